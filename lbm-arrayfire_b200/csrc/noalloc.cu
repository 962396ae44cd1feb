// noalloc.cu — FP64 conservation sums over a caller-owned population buffer without any device
// allocation (lbm_sums_fp64_noalloc).
//
// Some callers cannot let a library call cudaMalloc: applications whose device memory is owned by
// another allocator (a framework's caching allocator or a pool reserved up front to nearly all of
// HBM), where a cudaMalloc can fail or fragment the pool and a cudaFree synchronises the whole
// device, stalling the caller's other streams.  For them the reduction's scratch (one partial sum per
// block plus the folded result) lives in a fixed array of the library's device image instead of a
// per-context buffer.  The array exists on every device that loads the library and stays allocated
// until the process exits; it holds kMaxPartials + 1 entries of 40 bytes (640 KB).
#include "internal.h"
#include "kernels.cuh"

namespace lbm {
namespace {

constexpr int kThreads = 256;
constexpr long long kCellsPerBlock = 4096;  // 16 cells per thread
constexpr int kMaxPartials = 16384;         // -> LBM_NOALLOC_MAX_CELLS cells
static_assert(kCellsPerBlock * kMaxPartials == LBM_NOALLOC_MAX_CELLS, "scratch capacity and header limit differ");

// [0, kMaxPartials): one partial per block; [kMaxPartials]: the folded result of the call.
// Every entry a call reads was written earlier in the same call, so nothing has to be cleared.
static __device__ __align__(256) Sums g_noalloc_scratch[kMaxPartials + 1];

// Device address of the scratch array on the current device.  In host code the array's name is only a
// host-side stand-in, so the address is looked up with the device current, on every call: the lookup
// allocates nothing, and a cached address would go stale if the context were destroyed and recreated
// (cudaDeviceReset), when the library's module is loaded again and the array may move.
int scratch_address(Sums** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(noalloc scratch)");
    *out = static_cast<Sums*>(p);
    return LBM_OK;
}

template <class T>
struct Tag2 {
    using type = T;
};

template <class F>
void dispatch(int lattice, int storage, F&& f) {
    auto by_storage = [&](auto lt) {
        using L = typename decltype(lt)::type;
        switch (storage) {
            case LBM_F32: f(lt, Tag2<float>{}); break;
            case LBM_F16S: f(lt, Tag2<__half>{}); break;
            case LBM_BF16S: f(lt, Tag2<__nv_bfloat16>{}); break;
            default: f(lt, Tag2<double>{}); break;
        }
        (void)sizeof(L);
    };
    if (lattice == LBM_D2Q9)
        by_storage(Tag2<D2Q9>{});
    else
        by_storage(Tag2<D3Q27>{});
}

}  // namespace
}  // namespace lbm

using namespace lbm;

extern "C" int lbm_sums_fp64_noalloc(const void* populations, int lattice, int storage, int64_t nx, int64_t ny,
                                     int64_t nz, double storage_scale, void* stream, double out[4]) {
    if (!populations || !out) return set_error(LBM_ERR_INVALID, "NULL argument");
    if (lattice != LBM_D2Q9 && lattice != LBM_D3Q27) return set_error(LBM_ERR_INVALID, "unknown lattice");
    if (storage < LBM_F32 || storage > LBM_F64) return set_error(LBM_ERR_INVALID, "unknown storage");
    if (nx < 1 || ny < 1 || nz < 1 || (lattice == LBM_D2Q9 && nz != 1))
        return set_error(LBM_ERR_INVALID, "bad lattice extents");
    if (storage_scale < 0.0) return set_error(LBM_ERR_INVALID, "storage_scale must be >= 0");
    // bound the product by division first: each extent alone may pass while nx * ny * nz wraps
    const long long cap = LBM_NOALLOC_MAX_CELLS;
    if (nx > cap || ny > cap / nx || nz > cap / (nx * ny))
        return set_error(LBM_ERR_INVALID,
                         "lattice has more than LBM_NOALLOC_MAX_CELLS (67,108,864) cells: the fixed scratch "
                         "array of lbm_sums_fp64_noalloc is too small; use lbm_sums_fp64");
    const long long N = (long long)nx * ny * nz;
    Sums* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    const double scale = storage_scale > 0.0 ? storage_scale : default_scale(storage);
    const int blocks = (int)((N + kCellsPerBlock - 1) / kCellsPerBlock);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    dispatch(lattice, storage, [&](auto lt, auto st) {
        using L = typename decltype(lt)::type;
        using S = typename decltype(st)::type;
        k_sums_partial<L, S><<<blocks, kThreads, 0, s>>>(static_cast<const S*>(populations), N,
                                                         (float)(1.0 / scale), scratch);
    });
    k_sums_final<<<1, 32, 0, s>>>(scratch, blocks, scratch + kMaxPartials);
    LBM_CK(cudaGetLastError());
    Sums r;
    LBM_CK(cudaMemcpyAsync(&r, scratch + kMaxPartials, sizeof(Sums), cudaMemcpyDeviceToHost, s));
    LBM_CK(cudaStreamSynchronize(s));
    out[0] = r.m;
    out[1] = r.jx;
    out[2] = r.jy;
    out[3] = r.jz;
    if (r.bad) return set_error(LBM_ERR_DIVERGED, std::to_string(r.bad) + " non-finite populations");
    return LBM_OK;
}
