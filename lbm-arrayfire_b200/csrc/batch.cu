// batch.cu — an ensemble of independent BGK lattices (any mix of D2Q9 and D3Q27 extents and
// rates, one storage type) advanced together.  Each step is one kernel per lattice family over a
// tile table: a tile is one row segment (lattice, y, z, x0) of `tile_x` cells, so lattices of very
// different sizes share the SMs without per-lattice launches.  Chunks of steps are captured in a
// CUDA graph and replayed.  The tile width is picked by timing candidates on the real buffers.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"
#include "kernels.cuh"

namespace lbm {

// One ensemble member as the kernels see it (lives in device memory).
template <class R>
struct BatchLattice {
    void* f[2];
    const uint8_t* mask;
    int nx, ny, nz;
    long long N;
    R omega, one_m_omega;
    R scale, inv_scale;
    ClassTable<R> cls;
};

struct Tile {
    int lat, y, z, x0;
};

template <class L, class S>
__global__ void __launch_bounds__(256) k_batch_bgk(const BatchLattice<typename Codec<S>::Real>* __restrict__ lats,
                                                   const Tile* __restrict__ tiles, int parity) {
    using R = typename Codec<S>::Real;
    const Tile t = tiles[blockIdx.x];
    const BatchLattice<R>& p = lats[t.lat];
    const int x = t.x0 + threadIdx.x;
    if (x >= p.nx) return;
    bgk_cell<L, S, false>(p, static_cast<const S*>(p.f[parity]), static_cast<S*>(p.f[parity ^ 1]), x, t.y, t.z);
}

template <class T>
struct BTag {
    using type = T;
};
template <class F>
static void batch_dispatch(int storage, F&& f) {
    switch (storage) {
        case LBM_F32: f(BTag<float>{}); break;
        case LBM_F16S: f(BTag<__half>{}); break;
        case LBM_BF16S: f(BTag<__nv_bfloat16>{}); break;
        default: f(BTag<double>{}); break;
    }
}

}  // namespace lbm

using namespace lbm;

struct lbm_batch {
    std::vector<lbm_desc> descs;
    std::vector<lbm_ctx*> members;   // contexts owning each member's buffers (never stepped themselves)
    int storage = 0, device = 0;
    void* lats_d = nullptr;          // BatchLattice<R>[n]
    Tile* tiles_d[2] = {nullptr, nullptr};  // [0] D2Q9 tiles, [1] D3Q27 tiles
    long long n_tiles[2] = {0, 0};
    int tile_x = 0;
    int parity = 0;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int gsteps = 0;
    long long cells = 0;
    double bytes_per_step = 0;
};

namespace lbm {

static void batch_drop_graphs(lbm_batch* b) {
    for (auto& g : b->gexec)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    b->gsteps = 0;
}

static int batch_build_tiles(lbm_batch* b, int tile_x) {
    std::vector<Tile> t[2];
    for (int k = 0; k < (int)b->descs.size(); ++k) {
        const lbm_desc& d = b->descs[k];
        const int fam = d.lattice == LBM_D2Q9 ? 0 : 1;
        for (int z = 0; z < (int)d.nz; ++z)
            for (int y = 0; y < (int)d.ny; ++y)
                for (int x0 = 0; x0 < (int)d.nx; x0 += tile_x) t[fam].push_back(Tile{k, y, z, x0});
    }
    for (int fam = 0; fam < 2; ++fam) {
        if (b->tiles_d[fam]) cudaFree(b->tiles_d[fam]);
        b->tiles_d[fam] = nullptr;
        b->n_tiles[fam] = (long long)t[fam].size();
        if (t[fam].empty()) continue;
        if (t[fam].size() > 0x7fffffffULL) return set_error(LBM_ERR_INVALID, "tile table too large");
        if (cudaMalloc(&b->tiles_d[fam], sizeof(Tile) * t[fam].size()) != cudaSuccess) {
            cudaGetLastError();
            return set_error(LBM_ERR_NOMEM, "tile table allocation failed");
        }
        LBM_CK(cudaMemcpy(b->tiles_d[fam], t[fam].data(), sizeof(Tile) * t[fam].size(), cudaMemcpyHostToDevice));
    }
    b->tile_x = tile_x;
    return LBM_OK;
}

static void batch_launch(lbm_batch* b, int parity, cudaStream_t s) {
    batch_dispatch(b->storage, [&](auto tag) {
        using S = typename decltype(tag)::type;
        using R = typename Codec<S>::Real;
        const auto* lats = static_cast<const BatchLattice<R>*>(b->lats_d);
        if (b->n_tiles[0])
            k_batch_bgk<D2Q9, S><<<(unsigned)b->n_tiles[0], b->tile_x, 0, s>>>(lats, b->tiles_d[0], parity);
        if (b->n_tiles[1])
            k_batch_bgk<D3Q27, S><<<(unsigned)b->n_tiles[1], b->tile_x, 0, s>>>(lats, b->tiles_d[1], parity);
    });
}

static int batch_build_graphs(lbm_batch* b) {
    batch_drop_graphs(b);
    const double est_us = b->bytes_per_step / 5.0e6 + 4.0;
    int g = (int)std::ceil(400.0 / est_us);
    g = std::max(2, std::min(128, g + (g & 1)));
    for (int start = 0; start < 2; ++start) {
        cudaGraph_t graph;
        LBM_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        for (int s = 0; s < g; ++s) batch_launch(b, (start + s) & 1, b->stream);
        LBM_CK(cudaStreamEndCapture(b->stream, &graph));
        cudaError_t e = cudaGraphInstantiate(&b->gexec[start], graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate");
    }
    b->gsteps = g;
    return LBM_OK;
}

// Tile width: time one step for each candidate (reads the current buffers, writes the others).
static int batch_autotune(lbm_batch* b) {
    cudaEvent_t e0, e1;
    LBM_CK(cudaEventCreate(&e0));
    LBM_CK(cudaEventCreate(&e1));
    float best = 1e30f;
    int best_tx = 128;
    for (int tx : {64, 128, 256}) {
        int rc = batch_build_tiles(b, tx);
        if (rc) return rc;
        batch_launch(b, b->parity, b->stream);
        LBM_CK(cudaEventRecord(e0, b->stream));
        for (int r = 0; r < 2; ++r) batch_launch(b, b->parity, b->stream);
        LBM_CK(cudaEventRecord(e1, b->stream));
        LBM_CK(cudaEventSynchronize(e1));
        float ms = 0;
        LBM_CK(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
            best = ms;
            best_tx = tx;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    LBM_CK(cudaGetLastError());
    return batch_build_tiles(b, best_tx);
}

static void batch_free(lbm_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graphs(b);
    for (auto* m : b->members) lbm_destroy(m);
    cudaFree(b->lats_d);
    cudaFree(b->tiles_d[0]);
    cudaFree(b->tiles_d[1]);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

}  // namespace lbm

extern "C" {

int lbm_batch_create(const lbm_desc* descs, int n, lbm_batch** out) {
    if (!out || !descs || n < 1) return set_error(LBM_ERR_INVALID, "need n >= 1 descriptors and an out pointer");
    *out = nullptr;
    for (int k = 0; k < n; ++k) {
        int rc = validate_desc(&descs[k]);
        if (rc) return rc;
        if (descs[k].collision != LBM_BGK) return set_error(LBM_ERR_UNSUPPORTED, "batched ensembles are BGK only");
        if (descs[k].arithmetic != LBM_ARITH_DEVIATION)
            return set_error(LBM_ERR_UNSUPPORTED, "batched ensembles use deviation arithmetic");
        if (descs[k].storage != descs[0].storage) return set_error(LBM_ERR_INVALID, "one storage type per batch");
        if (descs[k].device != descs[0].device) return set_error(LBM_ERR_INVALID, "one device per batch");
    }
    lbm_batch* b = new lbm_batch();
    b->storage = descs[0].storage;
    b->device = descs[0].device;
    b->descs.assign(descs, descs + n);
    for (int k = 0; k < n; ++k) {
        lbm_ctx* m = nullptr;
        int rc = lbm_create(&descs[k], &m);
        if (rc) {
            batch_free(b);
            return rc;
        }
        b->members.push_back(m);
        b->descs[k].mask = nullptr;
        b->cells += (long long)descs[k].nx * descs[k].ny * descs[k].nz;
        b->bytes_per_step += 2.0 * (double)descs[k].nx * descs[k].ny * descs[k].nz * desc_q(&descs[k]) *
                             storage_bytes(b->storage);
    }
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) {
        batch_free(b);
        return set_error(LBM_ERR_CUDA, "stream creation failed");
    }
    int rc = LBM_OK;
    batch_dispatch(b->storage, [&](auto tag) {
        using S = typename decltype(tag)::type;
        using R = typename Codec<S>::Real;
        std::vector<BatchLattice<R>> h(n);
        for (int k = 0; k < n; ++k) {
            lbm_ctx* m = b->members[k];
            const lbm_desc& d = b->descs[k];
            BatchLattice<R>& L = h[k];
            std::memset(&L, 0, sizeof(L));
            (void)m;
            L.nx = (int)d.nx;
            L.ny = (int)d.ny;
            L.nz = (int)d.nz;
            L.N = (long long)d.nx * d.ny * d.nz;
            L.omega = R(d.omega);
            L.one_m_omega = R(1) - R(d.omega);
            const double sc = d.storage_scale > 0 ? d.storage_scale : default_scale(d.storage);
            L.scale = R(sc);
            L.inv_scale = R(1.0 / sc);
            for (int c = 0; c < kMaxClasses; ++c) {
                const bool used = c < d.n_classes;
                L.cls.flags[c] = used ? d.classes[c].flags : 0u;
                L.cls.rho[c] = R(used ? d.classes[c].rho : 1.0);
                L.cls.ux[c] = R(used ? d.classes[c].ux : 0.0);
                L.cls.uy[c] = R(used ? d.classes[c].uy : 0.0);
                L.cls.uz[c] = R(used ? d.classes[c].uz : 0.0);
            }
        }
        // population buffers and mask belong to the member contexts (both start on buffer 0)
        for (int k = 0; k < n && rc == LBM_OK; ++k)
            rc = ctx_buffers(b->members[k], &h[k].f[0], &h[k].f[1], &h[k].mask);
        if (rc == LBM_OK) {
            if (cudaMalloc(&b->lats_d, sizeof(BatchLattice<R>) * n) != cudaSuccess ||
                cudaMemcpy(b->lats_d, h.data(), sizeof(BatchLattice<R>) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
                cudaGetLastError();
                rc = set_error(LBM_ERR_NOMEM, "ensemble table allocation failed");
            }
        }
    });
    if (rc) {
        batch_free(b);
        return rc;
    }
    *out = b;
    return LBM_OK;
}

void lbm_batch_destroy(lbm_batch* b) { batch_free(b); }

int lbm_batch_size(const lbm_batch* b) { return b ? (int)b->descs.size() : 0; }
int64_t lbm_batch_cells(const lbm_batch* b) { return b ? b->cells : 0; }
void* lbm_batch_stream(lbm_batch* b) { return b ? (void*)b->stream : nullptr; }

int lbm_batch_tile_info(const lbm_batch* b, int* tile_x, int64_t* n_tiles) {
    if (!b) return set_error(LBM_ERR_INVALID, "batch is NULL");
    if (tile_x) *tile_x = b->tile_x;
    if (n_tiles) *n_tiles = b->n_tiles[0] + b->n_tiles[1];
    return LBM_OK;
}

int lbm_batch_step(lbm_batch* b, int64_t nsteps) {
    if (!b) return set_error(LBM_ERR_INVALID, "batch is NULL");
    if (nsteps < 0) return set_error(LBM_ERR_INVALID, "nsteps must be >= 0");
    if (nsteps == 0) return LBM_OK;
    LBM_CK(cudaSetDevice(b->device));
    if (!b->tile_x) {
        int rc = batch_autotune(b);
        if (rc) return rc;
    }
    long long n = nsteps;
    if (n >= 2) {
        if (!b->gsteps) {
            int rc = batch_build_graphs(b);
            if (rc) return rc;
        }
        while (n >= b->gsteps) {
            LBM_CK(cudaGraphLaunch(b->gexec[b->parity], b->stream));
            n -= b->gsteps;
        }
    }
    while (n > 0) {
        batch_launch(b, b->parity, b->stream);
        b->parity ^= 1;
        --n;
    }
    LBM_CK(cudaGetLastError());
    // members mirror the batch parity so their transfer/macro/sum calls see the current buffer
    for (auto* m : b->members) ctx_set_current(m, b->parity, true, nsteps);
    return LBM_OK;
}

int lbm_batch_sync(lbm_batch* b) {
    if (!b) return set_error(LBM_ERR_INVALID, "batch is NULL");
    LBM_CK(cudaSetDevice(b->device));
    LBM_CK(cudaStreamSynchronize(b->stream));
    return LBM_OK;
}

int lbm_batch_get_populations(lbm_batch* b, int k, void* dst, int dtype, int memory) {
    if (!b || k < 0 || k >= (int)b->members.size()) return set_error(LBM_ERR_INVALID, "bad batch member");
    int rc = lbm_batch_sync(b);
    return rc ? rc : lbm_get_populations(b->members[k], dst, dtype, memory);
}

int lbm_batch_set_populations(lbm_batch* b, int k, const void* src, int dtype, int memory) {
    if (!b || k < 0 || k >= (int)b->members.size()) return set_error(LBM_ERR_INVALID, "bad batch member");
    int rc = lbm_batch_sync(b);
    return rc ? rc : lbm_set_populations(b->members[k], src, dtype, memory);
}

int lbm_batch_get_macros(lbm_batch* b, int k, void* rho, void* u, int dtype, int memory) {
    if (!b || k < 0 || k >= (int)b->members.size()) return set_error(LBM_ERR_INVALID, "bad batch member");
    int rc = lbm_batch_sync(b);
    return rc ? rc : lbm_get_macros(b->members[k], rho, u, dtype, memory);
}

int lbm_batch_sums_fp64(lbm_batch* b, int k, double out[4]) {
    if (!b || k < 0 || k >= (int)b->members.size()) return set_error(LBM_ERR_INVALID, "bad batch member");
    int rc = lbm_batch_sync(b);
    return rc ? rc : lbm_sums_fp64(b->members[k], out);
}

}  // extern "C"
