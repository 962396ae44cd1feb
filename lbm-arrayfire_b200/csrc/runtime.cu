// runtime.cu — the single-lattice context behind the C ABI: device buffers (ping-pong
// populations, mask, Shan-Chen psi, reduction partials), kernel dispatch, CUDA-graph capture of
// step chunks, the block-width autotuner, population/field transfers and FP64 reductions.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <type_traits>
#include <vector>

#include "internal.h"
#include "cluster.cuh"
#include "kernels.cuh"
#include "rowpipe.cuh"

namespace lbm {

__global__ void k_sums_final(const Sums* __restrict__ partial, int n, Sums* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Sums s{0, 0, 0, 0, 0};
    for (int i = 0; i < n; ++i) {
        s.m += partial[i].m;
        s.jx += partial[i].jx;
        s.jy += partial[i].jy;
        s.jz += partial[i].jz;
        s.bad += partial[i].bad;
    }
    *out = s;
}

// One plane of populations (direction i) from plain values to the storage codec and back.
// The 16-bit codecs take the deviation in the caller's precision, so an FP64 source is rounded once.
template <class S, class In>
__global__ void k_encode_plane(const In* __restrict__ src, S* __restrict__ dst, long long n, double w, double scale) {
    using R = typename Codec<S>::Real;
    constexpr bool kShifted = Codec<S>::kBytes == 2;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        if constexpr (kShifted)
            Codec<S>::store_dev(dst + k, R(src[k] - In(w)), R(w), R(scale));
        else
            Codec<S>::store(dst + k, R(src[k]), R(w), R(scale));
    }
}
template <class S, class Out>
__global__ void k_decode_plane(const S* __restrict__ src, Out* __restrict__ dst, long long n, double w,
                               double inv_scale) {
    using R = typename Codec<S>::Real;
    constexpr bool kShifted = Codec<S>::kBytes == 2;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        if constexpr (kShifted)
            dst[k] = Out(w) + Out(Codec<S>::load_dev(src + k, R(w), R(inv_scale)));
        else
            dst[k] = Out(Codec<S>::load(src + k, R(w), R(inv_scale)));
    }
}

// F = feq(rho, u) for every cell; rho/u may be null (1 and 0).
template <class L, class S>
__global__ void k_init_eq(S* __restrict__ f, long long N, const double* __restrict__ rho,
                          const double* __restrict__ u, double scale) {
    using R = typename Codec<S>::Real;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x) {
        const R r = rho ? R(rho[c]) : R(1);
        const R ux = u ? R(u[c]) : R(0), uy = u ? R(u[N + c]) : R(0);
        const R uz = (u && L::DIM == 3) ? R(u[2 * N + c]) : R(0);
        R feq[L::Q];
        equilibrium<L, R>(r, ux, uy, uz, feq);
        static_for<L::Q>([&](auto I) {
            constexpr int i = I;
            Codec<S>::store(f + (long long)i * N + c, feq[i], R(L::w(i)), R(scale));
        });
    }
}

template <class T>
struct Tag {
    using type = T;
};

template <class F>
static void dispatch_storage(int storage, F&& f) {
    switch (storage) {
        case LBM_F32: f(Tag<float>{}); break;
        case LBM_F16S: f(Tag<__half>{}); break;
        case LBM_BF16S: f(Tag<__nv_bfloat16>{}); break;
        default: f(Tag<double>{}); break;
    }
}

template <class F>
static void dispatch_lattice(int lattice, F&& f) {
    if (lattice == LBM_D2Q9)
        f(Tag<D2Q9>{});
    else
        f(Tag<D3Q27>{});
}

static int grid_blocks(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    return (int)std::max(1LL, std::min(b, 148LL * 16));
}

}  // namespace lbm

using namespace lbm;

struct lbm_ctx {
    lbm_desc d{};
    int q = 0, dim = 0, sbytes = 0;
    long long N = 0;
    void* f[2] = {nullptr, nullptr};
    int cur = 0;
    uint8_t* mask = nullptr;
    void* psi = nullptr;
    void* staging = nullptr;
    size_t staging_bytes = 0;
    Sums* partial = nullptr;
    Sums* sums_out = nullptr;
    int reduce_blocks = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    bool timed = false;
    int block = 0;
    int kernel = LBM_KERNEL_AUTO;  // requested family
    int kernel_used = 0;           // family chosen (PLAIN or ROWS); 0 before the first step
    int rows_grid = 0;             // persistent grid of the row pipeline (a whole step)
    int rows_per_sm = 0, sms = 0;  // its CTAs per SM and the device's SMs
    int reserved_sms = 0;          // lbm_set_reserved_sms: SMs the persistent grids leave free
    int cl_ctas = 0, cl_rows = 0;  // cluster-resident kernel: CTAs of the cluster, rows per CTA
    int rows_rpg = 1;              // its rows per group (segmented rows: the segment width)
    long long scw_target = 0;      // Shan-Chen window kernel: resident CTAs of the device (0: not queried)
    int* err = nullptr;            // device error word of the row pipeline
    unsigned* tick = nullptr;      // the rounding's step counter pair (step_rounding)
    WaitLimits waits = kProductionWaits;  // the row pipeline's wait limits for the next launch
    bool stall_armed = false;      // lbm_test_stall_next_step: the next step launches with `stall`
    bool index64 = false;          // lbm_test_index64: 64-bit population indices in every kernel
    WaitLimits stall = kProductionWaits;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int gsteps = 0;
    bool has_prev = false;
    long long steps = 0;
    double scale = 1.0;
    bool mrt2 = false;             // two-rate Gram-Schmidt MRT (mrt2_collide) in use
    long long cell_offset = 0;     // lbm_set_cell_offset
    StepParams<float> pf{};
    StepParams<double> pd{};
};

namespace lbm {

template <class R>
static StepParams<R> make_params(const lbm_ctx* c) {
    StepParams<R> p{};
    const lbm_desc& d = c->d;
    p.mask = c->mask;
    p.nx = (int)d.nx;
    p.ny = (int)d.ny;
    p.nz = (int)d.nz;
    p.N = c->N;
    p.omega = R(d.omega);
    p.one_m_omega = R(1) - R(d.omega);
    p.scale = R(c->scale);
    p.inv_scale = R(1.0 / c->scale);
    p.G = R(d.sc_G);
    p.psi = static_cast<R*>(c->psi);
    p.tick = c->tick;
    p.sr = d.rounding == LBM_ROUND_STOCHASTIC ? 1 : 0;
    p.cell_base = (uint32_t)c->cell_offset;
    p.plo = 0;
    p.pcnt = (int)(d.lattice == LBM_D3Q27 ? d.nz : d.ny);
    p.pstride = 1;
    for (int k = 0; k < kMaxClasses; ++k) {
        const bool used = k < d.n_classes;
        p.cls.flags[k] = used ? d.classes[k].flags : 0u;
        p.cls.rho[k] = R(used ? d.classes[k].rho : 1.0);
        p.cls.ux[k] = R(used ? d.classes[k].ux : 0.0);
        p.cls.uy[k] = R(used ? d.classes[k].uy : 0.0);
        p.cls.uz[k] = R(used ? d.classes[k].uz : 0.0);
    }
    if (d.collision == LBM_MRT) {
        MrtCoef<double> k;
        mrt_coefficients(d.mrt_basis, d.mrt_s, k);
        // 16-bit storages carry (f - w) * scale through the (linear) transform; the equilibrium
        // moments are formed unscaled, so their coefficients take the scale (a power of two: exact).
        const double es = (d.storage == LBM_F16S || d.storage == LBM_BF16S) ? c->scale : 1.0;
        for (int t = 0; t < 27; ++t) {
            p.mrt.alpha[t] = R(k.alpha[t]);
            p.mrt.beta[t] = R(k.beta[t] * es);
        }
        for (int t = 0; t < 9; ++t) {
            p.mrt.A[t] = R(k.A[t]);
            p.mrt.B[t] = R(k.B[t] * es);
        }
        const int cslot[4] = {0, 1, 3, 9};
        for (int j = 0; j < 4; ++j) {
            const double dsc = mrt_slot_scale(d.mrt_basis, cslot[j]);
            p.mrt.cs[j] = R(d.mrt_s[mrt_slot_row(cslot[j])]);
            p.mrt.chi[j] = R(dsc);
            p.mrt.clo[j] = R(dsc - (double)R(dsc));
        }
        if (c->mrt2) {
            const double so = d.mrt_s[0], sv = d.mrt_s[4], dv = sv - so;
            p.mrt2.om1 = R(1.0 - so);
            p.mrt2.kxy = R(dv / 12.0);
            p.mrt2.k8 = R(dv / 36.0);
            p.mrt2.k9 = R(dv / 108.0);
            const double wc[4] = {D3Q27::w(0), D3Q27::w(1), D3Q27::w(7), D3Q27::w(19)};  // rest, face, edge, corner
            for (int k2 = 0; k2 < 4; ++k2) {
                p.mrt2.sw[k2] = R(so * wc[k2] * es);
                p.mrt2.sw45[k2] = R(4.5 * so * wc[k2] * es);
                p.mrt2.sw3[k2] = R(3.0 * so * wc[k2] * es);
            }
        }
    }
    return p;
}

// The two-rate collision (mrt2_collide) applies: Gram-Schmidt basis, 16-bit storage, and rates with one
// value on the shear rows 4-6, 8, 9 and one on every other row.
static bool mrt2_applies(const lbm_desc& d) {
    if (d.collision != LBM_MRT || d.mrt_basis != LBM_MRT_GRAM_SCHMIDT) return false;
    if (d.storage != LBM_F16S && d.storage != LBM_BF16S) return false;
    const double so = d.mrt_s[0], sv = d.mrt_s[4];
    for (int r = 0; r < 27; ++r) {
        const bool shear = r == 4 || r == 5 || r == 6 || r == 8 || r == 9;
        if (d.mrt_s[r] != (shear ? sv : so)) return false;
    }
    return true;
}

template <class R>
static StepParams<R>& params_of(lbm_ctx* c);
template <>
StepParams<float>& params_of<float>(lbm_ctx* c) {
    return c->pf;
}
template <>
StepParams<double>& params_of<double>(lbm_ctx* c) {
    return c->pd;
}

// ---- row pipeline (rowpipe.cuh) ------------------------------------------------------------
// D3Q27 BGK/MRT or D2Q9 BGK, deviation arithmetic, F32/F16S/BF16S, nx >= 32 and a multiple of 16:
// every bulk copy (population rows or segments, mask rows) must start on a 16-byte boundary and move a
// multiple of 16 bytes.  Rows wider than 1024 cells go by segments (k_step_rows_seg).
static bool rows_eligible(const lbm_ctx* c) {
    const lbm_desc& d = c->d;
    if (d.collision == LBM_SHANCHEN) return d.lattice == LBM_D2Q9;  // the one-pass window kernel: any shape
    const bool coll_ok = d.lattice == LBM_D3Q27 ? (d.collision == LBM_BGK || d.collision == LBM_MRT)
                                               : d.collision == LBM_BGK;
    // work items (row groups or row segments) are counted in 32 bits
    const bool items_ok = (long long)d.ny * d.nz * ((d.nx + 63) / 64) < (1LL << 31);
    return coll_ok && d.arithmetic == LBM_ARITH_DEVIATION && d.storage != LBM_F64 && d.nx >= 32 &&
           d.nx % 16 == 0 && items_ok;
}
static bool rows_segmented(const lbm_ctx* c) { return c->d.nx > 1024; }

// Segment width of the segmented row kernel (RowPipeShape::SEGW_RUN: 896 cells for D3Q27, 1008 for D2Q9).
#ifndef LBM_ROWPIPE_SEGW
#define LBM_ROWPIPE_SEGW 0  // > 0: a narrower segment width (a multiple of 16), for A/B builds
#endif
static int seg_width(int w) { return LBM_ROWPIPE_SEGW > 0 ? std::min(LBM_ROWPIPE_SEGW / 16 * 16, 1008) : w; }

// Persistent grid of the row pipeline for pcnt planes (pstride apart): one CTA per work item up to
// rows_per_sm x (SMs - reserved_sms), or, for a launch on a side stream (`side`), up to rows_per_sm x
// reserved_sms, the SMs left to it.  CTA b takes items b, b + grid, ...; where every plane (or
// row) ends in a short item, grid and the items per plane are kept coprime, so the short items do not
// all land on the same CTAs (148 = 4 x 37 CTAs and 4 segments per row would do that).
static int rows_grid_for(const lbm_ctx* c, int pcnt, int pstride, bool side = false) {
    const bool d3 = c->d.lattice == LBM_D3Q27;
    long long groups = 0, per_plane = 0;
    bool ragged = false;
    if (rows_segmented(c)) {
        per_plane = (c->d.nx + c->rows_rpg - 1) / c->rows_rpg;  // segments per row
        groups = per_plane * (d3 ? (long long)pcnt * c->d.ny : pcnt);
        ragged = true;
    } else if (d3) {
        per_plane = (c->d.ny + c->rows_rpg - 1) / c->rows_rpg;  // row groups per plane
        groups = per_plane * pcnt;
        ragged = c->d.ny % c->rows_rpg != 0;
    } else {
        // D2Q9: a plane is one row; a strided launch takes one row per group
        per_plane = groups = pstride > 1 ? pcnt : (pcnt + c->rows_rpg - 1) / c->rows_rpg;
        ragged = pstride == 1 && pcnt % c->rows_rpg != 0;
    }
    const int sms = side ? c->reserved_sms : c->sms - c->reserved_sms;
    const long long cap = (long long)c->rows_per_sm * std::max(1, sms);
    int grid = (int)std::max<long long>(1, std::min(groups, cap));
    if (ragged)
        while (grid > 1 && std::gcd((long long)grid, per_plane) != 1) --grid;
    return grid;
}

template <class L, class S, int PITCH, int COLL>
static void launch_rows_t(lbm_ctx* c, const StepParams<typename Codec<S>::Real>& p, cudaStream_t s, bool side) {
    const int grid = rows_grid_for(c, p.pcnt, p.pstride, side);
    if (rows_segmented(c)) {
        using Sh = SegShape<L, S, COLL>;
        k_step_rows_seg<L, S, COLL><<<grid, Sh::CONSUMERS + 32, Sh::smem_bytes(), s>>>(p, c->rows_rpg, c->err,
                                                                                       c->waits);
        return;
    }
    using Sh = RowShape<L, S, PITCH, COLL>;
    auto kern = k_step_rows<L, S, PITCH, COLL>;
    kern<<<grid, Sh::CONSUMERS + 32, Sh::smem_bytes(), s>>>(p, c->rows_rpg, c->err, c->waits);  // + producer warp
}

template <class L, class S, int PITCH, int COLL>
static int prepare_rows_t(lbm_ctx* c) {
    int per_sm = 0, sms = 0;
    LBM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->d.device));
    if (rows_segmented(c)) {
        using Sh = SegShape<L, S, COLL>;
        auto kern = k_step_rows_seg<L, S, COLL>;
        LBM_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::smem_bytes()));
        LBM_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Sh::CONSUMERS + 32, Sh::smem_bytes()));
        c->rows_rpg = seg_width(Sh::SEGW_RUN);
    } else {
        using Sh = RowShape<L, S, PITCH, COLL>;
        auto kern = k_step_rows<L, S, PITCH, COLL>;
        LBM_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::smem_bytes()));
        LBM_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Sh::CONSUMERS + 32, Sh::smem_bytes()));
        c->rows_rpg = Sh::rows_per_group((int)c->d.nx);
    }
    if (per_sm < 1) return set_error(LBM_ERR_UNSUPPORTED, "row pipeline does not fit on an SM");
    c->rows_per_sm = per_sm;
    c->sms = sms;
    c->rows_grid = rows_grid_for(c, (int)(c->d.lattice == LBM_D3Q27 ? c->d.nz : c->d.ny), 1);
    return LBM_OK;
}

// f(lattice tag, storage tag, collision constant, pitch constant)
template <class F>
static void dispatch_rows(const lbm_ctx* c, F&& f) {
    const int coll = c->d.collision == LBM_BGK ? 0 : c->mrt2 ? 3 : (c->d.mrt_basis == LBM_MRT_REF ? 1 : 2);
    auto by_pitch = [&](auto lt, auto st, auto co) {
        const long long nx = c->d.nx;
        if (nx <= 128)
            f(lt, st, co, std::integral_constant<int, 128>{});
        else if (nx <= 256)
            f(lt, st, co, std::integral_constant<int, 256>{});
        else if (nx <= 512)
            f(lt, st, co, std::integral_constant<int, 512>{});
        else
            f(lt, st, co, std::integral_constant<int, 1024>{});
    };
    auto by_coll = [&](auto lt, auto st) {
        if constexpr (std::is_same_v<typename decltype(lt)::type, D2Q9>) {
            by_pitch(lt, st, std::integral_constant<int, 0>{});
        } else {
            switch (coll) {
                case 0: by_pitch(lt, st, std::integral_constant<int, 0>{}); break;
                case 1: by_pitch(lt, st, std::integral_constant<int, 1>{}); break;
                case 2: by_pitch(lt, st, std::integral_constant<int, 2>{}); break;
                default:
                    // the two-rate collision exists for 16-bit storage only (mrt2_applies)
                    if constexpr (sizeof(typename decltype(st)::type) == 2)
                        by_pitch(lt, st, std::integral_constant<int, 3>{});
                    break;
            }
        }
    };
    auto by_storage = [&](auto lt) {
        switch (c->d.storage) {
            case LBM_F32: by_coll(lt, Tag<float>{}); break;
            case LBM_F16S: by_coll(lt, Tag<__half>{}); break;
            default: by_coll(lt, Tag<__nv_bfloat16>{}); break;
        }
    };
    if (c->d.lattice == LBM_D2Q9)
        by_storage(Tag<D2Q9>{});
    else
        by_storage(Tag<D3Q27>{});
}

#ifndef LBM_SCW_HMAX
#define LBM_SCW_HMAX 0  // > 0: at most this many rows per strip (several waves of CTAs on large lattices)
#endif
#ifndef LBM_IDX32
#define LBM_IDX32 1  // 0: the plain and window kernels always index populations in 64 bits (A/B)
#endif
// The plain step kernels (the two Shan-Chen passes included) and the Shan-Chen window kernel index
// populations in 32 bits when all Q N of them have 32-bit indices (largest index Q N - 1).
static bool idx32(const lbm_ctx* c) {
    const unsigned long long n = (unsigned long long)c->d.nx * (unsigned long long)c->d.ny * (unsigned long long)c->d.nz;
    const unsigned long long q = c->d.lattice == LBM_D3Q27 ? 27ULL : 9ULL;
    return LBM_IDX32 && !c->index64 && q * n <= (1ULL << 32);
}
static bool sc_window_i32(const lbm_ctx* c) { return idx32(c); }
// The window kernel instance of a context (storage S; absolute or deviation arithmetic; index width).
template <class S>
static auto sc_window_kernel(const lbm_ctx* c) {
    const bool abs_arith = c->d.arithmetic == LBM_ARITH_ABSOLUTE;
    if (sc_window_i32(c)) return abs_arith ? k_step_sc_window<S, true, true> : k_step_sc_window<S, false, true>;
    return abs_arith ? k_step_sc_window<S, true, false> : k_step_sc_window<S, false, false>;
}
// Rows per strip of the Shan-Chen window kernel over `rows` contiguous rows: one wave of CTAs.
static int sc_strip_rows(const lbm_ctx* c, long long rows) {
    const long long gx = (c->d.nx + kScwTX - 1) / kScwTX;
    const long long h = std::max<long long>(4, (rows * gx + c->scw_target - 1) / c->scw_target);
    return (int)(LBM_SCW_HMAX > 0 ? std::min<long long>(h, LBM_SCW_HMAX) : h);
}
static int prepare_rows(lbm_ctx* c) {
    if (c->d.collision == LBM_SHANCHEN) {
        // k_step_sc_window: strips of rows sized so that one wave of CTAs covers the lattice (A/B:
        // capping the strip height at 16/32/64 rows for several waves was slower or equal)
        int per_sm = 0, sms = 0, rc = LBM_OK;
        dispatch_storage(c->d.storage, [&](auto tag) {
            using S = typename decltype(tag)::type;
            auto kern = sc_window_kernel<S>(c);
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kScwTX, 0) != cudaSuccess)
                rc = set_error(LBM_ERR_CUDA, "occupancy query failed");
        });
        if (rc) return rc;
        LBM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->d.device));
        c->scw_target = std::max(1LL, (long long)std::max(per_sm, 1) * sms);
        c->rows_rpg = sc_strip_rows(c, c->d.ny);
        return LBM_OK;
    }
    int rc = LBM_OK;
    dispatch_rows(c, [&](auto lt, auto st, auto co, auto pi) {
        using L = typename decltype(lt)::type;
        using S = typename decltype(st)::type;
        rc = prepare_rows_t<L, S, decltype(pi)::value, decltype(co)::value>(c);
    });
    return rc;
}

// Launch one time step reading buffer `from` and writing the other one, over planes plo + k pstride,
// k < pcnt, of the slowest axis (pcnt < 0: all of them).  Plane sets of Shan-Chen take the one-pass
// window kernel whatever the family (bit-identical to the two passes): it writes psi of its own rows
// only, so launches of disjoint sets may run at the same time.
static void launch_step(lbm_ctx* c, int from, cudaStream_t s, int block, int plo = 0, int pcnt = -1,
                        int pstride = 1, bool side = false) {
    const int planes = (int)(c->d.lattice == LBM_D3Q27 ? c->d.nz : c->d.ny);
    if (pcnt < 0) {
        plo = 0;
        pcnt = planes;
        pstride = 1;
    }
    // the cluster-resident family runs whole multi-step launches (launch_cluster); anything else it is
    // asked for (plane sets, graph capture) takes the plain kernel, bit-identical to it
    if (c->kernel_used == LBM_KERNEL_CLUSTER && block <= 0) block = 128;
    const bool whole = plo == 0 && pcnt == planes && pstride == 1;
    if (c->d.collision == LBM_SHANCHEN && (c->kernel_used == LBM_KERNEL_ROWS || !whole)) {
        dispatch_storage(c->d.storage, [&](auto tag) {
            using S = typename decltype(tag)::type;
            using R = typename Codec<S>::Real;
            StepParams<R> p = params_of<R>(c);
            p.fin = c->f[from];
            p.fout = c->f[from ^ 1];
            p.parity = from;
            p.plo = plo;
            p.pcnt = pcnt;
            p.pstride = pstride;
            // contiguous rows: strips of h rows; a strided set: one row per strip
            const int h = whole ? c->rows_rpg : pstride > 1 ? 1 : sc_strip_rows(c, pcnt);
            const unsigned gy = (unsigned)(pstride > 1 ? pcnt : (pcnt + h - 1) / h);
            const dim3 wg((unsigned)((c->d.nx + kScwTX - 1) / kScwTX), gy, 1);
            sc_window_kernel<S>(c)<<<wg, kScwTX, 0, s>>>(p, h);
        });
        return;
    }
    if (c->kernel_used == LBM_KERNEL_ROWS) {
        dispatch_rows(c, [&](auto lt, auto st, auto co, auto pi) {
            using L = typename decltype(lt)::type;
            using S = typename decltype(st)::type;
            using R = typename Codec<S>::Real;
            StepParams<R> p = params_of<R>(c);
            p.fin = c->f[from];
            p.fout = c->f[from ^ 1];
            p.parity = from;
            p.plo = plo;
            p.pcnt = pcnt;
            p.pstride = pstride;
            launch_rows_t<L, S, decltype(pi)::value, decltype(co)::value>(c, p, s, side);
        });
        return;
    }
    const bool d3 = c->d.lattice == LBM_D3Q27;
    const dim3 blk(block), grid((unsigned)((c->d.nx + block - 1) / block), (unsigned)(d3 ? c->d.ny : pcnt),
                                (unsigned)(d3 ? pcnt : c->d.nz));
    dispatch_storage(c->d.storage, [&](auto tag) {
        using S = typename decltype(tag)::type;
        using R = typename Codec<S>::Real;
        StepParams<R> p = params_of<R>(c);
        p.fin = c->f[from];
        p.fout = c->f[from ^ 1];
        p.parity = from;
        p.plo = plo;
        p.pcnt = pcnt;
        p.pstride = pstride;
        const bool abs_arith = c->d.arithmetic == LBM_ARITH_ABSOLUTE;
        const bool i32 = idx32(c);
        switch (c->d.collision) {
            case LBM_BGK: {
                auto kern = [&](auto lt) {
                    using L = typename decltype(lt)::type;
                    if (abs_arith) return i32 ? k_step_bgk<L, S, true, true> : k_step_bgk<L, S, true, false>;
                    return i32 ? k_step_bgk<L, S, false, true> : k_step_bgk<L, S, false, false>;
                };
                if (c->d.lattice == LBM_D2Q9)
                    kern(Tag<D2Q9>{})<<<grid, blk, 0, s>>>(p);
                else
                    kern(Tag<D3Q27>{})<<<grid, blk, 0, s>>>(p);
                break;
            }
            case LBM_MRT:  // deviation arithmetic only (validate_desc)
                if (c->mrt2) {
                    if constexpr (sizeof(S) == 2) (i32 ? k_step_mrt2<S, true> : k_step_mrt2<S, false>)<<<grid, blk, 0, s>>>(p);
                } else if (c->d.mrt_basis == LBM_MRT_REF)
                    (i32 ? k_step_mrt<kMrtRef, S, true> : k_step_mrt<kMrtRef, S, false>)<<<grid, blk, 0, s>>>(p);
                else
                    (i32 ? k_step_mrt<kMrtGramSchmidt, S, true> : k_step_mrt<kMrtGramSchmidt, S, false>)<<<grid, blk, 0, s>>>(p);
                break;
            default:
                if (abs_arith) {
                    (i32 ? k_sc_psi<S, true, true> : k_sc_psi<S, true, false>)<<<grid, blk, 0, s>>>(p);
                    (i32 ? k_step_sc<S, true, true> : k_step_sc<S, true, false>)<<<grid, blk, 0, s>>>(p);
                } else {
                    (i32 ? k_sc_psi<S, false, true> : k_sc_psi<S, false, false>)<<<grid, blk, 0, s>>>(p);
                    (i32 ? k_step_sc<S, false, true> : k_step_sc<S, false, false>)<<<grid, blk, 0, s>>>(p);
                }
                break;
        }
    });
}

static int max_block(const lbm_ctx* c) { return c->d.collision == LBM_MRT ? 256 : 512; }

// ---- cluster-resident kernel (cluster.cuh) --------------------------------------------------
// D2Q9 BGK in deviation arithmetic whose two population buffers fit into the shared memory of one
// cluster (16 CTAs where the device launches that size, else 8; at most 200 KB per CTA).
static size_t cluster_smem(const lbm_ctx* c, int rows) {
    return (size_t)2 * c->q * rows * c->d.nx * c->sbytes + (size_t)rows * c->d.nx;
}

// The cluster kernel's dynamic shared-memory bound: the device's opt-in maximum per block.
static int cluster_smem_bound(const lbm_ctx* c) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->d.device) != cudaSuccess) {
        cudaGetLastError();
        v = 200 * 1024;
    }
    return v;
}

template <class F>
static void dispatch_cluster(const lbm_ctx* c, F&& f) {
    switch (c->d.storage) {
        case LBM_F32: f(k_step_cluster<float>); break;
        case LBM_F16S: f(k_step_cluster<__half>); break;
        case LBM_BF16S: f(k_step_cluster<__nv_bfloat16>); break;
        default: f(k_step_cluster<double>); break;
    }
}

// Sets cl_ctas / cl_rows and returns true when the lattice can run resident in one cluster.
static bool cluster_eligible(lbm_ctx* c) {
    const lbm_desc& d = c->d;
    if (d.lattice != LBM_D2Q9 || d.collision != LBM_BGK || d.arithmetic != LBM_ARITH_DEVIATION) return false;
    if ((long long)d.nx * d.ny > 16LL * kClusterThreads * 64) return false;
    bool ok = false;
    dispatch_cluster(c, [&](auto kern) {
        for (int ctas : {16, 8}) {
            const int rows = (int)((d.ny + ctas - 1) / ctas);
            const size_t smem = cluster_smem(c, rows);
            if (smem > 200 * 1024) continue;
            if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, cluster_smem_bound(c)) !=
                    cudaSuccess ||
                (ctas > 8 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
                cudaGetLastError();
                continue;
            }
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = (unsigned)ctas;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3((unsigned)ctas);
            cfg.blockDim = dim3(kClusterThreads);
            cfg.dynamicSmemBytes = smem;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            if (clusters >= 1) {
                c->cl_ctas = ctas;
                c->cl_rows = rows;
                ok = true;
                return;
            }
        }
    });
    return ok;
}

// One launch of k (<= kClusterMaxSteps) steps from buffer `from` into the other one; write_prev: also
// the state after k - 1 steps into buffer `from` (off for trial launches).
static void launch_cluster(lbm_ctx* c, int from, cudaStream_t s, int k, bool write_prev = true) {
    dispatch_storage(c->d.storage, [&](auto tag) {
        using S = typename decltype(tag)::type;
        using R = typename Codec<S>::Real;
        StepParams<R> p = params_of<R>(c);
        p.fin = c->f[from];
        p.fout = c->f[from ^ 1];
        p.parity = from;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)c->cl_ctas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        // the attribute is per kernel, not per context: every context sets the same bound (the
        // device's opt-in maximum), so contexts of different sizes, on any host thread, never lower it
        // below another's launch
        cudaFuncSetAttribute(k_step_cluster<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, cluster_smem_bound(c));
        cfg.gridDim = dim3((unsigned)c->cl_ctas);
        cfg.blockDim = dim3(kClusterThreads);
        cfg.dynamicSmemBytes = cluster_smem(c, c->cl_rows);
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k_step_cluster<S>, p, c->cl_rows, k, write_prev ? 1 : 0);
    });
}

static std::mutex g_tune_mu;
static std::map<std::string, int> g_tune_cache;

static std::string tune_key(const lbm_ctx* c) {
    const lbm_desc& d = c->d;
    char buf[160];
    snprintf(buf, sizeof(buf), "%d/%d/%d/%d/%lld/%lld/%lld", d.lattice, d.collision, d.storage, d.mrt_basis,
             (long long)d.nx, (long long)d.ny, (long long)d.nz);
    return buf;
}

// Pick the block width by timing candidates on the real buffers: each trial reads the current
// buffer and writes the other one, which the next step overwrites anyway.
// Choose the kernel family and, for the plain kernel, the block width.  An explicit block width or
// LBM_KERNEL_PLAIN selects the plain kernel, LBM_KERNEL_ROWS the row pipeline; otherwise every
// eligible candidate is timed (cached per problem shape).
static int autotune(lbm_ctx* c) {
    if (c->kernel == LBM_KERNEL_ROWS) {
        c->kernel_used = LBM_KERNEL_ROWS;
        return prepare_rows(c);
    }
    if (c->kernel == LBM_KERNEL_CLUSTER) {
        if (!cluster_eligible(c)) return set_error(LBM_ERR_UNSUPPORTED, "the lattice does not fit one cluster");
        c->kernel_used = LBM_KERNEL_CLUSTER;
        return LBM_OK;
    }
    if (c->kernel == LBM_KERNEL_PLAIN && c->block) {
        c->kernel_used = LBM_KERNEL_PLAIN;
        return LBM_OK;
    }
    if (c->block) {
        c->kernel_used = LBM_KERNEL_PLAIN;
        return LBM_OK;
    }
    const bool try_rows = c->kernel == LBM_KERNEL_AUTO && rows_eligible(c);
    const bool try_cluster = c->kernel == LBM_KERNEL_AUTO && cluster_eligible(c);
    const std::string key = tune_key(c) + (try_rows ? "/rows" : "/plain") + (try_cluster ? "/cluster" : "");
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            if (it->second == -2) {
                c->kernel_used = LBM_KERNEL_CLUSTER;
                return LBM_OK;
            }
            if (it->second < 0) {
                c->kernel_used = LBM_KERNEL_ROWS;
                return prepare_rows(c);
            }
            c->kernel_used = LBM_KERNEL_PLAIN;
            c->block = it->second;
            return LBM_OK;
        }
    }
    const int maxb = max_block(c);
    const long long nxr = ((c->d.nx + 31) / 32) * 32;
    std::vector<int> cands;  // block widths of the plain kernel; -1 = row pipeline, -2 = cluster-resident
    for (int b : {32, 64, 128, 256, 512})
        if (b <= maxb && (b <= nxr || b == 32)) cands.push_back(b);
    if (try_rows) {
        int rc = prepare_rows(c);
        if (rc) return rc;
        cands.push_back(-1);
    }
    if (try_cluster) cands.push_back(-2);
    int best_b = cands[0];
    if (cands.size() > 1) {
        cudaEvent_t a, b;
        LBM_CK(cudaEventCreate(&a));
        LBM_CK(cudaEventCreate(&b));
        float best = 1e30f;
        const long long bytes = c->N * c->q * (long long)c->sbytes * 2;
        // about 2 ms of timed launches per candidate at ~5 TB/s (small, L2-resident lattices take many
        // short launches to rank candidates a few percent apart), at least 2 and at most 50
        const int reps = (int)std::max(2LL, std::min(50LL, 10000000000LL / std::max(1LL, bytes)));
        for (int blk : cands) {
            if (blk == -2) {
                // one launch of `reps` steps, per step as the others' single launches (its output goes
                // to the other buffer, as every trial's does)
                c->kernel_used = LBM_KERNEL_CLUSTER;
                launch_cluster(c, c->cur, c->stream, 1, false);
                LBM_CK(cudaEventRecord(a, c->stream));
                launch_cluster(c, c->cur, c->stream, reps, false);
            } else {
                c->kernel_used = blk < 0 ? LBM_KERNEL_ROWS : LBM_KERNEL_PLAIN;
                launch_step(c, c->cur, c->stream, blk);
                LBM_CK(cudaEventRecord(a, c->stream));
                for (int r = 0; r < reps; ++r) launch_step(c, c->cur, c->stream, blk);
            }
            LBM_CK(cudaEventRecord(b, c->stream));
            LBM_CK(cudaEventSynchronize(b));
            float ms = 0;
            LBM_CK(cudaEventElapsedTime(&ms, a, b));
            if (ms < best) {
                best = ms;
                best_b = blk;
            }
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        LBM_CK(cudaGetLastError());
    }
    c->kernel_used = best_b == -2 ? LBM_KERNEL_CLUSTER : best_b < 0 ? LBM_KERNEL_ROWS : LBM_KERNEL_PLAIN;
    c->block = best_b < 0 ? 0 : best_b;
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune_cache[key] = best_b;
    return LBM_OK;
}

static void drop_graphs(lbm_ctx* c) {
    for (auto& g : c->gexec)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    c->gsteps = 0;
}

// Capture `gsteps` (even) consecutive steps starting from each buffer parity.
static int build_graphs(lbm_ctx* c) {
    drop_graphs(c);
    const double bytes = (double)c->N * c->q * c->sbytes * 2.0;
    const double est_us = bytes / 5.0e6 + 2.0;  // ~5 TB/s plus launch latency
    int g = (int)std::ceil(400.0 / est_us);
    g = std::max(2, std::min(256, g + (g & 1)));
    for (int start = 0; start < 2; ++start) {
        cudaGraph_t graph;
        LBM_CK(cudaStreamBeginCapture(c->own, cudaStreamCaptureModeThreadLocal));
        for (int s = 0; s < g; ++s) launch_step(c, (start + s) & 1, c->own, c->block);
        LBM_CK(cudaStreamEndCapture(c->own, &graph));
        cudaError_t e = cudaGraphInstantiate(&c->gexec[start], graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate");
    }
    c->gsteps = g;
    return LBM_OK;
}

static int ensure_staging(lbm_ctx* c, size_t bytes) {
    if (c->staging_bytes >= bytes) return LBM_OK;
    if (c->staging) cudaFree(c->staging);
    c->staging = nullptr;
    c->staging_bytes = 0;
    if (cudaMalloc(&c->staging, bytes) != cudaSuccess) {
        cudaGetLastError();
        return set_error(LBM_ERR_NOMEM, "staging allocation failed");
    }
    c->staging_bytes = bytes;
    return LBM_OK;
}

static void destroy_ctx(lbm_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->d.device);
    if (c->own) cudaStreamSynchronize(c->own);
    if (c->stream && c->stream != c->own) cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    cudaFree(c->f[0]);
    cudaFree(c->f[1]);
    cudaFree(c->mask);
    cudaFree(c->psi);
    cudaFree(c->staging);
    cudaFree(c->partial);
    cudaFree(c->sums_out);
    cudaFree(c->err);
    cudaFree(c->tick);
    if (c->e0) cudaEventDestroy(c->e0);
    if (c->e1) cudaEventDestroy(c->e1);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
}

int ctx_buffers(lbm_ctx* c, void** f0, void** f1, const uint8_t** mask) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    *f0 = c->f[0];
    *f1 = c->f[1];
    *mask = c->mask;
    return LBM_OK;
}

void ctx_set_current(lbm_ctx* c, int cur, bool has_prev, long long steps_added) {
    c->cur = cur;
    c->has_prev = has_prev;
    c->steps += steps_added;
}

static int check_device(int dev) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(LBM_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (dev < 0 || dev >= n) return set_error(LBM_ERR_INVALID, "device ordinal out of range");
    cudaDeviceProp prop;
    LBM_CK(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10 || prop.minor != 0)
        return set_error(LBM_ERR_NO_DEVICE, std::string("liblbm_b200 is built for sm_100a (B200); device is ") +
                                                prop.name);
    return LBM_OK;
}

}  // namespace lbm

extern "C" {

int lbm_create(const lbm_desc* d, lbm_ctx** out) {
    if (!out) return set_error(LBM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int rc = validate_desc(d);
    if (rc) return rc;
    if ((rc = check_device(d->device))) return rc;
    LBM_CK(cudaSetDevice(d->device));
    lbm_ctx* c = new lbm_ctx();
    c->d = *d;
    c->d.mask = nullptr;
    c->q = desc_q(d);
    c->dim = d->lattice == LBM_D2Q9 ? 2 : 3;
    c->N = desc_cells(d);
    c->sbytes = storage_bytes(d->storage);
    c->scale = d->storage_scale > 0 ? d->storage_scale : default_scale(d->storage);
    const size_t fbytes = (size_t)c->N * c->q * c->sbytes;
    c->reduce_blocks = grid_blocks(c->N, 256);
    bool ok = cudaMalloc(&c->f[0], fbytes) == cudaSuccess && cudaMalloc(&c->f[1], fbytes) == cudaSuccess &&
              cudaMalloc(&c->partial, sizeof(Sums) * c->reduce_blocks) == cudaSuccess &&
              cudaMalloc(&c->sums_out, sizeof(Sums)) == cudaSuccess &&
              cudaMalloc(&c->err, sizeof(int)) == cudaSuccess && cudaMemset(c->err, 0, sizeof(int)) == cudaSuccess &&
              cudaMalloc(&c->tick, 2 * sizeof(unsigned)) == cudaSuccess &&
              cudaMemset(c->tick, 0, 2 * sizeof(unsigned)) == cudaSuccess;
    if (ok && d->mask) ok = cudaMalloc(&c->mask, (size_t)c->N) == cudaSuccess;
    if (ok && d->collision == LBM_SHANCHEN)
        ok = cudaMalloc(&c->psi, (size_t)c->N * (d->storage == LBM_F64 ? 8 : 4)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        destroy_ctx(c);
        return set_error(LBM_ERR_NOMEM, "device allocation failed");
    }
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->e0) != cudaSuccess || cudaEventCreate(&c->e1) != cudaSuccess) {
        destroy_ctx(c);
        return set_error(LBM_ERR_CUDA, "stream/event creation failed");
    }
    c->stream = c->own;
    if (d->mask) {
        for (long long k = 0; k < c->N; ++k)
            if (d->mask[k] >= d->n_classes) {
                destroy_ctx(c);
                return set_error(LBM_ERR_INVALID, "mask holds a class id >= n_classes");
            }
        if (cudaMemcpy(c->mask, d->mask, (size_t)c->N, cudaMemcpyHostToDevice) != cudaSuccess) {
            destroy_ctx(c);
            return set_error(LBM_ERR_CUDA, "mask upload failed");
        }
    }
    c->mrt2 = mrt2_applies(c->d);
    c->pf = make_params<float>(c);
    c->pd = make_params<double>(c);
    rc = lbm_init_equilibrium(c, nullptr, nullptr);
    if (rc) {
        destroy_ctx(c);
        return rc;
    }
    *out = c;
    return LBM_OK;
}

void lbm_destroy(lbm_ctx* c) { destroy_ctx(c); }

int lbm_init_equilibrium(lbm_ctx* c, const double* rho, const double* u) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    LBM_CK(cudaSetDevice(c->d.device));
    double* drho = nullptr;
    double* du = nullptr;
    if (rho || u) {
        int rc = ensure_staging(c, sizeof(double) * (size_t)c->N * (1 + c->dim));
        if (rc) return rc;
        drho = static_cast<double*>(c->staging);
        du = drho + c->N;
        if (rho) LBM_CK(cudaMemcpyAsync(drho, rho, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
        if (u) LBM_CK(cudaMemcpyAsync(du, u, sizeof(double) * c->N * c->dim, cudaMemcpyHostToDevice, c->stream));
    }
    const int blocks = grid_blocks(c->N, 256);
    dispatch_storage(c->d.storage, [&](auto tag) {
        using S = typename decltype(tag)::type;
        dispatch_lattice(c->d.lattice, [&](auto lt) {
            using L = typename decltype(lt)::type;
            k_init_eq<L, S><<<blocks, 256, 0, c->stream>>>(static_cast<S*>(c->f[c->cur]), c->N,
                                                            rho ? drho : nullptr, u ? du : nullptr, c->scale);
        });
    });
    LBM_CK(cudaGetLastError());
    LBM_CK(cudaStreamSynchronize(c->stream));
    c->has_prev = false;
    return LBM_OK;
}

int lbm_set_populations(lbm_ctx* c, const void* src, int dtype, int memory) {
    if (!c || !src) return set_error(LBM_ERR_INVALID, "NULL argument");
    if (dtype != LBM_DTYPE_F32 && dtype != LBM_DTYPE_F64) return set_error(LBM_ERR_INVALID, "dtype must be F32 or F64");
    if (memory != LBM_HOST && memory != LBM_DEVICE) return set_error(LBM_ERR_INVALID, "memory must be HOST or DEVICE");
    LBM_CK(cudaSetDevice(c->d.device));
    const size_t elt = dtype == LBM_DTYPE_F32 ? 4 : 8;
    const cudaMemcpyKind kind = memory == LBM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const bool same = (dtype == LBM_DTYPE_F32 && c->d.storage == LBM_F32) ||
                      (dtype == LBM_DTYPE_F64 && c->d.storage == LBM_F64);
    if (same) {
        LBM_CK(cudaMemcpyAsync(c->f[c->cur], src, elt * c->N * c->q, kind, c->stream));
    } else {
        if (memory == LBM_HOST) {
            int rc = ensure_staging(c, elt * c->N);
            if (rc) return rc;
        }
        const int blocks = grid_blocks(c->N, 256);
        for (int i = 0; i < c->q; ++i) {
            const char* plane = static_cast<const char*>(src) + elt * c->N * i;
            const void* in = plane;
            if (memory == LBM_HOST) {
                LBM_CK(cudaMemcpyAsync(c->staging, plane, elt * c->N, kind, c->stream));
                in = c->staging;
            }
            const double w = c->d.lattice == LBM_D2Q9 ? D2Q9::w(i) : D3Q27::w(i);
            dispatch_storage(c->d.storage, [&](auto tag) {
                using S = typename decltype(tag)::type;
                S* dst = static_cast<S*>(c->f[c->cur]) + (long long)i * c->N;
                if (dtype == LBM_DTYPE_F32)
                    k_encode_plane<S, float><<<blocks, 256, 0, c->stream>>>(static_cast<const float*>(in), dst, c->N, w,
                                                                           c->scale);
                else
                    k_encode_plane<S, double><<<blocks, 256, 0, c->stream>>>(static_cast<const double*>(in), dst, c->N,
                                                                            w, c->scale);
            });
            LBM_CK(cudaGetLastError());
        }
    }
    LBM_CK(cudaStreamSynchronize(c->stream));
    c->has_prev = false;
    return LBM_OK;
}

int lbm_get_populations(lbm_ctx* c, void* dst, int dtype, int memory) {
    if (!c || !dst) return set_error(LBM_ERR_INVALID, "NULL argument");
    if (dtype != LBM_DTYPE_F32 && dtype != LBM_DTYPE_F64) return set_error(LBM_ERR_INVALID, "dtype must be F32 or F64");
    if (memory != LBM_HOST && memory != LBM_DEVICE) return set_error(LBM_ERR_INVALID, "memory must be HOST or DEVICE");
    LBM_CK(cudaSetDevice(c->d.device));
    const size_t elt = dtype == LBM_DTYPE_F32 ? 4 : 8;
    const cudaMemcpyKind kind = memory == LBM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    const bool same = (dtype == LBM_DTYPE_F32 && c->d.storage == LBM_F32) ||
                      (dtype == LBM_DTYPE_F64 && c->d.storage == LBM_F64);
    if (same) {
        LBM_CK(cudaMemcpyAsync(dst, c->f[c->cur], elt * c->N * c->q, kind, c->stream));
    } else {
        if (memory == LBM_HOST) {
            int rc = ensure_staging(c, elt * c->N);
            if (rc) return rc;
        }
        const int blocks = grid_blocks(c->N, 256);
        for (int i = 0; i < c->q; ++i) {
            char* plane = static_cast<char*>(dst) + elt * c->N * i;
            void* out = memory == LBM_HOST ? c->staging : plane;
            const double w = c->d.lattice == LBM_D2Q9 ? D2Q9::w(i) : D3Q27::w(i);
            dispatch_storage(c->d.storage, [&](auto tag) {
                using S = typename decltype(tag)::type;
                const S* srcp = static_cast<const S*>(c->f[c->cur]) + (long long)i * c->N;
                if (dtype == LBM_DTYPE_F32)
                    k_decode_plane<S, float><<<blocks, 256, 0, c->stream>>>(srcp, static_cast<float*>(out), c->N, w,
                                                                           1.0 / c->scale);
                else
                    k_decode_plane<S, double><<<blocks, 256, 0, c->stream>>>(srcp, static_cast<double*>(out), c->N, w,
                                                                            1.0 / c->scale);
            });
            LBM_CK(cudaGetLastError());
            if (memory == LBM_HOST) LBM_CK(cudaMemcpyAsync(plane, c->staging, elt * c->N, kind, c->stream));
        }
    }
    LBM_CK(cudaStreamSynchronize(c->stream));
    return LBM_OK;
}

int lbm_step(lbm_ctx* c, int64_t nsteps) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    if (nsteps < 0) return set_error(LBM_ERR_INVALID, "nsteps must be >= 0");
    if (nsteps == 0) return LBM_OK;
    LBM_CK(cudaSetDevice(c->d.device));
    if (!c->kernel_used) {
        int rc = autotune(c);
        if (rc) return rc;
    }
    LBM_CK(cudaEventRecord(c->e0, c->stream));
    long long n = nsteps;
    if (c->kernel_used == LBM_KERNEL_CLUSTER) {
        while (n > 0) {
            const int k = (int)std::min<long long>(n, kClusterMaxSteps);
            launch_cluster(c, c->cur, c->stream, k);
            c->cur ^= 1;
            n -= k;
        }
    }
    if (c->stall_armed) {
        // the armed test stall: one direct launch with its wait limits, before any graph (which
        // captures the production limits)
        c->stall_armed = false;
        c->waits = c->stall;
        launch_step(c, c->cur, c->stream, c->block);
        c->waits = kProductionWaits;
        c->cur ^= 1;
        --n;
    }
    if (n >= 2) {
        if (!c->gsteps) {
            int rc = build_graphs(c);
            if (rc) return rc;
        }
        while (n >= c->gsteps) {
            LBM_CK(cudaGraphLaunch(c->gexec[c->cur], c->stream));
            n -= c->gsteps;
        }
    }
    while (n > 0) {
        launch_step(c, c->cur, c->stream, c->block);
        c->cur ^= 1;
        --n;
    }
    LBM_CK(cudaGetLastError());
    LBM_CK(cudaEventRecord(c->e1, c->stream));
    c->timed = true;
    c->has_prev = true;
    c->steps += nsteps;
    return LBM_OK;
}

int lbm_sync(lbm_ctx* c) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    LBM_CK(cudaSetDevice(c->d.device));
    LBM_CK(cudaStreamSynchronize(c->stream));
    int err = 0;
    LBM_CK(cudaMemcpy(&err, c->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        LBM_CK(cudaMemset(c->err, 0, sizeof(int)));
        return set_error(LBM_ERR_TIMEOUT, "a row-pipeline wait on a shared-memory stage gave up; results are invalid");
    }
    return LBM_OK;
}

int lbm_last_step_ms(lbm_ctx* c, float* ms) {
    if (!c || !ms) return set_error(LBM_ERR_INVALID, "NULL argument");
    if (!c->timed) return set_error(LBM_ERR_STATE, "no step has been issued");
    LBM_CK(cudaSetDevice(c->d.device));
    LBM_CK(cudaEventSynchronize(c->e1));
    LBM_CK(cudaEventElapsedTime(ms, c->e0, c->e1));
    return LBM_OK;
}

int64_t lbm_steps_done(const lbm_ctx* c) { return c ? c->steps : -1; }

int lbm_get_macros(lbm_ctx* c, void* rho, void* u, int dtype, int memory) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    if (dtype != LBM_DTYPE_F32 && dtype != LBM_DTYPE_F64) return set_error(LBM_ERR_INVALID, "dtype must be F32 or F64");
    if (memory != LBM_HOST && memory != LBM_DEVICE) return set_error(LBM_ERR_INVALID, "memory must be HOST or DEVICE");
    if (!rho && !u) return LBM_OK;
    LBM_CK(cudaSetDevice(c->d.device));
    const size_t elt = dtype == LBM_DTYPE_F32 ? 4 : 8;
    void* drho = rho;
    void* du = u;
    if (memory == LBM_HOST) {
        int rc = ensure_staging(c, elt * c->N * (1 + c->dim));
        if (rc) return rc;
        drho = rho ? c->staging : nullptr;
        du = u ? static_cast<char*>(c->staging) + elt * c->N : nullptr;
    }
    const int pulled = c->has_prev ? 1 : 0;
    const int src = c->has_prev ? (c->cur ^ 1) : c->cur;
    const int block = 128;
    const dim3 grid((unsigned)((c->d.nx + block - 1) / block), (unsigned)c->d.ny, (unsigned)c->d.nz);
    dispatch_storage(c->d.storage, [&](auto tag) {
        using S = typename decltype(tag)::type;
        using R = typename Codec<S>::Real;
        StepParams<R> p = params_of<R>(c);
        p.fin = c->f[src];
        dispatch_lattice(c->d.lattice, [&](auto lt) {
            using L = typename decltype(lt)::type;
            if (dtype == LBM_DTYPE_F32)
                k_macros<L, S, float><<<grid, block, 0, c->stream>>>(p, pulled, c->d.collision, static_cast<float*>(drho),
                                                                     static_cast<float*>(du));
            else
                k_macros<L, S, double><<<grid, block, 0, c->stream>>>(p, pulled, c->d.collision,
                                                                      static_cast<double*>(drho), static_cast<double*>(du));
        });
    });
    LBM_CK(cudaGetLastError());
    if (memory == LBM_HOST) {
        if (rho) LBM_CK(cudaMemcpyAsync(rho, drho, elt * c->N, cudaMemcpyDeviceToHost, c->stream));
        if (u) LBM_CK(cudaMemcpyAsync(u, du, elt * c->N * c->dim, cudaMemcpyDeviceToHost, c->stream));
    }
    LBM_CK(cudaStreamSynchronize(c->stream));
    return LBM_OK;
}

int lbm_sums_fp64(lbm_ctx* c, double out[4]) {
    if (!c || !out) return set_error(LBM_ERR_INVALID, "NULL argument");
    LBM_CK(cudaSetDevice(c->d.device));
    dispatch_storage(c->d.storage, [&](auto tag) {
        using S = typename decltype(tag)::type;
        dispatch_lattice(c->d.lattice, [&](auto lt) {
            using L = typename decltype(lt)::type;
            k_sums_partial<L, S><<<c->reduce_blocks, 256, 0, c->stream>>>(static_cast<const S*>(c->f[c->cur]), c->N,
                                                                          (float)(1.0 / c->scale), c->partial);
        });
    });
    k_sums_final<<<1, 32, 0, c->stream>>>(c->partial, c->reduce_blocks, c->sums_out);
    LBM_CK(cudaGetLastError());
    Sums s;
    LBM_CK(cudaMemcpyAsync(&s, c->sums_out, sizeof(Sums), cudaMemcpyDeviceToHost, c->stream));
    LBM_CK(cudaStreamSynchronize(c->stream));
    out[0] = s.m;
    out[1] = s.jx;
    out[2] = s.jy;
    out[3] = s.jz;
    if (s.bad) return set_error(LBM_ERR_DIVERGED, std::to_string(s.bad) + " non-finite populations");
    return LBM_OK;
}

int lbm_residual_fp64(lbm_ctx* c, double* out) {
    if (!c || !out) return set_error(LBM_ERR_INVALID, "NULL argument");
    if (!c->has_prev) return set_error(LBM_ERR_STATE, "residual needs at least one step since the last set/init");
    LBM_CK(cudaSetDevice(c->d.device));
    dispatch_storage(c->d.storage, [&](auto tag) {
        using S = typename decltype(tag)::type;
        dispatch_lattice(c->d.lattice, [&](auto lt) {
            using L = typename decltype(lt)::type;
            k_residual_partial<L, S><<<c->reduce_blocks, 256, 0, c->stream>>>(
                static_cast<const S*>(c->f[c->cur]), static_cast<const S*>(c->f[c->cur ^ 1]), c->mask, c->N,
                (float)(1.0 / c->scale), c->partial);
        });
    });
    k_sums_final<<<1, 32, 0, c->stream>>>(c->partial, c->reduce_blocks, c->sums_out);
    LBM_CK(cudaGetLastError());
    Sums s;
    LBM_CK(cudaMemcpyAsync(&s, c->sums_out, sizeof(Sums), cudaMemcpyDeviceToHost, c->stream));
    LBM_CK(cudaStreamSynchronize(c->stream));
    *out = s.jx > 0 ? std::sqrt(s.m / s.jx) : 0.0;
    if (!std::isfinite(*out)) return set_error(LBM_ERR_DIVERGED, "residual is not finite");
    return LBM_OK;
}

void* lbm_stream(lbm_ctx* c) { return c ? (void*)c->stream : nullptr; }

int lbm_set_stream(lbm_ctx* c, void* stream) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    LBM_CK(cudaSetDevice(c->d.device));
    LBM_CK(cudaStreamSynchronize(c->stream));
    c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own;
    return LBM_OK;
}

void* lbm_device_populations(lbm_ctx* c, size_t* bytes) {
    if (!c) return nullptr;
    if (bytes) *bytes = (size_t)c->N * c->q * c->sbytes;
    return c->f[c->cur];
}

// One plane of the slowest axis is contiguous per direction in the [x, y(, z), i] layout, so a face is
// one copy per direction.
static int face_copy(lbm_ctx* c, int64_t plane, const int32_t* dirs, int32_t ndirs, void* host_or_dev,
                     int memory, bool get) {
    if (!c || !dirs || !host_or_dev) return set_error(LBM_ERR_INVALID, "NULL argument");
    if (memory != LBM_HOST && memory != LBM_DEVICE) return set_error(LBM_ERR_INVALID, "memory must be HOST or DEVICE");
    const long long planes = c->dim == 3 ? c->d.nz : c->d.ny;
    if (plane < 0 || plane >= planes) return set_error(LBM_ERR_INVALID, "plane outside the lattice");
    if (ndirs < 1 || ndirs > c->q) return set_error(LBM_ERR_INVALID, "ndirs must be in 1..Q");
    for (int k = 0; k < ndirs; ++k)
        if (dirs[k] < 0 || dirs[k] >= c->q) return set_error(LBM_ERR_INVALID, "direction outside 0..Q-1");
    LBM_CK(cudaSetDevice(c->d.device));
    const long long cells = c->N / planes;
    const size_t bytes = (size_t)cells * c->sbytes;
    char* f = static_cast<char*>(c->f[c->cur]);
    char* io = static_cast<char*>(host_or_dev);
    const cudaMemcpyKind kind = memory == LBM_HOST ? (get ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice)
                                                   : cudaMemcpyDeviceToDevice;
    for (int k = 0; k < ndirs; ++k) {
        char* dev = f + ((size_t)dirs[k] * c->N + (size_t)plane * cells) * c->sbytes;
        if (get)
            LBM_CK(cudaMemcpyAsync(io + k * bytes, dev, bytes, kind, c->stream));
        else
            LBM_CK(cudaMemcpyAsync(dev, io + k * bytes, bytes, kind, c->stream));
    }
    if (memory == LBM_HOST) LBM_CK(cudaStreamSynchronize(c->stream));
    return LBM_OK;
}

int lbm_face_get(lbm_ctx* c, int64_t plane, const int32_t* dirs, int32_t ndirs, void* dst, int memory) {
    return face_copy(c, plane, dirs, ndirs, dst, memory, true);
}

int lbm_face_set(lbm_ctx* c, int64_t plane, const int32_t* dirs, int32_t ndirs, const void* src, int memory) {
    return face_copy(c, plane, dirs, ndirs, const_cast<void*>(src), memory, false);
}

int lbm_get_desc(const lbm_ctx* c, lbm_desc* out) {
    if (!c || !out) return set_error(LBM_ERR_INVALID, "NULL argument");
    *out = c->d;
    return LBM_OK;
}

int lbm_set_block(lbm_ctx* c, int threads_x) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    if (threads_x != 0 && (threads_x < 32 || threads_x > max_block(c) || (threads_x & 31)))
        return set_error(LBM_ERR_INVALID, "block width must be 0 or a multiple of 32 within the kernel's launch bound");
    LBM_CK(cudaSetDevice(c->d.device));
    LBM_CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->block = threads_x;
    c->kernel_used = 0;
    return LBM_OK;
}

int lbm_get_block(const lbm_ctx* c) { return c ? c->block : 0; }

int lbm_set_kernel(lbm_ctx* c, int kind) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    if (kind != LBM_KERNEL_AUTO && kind != LBM_KERNEL_PLAIN && kind != LBM_KERNEL_ROWS && kind != LBM_KERNEL_CLUSTER)
        return set_error(LBM_ERR_INVALID, "unknown kernel family");
    if (kind == LBM_KERNEL_CLUSTER) {
        LBM_CK(cudaSetDevice(c->d.device));
        if (!cluster_eligible(c))
            return set_error(LBM_ERR_UNSUPPORTED,
                             "the cluster-resident kernel needs D2Q9 BGK, deviation arithmetic and both population "
                             "buffers within one cluster's shared memory");
    }
    if (kind == LBM_KERNEL_ROWS && !rows_eligible(c))
        return set_error(LBM_ERR_UNSUPPORTED,
                         "the row pipeline needs D3Q27 BGK/MRT or D2Q9 BGK, deviation arithmetic, F32/F16S/BF16S "
                         "and nx >= 32 a multiple of 16");
    LBM_CK(cudaSetDevice(c->d.device));
    LBM_CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->kernel = kind;
    c->kernel_used = 0;
    if (kind == LBM_KERNEL_ROWS || kind == LBM_KERNEL_CLUSTER) c->block = 0;
    return LBM_OK;
}

int lbm_get_kernel(const lbm_ctx* c) { return c ? c->kernel_used : 0; }

int lbm_step_planes(lbm_ctx* c, int64_t first, int64_t count, int64_t stride, int finish, void* stream) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    const long long planes = c->d.lattice == LBM_D3Q27 ? c->d.nz : c->d.ny;
    if (first < 0 || count < 1 || stride < 1 || first >= planes || (count - 1) > (planes - 1 - first) / stride)
        return set_error(LBM_ERR_INVALID, "planes outside the lattice's slowest axis");
    LBM_CK(cudaSetDevice(c->d.device));
    if (!c->kernel_used) {
        int rc = autotune(c);
        if (rc) return rc;
    }
    if (c->d.collision == LBM_SHANCHEN && !c->scw_target) {  // plane sets take the window kernel
        int rc = prepare_rows(c);
        if (rc) return rc;
    }
    // a launch on a side stream runs in the SMs that lbm_set_reserved_sms keeps from the context stream
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    launch_step(c, c->cur, s, c->block, (int)first, (int)count, (int)stride, s != c->stream && c->reserved_sms > 0);
    LBM_CK(cudaGetLastError());
    if (finish) {
        c->cur ^= 1;
        c->has_prev = true;
        c->steps += 1;
    }
    return LBM_OK;
}

int lbm_set_reserved_sms(lbm_ctx* c, int sms) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    if (sms < 0 || sms > 64) return set_error(LBM_ERR_INVALID, "reserved SMs must be in [0, 64]");
    LBM_CK(cudaSetDevice(c->d.device));
    LBM_CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);  // the graphs captured the persistent grid
    c->reserved_sms = sms;
    return LBM_OK;
}

int lbm_device_buffers(lbm_ctx* c, void** current, void** next, size_t* bytes) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    if (current) *current = c->f[c->cur];
    if (next) *next = c->f[c->cur ^ 1];
    if (bytes) *bytes = (size_t)c->N * c->q * c->sbytes;
    return LBM_OK;
}

int lbm_set_cell_offset(lbm_ctx* c, int64_t offset) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    LBM_CK(cudaSetDevice(c->d.device));
    LBM_CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);  // the graphs captured the old offset in their launch parameters
    c->cell_offset = offset;
    c->pf = make_params<float>(c);
    c->pd = make_params<double>(c);
    return LBM_OK;
}

int lbm_test_stall_next_step(lbm_ctx* c, int64_t item, int64_t wait_clocks) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    if (item < 0 || item >= 0xffffffffLL) return set_error(LBM_ERR_INVALID, "work item out of range");
    if (wait_clocks < (1LL << 10) || wait_clocks > (1LL << 32))
        return set_error(LBM_ERR_INVALID, "wait_clocks must be in [2^10, 2^32]");
    if (c->kernel != LBM_KERNEL_ROWS || c->d.collision == LBM_SHANCHEN)
        return set_error(LBM_ERR_STATE,
                         "the stall applies to the row pipeline's bulk-copy stages: pin LBM_KERNEL_ROWS (BGK/MRT) first");
    c->stall = WaitLimits{(unsigned)item, (long long)wait_clocks};
    c->stall_armed = true;
    return LBM_OK;
}

int lbm_test_index64(lbm_ctx* c, int on) {
    if (!c) return set_error(LBM_ERR_INVALID, "context is NULL");
    LBM_CK(cudaSetDevice(c->d.device));
    LBM_CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);  // captured launches name the kernel instance
    c->index64 = on != 0;
    return LBM_OK;
}

}  // extern "C"
