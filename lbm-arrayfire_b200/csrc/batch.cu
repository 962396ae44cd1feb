// batch.cu — an ensemble of independent BGK lattices (any mix of D2Q9 and D3Q27 extents and
// rates, one storage type) advanced together, so lattices of very different sizes share the SMs
// without per-lattice launches.  Each step is one persistent kernel over a work table:
//   - row pipeline, one launch (k_batch_rows_mix): items are (lattice, first row, z, rows, family)
//     groups of both lattice families staged in shared memory by bulk copies, for the members whose
//     rows the copies can move (nx a multiple of 16, at most 1024); the stage pitch is the widest such
//     row, narrower members put more rows into a stage and every consumer thread takes cells of the
//     flattened group;
//   - row pipeline per family (k_batch_rows): the same with one launch and table per lattice family
//     (kept for comparison);
//   - tile kernel (k_batch_bgk): a tile is one row segment (lattice, y, z, x0) of `tile_x` cells, one
//     thread per cell, for the other members (or all of them, if the autotuner finds that faster).
// Chunks of steps are captured in a CUDA graph and replayed.  The autotuner times the candidates on
// the real buffers.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"
#include "kernels.cuh"
#include "rowpipe.cuh"

namespace lbm {

template <class T>
struct BTag {
    using type = T;
};

// One ensemble member as the kernels see it (lives in device memory).
template <class R>
struct BatchLattice {
    void* f[2];
    const uint8_t* mask;
    int nx, ny, nz;
    long long N;
    R omega, one_m_omega;
    R scale, inv_scale;
    int sr;                         // 16-bit storage: stochastic rounding (1) or to nearest (0)
    uint32_t cell_base;             // 0: a member's cells are hashed by their own index
    alignas(16) ClassTable<R> cls;  // 16-byte aligned: the row pipeline bulk-copies it into shared memory
};

// The batch's rounding seed for a launch reading buffer `parity` (one counter pair for the whole batch,
// advanced once per step; a member stepped alone from the same start draws the same words).
template <class S>
__device__ __forceinline__ uint32_t batch_seed(unsigned* tick, int parity, bool designated) {
    if constexpr (!Codec<S>::kScaled)
        return 0u;
    else
        return step_seed(tick, parity, designated);
}

struct Tile {
    int lat, y, z, x0;
};

template <class L, class S>
__global__ void __launch_bounds__(256) k_batch_bgk(const BatchLattice<typename Codec<S>::Real>* __restrict__ lats,
                                                   const Tile* __restrict__ tiles, int parity, unsigned* tick,
                                                   int advance) {
    using R = typename Codec<S>::Real;
    const Tile t = tiles[blockIdx.x];
    const BatchLattice<R>& p = lats[t.lat];
    const int x = t.x0 + threadIdx.x;
    // every launch of a step reads the counter; the first one (advance) moves it on
    const uint32_t seed = batch_seed<S>(tick, parity, advance && (blockIdx.x | threadIdx.x) == 0);
    if (x >= p.nx) return;
    bgk_cell<L, S, false>(p, static_cast<const S*>(p.f[parity]), static_cast<S*>(p.f[parity ^ 1]), x, t.y, t.z,
                          Rounding{seed, p.sr != 0});
}

// A member's per-cell parameters for one row group: the scalars in registers (the stores of the group
// could alias the member table as far as the compiler knows, so reading them through `lats` would
// reload them after every cell) and the class table in the stage's shared memory.
template <class R>
struct MemberCell {
    long long N;
    R omega, one_m_omega;
    const ClassTable<R>& cls;
};

// One row group of one member: rows y0 .. y0 + nb - 1 at z; fam 0 = D2Q9, 1 = D3Q27.
struct RowItem {
    int lat, y0, z, nb, fam;
};

// The row pipeline's shape in the ensemble kernels (BGK: pairs of cells for 16-bit storage).
template <class L, class S, int PITCH>
using BatchShape = RowPipeShape<L, S, PITCH, false, kRowPair<L, S, 0>>;

// Shared memory of k_batch_rows: the row pipeline's stages plus one class table per stage.
template <class L, class S, int PITCH>
constexpr size_t batch_rows_smem() {
    using Sh = BatchShape<L, S, PITCH>;
    return Sh::smem_bytes() + (size_t)Sh::NS * sizeof(ClassTable<typename Codec<S>::Real>);
}

// The row pipeline of rowpipe.cuh over a work table of row groups of several lattices (BGK).
template <class L, class S, int PITCH>
__global__ void __launch_bounds__(BatchShape<L, S, PITCH>::CONSUMERS + 32, BatchShape<L, S, PITCH>::CTAS)
    k_batch_rows(const BatchLattice<typename Codec<S>::Real>* __restrict__ lats, const RowItem* __restrict__ items,
                 long long n_items, int parity, int* __restrict__ err, const WaitLimits wl, unsigned* tick,
                 int advance) {
    using R = typename Codec<S>::Real;
    using Sh = BatchShape<L, S, PITCH>;
    constexpr int Q = L::Q;
    constexpr int NS = Sh::NS;
    constexpr int SB = Sh::SB;
    constexpr int CONS = Sh::CONSUMERS;
    constexpr int W = CONS / 32;
    static_assert(NS <= 8, "barriers occupy the first 128 bytes");
    static_assert(CONS + 32 <= 2048 && PITCH <= 1024, "the reciprocal quotients below need numerators < 2^11, nx <= 1024");
    constexpr unsigned long long kCy = pack_c<L>(false), kCz = pack_c<L>(true);
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + NS;
    S* in = reinterpret_cast<S*>(smem + 128);                                 // [NS][Q][SB]
    uint8_t* mask_st = reinterpret_cast<uint8_t*>(in + (size_t)NS * Q * SB);  // [NS][SB]
    using CT = ClassTable<R>;
    static_assert(sizeof(CT) % 16 == 0 && (Sh::smem_bytes() % 16) == 0, "class-table copies need 16-byte multiples");
    CT* cls_st = reinterpret_cast<CT*>(smem + Sh::smem_bytes());              // [NS]
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    // item indices in 32 bits (the host keeps the item count below 2^31)
    const unsigned first = blockIdx.x, stride = gridDim.x, nit = (unsigned)n_items;

    auto issue = [&](unsigned g, int s) {
        if (g == wl.skip) return;  // test hook: this item's stage is never filled
        const RowItem it = items[g];
        const BatchLattice<R>& m = lats[it.lat];
        const int nx = m.nx, ny = m.ny, nz = m.nz, nb = it.nb;
        const uint32_t row_bytes = (uint32_t)(nx * sizeof(S));
        if (lane == 0)
            mbar_arrive_expect_tx(&full[s], (uint32_t)(Q * nb) * row_bytes + (m.mask ? (uint32_t)(nb * nx) : 0u) +
                                                (uint32_t)sizeof(CT));
        __syncwarp();
        if (lane < Q) {
            const int cy = (int)((kCy >> (2 * lane)) & 3) - 1, cz = (int)((kCz >> (2 * lane)) & 3) - 1;
            int zs = it.z - cz;
            zs = zs < 0 ? zs + nz : (zs >= nz ? zs - nz : zs);
            int ys = it.y0 - cy;
            ys = ys < 0 ? ys + ny : (ys >= ny ? ys - ny : ys);
            const int run = ny - ys < nb ? ny - ys : nb;
            const S* plane = static_cast<const S*>(m.f[parity]) + (long long)lane * m.N + (long long)zs * ny * nx;
            S* dst = in + ((long long)s * Q + lane) * SB;
            bulk_load(dst, plane + (long long)ys * nx, (uint32_t)run * row_bytes, &full[s]);
            if (run < nb) bulk_load(dst + run * nx, plane, (uint32_t)(nb - run) * row_bytes, &full[s]);
        } else if (lane == Q && m.mask) {
            bulk_load(mask_st + s * SB, m.mask + ((long long)it.z * ny + it.y0) * nx, (uint32_t)(nb * nx), &full[s]);
        } else if (lane == Q + 1) {
            bulk_load(cls_st + s, &m.cls, (uint32_t)sizeof(CT), &full[s]);
        }
    };

    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], W);
        }
        mbar_init_fence();
    }
    __syncthreads();
    if (tid >= CONS) {  // producer warp
        for (int s = 0; s < NS; ++s)
            if (first + s * stride < nit) issue(first + s * stride, s);
        for (unsigned k = 0; first + (k + NS) * stride < nit; ++k) {
            const int s = (int)(k % NS);
            if (!mbar_wait_bounded(&empty[s], (uint32_t)((k / NS) & 1), wl.limit)) {
                if (lane == 0) atomicExch(err, kRowPipeTimeout);
                return;
            }
            issue(first + (k + NS) * stride, s);
        }
        return;
    }
    const uint32_t seed = batch_seed<S>(tick, parity, advance && (blockIdx.x | tid) == 0);
    for (unsigned k = 0; first + k * stride < nit; ++k) {
        const unsigned g = first + k * stride;
        const int s = (int)(k % NS);
        if (!mbar_wait_bounded(&full[s], (uint32_t)((k / NS) & 1), wl.limit)) {
            if (lane == 0) atomicExch(err, kRowPipeTimeout);
            for (unsigned j = 1; j < NS && first + (k + j) * stride < nit; ++j)
                if (!mbar_wait_bounded(&full[(k + j) % NS], (uint32_t)(((k + j) / NS) & 1),
                                       wl.limit < (1LL << 28) ? wl.limit : (1LL << 28)))
                    break;
            return;
        }
        const RowItem it = items[g];
        const BatchLattice<R>& m = lats[it.lat];
        const int nx = m.nx;
        R sc, isc;
        storage_scale<S>(m, sc, isc);
        const MemberCell<R> mc{m.N, m.omega, m.one_m_omega, cls_st[s]};
        const S* st = in + (long long)s * Q * SB;
        const uint8_t* ms = m.mask ? mask_st + s * SB : nullptr;
        S* out0 = static_cast<S*>(m.f[parity ^ 1]) + ((long long)it.z * m.ny + it.y0) * nx;
        const uint32_t cell0 = (uint32_t)(((long long)it.z * m.ny + it.y0) * nx);
        const Rounding rnd{seed, m.sr != 0};
        // cells of the group, flattened (row b, column x), CONS apart.  tid / nx and CONS / nx by a
        // float reciprocal: exact here (numerators below 2^11, nx <= 1024: the quotient's distance to
        // the next integer, at least 1/(2 nx), is far above the rounding error)
        // 16-bit storage: pairs of adjacent cells (row_pair), nx / 2 per row
        constexpr bool kPair = kRowPair<L, S, 0>;
        const int cw = kPair ? nx >> 1 : nx;
        const float inv_nx = __frcp_rn((float)cw);
        int b = (int)(((float)tid + 0.5f) * inv_nx), x = tid - b * cw;
        const int cq = (int)(((float)CONS + 0.5f) * inv_nx), cr = CONS - cq * cw;
        const int nb = it.nb;
#pragma unroll 1
        while (b < nb) {
            if constexpr (kPair)
                row_pair_wrap<L, S, SB, 0>(mc, st + b * nx, ms ? ms + b * nx : nullptr, 2 * x, nx, sc, isc,
                                           out0 + (long long)b * nx, rnd, cell0 + (uint32_t)(b * nx));
            else
                row_cell_wrap<L, S, SB, 0>(mc, st + b * nx, ms ? ms + b * nx : nullptr, x, nx, sc, isc,
                                           out0 + (long long)b * nx, rnd, cell0 + (uint32_t)(b * nx));
            x += cr;
            b += cq;
            if (x >= cw) {
                x -= cw;
                ++b;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

// The whole ensemble in one persistent launch: one work table holds the row groups of both lattice
// families, and every CTA has the D3Q27 shape (BatchShape<D3Q27, S, PITCH>: consumer count, stage
// size, stages).  A stage keeps 27 direction slots of SB elements; a D2Q9 group fills the first 9 (its
// rows sized by the host so that nb * nx <= SB), a D3Q27 group all of them; the mask rows and the
// member's class table follow as in k_batch_rows.  Lanes 0 .. Q-1 of the producer copy the directions,
// lane 27 the mask rows, lane 28 the class table.  Each consumer runs the collision of the item's family
// (both are compiled into the kernel; the register budget is D3Q27's).
template <class S, int PITCH>
__global__ void __launch_bounds__(BatchShape<D3Q27, S, PITCH>::CONSUMERS + 32, BatchShape<D3Q27, S, PITCH>::CTAS)
    k_batch_rows_mix(const BatchLattice<typename Codec<S>::Real>* __restrict__ lats,
                     const RowItem* __restrict__ items, long long n_items, int parity, int* __restrict__ err,
                     const WaitLimits wl, unsigned* tick, int advance) {
    using R = typename Codec<S>::Real;
    using Sh = BatchShape<D3Q27, S, PITCH>;
    constexpr int NS = Sh::NS;
    constexpr int SB = Sh::SB;
    constexpr int CONS = Sh::CONSUMERS;
    constexpr int W = CONS / 32;
    static_assert(NS <= 8, "barriers occupy the first 128 bytes");
    static_assert(CONS + 32 <= 2048 && PITCH <= 1024, "the reciprocal quotients below need numerators < 2^11, nx <= 1024");
    constexpr unsigned long long kCy3 = pack_c<D3Q27>(false), kCz3 = pack_c<D3Q27>(true), kCy2 = pack_c<D2Q9>(false);
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + NS;
    S* in = reinterpret_cast<S*>(smem + 128);                                  // [NS][27][SB]
    uint8_t* mask_st = reinterpret_cast<uint8_t*>(in + (size_t)NS * 27 * SB);  // [NS][SB]
    using CT = ClassTable<R>;
    static_assert(sizeof(CT) % 16 == 0 && (Sh::smem_bytes() % 16) == 0, "class-table copies need 16-byte multiples");
    CT* cls_st = reinterpret_cast<CT*>(smem + Sh::smem_bytes());               // [NS]
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const unsigned first = blockIdx.x, stride = gridDim.x, nit = (unsigned)n_items;

    auto issue = [&](unsigned g, int s) {
        if (g == wl.skip) return;  // test hook: this item's stage is never filled
        const RowItem it = items[g];
        const BatchLattice<R>& m = lats[it.lat];
        const int nx = m.nx, ny = m.ny, nz = m.nz, nb = it.nb;
        const int Q = it.fam ? 27 : 9;
        const uint32_t row_bytes = (uint32_t)(nx * sizeof(S));
        if (lane == 0)
            mbar_arrive_expect_tx(&full[s], (uint32_t)(Q * nb) * row_bytes + (m.mask ? (uint32_t)(nb * nx) : 0u) +
                                                (uint32_t)sizeof(CT));
        __syncwarp();
        if (lane < Q) {
            const int cy = (int)(((it.fam ? kCy3 : kCy2) >> (2 * lane)) & 3) - 1;
            const int cz = it.fam ? (int)((kCz3 >> (2 * lane)) & 3) - 1 : 0;
            int zs = it.z - cz;
            zs = zs < 0 ? zs + nz : (zs >= nz ? zs - nz : zs);
            int ys = it.y0 - cy;
            ys = ys < 0 ? ys + ny : (ys >= ny ? ys - ny : ys);
            const int run = ny - ys < nb ? ny - ys : nb;
            const S* plane = static_cast<const S*>(m.f[parity]) + (long long)lane * m.N + (long long)zs * ny * nx;
            S* dst = in + ((long long)s * 27 + lane) * SB;
            bulk_load(dst, plane + (long long)ys * nx, (uint32_t)run * row_bytes, &full[s]);
            if (run < nb) bulk_load(dst + run * nx, plane, (uint32_t)(nb - run) * row_bytes, &full[s]);
        } else if (lane == 27 && m.mask) {
            bulk_load(mask_st + s * SB, m.mask + ((long long)it.z * ny + it.y0) * nx, (uint32_t)(nb * nx), &full[s]);
        } else if (lane == 28) {
            bulk_load(cls_st + s, &m.cls, (uint32_t)sizeof(CT), &full[s]);
        }
    };

    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], W);
        }
        mbar_init_fence();
    }
    __syncthreads();
    if (tid >= CONS) {  // producer warp
        for (int s = 0; s < NS; ++s)
            if (first + s * stride < nit) issue(first + s * stride, s);
        for (unsigned k = 0; first + (k + NS) * stride < nit; ++k) {
            const int s = (int)(k % NS);
            if (!mbar_wait_bounded(&empty[s], (uint32_t)((k / NS) & 1), wl.limit)) {
                if (lane == 0) atomicExch(err, kRowPipeTimeout);
                return;
            }
            issue(first + (k + NS) * stride, s);
        }
        return;
    }
    const uint32_t seed = batch_seed<S>(tick, parity, advance && (blockIdx.x | tid) == 0);
    for (unsigned k = 0; first + k * stride < nit; ++k) {
        const unsigned g = first + k * stride;
        const int s = (int)(k % NS);
        if (!mbar_wait_bounded(&full[s], (uint32_t)((k / NS) & 1), wl.limit)) {
            if (lane == 0) atomicExch(err, kRowPipeTimeout);
            for (unsigned j = 1; j < NS && first + (k + j) * stride < nit; ++j)
                if (!mbar_wait_bounded(&full[(k + j) % NS], (uint32_t)(((k + j) / NS) & 1),
                                       wl.limit < (1LL << 28) ? wl.limit : (1LL << 28)))
                    break;
            return;
        }
        const RowItem it = items[g];
        const BatchLattice<R>& m = lats[it.lat];
        const int nx = m.nx;
        R sc, isc;
        storage_scale<S>(m, sc, isc);
        const MemberCell<R> mc{m.N, m.omega, m.one_m_omega, cls_st[s]};
        const S* st = in + (long long)s * 27 * SB;
        const uint8_t* ms = m.mask ? mask_st + s * SB : nullptr;
        S* out0 = static_cast<S*>(m.f[parity ^ 1]) + ((long long)it.z * m.ny + it.y0) * nx;
        const uint32_t cell0 = (uint32_t)(((long long)it.z * m.ny + it.y0) * nx);
        const Rounding rnd{seed, m.sr != 0};
        // cells of the group, flattened (row b, column x), CONS apart (as k_batch_rows)
        // 16-bit storage: pairs of adjacent cells (row_pair), nx / 2 per row
        constexpr bool kPair = kRowPair<D3Q27, S, 0>;
        const int cw = kPair ? nx >> 1 : nx;
        const float inv_nx = __frcp_rn((float)cw);
        int b = (int)(((float)tid + 0.5f) * inv_nx), x = tid - b * cw;
        const int cq = (int)(((float)CONS + 0.5f) * inv_nx), cr = CONS - cq * cw;
        const int nb = it.nb;
        auto walk = [&](auto lt) {
            using L = typename decltype(lt)::type;
#pragma unroll 1
            while (b < nb) {
                if constexpr (kPair)
                    row_pair_wrap<L, S, SB, 0>(mc, st + b * nx, ms ? ms + b * nx : nullptr, 2 * x, nx, sc, isc,
                                               out0 + (long long)b * nx, rnd, cell0 + (uint32_t)(b * nx));
                else
                    row_cell_wrap<L, S, SB, 0>(mc, st + b * nx, ms ? ms + b * nx : nullptr, x, nx, sc, isc,
                                               out0 + (long long)b * nx, rnd, cell0 + (uint32_t)(b * nx));
                x += cr;
                b += cq;
                if (x >= cw) {
                    x -= cw;
                    ++b;
                }
            }
        };
        if (it.fam)
            walk(BTag<D3Q27>{});
        else
            walk(BTag<D2Q9>{});
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

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
    int mode = 0;                    // LBM_BATCH_AUTO / TILES / ROWS
    bool use_rows = false;           // row pipeline for the eligible members
    int rows_pitch[2] = {0, 0};      // shared-memory row pitch per family
    RowItem* items_d[2] = {nullptr, nullptr};
    long long n_items[2] = {0, 0};
    int rows_grid[2] = {0, 0};
    // the one-launch table of both families (k_batch_rows_mix), used when `mixed`
    bool mixed = false;
    int mix_pitch = 0;
    RowItem* mix_items_d = nullptr;
    long long mix_n = 0;
    int mix_grid = 0;
    int group_bytes[2] = {0, 0};     // copy-size targets of its row groups (D2Q9, D3Q27)
    int* err = nullptr;              // device error word of the row pipeline
    unsigned* tick = nullptr;        // the rounding's step counter pair (device)
    WaitLimits waits = kProductionWaits;  // wait limits of the next row-pipeline launches
    bool stall_armed = false;        // lbm_batch_test_stall_next_step
    WaitLimits stall = kProductionWaits;
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

// Row pipeline eligibility of one member: bulk copies move whole rows (nx a multiple of 16, <= 1024).
static bool batch_row_member(const lbm_batch* b, int k) {
    const lbm_desc& d = b->descs[k];
    return b->storage != LBM_F64 && d.nx >= 32 && d.nx <= 1024 && d.nx % 16 == 0;
}

static int pitch_for(long long nx) { return nx <= 128 ? 128 : nx <= 256 ? 256 : nx <= 512 ? 512 : 1024; }

// f(lattice tag, storage tag, pitch constant) for family fam (0 = D2Q9, 1 = D3Q27)
template <class F>
static void batch_rows_dispatch(const lbm_batch* b, int fam, F&& f) {
    auto by_pitch = [&](auto lt, auto st) {
        switch (b->rows_pitch[fam]) {
            case 128: f(lt, st, std::integral_constant<int, 128>{}); break;
            case 256: f(lt, st, std::integral_constant<int, 256>{}); break;
            case 512: f(lt, st, std::integral_constant<int, 512>{}); break;
            default: f(lt, st, std::integral_constant<int, 1024>{}); break;
        }
    };
    auto by_storage = [&](auto lt) {
        switch (b->storage) {
            case LBM_F32: by_pitch(lt, BTag<float>{}); break;
            case LBM_F16S: by_pitch(lt, BTag<__half>{}); break;
            default: by_pitch(lt, BTag<__nv_bfloat16>{}); break;
        }
    };
    if (fam == 0)
        by_storage(BTag<D2Q9>{});
    else
        by_storage(BTag<D3Q27>{});
}

// f(storage tag, pitch constant) for the one-launch kernel (pitch b->mix_pitch)
template <class F>
static void batch_mix_dispatch(const lbm_batch* b, F&& f) {
    auto by_pitch = [&](auto st) {
        switch (b->mix_pitch) {
            case 128: f(st, std::integral_constant<int, 128>{}); break;
            case 256: f(st, std::integral_constant<int, 256>{}); break;
            case 512: f(st, std::integral_constant<int, 512>{}); break;
            default: f(st, std::integral_constant<int, 1024>{}); break;
        }
    };
    switch (b->storage) {
        case LBM_F32: by_pitch(BTag<float>{}); break;
        case LBM_F16S: by_pitch(BTag<__half>{}); break;
        default: by_pitch(BTag<__nv_bfloat16>{}); break;
    }
}

// Work tables of the row pipeline: per family, the row groups of its eligible members.
static int batch_build_rows(lbm_batch* b) {
    int sms = 0;
    LBM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    for (int fam = 0; fam < 2; ++fam) {
        long long maxnx = 0;
        for (int k = 0; k < (int)b->descs.size(); ++k)
            if ((b->descs[k].lattice == LBM_D2Q9) == (fam == 0) && batch_row_member(b, k))
                maxnx = std::max<long long>(maxnx, b->descs[k].nx);
        if (!maxnx) continue;
        b->rows_pitch[fam] = pitch_for(maxnx);
        std::vector<RowItem> items;
        int rc = LBM_OK;
        batch_rows_dispatch(b, fam, [&](auto lt, auto st, auto pi) {
            using L = typename decltype(lt)::type;
            using S = typename decltype(st)::type;
            constexpr int PITCH = decltype(pi)::value;
            using Sh = BatchShape<L, S, PITCH>;
            for (int k = 0; k < (int)b->descs.size(); ++k) {
                const lbm_desc& d = b->descs[k];
                if ((d.lattice == LBM_D2Q9) != (fam == 0) || !batch_row_member(b, k)) continue;
                const int rpg = Sh::rows_per_group((int)d.nx);
                for (int z = 0; z < (int)d.nz; ++z)
                    for (int y0 = 0; y0 < (int)d.ny; y0 += rpg)
                        items.push_back(RowItem{k, y0, z, (int)std::min<long long>(rpg, d.ny - y0), fam});
            }
            auto kern = k_batch_rows<L, S, PITCH>;
            constexpr size_t smem = batch_rows_smem<L, S, PITCH>();
            if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
                rc = set_error(LBM_ERR_CUDA, "row pipeline shared-memory attribute");
                return;
            }
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Sh::CONSUMERS + 32, smem) != cudaSuccess ||
                per_sm < 1) {
                rc = set_error(LBM_ERR_UNSUPPORTED, "row pipeline does not fit on an SM");
                return;
            }
            b->rows_grid[fam] = (int)std::min<long long>((long long)items.size(), (long long)per_sm * sms);
        });
        if (rc) return rc;
        if (items.size() >= (1ull << 31)) return set_error(LBM_ERR_UNSUPPORTED, "row work table over 2^31 items");
        if (b->items_d[fam]) cudaFree(b->items_d[fam]);
        b->items_d[fam] = nullptr;
        b->n_items[fam] = (long long)items.size();
        if (cudaMalloc(&b->items_d[fam], sizeof(RowItem) * items.size()) != cudaSuccess) {
            cudaGetLastError();
            return set_error(LBM_ERR_NOMEM, "row work table allocation failed");
        }
        LBM_CK(cudaMemcpy(b->items_d[fam], items.data(), sizeof(RowItem) * items.size(), cudaMemcpyHostToDevice));
    }
    return LBM_OK;
}

// The one-launch work table (k_batch_rows_mix): the row groups of every eligible member of both
// families.  The stage pitch is the widest eligible row of the ensemble; a group's rows are sized for
// `scale` times the per-family copy target (RowPipeShape::kGroupBytes, per direction) and never exceed a
// stage (nb * nx <= SB).  The scale is the autotuner's cells-per-thread knob: a group of nb rows gives
// each consumer thread nb * nx / CONSUMERS cells per stage.
static int batch_build_mixed(lbm_batch* b, double scale) {
    int sms = 0;
    LBM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    long long maxnx = 0;
    for (int k = 0; k < (int)b->descs.size(); ++k)
        if (batch_row_member(b, k)) maxnx = std::max<long long>(maxnx, b->descs[k].nx);
    if (!maxnx) return set_error(LBM_ERR_UNSUPPORTED, "no member fits the row pipeline");
    b->mix_pitch = pitch_for(maxnx);
    std::vector<RowItem> items;
    int rc = LBM_OK;
    auto build = [&](auto st, auto pi) {
        using S = typename decltype(st)::type;
        constexpr int PITCH = decltype(pi)::value;
        using Sh = BatchShape<D3Q27, S, PITCH>;
        const int target[2] = {(int)(RowPipeShape<D2Q9, S, PITCH>::kGroupBytes * scale), (int)(Sh::kGroupBytes * scale)};
        b->group_bytes[0] = target[0];
        b->group_bytes[1] = target[1];
        for (int k = 0; k < (int)b->descs.size(); ++k) {
            if (!batch_row_member(b, k)) continue;
            const lbm_desc& d = b->descs[k];
            const int fam = d.lattice == LBM_D2Q9 ? 0 : 1;
            int rpg = target[fam] / (int)(d.nx * sizeof(S));
            rpg = std::max(1, std::min<int>(rpg, (int)(Sh::SB / d.nx)));
            for (int z = 0; z < (int)d.nz; ++z)
                for (int y0 = 0; y0 < (int)d.ny; y0 += rpg)
                    items.push_back(RowItem{k, y0, z, (int)std::min<long long>(rpg, d.ny - y0), fam});
        }
        auto kern = k_batch_rows_mix<S, PITCH>;
        constexpr size_t smem = batch_rows_smem<D3Q27, S, PITCH>();
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            rc = set_error(LBM_ERR_CUDA, "row pipeline shared-memory attribute");
            return;
        }
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Sh::CONSUMERS + 32, smem) != cudaSuccess ||
            per_sm < 1) {
            rc = set_error(LBM_ERR_UNSUPPORTED, "row pipeline does not fit on an SM");
            return;
        }
        b->mix_grid = (int)std::min<long long>((long long)items.size(), (long long)per_sm * sms);
    };
    batch_mix_dispatch(b, build);
    if (rc) return rc;
    if (items.size() >= (1ull << 31)) return set_error(LBM_ERR_UNSUPPORTED, "row work table over 2^31 items");
    if (b->mix_items_d) cudaFree(b->mix_items_d);
    b->mix_items_d = nullptr;
    b->mix_n = (long long)items.size();
    if (cudaMalloc(&b->mix_items_d, sizeof(RowItem) * items.size()) != cudaSuccess) {
        cudaGetLastError();
        return set_error(LBM_ERR_NOMEM, "row work table allocation failed");
    }
    LBM_CK(cudaMemcpy(b->mix_items_d, items.data(), sizeof(RowItem) * items.size(), cudaMemcpyHostToDevice));
    return LBM_OK;
}

static int batch_build_tiles(lbm_batch* b, int tile_x) {
    std::vector<Tile> t[2];
    for (int k = 0; k < (int)b->descs.size(); ++k) {
        const lbm_desc& d = b->descs[k];
        const int fam = d.lattice == LBM_D2Q9 ? 0 : 1;
        if (b->use_rows && batch_row_member(b, k)) continue;  // stepped by the row pipeline
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

// One step of the whole ensemble: the tile launches (members the row copies cannot move), then the row
// pipeline.  The first launch of the step advances the rounding counter (`advance`).
static void batch_launch(lbm_batch* b, int parity, cudaStream_t s) {
    int advance = 1;
    batch_dispatch(b->storage, [&](auto tag) {
        using S = typename decltype(tag)::type;
        using R = typename Codec<S>::Real;
        const auto* lats = static_cast<const BatchLattice<R>*>(b->lats_d);
        if (b->n_tiles[0])
            k_batch_bgk<D2Q9, S><<<(unsigned)b->n_tiles[0], b->tile_x, 0, s>>>(lats, b->tiles_d[0], parity, b->tick,
                                                                             advance);
        advance = advance && !b->n_tiles[0];
        if (b->n_tiles[1])
            k_batch_bgk<D3Q27, S><<<(unsigned)b->n_tiles[1], b->tile_x, 0, s>>>(lats, b->tiles_d[1], parity, b->tick,
                                                                              advance);
        advance = advance && !b->n_tiles[1];
    });
    if (!b->use_rows) return;
    if (b->mixed) {
        batch_mix_dispatch(b, [&](auto st, auto pi) {
            using S = typename decltype(st)::type;
            using R = typename Codec<S>::Real;
            constexpr int PITCH = decltype(pi)::value;
            using Sh = BatchShape<D3Q27, S, PITCH>;
            k_batch_rows_mix<S, PITCH><<<b->mix_grid, Sh::CONSUMERS + 32, batch_rows_smem<D3Q27, S, PITCH>(), s>>>(
                static_cast<const BatchLattice<R>*>(b->lats_d), b->mix_items_d, b->mix_n, parity, b->err, b->waits,
                b->tick, advance);
        });
        return;
    }
    for (int fam = 0; fam < 2; ++fam) {
        if (!b->n_items[fam]) continue;
        batch_rows_dispatch(b, fam, [&](auto lt, auto st, auto pi) {
            using L = typename decltype(lt)::type;
            using S = typename decltype(st)::type;
            using R = typename Codec<S>::Real;
            using Sh = BatchShape<L, S, decltype(pi)::value>;
            k_batch_rows<L, S, decltype(pi)::value><<<b->rows_grid[fam], Sh::CONSUMERS + 32,
                                                      batch_rows_smem<L, S, decltype(pi)::value>(), s>>>(
                static_cast<const BatchLattice<R>*>(b->lats_d), b->items_d[fam], b->n_items[fam], parity, b->err,
                b->waits, b->tick, advance);
            advance = 0;
        });
    }
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

// Configuration: time a step of each candidate on the real buffers (reads the current buffers, writes
// the others) and keep the fastest.  The candidates are the halo strategy and the cells per thread:
//   - tiles: every member on the one-thread-per-cell tile kernel (halos read straight from global
//     memory through L1/L2), tile widths 64 / 128 / 256;
//   - rows, one launch: the eligible members' row groups staged by bulk copies (halos in shared memory)
//     in one work table of both families (k_batch_rows_mix), group sizes 0.5x / 1x / 2x the per-family
//     copy target (the cells each consumer thread takes per stage), the best tile width for the rest;
//   - rows per family: one row-pipeline launch per lattice family (k_batch_rows), for comparison.
// lbm_batch_set_mode pins TILES, ROWS (one launch) or ROWS_PER_FAMILY.
static int batch_autotune(lbm_batch* b) {
    cudaEvent_t e0, e1;
    LBM_CK(cudaEventCreate(&e0));
    LBM_CK(cudaEventCreate(&e1));
    auto time_step = [&](float& ms) -> int {
        batch_launch(b, b->parity, b->stream);
        LBM_CK(cudaEventRecord(e0, b->stream));
        for (int r = 0; r < 2; ++r) batch_launch(b, b->parity, b->stream);
        LBM_CK(cudaEventRecord(e1, b->stream));
        LBM_CK(cudaEventSynchronize(e1));
        LBM_CK(cudaEventElapsedTime(&ms, e0, e1));
        return LBM_OK;
    };
    bool any_rows = false;
    for (int k = 0; k < (int)b->descs.size(); ++k) any_rows = any_rows || batch_row_member(b, k);
    float best = 1e30f;
    int best_tx = 128;
    int best_kind = 0;  // 0 tiles, 1 rows (one launch), 2 rows per family
    double best_scale = 1.0;
    int rc = LBM_OK;
    b->use_rows = false;
    b->mixed = false;
    for (int tx : {64, 128, 256}) {
        if (b->mode != LBM_BATCH_AUTO && b->mode != LBM_BATCH_TILES && tx != 128) continue;
        rc = batch_build_tiles(b, tx);
        float ms = 0;
        if (!rc) rc = time_step(ms);
        if (rc) return rc;
        if (ms < best && (b->mode == LBM_BATCH_AUTO || b->mode == LBM_BATCH_TILES || !any_rows)) {
            best = ms;
            best_tx = tx;
        }
    }
    if (any_rows && (b->mode == LBM_BATCH_AUTO || b->mode == LBM_BATCH_ROWS)) {
        b->use_rows = true;
        b->mixed = true;
        if ((rc = batch_build_tiles(b, best_tx))) return rc;
        for (double scale : {0.5, 1.0, 2.0}) {
            rc = batch_build_mixed(b, scale);
            float ms = 0;
            if (!rc) rc = time_step(ms);
            if (rc) return rc;
            if (ms < best || (b->mode == LBM_BATCH_ROWS && best_kind != 1)) {
                best = ms;
                best_kind = 1;
                best_scale = scale;
            }
        }
    }
    if (any_rows && (b->mode == LBM_BATCH_AUTO || b->mode == LBM_BATCH_ROWS_PER_FAMILY)) {
        b->use_rows = true;
        b->mixed = false;
        rc = batch_build_rows(b);
        if (!rc) rc = batch_build_tiles(b, best_tx);
        float ms = 0;
        if (!rc) rc = time_step(ms);
        if (rc) return rc;
        if (ms < best || (b->mode == LBM_BATCH_ROWS_PER_FAMILY && best_kind != 2)) {
            best = ms;
            best_kind = 2;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    LBM_CK(cudaGetLastError());
    b->use_rows = best_kind != 0;
    b->mixed = best_kind == 1;
    if (best_kind == 1 && (rc = batch_build_mixed(b, best_scale))) return rc;
    if (best_kind == 2 && (rc = batch_build_rows(b))) return rc;
    return batch_build_tiles(b, best_tx);
}

// Kernel launches per step of the configuration in use.
static int batch_launches(const lbm_batch* b) {
    int n = (b->n_tiles[0] > 0) + (b->n_tiles[1] > 0);
    if (b->use_rows) n += b->mixed ? (b->mix_n > 0) : (b->n_items[0] > 0) + (b->n_items[1] > 0);
    return n;
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
    cudaFree(b->items_d[0]);
    cudaFree(b->items_d[1]);
    cudaFree(b->mix_items_d);
    cudaFree(b->err);
    cudaFree(b->tick);
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
    if (cudaMalloc(&b->err, sizeof(int)) != cudaSuccess || cudaMemset(b->err, 0, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->tick, 2 * sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(b->tick, 0, 2 * sizeof(unsigned)) != cudaSuccess) {
        cudaGetLastError();
        batch_free(b);
        return set_error(LBM_ERR_NOMEM, "error word allocation failed");
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
            L.sr = d.rounding == LBM_ROUND_STOCHASTIC ? 1 : 0;
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
    if (b->stall_armed) {
        // the armed test stall: one direct launch with its wait limits, before any graph
        b->stall_armed = false;
        b->waits = b->stall;
        batch_launch(b, b->parity, b->stream);
        b->waits = kProductionWaits;
        b->parity ^= 1;
        --n;
    }
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
    int e = 0;
    LBM_CK(cudaMemcpy(&e, b->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        LBM_CK(cudaMemset(b->err, 0, sizeof(int)));
        return set_error(LBM_ERR_TIMEOUT, "a row-pipeline barrier wait ran out (the step did not complete)");
    }
    return LBM_OK;
}

int lbm_batch_test_stall_next_step(lbm_batch* b, int64_t item, int64_t wait_clocks) {
    if (!b) return set_error(LBM_ERR_INVALID, "batch is NULL");
    if (item < 0 || item >= 0xffffffffLL) return set_error(LBM_ERR_INVALID, "work item out of range");
    if (wait_clocks < (1LL << 10) || wait_clocks > (1LL << 32))
        return set_error(LBM_ERR_INVALID, "wait_clocks must be in [2^10, 2^32]");
    if (!b->tile_x || !b->use_rows)
        return set_error(LBM_ERR_STATE, "the stall applies to the row pipeline: step once in a row mode first");
    b->stall = WaitLimits{(unsigned)item, (long long)wait_clocks};
    b->stall_armed = true;
    return LBM_OK;
}

int lbm_batch_plan(const lbm_batch* b, int* launches_per_step, int* group_bytes_d2q9, int* group_bytes_d3q27) {
    if (!b) return set_error(LBM_ERR_INVALID, "batch is NULL");
    if (launches_per_step) *launches_per_step = b->tile_x ? batch_launches(b) : 0;
    if (group_bytes_d2q9) *group_bytes_d2q9 = b->mixed ? b->group_bytes[0] : 0;
    if (group_bytes_d3q27) *group_bytes_d3q27 = b->mixed ? b->group_bytes[1] : 0;
    return LBM_OK;
}

int lbm_batch_set_mode(lbm_batch* b, int mode) {
    if (!b) return set_error(LBM_ERR_INVALID, "batch is NULL");
    if (mode != LBM_BATCH_AUTO && mode != LBM_BATCH_TILES && mode != LBM_BATCH_ROWS &&
        mode != LBM_BATCH_ROWS_PER_FAMILY)
        return set_error(LBM_ERR_INVALID, "unknown batch mode");
    LBM_CK(cudaSetDevice(b->device));
    LBM_CK(cudaStreamSynchronize(b->stream));
    b->mode = mode;
    b->tile_x = 0;  // re-tune on the next step
    batch_drop_graphs(b);
    return LBM_OK;
}

int lbm_batch_get_mode(const lbm_batch* b) {
    if (!b) return set_error(LBM_ERR_INVALID, "batch is NULL");
    if (!b->tile_x) return LBM_BATCH_AUTO;
    return !b->use_rows ? LBM_BATCH_TILES : b->mixed ? LBM_BATCH_ROWS : LBM_BATCH_ROWS_PER_FAMILY;
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
