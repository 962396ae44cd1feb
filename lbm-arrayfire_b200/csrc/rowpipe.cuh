// rowpipe.cuh — the D3Q27 (BGK, MRT) and D2Q9 (BGK) step kernel with bulk-copy (TMA) staging of
// lattice rows.
//
// A CTA owns a group of up to B consecutive lattice rows (y0..y0+nb-1, z) at a time — one thread per
// x, each handling the nb cells of its column — and walks a strided list of row groups.  For each
// group it needs, per direction i, the source rows (y0+b - cy_i, z - cz_i) of plane i: one contiguous
// run of memory, split in two where the group wraps around y.  The x shift of the pull (af::shift
// semantics, periodic in x) becomes an index offset inside the staged rows.
//
// Warp specialisation: one producer warp issues `cp.async.bulk` global->shared copies (one or two per
// direction per group, plus the mask rows) into a ring of NS shared-memory stages; each stage's
// completion is counted in bytes on an mbarrier (full[s]).  The consumer warps wait on full[s], read
// the staged populations with immediate-offset shared loads, collide, store their cells straight to
// global memory (coalesced along x) and release the stage on empty[s]; the producer refills a stage as
// soon as empty[s] completes.  Measured on B200 (MRT, 256^3), against the alternatives:
//   - staging the outputs for bulk stores too: 25 vs 29 GLUPS (FP32) — twice the copies, each small;
//     every copy is a separate DRAM stream, so a group spans 1-4 KB per direction (RowPipeShape);
//   - no producer warp, the last consumer warp out of a stage refilling it: 40 vs 44 GLUPS (F16S),
//     25 vs 28 GLUPS (FP32) — the refill then waits for the slowest warp of the CTA;
//   - outputs through a per-warp shared-memory transpose and 16-byte stores along the planes (fewer
//     store and address instructions, smaller groups to make room): 43.0 vs 43.7 GLUPS (F16S MRT),
//     46.6 vs 48.1 (F16S BGK).
// Compared with the one-cell-per-thread kernel this removes the per-population 64-bit load-address
// arithmetic and decouples memory latency from occupancy.
//
// Every wait on an mbarrier is bounded (about two seconds, WaitLimits); a warp that times out records
// kRowPipeTimeout in *err and returns.  Consumers first wait (bounded, 2^28 clocks at most) for the
// copies already issued into their later stages.  Once any consumer warp has left, the stage it held is
// never released, so the producer issues nothing more and itself times out on that stage.  The one case
// left open: a copy that has not landed when that last bounded wait gives up (a DRAM read stalled for
// over 0.1 s) would still be in flight into the CTA's shared memory after it exits.
// No multicast: every copy moves data of this GPU's own memory into this CTA's shared memory.
#pragma once

#include <cstdint>

#include "kernels.cuh"

namespace lbm {

constexpr int kRowPipeTimeout = 1;

// Limits of a launch's mbarrier waits.  In production skip = ~0u (every work item is issued) and every
// wait gives up after `limit` = 2^32 clocks (about two seconds).  The test hook lbm_test_stall_next_step
// sets skip to one work item, whose copies the producer then never issues (nothing is in flight for it,
// so nothing can fault), and a short limit: the consumers waiting for that stage give up, then the
// producer, and the launch returns with kRowPipeTimeout in the error word.
struct WaitLimits {
    unsigned skip;
    long long limit;
};
constexpr WaitLimits kProductionWaits{~0u, 1LL << 32};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// try_wait with a suspend-time hint (1 ms): the warp may be parked until the phase completes.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity), "r"(1000000u)
        : "memory");
    return done != 0;
}
// Bounded wait: false after `limit` clocks (2^32 is about two seconds) without completion.
// (An explicit __nanosleep back-off between polls was measured: no change in throughput.)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit = 1LL << 32) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}
// A bounded wait with a chosen polling: SLEEP_NS = 0 the hinted wait; > 0 unhinted polls with a fixed
// sleep between them (bounded by the same clock limit).
template <int SLEEP_NS>
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t* bar, uint32_t parity, long long limit = 1LL << 32) {
    if constexpr (SLEEP_NS > 0) {
        const long long t0 = clock64();
        while (true) {
            uint32_t done;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(smem_addr(bar)), "r"(parity)
                : "memory");
            if (done) return true;
            if (clock64() - t0 > limit) return false;
            __nanosleep(SLEEP_NS);
        }
    }
    return mbar_wait_bounded(bar, parity, limit);
}
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst_smem)),
                 "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// (cy, cz) of direction i packed two bits each, so a lane can look its own up at run time.
template <class L>
constexpr unsigned long long pack_c(bool z) {
    unsigned long long v = 0;
    for (int i = 0; i < L::Q; ++i) v |= (unsigned long long)((z ? L::cz(i) : L::cy(i)) + 1) << (2 * i);
    return v;
}

#ifndef LBM_ROWPIPE_GROUP_BYTES
#define LBM_ROWPIPE_GROUP_BYTES 0  // target bytes per direction per row group; 0 = per storage type
#endif
#ifndef LBM_ROWPIPE_NS
#define LBM_ROWPIPE_NS 0  // stages; 0 = as many as the shared-memory budget holds
#endif
#ifndef LBM_ROWPIPE_THREADS
#define LBM_ROWPIPE_THREADS 256  // consumer threads per row set at most
#endif
#ifndef LBM_ROWPIPE_CONSUMER_SLEEP
#define LBM_ROWPIPE_CONSUMER_SLEEP 0  // > 0: overrides the consumers' polling sleep (ns) of every shape
#endif
#ifndef LBM_ROWPIPE_PRODUCER_SLEEP
#define LBM_ROWPIPE_PRODUCER_SLEEP 0  // > 0: overrides the producer's polling sleep (ns) of every shape
#endif
#ifndef LBM_ROWPIPE_CWARPS2
#define LBM_ROWPIPE_CWARPS2 0  // D2Q9 consumer warps (0: CR row sets of THREADS), for A/B
#endif
#ifndef LBM_ROWPIPE_CWARPS3
#define LBM_ROWPIPE_CWARPS3 0
#endif
#ifndef LBM_ROWPIPE_CR
#define LBM_ROWPIPE_CR 0  // consumer row sets per CTA; 0 = per lattice and storage type
#endif

// Shape of the row pipeline for lattice L, storage S and shared-memory row pitch PITCH (elements; the
// lattice's nx is at most PITCH).  Measured on B200 (D3Q27 MRT, 256^3): the size of each
// per-direction bulk copy matters most — every copy is a separate DRAM stream, so small copies lose
// row-buffer locality (F16S: 512 B 33 GLUPS, 1 KB 34-42, 2 KB 44, 4 KB 44.5).  FP32 reaches 0.97 of
// the measured copy bandwidth with 2 KB copies (2 rows at 256 wide, 1 KB target), two consumer row
// sets and three stages in one CTA per SM.  16-bit storage: 4 KB copies, two row sets, two stages,
// one CTA per SM (A/B on one B200: 43.8 vs 42.6 GLUPS for MRT 256^3 and 42.0 vs 40.3 for the config-5
// ensemble against 2 KB copies, one row set, two CTAs per SM).
//   THREADS   consumer threads per row set: at most 256 (768-wide F16S BGK: 43.9 vs 39.1 GLUPS
//             against 512)
//   CR        row sets; CONSUMERS = CR * THREADS consumer threads walk a group's cells flattened
//             (staged index b * nx + x), CONSUMERS apart and continued across stages
//   B         rows per group at nx == PITCH; the host may put more rows of a narrower lattice into
//             the same stage (runtime rows per group, at most B * PITCH / nx)
//   NS        stages
//   SEG       rows wider than PITCH: a work item is one row segment of up to SEGW = PITCH - 16 cells
//             (SEGW_RUN by default) staged with HALO = 8 cells on either side, one segment per stage;
//             CR only sets the consumer count, and every stage the CTA's shared memory holds is used
#ifndef LBM_ROWPIPE_PAIR
#define LBM_ROWPIPE_PAIR 1  // 16-bit storage, BGK / two-rate MRT: consumers take two adjacent cells (row_pair)
#endif
#ifndef LBM_ROWPIPE_PAIR_WARPS3
#define LBM_ROWPIPE_PAIR_WARPS3 15  // D3Q27 consumer warps with pairs: 16 warps in all, 4 per sub-partition
#endif
// D3Q27 consumer warps with pairs in the single-lattice row-group kernel (k_step_rows): 11 + the producer
// = 3 warps per sub-partition, up to 168 registers a thread.  A/B on B200 at 1965 MHz, 15 vs 11 warps,
// MLUPS: MRT 256^3 F16S 50.2k vs 51.8k, D3Q27 BGK 256^3 F16S 52.6k vs 54.0k; 9 warps (uneven across
// the sub-partitions) 44.0k, 7 warps 50.2k.  The segmented kernel (4096 x 64 x 64: 45.2k vs 45.1k) and
// the ensemble kernel (54.6k vs 53.7k) keep 15.
#ifndef LBM_ROWPIPE_PAIR_WARPS3_ROWS
#define LBM_ROWPIPE_PAIR_WARPS3_ROWS 11
#endif

// The row kernel's consumers take pairs of adjacent cells (row_pair) for this lattice, storage and collision.
template <class L, class S, int COLL>
constexpr bool kRowPair = LBM_ROWPIPE_PAIR && Codec<S>::kScaled && (COLL == 0 || COLL == 3);

template <class L, class S, int PITCH, bool SEG = false, bool PAIR = false, int PAIRW = LBM_ROWPIPE_PAIR_WARPS3>
struct RowPipeShape {
    static constexpr int HALO = 8;
    static constexpr int SEGW = PITCH - 2 * HALO;
    static constexpr int Q = L::Q;
    static constexpr bool k16 = sizeof(S) == 2;
    static constexpr bool k3 = L::DIM == 3;
    // segment width the segmented kernel runs with: a stage costs about max(floor, its cells' compute),
    // the floor (the stage's refill latency) near 900 D3Q27 cells; A/B, D3Q27 MRT F16S GLUPS at
    // 2048/3072/4096 x 128 x ...: 896 37.7/42.0/44.7, 1008 36.3/40.9/43.5, 832 36.8/40.6/43.7;
    // D2Q9 8192^2 F16S: 1008 134.6, 896 133.4
    static constexpr int SEGW_RUN = k3 ? 896 : SEGW;
    static constexpr int THREADS = PITCH > LBM_ROWPIPE_THREADS ? LBM_ROWPIPE_THREADS : PITCH;
    static constexpr int kRowBytes = PITCH * (int)sizeof(S);
    // the waits for stages: D3Q27 FP32 (memory-bound, often under the power cap) polls unhinted, the
    // producer every 512 ns and the consumers every 256 ns (A/B, MRT 256^3 GLUPS: 28.6 hinted, 29.35
    // with the producer's sleep, 29.6 with both); 16-bit storage and D2Q9 were unchanged or 1 % slower
    // and keep the hinted wait
    static constexpr int PRODUCER_SLEEP = LBM_ROWPIPE_PRODUCER_SLEEP > 0 ? LBM_ROWPIPE_PRODUCER_SLEEP : (k3 && !k16 ? 512 : 0);
    static constexpr int CONSUMER_SLEEP = LBM_ROWPIPE_CONSUMER_SLEEP > 0 ? LBM_ROWPIPE_CONSUMER_SLEEP : (k3 && !k16 ? 256 : 0);
    // D2Q9 (A/B, 1024 x 16384): one row set and 2 KB groups, i.e. more and smaller stages per SM
    // (FP32 85.1 vs 78.3 GLUPS against the D3Q27 shape)
    static constexpr int kGroupBytes =
        LBM_ROWPIPE_GROUP_BYTES > 0 ? LBM_ROWPIPE_GROUP_BYTES : (!k3 ? 2048 : k16 ? 4096 : 1024);
    // segments (SEG) stage one row segment per stage: CR only sets the consumer count (B stays 1)
    static constexpr int CRQ = LBM_ROWPIPE_CR > 0 ? LBM_ROWPIPE_CR : (k3 ? 2 : 1);
    static constexpr int CR0 = CRQ * THREADS > 512 ? 512 / THREADS : CRQ;
    static constexpr int CR = CR0 < 1 ? 1 : CR0;
    // D3Q27 consumer warps (0: CR row sets of THREADS): the register file holds 5 warps of 96
    // registers per SM sub-partition, i.e. up to 19 consumer warps beside the producer
    // with pairs a D3Q27 thread holds two cells' outputs: PAIRW consumer warps + the producer, 15 (every
    // sub-partition at 4 warps, up to 128 registers a thread; 17 warps put 5 on one: 96 at most) or 11
    // (3 warps each, up to 168 registers: the single-lattice row-group kernel)
    static constexpr int CONSUMERS = PAIR && k3                       ? PAIRW * 32
                                     : k3 && LBM_ROWPIPE_CWARPS3 > 0    ? LBM_ROWPIPE_CWARPS3 * 32
                                     : !k3 && LBM_ROWPIPE_CWARPS2 > 0 ? LBM_ROWPIPE_CWARPS2 * 32
                                                                       : CR * THREADS;
    // CTAs per SM: D3Q27 collisions need ~90-120 registers per thread, D2Q9 far fewer; fewer CTAs
    // where two stages of one row would not fit into a CTA's share of shared memory
    static constexpr int limit_of(int ctas) { return (ctas <= 1 ? 224 : ctas == 2 ? 112 : 74) * 1024; }
    static constexpr bool fits(int ctas) { return 2 * (Q * kRowBytes + PITCH) + 128 <= limit_of(ctas); }
    static constexpr int CTAS_R = k3 ? (CONSUMERS <= 256 ? 2 : 1) : (CONSUMERS <= 256 ? 3 : 2);
    static constexpr int CTAS = fits(CTAS_R) ? CTAS_R : (CTAS_R > 2 && fits(2) ? 2 : 1);
    static constexpr int kLimit = limit_of(CTAS);  // smem per CTA
    static constexpr int kBudget = (CTAS == 1 ? (k16 ? 216 : 166) : CTAS == 2 ? (k16 ? 110 : 83) : 72) * 1024;
    static constexpr int B0 = SEG ? 1 : kGroupBytes / kRowBytes;
    static constexpr int B1 = B0 < CR ? CR : B0;
    static constexpr int BMAX0 = (kLimit - 128) / (2 * (Q * kRowBytes + PITCH));
    static constexpr int BMAX = SEG ? 1 : BMAX0 > 8 ? 8 : BMAX0;
    static constexpr int B = B1 > BMAX ? BMAX : (B1 < 1 ? 1 : B1);
    static constexpr int SB = B * PITCH;  // elements per direction in a stage
    static constexpr int STAGE = Q * SB * (int)sizeof(S) + SB;  // populations + mask bytes
    // segments (one short row per stage) take every stage the CTA's shared memory holds: depth in flight
    static constexpr int NSB = (SEG || kBudget > kLimit - 128 ? kLimit - 128 : kBudget) / STAGE;
    static constexpr int NSF = (kLimit - 128) / STAGE;  // stages that fit at all
    static constexpr int NS0 = LBM_ROWPIPE_NS > 0 ? (LBM_ROWPIPE_NS < NSF ? LBM_ROWPIPE_NS : NSF) : NSB;
    static constexpr int NS = NS0 < 2 ? 2 : (NS0 > 8 ? 8 : NS0);
    static_assert(B >= 1, "a row group must fit twice into shared memory");
    static_assert((size_t)NS * STAGE + 128 <= (size_t)kLimit, "row pipeline stages exceed the shared-memory budget");

    static constexpr size_t smem_bytes() { return 128 + (size_t)NS * STAGE; }
    // rows per group for a lattice of width nx (host side): the target copy size, at least one row
    // per row set, within the stage
    static int rows_per_group(int nx) {
        const int cap = B * PITCH / nx;
        int b = kGroupBytes / (nx * (int)sizeof(S));
        if (b < CR) b = CR;
        if (b > cap) b = cap;
        return b < 1 ? 1 : b;
    }
};

// Staged pitch of the segmented kernel: segments of up to 1008 cells plus two 8-cell halos.  (512-cell
// segments in 528-cell stages, 7 of them in flight, were measured: 2048 x 128 x 64 D3Q27 MRT F16S
// 28.7 vs 35.8 GLUPS with 1008-cell segments; short segments mean small bulk copies.)
constexpr int kSegPitch = 1024;

// One cell of the row pipeline: st points at the staged row of direction 0 (direction i at
// st[i * SB]); x, xm, xp are the staged indices of the cell and of its left and right neighbours
// (periodic wrap already applied), mrow[mi] its class, orow[ox] its place in the output row.
template <class L, class S, int SB, int COLL, class P>
__device__ __forceinline__ void row_cell(const P& p, const S* st, const uint8_t* mrow, int x, int xm, int xp,
                                         int mi, int ox, typename Codec<S>::Real sc, typename Codec<S>::Real isc,
                                         S* orow, const Rounding& rnd, uint32_t cell) {
    using R = typename Codec<S>::Real;
    constexpr int Q = L::Q;
    R v[Q];
    static_for<Q>([&](auto I) {
        constexpr int i = I;
        constexpr int cx = L::cx(i);
        const int xs = cx == 1 ? xm : (cx == -1 ? xp : x);
        v[i] = Codec<S>::raw(st[i * SB + xs], R(L::w(i)));
    });
    const int cls = mrow ? (int)mrow[mi] : 0;
    const uint32_t fl = p.cls.flags[cls];
    if (fl & kZeroGradXp) {
        static_for<Q>([&](auto I) {
            constexpr int i = I;
            if constexpr (L::cx(i) == -1) v[i] = Codec<S>::raw(st[i * SB + x], R(L::w(i)));
        });
    }
    R out[Q];
    if constexpr (COLL == 0) {
        bgk_collide<L, false, kExactWeights<S>>(p, cls, fl, v, sc, isc, out);
    } else if constexpr (COLL == 3) {
        mrt2_collide(p, cls, fl, v, sc, isc, out);
    } else {
        R T[27];
        static_for<27>([&](auto I) {
            constexpr int i = I;
            T[L::slot(i)] = v[i];
        });
        mrt_collide<COLL == 1 ? kMrtRef : kMrtGramSchmidt, kExactWeights<S>>(p, cls, fl, T, sc, isc, out);
        if (fl & kBounce) {
            static_for<Q - 1>([&](auto I) {
                constexpr int i = I + 1;
                constexpr int cx = L::cx(i);
                int xs = cx == 1 ? xm : (cx == -1 ? xp : x);
                if (cx == -1 && (fl & kZeroGradXp)) xs = x;
                out[L::opp(i)] = Codec<S>::raw(st[i * SB + xs], R(L::w(i)));
            });
        }
    }
    S* __restrict__ fo = orow + ox;
    if constexpr (Codec<S>::kScaled) {
        store16<L, S>(fo, p.N, out, rnd, cell);
    } else {
        static_for<Q>([&](auto I) {
            constexpr int i = I;
            fo[(long long)i * p.N] = Codec<S>::enc(out[i], R(L::w(i)));
        });
    }
}

// A cell of a whole staged row of width nx (periodic in x); row0: the cell index of the row's x = 0.
template <class L, class S, int SB, int COLL, class P>
__device__ __forceinline__ void row_cell_wrap(const P& p, const S* st, const uint8_t* mrow, int x, int nx,
                                              typename Codec<S>::Real sc, typename Codec<S>::Real isc, S* orow,
                                              const Rounding& rnd, uint32_t row0) {
    const int xm = x == 0 ? nx - 1 : x - 1;
    const int xp = x == nx - 1 ? 0 : x + 1;
    row_cell<L, S, SB, COLL>(p, st, mrow, x, xm, xp, x, x, sc, isc, orow, rnd, row0 + (uint32_t)x);
}

// Two adjacent cells (x even and x + 1) of a staged row, for 16-bit
// storage and a collision that applies its own bounce-back (BGK, two-rate MRT).  Both cells collide as
// row_cell's would; then every direction's two outputs go through one paired conversion and one 32-bit
// store (cell x in the low half, x + 1 in the high half: both cells are adjacent in every plane), which
// halves the stores and their address arithmetic of one-cell threads, and the populations with c_x = 0
// of both cells come in one 32-bit shared load.  Stochastic rounding gives each value the same random
// bits as the one-cell path (pair_rbits), so the kernel families stay bit-identical.
// x: staged index of the first cell (even); xl, xr: staged indices of the pair's left and right neighbours
// (periodic wrap or halo already applied).
template <class L, class S, int SB, int COLL, class P>
__device__ __forceinline__ void row_pair(const P& p, const S* st, const uint8_t* mrow, int x, int xl, int xr,
                                         typename Codec<S>::Real sc, typename Codec<S>::Real isc, S* orow,
                                         const Rounding& rnd, uint32_t cell) {
    using R = typename Codec<S>::Real;
    constexpr int Q = L::Q;
    static_assert(Codec<S>::kScaled && (COLL == 0 || COLL == 3), "pairs: 16-bit storage, BGK or two-rate MRT");
    int clsA = 0, clsB = 0;
    if (mrow) {
        const uint32_t m2 = *reinterpret_cast<const unsigned short*>(mrow + x);
        clsA = (int)(m2 & 0xffu);
        clsB = (int)(m2 >> 8);
    }
    const uint32_t flA = p.cls.flags[clsA], flB = p.cls.flags[clsB];
    // D3Q27: the c_x = 0 populations of both cells come in one 32-bit shared load per direction (x
    // even, every staged row 4-byte aligned); cell x + 1's half waits in mid[] for its collision.
    // (D2Q9 loads them one by one: its ensemble kernel has no registers to spare for mid[].)
    constexpr bool kMid = Q == 27;
    uint32_t mid[Q];
    R outA[Q];
    {
        R v[Q];
        static_for<Q>([&](auto I) {
            constexpr int i = I;
            constexpr int cx = L::cx(i);
            if constexpr (kMid && cx == 0) {
                mid[i] = *reinterpret_cast<const uint32_t*>(st + i * SB + x);
                v[i] = Pair16<S>::lo_f(mid[i]);
            } else {
                v[i] = Codec<S>::raw(st[i * SB + (cx == 1 ? xl : (cx == -1 ? x + 1 : x))], R(L::w(i)));
            }
        });
        if (flA & kZeroGradXp) {
            static_for<Q>([&](auto I) {
                constexpr int i = I;
                if constexpr (L::cx(i) == -1) v[i] = Codec<S>::raw(st[i * SB + x], R(L::w(i)));
            });
        }
        if constexpr (COLL == 0)
            bgk_collide<L, false, false>(p, clsA, flA, v, sc, isc, outA);
        else
            mrt2_collide(p, clsA, flA, v, sc, isc, outA);
    }
    R outB[Q];
    {
        R v[Q];
        static_for<Q>([&](auto I) {
            constexpr int i = I;
            constexpr int cx = L::cx(i);
            if constexpr (kMid && cx == 0)
                v[i] = Pair16<S>::hi_f(mid[i]);
            else
                v[i] = Codec<S>::raw(st[i * SB + (cx == 1 ? x : (cx == -1 ? xr : x + 1))], R(L::w(i)));
        });
        if (flB & kZeroGradXp) {
            static_for<Q>([&](auto I) {
                constexpr int i = I;
                if constexpr (L::cx(i) == -1) v[i] = Codec<S>::raw(st[i * SB + x + 1], R(L::w(i)));
            });
        }
        if constexpr (COLL == 0)
            bgk_collide<L, false, false>(p, clsB, flB, v, sc, isc, outB);
        else
            mrt2_collide(p, clsB, flB, v, sc, isc, outB);
    }
    S* __restrict__ fo = orow + x;
    if (rnd.sr) {
        const PairBits pb{(cell_hash16(cell + 1u, rnd.seed) << 16) | cell_hash16(cell, rnd.seed)};
        static_for<Q>([&](auto I) {
            constexpr int i = I;
            *reinterpret_cast<uint32_t*>(fo + (long long)i * p.N) = Pair16<S>::rs(outB[i], outA[i], pb.template word<i, i>());
        });
    } else {
        static_for<Q>([&](auto I) {
            constexpr int i = I;
            *reinterpret_cast<uint32_t*>(fo + (long long)i * p.N) = Pair16<S>::rn(outB[i], outA[i]);
        });
    }
}

// A pair of a whole staged row of width nx (periodic in x); row0: the cell index of the row's x = 0.
template <class L, class S, int SB, int COLL, class P>
__device__ __forceinline__ void row_pair_wrap(const P& p, const S* st, const uint8_t* mrow, int x, int nx,
                                              typename Codec<S>::Real sc, typename Codec<S>::Real isc, S* orow,
                                              const Rounding& rnd, uint32_t row0) {
    row_pair<L, S, SB, COLL>(p, st, mrow, x, x == 0 ? nx - 1 : x - 1, x + 2 == nx ? 0 : x + 2, sc, isc, orow, rnd,
                             row0 + (uint32_t)x);
}

// COLL: 0 = BGK, 1 = MRT (reference basis), 2 = MRT (Gram-Schmidt), 3 = two-rate MRT (Gram-Schmidt,
// mrt2_collide).  Deviation arithmetic.
// Requires nx <= PITCH with nx * sizeof(S) a multiple of 16 bytes; `rows` = rows per group
// (RowPipeShape::rows_per_group).  Block = CR x THREADS consumer threads + one producer warp.
//   full[s]   tx-count barrier, completed by the bulk loads of stage s
//   empty[s]  every consumer warp has finished reading stage s
// Stage s holds, for direction i, the group's source rows at in[(s * Q + i) * SB + b * nx].
template <class L, class S, int PITCH, int COLL>
using RowShape = RowPipeShape<L, S, PITCH, false, kRowPair<L, S, COLL>, LBM_ROWPIPE_PAIR_WARPS3_ROWS>;

template <class L, class S, int PITCH, int COLL>
__global__ void __launch_bounds__(RowShape<L, S, PITCH, COLL>::CONSUMERS + 32, RowShape<L, S, PITCH, COLL>::CTAS)
    k_step_rows(const __grid_constant__ StepParams<typename Codec<S>::Real> p, int rows, int* __restrict__ err,
                  const WaitLimits wl) {
    using R = typename Codec<S>::Real;
    using Sh = RowShape<L, S, PITCH, COLL>;
    constexpr int Q = L::Q;
    constexpr int NS = Sh::NS;
    constexpr int SB = Sh::SB;
    constexpr int W = Sh::CONSUMERS / 32;  // consumer warps
    static_assert(NS <= 8, "barriers occupy the first 128 bytes");
    constexpr unsigned long long kCy = pack_c<L>(false), kCz = pack_c<L>(true);
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + NS;
    S* in = reinterpret_cast<S*>(smem + 128);                                 // [NS][Q][SB]
    uint8_t* mask_st = reinterpret_cast<uint8_t*>(in + (size_t)NS * Q * SB);  // [NS][SB]
    const bool has_mask = p.mask != nullptr;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    // the launch updates planes plo + k pstride, k < pcnt, of the slowest axis (z for D3Q27, y for
    // D2Q9); a strided D2Q9 launch takes one row per group
    const int ps = p.pstride;
    const int B = L::DIM == 2 && ps > 1 ? 1 : rows;
    const int ystep = L::DIM == 2 && ps > 1 ? ps : B, zstep = L::DIM == 3 ? ps : 1;
    const int ybeg = L::DIM == 2 ? p.plo : 0, yend = L::DIM == 2 ? p.plo + (p.pcnt - 1) * ps + 1 : ny;
    const int zbeg = L::DIM == 3 ? p.plo : 0, zcnt = L::DIM == 3 ? p.pcnt : nz;
    // row groups per z plane (the last one may be short)
    const int gy = L::DIM == 2 ? (p.pcnt + B - 1) / B : (ny + B - 1) / B;
    // item indices in 32 bits (the host keeps the item count below 2^31): a 64-bit division by a
    // runtime divisor is a long software sequence, paid once per stage by every consumer thread
    const unsigned groups = (unsigned)gy * (unsigned)zcnt, ugy = (unsigned)gy;
    const uint32_t row_bytes = (uint32_t)(nx * sizeof(S));
    const unsigned first = blockIdx.x, stride = gridDim.x;
    const S* __restrict__ fin = static_cast<const S*>(p.fin);

    // Issue the bulk loads of group g into stage s (one warp; lanes 0..Q-1 one direction each).
    auto issue = [&](unsigned g, int s) {
        if (g == wl.skip) return;  // test hook: this item's stage is never filled
        const int y0 = ybeg + (int)(g % ugy) * ystep, z = zbeg + (int)(g / ugy) * zstep;
        const int nb = yend - y0 < B ? yend - y0 : B;
        if (lane == 0)
            mbar_arrive_expect_tx(&full[s], (uint32_t)(Q * nb) * row_bytes + (has_mask ? (uint32_t)(nb * nx) : 0u));
        __syncwarp();
        if (lane < Q) {
            const int cy = (int)((kCy >> (2 * lane)) & 3) - 1, cz = (int)((kCz >> (2 * lane)) & 3) - 1;
            int zs = z - cz;
            zs = zs < 0 ? zs + nz : (zs >= nz ? zs - nz : zs);
            int ys = y0 - cy;  // first source row; the nb rows wrap around y at most once
            ys = ys < 0 ? ys + ny : (ys >= ny ? ys - ny : ys);
            const int run = ny - ys < nb ? ny - ys : nb;  // rows before the wrap
            const S* plane = fin + (long long)lane * p.N + (long long)zs * ny * nx;
            S* dst = in + ((long long)s * Q + lane) * SB;
            bulk_load(dst, plane + (long long)ys * nx, (uint32_t)run * row_bytes, &full[s]);
            if (run < nb) bulk_load(dst + run * nx, plane, (uint32_t)(nb - run) * row_bytes, &full[s]);
        } else if (lane == Q && has_mask) {
            bulk_load(mask_st + s * SB, p.mask + ((long long)z * ny + y0) * nx, (uint32_t)(nb * nx), &full[s]);
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
    if (tid >= Sh::CONSUMERS) {  // producer warp
        for (int s = 0; s < NS; ++s)
            if (first + s * stride < groups) issue(first + s * stride, s);
        for (unsigned k = 0; first + (k + NS) * stride < groups; ++k) {
            const int s = (int)(k % NS);
            if (!mbar_wait_sleep<Sh::PRODUCER_SLEEP>(&empty[s], (uint32_t)((k / NS) & 1), wl.limit)) {
                if (lane == 0) atomicExch(err, kRowPipeTimeout);
                return;
            }
            issue(first + (k + NS) * stride, s);
        }
        return;
    }

    R sc, isc;
    storage_scale<S>(p, sc, isc);
    const Rounding rnd = step_rounding<S>(p.tick, p.parity, p.sr, (blockIdx.x | tid) == 0);
    // cells of a group flattened (row b, column x; staged index b * nx + x), CONSUMERS apart and
    // continued across stages: the cells one stage leaves over go to other threads in the next
    // 16-bit BGK / two-rate MRT: threads take pairs of adjacent cells (row_pair), nx / 2 per row
    constexpr bool kPair = kRowPair<L, S, COLL>;
    const int cw = kPair ? nx >> 1 : nx;  // work units per row
    const int cq = Sh::CONSUMERS / cw, cr = Sh::CONSUMERS - cq * cw;
    int b = tid / cw, x = tid - b * cw;
    for (unsigned k = 0; first + k * stride < groups; ++k) {
        const unsigned g = first + k * stride;
        const int s = (int)(k % NS);
        if (!mbar_wait_sleep<Sh::CONSUMER_SLEEP>(&full[s], (uint32_t)((k / NS) & 1), wl.limit)) {
            if (lane == 0) atomicExch(err, kRowPipeTimeout);
            // wait, briefly and bounded, for copies that may still land in this CTA's stages
            for (int j = 1; j < NS && first + (k + j) * stride < groups; ++j)
                if (!mbar_wait_bounded(&full[(k + j) % NS], (uint32_t)(((k + j) / NS) & 1),
                                       wl.limit < (1LL << 28) ? wl.limit : (1LL << 28)))
                    break;
            return;
        }
        const int y0 = ybeg + (int)(g % ugy) * ystep, z = zbeg + (int)(g / ugy) * zstep;
        const int nb = yend - y0 < B ? yend - y0 : B;
        const S* st0 = in + (long long)s * Q * SB;
        const uint8_t* ms0 = has_mask ? mask_st + s * SB : nullptr;
        S* out0 = static_cast<S*>(p.fout) + ((long long)z * ny + y0) * nx;
        const uint32_t cell0 = (uint32_t)(((long long)z * ny + y0) * nx) + p.cell_base;
#pragma unroll 1
        while (b < nb) {
            if constexpr (kPair)
                row_pair_wrap<L, S, SB, COLL>(p, st0 + b * nx, ms0 ? ms0 + b * nx : nullptr, 2 * x, nx, sc, isc,
                                              out0 + (long long)b * nx, rnd, cell0 + (uint32_t)(b * nx));
            else
                row_cell_wrap<L, S, SB, COLL>(p, st0 + b * nx, ms0 ? ms0 + b * nx : nullptr, x, nx, sc, isc,
                                              out0 + (long long)b * nx, rnd, cell0 + (uint32_t)(b * nx));
            x += cr;
            b += cq;
            if (x >= cw) {
                x -= cw;
                ++b;
            }
        }
        b -= nb;
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);  // this warp is done with stage s
    }
}

// Rows wider than 1024 cells: a work item is one row segment [x0, x0 + w), x0 = seg * segw, w = segw
// except for the row's last segment, staged with HALO = 8 cells on either side, so the pull's x
// neighbours of every cell are in shared memory.  segw (host-chosen, seg_width in runtime.cu) is a
// multiple of 16 and at most SEGW = kSegPitch - 16 = 1008.  The halos of the first and the last
// segment of a row are the row's other end (periodic in x) and come by their own copies (16 bytes for
// 16-bit storage, 32 for FP32).  With nx a multiple of 16 every copy starts on a 16-byte boundary and moves a multiple of
// 16 bytes: population rows at x0 - 8, mask rows at x0 for w bytes.  Stage s, direction i, staged
// index j holds x = x0 - HALO + j.
template <class L, class S, int COLL>
using SegShape = RowPipeShape<L, S, kSegPitch, true, kRowPair<L, S, COLL>>;

template <class L, class S, int COLL>
__global__ void __launch_bounds__(SegShape<L, S, COLL>::CONSUMERS + 32, SegShape<L, S, COLL>::CTAS)
    k_step_rows_seg(const __grid_constant__ StepParams<typename Codec<S>::Real> p, int segw, int* __restrict__ err,
                  const WaitLimits wl) {
    using R = typename Codec<S>::Real;
    using Sh = SegShape<L, S, COLL>;
    constexpr int Q = L::Q;
    constexpr int NS = Sh::NS;
    constexpr int SB = Sh::SB;
    constexpr int H = Sh::HALO;
    constexpr int W = Sh::CONSUMERS / 32;
    static_assert(NS <= 8, "barriers occupy the first 128 bytes");
    static_assert(SB >= Sh::SEGW + 2 * H && Sh::SEGW % 16 == 0, "segment and halos must fit the staged row");
    const int SW = segw;
    constexpr unsigned long long kCy = pack_c<L>(false), kCz = pack_c<L>(true);
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + NS;
    S* in = reinterpret_cast<S*>(smem + 128);                                 // [NS][Q][SB]
    uint8_t* mask_st = reinterpret_cast<uint8_t*>(in + (size_t)NS * Q * SB);  // [NS][SB]
    const bool has_mask = p.mask != nullptr;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int nseg = (nx + SW - 1) / SW;
    // the launch updates nrows rows (global row index y + ny z): those of the planes plo + k pstride,
    // k < pcnt, of the slowest axis
    const unsigned row0 = L::DIM == 3 ? (unsigned)p.plo * (unsigned)ny : (unsigned)p.plo;
    const unsigned nrows = L::DIM == 3 ? (unsigned)p.pcnt * (unsigned)ny : (unsigned)p.pcnt;
    const unsigned groups = (unsigned)nseg * nrows;  // < 2^31 (host-checked)
    const unsigned useg = (unsigned)nseg, uny = (unsigned)ny, ups = (unsigned)p.pstride;
    // the q-th row of the launch
    auto row_of = [&](unsigned q) -> unsigned {
        if (ups == 1) return row0 + q;
        if (L::DIM == 2) return row0 + q * ups;
        const unsigned k = q / uny;
        return row0 + (k * ups) * uny + (q - k * uny);
    };
    const unsigned first = blockIdx.x, stride = gridDim.x;
    const S* __restrict__ fin = static_cast<const S*>(p.fin);

    auto issue = [&](unsigned g, int s) {
        if (g == wl.skip) return;  // test hook: this item's stage is never filled
        const unsigned gq = g / useg;
        const unsigned row = row_of(gq);
        const int seg = (int)(g - gq * useg);
        const int z = (int)(row / uny), y = (int)(row - (unsigned)z * uny);
        const int x0 = seg * SW;
        const int w = nx - x0 < SW ? nx - x0 : SW;
        if (lane == 0)
            mbar_arrive_expect_tx(&full[s], (uint32_t)(Q * (w + 2 * H) * sizeof(S)) + (has_mask ? (uint32_t)w : 0u));
        __syncwarp();
        if (lane < Q) {
            const int cy = (int)((kCy >> (2 * lane)) & 3) - 1, cz = (int)((kCz >> (2 * lane)) & 3) - 1;
            int zs = z - cz, ys = y - cy;
            zs = zs < 0 ? zs + nz : (zs >= nz ? zs - nz : zs);
            ys = ys < 0 ? ys + ny : (ys >= ny ? ys - ny : ys);
            const S* src = fin + (long long)lane * p.N + ((long long)zs * ny + ys) * nx;
            S* dst = in + ((long long)s * Q + lane) * SB;
            const bool left = x0 == 0, right = x0 + w == nx;
            if (!left && !right) {
                bulk_load(dst, src + x0 - H, (uint32_t)((w + 2 * H) * sizeof(S)), &full[s]);
            } else if (left) {  // nx > SW: the first segment is never the last
                bulk_load(dst + H, src, (uint32_t)((w + H) * sizeof(S)), &full[s]);
                bulk_load(dst, src + nx - H, (uint32_t)(H * sizeof(S)), &full[s]);
            } else {
                bulk_load(dst, src + x0 - H, (uint32_t)((w + H) * sizeof(S)), &full[s]);
                bulk_load(dst + H + w, src, (uint32_t)(H * sizeof(S)), &full[s]);
            }
        } else if (lane == Q && has_mask) {
            bulk_load(mask_st + s * SB, p.mask + ((long long)z * ny + y) * nx + x0, (uint32_t)w, &full[s]);
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
    if (tid >= Sh::CONSUMERS) {  // producer warp
        for (int s = 0; s < NS; ++s)
            if (first + s * stride < groups) issue(first + s * stride, s);
        for (unsigned k = 0; first + (k + NS) * stride < groups; ++k) {
            const int s = (int)(k % NS);
            if (!mbar_wait_sleep<Sh::PRODUCER_SLEEP>(&empty[s], (uint32_t)((k / NS) & 1), wl.limit)) {
                if (lane == 0) atomicExch(err, kRowPipeTimeout);
                return;
            }
            issue(first + (k + NS) * stride, s);
        }
        return;
    }
    R sc, isc;
    storage_scale<S>(p, sc, isc);
    const Rounding rnd = step_rounding<S>(p.tick, p.parity, p.sr, (blockIdx.x | tid) == 0);
    for (unsigned k = 0; first + k * stride < groups; ++k) {
        const unsigned g = first + k * stride;
        const int s = (int)(k % NS);
        if (!mbar_wait_sleep<Sh::CONSUMER_SLEEP>(&full[s], (uint32_t)((k / NS) & 1), wl.limit)) {
            if (lane == 0) atomicExch(err, kRowPipeTimeout);
            for (int j = 1; j < NS && first + (k + j) * stride < groups; ++j)
                if (!mbar_wait_bounded(&full[(k + j) % NS], (uint32_t)(((k + j) / NS) & 1),
                                       wl.limit < (1LL << 28) ? wl.limit : (1LL << 28)))
                    break;
            return;
        }
        const unsigned gq = g / useg;
        const unsigned row = row_of(gq);
        const int seg = (int)(g - gq * useg);
        const int x0 = seg * SW;
        const int w = nx - x0 < SW ? nx - x0 : SW;
        const S* st = in + (long long)s * Q * SB + H;  // staged index of x0 is 0
        const uint8_t* mrow = has_mask ? mask_st + s * SB : nullptr;
        S* orow = static_cast<S*>(p.fout) + (long long)row * nx + x0;
        const uint32_t cell0 = (uint32_t)((long long)row * nx + x0) + p.cell_base;
        if constexpr (kRowPair<L, S, COLL>) {
            // pairs (xl, xl + 1): w is even, the halos hold both neighbours
#pragma unroll 1
            for (int xl = 2 * tid; xl < w; xl += 2 * Sh::CONSUMERS)
                row_pair<L, S, SB, COLL>(p, st, mrow, xl, xl - 1, xl + 2, sc, isc, orow, rnd, cell0 + (uint32_t)xl);
        } else {
#pragma unroll 1
            for (int xl = tid; xl < w; xl += Sh::CONSUMERS)
                row_cell<L, S, SB, COLL>(p, st, mrow, xl, xl - 1, xl + 1, xl, xl, sc, isc, orow, rnd,
                                         cell0 + (uint32_t)xl);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

}  // namespace lbm
