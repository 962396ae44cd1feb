// rowpipe.cuh — D3Q27 step kernel with bulk-copy (TMA) staging of whole lattice rows.
//
// A CTA of nx threads owns one lattice row (y, z) at a time and walks a strided list of rows.  For
// each row it needs, per direction i, the full source row (y - cy_i, z - cz_i) of plane i; the x
// shift of the pull (af::shift semantics, periodic in x) then becomes an index offset inside that
// staged row.  Warp 0 issues one `cp.async.bulk` global->shared copy per direction into a ring of NS
// shared-memory stages (completion counted in bytes on one mbarrier per stage), so NS rows of loads
// are in flight per CTA without holding registers.  The collision reads the staged populations with
// immediate-offset shared loads, writes its results into one of two output stages, and warp 0 sends
// each output row back with `cp.async.bulk` shared->global copies.  Compared with the one-cell-per-
// thread kernel this removes the per-population 64-bit address arithmetic (the issue bottleneck of
// 16-bit storage) and decouples memory latency from occupancy.
//
// Every wait on an mbarrier is bounded (about two seconds); a CTA that times out records
// kRowPipeTimeout in *err, drains the copies it issued with bounded waits and returns.
// No multicast: every copy moves data of this GPU's own memory into this CTA's shared memory.
#pragma once

#include <cstdint>

#include "kernels.cuh"

namespace lbm {

constexpr int kRowPipeTimeout = 1;

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
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait: false after ~2^32 clocks (about two seconds) without completion.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > (1LL << 32)) return false;
    return true;
}
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst_smem)),
                 "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void bulk_store(void* dst_gmem, const void* src_smem, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem), "r"(smem_addr(src_smem)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// (cy, cz) of direction i packed two bits each, so a lane can look its own up at run time.
template <class L>
constexpr unsigned long long pack_c(bool z) {
    unsigned long long v = 0;
    for (int i = 0; i < L::Q; ++i) v |= (unsigned long long)((z ? L::cz(i) : L::cy(i)) + 1) << (2 * i);
    return v;
}

// Stage counts: input stages NS (loads in flight per CTA) and two output stages.
template <class S>
struct RowPipeStages {
    static constexpr int NS = sizeof(S) <= 2 ? 4 : 2;
    static constexpr int NO = 2;
};

template <class L, class S, int PITCH>
constexpr size_t rowpipe_smem_bytes() {
    return 128 + (size_t)(RowPipeStages<S>::NS + RowPipeStages<S>::NO) * L::Q * PITCH * sizeof(S);
}

// COLL: 0 = BGK, 1 = MRT (reference basis), 2 = MRT (Gram-Schmidt).  Deviation arithmetic.
// Requires nx == PITCH (one thread per cell of the row).
template <class L, class S, int PITCH, int COLL>
__global__ void __launch_bounds__(PITCH, PITCH <= 256 ? 2 : 1)
    k_step_rows(StepParams<typename Codec<S>::Real> p, int* __restrict__ err) {
    using R = typename Codec<S>::Real;
    constexpr int Q = L::Q;
    constexpr int NS = RowPipeStages<S>::NS;
    constexpr int NO = RowPipeStages<S>::NO;
    constexpr unsigned long long kCy = pack_c<L>(false), kCz = pack_c<L>(true);
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    S* in = reinterpret_cast<S*>(smem + 128);
    S* outs = in + NS * Q * PITCH;

    const int x = threadIdx.x;
    const int lane = x & 31, warp = x >> 5;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const long long rows = (long long)ny * nz;
    const uint32_t row_bytes = (uint32_t)(nx * sizeof(S));
    const S* __restrict__ fin = static_cast<const S*>(p.fin);
    S* __restrict__ fout = static_cast<S*>(p.fout);

    if (x == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&full[s], 1);
        mbar_init_fence();
    }
    __syncthreads();

    // warp 0: stage the Q source rows of destination row r into input stage s
    auto issue = [&](long long r, int s) {
        const int y = (int)(r % ny), z = (int)(r / ny);
        if (lane == 0) mbar_arrive_expect_tx(&full[s], (uint32_t)Q * row_bytes);
        __syncwarp();
        if (lane < Q) {
            const int cy = (int)((kCy >> (2 * lane)) & 3) - 1, cz = (int)((kCz >> (2 * lane)) & 3) - 1;
            int ys = y - cy, zs = z - cz;
            ys = ys < 0 ? ys + ny : (ys >= ny ? ys - ny : ys);
            zs = zs < 0 ? zs + nz : (zs >= nz ? zs - nz : zs);
            const S* src = fin + (long long)lane * p.N + ((long long)zs * ny + ys) * nx;
            bulk_load(in + (lane * PITCH) + (long long)s * Q * PITCH, src, row_bytes, &full[s]);
        }
    };

    const long long first = blockIdx.x, stride = gridDim.x;
    if (warp == 0)
        for (int s = 0; s < NS; ++s)
            if (first + s * stride < rows) issue(first + s * stride, s);

    const int xm = x == 0 ? nx - 1 : x - 1;
    const int xp = x == nx - 1 ? 0 : x + 1;
    long long k = 0;
    bool dead = false;
    for (;; ++k) {
        const long long r = first + k * stride;
        if (r >= rows) break;
        const int s = (int)(k % NS), o = (int)(k % NO);
        const uint32_t parity = (uint32_t)((k / NS) & 1);
        const bool ok = mbar_wait_bounded(&full[s], parity);
        const S* st = in + (long long)s * Q * PITCH;

        // gather the streamed deviations from the staged rows
        R v[Q];
        static_for<Q>([&](auto I) {
            constexpr int i = I;
            constexpr int cx = L::cx(i);
            const int xs = cx == 1 ? xm : (cx == -1 ? xp : x);
            v[i] = Codec<S>::dev(st[i * PITCH + xs], R(L::w(i)), R(p.inv_scale));
        });
        const long long c = r * nx + x;
        int cls;
        uint32_t fl;
        cell_class(p.mask, p.cls, c, cls, fl);
        if (fl & kZeroGradXp) {
            static_for<Q>([&](auto I) {
                constexpr int i = I;
                if constexpr (L::cx(i) == -1) v[i] = Codec<S>::dev(st[i * PITCH + x], R(L::w(i)), R(p.inv_scale));
            });
        }
        R out[Q];
        if constexpr (COLL == 0) {
            bgk_collide<L, false>(p, cls, fl, v, out);
        } else {
            R T[27];
            static_for<27>([&](auto I) {
                constexpr int i = I;
                T[L::slot(i)] = v[i];
            });
            mrt_collide<COLL == 1 ? kMrtRef : kMrtGramSchmidt>(p, cls, fl, T, out);
            if (fl & kBounce) {
                static_for<Q - 1>([&](auto I) {
                    constexpr int i = I + 1;
                    constexpr int cx = L::cx(i);
                    int xs = cx == 1 ? xm : (cx == -1 ? xp : x);
                    if (cx == -1 && (fl & kZeroGradXp)) xs = x;
                    out[L::opp(i)] = Codec<S>::dev(st[i * PITCH + xs], R(L::w(i)), R(p.inv_scale));
                });
            }
        }

        // (B) every thread is done with input stage s; warp 0's wait on output stage o is visible
        if (__syncthreads_or(!ok)) {
            dead = true;
            break;
        }
        if (warp == 0 && r + NS * stride < rows) issue(r + NS * stride, s);

        S* so = outs + (long long)o * Q * PITCH;
        static_for<Q>([&](auto I) {
            constexpr int i = I;
            Codec<S>::store_dev(so + i * PITCH + x, out[i], R(L::w(i)), R(p.scale));
        });
        fence_proxy_async_smem();
        __syncthreads();  // (C) output stage o complete
        if (warp == 0) {
            if (lane < Q) bulk_store(fout + (long long)lane * p.N + r * nx, so + lane * PITCH, row_bytes);
            bulk_commit();
            bulk_wait_read_1();  // output stage o^1 is free for the next row (NO == 2)
        }
    }
    if (dead) {
        if (x == 0) atomicExch(err, kRowPipeTimeout);
        // drain the loads this CTA issued (iterations k .. k+NS-1) with bounded waits
        for (int j = 0; j < NS; ++j) {
            const long long kk = k + j;
            if (first + kk * stride >= rows) break;
            if (!mbar_wait_bounded(&full[kk % NS], (uint32_t)((kk / NS) & 1))) break;
        }
    }
    if (warp == 0) bulk_wait_all();
}

}  // namespace lbm
