// cluster.cuh — small D2Q9 BGK lattices resident in the shared memory of one thread-block cluster.
//
// A 128^2 lattice (the reference's lid-driven cavity, cpp/d2q9_bgk_lid.cpp) holds 1.2 MB of FP32
// populations: one step is a few hundred nanoseconds of work, so a launch per step (or a CUDA graph of
// them) is bound by launch and drain latency.  Here one cluster of C CTAs (16 where the device allows
// that size, else 8) keeps both population buffers in its CTAs' shared memory for K steps of one
// launch: CTA r holds `rows` consecutive rows y, and a step is one pass over its cells followed by a
// cluster barrier.  Values that stream across a CTA boundary are stored into the neighbour CTA's shared
// memory (distributed shared memory, generic stores through cluster.map_shared_rank); the barrier
// (release/acquire) makes them visible before the next step reads them.
//
// Slot layout: buffer b, direction i, local row r, column x at ((b * Q + i) * rows + r) * nx + x.  Slot
// (i, y, x) of the current buffer holds f_i(x, y - c_iy) in stored words: the y part of the streaming
// happens when a value is written (to row y + c_iy), the x part when it is read (column x - c_ix), so a
// cell reads only its own CTA's memory and writes at most one row across.
//
// The cell update is the plain and row kernels' (bgk_collide, the codecs, encode16 with the same random
// words for stochastic rounding, step t's seed from the device step counter), so the results are
// bit-identical to theirs.  The launch reads buffer `parity`, leaves the state after K steps in the
// other buffer and the state after K - 1 steps in buffer `parity` (as K single steps would), and
// advances the step counter by K.
#pragma once

#include <cooperative_groups.h>

#include "kernels.cuh"

namespace lbm {

constexpr int kClusterThreads = 1024;
constexpr int kClusterMaxSteps = 4096;  // steps per launch (the host splits longer runs)

template <class S>
__global__ void __launch_bounds__(kClusterThreads, 1)
    k_step_cluster(const __grid_constant__ StepParams<typename Codec<S>::Real> p, int rows, int ksteps, int write_prev) {
    namespace cg = cooperative_groups;
    using L = D2Q9;
    using R = typename Codec<S>::Real;
    constexpr int Q = L::Q;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(128) unsigned char smem[];
    const int nx = p.nx, ny = p.ny;
    const int rank = (int)cluster.block_rank();
    const int y0 = rank * rows;
    const int nr = max(0, min(rows, ny - y0));  // rows of this CTA (the last CTAs may hold fewer or none)
    const int plane = rows * nx;                 // slots of one direction in one buffer
    S* buf = reinterpret_cast<S*>(smem);
    uint8_t* cls_s = reinterpret_cast<uint8_t*>(buf + 2 * Q * plane);
    const bool has_mask = p.mask != nullptr;
    const int cells = nr * nx;
    const int tid = (int)threadIdx.x;
    const int T = (int)blockDim.x;
    // the CTA and local row of global rows y0 - 1 and y0 + nr (periodic in y)
    const int last_rank = (ny - 1) / rows, last_row = ny - 1 - last_rank * rows;
    const int dn_rank = rank == 0 ? last_rank : rank - 1, dn_row = rank == 0 ? last_row : rows - 1;
    const int up_rank = y0 + nr >= ny ? 0 : rank + 1;

    // load: slot(0, i, y, x) = f_i(x, y - c_iy)
    {
        const S* __restrict__ fin = static_cast<const S*>(p.fin);
        for (int k = tid; k < cells; k += T) {
            const int r = k / nx, x = k - r * nx, y = y0 + r;
            static_for<Q>([&](auto I) {
                constexpr int i = I;
                constexpr int cy = L::cy(i);
                int ys = y - cy;
                ys = ys < 0 ? ys + ny : (ys >= ny ? ys - ny : ys);
                buf[i * plane + k] = fin[(long long)i * p.N + (long long)ys * nx + x];
            });
            cls_s[k] = has_mask ? p.mask[(long long)y * nx + x] : (uint8_t)0;
        }
    }
    const unsigned t0 = p.tick[p.parity];
    R sc, isc;
    storage_scale<S>(p, sc, isc);
    // this thread's first cell (row, column) and the stride T in rows and columns
    const int dr = T / nx, dx = T - dr * nx;
    const int r0 = tid / nx, x0 = tid - r0 * nx;
    cluster.sync();

    int cur = 0;
    for (int step = 0; step < ksteps; ++step) {
        Rounding rnd{0u, false};
        if constexpr (Codec<S>::kScaled) {
            if (p.sr) rnd = Rounding{seed_of_step(t0 + (unsigned)step), true};
        }
        const S* cb = buf + cur * Q * plane;
        S* nb = buf + (cur ^ 1) * Q * plane;
        int r = r0, x = x0;
#pragma unroll 1
        for (int k = tid; k < cells; k += T) {
            const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
            const S* st = cb + r * nx;
            R v[Q];
            static_for<Q>([&](auto I) {
                constexpr int i = I;
                constexpr int cx = L::cx(i);
                v[i] = Codec<S>::raw(st[i * plane + (cx == 1 ? xm : (cx == -1 ? xp : x))], R(L::w(i)));
            });
            const int cls = (int)cls_s[k];
            const uint32_t fl = p.cls.flags[cls];
            if (fl & kZeroGradXp) {
                static_for<Q>([&](auto I) {
                    constexpr int i = I;
                    if constexpr (L::cx(i) == -1) v[i] = Codec<S>::raw(st[i * plane + x], R(L::w(i)));
                });
            }
            R out[Q];
            bgk_collide<L, false, kExactWeights<S>>(p, cls, fl, v, sc, isc, out);
            // direction i goes to slot(next, i, y + c_iy, x): this CTA's unless the row is a neighbour's
            const bool up_here = r + 1 < nr, dn_here = r > 0;
            auto put = [&](auto I, S w) {
                constexpr int i = decltype(I)::value;
                constexpr int cy = L::cy(i);
                if constexpr (cy == 0) {
                    nb[i * plane + k] = w;
                } else if constexpr (cy == 1) {
                    if (up_here)
                        nb[i * plane + k + nx] = w;
                    else
                        *cluster.map_shared_rank(nb + i * plane + x, up_rank) = w;
                } else {
                    if (dn_here)
                        nb[i * plane + k - nx] = w;
                    else
                        *cluster.map_shared_rank(nb + i * plane + dn_row * nx + x, dn_rank) = w;
                }
            };
            const uint32_t cell = (uint32_t)((long long)(y0 + r) * nx + x) + p.cell_base;
            if constexpr (Codec<S>::kScaled) {
                encode16<L, S>(out, rnd, cell, put);
            } else {
                static_for<Q>([&](auto I) {
                    constexpr int i = I;
                    put(I, Codec<S>::enc(out[i], R(L::w(i))));
                });
            }
            r += dr;
            x += dx;
            if (x >= nx) {
                x -= nx;
                ++r;
            }
        }
        cluster.sync();
        cur ^= 1;
    }

    // store: f_i(x, y - c_iy) = slot(cur, i, y, x), this CTA's slots only.  The state after K steps goes
    // to the output buffer and the state after K - 1 steps (the other shared buffer) to the input
    // buffer, which every CTA finished reading before the first barrier: the pair is what K single
    // steps leave behind, so what reads the previous step's populations (lbm_get_macros pulls them)
    // sees the same.  (write_prev = 0, for the autotuner's trial launches, leaves the input alone.)
    {
        S* __restrict__ fout = static_cast<S*>(p.fout);
        S* __restrict__ fprev = const_cast<S*>(static_cast<const S*>(p.fin));
        const S* cb = buf + cur * Q * plane;
        const S* pb = buf + (cur ^ 1) * Q * plane;
        for (int k = tid; k < cells; k += T) {
            const int r = k / nx, x = k - r * nx, y = y0 + r;
            static_for<Q>([&](auto I) {
                constexpr int i = I;
                constexpr int cy = L::cy(i);
                int ys = y - cy;
                ys = ys < 0 ? ys + ny : (ys >= ny ? ys - ny : ys);
                const long long g = (long long)i * p.N + (long long)ys * nx + x;
                fout[g] = cb[i * plane + k];
                if (write_prev) fprev[g] = pb[i * plane + k];
            });
        }
    }
    // every CTA read tick[parity] before the first cluster barrier
    if (rank == 0 && tid == 0) p.tick[p.parity ^ 1] = t0 + (unsigned)ksteps;
}

}  // namespace lbm
