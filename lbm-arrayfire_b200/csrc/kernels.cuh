// kernels.cuh — the fused per-time-step kernels.
//
// One thread owns one cell.  Per step it
//   1. pulls Q populations from the previous buffer (periodic wrap: af::shift semantics,
//      cpp/d2q9_bgk_lid.cpp:18-28,124) — Q coalesced loads along x, one HBM read each;
//   2. forms rho and u (cpp/d2q9_bgk_lid.cpp:131-138), applies its cell class (the reference's
//      boundary overwrites, :141-146) and collides (BGK :149-153 / MRT / Shan-Chen);
//   3. applies full-way bounce-back for solid classes (:126,155) and writes Q populations.
// HBM traffic per cell and step: Q loads + Q stores of the storage type (+1 mask byte).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "arith.cuh"
#include "codec.cuh"
#include "lattice.cuh"
#include "mrt.cuh"

namespace lbm {

constexpr uint32_t kBounce = 0x01u, kSetRho = 0x02u, kSetUx = 0x04u, kSetUy = 0x08u, kSetUz = 0x10u,
                   kEquilibrium = 0x20u, kZeroGradXp = 0x40u, kZouHeVelXm = 0x80u, kZouHeRhoXp = 0x100u;
constexpr int kMaxClasses = 16;

template <class R>
struct ClassTable {
    uint32_t flags[kMaxClasses];
    R rho[kMaxClasses], ux[kMaxClasses], uy[kMaxClasses], uz[kMaxClasses];
};

template <class R>
struct StepParams {
    const void* fin;
    void* fout;
    const uint8_t* mask;  // nullptr: every cell is class 0
    int nx, ny, nz;
    long long N;          // cells
    R omega, one_m_omega;
    R scale, inv_scale;   // 16-bit storage codec
    R G;                  // Shan-Chen strength
    R* psi;               // Shan-Chen psi field (N)
    R* rho_out;           // macro kernel outputs
    R* u_out;
    unsigned* tick;       // the step counter pair of the rounding (see step_rounding)
    int parity;           // the input buffer of this launch: it reads tick[parity], writes tick[parity ^ 1]
    int sr;               // 16-bit storage: 1 stochastic rounding, 0 round to nearest
    uint32_t cell_base;   // index of cell 0 in the lattice this one is part of (the rounding's hash input)
    int plo, pcnt, pstride;  // the step kernels update planes plo + k pstride, k < pcnt, of the slowest axis
                             // (z for D3Q27, y for D2Q9; lbm_step_planes); 0, every plane and 1 for a
                             // whole step
    ClassTable<R> cls;
    MrtCoef<R> mrt;
    Mrt2Coef<R> mrt2;
};

// Row base offsets of the 3 (D2Q9) or 9 (D3Q27) neighbour rows of (y, z), wrap included, as cell
// indices of type I: long long, or uint32_t for lattices whose Q N populations all have 32-bit indices
// (one 32-bit add and one widening multiply-add per population address instead of 64-bit arithmetic).
template <class L, class I = long long>
struct RowsT {
    using Idx = I;
    I base[3][3];  // [dy+1][dz+1]
    __device__ __forceinline__ RowsT(int y, int z, int nx, int ny, int nz) {
        const int ys[3] = {y == 0 ? ny - 1 : y - 1, y, y == ny - 1 ? 0 : y + 1};
        const int zs[3] = {z == 0 ? nz - 1 : z - 1, z, z == nz - 1 ? 0 : z + 1};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
                base[a][b] = ((I)zs[b] * (I)ny + (I)ys[a]) * (I)nx;
    }
    // source row of direction (cy, cz): pull from y - cy, z - cz
    __device__ __forceinline__ I src(int cy, int cz) const { return base[1 - cy][1 - cz]; }
};
template <class L>
using Rows = RowsT<L, long long>;

// Pull gather of one cell.  ABS = false: deviations in storage units (Codec::raw: f_i - w_i, times
// the storage scale for the 16-bit codecs); ABS = true: the populations themselves.  x-wrap per thread; the source x of c_x = +1 is x-1 and of c_x = -1 is x+1
// (af::shift: out[x] = in[x - c]).
template <class L, class S, bool ABS, class P, class R, class Ix>
__device__ __forceinline__ void pull(const S* __restrict__ fin, const P& p, const RowsT<L, Ix>& rows, int x,
                                     R (&d)[L::Q]) {
    const int xm = x == 0 ? p.nx - 1 : x - 1;
    const int xp = x == p.nx - 1 ? 0 : x + 1;
    static_for<L::Q>([&](auto I) {
        constexpr int i = I;
        constexpr int cx = L::cx(i), cy = L::cy(i), cz = L::cz(i);
        const int xs = cx == 1 ? xm : (cx == -1 ? xp : x);
        const Ix idx = (Ix)i * (Ix)p.N + rows.src(cy, cz) + (Ix)xs;
        if constexpr (ABS)
            d[i] = Codec<S>::load(fin + idx, R(L::w(i)), R(p.inv_scale));
        else
            d[i] = Codec<S>::raw(__ldg(fin + idx), R(L::w(i)));
    });
}

// Zero-gradient outlet: populations arriving from +x are taken from cell x-1's streamed state,
// i.e. F_i(x - 1 - c_i) = F_i(x, y - cy, z - cz) for c_x = -1.
template <class L, class S, bool ABS, class P, class R, class Ix>
__device__ __forceinline__ void pull_zerograd(const S* __restrict__ fin, const P& p, const RowsT<L, Ix>& rows, int x,
                                              R (&d)[L::Q]) {
    static_for<L::Q>([&](auto I) {
        constexpr int i = I;
        if constexpr (L::cx(i) == -1) {
            const Ix idx = (Ix)i * (Ix)p.N + rows.src(L::cy(i), L::cz(i)) + (Ix)x;
            if constexpr (ABS)
                d[i] = Codec<S>::load(fin + idx, R(L::w(i)), R(p.inv_scale));
            else
                d[i] = Codec<S>::raw(__ldg(fin + idx), R(L::w(i)));
        }
    });
}

// Moments (cpp/d2q9_bgk_lid.cpp:131-138): rho = sum f, j = sum c f, u = j / rho.  On deviations
// sum d = rho - 1 and sum c d = j (sum c w = 0).  Both rho and drho = rho - 1 are returned.
// isc: 1 / storage scale of raw deviations (a power of two, so the rescaled sums are exact).
// The sums start from their first term (not from zero): no 0 + x whose folding could depend on the
// compiler's context.
template <class L, int AXIS>
LBM_HD constexpr int first_moving(int) {
    for (int i = 0; i < L::Q; ++i)
        if ((AXIS == 0 ? L::cx(i) : AXIS == 1 ? L::cy(i) : L::cz(i)) != 0) return i;
    return L::Q;
}
template <class L, int AXIS, class R>
__device__ __forceinline__ R momentum_sum(const R (&v)[L::Q]) {
    constexpr int f = first_moving<L, AXIS>(0);
    if constexpr (f == L::Q) {
        return R(0);
    } else {
        constexpr int cf = AXIS == 0 ? L::cx(f) : AXIS == 1 ? L::cy(f) : L::cz(f);
        R j = cf == 1 ? v[f] : -v[f];
        static_for<L::Q>([&](auto I) {
            constexpr int i = I;
            constexpr int c = AXIS == 0 ? L::cx(i) : AXIS == 1 ? L::cy(i) : L::cz(i);
            if constexpr (i > f && c == 1) j = j + v[i];
            if constexpr (i > f && c == -1) j = j - v[i];
        });
        return j;
    }
}

template <class L, bool ABS, class R>
__device__ __forceinline__ void moments(const R (&v)[L::Q], R sc, R isc, R& rho, R& drho, R& ux, R& uy, R& uz) {
    R r = v[0];
    static_for<L::Q - 1>([&](auto I) { r = r + v[I + 1]; });
    R jx = momentum_sum<L, 0>(v), jy = momentum_sum<L, 1>(v), jz = momentum_sum<L, 2>(v);
    if constexpr (ABS) {
        // the reference's arithmetic: u = j / rho
        rho = r;
        drho = r - R(1);
        ux = jx / rho;
        uy = jy / rho;
        uz = L::DIM == 3 ? jz / rho : R(0);
    } else {
        // One division whose numerator is the (power-of-two) storage scale, then a product and one
        // correction step per component (Markstein: q = j/rho, e = j - q rho exactly by fma, q + e/rho),
        // which returns the correctly rounded quotient in all but rare cases.  A plain j / rho per
        // component took the division's slow path for every zero or tiny momentum (cells at rest).
        drho = r * isc;
        rho = R(1) + drho;
        const R inv = isc / rho;  // (1 / rho) / scale
        const R rinv = inv * sc;  // 1 / rho: exact rescale by a power of two
        auto quot = [&](R j) {
            const R q = j * inv;
            const R e = mad(-q, rho, j * isc);
            return mad(e, rinv, q);
        };
        ux = quot(jx);
        uy = quot(jy);
        uz = L::DIM == 3 ? quot(jz) : R(0);
    }
}

// The reference's boundary overwrites of DENSITY/UX/UY/UZ (cpp/d2q9_bgk_lid.cpp:141-146).
template <class T, class R>
__device__ __forceinline__ void apply_class(const ClassTable<T>& ct, int cls, uint32_t fl, R& rho, R& drho,
                                            R& ux, R& uy, R& uz, int dim) {
    if (fl & kSetRho) {
        rho = R(ct.rho[cls]);
        drho = rho - R(1);
    }
    if (fl & kSetUx) ux = R(ct.ux[cls]);
    if (fl & kSetUy) uy = R(ct.uy[cls]);
    if ((fl & kSetUz) && dim == 3) uz = R(ct.uz[cls]);
}

// Equilibrium of direction I in the reference's form (cpp/d2q9_bgk_lid.cpp:151), absolute values:
//   feq_i = w_i rho (1 + 3 eu + 4.5 eu^2 - 1.5 u^2),   usq15 = 1.5 |u|^2
template <class L, int I, class R>
__device__ __forceinline__ R feq_abs_i(R rho, R usq15, R ux, R uy, R uz) {
    constexpr int cx = L::cx(I), cy = L::cy(I), cz = L::cz(I);
    R eu = R(0);
    if constexpr (cx == 1) eu = eu + ux;
    if constexpr (cx == -1) eu = eu - ux;
    if constexpr (cy == 1) eu = eu + uy;
    if constexpr (cy == -1) eu = eu - uy;
    if constexpr (cz == 1) eu = eu + uz;
    if constexpr (cz == -1) eu = eu - uz;
    return (R(L::w(I)) * rho) * ((R(1) - usq15) + eu * (R(3) + R(4.5) * eu));
}

// Deviation equilibrium feq_i - w_i = w_i ((rho - 1) + rho (4.5 eu^2 - 1.5 u^2)) +- w_i rho 3 eu,
// evaluated once per pair of opposite directions: the symmetric part is shared and the
// momentum-carrying part is exactly antisymmetric.  sc: storage scale of the result (power of two).
// Every multiply-add is explicit (mad): the rounding is fixed by the source (arith.cuh).
//
// EXACTW (FP32 storage): each weight is applied as a sum of two floats, w = hi + lo (hi the float
// nearest w, lo the float nearest the remainder), as mad(hi, x, lo * x).  No float equals 1/9, 2/27,
// ...: with the nearest floats alone the weights' moments miss their exact values by ~1e-8 (e.g.
// 3 sum_i w_i c_ix^2 = 9 fl(1/9) = 1 + 7.5e-9 for D2Q9), so every collision scales the momentum by
// 1 + omega * 7.5e-9 while the mass (rho - 1 = sum of deviations) stays put.  That systematic error
// drifts u linearly (the 128^2 lid cavity: rel. L2 1.8e-5 from the FP64 run after 10,000 steps).  The
// reference's own FP32 arithmetic scales mass and momentum alike (its density drifts instead, 8e-5
// there).  The two-float weights make the moments exact to ~1e-15; the rounding left is unbiased.
// 16-bit storage rounds each population far more coarsely than that bias, FP64 weights are exact to
// 1e-17: both keep the single multiply.
template <class L, bool EXACTW, class R>
__device__ __forceinline__ void equilibrium_dev(R rho, R drho, R ux, R uy, R uz, R sc, R (&fe)[L::Q]) {
    const R nusq15 = R(-1.5) * mad(uz, uz, mad(uy, uy, ux * ux));
    const R rho3 = R(3) * rho;
    const R rho45 = R(4.5) * rho;
    const R base = mad(rho, nusq15, drho);
    // w_i (times sc) applied to x: one multiply, or hi + lo by one multiply-add (EXACTW)
    auto wmul = [&](auto I, R x) {
        constexpr int i = decltype(I)::value;
        if constexpr (EXACTW) {
            constexpr R hi = R(L::w(i));
            constexpr R lo = R(L::w(i) - double(hi));
            return mad(hi * sc, x, (lo * sc) * x);
        } else {
            return (R(L::w(i)) * sc) * x;
        }
    };
    static_for<L::Q>([&](auto I) {
        constexpr int i = I;
        constexpr int o = L::opp(i);
        if constexpr (i == 0) {
            fe[0] = wmul(I, base);
        } else if constexpr (i < o) {
            constexpr int cx = L::cx(i), cy = L::cy(i), cz = L::cz(i);
            // c.u from its first nonzero term (no 0 + x)
            R eu = cx != 0 ? (cx == 1 ? ux : -ux) : (cy != 0 ? (cy == 1 ? uy : -uy) : (cz == 1 ? uz : -uz));
            if constexpr (cx != 0 && cy == 1) eu = eu + uy;
            if constexpr (cx != 0 && cy == -1) eu = eu - uy;
            if constexpr ((cx != 0 || cy != 0) && cz == 1) eu = eu + uz;
            if constexpr ((cx != 0 || cy != 0) && cz == -1) eu = eu - uz;
            const R sym = wmul(I, mad(rho45, eu * eu, base));
            const R anti = wmul(I, rho3 * eu);
            fe[i] = sym + anti;
            fe[o] = sym - anti;
        }
    });
}

template <class L, bool ABS, bool EXACTW, class R>
__device__ __forceinline__ void equilibrium_v(R rho, R drho, R ux, R uy, R uz, R sc, R (&feq)[L::Q]) {
    if constexpr (ABS) {
        const R usq15 = R(1.5) * (ux * ux + uy * uy + uz * uz);
        static_for<L::Q>([&](auto I) {
            constexpr int i = I;
            feq[i] = feq_abs_i<L, i>(rho, usq15, ux, uy, uz);
        });
    } else {
        equilibrium_dev<L, EXACTW, R>(rho, drho, ux, uy, uz, sc, feq);
    }
}

// Storage types whose equilibrium applies the weights as two floats (equilibrium_dev).
template <class S>
constexpr bool kExactWeights = std::is_same_v<S, float>;

// feq_i = w_i rho (1 + 3 eu + 4.5 eu^2 - 1.5 u^2) (absolute values, used to initialise)
template <class L, class R>
__device__ __forceinline__ void equilibrium(R rho, R ux, R uy, R uz, R (&feq)[L::Q]) {
    R dev[L::Q];
    equilibrium_dev<L, false, R>(rho, rho - R(1), ux, uy, uz, R(1), dev);
    static_for<L::Q>([&](auto I) {
        constexpr int i = I;
        feq[i] = R(L::w(i)) + dev[i];
    });
}

// How a launch rounds 16-bit stores: to nearest, or stochastically (sr) with random words hashed from
// the cell index and the step.  The step index lives on the device as a pair tick[2]: a launch reading
// buffer `parity` takes t = tick[parity] and one designated thread writes tick[parity ^ 1] = t + 1,
// which only the next launch reads.  Steps replayed from a CUDA graph, single launches, the autotuner's
// trial launches (they rewrite the same t + 1) and every kernel family therefore round with the same
// random words for the same step and cell: results stay bit-identical across them.
struct Rounding {
    uint32_t seed;
    bool sr;
};
// The seed of step t.
__device__ __forceinline__ uint32_t seed_of_step(unsigned t) { return mix32(t * 0x9e3779b9u + 0x7f4a7c15u); }
// The step's seed for a launch reading buffer `parity` (advances the counter pair, see above).
__device__ __forceinline__ uint32_t step_seed(unsigned* tick, int parity, bool designated) {
    const unsigned t = tick[parity];
    if (designated) tick[parity ^ 1] = t + 1u;
    return seed_of_step(t);
}
template <class S>
__device__ __forceinline__ Rounding step_rounding(unsigned* tick, int parity, int sr, bool designated) {
    if constexpr (!Codec<S>::kScaled) {
        return Rounding{0u, false};
    } else {
        if (!sr) return Rounding{0u, false};
        return Rounding{step_seed(tick, parity, designated), true};
    }
}

// Random bits of the stochastic rounding.  Every stored value (cell c, direction i) has its own 16-bit
// word g(c, i) = h(c) ^ salt(i), with h(c) a hash of the cell index and the step's seed; a paired
// conversion takes the upper value's word in bits 31..16 of its random operand and the lower value's in
// bits 15..0 (the layout cvt.rs uses, measured on B200).  A value therefore rounds with the same bits
// whichever value it is paired with: two directions of one cell (store16) or one direction of two
// adjacent cells (row_pair) -- the kernel families stay bit-identical.
__host__ __device__ constexpr uint32_t rs_salt(int i) { return ((0x9e3779b9u * (uint32_t)(i + 1)) >> 16) & 0xffffu; }
__device__ __forceinline__ uint32_t cell_hash16(uint32_t cell, uint32_t seed) {
    uint32_t h = (cell ^ seed) * 0x9e3779b1u;
    return (h ^ (h >> 16)) & 0xffffu;
}
// The random operands of one thread's paired conversions: base = (upper value's cell hash << 16) | lower's.
struct PairBits {
    uint32_t base;
    // directions i (upper) and j (lower)
    template <int I, int J>
    __device__ __forceinline__ uint32_t word() const {
        return base ^ ((rs_salt(I) << 16) | rs_salt(J));
    }
};

// The 16-bit encoding of a cell's outputs (raw, storage units): directions in pairs (i, i + 1, i in the
// upper half) through one paired conversion each; put(i, word) receives direction i's stored word.
template <class L, class S, class R, class Put>
__device__ __forceinline__ void encode16(const R (&out)[L::Q], const Rounding& rnd, uint32_t cell, Put&& put) {
    constexpr int NP = (L::Q + 1) / 2;
    auto put2 = [&](auto K, uint32_t w) {
        constexpr int i = 2 * decltype(K)::value, j = i + 1;
        put(std::integral_constant<int, i>{}, Pair16<S>::hi(w));
        if constexpr (j < L::Q) put(std::integral_constant<int, j>{}, Pair16<S>::lo(w));
    };
    auto second = [&](auto K) -> float {
        constexpr int j = 2 * decltype(K)::value + 1;
        if constexpr (j < L::Q)
            return out[j];
        else
            return 0.0f;
    };
    if (rnd.sr) {
        const uint32_t h = cell_hash16(cell, rnd.seed);
        const PairBits pb{(h << 16) | h};
        static_for<NP>([&](auto K) {
            constexpr int i = 2 * decltype(K)::value;
            put2(K, Pair16<S>::rs(out[i], second(K), pb.template word<i, i + 1>()));
        });
    } else {
        static_for<NP>([&](auto K) { put2(K, Pair16<S>::rn(out[2 * K], second(K))); });
    }
}

// The 16-bit store of a cell's outputs at fo[i * N].
template <class L, class S, class R>
__device__ __forceinline__ void store16(S* __restrict__ fo, long long N, const R (&out)[L::Q], const Rounding& rnd,
                                        uint32_t cell) {
    encode16<L, S>(out, rnd, cell, [&](auto I, S v) { fo[(long long)decltype(I)::value * N] = v; });
}

template <class L, class S, bool ABS, class P, class R>
__device__ __forceinline__ void store_cell(S* __restrict__ fout, const P& p, long long c, const R (&out)[L::Q],
                                           const Rounding& rnd) {
    if constexpr (!ABS && Codec<S>::kScaled) {
        store16<L, S>(fout + c, p.N, out, rnd, (uint32_t)c + p.cell_base);
    } else {
        static_for<L::Q>([&](auto I) {
            constexpr int i = I;
            if constexpr (ABS)
                Codec<S>::store(fout + (long long)i * p.N + c, out[i], R(L::w(i)), R(p.scale));
            else
                fout[(long long)i * p.N + c] = Codec<S>::enc(out[i], R(L::w(i)));
        });
    }
}

// store_cell with 32-bit population indices i N + c, for lattices whose Q N populations all have
// 32-bit indices: one 32-bit add and one widening multiply-add per address instead of 64-bit index
// arithmetic.  The same values, rounding bits and order as store_cell.
template <class L, class S, bool ABS, class P, class R>
__device__ __forceinline__ void store_cell32(S* __restrict__ fout, const P& p, uint32_t c, const R (&out)[L::Q],
                                             const Rounding& rnd) {
    const uint32_t N = (uint32_t)p.N;
    if constexpr (!ABS && Codec<S>::kScaled) {
        encode16<L, S>(out, rnd, c + p.cell_base,
                       [&](auto I, S v) { fout[(uint32_t)decltype(I)::value * N + c] = v; });
    } else {
        static_for<L::Q>([&](auto I) {
            constexpr int i = I;
            const uint32_t idx = (uint32_t)i * N + c;
            if constexpr (ABS)
                Codec<S>::store(fout + idx, out[i], R(L::w(i)), R(p.scale));
            else
                fout[idx] = Codec<S>::enc(out[i], R(L::w(i)));
        });
    }
}

// store_cell or store_cell32 by the index type of c.
template <class L, class S, bool ABS, class P, class R, class Ix>
__device__ __forceinline__ void store_cell_ix(S* __restrict__ fout, const P& p, Ix c, const R (&out)[L::Q],
                                              const Rounding& rnd) {
    if constexpr (std::is_same<Ix, uint32_t>::value)
        store_cell32<L, S, ABS>(fout, p, c, out, rnd);
    else
        store_cell<L, S, ABS>(fout, p, (long long)c, out, rnd);
}

// Storage scale and its inverse for raw deviations: the codec's scale for the 16-bit codecs,
// compile-time 1 otherwise.
template <class S, class P, class R>
__device__ __forceinline__ void storage_scale(const P& p, R& sc, R& isc) {
    if constexpr (Codec<S>::kScaled) {
        sc = R(p.scale);
        isc = R(p.inv_scale);
    } else {
        sc = R(1);
        isc = R(1);
    }
}

template <class T, class Ix>
__device__ __forceinline__ void cell_class(const uint8_t* __restrict__ mask, const ClassTable<T>& ct,
                                           Ix c, int& cls, uint32_t& fl) {
    cls = mask ? (int)__ldg(mask + c) : 0;
    fl = ct.flags[cls];
}

// Zou-He open boundaries of D2Q9 (Zou & He 1997, the velocity condition on the x = 0 face and the
// pressure condition on the x = nx-1 face): the streamed populations that arrive from outside the
// lattice (c_x = +1 at the inlet, c_x = -1 at the outlet) are rebuilt from the known ones so that the
// cell has the class's velocity (inlet) or density (outlet), with the non-equilibrium parts bounced
// back.  Directions 1 E, 2 N, 3 W, 4 S, 5 NE, 6 NW, 7 SW, 8 SE.  v: populations (ABS) or deviations in
// storage units (the weights of a rebuilt direction and its source agree, so deviations satisfy the
// same relations with every rho u term in storage units); sc / isc the storage scale and its inverse.
template <bool ABS, class T, class R>
__device__ __forceinline__ void zouhe_d2q9(const ClassTable<T>& ct, int cls, uint32_t fl, R (&v)[9], R sc, R isc) {
    const R k = ABS ? R(1) : sc;
    const R uy = R(ct.uy[cls]);
    const R half = R(0.5), sixth = R(1.0 / 6.0), two3 = R(2.0 / 3.0);
    const R t24 = half * (v[2] - v[4]);
    if (fl & kZouHeVelXm) {
        const R ux = R(ct.ux[cls]);
        const R s = v[0] + v[2] + v[4] + R(2) * (v[3] + v[6] + v[7]);
        const R rho = (ABS ? s : mad(s, isc, R(1))) / (R(1) - ux);
        const R ru = (rho * k) * ux, rv = (rho * k) * uy;
        v[1] = mad(two3, ru, v[3]);
        v[5] = mad(half, rv, mad(sixth, ru, v[7] - t24));
        v[8] = mad(-half, rv, mad(sixth, ru, v[6] + t24));
    } else {
        const R rho = R(ct.rho[cls]);
        const R s = v[0] + v[2] + v[4] + R(2) * (v[1] + v[5] + v[8]);
        const R ux = (ABS ? s : mad(s, isc, R(1))) / rho - R(1);
        const R ru = (rho * k) * ux, rv = (rho * k) * uy;
        v[3] = mad(-two3, ru, v[1]);
        v[7] = mad(-half, rv, mad(-sixth, ru, v[5] + t24));
        v[6] = mad(half, rv, mad(-sixth, ru, v[8] - t24));
    }
}

// ---- BGK ---------------------------------------------------------------------------------
// Collision of one cell from its streamed populations v (ABS) or deviations v = f - w:
// F = omega FEQ + (1 - omega) F_streamed (cpp/d2q9_bgk_lid.cpp:153), the class overwrites before it
// and the full-way bounce-back after it (:155).  P supplies cls, omega, one_m_omega.  Deviations
// are in storage units: sc / isc are the storage scale and its inverse (1 for ABS).  A Zou-He cell
// (D2Q9) first rebuilds its incoming populations in v.
template <class L, bool ABS, bool EXACTW, class P, class R>
__device__ __forceinline__ void bgk_collide(const P& p, int cls, uint32_t fl, R (&v)[L::Q], R sc, R isc,
                                            R (&out)[L::Q]) {
    if constexpr (L::Q == 9) {
        if (fl & (kZouHeVelXm | kZouHeRhoXp)) zouhe_d2q9<ABS>(p.cls, cls, fl, v, sc, isc);
    }
    R rho, drho, ux, uy, uz;
    moments<L, ABS>(v, sc, isc, rho, drho, ux, uy, uz);
    if (fl) apply_class(p.cls, cls, fl, rho, drho, ux, uy, uz, L::DIM);
    R fe[L::Q];
    equilibrium_v<L, ABS, EXACTW>(rho, drho, ux, uy, uz, sc, fe);
    const R omega = R(p.omega), one_m = R(p.one_m_omega);
    static_for<L::Q>([&](auto I) {
        constexpr int i = I;
        out[i] = (fl & kEquilibrium) ? fe[i] : mad(omega, fe[i], one_m * v[i]);
    });
    if (fl & kBounce) {
        // F(REFLECTED) = BOUNCEDBACK; w_opp(i) = w_i, so deviations bounce like populations
        static_for<L::Q - 1>([&](auto I) {
            constexpr int i = I + 1;
            out[L::opp(i)] = v[i];
        });
    }
}

// One cell of a BGK step read from and written to global memory.  P supplies mask, cls, nx, ny,
// nz, N, omega, one_m_omega, scale and inv_scale (StepParams for one lattice, BatchLattice for one
// member of an ensemble).
template <class L, class S, bool ABS, class Ix = long long, class P>
__device__ __forceinline__ void bgk_cell(const P& p, const S* __restrict__ fin, S* __restrict__ fout, int x, int y,
                                         int z, const Rounding& rnd) {
    using R = typename Codec<S>::Real;
    const RowsT<L, Ix> rows(y, z, p.nx, p.ny, p.nz);
    const Ix c = rows.base[1][1] + (Ix)x;
    R v[L::Q];
    pull<L, S, ABS>(fin, p, rows, x, v);
    int cls;
    uint32_t fl;
    cell_class(p.mask, p.cls, c, cls, fl);
    if (fl & kZeroGradXp) pull_zerograd<L, S, ABS>(fin, p, rows, x, v);
    R sc, isc;
    storage_scale<S>(p, sc, isc);
    R out[L::Q];
    bgk_collide<L, ABS, kExactWeights<S>>(p, cls, fl, v, sc, isc, out);
    store_cell_ix<L, S, ABS>(fout, p, c, out, rnd);
}

// I32: 32-bit population indices (lattices with Q N <= 2^32).
template <class L, class S, bool ABS, bool I32 = false>
__global__ void __launch_bounds__(512) k_step_bgk(const __grid_constant__ StepParams<typename Codec<S>::Real> p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= p.nx) return;
    const bool designated = (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x) == 0;
    const Rounding rnd = step_rounding<S>(p.tick, p.parity, p.sr, designated);
    const int y = L::DIM == 2 ? p.plo + (int)blockIdx.y * p.pstride : (int)blockIdx.y;
    const int z = L::DIM == 3 ? p.plo + (int)blockIdx.z * p.pstride : (int)blockIdx.z;
    bgk_cell<L, S, ABS, typename std::conditional<I32, uint32_t, long long>::type>(
        p, static_cast<const S*>(p.fin), static_cast<S*>(p.fout), x, y, z, rnd);
}

// ---- MRT (D3Q27) -------------------------------------------------------------------------
// Collision of one cell in deviation arithmetic.  T enters with the streamed deviations in tensor
// slot order (T[slot(i)] = f_i - w_i) and leaves with the post-collision deviations in direction
// order in out[].  The transform acts on d = f - w: M d = M f - M w, and M w = meq(rho = 1, u = 0) for
// both bases, so m* = m - S (m - meq) carries over with every equilibrium moment replaced by its
// deviation from rest, i.e. the cell quantity rho replaced by rho - 1 (mrt.cuh).  Bounce-back is left
// to the caller (it needs the streamed values, which the transform overwrote).  The deviations are in
// storage units (times sc); the transform is linear, so the scale rides along and enters only through
// isc here and through the equilibrium coefficients (beta and B carry sc, set on the host).
// Forward transform and the cell quantities: rho, rho - 1 and u from the moments of slots 0, 1, 3, 9.
template <int BASIS, class R>
__device__ __forceinline__ void mrt_pre(R (&T)[27], R isc, R& rho, R& drho, R& ux, R& uy, R& uz) {
    mrt_forward<BASIS>(T);
    drho = T[0] * isc;
    rho = R(1) + drho;
    const R inv = isc / rho;
    ux = T[1] * inv;
    uy = T[3] * inv;
    uz = T[9] * inv;
}

// Relaxation towards the equilibrium moments of (rho, u), inverse transform, direction order.
template <int BASIS, bool EXACT, class R, class K>
__device__ __forceinline__ void mrt_post(R (&T)[27], R rho, R drho, R ux, R uy, R uz, const MrtCoef<K>& k,
                                         R (&out)[27]) {
    using L = D3Q27;
    R q[11];
    q[0] = drho;
    q[1] = rho * ux;
    q[2] = rho * uy;
    q[3] = rho * uz;
    q[4] = q[1] * ux;
    q[5] = q[2] * uy;
    q[6] = q[3] * uz;
    q[7] = q[1] * uy;
    q[8] = q[1] * uz;
    q[9] = q[2] * uz;
    q[10] = mad(uz, uz, mad(uy, uy, ux * ux));
    mrt_relax<BASIS, EXACT>(T, q, k);
    mrt_inverse<BASIS>(T);
    static_for<27>([&](auto I) {
        constexpr int i = I;
        out[i] = T[L::slot(i)];
    });
}

template <int BASIS, bool EXACTW, class P, class R>
__device__ __forceinline__ void mrt_collide(const P& p, int cls, uint32_t fl, R (&T)[27], R sc, R isc,
                                            R (&out)[27]) {
    using L = D3Q27;
    R rho, drho, ux, uy, uz;
    mrt_pre<BASIS>(T, isc, rho, drho, ux, uy, uz);
    if (fl) apply_class(p.cls, cls, fl, rho, drho, ux, uy, uz, 3);
    mrt_post<BASIS, EXACTW>(T, rho, drho, ux, uy, uz, p.mrt, out);
    if (fl & kEquilibrium) equilibrium_dev<L, EXACTW, R>(rho, drho, ux, uy, uz, sc, out);
}

// ---- two-rate MRT (Gram-Schmidt basis) -----------------------------------------------------
// With the rows of M orthogonal (M M^T = D diagonal, M^-1 = M^T D^-1) and meq = M feq, a rate vector
// with two values -- s_v on the shear rows, s_o on every other row -- turns the collision
// f* = M^-1 (m - S (m - meq)) into
//   f* = f - s_o (f - feq) - (s_v - s_o) sum_{k in shear} M_k (m_k - meq_k) / D_k,
// the same map, evaluated without the full forward and inverse transforms: the moments needed are rho,
// j and the five shear moments (a partial tensor transform, 79 adds instead of 108), the equilibrium
// comes per pair of opposite directions as in BGK, and the shear correction is even in c, so each pair
// shares it.  In storage units on deviations like mrt_collide (the shear moments of w are zero).  The
// shear rows (Gram-Schmidt): cx cy, cx cz, cy cz (|row|^2 = 12), 3(cx^2 - cy^2) (108) and
// 3(cx^2 + cy^2 - 2 cz^2) (324); their equilibrium moments rho ux uy, rho ux uz, rho uy uz,
// 3 rho (ux^2 - uy^2), 3 rho (ux^2 + uy^2 - 2 uz^2).  v: streamed deviations in direction order (kept:
// bounce-back reads them).  Used for 16-bit storage when the rates have that structure (the benchmark
// cavity's); the general collision stays for every other case.
template <class P, class R>
__device__ __forceinline__ void mrt2_collide(const P& p, int cls, uint32_t fl, const R (&v)[27], R sc, R isc,
                                             R (&out)[27]) {
    using L = D3Q27;
    // x lines: (cy, cz) = line l = yb + 3 zc; X0 = sum, X1 = c-moment, X2 = (3c^2 - 2)-moment
    R X0[9], X1[9], X2[9];
    static_for<9>([&](auto Lc) {
        constexpr int l = Lc;
        constexpr int cy = l % 3 - 1, cz = l / 3 - 1;
        constexpr int im = L::dir_of(-1, cy, cz), i0 = L::dir_of(0, cy, cz), ip = L::dir_of(1, cy, cz);
        const R sum2 = v[im] + v[ip];
        X1[l] = v[ip] - v[im];
        X0[l] = sum2 + v[i0];
        X2[l] = minus_twice(sum2, v[i0]);
    });
    // y lines per z
    R Y00[3], Y01[3], Y02[3], Y10[3], Y11[3], Y20[3];
    static_for<3>([&](auto Zc) {
        constexpr int z = Zc;
        const R s0 = X0[3 * z] + X0[3 * z + 2];
        Y00[z] = s0 + X0[3 * z + 1];
        Y01[z] = X0[3 * z + 2] - X0[3 * z];
        Y02[z] = minus_twice(s0, X0[3 * z + 1]);
        Y10[z] = (X1[3 * z] + X1[3 * z + 2]) + X1[3 * z + 1];
        Y11[z] = X1[3 * z + 2] - X1[3 * z];
        Y20[z] = (X2[3 * z] + X2[3 * z + 2]) + X2[3 * z + 1];
    });
    // z: the ten moments
    const R sz = Y00[0] + Y00[2];
    const R m000 = sz + Y00[1], m001 = Y00[2] - Y00[0], m002 = minus_twice(sz, Y00[1]);
    const R m100 = (Y10[0] + Y10[2]) + Y10[1], m101 = Y10[2] - Y10[0];
    const R m010 = (Y01[0] + Y01[2]) + Y01[1], m011 = Y01[2] - Y01[0];
    const R m110 = (Y11[0] + Y11[2]) + Y11[1];
    const R m200 = (Y20[0] + Y20[2]) + Y20[1];
    const R m020 = (Y02[0] + Y02[2]) + Y02[1];
    // cell quantities (as mrt_pre) and the class overwrites
    R drho = m000 * isc;
    R rho = R(1) + drho;
    const R inv = isc / rho;
    R ux = m100 * inv, uy = m010 * inv, uz = m001 * inv;
    if (fl) apply_class(p.cls, cls, fl, rho, drho, ux, uy, uz, 3);
    const Mrt2Coef<R>& k = p.mrt2;
    // non-equilibrium parts of the shear moments, scaled by (s_v - s_o) / |row|^2
    const R rux = rho * ux, ruy = rho * uy, ruz = rho * uz;
    const R nsc = -sc, n3sc = R(-3) * sc;
    const R q4 = rux * ux, q5 = ruy * uy, q6 = ruz * uz;
    const R a = k.kxy * mad(nsc, rux * uy, m110);
    const R b = k.kxy * mad(nsc, rux * uz, m101);
    const R c = k.kxy * mad(nsc, ruy * uz, m011);
    const R e8 = k.k8 * mad(n3sc, q4 - q5, m200 - m020);
    const R e9 = k.k9 * mad(n3sc, minus_twice(q4 + q5, q6), minus_twice(m200 + m020, m002));
    // shear correction of each direction class (even in c)
    const R cfx = e8 + e9, cfy = e9 - e8, cfz = R(-2) * e9;
    const R exy = e9 + e9, exz = e8 - e9;
    // equilibrium parts per weight class: s_o w sc (drho + rho (4.5 eu^2 - 1.5 u^2)) +- s_o w sc 3 rho eu
    const R nusq15 = R(-1.5) * mad(uz, uz, mad(uy, uy, ux * ux));
    const R base = mad(rho, nusq15, drho);
    R wb[4], w45[4], w3[4];
    static_for<4>([&](auto Cc) {
        constexpr int cc = Cc;
        wb[cc] = k.sw[cc] * base;
        if constexpr (cc > 0) {
            w45[cc] = k.sw45[cc] * rho;
            w3[cc] = k.sw3[cc] * rho;
        }
    });
    const R om1 = k.om1;
    out[0] = mad(om1, v[0], wb[0]);
    static_for<27>([&](auto I) {
        constexpr int i = I;
        constexpr int o = L::opp(i);
        if constexpr (i > 0 && i < o) {
            constexpr int cx = L::cx(i), cy = L::cy(i), cz = L::cz(i);
            constexpr int nz = (cx != 0) + (cy != 0) + (cz != 0);  // 1 face, 2 edge, 3 corner
            R eu = cx != 0 ? (cx == 1 ? ux : -ux) : (cy != 0 ? (cy == 1 ? uy : -uy) : (cz == 1 ? uz : -uz));
            if constexpr (cx != 0 && cy == 1) eu = eu + uy;
            if constexpr (cx != 0 && cy == -1) eu = eu - uy;
            if constexpr ((cx != 0 || cy != 0) && cz == 1) eu = eu + uz;
            if constexpr ((cx != 0 || cy != 0) && cz == -1) eu = eu - uz;
            R corr;
            if constexpr (nz == 1) {
                corr = cx != 0 ? cfx : (cy != 0 ? cfy : cfz);
            } else if constexpr (nz == 2) {
                if constexpr (cz == 0)
                    corr = cx * cy == 1 ? exy + a : exy - a;
                else if constexpr (cy == 0)
                    corr = cx * cz == 1 ? exz + b : exz - b;
                else
                    corr = cy * cz == 1 ? c - cfx : -(c + cfx);
            } else {
                const R t1 = cx * cy == 1 ? a : -a;
                const R t2 = cx * cz == 1 ? t1 + b : t1 - b;
                corr = cy * cz == 1 ? t2 + c : t2 - c;
            }
            // the odd part (+- w3 eu) enters by multiply-adds: two FMAs instead of a product and two adds
            const R sym = mad(w45[nz], eu * eu, wb[nz]) - corr;
            out[i] = mad(om1, v[i], mad(w3[nz], eu, sym));
            out[o] = mad(om1, v[o], mad(-w3[nz], eu, sym));
        }
    });
    if (fl & kEquilibrium) equilibrium_dev<L, false, R>(rho, drho, ux, uy, uz, sc, out);
    if (fl & kBounce) {
        static_for<26>([&](auto I) {
            constexpr int i = I + 1;
            out[L::opp(i)] = v[i];
        });
    }
}

template <int BASIS, class S, bool I32 = false>
__global__ void __launch_bounds__(256) k_step_mrt(const __grid_constant__ StepParams<typename Codec<S>::Real> p) {
    using L = D3Q27;
    using R = typename Codec<S>::Real;
    using Ix = typename std::conditional<I32, uint32_t, long long>::type;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= p.nx) return;
    const int y = blockIdx.y, z = p.plo + (int)blockIdx.z * p.pstride;
    const RowsT<L, Ix> rows(y, z, p.nx, p.ny, p.nz);
    const Ix c = rows.base[1][1] + (Ix)x;
    const S* __restrict__ fin = static_cast<const S*>(p.fin);
    R T[27];
    int cls;
    uint32_t fl;
    {
        R v[27];
        pull<L, S, false>(fin, p, rows, x, v);
        cell_class(p.mask, p.cls, c, cls, fl);
        if (fl & kZeroGradXp) pull_zerograd<L, S, false>(fin, p, rows, x, v);
        static_for<27>([&](auto I) {
            constexpr int i = I;
            T[L::slot(i)] = v[i];
        });
    }
    R sc, isc;
    storage_scale<S>(p, sc, isc);
    R out[27];
    mrt_collide<BASIS, kExactWeights<S>>(p, cls, fl, T, sc, isc, out);
    if (fl & kBounce) {
        // reload the streamed deviations (the transform overwrote them in place)
        R v[27];
        pull<L, S, false>(fin, p, rows, x, v);
        if (fl & kZeroGradXp) pull_zerograd<L, S, false>(fin, p, rows, x, v);
        static_for<26>([&](auto I) {
            constexpr int i = I + 1;
            out[L::opp(i)] = v[i];
        });
    }
    const bool designated = (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x) == 0;
    const Rounding rnd = step_rounding<S>(p.tick, p.parity, p.sr, designated);
    store_cell_ix<L, S, false>(static_cast<S*>(p.fout), p, c, out, rnd);
}

// The plain (one thread per cell) step kernel of the two-rate collision.
template <class S, bool I32 = false>
__global__ void __launch_bounds__(256) k_step_mrt2(const __grid_constant__ StepParams<typename Codec<S>::Real> p) {
    using L = D3Q27;
    using R = typename Codec<S>::Real;
    using Ix = typename std::conditional<I32, uint32_t, long long>::type;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= p.nx) return;
    const RowsT<L, Ix> rows(blockIdx.y, p.plo + (int)blockIdx.z * p.pstride, p.nx, p.ny, p.nz);
    const Ix c = rows.base[1][1] + (Ix)x;
    const S* __restrict__ fin = static_cast<const S*>(p.fin);
    R v[27];
    pull<L, S, false>(fin, p, rows, x, v);
    int cls;
    uint32_t fl;
    cell_class(p.mask, p.cls, c, cls, fl);
    if (fl & kZeroGradXp) pull_zerograd<L, S, false>(fin, p, rows, x, v);
    R sc, isc;
    storage_scale<S>(p, sc, isc);
    R out[27];
    mrt2_collide(p, cls, fl, v, sc, isc, out);
    const bool designated = (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x) == 0;
    const Rounding rnd = step_rounding<S>(p.tick, p.parity, p.sr, designated);
    store_cell_ix<L, S, false>(static_cast<S*>(p.fout), p, c, out, rnd);
}

// ---- Shan-Chen (D2Q9) --------------------------------------------------------------------
// Pass 1: psi = 1 - exp(-rho) of the streamed density of every cell.
// psi = 1 - exp(-rho) of the streamed density of one cell (the pseudopotential of the Shan-Chen
// force); also returns the cell's pulled populations and class, which the collision reuses.
template <class S, bool ABS, class R, class Ix>
__device__ __forceinline__ void sc_pull_cell(const StepParams<R>& p, const S* __restrict__ fin,
                                             const RowsT<D2Q9, Ix>& rows, int x, Ix c, R (&v)[9], int& cls,
                                             uint32_t& fl) {
    using L = D2Q9;
    pull<L, S, ABS>(fin, p, rows, x, v);
    cell_class(p.mask, p.cls, c, cls, fl);
    if (fl & kZeroGradXp) pull_zerograd<L, S, ABS>(fin, p, rows, x, v);
}
template <class S, bool ABS, class R>
__device__ __forceinline__ R sc_psi_from(const StepParams<R>& p, const R (&v)[9], int cls, uint32_t fl) {
    R sc, isc;
    storage_scale<S>(p, sc, isc);
    R sum = R(0);
    static_for<9>([&](auto I) { sum += v[I]; });
    R rho = ABS ? sum : R(1) + sum * isc;
    if (fl & kSetRho) rho = R(p.cls.rho[cls]);
    return R(1) - exp(-rho);
}
template <class S, bool ABS, class R, class Ix>
__device__ __forceinline__ R sc_psi_of(const StepParams<R>& p, const S* __restrict__ fin, const RowsT<D2Q9, Ix>& rows,
                                       int x, Ix c, R (&v)[9], int& cls, uint32_t& fl) {
    sc_pull_cell<S, ABS>(p, fin, rows, x, c, v, cls, fl);
    return sc_psi_from<S, ABS>(p, v, cls, fl);
}

// Row offsets (y + dy) nx of the rows y - 1, y, y + 1 (periodic) as 32-bit cell indices, for the window
// kernel on lattices whose 9 N populations all have 32-bit indices.
struct WinRows {
    uint32_t base[3];  // [dy + 1]
    __device__ __forceinline__ WinRows(int y, int nx, int ny) {
        base[0] = (uint32_t)(y == 0 ? ny - 1 : y - 1) * (uint32_t)nx;
        base[1] = (uint32_t)y * (uint32_t)nx;
        base[2] = (uint32_t)(y == ny - 1 ? 0 : y + 1) * (uint32_t)nx;
    }
    // source row of direction cy: pull from y - cy
    __device__ __forceinline__ uint32_t src(int cy) const { return base[1 - cy]; }
};

// sc_pull_cell with 32-bit population indices i N + row + x (WinRows): the same loads, values and
// class as sc_pull_cell, each address one 32-bit add and one widening multiply-add.
template <class S, bool ABS, class R>
__device__ __forceinline__ void sc_pull_cell32(const StepParams<R>& p, const S* __restrict__ fin, const WinRows& rows,
                                               int x, uint32_t c, R (&v)[9], int& cls, uint32_t& fl) {
    using L = D2Q9;
    const uint32_t N = (uint32_t)p.N;
    const int xm = x == 0 ? p.nx - 1 : x - 1;
    const int xp = x == p.nx - 1 ? 0 : x + 1;
    static_for<9>([&](auto I) {
        constexpr int i = I;
        constexpr int cx = L::cx(i), cy = L::cy(i);
        const int xs = cx == 1 ? xm : (cx == -1 ? xp : x);
        const uint32_t idx = (uint32_t)i * N + rows.src(cy) + (uint32_t)xs;
        if constexpr (ABS)
            v[i] = Codec<S>::load(fin + idx, R(L::w(i)), R(p.inv_scale));
        else
            v[i] = Codec<S>::raw(__ldg(fin + idx), R(L::w(i)));
    });
    cls = p.mask ? (int)__ldg(p.mask + c) : 0;
    fl = p.cls.flags[cls];
    if (fl & kZeroGradXp) {  // pull_zerograd: c_x = -1 from the cell's own column
        static_for<9>([&](auto I) {
            constexpr int i = I;
            if constexpr (L::cx(i) == -1) {
                const uint32_t idx = (uint32_t)i * N + rows.src(L::cy(i)) + (uint32_t)x;
                if constexpr (ABS)
                    v[i] = Codec<S>::load(fin + idx, R(L::w(i)), R(p.inv_scale));
                else
                    v[i] = Codec<S>::raw(__ldg(fin + idx), R(L::w(i)));
            }
        });
    }
}

// I32: 32-bit population indices (lattices with 9 N <= 2^32).
template <class S, bool ABS, bool I32 = false>
__global__ void __launch_bounds__(512) k_sc_psi(const __grid_constant__ StepParams<typename Codec<S>::Real> p) {
    using L = D2Q9;
    using R = typename Codec<S>::Real;
    using Ix = typename std::conditional<I32, uint32_t, long long>::type;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= p.nx) return;
    const int y = blockIdx.y, z = blockIdx.z;
    const RowsT<L, Ix> rows(y, z, p.nx, p.ny, p.nz);
    const Ix c = rows.base[1][1] + (Ix)x;
    R v[9];
    int cls;
    uint32_t fl;
    p.psi[c] = sc_psi_of<S, ABS>(p, static_cast<const S*>(p.fin), rows, x, c, v, cls, fl);
}

// Shan-Chen force F = -G psi(x) sum_i w_i psi(x + c_i) c_i at one cell; psi_at(dx, dy) is psi of the
// neighbour (x + dx, y + dy).  One summation order for every caller.
template <class R, class PsiAt>
__device__ __forceinline__ void sc_force_from(const StepParams<R>& p, PsiAt&& psi_at, R& Fx, R& Fy) {
    using L = D2Q9;
    R sx = R(0), sy = R(0);
    static_for<8>([&](auto I) {
        constexpr int i = I + 1;
        constexpr int cx = L::cx(i), cy = L::cy(i);
        const R v = R(L::w(i)) * psi_at(cx, cy);
        if constexpr (cx == 1) sx += v;
        if constexpr (cx == -1) sx -= v;
        if constexpr (cy == 1) sy += v;
        if constexpr (cy == -1) sy -= v;
    });
    const R g = -p.G * psi_at(0, 0);
    Fx = g * sx;
    Fy = g * sy;
}

// The force at cell (x, y) from the psi field in global memory (periodic).
template <class R, class Ix>
__device__ __forceinline__ void sc_force(const StepParams<R>& p, const RowsT<D2Q9, Ix>& rows, int x, Ix c, R& Fx,
                                         R& Fy) {
    const int xm = x == 0 ? p.nx - 1 : x - 1;
    const int xp = x == p.nx - 1 ? 0 : x + 1;
    sc_force_from(p, [&](int dx, int dy) {
        if (dx == 0 && dy == 0) return __ldg(p.psi + c);
        // neighbour x + c_i: the source row of the opposite direction
        const int xn = dx == 1 ? xp : (dx == -1 ? xm : x);
        return __ldg(p.psi + (rows.src(-dy, 0) + (Ix)xn));
    }, Fx, Fy);
}

// The Shan-Chen collision of one cell from its pulled populations v (class cls, flags fl) and the
// force: moments, class overrides, velocity shift u_eq = u + tau F / rho (Shan & Chen 1993), BGK,
// bounce-back, store.
template <class S, bool ABS, class R, class Idx>
__device__ __forceinline__ void sc_collide_store(const StepParams<R>& p, Idx c, const R (&v)[9], int cls,
                                                 uint32_t fl, R Fx, R Fy, const Rounding& rnd) {
    using L = D2Q9;
    R sc, isc;
    storage_scale<S>(p, sc, isc);
    R rho, drho, ux, uy, uz;
    moments<L, ABS>(v, sc, isc, rho, drho, ux, uy, uz);
    if (fl) apply_class(p.cls, cls, fl, rho, drho, ux, uy, uz, 2);
    R vx = ux, vy = uy;
    if (rho > R(0)) {
        const R k = R(1) / (p.omega * rho);
        vx = ux + Fx * k;
        vy = uy + Fy * k;
    }
    R fe[9];
    equilibrium_v<L, ABS, kExactWeights<S>>(rho, drho, vx, vy, R(0), sc, fe);
    R out[9];
    static_for<9>([&](auto I) {
        constexpr int i = I;
        out[i] = (fl & kEquilibrium) ? fe[i] : p.omega * fe[i] + p.one_m_omega * v[i];
    });
    if (fl & kBounce) {
        static_for<8>([&](auto I) {
            constexpr int i = I + 1;
            out[L::opp(i)] = v[i];
        });
    }
    if constexpr (std::is_same<Idx, uint32_t>::value)
        store_cell32<L, S, ABS>(static_cast<S*>(p.fout), p, c, out, rnd);
    else
        store_cell<L, S, ABS>(static_cast<S*>(p.fout), p, (long long)c, out, rnd);
}

// Second pass of the two-pass Shan-Chen step (psi from k_sc_psi in global memory).
template <class S, bool ABS, bool I32 = false>
__global__ void __launch_bounds__(512) k_step_sc(const __grid_constant__ StepParams<typename Codec<S>::Real> p) {
    using L = D2Q9;
    using R = typename Codec<S>::Real;
    using Ix = typename std::conditional<I32, uint32_t, long long>::type;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= p.nx) return;
    const int y = blockIdx.y, z = blockIdx.z;
    const RowsT<L, Ix> rows(y, z, p.nx, p.ny, p.nz);
    const Ix c = rows.base[1][1] + (Ix)x;
    const S* __restrict__ fin = static_cast<const S*>(p.fin);
    R v[9];
    pull<L, S, ABS>(fin, p, rows, x, v);
    int cls;
    uint32_t fl;
    cell_class(p.mask, p.cls, c, cls, fl);
    if (fl & kZeroGradXp) pull_zerograd<L, S, ABS>(fin, p, rows, x, v);
    R Fx, Fy;
    sc_force(p, rows, x, c, Fx, Fy);
    const bool designated = (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x) == 0;
    const Rounding rnd = step_rounding<S>(p.tick, p.parity, p.sr, designated);
    sc_collide_store<S, ABS>(p, c, v, cls, fl, Fx, Fy, rnd);
}

// The whole Shan-Chen step in one pass, as a window sliding down y.  A CTA owns a strip of kScwTX
// columns and rows [y0, y0 + rows); thread tx owns column x0 + tx.  Per row y it pulls row y + 1 once
// (the populations stay in registers for the next row's collision), writes psi of row y + 1 into a
// ring of 4 shared rows (two threads add the strip's edge columns, periodic wrap), and after one
// block barrier takes the force at row y from ring rows y - 1 .. y + 1.  With 4 ring rows one barrier
// per row suffices: a row's slot is rewritten two barriers after its last read.  psi, force and
// collision are the two-pass kernels' device functions: bit-identical results.  I32: 32-bit
// population indices (lattices with 9 N <= 2^32), which take about a third of the address arithmetic
// of 64-bit ones; the same loads and stores.
#ifndef LBM_SCW_TX
#define LBM_SCW_TX 128
#endif
#ifndef LBM_SCW_MINB
#define LBM_SCW_MINB 8  // resident CTAs per SM asked of the compiler (FP64 storage: 4, up to 128 registers)
#endif
constexpr int kScwTX = LBM_SCW_TX;

template <class S, bool ABS, bool I32>
__global__ void __launch_bounds__(kScwTX, sizeof(typename Codec<S>::Real) == 8 ? 4 : LBM_SCW_MINB) k_step_sc_window(const __grid_constant__ StepParams<typename Codec<S>::Real> p,
                                                           int rows_per_strip) {
    using L = D2Q9;
    using R = typename Codec<S>::Real;
    using Idx = typename std::conditional<I32, uint32_t, long long>::type;
    constexpr int TX = kScwTX, PX = TX + 2;
    static_assert(TX >= 2, "two edge threads");
    __shared__ R ring[4][PX];
    const S* __restrict__ fin = static_cast<const S*>(p.fin);
    const int nx = p.nx, ny = p.ny;
    const int tx = threadIdx.x;
    const int x0 = blockIdx.x * TX;
    // rows plo + k pstride, k < pcnt: contiguous (pstride 1) in strips of rows_per_strip rows, else one
    // row per strip
    int ys, ye;
    if (p.pstride == 1) {
        const int end = p.plo + p.pcnt;
        ys = p.plo + (int)blockIdx.y * rows_per_strip;
        if (ys >= end) return;  // uniform over the block
        ye = ys + rows_per_strip < end ? ys + rows_per_strip : end;
    } else {
        ys = p.plo + (int)blockIdx.y * p.pstride;
        ye = ys + 1;
    }
    const int x = x0 + tx;
    const bool own_x = x < nx;
    const int xs = own_x ? x : x % nx;  // past the edge: the periodic image (only its psi is used)
    int xe = tx == 0 ? x0 - 1 : x0 + TX;  // the strip's edge columns (threads 0 and 1)
    xe = xe < 0 ? xe + nx : xe % nx;
    const int le = tx == 0 ? 0 : PX - 1;
    auto psi_row = [&](int y, R (&v)[9], int& cls, uint32_t& fl) {
        const int yw = y < 0 ? y + ny : (y >= ny ? y - ny : y);
        R w[9];
        int c2 = 0;
        uint32_t f2 = 0;
        Idx c;
        if constexpr (I32) {
            const WinRows rows(yw, nx, ny);
            c = rows.base[1] + (uint32_t)xs;
            sc_pull_cell32<S, ABS>(p, fin, rows, xs, c, v, cls, fl);
            if (tx < 2) sc_pull_cell32<S, ABS>(p, fin, rows, xe, rows.base[1] + (uint32_t)xe, w, c2, f2);
        } else {
            const Rows<L> rows(yw, 0, nx, ny, 1);
            c = rows.base[1][1] + xs;
            sc_pull_cell<S, ABS>(p, fin, rows, xs, c, v, cls, fl);
            if (tx < 2) sc_pull_cell<S, ABS>(p, fin, rows, xe, rows.base[1][1] + xe, w, c2, f2);
        }
        const R ps = sc_psi_from<S, ABS>(p, v, cls, fl);
        ring[y & 3][tx + 1] = ps;
        if (own_x && y >= ys && y < ye) p.psi[c] = ps;
        if (tx < 2) ring[y & 3][le] = sc_psi_from<S, ABS>(p, w, c2, f2);
    };
    const Rounding rnd = step_rounding<S>(p.tick, p.parity, p.sr, (blockIdx.x | blockIdx.y | threadIdx.x) == 0);
    R vc[9], vn[9];
    int cc = 0, cn = 0;
    uint32_t fc = 0, fn = 0;
    psi_row(ys - 1, vn, cn, fn);  // the row above the strip: psi only
    psi_row(ys, vc, cc, fc);
#pragma unroll 1
    for (int y = ys; y < ye; ++y) {
        psi_row(y + 1, vn, cn, fn);  // the next row (the row below the strip on the last pass)
        __syncthreads();
        if (own_x) {
            const Idx c = (Idx)y * (Idx)nx + (Idx)x;
            R Fx, Fy;
            sc_force_from(p, [&](int dx, int dy) { return ring[(y + dy) & 3][tx + 1 + dx]; }, Fx, Fy);
            sc_collide_store<S, ABS>(p, c, vc, cc, fc, Fx, Fy, rnd);
        }
        static_for<9>([&](auto I) { vc[I] = vn[I]; });
        cc = cn;
        fc = fn;
    }
}

// ---- macroscopic fields ------------------------------------------------------------------
// pulled = 1: the fields the last step's collision used (pull from the previous buffer, class
// overwrites, Shan-Chen velocity u + F/(2 rho)).  pulled = 0: local moments of p.fin.
template <class L, class S, class O>
__global__ void k_macros(const __grid_constant__ StepParams<typename Codec<S>::Real> p, int pulled, int collision, O* rho_out,
                         O* u_out) {
    using R = typename Codec<S>::Real;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= p.nx) return;
    const int y = blockIdx.y, z = blockIdx.z;
    const Rows<L> rows(y, z, p.nx, p.ny, p.nz);
    const long long c = rows.base[1][1] + x;
    const S* __restrict__ fin = static_cast<const S*>(p.fin);
    R d[L::Q];
    int cls;
    uint32_t fl;
    cell_class(p.mask, p.cls, c, cls, fl);
    if (pulled) {
        pull<L, S, false>(fin, p, rows, x, d);
        if (fl & kZeroGradXp) pull_zerograd<L, S, false>(fin, p, rows, x, d);
    } else {
        static_for<L::Q>([&](auto I) {
            constexpr int i = I;
            d[i] = Codec<S>::raw(__ldg(fin + (long long)i * p.N + c), R(L::w(i)));
        });
    }
    R sc, isc;
    storage_scale<S>(p, sc, isc);
    if constexpr (L::Q == 9) {
        if (pulled && (fl & (kZouHeVelXm | kZouHeRhoXp))) zouhe_d2q9<false>(p.cls, cls, fl, d, sc, isc);
    }
    R rho, drho, ux, uy, uz;
    moments<L, false>(d, sc, isc, rho, drho, ux, uy, uz);
    if (pulled && fl) apply_class(p.cls, cls, fl, rho, drho, ux, uy, uz, L::DIM);
    if constexpr (L::DIM == 2) {
        if (pulled && collision == 2) {
            R Fx, Fy;
            sc_force(p, rows, x, c, Fx, Fy);
            if (rho > R(0)) {
                ux = ux + Fx / (R(2) * rho);
                uy = uy + Fy / (R(2) * rho);
            }
        }
    }
    if (rho_out) rho_out[c] = O(rho);
    if (u_out) {
        u_out[c] = O(ux);
        u_out[p.N + c] = O(uy);
        if (L::DIM == 3) u_out[2 * p.N + c] = O(uz);
    }
}

// ---- FP64 conservation sums and steady-state residual ------------------------------------
struct Sums {
    double m, jx, jy, jz;
    unsigned long long bad;  // non-finite populations seen
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Stage 1: one partial per block over a grid-stride range of cells (fixed grid -> deterministic).
template <class L, class S>
__global__ void __launch_bounds__(256) k_sums_partial(const S* __restrict__ f, long long N, float inv_scale,
                                                       Sums* __restrict__ partial) {
    using R = typename Codec<S>::Real;
    double m = 0, jx = 0, jy = 0, jz = 0;
    unsigned long long bad = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N;
         c += (long long)gridDim.x * blockDim.x) {
        static_for<L::Q>([&](auto I) {
            constexpr int i = I;
            const double v = (double)Codec<S>::load(f + (long long)i * N + c, R(L::w(i)), R(inv_scale));
            if (!isfinite(v)) ++bad;
            m += v;
            if constexpr (L::cx(i) != 0) jx += L::cx(i) * v;
            if constexpr (L::cy(i) != 0) jy += L::cy(i) * v;
            if constexpr (L::cz(i) != 0) jz += L::cz(i) * v;
        });
    }
    __shared__ double sh[4][8];
    __shared__ unsigned long long shb[8];
    m = warp_sum(m);
    jx = warp_sum(jx);
    jy = warp_sum(jy);
    jz = warp_sum(jz);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][wid] = m;
        sh[1][wid] = jx;
        sh[2][wid] = jy;
        sh[3][wid] = jz;
        shb[wid] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Sums s{0, 0, 0, 0, 0};
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            s.m += sh[0][w];
            s.jx += sh[1][w];
            s.jy += sh[2][w];
            s.jz += sh[3][w];
            s.bad += shb[w];
        }
        partial[blockIdx.x] = s;
    }
}

// Stage 2: one thread folds the partials in index order.
__global__ void k_sums_final(const Sums* __restrict__ partial, int n, Sums* __restrict__ out);

// Residual partials: sum |u_a - u_b|^2 and |u_a|^2 over class-0 cells (local moments).
template <class L, class S>
__global__ void __launch_bounds__(256) k_residual_partial(const S* __restrict__ fa, const S* __restrict__ fb,
                                                           const uint8_t* __restrict__ mask, long long N,
                                                           float inv_scale, Sums* __restrict__ partial) {
    using R = typename Codec<S>::Real;
    double num = 0, den = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N;
         c += (long long)gridDim.x * blockDim.x) {
        if (mask && __ldg(mask + c) != 0) continue;
        double ra = 0, xa = 0, ya = 0, za = 0, rb = 0, xb = 0, yb = 0, zb = 0;
        static_for<L::Q>([&](auto I) {
            constexpr int i = I;
            const double a = (double)Codec<S>::load(fa + (long long)i * N + c, R(L::w(i)), R(inv_scale));
            const double b = (double)Codec<S>::load(fb + (long long)i * N + c, R(L::w(i)), R(inv_scale));
            ra += a;
            rb += b;
            xa += L::cx(i) * a;
            xb += L::cx(i) * b;
            ya += L::cy(i) * a;
            yb += L::cy(i) * b;
            za += L::cz(i) * a;
            zb += L::cz(i) * b;
        });
        const double dx = xa / ra - xb / rb, dy = ya / ra - yb / rb, dz = za / ra - zb / rb;
        num += dx * dx + dy * dy + dz * dz;
        den += (xa * xa + ya * ya + za * za) / (ra * ra);
    }
    __shared__ double sh[2][8];
    num = warp_sum(num);
    den = warp_sum(den);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][wid] = num;
        sh[1][wid] = den;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Sums s{0, 0, 0, 0, 0};
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            s.m += sh[0][w];
            s.jx += sh[1][w];
        }
        partial[blockIdx.x] = s;
    }
}

}  // namespace lbm
