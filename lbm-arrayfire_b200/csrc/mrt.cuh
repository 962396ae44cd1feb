// mrt.cuh — factorised D3Q27 multiple-relaxation-time collision, entirely in registers.
//
// The reference's moment matrix (rust/examples/d3q27_mrt_lid.rs:167-193) has rows that are
// monomials cx^a cy^b cz^c with a,b,c in {0,1,2}, except rows 7-9 which mix the three
// second-order diagonal monomials (e^2, ex^2-ey^2, ex^2-ez^2).  So m = M f factors into three
// 3-point transforms (one per axis) over the 3x3x3 tensor of populations, followed by a 3x3 mix
// of the tensor slots (2,0,0), (0,2,0), (0,0,2).  The reference multiplies by a dense 27x27
// matrix three times per cell (:336,385,387); here the forward transform costs 81 adds, the
// inverse 81-108, and the diagonal relaxation is folded into one multiply-add per slot.
//
// Two bases share the code:
//   REF (0)          1D rows {1, c, c^2}         (the reference's raw monomials, inverse exact)
//   GRAM_SCHMIDT (1) 1D rows {1, c, 3c^2 - 2}    (Gram-Schmidt of the reference rows in order,
//                    unweighted; rows 7-9 become (1,1,1), (1,-1,0), (1,1,-2) mixes of the slots)
// Tensor slot t = a + 3b + 9c holds the moment of order (a,b,c); direction i sits in slot
// (cx+1) + 3(cy+1) + 9(cz+1) before the transform.
#pragma once

#include <cmath>

#include "arith.cuh"
#include "lattice.cuh"

namespace lbm {

enum { kMrtRef = 0, kMrtGramSchmidt = 1 };

// Reference row that owns tensor slot t (-1: one of the mixed slots 2, 6, 18 -> rows 7, 8, 9).
LBM_HD constexpr int mrt_slot_row(int t) {
    constexpr int v[27] = {0,  1,  -1, 2,  4,  12, -1, 10, 17, 3,  5,  13, 6, 16,
                           20, 15, 21, 25, -1, 11, 18, 14, 22, 24, 19, 23, 26};
    return v[t];
}

// Per-axis scale of the inverse 1D transform (folded into the relaxation coefficients).
LBM_HD constexpr double mrt_axis_scale(int basis, int a) {
    return basis == kMrtRef ? (a == 0 ? 1.0 : 0.5) : (a == 0 ? 1.0 / 3.0 : (a == 1 ? 0.5 : 1.0 / 6.0));
}
LBM_HD constexpr double mrt_slot_scale(int basis, int t) {
    return mrt_axis_scale(basis, t % 3) * mrt_axis_scale(basis, (t / 3) % 3) * mrt_axis_scale(basis, t / 9);
}

// Equilibrium moment of slot t as a linear form in the cell quantities
//   k: 0 rho, 1 rho ux, 2 rho uy, 3 rho uz, 4 rho ux^2, 5 rho uy^2, 6 rho uz^2,
//      7 rho ux uy, 8 rho ux uz, 9 rho uy uz, 10 |u|^2
// REF: the table of rust/examples/d3q27_mrt_lid.rs:357-383 (rows 7-9 rewritten per slot:
//      (2,0,0) -> rho/3 + rho ux^2 etc., whose 7-9 mixes reproduce the table's rows).
// GRAM_SCHMIDT: moments of feq = w rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u^2); the D3Q27 weights
//      factor per axis (w1 = {1/6, 2/3, 1/6}), so each moment is a product of 1D weighted moments
//      E_a[1] = p_a, E_a[c] = q_a, E_a[c^2] = r_a of the 1D polynomials {1, c, 3c^2-2}.
LBM_HD constexpr double mrt_meq_coef(int basis, int t, int k) {
    const int a = t % 3, b = (t / 3) % 3, c = t / 9;
    if (basis == kMrtRef) {
        constexpr double cs2 = 1.0 / 3.0, cs4 = cs2 * cs2, cs6 = cs2 * cs2 * cs2;
        switch (t) {
            case 0: return k == 0 ? 1.0 : 0.0;
            case 1: return k == 1 ? 1.0 : 0.0;
            case 3: return k == 2 ? 1.0 : 0.0;
            case 9: return k == 3 ? 1.0 : 0.0;
            case 4: return k == 7 ? 1.0 : 0.0;
            case 10: return k == 8 ? 1.0 : 0.0;
            case 12: return k == 9 ? 1.0 : 0.0;
            case 2: return k == 0 ? cs2 : (k == 4 ? 1.0 : 0.0);
            case 6: return k == 0 ? cs2 : (k == 5 ? 1.0 : 0.0);
            case 18: return k == 0 ? cs2 : (k == 6 ? 1.0 : 0.0);
            case 7: case 19: return k == 1 ? cs2 : 0.0;
            case 5: case 21: return k == 2 ? cs2 : 0.0;
            case 11: case 15: return k == 3 ? cs2 : 0.0;
            case 13: return 0.0;
            case 8: return k == 0 ? cs4 : ((k == 4 || k == 5) ? cs2 : 0.0);
            case 20: return k == 0 ? cs4 : ((k == 4 || k == 6) ? cs2 : 0.0);
            case 24: return k == 0 ? cs4 : ((k == 5 || k == 6) ? cs2 : 0.0);
            case 14: return k == 9 ? cs2 : 0.0;
            case 16: return k == 8 ? cs2 : 0.0;
            case 22: return k == 7 ? cs2 : 0.0;
            case 25: return k == 1 ? cs4 : 0.0;
            case 23: return k == 2 ? cs4 : 0.0;
            case 17: return k == 3 ? cs4 : 0.0;
            case 26: return k == 10 ? 1.0 : (k == 0 ? cs6 : 0.0);
            default: return 0.0;
        }
    }
    const double p[3] = {1.0, 0.0, -1.0}, q[3] = {0.0, 1.0 / 3.0, 0.0}, r[3] = {1.0 / 3.0, 0.0, 1.0 / 3.0};
    const double P = p[a] * p[b] * p[c];
    switch (k) {
        case 0: return P;
        case 1: return 3.0 * q[a] * p[b] * p[c];
        case 2: return 3.0 * p[a] * q[b] * p[c];
        case 3: return 3.0 * p[a] * p[b] * q[c];
        case 4: return -1.5 * P + 4.5 * r[a] * p[b] * p[c];
        case 5: return -1.5 * P + 4.5 * p[a] * r[b] * p[c];
        case 6: return -1.5 * P + 4.5 * p[a] * p[b] * r[c];
        case 7: return 9.0 * q[a] * q[b] * p[c];
        case 8: return 9.0 * q[a] * p[b] * q[c];
        case 9: return 9.0 * p[a] * q[b] * q[c];
        default: return 0.0;
    }
}

// s - 2v as one fused multiply-add: 2v is exact, so this rounds exactly like the two-operation
// form, but stays one instruction (the compiler turns 2v into v + v otherwise).
template <class R>
LBM_HD R minus_twice(R s, R v) {
    return mad(R(-2), v, s);
}

template <int BASIS, class R>
LBM_HD void mrt_fwd3(R& v0, R& v1, R& v2) {
    // v0, v1, v2 = populations at c = -1, 0, +1 along one axis
    const R s = v0 + v2, d = v2 - v0;
    const R m0 = s + v1;
    const R m2 = BASIS == kMrtRef ? s : minus_twice(s, v1);
    v0 = m0;
    v1 = d;
    v2 = m2;
}

template <int BASIS, class R>
LBM_HD void mrt_inv3(R& m0, R& m1, R& m2) {
    // inverse of mrt_fwd3 after the per-axis scale has been applied
    const R v1 = minus_twice(m0, m2);
    const R t = BASIS == kMrtRef ? m2 : m0 + m2;
    const R v0 = t - m1, v2 = t + m1;
    m0 = v0;
    m1 = v1;
    m2 = v2;
}

// Forward tensor transform in place (slots -> moments).
template <int BASIS, class R>
LBM_HD void mrt_forward(R (&T)[27]) {
    static_for<9>([&](auto L) {  // x lines
        constexpr int o = 3 * L;
        mrt_fwd3<BASIS>(T[o], T[o + 1], T[o + 2]);
    });
    static_for<9>([&](auto L) {  // y lines
        constexpr int o = (L % 3) + 9 * (L / 3);
        mrt_fwd3<BASIS>(T[o], T[o + 3], T[o + 6]);
    });
    static_for<9>([&](auto L) {  // z lines
        constexpr int o = L;
        mrt_fwd3<BASIS>(T[o], T[o + 9], T[o + 18]);
    });
}

template <int BASIS, class R>
LBM_HD void mrt_inverse(R (&T)[27]) {
    static_for<9>([&](auto L) {
        constexpr int o = L;
        mrt_inv3<BASIS>(T[o], T[o + 9], T[o + 18]);
    });
    static_for<9>([&](auto L) {
        constexpr int o = (L % 3) + 9 * (L / 3);
        mrt_inv3<BASIS>(T[o], T[o + 3], T[o + 6]);
    });
    static_for<9>([&](auto L) {
        constexpr int o = 3 * L;
        mrt_inv3<BASIS>(T[o], T[o + 1], T[o + 2]);
    });
}

// Relaxation coefficients of one lattice: T'[t] = alpha[t] T[t] + beta[t] meq[t] for unmixed
// slots, and a 3x3 pair (A, B) for the mixed slots (2, 6, 18).  Scales of the inverse included.
// The conserved slots (rho and j: tensor slots 0, 1, 3, 9) also carry their rate s and slot scale d
// (the inverse's per-axis scales, e.g. 1/27 and 1/18 for the Gram-Schmidt basis) as d = dhi + dlo in
// two floats: see mrt_relax.
template <class R>
struct MrtCoef {
    R alpha[27], beta[27], A[9], B[9];
    R cs[4], chi[4], clo[4];
};
LBM_HD constexpr int mrt_conserved_index(int t) { return t == 0 ? 0 : t == 1 ? 1 : t == 3 ? 2 : t == 9 ? 3 : -1; }

// Coefficients of the two-rate Gram-Schmidt collision (mrt2_collide in kernels.cuh): every row relaxes
// at s_o except the five shear rows (4-6: cx cy, cx cz, cy cz; 8, 9: the traceless second-order
// mixes), which relax at s_v.  Storage units folded in (sc: the storage scale).
//   om1        1 - s_o
//   kxy, k8, k9  (s_v - s_o) / |row|^2 for the off-diagonal rows (12), row 8 (108 / 3) and row 9 (324 / 3)
//   sw[c]      s_o w_c sc for the weight classes c = rest, face, edge, corner; sw45 = 4.5 sw, sw3 = 3 sw
template <class R>
struct Mrt2Coef {
    R om1, kxy, k8, k9;
    R sw[4], sw45[4], sw3[4];
};

// First quantity with a nonzero coefficient in the equilibrium moment of slot t (11: none).
LBM_HD constexpr int mrt_meq_first(int basis, int t) {
    for (int k = 0; k < 11; ++k)
        if (mrt_meq_coef(basis, t, k) != 0.0) return k;
    return 11;
}

// Equilibrium moment of slot T from the cell quantities q[0..10]: a chain of explicit multiply-adds
// (unit coefficients as plain adds), the same IEEE operations for every real type.
template <int BASIS, int T, class R>
LBM_HD R mrt_meq(const R (&q)[11]) {
    constexpr int k0 = mrt_meq_first(BASIS, T);
    if constexpr (k0 == 11) {
        return R(0);
    } else {
        constexpr double c0 = mrt_meq_coef(BASIS, T, k0);
        R acc;
        if constexpr (c0 == 1.0)
            acc = q[k0];
        else if constexpr (c0 == -1.0)
            acc = -q[k0];
        else
            acc = R(c0) * q[k0];
        static_for<11>([&](auto K) {
            constexpr int kk = K;
            constexpr double c = mrt_meq_coef(BASIS, T, kk);
            if constexpr (kk > k0 && c != 0.0) {
                if constexpr (c == 1.0)
                    acc = acc + q[kk];
                else if constexpr (c == -1.0)
                    acc = acc - q[kk];
                else
                    acc = mad(R(c), q[kk], acc);
            }
        });
        return acc;
    }
}

// m* = relaxed, scaled moments.  q: cell quantities for the equilibrium.  K: coefficient type (the
// scalar of R).
// EXACT (FP32 storage): the conserved slots relax as d * (T + s (meq - T)) with d applied as two floats.
// alpha + beta of a single-float pair differs from the slot scale d by ~1e-8 whenever d is not a power
// of two (every Gram-Schmidt slot: 1/27, 1/18, ...), and a conserved moment has no restoring force, so
// that scale error compounds step after step: the FP32 MRT cavity's velocity drifted 1.2e-4 from FP64
// over 5,000 steps (256^3, config rates).  The other slots relax towards their equilibria, where a scale
// error of 1e-8 only shifts the relaxation rate by as much.
template <int BASIS, bool EXACT = false, class R, class K>
LBM_HD void mrt_relax(R (&T)[27], const R (&q)[11], const MrtCoef<K>& k) {
    static_for<27>([&](auto TI) {
        constexpr int t = TI;
        if constexpr (mrt_slot_row(t) >= 0) {
            const R e = mrt_meq<BASIS, t>(q);
            constexpr int ci = mrt_conserved_index(t);
            if constexpr (EXACT && ci >= 0) {
                const R x = mad(R(k.cs[ci]), e - T[t], T[t]);
                T[t] = mad(R(k.chi[ci]), x, R(k.clo[ci]) * x);
            } else {
                T[t] = mad(R(k.alpha[t]), T[t], R(k.beta[t]) * e);
            }
        }
    });
    const R a = T[2], b = T[6], c = T[18];
    const R ea = mrt_meq<BASIS, 2>(q), eb = mrt_meq<BASIS, 6>(q), ec = mrt_meq<BASIS, 18>(q);
    auto mix = [&](int r) {
        R acc = R(k.A[3 * r]) * a;
        acc = mad(R(k.A[3 * r + 1]), b, acc);
        acc = mad(R(k.A[3 * r + 2]), c, acc);
        acc = mad(R(k.B[3 * r]), ea, acc);
        acc = mad(R(k.B[3 * r + 1]), eb, acc);
        return mad(R(k.B[3 * r + 2]), ec, acc);
    };
    const R n2 = mix(0), n6 = mix(1), n18 = mix(2);
    T[2] = n2;
    T[6] = n6;
    T[18] = n18;
}

}  // namespace lbm
