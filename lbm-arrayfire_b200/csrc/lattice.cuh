// lattice.cuh — compile-time velocity sets, weights and opposites.
//
// D2Q9 ordering/weights: cpp/d2q9_bgk_lid.cpp:72-79 (opposites from nb_index_arr at :82).
// D3Q27 ordering/weights: cpp/d3q27_bgk_lid.cpp:98-107 (opposites from nb_index_arr at :111).
// The tables are constexpr functions so that every use inside the fully unrolled kernels folds to
// an immediate; nothing is read from memory.
#pragma once

#include <cstdint>
#include <utility>

#define LBM_HD __host__ __device__ __forceinline__

namespace lbm {

// Compile-time loop: f(std::integral_constant<int, 0>{}), ..., f(integral_constant<int, N-1>{}).
template <class F, int... Is>
LBM_HD constexpr void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
    (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F>
LBM_HD constexpr void static_for(F&& f) {
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

struct D2Q9 {
    static constexpr int Q = 9;
    static constexpr int DIM = 2;
    LBM_HD static constexpr int cx(int i) {
        constexpr int v[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
        return v[i];
    }
    LBM_HD static constexpr int cy(int i) {
        constexpr int v[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
        return v[i];
    }
    LBM_HD static constexpr int cz(int) { return 0; }
    LBM_HD static constexpr double w(int i) {
        return i == 0 ? 4.0 / 9.0 : (i < 5 ? 1.0 / 9.0 : 1.0 / 36.0);
    }
    LBM_HD static constexpr int opp(int i) {
        constexpr int v[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
        return v[i];
    }
};

struct D3Q27 {
    static constexpr int Q = 27;
    static constexpr int DIM = 3;
    LBM_HD static constexpr int cx(int i) {
        constexpr int v[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1,
                               -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
        return v[i];
    }
    LBM_HD static constexpr int cy(int i) {
        constexpr int v[27] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0,
                               0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1};
        return v[i];
    }
    LBM_HD static constexpr int cz(int i) {
        constexpr int v[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1,
                               -1, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1};
        return v[i];
    }
    LBM_HD static constexpr double w(int i) {
        return i == 0 ? 8.0 / 27.0 : (i < 7 ? 2.0 / 27.0 : (i < 19 ? 1.0 / 54.0 : 1.0 / 216.0));
    }
    LBM_HD static constexpr int opp(int i) {
        constexpr int v[27] = {0,  2,  1,  4,  3,  6,  5,  10, 9,  8,  7,  14, 13, 12,
                               11, 18, 17, 16, 15, 26, 25, 24, 23, 22, 21, 20, 19};
        return v[i];
    }
    // Tensor slot of direction i: (cx+1) + 3 (cy+1) + 9 (cz+1).  Used by the factorised MRT.
    LBM_HD static constexpr int slot(int i) { return (cx(i) + 1) + 3 * (cy(i) + 1) + 9 * (cz(i) + 1); }
    // The direction with velocity (x, y, z).
    LBM_HD static constexpr int dir_of(int x, int y, int z) {
        for (int i = 0; i < Q; ++i)
            if (cx(i) == x && cy(i) == y && cz(i) == z) return i;
        return -1;
    }
};

}  // namespace lbm
