// arith.cuh — explicit multiply-add for the collision code.
//
// Device code is compiled without multiply-add contraction (--fmad=false), and every multiply-add of
// the collision is written as mad(a, b, c): the rounding of each kernel is then fixed by the source,
// not by the compiler's contraction choices, so every kernel family that runs the same collision
// (the one-cell-per-thread kernels, the row pipeline, the batched ensemble) rounds identically
// (tested bit-exact).  The host instantiation (lbm_mrt_collide_host) uses std::fma.
//
// A packed FP32x2 variant of the collision (two cells per thread, add/mul/fma.f32x2) was built and
// measured on B200: it executes 470 instead of 767 instructions per cell for F16S MRT, but needs ~190
// registers, so only 10 warps fit on an SM and the kernel turned latency-bound (227 vs 187 us per
// launch); the compiler also contracted packed multiply/add pairs, which broke bit-identity with the
// scalar kernels.  It is not part of the build.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "lattice.cuh"

namespace lbm {

// a * b + c with one rounding (explicit single- and double-precision intrinsics on the device: no
// promotion of float arguments to double).
LBM_HD float mad(float a, float b, float c) {
#ifdef __CUDA_ARCH__
    return __fmaf_rn(a, b, c);
#else
    return std::fmaf(a, b, c);
#endif
}
LBM_HD double mad(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

}  // namespace lbm
