// codec.cuh — how one population is held in HBM.
//
//   F32   : the population itself (the reference's f32 arrays)
//   F64   : the population itself in double; the FP64 run of the same kernel
//   F16S  : half((f_i - w_i) * scale)            "shifted" storage, FP32 arithmetic
//   BF16S : bfloat16((f_i - w_i) * scale)
// Shifting by the rest weight keeps only the deviation from rest in the 16-bit word; `scale`
// (a power of two) lifts the small deviations out of the FP16 subnormal range.
//
// The step kernels compute on deviations d = f - w as well (load_dev / store_dev): for F32/F64 the
// subtraction is exact for populations within a factor of two of their weight (Sterbenz), and
// working on the small deviations avoids the cancellation of the O(w) parts in the moment sums and
// transforms; for the 16-bit codecs the stored word already is the deviation.
// load/load_dev read global memory through the read-only path (__ldg); dev() decodes a value that
// was read by other means (e.g. from shared memory, which __ldg must not be given).
//
// The BGK and MRT step kernels use the "raw" interface: raw() gives the deviation in storage units,
// i.e. (f - w) * scale for the 16-bit codecs (no multiply) and f - w for F32/F64 (scale 1), and enc()
// stores a value given in the same units.  The collision folds `scale` (a power of two, so every
// rescaling is exact) into its per-cell constants instead of rescaling 2*Q populations.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

namespace lbm {

template <class S>
struct Codec;

template <>
struct Codec<float> {
    using Real = float;
    static constexpr int kBytes = 4;
    __device__ __forceinline__ static float load(const float* p, float, float) { return __ldg(p); }
    __device__ __forceinline__ static void store(float* p, float v, float, float) { *p = v; }
    static constexpr bool kScaled = false;
    __device__ __forceinline__ static float raw(float v, float w) { return v - w; }
    __device__ __forceinline__ static float enc(float d, float w) { return w + d; }
    __device__ __forceinline__ static float dev(float raw, float w, float) { return raw - w; }
    __device__ __forceinline__ static float load_dev(const float* p, float w, float) { return __ldg(p) - w; }
    __device__ __forceinline__ static void store_dev(float* p, float d, float w, float) { *p = w + d; }
};

template <>
struct Codec<double> {
    using Real = double;
    static constexpr int kBytes = 8;
    __device__ __forceinline__ static double load(const double* p, double, double) { return __ldg(p); }
    __device__ __forceinline__ static void store(double* p, double v, double, double) { *p = v; }
    static constexpr bool kScaled = false;
    __device__ __forceinline__ static double raw(double v, double w) { return v - w; }
    __device__ __forceinline__ static double enc(double d, double w) { return w + d; }
    __device__ __forceinline__ static double dev(double raw, double w, double) { return raw - w; }
    __device__ __forceinline__ static double load_dev(const double* p, double w, double) { return __ldg(p) - w; }
    __device__ __forceinline__ static void store_dev(double* p, double d, double w, double) { *p = w + d; }
};

template <>
struct Codec<__half> {
    using Real = float;
    static constexpr int kBytes = 2;
    __device__ __forceinline__ static float load(const __half* p, float w, float inv_scale) {
        return fmaf(__half2float(__ldg(p)), inv_scale, w);
    }
    __device__ __forceinline__ static void store(__half* p, float v, float w, float scale) {
        *p = __float2half_rn((v - w) * scale);
    }
    static constexpr bool kScaled = true;
    __device__ __forceinline__ static float raw(__half v, float) { return __half2float(v); }
    __device__ __forceinline__ static __half enc(float d, float) { return __float2half_rn(d); }
    __device__ __forceinline__ static float dev(__half raw, float, float inv_scale) {
        return __half2float(raw) * inv_scale;
    }
    __device__ __forceinline__ static float load_dev(const __half* p, float, float inv_scale) {
        return __half2float(__ldg(p)) * inv_scale;
    }
    __device__ __forceinline__ static void store_dev(__half* p, float d, float, float scale) {
        *p = __float2half_rn(d * scale);
    }
};

template <>
struct Codec<__nv_bfloat16> {
    using Real = float;
    static constexpr int kBytes = 2;
    __device__ __forceinline__ static float load(const __nv_bfloat16* p, float w, float inv_scale) {
        return fmaf(__bfloat162float(__ldg(p)), inv_scale, w);
    }
    __device__ __forceinline__ static void store(__nv_bfloat16* p, float v, float w, float scale) {
        *p = __float2bfloat16_rn((v - w) * scale);
    }
    static constexpr bool kScaled = true;
    __device__ __forceinline__ static float raw(__nv_bfloat16 v, float) { return __bfloat162float(v); }
    __device__ __forceinline__ static __nv_bfloat16 enc(float d, float) { return __float2bfloat16_rn(d); }
    __device__ __forceinline__ static float dev(__nv_bfloat16 raw, float, float inv_scale) {
        return __bfloat162float(raw) * inv_scale;
    }
    __device__ __forceinline__ static float load_dev(const __nv_bfloat16* p, float, float inv_scale) {
        return __bfloat162float(__ldg(p)) * inv_scale;
    }
    __device__ __forceinline__ static void store_dev(__nv_bfloat16* p, float d, float, float scale) {
        *p = __float2bfloat16_rn(d * scale);
    }
};

// ---- paired 16-bit conversion and stochastic rounding ------------------------------------------
// The step kernels convert a cell's outputs two at a time (directions i, i + 1) with one paired
// conversion: `a` goes to the upper half, `b` to the lower.  rn: round to nearest even (identical to
// converting each value alone).  rs: stochastic rounding (sm_100a `cvt.rs`): a value between two
// representable neighbours rounds away from zero with probability equal to its distance from the lower
// one in units of their spacing, decided by the 32-bit random word `rbits` -- unbiased, so rounding
// errors that repeat step after step (a near-steady flow recomputes the same values) do not add up
// to a drift.  Measured on B200 over 2^20 random words: 1/4 and 1/2 ulp above a value round up
// 24.9 % and 50.0 % of the time (FP16), 25.0 % and 74.9 % at 1/4 and 3/4 ulp (BF16).
template <class S>
struct Pair16;

template <>
struct Pair16<__half> {
    __device__ __forceinline__ static uint32_t rn(float a, float b) {
        uint32_t d;
        asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(a), "f"(b));
        return d;
    }
    __device__ __forceinline__ static uint32_t rs(float a, float b, uint32_t rbits) {
        uint32_t d;
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(rbits));
        return d;
    }
    __device__ __forceinline__ static __half hi(uint32_t d) { return __ushort_as_half((unsigned short)(d >> 16)); }
    __device__ __forceinline__ static __half lo(uint32_t d) { return __ushort_as_half((unsigned short)(d & 0xffffu)); }
    // the two halves of a packed pair as floats (low: the first cell)
    __device__ __forceinline__ static float lo_f(uint32_t d) {
        return __low2float(*reinterpret_cast<const __half2*>(&d));
    }
    __device__ __forceinline__ static float hi_f(uint32_t d) {
        return __high2float(*reinterpret_cast<const __half2*>(&d));
    }
};

template <>
struct Pair16<__nv_bfloat16> {
    __device__ __forceinline__ static uint32_t rn(float a, float b) {
        uint32_t d;
        asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(a), "f"(b));
        return d;
    }
    __device__ __forceinline__ static uint32_t rs(float a, float b, uint32_t rbits) {
        uint32_t d;
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(rbits));
        return d;
    }
    __device__ __forceinline__ static __nv_bfloat16 hi(uint32_t d) {
        return __ushort_as_bfloat16((unsigned short)(d >> 16));
    }
    __device__ __forceinline__ static __nv_bfloat16 lo(uint32_t d) {
        return __ushort_as_bfloat16((unsigned short)(d & 0xffffu));
    }
    // the two halves of a packed pair as floats (a bfloat16 is the top half of its float)
    __device__ __forceinline__ static float lo_f(uint32_t d) { return __uint_as_float(d << 16); }
    __device__ __forceinline__ static float hi_f(uint32_t d) { return __uint_as_float(d & 0xffff0000u); }
};

// A 32-bit integer hash (xor-shift / multiply rounds): the random words of the stochastic rounding come
// from hashing the cell index with the step's seed.
__host__ __device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

}  // namespace lbm

