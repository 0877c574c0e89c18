// Device arithmetic for the block engine: float64, double-double in the two flavours KBSRC uses, and x87
// extended (x80.cuh) for Precision::LongDouble.
//
// Output must be byte-identical to the reference CPU engines, so every value is produced by the same IEEE
// operations in the same order (HongYue1/KBSRC src/dsp/double_double.hpp:59-79, src/dsp/simd.hpp:44-66).
// All operations are explicit round-to-nearest intrinsics, never contracted (the build also passes
// -fmad=false); the only fused multiply-add is the exact product error of the dd product.
#pragma once
#include <cuda_runtime.h>

#include "x80.cuh"

// Launch shapes the shared-memory passes are compiled for: at most KB_MAXT_* threads per CTA and KB_MINB_*
// resident CTAs per SM, which caps registers at 64K / (threads * CTAs). Double-double: 192 x 3 (96 registers,
// 18 warps per SM, measured fastest) for the row and direct passes, 320 x 2 for the column passes (their shared
// memory allows two CTAs: 20 warps per SM; C2 forward column 1.16 -> 1.05 ms, while the row passes lose with
// it); f64: 256 x 3 (80 registers); x87 extended: 192 x 2 (170 registers: the integer emulation holds 128-bit
// intermediates).
#ifndef KB_MINB_DD
#define KB_MINB_DD 3
#endif
#ifndef KB_MAXT_DD
#define KB_MAXT_DD 192
#endif
#ifndef KB_MINB_DD_COL
#define KB_MINB_DD_COL 2
#endif
#ifndef KB_MAXT_DD_COL
#define KB_MAXT_DD_COL 320
#endif
#ifndef KB_MINB_X80
#define KB_MINB_X80 2
#endif
#ifndef KB_MAXT_X80
#define KB_MAXT_X80 192
#endif
#ifndef KB_MINB_F64
#define KB_MINB_F64 3
#endif
#ifndef KB_MAXT_F64
#define KB_MAXT_F64 256
#endif

namespace kbsrc::dev {

struct alignas(16) dd {
    double hi, lo;
};

// Complex value in registers or shared/global memory. 16 B for f64, 32 B for dd; 16-byte aligned so that
// shared and global accesses are 128-bit.
template <class R>
struct alignas(16) cx {
    R re, im;
};

__device__ __forceinline__ dd make_dd(double h, double l) { return dd{h, l}; }

// quick two-sum: s = a + b, low part b - (s - a)
__device__ __forceinline__ dd qts(double a, double b) {
    const double s = __dadd_rn(a, b);
    return dd{s, __dsub_rn(b, __dsub_rn(s, a))};
}
// two-sum: exact error of a + b for any a, b
__device__ __forceinline__ dd two_sum(double a, double b) {
    const double s = __dadd_rn(a, b), v = __dsub_rn(s, a);
    return dd{s, __dadd_rn(__dsub_rn(a, __dsub_rn(s, v)), __dsub_rn(b, v))};
}
__device__ __forceinline__ dd dd_neg(dd a) { return dd{-a.hi, -a.lo}; }
// negation of a table value (exact, both parts)
__device__ __forceinline__ double w_neg(double a) { return -a; }
__device__ __forceinline__ dd w_neg(dd a) { return dd_neg(a); }
__device__ __forceinline__ x80 w_neg(x80 a) { return x80_neg(a); }

// Accurate sum of the scalar dd type (double_double.hpp:67-70): two two-sums and two renormalisations.
__device__ __forceinline__ dd add_accurate(dd a, dd b) {
    dd h = two_sum(a.hi, b.hi);
    const dd l = two_sum(a.lo, b.lo);
    h.lo = __dadd_rn(h.lo, l.hi);
    h = qts(h.hi, h.lo);
    h.lo = __dadd_rn(h.lo, l.lo);
    return qts(h.hi, h.lo);
}
// Short sum of the reference's 4-lane DD4 type (simd.hpp:44-49): one two-sum, low parts added, one
// renormalisation. Used by its four-step sub-FFTs.
__device__ __forceinline__ dd add_short(dd a, dd b) {
    const double s = __dadd_rn(a.hi, b.hi), v = __dsub_rn(s, a.hi);
    double e = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, v)), __dsub_rn(b.hi, v));
    e = __dadd_rn(e, __dadd_rn(a.lo, b.lo));
    return qts(s, e);
}
// Product (double_double.hpp:73-76): the error of hi*hi by fma, then the cross terms.
__device__ __forceinline__ dd mul_dd(dd a, dd b) {
    const double p = __dmul_rn(a.hi, b.hi);
    double e = __fma_rn(a.hi, b.hi, -p);
    e = __dadd_rn(e, __dadd_rn(__dmul_rn(a.hi, b.lo), __dmul_rn(a.lo, b.hi)));
    return qts(p, e);
}

// Arithmetic flavours. R: register type, W: table (twiddle / kernel) type.
// kLanes: used by the reference's 4-lane four-step, whose twiddle multiply includes column 0
// (fft.hpp:294); the 1-lane four-step skips it (fft.hpp:293). kLaneRenorm: four-step results are stored
// through qts(hi, lo) (fft.hpp:200-204). kWide: the real type is wider than float64, so the RFFT split and merge
// take conjugate pairs together (the reference's non-double branch, fft.hpp:374-407,417-457), and the passes stage
// their sub-FFT twiddles in shared memory.
struct ArF64 {  // Precision::Fast: float64 everywhere (V4 lanes and scalar alike)
    using R = double;
    using W = double;
    static constexpr bool kLanes = true, kLaneRenorm = false, kWide = false;
    static constexpr int kMinBlocks = KB_MINB_F64, kMaxThreads = KB_MAXT_F64;
    static constexpr int kColMinBlocks = KB_MINB_F64, kColMaxThreads = KB_MAXT_F64;
    static __device__ __forceinline__ R add(R a, R b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ R sub(R a, R b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ R mul(R a, R b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ R neg(R a) { return -a; }
    static __device__ __forceinline__ R zero() { return 0.0; }
    static __device__ __forceinline__ R from_w(W w) { return w; }
    static __device__ __forceinline__ R from_f64(double v) { return v; }
    static __device__ __forceinline__ double to_f64(R v) { return v; }
    static __device__ __forceinline__ R renorm(R v) { return v; }
};
struct ArDDShort {  // four-step sub-FFTs of Precision::Exact (DD4 lanes)
    using R = dd;
    using W = dd;
    static constexpr bool kLanes = true, kLaneRenorm = true, kWide = true;
    static constexpr int kMinBlocks = KB_MINB_DD, kMaxThreads = KB_MAXT_DD;
    static constexpr int kColMinBlocks = KB_MINB_DD_COL, kColMaxThreads = KB_MAXT_DD_COL;
    static __device__ __forceinline__ R add(R a, R b) { return add_short(a, b); }
    static __device__ __forceinline__ R sub(R a, R b) { return add_short(a, dd_neg(b)); }
    static __device__ __forceinline__ R mul(R a, R b) { return mul_dd(a, b); }
    static __device__ __forceinline__ R neg(R a) { return dd_neg(a); }
    static __device__ __forceinline__ R zero() { return dd{0.0, 0.0}; }
    static __device__ __forceinline__ R from_w(W w) { return w; }
    static __device__ __forceinline__ R from_f64(double v) { return dd{v, 0.0}; }
    static __device__ __forceinline__ double to_f64(R v) { return __dadd_rn(v.hi, v.lo); }
    // lane results leave the DD4 registers through qts(hi, lo) (fft.hpp:200-204)
    static __device__ __forceinline__ R renorm(R v) { return qts(v.hi, v.lo); }
};
struct ArDDAccurate {  // scalar dd: direct SFFT, Bluestein, RFFT split/merge, spectrum, kernel design
    using R = dd;
    using W = dd;
    static constexpr bool kLanes = false, kLaneRenorm = false, kWide = true;
    static constexpr int kMinBlocks = KB_MINB_DD, kMaxThreads = KB_MAXT_DD;
    static constexpr int kColMinBlocks = KB_MINB_DD_COL, kColMaxThreads = KB_MAXT_DD_COL;
    static __device__ __forceinline__ R add(R a, R b) { return add_accurate(a, b); }
    static __device__ __forceinline__ R sub(R a, R b) { return add_accurate(a, dd_neg(b)); }
    static __device__ __forceinline__ R mul(R a, R b) { return mul_dd(a, b); }
    static __device__ __forceinline__ R neg(R a) { return dd_neg(a); }
    static __device__ __forceinline__ R zero() { return dd{0.0, 0.0}; }
    static __device__ __forceinline__ R from_w(W w) { return w; }
    static __device__ __forceinline__ R from_f64(double v) { return dd{v, 0.0}; }
    static __device__ __forceinline__ double to_f64(R v) { return __dadd_rn(v.hi, v.lo); }
    static __device__ __forceinline__ R renorm(R v) { return qts(v.hi, v.lo); }
};

struct ArX80 {  // Precision::LongDouble: x87 extended everywhere, one lane (CFFT<long double, long double, long double>)
    using R = x80;
    using W = x80;
    static constexpr bool kLanes = false, kLaneRenorm = false, kWide = true;
    static constexpr int kMinBlocks = KB_MINB_X80, kMaxThreads = KB_MAXT_X80;
    static constexpr int kColMinBlocks = KB_MINB_X80, kColMaxThreads = KB_MAXT_X80;
    static __device__ __forceinline__ R add(R a, R b) { return x80_add(a, b); }
    static __device__ __forceinline__ R sub(R a, R b) { return x80_sub(a, b); }
    static __device__ __forceinline__ R mul(R a, R b) { return x80_mul(a, b); }
    static __device__ __forceinline__ R neg(R a) { return x80_neg(a); }
    static __device__ __forceinline__ R zero() { return x80{0ull, 0, 0}; }
    static __device__ __forceinline__ R from_w(W w) { return w; }
    static __device__ __forceinline__ R from_f64(double v) { return x80_from_f64(v); }
    static __device__ __forceinline__ double to_f64(R v) { return x80_to_f64(v); }
    static __device__ __forceinline__ R renorm(R v) { return v; }
};

template <class Ar>
using CxR = cx<typename Ar::R>;
template <class Ar>
using CxW = cx<typename Ar::W>;

template <class Ar>
__device__ __forceinline__ CxR<Ar> c_add(CxR<Ar> a, CxR<Ar> b) {
    return {Ar::add(a.re, b.re), Ar::add(a.im, b.im)};
}
template <class Ar>
__device__ __forceinline__ CxR<Ar> c_sub(CxR<Ar> a, CxR<Ar> b) {
    return {Ar::sub(a.re, b.re), Ar::sub(a.im, b.im)};
}
template <class Ar>
__device__ __forceinline__ CxR<Ar> c_conj(CxR<Ar> a) {
    return {a.re, Ar::neg(a.im)};
}
// a * (-i)
template <class Ar>
__device__ __forceinline__ CxR<Ar> c_mul_mi(CxR<Ar> a) {
    return {a.im, Ar::neg(a.re)};
}
// {a.re b.re - a.im b.im, a.re b.im + a.im b.re} (fft.hpp:46-51)
template <class Ar>
__device__ __forceinline__ CxR<Ar> c_mul(CxR<Ar> a, CxR<Ar> b) {
    return {Ar::sub(Ar::mul(a.re, b.re), Ar::mul(a.im, b.im)), Ar::add(Ar::mul(a.re, b.im), Ar::mul(a.im, b.re))};
}
template <class Ar>
__device__ __forceinline__ CxR<Ar> c_mulw(CxR<Ar> a, CxW<Ar> w) {
    return c_mul<Ar>(a, CxR<Ar>{Ar::from_w(w.re), Ar::from_w(w.im)});
}
template <class Ar>
__device__ __forceinline__ CxR<Ar> c_scale(CxR<Ar> a, typename Ar::R h) {
    return {Ar::mul(a.re, h), Ar::mul(a.im, h)};
}
template <class Ar>
__device__ __forceinline__ CxR<Ar> c_renorm(CxR<Ar> a) {
    return {Ar::renorm(a.re), Ar::renorm(a.im)};
}

}  // namespace kbsrc::dev
