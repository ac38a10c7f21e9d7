// Shared device/host helpers for the B200 transposition kernels.
//
// Element arithmetic restates the update rules of TTC's reference loop and CUDA kernels
// (GPUreference.py:90-137, CUDAtranspose.py:801-961):
//   real:     B = alpha*A + beta*B          alpha in A's precision, beta in B's precision,
//                                           C promotion: products in their own precision, the sum
//                                           in the wider one, then one rounding to B's type
//   complex:  B = cuCadd(cvt(cuCmul(alpha, A)), cuCmul(beta, B))
//             cuCmul(x, y) = (xr*yr - xi*yi, xr*yi + xi*yr), cvt = component-wise conversion
// Every operation uses the explicitly rounded intrinsics (__fmul_rn, __dadd_rn, ...), which the
// compiler never contracts into FMAs, so results are bit-identical to a C restatement compiled
// without floating-point contraction.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#ifndef TTCB_MAXR
#define TTCB_MAXR 10
#endif

// ------------------------------------------------------------------------------------------------
// Division by a run-time invariant divisor (Granlund & Montgomery, "Division by invariant integers
// using multiplication", PLDI 1994): for 1 <= d < 2^31 and 0 <= n < 2^31,
//   l = ceil(log2 d), m = floor(2^32 * (2^l - d) / d) + 1, n / d = (umulhi(n, m) + n) >> l.
// The sum cannot overflow 32 bits because umulhi(n, m) < n < 2^31.
struct FastDiv {
  uint32_t d;
  uint32_t m;
  uint32_t l;
  uint32_t pad_;
};

inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f;
  f.d = d;
  uint32_t l = 0;
  while ((1ull << l) < d) ++l;
  f.l = l;
  f.m = (uint32_t)((((1ull << l) - d) << 32) / d + 1);
  f.pad_ = 0;
  return f;
}

__host__ __device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
#ifdef __CUDA_ARCH__
  return (__umulhi(n, f.m) + n) >> f.l;
#else
  return (uint32_t)((((uint64_t)n * f.m) >> 32) + n) >> f.l;
#endif
}

// ------------------------------------------------------------------------------------------------
// Element types: float, double, float2 (float complex), double2 (double complex).
template <typename T> struct ElemInfo;
template <> struct ElemInfo<float>   { static constexpr int bytes = 4;  static constexpr bool cplx = false; };
template <> struct ElemInfo<double>  { static constexpr int bytes = 8;  static constexpr bool cplx = false; };
template <> struct ElemInfo<float2>  { static constexpr int bytes = 8;  static constexpr bool cplx = true; };
template <> struct ElemInfo<double2> { static constexpr int bytes = 16; static constexpr bool cplx = true; };

// alpha * a in A's precision
__device__ __forceinline__ float scale_a(float al, float a) { return __fmul_rn(al, a); }
__device__ __forceinline__ double scale_a(double al, double a) { return __dmul_rn(al, a); }
__device__ __forceinline__ float2 scale_a(float2 x, float2 y) {
  return make_float2(__fsub_rn(__fmul_rn(x.x, y.x), __fmul_rn(x.y, y.y)),
                     __fadd_rn(__fmul_rn(x.x, y.y), __fmul_rn(x.y, y.x)));
}
__device__ __forceinline__ double2 scale_a(double2 x, double2 y) {
  return make_double2(__dsub_rn(__dmul_rn(x.x, y.x), __dmul_rn(x.y, y.y)),
                      __dadd_rn(__dmul_rn(x.x, y.y), __dmul_rn(x.y, y.x)));
}

// B = convert(t) for beta == 0 (t = alpha*A already in A's precision)
template <typename TA, typename TB> __device__ __forceinline__ TB finish(TA t);
template <> __device__ __forceinline__ float finish<float, float>(float t) { return t; }
template <> __device__ __forceinline__ double finish<double, double>(double t) { return t; }
template <> __device__ __forceinline__ double finish<float, double>(float t) { return (double)t; }
template <> __device__ __forceinline__ float finish<double, float>(double t) { return __double2float_rn(t); }
template <> __device__ __forceinline__ float2 finish<float2, float2>(float2 t) { return t; }
template <> __device__ __forceinline__ double2 finish<double2, double2>(double2 t) { return t; }
template <> __device__ __forceinline__ double2 finish<float2, double2>(float2 t) {
  return make_double2((double)t.x, (double)t.y);
}
template <> __device__ __forceinline__ float2 finish<double2, float2>(double2 t) {
  return make_float2(__double2float_rn(t.x), __double2float_rn(t.y));
}

// B = t + beta*b with the reference's promotion rules
template <typename TA, typename TB> __device__ __forceinline__ TB combine(TA t, TB b, TB beta);
template <> __device__ __forceinline__ float combine<float, float>(float t, float b, float be) {
  return __fadd_rn(t, __fmul_rn(be, b));
}
template <> __device__ __forceinline__ double combine<double, double>(double t, double b, double be) {
  return __dadd_rn(t, __dmul_rn(be, b));
}
// sd: float product promoted, sum in double
template <> __device__ __forceinline__ double combine<float, double>(float t, double b, double be) {
  return __dadd_rn((double)t, __dmul_rn(be, b));
}
// ds: beta*b is a float product, promoted; the sum is in double and rounded once to float
template <> __device__ __forceinline__ float combine<double, float>(double t, float b, float be) {
  return __double2float_rn(__dadd_rn(t, (double)__fmul_rn(be, b)));
}
template <> __device__ __forceinline__ float2 combine<float2, float2>(float2 t, float2 b, float2 be) {
  float2 u = scale_a(be, b);
  return make_float2(__fadd_rn(t.x, u.x), __fadd_rn(t.y, u.y));
}
template <> __device__ __forceinline__ double2 combine<double2, double2>(double2 t, double2 b, double2 be) {
  double2 u = scale_a(be, b);
  return make_double2(__dadd_rn(t.x, u.x), __dadd_rn(t.y, u.y));
}
// cz: cuCadd(cuComplexFloatToDouble(t), cuCmul(beta, b))
template <> __device__ __forceinline__ double2 combine<float2, double2>(float2 t, double2 b, double2 be) {
  double2 u = scale_a(be, b);
  return make_double2(__dadd_rn((double)t.x, u.x), __dadd_rn((double)t.y, u.y));
}
// zc: cuCaddf(cuComplexDoubleToFloat(t), cuCmulf(beta, b))
template <> __device__ __forceinline__ float2 combine<double2, float2>(double2 t, float2 b, float2 be) {
  float2 u = scale_a(be, b);
  return make_float2(__fadd_rn(__double2float_rn(t.x), u.x), __fadd_rn(__double2float_rn(t.y), u.y));
}

// ------------------------------------------------------------------------------------------------
// Vectors of V elements moved as one 4/8/16-byte access.
template <typename T, int V> struct alignas(sizeof(T) * V) Vec { T v[V]; };

template <int BYTES> struct RawType;
template <> struct RawType<4> { using type = unsigned int; };
template <> struct RawType<8> { using type = uint2; };
template <> struct RawType<16> { using type = uint4; };

// Streaming (read-once) load: ld.global.cs
template <typename T, int V> __device__ __forceinline__ Vec<T, V> ld_stream(const T* p) {
  using R = typename RawType<sizeof(T) * V>::type;
  R r = __ldcs(reinterpret_cast<const R*>(p));
  Vec<T, V> out;
  static_assert(sizeof(R) == sizeof(Vec<T, V>), "vector size");
  __builtin_memcpy(&out, &r, sizeof(R));
  return out;
}

template <typename T, int V> __device__ __forceinline__ void st_vec(T* p, const Vec<T, V>& v, bool streaming) {
  using R = typename RawType<sizeof(T) * V>::type;
  R r;
  __builtin_memcpy(&r, &v, sizeof(R));
  if (streaming)
    __stcs(reinterpret_cast<R*>(p), r);
  else
    *reinterpret_cast<R*>(p) = r;
}

template <typename T> __device__ __forceinline__ T ld_scalar(const T* p) { return ld_stream<T, 1>(p).v[0]; }
template <typename T> __device__ __forceinline__ void st_scalar(T* p, T v, bool streaming) {
  Vec<T, 1> x;
  x.v[0] = v;
  st_vec<T, 1>(p, x, streaming);
}
