// Device building blocks of the spline push/pull path: storage types,
// boundary index/sign maps and centred B-spline weights (orders 0-7) with
// their first and second derivatives.
//
// Semantics follow nitorch's compiled backend:
//   index / sign maps  : nitorch/_C/src/impl/bounds_common.h:26-133,193-219
//   spline polynomials : nitorch/_C/src/impl/interpolation_common.h:57-815
//   support (low node) : interpolation_common.h bounds0..7 (round for
//                        order 0, floor of x - (p-1)/2 otherwise)
// The B-spline pieces are the standard centred B-spline polynomials; second
// derivatives for orders >= 5 use  B''_p(x) = B_{p-2}(x+1) - 2 B_{p-2}(x)
// + B_{p-2}(x-1)  (the reference leaves them at zero).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace ppk {

// Bound codes: identical to nitorch/_C/src/bounds.h (BoundType).
enum Bound : int {
  BND_REPLICATE = 0, BND_DCT1 = 1, BND_DCT2 = 2, BND_DST1 = 3,
  BND_DST2 = 4, BND_DFT = 5, BND_SLIDING = 6, BND_ZERO = 7
};

// ---------------------------------------------------------------------
// Storage <-> compute conversions
// ---------------------------------------------------------------------
template <class S> struct Acc { using type = float; };
template <> struct Acc<double> { using type = double; };

__device__ __forceinline__ float to_acc(float v) { return v; }
__device__ __forceinline__ double to_acc(double v) { return v; }
__device__ __forceinline__ float to_acc(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_acc(__half v) { return __half2float(v); }

template <class S> __device__ __forceinline__ S from_acc(float v);
template <> __device__ __forceinline__ float from_acc<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_acc<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __half from_acc<__half>(float v) { return __float2half_rn(v); }
template <class S> __device__ __forceinline__ S from_acc(double v);
template <> __device__ __forceinline__ double from_acc<double>(double v) { return v; }

// Read-only cached load of one storage element, converted to compute type.
template <class S>
__device__ __forceinline__ typename Acc<S>::type ldg_acc(const S* p) { return to_acc(__ldg(p)); }

// Atomic accumulation in compute type (push / count outputs are always
// float or double: 16-bit storage pushes accumulate into a float buffer).
__device__ __forceinline__ void atomic_acc(float* p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_acc(double* p, double v) { atomicAdd(p, v); }

// ---------------------------------------------------------------------
// Boundary conditions (bounds_common.h). I is int32_t or int64_t.
// ---------------------------------------------------------------------
template <class I>
__device__ __forceinline__ I bound_index(int b, I i, I n) {
  switch (b) {
    case BND_REPLICATE:
      return i <= 0 ? I(0) : (i >= n ? n - 1 : i);
    case BND_DCT1: {                               // reflect about centres
      if (n == 1) return 0;
      I p = (n - 1) * 2;
      i = i < 0 ? -i : i;
      i = i % p;
      return i >= n ? p - i : i;
    }
    case BND_DCT2: case BND_DST2: {                // reflect about edges
      I p = n * 2;
      i = i < 0 ? p - ((-i - 1) % p) - 1 : i % p;
      return i >= n ? p - i - 1 : i;
    }
    case BND_DST1: {                               // antisymmetric, centres
      if (n == 1) return 0;
      I p = (n + 1) * 2;
      i = i == -1 ? I(0) : (i < 0 ? -i - 2 : i);
      i = i % p;
      return i == n ? n - 1 : (i > n ? p - i - 2 : i);
    }
    case BND_DFT:
      return i < 0 ? (n + i % n) % n : i % n;
    default:
      return i;
  }
}

template <class I>
__device__ __forceinline__ int bound_sign(int b, I i, I n) {
  switch (b) {
    case BND_DST1: {
      if (n == 1) return 1;
      I p = (n + 1) * 2;
      i = i < 0 ? n - i - 1 : i;
      i = i % p;
      if (i % (n + 1) == n) return 0;
      return ((i / (n + 1)) % 2) ? -1 : 1;
    }
    case BND_DST2:
      i = i < 0 ? n - i - 1 : i;
      return ((i / n) % 2) ? -1 : 1;
    case BND_ZERO:
      return (i < 0 || i >= n) ? 0 : 1;
    default:
      return 1;
  }
}

// ---------------------------------------------------------------------
// B-spline pieces. x is the signed distance node - sample, |x| inside the
// support (the callers only evaluate nodes of the support).
// ---------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T bs_weight(int order, T x) {
  x = fabs(x);
  switch (order) {
    case 0: return T(1);
    case 1: return T(1) - x;
    case 2:
      if (x < T(0.5)) return T(0.75) - x * x;
      x = T(1.5) - x; return T(0.5) * x * x;
    case 3:
      if (x < T(1)) return (x * x * (x - T(2)) * T(3) + T(4)) * T(1.0 / 6.0);
      x = T(2) - x; return x * x * x * T(1.0 / 6.0);
    case 4:
      if (x < T(0.5)) { x *= x; return x * (x * T(0.25) - T(0.625)) + T(115.0 / 192.0); }
      if (x < T(1.5)) return x * (x * (x * (T(5) - x) * T(1.0 / 6.0) - T(1.25)) + T(5.0 / 24.0)) + T(55.0 / 96.0);
      x -= T(2.5); x *= x; return x * x * T(1.0 / 24.0);
    case 5:
      if (x < T(1)) { T f = x * x; return f * (f * (T(0.25) - x * T(1.0 / 12.0)) - T(0.5)) + T(0.55); }
      if (x < T(2)) return x * (x * (x * (x * (x * T(1.0 / 24.0) - T(0.375)) + T(1.25)) - T(1.75)) + T(0.625)) + T(0.425);
      { T f = T(3) - x; x = f * f; return f * x * x * T(1.0 / 120.0); }
    case 6:
      if (x < T(0.5)) { x *= x;
        return x * (x * (T(7.0 / 48.0) - x * T(1.0 / 36.0)) - T(77.0 / 192.0)) + T(5887.0 / 11520.0); }
      if (x < T(1.5))
        return x * (x * (x * (x * (x * (x * T(1.0 / 48.0) - T(7.0 / 48.0)) + T(0.328125))
               - T(35.0 / 288.0)) - T(91.0 / 256.0)) - T(7.0 / 768.0)) + T(7861.0 / 15360.0);
      if (x < T(2.5))
        return x * (x * (x * (x * (x * (T(7.0 / 60.0) - x * T(1.0 / 120.0)) - T(0.65625))
               + T(133.0 / 72.0)) - T(2.5703125)) + T(1267.0 / 960.0)) + T(1379.0 / 7680.0);
      x -= T(3.5); x *= x * x; return x * x * T(1.0 / 720.0);
    default:  // 7
      if (x < T(1)) { T f = x * x;
        return f * (f * (f * (x * T(1.0 / 144.0) - T(1.0 / 36.0)) + T(1.0 / 9.0)) - T(1.0 / 3.0)) + T(151.0 / 315.0); }
      if (x < T(2))
        return x * (x * (x * (x * (x * (x * (T(0.05) - x * T(1.0 / 240.0)) - T(7.0 / 30.0))
               + T(0.5)) - T(7.0 / 18.0)) - T(0.1)) - T(7.0 / 90.0)) + T(103.0 / 210.0);
      if (x < T(3))
        return x * (x * (x * (x * (x * (x * (x * T(1.0 / 720.0) - T(1.0 / 36.0)) + T(7.0 / 30.0))
               - T(19.0 / 18.0)) + T(49.0 / 18.0)) - T(23.0 / 6.0)) + T(217.0 / 90.0)) - T(139.0 / 630.0);
      { T f = T(4) - x; x = f * f * f; return x * x * f * T(1.0 / 5040.0); }
  }
}

// Weight with support test (0 outside), used for derivative identities.
template <class T>
__device__ __forceinline__ T bs_weight_full(int order, T x) {
  T a = fabs(x);
  if (a >= T(0.5) * T(order + 1)) return T(0);
  return bs_weight(order, x);
}

template <class T>
__device__ __forceinline__ T bs_grad(int order, T x) {
  bool neg = x < T(0);
  if (neg) x = -x;
  T r;
  switch (order) {
    case 0: return T(0);
    case 1: return neg ? T(1) : T(-1);
    case 2: r = x < T(0.5) ? T(-2) * x : x - T(1.5); break;
    case 3:
      if (x < T(1)) r = x * (x * T(1.5) - T(2));
      else { T t = T(2) - x; r = -(t * t) * T(0.5); }
      break;
    case 4:
      if (x < T(0.5)) r = x * (x * x - T(1.25));
      else if (x < T(1.5)) r = x * (x * (x * T(-2.0 / 3.0) + T(2.5)) - T(2.5)) + T(5.0 / 24.0);
      else { T t = x * T(2) - T(5); r = t * t * t * T(1.0 / 48.0); }
      break;
    case 5:
      if (x < T(1)) r = x * (x * (x * (x * T(-5.0 / 12.0) + T(1))) - T(1));
      else if (x < T(2)) r = x * (x * (x * (x * T(5.0 / 24.0) - T(1.5)) + T(3.75)) - T(3.5)) + T(0.625);
      else { T t = x - T(3); t *= t; r = -(t * t) * T(1.0 / 24.0); }
      break;
    case 6:
      if (x < T(0.5)) { T x2 = x * x; r = x * (x2 * T(7.0 / 12.0) - x2 * x2 * T(1.0 / 6.0) - T(77.0 / 96.0)); }
      else if (x < T(1.5))
        r = x * (x * (x * (x * (x * T(0.125) - T(35.0 / 48.0)) + T(1.3125)) - T(35.0 / 96.0)) - T(0.7109375)) - T(7.0 / 768.0);
      else if (x < T(2.5))
        r = x * (x * (x * (x * (x * T(-1.0 / 20.0) + T(7.0 / 12.0)) - T(2.625)) + T(133.0 / 24.0)) - T(5.140625)) + T(1267.0 / 960.0);
      else { T t = x * T(2) - T(7); T t2 = t * t; r = t2 * t2 * t * T(1.0 / 3840.0); }
      break;
    default:  // 7
      if (x < T(1)) { T x2 = x * x;
        r = x * (x2 * (x2 * (x * T(7.0 / 144.0) - T(1.0 / 6.0)) + T(4.0 / 9.0)) - T(2.0 / 3.0)); }
      else if (x < T(2))
        r = x * (x * (x * (x * (x * (x * T(-7.0 / 240.0) + T(3.0 / 10.0)) - T(7.0 / 6.0)) + T(2)) - T(7.0 / 6.0)) - T(1.0 / 5.0)) - T(7.0 / 90.0);
      else if (x < T(3))
        r = x * (x * (x * (x * (x * (x * T(7.0 / 720.0) - T(1.0 / 6.0)) + T(7.0 / 6.0)) - T(38.0 / 9.0)) + T(49.0 / 6.0)) - T(23.0 / 3.0)) + T(217.0 / 90.0);
      else { T t = x - T(4); T t3 = t * t * t; r = -(t3 * t3) * T(1.0 / 720.0); }
      break;
  }
  return neg ? -r : r;
}

template <class T>
__device__ __forceinline__ T bs_hess(int order, T x) {
  T a = fabs(x);
  switch (order) {
    case 0: case 1: return T(0);
    case 2: return a < T(0.5) ? T(-2) : T(1);
    case 3: return a < T(1) ? a * T(3) - T(2) : T(2) - a;
    case 4:
      if (a < T(0.5)) return a * a * T(3) - T(1.25);
      if (a < T(1.5)) return a * (a * T(-2) + T(5)) - T(2.5);
      { T t = a * T(2) - T(5); return t * t * T(0.125); }
    default:
      return bs_weight_full(order - 2, x + T(1)) - T(2) * bs_weight_full(order - 2, x)
           + bs_weight_full(order - 2, x - T(1));
  }
}

// Lowest support node.  Odd orders: floor(x) - (p-1)/2 (exact).  Even orders
// subtract a half in double, like the reference (whose double literals
// promote the float coordinate), so the node choice is bit-identical.
template <class I, class T>
__device__ __forceinline__ I support_low(int order, T x) {
  switch (order) {
    case 0: return static_cast<I>(round(x));
    case 1: return static_cast<I>(floor(x));
    case 3: return static_cast<I>(floor(x)) - 1;
    case 5: return static_cast<I>(floor(x)) - 2;
    case 7: return static_cast<I>(floor(x)) - 3;
    case 2: return static_cast<I>(floor(static_cast<double>(x) - 0.5));
    case 4: return static_cast<I>(floor(static_cast<double>(x) - 1.5));
    default: return static_cast<I>(floor(static_cast<double>(x) - 2.5));  // 6
  }
}

// Out-of-bound test of the compiled backend: inside [-tol, n-1+tol) with
// tol = 0.05 (or 0.55 with the half-voxel flag), in the grid's precision.
// nitorch/_C/src/impl/bounds_common.h:168-171, pushpull_common.cpp:58,895-918.
template <class T>
__device__ __forceinline__ bool in_fov(T x, int64_t n, T tol) {
  return x >= -tol && x < static_cast<T>(n - 1) + tol;
}

}  // namespace ppk
