// Device building blocks of the spline push/pull path: storage types,
// boundary index/sign maps and centred B-spline weights (orders 0-7) with
// their first and second derivatives.
//
// Semantics follow nitorch's compiled backend:
//   index / sign maps  : nitorch/_C/src/impl/bounds_common.h:26-133,193-219
//   spline polynomials : nitorch/_C/src/impl/interpolation_common.h:57-815
//   support (low node) : interpolation_common.h bounds0..7 (round for
//                        order 0, floor of x - (p-1)/2 otherwise)
// Weights and derivatives come from the Cox-de Boor recurrence
// (bspline_stencil); second derivatives are exact at every order (the
// reference leaves them at zero for orders 5-7).
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
// B-spline stencil of one axis.
//
// The p+1 non-zero weights of a sample are values of the cardinal B-spline
// M_p (support [0, p+1]; B_p(x) = M_p(x + (p+1)/2)) at f + i, i = 0..p,
// where f in [0,1) is the sample's offset from its support.  They are
// evaluated together by the Cox-de Boor recurrence
//     M_k(s) = ( s M_{k-1}(s) + (k+1-s) M_{k-1}(s-1) ) / k,
// whose terms are all non-negative (accurate to a few ulps at every order,
// where Horner forms of the order-7 pieces lose ~4 digits in float32).
// Derivatives use  M_p' (s) = M_{p-1}(s) - M_{p-1}(s-1)  and
// M_p''(s) = M_{p-2}(s) - 2 M_{p-2}(s-1) + M_{p-2}(s-2), i.e. the rows of
// the same recurrence at k = p-1 and k = p-2.
// Tap j sits on node low + j at signed distance dx_j = x - (low + j); its
// weight is B_p(dx_j) = M_p(f + p - j), i.e. row[p - j].
// NT: compile-time max taps (>= p+1); p may be a run-time value.
// ---------------------------------------------------------------------
template <int NT, bool NEED_G, bool NEED_H, class T>
__device__ __forceinline__ void bspline_stencil(int p, T f, T (&w)[NT], T (&g)[NT], T (&h)[NT]) {
  T b[NT + 1], c[NT + 1], d[NT + 1];
#pragma unroll
  for (int i = 0; i <= NT; ++i) { b[i] = i == 0 ? T(1) : T(0); c[i] = b[i]; d[i] = b[i]; }
#pragma unroll
  for (int k = 1; k < NT; ++k) {
    if (k <= p) {
      if (NEED_H && k == p - 1) {
#pragma unroll
        for (int i = 0; i <= NT; ++i) d[i] = b[i];
      }
      if (NEED_G && k == p) {
#pragma unroll
        for (int i = 0; i <= NT; ++i) c[i] = b[i];
      }
      const T ik = T(1) / T(k);
#pragma unroll
      for (int i = k; i >= 0; --i) {
        const T lo = i > 0 ? b[i - 1] : T(0);
        b[i] = ((f + T(i)) * b[i] + (T(k + 1 - i) - f) * lo) * ik;
      }
    }
  }
  if (NEED_H && p <= 1) {
#pragma unroll
    for (int i = 0; i <= NT; ++i) d[i] = T(0);
  }
#pragma unroll
  for (int j = 0; j < NT; ++j) {
    const int r = p - j;          // row index of tap j
    w[j] = (r >= 0) ? b[r < 0 ? 0 : r] : T(0);
    if (NEED_G) {
      const T c0 = (r >= 0 && r <= NT) ? c[r < 0 ? 0 : (r > NT ? NT : r)] : T(0);
      const T c1 = (r - 1 >= 0) ? c[r - 1 < 0 ? 0 : r - 1] : T(0);
      g[j] = p == 0 ? T(0) : c0 - c1;
    } else {
      g[j] = T(0);
    }
    if (NEED_H) {
      const T d0 = (r >= 0) ? d[r < 0 ? 0 : r] : T(0);
      const T d1 = (r - 1 >= 0) ? d[r - 1 < 0 ? 0 : r - 1] : T(0);
      const T d2 = (r - 2 >= 0) ? d[r - 2 < 0 ? 0 : r - 2] : T(0);
      h[j] = p <= 1 ? T(0) : d0 - T(2) * d1 + d2;
    } else {
      h[j] = T(0);
    }
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
