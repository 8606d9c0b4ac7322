// Push / pull kernel family for sm_100a.
//
// One thread per sampling point (grid voxel), Z fastest, so that grid reads,
// target reads and gather/scatter neighbourhoods of consecutive lanes are
// contiguous for near-identity deformations.  Per thread:
//   1. read the D coordinates, run the out-of-bound test
//      (nitorch/_C/src/impl/pushpull_common.cpp:925-974);
//   2. build a separable stencil: per axis, the support nodes, their B-spline
//      weights / first / second derivatives with the boundary sign folded in,
//      and the wrapped memory offsets (pushpull_common.cpp:1121-1171);
//   3. run the mode's tap loop with separable partial sums (x innermost,
//      then y, then z), so a tap costs one load (or one atomic) and one FMA.
//
// Modes (compile-time) and the reference op they implement
// (flag table of nitorch/_C/src/pushpull.cpp):
//   K_PULL     grid_pull                       out[c]   = sum w   src[c]
//   K_SGRAD    grid_grad                       out[c,d] = sum dw_d src[c]
//   K_PUSH     grid_push / pull_backward(in)   out[c]  += w t[c]          (atomics)
//   K_COUNT    grid_count                      out     += w               (atomics)
//   K_PULLGRAD push_backward (+grid)           optional pull, gg_d = sum_c t[c] sum dw_d src[c]
//   K_PUSHGRAD pull_backward (+grid), count_backward (no target: t = 1)
//   K_KD       grid_grad_backward              out[c] += sum_d dw_d t[c,d];
//                                              gg_d = sum_c sum_e t[c,e] sum d2w_de src[c]
// Runtime flags select the optional halves of the fused modes.
#pragma once
#include "pp_common.cuh"

namespace ppk {

enum Mode : int { K_PULL = 0, K_SGRAD, K_PUSH, K_COUNT, K_PULLGRAD, K_PUSHGRAD, K_KD, K_NMODES };
enum Flag : int { F_A = 1, F_GRAD = 2, F_NOTRGT = 4 };  // F_A: pull (PULLGRAD) / push (PUSHGRAD, KD)

struct PPArgs {
  const void* src;   // gathered tensor (N, C, *src_size)
  const void* trgt;  // per-sample values (N, C, *trgt_size[, K])
  const void* grid;  // (N, *trgt_size, D)
  void* out;         // pull/sgrad: (N, C, *trgt_size[, D]); push/count: (N, C, *src_size)
  void* gg;          // grid gradient (N, *trgt_size, D)
  int64_t N, C;
  int64_t src_size[3], trgt_size[3];
  int64_t src_sN, src_sC, src_s[3];
  int64_t trgt_sN, trgt_sC, trgt_s[3], trgt_sK;
  int64_t grid_sN, grid_s[3], grid_sD;
  int64_t out_sN, out_sC, out_s[3], out_sK;
  int64_t gg_sN, gg_s[3], gg_sD;
  int bound[3], order[3];
  int extrapolate;
  int flags;
  int64_t nvox;
};

template <int ORD> struct Taps { static constexpr int value = ORD < 0 ? 8 : (ORD == 0 ? 1 : ORD + 1); };
// Unroll factor of the outermost (z) tap loop: full up to cubic, rolled for
// higher and runtime orders (keeps code size and compile time bounded).
template <int ORD, int NZ> struct OuterUnroll { static constexpr int value = (ORD >= 0 && ORD <= 3) ? NZ : 1; };

// Per-axis stencil.  NT = max taps; unused axes have one tap of weight 1.
template <int NT, class T, class I>
struct Axis {
  T w[NT], g[NT], h[NT];
  I os[NT];   // offsets into the gathered tensor (src)
  I oo[NT];   // offsets into the scattered tensor (out)
  unsigned mask;  // bit t set: tap t is a real node (sign != 0)
  int nt;
};

template <int NT, bool NEED_G, bool NEED_H, bool NEED_OS, bool NEED_OO, class T, class I>
__device__ __forceinline__ void build_axis(Axis<NT, T, I>& ax, int ORDc, int bnd, T x, I n,
                                           I sts, I sto) {
  const int ord = ORDc;
  const int nt = ord == 0 ? 1 : ord + 1;
  ax.nt = nt;
  // Keep the node arithmetic defined for absurd or non-finite coordinates
  // (only reachable with extrapolation on): |x| <= 2^30, NaN -> -2^30.
  x = fmin(fmax(x, T(-1073741824.0)), T(1073741824.0));
  I low = support_low<I, T>(ord, x);
  const bool inside = low >= 0 && low + nt - 1 < n;
  ax.mask = 0;
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    if (t < nt) {
      I b = low + t;
      T dx = x - static_cast<T>(b);
      T w = bs_weight<T>(ord, dx);
      T g = NEED_G ? bs_grad<T>(ord, dx) : T(0);
      T h = NEED_H ? bs_hess<T>(ord, dx) : T(0);
      int s = 1;
      I idx = b;
      if (!inside) { s = bound_sign<I>(bnd, b, n); idx = bound_index<I>(bnd, b, n); }
      if (s == 0) { idx = 0; w = g = h = T(0); }
      else { ax.mask |= 1u << t; if (s < 0) { w = -w; g = -g; h = -h; } }
      ax.w[t] = w; ax.g[t] = g; ax.h[t] = h;
      if (NEED_OS) ax.os[t] = idx * sts;
      if (NEED_OO) ax.oo[t] = idx * sto;
    } else {
      ax.w[t] = T(0); ax.g[t] = T(0); ax.h[t] = T(0);
      if (NEED_OS) ax.os[t] = 0;
      if (NEED_OO) ax.oo[t] = 0;
    }
  }
}

template <int NT, class T, class I>
__device__ __forceinline__ void unit_axis(Axis<NT, T, I>& ax) {
  ax.nt = 1; ax.mask = 1u;
#pragma unroll
  for (int t = 0; t < NT; ++t) { ax.w[t] = t == 0 ? T(1) : T(0); ax.g[t] = T(0); ax.h[t] = T(0); ax.os[t] = 0; ax.oo[t] = 0; }
}

template <int D, int ORD, class S, int MODE, class I>
__global__ void __launch_bounds__(256) pp_kernel(const PPArgs a) {
  using T = typename Acc<S>::type;
  constexpr int NT = Taps<ORD>::value;
  constexpr int NX = NT, NY = D > 1 ? NT : 1, NZ = D > 2 ? NT : 1;
  constexpr bool NEED_G = MODE == K_SGRAD || MODE == K_PULLGRAD || MODE == K_PUSHGRAD || MODE == K_KD;
  constexpr bool NEED_H = MODE == K_KD;
  constexpr bool GATHER = MODE == K_PULL || MODE == K_SGRAD || MODE == K_PULLGRAD || MODE == K_PUSHGRAD || MODE == K_KD;
  constexpr bool SCATTER = MODE == K_PUSH || MODE == K_COUNT || MODE == K_PUSHGRAD || MODE == K_KD;

  const int64_t vid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (vid >= a.nvox) return;

  // ---- decode sampling point (n, x, y, z), Z fastest -------------------
  I sub[3] = {0, 0, 0};
  I n;
  {
    I v = static_cast<I>(vid);
    if (D > 2) { sub[2] = v % static_cast<I>(a.trgt_size[2]); v /= static_cast<I>(a.trgt_size[2]); }
    if (D > 1) { sub[1] = v % static_cast<I>(a.trgt_size[1]); v /= static_cast<I>(a.trgt_size[1]); }
    sub[0] = v % static_cast<I>(a.trgt_size[0]);
    n = v / static_cast<I>(a.trgt_size[0]);
  }

  // ---- coordinates ------------------------------------------------------
  const T* gp = static_cast<const T*>(a.grid) + static_cast<int64_t>(n) * a.grid_sN;
  int64_t goff = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) goff += static_cast<int64_t>(sub[d]) * a.grid_s[d];
  gp += goff;
  T coord[3];
#pragma unroll
  for (int d = 0; d < D; ++d) coord[d] = __ldg(gp + d * a.grid_sD);

  const bool do_a = (a.flags & F_A) != 0;
  const bool do_grad = (a.flags & F_GRAD) != 0;

  // per-voxel output locations (gathered outputs / grid gradient)
  int64_t ovox = static_cast<int64_t>(n) * a.out_sN;
  int64_t gvox = static_cast<int64_t>(n) * a.gg_sN;
  int64_t tvox = static_cast<int64_t>(n) * a.trgt_sN;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    ovox += static_cast<int64_t>(sub[d]) * a.out_s[d];
    gvox += static_cast<int64_t>(sub[d]) * a.gg_s[d];
    tvox += static_cast<int64_t>(sub[d]) * a.trgt_s[d];
  }

  // ---- out-of-bound test -------------------------------------------------
  {
    const T tol = (a.extrapolate & 2) ? static_cast<T>(0.5 + 5e-2) : static_cast<T>(5e-2);
    bool inb = true;
#pragma unroll
    for (int d = 0; d < D; ++d) inb = inb && in_fov<T>(coord[d], a.src_size[d], tol);
    if (!((a.extrapolate & 1) || inb)) {
      if (MODE == K_PULL || MODE == K_SGRAD || (MODE == K_PULLGRAD && do_a)) {
        S* op = static_cast<S*>(a.out) + ovox;
        for (int64_t c = 0; c < a.C; ++c) {
          if (MODE == K_SGRAD) {
#pragma unroll
            for (int d = 0; d < D; ++d) op[c * a.out_sC + d * a.out_sK] = from_acc<S>(T(0));
          } else {
            op[c * a.out_sC] = from_acc<S>(T(0));
          }
        }
      }
      if ((MODE == K_PULLGRAD || MODE == K_PUSHGRAD || MODE == K_KD) && do_grad) {
        T* g = static_cast<T*>(a.gg) + gvox;
#pragma unroll
        for (int d = 0; d < D; ++d) g[d * a.gg_sD] = T(0);
      }
      return;
    }
  }

  // ---- separable stencil --------------------------------------------------
  Axis<NX, T, I> ax;
  Axis<NY, T, I> ay;
  Axis<NZ, T, I> az;
  {
    const int o0 = ORD >= 0 ? ORD : a.order[0];
    build_axis<NX, NEED_G, NEED_H, GATHER, SCATTER, T, I>(
        ax, o0, a.bound[0], coord[0], static_cast<I>(a.src_size[0]),
        static_cast<I>(a.src_s[0]), static_cast<I>(a.out_s[0]));
    if (D > 1) {
      const int o1 = ORD >= 0 ? ORD : a.order[1];
      build_axis<NY, NEED_G, NEED_H, GATHER, SCATTER, T, I>(
          ay, o1, a.bound[1], coord[1], static_cast<I>(a.src_size[1]),
          static_cast<I>(a.src_s[1]), static_cast<I>(a.out_s[1]));
    } else {
      unit_axis(ay);
    }
    if (D > 2) {
      const int o2 = ORD >= 0 ? ORD : a.order[2];
      build_axis<NZ, NEED_G, NEED_H, GATHER, SCATTER, T, I>(
          az, o2, a.bound[2], coord[2], static_cast<I>(a.src_size[2]),
          static_cast<I>(a.src_s[2]), static_cast<I>(a.out_s[2]));
    } else {
      unit_axis(az);
    }
  }
  const bool full = (ax.mask == (1u << ax.nt) - 1u) && (ay.mask == (1u << ay.nt) - 1u) &&
                    (az.mask == (1u << az.nt) - 1u);
  const int tx = ORD >= 0 ? NX : ax.nt;
  const int ty = ORD >= 0 ? NY : ay.nt;
  const int tz = ORD >= 0 ? NZ : az.nt;

  const S* src_n = GATHER ? static_cast<const S*>(a.src) + static_cast<int64_t>(n) * a.src_sN : nullptr;
  T* outs_n = SCATTER ? static_cast<T*>(a.out) + static_cast<int64_t>(n) * a.out_sN : nullptr;
  const S* trg_v = static_cast<const S*>(a.trgt) + tvox;

#define PP_TAP_VALID(i, j, k) (full || ((((ax.mask >> (i)) & (ay.mask >> (j)) & (az.mask >> (k))) & 1u) != 0u))

  // ======================= gather-only modes ================================
  if constexpr (MODE == K_PULL) {
    S* op = static_cast<S*>(a.out) + ovox;
    for (int64_t c = 0; c < a.C; ++c) {
      const S* sp = src_n + c * a.src_sC;
      T acc = T(0);
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
          T accy = T(0);
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const I oyz = ay.os[j] + az.os[k];
              T accx = T(0);
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx) {
                  T v = ldg_acc(sp + (ax.os[i] + oyz));
                  if (!PP_TAP_VALID(i, j, k)) v = T(0);
                  accx = fma(ax.w[i], v, accx);
                }
              }
              accy = fma(ay.w[j], accx, accy);
            }
          }
          acc = fma(az.w[k], accy, acc);
        }
      }
      op[c * a.out_sC] = from_acc<S>(acc);
    }
  }

  if constexpr (MODE == K_SGRAD) {
    S* op = static_cast<S*>(a.out) + ovox;
    for (int64_t c = 0; c < a.C; ++c) {
      const S* sp = src_n + c * a.src_sC;
      T gx = T(0), gy = T(0), gz = T(0);
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
          T yw = T(0), ygx = T(0), ygy = T(0);
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const I oyz = ay.os[j] + az.os[k];
              T sx = T(0), dx = T(0);
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx) {
                  T v = ldg_acc(sp + (ax.os[i] + oyz));
                  if (!PP_TAP_VALID(i, j, k)) v = T(0);
                  sx = fma(ax.w[i], v, sx);
                  dx = fma(ax.g[i], v, dx);
                }
              }
              yw = fma(ay.w[j], sx, yw);
              ygx = fma(ay.w[j], dx, ygx);
              ygy = fma(ay.g[j], sx, ygy);
            }
          }
          gx = fma(az.w[k], ygx, gx);
          gy = fma(az.w[k], ygy, gy);
          gz = fma(az.g[k], yw, gz);
        }
      }
      S* oc = op + c * a.out_sC;
      oc[0] = from_acc<S>(gx);
      if (D > 1) oc[a.out_sK] = from_acc<S>(gy);
      if (D > 2) oc[2 * a.out_sK] = from_acc<S>(gz);
    }
  }

  if constexpr (MODE == K_PULLGRAD) {
    // push backward: src = incoming gradient, trgt = pushed values.
    S* op = static_cast<S*>(a.out) + ovox;
    T og0 = T(0), og1 = T(0), og2 = T(0);
    for (int64_t c = 0; c < a.C; ++c) {
      const S* sp = src_n + c * a.src_sC;
      T acc = T(0), gx = T(0), gy = T(0), gz = T(0);
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
          T yw = T(0), ygx = T(0), ygy = T(0);
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const I oyz = ay.os[j] + az.os[k];
              T sx = T(0), dx = T(0);
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx) {
                  T v = ldg_acc(sp + (ax.os[i] + oyz));
                  if (!PP_TAP_VALID(i, j, k)) v = T(0);
                  sx = fma(ax.w[i], v, sx);
                  dx = fma(ax.g[i], v, dx);
                }
              }
              yw = fma(ay.w[j], sx, yw);
              ygx = fma(ay.w[j], dx, ygx);
              ygy = fma(ay.g[j], sx, ygy);
            }
          }
          acc = fma(az.w[k], yw, acc);
          gx = fma(az.w[k], ygx, gx);
          gy = fma(az.w[k], ygy, gy);
          gz = fma(az.g[k], yw, gz);
        }
      }
      if (do_a) op[c * a.out_sC] = from_acc<S>(acc);
      const T t = ldg_acc(trg_v + c * a.trgt_sC);
      og0 = fma(t, gx, og0); og1 = fma(t, gy, og1); og2 = fma(t, gz, og2);
    }
    if (do_grad) {
      T* g = static_cast<T*>(a.gg) + gvox;
      g[0] = og0;
      if (D > 1) g[a.gg_sD] = og1;
      if (D > 2) g[2 * a.gg_sD] = og2;
    }
  }

  // ======================= scatter modes ====================================
  if constexpr (MODE == K_PUSH || MODE == K_COUNT) {
    const int64_t C = MODE == K_COUNT ? 1 : a.C;
    for (int64_t c = 0; c < C; ++c) {
      const T t = MODE == K_COUNT ? T(1) : ldg_acc(trg_v + c * a.trgt_sC);
      T* opc = outs_n + c * a.out_sC;
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
          const T tz_ = az.w[k] * t;
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const T tyz = ay.w[j] * tz_;
              const I oyz = ay.oo[j] + az.oo[k];
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx) {
                  const T v = ax.w[i] * tyz;
                  if (PP_TAP_VALID(i, j, k) && v != T(0)) atomic_acc(opc + (ax.oo[i] + oyz), v);
                }
              }
            }
          }
        }
      }
    }
  }

  if constexpr (MODE == K_PUSHGRAD) {
    // pull backward: src = pulled input, trgt = incoming gradient.
    // count backward: F_NOTRGT, t = 1, no push.
    const bool has_t = (a.flags & F_NOTRGT) == 0;
    T og0 = T(0), og1 = T(0), og2 = T(0);
    for (int64_t c = 0; c < a.C; ++c) {
      const S* sp = src_n + c * a.src_sC;
      T* opc = do_a ? outs_n + c * a.out_sC : nullptr;
      const T t = has_t ? ldg_acc(trg_v + c * a.trgt_sC) : T(1);
      T gx = T(0), gy = T(0), gz = T(0);
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
          T yw = T(0), ygx = T(0), ygy = T(0);
          const T tz_ = az.w[k] * t;
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const I oyz = ay.os[j] + az.os[k];
              const I ooyz = ay.oo[j] + az.oo[k];
              const T tyz = ay.w[j] * tz_;
              T sx = T(0), dx = T(0);
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx) {
                  const bool valid = PP_TAP_VALID(i, j, k);
                  if (do_grad) {
                    T v = ldg_acc(sp + (ax.os[i] + oyz));
                    if (!valid) v = T(0);
                    sx = fma(ax.w[i], v, sx);
                    dx = fma(ax.g[i], v, dx);
                  }
                  if (do_a) {
                    const T pv = ax.w[i] * tyz;
                    if (valid && pv != T(0)) atomic_acc(opc + (ax.oo[i] + ooyz), pv);
                  }
                }
              }
              yw = fma(ay.w[j], sx, yw);
              ygx = fma(ay.w[j], dx, ygx);
              ygy = fma(ay.g[j], sx, ygy);
            }
          }
          gx = fma(az.w[k], ygx, gx);
          gy = fma(az.w[k], ygy, gy);
          gz = fma(az.g[k], yw, gz);
        }
      }
      og0 = fma(t, gx, og0); og1 = fma(t, gy, og1); og2 = fma(t, gz, og2);
    }
    if (do_grad) {
      T* g = static_cast<T*>(a.gg) + gvox;
      g[0] = og0;
      if (D > 1) g[a.gg_sD] = og1;
      if (D > 2) g[2 * a.gg_sD] = og2;
    }
  }

  if constexpr (MODE == K_KD) {
    // grid_grad backward: trgt = incoming gradient (N, C, *grid, D).
    T og0 = T(0), og1 = T(0), og2 = T(0);
    for (int64_t c = 0; c < a.C; ++c) {
      const S* sp = src_n + c * a.src_sC;
      T* opc = do_a ? outs_n + c * a.out_sC : nullptr;
      const S* tp = trg_v + c * a.trgt_sC;
      const T t0 = ldg_acc(tp);
      const T t1 = D > 1 ? ldg_acc(tp + a.trgt_sK) : T(0);
      const T t2 = D > 2 ? ldg_acc(tp + 2 * a.trgt_sK) : T(0);
      // Hessian accumulators of the interpolant of channel c.
      T hxx = T(0), hxy = T(0), hxz = T(0), hyy = T(0), hyz = T(0), hzz = T(0);
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
          T yw = T(0), ygx = T(0), ygy = T(0), yhx = T(0), ygxy = T(0), yhy = T(0);
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const I oyz = ay.os[j] + az.os[k];
              const I ooyz = ay.oo[j] + az.oo[k];
              // push value of tap (i,j,k): gx_i*(wy wz t0) + wx_i*(gy wz t1 + wy gz t2)
              const T pa = ay.w[j] * az.w[k] * t0;
              const T pb = ay.g[j] * az.w[k] * t1 + ay.w[j] * az.g[k] * t2;
              T sx = T(0), dx = T(0), hx = T(0);
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx) {
                  const bool valid = PP_TAP_VALID(i, j, k);
                  if (do_grad) {
                    T v = ldg_acc(sp + (ax.os[i] + oyz));
                    if (!valid) v = T(0);
                    sx = fma(ax.w[i], v, sx);
                    dx = fma(ax.g[i], v, dx);
                    hx = fma(ax.h[i], v, hx);
                  }
                  if (do_a) {
                    const T pv = ax.g[i] * pa + ax.w[i] * pb;
                    if (valid && pv != T(0)) atomic_acc(opc + (ax.oo[i] + ooyz), pv);
                  }
                }
              }
              yw = fma(ay.w[j], sx, yw);
              ygx = fma(ay.w[j], dx, ygx);
              ygy = fma(ay.g[j], sx, ygy);
              yhx = fma(ay.w[j], hx, yhx);
              ygxy = fma(ay.g[j], dx, ygxy);
              yhy = fma(ay.h[j], sx, yhy);
            }
          }
          hxx = fma(az.w[k], yhx, hxx);
          hxy = fma(az.w[k], ygxy, hxy);
          hyy = fma(az.w[k], yhy, hyy);
          hxz = fma(az.g[k], ygx, hxz);
          hyz = fma(az.g[k], ygy, hyz);
          hzz = fma(az.h[k], yw, hzz);
        }
      }
      og0 += hxx * t0 + hxy * t1 + hxz * t2;
      og1 += hxy * t0 + hyy * t1 + hyz * t2;
      og2 += hxz * t0 + hyz * t1 + hzz * t2;
    }
    if (do_grad) {
      T* g = static_cast<T*>(a.gg) + gvox;
      g[0] = og0;
      if (D > 1) g[a.gg_sD] = og1;
      if (D > 2) g[2 * a.gg_sD] = og2;
    }
  }
#undef PP_TAP_VALID
}

// Orders that get a compile-time specialisation for a storage type; every
// other order (and any anisotropic order or 64-bit offset case) runs the
// runtime-order kernel (ORD = -1, 64-bit offsets).
template <class S> struct Specialised { static constexpr unsigned mask = 0; };
template <> struct Specialised<float> { static constexpr unsigned mask = 0xFFu; };
template <> struct Specialised<__nv_bfloat16> { static constexpr unsigned mask = (1u << 1) | (1u << 3); };

template <int D, int ORD, class S, int MODE, class I>
inline cudaError_t launch_one(const PPArgs& a, cudaStream_t st) {
  const int threads = 256;
  const int64_t blocks = (a.nvox + threads - 1) / threads;
  if (blocks == 0) return cudaSuccess;
  pp_kernel<D, ORD, S, MODE, I><<<static_cast<unsigned>(blocks), threads, 0, st>>>(a);
  return cudaGetLastError();
}

template <int D, class S, int MODE>
inline cudaError_t launch_ord(int ord, bool wide, const PPArgs& a, cudaStream_t st) {
  constexpr unsigned m = (D == 1) ? 0u : Specialised<S>::mask;
  if (!wide && ord >= 0) {
    switch (ord) {
#define PP_CASE(O) case O: if constexpr ((m >> O) & 1u) return launch_one<D, O, S, MODE, int32_t>(a, st); break;
      PP_CASE(0) PP_CASE(1) PP_CASE(2) PP_CASE(3) PP_CASE(4) PP_CASE(5) PP_CASE(6) PP_CASE(7)
#undef PP_CASE
      default: break;
    }
  }
  return launch_one<D, -1, S, MODE, int64_t>(a, st);
}

}  // namespace ppk

// One launcher per (storage type, dimension, mode); each is compiled in its
// own translation unit (pp_inst.cu) so the family builds in parallel.
using pp_launcher_t = cudaError_t (*)(int ord, bool wide, const ppk::PPArgs& a, cudaStream_t st);
