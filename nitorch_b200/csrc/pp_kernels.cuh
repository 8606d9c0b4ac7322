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
//   K_PP       push(pull(src)) in one pass: y = sum w src (gathered, rounded to
//              the storage type as a separate pull would store it), then
//              out += w y at the same taps (no counterpart in the reference,
//              which runs grid_pull then grid_push)
//   K_PP_BWD   its adjoint pass: P^T P is self-adjoint, so with W = trgt
//              (laid out like src) out += w (sum w W) and the grid gradient is
//              gg_d = sum_c [ (P src)_c d(P W)_c/dx_d + (P W)_c d(P src)_c/dx_d ]
// Runtime flags select the optional halves of the fused modes.
#pragma once
#include <atomic>
#include <type_traits>

#include "pp_common.cuh"

namespace ppk {

enum Mode : int { K_PULL = 0, K_SGRAD, K_PUSH, K_COUNT, K_PULLGRAD, K_PUSHGRAD, K_KD,
                  K_PP, K_PP_BWD, K_NMODES };
enum Flag : int { F_A = 1, F_GRAD = 2, F_NOTRGT = 4, F_VEC = 8, F_IDGRID = 16, F_ADDSELF = 32, F_AFFINE = 64 };
// F_A: pull (PULLGRAD) / push (PUSHGRAD, KD)
// F_VEC: `out` is a channel-interleaved float accumulator (pp_lanes_kernel)
// F_IDGRID: the sampling coordinate is the point's own voxel plus the grid
//   value (the grid holds a displacement, not a transformation)
// F_ADDSELF (with F_IDGRID, C = D; displacement self-composition):
//   K_PULL      out = src(point) + pulled value        (u + u o (id + u))
//   K_PUSHGRAD  out += g(point) + grid gradient at the point, atomically,
//               on top of the push of g (its adjoint w.r.t. u)
// F_AFFINE: no grid tensor: the coordinate of grid point `sub` is
//   A [sub; 1], A the D x (D+1) row-major matrix of batch item n at
//   grid + n * grid_sN (resize / reslice without a materialised grid)

struct PPArgs {
  const void* src;   // gathered tensor (N, C, *src_size)
  const void* trgt;  // per-sample values (N, C, *trgt_size[, K])
  const void* grid;  // (N, *trgt_size, D)
  void* out;         // pull/sgrad: (N, C, *trgt_size[, D]); push/count: (N, C, *src_size)
  void* gg;          // grid gradient (N, *trgt_size, D)
  void* aux;         // K_SGRAD with F_A: the interpolated values (N, C, *trgt_size) at the trgt_* strides
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
  const int32_t* perm;  // optional processing order of the sampling points
  // Deterministic scatter: when det_acc is set, scatter modes accumulate
  // round(v * 2^e) into this int64 buffer (contiguous (N, C, *src_size))
  // instead of float atomics into `out`; e is derived from the float bits of
  // max |target| (det_max, written by a reduction) times det_bound so that
  // no partial sum can overflow.  Integer addition is associative, so the
  // result does not depend on the order of the atomics.
  unsigned long long* det_acc;
  const unsigned int* det_max;
  double det_bound;
  // Brick-major order (pp_brick_order): with `perm` brick-major, brick b of
  // batch item n holds samples perm[brick_start[b] .. brick_start[b + 1]),
  // nbrick[] bricks per axis of the scatter target / gathered source.
  const int32_t* brick_start;
  int64_t nbrick[3];
  // With brick_start: the samples' coordinates and indices in perm order
  // (pp_brick_order's records), or NULL to read perm and the grid.
  const float4* brec;
};

// Power-of-two scale of the deterministic accumulators: bound * scale < 2^61.
__device__ __forceinline__ double det_scale(const PPArgs& a) {
  const float m = __uint_as_float(__ldg(a.det_max));
  const double bound = static_cast<double>(m) * a.det_bound;
  if (!(bound > 0.0)) return 1.0;
  int ex;
  frexp(bound, &ex);            // bound = f * 2^ex, f in [0.5, 1)
  return ldexp(1.0, 61 - ex);
}

template <int ORD> struct Taps { static constexpr int value = ORD < 0 ? 8 : (ORD == 0 ? 1 : ORD + 1); };
// Unroll factor of the outermost (z) tap loop: full up to cubic, rolled for
// higher and runtime orders (keeps code size and compile time bounded).
template <int ORD, int NZ> struct OuterUnroll { static constexpr int value = 1; };

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
  const I low = support_low<I, T>(ord, x);
  const bool inside = low >= 0 && low + nt - 1 < n;
  const T f = (x - static_cast<T>(low)) - T(0.5) * static_cast<T>(ord - 1);
  bspline_stencil<NT, NEED_G, NEED_H, T>(ord, ord == 0 ? T(0) : f, ax.w, ax.g, ax.h);
  ax.mask = 0;
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    if (t < nt) {
      const I b = low + t;
      int s = 1;
      I idx = b;
      if (!inside) { s = bound_sign<I>(bnd, b, n); idx = bound_index<I>(bnd, b, n); }
      if (s == 0) { idx = 0; ax.w[t] = ax.g[t] = ax.h[t] = T(0); }
      else { ax.mask |= 1u << t; if (s < 0) { ax.w[t] = -ax.w[t]; ax.g[t] = -ax.g[t]; ax.h[t] = -ax.h[t]; } }
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

// CTA tile: 32 (last spatial axis) x 8 (second-to-last axis) sampling
// points; blockIdx.x enumerates (outer index, tile along the last axis),
// blockIdx.y tiles the second-to-last axis.  Neighbouring lanes and warps
// then share most of their support, which the L1 serves.
constexpr int TILE_IN = 32, TILE_MID = 8, PP_THREADS = TILE_IN * TILE_MID;

// Vector reduction of CP interleaved float channels (red.global.add.v2/v4.f32).
template <int CP> __device__ __forceinline__ void red_vec(float* p, const float (&v)[CP]) {
  if constexpr (CP == 4)
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]),
                 "f"(v[3]) : "memory");
  else
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(v[0]), "f"(v[1]) : "memory");
}
// Channel blocks that can scatter into a channel-interleaved float
// accumulator (flag F_VEC): float arithmetic, 2-4 channels in one block.
template <class T, int CB> struct PPVec {
  static constexpr bool ok = std::is_same<T, float>::value && CB >= 2;
  static constexpr int CP = CB == 2 ? 2 : 4;
};

template <int MODE> struct MinBlocks { static constexpr int value = (MODE == K_PUSH || MODE == K_COUNT) ? 4 : 2; };

// One sampling point (batch item n, grid position sub) of mode MODE: the
// whole per-point computation, shared by the single-tensor kernel below and
// the batched kernel (batch.cu).
template <int D, int ORD, int CB, class S, int MODE, class I>
__device__ __forceinline__ void pp_point(const PPArgs& a, const I (&sub)[3], const I n) {
  using T = typename Acc<S>::type;
  constexpr int NT = Taps<ORD>::value;
  constexpr int NX = NT, NY = D > 1 ? NT : 1, NZ = D > 2 ? NT : 1;
  constexpr bool NEED_G = MODE == K_SGRAD || MODE == K_PULLGRAD || MODE == K_PUSHGRAD || MODE == K_KD ||
                          MODE == K_PP_BWD;
  constexpr bool NEED_H = MODE == K_KD;
  constexpr bool GATHER = MODE == K_PULL || MODE == K_SGRAD || MODE == K_PULLGRAD || MODE == K_PUSHGRAD ||
                          MODE == K_KD || MODE == K_PP || MODE == K_PP_BWD;
  constexpr bool SCATTER = MODE == K_PUSH || MODE == K_COUNT || MODE == K_PUSHGRAD || MODE == K_KD ||
                           MODE == K_PP || MODE == K_PP_BWD;

  // ---- coordinates ------------------------------------------------------
  T coord[3];
  if (a.flags & F_AFFINE) {
    const T* m = static_cast<const T*>(a.grid) + static_cast<int64_t>(n) * a.grid_sN;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      T x = __ldg(m + d * (D + 1) + D);
#pragma unroll
      for (int e = 0; e < D; ++e) x = fma(__ldg(m + d * (D + 1) + e), static_cast<T>(sub[e]), x);
      coord[d] = x;
    }
  } else {
    const T* gp = static_cast<const T*>(a.grid) + static_cast<int64_t>(n) * a.grid_sN;
    int64_t goff = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) goff += static_cast<int64_t>(sub[d]) * a.grid_s[d];
    gp += goff;
#pragma unroll
    for (int d = 0; d < D; ++d) coord[d] = __ldg(gp + d * a.grid_sD);
  }
  if (a.flags & F_IDGRID) {
#pragma unroll
    for (int d = 0; d < D; ++d) coord[d] += static_cast<T>(sub[d]);
  }

  const bool do_a = (a.flags & F_A) != 0;
  const bool do_grad = (a.flags & F_GRAD) != 0;
  const bool vec = (a.flags & F_VEC) != 0;  // channel-interleaved float accumulator

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
      if (a.flags & F_ADDSELF) {
        // self-composition outside the field of view: only the identity terms
        int64_t so = 0, oo = 0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          so += static_cast<int64_t>(sub[d]) * a.src_s[d];
          oo += static_cast<int64_t>(sub[d]) * a.out_s[d];
        }
        if (MODE == K_PULL) {
          const S* sp = static_cast<const S*>(a.src) + static_cast<int64_t>(n) * a.src_sN + so;
          S* op = static_cast<S*>(a.out) + ovox;
          for (int64_t c = 0; c < a.C; ++c) op[c * a.out_sC] = sp[c * a.src_sC];
        }
        if (MODE == K_PUSHGRAD) {
          const S* tp = static_cast<const S*>(a.trgt) + tvox;
          if (a.det_acc != nullptr) {  // deterministic: this point alone writes its terms (aux)
            T* sp = static_cast<T*>(a.aux) + static_cast<int64_t>(n) * a.out_sN + oo;
            for (int64_t c = 0; c < a.C; ++c) sp[c * a.out_sC] = ldg_acc(tp + c * a.trgt_sC);
          } else {
            T* op = static_cast<T*>(a.out) + static_cast<int64_t>(n) * a.out_sN + oo;
            for (int64_t c = 0; c < a.C; ++c) atomic_acc(op + c * a.out_sC, ldg_acc(tp + c * a.trgt_sC));
          }
        }
        return;
      }
      if (MODE == K_PULL || MODE == K_SGRAD || (MODE == K_PULLGRAD && do_a)) {
        S* op = static_cast<S*>(a.out) + ovox;
        for (int64_t c = 0; c < a.C; ++c) {
          if (MODE == K_SGRAD) {
#pragma unroll
            for (int d = 0; d < D; ++d) op[c * a.out_sC + d * a.out_sK] = from_acc<S>(T(0));
            if (do_a) (static_cast<S*>(a.aux) + tvox)[c * a.trgt_sC] = from_acc<S>(T(0));
          } else {
            op[c * a.out_sC] = from_acc<S>(T(0));
          }
        }
      }
      if ((MODE == K_PULLGRAD || MODE == K_PUSHGRAD || MODE == K_KD || MODE == K_PP_BWD) && do_grad) {
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
  const double dscale = (SCATTER && a.det_acc != nullptr) ? det_scale(a) : 0.0;
  unsigned long long* dacc_n = (SCATTER && a.det_acc != nullptr) ? a.det_acc + static_cast<int64_t>(n) * a.out_sN : nullptr;
  // scatter of v to tap offset `off` of channel cb of the current group
#define PP_SCATTER(off, v)                                                                   \
  do {                                                                                       \
    if (dacc_n != nullptr)                                                                   \
      atomicAdd(dacc_n + ((c0 + cb) * a.out_sC + (off)),                                     \
                static_cast<unsigned long long>(__double2ll_rn(static_cast<double>(v) * dscale))); \
    else                                                                                     \
      atomic_acc(opc + (cb * a.out_sC + (off)), (v));                                        \
  } while (0)

// scatter of one tap's channel values VAL(cb): one vector reduction into the
// interleaved accumulator when `vec`, else one reduction per nonzero value
#define PP_SCATTER_CH(off, VAL)                                                     \
  do {                                                                              \
    if constexpr (PPVec<T, CB>::ok) {                                               \
      if (vec) {                                                                    \
        float vals_[PPVec<T, CB>::CP];                                              \
        _Pragma("unroll") for (int q_ = 0; q_ < PPVec<T, CB>::CP; ++q_) vals_[q_] = 0.f; \
        _Pragma("unroll") for (int cb = 0; cb < CB; ++cb) vals_[cb] = VAL(cb);     \
        red_vec<PPVec<T, CB>::CP>(opc + (off), vals_);                              \
        break;                                                                      \
      }                                                                             \
    }                                                                               \
    _Pragma("unroll") PP_CB {                                                       \
      if (CB == 1 || cb < nc) {                                                     \
        const T v_ = VAL(cb);                                                       \
        if (v_ != T(0)) PP_SCATTER(off, v_);                                        \
      }                                                                             \
    }                                                                               \
  } while (0)

#define PP_TAP_VALID(i, j, k) (full || ((((ax.mask >> (i)) & (ay.mask >> (j)) & (az.mask >> (k))) & 1u) != 0u))

  // Channels are processed in groups of CB (compile-time): per tap, one
  // offset and one weight feed CB loads / atomics, and the accumulators of
  // the group live in registers.
#define PP_CB for (int cb = 0; cb < CB; ++cb)
  const int64_t C = MODE == K_COUNT ? 1 : a.C;

  // ======================= gather-only modes ================================
  if constexpr (MODE == K_PULL) {
    S* op = static_cast<S*>(a.out) + ovox;
    for (int64_t c0 = 0; c0 < C; c0 += CB) {
      const int nc = C - c0 < CB ? static_cast<int>(C - c0) : CB;
      const S* sp = src_n + c0 * a.src_sC;
      T acc[CB];
#pragma unroll
      PP_CB acc[cb] = T(0);
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
          T accy[CB];
#pragma unroll
          PP_CB accy[cb] = T(0);
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const I oyz = ay.os[j] + az.os[k];
              T accx[CB];
#pragma unroll
              PP_CB accx[cb] = T(0);
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx) {
                  const I off = ax.os[i] + oyz;
                  const bool valid = PP_TAP_VALID(i, j, k);
#pragma unroll
                  PP_CB {
                    if (CB == 1 || cb < nc) {
                      T v = ldg_acc(sp + (cb * a.src_sC + off));
                      if (!valid) v = T(0);
                      accx[cb] = fma(ax.w[i], v, accx[cb]);
                    }
                  }
                }
              }
#pragma unroll
              PP_CB accy[cb] = fma(ay.w[j], accx[cb], accy[cb]);
            }
          }
#pragma unroll
          PP_CB acc[cb] = fma(az.w[k], accy[cb], acc[cb]);
        }
      }
      if (a.flags & F_ADDSELF) {
        // self-composition: add the field's own value at the point
        int64_t so = 0;
#pragma unroll
        for (int d = 0; d < D; ++d) so += static_cast<int64_t>(sub[d]) * a.src_s[d];
#pragma unroll
        PP_CB if (CB == 1 || cb < nc) acc[cb] += ldg_acc(sp + cb * a.src_sC + so);
      }
#pragma unroll
      PP_CB if (CB == 1 || cb < nc) op[(c0 + cb) * a.out_sC] = from_acc<S>(acc[cb]);
    }
  }

  // Spatial-gradient accumulation shared by SGRAD and PULLGRAD: per channel
  // of the group, the interpolant (w) and its x/y/z derivatives.
#define PP_GRAD_GATHER(EXTRA_ROW, EXTRA_PLANE)                                   \
  T gx[CB], gy[CB], gz[CB], gw[CB];                                              \
  _Pragma("unroll") PP_CB { gx[cb] = gy[cb] = gz[cb] = gw[cb] = T(0); }          \
  _Pragma("unroll (OuterUnroll<ORD, NZ>::value)") for (int k = 0; k < NZ; ++k) {  \
    if (k < tz) {                                                                \
      T yw[CB], ygx[CB], ygy[CB];                                                \
      _Pragma("unroll") PP_CB { yw[cb] = ygx[cb] = ygy[cb] = T(0); }             \
      _Pragma("unroll") for (int j = 0; j < NY; ++j) {                           \
        if (j < ty) {                                                            \
          const I oyz = ay.os[j] + az.os[k];                                     \
          T sx[CB], dx[CB];                                                      \
          _Pragma("unroll") PP_CB { sx[cb] = dx[cb] = T(0); }                    \
          _Pragma("unroll") for (int i = 0; i < NX; ++i) {                       \
            if (i < tx) {                                                        \
              const I off = ax.os[i] + oyz;                                      \
              const bool valid = PP_TAP_VALID(i, j, k);                          \
              _Pragma("unroll") PP_CB {                                          \
                if (CB == 1 || cb < nc) {                                        \
                  T v = ldg_acc(sp + (cb * a.src_sC + off));                     \
                  if (!valid) v = T(0);                                          \
                  sx[cb] = fma(ax.w[i], v, sx[cb]);                              \
                  dx[cb] = fma(ax.g[i], v, dx[cb]);                              \
                }                                                                \
              }                                                                  \
              EXTRA_ROW                                                          \
            }                                                                    \
          }                                                                      \
          _Pragma("unroll") PP_CB {                                              \
            yw[cb] = fma(ay.w[j], sx[cb], yw[cb]);                               \
            ygx[cb] = fma(ay.w[j], dx[cb], ygx[cb]);                             \
            ygy[cb] = fma(ay.g[j], sx[cb], ygy[cb]);                             \
          }                                                                      \
        }                                                                        \
      }                                                                          \
      _Pragma("unroll") PP_CB {                                                  \
        gx[cb] = fma(az.w[k], ygx[cb], gx[cb]);                                  \
        gy[cb] = fma(az.w[k], ygy[cb], gy[cb]);                                  \
        gz[cb] = fma(az.g[k], yw[cb], gz[cb]);                                   \
        gw[cb] = fma(az.w[k], yw[cb], gw[cb]);                                   \
      }                                                                          \
      EXTRA_PLANE                                                                \
    }                                                                            \
  }

  if constexpr (MODE == K_SGRAD) {
    // spatial gradient; with F_A also the interpolated value (the fused
    // pull + grid_grad forward), the gw sum of the same taps
    S* op = static_cast<S*>(a.out) + ovox;
    S* vp = do_a ? static_cast<S*>(a.aux) + tvox : nullptr;
    for (int64_t c0 = 0; c0 < C; c0 += CB) {
      const int nc = C - c0 < CB ? static_cast<int>(C - c0) : CB;
      const S* sp = src_n + c0 * a.src_sC;
      PP_GRAD_GATHER(, )
#pragma unroll
      PP_CB {
        if (CB == 1 || cb < nc) {
          S* oc = op + (c0 + cb) * a.out_sC;
          oc[0] = from_acc<S>(gx[cb]);
          if (D > 1) oc[a.out_sK] = from_acc<S>(gy[cb]);
          if (D > 2) oc[2 * a.out_sK] = from_acc<S>(gz[cb]);
          if (vp) vp[(c0 + cb) * a.trgt_sC] = from_acc<S>(gw[cb]);
        }
      }
    }
  }

  if constexpr (MODE == K_PULLGRAD) {
    // push backward: src = incoming gradient, trgt = pushed values.
    S* op = static_cast<S*>(a.out) + ovox;
    T og0 = T(0), og1 = T(0), og2 = T(0);
    for (int64_t c0 = 0; c0 < C; c0 += CB) {
      const int nc = C - c0 < CB ? static_cast<int>(C - c0) : CB;
      const S* sp = src_n + c0 * a.src_sC;
      PP_GRAD_GATHER(, )
#pragma unroll
      PP_CB {
        if (CB == 1 || cb < nc) {
          if (do_a) op[(c0 + cb) * a.out_sC] = from_acc<S>(gw[cb]);
          const T t = ldg_acc(trg_v + (c0 + cb) * a.trgt_sC);
          og0 = fma(t, gx[cb], og0); og1 = fma(t, gy[cb], og1); og2 = fma(t, gz[cb], og2);
        }
      }
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
    for (int64_t c0 = 0; c0 < C; c0 += CB) {
      const int nc = C - c0 < CB ? static_cast<int>(C - c0) : CB;
      T* opc = outs_n + c0 * a.out_sC;
      T t[CB];
#pragma unroll
      PP_CB t[cb] = (MODE == K_COUNT) ? T(1) : ((CB == 1 || cb < nc) ? ldg_acc(trg_v + (c0 + cb) * a.trgt_sC) : T(0));
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const T wyz = ay.w[j] * az.w[k];
              const I oyz = ay.oo[j] + az.oo[k];
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx && PP_TAP_VALID(i, j, k)) {
                  const T wt = ax.w[i] * wyz;
                  const I off = ax.oo[i] + oyz;
                  auto val = [&](int cb) { return wt * t[cb]; };
                  PP_SCATTER_CH(off, val);
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
    for (int64_t c0 = 0; c0 < C; c0 += CB) {
      const int nc = C - c0 < CB ? static_cast<int>(C - c0) : CB;
      const S* sp = src_n + c0 * a.src_sC;
      T* opc = do_a ? outs_n + c0 * a.out_sC : nullptr;
      T t[CB];
#pragma unroll
      PP_CB t[cb] = (CB == 1 || cb < nc) ? (has_t ? ldg_acc(trg_v + (c0 + cb) * a.trgt_sC) : T(1)) : T(0);
      T gx[CB], gy[CB], gz[CB];
#pragma unroll
      PP_CB { gx[cb] = gy[cb] = gz[cb] = T(0); }
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
          T yw[CB], ygx[CB], ygy[CB];
#pragma unroll
          PP_CB { yw[cb] = ygx[cb] = ygy[cb] = T(0); }
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const I oyz = ay.os[j] + az.os[k];
              const I ooyz = ay.oo[j] + az.oo[k];
              const T wyz = ay.w[j] * az.w[k];
              T sx[CB], dx[CB];
#pragma unroll
              PP_CB { sx[cb] = dx[cb] = T(0); }
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx) {
                  const bool valid = PP_TAP_VALID(i, j, k);
                  if (do_grad) {
                    const I off = ax.os[i] + oyz;
#pragma unroll
                    PP_CB {
                      if (CB == 1 || cb < nc) {
                        T v = ldg_acc(sp + (cb * a.src_sC + off));
                        if (!valid) v = T(0);
                        sx[cb] = fma(ax.w[i], v, sx[cb]);
                        dx[cb] = fma(ax.g[i], v, dx[cb]);
                      }
                    }
                  }
                  if (do_a && valid) {
                    const T wt = ax.w[i] * wyz;
                    const I off = ax.oo[i] + ooyz;
                    auto val = [&](int cb) { return wt * t[cb]; };
                    PP_SCATTER_CH(off, val);
                  }
                }
              }
#pragma unroll
              PP_CB {
                yw[cb] = fma(ay.w[j], sx[cb], yw[cb]);
                ygx[cb] = fma(ay.w[j], dx[cb], ygx[cb]);
                ygy[cb] = fma(ay.g[j], sx[cb], ygy[cb]);
              }
            }
          }
#pragma unroll
          PP_CB {
            gx[cb] = fma(az.w[k], ygx[cb], gx[cb]);
            gy[cb] = fma(az.w[k], ygy[cb], gy[cb]);
            gz[cb] = fma(az.g[k], yw[cb], gz[cb]);
          }
        }
      }
#pragma unroll
      PP_CB { og0 = fma(t[cb], gx[cb], og0); og1 = fma(t[cb], gy[cb], og1); og2 = fma(t[cb], gz[cb], og2); }
    }
    if (a.flags & F_ADDSELF) {
      // self-composition backward: g and the grid gradient at the point go to
      // the same output as the push, atomically
      int64_t oo = 0;
#pragma unroll
      for (int d = 0; d < D; ++d) oo += static_cast<int64_t>(sub[d]) * a.out_s[d];
      const T og[3] = {og0, og1, og2};
      if (a.det_acc != nullptr) {
        // deterministic mode: the terms of this voxel have no other writer;
        // stored apart (aux, laid out like the fixed-point accumulator) and
        // added to the push by the finalize pass
        T* sp = static_cast<T*>(a.aux) + static_cast<int64_t>(n) * a.out_sN + oo;
#pragma unroll
        for (int d = 0; d < D; ++d) sp[d * a.out_sC] = og[d] + ldg_acc(trg_v + d * a.trgt_sC);
      } else {
        T* op = static_cast<T*>(a.out) + static_cast<int64_t>(n) * a.out_sN + oo;
#pragma unroll
        for (int d = 0; d < D; ++d) atomic_acc(op + d * a.out_sC, og[d] + ldg_acc(trg_v + d * a.trgt_sC));
      }
    } else if (do_grad) {
      T* g = static_cast<T*>(a.gg) + gvox;
      g[0] = og0;
      if (D > 1) g[a.gg_sD] = og1;
      if (D > 2) g[2 * a.gg_sD] = og2;
    }
  }

  if constexpr (MODE == K_KD) {
    // grid_grad backward: trgt = incoming gradient (N, C, *grid, D).
    T og0 = T(0), og1 = T(0), og2 = T(0);
    for (int64_t c0 = 0; c0 < C; c0 += CB) {
      const int nc = C - c0 < CB ? static_cast<int>(C - c0) : CB;
      const S* sp = src_n + c0 * a.src_sC;
      T* opc = do_a ? outs_n + c0 * a.out_sC : nullptr;
      T t0[CB], t1[CB], t2[CB];
#pragma unroll
      PP_CB {
        const bool on = CB == 1 || cb < nc;
        const S* tp = trg_v + (c0 + cb) * a.trgt_sC;
        t0[cb] = on ? ldg_acc(tp) : T(0);
        t1[cb] = (on && D > 1) ? ldg_acc(tp + a.trgt_sK) : T(0);
        t2[cb] = (on && D > 2) ? ldg_acc(tp + 2 * a.trgt_sK) : T(0);
      }
      T hxx[CB], hxy[CB], hxz[CB], hyy[CB], hyz[CB], hzz[CB];
#pragma unroll
      PP_CB { hxx[cb] = hxy[cb] = hxz[cb] = hyy[cb] = hyz[cb] = hzz[cb] = T(0); }
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
          T yw[CB], ygx[CB], ygy[CB], yhx[CB], ygxy[CB], yhy[CB];
#pragma unroll
          PP_CB { yw[cb] = ygx[cb] = ygy[cb] = yhx[cb] = ygxy[cb] = yhy[cb] = T(0); }
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const I oyz = ay.os[j] + az.os[k];
              const I ooyz = ay.oo[j] + az.oo[k];
              T sx[CB], dx[CB], hx[CB];
#pragma unroll
              PP_CB { sx[cb] = dx[cb] = hx[cb] = T(0); }
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx) {
                  const bool valid = PP_TAP_VALID(i, j, k);
                  if (do_grad) {
                    const I off = ax.os[i] + oyz;
#pragma unroll
                    PP_CB {
                      if (CB == 1 || cb < nc) {
                        T v = ldg_acc(sp + (cb * a.src_sC + off));
                        if (!valid) v = T(0);
                        sx[cb] = fma(ax.w[i], v, sx[cb]);
                        dx[cb] = fma(ax.g[i], v, dx[cb]);
                        hx[cb] = fma(ax.h[i], v, hx[cb]);
                      }
                    }
                  }
                  if (do_a && valid) {
                    const I off = ax.oo[i] + ooyz;
                    // push value: gx wy wz t0 + wx (gy wz t1 + wy gz t2)
                    auto val = [&](int cb) {
                      const T pa = ay.w[j] * az.w[k] * t0[cb];
                      const T pb = ay.g[j] * az.w[k] * t1[cb] + ay.w[j] * az.g[k] * t2[cb];
                      return ax.g[i] * pa + ax.w[i] * pb;
                    };
                    PP_SCATTER_CH(off, val);
                  }
                }
              }
#pragma unroll
              PP_CB {
                yw[cb] = fma(ay.w[j], sx[cb], yw[cb]);
                ygx[cb] = fma(ay.w[j], dx[cb], ygx[cb]);
                ygy[cb] = fma(ay.g[j], sx[cb], ygy[cb]);
                yhx[cb] = fma(ay.w[j], hx[cb], yhx[cb]);
                ygxy[cb] = fma(ay.g[j], dx[cb], ygxy[cb]);
                yhy[cb] = fma(ay.h[j], sx[cb], yhy[cb]);
              }
            }
          }
#pragma unroll
          PP_CB {
            hxx[cb] = fma(az.w[k], yhx[cb], hxx[cb]);
            hxy[cb] = fma(az.w[k], ygxy[cb], hxy[cb]);
            hyy[cb] = fma(az.w[k], yhy[cb], hyy[cb]);
            hxz[cb] = fma(az.g[k], ygx[cb], hxz[cb]);
            hyz[cb] = fma(az.g[k], ygy[cb], hyz[cb]);
            hzz[cb] = fma(az.h[k], yw[cb], hzz[cb]);
          }
        }
      }
#pragma unroll
      PP_CB {
        og0 += hxx[cb] * t0[cb] + hxy[cb] * t1[cb] + hxz[cb] * t2[cb];
        og1 += hxy[cb] * t0[cb] + hyy[cb] * t1[cb] + hyz[cb] * t2[cb];
        og2 += hxz[cb] * t0[cb] + hyz[cb] * t1[cb] + hzz[cb] * t2[cb];
      }
    }
    if (do_grad) {
      T* g = static_cast<T*>(a.gg) + gvox;
      g[0] = og0;
      if (D > 1) g[a.gg_sD] = og1;
      if (D > 2) g[2 * a.gg_sD] = og2;
    }
  }

  if constexpr (MODE == K_PP) {
    // One pass of push(pull(src)): the gather and the scatter share the
    // stencil; out has src's shape (its own strides, offsets `oo`).
    for (int64_t c0 = 0; c0 < C; c0 += CB) {
      const int nc = C - c0 < CB ? static_cast<int>(C - c0) : CB;
      const S* sp = src_n + c0 * a.src_sC;
      T* opc = outs_n + c0 * a.out_sC;
      T y[CB];
#pragma unroll
      PP_CB y[cb] = T(0);
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
          T accy[CB];
#pragma unroll
          PP_CB accy[cb] = T(0);
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const I oyz = ay.os[j] + az.os[k];
              T accx[CB];
#pragma unroll
              PP_CB accx[cb] = T(0);
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx) {
                  const I off = ax.os[i] + oyz;
                  const bool valid = PP_TAP_VALID(i, j, k);
#pragma unroll
                  PP_CB {
                    if (CB == 1 || cb < nc) {
                      T v = ldg_acc(sp + (cb * a.src_sC + off));
                      if (!valid) v = T(0);
                      accx[cb] = fma(ax.w[i], v, accx[cb]);
                    }
                  }
                }
              }
#pragma unroll
              PP_CB accy[cb] = fma(ay.w[j], accx[cb], accy[cb]);
            }
          }
#pragma unroll
          PP_CB y[cb] = fma(az.w[k], accy[cb], y[cb]);
        }
      }
      // the pulled value as a separate pull would have stored it
#pragma unroll
      PP_CB y[cb] = to_acc(from_acc<S>(y[cb]));
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const T wyz = ay.w[j] * az.w[k];
              const I oyz = ay.oo[j] + az.oo[k];
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx && PP_TAP_VALID(i, j, k)) {
                  const T wt = ax.w[i] * wyz;
                  const I off = ax.oo[i] + oyz;
                  auto val = [&](int cb) { return wt * y[cb]; };
                  PP_SCATTER_CH(off, val);
                }
              }
            }
          }
        }
      }
    }
  }

  if constexpr (MODE == K_PP_BWD) {
    // Adjoint of K_PP.  trgt = W = d loss / d out, laid out like src
    // (checked on the host), so it shares src's offsets `os`.
    const S* wsrc_n = static_cast<const S*>(a.trgt) + static_cast<int64_t>(n) * a.src_sN;
    T og0 = T(0), og1 = T(0), og2 = T(0);
    for (int64_t c0 = 0; c0 < C; c0 += CB) {
      const int nc = C - c0 < CB ? static_cast<int>(C - c0) : CB;
      const S* sp = src_n + c0 * a.src_sC;
      const S* wp = wsrc_n + c0 * a.src_sC;
      T* opc = do_a ? outs_n + c0 * a.out_sC : nullptr;
      // interpolants of src (yv) and W (dv) and their spatial derivatives
      T yv[CB], yx[CB], yy[CB], yz[CB], dv[CB], dxg[CB], dyg[CB], dzg[CB];
#pragma unroll
      PP_CB { yv[cb] = yx[cb] = yy[cb] = yz[cb] = dv[cb] = dxg[cb] = dyg[cb] = dzg[cb] = T(0); }
#pragma unroll (OuterUnroll<ORD, NZ>::value)
      for (int k = 0; k < NZ; ++k) {
        if (k < tz) {
          T pyw[CB], pygx[CB], pygy[CB], pdw[CB], pdgx[CB], pdgy[CB];
#pragma unroll
          PP_CB { pyw[cb] = pygx[cb] = pygy[cb] = pdw[cb] = pdgx[cb] = pdgy[cb] = T(0); }
#pragma unroll
          for (int j = 0; j < NY; ++j) {
            if (j < ty) {
              const I oyz = ay.os[j] + az.os[k];
              T sx[CB], sdx[CB], wx[CB], wdx[CB];
#pragma unroll
              PP_CB { sx[cb] = sdx[cb] = wx[cb] = wdx[cb] = T(0); }
#pragma unroll
              for (int i = 0; i < NX; ++i) {
                if (i < tx) {
                  const I off = ax.os[i] + oyz;
                  const bool valid = PP_TAP_VALID(i, j, k);
#pragma unroll
                  PP_CB {
                    if (CB == 1 || cb < nc) {
                      T v = ldg_acc(sp + (cb * a.src_sC + off));
                      T u = ldg_acc(wp + (cb * a.src_sC + off));
                      if (!valid) { v = T(0); u = T(0); }
                      sx[cb] = fma(ax.w[i], v, sx[cb]);
                      sdx[cb] = fma(ax.g[i], v, sdx[cb]);
                      wx[cb] = fma(ax.w[i], u, wx[cb]);
                      wdx[cb] = fma(ax.g[i], u, wdx[cb]);
                    }
                  }
                }
              }
#pragma unroll
              PP_CB {
                pyw[cb] = fma(ay.w[j], sx[cb], pyw[cb]);
                pygx[cb] = fma(ay.w[j], sdx[cb], pygx[cb]);
                pygy[cb] = fma(ay.g[j], sx[cb], pygy[cb]);
                pdw[cb] = fma(ay.w[j], wx[cb], pdw[cb]);
                pdgx[cb] = fma(ay.w[j], wdx[cb], pdgx[cb]);
                pdgy[cb] = fma(ay.g[j], wx[cb], pdgy[cb]);
              }
            }
          }
#pragma unroll
          PP_CB {
            yv[cb] = fma(az.w[k], pyw[cb], yv[cb]);
            yx[cb] = fma(az.w[k], pygx[cb], yx[cb]);
            yy[cb] = fma(az.w[k], pygy[cb], yy[cb]);
            yz[cb] = fma(az.g[k], pyw[cb], yz[cb]);
            dv[cb] = fma(az.w[k], pdw[cb], dv[cb]);
            dxg[cb] = fma(az.w[k], pdgx[cb], dxg[cb]);
            dyg[cb] = fma(az.w[k], pdgy[cb], dyg[cb]);
            dzg[cb] = fma(az.g[k], pdw[cb], dzg[cb]);
          }
        }
      }
      // the values a separate pull / push-backward would have stored
#pragma unroll
      PP_CB {
        yv[cb] = to_acc(from_acc<S>(yv[cb]));
        dv[cb] = to_acc(from_acc<S>(dv[cb]));
        if (CB == 1 || cb < nc) {
          og0 += yv[cb] * dxg[cb] + dv[cb] * yx[cb];
          og1 += yv[cb] * dyg[cb] + dv[cb] * yy[cb];
          og2 += yv[cb] * dzg[cb] + dv[cb] * yz[cb];
        }
      }
      if (do_a) {
#pragma unroll (OuterUnroll<ORD, NZ>::value)
        for (int k = 0; k < NZ; ++k) {
          if (k < tz) {
#pragma unroll
            for (int j = 0; j < NY; ++j) {
              if (j < ty) {
                const T wyz = ay.w[j] * az.w[k];
                const I oyz = ay.oo[j] + az.oo[k];
#pragma unroll
                for (int i = 0; i < NX; ++i) {
                  if (i < tx && PP_TAP_VALID(i, j, k)) {
                    const T wt = ax.w[i] * wyz;
                    const I off = ax.oo[i] + oyz;
                    auto val = [&](int cb) { return wt * dv[cb]; };
                    PP_SCATTER_CH(off, val);
                  }
                }
              }
            }
          }
        }
      }
    }
    if (do_grad) {
      T* g = static_cast<T*>(a.gg) + gvox;
      g[0] = og0;
      if (D > 1) g[a.gg_sD] = og1;
      if (D > 2) g[2 * a.gg_sD] = og2;
    }
  }
#undef PP_GRAD_GATHER
#undef PP_CB
#undef PP_SCATTER

#undef PP_TAP_VALID
#undef PP_SCATTER_CH
}

// Single-channel 3-D pull-backward at orders 2-3 fits three CTAs per SM
// (80 registers, a few bytes of spills; cubic 192^3: 1.43 -> 1.25 ms); other
// instances keep MinBlocks (higher orders spill hundreds of bytes at three).
template <int D, int ORD, int CB, class S, int MODE, class I>
__global__ void __launch_bounds__(PP_THREADS, (MODE == K_PUSHGRAD && CB == 1 && D == 3 && ORD >= 2 && ORD <= 3) ? 3 : MinBlocks<MODE>::value) pp_kernel(const PPArgs a) {
  // ---- sampling point (n, x, y, z) -------------------------------------
  I sub[3] = {0, 0, 0};
  I n = 0;
  if (a.perm != nullptr) {
    // explicit processing order (source-sorted): linear thread index
    const int64_t t = (static_cast<int64_t>(blockIdx.x) * TILE_MID + threadIdx.y) * TILE_IN + threadIdx.x;
    if (t >= a.nvox) return;
    I v = static_cast<I>(__ldg(a.perm + t));
    if (D > 2) { sub[2] = v % static_cast<I>(a.trgt_size[2]); v /= static_cast<I>(a.trgt_size[2]); }
    if (D > 1) { sub[1] = v % static_cast<I>(a.trgt_size[1]); v /= static_cast<I>(a.trgt_size[1]); }
    sub[0] = v % static_cast<I>(a.trgt_size[0]);
    n = v / static_cast<I>(a.trgt_size[0]);
  } else {
    // 2-D tile mapping over the grid
    const I inner = static_cast<I>(a.trgt_size[D - 1]);
    const I mid = D > 1 ? static_cast<I>(a.trgt_size[D - 2]) : I(1);
    const I ntile = (inner + TILE_IN - 1) / TILE_IN;
    const I outer_idx = static_cast<I>(blockIdx.x) / ntile;
    const I ii = (static_cast<I>(blockIdx.x) - outer_idx * ntile) * TILE_IN + static_cast<I>(threadIdx.x);
    const I mm = static_cast<I>(blockIdx.y) * TILE_MID + static_cast<I>(threadIdx.y);
    if (ii >= inner || mm >= mid) return;
    if (D == 3) {
      sub[2] = ii; sub[1] = mm;
      sub[0] = outer_idx % static_cast<I>(a.trgt_size[0]);
      n = outer_idx / static_cast<I>(a.trgt_size[0]);
    } else if (D == 2) {
      sub[1] = ii; sub[0] = mm; n = outer_idx;
    } else {
      sub[0] = ii; n = outer_idx;
    }
  }

  pp_point<D, ORD, CB, S, MODE, I>(a, sub, n);
}

// Push / count with the last axis' taps spread over lanes (3-D, orders 1
// and 3): NT = taps-per-axis consecutive lanes serve one sampling point,
// lane q adding the contributions of last-axis tap q.  Consecutive lanes
// then write consecutive floats -- a point's last-axis taps, followed by the
// next point's, which in source-sorted (or natural, last axis fastest) order
// sits one voxel further along the same row -- so a reduction instruction
// touches one or two sectors instead of one or more per lane.  Each lane
// builds the whole stencil (cheap next to the reductions it saves).
//
// With CP > 0 (flag F_VEC), `out` is a float accumulator with the channels
// of a voxel interleaved in CP slots ((N, X, Y, Z, CP), CP = 2 or 4): one
// vector reduction (red.global.add.v2/v4.f32) then adds all channels of a
// tap, C times fewer reduction instructions; the host converts the
// accumulator to the output layout afterwards.  The vector form fits five
// CTAs per SM (48 registers, no spills; 1.45 -> 1.40 ms on config 2); the
// scalar forms keep MinBlocks.
template <int ORD, int CB, class S, int MODE, class I, int CP>
__global__ void __launch_bounds__(PP_THREADS, (CP > 0 ? 5 : MinBlocks<MODE>::value)) pp_lanes_kernel(const PPArgs a) {
  using T = typename Acc<S>::type;
  constexpr int NT = Taps<ORD>::value;
  constexpr int PPB = PP_THREADS / NT;  // sampling points per CTA
  const int q = static_cast<int>(threadIdx.x) % NT;
  const int64_t t = static_cast<int64_t>(blockIdx.x) * PPB + static_cast<int64_t>(threadIdx.x) / NT;
  if (t >= a.nvox) return;
  I v = a.perm != nullptr ? static_cast<I>(__ldg(a.perm + t)) : static_cast<I>(t);
  I sub[3];
  sub[2] = v % static_cast<I>(a.trgt_size[2]); v /= static_cast<I>(a.trgt_size[2]);
  sub[1] = v % static_cast<I>(a.trgt_size[1]); v /= static_cast<I>(a.trgt_size[1]);
  sub[0] = v % static_cast<I>(a.trgt_size[0]);
  const I n = v / static_cast<I>(a.trgt_size[0]);

  const T* gp = static_cast<const T*>(a.grid) + static_cast<int64_t>(n) * a.grid_sN;
  int64_t tvox = static_cast<int64_t>(n) * a.trgt_sN;
#pragma unroll
  for (int d = 0; d < 3; ++d) tvox += static_cast<int64_t>(sub[d]) * a.trgt_s[d];
  T coord[3];
  if (a.flags & F_AFFINE) {
    // coordinate A [sub; 1] (gp points at this item's 3 x 4 matrix)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      T x = __ldg(gp + d * 4 + 3);
#pragma unroll
      for (int e = 0; e < 3; ++e) x = fma(__ldg(gp + d * 4 + e), static_cast<T>(sub[e]), x);
      coord[d] = x;
    }
  } else {
#pragma unroll
    for (int d = 0; d < 3; ++d) gp += static_cast<int64_t>(sub[d]) * a.grid_s[d];
#pragma unroll
    for (int d = 0; d < 3; ++d) coord[d] = __ldg(gp + d * a.grid_sD);
  }
  {
    const T tol = (a.extrapolate & 2) ? static_cast<T>(0.5 + 5e-2) : static_cast<T>(5e-2);
    bool inb = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) inb = inb && in_fov<T>(coord[d], a.src_size[d], tol);
    if (!((a.extrapolate & 1) || inb)) return;
  }
  Axis<NT, T, I> ax, ay, az;
  build_axis<NT, false, false, false, true, T, I>(ax, ORD, a.bound[0], coord[0], static_cast<I>(a.src_size[0]),
                                                   I(0), static_cast<I>(a.out_s[0]));
  build_axis<NT, false, false, false, true, T, I>(ay, ORD, a.bound[1], coord[1], static_cast<I>(a.src_size[1]),
                                                   I(0), static_cast<I>(a.out_s[1]));
  build_axis<NT, false, false, false, true, T, I>(az, ORD, a.bound[2], coord[2], static_cast<I>(a.src_size[2]),
                                                   I(0), static_cast<I>(a.out_s[2]));
  // this lane's last-axis tap (selected without dynamic register indexing)
  T wz = T(0);
  I oz = 0;
  bool vz = false;
#pragma unroll
  for (int k = 0; k < NT; ++k)
    if (k == q) { wz = az.w[k]; oz = az.oo[k]; vz = ((az.mask >> k) & 1u) != 0u; }
  if (!vz) return;

  const S* trg_v = static_cast<const S*>(a.trgt) + tvox;
  T* outs_n = a.det_acc == nullptr ? static_cast<T*>(a.out) + static_cast<int64_t>(n) * a.out_sN : nullptr;
  unsigned long long* dacc_n = a.det_acc != nullptr ? a.det_acc + static_cast<int64_t>(n) * a.out_sN : nullptr;
  const double dscale = a.det_acc != nullptr ? det_scale(a) : 0.0;
  if constexpr (CP > 0) {
    // all channels (C <= CP) of a tap in one vector reduction
    float tv[CP];
#pragma unroll
    for (int c = 0; c < CP; ++c) tv[c] = c < a.C ? static_cast<float>(ldg_acc(trg_v + c * a.trgt_sC)) : 0.f;
    float* acc_n = static_cast<float*>(a.out) + static_cast<int64_t>(n) * a.out_sN;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const T wyz = ay.w[j] * wz;
      const I oyz = ay.oo[j] + oz;
#pragma unroll
      for (int i = 0; i < NT; ++i) {
        if ((((ax.mask >> i) & (ay.mask >> j)) & 1u) == 0u) continue;
        const float wt = static_cast<float>(ax.w[i] * wyz);
        if (wt == 0.f) continue;
        float vals[CP];
#pragma unroll
        for (int c = 0; c < CP; ++c) vals[c] = wt * tv[c];
        red_vec<CP>(acc_n + (ax.oo[i] + oyz), vals);
      }
    }
    return;
  }
  const int64_t C = MODE == K_COUNT ? 1 : a.C;
  for (int64_t c0 = 0; c0 < C; c0 += CB) {
    const int nc = C - c0 < CB ? static_cast<int>(C - c0) : CB;
    T tv[CB];
#pragma unroll
    for (int cb = 0; cb < CB; ++cb)
      tv[cb] = (MODE == K_COUNT) ? T(1) : ((CB == 1 || cb < nc) ? ldg_acc(trg_v + (c0 + cb) * a.trgt_sC) : T(0));
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const T wyz = ay.w[j] * wz;
      const I oyz = ay.oo[j] + oz;
#pragma unroll
      for (int i = 0; i < NT; ++i) {
        if ((((ax.mask >> i) & (ay.mask >> j)) & 1u) == 0u) continue;
        const T wt = ax.w[i] * wyz;
        const I off = ax.oo[i] + oyz;
#pragma unroll
        for (int cb = 0; cb < CB; ++cb) {
          if (CB == 1 || cb < nc) {
            const T val = wt * tv[cb];
            if (val == T(0)) continue;
            if (dacc_n != nullptr)
              atomicAdd(dacc_n + ((c0 + cb) * a.out_sC + off),
                        static_cast<unsigned long long>(__double2ll_rn(static_cast<double>(val) * dscale)));
            else
              atomic_acc(outs_n + ((c0 + cb) * a.out_sC + off), val);
          }
        }
      }
    }
  }
}

// Pull backward (K_PUSHGRAD) with the last axis' taps spread over lanes
// (3-D, orders 1 and 3, float arithmetic, channel-interleaved float
// accumulator for the image gradient: flag F_VEC, C <= CP).  NT consecutive
// lanes serve one sampling point, lane q its last-axis tap q:
//  * image gradient: the incoming gradient t (C channels at the point)
//    times the tap weight, one vector reduction per tap -- consecutive lanes
//    add to consecutive voxels as in pp_lanes_kernel;
//  * grid gradient: per tap, the dot product of t with the image values
//    there, weighted by the three derivative stencils; each lane sums its
//    last-axis tap, the NT partial sums are added with shuffles inside the
//    lane group and lane 0 stores them.
// Lanes of one point stay together to the end (no early return between the
// point's first and last shuffle): a missing tap contributes zero instead.
// Four CTAs per SM (64 registers): the gathers' latency is the main stall,
// and 32 warps per SM hide it better than 24 (2.50 -> 2.37 ms on config 2).
template <int ORD, class S, class I, int CP, int CB>
__global__ void __launch_bounds__(PP_THREADS, 4) pp_lanes_pullbwd_kernel(const PPArgs a) {
  using T = float;
  constexpr int NT = Taps<ORD>::value;
  constexpr int PPB = PP_THREADS / NT;
  constexpr int NC = CP > 0 ? CP : CB;  // channel slots: vector width, or the channel block
  const bool self = (a.flags & F_ADDSELF) != 0;  // self-composition (C = 3, grid = displacement)
  const int q = static_cast<int>(threadIdx.x) % NT;
  const int64_t t = static_cast<int64_t>(blockIdx.x) * PPB + static_cast<int64_t>(threadIdx.x) / NT;
  if (t >= a.nvox) return;  // whole lane groups (t is per group)
  const unsigned lanes = ((1u << NT) - 1u) << ((threadIdx.x & 31u) & ~static_cast<unsigned>(NT - 1));
  I v = a.perm != nullptr ? static_cast<I>(__ldg(a.perm + t)) : static_cast<I>(t);
  I sub[3];
  sub[2] = v % static_cast<I>(a.trgt_size[2]); v /= static_cast<I>(a.trgt_size[2]);
  sub[1] = v % static_cast<I>(a.trgt_size[1]); v /= static_cast<I>(a.trgt_size[1]);
  sub[0] = v % static_cast<I>(a.trgt_size[0]);
  const I n = v / static_cast<I>(a.trgt_size[0]);

  const T* gp = static_cast<const T*>(a.grid) + static_cast<int64_t>(n) * a.grid_sN;
  int64_t tvox = static_cast<int64_t>(n) * a.trgt_sN, gvox = static_cast<int64_t>(n) * a.gg_sN;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    tvox += static_cast<int64_t>(sub[d]) * a.trgt_s[d];
    gvox += static_cast<int64_t>(sub[d]) * a.gg_s[d];
    gp += static_cast<int64_t>(sub[d]) * a.grid_s[d];
  }
  T coord[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) coord[d] = __ldg(gp + d * a.grid_sD);
  if (a.flags & F_IDGRID) {
#pragma unroll
    for (int d = 0; d < 3; ++d) coord[d] += static_cast<T>(sub[d]);
  }
  // the point's own voxel in `out` (self-composition terms)
  T* self_out = nullptr;
  if (self) {
    int64_t oo = static_cast<int64_t>(n) * a.out_sN;
#pragma unroll
    for (int d = 0; d < 3; ++d) oo += static_cast<int64_t>(sub[d]) * a.out_s[d];
    self_out = static_cast<T*>(a.out) + oo;
  }
  const bool do_a = (a.flags & F_A) != 0;
  const bool do_grad = (a.flags & F_GRAD) != 0;
  {
    const T tol = (a.extrapolate & 2) ? static_cast<T>(0.5 + 5e-2) : static_cast<T>(5e-2);
    bool inb = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) inb = inb && in_fov<T>(coord[d], a.src_size[d], tol);
    if (!((a.extrapolate & 1) || inb)) {  // the whole group: zero grid gradient, no push
      if (self) {  // only the identity terms: g at the point
        if (q == 0) {
          const S* tp = static_cast<const S*>(a.trgt) + tvox;
#pragma unroll
          for (int d = 0; d < 3; ++d) atomic_acc(self_out + d * a.out_sC, ldg_acc(tp + d * a.trgt_sC));
        }
      } else if (do_grad && q == 0) {
        T* g = static_cast<T*>(a.gg) + gvox;
        g[0] = T(0); g[a.gg_sD] = T(0); g[2 * a.gg_sD] = T(0);
      }
      return;
    }
  }
  Axis<NT, T, I> ax, ay, az;
  build_axis<NT, true, false, true, true, T, I>(ax, ORD, a.bound[0], coord[0], static_cast<I>(a.src_size[0]),
                                                 static_cast<I>(a.src_s[0]), static_cast<I>(a.out_s[0]));
  build_axis<NT, true, false, true, true, T, I>(ay, ORD, a.bound[1], coord[1], static_cast<I>(a.src_size[1]),
                                                 static_cast<I>(a.src_s[1]), static_cast<I>(a.out_s[1]));
  build_axis<NT, true, false, true, true, T, I>(az, ORD, a.bound[2], coord[2], static_cast<I>(a.src_size[2]),
                                                 static_cast<I>(a.src_s[2]), static_cast<I>(a.out_s[2]));
  // this lane's last-axis tap (selected without dynamic register indexing)
  T wz = T(0), gz = T(0);
  I osz = 0, ooz = 0;
  bool vz = false;
#pragma unroll
  for (int k = 0; k < NT; ++k)
    if (k == q) { wz = az.w[k]; gz = az.g[k]; osz = az.os[k]; ooz = az.oo[k]; vz = ((az.mask >> k) & 1u) != 0u; }

  const S* trg_v = static_cast<const S*>(a.trgt) + tvox;
  const S* src_n = static_cast<const S*>(a.src) + static_cast<int64_t>(n) * a.src_sN;
  float* acc_n = static_cast<float*>(a.out) + static_cast<int64_t>(n) * a.out_sN;
  float tv[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) tv[c] = c < a.C ? static_cast<float>(ldg_acc(trg_v + c * a.trgt_sC)) : 0.f;
  T og0 = T(0), og1 = T(0), og2 = T(0);
  if (vz) {
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      if (((ay.mask >> j) & 1u) == 0u) continue;
      const I osyz = ay.os[j] + osz, ooyz = ay.oo[j] + ooz;
      T sx = T(0), dx = T(0);  // sum_i w_i <t, src>, sum_i g_i <t, src>
#pragma unroll
      for (int i = 0; i < NT; ++i) {
        if (((ax.mask >> i) & 1u) == 0u) continue;
        if (do_grad) {
          const S* sp = src_n + (ax.os[i] + osyz);
          T dot = T(0);
#pragma unroll
          for (int c = 0; c < NC; ++c)
            if (c < a.C) dot = fma(tv[c], ldg_acc(sp + c * a.src_sC), dot);
          sx = fma(ax.w[i], dot, sx);
          dx = fma(ax.g[i], dot, dx);
        }
        if (do_a) {
          const float wt = ax.w[i] * ay.w[j] * wz;
          if (wt != 0.f) {
            if constexpr (CP > 0) {
              float vals[CP];
#pragma unroll
              for (int c = 0; c < CP; ++c) vals[c] = wt * tv[c];
              red_vec<CP>(acc_n + (ax.oo[i] + ooyz), vals);
            } else {
#pragma unroll
              for (int c = 0; c < NC; ++c)
                if (c < a.C) atomic_acc(acc_n + (c * a.out_sC + (ax.oo[i] + ooyz)), wt * tv[c]);
            }
          }
        }
      }
      og0 = fma(ay.w[j] * wz, dx, og0);
      og1 = fma(ay.g[j] * wz, sx, og1);
      og2 = fma(ay.w[j] * gz, sx, og2);
    }
  }
  if (do_grad) {
#pragma unroll
    for (int o = 1; o < NT; o <<= 1) {
      og0 += __shfl_xor_sync(lanes, og0, o);
      og1 += __shfl_xor_sync(lanes, og1, o);
      og2 += __shfl_xor_sync(lanes, og2, o);
    }
    if (q == 0) {
      if (self) {
        // self-composition backward: g and the grid gradient at the point go
        // to the same output as the push, atomically
        const T og[3] = {og0, og1, og2};
#pragma unroll
        for (int d = 0; d < 3; ++d) atomic_acc(self_out + d * a.out_sC, og[d] + ldg_acc(trg_v + d * a.trgt_sC));
      } else {
        T* g = static_cast<T*>(a.gg) + gvox;
        g[0] = og0; g[a.gg_sD] = og1; g[2 * a.gg_sD] = og2;
      }
    }
  }
}

}  // namespace ppk

#include "pp_brick.cuh"

namespace ppk {

void note_kernel(const char* family, int mode, int ord, int cb);

// Dynamic shared memory above 48 KB must be opted into, once per kernel and
// device: `done` is the caller's per-instantiation record of the devices
// already set up (bit d = device d).
template <class K>
inline cudaError_t brick_smem_optin(K kernel, size_t bytes, std::atomic<unsigned long long>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_relaxed) & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
  // the whole unified L1 / shared array as shared memory: several CTAs of
  // these window-sized allocations per SM
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e == cudaSuccess) done.fetch_or(bit);
  return e;
}

template <int MODE, int CB, class S>
inline cudaError_t launch_brick_scatter(const PPArgs& a, cudaStream_t st) {
  constexpr int CP = CB == 1 ? 1 : (CB == 2 ? 2 : (CB == 3 ? 3 : 4));  // 3: channel planes
  constexpr size_t bytes = BrickScatterSmem<CP>::bytes;
  const int64_t nb = a.N * a.nbrick[0] * a.nbrick[1] * a.nbrick[2];
  const int64_t grid = (nb + BRK_SCATTER_WARPS - 1) / BRK_SCATTER_WARPS;
  if (grid <= 0) return cudaSuccess;
  if (grid > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  static std::atomic<unsigned long long> optin_done{0};  // one per kernel instantiation
  cudaError_t e = brick_smem_optin(pp_brick_scatter_kernel<MODE, CB, CP, S>, bytes, optin_done);
  if (e != cudaSuccess) return e;
  note_kernel("pp_brick_scatter_kernel", MODE, 3, CB);
  pp_brick_scatter_kernel<MODE, CB, CP, S><<<static_cast<unsigned>(grid), 32 * BRK_SCATTER_WARPS, bytes, st>>>(a);
  return cudaGetLastError();
}

template <int MODE, int CB, class S>
inline cudaError_t launch_brick_gather(const PPArgs& a, cudaStream_t st) {
  constexpr int CP = CB == 1 ? 1 : (CB == 2 ? 2 : 4);
  constexpr size_t bytes = BrickGatherSmem<CP>::bytes;
  const int64_t nb = a.N * a.nbrick[0] * a.nbrick[1] * a.nbrick[2];
  if (nb <= 0) return cudaSuccess;
  if (nb > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  static std::atomic<unsigned long long> optin_done{0};
  cudaError_t e = brick_smem_optin(pp_brick_gather_kernel<MODE, CB, CP, S>, bytes, optin_done);
  if (e != cudaSuccess) return e;
  note_kernel("pp_brick_gather_kernel", MODE, 3, CB);
  pp_brick_gather_kernel<MODE, CB, CP, S><<<static_cast<unsigned>(nb), BRK_GATHER_THREADS, bytes, st>>>(a);
  return cudaGetLastError();
}

template <int CB, class S>
inline cudaError_t launch_brick_pullbwd(const PPArgs& a, cudaStream_t st) {
  constexpr int CP = CB == 1 ? 1 : (CB == 2 ? 2 : 4);
  constexpr size_t bytes = PullBwdSmem<CB, CP>::bytes;
  const int64_t nb = a.N * a.nbrick[0] * a.nbrick[1] * a.nbrick[2];
  if (nb <= 0) return cudaSuccess;
  if (nb > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  static std::atomic<unsigned long long> optin_done{0};
  cudaError_t e = brick_smem_optin(pp_brick_pullbwd_kernel<CB, CP, S>, bytes, optin_done);
  if (e != cudaSuccess) return e;
  note_kernel("pp_brick_pullbwd_kernel", K_PUSHGRAD, 3, CB);
  pp_brick_pullbwd_kernel<CB, CP, S><<<static_cast<unsigned>(nb), BRK_GATHER_THREADS, bytes, st>>>(a);
  return cudaGetLastError();
}

// Brick kernels of one mode: push / count scatter; pull gather; pull
// backward = the scatter of the incoming gradient (image gradient) plus the
// gather of the grid gradient, in one kernel when both are wanted.
template <int MODE, int CB, class S>
inline cudaError_t launch_brick(const PPArgs& a, cudaStream_t st) {
  if constexpr (MODE == K_PUSH || MODE == K_COUNT) {
    return launch_brick_scatter<MODE, CB, S>(a, st);
  } else if constexpr (MODE == K_PULL) {
    return launch_brick_gather<MODE, CB, S>(a, st);
  } else {
    static_assert(MODE == K_PUSHGRAD, "brick modes");
    if ((a.flags & F_A) && (a.flags & F_GRAD)) return launch_brick_pullbwd<CB, S>(a, st);
    if (a.flags & F_A) {
      PPArgs s = a;
      s.flags &= ~F_GRAD;
      const cudaError_t e = launch_brick_scatter<K_PUSH, CB, S>(s, st);
      if (e != cudaSuccess || !(a.flags & F_GRAD)) return e;
    }
    PPArgs g = a;
    g.flags &= ~F_A;
    return launch_brick_gather<K_PUSHGRAD, CB, S>(g, st);
  }
}

// The brick kernels apply to 3-D cubic pull, push, count and the pull's
// backward pass of float arithmetic and at most four channels, given a
// brick-major order.  (The push's backward pass -- a pull with derivatives --
// measured faster as one thread per point through L1: 1.1 vs 1.3 ms on a
// 3 x 192^3 image.)
template <int D, int ORD, int MODE> struct UseBrick {
  static constexpr bool value = D == 3 && ORD == 3 &&
                                (MODE == K_PUSH || MODE == K_COUNT || MODE == K_PUSHGRAD || MODE == K_PULL);
};

// The lane-split push applies to 3-D push / count at orders 1 and 3.
template <int D, int ORD, int MODE> struct UseLanes {
  static constexpr bool value = D == 3 && (ORD == 1 || ORD == 3) && (MODE == K_PUSH || MODE == K_COUNT);
};
bool lanes_enabled();  // host switch (pp_capi.cu), on unless PP_PUSH_LANES=0
// Records, per host thread, which kernel family (and mode, order, channel
// block) the last launch used (pp_capi.cu; read back by pp_last_kernel).
void note_kernel(const char* family, int mode, int ord, int cb);

template <int D, int ORD, int CB, class S, int MODE, class I>
inline cudaError_t launch_one(const PPArgs& a, cudaStream_t st) {
  if (a.nvox == 0) return cudaSuccess;
  if constexpr (UseBrick<D, ORD, MODE>::value && std::is_same<typename Acc<S>::type, float>::value &&
                std::is_same<I, int32_t>::value) {
    if (a.brick_start != nullptr && a.perm != nullptr && a.det_acc == nullptr && a.C <= CB && lanes_enabled() &&
        !(a.flags & (F_AFFINE | F_IDGRID | F_ADDSELF | F_NOTRGT)))
      return launch_brick<MODE, CB, S>(a, st);
  }
  if constexpr (D == 3 && (ORD == 1 || ORD == 3) && MODE == K_PUSHGRAD &&
                std::is_same<typename Acc<S>::type, float>::value) {
    constexpr int PPB = PP_THREADS / Taps<ORD>::value;
    const int64_t nb = (a.nvox + PPB - 1) / PPB;
    if (lanes_enabled() && a.det_acc == nullptr && !(a.flags & (F_AFFINE | F_NOTRGT)) && nb <= 0x7fffffffLL) {
      // pull backward into the interleaved accumulator: lane-split kernel
      if constexpr (CB >= 2) {
        if (a.flags & F_VEC) {
          note_kernel("pp_lanes_pullbwd_kernel", MODE, ORD, CB);
          pp_lanes_pullbwd_kernel<ORD, S, I, (CB == 2 ? 2 : 4), CB>
              <<<static_cast<unsigned>(nb), PP_THREADS, 0, st>>>(a);
          return cudaGetLastError();
        }
      }
      // linear pull backward with up to CB channels (the self-composition
      // backward of velocity exponentiation included): lane-split with
      // scalar reductions into the output.  (Cubic single-channel images
      // measured slower this way: 1.43 -> 1.59 ms on a 192^3 grid.)
      if constexpr (ORD == 1) {
        if (!(a.flags & F_VEC) && a.C <= CB) {
          note_kernel("pp_lanes_pullbwd_kernel", MODE, ORD, CB);
          pp_lanes_pullbwd_kernel<ORD, S, I, 0, CB><<<static_cast<unsigned>(nb), PP_THREADS, 0, st>>>(a);
          return cudaGetLastError();
        }
      }
    }
  }
  if constexpr (UseLanes<D, ORD, MODE>::value) {
    if (lanes_enabled()) {
      constexpr int PPB = PP_THREADS / Taps<ORD>::value;
      const int64_t nb = (a.nvox + PPB - 1) / PPB;
      if (nb > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
      if (a.flags & F_VEC) {
        if constexpr (MODE == K_PUSH && CB >= 2 && std::is_same<typename Acc<S>::type, float>::value) {
          note_kernel("pp_lanes_kernel", MODE, ORD, CB);
          pp_lanes_kernel<ORD, CB, S, MODE, I, (CB == 2 ? 2 : 4)><<<static_cast<unsigned>(nb), PP_THREADS, 0, st>>>(a);
          return cudaGetLastError();
        }
        return cudaErrorInvalidValue;  // the host only sets F_VEC where a vector kernel exists
      }
      note_kernel("pp_lanes_kernel", MODE, ORD, CB);
      pp_lanes_kernel<ORD, CB, S, MODE, I, 0><<<static_cast<unsigned>(nb), PP_THREADS, 0, st>>>(a);
      return cudaGetLastError();
    }
  }
  const int64_t inner = a.trgt_size[D - 1];
  const int64_t mid = D > 1 ? a.trgt_size[D - 2] : 1;
  const int64_t outer = a.N * (D == 3 ? a.trgt_size[0] : 1);
  const int64_t gx = a.perm ? (a.nvox + PP_THREADS - 1) / PP_THREADS : outer * ((inner + TILE_IN - 1) / TILE_IN);
  const int64_t gy = a.perm ? 1 : (mid + TILE_MID - 1) / TILE_MID;
  if (gx > 0x7fffffffLL || gy > 65535) return cudaErrorInvalidConfiguration;
  dim3 grid(static_cast<unsigned>(gx), static_cast<unsigned>(gy), 1);
  dim3 block(TILE_IN, TILE_MID, 1);
  note_kernel("pp_kernel", MODE, ORD, CB);
  pp_kernel<D, ORD, CB, S, MODE, I><<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

// Channel block: the whole channel set when C <= 4, else groups of 4.
// Only the specialised orders up to cubic get CB > 1.
template <int D, int ORD, class S, int MODE, class I>
inline cudaError_t launch_cb(const PPArgs& a, cudaStream_t st) {
  const int64_t C = MODE == K_COUNT ? 1 : a.C;
  if constexpr (ORD >= 0 && ORD <= 3) {
    switch (C >= 4 ? 4 : static_cast<int>(C)) {
      case 2: return launch_one<D, ORD, 2, S, MODE, I>(a, st);
      case 3: return launch_one<D, ORD, 3, S, MODE, I>(a, st);
      case 4: return launch_one<D, ORD, 4, S, MODE, I>(a, st);
      default: return launch_one<D, ORD, 1, S, MODE, I>(a, st);
    }
  } else {
    return launch_one<D, ORD, 1, S, MODE, I>(a, st);
  }
}

// Orders that get a compile-time specialisation for a storage type; every
// other order (and any anisotropic order or 64-bit offset case) runs the
// runtime-order kernel (ORD = -1, 64-bit offsets).
template <class S> struct Specialised { static constexpr unsigned mask = 0; };
template <> struct Specialised<float> { static constexpr unsigned mask = 0xFFu; };
template <> struct Specialised<__nv_bfloat16> { static constexpr unsigned mask = (1u << 1) | (1u << 3); };

template <int D, class S, int MODE>
inline cudaError_t launch_ord(int ord, bool wide, const PPArgs& a, cudaStream_t st) {
  constexpr unsigned m = (D == 1) ? 0u : Specialised<S>::mask;
  if (!wide && ord >= 0) {
    switch (ord) {
#define PP_CASE(O) case O: if constexpr ((m >> O) & 1u) return launch_cb<D, O, S, MODE, int32_t>(a, st); break;
      PP_CASE(0) PP_CASE(1) PP_CASE(2) PP_CASE(3) PP_CASE(4) PP_CASE(5) PP_CASE(6) PP_CASE(7)
#undef PP_CASE
      default: break;
    }
  }
  return launch_one<D, -1, 1, S, MODE, int64_t>(a, st);
}

}  // namespace ppk

// One launcher per (storage type, dimension, mode); each is compiled in its
// own translation unit (pp_inst.cu) so the family builds in parallel.
using pp_launcher_t = cudaError_t (*)(int ord, bool wide, const ppk::PPArgs& a, cudaStream_t st);
