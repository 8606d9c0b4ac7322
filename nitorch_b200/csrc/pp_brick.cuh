// Brick kernels for 3-D cubic sampling in brick-major order.
//
// pp_brick_order sorts the sampling points by the brick (PP_BRICK_X x
// PP_BRICK_Y x PP_BRICK_Z source voxels) of their floor voxel.  A brick's
// points then touch only the brick's source window: the brick plus the cubic
// support halo, 7 x 7 x 9 voxels.  Two kernels use that window in shared
// memory.
//
// pp_brick_scatter_kernel (push, count, and the image gradient of the pull's
// backward pass).  The reference scatters every tap with a global atomic add
// (nitorch/_C/src/impl/bounds_common.h:185-191, from the tap loop of
// pushpull_common.cpp:1232-1240): 64 * C float reductions per point.  Here a
// warp owns one brick and a shared accumulator window:
//   1. the window starts at zero;
//   2. points are read 32 at a time, one per lane (coordinates, the
//      out-of-bound test, B-spline weights), into shared records;
//   3. the warp walks the recorded points one at a time, lane (i, j, kk)
//      taking taps (i, j, kk) and (i, j, kk + 2) of the 4x4x4 support:
//      plain shared read-modify-writes (the 32 lanes touch 32 distinct
//      voxels and the window belongs to this warp alone, so no atomics);
//   4. the window is added to the output with one vector reduction per
//      touched window voxel (boundary index and sign applied there), ~14x
//      fewer global reductions than one per tap.
// Float shared-memory atomics are no alternative: on B200 they sustain
// ~0.7 T adds/s on scatter-like patterns, below the ~1-1.5 T of global
// reductions.
//
// pp_brick_gather_kernel (pull, and the grid gradient of the pull's backward
// pass).  A CTA owns one brick: its
// threads stage the source window in shared memory (boundary condition
// applied per window voxel: value times sign), then each thread takes one
// point and gathers its 64 taps from the window at compile-time offsets.
//
// pp_brick_pullbwd_kernel (the pull's backward pass with both outputs) does
// the two in one pass over a brick's points: each point's coordinates and
// incoming gradient are read once for the gather of the grid gradient and
// the scatter of the image gradient.
//
// Points whose support leaves the window (sampling outside the volume with
// extrapolation, or just below a volume edge) and points outside the field
// of view run the per-point body pp_point with global memory instead.
//
// Window layout: voxel (x, y, z) of the window at (x * PX + y * PY + z) * CP
// floats, CP channel slots per voxel (1, 2 or 4).  In the scatter, with
// lane = kk + 2j + 8i and PY = 10, PX = 72 (voxels), the 32 lanes of a step
// fall in distinct banks for 4-, 8- and 16-byte voxels alike; the gather's
// pitches are chosen for its own access pattern (GatherWin).
#pragma once
#include "../../include/nitorch_b200.h"

namespace ppk {

constexpr int BRK_X = PP_BRICK_X, BRK_Y = PP_BRICK_Y, BRK_Z = PP_BRICK_Z;

// Source window of one brick for cubic taps: floor(x) in [o, o + B) has taps
// [floor(x) - 1, floor(x) + 2], inside [o - 1, o + B + 2).
struct BrickWin {
  static constexpr int LO = 1;
  static constexpr int EX = BRK_X + 3, EY = BRK_Y + 3, EZ = BRK_Z + 3;
  static constexpr int PY = 10, PX = 72;
  static constexpr int NV = EX * PX;       // storage voxels
  static constexpr int NE = EX * EY * EZ;  // window voxels
  static_assert(PY >= EZ && PX >= EY * PY, "window pitches too small");
};

// Per-point scatter record in shared memory (floats, 16-byte aligned rows):
//   [0, 4) x tap weights   [4, 8) y tap weights
//   [8, 12) z tap weights in the order 0, 2, 1, 3   [12, 16) target values
//   [16] window offset of the lowest node
constexpr int BRK_REC = 20;

constexpr int BRK_SCATTER_WARPS = 4;  // warps (bricks) per scatter CTA
constexpr int BRK_GATHER_THREADS = 128;

template <int CP> struct BrickScatterSmem {
  static constexpr int PER_WARP = BrickWin::NV * CP + 32 * BRK_REC;  // floats
  static constexpr size_t bytes = size_t(PER_WARP) * 4 * BRK_SCATTER_WARPS;
};
// The gather kernel's window: the same extents, pitches for thread-per-point
// reads.  Eight consecutive points of a brick (one phase of a 16-byte shared
// load) are mostly runs along z of one or two (x, y) columns: with
// PY = 6 (mod 8) and PX = 0 (mod 8) voxels such runs fall in distinct
// 16-byte bank groups.
struct GatherWin {
  static constexpr int PY = 14, PX = 104;
  static constexpr int NV = BrickWin::EX * PX;
  static_assert(PY >= BrickWin::EZ && PX >= BrickWin::EY * PY, "window pitches too small");
};
template <int CP> struct BrickGatherSmem {
  static constexpr size_t bytes = size_t(GatherWin::NV) * CP * 4;
};
// Resident CTAs per SM the gather kernels are built for (register caps).
// (single-channel pulls: eight, 64 registers; single-channel grid
// gradients: five, 96 registers; both without spills, where more channels
// spill and keep six and four)
template <int MODE, int CB> struct GatherBlocks {
  static constexpr int value = MODE == K_PULL ? (CB == 1 ? 8 : 6) : (CB == 1 ? 5 : 4);
};

template <int CP> __device__ __forceinline__ void vload(const float* p, float (&v)[CP]) {
  if constexpr (CP == 4) { const float4 q = *reinterpret_cast<const float4*>(p); v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w; }
  else if constexpr (CP == 2) { const float2 q = *reinterpret_cast<const float2*>(p); v[0] = q.x; v[1] = q.y; }
  else v[0] = *p;
}
template <int CP> __device__ __forceinline__ void vstore(float* p, const float (&v)[CP]) {
  if constexpr (CP == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  else if constexpr (CP == 2) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  else *p = v[0];
}

// acc[p .. p + CP) += w * t
template <int CP> __device__ __forceinline__ void vaxpy(float* p, float w, const float (&t)[CP]) {
  float v[CP];
  vload<CP>(p, v);
#pragma unroll
  for (int c = 0; c < CP; ++c) v[c] = fmaf(w, t[c], v[c]);
  vstore<CP>(p, v);
}

// Accumulator windows of the scatters, by voxel: CP = 1, 2, 4 channel slots
// interleaved per voxel; CP = 3 three channel planes BrickWin::NV floats
// apart (no padding slot: a quarter less shared-memory traffic per tap).
template <int CP> __device__ __forceinline__ void win_axpy(float* acc, int vox, float w, const float (&t)[CP]) {
  if constexpr (CP == 3) {
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c * BrickWin::NV + vox] = fmaf(w, t[c], acc[c * BrickWin::NV + vox]);
  } else {
    vaxpy<CP>(acc + vox * CP, w, t);
  }
}
template <int CP> __device__ __forceinline__ void win_get(const float* acc, int vox, float (&v)[CP]) {
  if constexpr (CP == 3) {
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = acc[c * BrickWin::NV + vox];
  } else {
    vload<CP>(acc + vox * CP, v);
  }
}

// Brick b of the scatter target / gathered source: batch item, window origin
// (absolute voxel of window voxel 0) and whether the window lies inside the
// volume on every axis.
struct BrickPos {
  int n, ox, oy, oz;
  bool interior;
};
__device__ __forceinline__ BrickPos brick_pos(const PPArgs& a, int64_t b) {
  using W = BrickWin;
  BrickPos q;
  int64_t r = b;
  const int bz = static_cast<int>(r % a.nbrick[2]); r /= a.nbrick[2];
  const int by = static_cast<int>(r % a.nbrick[1]); r /= a.nbrick[1];
  const int bx = static_cast<int>(r % a.nbrick[0]);
  q.n = static_cast<int>(r / a.nbrick[0]);
  q.ox = bx * BRK_X - W::LO;
  q.oy = by * BRK_Y - W::LO;
  q.oz = bz * BRK_Z - W::LO;
  q.interior = q.ox >= 0 && q.oy >= 0 && q.oz >= 0 && q.ox + W::EX <= a.src_size[0] &&
               q.oy + W::EY <= a.src_size[1] && q.oz + W::EZ <= a.src_size[2];
  return q;
}

// Window voxel e (x slowest, z fastest) -> window coordinates.
__device__ __forceinline__ void win_coords(int e, int& wx, int& wy, int& wz) {
  using W = BrickWin;
  wx = e / (W::EY * W::EZ);
  const int rem = e - wx * (W::EY * W::EZ);
  wy = rem / W::EZ;
  wz = rem - wy * W::EZ;
}

// Offset (elements) and sign of absolute voxel (X, Y, Z) under the bound
// condition, for strides s[]; sign 0 = outside (zero bound, dst nodes).
__device__ __forceinline__ int64_t bound_offset(const PPArgs& a, int X, int Y, int Z, const int64_t (&s)[3],
                                                bool interior, int& sgn) {
  if (interior) {
    sgn = 1;
    return X * s[0] + Y * s[1] + Z * s[2];
  }
  const int nX = static_cast<int>(a.src_size[0]), nY = static_cast<int>(a.src_size[1]),
            nZ = static_cast<int>(a.src_size[2]);
  sgn = bound_sign<int>(a.bound[0], X, nX) * bound_sign<int>(a.bound[1], Y, nY) * bound_sign<int>(a.bound[2], Z, nZ);
  return bound_index<int>(a.bound[0], X, nX) * s[0] + bound_index<int>(a.bound[1], Y, nY) * s[1] +
         bound_index<int>(a.bound[2], Z, nZ) * s[2];
}

// One sampling point of a brick: its grid position, coordinates and whether
// its 4x4x4 support lies in the brick's window (lo: lowest support node).
struct BrickPoint {
  int sub[3], n;
  float x[3];
  int lo[3];
  bool fits;
};
// The point of sample index v at coordinates x (batch item, grid voxel, fit).
__device__ __forceinline__ BrickPoint brick_point_of(const PPArgs& a, int v, float x0, float x1, float x2,
                                                     const BrickPos& bp) {
  using W = BrickWin;
  BrickPoint q;
  q.x[0] = x0;
  q.x[1] = x1;
  q.x[2] = x2;
  q.sub[2] = v % static_cast<int>(a.trgt_size[2]); v /= static_cast<int>(a.trgt_size[2]);
  q.sub[1] = v % static_cast<int>(a.trgt_size[1]); v /= static_cast<int>(a.trgt_size[1]);
  q.sub[0] = v % static_cast<int>(a.trgt_size[0]);
  q.n = v / static_cast<int>(a.trgt_size[0]);
  const float tol = (a.extrapolate & 2) ? 0.55f : 0.05f;
  bool inb = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) inb = inb && in_fov<float>(q.x[d], a.src_size[d], tol);
  // window fit: lowest node floor(x) - 1 within [o, o + E - 4] on every axis
  q.fits = q.n == bp.n && ((a.extrapolate & 1) || inb);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float xc = fminf(fmaxf(q.x[d], -1073741824.f), 1073741824.f);
    q.lo[d] = static_cast<int>(floorf(xc)) - 1;
    const int o = d == 0 ? bp.ox : (d == 1 ? bp.oy : bp.oz);
    const int e = d == 0 ? W::EX : (d == 1 ? W::EY : W::EZ);
    q.fits = q.fits && q.lo[d] >= o && q.lo[d] <= o + e - 4;
  }
  return q;
}

// Sample p (in brick order): from its record, or through perm and the grid.
__device__ __forceinline__ BrickPoint brick_point(const PPArgs& a, int p, const BrickPos& bp) {
  if (a.brec) {  // coordinates and index in one record, in brick order
    const float4 r = __ldg(a.brec + p);
    return brick_point_of(a, __float_as_int(r.w), r.x, r.y, r.z, bp);
  }
  const int v = __ldg(a.perm + p);
  int r = v;
  const int s2 = r % static_cast<int>(a.trgt_size[2]); r /= static_cast<int>(a.trgt_size[2]);
  const int s1 = r % static_cast<int>(a.trgt_size[1]); r /= static_cast<int>(a.trgt_size[1]);
  const int s0 = r % static_cast<int>(a.trgt_size[0]);
  const int n = r / static_cast<int>(a.trgt_size[0]);
  const float* gp = static_cast<const float*>(a.grid) + static_cast<int64_t>(n) * a.grid_sN + s0 * a.grid_s[0] +
                    s1 * a.grid_s[1] + s2 * a.grid_s[2];
  return brick_point_of(a, v, __ldg(gp), __ldg(gp + a.grid_sD), __ldg(gp + 2 * a.grid_sD), bp);
}

// ===========================================================================
// Pieces shared by the brick kernels.
// ===========================================================================

// Weights, target values and window offset of one point, written to its
// shared scatter record (layout above).
__device__ __forceinline__ void write_record(const BrickPoint& q, const BrickPos& bp, const float (&w)[3][4],
                                             const float (&t)[4], float* rr) {
  using W = BrickWin;
  *reinterpret_cast<float4*>(rr + 0) = make_float4(w[0][0], w[0][1], w[0][2], w[0][3]);
  *reinterpret_cast<float4*>(rr + 4) = make_float4(w[1][0], w[1][1], w[1][2], w[1][3]);
  *reinterpret_cast<float4*>(rr + 8) = make_float4(w[2][0], w[2][2], w[2][1], w[2][3]);
  *reinterpret_cast<float4*>(rr + 12) = make_float4(t[0], t[1], t[2], t[3]);
  rr[16] = __int_as_float((q.lo[0] - bp.ox) * W::PX + (q.lo[1] - bp.oy) * W::PY + (q.lo[2] - bp.oz));
}

// The warp walks its recorded points (bit set in `todo`) one at a time,
// lane (i, j, kk) adding taps (i, j, kk) and (i, j, kk + 2) of the 4x4x4
// support into the warp's accumulator window.
template <int CP>
__device__ __forceinline__ void scatter_recorded(float* acc, const float* rec, unsigned todo, int lane) {
  using W = BrickWin;
  const int ti = lane >> 3, tj = (lane >> 1) & 3, tk = lane & 1;
  const int loff = ti * W::PX + tj * W::PY + tk;
  while (todo) {
    const int q = __ffs(todo) - 1;
    todo &= todo - 1;
    const float* rr = rec + q * BRK_REC;
    const float wxy = rr[ti] * rr[4 + tj];
    const float2 zp = *reinterpret_cast<const float2*>(rr + 8 + 2 * tk);  // (wz_k, wz_k+2)
    float t[CP];
    {
      const float4 tq = *reinterpret_cast<const float4*>(rr + 12);
      const float tt[4] = {tq.x, tq.y, tq.z, tq.w};
#pragma unroll
      for (int c = 0; c < CP; ++c) t[c] = tt[c];
    }
    const int vox0 = __float_as_int(rr[16]) + loff;
    win_axpy<CP>(acc, vox0, wxy * zp.x, t);
    win_axpy<CP>(acc, vox0 + 2, wxy * zp.y, t);
    __syncwarp();
  }
}

// Add NACC accumulator windows (`stride` floats apart) of brick bp to the
// output: one vector reduction per touched window voxel, boundary index and
// sign applied; threads `tid` of `nthreads`.
template <int CP, int NACC>
__device__ __forceinline__ void flush_windows(const PPArgs& a, const BrickPos& bp, const float* acc, int stride,
                                              int tid, int nthreads) {
  using W = BrickWin;
  float* out_n = static_cast<float*>(a.out) + static_cast<int64_t>(bp.n) * a.out_sN;
  const bool vec = (a.flags & F_VEC) != 0;
  const int64_t os[3] = {a.out_s[0], a.out_s[1], a.out_s[2]};
  for (int e = tid; e < W::NE; e += nthreads) {
    int wx, wy, wz;
    win_coords(e, wx, wy, wz);
    const int vox = wx * W::PX + wy * W::PY + wz;
    float v[CP];
    win_get<CP>(acc, vox, v);
#pragma unroll
    for (int k = 1; k < NACC; ++k) {
      float u[CP];
      win_get<CP>(acc + k * stride, vox, u);
#pragma unroll
      for (int c = 0; c < CP; ++c) v[c] += u[c];
    }
    bool any = false;
#pragma unroll
    for (int c = 0; c < CP; ++c) any = any || v[c] != 0.f;
    if (!any) continue;
    int sgn;
    const int64_t off = bound_offset(a, bp.ox + wx, bp.oy + wy, bp.oz + wz, os, bp.interior, sgn);
    if (sgn == 0) continue;
    if (sgn < 0) {
#pragma unroll
      for (int c = 0; c < CP; ++c) v[c] = -v[c];
    }
    if constexpr (CP == 3) {
      if (vec) {  // the interleaved accumulator has four slots for three channels
        const float v4[4] = {v[0], v[1], v[2], 0.f};
        red_vec<4>(out_n + off, v4);
        continue;
      }
    } else if constexpr (CP >= 2) {
      if (vec) {
        red_vec<CP>(out_n + off, v);
        continue;
      }
    }
#pragma unroll
    for (int c = 0; c < CP; ++c)
      if (c < a.C && v[c] != 0.f) atomicAdd(out_n + c * a.out_sC + off, v[c]);
  }
}

// The source window of brick bp at GatherWin pitches (value times boundary
// sign; 0 outside), in two halves: window_load issues every load of this
// thread into registers, window_store writes them to shared memory.
template <int NTHR> struct WinRegs {
  static constexpr int NIT = (BrickWin::NE + NTHR - 1) / NTHR;
};
template <int CB, int CP, class S, int NTHR>
__device__ __forceinline__ void window_load(const PPArgs& a, const BrickPos& bp,
                                            float (&v)[WinRegs<NTHR>::NIT][CP], int (&dst)[WinRegs<NTHR>::NIT]) {
  using W = BrickWin;
  using G = GatherWin;
  constexpr int NIT = WinRegs<NTHR>::NIT;
  const S* src_n = static_cast<const S*>(a.src) + static_cast<int64_t>(bp.n) * a.src_sN;
  const int64_t ss[3] = {a.src_s[0], a.src_s[1], a.src_s[2]};
#pragma unroll
  for (int it = 0; it < NIT; ++it) {
    const int e = static_cast<int>(threadIdx.x) + it * NTHR;
#pragma unroll
    for (int c = 0; c < CP; ++c) v[it][c] = 0.f;
    dst[it] = -1;
    if (e < W::NE) {
      int wx, wy, wz;
      win_coords(e, wx, wy, wz);
      dst[it] = (wx * G::PX + wy * G::PY + wz) * CP;
      int sgn;
      const int64_t so = bound_offset(a, bp.ox + wx, bp.oy + wy, bp.oz + wz, ss, bp.interior, sgn);
      if (sgn != 0) {
#pragma unroll
        for (int c = 0; c < CP; ++c)
          if (c < CB && c < a.C)
            v[it][c] = static_cast<float>(sgn) * static_cast<float>(ldg_acc(src_n + c * a.src_sC + so));
      }
    }
  }
}
template <int CP, int NTHR>
__device__ __forceinline__ void window_store(float* img, const float (&v)[WinRegs<NTHR>::NIT][CP],
                                             const int (&dst)[WinRegs<NTHR>::NIT]) {
#pragma unroll
  for (int it = 0; it < WinRegs<NTHR>::NIT; ++it)
    if (dst[it] >= 0) vstore<CP>(img + dst[it], v[it]);
}

// Stage the source window of brick bp: every thread issues all of its loads
// before its first shared store.
template <int CB, int CP, class S, int NTHR>
__device__ __forceinline__ void stage_window(const PPArgs& a, const BrickPos& bp, float* img) {
  float v[WinRegs<NTHR>::NIT][CP];
  int dst[WinRegs<NTHR>::NIT];
  window_load<CB, CP, S, NTHR>(a, bp, v, dst);
  window_store<CP, NTHR>(img, v, dst);
}

// One point's 64-tap gather from the staged window `ib` (its lowest node):
// separable partial sums, x innermost; per channel the interpolant (VAL),
// and for the grid gradient (GG) the dot product with t under w and dw.
template <int CB, int CP, bool VAL, bool GG>
__device__ __forceinline__ void gather_taps(const float* ib, const float (&w)[3][4], const float (&g)[3][4],
                                            const float (&t)[CP], float (&val)[CP], float& gx, float& gy,
                                            float& gz) {
  using G = GatherWin;
  gx = gy = gz = 0.f;
#pragma unroll
  for (int c = 0; c < CP; ++c) val[c] = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float yv[CP], yw = 0.f, ygx = 0.f, ygy = 0.f;
#pragma unroll
    for (int c = 0; c < CP; ++c) yv[c] = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float xv[CP], sx = 0.f, sdx = 0.f;
#pragma unroll
      for (int c = 0; c < CP; ++c) xv[c] = 0.f;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        float iv[CP];
        vload<CP>(ib + (i * G::PX + j * G::PY + k) * CP, iv);
        if (VAL) {
#pragma unroll
          for (int c = 0; c < CP; ++c)
            if (c < CB) xv[c] = fmaf(w[0][i], iv[c], xv[c]);
        }
        if (GG) {
          float dot = 0.f;
#pragma unroll
          for (int c = 0; c < CP; ++c)
            if (c < CB) dot = fmaf(t[c], iv[c], dot);
          sx = fmaf(w[0][i], dot, sx);
          sdx = fmaf(g[0][i], dot, sdx);
        }
      }
      if (VAL) {
#pragma unroll
        for (int c = 0; c < CP; ++c)
          if (c < CB) yv[c] = fmaf(w[1][j], xv[c], yv[c]);
      }
      if (GG) {
        yw = fmaf(w[1][j], sx, yw);
        ygx = fmaf(w[1][j], sdx, ygx);
        ygy = fmaf(g[1][j], sx, ygy);
      }
    }
    if (VAL) {
#pragma unroll
      for (int c = 0; c < CP; ++c)
        if (c < CB) val[c] = fmaf(w[2][k], yv[c], val[c]);
    }
    if (GG) {
      gx = fmaf(w[2][k], ygx, gx);
      gy = fmaf(w[2][k], ygy, gy);
      gz = fmaf(g[2][k], yw, gz);
    }
  }
}

// The target values of a point (CB channels, zero in the other slots).
template <int CB, int NS, class S>
__device__ __forceinline__ void load_target(const PPArgs& a, const BrickPoint& q, float (&t)[NS]) {
  const S* tp = static_cast<const S*>(a.trgt) + static_cast<int64_t>(q.n) * a.trgt_sN + q.sub[0] * a.trgt_s[0] +
                q.sub[1] * a.trgt_s[1] + q.sub[2] * a.trgt_s[2];
#pragma unroll
  for (int c = 0; c < NS; ++c) t[c] = (c < CB && c < a.C) ? static_cast<float>(ldg_acc(tp + c * a.trgt_sC)) : 0.f;
}

// ===========================================================================
// Scatter: one warp per brick (see the file comment).  CB: channel block of
// the per-point fallback body (= C for C <= 4); CP: channel slots per window
// voxel (1 for C = 1, 2 for C = 2, 4 for C = 3-4).
// ===========================================================================
// Six CTAs per SM (at most 85 registers; no spills): the shared-memory
// budget of 3-channel windows holds six.
template <int MODE, int CB, int CP, class S>
__global__ void __launch_bounds__(32 * BRK_SCATTER_WARPS, 6) pp_brick_scatter_kernel(const PPArgs a) {
  using W = BrickWin;
  using SM = BrickScatterSmem<CP>;
  static_assert(MODE == K_PUSH || MODE == K_COUNT, "scatter modes");
  extern __shared__ float4 brick_smem4[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  float* acc = reinterpret_cast<float*>(brick_smem4) + wid * SM::PER_WARP;
  float* rec = acc + W::NV * CP;

  const int64_t nbricks = a.N * a.nbrick[0] * a.nbrick[1] * a.nbrick[2];
  const int64_t b = static_cast<int64_t>(blockIdx.x) * BRK_SCATTER_WARPS + wid;
  if (b >= nbricks) return;  // whole warp
  const int p0 = __ldg(a.brick_start + b), p1 = __ldg(a.brick_start + b + 1);
  if (p0 >= p1) return;
  const BrickPos bp = brick_pos(a, b);

  {
    float4* a4 = reinterpret_cast<float4*>(acc);
    for (int e = lane; e < W::NV * CP / 4; e += 32) a4[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncwarp();

  for (int c0 = p0; c0 < p1; c0 += 32) {
    const int p = c0 + lane;
    bool mine = false;
    if (p < p1) {
      const BrickPoint q = brick_point(a, p, bp);
      if (!q.fits) {
        pp_point<3, 3, CB, S, MODE, int>(a, q.sub, q.n);  // global reductions
      } else {
        mine = true;
        float w[3][4], g[3][4], h[3][4];
#pragma unroll
        for (int d = 0; d < 3; ++d)
          bspline_stencil<4, false, false, float>(3, q.x[d] - static_cast<float>(q.lo[d] + 1), w[d], g[d], h[d]);
        float t[4] = {1.f, 0.f, 0.f, 0.f};
        if (MODE != K_COUNT) load_target<CB, 4, S>(a, q, t);
        write_record(q, bp, w, t, rec + lane * BRK_REC);
      }
    }
    const unsigned todo = __ballot_sync(0xffffffffu, mine);
    __syncwarp();
    scatter_recorded<CP>(acc, rec, todo, lane);
  }

  flush_windows<CP, 1>(a, bp, acc, 0, lane, 32);
}

// ===========================================================================
// Gather: one CTA per brick, one thread per point.  Modes:
//   K_PULL      out[c] = sum w src[c]
//   K_PUSHGRAD  pull backward's grid gradient only (flag F_GRAD, no F_A):
//               gg_d = sum_c t[c] sum dw_d src[c], src the pulled image and
//               t the incoming gradient at the point
// ===========================================================================
template <int MODE, int CB, int CP, class S>
__global__ void __launch_bounds__(BRK_GATHER_THREADS, GatherBlocks<MODE, CB>::value)
    pp_brick_gather_kernel(const PPArgs a) {
  using G = GatherWin;
  static_assert(MODE == K_PULL || MODE == K_PUSHGRAD, "gather modes");
  constexpr bool GG = MODE != K_PULL;
  extern __shared__ float4 brick_smem4[];
  float* img = reinterpret_cast<float*>(brick_smem4);

  const int64_t b = blockIdx.x;
  const int p0 = __ldg(a.brick_start + b), p1 = __ldg(a.brick_start + b + 1);
  if (p0 >= p1) return;  // whole CTA
  const BrickPos bp = brick_pos(a, b);
  constexpr bool want_val = MODE == K_PULL;
  const bool want_gg = GG && (a.flags & F_GRAD) != 0;

  stage_window<CB, CP, S, BRK_GATHER_THREADS>(a, bp, img);
  __syncthreads();

  for (int p = p0 + static_cast<int>(threadIdx.x); p < p1; p += BRK_GATHER_THREADS) {
    const BrickPoint q = brick_point(a, p, bp);
    if (!q.fits) {
      pp_point<3, 3, CB, S, MODE, int>(a, q.sub, q.n);  // global memory
      continue;
    }
    float w[3][4], g[3][4], h[3][4];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      bspline_stencil<4, GG, false, float>(3, q.x[d] - static_cast<float>(q.lo[d] + 1), w[d], g[d], h[d]);
    float t[CP];
#pragma unroll
    for (int c = 0; c < CP; ++c) t[c] = 0.f;
    if (GG && want_gg) load_target<CB, CP, S>(a, q, t);
    const float* ib = img + ((q.lo[0] - bp.ox) * G::PX + (q.lo[1] - bp.oy) * G::PY + (q.lo[2] - bp.oz)) * CP;
    float val[CP], gx, gy, gz;
    if (want_val) {
      gather_taps<CB, CP, true, false>(ib, w, g, t, val, gx, gy, gz);
      S* op = static_cast<S*>(a.out) + static_cast<int64_t>(q.n) * a.out_sN + q.sub[0] * a.out_s[0] +
              q.sub[1] * a.out_s[1] + q.sub[2] * a.out_s[2];
#pragma unroll
      for (int c = 0; c < CP; ++c)
        if (c < CB && c < a.C) op[c * a.out_sC] = from_acc<S>(val[c]);
    }
    if (GG && want_gg) {
      gather_taps<CB, CP, false, true>(ib, w, g, t, val, gx, gy, gz);
      float* gg = static_cast<float*>(a.gg) + static_cast<int64_t>(q.n) * a.gg_sN + q.sub[0] * a.gg_s[0] +
                  q.sub[1] * a.gg_s[1] + q.sub[2] * a.gg_s[2];
      gg[0] = gx; gg[a.gg_sD] = gy; gg[2 * a.gg_sD] = gz;
    }
  }
}

// ===========================================================================
// Pull backward in one pass over a brick's points (flags F_A and F_GRAD):
// one CTA per brick, one thread per point.  Each point's coordinates and
// incoming gradient t are read once and serve both outputs:
//   grid gradient  gg_d = sum_c t[c] sum dw_d src[c]  (gather from the staged
//                  source window, as pp_brick_gather_kernel)
//   image gradient out[c] += w t[c]  (scatter: each warp records its lanes'
//                  points and adds them into its own accumulator window, as
//                  pp_brick_scatter_kernel; the four windows are summed and
//                  flushed once at the end)
// ===========================================================================
template <int CB, int CP> struct PullBwdSmem {
  static constexpr int CPS = CB == 3 ? 3 : CP;     // accumulator layout (3: channel planes)
  static constexpr int ACC = BrickWin::NV * CPS;   // floats per accumulator window
  static constexpr int IMG = GatherWin::NV * CP;
  static constexpr int NWARP = BRK_GATHER_THREADS / 32;
  static_assert(NWARP == 4, "the scatter shares points out by k mod 4 (mask 0x11111111 << warp)");
  static constexpr size_t bytes = (size_t(IMG) + size_t(NWARP) * (ACC + 32 * BRK_REC)) * 4;
};

template <int CB, int CP, class S>
__global__ void __launch_bounds__(BRK_GATHER_THREADS, 4) pp_brick_pullbwd_kernel(const PPArgs a) {
  using W = BrickWin;
  using G = GatherWin;
  using SM = PullBwdSmem<CB, CP>;
  extern __shared__ float4 brick_smem4[];
  __shared__ unsigned recorded[SM::NWARP];     // per warp: lanes that recorded a point
  float* img = reinterpret_cast<float*>(brick_smem4);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  float* acc0 = img + SM::IMG;                 // NWARP windows, SM::ACC floats apart
  float* acc = acc0 + wid * SM::ACC;
  float* rec = acc0 + SM::NWARP * SM::ACC;     // one record per thread of the CTA

  const int64_t b = blockIdx.x;
  const int p0 = __ldg(a.brick_start + b), p1 = __ldg(a.brick_start + b + 1);
  if (p0 >= p1) return;  // whole CTA
  const BrickPos bp = brick_pos(a, b);

  stage_window<CB, CP, S, BRK_GATHER_THREADS>(a, bp, img);
  {
    float4* a4 = reinterpret_cast<float4*>(acc0);
    for (int e = threadIdx.x; e < SM::NWARP * SM::ACC / 4; e += BRK_GATHER_THREADS)
      a4[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();

  for (int c0 = p0; c0 < p1; c0 += BRK_GATHER_THREADS) {
    const int p = c0 + static_cast<int>(threadIdx.x);
    bool mine = false;
    if (p < p1) {
      const BrickPoint q = brick_point(a, p, bp);
      if (!q.fits) {
        pp_point<3, 3, CB, S, K_PUSHGRAD, int>(a, q.sub, q.n);  // both outputs, global memory
      } else {
        mine = true;
        float w[3][4], g[3][4], h[3][4];
#pragma unroll
        for (int d = 0; d < 3; ++d)
          bspline_stencil<4, true, false, float>(3, q.x[d] - static_cast<float>(q.lo[d] + 1), w[d], g[d], h[d]);
        float t4[4];
        load_target<CB, 4, S>(a, q, t4);
        float t[CP];
#pragma unroll
        for (int c = 0; c < CP; ++c) t[c] = t4[c];
        const float* ib = img + ((q.lo[0] - bp.ox) * G::PX + (q.lo[1] - bp.oy) * G::PY + (q.lo[2] - bp.oz)) * CP;
        float val[CP], gx, gy, gz;
        gather_taps<CB, CP, false, true>(ib, w, g, t, val, gx, gy, gz);
        float* gg = static_cast<float*>(a.gg) + static_cast<int64_t>(q.n) * a.gg_sN + q.sub[0] * a.gg_s[0] +
                    q.sub[1] * a.gg_s[1] + q.sub[2] * a.gg_s[2];
        gg[0] = gx; gg[a.gg_sD] = gy; gg[2 * a.gg_sD] = gz;
        write_record(q, bp, w, t4, rec + threadIdx.x * BRK_REC);
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, mine);
    if (lane == 0) recorded[wid] = m;
    __syncthreads();
    // warp w adds the recorded points k = w (mod NWARP) of this pass into
    // its own window: an even share whatever the number of points
    for (int s = 0; s < SM::NWARP; ++s)
      scatter_recorded<SM::CPS>(acc, rec + s * 32 * BRK_REC, recorded[s] & (0x11111111u << wid), lane);
    __syncthreads();  // records and masks are rewritten by the next pass
  }
  flush_windows<SM::CPS, SM::NWARP>(a, bp, acc0, SM::ACC, static_cast<int>(threadIdx.x), BRK_GATHER_THREADS);
}

}  // namespace ppk
