// Separable resampling at diagonal affine coordinates (resize): TMA-staged
// tiles and three one-dimensional passes.
//
// nitorch resizes an image by pulling it through the grid of a diagonal
// affine map, x_d = scale_d * o_d + shift_d (nitorch/spatial/_grid.py:618-754
// builds affine_grid and calls grid_pull; its native ni::resize,
// nitorch/_C/src/impl/resize_common.cpp:600-700, evaluates the same sum voxel
// by voxel).  With a diagonal map every output index o_d has one 1-D stencil
// per axis (its support nodes and B-spline weights), so the 64-tap cubic sum
// factors into three 4-tap passes.  One CTA per output tile of
// TX x TY x TZ voxels (z contiguous in memory):
//   1. per axis, each output index's lowest node, weights and field-of-view
//      test go to shared tables;
//   2. per channel, the input region the tile reads -- its nodes from the
//      tile's first to last output, per axis -- is staged in shared memory
//      by one TMA tensor copy (cp.async.bulk.tensor, mbarrier completion);
//      staged voxels outside the volume are then rewritten under the
//      boundary condition (sign times the mapped voxel, which the staged
//      region usually holds already);
//   3. x pass: T1[ox][y][z] = sum_i wx_i S[lx + i][y][z] over the staged y, z;
//      y pass: T2[ox][oy][z] = sum_j wy_j T1[ox][ly + j][z];
//      z pass: out = sum_k wz_k T2[ox][oy][lz + k], stored along z.
// Each partial sum is the fused multiply-add chain of the per-point kernel
// (x innermost, then y, then z, starting from zero), so the result equals
// pp_grid_pull's on the materialised affine grid.  Persistent CTAs walk the
// (tile, channel) items with two staging buffers: the next item's copy is
// in flight while the current item is filtered; the x and y passes move
// four z positions per thread (16-byte shared accesses).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "pp_capi_internal.cuh"

namespace ppk {
void note_kernel(const char* family, int mode, int ord, int cb);  // pp_capi.cu
}

namespace {

using namespace ppk;

constexpr int RZ_THREADS = 256;
constexpr int RZ_MAXT = 64;   // largest tile edge (tables)
constexpr int RZ_MAXE = 256;  // largest staged extent (boundary tables)

struct ResizeArgs {
  const void* src;
  void* out;
  int N, C;
  int in_size[3], out_size[3];
  int64_t src_sN, src_sC, src_s[3];
  int64_t out_sN, out_sC, out_s[3];
  float scale[3], shift[3];
  int bound[3], order;
  int extrapolate;
  int kind;  // 0: B-spline at scale * o + shift (field-of-view test); 1: multigrid
             // restriction, 2: multigrid prolongation (both at (o + 1/2) scale - 1/2)
  int tile[3];  // TX, TY, TZ
  int ext[3];   // staged extents EX, EY, EZ (EZ a multiple of 4: the TMA box)
  int ntile[3];
  int zls;  // log2 of the lanes per staged z row in the x and y passes (2^zls >= EZ / 4, at most 32)
  int use_tma;
};

__device__ unsigned int g_resize_status = 0;  // bit 0: a TMA wait gave up

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// Wait for phase `phase` of the mbarrier: try_wait with a suspend-time hint
// (1 ms), at most 4096 tries (a few seconds) before giving up.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned phase) {
  for (unsigned it = 0; it < 4096u; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar), "r"(phase), "r"(1000000u)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Per-axis stencil of output index o: lowest node, weights, field of view.
// Kinds 1 and 2 follow nitorch's multigrid operators
// (nitorch/_C/src/impl/multires_common.cpp:419-500, 587-660): the output
// voxel centre maps to x = (o + 1/2) scale - 1/2 in input voxels, with no
// field-of-view test; restriction (kind 1) weights the four nodes from
// floor(x) - 1 by the linear B-spline of width `scale`, L(|x - i| / scale) /
// scale; prolongation (kind 2) is the quadratic B-spline at x.
template <int NT>
__device__ __forceinline__ void axis_stencil(const ResizeArgs& a, int d, int o, int& lo, float (&w)[NT], bool& inb) {
  float x;
  if (a.kind == 0) {
    x = fmaf(a.scale[d], static_cast<float>(o), a.shift[d]);
    const float tol = (a.extrapolate & 2) ? 0.55f : 0.05f;
    inb = in_fov<float>(x, a.in_size[d], tol);
  } else {
    x = (static_cast<float>(o) + 0.5f) * a.scale[d] - 0.5f;
    inb = true;
  }
  x = fminf(fmaxf(x, -1073741824.f), 1073741824.f);
  if (NT == 4 && a.kind == 1) {
    const float s = a.scale[d];
    lo = static_cast<int>(floorf(x)) - 1;
#pragma unroll
    for (int k = 0; k < NT; ++k) {
      const float t = fabsf(x - static_cast<float>(lo + k)) / s;
      w[k] = (t < 1.f ? 1.f - t : 0.f) / s;
    }
    return;
  }
  lo = support_low<int, float>(a.order, x);
  const float f = (x - static_cast<float>(lo)) - 0.5f * static_cast<float>(a.order - 1);
  float g[NT], h[NT];
  bspline_stencil<NT, false, false, float>(a.order, a.order == 0 ? 0.f : f, w, g, h);
}

// One work item: channel c of output tile t (items are channel-minor).
struct RzItem {
  int n, c, o0[3], tn[3];
  int base[3];      // first staged node per axis (z on a 16-byte boundary)
  int fits;         // the tile's nodes lie within the staged extents
  int interior;     // ... and inside the volume
};

// Item setup by the 32 lanes of warp 0: lane d < 3 handles axis d.
template <int NT>
__device__ void rz_item(const ResizeArgs& a, int item, RzItem& it) {
  const int lane = threadIdx.x & 31;
  const int t = item / a.C;
  int r = t;
  const int tz = r % a.ntile[2]; r /= a.ntile[2];
  const int ty = r % a.ntile[1]; r /= a.ntile[1];
  const int tx = r % a.ntile[0];
  bool fits = true, interior = true;
  if (lane < 3) {
    const int d = lane;
    const int o0 = (d == 0 ? tx : (d == 1 ? ty : tz)) * a.tile[d];
    const int tn = min(a.tile[d], a.out_size[d] - o0);
    float w[NT];
    int lo0, lo1;
    bool inb;
    axis_stencil<NT>(a, d, o0, lo0, w, inb);
    axis_stencil<NT>(a, d, o0 + tn - 1, lo1, w, inb);
    const int b = d == 2 ? (lo0 & ~3) : lo0;
    const int hi = lo1 + NT - 1;
    it.o0[d] = o0;
    it.tn[d] = tn;
    it.base[d] = b;
    fits = hi - b < a.ext[d];
    interior = b >= 0 && hi < a.in_size[d];
  }
  const bool all_fit = __all_sync(0xffffffffu, fits), all_in = __all_sync(0xffffffffu, interior);
  if (lane == 0) {
    it.c = item - t * a.C;
    it.n = r / a.ntile[0];
    it.fits = all_fit;
    it.interior = all_fit && all_in;
  }
  __syncwarp();
}

// Persistent CTAs walk the (tile, channel) items, a tile's channels in a row,
// with two staging buffers: the TMA copy of the next item is in flight while
// the current one is filtered.
template <int NT, class S, bool TMA>
__global__ void __launch_bounds__(RZ_THREADS, 3) resize_sep_kernel(const __grid_constant__ ResizeArgs a,
                                                                 const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(128) float rz_smem[];
  __shared__ __align__(8) unsigned long long mbar[2];
  __shared__ unsigned uses[2];  // copies issued into each staging buffer
  __shared__ int lo_t[3][RZ_MAXT];
  __shared__ float4 w_t[3][RZ_MAXT];  // NT <= 4 weights per output index
  __shared__ unsigned char inb_t[3][RZ_MAXT];
  __shared__ int gidx_t[3][RZ_MAXE];           // boundary items: node each staged position maps to
  __shared__ signed char sgn_t[3][RZ_MAXE];    // ... and its sign
  __shared__ RzItem cur, nxt;
  __shared__ bool tma_ok;

  const int TX = a.tile[0], TY = a.tile[1];
  const int EX = a.ext[0], EY = a.ext[1], EZ = a.ext[2];
  const int EZ4 = EZ / 4;
  const int SZ = EX * EY * EZ;
  // TMA writes shared memory at 128-byte boundaries: the staging buffers
  // start at a 128-byte aligned base, one pitch (a multiple of 32 floats) apart
  const int SP = (SZ + 31) & ~31;
  float* smem = rz_smem + ((128u - (smem_addr(rz_smem) & 127u)) & 127u) / 4u;
  float* T1 = smem + 2 * SP;  // [TX][EY][EZ]
  float* T2 = T1 + TX * EY * EZ;  // [TX][TY][EZ]
  // CTA j walks the tiles j, j + G, ... and each tile's channels in turn:
  // its k-th item is channel k mod C of tile j + (k / C) G (items are
  // numbered tile * C + channel); a tile's tables serve all its channels
  const int ntiles = a.ntile[0] * a.ntile[1] * a.ntile[2] * a.N;
  auto item_of = [&](int k) { return (static_cast<int>(blockIdx.x) + (k / a.C) * static_cast<int>(gridDim.x)) * a.C + k % a.C; };
  const int lz = threadIdx.x & 31, lr = threadIdx.x >> 5;
  const bool oob_zero = !(a.extrapolate & 1);

  auto issue = [&](int buf, const RzItem& it) {  // one thread: TMA copy of an item's region
    const unsigned bar = smem_addr(&mbar[buf]);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                 "r"(static_cast<unsigned>(SZ * 4))
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
            smem_addr(smem + buf * SP)),
        "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(it.base[2]), "r"(it.base[1]), "r"(it.base[0]),
        "r"(it.n * a.C + it.c), "r"(bar)
        : "memory");
    ++uses[buf];
  };

  int item = item_of(0);
  if (threadIdx.x < 32) {
    if (threadIdx.x == 0) {
      if (TMA) {
        for (int b = 0; b < 2; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&mbar[b])), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      }
      uses[0] = uses[1] = 0;
    }
    if (item / a.C < ntiles) {
      rz_item<NT>(a, item, cur);
      if (TMA && threadIdx.x == 0 && cur.fits) issue(0, cur);
    }
  }
  __syncthreads();

  for (int k = 0; item / a.C < ntiles; ++k, item = item_of(k)) {
    const int buf = k & 1;
    float* Sst = smem + buf * SP;
    // per-axis tables of this item's tile (its first channel)
    for (int e = threadIdx.x; cur.c == 0 && e < a.tile[0] + a.tile[1] + a.tile[2]; e += RZ_THREADS) {
      const int d = e < a.tile[0] ? 0 : (e < a.tile[0] + a.tile[1] ? 1 : 2);
      const int i = e - (d == 0 ? 0 : (d == 1 ? a.tile[0] : a.tile[0] + a.tile[1]));
      float w[NT];
      int lo;
      bool inb;
      axis_stencil<NT>(a, d, cur.o0[d] + min(i, cur.tn[d] - 1), lo, w, inb);
      lo_t[d][i] = lo - cur.base[d];  // relative to the staged region
      float4 w4 = make_float4(0.f, 0.f, 0.f, 0.f);
      w4.x = w[0];
      if (NT > 1) w4.y = w[NT > 1 ? 1 : 0];
      if (NT > 2) w4.z = w[NT > 2 ? 2 : 0];
      if (NT > 3) w4.w = w[NT > 3 ? 3 : 0];
      w_t[d][i] = w4;
      inb_t[d][i] = inb;
    }
    if (cur.c == 0 && cur.fits && !cur.interior) {
      // per axis, where the boundary condition maps each staged position
      for (int e = threadIdx.x; e < EX + EY + EZ; e += RZ_THREADS) {
        const int d = e < EX ? 0 : (e < EX + EY ? 1 : 2);
        const int i = e - (d == 0 ? 0 : (d == 1 ? EX : EX + EY));
        const int P = cur.base[d] + i;
        gidx_t[d][i] = bound_index<int>(a.bound[d], P, a.in_size[d]);
        sgn_t[d][i] = static_cast<signed char>(bound_sign<int>(a.bound[d], P, a.in_size[d]));
      }
    }
    // the next item: its copy goes into the other buffer (its last reader,
    // item k - 1, has finished)
    const int ni = item_of(k + 1);
    const bool has_next = ni / a.C < ntiles;
    if (threadIdx.x < 32 && has_next) {
      if (ni % a.C != 0) {
        // the next channel of the same tile: the same staged region
        if (threadIdx.x == 0) {
          nxt = cur;
          nxt.c = cur.c + 1;
        }
        __syncwarp();
      } else {
        rz_item<NT>(a, ni, nxt);
      }
      if (TMA && threadIdx.x == 0 && nxt.fits) issue(buf ^ 1, nxt);
    }
    const S* sc = static_cast<const S*>(a.src) + static_cast<int64_t>(cur.n) * a.src_sN + cur.c * a.src_sC;
    const int bx = cur.base[0], by = cur.base[1], bz = cur.base[2];
    auto bounded = [&](int X, int Y, int Z) -> float {  // staged value under the boundary condition
      const int sgn = bound_sign<int>(a.bound[0], X, a.in_size[0]) * bound_sign<int>(a.bound[1], Y, a.in_size[1]) *
                      bound_sign<int>(a.bound[2], Z, a.in_size[2]);
      if (sgn == 0) return 0.f;
      const int64_t off = bound_index<int>(a.bound[0], X, a.in_size[0]) * a.src_s[0] +
                          bound_index<int>(a.bound[1], Y, a.in_size[1]) * a.src_s[1] +
                          bound_index<int>(a.bound[2], Z, a.in_size[2]) * a.src_s[2];
      return static_cast<float>(sgn) * static_cast<float>(ldg_acc(sc + off));
    };
    S* out_c = static_cast<S*>(a.out) + static_cast<int64_t>(cur.n) * a.out_sN + cur.c * a.out_sC;

    if (!cur.fits) {
      // the nodes of this tile span more than the staged region (float
      // rounding of the coordinates): its voxels straight from global memory
      __syncthreads();
      for (int e = threadIdx.x; e < a.tile[0] * a.tile[1] * a.tile[2]; e += RZ_THREADS) {
        const int oz = e % a.tile[2], r = e / a.tile[2], oy = r % TY, ox = r / TY;
        if (ox >= cur.tn[0] || oy >= cur.tn[1] || oz >= cur.tn[2]) continue;
        float acc = 0.f;
        if (!oob_zero || (inb_t[0][ox] && inb_t[1][oy] && inb_t[2][oz])) {
          const float* wx = &w_t[0][ox].x;
          const float* wy = &w_t[1][oy].x;
          const float* wz = &w_t[2][oz].x;
          for (int kk = 0; kk < NT; ++kk) {
            float accy = 0.f;
            for (int j = 0; j < NT; ++j) {
              float accx = 0.f;
              for (int i = 0; i < NT; ++i)
                accx = fmaf(wx[i], bounded(bx + lo_t[0][ox] + i, by + lo_t[1][oy] + j, bz + lo_t[2][oz] + kk), accx);
              accy = fmaf(wy[j], accx, accy);
            }
            acc = fmaf(wz[kk], accy, acc);
          }
        }
        out_c[(cur.o0[0] + ox) * a.out_s[0] + (cur.o0[1] + oy) * a.out_s[1] + (cur.o0[2] + oz) * a.out_s[2]] =
            from_acc<S>(acc);
      }
    } else {
      // staged region of this item
      if (TMA) {
        // one thread waits for the copy (the others sleep in the barrier),
        // then every thread observes the completed phase once
        const unsigned ph = (uses[buf] - 1) & 1u;
        if (threadIdx.x == 0) tma_ok = mbar_wait(smem_addr(&mbar[buf]), ph);
        __syncthreads();
        if (!tma_ok) {
          if (threadIdx.x == 0) {
            atomicOr(&g_resize_status, 1u);
            mbar_wait(smem_addr(&mbar[buf]), ph);  // the copy may still land: wait once more
            if (TMA && has_next && nxt.fits)
              mbar_wait(smem_addr(&mbar[buf ^ 1]), (uses[buf ^ 1] - 1) & 1u);
          }
          return;
        }
        mbar_wait(smem_addr(&mbar[buf]), ph);
      } else {
        // stage the voxels inside the volume
        __syncthreads();
        for (int r = lr; r < EX * EY; r += RZ_THREADS / 32) {
          const int x = r / EY, y = r - x * EY;
          const int X = bx + x, Y = by + y;
          if (X < 0 || X >= a.in_size[0] || Y < 0 || Y >= a.in_size[1]) continue;
          const S* rowp = sc + X * a.src_s[0] + Y * a.src_s[1];
          for (int z = lz; z < EZ; z += 32) {
            const int Z = bz + z;
            if (Z >= 0 && Z < a.in_size[2]) Sst[r * EZ + z] = static_cast<float>(ldg_acc(rowp + Z * a.src_s[2]));
          }
        }
        __syncthreads();
      }
      if (!cur.interior) {
        // the staged voxels outside the volume: the boundary condition maps
        // each to a voxel inside it (times a sign), read from the staged
        // region when it holds that voxel, else from global memory.  All
        // threads share three segments: x planes outside the volume, then
        // rows outside it in y, then the out-of-volume z of inside rows.
        int lo3[3], hi3[3];  // staged positions inside the volume: [lo, hi)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          lo3[d] = min(max(-cur.base[d], 0), a.ext[d]);
          hi3[d] = max(min(a.in_size[d] - cur.base[d], a.ext[d]), lo3[d]);
        }
        const int nxi = hi3[0] - lo3[0], nyi = hi3[1] - lo3[1], nzi = hi3[2] - lo3[2];
        const int nyo = EY - nyi, nzo = EZ - nzi;
        const int segA = (EX - nxi) * EY * EZ, segB = nxi * nyo * EZ, segC = nxi * nyi * nzo;
        for (int e = threadIdx.x; e < segA + segB + segC; e += RZ_THREADS) {
          int x, y, z;
          if (e < segA) {
            const int q = e / EZ;
            z = e - q * EZ;
            const int xo = q / EY;
            y = q - xo * EY;
            x = xo < lo3[0] ? xo : hi3[0] + (xo - lo3[0]);
          } else if (e < segA + segB) {
            const int f = e - segA, q = f / EZ;
            z = f - q * EZ;
            const int xi = q / nyo, yo = q - xi * nyo;
            x = lo3[0] + xi;
            y = yo < lo3[1] ? yo : hi3[1] + (yo - lo3[1]);
          } else {
            const int f = e - segA - segB, q = f / nzo, zo = f - q * nzo;
            const int xi = q / nyi;
            x = lo3[0] + xi;
            y = lo3[1] + (q - xi * nyi);
            z = zo < lo3[2] ? zo : hi3[2] + (zo - lo3[2]);
          }
          const int sgn = sgn_t[0][x] * sgn_t[1][y] * sgn_t[2][z];
          float v = 0.f;
          if (sgn != 0) {
            const int gx = gidx_t[0][x], gy = gidx_t[1][y], gz = gidx_t[2][z];
            const int mx = gx - bx, my = gy - by, mz = gz - bz;
            const float u = (mx >= 0 && mx < EX && my >= 0 && my < EY && mz >= 0 && mz < EZ)
                                ? Sst[(mx * EY + my) * EZ + mz]
                                : static_cast<float>(ldg_acc(sc + gx * a.src_s[0] + gy * a.src_s[1] + gz * a.src_s[2]));
            v = static_cast<float>(sgn) * u;
          }
          Sst[(x * EY + y) * EZ + z] = v;
        }
      }
      __syncthreads();
      // x pass over every staged (y, z), four z at a time: rows (ox, y),
      // 2^zls lanes per row
      const int ZL = 1 << a.zls, RW = 32 >> a.zls;
      const int zl = lz & (ZL - 1), rs = lz >> a.zls;
      {
        const float4* S4 = reinterpret_cast<const float4*>(Sst);
        float4* T14 = reinterpret_cast<float4*>(T1);
        for (int r = lr * RW + rs; r < TX * EY; r += (RZ_THREADS / 32) * RW) {
          const int ox = r / EY, y = r - ox * EY;
          const float4 w = w_t[0][ox];
          const float wi[4] = {w.x, w.y, w.z, w.w};
          const float4* sp = S4 + (lo_t[0][ox] * EY + y) * EZ4;
          for (int z = zl; z < EZ4; z += ZL) {
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int i = 0; i < NT; ++i) {
              const float4 v = sp[i * EY * EZ4 + z];
              acc.x = fmaf(wi[i], v.x, acc.x);
              acc.y = fmaf(wi[i], v.y, acc.y);
              acc.z = fmaf(wi[i], v.z, acc.z);
              acc.w = fmaf(wi[i], v.w, acc.w);
            }
            T14[r * EZ4 + z] = acc;
          }
        }
      }
      __syncthreads();
      // y pass, four z at a time: rows (ox, oy)
      {
        const float4* T14 = reinterpret_cast<const float4*>(T1);
        float4* T24 = reinterpret_cast<float4*>(T2);
        for (int r = lr * RW + rs; r < TX * TY; r += (RZ_THREADS / 32) * RW) {
          const int ox = r / TY, oy = r - ox * TY;
          const float4 w = w_t[1][oy];
          const float wj[4] = {w.x, w.y, w.z, w.w};
          const float4* tp = T14 + (ox * EY + lo_t[1][oy]) * EZ4;
          for (int z = zl; z < EZ4; z += ZL) {
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int j = 0; j < NT; ++j) {
              const float4 v = tp[j * EZ4 + z];
              acc.x = fmaf(wj[j], v.x, acc.x);
              acc.y = fmaf(wj[j], v.y, acc.y);
              acc.z = fmaf(wj[j], v.z, acc.z);
              acc.w = fmaf(wj[j], v.w, acc.w);
            }
            T24[r * EZ4 + z] = acc;
          }
        }
      }
      __syncthreads();
      // z pass and store: lanes along oz (the stencil of each lane's oz
      // read once), warps over rows (ox, oy)
      for (int oz = lz; oz < cur.tn[2]; oz += 32) {
        const float4 w = w_t[2][oz];
        const float wk[4] = {w.x, w.y, w.z, w.w};
        const int lzo = lo_t[2][oz];
        const bool inz = inb_t[2][oz];
        S* oc = out_c + (cur.o0[2] + oz) * a.out_s[2];
#pragma unroll 4
        for (int r = lr; r < TX * TY; r += RZ_THREADS / 32) {
          const int ox = r / TY, oy = r - ox * TY;
          if (ox >= cur.tn[0] || oy >= cur.tn[1]) continue;
          float acc = 0.f;
          if (!oob_zero || (inz && inb_t[0][ox] && inb_t[1][oy])) {
            const float* tz = T2 + r * EZ + lzo;
#pragma unroll
            for (int kk = 0; kk < NT; ++kk) acc = fmaf(wk[kk], tz[kk], acc);
          }
          oc[(cur.o0[0] + ox) * a.out_s[0] + (cur.o0[1] + oy) * a.out_s[1]] = from_acc<S>(acc);
        }
      }
    }
    // order this item's generic-proxy writes to the staging buffer (the
    // boundary fix-up) before the next TMA copy into it
    if (TMA && cur.fits && !cur.interior) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) cur = nxt;
    __syncthreads();
  }
}

// --- host side --------------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Working set of a tile: two staging buffers (each padded to 128 bytes, plus
// 128 bytes to align the first), the x-pass and y-pass results.
size_t smem_floats(const int (&t)[3], const int (&e)[3]) {
  const size_t sz = (static_cast<size_t>(e[0]) * e[1] * e[2] + 31) & ~static_cast<size_t>(31);
  return 32 + 2 * sz + static_cast<size_t>(t[0]) * e[1] * e[2] + static_cast<size_t>(t[0]) * t[1] * e[2];
}

// Staged extent of a tile edge of T outputs at step `scale` for NT taps:
// the nodes of T consecutive outputs span at most ceil((T - 1) scale) + NT
// positions; one more covers the rounding of the lowest node.
int extent(int T, double scale, int NT) {
  return static_cast<int>(std::ceil((T - 1) * scale)) + NT + 1;
}

// Largest tile whose working set fits `budget` floats of shared memory.
bool choose_tile(const double (&scale)[3], int NT, int (&t)[3], int (&e)[3], size_t budget) {
  static const int cand[][3] = {{4, 8, 64}, {2, 8, 64}, {4, 8, 32}, {2, 8, 32}, {2, 4, 32}, {1, 4, 32},
                                {2, 4, 16}, {1, 4, 16}, {1, 2, 16}, {1, 1, 16}, {1, 1, 8}};
  for (const auto& c : cand) {
    int ee[3];
    for (int d = 0; d < 3; ++d) ee[d] = extent(c[d], scale[d], NT);
    ee[2] = ((ee[2] + 3 + 3) / 4) * 4;  // room for the 16-byte alignment of the z start; TMA box multiple of 4
    if (ee[2] > 256 || ee[1] > 256 || ee[0] > 256) continue;
    const int tt[3] = {c[0], c[1], c[2]};
    if (smem_floats(tt, ee) <= budget) {
      for (int d = 0; d < 3; ++d) { t[d] = c[d]; e[d] = ee[d]; }
      return true;
    }
  }
  return false;
}

// Largest working set of a tile (floats of dynamic shared memory): three
// CTAs per SM.
constexpr size_t RZ_SMEM_FLOATS = 16 * 1024;

template <int NT, class S, bool TMA>
cudaError_t launch_resize(const ResizeArgs& a, const CUtensorMap& map, size_t smem, int64_t ntiles, cudaStream_t st) {
  // opt in, once per device, to the largest working set any call may use
  static std::atomic<unsigned long long> done{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(done.load() & bit)) {
    e = cudaFuncSetAttribute(resize_sep_kernel<NT, S, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(RZ_SMEM_FLOATS * 4));
    if (e != cudaSuccess) return e;
    done.fetch_or(bit);
  }
  if (smem > RZ_SMEM_FLOATS * 4) return cudaErrorInvalidValue;
  // persistent CTAs: as many as fit on the GPU at once
  int sms = 0, per_sm = 0;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, resize_sep_kernel<NT, S, TMA>, RZ_THREADS, smem)) !=
      cudaSuccess)
    return e;
  const int64_t grid = std::min<int64_t>(ntiles, static_cast<int64_t>(std::max(1, sms * per_sm)));
  ppk::note_kernel(TMA ? "resize_sep_kernel tma" : "resize_sep_kernel", a.kind, NT - 1, 1);
  resize_sep_kernel<NT, S, TMA><<<static_cast<unsigned>(grid), RZ_THREADS, smem, st>>>(a, map);
  return cudaGetLastError();
}

template <class S>
cudaError_t dispatch(int order, bool tma, const ResizeArgs& a, const CUtensorMap& map, size_t smem, int64_t nt,
                     cudaStream_t st) {
  switch (order) {
#define RZ_CASE(O)                                                                   \
  case O:                                                                            \
    return tma ? launch_resize<O + 1, S, true>(a, map, smem, nt, st)                 \
               : launch_resize<O + 1, S, false>(a, map, smem, nt, st);
    RZ_CASE(0) RZ_CASE(1) RZ_CASE(2) RZ_CASE(3)
#undef RZ_CASE
  }
  return cudaErrorInvalidValue;
}

int resize_launch(const pp_tensor* input, const pp_tensor* out, const double* scale, const double* shift,
                  const int (&bound)[3], int order, int extrapolate, int kind, void* stream) {
  using namespace ppc;
  int rc;
  if ((rc = check_tensor(input, "input")) || (rc = check_tensor(out, "output"))) return rc;
  if (input->ndim != 5 || out->ndim != 5)
    return fail(PP_ERR_UNSUPPORTED, "(): pp_resize takes 3-D images (N, C, X, Y, Z)");
  if (input->sizes[0] != out->sizes[0] || input->sizes[1] != out->sizes[1])
    return fail(PP_ERR_ARG, "(): expected input (N, C, *inshape) and output (N, C, *shape)");
  if (input->dtype != out->dtype) return fail(PP_ERR_DTYPE, "(): output dtype must match input");
  if (input->dtype != PP_FLOAT32 && input->dtype != PP_BFLOAT16)
    return fail(PP_ERR_UNSUPPORTED, "(): pp_resize takes float32 or bfloat16 images");
  for (int d = 0; d < 3; ++d) {
    if (!(scale[d] > 0.0) || !std::isfinite(scale[d]) || !std::isfinite(shift[d]))
      return fail(PP_ERR_UNSUPPORTED, "(): pp_resize takes positive finite scales and finite shifts");
    if (input->sizes[2 + d] <= 0 || out->sizes[2 + d] <= 0) return fail(PP_ERR_ARG, "(): expected non-empty sizes");
    if (input->sizes[2 + d] >= (1 << 24) || out->sizes[2 + d] >= (1 << 24))
      return fail(PP_ERR_UNSUPPORTED, "(): pp_resize takes axes shorter than 2^24 voxels");
  }
  if (max_offset(input, 0) >= (int64_t(1) << 31) || max_offset(out, 0) >= (int64_t(1) << 31) ||
      input->sizes[0] * input->sizes[1] >= (int64_t(1) << 31))
    return fail(PP_ERR_UNSUPPORTED, "(): pp_resize needs 32-bit element offsets");
  const int NT = kind == 1 ? 4 : (order == 0 ? 1 : order + 1);
  int tile[3], ext[3];
  const double sc3[3] = {scale[0], scale[1], scale[2]};
  if (!choose_tile(sc3, NT, tile, ext, RZ_SMEM_FLOATS))
    return fail(PP_ERR_UNSUPPORTED, "(): pp_resize: scales too large for a shared-memory tile");
  if (numel(out) == 0) return PP_OK;

  ResizeArgs a;
  std::memset(&a, 0, sizeof(a));
  a.src = input->data;
  a.out = out->data;
  a.N = static_cast<int>(input->sizes[0]);
  a.C = static_cast<int>(input->sizes[1]);
  a.src_sN = input->strides[0];
  a.src_sC = input->strides[1];
  a.out_sN = out->strides[0];
  a.out_sC = out->strides[1];
  int64_t ntiles = a.N;
  for (int d = 0; d < 3; ++d) {
    a.in_size[d] = static_cast<int>(input->sizes[2 + d]);
    a.out_size[d] = static_cast<int>(out->sizes[2 + d]);
    a.src_s[d] = input->strides[2 + d];
    a.out_s[d] = out->strides[2 + d];
    a.scale[d] = static_cast<float>(scale[d]);
    a.shift[d] = static_cast<float>(shift[d]);
    a.bound[d] = bound[d];
    a.tile[d] = tile[d];
    a.ext[d] = ext[d];
    a.ntile[d] = (a.out_size[d] + tile[d] - 1) / tile[d];
    ntiles *= a.ntile[d];
  }
  while ((1 << a.zls) < ext[2] / 4 && a.zls < 5) ++a.zls;
  a.order = order;
  a.extrapolate = extrapolate;
  a.kind = kind;
  if (ntiles * a.C >= (int64_t(1) << 31)) return fail(PP_ERR_UNSUPPORTED, "(): pp_resize: too many tiles");

  // TMA copies need a float32 image with the z axis contiguous, 16-byte
  // aligned rows and the batch and channel axes foldable into one.
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  bool tma = input->dtype == PP_FLOAT32 && input->strides[4] == 1 && input->strides[3] % 4 == 0 &&
             input->strides[2] % 4 == 0 && input->strides[1] % 4 == 0 &&
             input->strides[0] == input->sizes[1] * input->strides[1] &&
             reinterpret_cast<uintptr_t>(input->data) % 16 == 0;
  if (tma) {
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(input->sizes[4]), static_cast<cuuint64_t>(input->sizes[3]),
                                static_cast<cuuint64_t>(input->sizes[2]),
                                static_cast<cuuint64_t>(input->sizes[0] * input->sizes[1])};
    const cuuint64_t strides[3] = {static_cast<cuuint64_t>(input->strides[3]) * 4,
                                   static_cast<cuuint64_t>(input->strides[2]) * 4,
                                   static_cast<cuuint64_t>(input->strides[1]) * 4};
    const cuuint32_t box[4] = {static_cast<cuuint32_t>(ext[2]), static_cast<cuuint32_t>(ext[1]),
                               static_cast<cuuint32_t>(ext[0]), 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    tma = encode && encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, input->data, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  }
  a.use_tma = tma;
  const size_t smem = smem_floats(tile, ext) * 4;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int tap_order = NT - 1;  // the instance: NT taps
  // persistent CTAs: at most one per tile (each walks its tiles' channels)
  cudaError_t e = input->dtype == PP_FLOAT32 ? dispatch<float>(tap_order, tma, a, map, smem, ntiles, st)
                                             : dispatch<__nv_bfloat16>(tap_order, false, a, map, smem, ntiles, st);
  count_launch();
  return cuda_check(e, "resize launch");
}

}  // namespace

extern "C" {

int pp_resize(const pp_tensor* input, const pp_tensor* out, const double* scale, const double* shift,
              const pp_options* opt, void* stream) {
  using namespace ppc;
  if (!scale || !shift) return fail(PP_ERR_ARG, "(): expected scale and shift");
  int bound[3], order[3], rc;
  if ((rc = read_options(opt, 3, bound, order))) return rc;
  if (order[1] != order[0] || order[2] != order[0] || order[0] > 3)
    return fail(PP_ERR_UNSUPPORTED, "(): pp_resize takes one B-spline order of at most 3 for all axes");
  return resize_launch(input, out, scale, shift, bound, order[0], opt->extrapolate, 0, stream);
}

// Multigrid prolongation / restriction between the grids of `input` and
// `out`: scale = input size / output size per axis.
static int multires(const pp_tensor* input, const pp_tensor* out, const pp_options* opt, int kind, void* stream) {
  using namespace ppc;
  int rc;
  if ((rc = check_tensor(input, "input")) || (rc = check_tensor(out, "output"))) return rc;
  if (input->ndim != 5 || out->ndim != 5)
    return fail(PP_ERR_UNSUPPORTED, "(): expected 3-D images (N, C, X, Y, Z)");
  int bound[3], order[3];
  if ((rc = read_options(opt, 3, bound, order))) return rc;
  double scale[3], shift[3] = {0., 0., 0.};
  for (int d = 0; d < 3; ++d) {
    if (input->sizes[2 + d] <= 0 || out->sizes[2 + d] <= 0) return fail(PP_ERR_ARG, "(): expected non-empty sizes");
    scale[d] = static_cast<double>(input->sizes[2 + d]) / static_cast<double>(out->sizes[2 + d]);
  }
  return resize_launch(input, out, scale, shift, bound, kind == 1 ? 1 : 2, 1, kind, stream);
}

int pp_fmg_prolongation(const pp_tensor* input, const pp_tensor* out, const pp_options* opt, void* stream) {
  return multires(input, out, opt, 2, stream);
}

int pp_fmg_restriction(const pp_tensor* input, const pp_tensor* out, const pp_options* opt, void* stream) {
  return multires(input, out, opt, 1, stream);
}

int pp_resize_status(uint32_t* status) {
  if (!status) return ppc::fail(PP_ERR_ARG, "(): expected a status pointer");
  unsigned int s = 0;
  const cudaError_t e = cudaMemcpyFromSymbol(&s, g_resize_status, sizeof(s));
  if (e != cudaSuccess) return ppc::cuda_check(e, "resize status");
  *status = s;
  return PP_OK;
}

}  // extern "C"
