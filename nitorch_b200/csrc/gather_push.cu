// Gather-form push (3-D, orders 1 and 3).
//
// push scatters every sampling point's value t_p into the (ORD+1)^3 voxels
// of its stencil: out[v] += w(v - x_p) t_p (nitorch/_C/src/impl/
// pushpull_common.cpp, push3d).  As a scatter that is one float atomic per
// tap and channel -- on B200 the reduction path, not HBM, bounds it.  Here
// the same sum runs per output voxel instead:
//
//   out[v] = sum over the points p whose stencil covers v of w(v - x_p) t_p
//
// over the points sorted by source cell (the counting sort of order.cu; its
// per-cell offsets `cells` list the points whose floor(x) is each cell).  A
// point reaches voxel v iff its cell is in [v - LO, v + HI] along every axis
// (LO = (ORD+1)/2, HI = (ORD-1)/2), so voxel v reads the (ORD+1)^3 cells
// around it.  Only interior points -- every tap inside the volume, so no
// boundary condition applies (interior_axis) -- are gathered; the others
// (near the faces, outside the field of view, or clamped into an edge cell
// by the sort) get zero weight here and go through the atomic scatter with
// flag F_RESID afterwards.  No atomics, and every output voxel is written
// once, so the output needs no clearing.
//
// CTA = a GX x GY x GZ block of output voxels of one batch item, one thread
// each.  The block's cells form CX x CY rows of CZ cells (the block dilated
// by the stencil); in sorted order each row's points are contiguous.  The
// CTA lists the rows' point ranges (prefix sum of their counts), then stages
// up to G_CAP points at a time in shared memory: per-axis weights of every
// tap (from the same build_axis as the scatter kernels) and up to G_CB
// channel values.  Each thread then walks its (ORD+1)^3 cells and
// accumulates.  Denser regions than G_CAP points per block take several
// passes; more than G_CB channels take several channel passes.
#include "pp_capi_internal.cuh"
#include "pp_kernels.cuh"

namespace ppk {
namespace {

constexpr int GX = 4, GY = 8, GZ = 8;    // output voxels per CTA (z fastest)
constexpr int G_THREADS = GX * GY * GZ;  // one voxel per thread
constexpr int G_CAP = 1024;              // points staged per pass
constexpr int G_CB = 4;                  // channels per pass

template <int ORD>
constexpr size_t gather_smem_bytes() {
  return static_cast<size_t>(3 * (ORD + 1) + G_CB) * G_CAP * sizeof(float);
}

template <int ORD, class S>
__global__ void __launch_bounds__(G_THREADS) gather_push_kernel(const PPArgs a, const int32_t* __restrict__ cells,
                                                                int nbx, int nby, int nbz) {
  constexpr int NTAP = ORD + 1;
  constexpr int LO = (ORD + 1) / 2, HI = (ORD - 1) / 2;
  constexpr int CX = GX + ORD, CY = GY + ORD, CZ = GZ + ORD;  // cells of the dilated block
  constexpr int NROW = CX * CY;
  static_assert(NROW <= G_THREADS, "one thread per row");
  extern __shared__ __align__(16) float gsm[];
  float* wsm = gsm;                     // [3][NTAP][G_CAP]: weight of tap t along each axis
  float* vsm = gsm + 3 * NTAP * G_CAP;  // [G_CB][G_CAP]: channel values
  __shared__ int row_first[NROW];       // sorted position of the row's first staged point
  __shared__ int row_base[NROW + 1];    // the row's first point in the block's list
  __shared__ int cell_off[NROW * (CZ + 1)];

  int b = static_cast<int>(blockIdx.x);
  const int bz = b % nbz; b /= nbz;
  const int by = b % nby; b /= nby;
  const int bx = b % nbx;
  const int n = b / nbx;
  const int x0 = bx * GX, y0 = by * GY, z0 = bz * GZ;
  const int sx = static_cast<int>(a.src_size[0]), sy = static_cast<int>(a.src_size[1]),
            sz = static_cast<int>(a.src_size[2]);
  const int32_t* cn = cells + static_cast<int64_t>(n) * sx * sy * sz;
  const int tid = threadIdx.x;
  const int za = max(z0 - LO, 0), zb = min(z0 + GZ + HI, sz);  // cells [za, zb) of every row

  // 1. point ranges of the rows, their prefix sum, the cell boundaries
  if (tid < NROW) {
    const int cx = x0 - LO + tid / CY, cy = y0 - LO + tid % CY;
    int g0 = 0, cnt = 0;
    if (cx >= 0 && cx < sx && cy >= 0 && cy < sy) {
      const int64_t rk = (static_cast<int64_t>(cx) * sy + cy) * sz;
      g0 = cn[rk + za];
      cnt = cn[rk + zb] - g0;
    }
    row_first[tid] = g0;
    row_base[tid] = cnt;
  }
  __syncthreads();
  if (tid < 32) {
    int run = 0;
    for (int r0 = 0; r0 < NROW; r0 += 32) {
      const int r = r0 + tid;
      const int c = r < NROW ? row_base[r] : 0;
      int inc = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (tid >= o) inc += y;
      }
      if (r < NROW) row_base[r] = run + inc - c;
      run += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (tid == 0) row_base[NROW] = run;
  }
  __syncthreads();
  for (int e = tid; e < NROW * (CZ + 1); e += G_THREADS) {
    const int r = e / (CZ + 1), zi = e % (CZ + 1);
    const int cx = x0 - LO + r / CY, cy = y0 - LO + r % CY;
    int pos = row_base[r];
    if (cx >= 0 && cx < sx && cy >= 0 && cy < sy) {
      const int cz = min(max(z0 - LO + zi, za), zb);
      pos += cn[(static_cast<int64_t>(cx) * sy + cy) * sz + cz] - row_first[r];
    }
    cell_off[e] = pos;
  }
  __syncthreads();
  const int total = row_base[NROW];

  const int lx = tid / (GY * GZ), ly = (tid / GZ) % GY, lz = tid % GZ;
  const int vx = x0 + lx, vy = y0 + ly, vz = z0 + lz;
  const bool live = vx < sx && vy < sy && vz < sz;
  const int t0 = static_cast<int>(a.trgt_size[0]), t1 = static_cast<int>(a.trgt_size[1]),
            t2 = static_cast<int>(a.trgt_size[2]);
  const float* gbase = static_cast<const float*>(a.grid) + static_cast<int64_t>(n) * a.grid_sN;
  const S* tbase = static_cast<const S*>(a.trgt) + static_cast<int64_t>(n) * a.trgt_sN;
  float* obase = static_cast<float*>(a.out) + static_cast<int64_t>(n) * a.out_sN +
                 static_cast<int64_t>(vx) * a.out_s[0] + static_cast<int64_t>(vy) * a.out_s[1] +
                 static_cast<int64_t>(vz) * a.out_s[2];

  for (int c0 = 0; c0 < a.C; c0 += G_CB) {
    const int nc = a.C - c0 < G_CB ? static_cast<int>(a.C - c0) : G_CB;
    float acc[G_CB];
#pragma unroll
    for (int c = 0; c < G_CB; ++c) acc[c] = 0.f;
    for (int P0 = 0; P0 < total; P0 += G_CAP) {
      const int np = total - P0 < G_CAP ? total - P0 : G_CAP;
      // 2. stage points [P0, P0 + np): weights and values
      for (int j = tid; j < np; j += G_THREADS) {
        const int p = P0 + j;
        int lo = 0, hi = NROW - 1;  // row of p: the last r with row_base[r] <= p
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (row_base[mid] <= p) lo = mid; else hi = mid - 1;
        }
        int s = a.perm[row_first[lo] + (p - row_base[lo])];  // flat sample (item n)
        const int gz = s % t2; s /= t2;
        const int gy = s % t1; s /= t1;
        const int gx = s % t0;
        const float* gp = gbase + static_cast<int64_t>(gx) * a.grid_s[0] + static_cast<int64_t>(gy) * a.grid_s[1] +
                          static_cast<int64_t>(gz) * a.grid_s[2];
        float x[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d] = __ldg(gp + d * a.grid_sD);
        const bool inner = interior_axis<int, float>(ORD, x[0], sx) && interior_axis<int, float>(ORD, x[1], sy) &&
                           interior_axis<int, float>(ORD, x[2], sz);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          Axis<NTAP, float, int> ax;
          build_axis<NTAP, false, false, false, false, float, int>(ax, ORD, a.bound[d], x[d],
                                                                   static_cast<int>(a.src_size[d]), 0, 0);
#pragma unroll
          for (int t = 0; t < NTAP; ++t) wsm[(d * NTAP + t) * G_CAP + j] = inner ? ax.w[t] : 0.f;
        }
        const S* tp = tbase + static_cast<int64_t>(gx) * a.trgt_s[0] + static_cast<int64_t>(gy) * a.trgt_s[1] +
                      static_cast<int64_t>(gz) * a.trgt_s[2] + static_cast<int64_t>(c0) * a.trgt_sC;
#pragma unroll
        for (int c = 0; c < G_CB; ++c) vsm[c * G_CAP + j] = c < nc ? ldg_acc(tp + c * a.trgt_sC) : 0.f;
      }
      __syncthreads();
      // 3. every voxel sums the staged points of its (ORD+1)^3 cells
      if (live) {
        const int pend = P0 + np;
#pragma unroll
        for (int kx = 0; kx < NTAP; ++kx) {
          const float* wx = wsm + (0 * NTAP + (ORD - kx)) * G_CAP - P0;
#pragma unroll
          for (int ky = 0; ky < NTAP; ++ky) {
            const float* wy = wsm + (1 * NTAP + (ORD - ky)) * G_CAP - P0;
            const int* co = cell_off + ((lx + kx) * CY + (ly + ky)) * (CZ + 1) + lz;
#pragma unroll
            for (int kz = 0; kz < NTAP; ++kz) {
              const float* wz = wsm + (2 * NTAP + (ORD - kz)) * G_CAP - P0;
              const int pa = max(co[kz], P0), pb = min(co[kz + 1], pend);
              for (int p = pa; p < pb; ++p) {
                const float w = wx[p] * wy[p] * wz[p];
#pragma unroll
                for (int c = 0; c < G_CB; ++c) acc[c] = fmaf(w, vsm[c * G_CAP + p - P0], acc[c]);
              }
            }
          }
        }
      }
      __syncthreads();
    }
    if (live)
      for (int c = 0; c < nc; ++c) obase[static_cast<int64_t>(c0 + c) * a.out_sC] = acc[c];
  }
}

template <int ORD, class S>
int launch_gather(const PPArgs& a, const int32_t* cells, cudaStream_t st) {
  auto k = gather_push_kernel<ORD, S>;
  constexpr size_t smem = gather_smem_bytes<ORD>();
  if (smem > 48 * 1024 - 8 * 1024) {  // static tables take a few KB of the default 48
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return ppc::cuda_check(e, "gather push smem attribute");
  }
  const int nbx = static_cast<int>((a.src_size[0] + GX - 1) / GX);
  const int nby = static_cast<int>((a.src_size[1] + GY - 1) / GY);
  const int nbz = static_cast<int>((a.src_size[2] + GZ - 1) / GZ);
  const int64_t blocks = a.N * static_cast<int64_t>(nbx) * nby * nbz;
  if (blocks > 0x7fffffffLL) return ppc::fail(PP_ERR_UNSUPPORTED, "(): gather push grid too large");
  k<<<static_cast<unsigned>(blocks), G_THREADS, smem, st>>>(a, cells, nbx, nby, nbz);
  ppc::count_launch();
  return ppc::cuda_check(cudaGetLastError(), "gather push launch");
}

}  // namespace

// Host entry (pp_capi.cu): a describes the push (trgt = values, grid,
// out = float32 output, sizes and strides; perm = the source-sorted order of
// the samples), `cells` the per-cell offsets of that order (N * prod(src) + 1
// entries).  Writes every output voxel.
int gather_push(const PPArgs& a, int order, int trgt_dtype, const int32_t* cells, cudaStream_t st) {
  if (order == 1) {
    if (trgt_dtype == PP_FLOAT32) return launch_gather<1, float>(a, cells, st);
    if (trgt_dtype == PP_BFLOAT16) return launch_gather<1, __nv_bfloat16>(a, cells, st);
  } else if (order == 3) {
    if (trgt_dtype == PP_FLOAT32) return launch_gather<3, float>(a, cells, st);
    if (trgt_dtype == PP_BFLOAT16) return launch_gather<3, __nv_bfloat16>(a, cells, st);
  }
  return ppc::fail(PP_ERR_UNSUPPORTED, "(): gather push covers orders 1 and 3, float32 / bfloat16 values");
}

}  // namespace ppk
