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
//      tile's first to last output, per axis -- is staged in shared memory:
//      by one TMA tensor copy (cp.async.bulk.tensor, mbarrier completion)
//      when the region lies inside the volume, else by loads that apply the
//      boundary condition per voxel (value times sign);
//   3. x pass: T1[ox][y][z] = sum_i wx_i S[lx + i][y][z] over the staged y, z;
//      y pass: T2[ox][oy][z] = sum_j wy_j T1[ox][ly + j][z];
//      z pass: out = sum_k wz_k T2[ox][oy][lz + k], stored along z.
// Each partial sum is the fused multiply-add chain of the per-point kernel
// (x innermost, then y, then z, starting from zero), so the result equals
// pp_grid_pull's on the materialised affine grid.  The next channel's TMA
// copy is issued as soon as the x pass has read the staged region.
#include <cuda.h>
#include <cudaTypedefs.h>

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
constexpr int RZ_MAXT = 64;  // largest tile edge (tables)

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
  int tile[3];  // TX, TY, TZ
  int ext[3];   // staged extents EX, EY, EZ (EZ a multiple of 4: the TMA box)
  int ntile[3];
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
template <int NT>
__device__ __forceinline__ void axis_stencil(const ResizeArgs& a, int d, int o, int& lo, float (&w)[NT], bool& inb) {
  float x = fmaf(a.scale[d], static_cast<float>(o), a.shift[d]);
  const float tol = (a.extrapolate & 2) ? 0.55f : 0.05f;
  inb = in_fov<float>(x, a.in_size[d], tol);
  x = fminf(fmaxf(x, -1073741824.f), 1073741824.f);
  lo = support_low<int, float>(a.order, x);
  const float f = (x - static_cast<float>(lo)) - 0.5f * static_cast<float>(a.order - 1);
  float g[NT], h[NT];
  bspline_stencil<NT, false, false, float>(a.order, a.order == 0 ? 0.f : f, w, g, h);
}

template <int NT, class S, bool TMA>
__global__ void __launch_bounds__(RZ_THREADS) resize_sep_kernel(const __grid_constant__ ResizeArgs a,
                                                                 const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(128) float rz_smem[];
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ int lo_t[3][RZ_MAXT];
  __shared__ float w_t[3][RZ_MAXT][NT];
  __shared__ unsigned char inb_t[3][RZ_MAXT];
  __shared__ int base_t[3];  // first staged node per axis
  __shared__ int interior, fits;
  __shared__ bool tma_ok;

  const int TX = a.tile[0], TY = a.tile[1], TZ = a.tile[2];
  const int EX = a.ext[0], EY = a.ext[1], EZ = a.ext[2];
  float* Sst = rz_smem;                 // [EX][EY][EZ]
  float* T1 = Sst + EX * EY * EZ;       // [TX][EY][EZ]
  float* T2 = T1 + TX * EY * EZ;        // [TX][TY][EZ]

  int t = blockIdx.x;
  const int tz = t % a.ntile[2]; t /= a.ntile[2];
  const int ty = t % a.ntile[1]; t /= a.ntile[1];
  const int tx = t % a.ntile[0];
  const int n = t / a.ntile[0];
  const int o0[3] = {tx * TX, ty * TY, tz * TZ};
  int tn[3];
  for (int d = 0; d < 3; ++d) tn[d] = min(a.tile[d], a.out_size[d] - o0[d]);

  // 1. per-axis tables
  for (int e = threadIdx.x; e < TX + TY + TZ; e += RZ_THREADS) {
    const int d = e < TX ? 0 : (e < TX + TY ? 1 : 2);
    const int i = e - (d == 0 ? 0 : (d == 1 ? TX : TX + TY));
    float w[NT];
    int lo;
    bool inb;
    axis_stencil<NT>(a, d, o0[d] + min(i, tn[d] - 1), lo, w, inb);
    lo_t[d][i] = lo;
#pragma unroll
    for (int k = 0; k < NT; ++k) w_t[d][i][k] = w[k];
    inb_t[d][i] = inb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    bool in = true, fit = true;
    for (int d = 0; d < 3; ++d) {
      int b = lo_t[d][0];
      if (d == 2) b &= ~3;  // TMA: the innermost coordinate on a 16-byte boundary
      base_t[d] = b;
      const int hi = lo_t[d][tn[d] - 1] + NT - 1;  // last node the tile reads
      fit = fit && hi - b < a.ext[d];
      in = in && b >= 0 && hi < a.in_size[d];
    }
    fits = fit;
    interior = in && fit;
    if (TMA && fit) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&mbar)), "r"(1) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
  }
  __syncthreads();
  const S* src_n = static_cast<const S*>(a.src) + static_cast<int64_t>(n) * a.src_sN;
  S* out_n = static_cast<S*>(a.out) + static_cast<int64_t>(n) * a.out_sN;
  const bool oob_zero = !(a.extrapolate & 1);
  if (!fits) {
    // the nodes of this tile span more than its staged region (float
    // rounding of the coordinates): every voxel straight from global memory
    for (int e = threadIdx.x; e < TX * TY * TZ; e += RZ_THREADS) {
      const int oz = e % TZ, r = e / TZ, oy = r % TY, ox = r / TY;
      if (ox >= tn[0] || oy >= tn[1] || oz >= tn[2]) continue;
      const bool zero = oob_zero && !(inb_t[0][ox] && inb_t[1][oy] && inb_t[2][oz]);
      for (int c = 0; c < a.C; ++c) {
        const S* sc = src_n + c * a.src_sC;
        float acc = 0.f;
        for (int k = 0; zero == false && k < NT; ++k) {
          float accy = 0.f;
          for (int j = 0; j < NT; ++j) {
            float accx = 0.f;
            for (int i = 0; i < NT; ++i) {
              const int X = lo_t[0][ox] + i, Y = lo_t[1][oy] + j, Z = lo_t[2][oz] + k;
              const int sgn = bound_sign<int>(a.bound[0], X, a.in_size[0]) *
                              bound_sign<int>(a.bound[1], Y, a.in_size[1]) *
                              bound_sign<int>(a.bound[2], Z, a.in_size[2]);
              float v = 0.f;
              if (sgn != 0)
                v = static_cast<float>(sgn) *
                    static_cast<float>(ldg_acc(sc + bound_index<int>(a.bound[0], X, a.in_size[0]) * a.src_s[0] +
                                               bound_index<int>(a.bound[1], Y, a.in_size[1]) * a.src_s[1] +
                                               bound_index<int>(a.bound[2], Z, a.in_size[2]) * a.src_s[2]));
              accx = fmaf(w_t[0][ox][i], v, accx);
            }
            accy = fmaf(w_t[1][oy][j], accx, accy);
          }
          acc = fmaf(w_t[2][oz][k], accy, acc);
        }
        out_n[c * a.out_sC + (o0[0] + ox) * a.out_s[0] + (o0[1] + oy) * a.out_s[1] + (o0[2] + oz) * a.out_s[2]] =
            from_acc<S>(acc);
      }
    }
    return;
  }
  // TMA copies serve every tile (a box reaching outside the volume reads
  // zeros there; those voxels are rewritten with their boundary value)
  const bool use_tma = TMA;
  const int bx = base_t[0], by = base_t[1], bz = base_t[2];
  const unsigned bar = smem_addr(&mbar);
  const unsigned box_bytes = static_cast<unsigned>(EX * EY * EZ * 4);

  auto issue = [&](int c) {  // one thread: TMA copy of channel c's region
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(box_bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
            smem_addr(Sst)),
        "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(bz), "r"(by), "r"(bx), "r"(n * a.C + c), "r"(bar)
        : "memory");
  };
  if (use_tma && threadIdx.x == 0) issue(0);

  // thread (lz, lr): lanes along z (stride 32), warps along rows (stride 8)
  const int lz = threadIdx.x & 31, lr = threadIdx.x >> 5;
  for (int c = 0; c < a.C; ++c) {
    // 2. staged region of channel c
    const S* sc = src_n + c * a.src_sC;
    // value of staged voxel (x, y, z) under the boundary condition
    auto bounded = [&](int X, int Y, int Z) -> float {
      const int sgn = bound_sign<int>(a.bound[0], X, a.in_size[0]) * bound_sign<int>(a.bound[1], Y, a.in_size[1]) *
                      bound_sign<int>(a.bound[2], Z, a.in_size[2]);
      if (sgn == 0) return 0.f;
      const int64_t off = bound_index<int>(a.bound[0], X, a.in_size[0]) * a.src_s[0] +
                          bound_index<int>(a.bound[1], Y, a.in_size[1]) * a.src_s[1] +
                          bound_index<int>(a.bound[2], Z, a.in_size[2]) * a.src_s[2];
      return static_cast<float>(sgn) * static_cast<float>(ldg_acc(sc + off));
    };
    if (use_tma) {
      // one thread waits for the copy (the others sleep in the barrier),
      // then every thread observes the completed phase once: acquire order
      // on the copied data without 256 threads spinning
      if (threadIdx.x == 0) tma_ok = mbar_wait(bar, static_cast<unsigned>(c & 1));
      __syncthreads();
      if (!tma_ok) {
        if (threadIdx.x == 0) {
          atomicOr(&g_resize_status, 1u);
          mbar_wait(bar, static_cast<unsigned>(c & 1));  // the copy may still land: wait once more
        }
        return;
      }
      mbar_wait(bar, static_cast<unsigned>(c & 1));
      if (!interior) {
        // rewrite the staged voxels that lie outside the volume
        for (int r = lr; r < EX * EY; r += RZ_THREADS / 32) {
          const int x = r / EY, y = r - x * EY;
          const int X = bx + x, Y = by + y;
          const bool row_in = X >= 0 && X < a.in_size[0] && Y >= 0 && Y < a.in_size[1];
          for (int z = lz; z < EZ; z += 32) {
            const int Z = bz + z;
            if (row_in && Z >= 0 && Z < a.in_size[2]) continue;
            Sst[r * EZ + z] = bounded(X, Y, Z);
          }
        }
      }
    } else {
      for (int r = lr; r < EX * EY; r += RZ_THREADS / 32) {
        const int x = r / EY, y = r - x * EY;
        const int X = bx + x, Y = by + y;
        const bool row_in = X >= 0 && X < a.in_size[0] && Y >= 0 && Y < a.in_size[1];
        const S* rowp = sc + X * a.src_s[0] + Y * a.src_s[1];
        for (int z = lz; z < EZ; z += 32) {
          const int Z = bz + z;
          Sst[r * EZ + z] = (row_in && Z >= 0 && Z < a.in_size[2]) ? static_cast<float>(ldg_acc(rowp + Z * a.src_s[2]))
                                                                    : bounded(X, Y, Z);
        }
      }
    }
    __syncthreads();
    // 3a. x pass over every staged (y, z): rows (ox, y)
    for (int r = lr; r < TX * EY; r += RZ_THREADS / 32) {
      const int ox = r / EY, y = r - ox * EY;
      float w[NT];
#pragma unroll
      for (int i = 0; i < NT; ++i) w[i] = w_t[0][ox][i];
      const float* sp = Sst + ((lo_t[0][ox] - bx) * EY + y) * EZ;
      for (int z = lz; z < EZ; z += 32) {
        float acc = 0.f;
#pragma unroll
        for (int i = 0; i < NT; ++i) acc = fmaf(w[i], sp[i * EY * EZ + z], acc);
        T1[r * EZ + z] = acc;
      }
    }
    __syncthreads();
    if (use_tma && c + 1 < a.C && threadIdx.x == 0) issue(c + 1);  // S is free again
    // 3b. y pass: rows (ox, oy)
    for (int r = lr; r < TX * TY; r += RZ_THREADS / 32) {
      const int ox = r / TY, oy = r - ox * TY;
      float w[NT];
#pragma unroll
      for (int j = 0; j < NT; ++j) w[j] = w_t[1][oy][j];
      const float* tp = T1 + (ox * EY + (lo_t[1][oy] - by)) * EZ;
      for (int z = lz; z < EZ; z += 32) {
        float acc = 0.f;
#pragma unroll
        for (int j = 0; j < NT; ++j) acc = fmaf(w[j], tp[j * EZ + z], acc);
        T2[r * EZ + z] = acc;
      }
    }
    __syncthreads();
    // 3c. z pass and store: rows (ox, oy), lanes along oz
    for (int r = lr; r < TX * TY; r += RZ_THREADS / 32) {
      const int ox = r / TY, oy = r - ox * TY;
      if (ox >= tn[0] || oy >= tn[1]) continue;
      const bool inxy = inb_t[0][ox] && inb_t[1][oy];
      const float* tp = T2 + r * EZ - bz;
      S* op = out_n + c * a.out_sC + (o0[0] + ox) * a.out_s[0] + (o0[1] + oy) * a.out_s[1] + o0[2] * a.out_s[2];
      for (int oz = lz; oz < tn[2]; oz += 32) {
        float acc = 0.f;
        if (!oob_zero || (inxy && inb_t[2][oz])) {
          const float* tz = tp + lo_t[2][oz];
#pragma unroll
          for (int k = 0; k < NT; ++k) acc = fmaf(w_t[2][oz][k], tz[k], acc);
        }
        op[oz * a.out_s[2]] = from_acc<S>(acc);
      }
    }
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

size_t smem_floats(const int (&t)[3], const int (&e)[3]) {
  return static_cast<size_t>(e[0]) * e[1] * e[2] + static_cast<size_t>(t[0]) * e[1] * e[2] +
         static_cast<size_t>(t[0]) * t[1] * e[2];
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

// Largest working set of a tile (floats of dynamic shared memory).
constexpr size_t RZ_SMEM_FLOATS = 15 * 1024;

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
  ppk::note_kernel(TMA ? "resize_sep_kernel tma" : "resize_sep_kernel", 0, NT - 1, 1);
  resize_sep_kernel<NT, S, TMA><<<static_cast<unsigned>(ntiles), RZ_THREADS, smem, st>>>(a, map);
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

}  // namespace

extern "C" {

int pp_resize(const pp_tensor* input, const pp_tensor* out, const double* scale, const double* shift,
              const pp_options* opt, void* stream) {
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
  if (!scale || !shift) return fail(PP_ERR_ARG, "(): expected scale and shift");
  int bound[3], order[3];
  if ((rc = read_options(opt, 3, bound, order))) return rc;
  if (order[1] != order[0] || order[2] != order[0] || order[0] > 3)
    return fail(PP_ERR_UNSUPPORTED, "(): pp_resize takes one B-spline order of at most 3 for all axes");
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
  const int NT = order[0] == 0 ? 1 : order[0] + 1;
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
  a.order = order[0];
  a.extrapolate = opt->extrapolate;
  if (ntiles >= (int64_t(1) << 31)) return fail(PP_ERR_UNSUPPORTED, "(): pp_resize: too many tiles");

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
  cudaError_t e = input->dtype == PP_FLOAT32 ? dispatch<float>(order[0], tma, a, map, smem, ntiles, st)
                                             : dispatch<__nv_bfloat16>(order[0], false, a, map, smem, ntiles, st);
  count_launch();
  return cuda_check(e, "resize launch");
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
