// Field and grid regularisers: out = (H + L) x.
//
// nitorch's native regularisers (nitorch/_C/src/regulariser.cpp:19-64 and
// regulariser_grid.cpp, kernels nitorch/_C/src/impl/regulariser_common.cpp
// and regulariser_grid_common.cpp) apply the matrix of a quadratic energy --
// absolute values, membrane (first derivatives), bending (second
// derivatives) and, for displacement grids, the linear-elastic (Lame)
// shear and divergence terms -- plus a voxel-wise Hessian.  The reference
// writes one function per (dimension, penalty mix, weighting) with the
// stencil spelled out.  All of them share one shape, which is what the
// kernel here computes, per output channel c:
//   a_c * x_c                                              (centre)
//   + sum_axis c1_c[axis] * (d(-1) + d(+1))                (+-1 steps)
//   + sum_axis c2_c[axis] * (d(-2) + d(+2))                (+-2 steps, bending)
//   + sum_pair cd_c[pair] * (four diagonal differences)    (bending)
//   + w2 * (Lame coupling: other components on the diagonals of
//           (own axis, other axis), grids only)
//   + (H x)_c
// with d(o) = sign * x_c(neighbour o) - x_c(centre) under the boundary
// index and sign of every axis stepped along.  With a weight map (absolute
// and membrane only) the centre term is a_c * w * x_c and the +-1 terms
// c1_c[axis] * (w + sign * w(nbr)) * d.  The host fills the coefficients
// from the reference's set_kernel formulas (regulariser_common.cpp:285-299,
// regulariser_grid_common.cpp:265-298); the kernel is compiled per
// (dimension, stencil radius, weighted, Lame), so every neighbour offset
// and sign lives in registers.  Differences and their group sums are formed
// in the storage type as in the reference; the group terms are accumulated
// in the storage type too (the reference accumulates them in float64, which
// moves a float32 result by a few ulps at most).  Voxels at least R from
// every edge take a path without boundary signs.
// A thread per voxel, the last axis fastest (coalesced rows; the
// neighbours come from L1 / L2): HBM-bound, each input element read once
// from DRAM and each output element written once.
//
// Behaviour where the reference is defective: a call with every penalty
// zero returns the Hessian product (the reference's field kernel loops
// forever in its `zeros` function, regulariser_common.cpp:739-748); weights
// and Hessians are read per batch item (the reference's field kernel reads
// item 0's weights for every item, :862, and its grid kernel offsets the
// Hessian by the input's batch stride, regulariser_grid_common.cpp:817).
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>

#include "../../include/nitorch_b200.h"
#include "pp_capi_internal.cuh"
#include "pp_kernels.cuh"

namespace {

constexpr int kRegMaxChan = 64;

enum RegHess : int32_t { RH_NONE = 0, RH_EYE = 1, RH_DIAG = 2, RH_ESTATICS = 3, RH_SYM = 4 };

// Coefficients of one output channel (pairs: (0,1), (0,2), (1,2)), in the
// accumulation type of the storage type.
template <class T> struct Coef {
  T a, c1[3], c2[3], cd[3];
};

struct RegArgs {
  int32_t C, hess, CC;
  int32_t narrow;  // every neighbour offset fits 32 bits: int32 offset arithmetic
  int32_t bound[3];
  int32_t size[3];
  int64_t nvox;
  int64_t isN, isC, is[3];
  int64_t osN, osC, os[3];
  int64_t wsN, wsC, ws[3];
  int64_t hsN, hsC, hs[3];
  double w2;  // Lame coupling (grids)
  float w2f;
  int32_t pad2;
  const void* inp;
  void* out;
  const void* wgt;
  const void* hes;
  Coef<double> kd[kRegMaxChan];
  Coef<float> kf[kRegMaxChan];
};
static_assert(sizeof(RegArgs) <= 32764, "regulariser argument above the kernel-parameter limit");

template <class T> __device__ __forceinline__ const Coef<T>& coef(const RegArgs& A, int c);
template <> __device__ __forceinline__ const Coef<double>& coef<double>(const RegArgs& A, int c) { return A.kd[c]; }
template <> __device__ __forceinline__ const Coef<float>& coef<float>(const RegArgs& A, int c) { return A.kf[c]; }
template <class T> __device__ __forceinline__ T lame_w2(const RegArgs& A);
template <> __device__ __forceinline__ double lame_w2<double>(const RegArgs& A) { return A.w2; }
template <> __device__ __forceinline__ float lame_w2<float>(const RegArgs& A) { return A.w2f; }

// Index of the (i, j) entry, i < j, of a symmetric C x C matrix stored as its
// diagonal then the upper triangle row by row.
__device__ __forceinline__ int sym_index(int i, int j, int C) { return C + i * C - i * (i + 1) / 2 + (j - i - 1); }

// sign * x[off] (sign 0: outside the volume, nothing read) -- bound::get.
// INNER: every neighbour lies inside the volume (sign 1).
template <bool INNER, class S, class I>
__device__ __forceinline__ S nbr(const S* x, I off, int s) {
  if constexpr (INNER) return x[off];
  else return s == 0 ? S(0) : (s > 0 ? x[off] : -x[off]);
}

// I: int32 when every neighbour offset of every tensor fits, else int64.
template <class I> struct Nbrs {
  I im[3][2], ip[3][2], wm[3], wp[3];
  int sm[3][2], sp[3][2];
};

// One voxel: every output channel.  Accumulation in the storage type (float
// for float32 fields: the differences and group sums are formed in float as
// in the reference, whose float64 accumulation of the ten-odd group terms
// changes the float32 result by at most a few ulps).
// entry c of three registers, without indexing them (no local memory)
template <class V>
__device__ __forceinline__ V sel3(int c, V v0, V v1, V v2) { return c == 0 ? v0 : (c == 1 ? v1 : v2); }

template <class S, class I, int DIM, int R, bool W, bool LAME, bool G, bool INNER>
__device__ __forceinline__ void voxel(const RegArgs& A, const S* x, S* out, const S* w, int64_t ho, const Nbrs<I>& N) {
  using T = S;
#pragma unroll 1
  for (int c = 0; c < (G ? DIM : A.C); ++c) {
    const Coef<T>& K = coef<T>(A, c);
    const S* xc = x + c * A.isC;
    const S cen = xc[0];
    T acc;
    if constexpr (W) {
      const S* wc_ = w + c * A.wsC;
      const S wc = wc_[0];
      acc = K.a * wc * cen;
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        const S dm = nbr<INNER>(xc, N.im[a][0], N.sm[a][0]) - cen, dp = nbr<INNER>(xc, N.ip[a][0], N.sp[a][0]) - cen;
        const S gm = wc + nbr<INNER>(wc_, N.wm[a], N.sm[a][0]), gp = wc + nbr<INNER>(wc_, N.wp[a], N.sp[a][0]);
        acc += K.c1[a] * gm * dm + K.c1[a] * gp * dp;
      }
    } else {
      acc = K.a * cen;
#pragma unroll
      for (int a = 0; a < DIM; ++a)
        acc += K.c1[a] * ((nbr<INNER>(xc, N.im[a][0], N.sm[a][0]) - cen) + (nbr<INNER>(xc, N.ip[a][0], N.sp[a][0]) - cen));
      if constexpr (R == 2) {
#pragma unroll
        for (int a = 0; a < DIM; ++a)
          acc += K.c2[a] * ((nbr<INNER>(xc, N.im[a][1], N.sm[a][1]) - cen) +
                            (nbr<INNER>(xc, N.ip[a][1], N.sp[a][1]) - cen));
#pragma unroll
        for (int p = 0; p < (DIM == 3 ? 3 : DIM - 1); ++p) {
          const int ai = p == 2 ? 1 : 0, aj = p == 0 ? 1 : 2;
          const S s = (nbr<INNER>(xc, N.im[ai][0] + N.im[aj][0], N.sm[ai][0] * N.sm[aj][0]) - cen) +
                      (nbr<INNER>(xc, N.ip[ai][0] + N.im[aj][0], N.sp[ai][0] * N.sm[aj][0]) - cen) +
                      (nbr<INNER>(xc, N.im[ai][0] + N.ip[aj][0], N.sm[ai][0] * N.sp[aj][0]) - cen) +
                      (nbr<INNER>(xc, N.ip[ai][0] + N.ip[aj][0], N.sp[ai][0] * N.sp[aj][0]) - cen);
          acc += K.cd[p] * s;
        }
      }
      if constexpr (LAME) {
        // component c against each other component e on the diagonals of
        // (axis c, axis e): + (c+, e-) - (c+, e+) + (c-, e+) - (c-, e-)
        const I cp = sel3(c, N.ip[0][0], N.ip[DIM > 1 ? 1 : 0][0], N.ip[DIM > 2 ? 2 : 0][0]);
        const I cm = sel3(c, N.im[0][0], N.im[DIM > 1 ? 1 : 0][0], N.im[DIM > 2 ? 2 : 0][0]);
        const int scp = sel3(c, N.sp[0][0], N.sp[DIM > 1 ? 1 : 0][0], N.sp[DIM > 2 ? 2 : 0][0]);
        const int scm = sel3(c, N.sm[0][0], N.sm[DIM > 1 ? 1 : 0][0], N.sm[DIM > 2 ? 2 : 0][0]);
        S s = S(0);
#pragma unroll
        for (int e = 0; e < DIM; ++e) {
          if (e == c) continue;
          const S* xe = x + e * A.isC;
          s = s + nbr<INNER>(xe, cp + N.im[e][0], scp * N.sm[e][0]) - nbr<INNER>(xe, cp + N.ip[e][0], scp * N.sp[e][0]) +
              nbr<INNER>(xe, cm + N.ip[e][0], scm * N.sp[e][0]) - nbr<INNER>(xe, cm + N.im[e][0], scm * N.sm[e][0]);
        }
        acc += lame_w2<T>(A) * s;
      }
    }
    if (A.hess != RH_NONE) {
      const S* h = static_cast<const S*>(A.hes) + ho;
      const int C = A.C;
      switch (A.hess) {
        case RH_EYE: acc += h[0] * cen; break;
        case RH_DIAG: acc += h[c * A.hsC] * cen; break;
        case RH_ESTATICS:  // [[diag(d), b], [b^T, r]] stored as d_0..d_{C-2}, r, b_0..b_{C-2}
          if (c < C - 1) {
            acc += h[c * A.hsC] * cen + h[(C + c) * A.hsC] * x[(C - 1) * A.isC];
          } else {
            acc += h[(C - 1) * A.hsC] * cen;
            for (int k = 0; k < C - 1; ++k) acc += h[(C + k) * A.hsC] * x[k * A.isC];
          }
          break;
        default:  // RH_SYM
          acc += h[c * A.hsC] * cen;
          for (int k = 0; k < C; ++k) {
            if (k == c) continue;
            const int hk = k < c ? sym_index(k, c, C) : sym_index(c, k, C);
            acc += h[hk * A.hsC] * x[k * A.isC];
          }
          break;
      }
    }
    out[c * A.osC] = acc;
  }
}

// G: displacement grid (C = DIM components, channel loop unrolled so that the
// Lame terms index the per-axis registers at compile time).
// Resident blocks the register budget is set for (radius 1 without weights:
// at most 64 registers a thread, otherwise 85, float64 radius 2: 128):
// latency hiding needs the warps more than the registers.
template <class S, int R, bool W> struct RegBlocks {
  static constexpr int value = (R == 1 && !W) ? 4 : (sizeof(S) == 8 && R == 2 ? 2 : 3);
};

template <class S, class I, int DIM, int R, bool W, bool LAME, bool G>
__global__ void __launch_bounds__(256, RegBlocks<S, R, W>::value) regulariser_kernel(const __grid_constant__ RegArgs A) {
  static_assert(G || !LAME, "Lame terms are for grids");
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < A.nvox; i += step) {
    int sub[3] = {0, 0, 0};
    int64_t n;
    if (A.nvox <= 0x7fffffffLL) {  // 32-bit coordinate arithmetic
      unsigned r = static_cast<unsigned>(i);
#pragma unroll
      for (int a = DIM - 1; a >= 0; --a) {
        sub[a] = static_cast<int>(r % static_cast<unsigned>(A.size[a]));
        r /= static_cast<unsigned>(A.size[a]);
      }
      n = r;
    } else {
      int64_t r = i;
#pragma unroll
      for (int a = DIM - 1; a >= 0; --a) {
        sub[a] = static_cast<int>(r % A.size[a]);
        r /= A.size[a];
      }
      n = r;
    }
    // +-1 and +-2 neighbours per axis: element offsets (input, weights) and signs
    Nbrs<I> N;
    bool inner = true;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      if (sub[a] >= R && sub[a] < A.size[a] - R) {  // interior along this axis: plain steps
#pragma unroll
        for (int k = 0; k < R; ++k) {
          N.im[a][k] = static_cast<I>(-(k + 1) * A.is[a]);
          N.ip[a][k] = static_cast<I>((k + 1) * A.is[a]);
          N.sm[a][k] = N.sp[a][k] = 1;
          if (W && k == 0) {
            N.wm[a] = static_cast<I>(-A.ws[a]);
            N.wp[a] = static_cast<I>(A.ws[a]);
          }
        }
        continue;
      }
      inner = false;
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const int lo = sub[a] - (k + 1), hi = sub[a] + (k + 1), nn = A.size[a];
        const int slo = ppk::bound_sign<int>(A.bound[a], lo, nn), shi = ppk::bound_sign<int>(A.bound[a], hi, nn);
        const int ilo = slo ? ppk::bound_index<int>(A.bound[a], lo, nn) : sub[a];
        const int ihi = shi ? ppk::bound_index<int>(A.bound[a], hi, nn) : sub[a];
        N.im[a][k] = static_cast<I>(static_cast<int64_t>(ilo - sub[a]) * A.is[a]);
        N.ip[a][k] = static_cast<I>(static_cast<int64_t>(ihi - sub[a]) * A.is[a]);
        N.sm[a][k] = slo;
        N.sp[a][k] = shi;
        if (W && k == 0) {
          N.wm[a] = static_cast<I>(static_cast<int64_t>(ilo - sub[a]) * A.ws[a]);
          N.wp[a] = static_cast<I>(static_cast<int64_t>(ihi - sub[a]) * A.ws[a]);
        }
      }
    }
    int64_t io = n * A.isN, oo = n * A.osN, wo = n * A.wsN, ho = n * A.hsN;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      io += sub[a] * A.is[a];
      oo += sub[a] * A.os[a];
      wo += sub[a] * A.ws[a];
      ho += sub[a] * A.hs[a];
    }
    const S* x = static_cast<const S*>(A.inp) + io;
    S* out = static_cast<S*>(A.out) + oo;
    const S* w = W ? static_cast<const S*>(A.wgt) + wo : nullptr;
    if (inner)
      voxel<S, I, DIM, R, W, LAME, G, true>(A, x, out, w, ho, N);
    else
      voxel<S, I, DIM, R, W, LAME, G, false>(A, x, out, w, ho, N);
  }
}

// ---- host ------------------------------------------------------------------

// 1 / voxel_size^2 per axis, zero beyond the field's dimension
void voxel_factors(const double* vs, int dim, double (&vx)[3]) {
  for (int a = 0; a < 3; ++a) vx[a] = a < dim ? 1.0 / (vs[a] * vs[a]) : 0.0;
}

void set_layout(const pp_tensor* t, int dim, int chan_axis, int first_spatial, int64_t& sN, int64_t& sC,
                int64_t (&s)[3]) {
  sN = t->strides[0];
  sC = chan_axis >= 0 ? t->strides[chan_axis] : 0;
  for (int a = 0; a < 3; ++a) s[a] = a < dim ? t->strides[first_spatial + a] : 0;
}

int check_float(const pp_tensor* t, int dtype, const char* name) {
  int rc = ppc::check_tensor(t, name);
  if (rc) return rc;
  if (t->dtype != dtype) return ppc::fail(PP_ERR_DTYPE, "(): %s must have the input's dtype", name);
  return PP_OK;
}

// out must not share memory with the tensors the stencil reads
bool overlaps(const pp_tensor* a, const pp_tensor* b) {
  if (!a || !b || !a->data || !b->data) return false;
  const char* a0 = static_cast<const char*>(a->data);
  const char* b0 = static_cast<const char*>(b->data);
  const char* a1 = a0 + (ppc::max_offset(a, 0) + 1) * ppc::dtype_size(a->dtype);
  const char* b1 = b0 + (ppc::max_offset(b, 0) + 1) * ppc::dtype_size(b->dtype);
  return a0 < b1 && b0 < a1;
}

template <class S, int DIM, int R, bool W, bool LAME, bool G>
void launch_one(const RegArgs& A, cudaStream_t st) {
  const int64_t want = (A.nvox + 255) / 256;
  const unsigned nb = static_cast<unsigned>(want < 148 * 32 ? want : 148 * 32);
  if (A.narrow)
    regulariser_kernel<S, int32_t, DIM, R, W, LAME, G><<<nb, 256, 0, st>>>(A);
  else
    regulariser_kernel<S, int64_t, DIM, R, W, LAME, G><<<nb, 256, 0, st>>>(A);
}

template <class S, int DIM>
void launch_dim(const RegArgs& A, bool grid, int R, bool W, bool lame, cudaStream_t st) {
  if (grid) {
    if (W) return launch_one<S, DIM, 1, true, false, true>(A, st);
    if (R == 2) return lame ? launch_one<S, DIM, 2, false, true, true>(A, st) : launch_one<S, DIM, 2, false, false, true>(A, st);
    return lame ? launch_one<S, DIM, 1, false, true, true>(A, st) : launch_one<S, DIM, 1, false, false, true>(A, st);
  }
  if (W) return launch_one<S, DIM, 1, true, false, false>(A, st);
  if (R == 2) return launch_one<S, DIM, 2, false, false, false>(A, st);
  return launch_one<S, DIM, 1, false, false, false>(A, st);
}

// Neighbour offsets (at most two steps along each axis) of a tensor fit 32 bits.
bool narrow_ok(const pp_tensor* t) { return !t || 4 * ppc::max_offset(t, 1) < (int64_t(1) << 31); }

int launch(RegArgs& A, int dtype, int dim, bool grid, int R, bool W, bool lame, cudaStream_t st) {
  if (A.nvox == 0) return PP_OK;
  if (dtype == PP_FLOAT32) {
    if (dim == 1) launch_dim<float, 1>(A, grid, R, W, lame, st);
    else if (dim == 2) launch_dim<float, 2>(A, grid, R, W, lame, st);
    else launch_dim<float, 3>(A, grid, R, W, lame, st);
  } else {
    if (dim == 1) launch_dim<double, 1>(A, grid, R, W, lame, st);
    else if (dim == 2) launch_dim<double, 2>(A, grid, R, W, lame, st);
    else launch_dim<double, 3>(A, grid, R, W, lame, st);
  }
  ppc::count_launch();
  return ppc::cuda_check(cudaGetLastError(), "regulariser launch");
}

// The float copies of the coefficients (float32 fields accumulate in float).
void float_coefs(RegArgs& A, int C) {
  for (int c = 0; c < C; ++c) {
    const Coef<double>& d = A.kd[c];
    Coef<float>& f = A.kf[c];
    f.a = static_cast<float>(d.a);
    for (int k = 0; k < 3; ++k) {
      f.c1[k] = static_cast<float>(d.c1[k]);
      f.c2[k] = static_cast<float>(d.c2[k]);
      f.cd[k] = static_cast<float>(d.cd[k]);
    }
  }
  A.w2f = static_cast<float>(A.w2);
}

// Pair p of the diagonal terms: (0,1), (0,2), (1,2) in 3-D; (0,1) in 2-D.
void pair_axes(int p, int& i, int& j) {
  i = p == 2 ? 1 : 0;
  j = p == 0 ? 1 : 2;
}

}  // namespace

extern "C" {

int pp_regulariser(const pp_tensor* input, const pp_tensor* weight, const pp_tensor* hessian, const pp_tensor* out,
                   const double* absolute, const double* membrane, const double* bending, const double* voxel_size,
                   const int32_t* bound, void* stream) {
  int rc = ppc::check_tensor(input, "input");
  if (rc) return rc;
  if (input->ndim < 3 || input->ndim > 5) return ppc::fail(PP_ERR_ARG, "(): input must be (N, C, *spatial), 1-3-D");
  if (input->dtype != PP_FLOAT32 && input->dtype != PP_FLOAT64)
    return ppc::fail(PP_ERR_DTYPE, "(): the regulariser takes float32 or float64 fields");
  if (!absolute || !membrane || !bending || !voxel_size || !bound)
    return ppc::fail(PP_ERR_ARG, "(): expected penalties, voxel sizes and bounds");
  const int dim = input->ndim - 2;
  const int64_t C64 = input->sizes[1];
  if (C64 < 1 || C64 > kRegMaxChan) return ppc::fail(PP_ERR_UNSUPPORTED, "(): 1 to %d channels", kRegMaxChan);
  const int C = static_cast<int>(C64);
  if ((rc = check_float(out, input->dtype, "output"))) return rc;
  for (int i = 0; i < input->ndim; ++i)
    if (out->ndim != input->ndim || out->sizes[i] != input->sizes[i])
      return ppc::fail(PP_ERR_ARG, "(): output must have the input's shape");
  if (overlaps(out, input) || overlaps(out, weight) || overlaps(out, hessian))
    return ppc::fail(PP_ERR_ARG, "(): output must not overlap the inputs");
  bool has_b = false;
  for (int c = 0; c < C; ++c) has_b = has_b || bending[c] != 0.0;
  static thread_local RegArgs A;
  std::memset(&A, 0, sizeof(A));
  A.C = C;
  if (weight) {
    if ((rc = check_float(weight, input->dtype, "weight"))) return rc;
    for (int i = 0; i < input->ndim; ++i)
      if (weight->ndim != input->ndim || weight->sizes[i] != input->sizes[i])
        return ppc::fail(PP_ERR_ARG, "(): weight must be expanded to the input's shape");
    if (has_b) return ppc::fail(PP_ERR_UNSUPPORTED, "(): RLS only implemented for membrane or absolute");
  }
  if (hessian) {
    if ((rc = check_float(hessian, input->dtype, "hessian"))) return rc;
    bool same = hessian->ndim == input->ndim && hessian->sizes[0] == input->sizes[0];
    for (int i = 2; same && i < input->ndim; ++i) same = hessian->sizes[i] == input->sizes[i];
    if (!same) return ppc::fail(PP_ERR_ARG, "(): hessian must be (N, CC, *spatial) like the input");
    const int64_t CC = hessian->sizes[1];
    A.CC = static_cast<int>(CC);
    A.hess = CC == 1 ? RH_EYE : CC == C ? RH_DIAG : CC == 2 * C - 1 ? RH_ESTATICS : CC == C * (C + 1) / 2 ? RH_SYM : -1;
    if (A.hess < 0) return ppc::fail(PP_ERR_ARG, "(): hessian channels must be 1, C, 2C-1 or C(C+1)/2");
  }
  for (int a = 0; a < 3; ++a) {
    const int64_t n = a < dim ? input->sizes[2 + a] : 1;
    if (n > 0x7fffffff) return ppc::fail(PP_ERR_UNSUPPORTED, "(): axis too long");
    A.bound[a] = bound[a];
    A.size[a] = static_cast<int32_t>(n);
  }
  A.nvox = input->sizes[0] * int64_t(A.size[0]) * A.size[1] * A.size[2];
  set_layout(input, dim, 1, 2, A.isN, A.isC, A.is);
  set_layout(out, dim, 1, 2, A.osN, A.osC, A.os);
  if (weight) set_layout(weight, dim, 1, 2, A.wsN, A.wsC, A.ws);
  if (hessian) set_layout(hessian, dim, 1, 2, A.hsN, A.hsC, A.hs);
  A.inp = input->data;
  A.out = out->data;
  A.wgt = weight ? weight->data : nullptr;
  A.hes = hessian ? hessian->data : nullptr;
  double vx[3];
  voxel_factors(voxel_size, dim, vx);
  const double svx = vx[0] + vx[1] + vx[2];
  for (int c = 0; c < C; ++c) {
    Coef<double>& K = A.kd[c];
    const double a = absolute[c], m = membrane[c], b = bending[c];
    K.a = a;
    for (int ax = 0; ax < 3; ++ax) {
      if (weight) {  // vel2mom*_rls_membrane / _rls_absolute
        K.c1[ax] = m * 0.5 * -vx[ax];
      } else {       // vel2mom*_absolute / _membrane / _bending
        K.c1[ax] = m * -vx[ax] + b * (-4.0 * vx[ax] * svx);
        K.c2[ax] = b * vx[ax] * vx[ax];
      }
    }
    for (int p = 0; p < 3 && !weight; ++p) {
      int i, j;
      pair_axes(p, i, j);
      K.cd[p] = b * 2.0 * vx[i] * vx[j];
    }
  }
  float_coefs(A, C);
  A.narrow = narrow_ok(input) && narrow_ok(weight);
  return launch(A, input->dtype, dim, false, has_b ? 2 : 1, weight != nullptr, false,
                static_cast<cudaStream_t>(stream));
}

int pp_regulariser_grid(const pp_tensor* input, const pp_tensor* weight, const pp_tensor* hessian,
                        const pp_tensor* out, double absolute, double membrane, double bending, double shear,
                        double div, const double* voxel_size, const int32_t* bound, void* stream) {
  int rc = ppc::check_tensor(input, "input");
  if (rc) return rc;
  if (input->ndim < 3 || input->ndim > 5 || input->sizes[input->ndim - 1] != input->ndim - 2)
    return ppc::fail(PP_ERR_ARG, "(): input must be (N, *spatial, D) with D = 1-3 spatial dimensions");
  if (input->dtype != PP_FLOAT32 && input->dtype != PP_FLOAT64)
    return ppc::fail(PP_ERR_DTYPE, "(): the regulariser takes float32 or float64 fields");
  if (!voxel_size || !bound) return ppc::fail(PP_ERR_ARG, "(): expected voxel sizes and bounds");
  const int D = input->ndim - 2, last = input->ndim - 1;
  if ((rc = check_float(out, input->dtype, "output"))) return rc;
  for (int i = 0; i < input->ndim; ++i)
    if (out->ndim != input->ndim || out->sizes[i] != input->sizes[i])
      return ppc::fail(PP_ERR_ARG, "(): output must have the input's shape");
  if (overlaps(out, input) || overlaps(out, weight) || overlaps(out, hessian))
    return ppc::fail(PP_ERR_ARG, "(): output must not overlap the inputs");
  static thread_local RegArgs A;
  std::memset(&A, 0, sizeof(A));
  A.C = D;
  if (weight) {
    if ((rc = check_float(weight, input->dtype, "weight"))) return rc;
    bool same = weight->ndim == input->ndim - 1;
    for (int i = 0; same && i < input->ndim - 1; ++i) same = weight->sizes[i] == input->sizes[i];
    if (!same) return ppc::fail(PP_ERR_ARG, "(): weight must be (N, *spatial) like the input");
    if (bending != 0.0 || shear != 0.0 || div != 0.0)
      return ppc::fail(PP_ERR_UNSUPPORTED, "(): RLS only implemented for membrane or absolute");
  }
  if (hessian) {
    if ((rc = check_float(hessian, input->dtype, "hessian"))) return rc;
    bool same = hessian->ndim == input->ndim;
    for (int i = 0; same && i < input->ndim - 1; ++i) same = hessian->sizes[i] == input->sizes[i];
    if (!same) return ppc::fail(PP_ERR_ARG, "(): hessian must be (N, *spatial, DD) like the input");
    const int64_t DD = hessian->sizes[last];
    A.CC = static_cast<int>(DD);
    A.hess = DD == 1 ? RH_EYE : DD == D ? RH_DIAG : DD == D * (D + 1) / 2 ? RH_SYM : -1;
    if (A.hess < 0) return ppc::fail(PP_ERR_ARG, "(): hessian components must be 1, D or D(D+1)/2");
  }
  for (int a = 0; a < 3; ++a) {
    const int64_t n = a < D ? input->sizes[1 + a] : 1;
    if (n > 0x7fffffff) return ppc::fail(PP_ERR_UNSUPPORTED, "(): axis too long");
    A.bound[a] = bound[a];
    A.size[a] = static_cast<int32_t>(n);
  }
  A.nvox = input->sizes[0] * int64_t(A.size[0]) * A.size[1] * A.size[2];
  set_layout(input, D, last, 1, A.isN, A.isC, A.is);
  set_layout(out, D, last, 1, A.osN, A.osC, A.os);
  if (weight) set_layout(weight, D, -1, 1, A.wsN, A.wsC, A.ws);
  if (hessian) set_layout(hessian, D, last, 1, A.hsN, A.hsC, A.hs);
  A.inp = input->data;
  A.out = out->data;
  A.wgt = weight ? weight->data : nullptr;
  A.hes = hessian ? hessian->data : nullptr;
  double vx[3];
  voxel_factors(voxel_size, D, vx);
  const double svx = vx[0] + vx[1] + vx[2];
  const double lam0 = absolute, lam1 = membrane, lam2 = bending, mu = shear, lam = div;
  double w1[3];
  for (int a = 0; a < 3; ++a) w1[a] = lam2 * (-4.0 * vx[a] * svx) - lam1 * vx[a];
  A.w2 = weight ? 0.0 : 0.25 * mu + 0.25 * lam;
  for (int d = 0; d < D; ++d) {
    Coef<double>& K = A.kd[d];
    const double s = 1.0 / vx[d];  // component d in the units of its axis
    K.a = lam0 * s;
    for (int ax = 0; ax < D; ++ax) {
      if (weight) {  // vel2mom*_rls_membrane / _rls_absolute
        K.c1[ax] = 0.5 * w1[ax] * s;
      } else {       // vel2mom*_absolute / _membrane / _bending / _lame / _all
        K.c1[ax] = w1[ax] * s + (ax == d ? -2.0 * mu - lam : -mu * vx[ax] / vx[d]);
        K.c2[ax] = lam2 * vx[ax] * vx[ax] * s;
      }
    }
    for (int p = 0; p < 3 && !weight; ++p) {
      int i, j;
      pair_axes(p, i, j);
      K.cd[p] = lam2 * 2.0 * vx[i] * vx[j] * s;
    }
  }
  float_coefs(A, D);
  A.narrow = narrow_ok(input) && narrow_ok(weight);
  return launch(A, input->dtype, D, true, lam2 != 0.0 ? 2 : 1, weight != nullptr, A.w2 != 0.0,
                static_cast<cudaStream_t>(stream));
}

}  // extern "C"
