// Field and grid regularisers: out = (H + L) x.
//
// nitorch's native regularisers (nitorch/_C/src/regulariser.cpp:19-64 and
// regulariser_grid.cpp, kernels nitorch/_C/src/impl/regulariser_common.cpp
// and regulariser_grid_common.cpp) apply the matrix of a quadratic energy --
// absolute values, membrane (first derivatives), bending (second
// derivatives) and, for displacement grids, the linear-elastic (Lame)
// shear and divergence terms -- plus a voxel-wise Hessian.  The reference
// writes one function per (dimension, penalty mix, weighting) with the
// stencil spelled out; each of them is a linear stencil made of
//   * the centre value times a coefficient,
//   * differences sign * value(neighbour) - value(centre) along +-1 and +-2
//     steps of an axis and along the four diagonals of an axis pair,
//   * for grids with Lame terms, raw neighbour values of the other
//     components on the diagonals of (own axis, other axis),
//   * with a weight map (absolute / membrane only), the centre term and the
//     +-1 differences scaled by the local weights,
// plus the Hessian product at the voxel.  Here the host writes that stencil
// as a table of terms per output channel (offset, source channel, kind,
// coefficient: the reference's set_kernel formulas, regulariser_common.cpp:
// 285-299 and regulariser_grid_common.cpp:265-298) and one kernel applies
// any table: a thread per voxel, its neighbours gathered through the
// boundary index and sign of every axis they step along (differences
// formed in the storage type, accumulation in float64, as the reference
// does), the table read from the kernel parameter (constant bank, the same
// term for every thread of a warp).  HBM-bound: every input element is read
// once from DRAM (the neighbours come from L1 / L2) and every output
// element written once.
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
constexpr int kRegMaxTerms = 1600;

enum RegKind : int8_t {
  RK_CENTRE = 0,   // coef * value(src, centre)
  RK_DIFF = 1,     // coef * (sign * value(src, nbr) - value(src, centre))
  RK_RAW = 2,      // coef * sign * value(src, nbr)
  RK_WCENTRE = 3,  // coef * w(centre) * value(centre)
  RK_WDIFF = 4,    // coef * (w(centre) + sign * w(nbr)) * difference
};
enum RegHess : int32_t { RH_NONE = 0, RH_EYE = 1, RH_DIAG = 2, RH_ESTATICS = 3, RH_SYM = 4 };

struct RegTerm {
  int8_t o[3];  // step along each axis, -2..2
  int8_t src;   // source channel
  int8_t kind;
  int8_t pad[3];
  double coef;
};
static_assert(sizeof(RegTerm) == 16, "term layout");

struct RegLaunch {
  int32_t C, dim, hess, CC;
  int32_t bound[3];
  int32_t radius;
  int64_t size[3], nvox;
  int64_t isN, isC, is[3];
  int64_t osN, osC, os[3];
  int64_t wsN, wsC, ws[3];
  int64_t hsN, hsC, hs[3];
  const void* inp;
  void* out;
  const void* wgt;
  const void* hes;
  int32_t first[kRegMaxChan + 1];  // terms of output channel c: [first[c], first[c + 1])
  RegTerm t[kRegMaxTerms];
};
static_assert(sizeof(RegLaunch) <= 32764, "regulariser argument above the kernel-parameter limit");

// Index of the (i, j) entry, i < j, of a symmetric C x C matrix stored as its
// diagonal then the upper triangle row by row.
__device__ __forceinline__ int sym_index(int i, int j, int C) { return C + i * C - i * (i + 1) / 2 + (j - i - 1); }

template <class S>
__global__ void __launch_bounds__(256) regulariser_kernel(const __grid_constant__ RegLaunch L) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < L.nvox; i += step) {
    int64_t r = i;
    int sub[3] = {0, 0, 0};
    for (int a = L.dim - 1; a >= 0; --a) {
      sub[a] = static_cast<int>(r % L.size[a]);
      r /= L.size[a];
    }
    const int64_t n = r;
    // element offsets (input, weights) and signs of the +-1 / +-2 neighbours
    int64_t di[3][5], dw[3][5];
    int sg[3][5];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int k = 0; k < 5; ++k) { di[a][k] = 0; dw[a][k] = 0; sg[a][k] = 1; }
    for (int a = 0; a < L.dim; ++a) {
      const int nn = static_cast<int>(L.size[a]);
      for (int k = -L.radius; k <= L.radius; ++k) {
        if (k == 0) continue;
        const int j = sub[a] + k;
        const int s = ppk::bound_sign<int>(L.bound[a], j, nn);
        const int idx = s ? ppk::bound_index<int>(L.bound[a], j, nn) : sub[a];
        di[a][k + 2] = static_cast<int64_t>(idx - sub[a]) * L.is[a];
        dw[a][k + 2] = static_cast<int64_t>(idx - sub[a]) * L.ws[a];
        sg[a][k + 2] = s;
      }
    }
    int64_t io = n * L.isN, oo = n * L.osN, wo = n * L.wsN, ho = n * L.hsN;
    for (int a = 0; a < L.dim; ++a) {
      io += sub[a] * L.is[a];
      oo += sub[a] * L.os[a];
      wo += sub[a] * L.ws[a];
      ho += sub[a] * L.hs[a];
    }
    const S* inp = static_cast<const S*>(L.inp) + io;
    const S* wgt = L.wgt ? static_cast<const S*>(L.wgt) + wo : nullptr;
    const S* hes = L.hes ? static_cast<const S*>(L.hes) + ho : nullptr;
    S* out = static_cast<S*>(L.out) + oo;
    for (int c = 0; c < L.C; ++c) {
      const S cen = inp[c * L.isC];
      const S wc = wgt ? wgt[c * L.wsC] : S(0);
      double acc = 0.0;
      for (int e = L.first[c]; e < L.first[c + 1]; ++e) {
        const RegTerm& T = L.t[e];
        if (T.kind == RK_CENTRE) {
          acc += T.coef * static_cast<double>(inp[T.src * L.isC]);
          continue;
        }
        if (T.kind == RK_WCENTRE) {
          acc += T.coef * static_cast<double>(wc) * static_cast<double>(cen);
          continue;
        }
        const int k0 = T.o[0] + 2, k1 = T.o[1] + 2, k2 = T.o[2] + 2;
        const int s = sg[0][k0] * sg[1][k1] * sg[2][k2];
        const int64_t off = di[0][k0] + di[1][k1] + di[2][k2];
        const S v = s ? static_cast<S>(s) * inp[T.src * L.isC + off] : S(0);  // sign 0: outside, no read
        if (T.kind == RK_RAW) {
          acc += T.coef * static_cast<double>(v);
          continue;
        }
        const S d = v - cen;
        if (T.kind == RK_DIFF) {
          acc += T.coef * static_cast<double>(d);
        } else {
          const int64_t woff = dw[0][k0] + dw[1][k1] + dw[2][k2];
          const S wn = s ? static_cast<S>(s) * wgt[c * L.wsC + woff] : S(0);
          acc += T.coef * static_cast<double>(static_cast<S>(wc + wn)) * static_cast<double>(d);
        }
      }
      if (hes) {
        const int C = L.C;
        const double u = static_cast<double>(cen);
        switch (L.hess) {
          case RH_EYE: acc += static_cast<double>(hes[0]) * u; break;
          case RH_DIAG: acc += static_cast<double>(hes[c * L.hsC]) * u; break;
          case RH_ESTATICS:  // [[diag(d), b], [b^T, r]] stored as d_0..d_{C-2}, r, b_0..b_{C-2}
            if (c < C - 1) {
              acc += static_cast<double>(hes[c * L.hsC]) * u +
                     static_cast<double>(hes[(C + c) * L.hsC]) * static_cast<double>(inp[(C - 1) * L.isC]);
            } else {
              acc += static_cast<double>(hes[(C - 1) * L.hsC]) * u;
              for (int k = 0; k < C - 1; ++k)
                acc += static_cast<double>(hes[(C + k) * L.hsC]) * static_cast<double>(inp[k * L.isC]);
            }
            break;
          case RH_SYM:
            acc += static_cast<double>(hes[c * L.hsC]) * u;
            for (int k = 0; k < C; ++k) {
              if (k == c) continue;
              const int h = k < c ? sym_index(k, c, C) : sym_index(c, k, C);
              acc += static_cast<double>(hes[h * L.hsC]) * static_cast<double>(inp[k * L.isC]);
            }
            break;
          default: break;
        }
      }
      out[c * L.osC] = static_cast<S>(acc);
    }
  }
}

// ---- host: the term tables -------------------------------------------------

struct TableBuilder {
  RegLaunch& L;
  int n = 0;
  bool full = false;
  explicit TableBuilder(RegLaunch& l) : L(l) {}
  void add(int kind, int src, int o0, int o1, int o2, double coef) {
    if (coef == 0.0) return;
    if (n >= kRegMaxTerms) { full = true; return; }
    RegTerm& t = L.t[n++];
    std::memset(&t, 0, sizeof(t));
    t.o[0] = static_cast<int8_t>(o0);
    t.o[1] = static_cast<int8_t>(o1);
    t.o[2] = static_cast<int8_t>(o2);
    t.src = static_cast<int8_t>(src);
    t.kind = static_cast<int8_t>(kind);
    t.coef = coef;
  }
  // +-s steps along axis a
  void pair(int kind, int src, int a, int s, double coef) {
    int o[3] = {0, 0, 0};
    o[a] = -s;
    add(kind, src, o[0], o[1], o[2], coef);
    o[a] = s;
    add(kind, src, o[0], o[1], o[2], coef);
  }
  // the four diagonal neighbours of axes (i, j)
  void diagonals(int src, int i, int j, double coef) {
    for (int si = -1; si <= 1; si += 2)
      for (int sj = -1; sj <= 1; sj += 2) {
        int o[3] = {0, 0, 0};
        o[i] = si;
        o[j] = sj;
        add(RK_DIFF, src, o[0], o[1], o[2], coef);
      }
  }
};

// 1 / voxel_size^2 per axis, zero beyond the field's dimension
void voxel_factors(const double* vs, int dim, double (&vx)[3]) {
  for (int a = 0; a < 3; ++a) vx[a] = a < dim ? 1.0 / (vs[a] * vs[a]) : 0.0;
}

int set_layout(RegLaunch& L, const pp_tensor* t, int chan_axis, int first_spatial, int64_t& sN, int64_t& sC,
               int64_t (&s)[3]) {
  sN = t->strides[0];
  sC = chan_axis >= 0 ? t->strides[chan_axis] : 0;
  for (int a = 0; a < 3; ++a) s[a] = a < L.dim ? t->strides[first_spatial + a] : 0;
  return PP_OK;
}

int check_float(const pp_tensor* t, int dtype, const char* name) {
  int rc = ppc::check_tensor(t, name);
  if (rc) return rc;
  if (t->dtype != dtype) return ppc::fail(PP_ERR_DTYPE, "(): %s must have the input's dtype", name);
  return PP_OK;
}

int launch(RegLaunch& L, int dtype, cudaStream_t st) {
  if (L.nvox == 0) return PP_OK;
  const int64_t want = (L.nvox + 255) / 256;
  const unsigned nb = static_cast<unsigned>(want < 148 * 16 ? want : 148 * 16);
  if (dtype == PP_FLOAT32)
    regulariser_kernel<float><<<nb, 256, 0, st>>>(L);
  else
    regulariser_kernel<double><<<nb, 256, 0, st>>>(L);
  ppc::count_launch();
  return ppc::cuda_check(cudaGetLastError(), "regulariser launch");
}

// out must not share memory with the tensors the stencil reads
bool overlaps(const pp_tensor* a, const pp_tensor* b) {
  if (!a || !b || !a->data || !b->data) return false;
  const size_t es = ppc::dtype_size(a->dtype);
  const char* a0 = static_cast<const char*>(a->data);
  const char* b0 = static_cast<const char*>(b->data);
  const char* a1 = a0 + (ppc::max_offset(a, 0) + 1) * es;
  const char* b1 = b0 + (ppc::max_offset(b, 0) + 1) * ppc::dtype_size(b->dtype);
  return a0 < b1 && b0 < a1;
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
  static thread_local RegLaunch L;
  std::memset(&L, 0, offsetof(RegLaunch, t));
  L.dim = input->ndim - 2;
  const int64_t C64 = input->sizes[1];
  if (C64 < 1 || C64 > kRegMaxChan) return ppc::fail(PP_ERR_UNSUPPORTED, "(): 1 to %d channels", kRegMaxChan);
  L.C = static_cast<int>(C64);
  if ((rc = check_float(out, input->dtype, "output"))) return rc;
  for (int i = 0; i < input->ndim; ++i)
    if (out->ndim != input->ndim || out->sizes[i] != input->sizes[i])
      return ppc::fail(PP_ERR_ARG, "(): output must have the input's shape");
  if (overlaps(out, input) || overlaps(out, weight) || overlaps(out, hessian))
    return ppc::fail(PP_ERR_ARG, "(): output must not overlap the inputs");
  bool has_b = false;
  for (int c = 0; c < L.C; ++c) has_b = has_b || bending[c] != 0.0;
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
    const int64_t CC = hessian->sizes[1], C = L.C;
    L.CC = static_cast<int>(CC);
    L.hess = CC == 1 ? RH_EYE : CC == C ? RH_DIAG : CC == 2 * C - 1 ? RH_ESTATICS : CC == C * (C + 1) / 2 ? RH_SYM : -1;
    if (L.hess < 0) return ppc::fail(PP_ERR_ARG, "(): hessian channels must be 1, C, 2C-1 or C(C+1)/2");
  }
  for (int a = 0; a < 3; ++a) {
    L.bound[a] = bound[a];
    L.size[a] = a < L.dim ? input->sizes[2 + a] : 1;
  }
  L.nvox = input->sizes[0] * L.size[0] * L.size[1] * L.size[2];
  set_layout(L, input, 1, 2, L.isN, L.isC, L.is);
  set_layout(L, out, 1, 2, L.osN, L.osC, L.os);
  if (weight) set_layout(L, weight, 1, 2, L.wsN, L.wsC, L.ws);
  if (hessian) set_layout(L, hessian, 1, 2, L.hsN, L.hsC, L.hs);
  L.inp = input->data;
  L.out = out->data;
  L.wgt = weight ? weight->data : nullptr;
  L.hes = hessian ? hessian->data : nullptr;
  L.radius = has_b ? 2 : 1;
  double vx[3];
  voxel_factors(voxel_size, L.dim, vx);
  const double svx = vx[0] + vx[1] + vx[2];
  TableBuilder tb(L);
  for (int c = 0; c < L.C; ++c) {
    L.first[c] = tb.n;
    const double a = absolute[c], m = membrane[c], b = bending[c];
    if (weight) {  // vel2mom*_rls_membrane / _rls_absolute
      tb.add(RK_WCENTRE, c, 0, 0, 0, a);
      for (int ax = 0; ax < L.dim; ++ax) tb.pair(RK_WDIFF, c, ax, 1, m * 0.5 * -vx[ax]);
      continue;
    }
    tb.add(RK_CENTRE, c, 0, 0, 0, a);  // vel2mom*_absolute / _membrane / _bending
    for (int ax = 0; ax < L.dim; ++ax) tb.pair(RK_DIFF, c, ax, 1, m * -vx[ax] + b * (-4.0 * vx[ax] * svx));
    if (b != 0.0) {
      for (int ax = 0; ax < L.dim; ++ax) tb.pair(RK_DIFF, c, ax, 2, b * vx[ax] * vx[ax]);
      for (int i = 0; i < L.dim; ++i)
        for (int j = i + 1; j < L.dim; ++j) tb.diagonals(c, i, j, b * 2.0 * vx[i] * vx[j]);
    }
  }
  L.first[L.C] = tb.n;
  if (tb.full) return ppc::fail(PP_ERR_UNSUPPORTED, "(): too many stencil terms (fewer channels)");
  return launch(L, input->dtype, static_cast<cudaStream_t>(stream));
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
  static thread_local RegLaunch L;
  std::memset(&L, 0, offsetof(RegLaunch, t));
  L.dim = input->ndim - 2;
  L.C = L.dim;
  const int D = L.dim, last = input->ndim - 1;
  if ((rc = check_float(out, input->dtype, "output"))) return rc;
  for (int i = 0; i < input->ndim; ++i)
    if (out->ndim != input->ndim || out->sizes[i] != input->sizes[i])
      return ppc::fail(PP_ERR_ARG, "(): output must have the input's shape");
  if (overlaps(out, input) || overlaps(out, weight) || overlaps(out, hessian))
    return ppc::fail(PP_ERR_ARG, "(): output must not overlap the inputs");
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
    L.CC = static_cast<int>(DD);
    L.hess = DD == 1 ? RH_EYE : DD == D ? RH_DIAG : DD == D * (D + 1) / 2 ? RH_SYM : -1;
    if (L.hess < 0) return ppc::fail(PP_ERR_ARG, "(): hessian components must be 1, D or D(D+1)/2");
  }
  for (int a = 0; a < 3; ++a) {
    L.bound[a] = bound[a];
    L.size[a] = a < D ? input->sizes[1 + a] : 1;
  }
  L.nvox = input->sizes[0] * L.size[0] * L.size[1] * L.size[2];
  set_layout(L, input, last, 1, L.isN, L.isC, L.is);
  set_layout(L, out, last, 1, L.osN, L.osC, L.os);
  if (weight) set_layout(L, weight, -1, 1, L.wsN, L.wsC, L.ws);
  if (hessian) set_layout(L, hessian, last, 1, L.hsN, L.hsC, L.hs);
  L.inp = input->data;
  L.out = out->data;
  L.wgt = weight ? weight->data : nullptr;
  L.hes = hessian ? hessian->data : nullptr;
  L.radius = bending != 0.0 ? 2 : 1;
  double vx[3];
  voxel_factors(voxel_size, D, vx);
  const double svx = vx[0] + vx[1] + vx[2];
  const double lam0 = absolute, lam1 = membrane, lam2 = bending, mu = shear, lam = div;
  double w1[3];
  for (int a = 0; a < 3; ++a) w1[a] = lam2 * (-4.0 * vx[a] * svx) - lam1 * vx[a];
  const double wc2 = 0.25 * mu + 0.25 * lam;
  TableBuilder tb(L);
  for (int d = 0; d < D; ++d) {
    L.first[d] = tb.n;
    const double s = 1.0 / vx[d];  // component d in the units of its axis
    if (weight) {  // vel2mom*_rls_membrane / _rls_absolute
      tb.add(RK_WCENTRE, d, 0, 0, 0, lam0 * s);
      for (int ax = 0; ax < D; ++ax) tb.pair(RK_WDIFF, d, ax, 1, 0.5 * w1[ax] * s);
      continue;
    }
    tb.add(RK_CENTRE, d, 0, 0, 0, lam0 * s);
    for (int ax = 0; ax < D; ++ax) {
      const double lame = ax == d ? -2.0 * mu - lam : -mu * vx[ax] / vx[d];
      tb.pair(RK_DIFF, d, ax, 1, w1[ax] * s + lame);
    }
    if (lam2 != 0.0) {
      for (int ax = 0; ax < D; ++ax) tb.pair(RK_DIFF, d, ax, 2, lam2 * vx[ax] * vx[ax] * s);
      for (int i = 0; i < D; ++i)
        for (int j = i + 1; j < D; ++j) tb.diagonals(d, i, j, lam2 * 2.0 * vx[i] * vx[j] * s);
    }
    if (wc2 != 0.0) {  // the Lame coupling to the other components
      for (int e = 0; e < D; ++e) {
        if (e == d) continue;
        for (int sd = -1; sd <= 1; sd += 2)
          for (int se = -1; se <= 1; se += 2) {
            int o[3] = {0, 0, 0};
            o[d] = sd;
            o[e] = se;
            tb.add(RK_RAW, e, o[0], o[1], o[2], -wc2 * sd * se);
          }
      }
    }
  }
  L.first[D] = tb.n;
  return launch(L, input->dtype, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
