// One scaling-and-squaring step of a 3-D float32 displacement field at
// linear order: out = u + pull(u, id + u).
//
// nitorch's exp (nitorch/spatial/_svf.py:85-94, _pull_vel :323-362)
// materialises id + u and pulls every component at it, linear, dft by
// default.  The general pull kernel (flags F_IDGRID | F_ADDSELF) does the
// same for any order and dimension; this kernel is its 3-D linear float32
// case: a thread per voxel reads the voxel's three components once (they
// are the sampling offset and the added identity term), then the eight
// corners of the cell, the separable partial sums x innermost as the
// general kernel forms them.  A corner's boundary index and sign are only
// computed on axes where the cell leaves the volume; 32-bit offsets.
// Points outside the field of view without extrapolation keep the identity
// term alone, as there.
#include <cstdint>

#include "../../include/nitorch_b200.h"
#include "pp_capi_internal.cuh"
#include "pp_kernels.cuh"

namespace {

struct ComposeArgs {
  int32_t size[3], bound[3];
  int32_t extrapolate, pad;
  int64_t nvox;
  int64_t fN, oN;      // batch strides
  int32_t fs[3], fC;   // field strides (elements): spatial, component
  int32_t os[3], oC;   // output strides
  const float* u;
  float* out;
};

// UV4 / OV4: the field / the output is the first three slots of a four-slot
// buffer (strides (., 4YZ, 4Z, 4, 1), 16-byte aligned): one 16-byte access
// per voxel or corner instead of three.
template <bool UV4>
__device__ __forceinline__ void load3(const float* p, int fC, float (&v)[3]) {
  if constexpr (UV4) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z;
  } else {
    v[0] = __ldg(p); v[1] = __ldg(p + fC); v[2] = __ldg(p + 2 * fC);
  }
}

template <bool UV4, bool OV4>
__global__ void __launch_bounds__(256, UV4 ? 4 : 5) svf_compose_lin3(const ComposeArgs A) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < A.nvox; i += step) {
    int sub[3];
    int64_t n;
    {
      int64_t r = i;
      sub[2] = static_cast<int>(r % A.size[2]); r /= A.size[2];
      sub[1] = static_cast<int>(r % A.size[1]); r /= A.size[1];
      sub[0] = static_cast<int>(r % A.size[0]);
      n = r / A.size[0];
    }
    const float* un = A.u + n * A.fN;
    const int base = sub[0] * A.fs[0] + sub[1] * A.fs[1] + sub[2] * A.fs[2];
    float self[3], x[3];
    load3<UV4>(un + base, A.fC, self);
#pragma unroll
    for (int d = 0; d < 3; ++d) x[d] = static_cast<float>(sub[d]) + self[d];
    float* o = A.out + n * A.oN + sub[0] * A.os[0] + sub[1] * A.os[1] + sub[2] * A.os[2];
    const float tol = (A.extrapolate & 2) ? 0.55f : 0.05f;
    bool inb = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) inb = inb && ppk::in_fov<float>(x[d], A.size[d], tol);
    float res[3];
    if (!((A.extrapolate & 1) || inb)) {  // outside the field of view: the identity term alone
#pragma unroll
      for (int d = 0; d < 3; ++d) res[d] = self[d];
    } else {
      // per axis: the two nodes' offsets and weights (boundary sign folded in)
      int off[3][2];
      float w[3][2];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float xc = fminf(fmaxf(x[d], -1073741824.f), 1073741824.f);
        const float f = floorf(xc);
        const int i0 = static_cast<int>(f);
        const float t = xc - f;
        const int nn = A.size[d];
        if (i0 >= 0 && i0 + 1 < nn) {
          off[d][0] = i0 * A.fs[d];
          off[d][1] = off[d][0] + A.fs[d];
          w[d][0] = 1.f - t;
          w[d][1] = t;
        } else {
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            const int s = ppk::bound_sign<int>(A.bound[d], i0 + k, nn);
            const int idx = s ? ppk::bound_index<int>(A.bound[d], i0 + k, nn) : 0;
            off[d][k] = idx * A.fs[d];
            w[d][k] = static_cast<float>(s) * (k ? t : 1.f - t);
          }
        }
      }
      // separable partial sums, x innermost, the three components together
      float acc[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        float accy[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int oyz = off[1][j] + off[2][k];
          float c0[3], c1[3];
          load3<UV4>(un + off[0][0] + oyz, A.fC, c0);
          load3<UV4>(un + off[0][1] + oyz, A.fC, c1);
#pragma unroll
          for (int c = 0; c < 3; ++c) accy[c] = fmaf(w[1][j], fmaf(w[0][1], c1[c], w[0][0] * c0[c]), accy[c]);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] = fmaf(w[2][k], accy[c], acc[c]);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) res[c] = acc[c] + self[c];
    }
    if constexpr (OV4) {
      *reinterpret_cast<float4*>(o) = make_float4(res[0], res[1], res[2], 0.f);
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) o[c * A.oC] = res[c];
    }
  }
}

// Its adjoint with respect to u, for g = d loss / d out: the push of g
// through the cell's eight corners, the grid gradient sum_c g_c grad(u_c),
// and the identity term g, into a four-slot channel-interleaved float
// accumulator (acc[v * 4 + c]) with one vector reduction per corner.  A
// thread per voxel, consecutive lanes consecutive voxels along the last
// axis: for a smooth field a voxel's upper-z corner is often the next
// lane's lower-z corner, so the two contributions are added in registers
// (one shuffle) and one reduction is saved.  Both lanes test the same
// equality on valid addresses, so every contribution is added once.
struct ComposeBwdArgs {
  int32_t size[3], bound[3];
  int32_t extrapolate, pad;
  int64_t nvox;
  int64_t fN, gN, aN;
  int32_t fs[3], fC;   // field strides
  int32_t gs[3], gC;   // gradient strides
  int32_t as[3], pad2; // accumulator strides (floats): Y*Z*4, Z*4, 4
  const float* u;
  const float* g;
  float* acc;
};

template <bool UV4>
__global__ void __launch_bounds__(256, 5) svf_compose_backward_lin3(const ComposeBwdArgs A) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool live = i < A.nvox;
  int sub[3] = {0, 0, 0};
  int64_t n = 0;
  if (live) {
    int64_t r = i;
    sub[2] = static_cast<int>(r % A.size[2]); r /= A.size[2];
    sub[1] = static_cast<int>(r % A.size[1]); r /= A.size[1];
    sub[0] = static_cast<int>(r % A.size[0]);
    n = r / A.size[0];
  }
  const float* un = A.u + n * A.fN;
  float gv[3] = {0.f, 0.f, 0.f}, x[3] = {0.f, 0.f, 0.f};
  bool active = false;
  if (live) {
    const int fb = sub[0] * A.fs[0] + sub[1] * A.fs[1] + sub[2] * A.fs[2];
    const float* gp = A.g + n * A.gN + sub[0] * A.gs[0] + sub[1] * A.gs[1] + sub[2] * A.gs[2];
    float uu[3];
    load3<UV4>(un + fb, A.fC, uu);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      x[d] = static_cast<float>(sub[d]) + uu[d];
      gv[d] = __ldg(gp + d * A.gC);
    }
    const float tol = (A.extrapolate & 2) ? 0.55f : 0.05f;
    bool inb = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) inb = inb && ppk::in_fov<float>(x[d], A.size[d], tol);
    active = (A.extrapolate & 1) || inb;
  }
  float* acc_n = A.acc + n * A.aN;
  // per axis: the two nodes (field offsets, accumulator offsets, -1: none),
  // weights and derivative weights with the boundary sign folded in
  int fo[3][2], ao[3][2];
  float w[3][2], dw[3][2];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float xc = fminf(fmaxf(x[d], -1073741824.f), 1073741824.f);
    const float f = floorf(xc);
    const int i0 = static_cast<int>(f);
    const float t = xc - f;
    const int nn = A.size[d];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      int s = 1, idx = i0 + k;
      if (!(i0 >= 0 && i0 + 1 < nn)) {
        s = ppk::bound_sign<int>(A.bound[d], i0 + k, nn);
        idx = s ? ppk::bound_index<int>(A.bound[d], i0 + k, nn) : 0;
      }
      const bool ok = active && s != 0;
      fo[d][k] = idx * A.fs[d];
      ao[d][k] = ok ? idx * A.as[d] : -1;
      w[d][k] = ok ? static_cast<float>(s) * (k ? t : 1.f - t) : 0.f;
      dw[d][k] = ok ? static_cast<float>(s) * (k ? 1.f : -1.f) : 0.f;
    }
  }
  // grid gradient: og_d = sum over corners of (derivative along d of the
  // corner weight) * <g, u(corner)>
  float og0 = 0.f, og1 = 0.f, og2 = 0.f;
  if (active) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        float sx = 0.f, dx = 0.f;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          if (ao[0][q] < 0 || ao[1][j] < 0 || ao[2][k] < 0) continue;  // a node outside: no tap
          float cu[3];
          load3<UV4>(un + fo[0][q] + fo[1][j] + fo[2][k], A.fC, cu);
          const float dot = gv[0] * cu[0] + gv[1] * cu[1] + gv[2] * cu[2];
          sx = fmaf(w[0][q], dot, sx);
          dx = fmaf(dw[0][q], dot, dx);
        }
        og0 = fmaf(w[1][j] * w[2][k], dx, og0);
        og1 = fmaf(dw[1][j] * w[2][k], sx, og1);
        og2 = fmaf(w[1][j] * dw[2][k], sx, og2);
      }
    }
  }
  // the push of g, corner pairs (k = 0, 1) merged with the neighbouring lanes
#pragma unroll
  for (int q = 0; q < 2; ++q) {
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const bool xy = ao[0][q] >= 0 && ao[1][j] >= 0;
      const int a0 = xy && ao[2][0] >= 0 ? ao[0][q] + ao[1][j] + ao[2][0] : -1;
      const int a1 = xy && ao[2][1] >= 0 ? ao[0][q] + ao[1][j] + ao[2][1] : -1;
      const float wxy = w[0][q] * w[1][j];
      float v0[4] = {wxy * w[2][0] * gv[0], wxy * w[2][0] * gv[1], wxy * w[2][0] * gv[2], 0.f};
      const float c1 = wxy * w[2][1];
      // batch items differ: the neighbour's address is compared within one item
      const int64_t nn_prev = __shfl_up_sync(0xffffffffu, n, 1);
      const int64_t nn_next = __shfl_down_sync(0xffffffffu, n, 1);
      const int prev_a1 = __shfl_up_sync(0xffffffffu, a1, 1);
      const int next_a0 = __shfl_down_sync(0xffffffffu, a0, 1);
      const float p0 = __shfl_up_sync(0xffffffffu, c1 * gv[0], 1);
      const float p1 = __shfl_up_sync(0xffffffffu, c1 * gv[1], 1);
      const float p2 = __shfl_up_sync(0xffffffffu, c1 * gv[2], 1);
      const bool take_prev = lane > 0 && a0 >= 0 && prev_a1 == a0 && nn_prev == n;
      const bool given_next = lane < 31 && a1 >= 0 && next_a0 == a1 && nn_next == n;
      if (take_prev) {
        v0[0] += p0;
        v0[1] += p1;
        v0[2] += p2;
      }
      if (a0 >= 0) ppk::red_vec<4>(acc_n + a0, v0);
      if (a1 >= 0 && !given_next) {
        const float v1[4] = {c1 * gv[0], c1 * gv[1], c1 * gv[2], 0.f};
        ppk::red_vec<4>(acc_n + a1, v1);
      }
    }
  }
  // the identity term and the grid gradient at the voxel itself
  if (live) {
    const float vs[4] = {gv[0] + og0, gv[1] + og1, gv[2] + og2, 0.f};
    ppk::red_vec<4>(acc_n + sub[0] * A.as[0] + sub[1] * A.as[1] + sub[2] * A.as[2], vs);
  }
}

bool fits_int(int64_t v) { return v < (int64_t(1) << 31) - 1; }

// The first three slots of a 16-byte aligned four-slot (N, X, Y, Z, 4) buffer.
bool padded4(const pp_tensor* t) {
  if (t->ndim != 5 || t->sizes[4] != 3 || reinterpret_cast<uintptr_t>(t->data) % 16 != 0) return false;
  const int64_t want[5] = {t->strides[0], t->sizes[2] * t->sizes[3] * 4, t->sizes[3] * 4, 4, 1};
  if (t->strides[0] % 4 != 0) return false;
  for (int i = 1; i < 5; ++i)
    if (t->sizes[i] > 1 && t->strides[i] != want[i]) return false;
  return true;
}

}  // namespace

namespace ppc {

// The 3-D linear float32 self-composition above, or PP_ERR_UNSUPPORTED when
// the call is not that case (the caller then runs the general kernel).
int svf_compose_linear3(const pp_tensor* disp, const pp_tensor* out, const int32_t bound[3], int32_t extrapolate,
                        cudaStream_t st) {
  if (disp->ndim != 5 || disp->sizes[4] != 3 || disp->dtype != PP_FLOAT32 || out->dtype != PP_FLOAT32)
    return PP_ERR_UNSUPPORTED;
  const int64_t per_item_f = max_offset(disp, 1), per_item_o = max_offset(out, 1);
  if (!fits_int(per_item_f + 1) || !fits_int(per_item_o + 1)) return PP_ERR_UNSUPPORTED;
  for (int d = 1; d < 4; ++d)
    if (!fits_int(disp->sizes[d])) return PP_ERR_UNSUPPORTED;
  ComposeArgs A;
  for (int d = 0; d < 3; ++d) {
    A.size[d] = static_cast<int32_t>(disp->sizes[1 + d]);
    A.bound[d] = bound[d];
    A.fs[d] = static_cast<int32_t>(disp->strides[1 + d]);
    A.os[d] = static_cast<int32_t>(out->strides[1 + d]);
  }
  A.fC = static_cast<int32_t>(disp->strides[4]);
  A.oC = static_cast<int32_t>(out->strides[4]);
  A.fN = disp->strides[0];
  A.oN = out->strides[0];
  A.extrapolate = extrapolate;
  A.pad = 0;
  A.nvox = disp->sizes[0] * disp->sizes[1] * disp->sizes[2] * disp->sizes[3];
  A.u = static_cast<const float*>(disp->data);
  A.out = static_cast<float*>(out->data);
  if (A.nvox == 0) return PP_OK;
  const int64_t want = (A.nvox + 255) / 256;
  const unsigned nb = static_cast<unsigned>(want < 148 * 32 ? want : 148 * 32);
  ppk::note_kernel("svf_compose_lin3", ppk::K_PULL, 1, 3);
  const bool uv4 = padded4(disp), ov4 = padded4(out);
  if (uv4 && ov4) svf_compose_lin3<true, true><<<nb, 256, 0, st>>>(A);
  else if (uv4) svf_compose_lin3<true, false><<<nb, 256, 0, st>>>(A);
  else if (ov4) svf_compose_lin3<false, true><<<nb, 256, 0, st>>>(A);
  else svf_compose_lin3<false, false><<<nb, 256, 0, st>>>(A);
  count_launch();
  return cuda_check(cudaGetLastError(), "svf compose launch");
}

// The 3-D linear float32 self-composition backward into a four-slot
// channel-interleaved accumulator (zeroed by the caller, V * 4 floats per
// batch item, the last axis fastest), or PP_ERR_UNSUPPORTED (nothing
// launched) for any other field.
int svf_compose_backward_linear3(const pp_tensor* grad, const pp_tensor* disp, float* acc, const int32_t bound[3],
                                 int32_t extrapolate, cudaStream_t st) {
  if (disp->ndim != 5 || disp->sizes[4] != 3 || disp->dtype != PP_FLOAT32 || grad->dtype != PP_FLOAT32)
    return PP_ERR_UNSUPPORTED;
  const int64_t V = disp->sizes[1] * disp->sizes[2] * disp->sizes[3];
  if (!fits_int(max_offset(disp, 1) + 1) || !fits_int(max_offset(grad, 1) + 1) || !fits_int(V * 4))
    return PP_ERR_UNSUPPORTED;
  ComposeBwdArgs A;
  for (int d = 0; d < 3; ++d) {
    A.size[d] = static_cast<int32_t>(disp->sizes[1 + d]);
    A.bound[d] = bound[d];
    A.fs[d] = static_cast<int32_t>(disp->strides[1 + d]);
    A.gs[d] = static_cast<int32_t>(grad->strides[1 + d]);
  }
  A.as[2] = 4;
  A.as[1] = static_cast<int32_t>(disp->sizes[3] * 4);
  A.as[0] = static_cast<int32_t>(disp->sizes[2] * disp->sizes[3] * 4);
  A.fC = static_cast<int32_t>(disp->strides[4]);
  A.gC = static_cast<int32_t>(grad->strides[4]);
  A.fN = disp->strides[0];
  A.gN = grad->strides[0];
  A.aN = V * 4;
  A.extrapolate = extrapolate;
  A.pad = A.pad2 = 0;
  A.nvox = disp->sizes[0] * V;
  A.u = static_cast<const float*>(disp->data);
  A.g = static_cast<const float*>(grad->data);
  A.acc = acc;
  if (A.nvox == 0) return PP_OK;
  const int64_t nb = (A.nvox + 255) / 256;  // a thread per voxel: whole warps of consecutive voxels
  if (nb > 0x7fffffffLL) return PP_ERR_UNSUPPORTED;
  ppk::note_kernel("svf_compose_backward_lin3", ppk::K_PUSHGRAD, 1, 3);
  if (padded4(disp))
    svf_compose_backward_lin3<true><<<static_cast<unsigned>(nb), 256, 0, st>>>(A);
  else
    svf_compose_backward_lin3<false><<<static_cast<unsigned>(nb), 256, 0, st>>>(A);
  count_launch();
  return cuda_check(cudaGetLastError(), "svf compose backward launch");
}

}  // namespace ppc
