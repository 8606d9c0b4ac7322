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

__global__ void __launch_bounds__(256, 4) svf_compose_lin3(const ComposeArgs A) {
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
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      self[d] = __ldg(un + base + d * A.fC);
      x[d] = static_cast<float>(sub[d]) + self[d];
    }
    float* o = A.out + n * A.oN + sub[0] * A.os[0] + sub[1] * A.os[1] + sub[2] * A.os[2];
    const float tol = (A.extrapolate & 2) ? 0.55f : 0.05f;
    bool inb = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) inb = inb && ppk::in_fov<float>(x[d], A.size[d], tol);
    if (!((A.extrapolate & 1) || inb)) {  // outside the field of view: the identity term alone
#pragma unroll
      for (int d = 0; d < 3; ++d) o[d * A.oC] = self[d];
      continue;
    }
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
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float* uc = un + c * A.fC;
      float acc = 0.f;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        float accy = 0.f;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int oyz = off[1][j] + off[2][k];
          const float accx = fmaf(w[0][1], __ldg(uc + off[0][1] + oyz), w[0][0] * __ldg(uc + off[0][0] + oyz));
          accy = fmaf(w[1][j], accx, accy);
        }
        acc = fmaf(w[2][k], accy, acc);
      }
      o[c * A.oC] = acc + self[c];
    }
  }
}

bool fits_int(int64_t v) { return v < (int64_t(1) << 31) - 1; }

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
  svf_compose_lin3<<<nb, 256, 0, st>>>(A);
  count_launch();
  return cuda_check(cudaGetLastError(), "svf compose launch");
}

}  // namespace ppc
