// Jacobians of transformation / displacement fields.
//
// nitorch computes grid_jacobian (nitorch/spatial/_grid.py:917-969) as
// central finite differences of the displacement (diff, side 'c', order 1:
// nitorch/spatial/_finite_differences.py:32-222) with a boundary condition
// for the values beyond each end, then adds the identity; grid_jacdet
// (:972-1013) takes torch's determinant of the result.  Here one kernel
// reads each voxel's 2D neighbours and writes the D x D matrix and / or its
// determinant (no (N, *spatial, D, D) intermediate when only the
// determinant is wanted); its adjoint scatters the gradient back to the
// field.  With sampled coordinates the Jacobian comes from grid_grad
// instead, and pp_jacobian_det / pp_jacobian_det_backward give the
// determinant of any (..., D, D) matrices.
#include <cstdint>

#include "../../include/nitorch_b200.h"
#include "pp_capi_internal.cuh"
#include "pp_kernels.cuh"

namespace {

struct FieldArgs {
  int64_t N, size[3];
  int64_t fsN, fs[3], fsC;   // field (N, *spatial, D)
  int64_t jsN, js[3], jsI, jsJ;  // jacobian (N, *spatial, D, D)
  int64_t dsN, ds[3];        // determinant (N, *spatial)
  int bound;
  double inv2vs[3];          // 1 / (2 voxel_size)
  int is_grid, add_identity;
};

template <class T, int D>
__device__ __forceinline__ T det_of(const T (&J)[3][3]) {
  if constexpr (D == 1) return J[0][0];
  else if constexpr (D == 2) return J[0][0] * J[1][1] - J[0][1] * J[1][0];
  else
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

// d det / d J (the cofactor matrix)
template <class T, int D>
__device__ __forceinline__ void cofactor(const T (&J)[3][3], T (&K)[3][3]) {
  if constexpr (D == 1) {
    K[0][0] = T(1);
  } else if constexpr (D == 2) {
    K[0][0] = J[1][1]; K[0][1] = -J[1][0];
    K[1][0] = -J[0][1]; K[1][1] = J[0][0];
  } else {
    K[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    K[0][1] = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]);
    K[0][2] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    K[1][0] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]);
    K[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
    K[1][2] = -(J[0][0] * J[2][1] - J[0][1] * J[2][0]);
    K[2][0] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    K[2][1] = -(J[0][0] * J[1][2] - J[0][2] * J[1][0]);
    K[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  }
}

template <int D>
__device__ __forceinline__ void decode(const FieldArgs& a, int64_t v, int64_t& n, int64_t (&i)[3]) {
  i[0] = i[1] = i[2] = 0;
  for (int d = D - 1; d >= 0; --d) { i[d] = v % a.size[d]; v /= a.size[d]; }
  n = v;
}

// displacement component c at voxel p of item n
template <class T, int D>
__device__ __forceinline__ T disp_at(const T* f, const FieldArgs& a, int64_t n, const int64_t (&p)[3], int c) {
  int64_t off = n * a.fsN + c * a.fsC;
#pragma unroll
  for (int d = 0; d < D; ++d) off += p[d] * a.fs[d];
  T u = f[off];
  if (a.is_grid) u -= static_cast<T>(p[c]);
  return u;
}

// Jacobian at voxel i (central differences, the bound's values beyond the ends)
template <class T, int D>
__device__ __forceinline__ void jacobian_at(const T* f, const FieldArgs& a, int64_t n, const int64_t (&i)[3],
                                            T (&J)[3][3]) {
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const int64_t nj = a.size[j];
    if (nj == 1) {
      // a singleton axis: nitorch's diff returns the values themselves
#pragma unroll
      for (int c = 0; c < D; ++c) J[c][j] = disp_at<T, D>(f, a, n, i, c);
      continue;
    }
    int64_t pp[3] = {i[0], i[1], i[2]}, pm[3] = {i[0], i[1], i[2]};
    const int sp = ppk::bound_sign<int64_t>(a.bound, i[j] + 1, nj);
    const int sm = ppk::bound_sign<int64_t>(a.bound, i[j] - 1, nj);
    pp[j] = ppk::bound_index<int64_t>(a.bound, i[j] + 1, nj);
    pm[j] = ppk::bound_index<int64_t>(a.bound, i[j] - 1, nj);
    const T h = static_cast<T>(a.inv2vs[j]);
#pragma unroll
    for (int c = 0; c < D; ++c) {
      const T up = sp ? static_cast<T>(sp) * disp_at<T, D>(f, a, n, pp, c) : T(0);
      const T um = sm ? static_cast<T>(sm) * disp_at<T, D>(f, a, n, pm, c) : T(0);
      J[c][j] = (up - um) * h;
    }
  }
  if (a.add_identity) {
#pragma unroll
    for (int c = 0; c < D; ++c) J[c][c] += T(1);
  }
}

template <class T, int D>
__global__ void jacobian_fd(const T* f, FieldArgs a, T* jac, T* det, int64_t nvox) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nvox) return;
  int64_t n, i[3];
  decode<D>(a, v, n, i);
  T J[3][3];
  jacobian_at<T, D>(f, a, n, i, J);
  if (jac) {
    int64_t o = n * a.jsN;
#pragma unroll
    for (int d = 0; d < D; ++d) o += i[d] * a.js[d];
#pragma unroll
    for (int c = 0; c < D; ++c)
#pragma unroll
      for (int j = 0; j < D; ++j) jac[o + c * a.jsI + j * a.jsJ] = J[c][j];
  }
  if (det) {
    int64_t o = n * a.dsN;
#pragma unroll
    for (int d = 0; d < D; ++d) o += i[d] * a.ds[d];
    det[o] = det_of<T, D>(J);
  }
}

// Adjoint: G = grad_jac + grad_det * cofactor(J), scattered to the field
// values each entry was differenced from (atomics; gfield zero-filled).
template <class T, int D>
__global__ void jacobian_fd_backward(const T* f, FieldArgs a, const T* gjac, const T* gdet, T* gfield,
                                     int64_t gsN, int64_t gs0, int64_t gs1, int64_t gs2, int64_t gsC,
                                     int64_t nvox) {
  const int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nvox) return;
  int64_t n, i[3];
  decode<D>(a, v, n, i);
  T G[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int j = 0; j < 3; ++j) G[c][j] = T(0);
  if (gjac) {
    int64_t o = n * a.jsN;
#pragma unroll
    for (int d = 0; d < D; ++d) o += i[d] * a.js[d];
#pragma unroll
    for (int c = 0; c < D; ++c)
#pragma unroll
      for (int j = 0; j < D; ++j) G[c][j] = gjac[o + c * a.jsI + j * a.jsJ];
  }
  if (gdet) {
    int64_t o = n * a.dsN;
#pragma unroll
    for (int d = 0; d < D; ++d) o += i[d] * a.ds[d];
    const T g = gdet[o];
    T J[3][3], K[3][3];
    jacobian_at<T, D>(f, a, n, i, J);
    cofactor<T, D>(J, K);
#pragma unroll
    for (int c = 0; c < D; ++c)
#pragma unroll
      for (int j = 0; j < D; ++j) G[c][j] += g * K[c][j];
  }
  const int64_t gs[3] = {gs0, gs1, gs2};
  auto goff = [&](const int64_t (&p)[3], int c) {
    int64_t o = n * gsN + c * gsC;
#pragma unroll
    for (int d = 0; d < D; ++d) o += p[d] * gs[d];
    return o;
  };
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const int64_t nj = a.size[j];
    if (nj == 1) {
#pragma unroll
      for (int c = 0; c < D; ++c) ppk::atomic_acc(gfield + goff(i, c), G[c][j]);
      continue;
    }
    int64_t pp[3] = {i[0], i[1], i[2]}, pm[3] = {i[0], i[1], i[2]};
    const int sp = ppk::bound_sign<int64_t>(a.bound, i[j] + 1, nj);
    const int sm = ppk::bound_sign<int64_t>(a.bound, i[j] - 1, nj);
    pp[j] = ppk::bound_index<int64_t>(a.bound, i[j] + 1, nj);
    pm[j] = ppk::bound_index<int64_t>(a.bound, i[j] - 1, nj);
    const T h = static_cast<T>(a.inv2vs[j]);
#pragma unroll
    for (int c = 0; c < D; ++c) {
      if (sp) ppk::atomic_acc(gfield + goff(pp, c), static_cast<T>(sp) * G[c][j] * h);
      if (sm) ppk::atomic_acc(gfield + goff(pm, c), -static_cast<T>(sm) * G[c][j] * h);
    }
  }
}

// determinant of (M, D, D) matrices (and its adjoint)
template <class T, int D>
__global__ void det_kernel(const T* jac, int64_t jsM, int64_t jsI, int64_t jsJ, T* det, int64_t dsM, int64_t M,
                           const T* gdet, T* gjac, int64_t gsM, int64_t gsI, int64_t gsJ) {
  const int64_t m = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (m >= M) return;
  T J[3][3];
#pragma unroll
  for (int c = 0; c < D; ++c)
#pragma unroll
    for (int j = 0; j < D; ++j) J[c][j] = jac[m * jsM + c * jsI + j * jsJ];
  if (det) det[m * dsM] = det_of<T, D>(J);
  if (gjac) {
    T K[3][3];
    cofactor<T, D>(J, K);
    const T g = gdet[m * dsM];
#pragma unroll
    for (int c = 0; c < D; ++c)
#pragma unroll
      for (int j = 0; j < D; ++j) gjac[m * gsM + c * gsI + j * gsJ] = g * K[c][j];
  }
}

int field_args(const pp_tensor* field, int32_t bound, const double* voxel_size, int32_t is_grid,
               int32_t add_identity, FieldArgs& a, int& D, int64_t& nvox) {
  int rc = ppc::check_tensor(field, "field");
  if (rc) return rc;
  if (field->ndim < 3 || field->ndim > 5) return ppc::fail(PP_ERR_ARG, "(): expected a (N, *spatial, D) field, D = 1-3");
  D = field->ndim - 2;
  if (field->sizes[field->ndim - 1] != D)
    return ppc::fail(PP_ERR_ARG, "(): expected the field's last dimension to be %d", D);
  if (field->dtype != PP_FLOAT32 && field->dtype != PP_FLOAT64)
    return ppc::fail(PP_ERR_DTYPE, "(): expected a float32 or float64 field");
  if (!(bound >= 0 && bound <= 5) && bound != PP_BOUND_ZERO) return ppc::fail(PP_ERR_ARG, "(): unsupported bound code %d", bound);
  a = FieldArgs{};
  a.N = field->sizes[0];
  nvox = a.N;
  for (int d = 0; d < 3; ++d) {
    a.size[d] = d < D ? field->sizes[1 + d] : 1;
    if (a.size[d] <= 0) return ppc::fail(PP_ERR_ARG, "(): expected non-empty spatial dimensions");
    nvox *= a.size[d];
    const double vs = voxel_size ? voxel_size[d < D ? d : 0] : 1.0;
    if (!(vs != 0.0)) return ppc::fail(PP_ERR_ARG, "(): voxel sizes must be non-zero");
    a.inv2vs[d] = 1.0 / (2.0 * vs);
  }
  a.fsN = field->strides[0];
  for (int d = 0; d < 3; ++d) a.fs[d] = d < D ? field->strides[1 + d] : 0;
  a.fsC = field->strides[1 + D];
  a.bound = bound;
  a.is_grid = is_grid ? 1 : 0;
  a.add_identity = add_identity ? 1 : 0;
  return PP_OK;
}

int jac_det_layout(const pp_tensor* field, const pp_tensor* jac, const pp_tensor* det, int D, FieldArgs& a) {
  int rc;
  if (jac) {
    if ((rc = ppc::check_tensor(jac, "jacobian"))) return rc;
    if (jac->ndim != D + 3 || jac->dtype != field->dtype) return ppc::fail(PP_ERR_ARG, "(): jacobian must be (N, *spatial, D, D) of the field dtype");
    for (int i = 0; i <= D; ++i)
      if (jac->sizes[i] != field->sizes[i]) return ppc::fail(PP_ERR_ARG, "(): jacobian has the wrong shape");
    if (jac->sizes[D + 1] != D || jac->sizes[D + 2] != D) return ppc::fail(PP_ERR_ARG, "(): jacobian must end in (D, D)");
    a.jsN = jac->strides[0];
    for (int d = 0; d < 3; ++d) a.js[d] = d < D ? jac->strides[1 + d] : 0;
    a.jsI = jac->strides[1 + D];
    a.jsJ = jac->strides[2 + D];
  }
  if (det) {
    if ((rc = ppc::check_tensor(det, "determinant"))) return rc;
    if (det->ndim != D + 1 || det->dtype != field->dtype) return ppc::fail(PP_ERR_ARG, "(): determinant must be (N, *spatial) of the field dtype");
    for (int i = 0; i <= D; ++i)
      if (det->sizes[i] != field->sizes[i]) return ppc::fail(PP_ERR_ARG, "(): determinant has the wrong shape");
    a.dsN = det->strides[0];
    for (int d = 0; d < 3; ++d) a.ds[d] = d < D ? det->strides[1 + d] : 0;
  }
  return PP_OK;
}

template <class T>
cudaError_t launch_fd(int D, const T* f, const FieldArgs& a, T* jac, T* det, int64_t nvox, cudaStream_t st) {
  const unsigned nb = static_cast<unsigned>((nvox + 255) / 256);
  switch (D) {
    case 1: jacobian_fd<T, 1><<<nb, 256, 0, st>>>(f, a, jac, det, nvox); break;
    case 2: jacobian_fd<T, 2><<<nb, 256, 0, st>>>(f, a, jac, det, nvox); break;
    default: jacobian_fd<T, 3><<<nb, 256, 0, st>>>(f, a, jac, det, nvox); break;
  }
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_fd_bwd(int D, const T* f, const FieldArgs& a, const T* gj, const T* gd, T* gf,
                          const pp_tensor* g, int64_t nvox, cudaStream_t st) {
  const unsigned nb = static_cast<unsigned>((nvox + 255) / 256);
  const int64_t gsN = g->strides[0], gs0 = g->strides[1], gs1 = D > 1 ? g->strides[2] : 0,
                gs2 = D > 2 ? g->strides[3] : 0, gsC = g->strides[1 + D];
  switch (D) {
    case 1: jacobian_fd_backward<T, 1><<<nb, 256, 0, st>>>(f, a, gj, gd, gf, gsN, gs0, gs1, gs2, gsC, nvox); break;
    case 2: jacobian_fd_backward<T, 2><<<nb, 256, 0, st>>>(f, a, gj, gd, gf, gsN, gs0, gs1, gs2, gsC, nvox); break;
    default: jacobian_fd_backward<T, 3><<<nb, 256, 0, st>>>(f, a, gj, gd, gf, gsN, gs0, gs1, gs2, gsC, nvox); break;
  }
  return cudaGetLastError();
}

}  // namespace

extern "C" {

int pp_grid_jacobian(const pp_tensor* field, const pp_tensor* jac, const pp_tensor* det, int32_t bound,
                     const double* voxel_size, int32_t is_grid, int32_t add_identity, void* stream) {
  FieldArgs a;
  int D;
  int64_t nvox;
  int rc = field_args(field, bound, voxel_size, is_grid, add_identity, a, D, nvox);
  if (rc) return rc;
  if (!jac && !det) return ppc::fail(PP_ERR_ARG, "(): expected a jacobian and / or a determinant output");
  if ((rc = jac_det_layout(field, jac, det, D, a))) return rc;
  if (nvox == 0) return PP_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (field->dtype == PP_FLOAT32)
    e = launch_fd<float>(D, static_cast<const float*>(field->data), a, jac ? static_cast<float*>(jac->data) : nullptr,
                         det ? static_cast<float*>(det->data) : nullptr, nvox, st);
  else
    e = launch_fd<double>(D, static_cast<const double*>(field->data), a,
                          jac ? static_cast<double*>(jac->data) : nullptr,
                          det ? static_cast<double*>(det->data) : nullptr, nvox, st);
  ppc::count_launch();
  return ppc::cuda_check(e, "jacobian launch");
}

int pp_grid_jacobian_backward(const pp_tensor* grad_jac, const pp_tensor* grad_det, const pp_tensor* field,
                              const pp_tensor* grad_field, int32_t bound, const double* voxel_size, int32_t is_grid,
                              int32_t add_identity, void* stream) {
  FieldArgs a;
  int D;
  int64_t nvox;
  int rc = field_args(field, bound, voxel_size, is_grid, add_identity, a, D, nvox);
  if (rc) return rc;
  if (!grad_jac && !grad_det) return ppc::fail(PP_ERR_ARG, "(): expected grad_jac and / or grad_det");
  if ((rc = jac_det_layout(field, grad_jac, grad_det, D, a))) return rc;
  if ((rc = ppc::check_tensor(grad_field, "grad_field"))) return rc;
  for (int i = 0; i < field->ndim; ++i)
    if (grad_field->sizes[i] != field->sizes[i]) return ppc::fail(PP_ERR_ARG, "(): grad_field must have the field's shape");
  if (grad_field->dtype != field->dtype) return ppc::fail(PP_ERR_DTYPE, "(): grad_field must have the field dtype");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((rc = ppc::zero_fill(grad_field, st))) return rc;
  if (nvox == 0) return PP_OK;
  cudaError_t e;
  if (field->dtype == PP_FLOAT32)
    e = launch_fd_bwd<float>(D, static_cast<const float*>(field->data), a,
                             grad_jac ? static_cast<const float*>(grad_jac->data) : nullptr,
                             grad_det ? static_cast<const float*>(grad_det->data) : nullptr,
                             static_cast<float*>(grad_field->data), grad_field, nvox, st);
  else
    e = launch_fd_bwd<double>(D, static_cast<const double*>(field->data), a,
                              grad_jac ? static_cast<const double*>(grad_jac->data) : nullptr,
                              grad_det ? static_cast<const double*>(grad_det->data) : nullptr,
                              static_cast<double*>(grad_field->data), grad_field, nvox, st);
  ppc::count_launch();
  return ppc::cuda_check(e, "jacobian backward launch");
}

// det of jac (M, D, D) into det (M), or, with grad_det / grad_jac given,
// grad_jac = grad_det * cofactor(jac).  M-dimensional batches are flattened
// by the caller into one leading dimension.
int pp_jacobian_det(const pp_tensor* jac, const pp_tensor* det, const pp_tensor* grad_det, const pp_tensor* grad_jac,
                    void* stream) {
  int rc = ppc::check_tensor(jac, "jacobian");
  if (rc) return rc;
  if (jac->ndim != 3 || jac->sizes[1] != jac->sizes[2] || jac->sizes[1] < 1 || jac->sizes[1] > 3)
    return ppc::fail(PP_ERR_ARG, "(): expected (M, D, D) matrices, D = 1-3");
  if (jac->dtype != PP_FLOAT32 && jac->dtype != PP_FLOAT64) return ppc::fail(PP_ERR_DTYPE, "(): expected float32 or float64");
  const int D = static_cast<int>(jac->sizes[1]);
  const int64_t M = jac->sizes[0];
  const pp_tensor* dref = det ? det : grad_det;
  if (!dref) return ppc::fail(PP_ERR_ARG, "(): expected det or grad_det");
  if ((rc = ppc::check_tensor(dref, "determinant"))) return rc;
  if (dref->ndim != 1 || dref->sizes[0] != M || dref->dtype != jac->dtype) return ppc::fail(PP_ERR_ARG, "(): determinant must be (M)");
  if (det && grad_det) return ppc::fail(PP_ERR_ARG, "(): give det (forward) or grad_det and grad_jac (backward)");
  if (grad_det) {
    if ((rc = ppc::check_tensor(grad_jac, "grad_jac"))) return rc;
    if (grad_jac->ndim != 3 || grad_jac->sizes[0] != M || grad_jac->sizes[1] != D || grad_jac->sizes[2] != D ||
        grad_jac->dtype != jac->dtype)
      return ppc::fail(PP_ERR_ARG, "(): grad_jac must have the matrices' shape");
  }
  if (M == 0) return PP_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned nb = static_cast<unsigned>((M + 255) / 256);
  const int64_t gsM = grad_jac ? grad_jac->strides[0] : 0, gsI = grad_jac ? grad_jac->strides[1] : 0,
                gsJ = grad_jac ? grad_jac->strides[2] : 0;
#define PP_DET_LAUNCH(T, DD)                                                                                   \
  det_kernel<T, DD><<<nb, 256, 0, st>>>(static_cast<const T*>(jac->data), jac->strides[0], jac->strides[1],  \
                                        jac->strides[2], det ? static_cast<T*>(det->data) : nullptr,          \
                                        dref->strides[0], M,                                                   \
                                        grad_det ? static_cast<const T*>(grad_det->data) : nullptr,           \
                                        grad_det ? static_cast<T*>(grad_jac->data) : nullptr, gsM, gsI, gsJ)
  if (jac->dtype == PP_FLOAT32) {
    if (D == 1) PP_DET_LAUNCH(float, 1); else if (D == 2) PP_DET_LAUNCH(float, 2); else PP_DET_LAUNCH(float, 3);
  } else {
    if (D == 1) PP_DET_LAUNCH(double, 1); else if (D == 2) PP_DET_LAUNCH(double, 2); else PP_DET_LAUNCH(double, 3);
  }
#undef PP_DET_LAUNCH
  ppc::count_launch();
  return ppc::cuda_check(cudaGetLastError(), "determinant launch");
}

}  // extern "C"
