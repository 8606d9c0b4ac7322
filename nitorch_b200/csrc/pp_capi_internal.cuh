// Host helpers shared by the C-ABI translation units (error state,
// tensor checks, strided elementwise kernels).
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <atomic>
#include <string>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include "../../include/nitorch_b200.h"
#include "pp_common.cuh"

namespace ppc {

extern thread_local std::string g_err;

// pp_options -> per-axis bound codes and orders (padded with the last
// entry); validates them (pp_capi.cu).
int read_options(const pp_options* o, int D, int bound[3], int order[3]);

// Number of kernels this library has launched (all threads, all devices);
// exported as pp_kernel_launches() so callers can audit what ran.
extern std::atomic<unsigned long long> g_launches;
inline void count_launch(unsigned long long n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

inline int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

inline int cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return PP_OK;
  return fail(PP_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

inline size_t dtype_size(int dt) {
  switch (dt) {
    case PP_FLOAT32: return 4;
    case PP_FLOAT64: return 8;
    case PP_BFLOAT16: case PP_FLOAT16: return 2;
  }
  return 0;
}

inline int64_t numel(const pp_tensor* t) {
  int64_t n = 1;
  for (int i = 0; i < t->ndim; ++i) n *= t->sizes[i];
  return n;
}

inline bool contiguous(const pp_tensor* t) {
  int64_t s = 1;
  for (int i = t->ndim - 1; i >= 0; --i) {
    if (t->sizes[i] != 1 && t->strides[i] != s) return false;
    s *= t->sizes[i];
  }
  return true;
}

inline int64_t max_offset(const pp_tensor* t, int first) {
  int64_t o = 0;
  for (int i = first; i < t->ndim; ++i) o += (t->sizes[i] - 1) * t->strides[i];
  return o;
}

inline int check_tensor(const pp_tensor* t, const char* name) {
  if (!t) return fail(PP_ERR_ARG, "(): expected %s not be undefined, but it is", name);
  if (t->ndim < 0 || t->ndim > PP_MAX_DIM) return fail(PP_ERR_ARG, "(): %s has an invalid number of dimensions %d", name, t->ndim);
  if (dtype_size(t->dtype) == 0) return fail(PP_ERR_DTYPE, "(): %s has an unsupported dtype code %d", name, t->dtype);
  for (int i = 0; i < t->ndim; ++i) {
    if (t->sizes[i] < 0) return fail(PP_ERR_ARG, "(): %s has a negative size", name);
    if (t->strides[i] < 0) return fail(PP_ERR_ARG, "(): %s has a negative stride", name);
  }
  if (!t->data && numel(t) > 0) return fail(PP_ERR_ARG, "(): %s has a null data pointer", name);
  return PP_OK;
}

// --- strided elementwise helpers -------------------------------------------
struct Strided {
  int ndim;
  int64_t sizes[PP_MAX_DIM];
  int64_t strides[PP_MAX_DIM];
  int64_t numel;
};

inline Strided make_strided(const pp_tensor* t) {
  Strided s;
  s.ndim = t->ndim;
  for (int i = 0; i < t->ndim; ++i) { s.sizes[i] = t->sizes[i]; s.strides[i] = t->strides[i]; }
  s.numel = numel(t);
  return s;
}

__device__ __forceinline__ int64_t strided_offset(const Strided& s, int64_t i) {
  int64_t off = 0;
  for (int d = s.ndim - 1; d >= 0; --d) {
    const int64_t q = i / s.sizes[d];
    off += (i - q * s.sizes[d]) * s.strides[d];
    i = q;
  }
  return off;
}

template <class S>
__global__ void zero_strided(S* p, Strided s) {
  int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (; i < s.numel; i += step) p[strided_offset(s, i)] = S(0);
}

// dense float accumulator -> strided 16-bit storage
template <class S>
__global__ void store_from_f32(const float* acc, S* dst, Strided s) {
  int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (; i < s.numel; i += step) dst[strided_offset(s, i)] = ppk::from_acc<S>(acc[i]);
}

inline int grid_blocks(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  const int64_t cap = 148LL * 16;
  return static_cast<int>(b < 1 ? 1 : (b > cap ? cap : b));
}

inline int zero_fill(const pp_tensor* t, cudaStream_t st) {
  const int64_t n = numel(t);
  if (n == 0) return PP_OK;
  if (contiguous(t))
    return cuda_check(cudaMemsetAsync(t->data, 0, n * dtype_size(t->dtype), st), "zero fill");
  Strided s = make_strided(t);
  switch (t->dtype) {
    case PP_FLOAT32: zero_strided<float><<<grid_blocks(n), 256, 0, st>>>(static_cast<float*>(t->data), s); break;
    case PP_FLOAT64: zero_strided<double><<<grid_blocks(n), 256, 0, st>>>(static_cast<double*>(t->data), s); break;
    case PP_BFLOAT16: zero_strided<__nv_bfloat16><<<grid_blocks(n), 256, 0, st>>>(static_cast<__nv_bfloat16*>(t->data), s); break;
    case PP_FLOAT16: zero_strided<__half><<<grid_blocks(n), 256, 0, st>>>(static_cast<__half*>(t->data), s); break;
  }
  count_launch();
  return cuda_check(cudaGetLastError(), "zero fill");
}

inline int store_f32(const float* acc, const pp_tensor* t, cudaStream_t st) {
  const int64_t n = numel(t);
  if (n == 0) return PP_OK;
  Strided s = make_strided(t);
  if (t->dtype == PP_BFLOAT16)
    store_from_f32<__nv_bfloat16><<<grid_blocks(n), 256, 0, st>>>(acc, static_cast<__nv_bfloat16*>(t->data), s);
  else
    store_from_f32<__half><<<grid_blocks(n), 256, 0, st>>>(acc, static_cast<__half*>(t->data), s);
  count_launch();
  return cuda_check(cudaGetLastError(), "16-bit store");
}

// Defined in pp_capi.cu, shared with the batched entry points.
int read_options(const pp_options* o, int D, int bound[3], int order[3]);
void set_image(const pp_tensor* t, int D, int64_t& sN, int64_t& sC, int64_t s[3]);
void set_grid(const pp_tensor* t, int D, int64_t& sN, int64_t s[3], int64_t& sD);
bool fits32(int64_t v);

// Deterministic scatters (pp_capi.cu): max |t| of a tensor as float bits
// into *out (which starts at zero), and the int64 fixed-point accumulator
// (contiguous in out's logical order, scale from *mx times bound) -> out,
// plus `self` (accumulation-type values laid out like acc) where given.
int det_absmax_of(const pp_tensor* t, unsigned int* out, cudaStream_t st);
// The 3-D linear float32 displacement self-composition (svf_compose.cu), or
// PP_ERR_UNSUPPORTED (nothing launched) for any other field.
int svf_compose_linear3(const pp_tensor* disp, const pp_tensor* out, const int32_t bound[3], int32_t extrapolate,
                        cudaStream_t st);
// Its backward into a zeroed four-slot channel-interleaved accumulator, or
// PP_ERR_UNSUPPORTED (nothing launched).
int svf_compose_backward_linear3(const pp_tensor* grad, const pp_tensor* disp, float* acc, const int32_t bound[3],
                                 int32_t extrapolate, cudaStream_t st);
int det_finalize_to(const unsigned long long* acc, const pp_tensor* out, const unsigned int* mx, double bound,
                    cudaStream_t st, const void* self = nullptr);

}  // namespace ppc
