// C ABI of the push/pull library: argument validation (the checks of
// nitorch/_C/src/pushpull.cpp:19-72), output preparation (the zero-filled
// allocations of pushpull_common.cpp:476-571), mode wiring (pushpull.cpp
// flag table) and dispatch to the kernel family of pp_kernels.cuh.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <string>

#include "../../include/nitorch_b200.h"
#include "pp_capi_internal.cuh"
#include "pp_kernels.cuh"

// Launchers compiled from pp_inst.cu, one per (dtype, dim, mode).
#define PP_DECL_MODES(S, D)                                                        \
  cudaError_t pp_launch_##S##_d##D##_m0(int, bool, const ppk::PPArgs&, cudaStream_t); \
  cudaError_t pp_launch_##S##_d##D##_m1(int, bool, const ppk::PPArgs&, cudaStream_t); \
  cudaError_t pp_launch_##S##_d##D##_m2(int, bool, const ppk::PPArgs&, cudaStream_t); \
  cudaError_t pp_launch_##S##_d##D##_m3(int, bool, const ppk::PPArgs&, cudaStream_t); \
  cudaError_t pp_launch_##S##_d##D##_m4(int, bool, const ppk::PPArgs&, cudaStream_t); \
  cudaError_t pp_launch_##S##_d##D##_m5(int, bool, const ppk::PPArgs&, cudaStream_t); \
  cudaError_t pp_launch_##S##_d##D##_m6(int, bool, const ppk::PPArgs&, cudaStream_t); \
  cudaError_t pp_launch_##S##_d##D##_m7(int, bool, const ppk::PPArgs&, cudaStream_t); \
  cudaError_t pp_launch_##S##_d##D##_m8(int, bool, const ppk::PPArgs&, cudaStream_t);
#define PP_DECL_DIMS(S) PP_DECL_MODES(S, 1) PP_DECL_MODES(S, 2) PP_DECL_MODES(S, 3)
PP_DECL_DIMS(f32)
PP_DECL_DIMS(f64)
PP_DECL_DIMS(bf16)
PP_DECL_DIMS(f16)
#undef PP_DECL_DIMS
#undef PP_DECL_MODES

#define PP_ROW(S, D)                                                                          \
  {pp_launch_##S##_d##D##_m0, pp_launch_##S##_d##D##_m1, pp_launch_##S##_d##D##_m2,          \
   pp_launch_##S##_d##D##_m3, pp_launch_##S##_d##D##_m4, pp_launch_##S##_d##D##_m5,          \
   pp_launch_##S##_d##D##_m6, pp_launch_##S##_d##D##_m7, pp_launch_##S##_d##D##_m8}
#define PP_TYPE(S) {PP_ROW(S, 1), PP_ROW(S, 2), PP_ROW(S, 3)}
static const pp_launcher_t kLaunchers[4][3][ppk::K_NMODES] = {PP_TYPE(f32), PP_TYPE(f64), PP_TYPE(bf16),
                                                              PP_TYPE(f16)};
#undef PP_TYPE
#undef PP_ROW

namespace ppk {
thread_local char g_last_kernel[64] = "";
void note_kernel(const char* family, int mode, int ord, int cb) {
  std::snprintf(g_last_kernel, sizeof(g_last_kernel), "%s mode=%d order=%d cb=%d", family, mode, ord, cb);
}

// Lane-split push (pp_lanes_kernel) and vectorised scatters (F_VEC): on
// unless the environment sets PP_PUSH_LANES=0 (read once), which falls back
// to one scalar reduction per channel and tap everywhere.
bool lanes_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("PP_PUSH_LANES");
    return !(e && e[0] == '0');
  }();
  return on;
}
}  // namespace ppk


namespace ppc {

thread_local std::string g_err;
std::atomic<unsigned long long> g_launches{0};

// --- options ----------------------------------------------------------------
int read_options(const pp_options* o, int D, int bound[3], int order[3]) {
  if (!o) return fail(PP_ERR_ARG, "(): expected options not be undefined");
  if (o->nbound < 1 || o->nbound > 3) return fail(PP_ERR_ARG, "(): expected non empty parameter bound_mode");
  if (o->norder < 1 || o->norder > 3) return fail(PP_ERR_ARG, "(): expected non empty parameter interpolation_mode");
  for (int a = 0; a < 3; ++a) {
    bound[a] = o->bound[a < o->nbound ? a : o->nbound - 1];
    order[a] = o->order[a < o->norder ? a : o->norder - 1];
  }
  for (int a = 0; a < D; ++a) {
    const int b = bound[a];
    if (!(b >= 0 && b <= 5) && b != PP_BOUND_ZERO)
      return fail(PP_ERR_ARG, "(): unsupported bound code %d", b);
    if (order[a] < 0 || order[a] > 7)
      return fail(PP_ERR_ARG, "(): unsupported interpolation order %d", order[a]);
  }
  return PP_OK;
}

int iso_order(int D, const int order[3]) {
  for (int a = 1; a < D; ++a)
    if (order[a] != order[0]) return -1;
  return order[0];
}

// --- tensor -> kernel argument helpers ----------------------------------------
void set_image(const pp_tensor* t, int D, int64_t& sN, int64_t& sC, int64_t s[3]) {
  sN = t->strides[0];
  sC = t->strides[1];
  for (int a = 0; a < 3; ++a) s[a] = a < D ? t->strides[2 + a] : 0;
}

void set_grid(const pp_tensor* t, int D, int64_t& sN, int64_t s[3], int64_t& sD) {
  sN = t->strides[0];
  for (int a = 0; a < 3; ++a) s[a] = a < D ? t->strides[1 + a] : 0;
  sD = t->strides[1 + D];
}

bool fits32(int64_t v) { return v < (int64_t(1) << 31) - 1; }

cudaError_t launch(int dtype, int D, int mode, int ord, bool wide, const ppk::PPArgs& a, cudaStream_t st) {
  if (dtype < 0 || dtype > 3 || D < 1 || D > 3 || mode < 0 || mode >= ppk::K_NMODES) return cudaErrorInvalidValue;
  count_launch();
  return kLaunchers[dtype][D - 1][mode](ord, wide, a, st);
}

int grid_dtype_for(int image_dtype) { return image_dtype == PP_FLOAT64 ? PP_FLOAT64 : PP_FLOAT32; }

// Common checks of grid (pushpull.cpp:19-72): 3-5 dims, last dim = ndim-2,
// non-empty spatial dims.
int check_grid(const pp_tensor* grid, int& D) {
  int rc = check_tensor(grid, "grid");
  if (rc) return rc;
  if (grid->ndim < 3 || grid->ndim > 5)
    return fail(PP_ERR_ARG, "(): expected 3D, 4D or 5D grid but got input with %d dimensions", grid->ndim);
  D = grid->ndim - 2;
  if (grid->sizes[grid->ndim - 1] != D)
    return fail(PP_ERR_ARG, "(): expected grid to have size %d in last dimension, but got %lld", D,
                (long long)grid->sizes[grid->ndim - 1]);
  for (int i = 1; i < grid->ndim - 1; ++i)
    if (grid->sizes[i] <= 0)
      return fail(PP_ERR_ARG, "(): expected grid to have non-empty spatial dimensions, but dimension %d is empty", i);
  if (grid->dtype != PP_FLOAT32 && grid->dtype != PP_FLOAT64)
    return fail(PP_ERR_DTYPE, "(): expected grid to be float32 or float64");
  return PP_OK;
}

int check_image(const pp_tensor* t, const char* name, int D, int grid_dtype) {
  int rc = check_tensor(t, name);
  if (rc) return rc;
  if (t->ndim != D + 2)
    return fail(PP_ERR_ARG, "(): expected %s to have %d dimensions, but it has %d", name, D + 2, t->ndim);
  for (int i = 2; i < t->ndim; ++i)
    if (t->sizes[i] <= 0)
      return fail(PP_ERR_ARG, "(): expected %s to have non-empty spatial dimensions, but dimension %d is empty", name, i);
  if (grid_dtype_for(t->dtype) != grid_dtype)
    return fail(PP_ERR_DTYPE, "(): expected %s and grid to have the same dtype (or a 16-bit %s with a float32 grid)", name, name);
  return PP_OK;
}

int check_same_sizes(const pp_tensor* t, const int64_t* sizes, int nd, const char* name) {
  if (t->ndim != nd) return fail(PP_ERR_ARG, "(): %s has %d dimensions, expected %d", name, t->ndim, nd);
  for (int i = 0; i < nd; ++i)
    if (t->sizes[i] != sizes[i])
      return fail(PP_ERR_ARG, "(): %s has size %lld in dimension %d, expected %lld", name,
                  (long long)t->sizes[i], i, (long long)sizes[i]);
  return PP_OK;
}

}  // namespace ppc

using namespace ppc;

namespace {

// Core dispatcher shared by the entry points.
struct Call {
  int D = 0;
  int bound[3] = {0, 0, 0}, order[3] = {1, 1, 1};
  int dtype = PP_FLOAT32;  // image storage dtype
  ppk::PPArgs a;
  Call() { std::memset(&a, 0, sizeof(a)); }
};

int prepare(Call& k, const pp_tensor* grid, const pp_options* opt) {
  int rc = check_grid(grid, k.D);
  if (rc) return rc;
  rc = read_options(opt, k.D, k.bound, k.order);
  if (rc) return rc;
  for (int a = 0; a < 3; ++a) { k.a.bound[a] = k.bound[a]; k.a.order[a] = k.order[a]; }
  k.a.extrapolate = opt->extrapolate;
  k.a.perm = opt->sample_order;
  k.a.brick_start = (k.D == 3 && opt->sample_order) ? opt->brick_start : nullptr;
  k.a.brec = k.a.brick_start ? reinterpret_cast<const float4*>(opt->brick_records) : nullptr;
  k.a.grid = grid->data;
  set_grid(grid, k.D, k.a.grid_sN, k.a.grid_s, k.a.grid_sD);
  k.a.N = grid->sizes[0];
  int64_t nv = grid->sizes[0];
  for (int a = 0; a < 3; ++a) {
    k.a.trgt_size[a] = a < k.D ? grid->sizes[1 + a] : 1;
    nv *= k.a.trgt_size[a];
  }
  k.a.nvox = nv;
  return PP_OK;
}

bool need_wide(const Call& k, std::initializer_list<const pp_tensor*> spatial) {
  if (!fits32(k.a.nvox)) return true;
  for (const pp_tensor* t : spatial)
    if (t && !fits32(max_offset(t, 2))) return true;
  return false;
}

int run(Call& k, int mode, bool wide, cudaStream_t st) {
  const int ord = iso_order(k.D, k.order);
  if (k.a.nvox == 0) return PP_OK;
  if (k.a.brick_start) {
    // bricks of the scatter target / gathered source, as pp_brick_order cut it
    const int bs[3] = {PP_BRICK_X, PP_BRICK_Y, PP_BRICK_Z};
    for (int a = 0; a < 3; ++a) k.a.nbrick[a] = (k.a.src_size[a] + bs[a] - 1) / bs[a];
  }
  return cuda_check(launch(k.dtype, k.D, mode, ord, wide, k.a, st), "push/pull kernel launch");
}

// Scatter-mode workspace: 16-bit outputs accumulate into a float buffer;
// deterministic mode accumulates into int64 fixed point (256-byte header
// holding the float bits of max |target|, then N*C*spatial int64).
// Channel slots of the interleaved push accumulator for C channels (0: none).
int vec_slots(int64_t C) { return C == 2 ? 2 : (C == 3 || C == 4) ? 4 : 0; }

// Workspace a scatter into `out` cannot do without: the float accumulator of
// 16-bit outputs, the fixed-point accumulator of the deterministic mode.
size_t scatter_ws_required(const pp_tensor* out, int flags) {
  if (!out) return 0;
  const int64_t n = numel(out);
  if (flags & PP_DETERMINISTIC) return 256 + ((n * 8 + 255) / 256) * 256;
  if (out->dtype == PP_BFLOAT16 || out->dtype == PP_FLOAT16) return ((n * 4 + 255) / 256) * 256;
  return 0;
}

// Channel-interleaved float accumulator of the vectorised push (3-D images
// of 2-4 channels, see pp_lanes_kernel); 0 where it does not apply.
size_t scatter_ws_vec(const pp_tensor* out, int flags) {
  if (!out || (flags & PP_DETERMINISTIC) || out->ndim != 5 || out->sizes[1] <= 0) return 0;
  const int CP = vec_slots(out->sizes[1]);
  if (!CP) return 0;
  const int64_t vox = numel(out) / out->sizes[1];
  return ((vox * CP * 4 + 255) / 256) * 256;
}

// Workspace size reported to callers: enough for the fastest path.
size_t scatter_ws_bytes(const pp_tensor* out, int flags) {
  const size_t r = scatter_ws_required(out, flags), v = scatter_ws_vec(out, flags);
  return r > v ? r : v;
}

// interleaved float accumulator (N, *spatial, CP) -> strided output
template <class S>
__global__ void store_interleaved(const float* acc, S* dst, Strided s, int64_t V, int64_t C, int CP) {
  int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (; i < s.numel; i += step) {
    const int64_t lin = i % V, nc = i / V;
    const int64_t c = nc % C, nb = nc / C;
    dst[strided_offset(s, i)] = ppk::from_acc<S>(static_cast<typename ppk::Acc<S>::type>(acc[(nb * V + lin) * CP + c]));
  }
}

// Contiguous (N, C, *spatial) output: one thread per voxel, one vector load
// of its CP accumulator slots, C coalesced stores.  blockIdx.y = batch item.
template <class S, int CP>
__global__ void store_interleaved_vox(const float* __restrict__ acc, S* __restrict__ dst, int64_t V, int C) {
  using VT = typename std::conditional<CP == 4, float4, float2>::type;
  const int64_t nb = blockIdx.y;
  const float* a = acc + nb * V * CP;
  S* o = dst + nb * C * V;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < V; i += step) {
    const VT v = *reinterpret_cast<const VT*>(a + i * CP);
    const float* f = reinterpret_cast<const float*>(&v);
#pragma unroll
    for (int c = 0; c < CP; ++c)
      if (c < C) o[c * V + i] = ppk::from_acc<S>(static_cast<typename ppk::Acc<S>::type>(f[c]));
  }
}

template <class S>
int store_interleaved_fast(const float* acc, S* dst, int64_t N, int64_t V, int C, int CP, cudaStream_t st) {
  const int64_t want = (V + 255) / 256;
  const unsigned bx = static_cast<unsigned>(want < 148 * 16 ? want : 148 * 16);
  const dim3 grid(bx > 0 ? bx : 1, static_cast<unsigned>(N));
  if (CP == 4) store_interleaved_vox<S, 4><<<grid, 256, 0, st>>>(acc, dst, V, C);
  else store_interleaved_vox<S, 2><<<grid, 256, 0, st>>>(acc, dst, V, C);
  count_launch();
  return cuda_check(cudaGetLastError(), "interleaved store");
}

// A 4-slot channel-interleaved accumulator -> a float32 (N, X, Y, Z, 3)
// field: contiguous fields copy three floats per voxel, others go through
// the strided store on an (N, 3, X, Y, Z) view of the field.
__global__ void store_field3(const float4* __restrict__ acc, float* __restrict__ dst, int64_t nvox) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < nvox; v += step) {
    const float4 q = acc[v];
    dst[3 * v] = q.x;
    dst[3 * v + 1] = q.y;
    dst[3 * v + 2] = q.z;
  }
}

int store_interleaved_to(const float* acc, const pp_tensor* out, int CP, cudaStream_t st);

int store_field_from4(const float* acc, const pp_tensor* field, cudaStream_t st) {
  const int64_t n = numel(field);
  if (n == 0) return PP_OK;
  bool contiguous = true;
  {
    int64_t e = 1;
    for (int i = field->ndim - 1; i >= 0 && contiguous; --i) {
      if (field->sizes[i] > 1 && field->strides[i] != e) contiguous = false;
      e *= field->sizes[i];
    }
  }
  if (contiguous) {
    const int64_t nvox = n / 3, want = (nvox + 255) / 256;
    const unsigned nb = static_cast<unsigned>(want < 148 * 16 ? (want > 0 ? want : 1) : 148 * 16);
    store_field3<<<nb, 256, 0, st>>>(reinterpret_cast<const float4*>(acc), static_cast<float*>(field->data), nvox);
    count_launch();
    return cuda_check(cudaGetLastError(), "field store");
  }
  pp_tensor view = *field;  // (N, X, Y, Z, 3) as (N, 3, X, Y, Z)
  view.sizes[1] = 3;
  view.strides[1] = field->strides[4];
  for (int d = 0; d < 3; ++d) {
    view.sizes[2 + d] = field->sizes[1 + d];
    view.strides[2 + d] = field->strides[1 + d];
  }
  return store_interleaved_to(acc, &view, 4, st);
}

int store_interleaved_to(const float* acc, const pp_tensor* out, int CP, cudaStream_t st) {
  const int64_t n = numel(out);
  if (n == 0) return PP_OK;
  Strided s = make_strided(out);
  const int64_t C = out->sizes[1], V = n / (out->sizes[0] * C);
  bool contiguous = out->sizes[0] <= 65535 && (CP == 2 || CP == 4) && C <= CP;
  {
    int64_t e = 1;
    for (int i = out->ndim - 1; i >= 0 && contiguous; --i) {
      if (out->sizes[i] > 1 && out->strides[i] != e) contiguous = false;
      e *= out->sizes[i];
    }
  }
  if (contiguous) {
    if (out->dtype == PP_FLOAT32)
      return store_interleaved_fast(acc, static_cast<float*>(out->data), out->sizes[0], V, static_cast<int>(C), CP, st);
    if (out->dtype == PP_BFLOAT16)
      return store_interleaved_fast(acc, static_cast<__nv_bfloat16*>(out->data), out->sizes[0], V,
                                    static_cast<int>(C), CP, st);
  }
  const int nb = grid_blocks(n);
  switch (out->dtype) {
    case PP_FLOAT32: store_interleaved<float><<<nb, 256, 0, st>>>(acc, static_cast<float*>(out->data), s, V, C, CP); break;
    case PP_BFLOAT16: store_interleaved<__nv_bfloat16><<<nb, 256, 0, st>>>(acc, static_cast<__nv_bfloat16*>(out->data), s, V, C, CP); break;
    default: return fail(PP_ERR_DTYPE, "(): no interleaved store for this dtype");
  }
  count_launch();
  return cuda_check(cudaGetLastError(), "interleaved store");
}

// max |t| over a strided tensor, as float bits (non-negative floats order
// like their bit patterns, so an integer atomicMax is exact and
// order-independent).
template <class S>
__global__ void det_absmax(const S* t, Strided s, unsigned int* out) {
  int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  float m = 0.f;
  for (; i < s.numel; i += step) m = fmaxf(m, fabsf(static_cast<float>(ppk::to_acc(t[strided_offset(s, i)]))));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

__global__ void det_set_one(unsigned int* out) { *out = __float_as_uint(1.0f); }

// int64 fixed point (plus, when `self` is set, a term per element in the
// accumulation type laid out like acc) -> strided output
template <class S>
__global__ void det_finalize(const unsigned long long* acc, S* dst, Strided s, const unsigned int* mx,
                             double bound, const typename ppk::Acc<S>::type* self) {
  using A = typename ppk::Acc<S>::type;
  const float m = __uint_as_float(*mx);
  const double b = static_cast<double>(m) * bound;
  double inv = 1.0;
  if (b > 0.0) {
    int ex;
    frexp(b, &ex);
    inv = ldexp(1.0, ex - 61);
  }
  int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (; i < s.numel; i += step) {
    const double v = static_cast<double>(static_cast<long long>(acc[i])) * inv;
    A r = static_cast<A>(v);
    if (self) r += self[i];
    dst[strided_offset(s, i)] = ppk::from_acc<S>(r);
  }
}

}  // namespace

namespace ppc {

int det_absmax_of(const pp_tensor* t, unsigned int* out, cudaStream_t st) {
  const int64_t n = numel(t);
  if (n == 0) return PP_OK;
  Strided s = make_strided(t);
  const int nb = grid_blocks(n);
  switch (t->dtype) {
    case PP_FLOAT32: det_absmax<float><<<nb, 256, 0, st>>>(static_cast<const float*>(t->data), s, out); break;
    case PP_FLOAT64: det_absmax<double><<<nb, 256, 0, st>>>(static_cast<const double*>(t->data), s, out); break;
    case PP_BFLOAT16: det_absmax<__nv_bfloat16><<<nb, 256, 0, st>>>(static_cast<const __nv_bfloat16*>(t->data), s, out); break;
    default: det_absmax<__half><<<nb, 256, 0, st>>>(static_cast<const __half*>(t->data), s, out); break;
  }
  count_launch();
  return cuda_check(cudaGetLastError(), "deterministic max");
}

int det_finalize_to(const unsigned long long* acc, const pp_tensor* out, const unsigned int* mx, double bound,
                    cudaStream_t st, const void* self) {
  const int64_t n = numel(out);
  if (n == 0) return PP_OK;
  Strided s = make_strided(out);
  const int nb = grid_blocks(n);
  switch (out->dtype) {
    case PP_FLOAT32:
      det_finalize<float><<<nb, 256, 0, st>>>(acc, static_cast<float*>(out->data), s, mx, bound,
                                              static_cast<const float*>(self));
      break;
    case PP_FLOAT64:
      det_finalize<double><<<nb, 256, 0, st>>>(acc, static_cast<double*>(out->data), s, mx, bound,
                                               static_cast<const double*>(self));
      break;
    case PP_BFLOAT16:
      det_finalize<__nv_bfloat16><<<nb, 256, 0, st>>>(acc, static_cast<__nv_bfloat16*>(out->data), s, mx, bound,
                                                      static_cast<const float*>(self));
      break;
    default:
      det_finalize<__half><<<nb, 256, 0, st>>>(acc, static_cast<__half*>(out->data), s, mx, bound,
                                               static_cast<const float*>(self));
      break;
  }
  count_launch();
  return cuda_check(cudaGetLastError(), "deterministic finalize");
}

}  // namespace ppc

extern "C" {

int pp_abi_version(void) { return 105; }

const char* pp_last_error(void) { return g_err.c_str(); }

unsigned long long pp_kernel_launches(void) { return g_launches.load(); }

const char* pp_last_kernel(void) { return ppk::g_last_kernel; }

size_t pp_push_workspace_bytes(const pp_tensor* out, int32_t flags) {
  return scatter_ws_bytes(out, flags);
}

int pp_grid_pull(const pp_tensor* input, const pp_tensor* grid, const pp_tensor* out,
                 const pp_options* opt, void* stream) {
  Call k;
  int rc = prepare(k, grid, opt);
  if (rc) return rc;
  if ((rc = check_image(input, "input", k.D, grid->dtype))) return rc;
  if (input->sizes[0] != grid->sizes[0])
    return fail(PP_ERR_ARG, "(): expected input and grid to have the same batch size");
  if ((rc = check_tensor(out, "output"))) return rc;
  int64_t osz[5] = {grid->sizes[0], input->sizes[1], 1, 1, 1};
  for (int a = 0; a < k.D; ++a) osz[2 + a] = grid->sizes[1 + a];
  if ((rc = check_same_sizes(out, osz, k.D + 2, "output"))) return rc;
  if (out->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): output dtype must match input");
  k.dtype = input->dtype;
  k.a.src = input->data;
  k.a.C = input->sizes[1];
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? input->sizes[2 + a] : 1;
  set_image(input, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.out = out->data;
  set_image(out, k.D, k.a.out_sN, k.a.out_sC, k.a.out_s);
  return run(k, ppk::K_PULL, need_wide(k, {input, out}), static_cast<cudaStream_t>(stream));
}

int pp_grid_grad(const pp_tensor* input, const pp_tensor* grid, const pp_tensor* out,
                 const pp_options* opt, void* stream) {
  Call k;
  int rc = prepare(k, grid, opt);
  if (rc) return rc;
  if ((rc = check_image(input, "input", k.D, grid->dtype))) return rc;
  if (input->sizes[0] != grid->sizes[0])
    return fail(PP_ERR_ARG, "(): expected input and grid to have the same batch size");
  if ((rc = check_tensor(out, "output"))) return rc;
  int64_t osz[6] = {grid->sizes[0], input->sizes[1], 1, 1, 1, 1};
  for (int a = 0; a < k.D; ++a) osz[2 + a] = grid->sizes[1 + a];
  osz[2 + k.D] = k.D;
  if ((rc = check_same_sizes(out, osz, k.D + 3, "output"))) return rc;
  if (out->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): output dtype must match input");
  k.dtype = input->dtype;
  k.a.src = input->data;
  k.a.C = input->sizes[1];
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? input->sizes[2 + a] : 1;
  set_image(input, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.out = out->data;
  set_image(out, k.D, k.a.out_sN, k.a.out_sC, k.a.out_s);
  k.a.out_sK = out->strides[2 + k.D];
  return run(k, ppk::K_SGRAD, need_wide(k, {input, out}), static_cast<cudaStream_t>(stream));
}

int pp_grid_pull_grad(const pp_tensor* input, const pp_tensor* grid, const pp_tensor* out,
                      const pp_tensor* out_grad, const pp_options* opt, void* stream) {
  Call k;
  int rc = prepare(k, grid, opt);
  if (rc) return rc;
  if ((rc = check_image(input, "input", k.D, grid->dtype))) return rc;
  if (input->sizes[0] != grid->sizes[0])
    return fail(PP_ERR_ARG, "(): expected input and grid to have the same batch size");
  if ((rc = check_tensor(out, "output")) || (rc = check_tensor(out_grad, "output gradient"))) return rc;
  int64_t osz[6] = {grid->sizes[0], input->sizes[1], 1, 1, 1, 1};
  for (int a = 0; a < k.D; ++a) osz[2 + a] = grid->sizes[1 + a];
  if ((rc = check_same_sizes(out, osz, k.D + 2, "output"))) return rc;
  osz[2 + k.D] = k.D;
  if ((rc = check_same_sizes(out_grad, osz, k.D + 3, "output gradient"))) return rc;
  if (out->dtype != input->dtype || out_grad->dtype != input->dtype)
    return fail(PP_ERR_DTYPE, "(): output dtype must match input");
  k.dtype = input->dtype;
  k.a.src = input->data;
  k.a.C = input->sizes[1];
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? input->sizes[2 + a] : 1;
  set_image(input, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.out = out_grad->data;
  set_image(out_grad, k.D, k.a.out_sN, k.a.out_sC, k.a.out_s);
  k.a.out_sK = out_grad->strides[2 + k.D];
  k.a.aux = out->data;  // the pulled values, at the target strides
  set_image(out, k.D, k.a.trgt_sN, k.a.trgt_sC, k.a.trgt_s);
  k.a.flags |= ppk::F_A;
  return run(k, ppk::K_SGRAD, need_wide(k, {input, out, out_grad}), static_cast<cudaStream_t>(stream));
}

// Scatter helper: push `trgt` (N,C,*grid[,K]) into `out` (N,C,*shape) with
// `mode`, optionally fused with a grid gradient of `src`.  `trgt_t` is the
// target tensor (NULL for count), used by the deterministic mode's bound.
static int scatter_into(Call& k, int mode, const pp_tensor* out, const pp_tensor* trgt_t, bool wide,
                        int flags, void* ws, size_t ws_bytes, cudaStream_t st) {
  int rc;
  const bool det = (flags & PP_DETERMINISTIC) != 0;
  const bool half = out->dtype == PP_BFLOAT16 || out->dtype == PP_FLOAT16;
  const size_t need = scatter_ws_required(out, flags);
  if (need && (!ws || ws_bytes < need))
    return fail(PP_ERR_WORKSPACE, "(): this push output needs %zu bytes of workspace", need);
  // contiguous (N, C, *shape) strides of the accumulation buffers
  int64_t cs[PP_MAX_DIM];
  {
    int64_t s = 1;
    for (int i = out->ndim - 1; i >= 0; --i) { cs[i] = s; s *= out->sizes[i]; }
  }
  if (det) {
    unsigned char* w = static_cast<unsigned char*>(ws);
    unsigned int* mx = reinterpret_cast<unsigned int*>(w);
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(w + 256);
    if ((rc = cuda_check(cudaMemsetAsync(ws, 0, need, st), "workspace clear"))) return rc;
    if (trgt_t) {
      if ((rc = det_absmax_of(trgt_t, mx, st))) return rc;
    } else {
      det_set_one<<<1, 1, 0, st>>>(mx);
      count_launch();
    }
    int64_t per_item = 1;
    for (int a = 0; a < k.D; ++a) per_item *= k.a.trgt_size[a];
    k.a.det_acc = acc;
    k.a.det_max = mx;
    k.a.det_bound = static_cast<double>(per_item) * (mode == ppk::K_KD ? 2.0 * k.D : 1.0);
    k.a.out = nullptr;
    k.a.out_sN = cs[0];
    k.a.out_sC = cs[1];
    for (int a = 0; a < 3; ++a) k.a.out_s[a] = a < k.D ? cs[2 + a] : 0;
    if ((rc = run(k, mode, wide, st))) return rc;
    return det_finalize_to(acc, out, mx, k.a.det_bound, st);
  }
  // Vectorised scatter: 3-D, 2-4 channels, orders >= 2 with a compile-time
  // kernel (float32: all, bfloat16: cubic), 32-bit offsets, not
  // deterministic, a caller workspace large enough and 16-byte aligned.
  // Contributions go to a channel-interleaved float accumulator, one vector
  // reduction per tap, and are stored to `out` afterwards.
  const int iso = iso_order(k.D, k.order);
  const int CP = vec_slots(k.a.C);
  const bool spec = (out->dtype == PP_FLOAT32 && iso >= 0) || (out->dtype == PP_BFLOAT16 && iso == 3);
  if (k.D == 3 && CP > 0 && iso >= 2 && spec && !wide && !det && ppk::lanes_enabled() && ws &&
      ws_bytes >= scatter_ws_vec(out, flags) && reinterpret_cast<uintptr_t>(ws) % 16 == 0 &&
      fits32(numel(out) / k.a.C * CP)) {
    // the lane-split cubic push runs fastest in the grid's own order (1.69
    // vs 1.89 ms on config 2); the other scatters keep the sample order
    if (mode == ppk::K_PUSH && iso == 3 && !k.a.brick_start) k.a.perm = nullptr;
    float* acc = static_cast<float*>(ws);
    const int64_t vox = numel(out) / k.a.C;
    if ((rc = cuda_check(cudaMemsetAsync(acc, 0, static_cast<size_t>(vox) * CP * 4, st), "workspace clear"))) return rc;
    const int64_t V = vox / out->sizes[0];
    k.a.out = acc;
    k.a.out_sN = V * CP;
    k.a.out_sC = 1;
    k.a.out_s[2] = CP;
    k.a.out_s[1] = out->sizes[4] * CP;
    k.a.out_s[0] = out->sizes[3] * out->sizes[4] * CP;
    k.a.flags |= ppk::F_VEC;
    if ((rc = run(k, mode, wide, st))) return rc;
    return store_interleaved_to(acc, out, CP, st);
  }
  float* acc = nullptr;
  if (half) {
    acc = static_cast<float*>(ws);
    if ((rc = cuda_check(cudaMemsetAsync(acc, 0, numel(out) * 4, st), "workspace clear"))) return rc;
    k.a.out = acc;
    k.a.out_sN = cs[0];
    k.a.out_sC = cs[1];
    for (int a = 0; a < 3; ++a) k.a.out_s[a] = a < k.D ? cs[2 + a] : 0;
  } else {
    if ((rc = zero_fill(out, st))) return rc;
    k.a.out = out->data;
    set_image(out, k.D, k.a.out_sN, k.a.out_sC, k.a.out_s);
  }
  if ((rc = run(k, mode, wide, st))) return rc;
  if (half) return store_f32(acc, out, st);
  return PP_OK;
}

int pp_grid_push(const pp_tensor* input, const pp_tensor* grid, const pp_tensor* out,
                 const pp_options* opt, void* stream, void* workspace, size_t workspace_bytes) {
  Call k;
  int rc = prepare(k, grid, opt);
  if (rc) return rc;
  if ((rc = check_image(input, "input", k.D, grid->dtype))) return rc;
  // pushpull.cpp:131-150: input spatial size must match the grid's
  for (int a = 0; a < k.D; ++a)
    if (input->sizes[2 + a] != grid->sizes[1 + a] || input->sizes[0] != grid->sizes[0])
      return fail(PP_ERR_ARG, "(): expected input and grid to have same batch, width, height and (optionally) depth sizes");
  if ((rc = check_tensor(out, "output"))) return rc;
  if (out->ndim != k.D + 2 || out->sizes[0] != grid->sizes[0] || out->sizes[1] != input->sizes[1])
    return fail(PP_ERR_ARG, "(): output must be (N, C, *shape)");
  for (int i = 2; i < out->ndim; ++i)
    if (out->sizes[i] <= 0) return fail(PP_ERR_ARG, "(): expected non-empty output shape");
  if (out->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): output dtype must match input");
  k.dtype = input->dtype;
  k.a.trgt = input->data;
  k.a.C = input->sizes[1];
  set_image(input, k.D, k.a.trgt_sN, k.a.trgt_sC, k.a.trgt_s);
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? out->sizes[2 + a] : 1;
  return scatter_into(k, ppk::K_PUSH, out, input, need_wide(k, {input, out}), opt->flags, workspace,
                      workspace_bytes, static_cast<cudaStream_t>(stream));
}

int pp_grid_count(const pp_tensor* grid, const pp_tensor* out, const pp_options* opt, void* stream,
                  void* workspace, size_t workspace_bytes) {
  Call k;
  int rc = prepare(k, grid, opt);
  if (rc) return rc;
  if ((rc = check_tensor(out, "output"))) return rc;
  if (out->ndim != k.D + 2 || out->sizes[0] != grid->sizes[0] || out->sizes[1] != 1)
    return fail(PP_ERR_ARG, "(): output must be (N, 1, *shape)");
  for (int i = 2; i < out->ndim; ++i)
    if (out->sizes[i] <= 0) return fail(PP_ERR_ARG, "(): expected non-empty output shape");
  if (out->dtype != grid->dtype) return fail(PP_ERR_DTYPE, "(): count output must have the grid dtype");
  k.dtype = grid->dtype;
  k.a.C = 1;
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? out->sizes[2 + a] : 1;
  return scatter_into(k, ppk::K_COUNT, out, nullptr, need_wide(k, {out}), opt->flags, workspace,
                      workspace_bytes, static_cast<cudaStream_t>(stream));
}

static int check_ggrad(const pp_tensor* gg, const pp_tensor* grid) {
  int rc = check_tensor(gg, "grad_grid");
  if (rc) return rc;
  if ((rc = check_same_sizes(gg, grid->sizes, grid->ndim, "grad_grid"))) return rc;
  if (gg->dtype != grid->dtype) return fail(PP_ERR_DTYPE, "(): grad_grid must have the grid dtype");
  return PP_OK;
}

int pp_grid_pull_backward(const pp_tensor* grad, const pp_tensor* input, const pp_tensor* grid,
                          const pp_tensor* grad_input, const pp_tensor* grad_grid,
                          const pp_options* opt, void* stream, void* workspace, size_t workspace_bytes) {
  Call k;
  int rc = prepare(k, grid, opt);
  if (rc) return rc;
  if ((rc = check_image(input, "input", k.D, grid->dtype))) return rc;
  if ((rc = check_tensor(grad, "grad"))) return rc;
  int64_t gsz[5] = {grid->sizes[0], input->sizes[1], 1, 1, 1};
  for (int a = 0; a < k.D; ++a) gsz[2 + a] = grid->sizes[1 + a];
  if ((rc = check_same_sizes(grad, gsz, k.D + 2, "grad"))) return rc;
  if (grad->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): grad dtype must match input");
  if (grad_input && (rc = check_same_sizes(grad_input, input->sizes, input->ndim, "grad_input"))) return rc;
  if (grad_input && grad_input->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): grad_input dtype must match input");
  if (grad_grid && (rc = check_ggrad(grad_grid, grid))) return rc;
  if (!grad_input && !grad_grid) return PP_OK;
  k.dtype = input->dtype;
  k.a.C = input->sizes[1];
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? input->sizes[2 + a] : 1;
  k.a.src = input->data;
  set_image(input, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.trgt = grad->data;
  set_image(grad, k.D, k.a.trgt_sN, k.a.trgt_sC, k.a.trgt_s);
  const bool wide = need_wide(k, {input, grad, grad_input});
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (grad_grid) {
    k.a.gg = grad_grid->data;
    set_grid(grad_grid, k.D, k.a.gg_sN, k.a.gg_s, k.a.gg_sD);
    k.a.flags = ppk::F_GRAD | (grad_input ? ppk::F_A : 0);
    if (!grad_input) return run(k, ppk::K_PUSHGRAD, wide, st);
    return scatter_into(k, ppk::K_PUSHGRAD, grad_input, grad, wide, opt->flags, workspace, workspace_bytes, st);
  }
  return scatter_into(k, ppk::K_PUSH, grad_input, grad, wide, opt->flags, workspace, workspace_bytes, st);
}

int pp_grid_push_backward(const pp_tensor* grad, const pp_tensor* input, const pp_tensor* grid,
                          const pp_tensor* grad_input, const pp_tensor* grad_grid,
                          const pp_options* opt, void* stream) {
  Call k;
  int rc = prepare(k, grid, opt);
  if (rc) return rc;
  if ((rc = check_image(input, "input", k.D, grid->dtype))) return rc;
  if ((rc = check_image(grad, "grad", k.D, grid->dtype))) return rc;
  if (grad->sizes[0] != grid->sizes[0] || grad->sizes[1] != input->sizes[1])
    return fail(PP_ERR_ARG, "(): grad must be (N, C, *shape)");
  if (grad->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): grad dtype must match input");
  if (grad_input && (rc = check_same_sizes(grad_input, input->sizes, input->ndim, "grad_input"))) return rc;
  if (grad_input && grad_input->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): grad_input dtype must match input");
  if (grad_grid && (rc = check_ggrad(grad_grid, grid))) return rc;
  if (!grad_input && !grad_grid) return PP_OK;
  k.dtype = input->dtype;
  k.a.C = input->sizes[1];
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? grad->sizes[2 + a] : 1;
  k.a.src = grad->data;
  set_image(grad, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.trgt = input->data;
  set_image(input, k.D, k.a.trgt_sN, k.a.trgt_sC, k.a.trgt_s);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (grad_input) {
    k.a.out = grad_input->data;
    set_image(grad_input, k.D, k.a.out_sN, k.a.out_sC, k.a.out_s);
  }
  const bool wide = need_wide(k, {grad, input, grad_input});
  if (grad_grid) {
    k.a.gg = grad_grid->data;
    set_grid(grad_grid, k.D, k.a.gg_sN, k.a.gg_s, k.a.gg_sD);
    k.a.flags = ppk::F_GRAD | (grad_input ? ppk::F_A : 0);
    return run(k, ppk::K_PULLGRAD, wide, st);
  }
  return run(k, ppk::K_PULL, wide, st);
}

int pp_grid_count_backward(const pp_tensor* grad, const pp_tensor* grid, const pp_tensor* grad_grid,
                           const pp_options* opt, void* stream) {
  Call k;
  int rc = prepare(k, grid, opt);
  if (rc) return rc;
  if ((rc = check_image(grad, "grad", k.D, grid->dtype))) return rc;
  if (grad->sizes[0] != grid->sizes[0] || grad->sizes[1] != 1)
    return fail(PP_ERR_ARG, "(): grad must be (N, 1, *shape)");
  if (grad->dtype != grid->dtype) return fail(PP_ERR_DTYPE, "(): grad must have the grid dtype");
  if ((rc = check_ggrad(grad_grid, grid))) return rc;
  k.dtype = grid->dtype;
  k.a.C = 1;
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? grad->sizes[2 + a] : 1;
  k.a.src = grad->data;
  set_image(grad, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.gg = grad_grid->data;
  set_grid(grad_grid, k.D, k.a.gg_sN, k.a.gg_s, k.a.gg_sD);
  k.a.flags = ppk::F_GRAD | ppk::F_NOTRGT;
  return run(k, ppk::K_PUSHGRAD, need_wide(k, {grad}), static_cast<cudaStream_t>(stream));
}

int pp_grid_grad_backward(const pp_tensor* grad, const pp_tensor* input, const pp_tensor* grid,
                          const pp_tensor* grad_input, const pp_tensor* grad_grid,
                          const pp_options* opt, void* stream, void* workspace, size_t workspace_bytes) {
  Call k;
  int rc = prepare(k, grid, opt);
  if (rc) return rc;
  if ((rc = check_image(input, "input", k.D, grid->dtype))) return rc;
  if ((rc = check_tensor(grad, "grad"))) return rc;
  int64_t gsz[6] = {grid->sizes[0], input->sizes[1], 1, 1, 1, 1};
  for (int a = 0; a < k.D; ++a) gsz[2 + a] = grid->sizes[1 + a];
  gsz[2 + k.D] = k.D;
  if ((rc = check_same_sizes(grad, gsz, k.D + 3, "grad"))) return rc;
  if (grad->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): grad dtype must match input");
  if (grad_input && (rc = check_same_sizes(grad_input, input->sizes, input->ndim, "grad_input"))) return rc;
  if (grad_input && grad_input->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): grad_input dtype must match input");
  if (grad_grid && (rc = check_ggrad(grad_grid, grid))) return rc;
  if (!grad_input && !grad_grid) return PP_OK;
  k.dtype = input->dtype;
  k.a.C = input->sizes[1];
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? input->sizes[2 + a] : 1;
  k.a.src = input->data;
  set_image(input, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.trgt = grad->data;
  set_image(grad, k.D, k.a.trgt_sN, k.a.trgt_sC, k.a.trgt_s);
  k.a.trgt_sK = grad->strides[2 + k.D];
  const bool wide = need_wide(k, {input, grad, grad_input});
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k.a.flags = (grad_grid ? ppk::F_GRAD : 0) | (grad_input ? ppk::F_A : 0);
  if (grad_grid) {
    k.a.gg = grad_grid->data;
    set_grid(grad_grid, k.D, k.a.gg_sN, k.a.gg_s, k.a.gg_sD);
  }
  if (!grad_input) return run(k, ppk::K_KD, wide, st);
  return scatter_into(k, ppk::K_KD, grad_input, grad, wide, opt->flags, workspace, workspace_bytes, st);
}

// Fused push(pull(input)): out (laid out freely, input's shape) =
// P^T P input for the sampling points of `grid`.  No counterpart in the
// reference (where it is grid_pull then grid_push on the same grid).
int pp_grid_pull_push(const pp_tensor* input, const pp_tensor* grid, const pp_tensor* out,
                      const pp_options* opt, void* stream, void* workspace, size_t workspace_bytes) {
  Call k;
  int rc = prepare(k, grid, opt);
  if (rc) return rc;
  if ((rc = check_image(input, "input", k.D, grid->dtype))) return rc;
  if (input->sizes[0] != grid->sizes[0])
    return fail(PP_ERR_ARG, "(): expected input and grid to have the same batch size");
  if ((rc = check_tensor(out, "output"))) return rc;
  if ((rc = check_same_sizes(out, input->sizes, input->ndim, "output"))) return rc;
  if (out->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): output dtype must match input");
  k.dtype = input->dtype;
  k.a.C = input->sizes[1];
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? input->sizes[2 + a] : 1;
  k.a.src = input->data;
  set_image(input, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  return scatter_into(k, ppk::K_PP, out, input, need_wide(k, {input, out}), opt->flags, workspace,
                      workspace_bytes, static_cast<cudaStream_t>(stream));
}

// Backward of pp_grid_pull_push for a loss gradient `grad` (input's shape
// and strides): grad_input = P^T P grad, grad_grid as described in
// pp_kernels.cuh (K_PP_BWD).  Either output may be NULL.
int pp_grid_pull_push_backward(const pp_tensor* grad, const pp_tensor* input, const pp_tensor* grid,
                               const pp_tensor* grad_input, const pp_tensor* grad_grid, const pp_options* opt,
                               void* stream, void* workspace, size_t workspace_bytes) {
  Call k;
  int rc = prepare(k, grid, opt);
  if (rc) return rc;
  if ((rc = check_image(input, "input", k.D, grid->dtype))) return rc;
  if (input->sizes[0] != grid->sizes[0])
    return fail(PP_ERR_ARG, "(): expected input and grid to have the same batch size");
  if ((rc = check_tensor(grad, "grad"))) return rc;
  if ((rc = check_same_sizes(grad, input->sizes, input->ndim, "grad"))) return rc;
  if (grad->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): grad dtype must match input");
  for (int i = 0; i < input->ndim; ++i)
    if (input->sizes[i] > 1 && grad->strides[i] != input->strides[i])
      return fail(PP_ERR_UNSUPPORTED, "(): fused pull-push backward needs grad laid out like the input");
  if (grad_input && (rc = check_same_sizes(grad_input, input->sizes, input->ndim, "grad_input"))) return rc;
  if (grad_input && grad_input->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): grad_input dtype must match input");
  if (grad_grid && (rc = check_ggrad(grad_grid, grid))) return rc;
  if (!grad_input && !grad_grid) return PP_OK;
  k.dtype = input->dtype;
  k.a.C = input->sizes[1];
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? input->sizes[2 + a] : 1;
  k.a.src = input->data;
  set_image(input, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.trgt = grad->data;
  k.a.flags = (grad_grid ? ppk::F_GRAD : 0) | (grad_input ? ppk::F_A : 0);
  if (grad_grid) {
    k.a.gg = grad_grid->data;
    set_grid(grad_grid, k.D, k.a.gg_sN, k.a.gg_s, k.a.gg_sD);
  }
  const bool wide = need_wide(k, {input, grad, grad_input});
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!grad_input) return run(k, ppk::K_PP_BWD, wide, st);
  return scatter_into(k, ppk::K_PP_BWD, grad_input, grad, wide, opt->flags, workspace, workspace_bytes, st);
}

// Displacement self-composition, the step of scaling-and-squaring
// (nitorch/spatial/_svf.py:85-94 with _pull_vel, :323-362):
//   out = u + pull(u, id + u)
// u, out: (N, *spatial, D) fields, component last (any strides); the pull
// reads the components of u as its D channels.  out must not alias u.
static void field_as_image(const pp_tensor* f, int D, int64_t& sN, int64_t& sC, int64_t s[3]) {
  sN = f->strides[0];
  sC = f->strides[1 + D];
  for (int a = 0; a < 3; ++a) s[a] = a < D ? f->strides[1 + a] : 0;
}

int pp_svf_compose(const pp_tensor* disp, const pp_tensor* out, const pp_options* opt, void* stream) {
  Call k;
  int rc = prepare(k, disp, opt);
  if (rc) return rc;
  if ((rc = check_tensor(out, "output"))) return rc;
  if ((rc = check_same_sizes(out, disp->sizes, disp->ndim, "output"))) return rc;
  if (out->dtype != disp->dtype) return fail(PP_ERR_DTYPE, "(): output dtype must match the field");
  if (out->data == disp->data) return fail(PP_ERR_ARG, "(): output must not alias the field");
  k.a.perm = nullptr;
  k.dtype = disp->dtype;
  k.a.C = k.D;
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? disp->sizes[1 + a] : 1;
  k.a.src = disp->data;
  field_as_image(disp, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.out = out->data;
  field_as_image(out, k.D, k.a.out_sN, k.a.out_sC, k.a.out_s);
  k.a.flags = ppk::F_IDGRID | ppk::F_ADDSELF;
  if (k.D == 3 && iso_order(k.D, k.order) == 1 && ppk::lanes_enabled()) {
    // 3-D linear float32: the dedicated composition kernel (svf_compose.cu)
    rc = svf_compose_linear3(disp, out, k.a.bound, k.a.extrapolate, static_cast<cudaStream_t>(stream));
    if (rc != PP_ERR_UNSUPPORTED) return rc;
  }
  return run(k, ppk::K_PULL, need_wide(k, {disp, out}), static_cast<cudaStream_t>(stream));
}

// Its backward: grad_disp = g + push(g, id + u) + sum_c g_c grad(u_c)(id + u),
// the gradient of <g, u + pull(u, id + u)> with respect to u, in one pass
// (the push and the point's own terms accumulate atomically).
static size_t round256(size_t b) { return (b + 255) / 256 * 256; }

size_t pp_svf_workspace_bytes(const pp_tensor* disp, int32_t flags) {
  if (!disp || disp->ndim < 3 || disp->ndim > 5 || disp->sizes[disp->ndim - 1] != disp->ndim - 2) return 0;
  const int64_t n = numel(disp);
  if (flags & PP_DETERMINISTIC) {
    // max |grad| (256 B), the push part as int64 fixed point, the identity
    // and grid-gradient terms of every voxel in the accumulation type
    if (disp->dtype != PP_FLOAT32 && disp->dtype != PP_FLOAT64) return 0;
    return 256 + round256(static_cast<size_t>(n) * 8) + round256(static_cast<size_t>(n) * (disp->dtype == PP_FLOAT64 ? 8 : 4));
  }
  if (disp->ndim != 5 || disp->dtype != PP_FLOAT32) return 0;
  return round256(static_cast<size_t>(n / 3) * 16);
}

int pp_svf_compose_backward(const pp_tensor* grad, const pp_tensor* disp, const pp_tensor* grad_disp,
                            const pp_options* opt, void* stream, void* workspace, size_t workspace_bytes) {
  Call k;
  int rc = prepare(k, disp, opt);
  if (rc) return rc;
  const bool det = (opt->flags & PP_DETERMINISTIC) != 0;
  if ((rc = check_tensor(grad, "grad"))) return rc;
  if ((rc = check_same_sizes(grad, disp->sizes, disp->ndim, "grad"))) return rc;
  if ((rc = check_tensor(grad_disp, "grad_disp"))) return rc;
  if ((rc = check_same_sizes(grad_disp, disp->sizes, disp->ndim, "grad_disp"))) return rc;
  if (grad->dtype != disp->dtype || grad_disp->dtype != disp->dtype)
    return fail(PP_ERR_DTYPE, "(): grad and grad_disp must have the field's dtype");
  if (grad_disp->data == disp->data || grad_disp->data == grad->data)
    return fail(PP_ERR_ARG, "(): grad_disp must not alias its inputs");
  k.a.perm = nullptr;
  k.dtype = disp->dtype;
  k.a.C = k.D;
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? disp->sizes[1 + a] : 1;
  k.a.src = disp->data;
  field_as_image(disp, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.trgt = grad->data;
  field_as_image(grad, k.D, k.a.trgt_sN, k.a.trgt_sC, k.a.trgt_s);
  k.a.out = grad_disp->data;
  field_as_image(grad_disp, k.D, k.a.out_sN, k.a.out_sC, k.a.out_s);
  k.a.flags = ppk::F_A | ppk::F_GRAD | ppk::F_IDGRID | ppk::F_ADDSELF;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool wide = need_wide(k, {disp, grad, grad_disp});
  const int iso = iso_order(k.D, k.order);
  if (det) {
    // Deterministic: the push of grad into int64 fixed point (order-free
    // integer atomics), the identity and grid-gradient terms of each voxel
    // stored by the voxel's own point into a separate buffer, the two added
    // by the finalize pass.
    const size_t dneed = pp_svf_workspace_bytes(disp, PP_DETERMINISTIC);
    if (!dneed) return fail(PP_ERR_DTYPE, "(): the deterministic self-composition backward needs float32/64 fields");
    if (!workspace || workspace_bytes < dneed || reinterpret_cast<uintptr_t>(workspace) % 16 != 0)
      return fail(PP_ERR_WORKSPACE, "(): the deterministic mode needs %zu bytes of 16-byte aligned workspace", dneed);
    const int64_t n = numel(disp);
    unsigned char* w = static_cast<unsigned char*>(workspace);
    unsigned int* mx = reinterpret_cast<unsigned int*>(w);
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(w + 256);
    void* self = w + 256 + round256(static_cast<size_t>(n) * 8);
    if ((rc = cuda_check(cudaMemsetAsync(w, 0, 256 + static_cast<size_t>(n) * 8, st), "workspace clear"))) return rc;
    if ((rc = det_absmax_of(grad, mx, st))) return rc;
    // accumulators in the field's own (N, *spatial, D) order
    int64_t per_item = 1;
    for (int a = 0; a < k.D; ++a) per_item *= disp->sizes[1 + a];
    k.a.det_acc = acc;
    k.a.det_max = mx;
    k.a.det_bound = static_cast<double>(per_item);
    k.a.aux = self;
    k.a.out = nullptr;
    k.a.out_sN = per_item * k.D;
    k.a.out_sC = 1;
    {
      int64_t s = k.D;
      for (int a = 2; a >= 0; --a) {
        k.a.out_s[a] = a < k.D ? s : 0;
        if (a < k.D) s *= disp->sizes[1 + a];
      }
    }
    if ((rc = run(k, ppk::K_PUSHGRAD, wide, st))) return rc;
    return det_finalize_to(acc, grad_disp, mx, k.a.det_bound, st, self);
  }
  const size_t need = pp_svf_workspace_bytes(disp, 0);
  if (need && workspace && workspace_bytes >= need && reinterpret_cast<uintptr_t>(workspace) % 16 == 0 &&
      (iso == 1 || iso == 3) && !wide && ppk::lanes_enabled() && grad_disp->dtype == PP_FLOAT32 &&
      fits32(numel(disp) / 3 * 4)) {
    // channel-interleaved accumulator (4 slots per voxel), one vector
    // reduction per tap, then copied to the field
    float* acc = static_cast<float*>(workspace);
    const int64_t vox = numel(disp) / 3, V = vox / disp->sizes[0];
    if ((rc = cuda_check(cudaMemsetAsync(acc, 0, static_cast<size_t>(vox) * 16, st), "workspace clear"))) return rc;
    k.a.out = acc;
    k.a.out_sN = V * 4;
    k.a.out_sC = 1;
    k.a.out_s[2] = 4;
    k.a.out_s[1] = disp->sizes[3] * 4;
    k.a.out_s[0] = disp->sizes[2] * disp->sizes[3] * 4;
    k.a.flags |= ppk::F_VEC;
    // 3-D linear: the dedicated kernel (svf_compose.cu), else the lane-split one
    rc = iso == 1 ? svf_compose_backward_linear3(grad, disp, acc, k.a.bound, k.a.extrapolate, st) : PP_ERR_UNSUPPORTED;
    if (rc == PP_ERR_UNSUPPORTED) rc = run(k, ppk::K_PUSHGRAD, wide, st);
    if (rc) return rc;
    // grad_disp given as the first three slots of the workspace itself: done
    bool in_place = grad_disp->data == workspace;
    {
      const int64_t want[5] = {V * 4, disp->sizes[2] * disp->sizes[3] * 4, disp->sizes[3] * 4, 4, 1};
      for (int i = 0; i < 5 && in_place; ++i) in_place = grad_disp->sizes[i] == 1 || grad_disp->strides[i] == want[i];
    }
    return in_place ? PP_OK : store_field_from4(acc, grad_disp, st);
  }
  if ((rc = zero_fill(grad_disp, st))) return rc;
  return run(k, ppk::K_PUSHGRAD, wide, st);
}

// ---------------------------------------------------------------------------
// Affine sampling without a materialised grid (resize / reslice):
// nitorch/spatial/_grid.py builds affine_grid(mat, shape) (:579-615) and
// calls grid_pull on it (resize :618-754, reslice :860-914).  Here the
// kernels compute the coordinate A [sub; 1] of every grid point.
// ---------------------------------------------------------------------------

// mat: (N, D, D+1) or (N, D+1, D+1), rows of D+1 contiguous entries.
static int check_matrix(const pp_tensor* mat, int D, int64_t N, int dtype) {
  int rc = check_tensor(mat, "affine");
  if (rc) return rc;
  if (mat->ndim != 3 || mat->sizes[2] != D + 1 || (mat->sizes[1] != D && mat->sizes[1] != D + 1))
    return fail(PP_ERR_ARG, "(): expected affine matrices of shape (N, %d[+1], %d)", D, D + 1);
  if (mat->sizes[0] != N) return fail(PP_ERR_ARG, "(): expected one affine matrix per batch item");
  if (mat->strides[2] != 1 || (mat->sizes[1] > 1 && mat->strides[1] != D + 1))
    return fail(PP_ERR_ARG, "(): affine matrices must have contiguous rows");
  if (mat->dtype != dtype) return fail(PP_ERR_DTYPE, "(): affine matrices must have the grid dtype");
  return PP_OK;
}

// Call set-up of an affine op whose sampling lattice is `lat` (N, C, *shape).
static int prepare_affine(Call& k, const pp_tensor* lat, const pp_tensor* mat, const pp_options* opt,
                          int image_dtype) {
  int rc = check_tensor(lat, "image");
  if (rc) return rc;
  if (lat->ndim < 3 || lat->ndim > 5) return fail(PP_ERR_ARG, "(): expected a 1D, 2D or 3D image");
  k.D = lat->ndim - 2;
  if ((rc = read_options(opt, k.D, k.bound, k.order))) return rc;
  const int gdt = grid_dtype_for(image_dtype);
  if ((rc = check_matrix(mat, k.D, lat->sizes[0], gdt))) return rc;
  for (int a = 0; a < 3; ++a) { k.a.bound[a] = k.bound[a]; k.a.order[a] = k.order[a]; }
  k.a.extrapolate = opt->extrapolate;
  k.a.perm = nullptr;
  k.a.grid = mat->data;
  k.a.grid_sN = mat->strides[0];
  k.a.N = lat->sizes[0];
  int64_t nv = lat->sizes[0];
  for (int a = 0; a < 3; ++a) {
    k.a.trgt_size[a] = a < k.D ? lat->sizes[2 + a] : 1;
    if (k.a.trgt_size[a] <= 0) return fail(PP_ERR_ARG, "(): expected non-empty spatial dimensions");
    nv *= k.a.trgt_size[a];
  }
  k.a.nvox = nv;
  k.a.flags = ppk::F_AFFINE;
  return PP_OK;
}

int pp_affine_pull(const pp_tensor* input, const pp_tensor* mat, const pp_tensor* out, const pp_options* opt,
                   void* stream) {
  Call k;
  int rc = check_tensor(input, "input");
  if (rc) return rc;
  if ((rc = prepare_affine(k, out, mat, opt, input->dtype))) return rc;
  if (input->ndim != k.D + 2 || input->sizes[0] != out->sizes[0] || input->sizes[1] != out->sizes[1])
    return fail(PP_ERR_ARG, "(): expected input (N, C, *inshape) and output (N, C, *shape)");
  for (int i = 2; i < input->ndim; ++i)
    if (input->sizes[i] <= 0) return fail(PP_ERR_ARG, "(): expected non-empty input");
  if (out->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): output dtype must match input");
  k.dtype = input->dtype;
  k.a.C = input->sizes[1];
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? input->sizes[2 + a] : 1;
  k.a.src = input->data;
  set_image(input, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.out = out->data;
  set_image(out, k.D, k.a.out_sN, k.a.out_sC, k.a.out_s);
  return run(k, ppk::K_PULL, need_wide(k, {input, out}), static_cast<cudaStream_t>(stream));
}

// Adjoint of pp_affine_pull: out (N, C, *outshape) = push of `input`
// (N, C, *shape, sampled at A [sub; 1]).  Workspace: pp_push_workspace_bytes(out).
int pp_affine_push(const pp_tensor* input, const pp_tensor* mat, const pp_tensor* out, const pp_options* opt,
                   void* stream, void* workspace, size_t workspace_bytes) {
  Call k;
  int rc = check_tensor(out, "output");
  if (rc) return rc;
  if ((rc = prepare_affine(k, input, mat, opt, input->dtype))) return rc;
  if (out->ndim != k.D + 2 || out->sizes[0] != input->sizes[0] || out->sizes[1] != input->sizes[1])
    return fail(PP_ERR_ARG, "(): output must be (N, C, *outshape)");
  for (int i = 2; i < out->ndim; ++i)
    if (out->sizes[i] <= 0) return fail(PP_ERR_ARG, "(): expected non-empty output shape");
  if (out->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): output dtype must match input");
  k.dtype = input->dtype;
  k.a.trgt = input->data;
  k.a.C = input->sizes[1];
  set_image(input, k.D, k.a.trgt_sN, k.a.trgt_sC, k.a.trgt_s);
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? out->sizes[2 + a] : 1;
  return scatter_into(k, ppk::K_PUSH, out, input, need_wide(k, {input, out}), opt->flags, workspace,
                      workspace_bytes, static_cast<cudaStream_t>(stream));
}

size_t pp_affine_grad_workspace_bytes(const pp_tensor* grad) {
  if (!grad || grad->ndim < 3 || grad->ndim > 5) return 0;
  const int D = grad->ndim - 2;
  int64_t n = grad->sizes[0] * D;
  for (int i = 2; i < grad->ndim; ++i) n *= grad->sizes[i];
  return ((static_cast<size_t>(n) * 4 + 255) / 256) * 256;
}

}  // extern "C"

namespace {
// grad_mat[n, d, e] += sum over the grid points p of item n of
// gg[p, d] * h_e(p), h = (sub_0, .., sub_{D-1}, 1): one partial sum per
// CTA (block reduction in shared memory), then D (D+1) atomics per CTA.
template <int D>
__global__ void __launch_bounds__(256) affine_reduce(const float* gg, int64_t P, int64_t s1, int64_t s2,
                                                     float* gm, int64_t gm_sN, int64_t gm_sR) {
  constexpr int K = D * (D + 1);
  __shared__ float red[K][8];
  const int64_t n = blockIdx.y;
  float acc[K];
#pragma unroll
  for (int q = 0; q < K; ++q) acc[q] = 0.f;
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < P;
       p += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float h[D + 1];
    int64_t r = p;  // lattice index, last axis fastest
    if constexpr (D == 3) {
      h[2] = static_cast<float>(r % s2); r /= s2;
      h[1] = static_cast<float>(r % s1); r /= s1;
    } else if constexpr (D == 2) {
      h[1] = static_cast<float>(r % s1); r /= s1;
    }
    h[0] = static_cast<float>(r);
    h[D] = 1.f;
    const float* g = gg + (n * P + p) * D;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const float gd = g[d];
#pragma unroll
      for (int e = 0; e <= D; ++e) acc[d * (D + 1) + e] = fmaf(gd, h[e], acc[d * (D + 1) + e]);
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    float v = acc[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    float v = 0.f;
    for (int w = 0; w < 8; ++w) v += red[threadIdx.x][w];
    const int d = threadIdx.x / (D + 1), e = threadIdx.x % (D + 1);
    atomicAdd(gm + n * gm_sN + d * gm_sR + e, v);
  }
}
}  // namespace

extern "C" {

// Gradient of <grad, affine_pull(input, mat)> with respect to the first D
// rows of each matrix: per grid point the gradient of the pulled values with
// respect to the coordinate (sum_c grad_c * d/dx interp(input_c)), then
// grad_mat[n] = sum_p g(p) [sub_p; 1]^T.  grad_mat: (N, D, D+1) float32,
// contiguous rows; workspace: pp_affine_grad_workspace_bytes(grad) bytes.
// float32 / bfloat16 / float16 images only (float32 grid arithmetic).
int pp_affine_grad_matrix(const pp_tensor* grad, const pp_tensor* input, const pp_tensor* mat,
                          const pp_tensor* grad_mat, const pp_options* opt, void* stream, void* workspace,
                          size_t workspace_bytes) {
  Call k;
  int rc = check_tensor(input, "input");
  if (rc) return rc;
  if (input->dtype == PP_FLOAT64) return fail(PP_ERR_DTYPE, "(): affine matrix gradients are float32 only");
  if ((rc = prepare_affine(k, grad, mat, opt, input->dtype))) return rc;
  if (input->ndim != k.D + 2 || input->sizes[0] != grad->sizes[0] || input->sizes[1] != grad->sizes[1])
    return fail(PP_ERR_ARG, "(): expected input (N, C, *inshape) and grad (N, C, *shape)");
  if (grad->dtype != input->dtype) return fail(PP_ERR_DTYPE, "(): grad dtype must match input");
  if ((rc = check_tensor(grad_mat, "grad_affine"))) return rc;
  if (grad_mat->ndim != 3 || grad_mat->sizes[0] != grad->sizes[0] || grad_mat->sizes[1] != k.D ||
      grad_mat->sizes[2] != k.D + 1 || grad_mat->strides[2] != 1 || grad_mat->dtype != PP_FLOAT32)
    return fail(PP_ERR_ARG, "(): expected a float32 (N, %d, %d) grad_affine with contiguous rows", k.D, k.D + 1);
  const size_t need = pp_affine_grad_workspace_bytes(grad);
  if (!workspace || workspace_bytes < need)
    return fail(PP_ERR_WORKSPACE, "(): the affine gradient needs %zu bytes of workspace", need);
  k.dtype = input->dtype;
  k.a.C = input->sizes[1];
  for (int a = 0; a < 3; ++a) k.a.src_size[a] = a < k.D ? input->sizes[2 + a] : 1;
  k.a.src = input->data;
  set_image(input, k.D, k.a.src_sN, k.a.src_sC, k.a.src_s);
  k.a.trgt = grad->data;
  set_image(grad, k.D, k.a.trgt_sN, k.a.trgt_sC, k.a.trgt_s);
  // per-point coordinate gradients (N, *shape, D), contiguous
  float* gg = static_cast<float*>(workspace);
  const int64_t P = k.a.nvox / k.a.N;
  k.a.gg = gg;
  k.a.gg_sN = P * k.D;
  k.a.gg_sD = 1;
  {
    int64_t sd = k.D;
    for (int a = k.D - 1; a >= 0; --a) { k.a.gg_s[a] = sd; sd *= k.a.trgt_size[a]; }
    for (int a = k.D; a < 3; ++a) k.a.gg_s[a] = 0;
  }
  k.a.flags |= ppk::F_GRAD;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((rc = run(k, ppk::K_PULLGRAD, need_wide(k, {input, grad}), st))) return rc;
  if ((rc = zero_fill(grad_mat, st))) return rc;
  const int64_t blocks = std::min<int64_t>((P + 255) / 256, 148 * 4);
  dim3 g(static_cast<unsigned>(blocks), static_cast<unsigned>(k.a.N), 1);
  float* gm = static_cast<float*>(grad_mat->data);
  if (k.D == 3)
    affine_reduce<3><<<g, 256, 0, st>>>(gg, P, k.a.trgt_size[1], k.a.trgt_size[2], gm, grad_mat->strides[0],
                                        grad_mat->strides[1]);
  else if (k.D == 2)
    affine_reduce<2><<<g, 256, 0, st>>>(gg, P, k.a.trgt_size[1], 1, gm, grad_mat->strides[0],
                                        grad_mat->strides[1]);
  else
    affine_reduce<1><<<g, 256, 0, st>>>(gg, P, 1, 1, gm, grad_mat->strides[0], grad_mat->strides[1]);
  count_launch();
  return cuda_check(cudaGetLastError(), "affine gradient reduction");
}

}  // extern "C"
