// Interpolating B-spline prefilter (spline_coeff / spline_coeff_nd).
//
// Arithmetic restated from the vendored prefilter nitorch/_C/_ts/coeff.py
// (Unser-Aldroubi-Eden recursive filtering): gain (coeff.py:61-65), one
// causal and one anti-causal first-order recursion per pole (coeff.py:
// 254-281), initial / final conditions per boundary (coeff.py:69-251).
//
// B200 mapping: one line per thread, LINES lines per CTA staged in shared
// memory through a cooperative, coalesced load (whichever axis is filtered),
// so that the sequential recursions run out of shared memory and the global
// traffic is one read and one write of the volume per axis.  The recursions
// run in float (double for double storage); the initial / final condition
// sums are evaluated in double.  Lines longer than the shared-memory budget
// fall back to the same recursion directly on global memory.
#include "pp_capi_internal.cuh"

namespace {

constexpr int LINES = 128;    // lines per CTA: one per thread in the recursions
constexpr int THREADS = 128;
constexpr int UNROLL = 8;     // 16-bit storage: loads in flight per thread while staging

struct LineArgs {
  const void* in;
  void* out;
  int64_t nlines;
  int64_t n;          // line length
  int64_t in_st, out_st;  // element stride along the line
  int ndo;            // number of non-filtered dims
  int64_t osz[PP_MAX_DIM];     // their sizes (last fastest)
  int64_t ist[PP_MAX_DIM];     // their input strides
  int64_t ost[PP_MAX_DIM];     // their output strides
  int kind;           // 1 dct1, 2 dct2, 3 dft
  int npoles;
  double z[3];
  double gain;
  int line_major;     // 1: load element-major within a line (axis is the fastest)
};

__device__ __forceinline__ void line_base(const LineArgs& a, int64_t l, int64_t& bi, int64_t& bo) {
  bi = 0; bo = 0;
  for (int d = a.ndo - 1; d >= 0; --d) {
    const int64_t q = l / a.osz[d];
    const int64_t r = l - q * a.osz[d];
    bi += r * a.ist[d];
    bo += r * a.ost[d];
    l = q;
  }
}

__device__ __forceinline__ int64_t trunc_iter(double z) {
  return static_cast<int64_t>(ceil(-30.0 / log(fabs(z))));
}

// Accessors over one line: in global memory (any stride) or in the shared
// tile (element-major, one column per line, pitch = lines per CTA | 1).
template <class C>
struct LineRef {
  using value_type = C;
  using index_type = int64_t;
  C* p;
  int64_t st;
  __device__ __forceinline__ C& operator[](int64_t i) const { return p[i * st]; }
};

template <class C>
struct TileLine {
  using value_type = C;
  using index_type = int;
  C* p;
  int pitch;
  __device__ __forceinline__ C& operator[](int i) const { return p[i * pitch]; }
};

// Initial causal coefficient (coeff.py:69-170), double accumulation.  The
// samples are read as L[k] * g (g: the filter gain on the first pole's pass,
// 1 afterwards), so the gain pass costs no separate sweep.
template <class R, class C = typename R::value_type>
__device__ double initial(const R& L, int64_t n, int kind, double z, C g) {
  auto x = [&](int64_t k) { return static_cast<double>(L[k] * g); };
  if (kind == 2) {  // dct2 / replicate (coeff.py:137-170)
    const double zn = pow(z, static_cast<double>(n));
    const double zlast = zn * (1.0 + 1.0 / (z + zn * zn));
    double acc = x(0) + zlast * x(n - 1);
    // sum_{k=1}^{n-2} (z^k + z^(2n-1-k)) L[k]; both power series decay
    // geometrically, terms below 2^-64 of the leading one are dropped.
    const int64_t K = static_cast<int64_t>(ceil(-44.4 / log(fabs(z)))) + 1;
    const int64_t k1 = n - 2 < K ? n - 2 : K;
    double zk = z;
    for (int64_t k = 1; k <= k1; ++k, zk *= z) acc += zk * x(k);
    int64_t k2 = 2 * n - 1 - K;
    if (k2 < 1) k2 = 1;
    if (k2 <= n - 2) {
      double zq = pow(z, static_cast<double>(2 * n - 1 - k2));
      const double iz = 1.0 / z;
      for (int64_t k = k2; k <= n - 2; ++k, zq *= iz) acc += zq * x(k);
    }
    return acc * (z / (1.0 - zn * zn)) + x(0);
  }
  if (kind == 1) {  // dct1 / zero (coeff.py:94-134)
    const int64_t m = trunc_iter(z);
    if (m < n) {
      double acc = x(0), zk = z;
      for (int64_t k = 1; k < m; ++k, zk *= z) acc += zk * x(k);
      return acc;
    }
    const double zn = pow(z, static_cast<double>(n - 1));
    double acc = x(0) + zn * x(n - 1);
    double zk = z;
    for (int64_t k = 1; k < n - 1; ++k, zk *= z) acc += (zk + zn * zn / zk) * x(k);
    return acc / (1.0 - zn * zn);
  }
  // dft (coeff.py:69-91)
  int64_t m = trunc_iter(z);
  if (m > n) m = n;
  double acc = x(0), zj = z;
  for (int64_t j = 1; j < m; ++j, zj *= z) acc += zj * x(n - j);
  return acc / (1.0 - pow(z, static_cast<double>(m)));
}

// Final anti-causal coefficient (coeff.py:173-215).
template <class R>
__device__ double final_value(const R& L, int64_t n, int kind, double z) {
  if (kind == 2) return static_cast<double>(L[n - 1]) * (z / (z - 1.0));
  if (kind == 1) return (z * static_cast<double>(L[n - 2]) + static_cast<double>(L[n - 1])) * (z / (z * z - 1.0));
  int64_t m = trunc_iter(z);
  if (m > n) m = n;
  double acc = z * static_cast<double>(L[n - 1]), zj = z * z;
  for (int64_t j = 0; j < m - 1; ++j, zj *= z) acc += zj * static_cast<double>(L[j]);
  return acc / (pow(z, static_cast<double>(m)) - 1.0);
}

// Gain (coeff.py:61-65) folded into the first causal pass, then one causal
// and one anti-causal recursion per pole (coeff.py:254-281).
template <class R>
__device__ void filter_line(const R& L, typename R::index_type n, const LineArgs& a) {
  using C = typename R::value_type;
  using I = typename R::index_type;
  C g = static_cast<C>(a.gain);
  for (int q = 0; q < a.npoles; ++q) {
    const double zd = a.z[q];
    const C z = static_cast<C>(zd);
    C prev = static_cast<C>(initial(L, n, a.kind, zd, g));
    L[0] = prev;
    for (I i = 1; i < n; ++i) { prev = fma(z, prev, L[i] * g); L[i] = prev; }
    prev = static_cast<C>(final_value(L, n, a.kind, zd));
    L[n - 1] = prev;
    for (I i = n - 2; i >= 0; --i) { prev = z * (prev - L[i]); L[i] = prev; }
    g = C(1);
  }
}

// Asynchronous 4- / 8-byte global -> shared copy (no register round trip).
template <int B>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  if constexpr (B == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}

// Shared-memory line kernel: up to LINES lines per CTA, one per thread in
// the recursions, held element-major in shared memory (tile[i * pitch + l],
// odd pitch: conflict-free both for the per-thread walks along a line and
// for warps that stage whole lines).  Staging walks the tile so that a warp
// touches 32 consecutive addresses of global memory: 32 elements of one line
// when the filtered axis is the fastest, else element i of 32 adjacent
// lines.  float / double storage stage with asynchronous copies -- every
// element of the tile is in flight at once, which is what it takes to keep
// HBM busy with two CTAs per SM; 16-bit storage converts through registers,
// UNROLL loads in flight per thread.
template <class S>
__global__ void __launch_bounds__(THREADS) coeff_smem_kernel(LineArgs a, int pitch, int lines) {
  using C = typename ppk::Acc<S>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  const int64_t l0 = static_cast<int64_t>(blockIdx.x) * lines;
  const int nl = static_cast<int>(a.nlines - l0 < lines ? a.nlines - l0 : lines);
  const S* in = static_cast<const S*>(a.in);
  S* out = static_cast<S*>(a.out);
  __shared__ int64_t bin[LINES], bout[LINES];
  for (int l = threadIdx.x; l < nl; l += blockDim.x) line_base(a, l0 + l, bin[l], bout[l]);
  __syncthreads();
  const int n32 = static_cast<int>(a.n);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int outer_n = a.line_major ? nl : n32, inner_n = a.line_major ? n32 : nl;
  if constexpr (sizeof(S) == sizeof(C)) {
    for (int o = warp; o < outer_n; o += nwarps)
      for (int j = lane; j < inner_n; j += 32) {
        const int l = a.line_major ? o : j, i = a.line_major ? j : o;
        cp_async<sizeof(C)>(sm + i * pitch + l, in + bin[l] + static_cast<int64_t>(i) * a.in_st);
      }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  } else {
    for (int o = warp; o < outer_n; o += nwarps) {
      for (int j0 = 0; j0 < inner_n; j0 += 32 * UNROLL) {
        C v[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
          const int j = j0 + u * 32 + lane;
          const int l = a.line_major ? o : j, i = a.line_major ? j : o;
          v[u] = j < inner_n ? ppk::to_acc(in[bin[l] + static_cast<int64_t>(i) * a.in_st]) : C(0);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
          const int j = j0 + u * 32 + lane;
          const int l = a.line_major ? o : j, i = a.line_major ? j : o;
          if (j < inner_n) sm[i * pitch + l] = v[u];
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < nl) filter_line(TileLine<C>{sm + threadIdx.x, pitch}, n32, a);
  __syncthreads();
  for (int o = warp; o < outer_n; o += nwarps) {
    for (int j = lane; j < inner_n; j += 32) {
      const int l = a.line_major ? o : j, i = a.line_major ? j : o;
      out[bout[l] + static_cast<int64_t>(i) * a.out_st] = ppk::from_acc<S>(sm[i * pitch + l]);
    }
  }
}

// Global-memory fallback for lines too long for shared memory (more than
// ~50k elements): copy, then filter in place in the output.  float / double
// storage only.
template <class S>
__global__ void coeff_global_kernel(LineArgs a) {
  using C = typename ppk::Acc<S>::type;
  const int64_t l = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (l >= a.nlines) return;
  int64_t bi, bo;
  line_base(a, l, bi, bo);
  const S* in = static_cast<const S*>(a.in);
  S* out = static_cast<S*>(a.out);
  if (in != out || bi != bo || a.in_st != a.out_st)
    for (int64_t i = 0; i < a.n; ++i) out[bo + i * a.out_st] = in[bi + i * a.in_st];
  LineRef<S> L{out + bo, a.out_st};
  filter_line(L, a.n, a);
}

template <class S>
__global__ void copy_strided(const S* in, S* out, ppc::Strided si, ppc::Strided so) {
  int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (; i < si.numel; i += step) out[ppc::strided_offset(so, i)] = in[ppc::strided_offset(si, i)];
}

int poles(int order, double* z) {
  switch (order) {
    case 0: case 1: return 0;
    case 2: z[0] = sqrt(8.0) - 3.0; return 1;
    case 3: z[0] = sqrt(3.0) - 2.0; return 1;
    case 4:
      z[0] = sqrt(664.0 - sqrt(438976.0)) + sqrt(304.0) - 19.0;
      z[1] = sqrt(664.0 + sqrt(438976.0)) - sqrt(304.0) - 19.0;
      return 2;
    case 5:
      z[0] = sqrt(67.5 - sqrt(4436.25)) + sqrt(26.25) - 6.5;
      z[1] = sqrt(67.5 + sqrt(4436.25)) - sqrt(26.25) - 6.5;
      return 2;
    case 6:
      z[0] = -0.488294589303044755130118038883789062112279161239377608394;
      z[1] = -0.081679271076237512597937765737059080653379610398148178525368;
      z[2] = -0.00141415180832581775108724397655859252786416905534669851652709;
      return 3;
    case 7:
      z[0] = -0.5352804307964381655424037816816460718339231523426924148812;
      z[1] = -0.122554615192326690515272264359357343605486549427295558490763;
      z[2] = -0.0091486948096082769285930216516478534156925639545994482648003;
      return 3;
  }
  return -1;
}

template <class S>
int copy_tensor(const pp_tensor* in, const pp_tensor* out, cudaStream_t st) {
  const int64_t n = ppc::numel(in);
  if (n == 0 || in->data == out->data) return PP_OK;
  ppc::Strided si = ppc::make_strided(in), so = ppc::make_strided(out);
  copy_strided<S><<<ppc::grid_blocks(n), 256, 0, st>>>(static_cast<const S*>(in->data), static_cast<S*>(out->data), si, so);
  ppc::count_launch();
  return ppc::cuda_check(cudaGetLastError(), "copy");
}

int copy_any(const pp_tensor* in, const pp_tensor* out, cudaStream_t st) {
  switch (in->dtype) {
    case PP_FLOAT32: return copy_tensor<float>(in, out, st);
    case PP_FLOAT64: return copy_tensor<double>(in, out, st);
    case PP_BFLOAT16: return copy_tensor<__nv_bfloat16>(in, out, st);
    default: return copy_tensor<__half>(in, out, st);
  }
}

template <class S>
int run_axis(LineArgs& a, cudaStream_t st) {
  using C = typename ppk::Acc<S>::type;
  if (a.nlines == 0) return PP_OK;
  // two CTAs per SM where the lines allow; fewer, longer lines otherwise
  size_t budget = 110 * 1024;
  int lines = 0, pitch = 0;
  for (int pass = 0; pass < 2 && lines < 1; ++pass, budget = 200 * 1024) {
    const int64_t fit = static_cast<int64_t>(budget / (static_cast<size_t>(a.n) * sizeof(C)));
    lines = static_cast<int>(fit < LINES ? fit : LINES);
    pitch = lines | 1;
    if (static_cast<int64_t>(pitch) > fit) pitch = --lines;  // lines was even: drop one
  }
  if (lines >= 1) {
    const size_t smem = static_cast<size_t>(a.n) * pitch * sizeof(C);
    auto k = coeff_smem_kernel<S>;
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e != cudaSuccess) return ppc::cuda_check(e, "prefilter smem attribute");
    }
    const int64_t blocks = (a.nlines + lines - 1) / lines;
    k<<<static_cast<unsigned>(blocks), THREADS, smem, st>>>(a, pitch, lines);
    ppc::count_launch();
  } else {
    if constexpr (sizeof(S) < 4) {
      return ppc::fail(PP_ERR_UNSUPPORTED, "(): 16-bit spline_coeff lines longer than %lld elements",
                       (long long)(budget / sizeof(C)));
    } else {
      const int64_t blocks = (a.nlines + 127) / 128;
      coeff_global_kernel<S><<<static_cast<unsigned>(blocks), 128, 0, st>>>(a);
      ppc::count_launch();
    }
  }
  return ppc::cuda_check(cudaGetLastError(), "prefilter launch");
}

int coeff_axis(const pp_tensor* in, const pp_tensor* out, int bound, int order, int axis,
               cudaStream_t st) {
  LineArgs a;
  a.in = in->data;
  a.out = out->data;
  a.n = in->sizes[axis];
  a.in_st = in->strides[axis];
  a.out_st = out->strides[axis];
  a.npoles = poles(order, a.z);
  if (a.npoles < 0) return ppc::fail(PP_ERR_ARG, "(): unsupported interpolation order %d", order);
  if (a.npoles == 0) return copy_any(in, out, st);
  if (bound == 0 || bound == 2) a.kind = 1;
  else if (bound == 1 || bound == 3) a.kind = 2;
  else if (bound == 6) a.kind = 3;
  else return ppc::fail(PP_ERR_UNSUPPORTED, "(): spline_coeff is not implemented for bound code %d "
                        "(only zero, replicate, dct1, dct2 and dft)", bound);
  if (a.n == 1) return copy_any(in, out, st);
  a.gain = 1.0;
  for (int q = 0; q < a.npoles; ++q) a.gain *= (1.0 - a.z[q]) * (1.0 - 1.0 / a.z[q]);
  a.ndo = 0;
  a.nlines = 1;
  int64_t min_other = INT64_MAX;
  for (int d = 0; d < in->ndim; ++d) {
    if (d == axis) continue;
    a.osz[a.ndo] = in->sizes[d];
    a.ist[a.ndo] = in->strides[d];
    a.ost[a.ndo] = out->strides[d];
    if (in->sizes[d] > 1 && in->strides[d] < min_other) min_other = in->strides[d];
    a.nlines *= in->sizes[d];
    ++a.ndo;
  }
  a.line_major = (a.in_st <= min_other) ? 1 : 0;
  switch (in->dtype) {
    case PP_FLOAT32: return run_axis<float>(a, st);
    case PP_FLOAT64: return run_axis<double>(a, st);
    case PP_BFLOAT16: return run_axis<__nv_bfloat16>(a, st);
    default: return run_axis<__half>(a, st);
  }
}

int check_coeff_io(const pp_tensor* in, const pp_tensor* out) {
  int rc = ppc::check_tensor(in, "input");
  if (rc) return rc;
  if ((rc = ppc::check_tensor(out, "output"))) return rc;
  if (in->ndim != out->ndim) return ppc::fail(PP_ERR_ARG, "(): output must have the input's shape");
  for (int d = 0; d < in->ndim; ++d)
    if (in->sizes[d] != out->sizes[d]) return ppc::fail(PP_ERR_ARG, "(): output must have the input's shape");
  if (in->dtype != out->dtype) return ppc::fail(PP_ERR_DTYPE, "(): output dtype must match input");
  return PP_OK;
}

}  // namespace

extern "C" {

int pp_spline_coeff(const pp_tensor* input, const pp_tensor* out, int32_t bound, int32_t order,
                    int32_t axis, void* stream) {
  int rc = check_coeff_io(input, out);
  if (rc) return rc;
  if (input->ndim == 0) return copy_any(input, out, static_cast<cudaStream_t>(stream));
  if (axis < 0) axis += input->ndim;
  if (axis < 0 || axis >= input->ndim) return ppc::fail(PP_ERR_ARG, "(): axis out of range");
  if (order < 0 || order > 7) return ppc::fail(PP_ERR_ARG, "(): unsupported interpolation order %d", order);
  if (ppc::numel(input) == 0) return PP_OK;
  return coeff_axis(input, out, bound, order, axis, static_cast<cudaStream_t>(stream));
}

int pp_spline_coeff_nd(const pp_tensor* input, const pp_tensor* out, int32_t nbound, const int32_t* bound,
                       int32_t norder, const int32_t* order, int32_t dim, void* stream) {
  int rc = check_coeff_io(input, out);
  if (rc) return rc;
  if (dim < 0 || dim > input->ndim) return ppc::fail(PP_ERR_ARG, "(): dim out of range");
  if (nbound < 1 || norder < 1 || !bound || !order) return ppc::fail(PP_ERR_ARG, "(): empty bound / order list");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (ppc::numel(input) == 0) return PP_OK;
  const pp_tensor* src = input;
  bool wrote = false;
  for (int d = 0; d < dim; ++d) {
    const int b = bound[d < nbound ? d : nbound - 1];
    const int o = order[d < norder ? d : norder - 1];
    if (o < 0 || o > 7) return ppc::fail(PP_ERR_ARG, "(): unsupported interpolation order %d", o);
    const int axis = input->ndim - dim + d;
    if (o <= 1) continue;  // identity along this axis
    if ((rc = coeff_axis(src, out, b, o, axis, st))) return rc;
    src = out;
    wrote = true;
  }
  if (!wrote) return copy_any(input, out, st);
  return PP_OK;
}

}  // extern "C"
