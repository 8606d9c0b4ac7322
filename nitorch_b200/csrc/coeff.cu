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
#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "pp_capi_internal.cuh"

namespace {

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
  // per-pole boundary constants, the same for every line (host-computed):
  int64_t hz[3];      // dct2: series length K; dct1: truncation m; dft: min(m, n)
  double zp[3];       // dct2: z^n; dct1: z^(n-1); dft: z^hz
  double zq[3];       // dct2: z^(2n-1-k2), k2 = max(1, 2n-1-K): the mirrored tail's first weight
  int line_major;     // 1: the filtered axis is the fastest (warps stage whole lines)
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

template <class C, int P>  // P: compile-time pitch, 0 = runtime
struct TileLine {
  using value_type = C;
  using index_type = int;
  C* p;
  int pitch;
  __device__ __forceinline__ C& operator[](int i) const { return p[i * (P ? P : pitch)]; }
};

// Initial causal coefficient (coeff.py:69-170), double accumulation.  The
// samples are read as L[k] * g (g: the filter gain on the first pole's pass,
// 1 afterwards), so the gain pass costs no separate sweep.
template <class R, class C = typename R::value_type>
__device__ double initial(const R& L, int64_t n, const LineArgs& a, int q, C g) {
  const double z = a.z[q];
  auto x = [&](int64_t k) { return static_cast<double>(L[k] * g); };
  if (a.kind == 2) {  // dct2 / replicate (coeff.py:137-170)
    const double zn = a.zp[q];
    const double zlast = zn * (1.0 + 1.0 / (z + zn * zn));
    double acc = x(0) + zlast * x(n - 1);
    // sum_{k=1}^{n-2} (z^k + z^(2n-1-k)) L[k]; both power series decay
    // geometrically, terms below 2^-64 of the leading one are dropped.
    const int64_t K = a.hz[q];
    const int64_t k1 = n - 2 < K ? n - 2 : K;
    double zk = z;
    for (int64_t k = 1; k <= k1; ++k, zk *= z) acc += zk * x(k);
    int64_t k2 = 2 * n - 1 - K;
    if (k2 < 1) k2 = 1;
    if (k2 <= n - 2) {
      double zq = a.zq[q];
      const double iz = 1.0 / z;
      for (int64_t k = k2; k <= n - 2; ++k, zq *= iz) acc += zq * x(k);
    }
    return acc * (z / (1.0 - zn * zn)) + x(0);
  }
  if (a.kind == 1) {  // dct1 / zero (coeff.py:94-134)
    const int64_t m = a.hz[q];
    if (m < n) {
      double acc = x(0), zk = z;
      for (int64_t k = 1; k < m; ++k, zk *= z) acc += zk * x(k);
      return acc;
    }
    const double zn = a.zp[q];
    double acc = x(0) + zn * x(n - 1);
    double zk = z;
    for (int64_t k = 1; k < n - 1; ++k, zk *= z) acc += (zk + zn * zn / zk) * x(k);
    return acc / (1.0 - zn * zn);
  }
  // dft (coeff.py:69-91)
  const int64_t m = a.hz[q];
  double acc = x(0), zj = z;
  for (int64_t j = 1; j < m; ++j, zj *= z) acc += zj * x(n - j);
  return acc / (1.0 - a.zp[q]);
}

// Final anti-causal coefficient (coeff.py:173-215).
template <class R>
__device__ double final_value(const R& L, int64_t n, const LineArgs& a, int q) {
  const double z = a.z[q];
  if (a.kind == 2) return static_cast<double>(L[n - 1]) * (z / (z - 1.0));
  if (a.kind == 1) return (z * static_cast<double>(L[n - 2]) + static_cast<double>(L[n - 1])) * (z / (z * z - 1.0));
  const int64_t m = a.hz[q];
  double acc = z * static_cast<double>(L[n - 1]), zj = z * z;
  for (int64_t j = 0; j < m - 1; ++j, zj *= z) acc += zj * static_cast<double>(L[j]);
  return acc / (a.zp[q] - 1.0);
}

// Gain (coeff.py:61-65) folded into the first causal pass, then one causal
// and one anti-causal recursion per pole (coeff.py:254-281).  The walks go
// in chunks of RU samples held in registers, the next chunk loaded before the
// current one is filtered, so that the memory latency leaves the dependency
// chain (one FMA per sample); the accessor's stride is a runtime value, which
// keeps the compiler from reordering the loads past the stores by itself.
constexpr int RU = 8;

template <class R>
__device__ void filter_line(const R& L, typename R::index_type n, const LineArgs& a) {
  using C = typename R::value_type;
  using I = typename R::index_type;
  C g = static_cast<C>(a.gain);
  for (int q = 0; q < a.npoles; ++q) {
    const double zd = a.z[q];
    const C z = static_cast<C>(zd);
    C prev = static_cast<C>(initial(L, n, a, q, g));
    L[0] = prev;
    I i = 1;  // causal: i = 1 .. n-1
    if (n - 1 >= RU) {
      C x[RU];
#pragma unroll
      for (int u = 0; u < RU; ++u) x[u] = L[i + u];
      for (;;) {
        const bool more = i + 2 * RU <= n;
        C y[RU];
        if (more) {
#pragma unroll
          for (int u = 0; u < RU; ++u) y[u] = L[i + RU + u];
        }
#pragma unroll
        for (int u = 0; u < RU; ++u) { prev = fma(z, prev, x[u] * g); L[i + u] = prev; }
        i += RU;
        if (!more) break;
#pragma unroll
        for (int u = 0; u < RU; ++u) x[u] = y[u];
      }
    }
    for (; i < n; ++i) { prev = fma(z, prev, L[i] * g); L[i] = prev; }
    prev = static_cast<C>(final_value(L, n, a, q));
    L[n - 1] = prev;
    i = n - 2;  // anti-causal: i = n-2 .. 0
    if (i + 1 >= RU) {
      C x[RU];
#pragma unroll
      for (int u = 0; u < RU; ++u) x[u] = L[i - u];
      for (;;) {
        const bool more = i + 1 >= 2 * RU;
        C y[RU];
        if (more) {
#pragma unroll
          for (int u = 0; u < RU; ++u) y[u] = L[i - RU - u];
        }
#pragma unroll
        for (int u = 0; u < RU; ++u) { prev = z * (prev - x[u]); L[i - u] = prev; }
        i -= RU;
        if (!more) break;
#pragma unroll
        for (int u = 0; u < RU; ++u) x[u] = y[u];
      }
    }
    for (; i >= 0; --i) { prev = z * (prev - L[i]); L[i] = prev; }
    g = C(1);
  }
}

// Asynchronous global -> shared copies (no register round trip).
template <int B>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  if constexpr (B == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
  else if constexpr (B == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
  else asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}

// G adjacent samples of 16-bit storage <-> G floats (one 8-byte access).
template <class S, class C>
__device__ __forceinline__ void load_group(C* dst, const S* src) {
  static_assert(sizeof(S) == 2 && sizeof(C) == 4, "16-bit storage, float arithmetic");
  const uint2 r = *reinterpret_cast<const uint2*>(src);
  const S* v = reinterpret_cast<const S*>(&r);
  *reinterpret_cast<float4*>(dst) = make_float4(ppk::to_acc(v[0]), ppk::to_acc(v[1]), ppk::to_acc(v[2]),
                                                ppk::to_acc(v[3]));
}

// Shared-memory line kernel: NL threads, up to NL lines per CTA, one per
// thread, held element-major in shared memory (tile[i * pitch + l]).  Small
// CTAs (a few warps) several to an SM: each loads its tile, recurses and
// stores on its own schedule, so the loads of some overlap the recursions of
// others.  Staging walks the tile so that a warp touches consecutive
// addresses of global memory:
//  * filtered axis the fastest (line_major): a warp per line, lanes over
//    consecutive samples; odd pitch, so the lanes' column writes are
//    conflict-free;
//  * otherwise each thread a group of G = 16 / sizeof(C) adjacent lines on
//    every G-th sample row, moved as one 16-byte copy (8-byte load for
//    16-bit storage) when the G lines are adjacent and aligned in memory, else
//    G scalar copies; pitch a multiple of G.
// float / double storage stage with asynchronous copies, so that the whole
// tile is in flight at once; 16-bit storage converts through registers.
// P: the pitch as a compile-time constant for full tiles (NL + 1 for
// line_major, NL otherwise), 0 for the runtime pitch of long-line tiles.
template <class S, int NL, int P>
__global__ void __launch_bounds__(NL) coeff_smem_kernel(LineArgs a, int pitch_rt, int lines) {
  using C = typename ppk::Acc<S>::type;
  constexpr int G = 16 / static_cast<int>(sizeof(C));
  constexpr int GPR = NL / G;  // groups per sample row
  constexpr bool kAsync = sizeof(S) == sizeof(C);
  static_assert(NL % 32 == 0 && NL % G == 0, "tile of whole warps and groups");
  const int pitch = P ? P : pitch_rt;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  const int64_t l0 = static_cast<int64_t>(blockIdx.x) * lines;
  const int nl = static_cast<int>(a.nlines - l0 < lines ? a.nlines - l0 : lines);
  const S* in = static_cast<const S*>(a.in);
  S* out = static_cast<S*>(a.out);
  __shared__ int64_t bin[NL], bout[NL];
  for (int l = threadIdx.x; l < nl; l += NL) line_base(a, l0 + l, bin[l], bout[l]);
  __syncthreads();
  const int n32 = static_cast<int>(a.n);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int nwarps = NL / 32;
  // vector eligibility of the group at line l: G lines present, adjacent,
  // every row aligned
  auto group_vec = [&](const int64_t* base, const void* ptr, int64_t st, int l, int bytes) {
    if (l + G > nl || (pitch % G) != 0) return false;
    for (int k = 1; k < G; ++k)
      if (base[l + k] != base[l] + k) return false;
    const uintptr_t p = reinterpret_cast<uintptr_t>(ptr) + static_cast<uintptr_t>(base[l]) * sizeof(S);
    return (p % bytes) == 0 && ((st * static_cast<int64_t>(sizeof(S))) % bytes) == 0;
  };
  const int gl = (threadIdx.x % GPR) * G, r0 = threadIdx.x / GPR;  // strided: group line, first row
  if (a.line_major) {
    for (int l = warp; l < nl; l += nwarps) {
      const S* src = in + bin[l];
      C* dst = sm + l;
      if constexpr (kAsync) {
        for (int i = lane; i < n32; i += 32) cp_async<sizeof(C)>(dst + i * pitch, src + i * a.in_st);
      } else {
        for (int i0 = 0; i0 < n32; i0 += 32 * UNROLL) {
          C v[UNROLL];
#pragma unroll
          for (int u = 0; u < UNROLL; ++u) {
            const int i = i0 + u * 32 + lane;
            v[u] = i < n32 ? ppk::to_acc(src[i * a.in_st]) : C(0);
          }
#pragma unroll
          for (int u = 0; u < UNROLL; ++u) {
            const int i = i0 + u * 32 + lane;
            if (i < n32) dst[i * pitch] = v[u];
          }
        }
      }
    }
  } else if (gl < nl) {
    const bool vec = group_vec(bin, in, a.in_st, gl, G * static_cast<int>(sizeof(S)));
    const S* src = in + bin[gl];
    for (int i = r0; i < n32; i += G) {
      C* dst = sm + i * pitch + gl;
      const int64_t off = i * a.in_st;
      if (vec) {
        if constexpr (kAsync) cp_async<16>(dst, src + off);
        else load_group(dst, src + off);
      } else {
        for (int k = 0; k < G && gl + k < nl; ++k) {
          if constexpr (kAsync) cp_async<sizeof(C)>(dst + k, in + bin[gl + k] + off);
          else dst[k] = ppk::to_acc(in[bin[gl + k] + off]);
        }
      }
    }
  }
  if constexpr (kAsync) asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  if (threadIdx.x < nl) filter_line(TileLine<C, P>{sm + threadIdx.x, pitch}, n32, a);
  __syncthreads();
  if (a.line_major) {
    for (int l = warp; l < nl; l += nwarps) {
      S* dst = out + bout[l];
      const C* src = sm + l;
      for (int i = lane; i < n32; i += 32) dst[i * a.out_st] = ppk::from_acc<S>(src[i * pitch]);
    }
  } else if (gl < nl) {
    const bool vec = group_vec(bout, out, a.out_st, gl, G * static_cast<int>(sizeof(S)));
    S* dst = out + bout[gl];
    for (int i = r0; i < n32; i += G) {
      const C* src = sm + i * pitch + gl;
      const int64_t off = i * a.out_st;
      if (vec) {
        if constexpr (kAsync) {
          *reinterpret_cast<uint4*>(dst + off) = *reinterpret_cast<const uint4*>(src);
        } else {
          const float4 f = *reinterpret_cast<const float4*>(src);
          S v[4] = {ppk::from_acc<S>(f.x), ppk::from_acc<S>(f.y), ppk::from_acc<S>(f.z), ppk::from_acc<S>(f.w)};
          *reinterpret_cast<uint2*>(dst + off) = *reinterpret_cast<const uint2*>(v);
        }
      } else {
        for (int k = 0; k < G && gl + k < nl; ++k) out[bout[gl + k] + off] = ppk::from_acc<S>(src[k]);
      }
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

// Lines per CTA (= threads): small CTAs, several per SM.
int tile_lines() {
  static const int nl = [] {
    const char* e = std::getenv("PP_COEFF_LINES");
    const int v = e ? std::atoi(e) : 64;
    return (v == 32 || v == 64 || v == 128) ? v : 64;
  }();
  return nl;
}

template <class S, int NL>
int run_tiles(LineArgs& a, cudaStream_t st) {
  using C = typename ppk::Acc<S>::type;
  constexpr int G = 16 / static_cast<int>(sizeof(C));
  // pitch: odd when warps stage whole lines (conflict-free column writes),
  // else a multiple of the 16-byte group width; long lines take fewer lines
  // per CTA, up to 200 KB of shared memory.
  const size_t budget = 200 * 1024;
  const int64_t fit = static_cast<int64_t>(budget / (static_cast<size_t>(a.n) * sizeof(C)));
  int lines = static_cast<int>(fit < NL ? fit : NL), pitch = 0;
  if (a.line_major) {
    pitch = lines | 1;
    if (static_cast<int64_t>(pitch) > fit) pitch = --lines;  // lines was even: drop one
  } else {
    if (lines >= G) lines -= lines % G;
    pitch = lines;
  }
  if (lines >= 1) {
    const size_t smem = static_cast<size_t>(a.n) * pitch * sizeof(C);
    const bool full = lines == NL && pitch == (a.line_major ? NL + 1 : NL);
    auto k = !full ? coeff_smem_kernel<S, NL, 0>
                   : (a.line_major ? coeff_smem_kernel<S, NL, NL + 1> : coeff_smem_kernel<S, NL, NL>);
    // the 48 KB default covers static (line bases) plus dynamic shared memory
    if (smem + 2 * NL * sizeof(int64_t) > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e != cudaSuccess) return ppc::cuda_check(e, "prefilter smem attribute");
    }
    const int64_t blocks = (a.nlines + lines - 1) / lines;
    k<<<static_cast<unsigned>(blocks), NL, smem, st>>>(a, pitch, lines);
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

template <class S>
int run_axis(LineArgs& a, cudaStream_t st) {
  if (a.nlines == 0) return PP_OK;
  switch (tile_lines()) {
    case 32: return run_tiles<S, 32>(a, st);
    case 128: return run_tiles<S, 128>(a, st);
    default: return run_tiles<S, 64>(a, st);
  }
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
  for (int q = 0; q < a.npoles; ++q) {
    const double z = a.z[q];
    a.gain *= (1.0 - z) * (1.0 - 1.0 / z);
    // truncation of the causal initial sums (coeff.py:75, :100): |z|^m < 1e-13
    const int64_t m = static_cast<int64_t>(std::ceil(-30.0 / std::log(std::fabs(z))));
    if (a.kind == 2) {
      const int64_t K = static_cast<int64_t>(std::ceil(-44.4 / std::log(std::fabs(z)))) + 1;
      const int64_t k2 = std::max<int64_t>(1, 2 * a.n - 1 - K);
      a.hz[q] = K;
      a.zp[q] = std::pow(z, static_cast<double>(a.n));
      a.zq[q] = std::pow(z, static_cast<double>(2 * a.n - 1 - k2));
    } else if (a.kind == 1) {
      a.hz[q] = m;
      a.zp[q] = std::pow(z, static_cast<double>(a.n - 1));
      a.zq[q] = 0.0;
    } else {
      a.hz[q] = std::min<int64_t>(m, a.n);
      a.zp[q] = std::pow(z, static_cast<double>(a.hz[q]));
      a.zq[q] = 0.0;
    }
  }
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
