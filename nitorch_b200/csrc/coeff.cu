// Interpolating B-spline prefilter (spline_coeff / spline_coeff_nd).
//
// Arithmetic restated from the vendored prefilter nitorch/_C/_ts/coeff.py
// (Unser-Aldroubi-Eden recursive filtering): gain (coeff.py:61-65), one
// causal and one anti-causal first-order recursion per pole (coeff.py:
// 254-281), initial / final conditions per boundary (coeff.py:69-251).
//
// B200 mapping: one line per thread, a tile of lines per CTA staged in
// shared memory (element-major: warps of recursing threads read one sample of
// 32 adjacent lines per access) by asynchronous copies issued for the whole
// tile at once, 16 bytes at a time across adjacent lines when the filtered
// axis is strided.  The sequential recursions run out of shared memory and
// the global traffic is one read and one write of the volume per axis.  Tile
// widths are chosen per line length so that two CTAs share an SM, one's
// transfers overlapping the other's recursions.  The recursions run in float
// (double for double storage); the initial / final condition sums in double
// with per-pole constants computed on the host.  Lines too long for a shared
// tile fall back to the same recursion directly on global memory.
#include <algorithm>
#include <cmath>

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

// Accessors over V adjacent lines (V = 1: one line); load / store move
// sample i of the V lines.
template <class C>
struct LineRef {  // one line in global memory, any stride
  static constexpr int V = 1;
  using value_type = C;
  using index_type = int64_t;
  C* p;
  int64_t st;
  __device__ __forceinline__ void load(int64_t i, C (&x)[1]) const { x[0] = p[i * st]; }
  __device__ __forceinline__ void store(int64_t i, const C (&x)[1]) const { p[i * st] = x[0]; }
};

template <class C>
struct TileLine {  // one column of a shared tile, runtime pitch
  static constexpr int V = 1;
  using value_type = C;
  using index_type = int;
  C* p;
  int pitch;
  __device__ __forceinline__ void load(int i, C (&x)[1]) const { x[0] = p[i * pitch]; }
  __device__ __forceinline__ void store(int i, const C (&x)[1]) const { p[i * pitch] = x[0]; }
};

template <class C, int P, int V_>
struct TileCols {  // V_ adjacent columns of a shared tile (compile-time pitch), one access
  static constexpr int V = V_;
  using value_type = C;
  using index_type = int;
  C* p;
  __device__ __forceinline__ void load(int i, C (&x)[V]) const {
    const C* q = p + i * P;
    if constexpr (V == 4 && sizeof(C) == 4) {
      const float4 t = *reinterpret_cast<const float4*>(q);
      x[0] = t.x; x[1] = t.y; x[2] = t.z; x[3] = t.w;
    } else if constexpr (V == 2 && sizeof(C) == 4) {
      const float2 t = *reinterpret_cast<const float2*>(q);
      x[0] = t.x; x[1] = t.y;
    } else if constexpr (V == 2 && sizeof(C) == 8) {
      const double2 t = *reinterpret_cast<const double2*>(q);
      x[0] = t.x; x[1] = t.y;
    } else {
#pragma unroll
      for (int c = 0; c < V; ++c) x[c] = q[c];
    }
  }
  __device__ __forceinline__ void store(int i, const C (&x)[V]) const {
    C* q = p + i * P;
    if constexpr (V == 4 && sizeof(C) == 4) {
      *reinterpret_cast<float4*>(q) = make_float4(x[0], x[1], x[2], x[3]);
    } else if constexpr (V == 2 && sizeof(C) == 4) {
      *reinterpret_cast<float2*>(q) = make_float2(x[0], x[1]);
    } else if constexpr (V == 2 && sizeof(C) == 8) {
      *reinterpret_cast<double2*>(q) = make_double2(x[0], x[1]);
    } else {
#pragma unroll
      for (int c = 0; c < V; ++c) q[c] = x[c];
    }
  }
};

// Initial causal coefficient (coeff.py:69-170) of each of the V lines,
// double accumulation.  The samples are read as L[k] * g (g: the filter gain
// on the first pole's pass, 1 afterwards), so the gain costs no separate
// sweep.
template <class R, int V = R::V, class C = typename R::value_type>
__device__ void initial(const R& L, int64_t n, const LineArgs& a, int q, C g, double (&out)[V]) {
  const double z = a.z[q];
  C t[V];
  double xv[V], x0[V], acc[V];
  auto x = [&](int64_t k) {
    L.load(k, t);
#pragma unroll
    for (int c = 0; c < V; ++c) xv[c] = static_cast<double>(t[c] * g);
  };
  x(0);
#pragma unroll
  for (int c = 0; c < V; ++c) x0[c] = acc[c] = xv[c];
  if (a.kind == 2) {  // dct2 / replicate (coeff.py:137-170)
    const double zn = a.zp[q];
    const double zlast = zn * (1.0 + 1.0 / (z + zn * zn));
    x(n - 1);
#pragma unroll
    for (int c = 0; c < V; ++c) acc[c] += zlast * xv[c];
    // sum_{k=1}^{n-2} (z^k + z^(2n-1-k)) L[k]; both power series decay
    // geometrically, terms below 2^-64 of the leading one are dropped.
    const int64_t K = a.hz[q];
    const int64_t k1 = n - 2 < K ? n - 2 : K;
    double zk = z;
    for (int64_t k = 1; k <= k1; ++k, zk *= z) {
      x(k);
#pragma unroll
      for (int c = 0; c < V; ++c) acc[c] += zk * xv[c];
    }
    int64_t k2 = 2 * n - 1 - K;
    if (k2 < 1) k2 = 1;
    if (k2 <= n - 2) {
      double zq = a.zq[q];
      const double iz = 1.0 / z;
      for (int64_t k = k2; k <= n - 2; ++k, zq *= iz) {
        x(k);
#pragma unroll
        for (int c = 0; c < V; ++c) acc[c] += zq * xv[c];
      }
    }
    const double s = z / (1.0 - zn * zn);
#pragma unroll
    for (int c = 0; c < V; ++c) out[c] = acc[c] * s + x0[c];
    return;
  }
  if (a.kind == 1) {  // dct1 / zero (coeff.py:94-134)
    const int64_t m = a.hz[q];
    if (m < n) {
      double zk = z;
      for (int64_t k = 1; k < m; ++k, zk *= z) {
        x(k);
#pragma unroll
        for (int c = 0; c < V; ++c) acc[c] += zk * xv[c];
      }
#pragma unroll
      for (int c = 0; c < V; ++c) out[c] = acc[c];
      return;
    }
    const double zn = a.zp[q];
    x(n - 1);
#pragma unroll
    for (int c = 0; c < V; ++c) acc[c] += zn * xv[c];
    double zk = z;
    for (int64_t k = 1; k < n - 1; ++k, zk *= z) {
      x(k);
      const double w = zk + zn * zn / zk;
#pragma unroll
      for (int c = 0; c < V; ++c) acc[c] += w * xv[c];
    }
    const double s = 1.0 / (1.0 - zn * zn);
#pragma unroll
    for (int c = 0; c < V; ++c) out[c] = acc[c] * s;
    return;
  }
  // dft (coeff.py:69-91)
  const int64_t m = a.hz[q];
  double zj = z;
  for (int64_t j = 1; j < m; ++j, zj *= z) {
    x(n - j);
#pragma unroll
    for (int c = 0; c < V; ++c) acc[c] += zj * xv[c];
  }
  const double s = 1.0 / (1.0 - a.zp[q]);
#pragma unroll
  for (int c = 0; c < V; ++c) out[c] = acc[c] * s;
}

// Final anti-causal coefficient (coeff.py:173-215) of each of the V lines.
template <class R, int V = R::V, class C = typename R::value_type>
__device__ void final_value(const R& L, int64_t n, const LineArgs& a, int q, double (&out)[V]) {
  const double z = a.z[q];
  C t[V];
  L.load(n - 1, t);
  if (a.kind == 2) {
    const double s = z / (z - 1.0);
#pragma unroll
    for (int c = 0; c < V; ++c) out[c] = static_cast<double>(t[c]) * s;
    return;
  }
  if (a.kind == 1) {
    C u[V];
    L.load(n - 2, u);
    const double s = z / (z * z - 1.0);
#pragma unroll
    for (int c = 0; c < V; ++c) out[c] = (z * static_cast<double>(u[c]) + static_cast<double>(t[c])) * s;
    return;
  }
  const int64_t m = a.hz[q];
  double acc[V];
#pragma unroll
  for (int c = 0; c < V; ++c) acc[c] = z * static_cast<double>(t[c]);
  double zj = z * z;
  for (int64_t j = 0; j < m - 1; ++j, zj *= z) {
    L.load(j, t);
#pragma unroll
    for (int c = 0; c < V; ++c) acc[c] += zj * static_cast<double>(t[c]);
  }
  const double s = 1.0 / (a.zp[q] - 1.0);
#pragma unroll
  for (int c = 0; c < V; ++c) out[c] = acc[c] * s;
}

// Gain (coeff.py:61-65) folded into the first causal pass, then one causal
// and one anti-causal recursion per pole (coeff.py:254-281), on V lines at
// once (independent dependency chains).  The walks go in chunks of U samples
// held in registers, the next chunk loaded before the current one is
// filtered, so that the memory latency leaves the dependency chains.
template <class R>
__device__ void filter_line(const R& L, typename R::index_type n, const LineArgs& a) {
  using C = typename R::value_type;
  using I = typename R::index_type;
  constexpr int V = R::V;
  constexpr int U = V == 1 ? 8 : 4;
  C g = static_cast<C>(a.gain);
  for (int q = 0; q < a.npoles; ++q) {
    const C z = static_cast<C>(a.z[q]);
    double d[V];
    C prev[V];
    initial(L, n, a, q, g, d);
#pragma unroll
    for (int c = 0; c < V; ++c) prev[c] = static_cast<C>(d[c]);
    L.store(0, prev);
    I i = 1;  // causal: i = 1 .. n-1
    if (n - 1 >= U) {
      C x[U][V];
#pragma unroll
      for (int u = 0; u < U; ++u) L.load(i + u, x[u]);
      for (;;) {
        const bool more = i + 2 * U <= n;
        C y[U][V];
        if (more) {
#pragma unroll
          for (int u = 0; u < U; ++u) L.load(i + U + u, y[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
#pragma unroll
          for (int c = 0; c < V; ++c) prev[c] = fma(z, prev[c], x[u][c] * g);
          L.store(i + u, prev);
        }
        i += U;
        if (!more) break;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
          for (int c = 0; c < V; ++c) x[u][c] = y[u][c];
      }
    }
    for (; i < n; ++i) {
      C x[V];
      L.load(i, x);
#pragma unroll
      for (int c = 0; c < V; ++c) prev[c] = fma(z, prev[c], x[c] * g);
      L.store(i, prev);
    }
    final_value(L, n, a, q, d);
#pragma unroll
    for (int c = 0; c < V; ++c) prev[c] = static_cast<C>(d[c]);
    L.store(n - 1, prev);
    i = n - 2;  // anti-causal: i = n-2 .. 0
    if (i + 1 >= U) {
      C x[U][V];
#pragma unroll
      for (int u = 0; u < U; ++u) L.load(i - u, x[u]);
      for (;;) {
        const bool more = i + 1 >= 2 * U;
        C y[U][V];
        if (more) {
#pragma unroll
          for (int u = 0; u < U; ++u) L.load(i - U - u, y[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
#pragma unroll
          for (int c = 0; c < V; ++c) prev[c] = z * (prev[c] - x[u][c]);
          L.store(i - u, prev);
        }
        i -= U;
        if (!more) break;
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
          for (int c = 0; c < V; ++c) x[u][c] = y[u][c];
      }
    }
    for (; i >= 0; --i) {
      C x[V];
      L.load(i, x);
#pragma unroll
      for (int c = 0; c < V; ++c) prev[c] = z * (prev[c] - x[c]);
      L.store(i, prev);
    }
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

// Vector eligibility of the group of G adjacent lines starting at tile line
// l: all present, adjacent in memory, every sample row aligned to the group
// width in bytes.
template <class S, int G>
__device__ __forceinline__ bool group_vec(const int64_t* base, const void* ptr, int64_t st, int l, int nl) {
  constexpr int bytes = G * static_cast<int>(sizeof(S));
  if (l + G > nl) return false;
  for (int k = 1; k < G; ++k)
    if (base[l + k] != base[l] + k) return false;
  const uintptr_t p = reinterpret_cast<uintptr_t>(ptr) + static_cast<uintptr_t>(base[l]) * sizeof(S);
  return (p % bytes) == 0 && ((st * static_cast<int64_t>(sizeof(S))) % bytes) == 0;
}

// Full-tile kernel: NT lines per CTA (32, 64, 96 or 128: the widest that
// leaves room for two CTAs per SM and one's transfers overlap the
// other's recursions), held element-major in shared memory: tile[i * P + l],
// P = NT + 4 (16-byte rows; 4 mod 32 words).  TILE_THREADS stage and store;
// NT / V threads run the recursions, V adjacent lines each, read and written
// as one access.  Staging keeps warps on consecutive global addresses:
//  * filtered axis the fastest (line_major): a warp instruction covers 8
//    consecutive samples of 4 lines (32-byte segments); with P = 4 mod 32
//    words the 32 shared-memory writes fall in 32 distinct banks;
//  * otherwise each thread a group of G = 16 / sizeof(C) adjacent lines on
//    every few sample rows, moved as one 16-byte copy (8-byte load for 16-bit
//    storage) when the lines are adjacent and aligned in memory, else G
//    scalar copies.
// float / double storage stage with asynchronous copies, the whole tile in
// flight at once; 16-bit storage converts through registers.
constexpr int TILE_THREADS = 256;
// lines per recursion thread: 1, 2 and 4 (one 4-, 8- or 16-byte access per
// sample) measured within noise of each other on 3 x 192^3 and 3 x 256^3
// float volumes; one line per thread keeps the most warps in the recursions
constexpr int TILE_V = 1;

template <class S, int NT, int V>
__global__ void __launch_bounds__(TILE_THREADS, 2) coeff_tile_kernel(LineArgs a) {
  using C = typename ppk::Acc<S>::type;
  constexpr int G = 16 / static_cast<int>(sizeof(C));
  constexpr int P = NT + 4;
  constexpr int NW = TILE_THREADS / 32;
  constexpr int GPR = NT / G;                 // strided: groups per sample row
  constexpr int RS = TILE_THREADS / GPR;      // strided: rows per step (threads past RS * GPR idle)
  constexpr bool kAsync = sizeof(S) == sizeof(C);
  static_assert(NT % 32 == 0 && NT % G == 0 && RS >= 1 && NT / V <= TILE_THREADS, "tile shape");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  const int64_t l0 = static_cast<int64_t>(blockIdx.x) * NT;
  const int nl = static_cast<int>(a.nlines - l0 < NT ? a.nlines - l0 : NT);
  const S* in = static_cast<const S*>(a.in);
  S* out = static_cast<S*>(a.out);
  __shared__ int64_t bin[NT], bout[NT];
  for (int l = threadIdx.x; l < nl; l += TILE_THREADS) line_base(a, l0 + l, bin[l], bout[l]);
  __syncthreads();
  const int n32 = static_cast<int>(a.n);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int qs = lane >> 3, qj = lane & 7;  // line_major: line in the quad, first sample
  const int gl = threadIdx.x < RS * GPR ? (threadIdx.x % GPR) * G : NT;  // strided: group (NT: idle)
  const int r0 = threadIdx.x / GPR;                                       // strided: first row
  if (a.line_major) {
    for (int qd = warp; qd * 4 < nl; qd += NW) {
      const int l = qd * 4 + qs;
      if (l >= nl) continue;
      const S* src = in + bin[l];
      C* dst = sm + l;
      if constexpr (kAsync) {
        for (int i = qj; i < n32; i += 8) cp_async<sizeof(C)>(dst + i * P, src + i * a.in_st);
      } else {
        for (int i0 = qj; i0 < n32; i0 += 8 * UNROLL) {
          C v[UNROLL];
#pragma unroll
          for (int u = 0; u < UNROLL; ++u) {
            const int i = i0 + 8 * u;
            v[u] = i < n32 ? ppk::to_acc(src[i * a.in_st]) : C(0);
          }
#pragma unroll
          for (int u = 0; u < UNROLL; ++u) {
            const int i = i0 + 8 * u;
            if (i < n32) dst[i * P] = v[u];
          }
        }
      }
    }
  } else if (gl < nl) {
    const bool vec = group_vec<S, G>(bin, in, a.in_st, gl, nl);
    const S* src = in + bin[gl];
    for (int i = r0; i < n32; i += RS) {
      C* dst = sm + i * P + gl;
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
  // columns past nl (last tile) hold stale shared memory: filtered, never stored
  if (threadIdx.x * V < nl) filter_line(TileCols<C, P, V>{sm + threadIdx.x * V}, n32, a);
  __syncthreads();
  if (a.line_major) {
    for (int qd = warp; qd * 4 < nl; qd += NW) {
      const int l = qd * 4 + qs;
      if (l >= nl) continue;
      S* dst = out + bout[l];
      const C* src = sm + l;
      for (int i = qj; i < n32; i += 8) dst[i * a.out_st] = ppk::from_acc<S>(src[i * P]);
    }
  } else if (gl < nl) {
    const bool vec = group_vec<S, G>(bout, out, a.out_st, gl, nl);
    S* dst = out + bout[gl];
    for (int i = r0; i < n32; i += RS) {
      const C* src = sm + i * P + gl;
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

// Long-line kernel: LL threads, up to LL lines per CTA, one per thread, with
// a runtime pitch (fewer lines for longer lines, up to 200 KB of shared
// memory): odd when warps stage whole lines (conflict-free column writes),
// else a multiple of G = 16 / sizeof(C) for the group copies.
constexpr int LL = 64;

template <class S>
__global__ void __launch_bounds__(LL) coeff_smem_kernel(LineArgs a, int pitch, int lines) {
  using C = typename ppk::Acc<S>::type;
  constexpr int G = 16 / static_cast<int>(sizeof(C));
  constexpr int GPR = LL / G;  // groups per sample row
  constexpr int NW = LL / 32;
  constexpr bool kAsync = sizeof(S) == sizeof(C);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  const int64_t l0 = static_cast<int64_t>(blockIdx.x) * lines;
  const int nl = static_cast<int>(a.nlines - l0 < lines ? a.nlines - l0 : lines);
  const S* in = static_cast<const S*>(a.in);
  S* out = static_cast<S*>(a.out);
  __shared__ int64_t bin[LL], bout[LL];
  for (int l = threadIdx.x; l < nl; l += LL) line_base(a, l0 + l, bin[l], bout[l]);
  __syncthreads();
  const int n32 = static_cast<int>(a.n);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool gvec_ok = (pitch % G) == 0;
  const int gl = (threadIdx.x % GPR) * G, r0 = threadIdx.x / GPR;  // strided: group line, first row
  if (a.line_major) {
    for (int l = warp; l < nl; l += NW) {
      const S* src = in + bin[l];
      C* dst = sm + l;
      for (int i = lane; i < n32; i += 32) {
        if constexpr (kAsync) cp_async<sizeof(C)>(dst + i * pitch, src + i * a.in_st);
        else dst[i * pitch] = ppk::to_acc(src[i * a.in_st]);
      }
    }
  } else if (gl < nl) {
    const bool vec = gvec_ok && group_vec<S, G>(bin, in, a.in_st, gl, nl);
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
  if (threadIdx.x < nl) filter_line(TileLine<C>{sm + threadIdx.x, pitch}, n32, a);
  __syncthreads();
  if (a.line_major) {
    for (int l = warp; l < nl; l += NW) {
      S* dst = out + bout[l];
      const C* src = sm + l;
      for (int i = lane; i < n32; i += 32) dst[i * a.out_st] = ppk::from_acc<S>(src[i * pitch]);
    }
  } else if (gl < nl) {
    const bool vec = gvec_ok && group_vec<S, G>(bout, out, a.out_st, gl, nl);
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

template <class K>
int allow_smem(K k, size_t smem, size_t static_bytes) {
  // the 48 KB default covers static (line bases) plus dynamic shared memory
  if (smem + static_bytes <= 48 * 1024) return PP_OK;
  return ppc::cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                         "prefilter smem attribute");
}

template <class S, int NT, int V>
int launch_tile(const LineArgs& a, size_t smem, cudaStream_t st) {
  auto k = coeff_tile_kernel<S, NT, V>;
  if (int rc = allow_smem(k, smem, 2 * NT * sizeof(int64_t))) return rc;
  const int64_t blocks = (a.nlines + NT - 1) / NT;
  k<<<static_cast<unsigned>(blocks), TILE_THREADS, smem, st>>>(a);
  ppc::count_launch();
  return ppc::cuda_check(cudaGetLastError(), "prefilter launch");
}

template <class S>
int launch_tiles(const LineArgs& a, int NT, size_t smem, cudaStream_t st) {
  switch (NT) {
    case 128: return launch_tile<S, 128, TILE_V>(a, smem, st);
    case 96: return launch_tile<S, 96, TILE_V>(a, smem, st);
    case 64: return launch_tile<S, 64, TILE_V>(a, smem, st);
    default: return launch_tile<S, 32, TILE_V>(a, smem, st);
  }
}

template <class S>
int run_axis(LineArgs& a, cudaStream_t st) {
  using C = typename ppk::Acc<S>::type;
  constexpr int G = 16 / static_cast<int>(sizeof(C));
  if (a.nlines == 0) return PP_OK;
  const size_t budget = 200 * 1024;
  // full tiles: the widest NT (multiple of 32, at most 128) whose tile
  // leaves room for two CTAs per SM
  {
    const int64_t fit = static_cast<int64_t>(113 * 1024 / (static_cast<size_t>(a.n) * sizeof(C))) - 4;
    const int NT = fit >= 128 ? 128 : fit >= 96 ? 96 : fit >= 64 ? 64 : fit >= 32 ? 32 : 0;
    if (NT > 0) {
      const size_t smem = static_cast<size_t>(a.n) * (NT + 4) * sizeof(C);
      return launch_tiles<S>(a, NT, smem, st);
    }
  }
  // longer lines: fewer per CTA, one per thread
  const int64_t fit = static_cast<int64_t>(budget / (static_cast<size_t>(a.n) * sizeof(C)));
  int lines = static_cast<int>(fit < LL ? fit : LL), pitch = 0;
  if (a.line_major) {
    pitch = lines | 1;
    if (static_cast<int64_t>(pitch) > fit) pitch = --lines;  // lines was even: drop one
  } else {
    if (lines >= G) lines -= lines % G;
    pitch = lines;
  }
  if (lines >= 1) {
    const size_t smem = static_cast<size_t>(a.n) * pitch * sizeof(C);
    auto k = coeff_smem_kernel<S>;
    if (int rc = allow_smem(k, smem, 2 * LL * sizeof(int64_t))) return rc;
    const int64_t blocks = (a.nlines + lines - 1) / lines;
    k<<<static_cast<unsigned>(blocks), LL, smem, st>>>(a, pitch, lines);
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
