// Source-sorted processing order of the sampling points.
//
// With a rough deformation, the 32 lanes of a warp (consecutive grid voxels)
// sample source points scattered over a wide neighbourhood: every gather and
// every scatter instruction touches ~30 distinct 32-byte sectors.  Processing
// the sampling points in the order of their source voxel makes consecutive
// lanes sample neighbouring source voxels again, so taps coalesce and
// scatter atomics hit a few lines per instruction.
//
// pp_sample_order computes that order -- a permutation of the grid's sample
// indices sorted by the linear index (batch item, then the source voxel
// floor(coords) clamped into the volume, last axis fastest) -- with a
// counting sort.  (3-D grids of the cubic brick kernels use the brick-major
// order of pp_brick_order below instead.)
// Steps:
//   1. key / rank: key = source voxel, rank = atomicAdd(&count[key], 1);
//   2. exclusive scan of count (block reduce, scan of block sums, apply);
//   3. perm[offset[key] + rank] = sample.
// The permutation only depends on the grid, so the forward and backward
// kernels of a step share one.  Order within a source voxel is arbitrary.
#include <mutex>

#include "pp_capi_internal.cuh"
#include "pp_kernels.cuh"

namespace {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

struct KeyArgs {
  const void* grid;
  int64_t N;
  int64_t size[3];       // grid spatial sizes
  int64_t src[3];        // source spatial sizes
  int64_t gsN, gs[3], gsD;
  int D;
  int64_t nvox;
  int64_t nsrc;          // number of keys per batch item (source voxels)
};

// Number of keys per batch item (source voxels) for sizes src[0..D-1].
inline int64_t key_geometry(KeyArgs& a, int D, const int64_t* src) {
  int64_t n = 1;
  for (int d = 0; d < D; ++d) n *= src[d];
  a.nsrc = n;
  return n;
}

// One thread per sampling point.  Index arithmetic in 32 bits (the host
// guarantees fewer than 2^31 samples and keys); memory offsets in 64.
template <class T>
__global__ void order_keys(KeyArgs a, int32_t* count, int32_t* keys, int32_t* ranks) {
  const unsigned s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= static_cast<unsigned>(a.nvox)) return;
  int v = static_cast<int>(s), sub[3] = {0, 0, 0};
  for (int d = a.D - 1; d >= 0; --d) {
    const int n = static_cast<int>(a.size[d]);
    const int q = v / n;
    sub[d] = v - q * n;
    v = q;
  }
  const T* g = static_cast<const T*>(a.grid) + static_cast<int64_t>(v) * a.gsN;
  for (int d = 0; d < a.D; ++d) g += static_cast<int64_t>(sub[d]) * a.gs[d];
  int lin = 0;
  for (int d = 0; d < a.D; ++d) {
    const T c = g[d * a.gsD];
    const int n = static_cast<int>(a.src[d]);
    // floor, clamped into the volume (NaN -> 0)
    const int i = (c >= T(0)) ? static_cast<int>(fmin(c, static_cast<T>(n - 1))) : 0;
    lin = lin * n + i;
  }
  const int32_t key = v * static_cast<int>(a.nsrc) + lin;
  keys[s] = key;
  ranks[s] = atomicAdd(count + key, 1);
}

__device__ __forceinline__ int32_t block_exclusive_scan(int32_t x, int32_t& total) {
  __shared__ int32_t warp_sums[SCAN_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int32_t inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_sums[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int32_t ws = lane < SCAN_THREADS / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += y;
    }
    if (lane < SCAN_THREADS / 32) warp_sums[lane] = ws;
  }
  __syncthreads();
  const int32_t before = wid > 0 ? warp_sums[wid - 1] : 0;
  total = warp_sums[SCAN_THREADS / 32 - 1];
  __syncthreads();
  return before + inc - x;
}

// 2a. per-tile sums
__global__ void __launch_bounds__(SCAN_THREADS) scan_reduce(const int32_t* in, int64_t n, int32_t* partial) {
  const int64_t base = static_cast<int64_t>(blockIdx.x) * SCAN_TILE;
  int32_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const int64_t i = base + static_cast<int64_t>(k) * SCAN_THREADS + threadIdx.x;
    if (i < n) s += in[i];
  }
  int32_t total;
  block_exclusive_scan(s, total);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// 2b. exclusive scan of the tile sums, one CTA (sequential chunks of SCAN_THREADS)
__global__ void __launch_bounds__(SCAN_THREADS) scan_partials(int32_t* partial, int64_t np) {
  int32_t carry = 0;
  for (int64_t base = 0; base < np; base += SCAN_THREADS) {
    const int64_t i = base + threadIdx.x;
    const int32_t x = i < np ? partial[i] : 0;
    int32_t total;
    const int32_t ex = block_exclusive_scan(x, total);
    if (i < np) partial[i] = carry + ex;
    carry += total;
  }
}

// 2c. exclusive scan inside each tile, plus the tile's offset (in place)
__global__ void __launch_bounds__(SCAN_THREADS) scan_apply(int32_t* data, int64_t n, const int32_t* partial) {
  const int64_t base = static_cast<int64_t>(blockIdx.x) * SCAN_TILE + static_cast<int64_t>(threadIdx.x) * SCAN_ITEMS;
  int32_t v[SCAN_ITEMS];
  int32_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    v[k] = (base + k < n) ? data[base + k] : 0;
    s += v[k];
  }
  int32_t total;
  int32_t run = block_exclusive_scan(s, total) + partial[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    if (base + k < n) data[base + k] = run;
    run += v[k];
  }
}

__global__ void order_scatter(const int32_t* keys, const int32_t* ranks, const int32_t* offset,
                              int64_t nvox, int32_t* perm) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= nvox) return;
  perm[offset[keys[s]] + ranks[s]] = static_cast<int32_t>(s);
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

struct Layout {
  size_t count, keys, ranks, partial, total;
};

Layout layout(int64_t nvox, int64_t nsrc_total) {
  Layout L;
  const int64_t ntile = (nsrc_total + SCAN_TILE - 1) / SCAN_TILE;
  L.count = 0;
  L.keys = L.count + align256(static_cast<size_t>(nsrc_total) * 4);
  L.ranks = L.keys + align256(static_cast<size_t>(nvox) * 4);
  L.partial = L.ranks + align256(static_cast<size_t>(nvox) * 4);
  L.total = L.partial + align256(static_cast<size_t>(ntile > 0 ? ntile : 1) * 4);
  return L;
}

int sizes_of(const pp_tensor* grid, const int64_t* src_size, int& D, int64_t& nvox, int64_t& nsrc) {
  int rc = ppc::check_tensor(grid, "grid");
  if (rc) return rc;
  if (grid->ndim < 3 || grid->ndim > 5)
    return ppc::fail(PP_ERR_ARG, "(): expected 3D, 4D or 5D grid but got input with %d dimensions", grid->ndim);
  D = grid->ndim - 2;
  if (grid->sizes[grid->ndim - 1] != D)
    return ppc::fail(PP_ERR_ARG, "(): expected grid to have size %d in last dimension", D);
  if (grid->dtype != PP_FLOAT32 && grid->dtype != PP_FLOAT64)
    return ppc::fail(PP_ERR_DTYPE, "(): expected grid to be float32 or float64");
  if (!src_size) return ppc::fail(PP_ERR_ARG, "(): expected source sizes");
  nvox = grid->sizes[0];
  for (int d = 0; d < D; ++d) {
    if (src_size[d] <= 0 || grid->sizes[1 + d] <= 0) return ppc::fail(PP_ERR_ARG, "(): expected non-empty sizes");
    nvox *= grid->sizes[1 + d];
  }
  KeyArgs tmp;
  nsrc = key_geometry(tmp, D, src_size);
  if (nvox >= (int64_t(1) << 31) || nsrc * grid->sizes[0] >= (int64_t(1) << 31))
    return ppc::fail(PP_ERR_UNSUPPORTED, "(): sample ordering needs fewer than 2^31 samples and source voxels");
  return PP_OK;
}

// ---------------------------------------------------------------------------
// Brick-major order (3-D): the same counting sort with the key
//   ((n * NBX + bx) * NBY + by) * NBZ + bz) * BRICK + local
// of the clamped floor voxel (x, y, z), (bx, by, bz) its brick and `local`
// its index inside the brick (z fastest), so that the samples of one brick
// are consecutive.  The brick kernels read brick b's samples from
// perm[brick_start[b] .. brick_start[b + 1]).
// ---------------------------------------------------------------------------
constexpr int BRK[3] = {PP_BRICK_X, PP_BRICK_Y, PP_BRICK_Z};
constexpr int BRK_VOL = PP_BRICK_X * PP_BRICK_Y * PP_BRICK_Z;

struct BrickGeom {
  int64_t nb[3];     // bricks per axis
  int64_t per_item;  // bricks per batch item
  int64_t nkeys;     // N * per_item * BRK_VOL
};

BrickGeom brick_geometry(int64_t N, const int64_t* src) {
  BrickGeom g;
  g.per_item = 1;
  for (int d = 0; d < 3; ++d) {
    g.nb[d] = (src[d] + BRK[d] - 1) / BRK[d];
    g.per_item *= g.nb[d];
  }
  g.nkeys = N * g.per_item * BRK_VOL;
  return g;
}

template <class T>
__global__ void brick_keys(KeyArgs a, int nbx, int nby, int nbz, int32_t* count, int32_t* keys, int32_t* ranks) {
  const unsigned s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= static_cast<unsigned>(a.nvox)) return;
  int v = static_cast<int>(s), sub[3];
  for (int d = 2; d >= 0; --d) {
    const int n = static_cast<int>(a.size[d]);
    const int q = v / n;
    sub[d] = v - q * n;
    v = q;
  }
  const T* g = static_cast<const T*>(a.grid) + static_cast<int64_t>(v) * a.gsN;
  for (int d = 0; d < 3; ++d) g += static_cast<int64_t>(sub[d]) * a.gs[d];
  int f[3];
  for (int d = 0; d < 3; ++d) {
    const T c = g[d * a.gsD];
    const int n = static_cast<int>(a.src[d]);
    f[d] = (c >= T(0)) ? static_cast<int>(fmin(c, static_cast<T>(n - 1))) : 0;  // NaN -> 0
  }
  const int bx = f[0] / PP_BRICK_X, by = f[1] / PP_BRICK_Y, bz = f[2] / PP_BRICK_Z;
  const int local = ((f[0] - bx * PP_BRICK_X) * PP_BRICK_Y + (f[1] - by * PP_BRICK_Y)) * PP_BRICK_Z +
                    (f[2] - bz * PP_BRICK_Z);
  const int32_t key = (((v * nbx + bx) * nby + by) * nbz + bz) * BRK_VOL + local;
  keys[s] = key;
  ranks[s] = atomicAdd(count + key, 1);
}

// The brick pass's scatter: perm[pos] = s and, when `rec` is given, the
// sample's coordinates and index as one 16-byte record at the same position
// (read here once, coalesced by s, so that the brick kernels read each
// sample's data in brick order without the perm -> grid indirection).
__global__ void brick_scatter(KeyArgs a, const int32_t* keys, const int32_t* ranks, const int32_t* offset,
                              int32_t* perm, float4* rec) {
  const unsigned s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= static_cast<unsigned>(a.nvox)) return;
  const int32_t pos = offset[keys[s]] + ranks[s];
  perm[pos] = static_cast<int32_t>(s);
  if (rec) {
    int v = static_cast<int>(s), sub[3];
    for (int d = 2; d >= 0; --d) {
      const int n = static_cast<int>(a.size[d]);
      const int q = v / n;
      sub[d] = v - q * n;
      v = q;
    }
    const float* g = static_cast<const float*>(a.grid) + static_cast<int64_t>(v) * a.gsN;
    for (int d = 0; d < 3; ++d) g += static_cast<int64_t>(sub[d]) * a.gs[d];
    rec[pos] = make_float4(g[0], g[a.gsD], g[2 * a.gsD], __int_as_float(static_cast<int>(s)));
  }
}

// brick_start[b] = offset of brick b's first key; brick_start[nb] = nvox
__global__ void brick_starts(const int32_t* offset, int64_t nbricks, int32_t nvox, int32_t* start) {
  const int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b < nbricks) start[b] = offset[b * BRK_VOL];
  else if (b == nbricks) start[b] = nvox;
}

int brick_sizes_of(const pp_tensor* grid, const int64_t* src_size, int64_t& nvox, BrickGeom& g) {
  int D;
  int64_t nsrc;
  int rc = sizes_of(grid, src_size, D, nvox, nsrc);
  if (rc) return rc;
  if (D != 3) return ppc::fail(PP_ERR_UNSUPPORTED, "(): brick ordering needs a 3-D grid");
  g = brick_geometry(grid->sizes[0], src_size);
  if (g.nkeys >= (int64_t(1) << 31))
    return ppc::fail(PP_ERR_UNSUPPORTED, "(): brick ordering needs fewer than 2^31 brick voxels");
  return PP_OK;
}

}  // namespace

extern "C" {

int64_t pp_brick_count(const pp_tensor* grid, const int64_t* src_size) {
  int64_t nvox;
  BrickGeom g;
  if (brick_sizes_of(grid, src_size, nvox, g)) return -1;
  return grid->sizes[0] * g.per_item;
}

size_t pp_brick_order_workspace_bytes(const pp_tensor* grid, const int64_t* src_size) {
  int64_t nvox;
  BrickGeom g;
  if (brick_sizes_of(grid, src_size, nvox, g)) return 0;
  return layout(nvox, g.nkeys).total;
}

int pp_brick_order(const pp_tensor* grid, const int64_t* src_size, int32_t* perm, int32_t* brick_start,
                   float* records, void* workspace, size_t workspace_bytes, void* stream) {
  int64_t nvox;
  BrickGeom g;
  int rc = brick_sizes_of(grid, src_size, nvox, g);
  if (rc) return rc;
  if (!perm || !brick_start) return ppc::fail(PP_ERR_ARG, "(): expected an output permutation and brick offsets");
  if (records && (grid->dtype != PP_FLOAT32 || reinterpret_cast<uintptr_t>(records) % 16 != 0))
    return ppc::fail(PP_ERR_ARG, "(): brick records need a float32 grid and a 16-byte aligned buffer");
  const Layout L = layout(nvox, g.nkeys);
  if (!workspace || workspace_bytes < L.total)
    return ppc::fail(PP_ERR_WORKSPACE, "(): brick ordering needs %zu bytes of workspace", L.total);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t nbricks = grid->sizes[0] * g.per_item;
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  int32_t* count = reinterpret_cast<int32_t*>(ws + L.count);
  int32_t* keys = reinterpret_cast<int32_t*>(ws + L.keys);
  int32_t* ranks = reinterpret_cast<int32_t*>(ws + L.ranks);
  int32_t* partial = reinterpret_cast<int32_t*>(ws + L.partial);
  if ((rc = ppc::cuda_check(cudaMemsetAsync(count, 0, static_cast<size_t>(g.nkeys) * 4, st), "brick order clear")))
    return rc;
  KeyArgs a;
  a.grid = grid->data;
  a.N = grid->sizes[0];
  a.D = 3;
  a.gsN = grid->strides[0];
  a.gsD = grid->strides[4];
  for (int d = 0; d < 3; ++d) {
    a.size[d] = grid->sizes[1 + d];
    a.src[d] = src_size[d];
    a.gs[d] = grid->strides[1 + d];
  }
  a.nvox = nvox;
  a.nsrc = g.per_item * BRK_VOL;
  if (nvox > 0) {
    const unsigned nb = static_cast<unsigned>((nvox + 255) / 256);
    const int nbx = static_cast<int>(g.nb[0]), nby = static_cast<int>(g.nb[1]), nbz = static_cast<int>(g.nb[2]);
    if (grid->dtype == PP_FLOAT32) brick_keys<float><<<nb, 256, 0, st>>>(a, nbx, nby, nbz, count, keys, ranks);
    else brick_keys<double><<<nb, 256, 0, st>>>(a, nbx, nby, nbz, count, keys, ranks);
    const int64_t ntile = (g.nkeys + SCAN_TILE - 1) / SCAN_TILE;
    scan_reduce<<<static_cast<unsigned>(ntile), SCAN_THREADS, 0, st>>>(count, g.nkeys, partial);
    scan_partials<<<1, SCAN_THREADS, 0, st>>>(partial, ntile);
    scan_apply<<<static_cast<unsigned>(ntile), SCAN_THREADS, 0, st>>>(count, g.nkeys, partial);
    brick_scatter<<<nb, 256, 0, st>>>(a, keys, ranks, count, perm, reinterpret_cast<float4*>(records));
    ppc::count_launch(5);
  }
  brick_starts<<<static_cast<unsigned>((nbricks + 1 + 255) / 256), 256, 0, st>>>(count, nbricks,
                                                                                 static_cast<int32_t>(nvox), brick_start);
  ppc::count_launch();
  return ppc::cuda_check(cudaGetLastError(), "brick order launch");
}

size_t pp_sample_order_workspace_bytes(const pp_tensor* grid, const int64_t* src_size) {
  int D;
  int64_t nvox, nsrc;
  if (sizes_of(grid, src_size, D, nvox, nsrc)) return 0;
  return layout(nvox, nsrc * grid->sizes[0]).total;
}

int pp_sample_order(const pp_tensor* grid, const int64_t* src_size, int32_t* perm,
                    void* workspace, size_t workspace_bytes, void* stream) {
  int D;
  int64_t nvox, nsrc;
  int rc = sizes_of(grid, src_size, D, nvox, nsrc);
  if (rc) return rc;
  if (!perm) return ppc::fail(PP_ERR_ARG, "(): expected an output permutation");
  const int64_t nsrc_total = nsrc * grid->sizes[0];
  const Layout L = layout(nvox, nsrc_total);
  if (!workspace || workspace_bytes < L.total)
    return ppc::fail(PP_ERR_WORKSPACE, "(): sample ordering needs %zu bytes of workspace", L.total);
  if (nvox == 0) return PP_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  int32_t* count = reinterpret_cast<int32_t*>(ws + L.count);
  int32_t* keys = reinterpret_cast<int32_t*>(ws + L.keys);
  int32_t* ranks = reinterpret_cast<int32_t*>(ws + L.ranks);
  int32_t* partial = reinterpret_cast<int32_t*>(ws + L.partial);
  if ((rc = ppc::cuda_check(cudaMemsetAsync(count, 0, static_cast<size_t>(nsrc_total) * 4, st), "order clear"))) return rc;
  KeyArgs a;
  a.grid = grid->data;
  a.N = grid->sizes[0];
  a.D = D;
  a.gsN = grid->strides[0];
  a.gsD = grid->strides[1 + D];
  for (int d = 0; d < 3; ++d) {
    a.size[d] = d < D ? grid->sizes[1 + d] : 1;
    a.src[d] = d < D ? src_size[d] : 1;
    a.gs[d] = d < D ? grid->strides[1 + d] : 0;
  }
  a.nvox = nvox;
  a.nsrc = key_geometry(a, D, src_size);
  const unsigned nb = static_cast<unsigned>((nvox + 255) / 256);
  if (grid->dtype == PP_FLOAT32) order_keys<float><<<nb, 256, 0, st>>>(a, count, keys, ranks);
  else order_keys<double><<<nb, 256, 0, st>>>(a, count, keys, ranks);
  const int64_t ntile = (nsrc_total + SCAN_TILE - 1) / SCAN_TILE;
  scan_reduce<<<static_cast<unsigned>(ntile), SCAN_THREADS, 0, st>>>(count, nsrc_total, partial);
  scan_partials<<<1, SCAN_THREADS, 0, st>>>(partial, ntile);
  scan_apply<<<static_cast<unsigned>(ntile), SCAN_THREADS, 0, st>>>(count, nsrc_total, partial);
  order_scatter<<<nb, 256, 0, st>>>(keys, ranks, count, nvox, perm);
  ppc::count_launch(5);
  return ppc::cuda_check(cudaGetLastError(), "sample order launch");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Sample ordering without any device allocation.
//
// Some callers cannot allocate device memory at the moment they need an
// order: hosts that drive this library through its C ABI from a runtime that
// owns all device memory up front or works under a fixed memory budget
// (plugins of another framework, real-time pipelines).  For them,
// pp_sample_order_noalloc uses a scratch area that is part of the library
// image instead of a caller-provided workspace.
//
// The scratch is a file-scope device array of NOALLOC_SCRATCH_BYTES (16 MiB);
// every GPU that loads the library holds it until the process exits.  It
// covers grids whose counting-sort state fits in it: 4 bytes per source voxel
// (times the batch) plus 8 bytes per sampling point, e.g. up to ~1.3 M
// sampling points into a ~1.3 M-voxel source.  Larger requests are rejected
// with PP_ERR_WORKSPACE.  All calls share the one array: calls whose work
// overlaps on the GPU (different streams, or several host threads) race and
// must be serialised by the caller.  The scratch address is looked up once
// per device number, in the context current at the first call: callers must
// use the device's primary context (the runtime API's), and no
// cudaDeviceReset may follow the first call on that device.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(16) << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch per device, looked up once per device
// with that device current (host code cannot use the symbol itself).
constexpr int NOALLOC_MAX_DEVICES = 64;
void* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {nullptr};
std::mutex g_noalloc_mutex;

int noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return ppc::cuda_check(e, "noalloc: current device");
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return ppc::fail(PP_ERR_UNSUPPORTED, "(): device index %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return ppc::cuda_check(e, "noalloc: scratch address");
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return PP_OK;
}

}  // namespace

extern "C" {

int pp_sample_order_noalloc(const pp_tensor* grid, const int64_t* src_size, int32_t* perm, void* stream) {
  int D;
  int64_t nvox, nsrc;
  int rc = sizes_of(grid, src_size, D, nvox, nsrc);
  if (rc) return rc;
  if (!perm) return ppc::fail(PP_ERR_ARG, "(): expected an output permutation");
  const int64_t nsrc_total = nsrc * grid->sizes[0];
  const Layout L = layout(nvox, nsrc_total);
  if (L.total > NOALLOC_SCRATCH_BYTES)
    return ppc::fail(PP_ERR_WORKSPACE,
                     "(): pp_sample_order_noalloc needs %zu bytes of scratch for %lld sampling points "
                     "and %lld source voxels; its fixed scratch holds %zu bytes (use pp_sample_order "
                     "with a workspace instead)",
                     L.total, (long long)nvox, (long long)nsrc_total, NOALLOC_SCRATCH_BYTES);
  void* scratch = nullptr;
  if ((rc = noalloc_scratch(&scratch))) return rc;
  if (nvox == 0) return PP_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* ws = static_cast<unsigned char*>(scratch);
  int32_t* count = reinterpret_cast<int32_t*>(ws + L.count);
  int32_t* keys = reinterpret_cast<int32_t*>(ws + L.keys);
  int32_t* ranks = reinterpret_cast<int32_t*>(ws + L.ranks);
  int32_t* partial = reinterpret_cast<int32_t*>(ws + L.partial);
  // the histogram must start at zero; the scratch keeps the previous call's data
  if ((rc = ppc::cuda_check(cudaMemsetAsync(count, 0, static_cast<size_t>(nsrc_total) * 4, st), "noalloc clear")))
    return rc;
  KeyArgs a;
  a.grid = grid->data;
  a.N = grid->sizes[0];
  a.D = D;
  a.gsN = grid->strides[0];
  a.gsD = grid->strides[1 + D];
  for (int d = 0; d < 3; ++d) {
    a.size[d] = d < D ? grid->sizes[1 + d] : 1;
    a.src[d] = d < D ? src_size[d] : 1;
    a.gs[d] = d < D ? grid->strides[1 + d] : 0;
  }
  a.nvox = nvox;
  a.nsrc = key_geometry(a, D, src_size);
  const unsigned nb = static_cast<unsigned>((nvox + 255) / 256);
  if (grid->dtype == PP_FLOAT32) order_keys<float><<<nb, 256, 0, st>>>(a, count, keys, ranks);
  else order_keys<double><<<nb, 256, 0, st>>>(a, count, keys, ranks);
  const int64_t ntile = (nsrc_total + SCAN_TILE - 1) / SCAN_TILE;
  scan_reduce<<<static_cast<unsigned>(ntile), SCAN_THREADS, 0, st>>>(count, nsrc_total, partial);
  scan_partials<<<1, SCAN_THREADS, 0, st>>>(partial, ntile);
  scan_apply<<<static_cast<unsigned>(ntile), SCAN_THREADS, 0, st>>>(count, nsrc_total, partial);
  order_scatter<<<nb, 256, 0, st>>>(keys, ranks, count, nvox, perm);
  ppc::count_launch(5);
  return ppc::cuda_check(cudaGetLastError(), "sample order (no-alloc) launch");
}

}  // extern "C"
