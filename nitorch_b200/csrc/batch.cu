// Batched launches: many independent 3-D volumes (uneven shapes, 1-4+
// channels, isotropic orders 0-3, float32 or bfloat16 images) of one mode in
// a few launches, no device-side plan table.
//
// The reference processes one tensor per call (nitorch/_C/src/pushpull.cpp:
// 76-327); a loop over subjects pays a launch and a host round trip per
// volume and op.  Here pp_batch_plan sorts the volumes into groups of equal
// (order, channel block) -- the compile-time parameters of the per-point
// body -- and pp_batch_run launches each group as ONE kernel whose argument
// carries the per-volume arguments of up to kMaxEntries volumes by value
// (a __grid_constant__ kernel parameter of < 32 KB, read through the
// constant cache like the single-tensor kernel's arguments).  A CTA is one
// work item of kBatchPoints consecutive sampling points of one volume; it
// finds its volume by binary search over the item prefix sums.  With
// ctas > 0 the launch is persistent instead (ctas CTAs striding over the
// items).  Everything pp_batch_run issues (zero fills and kernels) is
// stream-ordered and takes no host synchronisation.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/nitorch_b200.h"
#include "batch_kernel.cuh"

#define PB_DECL(S)                                                                               \
  cudaError_t pp_batch_launch_##S##_m0(int, int, const ppb::BatchLaunch&, int, cudaStream_t);  \
  cudaError_t pp_batch_launch_##S##_m2(int, int, const ppb::BatchLaunch&, int, cudaStream_t);  \
  cudaError_t pp_batch_launch_##S##_m4(int, int, const ppb::BatchLaunch&, int, cudaStream_t);  \
  cudaError_t pp_batch_launch_##S##_m5(int, int, const ppb::BatchLaunch&, int, cudaStream_t);  \
  cudaError_t pp_batch_launch_##S##_m7(int, int, const ppb::BatchLaunch&, int, cudaStream_t);  \
  cudaError_t pp_batch_launch_##S##_m8(int, int, const ppb::BatchLaunch&, int, cudaStream_t);
PB_DECL(f32)
PB_DECL(bf16)
#undef PB_DECL
#define PB_ROW(S)                                                                                 \
  {pp_batch_launch_##S##_m0, nullptr, pp_batch_launch_##S##_m2, nullptr, pp_batch_launch_##S##_m4, \
   pp_batch_launch_##S##_m5, nullptr, pp_batch_launch_##S##_m7, pp_batch_launch_##S##_m8}
static const pb_launcher_t kBatchLaunchers[2][ppk::K_NMODES] = {PB_ROW(f32), PB_ROW(bf16)};
#undef PB_ROW

namespace ppb {

constexpr int kMaxGroups = 16;     // (order 0-3) x (channel block 1-4)
constexpr uint32_t kMagic = 0x50504231u;

// Interleaved float accumulator (X*Y*Z*CP floats, channel fastest) of one
// volume -> its contiguous float32 output (1, C, X, Y, Z).
struct VecStore {
  const float* acc;
  float* out;
  int64_t V;
  int32_t C, CP;
};
constexpr int kMaxStores = 256;
struct StoreLaunch {
  int32_t n, pad;
  int64_t first[kMaxStores + 1];  // voxel prefix sums (V per volume)
  VecStore s[kMaxStores];
};
static_assert(sizeof(StoreLaunch) <= 32764, "store argument above the kernel-parameter limit");

// One thread per voxel: its CP accumulator slots (consecutive, so a warp
// reads whole sectors) to the C channel planes of the output (coalesced).
__global__ void __launch_bounds__(256) batch_store_kernel(const __grid_constant__ StoreLaunch L) {
  const int64_t total = L.first[L.n];
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int lo = 0, hi = L.n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (L.first[mid] <= i) lo = mid; else hi = mid - 1;
    }
    const VecStore& v = L.s[lo];
    const int64_t lin = i - L.first[lo];
    const float* a = v.acc + lin * v.CP;
    float* o = v.out + lin;
    for (int c = 0; c < v.C; ++c) o[c * v.V] = a[c];
  }
}


// Deterministic scatter entry: its int64 fixed-point accumulator (after a
// 256-byte header holding max |t| as float bits) in the scratch, the tensor
// that max is taken over, and the output the accumulator is finalized into.
struct DetJob {
  unsigned int* mx;
  unsigned long long* acc;
  double bound;
  pp_tensor tmax, out;
};

struct PlanHeader {
  uint32_t magic;
  int32_t mode, ctas, nvol, dtype, ngroups, nfill, nstore, ndet, pad;
  int32_t gfirst[kMaxGroups], gcount[kMaxGroups], gorder[kMaxGroups], gcb[kMaxGroups];
};

struct Fill {  // a byte range to zero before the launches
  void* ptr;
  size_t bytes;
};

// Layout of the host plan buffer: header, then per volume its PPArgs and its
// item count (sorted by group), the fill ranges, the interleaved stores,
// then the deterministic entries.
inline size_t plan_bytes(int nvol) {
  return sizeof(PlanHeader) + static_cast<size_t>(nvol) * (sizeof(ppk::PPArgs) + sizeof(int64_t) + sizeof(Fill) +
                                                           sizeof(VecStore) + sizeof(DetJob));
}

// Scratch of a deterministic scatter entry: header + int64 per output element.
inline size_t det_bytes(const pp_tensor& out) {
  return 256 + ((static_cast<size_t>(ppc::numel(&out)) * 8 + 255) / 256) * 256;
}

// Channel slots of the interleaved accumulator of a scatter entry (0: the
// entry scatters with scalar reductions): 2-4 channels, orders 2 and 3
// (orders 0-1 scatter few taps, where the extra store pass does not pay).
inline int entry_slots(int mode, int64_t C, int iso) {
  const bool scatter = mode == ppk::K_PUSH || mode == ppk::K_PUSHGRAD || mode == ppk::K_PP || mode == ppk::K_PP_BWD;
  if (!scatter || iso < 2 || iso > 3 || !ppk::lanes_enabled()) return 0;
  return C == 2 ? 2 : (C == 3 || C == 4) ? 4 : 0;
}

bool is_scatter(int mode) {
  return mode == ppk::K_PUSH || mode == ppk::K_PUSHGRAD || mode == ppk::K_PP || mode == ppk::K_PP_BWD;
}

}  // namespace ppb

using namespace ppc;
using namespace ppb;

extern "C" {

size_t pp_batch_plan_bytes(int32_t nvol) { return nvol > 0 ? plan_bytes(nvol) : 0; }

// Device scratch for the channel-interleaved accumulators of the entries
// that scatter with vector reductions and the fixed-point accumulators of
// the deterministic scatter entries (0 if there are none).
size_t pp_batch_scratch_bytes(const pp_batch_entry* items, int32_t nvol, int32_t mode) {
  if (!items || nvol <= 0) return 0;
  size_t total = 0;
  for (int v = 0; v < nvol; ++v) {
    const pp_batch_entry& it = items[v];
    if (!it.out.data || it.out.ndim != 5) continue;
    if (it.opt.flags & PP_DETERMINISTIC) {
      if (is_scatter(mode)) total += det_bytes(it.out);
      continue;
    }
    int bound[3], ord[3];
    if (read_options(&it.opt, 3, bound, ord)) continue;
    const int iso = (ord[0] == ord[1] && ord[0] == ord[2]) ? ord[0] : -1;
    const int CP = entry_slots(mode, it.out.sizes[1], iso);
    if (!CP) continue;
    const int64_t V = it.out.sizes[2] * it.out.sizes[3] * it.out.sizes[4];
    total += ((static_cast<size_t>(V) * CP * 4 + 255) / 256) * 256;
  }
  return total;
}

int pp_batch_plan(const pp_batch_entry* items, int32_t nvol, int32_t mode, int32_t ctas, void* plan,
                  size_t plan_bytes_, void* scratch, size_t scratch_bytes) {
  if (!items || nvol <= 0) return fail(PP_ERR_ARG, "(): expected at least one batch entry");
  if (mode != ppk::K_PULL && mode != ppk::K_PUSH && mode != ppk::K_PULLGRAD && mode != ppk::K_PUSHGRAD &&
      mode != ppk::K_PP && mode != ppk::K_PP_BWD)
    return fail(PP_ERR_UNSUPPORTED, "(): batched mode %d not supported", mode);
  if (ctas < 0) return fail(PP_ERR_ARG, "(): expected ctas >= 0");
  if (!plan || plan_bytes_ < plan_bytes(nvol))
    return fail(PP_ERR_WORKSPACE, "(): batch plan needs %zu bytes", plan_bytes(nvol));
  std::vector<ppk::PPArgs> args(nvol);
  std::vector<int> order(nvol), cbs(nvol);
  std::vector<int64_t> nitems(nvol);
  std::vector<Fill> fills;
  std::vector<VecStore> stores;
  std::vector<DetJob> dets;
  size_t scratch_used = 0;
  const bool use_scratch = scratch && scratch_bytes >= pp_batch_scratch_bytes(items, nvol, mode) &&
                           reinterpret_cast<uintptr_t>(scratch) % 256 == 0;
  int dtype = -1;
  const bool scatter = is_scatter(mode);
  for (int v = 0; v < nvol; ++v) {
    const pp_batch_entry& it = items[v];
    ppk::PPArgs& a = args[v];
    std::memset(&a, 0, sizeof(a));
    const pp_tensor* grid = &it.grid;
    if (!grid->data || grid->ndim != 5 || grid->sizes[4] != 3 || grid->sizes[0] != 1)
      return fail(PP_ERR_ARG, "(): batch entry %d: expected a (1, X, Y, Z, 3) grid", v);
    if (grid->dtype != PP_FLOAT32) return fail(PP_ERR_DTYPE, "(): batch entry %d: grid must be float32", v);
    const bool det = (it.opt.flags & PP_DETERMINISTIC) != 0;
    int bound[3], ord[3];
    int rc = read_options(&it.opt, 3, bound, ord);
    if (rc) return rc;
    const int iso = (ord[0] == ord[1] && ord[0] == ord[2]) ? ord[0] : -1;
    if (iso < 0 || iso > 3)
      return fail(PP_ERR_UNSUPPORTED, "(): batch entry %d: batched volumes need one isotropic order 0-3", v);
    for (int d = 0; d < 3; ++d) { a.bound[d] = bound[d]; a.order[d] = ord[d]; }
    a.extrapolate = it.opt.extrapolate;
    a.perm = it.opt.sample_order;
    a.grid = grid->data;
    set_grid(grid, 3, a.grid_sN, a.grid_s, a.grid_sD);
    for (int d = 0; d < 3; ++d) a.trgt_size[d] = grid->sizes[1 + d];
    a.N = 1;
    a.nvox = grid->sizes[1] * grid->sizes[2] * grid->sizes[3];
    const pp_tensor* src = it.src.data ? &it.src : nullptr;
    const pp_tensor* trg = it.trgt.data ? &it.trgt : nullptr;
    const pp_tensor* out = it.out.data ? &it.out : nullptr;
    const pp_tensor* gg = it.gg.data ? &it.gg : nullptr;
    const pp_tensor* img = src ? src : trg;
    if (!img) return fail(PP_ERR_ARG, "(): batch entry %d: no image", v);
    for (const pp_tensor* t : {src, trg, out, gg})
      if (t && (rc = check_tensor(t, "batch tensor"))) return rc;
    if (dtype < 0) dtype = img->dtype;
    if (img->dtype != dtype || (dtype != PP_FLOAT32 && dtype != PP_BFLOAT16))
      return fail(PP_ERR_DTYPE, "(): batch entries must share one float32 or bfloat16 image dtype");
    if (img->ndim != 5 || img->sizes[0] != 1) return fail(PP_ERR_ARG, "(): batch entry %d: images are (1, C, X, Y, Z)", v);
    a.C = img->sizes[1];
    // roles of the tensors per mode (see the header)
    const bool need_src = mode != ppk::K_PUSH;
    const bool need_trg = mode == ppk::K_PUSH || mode == ppk::K_PULLGRAD || mode == ppk::K_PUSHGRAD ||
                          mode == ppk::K_PP_BWD;
    if (need_src && !src) return fail(PP_ERR_ARG, "(): batch entry %d: this mode needs src", v);
    if (need_trg && !trg) return fail(PP_ERR_ARG, "(): batch entry %d: this mode needs trgt", v);
    if ((mode == ppk::K_PULL || mode == ppk::K_PUSH || mode == ppk::K_PP) && !out)
      return fail(PP_ERR_ARG, "(): batch entry %d: this mode needs out", v);
    if (!out && !gg) return fail(PP_ERR_ARG, "(): batch entry %d: nothing to compute", v);
    for (const pp_tensor* t : {src, trg, out})
      if (t && (t->ndim != 5 || t->sizes[0] != 1 || t->sizes[1] != a.C))
        return fail(PP_ERR_ARG, "(): batch entry %d: images must be (1, C, X, Y, Z) with one C", v);
    if (src) {
      set_image(src, 3, a.src_sN, a.src_sC, a.src_s);
      a.src = src->data;
      for (int d = 0; d < 3; ++d) a.src_size[d] = src->sizes[2 + d];
    }
    if (trg) {
      set_image(trg, 3, a.trgt_sN, a.trgt_sC, a.trgt_s);
      a.trgt = trg->data;
    }
    if (out) {
      set_image(out, 3, a.out_sN, a.out_sC, a.out_s);
      a.out = out->data;
      if (mode == ppk::K_PUSH) for (int d = 0; d < 3; ++d) a.src_size[d] = out->sizes[2 + d];
      if (scatter && (out->dtype != PP_FLOAT32 || !contiguous(out)))
        return fail(PP_ERR_DTYPE, "(): batch entry %d: scatter outputs must be contiguous float32", v);
      if (!scatter && out->dtype != dtype) return fail(PP_ERR_DTYPE, "(): batch entry %d: output dtype", v);
    }
    // sizes of each tensor against its role
    const int64_t* gsz = grid->sizes + 1;
    auto same_grid = [&](const pp_tensor* t) {
      return t->sizes[2] == gsz[0] && t->sizes[3] == gsz[1] && t->sizes[4] == gsz[2];
    };
    auto same_src = [&](const pp_tensor* t) {
      return t->sizes[2] == a.src_size[0] && t->sizes[3] == a.src_size[1] && t->sizes[4] == a.src_size[2];
    };
    if (trg && mode != ppk::K_PP_BWD && !same_grid(trg))
      return fail(PP_ERR_ARG, "(): batch entry %d: trgt must have the grid's spatial shape", v);
    if (out) {
      const bool grid_shaped = mode == ppk::K_PULL || mode == ppk::K_PULLGRAD;
      if (grid_shaped ? !same_grid(out) : !same_src(out))
        return fail(PP_ERR_ARG, "(): batch entry %d: out has the wrong spatial shape", v);
    }
    if (mode == ppk::K_PP_BWD)
      for (int i = 0; i < 5; ++i)
        if (src->sizes[i] != trg->sizes[i] || (src->sizes[i] > 1 && src->strides[i] != trg->strides[i]))
          return fail(PP_ERR_ARG, "(): batch entry %d: trgt must be laid out like src", v);
    if (gg) {
      if (gg->ndim != 5 || gg->dtype != PP_FLOAT32)
        return fail(PP_ERR_ARG, "(): batch entry %d: gg must be a float32 grid", v);
      for (int i = 0; i < 5; ++i)
        if (gg->sizes[i] != grid->sizes[i]) return fail(PP_ERR_ARG, "(): batch entry %d: gg has the wrong shape", v);
      if (mode == ppk::K_PULL || mode == ppk::K_PUSH || mode == ppk::K_PP)
        return fail(PP_ERR_ARG, "(): batch entry %d: this mode has no grid gradient", v);
      set_grid(gg, 3, a.gg_sN, a.gg_s, a.gg_sD);
      a.gg = gg->data;
      a.flags |= ppk::F_GRAD;
    }
    if (out && (mode == ppk::K_PULLGRAD || mode == ppk::K_PUSHGRAD || mode == ppk::K_PP_BWD)) a.flags |= ppk::F_A;
    for (const pp_tensor* t : {src, trg, out, gg, grid})
      if (t && !fits32(max_offset(t, 0)))
        return fail(PP_ERR_UNSUPPORTED, "(): batch entry %d: volume too large for 32-bit offsets", v);
    if (!fits32(a.nvox)) return fail(PP_ERR_UNSUPPORTED, "(): batch entry %d: too many sampling points", v);
    order[v] = iso;
    cbs[v] = static_cast<int>(a.C >= 4 ? 4 : a.C);
    nitems[v] = (a.nvox + kBatchPoints - 1) / kBatchPoints;
    const int CP = scatter && out && use_scratch && !det ? entry_slots(mode, a.C, iso) : 0;
    if (scatter && out && det) {
      // order-independent int64 fixed-point accumulation (scale from
      // max |pushed values| and the point count), finalized into `out`
      if (!use_scratch)
        return fail(PP_ERR_WORKSPACE, "(): batch entry %d: the deterministic mode needs the plan's scratch", v);
      unsigned char* w = static_cast<unsigned char*>(scratch) + scratch_used;
      scratch_used += det_bytes(*out);
      DetJob j;
      j.mx = reinterpret_cast<unsigned int*>(w);
      j.acc = reinterpret_cast<unsigned long long*>(w + 256);
      j.bound = static_cast<double>(a.nvox);
      j.tmax = mode == ppk::K_PP ? *src : *trg;  // what is pushed: pulled src (K_PP) or trgt
      j.out = *out;
      const int64_t V = out->sizes[2] * out->sizes[3] * out->sizes[4];
      a.det_acc = j.acc;
      a.det_max = j.mx;
      a.det_bound = j.bound;
      a.out = nullptr;
      a.out_sN = a.C * V;
      a.out_sC = V;
      a.out_s[0] = out->sizes[3] * out->sizes[4];
      a.out_s[1] = out->sizes[4];
      a.out_s[2] = 1;
      fills.push_back({w, det_bytes(*out)});
      dets.push_back(j);
    } else if (CP) {
      // vector reductions into this entry's interleaved accumulator, stored
      // to `out` after the launches
      const int64_t V = out->sizes[2] * out->sizes[3] * out->sizes[4];
      float* acc = reinterpret_cast<float*>(static_cast<unsigned char*>(scratch) + scratch_used);
      scratch_used += ((static_cast<size_t>(V) * CP * 4 + 255) / 256) * 256;
      if (!fits32(V * CP)) return fail(PP_ERR_UNSUPPORTED, "(): batch entry %d: volume too large", v);
      a.out = acc;
      a.out_sN = V * CP;
      a.out_sC = 1;
      a.out_s[2] = CP;
      a.out_s[1] = out->sizes[4] * CP;
      a.out_s[0] = out->sizes[3] * out->sizes[4] * CP;
      a.flags |= ppk::F_VEC;
      fills.push_back({acc, static_cast<size_t>(V) * CP * 4});
      stores.push_back({acc, static_cast<float*>(out->data), V, static_cast<int32_t>(a.C), CP});
    } else if (scatter && out) {
      fills.push_back({out->data, static_cast<size_t>(numel(out)) * 4});
    }
  }
  // group by (order, channel block)
  std::vector<int> idx(nvol);
  for (int v = 0; v < nvol; ++v) idx[v] = v;
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
    return order[x] != order[y] ? order[x] < order[y] : cbs[x] < cbs[y];
  });
  unsigned char* p = static_cast<unsigned char*>(plan);
  PlanHeader* h = reinterpret_cast<PlanHeader*>(p);
  std::memset(h, 0, sizeof(PlanHeader));
  h->magic = kMagic;
  h->mode = mode;
  h->ctas = ctas;
  h->nvol = nvol;
  h->dtype = dtype;
  ppk::PPArgs* pa = reinterpret_cast<ppk::PPArgs*>(p + sizeof(PlanHeader));
  int64_t* pn = reinterpret_cast<int64_t*>(pa + nvol);
  Fill* pf = reinterpret_cast<Fill*>(pn + nvol);
  int g = -1;
  for (int k = 0; k < nvol; ++k) {
    const int v = idx[k];
    if (g < 0 || h->gorder[g] != order[v] || h->gcb[g] != cbs[v]) {
      ++g;
      h->gorder[g] = order[v];
      h->gcb[g] = cbs[v];
      h->gfirst[g] = k;
    }
    ++h->gcount[g];
    std::memcpy(pa + k, &args[v], sizeof(ppk::PPArgs));
    pn[k] = nitems[v];
  }
  h->ngroups = g + 1;
  // merge adjacent zero-fill ranges (arena-allocated outputs become one fill)
  std::sort(fills.begin(), fills.end(), [](const Fill& x, const Fill& y) { return x.ptr < y.ptr; });
  int nf = 0;
  for (const Fill& f : fills) {
    if (nf > 0 && static_cast<unsigned char*>(pf[nf - 1].ptr) + pf[nf - 1].bytes == f.ptr)
      pf[nf - 1].bytes += f.bytes;
    else
      pf[nf++] = f;
  }
  h->nfill = nf;
  VecStore* ps = reinterpret_cast<VecStore*>(pf + nvol);
  for (size_t i = 0; i < stores.size(); ++i) ps[i] = stores[i];
  h->nstore = static_cast<int32_t>(stores.size());
  DetJob* pd = reinterpret_cast<DetJob*>(ps + nvol);
  for (size_t i = 0; i < dets.size(); ++i) pd[i] = dets[i];
  h->ndet = static_cast<int32_t>(dets.size());
  return PP_OK;
}

int pp_batch_run(const void* plan, void* stream) {
  if (!plan) return fail(PP_ERR_ARG, "(): expected a batch plan");
  const unsigned char* p = static_cast<const unsigned char*>(plan);
  const PlanHeader* h = reinterpret_cast<const PlanHeader*>(p);
  if (h->magic != kMagic) return fail(PP_ERR_ARG, "(): not a batch plan (pp_batch_plan first)");
  const ppk::PPArgs* pa = reinterpret_cast<const ppk::PPArgs*>(p + sizeof(PlanHeader));
  const int64_t* pn = reinterpret_cast<const int64_t*>(pa + h->nvol);
  const Fill* pf = reinterpret_cast<const Fill*>(pn + h->nvol);
  const VecStore* ps = reinterpret_cast<const VecStore*>(pf + h->nvol);
  const DetJob* pd = reinterpret_cast<const DetJob*>(ps + h->nvol);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc;
  for (int f = 0; f < h->nfill; ++f)
    if ((rc = cuda_check(cudaMemsetAsync(pf[f].ptr, 0, pf[f].bytes, st), "batch zero fill"))) return rc;
  // deterministic entries: the scale of each fixed-point accumulator
  for (int d = 0; d < h->ndet; ++d)
    if ((rc = det_absmax_of(&pd[d].tmax, pd[d].mx, st))) return rc;
  static thread_local BatchLaunch L;  // 32 KB: not on the stack
  for (int g = 0; g < h->ngroups; ++g) {
    for (int c0 = 0; c0 < h->gcount[g]; c0 += kMaxEntries) {
      const int n = std::min(kMaxEntries, h->gcount[g] - c0);
      L.n = n;
      L.first[0] = 0;
      for (int e = 0; e < n; ++e) {
        const int k = h->gfirst[g] + c0 + e;
        L.e[e] = pa[k];
        L.first[e + 1] = L.first[e] + pn[k];
      }
      const pb_launcher_t fn = kBatchLaunchers[h->dtype == PP_FLOAT32 ? 0 : 1][h->mode];
      const cudaError_t err = fn ? fn(h->gorder[g], h->gcb[g], L, h->ctas, st) : cudaErrorInvalidValue;
      if ((rc = cuda_check(err, "batched kernel launch"))) return rc;
    }
  }
  // interleaved accumulators -> outputs
  static thread_local StoreLaunch SL;
  for (int s0 = 0; s0 < h->nstore; s0 += kMaxStores) {
    const int n = std::min(kMaxStores, h->nstore - s0);
    SL.n = n;
    SL.first[0] = 0;
    for (int e = 0; e < n; ++e) {
      SL.s[e] = ps[s0 + e];
      SL.first[e + 1] = SL.first[e] + SL.s[e].V;
    }
    const int nb = grid_blocks(SL.first[n]);
    batch_store_kernel<<<nb, 256, 0, st>>>(SL);
    count_launch();
    if ((rc = cuda_check(cudaGetLastError(), "batched interleaved store"))) return rc;
  }
  for (int d = 0; d < h->ndet; ++d)
    if ((rc = det_finalize_to(pd[d].acc, &pd[d].out, pd[d].mx, pd[d].bound, st))) return rc;
  return PP_OK;
}

}  // extern "C"
