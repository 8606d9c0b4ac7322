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

struct PlanHeader {
  uint32_t magic;
  int32_t mode, ctas, nvol, dtype, ngroups, nfill, pad;
  int32_t gfirst[kMaxGroups], gcount[kMaxGroups], gorder[kMaxGroups], gcb[kMaxGroups];
};

struct Fill {  // a byte range to zero before the launches
  void* ptr;
  size_t bytes;
};

// Layout of the host plan buffer: header, then per volume its PPArgs and its
// item count (sorted by group), then the fill ranges.
inline size_t plan_bytes(int nvol) {
  return sizeof(PlanHeader) + static_cast<size_t>(nvol) * (sizeof(ppk::PPArgs) + sizeof(int64_t) + sizeof(Fill));
}

bool is_scatter(int mode) {
  return mode == ppk::K_PUSH || mode == ppk::K_PUSHGRAD || mode == ppk::K_PP || mode == ppk::K_PP_BWD;
}

}  // namespace ppb

using namespace ppc;
using namespace ppb;

extern "C" {

size_t pp_batch_plan_bytes(int32_t nvol) { return nvol > 0 ? plan_bytes(nvol) : 0; }

int pp_batch_plan(const pp_batch_entry* items, int32_t nvol, int32_t mode, int32_t ctas, void* plan,
                  size_t plan_bytes_) {
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
    if (it.opt.flags & PP_DETERMINISTIC)
      return fail(PP_ERR_UNSUPPORTED, "(): batch entry %d: batched launches have no deterministic mode", v);
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
    if (scatter && out) fills.push_back({out->data, static_cast<size_t>(numel(out)) * 4});
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
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc;
  for (int f = 0; f < h->nfill; ++f)
    if ((rc = cuda_check(cudaMemsetAsync(pf[f].ptr, 0, pf[f].bytes, st), "batch zero fill"))) return rc;
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
  return PP_OK;
}

}  // extern "C"
