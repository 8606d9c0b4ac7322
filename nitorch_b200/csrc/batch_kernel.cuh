// Kernel side of the batched launches (see batch.cu): the launch argument
// carrying up to kMaxEntries volumes by value and the kernel over them.
#pragma once
#include "pp_capi_internal.cuh"
#include "pp_kernels.cuh"

namespace ppb {

constexpr int kBatchPoints = 256;  // sampling points per work item (= threads per CTA)
constexpr int kMaxEntries = 72;    // volumes per launch: keeps BatchLaunch under 32 KB

struct BatchLaunch {
  int32_t n;                       // volumes in this launch
  int32_t pad;
  int64_t first[kMaxEntries + 1];  // item prefix sums: items of volume e are [first[e], first[e+1])
  ppk::PPArgs e[kMaxEntries];
};
static_assert(sizeof(BatchLaunch) <= 32764, "batched kernel argument above the kernel-parameter limit");

// A CTA per work item (or, with gridDim.x below the item count, persistent
// CTAs striding over the items); the item's volume is found by binary
// search over the prefix sums, and its arguments are read in place from the
// kernel parameter (constant bank), never copied.
template <class S, int MODE, int ORD, int CB>
__global__ void __launch_bounds__(kBatchPoints, ppk::MinBlocks<MODE>::value)
    pp_batch_kernel(const __grid_constant__ BatchLaunch L) {
  const int64_t total = L.first[L.n];
  for (int64_t item = blockIdx.x; item < total; item += gridDim.x) {
    int lo = 0, hi = L.n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (L.first[mid] <= item) lo = mid; else hi = mid - 1;
    }
    const ppk::PPArgs& a = L.e[lo];
    const int64_t t = (item - L.first[lo]) * kBatchPoints + threadIdx.x;
    if (t < a.nvox) {
      int32_t v = a.perm != nullptr ? __ldg(a.perm + t) : static_cast<int32_t>(t);
      int32_t sub[3];
      const int32_t nz = static_cast<int32_t>(a.trgt_size[2]), ny = static_cast<int32_t>(a.trgt_size[1]);
      sub[2] = v % nz; v /= nz;
      sub[1] = v % ny;
      sub[0] = v / ny;
      ppk::pp_point<3, ORD, CB, S, MODE, int32_t>(a, sub, 0);
    }
  }
}

template <class S, int MODE, int ORD, int CB>
cudaError_t launch_chunk(const BatchLaunch& L, int ctas, cudaStream_t st) {
  const int64_t total = L.first[L.n];
  if (total == 0) return cudaSuccess;
  const int64_t blocks = ctas > 0 ? (ctas < total ? ctas : total) : total;
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  pp_batch_kernel<S, MODE, ORD, CB><<<static_cast<unsigned>(blocks), kBatchPoints, 0, st>>>(L);
  ppc::count_launch();
  return cudaGetLastError();
}

template <class S, int MODE, int ORD>
cudaError_t launch_cb(int cb, const BatchLaunch& L, int ctas, cudaStream_t st) {
  switch (cb) {
    case 1: return launch_chunk<S, MODE, ORD, 1>(L, ctas, st);
    case 2: return launch_chunk<S, MODE, ORD, 2>(L, ctas, st);
    case 3: return launch_chunk<S, MODE, ORD, 3>(L, ctas, st);
    default: return launch_chunk<S, MODE, ORD, 4>(L, ctas, st);
  }
}

template <class S, int MODE>
cudaError_t launch_group(int ord, int cb, const BatchLaunch& L, int ctas, cudaStream_t st) {
  switch (ord) {
    case 0: return launch_cb<S, MODE, 0>(cb, L, ctas, st);
    case 1: return launch_cb<S, MODE, 1>(cb, L, ctas, st);
    case 2: return launch_cb<S, MODE, 2>(cb, L, ctas, st);
    default: return launch_cb<S, MODE, 3>(cb, L, ctas, st);
  }
}

}  // namespace ppb

// One launcher per (image type, mode), compiled in its own translation unit
// (batch_inst.cu).
using pb_launcher_t = cudaError_t (*)(int ord, int cb, const ppb::BatchLaunch& L, int ctas, cudaStream_t st);
