// One (image type, mode) slice of the batched kernels.  Compiled several
// times by the Makefile with -DPB_STYPE=<float|__nv_bfloat16>
// -DPB_SNAME=<f32|bf16> -DPB_MODE=<0|2|4|5|7|8>; exports
// pp_batch_launch_<sname>_m<mode>(ord, cb, launch, ctas, stream).
#include "batch_kernel.cuh"

#define PB_CAT2(a, b) a##b
#define PB_CAT(a, b) PB_CAT2(a, b)
#define PB_NAME PB_CAT(PB_CAT(PB_CAT(pp_batch_launch_, PB_SNAME), _m), PB_MODE)

cudaError_t PB_NAME(int ord, int cb, const ppb::BatchLaunch& L, int ctas, cudaStream_t st) {
  return ppb::launch_group<PB_STYPE, PB_MODE>(ord, cb, L, ctas, st);
}
