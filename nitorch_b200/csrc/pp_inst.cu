// One (storage type, dimension, mode) slice of the push/pull kernel family.
// Compiled several times by the Makefile with
//   -DPP_STYPE=<float|double|__nv_bfloat16|__half> -DPP_SNAME=<f32|...>
//   -DPP_DIM=<1|2|3> -DPP_MODE=<0..8>
// and exports  pp_launch_<sname>_d<dim>_m<mode>(ord, wide, args, stream).
#include "pp_kernels.cuh"

#define PP_CAT2(a, b) a##b
#define PP_CAT(a, b) PP_CAT2(a, b)
#define PP_NAME PP_CAT(PP_CAT(PP_CAT(PP_CAT(PP_CAT(pp_launch_, PP_SNAME), _d), PP_DIM), _m), PP_MODE)

cudaError_t PP_NAME(int ord, bool wide, const ppk::PPArgs& a, cudaStream_t st) {
  return ppk::launch_ord<PP_DIM, PP_STYPE, PP_MODE>(ord, wide, a, st);
}
