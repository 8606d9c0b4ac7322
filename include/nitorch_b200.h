/*
 * nitorch_b200 -- C ABI of the B200 spline push/pull library.
 *
 * Plain pointers, sizes and strides; no framework types.  Every entry point
 * is asynchronous on the given CUDA stream (`void*` = cudaStream_t, NULL =
 * legacy default stream), validates its arguments on the host and returns
 * PP_OK (0) or a negative PP_ERR_* code; pp_last_error() then returns a
 * message (thread-local).  Device faults are reported by the CUDA runtime
 * at the next synchronising call, as for any kernel launch.
 *
 * Tensors are described by pp_tensor (sizes and strides in ELEMENTS, any
 * non-negative strides).  Layouts follow nitorch's native backend:
 *   image / volume : (N, C, X[, Y[, Z]])
 *   grid           : (N, X[, Y[, Z]], D)  voxel coordinates, grid[..., 0] -> X
 *   spatial grad   : (N, C, X[, Y[, Z]], D)
 * The spatial dimensionality D (1, 2 or 3) is taken from the grid.
 * Grids (and grid gradients) are float32 for float32 / bfloat16 / float16
 * images and float64 for float64 images; all arithmetic is float32
 * (float64 for float64 images).
 *
 * Ownership: inputs are borrowed read-only; outputs are caller-allocated
 * and FULLY written by the call (push / count outputs are zero-filled by
 * the library first, as the reference allocates them with zeros).
 *
 * Each entry point replaces the reference function named in its comment
 * (nitorch/_C/src/pushpull.h:10-57, implemented in pushpull.cpp:76-327;
 * prefilter: interpol.coeff, vendored as nitorch/_C/_ts/coeff.py:285-344).
 */
#ifndef NITORCH_B200_H
#define NITORCH_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PP_API __attribute__((visibility("default")))
#else
#define PP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define PP_OK               0
#define PP_ERR_ARG         -1   /* invalid shape / stride / option          */
#define PP_ERR_DTYPE       -2   /* unsupported or mismatched dtype          */
#define PP_ERR_CUDA        -3   /* CUDA launch / runtime error              */
#define PP_ERR_UNSUPPORTED -4   /* valid request the library does not do    */
#define PP_ERR_WORKSPACE   -5   /* workspace missing or too small           */
#define PP_ERR_TIMEOUT     -6   /* a bounded device wait gave up            */

/* Element types. */
#define PP_FLOAT32  0
#define PP_FLOAT64  1
#define PP_BFLOAT16 2
#define PP_FLOAT16  3

/* Bound codes: same values as nitorch's BoundType (nitorch/_C/src/bounds.h). */
#define PP_BOUND_REPLICATE 0
#define PP_BOUND_DCT1      1
#define PP_BOUND_DCT2      2
#define PP_BOUND_DST1      3
#define PP_BOUND_DST2      4
#define PP_BOUND_DFT       5
#define PP_BOUND_ZERO      7

/* pp_options.flags */
#define PP_DETERMINISTIC   1   /* push / count: order-independent exact
                                  accumulation (bit-stable run to run)    */

#define PP_MAX_DIM 8

typedef struct pp_tensor {
  void*   data;
  int32_t dtype;                 /* PP_FLOAT32 ...                          */
  int32_t ndim;
  int64_t sizes[PP_MAX_DIM];
  int64_t strides[PP_MAX_DIM];   /* in elements                             */
} pp_tensor;

typedef struct pp_options {
  int32_t nbound;                /* 1..3 entries, padded with the last one  */
  int32_t bound[3];              /* PP_BOUND_* per axis (X, Y, Z)           */
  int32_t norder;                /* 1..3 entries, padded with the last one  */
  int32_t order[3];              /* B-spline order 0..7 per axis            */
  int32_t extrapolate;           /* bit 0: sample outside the field of view;
                                    bit 1: half-voxel tolerance             */
  int32_t flags;                 /* PP_DETERMINISTIC                        */
  const int32_t* sample_order;   /* optional device array: the order in which
                                    the grid's N*prod(grid spatial) sampling
                                    points are processed (a permutation, e.g.
                                    from pp_sample_order); NULL = natural.
                                    Results do not depend on it beyond
                                    floating-point summation order.        */
  const int32_t* brick_start;    /* optional device array, 3-D grids only:
                                    with sample_order from pp_brick_order,
                                    its brick offsets (N * nbricks + 1
                                    entries).  Lets the cubic scatters
                                    accumulate each brick of the scatter
                                    target in on-chip memory.  NULL = no
                                    brick pass.                           */
  const float* brick_records;    /* optional device array with brick_start:
                                    the records pp_brick_order wrote for
                                    the same float32 grid (4 floats per
                                    sample, in perm order).  The brick
                                    kernels then read each sample's
                                    coordinates and index in one coalesced
                                    16-byte load.  NULL = read perm and the
                                    grid.                                 */
} pp_options;

/* Version of this ABI (major * 100 + minor). */
PP_API int pp_abi_version(void);

/* Message of the last error returned on this thread ("" if none). */
PP_API const char* pp_last_error(void);

/* Number of kernels this library has launched since it was loaded (all
 * threads and devices); for auditing what ran on the GPU. */
PP_API unsigned long long pp_kernel_launches(void);

/* Kernel family, mode, order and channel block of the last push/pull
 * launch made on this host thread, e.g. "pp_brick_kernel mode=5 order=3
 * cb=3" ("" if none); for auditing which code path a call took. */
PP_API const char* pp_last_kernel(void);

/* Workspace (device bytes, 256-byte aligned) that a push-type call with
 * output `out` needs: 0 for float32 / float64 outputs without
 * PP_DETERMINISTIC.  Pass it as `workspace` / `workspace_bytes`. */
PP_API size_t pp_push_workspace_bytes(const pp_tensor* out, int32_t flags);

/* ni::grid_pull (pushpull.h:10-13): out (N,C,*grid) = input sampled at grid. */
PP_API int pp_grid_pull(const pp_tensor* input, const pp_tensor* grid,
                 const pp_tensor* out, const pp_options* opt, void* stream);

/* ni::grid_pull_backward (pushpull.h:15-18).  grad_input (N,C,*in) and/or
 * grad_grid (N,*grid,D) may be NULL when not requested. */
PP_API int pp_grid_pull_backward(const pp_tensor* grad, const pp_tensor* input,
                          const pp_tensor* grid, const pp_tensor* grad_input,
                          const pp_tensor* grad_grid, const pp_options* opt,
                          void* stream, void* workspace, size_t workspace_bytes);

/* ni::grid_push (pushpull.h:20-23): out (N,C,*shape) = adjoint of pull. */
PP_API int pp_grid_push(const pp_tensor* input, const pp_tensor* grid,
                 const pp_tensor* out, const pp_options* opt, void* stream,
                 void* workspace, size_t workspace_bytes);

/* ni::grid_push_backward (pushpull.h:25-28). */
PP_API int pp_grid_push_backward(const pp_tensor* grad, const pp_tensor* input,
                          const pp_tensor* grid, const pp_tensor* grad_input,
                          const pp_tensor* grad_grid, const pp_options* opt,
                          void* stream);

/* ni::grid_count (pushpull.h:30-33): out (N,1,*shape), grid dtype. */
PP_API int pp_grid_count(const pp_tensor* grid, const pp_tensor* out,
                  const pp_options* opt, void* stream, void* workspace,
                  size_t workspace_bytes);

/* ni::grid_count_backward (pushpull.h:35-38): grad (N,1,*shape). */
PP_API int pp_grid_count_backward(const pp_tensor* grad, const pp_tensor* grid,
                           const pp_tensor* grad_grid, const pp_options* opt,
                           void* stream);

/* ni::grid_grad (pushpull.h:40-43): out (N,C,*grid,D). */
PP_API int pp_grid_grad(const pp_tensor* input, const pp_tensor* grid,
                 const pp_tensor* out, const pp_options* opt, void* stream);

/* Fused forward of pull and grid_grad: out (N, C, *grid) = pull(input, grid)
 * and out_grad (N, C, *grid, D) = grid_grad(input, grid) from one pass over
 * each point's taps (the two values ni::grid_pull and ni::grid_grad,
 * nitorch/_C/src/pushpull.h:10-13 and 40-43, compute separately).  Same
 * arguments and checks as pp_grid_grad, plus `out`. */
PP_API int pp_grid_pull_grad(const pp_tensor* input, const pp_tensor* grid, const pp_tensor* out,
                             const pp_tensor* out_grad, const pp_options* opt, void* stream);

/* ni::grid_grad_backward (pushpull.h:45-48): grad (N,C,*grid,D). */
PP_API int pp_grid_grad_backward(const pp_tensor* grad, const pp_tensor* input,
                          const pp_tensor* grid, const pp_tensor* grad_input,
                          const pp_tensor* grad_grid, const pp_options* opt,
                          void* stream, void* workspace, size_t workspace_bytes);

/* Fused normal operator push(pull(input, grid), grid) in one pass (no
 * counterpart in the reference, which calls ni::grid_pull then
 * ni::grid_push on the same grid): out (input's sizes, any strides) =
 * P^T P input, with the pulled values rounded to the storage type as a
 * separate pull would store them.  Workspace as for pp_grid_push
 * (pp_push_workspace_bytes of `out`). */
PP_API int pp_grid_pull_push(const pp_tensor* input, const pp_tensor* grid, const pp_tensor* out,
                             const pp_options* opt, void* stream, void* workspace,
                             size_t workspace_bytes);

/* Backward of pp_grid_pull_push for the loss gradient `grad` (input's sizes
 * AND strides): grad_input = P^T P grad (the operator is self-adjoint) and
 * the grid gradient (grid's sizes); either may be NULL.  One pass (the
 * reference runs ni::grid_push_backward then ni::grid_pull_backward). */
PP_API int pp_grid_pull_push_backward(const pp_tensor* grad, const pp_tensor* input,
                                      const pp_tensor* grid, const pp_tensor* grad_input,
                                      const pp_tensor* grad_grid, const pp_options* opt,
                                      void* stream, void* workspace, size_t workspace_bytes);

/* Displacement self-composition u <- u + pull(u, id + u), the step of the
 * scaling-and-squaring exponentiation of a stationary velocity field
 * (nitorch/spatial/_svf.py:85-94 with _pull_vel :323-362, which materialise
 * id + u and call ni::grid_pull).  disp and out: (N, *spatial, D) float32 or
 * float64 fields, displacement components last, any strides; out must not
 * alias disp.  The options' bound / order / extrapolate apply to the pull
 * (nitorch's defaults there: dft, linear, extrapolate). */
PP_API int pp_svf_compose(const pp_tensor* disp, const pp_tensor* out, const pp_options* opt,
                          void* stream);

/* Gradient of <grad, u + pull(u, id + u)> with respect to u (the exact
 * adjoint of pp_svf_compose), written to grad_disp (disp's sizes, every
 * element overwritten, must not alias the inputs).  Workspace: 16-byte
 * aligned, pp_svf_workspace_bytes(disp, opt->flags) bytes.
 *  - PP_DETERMINISTIC (float32 / float64 fields, workspace required): the
 *    push of the gradient accumulates in int64 fixed point (scaled from
 *    max |grad| and the voxel count) and each voxel's identity and
 *    grid-gradient terms are stored by its own point, so the result is
 *    bit-identical from run to run.
 *  - otherwise, for 3-D float32 fields at orders 1 and 3, the push goes to a
 *    four-slot channel-interleaved accumulator with one vector reduction
 *    per tap and is copied to grad_disp afterwards; with NULL / too small a
 *    workspace (or other fields), one reduction per component and tap
 *    straight into grad_disp.  grad_disp may be the first three slots of
 *    the workspace itself (data = workspace, strides (V*4, Y*Z*4, Z*4, 4,
 *    1)): the result is then left there, with no copy. */
PP_API size_t pp_svf_workspace_bytes(const pp_tensor* disp, int32_t flags);
PP_API int pp_svf_compose_backward(const pp_tensor* grad, const pp_tensor* disp,
                                   const pp_tensor* grad_disp, const pp_options* opt, void* stream,
                                   void* workspace, size_t workspace_bytes);

/* ---- Affine sampling without a materialised grid ----------------------
 * nitorch builds affine_grid(mat, shape) (nitorch/spatial/_grid.py:579-615)
 * and calls ni::grid_pull on it (resize :618-754, reslice :860-914); these
 * entry points compute the coordinate A [sub; 1] of every grid point in the
 * kernel instead (12 bytes per point less traffic, no grid allocation).
 * mat: (N, D, D+1) or (N, D+1, D+1) matrices of the grid dtype (float32 for
 * 16-bit images), rows of D+1 contiguous entries; the first D rows are used. */

/* out (N, C, *shape) = input (N, C, *inshape) sampled at A [sub; 1]. */
PP_API int pp_affine_pull(const pp_tensor* input, const pp_tensor* mat, const pp_tensor* out,
                          const pp_options* opt, void* stream);

/* Adjoint of pp_affine_pull: out (N, C, *outshape) = push of input
 * (N, C, *shape).  Workspace as for pp_grid_push (pp_push_workspace_bytes(out)). */
PP_API int pp_affine_push(const pp_tensor* input, const pp_tensor* mat, const pp_tensor* out,
                          const pp_options* opt, void* stream, void* workspace, size_t workspace_bytes);

/* Gradient of <grad, pp_affine_pull(input, mat)> with respect to the first
 * D rows of the matrices, into grad_mat (N, D, D+1) float32 with contiguous
 * rows (the input gradient is pp_affine_push of grad).  Needs
 * pp_affine_grad_workspace_bytes(grad) bytes of workspace; images of
 * float32 / 16-bit storage. */
PP_API size_t pp_affine_grad_workspace_bytes(const pp_tensor* grad);
PP_API int pp_affine_grad_matrix(const pp_tensor* grad, const pp_tensor* input, const pp_tensor* mat,
                                 const pp_tensor* grad_mat, const pp_options* opt, void* stream,
                                 void* workspace, size_t workspace_bytes);

/* Resize: out (N, C, *shape) = input (N, C, *inshape) sampled at
 * x_d = scale[d] * o_d + shift[d] for every output voxel o (3-D, float32 or
 * bfloat16, one B-spline order <= 3 for all axes, positive scales): the
 * diagonal affine sampling of nitorch's resize (nitorch/spatial/_grid.py:
 * 618-754, affine_grid then ni::grid_pull) and of its native ni::resize
 * (nitorch/_C/src/resize.h, resize_common.cpp:600-700, which extrapolates:
 * set bit 0 of opt->extrapolate).  Computed separably (three 4-tap passes
 * over TMA-staged tiles); equal to pp_affine_pull with the diagonal matrix.
 * Other cases return PP_ERR_UNSUPPORTED (use pp_affine_pull). */
PP_API int pp_resize(const pp_tensor* input, const pp_tensor* out, const double* scale, const double* shift,
                     const pp_options* opt, void* stream);

/* Device status of the resize kernels (bit 0: a bounded wait for a TMA copy
 * gave up; 0 in normal operation).  Synchronous. */
PP_API int pp_resize_status(uint32_t* status);

/* Multigrid prolongation / restriction between the grids of `input`
 * (N, C, *inshape) and `out` (N, C, *shape) of nitorch's native
 * fmg_prolongation / fmg_restriction (nitorch/_C/src/multires.h:10-19,
 * impl/multires_common.cpp:419-500 and 587-660): with scale = inshape /
 * shape per axis, output voxel o reads the input at x = (o + 1/2) scale -
 * 1/2; prolongation weights the three nodes around x by the quadratic
 * B-spline, restriction the four nodes from floor(x) - 1 by the linear
 * B-spline of width `scale` (divided by `scale`).  No field-of-view test;
 * opt->bound per axis (opt->order and opt->extrapolate are not read).
 * 3-D float32 or bfloat16; the same separable kernel as pp_resize. */
PP_API int pp_fmg_prolongation(const pp_tensor* input, const pp_tensor* out, const pp_options* opt, void* stream);
PP_API int pp_fmg_restriction(const pp_tensor* input, const pp_tensor* out, const pp_options* opt, void* stream);

/* ---- Regularisers: out = (H + L) x ------------------------------------
 * nitorch._C.solve.c_regulariser / c_regulariser_grid (nitorch/_C/solve.py:
 * 21-142; native nitorch/_C/src/regulariser.cpp:19-64, regulariser_grid.cpp;
 * kernels nitorch/_C/src/impl/regulariser_common.cpp,
 * regulariser_grid_common.cpp).  L is the matrix of the absolute, membrane
 * and bending energies (and, for displacement grids, the Lame shear and
 * divergence energies) with the boundary conditions `bound` per axis and
 * voxel sizes `voxel_size` per axis (three entries each, unfolded by the
 * caller: the last given entry repeated); H a voxel-wise Hessian.  float32
 * or float64; weights, Hessian and output have the input's dtype; the
 * output must not overlap the inputs.  A weight map scales the absolute and
 * membrane energies (PP_ERR_UNSUPPORTED with bending or Lame terms). */
/* Field: input / out (N, C, *spatial), 1-3-D, C <= 64; absolute / membrane /
 * bending: C entries each (already times the caller's factor); weight
 * (N, C, *spatial) or NULL (broadcast by strides); hessian (N, CC, *spatial),
 * CC in {1, C, 2C-1, C(C+1)/2} (identity, diagonal, the (diag, last row)
 * layout of regulariser_common.cpp:630-648, or the symmetric diagonal-then-
 * upper-triangle layout), or NULL. */
PP_API int pp_regulariser(const pp_tensor* input, const pp_tensor* weight, const pp_tensor* hessian,
                          const pp_tensor* out, const double* absolute, const double* membrane,
                          const double* bending, const double* voxel_size, const int32_t* bound, void* stream);
/* Grid: input / out (N, *spatial, D) displacements, components last, D = the
 * spatial dimension; component d is scaled by voxel_size[d]^2 as in the
 * reference; weight (N, *spatial) or NULL; hessian (N, *spatial, DD), DD in
 * {1, D, D(D+1)/2}, or NULL. */
PP_API int pp_regulariser_grid(const pp_tensor* input, const pp_tensor* weight, const pp_tensor* hessian,
                               const pp_tensor* out, double absolute, double membrane, double bending,
                               double shear, double div, const double* voxel_size, const int32_t* bound,
                               void* stream);

/* ---- Jacobians of transformation / displacement fields ----------------
 * nitorch.spatial.grid_jacobian / grid_jacdet (nitorch/spatial/_grid.py:
 * 917-1013) without `sample`: central finite differences of the
 * displacement (nitorch/spatial/_finite_differences.py:32-222, order 1,
 * side 'c'; the bound code gives the values beyond each end; a singleton
 * axis yields the values themselves, as there), plus the identity.
 * field: (N, *spatial, D) float32 / float64, components last (a
 * transformation if is_grid, else a displacement); jac: (N, *spatial, D, D)
 * with jac[..., i, j] = d psi_i / d x_j, and / or det: (N, *spatial); either
 * may be NULL.  voxel_size: D doubles (NULL: 1). */
PP_API int pp_grid_jacobian(const pp_tensor* field, const pp_tensor* jac, const pp_tensor* det, int32_t bound,
                            const double* voxel_size, int32_t is_grid, int32_t add_identity, void* stream);

/* Adjoint of pp_grid_jacobian: grad_field (field's shape, zero-filled by
 * the call) = gradient of <grad_jac, jac> + <grad_det, det> w.r.t. the field;
 * grad_jac or grad_det may be NULL. */
PP_API int pp_grid_jacobian_backward(const pp_tensor* grad_jac, const pp_tensor* grad_det,
                                     const pp_tensor* field, const pp_tensor* grad_field, int32_t bound,
                                     const double* voxel_size, int32_t is_grid, int32_t add_identity,
                                     void* stream);

/* Determinants of (M, D, D) matrices (torch.det in nitorch's grid_jacdet
 * with `sample`): det (M) forward, or grad_jac = grad_det * cofactor(jac)
 * backward (det = NULL). */
PP_API int pp_jacobian_det(const pp_tensor* jac, const pp_tensor* det, const pp_tensor* grad_det,
                           const pp_tensor* grad_jac, void* stream);

/* Source-sorted processing order of a grid's sampling points (no
 * counterpart in the reference; a scheduling aid for rough deformations):
 * writes to `perm` (int32, N*prod(grid spatial) entries) the sample indices
 * sorted by the source voxel floor(coordinate) they fall in, for a source
 * of spatial size `src_size` (D entries).  Needs
 * pp_sample_order_workspace_bytes() bytes of device workspace. */
PP_API size_t pp_sample_order_workspace_bytes(const pp_tensor* grid, const int64_t* src_size);
PP_API int pp_sample_order(const pp_tensor* grid, const int64_t* src_size, int32_t* perm,
                           void* workspace, size_t workspace_bytes, void* stream);

/* Brick-major processing order (no counterpart in the reference; a
 * scheduling aid for the cubic 3-D brick kernels).  The source volume (spatial
 * size `src_size`, 3 entries) is cut into bricks of PP_BRICK_X x PP_BRICK_Y
 * x PP_BRICK_Z voxels, nb = prod(ceil(src_size / brick)) per batch item.
 * Writes to `perm` (int32, N*prod(grid spatial) entries) the sample
 * indices sorted by (batch item, brick, voxel in brick) of the source voxel
 * floor(coordinate) they fall in (clamped into the volume), and to
 * `brick_start` (int32, N*nb + 1 entries) where each brick's samples start
 * in `perm` (the last entry is the number of samples).  Optional
 * `records` (float32 grids only; 4 * N*prod(grid spatial) floats, 16-byte
 * aligned, or NULL) receives, in perm order, each sample's coordinates and
 * its index (x, y, z, index as int32 bits).  Pass all three in pp_options.
 * 3-D grids only; needs pp_brick_order_workspace_bytes() bytes of device
 * workspace.  pp_brick_count() gives N*nb. */
#define PP_BRICK_X 4
#define PP_BRICK_Y 4
#define PP_BRICK_Z 6
PP_API int64_t pp_brick_count(const pp_tensor* grid, const int64_t* src_size);
PP_API size_t pp_brick_order_workspace_bytes(const pp_tensor* grid, const int64_t* src_size);
PP_API int pp_brick_order(const pp_tensor* grid, const int64_t* src_size, int32_t* perm,
                          int32_t* brick_start, float* records, void* workspace, size_t workspace_bytes,
                          void* stream);

/* pp_sample_order without any device allocation or caller workspace (no
 * counterpart in the reference).  For callers that cannot allocate device
 * memory when they need an order -- a host runtime that owns all device
 * memory up front, or one that works under a fixed budget.  Uses a fixed 16 MiB
 * scratch array compiled into the library (held on every device that loads
 * it): 4 bytes per source voxel (times the batch) plus 8 bytes per sampling
 * point must fit, else PP_ERR_WORKSPACE.  The first call on a device looks
 * up the scratch address for that device; make that first call before any
 * stream capture.  Only the device's primary context is supported, and no
 * cudaDeviceReset may follow the first call on that device.  All calls
 * share the scratch: calls that overlap on the GPU race and must be
 * serialised by the caller. */
PP_API int pp_sample_order_noalloc(const pp_tensor* grid, const int64_t* src_size, int32_t* perm,
                                   void* stream);

/* ---- Batched launches (no counterpart in the reference, which takes one
 * tensor per call: nitorch/_C/src/pushpull.cpp:76-327) --------------------
 * Many independent 3-D volumes (uneven shapes, one isotropic order 0-3 per
 * volume, float32 or bfloat16 images shared by all entries, float32 grids)
 * run one mode in a few launches: one per group of volumes with the same
 * (order, channel block), each carrying up to 80 volumes' arguments.
 * Tensors per mode (images (1, C, X, Y, Z), grids (1, X, Y, Z, 3); "grid
 * shaped" = the grid's spatial shape; scatter outputs contiguous float32,
 * zero-filled by pp_batch_run):
 *   PP_BATCH_PULL          src -> out (grid shaped, image dtype)
 *   PP_BATCH_PUSH          trgt (grid shaped) -> out (scatter, shape of out)
 *   PP_BATCH_PUSH_BACKWARD src = d loss/d push output, trgt = pushed values
 *                          -> out = d loss/d values (grid shaped, optional),
 *                             gg = d loss/d grid (optional)
 *   PP_BATCH_PULL_BACKWARD src = pulled image, trgt = d loss/d pulled
 *                          -> out = d loss/d image (scatter, optional), gg
 *   PP_BATCH_PULL_PUSH     src -> out = push(pull(src)) (scatter, src shaped)
 *   PP_BATCH_PULL_PUSH_BACKWARD src, trgt = d loss/d out laid out like src
 *                          -> out = d loss/d src (scatter, optional), gg
 * opt.sample_order (optional) is read when the plan runs.  An entry with
 * PP_DETERMINISTIC in opt.flags scatters into an int64 fixed-point
 * accumulator in the scratch (pp_batch_scratch_bytes counts it; the plan
 * fails with PP_ERR_WORKSPACE without it), scaled from max |pushed values|
 * taken when the plan runs, and is finalized into `out`: bit-identical
 * results from run to run. */
#define PP_BATCH_PULL 0
#define PP_BATCH_PUSH 2
#define PP_BATCH_PUSH_BACKWARD 4
#define PP_BATCH_PULL_BACKWARD 5
#define PP_BATCH_PULL_PUSH 7
#define PP_BATCH_PULL_PUSH_BACKWARD 8

typedef struct pp_batch_entry {
  pp_tensor src, trgt, grid, out, gg; /* unused: data = NULL */
  pp_options opt;
} pp_batch_entry;

/* Host bytes of a plan for `nvol` volumes. */
PP_API size_t pp_batch_plan_bytes(int32_t nvol);
/* Device scratch (bytes) that lets the scatter entries of 2-4 channels at
 * orders 2-3 accumulate with vector reductions, plus the fixed-point
 * accumulators of deterministic scatter entries (0 if no entry needs any). */
PP_API size_t pp_batch_scratch_bytes(const pp_batch_entry* entries, int32_t nvol, int32_t mode);
/* Validates the entries and writes a plan into `plan` (host memory of
 * pp_batch_plan_bytes(nvol) bytes, owned by the caller).  ctas = 0: one CTA
 * per 256 sampling points; ctas > 0: that many persistent CTAs.  `scratch`
 * (device, 256-byte aligned, pp_batch_scratch_bytes bytes) is optional:
 * without it every entry scatters with scalar reductions.  The tensors and
 * the scratch must stay alive and in place while the plan is used. */
PP_API int pp_batch_plan(const pp_batch_entry* entries, int32_t nvol, int32_t mode, int32_t ctas,
                         void* plan, size_t plan_bytes, void* scratch, size_t scratch_bytes);
/* Enqueues the plan's zero fills and launches on `stream`. */
PP_API int pp_batch_run(const void* plan, void* stream);

/* interpol.coeff.spline_coeff (vendored: _ts/coeff.py:285-310):
 * interpolating B-spline coefficients along one axis of `input`, written to
 * `out` (same sizes; may alias `input` for in-place).  `bound` uses the
 * prefilter's integer codes (_ts/bounds.py:7-14): 0 zero, 1 replicate,
 * 2 dct1, 3 dct2, 6 dft; other codes return PP_ERR_UNSUPPORTED, as the
 * reference raises NotImplementedError. */
PP_API int pp_spline_coeff(const pp_tensor* input, const pp_tensor* out,
                    int32_t bound, int32_t order, int32_t axis, void* stream);

/* interpol.coeff.spline_coeff_nd (_ts/coeff.py:314-344): the last `dim`
 * axes, per-axis bound / order lists padded with their last entry. */
PP_API int pp_spline_coeff_nd(const pp_tensor* input, const pp_tensor* out,
                       int32_t nbound, const int32_t* bound, int32_t norder,
                       const int32_t* order, int32_t dim, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NITORCH_B200_H */
