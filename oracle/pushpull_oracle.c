/*
 * CPU oracle for the spline push/pull path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is a plain-C restatement of nitorch's compiled push/pull
 * algorithm and of its spline prefilter.  It is the checker for the CUDA
 * product: only the tests, the package's smoke check and the CPU-baseline
 * leg of the benchmark load it.  The product never calls it.
 *
 * It is compiled twice (see oracle/Makefile):
 *   REAL=double -> liboracle_f64.so   (the FP64 oracle)
 *   REAL=float  -> liboracle_f32.so   (same arithmetic type as the
 *                                      reference's float instantiation,
 *                                      used for the bit-exact checks of
 *                                      order 0 and of the index maps)
 *
 * Parity is pinned against the reference's own compiled CPU backend
 * (oracle/build_ref.py) by tests/test_oracle_vs_reference.py and by the
 * golden fixtures under tests/golden/.
 *
 * Reference files followed (paths inside the nitorch project):
 *   nitorch/_C/src/impl/bounds_common.h         (index / sign maps)
 *   nitorch/_C/src/impl/interpolation_common.h  (B-spline weights)
 *   nitorch/_C/src/impl/pushpull_common.cpp     (tap loops, modes)
 *   nitorch/_C/_ts/coeff.py                     (prefilter)
 *
 * Known reference defects are corrected by default.  The `quirks` bitmask
 * re-enables them so that the oracle can be compared with the reference:
 *   OR_QUIRK_D1: the third axis uses the second axis' order
 *                (pushpull_common.cpp:591).
 *   OR_QUIRK_D3: second derivatives of orders 5-7 are zero
 *                (interpolation_common.h:1154-1156,1170-1172).
 * (Defect D2 -- uninitialised second derivatives when the target's last
 * stride is 1, pushpull_common.cpp:1137 -- reads indeterminate stack
 * values and is not reproducible; the oracle always computes them.)
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>
#include <string.h>

#ifndef REAL
#define REAL double
#endif

#define OR_QUIRK_D1 1
#define OR_QUIRK_D3 4

/* Bound codes of the compiled backend (nitorch/_C/src/bounds.h:5-15). */
enum { B_REPLICATE = 0, B_DCT1 = 1, B_DCT2 = 2, B_DST1 = 3, B_DST2 = 4,
       B_DFT = 5, B_SLIDING = 6, B_ZERO = 7, B_NOCHECK = 8 };

/* ------------------------------------------------------------------ */
/* Index maps: bounds_common.h:26-90                                   */
/* ------------------------------------------------------------------ */

static int64_t idx_reflect1c(int64_t i, int64_t n) {   /* bounds_common.h:36-43 */
  if (n == 1) return 0;
  int64_t p = (n - 1) * 2;
  i = i < 0 ? -i : i;
  i = i % p;
  return i >= n ? p - i : i;
}

static int64_t idx_reflect1s(int64_t i, int64_t n) {   /* bounds_common.h:52-59 */
  if (n == 1) return 0;
  int64_t p = (n + 1) * 2;
  i = i == -1 ? 0 : i < 0 ? -i - 2 : i;
  i = i % p;
  return i == n ? n - 1 : i > n ? p - i - 2 : i;
}

static int64_t idx_reflect2(int64_t i, int64_t n) {    /* bounds_common.h:66-71 */
  int64_t p = n * 2;
  i = i < 0 ? p - ((-i - 1) % p) - 1 : i % p;
  return i >= n ? p - i - 1 : i;
}

static int64_t idx_circular(int64_t i, int64_t n) {    /* bounds_common.h:78-81 */
  return i < 0 ? (n + i % n) % n : i % n;
}

static int64_t idx_replicate(int64_t i, int64_t n) {   /* bounds_common.h:88-91 */
  return i <= 0 ? 0 : i >= n ? n - 1 : i;
}

int64_t or_bound_index(int bound, int64_t i, int64_t n) { /* bounds_common.h:193-205 */
  switch (bound) {
    case B_REPLICATE: return idx_replicate(i, n);
    case B_DCT1:      return idx_reflect1c(i, n);
    case B_DCT2:      return idx_reflect2(i, n);
    case B_DST1:      return idx_reflect1s(i, n);
    case B_DST2:      return idx_reflect2(i, n);
    case B_DFT:       return idx_circular(i, n);
    default:          return i;
  }
}

/* Sign maps: bounds_common.h:101-133, 207-219 */
int or_bound_sign(int bound, int64_t i, int64_t n) {
  switch (bound) {
    case B_REPLICATE: case B_DCT1: case B_DCT2: case B_DFT:
      return 1;
    case B_DST1: {                                      /* periodic1 */
      if (n == 1) return 1;
      int64_t p = (n + 1) * 2;
      i = i < 0 ? n - i - 1 : i;
      i = i % p;
      if (i % (n + 1) == n) return 0;
      return ((i / (n + 1)) % 2) ? -1 : 1;
    }
    case B_DST2:                                        /* periodic2 */
      i = i < 0 ? n - i - 1 : i;
      return ((i / n) % 2) ? -1 : 1;
    default:                                            /* zero: inbounds */
      return (i < 0 || i >= n) ? 0 : 1;
  }
}

/* ------------------------------------------------------------------ */
/* B-spline weights, first and second derivatives                      */
/* interpolation_common.h:57-815 ("fast" variants: x inside support)   */
/* The piecewise polynomials are the standard centred B-splines; they  */
/* are evaluated here in REAL arithmetic, in Horner form.              */
/* ------------------------------------------------------------------ */

static REAL w_eval(int order, REAL x) {
  x = fabs(x);
  switch (order) {
    case 0: return 1;
    case 1: return 1 - x;
    case 2:
      if (x < 0.5) return 0.75 - x * x;
      x = 1.5 - x; return 0.5 * x * x;
    case 3:
      if (x < 1) return (x * x * (x - 2) * 3 + 4) / 6;
      x = 2 - x; return x * x * x / 6;
    case 4:
      if (x < 0.5) { x *= x; return x * (x * 0.25 - 0.625) + 115. / 192.; }
      if (x < 1.5) return x * (x * (x * (5. - x) / 6. - 1.25) + 5. / 24.) + 55. / 96.;
      x -= 2.5; x *= x; return x * x / 24.;
    case 5:
      if (x < 1) { REAL f = x * x; return f * (f * (0.25 - x * (1. / 12.)) - 0.5) + 0.55; }
      if (x < 2) return x * (x * (x * (x * (x * (1. / 24.) - 0.375) + 1.25) - 1.75) + 0.625) + 0.425;
      { REAL f = 3 - x; x = f * f; return f * x * x * (1. / 120.); }
    case 6:
      if (x < 0.5) { x *= x;
        return x * (x * (7. / 48. - x * (1. / 36.)) - 77. / 192.) + 5887. / 11520.; }
      if (x < 1.5)
        return x * (x * (x * (x * (x * (x * (1. / 48.) - 7. / 48.) + 0.328125)
               - 35. / 288.) - 91. / 256.) - 7. / 768.) + 7861. / 15360.;
      if (x < 2.5)
        return x * (x * (x * (x * (x * (7. / 60. - x * (1. / 120.)) - 0.65625)
               + 133. / 72.) - 2.5703125) + 1267. / 960.) + 1379. / 7680.;
      x -= 3.5; x *= x * x; return x * x * (1. / 720.);
    case 7:
      if (x < 1) { REAL f = x * x;
        return f * (f * (f * (x * (1. / 144.) - 1. / 36.) + 1. / 9.) - 1. / 3.) + 151. / 315.; }
      if (x < 2)
        return x * (x * (x * (x * (x * (x * (0.05 - x * (1. / 240.)) - 7. / 30.)
               + 0.5) - 7. / 18.) - 0.1) - 7. / 90.) + 103. / 210.;
      if (x < 3)
        return x * (x * (x * (x * (x * (x * (x * (1. / 720.) - 1. / 36.) + 7. / 30.)
               - 19. / 18.) + 49. / 18.) - 23. / 6.) + 217. / 90.) - 139. / 630.;
      { REAL f = 4 - x; x = f * f * f; return x * x * f / 5040.; }
  }
  return 0;
}

/* Derivative of the B-spline (odd function). interpolation_common.h
 * fastgrad0..7.  The signed result is computed on |x| then re-signed. */
static REAL g_eval(int order, REAL x) {
  int neg = x < 0;
  if (neg) x = -x;
  REAL r;
  switch (order) {
    case 0: return 0;
    case 1: return neg ? 1 : -1;             /* fastgrad1: x<0 -> 1 else -1 */
    case 2: r = x < 0.5 ? -2 * x : x - 1.5; break;
    case 3:
      if (x < 1) r = x * (x * 1.5 - 2);
      else { REAL t = 2 - x; r = -(t * t) * 0.5; }
      break;
    case 4:
      if (x < 0.5) r = x * (x * x - 1.25);
      else if (x < 1.5) r = x * (x * (x * (-2. / 3.) + 2.5) - 2.5) + 5. / 24.;
      else { REAL t = x * 2 - 5; r = t * t * t / 48.; }
      break;
    case 5:
      if (x < 1) r = x * (x * (x * (x * (-5. / 12.) + 1.)) - 1.);
      else if (x < 2) r = x * (x * (x * (x * (5. / 24.) - 1.5) + 3.75) - 3.5) + 0.625;
      else { REAL t = x - 3; t *= t; r = -(t * t) / 24.; }
      break;
    case 6:
      if (x < 0.5) { REAL x2 = x * x; r = x * (x2 * (7. / 12.) - (x2 * x2) / 6. - 77. / 96.); }
      else if (x < 1.5)
        r = x * (x * (x * (x * (x * 0.125 - 35. / 48.) + 1.3125) - 35. / 96.) - 0.7109375) - 7. / 768.;
      else if (x < 2.5)
        r = x * (x * (x * (x * (x * (-1. / 20.) + 7. / 12.) - 2.625) + 133. / 24.) - 5.140625) + 1267. / 960.;
      else { REAL t = x * 2 - 7; REAL t2 = t * t; r = t2 * t2 * t / 3840.; }
      break;
    case 7:
      if (x < 1) { REAL x2 = x * x;
        r = x * (x2 * (x2 * (x * (7. / 144.) - 1. / 6.) + 4. / 9.) - 2. / 3.); }
      else if (x < 2)
        r = x * (x * (x * (x * (x * (x * (-7. / 240.) + 3. / 10.) - 7. / 6.) + 2.) - 7. / 6.) - 1. / 5.) - 7. / 90.;
      else if (x < 3)
        r = x * (x * (x * (x * (x * (x * (7. / 720.) - 1. / 6.) + 7. / 6.) - 38. / 9.) + 49. / 6.) - 23. / 3.) + 217. / 90.;
      else { REAL t = x - 4; REAL t3 = t * t * t; r = -(t3 * t3) / 720.; }
      break;
    default: return 0;
  }
  return neg ? -r : r;
}

/* Second derivative (even function).  Orders 0-4 follow
 * interpolation_common.h fasthess0..4.  Orders 5-7 are not implemented by
 * the reference (it returns 0, defect D3); here they use the B-spline
 * identity  B''_p(x) = B_{p-2}(x+1) - 2 B_{p-2}(x) + B_{p-2}(x-1). */
static REAL w_full(int order, REAL x);
static REAL h_eval(int order, REAL x, int quirks) {
  REAL a = fabs(x);
  switch (order) {
    case 0: case 1: return 0;
    case 2: return a < 0.5 ? -2 : 1;
    case 3: return a < 1 ? a * 3 - 2 : 2 - a;
    case 4:
      if (a < 0.5) return a * a * 3 - 1.25;
      if (a < 1.5) return a * (a * (-2.) + 5.) - 2.5;
      { REAL t = a * 2 - 5; return t * t / 8.; }
    default:
      if (quirks & OR_QUIRK_D3) return 0;
      return w_full(order - 2, x + 1) - 2 * w_full(order - 2, x) + w_full(order - 2, x - 1);
  }
}

/* Weight with explicit support test (interpolation_common.h weight0..7). */
static REAL w_full(int order, REAL x) {
  REAL a = fabs(x);
  if (order == 0) return a < 0.5 ? 1 : 0;
  if (a >= 0.5 * (order + 1)) return 0;
  return w_eval(order, x);
}

/* Support: interpolation_common.h bounds0..7.  Order 0 rounds half away
 * from zero (std::round); odd orders floor(x - (p-1)/2); even orders
 * floor(x - p/2 + 1/2).  The subtraction is done in double as in the
 * reference (double literals promote the float coordinate). */
static void support(int order, REAL x, int64_t *low) {
  double xd = (double)x;
  switch (order) {
    case 0: *low = (int64_t)round(x); break;
    case 1: *low = (int64_t)floor(xd); break;
    case 2: *low = (int64_t)floor(xd - .5); break;
    case 3: *low = (int64_t)floor(xd - 1.); break;
    case 4: *low = (int64_t)floor(xd - 1.5); break;
    case 5: *low = (int64_t)floor(xd - 2.); break;
    case 6: *low = (int64_t)floor(xd - 2.5); break;
    case 7: *low = (int64_t)floor(xd - 3.); break;
  }
}

/* Exported scalar helpers (used by the exhaustive unit tests). */
REAL or_weight(int order, REAL x) { return w_full(order, x); }
REAL or_fastweight(int order, REAL x) { return w_eval(order, x); }
REAL or_fastgrad(int order, REAL x) { return g_eval(order, x); }
REAL or_fasthess(int order, REAL x, int quirks) { return h_eval(order, x, quirks); }
int64_t or_support_low(int order, REAL x) { int64_t l; support(order, x, &l); return l; }

/* ------------------------------------------------------------------ */
/* Push / pull: pushpull_common.cpp                                    */
/* ------------------------------------------------------------------ */

/* Mode flags (pushpull_common.h:8-25 boolean arguments). */
#define OR_PULL  1
#define OR_PUSH  2
#define OR_COUNT 4
#define OR_GRAD  8
#define OR_SGRAD 16

typedef struct {
  int dim;                 /* 1, 2 or 3 */
  int bound[3];            /* per axis, compiled-backend codes */
  int order[3];            /* per axis, 0..7 */
  int extrapolate;         /* bit 0: extrapolate; bit 1: half-voxel tolerance */
  int mode;                /* OR_* flags */
  int quirks;              /* OR_QUIRK_* flags */
  int64_t N, C;
  int64_t src_size[3];     /* spatial size of the source (pull input / push output) */
  int64_t trgt_size[3];    /* spatial size of the grid */
  int64_t trgt_K;          /* 0, or dim when the target carries a gradient */
  /* source (pull/sgrad/grad input) */
  const REAL *src; int64_t src_s[5];    /* N, C, X, Y, Z strides */
  /* target (push input / backward incoming gradient) */
  const REAL *trgt; int64_t trgt_s[6];  /* N, C, X, Y, Z, K */
  /* grid */
  const REAL *grid; int64_t grid_s[5];  /* N, X, Y, Z, D */
  /* output (pull / sgrad / push / count) */
  REAL *out; int64_t out_s[6];          /* N, C, X, Y, Z, K */
  /* grid gradient output */
  REAL *ggrad; int64_t ggrad_s[5];      /* N, X, Y, Z, D */
} or_params;

/* inbounds (bounds_common.h:163-171) with TINY = 5e-2
 * (pushpull_common.cpp:58, 895-918); computed in REAL as the reference. */
static int in_fov(REAL x, int64_t n, REAL tol) {
  return x >= -tol && x < (REAL)(n - 1) + tol;
}

static void one_voxel(const or_params *p, int64_t n, int64_t w, int64_t h, int64_t d) {
  const int D = p->dim;
  int64_t sub[3] = {w, h, d};
  const REAL *gp = p->grid + n * p->grid_s[0];
  for (int a = 0; a < D; ++a) gp += sub[a] * p->grid_s[1 + a];
  REAL coord[3] = {0, 0, 0};
  for (int a = 0; a < D; ++a) coord[a] = gp[a * p->grid_s[4]];

  const int do_pull = p->mode & OR_PULL, do_push = p->mode & OR_PUSH,
            do_count = p->mode & OR_COUNT, do_grad = p->mode & OR_GRAD,
            do_sgrad = p->mode & OR_SGRAD;
  const int64_t C = p->C, K = p->trgt_K;

  /* output / target base pointers at this voxel */
  REAL *outv = NULL;
  if (do_pull || do_sgrad) {
    outv = p->out + n * p->out_s[0];
    for (int a = 0; a < D; ++a) outv += sub[a] * p->out_s[2 + a];
  }
  REAL *ggv = NULL;
  if (do_grad) {
    ggv = p->ggrad + n * p->ggrad_s[0];
    for (int a = 0; a < D; ++a) ggv += sub[a] * p->ggrad_s[1 + a];
  }

  /* out-of-bound test: pushpull_common.cpp:925-974 */
  REAL tol = (REAL)((p->extrapolate & 2) ? 0.5 + 5e-2 : 5e-2);
  int inb = 1;
  for (int a = 0; a < D; ++a) inb = inb && in_fov(coord[a], p->src_size[a], tol);
  if (!((p->extrapolate & 1) || inb)) {
    if (do_pull || do_sgrad)
      for (int64_t c = 0; c < C; ++c) {
        outv[c * p->out_s[1]] = 0;
        if (do_sgrad)
          for (int k = 1; k < D; ++k) outv[c * p->out_s[1] + k * p->out_s[5]] = 0;
      }
    if (do_grad)
      for (int a = 0; a < D; ++a) ggv[a * p->ggrad_s[4]] = 0;
    return;
  }

  /* per-axis stencil: pushpull_common.cpp:1121-1171 */
  REAL W[3][8], G[3][8], H[3][8];
  int64_t I[3][8]; int S[3][8]; int T[3];
  for (int a = 0; a < 3; ++a) { T[a] = 1; W[a][0] = 1; G[a][0] = 0; H[a][0] = 0; I[a][0] = 0; S[a][0] = 1; }
  for (int a = 0; a < D; ++a) {
    int ord = p->order[a];
    if (a == 2 && (p->quirks & OR_QUIRK_D1)) ord = p->order[1];
    int64_t low; support(ord, coord[a], &low);
    T[a] = ord + 1;
    if (ord == 0) T[a] = 1;
    for (int t = 0; t < T[a]; ++t) {
      int64_t b = low + t;
      REAL dx = coord[a] - (REAL)b;
      W[a][t] = w_eval(ord, dx);
      G[a][t] = g_eval(ord, dx);
      H[a][t] = h_eval(ord, dx, p->quirks);
      S[a][t] = or_bound_sign(p->bound[a], b, p->src_size[a]);
      I[a][t] = or_bound_index(p->bound[a], b, p->src_size[a]);
    }
  }

  const REAL *src0 = p->src ? p->src + n * p->src_s[0] : NULL;
  REAL *out0 = (do_push || do_count) ? p->out + n * p->out_s[0] : NULL;
  const REAL *trgv = NULL;
  if (p->trgt) {
    trgv = p->trgt + n * p->trgt_s[0];
    for (int a = 0; a < D; ++a) trgv += sub[a] * p->trgt_s[2 + a];
  }

  REAL acc_out[1024 * 3];
  if (do_pull || do_sgrad)
    for (int64_t c = 0; c < C * D; ++c) acc_out[c] = 0;
  REAL og[3] = {0, 0, 0};

  /* tap loop z -> y -> x (pushpull_common.cpp:1176-1290) */
  for (int k = 0; k < T[2]; ++k)
  for (int j = 0; j < T[1]; ++j)
  for (int i = 0; i < T[0]; ++i) {
    int tt[3] = {i, j, k};
    int s = 1; int64_t so = 0, oo = 0;
    REAL wv[3], gv[3], hv[3];
    for (int a = 0; a < 3; ++a) {
      s *= S[a][tt[a]];
      wv[a] = W[a][tt[a]]; gv[a] = G[a][tt[a]]; hv[a] = H[a][tt[a]];
    }
    for (int a = 0; a < D; ++a) {
      if (src0) so += I[a][tt[a]] * p->src_s[2 + a];
      if (out0) oo += I[a][tt[a]] * p->out_s[2 + a];
    }
    REAL wt = wv[0] * wv[1] * wv[2];
    /* d(weight)/d(axis a) and second derivatives */
    REAL dw[3], hh[3][3];
    for (int a = 0; a < 3; ++a) {
      REAL prod = 1;
      for (int b = 0; b < 3; ++b) prod *= (b == a) ? gv[b] : wv[b];
      dw[a] = prod;
      for (int b = 0; b < 3; ++b) {
        REAL q = 1;
        for (int e = 0; e < 3; ++e) {
          if (a == b) q *= (e == a) ? hv[e] : wv[e];
          else q *= (e == a || e == b) ? gv[e] : wv[e];
        }
        hh[a][b] = q;
      }
    }
#define SRC(c) (s == 0 ? (REAL)0 : (s < 0 ? -src0[(c) * p->src_s[1] + so] : src0[(c) * p->src_s[1] + so]))
#define TRG(c, kk) (trgv[(c) * p->trgt_s[1] + (kk) * p->trgt_s[5]])
    if (do_pull) {
      for (int64_t c = 0; c < C; ++c) acc_out[c] += SRC(c) * wt;
    } else if (do_sgrad) {
      for (int64_t c = 0; c < C; ++c) {
        REAL v = SRC(c);
        for (int a = 0; a < D; ++a) acc_out[c * D + a] += v * dw[a];
      }
    } else if (do_push) {
      if (s != 0)
        for (int64_t c = 0; c < C; ++c) {
          REAL v;
          if (K == 0) v = wt * TRG(c, 0);
          else { v = 0; for (int a = 0; a < D; ++a) v += dw[a] * TRG(c, a); }
          out0[c * p->out_s[1] + oo] += (s < 0 ? -v : v);
        }
    } else if (do_count) {
      if (s != 0) out0[oo] += (s < 0 ? -wt : wt);
    }
    if (do_grad) {
      if (K == 0) {
        REAL dot = 0;
        for (int64_t c = 0; c < C; ++c) {
          REAL v = SRC(c);
          dot += trgv ? v * TRG(c, 0) : v;
        }
        for (int a = 0; a < D; ++a) og[a] += dw[a] * dot;
      } else {
        REAL dots[3] = {0, 0, 0};
        for (int64_t c = 0; c < C; ++c) {
          REAL v = SRC(c);
          for (int b = 0; b < D; ++b) dots[b] += v * TRG(c, b);
        }
        for (int a = 0; a < D; ++a)
          for (int b = 0; b < D; ++b) og[a] += hh[a][b] * dots[b];
      }
    }
#undef SRC
#undef TRG
  }

  if (do_pull)
    for (int64_t c = 0; c < C; ++c) outv[c * p->out_s[1]] = acc_out[c];
  if (do_sgrad)
    for (int64_t c = 0; c < C; ++c)
      for (int a = 0; a < D; ++a) outv[c * p->out_s[1] + a * p->out_s[5]] = acc_out[c * D + a];
  if (do_grad)
    for (int a = 0; a < D; ++a) ggv[a * p->ggrad_s[4]] = og[a];
}

/* Sequential loop over target voxels, Z fastest (pushpull_common.cpp:802-826).
 * Outputs are expected zero-filled for push/count/grad, as the reference's
 * allocator does (pushpull_common.cpp:476-571). Returns 0. */
int or_pushpull(const or_params *p) {
  if (p->C > 1024) return -1;
  int64_t X = p->trgt_size[0], Y = p->dim > 1 ? p->trgt_size[1] : 1,
          Z = p->dim > 2 ? p->trgt_size[2] : 1;
  for (int64_t n = 0; n < p->N; ++n)
    for (int64_t w = 0; w < X; ++w)
      for (int64_t h = 0; h < Y; ++h)
        for (int64_t d = 0; d < Z; ++d)
          one_voxel(p, n, w, h, d);
  return 0;
}

int or_params_size(void) { return (int)sizeof(or_params); }

/* ------------------------------------------------------------------ */
/* Spline prefilter: nitorch/_C/_ts/coeff.py                           */
/* Always evaluated in double, whatever REAL is.                       */
/* Bound codes here are the prefilter's integer codes                  */
/* (_ts/bounds.py:7-14): 0 zero, 1 replicate, 2 dct1, 3 dct2, 4 dst1,  */
/* 5 dst2, 6 dft.                                                      */
/* ------------------------------------------------------------------ */

int or_poles(int order, double *z) {                   /* coeff.py:34-57 */
  switch (order) {
    case 0: case 1: return 0;
    case 2: z[0] = sqrt(8.) - 3.; return 1;
    case 3: z[0] = sqrt(3.) - 2.; return 1;
    case 4:
      z[0] = sqrt(664. - sqrt(438976.)) + sqrt(304.) - 19.;
      z[1] = sqrt(664. + sqrt(438976.)) - sqrt(304.) - 19.;
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

#define L(i) line[(int64_t)(i) * st]

static int64_t trunc_iter(double z) {                    /* coeff.py:72 */
  return (int64_t)ceil(-30. / log(fabs(z)));
}

static double init_dct1(const double *line, int64_t n, int64_t st, double z) {  /* coeff.py:94-134 */
  int64_t m = trunc_iter(z);
  if (m < n) {
    double out = L(0), zk = z;
    for (int64_t k = 1; k < m; ++k, zk *= z) out += zk * L(k);
    return out;
  }
  double zn = pow(z, (double)(n - 1));
  double out = L(0) + zn * L(n - 1);
  for (int64_t k = 1; k < n - 1; ++k) {
    double zk = pow(z, (double)k);
    out += (zk + zn * zn / zk) * L(k);
  }
  return out / (1. - zn * zn);
}

static double init_dct2(const double *line, int64_t n, int64_t st, double z) {  /* coeff.py:137-170 */
  double zn = pow(z, (double)n);
  double zlast = zn * (1. + 1. / (z + zn * zn));
  double out = L(0) + zlast * L(n - 1);
  for (int64_t k = 1; k < n - 1; ++k)
    out += (pow(z, (double)k) + pow(z, (double)(2 * n - 1 - k))) * L(k);
  return out * (z / (1. - zn * zn)) + L(0);
}

static double init_dft(const double *line, int64_t n, int64_t st, double z) {   /* coeff.py:69-91 */
  int64_t m = trunc_iter(z);
  if (m > n) m = n;
  double out = L(0);
  for (int64_t j = 1; j < m; ++j) out += pow(z, (double)j) * L(n - j);
  return out / (1. - pow(z, (double)m));
}

static double final_dct1(const double *line, int64_t n, int64_t st, double z) { /* coeff.py:199-205 */
  return (z * L(n - 2) + L(n - 1)) * (z / (z * z - 1.));
}

static double final_dct2(const double *line, int64_t n, int64_t st, double z) { /* coeff.py:208-215 */
  return L(n - 1) * (z / (z - 1.));
}

static double final_dft(const double *line, int64_t n, int64_t st, double z) {  /* coeff.py:173-196 */
  int64_t m = trunc_iter(z);
  if (m > n) m = n;
  double out = z * L(n - 1);
  for (int64_t j = 0; j < m - 1; ++j) out += pow(z, (double)(j + 2)) * L(j);
  return out / (pow(z, (double)m) - 1.);
}

/* One line, in place (coeff.py:254-281). Returns -2 for unsupported bounds. */
int or_coeff_line(double *line, int64_t n, int64_t st, int bound_ts, int order) {
  double z[3];
  int np = or_poles(order, z);
  if (np < 0) return -1;
  if (np == 0 || n == 1) return 0;
  int kind;
  if (bound_ts == 0 || bound_ts == 2) kind = 1;         /* dct1 */
  else if (bound_ts == 1 || bound_ts == 3) kind = 2;    /* dct2 */
  else if (bound_ts == 6) kind = 3;                     /* dft */
  else return -2;
  double gain = 1.;
  for (int q = 0; q < np; ++q) gain *= (1. - z[q]) * (1. - 1. / z[q]);
  for (int64_t i = 0; i < n; ++i) L(i) *= gain;
  for (int q = 0; q < np; ++q) {
    double p = z[q];
    L(0) = kind == 1 ? init_dct1(line, n, st, p)
         : kind == 2 ? init_dct2(line, n, st, p) : init_dft(line, n, st, p);
    for (int64_t i = 1; i < n; ++i) L(i) += p * L(i - 1);
    L(n - 1) = kind == 1 ? final_dct1(line, n, st, p)
             : kind == 2 ? final_dct2(line, n, st, p) : final_dft(line, n, st, p);
    for (int64_t i = n - 2; i >= 0; --i) L(i) = p * (L(i + 1) - L(i));
  }
  return 0;
}
#undef L

/* Filter every line of a contiguous array along one axis.
 * shape: `ndim` sizes (C order); axis: the filtered axis. */
int or_coeff_axis(double *data, int ndim, const int64_t *shape, int axis,
                  int bound_ts, int order) {
  int64_t outer = 1, inner = 1, n = shape[axis];
  for (int a = 0; a < axis; ++a) outer *= shape[a];
  for (int a = axis + 1; a < ndim; ++a) inner *= shape[a];
  for (int64_t o = 0; o < outer; ++o)
    for (int64_t i = 0; i < inner; ++i) {
      int r = or_coeff_line(data + o * n * inner + i, n, inner, bound_ts, order);
      if (r) return r;
    }
  return 0;
}
