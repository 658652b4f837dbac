/*
 * andfn_oracle.c -- CPU oracle for the AnDFN analytic-element solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, function by function, the
 * Numba kernels of AnDFN v0.1.16 (the andfn/hpc package) so that tests and the
 * benchmark's CPU leg can check and time the CUDA implementation against the
 * reference algorithm.  Nothing in the product (andfn_b200/) links or calls it.
 *
 * Pinning: tests/test_oracle_golden.py compares this oracle (driven by
 * oracle/oracle.py) with golden vectors that tests/golden/make_golden.py wrote
 * by running the reference's own hpc_solve on seeded networks.
 *
 * Arithmetic follows Numba 0.65 semantics for complex128, so that results can
 * agree with the reference to the last bit where the operation order does:
 *   - a real operand of a complex operation is promoted to (x, +0.0);
 *   - complex division is Smith's algorithm (CPython _Py_c_quot, numba
 *     numbers.complex_div_impl);
 *   - sqrt(z) is Algorithm 312 with hypot (numba cmathimpl.sqrt_impl);
 *   - log(z) = (log(hypot(x, y)), atan2(y, x)) (numba cmathimpl.log_impl);
 *   - exp(i t) = (cos t, sin t) (numba cmathimpl.exp_impl with x = 0);
 *   - abs(z) = hypot(x, y).
 * Build with -ffp-contract=off and no -march so no FMA is contracted.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/andfn_b200.h"

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  double re, im;
} cplx;

static const double PI = 3.141592653589793115997963468544185161590576171875;

/* ---- complex helpers (numba semantics) ---------------------------------- */
static inline cplx C(double re, double im) {
  cplx z = {re, im};
  return z;
}
static inline cplx cadd(cplx a, cplx b) { return C(a.re + b.re, a.im + b.im); }
static inline cplx csub(cplx a, cplx b) { return C(a.re - b.re, a.im - b.im); }
static inline cplx cmul(cplx x, cplx y) {
  return C(x.re * y.re - x.im * y.im, x.re * y.im + x.im * y.re);
}
/* real * complex with the real promoted to (r, +0.0) */
static inline cplx rmul(double r, cplx y) { return cmul(C(r, 0.0), y); }
static inline cplx cdiv(cplx a, cplx b) {
  /* Smith's algorithm as in CPython _Py_c_quot */
  double br = b.re, bi = b.im;
  if (fabs(br) >= fabs(bi)) {
    if (br == 0.0 && bi == 0.0) return C(NAN, NAN);
    if (br == 0.0) return C(NAN, NAN);
    double ratio = bi / br;
    double denom = br + bi * ratio;
    return C((a.re + a.im * ratio) / denom, (a.im - a.re * ratio) / denom);
  } else {
    if (bi == 0.0) return C(NAN, NAN);
    double ratio = br / bi;
    double denom = br * ratio + bi;
    return C((a.re * ratio + a.im) / denom, (a.im * ratio - a.re) / denom);
  }
}
static inline cplx cdivr(cplx a, double r) { return cdiv(a, C(r, 0.0)); }
/* NumPy's complex true_divide as numba lowers np.divide (npyfuncs.np_complex_div_impl):
 * Smith's algorithm with a multiply by the reciprocal of the scaled denominator. */
static inline cplx cdiv_np(cplx a, cplx b) {
  double br = b.re, bi = b.im;
  if (fabs(br) >= fabs(bi)) {
    if (fabs(br) == 0.0 && fabs(bi) == 0.0) return C(a.re / fabs(br), a.im / fabs(bi));
    double rat = bi / br;
    double scl = 1.0 / (br + bi * rat);
    return C((a.re + a.im * rat) * scl, (a.im - a.re * rat) * scl);
  } else {
    double rat = br / bi;
    double scl = 1.0 / (bi + br * rat);
    return C((a.re * rat + a.im) * scl, (a.im * rat - a.re) * scl);
  }
}
static inline double cabs_(cplx z) { return hypot(z.re, z.im); }
static inline cplx clog_(cplx z) { return C(log(hypot(z.re, z.im)), atan2(z.im, z.re)); }
static inline cplx csqrt_(cplx z) {
  /* numba cmathimpl.sqrt_impl (NumPy npy_csqrt, Algorithm 312) */
  const double THRES = 1.7976931348623157e308 / (1.0 + 1.4142135623730951);
  double a = z.re, b = z.im;
  if (a == 0.0 && b == 0.0) return C(fabs(b), b);
  if (isinf(b)) return C(fabs(b), b);
  if (isnan(a)) return C(a, a);
  if (isinf(a)) {
    if (a < 0.0) return C(fabs(b - b), copysign(a, b));
    return C(a, copysign(b - b, b));
  }
  int scale = 0;
  if (fabs(a) >= THRES || fabs(b) >= THRES) {
    a *= 0.25;
    b *= 0.25;
    scale = 1;
  }
  double re, im;
  if (a >= 0) {
    double t = sqrt((a + hypot(a, b)) * 0.5);
    re = t;
    im = b / (2 * t);
  } else {
    double t = sqrt((-a + hypot(a, b)) * 0.5);
    re = fabs(b) / (2 * t);
    im = copysign(t, b);
  }
  if (scale) return C(re * 2, im);
  return C(re, im);
}
static inline cplx cexpi(double t) { return C(cos(t), sin(t)); }
static inline double sgn(double x) { return (x > 0) - (x < 0) + (x != x ? NAN : 0.0); }

/* ---- record access ------------------------------------------------------ */
typedef struct {
  const AndfnLayout *L;
  char *E; /* element records */
  char *F; /* fracture records */
  int64_t ne, nf;
} Net;

#define EI64(n, i, off) (*(int64_t *)((n)->E + (i) * (n)->L->elem_size + (n)->L->off))
#define EF64(n, i, off) (*(double *)((n)->E + (i) * (n)->L->elem_size + (n)->L->off))
#define EPTR(n, i, off) ((double *)((n)->E + (i) * (n)->L->elem_size + (n)->L->off))
#define FI64(n, f, off) (*(int64_t *)((n)->F + (f) * (n)->L->frac_size + (n)->L->off))
#define FF64(n, f, off) (*(double *)((n)->F + (f) * (n)->L->frac_size + (n)->L->off))
#define FPTR(n, f, off) ((int64_t *)((n)->F + (f) * (n)->L->frac_size + (n)->L->off))

static inline cplx ecoef(const Net *n, int64_t i, int64_t k) {
  double *p = EPTR(n, i, e_coef);
  return C(p[2 * k], p[2 * k + 1]);
}
static inline void set_ecoef(const Net *n, int64_t i, int64_t k, cplx v) {
  double *p = EPTR(n, i, e_coef);
  p[2 * k] = v.re;
  p[2 * k + 1] = v.im;
}
static inline cplx eptc(const Net *n, int64_t i, int64_t off, int64_t k) {
  double *p = (double *)(n->E + i * n->L->elem_size + off);
  return C(p[2 * k], p[2 * k + 1]);
}

/* ---- per-element work (andfn/hpc/hpc_solve.py:26-46 dtype_work) -------- */
typedef struct {
  double *phi, *psi, *dpsi;                      /* [2M] */
  cplx *coef, *coef0, *coef1, *old_coef;         /* [M]  */
  cplx *integral, *exp_m, *exp_p;                /* [2M] */
  int64_t *sign_array, *discharge_element, *element_pos; /* [MAXE] */
  int64_t len_discharge_element;
  int set_zero;
} Work;

typedef struct {
  int64_t ne, M, MAXE;
  Work *w;
  void *mem;
} OracleCtx;

/* ---- maps (andfn/hpc/hpc_geometry_functions.py:12-99) ------------------- */
static inline cplx map_z_line_to_chi(cplx z, cplx a, cplx b) {
  /* big_z = (2 z - a - b) / (b - a); chi = big_z + sqrt(big_z-1) sqrt(big_z+1) */
  cplx bz = cdiv(csub(csub(cmul(C(2.0, 0.0), z), a), b), csub(b, a));
  cplx s1 = csqrt_(C(bz.re - 1.0, bz.im - 0.0));
  cplx s2 = csqrt_(C(bz.re + 1.0, bz.im + 0.0));
  return cadd(bz, cmul(s1, s2));
}
static inline cplx map_chi_to_z_line(cplx chi, cplx a, cplx b) {
  /* big_z = 1/2 (chi + 1/chi); z = 1/2 (big_z (b - a) + a + b) */
  cplx bz = rmul(0.5, cadd(chi, cdiv(C(1.0, 0.0), chi)));
  return rmul(0.5, cadd(cadd(cmul(bz, csub(b, a)), a), b));
}
static inline cplx map_z_circle_to_chi(cplx z, double r, cplx c) { return cdivr(csub(z, c), r); }
static inline cplx map_chi_to_z_circle(cplx chi, double r, cplx c) { return cadd(rmul(r, chi), c); }

/* ---- series (andfn/hpc/hpc_math_functions.py:17-40, 104-128, 194-213) --- */
static inline cplx asym_expansion(cplx chi, const double *coef, int64_t m, double sign) {
  cplx res = C(0.0, 0.0);
  for (int64_t n = 0; n < m - 1; n++) {
    int64_t k = m - n - 1;
    res = cadd(res, C(sign * coef[2 * k], sign * coef[2 * k + 1]));
    res = cdiv(res, chi);
  }
  if (m > 0) res = cadd(res, C(sign * coef[0], sign * coef[1]));
  return res;
}
static inline cplx taylor_series(cplx chi, const double *coef, int64_t m) {
  cplx res = C(0.0, 0.0);
  for (int64_t n = 0; n < m - 1; n++) {
    int64_t k = m - n - 1;
    res = cadd(res, C(coef[2 * k], coef[2 * k + 1]));
    res = cmul(res, chi);
  }
  if (m > 0) res = cadd(res, C(coef[0], coef[1]));
  return res;
}
static inline cplx well_chi(cplx chi, double q) { return rmul(q / (2 * PI), clog_(chi)); }

/* ---- element potentials (andfn/hpc/hpc_*.py calc_omega) ---------------- */
static cplx element_omega(const Net *n, int64_t el, cplx z, int64_t frac_id) {
  int64_t type = EI64(n, el, e_type);
  int64_t m = EI64(n, el, e_ncoef);
  const double *coef = EPTR(n, el, e_coef);
  double q = EF64(n, el, e_q);
  switch (type) {
    case 0: { /* hpc_intersection.py:116-146 */
      if (frac_id == EI64(n, el, e_frac0)) {
        cplx chi = map_z_line_to_chi(z, eptc(n, el, n->L->e_endpoints0, 0), eptc(n, el, n->L->e_endpoints0, 1));
        return cadd(asym_expansion(chi, coef, m, 1.0), well_chi(chi, q));
      } else {
        cplx chi = map_z_line_to_chi(z, eptc(n, el, n->L->e_endpoints1, 0), eptc(n, el, n->L->e_endpoints1, 1));
        return cadd(asym_expansion(chi, coef, m, -1.0), well_chi(chi, -q));
      }
    }
    case 1: { /* hpc_bounding_circle.py:8-25, 53-71: the center is not used */
      cplx chi = map_z_circle_to_chi(z, EF64(n, el, e_radius), C(0.0, 0.0));
      /* map_z_circle_to_chi(z, r) has center=0.0 (a float): z - 0.0 */
      return taylor_series(chi, coef, m);
    }
    case 2: { /* hpc_well.py:39-60 */
      cplx chi = map_z_circle_to_chi(z, EF64(n, el, e_radius), eptc(n, el, n->L->e_center, 0));
      cplx om = well_chi(chi, q);
      if (cabs_(chi) < 1 - 1e-12) om = C(NAN, NAN);
      return om;
    }
    case 3: { /* hpc_const_head_line.py:89-108 */
      cplx chi = map_z_line_to_chi(z, eptc(n, el, n->L->e_endpoints0, 0), eptc(n, el, n->L->e_endpoints0, 1));
      cplx om = well_chi(chi, q);
      return cadd(om, asym_expansion(chi, coef, m, 1.0));
    }
    case 4: { /* hpc_imp_object.py:68-88 */
      cplx chi = map_z_circle_to_chi(z, EF64(n, el, e_radius), eptc(n, el, n->L->e_center, 0));
      if (cabs_(chi) < 1.0 - 1e-10) return C(NAN, NAN);
      return asym_expansion(chi, coef, m, 1.0);
    }
    case 5: { /* hpc_imp_object.py:187-205 */
      cplx chi = map_z_line_to_chi(z, eptc(n, el, n->L->e_endpoints0, 0), eptc(n, el, n->L->e_endpoints0, 1));
      return asym_expansion(chi, coef, m, 1.0);
    }
  }
  return C(0.0, 0.0);
}

/* hpc_fracture.py:52-94 */
static cplx calc_omega(const Net *n, int64_t f, cplx z, int64_t exclude) {
  cplx omega = C(FF64(n, f, f_constant), 0.0);
  int64_t ne = FI64(n, f, f_nelements);
  const int64_t *els = FPTR(n, f, f_elements);
  int64_t fid = FI64(n, f, f_id);
  for (int64_t k = 0; k < ne; k++) {
    int64_t el = els[k];
    if (el != exclude) omega = cadd(omega, element_omega(n, el, z, fid));
  }
  return omega;
}

/* ---- thetas / exp arrays (hpc_math_functions.py:674-723) ---------------- */
static void calc_thetas(int64_t nn, int64_t type, double *thetas) {
  double del = PI / nn;
  double start = del / 2;
  if (type == 1) {
    del = 2 * PI / nn;
    start = 0.0;
  }
  for (int64_t i = 0; i < nn; i++) thetas[i] = start + i * del;
}
static void fill_exp(int64_t nn, const double *thetas, cplx *out, int sign) {
  for (int64_t i = 0; i < nn; i++) {
    double t = thetas[i];
    /* exp(sign * 1j * t): the exponent's real part is a signed zero, exp(+-0)=1 */
    cplx e = cexpi(sign > 0 ? t : -t);
    out[i] = e;
  }
}

/* ---- Cauchy integrals (hpc_math_functions.py:244-297, 451-608) ---------- */
static void dft_coefs(int64_t nn, int64_t m, const double *vals, const cplx *exp_m, cplx *integral) {
  for (int64_t jj = 0; jj < m; jj++) {
    cplx res = C(0.0, 0.0);
    for (int64_t ii = 0; ii < nn; ii++) {
      cplx ev = C(1.0, 0.0);
      for (int64_t r = 0; r < jj; r++) ev = cmul(ev, exp_m[ii]);
      res = cadd(res, rmul(vals[ii], ev));
    }
    integral[jj] = res;
  }
}

static void cauchy_integral_real(const Net *n, Work *w, int64_t nn, int64_t m, int64_t f, int64_t self,
                                 cplx a, cplx b, cplx *coef) {
  for (int64_t ii = 0; ii < nn; ii++) {
    cplx z = map_chi_to_z_line(w->exp_p[ii], a, b);
    w->phi[ii] = calc_omega(n, f, z, self).re;
  }
  dft_coefs(nn, m, w->phi, w->exp_m, w->integral);
  for (int64_t ii = 0; ii < m; ii++) coef[ii] = cdivr(cmul(C(2.0, 0.0), w->integral[ii]), (double)nn);
  coef[0] = cdivr(coef[0], 2.0);
}

static void psi_unwrap(Work *w, int64_t nn, const double *dpsi_corr) {
  for (int64_t ii = 1; ii < nn; ii++) w->dpsi[ii] = (w->psi[ii] - w->psi[ii - 1]) - dpsi_corr[ii - 1];
  double psi0 = w->psi[0];
  for (int64_t ii = 0; ii < nn; ii++) {
    double psi1 = psi0 + w->dpsi[ii];
    w->psi[ii] = psi1;
    psi0 = psi1;
  }
}

static void cauchy_integral_domega(const Net *n, Work *w, int64_t nn, int64_t m, const double *dpsi_corr,
                                   int64_t f, int64_t self, int line, double radius, cplx center, cplx a,
                                   cplx b, cplx *coef) {
  for (int64_t ii = 0; ii < nn; ii++) {
    cplx z = line ? map_chi_to_z_line(w->exp_p[ii], a, b) : map_chi_to_z_circle(w->exp_p[ii], radius, center);
    w->psi[ii] = calc_omega(n, f, z, self).im;
  }
  psi_unwrap(w, nn, dpsi_corr);
  dft_coefs(nn, m, w->psi, w->exp_m, w->integral);
  for (int64_t ii = 0; ii < m; ii++) coef[ii] = cdivr(cmul(C(0.0, 2.0), w->integral[ii]), (double)nn);
  coef[0] = cdivr(coef[0], 2.0);
}

/* ---- branch cuts (hpc_math_functions.py:301-447) ------------------------ */
static void get_sign(int64_t self_type, Work *w, int64_t cnt, cplx chi0, cplx chi1, int64_t sign_default) {
  if (self_type != 1) {
    w->sign_array[cnt] = (chi0.im < chi1.im) ? -1 * sign_default : sign_default;
  } else {
    w->sign_array[cnt] = sign_default;
  }
}

static int find_branch_cuts(const Net *n, OracleCtx *ctx, int64_t self, const cplx *z_pos) {
  Work *w = &ctx->w[self];
  int64_t nint = EI64(n, self, e_nint);
  int64_t f = EI64(n, self, e_frac0);
  int64_t self_type = EI64(n, self, e_type);
  int64_t nel = FI64(n, f, f_nelements);
  const int64_t *els = FPTR(n, f, f_elements);
  w->len_discharge_element = 0;
  int64_t cnt = 0;
  for (int64_t ii = 0; ii < nint - 1; ii++) {
    for (int64_t k = 0; k < nel; k++) {
      int64_t e = els[k];
      int64_t t = EI64(n, e, e_type);
      int hit = 0;
      cplx chi0, chi1;
      int64_t sdef = -1;
      if (t == 0) {
        int64_t off = (EI64(n, e, e_frac0) == f) ? n->L->e_endpoints0 : n->L->e_endpoints1;
        sdef = (EI64(n, e, e_frac0) == f) ? -1 : 1;
        chi0 = map_z_line_to_chi(z_pos[ii], eptc(n, e, off, 0), eptc(n, e, off, 1));
        chi1 = map_z_line_to_chi(z_pos[ii + 1], eptc(n, e, off, 0), eptc(n, e, off, 1));
        double ln0 = clog_(chi0).im, ln1 = clog_(chi1).im;
        hit = (sgn(ln0) != sgn(ln1)) && (fabs(ln0) + fabs(ln1) > PI);
      } else if (t == 2) {
        cplx c = eptc(n, e, n->L->e_center, 0);
        double r = EF64(n, e, e_radius);
        chi0 = map_z_circle_to_chi(z_pos[ii], r, c);
        chi1 = map_z_circle_to_chi(z_pos[ii + 1], r, c);
        hit = (sgn(chi0.im) != sgn(chi1.im)) && (chi0.re < 0);
      } else if (t == 3) {
        chi0 = map_z_line_to_chi(z_pos[ii], eptc(n, e, n->L->e_endpoints0, 0), eptc(n, e, n->L->e_endpoints0, 1));
        chi1 = map_z_line_to_chi(z_pos[ii + 1], eptc(n, e, n->L->e_endpoints0, 0),
                                 eptc(n, e, n->L->e_endpoints0, 1));
        hit = (sgn(chi0.im) != sgn(chi1.im)) && (chi0.re < 0);
      }
      if (hit) {
        if (cnt >= ctx->MAXE) return -1;
        w->element_pos[cnt] = ii;
        w->discharge_element[cnt] = EI64(n, e, e_id);
        get_sign(self_type, w, cnt, chi0, chi1, sdef);
        w->len_discharge_element += 1;
        cnt += 1;
      }
    }
  }
  return 0;
}

static int get_dpsi_corr(const Net *n, OracleCtx *ctx, int64_t self) {
  Work *w = &ctx->w[self];
  int64_t nint = EI64(n, self, e_nint);
  int64_t type = EI64(n, self, e_type);
  if (w->len_discharge_element == 0) {
    cplx *z_pos = (cplx *)malloc(sizeof(cplx) * (nint > 0 ? nint : 1));
    for (int64_t i = 0; i < nint; i++) {
      if (type == 1 || type == 4)
        z_pos[i] = map_chi_to_z_circle(w->exp_p[i], EF64(n, self, e_radius), eptc(n, self, n->L->e_center, 0));
      else
        z_pos[i] = map_chi_to_z_line(w->exp_p[i], eptc(n, self, n->L->e_endpoints0, 0),
                                     eptc(n, self, n->L->e_endpoints0, 1));
    }
    int rc = find_branch_cuts(n, ctx, self, z_pos);
    free(z_pos);
    if (rc) return rc;
  }
  double *dc = EPTR(n, self, e_dpsi_corr);
  for (int64_t i = 0; i < nint - 1; i++) dc[i] = 0.0;
  for (int64_t i = 0; i < w->len_discharge_element; i++) {
    int64_t e = w->discharge_element[i];
    dc[w->element_pos[i]] += EF64(n, e, e_q) * (double)w->sign_array[i];
  }
  return 0;
}

/* ---- error metrics (hpc_math_functions.py:612-670) ---------------------- */
static double calc_error(const cplx *coef, const cplx *ref, int64_t m) {
  double s = 0.0;
  for (int64_t i = 0; i < 5 && i < m; i++) s += cabs_(ref[i]);
  if (s < 1e-15) return 0.0;
  cplx c1 = C(0.0, 0.0), c10 = C(0.0, 0.0);
  for (int64_t i = 0; i < m; i++) c1 = cadd(c1, coef[i]);
  for (int64_t i = (int64_t)(m * 0.9); i < m; i++) c10 = cadd(c10, coef[i]);
  return fabs(cabs_(csub(c1, c10)) / cabs_(C(c1.re + 1e-16, c1.im + 0.0)) - 1);
}
static double calc_coef_error(const cplx *coef, const cplx *ref, int64_t m) {
  double s = 0.0;
  for (int64_t i = 0; i < 5 && i < m; i++) s += cabs_(ref[i]);
  if (s < 1e-15) return 0.0;
  double err = 0.0;
  for (int64_t i = 0; i < m; i++) err += cabs_(csub(coef[i], ref[i]));
  return err / m;
}

static void push_errors(const Net *n, int64_t i, Work *w) {
  int64_t m = EI64(n, i, e_ncoef);
  EF64(n, i, e_error_old2) = EF64(n, i, e_error_old);
  EF64(n, i, e_error_old) = EF64(n, i, e_error);
  EF64(n, i, e_error) = calc_error(w->coef, w->old_coef, m);
  EF64(n, i, e_error_coef) = calc_coef_error(w->coef, w->old_coef, m);
}

static void save_old(const Net *n, int64_t i, Work *w) {
  int64_t m = EI64(n, i, e_ncoef);
  for (int64_t k = 0; k < m; k++) w->old_coef[k] = ecoef(n, i, k);
}

/* ---- per-type solves ---------------------------------------------------- */
static int solve_element(const Net *n, OracleCtx *ctx, int64_t i) {
  Work *w = &ctx->w[i];
  int64_t type = EI64(n, i, e_type);
  int64_t m = EI64(n, i, e_ncoef), nn = EI64(n, i, e_nint);
  int64_t f0 = EI64(n, i, e_frac0);
  int64_t self = EI64(n, i, e_id);
  switch (type) {
    case 0: { /* hpc_intersection.py:50-113 */
      int64_t f1 = EI64(n, i, e_frac1);
      save_old(n, i, w);
      cauchy_integral_real(n, w, nn, m, f0, self, eptc(n, i, n->L->e_endpoints0, 0),
                           eptc(n, i, n->L->e_endpoints0, 1), w->coef0);
      cauchy_integral_real(n, w, nn, m, f1, self, eptc(n, i, n->L->e_endpoints1, 0),
                           eptc(n, i, n->L->e_endpoints1, 1), w->coef1);
      double t0 = FF64(n, f0, f_t), t1 = FF64(n, f1, f_t);
      for (int64_t k = 0; k < m; k++)
        w->coef[k] = C(cdivr(csub(rmul(t0, w->coef1[k]), rmul(t1, w->coef0[k])), t0 + t1).re, 0.0);
      w->coef[0] = C(0.0, 0.0);
      push_errors(n, i, w);
      return 0;
    }
    case 1: { /* hpc_bounding_circle.py:119-163 */
      if (get_dpsi_corr(n, ctx, i)) return -1;
      save_old(n, i, w);
      cauchy_integral_domega(n, w, nn, m, EPTR(n, i, e_dpsi_corr), f0, self, 0, EF64(n, i, e_radius),
                             eptc(n, i, n->L->e_center, 0), C(0, 0), C(0, 0), w->coef);
      for (int64_t k = 0; k < m; k++) w->coef[k] = C(-w->coef[k].re, -w->coef[k].im);
      push_errors(n, i, w);
      return 0;
    }
    case 2: /* hpc_solve.py:366-368 */
      EF64(n, i, e_error) = 0.0;
      return 0;
    case 3: { /* hpc_const_head_line.py:39-85 */
      save_old(n, i, w);
      cauchy_integral_real(n, w, nn, m, f0, self, eptc(n, i, n->L->e_endpoints0, 0),
                           eptc(n, i, n->L->e_endpoints0, 1), w->coef);
      for (int64_t k = 0; k < m; k++) w->coef[k] = C(-w->coef[k].re, 0.0);
      w->coef[0] = C(0.0, 0.0);
      push_errors(n, i, w);
      return 0;
    }
    case 4: { /* hpc_imp_object.py:18-64 */
      if (get_dpsi_corr(n, ctx, i)) return -1;
      save_old(n, i, w);
      cauchy_integral_domega(n, w, nn, m, EPTR(n, i, e_dpsi_corr), f0, self, 0, EF64(n, i, e_radius),
                             eptc(n, i, n->L->e_center, 0), C(0, 0), C(0, 0), w->coef);
      for (int64_t k = 0; k < m; k++) w->coef[k] = C(w->coef[k].re, -w->coef[k].im);
      w->coef[0] = C(0.0, 0.0);
      push_errors(n, i, w);
      return 0;
    }
    case 5: { /* hpc_imp_object.py:125-183 */
      if (get_dpsi_corr(n, ctx, i)) return -1;
      save_old(n, i, w);
      cauchy_integral_domega(n, w, nn, m, EPTR(n, i, e_dpsi_corr), f0, self, 1, 0.0, C(0, 0),
                             eptc(n, i, n->L->e_endpoints0, 0), eptc(n, i, n->L->e_endpoints0, 1), w->coef);
      for (int64_t k = 0; k < m; k++) w->coef[k] = rmul(-w->coef[k].im, C(0.0, 1.0));
      w->coef[0] = C(0.0, 0.0);
      push_errors(n, i, w);
      return 0;
    }
  }
  return 0;
}

static void blend(const Net *n, OracleCtx *ctx, int64_t i, double damping) {
  int64_t m = EI64(n, i, e_ncoef);
  for (int64_t k = 0; k < m; k++) {
    cplx v = cadd(rmul(damping, ctx->w[i].coef[k]), rmul(1 - damping, ecoef(n, i, k)));
    set_ecoef(n, i, k, v);
  }
}

/* ======================= exported oracle entry points ===================== */

void *oracle_create(int64_t ne, int64_t max_ncoef, int64_t max_elements) {
  OracleCtx *ctx = (OracleCtx *)calloc(1, sizeof(OracleCtx));
  ctx->ne = ne;
  ctx->M = max_ncoef;
  ctx->MAXE = max_elements;
  ctx->w = (Work *)calloc(ne > 0 ? ne : 1, sizeof(Work));
  size_t per = sizeof(double) * 2 * max_ncoef * 3 + sizeof(cplx) * max_ncoef * 4 + sizeof(cplx) * 2 * max_ncoef * 3 +
               sizeof(int64_t) * max_elements * 3;
  char *mem = (char *)calloc((size_t)(ne > 0 ? ne : 1), per);
  ctx->mem = mem;
  for (int64_t i = 0; i < ne; i++) {
    char *p = mem + (size_t)i * per;
    Work *w = &ctx->w[i];
    w->phi = (double *)p; p += sizeof(double) * 2 * max_ncoef;
    w->psi = (double *)p; p += sizeof(double) * 2 * max_ncoef;
    w->dpsi = (double *)p; p += sizeof(double) * 2 * max_ncoef;
    w->coef = (cplx *)p; p += sizeof(cplx) * max_ncoef;
    w->coef0 = (cplx *)p; p += sizeof(cplx) * max_ncoef;
    w->coef1 = (cplx *)p; p += sizeof(cplx) * max_ncoef;
    w->old_coef = (cplx *)p; p += sizeof(cplx) * max_ncoef;
    w->integral = (cplx *)p; p += sizeof(cplx) * 2 * max_ncoef;
    w->exp_m = (cplx *)p; p += sizeof(cplx) * 2 * max_ncoef;
    w->exp_p = (cplx *)p; p += sizeof(cplx) * 2 * max_ncoef;
    w->sign_array = (int64_t *)p; p += sizeof(int64_t) * max_elements;
    w->discharge_element = (int64_t *)p; p += sizeof(int64_t) * max_elements;
    w->element_pos = (int64_t *)p; p += sizeof(int64_t) * max_elements;
  }
  return ctx;
}

void oracle_destroy(void *p) {
  OracleCtx *ctx = (OracleCtx *)p;
  if (!ctx) return;
  free(ctx->mem);
  free(ctx->w);
  free(ctx);
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* hpc_solve.py:124-137: error/error_old = 1e30, thetas and exp tables */
void oracle_init(void *p, const AndfnLayout *L, char *E, int64_t ne) {
  OracleCtx *ctx = (OracleCtx *)p;
  Net n = {L, E, NULL, ne, 0};
  for (int64_t i = 0; i < ne; i++) {
    EF64(&n, i, e_error_old) = 1e30;
    EF64(&n, i, e_error) = 1e30;
  }
  for (int64_t i = 0; i < ne; i++) {
    int64_t nn = EI64(&n, i, e_nint);
    double *th = EPTR(&n, i, e_thetas);
    calc_thetas(nn, EI64(&n, i, e_type), th);
    fill_exp(nn, th, ctx->w[i].exp_m, -1);
    fill_exp(nn, th, ctx->w[i].exp_p, 1);
  }
}

/* hpc_solve.py:1427-1447 and the per-type z_array functions:
 * D interior points of linspace(a, b, D+2) on line elements, r e^{i theta} + c on wells.
 * z0/z1: complex [n_de * D]. */
static void linspace_interior(cplx a, cplx b, int64_t D, cplx *out) {
  /* numba np.linspace(a, b, D + 2)[1 : D + 1] (numba/np/arrayobj.py linspace) */
  int64_t num = D + 2;
  a = rmul(1.0, a); /* start = start * 1.0 */
  b = rmul(1.0, b);
  cplx delta = csub(b, a);
  cplx step = cdiv_np(delta, C((double)(num - 1), 0.0));
  for (int64_t i = 1; i <= D; i++) {
    cplx v = cadd(a, cmul(C((double)i, 0.0), step));
    if (i == num - 1) v = b;
    out[i - 1] = v;
  }
}

void oracle_z_int(const AndfnLayout *L, char *E, const int64_t *de_ids, int64_t n_de, int64_t D, double *z0,
                  double *z1) {
  Net n = {L, E, NULL, 0, 0};
  for (int64_t j = 0; j < n_de; j++) {
    int64_t e = de_ids[j];
    int64_t t = EI64(&n, e, e_type);
    cplx *o0 = (cplx *)(z0 + 2 * j * D);
    cplx *o1 = (cplx *)(z1 + 2 * j * D);
    if (t == 0) {
      linspace_interior(eptc(&n, e, L->e_endpoints0, 0), eptc(&n, e, L->e_endpoints0, 1), D, o0);
      linspace_interior(eptc(&n, e, L->e_endpoints1, 0), eptc(&n, e, L->e_endpoints1, 1), D, o1);
    } else if (t == 3) {
      linspace_interior(eptc(&n, e, L->e_endpoints0, 0), eptc(&n, e, L->e_endpoints0, 1), D, o0);
    } else if (t == 2) {
      /* hpc_well.py:128-130: theta = linspace(0, 2pi - 2pi/D, D); z = r exp(i theta) + c */
      double stop = 2.0 * PI - 2 * PI / D;
      double r = EF64(&n, e, e_radius);
      cplx c = eptc(&n, e, L->e_center, 0);
      for (int64_t i = 0; i < D; i++) {
        double th;
        if (D - 1 > 0) {
          double step = (stop - 0.0) / (double)(D - 1);
          th = 0.0 + i * step;
          if (i == D - 1) th = stop;
        } else {
          th = 0.0;
        }
        o0[i] = cadd(rmul(r, cexpi(th)), c);
      }
    }
  }
}

static inline double discharge_term_(const Net *n, int64_t ee, const cplx *z, int64_t D, int64_t frac) {
  int64_t t = EI64(n, ee, e_type);
  double phi = 0.0;
  if (t == 0) { /* hpc_intersection.py:23-46 */
    double sign = 1.0;
    int64_t off = n->L->e_endpoints0;
    if (frac != EI64(n, ee, e_frac0)) {
      sign = -1.0;
      off = n->L->e_endpoints1;
    }
    for (int64_t i = 0; i < D; i++)
      phi += well_chi(map_z_line_to_chi(z[i], eptc(n, ee, off, 0), eptc(n, ee, off, 1)), sign).re;
    return phi / D;
  } else if (t == 2) { /* hpc_well.py:15-35 */
    for (int64_t i = 0; i < D; i++)
      phi += well_chi(map_z_circle_to_chi(z[i], EF64(n, ee, e_radius), eptc(n, ee, n->L->e_center, 0)), 1.0).re;
    return phi / D;
  } else if (t == 3) { /* hpc_const_head_line.py:15-35 */
    for (int64_t i = 0; i < D; i++)
      phi += well_chi(map_z_line_to_chi(z[i], eptc(n, ee, n->L->e_endpoints0, 0), eptc(n, ee, n->L->e_endpoints0, 1)),
                      1.0).re;
    return phi / D;
  }
  return 0.0;
}

static inline int is_disch(int64_t t) { return t == 0 || t == 2 || t == 3; }

/* hpc_solve.py:1061-1104: nonzeros per row */
int64_t oracle_count_nnz(const AndfnLayout *L, char *E, char *F, int64_t nf, const int64_t *de_ids, int64_t n_de,
                         int64_t *nnz_per_row) {
  Net n = {L, E, F, 0, nf};
  int64_t total = 0;
  for (int64_t j = 0; j < n_de; j++) {
    int64_t e = de_ids[j];
    int64_t cnt = 0;
    int64_t fr[2] = {EI64(&n, e, e_frac0), EI64(&n, e, e_frac1)};
    int nside = EI64(&n, e, e_type) == 0 ? 2 : 1;
    for (int s = 0; s < nside; s++) {
      int64_t f = fr[s];
      int64_t ne = FI64(&n, f, f_nelements);
      const int64_t *els = FPTR(&n, f, f_elements);
      for (int64_t k = 0; k < ne; k++) {
        int64_t ee = els[k];
        if (EI64(&n, ee, e_id) == EI64(&n, e, e_id) || !is_disch(EI64(&n, ee, e_type))) continue;
        cnt++;
      }
    }
    cnt += nside;
    nnz_per_row[j] = cnt;
    total += cnt;
  }
  for (int64_t f = 0; f < nf; f++) {
    int64_t cnt = 0;
    int64_t ne = FI64(&n, f, f_nelements);
    const int64_t *els = FPTR(&n, f, f_elements);
    for (int64_t k = 0; k < ne; k++)
      if (is_disch(EI64(&n, els[k], e_type))) cnt++;
    nnz_per_row[n_de + f] = cnt;
    total += cnt;
  }
  return total;
}

/* hpc_solve.py:1117-1201: COO entries; id_to_pos maps element id -> unknown */
void oracle_fill_matrix(const AndfnLayout *L, char *E, char *F, int64_t nf, const int64_t *de_ids, int64_t n_de,
                        const int64_t *id_to_pos, const double *z0, const double *z1, int64_t D,
                        const int64_t *row_offsets, int64_t *rows, int64_t *cols, double *data) {
  Net n = {L, E, F, 0, nf};
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t j = 0; j < n_de; j++) {
    int64_t e = de_ids[j];
    int64_t ptr = row_offsets[j];
    const cplx *zz0 = (const cplx *)(z0 + 2 * j * D);
    const cplx *zz1 = (const cplx *)(z1 + 2 * j * D);
    if (EI64(&n, e, e_type) == 0) {
      int64_t fr[2] = {EI64(&n, e, e_frac0), EI64(&n, e, e_frac1)};
      double sg[2] = {1.0, -1.0};
      for (int s = 0; s < 2; s++) {
        int64_t f = fr[s];
        int64_t ne = FI64(&n, f, f_nelements);
        const int64_t *els = FPTR(&n, f, f_elements);
        for (int64_t k = 0; k < ne; k++) {
          int64_t ee = els[k];
          if (EI64(&n, ee, e_id) == EI64(&n, e, e_id) || !is_disch(EI64(&n, ee, e_type))) continue;
          rows[ptr] = j;
          cols[ptr] = id_to_pos[EI64(&n, ee, e_id)];
          data[ptr] = (sg[s] * discharge_term_(&n, ee, s == 0 ? zz0 : zz1, D, f)) / FF64(&n, f, f_t);
          ptr++;
        }
      }
      rows[ptr] = j;
      cols[ptr] = n_de + fr[0];
      data[ptr] = 1.0 / FF64(&n, fr[0], f_t);
      ptr++;
      rows[ptr] = j;
      cols[ptr] = n_de + fr[1];
      data[ptr] = -1.0 / FF64(&n, fr[1], f_t);
    } else {
      int64_t f = EI64(&n, e, e_frac0);
      int64_t ne = FI64(&n, f, f_nelements);
      const int64_t *els = FPTR(&n, f, f_elements);
      for (int64_t k = 0; k < ne; k++) {
        int64_t ee = els[k];
        if (EI64(&n, ee, e_id) == EI64(&n, e, e_id) || !is_disch(EI64(&n, ee, e_type))) continue;
        rows[ptr] = j;
        cols[ptr] = id_to_pos[EI64(&n, ee, e_id)];
        data[ptr] = discharge_term_(&n, ee, zz0, D, f);
        ptr++;
      }
      rows[ptr] = j;
      cols[ptr] = n_de + f;
      data[ptr] = 1.0;
    }
  }
  for (int64_t f = 0; f < nf; f++) {
    int64_t ptr = row_offsets[n_de + f];
    int64_t ne = FI64(&n, f, f_nelements);
    const int64_t *els = FPTR(&n, f, f_elements);
    for (int64_t k = 0; k < ne; k++) {
      int64_t e = els[k];
      int64_t t = EI64(&n, e, e_type);
      if (!is_disch(t)) continue;
      rows[ptr] = n_de + f;
      cols[ptr] = id_to_pos[EI64(&n, e, e_id)];
      data[ptr] = (t != 0 || EI64(&n, e, e_frac0) == FI64(&n, f, f_id)) ? 1.0 : -1.0;
      ptr++;
    }
  }
}

/* hpc_solve.py:667-717 + 779-829: zero q and constants, then the head vector */
void oracle_head_vector(const AndfnLayout *L, char *E, int64_t ne, char *F, int64_t nf, const int64_t *de_ids,
                        int64_t n_de, const double *z0, const double *z1, int64_t D, double *head) {
  Net n = {L, E, F, ne, nf};
  for (int64_t i = 0; i < ne; i++) EF64(&n, i, e_q) = 0.0;
  for (int64_t f = 0; f < nf; f++) FF64(&n, f, f_constant) = 0.0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t j = 0; j < n_de; j++) {
    int64_t e = de_ids[j];
    int64_t f0 = EI64(&n, e, e_frac0);
    const cplx *zz0 = (const cplx *)(z0 + 2 * j * D);
    cplx om = C(0.0, 0.0);
    for (int64_t i = 0; i < D; i++) om = cadd(om, calc_omega(&n, f0, zz0[i], -1));
    om = cdiv(om, C((double)D, 0.0));
    int64_t t = EI64(&n, e, e_type);
    if (t == 0) {
      int64_t f1 = EI64(&n, e, e_frac1);
      const cplx *zz1 = (const cplx *)(z1 + 2 * j * D);
      cplx om1 = C(0.0, 0.0);
      for (int64_t i = 0; i < D; i++) om1 = cadd(om1, calc_omega(&n, f1, zz1[i], -1));
      om1 = cdiv(om1, C((double)D, 0.0));
      head[j] = om1.re / FF64(&n, f1, f_t) - om.re / FF64(&n, f0, f_t);
    } else if (t == 2 || t == 3) {
      head[j] = EF64(&n, e, e_phi) - om.re;
    }
  }
}

/* hpc_solve.py:721-761: scatter q of discharge elements and fracture constants */
void oracle_post_solve(const AndfnLayout *L, char *E, char *F, int64_t nf, const int64_t *de_ids, int64_t n_de,
                       const double *x) {
  Net n = {L, E, F, 0, nf};
  for (int64_t j = 0; j < n_de; j++) EF64(&n, de_ids[j], e_q) = x[j];
  for (int64_t f = 0; f < nf; f++) FF64(&n, f, f_constant) = x[n_de + f];
}

/* hpc_solve.py:311-390 element_solver: Jacobi sweep then damped blend */
int oracle_element_solver(void *p, const AndfnLayout *L, char *E, int64_t ne, char *F, int64_t nf, double damping) {
  OracleCtx *ctx = (OracleCtx *)p;
  Net n = {L, E, F, ne, nf};
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
  for (int64_t i = 0; i < ne; i++) {
    if (solve_element(&n, ctx, i)) bad = 1;
  }
  if (bad) return -1;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < ne; i++) blend(&n, ctx, i, damping);
  return 0;
}

/* hpc_solve.py:394-591 element_solver2: sweep, and for nit >= 2 the adaptive
 * ncoef growth (465-559) and a second damped blend (561-575). */
int oracle_element_solver2(void *p, const AndfnLayout *L, char *E, int64_t ne, char *F, int64_t nf, double max_error,
                           int64_t nit, double max_coef_ratio, int64_t max_coef, int64_t coef_increase,
                           double damping) {
  OracleCtx *ctx = (OracleCtx *)p;
  Net n = {L, E, F, ne, nf};
  if (oracle_element_solver(p, L, E, ne, F, nf, damping)) return -1;
  if (nit < 2) return 0;
  const int64_t ncc = 3;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
  for (int64_t i = 0; i < ne; i++) {
    Work *w = &ctx->w[i];
    w->set_zero = 0;
    int64_t type = EI64(&n, i, e_type);
    if (type == 2) continue;
    int64_t m = EI64(&n, i, e_ncoef);
    /* coefs = e.coef[:m] (already blended once) */
    double coef0 = 0.0, coef1 = 0.0;
    {
      /* np.mean(np.abs(coefs[1:ncc])) + 1e-30; np.max(np.abs(coefs[-ncc:])) */
      int64_t a0 = 1, a1 = ncc < m ? ncc : m;
      double s = 0.0;
      int64_t cntm = 0;
      for (int64_t k = a0; k < a1; k++) {
        s += cabs_(ecoef(&n, i, k));
        cntm++;
      }
      coef0 = (cntm > 0 ? s / cntm : NAN) + 1e-30;
      int64_t b0 = m - ncc < 0 ? 0 : m - ncc;
      coef1 = -INFINITY;
      for (int64_t k = b0; k < m; k++) {
        double v = cabs_(ecoef(&n, i, k));
        if (v > coef1 || v != v) coef1 = v;
        if (v != v) break;
      }
    }
    double ratio;
    if (coef0 == 0.0)
      ratio = 0.0;
    else
      ratio = coef1 / coef0 * 0;
    {
      double mx = -INFINITY;
      for (int64_t k = 1; k < 2 && k < m; k++) mx = cabs_(ecoef(&n, i, k));
      if (mx < max_error / 1e10) ratio = 0.0;
    }
    double err = EF64(&n, i, e_error), eo = EF64(&n, i, e_error_old), eo2 = EF64(&n, i, e_error_old2);
    if (err > eo && err > eo2 && err > max_error && nit > 5) {
      w->set_zero = 1;
      w->set_zero = 0;
      ratio = max_coef_ratio + 1.0;
    }
    {
      cplx s_last = C(0.0, 0.0), s_rest = C(0.0, 0.0);
      int64_t b0 = m - ncc < 0 ? 0 : m - ncc;
      for (int64_t k = b0; k < m; k++) s_last = cadd(s_last, ecoef(&n, i, k));
      for (int64_t k = 0; k < b0; k++) s_rest = cadd(s_rest, ecoef(&n, i, k));
      if (cabs_(cdiv(s_last, C(s_rest.re + 1e-30, s_rest.im + 0.0))) > max_coef_ratio && err > max_error)
        ratio = max_coef_ratio + 1.0;
    }
    int64_t cnt = 0;
    const int64_t max_cnt = 1;
    while (ratio > max_coef_ratio && EI64(&n, i, e_ncoef) < max_coef && cnt < max_cnt && nit > 1) {
      cnt++;
      EI64(&n, i, e_ncoef) = EI64(&n, i, e_ncoef) + coef_increase;
      EI64(&n, i, e_nint) = EI64(&n, i, e_ncoef) * 2;
      if (EI64(&n, i, e_ncoef) > ctx->M) {
        bad = 1;
        break;
      }
      int64_t nn = EI64(&n, i, e_nint);
      double *th = EPTR(&n, i, e_thetas);
      calc_thetas(nn, type, th);
      w->len_discharge_element = 0;
      fill_exp(nn, th, w->exp_m, -1);
      fill_exp(nn, th, w->exp_p, 1);
      if (solve_element(&n, ctx, i)) {
        bad = 1;
        break;
      }
      int64_t m2 = EI64(&n, i, e_ncoef);
      {
        int64_t a1 = ncc < m2 ? ncc : m2;
        double s = 0.0;
        int64_t cntm = 0;
        for (int64_t k = 1; k < a1; k++) {
          s += cabs_(w->coef[k]);
          cntm++;
        }
        coef0 = (cntm > 0 ? s / cntm : NAN) + 1e-30;
        int64_t b0 = m2 - ncc < 0 ? 0 : m2 - ncc;
        coef1 = -INFINITY;
        for (int64_t k = b0; k < m2; k++) {
          double v = cabs_(w->coef[k]);
          if (v > coef1 || v != v) coef1 = v;
          if (v != v) break;
        }
        ratio = coef1 / coef0;
        cplx s_last = C(0.0, 0.0), s_rest = C(0.0, 0.0);
        for (int64_t k = b0; k < m2; k++) s_last = cadd(s_last, w->coef[k]);
        for (int64_t k = 0; k < b0; k++) s_rest = cadd(s_rest, w->coef[k]);
        if (cabs_(cdiv(s_last, C(s_rest.re + 1e-30, s_rest.im + 0.0))) > max_coef_ratio)
          ratio = max_coef_ratio + 1.0;
      }
      if (cnt == max_cnt) {
        w->set_zero = 1;
        w->set_zero = 0;
      }
    }
  }
  if (bad) return -1;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < ne; i++) {
    if (ctx->w[i].set_zero) EF64(&n, i, e_error_old) = 1e30;
    blend(&n, ctx, i, damping);
  }
  return 0;
}

/* hpc_fracture.py:52-94 at arbitrary points (exclude = -1); out complex [npts] */
void oracle_eval_omega(const AndfnLayout *L, char *E, char *F, const int64_t *frac, const double *z, int64_t npts,
                       double *out) {
  Net n = {L, E, F, 0, 0};
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < npts; i++) {
    cplx om = calc_omega(&n, frac[i], C(z[2 * i], z[2 * i + 1]), -1);
    out[2 * i] = om.re;
    out[2 * i + 1] = om.im;
  }
}

/* hpc_fracture.py:205-231 calc_heads at arbitrary points: Re(Omega)/t */
void oracle_eval_heads(const AndfnLayout *L, char *E, char *F, const int64_t *frac, const double *z, int64_t npts,
                       double *out) {
  Net n = {L, E, F, 0, 0};
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < npts; i++) {
    cplx om = calc_omega(&n, frac[i], C(z[2 * i], z[2 * i + 1]), -1);
    out[i] = om.re / FF64(&n, frac[i], f_t);
  }
}

/* Collocation-point potentials of one element, excluding itself: used by the
 * tests to check the CUDA evaluation kernel in isolation.  side 0 = frac0 /
 * endpoints0, side 1 = frac1 / endpoints1.  out complex [nint]. */
void oracle_collocation_omega(void *p, const AndfnLayout *L, char *E, char *F, int64_t el, int side, double *out) {
  OracleCtx *ctx = (OracleCtx *)p;
  Net n = {L, E, F, 0, 0};
  Work *w = &ctx->w[el];
  int64_t type = EI64(&n, el, e_type), nn = EI64(&n, el, e_nint);
  int64_t f = side ? EI64(&n, el, e_frac1) : EI64(&n, el, e_frac0);
  int64_t off = side ? L->e_endpoints1 : L->e_endpoints0;
  for (int64_t ii = 0; ii < nn; ii++) {
    cplx z;
    if (type == 1 || type == 4)
      z = map_chi_to_z_circle(w->exp_p[ii], EF64(&n, el, e_radius), eptc(&n, el, L->e_center, 0));
    else
      z = map_chi_to_z_line(w->exp_p[ii], eptc(&n, el, off, 0), eptc(&n, el, off, 1));
    cplx om = calc_omega(&n, f, z, EI64(&n, el, e_id));
    out[2 * ii] = om.re;
    out[2 * ii + 1] = om.im;
  }
}
