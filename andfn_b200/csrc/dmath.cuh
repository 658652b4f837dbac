// Device-side complex arithmetic and conformal maps for the analytic elements.
//
// Two families of functions live here:
//  * fast forms used in the evaluation hot loop (FMA-based complex products,
//    one square root per line map, a reciprocal instead of a divide in every
//    Horner step).  They agree with the reference's arithmetic to rounding;
//  * reference-order forms (Smith division, sqrt(Z-1)*sqrt(Z+1)) used only
//    where the reference makes a discrete decision from the result (branch-cut
//    crossings, andfn/hpc/hpc_math_functions.py:301-403), so that the decision
//    is taken from the same formula.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace andfn {

struct cd {
  double re, im;
};

__host__ __device__ __forceinline__ cd mk(double re, double im) { return cd{re, im}; }
__host__ __device__ __forceinline__ cd operator+(cd a, cd b) { return mk(a.re + b.re, a.im + b.im); }
__host__ __device__ __forceinline__ cd operator-(cd a, cd b) { return mk(a.re - b.re, a.im - b.im); }
__host__ __device__ __forceinline__ cd operator*(cd a, cd b) {
  return mk(fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re));
}
__host__ __device__ __forceinline__ cd operator*(double s, cd a) { return mk(s * a.re, s * a.im); }
__host__ __device__ __forceinline__ double norm2(cd a) { return fma(a.re, a.re, a.im * a.im); }
__host__ __device__ __forceinline__ cd conjg(cd a) { return mk(a.re, -a.im); }
// r * w + c (Horner step), 4 FMAs
__host__ __device__ __forceinline__ cd fma_c(cd r, cd w, cd c) {
  return mk(fma(r.re, w.re, fma(-r.im, w.im, c.re)), fma(r.re, w.im, fma(r.im, w.re, c.im)));
}
__device__ __forceinline__ cd recip(cd a) {
  double s = 1.0 / norm2(a);
  return mk(a.re * s, -a.im * s);
}

// Principal square root (Algorithm 312 form, as numpy/numba compute it).
__host__ __device__ __forceinline__ cd csqrt_ref(cd z) {
  double a = z.re, b = z.im;
  if (a == 0.0 && b == 0.0) return mk(fabs(b), b);
  double h = hypot(a, b);
  if (a >= 0) {
    double t = sqrt((a + h) * 0.5);
    return mk(t, b / (2 * t));
  } else {
    double t = sqrt((-a + h) * 0.5);
    return mk(fabs(b) / (2 * t), copysign(t, b));
  }
}

// Smith's complex division (CPython _Py_c_quot), as the reference divides.
__host__ __device__ __forceinline__ cd cdiv_ref(cd a, cd b) {
  double br = b.re, bi = b.im;
  if (fabs(br) >= fabs(bi)) {
    if (br == 0.0) return mk(NAN, NAN);
    double ratio = bi / br;
    double denom = br + bi * ratio;
    return mk((a.re + a.im * ratio) / denom, (a.im - a.re * ratio) / denom);
  } else {
    double ratio = br / bi;
    double denom = br * ratio + bi;
    return mk((a.re * ratio + a.im) / denom, (a.im * ratio - a.re) / denom);
  }
}

// Reference-order line map (andfn/hpc/hpc_geometry_functions.py:12-31).
__host__ __device__ __forceinline__ cd map_z_line_to_chi_ref(cd z, cd a, cd b) {
  cd bz = cdiv_ref(mk(2.0 * z.re - a.re - b.re, 2.0 * z.im - a.im - b.im), b - a);
  cd s1 = csqrt_ref(mk(bz.re - 1.0, bz.im));
  cd s2 = csqrt_ref(mk(bz.re + 1.0, bz.im));
  cd p = mk(s1.re * s2.re - s1.im * s2.im, s1.re * s2.im + s1.im * s2.re);
  return bz + p;
}

// Exterior Joukowski inverse: chi = Z + sqrt(Z^2 - 1) on the branch with
// |chi| >= 1.  The reference's product sqrt(Z-1) sqrt(Z+1) is the analytic
// exterior branch with its cut on the segment [-1, 1]; (Z+s)(Z-s) = 1, so
// picking the root s with Re(conj(Z) s) >= 0 selects the same value off the
// segment with one square root.  On the segment both roots lie on |chi| = 1
// and give equal real parts for real coefficients.
__device__ __forceinline__ cd exterior_chi(cd Z) {
  cd w = mk(fma(Z.re, Z.re, -fma(Z.im, Z.im, 1.0)), 2.0 * Z.re * Z.im);
  double h = sqrt(norm2(w));
  double t = sqrt(0.5 * (fabs(w.re) + h));
  cd s;
  if (t == 0.0) {
    s = mk(0.0, 0.0);
  } else if (w.re >= 0) {
    s = mk(t, w.im / (2.0 * t));
  } else {
    s = mk(fabs(w.im) / (2.0 * t), copysign(t, w.im));
  }
  if (fma(Z.re, s.re, Z.im * s.im) < 0.0) s = mk(-s.re, -s.im);
  return Z + s;
}

}  // namespace andfn
