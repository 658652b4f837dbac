// Streamline (particle) tracking on a solved network: a group of TRACK_GROUP
// lanes per particle, which share the sum over the fracture's elements in every
// evaluation of w and otherwise run the same steps in lockstep.
//
// Follows the object layer of the reference, which is what DFN.streamline_tracking
// (andfn/dfn.py:2643-2722) runs on:
//  * the discharge vector w(z) of a fracture is Fracture.calc_w (andfn/fracture.py:453-478)
//    with the element methods of the object layer: intersections and constant-head
//    lines as in the consolidated solver, bounding circles with the minus sign and
//    the 1/R chain-rule factor and NaN beyond |z/R| > 1 + 1e-5 (bounding.py:49-108),
//    wells and impermeable circles NaN inside (well.py:129-153,
//    impermeable_object.py:131-156), impermeable lines (impermeable_object.py:205-224);
//  * a step is DFN.runge_kutta (andfn/dfn.py:2797-2846);
//  * exits are DFN.check_streamline_exit (andfn/dfn.py:2724-2741) with the crossing
//    tests of intersection.py:227-271, const_head.py:208-246 and well.py:162-200;
//  * at an intersection the particle moves to the other fracture by
//    DFN.get_exit_intersection (andfn/dfn.py:2743-2795).
//
// Every function is __host__ __device__ so that the same source runs in the
// kernel and, for tests, on the host.  Divisions use Smith's quotient and line
// maps the reference-order square roots (dmath.cuh), which is how the
// reference's compiled helpers compute them.
#pragma once
#include "dmath.cuh"

namespace andfn {

// Read-only view of a solved single network for tracking.
struct TrackView {
  int MC;                       // coefficient stride of coef
  const int *type, *frac0, *frac1, *ncoef;
  const cd *ep0, *ep1;          // [ne][2]
  const double *radius;         // element radius
  const cd *center;             // element center
  const double *q;              // element discharge
  const cd *coef;               // [ne][MC]
  const int *fptr, *felem;      // elements of each fracture, in record order
  const double *fgeo;           // [nf][TRACK_FGEO]: radius, center[3], x[3], y[3], normal[3]
  const double *aperture;       // [nf]
};
static constexpr int TRACK_FGEO = 13;
static constexpr int TRACK_GROUP = 8;  // lanes that trace one particle together
static constexpr double TRACK_PI = 3.141592653589793;

// Status of one particle.
enum TrackStatus { TRACK_DONE = 0, TRACK_TRUNCATED = 1 };

__host__ __device__ __forceinline__ double t_abs(cd a) { return hypot(a.re, a.im); }
__host__ __device__ __forceinline__ cd t_nan() { return mk(NAN, NAN); }
__host__ __device__ __forceinline__ cd t_scale(cd a, double s) { return mk(a.re * s, a.im * s); }
__host__ __device__ __forceinline__ cd t_mul(cd a, cd b) {
  return mk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}

// 1 / chi by Smith's quotient.
__host__ __device__ __forceinline__ cd t_recip(cd a) { return cdiv_ref(mk(1.0, 0.0), a); }

// d/dchi of sum_k s c_k chi^-k in the reference's Horner order
// (andfn/hpc/hpc_math_functions.py:76-100), each division by chi taken as a
// product with u = 1 / chi.
__host__ __device__ inline cd t_asym_d1(cd chi, const cd *c, int m, double s) {
  const cd u = t_recip(chi);
  cd res = mk(0.0, 0.0);
  for (int k = 0; k < m; k++) {
    const double n = (double)(m - 1 - k);
    res = t_mul(res - t_scale(c[m - 1 - k], s * n), u);
  }
  return res;
}

// d/dchi of sum_k c_k chi^k (andfn/hpc/hpc_math_functions.py:164-190); c1 is
// the record's slot 1, which the reference reads whatever ncoef is.
__host__ __device__ inline cd t_taylor_d1(cd chi, const cd *c, int m, cd c1) {
  cd res = mk(0.0, 0.0);
  for (int k = 0; k < m - 2; k++) {
    res = res + t_scale(c[m - 1 - k], (double)(m - 1 - k));
    res = t_mul(res, chi);
  }
  return res + c1;
}

// 2 chi^2 / (chi^2 - 1) * 2 / (b - a): dchi/dz of the line map.
__host__ __device__ __forceinline__ cd t_line_dchi(cd chi, cd a, cd b) {
  const cd c2 = t_mul(chi, chi);
  cd f = cdiv_ref(t_scale(c2, 2.0), mk(c2.re - 1.0, c2.im));
  return cdiv_ref(t_scale(f, 2.0), b - a);
}

// The object-layer w of element e seen from fracture f.
__host__ __device__ inline cd t_element_w(const TrackView &v, int f, int e, cd z) {
  const int ty = v.type[e];
  const int m = v.ncoef[e];
  const cd *c = v.coef + (size_t)e * v.MC;
  if (ty == 0 || ty == 3 || ty == 5) {
    const bool side1 = (ty == 0 && v.frac0[e] != f);
    const cd *ep = side1 ? v.ep1 + 2 * e : v.ep0 + 2 * e;
    const cd chi = map_z_line_to_chi_ref(z, ep[0], ep[1]);
    const double s = side1 ? -1.0 : 1.0;
    cd w = mk(0.0, 0.0) - t_asym_d1(chi, c, m, s);
    if (ty != 5) w = w - t_scale(cdiv_ref(mk(v.q[e], 0.0), t_scale(chi, 2 * TRACK_PI)), s);
    return t_mul(w, t_line_dchi(chi, ep[0], ep[1]));
  }
  const double r = v.radius[e];
  if (ty == 1) {
    cd chi = mk(z.re / r, z.im / r);
    if (t_abs(chi) > 1.0 + 1e-5) chi = t_nan();
    const cd c1 = v.MC > 1 ? c[1] : mk(0.0, 0.0);
    const cd w = mk(0.0, 0.0) - t_taylor_d1(chi, c, m, c1);
    return mk(w.re / r, w.im / r);
  }
  const cd d = z - v.center[e];
  const cd chi = mk(d.re / r, d.im / r);
  if (t_abs(chi) < 1.0 - 1e-10) return t_nan();
  cd w;
  if (ty == 2)
    w = cdiv_ref(mk(-v.q[e], 0.0), t_scale(chi, 2 * TRACK_PI));
  else
    w = mk(0.0, 0.0) - t_asym_d1(chi, c, m, 1.0);
  return mk(w.re / r, w.im / r);
}

// Fracture.calc_w: the sum over every element of fracture f in record order.
__host__ __device__ inline cd t_frac_w(const TrackView &v, int f, cd z) {
  cd w = mk(0.0, 0.0);
  for (int k = v.fptr[f]; k < v.fptr[f + 1]; k++) w = w + t_element_w(v, f, v.felem[k], z);
  return w;
}

// The share of lane `lane` of a group of G lanes: elements lane, lane + G, ...
__host__ __device__ inline cd t_frac_w_part(const TrackView &v, int f, cd z, int lane, int G) {
  cd w = mk(0.0, 0.0);
  for (int k = v.fptr[f] + lane; k < v.fptr[f + 1]; k += G) w = w + t_element_w(v, f, v.felem[k], z);
  return w;
}

// w of a fracture summed by a group of G lanes that trace one particle
// together: each lane sums its share, then a butterfly (lane l adds the value
// of lane l ^ o for o = G/2 ... 1) leaves the same total, bit for bit, in
// every lane (a + b == b + a), so all lanes take the same decisions.
#ifdef __CUDACC__
template <int G>
struct GroupW {
  TrackView v;
  int lane;
  unsigned mask;  // the G lanes of this group within the warp
  __device__ cd operator()(int f, cd z) const {
    cd w = t_frac_w_part(v, f, z, lane, G);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      const double re = __shfl_xor_sync(mask, w.re, o, G);
      const double im = __shfl_xor_sync(mask, w.im, o, G);
      w = w + mk(re, im);
    }
    return w;
  }
};
#endif

// The same sum on the host, lane by lane, in the butterfly's order.
template <int G>
struct HostGroupW {
  const TrackView *v;
  cd operator()(int f, cd z) const {
    cd p[G], q[G];
    for (int l = 0; l < G; l++) p[l] = t_frac_w_part(*v, f, z, l, G);
    for (int o = G / 2; o > 0; o >>= 1) {
      for (int l = 0; l < G; l++) q[l] = p[l] + p[l ^ o];
      for (int l = 0; l < G; l++) p[l] = q[l];
    }
    return p[0];
  }
};

__host__ __device__ __forceinline__ bool t_isnan(cd z) { return isnan(z.re) || isnan(z.im); }

// Unit step along conj(w) with up to max_it trapezoidal corrections; points
// beyond the fracture radius are pulled back inside (andfn/dfn.py:2797-2846).
// w0 is w at z0, which the caller has already evaluated for the velocity there.
template <class W>
__host__ __device__ inline cd t_runge_kutta(const TrackView &v, const W &wf, int f, cd z0, cd w0, double ds,
                                            bool backward) {
  const double R = v.fgeo[(size_t)f * TRACK_FGEO];
  if (backward) ds = -ds;
  if (isnan(w0.re)) return t_nan();
  const double a0 = t_abs(w0);
  cd z1 = z0 + t_scale(mk(w0.re / a0, -w0.im / a0), ds);
  double az = t_abs(z1);
  if (az > R) z1 = t_scale(z1, R / (az * (1 + 1e-5)));
  double dz = 1e99;
  int it = 0;
  while (dz > 1e-6 && it < 10) {
    const cd w1 = wf(f, z1);
    if (isnan(w1.re)) break;
    const cd sw = w0 + w1;
    const double as = t_abs(sw);
    cd z2 = z0 + t_scale(mk(sw.re / as, -sw.im / as), ds);
    az = t_abs(z2);
    if (az > R) z2 = t_scale(z2, R / (az * (1 + 1e-5)));
    dz = t_abs(z2 - z1);
    z1 = z2;
    it++;
  }
  return z1;
}

// andfn/geometry_functions.py:405-438; false when the lines are parallel.
__host__ __device__ inline bool t_line_line(cd z0, cd z1, cd z2, cd z3, cd *out) {
  const cd det = t_mul(conjg(z1) - conjg(z0), z3 - z2) - t_mul(z1 - z0, conjg(z3) - conjg(z2));
  if (det.re == 0.0 && det.im == 0.0) return false;
  const cd num = t_mul(t_mul(conjg(z1), z0) - t_mul(z1, conjg(z0)), z3 - z2) -
                 t_mul(z1 - z0, t_mul(conjg(z3), z2) - t_mul(z3, conjg(z2)));
  *out = cdiv_ref(num, det);
  return true;
}

// intersection.py:247-271, const_head.py:226-246 (atol 1e-12).
__host__ __device__ inline bool t_line_crossing(cd z0, cd z1, cd a, cd b, cd *out) {
  cd z;
  if (!t_line_line(z0, z1, a, b, &z)) return false;
  if (fabs(t_abs(z - z0) + t_abs(z1 - z) - t_abs(z0 - z1)) > 1e-12) return false;
  if (fabs(t_abs(z - a) + t_abs(z - b) - t_abs(a - b)) > 1e-12) return false;
  *out = z;
  return true;
}

// well.py:180-200 with andfn/geometry_functions.py:359-402 (atol 1e-10).
__host__ __device__ inline bool t_well_crossing(const TrackView &v, int e, cd z0, cd z1, cd *out) {
  const double r = v.radius[e];
  const cd c = v.center[e];
  const cd chi0 = mk((z0.re - c.re) / r, (z0.im - c.im) / r);
  const cd chi1 = mk((z1.re - c.re) / r, (z1.im - c.im) / r);
  cd chi2, chi3;
  const double dx = chi1.re - chi0.re, dy = chi1.im - chi0.im;
  if (dx == 0.0) {
    const double x = chi0.re;
    const double y1 = sqrt(1.0 - x * x);
    chi2 = mk(x, y1);
    chi3 = mk(x, -y1);
  } else {
    const double m = dy / dx;
    const double x0 = chi0.im - m * chi0.re;
    const double qa = 1 + m * m, qb = 2 * x0 * m, qc = x0 * x0 - 1.0;
    const double disc = qb * qb - 4 * qa * qc;
    if (disc < 0) return false;
    const double sq = sqrt(disc);
    const double x1 = (-qb + sq) / (2 * qa), x2 = (-qb - sq) / (2 * qa);
    chi2 = mk(x1, m * x1 + x0);
    chi3 = mk(x2, m * x2 + x0);
  }
  const double atol = 1e-10;
  const double d0 = fabs(t_abs(chi2 - chi0) + t_abs(chi2 - chi1) - t_abs(chi1 - chi0));
  const double d1 = fabs(t_abs(chi3 - chi0) + t_abs(chi3 - chi1) - t_abs(chi1 - chi0));
  if (d0 > atol && d1 > atol) return false;
  chi2 = t_scale(chi2, 1 + atol);
  chi3 = t_scale(chi3, 1 + atol);
  const cd za = t_scale(chi2, r) + c, zb = t_scale(chi3, r) + c;
  *out = (t_abs(za - z0) < t_abs(zb - z0)) ? za : zb;
  return true;
}

// The first discharge element of fracture f (record order) whose boundary the
// step z0 -> z1 crosses; -1 when there is none.
__host__ __device__ inline int t_check_exit(const TrackView &v, int f, cd z0, cd z1, cd *z3) {
  for (int k = v.fptr[f]; k < v.fptr[f + 1]; k++) {
    const int e = v.felem[k];
    const int ty = v.type[e];
    bool hit = false;
    if (ty == 0) {
      const cd *ep = (f == v.frac0[e]) ? v.ep0 + 2 * e : v.ep1 + 2 * e;
      hit = t_line_crossing(z0, z1, ep[0], ep[1], z3);
    } else if (ty == 3) {
      hit = t_line_crossing(z0, z1, v.ep0[2 * e], v.ep0[2 * e + 1], z3);
    } else if (ty == 2) {
      hit = t_well_crossing(v, e, z0, z1, z3);
    }
    if (hit) return e;
  }
  return -1;
}

__host__ __device__ __forceinline__ void t_to_3d(const TrackView &v, int f, cd z, double p[3]) {
  const double *g = v.fgeo + (size_t)f * TRACK_FGEO;
  for (int d = 0; d < 3; d++) p[d] = z.re * g[4 + d] + z.im * g[7 + d] + g[1 + d];
}

__host__ __device__ __forceinline__ cd t_to_2d(const TrackView &v, int f, const double p[3]) {
  const double *g = v.fgeo + (size_t)f * TRACK_FGEO;
  const double d0 = p[0] - g[1], d1 = p[1] - g[2], d2 = p[2] - g[3];
  return mk(d0 * g[4] + d1 * g[5] + d2 * g[6], d0 * g[7] + d1 * g[8] + d2 * g[9]);
}

__host__ __device__ __forceinline__ cd t_chi_to_z_line(cd chi, cd a, cd b) {
  const cd big_z = t_scale(chi + cdiv_ref(mk(1.0, 0.0), chi), 0.5);
  return t_scale(t_mul(big_z, b - a) + a + b, 0.5);
}

// The particle crosses intersection e from fracture f_old into f at p3: the two
// points just off the line on either side, the split of the flow by |w| there,
// and the side that the elevation selects (andfn/dfn.py:2743-2795).
template <class W>
__host__ __device__ inline void t_exit_intersection(const TrackView &v, const W &wf, const double p3[3], int e, int f,
                                                    int f_old, double *elevation, cd *z_next, cd *z_start) {
  const cd *ep = (f == v.frac0[e]) ? v.ep0 + 2 * e : v.ep1 + 2 * e;
  const cd z = t_to_2d(v, f, p3);
  const cd chi0 = map_z_line_to_chi_ref(z, ep[0], ep[1]);
  const cd chi1 = conjg(chi0);
  const double dchi = 1e-4;
  const cd za = t_chi_to_z_line(t_scale(chi0, 1 + dchi), ep[0], ep[1]);
  const cd zb = t_chi_to_z_line(t_scale(chi1, 1 + dchi), ep[0], ep[1]);
  const double a0 = t_abs(wf(f, za)), a1 = t_abs(wf(f, zb));
  double divide = a0 / (a0 + a1);
  double pa[3];
  t_to_3d(v, f, za, pa);
  const double *nrm = v.fgeo + (size_t)f_old * TRACK_FGEO + 10;
  const double nz0 = (pa[0] - p3[0]) * nrm[0] + (pa[1] - p3[1]) * nrm[1] + (pa[2] - p3[2]) * nrm[2];
  cd up, down;
  if (nz0 < 0) {
    up = zb;
    down = za;
  } else {
    up = za;
    down = zb;
    divide = 1 - divide;
  }
  double el = *elevation;
  if (el < divide) {
    *elevation = el / divide;
    *z_next = down;
  } else {
    *elevation = (el - divide) / (1 - divide);
    *z_next = up;
  }
  *z_start = za;
}

// One streamline (andfn/dfn.py:2643-2722).  Writes up to cap points into
// oz / ov / oseg / ofr (point, velocity, segment index, fracture); *n_out is
// the number of points, *elem_out the element the trace ended on (-1: none,
// the reference's False).  A segment whose first step is NaN is dropped, as in
// the reference.  TRACK_TRUNCATED when cap points did not suffice.  Only a
// `writer` stores; the other lanes of a group compute the same values.
template <class W>
__host__ __device__ inline int t_track(const TrackView &v, const W &wf, bool writer, int f, cd z0, double elevation,
                                       double ds, int max_length, bool backward, int cap, cd *oz, double *ov,
                                       int *oseg, int *ofr, int *n_out, int *elem_out) {
  int n = 0, nseg = 0, element = -1, status = TRACK_DONE;
  cd z_start = z0;
  for (;;) {
    const double ds_frac = v.fgeo[(size_t)f * TRACK_FGEO] * ds;
    const double ap = v.aperture[f];
    const int length = n;
    if (n >= cap) {
      status = TRACK_TRUNCATED;
      break;
    }
    int np = 1;
    cd w0 = wf(f, z0);
    if (writer) {
      oz[n] = z_start;
      ov[n] = t_abs(w0) / ap;
      oseg[n] = nseg;
      ofr[n] = f;
    }
    cd z1 = t_runge_kutta(v, wf, f, z0, w0, ds_frac, backward);
    if (t_isnan(z1)) break;
    cd z3;
    element = t_check_exit(v, f, z0, z1, &z3);
    bool stop = element >= 0;
    while (!stop) {
      if (n + np >= cap) {
        status = TRACK_TRUNCATED;
        break;
      }
      w0 = wf(f, z1);
      if (writer) {
        oz[n + np] = z1;
        ov[n + np] = t_abs(w0) / ap;
        oseg[n + np] = nseg;
        ofr[n + np] = f;
      }
      np++;
      z0 = z1;
      z1 = t_runge_kutta(v, wf, f, z0, w0, ds_frac, backward);
      if (t_isnan(z1)) {
        z3 = z0;
        break;
      }
      element = t_check_exit(v, f, z0, z1, &z3);
      stop = element >= 0;
      if (np > max_length - length) {
        z3 = z1;
        break;
      }
    }
    if (status == TRACK_DONE && n + np >= cap) status = TRACK_TRUNCATED;
    if (status != TRACK_DONE) {
      n += np;
      element = -1;
      break;
    }
    const cd w3 = wf(f, z3);
    if (writer) {
      oz[n + np] = z3;
      ov[n + np] = t_abs(w3) / ap;
      oseg[n + np] = nseg;
      ofr[n + np] = f;
    }
    n += np + 1;
    nseg++;
    if (element < 0 || v.type[element] != 0) break;
    double p3[3];
    t_to_3d(v, f, z3, p3);
    const int f_old = f;
    f = (f == v.frac0[element]) ? v.frac1[element] : v.frac0[element];
    t_exit_intersection(v, wf, p3, element, f, f_old, &elevation, &z0, &z_start);
  }
  *n_out = n;
  *elem_out = element;
  return status;
}

}  // namespace andfn
