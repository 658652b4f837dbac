// Runs the streamline tracker of andfn_b200/csrc/track.cuh -- the very
// functions that track_kernel runs on the GPU -- on the host, so that the CPU
// tests can compare it with the oracle without a GPU.  Test infrastructure only.
#include "track.cuh"

using namespace andfn;

namespace {
TrackView view(int MC, const int *type, const int *frac0, const int *frac1, const int *ncoef, const double *ep0,
               const double *ep1, const double *radius, const double *center, const double *q, const double *coef,
               const int *fptr, const int *felem, const double *fgeo, const double *aperture) {
  TrackView v;
  v.MC = MC;
  v.type = type;
  v.frac0 = frac0;
  v.frac1 = frac1;
  v.ncoef = ncoef;
  v.ep0 = reinterpret_cast<const cd *>(ep0);
  v.ep1 = reinterpret_cast<const cd *>(ep1);
  v.radius = radius;
  v.center = reinterpret_cast<const cd *>(center);
  v.q = q;
  v.coef = reinterpret_cast<const cd *>(coef);
  v.fptr = fptr;
  v.felem = felem;
  v.fgeo = fgeo;
  v.aperture = aperture;
  return v;
}
}  // namespace

extern "C" void w_object_host(int MC, const int *type, const int *frac0, const int *frac1, const int *ncoef,
                              const double *ep0, const double *ep1, const double *radius, const double *center,
                              const double *q, const double *coef, const int *fptr, const int *felem,
                              const double *fgeo, const double *aperture, int npts, const int *frac, const double *z,
                              double *out) {
  const TrackView v = view(MC, type, frac0, frac1, ncoef, ep0, ep1, radius, center, q, coef, fptr, felem, fgeo,
                           aperture);
  for (int i = 0; i < npts; i++) {
    const cd w = t_frac_w(v, frac[i], mk(z[2 * i], z[2 * i + 1]));
    out[2 * i] = w.re;
    out[2 * i + 1] = w.im;
  }
}

extern "C" void track_host(int MC, const int *type, const int *frac0, const int *frac1, const int *ncoef,
                           const double *ep0, const double *ep1, const double *radius, const double *center,
                           const double *q, const double *coef, const int *fptr, const int *felem, const double *fgeo,
                           const double *aperture, int npart, const int *pf, const double *pz, const double *pe,
                           double ds, int max_length, int backward, int cap, double *oz, double *ov, int *oseg,
                           int *ofr, int *on, int *oelem, int *ostat) {
  const TrackView v = view(MC, type, frac0, frac1, ncoef, ep0, ep1, radius, center, q, coef, fptr, felem, fgeo,
                           aperture);
  for (int i = 0; i < npart; i++) {
    const size_t b = (size_t)i * (size_t)cap;
    int n = 0, el = -1;
    ostat[i] = t_track(v, HostGroupW<TRACK_GROUP>{&v}, true, pf[i], mk(pz[2 * i], pz[2 * i + 1]), pe[i], ds,
                       max_length, backward != 0, cap, reinterpret_cast<cd *>(oz) + b, ov + b, oseg + b, ofr + b, &n,
                       &el);
    on[i] = n;
    oelem[i] = el;
  }
}
