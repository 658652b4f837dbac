// Network geometry on the device: disc-disc intersection segments and the
// connected clusters of a fracture set.
//
// Replaces the host steps that build a network before the solve:
//   * get_fracture_intersections (andfn/geometry_functions.py:623-713), which
//     applies fracture_intersection (:302-356; line_circle_intersection
//     :359-402 on both discs) to the pairs of discs a KD-tree query returns,
//     then shorten_line (:974-993) to each segment;
//   * the connected components of the intersection graph that
//     check_connectivity_hpc (:1121-1294) walks.
// The arithmetic restates andfn_b200/network.py (plane_disc_intersections,
// _line_circle, shorten, _candidate_pairs), which reproduces the reference's
// networks element for element, operation for operation in numpy's order:
// every product, sum, quotient and square root is rounded on its own
// (__dmul_rn / __dadd_rn / __dsub_rn / __ddiv_rn / __dsqrt_rn; no FMA
// contraction), so the device gives the same bits as the numpy restatement.
// All pairs i < k are tested: |c_i - c_k| <= r_i + r_k decides a candidate
// (the KD-tree of the host code is only a prefilter for the same test).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/andfn_b200.h"

namespace andfn_geo {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

struct V3 {
  double x, y, z;
};
struct Z {
  double re, im;
};

__device__ __forceinline__ V3 ld3(const double *p, int64_t i) { return V3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
// numpy.cross: (a1 b2 - a2 b1, a2 b0 - a0 b2, a0 b1 - a1 b0)
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return V3{sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)), sub(mul(a.x, b.y), mul(a.y, b.x))};
}
// network._dot: a0 b0 + a1 b1 + a2 b2, left to right
__device__ __forceinline__ double dot(V3 a, V3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return V3{sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)}; }
__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return V3{add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)}; }
// network._to2d: (dot(p - c, xv), dot(p - c, yv))
__device__ __forceinline__ Z to2d(V3 p, V3 c, V3 xv, V3 yv) {
  const V3 d = vsub(p, c);
  return Z{dot(d, xv), dot(d, yv)};
}
// network._to3d: re xv + im yv + c, per component
__device__ __forceinline__ V3 to3d(Z z, V3 c, V3 xv, V3 yv) {
  return V3{add(add(mul(z.re, xv.x), mul(z.im, yv.x)), c.x), add(add(mul(z.re, xv.y), mul(z.im, yv.y)), c.y),
            add(add(mul(z.re, xv.z), mul(z.im, yv.z)), c.z)};
}
// numpy.linalg.norm of a 3-vector: sqrt((x^2 + y^2) + z^2)
__device__ __forceinline__ double norm(V3 a) { return __dsqrt_rn(add(add(mul(a.x, a.x), mul(a.y, a.y)), mul(a.z, a.z))); }

// network._line_circle (line_circle_intersection, geometry_functions.py:359-402)
__device__ __forceinline__ bool line_circle(Z z0, Z z1, double R, Z &a, Z &b) {
  const double dx = sub(z1.re, z0.re), dy = sub(z1.im, z0.im);
  if (dx == 0.0) {  // vertical line: x = re z0
    const double x = z0.re;
    const double y1 = __dsqrt_rn(sub(mul(R, R), mul(x, x)));
    a = Z{x, y1};
    b = Z{x, -y1};
    return true;
  }
  const double m = dvd(dy, dx);
  const double x0 = sub(z0.im, mul(m, z0.re));
  const double A = add(1.0, mul(m, m));
  const double B = mul(mul(2.0, x0), m);
  const double C = sub(mul(x0, x0), mul(R, R));
  const double disc = sub(mul(B, B), mul(mul(4.0, A), C));
  const double sd = __dsqrt_rn(disc < 0.0 ? 0.0 : disc);
  const double x1 = dvd(add(-B, sd), mul(2.0, A));
  const double x2 = dvd(sub(-B, sd), mul(2.0, A));
  a = Z{x1, add(mul(m, x1), x0)};
  b = Z{x2, add(mul(m, x2), x0)};
  return disc >= 0.0;
}

// network.shorten (shorten_line, geometry_functions.py:974-993): c = (a + b) / 2,
// c + (a - c) se, c + (b - c) se
__device__ __forceinline__ void shorten(Z &a, Z &b, double se) {
  const Z c{dvd(add(a.re, b.re), 2.0), dvd(add(a.im, b.im), 2.0)};
  a = Z{add(c.re, mul(sub(a.re, c.re), se)), add(c.im, mul(sub(a.im, c.im), se))};
  b = Z{add(c.re, mul(sub(b.re, c.re), se)), add(c.im, mul(sub(b.im, c.im), se))};
}

// One thread per pair (i, k), i = blockIdx.y < k.  Valid segments are
// appended (atomic slot) with their endpoints in both discs' frames, shortened.
__global__ void intersections_kernel(int nf, const double *__restrict__ ctr, const double *__restrict__ nrm,
                                     const double *__restrict__ xvec, const double *__restrict__ yvec,
                                     const double *__restrict__ rad, double se, long long cap,
                                     unsigned long long *count, int2 *pairs, double *ep0, double *ep1) {
  const int i = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k <= i || k >= nf) return;
  const V3 c0 = ld3(ctr, i), c1 = ld3(ctr, k);
  const double R0 = rad[i], R1 = rad[k];
  // candidate: |c_i - c_k| <= r_i + r_k (network._candidate_pairs)
  if (!(norm(vsub(c0, c1)) <= add(R0, R1))) return;
  const V3 n0 = ld3(nrm, i), n1 = ld3(nrm, k);
  const V3 x0v = ld3(xvec, i), y0v = ld3(yvec, i), x1v = ld3(xvec, k), y1v = ld3(yvec, k);
  // fracture_intersection (network.plane_disc_intersections)
  const V3 d = cross(n0, n1);
  const double dn2 = dot(d, d);
  if (!(dn2 >= 1e-14)) return;
  const double cc0 = dot(n0, c0), cc1 = dot(n1, c1);
  const V3 a1 = cross(n1, d), b1 = cross(d, n0);
  const V3 p0{dvd(add(mul(cc0, a1.x), mul(cc1, b1.x)), dn2), dvd(add(mul(cc0, a1.y), mul(cc1, b1.y)), dn2),
              dvd(add(mul(cc0, a1.z), mul(cc1, b1.z)), dn2)};
  const V3 p1 = vadd(p0, d);
  Z a0, b0, a1z, b1z;
  const bool ok0 = line_circle(to2d(p0, c0, x0v, y0v), to2d(p1, c0, x0v, y0v), R0, a0, b0);
  const bool ok1 = line_circle(to2d(p0, c1, x1v, y1v), to2d(p1, c1, x1v, y1v), R1, a1z, b1z);
  if (!(ok0 && ok1)) return;
  const V3 cand[4] = {to3d(a0, c0, x0v, y0v), to3d(b0, c0, x0v, y0v), to3d(a1z, c1, x1v, y1v), to3d(b1z, c1, x1v, y1v)};
  int sel[2] = {-1, -1}, nin = 0;
  for (int j = 0; j < 4; j++) {
    const bool in0 = norm(vsub(cand[j], c0)) <= add(R0, 1e-8);
    const bool in1 = norm(vsub(cand[j], c1)) <= add(R1, 1e-8);
    if (in0 && in1) {
      if (nin < 2) sel[nin] = j;
      nin++;
    }
  }
  if (nin != 2) return;
  Z e00 = to2d(cand[sel[0]], c0, x0v, y0v), e01 = to2d(cand[sel[1]], c0, x0v, y0v);
  Z e10 = to2d(cand[sel[0]], c1, x1v, y1v), e11 = to2d(cand[sel[1]], c1, x1v, y1v);
  shorten(e00, e01, se);
  shorten(e10, e11, se);
  const unsigned long long slot = atomicAdd(count, 1ULL);
  if ((long long)slot >= cap) return;  // counted; the caller retries with room for all
  pairs[slot] = make_int2(i, k);
  double *o0 = ep0 + 4 * slot, *o1 = ep1 + 4 * slot;
  o0[0] = e00.re;
  o0[1] = e00.im;
  o0[2] = e01.re;
  o0[3] = e01.im;
  o1[0] = e10.re;
  o1[1] = e10.im;
  o1[2] = e11.re;
  o1[3] = e11.im;
}

// Connected clusters of the intersection graph: every edge hooks the larger
// of its two roots under the smaller (atomicMin), then every node jumps to
// its root; repeated until an edge pass changes nothing.  Parent values only
// decrease, so the loop ends; each root ends as its cluster's smallest index.
__device__ __forceinline__ int find_root(const int *parent, int x, int nf) {
  for (int s = 0; s < nf && parent[x] != x; s++) x = parent[x];
  return x;
}
__global__ void hook_kernel(int nf, const int2 *__restrict__ pairs, int np, int *parent, int *changed) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= np) return;
  const int a = find_root(parent, pairs[e].x, nf), b = find_root(parent, pairs[e].y, nf);
  if (a == b) return;
  atomicMin(&parent[max(a, b)], min(a, b));
  *changed = 1;
}
__global__ void jump_kernel(int nf, int *parent) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < nf) parent[f] = find_root(parent, f, nf);
}

}  // namespace andfn_geo

namespace {
thread_local std::string g_geo_error;
}

#define GEO_CK(call)                                                                   \
  do {                                                                                 \
    cudaError_t _e = (call);                                                           \
    if (_e != cudaSuccess) {                                                           \
      g_geo_error = std::string(#call) + ": " + cudaGetErrorString(_e);                \
      rc = ANDFN_CUDA_ERROR;                                                           \
      goto done;                                                                       \
    }                                                                                  \
  } while (0)

extern "C" const char *andfn_b200_geometry_last_error(void) { return g_geo_error.c_str(); }

extern "C" int andfn_b200_disc_intersections(int32_t device, int64_t nf, const double *centers,
                                             const double *normals, const double *xvec, const double *yvec,
                                             const double *radii, double se_factor, int64_t cap,
                                             int64_t *out_pairs, double *out_ep0, double *out_ep1,
                                             int64_t *out_n) {
  using namespace andfn_geo;
  if (nf < 0 || nf > 60000 || cap < 0 || !out_n || (nf > 0 && (!centers || !normals || !xvec || !yvec || !radii)) ||
      (cap > 0 && (!out_pairs || !out_ep0 || !out_ep1))) {
    g_geo_error = "disc_intersections: bad sizes or pointers (at most 60,000 discs)";
    return ANDFN_BAD_INPUT;
  }
  *out_n = 0;
  if (nf < 2) return ANDFN_OK;
  int rc = ANDFN_OK;
  double *d_in = nullptr, *d_ep0 = nullptr, *d_ep1 = nullptr;
  int2 *d_pairs = nullptr;
  unsigned long long *d_count = nullptr;
  unsigned long long count = 0;
  const size_t n3 = 3 * (size_t)nf;
  const long long dcap = std::max<long long>(1, cap);
  if (device >= 0) GEO_CK(cudaSetDevice(device));
  GEO_CK(cudaMalloc(&d_in, sizeof(double) * (4 * n3 + nf)));
  GEO_CK(cudaMalloc(&d_pairs, sizeof(int2) * dcap));
  GEO_CK(cudaMalloc(&d_ep0, sizeof(double) * 4 * dcap));
  GEO_CK(cudaMalloc(&d_ep1, sizeof(double) * 4 * dcap));
  GEO_CK(cudaMalloc(&d_count, sizeof(unsigned long long)));
  GEO_CK(cudaMemcpy(d_in, centers, sizeof(double) * n3, cudaMemcpyHostToDevice));
  GEO_CK(cudaMemcpy(d_in + n3, normals, sizeof(double) * n3, cudaMemcpyHostToDevice));
  GEO_CK(cudaMemcpy(d_in + 2 * n3, xvec, sizeof(double) * n3, cudaMemcpyHostToDevice));
  GEO_CK(cudaMemcpy(d_in + 3 * n3, yvec, sizeof(double) * n3, cudaMemcpyHostToDevice));
  GEO_CK(cudaMemcpy(d_in + 4 * n3, radii, sizeof(double) * nf, cudaMemcpyHostToDevice));
  GEO_CK(cudaMemset(d_count, 0, sizeof(unsigned long long)));
  {
    const dim3 grid((unsigned)((nf + 255) / 256), (unsigned)nf);
    intersections_kernel<<<grid, 256>>>((int)nf, d_in, d_in + n3, d_in + 2 * n3, d_in + 3 * n3, d_in + 4 * n3,
                                        se_factor, dcap, d_count, d_pairs, d_ep0, d_ep1);
    GEO_CK(cudaGetLastError());
  }
  GEO_CK(cudaMemcpy(&count, d_count, sizeof(count), cudaMemcpyDeviceToHost));
  *out_n = (int64_t)count;
  if ((long long)count > cap) {
    g_geo_error = "disc_intersections: " + std::to_string(count) + " segments, room for " + std::to_string(cap);
    rc = ANDFN_BAD_INPUT;
    goto done;
  }
  if (count > 0) {
    // the reference's order: pairs (i, k) sorted by i, then k
    std::vector<int2> pr(count);
    std::vector<double> e0(4 * count), e1(4 * count);
    GEO_CK(cudaMemcpy(pr.data(), d_pairs, sizeof(int2) * count, cudaMemcpyDeviceToHost));
    GEO_CK(cudaMemcpy(e0.data(), d_ep0, sizeof(double) * 4 * count, cudaMemcpyDeviceToHost));
    GEO_CK(cudaMemcpy(e1.data(), d_ep1, sizeof(double) * 4 * count, cudaMemcpyDeviceToHost));
    std::vector<size_t> ord(count);
    std::iota(ord.begin(), ord.end(), size_t(0));
    std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
      return pr[a].x != pr[b].x ? pr[a].x < pr[b].x : pr[a].y < pr[b].y;
    });
    for (size_t j = 0; j < count; j++) {
      const size_t o = ord[j];
      out_pairs[2 * j] = pr[o].x;
      out_pairs[2 * j + 1] = pr[o].y;
      for (int q = 0; q < 4; q++) {
        out_ep0[4 * j + q] = e0[4 * o + q];
        out_ep1[4 * j + q] = e1[4 * o + q];
      }
    }
  }
done:
  cudaFree(d_in);
  cudaFree(d_pairs);
  cudaFree(d_ep0);
  cudaFree(d_ep1);
  cudaFree(d_count);
  return rc;
}

extern "C" int andfn_b200_clusters(int32_t device, int64_t nf, int64_t npairs, const int64_t *pairs, int64_t *out_root) {
  using namespace andfn_geo;
  if (nf < 0 || nf > (1LL << 30) || npairs < 0 || npairs > (1LL << 30) || !out_root || (npairs > 0 && !pairs)) {
    g_geo_error = "clusters: bad sizes or pointers";
    return ANDFN_BAD_INPUT;
  }
  for (int64_t e = 0; e < npairs; e++)
    if (pairs[2 * e] < 0 || pairs[2 * e] >= nf || pairs[2 * e + 1] < 0 || pairs[2 * e + 1] >= nf) {
      g_geo_error = "clusters: a pair names a fracture out of range";
      return ANDFN_BAD_INPUT;
    }
  if (nf == 0) return ANDFN_OK;
  int rc = ANDFN_OK;
  int *d_parent = nullptr, *d_changed = nullptr;
  int2 *d_pairs = nullptr;
  std::vector<int> parent(nf), host_changed(1);
  std::vector<int2> pr(std::max<int64_t>(1, npairs));
  for (int64_t f = 0; f < nf; f++) parent[f] = (int)f;
  for (int64_t e = 0; e < npairs; e++) pr[e] = make_int2((int)pairs[2 * e], (int)pairs[2 * e + 1]);
  if (device >= 0) GEO_CK(cudaSetDevice(device));
  GEO_CK(cudaMalloc(&d_parent, sizeof(int) * nf));
  GEO_CK(cudaMalloc(&d_pairs, sizeof(int2) * pr.size()));
  GEO_CK(cudaMalloc(&d_changed, sizeof(int)));
  GEO_CK(cudaMemcpy(d_parent, parent.data(), sizeof(int) * nf, cudaMemcpyHostToDevice));
  GEO_CK(cudaMemcpy(d_pairs, pr.data(), sizeof(int2) * pr.size(), cudaMemcpyHostToDevice));
  for (int64_t round = 0; round <= nf; round++) {  // every productive round lowers some parent
    GEO_CK(cudaMemset(d_changed, 0, sizeof(int)));
    if (npairs > 0) {
      hook_kernel<<<(unsigned)((npairs + 255) / 256), 256>>>((int)nf, d_pairs, (int)npairs, d_parent, d_changed);
      GEO_CK(cudaGetLastError());
    }
    jump_kernel<<<(unsigned)((nf + 255) / 256), 256>>>((int)nf, d_parent);
    GEO_CK(cudaGetLastError());
    GEO_CK(cudaMemcpy(host_changed.data(), d_changed, sizeof(int), cudaMemcpyDeviceToHost));
    if (!host_changed[0]) break;
  }
  GEO_CK(cudaMemcpy(parent.data(), d_parent, sizeof(int) * nf, cudaMemcpyDeviceToHost));
  for (int64_t f = 0; f < nf; f++) out_root[f] = parent[f];
done:
  cudaFree(d_parent);
  cudaFree(d_pairs);
  cudaFree(d_changed);
  return rc;
}
