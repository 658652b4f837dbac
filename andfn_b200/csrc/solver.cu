// B200-native analytic-element DFN solve: kernels, host orchestration, C ABI.
//
// Replaces andfn.hpc.hpc_solve.solve (andfn/hpc/hpc_solve.py:55-257).  One
// outer iteration of the reference is
//   (1) head vector from the series part of every fracture potential at the
//       discharge elements' D points (build_head_matrix, hpc_solve.py:779-829),
//   (2) x = A^-1 b with the factorised discharge system (hpc_solve.py:651),
//       scatter q and fracture constants (post_matrix_solve, :721-761),
//   (3) a damped Jacobi sweep: every element re-fits its coefficients from the
//       potential of all *other* elements of its fracture(s) at its nint
//       collocation points (element_solver, :311-390, element_solver2
//       :394-591),
//   (4) max-reductions of the element errors and the convergence rule
//       (:196-239).
// Here (1) and (3) are one evaluation kernel (eval_kernel) in two modes,
// (2) is a single-CTA dependency-driven triangular solve (trisolve_kernel),
// the per-element fit is update_kernel and (4) is reduce_kernel.  Every kernel
// reads a device status word first and returns once the loop is finished, so
// iterations are launched in batches (CUDA graphs) without a host round trip
// per iteration.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/andfn_b200.h"
#include "dmath.cuh"
#include "sparse_lu.h"
#include "track.cuh"

namespace andfn {

static constexpr double PI = 3.141592653589793115997963468544185161590576171875;
static constexpr int EVAL_THREADS = 128;
static constexpr int HV_THREADS = 128;  // head_vector_kernel: one CTA per system row
static constexpr int UPDATE_WARPS = 4;
static constexpr int SOLVE_THREADS = 512;
// Discharge solves through the explicit inverse X take one refinement step
// in every iteration: x0 = X b alone carries errors of a few 1e-9 of the
// potential scale in the fracture constants of an ill-conditioned system
// (condition ~6e12 on the 2,118-fracture network), which show in the
// iterates of the first iterations; x0 + X (b - A x0) is accurate to
// round-off, so every iterate follows the reference's to 1e-13 or better.
static constexpr int ITER_BATCH = 8;  // iterations per graph launch (one host status read each)

enum GroupKind { KIND_PHI = 0, KIND_PSI = 1 };
// kernel classes of one outer iteration, in launch order
enum KClass { K_RHS = 0, K_TRISOLVE = 1, K_SWEEP = 2, K_UPDATE = 3, K_REDUCE = 4, KCLASSES = 5 };

// Target points of one element side (sweep) or one discharge element side (RHS).
struct Group {
  int elem, frac, side, npts;
  int out;   // offset into the value buffer
  int kind;  // KIND_PHI: real part (+ fracture constant); KIND_PSI: imaginary part
  int pad0, pad1;
};
struct Item {
  int frac, p0, p1, pad;
};
// A source element as seen from one fracture, staged in shared memory.
struct Src {
  int id, type, m, pad;
  cd p0, p1;  // line: Z = p0 * z + p1;  circle: p0 = center, p1.re = 1/r
  double qk;  // sign * q / (2 pi)
  double pad2;
};

struct SolveState {
  int nit, cnt_error, done, status;
  int worst, abort_flag, nonfinite, solve_q;
  double error_q, error, error_coef, pad;
  double max_error, damping;
  int max_it, fused_blend2;
  // explicit-inverse solves: 1 when the refinement step is applied (set at
  // the start of a run)
  int refine, n_refined;  // n_refined: solves that took the refinement step
  // SM clock cycles spent in the phases of trisolve_kernel, summed over
  // launches (thread 0's view): gather, L sparse, L coupling, L dense,
  // U dense, U coupling, U sparse, scatter
  long long tri_cycles[8];
};

struct TriDesc;

// Device view of one network.
struct Net {
  int ne, nf, n_de, N, MC, D;
  // elements
  const int *type, *frac0, *frac1;
  int *ncoef, *nint;
  const cd *ep0, *ep1;  // [ne][2]
  const double *radius, *phi;
  const cd *center;
  double *q;
  cd *coef, *wcoef;  // [ne][MC]
  double *err, *err_old, *err_old2, *err_coef;
  double *dpsi_corr;  // [ne][2*MC]
  // fractures
  const double *t;
  double *constant;
  const int *fptr, *felem;
  // discharge system
  const int *de_ids;
  cd *zint0, *zint1;  // [n_de][D]
  // branch cuts of psi elements: [ne][cut_cap]
  int cut_cap;
  int *cut_n, *cut_pos, *cut_elem, *cut_sign;
  // factors
  const int *pinv, *qcol, *l_ptr, *l_col, *u_ptr, *u_col;
  const double *l_val, *u_val, *u_inv;
  double *disc;  // current discharges [N]
  double *work;  // [N] scratch (solve in global memory when N is large)
  double *bvec;  // [N] head vector of the current iteration
  int *ready;    // [N]
  // Several independent networks (realizations) can share one launch: every
  // element, fracture and discharge-system row knows its realization, each
  // realization has its own loop state and its own factorised system.
  int R;
  SolveState *st;            // [R]
  const int *real_elem;      // [ne]
  const int *real_frac;      // [nf]
  const int *real_row;       // [N]
  const int *eoff;           // [R + 1] element range of each realization
  const int *row_de;         // [N] discharge-element index of a row, -1 for continuity rows
  const int *row_frac;       // [N] fracture of a continuity row, -1 otherwise
  int *ndone;                // realizations whose loop has finished
  const struct TriDesc *tri; // [R]
  // known part of the head vector [N] (wells with a prescribed discharge), or null
  const double *bknown;
  // DFT bases of the Cauchy-integral fits: element e's basis starts at
  // dft_tab + dft_off[e], entry (k, j) at k * MC + j = exp(-i theta_k)^j
  const cd *dft_tab;
  const int *dft_off;
};

// ------------------------------------------------------------------------
// small device helpers
// ------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ cd warp_sum(cd v) { return mk(warp_sum(v.re), warp_sum(v.im)); }

__device__ __forceinline__ void theta_of(int type, int n, int k, double &theta) {
  // hpc_math_functions.py:674-699 calc_thetas
  double del = PI / n;
  double start = del / 2;
  if (type == 1) {
    del = 2 * PI / n;
    start = 0.0;
  }
  theta = start + k * del;
}

// Collocation point k of element e on side s (hpc_math_functions.py:279-284,
// 491-495, 581-585: z = map_chi_to_z(exp(i theta_k))).
__device__ __forceinline__ cd sweep_point(const Net &net, int e, int side, int k) {
  int type = net.type[e];
  int n = net.nint[e];
  double th;
  theta_of(type, n, k, th);
  double s, c;
  sincos(th, &s, &c);
  cd chi = mk(c, s);
  if (type == 1 || type == 4) {
    double r = net.radius[e];
    cd ctr = net.center[e];
    return mk(chi.re * r - chi.im * 0.0 + ctr.re, chi.re * 0.0 + chi.im * r + ctr.im);
  }
  const cd *ep = side ? net.ep1 + 2 * e : net.ep0 + 2 * e;
  cd a = ep[0], b = ep[1];
  cd inv = cdiv_ref(mk(1.0, 0.0), chi);
  cd bz = 0.5 * (chi + inv);
  cd d = b - a;
  cd p = mk(bz.re * d.re - bz.im * d.im, bz.re * d.im + bz.im * d.re);
  return 0.5 * (p + a + b);
}

// ------------------------------------------------------------------------
// Evaluation kernel: Omega_f(z) over the elements of one fracture.
// RHS mode: series part only (q = C = 0 as after pre_matrix_solve), every
// element included (build_head_matrix).  Sweep mode: full potential without
// the target element itself (calc_omega(..., exclude=e)).
// ------------------------------------------------------------------------
template <bool RHS>
__global__ void __launch_bounds__(EVAL_THREADS) eval_kernel(Net net, const Item *__restrict__ items,
                                                              const int2 *__restrict__ pts,
                                                              const Group *__restrict__ groups,
                                                              double *__restrict__ out, int chunk) {
  const Item it = items[blockIdx.x];
  const SolveState *st = net.st + net.real_frac[it.frac];
  if (st->done) return;
  if (RHS && !st->solve_q) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Src *src = reinterpret_cast<Src *>(smem_raw);
  cd *scoef = reinterpret_cast<cd *>(smem_raw + sizeof(Src) * chunk);
  const int MC = net.MC;

  const int p = it.p0 + threadIdx.x;
  const bool active = p < it.p1;
  cd z = mk(0.0, 0.0);
  int exclude = -1, kind = KIND_PHI;
  int gout = 0;
  if (active) {
    int2 gk = pts[p];
    const Group g = groups[gk.x];
    gout = g.out + gk.y;
    if (RHS) {
      z = (g.side ? net.zint1 : net.zint0)[(size_t)g.elem * net.D + gk.y];
    } else {
      exclude = g.elem;
      kind = g.kind;
      z = sweep_point(net, g.elem, g.side, gk.y);
    }
  }
  const int f = it.frac;
  const int e0 = net.fptr[f], e1 = net.fptr[f + 1];
  double acc_re = 0.0, acc_im = 0.0;
  for (int base = e0; base < e1; base += chunk) {
    const int cnt = min(chunk, e1 - base);
    __syncthreads();
    for (int s = threadIdx.x; s < cnt; s += blockDim.x) {
      const int el = net.felem[base + s];
      Src h;
      h.id = el;
      h.type = net.type[el];
      h.m = net.ncoef[el];
      h.pad = 0;
      const int side = (h.type == 0 && net.frac0[el] != f) ? 1 : 0;
      const double sg = side ? -1.0 : 1.0;
      h.qk = RHS ? 0.0 : sg * net.q[el] / (2 * PI);
      h.pad2 = 0.0;
      if (h.type == 0 || h.type == 3 || h.type == 5) {
        const cd *ep = side ? net.ep1 + 2 * el : net.ep0 + 2 * el;
        cd a = ep[0], b = ep[1];
        cd inv = recip(b - a);
        h.p0 = 2.0 * inv;
        cd ab = a + b;
        h.p1 = mk(-(ab.re * inv.re - ab.im * inv.im), -(ab.re * inv.im + ab.im * inv.re));
      } else {
        h.p0 = (h.type == 1) ? mk(0.0, 0.0) : net.center[el];
        h.p1 = mk(1.0 / net.radius[el], 0.0);
      }
      src[s] = h;
    }
    for (int idx = threadIdx.x; idx < cnt * MC; idx += blockDim.x) {
      const int s = idx / MC, k = idx - s * MC;
      const int el = net.felem[base + s];
      const int m = net.ncoef[el];
      const int type = net.type[el];
      const bool neg = (type == 0 && net.frac0[el] != f);
      cd c = (k < m) ? net.coef[(size_t)el * MC + k] : mk(0.0, 0.0);
      if (neg) c = mk(-c.re, -c.im);
      scoef[idx] = c;
    }
    __syncthreads();
    if (active) {
      for (int s = 0; s < cnt; s++) {
        const Src &h = src[s];
        if (h.id == exclude) continue;
        const cd *c = scoef + s * MC;
        const int m = h.m;
        if (h.type == 0 || h.type == 3 || h.type == 5) {
          cd Z = fma_c(h.p0, z, h.p1);
          cd chi = exterior_chi(Z);
          if (m > 0) {
            cd w = recip(chi);
            cd r = c[m - 1];
            for (int k = m - 2; k >= 0; k--) r = fma_c(r, w, c[k]);
            acc_re += r.re;
            acc_im += r.im;
          }
          if (!RHS && h.type != 5) {
            if (kind == KIND_PSI)
              acc_im += h.qk * atan2(chi.im, chi.re);
            else
              acc_re += h.qk * (0.5 * log(norm2(chi)));
          }
        } else if (h.type == 1) {
          cd chi = h.p1.re * z;
          if (m > 0) {
            cd r = c[m - 1];
            for (int k = m - 2; k >= 0; k--) r = fma_c(r, chi, c[k]);
            acc_re += r.re;
            acc_im += r.im;
          }
        } else if (h.type == 2) {
          cd chi = h.p1.re * (z - h.p0);
          const double thr = (1.0 - 1e-12) * (1.0 - 1e-12);
          if (norm2(chi) < thr) {
            acc_re = NAN;
            acc_im = NAN;
          } else if (!RHS) {
            if (kind == KIND_PSI)
              acc_im += h.qk * atan2(chi.im, chi.re);
            else
              acc_re += h.qk * (0.5 * log(norm2(chi)));
          }
        } else if (h.type == 4) {
          cd chi = h.p1.re * (z - h.p0);
          const double thr = (1.0 - 1e-10) * (1.0 - 1e-10);
          if (norm2(chi) < thr) {
            acc_re = NAN;
            acc_im = NAN;
          } else if (m > 0) {
            cd w = recip(chi);
            cd r = c[m - 1];
            for (int k = m - 2; k >= 0; k--) r = fma_c(r, w, c[k]);
            acc_re += r.re;
            acc_im += r.im;
          }
        }
      }
    }
  }
  if (active) {
    if (RHS)
      out[gout] = acc_re;
    else
      out[gout] = (kind == KIND_PSI) ? acc_im : (acc_re + net.constant[f]);
  }
}

// ------------------------------------------------------------------------
// Pair tables of the sweep.  Within one solve the collocation points and the
// element geometry are fixed, so for every (collocation point, source
// element of the point's fracture) pair the map value the series needs and
// the log term are the same in every iteration:
//   x = 1/chi  (Laurent types 0, 3, 4, 5)   or   chi = z / R  (bounding
//       circle, type 1; Taylor series);
//   l = 0.5 log|chi|^2 (point of a phi element) or atan2(chi) (psi element)
//       for the discharge types 0, 2, 3, else 0; NaN where the reference's
//       potential is NaN (inside a well or an impermeable circle).
// The sweep then evaluates sum_k c_k x^k + qk * l per pair: the Horner chain
// alone instead of two square roots, a reciprocal and a logarithm.
// Layout, per fracture f: [source slot s][point of f] (points contiguous,
// so a warp's loads for one source are coalesced), from tab_off[f]; the
// points of f are the flattened sweep points [fpt0[f], fpt0[f] + fnp[f]).
// The values are computed with the same expressions as eval_kernel<false>,
// so both sweeps give the same results bit for bit.
// ------------------------------------------------------------------------
__device__ __forceinline__ void line_map_coeffs(const Net &net, int el, int f, cd &p0, cd &p1) {
  // Z = p0 z + p1 = (2 z - a - b) / (b - a) on the side of el that lies in f
  const int side = (net.type[el] == 0 && net.frac0[el] != f) ? 1 : 0;
  const cd *ep = side ? net.ep1 + 2 * el : net.ep0 + 2 * el;
  cd a = ep[0], b = ep[1];
  cd inv = recip(b - a);
  p0 = 2.0 * inv;
  cd ab = a + b;
  p1 = mk(-(ab.re * inv.re - ab.im * inv.im), -(ab.re * inv.im + ab.im * inv.re));
}

__global__ void __launch_bounds__(EVAL_THREADS) pair_table_kernel(Net net, const Item *__restrict__ items,
                                                                    const int2 *__restrict__ pts,
                                                                    const Group *__restrict__ groups,
                                                                    const int *__restrict__ fpt0,
                                                                    const int *__restrict__ fnp,
                                                                    const long long *__restrict__ tab_off,
                                                                    cd *__restrict__ tw, double *__restrict__ tl) {
  const Item it = items[blockIdx.x];
  const int p = it.p0 + threadIdx.x;
  if (p >= it.p1) return;
  const int f = it.frac;
  const int2 gk = pts[p];
  const Group g = groups[gk.x];
  const int exclude = g.elem, kind = g.kind;
  const cd z = sweep_point(net, g.elem, g.side, gk.y);
  const int np = fnp[f];
  const long long base = tab_off[f] + (p - fpt0[f]);
  const int e0 = net.fptr[f], e1 = net.fptr[f + 1];
  for (int s = 0; s < e1 - e0; s++) {
    const int el = net.felem[e0 + s];
    const int type = net.type[el];
    cd x = mk(0.0, 0.0);
    double l = 0.0;
    if (el != exclude) {
      if (type == 0 || type == 3 || type == 5) {
        cd p0, p1;
        line_map_coeffs(net, el, f, p0, p1);
        const cd chi = exterior_chi(fma_c(p0, z, p1));
        x = recip(chi);
        if (type != 5) l = (kind == KIND_PSI) ? atan2(chi.im, chi.re) : 0.5 * log(norm2(chi));
      } else if (type == 1) {
        const double ir = 1.0 / net.radius[el];
        x = ir * z;
      } else {
        const double ir = 1.0 / net.radius[el];
        const cd chi = ir * (z - net.center[el]);
        if (type == 2) {
          const double thr = (1.0 - 1e-12) * (1.0 - 1e-12);
          if (norm2(chi) < thr)
            l = NAN;
          else
            l = (kind == KIND_PSI) ? atan2(chi.im, chi.re) : 0.5 * log(norm2(chi));
        } else {  // type 4
          const double thr = (1.0 - 1e-10) * (1.0 - 1e-10);
          if (norm2(chi) < thr)
            l = NAN;
          else
            x = recip(chi);
        }
      }
    }
    tw[base + (long long)s * np] = x;
    tl[base + (long long)s * np] = l;
  }
}

// A complex128 load with the streaming (evict-first) cache policy.
__device__ __forceinline__ cd ldcs_cd(const cd *p) {
  const double2 v = __ldcs(reinterpret_cast<const double2 *>(p));
  return mk(v.x, v.y);
}

// The sweep from the pair tables, one item (fracture, <= EVAL_THREADS
// collocation points; one thread per point).  The item's sources are staged
// in shared memory (signed coefficients, zero-padded to MC, ncoef,
// q / 2 pi, id), and every thread walks them two at a time (two independent
// Horner chains), loading the next pair's table entries before the current
// pair's chains run.  The table loads are streaming (evict-first): the
// tables are read once per sweep, and the power sums and coefficients of the
// other kernels should stay in L2.  Output as eval_kernel<false>.
struct TabSrc {
  int id, m;
  double qk;
};

__device__ __forceinline__ void sweep_table_item(const Net &net, const Item it, const int2 *__restrict__ pts,
                                                 const Group *__restrict__ groups, const int *__restrict__ fpt0,
                                                 const int *__restrict__ fnp, const long long *__restrict__ tab_off,
                                                 const cd *__restrict__ tw, const double *__restrict__ tl,
                                                 double *__restrict__ out, int chunk) {
  const int f = it.frac;
  if (net.st[net.real_frac[f]].done) return;  // uniform over the CTA
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TabSrc *src = reinterpret_cast<TabSrc *>(smem_raw);
  cd *scoef = reinterpret_cast<cd *>(smem_raw + sizeof(TabSrc) * chunk);
  const int MC = net.MC;
  const int p = it.p0 + threadIdx.x;
  const bool active = p < it.p1;
  int exclude = -1, kind = KIND_PHI, gout = 0;
  long long base = 0;
  const int np = fnp[f];
  if (active) {
    const int2 gk = pts[p];
    const Group g = groups[gk.x];
    gout = g.out + gk.y;
    exclude = g.elem;
    kind = g.kind;
    base = tab_off[f] + (p - fpt0[f]);
  }
  const int e0 = net.fptr[f], e1 = net.fptr[f + 1];
  double acc_re = 0.0, acc_im = 0.0;
  for (int c0 = e0; c0 < e1; c0 += chunk) {
    const int cnt = min(chunk, e1 - c0);
    __syncthreads();
    for (int s = threadIdx.x; s < cnt; s += blockDim.x) {
      const int el = net.felem[c0 + s];
      const int type = net.type[el];
      const double sg = (type == 0 && net.frac0[el] != f) ? -1.0 : 1.0;
      TabSrc h;
      h.id = el;
      h.m = net.ncoef[el];
      h.qk = sg * net.q[el] / (2 * PI);
      src[s] = h;
    }
    for (int idx = threadIdx.x; idx < cnt * MC; idx += blockDim.x) {
      const int s = idx / MC, k = idx - s * MC;
      const int el = net.felem[c0 + s];
      const int m = net.ncoef[el];
      const bool neg = (net.type[el] == 0 && net.frac0[el] != f);
      cd c = (k < m) ? net.coef[(size_t)el * MC + k] : mk(0.0, 0.0);
      if (neg) c = mk(-c.re, -c.im);
      scoef[idx] = c;
    }
    __syncthreads();
    if (!active) continue;
    const cd *__restrict__ xw = tw + base + (long long)(c0 - e0) * np;
    const double *__restrict__ xl = tl + base + (long long)(c0 - e0) * np;
    int s = 0;
    cd xa = mk(0.0, 0.0), xb = mk(0.0, 0.0);
    double la = 0.0, lb = 0.0;
    if (cnt >= 2) {
      xa = ldcs_cd(xw);
      la = __ldcs(xl);
      xb = ldcs_cd(xw + np);
      lb = __ldcs(xl + np);
    }
    for (; s + 1 < cnt; s += 2) {
      // the next pair's table entries, in flight while this pair's chains run
      cd na = mk(0.0, 0.0), nb = mk(0.0, 0.0);
      double nla = 0.0, nlb = 0.0;
      if (s + 3 < cnt) {
        na = ldcs_cd(xw + (long long)(s + 2) * np);
        nla = __ldcs(xl + (long long)(s + 2) * np);
        nb = ldcs_cd(xw + (long long)(s + 3) * np);
        nlb = __ldcs(xl + (long long)(s + 3) * np);
      }
      const TabSrc ha = src[s], hb = src[s + 1];
      const int mm = max(ha.m, hb.m);
      cd ra = mk(0.0, 0.0), rb = mk(0.0, 0.0);
      if (mm > 0) {
        const cd *ca = scoef + s * MC, *cb = ca + MC;
        ra = ca[mm - 1];
        rb = cb[mm - 1];
        for (int k = mm - 2; k >= 0; k--) {
          ra = fma_c(ra, xa, ca[k]);
          rb = fma_c(rb, xb, cb[k]);
        }
      }
      if (ha.id != exclude) {
        acc_re += ra.re;
        acc_im += ra.im;
        if (kind == KIND_PSI)
          acc_im += ha.qk * la;
        else
          acc_re += ha.qk * la;
      }
      if (hb.id != exclude) {
        acc_re += rb.re;
        acc_im += rb.im;
        if (kind == KIND_PSI)
          acc_im += hb.qk * lb;
        else
          acc_re += hb.qk * lb;
      }
      xa = na;
      la = nla;
      xb = nb;
      lb = nlb;
    }
    if (s < cnt) {  // odd source count: the last one alone
      const TabSrc h = src[s];
      if (h.id != exclude) {
        const cd x = ldcs_cd(xw + (long long)s * np);
        const double l = __ldcs(xl + (long long)s * np);
        if (h.m > 0) {
          const cd *c = scoef + s * MC;
          cd r = c[h.m - 1];
          for (int k = h.m - 2; k >= 0; k--) r = fma_c(r, x, c[k]);
          acc_re += r.re;
          acc_im += r.im;
        }
        if (kind == KIND_PSI)
          acc_im += h.qk * l;
        else
          acc_re += h.qk * l;
      }
    }
  }
  if (active) out[gout] = (kind == KIND_PSI) ? acc_im : (acc_re + net.constant[f]);
}

// One CTA per item (the hardware block scheduler hands out the items, which
// are sorted by estimated cost, largest first).
// With an active list (batches), the CTAs walk the list's items
// (grid-stride, the list's length *acount on the device).
__global__ void __launch_bounds__(EVAL_THREADS) sweep_table_kernel(Net net, const Item *__restrict__ items,
                                                                     const int2 *__restrict__ pts,
                                                                     const Group *__restrict__ groups,
                                                                     const int *__restrict__ fpt0,
                                                                     const int *__restrict__ fnp,
                                                                     const long long *__restrict__ tab_off,
                                                                     const cd *__restrict__ tw,
                                                                     const double *__restrict__ tl,
                                                                     double *__restrict__ out, int chunk,
                                                                     const int *__restrict__ alist,
                                                                     const int *__restrict__ acount) {
  // one call site (a second inlined copy of the item body made the kernel slower)
  const int n = alist ? *acount : (int)gridDim.x;
  for (int i = blockIdx.x; i < n; i += gridDim.x)  // uniform over the CTA
    sweep_table_item(net, items[alist ? alist[i] : i], pts, groups, fpt0, fnp, tab_off, tw, tl, out, chunk);
}

// Persistent form: a grid of a few CTAs per SM takes the items (largest
// first) from a device work queue, one atomic fetch per item; the last CTA
// to finish resets the queue for the next launch.
struct WorkQueue {
  int next, done;
};
__global__ void __launch_bounds__(EVAL_THREADS) sweep_table_queue_kernel(
    Net net, const Item *__restrict__ items, int n_items, const int2 *__restrict__ pts,
    const Group *__restrict__ groups, const int *__restrict__ fpt0, const int *__restrict__ fnp,
    const long long *__restrict__ tab_off, const cd *__restrict__ tw, const double *__restrict__ tl,
    double *__restrict__ out, int chunk, WorkQueue *q, const int *__restrict__ alist,
    const int *__restrict__ acount) {
  __shared__ int s_next;
  if (alist) n_items = *acount;
  while (true) {
    if (threadIdx.x == 0) s_next = atomicAdd(&q->next, 1);
    __syncthreads();
    const int i = s_next;
    __syncthreads();  // every thread has read s_next before thread 0 fetches again
    if (i >= n_items) break;
    sweep_table_item(net, items[alist ? alist[i] : i], pts, groups, fpt0, fnp, tab_off, tw, tl, out, chunk);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&q->done, 1) == (int)gridDim.x - 1) {  // every CTA has stopped fetching
      q->next = 0;
      q->done = 0;
      __threadfence();
    }
  }
}

// ------------------------------------------------------------------------
// Active work lists of a batch.  Once realizations finish, their rows, sweep
// items and elements still occupy the grids of the per-iteration kernels
// (each CTA or warp returning at entry); in a batch's last iterations, with
// a few realizations left, those empty launches cost more than the work.
// The lists below hold, in their original order, the entries of the
// realizations still running; the kernels take entry alist[i] for i below
// the list's length.  They are rebuilt at the end of an iteration in which
// a realization finished (ndone changed), by two launches over chunks of
// ACT_CHUNK entries: per-chunk counts, then each chunk's prefix (the sum of
// the counts before it) and an order-preserving scatter.  Launches in which
// nothing changed return at entry.
// ------------------------------------------------------------------------
static constexpr int ACT_CHUNK = 1024;
// head-vector rows, sweep items, updated elements, realizations solved on a
// cluster (a prefix of the size order), realizations solved by one CTA (the
// rest of it), all realizations (the reduction)
static constexpr int ACT_LISTS = 6;

struct ActState {
  int seen;         // ndone when the lists were last built
  unsigned arrive;  // CTAs of the scatter launch that have finished
  int count[ACT_LISTS];
};

struct ActLists {
  int n[ACT_LISTS];       // entries of the full lists
  int chunk0[ACT_LISTS + 1];  // first compaction CTA of each list (chunk0[ACT_LISTS] = grid)
  int *list[ACT_LISTS];   // active entries (indices into the full list)
  int *ccnt;              // active entries per chunk, all lists
  const Item *items;      // the sweep items (list 1's realization lookup)
  const int *order;       // realizations by decreasing size (lists 3 and 4), or null
  int nbig;               // realizations solved on a cluster (list 3's length)
  ActState *st;
};

// the realization of entry i of list l
__device__ __forceinline__ int act_real(const Net &net, const ActLists &A, int l, int i) {
  switch (l) {
    case 0: return net.real_row[i];
    case 1: return net.real_frac[A.items[i].frac];
    case 2: return net.real_elem[i];
    case 3: return A.order[i];
    case 4: return A.order[A.nbig + i];
    default: return i;
  }
}

__device__ __forceinline__ void act_locate(const ActLists &A, int &l, int &c) {
  l = 0;
  while (l + 1 < ACT_LISTS && (int)blockIdx.x >= A.chunk0[l + 1]) l++;
  c = (int)blockIdx.x - A.chunk0[l];
}

__global__ void __launch_bounds__(ACT_CHUNK) act_count_kernel(Net net, ActLists A) {
  if (A.st->seen == *net.ndone) return;  // uniform: nothing finished since the last build
  int l, c;
  act_locate(A, l, c);
  const int i = c * ACT_CHUNK + threadIdx.x;
  const bool on = i < A.n[l] && !net.st[act_real(net, A, l, i)].done;
  const int n = __syncthreads_count(on);
  if (threadIdx.x == 0) A.ccnt[blockIdx.x] = n;
}

__global__ void __launch_bounds__(ACT_CHUNK) act_scatter_kernel(Net net, ActLists A) {
  __shared__ int s_w[ACT_CHUNK / 32];
  __shared__ int s_pre;
  const int nd = *net.ndone;
  if (A.st->seen == nd) return;
  int l, c;
  act_locate(A, l, c);
  // prefix: active entries of this list's chunks before this one
  int pre = 0;
  for (int k = A.chunk0[l] + (int)threadIdx.x; k < A.chunk0[l] + c; k += ACT_CHUNK) pre += A.ccnt[k];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) pre += __shfl_xor_sync(0xffffffffu, pre, o);
  if (lane == 0) s_w[warp] = pre;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < ACT_CHUNK / 32; w++) t += s_w[w];
    s_pre = t;
  }
  __syncthreads();
  const int base = s_pre;
  // order-preserving scatter of the chunk's active entries
  const int i = c * ACT_CHUNK + threadIdx.x;
  const bool on = i < A.n[l] && !net.st[act_real(net, A, l, i)].done;
  const unsigned m = __ballot_sync(0xffffffffu, on);
  if (lane == 0) s_w[warp] = __popc(m);  // thread 0's reads of s_w ended at the barrier above
  __syncthreads();
  int wpre = 0;
  for (int w = 0; w < warp; w++) wpre += s_w[w];
  if (on) A.list[l][base + wpre + __popc(m & ((1u << lane) - 1u))] = i;
  const int last_chunk = (A.n[l] + ACT_CHUNK - 1) / ACT_CHUNK - 1;
  if (c == last_chunk && threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < ACT_CHUNK / 32; w++) t += s_w[w];
    A.st->count[l] = base + t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&A.st->arrive, 1u) == gridDim.x - 1) {  // the last CTA of the rebuild
      A.st->arrive = 0;
      A.st->seen = nd;
      __threadfence();
    }
  }
}

// The full lists (identity) at the start of a run.
__global__ void act_init_kernel(ActLists A, int ndone0) {
  for (int l = 0; l < ACT_LISTS; l++)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n[l]; i += gridDim.x * blockDim.x) A.list[l][i] = i;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    A.st->seen = ndone0;
    A.st->arrive = 0;
    for (int l = 0; l < ACT_LISTS; l++) A.st->count[l] = A.n[l];
  }
}

// ------------------------------------------------------------------------
// Per-element fit: Cauchy-integral DFT, per-type transform, errors, blends.
// One warp per element.  vals holds phi (or psi) at the collocation points.
// ------------------------------------------------------------------------
__device__ __forceinline__ void dft_lane(const double *v, int n, int type, int j, bool imag_unit, cd &out) {
  // integral_j = sum_k v_k exp(-i j theta_k), theta_k = start + k del: the
  // phase advances by a fixed rotation; it is re-anchored every 32 points.
  double del = PI / n, start = del / 2;
  if (type == 1) {
    del = 2 * PI / n;
    start = 0.0;
  }
  double rs, rc;
  sincos((double)j * del, &rs, &rc);
  double sr = 0.0, si = 0.0;
  double c = 1.0, s = 0.0;
  for (int k = 0; k < n; k++) {
    if ((k & 31) == 0) sincos((double)j * (start + k * del), &s, &c);
    sr = fma(v[k], c, sr);
    si = fma(-v[k], s, si);
    const double c2 = fma(c, rc, -s * rs);
    s = fma(s, rc, c * rs);
    c = c2;
  }
  // coef_j = 2 * integral_j / n   (real Cauchy integral)
  // coef_j = 2i * integral_j / n  (stream-function Cauchy integral)
  if (imag_unit)
    out = mk(-2.0 * si / n, 2.0 * sr / n);
  else
    out = mk(2.0 * sr / n, 2.0 * si / n);
  if (j == 0) out = mk(out.re / 2, out.im / 2);
}

// The Cauchy-integral DFT of one lane's coefficient j from the element's
// basis B (entry (k, j) = exp(-i theta_k)^j, the powers the reference forms
// by repeated multiplication, hpc_math_functions.py:244-297): the products
// and sums in the reference's order (a product, then a sum, point by point).
// Two value sets (the sides of an intersection) share the basis loads.
template <int SETS>
__device__ __forceinline__ void dft_basis(const double *v0, const double *v1, int n, const cd *__restrict__ B,
                                          int MC, int j, bool imag_unit, cd &out0, cd &out1) {
  double r0 = 0.0, i0 = 0.0, r1 = 0.0, i1 = 0.0;
  for (int k = 0; k < n; k++) {
    const cd b = B[(size_t)k * MC + j];
    r0 = __dadd_rn(r0, __dmul_rn(v0[k], b.re));
    i0 = __dadd_rn(i0, __dmul_rn(v0[k], b.im));
    if (SETS == 2) {
      r1 = __dadd_rn(r1, __dmul_rn(v1[k], b.re));
      i1 = __dadd_rn(i1, __dmul_rn(v1[k], b.im));
    }
  }
  // coef_j = 2 integral_j / n (real Cauchy integral), 2i integral_j / n
  // (stream-function Cauchy integral); coef_0 halved
  if (imag_unit)
    out0 = mk(-2.0 * i0 / n, 2.0 * r0 / n);
  else
    out0 = mk(2.0 * r0 / n, 2.0 * i0 / n);
  out1 = mk(2.0 * r1 / n, 2.0 * i1 / n);
  if (j == 0) {
    out0 = mk(out0.re / 2, out0.im / 2);
    out1 = mk(out1.re / 2, out1.im / 2);
  }
}

// The running maximum of the element errors with its (first) index, the
// maximum of the coefficient errors and a non-finite flag, with np.max /
// np.argmax semantics: a NaN wins, the first index among equal maxima or
// NaNs.  merge() is associative and commutative, so any split of the
// elements gives the same result.
struct ErrAcc {
  double best = -INFINITY, bec = -INFINITY;
  int bidx = 0x7fffffff, nonfin = 0;
  // element i (visited in increasing order by one thread)
  __device__ __forceinline__ void add(double e, double ec, int i) {
    if (!(e == e)) {
      if (best == best) {
        best = NAN;
        bidx = i;
      } else {
        bidx = min(bidx, i);
      }
      nonfin = 1;
    } else if (best == best && (e > best || (e == best && i < bidx))) {
      best = e;
      bidx = i;
    }
    if (!(ec == ec)) {
      bec = NAN;
      nonfin = 1;
    } else if (bec == bec && ec > bec) {
      bec = ec;
    }
  }
  __device__ __forceinline__ void merge(double ob, int oi, double oec, int onf) {
    const bool onan = !(ob == ob), mnan = !(best == best);
    if (onan && (!mnan || oi < bidx)) {
      best = ob;
      bidx = oi;
    } else if (!onan && !mnan && (ob > best || (ob == best && oi < bidx))) {
      best = ob;
      bidx = oi;
    }
    if (!(oec == oec) || (bec == bec && oec > bec)) bec = oec;
    nonfin |= onf;
  }
  __device__ __forceinline__ void warp_merge() {
    for (int o = 16; o > 0; o >>= 1)
      merge(__shfl_xor_sync(0xffffffffu, best, o), __shfl_xor_sync(0xffffffffu, bidx, o),
            __shfl_xor_sync(0xffffffffu, bec, o), __shfl_xor_sync(0xffffffffu, nonfin, o));
  }
};

// The block's ErrAcc into thread 0 (every thread calls it).
template <int THREADS>
__device__ __forceinline__ void block_merge(ErrAcc &a) {
  __shared__ double s_err[THREADS / 32], s_ec[THREADS / 32];
  __shared__ int s_idx[THREADS / 32], s_nf[THREADS / 32];
  a.warp_merge();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    s_err[w] = a.best;
    s_idx[w] = a.bidx;
    s_ec[w] = a.bec;
    s_nf[w] = a.nonfin;
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 1; k < THREADS / 32; k++) a.merge(s_err[k], s_idx[k], s_ec[k], s_nf[k]);
}

// The convergence rule of realization r from its errors (one thread).
__device__ __forceinline__ void reduce_finish(Net &net, SolveState *st, const ErrAcc &a, int e0) {
  int nf = a.nonfin;
  st->error = a.best;
  st->worst = a.bidx - e0;
  st->error_coef = a.bec;
  if (!(st->error_q == st->error_q)) nf = 1;
  if (nf) st->nonfinite = 1;
  // hpc_solve.py:237-239
  if (a.bec < st->max_error && st->error_q < st->max_error) {
    st->cnt_error += 1;
    st->error_q = 1e30;
  }
  if (st->cnt_error >= 2 || st->nit >= st->max_it || st->nonfinite) {
    st->done = 1;
    atomicAdd(net.ndone, 1);
  }
  st->solve_q = (st->error_q > st->max_error / 1e30) ? 1 : 0;
}

static constexpr int REDUCE_SPLIT_THREADS = 256;
static constexpr int REDUCE_SPLIT_ELEMS = 4 * REDUCE_SPLIT_THREADS;
struct ReducePart {
  double best, bec;
  int bidx, nonfin;
};

// Returns false when the element's realization is done (nothing updated);
// otherwise lane 0's er / erc are the element's new errors.
__device__ __forceinline__ bool update_element(Net &net, int e, const int *__restrict__ group_of,
                                               const Group *__restrict__ groups, const double *__restrict__ vals,
                                               double *v0, double *v1, int blend_mode, double &er, double &erc);

// One warp per element of the list; with an active list (batches: its
// length *ncount on the device) the warps walk the list (grid-stride).
// (Reducing a single network's errors at the end of this kernel, the last
// CTA merging the CTAs' partial maxima, measured 5 us slower an iteration
// than the separate launch: 1,344 CTAs' fences and atomics on one ticket.)
__global__ void __launch_bounds__(UPDATE_WARPS * 32) update_kernel(Net net, const int *__restrict__ elist, int nlist,
                                                                    const int *__restrict__ group_of,
                                                                    const Group *__restrict__ groups,
                                                                    const double *__restrict__ vals, int nvmax,
                                                                    int blend_mode,
                                                                    const int *__restrict__ ncount = nullptr) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5;
  double *v0 = reinterpret_cast<double *>(smem_raw) + (size_t)warp * 2 * nvmax;
  double *v1 = v0 + nvmax;
  const int idx = blockIdx.x * UPDATE_WARPS + warp;
  const int n = ncount ? *ncount : nlist;
  for (int i = idx; i < n; i += gridDim.x * UPDATE_WARPS) {
    __syncwarp();  // the previous element's reads of v0 / v1 are done
    double er, erc;
    update_element(net, elist[i], group_of, groups, vals, v0, v1, blend_mode, er, erc);
  }
}

__device__ __forceinline__ bool update_element(Net &net, int e, const int *__restrict__ group_of,
                                               const Group *__restrict__ groups, const double *__restrict__ vals,
                                               double *v0, double *v1, int blend_mode, double &er_out,
                                               double &erc_out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  SolveState *st = net.st + net.real_elem[e];
  if (st->done) return false;
  const int type = net.type[e];
  const int MC = net.MC;
  if (type == 2) {  // hpc_solve.py:366-368
    if (lane == 0) net.err[e] = 0.0;
    er_out = 0.0;
    erc_out = net.err_coef[e];
    return true;
  }
  const int n = net.nint[e], m = net.ncoef[e];
  const Group g0 = groups[group_of[2 * e]];
  for (int k = lane; k < n; k += 32) v0[k] = vals[g0.out + k];
  if (type == 0) {
    const Group g1 = groups[group_of[2 * e + 1]];
    for (int k = lane; k < n; k += 32) v1[k] = vals[g1.out + k];
  }
  const bool psi = (type == 1 || type == 4 || type == 5);
  if (psi) {
    // get_dpsi_corr (hpc_math_functions.py:407-447) and the unwrapping of
    // psi in cauchy_integral_domega(_line) (:496-505, :586-595):
    // psi'_k = psi_k - sum_{i<k} dpsi_corr_i.  The cuts are staged 32 at a
    // time in shared memory (one load round by the warp's lanes); every lane
    // then adds them in cut order, as one serial loop over the cuts would.
    __shared__ int s_cp[UPDATE_WARPS][32];
    __shared__ double s_qv[UPDATE_WARPS][32];
    const int nc = net.cut_n[e];
    const int *cp = net.cut_pos + (size_t)e * net.cut_cap;
    const int *ce = net.cut_elem + (size_t)e * net.cut_cap;
    const int *cs = net.cut_sign + (size_t)e * net.cut_cap;
    double *dc = net.dpsi_corr + (size_t)e * 2 * MC;
    double cum0 = 0.0, here0 = 0.0, cum1 = 0.0, here1 = 0.0;  // points lane and lane + 32
    const int k0 = lane, k1 = lane + 32;
    for (int c0 = 0; c0 < nc; c0 += 32) {
      const int cnt = min(32, nc - c0);
      __syncwarp();
      if (lane < cnt) {
        s_cp[warp][lane] = cp[c0 + lane];
        s_qv[warp][lane] = net.q[ce[c0 + lane]] * (double)cs[c0 + lane];
      }
      __syncwarp();
      for (int c = 0; c < cnt; c++) {
        const int pos = s_cp[warp][c];
        const double qv = s_qv[warp][c];
        if (pos < k0) cum0 += qv;
        if (pos == k0) here0 += qv;
        if (pos < k1) cum1 += qv;
        if (pos == k1) here1 += qv;
      }
    }
    __syncwarp();
    if (k0 < n) {
      if (k0 < n - 1) dc[k0] = here0;
      v0[k0] -= cum0;
    }
    if (k1 < n) {
      if (k1 < n - 1) dc[k1] = here1;
      v0[k1] -= cum1;
    }
    for (int k = lane + 64; k < n; k += 32) {  // points beyond 64 (nint > 64), in the serial form
      double cum = 0.0, here = 0.0;
      for (int c = 0; c < nc; c++) {
        const double qv = net.q[ce[c]] * (double)cs[c];
        if (cp[c] < k) cum += qv;
        if (cp[c] == k) here += qv;
      }
      if (k < n - 1) dc[k] = here;
      v0[k] -= cum;
    }
  }
  __syncwarp();
  const double t0 = net.t[net.frac0[e]];
  const double t1 = (type == 0) ? net.t[net.frac1[e]] : 0.0;
  const cd *oldc = net.coef + (size_t)e * MC;
  cd *neww = net.wcoef + (size_t)e * MC;
  const int i90 = (int)(m * 0.9);
  double s5 = 0.0, ecoef = 0.0;
  cd c1 = mk(0.0, 0.0), c10 = mk(0.0, 0.0);
  const cd *B = net.dft_tab + net.dft_off[e];
  for (int j = lane; j < m; j += 32) {
    cd nj;
    if (type == 0) {
      cd a0, a1;
      dft_basis<2>(v0, v1, n, B, MC, j, false, a0, a1);
      // Re((t0 c1 - t1 c0) / (t0 + t1)), coef_0 = 0 (hpc_intersection.py:95-102)
      nj = mk((t0 * a1.re - t1 * a0.re) / (t0 + t1), 0.0);
      if (j == 0) nj = mk(0.0, 0.0);
    } else if (type == 3) {
      cd a, unused;
      dft_basis<1>(v0, v0, n, B, MC, j, false, a, unused);
      nj = mk(-a.re, 0.0);  // hpc_const_head_line.py:72-76
      if (j == 0) nj = mk(0.0, 0.0);
    } else {
      cd a, unused;
      dft_basis<1>(v0, v0, n, B, MC, j, true, a, unused);
      if (type == 1) {
        nj = mk(-a.re, -a.im);  // hpc_bounding_circle.py:154
      } else if (type == 4) {
        nj = mk(a.re, -a.im);  // hpc_imp_object.py:54-56
        if (j == 0) nj = mk(0.0, 0.0);
      } else {
        nj = mk(-a.im * 0.0 - 0.0, -a.im);  // hpc_imp_object.py:173-175
        if (j == 0) nj = mk(0.0, 0.0);
      }
    }
    neww[j] = nj;
    const cd oj = oldc[j];
    if (j < 5) s5 += hypot(oj.re, oj.im);
    c1 = c1 + nj;
    if (j >= i90) c10 = c10 + nj;
    ecoef += hypot(nj.re - oj.re, nj.im - oj.im);
  }
  s5 = warp_sum(s5);
  ecoef = warp_sum(ecoef);
  c1 = warp_sum(c1);
  c10 = warp_sum(c10);
  if (lane == 0) {
    // calc_error / calc_coef_error (hpc_math_functions.py:612-670)
    double er = 0.0, erc = 0.0;
    if (!(s5 < 1e-15)) {
      er = fabs(hypot(c1.re - c10.re, c1.im - c10.im) / hypot(c1.re + 1e-16, c1.im) - 1);
      erc = ecoef / m;
    }
    net.err_old2[e] = net.err_old[e];
    net.err_old[e] = net.err[e];
    net.err[e] = er;
    net.err_coef[e] = erc;
    er_out = er;
    erc_out = erc;
  }
  // damped blends (hpc_solve.py:383-388 and, for nit >= 2, 561-575)
  const double d = st->damping;
  const int nb = (blend_mode == 2) ? 0 : (blend_mode == 1 ? 1 : ((st->fused_blend2 && st->nit >= 2) ? 2 : 1));
  cd *cc = net.coef + (size_t)e * MC;
  for (int j = lane; j < m; j += 32) {
    cd w = neww[j], c = cc[j];
    for (int b = 0; b < nb; b++) c = mk(d * w.re + (1 - d) * c.re, d * w.im + (1 - d) * c.im);
    cc[j] = c;
    // a non-finite leading coefficient ends the realization's loop (read by reduce_kernel)
    if (j == 0 && !isfinite(c.re)) st->nonfinite = 1;
  }
  return true;
}

// ------------------------------------------------------------------------
// Adaptive coefficient growth (element_solver2, hpc_solve.py:465-559): after
// the first blend, an element whose tail coefficients are large relative to
// the rest, or whose error rose three times in a row, gets COEF_INCREASE more
// coefficients and nint = 2 ncoef, at most once per iteration.  The decision
// uses the reference's operation order (sequential complex sums, Smith
// division, hypot) on the blended coefficients.  One warp per element; the
// grown elements are appended to grow_list.
// ------------------------------------------------------------------------
__global__ void growth_kernel(Net net, const int *__restrict__ elist, int nlist, double max_coef_ratio,
                              int max_coef, int coef_increase, int *grow_list, int *grow_count) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nlist || lane != 0) return;
  const int e = elist[warp];
  const SolveState *st = net.st + net.real_elem[e];
  if (st->done) return;
  if (net.type[e] == 2) return;
  const int nit = st->nit;
  if (nit < 2) return;
  const int m = net.ncoef[e];
  const cd *c = net.coef + (size_t)e * net.MC;
  const int ncc = 3;
  double s = 0.0;
  int cnt = 0;
  for (int k = 1; k < min(ncc, m); k++) {
    s += hypot(c[k].re, c[k].im);
    cnt++;
  }
  const double coef0 = (cnt > 0 ? s / cnt : NAN) + 1e-30;
  double coef1 = -INFINITY;
  for (int k = max(0, m - ncc); k < m; k++) {
    const double v = hypot(c[k].re, c[k].im);
    if (v != v) {
      coef1 = v;
      break;
    }
    if (v > coef1) coef1 = v;
  }
  double ratio = (coef0 == 0.0) ? 0.0 : coef1 / coef0 * 0;
  if (m > 1 && hypot(c[1].re, c[1].im) < st->max_error / 1e10) ratio = 0.0;
  const double err = net.err[e], eo = net.err_old[e], eo2 = net.err_old2[e];
  if (err > eo && err > eo2 && err > st->max_error && nit > 5) ratio = max_coef_ratio + 1.0;
  cd sl = mk(0.0, 0.0), sr = mk(0.0, 0.0);
  for (int k = max(0, m - ncc); k < m; k++) sl = mk(sl.re + c[k].re, sl.im + c[k].im);
  for (int k = 0; k < max(0, m - ncc); k++) sr = mk(sr.re + c[k].re, sr.im + c[k].im);
  const cd qt = cdiv_ref(sl, mk(sr.re + 1e-30, sr.im + 0.0));
  if (hypot(qt.re, qt.im) > max_coef_ratio && err > st->max_error) ratio = max_coef_ratio + 1.0;
  if (ratio > max_coef_ratio && m < max_coef && nit > 1) {
    net.ncoef[e] = m + coef_increase;
    net.nint[e] = (m + coef_increase) * 2;
    const int slot = atomicAdd(grow_count, 1);
    grow_list[slot] = e;
  }
}

// Second damped blend of element_solver2 (hpc_solve.py:561-575), nit >= 2.
__global__ void blend2_kernel(Net net) {
  const long long tot = (long long)net.ne * net.MC;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(i / net.MC), j = (int)(i - (long long)e * net.MC);
    if (j >= net.ncoef[e]) continue;
    const SolveState *st = net.st + net.real_elem[e];
    if (st->done || st->nit < 2) continue;
    const double d = st->damping;
    const cd w = net.wcoef[i], c = net.coef[i];
    net.coef[i] = mk(d * w.re + (1 - d) * c.re, d * w.im + (1 - d) * c.im);
  }
}

// ------------------------------------------------------------------------
// Max-reductions of the element errors and the convergence rule.
// ------------------------------------------------------------------------

__device__ __forceinline__ void reduce_one(Net &net, int r) {
  SolveState *st = net.st + r;
  if (st->done) return;  // uniform over the CTA
  ErrAcc a;
  const int e0 = net.eoff[r], e1 = net.eoff[r + 1];
#pragma unroll 4
  for (int i = e0 + threadIdx.x; i < e1; i += blockDim.x) a.add(net.err[i], net.err_coef[i], i);
  block_merge<1024>(a);
  if (threadIdx.x == 0) reduce_finish(net, st, a, e0);
}

// One CTA per realization; with an active list (batches: its length
// *acount on the device) the CTAs walk the running realizations.
__global__ void __launch_bounds__(1024) reduce_kernel(Net net, const int *__restrict__ alist = nullptr,
                                                      const int *__restrict__ acount = nullptr) {
  const int n = alist ? *acount : (int)gridDim.x;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    __syncthreads();  // the previous realization's merge is read
    reduce_one(net, alist ? alist[i] : i);
  }
}

// A single network's reduction over several CTAs (REDUCE_SPLIT_ELEMS
// elements each, one element per thread and round): every CTA writes its
// partial result, the last to finish merges them in CTA order and applies
// the convergence rule, then resets the ticket for the next launch.
__global__ void __launch_bounds__(REDUCE_SPLIT_THREADS) reduce_split_kernel(Net net, ReducePart *parts,
                                                                           unsigned *ticket) {
  SolveState *st = net.st;
  if (st->done) return;
  ErrAcc a;
  const int e1 = net.eoff[1];
  const int c0 = blockIdx.x * REDUCE_SPLIT_ELEMS;
#pragma unroll
  for (int u = 0; u < REDUCE_SPLIT_ELEMS / REDUCE_SPLIT_THREADS; u++) {
    const int i = c0 + u * REDUCE_SPLIT_THREADS + threadIdx.x;
    if (i < e1) a.add(net.err[i], net.err_coef[i], i);
  }
  block_merge<REDUCE_SPLIT_THREADS>(a);
  __shared__ int s_last;
  if (threadIdx.x == 0) {
    parts[blockIdx.x] = ReducePart{a.best, a.bec, a.bidx, a.nonfin};
    __threadfence();
    s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  ErrAcc t;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += REDUCE_SPLIT_THREADS)
    t.merge(__ldcg(&parts[k].best), __ldcg(&parts[k].bidx), __ldcg(&parts[k].bec), __ldcg(&parts[k].nonfin));
  block_merge<REDUCE_SPLIT_THREADS>(t);
  if (threadIdx.x == 0) {
    reduce_finish(net, st, t, 0);
    *ticket = 0;
  }
}

// ------------------------------------------------------------------------
// Discharge solve: b from the RHS point values, x = Q U^-1 L^-1 P b, scatter.
// One CTA; rows are solved by warps in dependency order, each waiting on
// per-row ready flags (all warps are resident, and a row only waits on rows
// of smaller (L) / larger (U) index, so the waits always end).  Every wait is
// bounded; on timeout the CTA sets abort_flag and finishes without waiting.
// ------------------------------------------------------------------------
// Factor rows are stored in level order (rows of one level contiguous, each
// row's entries contiguous): a level's rows depend only on earlier levels.
struct LevelSolve {
  const int *lev_ptr;   // [nlev + 1] slot ranges of the levels
  const int *rows;      // [N] row solved in each slot
  const int *eptr;      // [N + 1] entry range of each slot
  const int *col;       // entries: column (pivot-step index)
  const double *val;    // entries: value
  const double *scale;  // [nslots] per-slot multiplier (1/U(i,i)) or null
  int nlev;
  int nslots;           // rows in this solve (rows[] has nslots, eptr[] nslots + 1 entries)
  int group;            // lanes per row: 4, 8, 16 or 32
};

static constexpr int PF = 4;  // factor entries per lane kept in registers

struct RowRegs {
  int row, beg, end;
  int c[PF];
  double v[PF];
  double scale;
};

// Slot metadata (row solved in a slot and its entry range) comes from shared
// memory when it fits, so a prefetch costs one global round trip.
struct SlotMeta {
  const int *rows, *eptr;
};

// A row is handled by a group of G lanes (G = 8, 16 or 32, chosen per factor
// part from its mean row length), so one warp solves 32/G rows of a level at
// once and every group keeps its row's first G*PF entries in registers.
template <int G>
__device__ __forceinline__ void load_row(RowRegs &r, const LevelSolve &F, const SlotMeta &M, int slot, bool valid,
                                         int sub) {
  r.row = valid ? M.rows[slot] : 0;
  r.beg = valid ? M.eptr[slot] : 0;
  r.end = valid ? M.eptr[slot + 1] : 0;
  r.scale = (valid && F.scale) ? __ldg(F.scale + slot) : 1.0;
#pragma unroll
  for (int k = 0; k < PF; k++) {
    const int p = r.beg + sub + G * k;
    r.c[k] = (p < r.end) ? __ldg(F.col + p) : 0;
    r.v[k] = (p < r.end) ? __ldg(F.val + p) : 0.0;
  }
}

template <int G>
__device__ __forceinline__ void solve_row(const RowRegs &r, const LevelSolve &F, bool valid, int sub, double *y) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < PF; k++) s = fma(r.v[k], y[r.c[k]], s);
  int p = r.beg + G * PF + sub;
  for (; p + 3 * G < r.end; p += 4 * G) {  // long rows: four independent loads in flight
    const double v0 = __ldg(F.val + p), v1 = __ldg(F.val + p + G), v2 = __ldg(F.val + p + 2 * G),
                 v3 = __ldg(F.val + p + 3 * G);
    const int c0 = __ldg(F.col + p), c1 = __ldg(F.col + p + G), c2 = __ldg(F.col + p + 2 * G),
              c3 = __ldg(F.col + p + 3 * G);
    s = fma(v0, y[c0], s);
    s = fma(v1, y[c1], s);
    s = fma(v2, y[c2], s);
    s = fma(v3, y[c3], s);
  }
  for (; p < r.end; p += G) s = fma(__ldg(F.val + p), y[__ldg(F.col + p)], s);
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (valid && sub == 0) y[r.row] = (y[r.row] - s) * r.scale;
}

// Rows of one level beyond the first ng: every group walks its extra slots
// with the next row's loads in flight.  The loop count is uniform across a
// warp (groups past the end are predicated off) so the shuffles stay
// converged.
template <int G>
__device__ __forceinline__ void extra_rows(const LevelSolve &F, const SlotMeta &M, int r0, int r1, int gid, int ng,
                                           int sub, double *y) {
  const int first = r0 + gid + ng;
  const int wfirst = r0 + (gid - gid % (32 / G)) + ng;  // first group of this warp
  const int cnt = (r1 > wfirst) ? (r1 - wfirst + ng - 1) / ng : 0;
  if (cnt == 0) return;
  RowRegs t0, t1;
  load_row<G>(t0, F, M, first, first < r1, sub);
  for (int k = 0; k < cnt; k++) {
    const int slot = first + k * ng;
    const bool nxt = k + 1 < cnt;
    if (nxt) load_row<G>(t1, F, M, slot + ng, slot + ng < r1, sub);
    solve_row<G>(t0, F, slot < r1, sub, y);
    if (!nxt) break;
    t0 = t1;
  }
}

// One triangular solve, level by level with a block barrier between levels.
// Levels are processed in pairs: registers a hold each group's first row of
// the even levels, b of the odd levels, each refilled two levels ahead right
// after it is consumed.  s_meta holds (row, entry start) per slot when there
// is room (meta_cap >= nslots + 1 ints each).
template <int G>
__device__ void level_solve_g(const LevelSolve &F, double *y, int *s_levptr, int cap_levptr, int *s_meta,
                              int meta_cap) {
  const int lane = threadIdx.x & 31, sub = lane % G;
  const int gid = threadIdx.x / G, ng = blockDim.x / G;
  const bool lev_in_smem = F.nlev + 1 <= cap_levptr;
  const bool meta_in_smem = F.nslots + 1 <= meta_cap;
  __syncthreads();
  if (lev_in_smem)
    for (int i = threadIdx.x; i <= F.nlev; i += blockDim.x) s_levptr[i] = F.lev_ptr[i];
  if (meta_in_smem) {
    for (int i = threadIdx.x; i < F.nslots; i += blockDim.x) s_meta[i] = F.rows[i];
    for (int i = threadIdx.x; i <= F.nslots; i += blockDim.x) s_meta[meta_cap + i] = F.eptr[i];
  }
  __syncthreads();
  const int *lp = lev_in_smem ? s_levptr : F.lev_ptr;
  SlotMeta M{meta_in_smem ? s_meta : F.rows, meta_in_smem ? s_meta + meta_cap : F.eptr};
  RowRegs a, b;
  bool ha = false, hb = false;
  if (F.nlev > 0) {
    ha = lp[0] + gid < lp[1];
    load_row<G>(a, F, M, lp[0] + gid, ha, sub);
  }
  if (F.nlev > 1) {
    hb = lp[1] + gid < lp[2];
    load_row<G>(b, F, M, lp[1] + gid, hb, sub);
  }
  // A level with at most 32 / G rows is solved by warp 0 alone (rows go to
  // groups in order); between two such levels a warp barrier suffices, and the
  // other warps run ahead to the next block barrier.  The condition depends on
  // the level pointers only, so every thread takes the same barriers.
  constexpr int WG = 32 / G;
  auto level_sync = [&](int l) {
    const bool small = lp[l + 1] - lp[l] <= WG;
    const bool small_next = l + 1 < F.nlev && lp[l + 2] - lp[l + 1] <= WG;
    if (small && small_next)
      __syncwarp();
    else
      __syncthreads();
  };
  for (int l = 0; l < F.nlev; l += 2) {
    {
      const int r0 = lp[l], r1 = lp[l + 1];
      solve_row<G>(a, F, ha, sub, y);
      extra_rows<G>(F, M, r0, r1, gid, ng, sub, y);
      ha = false;
      if (l + 2 < F.nlev) {
        ha = lp[l + 2] + gid < lp[l + 3];
        load_row<G>(a, F, M, lp[l + 2] + gid, ha, sub);
      }
      level_sync(l);
    }
    if (l + 1 < F.nlev) {
      const int r0 = lp[l + 1], r1 = lp[l + 2];
      solve_row<G>(b, F, hb, sub, y);
      extra_rows<G>(F, M, r0, r1, gid, ng, sub, y);
      hb = false;
      if (l + 3 < F.nlev) {
        hb = lp[l + 3] + gid < lp[l + 4];
        load_row<G>(b, F, M, lp[l + 3] + gid, hb, sub);
      }
      level_sync(l + 1);
    }
  }
}

static constexpr int RING_SLOTS = 4;  // staged levels in flight + 1 (see level_solve_staged)

// Byte offsets into the dynamic shared memory of the trisolve kernel (y at 0).
struct Ring {
  int levptr_off, meta_off, meta_cap;
  int val_off, scale_off, col_off;  // [RING_SLOTS][cap] values, [RING_SLOTS][rcap] scales, [RING_SLOTS][cap] columns
  int cap, rcap;
};

__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
// 8 bytes from src, or zeros when !valid (source size 0: nothing is read)
__device__ __forceinline__ void cp_async8_zfill(void *dst, const void *src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Copies level l's entries (and row scales) into ring slot l % RING_SLOTS
// when they fit; called by the staging threads (warps 1 and up), each of which
// commits one group per call.
__device__ __forceinline__ void stage_level(const LevelSolve &F, const int *lp, const int *meptr, int l,
                                            const Ring &R, unsigned char *smem, int t, int nt) {
  if (l < F.nlev) {
    const int s0 = lp[l], s1 = lp[l + 1];
    const int e0 = meptr[s0], e1 = meptr[s1];
    if (e1 - e0 <= R.cap && s1 - s0 <= R.rcap) {
      const int slot = l % RING_SLOTS;
      int *dc = reinterpret_cast<int *>(smem + R.col_off) + slot * R.cap;
      double *dv = reinterpret_cast<double *>(smem + R.val_off) + slot * R.cap;
      for (int i = t; i < e1 - e0; i += nt) {
        cp_async4(dc + i, F.col + e0 + i);
        cp_async8(dv + i, F.val + e0 + i);
      }
      if (F.scale) {
        double *ds = reinterpret_cast<double *>(smem + R.scale_off) + slot * R.rcap;
        for (int i = t; i < s1 - s0; i += nt) cp_async8(ds + i, F.scale + s0 + i);
      }
    }
  }
  cp_async_commit();
}

// The rows of one level: groups of G lanes, one row per group and pass; the
// pass count depends on the level only, so the shuffles stay converged.
// Column/value/scale pointers are indexed by entry / slot position; the row's
// own value and scale are loaded before its entries, off the critical path.
// STAGED (the pointers are shared memory) and !STAGED (global) are separate
// instantiations so that each has one address space.
template <int G, bool STAGED>
__device__ __forceinline__ void solve_level_rows(double *y, const int *mrows, const int *meptr, int s0, int s1,
                                                 const int *cc, const double *vv, const double *sc) {
  const int lane = threadIdx.x & 31, sub = lane % G;
  const int gid = threadIdx.x / G, ng = blockDim.x / G;
  for (int base = s0; base < s1; base += ng) {
    const int r = base + gid;
    const bool valid = r < s1;
    int row = 0, beg = 0, end = 0;
    if (valid) {
      row = mrows[r];
      beg = meptr[r];
      end = meptr[r + 1];
    }
    const double yr = (valid && sub == 0) ? y[row] : 0.0;
    const double scl = (valid && sub == 0 && sc) ? sc[r] : 1.0;
    double a0 = 0.0, a1 = 0.0;
    int p = beg + sub;
    for (; p + G < end; p += 2 * G) {
      a0 = fma(vv[p], y[cc[p]], a0);
      a1 = fma(vv[p + G], y[cc[p + G]], a1);
    }
    if (p < end) a0 = fma(vv[p], y[cc[p]], a0);
    double acc = a0 + a1;
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (valid && sub == 0) y[row] = (yr - acc) * scl;
  }
}

// Lanes per row for a level of nrows rows: as many as keep the level to one
// pass of the row warps (the warps below the staging warps; rows go to groups
// in order, so a level that fits stays off the staging warps), at least 4.
template <bool STAGED>
__device__ __forceinline__ void solve_level_any(double *y, const int *mrows, const int *meptr, int s0, int s1,
                                                const int *cc, const double *vv, const double *sc, int nw) {
  const int nr = s1 - s0;
  if (nr <= nw)
    solve_level_rows<32, STAGED>(y, mrows, meptr, s0, s1, cc, vv, sc);
  else if (nr <= 2 * nw)
    solve_level_rows<16, STAGED>(y, mrows, meptr, s0, s1, cc, vv, sc);
  else if (nr <= 4 * nw)
    solve_level_rows<8, STAGED>(y, mrows, meptr, s0, s1, cc, vv, sc);
  else
    solve_level_rows<4, STAGED>(y, mrows, meptr, s0, s1, cc, vv, sc);
}

// Staged level solve.  A deep level has few rows, so its cost is the latency
// of fetching its factor entries; here the entries (and row scales) of the
// next RING_SLOTS - 1 levels are copied into a shared-memory ring with
// asynchronous copies (cp.async) by warps 1 and up while the current level is
// solved, and a level reads only shared memory on its critical path (y, the
// slot metadata and the ring all live in the kernel's shared memory, so the
// loads are shared-space loads).  The copies are issued by the last warps,
// which small levels' rows do not reach.  Levels larger than the ring's capacity read global
// memory directly.
__device__ void level_solve_staged(const LevelSolve &F, const Ring &R) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *y = reinterpret_cast<double *>(smem_raw);
  const int *lp = reinterpret_cast<const int *>(smem_raw + R.levptr_off);
  const int *mrows = reinterpret_cast<const int *>(smem_raw + R.meta_off);
  const int *meptr = mrows + R.meta_cap;
  // the last STAGE_WARPS warps copy; the others solve the rows of small levels
  const int nwarps = blockDim.x >> 5;
  const int nst = nwarps >= 8 ? 4 : 1;
  const int nrow_w = nwarps - nst;
  const bool stager = (int)(threadIdx.x >> 5) >= nrow_w;
  const int t = threadIdx.x - nrow_w * 32, nt = nst * 32;
  if (stager) {
    for (int l = 0; l < RING_SLOTS - 1; l++) stage_level(F, lp, meptr, l, R, smem_raw, t, nt);
    cp_async_wait<RING_SLOTS - 2>();
  }
  __syncthreads();
  for (int l = 0; l < F.nlev; l++) {
    if (stager) stage_level(F, lp, meptr, l + RING_SLOTS - 1, R, smem_raw, t, nt);  // slot of level l - 1
    const int s0 = lp[l], s1 = lp[l + 1];
    const int e0 = meptr[s0], e1 = meptr[s1];
    if (e1 - e0 <= R.cap && s1 - s0 <= R.rcap) {
      const int slot = l % RING_SLOTS;
      const int *cc = reinterpret_cast<const int *>(smem_raw + R.col_off) + slot * R.cap - e0;
      const double *vv = reinterpret_cast<const double *>(smem_raw + R.val_off) + slot * R.cap - e0;
      const double *sc =
          F.scale ? reinterpret_cast<const double *>(smem_raw + R.scale_off) + slot * R.rcap - s0 : nullptr;
      solve_level_any<true>(y, mrows, meptr, s0, s1, cc, vv, sc, nrow_w);
    } else {
      solve_level_any<false>(y, mrows, meptr, s0, s1, F.col, F.val, F.scale, nrow_w);
    }
    if (stager) cp_async_wait<RING_SLOTS - 2>();  // level l + 1's slot is complete
    __syncthreads();
  }
  if (stager) cp_async_wait<0>();
}

__device__ void level_solve(const LevelSolve &F, double *y, int *s_levptr, int cap_levptr, int *s_meta,
                            int meta_cap, const Ring &R) {
  const bool lev_in_smem = F.nlev + 1 <= cap_levptr;
  const bool meta_in_smem = F.nslots + 1 <= meta_cap;
  if (R.cap > 0 && lev_in_smem && meta_in_smem && blockDim.x >= 64) {
    __syncthreads();
    for (int i = threadIdx.x; i <= F.nlev; i += blockDim.x) s_levptr[i] = F.lev_ptr[i];
    for (int i = threadIdx.x; i < F.nslots; i += blockDim.x) s_meta[i] = F.rows[i];
    for (int i = threadIdx.x; i <= F.nslots; i += blockDim.x) s_meta[meta_cap + i] = F.eptr[i];
    __syncthreads();
    level_solve_staged(F, R);
    return;
  }
  if (F.group == 4)
    level_solve_g<4>(F, y, s_levptr, cap_levptr, s_meta, meta_cap);
  else if (F.group == 8)
    level_solve_g<8>(F, y, s_levptr, cap_levptr, s_meta, meta_cap);
  else if (F.group == 16)
    level_solve_g<16>(F, y, s_levptr, cap_levptr, s_meta, meta_cap);
  else
    level_solve_g<32>(F, y, s_levptr, cap_levptr, s_meta, meta_cap);
}

// Head vector b (build_head_matrix, hpc_solve.py:811-829): the mean of the
// series potential over the D points of each discharge element side; one
// warp per row, lanes over the points.  Continuity rows are zero.
__global__ void rhs_reduce_kernel(Net net, const double *__restrict__ rhs_vals, const int *__restrict__ rhs_group,
                                  const Group *__restrict__ groups) {
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (g >= net.N) return;
  const SolveState *st = net.st + net.real_row[g];
  if (st->done || !st->solve_q) return;
  const int r = net.row_de[g];
  if (r < 0) {
    if (lane == 0) net.bvec[g] = net.bknown ? net.bknown[g] : 0.0;
    return;
  }
  const int D = net.D;
  const int e = net.de_ids[r];
  const double bk = net.bknown ? net.bknown[g] : 0.0;
  const Group g0 = groups[rhs_group[2 * r]];
  double s0 = 0.0;
  for (int k = lane; k < D; k += 32) s0 += rhs_vals[g0.out + k];
  s0 = warp_sum(s0);
  if (net.type[e] == 0) {
    const Group g1 = groups[rhs_group[2 * r + 1]];
    double s1 = 0.0;
    for (int k = lane; k < D; k += 32) s1 += rhs_vals[g1.out + k];
    s1 = warp_sum(s1);
    if (lane == 0) net.bvec[g] = ((s1 / D) / net.t[net.frac1[e]] - (s0 / D) / net.t[net.frac0[e]]) + bk;
  } else if (lane == 0) {
    net.bvec[g] = (net.phi[e] - s0 / D) + bk;
  }
}

// Dense trailing block of the factors (the last K pivot steps, where the LU
// of a minimum-degree order fills in): column-major K x K, solved in panels of
// 32 rows.  One warp solves the panel's triangle with its 32 rows in
// registers (shuffle broadcast of each solved value), then the whole CTA
// updates the rows below (lower) / above (upper) with coalesced column reads.
// One panel's contribution to row i of a dense tail: sum_j<nb M(i, r0 + j) p_j
// (col points at M(i, r0), column-major), all nb loads issued first.
__device__ __forceinline__ double panel_dot(const double *__restrict__ col, int K, const double *pv, int nb) {
  double v[32];
#pragma unroll
  for (int j = 0; j < 32; j++) v[j] = (j < nb) ? __ldg(col + (size_t)j * K) : 0.0;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
  for (int j = 0; j < 32; j += 4) {
    a0 = fma(v[j], pv[j], a0);
    a1 = fma(v[j + 1], pv[j + 1], a1);
    a2 = fma(v[j + 2], pv[j + 2], a2);
    a3 = fma(v[j + 3], pv[j + 3], a3);
  }
  return (a0 + a1) + (a2 + a3);
}

// The panels are pipelined: after the barrier that publishes panel p, warp 0
// first updates the 32 rows of the next panel and goes straight on to that
// panel's triangle, while the other warps update the remaining rows with
// panel p; one barrier per panel.  The solved panel values go to a
// double-buffered shared array (zero padded), so a warp still reading panel p
// never sees panel p + 1.
__device__ void dense_lower_solve(const double *__restrict__ Lcm, int K, double *y) {
  __shared__ double s_pan[2][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, bd = blockDim.x;
  const int npan = (K + 31) / 32;
  for (int p = 0; p < npan; p++) {
    const int r0 = p * 32, nb = min(32, K - r0);
    if (warp == 0) {
      double row[32];
#pragma unroll
      for (int j = 0; j < 32; j++)
        row[j] = (lane < nb && j < lane) ? __ldg(Lcm + (size_t)(r0 + j) * K + r0 + lane) : 0.0;
      double yi = (lane < nb) ? y[r0 + lane] : 0.0;
#pragma unroll
      for (int j = 0; j < 32; j++) {
        const double yj = __shfl_sync(0xffffffffu, yi, j);
        if (lane > j) yi = fma(-row[j], yj, yi);
      }
      if (lane < nb) y[r0 + lane] = yi;
      s_pan[p & 1][lane] = (lane < nb) ? yi : 0.0;
    }
    __syncthreads();
    const double *pv = s_pan[p & 1];
    if (warp == 0) {
      const int i = r0 + 32 + lane;
      if (i < K) y[i] -= panel_dot(Lcm + (size_t)r0 * K + i, K, pv, nb);
      if (bd == 32)
        for (int k = r0 + 64 + lane; k < K; k += 32) y[k] -= panel_dot(Lcm + (size_t)r0 * K + k, K, pv, nb);
      __syncwarp();
    } else {
      for (int i = r0 + 64 + threadIdx.x - 32; i < K; i += bd - 32)
        y[i] -= panel_dot(Lcm + (size_t)r0 * K + i, K, pv, nb);
    }
  }
  __syncthreads();
}

__device__ void dense_upper_solve(const double *__restrict__ Ucm, const double *__restrict__ uinv, int K, double *y) {
  __shared__ double s_pan[2][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, bd = blockDim.x;
  const int npan = (K + 31) / 32;
  for (int p = npan - 1; p >= 0; p--) {
    const int r0 = p * 32, nb = min(32, K - r0);
    if (warp == 0) {
      double row[32];
#pragma unroll
      for (int j = 0; j < 32; j++)
        row[j] = (lane < nb && j > lane && j < nb) ? __ldg(Ucm + (size_t)(r0 + j) * K + r0 + lane) : 0.0;
      const double di = (lane < nb) ? __ldg(uinv + r0 + lane) : 0.0;
      double yi = (lane < nb) ? y[r0 + lane] : 0.0;
#pragma unroll
      for (int j = 31; j >= 0; j--) {
        if (lane == j) yi *= di;
        const double xj = __shfl_sync(0xffffffffu, yi, j);
        if (lane < j) yi = fma(-row[j], xj, yi);
      }
      if (lane < nb) y[r0 + lane] = yi;
      s_pan[p & 1][lane] = (lane < nb) ? yi : 0.0;
    }
    __syncthreads();
    const double *pv = s_pan[p & 1];
    if (warp == 0) {
      if (p > 0) {
        const int i = r0 - 32 + lane;
        y[i] -= panel_dot(Ucm + (size_t)r0 * K + i, K, pv, nb);
      }
      if (bd == 32)
        for (int k = lane; k < r0 - 32; k += 32) y[k] -= panel_dot(Ucm + (size_t)r0 * K + k, K, pv, nb);
      __syncwarp();
    } else {
      for (int i = threadIdx.x - 32; i < r0 - 32; i += bd - 32) y[i] -= panel_dot(Ucm + (size_t)r0 * K + i, K, pv, nb);
    }
  }
  __syncthreads();
}

namespace cg = cooperative_groups;

// W = U^-1 L^-1 of a dense tail (L unit lower, U upper with 1/U(i,i) in
// uinv, both K x K column-major), column-major: the blocked solve of
// L U W = I.  A CTA takes nc (<= 16) columns of W and keeps them in shared
// memory (row-major [K][nc]); forward substitution with L and backward
// substitution with U go panel by panel (32 rows): a warp solves a panel's
// triangle for one column, then the CTA subtracts the panel from the rows
// below (L) or above (U).  Computed once per factorisation.
static constexpr int DINV_NC = 16;
static constexpr int CLUSTER_MIN_K = 256;  // dense tails this large use the cluster path

__global__ void __launch_bounds__(256) dense_inverse_kernel(const double *__restrict__ L, const double *__restrict__ U,
                                                            const double *__restrict__ uinv, int K, int nc,
                                                            double *__restrict__ W) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *X = reinterpret_cast<double *>(smem_raw);
  const int c0 = blockIdx.x * nc;
  const int ncl = min(nc, K - c0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int idx = threadIdx.x; idx < K * nc; idx += blockDim.x) {
    const int i = idx / nc, c = idx - i * nc;
    X[idx] = (c < ncl && i == c0 + c) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int r0 = (c0 / 32) * 32; r0 < K; r0 += 32) {
    const int nb = min(32, K - r0);
    double row[32];
#pragma unroll
    for (int j = 0; j < 32; j++) row[j] = (lane < nb && j < lane) ? L[(size_t)(r0 + j) * K + r0 + lane] : 0.0;
    for (int c = warp; c < ncl; c += nw) {
      double x = (lane < nb) ? X[(r0 + lane) * nc + c] : 0.0;
#pragma unroll
      for (int j = 0; j < 32; j++) {
        const double xj = __shfl_sync(0xffffffffu, x, j);
        if (lane > j) x = fma(-row[j], xj, x);
      }
      if (lane < nb) X[(r0 + lane) * nc + c] = x;
    }
    __syncthreads();
    for (int i = r0 + nb + threadIdx.x; i < K; i += blockDim.x) {
      double acc[DINV_NC];
#pragma unroll
      for (int c = 0; c < DINV_NC; c++) acc[c] = 0.0;
#pragma unroll 8
      for (int j = 0; j < nb; j++) {  // eight L loads in flight
        const double l = L[(size_t)(r0 + j) * K + i];
        const double *xr = X + (r0 + j) * nc;
#pragma unroll
        for (int c = 0; c < DINV_NC; c++)
          if (c < ncl) acc[c] = fma(l, xr[c], acc[c]);
      }
#pragma unroll
      for (int c = 0; c < DINV_NC; c++)
        if (c < ncl) X[i * nc + c] -= acc[c];
    }
    __syncthreads();
  }
  for (int p = (K + 31) / 32 - 1; p >= 0; p--) {
    const int r0 = p * 32, nb = min(32, K - r0);
    double row[32];
#pragma unroll
    for (int j = 0; j < 32; j++) row[j] = (lane < nb && j > lane && j < nb) ? U[(size_t)(r0 + j) * K + r0 + lane] : 0.0;
    const double di = (lane < nb) ? uinv[r0 + lane] : 0.0;
    for (int c = warp; c < ncl; c += nw) {
      double x = (lane < nb) ? X[(r0 + lane) * nc + c] : 0.0;
#pragma unroll
      for (int j = 31; j >= 0; j--) {
        if (lane == j) x *= di;
        const double xj = __shfl_sync(0xffffffffu, x, j);
        if (lane < j) x = fma(-row[j], xj, x);
      }
      if (lane < nb) X[(r0 + lane) * nc + c] = x;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < r0; i += blockDim.x) {
      double acc[DINV_NC];
#pragma unroll
      for (int c = 0; c < DINV_NC; c++) acc[c] = 0.0;
#pragma unroll 8
      for (int j = 0; j < nb; j++) {  // eight U loads in flight
        const double u = U[(size_t)(r0 + j) * K + i];
        const double *xr = X + (r0 + j) * nc;
#pragma unroll
        for (int c = 0; c < DINV_NC; c++)
          if (c < ncl) acc[c] = fma(u, xr[c], acc[c]);
      }
#pragma unroll
      for (int c = 0; c < DINV_NC; c++)
        if (c < ncl) X[i * nc + c] -= acc[c];
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < K * ncl; idx += blockDim.x) {
    const int c = idx / K, i = idx - c * K;
    W[(size_t)(c0 + c) * K + i] = X[i * nc + c];
  }
}

// ---------------------------------------------------------------------------
// The same W = U^-1 L^-1 by blocks of DINVB = 64 rows, GEMM-rich: the
// per-column kernel above streams all of L and U through every CTA (2.9 GB
// of L2 reads for K = 1,535, 2.6 TFLOP/s).  W (column-major, ld K) starts as
// the identity; then
//   forward, block i = 0, 1, ...: Y_i := L_ii^-1 Y_i on the columns up to
//     the block's end (Y = L^-1 is lower triangular), then
//     Y_below -= L_below,i Y_i (a GEMM with inner dimension 64);
//   backward, block i = last, ..., 0: W_i := U_ii^-1 W_i on every column,
//     then W_above -= U_above,i W_i.
static constexpr int DINVB = 64;

// Y[r0 .. r0+nb, c] := T^-1 Y[r0 .. r0+nb, c] for the columns c < ncols, T
// the diagonal block of LU (unit lower, or upper scaled by uinv): a warp per
// column, lane l holding rows l and l + 32, the solved value of each row
// broadcast by a shuffle (a thread per column ran each column as one chain
// of 2,016 dependent products, 29-86 us a block); the block is staged in
// shared memory, zero outside nb (rows past nb stay zero).
template <bool LOWER>
__global__ void __launch_bounds__(256) dinvb_diag_kernel(const double *__restrict__ LU,
                                                         const double *__restrict__ uinv, int K, int r0, int nb,
                                                         int ncols, double *__restrict__ W) {
  __shared__ double T[DINVB][DINVB + 1];  // T[row][col] of the diagonal block
  __shared__ double di[DINVB];
  for (int idx = threadIdx.x; idx < DINVB * DINVB; idx += blockDim.x) {
    const int c = idx / DINVB, r = idx - c * DINVB;
    T[r][c] = (r < nb && c < nb) ? LU[(size_t)(r0 + c) * K + r0 + r] : 0.0;
  }
  for (int r = threadIdx.x; r < DINVB; r += blockDim.x) di[r] = (LOWER || r >= nb) ? 1.0 : uinv[r0 + r];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (c >= ncols) return;  // uniform over the warp
  double *w = W + (size_t)c * K + r0;
  double x0 = (lane < nb) ? w[lane] : 0.0, x1 = (lane + 32 < nb) ? w[lane + 32] : 0.0;
  if (LOWER) {
    for (int j = 0; j < 32; j++) {
      const double xj = __shfl_sync(0xffffffffu, x0, j);
      if (lane > j) x0 = fma(-T[lane][j], xj, x0);
      x1 = fma(-T[lane + 32][j], xj, x1);
    }
    for (int j = 0; j < 32; j++) {
      const double xj = __shfl_sync(0xffffffffu, x1, j);
      if (lane > j) x1 = fma(-T[lane + 32][j + 32], xj, x1);
    }
  } else {
    for (int j = 31; j >= 0; j--) {
      if (lane == j) x1 *= di[j + 32];
      const double xj = __shfl_sync(0xffffffffu, x1, j);
      if (lane < j) x1 = fma(-T[lane + 32][j + 32], xj, x1);
      x0 = fma(-T[lane][j + 32], xj, x0);
    }
    for (int j = 31; j >= 0; j--) {
      if (lane == j) x0 *= di[j];
      const double xj = __shfl_sync(0xffffffffu, x0, j);
      if (lane < j) x0 = fma(-T[lane][j], xj, x0);
    }
  }
  if (lane < nb) w[lane] = x0;
  if (lane + 32 < nb) w[lane + 32] = x1;
}

// C[m0 .. m0+M, 0 .. N) -= A[m0 .. m0+M, k0 .. k0+kb) B[k0 .. k0+kb, 0 .. N),
// all column-major with leading dimension K (A a block column of L or U,
// B and C rows of W): 64 x 64 tiles, 16 x 16 threads with 4 x 4 outputs.
__global__ void __launch_bounds__(256, 3) dinvb_gemm_kernel(const double *__restrict__ A, double *__restrict__ W, int K,
                                                         int m0, int M, int k0, int kb, int N) {
  __shared__ double As[16][64], Bs[16][65];
  const int rb = blockIdx.x * 64, cb = blockIdx.y * 64;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[r][q] = 0.0;
  // a k step's tiles are loaded into registers while the step before it
  // computes (4 entries of A and 4 of B a thread), then stored to shared
  // memory: A's rows contiguous in a column, B's 16 k of a column together
  double la[4], lb[4];
  auto load_step = [&](int kk0) {
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int idx = threadIdx.x + 256 * u;
      const int kk = idx >> 6, i = idx & 63;
      la[u] = (kk0 + kk < kb && rb + i < M) ? A[(size_t)(k0 + kk0 + kk) * K + m0 + rb + i] : 0.0;
      const int c = idx >> 4, k2 = idx & 15;
      lb[u] = (kk0 + k2 < kb && cb + c < N) ? W[(size_t)(cb + c) * K + k0 + kk0 + k2] : 0.0;
    }
  };
  load_step(0);
  for (int kk0 = 0; kk0 < kb; kk0 += 16) {
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int idx = threadIdx.x + 256 * u;
      As[idx >> 6][idx & 63] = la[u];
      Bs[idx & 15][idx >> 4] = lb[u];
    }
    __syncthreads();
    if (kk0 + 16 < kb) load_step(kk0 + 16);
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      double a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; r++) a[r] = As[kk][tx + 16 * r];
#pragma unroll
      for (int q = 0; q < 4; q++) b[q] = Bs[kk][ty + 16 * q];
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[r][q] = fma(a[r], b[q], acc[r][q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int c = cb + ty + 16 * q;
    if (c >= N) continue;
    double *col = W + (size_t)c * K + m0;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int i = rb + tx + 16 * r;
      if (i < M) col[i] -= acc[r][q];
    }
  }
}

__global__ void identity_kernel(double *__restrict__ W, int K) {
  const size_t n = (size_t)K * K;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t c = i / K, r = i - c * K;
    W[i] = (r == c) ? 1.0 : 0.0;
  }
}

// out = in^T for K x K column-major matrices.
__global__ void transpose_kernel(const double *__restrict__ in, double *__restrict__ out, int K) {
  __shared__ double tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = bx + threadIdx.x, c = by + k;
    if (r < K && c < K) tile[k][threadIdx.x] = in[(size_t)c * K + r];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = by + threadIdx.x, c = bx + k;
    if (r < K && c < K) out[(size_t)c * K + r] = tile[threadIdx.x][k];
  }
}

// Dense-tail factors of the adjoint from the forward ones (one K x K
// column-major matrix holding L strictly below and U on and above the
// diagonal): out(i, j) = S(j, i) / U(j, j) below the diagonal ((D^-1 U)^T),
// S(j, i) above it (L^T), 0 on it.
__global__ void adj_tail_kernel(const double *__restrict__ S, const double *__restrict__ uinv, int K,
                                double *__restrict__ out) {
  __shared__ double tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = bx + threadIdx.x, c = by + k;
    if (r < K && c < K) tile[k][threadIdx.x] = S[(size_t)c * K + r];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int i = by + threadIdx.x, j = bx + k;
    if (i < K && j < K) {
      const double v = tile[threadIdx.x][k];
      out[(size_t)j * K + i] = (i > j) ? v * uinv[j] : (i < j ? v : 0.0);
    }
  }
}

// ---------------------------------------------------------------------------
// Dense LU of the Schur complement on the device (right-looking, partial
// pivoting, panels of DLU_NB columns), in place on a K x K column-major
// matrix: unit lower L below the diagonal, U on and above it, the pivot rule
// of the host factorisation (largest magnitude, first row on a tie).  Per
// panel: the panel kernel factorises the panel columns (one CTA; the panel's
// rows in shared memory when they fit), the update kernel applies the
// panel's row interchanges to every other column and solves U12 = L11^-1 A12,
// the GEMM kernel updates the trailing block A22 -= L21 U12.
static constexpr int DLU_NB = 16;
static constexpr int DLU_THREADS = 1024;
static constexpr int DLU_MIN_K = 64;
static constexpr int DLU_MAX_K = 16384;  // int panel indices: K * DLU_NB + K < 2^31
static constexpr size_t DLU_SMEM_MAX = 220 * 1024;

struct DluScratch {
  int *piv;       // [K] block row swapped with row j at step j
  double *diag;   // [K] U(j, j)
  int *swap_src;  // [2][2 DLU_NB] composite interchange of a panel (slot = panel
  int *swap_dst;  //   parity in the one-launch LU, slot 0 otherwise): row
  int *swap_cnt;  // [2]  swap_dst[k] receives the old row swap_src[k]
  int *flag;      // [1] first zero / non-finite pivot column + 1 (0 = none)
};

// Panel element (i, c) (rows from j0, columns from j0): shared memory
// row-major with a padded row, or the matrix itself (column-major).
template <bool SMEM>
__device__ __forceinline__ int dlu_at(int i, int c, int K) {
  return SMEM ? i * (DLU_NB + 1) + c : i + c * K;
}

// The interchanges of a panel (position j0 + jj swapped with j0 + s_piv[jj],
// jj in order) as one permutation of at most 2 nb rows, by one warp: lane k
// holds slot k (its row, and the row whose old content it gets).
__device__ void dlu_compose_swaps(const int *s_piv, int j0, int nb, int *dst, int *src, int *cnt_out) {
  const int lane = threadIdx.x & 31;
  __syncwarp();
  int row = -1, org = -1, cnt = 0;
  for (int jj = 0; jj < nb; jj++) {
    const int a = j0 + jj, b = j0 + s_piv[jj];
    if (a == b) continue;
    int ka, kb;
    const unsigned ma = __ballot_sync(0xffffffffu, row == a);
    if (ma) {
      ka = __ffs(ma) - 1;
    } else {
      ka = cnt++;
      if (lane == ka) row = org = a;
    }
    const unsigned mb = __ballot_sync(0xffffffffu, row == b);
    if (mb) {
      kb = __ffs(mb) - 1;
    } else {
      kb = cnt++;
      if (lane == kb) row = org = b;
    }
    const int oa = __shfl_sync(0xffffffffu, org, ka), ob = __shfl_sync(0xffffffffu, org, kb);
    if (lane == ka) org = ob;
    if (lane == kb) org = oa;
  }
  if (lane < cnt) {
    dst[lane] = row;
    src[lane] = org;
  }
  if (lane == 0) *cnt_out = cnt;
}

template <bool SMEM>
__global__ void __launch_bounds__(DLU_THREADS) dlu_panel_kernel(double *__restrict__ S, int K, int j0, int nb,
                                                                DluScratch D) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double s_wv[32];
  __shared__ int s_wi[32];
  __shared__ int s_piv[DLU_NB];
  const int tid = threadIdx.x, bd = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = bd >> 5;
  const int m = K - j0;
  double *const Sp = S + (size_t)j0 * K + j0;
  double *P;
  if (SMEM) {
    P = reinterpret_cast<double *>(smem_raw);
    for (int i = tid; i < m; i += bd) {  // a row's columns loaded together
      double v[DLU_NB];
#pragma unroll
      for (int c = 0; c < DLU_NB; c++) v[c] = (c < nb) ? Sp[i + c * K] : 0.0;
#pragma unroll
      for (int c = 0; c < DLU_NB; c++)
        if (c < nb) P[dlu_at<true>(i, c, K)] = v[c];
    }
    __syncthreads();
  } else {
    P = Sp;
  }
  for (int jj = 0; jj < nb; jj++) {
    double best = -1.0;
    int bi = m;
    int bad = 0;
    for (int i = jj + tid; i < m; i += bd) {
      const double v = fabs(P[dlu_at<SMEM>(i, jj, K)]);
      if (!(v <= DBL_MAX)) bad = 1;
      if (v > best) {
        best = v;
        bi = i;
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_down_sync(0xffffffffu, best, off);
      const int oi = __shfl_down_sync(0xffffffffu, bi, off);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if (lane == 0) {
      s_wv[warp] = best;
      s_wi[warp] = bi;
    }
    bad = __syncthreads_or(bad);
    if (warp == 0) {
      best = (lane < nw) ? s_wv[lane] : -1.0;
      bi = (lane < nw) ? s_wi[lane] : m;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, best, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ov > best || (ov == best && oi < bi)) {
          best = ov;
          bi = oi;
        }
      }
      if (lane == 0) {
        if (bi >= m) bi = jj;  // every entry NaN: keep the diagonal, flagged below
        s_piv[jj] = bi;
        D.piv[j0 + jj] = j0 + bi;
        if ((bad || !(best > 0.0)) && *D.flag == 0) *D.flag = j0 + jj + 1;
      }
    }
    __syncthreads();
    const int p = s_piv[jj];
    if (p != jj && tid < nb) {
      const double a = P[dlu_at<SMEM>(jj, tid, K)], b = P[dlu_at<SMEM>(p, tid, K)];
      P[dlu_at<SMEM>(jj, tid, K)] = b;
      P[dlu_at<SMEM>(p, tid, K)] = a;
    }
    __syncthreads();
    const double piv = P[dlu_at<SMEM>(jj, jj, K)];
    if (tid == 0) D.diag[j0 + jj] = piv;
    const double inv = (piv != 0.0) ? 1.0 / piv : 0.0;
    for (int i = jj + 1 + tid; i < m; i += bd) {
      const double l = P[dlu_at<SMEM>(i, jj, K)] * inv;
      P[dlu_at<SMEM>(i, jj, K)] = l;
      for (int c = jj + 1; c < nb; c++) P[dlu_at<SMEM>(i, c, K)] = fma(-l, P[dlu_at<SMEM>(jj, c, K)], P[dlu_at<SMEM>(i, c, K)]);
    }
    __syncthreads();
  }
  if (SMEM) {
    for (int c = 0; c < nb; c++)
      for (int i = tid; i < m; i += bd) Sp[i + c * K] = P[dlu_at<true>(i, c, K)];
  }
  if (warp == 0) dlu_compose_swaps(s_piv, j0, nb, D.swap_dst, D.swap_src, D.swap_cnt);
}

// One warp per column outside the panel: the panel's interchanges, then for
// the trailing columns U12 = L11^-1 A12 (unit lower triangle of the panel).
__global__ void __launch_bounds__(256) dlu_update_kernel(double *__restrict__ S, int K, int j0, int nb, DluScratch D) {
  __shared__ double L11[DLU_NB][DLU_NB + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int c = idx / nb, r = idx - c * nb;
    L11[r][c] = (r > c) ? S[(size_t)(j0 + c) * K + j0 + r] : 0.0;
  }
  __syncthreads();
  const int cidx = blockIdx.x * (blockDim.x >> 5) + warp;
  if (cidx >= K - nb) return;
  const int c = (cidx < j0) ? cidx : cidx + nb;
  double *col = S + (size_t)c * K;
  const int cnt = *D.swap_cnt;
  double v = 0.0;
  if (lane < cnt) v = col[D.swap_src[lane]];
  __syncwarp();
  if (lane < cnt) col[D.swap_dst[lane]] = v;
  __syncwarp();
  if (c < j0 + nb) return;
  double x = (lane < nb) ? col[j0 + lane] : 0.0;
#pragma unroll
  for (int j = 0; j < DLU_NB; j++) {
    const double xj = __shfl_sync(0xffffffffu, x, j);
    if (lane > j && lane < nb) x = fma(-L11[lane][j], xj, x);
  }
  if (lane < nb) col[j0 + lane] = x;
}

// A22 -= L21 U12 over 64 x 64 tiles of the trailing block (4 x 4 outputs a
// thread; the thread's rows are 16 apart so the column-major stores coalesce).
__global__ void __launch_bounds__(256) dlu_gemm_kernel(double *__restrict__ S, int K, int j0, int nb) {
  __shared__ double As[DLU_NB][64], Bs[DLU_NB][65];
  const int c0 = j0 + nb, m = K - c0;
  const int rb = blockIdx.x * 64, cb = blockIdx.y * 64;
  for (int idx = threadIdx.x; idx < DLU_NB * 64; idx += blockDim.x) {
    const int k = idx / 64, i = idx - k * 64;
    As[k][i] = (k < nb && rb + i < m) ? S[(size_t)(j0 + k) * K + c0 + rb + i] : 0.0;
    const int c = idx / DLU_NB, kk = idx - c * DLU_NB;
    Bs[kk][c] = (kk < nb && cb + c < m) ? S[(size_t)(c0 + cb + c) * K + j0 + kk] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[r][q] = 0.0;
#pragma unroll
  for (int k = 0; k < DLU_NB; k++) {
    double a[4], b[4];
#pragma unroll
    for (int r = 0; r < 4; r++) a[r] = As[k][tx + 16 * r];
#pragma unroll
    for (int q = 0; q < 4; q++) b[q] = Bs[k][ty + 16 * q];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[r][q] = fma(a[r], b[q], acc[r][q]);
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int c = cb + ty + 16 * q;
    if (c >= m) continue;
    double *col = S + (size_t)(c0 + c) * K + c0;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int i = rb + tx + 16 * r;
      if (i < m) col[i] -= acc[r][q];
    }
  }
}

// ---------------------------------------------------------------------------
// The same dense LU in one cooperative launch with a look-ahead of one panel:
// one grid barrier a panel step instead of three kernel launches, and CTA 0
// factorises panel k+1 while the other CTAs are still applying panel k to
// the rest of the trailing block.
//   phase S(k)  all CTAs, a warp per column outside panel k: the panel's row
//               interchanges, then U12 = L11^-1 A12 (as dlu_update_kernel);
//               panel k+1's columns are CTA 0's; every trailing column done
//               bumps the counter of its 16-column block;
//   phase P(k+1) CTA 0 at once: the update A22 -= L21 U12 of panel k+1's
//               columns (as dlu_gemm_kernel) straight into shared memory,
//               then the panel factorisation (as dlu_panel_kernel, the pivot
//               search of a column fused with the update by the column
//               before, the rows left in place);
//   phase G(k)  the other CTAs: A22 -= L21 U12 for the other columns in
//               items of DLUC_TR rows x DLU_NB columns, each item once its
//               column block's counter shows S(k) done there;
//   barrier.
// Every product, quotient and fused multiply-add is the one the three-kernel
// path computes, in the same order, so the factors are the same bit for bit.
// Waits are bounded: a barrier or the counter wait that runs out sets
// DluSync::err and every CTA returns at its next barrier.
static constexpr int DLUC_THREADS = 512;
static constexpr int DLUC_TR = 128;                 // rows of a G item
static constexpr unsigned DLUC_SPIN_LIMIT = 1u << 24;  // polls of a wait (>= 1 s with the sleeps)

// dynamic shared memory of dlu_coop_kernel for a K x K block
static size_t dluc_smem(int K) {
  return sizeof(double) * (DLU_NB + 1) * (size_t)std::max(K, DLUC_TR + 2 * DLU_NB);
}

struct DluSync {
  unsigned count;  // CTAs arrived at the current barrier
  unsigned gen;    // barrier generation
  int err;         // a wait ran out
};

__device__ __forceinline__ bool dluc_barrier(DluSync *sy, unsigned nblocks) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *gen = &sy->gen;
    volatile int *err = &sy->err;
    int ok = 1;
    const unsigned g = *gen;
    __threadfence();
    if (atomicAdd(&sy->count, 1u) == nblocks - 1) {
      atomicExch(&sy->count, 0u);
      __threadfence();
      atomicAdd(&sy->gen, 1u);
    } else {
      unsigned it = 0;
      while (*gen == g) {
        if (*err || ++it > DLUC_SPIN_LIMIT) {
          atomicExch(&sy->err, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = ok && !*err;
  }
  __syncthreads();
  return s_ok != 0;
}

// Rows of the panel a thread of dlu_coop_kernel holds: i = tid + r DLUC_THREADS.
static constexpr int DLUC_ROWS = 4;
static_assert(DLU_SMEM_MAX / (sizeof(double) * (DLU_NB + 1)) <= (size_t)DLUC_ROWS * DLUC_THREADS,
              "a panel of the one-launch LU has at most DLUC_ROWS rows a thread");
static_assert(DLUC_THREADS / 32 >= DLU_NB, "CTA 0's warps take the next panel's columns in phase S");

// Loads the panel (columns j0 .. j0+nb-1, rows j0 .. K-1) into shared memory
// P (row-major, padded rows) with L2 loads (other CTAs wrote it).
__device__ void dluc_panel_load(const double *__restrict__ S, int K, int j0, int nb, double *P) {
  const int m = K - j0;
  const double *const Sp = S + (size_t)j0 * K + j0;
  for (int i = threadIdx.x; i < m; i += DLUC_THREADS) {
    double v[DLU_NB];
#pragma unroll
    for (int c = 0; c < DLU_NB; c++) v[c] = (c < nb) ? __ldcg(Sp + i + (size_t)c * K) : 0.0;
#pragma unroll
    for (int c = 0; c < DLU_NB; c++)
      if (c < nb) P[i * (DLU_NB + 1) + c] = v[c];
  }
  __syncthreads();
}

// Warp argmax of (key, position): the largest key, the smallest position on
// a tie (key 0: no candidate); returns the winning lane.  Three redux
// instructions and a ballot instead of a shuffle tree.
__device__ __forceinline__ int dluc_warp_argmax(unsigned long long key, int pos) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  const bool top = hi == mhi && lo == mlo;
  const unsigned mpos = __reduce_min_sync(0xffffffffu, top ? (unsigned)pos : 0xffffffffu);
  return __ffs(__ballot_sync(0xffffffffu, top && (unsigned)pos == mpos)) - 1;
}

// Argmax key of a candidate magnitude v >= 0 (the bits of a non-negative
// double order as the values do); none (v < 0) is 0.
__device__ __forceinline__ unsigned long long dluc_key(double v) {
  return (v >= 0.0) ? (unsigned long long)__double_as_longlong(v) + 1ull : 0ull;
}

// Columns c0+1 .. nb-1 of a row update by the pivot row (distinct rows of
// P); column c0 < nb is updated first and returned (the next candidate).
__device__ __forceinline__ double dluc_row_update(double *__restrict__ Pi, const double *__restrict__ Pq, double l,
                                                  int c0, int nb) {
  double x0 = 0.0;
  if (c0 < nb) {
    x0 = fma(-l, Pq[c0], Pi[c0]);
    Pi[c0] = x0;
  }
#pragma unroll 4
  for (int c = c0 + 1; c < nb; c++) Pi[c] = fma(-l, Pq[c], Pi[c]);
  return x0;
}

// Panel factorisation of the panel in P (m = K - j0 rows) by one CTA.  The
// rows do not move: a thread keeps the positions of its rows in registers
// (position = the row's index after the interchanges so far), the pivot row
// of column jj takes position jj and the row that held position jj takes the
// pivot's old position, exactly the interchange of the row-swapping form.
// The pivot is the largest magnitude, the smallest position on a tie, and
// every quotient and fused multiply-add is the row-swapping form's, so the
// factors are the same bit for bit.  A column: each warp's argmax, a block
// barrier, warp 0's argmax over the warps and the one division, a block
// barrier (the warps' candidates are double-buffered by column parity).
// Stores the panel back in position order and writes the pivots, U's
// diagonal, the bad-pivot flag and the composite interchange (slot par).
__device__ void dluc_panel_factor(double *__restrict__ S, int K, int j0, int nb, const DluScratch &D, double *P,
                                  int par) {
  __shared__ unsigned long long s_wk[2][DLUC_THREADS / 32];
  __shared__ double s_wv[2][DLUC_THREADS / 32];
  __shared__ int s_wp[2][DLUC_THREADS / 32];
  __shared__ int s_wq[2][DLUC_THREADS / 32];
  __shared__ int s_bad[2][DLUC_THREADS / 32];
  __shared__ int s_piv[DLU_NB];
  __shared__ int s_p, s_q, s_found;
  __shared__ double s_inv;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = DLUC_THREADS / 32;
  const int m = K - j0;
  int pos[DLUC_ROWS];
  unsigned done = 0;  // bit r: the thread's row r is a pivot row
#pragma unroll
  for (int r = 0; r < DLUC_ROWS; r++) pos[r] = tid + r * DLUC_THREADS;
  // candidate of column 0 (rows in position order): magnitude, position,
  // row, signed value
  double best = -1.0, bval = 0.0;
  int bp = m, bq = m, bad = 0;
#pragma unroll
  for (int r = 0; r < DLUC_ROWS; r++) {
    const int i = tid + r * DLUC_THREADS;
    if (i < m) {
      const double x = P[i * (DLU_NB + 1)], v = fabs(x);
      if (!(v <= DBL_MAX)) bad = 1;
      if (v > best) {
        best = v;
        bp = i;
        bq = i;
        bval = x;
      }
    }
  }
  for (int jj = 0; jj < nb; jj++) {
    // block argmax of column jj: each warp's, then warp 0's over the warps
    const int pb = jj & 1;
    {
      const unsigned long long key = dluc_key(best);
      const int wl = dluc_warp_argmax(key, bp);
      bad = __any_sync(0xffffffffu, bad);
      if (lane == wl) {
        s_wk[pb][warp] = key;
        s_wp[pb][warp] = bp;
        s_wq[pb][warp] = bq;
        s_wv[pb][warp] = bval;
      }
      if (lane == 0) s_bad[pb][warp] = bad;
    }
    __syncthreads();  // also: every thread's update by column jj - 1 is done
    if (warp == 0) {
      const unsigned long long k2 = (lane < NW) ? s_wk[pb][lane] : 0ull;
      const int p2 = (lane < NW) ? s_wp[pb][lane] : m;
      const int bad2 = __any_sync(0xffffffffu, (lane < NW) ? s_bad[pb][lane] : 0);
      const int wl2 = dluc_warp_argmax(k2, p2);
      if (lane == wl2) {
        const bool found = k2 != 0ull;
        const double piv = s_wv[pb][lane];
        s_found = found;
        if (found) {
          s_p = p2;
          s_q = s_wq[pb][lane];
          s_inv = (piv != 0.0) ? 1.0 / piv : 0.0;
          s_piv[jj] = p2;
          D.piv[j0 + jj] = j0 + p2;
          D.diag[j0 + jj] = piv;
        }
        if ((bad2 || !found || !(fabs(piv) > 0.0)) && *D.flag == 0) *D.flag = j0 + jj + 1;
      }
    }
    __syncthreads();
    int p, q;
    double inv;
    if (s_found) {
      p = s_p;
      q = s_q;
      inv = s_inv;
    } else {
      // every entry NaN: the row at position jj stays (flagged above); its
      // holder names it (the same branch in every thread)
      p = jj;
#pragma unroll
      for (int r = 0; r < DLUC_ROWS; r++) {
        const int i = tid + r * DLUC_THREADS;
        if (i < m && !((done >> r) & 1u) && pos[r] == jj) s_q = i;
      }
      __syncthreads();
      q = s_q;
      const double piv = P[q * (DLU_NB + 1) + jj];
      inv = (piv != 0.0) ? 1.0 / piv : 0.0;
      if (tid == 0) {
        s_piv[jj] = p;
        D.piv[j0 + jj] = j0 + p;
        D.diag[j0 + jj] = piv;
      }
    }
    const double *const Pq = P + q * (DLU_NB + 1);
    // the interchange, in positions
#pragma unroll
    for (int r = 0; r < DLUC_ROWS; r++) {
      const int i = tid + r * DLUC_THREADS;
      if (i == q) {
        done |= 1u << r;
        pos[r] = jj;
      } else if (!((done >> r) & 1u) && pos[r] == jj) {
        pos[r] = p;
      }
    }
    // update by column jj, and the candidate of column jj + 1
    best = -1.0;
    bval = 0.0;
    bp = m;
    bq = m;
    bad = 0;
    const int nx = jj + 1;
#pragma unroll
    for (int r = 0; r < DLUC_ROWS; r++) {
      const int i = tid + r * DLUC_THREADS;
      if (i >= m || ((done >> r) & 1u)) continue;
      double *Pi = P + i * (DLU_NB + 1);
      const double l = Pi[jj] * inv;
      Pi[jj] = l;
      const double x = dluc_row_update(Pi, Pq, l, nx, nb);
      if (nx < nb) {
        const double v = fabs(x);
        if (!(v <= DBL_MAX)) bad = 1;
        if (v > best || (v == best && pos[r] < bp)) {
          best = v;
          bp = pos[r];
          bq = i;
          bval = x;
        }
      }
    }
  }
  __syncthreads();  // the last column's updates are done
  double *const Sp = S + (size_t)j0 * K + j0;
#pragma unroll
  for (int r = 0; r < DLUC_ROWS; r++) {
    const int i = tid + r * DLUC_THREADS;
    if (i < m)
      for (int c = 0; c < nb; c++) Sp[pos[r] + (size_t)c * K] = P[i * (DLU_NB + 1) + c];
  }
  if (warp == 0)
    dlu_compose_swaps(s_piv, j0, nb, D.swap_dst + par * 2 * DLU_NB, D.swap_src + par * 2 * DLU_NB,
                      D.swap_cnt + par);
}

// CTA 0's part of G(k) for panel k+1's columns c0 .. c0+ncols-1 (their
// interchanges and U12 rows are done by its own warps in S(k)): the update
// A22 -= L21 U12 of their rows c0 .. K-1, each entry the fused multiply-add
// chain of a G item, written straight into the panel buffer P of P(k+1).
__device__ void dluc_next_panel(const double *__restrict__ S, int K, int j0, int c0, int ncols, double *P) {
  __shared__ __align__(16) double s_u12[DLU_NB][DLU_NB];
  const int mt = K - c0;
  for (int idx = threadIdx.x; idx < DLU_NB * DLU_NB; idx += DLUC_THREADS) {
    const int c = idx / DLU_NB, kk = idx - c * DLU_NB;
    s_u12[kk][c] = (c < ncols) ? __ldcg(S + (size_t)(c0 + c) * K + j0 + kk) : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.x; r < mt; r += DLUC_THREADS) {
    // the row's L21 entries issued together; kk outer over the accumulators
    // of a quarter of the columns (each still summed in kk order), U12 rows
    // read 16 bytes at a time; a quarter's old values are loaded before its
    // products
    double a[DLU_NB];
#pragma unroll
    for (int kk = 0; kk < DLU_NB; kk++) a[kk] = __ldcg(S + (size_t)(j0 + kk) * K + c0 + r);
#pragma unroll 1
    for (int h = 0; h < 4; h++) {
      constexpr int HC = DLU_NB / 4;
      double acc[HC], o[HC];
#pragma unroll
      for (int c = 0; c < HC; c++) {
        const int cc = h * HC + c;
        o[c] = (cc < ncols) ? __ldcg(S + (size_t)(c0 + cc) * K + c0 + r) : 0.0;
        acc[c] = 0.0;
      }
#pragma unroll
      for (int kk = 0; kk < DLU_NB; kk++) {
        const double2 *u2 = reinterpret_cast<const double2 *>(&s_u12[kk][h * HC]);
#pragma unroll
        for (int c2 = 0; c2 < HC / 2; c2++) {
          const double2 u = u2[c2];
          acc[2 * c2] = fma(a[kk], u.x, acc[2 * c2]);
          acc[2 * c2 + 1] = fma(a[kk], u.y, acc[2 * c2 + 1]);
        }
      }
#pragma unroll
      for (int c = 0; c < HC; c++) {
        const int cc = h * HC + c;
        if (cc < ncols) P[r * (DLU_NB + 1) + cc] = o[c] - acc[c];
      }
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(DLUC_THREADS, 1) dlu_coop_kernel(double *__restrict__ S, int K, DluScratch D,
                                                                   DluSync *sy, unsigned *__restrict__ colcnt) {
  // one dynamic buffer, used by one phase at a time: the panel (CTA 0), or
  // L11 (phase S), or an item's L21 rows and U12 block (phase G)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *const P = reinterpret_cast<double *>(smem_raw);
  double(*const s_l)[DLU_NB + 1] = reinterpret_cast<double(*)[DLU_NB + 1]>(P);
  double(*const s_u)[DLU_NB + 1] = reinterpret_cast<double(*)[DLU_NB + 1]>(P + DLUC_TR * (DLU_NB + 1));
  double(*const L11)[DLU_NB + 1] =
      reinterpret_cast<double(*)[DLU_NB + 1]>(P + (DLUC_TR + DLU_NB) * (DLU_NB + 1));
  const unsigned G = gridDim.x;
  const int cta = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = DLUC_THREADS / 32;
  const int np = (K + DLU_NB - 1) / DLU_NB;
  if (cta == 0) {
    dluc_panel_load(S, K, 0, min(DLU_NB, K), P);
    dluc_panel_factor(S, K, 0, min(DLU_NB, K), D, P, 0);
  }
  if (!dluc_barrier(sy, G)) return;
  for (int k = 0; k < np; k++) {
    const int j0 = k * DLU_NB, nb = min(DLU_NB, K - j0), c0 = j0 + nb, mt = K - c0;
    const int par = k & 1;
    // S(k): interchanges for every column outside the panel, U12 for the trailing ones
    for (int idx = threadIdx.x; idx < nb * nb; idx += DLUC_THREADS) {
      const int c = idx / nb, r = idx - c * nb;
      L11[r][c] = (r > c) ? __ldcg(S + (size_t)(j0 + c) * K + j0 + r) : 0.0;
    }
    __syncthreads();
    const int cnt = __ldcg(D.swap_cnt + par);
    const int sw_src = (lane < cnt) ? __ldcg(D.swap_src + par * 2 * DLU_NB + lane) : 0;
    const int sw_dst = (lane < cnt) ? __ldcg(D.swap_dst + par * 2 * DLU_NB + lane) : 0;
    // the trailing columns first (from c0: panel k+1's columns are CTA 0's
    // warps 0 .. DLU_NB-1), then the columns left of the panel (interchanges
    // only); each trailing column done bumps its 16-column block's counter,
    // which the G items of that block wait for (no grid barrier between S and G)
    for (int cidx = cta * NW + warp; cidx < K - nb; cidx += G * NW) {
      const int c = (cidx < mt) ? c0 + cidx : cidx - mt;
      double *col = S + (size_t)c * K;
      double v = 0.0;
      if (lane < cnt) v = __ldcg(col + sw_src);
      __syncwarp();
      if (lane < cnt) col[sw_dst] = v;
      __syncwarp();
      if (c < c0) continue;
      double x = (lane < nb) ? __ldcg(col + j0 + lane) : 0.0;
#pragma unroll
      for (int j = 0; j < DLU_NB; j++) {
        const double xj = __shfl_sync(0xffffffffu, x, j);
        if (lane > j && lane < nb) x = fma(-L11[lane][j], xj, x);
      }
      if (lane < nb) col[j0 + lane] = x;
      if (c < c0 + DLU_NB) continue;  // panel k+1's columns: CTA 0's own, no counter
      __threadfence();
      __syncwarp();
      if (lane == 0) atomicAdd(&colcnt[c / DLU_NB], 1u);
    }
    if (mt <= 0) break;
    // P(k+1) on CTA 0 right away: it updates panel k+1's columns itself (G's
    // column block 0) and factorises them, while the other CTAs run G(k)'s
    // other column blocks
    const int ncols0 = min(DLU_NB, mt);
    if (cta == 0) {
      __syncthreads();  // S(k) of panel k+1's columns (this CTA's warps) is done; L11 reads too
      dluc_next_panel(S, K, j0, c0, ncols0, P);
      dluc_panel_factor(S, K, c0, ncols0, D, P, par ^ 1);
    }
    // G(k): items (row tile, column block >= 1)
    const int nrt = (mt + DLUC_TR - 1) / DLUC_TR, ncb = (mt + DLU_NB - 1) / DLU_NB;
    const int nitems = nrt * (ncb - 1);
    const int first = (G > 1) ? cta - 1 : 0, stride = (G > 1) ? (int)G - 1 : 1;
    if (G == 1 || cta > 0) {
      for (int it = first; it < nitems; it += stride) {
        const int cb = 1 + it / nrt, rt = it - (cb - 1) * nrt;
        const int r0 = rt * DLUC_TR, cc0 = cb * DLU_NB;
        const int ncols = min(DLU_NB, mt - cc0);
        // the block's columns have had S(0 .. k): ncols bumps a panel
        __shared__ int s_ok;
        if (threadIdx.x == 0) {
          volatile unsigned *cc = colcnt + (c0 + cc0) / DLU_NB;
          volatile int *err = &sy->err;
          const unsigned target = (unsigned)ncols * (unsigned)(k + 1);
          unsigned spin = 0;
          int ok = 1;
          while (*cc < target) {
            if (*err || ++spin > DLUC_SPIN_LIMIT) {
              atomicExch(&sy->err, 1);
              ok = 0;
              break;
            }
            __nanosleep(32);
          }
          __threadfence();
          s_ok = ok;
        }
        __syncthreads();  // also: the previous item's reads of s_l / s_u are done
        if (!s_ok) break;
        for (int idx = threadIdx.x; idx < DLUC_TR * DLU_NB; idx += DLUC_THREADS) {
          const int kk = idx / DLUC_TR, i = idx - kk * DLUC_TR;
          s_l[i][kk] = (kk < nb && r0 + i < mt) ? __ldcg(S + (size_t)(j0 + kk) * K + c0 + r0 + i) : 0.0;
        }
        for (int idx = threadIdx.x; idx < DLU_NB * DLU_NB; idx += DLUC_THREADS) {
          const int c = idx / DLU_NB, kk = idx - c * DLU_NB;
          s_u[kk][c] = (kk < nb && c < ncols) ? __ldcg(S + (size_t)(c0 + cc0 + c) * K + j0 + kk) : 0.0;
        }
        __syncthreads();
        // thread: row r0 + (tid % DLUC_TR), columns 4 (tid / DLUC_TR) .. +3
        const int i = threadIdx.x % DLUC_TR, q0 = 4 * (threadIdx.x / DLUC_TR);
        if (r0 + i < mt) {
          double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
          for (int kk = 0; kk < DLU_NB; kk++) {
            const double a = s_l[i][kk];
#pragma unroll
            for (int q = 0; q < 4; q++) acc[q] = fma(a, s_u[kk][q0 + q], acc[q]);
          }
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int c = q0 + q;
            if (c < ncols) {
              double *dst = S + (size_t)(c0 + cc0 + c) * K + c0 + r0 + i;
              *dst = __ldcg(dst) - acc[q];
            }
          }
        }
      }
    }
    if (!dluc_barrier(sy, G)) return;
  }
}

struct DenseTail {
  int K;                 // trailing block size (0 = none)
  const double *L;       // K x K column-major, strictly lower part
  const double *U;       // K x K column-major, strictly upper part
  const double *uinv;    // [K] 1 / U(i,i)
  const double *lscale;  // [K] multiplier after the unit lower solve, or null
  const double *W;       // K x K column-major inverse (cluster path), or null
};

namespace cg = cooperative_groups;

// Rows [i0, i1) of a column-major K x K product, restricted to the columns
// [jlo(i), jhi(i)) that mode selects (0: all, 1: j > i, 2: j < i):
// out[i] = sum_j M(i, j) v[j].  Threads take (row, part) pairs; the parts of
// a row (strided columns) are added through shared memory red[].
__device__ void slice_gemv(const double *__restrict__ M, int K, int i0, int i1, const double *v, int mode,
                           double *out, double *red) {
  const int nr = i1 - i0;
  if (nr <= 0) {
    __syncthreads();
    __syncthreads();
    return;
  }
  const int parts = max(1, min(32, (int)blockDim.x / nr));
  const int t = threadIdx.x;
  const int row = t % nr, part = t / nr;
  double acc = 0.0;
  if (part < parts) {
    const int i = i0 + row;
    const double *col = M + i;
    const int jlo = (mode == 1) ? i + 1 : 0, jhi = (mode == 2) ? i : K;
    int j = jlo + ((part - jlo % parts) % parts + parts) % parts;  // first j >= jlo with j % parts == part
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (; j + 3 * parts < jhi; j += 4 * parts) {
      const double m0 = __ldg(col + (size_t)j * K), m1 = __ldg(col + (size_t)(j + parts) * K),
                   m2 = __ldg(col + (size_t)(j + 2 * parts) * K), m3 = __ldg(col + (size_t)(j + 3 * parts) * K);
      a[0] = fma(m0, v[j], a[0]);
      a[1] = fma(m1, v[j + parts], a[1]);
      a[2] = fma(m2, v[j + 2 * parts], a[2]);
      a[3] = fma(m3, v[j + 3 * parts], a[3]);
    }
    for (; j < jhi; j += parts) a[0] = fma(__ldg(col + (size_t)j * K), v[j], a[0]);
    acc = (a[0] + a[1]) + (a[2] + a[3]);
    red[part * nr + row] = acc;
  }
  __syncthreads();
  if (t < nr) {
    double s = 0.0;
    for (int p = 0; p < parts; p++) s += red[p * nr + t];
    out[t] = s;
  }
  __syncthreads();
}

// The dense tail across a thread-block cluster: x = W b with one step of
// iterative refinement through the factors, r = b - L (U x0), x = x0 + W r
// (W = U^-1 L^-1 computed once per factorisation; applying an inverse alone
// loses accuracy on an ill-conditioned Schur complement, the refinement
// step restores the triangular solves' accuracy).  Each of the csize CTAs
// computes a slice of rows of every product and writes it into every CTA's
// copy of the vector through distributed shared memory; one cluster barrier
// per product, no sequential panel chain.  The adjoint passes W^T and the
// transposed factors: L = (D^-1 U)^T with lscale = D^-1, U = L^T (unit), so
// the residual product divides by lscale between the two triangles.
// buf holds b, x0, t, r (K each) and the reduction scratch.
__device__ void cluster_dense_refined(const DenseTail &T, double *y2, double *buf, cg::cluster_group &cluster,
                                      int csize, int crank) {
  const int K = T.K;
  double *b = buf, *x0 = buf + K, *tt = buf + 2 * K, *rr = buf + 3 * K, *red = buf + 4 * K;
  const int per = (K + csize - 1) / csize;
  const int i0 = min(K, crank * per), i1 = min(K, i0 + per);
  double *sl = red + 512;  // slice result scratch [per] (red holds parts x rows <= 512)
  for (int i = threadIdx.x; i < K; i += blockDim.x) b[i] = y2[i];
  __syncthreads();
  auto publish = [&](double *dst) {
    for (int c = 0; c < csize; c++) {
      double *d = (c == crank) ? dst : cluster.map_shared_rank(dst, c);
      for (int k = threadIdx.x; k < i1 - i0; k += blockDim.x) d[i0 + k] = sl[k];
    }
    cluster.sync();
  };
  // x0 = W b
  slice_gemv(T.W, K, i0, i1, b, 0, sl, red);
  publish(x0);
  // t = U x0 (strict upper part + diagonal 1/uinv), then / lscale
  slice_gemv(T.U, K, i0, i1, x0, 1, sl, red);
  for (int k = threadIdx.x; k < i1 - i0; k += blockDim.x) {
    const int i = i0 + k;
    double v = sl[k] + x0[i] / T.uinv[i];
    if (T.lscale) v /= T.lscale[i];
    sl[k] = v;
  }
  __syncthreads();
  publish(tt);
  // r = b - L t (unit lower)
  slice_gemv(T.L, K, i0, i1, tt, 2, sl, red);
  for (int k = threadIdx.x; k < i1 - i0; k += blockDim.x) sl[k] = b[i0 + k] - (tt[i0 + k] + sl[k]);
  __syncthreads();
  publish(rr);
  // x = x0 + W r, into every copy of the tail (CTA 0's is its solve vector)
  slice_gemv(T.W, K, i0, i1, rr, 0, sl, red);
  for (int k = threadIdx.x; k < i1 - i0; k += blockDim.x) sl[k] += x0[i0 + k];
  __syncthreads();
  publish(y2);
}


// The factorised discharge system of one realization (its rows are the
// global rows row0 .. row0 + n - 1; all indices inside are local).
struct TriDesc {
  LevelSolve Lf, Lx, Ux, Ub;
  DenseTail T;
  const int *pinv;  // [n] row -> pivot step
  const int *qcol;  // [n] pivot step -> column
  int row0, n;
};

// ADJ: the transposed solve of the adjoint (the factor parts passed in
// net.tri are those of A^T): reads net.bvec, writes net.disc only.
template <bool ADJ>
__global__ void __launch_bounds__(SOLVE_THREADS, 1) trisolve_kernel(Net net, int use_smem, int cap_levptr,
                                                                     int meta_cap, int ring_cap) {
  // launched either one CTA per realization or, for one network with a large
  // dense tail, as a cluster whose CTAs 1.. join only the dense phase
  cg::cluster_group cluster = cg::this_cluster();
  const int csize = (int)cluster.num_blocks();
  const int crank = (int)cluster.block_rank();
  const int r = blockIdx.x / csize;
  SolveState *st = net.st + r;
  if (st->done) return;
  const TriDesc &TD = net.tri[r];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = TD.n, row0 = TD.row0;
  size_t ycap = 0;
  if (use_smem) ycap = (size_t)use_smem;
  double *y = use_smem ? reinterpret_cast<double *>(smem_raw) : net.work + row0;
  int *s_levptr = reinterpret_cast<int *>(smem_raw + sizeof(double) * ycap);
  int *s_meta = s_levptr + cap_levptr;
  // factor-entry ring after the slot metadata (16-byte aligned); the staged
  // path needs y, the level pointers and the metadata in shared memory
  Ring ring{0, 0, 0, 0, 0, 0, 0, 0};
  if (ring_cap > 0 && use_smem) {
    const int off =
        (int)((sizeof(double) * ycap + sizeof(int) * ((size_t)cap_levptr + 2 * (size_t)meta_cap) + 15) & ~(size_t)15);
    ring.levptr_off = (int)(sizeof(double) * ycap);
    ring.meta_off = ring.levptr_off + (int)sizeof(int) * cap_levptr;
    ring.meta_cap = meta_cap;
    ring.val_off = off;
    ring.scale_off = off + (int)sizeof(double) * RING_SLOTS * ring_cap;
    ring.col_off = ring.scale_off + (int)sizeof(double) * RING_SLOTS * (ring_cap / 2);
    ring.cap = ring_cap;
    ring.rcap = ring_cap / 2;
  }
  // the cluster path keeps b, x0, t, r and scratch in the ring's shared memory
  double *dense_buf = reinterpret_cast<double *>(smem_raw + ring.val_off);
  const int dense_per = (TD.T.K + csize - 1) / csize;
  const bool coop = csize > 1 && TD.T.K > 0 && use_smem && TD.T.W && ring.cap > 0 &&
                    (size_t)64 * ring.cap >= sizeof(double) * (4 * (size_t)TD.T.K + 512 + dense_per);
  if (crank != 0) {
    if (!ADJ && !st->solve_q) return;  // the same exits as CTA 0, so the cluster barriers pair up
    if (!coop) return;
    const int K = TD.T.K;
    double *y2 = y + (N - K);
    cluster.sync();  // CTA 0 has finished the sparse L part and the coupling rows
    const double *src = cluster.map_shared_rank(y2, 0);
    for (int i = threadIdx.x; i < K; i += blockDim.x) y2[i] = src[i];
    cluster.sync();  // every copy is taken
    cluster_dense_refined(TD.T, y2, dense_buf, cluster, csize, crank);
    cluster.sync();  // no CTA leaves while another may still write into its shared memory
    return;
  }
  if (!ADJ) {
    if (threadIdx.x == 0) st->nit += 1;
    if (!st->solve_q) return;  // uniform: solve_q is written only by reduce_kernel
  }
  long long clk = clock64();
  auto phase = [&](int i) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const long long now = clock64();
      st->tri_cycles[i] += now - clk;
      clk = now;
    }
  };
  // y = P b (b from rhs_reduce_kernel)
  for (int i = threadIdx.x; i < N; i += blockDim.x) y[TD.pinv[i]] = net.bvec[row0 + i];
  phase(0);
  // L: sparse leading rows, coupling of the trailing rows to them, dense tail
  level_solve(TD.Lf, y, s_levptr, cap_levptr, s_meta, meta_cap, ring);
  phase(1);
  if (TD.T.K > 0) {
    level_solve(TD.Lx, y, s_levptr, cap_levptr, s_meta, meta_cap, ring);
    phase(2);
    if (coop) {
      double *y2 = y + (N - TD.T.K);
      cluster.sync();  // the helpers copy y2 after this
      cluster.sync();  // ... and have copied it
      cluster_dense_refined(TD.T, y2, dense_buf, cluster, csize, crank);
      phase(3);
      cluster.sync();
      phase(4);
    } else {
      dense_lower_solve(TD.T.L, TD.T.K, y + (N - TD.T.K));
      if (TD.T.lscale) {
        for (int i = threadIdx.x; i < TD.T.K; i += blockDim.x) y[N - TD.T.K + i] *= TD.T.lscale[i];
        __syncthreads();
      }
      phase(3);
      // U: dense tail, coupling of the leading rows to it, sparse leading rows
      dense_upper_solve(TD.T.U, TD.T.uinv, TD.T.K, y + (N - TD.T.K));
      phase(4);
    }
    level_solve(TD.Ux, y, s_levptr, cap_levptr, s_meta, meta_cap, ring);
    phase(5);
  }
  level_solve(TD.Ub, y, s_levptr, cap_levptr, s_meta, meta_cap, ring);  // scale = 1/U(i,i)
  phase(6);
  // x = Q y; error_q = max|x - x_old| / (max|x_old| + 1e-16) (hpc_solve.py:169-174)
  __shared__ double s_d[32], s_o[32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double md = 0.0, mo = 0.0;
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    const int c = row0 + TD.qcol[k];
    const double xv = y[k];
    const double xo = net.disc[c];
    double dd = fabs(xv - xo);
    if (!(dd == dd)) dd = INFINITY;
    md = fmax(md, dd);
    mo = fmax(mo, fabs(xo));
  }
  __syncthreads();
  if (ADJ) {
    for (int k = threadIdx.x; k < N; k += blockDim.x) net.disc[row0 + TD.qcol[k]] = y[k];
    return;
  }
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    const int c = row0 + TD.qcol[k];
    const double xv = y[k];
    net.disc[c] = xv;
    const int d = net.row_de[c];
    if (d >= 0)
      net.q[net.de_ids[d]] = xv;
    else
      net.constant[net.row_frac[c]] = xv;
  }
  for (int o = 16; o > 0; o >>= 1) {
    md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    mo = fmax(mo, __shfl_xor_sync(0xffffffffu, mo, o));
  }
  if (lane == 0) {
    s_d[warp] = md;
    s_o[warp] = mo;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, bb = 0.0;
    for (int k = 0; k < nw; k++) {
      a = fmax(a, s_d[k]);
      bb = fmax(bb, s_o[k]);
    }
    st->error_q = a / (bb + 1e-16);
    st->tri_cycles[7] += clock64() - clk;
  }
}

// ------------------------------------------------------------------------
// Explicit inverse of the discharge system of one network
// ------------------------------------------------------------------------
// X = (P A Q)^-1 = U^-1 L^-1 in pivot order, row-major with rows padded to
// ldw (a multiple of 32), formed once per factorisation from the
// level-ordered factors: the unit lower solve on the identity (one CTA per 32
// right-hand sides, lane = right-hand side, warps over the rows of a level;
// L^-1 is lower triangular, so rows and entries left of a CTA's columns are
// skipped), the dense tail's rows as W22 T with the tail inverse
// W22 = U22^-1 L22^-1 (one FP64 GEMM), then the upper solve.  A discharge
// solve is then x0 = Q X P b, r = b - A x0, x = x0 + Q X P r: two streaming
// passes over X and one over A instead of the level-by-level dependency
// chain; the refinement step makes the result as accurate as the inverse's
// condition allows (the triangular solves' own accuracy or better).
static constexpr int WINV_THREADS = 512;
static constexpr int WINV_MAX_N = 16384;

// sum over the entries e of slot sl with col(e) >= cmin of val(e) X(col(e), c)
__device__ __forceinline__ double winv_row_dot(const LevelSolve &F, int sl, const double *X, int ldw, int c,
                                               int cmin) {
  const int e0 = __ldg(F.eptr + sl), e1 = __ldg(F.eptr + sl + 1);
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int e = e0;
  for (; e + 7 < e1; e += 8) {  // eight loads of X in flight
    int j[8];
    double v[8], x[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      j[u] = __ldg(F.col + e + u);
      v[u] = __ldg(F.val + e + u);
    }
#pragma unroll
    for (int u = 0; u < 8; u++) x[u] = (j[u] >= cmin) ? X[(size_t)j[u] * ldw + c] : 0.0;
    a0 = fma(v[0], x[0], a0);
    a1 = fma(v[1], x[1], a1);
    a2 = fma(v[2], x[2], a2);
    a3 = fma(v[3], x[3], a3);
    a0 = fma(v[4], x[4], a0);
    a1 = fma(v[5], x[5], a1);
    a2 = fma(v[6], x[6], a2);
    a3 = fma(v[7], x[7], a3);
  }
  for (; e + 3 < e1; e += 4) {
    const int j0 = __ldg(F.col + e), j1 = __ldg(F.col + e + 1), j2 = __ldg(F.col + e + 2), j3 = __ldg(F.col + e + 3);
    const double v0 = __ldg(F.val + e), v1 = __ldg(F.val + e + 1), v2 = __ldg(F.val + e + 2),
                 v3 = __ldg(F.val + e + 3);
    const double x0 = (j0 >= cmin) ? X[(size_t)j0 * ldw + c] : 0.0;
    const double x1 = (j1 >= cmin) ? X[(size_t)j1 * ldw + c] : 0.0;
    const double x2 = (j2 >= cmin) ? X[(size_t)j2 * ldw + c] : 0.0;
    const double x3 = (j3 >= cmin) ? X[(size_t)j3 * ldw + c] : 0.0;
    a0 = fma(v0, x0, a0);
    a1 = fma(v1, x1, a1);
    a2 = fma(v2, x2, a2);
    a3 = fma(v3, x3, a3);
  }
  for (; e < e1; e++) {
    const int j = __ldg(F.col + e);
    if (j >= cmin) a0 = fma(__ldg(F.val + e), X[(size_t)j * ldw + c], a0);
  }
  return (a0 + a1) + (a2 + a3);
}

// The level kernels give a CTA WINV_CW right-hand sides: each half-warp
// solves one row of a level for them, so a warp has two rows in flight.
static constexpr int WINV_CW = 16;

// X = L^-1 on the leading rows (X zeroed beforehand); T = the trailing rows
// before the dense tail's solve (K x ldw, row-major).
__global__ void __launch_bounds__(WINV_THREADS) winv_lower_kernel(TriDesc TD, double *__restrict__ X, int ldw,
                                                                  double *__restrict__ T) {
  const int N = TD.n, K = TD.T.K;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int sub = lane / WINV_CW, hw = 2 * warp + sub, nhw = 2 * nw;
  const int c0 = blockIdx.x * WINV_CW, c = c0 + lane % WINV_CW;
  const LevelSolve &F = TD.Lf;
  for (int l = 0; l < F.nlev; l++) {
    const int s0 = __ldg(F.lev_ptr + l), s1 = __ldg(F.lev_ptr + l + 1);
    for (int sl = s0 + hw; sl < s1; sl += nhw) {
      const int i = __ldg(F.rows + sl);
      if (i < c0) continue;  // X(i, c) = 0 for i < c
      const double acc = winv_row_dot(F, sl, X, ldw, c, c0);
      X[(size_t)i * ldw + c] = ((i == c) ? 1.0 : 0.0) - acc;
    }
    __syncthreads();
  }
  if (K > 0) {
    const LevelSolve &G = TD.Lx;  // independent rows (entries in the leading columns only)
    for (int sl = hw; sl < G.nslots; sl += nhw) {
      const int i = __ldg(G.rows + sl);
      const double acc = winv_row_dot(G, sl, X, ldw, c, c0);
      T[(size_t)(i - (N - K)) * ldw + c] = ((i == c) ? 1.0 : 0.0) - acc;
    }
  }
}

// C (K x ldw, row-major) = W (K x K, column-major) T (K x ldw, row-major):
// 64 x 64 tiles, 16-deep slices of W and T in shared memory, 4 x 4 outputs a
// thread (rows and columns 16 apart, so loads and stores coalesce).
__global__ void __launch_bounds__(256, 2) winv_gemm_kernel(const double *__restrict__ W, int K,
                                                           const double *__restrict__ T, int ldw,
                                                           double *__restrict__ C) {
  // 128 x 64 tile of C a CTA, 8 x 4 a thread (rows ty + 16 r, columns
  // tx + 16 q: the A reads broadcast in half-warps, the B reads consecutive),
  // a 16-deep k step: 12 shared loads per 32 fused multiply-adds; every
  // entry is one chain over k in order, whatever the tile.  The next k
  // step's tiles arrive by asynchronous copies (zero-filled outside the
  // matrices) into the other half of a double buffer while this one computes.
  __shared__ __align__(16) double As[2][16][128], Bs[2][16][64];
  const int rb = blockIdx.x * 128, cb = blockIdx.y * 64;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[8][4];
#pragma unroll
  for (int r = 0; r < 8; r++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[r][q] = 0.0;
  auto issue = [&](int k0, int buf) {
    for (int idx = threadIdx.x; idx < 16 * 128; idx += blockDim.x) {
      const int kk = idx >> 7, i = idx & 127;
      const bool v = k0 + kk < K && rb + i < K;
      cp_async8_zfill(&As[buf][kk][i], v ? W + (size_t)(k0 + kk) * K + rb + i : W, v);
    }
    for (int idx = threadIdx.x; idx < 16 * 64; idx += blockDim.x) {
      const int kk = idx >> 6, i = idx & 63;
      const bool v = k0 + kk < K && cb + i < ldw;
      cp_async8_zfill(&Bs[buf][kk][i], v ? T + (size_t)(k0 + kk) * ldw + cb + i : T, v);
    }
    cp_async_commit();
  };
  issue(0, 0);
  int buf = 0;
  for (int k0 = 0; k0 < K; k0 += 16, buf ^= 1) {
    if (k0 + 16 < K) {
      issue(k0 + 16, buf ^ 1);  // that half was last read before the barrier ending the step before
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      double a[8], b[4];
#pragma unroll
      for (int r = 0; r < 8; r++) a[r] = As[buf][kk][ty + 16 * r];
#pragma unroll
      for (int q = 0; q < 4; q++) b[q] = Bs[buf][kk][tx + 16 * q];
#pragma unroll
      for (int r = 0; r < 8; r++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[r][q] = fma(a[r], b[q], acc[r][q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const int i = rb + ty + 16 * r;
    if (i >= K) continue;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int c = cb + tx + 16 * q;
      if (c < ldw) C[(size_t)i * ldw + c] = acc[r][q];
    }
  }
}

// X(i, :) -= sum_j U(i, j) X(j, :) for the leading rows i and the (final)
// trailing rows j: independent rows, so a CTA takes WINV_COUPLE_ROWS rows
// for one slab of 256 columns (every entry's row of X is read as one
// coalesced 2 KB slab, mostly from L2).
static constexpr int WINV_COUPLE_ROWS = 8;
__global__ void __launch_bounds__(256) winv_coupling_kernel(LevelSolve G, double *__restrict__ X, int ldw) {
  const int c = blockIdx.y * 256 + threadIdx.x;
  if (c >= ldw) return;
  const int s0 = blockIdx.x * WINV_COUPLE_ROWS, s1 = min(G.nslots, s0 + WINV_COUPLE_ROWS);
  for (int sl = s0; sl < s1; sl++) {
    const int i = __ldg(G.rows + sl);
    const double acc = winv_row_dot(G, sl, X, ldw, c, 0);
    X[(size_t)i * ldw + c] -= acc;
  }
}

// X = U^-1 X on the leading rows after the coupling: the sparse upper levels
// with 1/U(i,i).
__global__ void __launch_bounds__(WINV_THREADS) winv_upper_kernel(TriDesc TD, double *__restrict__ X, int ldw) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int sub = lane / WINV_CW, hw = 2 * warp + sub, nhw = 2 * nw;
  const int c = blockIdx.x * WINV_CW + lane % WINV_CW;
  const LevelSolve &F = TD.Ub;
  for (int l = 0; l < F.nlev; l++) {
    const int s0 = __ldg(F.lev_ptr + l), s1 = __ldg(F.lev_ptr + l + 1);
    for (int sl = s0 + hw; sl < s1; sl += nhw) {
      const int i = __ldg(F.rows + sl);
      const double acc = winv_row_dot(F, sl, X, ldw, c, 0);
      const double sc = F.scale ? __ldg(F.scale + sl) : 1.0;
      X[(size_t)i * ldw + c] = (X[(size_t)i * ldw + c] - acc) * sc;
    }
    __syncthreads();
  }
}

// One pass over X: y(k) = sum_j X(k, j) v(j) with v = P src (src in equation
// order, permuted into pivot order in shared memory), X streamed past the L2.
// Each CTA owns a contiguous block of at most WINV_RPC rows; its 16 warps
// split every row into equal segments, two rows in flight at a time, and the
// segment sums are added in a fixed order (deterministic).  STAGE 0 counts
// the loop iteration (as trisolve_kernel does) and, when the state asks for
// the refinement step, writes x0(Q k) = y(k); otherwise it is the final pass.
// STAGE 1 (refinement only): x(Q k) = x0(Q k) + y(k).  The final forward
// pass writes x to the discharges / constants with the max-change error of
// the solve (the last CTA to finish turns the grid's maxima into error_q and
// zeroes them for the next solve); the adjoint (ADJ: X holds the transposed
// inverse, P and Q those of the transposed system, no refinement) writes
// net.disc only.
//
// F32 (the refinement pass): X is read from a float copy (X32, the same
// layout), each entry widened to double before its product.  The pass forms
// the correction X r of a residual r that is about 1e-10 of b: single
// precision entries (relative error 6e-8) leave an error near 1e-17 of x,
// well below the double-precision pass's own (mixed-precision iterative
// refinement: the residual in double, the correction in single).  Half the
// bytes of that pass.
static constexpr int WINV_RPC = 64;
static_assert(WINV_THREADS == 512, "16 warps split each row of X");

// The end of a pass over X: the rows' sums (warp partials in s_part, added
// in warp order), x0 or the final discharges / constants, and for the final
// forward pass the max-change error of the solve (the last CTA turns the
// grid's maxima into error_q and zeroes them for the next solve).
template <int STAGE, bool ADJ>
__device__ __forceinline__ void winv_epilogue(Net &net, const TriDesc &TD, int r0, int r1,
                                              double (*s_part)[16], double *__restrict__ x0,
                                              unsigned long long *__restrict__ acc, bool fin) {
  SolveState *st = net.st;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double md = 0.0, mo = 0.0;
  for (int t = threadIdx.x; t < r1 - r0; t += blockDim.x) {
    double y = 0.0;
#pragma unroll
    for (int w = 0; w < 16; w++) y += s_part[t][w];
    const int cc = __ldg(TD.qcol + r0 + t);
    if (!fin) {
      x0[cc] = y;
    } else if (ADJ) {
      net.disc[cc] = (STAGE == 1 ? x0[cc] : 0.0) + y;
    } else {
      const double xv = (STAGE == 1 ? x0[cc] : 0.0) + y;
      const double xo = net.disc[cc];
      double dd = fabs(xv - xo);
      if (!(dd == dd)) dd = INFINITY;
      md = fmax(md, dd);
      mo = fmax(mo, fabs(xo));
      net.disc[cc] = xv;
      const int d = net.row_de[cc];
      if (d >= 0)
        net.q[net.de_ids[d]] = xv;
      else
        net.constant[net.row_frac[cc]] = xv;
    }
  }
  if (!fin || ADJ) return;
  __shared__ double s_d[32], s_o[32];
  __shared__ int s_last;
  for (int o = 16; o > 0; o >>= 1) {
    md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    mo = fmax(mo, __shfl_xor_sync(0xffffffffu, mo, o));
  }
  if (lane == 0) {
    s_d[warp] = md;
    s_o[warp] = mo;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < 16; k++) {
      a = fmax(a, s_d[k]);
      b = fmax(b, s_o[k]);
    }
    // non-negative doubles order like their bit patterns
    atomicMax(acc, (unsigned long long)__double_as_longlong(a));
    atomicMax(acc + 1, (unsigned long long)__double_as_longlong(b));
    __threadfence();
    s_last = atomicAdd(acc + 2, 1ull) == (unsigned long long)(gridDim.x - 1);
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    const double a = __longlong_as_double((long long)atomicAdd(acc, 0ull));
    const double b = __longlong_as_double((long long)atomicAdd(acc + 1, 0ull));
    st->error_q = a / (b + 1e-16);
    acc[0] = 0ull;  // every other CTA is done with them: zero for the next solve
    acc[1] = 0ull;
    acc[2] = 0ull;
  }
}

template <int STAGE, bool ADJ, bool F32 = false>
__global__ void __launch_bounds__(WINV_THREADS, 2) winv_gemv_kernel(Net net, const double *__restrict__ X, int ldw,
                                                                 const double *__restrict__ src,
                                                                 double *__restrict__ x0,
                                                                 unsigned long long *__restrict__ acc,
                                                                 const float *__restrict__ X32 = nullptr) {
  SolveState *st = net.st;
  if (st->done) return;
  // forward: without refinement (refine is set when the run starts) the
  // first pass writes the result itself and the second does not run; the
  // adjoint's transposed solves always take the refinement step
  const bool fin = (STAGE == 1) || (!ADJ && !st->refine);
  if (!ADJ) {
    if (STAGE == 0 && blockIdx.x == 0 && threadIdx.x == 0) st->nit += 1;
    if (!st->solve_q) return;  // uniform: solve_q is written only by reduce_kernel
    if (STAGE == 1 && !st->refine) return;
    if (STAGE == 1 && blockIdx.x == 0 && threadIdx.x == 0) st->n_refined += 1;
  }
  const TriDesc &TD = net.tri[0];
  const int N = TD.n;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double s_part[WINV_RPC][16];
  double *v = reinterpret_cast<double *>(smem_raw);
  for (int i = threadIdx.x; i < N; i += blockDim.x) v[__ldg(TD.pinv + i)] = src[i];
  for (int i = N + threadIdx.x; i < ldw; i += blockDim.x) v[i] = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rpc = (N + gridDim.x - 1) / gridDim.x;  // <= WINV_RPC (grid size chosen by the host)
  const int r0 = min(N, (int)blockIdx.x * rpc), r1 = min(N, r0 + rpc);
  const int seg = ldw / 32;  // double2 per warp and row
  const double2 *vs = reinterpret_cast<const double2 *>(v) + warp * seg;
  const double2 zero2 = make_double2(0.0, 0.0);
  // four rows at a time: per lane 8 loads of 16 B in flight per round (each
  // row's segment in two halves of 32 double2), half the latency rounds of
  // two rows at a time; rows beyond r1 reread row k (results not stored)
  for (int k = r0; k < r1; k += 4) {
    double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0, c0 = 0.0, c1 = 0.0, d0 = 0.0, d1 = 0.0;
    if (F32) {
      // float4 loads (four entries, 16 B): this warp's segment of a row is
      // seg / 2 of them (ldw is a multiple of 64 when the float copy exists)
      const int seg4 = seg / 2;
      const size_t rf = ldw / 4;
      const float4 *fa = reinterpret_cast<const float4 *>(X32) + (size_t)k * rf + (size_t)warp * seg4;
      const float4 *fb = (k + 1 < r1) ? fa + rf : fa, *fc = (k + 2 < r1) ? fa + 2 * rf : fa,
                   *fd = (k + 3 < r1) ? fa + 3 * rf : fa;
      // one float4 of each of the four rows in flight per lane (64 B; two
      // of each spilled in the budget of two CTAs an SM and ran at 43 us,
      // three at one CTA an SM ran at 37 us against 34 us)
      for (int j = lane; j < seg4; j += 32) {
        const float4 wa = __ldcs(fa + j), wb = __ldcs(fb + j), wc = __ldcs(fc + j), wd = __ldcs(fd + j);
        const double2 p = vs[2 * j], q = vs[2 * j + 1];
#define WINV_F4(ACC, F) \
  ACC = fma((double)F.w, q.y, fma((double)F.z, q.x, fma((double)F.y, p.y, fma((double)F.x, p.x, ACC))))
        WINV_F4(a0, wa);
        WINV_F4(b0, wb);
        WINV_F4(c0, wc);
        WINV_F4(d0, wd);
#undef WINV_F4
      }
    } else {
      const double2 *ra = reinterpret_cast<const double2 *>(X + (size_t)k * ldw) + warp * seg;
      const double2 *rb = (k + 1 < r1) ? ra + ldw / 2 : ra;
      const double2 *rc = (k + 2 < r1) ? ra + ldw : ra;
      const double2 *rd = (k + 3 < r1) ? ra + 3 * (size_t)(ldw / 2) : ra;
      for (int j = lane; j < seg; j += 64) {
        const bool h = j + 32 < seg;
        const double2 wa0 = __ldcs(ra + j), wb0 = __ldcs(rb + j), wc0 = __ldcs(rc + j), wd0 = __ldcs(rd + j);
        const double2 wa1 = h ? __ldcs(ra + j + 32) : zero2, wb1 = h ? __ldcs(rb + j + 32) : zero2;
        const double2 wc1 = h ? __ldcs(rc + j + 32) : zero2, wd1 = h ? __ldcs(rd + j + 32) : zero2;
        const double2 x0v = vs[j], x1v = h ? vs[j + 32] : zero2;
        a0 = fma(wa0.y, x0v.y, fma(wa0.x, x0v.x, a0));
        b0 = fma(wb0.y, x0v.y, fma(wb0.x, x0v.x, b0));
        c0 = fma(wc0.y, x0v.y, fma(wc0.x, x0v.x, c0));
        d0 = fma(wd0.y, x0v.y, fma(wd0.x, x0v.x, d0));
        a1 = fma(wa1.y, x1v.y, fma(wa1.x, x1v.x, a1));
        b1 = fma(wb1.y, x1v.y, fma(wb1.x, x1v.x, b1));
        c1 = fma(wc1.y, x1v.y, fma(wc1.x, x1v.x, c1));
        d1 = fma(wd1.y, x1v.y, fma(wd1.x, x1v.x, d1));
      }
    }
    const double sa = warp_sum(a0 + a1), sb = warp_sum(b0 + b1), sc = warp_sum(c0 + c1), sd = warp_sum(d0 + d1);
    if (lane == 0) {
      s_part[k - r0][warp] = sa;
      if (k + 1 < r1) s_part[k + 1 - r0][warp] = sb;
      if (k + 2 < r1) s_part[k + 2 - r0][warp] = sc;
      if (k + 3 < r1) s_part[k + 3 - r0][warp] = sd;
    }
  }
  __syncthreads();
  winv_epilogue<STAGE, ADJ>(net, TD, r0, r1, s_part, x0, acc, fin);
}

// r = b - M x0 with M's rows in CSR form (one warp per row): M = A (vals in
// entry order, map null) or A^T (CSC of A; map gives each entry's index in
// A's entry order).  The adjoint's state has no solve_q gate.
template <bool ADJ>
__global__ void winv_resid_kernel(Net net, const int *__restrict__ rp, const int *__restrict__ cols,
                                  const int *__restrict__ map, const double *__restrict__ vals,
                                  const double *__restrict__ x0, double *__restrict__ r, int N) {
  const SolveState *st = net.st;
  if (st->done || (!ADJ && (!st->solve_q || !st->refine))) return;
  const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (i >= N) return;
  double sum = 0.0;
  for (int p = __ldg(rp + i) + lane; p < __ldg(rp + i + 1); p += 32)
    sum = fma(__ldg(vals + (map ? __ldg(map + p) : p)), x0[__ldg(cols + p)], sum);
  sum = warp_sum(sum);
  if (lane == 0) r[i] = net.bvec[i] - sum;
}

// out (cols x ldo, row-major) = in^T for in (rows x ldi, row-major).
// ------------------------------------------------------------------------
// Batched realizations: an explicit inverse per realization.  A batch's
// systems are small (tens to a few hundred unknowns), and a level-scheduled
// triangular solve of one is a chain of dependent levels in one CTA; their
// inverses (26 MB for the 256 realizations of the batched workload) stay in
// L2, and each solve is two matrix-vector products of one CTA.
//
// batch_inverse_kernel: one CTA per realization forms X = A^-1 by in-place
// Gauss-Jordan elimination with partial pivoting (the largest |a_ik| of the
// column, the first row on a tie; the row interchanges are undone as column
// interchanges in reverse order at the end), in shared memory when the
// matrix fits, else in place in the output (global memory, L2-resident).  A
// zero or non-finite pivot marks the realization singular.  The dense A is
// scattered from the assembled entries (CSR: row g's entries [ptr[g],
// ptr[g+1]) of vals, local columns in col).
// ------------------------------------------------------------------------
static constexpr int BINV_THREADS = 512;
static constexpr int BINV_SOLVE_THREADS = 512;
static constexpr int BINV_MAX_N = 4096;  // three n-vectors of the solve kernel in shared memory

__global__ void __launch_bounds__(BINV_THREADS) batch_inverse_kernel(const int *__restrict__ order,
                                                                     const int *__restrict__ roff,
                                                                     const long long *__restrict__ xoff,
                                                                     double *__restrict__ Xall,
                                                                     const int *__restrict__ ptr,
                                                                     const int *__restrict__ col,
                                                                     const double *__restrict__ vals, int *sing,
                                                                     int smem_n) {
  const int r = order[blockIdx.x];
  const int row0 = roff[r], n = roff[r + 1] - row0;
  double *Xg = Xall + xoff[r];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sm = reinterpret_cast<double *>(smem_raw);
  const bool in_smem = n <= smem_n;
  double *A = in_smem ? sm : Xg;
  double *rowk = in_smem ? sm + (size_t)n * n : sm;
  double *colk = rowk + n;
  int *ip = reinterpret_cast<int *>(colk + n);
  __shared__ double s_best[BINV_THREADS / 32];
  __shared__ int s_idx[BINV_THREADS / 32];
  __shared__ int s_p, s_bad;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = BINV_THREADS / 32;
  for (long long i = tid; i < (long long)n * n; i += BINV_THREADS) A[i] = 0.0;
  if (tid == 0) s_bad = 0;
  __syncthreads();
  for (int i = tid; i < n; i += BINV_THREADS)
    for (int p = ptr[row0 + i]; p < ptr[row0 + i + 1]; p++) A[(size_t)i * n + col[p]] += vals[p];
  __syncthreads();
  for (int k = 0; k < n; k++) {
    // pivot: the largest |a_ik|, i >= k; the first such row on a tie; a
    // NaN anywhere in the column marks the system singular
    double best = -1.0;
    int bi = n, nan_seen = 0;
    for (int i = k + tid; i < n; i += BINV_THREADS) {
      const double v = fabs(A[(size_t)i * n + k]);
      if (!(v == v))
        nan_seen = 1;
      else if (v > best) {  // rows ascend per thread: strict > keeps the first
        best = v;
        bi = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      nan_seen |= __shfl_xor_sync(0xffffffffu, nan_seen, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (lane == 0) {
      s_best[warp] = best;
      s_idx[warp] = bi;
      if (nan_seen) s_bad = 1;
    }
    __syncthreads();
    if (tid == 0) {
      double b = s_best[0];
      int p = s_idx[0];
      for (int w = 1; w < nw; w++)
        if (s_best[w] > b || (s_best[w] == b && s_idx[w] < p)) {
          b = s_best[w];
          p = s_idx[w];
        }
      if (!(b > 0.0) || !(b < INFINITY) || p >= n) s_bad = 1;  // zero or infinite pivot
      s_p = p;
      ip[k] = p;
    }
    __syncthreads();
    if (s_bad) break;
    const int p = s_p;
    if (p != k)
      for (int j = tid; j < n; j += BINV_THREADS) {
        const double t = A[(size_t)k * n + j];
        A[(size_t)k * n + j] = A[(size_t)p * n + j];
        A[(size_t)p * n + j] = t;
      }
    __syncthreads();
    const double inv = 1.0 / A[(size_t)k * n + k];
    for (int j = tid; j < n; j += BINV_THREADS) {
      rowk[j] = (j == k ? 1.0 : A[(size_t)k * n + j]) * inv;
      colk[j] = A[(size_t)j * n + k];
    }
    __syncthreads();
    for (int i = warp; i < n; i += nw) {
      double *Ai = A + (size_t)i * n;
      if (i == k) {
        for (int j = lane; j < n; j += 32) Ai[j] = rowk[j];
      } else {
        const double ci = colk[i];
        for (int j = lane; j < n; j += 32) Ai[j] = (j == k) ? -ci * inv : fma(-ci, rowk[j], Ai[j]);
      }
    }
    __syncthreads();
  }
  if (s_bad) {
    if (tid == 0) sing[r] = 1;
    return;
  }
  // undo the row interchanges: columns k and ip[k], in reverse order
  for (int k = n - 1; k >= 0; k--) {
    const int p = ip[k];
    if (p != k)
      for (int i = tid; i < n; i += BINV_THREADS) {
        const double t = A[(size_t)i * n + k];
        A[(size_t)i * n + k] = A[(size_t)i * n + p];
        A[(size_t)i * n + p] = t;
      }
    __syncthreads();
  }
  if (in_smem)
    for (long long i = tid; i < (long long)n * n; i += BINV_THREADS) Xg[i] = A[i];
  if (tid == 0) sing[r] = 0;
}

// The same Gauss-Jordan elimination for a realization too large for one
// CTA's shared memory: a cluster of BINV_CLUSTER CTAs holds the matrix in
// their shared memories, CTA c the rows [c rpc, (c + 1) rpc), rpc =
// ceil(n / BINV_CLUSTER).  Pivot step k:
//   1. each CTA finds the largest |a_ik| of its rows i >= k (first on a tie;
//      NaN flags the system) and publishes it; cluster barrier;
//   2. every CTA reads the BINV_CLUSTER candidates (distributed shared
//      memory) and takes the same pivot row p;
//   3. every CTA copies the old row p into its own buffer, and p's owner
//      copies the old row k; cluster barrier (no row is written before every
//      remote read of it is done);
//   4. each CTA forms the scaled pivot row from its copy, p's owner stores
//      the old row k as row p, and every CTA updates its own rows (row k
//      becomes the scaled pivot row).
// A step's writes to a row happen after the step's second barrier, and the
// next step's remote reads after the next step's first barrier, which every
// CTA reaches only after finishing this step.  All CTAs take the same
// decisions (from the same candidates), so they pass the same barriers.
static constexpr int BINV_CLUSTER = 8;
static constexpr size_t BINV_CLUSTER_SMEM_MAX = 220 * 1024;

__host__ __device__ __forceinline__ size_t binv_cluster_smem(int n) {
  const size_t rpc = (size_t)(n + BINV_CLUSTER - 1) / BINV_CLUSTER;
  return sizeof(double) * (rpc * n + 3 * (size_t)n) + sizeof(int) * (size_t)n + 16;
}

__global__ void __launch_bounds__(BINV_THREADS) batch_inverse_cluster_kernel(
    const int *__restrict__ big, const int *__restrict__ roff, const long long *__restrict__ xoff,
    double *__restrict__ Xall, const int *__restrict__ ptr, const int *__restrict__ col,
    const double *__restrict__ vals, int *sing) {
  cg::cluster_group cluster = cg::this_cluster();
  const int crank = (int)cluster.block_rank();
  const int r = big[blockIdx.x / BINV_CLUSTER];
  const int row0 = roff[r], n = roff[r + 1] - row0;
  const int rpc = (n + BINV_CLUSTER - 1) / BINV_CLUSTER;
  const int my0 = min(n, crank * rpc), my1 = min(n, my0 + rpc);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *A = reinterpret_cast<double *>(smem_raw);  // my rows, row-major (rpc x n)
  double *prow = A + (size_t)rpc * n;                // old pivot row
  double *rowk = prow + n;                           // scaled pivot row
  double *rkold = rowk + n;                          // old row k (p's owner)
  int *ip = reinterpret_cast<int *>(rkold + n);
  __shared__ double s_cv[2];
  __shared__ int s_ci[2];
  __shared__ double s_best[BINV_THREADS / 32];
  __shared__ int s_idx[BINV_THREADS / 32];
  __shared__ int s_p, s_bad, s_nan;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = BINV_THREADS / 32;
  for (long long i = tid; i < (long long)rpc * n; i += BINV_THREADS) A[i] = 0.0;
  if (tid == 0) {
    s_bad = 0;
    s_nan = 0;
  }
  __syncthreads();
  for (int i = my0 + tid; i < my1; i += BINV_THREADS)
    for (int p = ptr[row0 + i]; p < ptr[row0 + i + 1]; p++) A[(size_t)(i - my0) * n + col[p]] += vals[p];
  __syncthreads();
  int bad = 0;
  for (int k = 0; k < n; k++) {
    const int par = k & 1;
    // 1. this CTA's candidate
    double best = -1.0;
    int bi = n, nan_seen = 0;
    for (int i = max(k, my0) + tid; i < my1; i += BINV_THREADS) {
      const double v = fabs(A[(size_t)(i - my0) * n + k]);
      if (!(v == v))
        nan_seen = 1;
      else if (v > best) {
        best = v;
        bi = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      nan_seen |= __shfl_xor_sync(0xffffffffu, nan_seen, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (lane == 0) {
      s_best[warp] = best;
      s_idx[warp] = bi;
      if (nan_seen) s_nan = 1;
    }
    __syncthreads();
    if (tid == 0) {
      double b = s_best[0];
      int p = s_idx[0];
      for (int w = 1; w < nw; w++)
        if (s_best[w] > b || (s_best[w] == b && s_idx[w] < p)) {
          b = s_best[w];
          p = s_idx[w];
        }
      s_cv[par] = s_nan ? NAN : b;
      s_ci[par] = p;
    }
    cluster.sync();
    // 2. the pivot, from every CTA's candidate
    if (tid == 0) {
      double b = -1.0;
      int p = n, anynan = 0;
      for (int c = 0; c < BINV_CLUSTER; c++) {
        const double cv = *cluster.map_shared_rank(&s_cv[par], c);
        const int ci = *cluster.map_shared_rank(&s_ci[par], c);
        if (!(cv == cv))
          anynan = 1;
        else if (cv > b || (cv == b && ci < p)) {
          b = cv;
          p = ci;
        }
      }
      s_bad = (anynan || !(b > 0.0) || !(b < INFINITY) || p >= n) ? 1 : 0;
      s_p = p;
    }
    __syncthreads();
    if (s_bad) {
      bad = 1;
      break;
    }
    const int p = s_p;
    const int ownk = k / rpc, ownp = p / rpc;
    // 3. copies of the old rows p (every CTA) and k (p's owner)
    {
      const double *rp = cluster.map_shared_rank(A, ownp) + (size_t)(p - ownp * rpc) * n;
      for (int j = tid; j < n; j += BINV_THREADS) prow[j] = rp[j];
      if (crank == ownp && p != k) {
        const double *rk = cluster.map_shared_rank(A, ownk) + (size_t)(k - ownk * rpc) * n;
        for (int j = tid; j < n; j += BINV_THREADS) rkold[j] = rk[j];
      }
    }
    cluster.sync();
    // 4. the scaled pivot row, the interchange, the update of this CTA's rows
    const double inv = 1.0 / prow[k];
    for (int j = tid; j < n; j += BINV_THREADS) rowk[j] = (j == k ? 1.0 : prow[j]) * inv;
    if (crank == ownp && p != k)
      for (int j = tid; j < n; j += BINV_THREADS) A[(size_t)(p - my0) * n + j] = rkold[j];
    if (tid == 0) ip[k] = p;
    __syncthreads();
    for (int i = my0 + warp; i < my1; i += nw) {
      double *Ai = A + (size_t)(i - my0) * n;
      if (i == k) {
        for (int j = lane; j < n; j += 32) Ai[j] = rowk[j];
      } else {
        const double ci = Ai[k];
        __syncwarp();
        for (int j = lane; j < n; j += 32) Ai[j] = (j == k) ? -ci * inv : fma(-ci, rowk[j], Ai[j]);
      }
    }
    __syncthreads();
  }
  if (!bad) {
    // undo the row interchanges: columns k and ip[k] of this CTA's rows, in reverse order
    for (int k = n - 1; k >= 0; k--) {
      const int p = ip[k];
      if (p != k)
        for (int i = my0 + tid; i < my1; i += BINV_THREADS) {
          double *Ai = A + (size_t)(i - my0) * n;
          const double t = Ai[k];
          Ai[k] = Ai[p];
          Ai[p] = t;
        }
      __syncthreads();
    }
    double *Xg = Xall + xoff[r];
    for (long long i = tid; i < (long long)(my1 - my0) * n; i += BINV_THREADS) Xg[(size_t)my0 * n + i] = A[i];
  }
  cluster.sync();  // no CTA leaves while another may still read its shared memory
  if (crank == 0 && tid == 0) sing[r] = bad;
}

// One discharge solve of every realization, one CTA each: x0 = X b,
// r = b - A x0 (the assembled entries), x = x0 + X r; then, as the
// triangular solve's epilogue, error_q = max|x - x_old| / (max|x_old| + 1e-16)
// (hpc_solve.py:169-174) and the scatter of q and the fracture constants
// (post_matrix_solve, hpc_solve.py:721-761).
// out = X v for rows x n of a row-major X (L2-resident) with n columns and v
// in shared memory (binv_gemv: the square case):
// each warp takes four rows at a time, its lanes split the columns, eight
// independent loads in flight per lane.
__device__ __forceinline__ void binv_gemv_rows(const double *__restrict__ X, int rows, int n, const double *v,
                                               double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = BINV_SOLVE_THREADS / 32;
  for (int i0 = warp * 4; i0 < rows; i0 += nw * 4) {
    const double *X0 = X + (size_t)i0 * n;
    const bool h1 = i0 + 1 < rows, h2 = i0 + 2 < rows, h3 = i0 + 3 < rows;
    const double *X1 = h1 ? X0 + n : X0, *X2 = h2 ? X0 + 2 * (size_t)n : X0, *X3 = h3 ? X0 + 3 * (size_t)n : X0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, b0 = 0.0, b1 = 0.0, b2 = 0.0, b3 = 0.0;
    int j = lane;
    for (; j + 32 < n; j += 64) {
      const double v0 = v[j], v1 = v[j + 32];
      const double x00 = __ldg(X0 + j), x10 = __ldg(X1 + j), x20 = __ldg(X2 + j), x30 = __ldg(X3 + j);
      const double x01 = __ldg(X0 + j + 32), x11 = __ldg(X1 + j + 32), x21 = __ldg(X2 + j + 32),
                   x31 = __ldg(X3 + j + 32);
      a0 = fma(x00, v0, a0);
      a1 = fma(x10, v0, a1);
      a2 = fma(x20, v0, a2);
      a3 = fma(x30, v0, a3);
      b0 = fma(x01, v1, b0);
      b1 = fma(x11, v1, b1);
      b2 = fma(x21, v1, b2);
      b3 = fma(x31, v1, b3);
    }
    if (j < n) {
      const double v0 = v[j];
      a0 = fma(__ldg(X0 + j), v0, a0);
      a1 = fma(__ldg(X1 + j), v0, a1);
      a2 = fma(__ldg(X2 + j), v0, a2);
      a3 = fma(__ldg(X3 + j), v0, a3);
    }
    const double s0 = warp_sum(a0 + b0), s1 = warp_sum(a1 + b1), s2 = warp_sum(a2 + b2), s3 = warp_sum(a3 + b3);
    if (lane == 0) {
      out[i0] = s0;
      if (h1) out[i0 + 1] = s1;
      if (h2) out[i0 + 2] = s2;
      if (h3) out[i0 + 3] = s3;
    }
  }
}

__device__ __forceinline__ void binv_gemv(const double *__restrict__ X, int n, const double *v, double *out) {
  binv_gemv_rows(X, n, n, v, out);
}

__device__ __forceinline__ void batch_winv_solve_one(Net &net, int r, const int *__restrict__ roff,
                                                     const long long *__restrict__ xoff,
                                                     const double *__restrict__ Xall, const int *__restrict__ ptr,
                                                     const int *__restrict__ col, const double *__restrict__ vals);

// One CTA per realization of order[]; with an active list (alist of
// positions in order[], its length *acount on the device) the CTAs walk the
// list (grid-stride).
__global__ void __launch_bounds__(BINV_SOLVE_THREADS) batch_winv_solve_kernel(
    Net net, const int *__restrict__ order, const int *__restrict__ roff, const long long *__restrict__ xoff,
    const double *__restrict__ Xall, const int *__restrict__ ptr, const int *__restrict__ col,
    const double *__restrict__ vals, const int *__restrict__ alist = nullptr, const int *__restrict__ acount = nullptr) {
  const int n = alist ? *acount : (int)gridDim.x;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    __syncthreads();  // the previous realization's shared memory reads are done
    batch_winv_solve_one(net, order[alist ? alist[i] : i], roff, xoff, Xall, ptr, col, vals);
  }
}

__device__ __forceinline__ void batch_winv_solve_one(Net &net, int r, const int *__restrict__ roff,
                                                     const long long *__restrict__ xoff,
                                                     const double *__restrict__ Xall, const int *__restrict__ ptr,
                                                     const int *__restrict__ col, const double *__restrict__ vals) {
  SolveState *st = net.st + r;
  if (st->done) return;
  if (threadIdx.x == 0) st->nit += 1;
  if (!st->solve_q) return;  // uniform: solve_q is written only by reduce_kernel
  const int row0 = roff[r], n = roff[r + 1] - row0;
  const double *X = Xall + xoff[r];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *b = reinterpret_cast<double *>(smem_raw);
  double *x0 = b + n;
  double *res = x0 + n;
  for (int i = threadIdx.x; i < n; i += BINV_SOLVE_THREADS) b[i] = net.bvec[row0 + i];
  __syncthreads();
  binv_gemv(X, n, b, x0);
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += BINV_SOLVE_THREADS) {
    double s = b[i];
    for (int p = ptr[row0 + i]; p < ptr[row0 + i + 1]; p++) s = fma(-vals[p], x0[col[p]], s);
    res[i] = s;
  }
  __syncthreads();
  binv_gemv(X, n, res, b);  // b now holds the correction X r
  __syncthreads();
  __shared__ double s_d[BINV_SOLVE_THREADS / 32], s_o[BINV_SOLVE_THREADS / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double md = 0.0, mo = 0.0;
  for (int i = threadIdx.x; i < n; i += BINV_SOLVE_THREADS) {
    const int c = row0 + i;
    const double xv = x0[i] + b[i];
    const double xo = net.disc[c];
    double dd = fabs(xv - xo);
    if (!(dd == dd)) dd = INFINITY;
    md = fmax(md, dd);
    mo = fmax(mo, fabs(xo));
    net.disc[c] = xv;
    const int d = net.row_de[c];
    if (d >= 0)
      net.q[net.de_ids[d]] = xv;
    else
      net.constant[net.row_frac[c]] = xv;
  }
  for (int o = 16; o > 0; o >>= 1) {
    md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    mo = fmax(mo, __shfl_xor_sync(0xffffffffu, mo, o));
  }
  if (lane == 0) {
    s_d[warp] = md;
    s_o[warp] = mo;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, bb = 0.0;
    for (int k = 0; k < BINV_SOLVE_THREADS / 32; k++) {
      a = fmax(a, s_d[k]);
      bb = fmax(bb, s_o[k]);
    }
    st->error_q = a / (bb + 1e-16);
    st->n_refined += 1;
  }
}

// The same solve for a realization with many unknowns, spread over a
// cluster of BINV_CLUSTER CTAs: CTA c computes the rows [c rpc, (c+1) rpc) of
// x0 = X b, of the residual and of the correction X r; x0 and the residual
// are gathered from every CTA's shared memory (distributed shared memory)
// between the passes, and error_q is the maximum of the CTAs' partial maxima.
// Every CTA takes the same exits (the loop state it reads is written by other
// kernels only) and the same four cluster barriers:
//   1. every CTA's rows of x0 are in its xp;
//   2. every CTA's residual rows are in its rp and every copy of x0 is taken
//      (so xp may take the correction);
//   3. every CTA's partial maxima are written;
//   4. CTA 0 has read them (no CTA leaves while its shared memory is read).
__device__ __forceinline__ void batch_winv_solve_cluster_one(Net &net, int r, const int *__restrict__ roff,
                                                             const long long *__restrict__ xoff,
                                                             const double *__restrict__ Xall,
                                                             const int *__restrict__ ptr, const int *__restrict__ col,
                                                             const double *__restrict__ vals);

// One cluster per realization of big[]; with an active list (positions in
// big[], its length *acount on the device) the clusters walk the list
// (every CTA of a cluster takes the same realizations).
__global__ void __launch_bounds__(BINV_SOLVE_THREADS) batch_winv_solve_cluster_kernel(
    Net net, const int *__restrict__ big, const int *__restrict__ roff, const long long *__restrict__ xoff,
    const double *__restrict__ Xall, const int *__restrict__ ptr, const int *__restrict__ col,
    const double *__restrict__ vals, const int *__restrict__ alist, const int *__restrict__ acount) {
  const int cid = blockIdx.x / BINV_CLUSTER, ncl = gridDim.x / BINV_CLUSTER;
  const int n = alist ? *acount : ncl;
  for (int i = cid; i < n; i += ncl)
    batch_winv_solve_cluster_one(net, big[alist ? alist[i] : i], roff, xoff, Xall, ptr, col, vals);
}

__device__ __forceinline__ void batch_winv_solve_cluster_one(Net &net, int r, const int *__restrict__ roff,
                                                             const long long *__restrict__ xoff,
                                                             const double *__restrict__ Xall,
                                                             const int *__restrict__ ptr, const int *__restrict__ col,
                                                             const double *__restrict__ vals) {
  cg::cluster_group cluster = cg::this_cluster();
  const int crank = (int)cluster.block_rank();
  SolveState *st = net.st + r;
  if (st->done) return;
  if (crank == 0 && threadIdx.x == 0) st->nit += 1;
  if (!st->solve_q) return;  // uniform: solve_q is written only by reduce_kernel
  const int row0 = roff[r], n = roff[r + 1] - row0;
  const int rpc = (n + BINV_CLUSTER - 1) / BINV_CLUSTER;
  const int my0 = min(n, crank * rpc), my1 = min(n, my0 + rpc), mine = my1 - my0;
  const double *X = Xall + xoff[r] + (size_t)my0 * n;  // this CTA's rows
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *b = reinterpret_cast<double *>(smem_raw);  // n: b, later the whole residual
  double *x0 = b + n;                                // n: the whole x0
  double *xp = x0 + n;                               // rpc: this CTA's rows of x0, later of X r
  double *rp = xp + rpc;                             // rpc: this CTA's rows of the residual
  __shared__ double s_d[BINV_SOLVE_THREADS / 32], s_o[BINV_SOLVE_THREADS / 32];
  __shared__ double s_md, s_mo;
  for (int i = threadIdx.x; i < n; i += BINV_SOLVE_THREADS) b[i] = net.bvec[row0 + i];
  __syncthreads();
  binv_gemv_rows(X, mine, n, b, xp);
  cluster.sync();  // 1
  for (int i = threadIdx.x; i < n; i += BINV_SOLVE_THREADS) {
    const int c = i / rpc;
    x0[i] = *cluster.map_shared_rank(xp + (i - c * rpc), c);
  }
  __syncthreads();
  for (int i = my0 + threadIdx.x; i < my1; i += BINV_SOLVE_THREADS) {
    double sres = b[i];
    for (int p = ptr[row0 + i]; p < ptr[row0 + i + 1]; p++) sres = fma(-vals[p], x0[col[p]], sres);
    rp[i - my0] = sres;
  }
  cluster.sync();  // 2
  for (int i = threadIdx.x; i < n; i += BINV_SOLVE_THREADS) {
    const int c = i / rpc;
    b[i] = *cluster.map_shared_rank(rp + (i - c * rpc), c);
  }
  __syncthreads();
  binv_gemv_rows(X, mine, n, b, xp);  // the correction of this CTA's rows
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double md = 0.0, mo = 0.0;
  for (int i = my0 + threadIdx.x; i < my1; i += BINV_SOLVE_THREADS) {
    const int c = row0 + i;
    const double xv = x0[i] + xp[i - my0];
    const double xo = net.disc[c];
    double dd = fabs(xv - xo);
    if (!(dd == dd)) dd = INFINITY;
    md = fmax(md, dd);
    mo = fmax(mo, fabs(xo));
    net.disc[c] = xv;
    const int d = net.row_de[c];
    if (d >= 0)
      net.q[net.de_ids[d]] = xv;
    else
      net.constant[net.row_frac[c]] = xv;
  }
  for (int o = 16; o > 0; o >>= 1) {
    md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    mo = fmax(mo, __shfl_xor_sync(0xffffffffu, mo, o));
  }
  if (lane == 0) {
    s_d[warp] = md;
    s_o[warp] = mo;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, bb = 0.0;
    for (int k = 0; k < BINV_SOLVE_THREADS / 32; k++) {
      a = fmax(a, s_d[k]);
      bb = fmax(bb, s_o[k]);
    }
    s_md = a;
    s_mo = bb;
  }
  cluster.sync();  // 3
  if (crank == 0 && threadIdx.x == 0) {
    double a = 0.0, bb = 0.0;
    for (int c = 0; c < BINV_CLUSTER; c++) {
      a = fmax(a, *cluster.map_shared_rank(&s_md, c));
      bb = fmax(bb, *cluster.map_shared_rank(&s_mo, c));
    }
    st->error_q = a / (bb + 1e-16);
    st->n_refined += 1;
  }
  cluster.sync();  // 4
}

static size_t binv_solve_cluster_smem(int n) {
  const int rpc = (n + BINV_CLUSTER - 1) / BINV_CLUSTER;
  return sizeof(double) * (2 * (size_t)n + 2 * (size_t)rpc);
}

__global__ void transpose_ld_kernel(const double *__restrict__ in, int ldi, int rows, int cols,
                                    double *__restrict__ out, int ldo) {
  __shared__ double tile[32][33];
  const int rb = blockIdx.y * 32, cb = blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = rb + k, c = cb + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = in[(size_t)r * ldi + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = cb + k, r = rb + threadIdx.x;
    if (r < rows && c < cols) out[(size_t)c * ldo + r] = tile[threadIdx.x][k];
  }
}

// ------------------------------------------------------------------------
// Setup kernels
// ------------------------------------------------------------------------
// numba np.linspace(a, b, D + 2)[1:D+1] (np.divide of a complex by an int is
// NumPy's Smith division with a reciprocal, numba npyfuncs.np_complex_div_impl)
__device__ __forceinline__ cd linspace_interior(cd a, cd b, int D, int i /*1..D*/) {
  const int num = D + 2;
  cd delta = b - a;
  const double br = (double)(num - 1);
  const double scl = 1.0 / (br + 0.0 * 0.0);
  cd step = mk((delta.re + delta.im * 0.0) * scl, (delta.im - delta.re * 0.0) * scl);
  if (i == num - 1) return b;
  return mk(a.re + (i * step.re - 0.0 * step.im), a.im + (i * step.im + 0.0 * step.re));
}

__global__ void zint_kernel(Net net) {
  const int D = net.D;
  const long long tot = (long long)net.n_de * D;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < tot;
       idx += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(idx / D), i = (int)(idx - (long long)j * D);
    const int e = net.de_ids[j];
    const int type = net.type[e];
    if (type == 0 || type == 3) {
      net.zint0[idx] = linspace_interior(net.ep0[2 * e], net.ep0[2 * e + 1], D, i + 1);
      if (type == 0) net.zint1[idx] = linspace_interior(net.ep1[2 * e], net.ep1[2 * e + 1], D, i + 1);
    } else if (type == 2) {
      // hpc_well.py:128-130
      const double stop = 2.0 * PI - 2 * PI / D;
      double th = (D > 1) ? (0.0 + i * ((stop - 0.0) / (double)(D - 1))) : 0.0;
      if (D > 1 && i == D - 1) th = stop;
      double s, c;
      sincos(th, &s, &c);
      const double r = net.radius[e];
      const cd ctr = net.center[e];
      net.zint0[idx] = mk(r * c - 0.0 * s + ctr.re, r * s + 0.0 * c + ctr.im);
    }
  }
}

// Branch-cut crossings of the discharge elements' log cuts through the
// collocation polygon of every psi element (find_branch_cuts / get_sign,
// hpc_math_functions.py:301-403), in the reference's (segment, element)
// order.  One warp per element; lanes take consecutive segments.
__device__ __forceinline__ cd psi_polygon_point(const Net &net, int e, int type, int n, int k) {
  double th;
  theta_of(type, n, k, th);
  double s, c;
  sincos(th, &s, &c);
  cd chi = mk(c, s);
  if (type == 1 || type == 4) {
    const double r = net.radius[e];
    const cd ctr = net.center[e];
    return mk(chi.re * r - chi.im * 0.0 + ctr.re, chi.re * 0.0 + chi.im * r + ctr.im);
  }
  cd a = net.ep0[2 * e], b = net.ep0[2 * e + 1];
  cd inv = cdiv_ref(mk(1.0, 0.0), chi);
  cd bz = 0.5 * (chi + inv);
  cd d = b - a;
  cd pp = mk(bz.re * d.re - bz.im * d.im, bz.re * d.im + bz.im * d.re);
  return 0.5 * (pp + a + b);
}

__global__ void cuts_kernel(Net net, const int *__restrict__ elist, int nlist) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nlist) return;
  const int e = elist[warp];
  const int type = net.type[e];
  const int n = net.nint[e];
  const int f = net.frac0[e];
  const int k0 = net.fptr[f], k1 = net.fptr[f + 1];
  int total = 0;
  for (int base = 0; base < n - 1; base += 32) {
    const int ii = base + lane;
    cd zp0 = mk(0, 0), zp1 = mk(0, 0);
    if (ii < n - 1) {
      zp0 = psi_polygon_point(net, e, type, n, ii);
      zp1 = psi_polygon_point(net, e, type, n, ii + 1);
    }
    int mine = 0, off = 0;
    // pass 0 counts this lane's crossings, pass 1 writes them after an
    // exclusive scan, so entries come out in (segment, element) order
    for (int pass = 0; pass < 2; pass++) {
      int wrote = 0;
      if (ii < n - 1) {
        for (int k = k0; k < k1; k++) {
          const int el = net.felem[k];
          const int t = net.type[el];
          bool hit = false;
          cd chi0 = mk(0, 0), chi1 = mk(0, 0);
          int sdef = -1;
          if (t == 0) {
            const bool s0 = (net.frac0[el] == f);
            const cd *ep = s0 ? net.ep0 + 2 * el : net.ep1 + 2 * el;
            sdef = s0 ? -1 : 1;
            chi0 = map_z_line_to_chi_ref(zp0, ep[0], ep[1]);
            chi1 = map_z_line_to_chi_ref(zp1, ep[0], ep[1]);
            const double ln0 = atan2(chi0.im, chi0.re), ln1 = atan2(chi1.im, chi1.re);
            const int sg0 = (ln0 > 0) - (ln0 < 0), sg1 = (ln1 > 0) - (ln1 < 0);
            hit = (sg0 != sg1) && (fabs(ln0) + fabs(ln1) > PI);
          } else if (t == 2 || t == 3) {
            if (t == 2) {
              const double r = net.radius[el];
              const cd c = net.center[el];
              chi0 = cdiv_ref(zp0 - c, mk(r, 0.0));
              chi1 = cdiv_ref(zp1 - c, mk(r, 0.0));
            } else {
              chi0 = map_z_line_to_chi_ref(zp0, net.ep0[2 * el], net.ep0[2 * el + 1]);
              chi1 = map_z_line_to_chi_ref(zp1, net.ep0[2 * el], net.ep0[2 * el + 1]);
            }
            const int sg0 = (chi0.im > 0) - (chi0.im < 0), sg1 = (chi1.im > 0) - (chi1.im < 0);
            hit = (sg0 != sg1) && (chi0.re < 0);
          }
          if (!hit) continue;
          if (pass == 0) {
            mine++;
          } else {
            const int slot = total + off + wrote;
            wrote++;
            if (slot < net.cut_cap) {
              const size_t o = (size_t)e * net.cut_cap + slot;
              net.cut_pos[o] = ii;
              net.cut_elem[o] = el;
              int sg = sdef;
              if (type != 1) sg = (chi0.im < chi1.im) ? -1 * sdef : sdef;  // get_sign
              net.cut_sign[o] = sg;
            } else {
              atomicExch(&net.st[net.real_elem[e]].status, (int)ANDFN_BAD_INPUT);
            }
          }
        }
      }
      if (pass == 0) {
        int v = mine;
        for (int o = 1; o < 32; o <<= 1) {
          int u = __shfl_up_sync(0xffffffffu, v, o);
          if (lane >= o) v += u;
        }
        off = v - mine;
      }
    }
    total += __shfl_sync(0xffffffffu, off + mine, 31);
  }
  if (lane == 0) net.cut_n[e] = min(total, net.cut_cap);
}

// Omega_f(z) of one point: C_f plus the potential of every element of
// fracture f (hpc_fracture.py:52-94, exclude = -1).  Shared by every
// point-evaluation kernel (heads, Omega), so they evaluate one formula.
__device__ __forceinline__ cd omega_at(const Net &net, int f, cd zz) {
  double ar = net.constant[f], ai = 0.0;
  for (int k = net.fptr[f]; k < net.fptr[f + 1]; k++) {
    const int el = net.felem[k];
    const int ty = net.type[el];
    const int m = net.ncoef[el];
    const cd *c = net.coef + (size_t)el * net.MC;
    const bool neg = (ty == 0 && net.frac0[el] != f);
    const double sg = neg ? -1.0 : 1.0;
    const double qk = sg * net.q[el] / (2 * PI);
    if (ty == 0 || ty == 3 || ty == 5) {
      const cd *ep = neg ? net.ep1 + 2 * el : net.ep0 + 2 * el;
      cd inv = recip(ep[1] - ep[0]);
      cd ab = ep[0] + ep[1];
      cd Z = fma_c(2.0 * inv, zz, mk(-(ab.re * inv.re - ab.im * inv.im), -(ab.re * inv.im + ab.im * inv.re)));
      cd chi = exterior_chi(Z);
      if (m > 0) {
        cd w = recip(chi);
        cd r = sg * c[m - 1];
        for (int j = m - 2; j >= 0; j--) r = fma_c(r, w, sg * c[j]);
        ar += r.re;
        ai += r.im;
      }
      if (ty != 5) {
        ar += qk * 0.5 * log(norm2(chi));
        ai += qk * atan2(chi.im, chi.re);
      }
    } else if (ty == 1) {
      cd chi = (1.0 / net.radius[el]) * zz;
      if (m > 0) {
        cd r = c[m - 1];
        for (int j = m - 2; j >= 0; j--) r = fma_c(r, chi, c[j]);
        ar += r.re;
        ai += r.im;
      }
    } else if (ty == 2) {
      cd chi = (1.0 / net.radius[el]) * (zz - net.center[el]);
      if (norm2(chi) < (1.0 - 1e-12) * (1.0 - 1e-12)) {
        ar = NAN;
        ai = NAN;
      } else {
        ar += qk * 0.5 * log(norm2(chi));
        ai += qk * atan2(chi.im, chi.re);
      }
    } else if (ty == 4) {
      cd chi = (1.0 / net.radius[el]) * (zz - net.center[el]);
      if (norm2(chi) < (1.0 - 1e-10) * (1.0 - 1e-10)) {
        ar = NAN;
        ai = NAN;
      } else if (m > 0) {
        cd w = recip(chi);
        cd r = c[m - 1];
        for (int j = m - 2; j >= 0; j--) r = fma_c(r, w, c[j]);
        ar += r.re;
        ai += r.im;
      }
    }
  }
  return mk(ar, ai);
}

// Omega_f(z) at arbitrary points, one thread per point; used for heads
// (hpc_fracture.py:205-252).
__global__ void points_kernel(Net net, const int *__restrict__ frac, const cd *__restrict__ z, int npts,
                              cd *__restrict__ out_omega, double *__restrict__ out_head) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const int f = frac[i];
  const cd om = omega_at(net, f, z[i]);
  if (out_omega) out_omega[i] = om;
  if (out_head) out_head[i] = om.re / net.t[f];
}

// Average discharge term of source element ee over the D points of row j
// (get_discharge_term, hpc_solve.py:1451-1459 and the per-type
// discharge_term functions).  One warp per matrix entry.
__global__ void matrix_values_kernel(Net net, const int *__restrict__ ent_row, const int *__restrict__ ent_src,
                                     const int *__restrict__ ent_side, const int *__restrict__ ent_kind,
                                     double *__restrict__ vals, long long nent) {
  const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= nent) return;
  const int kind = ent_kind[w];
  const int g = ent_row[w];   // global row
  const int j = net.row_de[g];  // discharge-element index (-1 for continuity rows)
  if (kind == 1) {  // fracture-constant column: 1/t0, -1/t1 (intersections) or 1
    if (lane == 0) {
      const int e = net.de_ids[j];
      const int side = ent_side[w];
      if (net.type[e] == 0)
        vals[w] = side ? -1.0 / net.t[net.frac1[e]] : 1.0 / net.t[net.frac0[e]];
      else
        vals[w] = 1.0;
    }
    return;
  }
  if (kind == 2) {  // continuity row: +1 / -1
    if (lane == 0) {
      const int el = ent_src[w];
      const int f = net.row_frac[g];
      vals[w] = (net.type[el] != 0 || net.frac0[el] == f) ? 1.0 : -1.0;
    }
    return;
  }
  const int e = net.de_ids[j];
  const int side = ent_side[w];
  const int ee = ent_src[w];
  const int f = side ? net.frac1[e] : net.frac0[e];
  const cd *z = (side ? net.zint1 : net.zint0) + (size_t)j * net.D;
  const int t = net.type[ee];
  double s = 0.0;
  for (int i = lane; i < net.D; i += 32) {
    cd chi;
    double sg = 1.0;
    if (t == 2) {
      chi = (1.0 / net.radius[ee]) * (z[i] - net.center[ee]);
    } else {
      const bool s0 = (t != 0) || (net.frac0[ee] == f);
      if (t == 0 && !s0) sg = -1.0;
      const cd *ep = s0 ? net.ep0 + 2 * ee : net.ep1 + 2 * ee;
      cd inv = recip(ep[1] - ep[0]);
      cd Z = fma_c(2.0 * inv, z[i], mk(-((ep[0] + ep[1]).re * inv.re - (ep[0] + ep[1]).im * inv.im),
                                        -((ep[0] + ep[1]).re * inv.im + (ep[0] + ep[1]).im * inv.re)));
      chi = exterior_chi(Z);
    }
    s += sg / (2 * PI) * (0.5 * log(norm2(chi)));
  }
  s = warp_sum(s);
  if (lane == 0) {
    double v = s / net.D;
    if (net.type[e] == 0) v = (side ? -v : v) / net.t[f];
    vals[w] = v;
  }
}

// hpc_solve.py:124-128: error and error_old start at 1e30.
__global__ void init_state_kernel(Net net) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < net.ne; i += gridDim.x * blockDim.x) {
    net.err_old[i] = 1e30;
    net.err[i] = 1e30;
  }
}

// FP64 FMA throughput probe: 8 independent dependent chains per thread.
__global__ void fp64_peak_kernel(double *out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = threadIdx.x * 1e-9 + k;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = fma(x[k], a, b);
  }
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  if (s == 12345.678) out[0] = s;
}

// ------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------
static thread_local std::string g_last_error;
static void set_error(const std::string &s) { g_last_error = s; }

#define CK(call)                                                                                    \
  do {                                                                                              \
    cudaError_t _e = (call);                                                                        \
    if (_e != cudaSuccess) {                                                                        \
      set_error(std::string(#call) + ": " + cudaGetErrorString(_e));                                \
      return ANDFN_CUDA_ERROR;                                                                      \
    }                                                                                               \
  } while (0)

// Host milliseconds spent in device allocation and release on this thread
// (reported per solve as ms_alloc).
static thread_local double g_alloc_ms = 0.0;

// ------------------------------------------------------------------------
// Device memory cache shared by every handle of the process.
//
// cudaMalloc and cudaFree of the large buffers (an explicit inverse of
// hundreds of MB, the pair tables) cost milliseconds each, and cudaFree waits
// for the whole device; a one-call solve that creates and destroys a handle
// would pay that every call.  Released blocks are therefore kept and handed
// to later buffers of any handle:
//   * a block is released while the releasing thread has a handle's stream
//     current (PoolStream, set by the entry points), and it is tagged with an
//     event recorded on that stream; a later user waits for the event on its
//     own current stream (cudaStreamWaitEvent) before touching the block, so
//     reuse is ordered after every use of the earlier owner;
//   * without a current stream a block is freed and allocated the plain way
//     (cudaFree's device-wide wait keeps that safe);
//   * a request takes the smallest cached block of at least its size and at
//     most twice it (plus 1 MiB), and blocks are allocated in 256-byte steps;
//   * the cache holds at most ANDFN_B200_POOL_MB MiB per device (default
//     8192, 0 turns it off); a block that would exceed it is freed, and a
//     failed cudaMalloc frees every cached block of the device and retries;
//   * andfn_b200_release_cached_memory() returns every cached block.
// ------------------------------------------------------------------------
static thread_local cudaStream_t g_pool_stream = nullptr;
static thread_local bool g_pool_stream_set = false;

struct PoolStream {
  cudaStream_t prev;
  bool prev_set;
  explicit PoolStream(cudaStream_t s) : prev(g_pool_stream), prev_set(g_pool_stream_set) {
    g_pool_stream = s;
    g_pool_stream_set = true;
  }
  ~PoolStream() {
    g_pool_stream = prev;
    g_pool_stream_set = prev_set;
  }
};

struct PoolBlock {
  void *p;
  size_t bytes;
  cudaEvent_t ev;
};

struct DevicePool {
  std::mutex m;
  std::multimap<size_t, PoolBlock> free_blocks[64];  // by device
  size_t held[64] = {};
  std::vector<cudaEvent_t> spare_events;
  int64_t hits = 0, misses = 0;
};

static DevicePool &device_pool() {
  static DevicePool *pool = new DevicePool();  // never destroyed: the driver may be gone at exit
  return *pool;
}

static size_t pool_cap_bytes() {
  static const size_t cap = [] {
    long long mb = 8192;
    if (const char *e = getenv("ANDFN_B200_POOL_MB")) mb = std::max(0LL, atoll(e));
    return (size_t)mb << 20;
  }();
  return cap;
}

static size_t pool_round(size_t bytes) { return (bytes + 255) & ~(size_t)255; }

// Frees every cached block of device dev (waiting for each block's event).
static void pool_flush_device(DevicePool &P, int dev) {
  for (auto &kv : P.free_blocks[dev]) {
    if (kv.second.ev) {
      cudaEventSynchronize(kv.second.ev);
      P.spare_events.push_back(kv.second.ev);
    }
    cudaFree(kv.second.p);
  }
  P.free_blocks[dev].clear();
  P.held[dev] = 0;
}

// The cache is used only with a current stream that is not being captured
// into a graph (an event wait there would tie the graph to this moment).
static bool pool_usable() {
  if (!g_pool_stream_set || pool_cap_bytes() == 0) return false;
  if (!g_pool_stream) return true;  // idle: the handle's stream has been synchronised
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(g_pool_stream, &cs) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return cs == cudaStreamCaptureStatusNone;
}

static cudaError_t pool_alloc(void **out, size_t bytes) {
  bytes = pool_round(bytes);
  int dev = 0;
  cudaGetDevice(&dev);
  DevicePool &P = device_pool();
  if (dev >= 0 && dev < 64 && pool_usable()) {
    std::lock_guard<std::mutex> lk(P.m);
    auto &fb = P.free_blocks[dev];
    auto it = fb.lower_bound(bytes);
    if (it != fb.end() && it->first <= 2 * bytes + ((size_t)1 << 20)) {
      PoolBlock b = it->second;
      fb.erase(it);
      P.held[dev] -= b.bytes;
      if (b.ev) {
        if (g_pool_stream)
          cudaStreamWaitEvent(g_pool_stream, b.ev, 0);
        else
          cudaEventSynchronize(b.ev);
        P.spare_events.push_back(b.ev);
      }
      *out = b.p;
      P.hits++;
      return cudaSuccess;
    }
    P.misses++;
  }
  cudaError_t e = cudaMalloc(out, bytes);
  if (e == cudaErrorMemoryAllocation && dev >= 0 && dev < 64) {
    cudaGetLastError();
    {
      std::lock_guard<std::mutex> lk(P.m);
      pool_flush_device(P, dev);
    }
    e = cudaMalloc(out, bytes);
  }
  return e;
}

static void pool_release(void *p, size_t bytes) {
  bytes = pool_round(bytes);
  int dev = 0;
  cudaGetDevice(&dev);
  DevicePool &P = device_pool();
  if (dev >= 0 && dev < 64 && pool_usable()) {
    std::lock_guard<std::mutex> lk(P.m);
    if (P.held[dev] + bytes <= pool_cap_bytes()) {
      if (!g_pool_stream) {  // idle: nothing in flight uses the block
        P.free_blocks[dev].emplace(bytes, PoolBlock{p, bytes, nullptr});
        P.held[dev] += bytes;
        return;
      }
      cudaEvent_t ev = nullptr;
      if (!P.spare_events.empty()) {
        ev = P.spare_events.back();
        P.spare_events.pop_back();
      } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        ev = nullptr;
      }
      if (ev && cudaEventRecord(ev, g_pool_stream) == cudaSuccess) {
        P.free_blocks[dev].emplace(bytes, PoolBlock{p, bytes, ev});
        P.held[dev] += bytes;
        return;
      }
      cudaGetLastError();
      if (ev) P.spare_events.push_back(ev);
    }
  }
  cudaFree(p);
}

// Device buffer that keeps its allocation when it is re-filled with no more
// elements than it holds; its blocks come from, and go back to, the device
// memory cache above.
template <class T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0, cap = 0;
  DBuf() = default;
  DBuf(const DBuf &) = delete;  // one owner per block (the cache would hand out a doubly released block twice)
  DBuf &operator=(const DBuf &) = delete;
  cudaError_t alloc(size_t count) {
    n = count;
    if (count <= cap && p) return cudaSuccess;
    release();
    n = count;
    if (count == 0) return cudaSuccess;
    cap = count;
    const auto t0 = std::chrono::steady_clock::now();
    void *q = nullptr;
    const cudaError_t e = pool_alloc(&q, sizeof(T) * count);
    p = static_cast<T *>(q);
    if (e != cudaSuccess) {
      p = nullptr;
      cap = 0;
    }
    g_alloc_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return e;
  }
  void release() {
    if (p) {
      const auto t0 = std::chrono::steady_clock::now();
      pool_release(p, sizeof(T) * cap);
      g_alloc_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    p = nullptr;
    n = cap = 0;
  }
  ~DBuf() { release(); }
};

// Page-locked host blocks (the Schur complement's staging buffer), kept
// for later handles of the process like the device blocks above: a block is
// handed out only after its owner's copies have finished (the owner
// synchronises before it releases).  At most ANDFN_B200_PINNED_POOL_MB MiB
// (default 1024) are kept; andfn_b200_release_cached_memory() frees them.
struct PinnedPool {
  std::mutex m;
  std::multimap<size_t, void *> blocks;
  size_t held = 0;
};
static PinnedPool &pinned_pool() {
  static PinnedPool *pool = new PinnedPool();
  return *pool;
}
static void *pinned_get(size_t bytes, size_t *cap) {
  PinnedPool &P = pinned_pool();
  {
    std::lock_guard<std::mutex> lk(P.m);
    auto it = P.blocks.lower_bound(bytes);
    if (it != P.blocks.end() && it->first <= 2 * bytes) {
      void *p = it->second;
      *cap = it->first;
      P.held -= it->first;
      P.blocks.erase(it);
      return p;
    }
  }
  void *p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  *cap = bytes;
  return p;
}
static void pinned_put(void *p, size_t cap) {
  if (!p) return;
  static const size_t limit = [] {
    long long mb = 1024;
    if (const char *e = getenv("ANDFN_B200_PINNED_POOL_MB")) mb = std::max(0LL, atoll(e));
    return (size_t)mb << 20;
  }();
  PinnedPool &P = pinned_pool();
  {
    std::lock_guard<std::mutex> lk(P.m);
    if (P.held + cap <= limit) {
      P.blocks.emplace(cap, p);
      P.held += cap;
      return;
    }
  }
  cudaFreeHost(p);
}
static void pinned_flush() {
  PinnedPool &P = pinned_pool();
  std::lock_guard<std::mutex> lk(P.m);
  for (auto &kv : P.blocks) cudaFreeHost(kv.second);
  P.blocks.clear();
  P.held = 0;
}

struct HostNet {
  // element SoA of all realizations (host copies of the geometry and of the initial state)
  std::vector<int> type, frac0, frac1, ncoef, nint;
  std::vector<cd> ep0, ep1, center;
  std::vector<double> radius, phi, q, err, err_old, err_old2, err_coef;
  std::vector<cd> coef;  // [ne][MC]
  std::vector<double> t, constant;
  std::vector<int> fptr, felem;
  std::vector<int> de_ids, elem_de;
  // realization r owns elements [eoff[r], eoff[r+1]), fractures [foff[r], foff[r+1]),
  // discharge elements [doff[r], doff[r+1]) and system rows [roff[r], roff[r+1])
  std::vector<int> eoff, foff, doff, roff;
  std::vector<int> real_elem, real_frac, real_row, row_de, row_frac;
  std::vector<double> head;  // prescribed head of constant-head lines and wells
  // wells whose discharge is prescribed (NaN head): not unknowns of the system
  std::vector<char> spec_q;
};

// Discharge system of one realization (local row / column indices).
struct RealSys {
  int n = 0, n_de = 0;
  std::vector<int> mrow_ptr, mcol;  // CSR pattern (row = equation, col = unknown)
  int ent0 = 0;                     // first entry in the global assembly arrays
  std::vector<int> colorder;        // cached symbolic analysis (pattern only)
  int dense_k = 0;
  // factor statistics of the last run
  int tail_k = 0, nlev_l = 0, nlev_u = 0;
  int64_t nnz = 0;
};

// Level-ordered factor part of all realizations, concatenated.
struct LevelParts {
  std::vector<int> lev, rows, eptr, col;
  std::vector<double> val, scale;
};

struct AdjBufs;
static void destroy_adj(AdjBufs *a);

// Power sums of the head-vector points: for every (discharge row side g =
// 2 j + side, source element of that side's fracture with coefficients) pair,
// S[x] = sign * sum over the side's D points of x^k (k < ncoef of the
// source; x the source's 1/chi or chi).  They depend on the geometry and ncoef
// only, so they are computed once per handle; the head vector is then
// b = sum Re(coef * S) / D per row side, and its transpose reuses them.
struct HeadSums {
  DBuf<int> pair_g, pair_src, pair_off, src_ptr, src_pairs, gptr, sidx;
  DBuf<cd> S;
  int npairs = 0;
  bool valid = false;
  bool long_rows = false;  // > 256 entries a row on average: a CTA per row, else a warp
  int mc = 0;
  std::vector<int> ncoef;  // the ncoef the sums were computed for
};

}  // namespace andfn

using namespace andfn;

struct AndfnHandle {
  int device = 0;
  cudaStream_t stream = nullptr;
  AndfnLayout L;
  int R = 1;
  int64_t ne = 0, nf = 0, D = 0;
  int MC = 0;  // coefficient capacity (per element, device)
  HostNet h;
  // device arrays
  DBuf<int> type, frac0, frac1, ncoef, nint, ncoef0, nint0;
  DBuf<cd> ep0, ep1, center, coef, coef0, wcoef;
  DBuf<double> radius, phi, q, q0, err, err_old, err_old2, err_coef, err_in, err_old_in, err_old2_in, err_coef_in;
  DBuf<double> dpsi_corr, t, constant, constant0;
  DBuf<int> fptr, felem, de_ids;
  DBuf<int> real_elem, real_frac, real_row, eoff, row_de, row_frac, ndone;
  DBuf<cd> zint0, zint1;
  DBuf<int> cut_n, cut_pos, cut_elem, cut_sign;
  int cut_cap = 0;
  // discharge systems
  int N = 0;  // rows of all realizations
  std::vector<RealSys> sys;
  std::vector<int> ent_row, ent_src, ent_side, ent_kind;
  // known terms of wells with a prescribed discharge: matrix-like entries
  // (row, source well, side; their values follow the pattern entries in the
  // assembly arrays from known0 on) and continuity-row terms (row, well)
  std::vector<int> known_row, known_src, known_side, known_cont_row, known_cont_src;
  int known0 = 0;
  bool has_spec = false;
  DBuf<double> bknown;
  DBuf<int> d_ent_row, d_ent_src, d_ent_side, d_ent_kind;
  DBuf<double> d_mvals;
  double ms_create_upload = 0, ms_create_tables = 0, ms_create_order = 0;
  // the column orders are computed on this host thread while the evaluation
  // tables are built and the first run's device set-up goes on; joined
  // before the first factorisation (and on destruction).  A single network's
  // order is also published column by column (order_prog), and the first
  // factorisation takes its leading pivot steps as the columns arrive.
  std::thread order_thread;
  OrderProgress order_prog;
  bool order_follow = false;
  DBuf<double> disc, work, bvec;
  DBuf<int> ready;
  // factors of all realizations (level-ordered parts, dense tails, permutations)
  DBuf<int> lf_lev, lf_rows, lf_eptr, lf_col, ub_lev, ub_rows, ub_eptr, ub_col;
  DBuf<double> lf_val, ub_val, ub_scale;
  DBuf<int> lx_lev, lx_rows, lx_eptr, lx_col, ux_lev, ux_rows, ux_eptr, ux_col;
  DBuf<double> lx_val, ux_val;
  // dense tails: L strictly below and U on and above the diagonal in one
  // K x K column-major matrix per realization (diagonal of U in tail_uinv)
  DBuf<double> tail_l, tail_uinv, tail_w;
  DBuf<int> dlu_i;  // device dense-LU scratch
  DBuf<double> dlu_d;
  cudaEvent_t mv_ev = nullptr;  // the matrix values' copy to the host has landed
  DBuf<DluSync> dlu_sync;  // barrier state of the one-launch dense LU
  DBuf<unsigned> dlu_colcnt;  // its per-16-column-block counters of finished S steps
  // explicit inverse of a single network's system (pivot order, rows padded
  // to winv_ldw), the system's CSR pattern and the solve's work arrays
  DBuf<double> winv, winv_t, wx0, wr;
  DBuf<float> winv32;  // float copy of winv for the refinement pass
  float *winv32_p = nullptr;
  DBuf<int> a_ptr, a_col;
  DBuf<unsigned long long> wacc;
  int winv_ldw = 0, num_sms = 148;
  cudaEvent_t dlu_ev = nullptr;  // the dense LU's pivots are on the host
  double *pin_schur = nullptr;   // page-locked Schur complement (repeated factorisations)
  size_t pin_schur_n = 0;
  int factor_runs = 0;
  double ms_fac[4] = {};  // factorisation phases of the last run (see AndfnSolveStats)
  bool winv_ready = false;
  bool winv_enabled = true;
  // batches: one explicit inverse per realization (batch_inverse_kernel)
  bool binv_ready = false;
  DBuf<double> binv;
  DBuf<long long> binv_off;
  DBuf<int> binv_order, binv_roff, bcsr_ptr, bcsr_col, bsing, binv_small, binv_big;
  int binv_maxn = 0, binv_nsmall = 0, binv_nbig = 0, binv_smem_n = 0, binv_bign = 0;
  // realizations (the largest, a prefix of binv_order) whose per-iteration
  // solve runs on a cluster of CTAs, and binv_order on the host
  int binv_ncsolve = 0;
  std::vector<int> binv_order_h;
  double dense_frac = 0.15;  // ordering: dense tail once the minimum degree reaches this fraction
  bool bcsr_built = false;
  DBuf<int> pinv, qcol;
  DBuf<TriDesc> tri;
  int max_n = 0, max_nlev = 0, max_k = 0;
  int cluster_fwd = -1, cluster_adj = -1;  // CTAs of the dense-tail cluster (1: no cluster; -1: not yet chosen)
  int64_t nnz_factors = 0;
  // evaluation tables
  std::vector<Group> groups;
  DBuf<Group> d_groups;
  DBuf<Item> sweep_items, rhs_items;
  DBuf<int2> sweep_pts, rhs_pts;
  int n_sweep_items = 0, n_rhs_items = 0;
  DBuf<int> group_of;   // [ne][2] -> sweep group
  DBuf<int> rhs_group;  // [n_de][2] -> rhs group
  DBuf<double> sweep_vals, rhs_vals;
  // sweep pair tables (see pair_table_kernel): layout, values, and whether
  // the values belong to this run's geometry and points
  DBuf<long long> tab_off;
  DBuf<int> tab_fpt0, tab_fnp;
  std::vector<int> h_tab_fpt0, h_tab_fnp;
  DBuf<cd> tab_w;
  DBuf<double> tab_l;
  long long tab_pairs = 0;
  int tab_chunk = 2;
  size_t tab_smem = 0;
  bool tab_valid = false, use_tab = false;
  // launch form of the table sweep (SWEEP_* below), picked by sweep_autotune
  DBuf<WorkQueue> sweep_q;
  int sweep_variant = -1;
  bool tune_sweep = true;  // false: the one-call solve uses a cached choice or the default
  DBuf<int> upd_list, psi_list;
  DBuf<cd> dft_tab;  // DFT bases, one per (nint, theta layout) in use
  DBuf<int> dft_off;
  // a single network's split reduction: partial results and the ticket
  DBuf<ReducePart> red_parts;
  DBuf<unsigned> red_ticket;
  // a batch's active work lists (rows, sweep items, elements) and their state
  DBuf<int> act_l[ACT_LISTS], act_ccnt;
  DBuf<ActState> act_st;
  ActLists act{};
  bool act_on = false;
  int n_upd = 0, n_psi = 0;
  int nvmax = 0;
  // current ncoef / nint the tables were built for (they change with adaptive growth)
  std::vector<int> cur_ncoef, cur_nint;
  bool tables_dirty = false;
  // re-solve tables of the elements grown in one iteration
  DBuf<Group> rs_groups;
  DBuf<Item> rs_items;
  DBuf<int2> rs_pts;
  DBuf<int> rs_group_of, rs_list, grow_list, grow_count;
  DBuf<double> rs_vals;
  int chunk = 0;
  size_t eval_smem = 0;
  DBuf<SolveState> st;
  std::vector<SolveState> h_st;  // host copy of the R loop states
  int *h_ndone = nullptr;        // pinned
  cudaGraphExec_t graph_exec = nullptr;
  // the whole iteration loop as one graph launch (a device-side while node)
  cudaGraphExec_t loop_exec = nullptr;
  DBuf<int> loop_count;
  int solve_threads = SOLVE_THREADS;
  // per-kernel timing: event pairs recorded as graph nodes around every
  // kernel of every captured iteration
  int profiling = 0;
  cudaEvent_t ev[ITER_BATCH][KCLASSES][2] = {};
  double k_ms[KCLASSES] = {};
  int64_t k_n[KCLASSES] = {};
  int64_t launches = 0;
  std::vector<AndfnSolveStats> last;  // per realization
  // adjoint (single network): factors of the last run and their transposed
  // device form, loop state and work arrays
  LuFactors lu_keep;
  bool adj_factors_ready = false;
  bool have_solution = false;
  AdjBufs *adj = nullptr;
  HeadSums hs;
  bool use_head_sums = false;

  Net net() const {
    Net n;
    n.ne = (int)ne;
    n.nf = (int)nf;
    n.n_de = (int)h.de_ids.size();
    n.N = N;
    n.MC = MC;
    n.D = (int)D;
    n.type = type.p;
    n.frac0 = frac0.p;
    n.frac1 = frac1.p;
    n.ncoef = ncoef.p;
    n.nint = nint.p;
    n.ep0 = ep0.p;
    n.ep1 = ep1.p;
    n.radius = radius.p;
    n.phi = phi.p;
    n.center = center.p;
    n.q = q.p;
    n.coef = coef.p;
    n.wcoef = wcoef.p;
    n.err = err.p;
    n.err_old = err_old.p;
    n.err_old2 = err_old2.p;
    n.err_coef = err_coef.p;
    n.dpsi_corr = dpsi_corr.p;
    n.t = t.p;
    n.constant = constant.p;
    n.fptr = fptr.p;
    n.felem = felem.p;
    n.de_ids = de_ids.p;
    n.zint0 = zint0.p;
    n.zint1 = zint1.p;
    n.cut_cap = cut_cap;
    n.cut_n = cut_n.p;
    n.cut_pos = cut_pos.p;
    n.cut_elem = cut_elem.p;
    n.cut_sign = cut_sign.p;
    n.pinv = pinv.p;
    n.qcol = qcol.p;
    n.l_ptr = nullptr;
    n.l_col = nullptr;
    n.u_ptr = nullptr;
    n.u_col = nullptr;
    n.l_val = nullptr;
    n.u_val = nullptr;
    n.u_inv = nullptr;
    n.disc = disc.p;
    n.work = work.p;
    n.bvec = bvec.p;
    n.ready = ready.p;
    n.R = R;
    n.st = st.p;
    n.real_elem = real_elem.p;
    n.real_frac = real_frac.p;
    n.real_row = real_row.p;
    n.eoff = eoff.p;
    n.row_de = row_de.p;
    n.row_frac = row_frac.p;
    n.ndone = ndone.p;
    n.tri = tri.p;
    n.bknown = has_spec ? bknown.p : nullptr;
    n.dft_tab = dft_tab.p;
    n.dft_off = dft_off.p;
    return n;
  }
  ~AndfnHandle() {
    if (order_thread.joinable()) order_thread.join();
    if (dlu_ev) cudaEventDestroy(dlu_ev);
    if (mv_ev) cudaEventDestroy(mv_ev);
    if (pin_schur) pinned_put(pin_schur, sizeof(double) * pin_schur_n);
    andfn::destroy_adj(adj);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (loop_exec) cudaGraphExecDestroy(loop_exec);
    for (auto &b : ev)
      for (auto &c : b)
        for (auto &e : c)
          if (e) cudaEventDestroy(e);
    if (h_ndone) cudaFreeHost(h_ndone);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace andfn {

static inline int64_t rd_i64(const char *rec, int64_t off) {
  int64_t v;
  std::memcpy(&v, rec + off, 8);
  return v;
}
static inline double rd_f64(const char *rec, int64_t off) {
  double v;
  std::memcpy(&v, rec + off, 8);
  return v;
}
static inline cd rd_cd(const char *rec, int64_t off, int k) {
  cd v;
  std::memcpy(&v, rec + off + 16 * k, 16);
  return v;
}

static int check_layout(const AndfnLayout *L) {
  if (!L || L->elem_size <= 0 || L->frac_size <= 0 || L->max_ncoef <= 0 || L->max_elements <= 0) return 1;
  const int64_t eo[] = {L->e_id, L->e_type, L->e_frac0, L->e_frac1, L->e_radius, L->e_head, L->e_phi, L->e_ncoef,
                        L->e_nint, L->e_q, L->e_error, L->e_error_old, L->e_error_old2, L->e_error_coef};
  for (int64_t o : eo)
    if (o < 0 || o + 8 > L->elem_size) return 1;
  if (L->e_endpoints0 < 0 || L->e_endpoints0 + 32 > L->elem_size) return 1;
  if (L->e_endpoints1 < 0 || L->e_endpoints1 + 32 > L->elem_size) return 1;
  if (L->e_center < 0 || L->e_center + 16 > L->elem_size) return 1;
  if (L->e_coef < 0 || L->e_coef + 16 * L->max_ncoef > L->elem_size) return 1;
  if (L->e_thetas < 0 || L->e_thetas + 16 * L->max_ncoef > L->elem_size) return 1;
  if (L->e_dpsi_corr < 0 || L->e_dpsi_corr + 16 * L->max_ncoef > L->elem_size) return 1;
  const int64_t fo[] = {L->f_id, L->f_t, L->f_radius, L->f_nelements, L->f_constant};
  for (int64_t o : fo)
    if (o < 0 || o + 8 > L->frac_size) return 1;
  if (L->f_elements < 0 || L->f_elements + 8 * L->max_elements > L->frac_size) return 1;
  return 0;
}

// Appends realization r's records to the host SoA (ids shifted by the
// realization's offsets) and validates them.
static int parse_records(AndfnHandle *H, int r, const char *F, int64_t nf, const char *E, int64_t ne) {
  const AndfnLayout &L = H->L;
  HostNet &h = H->h;
  const int e0 = h.eoff[r], f0 = h.foff[r];
  int maxm = 0;
  for (int64_t i = 0; i < ne; i++) {
    const char *rec = E + i * L.elem_size;
    if (rd_i64(rec, L.e_id) != i) {
      set_error("element _id must equal its index (andfn/dfn.py:1062-1063)");
      return ANDFN_BAD_INPUT;
    }
    int64_t ty = rd_i64(rec, L.e_type);
    if (ty < 0 || ty > 5) {
      set_error("element type out of range");
      return ANDFN_BAD_INPUT;
    }
    int64_t fa = rd_i64(rec, L.e_frac0), fb = rd_i64(rec, L.e_frac1);
    if (fa < 0 || fa >= nf || (ty == 0 && (fb < 0 || fb >= nf))) {
      set_error("element fracture id out of range");
      return ANDFN_BAD_INPUT;
    }
    int64_t m = rd_i64(rec, L.e_ncoef), n = rd_i64(rec, L.e_nint);
    if (m < 0 || m > L.max_ncoef || n < 0 || n > 2 * L.max_ncoef || (ty != 2 && (m < 1 || n < 2))) {
      set_error("ncoef/nint out of range for the record capacity");
      return ANDFN_BAD_INPUT;
    }
    h.type.push_back((int)ty);
    h.frac0.push_back(f0 + (int)fa);
    h.frac1.push_back(ty == 0 ? f0 + (int)fb : -1);
    h.ncoef.push_back((int)m);
    h.nint.push_back((int)n);
    maxm = std::max(maxm, (int)m);
    h.ep0.push_back(rd_cd(rec, L.e_endpoints0, 0));
    h.ep0.push_back(rd_cd(rec, L.e_endpoints0, 1));
    h.ep1.push_back(rd_cd(rec, L.e_endpoints1, 0));
    h.ep1.push_back(rd_cd(rec, L.e_endpoints1, 1));
    h.center.push_back(rd_cd(rec, L.e_center, 0));
    h.radius.push_back(rd_f64(rec, L.e_radius));
    h.phi.push_back(rd_f64(rec, L.e_phi));
    h.q.push_back(rd_f64(rec, L.e_q));
    h.err.push_back(rd_f64(rec, L.e_error));
    h.err_old.push_back(rd_f64(rec, L.e_error_old));
    h.err_old2.push_back(rd_f64(rec, L.e_error_old2));
    h.err_coef.push_back(rd_f64(rec, L.e_error_coef));
    h.head.push_back(rd_f64(rec, L.e_head));
    h.spec_q.push_back(ty == 2 && std::isnan(h.head.back()) ? 1 : 0);
    if (h.spec_q.back() && !std::isfinite(h.q.back())) {
      set_error("a well with a prescribed discharge (NaN head) needs a finite q");
      return ANDFN_BAD_INPUT;
    }
    h.real_elem.push_back(r);
  }
  H->MC = std::max(H->MC, std::max(1, maxm));
  for (int64_t f = 0; f < nf; f++) {
    const char *rec = F + f * L.frac_size;
    if (rd_i64(rec, L.f_id) != f) {
      set_error("fracture _id must equal its index (andfn/dfn.py:1119-1120)");
      return ANDFN_BAD_INPUT;
    }
    h.t.push_back(rd_f64(rec, L.f_t));
    h.constant.push_back(rd_f64(rec, L.f_constant));
    int64_t nel = rd_i64(rec, L.f_nelements);
    if (nel < 0 || nel > L.max_elements) {
      set_error("fracture nelements out of range");
      return ANDFN_BAD_INPUT;
    }
    for (int64_t k = 0; k < nel; k++) {
      int64_t el = rd_i64(rec, L.f_elements + 8 * k);
      if (el < 0 || el >= ne) {
        set_error("fracture element id out of range");
        return ANDFN_BAD_INPUT;
      }
      h.felem.push_back(e0 + (int)el);
    }
    h.fptr.push_back((int)h.felem.size());
    h.real_frac.push_back(r);
  }
  // discharge elements (types 0, 2, 3 in element order) and system rows
  h.elem_de.resize(h.type.size(), -1);
  const int d0 = (int)h.de_ids.size();
  for (int64_t i = 0; i < ne; i++) {
    const int ty = h.type[e0 + i];
    if ((ty == 0 || ty == 2 || ty == 3) && !h.spec_q[e0 + i]) {
      h.elem_de[e0 + i] = (int)h.de_ids.size();
      h.de_ids.push_back(e0 + (int)i);
    }
  }
  const int nde = (int)h.de_ids.size() - d0;
  for (int j = 0; j < nde; j++) {
    h.row_de.push_back(d0 + j);
    h.row_frac.push_back(-1);
    h.real_row.push_back(r);
  }
  for (int64_t f = 0; f < nf; f++) {
    h.row_de.push_back(-1);
    h.row_frac.push_back(f0 + (int)f);
    h.real_row.push_back(r);
  }
  h.eoff[r + 1] = e0 + (int)ne;
  h.foff[r + 1] = f0 + (int)nf;
  h.doff[r + 1] = (int)h.de_ids.size();
  h.roff[r + 1] = h.roff[r] + nde + (int)nf;
  return 0;
}

static void read_coefs(AndfnHandle *H, int r, const char *E) {
  const AndfnLayout &L = H->L;
  const int e0 = H->h.eoff[r], e1 = H->h.eoff[r + 1];
  for (int i = e0; i < e1; i++) {
    const char *rec = E + (int64_t)(i - e0) * L.elem_size;
    const int m = H->h.ncoef[i];
    for (int k = 0; k < m && k < H->MC; k++) H->h.coef[(size_t)i * H->MC + k] = rd_cd(rec, L.e_coef, k);
  }
}

static thread_local int64_t g_h2d_bytes = 0, g_d2h_bytes = 0;

static double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Phase trace: with ANDFN_B200_TRACE set (to anything but 0), the host
// phases of handle creation and of a run's set-up print their wall time to
// stderr as they end (host time; a phase that waits for the stream includes
// the device work queued before it).
static bool trace_on() {
  static const bool on = [] {
    const char *e = getenv("ANDFN_B200_TRACE");
    return e && atoi(e) != 0;
  }();
  return on;
}

struct PhaseTimer {
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  void lap(const char *name) {
    if (trace_on()) fprintf(stderr, "[andfn_b200] %-28s %8.3f ms\n", name, ms_since(t));
    t = std::chrono::steady_clock::now();
  }
};

template <class T>
static cudaError_t upload(DBuf<T> &d, const std::vector<T> &v, cudaStream_t s) {
  cudaError_t e = d.alloc(v.size());
  if (e != cudaSuccess || v.empty()) return e;
  g_h2d_bytes += (int64_t)(sizeof(T) * v.size());
  return cudaMemcpyAsync(d.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s);
}

// Discharge-system pattern of realization r, row by row exactly as
// fill_discharge_matrix (hpc_solve.py:1117-1201) orders it; local indices
// (rows: its discharge elements then its fractures).  The assembly entries are
// appended to the global arrays (global row, global source element).
static void build_pattern(AndfnHandle *H, int r) {
  const HostNet &h = H->h;
  RealSys &S = H->sys[r];
  const int d0 = h.doff[r], d1 = h.doff[r + 1], f0 = h.foff[r], f1 = h.foff[r + 1];
  const int n_de = d1 - d0, nf = f1 - f0, row0 = h.roff[r];
  S.n_de = n_de;
  S.n = n_de + nf;
  S.mrow_ptr.assign(1, 0);
  S.mcol.clear();
  S.ent0 = (int)H->ent_row.size();
  auto disch = [&](int ty) { return ty == 0 || ty == 2 || ty == 3; };
  for (int j = 0; j < n_de; j++) {
    const int e = h.de_ids[d0 + j];
    const int sides = (h.type[e] == 0) ? 2 : 1;
    for (int s = 0; s < sides; s++) {
      const int f = s ? h.frac1[e] : h.frac0[e];
      for (int k = h.fptr[f]; k < h.fptr[f + 1]; k++) {
        const int ee = h.felem[k];
        if (ee == e || !disch(h.type[ee])) continue;
        if (h.spec_q[ee]) {  // prescribed discharge: a known term of the row
          H->known_row.push_back(row0 + j);
          H->known_src.push_back(ee);
          H->known_side.push_back(s);
          continue;
        }
        S.mcol.push_back(h.elem_de[ee] - d0);
        H->ent_row.push_back(row0 + j);
        H->ent_src.push_back(ee);
        H->ent_side.push_back(s);
        H->ent_kind.push_back(0);
      }
    }
    for (int s = 0; s < sides; s++) {
      const int f = s ? h.frac1[e] : h.frac0[e];
      S.mcol.push_back(n_de + (f - f0));
      H->ent_row.push_back(row0 + j);
      H->ent_src.push_back(-1);
      H->ent_side.push_back(s);
      H->ent_kind.push_back(1);
    }
    S.mrow_ptr.push_back((int)S.mcol.size());
  }
  for (int f = f0; f < f1; f++) {
    for (int k = h.fptr[f]; k < h.fptr[f + 1]; k++) {
      const int el = h.felem[k];
      if (!disch(h.type[el])) continue;
      if (h.spec_q[el]) {  // +q of the well in its fracture's continuity row
        H->known_cont_row.push_back(row0 + n_de + (f - f0));
        H->known_cont_src.push_back(el);
        continue;
      }
      S.mcol.push_back(h.elem_de[el] - d0);
      H->ent_row.push_back(row0 + n_de + (f - f0));
      H->ent_src.push_back(el);
      H->ent_side.push_back(0);
      H->ent_kind.push_back(2);
    }
    S.mrow_ptr.push_back((int)S.mcol.size());
  }
}

// CSC of realization r's system with the given entry values (vals indexed by
// global assembly entry).
static CscMatrix system_csc(const RealSys &S, const double *vals) {
  CscMatrix A;
  A.n = S.n;
  A.colptr.assign(S.n + 1, 0);
  for (int c : S.mcol) A.colptr[c + 1]++;
  for (int i = 0; i < S.n; i++) A.colptr[i + 1] += A.colptr[i];
  A.rowind.resize(S.mcol.size());
  A.val.resize(S.mcol.size());
  std::vector<int> fill(A.colptr.begin(), A.colptr.end() - 1);
  for (int rr = 0; rr < S.n; rr++)
    for (int p = S.mrow_ptr[rr]; p < S.mrow_ptr[rr + 1]; p++) {
      const int c = S.mcol[p];
      A.rowind[fill[c]] = rr;
      A.val[fill[c]++] = vals ? vals[S.ent0 + p] : 1.0;
    }
  return A;
}

static void build_tables(AndfnHandle *H, bool rhs, std::vector<Group> &groups, std::vector<int> &index_of,
                         std::vector<Item> &items, std::vector<int2> &pts, int &nvals,
                         const std::vector<char> *only = nullptr, std::vector<int> *fpt0 = nullptr,
                         std::vector<int> *fnp = nullptr) {
  const HostNet &h = H->h;
  const std::vector<int> &cnint = H->cur_nint;
  const std::vector<int> &cncoef = H->cur_ncoef;
  const int ne = (int)H->ne, nf = (int)H->nf;
  const int D = (int)H->D;
  const int n_de = (int)h.de_ids.size();
  // per fracture, the groups whose points lie in it
  std::vector<std::vector<int>> per_frac(nf);
  nvals = 0;
  if (!rhs) {
    index_of.assign(2 * (size_t)ne, -1);
    for (int e = 0; e < ne; e++) {
      const int ty = h.type[e];
      if (ty == 2) continue;
      if (only && !(*only)[e]) continue;
      const int sides = (ty == 0) ? 2 : 1;
      for (int s = 0; s < sides; s++) {
        Group g;
        g.elem = e;
        g.side = s;
        g.frac = s ? h.frac1[e] : h.frac0[e];
        g.npts = cnint[e];
        g.kind = (ty == 1 || ty == 4 || ty == 5) ? KIND_PSI : KIND_PHI;
        g.out = nvals;
        g.pad0 = g.pad1 = 0;
        nvals += g.npts;
        index_of[2 * (size_t)e + s] = (int)groups.size();
        per_frac[g.frac].push_back((int)groups.size());
        groups.push_back(g);
      }
    }
  } else {
    index_of.assign(2 * (size_t)n_de, -1);
    for (int j = 0; j < n_de; j++) {
      const int e = h.de_ids[j];
      const int sides = (h.type[e] == 0) ? 2 : 1;
      for (int s = 0; s < sides; s++) {
        Group g;
        g.elem = j;  // row index (z_int is per discharge element)
        g.side = s;
        g.frac = s ? h.frac1[e] : h.frac0[e];
        g.npts = D;
        g.kind = KIND_PHI;
        g.out = nvals;
        g.pad0 = g.pad1 = 0;
        nvals += D;
        index_of[2 * (size_t)j + s] = (int)groups.size();
        per_frac[g.frac].push_back((int)groups.size());
        groups.push_back(g);
      }
    }
  }
  // flatten: within a fracture, PSI groups first (bounding circles lead the
  // element order) so mixed warps are rare
  struct Cost {
    double c;
    Item it;
  };
  std::vector<Cost> costs;
  for (int f = 0; f < nf; f++) {
    auto &gl = per_frac[f];
    std::stable_sort(gl.begin(), gl.end(), [&](int a, int b) { return groups[a].kind > groups[b].kind; });
    const int start = (int)pts.size();
    for (int gi : gl)
      for (int k = 0; k < groups[gi].npts; k++) pts.push_back(make_int2(gi, k));
    const int end = (int)pts.size();
    if (fpt0) fpt0->push_back(start);
    if (fnp) fnp->push_back(end - start);
    double work_per_pt = 0.0;
    for (int k = h.fptr[f]; k < h.fptr[f + 1]; k++) work_per_pt += 30.0 + 4.0 * cncoef[h.felem[k]];
    for (int p = start; p < end; p += EVAL_THREADS) {
      Item it;
      it.frac = f;
      it.p0 = p;
      it.p1 = std::min(end, p + EVAL_THREADS);
      it.pad = 0;
      costs.push_back({work_per_pt * (it.p1 - it.p0), it});
    }
  }
  std::stable_sort(costs.begin(), costs.end(), [](const Cost &a, const Cost &b) { return a.c > b.c; });
  for (auto &c : costs) items.push_back(c.it);
}


static int reset_impl(AndfnHandle *H);

// Sweep / head-vector tables for the current ncoef and nint, uploaded.
// DFT bases of the elements' Cauchy-integral fits, one per (nint, theta
// layout) in use: entry (k, j) = exp_m[k]^j, exp_m[k] = exp(-i theta_k),
// theta_k = start + k del (del = pi / n, start = del / 2; del = 2 pi / n,
// start = 0 for bounding circles), the powers formed by repeated complex
// multiplication from 1 as the reference forms them
// (hpc_math_functions.py:244-297, 674-723).
static int build_dft_tables(AndfnHandle *H) {
  const HostNet &h = H->h;
  const int ne = (int)H->ne, MC = H->MC;
  std::map<std::pair<int, int>, int> where;
  std::vector<cd> tab;
  std::vector<int> off(std::max(1, ne), 0);
  for (int e = 0; e < ne; e++) {
    if (h.type[e] == 2) continue;
    const int n = H->cur_nint[e], kind = (h.type[e] == 1) ? 1 : 0;
    auto it = where.find({n, kind});
    if (it == where.end()) {
      const int o = (int)tab.size();
      it = where.emplace(std::make_pair(n, kind), o).first;
      tab.resize(tab.size() + (size_t)n * MC);
      const double del = kind ? 2 * PI / n : PI / n, start = kind ? 0.0 : del / 2;
      for (int k = 0; k < n; k++) {
        const double th = start + k * del;
        const double er = std::cos(-th), ei = std::sin(-th);
        double pr = 1.0, pi = 0.0;
        for (int j = 0; j < MC; j++) {
          tab[(size_t)o + (size_t)k * MC + j] = mk(pr, pi);
          const double nr = pr * er - pi * ei, ni = pr * ei + pi * er;
          pr = nr;
          pi = ni;
        }
      }
    }
    off[e] = it->second;
  }
  if (tab.empty()) tab.push_back(mk(0.0, 0.0));
  CK(upload(H->dft_tab, tab, H->stream));
  CK(upload(H->dft_off, off, H->stream));
  return 0;
}

static int build_eval_tables(AndfnHandle *H) {
  HostNet &h = H->h;
  cudaStream_t s = H->stream;
  const int ne = (int)H->ne;
  {
    const int rcd = build_dft_tables(H);
    if (rcd) return rcd;
  }
  std::vector<Group> groups;
  std::vector<int> group_of, rhs_group;
  std::vector<Item> sitems, ritems;
  std::vector<int2> spts, rpts;
  int nsv = 0, nrv = 0;
  std::vector<int> fpt0, fnp;
  build_tables(H, false, groups, group_of, sitems, spts, nsv, nullptr, &fpt0, &fnp);
  build_tables(H, true, groups, rhs_group, ritems, rpts, nrv);
  // pair tables: per fracture, (sources) x (points of the fracture)
  {
    const int nf = (int)H->nf;
    std::vector<long long> off(nf + 1, 0);
    for (int f = 0; f < nf; f++) off[f + 1] = off[f] + (long long)(h.fptr[f + 1] - h.fptr[f]) * fnp[f];
    H->tab_pairs = off[nf];
    CK(upload(H->tab_off, off, s));
    CK(upload(H->tab_fpt0, fpt0, s));
    CK(upload(H->tab_fnp, fnp, s));
    H->h_tab_fpt0 = fpt0;
    H->h_tab_fnp = fnp;
    const size_t np = (size_t)std::max<long long>(1, H->tab_pairs);
    if (H->tab_w.cap < np) CK(H->tab_w.alloc(np));
    if (H->tab_l.cap < np) CK(H->tab_l.alloc(np));
    H->tab_valid = false;
  }
  H->groups = groups;
  CK(upload(H->d_groups, groups, s));
  CK(upload(H->group_of, group_of, s));
  CK(upload(H->rhs_group, rhs_group, s));
  CK(upload(H->sweep_items, sitems, s));
  CK(upload(H->rhs_items, ritems, s));
  CK(upload(H->sweep_pts, spts, s));
  CK(upload(H->rhs_pts, rpts, s));
  H->n_sweep_items = (int)sitems.size();
  H->n_rhs_items = (int)ritems.size();
  if (H->sweep_vals.cap < (size_t)std::max(1, nsv)) CK(H->sweep_vals.alloc(std::max(1, nsv)));
  if (H->rhs_vals.cap < (size_t)std::max(1, nrv)) CK(H->rhs_vals.alloc(std::max(1, nrv)));
  std::vector<int> upd, psi;
  int nvmax = 2;
  for (int e = 0; e < ne; e++) {
    upd.push_back(e);
    if (h.type[e] == 1 || h.type[e] == 4 || h.type[e] == 5) psi.push_back(e);
    nvmax = std::max(nvmax, H->cur_nint[e]);
  }
  H->n_upd = (int)upd.size();
  H->n_psi = (int)psi.size();
  H->nvmax = nvmax;
  CK(upload(H->upd_list, upd, s));
  CK(upload(H->psi_list, psi, s));
  // eval staging: sources per chunk within the shared-memory budget
  int maxnf = 1;
  for (int f = 0; f < (int)H->nf; f++) maxnf = std::max(maxnf, h.fptr[f + 1] - h.fptr[f]);
  const size_t budget = 96 * 1024;
  int chunk = (int)(budget / (sizeof(Src) + sizeof(cd) * H->MC));
  chunk = std::max(1, std::min(chunk, maxnf));
  H->chunk = chunk;
  H->eval_smem = (sizeof(Src) + sizeof(cd) * H->MC) * chunk;
  // table sweep staging: at most 48 KB of sources per CTA (every source of
  // the largest fracture when they fit)
  int tchunk = (int)((48 * 1024) / (sizeof(TabSrc) + sizeof(cd) * H->MC));
  tchunk = std::max(2, std::min(tchunk, maxnf));
  H->tab_chunk = tchunk;
  H->tab_smem = (sizeof(TabSrc) + sizeof(cd) * H->MC) * tchunk;
  CK(cudaStreamSynchronize(s));
  H->tables_dirty = false;
  return 0;
}

// Coefficient capacity per element on the device (>= the largest ncoef the
// run can reach); re-strides the stored initial coefficients when it grows.
static int ensure_capacity(AndfnHandle *H, int mc) {
  if (mc <= H->MC) return 0;
  const int old = H->MC;
  std::vector<cd> nc((size_t)H->ne * mc, mk(0.0, 0.0));
  for (int64_t i = 0; i < H->ne; i++)
    for (int k = 0; k < old; k++) nc[(size_t)i * mc + k] = H->h.coef[(size_t)i * old + k];
  H->h.coef.swap(nc);
  H->MC = mc;
  cudaStream_t s = H->stream;
  CK(upload(H->coef0, H->h.coef, s));
  CK(H->coef.alloc((size_t)H->ne * mc));
  CK(H->wcoef.alloc((size_t)H->ne * mc));
  CK(H->dpsi_corr.alloc((size_t)H->ne * 2 * mc));
  H->tables_dirty = true;
  return 0;
}

static int create_impl(AndfnHandle *H, int R, const char *const *F, const int64_t *nf, const char *const *E,
                       const int64_t *ne) {
  auto tc0 = std::chrono::steady_clock::now();
  HostNet &h = H->h;
  H->R = R;
  h.eoff.assign(R + 1, 0);
  h.foff.assign(R + 1, 0);
  h.doff.assign(R + 1, 0);
  h.roff.assign(R + 1, 0);
  h.fptr.assign(1, 0);
  H->MC = 1;
  PhaseTimer pt;
  for (int r = 0; r < R; r++) {
    int rc = parse_records(H, r, F[r], nf[r], E[r], ne[r]);
    if (rc) return rc;
  }
  pt.lap("create: parse records");
  H->ne = h.eoff[R];
  H->nf = h.foff[R];
  H->N = h.roff[R];
  // discharge systems: patterns, then fill-reducing column orders from the
  // patterns alone, computed once per network (in parallel over
  // realizations) on a host thread of their own; nothing before the first
  // factorisation reads them
  H->sys.assign(R, RealSys());
  H->ent_row.clear();
  H->ent_src.clear();
  H->ent_side.clear();
  H->ent_kind.clear();
  for (int r = 0; r < R; r++) build_pattern(H, r);
  H->known0 = (int)H->ent_row.size();
  for (size_t k = 0; k < H->known_row.size(); k++) {
    H->ent_row.push_back(H->known_row[k]);
    H->ent_src.push_back(H->known_src[k]);
    H->ent_side.push_back(H->known_side[k]);
    H->ent_kind.push_back(0);
  }
  for (char c : H->h.spec_q) H->has_spec |= (c != 0);
  pt.lap("create: system patterns");
  // batches whose realizations the device inverts need no column order; it
  // is computed on first use if a run falls back to the sparse LU
  int maxn_sys = 0;
  for (int r = 0; r < R; r++) maxn_sys = std::max(maxn_sys, H->sys[r].n);
  const bool skip_order =
      R > 1 && H->winv_enabled && maxn_sys <= BINV_MAX_N && binv_cluster_smem(maxn_sys) <= BINV_CLUSTER_SMEM_MAX;
  // the ordering hands the remaining columns to the dense tail once the
  // minimum degree reaches this fraction of what remains: 0.15 balances the
  // host's serial sparse LU against the device's dense LU (2,118-fracture
  // network: 41.6 ms a solve at 0.4, 38.5 ms at 0.15, 38.7 ms at 0.1)
  double dense_frac = 0.15;
  if (const char *v = getenv("ANDFN_B200_DENSE_FRAC")) {
    const double x = atof(v);
    if (x > 0.0 && x <= 1.0) dense_frac = x;
  }
  H->dense_frac = dense_frac;
  H->order_follow = R == 1 && !skip_order;
  if (H->order_follow) H->order_prog.reset(H->sys[0].n);
  H->order_thread = std::thread([H, R, skip_order, dense_frac]() {
    auto tc2 = std::chrono::steady_clock::now();
    if (!skip_order) {
#pragma omp parallel for schedule(dynamic, 1) if (R > 1)
      for (int r = 0; r < R; r++) {
        CscMatrix P = system_csc(H->sys[r], nullptr);
        H->sys[r].colorder = column_min_degree_order(P, &H->sys[r].dense_k, dense_frac, 3072,
                                                     H->order_follow ? &H->order_prog : nullptr);
      }
    }
    H->ms_create_order = ms_since(tc2);
    if (trace_on()) fprintf(stderr, "[andfn_b200] %-28s %8.3f ms\n", "create: column orders (thread)", H->ms_create_order);
  });
  h.coef.assign((size_t)H->ne * H->MC, mk(0.0, 0.0));
  for (int r = 0; r < R; r++) read_coefs(H, r, E[r]);
  cudaStream_t s = H->stream;
  const int nel = (int)H->ne;
  CK(upload(H->type, h.type, s));
  CK(upload(H->frac0, h.frac0, s));
  CK(upload(H->frac1, h.frac1, s));
  CK(upload(H->ncoef0, h.ncoef, s));
  CK(upload(H->nint0, h.nint, s));
  CK(H->ncoef.alloc(nel));
  CK(H->nint.alloc(nel));
  CK(upload(H->ep0, h.ep0, s));
  CK(upload(H->ep1, h.ep1, s));
  CK(upload(H->center, h.center, s));
  CK(upload(H->radius, h.radius, s));
  CK(upload(H->phi, h.phi, s));
  CK(upload(H->q0, h.q, s));
  CK(H->q.alloc(nel));
  CK(upload(H->coef0, h.coef, s));
  CK(H->coef.alloc((size_t)nel * H->MC));
  CK(H->wcoef.alloc((size_t)nel * H->MC));
  CK(upload(H->err_in, h.err, s));
  CK(upload(H->err_old_in, h.err_old, s));
  CK(upload(H->err_old2_in, h.err_old2, s));
  CK(upload(H->err_coef_in, h.err_coef, s));
  CK(H->err.alloc(nel));
  CK(H->err_old.alloc(nel));
  CK(H->err_old2.alloc(nel));
  CK(H->err_coef.alloc(nel));
  CK(H->dpsi_corr.alloc((size_t)nel * 2 * H->MC));
  CK(upload(H->t, h.t, s));
  CK(upload(H->constant0, h.constant, s));
  CK(H->constant.alloc(h.constant.size()));
  CK(upload(H->fptr, h.fptr, s));
  CK(upload(H->felem, h.felem, s));
  CK(upload(H->de_ids, h.de_ids, s));
  CK(upload(H->real_elem, h.real_elem, s));
  CK(upload(H->real_frac, h.real_frac, s));
  CK(upload(H->real_row, h.real_row, s));
  CK(upload(H->eoff, h.eoff, s));
  CK(upload(H->row_de, h.row_de, s));
  CK(upload(H->row_frac, h.row_frac, s));
  CK(H->ndone.alloc(1));
  const int n_de = (int)h.de_ids.size();
  CK(H->zint0.alloc((size_t)std::max(1, n_de) * H->D));
  CK(H->zint1.alloc((size_t)std::max(1, n_de) * H->D));
  // branch-cut capacity: crossings per psi element are bounded by twice the
  // discharge elements of its fracture
  int maxd = 0;
  for (int f = 0; f < (int)H->nf; f++) {
    int c = 0;
    for (int k = h.fptr[f]; k < h.fptr[f + 1]; k++) {
      int ty = h.type[h.felem[k]];
      c += (ty == 0 || ty == 2 || ty == 3);
    }
    maxd = std::max(maxd, c);
  }
  H->cut_cap = 2 * maxd + 4;
  CK(H->cut_n.alloc(nel));
  CK(H->cut_pos.alloc((size_t)nel * H->cut_cap));
  CK(H->cut_elem.alloc((size_t)nel * H->cut_cap));
  CK(H->cut_sign.alloc((size_t)nel * H->cut_cap));
  CK(upload(H->d_ent_row, H->ent_row, s));
  CK(upload(H->d_ent_src, H->ent_src, s));
  CK(upload(H->d_ent_side, H->ent_side, s));
  CK(upload(H->d_ent_kind, H->ent_kind, s));
  CK(H->d_mvals.alloc(std::max<size_t>(1, H->ent_row.size())));
  H->ms_create_upload = ms_since(tc0);
  pt.lap("create: uploads");
  auto tc1 = std::chrono::steady_clock::now();
  H->cur_ncoef = h.ncoef;
  H->cur_nint = h.nint;
  int rc = build_eval_tables(H);
  if (rc) return rc;
  H->ms_create_tables = ms_since(tc1);
  pt.lap("create: evaluation tables");
  CK(H->disc.alloc(H->N));
  CK(H->work.alloc(H->N));
  CK(H->bvec.alloc(H->N));
  CK(H->ready.alloc(H->N));
  CK(H->st.alloc(R));
  if (R == 1) {  // partial results of the split reduction, one per CTA
    CK(H->red_parts.alloc((H->ne + REDUCE_SPLIT_ELEMS - 1) / REDUCE_SPLIT_ELEMS));
    CK(H->red_ticket.alloc(1));
    CK(cudaMemsetAsync(H->red_ticket.p, 0, sizeof(unsigned), s));
  }
  H->h_st.assign(R, SolveState());
  if (!H->h_ndone) CK(cudaMallocHost(&H->h_ndone, sizeof(int)));
  CK(cudaFuncSetAttribute(eval_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  CK(cudaFuncSetAttribute(eval_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  CK(cudaFuncSetAttribute(sweep_table_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  CK(cudaFuncSetAttribute(trisolve_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  CK(cudaFuncSetAttribute(trisolve_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  CK(cudaFuncSetAttribute(dense_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  CK(cudaFuncSetAttribute(dlu_panel_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DLU_SMEM_MAX));
  CK(cudaFuncSetAttribute(winv_gemv_kernel<0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(sizeof(double) * WINV_MAX_N)));
  CK(cudaFuncSetAttribute(winv_gemv_kernel<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(sizeof(double) * WINV_MAX_N)));
  CK(cudaFuncSetAttribute(winv_gemv_kernel<0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(sizeof(double) * WINV_MAX_N)));
  CK(cudaFuncSetAttribute(winv_gemv_kernel<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(sizeof(double) * WINV_MAX_N)));
  CK(cudaFuncSetAttribute(winv_gemv_kernel<1, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(sizeof(double) * WINV_MAX_N)));
  CK(cudaFuncSetAttribute(winv_gemv_kernel<1, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(sizeof(double) * WINV_MAX_N)));
  CK(cudaFuncSetAttribute(update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  rc = reset_impl(H);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s));
  return 0;
}

// Copies the initial state into the working arrays.
static int reset_impl(AndfnHandle *H) {
  cudaStream_t s = H->stream;
  const size_t ne = H->ne;
  CK(cudaMemcpyAsync(H->ncoef.p, H->ncoef0.p, sizeof(int) * ne, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(H->nint.p, H->nint0.p, sizeof(int) * ne, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(H->q.p, H->q0.p, sizeof(double) * ne, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(H->coef.p, H->coef0.p, sizeof(cd) * ne * H->MC, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(H->err.p, H->err_in.p, sizeof(double) * ne, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(H->err_old.p, H->err_old_in.p, sizeof(double) * ne, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(H->err_old2.p, H->err_old2_in.p, sizeof(double) * ne, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(H->err_coef.p, H->err_coef_in.p, sizeof(double) * ne, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(H->constant.p, H->constant0.p, sizeof(double) * H->nf, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemsetAsync(H->dpsi_corr.p, 0, sizeof(double) * ne * 2 * H->MC, s));
  return 0;
}

// Groups rows [row_lo, row_hi) of a triangular factor by dependency level and
// stores their entries with columns in [col_lo, col_hi) in that order
// (level_solve reads one contiguous range per level).  single_level puts all
// rows in one level (the coupling terms between the sparse part and the dense
// tail, whose rows are independent).
static void build_levels(int n, const std::vector<int> &ptr, const std::vector<int> &col,
                         const std::vector<double> &val, const std::vector<double> *scale, bool lower, int row_lo,
                         int row_hi, int col_lo, int col_hi, bool single_level, std::vector<int> &lev_ptr,
                         std::vector<int> &rows, std::vector<int> &eptr, std::vector<int> &ecol,
                         std::vector<double> &evals, std::vector<double> &escale) {
  (void)n;
  const int nr = std::max(0, row_hi - row_lo);
  std::vector<int> lev(std::max(1, row_hi), 0);
  int nlev = nr > 0 ? 1 : 0;
  if (!single_level) {
    for (int t = 0; t < nr; t++) {
      const int i = lower ? row_lo + t : row_hi - 1 - t;
      int l = 0;
      for (int p = ptr[i]; p < ptr[i + 1]; p++) {
        const int c = col[p];
        if (c >= col_lo && c < col_hi && c >= row_lo && c < row_hi) l = std::max(l, lev[c] + 1);
      }
      lev[i] = l;
      nlev = std::max(nlev, l + 1);
    }
  }
  lev_ptr.assign(nlev + 1, 0);
  for (int i = row_lo; i < row_hi; i++) lev_ptr[lev[i] + 1]++;
  for (int l = 0; l < nlev; l++) lev_ptr[l + 1] += lev_ptr[l];
  rows.assign(nr, 0);
  std::vector<int> fill(lev_ptr.begin(), lev_ptr.end() - 1);
  for (int t = 0; t < nr; t++) {
    const int i = lower ? row_lo + t : row_hi - 1 - t;
    rows[fill[lev[i]]++] = i;
  }
  eptr.assign(nr + 1, 0);
  ecol.clear();
  evals.clear();
  escale.assign(nr, 1.0);
  for (int sl = 0; sl < nr; sl++) {
    const int i = rows[sl];
    for (int p = ptr[i]; p < ptr[i + 1]; p++) {
      if (col[p] < col_lo || col[p] >= col_hi) continue;
      ecol.push_back(col[p]);
      evals.push_back(val[p]);
    }
    eptr[sl + 1] = (int)ecol.size();
    if (scale) escale[sl] = (*scale)[i];
  }
}

// Lanes per factor row: the smallest group whose registers hold a mean row.
// A single-level part (the coupling terms, independent rows) takes narrower
// groups, so more rows are in flight at once.
static int group_for(const std::vector<int> &eptr, bool single = false) {
  const int n = (int)eptr.size() - 1;
  const double mean = n > 0 ? (double)eptr[n] / n : 0.0;
  if (single) {
    if (mean <= 16.0 * PF) return 4;
    if (mean <= 32.0 * PF) return 8;
    return 16;
  }
  if (mean <= 8.0 * PF) return 8;
  if (mean <= 16.0 * PF) return 16;
  return 32;
}

// Factorises every realization's system (in parallel over realizations) and
// uploads the level-ordered factor parts, dense tails, permutations and one
// TriDesc per realization.
// Factorises the Schur complement F.schur (K x K, host) on the device into H->tail_l
// (panels of DLU_NB columns, three launches each) and completes F from the
// pivots and U's diagonal.  Returns 3 for a singular block.
__global__ void recip_kernel(const double *__restrict__ d, double *__restrict__ out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = 1.0 / d[i];
}

// W = (L U)^-1 of a single network's dense tail (H->tail_l, 1/U(i,i) in
// H->tail_uinv) into H->tail_w.
static int launch_tail_inverse(AndfnHandle *H, int K) {
  cudaStream_t s = H->stream;
  CK(H->tail_w.alloc((size_t)K * K));
  // by blocks (ANDFN_B200_DINV_BLOCKED=0: a CTA per group of columns)
  const char *eb = getenv("ANDFN_B200_DINV_BLOCKED");
  if (!(eb && atoi(eb) == 0)) {
    double *W = H->tail_w.p;
    const double *LU = H->tail_l.p;
    identity_kernel<<<4 * H->num_sms, 256, 0, s>>>(W, K);
    const int nbk = (K + DINVB - 1) / DINVB;
    for (int i = 0; i < nbk; i++) {  // forward: Y = L^-1, lower triangular
      const int r0 = i * DINVB, nb = std::min(DINVB, K - r0), e = r0 + nb;
      dinvb_diag_kernel<true><<<(e + 7) / 8, 256, 0, s>>>(LU, nullptr, K, r0, nb, e, W);
      if (e < K)
        dinvb_gemm_kernel<<<dim3((K - e + 63) / 64, (e + 63) / 64), 256, 0, s>>>(LU, W, K, e, K - e, r0, nb, e);
    }
    for (int i = nbk - 1; i >= 0; i--) {  // backward: W = U^-1 Y
      const int r0 = i * DINVB, nb = std::min(DINVB, K - r0);
      dinvb_diag_kernel<false><<<(K + 7) / 8, 256, 0, s>>>(LU, H->tail_uinv.p, K, r0, nb, K, W);
      if (r0 > 0) dinvb_gemm_kernel<<<dim3((r0 + 63) / 64, (K + 63) / 64), 256, 0, s>>>(LU, W, K, 0, r0, r0, nb, K);
    }
    H->launches += 1 + 4 * nbk;
    CK(cudaGetLastError());
    return 0;
  }
  // about one CTA per SM (nc columns of the inverse each)
  const int nc = std::max(1, std::min({DINV_NC, (int)(200 * 1024 / (sizeof(double) * (size_t)K)), K / H->num_sms}));
  dense_inverse_kernel<<<(K + nc - 1) / nc, 256, sizeof(double) * (size_t)K * nc, s>>>(H->tail_l.p, H->tail_l.p,
                                                                                       H->tail_uinv.p, K, nc,
                                                                                       H->tail_w.p);
  CK(cudaGetLastError());
  return 0;
}

// With want_w the tail inverse is launched right after the LU (1/U(i,i)
// computed on the device, the same IEEE quotients as the host's), and the
// host waits only for the pivots, so the inverse runs while the host
// completes the factors and builds the level tables.
static int gpu_dense_lu(AndfnHandle *H, LuFactors &F, bool want_w) {
  const int K = F.dense;
  cudaStream_t s = H->stream;
  CK(H->tail_l.alloc((size_t)K * K));
  CK(cudaMemcpyAsync(H->tail_l.p, F.schur, sizeof(double) * (size_t)K * K, cudaMemcpyHostToDevice, s));
  g_h2d_bytes += (int64_t)(sizeof(double) * (size_t)K * K);
  CK(H->dlu_i.alloc((size_t)K + 8 * DLU_NB + 3));
  CK(H->dlu_d.alloc((size_t)K));
  int *ib = H->dlu_i.p;
  DluScratch D{ib, H->dlu_d.p, ib + K, ib + K + 4 * DLU_NB, ib + K + 8 * DLU_NB, ib + K + 8 * DLU_NB + 2};
  CK(cudaMemsetAsync(D.flag, 0, sizeof(int), s));
  double *S = H->tail_l.p;
  // one cooperative launch when the panel fits one CTA's shared memory and
  // every SM can hold a CTA (ANDFN_B200_DLU_COOP=0: the three launches a panel)
  bool coop = sizeof(double) * (DLU_NB + 1) * (size_t)K <= DLU_SMEM_MAX;
  if (const char *e = getenv("ANDFN_B200_DLU_COOP")) coop = coop && atoi(e) != 0;
  if (coop) {
    const size_t sm = dluc_smem(K);
    CK(cudaFuncSetAttribute(dlu_coop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dlu_coop_kernel, DLUC_THREADS, sm));
    coop = per_sm >= 1;
    if (coop) {
      if (H->dlu_sync.cap < 1) CK(H->dlu_sync.alloc(1));
      CK(cudaMemsetAsync(H->dlu_sync.p, 0, sizeof(DluSync), s));
      const int nblk = (K + DLU_NB - 1) / DLU_NB;
      if (H->dlu_colcnt.cap < (size_t)nblk) CK(H->dlu_colcnt.alloc(nblk));
      CK(cudaMemsetAsync(H->dlu_colcnt.p, 0, sizeof(unsigned) * nblk, s));
      DluSync *sy = H->dlu_sync.p;
      unsigned *colcnt = H->dlu_colcnt.p;
      int Kv = K;
      void *args[] = {(void *)&S, (void *)&Kv, (void *)&D, (void *)&sy, (void *)&colcnt};
      CK(cudaLaunchCooperativeKernel((void *)dlu_coop_kernel, dim3(H->num_sms), dim3(DLUC_THREADS), args, sm, s));
      H->launches += 1;
    }
  }
  for (int j0 = 0; j0 < K && !coop; j0 += DLU_NB) {
    const int nb = std::min(DLU_NB, K - j0), m = K - j0, mt = m - nb;
    const size_t sm = sizeof(double) * (size_t)m * (DLU_NB + 1);
    const int use_smem = sm <= DLU_SMEM_MAX;
    if (use_smem)
      dlu_panel_kernel<true><<<1, DLU_THREADS, sm, s>>>(S, K, j0, nb, D);
    else
      dlu_panel_kernel<false><<<1, DLU_THREADS, 0, s>>>(S, K, j0, nb, D);
    if (K > nb) dlu_update_kernel<<<(K - nb + 7) / 8, 256, 0, s>>>(S, K, j0, nb, D);
    if (mt > 0) dlu_gemm_kernel<<<dim3((mt + 63) / 64, (mt + 63) / 64), 256, 0, s>>>(S, K, j0, nb);
    H->launches += 1 + (K > nb) + (mt > 0);
  }
  CK(cudaGetLastError());
  CK(H->tail_uinv.alloc((size_t)K));
  recip_kernel<<<(K + 255) / 256, 256, 0, s>>>(D.diag, H->tail_uinv.p, K);
  std::vector<int> piv(K), flag(1);
  std::vector<double> dg(K);
  DluSync syh = {};
  CK(cudaMemcpyAsync(piv.data(), D.piv, sizeof(int) * K, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(dg.data(), D.diag, sizeof(double) * K, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(flag.data(), D.flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (coop) CK(cudaMemcpyAsync(&syh, H->dlu_sync.p, sizeof(DluSync), cudaMemcpyDeviceToHost, s));
  g_d2h_bytes += (int64_t)(12 * K + 4);
  if (!H->dlu_ev) CK(cudaEventCreateWithFlags(&H->dlu_ev, cudaEventDisableTiming));
  CK(cudaEventRecord(H->dlu_ev, s));
  if (want_w) {
    const int rc = launch_tail_inverse(H, K);
    if (rc) return rc;
  }
  CK(cudaEventSynchronize(H->dlu_ev));
  if (syh.err) {
    set_error("dense LU of the Schur complement: a grid barrier wait ran out");
    return ANDFN_CUDA_ERROR;
  }
  if (flag[0]) return 3;
  return sparse_lu_finish(F, piv, dg);
}

static float *make_winv_f32(AndfnHandle *H, DBuf<float> &Y, const double *X, size_t n);

// Forms the explicit inverse of a single network's factorised system (its
// TriDesc, dense-tail inverse in H->tail_w) when the device has room for it,
// and the CSR pattern of the system for the refinement step.
static int build_inverse(AndfnHandle *H, const TriDesc &td) {
  cudaStream_t s = H->stream;
  const int N = td.n, K = td.T.K, m0 = N - K;
  const int ldw = (N + 63) / 64 * 64;  // rows of 64-entry multiples: 512 B (double) / 256 B (float) aligned
  const size_t xbytes = sizeof(double) * (size_t)N * ldw, tbytes = sizeof(double) * (size_t)std::max(1, K) * ldw;
  // free device memory is queried only when the buffers have to grow (a
  // driver query per run would contend with monitoring tools)
  if (H->winv.cap < (size_t)N * ldw || H->winv_t.cap < (size_t)std::max(1, K) * ldw) {
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    const size_t have = fr + sizeof(double) * (H->winv.cap + H->winv_t.cap);
    if (xbytes + tbytes + ((size_t)1 << 30) > have) return 0;  // keep the triangular solves
  }
  CK(H->winv.alloc((size_t)N * ldw));
  CK(H->winv_t.alloc((size_t)std::max(1, K) * ldw));
  CK(cudaMemsetAsync(H->winv.p, 0, xbytes, s));
  const int nchunk = ldw / WINV_CW;
  winv_lower_kernel<<<nchunk, WINV_THREADS, 0, s>>>(td, H->winv.p, ldw, H->winv_t.p);
  if (K > 0) {
    winv_gemm_kernel<<<dim3((K + 127) / 128, (ldw + 63) / 64), 256, 0, s>>>(H->tail_w.p, K, H->winv_t.p, ldw,
                                                                          H->winv.p + (size_t)m0 * ldw);
    if (td.Ux.nslots > 0)
      winv_coupling_kernel<<<dim3((td.Ux.nslots + WINV_COUPLE_ROWS - 1) / WINV_COUPLE_ROWS, (ldw + 255) / 256), 256,
                             0, s>>>(td.Ux, H->winv.p, ldw);
  }
  winv_upper_kernel<<<nchunk, WINV_THREADS, 0, s>>>(td, H->winv.p, ldw);
  CK(cudaGetLastError());
  H->launches += K > 0 ? 4 : 2;
  const RealSys &S = H->sys[0];
  if (H->a_ptr.n != S.mrow_ptr.size() || H->a_col.n != S.mcol.size()) {
    CK(upload(H->a_ptr, S.mrow_ptr, s));
    CK(upload(H->a_col, S.mcol, s));
  }
  CK(H->wx0.alloc(N));
  CK(H->wr.alloc(N));
  CK(H->wacc.alloc(3));
  CK(cudaMemsetAsync(H->wacc.p, 0, sizeof(unsigned long long) * 3, s));
  H->winv_ldw = ldw;
  H->winv_ready = true;
  H->winv32_p = make_winv_f32(H, H->winv32, H->winv.p, (size_t)N * ldw);
  return 0;
}

// Batched realizations: X_r = A_r^-1 for every realization on the device
// (batch_inverse_kernel), from the assembled entries already on the device.
static int factor_batch_inverse(AndfnHandle *H) {
  const int R = H->R;
  cudaStream_t s = H->stream;
  auto t0 = std::chrono::steady_clock::now();
  const std::vector<int> &roff = H->h.roff;
  if (!H->bcsr_built) {
    // CSR of every realization's pattern over the global rows; entry p of
    // realization r is assembly entry ent0_r + p
    std::vector<int> ptr(H->N + 1, 0), col;
    for (int r = 0; r < R; r++) {
      const RealSys &S = H->sys[r];
      for (int i = 0; i < S.n; i++) ptr[roff[r] + i + 1] = S.ent0 + S.mrow_ptr[i + 1];
      if (S.n > 0) ptr[roff[r]] = S.ent0 + S.mrow_ptr[0];
    }
    col.assign(H->ent_row.size(), 0);
    for (int r = 0; r < R; r++) {
      const RealSys &S = H->sys[r];
      for (size_t p = 0; p < S.mcol.size(); p++) col[S.ent0 + p] = S.mcol[p];
    }
    std::vector<int> order(R);
    for (int r = 0; r < R; r++) order[r] = r;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return H->sys[a].n > H->sys[b].n; });
    std::vector<long long> off(R);
    long long tot = 0;
    int maxn = 1;
    for (int r = 0; r < R; r++) {
      off[r] = tot;
      tot += (long long)H->sys[r].n * H->sys[r].n;
      maxn = std::max(maxn, H->sys[r].n);
    }
    CK(upload(H->bcsr_ptr, ptr, s));
    CK(upload(H->bcsr_col, col, s));
    CK(upload(H->binv_order, order, s));
    H->binv_order_h = order;
    CK(upload(H->binv_roff, roff, s));
    CK(upload(H->binv_off, off, s));
    CK(H->binv.alloc((size_t)std::max(1LL, tot)));
    CK(H->bsing.alloc(R));
    H->binv_maxn = maxn;
    // realizations whose matrix fits one CTA's shared memory (n <= smem_n)
    // are inverted by one CTA each, larger ones by a cluster
    const size_t budget = 200 * 1024;
    const size_t vec = 16 * (size_t)maxn + 4 * (size_t)maxn + 16;
    int smem_n = 0;
    if (budget > vec) smem_n = (int)std::floor(std::sqrt((double)(budget - vec) / 8.0));
    smem_n = std::min(smem_n, maxn);
    std::vector<int> small, big;
    int bign = 0;
    for (int r : order) {
      if (H->sys[r].n <= smem_n) {
        small.push_back(r);
      } else {
        big.push_back(r);
        bign = std::max(bign, H->sys[r].n);
      }
    }
    CK(upload(H->binv_small, small.empty() ? std::vector<int>{0} : small, s));
    CK(upload(H->binv_big, big.empty() ? std::vector<int>{0} : big, s));
    H->binv_nsmall = (int)small.size();
    H->binv_nbig = (int)big.size();
    H->binv_smem_n = smem_n;
    H->binv_bign = bign;
    // the per-iteration solve of a realization with at least
    // ANDFN_B200_BINV_CLUSTER_SOLVE_N (default 128) unknowns is spread over
    // a cluster: its two products with X then take 1/8 of the time and the
    // largest realizations, which set the pace of a batch's last iterations,
    // are not bound by one SM's share of L2 bandwidth
    int csolve_n = 128;
    if (const char *e = getenv("ANDFN_B200_BINV_CLUSTER_SOLVE_N")) csolve_n = std::max(1, atoi(e));
    int nc = 0;
    while (nc < R && H->sys[order[nc]].n >= csolve_n && H->sys[order[nc]].n >= BINV_CLUSTER) nc++;
    H->binv_ncsolve = nc;
    H->bcsr_built = true;
  }
  const int maxn = H->binv_maxn;
  const int smem_n = H->binv_smem_n;
  const size_t smem = 8 * (size_t)smem_n * smem_n + 16 * (size_t)maxn + 4 * (size_t)maxn + 16;
  CK(cudaFuncSetAttribute(batch_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CK(cudaFuncSetAttribute(batch_winv_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(24 * (size_t)maxn)));
  if (H->binv_ncsolve > 0)
    CK(cudaFuncSetAttribute(batch_winv_solve_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)binv_solve_cluster_smem(maxn)));
  if (H->binv_nbig > 0) {
    const size_t csmem = binv_cluster_smem(H->binv_bign);
    CK(cudaFuncSetAttribute(batch_inverse_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csmem));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = BINV_CLUSTER;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(BINV_CLUSTER * H->binv_nbig);
    cfg.blockDim = dim3(BINV_THREADS);
    cfg.dynamicSmemBytes = csmem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, batch_inverse_cluster_kernel, (const int *)H->binv_big.p, (const int *)H->binv_roff.p,
                          (const long long *)H->binv_off.p, H->binv.p, (const int *)H->bcsr_ptr.p,
                          (const int *)H->bcsr_col.p, (const double *)H->d_mvals.p, H->bsing.p));
    H->launches += 1;
  }
  if (H->binv_nsmall > 0) {
    batch_inverse_kernel<<<H->binv_nsmall, BINV_THREADS, smem, s>>>(H->binv_small.p, H->binv_roff.p, H->binv_off.p,
                                                                    H->binv.p, H->bcsr_ptr.p, H->bcsr_col.p,
                                                                    H->d_mvals.p, H->bsing.p, smem_n);
    H->launches += 1;
  }
  CK(cudaGetLastError());
  std::vector<int> sing(R, 0);
  CK(cudaMemcpyAsync(sing.data(), H->bsing.p, sizeof(int) * R, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int r = 0; r < R; r++)
    if (sing[r]) {
      set_error("discharge system of realization " + std::to_string(r) +
                " is singular (a fracture without a head boundary?)");
      return ANDFN_SINGULAR;
    }
  for (int r = 0; r < R; r++) {
    H->sys[r].tail_k = 0;
    H->sys[r].nlev_l = H->sys[r].nlev_u = 0;
    H->sys[r].nnz = (int64_t)H->sys[r].n * H->sys[r].n;
  }
  H->nnz_factors = 0;
  for (int r = 0; r < R; r++) H->nnz_factors += H->sys[r].nnz;
  H->winv_ready = false;
  H->binv_ready = true;
  H->adj_factors_ready = false;
  H->lu_keep = LuFactors();
  H->ms_fac[0] = H->ms_fac[2] = H->ms_fac[3] = 0.0;
  H->ms_fac[1] = ms_since(t0);
  return 0;
}

static int factor_all(AndfnHandle *H, const std::vector<double> &mv) {
  const int R = H->R;
  cudaStream_t s = H->stream;
  H->binv_ready = false;
  if (R > 1 && H->winv_enabled) {
    // batches: per-realization explicit inverses on the device when they are
    // small enough (the host's sparse LU is then not needed)
    int maxn = 0;
    long long tot = 0;
    for (int r = 0; r < R; r++) {
      maxn = std::max(maxn, H->sys[r].n);
      tot += (long long)H->sys[r].n * H->sys[r].n;
    }
    size_t fr = 0, totmem = 0;
    cudaMemGetInfo(&fr, &totmem);
    if (maxn <= BINV_MAX_N && binv_cluster_smem(maxn) <= BINV_CLUSTER_SMEM_MAX && 8.0 * (double)tot < 0.5 * (double)fr)
      return factor_batch_inverse(H);
  }
  std::vector<LuFactors> LU(R);
  std::vector<int> rcs(R, 0);
  auto tf0 = std::chrono::steady_clock::now();
  // a single network whose column order is still being computed: its
  // leading pivot steps follow the published order (the same steps in the
  // same order as after it), then the thread is joined
  LuLeading lead_st;
  CscMatrix A0;
  bool followed = false;
  int lead_rc = 0;
  if (H->order_thread.joinable()) {
    if (R == 1 && H->order_follow) {
      A0 = system_csc(H->sys[0], mv.data());
      lu_leading_init(lead_st, A0.n);
      lead_rc = lu_leading_follow(A0, H->order_prog, lead_st);
      followed = true;
    }
    H->order_thread.join();
  }
  // one realization: the Schur complement's columns use the host threads and
  // a large dense block is factorised on the device; several: one
  // realization per thread, dense blocks on the host
  const bool defer = R == 1 && H->sys[0].dense_k >= DLU_MIN_K && H->sys[0].dense_k <= DLU_MAX_K;
  // the Schur complement is formed straight into page-locked memory (from
  // the process's cache of such blocks), so its upload is a DMA
  double *schur_buf = nullptr;
  if (defer) {
    const size_t need = (size_t)H->sys[0].dense_k * H->sys[0].dense_k;
    if (H->pin_schur_n < need) {
      if (H->pin_schur) pinned_put(H->pin_schur, sizeof(double) * H->pin_schur_n);
      H->pin_schur = nullptr;
      H->pin_schur_n = 0;
      size_t cap = 0;
      if (void *p = pinned_get(sizeof(double) * need, &cap)) {
        H->pin_schur = static_cast<double *>(p);
        H->pin_schur_n = cap / sizeof(double);
      }
      else
        cudaGetLastError();
    }
    if (H->pin_schur_n >= need) schur_buf = H->pin_schur;
  }
  H->factor_runs += 1;
  auto factor_one = [&](int r) {
    if (H->sys[r].colorder.empty() && H->sys[r].n > 0) {  // column order not computed at creation
      CscMatrix P = system_csc(H->sys[r], nullptr);
      H->sys[r].colorder = column_min_degree_order(P, &H->sys[r].dense_k, H->dense_frac);
    }
    if (followed && r == 0) {
      rcs[0] = lead_rc ? lead_rc
                       : sparse_lu_factor_rest(A0, H->sys[0].colorder, lead_st, LU[0], H->sys[0].dense_k, defer,
                                               schur_buf);
      return;
    }
    CscMatrix A = system_csc(H->sys[r], mv.data());
    rcs[r] = sparse_lu_factor(A, H->sys[r].colorder, 1.0, LU[r], H->sys[r].dense_k, defer, schur_buf);
  };
  if (R == 1) {
    factor_one(0);
  } else {
#pragma omp parallel for schedule(dynamic, 1)
    for (int r = 0; r < R; r++) factor_one(r);
  }
  H->ms_fac[0] = ms_since(tf0);
  auto tf1 = std::chrono::steady_clock::now();
  H->ms_fac[1] = H->ms_fac[3] = 0.0;
  const bool dev_tail = defer && rcs[0] == 0 && LU[0].schur != nullptr;
  // explicit inverse of the whole system (one network), and of a dense tail
  // of one network (the inverse's tail rows; the cluster path of the
  // triangular solves, applied with one refinement step)
  const bool want_winv = R == 1 && H->winv_enabled && LU[0].n <= WINV_MAX_N;
  const bool want_w = R == 1 && LU[0].dense > 0 && (LU[0].dense >= CLUSTER_MIN_K || want_winv);
  if (dev_tail) {
    const int rc = gpu_dense_lu(H, LU[0], want_w);
    if (rc != 0 && rc != 3) return rc;
    rcs[0] = rc;
    H->ms_fac[1] = ms_since(tf1);
  }
  auto tf2 = std::chrono::steady_clock::now();
  for (int r = 0; r < R; r++)
    if (rcs[r]) {
      set_error("discharge system of realization " + std::to_string(r) +
                " is singular (a fracture without a head boundary?)");
      return ANDFN_SINGULAR;
    }
  struct PartOff {
    int lev, rows, ent;
  };
  LevelParts parts[4];  // lf, lx, ux, ub
  std::vector<std::array<PartOff, 4>> off(R);
  std::vector<std::array<int, 4>> nlev(R), nslots(R), grp(R);
  std::vector<double> tl, tui;
  std::vector<size_t> toff(R), tuoff(R);
  std::vector<int> pinv, qcol;
  H->nnz_factors = 0;
  H->max_k = 0;
  H->cluster_fwd = H->cluster_adj = -1;
  H->max_n = 0;
  H->max_nlev = 1;
  for (int r = 0; r < R; r++) {
    const LuFactors &F = LU[r];
    const int n = F.n, K = F.dense, m0 = n - K;
    H->max_n = std::max(H->max_n, n);
    H->max_k = std::max(H->max_k, K);
    H->nnz_factors += F.nnz() + 2LL * K * K;
    pinv.insert(pinv.end(), F.pinv.begin(), F.pinv.end());
    qcol.insert(qcol.end(), F.q.begin(), F.q.end());
    const struct {
      bool lower, single;
      int rlo, rhi, clo, chi;
      bool scaled;
    } spec[4] = {{true, false, 0, m0, 0, m0, false},
                 {true, true, m0, n, 0, m0, false},
                 {false, true, 0, m0, m0, n, false},
                 {false, false, 0, m0, 0, m0, true}};
    // the four parts' level tables, then appended in part order (building
    // them on four host threads measured slower on the box)
    std::vector<int> levk[4], rowsk[4], eptrk[4], ecolk[4];
    std::vector<double> evk[4], esck[4];
    for (int k = 0; k < 4; k++) {
      const auto &sp = spec[k];
      // without a dense tail the coupling parts are empty
      const int rlo = (K == 0 && (k == 1 || k == 2)) ? 0 : sp.rlo;
      const int rhi = (K == 0 && (k == 1 || k == 2)) ? 0 : sp.rhi;
      if (sp.lower)
        build_levels(n, F.l_ptr, F.l_col, F.l_val, nullptr, true, rlo, rhi, sp.clo, sp.chi, sp.single, levk[k],
                     rowsk[k], eptrk[k], ecolk[k], evk[k], esck[k]);
      else
        build_levels(n, F.u_ptr, F.u_col, F.u_val, sp.scaled ? &F.u_inv_diag : nullptr, false, rlo, rhi, sp.clo,
                     sp.chi, sp.single, levk[k], rowsk[k], eptrk[k], ecolk[k], evk[k], esck[k]);
    }
    for (int k = 0; k < 4; k++) {
      const auto &sp = spec[k];
      const std::vector<int> &lev = levk[k], &rows = rowsk[k], &eptr = eptrk[k], &ecol = ecolk[k];
      const std::vector<double> &ev = evk[k], &esc = esck[k];
      LevelParts &P = parts[k];
      off[r][k] = {(int)P.lev.size(), (int)P.rows.size(), (int)P.col.size()};
      nlev[r][k] = (int)lev.size() - 1;
      nslots[r][k] = (int)rows.size();
      grp[r][k] = group_for(eptr, sp.single);
      H->max_nlev = std::max(H->max_nlev, nlev[r][k]);
      P.lev.insert(P.lev.end(), lev.begin(), lev.end());
      P.rows.insert(P.rows.end(), rows.begin(), rows.end());
      P.eptr.insert(P.eptr.end(), eptr.begin(), eptr.end());
      P.col.insert(P.col.end(), ecol.begin(), ecol.end());
      P.val.insert(P.val.end(), ev.begin(), ev.end());
      P.scale.insert(P.scale.end(), esc.begin(), esc.end());
      // keep eptr and rows indexable by slot: eptr has nslots + 1 entries, so
      // the next part starts one entry later; rows pad to the same length
      P.rows.push_back(0);
      P.scale.push_back(1.0);
    }
    toff[r] = tl.size();
    tuoff[r] = tui.size();
    if (!dev_tail) {  // L and U (zero diagonals, disjoint parts) in one matrix
      tl.insert(tl.end(), F.l22.begin(), F.l22.end());
      for (size_t k = 0; k < F.u22.size(); k++) tl[toff[r] + k] += F.u22[k];
    }
    tui.insert(tui.end(), F.u_inv_diag.begin() + m0, F.u_inv_diag.end());
    H->sys[r].tail_k = K;
    H->sys[r].nlev_l = nlev[r][0];
    H->sys[r].nlev_u = nlev[r][3];
    H->sys[r].nnz = F.nnz() + 2LL * K * K;
  }
  DBuf<int> *dlev[4] = {&H->lf_lev, &H->lx_lev, &H->ux_lev, &H->ub_lev};
  DBuf<int> *drows[4] = {&H->lf_rows, &H->lx_rows, &H->ux_rows, &H->ub_rows};
  DBuf<int> *deptr[4] = {&H->lf_eptr, &H->lx_eptr, &H->ux_eptr, &H->ub_eptr};
  DBuf<int> *dcol[4] = {&H->lf_col, &H->lx_col, &H->ux_col, &H->ub_col};
  DBuf<double> *dval[4] = {&H->lf_val, &H->lx_val, &H->ux_val, &H->ub_val};
  for (int k = 0; k < 4; k++) {
    if (parts[k].col.empty()) {
      parts[k].col.push_back(0);
      parts[k].val.push_back(0.0);
    }
    CK(upload(*dlev[k], parts[k].lev, s));
    CK(upload(*drows[k], parts[k].rows, s));
    CK(upload(*deptr[k], parts[k].eptr, s));
    CK(upload(*dcol[k], parts[k].col, s));
    CK(upload(*dval[k], parts[k].val, s));
  }
  CK(upload(H->ub_scale, parts[3].scale, s));
  if (tui.empty()) tui.push_back(0.0);
  if (!dev_tail) {
    if (tl.empty()) tl.push_back(0.0);
    CK(upload(H->tail_l, tl, s));
  }
  if (!dev_tail) CK(upload(H->tail_uinv, tui, s));  // on the device already (gpu_dense_lu)
  if (want_w && !dev_tail) {
    const int rc = launch_tail_inverse(H, LU[0].dense);
    if (rc) return rc;
  }
  CK(upload(H->pinv, pinv, s));
  CK(upload(H->qcol, qcol, s));
  std::vector<TriDesc> td(R);
  for (int r = 0; r < R; r++) {
    const int n = LU[r].n, K = LU[r].dense;
    LevelSolve *ls[4] = {&td[r].Lf, &td[r].Lx, &td[r].Ux, &td[r].Ub};
    for (int k = 0; k < 4; k++) {
      LevelSolve &L = *ls[k];
      const PartOff &o = off[r][k];
      L.lev_ptr = dlev[k]->p + o.lev;
      L.rows = drows[k]->p + o.rows;
      L.eptr = deptr[k]->p + o.rows;
      L.col = dcol[k]->p + o.ent;
      L.val = dval[k]->p + o.ent;
      L.scale = (k == 3) ? H->ub_scale.p + o.rows : nullptr;
      L.nlev = nlev[r][k];
      L.nslots = nslots[r][k];
      L.group = grp[r][k];
    }
    td[r].T.K = K;
    td[r].T.L = H->tail_l.p + toff[r];
    td[r].T.U = H->tail_l.p + toff[r];
    td[r].T.uinv = H->tail_uinv.p + tuoff[r];
    td[r].T.lscale = nullptr;
    td[r].T.W = want_w ? H->tail_w.p : nullptr;
    td[r].pinv = H->pinv.p + H->h.roff[r];
    td[r].qcol = H->qcol.p + H->h.roff[r];
    td[r].row0 = H->h.roff[r];
    td[r].n = n;
  }
  CK(upload(H->tri, td, s));
  H->winv_ready = false;
  CK(cudaStreamSynchronize(s));
  H->ms_fac[2] = ms_since(tf2);
  if (want_winv) {
    auto tf3 = std::chrono::steady_clock::now();
    const int rc = build_inverse(H, td[0]);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s));
    H->ms_fac[3] = ms_since(tf3);
  }
  // the adjoint solves with the transposed factors of a single network
  H->adj_factors_ready = false;
  if (R == 1)
    H->lu_keep = std::move(LU[0]);
  else
    H->lu_keep = LuFactors();
  return 0;
}

// Factor-entry ring of the staged level solve: entries per slot (even), from
// the shared memory left under 200 KB; 0 (unstaged path) when y or the slot
// metadata are not in shared memory.
static size_t ring_bytes(int cap) {
  return (size_t)RING_SLOTS * (sizeof(double) * cap + sizeof(double) * (cap / 2) + sizeof(int) * cap);
}
static int ring_capacity(size_t used, int use_smem, int meta_cap) {
  if (!use_smem || !meta_cap) return 0;
  const size_t budget = 190 * 1024;
  const size_t base = (used + 15) & ~(size_t)15;
  if (base >= budget) return 0;
  // per entry: value and column in every slot, a row scale per two entries
  const size_t per_entry = (size_t)RING_SLOTS * (sizeof(double) + sizeof(int) + sizeof(double) / 2);
  int cap = (int)((budget - base) / per_entry) & ~1;
  cap = std::min(cap, 2048);
  if (cap < 64 || base + ring_bytes(cap) > budget) return 0;
  return cap;
}

// One network with a dense tail of at least CLUSTER_MIN_K rows: the trisolve
// runs as a cluster of CLUSTER_CTAS CTAs (the dense tail spread over their
// SMs) when the device can co-schedule such a cluster with this much shared
// memory per CTA; otherwise one CTA.
static constexpr int CLUSTER_CTAS = 8;

template <bool ADJ>
static int choose_cluster(AndfnHandle *H, size_t smem, int use_smem) {
  if (H->R != 1 || H->max_k < CLUSTER_MIN_K || !use_smem) return 1;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CLUSTER_CTAS;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(CLUSTER_CTAS);
  cfg.blockDim = dim3(H->solve_threads);
  cfg.dynamicSmemBytes = smem;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, trisolve_kernel<ADJ>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  return n >= 1 ? CLUSTER_CTAS : 1;
}

template <bool ADJ>
static void launch_trisolve_kernel(AndfnHandle *H, const Net &net, cudaStream_t s, int csize, size_t smem,
                                   int use_smem, int cap_levptr, int meta_cap, int ring_cap) {
  if (csize > 1) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(csize);
    cfg.blockDim = dim3(H->solve_threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, trisolve_kernel<ADJ>, net, use_smem, cap_levptr, meta_cap, ring_cap);
  } else {
    trisolve_kernel<ADJ><<<H->R, H->solve_threads, smem, s>>>(net, use_smem, cap_levptr, meta_cap, ring_cap);
  }
}

static int build_head_sums(AndfnHandle *H);
template <int T, int RPB>
__global__ void head_vector_kernel(Net net, const int *__restrict__ gptr, const int *__restrict__ sidx,
                                   const cd *__restrict__ S, const int *__restrict__ alist,
                                   const int *__restrict__ acount);

// Kernels one discharge solve launches.
static int tri_launches(const AndfnHandle *H) { return H->winv_ready ? 3 : 1; }  // batched inverses: 1

// A discharge solve through the explicit inverse X (forward) or its
// transpose (ADJ): x0 = Q X P b, r = b - M x0, x = x0 + Q X P r, with M = A
// or A^T in CSR form (map: value index of each entry, null = entry order).
template <bool ADJ>
static void launch_winv_solve(AndfnHandle *H, const Net &net, cudaStream_t s, const double *X, const int *rp,
                              const int *cols, const int *map, const float *X32 = nullptr) {
  const int N = H->N, ldw = H->winv_ldw;
  const size_t vsm = sizeof(double) * (size_t)ldw;
  // two CTAs of 512 threads per SM, at most WINV_RPC rows per CTA
  const int grid = std::max(2 * H->num_sms, (N + WINV_RPC - 1) / WINV_RPC);
  winv_gemv_kernel<0, ADJ><<<grid, WINV_THREADS, vsm, s>>>(net, X, ldw, net.bvec, H->wx0.p, H->wacc.p);
  winv_resid_kernel<ADJ><<<(N * 32 + 255) / 256, 256, 0, s>>>(net, rp, cols, map, H->d_mvals.p + H->sys[0].ent0,
                                                             H->wx0.p, H->wr.p, N);
  if (X32)
    winv_gemv_kernel<1, ADJ, true><<<grid, WINV_THREADS, vsm, s>>>(net, X, ldw, H->wr.p, H->wx0.p, H->wacc.p, X32);
  else
    winv_gemv_kernel<1, ADJ><<<grid, WINV_THREADS, vsm, s>>>(net, X, ldw, H->wr.p, H->wx0.p, H->wacc.p);
}

// A float copy of an N x ldw inverse for the refinement pass.
__global__ void winv_to_f32_kernel(const double *__restrict__ X, float *__restrict__ Y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    Y[i] = (float)X[i];
}

// Whether the refinement passes read float copies of the inverses
// (ANDFN_B200_WINV_F32=0 when the inverse is formed: the double inverse in
// both passes).
static bool winv_f32_enabled() {
  const char *e = getenv("ANDFN_B200_WINV_F32");
  return !(e && atoi(e) == 0);
}

// The float copy of X (N x ldw) when the device has room for it, else null.
static float *make_winv_f32(AndfnHandle *H, DBuf<float> &Y, const double *X, size_t n) {
  if (!winv_f32_enabled()) return nullptr;
  if (Y.cap < n) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    if (sizeof(float) * n + ((size_t)1 << 30) > fr + sizeof(float) * Y.cap) return nullptr;
  }
  if (Y.alloc(n) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  winv_to_f32_kernel<<<4 * H->num_sms, 256, 0, H->stream>>>(X, Y.p, n);
  H->launches += 1;
  return Y.p;
}

static void launch_trisolve(AndfnHandle *H, cudaStream_t s) {
  Net net = H->net();
  if (H->binv_ready) {
    // binv_order lists the realizations by decreasing size: the first
    // binv_ncsolve of them are solved by a cluster each, the rest by one CTA
    // with active lists (every batch iteration loop) the CTAs take the
    // running realizations from the lists
    const int nc = H->binv_ncsolve;
    const bool act = H->act_on;
    if (nc > 0) {
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = BINV_CLUSTER;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(BINV_CLUSTER * nc);
      cfg.blockDim = dim3(BINV_SOLVE_THREADS);
      cfg.dynamicSmemBytes = binv_solve_cluster_smem(H->sys[H->binv_order_h[0]].n);
      cfg.stream = s;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      const cudaError_t ce = cudaLaunchKernelEx(
          &cfg, batch_winv_solve_cluster_kernel, net, (const int *)H->binv_order.p, (const int *)H->binv_roff.p,
          (const long long *)H->binv_off.p, (const double *)H->binv.p, (const int *)H->bcsr_ptr.p,
          (const int *)H->bcsr_col.p, (const double *)H->d_mvals.p, act ? (const int *)H->act.list[3] : nullptr,
          act ? (const int *)&H->act.st->count[3] : nullptr);
      if (ce != cudaSuccess) set_error(std::string("batched cluster solve launch: ") + cudaGetErrorString(ce));
      H->launches += 1;
    }
    if (H->R > nc) {
      batch_winv_solve_kernel<<<H->R - nc, BINV_SOLVE_THREADS, 24 * (size_t)H->binv_maxn, s>>>(
          net, H->binv_order.p + nc, H->binv_roff.p, H->binv_off.p, H->binv.p, H->bcsr_ptr.p, H->bcsr_col.p,
          H->d_mvals.p, act ? H->act.list[4] : nullptr, act ? &H->act.st->count[4] : nullptr);
      H->launches += 1;
    }
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) set_error(std::string("batched explicit-inverse solve launch: ") + cudaGetErrorString(le));
    return;
  }
  if (H->winv_ready) {
    launch_winv_solve<false>(H, net, s, H->winv.p, H->a_ptr.p, H->a_col.p, nullptr, H->winv32_p);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) set_error(std::string("explicit-inverse solve launch: ") + cudaGetErrorString(le));
    return;
  }
  const size_t ybytes = sizeof(double) * (size_t)H->max_n;
  const int use_smem = ybytes <= 150 * 1024 ? H->max_n : 0;
  const int cap_levptr = std::min(H->max_nlev + 1, 10240);
  size_t solve_smem = (use_smem ? ybytes : 0) + sizeof(int) * (size_t)cap_levptr;
  const size_t meta_bytes = sizeof(int) * 2 * ((size_t)H->max_n + 1);
  const int meta_cap = (solve_smem + meta_bytes <= 200 * 1024) ? H->max_n + 1 : 0;
  if (meta_cap) solve_smem += meta_bytes;
  const int ring_cap = ring_capacity(solve_smem, use_smem, meta_cap);
  if (ring_cap) solve_smem = ((solve_smem + 15) & ~(size_t)15) + ring_bytes(ring_cap);
  if (H->cluster_fwd < 0) H->cluster_fwd = choose_cluster<false>(H, solve_smem, use_smem);
  launch_trisolve_kernel<false>(H, net, s, H->cluster_fwd, solve_smem, use_smem, cap_levptr, meta_cap, ring_cap);
  const cudaError_t le = cudaGetLastError();
  if (le != cudaSuccess)
    set_error(std::string("trisolve_kernel launch (shared memory ") + std::to_string(solve_smem) +
              " B, ring " + std::to_string(ring_cap) + "): " + cudaGetErrorString(le));
}

static inline void mark(AndfnHandle *H, cudaStream_t s, int b, int c, int w) {
  if (H->profiling && b >= 0) cudaEventRecordWithFlags(H->ev[b][c][w], s, cudaEventRecordExternal);
}

static int enqueue_iteration(AndfnHandle *H, cudaStream_t s, int blend_mode, int b = -1);

// Condition of the device-side iteration loop: another iteration while some
// realization is still running, at most cap iterations (a bound independent
// of the stopping logic).  One thread.
__global__ void loop_cond_kernel(cudaGraphConditionalHandle h, const int *ndone, int R, int *count, int cap) {
  const int c = ++(*count);
  cudaGraphSetConditional(h, (*ndone < R && c < cap) ? 1u : 0u);
}

// The iteration loop as one graph launch: a while node whose body is one
// outer iteration (enqueue_iteration) followed by loop_cond_kernel.  Returns
// 0 and sets *ran when the loop ran; *ran = false (nothing launched) when the
// runtime has no conditional graph nodes, so the caller falls back to
// launching batches of iterations from the host.
static int run_device_loop(AndfnHandle *H, const AndfnConstants *C, bool *ran, int *iterations_run) {
  *ran = false;
  cudaStream_t s = H->stream;
  if (H->loop_exec) {
    cudaGraphExecDestroy(H->loop_exec);
    H->loop_exec = nullptr;
  }
  if (!H->loop_count.p) CK(H->loop_count.alloc(1));
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle hc;
  if (cudaGraphConditionalHandleCreate(&hc, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return 0;
  }
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = hc;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  if (cudaGraphAddNode(&cnode, g, nullptr, 0, &cp) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return 0;
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  const int64_t launches0 = H->launches;
  CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  enqueue_iteration(H, s, 0, -1);
  const int cap = (int)std::min<int64_t>(C->max_iterations + 2, (int64_t)1 << 30);
  loop_cond_kernel<<<1, 1, 0, s>>>(hc, H->ndone.p, H->R, H->loop_count.p, cap);
  {
    const cudaError_t ec = cudaStreamEndCapture(s, &body);
    if (ec != cudaSuccess) {
      cudaGraphDestroy(g);
      set_error(std::string("capture of the iteration loop: ") + cudaGetErrorString(ec) + "; " + g_last_error);
      return ANDFN_CUDA_ERROR;
    }
  }
  const int64_t per_it = H->launches - launches0 + 1;  // kernels of one iteration, the condition included
  H->launches = launches0;                              // capture launches nothing
  const cudaError_t ei = cudaGraphInstantiate(&H->loop_exec, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    set_error(std::string("instantiation of the iteration loop: ") + cudaGetErrorString(ei));
    return ANDFN_CUDA_ERROR;
  }
  CK(cudaMemsetAsync(H->loop_count.p, 0, sizeof(int), s));
  CK(cudaGraphLaunch(H->loop_exec, s));
  int count = 0;
  CK(cudaMemcpyAsync(&count, H->loop_count.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  H->launches += per_it * count;
  *iterations_run = count;
  *ran = true;
  return 0;
}

// Launch forms of the table sweep: one CTA per item, or persistent CTAs
// (4 or 6 per SM) taking items from a device work queue.
enum SweepVariant { SWEEP_PER_ITEM = 0, SWEEP_QUEUE4 = 1, SWEEP_QUEUE6 = 2, SWEEP_VARIANTS = 3 };

static void launch_sweep_variant(AndfnHandle *H, const Net &net, cudaStream_t s, int v) {
  const int *alist = H->act_on ? H->act.list[1] : nullptr;
  const int *acount = H->act_on ? &H->act.st->count[1] : nullptr;
  if (v == SWEEP_PER_ITEM) {
    sweep_table_kernel<<<H->n_sweep_items, EVAL_THREADS, H->tab_smem, s>>>(
        net, H->sweep_items.p, H->sweep_pts.p, H->d_groups.p, H->tab_fpt0.p, H->tab_fnp.p, H->tab_off.p, H->tab_w.p,
        H->tab_l.p, H->sweep_vals.p, H->tab_chunk, alist, acount);
  } else {
    const int per_sm = (v == SWEEP_QUEUE4) ? 4 : 6;
    const int grid = std::min(H->n_sweep_items, per_sm * H->num_sms);
    sweep_table_queue_kernel<<<grid, EVAL_THREADS, H->tab_smem, s>>>(
        net, H->sweep_items.p, H->n_sweep_items, H->sweep_pts.p, H->d_groups.p, H->tab_fpt0.p, H->tab_fnp.p,
        H->tab_off.p, H->tab_w.p, H->tab_l.p, H->sweep_vals.p, H->tab_chunk, H->sweep_q.p, alist, acount);
  }
}

// The sweep evaluation into sweep_vals: from the pair tables when this run
// has them (fixed ncoef and nint), else the full evaluation.
static void launch_sweep(AndfnHandle *H, const Net &net, cudaStream_t s) {
  if (H->n_sweep_items <= 0) return;
  if (H->use_tab && H->tab_valid)
    launch_sweep_variant(H, net, s, H->sweep_variant < 0 ? SWEEP_PER_ITEM : H->sweep_variant);
  else
    eval_kernel<false><<<H->n_sweep_items, EVAL_THREADS, H->eval_smem, s>>>(net, H->sweep_items.p, H->sweep_pts.p,
                                                                             H->d_groups.p, H->sweep_vals.p, H->chunk);
}

// Autotuner of the table sweep's launch form: each form runs on this run's
// own tables (one warm-up launch, then three timed with CUDA events; the
// outputs are overwritten by the first iteration), the fastest is kept for
// the handle and cached for the process by the shape of the work (MC,
// items and largest fracture, bucketed).  ANDFN_B200_SWEEP_VARIANT=0/1/2
// forces a form.  A handle that may not tune (the one-call solve) takes a
// cached choice or the per-item form.
static std::mutex g_tune_mu;
static std::map<std::array<int, 4>, int> g_tune_cache;

static int sweep_autotune(AndfnHandle *H) {
  if (H->sweep_variant >= 0) return 0;
  if (const char *v = getenv("ANDFN_B200_SWEEP_VARIANT")) {
    const int x = atoi(v);
    if (x >= 0 && x < SWEEP_VARIANTS) {
      H->sweep_variant = x;
      return 0;
    }
  }
  int maxnf = 1;
  for (int f = 0; f < (int)H->nf; f++) maxnf = std::max(maxnf, H->h.fptr[f + 1] - H->h.fptr[f]);
  const std::array<int, 4> key = {H->device, H->MC, H->n_sweep_items / 256, maxnf / 8};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      H->sweep_variant = it->second;
      return 0;
    }
  }
  if (!H->tune_sweep || H->n_sweep_items <= 0) {
    H->sweep_variant = SWEEP_PER_ITEM;
    return 0;
  }
  cudaStream_t s = H->stream;
  const Net net = H->net();
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  float best = 1e30f;
  int bestv = SWEEP_PER_ITEM;
  for (int v = 0; v < SWEEP_VARIANTS; v++) {
    launch_sweep_variant(H, net, s, v);
    CK(cudaEventRecord(a, s));
    for (int r = 0; r < 3; r++) launch_sweep_variant(H, net, s, v);
    CK(cudaEventRecord(b, s));
    CK(cudaEventSynchronize(b));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, a, b));
    if (ms < best) {
      best = ms;
      bestv = v;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  CK(cudaGetLastError());
  H->launches += 4 * SWEEP_VARIANTS;
  H->sweep_variant = bestv;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = bestv;
  return 0;
}

// The pair tables of the current points and geometry (once per run).
static int build_pair_table(AndfnHandle *H) {
  H->tab_valid = false;
  if (H->n_sweep_items > 0 && H->tab_pairs > 0) {
    pair_table_kernel<<<H->n_sweep_items, EVAL_THREADS, 0, H->stream>>>(
        H->net(), H->sweep_items.p, H->sweep_pts.p, H->d_groups.p, H->tab_fpt0.p, H->tab_fnp.p, H->tab_off.p,
        H->tab_w.p, H->tab_l.p);
    CK(cudaGetLastError());
    H->launches += 1;
  }
  H->tab_valid = true;
  return 0;
}

static int enqueue_iteration(AndfnHandle *H, cudaStream_t s, int blend_mode, int b) {
  Net net = H->net();
  mark(H, s, b, K_RHS, 0);
  const int *arows = H->act_on ? H->act.list[0] : nullptr;
  const int *arow_n = H->act_on ? &H->act.st->count[0] : nullptr;
  if (H->use_head_sums) {
    if (H->hs.long_rows)
      head_vector_kernel<HV_THREADS, 1><<<H->N, HV_THREADS, 0, s>>>(net, H->hs.gptr.p, H->hs.sidx.p, H->hs.S.p,
                                                                     arows, arow_n);
    else
      head_vector_kernel<32, 4><<<(H->N + 3) / 4, 128, 0, s>>>(net, H->hs.gptr.p, H->hs.sidx.p, H->hs.S.p, arows,
                                                               arow_n);
  } else {
    if (H->n_rhs_items > 0)
      eval_kernel<true><<<H->n_rhs_items, EVAL_THREADS, H->eval_smem, s>>>(net, H->rhs_items.p, H->rhs_pts.p,
                                                                            H->d_groups.p, H->rhs_vals.p, H->chunk);
    rhs_reduce_kernel<<<(H->N * 32 + 255) / 256, 256, 0, s>>>(net, H->rhs_vals.p, H->rhs_group.p, H->d_groups.p);
    H->launches += 1;
  }
  mark(H, s, b, K_RHS, 1);
  mark(H, s, b, K_TRISOLVE, 0);
  launch_trisolve(H, s);
  mark(H, s, b, K_TRISOLVE, 1);
  mark(H, s, b, K_SWEEP, 0);
  launch_sweep(H, net, s);
  mark(H, s, b, K_SWEEP, 1);
  const int ub = (H->n_upd + UPDATE_WARPS - 1) / UPDATE_WARPS;
  const size_t usmem = sizeof(double) * 2 * H->nvmax * UPDATE_WARPS;
  mark(H, s, b, K_UPDATE, 0);
  if (ub > 0)
    update_kernel<<<ub, UPDATE_WARPS * 32, usmem, s>>>(
        net, H->act_on ? H->act.list[2] : H->upd_list.p, H->n_upd, H->group_of.p, H->d_groups.p, H->sweep_vals.p,
        H->nvmax, blend_mode, H->act_on ? &H->act.st->count[2] : nullptr);
  mark(H, s, b, K_UPDATE, 1);
  mark(H, s, b, K_REDUCE, 0);
  if (H->R == 1 && H->red_parts.p)
    reduce_split_kernel<<<(int)((H->ne + REDUCE_SPLIT_ELEMS - 1) / REDUCE_SPLIT_ELEMS), REDUCE_SPLIT_THREADS, 0, s>>>(
        net, H->red_parts.p, H->red_ticket.p);
  else if (H->act_on)
    reduce_kernel<<<H->R, 1024, 0, s>>>(net, H->act.list[5], &H->act.st->count[5]);
  else
    reduce_kernel<<<H->R, 1024, 0, s>>>(net);
  if (H->act_on) {  // the active lists of the next iteration (launches return at entry unless one finished)
    act_count_kernel<<<H->act.chunk0[ACT_LISTS], ACT_CHUNK, 0, s>>>(net, H->act);
    act_scatter_kernel<<<H->act.chunk0[ACT_LISTS], ACT_CHUNK, 0, s>>>(net, H->act);
    H->launches += 2;
  }
  mark(H, s, b, K_REDUCE, 1);
  H->launches += 4 + tri_launches(H);
  return 0;
}

// A batch's active work lists for the iterations of this run: the full
// lists, rebuilt after each iteration in which a realization finished.  The
// element list relies on the update list being every element in order.
static int act_setup(AndfnHandle *H, int ndone0) {
  cudaStream_t s = H->stream;
  const int nbig = H->binv_ready ? H->binv_ncsolve : 0;
  const int nsmall = H->binv_ready ? H->R - nbig : 0;
  const int n[ACT_LISTS] = {(int)H->N, H->n_sweep_items, H->n_upd, nbig, nsmall, H->R};
  ActLists &A = H->act;
  A.order = H->binv_ready ? H->binv_order.p : nullptr;
  A.nbig = nbig;
  int c0 = 0;
  for (int l = 0; l < ACT_LISTS; l++) {
    A.n[l] = n[l];
    A.chunk0[l] = c0;
    c0 += std::max(1, (n[l] + ACT_CHUNK - 1) / ACT_CHUNK);
    if (H->act_l[l].cap < (size_t)std::max(1, n[l])) CK(H->act_l[l].alloc(std::max(1, n[l])));
    A.list[l] = H->act_l[l].p;
  }
  A.chunk0[ACT_LISTS] = c0;
  if (H->act_ccnt.cap < (size_t)c0) CK(H->act_ccnt.alloc(c0));
  if (H->act_st.cap < 1) CK(H->act_st.alloc(1));
  A.ccnt = H->act_ccnt.p;
  A.items = H->sweep_items.p;
  A.st = H->act_st.p;
  const int mx = std::max({n[0], n[1], n[2], n[5], 1});
  act_init_kernel<<<std::min(4 * H->num_sms, (mx + 255) / 256), 256, 0, s>>>(A, ndone0);
  CK(cudaGetLastError());
  H->launches += 1;
  H->act_on = true;
  return 0;
}

// One outer iteration at a time with the coefficient growth of
// element_solver2 between the two blends (hpc_solve.py:394-591).
static int run_adaptive(AndfnHandle *H, const AndfnConstants *C) {
  cudaStream_t s = H->stream;
  const int ne = (int)H->ne;
  if (H->grow_list.cap < (size_t)ne) CK(H->grow_list.alloc(ne));
  if (H->grow_count.cap < 1) CK(H->grow_count.alloc(1));
  int guard = 0;
  while (true) {
    Net net = H->net();
    // head vector, discharge solve, sweep, fit + first blend (no fused second blend)
    if (H->n_rhs_items > 0)
      eval_kernel<true><<<H->n_rhs_items, EVAL_THREADS, H->eval_smem, s>>>(net, H->rhs_items.p, H->rhs_pts.p,
                                                                            H->d_groups.p, H->rhs_vals.p, H->chunk);
    rhs_reduce_kernel<<<(H->N * 32 + 255) / 256, 256, 0, s>>>(net, H->rhs_vals.p, H->rhs_group.p, H->d_groups.p);
    launch_trisolve(H, s);
    if (H->n_sweep_items > 0)
      eval_kernel<false><<<H->n_sweep_items, EVAL_THREADS, H->eval_smem, s>>>(
          net, H->sweep_items.p, H->sweep_pts.p, H->d_groups.p, H->sweep_vals.p, H->chunk);
    const int ub = (H->n_upd + UPDATE_WARPS - 1) / UPDATE_WARPS;
    const size_t usmem = sizeof(double) * 2 * H->nvmax * UPDATE_WARPS;
    if (ub > 0)
      update_kernel<<<ub, UPDATE_WARPS * 32, usmem, s>>>(net, H->upd_list.p, H->n_upd, H->group_of.p,
                                                          H->d_groups.p, H->sweep_vals.p, H->nvmax, 0);
    CK(cudaMemsetAsync(H->grow_count.p, 0, sizeof(int), s));
    growth_kernel<<<(H->n_upd * 32 + 127) / 128, 128, 0, s>>>(net, H->upd_list.p, H->n_upd, C->coef_ratio,
                                                               (int)C->max_ncoef, (int)C->coef_increase,
                                                               H->grow_list.p, H->grow_count.p);
    int ngrow = 0;
    CK(cudaMemcpyAsync(&ngrow, H->grow_count.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    H->launches += 6 + tri_launches(H);
    if (ngrow > 0) {
      std::vector<int> grown(ngrow);
      CK(cudaMemcpy(grown.data(), H->grow_list.p, sizeof(int) * ngrow, cudaMemcpyDeviceToHost));
      std::sort(grown.begin(), grown.end());
      std::vector<char> mask(ne, 0);
      std::vector<int> psi;
      for (int e : grown) {
        mask[e] = 1;
        H->cur_ncoef[e] += (int)C->coef_increase;
        H->cur_nint[e] = 2 * H->cur_ncoef[e];
        const int ty = H->h.type[e];
        if (ty == 1 || ty == 4 || ty == 5) psi.push_back(e);
      }
      // tables for the next iterations, and for re-solving the grown elements
      int rct = build_eval_tables(H);
      if (rct) return rct;
      std::vector<Group> rg;
      std::vector<int> rgo;
      std::vector<Item> ri;
      std::vector<int2> rp;
      int nrv = 0;
      build_tables(H, false, rg, rgo, ri, rp, nrv, &mask);
      CK(upload(H->rs_groups, rg, s));
      CK(upload(H->rs_group_of, rgo, s));
      CK(upload(H->rs_items, ri, s));
      CK(upload(H->rs_pts, rp, s));
      CK(upload(H->rs_list, grown, s));
      if (H->rs_vals.cap < (size_t)std::max(1, nrv)) CK(H->rs_vals.alloc(std::max(1, nrv)));
      net = H->net();
      if (!psi.empty()) {
        DBuf<int> dpsi;
        CK(upload(dpsi, psi, s));
        cuts_kernel<<<((int)psi.size() * 32 + 127) / 128, 128, 0, s>>>(net, dpsi.p, (int)psi.size());
        CK(cudaStreamSynchronize(s));
        H->launches += 1;
      }
      if (!ri.empty())
        eval_kernel<false><<<(int)ri.size(), EVAL_THREADS, H->eval_smem, s>>>(net, H->rs_items.p, H->rs_pts.p,
                                                                              H->rs_groups.p, H->rs_vals.p,
                                                                              H->chunk);
      const size_t us2 = sizeof(double) * 2 * H->nvmax * UPDATE_WARPS;
      update_kernel<<<(ngrow + UPDATE_WARPS - 1) / UPDATE_WARPS, UPDATE_WARPS * 32, us2, s>>>(
          net, H->rs_list.p, ngrow, H->rs_group_of.p, H->rs_groups.p, H->rs_vals.p, H->nvmax, 2);
      H->launches += 2;
    }
    blend2_kernel<<<std::max(1, std::min(1184, (int)((H->ne * H->MC + 255) / 256))), 256, 0, s>>>(net);
    reduce_kernel<<<H->R, 1024, 0, s>>>(net);
    H->launches += 2;
    CK(cudaMemcpyAsync(H->h_ndone, H->ndone.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (*H->h_ndone >= H->R) break;
    if (++guard > C->max_iterations + 2) break;
  }
  return 0;
}

static int read_states(AndfnHandle *H) {
  CK(cudaMemcpyAsync(H->h_st.data(), H->st.p, sizeof(SolveState) * H->R, cudaMemcpyDeviceToHost, H->stream));
  CK(cudaStreamSynchronize(H->stream));
  return 0;
}

static int run_impl(AndfnHandle *H, const AndfnConstants *C, AndfnSolveStats *S) {
  auto t_all = std::chrono::steady_clock::now();
  cudaStream_t s = H->stream;
  const int R = H->R;
  AndfnSolveStats base;
  std::memset(&base, 0, sizeof(base));
  base.device = H->device;
  H->launches = 0;
  if (C->max_ncoef > H->L.max_ncoef || C->max_iterations < 0) {
    set_error("constants out of range");
    return ANDFN_BAD_INPUT;
  }
  // Adaptive coefficient growth (hpc_solve.py:465-559) can happen when some
  // element may still grow (ncoef < MAX_NCOEF); it needs coefficient capacity
  // up to the largest reachable ncoef and the host-driven loop.
  bool growth_possible = false;
  for (int64_t i = 0; i < H->ne; i++)
    if (H->h.type[i] != 2 && H->h.ncoef[i] < C->max_ncoef) growth_possible = true;
  if (growth_possible) {
    if (C->coef_increase <= 0) {
      set_error("COEF_INCREASE must be positive");
      return ANDFN_BAD_INPUT;
    }
    // largest ncoef reachable: growth stops at the first step >= MAX_NCOEF
    int64_t top = 0;
    for (int64_t i = 0; i < H->ne; i++) {
      int64_t m = H->h.ncoef[i];
      if (H->h.type[i] != 2 && m < C->max_ncoef)
        m += C->coef_increase * ((C->max_ncoef - m + C->coef_increase - 1) / C->coef_increase);
      top = std::max(top, m);
    }
    if (top > H->L.max_ncoef) {
      set_error("adaptive growth can exceed the record capacity (element MAX_NCOEF)");
      return ANDFN_BAD_INPUT;
    }
    int rce = ensure_capacity(H, (int)top);
    if (rce) return rce;
  }
  if (H->cur_nint != H->h.nint || H->cur_ncoef != H->h.ncoef) {
    H->cur_nint = H->h.nint;
    H->cur_ncoef = H->h.ncoef;
    H->tables_dirty = true;
  }
  if (H->tables_dirty) {
    int rct = build_eval_tables(H);
    if (rct) return rct;
  }
  H->have_solution = false;
  int rc = reset_impl(H);
  if (rc) return rc;
  Net net = H->net();
  SolveState st0;
  std::memset(&st0, 0, sizeof(st0));
  st0.error_q = 1.0;
  st0.max_error = C->max_error;
  st0.damping = C->damping;
  st0.max_it = (int)C->max_iterations;
  st0.fused_blend2 = growth_possible ? 0 : 1;
  st0.solve_q = 1;
  st0.refine = 1;  // the refinement step in every explicit-inverse solve
  st0.n_refined = 0;
  st0.done = (C->max_iterations <= 0) ? 1 : 0;
  std::vector<SolveState> st_init(R, st0);
  CK(cudaMemcpyAsync(H->st.p, st_init.data(), sizeof(SolveState) * R, cudaMemcpyHostToDevice, s));
  const int ndone0 = st0.done ? R : 0;
  CK(cudaMemcpyAsync(H->ndone.p, &ndone0, sizeof(int), cudaMemcpyHostToDevice, s));
  auto t_setup = std::chrono::steady_clock::now();
  PhaseTimer pt;
  // initial discharges (get_old_discharges, hpc_solve.py:765-775), uploaded
  // before the set-up kernels (a pageable upload waits for the stream)
  {
    std::vector<double> disc0(H->N, 0.0);
    for (int g = 0; g < H->N; g++) {
      const int d = H->h.row_de[g];
      disc0[g] = d >= 0 ? H->h.q[H->h.de_ids[d]] : H->h.constant[H->h.row_frac[g]];
    }
    CK(cudaMemcpyAsync(H->disc.p, disc0.data(), sizeof(double) * H->N, cudaMemcpyHostToDevice, s));
    g_h2d_bytes += 8 * (int64_t)H->N;
  }
  init_state_kernel<<<std::max<int64_t>(1, (H->ne + 255) / 256), 256, 0, s>>>(net);
  const int n_de = (int)H->h.de_ids.size();
  if (n_de > 0) zint_kernel<<<std::max(1, std::min(1184, (int)((n_de * H->D + 255) / 256))), 256, 0, s>>>(net);
  // the matrix values first: the host factorisation waits for them only,
  // while the device goes on with the rest of the set-up
  const long long nent = (long long)H->ent_row.size();
  if (nent > 0)
    matrix_values_kernel<<<(unsigned)((nent * 32 + 255) / 256), 256, 0, s>>>(
        net, H->d_ent_row.p, H->d_ent_src.p, H->d_ent_side.p, H->d_ent_kind.p, H->d_mvals.p, nent);
  std::vector<double> mv(std::max<long long>(1, nent));
  if (nent > 0) CK(cudaMemcpyAsync(mv.data(), H->d_mvals.p, sizeof(double) * nent, cudaMemcpyDeviceToHost, s));
  g_d2h_bytes += 8 * nent;
  if (!H->mv_ev) CK(cudaEventCreateWithFlags(&H->mv_ev, cudaEventDisableTiming));
  CK(cudaEventRecord(H->mv_ev, s));
  if (H->n_psi > 0) cuts_kernel<<<(H->n_psi * 32 + 127) / 128, 128, 0, s>>>(net, H->psi_list.p, H->n_psi);
  // head vector from power sums and the sweep from pair tables, unless
  // coefficients may grow (then the points and series lengths change)
  H->use_head_sums = false;
  H->use_tab = false;
  H->tab_valid = false;
  if (!growth_possible) {
    int rch = build_head_sums(H);
    if (rch) return rch;
    pt.lap("setup: head-vector sums");
    H->use_head_sums = true;
    if (const char *v = getenv("ANDFN_B200_PAIR_TABLES"); !v || atoi(v) != 0) {
      int rcp = build_pair_table(H);
      if (rcp) return rcp;
      H->use_tab = true;
      if (!H->sweep_q.p) {
        CK(H->sweep_q.alloc(1));
        CK(cudaMemsetAsync(H->sweep_q.p, 0, sizeof(WorkQueue), s));
      }
      rcp = sweep_autotune(H);
      if (rcp) return rcp;
      pt.lap("setup: pair tables");
    }
  }
  H->launches += 4;
  CK(cudaEventSynchronize(H->mv_ev));
  pt.lap("setup: wait for matrix values");
  if (H->has_spec) {
    // the prescribed discharges' terms move to the right-hand side: minus
    // the entry times q in the rows, minus q in the continuity rows
    std::vector<double> bk(H->N, 0.0);
    for (size_t k = 0; k < H->known_row.size(); k++)
      bk[H->known_row[k]] -= mv[H->known0 + k] * H->h.q[H->known_src[k]];
    for (size_t k = 0; k < H->known_cont_row.size(); k++) bk[H->known_cont_row[k]] -= H->h.q[H->known_cont_src[k]];
    CK(upload(H->bknown, bk, s));
    g_h2d_bytes += 8 * (int64_t)H->N;
  }
  base.ms_setup = ms_since(t_setup);
  // factorisation (host)
  auto t_fac = std::chrono::steady_clock::now();
  pt.lap("setup: rest");
  if (H->order_thread.joinable() && !H->order_follow) H->order_thread.join();
  pt.lap("factor: wait for column order");
  rc = factor_all(H, mv);
  if (rc) return rc;
  pt.lap("factor");
  base.ms_factor = ms_since(t_fac);
  base.ms_factor_sparse = H->ms_fac[0];
  base.ms_factor_dense = H->ms_fac[1];
  base.ms_factor_levels = H->ms_fac[2];
  base.ms_inverse = H->ms_fac[3];
  // iterations, in graph batches
  auto t_it = std::chrono::steady_clock::now();
  int64_t loop_launches = 0;
  if (growth_possible) {
    int rca = run_adaptive(H, C);
    if (rca) return rca;
  } else {
    // a batch's kernels run over the work of its running realizations (the
    // lists are off again when the loop ends, also on an error return)
    struct ActOff {
      AndfnHandle *h;
      ~ActOff() { h->act_on = false; }
    } act_off{H};
    const char *al = getenv("ANDFN_B200_ACTIVE_LISTS");
    if (R > 1 && !(al && atoi(al) == 0)) {
      const int rca = act_setup(H, ndone0);
      if (rca) return rca;
    }
    // the whole loop in one launch (not with per-kernel event profiling,
    // whose event nodes a loop body cannot hold, nor with cluster-launched
    // triangular solves)
    bool looped = false;
    const char *dl = getenv("ANDFN_B200_DEVICE_LOOP");
    if (!H->profiling && (H->winv_ready || H->binv_ready) && !(dl && atoi(dl) == 0)) {
      int its_run = 0;
      int rcl = run_device_loop(H, C, &looped, &its_run);
      if (rcl) return rcl;
      if (looped) loop_launches = 1;
    }
    if (!looped) {
    int64_t launches_before = 0;
    if (H->graph_exec) {
      cudaGraphExecDestroy(H->graph_exec);
      H->graph_exec = nullptr;
    }
    {
      cudaGraph_t g;
      if (H->profiling && !H->ev[0][0][0])
        for (auto &bb : H->ev)
          for (auto &c : bb)
            for (auto &e : c) CK(cudaEventCreate(&e));
      launches_before = H->launches;
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      for (int b = 0; b < ITER_BATCH; b++) enqueue_iteration(H, s, 0, b);
      {
        const cudaError_t ec = cudaStreamEndCapture(s, &g);
        if (ec != cudaSuccess) {
          set_error(std::string("capture of the iteration graph: ") + cudaGetErrorString(ec) + "; " + g_last_error);
          return ANDFN_CUDA_ERROR;
        }
      }
      CK(cudaGraphInstantiate(&H->graph_exec, g, 0));
      cudaGraphDestroy(g);
    }
    const int64_t per_graph = H->launches - launches_before;  // kernels of the captured iterations
    H->launches = launches_before;                          // capture does not launch
    int guard = 0;
    int nit_before = 0;
    while (true) {
      CK(cudaGraphLaunch(H->graph_exec, s));
      CK(cudaMemcpyAsync(H->h_ndone, H->ndone.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      H->launches += per_graph;
      if (H->profiling) {
        // only the iterations that did work (later ones return at entry)
        int rcs = read_states(H);
        if (rcs) return rcs;
        int nit_max = 0;
        for (int r = 0; r < R; r++) nit_max = std::max(nit_max, H->h_st[r].nit);
        const int real = std::min(ITER_BATCH, nit_max - nit_before);
        for (int b = 0; b < real; b++)
          for (int c = 0; c < KCLASSES; c++) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, H->ev[b][c][0], H->ev[b][c][1]) == cudaSuccess) {
              H->k_ms[c] += ms;
              H->k_n[c] += 1;
            }
          }
        nit_before = nit_max;
      }
      loop_launches += 1;
      if (*H->h_ndone >= R) break;
      if (++guard > 1 + C->max_iterations / ITER_BATCH + 2) break;
    }
    }
  }
  H->act_on = false;
  rc = read_states(H);
  if (rc) return rc;
  std::vector<SolveState> fin = H->h_st;
  // hpc_solve.py:224-234: an extra element_solver sweep at nit == MAX_ITERATIONS,
  // for the realizations that stopped there
  {
    std::vector<SolveState> tmp = fin;
    bool any = false;
    for (int r = 0; r < R; r++) {
      const bool extra = fin[r].nit == C->max_iterations && !fin[r].nonfinite && fin[r].status == 0;
      tmp[r].done = extra ? 0 : 1;
      any |= extra;
    }
    if (any) {
      net = H->net();
      CK(cudaMemcpyAsync(H->st.p, tmp.data(), sizeof(SolveState) * R, cudaMemcpyHostToDevice, s));
      launch_sweep(H, net, s);
      const int ub = (H->n_upd + UPDATE_WARPS - 1) / UPDATE_WARPS;
      const size_t usmem = sizeof(double) * 2 * H->nvmax * UPDATE_WARPS;
      if (ub > 0)
        update_kernel<<<ub, UPDATE_WARPS * 32, usmem, s>>>(net, H->upd_list.p, H->n_upd, H->group_of.p,
                                                            H->d_groups.p, H->sweep_vals.p, H->nvmax, 1);
      H->launches += 2;
      CK(cudaMemcpyAsync(H->st.p, fin.data(), sizeof(SolveState) * R, cudaMemcpyHostToDevice, s));
    }
  }
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  base.ms_iterate = ms_since(t_it);
  base.gpu_launches = H->launches;
  base.ms_create_upload = H->ms_create_upload;
  base.ms_create_tables = H->ms_create_tables;
  base.ms_create_order = H->ms_create_order;
  int status = ANDFN_OK;
  H->last.assign(R, base);
  H->have_solution = true;
  for (int r = 0; r < R; r++) {
    AndfnSolveStats &st = H->last[r];
    const SolveState &f = fin[r];
    st.iterations = f.nit;
    st.cnt_error = f.cnt_error;
    st.error = f.error;
    st.error_coef = f.error_coef;
    st.error_q = f.error_q;
    st.worst_element = f.worst;
    st.n_unknowns = H->sys[r].n;
    st.nnz_matrix = (int64_t)H->sys[r].mcol.size();
    st.nnz_factors = H->sys[r].nnz;
    st.dense_tail = H->sys[r].tail_k;
    st.explicit_inverse = (H->winv_ready || H->binv_ready) ? 1 : 0;
    st.refined_solves = (H->winv_ready || H->binv_ready) ? f.n_refined : 0;
    st.sweep_variant = H->use_tab ? H->sweep_variant : -1;
    st.loop_launches = loop_launches;
    st.ms_alloc = g_alloc_ms;
    st.refine_f32 = (H->winv_ready && H->winv32_p) ? 1 : 0;
    st.levels_l = H->sys[r].nlev_l;
    st.levels_u = H->sys[r].nlev_u;
    for (int i = 0; i < 8; i++) st.tri_cycles[i] = f.tri_cycles[i];
    int sr = ANDFN_OK;
    if (f.status)
      sr = f.status;
    else if (f.nonfinite)
      sr = ANDFN_NONFINITE;
    else if (f.cnt_error < 2)
      sr = ANDFN_MAX_ITERATIONS;
    st.status = sr;
    if (sr >= ANDFN_BAD_LAYOUT)
      status = std::max(status, sr);
    else if (status < ANDFN_BAD_LAYOUT)
      status = std::max(status, sr);
    st.ms_total = ms_since(t_all);
  }
  if (S)
    for (int r = 0; r < R; r++) S[r] = H->last[r];
  return status;
}

static int download_impl(AndfnHandle *H, char *const *F, char *const *E) {
  cudaStream_t s = H->stream;
  const int64_t ne = H->ne, nf = H->nf;
  const int MC = H->MC;
  std::vector<cd> coef((size_t)ne * MC);
  std::vector<int> ncoef(ne), nint(ne);
  std::vector<double> q(ne), err(ne), eo(ne), eo2(ne), ec(ne), dc((size_t)ne * 2 * MC), cst(nf);
  CK(cudaMemcpyAsync(coef.data(), H->coef.p, sizeof(cd) * coef.size(), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(ncoef.data(), H->ncoef.p, sizeof(int) * ne, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(nint.data(), H->nint.p, sizeof(int) * ne, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(q.data(), H->q.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(err.data(), H->err.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(eo.data(), H->err_old.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(eo2.data(), H->err_old2.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(ec.data(), H->err_coef.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(dc.data(), H->dpsi_corr.p, sizeof(double) * dc.size(), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(cst.data(), H->constant.p, sizeof(double) * nf, cudaMemcpyDeviceToHost, s));
  g_d2h_bytes += (int64_t)(sizeof(cd) * coef.size() + 4 * 2 * ne + 8 * 5 * ne + 8 * dc.size() + 8 * nf);
  CK(cudaStreamSynchronize(s));
  const AndfnLayout &L = H->L;
  for (int r = 0; r < H->R; r++) {
    const int e0 = H->h.eoff[r], e1 = H->h.eoff[r + 1], f0 = H->h.foff[r], f1 = H->h.foff[r + 1];
    for (int i = e0; i < e1; i++) {
      char *rec = E[r] + (int64_t)(i - e0) * L.elem_size;
      const int m = ncoef[i], n = nint[i], ty = H->h.type[i];
      int64_t v;
      v = m;
      std::memcpy(rec + L.e_ncoef, &v, 8);
      v = n;
      std::memcpy(rec + L.e_nint, &v, 8);
      std::memcpy(rec + L.e_coef, &coef[(size_t)i * MC], sizeof(cd) * std::min(m, MC));
      // thetas as calc_thetas writes them (hpc_math_functions.py:693-699)
      double del = PI / n, start = del / 2;
      if (ty == 1) {
        del = 2 * PI / n;
        start = 0.0;
      }
      for (int k = 0; k < n; k++) {
        double th = start + k * del;
        std::memcpy(rec + L.e_thetas + 8 * k, &th, 8);
      }
      std::memcpy(rec + L.e_q, &q[i], 8);
      std::memcpy(rec + L.e_error, &err[i], 8);
      std::memcpy(rec + L.e_error_old, &eo[i], 8);
      if (ty != 2) {
        std::memcpy(rec + L.e_error_old2, &eo2[i], 8);
        std::memcpy(rec + L.e_error_coef, &ec[i], 8);
      }
      if (ty == 1 || ty == 4 || ty == 5)
        std::memcpy(rec + L.e_dpsi_corr, &dc[(size_t)i * 2 * MC], 8 * std::max(0, n - 1));
    }
    for (int f = f0; f < f1; f++) std::memcpy(F[r] + (int64_t)(f - f0) * L.frac_size + L.f_constant, &cst[f], 8);
  }
  return 0;
}

// Complex discharge vector w at points (andfn/hpc/hpc_fracture.py:139-175):
// the sum over the fracture's intersections and constant-head lines
// (derivative of the Laurent series and the log term times dchi/dz,
// hpc_intersection.py:179-225, hpc_const_head_line.py:135-164), bounding
// circle (derivative of the Taylor series in chi = z / R as the reference
// writes it, without dchi/dz, hpc_bounding_circle.py:97-115) and wells
// (hpc_well.py:89-108); impermeable elements do not contribute.
// With u = 1/chi and P(u) = sum_{k>=1} k c_k u^(k-1), the line term is
// sg (u^2 P - q u / (2 pi)) * 2 / (1 - u^2) * 2 / (b - a).
__global__ void points_w_kernel(Net net, const int *__restrict__ frac, const cd *__restrict__ z, int npts,
                                cd *__restrict__ out_w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const int f = frac[i];
  const cd zz = z[i];
  cd w = mk(0.0, 0.0);
  for (int k = net.fptr[f]; k < net.fptr[f + 1]; k++) {
    const int el = net.felem[k];
    const int ty = net.type[el];
    const int m = net.ncoef[el];
    const cd *c = net.coef + (size_t)el * net.MC;
    if (ty == 0 || ty == 3) {
      const bool neg = (ty == 0 && net.frac0[el] != f);
      const double sg = neg ? -1.0 : 1.0;
      const cd *ep = neg ? net.ep1 + 2 * el : net.ep0 + 2 * el;
      const cd inv = recip(ep[1] - ep[0]);
      const cd ab = ep[0] + ep[1];
      const cd Z = fma_c(2.0 * inv, zz, mk(-(ab.re * inv.re - ab.im * inv.im), -(ab.re * inv.im + ab.im * inv.re)));
      const cd u = recip(exterior_chi(Z));
      cd P = mk(0.0, 0.0);
      if (m >= 2) {
        P = (double)(m - 1) * c[m - 1];
        for (int j = m - 2; j >= 1; j--) P = fma_c(P, u, (double)j * c[j]);
      }
      const cd u2 = u * u;
      const cd t = u2 * P - (net.q[el] / (2 * PI)) * u;
      const cd fac = recip(mk(1.0 - u2.re, -u2.im)) * (4.0 * inv);  // 2 / (1 - u^2) * 2 / (b - a)
      w = w + (sg * t) * fac;
    } else if (ty == 1) {
      const cd chi = (1.0 / net.radius[el]) * zz;
      cd P = (net.MC > 1) ? c[1] : mk(0.0, 0.0);  // m < 2: the reference reads the record's slot 1
      if (m >= 2) {
        P = (double)(m - 1) * c[m - 1];
        for (int j = m - 2; j >= 1; j--) P = fma_c(P, chi, (double)j * c[j]);
      }
      w = w + P;
    } else if (ty == 2) {
      const double r = net.radius[el];
      const cd u = recip((1.0 / r) * (zz - net.center[el]));
      w = w + (-net.q[el] / (2 * PI * r)) * u;
    }
  }
  out_w[i] = w;
}

// Complex discharge vectors at the points of realization 0.
static int eval_w_impl(AndfnHandle *H, const int64_t *frac, const cd *z, int64_t npts, cd *out) {
  if (npts <= 0) return 0;
  if (npts > (1LL << 31) - 1) return ANDFN_BAD_INPUT;
  const int nfr = H->h.foff[1] - H->h.foff[0];
  std::vector<int> fr(npts);
  for (int64_t i = 0; i < npts; i++) {
    if (frac[i] < 0 || frac[i] >= nfr) {
      set_error("point fracture index out of range");
      return ANDFN_BAD_INPUT;
    }
    fr[i] = (int)frac[i];
  }
  cudaStream_t s = H->stream;
  DBuf<int> dfr;
  DBuf<cd> dz, dw;
  CK(dfr.alloc(npts));
  CK(dz.alloc(npts));
  CK(dw.alloc(npts));
  CK(cudaMemcpyAsync(dfr.p, fr.data(), sizeof(int) * npts, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dz.p, z, sizeof(cd) * npts, cudaMemcpyHostToDevice, s));
  points_w_kernel<<<(unsigned)((npts + 127) / 128), 128, 0, s>>>(H->net(), dfr.p, dz.p, (int)npts, dw.p);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, dw.p, sizeof(cd) * npts, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

// ---------------------------------------------------------------------------
// Streamline tracking (track.cuh): a group of TRACK_GROUP lanes per particle,
// tracing its whole streamline through the fractures it passes.
static TrackView track_view(const Net &n, const double *fgeo, const double *aperture) {
  TrackView v;
  v.MC = n.MC;
  v.type = n.type;
  v.frac0 = n.frac0;
  v.frac1 = n.frac1;
  v.ncoef = n.ncoef;
  v.ep0 = n.ep0;
  v.ep1 = n.ep1;
  v.radius = n.radius;
  v.center = n.center;
  v.q = n.q;
  v.coef = n.coef;
  v.fptr = n.fptr;
  v.felem = n.felem;
  v.fgeo = fgeo;
  v.aperture = aperture;
  return v;
}

__global__ void track_kernel(TrackView tv, int npart, const int *__restrict__ pf, const cd *__restrict__ pz,
                             const double *__restrict__ pe, double ds, int max_length, int backward, int cap,
                             cd *oz, double *ov, int *oseg, int *ofr, int *on, int *oelem, int *ostat) {
  // blockDim.x is a multiple of 32, so the TRACK_GROUP lanes of a particle sit
  // in one warp and leave (i >= npart) together.
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) / TRACK_GROUP;
  if (i >= npart) return;
  const int lane = threadIdx.x & (TRACK_GROUP - 1);
  const int base = (threadIdx.x & 31) & ~(TRACK_GROUP - 1);
  const GroupW<TRACK_GROUP> wf{tv, lane, ((1u << TRACK_GROUP) - 1u) << base};
  const size_t b = (size_t)i * (size_t)cap;
  int n = 0, el = -1;
  const int st = t_track(tv, wf, lane == 0, pf[i], pz[i], pe[i], ds, max_length, backward != 0, cap, oz + b, ov + b,
                         oseg + b, ofr + b, &n, &el);
  if (lane == 0) {
    ostat[i] = st;
    on[i] = n;
    oelem[i] = el;
  }
}

// Object-layer w (Fracture.calc_w, andfn/fracture.py:453-478) at points.
__global__ void points_w_object_kernel(TrackView tv, const int *__restrict__ frac, const cd *__restrict__ z, int npts,
                                       cd *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  out[i] = t_frac_w(tv, frac[i], z[i]);
}

static int check_frac_ids(AndfnHandle *H, const int64_t *frac, int64_t n, std::vector<int> &out) {
  if (H->R != 1) {
    set_error("tracking and object-layer fields need a single-network handle");
    return ANDFN_BAD_INPUT;
  }
  const int nfr = H->h.foff[1] - H->h.foff[0];
  out.resize(n);
  for (int64_t i = 0; i < n; i++) {
    if (frac[i] < 0 || frac[i] >= nfr) {
      set_error("point fracture index out of range");
      return ANDFN_BAD_INPUT;
    }
    out[i] = (int)frac[i];
  }
  return 0;
}

static int eval_w_object_impl(AndfnHandle *H, const int64_t *frac, const cd *z, int64_t npts, cd *out) {
  if (npts <= 0) return 0;
  if (npts > (1LL << 31) - 1) return ANDFN_BAD_INPUT;
  std::vector<int> fr;
  if (int rc = check_frac_ids(H, frac, npts, fr)) return rc;
  cudaStream_t s = H->stream;
  DBuf<int> dfr;
  DBuf<cd> dz, dw;
  CK(dfr.alloc(npts));
  CK(dz.alloc(npts));
  CK(dw.alloc(npts));
  CK(cudaMemcpyAsync(dfr.p, fr.data(), sizeof(int) * npts, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dz.p, z, sizeof(cd) * npts, cudaMemcpyHostToDevice, s));
  points_w_object_kernel<<<(unsigned)((npts + 127) / 128), 128, 0, s>>>(track_view(H->net(), nullptr, nullptr), dfr.p,
                                                                         dz.p, (int)npts, dw.p);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, dw.p, sizeof(cd) * npts, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

static int track_impl(AndfnHandle *H, const void *frac_recs, int64_t nf, const double *aperture, int64_t npart,
                      const int64_t *frac, const cd *z, const double *elev, double ds, int64_t max_length,
                      int backward, int64_t cap, cd *out_z, double *out_v, int64_t *out_seg, int64_t *out_frac,
                      int64_t *out_n, int64_t *out_elem, int32_t *out_status) {
  if (npart <= 0) return 0;
  std::vector<int> pf;
  if (int rc = check_frac_ids(H, frac, npart, pf)) return rc;
  if (nf != H->h.foff[1] - H->h.foff[0]) {
    set_error("fracture count differs from the handle's network");
    return ANDFN_BAD_INPUT;
  }
  if (cap < 2 || cap > (1LL << 30) || max_length < 0 || max_length > (1LL << 30) || npart > (1LL << 27) ||
      npart * cap > (1LL << 31)) {
    set_error("track: cap, max_length or the particle count out of range");
    return ANDFN_BAD_INPUT;
  }
  const AndfnLayout &L = H->L;
  std::vector<double> geo((size_t)nf * TRACK_FGEO);
  for (int64_t f = 0; f < nf; f++) {
    const char *rec = static_cast<const char *>(frac_recs) + f * L.frac_size;
    double *g = &geo[(size_t)f * TRACK_FGEO];
    std::memcpy(g, rec + L.f_radius, 8);
    std::memcpy(g + 1, rec + L.f_center, 24);
    std::memcpy(g + 4, rec + L.f_x_vector, 24);
    std::memcpy(g + 7, rec + L.f_y_vector, 24);
    std::memcpy(g + 10, rec + L.f_normal, 24);
  }
  cudaStream_t s = H->stream;
  const size_t slots = (size_t)npart * (size_t)cap;
  DBuf<double> dgeo, dap, dpe, dov;
  DBuf<int> dpf, dseg, dfr, dn, del, dst;
  DBuf<cd> dpz, doz;
  CK(dgeo.alloc(geo.size()));
  CK(dap.alloc(nf));
  CK(dpe.alloc(npart));
  CK(dpf.alloc(npart));
  CK(dpz.alloc(npart));
  CK(doz.alloc(slots));
  CK(dov.alloc(slots));
  CK(dseg.alloc(slots));
  CK(dfr.alloc(slots));
  CK(dn.alloc(npart));
  CK(del.alloc(npart));
  CK(dst.alloc(npart));
  CK(cudaMemcpyAsync(dgeo.p, geo.data(), sizeof(double) * geo.size(), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dap.p, aperture, sizeof(double) * nf, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dpe.p, elev, sizeof(double) * npart, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dpf.p, pf.data(), sizeof(int) * npart, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dpz.p, z, sizeof(cd) * npart, cudaMemcpyHostToDevice, s));
  track_kernel<<<(unsigned)((npart * TRACK_GROUP + 127) / 128), 128, 0, s>>>(track_view(H->net(), dgeo.p, dap.p),
                                                                              (int)npart, dpf.p,
                                                            dpz.p, dpe.p, ds, (int)max_length, backward, (int)cap,
                                                            doz.p, dov.p, dseg.p, dfr.p, dn.p, del.p, dst.p);
  CK(cudaGetLastError());
  std::vector<int> seg(slots), fr(slots), n(npart), el(npart);
  CK(cudaMemcpyAsync(out_z, doz.p, sizeof(cd) * slots, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(out_v, dov.p, sizeof(double) * slots, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(seg.data(), dseg.p, sizeof(int) * slots, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(fr.data(), dfr.p, sizeof(int) * slots, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(n.data(), dn.p, sizeof(int) * npart, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(el.data(), del.p, sizeof(int) * npart, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(out_status, dst.p, sizeof(int32_t) * npart, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int64_t i = 0; i < npart; i++) {
    out_n[i] = n[i];
    out_elem[i] = el[i];
    const size_t b = (size_t)i * (size_t)cap;
    for (int k = 0; k < n[i]; k++) {
      out_seg[b + k] = seg[b + k];
      out_frac[b + k] = fr[b + k];
    }
  }
  return 0;
}

// Points of realization r (fracture indices local to it).
static int eval_points_impl(AndfnHandle *H, int64_t r, const int64_t *frac, const double *z, int64_t npts,
                            double *omega, double *head) {
  if (r < 0 || r >= H->R) {
    set_error("realization index out of range");
    return ANDFN_BAD_INPUT;
  }
  if (npts <= 0) return 0;
  if (npts > (1LL << 31) - 1) return ANDFN_BAD_INPUT;
  const int f0 = H->h.foff[r], nfr = H->h.foff[r + 1] - f0;
  std::vector<int> fr(npts);
  for (int64_t i = 0; i < npts; i++) {
    if (frac[i] < 0 || frac[i] >= nfr) {
      set_error("point fracture index out of range");
      return ANDFN_BAD_INPUT;
    }
    fr[i] = f0 + (int)frac[i];
  }
  cudaStream_t s = H->stream;
  DBuf<int> dfr;
  DBuf<cd> dz, dom;
  DBuf<double> dh;
  CK(dfr.alloc(npts));
  CK(dz.alloc(npts));
  CK(cudaMemcpyAsync(dfr.p, fr.data(), sizeof(int) * npts, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(dz.p, z, sizeof(cd) * npts, cudaMemcpyHostToDevice, s));
  if (omega) CK(dom.alloc(npts));
  if (head) CK(dh.alloc(npts));
  points_kernel<<<(unsigned)((npts + 127) / 128), 128, 0, s>>>(H->net(), dfr.p, dz.p, (int)npts, dom.p, dh.p);
  CK(cudaGetLastError());
  if (omega) CK(cudaMemcpyAsync(omega, dom.p, sizeof(cd) * npts, cudaMemcpyDeviceToHost, s));
  if (head) CK(cudaMemcpyAsync(head, dh.p, sizeof(double) * npts, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

}  // namespace andfn

// ==========================================================================
// C ABI
// ==========================================================================
extern "C" {

const char *andfn_b200_last_error(void) { return g_last_error.c_str(); }
const char *andfn_b200_version(void) { return "andfn_b200 0.2.0 (sm_100a, fp64)"; }

int andfn_b200_batch_create(AndfnHandle **out, int64_t R, void *const *frac_recs, const int64_t *nf,
                            void *const *elem_recs, const int64_t *ne, const AndfnLayout *layout,
                            int64_t discharge_int, int32_t device) {
  if (!out) return ANDFN_BAD_INPUT;
  *out = nullptr;
  if (check_layout(layout)) {
    set_error("inconsistent record layout");
    return ANDFN_BAD_LAYOUT;
  }
  if (R < 1 || R > (1 << 20) || !frac_recs || !elem_recs || !nf || !ne || discharge_int < 1 ||
      discharge_int > 100000) {
    set_error("bad realization count, pointers or discharge_int");
    return ANDFN_BAD_INPUT;
  }
  int64_t tot_e = 0, tot_f = 0;
  for (int64_t r = 0; r < R; r++) {
    if (nf[r] <= 0 || ne[r] <= 0 || !frac_recs[r] || !elem_recs[r]) {
      set_error("empty network in the batch");
      return ANDFN_BAD_INPUT;
    }
    tot_e += ne[r];
    tot_f += nf[r];
  }
  if (tot_e > (1LL << 30) || tot_f > (1LL << 30)) {
    set_error("batch too large");
    return ANDFN_BAD_INPUT;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device visible");
    return ANDFN_NO_DEVICE;
  }
  AndfnHandle *H = new AndfnHandle();
  if (device >= 0) {
    if (cudaSetDevice(device) != cudaSuccess) {
      delete H;
      set_error("cudaSetDevice failed");
      return ANDFN_NO_DEVICE;
    }
  }
  cudaGetDevice(&H->device);
  // two attributes, not cudaGetDeviceProperties (which queries them all and
  // costs milliseconds a call)
  int major = 0;
  cudaDeviceGetAttribute(&H->num_sms, cudaDevAttrMultiProcessorCount, H->device);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, H->device);
  if (major < 10) {
    delete H;
    set_error("an sm_100 (Blackwell) device is required");
    return ANDFN_NO_DEVICE;
  }
  if (cudaStreamCreateWithFlags(&H->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete H;
    set_error("cudaStreamCreate failed");
    return ANDFN_CUDA_ERROR;
  }
  PoolStream pool_scope(H->stream);
  H->L = *layout;
  if (const char *v = getenv("ANDFN_B200_SOLVE_THREADS")) {
    int t = atoi(v);
    if (t >= 32 && t <= SOLVE_THREADS && t % 32 == 0) H->solve_threads = t;
  }
  H->D = discharge_int;
  if (const char *v = getenv("ANDFN_B200_EXPLICIT_INVERSE")) H->winv_enabled = atoi(v) != 0;
  int rc = create_impl(H, (int)R, (const char *const *)frac_recs, nf, (const char *const *)elem_recs, ne);
  if (rc) {
    delete H;
    return rc;
  }
  *out = H;
  return 0;
}

int andfn_b200_create(AndfnHandle **out, const void *frac_recs, int64_t nf, const void *elem_recs, int64_t ne,
                      const AndfnLayout *layout, int64_t discharge_int, int32_t device) {
  void *F[1] = {const_cast<void *>(frac_recs)};
  void *E[1] = {const_cast<void *>(elem_recs)};
  return andfn_b200_batch_create(out, 1, F, &nf, E, &ne, layout, discharge_int, device);
}

int64_t andfn_b200_realizations(AndfnHandle *H) { return H ? H->R : 0; }

int andfn_b200_upload_state(AndfnHandle *H, const void *frac_recs, const void *elem_recs) {
  if (!H || H->R != 1) {
    set_error("upload_state needs a single-network handle");
    return ANDFN_BAD_INPUT;
  }
  H->have_solution = false;
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  const char *E = (const char *)elem_recs;
  const char *F = (const char *)frac_recs;
  const AndfnLayout &L = H->L;
  for (int64_t i = 0; i < H->ne; i++) {
    const char *r = E + i * L.elem_size;
    H->h.q[i] = rd_f64(r, L.e_q);
    H->h.err[i] = rd_f64(r, L.e_error);
    H->h.err_old[i] = rd_f64(r, L.e_error_old);
    H->h.err_old2[i] = rd_f64(r, L.e_error_old2);
    H->h.err_coef[i] = rd_f64(r, L.e_error_coef);
    int64_t m = rd_i64(r, L.e_ncoef);
    if (m != H->h.ncoef[i]) {
      set_error("upload_state: ncoef changed; create a new handle");
      return ANDFN_BAD_INPUT;
    }
  }
  for (int64_t f = 0; f < H->nf; f++) H->h.constant[f] = rd_f64(F + f * L.frac_size, L.f_constant);
  std::fill(H->h.coef.begin(), H->h.coef.end(), mk(0.0, 0.0));
  read_coefs(H, 0, E);
  cudaStream_t s = H->stream;
  CK(cudaMemcpyAsync(H->q0.p, H->h.q.data(), 8 * H->ne, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(H->err_in.p, H->h.err.data(), 8 * H->ne, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(H->err_old_in.p, H->h.err_old.data(), 8 * H->ne, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(H->err_old2_in.p, H->h.err_old2.data(), 8 * H->ne, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(H->err_coef_in.p, H->h.err_coef.data(), 8 * H->ne, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(H->constant0.p, H->h.constant.data(), 8 * H->nf, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(H->coef0.p, H->h.coef.data(), sizeof(cd) * H->h.coef.size(), cudaMemcpyHostToDevice, s));
  int rc = reset_impl(H);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s));
  return 0;
}

int andfn_b200_reset_state(AndfnHandle *H) {
  if (!H) return ANDFN_BAD_INPUT;
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  H->have_solution = false;
  int rc = reset_impl(H);
  if (rc) return rc;
  CK(cudaStreamSynchronize(H->stream));
  return 0;
}

int andfn_b200_batch_run(AndfnHandle *H, const AndfnConstants *constants, AndfnSolveStats *stats) {
  if (!H || !constants) return ANDFN_BAD_INPUT;
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  return run_impl(H, constants, stats);
}

int andfn_b200_run(AndfnHandle *H, const AndfnConstants *constants, AndfnSolveStats *stats) {
  if (!H || !constants) return ANDFN_BAD_INPUT;
  if (H->R != 1) {
    set_error("run() on a batch handle: use andfn_b200_batch_run");
    return ANDFN_BAD_INPUT;
  }
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  return run_impl(H, constants, stats);
}

int andfn_b200_batch_download(AndfnHandle *H, void *const *frac_recs, void *const *elem_recs) {
  if (!H || !frac_recs || !elem_recs) return ANDFN_BAD_INPUT;
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  return download_impl(H, (char *const *)frac_recs, (char *const *)elem_recs);
}

int andfn_b200_download(AndfnHandle *H, void *frac_recs, void *elem_recs) {
  if (!H || !frac_recs || !elem_recs || H->R != 1) return ANDFN_BAD_INPUT;
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  char *F[1] = {(char *)frac_recs};
  char *E[1] = {(char *)elem_recs};
  return download_impl(H, F, E);
}

int andfn_b200_eval_heads(AndfnHandle *H, const int64_t *frac, const double *z, int64_t npts, double *out) {
  if (!H || (npts > 0 && (!frac || !z || !out))) return ANDFN_BAD_INPUT;
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  return eval_points_impl(H, 0, frac, z, npts, nullptr, out);
}

int andfn_b200_batch_eval_heads(AndfnHandle *H, int64_t r, const int64_t *frac, const double *z, int64_t npts,
                                double *out) {
  if (!H || (npts > 0 && (!frac || !z || !out))) return ANDFN_BAD_INPUT;
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  return eval_points_impl(H, r, frac, z, npts, nullptr, out);
}

int andfn_b200_eval_omega(AndfnHandle *H, const int64_t *frac, const double *z, int64_t npts, double *out) {
  if (!H || (npts > 0 && (!frac || !z || !out))) return ANDFN_BAD_INPUT;
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  return eval_points_impl(H, 0, frac, z, npts, out, nullptr);
}

int andfn_b200_eval_w(AndfnHandle *H, const int64_t *frac, const double *z, int64_t npts, double *out) {
  if (!H || (npts > 0 && (!frac || !z || !out))) return ANDFN_BAD_INPUT;
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  return eval_w_impl(H, frac, reinterpret_cast<const cd *>(z), npts, reinterpret_cast<cd *>(out));
}

int andfn_b200_eval_w_object(AndfnHandle *H, const int64_t *frac, const double *z, int64_t npts, double *out) {
  if (!H || (npts > 0 && (!frac || !z || !out))) return ANDFN_BAD_INPUT;
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  return eval_w_object_impl(H, frac, reinterpret_cast<const cd *>(z), npts, reinterpret_cast<cd *>(out));
}

int andfn_b200_track(AndfnHandle *H, const void *frac_recs, int64_t nf, const double *aperture, int64_t npart,
                     const int64_t *frac, const double *z, const double *elevation, double ds, int64_t max_length,
                     int32_t backward, int64_t cap, double *out_z, double *out_v, int64_t *out_seg,
                     int64_t *out_frac, int64_t *out_n, int64_t *out_elem, int32_t *out_status) {
  if (!H || (npart > 0 && (!frac_recs || !aperture || !frac || !z || !elevation || !out_z || !out_v || !out_seg ||
                           !out_frac || !out_n || !out_elem || !out_status)))
    return ANDFN_BAD_INPUT;
  cudaSetDevice(H->device);
  PoolStream pool_scope(H->stream);
  return track_impl(H, frac_recs, nf, aperture, npart, frac, reinterpret_cast<const cd *>(z), elevation, ds,
                    max_length, backward, cap, reinterpret_cast<cd *>(out_z), out_v, out_seg, out_frac, out_n,
                    out_elem, out_status);
}

void andfn_b200_destroy(AndfnHandle *H) {
  if (!H) return;
  cudaSetDevice(H->device);
  cudaStreamSynchronize(H->stream);
  PoolStream pool_scope(nullptr);  // the stream is idle: blocks go back to the cache with no event
  delete H;
}

void *andfn_b200_stream(AndfnHandle *H) { return H ? (void *)H->stream : nullptr; }

int andfn_b200_set_profiling(AndfnHandle *H, int on) {
  if (!H) return ANDFN_BAD_INPUT;
  H->profiling = on ? 1 : 0;
  for (int c = 0; c < KCLASSES; c++) {
    H->k_ms[c] = 0.0;
    H->k_n[c] = 0;
  }
  return 0;
}

int andfn_b200_kernel_times(AndfnHandle *H, double *ms, int64_t *launches, int n) {
  if (!H || n < KCLASSES) return ANDFN_BAD_INPUT;
  for (int c = 0; c < KCLASSES; c++) {
    ms[c] = H->k_ms[c];
    launches[c] = H->k_n[c];
  }
  return 0;
}

int andfn_b200_fp64_peak(int32_t device, double *tflops) {
  if (!tflops) return ANDFN_BAD_INPUT;
  if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return ANDFN_NO_DEVICE;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  double *d = nullptr;
  CK(cudaMalloc(&d, sizeof(double)));
  const int iters = 1 << 14, threads = 256, blocks = nsm * 8;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  fp64_peak_kernel<<<blocks, threads>>>(d, 64, 1.0000001, 1e-7);
  float best = 1e30f;
  for (int r = 0; r < 5; r++) {
    cudaEventRecord(a);
    fp64_peak_kernel<<<blocks, threads>>>(d, iters, 1.0000001, 1e-7);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d);
  CK(cudaGetLastError());
  *tflops = 2.0 * 8.0 * iters * (double)threads * blocks / (best * 1e-3) / 1e12;
  return 0;
}

void andfn_b200_release_cached_memory(void) {
  pinned_flush();
  DevicePool &P = device_pool();
  std::lock_guard<std::mutex> lk(P.m);
  int cur = 0;
  cudaGetDevice(&cur);
  for (int d = 0; d < 64; d++) {
    if (P.free_blocks[d].empty()) continue;
    cudaSetDevice(d);
    pool_flush_device(P, d);
  }
  cudaSetDevice(cur);
}

int andfn_b200_cached_memory(int32_t device, int64_t *bytes, int64_t *hits, int64_t *misses) {
  if (device < 0 || device >= 64) return ANDFN_BAD_INPUT;
  DevicePool &P = device_pool();
  std::lock_guard<std::mutex> lk(P.m);
  if (bytes) *bytes = (int64_t)P.held[device];
  if (hits) *hits = P.hits;
  if (misses) *misses = P.misses;
  return 0;
}

int andfn_b200_batch_solve(int64_t R, void *const *frac_recs, const int64_t *nf, void *const *elem_recs,
                           const int64_t *ne, const AndfnLayout *layout, int64_t discharge_int,
                           const AndfnConstants *constants, AndfnSolveStats *stats) {
  auto t0 = std::chrono::steady_clock::now();
  g_h2d_bytes = g_d2h_bytes = 0;
  g_alloc_ms = 0.0;
  AndfnHandle *H = nullptr;
  int rc = andfn_b200_batch_create(&H, R, frac_recs, nf, elem_recs, ne, layout, discharge_int, -1);
  if (rc) return rc;
  H->tune_sweep = false;  // a cached choice of an earlier handle, or the per-item form
  PoolStream pool_scope(H->stream);
  const double ms_up = ms_since(t0);
  rc = run_impl(H, constants, nullptr);
  double ms_down = 0;
  if (rc == ANDFN_OK || rc == ANDFN_MAX_ITERATIONS || rc == ANDFN_NONFINITE) {
    auto t1 = std::chrono::steady_clock::now();
    int rc2 = download_impl(H, (char *const *)frac_recs, (char *const *)elem_recs);
    ms_down = ms_since(t1);
    if (rc2) rc = rc2;
  }
  const double ms_tot = ms_since(t0);
  if (stats)
    for (int64_t r = 0; r < R && r < (int64_t)H->last.size(); r++) {
      stats[r] = H->last[r];
      stats[r].ms_upload = ms_up;
      stats[r].ms_download = ms_down;
      stats[r].ms_total = ms_tot;
      stats[r].h2d_bytes = g_h2d_bytes;
      stats[r].d2h_bytes = g_d2h_bytes;
    }
  andfn_b200_destroy(H);
  if (stats)
    for (int64_t r = 0; r < R; r++) stats[r].ms_alloc = g_alloc_ms;  // creation, run and destruction
  return rc;
}

int andfn_b200_solve(void *frac_recs, int64_t nf, void *elem_recs, int64_t ne, const AndfnLayout *layout,
                     int64_t discharge_int, const AndfnConstants *constants, AndfnSolveStats *stats) {
  void *F[1] = {frac_recs};
  void *E[1] = {elem_recs};
  return andfn_b200_batch_solve(1, F, &nf, E, &ne, layout, discharge_int, constants, stats);
}

}  // extern "C"

// ==========================================================================
// Head evaluation without device allocation.
//
// andfn_b200_eval_heads allocates device buffers for the points on every
// call (cudaMalloc, and cudaFree, which waits for the whole device).  Some
// callers cannot do that: a process whose memory pool already holds the
// device memory it is allowed, or a loop that must not stall other streams
// on the device.  This variant stages the points in one fixed device array
// of NOALLOC_MAX_POINTS entries that lives in the library image, so a call
// allocates nothing on the device or the host.
//
// * The first call on a device looks up the array's address
//   (cudaGetSymbolAddress, with that device current) and caches it; make
//   that first call before any stream capture on the device.  The address
//   belongs to the device's primary context: the cache assumes that context
//   lives as long as the library (no cudaDeviceReset in between).
// * Nothing in the array has to start at zero: every entry the kernel reads
//   is copied in by the same call first, and the kernel writes every result
//   entry that is copied out.
// * There is one array per device, shared by all handles: calls that
//   overlap in time on one device (from several host threads) race on it and
//   must be serialised by the caller.
// ==========================================================================
namespace andfn {

static constexpr int NOALLOC_MAX_POINTS = 65536;

struct NoAllocScratch {
  int64_t frac[NOALLOC_MAX_POINTS];  // fracture of each point (local index)
  cd z[NOALLOC_MAX_POINTS];          // point in the fracture's plane
  double head[NOALLOC_MAX_POINTS];   // result
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// One thread per point; fracture indices are local to the realization whose
// fractures start at f0.
__global__ void heads_noalloc_kernel(Net net, NoAllocScratch *s, int npts, int f0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const int f = f0 + (int)s->frac[i];
  s->head[i] = omega_at(net, f, s->z[i]).re / net.t[f];
}

static NoAllocScratch *g_noalloc_ptr[64] = {};

}  // namespace andfn

extern "C" int andfn_b200_eval_heads_noalloc(AndfnHandle *H, const int64_t *frac, const double *z, int64_t npts,
                                             double *out) {
  if (!H || (npts > 0 && (!frac || !z || !out)) || npts < 0) return ANDFN_BAD_INPUT;
  if (npts > NOALLOC_MAX_POINTS) {
    set_error("eval_heads_noalloc: more points than its fixed device array holds (65536); split the call or "
              "use andfn_b200_eval_heads");
    return ANDFN_BAD_INPUT;
  }
  const int64_t nfr = H->h.foff[1] - H->h.foff[0];
  for (int64_t i = 0; i < npts; i++)
    if (frac[i] < 0 || frac[i] >= nfr) {
      set_error("point fracture index out of range");
      return ANDFN_BAD_INPUT;
    }
  if (H->device < 0 || H->device >= 64) {
    set_error("eval_heads_noalloc: device ordinal above 63");
    return ANDFN_NO_DEVICE;
  }
  CK(cudaSetDevice(H->device));
  PoolStream pool_scope(H->stream);
  NoAllocScratch *s = g_noalloc_ptr[H->device];
  if (!s) {  // first call on this device: look the array up once
    void *p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    s = static_cast<NoAllocScratch *>(p);
    g_noalloc_ptr[H->device] = s;
  }
  if (npts == 0) return 0;
  cudaStream_t st = H->stream;
  CK(cudaMemcpyAsync(s->frac, frac, sizeof(int64_t) * npts, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(s->z, z, sizeof(cd) * npts, cudaMemcpyHostToDevice, st));
  heads_noalloc_kernel<<<(unsigned)((npts + 127) / 128), 128, 0, st>>>(H->net(), s, (int)npts, H->h.foff[0]);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, s->head, sizeof(double) * npts, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return 0;
}

// ==========================================================================
// Adjoint: the gradient of an objective J(coef, q, C, log t) with respect to
// the natural log of every fracture's transmissivity, through the converged
// solve (no reference counterpart; the reference computes no derivatives).
//
// At convergence the solve satisfies, with c the element coefficients, d =
// (q of the discharge elements, fracture constants C) and theta = log t,
//     c = Phi(c, d, theta)          element sweep (evaluation, DFT fit,
//                                   per-type update; hpc_solve.py:311-390)
//     A(theta) d = b(c, theta)      discharge system (hpc_solve.py:594-887)
// Both are linear in (c, d).  With the Lagrangian
//     L = J + lam^T (Phi - c) + mu^T (b - A d)
// the multipliers solve
//     mu  = A^-T (dJ/dd + Phi_d^T lam)
//     lam = dJ/dc + Phi_c^T lam + b_c^T mu
// and dJ/dtheta = J_theta + lam^T Phi_theta + mu^T (b_theta - A_theta d).
// Eliminating mu, lam solves the linear system (I - T^T) lam = F(0), T^T the
// transpose of the forward loop's (undamped) iteration operator; it is
// solved by restarted GMRES whose operator is one transposed sweep, so no
// forward iterate is stored.  A transposed sweep runs the transposes of the
// forward kernels:
//   adj_fit_kernel        the DFT fit and per-type update transposed: lam ->
//                         weights at the collocation points (+ the q terms of
//                         the stream-function branch-cut unwrapping)
//   adj_sweep_kernel      the sweep evaluation transposed: point weights ->
//                         dJ/d(coef, q, C) of the source elements
//   trisolve_kernel<1>    A^-T with the transposed factors of the last run
//   adj_rhs_gather_kernel the head-vector evaluation transposed (b_c^T mu),
//                         from power sums precomputed by rhs_sums_kernel
//   adj_combine_kernel    (I - T^T) x, or the residual F(x) - x
// theta enters Phi only through the intersection update
// (t0 c1 - t1 c0) / (t0 + t1), b through 1/t of the intersection rows and
// phi = t * head of constant-head lines and wells, and A through 1/t of the
// intersection rows.  Complex quantities are (d/dRe, d/dIm) pairs.
// ==========================================================================
namespace andfn {

static constexpr int ADJ_ITEM = EVAL_THREADS * 4;  // points of one adj_sweep_kernel item

// The kernels shared with the forward loop return at entry when s.done is set;
// the adjoint keeps it 0.
struct AdjState {
  SolveState s;
};

// GMRES cycle state of the adjoint on the device (see gm_givens_kernel).
static constexpr int GM_MK = 40;  // Krylov basis size before a restart
struct GmresDev {
  int j, stop, k, nonfinite;
  long long matvecs, max_it;
  double bnorm, tol, rel, scale;
  double cs[GM_MK], sn[GM_MK], gv[GM_MK + 1];
  double Hm[(GM_MK + 1) * GM_MK];  // row-major (GM_MK + 1) x GM_MK
};

struct AdjBufs {
  DBuf<AdjState> st;
  DBuf<SolveState> st_eval;
  DBuf<cd> lam, gobj, gc;          // [ne][MC]
  DBuf<double> gq, gC, gd, b, mu;  // [ne], [nf], [N], [N], [N]
  DBuf<double> wsw, gtheta, obar, gd0, hbuf;
  DBuf<cd> V, xin, wv;  // Krylov basis [restart + 1][ne][MC], sweep input and output
  DBuf<GmresDev> gm;    // GMRES cycle state
  cudaGraphExec_t step_graph = nullptr;  // one Arnoldi step
  // transposed explicit inverse (rows padded like the forward one) and A^T
  // in CSR form (value index of each entry in A's entry order)
  DBuf<double> xt;
  DBuf<float> xt32;  // float copy of xt for the refinement pass
  float *xt32_p = nullptr;
  DBuf<int> at_ptr, at_col, at_map;
  bool use_winv = false;
  DBuf<Item> items_sw;
  int n_items_sw = 0;
  DBuf<Item> items_tab;  // items of adj_sweep_table_kernel (ADJ_TAB_PTS points of one fracture)
  int n_items_tab = 0;
  DBuf<double> fac;  // [2 n_de] weight of a row side per unit mu
  int chunk = 1;
  size_t smem = 0;
  // transposed factors
  DBuf<int> lev[4], rows[4], eptr[4], col[4];
  DBuf<double> val[4], scale0, tl, tones, tw;
  DBuf<int> pinv, qcol;
  DBuf<TriDesc> tri;
  int max_nlev = 1;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // one transposed sweep, mode 0 / 1
  ~AdjBufs() {
    for (auto g : graph)
      if (g) cudaGraphExecDestroy(g);
    if (step_graph) cudaGraphExecDestroy(step_graph);
  }
};

static void destroy_adj(AdjBufs *a) { delete a; }

// The DFT fit and per-type update of one element transposed (one warp): lam
// (the multiplier of the element's new coefficients) -> weights of the
// values at its collocation points, written to wsw in the sweep-value
// layout.  For stream-function elements the branch-cut unwrapping
// (psi'_k = psi_k - sum over cuts before k of sign * q) adds
// -sign * (sum of the weights after the cut) to the cut's discharge element.
__global__ void __launch_bounds__(UPDATE_WARPS * 32) adj_fit_kernel(Net net, const cd *__restrict__ lam,
                                                                     const int *__restrict__ group_of,
                                                                     const Group *__restrict__ groups, double *wsw,
                                                                     double *gq, int nvmax, const AdjState *as) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (as->s.done) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *wk = reinterpret_cast<double *>(smem_raw) + (size_t)warp * nvmax;
  const int e = blockIdx.x * UPDATE_WARPS + warp;
  if (e >= net.ne) return;
  const int type = net.type[e];
  if (type == 2) return;
  const int n = net.nint[e], m = net.ncoef[e];
  const cd *L = lam + (size_t)e * net.MC;
  double del = PI / n, start = del / 2;
  if (type == 1) {
    del = 2 * PI / n;
    start = 0.0;
  }
  const double t0 = net.t[net.frac0[e]], t1 = (type == 0) ? net.t[net.frac1[e]] : 0.0;
  const int sides = (type == 0) ? 2 : 1;
  const double tn = 2.0 / n;
  for (int s = 0; s < sides; s++) {
    const Group g = groups[group_of[2 * e + s]];
    const double side_f = (type == 0) ? (s ? t0 / (t0 + t1) : -t1 / (t0 + t1)) : 0.0;
    for (int k = lane; k < n; k += 32) {
      double sn, cs;
      sincos(start + k * del, &sn, &cs);
      double cj = 1.0, sj = 0.0, acc = 0.0;
      for (int j = 0; j < m; j++) {
        const cd l = L[j];
        double a = 0.0, b = 0.0;  // weights of cos(j theta_k) and sin(j theta_k)
        if (type == 0) {
          if (j >= 1) a = side_f * l.re * tn;
        } else if (type == 3) {
          if (j >= 1) a = -l.re * tn;
        } else if (type == 1) {
          const double h = (j == 0) ? 0.5 : 1.0;
          a = -l.im * tn * h;
          b = -l.re * tn * h;
        } else if (type == 4) {
          if (j >= 1) {
            a = -l.im * tn;
            b = l.re * tn;
          }
        } else {  // type 5
          if (j >= 1) a = -l.im * tn;
        }
        acc = fma(a, cj, fma(b, sj, acc));
        const double c2 = cj * cs - sj * sn;
        sj = sj * cs + cj * sn;
        cj = c2;
      }
      wk[k] = acc;
      wsw[g.out + k] = acc;
    }
  }
  if (type == 1 || type == 4 || type == 5) {
    __syncwarp();
    const int nc = net.cut_n[e];
    const int *cp = net.cut_pos + (size_t)e * net.cut_cap;
    const int *ce = net.cut_elem + (size_t)e * net.cut_cap;
    const int *cs = net.cut_sign + (size_t)e * net.cut_cap;
    for (int c = lane; c < nc; c += 32) {
      double sum = 0.0;
      for (int k = cp[c] + 1; k < n; k++) sum += wk[k];
      atomicAdd(&gq[ce[c]], -(double)cs[c] * sum);
    }
  }
}

// The sweep evaluation transposed: every collocation point carries a weight
// w (the adjoint of the value eval_kernel writes there); every source element
// of the point's fracture except the point's own element receives w times the
// derivative of that value with respect to its coefficients (complex pairs),
// its discharge (log term) and the fracture constant (phi points).  An item
// holds up to EVAL_THREADS * P points of one fracture, P = 1, 2 or 4 (in
// item.pad), each thread P of them.  Per source and coefficient every lane
// sums its points, the lanes' sums go to a per-warp shared-memory table and
// lane j adds up column j, so a warp spends one table write per coefficient
// instead of a shuffle reduction; the block's sums go to global memory once
// per source chunk.
static constexpr int ADJ_RED_STRIDE = 33;  // lanes + 1 (bank spread)

template <int P>
__device__ __forceinline__ void adj_sweep_body(const Net &net, const Item &it, const int2 *__restrict__ pts,
                                               const Group *__restrict__ groups, const double *__restrict__ wsw,
                                               cd *gc, double *gq, double *gC, int chunk, unsigned char *smem) {
  const int MC = net.MC;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Src *src = reinterpret_cast<Src *>(smem);
  cd *sacc = reinterpret_cast<cd *>(smem + sizeof(Src) * chunk);
  double *sq = reinterpret_cast<double *>(sacc + (size_t)chunk * MC);
  double *red_re = sq + chunk + (size_t)warp * 2 * MC * ADJ_RED_STRIDE;
  double *red_im = red_re + (size_t)MC * ADJ_RED_STRIDE;
  __shared__ double s_cw[EVAL_THREADS / 32];
  const int f = it.frac;
  cd z[P];
  double w[P];
  int excl[P], kind[P];
  double cw = 0.0;
#pragma unroll
  for (int i = 0; i < P; i++) {
    const int p = it.p0 + threadIdx.x + i * EVAL_THREADS;
    z[i] = mk(0.0, 0.0);
    w[i] = 0.0;
    excl[i] = -1;
    kind[i] = KIND_PHI;
    if (p < it.p1) {
      const int2 gk = pts[p];
      const Group g = groups[gk.x];
      w[i] = wsw[g.out + gk.y];
      excl[i] = g.elem;
      kind[i] = g.kind;
      z[i] = sweep_point(net, g.elem, g.side, gk.y);
      if (g.kind == KIND_PHI) cw += w[i];
    }
  }
  const int e0 = net.fptr[f], e1 = net.fptr[f + 1];
  for (int base = e0; base < e1; base += chunk) {
    const int cnt = min(chunk, e1 - base);
    __syncthreads();
    for (int s = threadIdx.x; s < cnt; s += blockDim.x) {
      const int el = net.felem[base + s];
      Src h;
      h.id = el;
      h.type = net.type[el];
      h.m = net.ncoef[el];
      h.pad = (h.type == 0 && net.frac0[el] != f) ? 1 : 0;  // frac1 side of an intersection: -c, -q
      h.qk = 0.0;
      h.pad2 = 0.0;
      if (h.type == 0 || h.type == 3 || h.type == 5) {
        const cd *ep = h.pad ? net.ep1 + 2 * el : net.ep0 + 2 * el;
        cd a = ep[0], b = ep[1];
        cd inv = recip(b - a);
        h.p0 = 2.0 * inv;
        cd ab = a + b;
        h.p1 = mk(-(ab.re * inv.re - ab.im * inv.im), -(ab.re * inv.im + ab.im * inv.re));
      } else {
        h.p0 = (h.type == 1) ? mk(0.0, 0.0) : net.center[el];
        h.p1 = mk(1.0 / net.radius[el], 0.0);
      }
      src[s] = h;
      sq[s] = 0.0;
    }
    for (int idx = threadIdx.x; idx < cnt * MC; idx += blockDim.x) sacc[idx] = mk(0.0, 0.0);
    __syncthreads();
    for (int s = 0; s < cnt; s++) {
      const Src h = src[s];
      const double sg = h.pad ? -1.0 : 1.0;
      cd rt[P], pw[P];
      double wv[P];
      double qc = 0.0;
#pragma unroll
      for (int i = 0; i < P; i++) {
        rt[i] = mk(0.0, 0.0);
        pw[i] = mk(1.0, 0.0);
        wv[i] = 0.0;
        if (w[i] == 0.0 || h.id == excl[i]) continue;
        cd chi;
        if (h.type == 0 || h.type == 3 || h.type == 5) {
          chi = exterior_chi(fma_c(h.p0, z[i], h.p1));
          rt[i] = recip(chi);
        } else if (h.type == 1) {
          chi = h.p1.re * z[i];
          rt[i] = chi;
        } else {
          chi = h.p1.re * (z[i] - h.p0);
          if (h.type == 4) rt[i] = recip(chi);
        }
        wv[i] = w[i] * sg;
        if (h.type == 0 || h.type == 2 || h.type == 3) {
          const double lg = (kind[i] == KIND_PSI) ? atan2(chi.im, chi.re) : 0.5 * log(norm2(chi));
          qc += wv[i] / (2 * PI) * lg;
        }
      }
      if (h.type == 0 || h.type == 2 || h.type == 3) {
        qc = warp_sum(qc);
        if (lane == 0) atomicAdd(&sq[s], qc);
      }
      if (h.m == 0) continue;
      for (int j = 0; j < h.m; j++) {
        double ar = 0.0, ai = 0.0;
#pragma unroll
        for (int i = 0; i < P; i++) {
          // d(value)/d(Re c_j, Im c_j) = conj(x^j) (phi) or i conj(x^j) (psi), x^j = pw
          const double cr = wv[i] * pw[i].re, ci = wv[i] * pw[i].im;
          if (kind[i] == KIND_PSI) {
            ar += ci;
            ai += cr;
          } else {
            ar += cr;
            ai -= ci;
          }
          pw[i] = mk(pw[i].re * rt[i].re - pw[i].im * rt[i].im, pw[i].re * rt[i].im + pw[i].im * rt[i].re);
        }
        red_re[j * ADJ_RED_STRIDE + lane] = ar;
        red_im[j * ADJ_RED_STRIDE + lane] = ai;
      }
      __syncwarp();
      for (int j = lane; j < h.m; j += 32) {
        double sr = 0.0, si = 0.0;
        for (int l = 0; l < 32; l++) {
          sr += red_re[j * ADJ_RED_STRIDE + l];
          si += red_im[j * ADJ_RED_STRIDE + l];
        }
        atomicAdd(&sacc[s * MC + j].re, sr);
        atomicAdd(&sacc[s * MC + j].im, si);
      }
      __syncwarp();
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < cnt * MC; idx += blockDim.x) {
      const int s = idx / MC, j = idx - s * MC;
      if (j >= src[s].m) continue;
      const cd v = sacc[idx];
      cd *g = gc + (size_t)src[s].id * MC + j;
      atomicAdd(&g->re, v.re);
      atomicAdd(&g->im, v.im);
    }
    for (int s = threadIdx.x; s < cnt; s += blockDim.x)
      if (sq[s] != 0.0) atomicAdd(&gq[src[s].id], sq[s]);
  }
  cw = warp_sum(cw);
  if (lane == 0) s_cw[warp] = cw;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < EVAL_THREADS / 32; k++) t += s_cw[k];
    if (t != 0.0) atomicAdd(&gC[f], t);
  }
}

__global__ void __launch_bounds__(EVAL_THREADS) adj_sweep_kernel(Net net, const Item *__restrict__ items,
                                                                   const int2 *__restrict__ pts,
                                                                   const Group *__restrict__ groups,
                                                                   const double *__restrict__ wsw, cd *gc, double *gq,
                                                                   double *gC, int chunk, const AdjState *as) {
  if (as->s.done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Item it = items[blockIdx.x];
  if (it.pad == 1)
    adj_sweep_body<1>(net, it, pts, groups, wsw, gc, gq, gC, chunk, smem_raw);
  else if (it.pad == 2)
    adj_sweep_body<2>(net, it, pts, groups, wsw, gc, gq, gC, chunk, smem_raw);
  else
    adj_sweep_body<4>(net, it, pts, groups, wsw, gc, gq, gC, chunk, smem_raw);
}

// The sweep evaluation transposed, from the forward sweep's pair tables
// (pair_table_kernel): for every source s of fracture f and every weighted
// collocation point p of f,
//   d/d(Re c_sj, Im c_sj) += w_p sg (Re x^j, -Im x^j)   (phi point)
//                         or w_p sg (Im x^j,  Re x^j)   (psi point)
//   d/dq_s += w_p sg l / (2 pi)                         (discharge types)
// with x, l the pair's table entries.  One item is up to ADJ_TAB_PTS points
// of one fracture; each warp takes sources round-robin, its lanes split the
// points, keep the MM coefficient sums of the source in registers and reduce
// them over the warp once per source (no shared-memory reduction tables).
static constexpr int ADJ_TAB_PTS = 256;
template <int MM>
__global__ void __launch_bounds__(EVAL_THREADS) adj_sweep_table_kernel(
    Net net, const Item *__restrict__ items, const int2 *__restrict__ pts, const Group *__restrict__ groups,
    const int *__restrict__ fpt0, const int *__restrict__ fnp, const long long *__restrict__ tab_off,
    const cd *__restrict__ tw, const double *__restrict__ tl, const double *__restrict__ wsw, cd *gc, double *gq,
    double *gC, const AdjState *as) {
  if (as->s.done) return;
  __shared__ double s_w[ADJ_TAB_PTS];
  __shared__ int s_ex[ADJ_TAB_PTS];
  __shared__ int s_psi[ADJ_TAB_PTS];
  __shared__ double s_cw[EVAL_THREADS / 32];
  const Item it = items[blockIdx.x];
  const int f = it.frac;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int npt = it.p1 - it.p0;
  double cw = 0.0;
  for (int i = threadIdx.x; i < ADJ_TAB_PTS; i += EVAL_THREADS) {
    double w = 0.0;
    int ex = -1, psi = 0;
    if (i < npt) {
      const int2 gk = pts[it.p0 + i];
      const Group g = groups[gk.x];
      w = wsw[g.out + gk.y];
      ex = g.elem;
      psi = (g.kind == KIND_PSI) ? 1 : 0;
      if (!psi) cw += w;
    }
    s_w[i] = w;
    s_ex[i] = ex;
    s_psi[i] = psi;
  }
  cw = warp_sum(cw);
  if (lane == 0) s_cw[warp] = cw;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < EVAL_THREADS / 32; k++) t += s_cw[k];
    if (t != 0.0) atomicAdd(&gC[f], t);
  }
  const int np = fnp[f];
  const long long base = tab_off[f] + (it.p0 - fpt0[f]);
  const int e0 = net.fptr[f], nsrc = net.fptr[f + 1] - e0;
  const int MC = net.MC;
  for (int s = warp; s < nsrc; s += EVAL_THREADS / 32) {
    const int el = net.felem[e0 + s];
    const int type = net.type[el];
    const int m = net.ncoef[el];
    const double sg = (type == 0 && net.frac0[el] != f) ? -1.0 : 1.0;
    const bool disch = (type == 0 || type == 2 || type == 3);
    const cd *__restrict__ xs = tw + base + (long long)s * np;
    const double *__restrict__ ls = tl + base + (long long)s * np;
    double ar[MM], ai[MM];
#pragma unroll
    for (int j = 0; j < MM; j++) ar[j] = ai[j] = 0.0;
    double qc = 0.0;
    for (int i = lane; i < npt; i += 32) {
      const double w = s_w[i];
      if (w == 0.0 || s_ex[i] == el) continue;
      const cd x = ldcs_cd(xs + i);
      const double wv = w * sg;
      if (disch) qc += wv / (2 * PI) * __ldcs(ls + i);
      const bool psi = s_psi[i] != 0;
      cd pw = mk(1.0, 0.0);
#pragma unroll
      for (int j = 0; j < MM; j++) {
        if (j < m) {
          const double cr = wv * pw.re, ci = wv * pw.im;
          ar[j] += psi ? ci : cr;
          ai[j] += psi ? cr : -ci;
          pw = mk(pw.re * x.re - pw.im * x.im, pw.re * x.im + pw.im * x.re);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < MM; j++) {
      if (j < m) {
        const double r = warp_sum(ar[j]), im = warp_sum(ai[j]);
        if (lane == 0 && (r != 0.0 || im != 0.0)) {
          atomicAdd(&gc[(size_t)el * MC + j].re, r);
          atomicAdd(&gc[(size_t)el * MC + j].im, im);
        }
      }
    }
    if (disch) {
      qc = warp_sum(qc);
      if (lane == 0 && qc != 0.0) atomicAdd(&gq[el], qc);
    }
  }
}

// The head-vector evaluation transposed.  Its points carry one weight per
// discharge row and side (mu of the row times -1/(D t0), +1/(D t1) for the
// sides of an intersection, -1/D for a constant-head line or well), so the
// sums over a side's D points of the series terms depend on the geometry
// only: rhs_sums_kernel computes them once, S[pair][j] = sign * sum_k x_k^j
// for every (row side, source element of that side's fracture) pair (one warp
// per pair), and each iteration gathers gc[s][j] += sum over the pairs of s of
// weight * conj(S[pair][j]) (one thread per source coefficient).
// The coefficient index (source * MC + power) of every power-sum entry: a
// warp per (row side, source) pair, whose entries are consecutive from its
// offset to the next pair's.
__global__ void hs_index_kernel(const int *__restrict__ pair_src, const int *__restrict__ pair_off, int npairs,
                                int total, int MC, int *__restrict__ sidx) {
  const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (p >= npairs) return;
  const int o0 = pair_off[p], o1 = (p + 1 < npairs) ? pair_off[p + 1] : total;
  const int base = pair_src[p] * MC;
  for (int k = lane; k < o1 - o0; k += 32) sidx[o0 + k] = base + k;
}

__global__ void rhs_sums_kernel(Net net, const int *__restrict__ pair_g, const int *__restrict__ pair_src,
                                const int *__restrict__ pair_off, int npairs, cd *S) {
  const int pr = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (pr >= npairs) return;
  const int g = pair_g[pr], el = pair_src[pr];
  const int j = g >> 1, side = g & 1;
  const int e = net.de_ids[j];
  const int f = side ? net.frac1[e] : net.frac0[e];
  const cd *zp = (side ? net.zint1 : net.zint0) + (size_t)j * net.D;
  const int type = net.type[el], m = net.ncoef[el];
  const bool neg = (type == 0 && net.frac0[el] != f);
  const double sg = neg ? -1.0 : 1.0;
  cd p0, p1;
  if (type == 0 || type == 3 || type == 5) {
    const cd *ep = neg ? net.ep1 + 2 * el : net.ep0 + 2 * el;
    cd inv = recip(ep[1] - ep[0]);
    cd ab = ep[0] + ep[1];
    p0 = 2.0 * inv;
    p1 = mk(-(ab.re * inv.re - ab.im * inv.im), -(ab.re * inv.im + ab.im * inv.re));
  } else {
    p0 = (type == 1) ? mk(0.0, 0.0) : net.center[el];
    p1 = mk(1.0 / net.radius[el], 0.0);
  }
  cd *out = S + pair_off[pr];
  // lanes take points k, k + 32, ... (KP per pass); powers advance per coefficient
  constexpr int KP = 4;
  for (int k0 = 0; k0 < net.D; k0 += 32 * KP) {
    cd pw[KP], rt[KP];
#pragma unroll
    for (int i = 0; i < KP; i++) {
      const int k = k0 + lane + 32 * i;
      pw[i] = mk(0.0, 0.0);
      rt[i] = mk(0.0, 0.0);
      if (k < net.D) {
        const cd zz = zp[k];
        cd chi;
        if (type == 0 || type == 3 || type == 5) {
          chi = exterior_chi(fma_c(p0, zz, p1));
          rt[i] = recip(chi);
        } else if (type == 1) {
          chi = p1.re * zz;
          rt[i] = chi;
        } else {
          chi = p1.re * (zz - p0);
          rt[i] = recip(chi);
        }
        pw[i] = mk(sg, 0.0);
      }
    }
    for (int jj = 0; jj < m; jj++) {
      double ar = 0.0, ai = 0.0;
#pragma unroll
      for (int i = 0; i < KP; i++) {
        ar += pw[i].re;
        ai += pw[i].im;
        pw[i] = mk(pw[i].re * rt[i].re - pw[i].im * rt[i].im, pw[i].re * rt[i].im + pw[i].im * rt[i].re);
      }
      ar = warp_sum(ar);
      ai = warp_sum(ai);
      if (lane == 0) out[jj] = (k0 == 0) ? mk(ar, ai) : mk(out[jj].re + ar, out[jj].im + ai);
    }
  }
}

// Head vector from the power sums (replaces the evaluation of the head-vector
// points): one warp per system row, b = (S1 / D) / t1 - (S0 / D) / t0 for an
// intersection, phi - S0 / D for a constant-head line or well, 0 for a
// continuity row, with S_side = sum over the side's pairs of Re(coef * S).
// The head vector, a group of T threads per system row (RPB rows per CTA):
// the row side's power-sum entries are split over the group's threads (four
// index -> coefficient chains in flight per thread) and summed with a
// fixed-order tree, so the result does not depend on timing.  Long rows
// (one network: ~380 entries on average, 1,700 at most) take a 128-thread
// CTA each, so they no longer sit on one warp's dependent loads; short rows
// (batches of small realizations) a warp each, four to a CTA.
template <int T>
__device__ __forceinline__ double hv_group_sum(double v, double *red) {
  v = warp_sum(v);
  if (T == 32) return v;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();  // red is free (a previous sum's readers are done)
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < T / 32; w++) t += red[w];
  return t;
}
// One row group (a warp for T = 32, the CTA otherwise) per row; with an
// active list (batches) the groups walk the list's rows (grid-stride; the
// list's length on the device), else one row each.
template <int T>
__device__ __forceinline__ void head_row(const Net &net, int g, int t, const int *__restrict__ gptr,
                                         const int *__restrict__ sidx, const cd *__restrict__ S, double *red) {
  const SolveState *st = net.st + net.real_row[g];
  if (st->done || !st->solve_q) return;  // uniform over the row's group
  const int r = net.row_de[g];
  if (r < 0) {
    if (t == 0) net.bvec[g] = net.bknown ? net.bknown[g] : 0.0;
    return;
  }
  const int e = net.de_ids[r];
  double sum[2] = {0.0, 0.0};
  const int sides = (net.type[e] == 0) ? 2 : 1;
  for (int sd = 0; sd < sides; sd++) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    const int x1 = gptr[2 * r + sd + 1];
    int x = gptr[2 * r + sd] + t;
    for (; x + 3 * T < x1; x += 4 * T) {  // four index -> coefficient chains in flight
      const int i0 = sidx[x], i1 = sidx[x + T], i2 = sidx[x + 2 * T], i3 = sidx[x + 3 * T];
      const cd v0 = S[x], v1 = S[x + T], v2 = S[x + 2 * T], v3 = S[x + 3 * T];
      const cd c0 = net.coef[i0], c1 = net.coef[i1], c2 = net.coef[i2], c3 = net.coef[i3];
      a0 = fma(c0.re, v0.re, fma(-c0.im, v0.im, a0));
      a1 = fma(c1.re, v1.re, fma(-c1.im, v1.im, a1));
      a2 = fma(c2.re, v2.re, fma(-c2.im, v2.im, a2));
      a3 = fma(c3.re, v3.re, fma(-c3.im, v3.im, a3));
    }
    for (; x < x1; x += T) {
      const cd c = net.coef[sidx[x]], v = S[x];
      a0 = fma(c.re, v.re, fma(-c.im, v.im, a0));
    }
    sum[sd] = hv_group_sum<T>((a0 + a1) + (a2 + a3), red);
  }
  if (t == 0) {
    const double D = net.D;
    double b;
    if (sides == 2)
      b = (sum[1] / D) / net.t[net.frac1[e]] - (sum[0] / D) / net.t[net.frac0[e]];
    else
      b = net.phi[e] - sum[0] / D;
    net.bvec[g] = net.bknown ? b + net.bknown[g] : b;
  }
}

template <int T, int RPB>
__global__ void __launch_bounds__(T * RPB) head_vector_kernel(Net net, const int *__restrict__ gptr,
                                                               const int *__restrict__ sidx,
                                                               const cd *__restrict__ S,
                                                               const int *__restrict__ alist,
                                                               const int *__restrict__ acount) {
  __shared__ double red[T / 32 > 0 ? T / 32 : 1];
  const int t = (T == 32) ? (threadIdx.x & 31) : threadIdx.x;
  const int g0 = blockIdx.x * RPB + ((T == 32) ? (threadIdx.x >> 5) : 0);
  // a batch's rows of running realizations, or every row
  const int n = alist ? *acount : net.N;
  for (int v = g0; v < n; v += gridDim.x * RPB) head_row<T>(net, alist ? alist[v] : v, t, gptr, sidx, S, red);
}

__global__ void adj_rhs_gather_kernel(Net net, const int *__restrict__ src_ptr, const int *__restrict__ src_pairs,
                                      const int *__restrict__ pair_g, const int *__restrict__ pair_off,
                                      const cd *__restrict__ S, const double *__restrict__ mu,
                                      const double *__restrict__ fac, cd *gc, const AdjState *as) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (as->s.done || i >= (long long)net.ne * net.MC) return;
  const int el = (int)(i / net.MC), j = (int)(i - (long long)el * net.MC);
  if (j >= net.ncoef[el]) return;
  // weight * conj(S) per pair: the derivative of a phi value; four pair
  // chains (pair -> row side, offset -> weight, S) in flight
  double ar[4] = {0.0, 0.0, 0.0, 0.0}, ai[4] = {0.0, 0.0, 0.0, 0.0};
  const int k1 = src_ptr[el + 1];
  int k = src_ptr[el];
  for (; k + 3 < k1; k += 4) {
    int pr[4], g[4], off[4];
#pragma unroll
    for (int u = 0; u < 4; u++) pr[u] = src_pairs[k + u];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      g[u] = pair_g[pr[u]];
      off[u] = pair_off[pr[u]];
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const double wg = mu[g[u] >> 1] * fac[g[u]];
      const cd v = S[off[u] + j];
      ar[u] += wg * v.re;
      ai[u] -= wg * v.im;
    }
  }
  for (; k < k1; k++) {
    const int pr = src_pairs[k];
    const int g = pair_g[pr];
    const double wg = mu[g >> 1] * fac[g];
    const cd v = S[pair_off[pr] + j];
    ar[0] += wg * v.re;
    ai[0] -= wg * v.im;
  }
  gc[i].re += (ar[0] + ar[1]) + (ar[2] + ar[3]);
  gc[i].im += (ai[0] + ai[1]) + (ai[2] + ai[3]);
}

// Right-hand side of the transposed discharge solve: dJ/dd + Phi_d^T lam.
__global__ void adj_rhs_kernel(Net net, const double *gd, const double *gq, const double *gC, double *b,
                               const AdjState *as) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (as->s.done || g >= net.N) return;
  const int d = net.row_de[g];
  b[g] = gd[g] + (d >= 0 ? gq[net.de_ids[d]] : gC[net.row_frac[g]]);
}

// dJ/dd in system-row order from the caller's dJ/dq and dJ/dC.
__global__ void adj_gd_kernel(Net net, const double *gq_user, const double *gC_user, double *gd) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= net.N) return;
  const int d = net.row_de[g];
  gd[g] = d >= 0 ? gq_user[net.de_ids[d]] : gC_user[net.row_frac[g]];
}

// The multiplier components the update can change: every coefficient below
// ncoef, except the imaginary parts of intersections and constant-head lines
// (real coefficients), the real parts of impermeable lines and c_0 of all
// types but bounding circles (fixed at 0); wells have none.
__device__ __forceinline__ cd adj_mask(const Net &net, int e, int j, cd v) {
  const int type = net.type[e];
  if (type == 2 || j >= net.ncoef[e] || (j == 0 && type != 1)) return mk(0.0, 0.0);
  if (type == 0 || type == 3) v.im = 0.0;
  if (type == 5) v.re = 0.0;
  return v;
}

// With gc = Phi_c^T x + b_c^T mu(x) from one transposed sweep at lam = x:
//   mode 0 (sweep with dJ/dd = 0):    y = mask(x - gc)          = (I - T^T) x
//   mode 1 (sweep with the real dJ/dd): y = mask(dJ/dc + gc) - x = F(x) - x,
// the residual of the multiplier equation lam = F(lam) (the right-hand side
// when x = 0).
__global__ void adj_combine_kernel(Net net, const cd *x, const cd *gc, const cd *gobj, cd *y, int mode) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)net.ne * net.MC) return;
  const int e = (int)(i / net.MC), j = (int)(i - (long long)e * net.MC);
  const cd xv = x[i], g = gc[i];
  if (mode == 0) {
    y[i] = adj_mask(net, e, j, mk(xv.re - g.re, xv.im - g.im));
  } else {
    const cd f = adj_mask(net, e, j, mk(gobj[i].re + g.re, gobj[i].im + g.im));
    y[i] = mk(f.re - xv.re, f.im - xv.im);
  }
}

// Dense vector kernels of the Krylov solve (vectors of n doubles, a basis of
// nv vectors at stride `stride`): h[i] += V_i . w, w += sign sum_i h[i] V_i,
// out = a w.
__global__ void vec_mdot_kernel(const double *__restrict__ V, long long stride, int nv, const double *__restrict__ w,
                                long long n, double *h) {
  __shared__ double red[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = 0; i < nv; i++) {
    const double *v = V + (size_t)i * stride;
    double acc = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
      acc = fma(v[k], w[k], acc);
    acc = warp_sum(acc);
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += red[k];
      atomicAdd(&h[i], t);
    }
    __syncthreads();
  }
}

__global__ void vec_update_kernel(double *w, const double *__restrict__ V, long long stride, int nv,
                                  const double *__restrict__ h, double sign, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int i = 0; i < nv; i++) acc = fma(h[i], V[(size_t)i * stride + k], acc);
    w[k] = fma(sign, acc, w[k]);
  }
}

__global__ void vec_scale_kernel(const double *w, double *out, double a, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    out[k] = a * w[k];
}

// ---------------------------------------------------------------------------
// GMRES cycle state on the device.  One Arnoldi step (basis copy, transposed
// sweep, two classical Gram-Schmidt passes, norm, Givens update, scaling) is
// one captured graph whose kernels read the step index j and the stop flag
// from here, so the host launches several steps between synchronisations;
// the steps after a stop return at entry (the sweep's kernels through the
// adjoint state's done flag, which the Givens kernel sets with stop).

// Start of a cycle: V_0 = r / beta was written by the host; j = 0.
__global__ void gm_reset_kernel(GmresDev *g, AdjState *as, double beta, double bnorm, double tol,
                                long long matvecs, long long max_it) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  g->j = 0;
  g->stop = 0;
  g->k = 0;
  g->nonfinite = 0;
  g->matvecs = matvecs;
  g->max_it = max_it;
  g->bnorm = bnorm;
  g->tol = tol;
  g->rel = beta / bnorm;
  g->scale = 0.0;
  for (int i = 0; i <= GM_MK; i++) g->gv[i] = 0.0;
  g->gv[0] = beta;
  as->s.done = 0;
}

// xin = V_j
__global__ void gm_copy_kernel(const GmresDev *g, const double *__restrict__ V, double *__restrict__ xin, long long n) {
  if (g->stop) return;
  const double *v = V + (size_t)g->j * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    xin[k] = v[k];
}

// h[i] += <V_i, w> for i <= j (nv1: one vector only, V itself); eight
// basis vectors per pass over w, their block sums reduced together.
static constexpr int GM_GROUP = 8;
__global__ void gm_mdot_kernel(const GmresDev *g, const double *__restrict__ V, long long stride, int nv1,
                               const double *__restrict__ w, long long n, double *h) {
  if (g->stop) return;
  __shared__ double red[GM_GROUP][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int nv = nv1 ? 1 : g->j + 1;
  for (int i0 = 0; i0 < nv; i0 += GM_GROUP) {
    double acc[GM_GROUP];
#pragma unroll
    for (int u = 0; u < GM_GROUP; u++) acc[u] = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
      const double wk = w[k];
#pragma unroll
      for (int u = 0; u < GM_GROUP; u++)
        if (i0 + u < nv) acc[u] = fma(V[(size_t)(i0 + u) * stride + k], wk, acc[u]);
    }
#pragma unroll
    for (int u = 0; u < GM_GROUP; u++) {
      const double a = warp_sum(acc[u]);
      if (lane == 0) red[u][warp] = a;
    }
    __syncthreads();
    if (threadIdx.x < GM_GROUP && i0 + (int)threadIdx.x < nv) {
      double t = 0.0;
      for (int k = 0; k < nwarp; k++) t += red[threadIdx.x][k];
      atomicAdd(&h[i0 + threadIdx.x], t);
    }
    __syncthreads();
  }
}

// w -= sum_{i <= j} h[i] V_i
__global__ void gm_update_kernel(const GmresDev *g, double *w, const double *__restrict__ V, long long stride,
                                 const double *__restrict__ h, long long n) {
  if (g->stop) return;
  const int nv = g->j + 1;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int i = 0; i < nv; i++) acc = fma(h[i], V[(size_t)i * stride + k], acc);
    w[k] -= acc;
  }
}

// Hessenberg column j from the two Gram-Schmidt passes (hd[0..], hd[GM_MK + 2 ..])
// and |w|^2 (hd[2 GM_MK + 3]), the previous rotations, a new one zeroing
// H(j+1, j), the residual estimate, and the decision to stop the cycle.
__global__ void gm_givens_kernel(GmresDev *g, const double *hd, AdjState *as) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || g->stop) return;
  const int j = g->j;
  g->matvecs += 1;
  const double hn = sqrt(hd[2 * (GM_MK + 2) - 1]);
  double *Hm = g->Hm;
  for (int i = 0; i <= j; i++) Hm[i * GM_MK + j] = hd[i] + hd[GM_MK + 2 + i];
  Hm[(j + 1) * GM_MK + j] = hn;
  for (int i = 0; i < j; i++) {
    const double a = Hm[i * GM_MK + j], b = Hm[(i + 1) * GM_MK + j];
    Hm[i * GM_MK + j] = g->cs[i] * a + g->sn[i] * b;
    Hm[(i + 1) * GM_MK + j] = -g->sn[i] * a + g->cs[i] * b;
  }
  const double a = Hm[j * GM_MK + j], b = hn;
  const double r = hypot(a, b);
  g->cs[j] = r > 0 ? a / r : 1.0;
  g->sn[j] = r > 0 ? b / r : 0.0;
  Hm[j * GM_MK + j] = r;
  Hm[(j + 1) * GM_MK + j] = 0.0;
  g->gv[j + 1] = -g->sn[j] * g->gv[j];
  g->gv[j] = g->cs[j] * g->gv[j];
  g->k = j + 1;
  const bool bad = !isfinite(hn) || !isfinite(g->gv[j + 1]);
  g->rel = fabs(g->gv[j + 1]) / g->bnorm;
  g->scale = hn > 0.0 ? 1.0 / hn : 0.0;
  if (bad || g->rel <= g->tol || g->matvecs >= g->max_it || hn == 0.0 || j + 1 == GM_MK) {
    g->nonfinite = bad ? 1 : 0;
    g->stop = 1;
    as->s.done = 1;
  } else {
    g->j = j + 1;
  }
}

// V_{j+1} = w / |w| (j already advanced)
__global__ void gm_scale_kernel(const GmresDev *g, const double *__restrict__ w, double *V, long long n) {
  if (g->stop) return;
  double *v = V + (size_t)g->j * n;
  const double a = g->scale;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    v[k] = a * w[k];
}

// lam^T Phi_theta: for every intersection, sum_j>=1 lam_j.re (Re a0_j + Re a1_j)
// times t0 t1 / (t0 + t1)^2, added to theta of frac0 and subtracted from
// theta of frac1 (a0, a1: the DFTs of the two sides' values at convergence).
__global__ void adj_theta_kernel(Net net, const cd *lam, const int *group_of, const Group *groups,
                                 const double *sweep_vals, double *gtheta) {
  const int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (e >= net.ne || net.type[e] != 0) return;
  const int n = net.nint[e], m = net.ncoef[e];
  const double *v0 = sweep_vals + groups[group_of[2 * e]].out;
  const double *v1 = sweep_vals + groups[group_of[2 * e + 1]].out;
  double s = 0.0;
  for (int j = 1 + lane; j < m; j += 32) {
    cd a0, a1;
    dft_lane(v0, n, 0, j, false, a0);
    dft_lane(v1, n, 0, j, false, a1);
    s += lam[(size_t)e * net.MC + j].re * (a0.re + a1.re);
  }
  s = warp_sum(s);
  if (lane == 0) {
    const int f0 = net.frac0[e], f1 = net.frac1[e];
    const double t0 = net.t[f0], t1 = net.t[f1];
    const double K = t0 * t1 / ((t0 + t1) * (t0 + t1));
    atomicAdd(&gtheta[f0], s * K);
    atomicAdd(&gtheta[f1], -s * K);
  }
}

// Mean of Re Omega over the D points of each side of each discharge element.
__global__ void adj_obar_kernel(Net net, double *obar) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= 2 * net.n_de) return;
  const int j = w >> 1, side = w & 1;
  const int e = net.de_ids[j];
  if (side && net.type[e] != 0) {
    if (lane == 0) obar[w] = 0.0;
    return;
  }
  const int f = side ? net.frac1[e] : net.frac0[e];
  const cd *z = (side ? net.zint1 : net.zint0) + (size_t)j * net.D;
  double s = 0.0;
  for (int k = lane; k < net.D; k += 32) s += omega_at(net, f, z[k]).re;
  s = warp_sum(s);
  if (lane == 0) obar[w] = s / net.D;
}

// Heads Re Omega_f(z) / t_f at device-resident points.
__global__ void heads_dev_kernel(Net net, const int64_t *__restrict__ frac, const cd *__restrict__ z, int n,
                                 double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int f = (int)frac[i];
  out[i] = omega_at(net, f, z[i]).re / net.t[f];
}

// Vector-Jacobian product of heads_dev_kernel: given dJ/dh per point, adds
// dJ/d(coef) ([ne][mco] complex pairs), dJ/dq, dJ/dC and the explicit
// dJ/dlog t (h = Re Omega / t, so dh/dlog t = -h) of the current state.
__global__ void heads_vjp_kernel(Net net, const int64_t *__restrict__ frac, const cd *__restrict__ z, int n,
                                 const double *__restrict__ gh, double *gcoef, int mco, double *gq, double *gC,
                                 double *glogt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double g = gh[i];
  if (g == 0.0) return;
  const int f = (int)frac[i];
  const cd zz = z[i];
  const double t = net.t[f];
  const double w = g / t;
  const double h = omega_at(net, f, zz).re / t;
  if (!(h == h)) return;
  atomicAdd(&glogt[f], -g * h);
  atomicAdd(&gC[f], w);
  for (int k = net.fptr[f]; k < net.fptr[f + 1]; k++) {
    const int el = net.felem[k];
    const int ty = net.type[el];
    const int m = min(net.ncoef[el], mco);
    const bool neg = (ty == 0 && net.frac0[el] != f);
    const double sg = neg ? -1.0 : 1.0;
    cd chi, rt = mk(0.0, 0.0);
    if (ty == 0 || ty == 3 || ty == 5) {
      const cd *ep = neg ? net.ep1 + 2 * el : net.ep0 + 2 * el;
      cd inv = recip(ep[1] - ep[0]);
      cd ab = ep[0] + ep[1];
      chi = exterior_chi(
          fma_c(2.0 * inv, zz, mk(-(ab.re * inv.re - ab.im * inv.im), -(ab.re * inv.im + ab.im * inv.re))));
      rt = recip(chi);
    } else if (ty == 1) {
      chi = (1.0 / net.radius[el]) * zz;
      rt = chi;
    } else {
      chi = (1.0 / net.radius[el]) * (zz - net.center[el]);
      if (ty == 4) rt = recip(chi);
    }
    if (ty == 0 || ty == 2 || ty == 3) atomicAdd(&gq[el], w * sg / (2 * PI) * (0.5 * log(norm2(chi))));
    cd pw = mk(1.0, 0.0);
    for (int j = 0; j < m; j++) {
      double *gp = gcoef + 2 * ((size_t)el * mco + j);
      atomicAdd(gp, w * sg * pw.re);
      atomicAdd(gp + 1, -w * sg * pw.im);
      pw = mk(pw.re * rt.re - pw.im * rt.im, pw.re * rt.im + pw.im * rt.re);
    }
  }
}

}  // namespace andfn

namespace andfn {

// Point tables of the transposed evaluation: the forward point lists (same
// order), cut into items of at most ADJ_ITEM points of one fracture.
static void adj_items(const std::vector<Group> &groups, const std::vector<int2> &pts, std::vector<Item> &items) {
  items.clear();
  size_t p = 0;
  while (p < pts.size()) {
    const int f = groups[pts[p].x].frac;
    size_t q = p;
    while (q < pts.size() && groups[pts[q].x].frac == f) q++;
    for (size_t a = p; a < q; a += ADJ_ITEM) {
      Item it;
      it.frac = f;
      it.p0 = (int)a;
      it.p1 = (int)std::min(q, a + ADJ_ITEM);
      const int np = it.p1 - it.p0;
      it.pad = np <= EVAL_THREADS ? 1 : (np <= 2 * EVAL_THREADS ? 2 : 4);  // points per thread
      items.push_back(it);
    }
    p = q;
  }
}

// Builds the head-vector power sums for the current ncoef (once per handle;
// again only if ncoef or the coefficient capacity changed).  Needs z_int.
static int build_head_sums(AndfnHandle *H) {
  HeadSums &hs = H->hs;
  if (hs.valid && hs.ncoef == H->cur_ncoef && hs.mc == H->MC) return 0;
  const HostNet &h = H->h;
  const int ne = (int)H->ne, n_de = (int)h.de_ids.size(), MC = H->MC;
  cudaStream_t s = H->stream;
  // pairs (row side, source element) in row order; the power-sum entries
  // of a pair are consecutive (offset po, ncoef of the source entries), and
  // the coefficient index of each entry is written on the device
  std::vector<int> pg, ps, po, gptr(2 * (size_t)n_de + 1, 0);
  std::vector<int> sp(ne + 1, 0);
  int off = 0;
  for (int j = 0; j < n_de; j++) {
    const int e = h.de_ids[j];
    const int sides = (h.type[e] == 0) ? 2 : 1;
    for (int sd = 0; sd < 2; sd++) {
      gptr[2 * j + sd] = off;
      if (sd >= sides) continue;
      const int f = sd ? h.frac1[e] : h.frac0[e];
      for (int k = h.fptr[f]; k < h.fptr[f + 1]; k++) {
        const int el = h.felem[k];
        const int m = H->cur_ncoef[el];
        if (h.type[el] == 2 || m <= 0) continue;
        sp[el + 1]++;
        pg.push_back(2 * j + sd);
        ps.push_back(el);
        po.push_back(off);
        off += m;
      }
    }
  }
  gptr[2 * (size_t)n_de] = off;
  // the pairs of each source element, in pair order (counting sort)
  for (int el = 0; el < ne; el++) sp[el + 1] += sp[el];
  std::vector<int> spairs(pg.size()), fillp(sp.begin(), sp.end() - 1);
  for (int p = 0; p < (int)ps.size(); p++) spairs[fillp[ps[p]]++] = p;
  hs.npairs = (int)pg.size();
  hs.long_rows = off > 256LL * std::max(1, H->N);
  CK(upload(hs.gptr, gptr, s));
  if (hs.npairs > 0) {
    CK(upload(hs.pair_g, pg, s));
    CK(upload(hs.pair_src, ps, s));
    CK(upload(hs.pair_off, po, s));
    CK(upload(hs.src_ptr, sp, s));
    CK(upload(hs.src_pairs, spairs, s));
    CK(hs.sidx.alloc(std::max(1, off)));
    hs_index_kernel<<<(hs.npairs * 32 + 127) / 128, 128, 0, s>>>(hs.pair_src.p, hs.pair_off.p, hs.npairs, off, MC,
                                                                  hs.sidx.p);
    CK(hs.S.alloc(std::max(1, off)));
    rhs_sums_kernel<<<(hs.npairs * 32 + 127) / 128, 128, 0, s>>>(H->net(), hs.pair_g.p, hs.pair_src.p,
                                                                  hs.pair_off.p, hs.npairs, hs.S.p);
    CK(cudaGetLastError());
  }
  hs.ncoef = H->cur_ncoef;
  hs.mc = MC;
  hs.valid = true;
  return 0;
}

// Transposed factors of the last run's LU (P A Q = L U, so A^T = Q U^T L^T P):
// the lower solve is U^T (rows scaled by 1/U(i,i)), the upper one L^T (unit);
// the dense tail's lower part is (D^-1 U22)^T followed by D^-1, its upper
// part L22^T; y = Q^T b on entry, x = P^T y on exit.
static int adj_build_factors(AndfnHandle *H) {
  AdjBufs &A = *H->adj;
  const LuFactors &F = H->lu_keep;
  const int n = F.n, K = F.dense, m0 = n - K;
  cudaStream_t s = H->stream;
  auto transpose = [n](const std::vector<int> &ptr, const std::vector<int> &col, const std::vector<double> &val,
                       std::vector<int> &tp, std::vector<int> &tc, std::vector<double> &tv) {
    tp.assign(n + 1, 0);
    for (int c : col) tp[c + 1]++;
    for (int i = 0; i < n; i++) tp[i + 1] += tp[i];
    tc.resize(col.size());
    tv.resize(col.size());
    std::vector<int> fill(tp.begin(), tp.end() - 1);
    for (int r = 0; r < n; r++)
      for (int p = ptr[r]; p < ptr[r + 1]; p++) {
        const int c = col[p];
        tc[fill[c]] = r;
        tv[fill[c]++] = val[p];
      }
  };
  std::vector<int> ut_p, ut_c, lt_p, lt_c;
  std::vector<double> ut_v, lt_v;
  transpose(F.u_ptr, F.u_col, F.u_val, ut_p, ut_c, ut_v);  // U^T: strictly lower
  transpose(F.l_ptr, F.l_col, F.l_val, lt_p, lt_c, lt_v);  // L^T: strictly upper
  TriDesc td;
  std::memset(&td, 0, sizeof(td));
  LevelSolve *ls[4] = {&td.Lf, &td.Lx, &td.Ux, &td.Ub};
  A.max_nlev = 1;
  for (int k = 0; k < 4; k++) {
    std::vector<int> lev, rows, eptr, ecol;
    std::vector<double> ev, esc;
    const bool lower = (k <= 1);
    int rlo = 0, rhi = m0, clo = 0, chi = m0;
    if (k == 1) rlo = m0, rhi = n;
    if (k == 2) clo = m0, chi = n;
    if (K == 0 && (k == 1 || k == 2)) rlo = rhi = 0;
    if (lower)
      build_levels(n, ut_p, ut_c, ut_v, k == 0 ? &F.u_inv_diag : nullptr, true, rlo, rhi, clo, chi, k == 1, lev, rows,
                   eptr, ecol, ev, esc);
    else
      build_levels(n, lt_p, lt_c, lt_v, nullptr, false, rlo, rhi, clo, chi, k == 2, lev, rows, eptr, ecol, ev, esc);
    const int nslots = (int)rows.size();
    const int group = group_for(eptr, k == 1 || k == 2);
    rows.push_back(0);
    if (ecol.empty()) {
      ecol.push_back(0);
      ev.push_back(0.0);
    }
    CK(upload(A.lev[k], lev, s));
    CK(upload(A.rows[k], rows, s));
    CK(upload(A.eptr[k], eptr, s));
    CK(upload(A.col[k], ecol, s));
    CK(upload(A.val[k], ev, s));
    if (k == 0) {
      esc.push_back(1.0);
      CK(upload(A.scale0, esc, s));
    }
    LevelSolve &L = *ls[k];
    L.lev_ptr = A.lev[k].p;
    L.rows = A.rows[k].p;
    L.eptr = A.eptr[k].p;
    L.col = A.col[k].p;
    L.val = A.val[k].p;
    L.scale = (k == 0) ? A.scale0.p : nullptr;
    L.nlev = (int)lev.size() - 1;
    L.nslots = nslots;
    L.group = group;
    A.max_nlev = std::max(A.max_nlev, L.nlev);
  }
  // the forward tail (one network: offset 0) transposed on the device
  std::vector<double> ones(std::max(1, K), 1.0);
  CK(A.tl.alloc((size_t)std::max(1, K * K)));
  if (K > 0) {
    adj_tail_kernel<<<dim3((K + 31) / 32, (K + 31) / 32), dim3(32, 8), 0, s>>>(H->tail_l.p, H->tail_uinv.p, K,
                                                                                 A.tl.p);
    CK(cudaGetLastError());
  }
  CK(upload(A.tones, ones, s));
  td.T.K = K;
  td.T.L = A.tl.p;
  td.T.U = A.tl.p;
  td.T.uinv = A.tones.p;
  td.T.lscale = H->tail_uinv.p;
  td.T.W = nullptr;
  A.use_winv = false;
  A.xt32_p = nullptr;
  if (H->winv_ready) {  // A^-T = (Q X P)^T: X^T with the transposed system's P and Q
    const int ldw = H->winv_ldw;
    const size_t xbytes = sizeof(double) * (size_t)n * ldw;
    size_t fr = 0, tot = 0;
    if (A.xt.cap < (size_t)n * ldw) CK(cudaMemGetInfo(&fr, &tot));
    if (A.xt.cap >= (size_t)n * ldw || xbytes + ((size_t)1 << 30) <= fr + sizeof(double) * A.xt.cap) {
      CK(A.xt.alloc((size_t)n * ldw));
      CK(cudaMemsetAsync(A.xt.p, 0, xbytes, s));
      transpose_ld_kernel<<<dim3((n + 31) / 32, (n + 31) / 32), dim3(32, 8), 0, s>>>(H->winv.p, ldw, n, n, A.xt.p,
                                                                                     ldw);
      CK(cudaGetLastError());
      A.xt32_p = make_winv_f32(H, A.xt32, A.xt.p, (size_t)n * ldw);
      const RealSys &S = H->sys[0];
      std::vector<int> cp(n + 1, 0), ri(S.mcol.size()), mp(S.mcol.size());
      for (int c : S.mcol) cp[c + 1]++;
      for (int i = 0; i < n; i++) cp[i + 1] += cp[i];
      std::vector<int> fill(cp.begin(), cp.end() - 1);
      for (int rr = 0; rr < n; rr++)
        for (int p = S.mrow_ptr[rr]; p < S.mrow_ptr[rr + 1]; p++) {
          const int c = S.mcol[p];
          ri[fill[c]] = rr;
          mp[fill[c]++] = p;
        }
      CK(upload(A.at_ptr, cp, s));
      CK(upload(A.at_col, ri, s));
      CK(upload(A.at_map, mp, s));
      A.use_winv = true;
    }
  }
  if (K >= CLUSTER_MIN_K && H->tail_w.p && H->tail_w.n == (size_t)K * K) {  // (L U)^-T = W^T
    CK(A.tw.alloc((size_t)K * K));
    transpose_kernel<<<dim3((K + 31) / 32, (K + 31) / 32), dim3(32, 8), 0, s>>>(H->tail_w.p, A.tw.p, K);
    CK(cudaGetLastError());
    td.T.W = A.tw.p;
  }
  std::vector<int> qinv(n), pinvinv(n);
  for (int k = 0; k < n; k++) qinv[F.q[k]] = k;
  for (int i = 0; i < n; i++) pinvinv[F.pinv[i]] = i;
  CK(upload(A.pinv, qinv, s));
  CK(upload(A.qcol, pinvinv, s));
  td.pinv = A.pinv.p;
  td.qcol = A.qcol.p;
  td.row0 = 0;
  td.n = n;
  std::vector<TriDesc> tdv(1, td);
  CK(upload(A.tri, tdv, s));
  CK(cudaStreamSynchronize(s));
  H->adj_factors_ready = true;
  return 0;
}

static void launch_trisolve_adj(AndfnHandle *H, const Net &net, cudaStream_t s) {
  if (H->adj->use_winv) {
    const AdjBufs &A = *H->adj;
    launch_winv_solve<true>(H, net, s, A.xt.p, A.at_ptr.p, A.at_col.p, A.at_map.p, A.xt32_p);
    return;
  }
  const size_t ybytes = sizeof(double) * (size_t)H->max_n;
  const int use_smem = ybytes <= 150 * 1024 ? H->max_n : 0;
  const int cap_levptr = std::min(H->adj->max_nlev + 1, 10240);
  size_t solve_smem = (use_smem ? ybytes : 0) + sizeof(int) * (size_t)cap_levptr;
  const size_t meta_bytes = sizeof(int) * 2 * ((size_t)H->max_n + 1);
  const int meta_cap = (solve_smem + meta_bytes <= 200 * 1024) ? H->max_n + 1 : 0;
  if (meta_cap) solve_smem += meta_bytes;
  const int ring_cap = ring_capacity(solve_smem, use_smem, meta_cap);
  if (ring_cap) solve_smem = ((solve_smem + 15) & ~(size_t)15) + ring_bytes(ring_cap);
  if (H->cluster_adj < 0) H->cluster_adj = choose_cluster<true>(H, solve_smem, use_smem);
  launch_trisolve_kernel<true>(H, net, s, H->cluster_adj, solve_smem, use_smem, cap_levptr, meta_cap, ring_cap);
}

// per transposed sweep: 3 memsets + 5 kernels + the transposed discharge solve
// operations of one transposed sweep (3 memsets, 5 kernels, the transposed
// discharge solve: 3 kernels through X^T with its refinement step, else 1)
static int adj_sweep_launches(const AndfnHandle *H) { return 8 + ((H->adj && H->adj->use_winv) ? 3 : 1); }
static constexpr int ADJ_RESTART = GM_MK;     // Krylov basis size before a restart

// One transposed sweep at lam = x: gc = Phi_c^T x + b_c^T A^-T (gd + Phi_d^T x),
// then y = (I - T^T) x (mode 0, gd = 0) or y = F(x) - x (mode 1, the real dJ/dd).
static void adj_enqueue_sweep(AndfnHandle *H, const Net &net, const Net &net_t, cudaStream_t s, const cd *x,
                              const double *gd, cd *y, int mode) {
  AdjBufs &A = *H->adj;
  const int ne = (int)H->ne, nf = (int)H->nf, N = H->N, MC = H->MC;
  const unsigned ce = (unsigned)(((long long)ne * MC + 255) / 256);
  cudaMemsetAsync(A.gc.p, 0, sizeof(cd) * (size_t)ne * MC, s);
  cudaMemsetAsync(A.gq.p, 0, sizeof(double) * ne, s);
  cudaMemsetAsync(A.gC.p, 0, sizeof(double) * nf, s);
  adj_fit_kernel<<<(ne + UPDATE_WARPS - 1) / UPDATE_WARPS, UPDATE_WARPS * 32, sizeof(double) * H->nvmax * UPDATE_WARPS,
                   s>>>(net, x, H->group_of.p, H->d_groups.p, A.wsw.p, A.gq.p, H->nvmax, A.st.p);
  if (H->use_tab && H->tab_valid && MC <= 32 && A.n_items_tab > 0) {
#define ANDFN_ADJ_TAB(MMV)                                                                                      \
  adj_sweep_table_kernel<MMV><<<A.n_items_tab, EVAL_THREADS, 0, s>>>(                                          \
      net, A.items_tab.p, H->sweep_pts.p, H->d_groups.p, H->tab_fpt0.p, H->tab_fnp.p, H->tab_off.p, H->tab_w.p, \
      H->tab_l.p, A.wsw.p, A.gc.p, A.gq.p, A.gC.p, A.st.p)
    if (MC <= 16)
      ANDFN_ADJ_TAB(16);
    else if (MC <= 24)
      ANDFN_ADJ_TAB(24);
    else
      ANDFN_ADJ_TAB(32);
#undef ANDFN_ADJ_TAB
  } else if (A.n_items_sw > 0) {
    adj_sweep_kernel<<<A.n_items_sw, EVAL_THREADS, A.smem, s>>>(net, A.items_sw.p, H->sweep_pts.p, H->d_groups.p,
                                                                 A.wsw.p, A.gc.p, A.gq.p, A.gC.p, A.chunk, A.st.p);
  }
  adj_rhs_kernel<<<(N + 255) / 256, 256, 0, s>>>(net, gd, A.gq.p, A.gC.p, A.b.p, A.st.p);
  launch_trisolve_adj(H, net_t, s);
  if (H->hs.npairs > 0)
    adj_rhs_gather_kernel<<<ce, 256, 0, s>>>(net, H->hs.src_ptr.p, H->hs.src_pairs.p, H->hs.pair_g.p,
                                             H->hs.pair_off.p, H->hs.S.p, A.mu.p, A.fac.p, A.gc.p, A.st.p);
  adj_combine_kernel<<<ce, 256, 0, s>>>(net, x, A.gc.p, A.gobj.p, y, mode);
}

static int adjoint_impl(AndfnHandle *H, const double *gcoef, int64_t mco, const double *gq_user,
                        const double *gC_user, double tol, int64_t max_it, double *glogt, AndfnAdjointStats *S) {
  auto t0 = std::chrono::steady_clock::now();
  if (H->R != 1) {
    set_error("the adjoint needs a single-network handle");
    return ANDFN_BAD_INPUT;
  }
  if (H->has_spec) {
    set_error("the adjoint does not cover wells with a prescribed discharge (NaN head)");
    return ANDFN_BAD_INPUT;
  }
  if (!H->have_solution || H->lu_keep.n != H->N) {
    set_error("the adjoint needs a completed run() on this handle (and no reset since)");
    return ANDFN_BAD_INPUT;
  }
  if (!gcoef || !gq_user || !gC_user || !glogt || mco < 0 || !(tol > 0) || max_it < 1) {
    set_error("adjoint: bad pointers, mco, tol or max_iterations");
    return ANDFN_BAD_INPUT;
  }
  cudaStream_t s = H->stream;
  if (!H->adj) H->adj = new AdjBufs();
  AdjBufs &A = *H->adj;
  const int ne = (int)H->ne, nf = (int)H->nf, N = H->N, MC = H->MC, n_de = (int)H->h.de_ids.size();
  if (!H->adj_factors_ready) {
    int rc = adj_build_factors(H);
    if (rc) return rc;
  }
  // sweep point tables: the forward list (rebuilt in the same order), in
  // items of up to ADJ_ITEM points of one fracture
  {
    std::vector<Group> groups;
    std::vector<int> go;
    std::vector<Item> si, items;
    std::vector<int2> spts;
    int nsv = 0;
    build_tables(H, false, groups, go, si, spts, nsv);
    adj_items(groups, spts, items);
    CK(upload(A.items_sw, items, s));
    A.n_items_sw = (int)items.size();
    CK(A.wsw.alloc(std::max(1, nsv)));
    int maxnf = 1;
    for (int f = 0; f < nf; f++) maxnf = std::max(maxnf, H->h.fptr[f + 1] - H->h.fptr[f]);
    const size_t red = sizeof(double) * 2 * MC * ADJ_RED_STRIDE * (EVAL_THREADS / 32);
    const size_t per = sizeof(Src) + sizeof(cd) * MC + sizeof(double);
    const size_t budget = 100 * 1024 > red + per ? 100 * 1024 - red : per;
    A.chunk = std::max(1, std::min((int)(budget / per), maxnf));
    A.smem = per * A.chunk + red;
    if (A.smem > 200 * 1024) {
      set_error("adjoint: coefficient capacity too large for the transposed evaluation");
      return ANDFN_BAD_INPUT;
    }
    CK(cudaFuncSetAttribute(adj_sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    // items of the table-driven transposed sweep
    std::vector<Item> ti;
    for (int f = 0; f < nf && f < (int)H->h_tab_fpt0.size(); f++)
      for (int a = 0; a < H->h_tab_fnp[f]; a += ADJ_TAB_PTS) {
        Item it;
        it.frac = f;
        it.p0 = H->h_tab_fpt0[f] + a;
        it.p1 = H->h_tab_fpt0[f] + std::min(H->h_tab_fnp[f], a + ADJ_TAB_PTS);
        it.pad = 0;
        ti.push_back(it);
      }
    CK(upload(A.items_tab, ti, s));
    A.n_items_tab = (int)ti.size();
  }
  {
    int rcs = build_head_sums(H);
    if (rcs) return rcs;
  }
  {
    // row-side weights per unit mu (t may have changed since the sums)
    const HostNet &h = H->h;
    std::vector<double> fac(2 * (size_t)std::max(1, n_de), 0.0);
    for (int j = 0; j < n_de; j++) {
      const int e = h.de_ids[j];
      if (h.type[e] == 0) {
        fac[2 * j] = -1.0 / (H->D * h.t[h.frac0[e]]);
        fac[2 * j + 1] = 1.0 / (H->D * h.t[h.frac1[e]]);
      } else {
        fac[2 * j] = -1.0 / H->D;
      }
    }
    CK(upload(A.fac, fac, s));
  }
  CK(A.st.alloc(1));
  CK(A.st_eval.alloc(1));
  CK(A.lam.alloc((size_t)ne * MC));
  CK(A.gobj.alloc((size_t)ne * MC));
  CK(A.gc.alloc((size_t)ne * MC));
  CK(A.gq.alloc(ne));
  CK(A.gC.alloc(nf));
  CK(A.gd.alloc(N));
  CK(A.b.alloc(N));
  CK(A.mu.alloc(N));
  CK(A.gtheta.alloc(nf));
  CK(A.obar.alloc(2 * (size_t)std::max(1, n_de)));
  // objective gradients
  CK(cudaMemsetAsync(A.gobj.p, 0, sizeof(cd) * (size_t)ne * MC, s));
  const int64_t w = std::min<int64_t>(mco, MC);
  if (w > 0)
    CK(cudaMemcpy2DAsync(A.gobj.p, sizeof(cd) * MC, gcoef, sizeof(cd) * mco, sizeof(cd) * w, ne,
                         cudaMemcpyDeviceToDevice, s));
  Net net = H->net();
  adj_gd_kernel<<<(N + 255) / 256, 256, 0, s>>>(net, gq_user, gC_user, A.gd.p);
  // sweep values at the converged state (for lam^T Phi_theta)
  SolveState se;
  std::memset(&se, 0, sizeof(se));
  se.solve_q = 1;
  CK(cudaMemcpyAsync(A.st_eval.p, &se, sizeof(se), cudaMemcpyHostToDevice, s));
  Net net_e = net;
  net_e.st = A.st_eval.p;
  launch_sweep(H, net_e, s);
  // The multipliers solve the linear system (I - T^T) lam = F(0), F(lam) =
  // mask(dJ/dc + gc(lam)) with gc from one transposed sweep (the damped
  // fixed-point iteration lam <- F(lam) contracts only as fast as the forward
  // loop).  Restarted GMRES with this operator, classical Gram-Schmidt
  // applied twice; the start vector is 0.
  AdjState as0;
  std::memset(&as0, 0, sizeof(as0));
  CK(cudaMemcpyAsync(A.st.p, &as0, sizeof(as0), cudaMemcpyHostToDevice, s));
  const long long nd = (long long)ne * MC, n2 = 2 * nd;
  const int mk_ = ADJ_RESTART;
  CK(A.V.alloc((size_t)(mk_ + 1) * nd));
  CK(A.xin.alloc(nd));
  CK(A.wv.alloc(nd));
  CK(A.gd0.alloc(N));
  CK(A.hbuf.alloc(2 * (size_t)(mk_ + 2)));
  CK(cudaMemsetAsync(A.gd0.p, 0, sizeof(double) * N, s));
  CK(cudaMemsetAsync(A.lam.p, 0, sizeof(cd) * nd, s));
  CK(cudaMemsetAsync(A.mu.p, 0, sizeof(double) * N, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  const double ms_setup = ms_since(t0);
  auto t1 = std::chrono::steady_clock::now();
  Net net_t = net;  // the transposed discharge solve: b -> mu
  net_t.st = reinterpret_cast<SolveState *>(A.st.p);
  net_t.bvec = A.b.p;
  net_t.disc = A.mu.p;
  net_t.tri = A.tri.p;
  for (auto &g : A.graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  for (int mode = 0; mode < 2; mode++) {
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    adj_enqueue_sweep(H, net, net_t, s, A.xin.p, mode ? A.gd.p : A.gd0.p, A.wv.p, mode);
    CK(cudaStreamEndCapture(s, &g));
    CK(cudaGraphInstantiate(&A.graph[mode], g, 0));
    cudaGraphDestroy(g);
  }
  double *V = reinterpret_cast<double *>(A.V.p);
  double *wv = reinterpret_cast<double *>(A.wv.p);
  double *hd = A.hbuf.p;
  const int vb = 4 * 148, vt = 256;
  // one Arnoldi step as a graph (its kernels read j and stop from A.gm)
  CK(A.gm.alloc(1));
  if (A.step_graph) {
    cudaGraphExecDestroy(A.step_graph);
    A.step_graph = nullptr;
  }
  {
    GmresDev *gd = A.gm.p;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    gm_copy_kernel<<<vb, vt, 0, s>>>(gd, V, reinterpret_cast<double *>(A.xin.p), n2);
    adj_enqueue_sweep(H, net, net_t, s, A.xin.p, A.gd0.p, A.wv.p, 0);
    cudaMemsetAsync(hd, 0, sizeof(double) * 2 * (GM_MK + 2), s);
    for (int pass = 0; pass < 2; pass++) {
      double *hp = hd + pass * (GM_MK + 2);
      gm_mdot_kernel<<<vb, vt, 0, s>>>(gd, V, n2, 0, wv, n2, hp);
      gm_update_kernel<<<vb, vt, 0, s>>>(gd, wv, V, n2, hp, n2);
    }
    gm_mdot_kernel<<<vb, vt, 0, s>>>(gd, wv, 0, 1, wv, n2, hd + 2 * (GM_MK + 2) - 1);
    gm_givens_kernel<<<1, 32, 0, s>>>(gd, hd, A.st.p);
    gm_scale_kernel<<<vb, vt, 0, s>>>(gd, wv, V, n2);
    const cudaError_t ec = cudaStreamEndCapture(s, &g);
    if (ec != cudaSuccess) {
      set_error(std::string("capture of the Arnoldi step: ") + cudaGetErrorString(ec));
      return ANDFN_CUDA_ERROR;
    }
    CK(cudaGraphInstantiate(&A.step_graph, g, 0));
    cudaGraphDestroy(g);
  }
  // kernels of one Arnoldi step: copy + sweep + memset + 5 + Givens + scale
  const int step_launches = 1 + adj_sweep_launches(H) + 1 + 5 + 2;
  constexpr int STEPS_PER_SYNC = 8;
  int64_t matvecs = 0, launches = 4;
  // |w|^2 on the device into hd[0], read back
  auto norm2_of = [&](const double *w, double &out) -> int {
    CK(cudaMemsetAsync(hd, 0, sizeof(double), s));
    vec_mdot_kernel<<<vb, vt, 0, s>>>(w, 0, 1, w, n2, hd);
    CK(cudaMemcpyAsync(&out, hd, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    launches += 1;
    return 0;
  };
  auto sweep = [&](const double *x, int mode) -> int {  // wv = (I - T^T) x or F(x) - x
    CK(cudaMemcpyAsync(A.xin.p, x, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
    CK(cudaGraphLaunch(A.graph[mode], s));
    matvecs++;
    launches += adj_sweep_launches(H);
    return 0;
  };
  double bnorm = 0.0, rel = 1.0;
  int nonfinite = 0;
  std::vector<double> Hm((size_t)(mk_ + 1) * mk_), gv(mk_ + 1);
  while (true) {
    // residual r = F(x) - x
    if (sweep(reinterpret_cast<const double *>(A.lam.p), 1)) return ANDFN_CUDA_ERROR;
    double r2 = 0.0;
    if (norm2_of(wv, r2)) return ANDFN_CUDA_ERROR;
    const double beta = std::sqrt(r2);
    if (!std::isfinite(beta)) {
      nonfinite = 1;
      break;
    }
    if (matvecs == 1) bnorm = beta;
    if (bnorm == 0.0) {
      rel = 0.0;
      break;
    }
    rel = beta / bnorm;
    if (rel <= tol || matvecs >= max_it) break;
    vec_scale_kernel<<<vb, vt, 0, s>>>(wv, V, 1.0 / beta, n2);
    gm_reset_kernel<<<1, 32, 0, s>>>(A.gm.p, A.st.p, beta, bnorm, tol, matvecs, max_it);
    launches += 2;
    // Arnoldi steps in batches; the device stops the cycle
    GmresDev gh;
    for (int done_steps = 0; done_steps < mk_;) {
      const int nb = std::min(STEPS_PER_SYNC, mk_ - done_steps);
      for (int b = 0; b < nb; b++) CK(cudaGraphLaunch(A.step_graph, s));
      launches += (int64_t)nb * step_launches;
      done_steps += nb;
      CK(cudaMemcpyAsync(&gh, A.gm.p, sizeof(GmresDev), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      if (gh.stop) break;
    }
    matvecs = gh.matvecs;
    rel = gh.rel;
    const int k = gh.k;
    if (gh.nonfinite) {
      nonfinite = 1;
      break;
    }
    for (int i = 0; i <= k && i <= mk_; i++) gv[i] = gh.gv[i];
    for (int i = 0; i < k; i++)
      for (int c = 0; c < k; c++) Hm[(size_t)i * mk_ + c] = gh.Hm[i * GM_MK + c];
    // the sweeps of the next cycle (or the final residual) run again
    {
      const int zero = 0;
      CK(cudaMemcpyAsync(&A.st.p->s.done, &zero, sizeof(int), cudaMemcpyHostToDevice, s));
    }
    // x += V y, H y = g (upper triangular k x k)
    std::vector<double> y(k, 0.0);
    for (int i = k - 1; i >= 0; i--) {
      double t = gv[i];
      for (int c = i + 1; c < k; c++) t -= Hm[(size_t)i * mk_ + c] * y[c];
      y[i] = t / Hm[(size_t)i * mk_ + i];
    }
    CK(cudaMemcpyAsync(hd, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
    vec_update_kernel<<<vb, vt, 0, s>>>(reinterpret_cast<double *>(A.lam.p), V, n2, k, hd, 1.0, n2);
    CK(cudaStreamSynchronize(s));
    launches += 1;
  }
  // the multiplier of the discharge system at the final lam, and the true
  // residual of the final lam (mode 1 sweep)
  if (sweep(reinterpret_cast<const double *>(A.lam.p), 1)) return ANDFN_CUDA_ERROR;
  double rf2 = 0.0;
  if (norm2_of(wv, rf2)) return ANDFN_CUDA_ERROR;
  const double rel_true = bnorm > 0 ? std::sqrt(rf2) / bnorm : 0.0;
  double l2 = 0.0;
  if (norm2_of(reinterpret_cast<const double *>(A.lam.p), l2)) return ANDFN_CUDA_ERROR;
  // lam^T Phi_theta and the mean potentials of the discharge rows
  CK(cudaMemsetAsync(A.gtheta.p, 0, sizeof(double) * nf, s));
  adj_theta_kernel<<<(ne * 32 + 127) / 128, 128, 0, s>>>(net, A.lam.p, H->group_of.p, H->d_groups.p,
                                                          H->sweep_vals.p, A.gtheta.p);
  if (n_de > 0) adj_obar_kernel<<<(2 * n_de * 32 + 127) / 128, 128, 0, s>>>(net, A.obar.p);
  launches += 2;
  std::vector<double> mu(N), obar(2 * (size_t)std::max(1, n_de)), gth(nf), tt(nf);
  CK(cudaMemcpyAsync(mu.data(), A.mu.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(obar.data(), A.obar.p, sizeof(double) * obar.size(), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(gth.data(), A.gtheta.p, sizeof(double) * nf, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(tt.data(), H->t.p, sizeof(double) * nf, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  // mu^T (b_theta - A_theta d): an intersection row gives mu * mean(Re Omega)
  // / t on each side (+ on frac0, - on frac1); a constant-head line or well
  // row gives mu * head * t
  const HostNet &h = H->h;
  for (int j = 0; j < n_de; j++) {
    const int e = h.de_ids[j];
    const int f0 = h.frac0[e];
    if (h.type[e] == 0) {
      const int f1 = h.frac1[e];
      gth[f0] += mu[j] * obar[2 * j] / tt[f0];
      gth[f1] -= mu[j] * obar[2 * j + 1] / tt[f1];
    } else {
      gth[f0] += mu[j] * h.head[e] * tt[f0];
    }
  }
  CK(cudaMemcpyAsync(glogt, gth.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  int status = ANDFN_OK;
  if (nonfinite || !std::isfinite(rel_true))
    status = ANDFN_NONFINITE;
  else if (!(rel_true <= 10.0 * tol))
    status = ANDFN_MAX_ITERATIONS;
  if (S) {
    std::memset(S, 0, sizeof(*S));
    S->iterations = matvecs;
    S->residual = rel_true;
    S->lam_norm = std::sqrt(l2);
    S->restart = ADJ_RESTART;
    S->ms_setup = ms_setup;
    S->ms_iterate = ms_since(t1);
    S->ms_total = ms_since(t0);
    S->gpu_launches = launches;
    S->status = status;
  }
  return status;
}

static int set_transmissivity_impl(AndfnHandle *H, const double *t) {
  for (int64_t f = 0; f < H->nf; f++)
    if (!(t[f] > 0) || !std::isfinite(t[f])) {
      set_error("transmissivity must be positive and finite");
      return ANDFN_BAD_INPUT;
    }
  HostNet &h = H->h;
  for (int64_t f = 0; f < H->nf; f++) h.t[f] = t[f];
  // phi = head * t of constant-head lines and wells (Fracture.phi_from_head)
  for (int64_t e = 0; e < H->ne; e++)
    if (h.type[e] == 2 || h.type[e] == 3) h.phi[e] = h.head[e] * h.t[h.frac0[e]];
  cudaStream_t s = H->stream;
  CK(cudaMemcpyAsync(H->t.p, h.t.data(), sizeof(double) * H->nf, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(H->phi.p, h.phi.data(), sizeof(double) * H->ne, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  H->have_solution = false;
  return 0;
}

}  // namespace andfn

extern "C" {

int andfn_b200_set_transmissivity(AndfnHandle *H, const double *t) {
  if (!H || !t) return ANDFN_BAD_INPUT;
  CK(cudaSetDevice(H->device));
  PoolStream pool_scope(H->stream);
  return set_transmissivity_impl(H, t);
}

int andfn_b200_state_device(AndfnHandle *H, double *coef, int64_t mco, double *q, double *constant) {
  if (!H || mco < 0 || (mco > 0 && !coef) || !q || !constant) return ANDFN_BAD_INPUT;
  CK(cudaSetDevice(H->device));
  PoolStream pool_scope(H->stream);
  cudaStream_t s = H->stream;
  const int64_t w = std::min<int64_t>(mco, H->MC);
  if (mco > 0) {
    CK(cudaMemsetAsync(coef, 0, sizeof(cd) * mco * H->ne, s));
    if (w > 0)
      CK(cudaMemcpy2DAsync(coef, sizeof(cd) * mco, H->coef.p, sizeof(cd) * H->MC, sizeof(cd) * w, H->ne,
                           cudaMemcpyDeviceToDevice, s));
  }
  CK(cudaMemcpyAsync(q, H->q.p, sizeof(double) * H->ne, cudaMemcpyDeviceToDevice, s));
  CK(cudaMemcpyAsync(constant, H->constant.p, sizeof(double) * H->nf, cudaMemcpyDeviceToDevice, s));
  CK(cudaStreamSynchronize(s));
  return 0;
}

int andfn_b200_heads_device(AndfnHandle *H, const int64_t *frac, const double *z, int64_t npts, double *out) {
  if (!H || npts < 0 || (npts > 0 && (!frac || !z || !out)) || npts > (1LL << 31) - 1) return ANDFN_BAD_INPUT;
  if (H->R != 1) {
    set_error("heads_device needs a single-network handle");
    return ANDFN_BAD_INPUT;
  }
  if (npts == 0) return 0;
  CK(cudaSetDevice(H->device));
  PoolStream pool_scope(H->stream);
  heads_dev_kernel<<<(unsigned)((npts + 127) / 128), 128, 0, H->stream>>>(H->net(), frac, (const cd *)z, (int)npts,
                                                                           out);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(H->stream));
  return 0;
}

int andfn_b200_heads_vjp(AndfnHandle *H, const int64_t *frac, const double *z, int64_t npts, const double *gh,
                         double *gcoef, int64_t mco, double *gq, double *gC, double *glogt) {
  if (!H || npts < 0 || (npts > 0 && (!frac || !z || !gh)) || !gcoef || !gq || !gC || !glogt || mco < 0 ||
      npts > (1LL << 31) - 1)
    return ANDFN_BAD_INPUT;
  if (H->R != 1) {
    set_error("heads_vjp needs a single-network handle");
    return ANDFN_BAD_INPUT;
  }
  if (npts == 0) return 0;
  CK(cudaSetDevice(H->device));
  PoolStream pool_scope(H->stream);
  heads_vjp_kernel<<<(unsigned)((npts + 127) / 128), 128, 0, H->stream>>>(H->net(), frac, (const cd *)z, (int)npts,
                                                                           gh, gcoef, (int)mco, gq, gC, glogt);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(H->stream));
  return 0;
}

int andfn_b200_adjoint(AndfnHandle *H, const double *gcoef, int64_t mco, const double *gq, const double *gC,
                       double tol, int64_t max_iterations, double *glogt, AndfnAdjointStats *stats) {
  if (!H) return ANDFN_BAD_INPUT;
  CK(cudaSetDevice(H->device));
  PoolStream pool_scope(H->stream);
  return adjoint_impl(H, gcoef, mco, gq, gC, tol, max_iterations, glogt, stats);
}

}  // extern "C"

// ==========================================================================
// Boundary-condition residual and flux balance of the current state (no
// reference counterpart for the residual; the flux balance is
// Fracture.check_discharge, andfn/fracture.py:377-394).
//   intersection:   max_k |h0(z_k) - h1(z_k)| / h_scale at its collocation
//                   points (h = Re Omega_f / t_f, both sides)
//   constant head:  max_k |h(z_k) - head| / h_scale
//   well:           max over 16 points on its circle of |h - head| / h_scale
//   bounding circle, impermeable circle / line: (max_k - min_k) psi'_k /
//                   q_scale, psi' the stream function unwrapped across the
//                   branch cuts (the no-flow condition makes it constant)
// h_scale = max |head| of the constant-head lines and wells (1 if none);
// q_scale = the largest total |q| of a fracture's discharge elements
// (get_total_discharge, andfn/fracture.py:365-375), the network's flow scale.
// ==========================================================================
namespace andfn {

__global__ void bc_residual_kernel(Net net, double hscale, double qscale, double *res) {
  const int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (e >= net.ne) return;
  const int type = net.type[e];
  const int f0 = net.frac0[e];
  double r = 0.0;
  if (type == 0 || type == 3) {
    const int n = net.nint[e];
    const double t0 = net.t[f0];
    const double head = (type == 3) ? net.phi[e] / t0 : 0.0;
    for (int k = lane; k < n; k += 32) {
      const double h0 = omega_at(net, f0, sweep_point(net, e, 0, k)).re / t0;
      double d;
      if (type == 0) {
        const int f1 = net.frac1[e];
        d = h0 - omega_at(net, f1, sweep_point(net, e, 1, k)).re / net.t[f1];
      } else {
        d = h0 - head;
      }
      r = fmax(r, fabs(d) / hscale);
    }
  } else if (type == 2) {
    const double t0 = net.t[f0], head = net.phi[e] / t0;
    if (lane < 16 && head == head) {  // a NaN head: the well's discharge is prescribed instead
      double sn, cs;
      sincos(2 * PI * lane / 16, &sn, &cs);
      const cd z = mk(net.center[e].re + net.radius[e] * cs, net.center[e].im + net.radius[e] * sn);
      r = fabs(omega_at(net, f0, z).re / t0 - head) / hscale;
    }
  } else {
    const int n = net.nint[e];
    const int nc = net.cut_n[e];
    const int *cp = net.cut_pos + (size_t)e * net.cut_cap;
    const int *ce = net.cut_elem + (size_t)e * net.cut_cap;
    const int *cs = net.cut_sign + (size_t)e * net.cut_cap;
    double mx = -INFINITY, mn = INFINITY;
    for (int k = lane; k < n; k += 32) {
      double cum = 0.0;
      for (int c = 0; c < nc; c++)
        if (cp[c] < k) cum += net.q[ce[c]] * (double)cs[c];
      const double psi = omega_at(net, f0, sweep_point(net, e, 0, k)).im - cum;
      mx = fmax(mx, psi);
      mn = fmin(mn, psi);
    }
    for (int o = 16; o > 0; o >>= 1) {
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    }
    r = (mx >= mn) ? (mx - mn) / qscale : 0.0;
  }
  for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
  if (lane == 0) res[e] = r;
}

}  // namespace andfn

extern "C" int andfn_b200_bc_residual(AndfnHandle *H, double *elem_res, double *frac_flux, AndfnResidual *out) {
  if (!H || !out) return ANDFN_BAD_INPUT;
  if (H->R != 1) {
    set_error("bc_residual needs a single-network handle");
    return ANDFN_BAD_INPUT;
  }
  CK(cudaSetDevice(H->device));
  PoolStream pool_scope(H->stream);
  const HostNet &h = H->h;
  const int ne = (int)H->ne, nf = (int)H->nf;
  cudaStream_t s = H->stream;
  std::vector<double> tt(nf), phi(ne), q(ne);
  CK(cudaMemcpyAsync(tt.data(), H->t.p, sizeof(double) * nf, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(phi.data(), H->phi.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(q.data(), H->q.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  double hscale = 0.0;
  for (int e = 0; e < ne; e++)
    if (h.type[e] == 2 || h.type[e] == 3) hscale = std::max(hscale, std::fabs(phi[e] / tt[h.frac0[e]]));
  if (!(hscale > 0.0)) hscale = 1.0;
  // flow scale and the per-fracture balance (check_discharge,
  // andfn/fracture.py:377-394)
  std::vector<double> fsum(nf, 0.0), ftot(nf, 0.0);
  double qscale = 0.0;
  for (int f = 0; f < nf; f++) {
    for (int k = h.fptr[f]; k < h.fptr[f + 1]; k++) {
      const int el = h.felem[k], ty = h.type[el];
      if (ty != 0 && ty != 2 && ty != 3) continue;
      fsum[f] += (ty == 0 && h.frac1[el] == f) ? -q[el] : q[el];
      ftot[f] += std::fabs(q[el]);
    }
    qscale = std::max(qscale, ftot[f]);
  }
  if (!(qscale > 0.0)) qscale = 1.0;
  DBuf<double> dres;
  CK(dres.alloc(ne));
  // branch cuts of the current nint (also valid for a handle that has not run)
  if (H->n_psi > 0) cuts_kernel<<<(H->n_psi * 32 + 127) / 128, 128, 0, s>>>(H->net(), H->psi_list.p, H->n_psi);
  bc_residual_kernel<<<(ne * 32 + 127) / 128, 128, 0, s>>>(H->net(), hscale, qscale, dres.p);
  CK(cudaGetLastError());
  std::vector<double> res(ne);
  CK(cudaMemcpyAsync(res.data(), dres.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  std::memset(out, 0, sizeof(*out));
  out->h_scale = hscale;
  out->bc_worst = -1;
  for (int e = 0; e < ne; e++)
    if (!(res[e] <= out->bc_max)) {  // NaN propagates
      out->bc_max = res[e];
      out->bc_worst = e;
      if (!(res[e] == res[e])) break;
    }
  out->q_scale = qscale;
  out->flux_worst = -1;
  for (int f = 0; f < nf; f++) {
    const double rel = std::fabs(fsum[f]) / qscale;
    if (frac_flux) frac_flux[f] = std::fabs(fsum[f]);
    if (rel > out->flux_max) {
      out->flux_max = rel;
      out->flux_worst = f;
    }
  }
  if (elem_res) std::memcpy(elem_res, res.data(), sizeof(double) * ne);
  return 0;
}
