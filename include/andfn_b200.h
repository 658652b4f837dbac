/*
 * andfn_b200.h -- C ABI of the B200-native AnDFN analytic-element solve.
 *
 * The library replaces AnDFN's iterative solve
 *     andfn.hpc.hpc_solve.solve(fracture_struc_array, element_struc_array,
 *                               discharge_int, constants, ntype_elements)
 * (andfn/hpc/hpc_solve.py:55-257), which andfn.dfn.DFN.solve calls at
 * andfn/dfn.py:1840-1846 through the module-level name bound at andfn/dfn.py:21.
 *
 * Records are the reference's packed numpy structured arrays:
 *   element_dtype_hpc   (andfn/element.py:45-69)
 *   fracture_dtype_hpc  (andfn/element.py:146-159)
 * Their field offsets depend on the YAML-configurable MAX_NCOEF / MAX_ELEMENTS
 * (andfn/element.py:13-20), so every entry point takes an AndfnLayout that the
 * caller derives from dtype.fields.  Records are read and written in place with
 * the reference's semantics: elements get coef[:ncoef], ncoef, nint, thetas, q,
 * error, error_old, error_old2, error_coef and dpsi_corr; fractures get
 * constant.
 *
 * All arithmetic is IEEE binary64 / complex128.  No entry point allocates on
 * the calling thread's CUDA stream other than its own; handles are not
 * re-entrant (use one handle per host thread).
 */
#ifndef ANDFN_B200_H
#define ANDFN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes (int).  0 is success; the solve-outcome codes (1..3) still
 * leave the records updated with the last iterate, like the reference, which
 * returns silently in those cases (andfn/hpc/hpc_solve.py:152,257). */
enum {
  ANDFN_OK = 0,
  ANDFN_MAX_ITERATIONS = 1, /* loop stopped at MAX_ITERATIONS before 2 converged rounds */
  ANDFN_NONFINITE = 2,      /* a coefficient, discharge or error became NaN/Inf        */
  ANDFN_SINGULAR = 3,       /* discharge system has a zero pivot (disconnected fracture) */
  ANDFN_BAD_LAYOUT = 10,    /* offsets/strides inconsistent or sizes out of range      */
  ANDFN_BAD_INPUT = 11,     /* ids out of range, ncoef > capacity, nint/ncoef mismatch */
  ANDFN_CUDA_ERROR = 12,    /* a CUDA runtime call failed (message via andfn_b200_last_error) */
  ANDFN_NO_DEVICE = 13,     /* no sm_100 device visible                                */
  ANDFN_OUT_OF_MEMORY = 14
};

/* Byte offsets of the record fields, as given by numpy dtype.fields[name][1].
 * Complex fields are (re, im) double pairs; integer fields are int64. */
typedef struct AndfnLayout {
  int64_t elem_size; /* element_dtype_hpc.itemsize */
  int64_t e_id, e_type, e_frac0, e_frac1, e_endpoints0, e_endpoints1, e_radius,
      e_center, e_head, e_phi, e_ncoef, e_nint, e_q, e_thetas, e_coef,
      e_old_coef, e_dpsi_corr, e_error, e_error_old, e_error_old2, e_error_coef;
  int64_t max_ncoef; /* capacity of coef / old_coef; thetas and dpsi_corr hold 2*max_ncoef */
  int64_t frac_size; /* fracture_dtype_hpc.itemsize */
  int64_t f_id, f_t, f_radius, f_center, f_normal, f_x_vector, f_y_vector,
      f_elements, f_nelements, f_constant;
  int64_t max_elements; /* capacity of fracture.elements */
} AndfnLayout;

/* Solver fields of the reference's dtype_constants record
 * (andfn/constants.py:13-29), as read at andfn/hpc/hpc_solve.py:81-86. */
typedef struct AndfnConstants {
  double max_error;       /* MAX_ERROR      */
  int64_t max_iterations; /* MAX_ITERATIONS */
  int64_t max_ncoef;      /* MAX_NCOEF (runtime cap on adaptive growth) */
  double damping;         /* DAMPING        */
  int64_t coef_increase;  /* COEF_INCREASE  */
  double coef_ratio;      /* COEF_RATIO     */
} AndfnConstants;

/* What the reference only logs (andfn/hpc/hpc_solve.py:196-255), returned. */
typedef struct AndfnSolveStats {
  int64_t iterations;    /* nit at exit                                   */
  int64_t cnt_error;     /* converged rounds seen (2 = converged)         */
  double error;          /* max element error (truncation indicator)      */
  double error_coef;     /* max element mean |delta coef|                 */
  double error_q;        /* relative max |delta discharge| of last round  */
  int64_t worst_element; /* argmax of error                               */
  int64_t n_unknowns;    /* discharge-system size                         */
  int64_t nnz_matrix;    /* discharge-system nonzeros                     */
  int64_t nnz_factors;   /* nonzeros of L+U                               */
  int64_t gpu_launches;  /* kernels this library launched for the solve   */
  double ms_upload, ms_setup, ms_factor, ms_iterate, ms_download, ms_total;
  int32_t status;        /* same as the return code                       */
  int32_t device;        /* CUDA ordinal used                             */
  int64_t h2d_bytes;     /* host->device bytes of andfn_b200_solve        */
  int64_t d2h_bytes;     /* device->host bytes of andfn_b200_solve        */
  int64_t dense_tail;    /* pivot steps solved as a dense trailing block  */
  int64_t levels_l;      /* dependency levels of the sparse part of L     */
  int64_t levels_u;      /* dependency levels of the sparse part of U     */
  double ms_create_upload, ms_create_tables, ms_create_order; /* handle creation phases (the column
                            ordering runs on a host thread of its own, alongside the tables and the first
                            run's device set-up; ms_create_order is that thread's time) */
  int64_t tri_cycles[8]; /* SM cycles of the discharge-solve phases, summed over iterations:
                            head vector, L sparse, L coupling, L dense, U dense,
                            U coupling, U sparse, scatter */
  int64_t explicit_inverse; /* 1: each discharge solve applied the system's explicit inverse
                               (formed once per factorisation) with one refinement step;
                               0: level-scheduled triangular solves */
  double ms_factor_sparse;  /* ms_factor parts: sparse LU + Schur complement (host),          */
  double ms_factor_dense;   /*   dense LU of the Schur complement (device, incl. its upload), */
  double ms_factor_levels;  /*   level-ordered factor tables + dense-tail inverse,            */
  double ms_inverse;        /*   explicit inverse of the system (device)                      */
  int64_t refined_solves;   /* explicit-inverse solves that took the refinement step */
  int64_t sweep_variant;    /* launch form of the sweep from pair tables, picked by the autotuner:
                               0 one CTA per work item, 1 / 2 persistent CTAs (4 / 6 per SM) on a
                               device work queue; -1: no pair tables (adaptive coefficient growth) */
  int64_t loop_launches;    /* graph launches of the iteration loop (1: the whole loop runs on the
                               device in one launch) */
  double ms_alloc;          /* host milliseconds in device allocation and release on the calling
                               thread (andfn_b200_solve: the whole call; a run: since the thread's
                               previous one-call solve) */
  int64_t refine_f32;       /* 1: the refinement pass read a float copy of the explicit inverse */
} AndfnSolveStats;

/* ---- one-call drop-in (replaces andfn/hpc/hpc_solve.py:55 solve) --------
 * frac_recs/elem_recs: host pointers to the structured arrays (C-contiguous).
 * ntype_elements is ignored by the reference (andfn/hpc/hpc_solve.py:55-79)
 * and is therefore not part of this signature.  stats may be NULL. */
int andfn_b200_solve(void *frac_recs, int64_t nf, void *elem_recs, int64_t ne,
                     const AndfnLayout *layout, int64_t discharge_int,
                     const AndfnConstants *constants, AndfnSolveStats *stats);

/* ---- handle API: keep a network resident in HBM across calls ------------ */
typedef struct AndfnHandle AndfnHandle;

/* Uploads the records, builds device tables.  device < 0 = current device. */
int andfn_b200_create(AndfnHandle **out, const void *frac_recs, int64_t nf,
                      const void *elem_recs, int64_t ne,
                      const AndfnLayout *layout, int64_t discharge_int,
                      int32_t device);
/* Re-uploads coefficient/discharge state (warm start) from host records. */
int andfn_b200_upload_state(AndfnHandle *h, const void *frac_recs,
                            const void *elem_recs);
/* Restores the state captured at create()/upload_state() on the device. */
int andfn_b200_reset_state(AndfnHandle *h);
/* Full solve on device-resident data (assembly, factorisation, iterations). */
int andfn_b200_run(AndfnHandle *h, const AndfnConstants *constants,
                   AndfnSolveStats *stats);
/* Writes the solved fields back into host records in place. */
int andfn_b200_download(AndfnHandle *h, void *frac_recs, void *elem_recs);
/* Heads h = Re(Omega_f(z)) / t_f at npts points of fracture frac[i]
 * (andfn/hpc/hpc_fracture.py:205-252).  z: complex128 [npts]; out: [npts]. */
int andfn_b200_eval_heads(AndfnHandle *h, const int64_t *frac, const double *z,
                          int64_t npts, double *out);
/* Complex potential Omega_f(z) at npts points (andfn/hpc/hpc_fracture.py:52-94,
 * exclude = -1).  out: complex128 [npts]. */
int andfn_b200_eval_omega(AndfnHandle *h, const int64_t *frac, const double *z,
                          int64_t npts, double *out);
/* Complex discharge vector w at npts points of fracture frac[i] of a
 * single-network handle (replaces andfn/hpc/hpc_fracture.py:139-175 calc_w,
 * exclude = -1; the velocity magnitude of Fracture.calc_velocity,
 * andfn/fracture.py:481-497, is |w| / aperture).  z, out: complex128 [npts]. */
int andfn_b200_eval_w(AndfnHandle *h, const int64_t *frac, const double *z,
                      int64_t npts, double *out);
/* The discharge vector of the reference's object layer, which its streamline
 * tracking uses: Fracture.calc_w (andfn/fracture.py:453-478), where bounding
 * circles carry -1/R (bounding.py:91-108) and are NaN beyond |z/R| > 1 + 1e-5,
 * wells and impermeable circles are NaN inside, and impermeable elements
 * contribute (impermeable_object.py:131-156, 205-224).  Single-network handle;
 * z, out: complex128 [npts]. */
int andfn_b200_eval_w_object(AndfnHandle *h, const int64_t *frac, const double *z,
                             int64_t npts, double *out);
/* Streamline tracking of npart particles on the handle's solved single network
 * (replaces DFN.streamline_tracking, andfn/dfn.py:2643-2722, called per start
 * point and elevation as DFN.plot_streamline_tracking does, dfn.py:2558-2641).
 * frac_recs: the nf fracture records of the handle (their frames are read with
 * the handle's layout); aperture: [nf] (the Fracture objects' aperture, which the
 * records do not hold).  Particle i starts at z[i] (complex128) on fracture
 * frac[i] with elevation[i]; ds is the step as a fraction of the fracture
 * radius, max_length the reference's point limit, backward != 0 traces against
 * the flow.  Outputs, cap slots per particle: out_z (complex128 [npart][cap]),
 * out_v (velocity |w| / aperture), out_seg (segment index of the point),
 * out_frac (fracture of the point); out_n [npart] points written, out_elem
 * [npart] the element the trace ended on (-1 = the reference's False),
 * out_status [npart] 0 = done, 1 = cap slots were not enough (trace cut). */
int andfn_b200_track(AndfnHandle *h, const void *frac_recs, int64_t nf,
                     const double *aperture, int64_t npart, const int64_t *frac,
                     const double *z, const double *elevation, double ds,
                     int64_t max_length, int32_t backward, int64_t cap,
                     double *out_z, double *out_v, int64_t *out_seg,
                     int64_t *out_frac, int64_t *out_n, int64_t *out_elem,
                     int32_t *out_status);
void andfn_b200_destroy(AndfnHandle *h);

/* CUDA stream the handle launches on (cudaStream_t as void*). */
void *andfn_b200_stream(AndfnHandle *h);

/* ---- batched realizations ------------------------------------------------
 * R independent networks (e.g. Monte-Carlo realizations of one fracture
 * statistics) solved by one launch sequence: every kernel of an outer
 * iteration covers all realizations, each realization keeps its own loop
 * state, factorisation and convergence test, and stops iterating on its own
 * (the reference solves them one at a time with hpc_solve.solve,
 * andfn/hpc/hpc_solve.py:55-257; each realization's result equals that
 * call's).  Arrays of length R give each realization's records and sizes;
 * stats, where given, has R entries.  The single-network functions above are
 * the R = 1 case; run() and download() refuse handles with R > 1. */
int andfn_b200_batch_solve(int64_t R, void *const *frac_recs, const int64_t *nf,
                           void *const *elem_recs, const int64_t *ne,
                           const AndfnLayout *layout, int64_t discharge_int,
                           const AndfnConstants *constants,
                           AndfnSolveStats *stats);
int andfn_b200_batch_create(AndfnHandle **out, int64_t R,
                            void *const *frac_recs, const int64_t *nf,
                            void *const *elem_recs, const int64_t *ne,
                            const AndfnLayout *layout, int64_t discharge_int,
                            int32_t device);
/* Returns the worst status over the realizations (per-realization status in
 * stats[r].status). */
int andfn_b200_batch_run(AndfnHandle *h, const AndfnConstants *constants,
                         AndfnSolveStats *stats);
int andfn_b200_batch_download(AndfnHandle *h, void *const *frac_recs,
                              void *const *elem_recs);
/* Heads at points of realization r (frac[] indexes that realization's
 * fractures). */
int andfn_b200_batch_eval_heads(AndfnHandle *h, int64_t r, const int64_t *frac,
                                const double *z, int64_t npts, double *out);
/* Number of realizations held by a handle. */
int64_t andfn_b200_realizations(AndfnHandle *h);

/* Per-kernel device timing of the outer iterations (no reference
 * counterpart; the reference only logs wall-clock phases,
 * andfn/hpc/hpc_solve.py:109-122,149-215).  When on, run() records CUDA
 * events around every kernel of every iteration; kernel_times() returns the
 * accumulated milliseconds and launch counts per kernel class, in the order
 * head-vector evaluation, triangular solve, sweep evaluation, element update,
 * reduction (n >= 5).  Turning it on resets the accumulators. */
int andfn_b200_set_profiling(AndfnHandle *h, int on);
int andfn_b200_kernel_times(AndfnHandle *h, double *ms, int64_t *launches, int n);

/* Measured FP64 FMA throughput of a device in TFLOP/s (the denominator of
 * the evaluation kernels' roofline). */
int andfn_b200_fp64_peak(int32_t device, double *tflops);

/* Device memory cache (no reference counterpart).  Device buffers released
 * by handles (andfn_b200_destroy, or a buffer that grows) are kept by the
 * library and reused by later handles of the process, so a one-call solve
 * does not pay cudaMalloc / cudaFree for its large buffers every call.  The
 * cache holds at most ANDFN_B200_POOL_MB MiB per device (environment,
 * default 8192; 0 turns it off) and gives its memory back when an
 * allocation fails.  release_cached_memory() frees every cached block of
 * every device; cached_memory() reports the bytes held on `device` and the
 * cache's hits and misses since the process started.  The page-locked host
 * blocks that stage the Schur complement of a factorisation are cached the
 * same way (ANDFN_B200_PINNED_POOL_MB, default 1024) and released with them. */
void andfn_b200_release_cached_memory(void);
int andfn_b200_cached_memory(int32_t device, int64_t *bytes, int64_t *hits, int64_t *misses);

/* Heads like andfn_b200_eval_heads, without allocating any memory (no
 * reference counterpart: the reference evaluates heads on the host).
 * For callers that cannot allocate device memory during a call -- a process
 * whose memory pool already holds all the device memory it may use, or a
 * loop that must not stall the device's other streams, which cudaFree does.
 * The points are staged in one fixed device array inside the library, so:
 *   - npts is at most ANDFN_NOALLOC_MAX_POINTS; larger calls are refused
 *     with ANDFN_BAD_INPUT (split them, or use andfn_b200_eval_heads);
 *   - the first call on a device looks the array up and caches its address:
 *     make it before any stream capture on that device.  The cached address
 *     belongs to the device's primary context, so it assumes that context
 *     lives as long as the library is loaded: after cudaDeviceReset the
 *     library must not be used again in that process;
 *   - the array is shared by all handles on a device: calls that overlap in
 *     time on one device race on it and must be serialised by the caller.
 * Fracture indices are those of the handle's first (or only) network. */
#define ANDFN_NOALLOC_MAX_POINTS 65536
int andfn_b200_eval_heads_noalloc(AndfnHandle *h, const int64_t *frac,
                                  const double *z, int64_t npts, double *out);

/* ---- network geometry on the device ---------------------------------------
 * Replace the host steps that build a network before the solve:
 * andfn_b200_disc_intersections is get_fracture_intersections
 * (andfn/geometry_functions.py:623-713) with fracture_intersection (:302-356)
 * and shorten_line (:974-993) by se_factor, for every pair of discs i < k
 * with |c_i - c_k| <= r_i + r_k.  Inputs are nf x 3 arrays (centers,
 * normals, the discs' in-plane x / y unit vectors as andfn/fracture.py:60-68
 * builds them) and the radii.  Output, sorted by (i, k): out_pairs[j] =
 * (i, k), out_ep0[j] / out_ep1[j] = the segment's two endpoints (complex,
 * re/im interleaved) in disc i's / disc k's frame.  *out_n receives the
 * number of segments; when it exceeds cap the call returns ANDFN_BAD_INPUT
 * and writes nothing (call again with cap >= *out_n).  Every operation is
 * rounded on its own in numpy's order, so the results equal the host
 * restatement (andfn_b200/network.py) bit for bit.
 * andfn_b200_clusters: the connected components of a pair list (the graph
 * check_connectivity_hpc walks, :1121-1294); out_root[f] is the smallest
 * fracture index of f's component.  device < 0: the current device.
 * andfn_b200_geometry_last_error: message of the last failing call of the two. */
int andfn_b200_disc_intersections(int32_t device, int64_t nf, const double *centers, const double *normals,
                                  const double *xvec, const double *yvec, const double *radii, double se_factor,
                                  int64_t cap, int64_t *out_pairs, double *out_ep0, double *out_ep1,
                                  int64_t *out_n);
int andfn_b200_clusters(int32_t device, int64_t nf, int64_t npairs, const int64_t *pairs, int64_t *out_root);
const char *andfn_b200_geometry_last_error(void);

/* ---- adjoint: gradient with respect to log-transmissivity ---------------
 * No reference counterpart (the reference computes no derivatives).  For an
 * objective J(coef, q, C, log t) of the converged solve of a single-network
 * handle, andfn_b200_adjoint returns dJ/dlog t_f (natural log) for every
 * fracture, given the partial derivatives of J with respect to the solved
 * state.  The multipliers of the solve's two equations (element sweep and
 * discharge system) solve a linear system whose operator is one transposed
 * sweep (the transposes of the sweep evaluation, the DFT fit and the
 * discharge solve, with the transposed factors of the last run); it is
 * solved by restarted GMRES, so no forward iterate is stored.  The solve
 * stops when the relative residual |F(lam) - lam| / |F(0)| <= tol or after
 * max_iterations transposed sweeps.
 * All array arguments of the functions in this block are DEVICE pointers on
 * the handle's device; complex values are (re, im) double pairs:
 *   gcoef [ne][mco][2]  dJ/d(Re, Im) coef (entries beyond ncoef are ignored)
 *   gq    [ne]          dJ/dq (read for the discharge elements only:
 *                       intersections, constant-head lines, wells)
 *   gC    [nf]          dJ/dC (fracture constants)
 *   glogt [nf]          output, overwritten: the part of dJ/dlog t that
 *                       flows through the solve (add the explicit part of J,
 *                       e.g. from andfn_b200_heads_vjp)
 * Requires a completed andfn_b200_run on the handle (with MAX_NCOEF =
 * ncoef, so that no coefficients grow) and no reset since.  Returns 0, or
 * ANDFN_MAX_ITERATIONS when the final residual is above 10 tol (the gradient
 * of the last iterate is still written). */
typedef struct {
  int64_t iterations;     /* transposed sweeps (operator applications) */
  double residual;        /* final relative residual                  */
  double lam_norm;        /* |lam|                                     */
  int64_t restart;        /* Krylov basis size between restarts        */
  double ms_setup, ms_iterate, ms_total;
  int64_t gpu_launches;
  int32_t status;
  int32_t pad;
} AndfnAdjointStats;
int andfn_b200_adjoint(AndfnHandle *h, const double *gcoef, int64_t mco,
                       const double *gq, const double *gC, double tol,
                       int64_t max_iterations, double *glogt,
                       AndfnAdjointStats *stats);
/* Replaces the fractures' transmissivities (host array [nf]) and with them
 * phi = head * t of constant-head lines and wells (the reference sets phi
 * once, at construction: andfn/const_head.py:45, andfn/well.py:38); the next
 * run() solves with them. */
int andfn_b200_set_transmissivity(AndfnHandle *h, const double *t);
/* Copies the solved state to device arrays: coef [ne][mco][2] (zero beyond
 * the handle's capacity), q [ne], C [nf]. */
int andfn_b200_state_device(AndfnHandle *h, double *coef, int64_t mco,
                            double *q, double *C);
/* Heads at device-resident points (frac int64 [n], z complex [n][2], out [n])
 * and the vector-Jacobian product of that map: given gh = dJ/dh, ADDS
 * dJ/d(coef, q, C) of the current state and the explicit dJ/dlog t
 * (-h gh) into gcoef [ne][mco][2], gq [ne], gC [nf], glogt [nf]. */
int andfn_b200_heads_device(AndfnHandle *h, const int64_t *frac,
                            const double *z, int64_t npts, double *out);
int andfn_b200_heads_vjp(AndfnHandle *h, const int64_t *frac, const double *z,
                         int64_t npts, const double *gh, double *gcoef,
                         int64_t mco, double *gq, double *gC, double *glogt);

/* ---- boundary-condition residual and flux balance -----------------------
 * Of the handle's current state (single network; after run() or download()).
 * Per element, the relative boundary-condition error at its collocation
 * points (no reference counterpart): intersections |h0 - h1|, constant-head
 * lines and wells |h - head|, both over h_scale = max |prescribed head|;
 * bounding circles and impermeable elements the spread of the stream
 * function unwrapped across branch cuts, over q_scale = the largest total
 * |q| of a fracture (get_total_discharge, andfn/fracture.py:365-375).  Per
 * fracture, |sum of signed discharges| as Fracture.check_discharge
 * (andfn/fracture.py:377-394); the summary gives its maximum over q_scale.
 * elem_res [ne] and frac_flux [nf] are host arrays or NULL. */
typedef struct {
  double bc_max;        /* max element residual                 */
  int64_t bc_worst;     /* its element                          */
  double flux_max;      /* max flux imbalance / q_scale         */
  int64_t flux_worst;   /* its fracture                         */
  double h_scale;       /* head scale of the residual           */
  double q_scale;       /* discharge scale                      */
} AndfnResidual;
int andfn_b200_bc_residual(AndfnHandle *h, double *elem_res, double *frac_flux,
                           AndfnResidual *out);

/* Thread-local text of the last error. */
const char *andfn_b200_last_error(void);
/* Library version string. */
const char *andfn_b200_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ANDFN_B200_H */
