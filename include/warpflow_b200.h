/*
 * warpflow_b200.h -- C ABI of libwfb200.so, the B200 (sm_100a) kernels for
 * the warpflow-les per-step hot path: Heun RK2 stage (4th-order convection,
 * 4th-order variable-viscosity diffusion, WALE, ghost fills) and the
 * fractional-step projection with its red-black Gauss-Seidel multigrid.
 *
 * Conventions
 *   - Every field is a C-contiguous float64 device array of (n+6)^3 doubles
 *     indexed [i][j][k], k fastest, real cells NPL..NPL+n-1 with NPL = 3
 *     (reference kernels.py:9-12, topology.py:15).  Only cubic grids.
 *   - Multigrid level l >= 1 arrays are (n_l+2)^3, n_l = n >> l, one ring.
 *     Level 0 has no arrays of its own: it reads `su` and solves into `pp`
 *     in place.  Element type is double, or float when `mg_fp32` is set.
 *   - All memory is allocated and owned by the caller.  Nothing here calls
 *     cudaMalloc / cudaFree on the step path.  Only the step context keeps
 *     CUDA graph handles.
 *   - Every entry returns 0 on success or a WF_E* code; wf_last_error()
 *     gives a thread-local message.  Launches are asynchronous on `stream`
 *     (a cudaStream_t passed as void*); there are no host syncs inside
 *     except where a function says so.
 *   - Device-detected conditions (dt collapse, divergence, non-convergence)
 *     are written to wf_scalars.status, which the caller reads.
 */
#ifndef WARPFLOW_B200_H
#define WARPFLOW_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define WF_API __attribute__((visibility("default")))
#else
#define WF_API
#endif

#define WF_NPL 3
#define WF_MAX_LEVELS 8
#define WF_NFIELDS 13

/* field slots, in the order of the reference FlowSolver.f (solver.py:43-46) */
enum wf_field {
  WF_U = 0, WF_V, WF_W, WF_P, WF_USTAR, WF_VSTAR, WF_WSTAR,
  WF_UOO, WF_VOO, WF_WOO, WF_VIS, WF_SU, WF_PP
};

enum wf_err {
  WF_OK = 0,
  WF_EINVAL = 1,     /* bad extent / pointer / configuration */
  WF_EUNSUPPORTED = 2,
  WF_ECUDA = 3,      /* a CUDA call or launch failed */
  WF_ESTATUS = 4     /* device status word reports a failure */
};

/* device status word values (wf_scalars.status) */
enum wf_status {
  WF_ST_OK = 0,
  WF_ST_DT_COLLAPSE = 1,   /* solver.py:143-144 */
  WF_ST_DIVERGED = 2,      /* solver.py:190-193 */
  WF_ST_NOT_CONVERGED = 3, /* solver.py:205-209 (warning only) */
  WF_ST_WAIT_TIMEOUT = 4   /* a bounded device-side wait gave up */
};

/* Device-resident scalar block of one case.  The step kernels read dt from
 * here and write every per-step scalar back, so the host reads one small
 * struct per step instead of the reference's 5+ blocking readbacks. */
typedef struct wf_scalars {
  double dt;          /* time step in use (FlowSolver.dt) */
  double ctime;       /* simulated time (FlowSolver.ctime) */
  double rmax;        /* last 4th-order divergence max (FlowSolver.rmax) */
  double cfl;         /* dt_old / dtmax (FlowSolver.cfl) */
  double dtmax;       /* min(dtvisc, dtcfl) of the last checkdt */
  double umax, vmax, wmax, dtvisc;      /* last checkdt reductions */
  double rrey, ulid;  /* 1/Re and lid velocity: the step reads them here, so a built step
                         serves a new case of the same size after wf_scalars_init */
  double rmax_trace[32];                /* rmax of every outer iteration */
  unsigned long long red[6];            /* reduction scratch (bit patterns) */
  int32_t itime;      /* step counter (FlowSolver.itime) */
  int32_t iters;      /* outer iterations of the last step (outer_iters) */
  int32_t status;     /* wf_status */
  int32_t loop;       /* device loop flag of the projection */
  uint32_t ticket;    /* last-block-done counter */
  int32_t nmg;        /* multigrid solves run in the last step */
  uint32_t gbar[2];   /* grid barrier of the persistent relax (count, generation) */
  uint32_t bticket;   /* bucket stepping (first case of a bucket): cases reported */
  int32_t bflags;     /* bucket stepping: OR of the cases' loop decisions */
} wf_scalars;

/* One cavity case: geometry, physics, numerics and the caller's buffers. */
typedef struct wf_case {
  int32_t n;            /* cells per axis */
  int32_t nlev;         /* multigrid levels (config mg_levels) */
  int32_t sgs;          /* WALE on (physics.sgs.enabled) */
  int32_t variable_dt;  /* time.variable_dt */
  int32_t maxcy;        /* numerics.max_outer_iters */
  int32_t mg_fp32;      /* 0: FP64 multigrid, 1: FP32 V-cycle in FP64 defect correction */
  int32_t n_pre, n_post, n_coarse, n_vcycles;   /* multigrid.py:257-260 */
  double dx, dy, dz;    /* cell sizes */
  double rrey;          /* 1/Re */
  double cw;            /* WALE coefficient */
  double ulid;          /* lid velocity */
  double dt_growth, safety, eps;  /* time.dt_growth, time.safety_factor, div_tolerance */
  double* fld[WF_NFIELDS];        /* (n+6)^3 each, order of enum wf_field */
  void* mg_phi[WF_MAX_LEVELS];    /* level l >= 1 (entry 0 unused in FP64) */
  void* mg_rhs[WF_MAX_LEVELS];    /* level l >= 1; in FP32 mode entry 0 is the FP32 level-0 pair */
  void* mg_tmp[WF_MAX_LEVELS];    /* optional scratch of 2*(n_l+2)^3 elements per level
                                     (level 0 included, element type of the level): large
                                     levels relax on row-parity-split copies of phi and rhs
                                     held there; NULL = relax in place */
  wf_scalars* sc;                 /* device scalar block */
  void* mg_cop;                   /* optional coarse-level operator (may be shared
                                     by cases), see wf_mg_build_coarse_op; NULL = sweeps */
  void* mg_cop_part;              /* this case's scratch for it (N/2 elements) */
} wf_case;

/* ---- library ---------------------------------------------------------- */
WF_API int wf_version(void);
WF_API const char* wf_last_error(void);
/* sizeof(wf_scalars), sizeof(wf_case) as compiled, for binding checks */
WF_API int wf_struct_sizes(int64_t* scalars, int64_t* casebytes);
/* solver.py:60-65 initial scalars: dt = dt0, ctime = 0, itime = 0, ...,
 * and the case's 1/Re and lid velocity (sc->rrey, sc->ulid), which the step
 * of wf_stepper_create reads from the block rather than from its wf_case */
WF_API int wf_scalars_init(wf_scalars* sc, double dt0, double rrey, double ulid, void* stream);
/* Tuning knob (no reference counterpart): how a many-sweep relax of an n^3
 * level (n <= 64) runs -- 0 one CTA, 1 cluster with a barrier per
 * half-sweep, 2 cluster with point-to-point halo pushes.  Process-wide;
 * set before graphs are built.  fp32 selects the mixed-precision table. */
WF_API int wf_set_coarse_strategy(int32_t n, int32_t fp32, int32_t strategy);
/* Tuning knob (no reference counterpart): the launch shape of a kernel for
 * size n.  kind 0 = the convection pass (k_conv): a x b threads per CTA, a
 * along k (a power of two), b along j, a*b a multiple of 32 and <= 256,
 * and c consecutive planes i per thread (1..16); default 32 x 8 x 1.
 * kind 1 = the split red-black half-sweep of an n^3 level (k_rbgs_split):
 * a = cells per thread (1, 2, 4), b = rows per CTA (1, 2, 4, 8), c = 1;
 * default 2 x 8 x 1.  a = b = c = 0 restores the default.  Results do not
 * depend on the shape (each cell's arithmetic is the same).  Process-wide;
 * read when a launch is issued, so set it before steppers are built.
 * wf_launch_shape reads the shape in force. */
WF_API int wf_set_launch_shape(int32_t kind, int32_t n, int32_t a, int32_t b, int32_t c);
WF_API int wf_launch_shape(int32_t kind, int32_t n, int32_t* a, int32_t* b, int32_t* c);
/* bytes of MG workspace a case needs at each level (caller allocates) */
WF_API int wf_mg_level_elems(int32_t n, int32_t nlev, int32_t level, int64_t* elems);
/* No counterpart in the reference.  The coarsest-level relax of a V-cycle
 * (multigrid.py:301-322: n_coarse RBGS sweeps starting from phi = 0) is a
 * fixed linear map of the level's rhs.  Every cell neighbours only cells of
 * the other parity of i+j+k, so after the first sweep from zero the
 * even-parity half of phi evolves on its own: after n_coarse - 1 sweeps it
 * is S v, v = the even-parity numerators of the first sweep, S a fixed
 * symmetric (N/2)^2 matrix (N = n_c^3) that commutes with the level's
 * colour-preserving symmetries (axis permutations between axes of equal
 * spacing, reflections of two axes: 24 on a cube).  wf_mg_build_coarse_op
 * stores, for the case's n, nlev, spacing, n_coarse and precision
 * (c->mg_fp32 selects FP32), in c->mg_cop the columns of S at one
 * representative cell of every orbit of those symmetries (about N/48
 * columns of N/2 entries on a cube) followed by an integer table.  With
 * c->mg_cop set, V-cycles run the coarse relax as v, the product S v formed
 * from the stored columns in shared memory, and the last sweep, instead of
 * the latency-bound sweeps; the results agree to rounding.  Coarsest edges
 * 4, 8, 12, 16, 20, 24 and n_coarse >= 2 only (WF_EUNSUPPORTED /
 * WF_EINVAL).  The operator is read-only once built and can be shared by
 * cases of the same size and spacing; each case needs its own scratch of
 * N/2 elements (c->mg_cop_part).  wf_mg_coarse_op_elems gives both element
 * counts (they depend on which spacings are equal). */
WF_API int wf_mg_coarse_op_elems(const wf_case* c, int64_t* op_elems, int64_t* scratch_elems);
WF_API int wf_mg_build_coarse_op(const wf_case* c, void* stream);
/* The coarsest-level solve of a V-cycle (multigrid.py:301-322, coarsest
 * level: phi from zero, n_coarse sweeps) on an explicit FP64 pair of
 * (n_c+2)^3 doubles: through c->mg_cop when it is set, else as sweeps. */
WF_API int wf_mg_coarse_solve(const wf_case* c, double* phi, const double* rhs, void* stream);

/* ---- initial state ---------------------------------------------------- */
/* kernels.py:452-471 init_noise: u = v = amp*r, w = -amp*r (uint32 hash). */
WF_API int wf_init_noise(double* u, double* v, double* w, int32_t n, double amp,
                  int32_t seed, void* stream);
/* bcs.py:313-323 BoundaryKernels.apply: boundu/v/w + full-depth p mirror. */
WF_API int wf_fill_initial(const wf_case* c, void* stream);

/* ---- ghost fills (bcs.py) --------------------------------------------- */
/* bcs.py:201-223 apply_u */
WF_API int wf_fill_u(double* u, int32_t n, double ulid, void* stream);
/* bcs.py:225-244 apply_v */
WF_API int wf_fill_v(double* v, int32_t n, void* stream);
/* bcs.py:246-265 apply_w */
WF_API int wf_fill_w(double* w, int32_t n, void* stream);
/* bcs.py:267-293 apply_vis */
WF_API int wf_fill_vis(double* vis, int32_t n, double rrey, void* stream);
/* bcs.py:295-302 apply_pbound */
WF_API int wf_fill_pbound(double* p, int32_t n, void* stream);
/* bcs.py:304-311 apply_p_mirror */
WF_API int wf_fill_p_mirror(double* p, int32_t n, void* stream);

/* ---- stencil operators (kernels.py) ----------------------------------- */
/* kernels.py:53-168 conv4th_{u,v,w}; comp 0/1/2; dt read from *dt_dev. */
WF_API int wf_conv(const wf_case* c, int32_t comp, double alpha, const double* dt_dev,
            void* stream);
/* kernels.py:189-225 diff4th_{u,v,w} */
WF_API int wf_diff(const wf_case* c, int32_t comp, double alpha, const double* dt_dev,
            void* stream);
/* kernels.py:232-264 calvel_{u,v,w} (all three components, one launch) */
WF_API int wf_calvel(const wf_case* c, double alpha, const double* dt_dev, void* stream);
/* kernels.py:271-289 calmas: su = div/dt, sc->rmax = max|div dV| */
WF_API int wf_calmas(const wf_case* c, void* stream);
/* kernels.py:297-367 wale_viscosity (or kernels.py:442-449 fill_const when
 * sgs is off) followed by bcs.py:267-293 apply_vis. */
WF_API int wf_wale_vis(const wf_case* c, void* stream);
/* solver.py:122-150 compute_dt with kernels.py:374-402: reductions and the
 * dt / cfl update, all on the device; also itime += 1, ctime += dt. */
WF_API int wf_checkdt(const wf_case* c, void* stream);
/* kernels.py:405-414 add_inplace: p += pp over real cells + one ring. */
WF_API int wf_add_ring(double* p, const double* pp, int32_t n, void* stream);

/* ---- multigrid (multigrid.py) ----------------------------------------- */
/* multigrid.py:324-337 Multigrid.solve(su, pp): pp = 4 V-cycles from zero
 * on A pp = su (7-point Neumann, RBGS 6/6/300).  Level 0 works in place in
 * `pp`; level >= 1 buffers come from the case. */
WF_API int wf_mg_solve(const wf_case* c, void* stream);
/* No counterpart in the reference.  The same solve as wf_mg_solve (6/6/300
 * sweeps, 4 V-cycles from zero, pp written in place from su) for callers
 * that cannot allocate device memory -- host codes that hand out every GPU
 * buffer from their own fixed pool or memory budget.  The coarse levels live
 * in a 4 MiB array compiled into the library (held on every GPU that loads
 * it until the process exits), enough for n <= 112 at 3 levels; larger
 * problems return WF_EINVAL.  Nothing is allocated.  The first call in a
 * CUDA context looks up the array's address; make it before any stream
 * capture.  Calls share the array: calls that overlap on the GPU race. */
WF_API int wf_mg_solve_noalloc(const double* su, double* pp, int32_t n, int32_t nlev,
                               double dx, double dy, double dz, void* stream);
/* No counterpart in the reference.  The device status word of the last
 * wf_mg_solve_noalloc call (it clears the word when it starts): waits for
 * `stream`, then *status = WF_ST_OK, or WF_ST_WAIT_TIMEOUT when a bounded
 * device-side wait of its coarse-level kernels gave up (pp is then
 * invalid).  Allocates nothing. */
WF_API int wf_mg_noalloc_status(void* stream, int32_t* status);
/* No counterpart in the reference.  wf_mg_solve for `ncases` cases of the
 * same size and numerics at once: every launch of the solve serves all of
 * them (grids stacked along z), each case computing what wf_mg_solve
 * computes for it alone.  `table` is caller-owned device memory of
 * wf_mg_bucket_table_bytes(ncases) bytes, which receives the cases' buffer
 * pointers (the call waits for that copy, then enqueues the solve). */
WF_API int wf_mg_solve_bucket(const wf_case* cases, int32_t ncases, void* table, void* stream);
WF_API int wf_mg_bucket_table_bytes(int32_t ncases, int64_t* bytes);
/* multigrid.py:301-322 one V-cycle on an explicit level-0 pair (phi, rhs)
 * of (n+2)^3 doubles each (the standalone harness of tests/test_mg.py). */
WF_API int wf_mg_vcycle(const wf_case* c, double* phi0, const double* rhs0, void* stream);
/* multigrid.py:301-322 as an FP64 defect correction around an FP32 V-cycle:
 * r = rhs0 - A phi0 (FP64), e = FP32 V-cycle from zero on A e = r, phi0 += e.
 * FP32 level buffers (level 0 included) come from c->mg_phi / c->mg_rhs. */
WF_API int wf_mg_dc_cycle(const wf_case* c, double* phi0, const double* rhs0, void* stream);
/* multigrid.py:289-299 `nsweeps` RBGS sweeps + ring refill on level 0 pair */
WF_API int wf_mg_relax(const wf_case* c, double* phi0, const double* rhs0,
                int32_t nsweeps, void* stream);
/* tests/test_mg.py:16-32 residual: *out = max|rhs - A phi| over level 0. */
WF_API int wf_mg_residual_max(const wf_case* c, const double* phi0, const double* rhs0,
                       double* out_dev, void* stream);
/* bcs.py:326-360 _mk_neumann on all six faces of a level-0 pair. */
WF_API int wf_mg_refill(const wf_case* c, double* phi0, void* stream);

/* No counterpart in the reference (its fills are ordered face launches,
 * bcs.py:201-323).  The composed one-launch program of a ghost fill, for
 * checking on the host: kind 0 u, 1 v, 2 w, 3 vis, 4 pbound, 5 the initial p
 * mirror; 4 <= n <= 256.  Entries are (dst, code) pairs of offsets into the
 * padded (n+6)^3 field: code bit 0 set = a constant (bits 2.. : 0 for 0.0,
 * 1 for the fill's value), else bits 2.. = the source offset; bit 1 set =
 * negated.  The first nsimple entries are independent gathers; the rest are
 * ngroup groups (entries gstart[g] .. gstart[g+1]-1 after the simple ones),
 * each applied by one thread that reads every source before it writes.
 * Sources always hold the values from before the fill.  Call with null ent
 * and gstart to get the counts (2 * nent ints, ngroup + 1 ints). */
WF_API int wf_fill_program(int32_t kind, int32_t n, int32_t* nsimple, int32_t* ngroup,
                           int64_t* nent, int32_t* ent, int32_t* gstart);

/* ---- sub-domains (more than one rank per case) --------------------------
 * The reference decomposes a case over MPI ranks (topology.py:30-53): each
 * rank steps its own cube of cells, and halo.py:59-130 HaloExchanger.exchange
 * copies ghost slabs between neighbours along x, then y, then z, each slab
 * the full extent of the other two axes (so edge and corner ghosts follow
 * without diagonal messages).  These entries are the device side of that:
 * the host moves the buffers between ranks (NCCL or gloo). */
/* halo.py:16-55 _gather_{x,y,z} (unpack = 0) and _scatter_{x,y,z}
 * (unpack = 1): the box [i0,i0+ni) x [j0,j0+nj) x [k0,k0+nk) of a 3-D
 * array with strides (sI, sJ, 1) to / from a dense buffer ordered
 * [i][j][k]. */
WF_API int wf_box_copy(double* arr, int64_t sI, int64_t sJ, int32_t i0, int32_t j0, int32_t k0,
                       int32_t ni, int32_t nj, int32_t nk, double* buf, int32_t unpack,
                       void* stream);
/* solver.py:222-225: uoo/voo/woo = u/v/w over the whole padded arrays. */
WF_API int wf_copy_oo(const wf_case* c, void* stream);
/* One pass of the reference multigrid at a sub-domain, on level `level` of
 * the case (level 0 = the one-ring core of pp and su, as wf_mg_solve):
 * op 0 one colour half-sweep (multigrid.py:70-90) with the face
 * coefficients of multigrid.py:23-67, zero only across a physical face;
 * op 1 the Neumann mirror of the physical faces (bcs.py:326-360, the
 * mgbound half of multigrid.py:264-287; the seams are the host's exchange);
 * op 2 restriction from level-1 (multigrid.py:93-119) and the coarse phi
 * zeroed (multigrid.py:310-312); op 3 prolongation from level+1 onto the
 * real cells (multigrid.py:122-146); op 4 pp zeroed (multigrid.py:332-333).
 * `phys`: bit f set when face f is physical (0 west, 1 east, 2 south,
 * 3 north, 4 bottom, 5 top). */
WF_API int wf_rk_mg_op(const wf_case* c, int32_t op, int32_t level, int32_t phys,
                       int32_t color, void* stream);
/* Where level `level` of the case lives: the ring cell (0,0,0) of its phi,
 * its strides (k stride 1) and its edge m = n_l + 2. */
WF_API int wf_rk_level_view(const wf_case* c, int32_t level, double** phi, int64_t* sI,
                            int64_t* sJ, int32_t* m);

/* No counterpart in the reference: a check of the library's bounded
 * device-side waits.  One CTA runs one wait that can never complete and
 * must give up after `tries` tries (1 .. 2^22): kind 0 the grid barrier of
 * the cooperative relax (gbar: two zeroed words, declared block count one
 * above the launched one), kind 1 the mbarrier wait of the point-to-point
 * coarse kernels on bytes that nobody sends.  *err (device) receives
 * WF_ST_WAIT_TIMEOUT; the kernel returns with nothing in flight. */
WF_API int wf_wait_probe(uint32_t* gbar, int32_t* err, int32_t kind, int32_t tries,
                         void* stream);

/* ---- whole step (solver.py:217-271) ------------------------------------ */
typedef struct wf_stepper wf_stepper;
/* Build the per-case step as one CUDA graph (device-side dt control and a
 * device-driven projection loop through conditional graph nodes).  `c` is
 * copied.  mode 0 = graph, 1 = plain stream launches with host-driven
 * projection loop (one 8-byte readback per outer iteration).  OR-ing
 * WF_STEP_SERIAL into the mode launches every kernel of the step without
 * programmatic dependent launch: a kernel's CTAs then become resident only
 * after its predecessor finished, which frees SMs for other streams when
 * many steppers run concurrently (ensembles, serving). */
#define WF_STEP_SERIAL 2
WF_API int wf_stepper_create(const wf_case* c, int32_t mode, wf_stepper** out);
/* One FlowSolver.step(): enqueue the step on `stream`.  No host sync. */
WF_API int wf_stepper_step(wf_stepper* s, void* stream);
/* kernel launches per part of the step: prologue, one projection-loop
 * pass (calmas), one multigrid part, epilogue */
WF_API int wf_stepper_launch_counts(const wf_stepper* s, int32_t counts[4]);
WF_API int wf_stepper_destroy(wf_stepper* s);

/* No counterpart in the reference (its cases run one at a time).  Many
 * independent cases stepped by ONE graph launch: wf_ensemble_create appends
 * every case's step (as wf_stepper_create builds it) to a single CUDA graph
 * as independent branches, so the device schedules all cases' kernels
 * concurrently without a stream per case.  `cases` are copied; mode 0 or
 * WF_STEP_SERIAL, optionally | WF_ENS_BUCKETS: cases of the same size and
 * numerics (any Re and lid velocity; the same shared coarse operator) then
 * form buckets, and each bucket is ONE branch whose every kernel launch
 * serves all its cases (grids stacked along z, a device table of the cases'
 * buffers allocated at creation and freed by wf_ensemble_destroy); the
 * bucket's projection loop runs while any of its cases' loops does, each
 * case's multigrid part only while its own loop runs it, so every case
 * computes what it computes alone.  wf_ensemble_step enqueues one step of
 * every case; read each case's scalar block after the stream finishes.
 * wf_ensemble_layout gives the bucket count (the case count without
 * buckets), each case's bucket (-1 without buckets) and 4 launch counts
 * per bucket or case (prologue, calmas pass, multigrid part, epilogue).
 * A bucket holds at most wf_bucket_cap(n, mg_fp32) cases of its size: by
 * default as many as keep their finest multigrid level within half the L2
 * (and the stacked grid within the z limit); wf_set_bucket_cap(n, fp32,
 * cap) overrides it per size (1 = a branch per case, 0 restores the
 * default; process-wide, read when an ensemble is created).  Buckets pay
 * for ensembles of one size; for a mix of sizes a branch per case (mode
 * without WF_ENS_BUCKETS) measured faster on B200. */
#define WF_ENS_BUCKETS 4
WF_API int wf_set_bucket_cap(int32_t n, int32_t fp32, int32_t cap);
WF_API int wf_bucket_cap(int32_t n, int32_t fp32, int32_t* cap);
typedef struct wf_ensemble wf_ensemble;
WF_API int wf_ensemble_create(const wf_case* cases, int32_t ncases, int32_t mode,
                              wf_ensemble** out);
WF_API int wf_ensemble_layout(const wf_ensemble* e, int32_t* nbuckets, int32_t* bucket_of_case,
                              int32_t* counts);
WF_API int wf_ensemble_step(wf_ensemble* e, void* stream);
WF_API int wf_ensemble_destroy(wf_ensemble* e);

#ifdef __cplusplus
}
#endif
#endif /* WARPFLOW_B200_H */
