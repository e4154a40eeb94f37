// One FlowSolver.step() (reference solver.py:217-271) on the device, the
// C ABI entry points, and error plumbing.
//
// Step layout (launch order follows solver.py exactly):
//   prologue : checkdt -> uoo/voo/woo copy -> WALE + vis fill ->
//              2 x RK stage (fill + convection-diffusion per component,
//              fill u,v,w, calvel(0.5) after stage 1) -> calvel(1.0)
//   loop     : calmas + control  [if run] MG solve, p += pp, pbound,
//              calvel(1.0)  -- repeated while the control says so
//   epilogue : fill u, v, w
// In graph mode the loop is a conditional WHILE node whose body holds the
// calmas kernel and a conditional IF node for the multigrid part; the
// calmas kernel's last block sets both conditions on the device, so a
// whole step is one graph launch with no host round trip.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "wf_internal.h"

namespace wf {

static thread_local std::string g_err;
thread_local long g_launches = 0;
// Set while a stepper created with WF_STEP_SERIAL captures or launches.
static thread_local int g_pdl_off = 0;

bool pdl_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("WF_PDL");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1 && !g_pdl_off;
}

BatchCtx& batch_ctx() {
  static thread_local BatchCtx ctx;
  return ctx;
}

// Launches of this thread serve the bucket `tab` (ncases cases) for one
// scope; tab null = one case.
struct BatchScope {
  BatchCtx prev;
  BatchScope(const CasePtrs* tab, int ncases, int skip) : prev(batch_ctx()) {
    batch_ctx().tab = tab;
    batch_ctx().ncases = tab ? ncases : 1;
    batch_ctx().skip = tab ? skip : 0;
  }
  ~BatchScope() { batch_ctx() = prev; }
};

// Turns programmatic dependent launch off on this thread for one scope.
struct PdlOff {
  int prev;
  explicit PdlOff(bool on) : prev(g_pdl_off) { if (on) g_pdl_off = 1; }
  ~PdlOff() { g_pdl_off = prev; }
};

void set_error(const std::string& msg) { g_err = msg; }
int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return WF_ECUDA;
}

int validate_case(const wf_case& c) {
  if (c.n < 4) return fail(WF_EINVAL, "n must be >= 4");
  if (c.nlev < 1 || c.nlev > WF_MAX_LEVELS) return fail(WF_EINVAL, "mg_levels out of range");
  if (c.n % (1 << (c.nlev - 1)) != 0)
    return fail(WF_EINVAL, "n must be divisible by 2**(mg_levels-1)");
  for (int f = 0; f < WF_NFIELDS; ++f)
    if (!c.fld[f]) return fail(WF_EINVAL, "null field pointer");
  if (!c.sc) return fail(WF_EINVAL, "null scalar block");
  for (int l = 1; l < c.nlev; ++l)
    if (!c.mg_phi[l] || !c.mg_rhs[l]) return fail(WF_EINVAL, "missing multigrid level buffer");
  if (c.mg_fp32 && (!c.mg_phi[0] || !c.mg_rhs[0]))
    return fail(WF_EINVAL, "mixed precision needs FP32 level-0 buffers");
  if (c.maxcy < 1 || c.maxcy > 32) return fail(WF_EINVAL, "max_outer_iters must be 1..32");
  if (c.dx <= 0 || c.dy <= 0 || c.dz <= 0) return fail(WF_EINVAL, "cell sizes must be > 0");
  if (c.n_pre < 0 || c.n_post < 0 || c.n_coarse < 0 || c.n_vcycles < 0)
    return fail(WF_EINVAL, "negative sweep count");
  return WF_OK;
}

// The step reads 1/Re and the lid velocity from the case's scalar block
// (wf_scalars_init writes them), so that a built step can serve a new case
// of the same size without being rebuilt.
static int fill_comp(const wf_case& c, int comp, cudaStream_t s) {
  FillReq r{c.fld[WF_U + comp], comp == 0 ? FILL_U : (comp == 1 ? FILL_V : FILL_W), c.ulid,
            comp == 0 ? &c.sc->ulid : nullptr, WF_U + comp, comp == 0 ? 1 : 0};
  return launch_fills(&r, 1, c.n, s);
}

static int fill_uvw(const wf_case& c, cudaStream_t s) {
  FillReq r[3] = {{c.fld[WF_U], FILL_U, c.ulid, &c.sc->ulid, WF_U, 1},
                  {c.fld[WF_V], FILL_V, 0.0, nullptr, WF_V, 0},
                  {c.fld[WF_W], FILL_W, 0.0, nullptr, WF_W, 0}};
  return launch_fills(r, 3, c.n, s);
}

static int step_prologue(const wf_case& c, cudaStream_t s) {
  WF_TRY(launch_checkdt(c, s));
  WF_TRY(launch_copy_oo(c, s));
  WF_TRY(launch_wale(c, s, &c.sc->rrey));
  const double* dt = &c.sc->dt;
  const double alfark[2] = {0.5, 1.0};  // solver.py:26
  for (int st = 0; st < 2; ++st) {
    // each component's diffusion runs inside its convection pass (k_conv
    // with DIFF: the fill between them changes no cell the diffusion reads)
    for (int comp = 0; comp < 3; ++comp) {
      WF_TRY(fill_comp(c, comp, s));
      WF_TRY(launch_conv(c, comp, alfark[st], dt, s, true));
    }
    // the fills solver.py:258-263 runs before each diffusion still set the
    // ghost edges and corners that later fills read
    WF_TRY(fill_uvw(c, s));
    if (st == 0) WF_TRY(launch_calvel(c, alfark[st], dt, s));
  }
  return launch_calvel(c, 1.0, dt, s);
}

static int step_mg_part(const wf_case& c, cudaStream_t s) {
  WF_TRY(mg_solve(c, s));
  WF_TRY(launch_add_ring(c.fld[WF_P], c.fld[WF_PP], c.n, s));
  FillReq r{c.fld[WF_P], FILL_PBOUND, 0.0, nullptr, WF_P, 0};
  WF_TRY(launch_fills(&r, 1, c.n, s));
  return launch_calvel(c, 1.0, &c.sc->dt, s);
}

static int step_epilogue(const wf_case& c, cudaStream_t s) { return fill_uvw(c, s); }

}  // namespace wf

using namespace wf;

struct wf_stepper {
  wf_case c;
  int mode;     // 0 graph, 1 host loop
  int serial;   // WF_STEP_SERIAL: no programmatic dependent launch
  int32_t counts[4];  // launches: prologue, calmas pass, multigrid part, epilogue
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  int32_t* hflag;  // pinned, host-loop mode
};

// Append one case's step to graph g as an independent branch (its first
// nodes have no dependencies): the prologue, a WHILE node over calmas and
// an IF node holding the multigrid part, then the epilogue.  counts gets the
// launches of each part.  With `tab` (ncases rows, c = the first case) the
// branch steps the whole bucket: every launch serves every case, the
// multigrid part only the cases whose own loop runs it this iteration, and
// the loop runs while any case's loop does.
static int append_step(cudaGraph_t g, const wf_case& c, int32_t counts[4],
                       const CasePtrs* tab = nullptr, int ncases = 1) {
  cudaStream_t cap;
  WF_CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  int rc = WF_OK;
  do {
    cudaGraphConditionalHandle h_loop;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h_loop, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) { rc = cuda_fail(e, "cudaGraphConditionalHandleCreate(loop)"); break; }
    e = cudaStreamBeginCaptureToGraph(cap, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { rc = cuda_fail(e, "cudaStreamBeginCaptureToGraph"); break; }
    long l0 = g_launches;
    {
      BatchScope bs(tab, ncases, 0);
      rc = step_prologue(c, cap);
    }
    counts[0] = (int32_t)(g_launches - l0);
    cudaGraphNode_t wnode = nullptr;
    cudaGraph_t wbody = nullptr;
    if (rc == WF_OK) {
      cudaStreamCaptureStatus cst;
      const cudaGraphNode_t* deps = nullptr;
      size_t ndeps = 0;
      e = cudaStreamGetCaptureInfo(cap, &cst, nullptr, nullptr, &deps, &ndeps);
      if (e != cudaSuccess) rc = cuda_fail(e, "cudaStreamGetCaptureInfo");
      if (rc == WF_OK) {
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = h_loop;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&wnode, g, deps, ndeps, &cp);
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaGraphAddNode(while)");
        else wbody = cp.conditional.phGraph_out[0];
      }
      if (rc == WF_OK) {
        e = cudaStreamUpdateCaptureDependencies(cap, &wnode, 1, cudaStreamSetCaptureDependencies);
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaStreamUpdateCaptureDependencies");
      }
      l0 = g_launches;
      if (rc == WF_OK) {
        BatchScope bs(tab, ncases, 0);
        rc = step_epilogue(c, cap);
      }
      counts[3] = (int32_t)(g_launches - l0);
    }
    cudaGraph_t gout = nullptr;
    e = cudaStreamEndCapture(cap, &gout);
    if (rc == WF_OK && e != cudaSuccess) rc = cuda_fail(e, "cudaStreamEndCapture(step)");
    if (rc != WF_OK) break;

    // while body: calmas + control, then IF(run) multigrid part
    cudaGraphConditionalHandle h_if;
    e = cudaGraphConditionalHandleCreate(&h_if, wbody, 0, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) { rc = cuda_fail(e, "cudaGraphConditionalHandleCreate(if)"); break; }
    e = cudaStreamBeginCaptureToGraph(cap, wbody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { rc = cuda_fail(e, "cudaStreamBeginCaptureToGraph(while)"); break; }
    l0 = g_launches;
    {
      BatchScope bs(tab, ncases, 0);
      rc = launch_calmas(c, (unsigned long long)h_if, (unsigned long long)h_loop, cap);
    }
    counts[1] = (int32_t)(g_launches - l0);
    cudaGraph_t ibody = nullptr;
    if (rc == WF_OK) {
      cudaStreamCaptureStatus cst;
      const cudaGraphNode_t* deps = nullptr;
      size_t ndeps = 0;
      e = cudaStreamGetCaptureInfo(cap, &cst, nullptr, nullptr, &deps, &ndeps);
      if (e != cudaSuccess) rc = cuda_fail(e, "cudaStreamGetCaptureInfo(while)");
      cudaGraphNode_t inode = nullptr;
      if (rc == WF_OK) {
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = h_if;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&inode, wbody, deps, ndeps, &cp);
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaGraphAddNode(if)");
        else ibody = cp.conditional.phGraph_out[0];
      }
      if (rc == WF_OK) {
        e = cudaStreamUpdateCaptureDependencies(cap, &inode, 1, cudaStreamSetCaptureDependencies);
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaStreamUpdateCaptureDependencies(while)");
      }
    }
    e = cudaStreamEndCapture(cap, &gout);
    if (rc == WF_OK && e != cudaSuccess) rc = cuda_fail(e, "cudaStreamEndCapture(while)");
    if (rc != WF_OK) break;

    e = cudaStreamBeginCaptureToGraph(cap, ibody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { rc = cuda_fail(e, "cudaStreamBeginCaptureToGraph(if)"); break; }
    l0 = g_launches;
    {
      BatchScope bs(tab, ncases, 2);   // only cases whose loop runs the multigrid part
      rc = step_mg_part(c, cap);
    }
    counts[2] = (int32_t)(g_launches - l0);
    e = cudaStreamEndCapture(cap, &gout);
    if (rc == WF_OK && e != cudaSuccess) rc = cuda_fail(e, "cudaStreamEndCapture(if)");
    if (rc != WF_OK) break;

  } while (0);
  cudaStreamDestroy(cap);
  return rc;
}

static int build_graph(wf_stepper* st) {
  cudaGraph_t g = nullptr;
  WF_CK(cudaGraphCreate(&g, 0));
  int rc = append_step(g, st->c, st->counts);
  if (rc == WF_OK) {
    const cudaError_t e = cudaGraphInstantiate(&st->exec, g, 0);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaGraphInstantiate(step)");
  }
  if (rc == WF_OK) st->graph = g;
  else cudaGraphDestroy(g);
  return rc;
}

struct wf_ensemble {
  int ncases;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  std::vector<void*> tables;            // device pointer tables of the buckets
  std::vector<int32_t> bucket_of_case;  // -1 without buckets
  std::vector<int32_t> counts;          // 4 per bucket (or per case)
};

// Cases that can share a bucket: the same size, numerics and physics flags
// (1/Re and the lid velocity are read from each case's scalar block), the
// same shared coarse operator, and the same optional buffers present.
static bool same_bucket(const wf_case& a, const wf_case& b) {
  if (a.n != b.n || a.nlev != b.nlev || a.sgs != b.sgs || a.variable_dt != b.variable_dt ||
      a.maxcy != b.maxcy || a.mg_fp32 != b.mg_fp32 || a.n_pre != b.n_pre ||
      a.n_post != b.n_post || a.n_coarse != b.n_coarse || a.n_vcycles != b.n_vcycles)
    return false;
  if (a.dx != b.dx || a.dy != b.dy || a.dz != b.dz || a.cw != b.cw ||
      a.dt_growth != b.dt_growth || a.safety != b.safety || a.eps != b.eps)
    return false;
  if (a.mg_cop != b.mg_cop || (a.mg_cop_part == nullptr) != (b.mg_cop_part == nullptr))
    return false;
  for (int l = 0; l < WF_MAX_LEVELS; ++l)
    if ((a.mg_tmp[l] == nullptr) != (b.mg_tmp[l] == nullptr)) return false;
  return true;
}

// Largest bucket for cases of size n (per precision of their multigrid).
// 0 in the table means the built-in rule: a bucket's grids stack its cases
// along z (< 65536), and its cases' finest multigrid level (phi and rhs)
// should fit in about half the L2 (64 MB), so the half-sweeps, which
// dominate a step, keep the bucket's level resident across launches.
// Measured on B200 with 13 equal mixed-precision cases per size, one bucket
// against a branch per case (ms per ensemble step): 32^3 1.07 vs 1.84,
// 48^3 2.45 vs 3.29, 64^3 3.88 vs 4.44, 80^3 8.49 vs 8.94, 96^3 12.49 vs
// 12.61.  wf_set_bucket_cap overrides the rule per size (the autotuner's
// measurement).
static constexpr int BUCKET_MAX_N = 1024;
static int g_bucket_cap[2][BUCKET_MAX_N + 1];

static int bucket_cap(const wf_case& c) {
  const int set = (c.n >= 0 && c.n <= BUCKET_MAX_N) ? g_bucket_cap[c.mg_fp32 ? 1 : 0][c.n] : 0;
  if (set > 0) return std::min(set, std::max(1, 60000 / (c.n + 2 * NPL)));
  const long m = c.n + 2;
  const long lvl_bytes = 2 * m * m * m * (c.mg_fp32 ? 4 : 8);
  return (int)std::max(1L, std::min(60000L / (c.n + 2 * NPL), (64L << 20) / lvl_bytes));
}

static CasePtrs ptrs_of(const wf_case& c) {
  CasePtrs p{};
  for (int f = 0; f < WF_NFIELDS; ++f) p.fld[f] = c.fld[f];
  p.sc = c.sc;
  for (int l = 0; l < WF_MAX_LEVELS; ++l) {
    p.mg_phi[l] = c.mg_phi[l];
    p.mg_rhs[l] = c.mg_rhs[l];
    p.mg_tmp[l] = c.mg_tmp[l];
  }
  p.mg_cop_part = c.mg_cop_part;
  return p;
}

extern "C" {

int wf_version(void) { return 100; }

const char* wf_last_error(void) { return g_err.c_str(); }

int wf_struct_sizes(int64_t* scalars, int64_t* casebytes) {
  if (scalars) *scalars = (int64_t)sizeof(wf_scalars);
  if (casebytes) *casebytes = (int64_t)sizeof(wf_case);
  return WF_OK;
}

int wf_set_coarse_strategy(int32_t n, int32_t fp32, int32_t strategy) {
  return set_coarse_strategy(n, fp32, strategy);
}

int wf_set_launch_shape(int32_t kind, int32_t n, int32_t a, int32_t b, int32_t c) {
  return set_launch_shape(kind, n, a, b, c);
}

int wf_launch_shape(int32_t kind, int32_t n, int32_t* a, int32_t* b, int32_t* c) {
  if (!a || !b || !c || (kind != SHAPE_CONV && kind != SHAPE_SPLIT))
    return fail(WF_EINVAL, "wf_launch_shape: kind 0 or 1, non-null outputs");
  int x, y, z;
  launch_shape(kind, n, &x, &y, &z);
  *a = x;
  *b = y;
  *c = z;
  return WF_OK;
}

int wf_set_bucket_cap(int32_t n, int32_t fp32, int32_t cap) {
  if (n < 4 || n > BUCKET_MAX_N || cap < 0)
    return fail(WF_EINVAL, "wf_set_bucket_cap: n in 4..1024, cap >= 0");
  g_bucket_cap[fp32 ? 1 : 0][n] = cap;
  return WF_OK;
}

int wf_bucket_cap(int32_t n, int32_t fp32, int32_t* cap) {
  if (!cap || n < 4 || n > BUCKET_MAX_N) return fail(WF_EINVAL, "wf_bucket_cap: n in 4..1024");
  wf_case c{};
  c.n = n;
  c.mg_fp32 = fp32 ? 1 : 0;
  *cap = bucket_cap(c);
  return WF_OK;
}

int wf_mg_level_elems(int32_t n, int32_t nlev, int32_t level, int64_t* elems) {
  if (!elems || level < 0 || level >= nlev || nlev > WF_MAX_LEVELS)
    return fail(WF_EINVAL, "wf_mg_level_elems: bad level");
  const int64_t m = (int64_t)(n >> level) + 2;
  *elems = m * m * m;
  return WF_OK;
}

int wf_scalars_init(wf_scalars* sc, double dt0, double rrey, double ulid, void* stream) {
  return launch_scalars_init(sc, dt0, rrey, ulid, (cudaStream_t)stream);
}

int wf_init_noise(double* u, double* v, double* w, int32_t n, double amp, int32_t seed,
                  void* stream) {
  return launch_init_noise(u, v, w, n, amp, seed, (cudaStream_t)stream);
}

int wf_fill_initial(const wf_case* c, void* stream) {
  if (!c) return fail(WF_EINVAL, "null case");
  cudaStream_t s = (cudaStream_t)stream;
  FillReq r[3] = {{c->fld[WF_U], FILL_U, c->ulid}, {c->fld[WF_V], FILL_V, 0.0},
                  {c->fld[WF_W], FILL_W, 0.0}};
  WF_TRY(launch_fills(r, 3, c->n, s));
  FillReq p{c->fld[WF_P], FILL_PMIRROR, 0.0};
  return launch_fills(&p, 1, c->n, s);
}

static int fill_one(double* f, int kind, double val, int32_t n, void* stream) {
  FillReq r{f, kind, val};
  return launch_fills(&r, 1, n, (cudaStream_t)stream);
}
int wf_fill_u(double* u, int32_t n, double ulid, void* s) { return fill_one(u, FILL_U, ulid, n, s); }
int wf_fill_v(double* v, int32_t n, void* s) { return fill_one(v, FILL_V, 0.0, n, s); }
int wf_fill_w(double* w, int32_t n, void* s) { return fill_one(w, FILL_W, 0.0, n, s); }
int wf_fill_vis(double* vis, int32_t n, double rrey, void* s) {
  return fill_one(vis, FILL_VIS, rrey, n, s);
}
int wf_fill_pbound(double* p, int32_t n, void* s) { return fill_one(p, FILL_PBOUND, 0.0, n, s); }
int wf_fill_p_mirror(double* p, int32_t n, void* s) {
  return fill_one(p, FILL_PMIRROR, 0.0, n, s);
}

int wf_conv(const wf_case* c, int32_t comp, double alpha, const double* dt, void* s) {
  if (!c || !dt) return fail(WF_EINVAL, "null argument");
  return launch_conv(*c, comp, alpha, dt, (cudaStream_t)s);
}
int wf_diff(const wf_case* c, int32_t comp, double alpha, const double* dt, void* s) {
  if (!c || !dt) return fail(WF_EINVAL, "null argument");
  return launch_diff(*c, comp, alpha, dt, (cudaStream_t)s);
}
int wf_calvel(const wf_case* c, double alpha, const double* dt, void* s) {
  if (!c || !dt) return fail(WF_EINVAL, "null argument");
  return launch_calvel(*c, alpha, dt, (cudaStream_t)s);
}
int wf_calmas(const wf_case* c, void* s) {
  if (!c) return fail(WF_EINVAL, "null case");
  return launch_calmas(*c, 0, 0, (cudaStream_t)s);
}
int wf_wale_vis(const wf_case* c, void* s) {
  if (!c) return fail(WF_EINVAL, "null case");
  return launch_wale(*c, (cudaStream_t)s);
}
int wf_checkdt(const wf_case* c, void* s) {
  if (!c) return fail(WF_EINVAL, "null case");
  return launch_checkdt(*c, (cudaStream_t)s);
}
int wf_add_ring(double* p, const double* pp, int32_t n, void* s) {
  if (!p || !pp) return fail(WF_EINVAL, "null field");
  return launch_add_ring(p, pp, n, (cudaStream_t)s);
}

int wf_mg_solve(const wf_case* c, void* s) {
  if (!c) return fail(WF_EINVAL, "null case");
  WF_TRY(validate_case(*c));
  return mg_solve(*c, (cudaStream_t)s);
}
int wf_mg_solve_noalloc(const double* su, double* pp, int32_t n, int32_t nlev, double dx,
                        double dy, double dz, void* s) {
  return mg_solve_noalloc(su, pp, n, nlev, dx, dy, dz, (cudaStream_t)s);
}
int wf_mg_noalloc_status(void* s, int32_t* status) { return mg_noalloc_status(s, status); }
int wf_wait_probe(uint32_t* gbar, int32_t* err, int32_t kind, int32_t tries, void* s) {
  return wait_probe(gbar, err, kind, tries, (cudaStream_t)s);
}
int wf_mg_vcycle(const wf_case* c, double* phi0, const double* rhs0, void* s) {
  if (!c || !phi0 || !rhs0) return fail(WF_EINVAL, "null argument");
  return mg_vcycle_pair(*c, phi0, rhs0, (cudaStream_t)s);
}
int wf_mg_dc_cycle(const wf_case* c, double* phi0, const double* rhs0, void* s) {
  if (!c || !phi0 || !rhs0) return fail(WF_EINVAL, "null argument");
  return mg_dc_cycle_pair(*c, phi0, rhs0, (cudaStream_t)s);
}
int wf_mg_relax(const wf_case* c, double* phi0, const double* rhs0, int32_t nsweeps, void* s) {
  if (!c || !phi0 || !rhs0) return fail(WF_EINVAL, "null argument");
  return mg_relax_pair(*c, phi0, rhs0, nsweeps, (cudaStream_t)s);
}
int wf_mg_residual_max(const wf_case* c, const double* phi0, const double* rhs0, double* out,
                       void* s) {
  if (!c || !phi0 || !rhs0 || !out) return fail(WF_EINVAL, "null argument");
  return mg_residual_max_pair(*c, phi0, rhs0, out, (cudaStream_t)s);
}
int wf_mg_coarse_op_elems(const wf_case* c, int64_t* op_elems, int64_t* scratch_elems) {
  if (!c) return fail(WF_EINVAL, "null case");
  return coarse_op_elems(*c, op_elems, scratch_elems);
}

int wf_mg_coarse_solve(const wf_case* c, double* phi, const double* rhs, void* s) {
  if (!c || !phi || !rhs) return fail(WF_EINVAL, "null argument");
  return mg_coarse_solve_pair(*c, phi, rhs, (cudaStream_t)s);
}

int wf_mg_build_coarse_op(const wf_case* c, void* s) {
  if (!c) return fail(WF_EINVAL, "null argument");
  return build_coarse_op_case(*c, (cudaStream_t)s);
}

int wf_fill_program(int32_t kind, int32_t n, int32_t* nsimple, int32_t* ngroup, int64_t* nent,
                    int32_t* ent, int32_t* gstart) {
  if (!nsimple || !ngroup || !nent) return fail(WF_EINVAL, "null argument");
  return fill_program(kind, n, nsimple, ngroup, nent, ent, gstart);
}
int wf_box_copy(double* arr, int64_t sI, int64_t sJ, int32_t i0, int32_t j0, int32_t k0,
                int32_t ni, int32_t nj, int32_t nk, double* buf, int32_t unpack, void* s) {
  return launch_box(arr, sI, sJ, i0, j0, k0, ni, nj, nk, buf, unpack ? 1 : 0, (cudaStream_t)s);
}
int wf_copy_oo(const wf_case* c, void* s) {
  if (!c) return fail(WF_EINVAL, "null case");
  for (int f : {WF_U, WF_V, WF_W, WF_UOO, WF_VOO, WF_WOO})
    if (!c->fld[f]) return fail(WF_EINVAL, "null field pointer");
  return launch_copy_oo(*c, (cudaStream_t)s);
}
int wf_rk_mg_op(const wf_case* c, int32_t op, int32_t level, int32_t phys, int32_t color,
                void* s) {
  if (!c) return fail(WF_EINVAL, "null case");
  return rk_mg_op(*c, op, level, phys, color, (cudaStream_t)s);
}
int wf_rk_level_view(const wf_case* c, int32_t level, double** phi, int64_t* sI, int64_t* sJ,
                     int32_t* m) {
  if (!c || !phi || !sI || !sJ || !m) return fail(WF_EINVAL, "null argument");
  return rk_level_view(*c, level, phi, sI, sJ, m);
}

int wf_mg_refill(const wf_case* c, double* phi0, void* s) {
  if (!c || !phi0) return fail(WF_EINVAL, "null argument");
  return mg_refill_pair(*c, phi0, (cudaStream_t)s);
}

int wf_stepper_create(const wf_case* c, int32_t mode, wf_stepper** out) {
  if (!c || !out) return fail(WF_EINVAL, "null argument");
  *out = nullptr;
  WF_TRY(validate_case(*c));
  if (mode & ~(1 | WF_STEP_SERIAL))
    return fail(WF_EINVAL, "mode must be 0 (graph) or 1 (host loop), optionally | WF_STEP_SERIAL");
  prepare_fills(c->n);   // the fill programs are built outside the capture
  wf_stepper* st = new wf_stepper();
  st->c = *c;
  st->mode = mode & 1;
  st->serial = (mode & WF_STEP_SERIAL) != 0;
  PdlOff guard(st->serial);
  st->graph = nullptr;
  st->exec = nullptr;
  st->hflag = nullptr;
  for (int i = 0; i < 4; ++i) st->counts[i] = 0;
  int rc = WF_OK;
  if (st->mode == 0) {
    rc = build_graph(st);
  } else {
    cudaError_t e = cudaMallocHost((void**)&st->hflag, sizeof(int32_t));
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMallocHost");
  }
  if (rc != WF_OK) {
    wf_stepper_destroy(st);
    return rc;
  }
  *out = st;
  return WF_OK;
}

int wf_stepper_step(wf_stepper* st, void* stream) {
  if (!st) return fail(WF_EINVAL, "null stepper");
  cudaStream_t s = (cudaStream_t)stream;
  if (st->mode == 0) {
    WF_CK(cudaGraphLaunch(st->exec, s));
    return WF_OK;
  }
  const wf_case& c = st->c;
  PdlOff guard(st->serial);
  long l0 = g_launches;
  WF_TRY(step_prologue(c, s));
  st->counts[0] = (int32_t)(g_launches - l0);
  for (int it = 0; it < 64; ++it) {
    l0 = g_launches;
    WF_TRY(launch_calmas(c, 0, 0, s));
    st->counts[1] = (int32_t)(g_launches - l0);
    WF_CK(cudaMemcpyAsync(st->hflag, &c.sc->loop, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    WF_CK(cudaStreamSynchronize(s));
    const int32_t f = *st->hflag;
    if (f & 2) {
      l0 = g_launches;
      WF_TRY(step_mg_part(c, s));
      st->counts[2] = (int32_t)(g_launches - l0);
    }
    if (!(f & 1)) break;
  }
  l0 = g_launches;
  WF_TRY(step_epilogue(c, s));
  st->counts[3] = (int32_t)(g_launches - l0);
  return WF_OK;
}

int wf_ensemble_create(const wf_case* cases, int32_t ncases, int32_t mode, wf_ensemble** out) {
  if (!cases || !out || ncases < 1) return fail(WF_EINVAL, "null argument or no cases");
  *out = nullptr;
  if (mode & ~(WF_STEP_SERIAL | WF_ENS_BUCKETS))
    return fail(WF_EINVAL, "ensemble mode: 0, WF_STEP_SERIAL and/or WF_ENS_BUCKETS");
  for (int i = 0; i < ncases; ++i) WF_TRY(validate_case(cases[i]));
  for (int i = 0; i < ncases; ++i) prepare_fills(cases[i].n);
  PdlOff guard((mode & WF_STEP_SERIAL) != 0);
  wf_ensemble* en = new wf_ensemble();
  en->ncases = ncases;
  en->graph = nullptr;
  en->exec = nullptr;
  en->bucket_of_case.assign(ncases, -1);
  cudaError_t e = cudaGraphCreate(&en->graph, 0);
  if (e != cudaSuccess) {
    delete en;
    return cuda_fail(e, "cudaGraphCreate(ensemble)");
  }
  int rc = WF_OK;
  if (mode & WF_ENS_BUCKETS) {
    // group the cases, at most bucket_cap(case) to a bucket
    std::vector<std::vector<int>> buckets;
    for (int i = 0; i < ncases; ++i) {
      const int cap = bucket_cap(cases[i]);
      bool placed = false;
      for (auto& b : buckets)
        if ((int)b.size() < cap && same_bucket(cases[b[0]], cases[i])) {
          b.push_back(i);
          placed = true;
          break;
        }
      if (!placed) buckets.push_back({i});
    }
    for (size_t bi = 0; bi < buckets.size() && rc == WF_OK; ++bi) {
      const auto& b = buckets[bi];
      std::vector<CasePtrs> rows;
      for (int i : b) {
        rows.push_back(ptrs_of(cases[i]));
        en->bucket_of_case[i] = (int32_t)bi;
      }
      void* tab = nullptr;
      e = cudaMalloc(&tab, rows.size() * sizeof(CasePtrs));
      if (e != cudaSuccess) { rc = cuda_fail(e, "cudaMalloc(bucket table)"); break; }
      en->tables.push_back(tab);
      e = cudaMemcpy(tab, rows.data(), rows.size() * sizeof(CasePtrs), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) { rc = cuda_fail(e, "cudaMemcpy(bucket table)"); break; }
      int32_t counts[4] = {0, 0, 0, 0};
      rc = append_step(en->graph, cases[b[0]], counts, (const CasePtrs*)tab, (int)b.size());
      en->counts.insert(en->counts.end(), counts, counts + 4);
    }
  } else {
    for (int i = 0; i < ncases && rc == WF_OK; ++i) {
      int32_t counts[4] = {0, 0, 0, 0};
      rc = append_step(en->graph, cases[i], counts);
      en->counts.insert(en->counts.end(), counts, counts + 4);
    }
  }
  if (rc == WF_OK) {
    e = cudaGraphInstantiate(&en->exec, en->graph, 0);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaGraphInstantiate(ensemble)");
  }
  if (rc != WF_OK) {
    wf_ensemble_destroy(en);
    return rc;
  }
  *out = en;
  return WF_OK;
}

int wf_mg_solve_bucket(const wf_case* cases, int32_t ncases, void* table, void* stream) {
  if (!cases || ncases < 1 || !table) return fail(WF_EINVAL, "null argument or no cases");
  if (ncases > std::max(1, 60000 / (cases[0].n + 2 * NPL)))
    return fail(WF_EINVAL, "wf_mg_solve_bucket: too many cases for one launch");
  for (int i = 0; i < ncases; ++i) {
    WF_TRY(validate_case(cases[i]));
    if (!same_bucket(cases[0], cases[i]))
      return fail(WF_EINVAL, "wf_mg_solve_bucket: the cases differ in size or numerics");
  }
  std::vector<CasePtrs> rows;
  for (int i = 0; i < ncases; ++i) rows.push_back(ptrs_of(cases[i]));
  cudaStream_t s = (cudaStream_t)stream;
  WF_CK(cudaMemcpyAsync(table, rows.data(), rows.size() * sizeof(CasePtrs),
                        cudaMemcpyHostToDevice, s));
  WF_CK(cudaStreamSynchronize(s));   // the rows live on this thread's stack
  BatchScope bs((const CasePtrs*)table, ncases, 0);
  return mg_solve(cases[0], s);
}

int wf_mg_bucket_table_bytes(int32_t ncases, int64_t* bytes) {
  if (!bytes || ncases < 1) return fail(WF_EINVAL, "null argument or no cases");
  *bytes = (int64_t)ncases * (int64_t)sizeof(CasePtrs);
  return WF_OK;
}

int wf_ensemble_layout(const wf_ensemble* en, int32_t* nbuckets, int32_t* bucket_of_case,
                       int32_t* counts) {
  if (!en || !nbuckets) return fail(WF_EINVAL, "null argument");
  const int nb = en->tables.empty() ? en->ncases : (int)en->tables.size();
  *nbuckets = nb;
  if (bucket_of_case)
    for (int i = 0; i < en->ncases; ++i) bucket_of_case[i] = en->bucket_of_case[i];
  if (counts)
    for (size_t i = 0; i < en->counts.size(); ++i) counts[i] = en->counts[i];
  return WF_OK;
}

int wf_ensemble_step(wf_ensemble* en, void* stream) {
  if (!en) return fail(WF_EINVAL, "null ensemble");
  WF_CK(cudaGraphLaunch(en->exec, (cudaStream_t)stream));
  return WF_OK;
}

int wf_ensemble_destroy(wf_ensemble* en) {
  if (!en) return WF_OK;
  if (en->exec) cudaGraphExecDestroy(en->exec);
  if (en->graph) cudaGraphDestroy(en->graph);
  for (void* t : en->tables) cudaFree(t);
  delete en;
  return WF_OK;
}

int wf_stepper_launch_counts(const wf_stepper* st, int32_t counts[4]) {
  if (!st || !counts) return fail(WF_EINVAL, "null argument");
  for (int i = 0; i < 4; ++i) counts[i] = st->counts[i];
  return WF_OK;
}

int wf_stepper_destroy(wf_stepper* st) {
  if (!st) return WF_OK;
  if (st->exec) cudaGraphExecDestroy(st->exec);
  if (st->graph) cudaGraphDestroy(st->graph);
  if (st->hflag) cudaFreeHost(st->hflag);
  delete st;
  return WF_OK;
}

}  // extern "C"
