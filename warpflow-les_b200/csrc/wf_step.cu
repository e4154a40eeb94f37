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
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

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
            comp == 0 ? &c.sc->ulid : nullptr};
  return launch_fills(&r, 1, c.n, s);
}

static int fill_uvw(const wf_case& c, cudaStream_t s) {
  FillReq r[3] = {{c.fld[WF_U], FILL_U, c.ulid, &c.sc->ulid}, {c.fld[WF_V], FILL_V, 0.0},
                  {c.fld[WF_W], FILL_W, 0.0}};
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
  FillReq r{c.fld[WF_P], FILL_PBOUND, 0.0};
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
// launches of each part.
static int append_step(cudaGraph_t g, const wf_case& c, int32_t counts[4]) {
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
    rc = step_prologue(c, cap);
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
      if (rc == WF_OK) rc = step_epilogue(c, cap);
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
    rc = launch_calmas(c, (unsigned long long)h_if, (unsigned long long)h_loop, cap);
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
    rc = step_mg_part(c, cap);
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
};

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
  if (mode & ~WF_STEP_SERIAL) return fail(WF_EINVAL, "ensemble mode: 0 or WF_STEP_SERIAL");
  for (int i = 0; i < ncases; ++i) WF_TRY(validate_case(cases[i]));
  PdlOff guard((mode & WF_STEP_SERIAL) != 0);
  cudaGraph_t g = nullptr;
  WF_CK(cudaGraphCreate(&g, 0));
  int rc = WF_OK;
  int32_t counts[4];
  for (int i = 0; i < ncases && rc == WF_OK; ++i) rc = append_step(g, cases[i], counts);
  wf_ensemble* en = nullptr;
  if (rc == WF_OK) {
    en = new wf_ensemble();
    en->ncases = ncases;
    en->graph = g;
    en->exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&en->exec, g, 0);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaGraphInstantiate(ensemble)");
  }
  if (rc != WF_OK) {
    if (en) {
      wf_ensemble_destroy(en);
    } else {
      cudaGraphDestroy(g);
    }
    return rc;
  }
  *out = en;
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
