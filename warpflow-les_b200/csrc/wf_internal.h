// Internal declarations shared by the libwfb200 translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "warpflow_b200.h"

namespace wf {

constexpr int NPL = WF_NPL;

// ---- error plumbing ------------------------------------------------------
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define WF_CK(expr)                                                  \
  do {                                                               \
    cudaError_t _e = (expr);                                         \
    if (_e != cudaSuccess) return ::wf::cuda_fail(_e, #expr);        \
  } while (0)

// every kernel launch is followed by WF_CKL, which also counts it
extern thread_local long g_launches;
#define WF_CKL(what)                                                 \
  do {                                                               \
    ++::wf::g_launches;                                              \
    cudaError_t _e = cudaGetLastError();                             \
    if (_e != cudaSuccess) return ::wf::cuda_fail(_e, what);         \
  } while (0)

#define WF_TRY(expr)                                                 \
  do {                                                               \
    int _r = (expr);                                                 \
    if (_r != WF_OK) return _r;                                      \
  } while (0)

inline int64_t padded(int n) { return (int64_t)n + 2 * NPL; }

// programmatic dependent launch on (default) or off (WF_PDL=0)
bool pdl_enabled();

// one thread per cell of an ni x nj x nk box: CTAs of 32 (k) x 8 (j) threads,
// grid z = i
inline dim3 cells3(int ni, int nj, int nk) { return dim3((nk + 31) / 32, (nj + 7) / 8, ni); }
inline dim3 cell_block() { return dim3(32, 8); }

// launch a kernel of this library, with the programmatic-serialization
// attribute when enabled and an optional cluster shape
template <typename... ExpTypes, typename... ActTypes>
inline cudaError_t launch_k(void (*kernel)(ExpTypes...), dim3 grid, dim3 block, size_t smem,
                            cudaStream_t s, ActTypes&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  int na = 0;
  if (pdl_enabled()) {
    at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
  }
  cfg.attrs = at;
  cfg.numAttrs = na;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<ActTypes&&>(args)...);
}

int validate_case(const wf_case& c);

// ---- ghost fills ---------------------------------------------------------
enum FillKind { FILL_U = 0, FILL_V, FILL_W, FILL_VIS, FILL_PBOUND, FILL_PMIRROR };
struct FillReq {
  double* fld;
  int kind;
  double val;               // ulid for u, 1/Re for vis
  const double* valp = nullptr;  // the same value read on the device, when set
};
// up to 3 independent field fills, executed as 3 ordered axis phases
int launch_fills(const FillReq* reqs, int nreq, int n, cudaStream_t s);

// ---- operators -----------------------------------------------------------
int launch_init_noise(double* u, double* v, double* w, int n, double amp,
                      int seed, cudaStream_t s);
int launch_checkdt(const wf_case& c, cudaStream_t s);
int launch_copy_oo(const wf_case& c, cudaStream_t s);
// rrey_dev: 1/Re read on the device (the step), or null for c.rrey
int launch_wale(const wf_case& c, cudaStream_t s, const double* rrey_dev = nullptr);
int launch_conv(const wf_case& c, int comp, double alpha, const double* dt, cudaStream_t s,
                bool with_diff = false);
int launch_diff(const wf_case& c, int comp, double alpha, const double* dt, cudaStream_t s);
int launch_calvel(const wf_case& c, double alpha, const double* dt, cudaStream_t s);
// calmas + projection-loop control (sets graph conditionals when h != 0)
int launch_calmas(const wf_case& c, unsigned long long h_if,
                  unsigned long long h_loop, cudaStream_t s);
int launch_add_ring(double* p, const double* pp, int n, cudaStream_t s);
int launch_scalars_init(wf_scalars* sc, double dt0, double rrey, double ulid, cudaStream_t s);

// ---- multigrid -----------------------------------------------------------
int mg_solve(const wf_case& c, cudaStream_t s);
int coarse_op_elems(const wf_case& c, int64_t* op_elems, int64_t* scratch_elems);
int build_coarse_op_case(const wf_case& c, cudaStream_t s);
int mg_coarse_solve_pair(const wf_case& c, double* phi, const double* rhs, cudaStream_t s);
int mg_vcycle_pair(const wf_case& c, double* phi0, const double* rhs0, cudaStream_t s);
int mg_relax_pair(const wf_case& c, double* phi0, const double* rhs0, int nsweeps,
                  cudaStream_t s);
int mg_refill_pair(const wf_case& c, double* phi0, cudaStream_t s);
int set_coarse_strategy(int n, int fp32, int strategy);
int mg_dc_cycle_pair(const wf_case& c, double* phi0, const double* rhs0, cudaStream_t s);
int mg_solve_noalloc(const double* su, double* pp, int n, int nlev, double dx, double dy,
                     double dz, cudaStream_t s);
int mg_noalloc_status(void* stream, int32_t* status);
int wait_probe(unsigned* gbar, int* err, int kind, int tries, cudaStream_t s);
int mg_residual_max_pair(const wf_case& c, const double* phi0, const double* rhs0,
                         double* out, cudaStream_t s);

}  // namespace wf
