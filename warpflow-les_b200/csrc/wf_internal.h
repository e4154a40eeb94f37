// Internal declarations shared by the libwfb200 translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <tuple>
#include <type_traits>

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

// ---- bucket batching ------------------------------------------------------
// A bucket is a set of cases of the same size and numerics stepped together:
// one launch of a kernel serves every case of the bucket.  The cases differ
// only in their buffers (1/Re and the lid velocity live in each case's
// scalar block), so a launch carries the first case's arguments and a device
// table of every case's buffers; a kernel takes its case from blockIdx.z
// (grid z = cases x the single case's z extent) and rebuilds its pointers
// from that case's row.
struct CasePtrs {
  double* fld[WF_NFIELDS];
  wf_scalars* sc;
  void* mg_phi[WF_MAX_LEVELS];
  void* mg_rhs[WF_MAX_LEVELS];
  void* mg_tmp[WF_MAX_LEVELS];
  void* mg_cop_part;
};

// the batch argument every bucket-capable kernel takes last: tab null = one
// case; nz = the single case's grid z extent; skip = a bit of wf_scalars.loop
// a case must have set for the launch to work on it (0: every case)
struct Batch {
  const CasePtrs* tab;
  int nz;
  int skip;
};

// the bucket the calling thread is building launches for (tab null: none)
struct BatchCtx {
  const CasePtrs* tab = nullptr;
  int ncases = 1;
  int skip = 0;
};
BatchCtx& batch_ctx();

template <typename... E>
constexpr bool takes_batch() {
  if constexpr (sizeof...(E) == 0) {
    return false;
  } else {
    return std::is_same<typename std::tuple_element<sizeof...(E) - 1, std::tuple<E...>>::type,
                        Batch>::value;
  }
}

// launch a kernel of this library, with the programmatic-serialization
// attribute when enabled.  A kernel whose last parameter is a Batch gets the
// calling thread's bucket (grid z multiplied by its case count); any other
// kernel refuses to launch while a bucket is being built.
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
  const BatchCtx& bc = batch_ctx();
  if constexpr (takes_batch<ExpTypes...>()) {
    Batch b{bc.tab, (int)grid.z, bc.skip};
    if (bc.tab) cfg.gridDim.z = grid.z * (unsigned)bc.ncases;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<ActTypes&&>(args)..., b);
  } else {
    if (bc.tab) return cudaErrorNotSupported;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<ActTypes&&>(args)...);
  }
}

int validate_case(const wf_case& c);

// ---- ghost fills ---------------------------------------------------------
enum FillKind { FILL_U = 0, FILL_V, FILL_W, FILL_VIS, FILL_PBOUND, FILL_PMIRROR };
struct FillReq {
  double* fld;
  int kind;
  double val;               // ulid for u, 1/Re for vis
  const double* valp = nullptr;  // the same value read on the device, when set
  int fid = -1;             // the field's slot (enum wf_field), for bucket launches
  int vsrc = 0;             // valp in the scalar block: 1 ulid, 2 rrey (bucket launches)
};
// up to 3 independent field fills: one launch of the composed fill program
// (sizes up to 256), else 3 ordered axis phases
int launch_fills(const FillReq* reqs, int nreq, int n, cudaStream_t s);
// build the composed fill programs of size n now (outside any stream capture)
int prepare_fills(int n);
int fill_program(int kind, int n, int32_t* nsimple, int32_t* ngroup, int64_t* nent,
                 int32_t* ent, int32_t* gstart);

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

// ---- launch shapes chosen per size --------------------------------------
// kind SHAPE_CONV: k_conv's CTA, a = extent along k (x), b = along j (y),
// c = planes i per thread; kind SHAPE_SPLIT: k_rbgs_split, a = cells per
// thread, b = rows per CTA (c = 1).  Process-wide, read when a launch is
// issued (a graph keeps the shapes it was captured with); set by
// wf_set_launch_shape (the autotuner).
constexpr int SHAPE_CONV = 0, SHAPE_SPLIT = 1;
void launch_shape(int kind, int n, int* a, int* b, int* c);
int set_launch_shape(int kind, int n, int a, int b, int c);

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
// sub-domains (more than one rank per case)
int launch_box(double* arr, long sI, long sJ, int i0, int j0, int k0, int ni, int nj, int nk,
               double* buf, int unpack, cudaStream_t s);
int rk_mg_op(const wf_case& c, int op, int level, int phys, int color, cudaStream_t s);
int rk_level_view(const wf_case& c, int level, double** phi, int64_t* sI, int64_t* sJ,
                  int32_t* m);
int mg_residual_max_pair(const wf_case& c, const double* phi0, const double* rhs0,
                         double* out, cudaStream_t s);

}  // namespace wf
