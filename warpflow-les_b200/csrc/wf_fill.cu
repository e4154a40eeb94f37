// Ghost-layer fills of the cavity benchmark (reference bcs.py).
//
// The reference issues each fill as an ordered list of face launches
// (bcs.py:201-311), and later faces read what earlier faces wrote at edges
// and corners, so the corner values depend on the order.  Up to n = 256 a
// fill runs as ONE launch of its composed program (k_fill_one, below): the
// host composes the ordered face ops into independent gathers.  Larger
// fills use the ordered form: the faces of one axis never touch each other
// (for n >= 4), so the list splits into three ordered phases -- x faces, y
// faces, z faces -- and each phase runs as one launch (k_fill_phase) in
// which a thread owns one (a, b) line of every face op of that phase and
// walks its layers in order.  Up to three fields share a launch either way.
#include <algorithm>
#include <cstdlib>
#include <functional>
#include <map>
#include <mutex>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "wf_dev.cuh"
#include "wf_internal.h"

namespace wf {

struct FaceOp {
  int axis, high, lin, nlay;
  int g0, s0;
  double val;  // sign for lin, value for const
  int a0, na, b0, nb;
  const double* valp;  // const: the value read on the device instead, when set
};

constexpr int MAX_OPS_PER_PHASE = 4;
constexpr int MAX_JOBS = 3;

constexpr int MAX_LAYERS = NPL;

struct PhaseJob {
  double* fld;
  int fid, vsrc;   // bucket launches: the field's slot, the source of valp (1 ulid, 2 rrey)
  int nops;
  int indep;       // no op reads a cell that an op of this job writes: loads may go first
  FaceOp ops[MAX_OPS_PER_PHASE];
};

struct PhaseArgs {
  PhaseJob job[MAX_JOBS];
  int njob;
  int amax, bmax;
  int P;  // padded extent n + 6
};

__global__ void k_fill_phase(const PhaseArgs args, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  // b (k for x/y faces) is the fast lane index so stores coalesce
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = blockIdx.y * blockDim.y + threadIdx.y;
  const int jb = bt_z(bt);
  if (jb >= args.njob) return;
  const PhaseJob& J = args.job[jb];
  const long P = args.P;
  double* f = J.fld;
  const double* valp = nullptr;
  if (bt.tab) {
    const CasePtrs& cp = bt.tab[bt_case(bt)];
    f = cp.fld[J.fid];
    valp = J.vsrc == 1 ? &cp.sc->ulid : (J.vsrc == 2 ? &cp.sc->rrey : nullptr);
  }
  if (J.indep) {
    // every source of the job is read before any ghost is written (the host
    // checked that no source is a cell the job writes), so a thread's loads
    // are independent and in flight together instead of one per layer
    double val[MAX_OPS_PER_PHASE][MAX_LAYERS];
    long gidx[MAX_OPS_PER_PHASE][MAX_LAYERS];
#pragma unroll
    for (int o = 0; o < MAX_OPS_PER_PHASE; ++o) {
#pragma unroll
      for (int m = 0; m < MAX_LAYERS; ++m) gidx[o][m] = -1;
      if (o >= J.nops) continue;
      const FaceOp& op = J.ops[o];
      if (a >= op.na || b >= op.nb) continue;
      const int pa = op.a0 + a, pb = op.b0 + b;
#pragma unroll
      for (int m = 0; m < MAX_LAYERS; ++m) {
        if (m >= op.nlay) continue;
        const int g = op.high ? op.g0 + m : op.g0 - m;
        gidx[o][m] = op.axis == 0 ? ((long)g * P + pa) * P + pb
                                  : (op.axis == 1 ? ((long)pa * P + g) * P + pb
                                                  : ((long)pa * P + pb) * P + g);
        if (op.lin) {
          const int sidx = op.high ? op.s0 - m : op.s0 + m;
          const long si = op.axis == 0 ? ((long)sidx * P + pa) * P + pb
                                       : (op.axis == 1 ? ((long)pa * P + sidx) * P + pb
                                                       : ((long)pa * P + pb) * P + sidx);
          val[o][m] = op.val * f[si];
        } else {
          val[o][m] = op.valp ? *(valp ? valp : op.valp) : op.val;
        }
      }
    }
#pragma unroll
    for (int o = 0; o < MAX_OPS_PER_PHASE; ++o)
#pragma unroll
      for (int m = 0; m < MAX_LAYERS; ++m)
        if (gidx[o][m] >= 0) f[gidx[o][m]] = val[o][m];
    return;
  }
  for (int o = 0; o < J.nops; ++o) {
    const FaceOp& op = J.ops[o];
    if (a >= op.na || b >= op.nb) continue;
    const int pa = op.a0 + a, pb = op.b0 + b;
    for (int m = 0; m < op.nlay; ++m) {
      const int g = op.high ? op.g0 + m : op.g0 - m;
      long gi, si = 0;
      if (op.axis == 0) {
        gi = ((long)g * P + pa) * P + pb;
      } else if (op.axis == 1) {
        gi = ((long)pa * P + g) * P + pb;
      } else {
        gi = ((long)pa * P + pb) * P + g;
      }
      if (op.lin) {
        const int sidx = op.high ? op.s0 - m : op.s0 + m;
        if (op.axis == 0) {
          si = ((long)sidx * P + pa) * P + pb;
        } else if (op.axis == 1) {
          si = ((long)pa * P + sidx) * P + pb;
        } else {
          si = ((long)pa * P + pb) * P + sidx;
        }
        f[gi] = op.val * f[si];
      } else {
        f[gi] = op.valp ? *(valp ? valp : op.valp) : op.val;
      }
    }
  }
}

// ---- fill programs: the reference launch lists, split into axis phases ----
static FaceOp lin(int axis, int high, int g0, int s0, double sign, int a0, int na,
                  int b0, int nb, int nlay) {
  return FaceOp{axis, high, 1, nlay, g0, s0, sign, a0, na, b0, nb, nullptr};
}
static FaceOp cst(int axis, int high, int g0, double val, int a0, int na, int b0,
                  int nb, int nlay, const double* valp = nullptr) {
  return FaceOp{axis, high, 0, nlay, g0, 0, val, a0, na, b0, nb, valp};
}

// true when no op of the list reads a cell that an op of the list writes
// (the ops of one phase share its axis, so it suffices to compare the layer
// indices along the axis and the (a, b) rectangles): then every load may
// precede every store and the result is the same as in program order
static bool ops_independent(const FaceOp* ops, int nops) {
  for (int w = 0; w < nops; ++w)
    if (ops[w].nlay > MAX_LAYERS) return false;   // the kernel's hoisted form holds MAX_LAYERS
  for (int r = 0; r < nops; ++r) {
    if (!ops[r].lin) continue;
    for (int w = 0; w < nops; ++w) {
      if (ops[w].axis != ops[r].axis) return false;
      const bool overlap_ab = ops[r].a0 < ops[w].a0 + ops[w].na && ops[w].a0 < ops[r].a0 + ops[r].na &&
                              ops[r].b0 < ops[w].b0 + ops[w].nb && ops[w].b0 < ops[r].b0 + ops[r].nb;
      if (!overlap_ab) continue;
      for (int mr = 0; mr < ops[r].nlay; ++mr) {
        const int src = ops[r].high ? ops[r].s0 - mr : ops[r].s0 + mr;
        for (int mw = 0; mw < ops[w].nlay; ++mw) {
          const int dst = ops[w].high ? ops[w].g0 + mw : ops[w].g0 - mw;
          if (src == dst) return false;
        }
      }
    }
  }
  return true;
}

// phase ops of one fill kind; returns op count for `phase` (0 = x, 1 = y, 2 = z)
static int program(int kind, int n, double val, const double* valp, int phase, FaceOp* out) {
  const int P = NPL;
  int k = 0;
  switch (kind) {
    case FILL_U:  // bcs.py:201-223
      if (phase == 0) {
        out[k++] = cst(0, 0, P - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3);
        out[k++] = cst(0, 1, P + n - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3);
      } else if (phase == 1) {
        out[k++] = lin(1, 0, P - 1, P, 1.0, P - 1, n + 1, P - 1, n + 2, 3);
        out[k++] = lin(1, 1, P + n, P + n - 1, 1.0, P - 1, n + 1, P - 1, n + 2, 3);
      } else {
        out[k++] = lin(2, 0, P - 1, P, -1.0, P - 1, n + 1, P - 1, n + 2, 3);
        out[k++] = cst(2, 1, P + n, val, P - 1, n + 1, P - 1, n + 2, 3, valp);
      }
      break;
    case FILL_V:  // bcs.py:225-244
      if (phase == 0) {
        out[k++] = lin(0, 0, P - 1, P, -1.0, P - 1, n + 1, P - 1, n + 2, 3);
        out[k++] = lin(0, 1, P + n, P + n - 1, -1.0, P - 1, n + 1, P - 1, n + 2, 3);
      } else if (phase == 1) {
        out[k++] = cst(1, 0, P - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3);
        out[k++] = cst(1, 1, P + n - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3);
      } else {
        out[k++] = lin(2, 0, P - 1, P, -1.0, P - 1, n + 2, P - 1, n + 1, 3);
        out[k++] = lin(2, 1, P + n, P + n - 1, 1.0, P - 1, n + 2, P - 1, n + 1, 3);
      }
      break;
    case FILL_W:  // bcs.py:246-265
      if (phase == 0) {
        out[k++] = lin(0, 0, P - 1, P, -1.0, P - 1, n + 2, P - 1, n + 1, 3);
        out[k++] = lin(0, 1, P + n, P + n - 1, -1.0, P - 1, n + 2, P - 1, n + 1, 3);
      } else if (phase == 1) {
        out[k++] = lin(1, 0, P - 1, P, 1.0, P - 1, n + 2, P - 1, n + 1, 3);
        out[k++] = lin(1, 1, P + n, P + n - 1, 1.0, P - 1, n + 2, P - 1, n + 1, 3);
      } else {
        out[k++] = cst(2, 0, P - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3);
        out[k++] = cst(2, 1, P + n - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3);
      }
      break;
    case FILL_VIS:  // bcs.py:267-293
      if (phase == 0) {
        out[k++] = cst(0, 0, P, val, P - 1, n + 2, P - 1, n + 2, 1, valp);
        out[k++] = lin(0, 0, P - 1, P, 1.0, P - 1, n + 2, P - 1, n + 2, 1);
        out[k++] = cst(0, 1, P + n - 1, val, P - 1, n + 2, P - 1, n + 2, 1, valp);
        out[k++] = lin(0, 1, P + n, P + n - 1, 1.0, P - 1, n + 2, P - 1, n + 2, 1);
      } else if (phase == 1) {
        out[k++] = lin(1, 0, P - 1, P, 1.0, P - 1, n + 2, P - 1, n + 2, 1);
        out[k++] = lin(1, 1, P + n, P + n - 1, 1.0, P - 1, n + 2, P - 1, n + 2, 1);
      } else {
        out[k++] = cst(2, 0, P, val, P - 1, n + 2, P - 1, n + 2, 1, valp);
        out[k++] = lin(2, 0, P - 1, P, 1.0, P - 1, n + 2, P - 1, n + 2, 1);
        out[k++] = lin(2, 1, P + n, P + n - 1, 1.0, P - 1, n + 2, P - 1, n + 2, 1);
      }
      break;
    case FILL_PBOUND:  // bcs.py:295-302
      out[k++] = lin(phase, 0, P - 1, P, 1.0, P - 1, n + 3, P - 1, n + 3, 1);
      out[k++] = lin(phase, 1, P + n, P + n - 1, 1.0, P - 1, n + 3, P - 1, n + 3, 1);
      break;
    case FILL_PMIRROR:  // bcs.py:304-311
      out[k++] = lin(phase, 0, P - 1, P, 1.0, 0, n + 2 * P, 0, n + 2 * P, P);
      out[k++] = lin(phase, 1, P + n, P + n - 1, 1.0, 0, n + 2 * P, 0, n + 2 * P, P);
      break;
  }
  return k;
}


// ---- one-launch fills -------------------------------------------------------
// The ordered face ops of a fill only copy (times +-1) and set constants, so
// every cell a fill writes ends as s * old(x) -- the value some cell x held
// before the fill -- or s * K, K = 0 or the fill's value, s = +-1.  The host
// composes the ops in the reference's order once per (fill kind, n) and the
// fill then runs as ONE launch of independent gathers instead of three
// ordered phases whose threads walk their layers load by load.  Where a
// written cell's final value needs the old value of a cell that the same
// fill also overwrites, both cells (and any others chained to them) go to
// one thread, which loads every value it needs before it stores any: a
// "group".  Every other written cell is one thread's single gather.  The
// products by +-1 are exact, so the result is the phases' bit for bit.
//
// Table entries are (dst, code): dst the cell's offset in the field; code
// bit 0 set: a constant (bits 2.. = 0 for 0.0, 1 for the fill's value),
// else bits 2.. = the source offset; bit 1 set: negate.
constexpr int ONE_GMAX = 16;        // cells of one group
constexpr int ONE_NMAX = 256;       // largest n served by one-launch fills

struct OneProg {
  const int2* ent = nullptr;   // nsimple entries, then the groups' entries
  const int* gstart = nullptr; // ngroup + 1 offsets into ent (from nsimple)
  int nsimple = 0, ngroup = 0;
};

struct OneJob {
  double* fld;
  int fid, vsrc;
  double val;
  const double* valp;
  OneProg prog;
};

struct OneArgs {
  OneJob job[MAX_JOBS];
  int njob;
};

__device__ __forceinline__ double one_value(const double* f, int code, double K) {
  const double v = (code & 1) ? ((code >> 2) ? K : 0.0) : f[code >> 2];
  return (code & 2) ? -v : v;
}

__global__ void k_fill_one(const OneArgs args, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const int jb = bt_z(bt);
  if (jb >= args.njob) return;
  const OneJob& J = args.job[jb];
  double* f = J.fld;
  const double* valp = J.valp;
  if (bt.tab) {
    const CasePtrs& cp = bt.tab[bt_case(bt)];
    f = cp.fld[J.fid];
    if (J.vsrc) valp = J.vsrc == 1 ? &cp.sc->ulid : &cp.sc->rrey;
  }
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double K = valp ? *valp : J.val;
  if (t < J.prog.nsimple) {
    const int2 e = J.prog.ent[t];
    f[e.x] = one_value(f, e.y, K);
    return;
  }
  const int g = t - J.prog.nsimple;
  if (g >= J.prog.ngroup) return;
  const int a = J.prog.nsimple + J.prog.gstart[g], b = J.prog.nsimple + J.prog.gstart[g + 1];
  double v[ONE_GMAX];
#pragma unroll
  for (int q = 0; q < ONE_GMAX; ++q)
    if (a + q < b) v[q] = one_value(f, J.prog.ent[a + q].y, K);
#pragma unroll
  for (int q = 0; q < ONE_GMAX; ++q)
    if (a + q < b) f[J.prog.ent[a + q].x] = v[q];
}

// compose the fill's ops (reference order) into its one-launch program;
// false when a group would exceed ONE_GMAX cells
static bool one_build(int kind, int n, std::vector<int2>& ent, std::vector<int>& gstart,
                      int& nsimple) {
  const long P = n + 2 * NPL;
  // expression of every written cell: (source offset or constant id, const, negate)
  struct Ex { long ref; bool cst, neg; };
  std::unordered_map<long, Ex> ex;
  ex.reserve((size_t)6 * NPL * P * P);
  auto cur = [&](long c) -> Ex {
    auto it = ex.find(c);
    return it == ex.end() ? Ex{c, false, false} : it->second;
  };
  std::vector<long> order;   // written cells, first write order
  for (int phase = 0; phase < 3; ++phase) {
    FaceOp ops[MAX_OPS_PER_PHASE];
    const int nops = program(kind, n, 1.0, nullptr, phase, ops);
    for (int o = 0; o < nops; ++o) {
      const FaceOp& op = ops[o];
      for (int a = 0; a < op.na; ++a)
        for (int b = 0; b < op.nb; ++b)
          for (int m = 0; m < op.nlay; ++m) {
            const long pa = op.a0 + a, pb = op.b0 + b;
            const long gidx = op.high ? op.g0 + m : op.g0 - m;
            auto at = [&](long x) {
              return op.axis == 0 ? (x * P + pa) * P + pb
                                  : (op.axis == 1 ? (pa * P + x) * P + pb : (pa * P + pb) * P + x);
            };
            const long dst = at(gidx);
            Ex e;
            if (op.lin) {
              e = cur(at(op.high ? op.s0 - m : op.s0 + m));
              if (op.val < 0) e.neg = !e.neg;
            } else {
              // a constant op writes 0.0 or the fill's value (ulid, 1/Re),
              // which program() was given as 1.0 here
              e = Ex{op.val == 0.0 ? 0 : 1, true, false};
            }
            if (!ex.count(dst)) order.push_back(dst);
            ex[dst] = e;
          }
    }
  }
  // union-find over written cells: a cell whose value is the old value of
  // another written cell goes with it
  std::unordered_map<long, long> parent;
  parent.reserve(order.size());
  std::function<long(long)> find = [&](long x) {
    long r = x;
    while (parent[r] != r) r = parent[r];
    while (parent[x] != r) {
      const long nx = parent[x];
      parent[x] = r;
      x = nx;
    }
    return r;
  };
  for (long c : order) parent[c] = c;
  for (long c : order) {
    const Ex& e = ex[c];
    if (!e.cst && e.ref != c && ex.count(e.ref)) {
      const long ra = find(c), rb = find(e.ref);
      if (ra != rb) parent[ra] = rb;
    }
  }
  std::unordered_map<long, std::vector<long>> comp;
  for (long c : order) {
    const Ex& e = ex[c];
    if (!e.cst && e.ref == c && !e.neg) continue;   // unchanged: nothing to write
    comp[find(c)].push_back(c);
  }
  auto code = [&](const Ex& e) {
    return (int)((e.ref << 2) | (e.neg ? 2 : 0) | (e.cst ? 1 : 0));
  };
  std::vector<int2> simple;
  std::vector<std::vector<long>> groups;
  for (auto& kv : comp) {
    if (kv.second.size() == 1) {
      const long c = kv.second[0];
      simple.push_back(make_int2((int)c, code(ex[c])));
    } else {
      if (kv.second.size() > (size_t)ONE_GMAX) return false;
      groups.push_back(kv.second);
    }
  }
  std::sort(simple.begin(), simple.end(), [](const int2& p, const int2& q) { return p.x < q.x; });
  std::sort(groups.begin(), groups.end());
  ent = simple;
  nsimple = (int)simple.size();
  gstart.assign(1, 0);
  for (auto& gr : groups) {
    std::sort(gr.begin(), gr.end());
    for (long c : gr) ent.push_back(make_int2((int)c, code(ex[c])));
    gstart.push_back((int)(ent.size() - nsimple));
  }
  return true;
}

// the device program of (kind, n) on the current device, built on first use;
// null while the stream is being captured and it does not exist yet (the
// phased fill then runs), or for sizes above ONE_NMAX
static const OneProg* one_prog(int kind, int n, cudaStream_t s) {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("WF_FILL1");
    on = (e && e[0] == '0') ? 0 : 1;
  }
  if (n > ONE_NMAX || !on) return nullptr;
  static std::mutex mu;
  static std::map<std::tuple<int, int, int>, OneProg*> progs;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_tuple(dev, kind, n);
  auto it = progs.find(key);
  if (it != progs.end()) return it->second;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (s && cudaStreamIsCapturing(s, &cs) != cudaSuccess) return nullptr;
  if (cs != cudaStreamCaptureStatusNone) return nullptr;
  std::vector<int2> ent;
  std::vector<int> gstart;
  int nsimple = 0;
  OneProg* p = new OneProg();
  if (one_build(kind, n, ent, gstart, nsimple)) {
    int2* de = nullptr;
    int* dg = nullptr;
    if (cudaMalloc(&de, ent.size() * sizeof(int2)) != cudaSuccess ||
        cudaMalloc(&dg, gstart.size() * sizeof(int)) != cudaSuccess ||
        cudaMemcpy(de, ent.data(), ent.size() * sizeof(int2), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(dg, gstart.data(), gstart.size() * sizeof(int), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
      cudaGetLastError();
      delete p;
      return nullptr;
    }
    p->ent = de;
    p->gstart = dg;
    p->nsimple = nsimple;
    p->ngroup = (int)gstart.size() - 1;
  }
  progs[key] = p->ent ? p : nullptr;
  if (!p->ent) delete p;
  return progs[key];
}

int fill_program(int kind, int n, int32_t* nsimple, int32_t* ngroup, int64_t* nent,
                 int32_t* ent, int32_t* gstart) {
  if (kind < FILL_U || kind > FILL_PMIRROR) return fail(WF_EINVAL, "fill kind out of range");
  if (n < 4 || n > ONE_NMAX) return fail(WF_EINVAL, "fill program: n in 4..256");
  std::vector<int2> e;
  std::vector<int> g;
  int ns = 0;
  if (!one_build(kind, n, e, g, ns)) return fail(WF_EUNSUPPORTED, "fill program: group too large");
  *nsimple = ns;
  *ngroup = (int32_t)g.size() - 1;
  *nent = (int64_t)e.size();
  if (ent)
    for (size_t q = 0; q < e.size(); ++q) {
      ent[2 * q] = e[q].x;
      ent[2 * q + 1] = e[q].y;
    }
  if (gstart)
    for (size_t q = 0; q < g.size(); ++q) gstart[q] = g[q];
  return WF_OK;
}

int prepare_fills(int n) {
  for (int kind = FILL_U; kind <= FILL_PMIRROR; ++kind) one_prog(kind, n, nullptr);
  return WF_OK;
}

// the one-launch form of launch_fills; false when a job has no program
static bool launch_fills_one(const FillReq* reqs, int nreq, int n, cudaStream_t s, int* rc) {
  OneArgs a{};
  a.njob = nreq;
  int maxthreads = 0;
  for (int r = 0; r < nreq; ++r) {
    const OneProg* p = one_prog(reqs[r].kind, n, s);
    if (!p) return false;
    a.job[r] = OneJob{reqs[r].fld, reqs[r].fid, reqs[r].vsrc, reqs[r].val, reqs[r].valp, *p};
    maxthreads = std::max(maxthreads, p->nsimple + p->ngroup);
  }
  *rc = WF_OK;
  cudaError_t e = launch_k(k_fill_one, dim3((maxthreads + 255) / 256, 1, nreq), dim3(256), 0, s, a);
  ++g_launches;
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) *rc = cuda_fail(e, "k_fill_one");
  return true;
}

int launch_fills(const FillReq* reqs, int nreq, int n, cudaStream_t s) {
  if (nreq < 1 || nreq > MAX_JOBS) return fail(WF_EINVAL, "launch_fills: 1..3 fields");
  if (n < 4) return fail(WF_EINVAL, "ghost fills need n >= 4");
  for (int r = 0; r < nreq; ++r) {
    if (!reqs[r].fld) return fail(WF_EINVAL, "launch_fills: null field");
    if (batch_ctx().tab && reqs[r].fid < 0)
      return fail(WF_EUNSUPPORTED, "launch_fills: a bucket fill needs field slots");
  }
  {
    int rc = WF_OK;
    if (launch_fills_one(reqs, nreq, n, s, &rc)) return rc;
  }
  for (int phase = 0; phase < 3; ++phase) {
    PhaseArgs a{};
    a.njob = nreq;
    a.P = n + 2 * NPL;
    a.amax = a.bmax = 0;
    for (int r = 0; r < nreq; ++r) {
      if (!reqs[r].fld) return fail(WF_EINVAL, "launch_fills: null field");
      if (batch_ctx().tab && reqs[r].fid < 0)
        return fail(WF_EUNSUPPORTED, "launch_fills: a bucket fill needs field slots");
      a.job[r].fld = reqs[r].fld;
      a.job[r].fid = reqs[r].fid;
      a.job[r].vsrc = reqs[r].vsrc;
      a.job[r].nops = program(reqs[r].kind, n, reqs[r].val, reqs[r].valp, phase, a.job[r].ops);
      a.job[r].indep = ops_independent(a.job[r].ops, a.job[r].nops) ? 1 : 0;
      for (int o = 0; o < a.job[r].nops; ++o) {
        a.amax = a.job[r].ops[o].na > a.amax ? a.job[r].ops[o].na : a.amax;
        a.bmax = a.job[r].ops[o].nb > a.bmax ? a.job[r].ops[o].nb : a.bmax;
      }
    }
    dim3 tb(32, 8);
    dim3 gb((a.bmax + 31) / 32, (a.amax + 7) / 8, nreq);
    WF_CK(launch_k(k_fill_phase, gb, tb, 0, s, a));
    WF_CKL("k_fill_phase");
  }
  return WF_OK;
}

}  // namespace wf
