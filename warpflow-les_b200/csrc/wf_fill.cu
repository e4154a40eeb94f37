// Ghost-layer fills of the cavity benchmark (reference bcs.py).
//
// The reference issues each fill as an ordered list of face launches
// (bcs.py:201-311), and later faces read what earlier faces wrote at edges
// and corners, so the corner values depend on the order.  The faces of one
// axis never touch each other (for n >= 4), so the list splits into three
// ordered phases -- x faces, y faces, z faces -- and each phase runs as one
// launch in which a thread owns one (a, b) line of every face op of that
// phase and walks its layers in order.  Up to three fields share a launch.
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

int launch_fills(const FillReq* reqs, int nreq, int n, cudaStream_t s) {
  if (nreq < 1 || nreq > MAX_JOBS) return fail(WF_EINVAL, "launch_fills: 1..3 fields");
  if (n < 4) return fail(WF_EINVAL, "ghost fills need n >= 4");
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
