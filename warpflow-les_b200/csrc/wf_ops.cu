// Stencil operators of one LES step (reference kernels.py) and the device
// side of the time-step control (solver.py compute_dt) and of the
// projection loop (solver.py _project).
//
// Field layout: (n+6)^3 doubles, [i][j][k] with k contiguous, real cells
// NPL..NPL+n-1.  One thread per output cell; consecutive threads walk k so
// every access of a warp is a contiguous run.
#include <algorithm>
#include <cmath>

#include "wf_dev.cuh"
#include "wf_internal.h"

namespace wf {

constexpr int TPB = 256;

struct Geo {
  long P, sI, sJ;   // padded extent and strides
  int n;
  __device__ __forceinline__ long at(int i, int j, int k) const {
    return (long)i * sI + (long)j * sJ + k;
  }
};

// The constant divisors of the stage kernels with their reciprocals
// RN(1/d), computed on the host with the same expressions the kernels use
// (24h, 12h*h, h, 3): x/d is then div_by_recip(x, d, RN(1/d)), the same
// correctly rounded quotient as the division.
struct Divs {
  double d24[3], y24[3], d12[3], y12[3], dh[3], yh[3], d3, y3;
};

static inline Divs divs_of(const wf_case& c) {
  Divs v;
  const double h[3] = {c.dx, c.dy, c.dz};
  for (int a = 0; a < 3; ++a) {
    v.d24[a] = 24.0 * h[a];
    v.y24[a] = 1.0 / v.d24[a];
    v.d12[a] = 12.0 * h[a] * h[a];
    v.y12[a] = 1.0 / v.d12[a];
    v.dh[a] = h[a];
    v.yh[a] = 1.0 / h[a];
  }
  v.d3 = 3.0;
  v.y3 = 1.0 / 3.0;
  return v;
}

static inline Geo geo_of(int n) {
  Geo g;
  g.n = n;
  g.P = n + 2 * NPL;
  g.sJ = g.P;
  g.sI = g.P * g.P;
  return g;
}

// reductions over the n^3 real cells: 1-D CTAs of 32 (k) x 8 (j) threads,
// grid (k runs, j groups, G) with each CTA stepping through planes i by G;
// G keeps the grid near 32 CTAs per SM: enough independent planes in flight,
// few enough CTAs meeting at the reduction atomics
static inline dim3 reduce_grid(int n) {
  const int gx = (n + 31) / 32, gy = (n + 7) / 8;
  const int g = std::max(1, std::min(n, (148 * 32) / (gx * gy)));
  return dim3(gx, gy, g);
}

static inline int nblocks(long work, int tpb = TPB, int cap = 148 * 16) {
  long b = (work + tpb - 1) / tpb;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

#define LD(p, idx) ((p)[(idx)])

// --------------------------------------------------------------------------
// scalar block
// --------------------------------------------------------------------------
__global__ void k_scalars_init(wf_scalars* sc, double dt0, double rrey, double ulid) {
  pdl_entry();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  sc->dt = dt0;
  sc->rrey = rrey;
  sc->ulid = ulid;
  sc->ctime = 0.0;
  sc->rmax = 0.0;
  sc->cfl = 0.0;
  sc->dtmax = 0.0;
  sc->umax = sc->vmax = sc->wmax = 0.0;
  sc->dtvisc = 0.0;
  for (int i = 0; i < 32; ++i) sc->rmax_trace[i] = 0.0;
  sc->red[0] = sc->red[1] = sc->red[2] = okey(0.0);
  sc->red[3] = 0ull;          // rate key of k_checkdt (0: the key of +0)
  sc->red[4] = okey(0.0);
  sc->red[5] = okey(0.0);
  sc->itime = 0;
  sc->iters = 0;
  sc->status = WF_ST_OK;
  sc->loop = 0;
  sc->ticket = 0u;
  sc->nmg = 0;
  sc->gbar[0] = sc->gbar[1] = 0u;
}

int launch_scalars_init(wf_scalars* sc, double dt0, double rrey, double ulid, cudaStream_t s) {
  if (!sc) return fail(WF_EINVAL, "null scalar block");
  WF_CK(launch_k(k_scalars_init, 1, 32, 0, s, sc, dt0, rrey, ulid));
  WF_CKL("k_scalars_init");
  return WF_OK;
}

// --------------------------------------------------------------------------
// init_noise (kernels.py:452-471)
// --------------------------------------------------------------------------
__global__ void k_init_noise(double* u, double* v, double* w, Geo g, double amp,
                             int seed) {
  pdl_entry();
  const long tot = (long)g.n * g.n * g.n;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot;
       t += (long)gridDim.x * blockDim.x) {
    const int k = NPL + (int)(t % g.n);
    const int j = NPL + (int)((t / g.n) % g.n);
    const int i = NPL + (int)(t / ((long)g.n * g.n));
    uint32_t h = ((uint32_t)i * 73856093u) ^ ((uint32_t)j * 19349663u) ^
                 ((uint32_t)k * 83492791u) ^ (uint32_t)seed;
    h = h ^ (h >> 13);
    h = h * 1274126177u;
    h = h ^ (h >> 16);
    const double r = ((double)h / 4294967295.0) * 2.0 - 1.0;
    const long id = g.at(i, j, k);
    u[id] = amp * r;
    v[id] = amp * r;
    w[id] = -amp * r;
  }
}

int launch_init_noise(double* u, double* v, double* w, int n, double amp, int seed,
                      cudaStream_t s) {
  if (!u || !v || !w || n < 1) return fail(WF_EINVAL, "init_noise: bad args");
  Geo g = geo_of(n);
  WF_CK(launch_k(k_init_noise, nblocks((long)n * n * n), TPB, 0, s, u, v, w, g, amp, seed));
  WF_CKL("k_init_noise");
  return WF_OK;
}

// --------------------------------------------------------------------------
// checkdt (solver.py:122-150, kernels.py:374-402): max|u|, max|v|, max|w|
// and the viscous/advective min in one pass; the last block finishes the
// dt update on the device.
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(TPB) k_checkdt(const wf_case c, Geo g, const Divs dv,
                                                const Batch bt) {
  pdl_entry();
  __shared__ double sm[32];
  const double* u = bt_fld(c, bt, WF_U);
  const double* v = bt_fld(c, bt, WF_V);
  const double* w = bt_fld(c, bt, WF_W);
  const double* vis = bt_fld(c, bt, WF_VIS);
  const double dx = c.dx, dy = c.dy, dz = c.dz;
  const double inv2 = 1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz);
  // The reference's dtvisc is the min over cells of RN(1/x), x the cell's
  // viscous/advective rate, initialised with 1e10 (solver.py:127).  On each
  // side of zero the correctly rounded reciprocal falls as x grows, and
  // every negative x gives a smaller reciprocal than every positive one, so
  // the min is RN(1/x*) for the x* that maximises the order key of x with
  // its top bit flipped (negatives above positives, ascending x within
  // each sign; NaN skipped as fmin skips it): one division per step instead
  // of one per cell, the same bits for every input.
  double mu = 0.0, mv = 0.0, mw = 0.0;
  unsigned long long kx = 0ull;
  __shared__ unsigned long long skx[32];
  const int k = NPL + blockIdx.x * 32 + (threadIdx.x & 31);
  const int j = NPL + blockIdx.y * 8 + (threadIdx.x >> 5);
  const bool in = k < NPL + g.n && j < NPL + g.n;
  for (int i = NPL + bt_z(bt); in && i < NPL + g.n; i += bt_gz(bt)) {
    const long id = g.at(i, j, k);
    const double uu = LD(u, id), vv = LD(v, id), ww = LD(w, id);
    mu = fmax(mu, fabs(uu));
    mv = fmax(mv, fabs(vv));
    mw = fmax(mw, fabs(ww));
    const double uc = 0.5 * (uu + LD(u, id - g.sI));
    const double vc = 0.5 * (vv + LD(v, id - g.sJ));
    const double wc = 0.5 * (ww + LD(w, id - 1));
    const double x = div_by_recip(fabs(uc), dv.dh[0], dv.yh[0]) +
                     div_by_recip(fabs(vc), dv.dh[1], dv.yh[1]) +
                     div_by_recip(fabs(wc), dv.dh[2], dv.yh[2]) + 2.0 * LD(vis, id) * inv2 +
                     1.0e-30;
    if (x == x) kx = max(kx, okey(x) ^ 0x8000000000000000ull);
  }
  mu = block_max(mu, sm);
  mv = block_max(mv, sm);
  mw = block_max(mw, sm);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) kx = max(kx, __shfl_xor_sync(0xffffffffu, kx, o));
  if ((threadIdx.x & 31) == 0) skx[threadIdx.x >> 5] = kx;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int q = 1; q < (int)((blockDim.x + 31) >> 5); ++q) kx = max(kx, skx[q]);
  wf_scalars* sc = bt_sc(c, bt);
  if (threadIdx.x == 0) {
    atomicMax(&sc->red[0], okey(mu));
    atomicMax(&sc->red[1], okey(mv));
    atomicMax(&sc->red[2], okey(mw));
    atomicMax(&sc->red[3], kx);
  }
  if (!last_block(&sc->ticket, gridDim.x * gridDim.y * bt_gz(bt))) return;
  if (threadIdx.x != 0) return;
  const double umax = okey_inv(atomicAdd(&sc->red[0], 0ull));
  const double vmax = okey_inv(atomicAdd(&sc->red[1], 0ull));
  const double wmax = okey_inv(atomicAdd(&sc->red[2], 0ull));
  const double dtvisc =
      fmin(1.0e10, 1.0 / okey_inv(atomicAdd(&sc->red[3], 0ull) ^ 0x8000000000000000ull));
  sc->red[0] = sc->red[1] = sc->red[2] = okey(0.0);
  sc->red[3] = 0ull;
  const double big = 1.0e10;
  double dtcfl = big;
  if (umax > 0.0) dtcfl = fmin(dtcfl, dx / umax);
  if (vmax > 0.0) dtcfl = fmin(dtcfl, dy / vmax);
  if (wmax > 0.0) dtcfl = fmin(dtcfl, dz / wmax);
  const double dtmax = fmin(dtvisc, dtcfl);
  sc->umax = umax;
  sc->vmax = vmax;
  sc->wmax = wmax;
  sc->dtvisc = dtvisc;
  sc->dtmax = dtmax;
  sc->itime += 1;
  sc->iters = 0;
  sc->nmg = 0;
  sc->loop = 1;   // the case takes part in this step's projection loop
  if (dtmax <= 0.0 || !(dtmax < big)) sc->status = WF_ST_DT_COLLAPSE;
  const double dt_old = sc->dt;
  sc->cfl = dt_old / dtmax;
  double dt = dt_old;
  if (c.variable_dt) dt = fmin(dt_old * c.dt_growth, c.safety * dtmax);
  sc->dt = dt;
  sc->ctime += dt;
}

int launch_checkdt(const wf_case& c, cudaStream_t s) {
  Geo g = geo_of(c.n);
  WF_CK(launch_k(k_checkdt, reduce_grid(c.n), TPB, 0, s, c, g, divs_of(c)));
  WF_CKL("k_checkdt");
  return WF_OK;
}

// --------------------------------------------------------------------------
// uoo/voo/woo = u/v/w over the full padded arrays (solver.py:223-225)
// --------------------------------------------------------------------------
__global__ void k_copy3(const double2* a0, double2* b0,
                        const double2* a1, double2* b1,
                        const double2* a2, double2* b2,
                        long n2, const Batch bt) {
  pdl_entry();
  if (bt.tab) {
    const CasePtrs& cp = bt.tab[bt_case(bt)];
    a0 = (const double2*)cp.fld[WF_U];
    b0 = (double2*)cp.fld[WF_UOO];
    a1 = (const double2*)cp.fld[WF_V];
    b1 = (double2*)cp.fld[WF_VOO];
    a2 = (const double2*)cp.fld[WF_W];
    b2 = (double2*)cp.fld[WF_WOO];
  }
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n2;
       t += (long)gridDim.x * blockDim.x) {
    b0[t] = a0[t];
    b1[t] = a1[t];
    b2[t] = a2[t];
  }
}
__global__ void k_copy_tail(const double* a0, double* b0, const double* a1, double* b1,
                            const double* a2, double* b2, long idx) {
  pdl_entry();
  b0[idx] = a0[idx];
  b1[idx] = a1[idx];
  b2[idx] = a2[idx];
}

int launch_copy_oo(const wf_case& c, cudaStream_t s) {
  const long tot = padded(c.n) * padded(c.n) * padded(c.n);
  const long n2 = tot / 2;
  WF_CK(launch_k(k_copy3, nblocks(n2, TPB, 148 * 8), TPB, 0, s, 
      (const double2*)c.fld[WF_U], (double2*)c.fld[WF_UOO], (const double2*)c.fld[WF_V],
      (double2*)c.fld[WF_VOO], (const double2*)c.fld[WF_W], (double2*)c.fld[WF_WOO], n2));
  WF_CKL("k_copy3");
  if (tot & 1) {
    WF_CK(launch_k(k_copy_tail, 1, 1, 0, s, c.fld[WF_U], c.fld[WF_UOO], c.fld[WF_V], c.fld[WF_VOO],
                                c.fld[WF_W], c.fld[WF_WOO], tot - 1));
    WF_CKL("k_copy_tail");
  }
  return WF_OK;
}

// --------------------------------------------------------------------------
// WALE eddy viscosity (kernels.py:297-367)
// --------------------------------------------------------------------------
// ls = cw * (dx dy dz)^(1/3) comes from the host (kernels.py:360-361 compute
// it in every thread; one host pow gives the same value without a device
// pow per cell)
__global__ void __launch_bounds__(TPB) k_wale(const wf_case c, Geo g, const Divs dv,
                                             const double ls, const double* rrey_dev,
                                             const Batch bt) {
  pdl_entry();
  const double* u = bt_fld(c, bt, WF_U);
  const double* v = bt_fld(c, bt, WF_V);
  const double* w = bt_fld(c, bt, WF_W);
  double* vis = bt_fld(c, bt, WF_VIS);
  if (bt.tab) rrey_dev = &bt_sc(c, bt)->rrey;
  const long sI = g.sI, sJ = g.sJ;
  {  // one thread per cell: x = k (runs of 32), y = j (groups of 8), z = i
    const int kx_ = blockIdx.x * 32 + threadIdx.x, jy_ = blockIdx.y * 8 + threadIdx.y;
    if (kx_ >= g.n || jy_ >= g.n) return;
    const int k = NPL + kx_;
    const int j = NPL + jy_;
    const int i = NPL + bt_z(bt);
    const long id = g.at(i, j, k);
#define U_(a) LD(u, id + (a))
#define V_(a) LD(v, id + (a))
#define W_(a) LD(w, id + (a))
    const double dudx = div_by_recip(U_(0) - U_(-sI), dv.dh[0], dv.yh[0]);
    const double dudy = div_by_recip(0.25 * (U_(sJ) + U_(-sI + sJ) - U_(-sJ) - U_(-sI - sJ)), dv.dh[1], dv.yh[1]);
    const double dudz = div_by_recip(0.25 * (U_(1) + U_(-sI + 1) - U_(-1) - U_(-sI - 1)), dv.dh[2], dv.yh[2]);
    const double dvdx = div_by_recip(0.25 * (V_(sI) + V_(sI - sJ) - V_(-sI) - V_(-sI - sJ)), dv.dh[0], dv.yh[0]);
    const double dvdy = div_by_recip(V_(0) - V_(-sJ), dv.dh[1], dv.yh[1]);
    const double dvdz = div_by_recip(0.25 * (V_(1) + V_(-sJ + 1) - V_(-1) - V_(-sJ - 1)), dv.dh[2], dv.yh[2]);
    const double dwdx = div_by_recip(0.25 * (W_(sI) + W_(sI - 1) - W_(-sI) - W_(-sI - 1)), dv.dh[0], dv.yh[0]);
    const double dwdy = div_by_recip(0.25 * (W_(sJ) + W_(sJ - 1) - W_(-sJ) - W_(-sJ - 1)), dv.dh[1], dv.yh[1]);
    const double dwdz = div_by_recip(W_(0) - W_(-1), dv.dh[2], dv.yh[2]);
#undef U_
#undef V_
#undef W_
    const double g2xx = dudx * dudx + dudy * dvdx + dudz * dwdx;
    const double g2yy = dvdx * dudy + dvdy * dvdy + dvdz * dwdy;
    const double g2zz = dwdx * dudz + dwdy * dvdz + dwdz * dwdz;
    const double g2xy = dudx * dudy + dudy * dvdy + dudz * dwdy;
    const double g2yx = dvdx * dudx + dvdy * dvdx + dvdz * dwdx;
    const double g2xz = dudx * dudz + dudy * dvdz + dudz * dwdz;
    const double g2zx = dwdx * dudx + dwdy * dvdx + dwdz * dudz;
    const double g2yz = dvdx * dudz + dvdy * dvdz + dvdz * dwdz;
    const double g2zy = dwdx * dudy + dwdy * dvdy + dwdz * dudy;
    const double tr = div_by_recip(g2xx + g2yy + g2zz, dv.d3, dv.y3);
    const double sdxx = g2xx - tr, sdyy = g2yy - tr, sdzz = g2zz - tr;
    const double sdxy = 0.5 * (g2xy + g2yx);
    const double sdxz = 0.5 * (g2xz + g2zx);
    const double sdyz = 0.5 * (g2yz + g2zy);
    const double sdsd = sdxx * sdxx + sdyy * sdyy + sdzz * sdzz +
                        2.0 * (sdxy * sdxy + sdxz * sdxz + sdyz * sdyz);
    const double sxy = 0.5 * (dudy + dvdx);
    const double sxz = 0.5 * (dudz + dwdx);
    const double syz = 0.5 * (dvdz + dwdy);
    const double ss = dudx * dudx + dvdy * dvdy + dwdz * dwdz +
                      2.0 * (sxy * sxy + sxz * sxz + syz * syz);
    // kernels.py:362-365 with x^1.5 = x sqrt(x), x^2.5 = x^2 sqrt(x) and
    // x^1.25 = x sqrt(sqrt(x)) (correctly rounded sqrt; a few ulp from pow)
    double nut = 0.0;
    if (sdsd > 1.0e-8) {
      const double rs = sqrt(sdsd);
      const double sdsd15 = sdsd * rs;
      const double as = fabs(ss);
      const double denom = as * as * sqrt(as) + sdsd * sqrt(rs);
      nut = ls * ls * sdsd15 / denom;
    }
    vis[id] = (rrey_dev ? *rrey_dev : c.rrey) + nut;
  }
}

// vis = 1/Re on real cells (kernels.py:442-449)
__global__ void k_fill_real(double* f, Geo g, double val, const double* valp, const Batch bt) {
  pdl_entry();
  if (bt.tab) {
    f = bt.tab[bt_case(bt)].fld[WF_VIS];
    valp = &bt.tab[bt_case(bt)].sc->rrey;
  }
  if (valp) val = *valp;
  const long tot = (long)g.n * g.n * g.n;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot;
       t += (long)gridDim.x * blockDim.x) {
    const int k = NPL + (int)(t % g.n);
    const int j = NPL + (int)((t / g.n) % g.n);
    const int i = NPL + (int)(t / ((long)g.n * g.n));
    f[g.at(i, j, k)] = val;
  }
}

int launch_wale(const wf_case& c, cudaStream_t s, const double* rrey_dev) {
  Geo g = geo_of(c.n);
  const long tot = (long)c.n * c.n * c.n;
  if (c.sgs) {
    const double ls = c.cw * std::pow(c.dx * c.dy * c.dz, 1.0 / 3.0);
    WF_CK(launch_k(k_wale, cells3(c.n, c.n, c.n), cell_block(), 0, s, c, g, divs_of(c), ls,
                   rrey_dev));
    WF_CKL("k_wale");
    FillReq r{c.fld[WF_VIS], FILL_VIS, c.rrey, rrey_dev, WF_VIS, rrey_dev ? 2 : 0};
    return launch_fills(&r, 1, c.n, s);
  }
  WF_CK(launch_k(k_fill_real, nblocks(tot), TPB, 0, s, c.fld[WF_VIS], g, c.rrey, rrey_dev));
  WF_CKL("k_fill_real");
  return WF_OK;
}

// --------------------------------------------------------------------------
// convection (kernels.py:53-168) and diffusion (kernels.py:177-225)
// --------------------------------------------------------------------------
// 4th-order interpolation I at `id` along stride s (kernels.py:31-46)
__device__ __forceinline__ double I4(const double* f, long id, long s) {
  return (-LD(f, id + s) + 9.0 * LD(f, id) + 9.0 * LD(f, id - s) - LD(f, id - 2 * s)) / 16.0;
}

// op-range dims (solver.py:99-110): the component's own axis is n-1 long
__host__ __device__ __forceinline__ void op_dims(int comp, int n, int& ni, int& nj, int& nk) {
  ni = nj = nk = n;
  if (comp == 0) ni = n - 1;
  if (comp == 1) nj = n - 1;
  if (comp == 2) nk = n - 1;
}

__device__ __forceinline__ double lap1(const double* f, long id, long s, double d,
                                       double y) {
  return div_by_recip(-LD(f, id + 2 * s) + 16.0 * LD(f, id + s) - 30.0 * LD(f, id) +
                          16.0 * LD(f, id - s) - LD(f, id - 2 * s),
                      d, y);
}

// star + dt*alpha*diff (kernels.py:221-225), the one form both the separate
// diffusion and the diffusion fused into the convection use
__device__ __forceinline__ double diff_add(double star, double dt, double alpha, double diff) {
  return star + dt * alpha * diff;
}

// vis * lap4(f) at cell id of component COMP (kernels.py:189-225); f the
// component, vis the viscosity field
template <int COMP>
__device__ __forceinline__ double diff_term(const double* f, const double* vis, long sI,
                                            long sJ, const Divs& dv, long id) {
  const long vofs = COMP == 0 ? 0 : (COMP == 1 ? sJ : 1);
  const double l4 = lap1(f, id, sI, dv.d12[0], dv.y12[0]) +
                    lap1(f, id, sJ, dv.d12[1], dv.y12[1]) + lap1(f, id, 1, dv.d12[2], dv.y12[2]);
  return LD(vis, id + vofs) * l4;
}

// one cell (i0, j0, k0 from 0 within the op range) of component COMP
template <int COMP>
__device__ __forceinline__ void diff_cell(const wf_case& c, const Geo& g, double alpha,
                                          double dt, const Divs& dv, int i0, int j0, int k0) {
  double* star = c.fld[WF_USTAR + COMP];
  const long id = g.at(NPL + i0, NPL + j0, NPL + k0);
  star[id] = diff_add(star[id], dt, alpha,
                      diff_term<COMP>(c.fld[WF_U + COMP], c.fld[WF_VIS], g.sI, g.sJ, dv, id));
}

// PC: the padded extent n + 6 as a compile-time constant for the common
// sizes (0: read from g), so that every neighbour load is one base address
// plus an immediate offset instead of a runtime 64-bit address sum -- the
// pass is instruction-bound; the arithmetic is the same.
// DIFF: also add the component's diffusion to star in the same pass.  The
// step's fill of the component between its convection and its diffusion
// (solver.py:253-263) changes only ghost cells that lie outside the grid in
// two or more directions -- its other ghost cells are functions of real
// cells, which do not change in between -- and the diffusion stencil never
// reaches such cells, so the fused update reads the same values and gives
// the same star.
template <int COMP, bool DIFF, int PC>
__global__ void __launch_bounds__(TPB) k_conv(const wf_case c, Geo g, double alpha,
                                             const double* dtp, const Divs dv, int planes,
                                             const Batch bt) {
  pdl_entry();
  const double* u = bt_fld(c, bt, WF_U);
  const double* v = bt_fld(c, bt, WF_V);
  const double* w = bt_fld(c, bt, WF_W);
  const double* oo = bt_fld(c, bt, WF_UOO + COMP);
  double* star = bt_fld(c, bt, WF_USTAR + COMP);
  if (bt.tab) dtp = &bt_sc(c, bt)->dt;
  const double dt = *dtp;
  const long X = PC ? (long)PC * PC : g.sI, Y = PC ? (long)PC : g.sJ, Z = 1;
  int ni, nj, nk;
  op_dims(COMP, PC ? PC - 2 * NPL : g.n, ni, nj, nk);
  // one thread per (j, k) column and `planes` consecutive planes i: x = k,
  // y = j (the CTA's shape and the planes are chosen per size, 32 x 8 x 1 by
  // default), z = group of planes.  A CTA that walks through several planes
  // finds a cell's neighbours across i in L1, loaded for the planes before.
  const int kx_ = blockIdx.x * blockDim.x + threadIdx.x;
  const int jy_ = blockIdx.y * blockDim.y + threadIdx.y;
  if (kx_ >= nk || jy_ >= nj) return;
  const int k = NPL + kx_;
  const int j = NPL + jy_;
  const int i_end = min(ni, (bt_z(bt) + 1) * planes);
#pragma unroll 1
  for (int ii = bt_z(bt) * planes; ii < i_end; ++ii) {
    const int i = NPL + ii;
    const long id = (long)i * X + (long)j * Y + k;
    double tot3;
    if (COMP == 0) {
      double a;
      a = I4(u, id + 2 * X, X); const double sp2 = a * a;
      a = I4(u, id + X, X); const double sp1 = a * a;
      a = I4(u, id, X); const double sn = a * a;
      a = I4(u, id - X, X); const double sm1 = a * a;
      const double du2dx = div_by_recip(-sp2 + 27.0 * sp1 - 27.0 * sn + sm1, dv.d24[0], dv.y24[0]);
      double p1 = I4(u, id + 2 * Y, Y) * I4(v, id + X + Y, X);
      double p0 = I4(u, id + Y, Y) * I4(v, id + X, X);
      double m1 = I4(u, id, Y) * I4(v, id + X - Y, X);
      double m2 = I4(u, id - Y, Y) * I4(v, id + X - 2 * Y, X);
      const double duvdy = div_by_recip(-p1 + 27.0 * p0 - 27.0 * m1 + m2, dv.d24[1], dv.y24[1]);
      p1 = I4(u, id + 2 * Z, Z) * I4(w, id + X + Z, X);
      p0 = I4(u, id + Z, Z) * I4(w, id + X, X);
      m1 = I4(u, id, Z) * I4(w, id + X - Z, X);
      m2 = I4(u, id - Z, Z) * I4(w, id + X - 2 * Z, X);
      const double duwdz = div_by_recip(-p1 + 27.0 * p0 - 27.0 * m1 + m2, dv.d24[2], dv.y24[2]);
      tot3 = du2dx + duvdy + duwdz;
    } else if (COMP == 1) {
      double a;
      a = I4(v, id + 2 * Y, Y); const double sp2 = a * a;
      a = I4(v, id + Y, Y); const double sp1 = a * a;
      a = I4(v, id, Y); const double sn = a * a;
      a = I4(v, id - Y, Y); const double sm1 = a * a;
      const double dv2dy = div_by_recip(-sp2 + 27.0 * sp1 - 27.0 * sn + sm1, dv.d24[1], dv.y24[1]);
      double p1 = I4(v, id + 2 * X, X) * I4(u, id + X + Y, Y);
      double p0 = I4(v, id + X, X) * I4(u, id + Y, Y);
      double m1 = I4(v, id, X) * I4(u, id - X + Y, Y);
      double m2 = I4(v, id - X, X) * I4(u, id - 2 * X + Y, Y);
      const double duvdx = div_by_recip(-p1 + 27.0 * p0 - 27.0 * m1 + m2, dv.d24[0], dv.y24[0]);
      p1 = I4(v, id + 2 * Z, Z) * I4(w, id + Y + Z, Y);
      p0 = I4(v, id + Z, Z) * I4(w, id + Y, Y);
      m1 = I4(v, id, Z) * I4(w, id + Y - Z, Y);
      m2 = I4(v, id - Z, Z) * I4(w, id + Y - 2 * Z, Y);
      const double dvwdz = div_by_recip(-p1 + 27.0 * p0 - 27.0 * m1 + m2, dv.d24[2], dv.y24[2]);
      tot3 = duvdx + dv2dy + dvwdz;
    } else {
      double a;
      a = I4(w, id + 2 * Z, Z); const double sp2 = a * a;
      a = I4(w, id + Z, Z); const double sp1 = a * a;
      a = I4(w, id, Z); const double sn = a * a;
      a = I4(w, id - Z, Z); const double sm1 = a * a;
      const double dw2dz = div_by_recip(-sp2 + 27.0 * sp1 - 27.0 * sn + sm1, dv.d24[2], dv.y24[2]);
      double p1 = I4(w, id + 2 * X, X) * I4(u, id + X + Z, Z);
      double p0 = I4(w, id + X, X) * I4(u, id + Z, Z);
      double m1 = I4(w, id, X) * I4(u, id - X + Z, Z);
      double m2 = I4(w, id - X, X) * I4(u, id - 2 * X + Z, Z);
      const double duwdx = div_by_recip(-p1 + 27.0 * p0 - 27.0 * m1 + m2, dv.d24[0], dv.y24[0]);
      p1 = I4(w, id + 2 * Y, Y) * I4(v, id + Y + Z, Z);
      p0 = I4(w, id + Y, Y) * I4(v, id + Z, Z);
      m1 = I4(w, id, Y) * I4(v, id - Y + Z, Z);
      m2 = I4(w, id - Y, Y) * I4(v, id - 2 * Y + Z, Z);
      const double dvwdy = div_by_recip(-p1 + 27.0 * p0 - 27.0 * m1 + m2, dv.d24[1], dv.y24[1]);
      tot3 = duwdx + dvwdy + dw2dz;
    }
    const double s1 = LD(oo, id) - dt * alpha * tot3;
    star[id] = DIFF ? diff_add(s1, dt, alpha,
                               diff_term<COMP>(COMP == 0 ? u : (COMP == 1 ? v : w),
                                               bt_fld(c, bt, WF_VIS), X, Y, dv, id))
                    : s1;
  }
}

template <int COMP>
__global__ void __launch_bounds__(TPB) k_diff(const wf_case c, Geo g, double alpha,
                                             const double* dtp, const Divs dv) {
  pdl_entry();
  int ni, nj, nk;
  op_dims(COMP, g.n, ni, nj, nk);
  // one thread per cell: x = k (runs of 32), y = j (groups of 8), z = i
  const int kx_ = blockIdx.x * 32 + threadIdx.x, jy_ = blockIdx.y * 8 + threadIdx.y;
  if (kx_ >= nk || jy_ >= nj) return;
  diff_cell<COMP>(c, g, alpha, *dtp, dv, (int)blockIdx.z, jy_, kx_);
}


// ---- launch shapes per size ------------------------------------------------
// 0 = the default: k_conv 32 x 8 threads (a warp along k, 8 rows j), one
// plane i per thread; k_rbgs_split 2 cells per thread (WF_SPLIT_CPT
// overrides), 8 rows per CTA
static constexpr int SHAPE_MAX_N = 1024;
static int g_shape[2][SHAPE_MAX_N + 1][3];

// built-in shapes by size, from the tuner's measurements on B200 (80^3,
// 128^3, 256^3): the convection pass walks more planes per thread as the
// grid grows (neighbours across i found in L1), and the split half-sweep of
// large levels takes 4 cells per thread in CTAs of 2 rows
// (us per pass / half-sweep, default -> tuned: conv 39.5 -> 35.8 at 80,
// 145.6 -> 131.2 at 128, 1019 -> 855 at 256; split 3.57 -> 3.29 at 80,
// 51.7 -> 41.5 at 256)
static void shape_default(int kind, int n, int* a, int* b, int* c) {
  if (kind == SHAPE_CONV) {
    *a = 32;
    *b = n >= 64 ? 4 : 8;
    *c = n >= 192 ? 4 : (n >= 64 ? 2 : 1);
  } else {
    const char* e = getenv("WF_SPLIT_CPT");
    const int forced = e ? atoi(e) : 0;
    *a = (forced == 1 || forced == 2 || forced == 4 || forced == 8) ? forced
                                                                    : (n >= 192 || n < 100 ? 4 : 2);
    *b = n >= 192 ? 2 : 8;
    *c = 1;
  }
}

void launch_shape(int kind, int n, int* a, int* b, int* c) {
  const bool set = kind >= 0 && kind <= 1 && n >= 0 && n <= SHAPE_MAX_N && g_shape[kind][n][0];
  shape_default(kind, n, a, b, c);
  if (set) {
    *a = g_shape[kind][n][0];
    *b = g_shape[kind][n][1];
    *c = kind == SHAPE_CONV ? g_shape[kind][n][2] : 1;
  }
}

int set_launch_shape(int kind, int n, int a, int b, int c) {
  if (n < 4 || n > SHAPE_MAX_N) return fail(WF_EINVAL, "wf_set_launch_shape: n in 4..1024");
  if (kind != SHAPE_CONV && kind != SHAPE_SPLIT)
    return fail(WF_EINVAL, "wf_set_launch_shape: kind 0 (k_conv) or 1 (k_rbgs_split)");
  if (a == 0 && b == 0 && c == 0) {
    g_shape[kind][n][0] = g_shape[kind][n][1] = g_shape[kind][n][2] = 0;
    return WF_OK;
  }
  if (kind == SHAPE_CONV) {
    // whole warps, at most TPB threads (the kernel's launch bound)
    if (a < 1 || b < 1 || a > 256 || (a & (a - 1)) || a * b > TPB || (a * b) % 32 || c < 1 ||
        c > 16)
      return fail(WF_EINVAL, "wf_set_launch_shape(k_conv): a a power of two, a*b a multiple "
                             "of 32 and at most 256, c in 1..16");
  } else if ((a != 1 && a != 2 && a != 4 && a != 8) || (b != 1 && b != 2 && b != 4 && b != 8) ||
             c != 1) {
    return fail(WF_EINVAL,
                "wf_set_launch_shape(k_rbgs_split): a in {1,2,4,8}, b in {1,2,4,8}, c = 1");
  }
  g_shape[kind][n][0] = a;
  g_shape[kind][n][1] = b;
  g_shape[kind][n][2] = c;
  return WF_OK;
}

int launch_conv(const wf_case& c, int comp, double alpha, const double* dt,
                cudaStream_t s, bool with_diff) {
  Geo g = geo_of(c.n);
  int ni, nj, nk;
  op_dims(comp, c.n, ni, nj, nk);
  int bx, by, planes;
  launch_shape(SHAPE_CONV, c.n, &bx, &by, &planes);
  const dim3 gr((nk + bx - 1) / bx, (nj + by - 1) / by, (ni + planes - 1) / planes), bl(bx, by);
  if (comp < 0 || comp > 2) return fail(WF_EINVAL, "conv: comp must be 0, 1 or 2");
  using KC = void (*)(const wf_case, Geo, double, const double*, const Divs, int, const Batch);
  static const KC kern[3][2][3] = {
      {{k_conv<0, false, 0>, k_conv<1, false, 0>, k_conv<2, false, 0>},
       {k_conv<0, true, 0>, k_conv<1, true, 0>, k_conv<2, true, 0>}},
      {{k_conv<0, false, 86>, k_conv<1, false, 86>, k_conv<2, false, 86>},
       {k_conv<0, true, 86>, k_conv<1, true, 86>, k_conv<2, true, 86>}},
      {{k_conv<0, false, 262>, k_conv<1, false, 262>, k_conv<2, false, 262>},
       {k_conv<0, true, 262>, k_conv<1, true, 262>, k_conv<2, true, 262>}}};
  // the size-specialised forms (80^3 and 256^3); WF_CONV_PC=0 keeps the generic one
  static int spec = -1;
  if (spec < 0) {
    const char* e = getenv("WF_CONV_PC");
    spec = (e && e[0] == '0') ? 0 : 1;
  }
  const int form = !spec ? 0 : (c.n == 80 ? 1 : (c.n == 256 ? 2 : 0));
  WF_CK(launch_k(kern[form][with_diff ? 1 : 0][comp], gr, bl, 0, s, c, g, alpha, dt, divs_of(c),
                 planes));
  WF_CKL("k_conv");
  return WF_OK;
}

int launch_diff(const wf_case& c, int comp, double alpha, const double* dt,
                cudaStream_t s) {
  Geo g = geo_of(c.n);
  const long tot = (long)c.n * c.n * (c.n - 1);
  const int nb = nblocks(tot);
  int ni, nj, nk;
  op_dims(comp, c.n, ni, nj, nk);
  const dim3 gr = cells3(ni, nj, nk), bl = cell_block();
  if (comp == 0) WF_CK(launch_k(k_diff<0>, gr, bl, 0, s, c, g, alpha, dt, divs_of(c)));
  else if (comp == 1) WF_CK(launch_k(k_diff<1>, gr, bl, 0, s, c, g, alpha, dt, divs_of(c)));
  else if (comp == 2) WF_CK(launch_k(k_diff<2>, gr, bl, 0, s, c, g, alpha, dt, divs_of(c)));
  else return fail(WF_EINVAL, "diff: comp must be 0, 1 or 2");
  WF_CKL("k_diff");
  return WF_OK;
}


// --------------------------------------------------------------------------
// calvel (kernels.py:232-264): the three components in one launch
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(TPB) k_calvel(const wf_case c, Geo g, double alpha,
                                               const double* dtp, const Divs dv,
                                               const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const double* p = bt_fld(c, bt, WF_P);
  if (bt.tab) dtp = &bt_sc(c, bt)->dt;
  const double dt = *dtp;
  double* fu = bt_fld(c, bt, WF_U);
  double* fv = bt_fld(c, bt, WF_V);
  double* fw = bt_fld(c, bt, WF_W);
  const double* us = bt_fld(c, bt, WF_USTAR);
  const double* vs = bt_fld(c, bt, WF_VSTAR);
  const double* ws = bt_fld(c, bt, WF_WSTAR);
  const int hi = NPL + g.n - 1;  // last real index; the component's own axis stops before it
  {  // one thread per cell: x = k (runs of 32), y = j (groups of 8), z = i
    const int kx_ = blockIdx.x * 32 + threadIdx.x, jy_ = blockIdx.y * 8 + threadIdx.y;
    if (kx_ >= g.n || jy_ >= g.n) return;
    const int k = NPL + kx_;
    const int j = NPL + jy_;
    const int i = NPL + bt_z(bt);
    const long id = g.at(i, j, k);
    // every load before the first store: the stores go through pointers the
    // compiler cannot separate from the loads, so a load placed after a
    // store would wait for the round trip of the loads before it
    const double p0 = LD(p, id);
    const double pi1 = LD(p, id + g.sI), pj1 = LD(p, id + g.sJ), pk1 = LD(p, id + 1);
    const double u0 = LD(us, id), v0 = LD(vs, id), w0 = LD(ws, id);
    if (i < hi) fu[id] = u0 - div_by_recip(dt * alpha * (pi1 - p0), dv.dh[0], dv.yh[0]);
    if (j < hi) fv[id] = v0 - div_by_recip(dt * alpha * (pj1 - p0), dv.dh[1], dv.yh[1]);
    if (k < hi) fw[id] = w0 - div_by_recip(dt * alpha * (pk1 - p0), dv.dh[2], dv.yh[2]);
  }
}

int launch_calvel(const wf_case& c, double alpha, const double* dt, cudaStream_t s) {
  Geo g = geo_of(c.n);
  WF_CK(launch_k(k_calvel, cells3(c.n, c.n, c.n), cell_block(), 0, s, c, g, alpha, dt, divs_of(c)));
  WF_CKL("k_calvel");
  return WF_OK;
}

// one case of a bucket reports its loop decision (wf_scalars.loop bits:
// 1 continue, 2 run the multigrid part); the last case to report sets the
// bucket loop's graph conditions from the OR of all decisions and resets
// the count (kept in the first case's scalar block)
__device__ __forceinline__ void bucket_report(const Batch& bt, int loop,
                                              unsigned long long h_if,
                                              unsigned long long h_loop) {
  wf_scalars* s0 = bt.tab[0].sc;
  const unsigned ncases = gridDim.z / (unsigned)bt.nz;
  atomicOr((unsigned*)&s0->bflags, (unsigned)loop);
  __threadfence();
  if (atomicAdd(&s0->bticket, 1u) != ncases - 1) return;
  __threadfence();
  const unsigned any = atomicExch((unsigned*)&s0->bflags, 0u);
  s0->bticket = 0u;
  if (h_if) cudaGraphSetConditional((cudaGraphConditionalHandle)h_if, (any & 2) ? 1u : 0u);
  if (h_loop) cudaGraphSetConditional((cudaGraphConditionalHandle)h_loop, (any & 1) ? 1u : 0u);
}

// --------------------------------------------------------------------------
// calmas (kernels.py:271-289) + one iteration of the projection control
// (solver.py:185-209), decided by the last block on the device
// --------------------------------------------------------------------------
// In a bucket (bt.tab set) a case whose loop has ended does no work: one of
// its blocks only reports it to the bucket; the conditions of the bucket's
// loop are set by whichever case reports last, from the OR of all cases'
// decisions (collected in the first case's scalar block).
__global__ void __launch_bounds__(TPB) k_calmas(const wf_case c, Geo g,
                                               unsigned long long h_if,
                                               unsigned long long h_loop, const Divs dv,
                                               const Batch bt) {
  pdl_entry();
  __shared__ double sm[32];
  const double* u = bt_fld(c, bt, WF_U);
  const double* v = bt_fld(c, bt, WF_V);
  const double* w = bt_fld(c, bt, WF_W);
  double* su = bt_fld(c, bt, WF_SU);
  wf_scalars* sc = bt_sc(c, bt);
  if (bt.tab && !(sc->loop & 1)) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && bt_z(bt) == 0 && threadIdx.x == 0)
      bucket_report(bt, 0, h_if, h_loop);
    return;
  }
  const double dt = sc->dt;
  const double rdt = 1.0 / dt;   // fact / dt below as div_by_recip(fact, dt, rdt)
  const double dx = c.dx, dy = c.dy, dz = c.dz;
  double mloc = 0.0;
  const int k = NPL + blockIdx.x * 32 + (threadIdx.x & 31);
  const int j = NPL + blockIdx.y * 8 + (threadIdx.x >> 5);
  const bool in = k < NPL + g.n && j < NPL + g.n;
  for (int i = NPL + bt_z(bt); in && i < NPL + g.n; i += bt_gz(bt)) {
    const long id = g.at(i, j, k);
    const long X = g.sI, Y = g.sJ;
    const double dudx = div_by_recip(-LD(u, id + X) + 27.0 * LD(u, id) - 27.0 * LD(u, id - X) +
                                         LD(u, id - 2 * X), dv.d24[0], dv.y24[0]);
    const double dvdy = div_by_recip(-LD(v, id + Y) + 27.0 * LD(v, id) - 27.0 * LD(v, id - Y) +
                                         LD(v, id - 2 * Y), dv.d24[1], dv.y24[1]);
    const double dwdz = div_by_recip(-LD(w, id + 1) + 27.0 * LD(w, id) - 27.0 * LD(w, id - 1) +
                                         LD(w, id - 2), dv.d24[2], dv.y24[2]);
    const double fact = dudx + dvdy + dwdz;
    su[id] = div_by_recip(fact, dt, rdt);
    mloc = fmax(mloc, fabs(fact * dx * dy * dz));
  }
  mloc = block_max(mloc, sm);
  if (threadIdx.x == 0) atomicMax(&sc->red[4], okey(mloc));
  if (!last_block(&sc->ticket, gridDim.x * gridDim.y * bt_gz(bt))) return;
  if (threadIdx.x != 0) return;
  const double rmax = okey_inv(atomicAdd(&sc->red[4], 0ull));
  sc->red[4] = okey(0.0);
  sc->rmax = rmax;
  const int it = ++sc->iters;
  if (it <= 32) sc->rmax_trace[it - 1] = rmax;
  const bool conv = (it > 1) && (rmax < c.eps);
  const bool div = !conv && (rmax > 10.0);
  const bool run = !conv && !div;
  if (div) sc->status = WF_ST_DIVERGED;
  if (run) sc->nmg += 1;
  if (run && it >= c.maxcy && sc->status == WF_ST_OK) sc->status = WF_ST_NOT_CONVERGED;
  const int more = (run && it < c.maxcy) ? 1 : 0;
  sc->loop = (run ? 2 : 0) | more;
  if (bt.tab) {
    bucket_report(bt, sc->loop, h_if, h_loop);
    return;
  }
  if (h_if) cudaGraphSetConditional((cudaGraphConditionalHandle)h_if, run ? 1u : 0u);
  if (h_loop) cudaGraphSetConditional((cudaGraphConditionalHandle)h_loop, (unsigned)more);
}

int launch_calmas(const wf_case& c, unsigned long long h_if, unsigned long long h_loop,
                  cudaStream_t s) {
  Geo g = geo_of(c.n);
  WF_CK(launch_k(k_calmas, reduce_grid(c.n), TPB, 0, s, c, g, h_if, h_loop, divs_of(c)));
  WF_CKL("k_calmas");
  return WF_OK;
}

// --------------------------------------------------------------------------
// p += pp over real cells plus one ring (kernels.py:405-414)
// --------------------------------------------------------------------------
__global__ void k_add_ring(double* p, const double* pp, Geo g, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  if (bt.tab) {
    p = bt.tab[bt_case(bt)].fld[WF_P];
    pp = bt.tab[bt_case(bt)].fld[WF_PP];
  }
  const int m = g.n + 2;
  {  // one thread per cell: x = k (runs of 32), y = j (groups of 8), z = i
    const int kx_ = blockIdx.x * 32 + threadIdx.x, jy_ = blockIdx.y * 8 + threadIdx.y;
    if (kx_ >= m || jy_ >= m) return;
    const int k = NPL - 1 + kx_;
    const int j = NPL - 1 + jy_;
    const int i = NPL - 1 + bt_z(bt);
    const long id = g.at(i, j, k);
    p[id] = p[id] + pp[id];
  }
}

int launch_add_ring(double* p, const double* pp, int n, cudaStream_t s) {
  Geo g = geo_of(n);
  WF_CK(launch_k(k_add_ring, cells3(n + 2, n + 2, n + 2), cell_block(), 0, s, p, pp, g));
  WF_CKL("k_add_ring");
  return WF_OK;
}


// --------------------------------------------------------------------------
// halo slabs of a sub-domain (reference halo.py:16-55 gather/scatter): a box
// of a strided 3-D array (k contiguous) to and from a dense buffer ordered
// [i][j][k], so a slab along any axis is one contiguous message
// --------------------------------------------------------------------------
__global__ void k_box(double* arr, long sI, long sJ, int i0, int j0, int k0, int ni, int nj,
                      int nk, double* buf, int unpack) {
  pdl_entry();
  const long tot = (long)ni * nj * nk;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot;
       t += (long)gridDim.x * blockDim.x) {
    const int k = (int)(t % nk);
    const long r = t / nk;
    const int j = (int)(r % nj), i = (int)(r / nj);
    const long a = (long)(i0 + i) * sI + (long)(j0 + j) * sJ + (k0 + k);
    if (unpack)
      arr[a] = buf[t];
    else
      buf[t] = arr[a];
  }
}

int launch_box(double* arr, long sI, long sJ, int i0, int j0, int k0, int ni, int nj, int nk,
               double* buf, int unpack, cudaStream_t s) {
  if (!arr || !buf) return fail(WF_EINVAL, "null array or buffer");
  if (ni < 0 || nj < 0 || nk < 0 || i0 < 0 || j0 < 0 || k0 < 0 || sJ < nk + k0 || sI < sJ)
    return fail(WF_EINVAL, "box out of range");
  const long tot = (long)ni * nj * nk;
  if (tot == 0) return WF_OK;
  WF_CK(launch_k(k_box, nblocks(tot), TPB, 0, s, arr, sI, sJ, i0, j0, k0, ni, nj, nk, buf,
                 unpack));
  WF_CKL("k_box");
  return WF_OK;
}

}  // namespace wf
