// Geometric multigrid for the pressure Poisson equation (reference
// multigrid.py): 7-point Neumann operator with the boundary coefficients
// zeroed (multigrid.py:23-67), red-black Gauss-Seidel with one ring refill
// per full sweep (multigrid.py:70-90, 289-299), full-weighting residual
// restriction (93-119), trilinear prolongation (122-146) and the fixed
// V-cycle schedule (301-337).
//
// No coefficient arrays: the face coefficient is 1/h^2 of the level or 0
// across a physical face, decided from the cell index.
//
// Ring refill fused into the updates: a ring cell of a face has exactly one
// real neighbour and is multiplied by a zero coefficient everywhere, so the
// thread that updates that neighbour writes the mirror right away.  At the
// end of each sweep (and after prolongation) the ring therefore holds what
// the reference's separate refill launch writes; edge and corner ring cells
// are never written, as in bcs.py:326-360.
//
// Level 0 works in place: phi is the (n+2)^3 core of `pp` and rhs the core
// of `su`, both with the padded (n+6) strides.
#include <cooperative_groups.h>
#include <cuda.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "wf_dev.cuh"
#include "wf_internal.h"

namespace wf {

constexpr int MG_TPB = 256;

template <class T>
struct Lvl {
  T* phi;        // ring cell (0,0,0)
  const T* rhs;  // same layout as phi
  int n;         // real cells per axis
  long sI, sJ;   // strides (k stride 1)
  T ax, ay, az;  // 1/h^2 per axis of this level
  int* err;      // where a device-side wait records a timeout (may be null)
  T* tmp;        // scratch of two level arrays: split copies / one-launch sweeps (may be null)
  long tI, tJ;   // its strides
  unsigned* gbar;  // two words of grid-barrier state (may be null)
  int split = 0;   // phi/rhs stored row-parity split (see k_rbgs_split)
  // where the level's arrays sit in a case's buffers, so that a bucket launch
  // can find them for every case: bits 0-3 the level; LV_PP the FP64 level 0
  // inside pp (phi) and su (rhs); LV_SPLIT the split copies in mg_tmp;
  // otherwise mg_phi / mg_rhs of the level
  int role = 0;
};
constexpr int LV_PP = 16, LV_SPLIT = 32;

// the level L of the case this block serves in a bucket launch (L itself
// outside one)
template <class T>
__device__ __forceinline__ Lvl<T> rebase(const Lvl<T>& L, const Batch& bt) {
  if (!bt.tab) return L;
  const CasePtrs& cp = bt.tab[bt_case(bt)];
  Lvl<T> R = L;
  const int l = L.role & 15;
  const long m = (long)L.n + 2;
  T* tmp = (T*)cp.mg_tmp[l];
  if (L.role & LV_SPLIT) {
    R.phi = tmp;
    R.rhs = tmp + m * m * m;
  } else if (L.role & LV_PP) {
    const long P = (long)L.n + 2 * NPL;
    const long off = (long)(NPL - 1) * (P * P + P + 1);
    R.phi = (T*)(cp.fld[WF_PP] + off);
    R.rhs = (const T*)(cp.fld[WF_SU] + off);
  } else {
    R.phi = (T*)cp.mg_phi[l];
    R.rhs = (const T*)cp.mg_rhs[l];
  }
  R.tmp = tmp;
  R.err = &cp.sc->status;
  R.gbar = cp.sc->gbar;
  return R;
}

// position of array index a within a row of the row-parity-split layout
__host__ __device__ __forceinline__ int spos(int a, int H) { return (a & 1) * H + (a >> 1); }

template <class T>
__device__ __forceinline__ long lid(const Lvl<T>& L, int i, int j, int k) {
  return (long)i * L.sI + (long)j * L.sJ + (L.split ? spos(k, (L.n + 2) >> 1) : k);
}

// write the face-ring mirrors of real cell (i,j,k) (0-based) with value x
template <class T>
__device__ __forceinline__ void ring_mirror(const Lvl<T>& L, int i, int j, int k, long c,
                                            T x) {
  const int n = L.n;
  if (i == 0) L.phi[c - L.sI] = x;
  if (i == n - 1) L.phi[c + L.sI] = x;
  if (j == 0) L.phi[c - L.sJ] = x;
  if (j == n - 1) L.phi[c + L.sJ] = x;
  if (k == 0) L.phi[c - 1] = x;
  if (k == n - 1) L.phi[c + 1] = x;
}


// RN(1/ap) for every boundary pattern of a cell: index 9*cx + 3*cy + cz,
// c = number of non-zero coefficients along the axis (0, 1 or 2).  ap is
// summed in the kernels' order; zero terms do not change an IEEE sum, so
// the pattern counts fix ap exactly.
template <class T>
struct ApRecip {
  T y[27];
};

template <class T>
static ApRecip<T> ap_recip(const Lvl<T>& L) {
  ApRecip<T> t;
  for (int cx = 0; cx < 3; ++cx)
    for (int cy = 0; cy < 3; ++cy)
      for (int cz = 0; cz < 3; ++cz) {
        const T aw = cx > 0 ? L.ax : T(0), ae = cx > 1 ? L.ax : T(0);
        const T as = cy > 0 ? L.ay : T(0), an = cy > 1 ? L.ay : T(0);
        const T ab = cz > 0 ? L.az : T(0), at = cz > 1 ? L.az : T(0);
        const T ap = -(aw + ae + as + an + ab + at);
        t.y[9 * cx + 3 * cy + cz] = ap != T(0) ? T(1) / ap : T(0);
      }
  return t;
}

// one colour half-sweep (multigrid.py:70-90): update where (i+j+k+color)%2==1
template <class T>
__global__ void __launch_bounds__(MG_TPB) k_rbgs(const Lvl<T> L0, int color, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> L = rebase(L0, bt);
  const int n = L.n;
  const int nh = (n + 1) >> 1;
  {  // one thread per cell: x = kk (runs of 32), y = j (groups of 8), z = i
    const int kx_ = blockIdx.x * 32 + threadIdx.x, jy_ = blockIdx.y * 8 + threadIdx.y;
    if (kx_ >= nh || jy_ >= n) return;
    const int kk = kx_;
    const int j = jy_;
    const int i = bt_z(bt);
    const int k = 2 * kk + ((1 + i + j + color) & 1);
    if (k >= n) return;
    const long c = lid(L, i + 1, j + 1, k + 1);
    const T aw = i > 0 ? L.ax : T(0), ae = i < n - 1 ? L.ax : T(0);
    const T as = j > 0 ? L.ay : T(0), an = j < n - 1 ? L.ay : T(0);
    const T ab = k > 0 ? L.az : T(0), at = k < n - 1 ? L.az : T(0);
    const T ap = -(aw + ae + as + an + ab + at);
    const T* phi = L.phi;
    const T s = aw * phi[c - L.sI] + ae * phi[c + L.sI] + as * phi[c - L.sJ] +
                an * phi[c + L.sJ] + ab * phi[c - 1] + at * phi[c + 1];
    const T x = (L.rhs[c] - s) / ap;
    L.phi[c] = x;
    ring_mirror(L, i, j, k, c, x);
  }
}

// restriction (multigrid.py:93-119): rhs_c = 1/8 sum of the 8 fine residuals;
// also zeroes the coarse level's phi, ring included
template <class T>
__global__ void __launch_bounds__(MG_TPB) k_restrict(const Lvl<T> F0, T* rhs_c, Lvl<T> C0,
                                                     const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> F = rebase(F0, bt);
  const Lvl<T> C = rebase(C0, bt);
  if (bt.tab) rhs_c = const_cast<T*>(C.rhs);
  const int nc = C.n, n = F.n;
  {  // one thread per cell: x = ck (runs of 32), y = cj (groups of 8), z = ci
    const int kx_ = blockIdx.x * 32 + threadIdx.x, jy_ = blockIdx.y * 8 + threadIdx.y;
    if (kx_ >= nc || jy_ >= nc) return;
    const int ck = kx_;
    const int cj = jy_;
    const int ci = bt_z(bt);
    // the fine phi values the 8 residuals read -- the 2x2x2 block and its
    // face neighbours, P[a][b][c] at fine cell (2ci-1+a, 2cj-1+b, 2ck-1+c)
    // -- each loaded once (32 loads instead of 56)
    const int i0 = 2 * ci, j0 = 2 * cj, k0 = 2 * ck;
    const int H = (n + 2) >> 1;
    long kp[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) kp[q] = F.split ? spos(k0 + q, H) : (k0 + q);
    const T* p = F.phi;
    T P[4][4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if ((a == 0 || a == 3) + (b == 0 || b == 3) + (q == 0 || q == 3) <= 1)
            P[a][b][q] = p[(long)(i0 + a) * F.sI + (long)(j0 + b) * F.sJ + kp[q]];
    T acc = T(0);
#pragma unroll
    for (int di = 0; di < 2; ++di)
#pragma unroll
      for (int dj = 0; dj < 2; ++dj)
#pragma unroll
        for (int dk = 0; dk < 2; ++dk) {
          const int i = i0 + di, j = j0 + dj, k = k0 + dk;
          const T aw = i > 0 ? F.ax : T(0), ae = i < n - 1 ? F.ax : T(0);
          const T as = j > 0 ? F.ay : T(0), an = j < n - 1 ? F.ay : T(0);
          const T ab = k > 0 ? F.az : T(0), at = k < n - 1 ? F.az : T(0);
          const T ap = -(aw + ae + as + an + ab + at);
          const int a = 1 + di, b = 1 + dj, q = 1 + dk;
          const T r = F.rhs[(long)(i + 1) * F.sI + (long)(j + 1) * F.sJ + kp[q]];
          const T res = r - (aw * P[a - 1][b][q] + ae * P[a + 1][b][q] + as * P[a][b - 1][q] +
                             an * P[a][b + 1][q] + ab * P[a][b][q - 1] + at * P[a][b][q + 1] +
                             ap * P[a][b][q]);
          acc = acc + res;
        }
    rhs_c[lid(C, ci + 1, cj + 1, ck + 1)] = acc * T(0.125);
    // the coarse phi starts from zero (multigrid.py:314): this cell and the
    // ring cells nearest to it (faces, edges, corners), so that every cell
    // of the (nc+2)^3 array is zeroed exactly once
    const int zi0 = ci == 0 ? -1 : 0, zi1 = ci == nc - 1 ? 1 : 0;
    const int zj0 = cj == 0 ? -1 : 0, zj1 = cj == nc - 1 ? 1 : 0;
    const int zk0 = ck == 0 ? -1 : 0, zk1 = ck == nc - 1 ? 1 : 0;
    for (int oi = zi0; oi <= zi1; ++oi)
      for (int oj = zj0; oj <= zj1; ++oj)
        for (int ok = zk0; ok <= zk1; ++ok)
          C.phi[lid(C, ci + 1 + oi, cj + 1 + oj, ck + 1 + ok)] = T(0);
  }
}

// zero a whole array (in a bucket launch: field slot `fid` of every case)
template <class T>
__global__ void k_zero(T* a, long cnt, int fid, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  if (bt.tab) a = (T*)bt.tab[bt_case(bt)].fld[fid];
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < cnt;
       t += (long)gridDim.x * blockDim.x)
    a[t] = T(0);
}

// zero a (n+2)^3 block embedded with strides (sI, sJ)
template <class T>
__global__ void k_zero_strided(T* a, int m, long sI, long sJ) {
  pdl_entry();
  const long tot = (long)m * m * m;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot;
       t += (long)gridDim.x * blockDim.x) {
    const int k = (int)(t % m);
    const int j = (int)((t / m) % m);
    const int i = (int)(t / ((long)m * m));
    a[(long)i * sI + (long)j * sJ + k] = T(0);
  }
}

// prolongation (multigrid.py:122-146) + the ring refill that follows it
template <class T>
__global__ void __launch_bounds__(MG_TPB) k_prolong(const Lvl<T> C0, Lvl<T> F0, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> C = rebase(C0, bt);
  const Lvl<T> F = rebase(F0, bt);
  const int n = F.n;
  {  // one thread per cell: x = k (runs of 32), y = j (groups of 8), z = i
    const int kx_ = blockIdx.x * 32 + threadIdx.x, jy_ = blockIdx.y * 8 + threadIdx.y;
    if (kx_ >= n || jy_ >= n) return;
    const int k = kx_;
    const int j = jy_;
    const int i = bt_z(bt);
    const int c0x = (i % 2 == 0) ? i / 2 - 1 : i / 2;
    const T wx0 = (i % 2 == 0) ? T(0.25) : T(0.75);
    const int c0y = (j % 2 == 0) ? j / 2 - 1 : j / 2;
    const T wy0 = (j % 2 == 0) ? T(0.25) : T(0.75);
    const int c0z = (k % 2 == 0) ? k / 2 - 1 : k / 2;
    const T wz0 = (k % 2 == 0) ? T(0.25) : T(0.75);
    T acc = T(0);
#pragma unroll
    for (int di = 0; di < 2; ++di) {
      const T wxi = di == 0 ? wx0 : T(1) - wx0;
#pragma unroll
      for (int dj = 0; dj < 2; ++dj) {
        const T wyj = dj == 0 ? wy0 : T(1) - wy0;
#pragma unroll
        for (int dk = 0; dk < 2; ++dk) {
          const T wzk = dk == 0 ? wz0 : T(1) - wz0;
          acc = acc + wxi * wyj * wzk * C.phi[lid(C, c0x + di + 1, c0y + dj + 1, c0z + dk + 1)];
        }
      }
    }
    const long c = lid(F, i + 1, j + 1, k + 1);
    const T x = F.phi[c] + acc;
    F.phi[c] = x;
    if (!F.split) ring_mirror(F, i, j, k, c, x);
  }
}

// the same prolongation with one thread per COARSE cell writing its 2x2x2
// fine cells from the 27 coarse values around it, each loaded once (27 loads
// for 8 outputs instead of 64); every output sums the same terms in the
// same order as k_prolong, so the results are the same bits.  The 8 fine
// values are loaded before the first store: the stores go through the same
// pointer, so the compiler would otherwise issue each load after the
// previous cell's store, eight dependent memory round trips per thread.
// Loading them first is safe because each fine cell is written by this
// thread only, and ring_mirror writes ring cells, which are never loaded.
template <class T>
__global__ void __launch_bounds__(MG_TPB) k_prolong8(const Lvl<T> C0, Lvl<T> F0, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> C = rebase(C0, bt);
  const Lvl<T> F = rebase(F0, bt);
  const int nc = C.n;
  const int ck = blockIdx.x * 32 + threadIdx.x, cj = blockIdx.y * 8 + threadIdx.y;
  if (ck >= nc || cj >= nc) return;
  const int ci = bt_z(bt);
  const int Hc = (nc + 2) >> 1;
  long kq[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) kq[q] = C.split ? spos(ck + q, Hc) : (ck + q);
  T Q[3][3][3];   // coarse (ci-1+a, cj-1+b, ck-1+q), ring included
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        Q[a][b][q] = C.phi[(long)(ci + a) * C.sI + (long)(cj + b) * C.sJ + kq[q]];
  long fc[2][2][2];
  T fv[2][2][2];
#pragma unroll
  for (int pi = 0; pi < 2; ++pi)
#pragma unroll
    for (int pj = 0; pj < 2; ++pj)
#pragma unroll
      for (int pk = 0; pk < 2; ++pk) {
        fc[pi][pj][pk] = lid(F, 2 * ci + pi + 1, 2 * cj + pj + 1, 2 * ck + pk + 1);
        fv[pi][pj][pk] = F.phi[fc[pi][pj][pk]];
      }
#pragma unroll
  for (int pi = 0; pi < 2; ++pi)
#pragma unroll
    for (int pj = 0; pj < 2; ++pj)
#pragma unroll
      for (int pk = 0; pk < 2; ++pk) {
        const T wx0 = pi == 0 ? T(0.25) : T(0.75);
        const T wy0 = pj == 0 ? T(0.25) : T(0.75);
        const T wz0 = pk == 0 ? T(0.25) : T(0.75);
        T acc = T(0);
#pragma unroll
        for (int di = 0; di < 2; ++di) {
          const T wxi = di == 0 ? wx0 : T(1) - wx0;
#pragma unroll
          for (int dj = 0; dj < 2; ++dj) {
            const T wyj = dj == 0 ? wy0 : T(1) - wy0;
#pragma unroll
            for (int dk = 0; dk < 2; ++dk) {
              const T wzk = dk == 0 ? wz0 : T(1) - wz0;
              acc = acc + wxi * wyj * wzk * Q[pi + di][pj + dj][pk + dk];
            }
          }
        }
        const int i = 2 * ci + pi, j = 2 * cj + pj, k = 2 * ck + pk;
        const long c = fc[pi][pj][pk];
        const T x = fv[pi][pj][pk] + acc;
        F.phi[c] = x;
        if (!F.split) ring_mirror(F, i, j, k, c, x);
      }
}

// ---- a whole relax() of a small level inside one CTA's shared memory ------
// phi and rhs of the real cells live in shared memory ([i][j][k]); the
// ring is not needed there because every ring term has a zero coefficient.
// After the last sweep the interior and the face rings go back to global.
template <class T>
__global__ void __launch_bounds__(1024) k_relax_smem(Lvl<T> L0, int nsweeps, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> L = rebase(L0, bt);
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sphi = reinterpret_cast<T*>(smraw);
  const int n = L.n;
  const int n3 = n * n * n;
  T* srhs = sphi + n3;
  for (int t = threadIdx.x; t < n3; t += blockDim.x) {
    const int k = t % n, j = (t / n) % n, i = t / (n * n);
    const long c = lid(L, i + 1, j + 1, k + 1);
    sphi[t] = L.phi[c];
    srhs[t] = L.rhs[c];
  }
  __syncthreads();
  const int nh = (n + 1) >> 1;
  const int half = n * n * nh;
  const int SI = n * n, SJ = n;
  for (int s = 0; s < nsweeps; ++s) {
    for (int color = 0; color < 2; ++color) {
      for (int t = threadIdx.x; t < half; t += blockDim.x) {
        const int kk = t % nh;
        const int j = (t / nh) % n;
        const int i = t / (nh * n);
        const int k = 2 * kk + ((1 + i + j + color) & 1);
        if (k >= n) continue;
        const int c = i * SI + j * SJ + k;
        const T aw = i > 0 ? L.ax : T(0), ae = i < n - 1 ? L.ax : T(0);
        const T as = j > 0 ? L.ay : T(0), an = j < n - 1 ? L.ay : T(0);
        const T ab = k > 0 ? L.az : T(0), at = k < n - 1 ? L.az : T(0);
        const T ap = -(aw + ae + as + an + ab + at);
        // out-of-range neighbours have a zero coefficient; read a valid
        // cell instead (the product is then exactly zero)
        const T W = sphi[i > 0 ? c - SI : c], E = sphi[i < n - 1 ? c + SI : c];
        const T S = sphi[j > 0 ? c - SJ : c], N = sphi[j < n - 1 ? c + SJ : c];
        const T B = sphi[k > 0 ? c - 1 : c], Tt = sphi[k < n - 1 ? c + 1 : c];
        const T sum = aw * W + ae * E + as * S + an * N + ab * B + at * Tt;
        sphi[c] = (srhs[c] - sum) / ap;
      }
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < n3; t += blockDim.x) {
    const int k = t % n, j = (t / n) % n, i = t / (n * n);
    const long c = lid(L, i + 1, j + 1, k + 1);
    const T x = sphi[t];
    L.phi[c] = x;
    if (nsweeps > 0) ring_mirror(L, i, j, k, c, x);
  }
}

// One colour of one column: the cells k = KP, KP+2, ... of the column.
// Phase 1 gathers the four in-plane neighbour sums of every cell (all loads
// independent), phase 2 updates the column top-down and publishes the new
// values, so no shared-memory store sits between two loads.  The sum keeps
// the reference's term order aw W + ae E + as S + an N + ab B + at T.
template <class T, int NC, int KP, bool RHS_SMEM>
__device__ __forceinline__ void half_sweep_cols(const T* __restrict__ oth, T* __restrict__ own,
                                                int PLANE, int me, int oW, int oE, int oS,
                                                int oN, T aw, T ae, T as, T an, T az, T inv_in,
                                                T inv_lo, T inv_hi, T (&ph)[NC],
                                                const T (&rh)[RHS_SMEM ? 1 : NC],
                                                const T* __restrict__ srh) {
  constexpr int NK = (NC - KP + 1) / 2;
  T nb[NK];
#pragma unroll
  for (int t = 0; t < NK; ++t) {
    const T* pl = oth + (KP + 2 * t) * PLANE;
    nb[t] = aw * pl[oW] + ae * pl[oE] + as * pl[oS] + an * pl[oN];
  }
  T rr[RHS_SMEM ? NK : 1];
  if (RHS_SMEM) {
#pragma unroll
    for (int t = 0; t < NK; ++t) rr[RHS_SMEM ? t : 0] = srh[(KP + 2 * t) * PLANE + me];
  }
#pragma unroll
  for (int t = 0; t < NK; ++t) {
    const int k = KP + 2 * t;
    T sum = nb[t];
    if (k > 0) sum = sum + az * ph[k - 1];
    if (k < NC - 1) sum = sum + az * ph[k + 1];
    const T r = RHS_SMEM ? rr[RHS_SMEM ? t : 0] : rh[RHS_SMEM ? 0 : k];
    const T x = (r - sum) * (k == 0 ? inv_lo : (k == NC - 1 ? inv_hi : inv_in));
    ph[k] = x;
  }
#pragma unroll
  for (int t = 0; t < NK; ++t) own[(KP + 2 * t) * PLANE + me] = ph[KP + 2 * t];
}

// ---- the coarse level: many sweeps of an even n <= 24 in one CTA ----------
// One thread per (i,j) column.  Columns are split by the parity of i+j into
// two groups of warps, so within a warp every thread updates the same k
// parity in a given half-sweep (no divergence, register indices fixed at
// compile time).  The column's phi and rhs live in registers; phi is also
// published to shared memory, stored red/black-split as
// [column parity][k][i][j/2], where the four in-plane neighbours of a
// column (all of the other parity) are contiguous across the lanes of a
// warp.  The diagonal is applied as a reciprocal (one rounding away from the
// division; correcting it to the exact quotient lengthens the dependent
// chain of every update, which is what these latency-bound kernels cannot
// afford).  Ring terms have zero coefficients and are not read.
template <int NC>
struct CoarseShape {
  static constexpr int THREADS = 2 * (((NC * (NC / 2)) + 31) / 32) * 32;
};

// With unit_out set, CTA b relaxes rhs = e_u from phi = 0, u the b-th cell
// of even i+j+k in (i, j, k) order (cell index 2b or 2b+1), and writes the
// even-parity cells of the result as row b of unit_out (position = cell
// index / 2): the rows of the coarse-level operator.
template <class T, int NC, bool RHS_SMEM>
__global__ void __launch_bounds__(CoarseShape<NC>::THREADS) k_coarse_cols(Lvl<T> L0,
                                                                           int nsweeps,
                                                                           T* unit_out,
                                                                           const int* unit_ids,
                                                                           const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> L = rebase(L0, bt);
  constexpr int H = NC / 2;
  constexpr int HALF = NC * H;                  // columns per parity
  constexpr int GROUP = ((HALF + 31) / 32) * 32;
  constexpr int PLANE = NC * H;                 // one parity, one k plane
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sp = reinterpret_cast<T*>(smraw);
  T* srh = sp + NC * NC * NC;                   // rhs, when it stays in smem
  const int tid = threadIdx.x;
  const int g = tid / GROUP;                    // 0: (i+j) even, 1: odd
  const int q = tid - g * GROUP;
  const bool active = q < HALF;
  const int i = active ? q / H : 0;
  const int m = active ? q - i * H : 0;
  const int j = 2 * m + ((i + g) & 1);
  T* own = sp + g * NC * PLANE;
  const T* oth = sp + (1 - g) * NC * PLANE;
  const int me = q < HALF ? q : 0;
  const int oW = i > 0 ? me - H : me;
  const int oE = i < NC - 1 ? me + H : me;
  const int oS = j > 0 ? i * H + ((j - 1) >> 1) : me;
  const int oN = j < NC - 1 ? i * H + ((j + 1) >> 1) : me;
  const T aw = i > 0 ? L.ax : T(0), ae = i < NC - 1 ? L.ax : T(0);
  const T as = j > 0 ? L.ay : T(0), an = j < NC - 1 ? L.ay : T(0);
  const T az = L.az;
  // multigrid.py:58-67: ap = -(aw + ae + as + an + ab + at)
  const T inv_in = T(1) / (-(aw + ae + as + an + az + az));
  const T inv_lo = T(1) / (-(aw + ae + as + an + T(0) + az));
  const T inv_hi = T(1) / (-(aw + ae + as + an + az + T(0)));
  T ph[NC];
  T rh[RHS_SMEM ? 1 : NC];
  const long c0 = lid(L, i + 1, j + 1, 1);
  // the unit cell of this CTA: the one of cells 2b, 2b+1 with even i+j+k,
  // b = unit_ids[blockIdx.x] (or blockIdx.x)
  const int ub = unit_ids ? unit_ids[blockIdx.x] : (int)blockIdx.x;
  const int unit = 2 * ub + (((2 * ub / NC) / NC + (2 * ub / NC) % NC) & 1);
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    T r;
    if (unit_out) {
      ph[k] = T(0);
      r = (active && (i * NC + j) * NC + k == unit) ? T(1) : T(0);
    } else {
      ph[k] = active ? L.phi[c0 + k] : T(0);
      r = active ? L.rhs[c0 + k] : T(0);
    }
    if (RHS_SMEM) {
      if (active) srh[(g * NC + k) * PLANE + me] = r;
    } else {
      rh[RHS_SMEM ? 0 : k] = r;
    }
    if (active) own[k * PLANE + me] = ph[k];
  }
  __syncthreads();
  for (int sw = 0; sw < nsweeps; ++sw) {
#pragma unroll
    for (int color = 0; color < 2; ++color) {
      // (i+j+k+color) odd  <=>  k parity = (1 + g + color) & 1
      const int kp = (1 + g + color) & 1;
      if (active) {
        if (kp == 0) half_sweep_cols<T, NC, 0, RHS_SMEM>(oth, own, PLANE, me, oW, oE, oS, oN, aw, ae, as,
                                                    an, az, inv_in, inv_lo, inv_hi, ph, rh,
                                                    srh + g * NC * PLANE);
        else half_sweep_cols<T, NC, 1, RHS_SMEM>(oth, own, PLANE, me, oW, oE, oS, oN, aw, ae, as, an,
                                                 az, inv_in, inv_lo, inv_hi, ph, rh,
                                                 srh + g * NC * PLANE);
      }
      __syncthreads();
    }
  }
  if (!active) return;
  if (unit_out) {
    T* row = unit_out + (long)blockIdx.x * (NC * NC * NC / 2) + ((i * NC + j) * NC >> 1);
#pragma unroll
    for (int k = 0; k < NC; ++k)
      if (((i + j + k) & 1) == 0) row[k >> 1] = ph[k];
    return;
  }
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    const long c = c0 + k;
    L.phi[c] = ph[k];
    if (nsweeps > 0) ring_mirror(L, i, j, k, c, ph[k]);
  }
}

template <class T, int NC, bool RHS_SMEM>
static int launch_coarse(const Lvl<T>& L, int nsweeps, cudaStream_t s, T* unit_out = nullptr,
                         const int* unit_ids = nullptr, int nunits = 0) {
  constexpr int HALF = NC * (NC / 2);
  constexpr int GROUP = ((HALF + 31) / 32) * 32;
  const size_t sb = (size_t)NC * NC * NC * sizeof(T) * (RHS_SMEM ? 2 : 1);
  WF_CK(cudaFuncSetAttribute(k_coarse_cols<T, NC, RHS_SMEM>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb));
  const int nb = unit_out ? (unit_ids ? nunits : NC * NC * NC / 2) : 1;
  WF_CK(launch_k(k_coarse_cols<T, NC, RHS_SMEM>, nb, 2 * GROUP, sb, s, L, nsweeps, unit_out,
                 unit_ids));
  WF_CKL("k_coarse_cols");
  return WF_OK;
}

// returns 1 when a specialised coarse kernel handled the level
template <class T>
static int try_coarse(const Lvl<T>& L, int nsweeps, cudaStream_t s, int* rc) {
  switch (L.n) {
    case 4: *rc = launch_coarse<T, 4, false>(L, nsweeps, s); return 1;
    case 8: *rc = launch_coarse<T, 8, false>(L, nsweeps, s); return 1;
    case 12: *rc = launch_coarse<T, 12, false>(L, nsweeps, s); return 1;
    case 16: *rc = launch_coarse<T, 16, false>(L, nsweeps, s); return 1;
    case 20: *rc = launch_coarse<T, 20, false>(L, nsweeps, s); return 1;
    case 24: *rc = launch_coarse<T, 24, true>(L, nsweeps, s); return 1;
    default: return 0;
  }
}

// ---- the coarse level spread over a thread-block cluster ------------------
// The level is cut into C = NC/NCL slabs of NCL i-planes, one CTA per slab,
// the CTAs forming one cluster.  A CTA keeps its slab plus one halo plane
// on each side in shared memory ([parity][k][NCL+2][NC/2], red/black split
// as in k_coarse_cols), so every neighbour read is local.  After updating a
// cell on its first or last plane a thread also stores the value into the
// neighbouring CTA's halo plane (distributed shared memory), and the cluster
// barrier that ends each half-sweep publishes those stores.
template <int NC, int NCL>
struct ClusterShape {
  static constexpr int C = NC / NCL;
  static constexpr int H = NC / 2;
  static constexpr int HALF = NCL * H;
  static constexpr int GROUP = ((HALF + 31) / 32) * 32;
  static constexpr int THREADS = 2 * GROUP;
  static constexpr int PL = (NCL + 2) * H;  // one parity, one k
};

template <class T, int NC, int NCL>
__global__ void __launch_bounds__(ClusterShape<NC, NCL>::THREADS)
    k_coarse_cluster(Lvl<T> L, int nsweeps) {
  pdl_entry();
  using S = ClusterShape<NC, NCL>;
  constexpr int H = S::H, HALF = S::HALF, GROUP = S::GROUP, PL = S::PL, C = S::C;
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  extern __shared__ __align__(16) unsigned char smraw[];
  T* sp = reinterpret_cast<T*>(smraw);
  const int tid = threadIdx.x;
  for (int t = tid; t < 2 * NC * PL; t += blockDim.x) sp[t] = T(0);
  const int g = tid / GROUP;
  const int q = tid - g * GROUP;
  const bool active = q < HALF;
  const int il = active ? q / H : 0;
  const int m = active ? q - il * H : 0;
  const int i = rank * NCL + il;
  const int j = 2 * m + ((i + g) & 1);
  T* own = sp + g * NC * PL;
  const T* oth = sp + (1 - g) * NC * PL;
  const int me = (il + 1) * H + m;
  const int oW = me - H, oE = me + H;
  const int oS = j > 0 ? (il + 1) * H + ((j - 1) >> 1) : me;
  const int oN = j < NC - 1 ? (il + 1) * H + ((j + 1) >> 1) : me;
  const T aw = i > 0 ? L.ax : T(0), ae = i < NC - 1 ? L.ax : T(0);
  const T as = j > 0 ? L.ay : T(0), an = j < NC - 1 ? L.ay : T(0);
  const T az = L.az;
  const T inv_in = T(1) / (-(aw + ae + as + an + az + az));
  const T inv_lo = T(1) / (-(aw + ae + as + an + T(0) + az));
  const T inv_hi = T(1) / (-(aw + ae + as + an + az + T(0)));
  // halo slots of the neighbouring CTAs that mirror this thread's column
  T* rW = nullptr;  // my first plane -> rank-1's east halo (plane NCL+1)
  T* rE = nullptr;  // my last plane  -> rank+1's west halo (plane 0)
  if (active && il == 0 && rank > 0)
    rW = cl.map_shared_rank(own, rank - 1) + (NCL + 1) * H + m;
  if (active && il == NCL - 1 && rank < C - 1)
    rE = cl.map_shared_rank(own, rank + 1) + m;
  T ph[NC], rh[NC];
  const long c0 = lid(L, i + 1, j + 1, 1);
  cl.sync();  // every CTA's halos are zeroed before anyone writes into them
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    ph[k] = active ? L.phi[c0 + k] : T(0);
    rh[k] = active ? L.rhs[c0 + k] : T(0);
    if (active) {
      own[k * PL + me] = ph[k];
      if (rW) rW[k * PL] = ph[k];
      if (rE) rE[k * PL] = ph[k];
    }
  }
  cl.sync();
  for (int sw = 0; sw < nsweeps; ++sw) {
#pragma unroll
    for (int color = 0; color < 2; ++color) {
      const int kp = (1 + g + color) & 1;
      if (active) {
        if (kp == 0) {
          half_sweep_cols<T, NC, 0, false>(oth, own, PL, me, oW, oE, oS, oN, aw, ae, as, an, az,
                                           inv_in, inv_lo, inv_hi, ph, rh, nullptr);
          if (rW) {
#pragma unroll
            for (int k = 0; k < NC; k += 2) rW[k * PL] = ph[k];
          }
          if (rE) {
#pragma unroll
            for (int k = 0; k < NC; k += 2) rE[k * PL] = ph[k];
          }
        } else {
          half_sweep_cols<T, NC, 1, false>(oth, own, PL, me, oW, oE, oS, oN, aw, ae, as, an, az,
                                           inv_in, inv_lo, inv_hi, ph, rh, nullptr);
          if (rW) {
#pragma unroll
            for (int k = 1; k < NC; k += 2) rW[k * PL] = ph[k];
          }
          if (rE) {
#pragma unroll
            for (int k = 1; k < NC; k += 2) rE[k * PL] = ph[k];
          }
        }
      }
      cl.sync();
    }
  }
  if (!active) return;
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    const long c = c0 + k;
    L.phi[c] = ph[k];
    if (nsweeps > 0) ring_mirror(L, i, j, k, c, ph[k]);
  }
}

template <class T, int NC, int NCL>
static int launch_coarse_cluster(const Lvl<T>& L, int nsweeps, cudaStream_t s) {
  if (batch_ctx().tab) return fail(WF_EUNSUPPORTED, "cluster and cooperative relaxes do not run in a bucket");
  using S = ClusterShape<NC, NCL>;
  const size_t sb = 2ull * NC * S::PL * sizeof(T);
  auto kern = k_coarse_cluster<T, NC, NCL>;
  WF_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(S::C, 1, 1);
  cfg.blockDim = dim3(S::THREADS, 1, 1);
  cfg.dynamicSmemBytes = sb;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = S::C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 2 : 1;
  WF_CK(cudaLaunchKernelEx(&cfg, kern, L, nsweeps));
  WF_CKL("k_coarse_cluster");
  return WF_OK;
}

// ---- point-to-point variant: halo pushes complete on the receiver's mbarrier
// Same slab decomposition as k_coarse_cluster, but no cluster-wide barrier
// inside the sweep loop.  A thread on a slab's first/last plane sends each
// value it updates straight into the neighbouring CTA's halo plane with
// st.async, whose completion is counted in bytes on that CTA's mbarrier for
// the colour of the data.  Before a half-sweep reads halo values of one
// colour, every thread waits on its own CTA's barrier for that colour, so
// nobody waits for a memory fence or for CTAs it does not exchange with.
// Ordering: a neighbour can only produce the next values of a colour after
// receiving the values this CTA computes from the current ones, so a halo
// cell is never overwritten while it may still be read.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint32_t mapa_u32(uint32_t a, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t a, uint32_t tx) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(tx)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t a, uint32_t parity, int mode) {
  uint32_t ok;
  if (mode == 0) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity), "r"(1000u)
        : "memory");
  } else if (mode == 1) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
  }
  return ok != 0;
}
__device__ __forceinline__ void st_async(uint32_t raddr, double v, uint32_t rmbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b64 [%0], %1, [%2];" ::"r"(
                   raddr),
               "l"(__double_as_longlong(v)), "r"(rmbar)
               : "memory");
}
__device__ __forceinline__ void st_async(uint32_t raddr, float v, uint32_t rmbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];" ::"r"(
                   raddr),
               "r"(__float_as_uint(v)), "r"(rmbar)
               : "memory");
}

// bounded wait: at most 2^22 tries (about a second with suspending tries,
// much less when spinning)
constexpr int MBAR_WAIT_TRIES = 1 << 22;

template <class T, int NC, int NCL>
__global__ void __launch_bounds__(ClusterShape<NC, NCL>::THREADS)
    k_coarse_p2p(Lvl<T> L, int nsweeps, int wmode) {
  pdl_entry();
  using S = ClusterShape<NC, NCL>;
  constexpr int H = S::H, HALF = S::HALF, GROUP = S::GROUP, PL = S::PL, C = S::C;
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(8) unsigned long long mbar[2];
  __shared__ int s_bail;
  T* sp = reinterpret_cast<T*>(smraw);
  const int tid = threadIdx.x;
  const uint32_t mb[2] = {smem_u32(&mbar[0]), smem_u32(&mbar[1])};
  if (tid == 0) {
    mbar_init(mb[0], 1);
    mbar_init(mb[1], 1);
    s_bail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int t = tid; t < 2 * NC * PL; t += blockDim.x) sp[t] = T(0);
  const int g = tid / GROUP;
  const int q = tid - g * GROUP;
  const bool active = q < HALF;
  const int il = active ? q / H : 0;
  const int m = active ? q - il * H : 0;
  const int i = rank * NCL + il;
  const int j = 2 * m + ((i + g) & 1);
  T* own = sp + g * NC * PL;
  const T* oth = sp + (1 - g) * NC * PL;
  const int me = (il + 1) * H + m;
  const int oW = me - H, oE = me + H;
  const int oS = j > 0 ? (il + 1) * H + ((j - 1) >> 1) : me;
  const int oN = j < NC - 1 ? (il + 1) * H + ((j + 1) >> 1) : me;
  const T aw = i > 0 ? L.ax : T(0), ae = i < NC - 1 ? L.ax : T(0);
  const T as = j > 0 ? L.ay : T(0), an = j < NC - 1 ? L.ay : T(0);
  const T az = L.az;
  const T inv_in = T(1) / (-(aw + ae + as + an + az + az));
  const T inv_lo = T(1) / (-(aw + ae + as + an + T(0) + az));
  const T inv_hi = T(1) / (-(aw + ae + as + an + az + T(0)));
  const bool sendW = active && il == 0 && rank > 0;
  const bool sendE = active && il == NCL - 1 && rank < C - 1;
  // this column's halo slot in the neighbour (same parity array, k = 0)
  const uint32_t own_u32 = smem_u32(own);
  uint32_t aW = 0, aE = 0, mW[2] = {0, 0}, mE[2] = {0, 0};
  if (sendW) {
    aW = mapa_u32(own_u32 + (uint32_t)(((NCL + 1) * H + m) * sizeof(T)), rank - 1);
    mW[0] = mapa_u32(mb[0], rank - 1);
    mW[1] = mapa_u32(mb[1], rank - 1);
  }
  if (sendE) {
    aE = mapa_u32(own_u32 + (uint32_t)(m * sizeof(T)), rank + 1);
    mE[0] = mapa_u32(mb[0], rank + 1);
    mE[1] = mapa_u32(mb[1], rank + 1);
  }
  const int nbr = (rank > 0 ? 1 : 0) + (rank < C - 1 ? 1 : 0);
  const uint32_t tx = (uint32_t)(nbr * (NC * NC / 2) * sizeof(T));
  T ph[NC], rh[NC];
  const long c0 = lid(L, i + 1, j + 1, 1);
  cl.sync();  // barriers initialised and halos zeroed in every CTA
  T* rWp = sendW ? cl.map_shared_rank(own, rank - 1) + (NCL + 1) * H + m : nullptr;
  T* rEp = sendE ? cl.map_shared_rank(own, rank + 1) + m : nullptr;
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    ph[k] = active ? L.phi[c0 + k] : T(0);
    rh[k] = active ? L.rhs[c0 + k] : T(0);
    if (active) {
      own[k * PL + me] = ph[k];
      if (rWp) rWp[k * PL] = ph[k];
      if (rEp) rEp[k * PL] = ph[k];
    }
  }
  if (tid == 0 && nsweeps > 0) {
    mbar_arrive_expect_tx(mb[0], tx);
    mbar_arrive_expect_tx(mb[1], tx);
  }
  cl.sync();  // initial halos in place everywhere
  const int nh = 2 * nsweeps;
  bool bailed = false;
  for (int t = 0; t < nh; ++t) {
    if (t > 0) {
      // halo values of the colour read now were produced at t-1
      const int c = (t - 1) & 1;
      const uint32_t par = (uint32_t)(((t - 1) >> 1) & 1);
      bool ok = false;
      for (int it = 0; it < MBAR_WAIT_TRIES && !ok; ++it) ok = mbar_try_wait(mb[c], par, wmode);
      if (!ok) s_bail = 1;
      if (tid == 0 && t + 1 < nh) mbar_arrive_expect_tx(mb[c], tx);
    }
    __syncthreads();  // local values of t-1 visible; bail decision uniform
    if (s_bail) {
      bailed = true;
      break;
    }
    const int kp = (1 + g + (t & 1)) & 1;
    if (active) {
      if (kp == 0)
        half_sweep_cols<T, NC, 0, false>(oth, own, PL, me, oW, oE, oS, oN, aw, ae, as, an, az,
                                         inv_in, inv_lo, inv_hi, ph, rh, nullptr);
      else
        half_sweep_cols<T, NC, 1, false>(oth, own, PL, me, oW, oE, oS, oN, aw, ae, as, an, az,
                                         inv_in, inv_lo, inv_hi, ph, rh, nullptr);
      const uint32_t mc = (uint32_t)(t & 1);
      if (sendW) {
#pragma unroll
        for (int k = 0; k < NC; ++k)
          if ((k & 1) == kp) st_async(aW + (uint32_t)(k * PL * sizeof(T)), ph[k], mW[mc]);
      }
      if (sendE) {
#pragma unroll
        for (int k = 0; k < NC; ++k)
          if ((k & 1) == kp) st_async(aE + (uint32_t)(k * PL * sizeof(T)), ph[k], mE[mc]);
      }
    }
  }
  if (!bailed && nh > 0) {
    // the neighbours' last pushes (colour of t = nh-1) must land before exit
    const int c = (nh - 1) & 1;
    const uint32_t par = (uint32_t)(((nh - 1) >> 1) & 1);
    bool ok = false;
    for (int it = 0; it < MBAR_WAIT_TRIES && !ok; ++it) ok = mbar_try_wait(mb[c], par, wmode);
    if (!ok) s_bail = 1;
  }
  __syncthreads();
  if (s_bail && tid == 0 && L.err) atomicExch(L.err, (int)WF_ST_WAIT_TIMEOUT);
  cl.sync();
  if (!active) return;
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    const long c = c0 + k;
    L.phi[c] = ph[k];
    if (nsweeps > 0) ring_mirror(L, i, j, k, c, ph[k]);
  }
}

template <class T, int NC, int NCL>
static int launch_coarse_p2p(const Lvl<T>& L, int nsweeps, cudaStream_t s) {
  if (batch_ctx().tab) return fail(WF_EUNSUPPORTED, "cluster and cooperative relaxes do not run in a bucket");
  using S = ClusterShape<NC, NCL>;
  const size_t sb = 2ull * NC * S::PL * sizeof(T);
  auto kern = k_coarse_p2p<T, NC, NCL>;
  WF_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb));
  if (S::C > 8) WF_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(S::C, 1, 1);
  cfg.blockDim = dim3(S::THREADS, 1, 1);
  cfg.dynamicSmemBytes = sb;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = S::C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 2 : 1;
  static int wmode = -1;
  if (wmode < 0) {
    const char* e = getenv("WF_MBWAIT");
    wmode = (e && e[0] >= '0' && e[0] <= '2') ? e[0] - '0' : 1;
  }
  WF_CK(cudaLaunchKernelEx(&cfg, kern, L, nsweeps, wmode));
  WF_CKL("k_coarse_p2p");
  return WF_OK;
}

// thin slabs: more CTAs per cluster (up to 16, non-portable sizes)
template <class T>
static int try_coarse_p2p_thin(const Lvl<T>& L, int nsweeps, cudaStream_t s, int* rc) {
  switch (L.n) {
    case 12: *rc = launch_coarse_p2p<T, 12, 1>(L, nsweeps, s); return 1;
    case 16: *rc = launch_coarse_p2p<T, 16, 1>(L, nsweeps, s); return 1;
    case 20: *rc = launch_coarse_p2p<T, 20, 2>(L, nsweeps, s); return 1;
    case 24: *rc = launch_coarse_p2p<T, 24, 2>(L, nsweeps, s); return 1;
    case 28: *rc = launch_coarse_p2p<T, 28, 2>(L, nsweeps, s); return 1;
    case 32: *rc = launch_coarse_p2p<T, 32, 2>(L, nsweeps, s); return 1;
    default: return 0;
  }
}

template <class T>
static int try_coarse_p2p(const Lvl<T>& L, int nsweeps, cudaStream_t s, int* rc) {
  switch (L.n) {
    case 6: *rc = launch_coarse_p2p<T, 6, 1>(L, nsweeps, s); return 1;
    case 8: *rc = launch_coarse_p2p<T, 8, 1>(L, nsweeps, s); return 1;
    case 10: *rc = launch_coarse_p2p<T, 10, 2>(L, nsweeps, s); return 1;
    case 12: *rc = launch_coarse_p2p<T, 12, 2>(L, nsweeps, s); return 1;
    case 14: *rc = launch_coarse_p2p<T, 14, 2>(L, nsweeps, s); return 1;
    case 16: *rc = launch_coarse_p2p<T, 16, 2>(L, nsweeps, s); return 1;
    case 20: *rc = launch_coarse_p2p<T, 20, 4>(L, nsweeps, s); return 1;
    case 24: *rc = launch_coarse_p2p<T, 24, 3>(L, nsweeps, s); return 1;
    case 28: *rc = launch_coarse_p2p<T, 28, 4>(L, nsweeps, s); return 1;
    case 32: *rc = launch_coarse_p2p<T, 32, 4>(L, nsweeps, s); return 1;
    default: return 0;
  }
}

// mid-size levels (a few sweeps of 28^3..48^3): the whole level resident in
// the distributed shared memory of one cluster, so a 6-sweep relax is one
// launch instead of twelve.  Off by default (WF_MID=1 turns it on): inside
// the step graph, programmatic dependent launch already brings a
// one-colour half-sweep of these levels to about 1.3 us, and the 80^3 step
// measured 2.47 ms with it against 2.41 ms without.
static bool mid_p2p_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("WF_MID");
    v = (e && e[0] == '1') ? 1 : 0;
  }
  return v == 1;
}

template <class T>
static int try_relax_mid(const Lvl<T>& L, int nsweeps, cudaStream_t s, int* rc) {
  if (!mid_p2p_enabled()) return 0;
  switch (L.n) {
    case 28: *rc = launch_coarse_p2p<T, 28, 4>(L, nsweeps, s); return 1;
    case 32: *rc = launch_coarse_p2p<T, 32, 4>(L, nsweeps, s); return 1;
    case 40: *rc = launch_coarse_p2p<T, 40, 4>(L, nsweeps, s); return 1;
    case 48: *rc = launch_coarse_p2p<T, 48, 4>(L, nsweeps, s); return 1;
    default: return 0;
  }
}

// ---- temporal blocking: one exchange per full sweep ----------------------
// As k_coarse_p2p, but each CTA also keeps two halo planes on each side, so
// it can run a whole sweep locally: red on its slab plus one plane on each
// side (the extra planes redundantly, from the neighbours' values of the
// previous sweep), then black on its slab.  Only then do the slab's two
// outer planes (both colours) go to the neighbours, into a staging buffer
// that alternates between sweeps so that a sender one sweep ahead never
// overwrites values still being read; the receiver copies them into its
// halo planes before the next sweep.  Half as many exchanges as k_coarse_p2p
// for 25 % more red work.
template <int NC, int NCL>
struct TbShape {
  static constexpr int C = NC / NCL;
  static constexpr int H = NC / 2;
  static constexpr int NLP = NCL + 4;          // local planes incl. halos
  static constexpr int HALF = NLP * H;         // columns per parity
  static constexpr int GROUP = ((HALF + 31) / 32) * 32;
  static constexpr int THREADS = 2 * GROUP;
  static constexpr int PL = NLP * H;           // one parity, one k
  static constexpr int SIDE = 2 * NC * NC;     // staged values per side
};

template <class T, int NC, int NCL>
__global__ void __launch_bounds__(TbShape<NC, NCL>::THREADS)
    k_coarse_tb(Lvl<T> L, int nsweeps, int wmode) {
  pdl_entry();
  using S = TbShape<NC, NCL>;
  constexpr int H = S::H, HALF = S::HALF, GROUP = S::GROUP, PL = S::PL, C = S::C;
  constexpr int SIDE = S::SIDE;
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ __align__(8) unsigned long long mbar[2];
  __shared__ int s_bail;
  T* sp = reinterpret_cast<T*>(smraw);
  T* stage = sp + 2 * NC * PL;  // [buf 2][side 2 (0 = from rank-1, 1 = from rank+1)][SIDE]
  const int tid = threadIdx.x;
  const uint32_t mb[2] = {smem_u32(&mbar[0]), smem_u32(&mbar[1])};
  if (tid == 0) {
    mbar_init(mb[0], 1);
    mbar_init(mb[1], 1);
    s_bail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int t = tid; t < 2 * NC * PL; t += blockDim.x) sp[t] = T(0);
  const int g = tid / GROUP;
  const int q = tid - g * GROUP;
  const bool slot = q < HALF;
  const int il = slot ? q / H : 0;                 // local plane 0 .. NCL+3
  const int m = slot ? q - il * H : 0;
  const int i = rank * NCL - 2 + il;               // global plane (may be outside)
  const bool active = slot && i >= 0 && i < NC;
  const int j = 2 * m + ((i + g) & 1);
  T* own = sp + g * NC * PL;
  const T* oth = sp + (1 - g) * NC * PL;
  const int me = il * H + m;
  const int oW = il > 0 ? me - H : me, oE = il < S::NLP - 1 ? me + H : me;
  const int oS = j > 0 ? il * H + ((j - 1) >> 1) : me;
  const int oN = j < NC - 1 ? il * H + ((j + 1) >> 1) : me;
  const T aw = i > 0 ? L.ax : T(0), ae = i < NC - 1 ? L.ax : T(0);
  const T as = j > 0 ? L.ay : T(0), an = j < NC - 1 ? L.ay : T(0);
  const T az = L.az;
  const T inv_in = T(1) / (-(aw + ae + as + an + az + az));
  const T inv_lo = T(1) / (-(aw + ae + as + an + T(0) + az));
  const T inv_hi = T(1) / (-(aw + ae + as + an + az + T(0)));
  const int olo = rank * NCL, ohi = olo + NCL;      // owned planes [olo, ohi)
  const bool do_red = active && i >= olo - 1 && i < ohi + 1;
  const bool do_black = active && i >= olo && i < ohi;
  const bool halo_lo = active && i < olo;           // filled from rank-1
  const bool halo_hi = active && i >= ohi;          // filled from rank+1
  // my column goes to a neighbour when it is one of my two outer planes
  const bool sendW = active && rank > 0 && i >= olo && i < olo + 2;
  const bool sendE = active && rank < C - 1 && i >= ohi - 2 && i < ohi;
  uint32_t aW[2] = {0, 0}, aE[2] = {0, 0}, mW[2] = {0, 0}, mE[2] = {0, 0};
  const uint32_t st_u32 = smem_u32(stage);
  if (sendW) {  // rank-1 stores me as side 1 (from its right), plane i - olo
    const int pw = i - olo;
    for (int b = 0; b < 2; ++b) {
      aW[b] = mapa_u32(st_u32 + (uint32_t)(((b * 2 + 1) * SIDE + (pw * NC + j) * NC) * sizeof(T)),
                       rank - 1);
      mW[b] = mapa_u32(mb[b], rank - 1);
    }
  }
  if (sendE) {  // rank+1 stores me as side 0 (from its left), plane i - (ohi - 2)
    const int pe = i - (ohi - 2);
    for (int b = 0; b < 2; ++b) {
      aE[b] = mapa_u32(st_u32 + (uint32_t)(((b * 2 + 0) * SIDE + (pe * NC + j) * NC) * sizeof(T)),
                       rank + 1);
      mE[b] = mapa_u32(mb[b], rank + 1);
    }
  }
  // where a halo column of mine finds its staged values
  const int hside = halo_lo ? 0 : 1;
  const int hplane = halo_lo ? i - (olo - 2) : i - ohi;
  const int hoff = hside * SIDE + (hplane * NC + j) * NC;
  const int nbr = (rank > 0 ? 1 : 0) + (rank < C - 1 ? 1 : 0);
  const uint32_t tx = (uint32_t)(nbr * SIDE * sizeof(T));
  T ph[NC], rh[NC];
  const long c0 = lid(L, (active ? i : 0) + 1, j + 1, 1);
  cl.sync();  // barriers initialised everywhere before any push
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    ph[k] = active ? L.phi[c0 + k] : T(0);
    rh[k] = active ? L.rhs[c0 + k] : T(0);
    if (slot) own[k * PL + me] = ph[k];
  }
  // data of sweep s (s < nsweeps-1) lands in staging buffer s&1
  if (tid == 0) {
    if (nsweeps > 1) mbar_arrive_expect_tx(mb[0], tx);
    if (nsweeps > 2) mbar_arrive_expect_tx(mb[1], tx);
  }
  __syncthreads();
  bool bailed = false;
  for (int sw = 0; sw < nsweeps; ++sw) {
    if (sw > 0) {
      const int b = (sw - 1) & 1;
      const uint32_t par = (uint32_t)(((sw - 1) >> 1) & 1);
      bool ok = false;
      for (int it = 0; it < MBAR_WAIT_TRIES && !ok; ++it) ok = mbar_try_wait(mb[b], par, wmode);
      if (!ok) s_bail = 1;
      if (tid == 0 && sw + 1 < nsweeps - 1) mbar_arrive_expect_tx(mb[b], tx);
      if (ok && (halo_lo || halo_hi)) {
        const T* src = stage + b * 2 * SIDE + hoff;
#pragma unroll
        for (int k = 0; k < NC; ++k) {
          ph[k] = src[k];
          own[k * PL + me] = ph[k];
        }
      }
    }
    __syncthreads();
    if (s_bail) {
      bailed = true;
      break;
    }
    // red: colour 0, cells with (i+j+k) odd  <=>  k parity (1 + g) & 1
    if (do_red) {
      if (((1 + g) & 1) == 0)
        half_sweep_cols<T, NC, 0, false>(oth, own, PL, me, oW, oE, oS, oN, aw, ae, as, an, az,
                                         inv_in, inv_lo, inv_hi, ph, rh, nullptr);
      else
        half_sweep_cols<T, NC, 1, false>(oth, own, PL, me, oW, oE, oS, oN, aw, ae, as, an, az,
                                         inv_in, inv_lo, inv_hi, ph, rh, nullptr);
    }
    __syncthreads();
    if (do_black) {
      if ((g & 1) == 0)
        half_sweep_cols<T, NC, 0, false>(oth, own, PL, me, oW, oE, oS, oN, aw, ae, as, an, az,
                                         inv_in, inv_lo, inv_hi, ph, rh, nullptr);
      else
        half_sweep_cols<T, NC, 1, false>(oth, own, PL, me, oW, oE, oS, oN, aw, ae, as, an, az,
                                         inv_in, inv_lo, inv_hi, ph, rh, nullptr);
    }
    if (sw + 1 < nsweeps) {
      const int b = sw & 1;
      if (sendW) {
#pragma unroll
        for (int k = 0; k < NC; ++k) st_async(aW[b] + (uint32_t)(k * sizeof(T)), ph[k], mW[b]);
      }
      if (sendE) {
#pragma unroll
        for (int k = 0; k < NC; ++k) st_async(aE[b] + (uint32_t)(k * sizeof(T)), ph[k], mE[b]);
      }
    }
    __syncthreads();  // this sweep's reads of the halo planes are done
  }
  __syncthreads();
  if (s_bail && tid == 0 && L.err) atomicExch(L.err, (int)WF_ST_WAIT_TIMEOUT);
  cl.sync();
  if (!do_black) return;
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    const long c = c0 + k;
    L.phi[c] = ph[k];
    if (nsweeps > 0) ring_mirror(L, i, j, k, c, ph[k]);
  }
  (void)bailed;
}

template <class T, int NC, int NCL>
static int launch_coarse_tb(const Lvl<T>& L, int nsweeps, cudaStream_t s) {
  if (batch_ctx().tab) return fail(WF_EUNSUPPORTED, "cluster and cooperative relaxes do not run in a bucket");
  using S = TbShape<NC, NCL>;
  const size_t sb = (2ull * NC * S::PL + 4ull * S::SIDE) * sizeof(T);
  auto kern = k_coarse_tb<T, NC, NCL>;
  WF_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(S::C, 1, 1);
  cfg.blockDim = dim3(S::THREADS, 1, 1);
  cfg.dynamicSmemBytes = sb;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = S::C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 2 : 1;
  WF_CK(cudaLaunchKernelEx(&cfg, kern, L, nsweeps, 1));
  WF_CKL("k_coarse_tb");
  return WF_OK;
}

template <class T>
static int try_coarse_tb(const Lvl<T>& L, int nsweeps, cudaStream_t s, int* rc) {
  switch (L.n) {
    case 8: *rc = launch_coarse_tb<T, 8, 2>(L, nsweeps, s); return 1;
    case 10: *rc = launch_coarse_tb<T, 10, 2>(L, nsweeps, s); return 1;
    case 12: *rc = launch_coarse_tb<T, 12, 2>(L, nsweeps, s); return 1;
    case 14: *rc = launch_coarse_tb<T, 14, 2>(L, nsweeps, s); return 1;
    case 16: *rc = launch_coarse_tb<T, 16, 2>(L, nsweeps, s); return 1;
    case 20: *rc = launch_coarse_tb<T, 20, 4>(L, nsweeps, s); return 1;
    case 24: *rc = launch_coarse_tb<T, 24, 3>(L, nsweeps, s); return 1;
    case 28: *rc = launch_coarse_tb<T, 28, 4>(L, nsweeps, s); return 1;
    case 32: *rc = launch_coarse_tb<T, 32, 4>(L, nsweeps, s); return 1;
    default: return 0;
  }
}

// ---- the coarse-level relax as a precomputed operator ----------------------
// Colour A = cells of odd i+j+k (each sweep updates them first), colour B =
// even i+j+k; every neighbour of a cell has the other colour.  From phi = 0
// the first sweep gives x_A = b_A / ap and then x_B = v_B / ap with
// v_B = b_B - sum_nb a_nb x_A(nb); every later sweep maps x_B linearly
// (x_B <- x_B1 + G x_B, G = D_B^-1 A_BA D_A^-1 A_AB).  So after
// m = n_coarse - 1 sweeps x_B = S v_B with S = sum_{s<m} G^s D_B^-1, and the
// n_coarse-th sweep is run as such from that x_B.
//
// S is symmetric (D_B G is, because A is), and it commutes with every map
// of the level's cells onto themselves that keeps the colour of each cell
// and the operator: the permutations of axes of equal coefficient combined
// with reflections of an even number of axes (n is even, so one reflection
// swaps the colours) -- 24 maps on a cube of equal spacings.  So S is fixed
// by its columns at one representative B cell r of every orbit of these
// maps, and for an output o = g(r):  x_B[o] = sum_u S[u, r] v_B[g(u)]
// (S[g r, w] = S[r, g^-1 w] = S[g^-1 w, r]).  Only the representative
// columns are stored (about N/48 of the (N/2)^2 entries of S, N = n^3:
// 5.8 MB instead of 128 MB at 20^3), built like the full map was (one CTA
// of the column kernel per representative, unit rhs).  The product is a
// small GEMM: with the permuted copies V[g][u] = v_B[g(u)] (k_cop_vg),
// Y[r][g] = sum_u C[r][u] V[g][u] over slices of u (k_cop_gemm), and
// x_B[g(r)] = the slices of Y[r][g] added in order (k_cop_out).  Every sum
// runs in a fixed order (per lane over its cells, a lane butterfly, the
// slices in order), so results do not depend on scheduling and a case
// computes the same bits alone or beside other cases.  The stored columns
// equal the mathematical S to rounding, so the relax agrees with the
// sweeps to rounding.
constexpr int COP_GMAX = 24;
static_assert(COP_GMAX <= 32, "k_cop_gemm writes symmetry q from lane q");

static bool cop_size_ok(int nc) {
  return nc == 4 || nc == 8 || nc == 12 || nc == 16 || nc == 20 || nc == 24;
}

static bool cop_full(int nc, bool fp32) { return fp32 && nc <= 4; }

// one colour-preserving symmetry of an n^3 level: c'_d = sgn_d * c[src_d] + off_d,
// and its inverse (same form) in isrc/isgn/ioff
struct CopSyms {
  int ng;
  int src[COP_GMAX][3], sgn[COP_GMAX][3], off[COP_GMAX][3];
  int isrc[COP_GMAX][3], isgn[COP_GMAX][3], ioff[COP_GMAX][3];
};

// the orbit structure of the B cells of an n^3 level under the symmetries
// its coefficients allow: the representatives, and for every B cell o the
// (representative, symmetry) pair that produces it (o = g(r), every o once)
struct CopPlan {
  int n = 0, M = 0, nrep = 0;
  int eq = 0;              // which coefficients are equal (bits: xy, xz, yz; 8 = full)
  CopSyms G{};
  std::vector<int> ints;   // nrep representative B indices, then for each B cell o
                           // (representative index << 5) | symmetry
  template <class T>
  int64_t op_elems() const {
    return (int64_t)nrep * M + ((int64_t)ints.size() * 4 + sizeof(T) - 1) / sizeof(T);
  }
};

constexpr int COP_RB = 16;  // representatives per CTA of k_cop_gemm (2 per warp)
constexpr int COP_KS = 8;   // slices of the B cells (the product's sum) per output

// per-case scratch of the operator product: the permuted copies of v_B
// (COP_GMAX x M) and the slice partials (COP_KS x nrep x COP_GMAX)
static int64_t cop_scratch_elems(const CopPlan& P) {
  return (int64_t)COP_GMAX * P.M + (int64_t)COP_KS * P.nrep * COP_GMAX;
}

static void b_cell_host(int b, int n, int& i, int& j, int& k) {
  const int rw = 2 * b / n;
  i = rw / n;
  j = rw - i * n;
  k = 2 * b - rw * n + ((i + j) & 1);
}

// full: the identity map only (every column stored).  An FP32 operator of a
// 4^3 level is kept full: after hundreds of sweeps its map is nearly the
// rank-one projection on the constant mode of the Neumann problem, so the
// product is a large cancellation, and columns that equal the wanted
// entries only to FP32 rounding would not cancel (2e-1 relative error,
// against 1e-7 from 8^3 up and 1e-14 in FP64 at 4^3).
static const CopPlan& cop_plan(int n, double ax, double ay, double az, bool full) {
  static std::mutex mu;
  static std::vector<CopPlan*> plans;
  const double a[3] = {ax, ay, az};
  const int eq = full ? 8 : (a[0] == a[1]) | ((a[0] == a[2]) << 1) | ((a[1] == a[2]) << 2);
  std::lock_guard<std::mutex> lock(mu);
  for (CopPlan* p : plans)
    if (p->n == n && p->eq == eq) return *p;
  CopPlan* P = new CopPlan();
  P->n = n;
  P->M = n * n * n / 2;
  P->eq = eq;
  static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  static const int masks[4] = {0, 3, 5, 6};
  int ng = 0;
  for (const auto& pm : perms) {
    if (a[pm[0]] != a[0] || a[pm[1]] != a[1] || a[pm[2]] != a[2]) continue;
    if (full && (pm[0] != 0 || pm[1] != 1)) continue;
    for (int mk : masks) {
      if (full && mk != 0) continue;
      for (int d = 0; d < 3; ++d) {
        const int sg = (mk >> d) & 1 ? -1 : 1, of = (mk >> d) & 1 ? n - 1 : 0;
        P->G.src[ng][d] = pm[d];
        P->G.sgn[ng][d] = sg;
        P->G.off[ng][d] = of;
        // inverse: c[src_d] = sg * c'_d - sg * off
        P->G.isrc[ng][pm[d]] = d;
        P->G.isgn[ng][pm[d]] = sg;
        P->G.ioff[ng][pm[d]] = -sg * of;
      }
      ++ng;
    }
  }
  P->G.ng = ng;
  const int M = P->M;
  auto image = [&](int g, int b) {
    int c[3];
    b_cell_host(b, n, c[0], c[1], c[2]);
    int q[3];
    for (int d = 0; d < 3; ++d) q[d] = P->G.sgn[g][d] * c[P->G.src[g][d]] + P->G.off[g][d];
    return ((q[0] * n + q[1]) * n + q[2]) >> 1;
  };
  std::vector<int> reps;
  for (int b = 0; b < M; ++b) {
    int r = b;
    for (int g = 0; g < ng; ++g) r = std::min(r, image(g, b));
    if (r == b) reps.push_back(b);
  }
  P->nrep = (int)reps.size();
  P->ints.assign((size_t)P->nrep + M, -1);
  for (int x = 0; x < P->nrep; ++x) {
    P->ints[x] = reps[x];
    for (int g = 0; g < ng; ++g) {
      const int o = image(g, reps[x]);
      if (P->ints[P->nrep + o] < 0) P->ints[P->nrep + o] = (x << 5) | g;
    }
  }
  plans.push_back(P);
  return *P;
}

// (i, j, k) of the B cell at position b of the B-only order (n even: cells
// 2b and 2b+1 share i and j, and exactly one of them has even i+j+k)
__device__ __forceinline__ void b_cell(int b, int n, int& i, int& j, int& k) {
  const int rw = 2 * b / n;
  i = rw / n;
  j = rw - i * n;
  k = 2 * b - rw * n + ((i + j) & 1);
}

// v_B of B cell (i,j,k): its rhs minus its neighbours' first-sweep values
// b/ap (every neighbour is an A cell, updated from phi = 0); the terms in
// the order of k_rbgs, absent faces with zero coefficients
template <class T>
__device__ __forceinline__ T first_sweep_v(const Lvl<T>& L, int i, int j, int k) {
  const int n = L.n;
  auto x1 = [&](int a, int bq, int cq) -> T {
    const T aw = a > 0 ? L.ax : T(0), ae = a < n - 1 ? L.ax : T(0);
    const T as = bq > 0 ? L.ay : T(0), an = bq < n - 1 ? L.ay : T(0);
    const T ab = cq > 0 ? L.az : T(0), at = cq < n - 1 ? L.az : T(0);
    return L.rhs[lid(L, a + 1, bq + 1, cq + 1)] / (-(aw + ae + as + an + ab + at));
  };
  const T W = i > 0 ? L.ax * x1(i - 1, j, k) : T(0);
  const T E = i < n - 1 ? L.ax * x1(i + 1, j, k) : T(0);
  const T S = j > 0 ? L.ay * x1(i, j - 1, k) : T(0);
  const T N = j < n - 1 ? L.ay * x1(i, j + 1, k) : T(0);
  const T B = k > 0 ? L.az * x1(i, j, k - 1) : T(0);
  const T U = k < n - 1 ? L.az * x1(i, j, k + 1) : T(0);
  return L.rhs[lid(L, i + 1, j + 1, k + 1)] - (W + E + S + N + B + U);
}

// v_B of B cell w, stored into every permuted copy that holds it:
// V[g][u] = v_B[g(u)], so V[g][g^-1(w)] = v_B[w].  Eight threads per cell:
// thread t < 6 forms the t-th neighbour term of first_sweep_v (W, E, S, N,
// B, U: one division each), thread 0 adds them in that order, and the eight
// threads then store the copies (g = t, t+8, t+16)
template <class T>
__global__ void __launch_bounds__(256) k_cop_vg(const Lvl<T> L0, T* V,
                                                const __grid_constant__ CopSyms G,
                                                const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> L = rebase(L0, bt);
  if (bt.tab) V = (T*)bt.tab[bt_case(bt)].mg_cop_part;
  const int n = L.n, M = n * n * n / 2;
  const int t = threadIdx.x & 7;
  const int w = blockIdx.x * 32 + (threadIdx.x >> 3);
  const bool on = w < M;
  int c[3] = {0, 0, 0};
  if (on) b_cell(w, n, c[0], c[1], c[2]);
  const int i = c[0], j = c[1], k = c[2];
  // the cell's own rhs, loaded together with the neighbour's (one round of
  // memory latency instead of two)
  const T own = on ? L.rhs[lid(L, i + 1, j + 1, k + 1)] : T(0);
  // the neighbour of this thread's term and the coefficient towards it
  T term = T(0);
  if (on && t < 6) {
    const int a = i + (t == 0 ? -1 : t == 1 ? 1 : 0);
    const int bq = j + (t == 2 ? -1 : t == 3 ? 1 : 0);
    const int cq = k + (t == 4 ? -1 : t == 5 ? 1 : 0);
    const T coef = t < 2 ? L.ax : (t < 4 ? L.ay : L.az);
    if (a >= 0 && a < n && bq >= 0 && bq < n && cq >= 0 && cq < n) {
      const T aw = a > 0 ? L.ax : T(0), ae = a < n - 1 ? L.ax : T(0);
      const T as = bq > 0 ? L.ay : T(0), an = bq < n - 1 ? L.ay : T(0);
      const T ab = cq > 0 ? L.az : T(0), at = cq < n - 1 ? L.az : T(0);
      term = coef * (L.rhs[lid(L, a + 1, bq + 1, cq + 1)] / (-(aw + ae + as + an + ab + at)));
    }
  }
  T nb[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) nb[q] = __shfl_sync(0xffffffffu, term, (threadIdx.x & 24) | q);
  T x = T(0);
  if (on) x = own - (nb[0] + nb[1] + nb[2] + nb[3] + nb[4] + nb[5]);
  if (!on) return;
  for (int g = t; g < G.ng; g += 8) {
    int q[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int sd = G.isrc[g][d];
      q[d] = G.isgn[g][d] * (sd == 0 ? i : (sd == 1 ? j : k)) + G.ioff[g][d];
    }
    V[(long)g * M + (((q[0] * n + q[1]) * n + q[2]) >> 1)] = x;
  }
}

template <class T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// Y_s[x][g] = sum over the s-th slice of B cells u of C[x][u] * V[g][u]:
// a CTA takes COP_RB representatives x and one slice, and first copies the
// slice of every permuted copy V[g] into shared memory (each CTA reads it
// once from L2; the operator rows are read once in all) -- COP_SB loads per
// thread issued before any is stored, a few rounds of L2 latency instead of
// one per element (the 20^3 relax 28.8 -> 24.7 us); warp w takes the
// representatives x0 + 2w, x0 + 2w + 1 and every symmetry; lanes step
// through the slice two cells at a time (2-vector loads), each summing its
// cells in ascending order, then the lanes are added by a butterfly (fixed
// order)
constexpr int COP_SB = 16;   // staging loads in flight per thread

template <class T>
__global__ void __launch_bounds__(256) k_cop_gemm(const T* C, const T* V, T* Y, int nrep,
                                                  int M, int ng, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  if (bt.tab) {
    V = (const T*)bt.tab[bt_case(bt)].mg_cop_part;
    Y = (T*)bt.tab[bt_case(bt)].mg_cop_part + (long)COP_GMAX * M;
  }
  using V2 = typename Vec2<T>::type;
  extern __shared__ __align__(16) unsigned char cop_smem[];
  V2* sv = reinterpret_cast<V2*>(cop_smem);   // [ng][nh]: this slice of every V[g]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x0 = blockIdx.x * COP_RB, s = blockIdx.y;
  const int per = (((M + COP_KS - 1) / COP_KS) + 1) & ~1;   // even: 2-vector aligned
  const int h0 = s * per / 2, h1 = min(M, s * per + per) / 2;   // 2-vector range
  const int nh = max(0, h1 - h0);
  const int nv = ng * nh;
  for (int t0 = threadIdx.x; t0 < nv; t0 += blockDim.x * COP_SB) {
    V2 buf[COP_SB];
#pragma unroll
    for (int b = 0; b < COP_SB; ++b) {
      const int t = t0 + b * blockDim.x;
      if (t < nv) {
        const int g = t / nh, h = t - g * nh;
        buf[b] = reinterpret_cast<const V2*>(V + (long)g * M)[h0 + h];
      }
    }
#pragma unroll
    for (int b = 0; b < COP_SB; ++b) {
      const int t = t0 + b * blockDim.x;
      if (t < nv) sv[t] = buf[b];
    }
  }
  __syncthreads();
  const int r0 = x0 + 2 * w;
  T acc[2][COP_GMAX];
#pragma unroll
  for (int q = 0; q < COP_GMAX; ++q) acc[0][q] = acc[1][q] = T(0);
  if (r0 < nrep) {
    const V2* c0p = reinterpret_cast<const V2*>(C + (long)r0 * M);
    const V2* c1p = reinterpret_cast<const V2*>(C + (long)min(r0 + 1, nrep - 1) * M);
#pragma unroll 1
    for (int h = h0 + lane; h < h1; h += 32) {
      const V2 c0 = c0p[h], c1 = c1p[h];
      const V2* vh = sv + (h - h0);
#pragma unroll
      for (int q = 0; q < COP_GMAX; ++q) {
        if (q < ng) {
          const V2 v = vh[q * nh];
          acc[0][q] = fma(c0.x, v.x, acc[0][q]);
          acc[0][q] = fma(c0.y, v.y, acc[0][q]);
          acc[1][q] = fma(c1.x, v.x, acc[1][q]);
          acc[1][q] = fma(c1.y, v.y, acc[1][q]);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int q = 0; q < COP_GMAX; ++q) {
      T y = acc[r][q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
      acc[r][q] = y;
    }
  // lane q writes symmetry q of both representatives
  T y0 = T(0), y1 = T(0);
#pragma unroll
  for (int q = 0; q < COP_GMAX; ++q)
    if (lane == q) {
      y0 = acc[0][q];
      y1 = acc[1][q];
    }
  if (lane < ng) {
    if (r0 < nrep) Y[((long)s * nrep + r0) * COP_GMAX + lane] = y0;
    if (r0 + 1 < nrep) Y[((long)s * nrep + r0 + 1) * COP_GMAX + lane] = y1;
  }
}

// shared memory of k_cop_gemm: the slice of every permuted copy
template <class T>
static size_t cop_gemm_smem(int M, int ng) {
  const int per = (((M + COP_KS - 1) / COP_KS) + 1) & ~1;
  return (size_t)ng * (per / 2) * 2 * sizeof(T);
}

// x_B[o] = the slices of Y[x][g] added in ascending order, (x, g) the pair
// producing o; written into phi, and the A cell beside o zeroed (the
// closing sweep overwrites it first)
template <class T>
__global__ void __launch_bounds__(256) k_cop_out(const T* Y, const int* prod, int nrep,
                                                 Lvl<T> L0, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> L = rebase(L0, bt);
  const int n = L.n, M = n * n * n / 2;
  if (bt.tab) Y = (const T*)bt.tab[bt_case(bt)].mg_cop_part + (long)COP_GMAX * M;
  const int o = blockIdx.x * 256 + threadIdx.x;
  if (o >= M) return;
  const int pv = prod[o];
  const long at = (long)(pv >> 5) * COP_GMAX + (pv & 31);
  T y = Y[at];
#pragma unroll
  for (int s = 1; s < COP_KS; ++s) y += Y[(long)s * nrep * COP_GMAX + at];
  int i, j, k;
  b_cell(o, n, i, j, k);
  L.phi[lid(L, i + 1, j + 1, k + 1)] = y;
  L.phi[lid(L, i + 1, j + 1, (k ^ 1) + 1)] = T(0);
}

// phi of the coarsest level = the n_coarse-sweep relax of rhs from zero (the
// level's phi is overwritten): v_B and its permuted copies, the product of
// the representative columns with them, the B cells from their producing
// pairs, then the last sweep (k_rbgs, colour A then B, which also writes the
// face-ring mirrors); part: this case's scratch (cop_scratch_elems)
template <class T>
static int apply_coarse_op(const Lvl<T>& L, const T* op, T* part, cudaStream_t s) {
  const CopPlan& P =
      cop_plan(L.n, (double)L.ax, (double)L.ay, (double)L.az, cop_full(L.n, sizeof(T) == 4));
  T* V = part;
  T* Y = part + (long)COP_GMAX * P.M;
  const int* prod = reinterpret_cast<const int*>(op + (long)P.nrep * P.M) + P.nrep;
  WF_CK(launch_k(k_cop_vg<T>, (P.M + 31) / 32, 256, 0, s, L, V, P.G));
  WF_CKL("k_cop_vg");
  const size_t sm = cop_gemm_smem<T>(P.M, P.G.ng);
  WF_CK(cudaFuncSetAttribute(k_cop_gemm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  WF_CK(launch_k(k_cop_gemm<T>, dim3((P.nrep + COP_RB - 1) / COP_RB, COP_KS), 256, sm, s, op,
                 (const T*)V, Y, P.nrep, P.M, P.G.ng));
  WF_CKL("k_cop_gemm");
  WF_CK(launch_k(k_cop_out<T>, (P.M + 255) / 256, 256, 0, s, (const T*)Y, prod, P.nrep, L));
  WF_CKL("k_cop_out");
  for (int color = 0; color < 2; ++color) {
    WF_CK(launch_k(k_rbgs<T>, cells3(L.n, L.n, (L.n + 1) / 2), cell_block(), 0, s, L, color));
    WF_CKL("k_rbgs");
  }
  return WF_OK;
}

// the representative columns: n_coarse - 1 sweeps from zero per unit
// representative B cell; the plan's integers go after them
template <class T>
static int build_coarse_op(const Lvl<T>& L, int n_coarse, T* op, cudaStream_t s) {
  if (n_coarse < 2) return fail(WF_EINVAL, "coarse operator needs n_coarse >= 2");
  if (!cop_size_ok(L.n))
    return fail(WF_EUNSUPPORTED, "coarse operator: coarsest edge must be 4..24, step 4");
  const CopPlan& P =
      cop_plan(L.n, (double)L.ax, (double)L.ay, (double)L.az, cop_full(L.n, sizeof(T) == 4));
  int* ints = reinterpret_cast<int*>(op + (long)P.nrep * P.M);
  WF_CK(cudaMemcpyAsync(ints, P.ints.data(), P.ints.size() * sizeof(int),
                        cudaMemcpyHostToDevice, s));
  // the copy reads host memory that outlives it (the plan is kept for the
  // process), so it may stay asynchronous
  const int nsweeps = n_coarse - 1;
  switch (L.n) {
    case 4: return launch_coarse<T, 4, false>(L, nsweeps, s, op, ints, P.nrep);
    case 8: return launch_coarse<T, 8, false>(L, nsweeps, s, op, ints, P.nrep);
    case 12: return launch_coarse<T, 12, false>(L, nsweeps, s, op, ints, P.nrep);
    case 16: return launch_coarse<T, 16, false>(L, nsweeps, s, op, ints, P.nrep);
    case 20: return launch_coarse<T, 20, false>(L, nsweeps, s, op, ints, P.nrep);
    default: return launch_coarse<T, 24, true>(L, nsweeps, s, op, ints, P.nrep);
  }
}

// coarse strategy: 0 = one CTA (k_coarse_cols), 1 = cluster with a cluster
// barrier per half-sweep (k_coarse_cluster), 2 = cluster with point-to-point
// halo pushes (k_coarse_p2p).  Chosen per level size and precision from a
// table that the autotuner (warpflow/autotune.py) can overwrite through
// wf_set_coarse_strategy; WF_COARSE forces one strategy for every size.
// Defaults measured on B200 (ns per half-sweep, FP64, 300-sweep relax):
//   n:             8    12    16    20    24    32
//   0 one CTA:   133   263   407   903  1530  4090
//   1 barrier:   442   449   488   651   686   921
//   2 p2p:       402   487   501   596   905   860
//   3 tb:        499   625  1143  1281  1962  3802
//   4 p2p thin:    -   427   464   762   631   776
static int g_strategy[2][65];
static bool g_strategy_init = false;

static void strategy_defaults() {
  for (int f = 0; f < 2; ++f)
    for (int n = 0; n <= 64; ++n) g_strategy[f][n] = n <= 16 ? 0 : (n == 20 ? 2 : 4);
  g_strategy_init = true;
}

static int coarse_strategy(int n, bool fp32) {
  const char* e = getenv("WF_COARSE");
  if (e && e[0] >= '0' && e[0] <= '4') return e[0] - '0';
  if (!g_strategy_init) strategy_defaults();
  return (n >= 0 && n <= 64) ? g_strategy[fp32 ? 1 : 0][n] : 2;
}

int set_coarse_strategy(int n, int fp32, int strategy) {
  if (n < 0 || n > 64 || strategy < 0 || strategy > 4)
    return fail(WF_EINVAL, "wf_set_coarse_strategy: n in 0..64, strategy in 0..4");
  if (!g_strategy_init) strategy_defaults();
  g_strategy[fp32 ? 1 : 0][n] = strategy;
  return WF_OK;
}

template <class T>
static int try_coarse_cluster(const Lvl<T>& L, int nsweeps, cudaStream_t s, int* rc) {
  switch (L.n) {
    case 6: *rc = launch_coarse_cluster<T, 6, 1>(L, nsweeps, s); return 1;
    case 8: *rc = launch_coarse_cluster<T, 8, 1>(L, nsweeps, s); return 1;
    case 10: *rc = launch_coarse_cluster<T, 10, 2>(L, nsweeps, s); return 1;
    case 12: *rc = launch_coarse_cluster<T, 12, 2>(L, nsweeps, s); return 1;
    case 14: *rc = launch_coarse_cluster<T, 14, 2>(L, nsweeps, s); return 1;
    case 16: *rc = launch_coarse_cluster<T, 16, 2>(L, nsweeps, s); return 1;
    case 20: *rc = launch_coarse_cluster<T, 20, 4>(L, nsweeps, s); return 1;
    case 24: *rc = launch_coarse_cluster<T, 24, 3>(L, nsweeps, s); return 1;
    case 28: *rc = launch_coarse_cluster<T, 28, 4>(L, nsweeps, s); return 1;
    case 32: *rc = launch_coarse_cluster<T, 32, 4>(L, nsweeps, s); return 1;
    default: return 0;
  }
}

// ---- red-black sweeps on a row-parity-split copy (large levels) -----------
// A large level relaxes on a scratch copy whose rows are stored split by the
// parity of the array index a = k+1: position of a in its row is
// (a&1)*H + (a>>1), H = (n+2)/2.  Within a row the cells of one colour then
// form one contiguous half-row, so a half-sweep reads the other colour (half
// the level), the rhs of its own colour (from a split copy of rhs) and writes
// its own colour: 1.5 words per cell, against 3 words of whole cache lines in
// the interleaved layout.  Every cell keeps k_rbgs's arithmetic (same terms,
// same order, division by ap), so results are bit-identical to it.  The copy
// has the ring of the original (face-ring values only ever meet a zero
// coefficient); copying back writes the real cells and their face-ring
// mirrors, which is what k_rbgs leaves in the ring after the last sweep.
constexpr int SPLIT_ROWS = 8;  // rows (one warp each) per CTA

// level phi (all (n+2)^3 cells) and rhs -> split copies sp, sr (dense strides)
template <class T>
__global__ void __launch_bounds__(32 * SPLIT_ROWS)
    k_split_in(const Lvl<T> L0, T* sp, T* sr, int with_rhs, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> L = rebase(L0, bt);
  if (bt.tab) {
    sp = L.tmp;
    sr = L.tmp + (long)(L.n + 2) * (L.n + 2) * (L.n + 2);
  }
  const int m = L.n + 2, H = m >> 1;
  const int row = blockIdx.x * SPLIT_ROWS + (threadIdx.x >> 5);
  if (row >= m * m) return;
  const int i = row / m, j = row - i * m;
  const long src = (long)i * L.sI + (long)j * L.sJ;
  const long dst = (long)i * L.tI + (long)j * L.tJ;
  for (int a = threadIdx.x & 31; a < m; a += 32) {
    const int q = spos(a, H);
    const T x = L.phi[src + a];
    const T y = with_rhs ? L.rhs[src + a] : T(0);   // both loads before the stores
    sp[dst + q] = x;
    if (with_rhs) sr[dst + q] = y;
  }
}

// one colour half-sweep on the split copy: a warp updates CPT runs of 32
// consecutive cells of one colour in one real row (cells h, h+32, ...); grid
// x = chunk of 32*CPT cells of the half-row, y = group of blockDim.y rows j
// (at most SPLIT_ROWS; CPT and the rows are chosen per size), z = plane i.  All loads of a thread come before its stores: a half-sweep
// reads only the other colour and rhs, which it does not write.
template <class T, int CPT>
__global__ void __launch_bounds__(32 * SPLIT_ROWS)
    k_rbgs_split(const Lvl<T> L0, T* sp, const T* sr, int color,
                 const __grid_constant__ ApRecip<T> rt, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> L = rebase(L0, bt);
  if (bt.tab) {
    sp = L.tmp;
    sr = L.tmp + (long)(L.n + 2) * (L.n + 2) * (L.n + 2);
  }
  const int n = L.n, nh = n >> 1;
  const int h0 = blockIdx.x * 32 * CPT + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = bt_z(bt);
  if (j >= n || h0 >= nh) return;
  const int H = (n + 2) >> 1, tI = (int)L.tI, tJ = (int)L.tJ;
  const int pr = (i + j + color) & 1;       // parity of a = k+1 of this row's colour
  const long r = (long)(i + 1) * L.tI + (long)(j + 1) * L.tJ;
  T* own = sp + r + (pr * H + 1 - pr + h0);  // a = 2*(h+1-pr) + pr
  const T* oth = sp + r + ((1 - pr) * H + h0);  // a-1, a+1
  const T* rr = sr + r + (pr * H + 1 - pr + h0);
  const T aw = i > 0 ? L.ax : T(0), ae = i < n - 1 ? L.ax : T(0);
  const T as = j > 0 ? L.ay : T(0), an = j < n - 1 ? L.ay : T(0);
  const int pij = 9 * ((i > 0) + (i < n - 1)) + 3 * ((j > 0) + (j < n - 1));
  T vw[CPT], ve[CPT], vs[CPT], vn[CPT], vb[CPT], vt[CPT], vr[CPT];
#pragma unroll
  for (int u = 0; u < CPT; ++u) {
    if (u == 0 || h0 + 32 * u < nh) {
      vw[u] = own[32 * u - tI];
      ve[u] = own[32 * u + tI];
      vs[u] = own[32 * u - tJ];
      vn[u] = own[32 * u + tJ];
      vb[u] = oth[32 * u];
      vt[u] = oth[32 * u + 1];
      vr[u] = rr[32 * u];
    }
  }
#pragma unroll
  for (int u = 0; u < CPT; ++u) {
    if (u == 0 || h0 + 32 * u < nh) {
      const int k = 2 * (h0 + 32 * u) + 1 - pr;
      const T ab = k > 0 ? L.az : T(0), at = k < n - 1 ? L.az : T(0);
      const T ap = -(aw + ae + as + an + ab + at);
      const T s = aw * vw[u] + ae * ve[u] + as * vs[u] + an * vn[u] + ab * vb[u] + at * vt[u];
      own[32 * u] = div_by_recip(vr[u] - s, ap, rt.y[pij + (k > 0) + (k < n - 1)]);
    }
  }
}

// split copy -> real cells of the level and their face-ring mirrors
template <class T>
__global__ void __launch_bounds__(32 * SPLIT_ROWS)
    k_split_out(const Lvl<T> L0, const T* sp, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> L = rebase(L0, bt);
  if (bt.tab) sp = L.tmp;
  const int n = L.n, H = (n + 2) >> 1;
  const int row = blockIdx.x * SPLIT_ROWS + (threadIdx.x >> 5);
  if (row >= n * n) return;
  const int i = row / n, j = row - i * n;
  const long r = (long)(i + 1) * L.tI + (long)(j + 1) * L.tJ;
  // four loads in flight before their stores (the copy and the level are
  // different buffers; the compiler cannot tell, and would otherwise wait
  // for each load's round trip after the previous store)
  for (int k0 = threadIdx.x & 31; k0 < n; k0 += 128) {
    T x[4];
#pragma unroll
    for (int b = 0; b < 4; ++b)
      if (k0 + 32 * b < n) x[b] = sp[r + spos(k0 + 32 * b + 1, H)];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int k = k0 + 32 * b;
      if (k < n) {
        const long c = lid(L, i + 1, j + 1, k + 1);
        L.phi[c] = x[b];
        ring_mirror(L, i, j, k, c, x[b]);
      }
    }
  }
}

// smallest even level edge that relaxes on the split copy (WF_SPLIT_MIN
// overrides both): 80 for FP64, 128 for FP32, whose 80^3 level stays in L2
// (step time at 80^3, FP64 1.332 ms split vs 1.348 in place; mixed 1.255 vs 1.184)
static int split_min_n(bool fp32) {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("WF_SPLIT_MIN");
    v = e ? atoi(e) : 0;
  }
  return v > 0 ? v : (fp32 ? 128 : 80);
}

// level -> split copies (phi, and rhs unless the scratch already holds it)
template <class T>
static int split_in(const Lvl<T>& L, bool with_rhs, cudaStream_t s) {
  const int m = L.n + 2;
  T* sp = L.tmp;
  T* sr = L.tmp + (long)m * m * m;
  WF_CK(launch_k(k_split_in<T>, (m * m + SPLIT_ROWS - 1) / SPLIT_ROWS, 32 * SPLIT_ROWS, 0, s, L,
                 sp, sr, with_rhs ? 1 : 0));
  WF_CKL("k_split_in");
  return WF_OK;
}

// the half-sweeps of a relax on the split copies
template <class T>
static int split_sweeps(const Lvl<T>& L, int nsweeps, cudaStream_t s) {
  const int m = L.n + 2;
  T* sp = L.tmp;
  const T* sr = L.tmp + (long)m * m * m;
  int cpt, rows, one;
  launch_shape(SHAPE_SPLIT, L.n, &cpt, &rows, &one);   // cpt in {1, 2, 4, 8}, rows <= SPLIT_ROWS
  const dim3 grid((L.n / 2 + 32 * cpt - 1) / (32 * cpt), (L.n + rows - 1) / rows, L.n);
  const ApRecip<T> rt = ap_recip(L);
  auto kern = cpt == 8   ? k_rbgs_split<T, 8>
              : cpt == 4 ? k_rbgs_split<T, 4>
              : cpt == 2 ? k_rbgs_split<T, 2>
                         : k_rbgs_split<T, 1>;
  for (int it = 0; it < nsweeps; ++it) {
    for (int color = 0; color < 2; ++color) {
      WF_CK(launch_k(kern, grid, dim3(32, rows), 0, s, L, sp, sr, color, rt));
      WF_CKL("k_rbgs_split");
    }
  }
  return WF_OK;
}

// split copy of phi -> the level's real cells and face-ring mirrors
template <class T>
static int split_out(const Lvl<T>& L, cudaStream_t s) {
  WF_CK(launch_k(k_split_out<T>, (L.n * L.n + SPLIT_ROWS - 1) / SPLIT_ROWS, 32 * SPLIT_ROWS, 0,
                 s, L, (const T*)L.tmp));
  WF_CKL("k_split_out");
  return WF_OK;
}

// rhs_ready: the scratch already holds the split rhs of this level (the
// level's rhs has not changed since the last split relax of it)
template <class T>
static int relax_split(const Lvl<T>& L, int nsweeps, bool rhs_ready, cudaStream_t s) {
  WF_TRY(split_in(L, !rhs_ready, s));
  WF_TRY(split_sweeps(L, nsweeps, s));
  return split_out(L, s);
}

// The V-cycle keeps large levels in the split layout from their
// pre-smoothing to their post-smoothing: restriction reads and writes split
// views, prolongation adds into them, and only level 0 is copied in and out
// once per V-cycle.  A split view addresses the scratch copies through lid().
template <class T>
static Lvl<T> split_view(const Lvl<T>& L) {
  Lvl<T> V = L;
  V.role = L.role | LV_SPLIT;
  const long m = (long)L.n + 2;
  V.phi = L.tmp;
  V.rhs = L.tmp + m * m * m;
  V.sI = L.tI;
  V.sJ = L.tJ;
  V.split = 1;
  return V;
}

// face-ring mirrors of a split view (what k_rbgs leaves in the ring; the
// prolongation out of this level reads them)
template <class T>
__global__ void __launch_bounds__(256) k_split_ring(const Lvl<T> V0, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<T> V = rebase(V0, bt);
  const int n = V.n;
  const int t = blockIdx.x * 256 + threadIdx.x;
  if (t >= 6 * n * n) return;
  const int face = t / (n * n), r = t - face * n * n;
  const int a = r / n + 1, b = r % n + 1;   // the two in-face coordinates, 1..n
  const int lo = (face & 1) ? n + 1 : 0, in = (face & 1) ? n : 1;
  long dst, src;
  if (face < 2) {
    dst = lid(V, lo, a, b);
    src = lid(V, in, a, b);
  } else if (face < 4) {
    dst = lid(V, a, lo, b);
    src = lid(V, a, in, b);
  } else {
    dst = lid(V, a, b, lo);
    src = lid(V, a, b, in);
  }
  V.phi[dst] = V.phi[src];
}

// ---- one whole red-black sweep per launch (fine levels) -------------------
// Red values depend only on the old black values, so a sweep can run as one
// launch if every CTA reads the old state from `src` and writes the new
// state to a different buffer `dst` (the two buffers alternate over the
// sweeps of a relax; an even sweep count ends in the level's own array).
// A CTA owns a TJ x TK tile of (j,k) columns and a segment of i-planes and
// marches along i with a 4-plane window in shared memory covering the tile
// plus a 2-cell halo: at plane p it computes red on the tile plus a 1-cell
// halo (the halo redundantly, from old black values), then black on plane
// p-1 of the tile, and stores both colours of plane p-1.  Red is also
// computed redundantly on the plane before and after the segment.  Every
// cell keeps the reference's arithmetic (same terms, same order, division by
// ap), so results equal the one-colour-per-launch kernel bit for bit.  The
// face-ring mirrors are written on the last sweep of a relax only; no sweep
// reads the ring (its coefficients are zero).
template <int TJ, int TK>
struct SweepTile {
  static constexpr int WJ = TJ + 4, WK = TK + 4;
  static constexpr int WH = WK / 2;            // cells per parity half-row
  static constexpr int PLANE = WJ * WK;
  static constexpr int THREADS = 32 * (TJ + 2);  // one warp per row of the red region
};

// Window layout: [plane slot 4][k parity 2][row WJ][WH].  Cell (jj, kk) sits
// in half-row kk&1 at index kk>>1; k k0 is even, so within a row of plane q
// the red cells are exactly one parity half-row ((1 + q + j) & 1) and the
// black cells the other.  A warp owns a row, lane = index in the half-row:
// every access of a warp (its own cells, k+-1 in the other half-row, j+-1
// in the same half-row of the adjacent rows, i+-1 in the adjacent planes)
// is a contiguous run, free of bank conflicts.
template <class T, int TJ, int TK>
__global__ void __launch_bounds__(SweepTile<TJ, TK>::THREADS)
    k_sweep2(const T* src, long sIs, long sJs, T* dst, long sId,
             long sJd, const T* rhs, long sIr, long sJr, int n, T ax, T ay,
             T az, int seg, int write_ring) {
  pdl_entry();
  using W = SweepTile<TJ, TK>;
  constexpr int WJ = W::WJ, WK = W::WK, WH = W::WH, PLANE = W::PLANE, NT = W::THREADS;
  constexpr int HALF = WJ * WH;                // one parity of a plane
  constexpr int PER = (PLANE + NT - 1) / NT;
  static_assert(TK == 64, "lane mapping assumes 32 cells per parity half-row");
  __shared__ T win[4][PLANE];
  __shared__ T rb[2][PLANE];
  const int ntk = (n + TK - 1) / TK;
  const int j0 = (blockIdx.x / ntk) * TJ;
  const int k0 = (blockIdx.x % ntk) * TK;
  const int i0 = blockIdx.y * seg;
  const int i1 = min(n, i0 + seg);
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  // loader mapping: element e of this thread = window cell (jj, kk), kk fastest
  long offs[PER], roff[PER];
  int sidx[PER];
  bool okp[PER], okr[PER];
#pragma unroll
  for (int e = 0; e < PER; ++e) {
    const int t = tid + e * NT;
    const int jj = t / WK, kk = t - jj * WK;
    const int j = j0 - 2 + jj, k = k0 - 2 + kk;
    okp[e] = t < PLANE && j >= -1 && j <= n && k >= -1 && k <= n;
    okr[e] = t < PLANE && j >= 0 && j < n && k >= 0 && k < n;
    offs[e] = okp[e] ? (long)(j + 1) * sJs + (k + 1) : 0;
    roff[e] = okr[e] ? (long)(j + 1) * sJr + (k + 1) : 0;
    sidx[e] = t < PLANE ? (kk & 1) * HALF + jj * WH + (kk >> 1) : 0;
  }
  T pf[PER], rf[PER];
  auto fetch = [&](int q) {  // phi of plane q and rhs of plane q-1 into registers
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      pf[e] = (okp[e] && q <= n) ? src[(long)(q + 1) * sIs + offs[e]] : T(0);
      rf[e] = (okr[e] && q - 1 >= 0 && q - 1 < n) ? rhs[(long)q * sIr + roff[e]] : T(0);
    }
  };
  auto deposit = [&](int q) {
    T* w = win[(q + 4) & 3];
    T* r = rb[(q + 3) & 1];
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      if (tid + e * NT < PLANE) {
        w[sidx[e]] = pf[e];
        r[sidx[e]] = rf[e];
      }
    }
  };
  // one update of cell (row jj, parity par, index h) of plane pl (real index)
  auto update = [&](int pl, int jj, int par, int h, T* wc, const T* wm, const T* wp,
                    const T* rr) {
    const int kk = 2 * h + par;
    const int j = j0 - 2 + jj, k = k0 - 2 + kk;
    if (j < 0 || j >= n || k < 0 || k >= n) return;
    const int c = par * HALF + jj * WH + h;
    const int ck = (1 - par) * HALF + jj * WH;          // other half-row of this row
    const int km = ck + (par ? h : h - 1);              // kk-1
    const int kp = ck + (par ? h + 1 : h);              // kk+1
    const T aw = pl > 0 ? ax : T(0), ae = pl < n - 1 ? ax : T(0);
    const T as = j > 0 ? ay : T(0), an = j < n - 1 ? ay : T(0);
    const T ab = k > 0 ? az : T(0), at = k < n - 1 ? az : T(0);
    const T ap = -(aw + ae + as + an + ab + at);
    const T sum = aw * wm[c] + ae * wp[c] + as * wc[c - WH] + an * wc[c + WH] +
                  ab * wc[km] + at * wc[kp];
    wc[c] = (rr[c] - sum) / ap;
  };
  if (i0 - 2 >= -1) {
    fetch(i0 - 2);
    deposit(i0 - 2);
  }
  fetch(i0 - 1);
  deposit(i0 - 1);
  fetch(i0);
  for (int p = i0 - 1; p <= i1; ++p) {
    __syncthreads();
    deposit(p + 1);
    __syncthreads();
    if (p + 2 <= i1 + 1) fetch(p + 2);
    // red on plane p over rows 1..TJ+2 (warp = row), cells kk in 1..TK+2
    if (p >= 0 && p < n) {
      T* wc = win[(p + 4) & 3];
      const T* wm = win[(p + 3) & 3];
      const T* wp = win[(p + 5) & 3];
      const T* rr = rb[p & 1];
      const int jj = 1 + warp;
      const int j = j0 - 2 + jj;
      const int par = (1 + p + j) & 1;  // half-row holding the red cells (k0 even)
      // red kk range [1, TK+2]: parity 1 -> h 0..TK/2, parity 0 -> h 1..TK/2+1
      const int hlo = par ? 0 : 1;
      update(p, jj, par, hlo + lane, wc, wm, wp, rr);
      if (lane == 0) update(p, jj, par, hlo + 32, wc, wm, wp, rr);
    }
    __syncthreads();
    // black on plane q = p-1, rows 2..TJ+1, then store both colours of q
    const int q = p - 1;
    if (q >= i0 && q < i1 && warp < TJ) {
      T* wc = win[(q + 4) & 3];
      const T* wm = win[(q + 3) & 3];
      const T* wp = win[(q + 5) & 3];
      const T* rr = rb[q & 1];
      const int jj = 2 + warp;
      const int j = j0 - 2 + jj;
      const int par = (q + j) & 1;      // half-row holding the black cells
      update(q, jj, par, 1 + lane, wc, wm, wp, rr);
      __syncwarp();
      if (j < n) {
#pragma unroll
        for (int pp = 0; pp < 2; ++pp) {
          const int kk = 2 * (1 + lane) + pp;   // tile cells kk 2..TK+1
          const int k = k0 - 2 + kk;
          if (k >= n) continue;
          const T x = wc[pp * HALF + jj * WH + 1 + lane];
          const long o = (long)(q + 1) * sId + (long)(j + 1) * sJd + (k + 1);
          dst[o] = x;
          if (write_ring) {
            if (q == 0) dst[o - sId] = x;
            if (q == n - 1) dst[o + sId] = x;
            if (j == 0) dst[o - sJd] = x;
            if (j == n - 1) dst[o + sJd] = x;
            if (k == 0) dst[o - 1] = x;
            if (k == n - 1) dst[o + 1] = x;
          }
        }
      }
    }
  }
}

constexpr int SWEEP_TJ = 8, SWEEP_TK = 64;

// smallest level edge that uses one-launch sweeps (WF_SWEEP2_MIN overrides)
static int sweep2_min_n() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("WF_SWEEP2_MIN");
    v = e ? atoi(e) : 1 << 30;
  }
  return v;
}

template <class T>
static int launch_sweep2(const T* src, long sIs, long sJs, T* dst, long sId, long sJd,
                         const Lvl<T>& L, int write_ring, cudaStream_t s) {
  const int n = L.n;
  const int ntj = (n + SWEEP_TJ - 1) / SWEEP_TJ, ntk = (n + SWEEP_TK - 1) / SWEEP_TK;
  // at least ~2 CTAs per SM, segments of 4 to 32 planes
  int nseg = std::max(1, (2 * 148 + ntj * ntk - 1) / (ntj * ntk));
  int seg = std::min(32, std::max(4, (n + nseg - 1) / nseg));
  nseg = (n + seg - 1) / seg;
  WF_CK(launch_k(k_sweep2<T, SWEEP_TJ, SWEEP_TK>, dim3(ntj * ntk, nseg), SweepTile<SWEEP_TJ, SWEEP_TK>::THREADS, 0, s, src, sIs, sJs, dst, sId, sJd, L.rhs, L.sI, L.sJ, n,
                                            L.ax, L.ay, L.az, seg, write_ring));
  WF_CKL("k_sweep2");
  return WF_OK;
}

// ---- a whole relax of a fine level in one cooperative launch --------------
// The same half-sweep body as k_rbgs, all 2*nsweeps half-sweeps in one
// launch with a grid barrier between them, so a 6-sweep relax costs one
// launch instead of twelve.  The launch is cooperative (all CTAs resident);
// the barrier is a sense-reversing counter in the case's scalar block whose
// waits are bounded: a timeout records WF_ST_WAIT_TIMEOUT and the kernel
// finishes its remaining half-sweeps without waiting (results then invalid,
// the host raises).
constexpr int GBAR_SPINS = 1 << 22;

__device__ __forceinline__ void grid_barrier(unsigned* gbar, unsigned nblocks, int* err,
                                             bool& timed_out, int spins = GBAR_SPINS) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = gbar + 1;
    const unsigned gen = *vgen;
    __threadfence();
    if (atomicAdd(gbar, 1u) == nblocks - 1) {
      gbar[0] = 0u;
      __threadfence();
      atomicAdd(gbar + 1, 1u);
    } else if (!timed_out) {
      int it = 0;
      while (*vgen == gen) {
        if (++it > spins) {
          timed_out = true;
          if (err) atomicExch(err, (int)WF_ST_WAIT_TIMEOUT);
          break;
        }
        __nanosleep(20);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(MG_TPB) k_relax_persist(const Lvl<T> L, int nsweeps) {
  pdl_entry();
  const int n = L.n;
  const int nh = (n + 1) >> 1;
  const long tot = (long)n * n * nh;
  bool timed_out = false;
  for (int hs = 0; hs < 2 * nsweeps; ++hs) {
    const int color = hs & 1;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot;
         t += (long)gridDim.x * blockDim.x) {
      const int kk = (int)(t % nh);
      const int j = (int)((t / nh) % n);
      const int i = (int)(t / ((long)nh * n));
      const int k = 2 * kk + ((1 + i + j + color) & 1);
      if (k >= n) continue;
      const long c = lid(L, i + 1, j + 1, k + 1);
      const T aw = i > 0 ? L.ax : T(0), ae = i < n - 1 ? L.ax : T(0);
      const T as = j > 0 ? L.ay : T(0), an = j < n - 1 ? L.ay : T(0);
      const T ab = k > 0 ? L.az : T(0), at = k < n - 1 ? L.az : T(0);
      const T ap = -(aw + ae + as + an + ab + at);
      const T* phi = L.phi;
      const T s = aw * phi[c - L.sI] + ae * phi[c + L.sI] + as * phi[c - L.sJ] +
                  an * phi[c + L.sJ] + ab * phi[c - 1] + at * phi[c + 1];
      const T x = (L.rhs[c] - s) / ap;
      L.phi[c] = x;
      ring_mirror(L, i, j, k, c, x);
    }
    if (hs + 1 < 2 * nsweeps) grid_barrier(L.gbar, gridDim.x, L.err, timed_out);
  }
}

template <class T>
static int launch_relax_persist(const Lvl<T>& L, int nsweeps, cudaStream_t s, bool* done) {
  if (batch_ctx().tab) return fail(WF_EUNSUPPORTED, "cluster and cooperative relaxes do not run in a bucket");
  *done = false;
  static int blocks_per_sm[2] = {-1, -1};
  int& bps = blocks_per_sm[sizeof(T) == 4 ? 1 : 0];
  if (bps < 0) {
    WF_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_relax_persist<T>, MG_TPB, 0));
  }
  int dev = 0, nsm = 0;
  WF_CK(cudaGetDevice(&dev));
  WF_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const long half = (long)L.n * L.n * ((L.n + 1) / 2);
  long want = (half + MG_TPB - 1) / MG_TPB;
  const long cap = (long)nsm * std::max(1, std::min(bps, 4));
  const int nb = (int)std::max(1L, std::min(want, cap));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nb, 1, 1);
  cfg.blockDim = dim3(MG_TPB, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  WF_CK(cudaLaunchKernelEx(&cfg, k_relax_persist<T>, L, nsweeps));
  WF_CKL("k_relax_persist");
  *done = true;
  return WF_OK;
}

// smallest level edge that relaxes in one cooperative launch (WF_PERSIST_MIN)
static int persist_min_n() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("WF_PERSIST_MIN");
    v = e ? atoi(e) : 1 << 30;
  }
  return v;
}

// ---- a check of the bounded waits ------------------------------------------
// kind 0: the grid barrier above, entered by the one launched CTA with a
// declared count of two, so the barrier can never open; kind 1: the
// mbarrier wait of the point-to-point coarse kernel on a barrier that
// expects 8 bytes which nobody sends.  Either wait gives up after `tries`
// tries and records WF_ST_WAIT_TIMEOUT in *err; nothing is in flight when
// the kernel returns.
__global__ void k_wait_probe(unsigned* gbar, int* err, int kind, int tries) {
  if (kind == 0) {
    bool timed_out = false;
    grid_barrier(gbar, gridDim.x + 1, err, timed_out, tries);
    return;
  }
  __shared__ __align__(8) unsigned long long mbar;
  const uint32_t mb = smem_u32(&mbar);
  if (threadIdx.x == 0) {
    mbar_init(mb, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_arrive_expect_tx(mb, 8u);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    bool ok = false;
    for (int it = 0; it < tries && !ok; ++it) ok = mbar_try_wait(mb, 0u, 1);
    if (!ok && err) atomicExch(err, (int)WF_ST_WAIT_TIMEOUT);
  }
  __syncthreads();
}

int wait_probe(unsigned* gbar, int* err, int kind, int tries, cudaStream_t s) {
  if (!gbar || !err) return fail(WF_EINVAL, "wf_wait_probe: null gbar or err");
  if (kind != 0 && kind != 1) return fail(WF_EINVAL, "wf_wait_probe: kind must be 0 or 1");
  if (tries < 1 || tries > MBAR_WAIT_TRIES)
    return fail(WF_EINVAL, "wf_wait_probe: tries must be 1 .. 2^22");
  k_wait_probe<<<1, 32, 0, s>>>(gbar, err, kind, tries);
  WF_CKL("k_wait_probe");
  return WF_OK;
}

// max |rhs - A phi| over a level (tests/test_mg.py:16-32)
__global__ void k_resmax(const Lvl<double> L, double* out, unsigned int* ticket,
                         unsigned long long* acc) {
  pdl_entry();
  __shared__ double sm[32];
  const int n = L.n;
  double m = 0.0;
  // 1-D CTAs of 32 (k) x 8 (j) threads stepping through planes i by gridDim.z
  const int k = blockIdx.x * 32 + (threadIdx.x & 31);
  const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
  const bool in = k < n && j < n;
  for (int i = blockIdx.z; in && i < n; i += gridDim.z) {
    const long c = lid(L, i + 1, j + 1, k + 1);
    const double aw = i > 0 ? L.ax : 0.0, ae = i < n - 1 ? L.ax : 0.0;
    const double as = j > 0 ? L.ay : 0.0, an = j < n - 1 ? L.ay : 0.0;
    const double ab = k > 0 ? L.az : 0.0, at = k < n - 1 ? L.az : 0.0;
    const double ap = -(aw + ae + as + an + ab + at);
    const double* p = L.phi;
    const double r = L.rhs[c] - (ap * p[c] + aw * p[c - L.sI] + ae * p[c + L.sI] +
                                 as * p[c - L.sJ] + an * p[c + L.sJ] + ab * p[c - 1] +
                                 at * p[c + 1]);
    m = fmax(m, fabs(r));
  }
  m = block_max(m, sm);
  if (threadIdx.x == 0) atomicMax(acc, okey(m));
  if (!last_block(ticket, gridDim.x * gridDim.y * gridDim.z)) return;
  if (threadIdx.x == 0) {
    *out = okey_inv(atomicAdd(acc, 0ull));
    *acc = okey(0.0);
  }
}

// --------------------------------------------------------------------------
// host side
// --------------------------------------------------------------------------
static inline int mg_blocks(long work) {
  long b = (work + MG_TPB - 1) / MG_TPB;
  b = std::min<long>(b, 148L * 8);
  return (int)std::max<long>(b, 1);
}

template <class T>
static size_t smem_bytes(int n) {
  return 2ull * (size_t)n * n * n * sizeof(T);
}

constexpr size_t SMEM_CAP = 220 * 1024;

// rhs_ready: the level's rhs is unchanged since its last relax, so a split
// copy of it made then can be reused
template <class T>
static int relax(const Lvl<T>& L, int nsweeps, cudaStream_t s, bool rhs_ready = false) {
  if (nsweeps <= 0) return WF_OK;
  // a bucket launch serves many cases through their table: only kernels that
  // take one (the one-CTA column kernel, split and plain sweeps, the
  // shared-memory relax) run there
  const bool bucket = batch_ctx().tab != nullptr;
  // small levels with many sweeps: the column kernel
  if (nsweeps > 12 || L.n <= 24) {
    // small levels: one CTA, or a cluster when there are many sweeps
    int rc = WF_OK;
    const int strat = bucket ? 0 : coarse_strategy(L.n, sizeof(T) == 4);
    if (nsweeps > 12 && strat == 4 && try_coarse_p2p_thin<T>(L, nsweeps, s, &rc)) return rc;
    if (nsweeps > 12 && strat == 3 && try_coarse_tb<T>(L, nsweeps, s, &rc)) return rc;
    if (nsweeps > 12 && strat == 2 && try_coarse_p2p<T>(L, nsweeps, s, &rc)) return rc;
    if (nsweeps > 12 && strat == 1 && try_coarse_cluster<T>(L, nsweeps, s, &rc)) return rc;
    if (try_coarse<T>(L, nsweeps, s, &rc)) return rc;
  }
  if (L.tmp && (L.n & 1) == 0 && L.n >= split_min_n(sizeof(T) == 4))
    return relax_split<T>(L, nsweeps, rhs_ready, s);
  if (!bucket) {
    int rc = WF_OK;
    if (try_relax_mid<T>(L, nsweeps, s, &rc)) return rc;
  }
  if (!bucket && L.tmp && nsweeps >= 2 && L.n >= sweep2_min_n()) {
    // pairs of one-launch sweeps: phi -> tmp -> phi
    const int pairs = nsweeps / 2;
    for (int p = 0; p < pairs; ++p) {
      WF_TRY(launch_sweep2<T>(L.phi, L.sI, L.sJ, L.tmp, L.tI, L.tJ, L, 0, s));
      const int ring = (p == pairs - 1 && (nsweeps & 1) == 0) ? 1 : 0;
      WF_TRY(launch_sweep2<T>(L.tmp, L.tI, L.tJ, L.phi, L.sI, L.sJ, L, ring, s));
    }
    if (nsweeps & 1) {
      const long half = (long)L.n * L.n * ((L.n + 1) / 2);
      const int nb = mg_blocks(half);
      WF_CK(launch_k(k_rbgs<T>, cells3(L.n, L.n, (L.n + 1) / 2), cell_block(), 0, s, L, 0));
      WF_CKL("k_rbgs");
      WF_CK(launch_k(k_rbgs<T>, cells3(L.n, L.n, (L.n + 1) / 2), cell_block(), 0, s, L, 1));
      WF_CKL("k_rbgs");
    }
    return WF_OK;
  }
  if (!bucket && L.gbar && nsweeps >= 1 && L.n >= persist_min_n()) {
    bool done = false;
    WF_TRY(launch_relax_persist<T>(L, nsweeps, s, &done));
    if (done) return WF_OK;
  }
  const size_t sb = smem_bytes<T>(L.n);
  if (sb <= SMEM_CAP) {
    WF_CK(cudaFuncSetAttribute(k_relax_smem<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)SMEM_CAP));
    const int n3 = L.n * L.n * L.n;
    int tpb = 1024;
    if (n3 / 2 < 1024) tpb = std::max(32, ((n3 / 2 + 31) / 32) * 32);
    WF_CK(launch_k(k_relax_smem<T>, 1, tpb, sb, s, L, nsweeps));
    WF_CKL("k_relax_smem");
    return WF_OK;
  }
  const long half = (long)L.n * L.n * ((L.n + 1) / 2);
  const int nb = mg_blocks(half);
  for (int sw = 0; sw < nsweeps; ++sw) {
    WF_CK(launch_k(k_rbgs<T>, cells3(L.n, L.n, (L.n + 1) / 2), cell_block(), 0, s, L, 0));
    WF_CKL("k_rbgs");
    WF_CK(launch_k(k_rbgs<T>, cells3(L.n, L.n, (L.n + 1) / 2), cell_block(), 0, s, L, 1));
    WF_CKL("k_rbgs");
  }
  return WF_OK;
}

// a level the V-cycle keeps in the split layout: one that relax() would send
// to relax_split for both smoothings
template <class T>
static bool split_resident(const Lvl<T>& L, const wf_case& c) {
  return L.tmp && (L.n & 1) == 0 && L.n > 24 && L.n >= split_min_n(sizeof(T) == 4) &&
         c.n_pre >= 1 && c.n_pre <= 12 && c.n_post >= 1 && c.n_post <= 12;
}

// rhs0_ready: level 0's rhs is unchanged since the previous V-cycle relaxed
// it (a solve's V-cycles share rhs = su).  split0_in: level 0's split copy
// already holds its current phi (left there by the previous V-cycle);
// split0_keep: leave the result in the split copy (the next V-cycle of the
// same solve continues from it) instead of copying it back.
template <class T>
static int vcycle(std::vector<Lvl<T>>& lv, const wf_case& c, cudaStream_t s,
                  bool rhs0_ready = false, bool split0_in = false, bool split0_keep = false) {
  const int L = (int)lv.size();
  std::vector<Lvl<T>> vw(lv);    // the views restriction and prolongation work on
  std::vector<char> res(L, 0);   // level kept split from pre- to post-smoothing
  for (int l = 0; l + 1 < L; ++l)
    if (split_resident(lv[l], c)) {
      res[l] = 1;
      vw[l] = split_view(lv[l]);
    }
  for (int l = 0; l < L; ++l) {
    if (l > 0) {
      Lvl<T>& C = vw[l];
      WF_CK(launch_k(k_restrict<T>, cells3(C.n, C.n, C.n), cell_block(), 0, s,
          vw[l - 1], const_cast<T*>(C.rhs), C));
      WF_CKL("k_restrict");
    } else if (res[0] && !split0_in) {
      WF_TRY(split_in(lv[0], !rhs0_ready, s));
    }
    if (l == L - 1 && L > 1 && c.mg_cop && c.mg_cop_part && c.n_coarse >= 2 &&
        cop_size_ok(lv[l].n))
      WF_TRY(apply_coarse_op<T>(lv[l], (const T*)c.mg_cop, (T*)c.mg_cop_part, s));
    else if (res[l])
      WF_TRY(split_sweeps(lv[l], c.n_pre, s));
    else
      WF_TRY(relax(lv[l], l < L - 1 ? c.n_pre : c.n_coarse, s, l == 0 && rhs0_ready));
  }
  for (int l = L - 2; l >= 0; --l) {
    // fine levels from 64: one thread per coarse cell (fewer loads); smaller
    // ones keep one thread per fine cell (more threads in flight)
    if (lv[l].n >= 64 && (lv[l].n & 1) == 0) {
      WF_CK(launch_k(k_prolong8<T>, cells3(lv[l + 1].n, lv[l + 1].n, lv[l + 1].n), cell_block(),
                     0, s, vw[l + 1], vw[l]));
      WF_CKL("k_prolong8");
    } else {
      WF_CK(launch_k(k_prolong<T>, cells3(lv[l].n, lv[l].n, lv[l].n), cell_block(), 0, s,
                     vw[l + 1], vw[l]));
      WF_CKL("k_prolong");
    }
    if (res[l]) {
      WF_TRY(split_sweeps(lv[l], c.n_post, s));
      if (l > 0) {
        WF_CK(launch_k(k_split_ring<T>, (6 * lv[l].n * lv[l].n + 255) / 256, 256, 0, s, vw[l]));
        WF_CKL("k_split_ring");
      } else if (!split0_keep) {
        WF_TRY(split_out(lv[0], s));
      }
    } else {
      // the rhs of level l is the one its pre-smoothing saw
      WF_TRY(relax(lv[l], c.n_post, s, c.n_pre > 0 || (l == 0 && rhs0_ready)));
    }
  }
  return WF_OK;
}

// build the level views of a case; level 0 = (phi0, rhs0) with strides sI, sJ
template <class T>
static int build_levels(const wf_case& c, T* phi0, const T* rhs0, long sI, long sJ,
                        std::vector<Lvl<T>>& lv) {
  lv.clear();
  if (c.nlev < 1 || c.nlev > WF_MAX_LEVELS) return fail(WF_EINVAL, "nlev out of range");
  for (int l = 0; l < c.nlev; ++l) {
    Lvl<T> L;
    const double s2 = (double)(1 << l);
    const double dxl = c.dx * s2, dyl = c.dy * s2, dzl = c.dz * s2;
    L.ax = (T)(1.0 / (dxl * dxl));
    L.ay = (T)(1.0 / (dyl * dyl));
    L.az = (T)(1.0 / (dzl * dzl));
    L.n = c.n >> l;
    L.err = c.sc ? &c.sc->status : nullptr;
    L.tmp = (T*)c.mg_tmp[l];
    L.gbar = c.sc ? c.sc->gbar : nullptr;
    L.role = l;
    L.tJ = L.n + 2;
    L.tI = (long)(L.n + 2) * (L.n + 2);
    if ((L.n << l) != c.n || L.n < 1)
      return fail(WF_EINVAL, "n must be divisible by 2^(nlev-1)");
    if (l == 0) {
      L.phi = phi0;
      L.rhs = rhs0;
      L.sI = sI;
      L.sJ = sJ;
    } else {
      if (!c.mg_phi[l] || !c.mg_rhs[l]) return fail(WF_EINVAL, "missing multigrid level buffer");
      L.phi = (T*)c.mg_phi[l];
      L.rhs = (const T*)c.mg_rhs[l];
      L.sJ = L.n + 2;
      L.sI = (long)(L.n + 2) * (L.n + 2);
    }
    lv.push_back(L);
  }
  return WF_OK;
}

// ---- mixed precision: FP32 V-cycles inside an FP64 defect correction -------
// One cycle on the FP64 level-0 pair (phi, rhs):
//   r = rhs - A phi            (FP64, rounded once to FP32)
//   e = V-cycle from zero on A e = r, every level in FP32
//   phi += e                   (FP64, over the real cells and the ring)
// In exact arithmetic a V-cycle from phi equals phi + V(rhs - A phi), so the
// FP64 schedule of n_vcycles cycles is reproduced up to FP32 rounding of the
// corrections; residual and accumulation stay FP64.
// One thread per real cell (x = k in runs of 32, y = j in groups of 8, z = i),
// as the other stencil kernels: no 64-bit index division per cell.
__device__ __forceinline__ double defect_at(const Lvl<double>& F, int n, int i, int j, int k) {
  const long c = lid(F, i + 1, j + 1, k + 1);
  const double aw = i > 0 ? F.ax : 0.0, ae = i < n - 1 ? F.ax : 0.0;
  const double as = j > 0 ? F.ay : 0.0, an = j < n - 1 ? F.ay : 0.0;
  const double ab = k > 0 ? F.az : 0.0, at = k < n - 1 ? F.az : 0.0;
  const double ap = -(aw + ae + as + an + ab + at);
  const double* p = F.phi;
  return F.rhs[c] - (aw * p[c - F.sI] + ae * p[c + F.sI] + as * p[c - F.sJ] +
                     an * p[c + F.sJ] + ab * p[c - 1] + at * p[c + 1] + ap * p[c]);
}

// zero cell (i, j, k) (0-based real index) of an FP32 level array and the
// ring cells nearest to it (faces, edges, corners), so that the real cells'
// threads together zero every cell of the (n+2)^3 array exactly once
__device__ __forceinline__ void zero_with_ring(const Lvl<float>& L, int n, int i, int j, int k) {
  const int zi0 = i == 0 ? -1 : 0, zi1 = i == n - 1 ? 1 : 0;
  const int zj0 = j == 0 ? -1 : 0, zj1 = j == n - 1 ? 1 : 0;
  const int zk0 = k == 0 ? -1 : 0, zk1 = k == n - 1 ? 1 : 0;
  for (int oi = zi0; oi <= zi1; ++oi)
    for (int oj = zj0; oj <= zj1; ++oj)
      for (int ok = zk0; ok <= zk1; ++ok) L.phi[lid(L, i + 1 + oi, j + 1 + oj, k + 1 + ok)] = 0.0f;
}

// Lf: the FP32 level 0 (its own arrays, or with LV_SPLIT its split copies)
__global__ void __launch_bounds__(MG_TPB) k_defect(const Lvl<double> F0, const Lvl<float> Lf0,
                                                   const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<double> F = rebase(F0, bt);
  const Lvl<float> Lf = rebase(Lf0, bt);
  const int n = F.n;
  const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  if (k >= n || j >= n) return;
  const int i = bt_z(bt);
  const double r = defect_at(F, n, i, j, k);
  const_cast<float*>(Lf.rhs)[lid(Lf, i + 1, j + 1, k + 1)] = (float)r;
  // the FP32 correction starts from zero, ring included
  zero_with_ring(Lf, n, i, j, k);
}

// phi += the FP32 correction over the real cells and the ring.  With a split
// Lf the correction is read from the split copy, and the ring gets exactly
// what copying it back would have left in the level's own array: the face
// ring the value of the real cell next to it, edges and corners zero.
__global__ void k_correct(const Lvl<double> F0, const Lvl<float> Lf0, const Batch bt) {
  pdl_entry();
  if (bt_skip(bt)) return;
  const Lvl<double> F = rebase(F0, bt);
  const Lvl<float> Lf = rebase(Lf0, bt);
  const int n = F.n, m = n + 2;
  const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  if (k >= m || j >= m) return;
  const int i = bt_z(bt);
  float v;
  if (Lf.split) {
    const int oi = i == 0 || i == m - 1, oj = j == 0 || j == m - 1, ok = k == 0 || k == m - 1;
    v = 0.0f;
    if (oi + oj + ok <= 1) {
      const int ri = i == 0 ? 1 : (i == m - 1 ? n : i);
      const int rj = j == 0 ? 1 : (j == m - 1 ? n : j);
      const int rk = k == 0 ? 1 : (k == m - 1 ? n : k);
      v = Lf.phi[lid(Lf, ri, rj, rk)];
    }
  } else {
    v = Lf.phi[lid(Lf, i, j, k)];
  }
  F.phi[lid(F, i, j, k)] += (double)v;
}

static int build_levels_f32(const wf_case& c, std::vector<Lvl<float>>& lv) {
  lv.clear();
  for (int l = 0; l < c.nlev; ++l) {
    if (!c.mg_phi[l] || !c.mg_rhs[l]) return fail(WF_EINVAL, "missing FP32 multigrid buffer");
    Lvl<float> L;
    const double s2 = (double)(1 << l);
    const double dxl = c.dx * s2, dyl = c.dy * s2, dzl = c.dz * s2;
    L.ax = (float)(1.0 / (dxl * dxl));
    L.ay = (float)(1.0 / (dyl * dyl));
    L.az = (float)(1.0 / (dzl * dzl));
    L.n = c.n >> l;
    L.err = c.sc ? &c.sc->status : nullptr;
    L.tmp = (float*)c.mg_tmp[l];
    L.gbar = c.sc ? c.sc->gbar : nullptr;
    L.role = l;
    L.tJ = L.n + 2;
    L.tI = (long)(L.n + 2) * (L.n + 2);
    L.phi = (float*)c.mg_phi[l];
    L.rhs = (const float*)c.mg_rhs[l];
    L.sJ = L.n + 2;
    L.sI = (long)(L.n + 2) * (L.n + 2);
    lv.push_back(L);
  }
  return WF_OK;
}

static int dc_cycle(const Lvl<double>& F, std::vector<Lvl<float>>& lvf, const wf_case& c,
                    cudaStream_t s) {
  const int n = F.n, m = n + 2;
  // a split-resident FP32 level 0 stays in its split copy from the defect to
  // the correction: no copy into the split layout and none back
  const bool sp = lvf.size() > 1 && split_resident(lvf[0], c);
  const Lvl<float> Lf = sp ? split_view(lvf[0]) : lvf[0];
  WF_CK(launch_k(k_defect, cells3(n, n, n), cell_block(), 0, s, F, Lf));
  WF_CKL("k_defect");
  WF_TRY(vcycle<float>(lvf, c, s, sp, sp, sp));
  WF_CK(launch_k(k_correct, cells3(m, m, m), cell_block(), 0, s, F, Lf));
  WF_CKL("k_correct");
  return WF_OK;
}

static Lvl<double> level0_view(const wf_case& c, double* phi, const double* rhs, long sI,
                               long sJ) {
  Lvl<double> L;
  L.phi = phi;
  L.rhs = rhs;
  L.n = c.n;
  L.sI = sI;
  L.sJ = sJ;
  L.err = c.sc ? &c.sc->status : nullptr;
  L.tmp = nullptr;
  L.gbar = c.sc ? c.sc->gbar : nullptr;
  L.ax = 1.0 / (c.dx * c.dx);
  L.ay = 1.0 / (c.dy * c.dy);
  L.az = 1.0 / (c.dz * c.dz);
  return L;
}

int mg_dc_cycle_pair(const wf_case& c, double* phi0, const double* rhs0, cudaStream_t s) {
  const long m = c.n + 2;
  std::vector<Lvl<float>> lvf;
  WF_TRY(build_levels_f32(c, lvf));
  return dc_cycle(level0_view(c, phi0, rhs0, m * m, m), lvf, c, s);
}

// the coarsest level's coefficients 1/h^2 of case c, in the level's precision
static void coarse_coeffs(const wf_case& c, double a[3]) {
  const int l = c.nlev - 1;
  const double s2 = (double)(1 << l);
  const double dxl = c.dx * s2, dyl = c.dy * s2, dzl = c.dz * s2;
  a[0] = 1.0 / (dxl * dxl);
  a[1] = 1.0 / (dyl * dyl);
  a[2] = 1.0 / (dzl * dzl);
  if (c.mg_fp32)
    for (int d = 0; d < 3; ++d) a[d] = (double)(float)a[d];
}

int coarse_op_elems(const wf_case& c, int64_t* op_elems, int64_t* scratch_elems) {
  const int n = c.n, nlev = c.nlev;
  if (nlev < 2 || nlev > WF_MAX_LEVELS || n < 1) return fail(WF_EINVAL, "bad n or nlev");
  const int nc = n >> (nlev - 1);
  if ((nc << (nlev - 1)) != n) return fail(WF_EINVAL, "n must be divisible by 2^(nlev-1)");
  if (!cop_size_ok(nc))
    return fail(WF_EUNSUPPORTED, "coarse operator: coarsest edge must be 4..24, step 4");
  if (!(c.dx > 0 && c.dy > 0 && c.dz > 0)) return fail(WF_EINVAL, "cell sizes must be > 0");
  double a[3];
  coarse_coeffs(c, a);
  const CopPlan& P = cop_plan(nc, a[0], a[1], a[2], cop_full(nc, c.mg_fp32 != 0));
  if (op_elems) *op_elems = c.mg_fp32 ? P.op_elems<float>() : P.op_elems<double>();
  if (scratch_elems) *scratch_elems = cop_scratch_elems(P);
  return WF_OK;
}

int build_coarse_op_case(const wf_case& c, cudaStream_t s) {
  if (!c.mg_cop) return fail(WF_EINVAL, "mg_cop is null");
  WF_TRY(coarse_op_elems(c, nullptr, nullptr));
  const int l = c.nlev - 1;
  double a[3];
  coarse_coeffs(c, a);
  if (c.mg_fp32) {
    Lvl<float> L = {};
    L.n = c.n >> l;
    L.ax = (float)a[0];
    L.ay = (float)a[1];
    L.az = (float)a[2];
    return build_coarse_op<float>(L, c.n_coarse, (float*)c.mg_cop, s);
  }
  Lvl<double> L = {};
  L.n = c.n >> l;
  L.ax = a[0];
  L.ay = a[1];
  L.az = a[2];
  return build_coarse_op<double>(L, c.n_coarse, (double*)c.mg_cop, s);
}

int mg_solve(const wf_case& c, cudaStream_t s) {
  if (c.mg_fp32) {
    const long P = padded(c.n);
    const long off = (long)(NPL - 1) * (P * P + P + 1);
    double* pp = c.fld[WF_PP];
    std::vector<Lvl<float>> lvf;
    WF_TRY(build_levels_f32(c, lvf));
    Lvl<double> F = level0_view(c, pp + off, c.fld[WF_SU] + off, P * P, P);
    F.role = LV_PP;
    WF_CK(launch_k(k_zero<double>, mg_blocks(P * P * P), MG_TPB, 0, s, pp, P * P * P, (int)WF_PP));
    WF_CKL("k_zero pp");
    for (int cyc = 0; cyc < c.n_vcycles; ++cyc) WF_TRY(dc_cycle(F, lvf, c, s));
    return WF_OK;
  }
  const long P = padded(c.n);
  const long off = (long)(NPL - 1) * (P * P + P + 1);
  double* pp = c.fld[WF_PP];
  const double* su = c.fld[WF_SU];
  std::vector<Lvl<double>> lv;
  WF_TRY(build_levels<double>(c, pp + off, su + off, P * P, P, lv));
  lv[0].role = LV_PP;   // level 0 is the core of pp and su
  // multigrid.py:332-333: pp and level-0 phi start from zero
  WF_CK(launch_k(k_zero<double>, mg_blocks(P * P * P), MG_TPB, 0, s, pp, P * P * P, (int)WF_PP));
  WF_CKL("k_zero pp");
  // a level 0 kept in the split layout stays there from the first V-cycle's
  // copy-in to the last one's copy-out
  const bool keep = split_resident(lv[0], c) && lv.size() > 1;
  for (int cyc = 0; cyc < c.n_vcycles; ++cyc)
    WF_TRY(vcycle<double>(lv, c, s, cyc > 0 && (c.n_pre > 0 || c.n_post > 0),
                          keep && cyc > 0, keep && cyc + 1 < c.n_vcycles));
  return WF_OK;
}

int mg_vcycle_pair(const wf_case& c, double* phi0, const double* rhs0, cudaStream_t s) {
  const long m = c.n + 2;
  std::vector<Lvl<double>> lv;
  WF_TRY(build_levels<double>(c, phi0, rhs0, m * m, m, lv));
  return vcycle<double>(lv, c, s);
}

int mg_relax_pair(const wf_case& c, double* phi0, const double* rhs0, int nsweeps,
                  cudaStream_t s) {
  const long m = c.n + 2;
  std::vector<Lvl<double>> lv;
  WF_TRY(build_levels<double>(c, phi0, rhs0, m * m, m, lv));
  return relax<double>(lv[0], nsweeps, s);
}

// the coarsest-level solve of a V-cycle on an explicit (n_c+2)^3 pair: phi
// from zero by the case's coarse operator when it has one, else n_coarse
// sweeps
int mg_coarse_solve_pair(const wf_case& c, double* phi, const double* rhs, cudaStream_t s) {
  if (c.nlev < 2) return fail(WF_EINVAL, "coarse solve needs nlev >= 2");
  const int l = c.nlev - 1;
  Lvl<double> L = {};
  L.n = c.n >> l;
  if ((L.n << l) != c.n || L.n < 1) return fail(WF_EINVAL, "n must be divisible by 2^(nlev-1)");
  const double s2 = (double)(1 << l);
  const double dxl = c.dx * s2, dyl = c.dy * s2, dzl = c.dz * s2;
  L.ax = 1.0 / (dxl * dxl);
  L.ay = 1.0 / (dyl * dyl);
  L.az = 1.0 / (dzl * dzl);
  L.phi = phi;
  L.rhs = rhs;
  L.sJ = L.n + 2;
  L.sI = (long)(L.n + 2) * (L.n + 2);
  L.err = c.sc ? &c.sc->status : nullptr;
  L.gbar = c.sc ? c.sc->gbar : nullptr;
  const long m = (long)L.n + 2;
  WF_CK(launch_k(k_zero<double>, mg_blocks(m * m * m), MG_TPB, 0, s, phi, m * m * m, -1));
  WF_CKL("k_zero");
  if (c.mg_cop && c.mg_cop_part && !c.mg_fp32 && c.n_coarse >= 2 && cop_size_ok(L.n))
    return apply_coarse_op<double>(L, (const double*)c.mg_cop, (double*)c.mg_cop_part, s);
  return relax<double>(L, c.n_coarse, s);
}

__global__ void k_refill(Lvl<double> L) {
  pdl_entry();
  const int n = L.n;
  const long tot = (long)n * n;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot;
       t += (long)gridDim.x * blockDim.x) {
    const int a = 1 + (int)(t / n), b = 1 + (int)(t % n);
    double* p = L.phi;
    p[lid(L, 0, a, b)] = p[lid(L, 1, a, b)];
    p[lid(L, n + 1, a, b)] = p[lid(L, n, a, b)];
    p[lid(L, a, 0, b)] = p[lid(L, a, 1, b)];
    p[lid(L, a, n + 1, b)] = p[lid(L, a, n, b)];
    p[lid(L, a, b, 0)] = p[lid(L, a, b, 1)];
    p[lid(L, a, b, n + 1)] = p[lid(L, a, b, n)];
  }
}

int mg_refill_pair(const wf_case& c, double* phi0, cudaStream_t s) {
  const long m = c.n + 2;
  std::vector<Lvl<double>> lv;
  WF_TRY(build_levels<double>(c, phi0, phi0, m * m, m, lv));
  WF_CK(launch_k(k_refill, mg_blocks((long)c.n * c.n), MG_TPB, 0, s, lv[0]));
  WF_CKL("k_refill");
  return WF_OK;
}

int mg_residual_max_pair(const wf_case& c, const double* phi0, const double* rhs0,
                         double* out, cudaStream_t s) {
  if (!c.sc) return fail(WF_EINVAL, "residual needs the case scalar block");
  const long m = c.n + 2;
  std::vector<Lvl<double>> lv;
  WF_TRY(build_levels<double>(c, const_cast<double*>(phi0), rhs0, m * m, m, lv));
  const int gx = (c.n + 31) / 32, gy = (c.n + 7) / 8;
  const dim3 rg(gx, gy, std::max(1, std::min(c.n, (148 * 32) / (gx * gy))));
  WF_CK(launch_k(k_resmax, rg, MG_TPB, 0, s, lv[0], out, &c.sc->ticket,
                                                               &c.sc->red[5]));
  WF_CKL("k_resmax");
  return WF_OK;
}

// ---------------------------------------------------------------------------
// Multigrid solve for callers that cannot allocate device memory.
//
// Some host programs do not let a library allocate GPU memory at all: a
// Fortran or C++ flow solver that links this library through the C ABI and
// hands out every device buffer from its own fixed pool, or a service that
// admits work against a fixed memory budget and must know every byte in
// advance.  For them, wf_mg_solve_noalloc keeps the coarse multigrid levels
// (1 .. nlev-1) in one fixed array compiled into this library, so the
// caller passes only the right-hand side and the solution and nothing is
// allocated on any call.
//
// The array holds MG_NOALLOC_DOUBLES doubles (4 MiB) on every GPU that
// loads the library, for the life of the process; that is enough for n up
// to 112 at 3 levels.  Larger problems are rejected with WF_EINVAL.
// Host code cannot use the array's name as a device address, so the first
// call in each CUDA context looks the address up (with that context
// current) and caches it per context; make that first call before any
// stream capture.  The cache is keyed on the context's unique id, so a
// context created after cudaDeviceReset, or a host program's own driver
// context, gets its own lookup.  All calls share the array and only the
// last call's contents remain: every level is rewritten before it is read,
// and calls that overlap on the GPU (two streams, or two host threads) race
// on it.
//
// A device-side wait that gives up in a coarse-level kernel (a bounded
// wait, see WF_ST_WAIT_TIMEOUT) is recorded in a status word that sits next
// to the array; each call clears it first, and wf_mg_noalloc_status reads
// it after the caller's stream has finished.
// ---------------------------------------------------------------------------
constexpr long MG_NOALLOC_DOUBLES = 1L << 19;
static __device__ __align__(256) double g_mg_noalloc_scratch[MG_NOALLOC_DOUBLES];
static __device__ int g_mg_noalloc_status;

struct NoallocAddrs {
  unsigned long long ctx_id;
  double* scratch;
  int* status;
};

// unique id of the calling thread's current CUDA context (0: none current);
// the driver functions are looked up through the runtime, so the library
// does not link libcuda and still loads on a machine without a GPU
static int current_ctx_id(unsigned long long* id) {
  typedef CUresult (*GetCur)(CUcontext*);
  typedef CUresult (*GetId)(CUcontext, unsigned long long*);
  static GetCur get_cur = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_cur = reinterpret_cast<GetCur>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  if (!get_cur || !get_id) return fail(WF_EUNSUPPORTED, "driver lacks cuCtxGetCurrent/cuCtxGetId");
  CUcontext ctx = nullptr;
  *id = 0;
  if (get_cur(&ctx) != CUDA_SUCCESS) return fail(WF_ECUDA, "cuCtxGetCurrent failed");
  if (ctx && get_id(ctx, id) != CUDA_SUCCESS) return fail(WF_ECUDA, "cuCtxGetId failed");
  return WF_OK;
}

static int noalloc_addrs(NoallocAddrs* out) {
  static std::mutex mu;
  static std::vector<NoallocAddrs> cache;
  unsigned long long id = 0;
  WF_TRY(current_ctx_id(&id));
  std::lock_guard<std::mutex> lock(mu);
  if (id)
    for (const NoallocAddrs& a : cache)
      if (a.ctx_id == id) {
        *out = a;
        return WF_OK;
      }
  NoallocAddrs a{};
  void* p = nullptr;
  // the first runtime call of a thread without a current context makes the
  // device's primary context current; its id is read after the lookup
  cudaError_t e = cudaGetSymbolAddress(&p, g_mg_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(multigrid scratch)");
  a.scratch = static_cast<double*>(p);
  e = cudaGetSymbolAddress(&p, g_mg_noalloc_status);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(multigrid status)");
  a.status = static_cast<int*>(p);
  if (!id) WF_TRY(current_ctx_id(&id));
  if (!id) return fail(WF_ECUDA, "no current CUDA context after the symbol lookup");
  a.ctx_id = id;
  for (const NoallocAddrs& b : cache)
    if (b.ctx_id == id) {
      *out = b;
      return WF_OK;
    }
  cache.push_back(a);
  *out = a;
  return WF_OK;
}

// the V-cycle of multigrid.py:301-322 over a fixed array of level views
static int vcycle_fixed(Lvl<double>* lv, int L, const wf_case& c, cudaStream_t s) {
  for (int l = 0; l < L; ++l) {
    if (l > 0) {
      // k_restrict also zeroes the coarse phi, ring included
      WF_CK(launch_k(k_restrict<double>, cells3(lv[l].n, lv[l].n, lv[l].n), cell_block(), 0, s,
          lv[l - 1], const_cast<double*>(lv[l].rhs), lv[l]));
      WF_CKL("k_restrict");
    }
    WF_TRY(relax(lv[l], l < L - 1 ? c.n_pre : c.n_coarse, s));
  }
  for (int l = L - 2; l >= 0; --l) {
    WF_CK(launch_k(k_prolong<double>, cells3(lv[l].n, lv[l].n, lv[l].n), cell_block(), 0, s, 
        lv[l + 1], lv[l]));
    WF_CKL("k_prolong");
    WF_TRY(relax(lv[l], c.n_post, s));
  }
  return WF_OK;
}

int mg_solve_noalloc(const double* su, double* pp, int n, int nlev, double dx, double dy,
                     double dz, cudaStream_t s) {
  if (!su || !pp) return fail(WF_EINVAL, "wf_mg_solve_noalloc: null su or pp");
  if (n < 4 || nlev < 1 || nlev > WF_MAX_LEVELS || n % (1 << (nlev - 1)) != 0)
    return fail(WF_EINVAL, "wf_mg_solve_noalloc: n must be >= 4 and divisible by "
                           "2**(nlev-1), 1 <= nlev <= 8");
  if (!(dx > 0 && dy > 0 && dz > 0)) return fail(WF_EINVAL, "wf_mg_solve_noalloc: bad spacing");
  long need = 0;
  for (int l = 1; l < nlev; ++l) {
    const long m = (long)(n >> l) + 2;
    need += 2 * (((m * m * m) + 31) / 32) * 32;
  }
  if (need > MG_NOALLOC_DOUBLES)
    return fail(WF_EINVAL, "wf_mg_solve_noalloc: n=" + std::to_string(n) + " with " +
                               std::to_string(nlev) + " levels needs " + std::to_string(need) +
                               " doubles of multigrid scratch; the static array holds " +
                               std::to_string(MG_NOALLOC_DOUBLES) +
                               " (n <= 112 at 3 levels); use wf_mg_solve with caller buffers");
  NoallocAddrs ad{};
  WF_TRY(noalloc_addrs(&ad));
  double* base = ad.scratch;
  const long P = padded(n);
  const long off = (long)(NPL - 1) * (P * P + P + 1);
  Lvl<double> lv[WF_MAX_LEVELS];
  long used = 0;
  for (int l = 0; l < nlev; ++l) {
    const double s2 = (double)(1 << l);
    const double dxl = dx * s2, dyl = dy * s2, dzl = dz * s2;
    Lvl<double>& L = lv[l];
    L.err = ad.status;
    L.tmp = nullptr;
    L.gbar = nullptr;
    L.ax = 1.0 / (dxl * dxl);
    L.ay = 1.0 / (dyl * dyl);
    L.az = 1.0 / (dzl * dzl);
    L.n = n >> l;
    if (l == 0) {
      L.phi = pp + off;
      L.rhs = su + off;
      L.sI = P * P;
      L.sJ = P;
    } else {
      const long m = (long)L.n + 2;
      const long cnt = ((m * m * m + 31) / 32) * 32;
      L.phi = base + used;
      L.rhs = base + used + cnt;
      used += 2 * cnt;
      L.sJ = m;
      L.sI = m * m;
    }
  }
  wf_case c{};
  c.n_pre = 6;      // multigrid.py:257-260
  c.n_post = 6;
  c.n_coarse = 300;
  c.n_vcycles = 4;
  WF_CK(cudaMemsetAsync(ad.status, 0, sizeof(int), s));
  WF_CK(launch_k(k_zero<double>, mg_blocks(P * P * P), MG_TPB, 0, s, pp, P * P * P, (int)WF_PP));
  WF_CKL("k_zero pp");
  for (int cyc = 0; cyc < c.n_vcycles; ++cyc) WF_TRY(vcycle_fixed(lv, nlev, c, s));
  return WF_OK;
}

int mg_noalloc_status(void* stream, int32_t* status) {
  if (!status) return fail(WF_EINVAL, "wf_mg_noalloc_status: null status");
  NoallocAddrs ad{};
  WF_TRY(noalloc_addrs(&ad));
  WF_CK(cudaStreamSynchronize((cudaStream_t)stream));
  int v = 0;
  WF_CK(cudaMemcpy(&v, ad.status, sizeof(int), cudaMemcpyDeviceToHost));
  *status = v;
  return WF_OK;
}


// ---------------------------------------------------------------------------
// Sub-domains (the reference's multigrid.py and halo.py at more than one
// rank).  At a seam between ranks the reference keeps the face coefficient
// (multigrid.py:23-67 zeroes it only across a physical face) and refreshes
// the one-cell ring by a halo exchange once per full sweep, after the
// Neumann mirror of the physical faces (multigrid.py:264-299).  These
// kernels do one reference pass each, on a level of a case whose level 0 is
// the core of pp and su (as mg_solve); the ring at the seams is the host's:
//   op 0  one colour half-sweep (multigrid.py:70-90), no ring writes
//   op 1  Neumann mirror of the physical faces' interiors (bcs.py:326-360)
//   op 2  restriction from level-1 to level (multigrid.py:93-119), the
//         coarse phi zeroed, ring included (multigrid.py:310-312)
//   op 3  prolongation from level+1 to level, real cells only (122-146)
//   op 4  pp zeroed over the whole padded array (multigrid.py:332-333)
// `phys` holds one bit per face, set when the face is physical: bit 0 west,
// 1 east, 2 south, 3 north, 4 bottom, 5 top.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double seam_coef(bool edge, int phys, int bit, double a) {
  return (edge && ((phys >> bit) & 1)) ? 0.0 : a;
}

__global__ void __launch_bounds__(MG_TPB) k_rk_rbgs(const Lvl<double> L, int phys, int color) {
  pdl_entry();
  const int n = L.n;
  const int kx = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  const int i = blockIdx.z;
  if (kx >= (n + 1) / 2 || j >= n) return;
  const int k = 2 * kx + ((1 + i + j + color) & 1);
  if (k >= n) return;
  const long c = lid(L, i + 1, j + 1, k + 1);
  const double aw = seam_coef(i == 0, phys, 0, L.ax), ae = seam_coef(i == n - 1, phys, 1, L.ax);
  const double as = seam_coef(j == 0, phys, 2, L.ay), an = seam_coef(j == n - 1, phys, 3, L.ay);
  const double ab = seam_coef(k == 0, phys, 4, L.az), at = seam_coef(k == n - 1, phys, 5, L.az);
  const double ap = -(aw + ae + as + an + ab + at);
  const double* p = L.phi;
  const double s = aw * p[c - L.sI] + ae * p[c + L.sI] + as * p[c - L.sJ] + an * p[c + L.sJ] +
                   ab * p[c - 1] + at * p[c + 1];
  L.phi[c] = (L.rhs[c] - s) / ap;
}

__global__ void k_rk_mirror(const Lvl<double> L, int phys) {
  pdl_entry();
  const int n = L.n;
  const long tot = (long)n * n;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot;
       t += (long)gridDim.x * blockDim.x) {
    const int a = 1 + (int)(t / n), b = 1 + (int)(t % n);
    double* p = L.phi;
    if (phys & 1) p[lid(L, 0, a, b)] = p[lid(L, 1, a, b)];
    if (phys & 2) p[lid(L, n + 1, a, b)] = p[lid(L, n, a, b)];
    if (phys & 4) p[lid(L, a, 0, b)] = p[lid(L, a, 1, b)];
    if (phys & 8) p[lid(L, a, n + 1, b)] = p[lid(L, a, n, b)];
    if (phys & 16) p[lid(L, a, b, 0)] = p[lid(L, a, b, 1)];
    if (phys & 32) p[lid(L, a, b, n + 1)] = p[lid(L, a, b, n)];
  }
}

__global__ void __launch_bounds__(MG_TPB) k_rk_restrict(const Lvl<double> F, Lvl<double> C,
                                                        int phys) {
  pdl_entry();
  const int nc = C.n, n = F.n;
  const int ck = blockIdx.x * 32 + threadIdx.x, cj = blockIdx.y * 8 + threadIdx.y;
  const int ci = blockIdx.z;
  if (ck >= nc || cj >= nc) return;
  const double* p = F.phi;
  double acc = 0.0;
  for (int di = 0; di < 2; ++di)
    for (int dj = 0; dj < 2; ++dj)
      for (int dk = 0; dk < 2; ++dk) {
        const int i = 2 * ci + di, j = 2 * cj + dj, k = 2 * ck + dk;
        const long c = lid(F, i + 1, j + 1, k + 1);
        const double aw = seam_coef(i == 0, phys, 0, F.ax), ae = seam_coef(i == n - 1, phys, 1, F.ax);
        const double as = seam_coef(j == 0, phys, 2, F.ay), an = seam_coef(j == n - 1, phys, 3, F.ay);
        const double ab = seam_coef(k == 0, phys, 4, F.az), at = seam_coef(k == n - 1, phys, 5, F.az);
        const double ap = -(aw + ae + as + an + ab + at);
        const double res = F.rhs[c] - (aw * p[c - F.sI] + ae * p[c + F.sI] + as * p[c - F.sJ] +
                                       an * p[c + F.sJ] + ab * p[c - 1] + at * p[c + 1] +
                                       ap * p[c]);
        acc = acc + res;
      }
  const_cast<double*>(C.rhs)[lid(C, ci + 1, cj + 1, ck + 1)] = acc * 0.125;
  // every cell of the (nc+2)^3 coarse phi zeroed once: this cell and the
  // ring cells nearest to it
  const int zi0 = ci == 0 ? -1 : 0, zi1 = ci == nc - 1 ? 1 : 0;
  const int zj0 = cj == 0 ? -1 : 0, zj1 = cj == nc - 1 ? 1 : 0;
  const int zk0 = ck == 0 ? -1 : 0, zk1 = ck == nc - 1 ? 1 : 0;
  for (int oi = zi0; oi <= zi1; ++oi)
    for (int oj = zj0; oj <= zj1; ++oj)
      for (int ok = zk0; ok <= zk1; ++ok)
        C.phi[lid(C, ci + 1 + oi, cj + 1 + oj, ck + 1 + ok)] = 0.0;
}

__global__ void __launch_bounds__(MG_TPB) k_rk_prolong(const Lvl<double> C, Lvl<double> F) {
  pdl_entry();
  const int n = F.n;
  const int k = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= n || j >= n) return;
  const int c0x = (i % 2 == 0) ? i / 2 - 1 : i / 2;
  const double wx0 = (i % 2 == 0) ? 0.25 : 0.75;
  const int c0y = (j % 2 == 0) ? j / 2 - 1 : j / 2;
  const double wy0 = (j % 2 == 0) ? 0.25 : 0.75;
  const int c0z = (k % 2 == 0) ? k / 2 - 1 : k / 2;
  const double wz0 = (k % 2 == 0) ? 0.25 : 0.75;
  double acc = 0.0;
  for (int di = 0; di < 2; ++di) {
    const double wxi = di == 0 ? wx0 : 1.0 - wx0;
    for (int dj = 0; dj < 2; ++dj) {
      const double wyj = dj == 0 ? wy0 : 1.0 - wy0;
      for (int dk = 0; dk < 2; ++dk) {
        const double wzk = dk == 0 ? wz0 : 1.0 - wz0;
        acc = acc + wxi * wyj * wzk * C.phi[lid(C, c0x + di + 1, c0y + dj + 1, c0z + dk + 1)];
      }
    }
  }
  const long c = lid(F, i + 1, j + 1, k + 1);
  F.phi[c] = F.phi[c] + acc;
}

// the levels of a case, level 0 the one-ring core of pp (phi) and su (rhs)
static int rank_levels(const wf_case& c, std::vector<Lvl<double>>& lv) {
  const long P = padded(c.n);
  const long off = (long)(NPL - 1) * (P * P + P + 1);
  WF_TRY(build_levels<double>(c, c.fld[WF_PP] + off, c.fld[WF_SU] + off, P * P, P, lv));
  for (auto& L : lv) {
    L.tmp = nullptr;
    L.split = 0;
  }
  return WF_OK;
}

int rk_mg_op(const wf_case& c, int op, int level, int phys, int color, cudaStream_t s) {
  if (c.mg_fp32) return fail(WF_EUNSUPPORTED, "sub-domain multigrid runs in FP64");
  if (!c.fld[WF_PP] || !c.fld[WF_SU]) return fail(WF_EINVAL, "null pp or su");
  if (phys < 0 || phys > 63) return fail(WF_EINVAL, "face mask out of range");
  std::vector<Lvl<double>> lv;
  WF_TRY(rank_levels(c, lv));
  const int L = (int)lv.size();
  if (level < 0 || level >= L) return fail(WF_EINVAL, "level out of range");
  const Lvl<double>& V = lv[level];
  switch (op) {
    case 0:
      if (color != 0 && color != 1) return fail(WF_EINVAL, "colour must be 0 or 1");
      WF_CK(launch_k(k_rk_rbgs, cells3(V.n, V.n, (V.n + 1) / 2), cell_block(), 0, s, V, phys,
                     color));
      WF_CKL("k_rk_rbgs");
      return WF_OK;
    case 1:
      WF_CK(launch_k(k_rk_mirror, mg_blocks((long)V.n * V.n), MG_TPB, 0, s, V, phys));
      WF_CKL("k_rk_mirror");
      return WF_OK;
    case 2:
      if (level < 1) return fail(WF_EINVAL, "restriction needs level >= 1");
      WF_CK(launch_k(k_rk_restrict, cells3(V.n, V.n, V.n), cell_block(), 0, s, lv[level - 1],
                     V, phys));
      WF_CKL("k_rk_restrict");
      return WF_OK;
    case 3:
      if (level > L - 2) return fail(WF_EINVAL, "prolongation needs a coarser level");
      WF_CK(launch_k(k_rk_prolong, cells3(V.n, V.n, V.n), cell_block(), 0, s, lv[level + 1], V));
      WF_CKL("k_rk_prolong");
      return WF_OK;
    case 4: {
      const long P = padded(c.n);
      WF_CK(launch_k(k_zero<double>, mg_blocks(P * P * P), MG_TPB, 0, s, c.fld[WF_PP], P * P * P,
                     (int)WF_PP));
      WF_CKL("k_zero pp");
      return WF_OK;
    }
    default:
      return fail(WF_EINVAL, "unknown sub-domain multigrid op");
  }
}

int rk_level_view(const wf_case& c, int level, double** phi, int64_t* sI, int64_t* sJ,
                  int32_t* m) {
  std::vector<Lvl<double>> lv;
  WF_TRY(rank_levels(c, lv));
  if (level < 0 || level >= (int)lv.size()) return fail(WF_EINVAL, "level out of range");
  *phi = lv[level].phi;
  *sI = lv[level].sI;
  *sJ = lv[level].sJ;
  *m = lv[level].n + 2;
  return WF_OK;
}

}  // namespace wf
