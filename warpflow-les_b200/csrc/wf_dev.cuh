// Device helpers shared by the libwfb200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "wf_internal.h"

namespace wf {

// Programmatic dependent launch: every kernel of this library starts by
// allowing its successor to begin launching, then waits until its
// predecessor has completed and its memory is visible.  Without the launch
// attribute both instructions are no-ops.
//
// The wait orders a kernel's global loads only if the compiler cannot move
// them above it.  It is an asm statement with a memory clobber, but a load
// through a __restrict__ pointer (or the read-only path, __ldg) may legally
// be hoisted above such a statement -- the asm does not name the pointer --
// and would then read data the predecessor is still writing (this happened
// to a coarse-level kernel whose whole input load was provably in bounds).
// So no kernel of this library marks a global-memory pointer __restrict__
// or loads through __ldg; shared-memory pointers may be restrict.
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// ---- bucket batching (see Batch in wf_internal.h) -------------------------
// the case of this block, its z index within the case's grid, the case's z
// extent; a case's buffers
__device__ __forceinline__ int bt_case(const Batch& b) {
  return b.tab ? (int)(blockIdx.z / (unsigned)b.nz) : 0;
}
__device__ __forceinline__ int bt_z(const Batch& b) {
  return b.tab ? (int)(blockIdx.z % (unsigned)b.nz) : (int)blockIdx.z;
}
__device__ __forceinline__ int bt_gz(const Batch& b) { return b.tab ? b.nz : (int)gridDim.z; }
__device__ __forceinline__ double* bt_fld(const wf_case& c, const Batch& b, int f) {
  return b.tab ? b.tab[bt_case(b)].fld[f] : c.fld[f];
}
__device__ __forceinline__ wf_scalars* bt_sc(const wf_case& c, const Batch& b) {
  return b.tab ? b.tab[bt_case(b)].sc : c.sc;
}
// true when this block's case does not take part in the launch
__device__ __forceinline__ bool bt_skip(const Batch& b) {
  return b.tab && b.skip && !(b.tab[bt_case(b)].sc->loop & b.skip);
}

__device__ __forceinline__ unsigned long long dbits(double x) {
  return (unsigned long long)__double_as_longlong(x);
}
__device__ __forceinline__ double bitsd(unsigned long long b) {
  return __longlong_as_double((long long)b);
}
// order-preserving key: okey(a) < okey(b) as unsigned iff a < b as doubles
// (any sign), so device-wide max/min reductions are integer atomics
__device__ __forceinline__ unsigned long long okey(double x) {
  const unsigned long long b = dbits(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double okey_inv(unsigned long long k) {
  return bitsd((k >> 63) ? (k & 0x7fffffffffffffffull) : ~k);
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// block-wide max / min; every thread gets the result (blockDim <= 1024)
__device__ __forceinline__ double block_max(double v, double* sm) {
  v = warp_max(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (l == 0) sm[w] = v;
  __syncthreads();
  v = (threadIdx.x < nw) ? sm[threadIdx.x] : 0.0;
  if (w == 0) v = warp_max(v);
  if (threadIdx.x == 0) sm[0] = v;
  __syncthreads();
  return sm[0];
}
__device__ __forceinline__ double block_min(double v, double* sm, double ident) {
  v = warp_min(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (l == 0) sm[w] = v;
  __syncthreads();
  v = (threadIdx.x < nw) ? sm[threadIdx.x] : ident;
  if (w == 0) v = warp_min(v);
  if (threadIdx.x == 0) sm[0] = v;
  __syncthreads();
  return sm[0];
}

// "last block done" among `count` blocks: returns true in exactly one block,
// after every other block's preceding global writes are visible; resets the
// ticket.
__device__ __forceinline__ bool last_block(unsigned int* ticket, unsigned count) {
  __shared__ bool is_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == count - 1);
    if (is_last) {
      __threadfence();
      *ticket = 0u;
    }
  }
  __syncthreads();
  return is_last;
}

// x / d, correctly rounded, from y = RN(1/d): one residual correction makes
// the quotient faithful, a second rounds it correctly (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990).  Valid away from overflow and
// underflow, which the solver's values stay far from; four FMAs and a
// multiply in place of a full division.
template <class T>
__device__ __forceinline__ T div_by_recip(T x, T d, T y) {
  T q = x * y;
  T r = fma(-q, d, x);
  q = fma(r, y, q);
  r = fma(-q, d, x);
  return fma(r, y, q);
}

}  // namespace wf
