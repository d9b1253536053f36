// Per-system PCG reductions, shared by the reduction kernel of the solver and the node-slice
// kernels that finish them in their last CTA of each system.
//
// The scalars of a PCG iteration (p.q for alpha; r.z and r.r for beta and the convergence test)
// are sums of partials, one per slice (node-slice kernels) or per row block (row kernels), summed
// per system in a fixed order by one CTA of kRedThreads threads.  The same function produces the
// sums in the separate reduction kernel and in the fused form, so both give the same bits.
#pragma once
#include "ua_internal.h"

namespace ua {

constexpr int kRedThreads = 256;
// per-system scalars; SV_RH = |rhat|^2, SV_RST = BiCGStab restart pending, SV_NRST = restarts so far
enum { SV_RZ = 0, SV_PQ, SV_ALPHA, SV_BETA, SV_RR, SV_RR0, SV_TOL2, SV_NORM, SV_FF, SV_FD, SV_OMEGA, SV_RH, SV_RST,
       SV_NRST, SV_COUNT };

// Sum NV partial arrays of one system in a fixed order (a strided per-thread sum, then a tree
// over the kRedThreads threads).  CG: read through L2 only (partials written by other CTAs of
// the running kernel).
template <int NV, bool CG = false>
__device__ __forceinline__ void sys_sum(const double* part, int nrb, int b0, int b1, double (&out)[NV]) {
  __shared__ double red[NV][kRedThreads];
  double acc[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) acc[j] = 0;
  for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x)
#pragma unroll
    for (int j = 0; j < NV; ++j) acc[j] += CG ? __ldcg(part + j * nrb + b) : part[j * nrb + b];
#pragma unroll
  for (int j = 0; j < NV; ++j) red[j][threadIdx.x] = acc[j];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
#pragma unroll
      for (int j = 0; j < NV; ++j) red[j][threadIdx.x] += red[j][threadIdx.x + st];
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < NV; ++j) out[j] = red[j][0];
}

// alpha = rz / pq, or breakdown (pq not positive: not SPD on the free dofs)
__device__ __forceinline__ void pcg_stage1(int s, double pq, double* sysv, int nsys, int* status, int* done) {
  if (!(pq > 0)) {
    status[s] = 1;
    done[s] = 1;
    sysv[SV_ALPHA * nsys + s] = 0;
  } else {
    sysv[SV_ALPHA * nsys + s] = sysv[SV_RZ * nsys + s] / pq;
  }
}

// beta = rz_new / rz, and the convergence test on r.r
__device__ __forceinline__ void pcg_stage2(int s, double rz_new, double rr, double* sysv, int nsys, int* its,
                                           int* done, int maxit) {
  its[s] += 1;
  sysv[SV_RR * nsys + s] = rr;
  sysv[SV_BETA * nsys + s] = rz_new / sysv[SV_RZ * nsys + s];
  sysv[SV_RZ * nsys + s] = rz_new;
  if (rr <= sysv[SV_TOL2 * nsys + s] * sysv[SV_RR0 * nsys + s] || its[s] >= maxit || !(rr == rr)) done[s] = 1;
}

// The reduction of a PCG stage done by the last CTA of each system inside the node-slice kernel
// that writes its partials (stage 1 after the SpMV's p.q, stage 2 after the smoothing's r.z);
// stage 0 = off (the separate reduction kernel runs instead).
struct PcgFuse {
  int stage = 0;
  int* cnt = nullptr;              // per system: slice blocks finished in this launch
  const int* sys_sl_off = nullptr; // per-system slice prefix (spart)
  const double* rb_part = nullptr; // row-block partials (r.r in its second array)
  int nrb = 0;
  const int* sys_rb_off = nullptr;
  const int* sel = nullptr;
  int* done = nullptr;
  int* status = nullptr;
  int* its = nullptr;
  double* sysv = nullptr;
  int nsys = 0;
  int maxit = 0;
};

// Called by every thread of a CTA after the CTA wrote the slice partials of slice block sb of
// system s (spart).  The CTA that finishes a system's last slice block sums its partials and
// applies the stage; the count is reset for the next launch.  Visibility: each CTA makes its
// partials visible (__threadfence) before counting; the last one reads them through L2.
__device__ __forceinline__ void pcg_fused_tail(const PcgFuse& f, int s, int slices_per_block, const double* spart) {
  __shared__ int s_last;
  __syncthreads();  // the CTA's partials are written
  if (threadIdx.x == 0) {
    __threadfence();
    const int nb = (f.sys_sl_off[s + 1] - f.sys_sl_off[s]) / slices_per_block;
    const int old = atomicAdd(f.cnt + s, 1);
    s_last = old == nb - 1;
    if (s_last) f.cnt[s] = 0;
  }
  __syncthreads();
  if (!s_last) return;  // uniform over the CTA
  __threadfence();
  if (!f.sel[s] || f.done[s]) return;
  const int l0 = f.sys_sl_off[s], l1 = f.sys_sl_off[s + 1];
  if (f.stage == 1) {
    double o[1];
    sys_sum<1, true>(spart, 0, l0, l1, o);
    if (threadIdx.x == 0) pcg_stage1(s, o[0], f.sysv, f.nsys, f.status, f.done);
  } else {
    double a[1], b[1];
    sys_sum<1, true>(spart, 0, l0, l1, a);
    __syncthreads();  // sys_sum's shared array is rewritten by the next call
    sys_sum<1, true>(f.rb_part + f.nrb, 0, f.sys_rb_off[s], f.sys_rb_off[s + 1], b);
    if (threadIdx.x == 0) pcg_stage2(s, a[0], b[0], f.sysv, f.nsys, f.its, f.done, f.maxit);
  }
  __syncthreads();  // the shared sums are rewritten by a later slice block of this CTA
}

}  // namespace ua
