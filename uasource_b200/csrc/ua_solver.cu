// uv Newton-Raphson solve on the device: SSTREAM2dNR2.m:3-431 with the inner
// linear solve of ABfgPreEliminate.m replaced by a constrained, Jacobi-
// preconditioned conjugate-gradient solve, and the cost function of
// CalcCostFunctionNR.m:14-47 fused into residual-only assembly launches.
//
// All kernels work on every system of a handle at once (batched form):
// per-system scalars live in small device arrays and a per-system selection
// flag masks systems that have converged or are not part of the current
// stage.  Reductions are deterministic: each CTA writes one partial sum and a
// one-CTA-per-system kernel adds the partials in a fixed order, so a
// system's result does not depend on which other systems share the launch.
#include <algorithm>
#include <array>
#include <iterator>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include "ua_internal.h"
#include "ua_kernels.h"
#include <type_traits>
#include "ua_linesearch.h"
#include "ua_amg.h"

namespace ua {

constexpr int kRB = 256;        // rows per row block (one CTA)

// Calls f(std::integral_constant<int, LPR>) for the lanes-per-row value lpr (1, 2, 4, 8, 16 or 32).
template <class F>
static void dispatch_lpr(int lpr, F&& f) {
  switch (lpr) {
    case 1: f(std::integral_constant<int, 1>()); break;
    case 2: f(std::integral_constant<int, 2>()); break;
    case 4: f(std::integral_constant<int, 4>()); break;
    case 16: f(std::integral_constant<int, 16>()); break;
    case 32: f(std::integral_constant<int, 32>()); break;
    default: f(std::integral_constant<int, 8>());
  }
}

// Kernel launches issued by the library on the calling thread (reported per call).
static thread_local long long g_launches = 0;

// Optional per-launch timing with CUDA events recorded on the handle's stream.
struct Prof {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;  // (kind, (start, stop))
  cudaEvent_t get() {
    if (used == pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[used++];
  }
  void reset() { used = 0; marks.clear(); }
  ~Prof() { for (auto e : pool) cudaEventDestroy(e); }
  // per mark: tangent non-zeros and rows of the systems the timed launch works on
  long long* d_act = nullptr;
  int act_cap = 0;
};
enum { PK_ASMK = 0, PK_ASMR = 1, PK_SPMV = 2, PK_AMGR = 3, PK_AMGP = 4, PK_SETUP = 5, PK_KRYLOV = 6, PK_COUNT = 7 };
constexpr int PK_WORK = 5;  // classes with work counts (ua_newton_report.kwork_*)
constexpr int kRedThreads = 256;
// per-system scalars; SV_RH = |rhat|^2, SV_RST = BiCGStab restart pending, SV_NRST = restarts so far
enum { SV_RZ = 0, SV_PQ, SV_ALPHA, SV_BETA, SV_RR, SV_RR0, SV_TOL2, SV_NORM, SV_FF, SV_FD, SV_OMEGA, SV_RH, SV_RST,
       SV_NRST, SV_COUNT };
constexpr int kBicgMaxRestarts = 64;

struct Work {
  int nsys = 0, nrb = 0, nc = 0;
  int prec = -1;
  // dof CSR
  int *rowptr = nullptr, *colind = nullptr, *diagpos = nullptr;
  int *rb_start = nullptr, *rb_sys = nullptr, *sys_rb_off = nullptr;
  // nodal fields
  double *h, *s, *S, *B, *rho, *A, *n, *C, *m;
  SysScal* scal;
  // sliding-law and melange fields (q, muk, V0, uo, vo, Co, mo, ua, va, Ca, ma): buffers allocated
  // on first use, dragf[k] = dragbuf[k] while the configured law reads field k, else null
  double* dragbuf[11] = {};
  const double* dragf[11] = {};
  // adjoint gradient work (mass matrix values, measurements, misfit and CG vectors)
  double* adj_buf = nullptr;
  size_t adj_cap = 0;
  // two-entry constraint rows (ties, normal velocities): second dof and the scaled coefficients of
  // every row (dof2 = -1 for one-entry rows), the list of two-entry rows and its length
  int* con_dof2 = nullptr;
  double *con_v1 = nullptr, *con_v2 = nullptr;
  int* pair_rows = nullptr;
  std::vector<int> h_sel;  // host copy of sel (set_sel)
  int npair = 0;
  size_t pair_cap = 0;
  // dof vectors
  double *X, *X0, *dX, *R, *frhs, *Tint, *Fext;
  double* Kd = nullptr;
  float* Kf = nullptr;
  // Krylov (VT = double or float, allocated as double-sized)
  void *kr, *kz, *kp, *kq, *invd;
  void* kx0 = nullptr;   // AMG: pre-smoothed fine vector
  double* part;    // [4][nrb]
  double* sysv;    // [SV_COUNT][nsys]
  int* done;       // [nsys]
  int* its;        // [nsys]
  int* status;     // [nsys] 0 ok, 1 breakdown
  int* sel;        // [nsys]
  double* gamma;   // [nsys]
  unsigned char* cmask;  // [ndof]
  int* dof_con;    // [ndof]
  // constraints (mask form: one unit entry per row)
  int* con_dof = nullptr;
  int* con_sys = nullptr;
  int* sys_con_off = nullptr;
  double* con_rhs = nullptr;
  double *lam = nullptr, *dlam = nullptr, *grhs = nullptr;
  // uvh: level-0 state and mass balance (nodal), BiCGStab vectors
  double *h0 = nullptr, *u0 = nullptr, *v0 = nullptr, *as0 = nullptr, *ab0 = nullptr, *as1 = nullptr,
         *ab1 = nullptr, *dadh = nullptr;
  void *krh = nullptr, *ks = nullptr, *ksh = nullptr, *kt = nullptr;
  // uvh GMRES(m): basis, work vectors, per-system coefficients
  double *gm_V = nullptr, *gm_w = nullptr, *gm_z = nullptr, *gm_u = nullptr, *gm_part = nullptr;
  double *gm_hb = nullptr, *gm_ht = nullptr, *gm_hl1 = nullptr;  // thickness-block sweeps: b_h, ping-pong, l1
  double *gm_coef = nullptr, *gm_scal = nullptr;
  int *gm_act = nullptr, *gm_ny = nullptr;
  int gm_m = 0;
  // pinned host staging
  double* h_sysv = nullptr;
  int* h_int = nullptr;
  int* nan_first = nullptr;  // device NaN scan result (9 ints) and its pinned host copy
  int* h_nan = nullptr;
  double* h_gamma = nullptr;
  std::vector<int> h_sys_rb_off, h_sys_con_off;
  Prof prof;
  struct ServeState* serve = nullptr;
  // replayable PCG chunks, index (fp32 ? 2 : 0) + (amg ? 1 : 0) + (BF16 V-cycle ? 4 : 0) + (active lists ? 8 : 0)
  bool no_graph = false;
  cudaGraphExec_t pcg_exec[32] = {};
  long long pcg_exec_nodes[32] = {};
  int pcg_exec_maxit[32] = {};
  int pcg_exec_lpr[32] = {};
  int nsm = 148;  // SMs of the handle's device (grid of the list-driven kernels)
};

// Two-entry constraint rows (ties, normal velocities): the second dof and the scaled coefficients
// of every row; all null when every row has one unit entry (a dof selection).
struct ConPairs {
  const int* dof2;
  const double *v1, *v2;
};

static ConPairs con_pairs(const Work* w) {
  return w->npair ? ConPairs{w->con_dof2, w->con_v1, w->con_v2} : ConPairs{nullptr, nullptr, nullptr};
}

// Work of a timed launch: sum of the tangent non-zeros and dof rows of the
// systems it processes (selected; for Krylov kernels also not yet converged).
__global__ void k_count_active(int nsys, const int* sel, const int* done, const int* knz_off, const int* dof_off,
                               long long* out) {
  __shared__ long long a[256], b[256];
  long long x = 0, y = 0;
  for (int s = threadIdx.x; s < nsys; s += blockDim.x)
    if (sel[s] && !(done && done[s])) {
      x += knz_off[s + 1] - knz_off[s];
      y += dof_off[s + 1] - dof_off[s];
    }
  a[threadIdx.x] = x;
  b[threadIdx.x] = y;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) { a[threadIdx.x] += a[threadIdx.x + st]; b[threadIdx.x] += b[threadIdx.x + st]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { out[0] = a[0]; out[1] = b[0]; }
}

static void prof_begin(ua_mesh* m, int kind, cudaEvent_t* ev) {
  Work* w = m->work;
  if (!w->prof.on) return;
  ev[0] = w->prof.get();
  ev[1] = w->prof.get();
  const int idx = (int)w->prof.marks.size();
  if (!w->prof.d_act) {
    w->prof.act_cap = 1 << 16;
    w->prof.d_act = (long long*)dev_alloc(m, sizeof(long long) * 2 * w->prof.act_cap);
  }
  if (w->prof.d_act && idx < w->prof.act_cap)
    k_count_active<<<1, 256, 0, m->stream>>>(w->nsys, w->sel, kind >= PK_SPMV ? w->done : nullptr,
                                             m->dm.sys_knz_off, m->dm.sys_dof_off, w->prof.d_act + 2 * idx),
        ++g_launches;
  cudaEventRecord(ev[0], m->stream);
  w->prof.marks.push_back({kind, {ev[0], ev[1]}});
}

// Summed launch times, launch counts and work per timed kernel class.
static void prof_collect(Work* w, double* kms, int* kn, double* knnz, double* krows) {
  const int nm = (int)w->prof.marks.size();
  std::vector<long long> act;
  if (w->prof.d_act && nm) {
    act.resize(2 * (size_t)std::min(nm, w->prof.act_cap));
    cudaMemcpy(act.data(), w->prof.d_act, act.size() * sizeof(long long), cudaMemcpyDeviceToHost);
  }
  for (int i = 0; i < nm; ++i) {
    const auto& mk = w->prof.marks[i];
    float t = 0;
    cudaEventElapsedTime(&t, mk.second.first, mk.second.second);
    kms[mk.first] += t;
    kn[mk.first]++;
    if (2 * i + 1 < (int)act.size()) { knnz[mk.first] += (double)act[2 * i]; krows[mk.first] += (double)act[2 * i + 1]; }
  }
}

static void prof_report(ua_newton_report* r, const double* kms, const int* kn, const double* knnz,
                        const double* krows) {
  r->kasmK_ms = kms[PK_ASMK]; r->kasmK_n = kn[PK_ASMK];
  r->kasmR_ms = kms[PK_ASMR]; r->kasmR_n = kn[PK_ASMR];
  r->kspmv_ms = kms[PK_SPMV]; r->kspmv_n = kn[PK_SPMV];
  r->kamgR_ms = kms[PK_AMGR]; r->kamgR_n = kn[PK_AMGR];
  r->kamgP_ms = kms[PK_AMGP]; r->kamgP_n = kn[PK_AMGP];
  r->ksetup_ms = kms[PK_SETUP]; r->ksetup_n = kn[PK_SETUP];
  r->kkrylov_ms = kms[PK_KRYLOV]; r->kkrylov_n = kn[PK_KRYLOV];
  for (int k = 0; k < PK_WORK; ++k) { r->kwork_nnz[k] = knnz[k]; r->kwork_rows[k] = krows[k]; }
}

static void prof_end(ua_mesh* m, cudaEvent_t* ev) {
  if (!m->work->prof.on) return;
  cudaEventRecord(ev[1], m->stream);
}
// timing hook of the fine-level AMG launches (kind: 0 restriction, 1 prolongation)
static void prof_amg(void* ctx, int kind, int phase) {
  static thread_local cudaEvent_t ev[2];
  ua_mesh* m = (ua_mesh*)ctx;
  if (phase == 0) prof_begin(m, kind == 0 ? PK_AMGR : PK_AMGP, ev);
  else prof_end(m, ev);
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// Dof-level CSR rows of node g (all ndof components).
__global__ void k_dof_csr(DevMesh M, int* rowptr, int* colind, int* diagpos) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= M.nn) return;
  const int s = M.node_sys[g];
  const int no = M.sys_node_off[s], nn_s = M.sys_node_off[s + 1] - no;
  const int doff = M.sys_dof_off[s];
  const int np0 = M.nodeptr[g], deg = M.nodeptr[g + 1] - np0;
  const int lp = np0 - M.nodeptr[no];
  const int nd = M.ndof;
  int kd = 0;
  for (int k = 0; k < deg; ++k)
    if (M.nodecol[np0 + k] == g) kd = k;
  for (int c = 0; c < nd; ++c) {
    const int dof = doff + c * nn_s + (g - no);
    const int start = M.sys_knz_off[s] + c * nd * M.sys_nnzn[s] + nd * lp;
    rowptr[dof] = start;
    diagpos[dof] = start + c * deg + kd;
    for (int b = 0; b < nd; ++b)
      for (int k = 0; k < deg; ++k) colind[start + b * deg + k] = doff + b * nn_s + (M.nodecol[np0 + k] - no);
  }
}

// Calc_bs_From_hBS.m:71-79,109 (nodal flotation mask, b and s).
__global__ void k_calc_bs(int nn, const int* node_sys, const SysScal* scal, double kH, double Hh0, const double* h,
                          const double* S, const double* B, const double* rho, double* s) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nn) return;
  const double rhow = scal[node_sys[g]].rhow;
  const double hf = rhow * (S[g] - B[g]) / rho[g];
  const double GF = heaviside_approx(kH, h[g] - hf, Hh0);
  const double bfloat = S[g] - rho[g] * h[g] / rhow;
  const double b = GF * B[g] + (1 - GF) * bfloat;
  s[g] = b + h[g];
}

// per-system flag n = m = 3 at every node (the assembly then takes reciprocal cube roots for the
// powers): set, then cleared by any node with another exponent (every writer stores the same value)
__global__ void k_cube_set(int nsys, SysScal* scal) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nsys) scal[s].cube = 1.0;
}
__global__ void k_cube_check(int nn, const int* node_sys, const double* n, const double* m, SysScal* scal) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < nn && (n[g] != 3.0 || m[g] != 3.0)) scal[node_sys[g]].cube = 0.0;
}

template <typename KT, typename VT>
__global__ void k_invdiag(int n, const KT* K, const int* diagpos, const unsigned char* cmask, VT* invd) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double d = (double)K[diagpos[i]];
  invd[i] = (VT)((cmask[i] || d == 0.0) ? 0.0 : 1.0 / d);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block reduction of up to 4 values; thread 0 writes part[j*nrb + blk].
template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], double* part, int nrb, int blk) {
  __shared__ double red[NV][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double t = warp_sum(v[j]);
    if (lane == 0) red[j][w] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double t = 0;
      for (int i = 0; i < nw; ++i) t += red[j][i];
      part[j * nrb + blk] = t;
    }
  }
  __syncthreads();  // red is rewritten by the next row block of a list-driven launch
}

// Row-block SpMV with LPR lanes per row: y = mask(K x) (or mask(f - K x) in init mode).
template <typename KT, typename XT, int LPR>
__device__ __forceinline__ double row_dot(const int* rowptr, const int* colind, const KT* K, const XT* x, int row,
                                          bool valid, int lane) {
  // every lane of the warp reaches the shuffles; `valid` masks rows past the block end
  double acc = 0;
  if (valid) {
    const int r0 = rowptr[row], r1 = rowptr[row + 1];
    for (int j = r0 + lane; j < r1; j += LPR) acc += (double)K[j] * (double)x[colind[j]];
  }
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, LPR);
  return acc;
}

// Row product in the uv block layout: row (c, g) holds the u block then the v
// block of deg(g) entries with the same node columns, v columns = u columns +
// nhalf (the system's node count), so only the u block's column indices are
// read: 6 bytes per FP32 non-zero instead of 8.
template <typename KT, typename XT, int LPR>
__device__ __forceinline__ double row_dot_uv(const int* rowptr, const int* colind, const KT* K, const XT* x, int row,
                                             bool valid, int lane, int nhalf) {
  double acc = 0;
  if (valid) {
    const int r0 = rowptr[row], deg = (rowptr[row + 1] - r0) >> 1;
    for (int k = lane; k < deg; k += LPR) {
      const int j = colind[r0 + k];
      acc += (double)K[r0 + k] * (double)x[j] + (double)K[r0 + deg + k] * (double)x[j + nhalf];
    }
  }
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, LPR);
  return acc;
}

// PCG initial residual: r = mask(f - K x0), z = invd r, p = z; partials rz, rr.
// UV: the uv block layout (row_dot_uv, dof_off = per-system dof offsets); else plain CSR.
template <typename KT, typename VT, int LPR, bool UV>
__global__ void __launch_bounds__(256) k_pcg_init(const int* rb_start, const int* rb_sys, int nrb, const int* sel,
                                                  const int* rowptr, const int* colind, const KT* K,
                                                  const double* x0, const double* f, const unsigned char* cmask,
                                                  const VT* invd, VT* r, VT* z, VT* p, double* part,
                                                  const int* dof_off) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  double v[2] = {0, 0};
  if (sel[s]) {
    const int rs = rb_start[blk], re = rb_start[blk + 1];
    const int nhalf = UV ? (dof_off[s + 1] - dof_off[s]) >> 1 : 0;
    const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR, ngrp = blockDim.x / LPR;
    for (int row0 = rs; row0 < re; row0 += ngrp) {  // same trip count for every thread
      const int row = row0 + grp;
      const bool valid = row < re;
      double ax = UV ? row_dot_uv<KT, double, LPR>(rowptr, colind, K, x0, row, valid, lane, nhalf)
                     : row_dot<KT, double, LPR>(rowptr, colind, K, x0, row, valid, lane);
      if (valid && lane == 0) {
        double rv = cmask[row] ? 0.0 : f[row] - ax;
        VT rr = (VT)rv;
        VT zz = (VT)((double)invd[row] * (double)rr);
        r[row] = rr; z[row] = zz; p[row] = zz;
        v[0] += (double)rr * (double)zz;
        v[1] += (double)rr * (double)rr;
      }
    }
  }
  block_partials<2>(v, part, nrb, blk);
}

// q = mask(K p); partial p.q
// (list-driven when act.cnt is set: the CTAs loop over the active row blocks)
template <typename KT, typename VT, int LPR, bool UV>
__global__ void __launch_bounds__(256) k_pcg_spmv(const int* rb_start, const int* rb_sys, int nrb, ActList act,
                                                  const int* sel, const int* done, const int* rowptr,
                                                  const int* colind, const KT* K, const VT* p,
                                                  const unsigned char* cmask, VT* q, double* part,
                                                  const int* dof_off) {
  const int nv = act.cnt ? *act.cnt : gridDim.x;
  for (int vb = blockIdx.x; vb < nv; vb += gridDim.x) {
    const int blk = act.map ? act.map[vb] : vb;
    const int s = rb_sys[blk];
    double v[1] = {0};
    if (sel[s] && !done[s]) {
      const int rs = rb_start[blk], re = rb_start[blk + 1];
      const int nhalf = UV ? (dof_off[s + 1] - dof_off[s]) >> 1 : 0;
      const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR, ngrp = blockDim.x / LPR;
      for (int row0 = rs; row0 < re; row0 += ngrp) {  // same trip count for every thread
        const int row = row0 + grp;
        const bool valid = row < re;
        double ax = UV ? row_dot_uv<KT, VT, LPR>(rowptr, colind, K, p, row, valid, lane, nhalf)
                       : row_dot<KT, VT, LPR>(rowptr, colind, K, p, row, valid, lane);
        if (valid && lane == 0) {
          double qv = cmask[row] ? 0.0 : ax;
          q[row] = (VT)qv;
          v[0] += (double)p[row] * qv;
        }
      }
    }
    block_partials<1>(v, part, nrb, blk);
  }
}

// x += alpha p; r -= alpha q; z = invd r; partials rz, rr
template <typename VT>
__global__ void __launch_bounds__(256) k_pcg_update1(const int* rb_start, const int* rb_sys, int nrb, ActList act,
                                                     const int* sel, const int* done, const double* sysv,
                                                     int nsys, double* x, VT* r, VT* z, const VT* p, const VT* q,
                                                     const VT* invd, double* part) {
  pdl_enter();
  const int nv = act.cnt ? *act.cnt : gridDim.x;
  for (int vb = blockIdx.x; vb < nv; vb += gridDim.x) {
    const int blk = act.map ? act.map[vb] : vb;
    const int s = rb_sys[blk];
    double v[2] = {0, 0};
    if (sel[s] && !done[s]) {
      const double alpha = sysv[SV_ALPHA * nsys + s];
      const int rs = rb_start[blk], re = rb_start[blk + 1];
      for (int i = rs + threadIdx.x; i < re; i += blockDim.x) {
        x[i] += alpha * (double)p[i];
        VT rr = (VT)((double)r[i] - alpha * (double)q[i]);
        VT zz = (VT)((double)invd[i] * (double)rr);
        r[i] = rr; z[i] = zz;
        v[0] += (double)rr * (double)zz;
        v[1] += (double)rr * (double)rr;
      }
    }
    block_partials<2>(v, part, nrb, blk);
  }
}

template <typename VT>
__global__ void __launch_bounds__(256) k_pcg_update2(const int* rb_start, const int* rb_sys, ActList act,
                                                     const int* sel, const int* done, const double* sysv, int nsys,
                                                     VT* p, const VT* z) {
  pdl_enter();
  const int nv = act.cnt ? *act.cnt : gridDim.x;
  for (int vb = blockIdx.x; vb < nv; vb += gridDim.x) {
    const int blk = act.map ? act.map[vb] : vb;
    const int s = rb_sys[blk];
    if (!sel[s] || done[s]) continue;  // uniform over the block
    const double beta = sysv[SV_BETA * nsys + s];
    const int rs = rb_start[blk], re = rb_start[blk + 1];
    for (int i = rs + threadIdx.x; i < re; i += blockDim.x) p[i] = (VT)((double)z[i] + beta * (double)p[i]);
  }
}

// Sum NV partial arrays of one system in a fixed order.
template <int NV>
__device__ __forceinline__ void sys_sum(const double* part, int nrb, int b0, int b1, double (&out)[NV]) {
  __shared__ double red[NV][kRedThreads];
  double acc[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) acc[j] = 0;
  for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x)
#pragma unroll
    for (int j = 0; j < NV; ++j) acc[j] += part[j * nrb + b];
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

// stage: 0 = init (rz, rr0), 1 = alpha (pq), 2 = beta (rz_new, rr)
// spart (node slices): the p.q and r.z partials come per slice (sys_sl_off: per-system slice
// prefix) instead of from part's first array; r.r stays in part's second array.
__global__ void k_pcg_reduce(int stage, const int* sys_rb_off, int nrb, const int* sel, int* done, int* its,
                             int* status, double* sysv, int nsys, const double* part, int maxit,
                             const double* spart = nullptr, const int* sys_sl_off = nullptr) {
  pdl_enter();
  const int s = blockIdx.x;
  if (!sel[s] || (stage > 0 && done[s])) return;
  const int b0 = sys_rb_off[s], b1 = sys_rb_off[s + 1];
  if (stage == 1) {
    double o[1];
    if (spart) sys_sum<1>(spart, 0, sys_sl_off[s], sys_sl_off[s + 1], o);
    else sys_sum<1>(part, nrb, b0, b1, o);
    if (threadIdx.x == 0) {
      const double pq = o[0];
      if (!(pq > 0)) {  // not positive definite on the free dofs, or breakdown
        status[s] = 1;
        done[s] = 1;
        sysv[SV_ALPHA * nsys + s] = 0;
      } else {
        sysv[SV_ALPHA * nsys + s] = sysv[SV_RZ * nsys + s] / pq;
      }
    }
    return;
  }
  double o[2];
  if (spart) {
    double a[1], b[1];
    sys_sum<1>(spart, 0, sys_sl_off[s], sys_sl_off[s + 1], a);
    __syncthreads();  // sys_sum's shared array is rewritten by the next call
    sys_sum<1>(part + nrb, 0, b0, b1, b);
    o[0] = a[0];
    o[1] = b[0];
  } else {
    sys_sum<2>(part, nrb, b0, b1, o);
  }
  if (threadIdx.x != 0) return;
  if (stage == 0) {
    sysv[SV_RZ * nsys + s] = o[0];
    sysv[SV_RR0 * nsys + s] = o[1];
    sysv[SV_RR * nsys + s] = o[1];
    its[s] = 0;
    status[s] = 0;
    done[s] = (o[1] == 0.0) ? 1 : 0;
    return;
  }
  const double rz_new = o[0], rr = o[1];
  its[s] += 1;
  sysv[SV_RR * nsys + s] = rr;
  sysv[SV_BETA * nsys + s] = rz_new / sysv[SV_RZ * nsys + s];
  sysv[SV_RZ * nsys + s] = rz_new;
  if (rr <= sysv[SV_TOL2 * nsys + s] * sysv[SV_RR0 * nsys + s] || its[s] >= maxit || !(rr == rr)) done[s] = 1;
}

// Constraint rows of the Newton system (mask form):
// dX[dof_c] = grhs_c = c_c - X[dof_c] (particular solution x_p = L' g).
__device__ __forceinline__ bool con_is_pair(const ConPairs& cp, int c) { return cp.dof2 && cp.dof2[c] >= 0; }
// coefficient of row c at dof i (1 for a one-entry row)
__device__ __forceinline__ double con_coef(const ConPairs& cp, const int* con_dof, int c, int i) {
  if (!con_is_pair(cp, c)) return 1.0;
  return con_dof[c] == i ? cp.v1[c] : cp.v2[c];
}

// Particular solution of B dX = g - B X (ABfgPreEliminate.m:63 with unit rows): a one-entry row
// sets its dof, a two-entry row b puts b (g - b'X) on its pair.
__global__ void k_con_particular(int nc, const int* con_dof, const int* con_sys, const int* sel,
                                 const double* con_rhs, const double* X, double* dX, double* grhs, ConPairs cp) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc || !sel[con_sys[c]]) return;
  const int d = con_dof[c];
  if (con_is_pair(cp, c)) {
    const int d2 = cp.dof2[c];
    const double t = con_rhs[c] - (cp.v1[c] * X[d] + cp.v2[c] * X[d2]);
    grhs[c] = t;
    dX[d] = cp.v1[c] * t;
    dX[d2] = cp.v2[c] * t;
    return;
  }
  const double gv = con_rhs[c] - X[d];
  grhs[c] = gv;
  dX[d] = gv;
}

// z <- (I - b b') z on the two-entry rows (their dofs are free; rows have disjoint support).
template <typename VT>
__global__ void k_pair_project(int npair, const int* pair_rows, const int* con_dof, const int* con_sys,
                               const int* sel, const int* done, ConPairs cp, VT* z) {
  pdl_enter();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npair) return;
  const int c = pair_rows[k];
  const int s = con_sys[c];
  if (!sel[s] || (done && done[s])) return;
  const int a = con_dof[c], b = cp.dof2[c];
  const double t = cp.v1[c] * (double)z[a] + cp.v2[c] * (double)z[b];
  z[a] = (VT)((double)z[a] - cp.v1[c] * t);
  z[b] = (VT)((double)z[b] - cp.v2[c] * t);
}

// The first residual projected, and the l1-Jacobi pre-smoothed vector of the V-cycle refreshed on
// the projected entries (x0 = D^-1 r is diagonal).
template <typename VT>
__global__ void k_pair_project_r0(int npair, const int* pair_rows, const int* con_dof, const int* con_sys,
                                  const int* sel, ConPairs cp, VT* r, VT* x0, const VT* invd) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npair) return;
  const int c = pair_rows[k];
  if (!sel[con_sys[c]]) return;
  const int a = con_dof[c], b = cp.dof2[c];
  const double t = cp.v1[c] * (double)r[a] + cp.v2[c] * (double)r[b];
  r[a] = (VT)((double)r[a] - cp.v1[c] * t);
  r[b] = (VT)((double)r[b] - cp.v2[c] * t);
  if (x0) {
    x0[a] = (VT)((double)invd[a] * (double)r[a]);
    x0[b] = (VT)((double)invd[b] * (double)r[b]);
  }
}

// dl_c = (frhs - K dX)[dof_c]  (ABfgPreEliminate.m:138 with B a selection)
template <typename KT>
__global__ void k_con_multiplier(int nc, const int* con_dof, const int* con_sys, const int* sel, const int* rowptr,
                                 const int* colind, const KT* K, const double* dX, const double* frhs,
                                 double* dlam, ConPairs cp) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc || !sel[con_sys[c]]) return;
  auto row_res = [&](int d) {
    double acc = 0;
    for (int j = rowptr[d]; j < rowptr[d + 1]; ++j) acc += (double)K[j] * dX[colind[j]];
    return frhs[d] - acc;
  };
  const int d = con_dof[c];
  if (con_is_pair(cp, c)) {  // y = b'(f - K x) (ABfgPreEliminate.m:138)
    dlam[c] = cp.v1[c] * row_res(d) + cp.v2[c] * row_res(cp.dof2[c]);
    return;
  }
  dlam[c] = row_res(d);
}

// frhs = -R - L' l  (SSTREAM2dNR2.m:235)
__global__ void k_frhs(const int* rb_start, const int* rb_sys, const int* sel, const double* R, const int* dof_con,
                       const double* lam, double* frhs, const int* con_dof, ConPairs cp) {
  const int blk = blockIdx.x;
  if (!sel[rb_sys[blk]]) return;
  for (int i = rb_start[blk] + threadIdx.x; i < rb_start[blk + 1]; i += blockDim.x) {
    const int c = dof_con[i];
    frhs[i] = -R[i] - (c >= 0 ? con_coef(cp, con_dof, c, i) * lam[c] : 0.0);
  }
}

// Cost function rows (CalcCostFunctionNR.m:24-41): f = -R - L'(l + gamma dl);
// partials sum f^2 and sum f.dX
__global__ void __launch_bounds__(256) k_cost_rows(const int* rb_start, const int* rb_sys, int nrb, const int* sel,
                                                   const double* R, const int* dof_con, const double* lam,
                                                   const double* dlam, const double* gamma, const double* dX,
                                                   double* part, const int* con_dof, ConPairs cp) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  double v[2] = {0, 0};
  if (sel[s]) {
    const double gm = gamma ? gamma[s] : 0.0;
    for (int i = rb_start[blk] + threadIdx.x; i < rb_start[blk + 1]; i += blockDim.x) {
      const int c = dof_con ? dof_con[i] : -1;
      double f = -R[i];
      if (c >= 0) f -= con_coef(cp, con_dof, c, i) * (lam[c] + gm * dlam[c]);
      v[0] += f * f;
      if (dX) v[1] += f * dX[i];
    }
  }
  block_partials<2>(v, part, nrb, blk);
}

// Per-system cost: adds the constraint rows g = c - L(X + gamma dX), then
// rForce = (f'f + g'g)/Normalisation and D2 = [f;g]'[dX;dl].
__global__ void k_cost_reduce(const int* sys_rb_off, int nrb, const int* sel, const double* part, int nsys,
                              double* sysv, const int* sys_con_off, const int* con_dof, const double* con_rhs,
                              const double* X, const double* dX, const double* dlam, const double* gamma,
                              int write_norm, ConPairs cp) {
  const int s = blockIdx.x;
  if (!sel[s]) return;
  double o[2];
  sys_sum<2>(part, nrb, sys_rb_off[s], sys_rb_off[s + 1], o);
  // constraint rows, strided over the block, then a fixed-order tree sum
  __shared__ double cg[2][kRedThreads];
  double gg = 0, gd = 0;
  if (sys_con_off) {
    const double gm = gamma ? gamma[s] : 0.0;
    for (int c = sys_con_off[s] + threadIdx.x; c < sys_con_off[s + 1]; c += blockDim.x) {
      const int d = con_dof[c];
      double xv = X[d] + (dX ? gm * dX[d] : 0.0);
      if (con_is_pair(cp, c)) {  // g = c - L X on a two-entry row
        const int d2 = cp.dof2[c];
        xv = cp.v1[c] * xv + cp.v2[c] * (X[d2] + (dX ? gm * dX[d2] : 0.0));
      }
      const double gv = con_rhs[c] - xv;
      gg += gv * gv;
      if (dlam) gd += gv * dlam[c];
    }
  }
  cg[0][threadIdx.x] = gg;
  cg[1][threadIdx.x] = gd;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      cg[0][threadIdx.x] += cg[0][threadIdx.x + st];
      cg[1][threadIdx.x] += cg[1][threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  gg = cg[0][0];
  gd = cg[1][0];
  if (write_norm) {
    sysv[SV_NORM * nsys + s] = o[0] + 1000.0 * 2.220446049250313e-16;  // fext0'fext0+1000*eps
    return;
  }
  sysv[SV_FF * nsys + s] = (o[0] + gg) / sysv[SV_NORM * nsys + s];
  sysv[SV_FD * nsys + s] = o[1] + gd;
}

// X += gamma dX, l += gamma dl for selected systems.
__global__ void k_newton_update(const int* rb_start, const int* rb_sys, const int* sel, const double* gamma,
                                double* X, const double* dX) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s]) return;
  const double gm = gamma[s];
  for (int i = rb_start[blk] + threadIdx.x; i < rb_start[blk + 1]; i += blockDim.x) X[i] += gm * dX[i];
}

__global__ void k_lam_update(int nc, const int* con_sys, const int* sel, const double* gamma, double* lam,
                             const double* dlam) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc || !sel[con_sys[c]]) return;
  lam[c] += gamma[con_sys[c]] * dlam[c];
}

// Constraint masks: cmask[dof] = 1 and dof_con[dof] = c for every constraint c.
__global__ void k_con_masks(int nc, const int* con_dof, ConPairs cp, unsigned char* cmask, int* dof_con) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int d = con_dof[c];
  dof_con[d] = c;
  if (con_is_pair(cp, c)) {  // both dofs stay free: the Krylov iteration projects them
    dof_con[cp.dof2[c]] = c;
    return;
  }
  cmask[d] = 1;
}

// Fixed values into the iterate (SSTREAM2dNR2.m:101-104); two-entry rows are left to the Newton
// update, as the reference sets only fixed nodes.
__global__ void k_set_con_values(int nc, const int* con_dof, const int* con_sys, const int* sel,
                                 const double* con_rhs, double* X, ConPairs cp) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nc && (!sel || sel[con_sys[c]]) && !con_is_pair(cp, c)) X[con_dof[c]] = con_rhs[c];
}

__global__ void k_zero_sel(const int* rb_start, const int* rb_sys, const int* sel, double* v) {
  const int blk = blockIdx.x;
  if (!sel[rb_sys[blk]]) return;
  for (int i = rb_start[blk] + threadIdx.x; i < rb_start[blk + 1]; i += blockDim.x) v[i] = 0;
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------

template <class T>
static T* walloc(ua_mesh* m, size_t n) {
  return (T*)dev_alloc(m, n * sizeof(T));
}

// The patch plan the parameters ask for: patch_nodes > 0 cuts every system into patches of that
// many nodes; 0 takes the shape tuned for this device, element type and dof count by
// ua_autotune, or the default.  K and R do not depend on the plan.
static int ensure_plan(ua_mesh* m, const ua_params* p) {
  if (!p) return UA_OK;
  if (p->patch_nodes < 0 || p->patch_nodes > 1024)
    return set_error(UA_ERR_INVALID, "patch_nodes must be 0 (tuned or default) or 1..1024");
  if (p->asm_threads != 0 && p->asm_threads != 128 && p->asm_threads != 256)
    return set_error(UA_ERR_INVALID, "asm_threads must be 0 (tuned or default), 128 or 256");
  if (p->asm_regs != 0 && p->asm_regs != 128 && p->asm_regs != 96 && p->asm_regs != 80)
    return set_error(UA_ERR_INVALID, "asm_regs must be 0 (tuned or default), 128, 96 or 80");
  const AsmTuning t = tuned_assembly(m->device, m->nod, m->ndof);
  m->asm_threads = p->asm_threads > 0 ? p->asm_threads : t.threads;
  m->asm_regs = p->asm_regs > 0 ? p->asm_regs : t.regs;
  if (m->asm_regs == 96 && m->asm_threads != 128)
    return set_error(UA_ERR_INVALID, "asm_regs = 96 runs 128-thread CTAs only (asm_threads = 128)");
  return rebuild_patches(m, p->patch_nodes > 0 ? PatchShape{0, p->patch_nodes} : t.shape);
}

static int ensure_work(ua_mesh* m, const ua_params* p) {
  if (int rc = ensure_plan(m, p)) return rc;
  if (m->work) return UA_OK;
  UA_CUDA_TRY(cudaSetDevice(m->device));
  Work* w = new Work();
  const int nsys = m->dm.nsys, N = m->ndof_total, NN = m->nn_total;
  w->nsys = nsys;
  cudaDeviceGetAttribute(&w->nsm, cudaDevAttrMultiProcessorCount, m->device);
  // row blocks: per system and per dof component (u rows, v rows, ...), so that row block i
  // of every component covers the same nodes (the node-sliced kernels write both rows of a node)
  std::vector<int> rb_start, rb_sys;
  w->h_sys_rb_off.assign(nsys + 1, 0);
  for (int s = 0; s < nsys; ++s) {
    const int d0 = m->h_dof_off[s], nd = m->h_dof_off[s + 1] - d0;
    const int ncomp = (m->ndof > 1 && nd % m->ndof == 0) ? m->ndof : 1, nc = nd / ncomp;
    for (int c = 0; c < ncomp; ++c)
      for (int r = d0 + c * nc; r < d0 + (c + 1) * nc; r += kRB) {
        rb_start.push_back(r);
        rb_sys.push_back(s);
      }
    w->h_sys_rb_off[s + 1] = (int)rb_start.size();
  }
  rb_start.push_back(N);
  w->nrb = (int)rb_sys.size();
  bool ok = true;
  auto up = [&](const std::vector<int>& v) -> int* {
    int* d = walloc<int>(m, v.size());
    if (!d) { ok = false; return nullptr; }
    cudaMemcpy(d, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice);
    return d;
  };
  w->rb_start = up(rb_start);
  w->rb_sys = up(rb_sys);
  w->sys_rb_off = up(w->h_sys_rb_off);
  w->rowptr = walloc<int>(m, N + 1);
  w->colind = walloc<int>(m, (size_t)m->nnz_total);
  w->diagpos = walloc<int>(m, N);
  double** fp[] = {&w->h, &w->s, &w->S, &w->B, &w->rho, &w->A, &w->n, &w->C, &w->m};
  for (auto f : fp) { *f = walloc<double>(m, NN); ok = ok && *f; }
  w->scal = walloc<SysScal>(m, nsys);
  double** dv[] = {&w->X, &w->X0, &w->dX, &w->R, &w->frhs, &w->Tint, &w->Fext};
  for (auto f : dv) { *f = walloc<double>(m, N); ok = ok && *f; }
  void** kv[] = {&w->kr, &w->kz, &w->kp, &w->kq, &w->invd};
  for (auto f : kv) { *f = walloc<double>(m, N); ok = ok && *f; }
  if (m->ndof == 3) {
    double** uf[] = {&w->h0, &w->u0, &w->v0, &w->as0, &w->ab0, &w->as1, &w->ab1, &w->dadh};
    for (auto f : uf) { *f = walloc<double>(m, NN); ok = ok && *f; }
    void** bv[] = {&w->krh, &w->ks, &w->ksh, &w->kt};
    for (auto f : bv) { *f = walloc<double>(m, N); ok = ok && *f; }
  }
  w->part = walloc<double>(m, 4 * (size_t)w->nrb);
  w->sysv = walloc<double>(m, SV_COUNT * (size_t)nsys);
  w->done = walloc<int>(m, nsys);
  w->its = walloc<int>(m, nsys);
  w->status = walloc<int>(m, nsys);
  w->sel = walloc<int>(m, nsys);
  w->gamma = walloc<double>(m, nsys);
  w->cmask = walloc<unsigned char>(m, N);
  w->dof_con = walloc<int>(m, N);
  ok = ok && w->rowptr && w->colind && w->diagpos && w->scal && w->part && w->sysv && w->done && w->its &&
       w->status && w->sel && w->gamma && w->cmask && w->dof_con && w->rb_start && w->rb_sys && w->sys_rb_off;
  if (!ok) { delete w; return set_error(UA_ERR_OOM, "device allocation of work buffers failed"); }
  w->nan_first = walloc<int>(m, 16);
  if (!w->nan_first) { delete w; return set_error(UA_ERR_OOM, "device allocation of work buffers failed"); }
  if (cudaMallocHost(&w->h_sysv, SV_COUNT * sizeof(double) * nsys) != cudaSuccess ||
      cudaMallocHost(&w->h_int, 4 * sizeof(int) * (nsys + 1)) != cudaSuccess ||
      cudaMallocHost(&w->h_nan, 16 * sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&w->h_gamma, sizeof(double) * nsys) != cudaSuccess) {
    delete w;
    return set_error(UA_ERR_OOM, "pinned host allocation failed");
  }
  k_dof_csr<<<(NN + 127) / 128, 128, 0, m->stream>>>(m->dm, w->rowptr, w->colind, w->diagpos), ++g_launches;
  int nnz = (int)m->nnz_total;
  UA_CUDA_TRY(cudaMemcpyAsync(w->rowptr + N, &nnz, sizeof(int), cudaMemcpyHostToDevice, m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  m->work = w;
  return UA_OK;
}

static int ensure_K(ua_mesh* m, int prec) {
  Work* w = m->work;
  if (prec == UA_PREC_MIXED) {
    if (!w->Kf) w->Kf = walloc<float>(m, (size_t)m->nnz_total);
    if (!w->Kf) return set_error(UA_ERR_OOM, "device allocation of the FP32 tangent failed");
  } else {
    if (!w->Kd) w->Kd = walloc<double>(m, (size_t)m->nnz_total);
    if (!w->Kd) return set_error(UA_ERR_OOM, "device allocation of the FP64 tangent failed");
  }
  return UA_OK;
}

static UvPhys make_phys(const ua_params* p) {
  UvPhys P;
  P.kH = p->kH; P.Hh0 = p->Hh0; P.SpeedZero = p->SpeedZero; P.EpsZero = p->EpsZero; P.etaZero = p->etaZero;
  P.Czero = p->Czero; P.Cmin = p->Cmin; P.AGlenmin = p->AGlenmin;
  P.Dvisk = p->Picard ? 0.0 : p->NRviscosity;  // uvMatrixAssemblySSTREAM.m:67-71
  P.Nzero = p->Nzero;
  P.law = p->SlidingLaw;
  P.melange = p->IncludeMelangeModelPhysics != 0;
  return P;
}

// The sliding-law and melange fields the configured law reads (BasalDrag.m), copied to the
// device for every system; the others stay null.  A law whose fields are missing is refused.
static int upload_drag_fields(ua_mesh* m, const ua_params* p, const ua_fields* F, int nF) {
  Work* w = m->work;
  if (p->SlidingLaw < UA_SLIDING_WEERTMAN || p->SlidingLaw > UA_SLIDING_JOUGHIN)
    return set_error(UA_ERR_INVALID, "BasalDrag:CaseNotFound unknown SlidingLaw %d", p->SlidingLaw);
  const int law = p->SlidingLaw;
  bool need[11] = {};
  need[0] = law == UA_SLIDING_BUDD;
  need[1] = law == UA_SLIDING_TSAI || law == UA_SLIDING_COULOMB || law == UA_SLIDING_CORNFORD ||
            law == UA_SLIDING_UMBI;
  need[2] = law == UA_SLIDING_JOUGHIN;
  for (int k = 3; k < 11; ++k) need[k] = p->IncludeMelangeModelPhysics != 0;
  const char* names[11] = {"q", "muk", "V0", "uo", "vo", "Co", "mo", "ua", "va", "Ca", "ma"};
  for (int k = 0; k < 11; ++k) {
    w->dragf[k] = nullptr;
    if (!need[k]) continue;
    if (!w->dragbuf[k]) w->dragbuf[k] = walloc<double>(m, (size_t)m->nn_total);
    if (!w->dragbuf[k]) return set_error(UA_ERR_OOM, "device allocation of F.%s failed", names[k]);
    for (int s = 0; s < m->dm.nsys; ++s) {
      const ua_fields& f = F[nF == 1 ? 0 : s];
      const double* src[11] = {f.q, f.muk, f.V0, f.uo, f.vo, f.Co, f.mo, f.ua, f.va, f.Ca, f.ma};
      if (!src[k]) return set_error(UA_ERR_INVALID, "system %d: the sliding law needs F.%s", s, names[k]);
      UA_CUDA_TRY(cudaMemcpyAsync(w->dragbuf[k] + m->h_node_off[s], src[k], m->sys[s].nn * sizeof(double),
                                  f.location == UA_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                  m->stream));
    }
    w->dragf[k] = w->dragbuf[k];
  }
  return UA_OK;
}

static DragFields drag_fields(const Work* w) {
  DragFields D{};
  D.q = w->dragf[0]; D.muk = w->dragf[1]; D.V0 = w->dragf[2];
  for (int k = 0; k < 8; ++k) D.mel[k] = w->dragf[3 + k];
  return D;
}

static bool any_nan(const double* v, int n) {
  for (int i = 0; i < n; ++i)
    if (v[i] != v[i]) return true;
  return false;
}

// NaN scan of uploaded arrays on the device (the reference's anynan tests, SSTREAM2dNR2.m:42-66):
// per array k, first[k] = the lowest system with a NaN (node-indexed arrays map a node to its
// system, dof-indexed ones search the system dof offsets).  first[] starts at INT_MAX.
struct NanScan {
  const double* a[10];
  int len[10];
  int dof[10];
};

__global__ void k_nan_scan(NanScan S, const int* node_sys, const int* sys_dof_off, int nsys, int* first) {
  const int k = blockIdx.y;
  const double* a = S.a[k];
  const int n = S.len[k];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = a[i];
    if (v != v) {
      int sys = 0;
      if (S.dof[k]) {
        int lo = 0, hi = nsys - 1;  // largest sys with sys_dof_off[sys] <= i
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (sys_dof_off[mid] <= i) lo = mid; else hi = mid - 1;
        }
        sys = lo;
      } else {
        sys = node_sys[i];
      }
      atomicMin(first + k, sys);
    }
  }
}

// Nodal fields of system s (host or device pointers); SysScal staged in sc.  host_nan: scan host
// arrays for NaN here (else the caller scans the uploaded fields on the device).
static int upload_fields_sys(ua_mesh* m, const ua_fields& f, int s, SysScal& sc, bool host_nan = true,
                             bool copy = true) {
  Work* w = m->work;
  const int no = m->h_node_off[s], nn = m->sys[s].nn;
  const double* src[] = {f.h, f.S, f.B, f.rho, f.AGlen, f.n, f.C, f.m};
  double* dst[] = {w->h, w->S, w->B, w->rho, w->A, w->n, w->C, w->m};
  const char* names[] = {"h", "S", "B", "rho", "AGlen", "n", "C", "m"};
  for (int k = 0; k < 8; ++k) {
    if (!src[k]) return set_error(UA_ERR_INVALID, "system %d: null field pointer %s", s, names[k]);
    // SSTREAM2dNR2.m:42-65: NaN in C or A (warning + NaN solution in the
    // reference) and NaN in S, h, rho (error) all stop the solve here.
    if (host_nan && f.location == UA_HOST && any_nan(src[k], nn))
      return set_error(UA_ERR_NAN_INPUT, "SSTREAM2dNR2: nan in %s (system %d)", names[k], s);
    if (copy)
      UA_CUDA_TRY(cudaMemcpyAsync(dst[k] + no, src[k], nn * sizeof(double),
                                f.location == UA_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                m->stream));
  }
  sc.rhow = f.rhow; sc.g = f.g; sc.ca = std::cos(f.alpha); sc.sa = std::sin(f.alpha);
  sc.dt = f.dt;
  return UA_OK;
}

static void set_cube_flags(ua_mesh* m) {
  Work* w = m->work;
  k_cube_set<<<(m->dm.nsys + 255) / 256, 256, 0, m->stream>>>(m->dm.nsys, w->scal), ++g_launches;
  k_cube_check<<<(m->nn_total + 255) / 256, 256, 0, m->stream>>>(m->nn_total, m->dm.node_sys, w->n, w->m, w->scal),
      ++g_launches;
}

static int finish_fields(ua_mesh* m, const ua_params* p, const std::vector<SysScal>& sc, int s0, int count) {
  Work* w = m->work;
  UA_CUDA_TRY(cudaMemcpyAsync(w->scal + s0, sc.data(), count * sizeof(SysScal), cudaMemcpyHostToDevice, m->stream));
  set_cube_flags(m);
  k_calc_bs<<<(m->nn_total + 255) / 256, 256, 0, m->stream>>>(m->nn_total, m->dm.node_sys, w->scal, p->kH, p->Hh0,
                                                               w->h, w->S, w->B, w->rho, w->s), ++g_launches;
  UA_CUDA_TRY(cudaGetLastError());
  return UA_OK;
}

// Upload nodal fields of every system (host or device pointers) and compute s.  The NaN tests
// of host fields run on the device after the copies (device_nan_check).
static int upload_fields(ua_mesh* m, const ua_params* p, const ua_fields* F, int nF) {
  Work* w = m->work;
  const int nsys = m->dm.nsys;
  std::vector<SysScal> sc(nsys);
  for (int s = 0; s < nsys; ++s) {
    int rc = upload_fields_sys(m, F[nF == 1 ? 0 : s], s, sc[s], false, false);
    if (rc) return rc;
  }
  // one copy per run of systems whose arrays follow each other in memory (a batch passed as
  // slices of one array per field), else one per system
  double* dst[] = {w->h, w->S, w->B, w->rho, w->A, w->n, w->C, w->m};
  auto src_of = [&](int s, int k) -> const double* {
    const ua_fields& f = F[nF == 1 ? 0 : s];
    const double* a[] = {f.h, f.S, f.B, f.rho, f.AGlen, f.n, f.C, f.m};
    return a[k];
  };
  for (int k = 0; k < 8; ++k)
    for (int s = 0; s < nsys;) {
      const int loc = F[nF == 1 ? 0 : s].location;
      const double* a = src_of(s, k);
      size_t len = (size_t)m->sys[s].nn;
      int e = s + 1;
      while (e < nsys && F[nF == 1 ? 0 : e].location == loc && src_of(e, k) == a + len) len += m->sys[e++].nn;
      UA_CUDA_TRY(cudaMemcpyAsync(dst[k] + m->h_node_off[s], a, len * sizeof(double),
                                  loc == UA_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, m->stream));
      s = e;
    }
  if (int rc = upload_drag_fields(m, p, F, nF)) return rc;
  return finish_fields(m, p, sc, 0, nsys);
}

// The NaN tests of upload_fields + upload_velocity on the device, over every system whose fields
// came from host memory, with the host scan's errors and order: fields before velocities, then
// the lowest system, then the field order h, S, B, rho, AGlen, n, C, m.
static int device_nan_check(ua_mesh* m, const ua_fields* F, int nF) {
  Work* w = m->work;
  const int nsys = m->dm.nsys;
  bool any_host = false;
  for (int s = 0; s < nsys; ++s) any_host = any_host || F[nF == 1 ? 0 : s].location == UA_HOST;
  if (!any_host) return UA_OK;
  NanScan S{};
  const double* arr[] = {w->h, w->S, w->B, w->rho, w->A, w->n, w->C, w->m, w->X};
  const int na = 9;
  for (int k = 0; k < na; ++k) {
    S.a[k] = arr[k];
    S.len[k] = k < 8 ? m->nn_total : m->ndof_total;
    S.dof[k] = k == 8;
  }
  UA_CUDA_TRY(cudaMemsetAsync(w->nan_first, 0x7f, na * sizeof(int), m->stream));
  k_nan_scan<<<dim3(296, na), 256, 0, m->stream>>>(S, m->dm.node_sys, m->dm.sys_dof_off, nsys, w->nan_first),
      ++g_launches;
  UA_CUDA_TRY(cudaGetLastError());
  int first[9];
  UA_CUDA_TRY(cudaMemcpyAsync(w->h_nan, w->nan_first, na * sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  std::memcpy(first, w->h_nan, sizeof(first));
  const char* names[] = {"h", "S", "B", "rho", "AGlen", "n", "C", "m"};
  auto host_sys = [&](int s) { return s >= 0 && s < nsys && F[nF == 1 ? 0 : s].location == UA_HOST; };
  int bs = nsys, bk = -1;
  for (int k = 0; k < 8; ++k)
    if (host_sys(first[k]) && first[k] < bs) { bs = first[k]; bk = k; }
  if (bk >= 0) return set_error(UA_ERR_NAN_INPUT, "SSTREAM2dNR2: nan in %s (system %d)", names[bk], bs);
  if (host_sys(first[8])) return set_error(UA_ERR_NAN_INPUT, "uvMatrixAssembly:NaN NaN in F.ub or F.vb");
  return UA_OK;
}

// Velocities of system s into the dof vector X (host_nan as upload_fields_sys).
static int upload_velocity_sys(ua_mesh* m, const ua_fields& f, int s, bool host_nan = true) {
  Work* w = m->work;
  const int d0 = m->h_dof_off[s], nn = m->sys[s].nn;
  if (!f.ub || !f.vb) return set_error(UA_ERR_INVALID, "null ub/vb");
  if (host_nan && f.location == UA_HOST && (any_nan(f.ub, nn) || any_nan(f.vb, nn)))
    return set_error(UA_ERR_NAN_INPUT, "uvMatrixAssembly:NaN NaN in F.ub or F.vb");
  auto kind = f.location == UA_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  UA_CUDA_TRY(cudaMemcpyAsync(w->X + d0, f.ub, nn * sizeof(double), kind, m->stream));
  UA_CUDA_TRY(cudaMemcpyAsync(w->X + d0 + nn, f.vb, nn * sizeof(double), kind, m->stream));
  return UA_OK;
}

// Velocities of the fields into the dof vector X.
static int upload_velocity(ua_mesh* m, const ua_fields* F, int nF) {
  for (int s = 0; s < m->dm.nsys; ++s) {
    int rc = upload_velocity_sys(m, F[nF == 1 ? 0 : s], s, false);
    if (rc) return rc;
  }
  return device_nan_check(m, F, nF);
}

// BCs2MLC.m:19-25 + CreateLuv.m:28-76 + ScaleL.m for fixed-node BCs: one unit row
// per unique fixed node (first occurrence's value), u rows then v rows.
// Nodal normals of the boundary (CalcEdgeAndNodalNormals.m): the boundary edges are the element
// edges that belong to one element, each traversed in its element's node order; an edge A->B has
// the unit normal (-dy, dx)/l, a boundary node gets the normal of the edge starting at it plus that
// of the edge ending at it (a P2 mid-edge node the mean of its two sub-edges), normalised.
static void nodal_normals(const HostSystem& hs, int nod, std::vector<double>& Nx, std::vector<double>& Ny) {
  const int ne = hs.ne;
  const int cl[3] = {0, nod == 3 ? 1 : 2, nod == 3 ? 2 : 4};
  std::vector<std::array<int, 3>> edges;  // (start corner, mid or -1, end corner)
  std::vector<std::pair<long long, int>> key;
  for (int e = 0; e < ne; ++e)
    for (int k = 0; k < 3; ++k) {
      const int a = hs.conn[(size_t)cl[k] * ne + e], b = hs.conn[(size_t)cl[(k + 1) % 3] * ne + e];
      const int mid = nod == 6 ? hs.conn[(size_t)(cl[k] + 1) * ne + e] : -1;
      key.push_back({(long long)std::min(a, b) * hs.nn + std::max(a, b), (int)edges.size()});
      edges.push_back({a, mid, b});
    }
  std::sort(key.begin(), key.end());
  Nx.assign(hs.nn, 0.0); Ny.assign(hs.nn, 0.0);
  std::vector<int> bnd;
  for (size_t i = 0; i < key.size(); ++i) {
    const bool dup = (i > 0 && key[i].first == key[i - 1].first) ||
                     (i + 1 < key.size() && key[i].first == key[i + 1].first);
    if (!dup) bnd.push_back(key[i].second);
  }
  std::sort(bnd.begin(), bnd.end());
  auto unit_normal = [&](int a, int b, double& nx, double& ny) {
    const double dx = hs.x[b] - hs.x[a], dy = hs.y[b] - hs.y[a];
    nx = -dy; ny = dx;
    const double l = std::sqrt(nx * nx + ny * ny);
    nx = nx / l; ny = ny / l;
  };
  for (int ei : bnd) {  // start nodes: assignment
    const auto& E = edges[ei];
    double nx, ny;
    unit_normal(E[0], E[1] >= 0 ? E[1] : E[2], nx, ny);
    Nx[E[0]] = nx; Ny[E[0]] = ny;
  }
  for (int ei : bnd) {  // end nodes and mid nodes: sums
    const auto& E = edges[ei];
    double nx2, ny2;
    unit_normal(E[1] >= 0 ? E[1] : E[0], E[2], nx2, ny2);
    Nx[E[2]] = Nx[E[2]] + nx2; Ny[E[2]] = Ny[E[2]] + ny2;
    if (E[1] >= 0) {
      double nx1, ny1;
      unit_normal(E[0], E[1], nx1, ny1);
      Nx[E[1]] = Nx[E[1]] + (nx1 + nx2) / 2; Ny[E[1]] = Ny[E[1]] + (ny1 + ny2) / 2;
    }
  }
  for (int i = 0; i < hs.nn; ++i) {
    const double l = std::sqrt(Nx[i] * Nx[i] + Ny[i] * Ny[i]);
    Nx[i] = Nx[i] / l; Ny[i] = Ny[i] / l;
  }
}

// The constraint rows of the BCs, host side (BCs2MLC.m:19-29, CreateLuv.m:28-76, ScaleL.m:28-33,
// createLh.m): per system the u ties, the v ties, the fixed u nodes (increasing, first occurrence
// of a repeated node), the fixed v nodes, the fixed-normal-velocity nodes, then (ndof 3) the fixed
// h nodes as given.  Row c has the entry con_v1[c] at dof con_dof[c] and, for ties and normal
// rows, con_v2[c] at con_dof2[c] (else -1), all scaled to a unit row like the right-hand side.
// The rows must have disjoint support (B B' diagonal, ABfgPreEliminate.m:35).
static int constraint_rows(const ua_mesh* m, const ua_bcs* bcs, int nB, std::vector<int>& con_dof,
                           std::vector<int>& con_sys, std::vector<double>& rhs, std::vector<int>& sys_off,
                           std::vector<int>* con_dof2 = nullptr, std::vector<double>* con_v1 = nullptr,
                           std::vector<double>* con_v2 = nullptr) {
  const int nsys = m->dm.nsys;
  con_dof.clear(); con_sys.clear(); rhs.clear();
  std::vector<int> d2;
  std::vector<double> v1, v2;
  sys_off.assign(nsys + 1, 0);
  for (int s = 0; s < nsys; ++s) {
    const ua_bcs* b = bcs ? &bcs[nB == 1 ? 0 : s] : nullptr;
    const int nn = m->sys[s].nn, d0 = m->h_dof_off[s];
    auto push = [&](int da, double a, int db, double bval, double r) {
      const double scale = 1.0 / std::sqrt(a * a + (db >= 0 ? bval * bval : 0.0));  // ScaleL.m:28-33
      con_dof.push_back(da); d2.push_back(db); v1.push_back(a * scale); v2.push_back(db >= 0 ? bval * scale : 0.0);
      con_sys.push_back(s); rhs.push_back(r * scale);
    };
    for (int comp = 0; b && comp < 2; ++comp) {  // ties (CreateLuv.m:35-48)
      const int n = comp == 0 ? b->n_utied : b->n_vtied;
      const int* A = comp == 0 ? b->utied_a : b->vtied_a;
      const int* B = comp == 0 ? b->utied_b : b->vtied_b;
      for (int i = 0; i < n; ++i) {
        if (A[i] < 0 || A[i] >= nn || B[i] < 0 || B[i] >= nn || A[i] == B[i])
          return set_error(UA_ERR_INVALID, "system %d: tied node index out of range or tied to itself", s);
        push(d0 + comp * nn + A[i], 1.0, d0 + comp * nn + B[i], -1.0, 0.0);
      }
    }
    const int base = 0;  // indices are 0-based at this layer
    for (int comp = 0; b && comp < 2; ++comp) {
      int n = comp == 0 ? b->n_ufixed : b->n_vfixed;
      const int* nodes = comp == 0 ? b->ufixed_node : b->vfixed_node;
      const double* vals = comp == 0 ? b->ufixed_value : b->vfixed_value;
      std::vector<std::pair<int, int>> idx;  // (node, first position)
      for (int i = 0; i < n; ++i) {
        int nd = nodes[i] - base;
        if (nd < 0 || nd >= nn) return set_error(UA_ERR_INVALID, "system %d: fixed node index out of range", s);
        idx.push_back({nd, i});
      }
      std::stable_sort(idx.begin(), idx.end(), [](auto& x, auto& y) { return x.first < y.first; });
      for (size_t i = 0; i < idx.size(); ++i) {
        if (i > 0 && idx[i].first == idx[i - 1].first) continue;  // unique, first occurrence
        double v = vals ? vals[idx[i].second] : 0.0;
        if (v != v) return set_error(UA_ERR_NAN_INPUT, "nan in fixed value");
        push(d0 + comp * nn + idx[i].first, 1.0, -1, 0.0, v);
      }
    }
    if (b && b->n_normal > 0) {  // fixed normal velocity (CreateLuv.m:62-72): Nx u + Ny v = -value
      std::vector<double> Nx, Ny;
      nodal_normals(m->sys[s], m->nod, Nx, Ny);
      for (int i = 0; i < b->n_normal; ++i) {
        const int nd = b->normal_node[i];
        if (nd < 0 || nd >= nn) return set_error(UA_ERR_INVALID, "system %d: normal-velocity node out of range", s);
        if (!std::isfinite(Nx[nd]) || !std::isfinite(Ny[nd]) || Nx[nd] * Nx[nd] + Ny[nd] * Ny[nd] < 0.25)
          return set_error(UA_ERR_INVALID, "system %d: normal-velocity node %d is not on the mesh boundary", s, nd);
        const double v = b->normal_value ? b->normal_value[i] : 0.0;
        if (v != v) return set_error(UA_ERR_NAN_INPUT, "nan in fixed normal velocity");
        push(d0 + nd, Nx[nd], d0 + nn + nd, Ny[nd], -v);
      }
    }
    if (b && m->ndof == 3 && b->n_hfixed > 0) {  // createLh.m: fixed h nodes in the given order
      std::vector<unsigned char> seen(nn, 0);
      for (int i = 0; i < b->n_hfixed; ++i) {
        int nd = b->hfixed_node[i];
        if (nd < 0 || nd >= nn) return set_error(UA_ERR_INVALID, "system %d: fixed h node index out of range", s);
        if (seen[nd]) return set_error(UA_ERR_INVALID, "ABfgPreEliminate:B B*B^T not diagonal (h node %d fixed twice)", nd);
        seen[nd] = 1;
        double v = b->hfixed_value ? b->hfixed_value[i] : 0.0;
        if (v != v) return set_error(UA_ERR_NAN_INPUT, "nan in fixed h value");
        push(d0 + 2 * nn + nd, 1.0, -1, 0.0, v);
      }
    }
    sys_off[s + 1] = (int)con_dof.size();
  }
  // disjoint support: every dof in at most one row
  {
    std::vector<int> all(con_dof);
    for (int d : d2)
      if (d >= 0) all.push_back(d);
    std::sort(all.begin(), all.end());
    for (size_t i = 1; i < all.size(); ++i)
      if (all[i] == all[i - 1])
        return set_error(UA_ERR_INVALID, "ABfgPreEliminate:B B*B^T not diagonal (dof %d is in two constraints)",
                         all[i]);
  }
  if (con_dof2) *con_dof2 = d2;
  if (con_v1) *con_v1 = v1;
  if (con_v2) *con_v2 = v2;
  return UA_OK;
}

static int build_constraints(ua_mesh* m, const ua_bcs* bcs, int nB) {
  Work* w = m->work;
  const int nsys = m->dm.nsys;
  std::vector<int> con_dof, con_sys, sys_off, con_dof2;
  std::vector<double> rhs, con_v1, con_v2;
  if (int rc = constraint_rows(m, bcs, nB, con_dof, con_sys, rhs, sys_off, &con_dof2, &con_v1, &con_v2)) return rc;
  const int nc = (int)con_dof.size();
  // two-entry rows (ties, normal velocities): their coefficients and the list of those rows
  std::vector<int> pairs;
  for (int c = 0; c < nc; ++c)
    if (con_dof2[c] >= 0) pairs.push_back(c);
  w->npair = (int)pairs.size();
  if (w->npair) {
    if ((size_t)nc > w->pair_cap) {
      w->con_dof2 = walloc<int>(m, nc);
      w->con_v1 = walloc<double>(m, nc);
      w->con_v2 = walloc<double>(m, nc);
      w->pair_rows = walloc<int>(m, nc);
      if (!w->con_dof2 || !w->con_v1 || !w->con_v2 || !w->pair_rows)
        return set_error(UA_ERR_OOM, "constraint allocation failed");
      w->pair_cap = nc;
    }
    UA_CUDA_TRY(cudaMemcpyAsync(w->con_dof2, con_dof2.data(), nc * sizeof(int), cudaMemcpyHostToDevice, m->stream));
    UA_CUDA_TRY(cudaMemcpyAsync(w->con_v1, con_v1.data(), nc * sizeof(double), cudaMemcpyHostToDevice, m->stream));
    UA_CUDA_TRY(cudaMemcpyAsync(w->con_v2, con_v2.data(), nc * sizeof(double), cudaMemcpyHostToDevice, m->stream));
    UA_CUDA_TRY(cudaMemcpyAsync(w->pair_rows, pairs.data(), w->npair * sizeof(int), cudaMemcpyHostToDevice,
                                m->stream));
  }
  if (nc > w->nc || !w->con_dof) {
    int cap = std::max(nc, 1);
    w->con_dof = walloc<int>(m, cap);
    w->con_sys = walloc<int>(m, cap);
    w->con_rhs = walloc<double>(m, cap);
    w->lam = walloc<double>(m, cap);
    w->dlam = walloc<double>(m, cap);
    w->grhs = walloc<double>(m, cap);
    if (!w->sys_con_off) w->sys_con_off = walloc<int>(m, nsys + 1);
    if (!w->con_dof || !w->con_sys || !w->con_rhs || !w->lam || !w->dlam || !w->grhs || !w->sys_con_off)
      return set_error(UA_ERR_OOM, "constraint allocation failed");
  }
  w->nc = nc;
  w->h_sys_con_off = sys_off;
  if (nc) {
    UA_CUDA_TRY(cudaMemcpyAsync(w->con_dof, con_dof.data(), nc * sizeof(int), cudaMemcpyHostToDevice, m->stream));
    UA_CUDA_TRY(cudaMemcpyAsync(w->con_sys, con_sys.data(), nc * sizeof(int), cudaMemcpyHostToDevice, m->stream));
    UA_CUDA_TRY(cudaMemcpyAsync(w->con_rhs, rhs.data(), nc * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  }
  UA_CUDA_TRY(cudaMemcpyAsync(w->sys_con_off, sys_off.data(), (nsys + 1) * sizeof(int), cudaMemcpyHostToDevice,
                              m->stream));
  // dof masks, on the device: cmask = 0 and dof_con = -1 everywhere, then one thread per
  // constraint (its dof is unique: repeated nodes were dropped above)
  UA_CUDA_TRY(cudaMemsetAsync(w->cmask, 0, m->ndof_total, m->stream));
  UA_CUDA_TRY(cudaMemsetAsync(w->dof_con, 0xff, m->ndof_total * sizeof(int), m->stream));
  if (nc)
    k_con_masks<<<(nc + 255) / 256, 256, 0, m->stream>>>(nc, w->con_dof, con_pairs(w), w->cmask, w->dof_con),
        ++g_launches;
  UA_CUDA_TRY(cudaGetLastError());
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  return UA_OK;
}

// The host staging buffers (pinned) are rewritten only after the stream has drained, so an
// earlier asynchronous copy from them cannot pick up the new values.
static int set_sel(ua_mesh* m, const std::vector<int>& sel) {
  Work* w = m->work;
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  w->h_sel.assign(sel.begin(), sel.begin() + w->nsys);
  for (int s = 0; s < w->nsys; ++s) w->h_int[s] = sel[s];
  UA_CUDA_TRY(cudaMemcpyAsync(w->sel, w->h_int, w->nsys * sizeof(int), cudaMemcpyHostToDevice, m->stream));
  return UA_OK;
}

static int set_gamma(ua_mesh* m, const std::vector<double>& g) {
  Work* w = m->work;
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  for (int s = 0; s < w->nsys; ++s) w->h_gamma[s] = g[s];
  UA_CUDA_TRY(cudaMemcpyAsync(w->gamma, w->h_gamma, w->nsys * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  return UA_OK;
}

// Residual-only or residual+tangent assembly of the selected systems at X (+gamma dX).
static int assemble(ua_mesh* m, const ua_params* p, bool withK, bool useDir, const double* X, bool parts) {
  Work* w = m->work;
  UvIn in{w->h, w->s, w->S, w->B, w->rho, w->A, w->n, w->C, w->m, X, useDir ? w->dX : nullptr,
          useDir ? w->gamma : nullptr, w->scal, w->sel};
  in.drag = drag_fields(w);
  bool fp32 = p->precision == UA_PREC_MIXED;
  UvOut out{w->R, withK ? (fp32 ? (void*)w->Kf : (void*)w->Kd) : nullptr, parts ? w->Tint : nullptr,
            parts ? w->Fext : nullptr};
  cudaEvent_t ev[2];
  prof_begin(m, withK ? PK_ASMK : PK_ASMR, ev);
  cudaError_t e = launch_uv_assembly(m, make_phys(p), in, out, withK, fp32, m->asm_threads, m->asm_regs);
  prof_end(m, ev);
  ++g_launches;
  if (e != cudaSuccess) return set_error(UA_ERR_CUDA, "uv assembly launch: %s", cudaGetErrorString(e));
  return UA_OK;
}

// Cost function of every selected system at X + gamma dX with direction (dX, dl):
// CalcCostFunctionNR.m:14-41.  Result in sysv[SV_FF] (rForce) and sysv[SV_FD] (D2).
// Cost function at X + gamma dX.  assembleR = false takes w->R as it stands:
// the residual just assembled at X, which is the R-only assembly at gamma = 0.
// withK: assemble the tangent too (the next Newton system's, if this point is accepted).
static int cost_eval(ua_mesh* m, const ua_params* p, bool useDir, bool assembleR = true, bool withK = false) {
  Work* w = m->work;
  if (assembleR) {
    int rc = assemble(m, p, withK, useDir, w->X, false);
    if (rc) return rc;
  }
  k_cost_rows<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->R, w->dof_con, w->lam,
                                             w->dlam, useDir ? w->gamma : nullptr, w->dX, w->part, w->con_dof, con_pairs(w)), ++g_launches;
  k_cost_reduce<<<w->nsys, kRedThreads, 0, m->stream>>>(w->sys_rb_off, w->nrb, w->sel, w->part, w->nsys, w->sysv,
                                                         w->sys_con_off, w->con_dof, w->con_rhs, w->X,
                                                         useDir ? w->dX : nullptr, w->dlam,
                                                         useDir ? w->gamma : nullptr, 0, con_pairs(w)), ++g_launches;
  UA_CUDA_TRY(cudaGetLastError());
  UA_CUDA_TRY(cudaMemcpyAsync(w->h_sysv, w->sysv, SV_COUNT * w->nsys * sizeof(double), cudaMemcpyDeviceToHost,
                              m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  return UA_OK;
}

template <typename KT, typename VT>
static int pcg_t(ua_mesh* m, const ua_params* p, const KT* K, int* its_out, const double* eta = nullptr) {
  Work* w = m->work;
  const int N = m->ndof_total;
  // lanes per row of the row-block products: the caller's choice, else one thread per row for
  // P1 uv rows (about 14 entries) and two lanes for P2 rows (about 30); measured on B200 over
  // 1/2/4/8/16 lanes, thread-per-row keeps the most independent loads in flight per warp
  const int lpr = p->spmv_lanes ? p->spmv_lanes : (m->nod == 3 ? 1 : 2);
  if (lpr != 1 && lpr != 2 && lpr != 4 && lpr != 8 && lpr != 16 && lpr != 32)
    return set_error(UA_ERR_INVALID, "spmv_lanes must be 0, 1, 2, 4, 8, 16 or 32");
  // per-system tolerance (relative residual of the preconditioned solve)
  for (int s = 0; s < w->nsys; ++s) {
    const double e = eta ? eta[s] : p->krylov_rtol;
    w->h_sysv[s] = e * e;
  }
  UA_CUDA_TRY(cudaMemcpyAsync(w->sysv + SV_TOL2 * w->nsys, w->h_sysv, w->nsys * sizeof(double),
                              cudaMemcpyHostToDevice, m->stream));
  // the uv block layout of a mesh handle (a bare matrix from ua_solve_kape_symmetric has none);
  // reading only the u block's column indices pays off for FP64 values (measured on B200: 5%
  // faster for FP64, 9% slower for FP32, where the second value stream costs more than the
  // index bytes saved)
  const bool uvlay = m->ndof == 2 && !m->h_nodeptr.empty() && sizeof(KT) == 8;
  // preconditioner: aggregation AMG V(1,1) for the uv tangent of a mesh handle, else point Jacobi
  bool amg = p->krylov_precond == UA_PC_AMG && m->ndof == 2 && !m->h_nodeptr.empty();
  if (amg && !w->kx0) {
    w->kx0 = walloc<double>(m, N);
    if (!w->kx0) return set_error(UA_ERR_OOM, "device allocation of the AMG work vector failed");
  }
  if (amg && amg_setup(m, p->amg_smoothed != 0) != UA_OK) amg = false;  // shapes the hierarchy cannot take keep point Jacobi
  const bool fp32 = sizeof(KT) == 4;
  if (amg) {
    // the systems of this Newton step only (the others' hierarchies are not read)
    // prolongator refresh: every Newton step in FP64 (the Newton trajectory of the reference's
    // direct solves), every fourth in the mixed form, unless set
    const int prefresh = p->amg_P_refresh > 0 ? p->amg_P_refresh : (fp32 ? 4 : 1);
    cudaEvent_t ev[2];
    prof_begin(m, PK_SETUP, ev);
    int rc = amg_numeric(m, w->rowptr, w->colind, K, fp32, w->cmask, &g_launches, w->sel, &w->h_sel, prefresh,
                         !w->no_graph && !p->profile);
    prof_end(m, ev);
    if (rc) return rc;
  } else {
    k_invdiag<KT, VT><<<(N + 255) / 256, 256, 0, m->stream>>>(N, K, w->diagpos, w->cmask, (VT*)w->invd), ++g_launches;
  }
  // particular solution on the constrained dofs
  k_zero_sel<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->sel, w->dX), ++g_launches;
  if (w->nc)
    k_con_particular<<<(w->nc + 255) / 256, 256, 0, m->stream>>>(w->nc, w->con_dof, w->con_sys, w->sel, w->con_rhs,
                                                                 w->X, w->dX, w->grhs, con_pairs(w)), ++g_launches;
  VT *r = (VT*)w->kr, *z = (VT*)w->kz, *pp = (VT*)w->kp, *q = (VT*)w->kq;
  // with AMG the Jacobi-type kernels write the l1 pre-smoothed vector x0 and the V-cycle writes z (and r.z)
  const VT* invd = amg ? (const VT*)amg_invd0(m) : (const VT*)w->invd;
  VT* zj = amg ? (VT*)w->kx0 : z;
  // q is free between update1 and the next SpMV: the V-cycle's fine-level scratch
  AmgPcgView view{w->rowptr, w->colind, K, r, w->kx0, z, nullptr, w->part, w->cmask, w->sel, w->done,
                  w->rb_start, w->rb_sys, w->nrb, lpr, q};
  if (w->prof.on) { view.mark = prof_amg; view.mark_ctx = m; }
  // mixed precision: the V-cycle's finest-level residual and smoothing read a BF16 copy of K (the
  // l1 diagonal and the Galerkin products come from the FP32 values; the cycle stays symmetric and,
  // with the l1 diagonal above half the row sums, positive definite)
  // node slices (default): the PCG SpMV and the V-cycle's finest-level passes read per-tangent
  // sliced-ELL copies of K (FP32/FP64, plus BF16 for the mixed V-cycle) instead of the CSR
  const bool sell = amg && p->krylov_sell && amg_sell_init(m, w->h_sys_rb_off) == UA_OK;
  // with node slices the p.q and r.z partials are per slice
  const double* spart = nullptr;
  const int* sys_sl_off = nullptr;
  if (sell) amg_sell_partials(m, &spart, &sys_sl_off);
  if (sell) {
    cudaEvent_t ev[2];
    prof_begin(m, PK_SETUP, ev);
    int rc = amg_sell_fill(m, K, fp32, fp32 && p->precond_bf16, &g_launches, w->sel);
    prof_end(m, ev);
    if (rc) return rc;
    view.sell = true;
    view.sell_lo = fp32 && p->precond_bf16;
  }
  if (amg && fp32 && p->precond_bf16 && !sell)
    view.K0lo = amg_bf16_copy(m, (const float*)K, m->nnz_total, &g_launches);
  // with AMG the finest-level Krylov kernels and the V-cycle loop over the row and node blocks of
  // the systems still iterating (lists recompacted after every convergence check)
  if (amg && !p->krylov_full_grid) {
    int rc = amg_act_init(m, w->h_sys_rb_off);
    if (rc) return rc;
    view.act = true;
  }
  const ActList act0 = view.act ? amg_act_rows0(m) : ActList{};
  const int grid0 = view.act ? act_grid(w->nrb, w->nsm) : w->nrb;
  cudaEvent_t kev[2];  // the Krylov iterations, from the initial residual to the last chunk
  prof_begin(m, PK_KRYLOV, kev);
  dispatch_lpr(lpr, [&](auto L) {
    if (uvlay)
      k_pcg_init<KT, VT, decltype(L)::value, true><<<w->nrb, 256, 0, m->stream>>>(
          w->rb_start, w->rb_sys, w->nrb, w->sel, w->rowptr, w->colind, K, w->dX, w->frhs, w->cmask, invd, r, zj,
          pp, w->part, m->dm.sys_dof_off);
    else
      k_pcg_init<KT, VT, decltype(L)::value, false><<<w->nrb, 256, 0, m->stream>>>(
          w->rb_start, w->rb_sys, w->nrb, w->sel, w->rowptr, w->colind, K, w->dX, w->frhs, w->cmask, invd, r, zj,
          pp, w->part, nullptr);
  });
  ++g_launches;
  // two-entry constraint rows (ties, normal velocities): the iteration runs in the range of the
  // projector I - B'B on their pairs; the fused p.q and r.z partials stay exact because p and r
  // stay in that range
  const ConPairs cp = con_pairs(w);
  const int npb = (w->npair + 255) / 256;
  if (w->npair && !amg)
    return set_error(UA_ERR_INVALID, "tied and normal-velocity constraints need the AMG preconditioner");
  if (w->npair)
    k_pair_project_r0<VT><<<npb, 256, 0, m->stream>>>(w->npair, w->pair_rows, w->con_dof, w->con_sys, w->sel, cp, r,
                                                      zj, invd), ++g_launches;
  if (amg) {
    // done[] is reset by the stage-0 reduction below; the V-cycle must see every selected system
    UA_CUDA_TRY(cudaMemsetAsync(w->done, 0, w->nsys * sizeof(int), m->stream));
    if (view.act) amg_act_compact(m, w->sel, w->done, &g_launches);
    view.pcopy = pp;
    int rc = amg_vcycle(m, fp32, view, &g_launches);
    if (rc) return rc;
    view.pcopy = nullptr;
    if (w->npair) {
      k_pair_project<VT><<<npb, 256, 0, m->stream>>>(w->npair, w->pair_rows, w->con_dof, w->con_sys, w->sel,
                                                     nullptr, cp, z), ++g_launches;
      k_pair_project<VT><<<npb, 256, 0, m->stream>>>(w->npair, w->pair_rows, w->con_dof, w->con_sys, w->sel,
                                                     nullptr, cp, pp), ++g_launches;
    }
  }
  k_pcg_reduce<<<w->nsys, kRedThreads, 0, m->stream>>>(0, w->sys_rb_off, w->nrb, w->sel, w->done, w->its,
                                                        w->status, w->sysv, w->nsys, w->part, p->krylov_maxit, spart, sys_sl_off), ++g_launches;
  if (view.act) amg_act_compact(m, w->sel, w->done, &g_launches);
  UA_CUDA_TRY(cudaGetLastError());
  const int chunk = 16;
  // one PCG iteration for every selected, unfinished system
  auto iteration = [&]() -> int {
    cudaEvent_t ev[2];
    prof_begin(m, PK_SPMV, ev);
    if (view.sell)
      amg_sell_spmv(m, fp32, view.act, w->sel, w->done, pp, w->cmask, q, &g_launches);
    else {
      dispatch_lpr(lpr, [&](auto L) {
        if (uvlay)
          k_pcg_spmv<KT, VT, decltype(L)::value, true><<<grid0, 256, 0, m->stream>>>(
              w->rb_start, w->rb_sys, w->nrb, act0, w->sel, w->done, w->rowptr, w->colind, K, pp, w->cmask, q,
              w->part, m->dm.sys_dof_off);
        else
          k_pcg_spmv<KT, VT, decltype(L)::value, false><<<grid0, 256, 0, m->stream>>>(
              w->rb_start, w->rb_sys, w->nrb, act0, w->sel, w->done, w->rowptr, w->colind, K, pp, w->cmask, q,
              w->part, nullptr);
      });
      ++g_launches;
    }
    prof_end(m, ev);
    launch_pdl(k_pcg_reduce, w->nsys, kRedThreads, 0, m->stream, 1, w->sys_rb_off, w->nrb, w->sel, w->done, w->its,
                                                          w->status, w->sysv, w->nsys, w->part, p->krylov_maxit, spart, sys_sl_off), ++g_launches;
    if (w->npair)
      launch_pdl(k_pair_project<VT>, npb, 256, 0, m->stream, w->npair, w->pair_rows, w->con_dof, w->con_sys, w->sel,
                                                     w->done, cp, q), ++g_launches;
    launch_pdl(k_pcg_update1<VT>, grid0, 256, 0, m->stream, w->rb_start, w->rb_sys, w->nrb, act0, w->sel, w->done, w->sysv,
                                                     w->nsys, w->dX, r, zj, pp, q, invd, w->part), ++g_launches;
    if (amg) {
      int rc = amg_vcycle(m, fp32, view, &g_launches);
      if (rc) return rc;
      if (w->npair)
        launch_pdl(k_pair_project<VT>, npb, 256, 0, m->stream, w->npair, w->pair_rows, w->con_dof, w->con_sys, w->sel,
                                                       w->done, cp, z), ++g_launches;
    }
    launch_pdl(k_pcg_reduce, w->nsys, kRedThreads, 0, m->stream, 2, w->sys_rb_off, w->nrb, w->sel, w->done, w->its,
                                                          w->status, w->sysv, w->nsys, w->part, p->krylov_maxit, spart, sys_sl_off), ++g_launches;
    if (view.act) amg_act_compact(m, w->sel, w->done, &g_launches);
    launch_pdl(k_pcg_update2<VT>, grid0, 256, 0, m->stream, w->rb_start, w->rb_sys, act0, w->sel, w->done, w->sysv,
                                                     w->nsys, pp, z), ++g_launches;
    return UA_OK;
  };
  // A chunk of iterations is captured once per (handle, precision, preconditioner) as a CUDA
  // graph and replayed: every argument is a fixed device buffer of the handle, and systems that
  // have converged skip their rows on the device (done[s]), so a replay equals the launches.
  const bool graph = !w->no_graph && !p->profile && w->npair == 0;
  const int gk = (fp32 ? 2 : 0) + (amg ? 1 : 0) + (view.K0lo || view.sell_lo ? 4 : 0) + (view.act ? 8 : 0) +
                 (view.sell ? 16 : 0);
  if (graph && w->pcg_exec[gk] && (w->pcg_exec_maxit[gk] != p->krylov_maxit || w->pcg_exec_lpr[gk] != lpr)) {
    cudaGraphExecDestroy(w->pcg_exec[gk]);
    w->pcg_exec[gk] = nullptr;
  }
  if (graph && !w->pcg_exec[gk]) {
    const long long l0 = g_launches;
    cudaGraph_t gr = nullptr;
    UA_CUDA_TRY(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
    int rc = UA_OK;
    for (int k = 0; k < chunk && rc == UA_OK; ++k) rc = iteration();
    cudaError_t ce = cudaStreamEndCapture(m->stream, &gr);
    if (rc) { if (gr) cudaGraphDestroy(gr); return rc; }
    if (ce != cudaSuccess) return set_error(UA_ERR_CUDA, "PCG graph capture: %s", cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&w->pcg_exec[gk], gr, 0);
    cudaGraphDestroy(gr);
    if (ce != cudaSuccess) return set_error(UA_ERR_CUDA, "PCG graph instantiation: %s", cudaGetErrorString(ce));
    w->pcg_exec_nodes[gk] = g_launches - l0;
    w->pcg_exec_maxit[gk] = p->krylov_maxit;
    w->pcg_exec_lpr[gk] = lpr;
    g_launches = l0;  // capture launches nothing
  }
  int it = 0;
  while (true) {
    if (graph) {
      UA_CUDA_TRY(cudaGraphLaunch(w->pcg_exec[gk], m->stream));
      g_launches += w->pcg_exec_nodes[gk];
    } else {
      for (int k = 0; k < chunk; ++k) {
        int rc = iteration();
        if (rc) return rc;
      }
    }
    it += chunk;
    UA_CUDA_TRY(cudaGetLastError());
    UA_CUDA_TRY(cudaMemcpyAsync(w->h_int, w->done, w->nsys * sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    bool all = true;
    for (int s = 0; s < w->nsys; ++s) all = all && (w->h_int[s] || !its_out[s]);
    if (all || it >= p->krylov_maxit + chunk) break;
  }
  prof_end(m, kev);
  if (w->nc)
    k_con_multiplier<KT><<<(w->nc + 255) / 256, 256, 0, m->stream>>>(w->nc, w->con_dof, w->con_sys, w->sel,
                                                                     w->rowptr, w->colind, K, w->dX, w->frhs,
                                                                     w->dlam, con_pairs(w)), ++g_launches;
  UA_CUDA_TRY(cudaMemcpyAsync(w->h_int, w->its, w->nsys * sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  for (int s = 0; s < w->nsys; ++s) its_out[s] = its_out[s] ? w->h_int[s] : 0;
  return UA_OK;
}

// Solve [K L';L 0][dX;dl] = [frhs;grhs] for the selected systems (sel set on device,
// its_out[s] != 0 marks selected on input).
static int linear_solve(ua_mesh* m, const ua_params* p, std::vector<int>& its_out, const double* eta) {
  Work* w = m->work;
  if (p->precision == UA_PREC_MIXED) return pcg_t<float, float>(m, p, w->Kf, its_out.data(), eta);
  return pcg_t<double, double>(m, p, w->Kd, its_out.data(), eta);
}

// Inner tolerance of Newton iteration with cost rForce: the forcing term
// eta = c*sqrt(rForce) (relative residual ~ ||[f;g]||/||fext0||), clamped to
// [krylov_rtol, max] (defaults c = 0.5, max = 0.1, the fastest safe pair of a
// sweep on B200); krylov_rtol itself when adaptive tolerances are off.
static double forcing_term(const ua_params* p, double rForce) {
  if (!p->krylov_adaptive || !(rForce == rForce)) return p->krylov_rtol;
  const double c = p->krylov_eta_c > 0 ? p->krylov_eta_c : 0.5;
  const double hi = p->krylov_eta_max > 0 ? p->krylov_eta_max : 0.1;
  return std::min(hi, std::max(p->krylov_rtol, c * std::sqrt(std::max(rForce, 0.0))));
}

// The uvh step always takes the line search (SSTREAM_TransientImplicit.m:418) and its cost
// mixes momentum and mass-conservation rows, which loose directions stall: the uvh forcing
// term stays at or below 1e-6 (1e-3 sqrt(rForce), clamped to [krylov_rtol, 1e-6]).
static double forcing_term_uvh(const ua_params* p, double rForce) {
  if (!p->krylov_adaptive || !(rForce == rForce)) return p->krylov_rtol;
  return std::min(1e-6, std::max(p->krylov_rtol, 1e-3 * std::sqrt(std::max(rForce, 0.0))));
}

// uvResidualsCriteria.m:1-23
static bool residual_criteria(const ua_params* p, double rForce, double rWork, int iteration, double gamma) {
  const double *a, *o;
  if (gamma > std::max(p->uvExitBackTrackingStepLength, p->BacktrackingGammaMin)) {
    a = p->uvDesiredWorkAndForceTolerances; o = p->uvDesiredWorkOrForceTolerances;
  } else {
    a = p->uvAcceptableWorkAndForceTolerances; o = p->uvAcceptableWorkOrForceTolerances;
  }
  return (rWork < a[0] && rForce < a[1]) && (rWork < o[0] || rForce < o[1]) && iteration >= p->NRitmin;
}

struct SysState {
  bool active = false, converged = false;
  int iteration = 0, iarm = 0;
  double r = 0, rForce = 0, rWork = 0, gamma = 1, ResidualReduction = 1e10;
  double r0 = 0, rForce0 = 0, rWork0 = 0, r1 = 0, rForce1 = 0, rWork1 = 0;
  int kits = 0;
  // K and R in the work buffers are those of the current iterate (assembled ahead, at the
  // cost evaluation that found the iterate), so the next Newton system needs no assembly
  bool kfresh = false;
  // line search
  bool in_ls = false;
  BackTrack bt;
  std::vector<double> ls_g, ls_rF, ls_D2;
};

// Per-slot state of the serving loop (ua_serve_*).
struct ServeState {
  std::vector<SysState> st;
  std::vector<ua_newton_report> rep;
  std::vector<std::vector<ua_newton_iter>> recs;
  std::vector<int> retried, busy;
  double t_asm = 0, t_sol = 0;
};

static double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Tangent assembled ahead: the cost evaluations at the start iterate and at the full Newton
// step (gamma = 1) assemble K with R.  When the point becomes the next iterate (the start, or a
// full step accepted without backtracking) the next Newton system needs no assembly: K and R
// at X_k + 1.0 dX_k are the ones an assembly at X_{k+1} gives, bit for bit.  Off when the
// caller reads the last Newton system's tangent back, and for the modified Newton variant
// (ModifiedNRuvIntervalCriterion > 1) that keeps old tangents.
static bool tangent_ahead(const ua_mesh* m, const ua_params* p) {
  return !m->keep_last_tangent && p->ModifiedNRuvIntervalCriterion <= 1;
}

// Start the Newton solve of the systems with run[s]=1 (SSTREAM2dNR2.m:100-156):
// make the iterate feasible, fext0 at ZeroFields, cost at the start iterate.
// Other systems are left untouched, so a system can join while others iterate.
static int newton_init(ua_mesh* m, const ua_params* p, const std::vector<int>& run, std::vector<SysState>& st) {
  Work* w = m->work;
  const int nsys = w->nsys;
  int rc;
  // make the iterate feasible (:101-104) and compute fext0 at ZeroFields (:122-124)
  UA_CUDA_TRY(cudaMemsetAsync(w->X0, 0, m->ndof_total * sizeof(double), m->stream));
  if ((rc = set_sel(m, run))) return rc;
  amg_restart_P(m, run);  // a new solve: its first AMG set-up recomputes the prolongators
  if (w->nc) {
    k_set_con_values<<<(w->nc + 255) / 256, 256, 0, m->stream>>>(w->nc, w->con_dof, w->con_sys, w->sel,
                                                                 w->con_rhs, w->X, con_pairs(w)), ++g_launches;
    k_set_con_values<<<(w->nc + 255) / 256, 256, 0, m->stream>>>(w->nc, w->con_dof, w->con_sys, w->sel,
                                                                 w->con_rhs, w->X0, con_pairs(w)), ++g_launches;
  }
  {
    if ((rc = assemble(m, p, false, false, w->X0, false))) return rc;
    k_cost_rows<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->R, nullptr, nullptr,
                                               nullptr, nullptr, nullptr, w->part, nullptr, ConPairs{}), ++g_launches;
    k_cost_reduce<<<nsys, kRedThreads, 0, m->stream>>>(w->sys_rb_off, w->nrb, w->sel, w->part, nsys, w->sysv,
                                                       nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                                       nullptr, 1, con_pairs(w)), ++g_launches;
    UA_CUDA_TRY(cudaGetLastError());
  }
  // initial cost (:149-152) with zero direction
  UA_CUDA_TRY(cudaMemsetAsync(w->dX, 0, m->ndof_total * sizeof(double), m->stream));
  if (w->nc) UA_CUDA_TRY(cudaMemsetAsync(w->dlam, 0, w->nc * sizeof(double), m->stream));
  const bool ahead = tangent_ahead(m, p);
  if ((rc = cost_eval(m, p, false, true, ahead))) return rc;
  for (int s = 0; s < nsys; ++s) {
    if (!run[s]) continue;
    st[s] = SysState();
    st[s].kfresh = ahead;
    st[s].active = true;
    st[s].r = st[s].rForce = w->h_sysv[SV_FF * nsys + s];
    st[s].rWork = 0;
    st[s].gamma = 1;
  }
  return UA_OK;
}

// Clears a report, keeping the caller-owned record and update buffers.
static void reset_report(ua_newton_report* r) {
  const int cap = r->iters_capacity;
  ua_newton_iter* it = r->iters;
  double* up = r->updates;
  const int64_t stride = r->update_stride;
  int32_t* hp = r->hpos_node;
  const int hcap = r->hpos_capacity;
  std::memset(r, 0, sizeof(*r));
  r->iters_capacity = cap;
  r->iters = it;
  r->updates = up;
  r->update_stride = stride;
  r->hpos_node = hp;
  r->hpos_capacity = hcap;
}

// A caller-owned update buffer must hold ndof*Nnodes + nl doubles per record.
static int check_update_stride(const ua_mesh* m, const std::vector<ua_newton_report*>& rep) {
  const Work* w = m->work;
  for (size_t s = 0; s < rep.size(); ++s) {
    const ua_newton_report* r = rep[s];
    if (!r || !r->updates) continue;
    const int64_t need = (int64_t)(m->h_dof_off[s + 1] - m->h_dof_off[s]) +
                         (w->h_sys_con_off[s + 1] - w->h_sys_con_off[s]);
    if (r->update_stride < need)
      return set_error(UA_ERR_INVALID, "update_stride %lld of system %d is below ndof*Nnodes + nl = %lld",
                       (long long)r->update_stride, (int)s, (long long)need);
  }
  return UA_OK;
}

// Copies the accepted update gamma*[dX; dlam] of each system updated in this
// iteration (sel[s]) into record n_iter_records-1 of its caller-owned buffer
// (SSTREAM2dNR2.m:367-369).  The product by gamma is the one the update kernel
// applies, so record and iterate agree bit for bit.
static int record_updates(ua_mesh* m, const std::vector<ua_newton_report*>& rep, const std::vector<int>& sel,
                          const std::vector<double>& gam) {
  Work* w = m->work;
  bool any = false;
  for (size_t s = 0; s < rep.size(); ++s) {
    ua_newton_report* r = rep[s];
    if (!sel[s] || !r || !r->updates || r->n_iter_records <= 0 || r->n_iter_records > r->iters_capacity) continue;
    double* dst = r->updates + (int64_t)(r->n_iter_records - 1) * r->update_stride;
    const int d0 = m->h_dof_off[s], nd = m->h_dof_off[s + 1] - d0;
    const int c0 = w->h_sys_con_off[s], nc = w->h_sys_con_off[s + 1] - c0;
    UA_CUDA_TRY(cudaMemcpyAsync(dst, w->dX + d0, nd * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    if (nc) UA_CUDA_TRY(cudaMemcpyAsync(dst + nd, w->dlam + c0, nc * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    any = true;
  }
  if (!any) return UA_OK;
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  for (size_t s = 0; s < rep.size(); ++s) {
    ua_newton_report* r = rep[s];
    if (!sel[s] || !r || !r->updates || r->n_iter_records <= 0 || r->n_iter_records > r->iters_capacity) continue;
    double* dst = r->updates + (int64_t)(r->n_iter_records - 1) * r->update_stride;
    const int n = (m->h_dof_off[s + 1] - m->h_dof_off[s]) + (w->h_sys_con_off[s + 1] - w->h_sys_con_off[s]);
    for (int i = 0; i < n; ++i) dst[i] = gam[s] * dst[i];
  }
  return UA_OK;
}

// One Newton iteration (SSTREAM2dNR2.m:157-392) of every active system.
// *any is false when no system was active.
static int newton_step(ua_mesh* m, const ua_params* p, std::vector<ua_newton_report*>& rep,
                       std::vector<SysState>& st, double& t_asm, double& t_sol, bool* any_out) {
  Work* w = m->work;
  const int nsys = w->nsys;
  int rc;
  std::vector<int> sel(nsys), its(nsys);
  std::vector<double> gam(nsys, 0.0);
  {
    // convergence / iteration cap (:160-190)
    bool any = false;
    for (int s = 0; s < nsys; ++s) {
      SysState& S = st[s];
      if (!S.active) continue;
      if (residual_criteria(p, S.rForce, S.rWork, S.iteration, S.gamma)) { S.converged = true; S.active = false; continue; }
      if (S.iteration > p->NRitmax) { S.converged = false; S.active = false; continue; }
      S.iteration++;
      any = true;
    }
    *any_out = any;
    if (!any) return UA_OK;
    for (int s = 0; s < nsys; ++s) sel[s] = st[s].active ? 1 : 0;
    if ((rc = set_sel(m, sel))) return rc;
    // R and K (:197-213); the interval criterion 1 (default) always refreshes K
    double t0 = now_ms();
    bool refreshK = false;
    for (int s = 0; s < nsys; ++s)
      if (st[s].active && (((st[s].iteration - 1) % std::max(1, p->ModifiedNRuvIntervalCriterion)) == 0 ||
                           st[s].ResidualReduction > p->ModifiedNRuvReductionCriterion))
        refreshK = true;
    const bool ahead = tangent_ahead(m, p);
    std::vector<int> asel(nsys);
    int n_asm = 0, n_fresh = 0;
    for (int s = 0; s < nsys; ++s) {
      asel[s] = sel[s] && !(ahead && st[s].kfresh);
      n_asm += asel[s];
      n_fresh += sel[s] && !asel[s];
      st[s].kfresh = false;
    }
    if (n_fresh == 0) {
      if ((rc = assemble(m, p, refreshK, false, w->X, false))) return rc;
    } else if (n_asm > 0) {  // only the systems whose K and R were not assembled ahead
      if ((rc = set_sel(m, asel))) return rc;
      if ((rc = assemble(m, p, refreshK, false, w->X, false))) return rc;
      if ((rc = set_sel(m, sel))) return rc;
    }
    k_frhs<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->sel, w->R, w->dof_con, w->lam, w->frhs, w->con_dof, con_pairs(w)), ++g_launches;
    UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    double t1 = now_ms();
    t_asm += t1 - t0;
    // linear solve (:242-257)
    for (int s = 0; s < nsys; ++s) its[s] = sel[s];
    std::vector<double> eta(nsys);
    for (int s = 0; s < nsys; ++s) eta[s] = forcing_term(p, st[s].rForce);
    if ((rc = linear_solve(m, p, its, eta.data()))) return rc;
    double t2 = now_ms();
    t_sol += t2 - t1;
    for (int s = 0; s < nsys; ++s) if (sel[s]) st[s].kits = its[s];
    // gamma=0 (:260-283): R at X is the residual assembled with K above
    for (int s = 0; s < nsys; ++s) gam[s] = 0.0;
    if ((rc = set_gamma(m, gam))) return rc;
    if ((rc = cost_eval(m, p, true, false))) return rc;
    for (int s = 0; s < nsys; ++s) {
      if (!sel[s]) continue;
      SysState& S = st[s];
      S.r0 = S.rForce0 = w->h_sysv[SV_FF * nsys + s];
      double D2 = w->h_sysv[SV_FD * nsys + s];
      S.rWork0 = D2 * D2;
      if (S.iteration == 1 && residual_criteria(p, S.rForce0, S.rWork0, S.iteration, 1.0)) {
        S.iteration -= 1; S.converged = true; S.active = false; sel[s] = 0;
      }
    }
    // gamma=1 (:288), with the tangent there when it is assembled ahead
    for (int s = 0; s < nsys; ++s) gam[s] = 1.0;
    if ((rc = set_sel(m, sel))) return rc;
    if ((rc = set_gamma(m, gam))) return rc;
    if ((rc = cost_eval(m, p, true, true, ahead))) return rc;
    for (int s = 0; s < nsys; ++s) {
      if (!sel[s]) continue;
      SysState& S = st[s];
      S.r1 = S.rForce1 = w->h_sysv[SV_FF * nsys + s];
      double D2 = w->h_sysv[SV_FD * nsys + s];
      S.rWork1 = D2 * D2;
      if (S.r1 / S.r0 < p->NewtonAcceptRatio) {  // :290-296
        S.in_ls = false;
        S.kfresh = ahead;
        S.gamma = 1.0; S.r = S.r1; S.rForce = S.rForce1; S.rWork = S.rWork1; S.iarm = 0;
      } else {  // rLineminUa.m:57-135 (Newton-direction backtracking)
        S.in_ls = true;
        S.bt = BackTrack();
        BTConfig& c = S.bt.cfg;
        c.beta = p->BackTrackBeta; c.ExtrapolationRatio = p->BackTrackExtrapolationRatio;
        c.MinXfracRel = p->BackTrackMinXfrac; c.GL = p->BackTrackGuardLower; c.GU = p->BackTrackGuardUpper;
        c.NewtonAcceptRatio = p->NewtonAcceptRatio; c.GammaMin = 0.001; c.NLtol = p->NLtol;
        c.MaxIterations = p->BackTrackMaxIterations; c.MaxExtrapolations = p->BackTrackMaxExtrapolations;
        c.MaxFuncSame = p->BackTrackMaxFuncSame; c.allow_ext = p->LineSearchAllowedToUseExtrapolation != 0;
        S.ls_g.assign({0.0, 1.0});
        S.ls_rF.assign({S.rForce0, S.rForce1});
        S.ls_D2.assign({std::sqrt(S.rWork0), std::sqrt(S.rWork1)});
        S.bt.start(-2 * S.r0, 1.0, S.r0, S.r1);
      }
    }
    // line-search rounds
    while (true) {
      bool need = false;
      for (int s = 0; s < nsys; ++s) {
        sel[s] = (st[s].active && st[s].in_ls && !st[s].bt.done) ? 1 : 0;
        gam[s] = sel[s] ? st[s].bt.request : 0.0;
        need = need || sel[s];
      }
      if (!need) break;
      if ((rc = set_sel(m, sel))) return rc;
      if ((rc = set_gamma(m, gam))) return rc;
      if ((rc = cost_eval(m, p, true))) return rc;
      for (int s = 0; s < nsys; ++s) {
        if (!sel[s]) continue;
        double rf = w->h_sysv[SV_FF * nsys + s], d2 = w->h_sysv[SV_FD * nsys + s];
        st[s].ls_g.push_back(gam[s]); st[s].ls_rF.push_back(rf); st[s].ls_D2.push_back(d2);
        st[s].bt.feed(rf);
      }
    }
    // finish line searches, update (:313-371)
    for (int s = 0; s < nsys; ++s) {
      sel[s] = 0;
      SysState& S = st[s];
      if (!S.active) continue;
      int bt_conv = 1;
      if (S.in_ls) {
        BackTrack& bt = S.bt;
        double gN = bt.gmin, rN = bt.fmin;
        if (rep[s] && gN < 0.75 && rN / S.r0 > 0.7) rep[s]->cauchy_fallbacks++;  // rLineminUa.m:96
        S.iarm = bt.iarm;
        bt_conv = bt.converged && !bt.error;
        if (rN < S.r0) {
          S.gamma = gN; S.r = rN; S.rForce = rN;
          S.rWork = std::nan("");
          for (size_t k = 0; k < S.ls_g.size(); ++k)
            if (S.ls_g[k] == gN) { S.rWork = S.ls_D2[k] * S.ls_D2[k]; break; }
        } else {
          S.gamma = 0; S.r = S.r0; S.rForce = S.r0; S.rWork = std::nan("");
        }
      }
      if (rep[s] && rep[s]->iters && rep[s]->n_iter_records < rep[s]->iters_capacity) {
        ua_newton_iter& it = rep[s]->iters[rep[s]->n_iter_records++];
        it.iteration = S.iteration; it.iarm = S.iarm; it.krylov_its = S.kits; it.direction = S.in_ls ? 1 : 0;
        it.gamma = S.gamma; it.r0 = S.r0; it.r = S.r; it.rForce = S.rForce; it.rWork = S.rWork;
      }
      if (rep[s]) rep[s]->krylov_its_total += S.kits;
      if (p->verbose)
        fprintf(stderr, "NR-SSTREAM(uv)[%d]:%3d/%-2d g=%-14.7g , r/r0=%-14.7g ,  r0=%-14.7g , r=%-14.7g , rForce=%-14.7g , rWork=%-14.7g , pcg=%d\n",
                s, S.iteration, S.iarm, S.gamma, S.r / S.r0, S.r0, S.r, S.rForce, S.rWork, S.kits);
      if (!bt_conv) { S.converged = false; S.active = false; continue; }  // :322-327
      sel[s] = 1;
      gam[s] = S.gamma;
      S.ResidualReduction = S.r / S.r0;
    }
    if ((rc = set_sel(m, sel))) return rc;
    if ((rc = set_gamma(m, gam))) return rc;
    k_newton_update<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->sel, w->gamma, w->X, w->dX), ++g_launches;
    if (w->nc)
      k_lam_update<<<(w->nc + 255) / 256, 256, 0, m->stream>>>(w->nc, w->con_sys, w->sel, w->gamma, w->lam,
                                                               w->dlam), ++g_launches;
    UA_CUDA_TRY(cudaGetLastError());
    if ((rc = record_updates(m, rep, sel, gam))) return rc;
  }
  return UA_OK;
}

// Newton driver for the systems with run[s]=1 (SSTREAM2dNR2.m:100-392).
static int newton_run(ua_mesh* m, const ua_params* p, std::vector<int> run, std::vector<ua_newton_report*>& rep,
                      std::vector<SysState>& st) {
  Work* w = m->work;
  const int nsys = w->nsys;
  double t_asm = 0, t_sol = 0;
  int rc;
  if ((rc = newton_init(m, p, run, st))) return rc;
  for (int s = 0; s < nsys; ++s)
    if (!run[s]) st[s].active = false;
  bool any = true;
  while (any)
    if ((rc = newton_step(m, p, rep, st, t_asm, t_sol, &any))) return rc;
  for (int s = 0; s < nsys; ++s) {
    if (!run[s] || !rep[s]) continue;
    rep[s]->converged = st[s].converged ? 1 : 0;
    rep[s]->iterations = st[s].iteration;
    rep[s]->backtrack_steps = st[s].iarm;
    rep[s]->r = st[s].r; rep[s]->rForce = st[s].rForce; rep[s]->rWork = st[s].rWork;
    rep[s]->assembly_ms += t_asm; rep[s]->solve_ms += t_sol;
  }
  return UA_OK;
}

// ---------------------------------------------------------------------------
// BiCGStab for the unsymmetric uvh tangent (the reference's solveKApe ->
// ABfgPreEliminate direct solve, SSTREAM_TransientImplicit.m:136), Jacobi
// right-preconditioned, on the free dofs; constrained dofs are masked as in
// the PCG.  Per-system scalars, deterministic reductions.
// ---------------------------------------------------------------------------

// y = mask(K x); partials: a.y (a may be null), y.y
template <typename KT, int LPR>
__global__ void __launch_bounds__(256) k_bicg_spmv(const int* rb_start, const int* rb_sys, int nrb, const int* sel,
                                                   const int* done, const int* rowptr, const int* colind,
                                                   const KT* K, const double* x, const unsigned char* cmask,
                                                   double* y, const double* a, double* part) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  double v[2] = {0, 0};
  if (sel[s] && !done[s]) {
    const int rs = rb_start[blk], re = rb_start[blk + 1];
    const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR, ngrp = blockDim.x / LPR;
    for (int row0 = rs; row0 < re; row0 += ngrp) {
      const int row = row0 + grp;
      const bool valid = row < re;
      double ax = row_dot<KT, double, LPR>(rowptr, colind, K, x, row, valid, lane);
      if (valid && lane == 0) {
        const double yv = cmask[row] ? 0.0 : ax;
        y[row] = yv;
        if (a) v[0] += a[row] * yv;
        v[1] += yv * yv;
      }
    }
  }
  block_partials<2>(v, part, nrb, blk);
}

// r = mask(f - K x0), rhat = r, p = v = 0; partials rhat.r, r.r
template <typename KT, int LPR>
__global__ void __launch_bounds__(256) k_bicg_init(const int* rb_start, const int* rb_sys, int nrb, const int* sel,
                                                   const int* rowptr, const int* colind, const KT* K,
                                                   const double* x0, const double* f, const unsigned char* cmask,
                                                   double* r, double* rhat, double* p, double* vv, double* part) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  double v[2] = {0, 0};
  if (sel[s]) {
    const int rs = rb_start[blk], re = rb_start[blk + 1];
    const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR, ngrp = blockDim.x / LPR;
    for (int row0 = rs; row0 < re; row0 += ngrp) {
      const int row = row0 + grp;
      const bool valid = row < re;
      double ax = row_dot<KT, double, LPR>(rowptr, colind, K, x0, row, valid, lane);
      if (valid && lane == 0) {
        const double rv = cmask[row] ? 0.0 : f[row] - ax;
        r[row] = rv; rhat[row] = rv; p[row] = 0; vv[row] = 0;
        v[0] += rv * rv;
        v[1] += rv * rv;
      }
    }
  }
  block_partials<2>(v, part, nrb, blk);
}

// out = invd in (point-Jacobi preconditioner), selected unfinished systems
__global__ void __launch_bounds__(256) k_scale_vec(const int* rb_start, const int* rb_sys, const int* sel,
                                                   const int* done, const double* in, const double* invd,
                                                   double* out) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s] || done[s]) return;
  for (int i = rb_start[blk] + threadIdx.x; i < rb_start[blk + 1]; i += blockDim.x) out[i] = invd[i] * in[i];
}

// p = r + beta (p - omega v), phat = invd p; after a breakdown (restart pending, beta = 0)
// the shadow residual restarts from the current residual: rhat = r.
__global__ void __launch_bounds__(256) k_bicg_p(const int* rb_start, const int* rb_sys, const int* sel,
                                                const int* done, const double* sysv, int nsys, const double* r,
                                                double* p, const double* vv, const double* invd, double* phat,
                                                double* rhat) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s] || done[s]) return;
  const double beta = sysv[SV_BETA * nsys + s], omega = sysv[SV_OMEGA * nsys + s];
  const bool restart = sysv[SV_RST * nsys + s] != 0.0;
  for (int i = rb_start[blk] + threadIdx.x; i < rb_start[blk + 1]; i += blockDim.x) {
    const double pv = r[i] + beta * (p[i] - omega * vv[i]);
    p[i] = pv;
    phat[i] = invd[i] * pv;
    if (restart) rhat[i] = r[i];
  }
}

// s = r - alpha v; shat = invd s
__global__ void __launch_bounds__(256) k_bicg_s(const int* rb_start, const int* rb_sys, const int* sel,
                                                const int* done, const double* sysv, int nsys, const double* r,
                                                const double* vv, const double* invd, double* sv, double* shat) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s] || done[s]) return;
  const double alpha = sysv[SV_ALPHA * nsys + s];
  for (int i = rb_start[blk] + threadIdx.x; i < rb_start[blk + 1]; i += blockDim.x) {
    const double x = r[i] - alpha * vv[i];
    sv[i] = x;
    shat[i] = invd[i] * x;
  }
}

// x += alpha phat + omega shat; r = s - omega t; partials rhat.r, r.r
__global__ void __launch_bounds__(256) k_bicg_x(const int* rb_start, const int* rb_sys, int nrb, const int* sel,
                                                const int* done, const double* sysv, int nsys, double* x,
                                                const double* phat, const double* shat, const double* sv,
                                                const double* t, double* r, const double* rhat, double* part) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  double v[2] = {0, 0};
  if (sel[s] && !done[s]) {
    const double alpha = sysv[SV_ALPHA * nsys + s], omega = sysv[SV_OMEGA * nsys + s];
    for (int i = rb_start[blk] + threadIdx.x; i < rb_start[blk + 1]; i += blockDim.x) {
      x[i] += alpha * phat[i] + omega * shat[i];
      const double rv = sv[i] - omega * t[i];
      r[i] = rv;
      v[0] += rhat[i] * rv;
      v[1] += rv * rv;
    }
  }
  block_partials<2>(v, part, nrb, blk);
}

// stage 0: init (rho, rr0); 1: alpha = rho/(rhat.v); 2: omega = (t.s)/(t.t); 3: rho, beta, convergence
__global__ void k_bicg_reduce(int stage, const int* sys_rb_off, int nrb, const int* sel, int* done, int* its,
                              int* status, double* sysv, int nsys, const double* part, int maxit) {
  const int s = blockIdx.x;
  if (!sel[s] || (stage > 0 && done[s])) return;
  double o[2];
  sys_sum<2>(part, nrb, sys_rb_off[s], sys_rb_off[s + 1], o);
  if (threadIdx.x != 0) return;
  double* sv = sysv;
  if (stage == 0) {
    sv[SV_RZ * nsys + s] = o[0];
    sv[SV_RR0 * nsys + s] = o[1];
    sv[SV_RR * nsys + s] = o[1];
    sv[SV_ALPHA * nsys + s] = 1.0;
    sv[SV_OMEGA * nsys + s] = 1.0;
    sv[SV_BETA * nsys + s] = 0.0;  // first direction p = r
    sv[SV_RH * nsys + s] = o[1];   // rhat = r
    sv[SV_RST * nsys + s] = 0.0;
    sv[SV_NRST * nsys + s] = 0.0;
    its[s] = 0;
    status[s] = 0;
    done[s] = (o[1] == 0.0) ? 1 : 0;
  } else if (stage == 1) {
    const double rv = o[0];
    sv[SV_RST * nsys + s] = 0.0;  // every block of k_bicg_p has consumed a pending restart
    if (rv == 0.0 || !(rv == rv)) { status[s] = 1; done[s] = 1; sv[SV_ALPHA * nsys + s] = 0; return; }
    sv[SV_ALPHA * nsys + s] = sv[SV_RZ * nsys + s] / rv;
  } else if (stage == 2) {
    // partials: [0] = s.t, [1] = t.t
    sv[SV_OMEGA * nsys + s] = o[1] > 0 ? o[0] / o[1] : 0.0;
  } else {
    const double rho_new = o[0], rr = o[1];
    its[s] += 1;
    sv[SV_RR * nsys + s] = rr;
    const double omega = sv[SV_OMEGA * nsys + s];
    if (rr <= sv[SV_TOL2 * nsys + s] * sv[SV_RR0 * nsys + s] || its[s] >= maxit || !(rr == rr)) {
      done[s] = 1;
    } else if (omega == 0.0 || fabs(rho_new) <= 1e-12 * sqrt(sv[SV_RH * nsys + s] * rr)) {
      // breakdown (rhat nearly orthogonal to r, or a zero stabilisation step): restart from the
      // current residual with rhat = r, p = r, a bounded number of times
      if (sv[SV_NRST * nsys + s] >= kBicgMaxRestarts) { status[s] = 1; done[s] = 1; return; }
      sv[SV_NRST * nsys + s] += 1.0;
      sv[SV_RST * nsys + s] = 1.0;
      sv[SV_BETA * nsys + s] = 0.0;
      sv[SV_RZ * nsys + s] = rr;
      sv[SV_RH * nsys + s] = rr;
    } else {
      sv[SV_BETA * nsys + s] = (rho_new / sv[SV_RZ * nsys + s]) * (sv[SV_ALPHA * nsys + s] / omega);
      sv[SV_RZ * nsys + s] = rho_new;
    }
  }
}

// (s.t) partials: the spmv kernel gives a.y with a = s
template <typename KT>
static int bicgstab_t(ua_mesh* m, const ua_params* p, const KT* K, int* its_out, const double* eta = nullptr) {
  Work* w = m->work;
  const int N = m->ndof_total;
  const int lpr = 16;
  if (w->npair)
    return set_error(UA_ERR_INVALID, "tied nodes and fixed normal velocities need the GMRES uvh solver "
                                     "(uvh_krylov = UA_KRYLOV_GMRES)");
  for (int s = 0; s < w->nsys; ++s) {
    const double e = eta ? eta[s] : p->krylov_rtol;
    w->h_sysv[s] = e * e;
  }
  UA_CUDA_TRY(cudaMemcpyAsync(w->sysv + SV_TOL2 * w->nsys, w->h_sysv, w->nsys * sizeof(double),
                              cudaMemcpyHostToDevice, m->stream));
  double *r = (double*)w->kr, *rhat = (double*)w->krh, *pp = (double*)w->kp, *phat = (double*)w->kz;
  double *vv = (double*)w->kq, *sv = (double*)w->ks, *shat = (double*)w->ksh, *t = (double*)w->kt;
  double* invd = (double*)w->invd;
  k_invdiag<KT, double><<<(N + 255) / 256, 256, 0, m->stream>>>(N, K, w->diagpos, w->cmask, invd), ++g_launches;
  // block preconditioner: the aggregation-AMG V-cycle of the velocity block on the u, v rows,
  // point Jacobi on the h rows (the coupling blocks are left to the Krylov iteration)
  bool amg = p->krylov_precond == UA_PC_AMG && m->ndof == 3 && !m->h_nodeptr.empty() && sizeof(KT) == 8;
  if (amg && amg_setup(m, p->amg_smoothed != 0) != UA_OK) amg = false;
  if (amg) {
    int rc = amg_numeric_uvh(m, (const double*)K, w->cmask, &g_launches);
    if (rc) return rc;
  }
  const int lpr_uv = m->nod == 3 ? 1 : 2;
  k_zero_sel<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->sel, w->dX), ++g_launches;
  if (w->nc)
    k_con_particular<<<(w->nc + 255) / 256, 256, 0, m->stream>>>(w->nc, w->con_dof, w->con_sys, w->sel, w->con_rhs,
                                                                 w->X, w->dX, w->grhs, con_pairs(w)), ++g_launches;
  k_bicg_init<KT, 16><<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->rowptr, w->colind, K,
                                                     w->dX, w->frhs, w->cmask, r, rhat, pp, vv, w->part), ++g_launches;
  k_bicg_reduce<<<w->nsys, kRedThreads, 0, m->stream>>>(0, w->sys_rb_off, w->nrb, w->sel, w->done, w->its, w->status,
                                                         w->sysv, w->nsys, w->part, p->krylov_maxit), ++g_launches;
  UA_CUDA_TRY(cudaGetLastError());
  (void)lpr;
  const int chunk = 8;
  int it = 0;
  while (true) {
    for (int k = 0; k < chunk; ++k) {
      k_bicg_p<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->sel, w->done, w->sysv, w->nsys, r, pp, vv,
                                              invd, phat, rhat), ++g_launches;
      if (amg) {
        int rc = amg_apply_uvh(m, pp, phat, w->sel, w->done, lpr_uv, &g_launches);
        if (rc) return rc;
      }
      cudaEvent_t ev[2];
      prof_begin(m, PK_SPMV, ev);
      k_bicg_spmv<KT, 16><<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->done, w->rowptr,
                                                         w->colind, K, phat, w->cmask, vv, rhat, w->part), ++g_launches;
      prof_end(m, ev);
      k_bicg_reduce<<<w->nsys, kRedThreads, 0, m->stream>>>(1, w->sys_rb_off, w->nrb, w->sel, w->done, w->its,
                                                             w->status, w->sysv, w->nsys, w->part, p->krylov_maxit), ++g_launches;
      k_bicg_s<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->sel, w->done, w->sysv, w->nsys, r, vv, invd,
                                              sv, shat), ++g_launches;
      if (amg) {
        int rc = amg_apply_uvh(m, sv, shat, w->sel, w->done, lpr_uv, &g_launches);
        if (rc) return rc;
      }
      k_bicg_spmv<KT, 16><<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->done, w->rowptr,
                                                         w->colind, K, shat, w->cmask, t, sv, w->part), ++g_launches;
      k_bicg_reduce<<<w->nsys, kRedThreads, 0, m->stream>>>(2, w->sys_rb_off, w->nrb, w->sel, w->done, w->its,
                                                             w->status, w->sysv, w->nsys, w->part, p->krylov_maxit), ++g_launches;
      k_bicg_x<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->done, w->sysv, w->nsys, w->dX,
                                              phat, shat, sv, t, r, rhat, w->part), ++g_launches;
      k_bicg_reduce<<<w->nsys, kRedThreads, 0, m->stream>>>(3, w->sys_rb_off, w->nrb, w->sel, w->done, w->its,
                                                             w->status, w->sysv, w->nsys, w->part, p->krylov_maxit), ++g_launches;
    }
    it += chunk;
    UA_CUDA_TRY(cudaGetLastError());
    UA_CUDA_TRY(cudaMemcpyAsync(w->h_int, w->done, w->nsys * sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    bool all = true;
    for (int s = 0; s < w->nsys; ++s) all = all && (w->h_int[s] || !its_out[s]);
    if (all || it >= p->krylov_maxit + chunk) break;
  }
  if (w->nc)
    k_con_multiplier<KT><<<(w->nc + 255) / 256, 256, 0, m->stream>>>(w->nc, w->con_dof, w->con_sys, w->sel, w->rowptr,
                                                                     w->colind, K, w->dX, w->frhs, w->dlam, con_pairs(w)), ++g_launches;
  UA_CUDA_TRY(cudaMemcpyAsync(w->h_int, w->its, w->nsys * sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  for (int s = 0; s < w->nsys; ++s) its_out[s] = its_out[s] ? w->h_int[s] : 0;
  return UA_OK;
}

// ---------------------------------------------------------------------------
// uvh driver: SSTREAM_TransientImplicit.m:6-717
// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// Restarted GMRES(m) for the unsymmetric uvh system (replaces the direct
// solve of solveKApe.m:104-107 like BiCGStab does), right-preconditioned, all
// systems of the handle in lockstep with per-system Hessenberg matrices on the
// host.  Classical Gram-Schmidt with one re-orthogonalisation pass.
// ---------------------------------------------------------------------------

// part[i*nrb + blk] = block partial of (w, V_i) for i < nv (grid: row blocks x nv)
__global__ void __launch_bounds__(256) k_gm_dots(const int* rb_start, const int* rb_sys, int nrb, const int* sel,
                                                 const int* done, const double* w, const double* V, size_t ldv,
                                                 double* part) {
  const int blk = blockIdx.x, i = blockIdx.y;
  const int s = rb_sys[blk];
  double v[1] = {0};
  if (sel[s] && !done[s]) {
    const double* vi = V + (size_t)i * ldv;
    for (int r = rb_start[blk] + threadIdx.x; r < rb_start[blk + 1]; r += blockDim.x) v[0] += w[r] * vi[r];
  }
  __shared__ double red[8];
  double t = v[0];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sum = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) sum += red[k];
    part[(size_t)i * nrb + blk] = sum;
  }
}

// out[s*ld + i] = sum over the system's row blocks of part[i*nrb + b] (grid: systems x nv)
__global__ void k_gm_reduce(const int* sys_rb_off, int nrb, const int* sel, const int* done, const double* part,
                            double* out, int ld) {
  const int s = blockIdx.x, i = blockIdx.y;
  if (!sel[s] || done[s]) return;
  double o[1];
  sys_sum<1>(part + (size_t)i * nrb, nrb, sys_rb_off[s], sys_rb_off[s + 1], o);
  if (threadIdx.x == 0) out[(size_t)s * ld + i] = o[0];
}

// out = w / sqrt(nrm[s*ld]) per system (0 where the norm is 0)
__global__ void __launch_bounds__(256) k_gm_scale_norm(const int* rb_start, const int* rb_sys, const int* sel,
                                                       const int* done, const double* w, double* out,
                                                       const double* nrm, int ld) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s] || done[s]) return;
  const double hn = sqrt(fmax(nrm[(size_t)s * ld], 0.0));
  const double sc = hn > 0 ? 1.0 / hn : 0.0;
  for (int i = rb_start[blk] + threadIdx.x; i < rb_start[blk + 1]; i += blockDim.x) out[i] = w[i] * sc;
}

// w -= sum_i coef[s*ld + i] V_i (i < nv)
__global__ void __launch_bounds__(256) k_gm_orth(const int* rb_start, const int* rb_sys, const int* sel,
                                                 const int* done, double* w, const double* V, size_t ldv, int nv,
                                                 const double* coef, int ld) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s] || done[s]) return;
  const double* c = coef + (size_t)s * ld;
  for (int r = rb_start[blk] + threadIdx.x; r < rb_start[blk + 1]; r += blockDim.x) {
    double acc = w[r];
    for (int i = 0; i < nv; ++i) acc -= c[i] * V[(size_t)i * ldv + r];
    w[r] = acc;
  }
}

// dst = src * scale[s]
__global__ void __launch_bounds__(256) k_gm_scale(const int* rb_start, const int* rb_sys, const int* sel,
                                                  const int* done, const double* src, double* dst,
                                                  const double* scale) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s] || done[s]) return;
  const double a = scale[s];
  for (int r = rb_start[blk] + threadIdx.x; r < rb_start[blk + 1]; r += blockDim.x) dst[r] = src[r] * a;
}

// u = sum_i y[s*ld + i] V_i for i < ny[s]
__global__ void __launch_bounds__(256) k_gm_combine(const int* rb_start, const int* rb_sys, const int* sel,
                                                    const int* act, double* u, const double* V, size_t ldv,
                                                    const double* y, const int* ny, int ld) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s] || !act[s]) return;
  const double* c = y + (size_t)s * ld;
  const int n = ny[s];
  for (int r = rb_start[blk] + threadIdx.x; r < rb_start[blk + 1]; r += blockDim.x) {
    double acc = 0;
    for (int i = 0; i < n; ++i) acc += c[i] * V[(size_t)i * ldv + r];
    u[r] = acc;
  }
}

// x += z for systems with act[s]
__global__ void __launch_bounds__(256) k_gm_axpy(const int* rb_start, const int* rb_sys, const int* sel,
                                                 const int* act, double* x, const double* z) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s] || !act[s]) return;
  for (int r = rb_start[blk] + threadIdx.x; r < rb_start[blk + 1]; r += blockDim.x) x[r] += z[r];
}

// r = mask(f - K x) and the block partial of r.r (systems with act[s])
template <typename KT, int LPR>
__global__ void __launch_bounds__(256) k_gm_resid(const int* rb_start, const int* rb_sys, int nrb, const int* sel,
                                                  const int* act, const int* rowptr, const int* colind, const KT* K,
                                                  const double* x, const double* f, const unsigned char* cmask,
                                                  double* r, double* part) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  double v[1] = {0};
  if (sel[s] && act[s]) {
    const int rs = rb_start[blk], re = rb_start[blk + 1];
    const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR, ngrp = blockDim.x / LPR;
    for (int row0 = rs; row0 < re; row0 += ngrp) {  // same trip count for every thread
      const int row = row0 + grp;
      const bool valid = row < re;
      const double ax = row_dot<KT, double, LPR>(rowptr, colind, K, x, row, valid, lane);
      if (valid && lane == 0) {
        const double rv = cmask[row] ? 0.0 : f[row] - ax;
        r[row] = rv;
        v[0] += rv * rv;
      }
    }
  }
  block_partials<1>(v, part, nrb, blk);
}

// Thickness rows of the block lower-triangular preconditioner:
// z_h = invd_h (p_h - K_hu z_u - K_hv z_v), the velocity part z already set
// (row (2, g) of a uvh tangent: blocks u, v, h of deg entries each).
// Thickness rows of the block lower-triangular preconditioner: b_h = p_h - K_hu z_u (z_u
// already in z), then the first l1-Jacobi sweep zt_h = b_h / l1_h.  A row of the uvh tangent
// holds three blocks of deg columns (u, v, h).
__global__ void __launch_bounds__(256) k_uvh_hrows(const int* rb_start, const int* rb_sys, const int* sel,
                                                   const int* done, const int* dof_off, const int* rowptr,
                                                   const int* colind, const double* K, const double* hl1,
                                                   const unsigned char* cmask, const double* p, const double* z,
                                                   double* bh, double* zt) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s] || done[s]) return;
  const int nn = (dof_off[s + 1] - dof_off[s]) / 3, h0 = dof_off[s] + 2 * nn;
  const int r0 = max(rb_start[blk], h0), r1 = rb_start[blk + 1];
  for (int row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
    if (cmask[row]) { bh[row] = 0; zt[row] = 0; continue; }
    const int q0 = rowptr[row], deg = (rowptr[row + 1] - q0) / 3;
    double acc = 0;
    for (int q = q0; q < q0 + 2 * deg; ++q) acc += K[q] * z[colind[q]];
    const double b = p[row] - acc;
    bh[row] = b;
    zt[row] = b / hl1[row];
  }
}

// l1 row sums of the thickness block K_hh (the h columns of the h rows)
__global__ void __launch_bounds__(256) k_uvh_hl1(const int* rb_start, const int* rb_sys, const int* sel,
                                                 const int* dof_off, const int* rowptr, const double* K,
                                                 double* hl1) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s]) return;
  const int nn = (dof_off[s + 1] - dof_off[s]) / 3, h0 = dof_off[s] + 2 * nn;
  const int r0 = max(rb_start[blk], h0), r1 = rb_start[blk + 1];
  for (int row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
    const int q0 = rowptr[row], deg = (rowptr[row + 1] - q0) / 3;
    double a = 0;
    for (int q = q0 + 2 * deg; q < q0 + 3 * deg; ++q) a += fabs(K[q]);
    hl1[row] = a > 0 ? a : 1.0;
  }
}

// one l1-Jacobi sweep on the thickness block: zout_h = zin_h + (b_h - K_hh zin_h) / l1_h
__global__ void __launch_bounds__(256) k_uvh_hsweep(const int* rb_start, const int* rb_sys, const int* sel,
                                                    const int* done, const int* dof_off, const int* rowptr,
                                                    const int* colind, const double* K, const double* hl1,
                                                    const unsigned char* cmask, const double* bh,
                                                    const double* zin, double* zout) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s] || done[s]) return;
  const int nn = (dof_off[s + 1] - dof_off[s]) / 3, h0 = dof_off[s] + 2 * nn;
  const int r0 = max(rb_start[blk], h0), r1 = rb_start[blk + 1];
  for (int row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
    if (cmask[row]) { zout[row] = 0; continue; }
    const int q0 = rowptr[row], deg = (rowptr[row + 1] - q0) / 3;
    double acc = 0;
    for (int q = q0 + 2 * deg; q < q0 + 3 * deg; ++q) acc += K[q] * zin[colind[q]];
    zout[row] = zin[row] + (bh[row] - acc) / hl1[row];
  }
}

struct GmSys {
  std::vector<double> H, cs, sn, g;  // (m+1) x m column-major Hessenberg, rotations, rhs
  double beta0 = 0, beta = 0, tol = 0;
  int its = 0, j = 0;
  bool active = false, cycle_done = false;
};

template <typename KT>
static int gmres_t(ua_mesh* m, const ua_params* p, const KT* K, int* its_out, const double* eta) {
  Work* w = m->work;
  const int nsys = w->nsys, N = m->ndof_total;
  const int mr = std::max(4, std::min(200, p->krylov_restart > 0 ? p->krylov_restart : 40));
  const size_t ldv = (size_t)N;
  const int ld = mr + 1;
  // work space: basis V (mr+1 vectors), w, z, u; per-system coefficient arrays
  if (!w->gm_V || w->gm_m != mr) {
    w->gm_V = walloc<double>(m, (size_t)(mr + 1) * ldv);
    w->gm_w = walloc<double>(m, ldv);
    w->gm_z = walloc<double>(m, ldv);
    w->gm_u = walloc<double>(m, ldv);
    w->gm_part = walloc<double>(m, (size_t)(mr + 1) * w->nrb);
    w->gm_coef = walloc<double>(m, (size_t)3 * nsys * ld);  // two orthogonalisation passes and the norm
    w->gm_scal = walloc<double>(m, (size_t)nsys * ld);
    w->gm_act = walloc<int>(m, nsys);
    w->gm_ny = walloc<int>(m, nsys);
    w->gm_hb = walloc<double>(m, ldv);
    w->gm_ht = walloc<double>(m, ldv);
    w->gm_hl1 = walloc<double>(m, ldv);
    if (!w->gm_V || !w->gm_w || !w->gm_z || !w->gm_u || !w->gm_part || !w->gm_coef || !w->gm_scal || !w->gm_act ||
        !w->gm_ny || !w->gm_hb || !w->gm_ht || !w->gm_hl1)
      return set_error(UA_ERR_OOM, "device allocation of the GMRES basis failed");
    w->gm_m = mr;
  }
  double *V = w->gm_V, *wv = w->gm_w, *zv = w->gm_z, *uv = w->gm_u;
  cudaStream_t st = m->stream;
  double* invd = (double*)w->invd;
  k_invdiag<KT, double><<<(N + 255) / 256, 256, 0, st>>>(N, K, w->diagpos, w->cmask, invd), ++g_launches;
  bool amg = p->krylov_precond == UA_PC_AMG && m->ndof == 3 && !m->h_nodeptr.empty() && sizeof(KT) == 8;
  if (amg && amg_setup(m, p->amg_smoothed != 0) != UA_OK) amg = false;
  if (amg) {
    int rc = amg_numeric_uvh(m, (const double*)K, w->cmask, &g_launches);
    if (rc) return rc;
  }
  const int lpr_uv = m->nod == 3 ? 1 : 2;
  // thickness block: l1-Jacobi sweeps on K_hh (the P2 consistent mass in K_hh is not diagonally
  // dominant, so a plain Jacobi step is a poor inverse and a plain Jacobi iteration diverges)
  const int hsw = p->uvh_h_sweeps > 0 ? p->uvh_h_sweeps : 8;
  if (m->ndof == 3)
    k_uvh_hl1<<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->sel, m->dm.sys_dof_off, w->rowptr,
                                      (const double*)K, w->gm_hl1), ++g_launches;
  // preconditioner: velocity rows by the AMG V-cycle (else Jacobi), thickness rows by the block
  // lower-triangular step z_h = K_hh^-1 (r_h - K_hu z_u), K_hh^-1 by hsw l1-Jacobi sweeps from zero
  auto precond = [&](const double* in, double* out) -> int {
    k_scale_vec<<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->sel, w->done, in, invd, out), ++g_launches;
    if (amg) {
      int rc = amg_apply_uvh(m, in, out, w->sel, w->done, lpr_uv, &g_launches);
      if (rc) return rc;
    }
    if (m->ndof == 3) {
      // ping-pong between gm_ht and out so that the last sweep writes out (h rows only)
      double* bufs[2] = {out, w->gm_ht};
      int cur = (hsw - 1) % 2 == 0 ? 0 : 1;
      k_uvh_hrows<<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->sel, w->done, m->dm.sys_dof_off, w->rowptr,
                                          w->colind, (const double*)K, w->gm_hl1, w->cmask, in, out, w->gm_hb,
                                          bufs[cur]), ++g_launches;
      for (int k = 1; k < hsw; ++k) {
        k_uvh_hsweep<<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->sel, w->done, m->dm.sys_dof_off,
                                             w->rowptr, w->colind, (const double*)K, w->gm_hl1, w->cmask, w->gm_hb,
                                             bufs[cur], bufs[1 - cur]), ++g_launches;
        cur = 1 - cur;
      }
    }
    return UA_OK;
  };
  auto spmv = [&](const double* x, double* y) {
    k_bicg_spmv<KT, 16><<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->done, w->rowptr,
                                                w->colind, K, x, w->cmask, y, nullptr, w->part), ++g_launches;
  };
  // Two-entry constraint rows (ties, normal velocities): the Krylov space is kept in the range of
  // I - B'B by projecting the residual, every preconditioned vector and every product, so GMRES
  // solves the projected system (P K P) x = P f on it.
  const int npb = (w->npair + 255) / 256;
  auto project = [&](double* v) {
    if (w->npair)
      k_pair_project<double><<<npb, 256, 0, st>>>(w->npair, w->pair_rows, w->con_dof, w->con_sys, w->sel, w->done,
                                                  con_pairs(w), v), ++g_launches;
  };
  // host-side reduction results
  std::vector<double> hco((size_t)nsys * ld), hco2((size_t)nsys * ld), hnrm((size_t)nsys * ld), hsc(nsys),
      hy((size_t)nsys * ld), hco3((size_t)3 * nsys * ld);
  bool flags_changed = false;
  std::vector<int> hact(nsys), hny(nsys), hdone(nsys);
  // per-system sums of nv partial arrays into coef (device), without a host copy
  auto reduce_dev = [&](const double* part, int nv, double* coef) {
    k_gm_reduce<<<dim3(nsys, nv), kRedThreads, 0, st>>>(w->sys_rb_off, w->nrb, w->sel, w->done, part, coef, ld),
        ++g_launches;
  };
  auto reduce_to_host = [&](const double* part, int nv, std::vector<double>& dst) -> int {
    k_gm_reduce<<<dim3(nsys, nv), kRedThreads, 0, st>>>(w->sys_rb_off, w->nrb, w->sel, w->done, part, w->gm_coef,
                                                        ld), ++g_launches;
    UA_CUDA_TRY(cudaMemcpyAsync(dst.data(), w->gm_coef, sizeof(double) * nsys * ld, cudaMemcpyDeviceToHost, st));
    UA_CUDA_TRY(cudaStreamSynchronize(st));
    return UA_OK;
  };
  // x0: zero plus the particular solution on the constrained dofs
  k_zero_sel<<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->sel, w->dX), ++g_launches;
  if (w->nc)
    k_con_particular<<<(w->nc + 255) / 256, 256, 0, st>>>(w->nc, w->con_dof, w->con_sys, w->sel, w->con_rhs, w->X,
                                                         w->dX, w->grhs, con_pairs(w)), ++g_launches;
  std::vector<GmSys> S(nsys);
  for (int s = 0; s < nsys; ++s) {
    S[s].active = its_out[s] != 0;
    S[s].H.assign((size_t)ld * mr, 0.0);
    S[s].cs.assign(mr, 0.0);
    S[s].sn.assign(mr, 0.0);
    S[s].g.assign(ld, 0.0);
    S[s].tol = eta ? eta[s] : p->krylov_rtol;
  }
  auto upload_flags = [&]() -> int {
    for (int s = 0; s < nsys; ++s) { hact[s] = S[s].active ? 1 : 0; hdone[s] = (S[s].active && !S[s].cycle_done) ? 0 : 1; }
    UA_CUDA_TRY(cudaMemcpyAsync(w->gm_act, hact.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, st));
    UA_CUDA_TRY(cudaMemcpyAsync(w->done, hdone.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, st));
    return UA_OK;
  };
  int total_cycles = 0;
  const int max_cycles = std::max(1, p->krylov_maxit / mr + 1);
  bool first = true;
  while (true) {
    // residual of the current iterate, v0 = r / |r|
    for (int s = 0; s < nsys; ++s) S[s].cycle_done = false;
    int rc = upload_flags();
    if (rc) return rc;
    dispatch_lpr(16, [&](auto L) {
      k_gm_resid<KT, decltype(L)::value><<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->gm_act,
                                                                  w->rowptr, w->colind, K, w->dX, w->frhs, w->cmask,
                                                                  wv, w->gm_part);
    });
    ++g_launches;
    if (w->npair) {  // project the residual before its norm is taken
      project(wv);
      k_gm_dots<<<dim3(w->nrb, 1), 256, 0, st>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->done, wv, wv, 0,
                                                 w->gm_part), ++g_launches;
    }
    if ((rc = reduce_to_host(w->gm_part, 1, hco))) return rc;
    bool any = false;
    for (int s = 0; s < nsys; ++s) {
      GmSys& G = S[s];
      if (!G.active) continue;
      const double b = std::sqrt(std::max(hco[(size_t)s * ld], 0.0));
      if (first) G.beta0 = b;
      G.beta = b;
      if (!(b == b) || b <= G.tol * G.beta0 || b == 0.0 || G.its >= p->krylov_maxit || total_cycles >= max_cycles) {
        G.active = false;
        continue;
      }
      std::fill(G.g.begin(), G.g.end(), 0.0);
      G.g[0] = b;
      G.j = 0;
      hsc[s] = 1.0 / b;
      any = true;
    }
    first = false;
    if (!any) break;
    if ((rc = upload_flags())) return rc;
    UA_CUDA_TRY(cudaMemcpyAsync(w->gm_scal, hsc.data(), sizeof(double) * nsys, cudaMemcpyHostToDevice, st));
    k_gm_scale<<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->sel, w->done, wv, V, w->gm_scal), ++g_launches;
    // Arnoldi steps
    for (int j = 0; j < mr; ++j) {
      if ((rc = precond(V + (size_t)j * ldv, zv))) return rc;
      project(zv);
      spmv(zv, wv);
      project(wv);
      // classical Gram-Schmidt twice, then the norm and the next basis vector w / |w|, all on the
      // device (coefficients in gm_coef: pass 1, pass 2, norm); one host copy per Arnoldi step
      // for the Hessenberg column, the rotations and the convergence test
      double* const cf[3] = {w->gm_coef, w->gm_coef + (size_t)nsys * ld, w->gm_coef + (size_t)2 * nsys * ld};
      for (int pass = 0; pass < 2; ++pass) {
        k_gm_dots<<<dim3(w->nrb, j + 1), 256, 0, st>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->done, wv, V, ldv,
                                                       w->gm_part), ++g_launches;
        reduce_dev(w->gm_part, j + 1, cf[pass]);
        k_gm_orth<<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->sel, w->done, wv, V, ldv, j + 1, cf[pass],
                                          ld), ++g_launches;
      }
      k_gm_dots<<<dim3(w->nrb, 1), 256, 0, st>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->done, wv, wv, 0,
                                                 w->gm_part), ++g_launches;
      reduce_dev(w->gm_part, 1, cf[2]);
      // V_{j+1} = w / |w| for every system still in the cycle (a system whose cycle ends here
      // never reads it)
      if (j + 1 < mr)
        k_gm_scale_norm<<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->sel, w->done, wv,
                                                V + (size_t)(j + 1) * ldv, cf[2], ld), ++g_launches;
      UA_CUDA_TRY(cudaMemcpyAsync(hco3.data(), w->gm_coef, sizeof(double) * 3 * nsys * ld, cudaMemcpyDeviceToHost,
                                  st));
      UA_CUDA_TRY(cudaStreamSynchronize(st));
      std::copy(hco3.begin(), hco3.begin() + (size_t)nsys * ld, hco.begin());
      std::copy(hco3.begin() + (size_t)nsys * ld, hco3.begin() + (size_t)2 * nsys * ld, hco2.begin());
      std::copy(hco3.begin() + (size_t)2 * nsys * ld, hco3.end(), hnrm.begin());
      bool more = false;
      for (int s = 0; s < nsys; ++s) {
        GmSys& G = S[s];
        if (!G.active || G.cycle_done) continue;
        double* h = &G.H[(size_t)j * ld];
        for (int i = 0; i <= j; ++i) h[i] = hco[(size_t)s * ld + i] + hco2[(size_t)s * ld + i];
        const double hn = std::sqrt(std::max(hnrm[(size_t)s * ld], 0.0));
        h[j + 1] = hn;
        for (int i = 0; i < j; ++i) {  // previous rotations
          const double a = h[i], b = h[i + 1];
          h[i] = G.cs[i] * a + G.sn[i] * b;
          h[i + 1] = -G.sn[i] * a + G.cs[i] * b;
        }
        const double den = std::hypot(h[j], h[j + 1]);
        G.cs[j] = den > 0 ? h[j] / den : 1.0;
        G.sn[j] = den > 0 ? h[j + 1] / den : 0.0;
        h[j] = den;
        h[j + 1] = 0.0;
        G.g[j + 1] = -G.sn[j] * G.g[j];
        G.g[j] = G.cs[j] * G.g[j];
        G.its++;
        G.j = j + 1;
        const double res = std::fabs(G.g[j + 1]);
        if (res <= G.tol * G.beta0 || hn == 0.0 || !(res == res) || G.its >= p->krylov_maxit || j + 1 == mr) {
          G.cycle_done = true;
          flags_changed = true;
        } else {
          more = true;
        }
      }
      if (!more) break;
      if (flags_changed) {
        if ((rc = upload_flags())) return rc;
        flags_changed = false;
      }
    }
    // x += M^-1 (V y), y from the triangular system of each active system
    for (int s = 0; s < nsys; ++s) {
      GmSys& G = S[s];
      hny[s] = 0;
      if (!G.active) continue;
      const int k = G.j;
      for (int i = k - 1; i >= 0; --i) {
        double acc = G.g[i];
        for (int c = i + 1; c < k; ++c) acc -= G.H[(size_t)c * ld + i] * hy[(size_t)s * ld + c];
        const double d = G.H[(size_t)i * ld + i];
        hy[(size_t)s * ld + i] = d != 0.0 ? acc / d : 0.0;
      }
      hny[s] = k;
    }
    for (int s = 0; s < nsys; ++s) S[s].cycle_done = false;
    if ((rc = upload_flags())) return rc;
    UA_CUDA_TRY(cudaMemcpyAsync(w->gm_scal, hy.data(), sizeof(double) * nsys * ld, cudaMemcpyHostToDevice, st));
    UA_CUDA_TRY(cudaMemcpyAsync(w->gm_ny, hny.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, st));
    k_gm_combine<<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->sel, w->gm_act, uv, V, ldv, w->gm_scal,
                                         w->gm_ny, ld), ++g_launches;
    if ((rc = precond(uv, zv))) return rc;
    project(zv);
    k_gm_axpy<<<w->nrb, 256, 0, st>>>(w->rb_start, w->rb_sys, w->sel, w->gm_act, w->dX, zv), ++g_launches;
    ++total_cycles;
  }
  // restore selection semantics for the callers (done = finished)
  for (int s = 0; s < nsys; ++s) hdone[s] = 1;
  UA_CUDA_TRY(cudaMemcpyAsync(w->done, hdone.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, st));
  if (w->nc)
    k_con_multiplier<KT><<<(w->nc + 255) / 256, 256, 0, st>>>(w->nc, w->con_dof, w->con_sys, w->sel, w->rowptr,
                                                              w->colind, K, w->dX, w->frhs, w->dlam, con_pairs(w)), ++g_launches;
  UA_CUDA_TRY(cudaGetLastError());
  UA_CUDA_TRY(cudaStreamSynchronize(st));
  for (int s = 0; s < nsys; ++s) its_out[s] = its_out[s] ? S[s].its : 0;
  return UA_OK;
}

static UvhPhys make_uvh_phys(const ua_params* p) {
  UvhPhys P;
  P.uv = make_phys(p);
  P.kH = p->kH; P.Hh0 = p->Hh0; P.SpeedZero = p->SpeedZero;
  P.theta = p->theta; P.beta0 = p->SUPG_beta0; P.tau_mult = p->uvh_SUPG_tauMultiplier;
  P.tau_kind = p->uvh_SUPG_tau;
  return P;
}

static int upload_fields_uvh(ua_mesh* m, const ua_params* p, const ua_fields* F, int nF) {
  Work* w = m->work;
  std::vector<SysScal> sc(m->dm.nsys);
  for (int s = 0; s < m->dm.nsys; ++s) {
    const ua_fields& f = F[nF == 1 ? 0 : s];
    const int no = m->h_node_off[s], nn = m->sys[s].nn, d0 = m->h_dof_off[s];
    const double* src[] = {f.S, f.B, f.rho, f.AGlen, f.n, f.C, f.m, f.h0, f.u0, f.v0, f.as0, f.ab0, f.as1, f.ab1};
    double* dst[] = {w->S, w->B, w->rho, w->A, w->n, w->C, w->m, w->h0, w->u0, w->v0, w->as0, w->ab0, w->as1, w->ab1};
    const char* names[] = {"S", "B", "rho", "AGlen", "n", "C", "m", "h0", "u0", "v0", "as0", "ab0", "as1", "ab1"};
    auto kind = f.location == UA_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    for (int k = 0; k < 14; ++k) {
      if (!src[k]) return set_error(UA_ERR_INVALID, "system %d: null uvh field %s", s, names[k]);
      if (f.location == UA_HOST && any_nan(src[k], nn))
        return set_error(UA_ERR_NAN_INPUT, "uvhMatrixAssembly:NaN nan in %s (system %d)", names[k], s);
      UA_CUDA_TRY(cudaMemcpyAsync(dst[k] + no, src[k], nn * sizeof(double), kind, m->stream));
    }
    if (f.dadh) UA_CUDA_TRY(cudaMemcpyAsync(w->dadh + no, f.dadh, nn * sizeof(double), kind, m->stream));
    else UA_CUDA_TRY(cudaMemsetAsync(w->dadh + no, 0, nn * sizeof(double), m->stream));
    if (!f.ub || !f.vb || !f.h1) return set_error(UA_ERR_INVALID, "system %d: null ub/vb/h1", s);
    if (f.location == UA_HOST && (any_nan(f.ub, nn) || any_nan(f.vb, nn) || any_nan(f.h1, nn)))
      return set_error(UA_ERR_NAN_INPUT, "uvhMatrixAssembly:NaN nan in F1.ub, F1.vb or F1.h");
    UA_CUDA_TRY(cudaMemcpyAsync(w->X + d0, f.ub, nn * sizeof(double), kind, m->stream));
    UA_CUDA_TRY(cudaMemcpyAsync(w->X + d0 + nn, f.vb, nn * sizeof(double), kind, m->stream));
    UA_CUDA_TRY(cudaMemcpyAsync(w->X + d0 + 2 * nn, f.h1, nn * sizeof(double), kind, m->stream));
    sc[s].rhow = f.rhow; sc[s].g = f.g; sc[s].ca = std::cos(f.alpha); sc[s].sa = std::sin(f.alpha);
    sc[s].dt = f.dt;
  }
  UA_CUDA_TRY(cudaMemcpyAsync(w->scal, sc.data(), sc.size() * sizeof(SysScal), cudaMemcpyHostToDevice, m->stream));
  set_cube_flags(m);
  return upload_drag_fields(m, p, F, nF);
}

static int assemble_uvh(ua_mesh* m, const ua_params* p, bool withK, bool useDir, bool zero, bool parts) {
  Work* w = m->work;
  UvhIn in{w->S, w->B, w->rho, w->A, w->n, w->C, w->m, w->h0, w->u0, w->v0, w->as0, w->ab0, w->as1, w->ab1,
           w->dadh, w->X, useDir ? w->dX : nullptr, useDir ? w->gamma : nullptr, w->scal, w->sel, zero ? 1 : 0};
  in.drag = drag_fields(w);
  UvOut out{w->R, withK ? (void*)w->Kd : nullptr, parts ? w->Tint : nullptr, parts ? w->Fext : nullptr};
  cudaEvent_t ev[2];
  prof_begin(m, withK ? PK_ASMK : PK_ASMR, ev);
  cudaError_t e = launch_uvh_assembly(m, make_uvh_phys(p), in, out, withK);
  prof_end(m, ev);
  ++g_launches;
  if (e != cudaSuccess) return set_error(UA_ERR_CUDA, "uvh assembly launch: %s", cudaGetErrorString(e));
  return UA_OK;
}

// CalcCostFunctionNRuvh.m:12-105 for the selected systems
// uvh cost function at X + gamma dX; assembleR = false takes w->R as it stands
// (the residual just assembled at X, i.e. gamma = 0).
static int cost_eval_uvh(ua_mesh* m, const ua_params* p, bool assembleR = true) {
  Work* w = m->work;
  if (assembleR) {
    int rc = assemble_uvh(m, p, false, true, false, false);
    if (rc) return rc;
  }
  k_cost_rows<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->R, w->dof_con, w->lam,
                                             w->dlam, w->gamma, w->dX, w->part, w->con_dof, con_pairs(w)), ++g_launches;
  k_cost_reduce<<<w->nsys, kRedThreads, 0, m->stream>>>(w->sys_rb_off, w->nrb, w->sel, w->part, w->nsys, w->sysv,
                                                         w->sys_con_off, w->con_dof, w->con_rhs, w->X, w->dX, w->dlam,
                                                         w->gamma, 0, con_pairs(w)), ++g_launches;
  UA_CUDA_TRY(cudaGetLastError());
  UA_CUDA_TRY(cudaMemcpyAsync(w->h_sysv, w->sysv, SV_COUNT * w->nsys * sizeof(double), cudaMemcpyDeviceToHost,
                              m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  return UA_OK;
}

static bool uvh_criteria(const ua_params* p, double rForce, double rWork, int iteration, double gamma) {
  const double *a, *o;
  if (gamma > std::max(p->uvhExitBackTrackingStepLength, p->BacktrackingGammaMin)) {
    a = p->uvhDesiredWorkAndForceTolerances; o = p->uvhDesiredWorkOrForceTolerances;
  } else {
    a = p->uvhAcceptableWorkAndForceTolerances; o = p->uvhAcceptableWorkOrForceTolerances;
  }
  return (rWork < a[0] && rForce < a[1]) && (rWork < o[0] || rForce < o[1]) && iteration >= p->NRitmin;
}

struct UvhSys {
  bool active = false, converged = false, bt_ok = true;
  int iteration = 0, iarm = 0, kits = 0;
  double r = INFINITY, r0 = INFINITY, rForce = INFINITY, rWork = NAN, gamma = 1, r1 = 0;
  double rRatio[3] = {0, 0, 0};
  BackTrack bt;
  std::vector<double> ls_g, ls_D2;
};

static int newton_run_uvh(ua_mesh* m, const ua_params* p, std::vector<ua_newton_report*>& rep,
                          std::vector<UvhSys>& st) {
  Work* w = m->work;
  const int nsys = w->nsys;
  int rc;
  double t_asm = 0, t_sol = 0;
  std::vector<int> sel(nsys, 1), its(nsys);
  std::vector<double> gam(nsys, 0.0);
  if ((rc = set_sel(m, sel))) return rc;
  // uvhMakeInitialIterateFeasible (:37-41)
  if (w->nc)
    k_set_con_values<<<(w->nc + 255) / 256, 256, 0, m->stream>>>(w->nc, w->con_dof, w->con_sys, w->sel, w->con_rhs,
                                                                 w->X, con_pairs(w)), ++g_launches;
  // Fext0 at ZeroFields (:53-56); the normalisation of CalcCostFunctionNRuvh
  if ((rc = assemble_uvh(m, p, false, false, true, false))) return rc;
  k_cost_rows<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->nrb, w->sel, w->R, nullptr, nullptr, nullptr,
                                             nullptr, nullptr, w->part, nullptr, ConPairs{}), ++g_launches;
  k_cost_reduce<<<nsys, kRedThreads, 0, m->stream>>>(w->sys_rb_off, w->nrb, w->sel, w->part, nsys, w->sysv, nullptr,
                                                     nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 1, con_pairs(w)), ++g_launches;
  UA_CUDA_TRY(cudaGetLastError());
  for (int s = 0; s < nsys; ++s) { st[s] = UvhSys(); st[s].active = true; }
  while (true) {
    bool any = false;
    for (int s = 0; s < nsys; ++s) {
      UvhSys& S = st[s];
      if (!S.active) continue;
      if (S.rWork != S.rWork) S.rWork = 0;  // :78-80
      if (uvh_criteria(p, S.rForce, S.rWork, S.iteration, S.gamma)) { S.converged = true; S.active = false; continue; }
      if (S.iteration > p->NRitmax) { S.converged = false; S.active = false; continue; }
      if (!S.bt_ok || S.gamma == 0) { S.converged = false; S.active = false; continue; }  // :104-110
      const double ratio = S.r / S.r0;
      S.rRatio[S.iteration % 3] = ratio;  // :111-124 stagnation
      if (S.rRatio[0] > 0.98 && S.rRatio[1] > 0.98 && S.rRatio[2] > 0.98) {
        S.converged = S.rWork < 1e-14; S.active = false; continue;
      }
      S.iteration++;
      any = true;
    }
    if (!any) break;
    for (int s = 0; s < nsys; ++s) sel[s] = st[s].active ? 1 : 0;
    if ((rc = set_sel(m, sel))) return rc;
    double t0 = now_ms();
    if ((rc = assemble_uvh(m, p, true, false, false, false))) return rc;  // :127
    k_frhs<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->sel, w->R, w->dof_con, w->lam, w->frhs, w->con_dof, con_pairs(w)), ++g_launches;
    UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    double t1 = now_ms();
    t_asm += t1 - t0;
    for (int s = 0; s < nsys; ++s) its[s] = sel[s];
    std::vector<double> eta(nsys);
    for (int s = 0; s < nsys; ++s) eta[s] = forcing_term_uvh(p, st[s].rForce == INFINITY ? 1.0 : st[s].rForce);
    if (p->uvh_krylov == UA_KRYLOV_BICGSTAB) {
      if ((rc = bicgstab_t<double>(m, p, w->Kd, its.data(), eta.data()))) return rc;  // :136
    } else {
      if ((rc = gmres_t<double>(m, p, w->Kd, its.data(), eta.data()))) return rc;
    }
    t_sol += now_ms() - t1;
    for (int s = 0; s < nsys; ++s) if (sel[s]) st[s].kits = its[s];
    // r0 = func(0), r1 = func(1) (:155-156)
    for (int g1 = 0; g1 < 2; ++g1) {
      for (int s = 0; s < nsys; ++s) gam[s] = (double)g1;
      if ((rc = set_gamma(m, gam))) return rc;
      if ((rc = cost_eval_uvh(m, p, g1 != 0))) return rc;  // R at gamma = 0 was assembled with K
      for (int s = 0; s < nsys; ++s) {
        if (!sel[s]) continue;
        const double rf = w->h_sysv[SV_FF * nsys + s], d2 = w->h_sysv[SV_FD * nsys + s];
        UvhSys& S = st[s];
        if (g1 == 0) { S.r0 = rf; S.ls_g.assign({0.0}); S.ls_D2.assign({d2}); }
        else { S.r1 = rf; S.ls_g.push_back(1.0); S.ls_D2.push_back(d2); }
      }
    }
    // rLineminUa (:157): Newton-direction backtracking, BackTracking accepts
    // gamma=1 at once when r1 is below its target
    for (int s = 0; s < nsys; ++s) {
      if (!sel[s]) continue;
      UvhSys& S = st[s];
      S.bt = BackTrack();
      BTConfig& c = S.bt.cfg;
      c.beta = p->BackTrackBeta; c.ExtrapolationRatio = p->BackTrackExtrapolationRatio;
      c.MinXfracRel = p->BackTrackMinXfrac; c.GL = p->BackTrackGuardLower; c.GU = p->BackTrackGuardUpper;
      c.NewtonAcceptRatio = p->NewtonAcceptRatio; c.GammaMin = 0.001; c.NLtol = p->NLtol;
      c.MaxIterations = p->BackTrackMaxIterations; c.MaxExtrapolations = p->BackTrackMaxExtrapolations;
      c.MaxFuncSame = p->BackTrackMaxFuncSame; c.allow_ext = p->LineSearchAllowedToUseExtrapolation != 0;
      S.bt.start(-2 * S.r0, 1.0, S.r0, S.r1);
    }
    while (true) {
      bool need = false;
      for (int s = 0; s < nsys; ++s) {
        sel[s] = (st[s].active && !st[s].bt.done) ? 1 : 0;
        gam[s] = sel[s] ? st[s].bt.request : 0.0;
        need = need || sel[s];
      }
      if (!need) break;
      if ((rc = set_sel(m, sel))) return rc;
      if ((rc = set_gamma(m, gam))) return rc;
      if ((rc = cost_eval_uvh(m, p))) return rc;
      for (int s = 0; s < nsys; ++s) {
        if (!sel[s]) continue;
        st[s].ls_g.push_back(gam[s]);
        st[s].ls_D2.push_back(w->h_sysv[SV_FD * nsys + s]);
        st[s].bt.feed(w->h_sysv[SV_FF * nsys + s]);
      }
    }
    for (int s = 0; s < nsys; ++s) {
      sel[s] = 0;
      UvhSys& S = st[s];
      if (!S.active) continue;
      const double gN = S.bt.gmin, rN = S.bt.fmin;
      if (rep[s] && gN < 0.75 && rN / S.r0 > 0.7) rep[s]->cauchy_fallbacks++;  // rLineminUa.m:96
      S.iarm = S.bt.iarm;
      S.bt_ok = S.bt.converged && !S.bt.error;
      if (rN < S.r0) {
        S.gamma = gN; S.r = rN; S.rForce = rN; S.rWork = NAN;
        for (size_t k = 0; k < S.ls_g.size(); ++k)
          if (S.ls_g[k] == gN) { S.rWork = S.ls_D2[k] * S.ls_D2[k]; break; }
      } else {
        S.gamma = 0; S.r = S.r0; S.rForce = S.r0; S.rWork = NAN;  // rLineminUa.m:27-28
      }
      if (rep[s] && rep[s]->iters && rep[s]->n_iter_records < rep[s]->iters_capacity) {
        ua_newton_iter& it = rep[s]->iters[rep[s]->n_iter_records++];
        it.iteration = S.iteration; it.iarm = S.iarm; it.krylov_its = S.kits; it.direction = S.iarm > 0;
        it.gamma = S.gamma; it.r0 = S.r0; it.r = S.r; it.rForce = S.rForce; it.rWork = S.rWork;
      }
      if (rep[s]) rep[s]->krylov_its_total += S.kits;
      if (p->verbose)
        fprintf(stderr, "NR-SSTREAM(uvh)[%d]:%3d/%-2d g=%-14.7g , r/r0=%-14.7g ,  r0=%-14.7g , r=%-14.7g , rForce=%-14.7g , rWork=%-14.7g , bicg=%d\n",
                s, S.iteration, S.iarm, S.gamma, S.r / S.r0, S.r0, S.r, S.rForce, S.rWork, S.kits);
      sel[s] = 1;
      gam[s] = S.gamma;
    }
    if ((rc = set_sel(m, sel))) return rc;
    if ((rc = set_gamma(m, gam))) return rc;
    k_newton_update<<<w->nrb, 256, 0, m->stream>>>(w->rb_start, w->rb_sys, w->sel, w->gamma, w->X, w->dX), ++g_launches;
    if (w->nc)
      k_lam_update<<<(w->nc + 255) / 256, 256, 0, m->stream>>>(w->nc, w->con_sys, w->sel, w->gamma, w->lam, w->dlam), ++g_launches;
    UA_CUDA_TRY(cudaGetLastError());
    if ((rc = record_updates(m, rep, sel, gam))) return rc;
  }
  for (int s = 0; s < nsys; ++s) {
    if (!rep[s]) continue;
    rep[s]->converged = st[s].converged ? 1 : 0;
    rep[s]->iterations = st[s].iteration;
    rep[s]->backtrack_steps = st[s].iarm;
    rep[s]->r = st[s].r; rep[s]->rForce = st[s].rForce; rep[s]->rWork = st[s].rWork;
    rep[s]->assembly_ms += t_asm; rep[s]->solve_ms += t_sol;
  }
  return UA_OK;
}

}  // namespace ua

using namespace ua;

extern "C" void ua_params_default(ua_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->kH = 1; p->Hh0 = 0;
  p->SpeedZero = 1e-4; p->EpsZero = 1e-10; p->etaZero = 10;
  p->Czero = 0; p->Cmin = 1e-20; p->AGlenmin = 1e-20;
  p->Picard = 0; p->NRviscosity = 1;
  p->NRitmax = 50; p->NRitmin = 1; p->NewtonAcceptRatio = 0.5; p->BacktrackingGammaMin = 1e-10;
  p->LineSearchAllowedToUseExtrapolation = 0;
  p->BackTrackBeta = 0.1; p->BackTrackMaxIterations = 50; p->BackTrackMaxExtrapolations = 50;
  p->BackTrackExtrapolationRatio = 2.5; p->BackTrackMinXfrac = 1e-10; p->BackTrackMaxFuncSame = 3;
  p->BackTrackGuardLower = 0.25; p->BackTrackGuardUpper = 0.95; p->NLtol = 1e-15;
  const double inf = INFINITY;
  double d[2] = {inf, 1e-15};
  std::memcpy(p->uvDesiredWorkAndForceTolerances, d, sizeof d);
  std::memcpy(p->uvDesiredWorkOrForceTolerances, d, sizeof d);
  std::memcpy(p->uvAcceptableWorkAndForceTolerances, d, sizeof d);
  std::memcpy(p->uvAcceptableWorkOrForceTolerances, d, sizeof d);
  p->uvExitBackTrackingStepLength = 1e-10;
  p->ModifiedNRuvIntervalCriterion = 1; p->ModifiedNRuvReductionCriterion = 0.5;
  p->theta = 0.5; p->SUPG_beta0 = 1; p->uvh_SUPG_tauMultiplier = 1; p->uvh_SUPG_tau = 0;
  std::memcpy(p->uvhDesiredWorkAndForceTolerances, d, sizeof d);
  std::memcpy(p->uvhDesiredWorkOrForceTolerances, d, sizeof d);
  p->uvhExitBackTrackingStepLength = 1e-3;
  double a1[2] = {inf, 1e-6}, a2[2] = {1, 1e-8};
  std::memcpy(p->uvhAcceptableWorkAndForceTolerances, a1, sizeof a1);
  std::memcpy(p->uvhAcceptableWorkOrForceTolerances, a2, sizeof a2);
  p->krylov_rtol = 1e-12; p->krylov_maxit = 20000; p->precision = UA_PREC_FP64;
  p->patch_nodes = 0; p->verbose = 0; p->profile = 0; p->krylov_adaptive = 1; p->spmv_lanes = 0; p->asm_threads = 0; p->asm_regs = 0;
  p->uvh_krylov = UA_KRYLOV_GMRES; p->krylov_restart = 40;
  p->krylov_eta_c = 0.5; p->krylov_eta_max = 0.1; p->precond_bf16 = 1;
  p->amg_smoothed = 1;
  p->krylov_full_grid = 0;
  p->amg_P_refresh = 0;
  p->uvh_h_sweeps = 0;
  p->krylov_sell = 1;
  p->krylov_precond = UA_PC_AMG;
  p->SlidingLaw = UA_SLIDING_WEERTMAN;  // :171
  p->Nzero = 1e-20;                     // :445
  p->IncludeMelangeModelPhysics = 0;
  p->ThicknessConstraints = 1;          // :1478
  p->ThickMin = 1.0;                    // :1469
  p->ThicknessConstraintsItMax = 10;    // :1479
  p->MaxNumberOfNewlyIntroducedActiveThicknessConstraints = 1000;  // :1500
  p->MinNumberOfNewlyIntroducedActiveThicknessConstraints = 0;     // :1502
}

extern "C" int ua_uv_assemble(ua_mesh* m, const ua_params* p, const ua_fields* F, const ua_bcs* bcs, int32_t mode,
                              double* R, double* Kvals, double* Tint, double* Fext) {
  if (!m || !p || !F) return set_error(UA_ERR_INVALID, "ua_uv_assemble: null argument");
  if (m->ndof != 2) return set_error(UA_ERR_INVALID, "ua_uv_assemble needs a ndof=2 mesh handle");
  if (m->dm.nsys != 1) return set_error(UA_ERR_INVALID, "ua_uv_assemble takes a single-mesh handle");
  if (mode != UA_ASM_R && mode != UA_ASM_RK && mode != UA_ASM_ZERO_R) return set_error(UA_ERR_INVALID, "bad mode");
  UA_CUDA_TRY(cudaSetDevice(m->device));
  int rc;
  if ((rc = ensure_work(m, p))) return rc;
  Work* w = m->work;
  bool withK = mode == UA_ASM_RK;
  if (withK && (rc = ensure_K(m, p->precision))) return rc;
  if ((rc = upload_fields(m, p, F, 1))) return rc;
  if ((rc = upload_velocity(m, F, 1))) return rc;
  if (mode == UA_ASM_ZERO_R) {  // uvMatrixAssemblySSTREAM.m:24-28
    if ((rc = build_constraints(m, bcs, 1))) return rc;
    UA_CUDA_TRY(cudaMemsetAsync(w->X, 0, m->ndof_total * sizeof(double), m->stream));
    if (w->nc)
      k_set_con_values<<<(w->nc + 255) / 256, 256, 0, m->stream>>>(w->nc, w->con_dof, w->con_sys, nullptr,
                                                                   w->con_rhs, w->X, con_pairs(w)), ++g_launches;
  }
  std::vector<int> sel(1, 1);
  if ((rc = set_sel(m, sel))) return rc;
  if ((rc = assemble(m, p, withK, false, w->X, Tint || Fext))) return rc;
  const int N = m->ndof_total;
  if (R) UA_CUDA_TRY(cudaMemcpyAsync(R, w->R, N * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if (Tint) UA_CUDA_TRY(cudaMemcpyAsync(Tint, w->Tint, N * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if (Fext) UA_CUDA_TRY(cudaMemcpyAsync(Fext, w->Fext, N * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if (withK && Kvals) {
    if (p->precision == UA_PREC_MIXED) {
      std::vector<float> tmp(m->nnz_total);
      UA_CUDA_TRY(cudaMemcpyAsync(tmp.data(), w->Kf, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
      UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
      for (size_t i = 0; i < tmp.size(); ++i) Kvals[i] = tmp[i];
    } else {
      UA_CUDA_TRY(cudaMemcpyAsync(Kvals, w->Kd, m->nnz_total * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    }
  }
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  return UA_OK;
}

// The assembly autotuner: times the tangent+residual assembly (the dominant kernel of the uv
// Newton solve) of this handle's systems at the given fields for each candidate schedule (patch
// shape x CTA size), keeps the fastest for the handle and records it as the tuned schedule of
// this device, element type and dof count, which every handle then takes with patch_nodes = 0
// and asm_threads = 0.  The schedules change where the element work runs, not what is summed in
// which order, so K and R are the same under every one of them.
extern "C" int ua_autotune(ua_mesh* m, const ua_params* p, const ua_fields* F, int32_t nF, int32_t reps,
                           ua_tune_report* rep) {
  if (!m || !p || !F || !rep) return set_error(UA_ERR_INVALID, "ua_autotune: null argument");
  if (m->ndof != 2) return set_error(UA_ERR_INVALID, "ua_autotune tunes the uv assembly (ndof=2 handle)");
  if (nF != 1 && nF != m->dm.nsys) return set_error(UA_ERR_INVALID, "ua_autotune: nF must be 1 or the system count");
  if (reps < 1) reps = 3;
  UA_CUDA_TRY(cudaSetDevice(m->device));
  int rc;
  if ((rc = ensure_work(m, nullptr))) return rc;
  Work* w = m->work;
  if ((rc = ensure_K(m, p->precision))) return rc;
  if ((rc = upload_fields(m, p, F, nF))) return rc;
  if ((rc = upload_velocity(m, F, nF))) return rc;
  std::vector<int> sel(w->nsys, 1);
  if ((rc = set_sel(m, sel))) return rc;
  ua_params q = *p;
  q.profile = 0;
  // candidates: the default shape first; P2 elements run 128-thread CTAs only
  const PatchShape shapes[] = {{600, 128}, {300, 128}, {150, 128}, {1200, 128}, {300, 64}, {150, 64}, {0, 48}};
  // P1 schedules (CTA size, register budget); P2 elements run 128-thread CTAs of one budget
  const int sched[5][2] = {{256, 128}, {128, 128}, {128, 96}, {256, 80}, {128, 80}};
  const int nsched = m->nod == 3 ? 5 : 1;
  std::memset(rep, 0, sizeof(*rep));
  const PatchShape keep_shape = m->patch_shape;
  const int keep_threads = m->asm_threads, keep_regs = m->asm_regs;
  cudaEvent_t e0, e1;
  UA_CUDA_TRY(cudaEventCreate(&e0));
  UA_CUDA_TRY(cudaEventCreate(&e1));
  int best = -1;
  for (const PatchShape& sh : shapes) {
    if ((rc = rebuild_patches(m, sh))) break;
    for (int ti = 0; ti < nsched && rep->n_candidates < UA_TUNE_MAX; ++ti) {
      m->asm_threads = m->nod == 3 ? sched[ti][0] : 128;
      m->asm_regs = sched[ti][1];
      if ((rc = assemble(m, &q, true, false, w->X, false))) break;  // warm-up
      UA_CUDA_TRY(cudaEventRecord(e0, m->stream));
      for (int r = 0; r < reps && !rc; ++r) rc = assemble(m, &q, true, false, w->X, false);
      if (rc) break;
      UA_CUDA_TRY(cudaEventRecord(e1, m->stream));
      UA_CUDA_TRY(cudaEventSynchronize(e1));
      float ms = 0;
      UA_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
      const int k = rep->n_candidates++;
      rep->div[k] = sh.div; rep->cap[k] = sh.cap; rep->threads[k] = m->asm_threads; rep->regs[k] = m->asm_regs;
      rep->ms[k] = ms / reps;
      if (best < 0 || rep->ms[k] < rep->ms[best]) best = k;
    }
    if (rc) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc || best < 0) {  // leave the handle as it was
    m->asm_threads = keep_threads;
    m->asm_regs = keep_regs;
    int rc2 = rebuild_patches(m, keep_shape);
    return rc ? rc : (rc2 ? rc2 : set_error(UA_ERR_INVALID, "ua_autotune: no candidate ran"));
  }
  AsmTuning t;
  t.shape = PatchShape{rep->div[best], rep->cap[best]};
  t.threads = rep->threads[best];
  t.regs = rep->regs[best];
  if ((rc = rebuild_patches(m, t.shape))) return rc;
  m->asm_threads = t.threads;
  m->asm_regs = t.regs;
  set_tuned_assembly(m->device, m->nod, m->ndof, t);
  rep->chosen = best;
  rep->default_ms = rep->ms[0];
  return UA_OK;
}

static int newton_common(ua_mesh* m, const ua_params* p, ua_fields* F, const ua_bcs* bcs, int nF,
                         std::vector<ua_newton_report*>& rep, double** lam_io, const int* nl_io) {
  if (m->ndof != 2) return set_error(UA_ERR_INVALID, "uv Newton needs a ndof=2 mesh handle");
  UA_CUDA_TRY(cudaSetDevice(m->device));
  int rc;
  double t0 = now_ms();
  if ((rc = ensure_work(m, p))) return rc;
  if ((rc = ensure_K(m, p->precision))) return rc;
  if ((rc = upload_fields(m, p, F, nF))) return rc;
  if ((rc = upload_velocity(m, F, nF))) return rc;
  if ((rc = build_constraints(m, bcs, nF))) return rc;
  Work* w = m->work;
  const int nsys = w->nsys;
  g_launches = 0;
  w->prof.reset();
  w->prof.on = p->profile != 0;
  cudaEvent_t call_ev[2];
  {
    bool on = w->prof.on;
    w->prof.on = true;
    call_ev[0] = w->prof.get();
    call_ev[1] = w->prof.get();
    w->prof.on = on;
  }
  UA_CUDA_TRY(cudaEventRecord(call_ev[0], m->stream));
  // Lagrange multipliers l.ubvb (:35-39): zero unless the caller's vector matches
  if (w->nc) UA_CUDA_TRY(cudaMemsetAsync(w->lam, 0, w->nc * sizeof(double), m->stream));
  for (int s = 0; s < nsys && lam_io; ++s) {
    int nc_s = w->h_sys_con_off[s + 1] - w->h_sys_con_off[s];
    if (lam_io[s] && nl_io[s] == nc_s && nc_s > 0)
      UA_CUDA_TRY(cudaMemcpyAsync(w->lam + w->h_sys_con_off[s], lam_io[s], nc_s * sizeof(double),
                                  cudaMemcpyHostToDevice, m->stream));
  }
  for (auto r : rep)
    if (r) reset_report(r);
  if ((rc = check_update_stride(m, rep))) return rc;
  std::vector<SysState> st(nsys);
  std::vector<int> run(nsys, 1);
  if ((rc = newton_run(m, p, run, rep, st))) return rc;
  // uv.m:107-112: reset u=v=l=0 and solve again once
  std::vector<int> retry(nsys, 0);
  bool any = false;
  for (int s = 0; s < nsys; ++s)
    if (!st[s].converged) { retry[s] = 1; any = true; }
  if (any) {
    for (int s = 0; s < nsys; ++s) {
      if (!retry[s]) continue;
      const int d0 = m->h_dof_off[s], nd = m->h_dof_off[s + 1] - d0;
      UA_CUDA_TRY(cudaMemsetAsync(w->X + d0, 0, nd * sizeof(double), m->stream));
      int c0 = w->h_sys_con_off[s], nc_s = w->h_sys_con_off[s + 1] - c0;
      if (nc_s) UA_CUDA_TRY(cudaMemsetAsync(w->lam + c0, 0, nc_s * sizeof(double), m->stream));
      if (rep[s]) rep[s]->retried = 1;
    }
    if ((rc = newton_run(m, p, retry, rep, st))) return rc;
  }
  // results back
  for (int s = 0; s < nsys; ++s) {
    ua_fields& f = F[nF == 1 ? 0 : s];
    const int d0 = m->h_dof_off[s], nn = m->sys[s].nn;
    auto kind = f.location == UA_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    UA_CUDA_TRY(cudaMemcpyAsync(f.ub_out ? f.ub_out : f.ub, w->X + d0, nn * sizeof(double), kind, m->stream));
    UA_CUDA_TRY(cudaMemcpyAsync(f.vb_out ? f.vb_out : f.vb, w->X + d0 + nn, nn * sizeof(double), kind, m->stream));
    if (lam_io && lam_io[s]) {
      int nc_s = w->h_sys_con_off[s + 1] - w->h_sys_con_off[s];
      if (nl_io[s] >= nc_s && nc_s > 0)
        UA_CUDA_TRY(cudaMemcpyAsync(lam_io[s], w->lam + w->h_sys_con_off[s], nc_s * sizeof(double),
                                    cudaMemcpyDeviceToHost, m->stream));
    }
  }
  UA_CUDA_TRY(cudaEventRecord(call_ev[1], m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  double t1 = now_ms();
  float dev_ms = 0;
  cudaEventElapsedTime(&dev_ms, call_ev[0], call_ev[1]);
  double kms[PK_COUNT] = {}, knnz[PK_COUNT] = {}, krows[PK_COUNT] = {};
  int kn[PK_COUNT] = {};
  prof_collect(w, kms, kn, knnz, krows);
  bool all_conv = true;
  for (int s = 0; s < nsys; ++s) {
    if (rep[s]) {
      rep[s]->total_ms = t1 - t0;
      rep[s]->device_ms = dev_ms;
      prof_report(rep[s], kms, kn, knnz, krows);
      rep[s]->gpu_launches = (int)g_launches;
    }
    all_conv = all_conv && st[s].converged;
  }
  return all_conv ? UA_OK : UA_ERR_NOT_CONVERGED;
}

extern "C" int ua_uv_newton(ua_mesh* m, const ua_params* p, ua_fields* F, const ua_bcs* bcs, double* lubvb,
                            int32_t nl, ua_newton_report* rep, double* Kvals, double* R) {
  if (!m || !p || !F) return set_error(UA_ERR_INVALID, "ua_uv_newton: null argument");
  if (m->dm.nsys != 1) return set_error(UA_ERR_INVALID, "ua_uv_newton takes a single-mesh handle");
  std::vector<ua_newton_report*> reps(1, rep);
  double* lam[1] = {lubvb};
  int nls[1] = {nl};
  m->keep_last_tangent = Kvals != nullptr;
  int rc = newton_common(m, p, F, bcs, 1, reps, lam, nls);
  m->keep_last_tangent = false;
  if (rc != UA_OK && rc != UA_ERR_NOT_CONVERGED) return rc;
  Work* w = m->work;
  if (R) UA_CUDA_TRY(cudaMemcpy(R, w->R, m->ndof_total * sizeof(double), cudaMemcpyDeviceToHost));
  if (Kvals) {
    if (p->precision == UA_PREC_MIXED) {
      std::vector<float> tmp(m->nnz_total);
      UA_CUDA_TRY(cudaMemcpy(tmp.data(), w->Kf, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < tmp.size(); ++i) Kvals[i] = tmp[i];
    } else {
      UA_CUDA_TRY(cudaMemcpy(Kvals, w->Kd, m->nnz_total * sizeof(double), cudaMemcpyDeviceToHost));
    }
  }
  return rc;
}

extern "C" int ua_uv_newton_batch(ua_mesh* m, const ua_params* p, ua_fields* fields, const ua_bcs* bcs,
                                  ua_newton_report* reports) {
  if (!m || !p || !fields) return set_error(UA_ERR_INVALID, "ua_uv_newton_batch: null argument");
  std::vector<ua_newton_report*> reps(m->dm.nsys);
  for (int s = 0; s < m->dm.nsys; ++s) reps[s] = reports ? &reports[s] : nullptr;
  return newton_common(m, p, fields, bcs, m->dm.nsys, reps, nullptr, nullptr);
}

extern "C" int ua_constraint_count(const ua_mesh* m, const ua_bcs* bcs, int32_t ndof, int32_t* nc) {
  if (!m || !nc) return set_error(UA_ERR_INVALID, "null argument");
  int n = 0;
  if (bcs) {
    for (int comp = 0; comp < 2; ++comp) {
      int k = comp == 0 ? bcs->n_ufixed : bcs->n_vfixed;
      const int* nodes = comp == 0 ? bcs->ufixed_node : bcs->vfixed_node;
      std::vector<int> v(nodes, nodes + k);
      std::sort(v.begin(), v.end());
      n += (int)(std::unique(v.begin(), v.end()) - v.begin());
    }
    n += bcs->n_utied + bcs->n_vtied + bcs->n_normal;
    if (ndof == 3) n += bcs->n_hfixed;
  }
  *nc = n;
  return UA_OK;
}

extern "C" int ua_constraint_matrix(const ua_mesh* m, const ua_bcs* bcs, int32_t* nc, int32_t* dof, double* val,
                                    double* rhs) {
  if (!m || !nc) return set_error(UA_ERR_INVALID, "ua_constraint_matrix: null argument");
  if (m->dm.nsys != 1) return set_error(UA_ERR_INVALID, "ua_constraint_matrix takes a single-mesh handle");
  std::vector<int> cd, cs, off, cd2;
  std::vector<double> r, v1, v2;
  if (int rc = constraint_rows(m, bcs, 1, cd, cs, r, off, &cd2, &v1, &v2)) return rc;
  *nc = (int32_t)cd.size();
  for (size_t k = 0; k < cd.size(); ++k) {
    if (dof) { dof[2 * k] = cd[k]; dof[2 * k + 1] = cd2[k]; }
    if (val) { val[2 * k] = v1[k]; val[2 * k + 1] = v2[k]; }
    if (rhs) rhs[k] = r[k];
  }
  return UA_OK;
}

extern "C" void ua_mesh_destroy(ua_mesh* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  if (m->work) {
    Work* w = m->work;
    delete w->serve;
    for (auto& e : w->pcg_exec)
      if (e) cudaGraphExecDestroy(e);
    if (w->h_sysv) cudaFreeHost(w->h_sysv);
    if (w->h_int) cudaFreeHost(w->h_int);
    if (w->h_nan) cudaFreeHost(w->h_nan);
    if (w->h_gamma) cudaFreeHost(w->h_gamma);
    delete w;
  }
  amg_free(m->amg);
  m->amg = nullptr;
  dev_free_all(m);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

// solveKApeSymmetric.m:71-113 -> ABfgPreEliminate.m:29-160 for an SPD A with
// selection-type constraints (one non-zero per row of L): x_d = g/l on the
// constrained dofs, projected PCG on the rest, y = (f - A x)_d / l
// (ABfgPreEliminate.m:138 with the ScaleL factor undone as at :159).
extern "C" int ua_solve_kape_symmetric(int32_t n, const int64_t* Arowptr, const int64_t* Acol, const double* Aval,
                                       int32_t nl, const int64_t* Lrowptr, const int64_t* Lcol, const double* Lval,
                                       const double* f, const double* g, double* x, double* y, double rtol,
                                       int32_t maxit, int32_t* its, int32_t device) {
  if (n <= 0 || !Arowptr || !Acol || !Aval || !f || !x) return set_error(UA_ERR_INVALID, "ua_solve_kape_symmetric: bad arguments");
  if (nl > 0 && (!Lrowptr || !Lcol || !Lval || !g || !y)) return set_error(UA_ERR_INVALID, "constraint arrays missing");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return set_error(UA_ERR_NO_DEVICE, "no CUDA device"); }
  UA_CUDA_TRY(cudaSetDevice(device));
  const long long nnz = Arowptr[n] - Arowptr[0];
  if (nnz >= (1LL << 31)) return set_error(UA_ERR_INVALID, "too many non-zeros");
  std::vector<int> rowptr(n + 1), col(nnz), diagpos(n, -1);
  for (int i = 0; i <= n; ++i) rowptr[i] = (int)(Arowptr[i] - Arowptr[0]);
  for (long long j = 0; j < nnz; ++j) {
    long long c = Acol[Arowptr[0] + j];
    if (c < 0 || c >= n) return set_error(UA_ERR_INVALID, "column index out of range");
    col[j] = (int)c;
  }
  for (int i = 0; i < n; ++i)
    for (int j = rowptr[i]; j < rowptr[i + 1]; ++j)
      if (col[j] == i) diagpos[i] = j;
  std::vector<int> con_dof;
  std::vector<double> con_rhs, con_l;
  std::vector<unsigned char> cmask(n, 0);
  std::vector<int> dof_con(n, -1);
  for (int c = 0; c < nl; ++c) {
    if (Lrowptr[c + 1] - Lrowptr[c] != 1)
      return set_error(UA_ERR_INVALID, "constraint row %d: only single-entry rows are supported", c);
    long long d = Lcol[Lrowptr[c]];
    double l = Lval[Lrowptr[c]];
    if (d < 0 || d >= n || l == 0) return set_error(UA_ERR_INVALID, "constraint row %d: bad entry", c);
    if (cmask[d]) return set_error(UA_ERR_INVALID, "B*B' not diagonal (dof %lld constrained twice)", d);
    cmask[d] = 1; dof_con[d] = c;
    con_dof.push_back((int)d); con_rhs.push_back(g[c] / l); con_l.push_back(l);
  }
  for (int i = 0; i < n; ++i)
    if (diagpos[i] < 0 && !cmask[i]) return set_error(UA_ERR_INVALID, "row %d has no diagonal entry", i);
    else if (diagpos[i] < 0) diagpos[i] = rowptr[i];
  // a one-system scratch handle
  ua_mesh tmp;
  tmp.device = device; tmp.ndof = 2; tmp.nod = 6; tmp.ndof_total = n; tmp.nnz_total = nnz;
  tmp.dm.nsys = 1;
  tmp.h_dof_off = {0, n};
  int rc = UA_OK;
  Work* w = new Work();
  w->no_graph = true;  // a one-off solve: nothing to replay
  tmp.work = w;
  UA_CUDA_TRY(cudaStreamCreateWithFlags(&tmp.stream, cudaStreamNonBlocking));
  auto cleanup = [&]() {
    cudaStreamSynchronize(tmp.stream);
    if (w->h_sysv) cudaFreeHost(w->h_sysv);
    if (w->h_int) cudaFreeHost(w->h_int);
    if (w->h_nan) cudaFreeHost(w->h_nan);
    if (w->h_gamma) cudaFreeHost(w->h_gamma);
    delete w;
    tmp.work = nullptr;
    dev_free_all(&tmp);
    cudaStreamDestroy(tmp.stream);
  };
  {
    w->nsys = 1;
    std::vector<int> rb_start, rb_sys;
    for (int r = 0; r < n; r += kRB) { rb_start.push_back(r); rb_sys.push_back(0); }
    w->nrb = (int)rb_sys.size();
    rb_start.push_back(n);
    w->h_sys_rb_off = {0, w->nrb};
    std::vector<int> sel1 = {1}, coff = {0, (int)con_dof.size()}, csys(con_dof.size(), 0);
    auto up_i = [&](const std::vector<int>& v) { int* d = walloc<int>(&tmp, v.size()); if (d) cudaMemcpy(d, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice); return d; };
    auto up_d = [&](const double* v, size_t k) { double* d = walloc<double>(&tmp, k); if (d && k) cudaMemcpy(d, v, k * sizeof(double), cudaMemcpyHostToDevice); return d; };
    w->rb_start = up_i(rb_start); w->rb_sys = up_i(rb_sys); w->sys_rb_off = up_i(w->h_sys_rb_off);
    w->rowptr = up_i(rowptr); w->colind = up_i(col); w->diagpos = up_i(diagpos);
    w->Kd = up_d(Aval + Arowptr[0], nnz);
    w->frhs = up_d(f, n);
    w->X = walloc<double>(&tmp, n); w->dX = walloc<double>(&tmp, n);
    void** kv[] = {&w->kr, &w->kz, &w->kp, &w->kq, &w->invd};
    for (auto v : kv) *v = walloc<double>(&tmp, n);
    w->part = walloc<double>(&tmp, 4 * (size_t)w->nrb);
    w->sysv = walloc<double>(&tmp, SV_COUNT);
    w->done = walloc<int>(&tmp, 1); w->its = walloc<int>(&tmp, 1); w->status = walloc<int>(&tmp, 1);
    w->sel = up_i(sel1);
    w->cmask = walloc<unsigned char>(&tmp, n);
    w->dof_con = up_i(dof_con);
    w->nc = (int)con_dof.size();
    if (w->nc) {
      w->con_dof = up_i(con_dof); w->con_sys = up_i(csys); w->sys_con_off = up_i(coff);
      w->con_rhs = up_d(con_rhs.data(), w->nc);
      w->dlam = walloc<double>(&tmp, w->nc); w->grhs = walloc<double>(&tmp, w->nc);
    }
    if (!w->Kd || !w->X || !w->dX || !w->kr || !w->kz || !w->kp || !w->kq || !w->invd || !w->part || !w->cmask ||
        cudaMallocHost(&w->h_sysv, SV_COUNT * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&w->h_int, 8 * sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&w->h_gamma, sizeof(double)) != cudaSuccess) {
      cleanup();
      return set_error(UA_ERR_OOM, "allocation failed");
    }
    cudaMemcpy(w->cmask, cmask.data(), n, cudaMemcpyHostToDevice);
    cudaMemset(w->X, 0, n * sizeof(double));
    ua_params p;
    ua_params_default(&p);
    p.krylov_rtol = rtol > 0 ? rtol : 1e-12;
    p.krylov_maxit = maxit > 0 ? maxit : 10 * n + 100;
    p.krylov_precond = UA_PC_JACOBI;  // a bare matrix has no mesh to aggregate
    std::vector<int> kits(1, 1);
    rc = pcg_t<double, double>(&tmp, &p, w->Kd, kits.data());
    if (rc == UA_OK) {
      std::vector<double> dl(w->nc);
      int st = 0;
      cudaMemcpy(x, w->dX, n * sizeof(double), cudaMemcpyDeviceToHost);
      if (w->nc) cudaMemcpy(dl.data(), w->dlam, w->nc * sizeof(double), cudaMemcpyDeviceToHost);
      cudaMemcpy(&st, w->status, sizeof(int), cudaMemcpyDeviceToHost);
      for (int c = 0; c < w->nc; ++c) y[c] = dl[c] / con_l[c];
      if (its) *its = kits[0];
      if (st) rc = set_error(UA_ERR_KRYLOV, "PCG breakdown: A is not positive definite on the free dofs");
    }
  }
  cleanup();
  return rc;
}

// ---------------------------------------------------------------------------
// Allocation-free constrained PCG solve.
//
// For callers that cannot allocate device memory themselves: a MEX file that
// works on gpuArray data (MATLAB owns the device allocator and its memory
// pool), a plugin inside a host application that forbids cudaMalloc on its
// solve path, or a code running under a fixed device-memory budget.  Inputs
// and outputs are the caller's device arrays; every temporary (Krylov
// vectors, partial sums, constraint masks, per-solve scalars) lives in the
// file-scope array g_na_scratch, sized for at most UA_NOALLOC_MAX_ROWS
// unknowns and UA_NOALLOC_MAX_CONSTRAINTS constraint rows (about 8.5 MB).
// Every device that loads the library holds this array until the process
// exits.  All calls on a device share it and each call overwrites it, so
// calls that overlap on the GPU (two host threads, or calls queued on
// different streams) race and must be serialised by the caller.  The first
// call on a device looks up the array's device address with
// cudaGetSymbolAddress (make that first call before any stream capture);
// later calls reuse the address.  Work is queued on cudaStreamPerThread.
// ---------------------------------------------------------------------------
constexpr size_t kNaAlign = 256;
constexpr size_t na_align(size_t b) { return (b + kNaAlign - 1) & ~(kNaAlign - 1); }
constexpr int kNaMaxRb = (UA_NOALLOC_MAX_ROWS + kRB - 1) / kRB;
constexpr int kNaSmallInts = 2 * kNaMaxRb + 16;
constexpr size_t kNaScratchBytes =
    na_align(6 * sizeof(double) * (size_t)UA_NOALLOC_MAX_ROWS) +        // X, r, z, p, q, invd
    na_align(2 * sizeof(int) * (size_t)UA_NOALLOC_MAX_ROWS) +           // diagpos, dof_con
    na_align((size_t)UA_NOALLOC_MAX_ROWS) +                             // cmask
    na_align(sizeof(int) * (size_t)kNaSmallInts) +                      // row blocks, offsets, flags
    na_align(sizeof(double) * (4 * (size_t)kNaMaxRb + SV_COUNT)) +     // partial sums, scalars
    na_align(2 * sizeof(int) * (size_t)UA_NOALLOC_MAX_CONSTRAINTS) +    // con_dof, con_sys
    na_align(3 * sizeof(double) * (size_t)UA_NOALLOC_MAX_CONSTRAINTS);  // con_rhs, dlam, grhs

static __device__ __align__(256) unsigned char g_na_scratch[kNaScratchBytes];

constexpr int kNaMaxDevices = 64;
// device address of g_na_scratch per device, looked up once; atomic because
// host threads may make their first call on a device at the same time
static std::atomic<void*> g_na_addr[kNaMaxDevices];

// Clears the per-call state and checks the caller's CSR (flags are zeroed by
// the host before this launch).  flags[0]: a free row has no diagonal entry;
// flags[1]: a dof is constrained twice (B*B' not diagonal); flags[2]: a
// constraint entry is out of range or zero; flags[3]: the CSR of A is
// malformed (a column outside [0,n), a negative or decreasing row pointer,
// or no non-zero at all), so no later kernel may index with it.
__global__ void k_na_setup(int n, const int* rowptr, const int* col, int* diagpos, unsigned char* cmask,
                           int* dof_con, double* X, int* rb_start, int* rb_sys, int nrb, int* sys_rb_off,
                           int* sys_con_off, int nl, int* sel, int* flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    int dp = -1;
    const int r0 = rowptr[i], r1 = rowptr[i + 1];
    if (r0 < 0 || r1 < r0) {
      atomicExch(&flags[3], 1);
    } else {
      for (int j = r0; j < r1; ++j) {
        const int c = col[j];
        if (c < 0 || c >= n) atomicExch(&flags[3], 1);
        else if (c == i) dp = j;
      }
    }
    diagpos[i] = dp;
    cmask[i] = 0;
    dof_con[i] = -1;
    X[i] = 0.0;
  }
  if (i <= nrb) rb_start[i] = i < nrb ? i * kRB : n;
  if (i < nrb) rb_sys[i] = 0;
  if (i == 0) {
    sys_rb_off[0] = 0; sys_rb_off[1] = nrb;
    sys_con_off[0] = 0; sys_con_off[1] = nl;
    sel[0] = 1;
    if (rowptr[n] <= rowptr[0]) atomicExch(&flags[3], 1);
  }
}

__global__ void k_na_constraints(int n, int nl, const int* Ldof, const double* Lval, const double* g,
                                 unsigned char* cmask, int* dof_con, int* con_dof, int* con_sys, double* con_rhs,
                                 int* flags) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nl) return;
  const int d = Ldof[c];
  const double l = Lval[c];
  con_sys[c] = 0;
  if (d < 0 || d >= n || l == 0.0) {
    atomicExch(&flags[2], 1);
    con_dof[c] = 0;
    con_rhs[c] = 0;
    return;
  }
  if (atomicCAS(&dof_con[d], -1, c) != -1) atomicExch(&flags[1], 1);
  cmask[d] = 1;
  con_dof[c] = d;
  con_rhs[c] = g[c] / l;  // x_d = g/l (ABfgPreEliminate.m:63 with the row scaled to unit norm)
}

__global__ void k_na_check_diag(int n, const unsigned char* cmask, int* diagpos, const int* rowptr, int* flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || diagpos[i] >= 0) return;
  if (!cmask[i]) atomicExch(&flags[0], 1);
  // constrained row without entries: any valid index (the set-up rejects a CSR without non-zeros);
  // the value read is not used
  diagpos[i] = rowptr[i] < rowptr[n] ? rowptr[i] : rowptr[0];
}

__global__ void k_na_multiplier(int nl, const double* dlam, const double* Lval, double* y) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nl) y[c] = dlam[c] / Lval[c];
}

extern "C" int ua_solve_kape_symmetric_noalloc(int32_t n, const int32_t* Arowptr, const int32_t* Acol,
                                               const double* Aval, int32_t nl, const int32_t* Ldof,
                                               const double* Lval, const double* f, const double* g, double* x,
                                               double* y, double rtol, int32_t maxit, int32_t* its,
                                               int32_t device) {
  if (n <= 0 || n > UA_NOALLOC_MAX_ROWS)
    return set_error(UA_ERR_INVALID, "ua_solve_kape_symmetric_noalloc: n=%d is outside 1..%d (UA_NOALLOC_MAX_ROWS)",
                     n, UA_NOALLOC_MAX_ROWS);
  if (nl < 0 || nl > UA_NOALLOC_MAX_CONSTRAINTS)
    return set_error(UA_ERR_INVALID,
                     "ua_solve_kape_symmetric_noalloc: nl=%d is outside 0..%d (UA_NOALLOC_MAX_CONSTRAINTS)", nl,
                     UA_NOALLOC_MAX_CONSTRAINTS);
  if (!Arowptr || !Acol || !Aval || !f || !x || (nl > 0 && (!Ldof || !Lval || !g || !y)))
    return set_error(UA_ERR_INVALID, "ua_solve_kape_symmetric_noalloc: null device pointer");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(UA_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= ndev || device >= kNaMaxDevices) return set_error(UA_ERR_INVALID, "bad device ordinal %d", device);
  UA_CUDA_TRY(cudaSetDevice(device));
  void* na_base = g_na_addr[device].load(std::memory_order_acquire);
  if (!na_base) {  // once per device, with that device current
    UA_CUDA_TRY(cudaGetSymbolAddress(&na_base, g_na_scratch));
    g_na_addr[device].store(na_base, std::memory_order_release);
  }
  // carve the scratch array
  unsigned char* base = (unsigned char*)na_base;
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    void* q = base + off;
    off += na_align(bytes);
    return q;
  };
  const size_t R = UA_NOALLOC_MAX_ROWS, Cn = UA_NOALLOC_MAX_CONSTRAINTS;
  double* vec = (double*)carve(6 * sizeof(double) * R);
  int* ivec = (int*)carve(2 * sizeof(int) * R);
  unsigned char* cmask = (unsigned char*)carve(R);
  int* small = (int*)carve(sizeof(int) * kNaSmallInts);
  double* dsmall = (double*)carve(sizeof(double) * (4 * (size_t)kNaMaxRb + SV_COUNT));
  int* con_i = (int*)carve(2 * sizeof(int) * Cn);
  double* con_d = (double*)carve(3 * sizeof(double) * Cn);
  const int nrb = (n + kRB - 1) / kRB;

  // a one-system view: scratch for temporaries, the caller's arrays in place
  ua_mesh view;
  view.device = device;
  view.ndof = 2;
  view.nod = 6;
  view.ndof_total = n;
  view.dm.nsys = 1;
  view.stream = cudaStreamPerThread;
  Work w;
  w.no_graph = true;  // no graph instantiation (it may allocate)
  static thread_local double h_sysv[SV_COUNT];
  static thread_local int h_int[8];
  w.nsys = 1; w.nrb = nrb; w.nc = nl;
  w.X = vec; w.kr = vec + R; w.kz = vec + 2 * R; w.kp = vec + 3 * R; w.kq = vec + 4 * R; w.invd = vec + 5 * R;
  w.diagpos = ivec; w.dof_con = ivec + R;
  w.cmask = cmask;
  w.rb_start = small;                          // kNaMaxRb + 1
  w.rb_sys = small + kNaMaxRb + 1;             // kNaMaxRb
  w.sys_rb_off = small + 2 * kNaMaxRb + 1;     // 2
  w.sys_con_off = small + 2 * kNaMaxRb + 3;    // 2
  w.sel = small + 2 * kNaMaxRb + 5;
  w.done = small + 2 * kNaMaxRb + 6;
  w.its = small + 2 * kNaMaxRb + 7;
  w.status = small + 2 * kNaMaxRb + 8;
  int* flags = small + 2 * kNaMaxRb + 9;       // 4
  w.part = dsmall; w.sysv = dsmall + 4 * kNaMaxRb;
  w.con_dof = con_i; w.con_sys = con_i + Cn;
  w.con_rhs = con_d; w.dlam = con_d + Cn; w.grhs = con_d + 2 * Cn;
  w.rowptr = const_cast<int*>(Arowptr);
  w.colind = const_cast<int*>(Acol);
  w.Kd = const_cast<double*>(Aval);
  w.frhs = const_cast<double*>(f);
  w.dX = x;
  w.h_sysv = h_sysv;
  w.h_int = h_int;
  view.work = &w;
  cudaStream_t st = view.stream;
  const int nb = (std::max(n, nrb + 1) + 255) / 256;
  if (cudaMemsetAsync(flags, 0, 4 * sizeof(int), st) != cudaSuccess) {
    view.work = nullptr;
    return set_error(UA_ERR_CUDA, "no-alloc set-up failed");
  }
  k_na_setup<<<nb, 256, 0, st>>>(n, Arowptr, Acol, w.diagpos, cmask, w.dof_con, w.X, w.rb_start, w.rb_sys, nrb,
                                 w.sys_rb_off, w.sys_con_off, nl, w.sel, flags);
  if (nl)
    k_na_constraints<<<(nl + 255) / 256, 256, 0, st>>>(n, nl, Ldof, Lval, g, cmask, w.dof_con, w.con_dof, w.con_sys,
                                                      w.con_rhs, flags);
  k_na_check_diag<<<(n + 255) / 256, 256, 0, st>>>(n, cmask, w.diagpos, Arowptr, flags);
  int rc = UA_OK;
  int hf[4] = {0, 0, 0, 0};
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    view.work = nullptr;
    return set_error(UA_ERR_CUDA, "no-alloc set-up failed");
  }
  if (hf[3])
    rc = set_error(UA_ERR_INVALID,
                   "A's CSR is invalid: a column index outside [0,n), a negative or decreasing row pointer, "
                   "or no non-zeros");
  else if (hf[2]) rc = set_error(UA_ERR_INVALID, "constraint row with a dof out of range or a zero coefficient");
  else if (hf[1]) rc = set_error(UA_ERR_INVALID, "B*B' not diagonal (a dof constrained twice)");
  else if (hf[0]) rc = set_error(UA_ERR_INVALID, "a free row has no diagonal entry");
  if (rc == UA_OK) {
    ua_params p;
    ua_params_default(&p);
    p.krylov_rtol = rtol > 0 ? rtol : 1e-12;
    p.krylov_maxit = maxit > 0 ? maxit : 10 * n + 100;
    p.krylov_precond = UA_PC_JACOBI;  // a bare matrix has no mesh to aggregate (and no allocation here)
    int kits[1] = {1};
    rc = pcg_t<double, double>(&view, &p, w.Kd, kits);
    if (rc == UA_OK) {
      if (nl) k_na_multiplier<<<(nl + 255) / 256, 256, 0, st>>>(nl, w.dlam, Lval, y), ++g_launches;
      int status = 0;
      if (cudaMemcpyAsync(&status, w.status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        rc = set_error(UA_ERR_CUDA, "no-alloc solve failed");
      else if (status)
        rc = set_error(UA_ERR_KRYLOV, "PCG breakdown: A is not positive definite on the free dofs");
      if (its) *its = kits[0];
    }
  }
  view.work = nullptr;
  return rc;
}

// Device work of the adjoint gradient and of the active-set reactions (mass matrix, vectors).
static int ensure_adj_buf(ua_mesh* m, size_t need) {
  Work* w = m->work;
  if (w->adj_cap >= need) return UA_OK;
  w->adj_buf = walloc<double>(m, need);
  if (!w->adj_buf) return set_error(UA_ERR_OOM, "device allocation of the adjoint work failed");
  w->adj_cap = need;
  return UA_OK;
}

// ---------------------------------------------------------------------------
// Adjoint gradient of the velocity misfit with respect to C (Misfit.m adjoint
// branch with "-uv-" data, dIdCq.m, ApplyAdjointGradientPreMultiplier.m).
// ---------------------------------------------------------------------------
extern "C" int ua_uv_adjoint_dIdC(ua_mesh* m, const ua_params* p, const ua_fields* F, const ua_bcs* bcs_adjoint,
                                  const ua_measurements* meas, int32_t flags, double* I, double* dIduv,
                                  double* lambda, double* dIdC, int32_t* krylov_its) {
  if (!m || !p || !F || !meas) return set_error(UA_ERR_INVALID, "ua_uv_adjoint_dIdC: null argument");
  if (m->ndof != 2 || m->dm.nsys != 1)
    return set_error(UA_ERR_INVALID, "ua_uv_adjoint_dIdC takes a single-mesh uv (ndof=2) handle");
  if (!meas->us || !meas->vs || !meas->usErr || !meas->vsErr)
    return set_error(UA_ERR_INVALID, "Misfit:us Meas.us, Meas.vs and their errors are required for -uv- data");
  if (p->SlidingLaw == UA_SLIDING_COULOMB)
    return set_error(UA_ERR_INVALID, "BasalDrag:InvalidCase inversion for C with the Coulomb sliding law is not "
                                     "implemented");
  UA_CUDA_TRY(cudaSetDevice(m->device));
  ua_params q = *p;  // the adjoint runs in FP64 at a fixed inner tolerance
  q.precision = UA_PREC_FP64;
  q.krylov_adaptive = 0;
  int rc;
  if ((rc = ensure_work(m, p))) return rc;
  if ((rc = ensure_K(m, UA_PREC_FP64))) return rc;
  if ((rc = upload_fields(m, &q, F, 1))) return rc;
  if ((rc = upload_velocity(m, F, 1))) return rc;
  if ((rc = build_constraints(m, bcs_adjoint, 1))) return rc;
  Work* w = m->work;
  const int nn = m->nn_total, N = m->ndof_total;
  const size_t nnzn = m->h_nodeptr.empty() ? 0 : (size_t)m->h_nodeptr.back();
  const size_t need = nnzn + 18 * (size_t)nn + 2 * (size_t)N + kAdjDotBlocks + 16;
  if ((rc = ensure_adj_buf(m, need))) return rc;
  double* Mval = w->adj_buf;
  double *us = Mval + nnzn, *vs = us + nn, *ue = vs + nn, *ve = ue + nn;
  double *ru = ve + nn, *rv = ru + nn, *Mru = rv + nn, *Mrv = Mru + nn, *gv = Mrv + nn, *gout = gv + nn;
  double* cgw = gout + nn;       // 6 nn + kAdjDotBlocks + 8
  double* xsave = cgw + 6 * (size_t)nn + kAdjDotBlocks + 8;  // N
  double* sc = cgw + 6 * (size_t)nn + kAdjDotBlocks;        // dot results (slots used here: 0, 1)
  const double* src[4] = {meas->us, meas->vs, meas->usErr, meas->vsErr};
  double* dst[4] = {us, vs, ue, ve};
  for (int k = 0; k < 4; ++k)
    UA_CUDA_TRY(cudaMemcpyAsync(dst[k], src[k], nn * sizeof(double),
                                F->location == UA_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                m->stream));
  // total area (CreateMUA.m:97-98): TriAreaFE over the corner nodes
  double area = 0.0;
  {
    const HostSystem& hs = m->sys[0];
    const int c1 = m->nod == 3 ? 1 : 2, c2 = m->nod == 3 ? 2 : 4;
    for (int e = 0; e < hs.ne; ++e) {
      const int a = hs.conn[e], b = hs.conn[(size_t)c1 * hs.ne + e], c = hs.conn[(size_t)c2 * hs.ne + e];
      area += 0.5 * std::fabs((hs.x[a] - hs.x[c]) * (hs.y[b] - hs.y[a]) - (hs.x[a] - hs.x[b]) * (hs.y[c] - hs.y[a]));
    }
  }
  // K at the state (the last Newton tangent the reference reuses as dfuv)
  std::vector<int> sel(1, 1);
  if ((rc = set_sel(m, sel))) return rc;
  if ((rc = assemble(m, &q, true, false, w->X, false))) return rc;
  // misfit and its gradient (Misfit.m:56-63, :117-120)
  UA_CUDA_TRY(adj_mass_matrix(m, Mval));
  UA_CUDA_TRY(adj_misfit(m, w->X, w->X + nn, us, vs, ue, ve, ru, rv));
  UA_CUDA_TRY(adj_node_spmv(m, m->dm.nodeptr, m->dm.nodecol, Mval, ru, Mru));
  UA_CUDA_TRY(adj_node_spmv(m, m->dm.nodeptr, m->dm.nodecol, Mval, rv, Mrv));
  UA_CUDA_TRY(adj_dot(m->stream, nn, ru, Mru, cgw + 6 * (size_t)nn, sc, 0));
  UA_CUDA_TRY(adj_dot(m->stream, nn, rv, Mrv, cgw + 6 * (size_t)nn, sc, 1));
  UA_CUDA_TRY(adj_misfit_grad(m, Mru, Mrv, ue, ve, area, w->frhs));
  g_launches += 8;
  double hs2[2];
  UA_CUDA_TRY(cudaMemcpyAsync(hs2, sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  // adjoint solve [K L'; L 0][lambda; mu] = [dI/duv; c] (Misfit.m:182-187): the constrained PCG
  // takes dX_c = c - X_c on the constrained dofs, so X is parked at zero for the solve
  UA_CUDA_TRY(cudaMemcpyAsync(xsave, w->X, N * sizeof(double), cudaMemcpyDeviceToDevice, m->stream));
  UA_CUDA_TRY(cudaMemsetAsync(w->X, 0, N * sizeof(double), m->stream));
  std::vector<int> its(1, 1);
  rc = pcg_t<double, double>(m, &q, w->Kd, its.data(), nullptr);
  UA_CUDA_TRY(cudaMemcpyAsync(w->X, xsave, N * sizeof(double), cudaMemcpyDeviceToDevice, m->stream));
  if (rc) return rc;
  int status = 0;
  UA_CUDA_TRY(cudaMemcpyAsync(&status, w->status, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  if (status) return set_error(UA_ERR_KRYLOV, "adjoint PCG breakdown: K is not positive definite on the free dofs");
  if (krylov_its) *krylov_its = its[0];
  if (I) *I = (hs2[0] + hs2[1]) / 2 / area;
  // dIdCq.m: the gradient assembly at (u, v, lambda)
  AdjIn in{w->h, w->S, w->B, w->rho, w->C, w->m, w->dragf[0], w->dragf[1], w->dragf[2],
           w->X, w->X + nn, w->dX, w->dX + nn, F->rhow, F->g};
  UA_CUDA_TRY(adj_dIdC(m, make_phys(&q), in, gv));
  ++g_launches;
  if (flags & UA_ADJ_LOGC) {
    UA_CUDA_TRY(adj_logc(m, w->C, gv));
    ++g_launches;
  }
  double* g = gv;
  if (flags & UA_ADJ_PREMUL_M) {  // (M/Area)\dIdC = Area (M\dIdC)
    double hsc[1];
    const int cits = adj_cg(m, m->dm.nodeptr, m->dm.nodecol, Mval, gv, gout, 1e-14, 20 * 1000, cgw, hsc);
    if (cits == -2) return set_error(UA_ERR_CUDA, "mass-matrix solve failed");
    if (cits == -1) return set_error(UA_ERR_KRYLOV, "mass-matrix CG reached its iteration cap");
    UA_CUDA_TRY(adj_scale(m, area, gout));
    g = gout;
  }
  if (dIduv) UA_CUDA_TRY(cudaMemcpyAsync(dIduv, w->frhs, N * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if (lambda) UA_CUDA_TRY(cudaMemcpyAsync(lambda, w->dX, N * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if (dIdC) UA_CUDA_TRY(cudaMemcpyAsync(dIdC, g, nn * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  return UA_OK;
}

// ---------------------------------------------------------------------------
// uvh C-ABI
// ---------------------------------------------------------------------------
extern "C" int ua_uvh_assemble(ua_mesh* m, const ua_params* p, const ua_fields* F, int32_t mode, double* R,
                               double* Kvals, double* Tint, double* Fext) {
  if (!m || !p || !F) return set_error(UA_ERR_INVALID, "ua_uvh_assemble: null argument");
  if (m->ndof != 3) return set_error(UA_ERR_INVALID, "ua_uvh_assemble needs a ndof=3 mesh handle");
  if (m->dm.nsys != 1) return set_error(UA_ERR_INVALID, "ua_uvh_assemble takes a single-mesh handle");
  if (mode != UA_ASM_R && mode != UA_ASM_RK && mode != UA_ASM_ZERO_R) return set_error(UA_ERR_INVALID, "bad mode");
  UA_CUDA_TRY(cudaSetDevice(m->device));
  int rc;
  if ((rc = ensure_work(m, p))) return rc;
  Work* w = m->work;
  const bool withK = mode == UA_ASM_RK;
  if (withK && (rc = ensure_K(m, UA_PREC_FP64))) return rc;
  if ((rc = upload_fields_uvh(m, p, F, 1))) return rc;
  std::vector<int> sel(1, 1);
  if ((rc = set_sel(m, sel))) return rc;
  if ((rc = assemble_uvh(m, p, withK, false, mode == UA_ASM_ZERO_R, Tint || Fext))) return rc;
  const int N = m->ndof_total;
  if (R) UA_CUDA_TRY(cudaMemcpyAsync(R, w->R, N * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if (Tint) UA_CUDA_TRY(cudaMemcpyAsync(Tint, w->Tint, N * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if (Fext) UA_CUDA_TRY(cudaMemcpyAsync(Fext, w->Fext, N * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if (withK && Kvals)
    UA_CUDA_TRY(cudaMemcpyAsync(Kvals, w->Kd, m->nnz_total * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  return UA_OK;
}

static int uvh_common(ua_mesh* m, const ua_params* p, ua_fields* F, const ua_bcs* bcs, int nF,
                      std::vector<ua_newton_report*>& rep, double* luvh, int32_t nl) {
  if (m->ndof != 3) return set_error(UA_ERR_INVALID, "uvh Newton needs a ndof=3 mesh handle");
  if (p->precision != UA_PREC_FP64) return set_error(UA_ERR_INVALID, "the uvh solve runs in FP64 only");
  UA_CUDA_TRY(cudaSetDevice(m->device));
  int rc;
  double t0 = now_ms();
  if ((rc = ensure_work(m, p))) return rc;
  if ((rc = ensure_K(m, UA_PREC_FP64))) return rc;
  if ((rc = upload_fields_uvh(m, p, F, nF))) return rc;
  if ((rc = build_constraints(m, bcs, nF))) return rc;
  Work* w = m->work;
  const int nsys = w->nsys;
  g_launches = 0;
  w->prof.reset();
  w->prof.on = p->profile != 0;
  cudaEvent_t call_ev[2];
  {
    bool on = w->prof.on;
    w->prof.on = true;
    call_ev[0] = w->prof.get();
    call_ev[1] = w->prof.get();
    w->prof.on = on;
  }
  UA_CUDA_TRY(cudaEventRecord(call_ev[0], m->stream));
  if (w->nc) UA_CUDA_TRY(cudaMemsetAsync(w->lam, 0, w->nc * sizeof(double), m->stream));
  if (luvh && nsys == 1 && nl == w->nc && nl > 0)
    UA_CUDA_TRY(cudaMemcpyAsync(w->lam, luvh, nl * sizeof(double), cudaMemcpyHostToDevice, m->stream));
  for (auto r : rep)
    if (r) reset_report(r);
  if ((rc = check_update_stride(m, rep))) return rc;
  std::vector<UvhSys> st(nsys);
  if ((rc = newton_run_uvh(m, p, rep, st))) return rc;
  for (int s = 0; s < nsys; ++s) {
    ua_fields& f = F[nF == 1 ? 0 : s];
    const int d0 = m->h_dof_off[s], nn = m->sys[s].nn;
    auto kind = f.location == UA_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    UA_CUDA_TRY(cudaMemcpyAsync(f.ub, w->X + d0, nn * sizeof(double), kind, m->stream));
    UA_CUDA_TRY(cudaMemcpyAsync(f.vb, w->X + d0 + nn, nn * sizeof(double), kind, m->stream));
    UA_CUDA_TRY(cudaMemcpyAsync(f.h1, w->X + d0 + 2 * nn, nn * sizeof(double), kind, m->stream));
  }
  if (luvh && nsys == 1 && nl >= w->nc && w->nc > 0)
    UA_CUDA_TRY(cudaMemcpyAsync(luvh, w->lam, w->nc * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  UA_CUDA_TRY(cudaEventRecord(call_ev[1], m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  float dev_ms = 0;
  cudaEventElapsedTime(&dev_ms, call_ev[0], call_ev[1]);
  double kms[PK_COUNT] = {}, knnz[PK_COUNT] = {}, krows[PK_COUNT] = {};
  int kn[PK_COUNT] = {};
  prof_collect(w, kms, kn, knnz, krows);
  bool all_conv = true;
  const double t1 = now_ms();
  for (int s = 0; s < nsys; ++s) {
    if (rep[s]) {
      rep[s]->total_ms = t1 - t0; rep[s]->device_ms = dev_ms;
      prof_report(rep[s], kms, kn, knnz, krows);
      rep[s]->gpu_launches = (int)g_launches;
    }
    all_conv = all_conv && st[s].converged;
  }
  return all_conv ? UA_OK : UA_ERR_NOT_CONVERGED;
}

// Sorted-set helpers with MATLAB's setdiff/setxor semantics (sorted unique results).
static std::vector<int> sorted_unique(std::vector<int> a) {
  std::sort(a.begin(), a.end());
  a.erase(std::unique(a.begin(), a.end()), a.end());
  return a;
}
static std::vector<int> set_diff(const std::vector<int>& a, const std::vector<int>& b) {
  std::vector<int> A = sorted_unique(a), B = sorted_unique(b), out;
  std::set_difference(A.begin(), A.end(), B.begin(), B.end(), std::back_inserter(out));
  return out;
}
static std::vector<int> set_xor(const std::vector<int>& a, const std::vector<int>& b) {
  std::vector<int> A = sorted_unique(a), B = sorted_unique(b), out;
  std::set_symmetric_difference(A.begin(), A.end(), B.begin(), B.end(), std::back_inserter(out));
  return out;
}

// uvh.m:64-212: the implicit step inside the active-set loop of minimum-thickness constraints
// (ActiveSetInitialisation.m, ActiveSetUpdate.m, CalculateReactions.m).  Host orchestration of
// device solves; the sets follow MATLAB's sorted setdiff, and the reactions pair the h
// multipliers with the re-sorted active set as CalculateReactions does.
static int uvh_active_set(ua_mesh* m, const ua_params* p, ua_fields* F, const ua_bcs* bcs, ua_newton_report* rep,
                          double* luvh, int32_t nl) {
  if (F->location != UA_HOST) return set_error(UA_ERR_INVALID, "the uvh active set takes host fields");
  if (!F->ub || !F->vb || !F->h1 || !F->rho) return set_error(UA_ERR_INVALID, "ua_uvh_newton: null field");
  const int nn = m->sys[0].nn;
  const double tmin = p->ThickMin, dt = F->dt;
  std::vector<double> ub(F->ub, F->ub + nn), vb(F->vb, F->vb + nn), h(F->h1, F->h1 + nn), rho(F->rho, F->rho + nn);
  std::vector<int> hfixed;
  std::vector<double> hfixv;
  for (int i = 0; bcs && i < bcs->n_hfixed; ++i) {
    hfixed.push_back(bcs->hfixed_node[i]);
    hfixv.push_back(bcs->hfixed_value ? bcs->hfixed_value[i] : 0.0);
  }
  std::vector<int> hpos_in;
  for (int i = 0; bcs && i < bcs->n_hpos; ++i) {
    const int k = bcs->hpos_node[i];
    if (k < 0 || k >= nn) return set_error(UA_ERR_INVALID, "hPosNode index %d out of range", k);
    hpos_in.push_back(k);
  }
  const int minnew = p->MinNumberOfNewlyIntroducedActiveThicknessConstraints;
  // ActiveSetInitialisation.m
  std::vector<int> hpos = set_diff(hpos_in, hfixed);
  const std::vector<int> last_active0 = hpos;
  if (*std::min_element(h.begin(), h.end()) > 1.1 * tmin) hpos.clear();
  if (hpos.empty()) {
    std::vector<int> thin;
    for (int i = 0; i < nn; ++i)
      if (h[i] < tmin) thin.push_back(i);
    hpos = set_diff(thin, hfixed);
  }
  std::vector<int> deact = set_diff(last_active0, hpos), act = set_diff(hpos, last_active0);
  if ((!deact.empty() || !act.empty()) && (int)deact.size() < minnew && (int)act.size() < minnew) {
    hpos = last_active0; deact.clear(); act.clear();
  }
  std::vector<int> last_released = deact, last_activated = act;
  // the consistent mass matrix for the reactions (MassMatrix2D1dof.m)
  int rc;
  UA_CUDA_TRY(cudaSetDevice(m->device));
  if ((rc = ensure_work(m, p))) return rc;
  const size_t nnzn = (size_t)m->h_nodeptr.back();
  if ((rc = ensure_adj_buf(m, nnzn + 9 * (size_t)nn + kAdjDotBlocks + 16))) return rc;
  double* Mval = m->work->adj_buf;
  double *d_rhs = Mval + nnzn, *d_r = d_rhs + nn, *cgw = d_r + nn;
  UA_CUDA_TRY(adj_mass_matrix(m, Mval));
  int it = 1, max_newton = 0, kits = 0;
  bool cyclical = false, as_conv = true;
  std::vector<double> lam;
  ua_fields f = *F;
  f.ub = ub.data(); f.vb = vb.data(); f.h1 = h.data();
  int solve_rc = UA_OK;
  while (true) {
    for (int k : hpos) h[k] = tmin;
    std::vector<int> hf2 = hfixed;
    std::vector<double> hv2 = hfixv;
    for (int k : hpos) { hf2.push_back(k); hv2.push_back(tmin); }
    ua_bcs b2{};
    if (bcs) b2 = *bcs;
    b2.n_hfixed = (int32_t)hf2.size(); b2.hfixed_node = hf2.data(); b2.hfixed_value = hv2.data();
    b2.n_hpos = 0; b2.hpos_node = nullptr;
    int32_t nc = 0;
    if ((rc = ua_constraint_count(m, &b2, 3, &nc))) return rc;
    lam.assign(std::max(nc, 1), 0.0);
    std::vector<ua_newton_report*> reps(1, rep);
    solve_rc = uvh_common(m, p, &f, &b2, 1, reps, lam.data(), nc);
    if (rep) { max_newton = std::max(max_newton, rep->iterations); kits += rep->krylov_its_total; }
    if (solve_rc == UA_ERR_NOT_CONVERGED) break;
    if (solve_rc) return solve_rc;
    for (int k : hpos)
      if (h[k] < tmin) h[k] = tmin;
    // ActiveSetUpdate.m
    hpos = set_diff(hpos, hfixed);
    const std::vector<int> last_set = hpos;
    const int nuv = nc - (int)hf2.size();
    std::vector<int> released;
    if (!hpos.empty()) {
      std::vector<double> rhs(nn, 0.0), r(nn, 0.0);
      for (size_t k = 0; k < hfixed.size(); ++k) rhs[hfixed[k]] += lam[nuv + k];
      for (size_t k = 0; k < last_set.size(); ++k) rhs[last_set[k]] += lam[nuv + hfixed.size() + k];
      UA_CUDA_TRY(cudaMemcpyAsync(d_rhs, rhs.data(), nn * sizeof(double), cudaMemcpyHostToDevice, m->stream));
      double hsc[1];
      const int cits = adj_cg(m, m->dm.nodeptr, m->dm.nodecol, Mval, d_rhs, d_r, 1e-14, 20000, cgw, hsc);
      if (cits < 0) return set_error(UA_ERR_KRYLOV, "mass-matrix solve of the thickness reactions failed");
      UA_CUDA_TRY(cudaMemcpyAsync(r.data(), d_r, nn * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
      UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
      std::vector<int> keep;
      for (int k : hpos) {
        const double ah = -r[k] / (rho[k] * dt);
        if (ah < -0.0 * tmin / dt) released.push_back(k);
        else keep.push_back(k);
      }
      hpos = keep;
    }
    std::vector<int> thin;
    for (int i = 0; i < nn; ++i)
      if (h[i] < tmin) thin.push_back(i);
    std::vector<int> newact = set_diff(set_diff(set_diff(thin, hfixed), hpos), released);
    const int maxnew = p->MaxNumberOfNewlyIntroducedActiveThicknessConstraints;
    if ((int)newact.size() > maxnew) {
      std::vector<int> order(nn);
      for (int i = 0; i < nn; ++i) order[i] = i;
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return h[a] < h[b]; });
      newact.assign(order.begin(), order.begin() + maxnew);
    }
    hpos.insert(hpos.end(), newact.begin(), newact.end());
    deact = set_diff(last_set, hpos);
    act = set_diff(hpos, last_set);
    cyclical = (!act.empty() || !deact.empty()) && set_xor(act, last_released).empty() &&
               set_xor(deact, last_activated).empty();
    if (cyclical) hpos.insert(hpos.end(), deact.begin(), deact.end());
    if ((!deact.empty() || !act.empty()) && (int)deact.size() < minnew && (int)act.size() < minnew) {
      hpos = last_set; deact.clear(); act.clear();
    }
    const bool modified = !set_xor(hpos, last_set).empty();
    last_released = deact;
    last_activated = act;
    ++it;
    if (!modified || cyclical) break;
    if (it > p->ThicknessConstraintsItMax) { as_conv = false; break; }
  }
  std::memcpy(F->ub, ub.data(), nn * sizeof(double));
  std::memcpy(F->vb, vb.data(), nn * sizeof(double));
  std::memcpy(F->h1, h.data(), nn * sizeof(double));
  if (luvh && nl == (int)lam.size()) std::memcpy(luvh, lam.data(), nl * sizeof(double));
  if (rep) {
    rep->iterations = max_newton;  // uvh.m:89-90: the largest Newton count of the active-set iterations
    rep->krylov_its_total = kits;
    rep->active_set_iterations = it - 1;
    rep->active_set_cyclical = cyclical ? 1 : 0;
    rep->active_set_converged = as_conv ? 1 : 0;
    rep->n_hpos = (int32_t)hpos.size();
    if (rep->hpos_node)
      for (int k = 0; k < (int)hpos.size() && k < rep->hpos_capacity; ++k) rep->hpos_node[k] = hpos[k];
  }
  return solve_rc;
}

extern "C" int ua_uvh_newton(ua_mesh* m, const ua_params* p, ua_fields* F, const ua_bcs* bcs, double* luvh,
                             int32_t nl, ua_newton_report* rep) {
  if (!m || !p || !F) return set_error(UA_ERR_INVALID, "ua_uvh_newton: null argument");
  if (m->dm.nsys != 1) return set_error(UA_ERR_INVALID, "ua_uvh_newton takes a single-mesh handle");
  if (p->ThicknessConstraints) return uvh_active_set(m, p, F, bcs, rep, luvh, nl);
  std::vector<ua_newton_report*> reps(1, rep);
  return uvh_common(m, p, F, bcs, 1, reps, luvh, nl);
}

extern "C" int ua_uvh_newton_batch(ua_mesh* m, const ua_params* p, ua_fields* fields, const ua_bcs* bcs,
                                   ua_newton_report* reports) {
  if (!m || !p || !fields) return set_error(UA_ERR_INVALID, "ua_uvh_newton_batch: null argument");
  std::vector<ua_newton_report*> reps(m->dm.nsys);
  for (int s = 0; s < m->dm.nsys; ++s) reps[s] = reports ? &reports[s] : nullptr;
  return uvh_common(m, p, fields, bcs, m->dm.nsys, reps, nullptr, 0);
}

// ---------------------------------------------------------------------------
// Serving: continuous batching over the systems (slots) of a handle.  A
// request is admitted into a free slot with ua_serve_begin (its fields and
// warm start are uploaded and its Newton solve initialised) while the other
// slots keep iterating; ua_serve_step advances every active slot by one
// Newton iteration and reports the slots that finished.  Each slot's
// arithmetic is independent of the others (per-system reductions and line
// searches), so a result is the same alone and in the mix.
// ---------------------------------------------------------------------------

extern "C" int ua_serve_setup(ua_mesh* m, const ua_params* p, const ua_bcs* bcs) {
  if (!m || !p || !bcs) return set_error(UA_ERR_INVALID, "ua_serve_setup: null argument");
  if (m->ndof != 2) return set_error(UA_ERR_INVALID, "serving runs the uv solve (ndof=2 handle)");
  UA_CUDA_TRY(cudaSetDevice(m->device));
  int rc;
  if ((rc = ensure_work(m, p))) return rc;
  if ((rc = ensure_K(m, p->precision))) return rc;
  if ((rc = build_constraints(m, bcs, m->dm.nsys))) return rc;
  Work* w = m->work;
  delete w->serve;
  w->serve = new ServeState();
  const int nsys = w->nsys;
  w->serve->st.assign(nsys, SysState());
  w->serve->rep.assign(nsys, ua_newton_report());
  w->serve->recs.assign(nsys, std::vector<ua_newton_iter>(2 * (p->NRitmax + 2)));
  w->serve->retried.assign(nsys, 0);
  w->serve->busy.assign(nsys, 0);
  if (w->nc) UA_CUDA_TRY(cudaMemsetAsync(w->lam, 0, w->nc * sizeof(double), m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  return UA_OK;
}

static int serve_reset_lam(ua_mesh* m, int s) {
  Work* w = m->work;
  const int c0 = w->h_sys_con_off[s], nc_s = w->h_sys_con_off[s + 1] - c0;
  if (nc_s) UA_CUDA_TRY(cudaMemsetAsync(w->lam + c0, 0, nc_s * sizeof(double), m->stream));
  return UA_OK;
}

extern "C" int ua_serve_begin(ua_mesh* m, const ua_params* p, int32_t count, const int32_t* sys,
                              const ua_fields* F) {
  if (!m || !p || !sys || !F || count <= 0) return set_error(UA_ERR_INVALID, "ua_serve_begin: bad arguments");
  if (!m->work || !m->work->serve) return set_error(UA_ERR_INVALID, "ua_serve_setup has not been called");
  UA_CUDA_TRY(cudaSetDevice(m->device));
  Work* w = m->work;
  ServeState& S = *w->serve;
  const int nsys = w->nsys;
  std::vector<int> run(nsys, 0);
  std::vector<SysScal> sc(nsys);
  UA_CUDA_TRY(cudaMemcpy(sc.data(), w->scal, nsys * sizeof(SysScal), cudaMemcpyDeviceToHost));
  int rc;
  for (int k = 0; k < count; ++k) {
    const int s = sys[k];
    if (s < 0 || s >= nsys) return set_error(UA_ERR_INVALID, "slot %d out of range", s);
    if (S.busy[s]) return set_error(UA_ERR_INVALID, "slot %d is busy", s);
    if ((rc = upload_fields_sys(m, F[k], s, sc[s]))) return rc;
    if ((rc = upload_velocity_sys(m, F[k], s))) return rc;
    if ((rc = serve_reset_lam(m, s))) return rc;
    run[s] = 1;
  }
  if ((rc = finish_fields(m, p, sc, 0, nsys))) return rc;
  if ((rc = newton_init(m, p, run, S.st))) return rc;
  for (int s = 0; s < nsys; ++s) {
    if (!run[s]) continue;
    S.busy[s] = 1;
    S.retried[s] = 0;
    ua_newton_report& r = S.rep[s];
    std::memset(&r, 0, sizeof(r));
    r.iters = S.recs[s].data();
    r.iters_capacity = (int)S.recs[s].size();
  }
  return UA_OK;
}

extern "C" int ua_serve_step(ua_mesh* m, const ua_params* p, int32_t* finished, int32_t* nactive) {
  if (!m || !p || !m->work || !m->work->serve) return set_error(UA_ERR_INVALID, "ua_serve_step: not set up");
  UA_CUDA_TRY(cudaSetDevice(m->device));
  Work* w = m->work;
  ServeState& S = *w->serve;
  const int nsys = w->nsys;
  std::vector<ua_newton_report*> rep(nsys);
  for (int s = 0; s < nsys; ++s) rep[s] = S.busy[s] ? &S.rep[s] : nullptr;
  bool any = false;
  int rc;
  if ((rc = newton_step(m, p, rep, S.st, S.t_asm, S.t_sol, &any))) return rc;
  // systems that stopped during this step (checked at the start of the next
  // step in the batch driver; here they are retired at once)
  std::vector<int> retry(nsys, 0);
  bool need_retry = false;
  int act = 0;
  for (int s = 0; s < nsys; ++s) {
    if (finished) finished[s] = 0;
    if (!S.busy[s]) continue;
    SysState& T = S.st[s];
    bool stop = !T.active;
    if (T.active) {  // apply the exit tests of the next iteration now (:160-190)
      if (residual_criteria(p, T.rForce, T.rWork, T.iteration, T.gamma)) { T.converged = true; T.active = false; stop = true; }
      else if (T.iteration > p->NRitmax) { T.converged = false; T.active = false; stop = true; }
    }
    if (stop && !T.converged && !S.retried[s]) {  // uv.m:107-112 reset-and-retry
      retry[s] = 1;
      need_retry = true;
      continue;
    }
    if (stop) {
      ua_newton_report& r = S.rep[s];
      r.converged = T.converged ? 1 : 0;
      r.iterations = T.iteration;
      r.backtrack_steps = T.iarm;
      r.r = T.r; r.rForce = T.rForce; r.rWork = T.rWork;
      r.retried = S.retried[s];
      S.busy[s] = 0;
      if (finished) finished[s] = 1;
    } else {
      ++act;
    }
  }
  if (need_retry) {
    for (int s = 0; s < nsys; ++s) {
      if (!retry[s]) continue;
      const int d0 = m->h_dof_off[s], nd = m->h_dof_off[s + 1] - d0;
      UA_CUDA_TRY(cudaMemsetAsync(w->X + d0, 0, nd * sizeof(double), m->stream));
      if ((rc = serve_reset_lam(m, s))) return rc;
      S.retried[s] = 1;
      ++act;
    }
    if ((rc = newton_init(m, p, retry, S.st))) return rc;
  }
  if (nactive) *nactive = act;
  (void)any;
  return UA_OK;
}

// Cancels active slots between steps: they leave the Newton iteration at once and are free for
// new requests.  The other slots' arithmetic does not see them (per-system reductions and line
// searches), so their results stay bit-identical.  A slot that is not busy is ignored.
extern "C" int ua_serve_cancel(ua_mesh* m, int32_t count, const int32_t* sys) {
  if (!m || !m->work || !m->work->serve) return set_error(UA_ERR_INVALID, "ua_serve_cancel: not set up");
  if (count < 0 || (count > 0 && !sys)) return set_error(UA_ERR_INVALID, "ua_serve_cancel: bad arguments");
  ServeState& S = *m->work->serve;
  for (int k = 0; k < count; ++k) {
    const int s = sys[k];
    if (s < 0 || s >= (int)S.busy.size()) return set_error(UA_ERR_INVALID, "slot %d out of range", s);
    if (!S.busy[s]) continue;
    S.busy[s] = 0;
    S.st[s].active = false;
    S.st[s].converged = false;
    S.st[s].in_ls = false;
    S.st[s].kfresh = false;
  }
  return UA_OK;
}

extern "C" int ua_serve_result(ua_mesh* m, int32_t sys, double* ub, double* vb, ua_newton_report* rep) {
  if (!m || !m->work || !m->work->serve) return set_error(UA_ERR_INVALID, "ua_serve_result: not set up");
  if (sys < 0 || sys >= m->work->nsys) return set_error(UA_ERR_INVALID, "slot %d out of range", sys);
  UA_CUDA_TRY(cudaSetDevice(m->device));
  Work* w = m->work;
  const int d0 = m->h_dof_off[sys], nn = m->sys[sys].nn;
  if (ub) UA_CUDA_TRY(cudaMemcpyAsync(ub, w->X + d0, nn * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  if (vb) UA_CUDA_TRY(cudaMemcpyAsync(vb, w->X + d0 + nn, nn * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  if (rep) {
    ua_newton_iter* it = rep->iters;
    int cap = rep->iters_capacity;
    double* up = rep->updates;
    const int64_t stride = rep->update_stride;
    *rep = w->serve->rep[sys];
    rep->iters = it;
    rep->iters_capacity = cap;
    rep->updates = up;  // served solves keep no update records
    rep->update_stride = stride;
    if (it) {
      int n = std::min(cap, w->serve->rep[sys].n_iter_records);
      for (int k = 0; k < n; ++k) it[k] = w->serve->recs[sys][k];
      rep->n_iter_records = n;
    } else {
      rep->n_iter_records = 0;
    }
  }
  return UA_OK;
}

extern "C" int ua_mem_info(int32_t device, int64_t* free_bytes, int64_t* total_bytes) {
  UA_CUDA_TRY(cudaSetDevice(device));
  size_t f = 0, t = 0;
  UA_CUDA_TRY(cudaMemGetInfo(&f, &t));
  if (free_bytes) *free_bytes = (int64_t)f;
  if (total_bytes) *total_bytes = (int64_t)t;
  return UA_OK;
}
