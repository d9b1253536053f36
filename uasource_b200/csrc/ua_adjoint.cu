// Kernels of the adjoint gradient of the velocity misfit with respect to C
// (Misfit.m "-uv-" adjoint branch, dIdCq.m, MassMatrix2D1dof.m,
// ApplyAdjointGradientPreMultiplier.m).  The adjoint solve itself is the uv
// constrained PCG of the Newton driver; these kernels form its right-hand
// side, the gradient assembly and the mass-matrix pre-multiplier.
//
// Every nodal sum is produced by one thread in a fixed order (the patch
// contribution lists, or one thread per node row), and the dot products are
// a fixed grid of block partials finished by one block: results do not depend
// on the launch schedule.
#include "ua_internal.h"
#include "ua_kernels.h"
#include "ua_physics.cuh"

namespace ua {

namespace {

// detJ of element e at integration point ip (derivVector.m:96-109)
template <int NOD>
__device__ __forceinline__ double elem_detj(const DevMesh& M, const QuadTable& Q, int e, int ip, int (&gn)[NOD]) {
  double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
#pragma unroll
  for (int a = 0; a < NOD; ++a) {
    const double x = __ldg(M.x + gn[a]), y = __ldg(M.y + gn[a]);
    J11 += x * Q.der[ip][0][a];
    J12 += y * Q.der[ip][0][a];
    J21 += x * Q.der[ip][1][a];
    J22 += y * Q.der[ip][1][a];
  }
  return J11 * J22 - J12 * J21;
}

template <int NOD>
__device__ __forceinline__ void elem_nodes(const DevMesh& M, int e, int (&gn)[NOD]) {
#pragma unroll
  for (int a = 0; a < NOD; ++a) gn[a] = __ldg(M.conn + (size_t)a * M.ne + e);
}

// Consistent mass matrix (MassMatrix2D1dof.m) on the node-level pattern: one thread per
// node-level non-zero of a patch's rows sums int N_a N_b over the elements sharing the pair,
// in increasing element order (the patch contribution list).  The result is symmetric bit for
// bit, which is what (M+M.')/2 leaves.
template <int NOD>
__global__ void k_mass_patch(DevMesh M, QuadTable Q, double* Mval) {
  const int p = blockIdx.x;
  const int pn0 = M.patch_node_ptr[p], e0 = M.patch_elem_ptr[p];
  const int q0 = M.patch_q_ptr[p], q1 = M.patch_q_ptr[p + 1];
  for (int t = q0 + threadIdx.x; t < q1; t += blockDim.x) {
    const uint32_t rk = __ldg(M.pq_rk + t);
    const int r = rk >> 16, k = rk & 0xffff;
    const int g = __ldg(M.patch_nodes + pn0 + r);
    double sum = 0.0;
    const int c1 = __ldg(M.pq_cptr + t + 1);
    for (int c = __ldg(M.pq_cptr + t); c < c1; ++c) {
      const uint16_t code = __ldg(M.contrib + c);
      const int el = code >> 6, a = (code >> 3) & 7, b = code & 7;
      const int e = __ldg(M.patch_elems + e0 + el);
      int gn[NOD];
      elem_nodes<NOD>(M, e, gn);
      double me = 0.0;
      for (int ip = 0; ip < Q.nip; ++ip) {
        const double detJw = elem_detj<NOD>(M, Q, e, ip, gn) * Q.w[ip];
        me += Q.fun[ip][b] * Q.fun[ip][a] * detJw;
      }
      sum += me;
    }
    Mval[__ldg(M.nodeptr + g) + k] = sum;
  }
}

// dIdCq.m:40-150 for the elements of one patch (one thread per element), then the nodal sums
// of the patch's nodes over their elements (the diagonal contribution list), fixed order.
template <int NOD>
__global__ void __launch_bounds__(128) k_dIdC_patch(DevMesh M, QuadTable Q, UvPhys P, AdjIn in, double* out) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* sT = reinterpret_cast<double*>(smem);  // [NOD][E]
  const int p = blockIdx.x;
  const int E = M.max_patch_elems;
  const int e0 = M.patch_elem_ptr[p], ne = M.patch_elem_ptr[p + 1] - e0;
  const double rhow = in.rhow, g = in.g;
  for (int t = threadIdx.x; t < ne; t += blockDim.x) {
    const int e = __ldg(M.patch_elems + e0 + t);
    int gn[NOD];
    elem_nodes<NOD>(M, e, gn);
    double T[NOD];
#pragma unroll
    for (int a = 0; a < NOD; ++a) T[a] = 0.0;
    for (int ip = 0; ip < Q.nip; ++ip) {
      const double* N = Q.fun[ip];
      auto itp = [&](const double* f) {
        if (!f) return 0.0;
        double v = 0.0;
#pragma unroll
        for (int a = 0; a < NOD; ++a) v += __ldg(f + gn[a]) * N[a];
        return v;
      };
      double hfint = 0.0;  // the nodal flotation thickness rhow (S - B)/rho, interpolated (:33, :97)
#pragma unroll
      for (int a = 0; a < NOD; ++a)
        hfint += rhow * (__ldg(in.S + gn[a]) - __ldg(in.B + gn[a])) / __ldg(in.rho + gn[a]) * N[a];
      const double hint = itp(in.h), uint = itp(in.u), vint = itp(in.v);
      double Cint = itp(in.C);
      if (Cint < P.Cmin) Cint = P.Cmin;
      const double mint = itp(in.m), qint = itp(in.q), mukint = itp(in.muk), V0int = itp(in.V0);
      const double Hint = itp(in.S) - itp(in.B), rhoint = itp(in.rho);
      const double uA = itp(in.uA), vA = itp(in.vA);
      const double He = heaviside_approx(P.kH, hint - hfint, P.Hh0);
      const double Ct = dFuvdC(P, He, hint, Hint, rhoint, rhow, g, uint, vint, Cint, mint, qint, mukint, V0int);
      const double detJw = elem_detj<NOD>(M, Q, e, ip, gn) * Q.w[ip];
#pragma unroll
      for (int a = 0; a < NOD; ++a) T[a] += Ct * (uint * uA + vint * vA) * N[a] * detJw;
    }
#pragma unroll
    for (int a = 0; a < NOD; ++a) sT[a * E + t] = T[a];
  }
  __syncthreads();
  const int pn0 = M.patch_node_ptr[p];
  const int nr = M.patch_node_ptr[p + 1] - pn0;
  for (int r = threadIdx.x; r < nr; r += blockDim.x) {
    const int gnode = __ldg(M.patch_nodes + pn0 + r);
    const int t = __ldg(M.prow_diag + pn0 + r);
    double s = 0.0;
    const int c1 = __ldg(M.pq_cptr + t + 1);
    for (int c = __ldg(M.pq_cptr + t); c < c1; ++c) {
      const uint16_t code = __ldg(M.contrib + c);
      s += sT[((code >> 3) & 7) * E + (code >> 6)];
    }
    out[gnode] = s;
  }
}

__global__ void k_node_spmv(int nn, const int* nodeptr, const int* nodecol, const double* A, const double* x,
                            double* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  double s = 0.0;
  for (int k = nodeptr[i]; k < nodeptr[i + 1]; ++k) s += A[k] * x[nodecol[k]];
  y[i] = s;
}

__global__ void k_node_diag(int nn, const int* nodeptr, const int* nodecol, const double* A, double* d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  double v = 0.0;
  for (int k = nodeptr[i]; k < nodeptr[i + 1]; ++k)
    if (nodecol[k] == i) v = A[k];
  d[i] = v;
}

// (u - us)/uErr and (v - vs)/vErr (Misfit.m:56, :63)
__global__ void k_misfit_res(int nn, const double* u, const double* v, const double* us, const double* vs,
                             const double* ue, const double* ve, double* ru, double* rv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  ru[i] = (u[i] - us[i]) / ue[i];
  rv[i] = (v[i] - vs[i]) / ve[i];
}

// dI/d(u,v) = [(M ru)./uErr; (M rv)./vErr]/Area (Misfit.m:118-119) into the dof vector
__global__ void k_misfit_grad(int nn, const double* Mru, const double* Mrv, const double* ue, const double* ve,
                              double area, double* f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  f[i] = Mru[i] / ue[i] / area;
  f[nn + i] = Mrv[i] / ve[i] / area;
}

// log(10) C .* dIdC (dIdCq.m:153-156)
__global__ void k_logc_scale(int nn, const double* C, double* g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn) g[i] = 2.302585092994045684 * C[i] * g[i];
}

constexpr int kDotBlocks = kAdjDotBlocks;

// block partials of sum a.b (grid-stride, fixed grid of kDotBlocks blocks x 256 threads)
__global__ void k_dot_part(int n, const double* a, const double* b, double* part) {
  __shared__ double s[256];
  double v = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v += a[i] * b[i];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) s[threadIdx.x] += s[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

// the partials summed by one block in a fixed order; out[slot] = sum
__global__ void k_dot_final(const double* part, double* out, int slot) {
  __shared__ double s[kDotBlocks];
  s[threadIdx.x] = part[threadIdx.x];
  __syncthreads();
  for (int st = kDotBlocks / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) s[threadIdx.x] += s[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[slot] = s[0];
}

// CG scalars in sc[]: 0 rz, 1 pq, 2 rz_new, 3 alpha, 4 beta, 5 rr
__global__ void k_cg_alpha(double* sc) { sc[3] = sc[1] != 0.0 ? sc[0] / sc[1] : 0.0; }
__global__ void k_cg_beta(double* sc) {
  sc[4] = sc[0] != 0.0 ? sc[2] / sc[0] : 0.0;
  sc[0] = sc[2];
}

__global__ void k_cg_xr(int n, const double* sc, const double* p, const double* q, const double* dinv, double* x,
                        double* r, double* z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = sc[3];
  x[i] += a * p[i];
  r[i] -= a * q[i];
  z[i] = r[i] * dinv[i];
}

__global__ void k_cg_p(int n, const double* sc, const double* z, double* p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = z[i] + sc[4] * p[i];
}

__global__ void k_cg_init(int n, const double* b, const double* d, double* x, double* r, double* z, double* p,
                          double* dinv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = 0.0;
  r[i] = b[i];
  dinv[i] = d[i] != 0.0 ? 1.0 / d[i] : 0.0;
  z[i] = r[i] * dinv[i];
  p[i] = z[i];
}

__global__ void k_scale(int n, double s, double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] *= s;
}

}  // namespace

static int nblk(int n) { return (n + 255) / 256; }

cudaError_t adj_mass_matrix(const ua_mesh* m, double* Mval) {
  if (m->nod == 3) k_mass_patch<3><<<m->dm.npatch, 128, 0, m->stream>>>(m->dm, quad_table(3), Mval);
  else k_mass_patch<6><<<m->dm.npatch, 128, 0, m->stream>>>(m->dm, quad_table(6), Mval);
  return cudaGetLastError();
}

cudaError_t adj_dIdC(const ua_mesh* m, const UvPhys& P, const AdjIn& in, double* out) {
  const size_t sm = (size_t)m->nod * m->dm.max_patch_elems * sizeof(double);
  if (m->nod == 3) {
    cudaFuncSetAttribute(k_dIdC_patch<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_dIdC_patch<3><<<m->dm.npatch, 128, sm, m->stream>>>(m->dm, quad_table(3), P, in, out);
  } else {
    cudaFuncSetAttribute(k_dIdC_patch<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_dIdC_patch<6><<<m->dm.npatch, 128, sm, m->stream>>>(m->dm, quad_table(6), P, in, out);
  }
  return cudaGetLastError();
}

cudaError_t adj_node_spmv(const ua_mesh* m, const int* nodeptr, const int* nodecol, const double* A,
                          const double* x, double* y) {
  k_node_spmv<<<nblk(m->nn_total), 256, 0, m->stream>>>(m->nn_total, nodeptr, nodecol, A, x, y);
  return cudaGetLastError();
}

cudaError_t adj_misfit(const ua_mesh* m, const double* u, const double* v, const double* us, const double* vs,
                       const double* ue, const double* ve, double* ru, double* rv) {
  k_misfit_res<<<nblk(m->nn_total), 256, 0, m->stream>>>(m->nn_total, u, v, us, vs, ue, ve, ru, rv);
  return cudaGetLastError();
}

cudaError_t adj_misfit_grad(const ua_mesh* m, const double* Mru, const double* Mrv, const double* ue,
                            const double* ve, double area, double* f) {
  k_misfit_grad<<<nblk(m->nn_total), 256, 0, m->stream>>>(m->nn_total, Mru, Mrv, ue, ve, area, f);
  return cudaGetLastError();
}

cudaError_t adj_logc(const ua_mesh* m, const double* C, double* g) {
  k_logc_scale<<<nblk(m->nn_total), 256, 0, m->stream>>>(m->nn_total, C, g);
  return cudaGetLastError();
}

// out[slot] = a.b over n entries, deterministic; part holds kDotBlocks doubles
cudaError_t adj_dot(cudaStream_t st, int n, const double* a, const double* b, double* part, double* out, int slot) {
  k_dot_part<<<kDotBlocks, 256, 0, st>>>(n, a, b, part);
  k_dot_final<<<1, kDotBlocks, 0, st>>>(part, out, slot);
  return cudaGetLastError();
}

// x = A^-1 b for the symmetric positive definite node matrix A (Jacobi-preconditioned CG, fixed-order
// reductions), to ||r|| <= rtol ||b||; work: 6 node vectors + kDotBlocks + 8 doubles.  Returns the
// iteration count, or -1 if the cap was reached.
int adj_cg(const ua_mesh* m, const int* nodeptr, const int* nodecol, const double* A, const double* b, double* x,
           double rtol, int maxit, double* work, double* h_sc) {
  const int n = m->nn_total;
  cudaStream_t st = m->stream;
  double *r = work, *z = work + n, *p = work + 2 * (size_t)n, *q = work + 3 * (size_t)n, *d = work + 4 * (size_t)n,
         *dinv = work + 5 * (size_t)n, *part = work + 6 * (size_t)n, *sc = part + kDotBlocks;
  k_node_diag<<<nblk(n), 256, 0, st>>>(n, nodeptr, nodecol, A, d);
  k_cg_init<<<nblk(n), 256, 0, st>>>(n, b, d, x, r, z, p, dinv);
  adj_dot(st, n, b, b, part, sc, 6);
  adj_dot(st, n, r, z, part, sc, 0);
  if (cudaMemcpyAsync(h_sc, sc + 6, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return -2;
  const double bb = h_sc[0];
  if (bb == 0.0) return 0;
  for (int it = 1; it <= maxit; ++it) {
    k_node_spmv<<<nblk(n), 256, 0, st>>>(n, nodeptr, nodecol, A, p, q);
    adj_dot(st, n, p, q, part, sc, 1);
    k_cg_alpha<<<1, 1, 0, st>>>(sc);
    k_cg_xr<<<nblk(n), 256, 0, st>>>(n, sc, p, q, dinv, x, r, z);
    adj_dot(st, n, r, z, part, sc, 2);
    k_cg_beta<<<1, 1, 0, st>>>(sc);
    k_cg_p<<<nblk(n), 256, 0, st>>>(n, sc, z, p);
    if (it % 8 == 0 || it == maxit) {
      adj_dot(st, n, r, r, part, sc, 5);
      if (cudaMemcpyAsync(h_sc, sc + 5, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        return -2;
      if (h_sc[0] <= rtol * rtol * bb) return it;
    }
  }
  return -1;
}

cudaError_t adj_scale(const ua_mesh* m, double s, double* x) {
  k_scale<<<nblk(m->nn_total), 256, 0, m->stream>>>(m->nn_total, s, x);
  return cudaGetLastError();
}

}  // namespace ua
