// uv residual/tangent assembly: uvMatrixAssemblySSTREAM.m:6-553 on the device.
//
// One CTA per node patch.  Phase 1: one thread per element of the patch
// gathers its nodal fields, loops over the integration points and writes the
// element tangent (uu and vv blocks symmetric, uv block full) and the four
// residual parts Tx, Fx, Ty, Fy into shared memory (element-fastest layout,
// so the writes are bank-conflict free).  Phase 2: one thread per node-level
// non-zero of the patch's rows sums the element contributions listed for it
// (increasing global element order) and writes the four dof-level values;
// the same for the residual on the diagonal entries.  No atomics: every
// matrix entry is produced by exactly one thread, in a fixed order.
#include "ua_internal.h"
#include "ua_physics.cuh"
#include "ua_kernels.h"

namespace ua {

template <int NOD>
struct ElemIdx {
  static constexpr int NS = NOD * (NOD + 1) / 2;
  static constexpr int NKE = 2 * NS + NOD * NOD;
  // packed upper triangle, row-major
  __host__ __device__ static constexpr int sym(int a, int b) {
    return a <= b ? a * NOD - a * (a - 1) / 2 + (b - a) : b * NOD - b * (b - 1) / 2 + (a - b);
  }
};

// derivVector.m:96-109 at integration point ip
template <int NOD>
__device__ __forceinline__ void uv_deriv(const QuadTable& Q, int ip, const double (&xe)[NOD], const double (&ye)[NOD],
                                         double (&Dx)[NOD], double (&Dy)[NOD], double& detJ) {
  double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
#pragma unroll
  for (int a = 0; a < NOD; ++a) {
    J11 += xe[a] * Q.der[ip][0][a];
    J12 += ye[a] * Q.der[ip][0][a];
    J21 += xe[a] * Q.der[ip][1][a];
    J22 += ye[a] * Q.der[ip][1][a];
  }
  detJ = J11 * J22 - J12 * J21;
#pragma unroll
  for (int a = 0; a < NOD; ++a) {
    Dx[a] = (J22 * Q.der[ip][0][a] - J12 * Q.der[ip][1][a]) / detJ;
    Dy[a] = (-J21 * Q.der[ip][0][a] + J11 * Q.der[ip][1][a]) / detJ;
  }
}

// Contribution of integration point ip to the element tangent and residual
// parts (accumulated into the outputs).
template <int NOD, bool WITHK, typename KT>
__device__ __forceinline__ void uv_ip(const QuadTable& Q, const UvPhys& P, const SysScal& S, int ip,
                                      const double (&Dx)[NOD], const double (&Dy)[NOD], double detJ,
                                      const double (&hn)[NOD], const double (&sn)[NOD], const double (&un)[NOD],
                                      const double (&vn)[NOD], const double (&Cn)[NOD], const double (&mn)[NOD],
                                      const double (&An)[NOD], const double (&nn)[NOD], const double (&Sn)[NOD],
                                      const double (&Bn)[NOD], const double (&rn)[NOD], KT* Kuu, KT* Kvv, KT* Kuv,
                                      double* Tx, double* Fx, double* Ty, double* Fy) {
  using I = ElemIdx<NOD>;
  const double rhow = S.rhow, g = S.g, ca = S.ca, sa = S.sa;
  {
    double N[NOD];
#pragma unroll
    for (int a = 0; a < NOD; ++a) N[a] = Q.fun[ip][a];
    double hint = 0, sint = 0, uint = 0, vint = 0, Cint = 0, mint = 0, Aint = 0, nint = 0, Bint = 0, Sint = 0,
           rhoint = 0;
#pragma unroll
    for (int a = 0; a < NOD; ++a) {
      hint += hn[a] * N[a]; sint += sn[a] * N[a];
      uint += un[a] * N[a]; vint += vn[a] * N[a];
      Cint += Cn[a] * N[a]; mint += mn[a] * N[a];
      Aint += An[a] * N[a]; nint += nn[a] * N[a];
      Bint += Bn[a] * N[a]; Sint += Sn[a] * N[a];
      rhoint += rn[a] * N[a];
    }
    if (Cint < P.Cmin) Cint = P.Cmin;        // :205
    if (Aint < P.AGlenmin) Aint = P.AGlenmin;  // :243
    const double Hint = Sint - Bint;
    const double hfint = rhow * Hint / rhoint;  // :300
    // flotation steps (:300-310): one expm1 per argument
    const StepPulse fl = step_pulse(P.kH, hint - hfint, P.Hh0);
    const double Heint = 0.5 + 0.5 * fl.t;
    const double HEint = P.Hh0 == 0.0 ? 0.5 - 0.5 * fl.t : heaviside_approx(P.kH, hfint - hint, P.Hh0);
    const double deltaint = fl.delta;
    const double Hposint = (0.5 + 0.5 * step_pulse(P.kH, Hint, P.Hh0).t) * Hint;
    const bool cube = S.cube != 0.0;  // n = m = 3 at every node of the system
    const double dint = HEint * rhoint * hint / rhow + Heint * Hposint;  // :310
    double dsdx = 0, dhdx = 0, dsdy = 0, dhdy = 0, exx = 0, eyy = 0, exy = 0;
#pragma unroll
    for (int a = 0; a < NOD; ++a) {  // :332-347
      dsdx += Dx[a] * sn[a]; dhdx += Dx[a] * hn[a];
      dsdy += Dy[a] * sn[a]; dhdy += Dy[a] * hn[a];
      exx += Dx[a] * un[a]; eyy += Dy[a] * vn[a];
      exy += 0.5 * (Dx[a] * vn[a] + Dy[a] * un[a]);
    }
    const Drag d = basal_drag_weertman(P, Heint, deltaint, uint, vint, Cint, mint, cube);
    double eta, E;
    effective_viscosity(P, Aint, nint, exx, eyy, exy, eta, E, cube);
    const double dbdx = dsdx - dhdx, dbdy = dsdy - dhdy;
    const double detJw = detJ * Q.w[ip];
    if (WITHK) {
      const KT cxu = (KT)(d.dxu * detJw), cyv = (KT)(d.dyv * detJw), cxv = (KT)(d.dxv * detJw);
      KT Nk[NOD];
#pragma unroll
      for (int a = 0; a < NOD; ++a) Nk[a] = (KT)N[a];
      if constexpr (sizeof(KT) == 8) {
        const KT he = hint * eta * detJw;
        const KT hE2 = P.Dvisk * 2.0 * hint * E * detJw;
        KT Pu[NOD], Pv[NOD];
#pragma unroll
        for (int a = 0; a < NOD; ++a) {
          Pu[a] = (2 * exx + eyy) * Dx[a] + exy * Dy[a];
          Pv[a] = (2 * eyy + exx) * Dy[a] + exy * Dx[a];
        }
#pragma unroll
        for (int a = 0; a < NOD; ++a) {
#pragma unroll
          for (int b = a; b < NOD; ++b) {
            const int i = I::sym(a, b);
            const KT NN = Nk[a] * Nk[b];
            Kuu[i] += he * (4 * Dx[a] * Dx[b] + Dy[a] * Dy[b]) + cxu * NN + hE2 * Pu[a] * Pu[b];
            Kvv[i] += he * (4 * Dy[a] * Dy[b] + Dx[a] * Dx[b]) + cyv * NN + hE2 * Pv[a] * Pv[b];
          }
#pragma unroll
          for (int b = 0; b < NOD; ++b)
            Kuv[a * NOD + b] += he * (2 * Dx[a] * Dy[b] + Dy[a] * Dx[b]) + cxv * Nk[a] * Nk[b] + hE2 * Pu[a] * Pv[b];
        }
      } else {
        // FP32 tangent: h*eta*detJw and 2*h*E*detJw span far beyond the float
        // range (E grows as e^((1-3n)/n) when the strain rate e -> EpsZero), so
        // their square roots are folded into the per-node vectors in FP64 and
        // only the bounded products are rounded to float.
        const double he = hint * eta * detJw;
        const double hE2 = P.Dvisk * 2.0 * hint * E * detJw;
        const double sh = sqrt(he), sE = sqrt(fabs(hE2));
        const KT sgn = hE2 < 0 ? KT(-1) : KT(1);
        KT dx[NOD], dy[NOD], Pu[NOD], Pv[NOD];
#pragma unroll
        for (int a = 0; a < NOD; ++a) {
          dx[a] = (KT)(sh * Dx[a]); dy[a] = (KT)(sh * Dy[a]);
          Pu[a] = (KT)(sE * ((2 * exx + eyy) * Dx[a] + exy * Dy[a]));
          Pv[a] = (KT)(sE * ((2 * eyy + exx) * Dy[a] + exy * Dx[a]));
        }
#pragma unroll
        for (int a = 0; a < NOD; ++a) {
#pragma unroll
          for (int b = a; b < NOD; ++b) {
            const int i = I::sym(a, b);
            const KT NN = Nk[a] * Nk[b];
            Kuu[i] += (4 * dx[a] * dx[b] + dy[a] * dy[b]) + cxu * NN + sgn * Pu[a] * Pu[b];
            Kvv[i] += (4 * dy[a] * dy[b] + dx[a] * dx[b]) + cyv * NN + sgn * Pv[a] * Pv[b];
          }
#pragma unroll
          for (int b = 0; b < NOD; ++b)
            Kuv[a * NOD + b] += (2 * dx[a] * dy[b] + dy[a] * dx[b]) + cxv * Nk[a] * Nk[b] + sgn * Pu[a] * Pv[b];
        }
      }
    }
    const double rr = rhoint * hint - rhow * dint;
    const double pp = 0.5 * g * ca * (rhoint * hint * hint - rhow * dint * dint);
#pragma unroll
    for (int a = 0; a < NOD; ++a) {  // :431-449
      double t1 = -g * rr * dbdx * N[a] * ca + rhoint * g * hint * sa * N[a];
      double t2 = pp * Dx[a];
      double t3 = hint * eta * (4 * exx + 2 * eyy) * Dx[a];
      double t4 = hint * eta * 2 * exy * Dy[a];
      double t5 = d.taux * N[a];
      Tx[a] += (t3 + t4 + t5) * detJw;
      Fx[a] += (t1 + t2) * detJw;
      t1 = -g * rr * dbdy * N[a] * ca;
      t2 = pp * Dy[a];
      t3 = hint * eta * (4 * eyy + 2 * exx) * Dy[a];
      t4 = hint * eta * 2 * exy * Dx[a];
      t5 = d.tauy * N[a];
      Ty[a] += (t3 + t4 + t5) * detJw;
      Fy[a] += (t1 + t2) * detJw;
    }
  }
}

template <int NOD, bool WITHK, typename KT>
__device__ __forceinline__ void uv_zero(KT* Kuu, KT* Kvv, KT* Kuv, double* Tx, double* Fx, double* Ty, double* Fy) {
  using I = ElemIdx<NOD>;
#pragma unroll
  for (int a = 0; a < NOD; ++a) { Tx[a] = 0; Fx[a] = 0; Ty[a] = 0; Fy[a] = 0; }
  if (WITHK) {
#pragma unroll
    for (int i = 0; i < I::NS; ++i) { Kuu[i] = 0; Kvv[i] = 0; }
#pragma unroll
    for (int i = 0; i < NOD * NOD; ++i) Kuv[i] = 0;
  }
}

// Element computation.  Follows uvMatrixAssemblySSTREAM.m :168-455 for one
// element: interpolation and clamps (:186-254), post-2025 flotation at the
// integration points (:300-310), nodal-derivative sums (:332-347), drag and
// viscosity (:351-353), tangent blocks including the Newton viscosity terms
// (:362-425) and residual terms (:431-449).
//
// The Newton viscosity terms E11..E22 are written as the rank-one product
// 2 h E P_I P_J with P_u = (2exx+eyy) dN/dx + exy dN/dy and
// P_v = (2eyy+exx) dN/dy + exy dN/dx, which is the same expression as
// :398-417 regrouped (E11 = h(4exx+2eyy) Deu dNI/dx + 2h exy Deu dNI/dy with
// Deu = E P_u(J)).  The tangent is produced symmetric, which is what
// (K+K.')/2 at :530-531 yields.
template <int NOD, bool WITHK, typename KT>
__device__ __forceinline__ void uv_element(const QuadTable& Q, const UvPhys& P, const SysScal& S,
                                           const double (&xe)[NOD], const double (&ye)[NOD],
                                           const double (&hn)[NOD], const double (&sn)[NOD],
                                           const double (&un)[NOD], const double (&vn)[NOD],
                                           const double (&Cn)[NOD], const double (&mn)[NOD],
                                           const double (&An)[NOD], const double (&nn)[NOD],
                                           const double (&Sn)[NOD], const double (&Bn)[NOD],
                                           const double (&rn)[NOD], KT* Kuu, KT* Kvv, KT* Kuv,
                                           double* Tx, double* Fx, double* Ty, double* Fy) {
  uv_zero<NOD, WITHK, KT>(Kuu, Kvv, Kuv, Tx, Fx, Ty, Fy);
  double Dx[NOD], Dy[NOD], detJ = 0;
  if (NOD == 3) uv_deriv<NOD>(Q, 0, xe, ye, Dx, Dy, detJ);  // P1: constant over the element
#pragma unroll 1
  for (int ip = 0; ip < Q.nip; ++ip) {
    if (NOD != 3) uv_deriv<NOD>(Q, ip, xe, ye, Dx, Dy, detJ);
    uv_ip<NOD, WITHK, KT>(Q, P, S, ip, Dx, Dy, detJ, hn, sn, un, vn, Cn, mn, An, nn, Sn, Bn, rn, Kuu, Kvv, Kuv, Tx,
                          Fx, Ty, Fy);
  }
}

// P1 runs integration-point-parallel (at most 128 registers: two 256-thread or four
// 128-thread blocks per SM); P2 keeps one element per thread in 128-thread blocks.
template <int NOD, bool WITHK, typename KT>
__global__ void __launch_bounds__(NOD == 3 ? 256 : 128, NOD == 3 ? 2 : 1) uv_patch_kernel(DevMesh M, QuadTable Q, UvPhys P, UvIn in, UvOut out) {
  using I = ElemIdx<NOD>;
  extern __shared__ __align__(16) unsigned char smem[];
  const int p = blockIdx.x;
  const int s = M.patch_sys[p];
  if (in.active && !in.active[s]) return;
  const int E = M.max_patch_elems;
  KT* sK = reinterpret_cast<KT*>(smem);
  size_t koff = WITHK ? (((size_t)I::NKE * E * sizeof(KT) + 15) & ~(size_t)15) : 0;
  double* sR = reinterpret_cast<double*>(smem + koff);
  const int e0 = M.patch_elem_ptr[p], ne = M.patch_elem_ptr[p + 1] - e0;
  const int uoff = M.sys_dof_off[s] - M.sys_node_off[s];
  const int nn_s = M.sys_node_off[s + 1] - M.sys_node_off[s];
  const int voff = uoff + nn_s;
  const double gam = in.gamma ? in.gamma[s] : 0.0;
  const SysScal S = in.scal[s];
  // nodal values of element e (u, v at X + gamma dX)
  auto gather = [&](int e, double (&xe)[NOD], double (&ye)[NOD], double (&hn)[NOD], double (&sn)[NOD],
                    double (&un)[NOD], double (&vn)[NOD], double (&Cn)[NOD], double (&mn)[NOD], double (&An)[NOD],
                    double (&nn)[NOD], double (&Sn)[NOD], double (&Bn)[NOD], double (&rn)[NOD]) {
#pragma unroll
    for (int a = 0; a < NOD; ++a) {
      const int gnode = __ldg(M.conn + (size_t)a * M.ne + e);
      xe[a] = __ldg(M.x + gnode); ye[a] = __ldg(M.y + gnode);
      hn[a] = __ldg(in.h + gnode); sn[a] = __ldg(in.s + gnode);
      double u = __ldg(in.X + uoff + gnode), v = __ldg(in.X + voff + gnode);
      if (in.dX) { u += gam * __ldg(in.dX + uoff + gnode); v += gam * __ldg(in.dX + voff + gnode); }
      un[a] = u; vn[a] = v;
      Cn[a] = __ldg(in.C + gnode); mn[a] = __ldg(in.m + gnode);
      An[a] = __ldg(in.A + gnode); nn[a] = __ldg(in.n + gnode);
      Sn[a] = __ldg(in.S + gnode); Bn[a] = __ldg(in.B + gnode);
      rn[a] = __ldg(in.rho + gnode);
    }
  };
  auto store = [&](int t, const KT* Kuu, const KT* Kvv, const KT* Kuv, const double* Tx, const double* Fx,
                   const double* Ty, const double* Fy) {
    if (WITHK) {
#pragma unroll
      for (int i = 0; i < I::NS; ++i) { sK[i * E + t] = Kuu[i]; sK[(I::NS + i) * E + t] = Kvv[i]; }
#pragma unroll
      for (int i = 0; i < NOD * NOD; ++i) sK[(2 * I::NS + i) * E + t] = Kuv[i];
    }
#pragma unroll
    for (int a = 0; a < NOD; ++a) {
      sR[(0 * NOD + a) * E + t] = Tx[a];
      sR[(1 * NOD + a) * E + t] = Fx[a];
      sR[(2 * NOD + a) * E + t] = Ty[a];
      sR[(3 * NOD + a) * E + t] = Fy[a];
    }
  };
  if constexpr (NOD == 3) {
    // P1: the integration points of an element on the lanes of a group (one each), summed in
    // a fixed order; no loop-carried element state, so far fewer registers per thread than an
    // element-per-thread loop.  The 6-point (degree-4) rule runs in 6-lane groups, five per
    // warp (lanes 30 and 31 idle: ip >= 6), so 30 of 32 lanes compute (the launch checks
    // nip <= 6).
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int ip = lane < 30 ? lane % 6 : 6 + lane - 30;
    const int grp = wid * 5 + min(lane / 6, 4);
    const int ngrp = (int)(blockDim.x >> 5) * 5;
    // fixed-order sum of a 6-lane group at its lane 0: ((v0 + v3) + (v1 + v4)) + (v2 + v5)
    auto sum6 = [](auto v) {
      v += __shfl_down_sync(0xffffffffu, v, 3);
      const auto a = __shfl_down_sync(0xffffffffu, v, 1);
      const auto b = __shfl_down_sync(0xffffffffu, v, 2);
      return (v + a) + b;
    };
    for (int base = 0; base < ne; base += ngrp) {  // same trip count for every thread of the block
      const int t = base + grp;
      KT Kuu[I::NS], Kvv[I::NS], Kuv[NOD * NOD];
      double Tx[NOD], Fx[NOD], Ty[NOD], Fy[NOD];
      uv_zero<NOD, WITHK, KT>(Kuu, Kvv, Kuv, Tx, Fx, Ty, Fy);
      if (t < ne && ip < Q.nip) {
        double xe[NOD], ye[NOD], hn[NOD], sn[NOD], un[NOD], vn[NOD], Cn[NOD], mn[NOD], An[NOD], nn[NOD], Sn[NOD],
            Bn[NOD], rn[NOD];
        gather(__ldg(M.patch_elems + e0 + t), xe, ye, hn, sn, un, vn, Cn, mn, An, nn, Sn, Bn, rn);
        double Dx[NOD], Dy[NOD], detJ;
        uv_deriv<NOD>(Q, 0, xe, ye, Dx, Dy, detJ);
        uv_ip<NOD, WITHK, KT>(Q, P, S, ip, Dx, Dy, detJ, hn, sn, un, vn, Cn, mn, An, nn, Sn, Bn, rn, Kuu, Kvv, Kuv,
                              Tx, Fx, Ty, Fy);
      }
      if (WITHK) {
#pragma unroll
        for (int i = 0; i < I::NS; ++i) { Kuu[i] = sum6(Kuu[i]); Kvv[i] = sum6(Kvv[i]); }
#pragma unroll
        for (int i = 0; i < NOD * NOD; ++i) Kuv[i] = sum6(Kuv[i]);
      }
#pragma unroll
      for (int a = 0; a < NOD; ++a) {
        Tx[a] = sum6(Tx[a]); Fx[a] = sum6(Fx[a]); Ty[a] = sum6(Ty[a]); Fy[a] = sum6(Fy[a]);
      }
      if (t < ne && ip == 0) store(t, Kuu, Kvv, Kuv, Tx, Fx, Ty, Fy);
    }
  } else {
    for (int t = threadIdx.x; t < ne; t += blockDim.x) {
      double xe[NOD], ye[NOD], hn[NOD], sn[NOD], un[NOD], vn[NOD], Cn[NOD], mn[NOD], An[NOD], nn[NOD], Sn[NOD],
          Bn[NOD], rn[NOD];
      gather(__ldg(M.patch_elems + e0 + t), xe, ye, hn, sn, un, vn, Cn, mn, An, nn, Sn, Bn, rn);
      KT Kuu[I::NS], Kvv[I::NS], Kuv[NOD * NOD];
      double Tx[NOD], Fx[NOD], Ty[NOD], Fy[NOD];
      uv_element<NOD, WITHK, KT>(Q, P, S, xe, ye, hn, sn, un, vn, Cn, mn, An, nn, Sn, Bn, rn, Kuu, Kvv, Kuv, Tx, Fx,
                                 Ty, Fy);
      store(t, Kuu, Kvv, Kuv, Tx, Fx, Ty, Fy);
    }
  }
  __syncthreads();
  const int pn0 = M.patch_node_ptr[p];
  const int nr = M.patch_node_ptr[p + 1] - pn0;
  if (WITHK) {
    const int q0 = M.patch_q_ptr[p], q1 = M.patch_q_ptr[p + 1];
    const int nbase = M.nodeptr[M.sys_node_off[s]];
    const int nnzn = M.sys_nnzn[s];
    const int kbase = M.sys_knz_off[s];
    for (int t = q0 + threadIdx.x; t < q1; t += blockDim.x) {
      const uint32_t rk = __ldg(M.pq_rk + t);
      const int r = rk >> 16, k = rk & 0xffff;
      const int g = __ldg(M.patch_nodes + pn0 + r);
      const int np0 = __ldg(M.nodeptr + g);
      const int deg = __ldg(M.nodeptr + g + 1) - np0;
      const int lp = np0 - nbase;
      KT uu = 0, vv = 0, uv = 0, vu = 0;
      const int c1 = __ldg(M.pq_cptr + t + 1);
      for (int c = __ldg(M.pq_cptr + t); c < c1; ++c) {
        const uint16_t code = __ldg(M.contrib + c);
        const int el = code >> 6, a = (code >> 3) & 7, b = code & 7;
        const int sy = I::sym(a, b);
        uu += sK[sy * E + el];
        vv += sK[(I::NS + sy) * E + el];
        uv += sK[(2 * I::NS + a * NOD + b) * E + el];
        vu += sK[(2 * I::NS + b * NOD + a) * E + el];
      }
      const size_t b0 = (size_t)kbase + 2 * (size_t)lp;
      const size_t b1 = (size_t)kbase + 2 * (size_t)nnzn + 2 * (size_t)lp;
      KT* Ko = reinterpret_cast<KT*>(out.K);
      Ko[b0 + k] = uu;
      Ko[b0 + deg + k] = uv;
      Ko[b1 + k] = vu;
      Ko[b1 + deg + k] = vv;
    }
  }
  for (int r = threadIdx.x; r < nr; r += blockDim.x) {
    const int g = __ldg(M.patch_nodes + pn0 + r);
    const int t = __ldg(M.prow_diag + pn0 + r);
    double tx = 0, fx = 0, ty = 0, fy = 0;
    const int c1 = __ldg(M.pq_cptr + t + 1);
    for (int c = __ldg(M.pq_cptr + t); c < c1; ++c) {
      const uint16_t code = __ldg(M.contrib + c);
      const int el = code >> 6, a = (code >> 3) & 7;
      tx += sR[(0 * NOD + a) * E + el];
      fx += sR[(1 * NOD + a) * E + el];
      ty += sR[(2 * NOD + a) * E + el];
      fy += sR[(3 * NOD + a) * E + el];
    }
    out.R[uoff + g] = tx - fx;
    out.R[voff + g] = ty - fy;
    if (out.Tint) { out.Tint[uoff + g] = tx; out.Tint[voff + g] = ty; }
    if (out.Fext) { out.Fext[uoff + g] = fx; out.Fext[voff + g] = fy; }
  }
}

size_t uv_patch_smem(int nod, bool withK, bool fp32, int E) {
  int NS = nod * (nod + 1) / 2, NKE = 2 * NS + nod * nod;
  size_t k = withK ? (((size_t)NKE * E * (fp32 ? 4 : 8) + 15) & ~(size_t)15) : 0;
  return k + (size_t)4 * nod * E * 8;
}

template <int NOD, bool WITHK, typename KT>
static cudaError_t launch_t(const ua_mesh* m, const UvPhys& P, const UvIn& in, const UvOut& out, int threads) {
  if (NOD == 3 && quad_table(3).nip > 6) return cudaErrorInvalidConfiguration;  // 6-lane groups of the P1 kernel
  size_t sm = uv_patch_smem(NOD, WITHK, sizeof(KT) == 4, m->dm.max_patch_elems);
  auto kern = uv_patch_kernel<NOD, WITHK, KT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  // all of the unified L1/shared storage as shared memory: several patch blocks per SM
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return e;
  kern<<<m->dm.npatch, NOD == 3 ? threads : 128, sm, m->stream>>>(m->dm, quad_table(NOD), P, in, out);
  return cudaGetLastError();
}

// threads: CTA size of the P1 kernels (128 or 256; 0 = 256 with K, 128 residual-only)
cudaError_t launch_uv_assembly(const ua_mesh* m, const UvPhys& P, const UvIn& in, const UvOut& out, bool withK,
                               bool fp32K, int threads) {
  if (threads != 128 && threads != 256) threads = withK ? 256 : 128;
  if (m->nod == 3) {
    if (!withK) return launch_t<3, false, double>(m, P, in, out, threads);
    return fp32K ? launch_t<3, true, float>(m, P, in, out, threads) : launch_t<3, true, double>(m, P, in, out, threads);
  }
  if (!withK) return launch_t<6, false, double>(m, P, in, out, 128);
  return fp32K ? launch_t<6, true, float>(m, P, in, out, 128) : launch_t<6, true, double>(m, P, in, out, 128);
}

}  // namespace ua
