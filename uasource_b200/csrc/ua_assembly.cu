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
template <int NOD, bool WITHK, typename KT, bool GEN>
__device__ __forceinline__ void uv_ip(const QuadTable& Q, const UvPhys& P, const SysScal& S, int ip,
                                      const int (&gn)[NOD], const DragFields& DF,
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
    // GEN: any sliding law and the melange terms; else Weertman (the general code stays out of
    // the Weertman build, whose registers it would crowd)
    const Drag d = !GEN ? basal_drag_weertman(P, Heint, deltaint, uint, vint, Cint, mint, cube)
                        : basal_drag_general(P, Heint, deltaint, hint, Hint, rhoint, rhow, g, uint, vint, Cint, mint,
                                             drag_interp<NOD>(DF, gn, N));
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
template <int NOD, bool WITHK, typename KT, bool GEN>
__device__ __forceinline__ void uv_element(const QuadTable& Q, const UvPhys& P, const SysScal& S,
                                           const int (&gn)[NOD], const DragFields& DF,
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
    uv_ip<NOD, WITHK, KT, GEN>(Q, P, S, ip, gn, DF, Dx, Dy, detJ, hn, sn, un, vn, Cn, mn, An, nn, Sn, Bn, rn, Kuu, Kvv,
                          Kuv, Tx, Fx, Ty, Fy);
  }
}

// Phase 2 of the patch kernels: one thread per node-level non-zero of the
// patch's rows sums the element contributions listed for it (increasing global
// element order) and writes the four dof-level values; the same for the
// residual on the diagonal entries.  No atomics: every matrix entry is produced
// by exactly one thread, in a fixed order, whatever the patch partition.
template <int NOD, bool WITHK, typename KT>
__device__ __forceinline__ void patch_scatter(const DevMesh& M, const UvOut& out, int p, int s, int uoff, int voff,
                                              const KT* sK, const double* sR, int E) {
  using I = ElemIdx<NOD>;
  const int pn0 = M.patch_node_ptr[p];
  const int nr = M.patch_node_ptr[p + 1] - pn0;
  const int nep = M.patch_elem_ptr[p + 1] - M.patch_elem_ptr[p];  // elements of this patch
  (void)nep;
  if (WITHK && out.K) {
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
        int el = code >> 6;
        const int a = (code >> 3) & 7, b = code & 7;
        bool ok = true;
        UA_CHECK_INDEX(M.dbg, el, 0, nep, BS_CONTRIB_ELEM, ok);
        if (!ok) continue;
        const int sy = I::sym(a, b);
        uu += sK[sy * E + el];
        vv += sK[(I::NS + sy) * E + el];
        uv += sK[(2 * I::NS + a * NOD + b) * E + el];
        vu += sK[(2 * I::NS + b * NOD + a) * E + el];
      }
      size_t b0 = (size_t)kbase + 2 * (size_t)lp;
      size_t b1 = (size_t)kbase + 2 * (size_t)nnzn + 2 * (size_t)lp;
      bool okk = true;
      UA_CHECK_INDEX(M.dbg, b0, (size_t)kbase, (size_t)M.sys_knz_off[s + 1] - deg - k, BS_K_INDEX, okk);
      UA_CHECK_INDEX(M.dbg, b1, (size_t)kbase, (size_t)M.sys_knz_off[s + 1] - deg - k, BS_K_INDEX, okk);
      if (!okk) continue;
      KT* Ko = reinterpret_cast<KT*>(out.K);
      Ko[b0 + k] = uu;
      Ko[b0 + deg + k] = uv;
      Ko[b1 + k] = vu;
      Ko[b1 + deg + k] = vv;
    }
  }
  for (int r = threadIdx.x; r < nr; r += blockDim.x) {
    int g = __ldg(M.patch_nodes + pn0 + r);
    bool okr = true;
    UA_CHECK_INDEX(M.dbg, g, M.sys_node_off[s], M.sys_node_off[s + 1], BS_R_INDEX, okr);
    if (!okr) continue;
    const int t = __ldg(M.prow_diag + pn0 + r);
    double tx = 0, fx = 0, ty = 0, fy = 0;
    const int c1 = __ldg(M.pq_cptr + t + 1);
    for (int c = __ldg(M.pq_cptr + t); c < c1; ++c) {
      const uint16_t code = __ldg(M.contrib + c);
      int el = code >> 6;
      const int a = (code >> 3) & 7;
      bool ok = true;
      UA_CHECK_INDEX(M.dbg, el, 0, nep, BS_CONTRIB_ELEM, ok);
      if (!ok) continue;
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

// ---------------------------------------------------------------------------
// P1 tangent and residual, re-derived for linear elements.
//
// On a 3-node triangle the basis gradients Dx, Dy, the strain rates exx, eyy,
// exy and the slopes dbdx, dbdy are constant over the element
// (uvMatrixAssemblySSTREAM.m:322-347 evaluate the same values at every
// integration point).  The integration-point loop (:362-449) therefore
// reduces to a handful of scalars per point, and
//   Kuu_ab = S1 (4 Dx_a Dx_b + Dy_a Dy_b) + S2 Pu_a Pu_b + sum_ip cxu N_a N_b
//   Kvv_ab = S1 (4 Dy_a Dy_b + Dx_a Dx_b) + S2 Pv_a Pv_b + sum_ip cyv N_a N_b
//   Kuv_ab = S1 (2 Dx_a Dy_b + Dy_a Dx_b) + S2 Pu_a Pv_b + sum_ip cxv N_a N_b
//   Tx_a = S1 ((4exx+2eyy) Dx_a + 2exy Dy_a) + sum_ip tx N_a,  Fx_a = P Dx_a + sum_ip fx N_a
//   Ty_a = S1 ((4eyy+2exx) Dy_a + 2exy Dx_a) + sum_ip ty N_a,  Fy_a = P Dy_a + sum_ip fy N_a
// with S1 = sum_ip h eta detJw, S2 = sum_ip 2 Dvisk h E detJw, P = sum_ip pp detJw,
// Pu = (2exx+eyy) Dx + exy Dy, Pv = (2eyy+exx) Dy + exy Dx, and per point
// tx = taux detJw, ty = tauy detJw, fx = (-g rr dbdx ca + rho g h sa) detJw,
// fy = -g rr dbdy ca detJw, pp = g ca (rho h^2 - rhow d^2)/2, rr = rho h - rhow d,
// and the drag derivatives cxu, cyv, cxv times detJw (BasalDrag.m:414-429).
// The terms are the reference's, regrouped; the tangent is symmetric as
// (K+K.')/2 makes it (:530-531).
//
// Mapping: six lanes per element, one integration point each (five elements per
// warp, lanes 30-31 idle).  Each lane evaluates its point's physics and writes
// its scalars to a per-warp scratch in shared memory; S1, S2 and P are summed
// over the six lanes in a fixed order.  The six lanes of the element then form
// the 21 tangent entries and 12 residual parts in six uniform steps, reading
// the point scalars (same-address broadcasts) instead of reducing 33 values
// across lanes.  The element tangents and residual parts go to shared memory
// for the segmented sum of phase 2.
// ---------------------------------------------------------------------------
namespace p1 {

constexpr int kThreads = 256;  // the largest CTA (launch bounds); 128 also runs (asm_threads)
// scratch slots per lane: residual scalars first, then the drag derivatives
enum { TX = 0, TY = 1, FX = 2, FY = 3, CXU = 4, CYV = 5, CXV = 6, NSC = 7 };
// staged fields of a patch's element nodes
enum { ND_X = 0, ND_Y, ND_U, ND_V, ND_H, ND_S, ND_C, ND_A, ND_SS, ND_B, ND_RHO, ND_M, ND_N, ND_COUNT };

__device__ __forceinline__ double sel3(double a0, double a1, double a2, int i) {
  return i == 0 ? a0 : (i == 1 ? a1 : a2);
}

// tanh z of z = k (x - x0), the argument of HeavisideApprox.m:86, from one expm1
// (tanh z = sign(z) (1 - e^-2|z|) / (1 + e^-2|z|)); for |z| >= 20, tanh z rounds to
// +-1 exactly in FP64, so the saturated value is returned without the transcendental.
__device__ __forceinline__ double tanh_step(double k, double x, double x0) {
  const double z = k * (x - x0);
  if (fabs(z) >= 20.0) return z > 0 ? 1.0 : -1.0;
  const double em = expm1(-2.0 * fabs(z));
  return copysign(-em / (2.0 + em), z);
}

}  // namespace p1

// GEN: any sliding law and the melange terms (basal_drag_general); else Weertman, with the
// reciprocal-cube-root powers when n = m = 3 at every node of the system.
// RV: register budget (launch bounds): 0 = 128 registers (two 256-thread CTAs per SM), 1 = 96
// (five 128-thread CTAs), 2 = 80 (three 256-thread CTAs); fewer registers, more warps to hide
// the gathers' latency, against spills to local memory.
namespace p1 {
constexpr int max_threads(int rv) { return rv == 1 ? 128 : 256; }
constexpr int min_blocks(int rv) { return rv == 0 ? 2 : (rv == 1 ? 5 : 3); }
}  // namespace p1
template <bool WITHK, typename KT, bool GEN, int RV>
__global__ void __launch_bounds__(p1::max_threads(RV), p1::min_blocks(RV))
    uv_p1_kernel(DevMesh M, QuadTable Q, UvPhys P, UvIn in, UvOut out) {
  using I = ElemIdx<3>;
  using namespace p1;
  extern __shared__ __align__(16) unsigned char smem[];
  const int p = blockIdx.x;
  const int s = M.patch_sys[p];
  if (in.active && !in.active[s]) return;
  const int E = M.max_patch_elems;
  // residual-only calls run the same instantiation as the tangent calls of their precision with
  // out.K null, so both compute R with the same instructions (bit-identical R)
  const bool kw = WITHK && out.K != nullptr;
  KT* sK = reinterpret_cast<KT*>(smem);
  const size_t koff = WITHK ? (((size_t)I::NKE * E * sizeof(KT) + 15) & ~(size_t)15) : 0;
  double* sR = reinterpret_cast<double*>(smem + koff);  // 12 E
  double* sN = sR + 12 * E;                              // N_a(ip) at [ip*3 + a], weights at [18 + ip]
  double* scr = sN + 24;                                 // NSC x 32 per warp
  double* nd = scr + (blockDim.x >> 5) * (NSC * 32);     // staged node fields [ND_COUNT][MH]
  const int MH = M.max_patch_hnodes;
  const int e0 = M.patch_elem_ptr[p], ne = M.patch_elem_ptr[p + 1] - e0;
  const int uoff = M.sys_dof_off[s] - M.sys_node_off[s];
  const int nn_s = M.sys_node_off[s + 1] - M.sys_node_off[s];
  const int voff = uoff + nn_s;
  const double gam = in.gamma ? in.gamma[s] : 0.0;
  const SysScal S = in.scal[s];
  const bool cube = S.cube != 0.0;
  if (threadIdx.x < 18) sN[threadIdx.x] = Q.fun[threadIdx.x / 3][threadIdx.x % 3];
  else if (threadIdx.x < 24) sN[threadIdx.x] = Q.w[threadIdx.x - 18];
  // stage the fields of the patch's element nodes: every load of the element loop then comes
  // from shared memory, and the gathers of the whole patch are in flight together
  const int hb0 = M.patch_hnode_ptr[p], nh = M.patch_hnode_ptr[p + 1] - hb0;
  for (int t = threadIdx.x; t < nh; t += blockDim.x) {
    int gn = __ldg(M.patch_hnodes + hb0 + t);
    bool okn = true;
    UA_CHECK_INDEX(M.dbg, gn, M.sys_node_off[s], M.sys_node_off[s + 1], BS_ELEM_NODE, okn);
    (void)okn;
    double u = __ldg(in.X + uoff + gn), v = __ldg(in.X + voff + gn);  // at X + gamma dX (CalcCostFunctionNR.m:14-16)
    if (in.dX) { u += gam * __ldg(in.dX + uoff + gn); v += gam * __ldg(in.dX + voff + gn); }
    nd[ND_X * MH + t] = __ldg(M.x + gn); nd[ND_Y * MH + t] = __ldg(M.y + gn);
    nd[ND_U * MH + t] = u; nd[ND_V * MH + t] = v;
    nd[ND_H * MH + t] = __ldg(in.h + gn); nd[ND_S * MH + t] = __ldg(in.s + gn);
    nd[ND_C * MH + t] = __ldg(in.C + gn); nd[ND_A * MH + t] = __ldg(in.A + gn);
    nd[ND_SS * MH + t] = __ldg(in.S + gn); nd[ND_B * MH + t] = __ldg(in.B + gn);
    nd[ND_RHO * MH + t] = __ldg(in.rho + gn); nd[ND_M * MH + t] = __ldg(in.m + gn);
    nd[ND_N * MH + t] = cube ? 3.0 : __ldg(in.n + gn);
  }
  __syncthreads();

  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int j = lane < 30 ? lane % 6 : lane - 30;  // integration point of this lane, and its output slot
  const int grp = lane < 30 ? lane / 6 : 4;
  const int g0 = grp * 6;                          // first lane of the element's group
  double* ws = scr + wid * (NSC * 32);
  const double N0 = sN[j * 3 + 0], N1 = sN[j * 3 + 1], N2 = sN[j * 3 + 2], wj = sN[18 + j];
  const double rhow = S.rhow, g = S.g, ca = S.ca, sa = S.sa;
  const int ngrp = (blockDim.x >> 5) * 5;  // five elements per warp

  for (int base = 0; base < ne; base += ngrp) {  // same trip count for every thread of the block
    const int t = base + wid * 5 + grp;
    bool inb = true;
    // the element's nodes as indices into the staged fields
    const size_t eln = (size_t)(e0 + min(t, ne - 1)) * 3;
    int n0 = __ldg(M.patch_elnodes + eln), n1 = __ldg(M.patch_elnodes + eln + 1), n2 = __ldg(M.patch_elnodes + eln + 2);
    UA_CHECK_INDEX(M.dbg, n0, 0, nh, BS_ELEM_NODE, inb);
    UA_CHECK_INDEX(M.dbg, n1, 0, nh, BS_ELEM_NODE, inb);
    UA_CHECK_INDEX(M.dbg, n2, 0, nh, BS_ELEM_NODE, inb);
    const bool valid = lane < 30 && t < ne && inb;
    auto nf = [&](int f, int l) { return nd[f * MH + l]; };
    // element geometry (derivVector.m:96-109 with the constant P1 derivatives of the
    // basis [xi, 1-xi-eta, eta]); one reciprocal of detJ
    const double x0 = nf(ND_X, n0), x1 = nf(ND_X, n1), x2 = nf(ND_X, n2);
    const double y0 = nf(ND_Y, n0), y1 = nf(ND_Y, n1), y2 = nf(ND_Y, n2);
    const double J11 = x0 - x1, J12 = y0 - y1, J21 = x2 - x1, J22 = y2 - y1;
    const double detJ = J11 * J22 - J12 * J21;
    const double rd = 1.0 / detJ;
    const double Dx0 = J22 * rd, Dx1 = (J12 - J22) * rd, Dx2 = -J12 * rd;
    const double Dy0 = -J21 * rd, Dy1 = (J21 - J11) * rd, Dy2 = J11 * rd;
    // nodal values (velocities staged at X + gamma dX)
    const double u0 = nf(ND_U, n0), u1 = nf(ND_U, n1), u2 = nf(ND_U, n2);
    const double v0 = nf(ND_V, n0), v1 = nf(ND_V, n1), v2 = nf(ND_V, n2);
    const double h0 = nf(ND_H, n0), h1 = nf(ND_H, n1), h2 = nf(ND_H, n2);
    const double s0 = nf(ND_S, n0), s1 = nf(ND_S, n1), s2 = nf(ND_S, n2);
    // element constants (:322-347)
    const double dsdx = (Dx0 * s0 + Dx1 * s1) + Dx2 * s2, dhdx = (Dx0 * h0 + Dx1 * h1) + Dx2 * h2;
    const double dsdy = (Dy0 * s0 + Dy1 * s1) + Dy2 * s2, dhdy = (Dy0 * h0 + Dy1 * h1) + Dy2 * h2;
    const double exx = (Dx0 * u0 + Dx1 * u1) + Dx2 * u2;
    const double eyy = (Dy0 * v0 + Dy1 * v1) + Dy2 * v2;
    const double exy = (0.5 * (Dx0 * v0 + Dy0 * u0) + 0.5 * (Dx1 * v1 + Dy1 * u1)) + 0.5 * (Dx2 * v2 + Dy2 * u2);
    const double dbdx = dsdx - dhdx, dbdy = dsdy - dhdy;
    const double e2 = P.EpsZero * P.EpsZero + exx * exx + eyy * eyy + exx * eyy + exy * exy;
    // this lane's integration point: interpolation and clamps (:186-254)
    const double hint = (h0 * N0 + h1 * N1) + h2 * N2;
    const double uint = (u0 * N0 + u1 * N1) + u2 * N2;
    const double vint = (v0 * N0 + v1 * N1) + v2 * N2;
    auto interp = [&](int f) { return (nf(f, n0) * N0 + nf(f, n1) * N1) + nf(f, n2) * N2; };
    double Cint = interp(ND_C), Aint = interp(ND_A);
    if (Cint < P.Cmin) Cint = P.Cmin;        // :205
    if (Aint < P.AGlenmin) Aint = P.AGlenmin;  // :243
    const double Hint = interp(ND_SS) - interp(ND_B);
    const double rhoint = interp(ND_RHO);
    // flotation at the integration point (:300-310)
    const double hfint = rhow * Hint / rhoint;
    const double tf = tanh_step(P.kH, hint - hfint, P.Hh0);
    const double Heint = 0.5 + 0.5 * tf;
    // H(hf - h): the mirror 0.5 - 0.5 tanh for x0 = 0 (tanh is odd)
    const double HEint = P.Hh0 == 0.0 ? 0.5 - 0.5 * tf : 0.5 + 0.5 * tanh_step(P.kH, hfint - hint, P.Hh0);
    const double Hposint = (0.5 + 0.5 * tanh_step(P.kH, Hint, P.Hh0)) * Hint;
    const double dint = HEint * rhoint * hint / rhow + Heint * Hposint;
    // drag (BasalDrag.m:54-77, :410-446): Weertman drag is identically zero on floating ice (He = 0)
    double taux = 0, tauy = 0, dxu = 0, dyv = 0, dxv = 0;
    if (GEN) {
      const int gn[3] = {__ldg(M.patch_hnodes + hb0 + n0), __ldg(M.patch_hnodes + hb0 + n1),
                         __ldg(M.patch_hnodes + hb0 + n2)};
      const double Nw[3] = {N0, N1, N2};
      const Drag d = basal_drag_general(P, Heint, 0.0, hint, Hint, rhoint, rhow, g, uint, vint, Cint,
                                        interp(ND_M), drag_interp<3>(in.drag, gn, Nw));
      taux = d.taux; tauy = d.tauy; dxu = d.dxu; dyv = d.dyv; dxv = d.dxv;
    } else if (Heint > 0) {
      const double sp2 = uint * uint + vint * vint + P.SpeedZero * P.SpeedZero;
      double Cm, ps, cD;
      if (cube) {
        Cm = rcbrt(Cint + P.Czero); ps = rcbrt(sp2); cD = -2.0 / 3.0;
      } else {
        const double mint = interp(ND_M);
        Cm = pow(Cint + P.Czero, -1.0 / mint); ps = pow(sp2, (1.0 - mint) / (2.0 * mint)); cD = 1.0 / mint - 1.0;
      }
      const double beta2 = Cm * ps, Dbeta2 = cD * Cm * ps / sp2;
      taux = Heint * beta2 * uint; tauy = Heint * beta2 * vint;
      dxu = Heint * (beta2 + Dbeta2 * uint * uint);
      dyv = Heint * (beta2 + Dbeta2 * vint * vint);
      dxv = Heint * Dbeta2 * uint * vint;
    }
    // viscosity (EffectiveViscositySSTREAM.m:7-9)
    double Am, pe, cE;
    if (cube) {
      Am = rcbrt(Aint); pe = rcbrt(e2); cE = -1.0 / 6.0;
    } else {
      const double nint = interp(ND_N);
      Am = pow(Aint, -1.0 / nint); pe = pow(sqrt(e2), (1.0 - nint) / nint); cE = (1.0 - nint) / (4.0 * nint);
    }
    const double eta = 0.5 * Am * pe + P.etaZero;
    const double detJw = detJ * wj;
    const double rr = rhoint * hint - rhow * dint;
    double s_he = hint * eta * detJw;
    double s_pp = 0.5 * g * ca * (rhoint * hint * hint - rhow * dint * dint) * detJw;
    double s_hE = 0;
    if (kw) s_hE = P.Dvisk * 2.0 * hint * (cE * Am * pe / e2) * detJw;
    ws[TX * 32 + lane] = taux * detJw;
    ws[TY * 32 + lane] = tauy * detJw;
    ws[FX * 32 + lane] = (-g * rr * dbdx * ca + rhoint * g * hint * sa) * detJw;
    ws[FY * 32 + lane] = (-g * rr * dbdy * ca) * detJw;
    if (kw) {
      ws[CXU * 32 + lane] = dxu * detJw;
      ws[CYV * 32 + lane] = dyv * detJw;
      ws[CXV * 32 + lane] = dxv * detJw;
    }
    // S1, S2, P over the element's six points, fixed order ((0+3)+(1+4))+(2+5), to every lane
    auto sum6 = [&](double v) {
      v += __shfl_down_sync(0xffffffffu, v, 3);
      const double a = __shfl_down_sync(0xffffffffu, v, 1);
      const double b = __shfl_down_sync(0xffffffffu, v, 2);
      return __shfl_sync(0xffffffffu, (v + a) + b, g0);
    };
    const double S1 = sum6(s_he), Pp = sum6(s_pp);
    const double S2 = kw ? sum6(s_hE) : 0.0;
    __syncwarp();
    // sum_ip sc(kind, ip) w(ip) for the element of this lane's group, ip in order
    auto dot = [&](int kind, int a, int b, bool pair) {
      const double* src = ws + kind * 32 + g0;
      double acc = 0.0;
#pragma unroll
      for (int ip = 0; ip < 6; ++ip) {
        const double w = pair ? sN[ip * 3 + a] * sN[ip * 3 + b] : sN[ip * 3 + a];
        acc += src[ip] * w;
      }
      return acc;
    };
    if (valid) {
      if (kw) {
        const double Pu0 = (2 * exx + eyy) * Dx0 + exy * Dy0, Pu1 = (2 * exx + eyy) * Dx1 + exy * Dy1,
                     Pu2 = (2 * exx + eyy) * Dx2 + exy * Dy2;
        const double Pv0 = (2 * eyy + exx) * Dy0 + exy * Dx0, Pv1 = (2 * eyy + exx) * Dy1 + exy * Dx1,
                     Pv2 = (2 * eyy + exx) * Dy2 + exy * Dx2;
        // symmetric blocks: packed upper-triangle pair j (row-major: 00 01 02 11 12 22)
        const int a = j < 3 ? 0 : (j < 5 ? 1 : 2);
        const int b = j < 3 ? j : (j < 5 ? j - 2 : 2);
        const double dxa = sel3(Dx0, Dx1, Dx2, a), dxb = sel3(Dx0, Dx1, Dx2, b);
        const double dya = sel3(Dy0, Dy1, Dy2, a), dyb = sel3(Dy0, Dy1, Dy2, b);
        const double kuu = S1 * (4 * dxa * dxb + dya * dyb) + S2 * (sel3(Pu0, Pu1, Pu2, a) * sel3(Pu0, Pu1, Pu2, b)) +
                           dot(CXU, a, b, true);
        const double kvv = S1 * (4 * dya * dyb + dxa * dxb) + S2 * (sel3(Pv0, Pv1, Pv2, a) * sel3(Pv0, Pv1, Pv2, b)) +
                           dot(CYV, a, b, true);
        sK[j * E + t] = (KT)kuu;
        sK[(I::NS + j) * E + t] = (KT)kvv;
        // uv block, full: entries (j/3, j%3) for j < 6, then (2, j) on lanes 0-2
#pragma unroll
        for (int step = 0; step < 2; ++step) {
          const int q = step * 6 + j;
          if (q < 9) {
            const int ua = q / 3, ub = q % 3;
            const double kuv = S1 * (2 * sel3(Dx0, Dx1, Dx2, ua) * sel3(Dy0, Dy1, Dy2, ub) +
                                     sel3(Dy0, Dy1, Dy2, ua) * sel3(Dx0, Dx1, Dx2, ub)) +
                               S2 * (sel3(Pu0, Pu1, Pu2, ua) * sel3(Pv0, Pv1, Pv2, ub)) + dot(CXV, ua, ub, true);
            sK[(2 * I::NS + q) * E + t] = (KT)kuv;
          }
        }
      }
      // residual parts: lanes 0-2 the x rows of nodes 0-2, lanes 3-5 the y rows
      const bool yrow = j >= 3;
      const int a = yrow ? j - 3 : j;
      const double da = sel3(Dx0, Dx1, Dx2, a), db = sel3(Dy0, Dy1, Dy2, a);
      const double d1 = yrow ? db : da, d2 = yrow ? da : db;      // Dy, Dx for the y rows
      const double e1 = yrow ? eyy : exx, e2_ = yrow ? exx : eyy;
      const double T = S1 * ((4 * e1 + 2 * e2_) * d1 + 2 * exy * d2) + dot(yrow ? TY : TX, a, 0, false);
      const double F = Pp * d1 + dot(yrow ? FY : FX, a, 0, false);
      sR[((yrow ? 2 : 0) * 3 + a) * E + t] = T;
      sR[((yrow ? 3 : 1) * 3 + a) * E + t] = F;
    }
    __syncwarp();  // the scratch is rewritten by the next element group
  }
  __syncthreads();
  patch_scatter<3, WITHK, KT>(M, out, p, s, uoff, voff, sK, sR, E);
}

size_t uv_p1_smem(bool withK, bool fp32, int E, int threads, int MH) {
  size_t k = withK ? (((size_t)ElemIdx<3>::NKE * E * (fp32 ? 4 : 8) + 15) & ~(size_t)15) : 0;
  return k + (size_t)12 * E * 8 + 24 * 8 + (size_t)(threads / 32) * p1::NSC * 32 * 8 +
         (size_t)p1::ND_COUNT * MH * 8;
}

// P2 (6-node elements): one element per thread in 128-thread blocks, the
// integration points in a loop (the derivatives vary over the element).
template <int NOD, bool WITHK, typename KT, bool GEN>
__global__ void __launch_bounds__(128, 1) uv_patch_kernel(DevMesh M, QuadTable Q, UvPhys P, UvIn in, UvOut out) {
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
  auto gather = [&](int e, int (&gn)[NOD], double (&xe)[NOD], double (&ye)[NOD], double (&hn)[NOD],
                    double (&sn)[NOD], double (&un)[NOD], double (&vn)[NOD], double (&Cn)[NOD], double (&mn)[NOD],
                    double (&An)[NOD], double (&nn)[NOD], double (&Sn)[NOD], double (&Bn)[NOD], double (&rn)[NOD]) {
#pragma unroll
    for (int a = 0; a < NOD; ++a) {
      int gnode = __ldg(M.conn + (size_t)a * M.ne + e);
      bool okn = true;
      UA_CHECK_INDEX(M.dbg, gnode, 0, M.nn, BS_ELEM_NODE, okn);
      (void)okn;
      gn[a] = gnode;
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
  for (int t = threadIdx.x; t < ne; t += blockDim.x) {
    int gn[NOD];
    double xe[NOD], ye[NOD], hn[NOD], sn[NOD], un[NOD], vn[NOD], Cn[NOD], mn[NOD], An[NOD], nn[NOD], Sn[NOD],
        Bn[NOD], rn[NOD];
    gather(__ldg(M.patch_elems + e0 + t), gn, xe, ye, hn, sn, un, vn, Cn, mn, An, nn, Sn, Bn, rn);
    KT Kuu[I::NS], Kvv[I::NS], Kuv[NOD * NOD];
    double Tx[NOD], Fx[NOD], Ty[NOD], Fy[NOD];
    uv_element<NOD, WITHK, KT, GEN>(Q, P, S, gn, in.drag, xe, ye, hn, sn, un, vn, Cn, mn, An, nn, Sn, Bn, rn, Kuu, Kvv,
                               Kuv, Tx, Fx, Ty, Fy);
    store(t, Kuu, Kvv, Kuv, Tx, Fx, Ty, Fy);
  }
  __syncthreads();
  patch_scatter<NOD, WITHK, KT>(M, out, p, s, uoff, voff, sK, sR, E);
}

size_t uv_patch_smem(int nod, bool withK, bool fp32, int E) {
  int NS = nod * (nod + 1) / 2, NKE = 2 * NS + nod * nod;
  size_t k = withK ? (((size_t)NKE * E * (fp32 ? 4 : 8) + 15) & ~(size_t)15) : 0;
  return k + (size_t)4 * nod * E * 8;
}

template <bool WITHK, typename KT, bool GEN>
static auto p1_kernel(int rv) {
  return rv == 1 ? uv_p1_kernel<WITHK, KT, GEN, 1> : (rv == 2 ? uv_p1_kernel<WITHK, KT, GEN, 2>
                                                               : uv_p1_kernel<WITHK, KT, GEN, 0>);
}

template <bool WITHK, typename KT>
static cudaError_t launch_p1(const ua_mesh* m, const UvPhys& P, const UvIn& in, const UvOut& out, int threads,
                             int regs) {
  if (quad_table(3).nip != 6) return cudaErrorInvalidConfiguration;  // six lanes, one point each
  if (threads != 128 && threads != 256) return cudaErrorInvalidConfiguration;
  const int rv = regs == 96 ? 1 : (regs == 80 ? 2 : 0);
  if (rv == 1 && threads != 128) return cudaErrorInvalidConfiguration;
  size_t sm = uv_p1_smem(WITHK, sizeof(KT) == 4, m->dm.max_patch_elems, threads, m->dm.max_patch_hnodes);
  const bool gen = P.law != UA_SLIDING_WEERTMAN || P.melange;
  auto kern = gen ? p1_kernel<WITHK, KT, true>(rv) : p1_kernel<WITHK, KT, false>(rv);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return e;
  kern<<<m->dm.npatch, threads, sm, m->stream>>>(m->dm, quad_table(3), P, in, out);
  return cudaGetLastError();
}

template <int NOD, bool WITHK, typename KT>
static cudaError_t launch_t(const ua_mesh* m, const UvPhys& P, const UvIn& in, const UvOut& out, int threads) {
  size_t sm = uv_patch_smem(NOD, WITHK, sizeof(KT) == 4, m->dm.max_patch_elems);
  const bool gen = P.law != UA_SLIDING_WEERTMAN || P.melange;
  auto kern = gen ? uv_patch_kernel<NOD, WITHK, KT, true> : uv_patch_kernel<NOD, WITHK, KT, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  // all of the unified L1/shared storage as shared memory: several patch blocks per SM
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return e;
  kern<<<m->dm.npatch, NOD == 3 ? threads : 128, sm, m->stream>>>(m->dm, quad_table(NOD), P, in, out);
  return cudaGetLastError();
}

// threads: CTA size of the P1 kernel (128 or 256; 0 = 256); regs: its register budget (128, 96, 80)
cudaError_t launch_uv_assembly(const ua_mesh* m, const UvPhys& P, const UvIn& in, const UvOut& out, bool withK,
                               bool fp32K, int threads, int regs) {
  if (m->nod == 3) {  // residual-only: the tangent instantiation of the precision with out.K null
    UvOut o = out;
    if (!withK) o.K = nullptr;
    const int t = threads > 0 ? threads : p1::kThreads;
    return fp32K ? launch_p1<true, float>(m, P, in, o, t, regs) : launch_p1<true, double>(m, P, in, o, t, regs);
  }
  if (!withK) return launch_t<6, false, double>(m, P, in, out, 128);
  return fp32K ? launch_t<6, true, float>(m, P, in, out, 128) : launch_t<6, true, double>(m, P, in, out, 128);
}

}  // namespace ua
