// uvh residual/tangent assembly of the fully implicit transient step:
// uvhMatrixAssembly.m:6-585 -> uvhAssemblyIntPointImplicitSUPG.m:10-531 ->
// uvhNodalLoopSSTREAM.m:1-229 on the device.
//
// One CTA per node patch.  Threads map to (element, local node I): each
// thread evaluates the integration-point quantities of its element (the
// nodal fields are staged in shared memory) and accumulates the three rows
// (x-momentum, y-momentum, mass conservation) of its node I against all nodes
// J in the nine blocks Kxu..Khh, directly in shared memory slots it alone
// owns.  The patch's node-level non-zeros are then summed over their element
// contributions in increasing global element order (deterministic segmented
// sum, no atomics), nine dof-level values each.
#include "ua_internal.h"
#include "ua_physics.cuh"
#include "ua_kernels.h"

namespace ua {

// Nodal quantities staged per element (index into the field block).
enum { F_X = 0, F_Y, F_H1, F_U1, F_V1, F_S, F_B, F_RHO, F_A, F_N, F_C, F_M, F_H0, F_U0, F_V0, F_A0, F_A1, F_DADH,
       F_B1, F_COUNT };

// SUPGtau.m:7-111
__device__ __forceinline__ double supg_tau(const UvhPhys& P, double v, double l, double dt) {
  const double eps = 2.220446049250313e-16;
  const double taut = dt / 2 + eps;
  const double taus = l / (2 * v + P.SpeedZero);
  double tau;
  switch (P.tau_kind) {
    case 1: tau = taut; break;                                  // "taut"
    case 2: {                                                   // "tau1"
      const double ECN = taut / taus;
      tau = (ECN < 1e-6 ? ECN / 3 : 1.0 / tanh(ECN) - 1.0 / ECN) * taus;
      break;
    }
    case 3: tau = (dt / 2) / (1 + taut / taus); break;          // "tau2"
    default: tau = taus;                                        // "taus" (:61-62)
  }
  return P.tau_mult * tau;
}

// GEN: any sliding law and the melange terms (Weertman chosen at run time); else Weertman only
// (the general code stays out of that build)
template <int NOD, bool WITHK, typename KT, bool GEN>
__global__ void __launch_bounds__(NOD == 3 ? 512 : 320) uvh_patch_kernel(DevMesh M, QuadTable Q, UvhPhys P,
                                                                          UvhIn in, UvOut out) {
  constexpr int NB = 9 * NOD * NOD;   // tangent entries per element
  extern __shared__ __align__(16) unsigned char smem[];
  const int p = blockIdx.x;
  const int s = M.patch_sys[p];
  if (in.active && !in.active[s]) return;
  const int E = M.max_patch_elems;
  KT* sK = reinterpret_cast<KT*>(smem);
  size_t off = WITHK ? (((size_t)NB * E * sizeof(KT) + 15) & ~(size_t)15) : 0;
  double* sR = reinterpret_cast<double*>(smem + off);                 // [6*NOD][E]
  double* sF = sR + (size_t)6 * NOD * E;                               // [F_COUNT][E*NOD]
  const int e0 = M.patch_elem_ptr[p], ne = M.patch_elem_ptr[p + 1] - e0;
  const int no = M.sys_node_off[s];
  const int nn_s = M.sys_node_off[s + 1] - no;
  const int uoff = M.sys_dof_off[s] - no, voff = uoff + nn_s, hoff = voff + nn_s;
  const double gam = in.gamma ? in.gamma[s] : 0.0;
  const SysScal S = in.scal[s];
  const double rhow = S.rhow, g = S.g, ca = S.ca, sa = S.sa, dt = S.dt;
  const double theta = P.theta;
  const int EN = E * NOD;
  // stage the nodal fields (one thread per element node)
  for (int t = threadIdx.x; t < ne * NOD; t += blockDim.x) {
    const int el = t / NOD, a = t % NOD;
    bool inb = true;
    int e = __ldg(M.patch_elems + e0 + el);
    UA_CHECK_INDEX(M.dbg, e, 0, M.ne, BS_PATCH_ELEM, inb);
    int gn = __ldg(M.conn + (size_t)a * M.ne + e);
    UA_CHECK_INDEX(M.dbg, gn, 0, M.nn, BS_ELEM_NODE, inb);
    (void)inb;
    double h1 = in.X[hoff + gn], u1 = in.X[uoff + gn], v1 = in.X[voff + gn];
    if (in.dX) { h1 += gam * in.dX[hoff + gn]; u1 += gam * in.dX[uoff + gn]; v1 += gam * in.dX[voff + gn]; }
    const double h0 = __ldg(in.h0 + gn);
    double u0 = __ldg(in.u0 + gn), v0 = __ldg(in.v0 + gn);
    double a0 = __ldg(in.as0 + gn) + __ldg(in.ab0 + gn), a1 = __ldg(in.as1 + gn) + __ldg(in.ab1 + gn);
    if (in.zero_fields) {  // uvhMatrixAssembly.m:9-15
      u1 = v1 = u0 = v0 = 0;
      h1 = h0;
      a0 = 2 * fabs(__ldg(in.ab0 + gn)) + 1;
      a1 = 2 * fabs(__ldg(in.ab1 + gn)) + 1;
    }
    const double Sg = __ldg(in.S + gn), Bg = __ldg(in.B + gn), rg = __ldg(in.rho + gn);
    // Calc_bs_From_hBS.m:71-79 at the current h (uvhMatrixAssembly.m:36)
    const double hf = rhow * (Sg - Bg) / rg;
    const double GF = heaviside_approx(P.kH, h1 - hf, P.Hh0);
    const double b1 = GF * Bg + (1 - GF) * (Sg - rg * h1 / rhow);
    double* f = sF + el * NOD + a;
    f[F_X * EN] = __ldg(M.x + gn); f[F_Y * EN] = __ldg(M.y + gn);
    f[F_H1 * EN] = h1; f[F_U1 * EN] = u1; f[F_V1 * EN] = v1;
    f[F_S * EN] = Sg; f[F_B * EN] = Bg; f[F_RHO * EN] = rg;
    f[F_A * EN] = __ldg(in.A + gn); f[F_N * EN] = __ldg(in.n + gn);
    f[F_C * EN] = __ldg(in.C + gn); f[F_M * EN] = __ldg(in.m + gn);
    f[F_H0 * EN] = h0; f[F_U0 * EN] = u0; f[F_V0 * EN] = v0;
    f[F_A0 * EN] = a0; f[F_A1 * EN] = a1;
    f[F_DADH * EN] = in.dadh ? __ldg(in.dadh + gn) : 0.0;
    f[F_B1 * EN] = b1;
  }
  __syncthreads();
  const int t = threadIdx.x;
  const int el = t / NOD, I = t % NOD;
  if (el < ne) {
    const double* f = sF + el * NOD;
    auto fv = [&](int k, int a) { return f[k * EN + a]; };
    if (WITHK) {
      for (int k = 0; k < 9 * NOD; ++k) sK[(size_t)(I * 9 * NOD + k) * E + el] = 0;
    }
    double Tx = 0, Fx = 0, Ty = 0, Fy = 0, Th = 0, Fh = 0;
    // element area from the corner nodes (TriAreaFE.m / TriArea.m) -> l = sqrt(2*area) (:156)
    const int c0 = 0, c1 = NOD == 3 ? 1 : 2, c2 = NOD == 3 ? 2 : 4;
    const double area = 0.5 * fabs((fv(F_X, c0) - fv(F_X, c2)) * (fv(F_Y, c1) - fv(F_Y, c0)) -
                                   (fv(F_X, c0) - fv(F_X, c1)) * (fv(F_Y, c2) - fv(F_Y, c0)));
    const double lsupg = sqrt(2 * area);
    double Dx[NOD], Dy[NOD], detJ = 0;
    auto deriv = [&](int ip) {  // derivVector.m:96-109
      double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
#pragma unroll
      for (int a = 0; a < NOD; ++a) {
        J11 += fv(F_X, a) * Q.der[ip][0][a];
        J12 += fv(F_Y, a) * Q.der[ip][0][a];
        J21 += fv(F_X, a) * Q.der[ip][1][a];
        J22 += fv(F_Y, a) * Q.der[ip][1][a];
      }
      detJ = J11 * J22 - J12 * J21;
#pragma unroll
      for (int a = 0; a < NOD; ++a) {
        Dx[a] = (J22 * Q.der[ip][0][a] - J12 * Q.der[ip][1][a]) / detJ;
        Dy[a] = (-J21 * Q.der[ip][0][a] + J11 * Q.der[ip][1][a]) / detJ;
      }
    };
    if (NOD == 3) deriv(0);
#pragma unroll 1
    for (int ip = 0; ip < Q.nip; ++ip) {
      if (NOD != 3) deriv(ip);
      double N[NOD];
#pragma unroll
      for (int a = 0; a < NOD; ++a) N[a] = Q.fun[ip][a];
      auto itp = [&](int k) {
        double v = 0;
#pragma unroll
        for (int a = 0; a < NOD; ++a) v += fv(k, a) * N[a];
        return v;
      };
      auto ddx = [&](int k) {
        double v = 0;
#pragma unroll
        for (int a = 0; a < NOD; ++a) v += Dx[a] * fv(k, a);
        return v;
      };
      auto ddy = [&](int k) {
        double v = 0;
#pragma unroll
        for (int a = 0; a < NOD; ++a) v += Dy[a] * fv(k, a);
        return v;
      };
      // uvhAssemblyIntPointImplicitSUPG.m:62-121 (no level set, no thickness penalty/barrier)
      const double hint = itp(F_H1), uint = itp(F_U1), vint = itp(F_V1);
      const double Cint = itp(F_C), mint = itp(F_M), Aint = itp(F_A), nint = itp(F_N);
      const double h0int = itp(F_H0), u0int = itp(F_U0), v0int = itp(F_V0);
      const double a1int = itp(F_A1), a0int = itp(F_A0), dadhint = itp(F_DADH);
      const double Bint = itp(F_B), Sint = itp(F_S), rhoint = itp(F_RHO);
      const double Hint = Sint - Bint;
      const double hfint = rhow * Hint / rhoint;
      // flotation steps and pulses: one expm1 per argument (for Hh0 = 0 the mirrored step is
      // 1 - the step and the pulse is even)
      const StepPulse fl = step_pulse(P.kH, hint - hfint, P.Hh0);
      const double Heint = 0.5 + 0.5 * fl.t;
      const double deltaint = fl.delta;
      double HEint, Deltaint;
      if (P.Hh0 == 0.0) {
        HEint = 0.5 - 0.5 * fl.t;
        Deltaint = fl.delta;
      } else {
        const StepPulse fm = step_pulse(P.kH, hfint - hint, P.Hh0);
        HEint = 0.5 + 0.5 * fm.t;
        Deltaint = fm.delta;
      }
      const double Hposint = (0.5 + 0.5 * step_pulse(P.kH, Hint, P.Hh0).t) * Hint;
      const bool cube = S.cube != 0.0;  // n = m = 3 at every node of the system
      const double dint = HEint * rhoint * hint / rhow + Heint * Hposint;
      const double Dddhint = HEint * rhoint / rhow - Deltaint * hint * rhoint / rhow + deltaint * Hposint;
      // :132-148
      const double dhdx = ddx(F_H1), dhdy = ddy(F_H1), dh0dx = ddx(F_H0), dh0dy = ddy(F_H0);
      const double exx0 = ddx(F_U0), eyy0 = ddy(F_V0);
      const double dbdx = ddx(F_B1), dbdy = ddy(F_B1), drhodx = ddx(F_RHO), drhody = ddy(F_RHO);
      const double exx = ddx(F_U1), eyy = ddy(F_V1);
      const double exy = 0.5 * (ddx(F_V1) + ddy(F_U1));
      double eta, Ev;
      effective_viscosity(P.uv, Aint, nint, exx, eyy, exy, eta, Ev, cube);  // :149
      Drag d;  // :150
      if (!GEN || (P.uv.law == UA_SLIDING_WEERTMAN && !P.uv.melange)) {
        d = basal_drag_weertman(P.uv, Heint, deltaint, uint, vint, Cint, mint, cube);
      } else {
        int gn[NOD];
        const int e = __ldg(M.patch_elems + e0 + el);
#pragma unroll
        for (int a = 0; a < NOD; ++a) gn[a] = __ldg(M.conn + (size_t)a * M.ne + e);
        d = basal_drag_general(P.uv, Heint, deltaint, hint, Hint, rhoint, rhow, g, uint, vint, Cint, mint,
                               drag_interp<NOD>(in.drag, gn, N));
      }
      const double speed0 = sqrt(u0int * u0int + v0int * v0int + P.SpeedZero * P.SpeedZero);  // :157
      const double tau0 = P.beta0 * supg_tau(P, speed0, lsupg, dt);                         // :158-159
      const double detJw = detJ * Q.w[ip];
      // uvhNodalLoopSSTREAM.m
      const double qx1dx = rhoint * exx * hint + rhoint * uint * dhdx + drhodx * uint * hint;  // :39
      const double qy1dy = rhoint * eyy * hint + rhoint * vint * dhdy + drhody * vint * hint;
      const double qx0dx = rhoint * exx0 * h0int + rhoint * u0int * dh0dx + drhodx * u0int * h0int;
      const double qy0dy = rhoint * eyy0 * h0int + rhoint * v0int * dh0dy + drhody * v0int * h0int;
      const double DxI = Dx[I], DyI = Dy[I], funI = N[I];
      const double SUPG = funI + 0.5 * tau0 * (u0int * DxI + v0int * DyI);  // :55
      if (WITHK) {
        const double Pu_I = (4 * exx + 2 * eyy) * DxI + 2 * exy * DyI;   // h-derivative of t3+t4 / h eta
        const double Pv_I = (4 * eyy + 2 * exx) * DyI + 2 * exy * DxI;
        const double cxh_nn = d.dxh + ca * g * (rhoint - rhow * Dddhint) * dbdx - sa * g * rhoint;
        const double cyh_nn = d.dyh + ca * g * (rhoint - rhow * Dddhint) * dbdy;
        const double ch_d = -ca * g * (rhoint * hint - rhow * dint * Dddhint);
        const double khh_n = rhoint - dt * theta * rhoint * dadhint +
                             dt * theta * (rhoint * exx + drhodx * uint + rhoint * eyy + drhody * vint);
        KT* row = sK + (size_t)I * 9 * NOD * E + el;
#pragma unroll
        for (int J = 0; J < NOD; ++J) {
          const double DxJ = Dx[J], DyJ = Dy[J], fJ = N[J];
          const double Deu = Ev * ((2 * exx + eyy) * DxJ + exy * DyJ);
          const double Dev = Ev * ((2 * eyy + exx) * DyJ + exy * DxJ);
          const double E11 = hint * (4 * exx + 2 * eyy) * Deu * DxI + 2 * hint * exy * Deu * DyI;
          const double E12 = hint * (4 * exx + 2 * eyy) * Dev * DxI + 2 * hint * exy * Dev * DyI;
          const double E22 = hint * (4 * eyy + 2 * exx) * Dev * DyI + 2 * hint * exy * Dev * DxI;
          const double E21 = hint * (4 * eyy + 2 * exx) * Deu * DyI + 2 * hint * exy * Deu * DxI;
          const double he = hint * eta;
          // :84-110 (Kxu, Kyv, Kxv, Kyu), :141-157 post-2025 (Kxh, Kyh), :164-179 (Khu, Khv, Khh)
          row[(0 * NOD + J) * E] += (KT)((4 * he * DxI * DxJ + he * DyI * DyJ + E11 + d.dxu * fJ * funI) * detJw);
          row[(1 * NOD + J) * E] += (KT)((he * (2 * DxI * DyJ + DyI * DxJ) + E12 + d.dxv * fJ * funI) * detJw);
          row[(2 * NOD + J) * E] += (KT)((eta * Pu_I * fJ + cxh_nn * funI * fJ + ch_d * DxI * fJ) * detJw);
          row[(3 * NOD + J) * E] += (KT)((he * (2 * DyI * DxJ + DxI * DyJ) + E21 + d.dxv * fJ * funI) * detJw);
          row[(4 * NOD + J) * E] += (KT)((4 * he * DyI * DyJ + he * DxI * DxJ + E22 + d.dyv * fJ * funI) * detJw);
          row[(5 * NOD + J) * E] += (KT)((eta * Pv_I * fJ + cyh_nn * funI * fJ + ch_d * DyI * fJ) * detJw);
          row[(6 * NOD + J) * E] += (KT)(theta * (rhoint * dhdx * fJ + drhodx * hint * fJ + rhoint * hint * DxJ) *
                                         SUPG * detJw * dt);
          row[(7 * NOD + J) * E] += (KT)(theta * (rhoint * dhdy * fJ + drhody * hint * fJ + rhoint * hint * DyJ) *
                                         SUPG * detJw * dt);
          row[(8 * NOD + J) * E] += (KT)((khh_n * fJ + dt * theta * (rhoint * uint * DxJ + rhoint * vint * DyJ)) *
                                         SUPG * detJw);
        }
      }
      // :189-226 residual
      const double rr = rhoint * hint - rhow * dint;
      const double pp = 0.5 * ca * g * (rhoint * hint * hint - rhow * dint * dint);
      Tx += (hint * eta * (4 * exx + 2 * eyy) * DxI + hint * eta * 2 * exy * DyI + d.taux * funI) * detJw;
      Fx += (-ca * g * rr * dbdx * funI + rhoint * g * hint * sa * funI + pp * DxI) * detJw;
      Ty += (hint * eta * (4 * eyy + 2 * exx) * DyI + hint * eta * 2 * exy * DxI + d.tauy * funI) * detJw;
      Fy += (-ca * g * rr * dbdy * funI + pp * DyI) * detJw;
      const double qterm = dt * (theta * qx1dx + (1 - theta) * qx0dx + theta * qy1dy + (1 - theta) * qy0dy) * SUPG;
      const double dhdt = rhoint * (h0int - hint) * SUPG;  // h0barr = h1barr = 0
      const double accterm = dt * rhoint * ((1 - theta) * a0int + theta * a1int) * SUPG;
      Th += -dhdt * detJw;
      Fh += (accterm - qterm) * detJw;
    }
    sR[(0 * NOD + I) * E + el] = Tx;
    sR[(1 * NOD + I) * E + el] = Fx;
    sR[(2 * NOD + I) * E + el] = Ty;
    sR[(3 * NOD + I) * E + el] = Fy;
    sR[(4 * NOD + I) * E + el] = Th;
    sR[(5 * NOD + I) * E + el] = Fh;
  }
  __syncthreads();
  const int pn0 = M.patch_node_ptr[p];
  const int nr = M.patch_node_ptr[p + 1] - pn0;
  if (WITHK) {
    const int q0 = M.patch_q_ptr[p], q1 = M.patch_q_ptr[p + 1];
    const int nbase = M.nodeptr[no];
    const int nnzn = M.sys_nnzn[s];
    const int kbase = M.sys_knz_off[s];
    KT* Ko = reinterpret_cast<KT*>(out.K);
    for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
      const uint32_t rk = __ldg(M.pq_rk + q);
      const int r = rk >> 16, k = rk & 0xffff;
      const int gnd = __ldg(M.patch_nodes + pn0 + r);
      const int np0 = __ldg(M.nodeptr + gnd);
      const int deg = __ldg(M.nodeptr + gnd + 1) - np0;
      const int lp = np0 - nbase;
      KT v[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) v[i] = 0;
      const int cend = __ldg(M.pq_cptr + q + 1);
      for (int c = __ldg(M.pq_cptr + q); c < cend; ++c) {
        const uint16_t code = __ldg(M.contrib + c);
        int ce = code >> 6;
        const int a = (code >> 3) & 7, b = code & 7;
        bool ok = true;
        UA_CHECK_INDEX(M.dbg, ce, 0, ne, BS_CONTRIB_ELEM, ok);
        if (!ok) continue;
        const KT* src = sK + (size_t)(a * 9 * NOD + b) * E + ce;
#pragma unroll
        for (int i = 0; i < 9; ++i) v[i] += src[(size_t)i * NOD * E];
      }
      {
        size_t last = (size_t)kbase + 6 * (size_t)nnzn + 3 * (size_t)lp + 2 * (size_t)deg + k;  // largest index
        bool okk = true;
        UA_CHECK_INDEX(M.dbg, last, (size_t)kbase, (size_t)M.sys_knz_off[s + 1], BS_K_INDEX, okk);
        (void)last;
        if (!okk) continue;
      }
#pragma unroll
      for (int cr = 0; cr < 3; ++cr) {
        const size_t base = (size_t)kbase + (size_t)cr * 3 * nnzn + 3 * (size_t)lp;
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) Ko[base + (size_t)cc * deg + k] = v[cr * 3 + cc];
      }
    }
  }
  for (int r = threadIdx.x; r < nr; r += blockDim.x) {
    int gnd = __ldg(M.patch_nodes + pn0 + r);
    bool okr = true;
    UA_CHECK_INDEX(M.dbg, gnd, M.sys_node_off[s], M.sys_node_off[s + 1], BS_R_INDEX, okr);
    if (!okr) continue;
    const int q = __ldg(M.prow_diag + pn0 + r);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const int cend = __ldg(M.pq_cptr + q + 1);
    for (int c = __ldg(M.pq_cptr + q); c < cend; ++c) {
      const uint16_t code = __ldg(M.contrib + c);
      int ce = code >> 6;
      const int a = (code >> 3) & 7;
      bool ok = true;
      UA_CHECK_INDEX(M.dbg, ce, 0, ne, BS_CONTRIB_ELEM, ok);
      if (!ok) continue;
#pragma unroll
      for (int i = 0; i < 6; ++i) acc[i] += sR[(i * NOD + a) * E + ce];
    }
    out.R[uoff + gnd] = acc[0] - acc[1];
    out.R[voff + gnd] = acc[2] - acc[3];
    out.R[hoff + gnd] = acc[4] - acc[5];
    if (out.Tint) { out.Tint[uoff + gnd] = acc[0]; out.Tint[voff + gnd] = acc[2]; out.Tint[hoff + gnd] = acc[4]; }
    if (out.Fext) { out.Fext[uoff + gnd] = acc[1]; out.Fext[voff + gnd] = acc[3]; out.Fext[hoff + gnd] = acc[5]; }
  }
}

size_t uvh_patch_smem(int nod, bool withK, bool fp32, int E) {
  const int NB = 9 * nod * nod;
  size_t k = withK ? (((size_t)NB * E * (fp32 ? 4 : 8) + 15) & ~(size_t)15) : 0;
  return k + (size_t)6 * nod * E * 8 + (size_t)F_COUNT * E * nod * 8;
}

int uvh_fields_per_node() { return F_COUNT; }

template <int NOD, bool WITHK, typename KT>
static cudaError_t launch_t(const ua_mesh* m, const UvhPhys& P, const UvhIn& in, const UvOut& out) {
  const int E = m->dm.max_patch_elems;
  size_t sm = uvh_patch_smem(NOD, WITHK, sizeof(KT) == 4, E);
  // the residual-only pass keeps the general build: without the tangent its Weertman-only build
  // spills more registers than the general one
  auto kern = uvh_patch_kernel<NOD, WITHK, KT, true>;
  if constexpr (WITHK) {
    if (P.uv.law == UA_SLIDING_WEERTMAN && !P.uv.melange) kern = uvh_patch_kernel<NOD, WITHK, KT, false>;
  }
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  int threads = ((E * NOD + 31) / 32) * 32;
  if (threads > (NOD == 3 ? 512 : 320)) return cudaErrorInvalidConfiguration;
  kern<<<m->dm.npatch, threads, sm, m->stream>>>(m->dm, quad_table(NOD), P, in, out);
  return cudaGetLastError();
}

cudaError_t launch_uvh_assembly(const ua_mesh* m, const UvhPhys& P, const UvhIn& in, const UvOut& out, bool withK) {
  if (m->nod == 3) return withK ? launch_t<3, true, double>(m, P, in, out) : launch_t<3, false, double>(m, P, in, out);
  return withK ? launch_t<6, true, double>(m, P, in, out) : launch_t<6, false, double>(m, P, in, out);
}

}  // namespace ua
