// Device restatement of the SSA constitutive, drag and flotation functions.
#pragma once
#include <cuda_runtime.h>
#include "../../include/ua_ssa.h"

namespace ua {

struct UvPhys {            // CtrlVar subset used inside the element loop
  double kH, Hh0, SpeedZero, EpsZero, etaZero, Czero, Cmin, AGlenmin, Dvisk;
  double Nzero;            // CtrlVar.Nzero (effective pressure floor)
  int law;                 // CtrlVar.SlidingLaw (UA_SLIDING_*)
  int melange;             // CtrlVar.IncludeMelangeModelPhysics
};

// Integration-point values of the fields the other sliding laws and the melange
// terms read (uvMatrixAssemblySSTREAM.m:210-254); unused ones are zero.
struct DragIp {
  double q, muk, V0;
  double uo, vo, Co, mo, ua, va, Ca, ma;
};

// Nodal arrays of those fields (global node index; null when the law does not use them).
struct DragFields {
  const double *q, *muk, *V0;
  const double* mel[8];  // uo, vo, Co, mo, ua, va, Ca, ma
};

struct SysScal {           // per-system F scalars
  double rhow, g, ca, sa;  // F.rhow, F.g, cos(F.alpha), sin(F.alpha)
  double dt;               // uvh time step
  double cube;             // 1 when n = m = 3 at every node of the system (set on the device)
  double pad[2];
};

// HeavisideApprox.m:86
__device__ __forceinline__ double heaviside_approx(double k, double x, double x0) {
  return 0.5 + 0.5 * tanh(k * (x - x0));
}

// DiracDelta.m:29 (0.5 k sech^2); cosh overflow gives +inf and a zero result.
__device__ __forceinline__ double dirac_delta(double k, double x, double x0) {
  double c = cosh(k * (x - x0));
  return 0.5 * k / (c * c);
}

// tanh z and 0.5 k sech^2 z of z = k (x - x0) from one expm1, by the identities
// tanh z = sign(z) (1 - e^-2|z|) / (1 + e^-2|z|) and sech^2 z = 4 e^-2|z| / (1 + e^-2|z|)^2
// (expm1 keeps small |z| accurate).  The smooth step HeavisideApprox.m:86 is 0.5 + 0.5 t, its
// mirror H(x0 - x) for x0 = 0 is 0.5 - 0.5 t, and delta is DiracDelta.m:29 (even in z).
struct StepPulse {
  double t, delta;
};
__device__ __forceinline__ StepPulse step_pulse(double k, double x, double x0) {
  const double z = k * (x - x0);
  const double em = expm1(-2.0 * fabs(z));
  const double q = 2.0 + em;
  StepPulse r;
  r.t = copysign(-em / q, z);
  r.delta = 2.0 * k * (1.0 + em) / (q * q);
  return r;
}

// EffectiveViscositySSTREAM.m:7-9.  e^((1-3n)/n) = e^((1-n)/n) / e^2, so one
// power of the strain rate serves eta and E (e >= EpsZero > 0).
// With n = 3 (cube) the powers are reciprocal cube roots: A^(-1/3) and e^(-2/3) = (e^2)^(-1/3).
__device__ __forceinline__ void effective_viscosity(const UvPhys& P, double A, double n, double exx, double eyy,
                                                    double exy, double& eta, double& E, bool cube = false) {
  const double e2 = P.EpsZero * P.EpsZero + exx * exx + eyy * eyy + exx * eyy + exy * exy;
  double Am, pe, c;
  if (cube) {
    Am = rcbrt(A);
    pe = rcbrt(e2);
    c = -1.0 / 6.0;
  } else {
    Am = pow(A, -1.0 / n);
    pe = pow(sqrt(e2), (1.0 - n) / n);
    c = (1.0 - n) / (4.0 * n);
  }
  eta = 0.5 * Am * pe + P.etaZero;
  E = c * Am * pe / e2;
}

// BasalDrag.m:54-77 (clamps, beta^2, Dbeta^2) and the Weertman branch
// (BasalDrag.m:184-186, :410-446).  dtauydu equals dtauxdv (BasalDrag.m:427).
struct Drag {
  double taux, tauy, dxu, dxv, dyv, dxh, dyh;
};

// With m = 3 (cube): (C+C0)^(-1/3) and sp2^(-1/3) by reciprocal cube roots.
__device__ __forceinline__ Drag basal_drag_weertman(const UvPhys& P, double He, double delta, double u, double v,
                                                    double C, double m, bool cube = false) {
  if (delta < 0) delta = 0;
  if (He < 0) He = 0;
  const double u0 = P.SpeedZero;
  const double sp2 = u * u + v * v + u0 * u0;
  // speed^(1/m-1) = sp2^((1-m)/(2m)), and sp2^((1-3m)/(2m)) = sp2^((1-m)/(2m)) / sp2:
  // one power serves beta^2 and its derivative (sp2 >= SpeedZero^2 > 0)
  const double Cm = cube ? rcbrt(C + P.Czero) : pow(C + P.Czero, -1.0 / m);
  const double ps = cube ? rcbrt(sp2) : pow(sp2, (1.0 - m) / (2.0 * m));
  const double beta2 = Cm * ps;
  const double Dbeta2 = (cube ? -2.0 / 3.0 : 1.0 / m - 1.0) * Cm * ps / sp2;
  Drag d;
  d.taux = He * beta2 * u;
  d.tauy = He * beta2 * v;
  d.dxu = He * (beta2 + Dbeta2 * u * u);
  d.dyv = He * (beta2 + Dbeta2 * v * v);
  d.dxv = He * Dbeta2 * u * v;
  d.dxh = delta * beta2 * u;
  d.dyh = delta * beta2 * v;
  return d;
}

// N0 of BasalDrag.m (zeroth-order hydrology): N = rho g max(h - hf, 0) + Nzero with
// hf = rhow H / rho (values below eps taken as 0), dN/dh = rho g where h > hf.
__device__ __forceinline__ void effective_pressure_n0(const UvPhys& P, double h, double H, double rho, double rhow,
                                                      double g, double& N, double& dNdh, double& Dh) {
  const double eps = 2.220446049250313e-16;
  double hf = rhow * H / rho;
  if (hf < eps) hf = 0.0;
  Dh = h - hf;
  const bool dry = Dh < eps;
  if (dry) Dh = 0.0;
  N = rho * g * Dh + P.Nzero;
  dNdh = dry ? 0.0 : rho * g;
}

// An isotropic law |tau| = T(U) with tau = T (u, v) / U: A = T/U, B = (T' - T/U)/U^2 give
// tau_x = A u, d tau_x/du = A + B u^2, d tau_x/dv = B u v, d tau_y/dv = A + B v^2.
__device__ __forceinline__ void isotropic_drag(double A, double B, double u, double v, Drag& d) {
  d.taux = A * u; d.tauy = A * v;
  d.dxu = A + B * u * u; d.dyv = A + B * v * v; d.dxv = B * u * v;
}

// BasalDrag.m:44-363 for every CtrlVar.SlidingLaw, plus the melange terms (:275-343).
// Weertman, Budd and Coulomb follow the reference's expressions (:410-490, :365-408);
// Tsai takes the smaller of the Weertman and Coulomb stresses pointwise (:207-244).
// Cornford (rpCWN0.m), Umbi (rCWN0.m) and Joughin (rCWV0.m) are written through their
// stresses |tau| = mu N W / ((mu N)^m + W^m)^(1/m), mu N W / (mu N + W) and
// W (U + V0)^(-1/m), W = He (C + C0)^(-1/m) U^(1/m), and their velocity derivatives
// (isotropic_drag); their thickness derivatives are the reference's expressions, which
// evaluate the Heaviside factor of the delta term at 1/2.
__device__ inline Drag basal_drag_general(const UvPhys& P, double He, double delta, double h, double H,
                                          double rho, double rhow, double g, double u, double v, double C,
                                          double m, const DragIp& x) {
  const double eps = 2.220446049250313e-16;
  if (delta < 0) delta = 0;
  if (He < 0) He = 0;
  const double C0 = P.Czero, u0 = P.SpeedZero;
  const double sp2 = u * u + v * v + u0 * u0;
  const double speed = sqrt(sp2);
  const double cm = pow(C + C0, -1.0 / m);
  const double beta2 = cm * pow(speed, 1.0 / m - 1);
  const double Dbeta2 = (1.0 / m - 1) * cm * pow(sp2, (1 - 3 * m) / (2 * m));
  Drag d{};
  auto weertman = [&](Drag& r) {
    r.taux = He * beta2 * u; r.tauy = He * beta2 * v;
    r.dxu = He * (beta2 + Dbeta2 * u * u); r.dyv = He * (beta2 + Dbeta2 * v * v); r.dxv = He * Dbeta2 * u * v;
    r.dxh = delta * beta2 * u; r.dyh = delta * beta2 * v;
  };
  auto coulomb = [&](Drag& r, double N, double dNdh, double Dh) {
    const double Tau = x.muk * N;
    r.taux = Tau * u / speed; r.tauy = Tau * v / speed;
    const double temp = speed * speed * speed;
    r.dxu = Tau * (1 / speed - u * u / temp); r.dyv = Tau * (1 / speed - v * v / temp);
    r.dxv = -Tau * u * v / temp;
    const double E = Dh < eps ? 0.0 : x.muk * dNdh / speed;
    r.dxh = E * u; r.dyh = E * v;
  };
  double N = 0, dNdh = 0, Dh = 0;
  if (P.law != UA_SLIDING_WEERTMAN && P.law != UA_SLIDING_JOUGHIN)
    effective_pressure_n0(P, h, H, rho, rhow, g, N, dNdh, Dh);
  switch (P.law) {
    case UA_SLIDING_BUDD: {
      const double qm = x.q / m, Nqm = pow(N, qm);
      const double T = He * Nqm * beta2;
      const double E = delta * T + He * qm * pow(N, qm - 1) * dNdh * beta2;
      d.taux = T * u; d.tauy = T * v;
      d.dxu = He * Nqm * (beta2 + Dbeta2 * u * u); d.dyv = He * Nqm * (beta2 + Dbeta2 * v * v);
      d.dxv = He * Nqm * Dbeta2 * u * v;
      d.dxh = E * u; d.dyh = E * v;
      break;
    }
    case UA_SLIDING_COULOMB:
      coulomb(d, N, dNdh, Dh);
      break;
    case UA_SLIDING_TSAI: {
      Drag w{}, c{};
      weertman(w);
      coulomb(c, N, dNdh, Dh);
      d = (c.taux * c.taux + c.tauy * c.tauy < w.taux * w.taux + w.tauy * w.tauy) ? c : w;
      break;
    }
    case UA_SLIDING_CORNFORD: {
      const double muN = x.muk * N, cu = cm * pow(speed, 1.0 / m);
      const double W = He * cu, S = pow(muN, m) + pow(W, m);
      const double TU = muN * He * cm * pow(speed, 1.0 / m - 1) * pow(S, -1.0 / m);
      const double Tp = muN * (W / (m * speed)) * pow(muN, m) * pow(S, -1.0 / m - 1);
      isotropic_drag(TU, (Tp - TU) / sp2, u, v, d);
      const double Wm = pow(cu, m), us = cm * pow(speed, 1.0 / m - 1);
      const double E = pow(2.0, m + 1) * pow(muN, m + 1) * delta * us * pow(pow(2.0, m) * pow(muN, m) + Wm, -(m + 1) / m) +
                       x.muk * dNdh * pow(He, m + 1) * us * Wm * pow(S, -(m + 1) / m);
      d.dxh = E * u; d.dyh = E * v;
      break;
    }
    case UA_SLIDING_UMBI: {
      const double c1 = pow(C + C0, 1.0 / m), muN = x.muk * N, sm = pow(speed, 1.0 / m);
      const double den = muN * c1 + He * sm;
      const double TU = muN * He * pow(speed, 1.0 / m - 1) / den;
      const double W = He * sm / c1;
      const double Tp = muN * muN * W / (m * speed * (muN + W) * (muN + W));
      isotropic_drag(TU, (Tp - TU) / sp2, u, v, d);
      const double den2 = 2 * muN * c1 + sm;
      const double E = x.muk * dNdh * He * pow(speed, 2.0 / m - 1) / (den * den) +
                       4.0 * x.muk * x.muk * N * N * delta * c1 * pow(speed, 1.0 / m - 1) / (den2 * den2);
      d.dxh = E * u; d.dyh = E * v;
      break;
    }
    case UA_SLIDING_JOUGHIN: {
      const double us = cm * pow(x.V0 + speed, -1.0 / m) * pow(speed, 1.0 / m - 1);
      const double TU = He * us;
      const double Tp = TU * x.V0 / (m * (speed + x.V0));
      isotropic_drag(TU, (Tp - TU) / sp2, u, v, d);
      d.dxh = delta * us * u; d.dyh = delta * us * v;
      break;
    }
    default:
      weertman(d);
  }
  if (P.melange) {  // ocean and atmosphere drag on the floating part
    const double w0[2][4] = {{x.uo, x.vo, x.Co, x.mo}, {x.ua, x.va, x.Ca, x.ma}};
    for (int k = 0; k < 2; ++k) {
      const double U = u - w0[k][0], V = v - w0[k][1], Cw = w0[k][2], mw = w0[k][3];
      const double s2 = U * U + V * V + u0 * u0;
      const double cw = pow(Cw + C0, -1.0 / mw);
      const double b2 = cw * pow(sqrt(s2), 1.0 / mw - 1);
      const double Db2 = (1.0 / mw - 1) * cw * pow(s2, (1 - 3 * mw) / (2 * mw));
      d.taux += (1 - He) * b2 * U; d.tauy += (1 - He) * b2 * V;
      d.dxu += (1 - He) * (b2 + Db2 * U * U); d.dyv += (1 - He) * (b2 + Db2 * V * V);
      d.dxv += (1 - He) * (Db2 * U * V);
      d.dxh += -delta * b2 * U; d.dyh += -delta * b2 * V;
    }
  }
  return d;
}

// BasalDrag.m:80-160 (CtrlVar.Inverse.dFuvdClambda): the derivative with respect to C of the drag
// magnitude over speed, per sliding law, as the adjoint gradient dIdCq.m uses it.  Budd takes
// N = rho g max(h - hf, 0) without Nzero (:120-126); Tsai is the Weertman term where the Weertman
// stress is the smaller one and 0 where Coulomb applies (:137-147).  Coulomb has none (the host
// refuses it).
__device__ inline double dFuvdC(const UvPhys& P, double He, double h, double H, double rho, double rhow, double g,
                                double u, double v, double C, double m, double q, double muk, double V0) {
  const double eps = 2.220446049250313e-16;
  if (He < 0) He = 0;
  const double C0 = P.Czero, u0 = P.SpeedZero;
  const double speed = sqrt(u * u + v * v + u0 * u0);
  const double Um = pow(speed, 1.0 / m - 1);
  double N = 0, dNdh = 0, Dh = 0;
  switch (P.law) {
    case UA_SLIDING_BUDD: {
      double hf = rhow * H / rho;
      if (hf < eps) hf = 0;
      double D = h - hf;
      if (D < eps) D = 0;
      const double Nb = rho * g * D;
      return He * pow(Nb, q / m) * (1.0 / m) * pow(C + C0, -1.0 / m - 1) * Um;
    }
    case UA_SLIDING_CORNFORD:
      effective_pressure_n0(P, h, H, rho, rhow, g, N, dNdh, Dh);
      return (pow(speed, 1.0 / m - 1) * pow(muk, m + 1) * pow(N, m + 1) * He *
              pow(pow(muk, m) * pow(N, m) + speed * pow(He * pow(C + C0, -1.0 / m), m), -1.0 / m - 1) *
              pow(C + C0, -1.0 / m - 1)) / m;
    case UA_SLIDING_UMBI: {
      effective_pressure_n0(P, h, H, rho, rhow, g, N, dNdh, Dh);
      const double den = pow(speed, 1.0 / m) * He + muk * N * pow(C + C0, 1.0 / m);
      return (pow(speed, 1.0 / m) * muk * muk * N * N * He / (den * den) * pow(C + C0, 1.0 / m - 1)) / (speed * m);
    }
    case UA_SLIDING_TSAI: {
      effective_pressure_n0(P, h, H, rho, rhow, g, N, dNdh, Dh);
      const double beta2 = pow(C + C0, -1.0 / m) * Um;
      const double tw2 = (He * beta2 * u) * (He * beta2 * u) + (He * beta2 * v) * (He * beta2 * v);
      const double Tau = muk * N;
      const double tc2 = (Tau * u / speed) * (Tau * u / speed) + (Tau * v / speed) * (Tau * v / speed);
      return tc2 < tw2 ? 0.0 : He * (1.0 / m) * pow(C + C0, -1.0 / m - 1) * Um;
    }
    case UA_SLIDING_JOUGHIN:
      return (pow(speed, 1.0 / m - 1) * He * pow(speed + V0, -1.0 / m) * pow(C + C0, -1.0 / m - 1)) / m;
    default:
      return He * (1.0 / m) * pow(C + C0, -1.0 / m - 1) * Um;
  }
}

// Interpolated sliding-law fields at an integration point (nodal values times N).
template <int NOD>
__device__ __forceinline__ DragIp drag_interp(const DragFields& F, const int (&gn)[NOD], const double* N) {
  DragIp x{};
  auto at = [&](const double* f) {
    double r = 0.0;
    if (f)
#pragma unroll
      for (int a = 0; a < NOD; ++a) r += __ldg(f + gn[a]) * N[a];
    return r;
  };
  x.q = at(F.q); x.muk = at(F.muk); x.V0 = at(F.V0);
  x.uo = at(F.mel[0]); x.vo = at(F.mel[1]); x.Co = at(F.mel[2]); x.mo = at(F.mel[3]);
  x.ua = at(F.mel[4]); x.va = at(F.mel[5]); x.Ca = at(F.mel[6]); x.ma = at(F.mel[7]);
  return x;
}

}  // namespace ua
