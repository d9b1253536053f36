// Device restatement of the SSA constitutive, drag and flotation functions.
#pragma once
#include <cuda_runtime.h>

namespace ua {

struct UvPhys {            // CtrlVar subset used inside the element loop
  double kH, Hh0, SpeedZero, EpsZero, etaZero, Czero, Cmin, AGlenmin, Dvisk;
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

}  // namespace ua
