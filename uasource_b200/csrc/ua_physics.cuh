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
  double pad[3];
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

// EffectiveViscositySSTREAM.m:7-9.  e^((1-3n)/n) = e^((1-n)/n) / e^2, so one
// power of the strain rate serves eta and E (e >= EpsZero > 0).
__device__ __forceinline__ void effective_viscosity(const UvPhys& P, double A, double n, double exx, double eyy,
                                                    double exy, double& eta, double& E) {
  const double e2 = P.EpsZero * P.EpsZero + exx * exx + eyy * eyy + exx * eyy + exy * exy;
  const double e = sqrt(e2);
  const double Am = pow(A, -1.0 / n);
  const double pe = pow(e, (1.0 - n) / n);
  eta = 0.5 * Am * pe + P.etaZero;
  E = (1.0 - n) / (4.0 * n) * Am * pe / e2;
}

// BasalDrag.m:54-77 (clamps, beta^2, Dbeta^2) and the Weertman branch
// (BasalDrag.m:184-186, :410-446).  dtauydu equals dtauxdv (BasalDrag.m:427).
struct Drag {
  double taux, tauy, dxu, dxv, dyv, dxh, dyh;
};

__device__ __forceinline__ Drag basal_drag_weertman(const UvPhys& P, double He, double delta, double u, double v,
                                                    double C, double m) {
  if (delta < 0) delta = 0;
  if (He < 0) He = 0;
  const double u0 = P.SpeedZero;
  const double sp2 = u * u + v * v + u0 * u0;
  const double Cm = pow(C + P.Czero, -1.0 / m);
  // speed^(1/m-1) = sp2^((1-m)/(2m)), and sp2^((1-3m)/(2m)) = sp2^((1-m)/(2m)) / sp2:
  // one power serves beta^2 and its derivative (sp2 >= SpeedZero^2 > 0)
  const double ps = pow(sp2, (1.0 - m) / (2.0 * m));
  const double beta2 = Cm * ps;
  const double Dbeta2 = (1.0 / m - 1.0) * Cm * ps / sp2;
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
