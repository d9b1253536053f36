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

// EffectiveViscositySSTREAM.m:7-9
__device__ __forceinline__ void effective_viscosity(const UvPhys& P, double A, double n, double exx, double eyy,
                                                    double exy, double& eta, double& E) {
  double e = sqrt(P.EpsZero * P.EpsZero + exx * exx + eyy * eyy + exx * eyy + exy * exy);
  double Am = pow(A, -1.0 / n);
  eta = 0.5 * Am * pow(e, (1.0 - n) / n) + P.etaZero;
  E = (1.0 - n) / (4.0 * n) * Am * pow(e, (1.0 - 3.0 * n) / n);
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
  double u0 = P.SpeedZero;
  double sp2 = u * u + v * v + u0 * u0;
  double speed = sqrt(sp2);
  double Cm = pow(C + P.Czero, -1.0 / m);
  double beta2 = Cm * pow(speed, 1.0 / m - 1.0);
  double Dbeta2 = (1.0 / m - 1.0) * Cm * pow(sp2, (1.0 - 3.0 * m) / (2.0 * m));
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
