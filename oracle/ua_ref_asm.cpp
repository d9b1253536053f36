// CPU restatement of the uv element loop of Úa's SSA assembly, in C++ with
// host threads over element ranges.
//
// TEST INFRASTRUCTURE ONLY.  This is the compiled twin of the numpy element
// loop in oracle/ua_ref.py (uv_matrix_assembly): the timed CPU baseline of the
// benchmark and a second, independent restatement that the tests compare
// with the numpy one.  The CUDA library never links or calls it.
//
// It follows UaMain/uvMatrixAssemblySSTREAM.m element by element, in the
// reference's operation order:
//   interpolation at the integration points with the clamps Cint >= Cmin
//   (:205) and AGlenint >= AGlenmin (:243); post-2025 flotation at the
//   integration points (:300-310); nodal-derivative sums (:322-347); drag
//   and viscosity (:351-353, BasalDrag.m:54-77,410-446,
//   EffectiveViscositySSTREAM.m:7-9); the tangent blocks d1d1, d2d2, d1d2,
//   d2d1 with the Newton viscosity terms E11..E22 (:362-425) and the
//   residual terms t1..t5 (:431-449).
// The scatter into the sparse tangent and the residual vector stays in the
// Python oracle (uvMatrixAssemblySSTREAM.m:462-534, MATLAB sparse semantics).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

namespace {

struct Par {
  double kH, Hh0, SpeedZero, EpsZero, etaZero, Czero, Cmin, AGlenmin, Dvisk, rhow, g, ca, sa;
};

// HeavisideApprox.m:86
inline double heaviside_approx(double k, double x, double x0) { return 0.5 + 0.5 * std::tanh(k * (x - x0)); }

// DiracDelta.m:29 (an overflowing cosh gives +inf and a zero result)
inline double dirac_delta(double k, double x, double x0) {
  const double sech = 1.0 / std::cosh(k * (x - x0));
  return 0.5 * k * (sech * sech);
}

}  // namespace

extern "C" {

// Element loop of uvMatrixAssemblySSTREAM.m for all Nele elements.
//   conn    : Nele x nod, row-major, 0-based node ids
//   Deriv   : Nele x 2 x nod x nip, row-major (MUA.Deriv)
//   DetJ    : Nele x nip, row-major (MUA.DetJ)
//   weights : nip;  fun : nip x nod (shape functions at the points)
//   nodal fields h, s, ub, vb, C, m, AGlen, n, S, B, rho (length Nnodes)
//   par     : kH, Hh0, SpeedZero, EpsZero, etaZero, Czero, Cmin, AGlenmin,
//             Dvisk (0 for Picard), rhow, g, cos(alpha), sin(alpha)
//   outputs : d1d1, d2d2, d1d2, d2d1 (Nele x nod x nod, row-major; ignored
//             when Ronly) and Tx, Fx, Ty, Fy (Nele x nod, row-major)
// nthreads <= 0 uses every hardware thread.  Returns 0.
int uvref_element_loop(int64_t Nele, int nod, int nip, const int64_t* conn, const double* Deriv,
                       const double* DetJ, const double* weights, const double* fun, const double* h,
                       const double* s, const double* ub, const double* vb, const double* C, const double* m,
                       const double* AGlen, const double* n, const double* S, const double* B, const double* rho,
                       const double* par_in, int Ronly, int nthreads, double* d1d1, double* d2d2, double* d1d2,
                       double* d2d1, double* Tx, double* Fx, double* Ty, double* Fy) {
  const Par p{par_in[0], par_in[1], par_in[2], par_in[3], par_in[4], par_in[5], par_in[6],
              par_in[7], par_in[8], par_in[9], par_in[10], par_in[11], par_in[12]};
  const int nn2 = nod * nod;
  auto range = [&](int64_t e0, int64_t e1) {
    for (int64_t e = e0; e < e1; ++e) {
      double hn[8], sn[8], un[8], vn[8], Cn[8], mn[8], An[8], nnv[8], Sn[8], Bn[8], rn[8];
      for (int a = 0; a < nod; ++a) {
        const int64_t g = conn[e * nod + a];
        hn[a] = h[g]; sn[a] = s[g]; un[a] = ub[g]; vn[a] = vb[g];
        Cn[a] = C[g]; mn[a] = m[g]; An[a] = AGlen[g]; nnv[a] = n[g];
        Sn[a] = S[g]; Bn[a] = B[g]; rn[a] = rho[g];
      }
      double* K11 = Ronly ? nullptr : d1d1 + e * nn2;
      double* K22 = Ronly ? nullptr : d2d2 + e * nn2;
      double* K12 = Ronly ? nullptr : d1d2 + e * nn2;
      double* K21 = Ronly ? nullptr : d2d1 + e * nn2;
      if (!Ronly)
        for (int i = 0; i < nn2; ++i) K11[i] = K22[i] = K12[i] = K21[i] = 0.0;
      double* tx = Tx + e * nod; double* fx = Fx + e * nod;
      double* ty = Ty + e * nod; double* fy = Fy + e * nod;
      for (int a = 0; a < nod; ++a) tx[a] = fx[a] = ty[a] = fy[a] = 0.0;
      for (int ip = 0; ip < nip; ++ip) {  // :168
        const double* N = fun + ip * nod;
        auto interp = [&](const double* v) {
          double r = 0.0;
          for (int a = 0; a < nod; ++a) r += v[a] * N[a];
          return r;
        };
        const double hint = interp(hn), sint = interp(sn), uint = interp(un), vint = interp(vn);
        double Cint = interp(Cn);
        if (Cint < p.Cmin) Cint = p.Cmin;  // :205
        const double mint = interp(mn);
        double Aint = interp(An);
        if (Aint < p.AGlenmin) Aint = p.AGlenmin;  // :243
        const double nint = interp(nnv), Bint = interp(Bn), Sint = interp(Sn);
        const double Hint = Sint - Bint;
        const double rhoint = interp(rn);
        // flotation at the integration points (:300-310)
        const double hfint = p.rhow * Hint / rhoint;
        const double Heint = heaviside_approx(p.kH, hint - hfint, p.Hh0);
        const double HEint = heaviside_approx(p.kH, hfint - hint, p.Hh0);
        const double deltaint = dirac_delta(p.kH, hint - hfint, p.Hh0);
        const double Hposint = heaviside_approx(p.kH, Hint, p.Hh0) * Hint;
        const double dint = HEint * rhoint * hint / p.rhow + Heint * Hposint;
        // nodal-derivative sums (:322-347)
        const double* Dx = Deriv + ((e * 2 + 0) * nod) * nip;  // Dx[a] = Dx[a*nip + ip]
        const double* Dy = Deriv + ((e * 2 + 1) * nod) * nip;
        double dsdx = 0, dhdx = 0, dsdy = 0, dhdy = 0, exx = 0, eyy = 0, exy = 0;
        for (int a = 0; a < nod; ++a) {
          const double dx = Dx[a * nip + ip], dy = Dy[a * nip + ip];
          dsdx = dsdx + dx * sn[a];
          dhdx = dhdx + dx * hn[a];
          dsdy = dsdy + dy * sn[a];
          dhdy = dhdy + dy * hn[a];
          exx = exx + dx * un[a];
          eyy = eyy + dy * vn[a];
          exy = exy + 0.5 * (dx * vn[a] + dy * un[a]);
        }
        // BasalDrag.m:54-77 and the Weertman branch :410-446
        const double He = Heint < 0 ? 0.0 : Heint;
        const double u0 = p.SpeedZero;
        const double speed = std::sqrt(uint * uint + vint * vint + u0 * u0);
        const double Um = std::pow(speed, 1.0 / mint - 1);
        const double beta2 = std::pow(Cint + p.Czero, -1.0 / mint) * Um;
        const double Dbeta2 = (1.0 / mint - 1) * std::pow(Cint + p.Czero, -1.0 / mint) *
                              std::pow(uint * uint + vint * vint + u0 * u0, (1 - 3 * mint) / (2 * mint));
        const double taux = He * beta2 * uint;
        const double tauy = He * beta2 * vint;
        const double dtauxdu = He * (beta2 + Dbeta2 * uint * uint);
        const double dtauydv = He * (beta2 + Dbeta2 * vint * vint);
        const double dtauxdv = He * Dbeta2 * uint * vint;
        const double dtauydu = dtauxdv;
        (void)deltaint;  // enters only the thickness derivatives of the uvh tangent
        // EffectiveViscositySSTREAM.m:7-9
        const double ee = std::sqrt(p.EpsZero * p.EpsZero + exx * exx + eyy * eyy + exx * eyy + exy * exy);
        const double etaint = 0.5 * std::pow(Aint, -1.0 / nint) * std::pow(ee, (1 - nint) / nint) + p.etaZero;
        const double Eint = (1 - nint) / (4 * nint) * std::pow(Aint, -1.0 / nint) * std::pow(ee, (1 - 3 * nint) / nint);
        const double dbdx = dsdx - dhdx, dbdy = dsdy - dhdy;  // :357
        const double detJw = DetJ[e * nip + ip] * weights[ip];  // :359
        for (int I = 0; I < nod; ++I) {  // :362
          const double dxI = Dx[I * nip + ip], dyI = Dy[I * nip + ip];
          if (!Ronly) {
            for (int J = 0; J < nod; ++J) {
              const double dxJ = Dx[J * nip + ip], dyJ = Dy[J * nip + ip];
              const int k = I * nod + J;
              K11[k] += (4 * hint * etaint * dxI * dxJ + hint * etaint * dyI * dyJ + dtauxdu * N[J] * N[I]) * detJw;
              K22[k] += (4 * hint * etaint * dyI * dyJ + hint * etaint * dxI * dxJ + dtauydv * N[J] * N[I]) * detJw;
              K12[k] += (etaint * hint * (2 * dxI * dyJ + dyI * dxJ) + dtauxdv * N[J] * N[I]) * detJw;
              K21[k] += (etaint * hint * (2 * dyI * dxJ + dxI * dyJ) + dtauydu * N[J] * N[I]) * detJw;
              const double Deu = Eint * ((2 * exx + eyy) * dxJ + exy * dyJ);  // :398
              const double Dev = Eint * ((2 * eyy + exx) * dyJ + exy * dxJ);
              const double E11 = hint * (4 * exx + 2 * eyy) * Deu * dxI + 2 * hint * exy * Deu * dyI;
              const double E12 = hint * (4 * exx + 2 * eyy) * Dev * dxI + 2 * hint * exy * Dev * dyI;
              const double E22 = hint * (4 * eyy + 2 * exx) * Dev * dyI + 2 * hint * exy * Dev * dxI;
              const double E21 = hint * (4 * eyy + 2 * exx) * Deu * dyI + 2 * hint * exy * Deu * dxI;
              K11[k] += p.Dvisk * E11 * detJw;  // :421-424
              K22[k] += p.Dvisk * E22 * detJw;
              K12[k] += p.Dvisk * E12 * detJw;
              K21[k] += p.Dvisk * E21 * detJw;
            }
          }
          // residual terms :431-449
          double t1 = -p.g * (rhoint * hint - p.rhow * dint) * dbdx * N[I] * p.ca + rhoint * p.g * hint * p.sa * N[I];
          double t2 = 0.5 * p.g * p.ca * (rhoint * hint * hint - p.rhow * dint * dint) * dxI;
          double t3 = hint * etaint * (4 * exx + 2 * eyy) * dxI;
          double t4 = hint * etaint * 2 * exy * dyI;
          double t5 = taux * N[I];
          tx[I] += (t3 + t4 + t5) * detJw;
          fx[I] += (t1 + t2) * detJw;
          t1 = -p.g * (rhoint * hint - p.rhow * dint) * dbdy * N[I] * p.ca;
          t2 = 0.5 * p.ca * p.g * (rhoint * hint * hint - p.rhow * dint * dint) * dyI;
          t3 = hint * etaint * (4 * eyy + 2 * exx) * dyI;
          t4 = hint * etaint * 2 * exy * dxI;
          t5 = tauy * N[I];
          ty[I] += (t3 + t4 + t5) * detJw;
          fy[I] += (t1 + t2) * detJw;
        }
      }
    }
  };
  // elements are independent: contiguous ranges on nthreads host threads (1 = the calling thread)
  int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  nt = (int)std::min<int64_t>(nt, std::max<int64_t>(1, Nele / 1024));
  if (nt <= 1) {
    range(0, Nele);
    return 0;
  }
  std::vector<std::thread> pool;
  const int64_t chunk = (Nele + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const int64_t a = t * chunk, b = std::min(Nele, a + chunk);
    if (a < b) pool.emplace_back(range, a, b);
  }
  for (auto& th : pool) th.join();
  return 0;
}

}  // extern "C"
