// Resumable restatement of BackTracking.m (plus CubicFit.m, parabolamin.m).
//
// The reference calls the cost function from inside BackTracking; here the
// search is a state machine so that many systems of a batch can advance
// together: next() returns true and sets `request` when the cost at gamma =
// request is needed, and feed(f) supplies it.  The sequence of requested
// gammas and the returned (gmin, fmin, Converged, iarm) are those of
// BackTracking.m:54-759 with plotting removed.
#pragma once
#include <cmath>
#include <limits>
#include <vector>

namespace ua {

struct BTConfig {
  double beta = 0.1, ExtrapolationRatio = 2.5, MinXfracRel = 1e-10, GL = 0.25, GU = 0.95;
  double NewtonAcceptRatio = 0.5, GammaMin = 1e-10, NLtol = 1e-15;
  int MaxIterations = 50, MaxExtrapolations = 50, MaxFuncSame = 3;
  bool allow_ext = false;
};

// parabolamin.m
inline double parabolamin(double a, double b, double c, double fa, double fb, double fc) {
  if (c < b) { std::swap(b, c); std::swap(fb, fc); }
  if (!(a < b && b < c)) return std::numeric_limits<double>::quiet_NaN();
  if (std::isinf(fa) && std::isinf(fb) && std::isinf(fc)) return a / 100;
  if (std::isinf(fb) && std::isinf(fc)) return b == b ? b / 100 : 1e-5;
  double t1 = (b - a) * (b - a) * (fb - fc);
  double t2 = (b - c) * (b - c) * (fb - fa);
  double t3 = (b - a) * (fb - fc);
  double t4 = (b - c) * (fb - fa);
  double xmin = t3 != t4 ? b - 0.5 * (t1 - t2) / (t3 - t4) : std::numeric_limits<double>::quiet_NaN();
  if (xmin != xmin || (fa + (b - a) * (fc - fa) / (c - a) < fb)) {
    if (fc < fb && fb < fa) xmin = 5 * c;
    else if (fc > fb && fb > fa) xmin = a + b / 10;
    else if (fc > fa && fb > fa) xmin = a + b / 100;
    else xmin = (a + b) / 3;
  }
  return xmin;
}

// CubicFit.m
inline double cubic_fit(double slope, double y0, double y1, double y2, double x1, double x2) {
  const double nan = std::numeric_limits<double>::quiet_NaN();
  if (x1 > x2) { std::swap(x1, x2); std::swap(y1, y2); }
  double xmin;
  if (x1 == x2) {
    double D = (y1 - y0) / x1 - slope;
    xmin = D != 0 ? -x1 * slope / 2 / D : x1 * 0.9;
  } else {
    double r1 = y1 - slope * x1 - y0, r2 = y2 - slope * x2 - y0;
    double a = (r1 / (x1 * x1) - r2 / (x2 * x2)) / (x1 - x2);
    double b = (-x2 * r1 / (x1 * x1) + x1 * r2 / (x2 * x2)) / (x1 - x2);
    double disc = b * b - 3 * a * slope;
    xmin = (a == 0 || disc < 0) ? nan : (-b + std::sqrt(disc)) / 3 / a;
    if (a == 0 || xmin != xmin) {
      if (slope == slope) {
        double D = (y1 - y0) / x1 - slope;
        xmin = D != 0 ? -x1 * slope / 2 / D : nan;
      } else {
        xmin = parabolamin(0, x1, x2, y0, y1, y2);
      }
    }
  }
  if (xmin != xmin) {
    if (y0 < y1 && y1 < y2) xmin = x1 / 2;
    else if (y0 > y1 && y1 > y2) xmin = x1 + (x2 - x1) / 2;
    else if (y0 < y1 && y1 > y2) xmin = y2 < y0 ? x1 + (x2 - x1) / 2 : x1 / 2;
  }
  return xmin;
}

class BackTrack {
 public:
  BTConfig cfg;
  // results
  double gmin = 0, fmin = 0;
  int iarm = 0, converged = 0, nfe = 0, nextrap = 0;
  bool done = false, error = false;
  double request = 0;
  std::vector<double> xs, fs;  // Infovector

  // BackTracking(slope0, b, fa, fb, Func, CtrlVar); returns true if an evaluation is requested.
  bool start(double slope0_, double b_, double fa_, double fb_) {
    slope0 = slope0_; b = b_; fa = fa_; fb = fb_;
    MinXfrac = cfg.MinXfracRel * b;
    NoSlope = !(slope0 == slope0);
    if (!NoSlope && slope0 > 0) { done = true; error = true; gmin = fmin = std::nan(""); return false; }
    target = std::max(cfg.NewtonAcceptRatio * fa, cfg.NLtol);  // :160
    if (!NoSlope) {
      double tws = std::min(fa + cfg.beta * slope0 * b, cfg.NewtonAcceptRatio * fa);
      target = std::max(target, tws);
      if (target < 0) target = std::max(cfg.NewtonAcceptRatio * fa, cfg.NLtol);
    }
    a = 0; f0 = fa;
    push(a, fa); push(b, fb);
    if (fb < target) { converged = 1; return finish_early(); }  // :239-265
    gamma = !NoSlope ? -b * slope0 / 2 / ((fb - fa) / b - slope0) : a + 0.9 * (b - a);  // :268
    if (gamma > cfg.GU * b) gamma = cfg.GU * b;
    else if (gamma < cfg.GL * b) gamma = cfg.GL * b;
    if (fmin > target) {  // :282
      iarm = 1;
      state = S_FIRST;
      return ask(gamma);
    }
    gammaOld = gamma; gamma = b; fgamma = fb;
    return after_first();
  }

  // supply f(request); returns true if another evaluation is requested.
  bool feed(double f) {
    nfe++;
    switch (state) {
      case S_FIRST:
        fgamma = f; gammaOld = gamma; push(gamma, fgamma);
        return after_first();
      case S_EXTRAP: {
        fgamma = f; push(gamma, fgamma);
        fbOld = fb; bOld = b; fb = fc; b = c; fc = fgamma; c = gamma;
        if (nextrap > cfg.MaxExtrapolations) return after_extrap();
        return extrap_loop();
      }
      case S_MID:
        fb = f; push(b, fb);
        fLastReduction = 1;
        return loop_head();
      case S_LOOP:
        return loop_tail(f);
      default:
        return false;
    }
  }

 private:
  enum State { S_NONE, S_FIRST, S_EXTRAP, S_MID, S_LOOP };
  State state = S_NONE;
  double slope0 = 0, a = 0, b = 1, c = 0, fa = 0, fb = 0, fc = 0, f0 = 0, target = 0, gamma = 0, fgamma = 0;
  double gammaOld = 0, xfrac = 1e10, MinXfrac = 0, fLastReduction = 1, bOld = 0, fbOld = 0;
  int iMinSame = 0, iMinSameWB = 0;
  bool NoSlope = false;

  void push(double x, double f) {
    xs.push_back(x); fs.push_back(f);
    // [fmin,I]=min(Infovector(:,2)) -- first index of the minimum, NaN ignored
    int I = -1;
    for (size_t i = 0; i < fs.size(); ++i)
      if (fs[i] == fs[i] && (I < 0 || fs[i] < fs[I])) I = (int)i;
    if (I >= 0) { fmin = fs[I]; gmin = xs[I]; }
  }
  bool ask(double g) { request = g; return true; }
  bool finish_early() { done = true; return false; }

  bool after_first() {  // :304-372
    c = b; fc = fb; b = gamma; fb = fgamma;
    if (cfg.allow_ext) return extrap_loop();
    return after_extrap();
  }
  bool extrap_loop() {
    if (fb < fa && fc < fb && fmin > target) {
      nextrap++;
      gamma = cfg.ExtrapolationRatio * c;
      gammaOld = gamma;
      state = S_EXTRAP;
      return ask(gamma);
    }
    return after_extrap();
  }
  bool after_extrap() {  // :388-405
    if (nextrap > 0) {
      a = bOld; fa = fbOld; b = (a + c) / 2;
      NoSlope = true;
      state = S_MID;
      return ask(b);
    }
    fLastReduction = 1;
    return loop_head();
  }
  bool loop_head() {  // :408-431
    if (!((fgamma > target || fLastReduction < 0.5))) return finish();
    iarm++;
    gamma = NoSlope ? parabolamin(a, b, c, fa, fb, fc) : cubic_fit(slope0, fa, fb, fc, b, c);
    if (gamma != gamma) { error = true; return finish(); }
    if (iarm == 2 && nextrap > 0) {
      if (gamma > b + 0.95 * (c - b)) gamma = b + 0.95 * (c - b);
      else if (gamma < a + 0.25 * (b - a)) gamma = a + 0.25 * (b - a);
      branch = 0;
    } else if (gamma > b && gamma < c) {
      if (gamma < (b + cfg.GU * (c - a))) gamma = b + cfg.GU * (c - a);
      else if (gamma > (c - cfg.GL * (c - b))) gamma = c - cfg.GL * (c - b);
      branch = 1;
    } else {
      if (gamma > (a + cfg.GU * (b - a))) gamma = a + cfg.GU * (b - a);
      else if (gamma < (a + cfg.GL * (b - a))) gamma = a + cfg.GL * (b - a);
      branch = 2;
    }
    state = S_LOOP;
    return ask(gamma);
  }
  int branch = 0;
  bool loop_tail(double f) {  // :433-624
    fgamma = f;
    if (branch == 0) {
      if (gamma < b && fgamma < fb) { c = b; fc = fb; b = gamma; fb = fgamma; }
      else if (gamma > b && fgamma < fb) { b = c; fb = fc; c = gamma; fc = fgamma; }
    } else if (branch == 1) {
      b = gamma; fb = fgamma;
    } else {
      c = b; fc = fb; b = gamma; fb = fgamma;
    }
    double fminOld = fmin, gminOld = gmin;
    push(gamma, fgamma);
    fLastReduction = fmin / fminOld;
    if (gmin != gminOld) { xfrac = std::fabs(gmin - gminOld); MinXfrac = gmin * 1e-10; }
    iMinSame = (fmin == fminOld) ? iMinSame + 1 : 0;
    iMinSameWB = (gamma < gammaOld && fmin == fminOld) ? iMinSameWB + 1 : 0;
    gammaOld = gamma;
    if (!NoSlope) {
      target = fa + cfg.beta * slope0 * b;  // :567
      if (target < 0) target = std::max(cfg.NewtonAcceptRatio * fa, cfg.NLtol);
    }
    if (iMinSame > cfg.MaxFuncSame && fmin < f0) return finish();
    if (iarm > 5 && iMinSameWB > 2 && fmin < f0) return finish();
    if (xfrac < MinXfrac && fmin < f0) return finish();
    if (b < cfg.GammaMin) return finish();
    if (iarm > cfg.MaxIterations) return finish();
    return loop_head();
  }
  bool finish() {  // :626-633
    const double eps = 2.220446049250313e-16;
    if (fgamma < (target - eps)) converged = 1;
    else if (std::fabs(fmin - fa) / fa > 1e-5 && gamma > cfg.GammaMin) converged = 1;
    else converged = 0;
    done = true;
    return false;
  }
};

}  // namespace ua
