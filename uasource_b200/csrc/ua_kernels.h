// Kernel launch interfaces shared between the library's translation units.
#pragma once
#include "ua_internal.h"
#include "ua_physics.cuh"

namespace ua {

// Inputs of the uv assembly.  Nodal fields are indexed by global node id;
// velocities live in the dof vector X (system-major [u_s; v_s]) and the
// assembly evaluates at X + gamma[s]*dX when dX is given (CalcCostFunctionNR.m:14-16).
struct UvIn {
  const double *h, *s, *S, *B, *rho, *A, *n, *C, *m;
  const double* X;
  const double* dX;       // may be null
  const double* gamma;    // [nsys], may be null
  const SysScal* scal;    // [nsys]
  const int* active;      // [nsys], may be null (all active)
};

struct UvOut {
  double* R;              // dof vector
  void* K;                // nnz values (double or float), null for R only
  double* Tint;           // optional
  double* Fext;           // optional
};

size_t uv_patch_smem(int nod, bool withK, bool fp32, int E);
cudaError_t launch_uv_assembly(const ua_mesh* m, const UvPhys& P, const UvIn& in, const UvOut& out, bool withK,
                               bool fp32K);

}  // namespace ua
