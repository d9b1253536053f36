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
  DragFields drag;        // sliding-law and melange fields (null unless the law reads them)
};

struct UvOut {
  double* R;              // dof vector
  void* K;                // nnz values (double or float), null for R only
  double* Tint;           // optional
  double* Fext;           // optional
};

// Inputs of the uvh assembly (fields at both time levels; level-1 u, v, h in
// the dof vector X, evaluated at X + gamma[s]*dX when dX is given).
struct UvhIn {
  const double *S, *B, *rho, *A, *n, *C, *m;
  const double *h0, *u0, *v0, *as0, *ab0, *as1, *ab1, *dadh;  // dadh may be null (zero)
  const double* X;
  const double* dX;
  const double* gamma;
  const SysScal* scal;
  const int* active;
  int zero_fields;        // uvhMatrixAssembly.m:9-15
  DragFields drag;        // sliding-law and melange fields (null unless the law reads them)
};

struct UvhPhys {
  UvPhys uv;
  double kH, Hh0, SpeedZero, theta, beta0, tau_mult;
  int tau_kind;           // 0 taus, 1 taut, 2 tau1, 3 tau2
};

// Inputs of the adjoint gradient assembly (dIdCq.m): nodal fields, the state and the adjoint
// velocities, all indexed by global node (q, muk, V0 null where the law does not use them).
struct AdjIn {
  const double *h, *S, *B, *rho, *C, *m, *q, *muk, *V0;
  const double *u, *v;
  const double *uA, *vA;
  double rhow, g;
};

cudaError_t adj_mass_matrix(const ua_mesh* m, double* Mval);
cudaError_t adj_dIdC(const ua_mesh* m, const UvPhys& P, const AdjIn& in, double* out);
cudaError_t adj_node_spmv(const ua_mesh* m, const int* nodeptr, const int* nodecol, const double* A,
                          const double* x, double* y);
cudaError_t adj_misfit(const ua_mesh* m, const double* u, const double* v, const double* us, const double* vs,
                       const double* ue, const double* ve, double* ru, double* rv);
cudaError_t adj_misfit_grad(const ua_mesh* m, const double* Mru, const double* Mrv, const double* ue,
                            const double* ve, double area, double* f);
cudaError_t adj_logc(const ua_mesh* m, const double* C, double* g);
cudaError_t adj_dot(cudaStream_t st, int n, const double* a, const double* b, double* part, double* out, int slot);
int adj_cg(const ua_mesh* m, const int* nodeptr, const int* nodecol, const double* A, const double* b, double* x,
           double rtol, int maxit, double* work, double* h_sc);
cudaError_t adj_scale(const ua_mesh* m, double s, double* x);
constexpr int kAdjDotBlocks = 256;  // block partials of the adjoint's dot products

size_t uv_patch_smem(int nod, bool withK, bool fp32, int E);
size_t uvh_patch_smem(int nod, bool withK, bool fp32, int E);
int uvh_fields_per_node();
cudaError_t launch_uvh_assembly(const ua_mesh* m, const UvhPhys& P, const UvhIn& in, const UvOut& out, bool withK);
cudaError_t launch_uv_assembly(const ua_mesh* m, const UvPhys& P, const UvIn& in, const UvOut& out, bool withK,
                               bool fp32K, int threads = 0, int regs = 0);

}  // namespace ua
