// Aggregation AMG preconditioner of the uv tangent (internal interface).
#pragma once
#include "ua_internal.h"

namespace ua {

struct Amg;

// Fine-level view of one preconditioner application z = M^-1 r inside PCG.
// x0 holds the pre-smoothed fine vector (l1-Jacobi of r, written by the
// caller with amg_invd0); z receives the result (and pcopy, if set, a copy);
// part_rz the row-block partials of r.z.
struct AmgPcgView {
  const int *rowptr0, *colind0;
  const void* K0;
  const void* r;
  const void* x0;
  void* z;
  void* pcopy;
  double* part_rz;
  const unsigned char* cmask;
  const int *sel, *done;
  const int *rb_start0, *rb_sys0;
  int nrb0;
  int lpr;     // lanes per fine row (8 or 16)
  void* tmp;   // a free fine-level vector (residual, then corrected iterate)
  // optional timing hook around the fine-level launches (kind 0 restriction, 1 prolongation;
  // phase 0 before, 1 after)
  void (*mark)(void* ctx, int kind, int phase) = nullptr;
  void* mark_ctx = nullptr;
  // optional BF16 copy of K0 for the finest-level residual and smoothing (mixed precision)
  const void* K0lo = nullptr;
  // loop the row-block and node-block kernels over the active-block lists (amg_act_compact)
  bool act = false;
  // finest-level residual and smoothing over the node slices (amg_sell_fill done for this
  // tangent); sell_lo: read their BF16 values
  bool sell = false, sell_lo = false;
};

// Active-block lists.  After every convergence check the row blocks (and, for the smoothed
// transfers, the node blocks) of the systems still iterating are compacted on the device,
// in ascending order; list-driven kernels run a grid of about one wave that loops over the
// list, so converged systems of a batch cost no blocks.
struct ActList {
  const int* map = nullptr;  // list entry -> block id
  const int* cnt = nullptr;  // number of entries (device scalar)
  int cap = 0;               // blocks of the full structure
};
// Build the lists of a uv handle's hierarchy (level 0 uses the handle's row blocks,
// sys_rb_off0 = per-system prefix of those blocks); no-op when built.
int amg_act_init(ua_mesh* m, const std::vector<int>& sys_rb_off0);
// Recompute every list from sel/done (one launch).
void amg_act_compact(ua_mesh* m, const int* sel, const int* done, long long* launches);
ActList amg_act_rows0(const ua_mesh* m);
// grid of a list-driven kernel over at most nblocks blocks of 256 threads
int act_grid(int nblocks, int nsm);

// Build the hierarchy of every system of the handle (host aggregation,
// device structures; smoothed = smoothed-aggregation prolongators, else
// piecewise constant); no-op when built (the first call fixes the kind).  Returns UA_OK or an error code
// (the handle then keeps point-Jacobi).
int amg_setup(ua_mesh* m, bool smoothed);
void amg_free(Amg* a);
int amg_levels(const ua_mesh* m);
// l1-Jacobi inverse row sums of the fine level (VT-typed, valid after amg_numeric)
const void* amg_invd0(const ua_mesh* m);
// Numeric phase for a new tangent K0 (Galerkin products, smoother, coarsest inverses).
// sel (device): the systems of this Newton step (others keep their hierarchies); h_sel (host copy)
// and p_refresh > 1: each system's prolongators are recomputed on the first set-up of its solve
// (amg_restart_P) and then every p_refresh-th set-up, the coarse operators every time.
// graph: run the set-up's launches as a captured CUDA graph (captured once per kind of call).
int amg_numeric(ua_mesh* m, const int* rowptr0, const int* colind0, const void* K0, bool fp32,
                const unsigned char* cmask, long long* launches, const int* sel = nullptr,
                const std::vector<int>* h_sel = nullptr, int p_refresh = 1, bool graph = false);
// the systems of `run` start a solve: their next set-up recomputes the prolongators
void amg_restart_P(ua_mesh* m, const std::vector<int>& run);
// uvh handles: extract the velocity block of the 3-dof tangent K3 (and its
// constraint mask) into the hierarchy's own finest level, then the numeric
// phase (FP64).
int amg_numeric_uvh(ua_mesh* m, const double* K3, const unsigned char* cmask3, long long* launches);
// out3 = V-cycle(p3) on the velocity rows of 3-dof vectors (other rows untouched).
int amg_apply_uvh(ua_mesh* m, const double* p3, double* out3, const int* sel, const int* done, int lpr,
                  long long* launches);
// Node slices of a uv handle's finest level (structure once per handle; call before
// amg_act_init so that the slice blocks get an active list).  sys_rb_off0 is the handle's
// per-system row-block prefix; its row blocks must split at the u/v boundary.  UA_OK, else an
// error code and the CSR kernels stay in use.
int amg_sell_init(ua_mesh* m, const std::vector<int>& sys_rb_off0);
// Slice values of a new tangent K0 (KT = float if fp32, else double); lo: also the BF16 copy.
int amg_sell_fill(ua_mesh* m, const void* K0, bool fp32, bool lo, long long* launches, const int* sel = nullptr);
// Per-slice partials of the node-slice SpMV (p.q) and smoothing (r.z), and the per-system
// slice prefix (the PCG reductions sum these instead of the row-block partials).
void amg_sell_partials(const ua_mesh* m, const double** spart, const int** sys_sl_off);
// PCG SpMV over the node slices: q = mask(K p), partials p.q per slice (amg_sell_partials).
int amg_sell_spmv(ua_mesh* m, bool fp32, bool act, const int* sel, const int* done, const void* p,
                  const unsigned char* cmask, void* q, long long* launches);
// Refresh the BF16 copy of an FP32 finest-level tangent (allocated on first use;
// nullptr if that fails).
const void* amg_bf16_copy(ua_mesh* m, const float* K0, long long nnz, long long* launches);
// One V(1,1) cycle.  The finest level runs as row-block kernels (residual,
// aggregation, correction, smoothing); coarser levels use one thread per aggregate.
int amg_vcycle(ua_mesh* m, bool fp32, const AmgPcgView& v, long long* launches);

}  // namespace ua
