// Aggregation AMG preconditioner for the constrained uv tangent.
//
// Preconditions the inner PCG that replaces the reference's direct solve of
// the Newton system (ABfgPreEliminate.m:110).  Node-based plain aggregation:
// every level keeps Úa's dof layout [u; v] per system, a coarse node is an
// aggregate of fine nodes and coarse dof (c, I) gathers the c-components of
// its member nodes, so the prolongation P is piecewise constant per component
// and the Galerkin operator P' A P is a pure summation.  Smoother: one
// l1-Jacobi sweep (x += (b - A x) / sum_j |a_ij|) before and after the coarse
// correction, a symmetric V(1,1) cycle and so an SPD preconditioner for CG.
// Coarsest level: a dense inverse per system (at most 2*kAmgCoarseNodes dofs)
// applied as a matrix-vector product.
//
// The hierarchy of a system depends only on that system's mesh and every
// kernel works on per-system ranges in a fixed summation order, so a
// system's result is the same alone and in a batch.  Constrained dofs (the
// masked rows and columns of the projected system) have no coarse image:
// they are left out of the Galerkin sums, the restriction and the
// prolongation.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include <type_traits>
#include <cuda_bf16.h>
#include "ua_amg.h"

namespace ua {

constexpr int kAmgCoarseNodes = 48;   // a system stops coarsening at this many nodes
constexpr int kAmgMaxRow = 32;        // longest coarse dof row (2 x coarse node degree)
constexpr int kSaMaxDeg = 256;        // largest coarse node degree of a smoothed hierarchy (shared-memory rows)
constexpr int kAmgMaxDense = 2 * kAmgCoarseNodes;
constexpr int kAmgRB = 256;           // rows per row block of a coarse level
constexpr int kSaRB = 128, kSaLPR = 2;
constexpr int kAmgNB = 32;            // nodes per node block of the smoothed transfers (one warp's worth)  // smoothed hierarchies (longer coarse rows): rows per block, lanes per row

// Calls f(std::integral_constant<int, LPR>) for the lanes-per-row value lpr (1, 2, 4, 8, 16 or 32).
template <class F>
static void dispatch_lpr(int lpr, F&& f) {
  switch (lpr) {
    case 1: f(std::integral_constant<int, 1>()); break;
    case 2: f(std::integral_constant<int, 2>()); break;
    case 4: f(std::integral_constant<int, 4>()); break;
    case 16: f(std::integral_constant<int, 16>()); break;
    case 32: f(std::integral_constant<int, 32>()); break;
    default: f(std::integral_constant<int, 8>());
  }
}

struct AmgLevel {
  int nn = 0, ndof = 0;
  long long nnz = 0;
  int ap_maxrow = 0;  // longest A P row (coarse columns) of the level
  int ac_maxdeg = 0;  // largest node degree of the next (coarse) level
  std::vector<int> node_off, dof_off, knz_off, nnzn;  // per system (0-sized when the system has no such level)
  // dof-level CSR of a coarse level, same layout rule as the finest level
  int *rowptr = nullptr, *colind = nullptr;
  int* dof_sys = nullptr;
  int* d_dof_off = nullptr;               // per-system dof offsets on the device
  int* d_knz_off = nullptr;               // per-system non-zero offsets (uvh finest level)
  int *rb_start = nullptr, *rb_sys = nullptr;
  int nrb = 0;
  int* cmap = nullptr;                    // this level's dof -> next level's dof
  int *mptr = nullptr, *mlist = nullptr;  // per dof of this (coarse) level: member dofs of the finer level
  void* A = nullptr;                      // coarse values (KT)
  void* invd = nullptr;                   // l1-Jacobi inverse row sums (VT)
  void *b = nullptr, *x = nullptr, *x2 = nullptr;  // rhs, pre-smoothed, post-smoothed (VT)
  int* d_node_off = nullptr;              // per-system node offsets on the device
  int* node_sys = nullptr;                // node -> system (smoothed hierarchies)
  std::vector<int> h_sys_rb_off;          // per-system prefix of the row blocks
  // node blocks (kAmgNB nodes, never straddling two systems) for the smoothed transfers
  int *nb_start = nullptr, *nb_sys = nullptr;
  int nnb = 0;
  std::vector<int> h_sys_nb_off;
  // smoothed aggregation, transfer from this level to the next (node-level lists, global ids):
  // pn: fine node -> coarse nodes of its neighbours' aggregates (the prolongator's node pattern);
  // apn: fine node -> coarse nodes of A P; ptn: coarse node -> (fine node, position in pn)
  int *sa_agg = nullptr, *pn_ptr = nullptr, *pn_col = nullptr, *apn_ptr = nullptr, *apn_col = nullptr;
  int *ptn_ptr = nullptr, *ptn_fine = nullptr, *ptn_k = nullptr;
  int *pbase = nullptr, *pnnz = nullptr, *poff = nullptr, *apbase = nullptr, *apnnz = nullptr, *apoff = nullptr;
  double *sa_p = nullptr, *sa_ap = nullptr;  // set-up values (FP64 form): 4 per node-level entry
  float* sa_plo = nullptr;                   // set-up values of P (mixed form)
  // P in the transfer layout, one quad per node-level entry: pn order (sa_q*) and ptn order
  // (sa_qt*); BF16 quads for the mixed form, FP64 quads for the FP64 form (allocated on first use)
  long long np = 0;  // node-level prolongator entries of the level (all systems)
  void *sa_qh = nullptr, *sa_qth = nullptr, *sa_qd = nullptr, *sa_qtd = nullptr;
};

// one active-block list to compact: blocks blk_off[s] .. blk_off[s+1] of every system s with
// sel, !done and depth > lmin, in ascending order
struct ActSpec {
  const int* blk_off;
  int lmin;
  int* map;
  int* cnt;
};

// Finest-level node slices of a uv handle (sliced ELL over nodes).  A slice block is the set of
// nodes of one u-row block of the handle's Krylov rows (at most kSellNodes nodes of one system);
// inside it the nodes are ordered by decreasing degree and cut into slices of 32, one warp each.
// Slice j holds width W_j = its largest degree; its slots are 32 * W_j, entry k of lane t at slot
// off_j + 32 k + t.  Per slot: the u column (global u dof of the k-th neighbour; v column = u column
// + the system's node count) and four values (blocks uu, uv, vu, vv at value offsets
// 4 off_j + b 32 W_j + 32 k + t).  Padding slots hold zeros and the node's own column.  One column
// index then serves four values, and a warp's loads of one k are contiguous.
constexpr int kSellNodes = 256;  // nodes per slice block (= rows per row block)
constexpr int kSellSlices = kSellNodes / 32;

struct Sell {
  bool ready = false, failed = false;
  int nsb = 0;
  long long slots = 0;
  std::vector<int> h_sys_sb_off;  // per-system prefix of the slice blocks
  int *sb_sys = nullptr, *sb_n0 = nullptr, *sb_cnt = nullptr, *sb_rbu = nullptr, *sb_rbv = nullptr;
  int* perm = nullptr;             // [nn_total]: per block, its global node ids in slice order
  long long* sl_off = nullptr;     // [nsb * kSellSlices + 1] slot offsets of the slices
  int* cols = nullptr;             // [slots]
  float* v32 = nullptr;            // [4 slots] FP32 values (mixed-precision PCG operator)
  double* v64 = nullptr;           // [4 slots] FP64 values
  __nv_bfloat16* vlo = nullptr;    // [4 slots] BF16 values (mixed-precision V-cycle)
  double* spart = nullptr;         // [nsb * kSellSlices] per-slice partials (p.q, r.z)
  int* sys_sl_off = nullptr;       // [nsys + 1] per-system slice prefix
  ActList act;                     // slice blocks of the systems still iterating
};

struct Amg {
  int nsys = 0, nlev = 0, maxdn = 0;
  Sell sell;
  // node slices of the coarse levels 1 .. nlev-2 (smoothed hierarchies): BF16 copies of the
  // coarse operators for the mixed-precision V-cycle's residual and smoothing there
  std::vector<Sell> csell;
  // active-block lists: rows[l] (level-l row blocks, depth > l; level 0 = the handle's blocks),
  // fnodes[l] (level-l node blocks, depth > l), cnodes[l] (level-(l+1) node blocks, depth > l)
  bool act_ready = false;
  int nsm = 148;
  std::vector<ActList> rows, fnodes, cnodes;
  ActSpec* d_specs = nullptr;
  int nspecs = 0;
  bool sa = false;            // smoothed aggregation (else plain)
  std::vector<AmgLevel> lev;  // lev[0] = the handle's own system
  std::vector<int> depth;     // per system: its coarsest level (>= 1)
  std::vector<int> h_dn, h_doff;
  int *d_depth = nullptr, *d_dn = nullptr, *d_doff = nullptr;
  double* dense = nullptr;    // per system dn x dn inverse (row-major)
  void **d_lev_b = nullptr, **d_lev_x2 = nullptr, **d_lev_A = nullptr;
  int **d_lev_rowptr = nullptr, **d_lev_colind = nullptr, **d_lev_dofoff = nullptr;
  size_t bytes = 0;
  __nv_bfloat16* k0lo = nullptr;  // mixed precision: BF16 copy of the finest-level tangent
  // uvh handles: constraint mask and vectors of the velocity rows (2-dof layout)
  unsigned char* uvh_mask = nullptr;
  double *uvh_r = nullptr, *uvh_x0 = nullptr, *uvh_z = nullptr, *uvh_t = nullptr;
  // per system: numeric set-ups since its solve started (prolongator refresh), and the systems
  // whose prolongators the current set-up recomputes
  std::vector<int> p_age, h_prefresh;
  int* d_prefresh = nullptr;
  // the numeric set-up of a Newton step captured as one CUDA graph per (precision, selection
  // kind) and replayed: every argument is a fixed device buffer of the handle
  cudaGraphExec_t setup_exec[8] = {};
  long long setup_nodes[8] = {};
  ~Amg() {
    for (auto& e : setup_exec)
      if (e) cudaGraphExecDestroy(e);
  }
};

// ---------------------------------------------------------------------------
// host: aggregation and hierarchy
// ---------------------------------------------------------------------------

// Greedy aggregation of a node graph (system-local ids, self included):
// (1) a node whose neighbourhood is entirely unassigned becomes the root of
// an aggregate of that neighbourhood; (2) an unassigned node joins the
// aggregate of its first assigned neighbour; (3) what is left forms
// aggregates with its unassigned neighbours.
static int aggregate(int n, const std::vector<int>& ptr, const std::vector<int>& col, std::vector<int>& agg) {
  agg.assign(n, -1);
  int na = 0;
  for (int i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    bool free_nb = true;
    for (int k = ptr[i]; k < ptr[i + 1] && free_nb; ++k) free_nb = agg[col[k]] < 0;
    if (!free_nb) continue;
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) agg[col[k]] = na;
    ++na;
  }
  for (int i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    for (int k = ptr[i]; k < ptr[i + 1]; ++k)
      if (agg[col[k]] >= 0) { agg[i] = agg[col[k]]; break; }
  }
  for (int i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    for (int k = ptr[i]; k < ptr[i + 1]; ++k)
      if (agg[col[k]] < 0) agg[col[k]] = na;
    agg[i] = na++;
  }
  return na;
}

template <class T>
static T* upload(ua_mesh* m, Amg* a, const std::vector<T>& v, bool& ok) {
  T* d = (T*)dev_alloc(m, std::max<size_t>(1, v.size()) * sizeof(T));
  if (!d) { ok = false; return nullptr; }
  if (!v.empty() && cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) ok = false;
  a->bytes += v.size() * sizeof(T);
  return d;
}

static void* dalloc(ua_mesh* m, Amg* a, size_t bytes, bool& ok) {
  void* d = dev_alloc(m, std::max<size_t>(bytes, 16));
  if (!d) ok = false;
  a->bytes += bytes;
  return d;
}

// Dof-level CSR of a level from its node graph (global ids of the level):
// row (c, I) holds 2 blocks of deg(I) columns (block b, k-th neighbour).
static void level_csr(AmgLevel& L, const std::vector<int>& gptr, const std::vector<int>& gcol, int nsys,
                      std::vector<int>& rowptr, std::vector<int>& colind, std::vector<int>& dof_sys) {
  const std::vector<int>& no = L.node_off;
  L.dof_off.assign(nsys + 1, 0);
  L.knz_off.assign(nsys + 1, 0);
  L.nnzn.assign(nsys, 0);
  for (int s = 0; s < nsys; ++s) {
    const int n = no[s + 1] - no[s];
    L.dof_off[s + 1] = L.dof_off[s] + 2 * n;
    L.nnzn[s] = gptr[no[s + 1]] - gptr[no[s]];
    L.knz_off[s + 1] = L.knz_off[s] + 4 * L.nnzn[s];
  }
  const int N = L.dof_off[nsys];
  rowptr.assign(N + 1, 0);
  colind.assign(L.knz_off[nsys], 0);
  dof_sys.assign(N, 0);
  for (int s = 0; s < nsys; ++s) {
    const int n0 = no[s], n = no[s + 1] - n0, base = gptr[n0];
    for (int I = n0; I < n0 + n; ++I) {
      const int p0 = gptr[I], deg = gptr[I + 1] - p0;
      for (int c = 0; c < 2; ++c) {
        const int dof = L.dof_off[s] + c * n + (I - n0);
        const int start = L.knz_off[s] + c * 2 * L.nnzn[s] + 2 * (p0 - base);
        rowptr[dof] = start;
        dof_sys[dof] = s;
        for (int b = 0; b < 2; ++b)
          for (int k = 0; k < deg; ++k) colind[start + b * deg + k] = L.dof_off[s] + b * n + (gcol[p0 + k] - n0);
      }
    }
  }
  rowptr[N] = L.knz_off[nsys];
  L.nn = no[nsys];
  L.ndof = N;
  L.nnz = L.knz_off[nsys];
}

static int amg_build(ua_mesh* m, bool smoothed) {
  const int nsys = m->dm.nsys;
  Amg* a = new Amg();
  a->nsys = nsys;
  a->depth.assign(nsys, 0);
  // node graphs per level (global ids of the level)
  std::vector<std::vector<int>> g_off{m->h_node_off}, g_ptr{m->h_nodeptr}, g_col{m->h_nodecol}, g_agg;
  // smoothed aggregation lists per transfer (index = fine level)
  std::vector<std::vector<int>> g_pnp, g_pnc, g_apnp, g_apnc, g_ptnp, g_ptnf, g_ptnk;
  a->sa = smoothed;
  std::vector<char> live(nsys, 1);
  auto fail = [&](const char* why) {
    delete a;
    return set_error(UA_ERR_INVALID, "AMG setup: %s", why);
  };
  while (std::find(live.begin(), live.end(), 1) != live.end()) {
    const std::vector<int>& no = g_off.back();
    const std::vector<int>& fp = g_ptr.back();
    const std::vector<int>& fc = g_col.back();
    std::vector<int> agg(no[nsys], -1), cno(nsys + 1, 0), cptr(1, 0), ccol;
    std::vector<int> pnp(1, 0), pnc, apnp(1, 0), apnc, ptnp(1, 0), ptnf, ptnk;
    for (int s = 0; s < nsys; ++s) {
      const int n = no[s + 1] - no[s];
      if (!live[s] || n == 0) {
        cno[s + 1] = cno[s];
        for (int i = 0; i < n; ++i) { pnp.push_back((int)pnc.size()); apnp.push_back((int)apnc.size()); }
        continue;
      }
      std::vector<int> lp(n + 1, 0), lc, la;
      for (int i = 0; i < n; ++i) {
        for (int k = fp[no[s] + i]; k < fp[no[s] + i + 1]; ++k) lc.push_back(fc[k] - no[s]);
        lp[i + 1] = (int)lc.size();
      }
      const int na = aggregate(n, lp, lc, la);
      for (int i = 0; i < n; ++i) agg[no[s] + i] = cno[s] + la[i];
      cno[s + 1] = cno[s] + na;
      std::vector<std::vector<int>> adj(na);
      if (!smoothed) {
        for (int i = 0; i < n; ++i)
          for (int k = lp[i]; k < lp[i + 1]; ++k) adj[la[i]].push_back(la[lc[k]]);
      } else {
        // prolongator pattern: node i reaches the aggregates of its neighbours (P = (I - w D^-1 A) P0)
        std::vector<int> lpn(n + 1, 0), lpc, stamp(na, -1);
        for (int i = 0; i < n; ++i) {
          const size_t b0 = lpc.size();
          for (int k = lp[i]; k < lp[i + 1]; ++k) {
            const int J = la[lc[k]];
            if (stamp[J] != i) { stamp[J] = i; lpc.push_back(J); }
          }
          std::sort(lpc.begin() + b0, lpc.end());
          lpn[i + 1] = (int)lpc.size();
        }
        // A P pattern: node i reaches the union of its neighbours' prolongator rows
        std::vector<int> lapn(n + 1, 0), lapc;
        std::fill(stamp.begin(), stamp.end(), -1);
        for (int i = 0; i < n; ++i) {
          const size_t b0 = lapc.size();
          for (int k = lp[i]; k < lp[i + 1]; ++k) {
            const int h = lc[k];
            for (int t = lpn[h]; t < lpn[h + 1]; ++t)
              if (stamp[lpc[t]] != i) { stamp[lpc[t]] = i; lapc.push_back(lpc[t]); }
          }
          std::sort(lapc.begin() + b0, lapc.end());
          lapn[i + 1] = (int)lapc.size();
        }
        // transpose of the prolongator pattern, with each entry's position in its fine row
        std::vector<int> ltp(na + 1, 0), ltf(lpc.size()), ltk(lpc.size());
        for (int t = 0; t < (int)lpc.size(); ++t) ltp[lpc[t] + 1]++;
        for (int J = 0; J < na; ++J) ltp[J + 1] += ltp[J];
        {
          std::vector<int> nx(ltp.begin(), ltp.end() - 1);
          for (int i = 0; i < n; ++i)
            for (int t = lpn[i]; t < lpn[i + 1]; ++t) { ltf[nx[lpc[t]]] = i; ltk[nx[lpc[t]]++] = t - lpn[i]; }
        }
        // coarse node graph of P' A P
        std::fill(stamp.begin(), stamp.end(), -1);
        for (int I = 0; I < na; ++I)
          for (int u = ltp[I]; u < ltp[I + 1]; ++u) {
            const int i = ltf[u];
            for (int t = lapn[i]; t < lapn[i + 1]; ++t)
              if (stamp[lapc[t]] != I) { stamp[lapc[t]] = I; adj[I].push_back(lapc[t]); }
          }
        for (int i = 0; i < n; ++i) {
          for (int t = lpn[i]; t < lpn[i + 1]; ++t) pnc.push_back(cno[s] + lpc[t]);
          pnp.push_back((int)pnc.size());
          for (int t = lapn[i]; t < lapn[i + 1]; ++t) apnc.push_back(cno[s] + lapc[t]);
          apnp.push_back((int)apnc.size());
        }
        for (int J = 0; J < na; ++J) {
          for (int u = ltp[J]; u < ltp[J + 1]; ++u) { ptnf.push_back(no[s] + ltf[u]); ptnk.push_back(ltk[u]); }
          ptnp.push_back((int)ptnf.size());
        }
      }
      for (int I = 0; I < na; ++I) {
        std::sort(adj[I].begin(), adj[I].end());
        adj[I].erase(std::unique(adj[I].begin(), adj[I].end()), adj[I].end());
        if (!smoothed && 2 * (int)adj[I].size() > kAmgMaxRow) return fail("coarse node degree above the row limit");
        if (smoothed && (int)adj[I].size() > kSaMaxDeg) return fail("smoothed coarse node degree above the limit");
        for (int J : adj[I]) ccol.push_back(cno[s] + J);
        cptr.push_back((int)ccol.size());
      }
      a->depth[s]++;
      if (na <= kAmgCoarseNodes) live[s] = 0;
      else if (na >= n) return fail("aggregation made no progress");
    }
    g_agg.push_back(agg);
    g_off.push_back(cno);
    g_ptr.push_back(cptr);
    g_col.push_back(ccol);
    g_pnp.push_back(pnp); g_pnc.push_back(pnc); g_apnp.push_back(apnp); g_apnc.push_back(apnc);
    g_ptnp.push_back(ptnp); g_ptnf.push_back(ptnf); g_ptnk.push_back(ptnk);
  }
  a->nlev = (int)g_off.size();
  a->lev.resize(a->nlev);
  bool ok = true;
  for (int l = 0; l < a->nlev; ++l) {
    AmgLevel& L = a->lev[l];
    L.node_off = g_off[l];
    std::vector<int> rowptr, colind, dof_sys;
    level_csr(L, g_ptr[l], g_col[l], nsys, rowptr, colind, dof_sys);
    if (l == 0 && m->ndof == 2 && (L.ndof != m->ndof_total || L.nnz != m->nnz_total))
      return fail("fine level does not match the handle");
    std::vector<int> rb_start, rb_sys;
    L.h_sys_rb_off.assign(nsys + 1, 0);
    for (int s = 0; s < nsys; ++s) {
      for (int r = L.dof_off[s]; r < L.dof_off[s + 1]; r += smoothed ? kSaRB : kAmgRB) {
        rb_start.push_back(r);
        rb_sys.push_back(s);
      }
      L.h_sys_rb_off[s + 1] = (int)rb_sys.size();
    }
    rb_start.push_back(L.ndof);
    L.nrb = (int)rb_sys.size();
    L.invd = dalloc(m, a, sizeof(double) * (size_t)L.ndof, ok);
    if (l == 0 && m->ndof == 3) {
      // uvh handle: the finest level is the velocity block, held apart from the 3-dof
      // tangent (values extracted per Newton step), with its own rows and vectors
      L.rb_start = upload(m, a, rb_start, ok);
      L.rb_sys = upload(m, a, rb_sys, ok);
      L.dof_sys = upload(m, a, dof_sys, ok);
      L.rowptr = upload(m, a, rowptr, ok);
      L.colind = upload(m, a, colind, ok);
      L.d_knz_off = upload(m, a, L.knz_off, ok);
      L.A = dalloc(m, a, sizeof(double) * (size_t)L.nnz, ok);
      a->uvh_mask = (unsigned char*)dalloc(m, a, (size_t)L.ndof, ok);
      for (double** v : {&a->uvh_r, &a->uvh_x0, &a->uvh_z, &a->uvh_t})
        *v = (double*)dalloc(m, a, sizeof(double) * (size_t)L.ndof, ok);
    }
    if (l > 0) {  // the fine level of a uv handle uses the handle's tangent structure and PCG vectors
      L.rb_start = upload(m, a, rb_start, ok);
      L.rb_sys = upload(m, a, rb_sys, ok);
      L.dof_sys = upload(m, a, dof_sys, ok);
      L.rowptr = upload(m, a, rowptr, ok);
      L.colind = upload(m, a, colind, ok);
      L.A = dalloc(m, a, sizeof(double) * (size_t)L.nnz, ok);
      L.b = dalloc(m, a, sizeof(double) * (size_t)L.ndof, ok);
      L.x = dalloc(m, a, sizeof(double) * (size_t)L.ndof, ok);
      L.x2 = dalloc(m, a, sizeof(double) * (size_t)L.ndof, ok);
      // coarse dof (c, I) gathers fine dofs (c, i) with agg[i] = I, in ascending order
      AmgLevel& F = a->lev[l - 1];
      const std::vector<int>& agg = g_agg[l - 1];
      std::vector<int> cmap(F.ndof, -1), cnt(L.ndof + 1, 0), mlist(F.ndof);
      for (int s = 0; s < nsys; ++s) {
        const int fno = F.node_off[s], fn = F.node_off[s + 1] - fno;
        const int cno = L.node_off[s], cn = L.node_off[s + 1] - cno;
        if (cn == 0) continue;
        for (int c = 0; c < 2; ++c)
          for (int i = 0; i < fn; ++i)
            cmap[F.dof_off[s] + c * fn + i] = L.dof_off[s] + c * cn + (agg[fno + i] - cno);
      }
      for (int d = 0; d < F.ndof; ++d)
        if (cmap[d] >= 0) cnt[cmap[d] + 1]++;
      for (int d = 0; d < L.ndof; ++d) cnt[d + 1] += cnt[d];
      std::vector<int> mptr = cnt;
      for (int d = 0; d < F.ndof; ++d)
        if (cmap[d] >= 0) mlist[cnt[cmap[d]]++] = d;
      mlist.resize(mptr[L.ndof]);
      F.cmap = upload(m, a, cmap, ok);
      L.mptr = upload(m, a, mptr, ok);
      L.mlist = upload(m, a, mlist, ok);
    }
  }
  a->h_dn.assign(nsys, 0);
  a->h_doff.assign(nsys + 1, 0);
  for (int s = 0; s < nsys; ++s) {
    const AmgLevel& L = a->lev[a->depth[s]];
    a->h_dn[s] = L.dof_off[s + 1] - L.dof_off[s];
    if (a->h_dn[s] > kAmgMaxDense) return fail("coarsest system above the dense limit");
    a->maxdn = std::max(a->maxdn, a->h_dn[s]);
    a->h_doff[s + 1] = a->h_doff[s] + a->h_dn[s] * a->h_dn[s];
  }
  a->dense = (double*)dalloc(m, a, sizeof(double) * (size_t)a->h_doff[nsys], ok);
  a->d_depth = upload(m, a, a->depth, ok);
  a->d_dn = upload(m, a, a->h_dn, ok);
  a->d_doff = upload(m, a, a->h_doff, ok);
  std::vector<void*> pb(a->nlev), px2(a->nlev), pA(a->nlev);
  std::vector<int*> prp(a->nlev), pci(a->nlev), pdo(a->nlev);
  for (int l = 0; l < a->nlev; ++l) {
    a->lev[l].d_node_off = upload(m, a, a->lev[l].node_off, ok);
    if (a->sa) {
      std::vector<int> ns(std::max(a->lev[l].node_off[nsys], 1), 0);
      for (int s = 0; s < nsys; ++s)
        for (int g = a->lev[l].node_off[s]; g < a->lev[l].node_off[s + 1]; ++g) ns[g] = s;
      a->lev[l].node_sys = upload(m, a, ns, ok);
      std::vector<int> nbs, nbsys;
      AmgLevel& L = a->lev[l];
      L.h_sys_nb_off.assign(nsys + 1, 0);
      for (int s = 0; s < nsys; ++s) {
        for (int g = L.node_off[s]; g < L.node_off[s + 1]; g += kAmgNB) {
          nbs.push_back(g);
          nbsys.push_back(s);
        }
        L.h_sys_nb_off[s + 1] = (int)nbsys.size();
      }
      nbs.push_back(L.node_off[nsys]);
      L.nnb = (int)nbsys.size();
      L.nb_start = upload(m, a, nbs, ok);
      L.nb_sys = upload(m, a, nbsys, ok);
    }
    if (!a->lev[l].dof_sys) {  // a uv handle's finest level: rows -> system, for the smoothed transfer
      std::vector<int> ds(a->lev[l].ndof);
      for (int s = 0; s < nsys; ++s)
        for (int d = a->lev[l].dof_off[s]; d < a->lev[l].dof_off[s + 1]; ++d) ds[d] = s;
      a->lev[l].dof_sys = upload(m, a, ds, ok);
    }
    if (a->sa && l + 1 < a->nlev) {
      AmgLevel& F = a->lev[l];
      const AmgLevel& C = a->lev[l + 1];
      F.sa_agg = upload(m, a, g_agg[l], ok);
      F.pn_ptr = upload(m, a, g_pnp[l], ok);
      F.pn_col = upload(m, a, g_pnc[l], ok);
      F.apn_ptr = upload(m, a, g_apnp[l], ok);
      F.apn_col = upload(m, a, g_apnc[l], ok);
      F.ptn_ptr = upload(m, a, g_ptnp[l], ok);
      F.ptn_fine = upload(m, a, g_ptnf[l], ok);
      F.ptn_k = upload(m, a, g_ptnk[l], ok);
      std::vector<int> pbase(nsys), pnnz(nsys), poff(nsys + 1, 0), apbase(nsys), apnnz(nsys), apoff(nsys + 1, 0);
      for (int s = 0; s < nsys; ++s) {
        pbase[s] = g_pnp[l][F.node_off[s]];
        pnnz[s] = g_pnp[l][F.node_off[s + 1]] - pbase[s];
        poff[s + 1] = poff[s] + 4 * pnnz[s];
        apbase[s] = g_apnp[l][F.node_off[s]];
        apnnz[s] = g_apnp[l][F.node_off[s + 1]] - apbase[s];
        apoff[s + 1] = apoff[s] + 4 * apnnz[s];
      }
      F.pbase = upload(m, a, pbase, ok); F.pnnz = upload(m, a, pnnz, ok); F.poff = upload(m, a, poff, ok);
      F.apbase = upload(m, a, apbase, ok); F.apnnz = upload(m, a, apnnz, ok); F.apoff = upload(m, a, apoff, ok);
      F.ap_maxrow = 0;
      for (size_t i = 0; i + 1 < g_apnp[l].size(); ++i)
        F.ap_maxrow = std::max(F.ap_maxrow, g_apnp[l][i + 1] - g_apnp[l][i]);
      F.ac_maxdeg = 0;
      for (size_t I = 0; I + 1 < g_ptr[l + 1].size(); ++I)
        F.ac_maxdeg = std::max(F.ac_maxdeg, g_ptr[l + 1][I + 1] - g_ptr[l + 1][I]);
      F.sa_p = (double*)dalloc(m, a, sizeof(double) * (size_t)poff[nsys], ok);
      F.np = g_pnp[l].back();
      F.sa_ap = (double*)dalloc(m, a, sizeof(double) * (size_t)apoff[nsys], ok);
      F.sa_plo = (float*)dalloc(m, a, sizeof(float) * (size_t)poff[nsys], ok);
    }
    pb[l] = a->lev[l].b;
    px2[l] = a->lev[l].x2;
    pA[l] = a->lev[l].A;
    prp[l] = a->lev[l].rowptr;
    pci[l] = a->lev[l].colind;
    pdo[l] = upload(m, a, a->lev[l].dof_off, ok);
    a->lev[l].d_dof_off = pdo[l];
  }
  a->d_lev_b = upload(m, a, pb, ok);
  a->d_lev_x2 = upload(m, a, px2, ok);
  a->d_lev_A = upload(m, a, pA, ok);
  a->d_lev_rowptr = upload(m, a, prp, ok);
  a->d_lev_colind = upload(m, a, pci, ok);
  a->d_lev_dofoff = upload(m, a, pdo, ok);
  if (!ok) {
    delete a;
    return set_error(UA_ERR_OOM, "AMG setup: device allocation failed");
  }
  m->amg = a;
  return UA_OK;
}

// smoothed aggregation first (when asked), plain aggregation if the smoothed hierarchy
// exceeds its limits; a shape neither can take keeps point Jacobi for the handle's life
int amg_setup(ua_mesh* m, bool smoothed) {
  if (m->amg) return UA_OK;
  if (m->amg_failed) return UA_ERR_INVALID;
  if (m->ndof != 2 && m->ndof != 3) return set_error(UA_ERR_INVALID, "the AMG preconditioner needs uv or uvh dofs");
  int rc = amg_build(m, smoothed);
  if (rc == UA_ERR_INVALID && smoothed) rc = amg_build(m, false);
  if (rc == UA_ERR_INVALID) m->amg_failed = true;
  return rc;
}

void amg_free(Amg* a) { delete a; }

int amg_levels(const ua_mesh* m) { return m->amg ? m->amg->nlev : 0; }

const void* amg_invd0(const ua_mesh* m) { return m->amg ? m->amg->lev[0].invd : nullptr; }

// ---------------------------------------------------------------------------
// device: numeric phase
// ---------------------------------------------------------------------------

// Galerkin product: coarse row R sums the unmasked entries of its member
// rows into the coarse columns cmap[j] (binary search in the sorted coarse row).
template <typename KT>
__global__ void k_amg_galerkin(int ncd, const int* mptr, const int* mlist, const int* frowptr, const int* fcolind,
                               const KT* fA, const int* cmap, const unsigned char* cmask, const int* crowptr,
                               const int* ccolind, KT* cA) {
  const int R = blockIdx.x * blockDim.x + threadIdx.x;
  if (R >= ncd) return;
  const int c0 = crowptr[R], len = crowptr[R + 1] - c0;
  double acc[kAmgMaxRow];
#pragma unroll
  for (int k = 0; k < kAmgMaxRow; ++k) acc[k] = 0;
  for (int t = mptr[R]; t < mptr[R + 1]; ++t) {
    const int i = mlist[t];
    if (cmask && cmask[i]) continue;
    for (int q = frowptr[i]; q < frowptr[i + 1]; ++q) {
      const int j = fcolind[q];
      if (cmask && cmask[j]) continue;
      const int C = cmap[j];
      int lo = 0, hi = len - 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ccolind[c0 + mid] < C) lo = mid + 1; else hi = mid;
      }
      acc[lo] += (double)fA[q];
    }
  }
  for (int k = 0; k < len; ++k) cA[c0 + k] = (KT)acc[k];
}

// l1-Jacobi: invd_i = 1 / sum_j |a_ij| over unmasked columns (0 on masked or empty rows)
template <typename KT, typename VT>
__global__ void k_amg_l1(int n, const int* rowptr, const int* colind, const KT* A, const unsigned char* cmask,
                         VT* invd, const int* dof_sys, const int* sel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (sel && !sel[dof_sys[i]]) return;  // systems not in this Newton step keep their values
  double s = 0;
  if (!(cmask && cmask[i]))
    for (int q = rowptr[i]; q < rowptr[i + 1]; ++q)
      if (!(cmask && cmask[colind[q]])) s += fabs((double)A[q]);
  invd[i] = (VT)(s > 0 ? 1.0 / s : 0.0);
}

// Inverse of each system's coarsest matrix: Gauss-Jordan on [A | I] in
// shared memory, one CTA per system, row-major result.  A is the Galerkin
// product of the SPD tangent (symmetric positive definite on the free dofs),
// so the diagonal pivots stay positive and no pivoting is needed.  At step k
// only columns k..n+k of the augmented matrix can be non-zero off the
// finished part, so the update covers those n+1 columns.  A zero row (an
// aggregate of constrained dofs only; its column is zero too) is replaced by
// the identity row.
template <typename KT>
__global__ void __launch_bounds__(256) k_amg_dense_inverse(const int* depth, const int* dn_arr, const int* doff,
                                                           int* const* lev_rowptr, int* const* lev_colind,
                                                           void* const* lev_A, int* const* lev_dofoff,
                                                           double* dense, const int* sel) {
  extern __shared__ double M[];
  __shared__ double fac[kAmgMaxDense];
  const int s = blockIdx.x;
  const int n = dn_arr[s];
  if (n == 0 || (sel && !sel[s])) return;
  const int l = depth[s];
  const int* rp = lev_rowptr[l];
  const int* ci = lev_colind[l];
  const KT* A = (const KT*)lev_A[l];
  const int d0 = lev_dofoff[l][s];
  const int w = 2 * n;
  for (int t = threadIdx.x; t < n * w; t += blockDim.x) M[t] = ((t % w) - n == t / w) ? 1.0 : 0.0;
  __syncthreads();
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    bool zero = true;
    for (int q = rp[d0 + r]; q < rp[d0 + r + 1]; ++q) {
      const double v = (double)A[q];
      M[r * w + (ci[q] - d0)] = v;
      zero = zero && v == 0.0;
    }
    if (zero) M[r * w + r] = 1.0;
  }
  __syncthreads();
  const int nc = n + 1;  // active columns k..n+k
  for (int k = 0; k < n; ++k) {
    const double inv = 1.0 / M[k * w + k];
    for (int r = threadIdx.x; r < n; r += blockDim.x) fac[r] = (r == k) ? 0.0 : M[r * w + k];
    __syncthreads();
    for (int c = k + threadIdx.x; c <= n + k; c += blockDim.x) M[k * w + c] *= inv;
    __syncthreads();
    for (int t = threadIdx.x; t < n * nc; t += blockDim.x) {
      const int r = t / nc, c = k + (t - r * nc);
      if (r != k) M[r * w + c] -= fac[r] * M[k * w + c];
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) dense[doff[s] + t] = M[(t / n) * w + n + (t % n)];
}

// ---------------------------------------------------------------------------
// device: V-cycle
// ---------------------------------------------------------------------------

// x2 = inv(A_L) b on each system's coarsest level L: grid (system, 32-row
// slab), one warp per row with the lanes over the columns (row-major inverse,
// coalesced), b staged in shared memory.
template <typename VT>
__global__ void __launch_bounds__(256) k_amg_dense_apply(const int* sel, const int* done, const int* depth,
                                                         const int* dn_arr, const int* doff, int* const* lev_dofoff,
                                                         void* const* lev_b, void* const* lev_x2,
                                                         const double* dense) {
  pdl_enter();
  __shared__ double sb[kAmgMaxDense];
  const int s = blockIdx.x;
  if (!sel[s] || done[s]) return;
  const int n = dn_arr[s], r0 = blockIdx.y * 32;
  if (r0 >= n) return;
  const int l = depth[s];
  const int d0 = lev_dofoff[l][s];
  const VT* b = (const VT*)lev_b[l] + d0;
  VT* x = (VT*)lev_x2[l] + d0;
  for (int c = threadIdx.x; c < n; c += blockDim.x) sb[c] = (double)b[c];
  __syncthreads();
  const double* Mi = dense + doff[s];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int r1 = min(r0 + 32, n);
  for (int r = r0 + warp; r < r1; r += nw) {  // warp-uniform
    double acc = 0;
    for (int c = lane; c < n; c += 32) acc += Mi[r * n + c] * sb[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) x[r] = (VT)acc;
  }
}

// Split V-cycle kernels (every level; coalesced row blocks with LPR lanes per
// row instead of one thread per aggregate).  Residual of the pre-smoothed
// vector of level l: res = mask(b - A x), for systems deeper than l.
// Row product in the uv block layout of every level: row (c, I) holds the u
// block then the v block of deg(I) entries on the same node columns, v column
// = u column + nhalf, so only the u block's indices are read (used for FP64
// values, where it is faster).
template <typename KT, typename XT, int LPR>
__device__ __forceinline__ double row_dot_uv(const int* rowptr, const int* colind, const KT* A, const XT* x, int row,
                                             bool valid, int lane, int nhalf) {
  double acc = 0;
  if (valid) {
    const int r0 = rowptr[row], deg = (rowptr[row + 1] - r0) >> 1;
    for (int k = lane; k < deg; k += LPR) {
      const int j = colind[r0 + k];
      acc += (double)A[r0 + k] * (double)x[j] + (double)A[r0 + deg + k] * (double)x[j + nhalf];
    }
  }
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, LPR);
  return acc;
}

__device__ __forceinline__ double to_d(double v) { return v; }
__device__ __forceinline__ double to_d(float v) { return (double)v; }
__device__ __forceinline__ double to_d(__nv_bfloat16 v) { return (double)__bfloat162float(v); }

// Plain CSR row product (every index read); the form that is faster for FP32 and BF16 values.
template <typename KT, typename XT, int LPR>
__device__ __forceinline__ double row_dot_csr(const int* rowptr, const int* colind, const KT* A, const XT* x, int row,
                                              bool valid, int lane) {
  double acc = 0;
  if (valid)
    for (int q = rowptr[row] + lane; q < rowptr[row + 1]; q += LPR) acc += to_d(A[q]) * (double)x[colind[q]];
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, LPR);
  return acc;
}

// BF16 copy of an FP32 tangent (the finest-level matrix of the mixed-precision
// V-cycle's residual and smoothing passes)
__global__ void k_to_bf16(long long n, const float* in, __nv_bfloat16* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

template <typename KT, typename VT, int LPR>
__global__ void __launch_bounds__(256) k_amg_residual(const int* rb_start, const int* rb_sys, ActList act,
                                                      const int* sel, const int* done, const int* depth, int l,
                                                      const int* rowptr, const int* colind, const KT* A,
                                                      const VT* b, const VT* x, const unsigned char* cmask, VT* res,
                                                      const int* dof_off) {
  pdl_enter();
  const int nv = act.cnt ? *act.cnt : gridDim.x;  // list entries, else one block per CTA
  for (int vb = blockIdx.x; vb < nv; vb += gridDim.x) {
    const int blk = act.map ? act.map[vb] : vb;
    const int s = rb_sys[blk];
    if (!sel[s] || done[s] || depth[s] <= l) continue;  // uniform over the block
    const int rs = rb_start[blk], re = rb_start[blk + 1];
    const int nhalf = (dof_off[s + 1] - dof_off[s]) >> 1;
    const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR, ngrp = blockDim.x / LPR;
    for (int row0 = rs; row0 < re; row0 += ngrp) {  // same trip count for every thread of the block
      const int row = row0 + grp;
      const bool valid = row < re;
      const double ax = sizeof(KT) == 8 ? row_dot_uv<KT, VT, LPR>(rowptr, colind, A, x, row, valid, lane, nhalf)
                                        : row_dot_csr<KT, VT, LPR>(rowptr, colind, A, x, row, valid, lane);
      if (valid && lane == 0) res[row] = (VT)((cmask && cmask[row]) ? 0.0 : (double)b[row] - ax);
    }
  }
}

// Aggregation of a fine vector: b(R) = sum over members (ascending) of res;
// coarse pre-smoothing x = invd b unless lc is the system's coarsest level.
template <typename VT>
__global__ void k_amg_gather(int ncd, const int* dof_sys_c, const int* depth, int lc, const int* sel,
                             const int* done, const int* mptr, const int* mlist, const VT* res, const VT* cinvd,
                             VT* cb, VT* cx) {
  const int R = blockIdx.x * blockDim.x + threadIdx.x;
  if (R >= ncd) return;
  const int s = dof_sys_c[R];
  if (!sel[s] || done[s]) return;
  double acc = 0;
  for (int t = mptr[R]; t < mptr[R + 1]; ++t) acc += (double)res[mlist[t]];
  cb[R] = (VT)acc;
  if (depth[s] > lc) cx[R] = (VT)((double)cinvd[R] * acc);
}

// Coarse correction of level l, in place: x = mask(x + xc[cmap]) for systems deeper than l.
template <typename VT>
__global__ void __launch_bounds__(256) k_amg_correct(const int* rb_start, const int* rb_sys, const int* sel,
                                                     const int* done, const int* depth, int l, VT* x,
                                                     const VT* xc, const int* cmap, const unsigned char* cmask) {
  const int blk = blockIdx.x;
  const int s = rb_sys[blk];
  if (!sel[s] || done[s] || depth[s] <= l) return;
  for (int i = rb_start[blk] + threadIdx.x; i < rb_start[blk + 1]; i += blockDim.x)
    x[i] = (cmask && cmask[i]) ? (VT)0 : (VT)((double)x[i] + (double)xc[cmap[i]]);
}

// Post-smoothing of level l: out = xp + invd (b - A xp) (0 on masked rows)
// for systems deeper than l; on the finest level pcopy (if set) receives a
// copy and part the block partials of b.out.
template <typename KT, typename VT, int LPR>
__global__ void __launch_bounds__(256) k_amg_smooth(const int* rb_start, const int* rb_sys, ActList act,
                                                    const int* sel, const int* done, const int* depth, int l,
                                                    const int* rowptr, const int* colind, const KT* A, const VT* b,
                                                    const VT* xp, const VT* invd, const unsigned char* cmask, VT* out,
                                                    VT* pcopy, double* part, const int* dof_off) {
  pdl_enter();
  __shared__ double red[8];
  const int nv = act.cnt ? *act.cnt : gridDim.x;  // list entries, else one block per CTA
  for (int vb = blockIdx.x; vb < nv; vb += gridDim.x) {
    const int blk = act.map ? act.map[vb] : vb;
    const int s = rb_sys[blk];
    double rz = 0;
    if (sel[s] && !done[s] && depth[s] > l) {
      const int rs = rb_start[blk], re = rb_start[blk + 1];
      const int nhalf = (dof_off[s + 1] - dof_off[s]) >> 1;
      const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR, ngrp = blockDim.x / LPR;
      for (int row0 = rs; row0 < re; row0 += ngrp) {  // same trip count for every thread of the block
        const int row = row0 + grp;
        const bool valid = row < re;
        const double ax = sizeof(KT) == 8 ? row_dot_uv<KT, VT, LPR>(rowptr, colind, A, xp, row, valid, lane, nhalf)
                                          : row_dot_csr<KT, VT, LPR>(rowptr, colind, A, xp, row, valid, lane);
        if (valid && lane == 0) {
          const double v =
              (cmask && cmask[row]) ? 0.0 : (double)xp[row] + (double)invd[row] * ((double)b[row] - ax);
          out[row] = (VT)v;
          if (pcopy) pcopy[row] = (VT)v;
          rz += (double)b[row] * v;
        }
      }
    }
    if (!part) continue;  // uniform per launch
    double t = rz;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double sum = 0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) sum += red[i];
      part[blk] = sum;
    }
    __syncthreads();  // red is rewritten by the next entry
  }
}

// ---------------------------------------------------------------------------
// device: finest-level node slices (both rows of a node per thread)
// ---------------------------------------------------------------------------

struct SellDev {
  const int *sb_sys, *sb_n0, *sb_cnt, *sb_rbu, *sb_rbv, *perm;
  const long long* sl_off;
  const int* cols;
  const int *dof_off, *node_off;  // per system, of the slices' level
  unsigned long long* dbg;        // first bounds violation (debug build)
  int lev;                        // the level (residual and smoothing: systems deeper than it)
};

// The four values of a slot (blocks uu, uv, vu, vv) are adjacent, so a lane reads them with one
// vector load: 8 bytes (BF16), 16 (FP32) or 32 (FP64, two loads).
template <typename KT> struct Quad;
template <> struct Quad<float> {
  static __device__ __forceinline__ void get(const float* p, double (&e)[4]) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(p));
    e[0] = q.x; e[1] = q.y; e[2] = q.z; e[3] = q.w;
  }
};
template <> struct Quad<double> {
  static __device__ __forceinline__ void get(const double* p, double (&e)[4]) {
    const double2 q0 = __ldg(reinterpret_cast<const double2*>(p)), q1 = __ldg(reinterpret_cast<const double2*>(p) + 1);
    e[0] = q0.x; e[1] = q0.y; e[2] = q1.x; e[3] = q1.y;
  }
};
template <> struct Quad<__nv_bfloat16> {
  static __device__ __forceinline__ void get(const __nv_bfloat16* p, double (&e)[4]) {
    const uint2 q = __ldg(reinterpret_cast<const uint2*>(p));
    // a BF16 value is the upper half of the FP32 value with the same bits
    e[0] = __uint_as_float(q.x << 16); e[1] = __uint_as_float(q.x & 0xffff0000u);
    e[2] = __uint_as_float(q.y << 16); e[3] = __uint_as_float(q.y & 0xffff0000u);
  }
};

// Slice values (and, once per handle, the columns) from the tangent's CSR layout: row (c, g)
// starts at knz_off[s] + 2 c nnzn[s] + 2 lp(g) and holds the u block then the v block of deg(g)
// entries.  One CTA per slice block, one warp per slice, one lane per node; writes are contiguous.
template <typename KT>
__global__ void __launch_bounds__(256) k_sell_fill(SellDev S, const DevMesh dm, const KT* K, KT* vk,
                                                   __nv_bfloat16* vlo, int* cols, const int* sel) {
  const int sb = blockIdx.x;
  const int w = threadIdx.x >> 5, t = threadIdx.x & 31, pos = w * 32 + t;
  const int sl = sb * kSellSlices + w;
  const long long o0 = S.sl_off[sl];
  const int W = (int)((S.sl_off[sl + 1] - o0) >> 5);
  if (W == 0) return;  // empty slice (warp-uniform)
  const int s = S.sb_sys[sb];
  if (sel && K && !sel[s]) return;  // values of the systems of this Newton step only
  const int no = dm.sys_node_off[s], d0 = dm.sys_dof_off[s];
  const bool has = pos < S.sb_cnt[sb];
  int g = no, np0 = 0, deg = 0;
  if (has) {
    g = S.perm[S.sb_n0[sb] + pos];
    np0 = dm.nodeptr[g];
    deg = dm.nodeptr[g + 1] - np0;
  }
  const long long lp = (long long)np0 - dm.nodeptr[no];
  const long long bu = (long long)dm.sys_knz_off[s] + 2 * lp, bv = bu + 2LL * dm.sys_nnzn[s];
  for (int k = 0; k < W; ++k) {
    const bool in = has && k < deg;
    const long long d = o0 + 32LL * k + t;
    if (cols) cols[d] = d0 + (in ? dm.nodecol[np0 + k] : g) - no;
    if (!K) continue;
    KT e0 = 0, e1 = 0, e2 = 0, e3 = 0;
    if (in) { e0 = K[bu + k]; e1 = K[bu + deg + k]; e2 = K[bv + k]; e3 = K[bv + deg + k]; }
    if (vk) { vk[4 * d] = e0; vk[4 * d + 1] = e1; vk[4 * d + 2] = e2; vk[4 * d + 3] = e3; }
    if (vlo) {
      vlo[4 * d] = __float2bfloat16_rn((float)e0); vlo[4 * d + 1] = __float2bfloat16_rn((float)e1);
      vlo[4 * d + 2] = __float2bfloat16_rn((float)e2); vlo[4 * d + 3] = __float2bfloat16_rn((float)e3);
    }
  }
}

// Coarse-level slice values (and, once, the columns) from the level's CSR: row (c, I) holds the
// u block then the v block of deg(I) entries.  Same slice layout as the finest level.
template <typename KT>
__global__ void __launch_bounds__(256) k_csell_fill(SellDev S, const int* rowptr, const int* colind, const KT* A,
                                                    __nv_bfloat16* vlo, int* cols, const int* sel) {
  const int sb = blockIdx.x;
  const int w = threadIdx.x >> 5, t = threadIdx.x & 31, pos = w * 32 + t;
  const int sl = sb * kSellSlices + w;
  const long long o0 = S.sl_off[sl];
  const int W = (int)((S.sl_off[sl + 1] - o0) >> 5);
  if (W == 0) return;  // empty slice (warp-uniform)
  const int s = S.sb_sys[sb];
  if (sel && A && !sel[s]) return;  // values of the systems of this Newton step only
  const int no = S.node_off[s], nn = S.node_off[s + 1] - no, d0 = S.dof_off[s];
  const bool has = pos < S.sb_cnt[sb];
  int R0 = d0, q0 = 0, q1 = 0, deg = 0;
  if (has) {
    R0 = d0 + (S.perm[S.sb_n0[sb] + pos] - no);
    q0 = rowptr[R0];
    q1 = rowptr[R0 + nn];
    deg = (rowptr[R0 + 1] - q0) >> 1;
  }
  for (int k = 0; k < W; ++k) {
    const bool in = has && k < deg;
    const long long d = o0 + 32LL * k + t;
    if (cols) cols[d] = in ? colind[q0 + k] : R0;
    if (!A) continue;
    float e0 = 0, e1 = 0, e2 = 0, e3 = 0;
    if (in) {
      e0 = (float)A[q0 + k];
      e1 = (float)A[q0 + deg + k];
      e2 = (float)A[q1 + k];
      e3 = (float)A[q1 + deg + k];
    }
    vlo[4 * d] = __float2bfloat16_rn(e0); vlo[4 * d + 1] = __float2bfloat16_rn(e1);
    vlo[4 * d + 2] = __float2bfloat16_rn(e2); vlo[4 * d + 3] = __float2bfloat16_rn(e3);
  }
}

// Finest-level row products over the node slices, both rows (u, v) of a node per thread.
//   MODE 0 (PCG SpMV):    out = mask(K x); partial x.out
//   MODE 1 (AMG residual): out = mask(b - K x)                 (systems deeper than level 0)
//   MODE 2 (AMG smoothing): out = mask(x + invd (b - K x)), pcopy = out; partial b.out
// The partials go per slice: part[slice block * kSellSlices + warp].  List-driven when act.cnt is
// set (the CTAs loop over the active slice blocks), else one slice block per CTA.
// The slot loop is unrolled eight deep (a P1 slice's width in one pass), so a thread has eight
// column loads and their gathers in flight.  FP32 vectors: the SpMV (FP32 values) at most 64
// registers, four CTAs per SM; the BF16 passes at most 48, five CTAs per SM; FP64 vectors: the
// compiler's choice.  Measured on B200 (256-mesh batch, algorithmic bytes): three deep at 40
// registers, SpMV 3.41 and smoothing 2.88 TB/s; eight deep, SpMV 4.10 at four CTAs per SM and
// the BF16 passes 3.56 at five.
template <typename KT, typename VT, int MODE>
__global__ void __launch_bounds__(256, sizeof(VT) == 4 ? (MODE == 0 ? 4 : 5) : 0) k_sell(SellDev S, int nsb, ActList act, const int* sel, const int* done,
                                              const int* depth, const KT* vals, const VT* x, const VT* b,
                                              const VT* invd, const unsigned char* cmask, VT* out, VT* pcopy,
                                              double* part) {
  pdl_enter();
  const int nv = act.cnt ? *act.cnt : nsb;
  const int w = threadIdx.x >> 5, t = threadIdx.x & 31, pos = w * 32 + t;
  for (int vb = blockIdx.x; vb < nv; vb += gridDim.x) {
    const int sb = act.map ? act.map[vb] : vb;
    const int s = S.sb_sys[sb];
    const bool live = sel[s] && !done[s] && (MODE == 0 || depth[s] > S.lev);
    if (MODE == 1 && !live) continue;  // uniform over the block
    double pv = 0;
    if (live && pos < S.sb_cnt[sb]) {
      const int sl = sb * kSellSlices + w;
      const long long o0 = S.sl_off[sl];
      const int W = (int)((S.sl_off[sl + 1] - o0) >> 5);
      const int no = S.node_off[s], nn = S.node_off[s + 1] - no;
      const int g = S.perm[S.sb_n0[sb] + pos];
      const int ru = S.dof_off[s] + (g - no), rv = ru + nn;
      // the node's own rows, loaded ahead of the row products
      const bool mu = cmask && cmask[ru], mv = cmask && cmask[rv];
      double xu0 = 0, xv0 = 0, bu0 = 0, bv0 = 0, du = 0, dv = 0;
      if (MODE != 1) { xu0 = to_d(x[ru]); xv0 = to_d(x[rv]); }
      if (MODE != 0) { bu0 = to_d(b[ru]); bv0 = to_d(b[rv]); }
      if (MODE == 2) { du = to_d(invd[ru]); dv = to_d(invd[rv]); }
      const int* cp = S.cols + o0 + t;
      const KT* vp = vals + 4 * (o0 + t);
      double au = 0, av = 0;
#pragma unroll 8
      for (int k = 0; k < W; ++k) {
        int j = __ldg(cp + 32 * k);
        bool okj = true;
        UA_CHECK_INDEX(S.dbg, j, S.dof_off[s], S.dof_off[s] + nn, BS_SELL_COL, okj);
        (void)okj;
        double e[4];
        Quad<KT>::get(vp + 128 * k, e);
        const double xu = to_d(x[j]), xv = to_d(x[j + nn]);
        au = fma(e[0], xu, au);
        au = fma(e[1], xv, au);
        av = fma(e[2], xu, av);
        av = fma(e[3], xv, av);
      }
      if (MODE == 0) {
        const double qu = mu ? 0.0 : au, qv = mv ? 0.0 : av;
        out[ru] = (VT)qu;
        out[rv] = (VT)qv;
        pv = xu0 * qu + xv0 * qv;
      } else if (MODE == 1) {
        out[ru] = (VT)(mu ? 0.0 : bu0 - au);
        out[rv] = (VT)(mv ? 0.0 : bv0 - av);
      } else {
        const double zu = mu ? 0.0 : xu0 + du * (bu0 - au);
        const double zv = mv ? 0.0 : xv0 + dv * (bv0 - av);
        out[ru] = (VT)zu;
        out[rv] = (VT)zv;
        if (pcopy) { pcopy[ru] = (VT)zu; pcopy[rv] = (VT)zv; }
        pv = bu0 * zu + bv0 * zv;
      }
    }
    if (MODE == 1 || !part) continue;  // uniform per launch
    // one partial per slice (a fixed-order warp sum): no CTA barrier, so the warps of the short
    // slices do not wait for the long ones
    double tw = pv;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tw += __shfl_down_sync(0xffffffffu, tw, o);
    if (t == 0) part[sb * kSellSlices + w] = tw;
  }
}

// ---------------------------------------------------------------------------
// device: smoothed aggregation (P = (I - w D^-1 A) P0, coarse operator P' A P)
// ---------------------------------------------------------------------------
//
// Values live on node-level lists with the tangent's layout rule: the entry of
// dof row (c, g), column component c2 and list position k of system s sits at
// off[s] + c*2*nnz[s] + 2*(ptr[g] - base[s]) + c2*deg(g) + k.  Every output
// entry is summed in a fixed order (no atomics), so results are reproducible.

constexpr double kSaOmega = 4.0 / 3.0;  // damping of the prolongator smoother (l1 diagonal: rho(D^-1 A) <= 1)

__device__ __forceinline__ int sa_find(const int* list, int n, int key) {  // list sorted ascending
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (list[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo < n && list[lo] == key ? lo : -1;
}

// dof row -> system, component, node (global) of a level
__device__ __forceinline__ void sa_decode(int i, const int* dof_sys, const int* dof_off, const int* node_off, int& s,
                                          int& c, int& g) {
  s = dof_sys[i];
  const int no = node_off[s], nn = node_off[s + 1] - no, loc = i - dof_off[s];
  c = loc / nn;
  g = no + (loc - c * nn);
}

// prolongator rows: P(i,:) = P0(i,:) - w invd_i A(i,:) P0 on unmasked rows and columns
// ST: the type the set-up stores and sums P, A P and P' in (FP32 for the mixed-precision form,
// whose V-cycle transfers read FP32 values, else FP64)
template <typename KT, typename VT, typename ST>
__global__ void k_sa_P(int nf, const int* dof_sys, const int* dof_off, const int* node_off, const int* rowptr,
                       const int* colind, const KT* A, const unsigned char* mask, const VT* invd, const int* agg,
                       const int* pn_ptr, const int* pn_col, const int* pbase, const int* pnnz, const int* poff,
                       ST* P, const int* sel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  int s, c, g;
  sa_decode(i, dof_sys, dof_off, node_off, s, c, g);
  if (sel && !sel[s]) return;
  const int pr = pn_ptr[g], dP = pn_ptr[g + 1] - pr;
  ST* row = P + poff[s] + (size_t)c * 2 * pnnz[s] + 2 * (size_t)(pr - pbase[s]);
  for (int t = 0; t < 2 * dP; ++t) row[t] = 0;
  if (mask && mask[i]) return;
  const int k0 = sa_find(pn_col + pr, dP, agg[g]);
  if (k0 >= 0) row[c * dP + k0] = 1;
  const ST f = (ST)(kSaOmega * (double)invd[i]);
  // the row holds the u block then the v block of the node's deg neighbours (the same nodes in
  // the same order), so one search per neighbour serves both blocks; each target still sums its
  // block's entries in row order
  const int q0 = rowptr[i], deg = (rowptr[i + 1] - q0) >> 1;
  const int d0 = dof_off[s], no = node_off[s], nn = node_off[s + 1] - no;
  for (int k = 0; k < deg; ++k) {
    const int ju = colind[q0 + k];
    const int kk = sa_find(pn_col + pr, dP, agg[no + (ju - d0)]);
    if (kk < 0) continue;
    if (!(mask && mask[ju])) row[kk] -= f * (ST)A[q0 + k];
    if (!(mask && mask[ju + nn])) row[dP + kk] -= f * (ST)A[q0 + deg + k];
  }
}

// P in the transfer layout: per node-level entry (fine node g, coarse node K) one quad of
// P((c,g),(c2,K)) in the order (c,c2) = (0,0), (0,1), (1,0), (1,1), read with one load.  The mixed
// form keeps BF16 quads (its set-up then reads the same rounded values, so the coarse operator is
// the Galerkin product of the prolongator the V-cycle applies), the FP64 form FP64 quads.
struct alignas(8) PQuadH {
  __nv_bfloat162 r0, r1;
};
struct alignas(16) PQuadD {
  double2 r0, r1;
};
template <typename VT>
struct PQuadOf {
  using T = PQuadD;
};
template <>
struct PQuadOf<float> {
  using T = PQuadH;
};
__device__ __forceinline__ void pq_get(const PQuadH* q, double (&v)[4]) {
  const uint2 u = __ldg(reinterpret_cast<const uint2*>(q));
  const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
  const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void pq_get(const PQuadH* q, float (&v)[4]) {
  const uint2 u = __ldg(reinterpret_cast<const uint2*>(q));
  const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
  const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void pq_get(const PQuadD* q, double (&v)[4]) {
  const double2 a = __ldg(&q->r0), b = __ldg(&q->r1);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void pq_set(PQuadH* q, double v0, double v1, double v2, double v3) {
  PQuadH h;
  h.r0 = __floats2bfloat162_rn((float)v0, (float)v1);
  h.r1 = __floats2bfloat162_rn((float)v2, (float)v3);
  *q = h;
}
__device__ __forceinline__ void pq_set(PQuadD* q, double v0, double v1, double v2, double v3) {
  q->r0 = make_double2(v0, v1);
  q->r1 = make_double2(v2, v3);
}

// A P rows: AP(i,:) = sum over unmasked columns j of A(i,j) P(j,:), kSaGL lanes per fine node g.
// Both rows (c = 0, 1) of the node share its neighbour list, so each neighbour h contributes
// A((c,g),(c2,h)) P((c2,h),:) to four output blocks (c, c3) at once.  The lanes first load the
// data of up to kSaGL neighbours (column, the four A entries, the row of P(h,:)); the neighbours
// then go in order.  A row of at most kSaApSm coarse columns is summed in shared memory (its
// column list there too, for the searches): the lanes split into kSaApG groups of kSaGL / kSaApG,
// group q takes the neighbours q, q + kSaApG, ... into its own copy of the row, its lanes the
// entries of P(h,:), whose targets in the AP row are distinct, and the copies are added in group
// order at the one write.  Longer rows are summed in place in global memory by all kSaGL lanes,
// neighbour after neighbour.  Either way a fixed summation order without atomics.  FP32 values:
// at most 48 registers, ten CTAs (40 warps) per SM for the gathers in flight.
constexpr int kSaGL = 8;
constexpr int kSaApG = 2;
constexpr int kSaApSm = 64;  // longest row summed in shared memory
// dynamic shared memory: per fine node kSaApG copies of 4 * ms sums and ms columns (ms = 0: none)
template <typename ST>
size_t sa_ap_smem(int ms) { return (size_t)(128 / kSaGL) * ms * (kSaApG * 4 * sizeof(ST) + sizeof(int)); }
template <typename KT, typename ST>
__global__ void __launch_bounds__(128, sizeof(ST) == 4 ? 10 : 0) k_sa_AP(int nfn, const int* node_sys, const int* dof_off, const int* node_off,
                                               const int* rowptr, const int* colind, const KT* A,
                                               const unsigned char* mask, const int* pn_ptr, const int* pn_col,
                                               const typename PQuadOf<KT>::T* Q, const int* apn_ptr,
                                               const int* apn_col, const int* apbase, const int* apnnz,
                                               const int* apoff, ST* AP, const int* sel, int ms) {
  extern __shared__ __align__(16) unsigned char sa_smem[];
  const int gi = threadIdx.x / kSaGL;
  ST* g_acc = reinterpret_cast<ST*>(sa_smem) + (size_t)gi * kSaApG * 4 * ms;
  int* g_col = reinterpret_cast<int*>(reinterpret_cast<ST*>(sa_smem) + (size_t)(128 / kSaGL) * kSaApG * 4 * ms) +
               gi * ms;
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) / kSaGL, lane = threadIdx.x % kSaGL;
  if (g >= nfn) return;  // whole groups leave together
  const unsigned gmask = ((1u << kSaGL) - 1u) << ((threadIdx.x & 31) & ~(kSaGL - 1));
  const int s = node_sys[g];
  if (sel && !sel[s]) return;  // whole groups
  const int no = node_off[s], nn = node_off[s + 1] - no, d0 = dof_off[s];
  const int i0 = d0 + (g - no), i1 = i0 + nn;
  const int ar = apn_ptr[g], dA = apn_ptr[g + 1] - ar;
  const size_t ars = (size_t)2 * apnnz[s];  // AP row stride between c = 0 and c = 1
  ST* r0 = AP + apoff[s] + 2 * (size_t)(ar - apbase[s]);
  const bool sm = ms > 0;  // every row of the launch fits (ms is the level's longest row)
  const int ng = sm ? kSaApG : 1, gw = kSaGL / ng;  // lane groups, lanes per group
  const int q = lane / gw, ql = lane % gw;
  ST* o0 = sm ? g_acc + (size_t)q * 4 * dA : r0;  // this group's copy
  const size_t o1 = sm ? (size_t)2 * dA : ars;   // offset of row c = 1
  const int* acol = apn_col + ar;
  if (sm) {
    for (int t = lane; t < dA; t += kSaGL) g_col[t] = acol[t];
    acol = g_col;
  }
  for (int t = lane; t < (sm ? kSaApG * 4 * dA : 2 * dA); t += kSaGL) {
    if (sm) g_acc[t] = 0;
    else { r0[t] = 0; r0[ars + t] = 0; }
  }
  const bool m0 = mask && mask[i0], m1 = mask && mask[i1];
  if (!(m0 && m1)) {
    const int q0 = rowptr[i0], q1 = rowptr[i1], deg = (rowptr[i0 + 1] - q0) >> 1;
    for (int k0 = 0; k0 < deg; k0 += kSaGL) {
      // lane k loads neighbour k0 + k
      ST b00 = 0, b01 = 0, b10 = 0, b11 = 0;
      int bpj = 0, bdP = 0;
      if (k0 + lane < deg) {
        const int k = k0 + lane;
        const int ju = colind[q0 + k], jv = ju + nn;  // u and v dofs of neighbour node h
        const bool cu = mask && mask[ju], cv = mask && mask[jv];
        b00 = (m0 || cu) ? ST(0) : (ST)A[q0 + k];
        b01 = (m0 || cv) ? ST(0) : (ST)A[q0 + deg + k];
        b10 = (m1 || cu) ? ST(0) : (ST)A[q1 + k];
        b11 = (m1 || cv) ? ST(0) : (ST)A[q1 + deg + k];
        const int h = no + (ju - d0);
        bpj = pn_ptr[h];
        bdP = pn_ptr[h + 1] - bpj;
      }
      const int nk = min(kSaGL, deg - k0);
      for (int e0 = 0; e0 < nk; e0 += ng) {
        const int e = e0 + q;  // this group's neighbour (lanes past nk read zeros)
        const ST a00 = __shfl_sync(gmask, b00, e, kSaGL), a01 = __shfl_sync(gmask, b01, e, kSaGL);
        const ST a10 = __shfl_sync(gmask, b10, e, kSaGL), a11 = __shfl_sync(gmask, b11, e, kSaGL);
        const int pj = __shfl_sync(gmask, bpj, e, kSaGL), dPj = __shfl_sync(gmask, bdP, e, kSaGL);
        __syncwarp(gmask);  // the previous neighbours' updates (and the zeroed rows) are visible
        if (e >= nk || (a00 == ST(0) && a01 == ST(0) && a10 == ST(0) && a11 == ST(0))) continue;
        for (int t = ql; t < dPj; t += gw) {
          // the P entries load beside the column, ahead of the search
          const int colp = pn_col[pj + t];
          double pq[4];
          pq_get(Q + pj + t, pq);
          const ST p00 = (ST)pq[0], p01 = (ST)pq[1], p10 = (ST)pq[2], p11 = (ST)pq[3];
          const int kk = sa_find(acol, dA, colp);
          if (kk < 0) continue;
          o0[kk] += a00 * p00 + a01 * p10;
          o0[dA + kk] += a00 * p01 + a01 * p11;
          o0[o1 + kk] += a10 * p00 + a11 * p10;
          o0[o1 + dA + kk] += a10 * p01 + a11 * p11;
        }
      }
    }
  }
  if (sm) {  // one write of the two rows, the group copies added in order
    __syncwarp(gmask);
    for (int t = lane; t < 2 * dA; t += kSaGL) {
      ST v0 = g_acc[t], v1 = g_acc[2 * dA + t];
#pragma unroll
      for (int c = 1; c < kSaApG; ++c) {
        v0 += g_acc[(size_t)c * 4 * dA + t];
        v1 += g_acc[(size_t)c * 4 * dA + 2 * dA + t];
      }
      r0[t] = v0;
      r0[ars + t] = v1;
    }
  }
}

// quads of the prolongator rows of fine node g (pn order): thread per fine node
template <typename ST, typename QT>
__global__ void k_sa_quads(int nfn, const int* node_sys, const int* pn_ptr, const int* pbase, const int* pnnz,
                           const int* poff, const ST* P, QT* Q, const int* sel) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nfn) return;
  const int s = node_sys[g];
  if (sel && !sel[s]) return;
  const int pr = pn_ptr[g], dP = pn_ptr[g + 1] - pr;
  const size_t prs = (size_t)2 * pnnz[s];  // row c = 1 after row c = 0
  const ST* p0 = P + poff[s] + 2 * (size_t)(pr - pbase[s]);  // row c: [c2 = 0 (dP)][c2 = 1 (dP)]
  for (int k = 0; k < dP; ++k)
    pq_set(Q + pr + k, (double)p0[k], (double)p0[dP + k], (double)p0[prs + k], (double)p0[prs + dP + k]);
}

// the same quads in ptn order (coarse node J, its fine nodes u): thread per ptn entry (its
// system is its fine node's); every P entry is the image of exactly one ptn entry
template <typename QT>
__global__ void k_sa_qt(long long np, const int* fnode_sys, const int* ptn_fine, const int* ptn_k,
                        const int* pn_ptr, const QT* Q, QT* QTr, const int* sel) {
  const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (u >= np) return;
  const int g = ptn_fine[u];
  if (sel && !sel[fnode_sys[g]]) return;
  QTr[u] = Q[pn_ptr[g] + ptn_k[u]];
}

// coarse operator rows: Ac((c2,J),:) = sum over P'((c2,J), (c,g)) AP((c,g),:), into the coarse
// level's CSR.  One warp per coarse node J: its two rows share the column list (sorted, in
// shared memory) and the fine nodes g of P'(J,:).  The lanes first load the fine-node data of 32
// list entries.  The warp is split into kSaAcG groups of kSaAcW lanes: group q takes the entries
// q, q + kSaAcG, ... in order, its lanes the entries of AP(g,:), whose columns are distinct, and
// sums into the group's own copy of the four FP64 blocks; the copies are added in group order at
// the end.  A fixed summation order without atomics.
constexpr int kSaAcWarps = 4;
constexpr int kSaAcG = 4, kSaAcW = 32 / kSaAcG;
// dynamic shared memory of a CTA for coarse rows of at most md nodes
inline size_t sa_ac_smem(int md) { return (size_t)kSaAcWarps * md * (kSaAcG * 4 * sizeof(double) + sizeof(int)); }
template <typename KT, typename ST>
__global__ void __launch_bounds__(32 * kSaAcWarps, sizeof(ST) == 4 ? 10 : 0) k_sa_Ac(int ncn, const int* cnode_sys, const int* cdof_off,
                                                           const int* cnode_off, const int* crowptr,
                                                           const int* ccolind, const int* ptn_ptr,
                                                           const int* ptn_fine, const typename PQuadOf<KT>::T* QTr,
                                                           const int* apn_ptr,
                                                           const int* apn_col, const int* apbase, const int* apnnz,
                                                           const int* apoff, const ST* AP, KT* Ac, const int* sel,
                                                           int md) {
  extern __shared__ __align__(16) unsigned char sa_smem[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int J = blockIdx.x * kSaAcWarps + wid;
  if (J >= ncn) return;  // whole warps leave together
  const int s = cnode_sys[J];
  if (sel && !sel[s]) return;  // whole warps
  const int cno = cnode_off[s], cnn = cnode_off[s + 1] - cno;
  const int R0 = cdof_off[s] + (J - cno), R1 = R0 + cnn;
  const int cr0 = crowptr[R0], cr1 = crowptr[R1], degc = min((crowptr[R0 + 1] - cr0) >> 1, md);
  const int cbase = cdof_off[s] - cno;  // u-column dof of coarse node K: cbase + K
  double* acc = reinterpret_cast<double*>(sa_smem) + (size_t)wid * kSaAcG * 4 * md;
  int* col = reinterpret_cast<int*>(reinterpret_cast<double*>(sa_smem) + (size_t)kSaAcWarps * kSaAcG * 4 * md) +
             wid * md;
  // copy q, block (c2, c3) at acc[(4 q + 2 c2 + c3) degc + pos]
  for (int t = lane; t < kSaAcG * 4 * degc; t += 32) acc[t] = 0;
  for (int t = lane; t < degc; t += 32) col[t] = ccolind[cr0 + t] - cbase;
  const int q = lane / kSaAcW, ql = lane % kSaAcW;
  double* ga = acc + (size_t)q * 4 * degc;
  const int tr = ptn_ptr[J], dT = ptn_ptr[J + 1] - tr;
  const size_t ars = (size_t)2 * apnnz[s];
  const ST* apb = AP + apoff[s];
  const int apb0 = apbase[s];
  for (int u0 = 0; u0 < dT; u0 += 32) {
    const int my = u0 + lane;
    int g_ar = 0, g_dA = 0;
    double w00 = 0, w01 = 0, w10 = 0, w11 = 0;
    if (my < dT) {
      const int g = ptn_fine[tr + my];
      g_ar = apn_ptr[g];
      g_dA = apn_ptr[g + 1] - g_ar;
      // w(c2, c) = P'((c2,J),(c,g)) = P((c,g),(c2,J)), quad entry 2 c + c2
      double pq[4];
      pq_get(QTr + tr + my, pq);
      w00 = pq[0];
      w01 = pq[2];
      w10 = pq[1];
      w11 = pq[3];
    }
    const int nstep = min(32, dT - u0);
    for (int e0 = 0; e0 < nstep; e0 += kSaAcG) {
      const int e = e0 + q;  // this group's entry (lanes past nstep hold dA = 0)
      const int ar = __shfl_sync(0xffffffffu, g_ar, e), dA = __shfl_sync(0xffffffffu, g_dA, e);
      const double v00 = __shfl_sync(0xffffffffu, w00, e), v01 = __shfl_sync(0xffffffffu, w01, e);
      const double v10 = __shfl_sync(0xffffffffu, w10, e), v11 = __shfl_sync(0xffffffffu, w11, e);
      const ST* a0 = apb + 2 * (size_t)(ar - apb0);  // AP((c,g),(c3,kk)) = a0[c ars + c3 dA + kk]
      __syncwarp();  // the previous entries' sums (and the zeroed copies) are visible to the warp
      for (int kk = ql; kk < dA; kk += kSaAcW) {
        // the AP entries load beside the column, ahead of the search
        const int cK = apn_col[ar + kk];
        const double x00 = (double)a0[kk], x01 = (double)a0[dA + kk], x10 = (double)a0[ars + kk],
                     x11 = (double)a0[ars + dA + kk];
        const int pos = sa_find(col, degc, cK);
        if (pos < 0) continue;
        ga[pos] += v00 * x00 + v01 * x10;
        ga[degc + pos] += v00 * x01 + v01 * x11;
        ga[2 * degc + pos] += v10 * x00 + v11 * x10;
        ga[3 * degc + pos] += v10 * x01 + v11 * x11;
      }
    }
  }
  __syncwarp();
  for (int t = lane; t < 2 * degc; t += 32) {
    double a0 = acc[t], a1 = acc[2 * degc + t];
#pragma unroll
    for (int c = 1; c < kSaAcG; ++c) {
      a0 += acc[(size_t)c * 4 * degc + t];
      a1 += acc[(size_t)c * 4 * degc + 2 * degc + t];
    }
    Ac[cr0 + t] = (KT)a0;
    Ac[cr1 + t] = (KT)a1;
  }
}

// The transfers are gather chains (list entry -> node block -> P list -> vector entries).  They
// load what a node block needs (its system, its nodes' P lists) ahead of the system's flags, and
// take the entries of a P list in chunks of kSaChunk (half that in FP64): the chunk's columns and
// P quads load together, then its vector entries, then the sums in list order.
constexpr int kSaChunk = 4;

// restriction b_c = P' res (coarse pre-smoothing x_c = invd b_c unless lc is the system's coarsest),
// kSaRL lanes per coarse node: both rows (c2 = 0, 1) of the node share the fine-node list and
// the gathered residuals; a lane sum in a fixed order.  A CTA of 32 kSaRL threads takes one node
// block (kAmgNB = 32 coarse nodes) per pass.
constexpr int kSaRL = 8;
template <typename VT>
__global__ void __launch_bounds__(32 * kSaRL, 4) k_sa_restrict(const int* nb_start, const int* nb_sys, ActList act,
                                                            const int* cdof_off, const int* cnode_off,
                                                            const int* depth, int lc, const int* sel,
                                                            const int* done, const int* ptn_ptr,
                                                            const int* ptn_fine,
                                                            const typename PQuadOf<VT>::T* QTr,
                                                            const int* fdof_off, const int* fnode_off,
                                                            const VT* res, const VT* cinvd, VT* cb, VT* cx) {
  pdl_enter();
  static_assert(kAmgNB == 32, "one coarse node per kSaRL-lane group of a 32 kSaRL-thread CTA");
  constexpr int CH = sizeof(VT) == 4 ? kSaChunk : kSaChunk / 2;  // FP64 chunks held to the register budget
  const int sub = threadIdx.x / kSaRL, lane = threadIdx.x % kSaRL;
  const int nv = act.cnt ? *act.cnt : gridDim.x;  // list entries, else one node block per CTA
  for (int vb = blockIdx.x; vb < nv; vb += gridDim.x) {
    const int b = act.map ? act.map[vb] : vb;
    const int s = nb_sys[b];
    const int J = nb_start[b] + sub;
    const bool valid = J < nb_start[b + 1];
    int tr = 0, t1 = 0;
    if (valid) {  // ahead of the flags
      tr = ptn_ptr[J];
      t1 = ptn_ptr[J + 1];
    }
    if (!sel[s] || done[s]) continue;  // uniform over the block
    const int cno = cnode_off[s], cnn = cnode_off[s + 1] - cno, cd = cdof_off[s];
    const int fno = fnode_off[s], fnn = fnode_off[s + 1] - fno, fd = fdof_off[s];
    const bool presmooth = depth[s] > lc;
    double a0 = 0, a1 = 0;
    for (int u0 = tr + lane; u0 < t1; u0 += kSaRL * CH) {
      int f[CH];
      VT q[CH][4];  // P((c,g),(c2,J)) at 2 c + c2 (BF16 quads widen exactly to FP32)
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        const int u = u0 + k * kSaRL;
        f[k] = -1;
        if (u < t1) {
          f[k] = fd + (ptn_fine[u] - fno);
          pq_get(QTr + u, q[k]);
        }
      }
      VT r0[CH], r1[CH];
#pragma unroll
      for (int k = 0; k < CH; ++k)
        if (f[k] >= 0) {
          r0[k] = res[f[k]];
          r1[k] = res[f[k] + fnn];
        }
#pragma unroll
      for (int k = 0; k < CH; ++k)
        if (f[k] >= 0) {
          a0 += (double)q[k][0] * (double)r0[k] + (double)q[k][2] * (double)r1[k];
          a1 += (double)q[k][1] * (double)r0[k] + (double)q[k][3] * (double)r1[k];
        }
    }
#pragma unroll
    for (int o = kSaRL / 2; o > 0; o >>= 1) {
      a0 += __shfl_down_sync(0xffffffffu, a0, o, kSaRL);
      a1 += __shfl_down_sync(0xffffffffu, a1, o, kSaRL);
    }
    if (valid && lane == 0) {
      const int R0 = cd + (J - cno), R1 = R0 + cnn;
      cb[R0] = (VT)a0;
      cb[R1] = (VT)a1;
      if (presmooth) {
        cx[R0] = (VT)((double)cinvd[R0] * a0);
        cx[R1] = (VT)((double)cinvd[R1] * a1);
      }
    }
  }
}

// prolongation x += P x_c on level l (systems deeper than l; masked rows have zero P rows),
// one thread per fine node of a node block: both rows share the coarse-node list and the gathered x_c
// (one warp per node block of kAmgNB = 32 nodes, kSaPW warps per CTA)
constexpr int kSaPW = 8;
template <typename VT>
__global__ void __launch_bounds__(32 * kSaPW, 4) k_sa_prolong(int nnb, const int* nb_start, const int* nb_sys,
                                                           ActList act, const int* dof_off, const int* node_off,
                                                           const int* depth, int l, const int* sel, const int* done,
                                                           const int* pn_ptr, const int* pn_col,
                                                           const typename PQuadOf<VT>::T* Q, const int* cdof_off,
                                                           const int* cnode_off, const VT* xc,
                                                           VT* x) {
  pdl_enter();
  static_assert(kAmgNB == 32, "one fine node per lane");
  constexpr int CH = sizeof(VT) == 4 ? kSaChunk : kSaChunk / 2;  // FP64 chunks held to the register budget
  const int nv = act.cnt ? *act.cnt : nnb;  // list entries, else every node block
  const int lane = threadIdx.x & 31;
  for (int vb = blockIdx.x * kSaPW + (threadIdx.x >> 5); vb < nv; vb += gridDim.x * kSaPW) {
    const int b = act.map ? act.map[vb] : vb;
    const int s = nb_sys[b];
    const int g = nb_start[b] + lane;
    const bool valid = g < nb_start[b + 1];
    int pr = 0, pe = 0;
    if (valid) {  // ahead of the flags
      pr = pn_ptr[g];
      pe = pn_ptr[g + 1];
    }
    if (!sel[s] || done[s] || depth[s] <= l) continue;  // uniform over the warp
    if (!valid) continue;
    const int cno = cnode_off[s], cnn = cnode_off[s + 1] - cno, cd = cdof_off[s];
    const int no = node_off[s], nn = node_off[s + 1] - no, d0 = dof_off[s];
    const int i0 = d0 + (g - no), i1 = i0 + nn;
    double a0 = (double)x[i0], a1 = (double)x[i1];
    for (int k0 = pr; k0 < pe; k0 += CH) {
      int K[CH];
      VT q[CH][4];  // P((c,g),(c2,K)) at 2 c + c2 (BF16 quads widen exactly to FP32)
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        K[k] = -1;
        if (k0 + k < pe) {
          K[k] = cd + (pn_col[k0 + k] - cno);
          pq_get(Q + k0 + k, q[k]);
        }
      }
      VT xu[CH], xv[CH];
#pragma unroll
      for (int k = 0; k < CH; ++k)
        if (K[k] >= 0) {
          xu[k] = xc[K[k]];
          xv[k] = xc[K[k] + cnn];
        }
#pragma unroll
      for (int k = 0; k < CH; ++k)
        if (K[k] >= 0) {
          a0 += (double)q[k][0] * (double)xu[k] + (double)q[k][1] * (double)xv[k];
          a1 += (double)q[k][2] * (double)xu[k] + (double)q[k][3] * (double)xv[k];
        }
    }
    x[i0] = (VT)a0;
    x[i1] = (VT)a1;
  }
}

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------

template <typename KT, typename VT>
static int numeric_t(ua_mesh* m, const int* rowptr0, const int* colind0, const KT* K0, const unsigned char* cmask,
                     const int* sel, const int* psel, long long* launches) {
  Amg* a = m->amg;
  cudaStream_t st = m->stream;
  auto l1 = [&](int l) {
    const AmgLevel& L = a->lev[l];
    k_amg_l1<KT, VT><<<(L.ndof + 255) / 256, 256, 0, st>>>(
        L.ndof, l == 0 ? rowptr0 : L.rowptr, l == 0 ? colind0 : L.colind, l == 0 ? K0 : (const KT*)L.A,
        l == 0 ? cmask : nullptr, (VT*)L.invd, L.dof_sys, sel), ++*launches;
  };
  if (a->sa) {
    // per level: smoother diagonal, smoothed prolongator, A P, P' values, coarse operator
    for (int l = 0; l + 1 < a->nlev; ++l) {
      AmgLevel& F = a->lev[l];
      AmgLevel& C = a->lev[l + 1];
      const int* rp = l == 0 ? rowptr0 : F.rowptr;
      const int* ci = l == 0 ? colind0 : F.colind;
      const KT* A = l == 0 ? K0 : (const KT*)F.A;
      const unsigned char* mk = l == 0 ? cmask : nullptr;
      l1(l);
      const int nbf = (F.ndof + 127) / 128;
      // the mixed form sets up in FP32, the FP64 form in FP64; P then goes into the transfer
      // layout (quads, pn and ptn order), which A P, the coarse operator and the V-cycle read
      using ST = typename std::conditional<sizeof(KT) == 4, float, double>::type;
      using QT = typename PQuadOf<KT>::T;
      ST* Pv = sizeof(KT) == 4 ? (ST*)F.sa_plo : (ST*)F.sa_p;
      ST* APv = (ST*)F.sa_ap;
      QT* Qv = (QT*)(sizeof(KT) == 4 ? F.sa_qh : F.sa_qd);
      QT* QTv = (QT*)(sizeof(KT) == 4 ? F.sa_qth : F.sa_qtd);
      k_sa_P<KT, VT, ST><<<nbf, 128, 0, st>>>(F.ndof, F.dof_sys, F.d_dof_off, F.d_node_off, rp, ci, A, mk,
                                              (const VT*)F.invd, F.sa_agg, F.pn_ptr, F.pn_col, F.pbase, F.pnnz,
                                              F.poff, Pv, psel), ++*launches;
      k_sa_quads<ST, QT><<<(F.nn + 127) / 128, 128, 0, st>>>(F.nn, F.node_sys, F.pn_ptr, F.pbase, F.pnnz, F.poff,
                                                            Pv, Qv, psel), ++*launches;
      k_sa_qt<QT><<<(int)((F.np + 255) / 256), 256, 0, st>>>(F.np, F.node_sys, F.ptn_fine, F.ptn_k, F.pn_ptr, Qv,
                                                               QTv, psel), ++*launches;
      const int ms = F.ap_maxrow <= kSaApSm ? F.ap_maxrow : 0;  // rows summed in shared memory
      k_sa_AP<KT, ST><<<(int)(((long long)F.nn * kSaGL + 127) / 128), 128, sa_ap_smem<ST>(ms), st>>>(
          F.nn, F.node_sys, F.d_dof_off, F.d_node_off, rp, ci, A, mk, F.pn_ptr, F.pn_col, Qv, F.apn_ptr, F.apn_col,
          F.apbase, F.apnnz, F.apoff, APv, sel, ms), ++*launches;
      k_sa_Ac<KT, ST><<<(C.nn + kSaAcWarps - 1) / kSaAcWarps, 32 * kSaAcWarps, sa_ac_smem(F.ac_maxdeg), st>>>(
          C.nn, C.node_sys, C.d_dof_off, C.d_node_off, C.rowptr, C.colind, F.ptn_ptr, F.ptn_fine, QTv, F.apn_ptr,
          F.apn_col, F.apbase, F.apnnz, F.apoff, APv, (KT*)C.A, sel, F.ac_maxdeg),
          ++*launches;
    }
    l1(a->nlev - 1);
  } else {
    for (int l = 0; l + 1 < a->nlev; ++l) {
      const AmgLevel& F = a->lev[l];
      const AmgLevel& C = a->lev[l + 1];
      k_amg_galerkin<KT><<<(C.ndof + 127) / 128, 128, 0, st>>>(
          C.ndof, C.mptr, C.mlist, l == 0 ? rowptr0 : F.rowptr, l == 0 ? colind0 : F.colind,
          l == 0 ? K0 : (const KT*)F.A, F.cmap, l == 0 ? cmask : nullptr, C.rowptr, C.colind, (KT*)C.A), ++*launches;
    }
    for (int l = 0; l < a->nlev; ++l) l1(l);
  }
  const int sm = (int)(sizeof(double) * (size_t)a->maxdn * 2 * a->maxdn);  // attribute set by the caller
  k_amg_dense_inverse<KT><<<a->nsys, 256, sm, st>>>(a->d_depth, a->d_dn, a->d_doff, a->d_lev_rowptr,
                                                     a->d_lev_colind, a->d_lev_A, a->d_lev_dofoff, a->dense, sel),
      ++*launches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(UA_ERR_CUDA, "AMG numeric phase: %s", cudaGetErrorString(e));
  return UA_OK;
}

static SellDev sell_dev(const ua_mesh* m, const Sell& S) {
  return SellDev{S.sb_sys, S.sb_n0, S.sb_cnt, S.sb_rbu, S.sb_rbv, S.perm, S.sl_off, S.cols,
                 m->dm.sys_dof_off, m->dm.sys_node_off, m->dm.dbg, 0};
}
static SellDev csell_dev(const ua_mesh* m, const Sell& S, const AmgLevel& L, int l) {
  return SellDev{S.sb_sys, S.sb_n0, S.sb_cnt, nullptr, nullptr, S.perm, S.sl_off, S.cols,
                 L.d_dof_off, L.d_node_off, m->dm.dbg, l};
}

// Node slices of the coarse levels that run a residual and a smoothing pass (1 .. nlev-2) and
// hold at least kCsellMinNodes nodes (below that the CSR row blocks, finer-grained than the slice
// blocks of 256 nodes, spread better over the SMs): per system, blocks of kSellNodes nodes
// ordered by decreasing degree, slices of 32 (the finest level's layout; node degrees from the
// level's CSR).
constexpr int kCsellMinNodes = 131072;
static void csell_init(ua_mesh* m) {
  Amg* a = m->amg;
  const int nsys = a->nsys;
  a->csell.assign(std::max(a->nlev, 1), Sell());
  for (int l = 1; l + 1 < a->nlev; ++l) {
    AmgLevel& L = a->lev[l];
    Sell& S = a->csell[l];
    if (L.nn < kCsellMinNodes) continue;
    std::vector<int> rowptr(L.ndof + 1);
    if (cudaMemcpy(rowptr.data(), L.rowptr, sizeof(int) * rowptr.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
      S.failed = true;
      return;
    }
    std::vector<int> sb_sys, sb_n0, sb_cnt, perm(std::max(L.nn, 1)), idx;
    std::vector<long long> sl_off(1, 0);
    S.h_sys_sb_off.assign(nsys + 1, 0);
    for (int s = 0; s < nsys; ++s) {
      const int no = L.node_off[s], nn = L.node_off[s + 1] - no, d0 = L.dof_off[s];
      auto deg = [&](int g) { return (rowptr[d0 + (g - no) + 1] - rowptr[d0 + (g - no)]) >> 1; };
      for (int n0 = no; n0 < no + nn; n0 += kSellNodes) {
        const int cnt = std::min(kSellNodes, no + nn - n0);
        idx.resize(cnt);
        for (int k = 0; k < cnt; ++k) idx[k] = n0 + k;
        std::stable_sort(idx.begin(), idx.end(), [&](int p, int q) { return deg(p) > deg(q); });
        for (int k = 0; k < cnt; ++k) perm[n0 + k] = idx[k];
        for (int j = 0; j < kSellSlices; ++j) {
          int W = 0;
          for (int k = j * 32; k < std::min(cnt, j * 32 + 32); ++k) W = std::max(W, deg(idx[k]));
          sl_off.push_back(sl_off.back() + 32LL * W);
        }
        sb_sys.push_back(s);
        sb_n0.push_back(n0);
        sb_cnt.push_back(cnt);
      }
      S.h_sys_sb_off[s + 1] = (int)sb_sys.size();
    }
    bool ok = true;
    S.nsb = (int)sb_sys.size();
    S.slots = sl_off.back();
    S.sb_sys = upload(m, a, sb_sys, ok);
    S.sb_n0 = upload(m, a, sb_n0, ok);
    S.sb_cnt = upload(m, a, sb_cnt, ok);
    S.perm = upload(m, a, perm, ok);
    S.sl_off = upload(m, a, sl_off, ok);
    S.cols = (int*)dalloc(m, a, sizeof(int) * (size_t)S.slots, ok);
    S.vlo = (__nv_bfloat16*)dalloc(m, a, sizeof(__nv_bfloat16) * 4 * (size_t)S.slots, ok);
    if (!ok) { S.failed = true; return; }
    if (S.nsb)
      k_csell_fill<float><<<S.nsb, 256, 0, m->stream>>>(csell_dev(m, S, L, l), L.rowptr, L.colind, nullptr,
                                                       nullptr, S.cols, nullptr);
    if (cudaGetLastError() != cudaSuccess) { S.failed = true; return; }
    S.ready = true;
  }
}

int amg_sell_init(ua_mesh* m, const std::vector<int>& sys_rb_off0) {
  Amg* a = m->amg;
  if (!a || m->ndof != 2 || m->h_nodeptr.empty()) return UA_ERR_INVALID;
  Sell& S = a->sell;
  if (S.ready) return UA_OK;
  if (S.failed) return UA_ERR_INVALID;
  const int nsys = a->nsys;
  if ((int)sys_rb_off0.size() != nsys + 1) { S.failed = true; return UA_ERR_INVALID; }
  std::vector<int> sb_sys, sb_n0, sb_cnt, sb_rbu, sb_rbv, perm(m->nn_total), idx;
  std::vector<long long> sl_off(1, 0);
  S.h_sys_sb_off.assign(nsys + 1, 0);
  auto deg = [&](int g) { return m->h_nodeptr[g + 1] - m->h_nodeptr[g]; };
  for (int s = 0; s < nsys; ++s) {
    const int no = m->h_node_off[s], nn = m->h_node_off[s + 1] - no;
    const int nbc = (nn + kSellNodes - 1) / kSellNodes;
    // the handle's row blocks must be the u blocks then the v blocks of kSellNodes rows each
    if (sys_rb_off0[s + 1] - sys_rb_off0[s] != 2 * nbc || 2 * nn != m->h_dof_off[s + 1] - m->h_dof_off[s]) {
      S.failed = true;
      return set_error(UA_ERR_INVALID, "node slices: row blocks of system %d do not split at the u/v boundary", s);
    }
    for (int i = 0; i < nbc; ++i) {
      const int n0 = no + i * kSellNodes, cnt = std::min(kSellNodes, nn - i * kSellNodes);
      idx.resize(cnt);
      for (int k = 0; k < cnt; ++k) idx[k] = n0 + k;
      std::stable_sort(idx.begin(), idx.end(), [&](int p, int q) { return deg(p) > deg(q); });
      for (int k = 0; k < cnt; ++k) perm[n0 + k] = idx[k];
      for (int j = 0; j < kSellSlices; ++j) {
        int W = 0;
        for (int k = j * 32; k < std::min(cnt, j * 32 + 32); ++k) W = std::max(W, deg(idx[k]));
        sl_off.push_back(sl_off.back() + 32LL * W);
      }
      sb_sys.push_back(s);
      sb_n0.push_back(n0);
      sb_cnt.push_back(cnt);
      sb_rbu.push_back(sys_rb_off0[s] + i);
      sb_rbv.push_back(sys_rb_off0[s] + nbc + i);
    }
    S.h_sys_sb_off[s + 1] = (int)sb_sys.size();
  }
  bool ok = true;
  S.nsb = (int)sb_sys.size();
  S.slots = sl_off.back();
  S.sb_sys = upload(m, a, sb_sys, ok);
  S.sb_n0 = upload(m, a, sb_n0, ok);
  S.sb_cnt = upload(m, a, sb_cnt, ok);
  S.sb_rbu = upload(m, a, sb_rbu, ok);
  S.sb_rbv = upload(m, a, sb_rbv, ok);
  S.perm = upload(m, a, perm, ok);
  S.sl_off = upload(m, a, sl_off, ok);
  S.cols = (int*)dalloc(m, a, sizeof(int) * (size_t)S.slots, ok);
  S.spart = (double*)dalloc(m, a, sizeof(double) * kSellSlices * (size_t)std::max(S.nsb, 1), ok);
  std::vector<int> sl_pre(nsys + 1);
  for (int s = 0; s <= nsys; ++s) sl_pre[s] = kSellSlices * S.h_sys_sb_off[s];
  S.sys_sl_off = upload(m, a, sl_pre, ok);
  if (!ok) { S.failed = true; return set_error(UA_ERR_OOM, "node slices: device allocation failed"); }
  if (S.nsb)
    k_sell_fill<double><<<S.nsb, 256, 0, m->stream>>>(sell_dev(m, S), m->dm, nullptr, nullptr, nullptr, S.cols,
                                                       nullptr);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { S.failed = true; return set_error(UA_ERR_CUDA, "node slices: %s", cudaGetErrorString(e)); }
  S.ready = true;
  if (a->sa) csell_init(m);  // the coarse levels keep their CSR passes if this fails
  return UA_OK;
}

int amg_sell_fill(ua_mesh* m, const void* K0, bool fp32, bool lo, long long* launches, const int* sel) {
  Amg* a = m->amg;
  if (!a || !a->sell.ready) return UA_ERR_INVALID;
  Sell& S = a->sell;
  bool ok = true;
  const size_t nv = 4 * (size_t)S.slots;
  if (fp32 && !S.v32) S.v32 = (float*)dalloc(m, a, sizeof(float) * nv, ok);
  if (!fp32 && !S.v64) S.v64 = (double*)dalloc(m, a, sizeof(double) * nv, ok);
  if (lo && !S.vlo) S.vlo = (__nv_bfloat16*)dalloc(m, a, sizeof(__nv_bfloat16) * nv, ok);
  if (!ok) return set_error(UA_ERR_OOM, "node slices: device allocation of the values failed");
  if (!S.nsb) return UA_OK;
  if (fp32)
    k_sell_fill<float><<<S.nsb, 256, 0, m->stream>>>(sell_dev(m, S), m->dm, (const float*)K0, S.v32,
                                                      lo ? S.vlo : nullptr, nullptr, sel);
  else
    k_sell_fill<double><<<S.nsb, 256, 0, m->stream>>>(sell_dev(m, S), m->dm, (const double*)K0, S.v64,
                                                       lo ? S.vlo : nullptr, nullptr, sel);
  ++*launches;
  if (lo && fp32)  // the coarse operators of this Newton step's set-up (FP32) into their BF16 slices
    for (int l = 1; l < (int)a->csell.size(); ++l) {
      const Sell& C = a->csell[l];
      if (!C.ready || !C.nsb) continue;
      const AmgLevel& L = a->lev[l];
      k_csell_fill<float><<<C.nsb, 256, 0, m->stream>>>(csell_dev(m, C, L, l), L.rowptr, L.colind,
                                                       (const float*)L.A, C.vlo, nullptr, sel), ++*launches;
    }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(UA_ERR_CUDA, "node slices: %s", cudaGetErrorString(e));
  return UA_OK;
}

// Grid of a slice kernel: one slice block per CTA, or, list-driven, the CTAs resident at once
// (per-instantiation occupancy, so that no partial second wave trails the list loop).
template <typename KT, typename VT, int MODE>
static int sell_grid(const Amg* a, bool listed, int nsb = -1) {
  if (nsb < 0) nsb = a->sell.nsb;
  if (!listed) return nsb;
  static int occ = 0;
  if (!occ && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sell<KT, VT, MODE>, 256, 0) != cudaSuccess ||
               occ < 1))
    occ = 1;
  return std::max(1, std::min(nsb, occ * a->nsm));
}

void amg_sell_partials(const ua_mesh* m, const double** spart, const int** sys_sl_off) {
  *spart = m->amg->sell.spart;
  *sys_sl_off = m->amg->sell.sys_sl_off;
}

int amg_sell_spmv(ua_mesh* m, bool fp32, bool act, const int* sel, const int* done, const void* p,
                  const unsigned char* cmask, void* q, long long* launches) {
  Amg* a = m->amg;
  const Sell& S = a->sell;
  const bool useact = act && S.act.map;
  const ActList L = useact ? S.act : ActList{};
  if (!S.nsb) return UA_OK;
  if (fp32)
    launch_pdl(k_sell<float, float, 0>, sell_grid<float, float, 0>(a, useact), 256, 0, m->stream, sell_dev(m, S), S.nsb, L, sel, done, a->d_depth, S.v32,
                                                         (const float*)p, nullptr, nullptr, cmask, (float*)q,
                                                         nullptr, S.spart);
  else
    launch_pdl(k_sell<double, double, 0>, sell_grid<double, double, 0>(a, useact), 256, 0, m->stream, sell_dev(m, S), S.nsb, L, sel, done, a->d_depth, S.v64,
                                                           (const double*)p, nullptr, nullptr, cmask, (double*)q,
                                                           nullptr, S.spart);
  ++*launches;
  return UA_OK;
}

const void* amg_bf16_copy(ua_mesh* m, const float* K0, long long nnz, long long* launches) {
  Amg* a = m->amg;
  if (!a) return nullptr;
  if (!a->k0lo) {
    a->k0lo = (__nv_bfloat16*)dev_alloc(m, sizeof(__nv_bfloat16) * (size_t)std::max(nnz, 1LL));
    if (!a->k0lo) return nullptr;
    a->bytes += sizeof(__nv_bfloat16) * (size_t)nnz;
  }
  k_to_bf16<<<1184, 256, 0, m->stream>>>(nnz, K0, a->k0lo), ++*launches;
  return a->k0lo;
}

int amg_numeric(ua_mesh* m, const int* rowptr0, const int* colind0, const void* K0, bool fp32,
                const unsigned char* cmask, long long* launches, const int* sel, const std::vector<int>* h_sel,
                int p_refresh, bool graph) {
  // prolongators: recomputed for the selected systems on the first set-up of their solve and then
  // every p_refresh-th one (all of them when no host selection is given)
  Amg* a = m->amg;
  const int* psel = sel;
  if (a && a->sa && h_sel && p_refresh > 1) {
    const int ns = a->nsys;
    if ((int)a->p_age.size() != ns) a->p_age.assign(ns, 0);
    a->h_prefresh.assign(ns, 0);
    for (int s = 0; s < ns; ++s) {
      if (!(*h_sel)[s]) continue;
      a->h_prefresh[s] = a->p_age[s] % p_refresh == 0 ? 1 : 0;
      a->p_age[s] += 1;
    }
    bool ok = true;
    if (!a->d_prefresh) a->d_prefresh = (int*)dalloc(m, a, sizeof(int) * ns, ok);
    if (!ok) return set_error(UA_ERR_OOM, "AMG: device allocation failed");
    UA_CUDA_TRY(cudaMemcpyAsync(a->d_prefresh, a->h_prefresh.data(), sizeof(int) * ns, cudaMemcpyHostToDevice,
                                m->stream));
    UA_CUDA_TRY(cudaStreamSynchronize(m->stream));  // h_prefresh is rewritten by the next set-up
    psel = a->d_prefresh;
  }
  const int sm = (int)(sizeof(double) * (size_t)a->maxdn * 2 * a->maxdn);
  if (fp32)
    UA_CUDA_TRY(cudaFuncSetAttribute(k_amg_dense_inverse<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  else
    UA_CUDA_TRY(cudaFuncSetAttribute(k_amg_dense_inverse<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  if (a->sa) {  // the set-up's shared-memory rows, sized by the hierarchy's longest ones
    int smd = 0;
    for (int l = 0; l + 1 < a->nlev; ++l) smd = std::max(smd, a->lev[l].ac_maxdeg);
    const int sac = (int)sa_ac_smem(smd);
    const int sap = fp32 ? (int)sa_ap_smem<float>(kSaApSm) : (int)sa_ap_smem<double>(kSaApSm);
    if (fp32) {
      UA_CUDA_TRY(cudaFuncSetAttribute(k_sa_Ac<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sac));
      UA_CUDA_TRY(cudaFuncSetAttribute(k_sa_AP<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sap));
    } else {
      UA_CUDA_TRY(cudaFuncSetAttribute(k_sa_Ac<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, sac));
      UA_CUDA_TRY(cudaFuncSetAttribute(k_sa_AP<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, sap));
    }
  }
  if (a->sa) {  // the transfer quads of this precision, allocated before any capture
    bool ok = true;
    for (int l = 0; l + 1 < a->nlev; ++l) {
      AmgLevel& F = a->lev[l];
      void*& q = fp32 ? F.sa_qh : F.sa_qd;
      void*& qt = fp32 ? F.sa_qth : F.sa_qtd;
      const size_t qb = fp32 ? sizeof(PQuadH) : sizeof(PQuadD);
      if (!q) q = dalloc(m, a, qb * (size_t)std::max(F.np, 1LL), ok);
      if (!qt) qt = dalloc(m, a, qb * (size_t)std::max(F.np, 1LL), ok);
    }
    if (!ok) return set_error(UA_ERR_OOM, "AMG: device allocation of the transfer values failed");
  }
  auto run = [&](long long* l) {
    return fp32 ? numeric_t<float, float>(m, rowptr0, colind0, (const float*)K0, cmask, sel, psel, l)
                : numeric_t<double, double>(m, rowptr0, colind0, (const double*)K0, cmask, sel, psel, l);
  };
  if (!graph) return run(launches);
  // one captured graph per kind of call (FP32/FP64 values, prolongator selection, handle's
  // selection), replayed at every later Newton step
  const int key = (fp32 ? 1 : 0) + (psel == a->d_prefresh && psel ? 2 : 0) + (sel ? 4 : 0);
  if (!a->setup_exec[key]) {
    long long n = 0;
    cudaGraph_t gr = nullptr;
    UA_CUDA_TRY(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
    int rc = run(&n);
    cudaError_t ce = cudaStreamEndCapture(m->stream, &gr);
    if (rc) { if (gr) cudaGraphDestroy(gr); return rc; }
    if (ce != cudaSuccess) return set_error(UA_ERR_CUDA, "AMG set-up graph capture: %s", cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&a->setup_exec[key], gr, 0);
    cudaGraphDestroy(gr);
    if (ce != cudaSuccess) return set_error(UA_ERR_CUDA, "AMG set-up graph: %s", cudaGetErrorString(ce));
    a->setup_nodes[key] = n;
  }
  UA_CUDA_TRY(cudaGraphLaunch(a->setup_exec[key], m->stream));
  *launches += a->setup_nodes[key];
  return UA_OK;
}

void amg_restart_P(ua_mesh* m, const std::vector<int>& run) {
  Amg* a = m->amg;
  if (!a) return;
  if ((int)a->p_age.size() != a->nsys) a->p_age.assign(a->nsys, 0);
  for (int s = 0; s < a->nsys && s < (int)run.size(); ++s)
    if (run[s]) a->p_age[s] = 0;
}

// the transfer quads of the vector precision
template <typename VT>
static const typename PQuadOf<VT>::T* sa_quads(void* qd, void* qh) {
  return (const typename PQuadOf<VT>::T*)(std::is_same<VT, float>::value ? qh : qd);
}

// Finest-level residual (MODE 1: W = mask(r - K x0)) or smoothing (MODE 2: z = mask(x + invd (r - K x)),
// pcopy, partials r.z) over the node slices, with BF16 values when v.sell_lo.
template <typename KT, typename VT, int MODE>
static void sell_pass(ua_mesh* m, const AmgPcgView& v, bool useact, const VT* invd, VT* out) {
  Amg* a = m->amg;
  const Sell& S = a->sell;
  if (!S.nsb) return;
  const bool la = useact && S.act.map;
  const ActList L = la ? S.act : ActList{};
  const VT* x = (const VT*)v.x0;
  VT* pcopy = MODE == 2 ? (VT*)v.pcopy : nullptr;
  double* part = MODE == 2 ? S.spart : nullptr;
  const VT* b = (const VT*)v.r;
  const KT* vk = nullptr;
  if constexpr (std::is_same<KT, float>::value) vk = S.v32;
  else vk = S.v64;
  if (v.sell_lo)
    launch_pdl(k_sell<__nv_bfloat16, VT, MODE>, sell_grid<__nv_bfloat16, VT, MODE>(a, la), 256, 0, m->stream, sell_dev(m, S), S.nsb, L, v.sel, v.done, a->d_depth,
                                                                 S.vlo, x, b, invd, v.cmask, out, pcopy, part);
  else
    launch_pdl(k_sell<KT, VT, MODE>, sell_grid<KT, VT, MODE>(a, la), 256, 0, m->stream, sell_dev(m, S), S.nsb, L, v.sel, v.done, a->d_depth, vk, x, b,
                                                      invd, v.cmask, out, pcopy, part);
}

// Coarse-level residual (MODE 1) or smoothing (MODE 2, no partials) over level l's BF16 node slices.
template <typename VT, int MODE>
static void csell_pass(ua_mesh* m, const AmgPcgView& v, int l, bool useact, const VT* x, const VT* b,
                       const VT* invd, VT* out) {
  Amg* a = m->amg;
  const Sell& S = a->csell[l];
  if (!S.nsb) return;
  const bool la = useact && S.act.map;
  const ActList L = la ? S.act : ActList{};
  launch_pdl(k_sell<__nv_bfloat16, VT, MODE>, sell_grid<__nv_bfloat16, VT, MODE>(a, la, S.nsb), 256, 0, m->stream, csell_dev(m, S, a->lev[l], l), S.nsb, L, v.sel, v.done, a->d_depth, S.vlo, x, b, invd, nullptr, out, nullptr,
      nullptr);
}

template <typename KT, typename VT>
static int vcycle_t(ua_mesh* m, const AmgPcgView& v, long long* launches) {
  Amg* a = m->amg;
  cudaStream_t st = m->stream;
  const int nl = a->nlev;
  // per level l: row blocks, matrix, rhs b, pre-smoothed x, residual / post-smoothed buffer
  auto rbs = [&](int l) { return l == 0 ? v.rb_start0 : a->lev[l].rb_start; };
  auto rbsys = [&](int l) { return l == 0 ? v.rb_sys0 : a->lev[l].rb_sys; };
  auto nrb = [&](int l) { return l == 0 ? v.nrb0 : a->lev[l].nrb; };
  auto rp = [&](int l) { return l == 0 ? v.rowptr0 : a->lev[l].rowptr; };
  auto ci = [&](int l) { return l == 0 ? v.colind0 : a->lev[l].colind; };
  auto A = [&](int l) { return l == 0 ? (const KT*)v.K0 : (const KT*)a->lev[l].A; };
  auto B = [&](int l) { return l == 0 ? (const VT*)v.r : (const VT*)a->lev[l].b; };
  auto X = [&](int l) { return l == 0 ? (VT*)v.x0 : (VT*)a->lev[l].x; };
  auto W = [&](int l) { return l == 0 ? (VT*)v.tmp : (VT*)a->lev[l].x2; };
  auto mask = [&](int l) { return l == 0 ? v.cmask : nullptr; };
  auto doff = [&](int l) { return (const int*)a->lev[l].d_dof_off; };
  const int lpr0 = v.lpr, lprc = a->sa ? kSaLPR : 1;  // lanes per row: finest level, coarse levels
  // list-driven launches (the PCG of a uv handle): a grid of about one wave over the active blocks
  const bool useact = v.act && a->act_ready;
  auto rows_act = [&](int l) { return useact ? a->rows[l] : ActList{}; };
  auto rows_grid = [&](int l) { return useact ? act_grid(nrb(l), a->nsm) : nrb(l); };
  // coarse levels on BF16 node slices: the mixed-precision cycle with node slices at the finest level
  auto cslices = [&](int l) { return v.sell && v.sell_lo && l < (int)a->csell.size() && a->csell[l].ready; };
  for (int l = 0; l + 1 < nl; ++l) {  // down: residual of level l, aggregated into level l+1
    const AmgLevel& C = a->lev[l + 1];
    if (l == 0 && v.mark) v.mark(v.mark_ctx, 0, 0);
    if (l == 0 && v.sell)
      sell_pass<KT, VT, 1>(m, v, useact, (const VT*)nullptr, W(0));
    else if (l > 0 && cslices(l))
      csell_pass<VT, 1>(m, v, l, useact, X(l), B(l), nullptr, W(l));
    else
    dispatch_lpr(l == 0 ? lpr0 : lprc, [&](auto L) {
      if (l == 0 && v.K0lo)
        launch_pdl(k_amg_residual<__nv_bfloat16, VT, decltype(L)::value>, rows_grid(l), 256, 0, st, rbs(l), rbsys(l), rows_act(l), v.sel, v.done, a->d_depth, l, rp(l), ci(l), (const __nv_bfloat16*)v.K0lo, B(l), X(l),
            mask(l), W(l), doff(l));
      else
        launch_pdl(k_amg_residual<KT, VT, decltype(L)::value>, rows_grid(l), 256, 0, st, rbs(l), rbsys(l), rows_act(l), v.sel, v.done, a->d_depth, l, rp(l), ci(l), A(l), B(l), X(l), mask(l), W(l), doff(l));
    });
    ++*launches;
    if (l == 0 && v.mark) v.mark(v.mark_ctx, 0, 1);
    const AmgLevel& F = a->lev[l];
    if (a->sa)
      launch_pdl(k_sa_restrict<VT>, useact ? act_grid(C.nnb, a->nsm) : C.nnb, 256, 0, st, C.nb_start, C.nb_sys, useact ? a->cnodes[l] : ActList{}, C.d_dof_off, C.d_node_off, a->d_depth, l + 1,
          v.sel, v.done, F.ptn_ptr, F.ptn_fine, sa_quads<VT>(F.sa_qtd, F.sa_qth), F.d_dof_off, F.d_node_off, W(l), (const VT*)C.invd, (VT*)C.b, (VT*)C.x), ++*launches;
    else
      k_amg_gather<VT><<<(C.ndof + 127) / 128, 128, 0, st>>>(C.ndof, C.dof_sys, a->d_depth, l + 1, v.sel, v.done,
                                                             C.mptr, C.mlist, W(l), (const VT*)C.invd, (VT*)C.b,
                                                             (VT*)C.x), ++*launches;
  }
  launch_pdl(k_amg_dense_apply<VT>, dim3(a->nsys, (a->maxdn + 31) / 32), 256, 0, st, v.sel, v.done, a->d_depth, a->d_dn, a->d_doff, a->d_lev_dofoff, a->d_lev_b, a->d_lev_x2, a->dense), ++*launches;
  for (int l = nl - 2; l >= 0; --l) {  // up: correction from level l+1's post-smoothed x2, then smoothing
    const AmgLevel& F = a->lev[l];
    const AmgLevel& C = a->lev[l + 1];
    if (a->sa)
      launch_pdl(k_sa_prolong<VT>, useact ? act_grid((F.nnb + kSaPW - 1) / kSaPW, a->nsm) : (F.nnb + kSaPW - 1) / kSaPW, 32 * kSaPW, 0, st, F.nnb, F.nb_start, F.nb_sys, useact ? a->fnodes[l] : ActList{}, F.d_dof_off, F.d_node_off, a->d_depth, l,
          v.sel, v.done, F.pn_ptr, F.pn_col, sa_quads<VT>(F.sa_qd, F.sa_qh), C.d_dof_off,
          C.d_node_off, (const VT*)C.x2, X(l)), ++*launches;
    else
      k_amg_correct<VT><<<nrb(l), 256, 0, st>>>(rbs(l), rbsys(l), v.sel, v.done, a->d_depth, l, X(l),
                                                (const VT*)C.x2, F.cmap, mask(l)), ++*launches;
    VT* out = l == 0 ? (VT*)v.z : (VT*)F.x2;
    VT* pcopy = l == 0 ? (VT*)v.pcopy : nullptr;
    double* part = l == 0 ? v.part_rz : nullptr;
    if (l == 0 && v.mark) v.mark(v.mark_ctx, 1, 0);
    if (l == 0 && v.sell)
      sell_pass<KT, VT, 2>(m, v, useact, (const VT*)F.invd, out);
    else if (l > 0 && cslices(l))
      csell_pass<VT, 2>(m, v, l, useact, X(l), B(l), (const VT*)F.invd, out);
    else
    dispatch_lpr(l == 0 ? lpr0 : lprc, [&](auto L) {
      if (l == 0 && v.K0lo)
        launch_pdl(k_amg_smooth<__nv_bfloat16, VT, decltype(L)::value>, rows_grid(l), 256, 0, st, rbs(l), rbsys(l), rows_act(l), v.sel, v.done, a->d_depth, l, rp(l), ci(l), (const __nv_bfloat16*)v.K0lo, B(l), X(l),
            (const VT*)F.invd, mask(l), out, pcopy, part, doff(l));
      else
        launch_pdl(k_amg_smooth<KT, VT, decltype(L)::value>, rows_grid(l), 256, 0, st, rbs(l), rbsys(l), rows_act(l), v.sel, v.done, a->d_depth, l, rp(l), ci(l), A(l), B(l), X(l), (const VT*)F.invd,
            mask(l), out, pcopy, part, doff(l));
    });
    ++*launches;
    if (l == 0 && v.mark) v.mark(v.mark_ctx, 1, 1);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(UA_ERR_CUDA, "AMG V-cycle: %s", cudaGetErrorString(e));
  return UA_OK;
}

int amg_vcycle(ua_mesh* m, bool fp32, const AmgPcgView& v, long long* launches) {
  if (fp32) return vcycle_t<float, float>(m, v, launches);
  return vcycle_t<double, double>(m, v, launches);
}

// ---------------------------------------------------------------------------
// uvh: block preconditioner, AMG on the velocity block
// ---------------------------------------------------------------------------

// 3-dof row (c, g) of a uvh tangent holds blocks b = u, v, h of deg(g)
// entries; its u and v blocks are the velocity block's row (c, g), c < 2.
// One thread per velocity row copies them, and the row's constraint mask.
__global__ void k_uvh_extract(const DevMesh dm, int n2, const int* dof_sys2, const int* dof2_off, const int* knz2_off,
                              const double* K3, const unsigned char* cmask3, double* K2, unsigned char* cmask2) {
  const int i2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (i2 >= n2) return;
  const int s = dof_sys2[i2];
  const int no = dm.sys_node_off[s], nn = dm.sys_node_off[s + 1] - no;
  const int local = i2 - dof2_off[s], c = local / nn, gl = local - c * nn;
  const int g = no + gl;
  const int np0 = dm.nodeptr[g], deg = dm.nodeptr[g + 1] - np0, lp = np0 - dm.nodeptr[no];
  const double* src = K3 + dm.sys_knz_off[s] + (size_t)c * 3 * dm.sys_nnzn[s] + 3 * (size_t)lp;
  double* dst = K2 + knz2_off[s] + (size_t)c * 2 * dm.sys_nnzn[s] + 2 * (size_t)lp;
  for (int k = 0; k < 2 * deg; ++k) dst[k] = src[k];
  cmask2[i2] = cmask3[dm.sys_dof_off[s] + local];
}

// r2 = mask(p3 on the velocity rows), x0 = l1-Jacobi of r2 (pre-smoothing).
__global__ void k_uvh_gather(const DevMesh dm, int n2, const int* dof_sys2, const int* dof2_off, const int* sel,
                             const int* done, const unsigned char* cmask2, const double* p3, const double* invd2,
                             double* r2, double* x0) {
  const int i2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (i2 >= n2) return;
  const int s = dof_sys2[i2];
  if (!sel[s] || done[s]) return;
  const double v = cmask2[i2] ? 0.0 : p3[dm.sys_dof_off[s] + (i2 - dof2_off[s])];
  r2[i2] = v;
  x0[i2] = invd2[i2] * v;
}

__global__ void k_uvh_scatter(const DevMesh dm, int n2, const int* dof_sys2, const int* dof2_off, const int* sel,
                              const int* done, const double* z2, double* out3) {
  const int i2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (i2 >= n2) return;
  const int s = dof_sys2[i2];
  if (!sel[s] || done[s]) return;
  out3[dm.sys_dof_off[s] + (i2 - dof2_off[s])] = z2[i2];
}

int amg_numeric_uvh(ua_mesh* m, const double* K3, const unsigned char* cmask3, long long* launches) {
  Amg* a = m->amg;
  if (!a || m->ndof != 3) return set_error(UA_ERR_INVALID, "no uvh AMG hierarchy");
  AmgLevel& F = a->lev[0];
  k_uvh_extract<<<(F.ndof + 255) / 256, 256, 0, m->stream>>>(m->dm, F.ndof, F.dof_sys, F.d_dof_off, F.d_knz_off,
                                                             K3, cmask3, (double*)F.A, a->uvh_mask), ++*launches;
  return amg_numeric(m, F.rowptr, F.colind, F.A, false, a->uvh_mask, launches);
}

int amg_apply_uvh(ua_mesh* m, const double* p3, double* out3, const int* sel, const int* done, int lpr,
                  long long* launches) {
  Amg* a = m->amg;
  AmgLevel& F = a->lev[0];
  const int nb = (F.ndof + 255) / 256;
  k_uvh_gather<<<nb, 256, 0, m->stream>>>(m->dm, F.ndof, F.dof_sys, F.d_dof_off, sel, done, a->uvh_mask, p3,
                                          (const double*)F.invd, a->uvh_r, a->uvh_x0), ++*launches;
  AmgPcgView v{F.rowptr, F.colind, F.A, a->uvh_r, a->uvh_x0, a->uvh_z, nullptr, nullptr, a->uvh_mask, sel, done,
               F.rb_start, F.rb_sys, F.nrb, lpr, a->uvh_t};
  int rc = vcycle_t<double, double>(m, v, launches);
  if (rc) return rc;
  k_uvh_scatter<<<nb, 256, 0, m->stream>>>(m->dm, F.ndof, F.dof_sys, F.d_dof_off, sel, done, a->uvh_z, out3),
      ++*launches;
  return UA_OK;
}

// ---------------------------------------------------------------------------
// active-block lists
// ---------------------------------------------------------------------------

int act_grid(int nblocks, int nsm) { return std::max(1, std::min(nblocks, 8 * nsm)); }

// exclusive block-wide scan of v (blockDim.x a multiple of 32, at most 1024); total = sum
__device__ int block_excl_scan(int v, int* sh, int& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int t = lane < nw ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    sh[lane] = t;
  }
  __syncthreads();
  const int pre = wid ? sh[wid - 1] : 0;
  total = sh[nw - 1];
  __syncthreads();  // sh is reused by the next call
  return pre + x - v;
}

// one CTA per list: scan the systems in order (a chunk of blockDim.x systems at a time), then
// one warp per active system writes its block ids, the lanes striding over them
__global__ void __launch_bounds__(1024) k_act_compact(const ActSpec* specs, int nsys, const int* sel,
                                                      const int* done, const int* depth) {
  pdl_enter();
  __shared__ int sh[32];
  __shared__ int s_ex[1024], s_n[1024], s_b0[1024];
  const ActSpec sp = specs[blockIdx.x];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int base = 0;
  for (int c0 = 0; c0 < nsys; c0 += blockDim.x) {  // same trip count for every thread
    const int s = c0 + threadIdx.x;
    int n = 0, b0 = 0;
    if (s < nsys && sel[s] && !done[s] && depth[s] > sp.lmin) {
      b0 = sp.blk_off[s];
      n = sp.blk_off[s + 1] - b0;
    }
    int tot;
    const int ex = block_excl_scan(n, sh, tot);
    s_ex[threadIdx.x] = ex;
    s_n[threadIdx.x] = n;
    s_b0[threadIdx.x] = b0;
    __syncthreads();
    const int cn = min((int)blockDim.x, nsys - c0);
    for (int t = wid; t < cn; t += nw) {
      const int nt = s_n[t], et = base + s_ex[t], bt = s_b0[t];
      for (int k = lane; k < nt; k += 32) sp.map[et + k] = bt + k;
    }
    __syncthreads();  // the shared arrays are rewritten by the next chunk
    base += tot;
  }
  if (threadIdx.x == 0) *sp.cnt = base;
}

int amg_act_init(ua_mesh* m, const std::vector<int>& sys_rb_off0) {
  Amg* a = m->amg;
  if (!a) return UA_ERR_INVALID;
  if (a->act_ready) return UA_OK;
  const int nsys = a->nsys;
  if ((int)sys_rb_off0.size() != nsys + 1) return set_error(UA_ERR_INVALID, "active lists: row-block prefix size");
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&a->nsm, cudaDevAttrMultiProcessorCount, dev);
  bool ok = true;
  std::vector<ActSpec> specs;
  auto make = [&](const std::vector<int>& off, int lmin) {
    ActList L;
    L.cap = off[nsys];
    int* map = (int*)dalloc(m, a, sizeof(int) * (size_t)std::max(L.cap, 1), ok);
    int* cnt = (int*)dalloc(m, a, sizeof(int), ok);
    int* doff = upload(m, a, off, ok);
    L.map = map;
    L.cnt = cnt;
    specs.push_back(ActSpec{doff, lmin, map, cnt});
    return L;
  };
  const int nl = a->nlev;
  a->rows.resize(std::max(nl - 1, 1));
  a->fnodes.resize(std::max(nl - 1, 0));
  a->cnodes.resize(std::max(nl - 1, 0));
  a->rows[0] = make(sys_rb_off0, -1);  // the handle's Krylov rows: every active system
  for (int l = 1; l + 1 < nl; ++l) a->rows[l] = make(a->lev[l].h_sys_rb_off, l);
  if (a->sa)
    for (int l = 0; l + 1 < nl; ++l) {
      a->fnodes[l] = make(a->lev[l].h_sys_nb_off, l);
      a->cnodes[l] = make(a->lev[l + 1].h_sys_nb_off, l);
    }
  if (a->sell.ready) a->sell.act = make(a->sell.h_sys_sb_off, -1);  // node slice blocks: every active system
  for (int l = 1; l < (int)a->csell.size(); ++l)
    if (a->csell[l].ready) a->csell[l].act = make(a->csell[l].h_sys_sb_off, l);  // depth > l
  a->d_specs = upload(m, a, specs, ok);
  a->nspecs = (int)specs.size();
  if (!ok) return set_error(UA_ERR_OOM, "active lists: device allocation failed");
  a->act_ready = true;
  return UA_OK;
}

void amg_act_compact(ua_mesh* m, const int* sel, const int* done, long long* launches) {
  Amg* a = m->amg;
  launch_pdl(k_act_compact, a->nspecs, 1024, 0, m->stream, a->d_specs, a->nsys, sel, done, a->d_depth), ++*launches;
}

ActList amg_act_rows0(const ua_mesh* m) { return m->amg && m->amg->act_ready ? m->amg->rows[0] : ActList{}; }

}  // namespace ua
