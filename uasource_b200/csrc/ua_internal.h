// Internal structures of libuassa: device layout of the resident mesh
// ("MUA" of Úa, CreateMUA.m) extended with the symbolic scatter plan.
//
// Layout in HBM (all systems of a handle concatenated, system-major):
//   nodes      : global node id g = node_off[s] + local node i
//   elements   : conn[a*ne_total + e] (SoA, element fastest) = global node id
//   dofs       : dof_off[s] + c*nn_s + i   (c = 0:u, 1:v, 2:h), Úa ordering
//   tangent    : CSR over dofs.  Row (c,g) of system s starts at
//                knz_off[s] + c*ndof*NNZn_s + ndof*(nodeptr[g]-nodeptr[node_off[s]])
//                and holds ndof blocks of deg(g) columns (block b, k-th neighbour).
//   scatter    : node patches.  A patch is a set of nodes of one system plus
//                every element touching them.  The assembly kernel computes
//                the patch's element tangents into shared memory, then sums
//                them per node-level non-zero through the precomputed
//                contribution list (element-local id, local row node,
//                local col node), in increasing global element order: a
//                deterministic segmented sum with no atomics whose result does
//                not depend on the patch partition.
#pragma once
#include <cstdint>
#include <vector>
#include <string>
#include <cuda_runtime.h>
#include "../../include/ua_ssa.h"

namespace ua {

// Programmatic dependent launch for the short kernels of a PCG step: launched with
// launch_pdl, a kernel may be scheduled while the kernel before it on the stream drains; it
// first calls pdl_enter, which waits for that kernel's completion and memory (a no-op for an
// ordinary launch) and then lets the next kernel be scheduled in turn.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <typename... P, typename... A>
inline cudaError_t launch_pdl(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... a) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, static_cast<A&&>(a)...);
}

constexpr int kMaxNip = 16;
constexpr int kMaxNod = 6;

// contribution packing: element-local id (10 bits) | row node a (3) | col node b (3)
__host__ __device__ inline uint16_t pack_contrib(int el, int a, int b) {
  return (uint16_t)((el << 6) | (a << 3) | b);
}

// Bounds checks of the debug build (`make debug`, -DUA_BOUNDS_CHECK): an index outside [lo, hi)
// records the check site and the index in the handle's flag (the first one wins), is replaced by
// lo and marks the access invalid (ok = false), so nothing is read or written out of range.  The
// release build compiles them out.
#ifdef UA_BOUNDS_CHECK
__device__ inline bool in_bounds(unsigned long long* dbg, long long i, long long lo, long long hi, int site) {
  if (i >= lo && i < hi) return true;
  if (dbg) atomicCAS(dbg, 0ULL, ((unsigned long long)(site & 0xffff) << 48) | ((unsigned long long)i & 0xffffffffffffULL));
  return false;
}
#define UA_CHECK_INDEX(dbg, i, lo, hi, site, ok)                                               \
  do {                                                                                         \
    if (!ua::in_bounds((dbg), (long long)(i), (long long)(lo), (long long)(hi), (site))) {     \
      (i) = (lo);                                                                              \
      (ok) = false;                                                                            \
    }                                                                                          \
  } while (0)
#else
#define UA_CHECK_INDEX(dbg, i, lo, hi, site, ok) \
  do {                                          \
  } while (0)
#endif
// check sites (bits 48-63 of the recorded flag)
enum BoundsSite {
  BS_PATCH_ELEM = 1, BS_ELEM_NODE = 2, BS_CONTRIB_ELEM = 3, BS_K_INDEX = 4, BS_R_INDEX = 5, BS_SELL_COL = 6
};

struct QuadTable {
  int nip;
  double w[kMaxNip];
  double fun[kMaxNip][kMaxNod];
  double der[kMaxNip][2][kMaxNod];
};

// Device view of a handle (passed to kernels by value).
struct DevMesh {
  int nsys, nn, ne, nod, nip, ndof;
  const int* conn;            // [nod][ne]
  const double* x;            // [nn]
  const double* y;            // [nn]
  const int* nodeptr;         // node-level CSR [nn+1] (global)
  const int* nodecol;         // node-level columns (global node ids)
  const int* node_sys;        // [nn]
  // per system
  const int* sys_node_off;    // [nsys+1]
  const int* sys_dof_off;     // [nsys+1]
  const int* sys_knz_off;     // [nsys+1] (dof-level nnz offset)
  const int* sys_nnzn;        // [nsys]  node-level nnz of the system
  // patches
  int npatch;
  const int* patch_sys;       // [npatch]
  const int* patch_node_ptr;  // [npatch+1]
  const int* patch_nodes;     // global node ids
  const int* patch_elem_ptr;  // [npatch+1]
  const int* patch_elems;     // global element ids (sorted)
  const int* patch_q_ptr;     // [npatch+1] into pq arrays
  const uint32_t* pq_rk;      // (local row << 16) | k
  const int* pq_cptr;         // [total_pq+1] into contrib
  const uint16_t* contrib;
  const int* prow_diag;       // per patch row (aligned with patch_nodes): pq index of diagonal
  int max_patch_elems;
  // the nodes of each patch's elements (its rows and their halo), sorted, and per patch element
  // the patch-local index of each of its nodes (element-local order), for staging node data
  const int* patch_hnode_ptr; // [npatch+1]
  const int* patch_hnodes;    // global node ids
  const uint16_t* patch_elnodes;  // [patch element][nod], aligned with patch_elems
  int max_patch_hnodes;
  unsigned long long* dbg;    // first bounds violation (debug build; null otherwise)
};

// Patch shape: the nodes of a system of nn nodes are cut, in Morton order, into patches of
// pn = clamp(nn / div, 16, cap) nodes (and at most the shared-memory element budget), so that
// a small mesh still gives enough patches to fill the SMs and a large one gets patches of cap
// nodes.  div = 0 means pn = cap for every system.
struct PatchShape {
  int div = 600;
  int cap = 128;
};

// The assembly schedule ua_autotune picks per (device, element type, dofs per node): the patch
// shape, the CTA size of the P1 kernel (128 or 256 threads) and its register budget.
struct AsmTuning {
  PatchShape shape;
  int threads = 256;
  int regs = 128;  // register budget of the P1 kernel: 128, 96 (128-thread CTAs) or 80
};

// Host-side mirror plus ownership of device buffers.
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
};

struct HostSystem {
  int nn = 0, ne = 0;
  std::vector<double> x, y;        // coordinates
  std::vector<int> conn;           // [nod][ne] local node ids (0-based)
  int nflipped = 0;
};

struct Constraints {
  // constraint matrix L (scaled rows), CSR by constraint row over global dofs
  int nc = 0;                      // total over systems
  std::vector<int> sys_c_off;      // [nsys+1]
  std::vector<int> rowptr;         // [nc+1]
  std::vector<int> col;            // global dof
  std::vector<double> val;
  std::vector<double> rhs;         // c (scaled)
  bool mask_only = true;           // every row has exactly one entry
};

struct Work;
struct Amg;

}  // namespace ua

struct ua_mesh {
  int device = 0;
  int ndof = 2;
  int nod = 3;
  int nip = 6;
  cudaStream_t stream = nullptr;
  std::vector<ua::HostSystem> sys;
  // host copies of symbolic data needed on the host
  std::vector<int> h_node_off, h_dof_off, h_knz_off, h_nnzn, h_elem_off;
  std::vector<int> h_nodeptr, h_nodecol;
  int nn_total = 0, ne_total = 0, ndof_total = 0;
  long long nnz_total = 0;
  ua::DevMesh dm{};
  std::vector<ua::DeviceBuffer> owned;
  size_t device_bytes = 0;
  // reusable work buffers
  ua::Work* work = nullptr;
  // aggregation AMG hierarchy of the uv tangent (built on first use)
  ua::Amg* amg = nullptr;
  bool amg_failed = false;
  // the caller reads the tangent back after a Newton solve (ua_uv_newton with Kvals): the
  // tangent must stay the one of the last Newton system, so no tangent is assembled ahead
  bool keep_last_tangent = false;
  // the shape of the current patch plan and the CTA size of the P1 assembly
  ua::PatchShape patch_shape;
  int asm_threads = 256;
  int asm_regs = 128;
};

namespace ua {
// allocation helpers (record ownership in the mesh)
void* dev_alloc(ua_mesh* m, size_t bytes);
void dev_free(ua_mesh* m, const void* p);
void dev_free_all(ua_mesh* m);
// rebuilds the patch plan of a handle with another shape (the results do not depend on it)
int rebuild_patches(ua_mesh* m, PatchShape shape);
// the process-wide tuning for (device, nod, ndof), set by ua_autotune; the default if none
AsmTuning tuned_assembly(int device, int nod, int ndof, bool* tuned = nullptr);
void set_tuned_assembly(int device, int nod, int ndof, AsmTuning t);
int set_error(int code, const char* fmt, ...);
const QuadTable& quad_table(int nod);
}  // namespace ua

#define UA_CUDA_TRY(call)                                                        \
  do {                                                                            \
    cudaError_t _e = (call);                                                      \
    if (_e != cudaSuccess)                                                        \
      return ua::set_error(UA_ERR_CUDA, "%s failed: %s (%s:%d)", #call,           \
                           cudaGetErrorString(_e), __FILE__, __LINE__);           \
  } while (0)
