// Mesh handle: CreateMUA.m:31-98 restated for the device, plus the symbolic
// scatter plan (node patches, CSR pattern, contribution lists).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <tuple>
#include "ua_internal.h"

namespace ua {

static thread_local char g_err[1024] = "";

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

const char* last_error_message() { return g_err; }

void* dev_alloc(ua_mesh* m, size_t bytes) {
  if (bytes == 0) bytes = 16;
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  m->owned.push_back({p, bytes});
  m->device_bytes += bytes;
  return p;
}

void dev_free(ua_mesh* m, const void* p) {
  if (!p) return;
  for (size_t i = 0; i < m->owned.size(); ++i)
    if (m->owned[i].ptr == p) {
      cudaFree(m->owned[i].ptr);
      m->device_bytes -= m->owned[i].bytes;
      m->owned.erase(m->owned.begin() + i);
      return;
    }
}

void dev_free_all(ua_mesh* m) {
  for (auto& b : m->owned) cudaFree(b.ptr);
  m->owned.clear();
  m->device_bytes = 0;
}

// ---------------------------------------------------------------------------
// Quadrature tables: quadtriangle.m nonproduct PI rules of degree 4 (6 points,
// :505-516) and degree 8 (16 points, :725-745), expanded over their symmetry
// orbits onto the domain [0 0;1 0;0 1] as quadTrianglePointsAndWeights does
// (:3674-3750): barycentric (b1,b2,b3) -> (x,y) = (b2,b3), weight = w/2.
// Shape functions shape_fun.m:52-71 and derivatives shape_der.m:54-98.
// ---------------------------------------------------------------------------
static void orbit(int mult, double p, double q, double w, std::vector<double>& X, std::vector<double>& Y,
                  std::vector<double>& W) {
  if (mult == 1) q = p;
  double r = 1.0 - (p + q);
  double o[6][3] = {{p, q, r}, {q, r, p}, {r, p, q}, {p, r, q}, {q, p, r}, {r, q, p}};
  for (int i = 0; i < mult; ++i) {
    X.push_back(o[i][1]);
    Y.push_back(o[i][2]);
    W.push_back(0.5 * w);
  }
}

static void shape(int nod, double c1, double c2, double* fun, double (*der)[kMaxNod]) {
  double c3 = 1.0 - c1 - c2;
  if (nod == 3) {
    fun[0] = c1; fun[1] = c3; fun[2] = c2;
    der[0][0] = 1; der[0][1] = -1; der[0][2] = 0;
    der[1][0] = 0; der[1][1] = -1; der[1][2] = 1;
  } else {
    fun[0] = (2 * c1 - 1) * c1; fun[1] = 4 * c3 * c1; fun[2] = (2 * c3 - 1) * c3;
    fun[3] = 4 * c2 * c3;       fun[4] = (2 * c2 - 1) * c2; fun[5] = 4 * c1 * c2;
    der[0][0] = 4 * c1 - 1; der[0][1] = 4 * (c3 - c1); der[0][2] = -(4 * c3 - 1);
    der[0][3] = -4 * c2;    der[0][4] = 0;             der[0][5] = 4 * c2;
    der[1][0] = 0;          der[1][1] = -4 * c1;       der[1][2] = -(4 * c3 - 1);
    der[1][3] = 4 * (c3 - c2); der[1][4] = 4 * c2 - 1; der[1][5] = 4 * c1;
  }
}

static QuadTable make_table(int nod) {
  QuadTable t{};
  std::vector<double> X, Y, W;
  if (nod == 3) {
    double s = std::sqrt(38.0 - 44.0 * std::sqrt(2.0 / 5.0));
    double b1 = (8.0 - std::sqrt(10.0) + s) / 18.0, b2 = (8.0 - std::sqrt(10.0) - s) / 18.0;
    double tt = std::sqrt(213125.0 - 53320.0 * std::sqrt(10.0));
    orbit(3, b1, b1, (620.0 + tt) / 3720.0, X, Y, W);
    orbit(3, b2, b2, (620.0 - tt) / 3720.0, X, Y, W);
  } else {
    const double b1[5] = {0.3333333333333333333333333333333333, 0.1705693077517602066222935014914645,
                          0.0505472283170309754584235505965989, 0.4592925882927231560288155144941693,
                          0.2631128296346381134217857862846436};
    const double b2_5 = 0.0083947774099576053372138345392944;
    const double w[5] = {0.1443156076777871682510911104890646, 0.1032173705347182502817915502921290,
                         0.0324584976231980803109259283417806, 0.0950916342672846247938961043885843,
                         0.0272303141744349942648446900739089};
    const int mult[5] = {1, 3, 3, 3, 6};
    for (int i = 0; i < 5; ++i) orbit(mult[i], b1[i], i == 4 ? b2_5 : b1[i], w[i], X, Y, W);
  }
  t.nip = (int)X.size();
  for (int i = 0; i < t.nip; ++i) {
    t.w[i] = W[i];
    shape(nod, X[i], Y[i], t.fun[i], t.der[i]);
  }
  return t;
}

const QuadTable& quad_table(int nod) {
  static QuadTable t3 = make_table(3);
  static QuadTable t6 = make_table(6);
  return nod == 3 ? t3 : t6;
}

// Morton code of 16-bit quantised coordinates.
static uint32_t spread16(uint32_t v) {
  v &= 0xffff;
  v = (v | (v << 8)) & 0x00FF00FF;
  v = (v | (v << 4)) & 0x0F0F0F0F;
  v = (v | (v << 2)) & 0x33333333;
  v = (v | (v << 1)) & 0x55555555;
  return v;
}

}  // namespace ua

using namespace ua;

static int upload(ua_mesh* m, const void* h, size_t bytes, void** d) {
  *d = dev_alloc(m, bytes);
  if (!*d) return set_error(UA_ERR_OOM, "device allocation of %zu bytes failed", bytes);
  if (bytes) UA_CUDA_TRY(cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice));
  return UA_OK;
}

template <class T>
static int upload_vec(ua_mesh* m, const std::vector<T>& v, const T** d) {
  void* p = nullptr;
  int rc = upload(m, v.data(), v.size() * sizeof(T), &p);
  *d = (const T*)p;
  return rc;
}

// Shared-memory bytes of one element in the assembly kernel (symmetric uu/vv
// blocks, full uv block, and Tx,Fx,Ty,Fy) for ndof=2; for ndof=3 nine full blocks
// and six residual parts.
static size_t elem_smem_bytes(int nod, int ndof) {
  if (ndof == 2) return (size_t)(nod * (nod + 1) + nod * nod + 4 * nod) * sizeof(double);
  return (size_t)(9 * nod * nod + 6 * nod + 19 * nod) * sizeof(double);  // + staged nodal fields
}

// Largest element count per patch: shared memory of the assembly kernel and,
// for the uvh kernel (one thread per element node), its block size.
static int max_patch_elements(int nod, int ndof) {
  const size_t budget = ndof == 2 ? 160 * 1024 : 200 * 1024;
  int e = (int)std::min<size_t>(1023, budget / elem_smem_bytes(nod, ndof));
  if (ndof == 3) e = std::min(e, (nod == 3 ? 512 : 320) / nod);
  return e;
}

// Node -> element lists (each sorted by global element id).
static void node_elements(int nod, int NN, int NE, const std::vector<int>& conn, std::vector<int>& n2e_ptr,
                          std::vector<int>& n2e) {
  n2e_ptr.assign(NN + 1, 0);
  for (int a = 0; a < nod; ++a)
    for (int e = 0; e < NE; ++e) n2e_ptr[conn[(size_t)a * NE + e] + 1]++;
  for (int i = 0; i < NN; ++i) n2e_ptr[i + 1] += n2e_ptr[i];
  n2e.resize(n2e_ptr[NN]);
  std::vector<int> fill(n2e_ptr.begin(), n2e_ptr.end() - 1);
  for (int e = 0; e < NE; ++e)  // increasing e => each list sorted; an element lists a node once
    for (int a = 0; a < nod; ++a) n2e[fill[conn[(size_t)a * NE + e]]++] = e;
}

// Global (batch) connectivity and coordinates of a handle from its per-system copies.
static void global_arrays(const ua_mesh* m, std::vector<int>& conn, std::vector<double>& X, std::vector<double>& Y,
                          std::vector<int>* node_sys) {
  const int nod = m->nod, nsys = (int)m->sys.size();
  const int NN = m->h_node_off[nsys], NE = m->h_elem_off[nsys];
  conn.assign((size_t)nod * NE, 0);
  X.assign(NN, 0.0); Y.assign(NN, 0.0);
  if (node_sys) node_sys->assign(NN, 0);
  for (int s = 0; s < nsys; ++s) {
    const HostSystem& hs = m->sys[s];
    int no = m->h_node_off[s], eo = m->h_elem_off[s];
    for (int i = 0; i < hs.nn; ++i) {
      X[no + i] = hs.x[i]; Y[no + i] = hs.y[i];
      if (node_sys) (*node_sys)[no + i] = s;
    }
    for (int a = 0; a < nod; ++a)
      for (int e = 0; e < hs.ne; ++e) conn[(size_t)a * NE + eo + e] = no + hs.conn[(size_t)a * hs.ne + e];
  }
}

// The symbolic scatter plan: node patches with their element lists and, per node-level
// non-zero of a patch row, the packed contribution list (element-local id, local row node,
// local column node) in increasing global element order.  The contributions of a non-zero
// are the same whatever the patches, so K and R do not depend on the shape.
struct PatchPlan {
  std::vector<int> patch_sys, patch_node_ptr{0}, patch_nodes, patch_elem_ptr{0}, patch_elems;
  std::vector<int> patch_q_ptr{0}, pq_cptr{0}, prow_diag;
  std::vector<uint32_t> pq_rk;
  std::vector<uint16_t> contrib;
  std::vector<int> hnode_ptr{0}, hnodes;
  std::vector<uint16_t> elnodes;
  int max_elems = 0, max_hnodes = 0;
};

static int build_patch_plan(const ua_mesh* m, const std::vector<int>& conn, const std::vector<double>& X,
                            const std::vector<double>& Y, const std::vector<int>& n2e_ptr, const std::vector<int>& n2e,
                            PatchShape shape, PatchPlan& P) {
  const int nod = m->nod, nsys = (int)m->sys.size();
  const int NE = m->h_elem_off[nsys];
  const std::vector<int>& nodeptr = m->h_nodeptr;
  const std::vector<int>& nodecol = m->h_nodecol;
  const int emax = max_patch_elements(nod, m->ndof);
  std::vector<int> mark(NE, -1), elocal(NE, -1);
  for (int s = 0; s < nsys; ++s) {
    int no = m->h_node_off[s], nn = m->sys[s].nn;
    double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
    for (int i = 0; i < nn; ++i) {
      xmin = std::min(xmin, X[no + i]); xmax = std::max(xmax, X[no + i]);
      ymin = std::min(ymin, Y[no + i]); ymax = std::max(ymax, Y[no + i]);
    }
    double span = std::max(xmax - xmin, ymax - ymin);
    if (!(span > 0)) span = 1;
    std::vector<std::pair<uint32_t, int>> key(nn);
    for (int i = 0; i < nn; ++i) {
      uint32_t qx = (uint32_t)std::min(65535.0, std::floor((X[no + i] - xmin) / span * 65535.0));
      uint32_t qy = (uint32_t)std::min(65535.0, std::floor((Y[no + i] - ymin) / span * 65535.0));
      key[i] = {spread16(qx) | (spread16(qy) << 1), no + i};
    }
    std::stable_sort(key.begin(), key.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    const int pn = shape.div > 0 ? std::max(16, std::min(shape.cap, nn / shape.div)) : std::max(1, shape.cap);
    size_t idx = 0;
    while (idx < key.size()) {
      std::vector<int> nodes, elems;
      int stamp = (int)P.patch_sys.size();
      while (idx < key.size() && (int)nodes.size() < pn) {
        int g = key[idx].second;
        int add = 0;
        for (int t = n2e_ptr[g]; t < n2e_ptr[g + 1]; ++t) add += (mark[n2e[t]] != stamp);
        if (!nodes.empty() && (int)elems.size() + add > emax) break;
        if ((int)elems.size() + add > emax) return set_error(UA_ERR_BAD_MESH, "node %d touches too many elements", g);
        nodes.push_back(g);
        for (int t = n2e_ptr[g]; t < n2e_ptr[g + 1]; ++t)
          if (mark[n2e[t]] != stamp) { mark[n2e[t]] = stamp; elems.push_back(n2e[t]); }
        ++idx;
      }
      std::sort(elems.begin(), elems.end());
      for (int i = 0; i < (int)elems.size(); ++i) elocal[elems[i]] = i;
      P.patch_sys.push_back(s);
      for (int r = 0; r < (int)nodes.size(); ++r) {
        int g = nodes[r];
        int deg = nodeptr[g + 1] - nodeptr[g];
        for (int k = 0; k < deg; ++k) {
          int j = nodecol[nodeptr[g] + k];
          if (j == g) P.prow_diag.push_back((int)P.pq_rk.size());
          P.pq_rk.push_back(((uint32_t)r << 16) | (uint32_t)k);
          for (int t = n2e_ptr[g]; t < n2e_ptr[g + 1]; ++t) {  // sorted global element order
            int e = n2e[t];
            int a = -1, b = -1;
            for (int c = 0; c < nod; ++c) {
              int v = conn[(size_t)c * NE + e];
              if (v == g) a = c;
              if (v == j) b = c;
            }
            if (b >= 0) P.contrib.push_back(pack_contrib(elocal[e], a, b));
          }
          P.pq_cptr.push_back((int)P.contrib.size());
        }
      }
      // the nodes of the patch's elements, sorted, and each element's nodes as indices into them
      {
        std::vector<int> hn;
        hn.reserve(elems.size() * nod);
        for (int e : elems)
          for (int c = 0; c < nod; ++c) hn.push_back(conn[(size_t)c * NE + e]);
        std::sort(hn.begin(), hn.end());
        hn.erase(std::unique(hn.begin(), hn.end()), hn.end());
        if (hn.size() > 65535) return set_error(UA_ERR_BAD_MESH, "patch with more than 65535 element nodes");
        for (int e : elems)
          for (int c = 0; c < nod; ++c) {
            const int v = conn[(size_t)c * NE + e];
            P.elnodes.push_back((uint16_t)(std::lower_bound(hn.begin(), hn.end(), v) - hn.begin()));
          }
        P.hnodes.insert(P.hnodes.end(), hn.begin(), hn.end());
        P.hnode_ptr.push_back((int)P.hnodes.size());
        P.max_hnodes = std::max(P.max_hnodes, (int)hn.size());
      }
      P.patch_nodes.insert(P.patch_nodes.end(), nodes.begin(), nodes.end());
      P.patch_node_ptr.push_back((int)P.patch_nodes.size());
      P.patch_elems.insert(P.patch_elems.end(), elems.begin(), elems.end());
      P.patch_elem_ptr.push_back((int)P.patch_elems.size());
      P.patch_q_ptr.push_back((int)P.pq_rk.size());
      P.max_elems = std::max(P.max_elems, (int)elems.size());
    }
  }
  return UA_OK;
}

// Uploads a plan into the handle, releasing the buffers of the plan it replaces.
static int install_patch_plan(ua_mesh* m, const PatchPlan& P) {
  DevMesh& dm = m->dm;
  const void* old[13] = {dm.patch_sys, dm.patch_node_ptr, dm.patch_nodes, dm.patch_elem_ptr, dm.patch_elems,
                         dm.patch_q_ptr, dm.pq_rk, dm.pq_cptr, dm.contrib, dm.prow_diag,
                         dm.patch_hnode_ptr, dm.patch_hnodes, dm.patch_elnodes};
  if (m->stream) UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  for (const void* q : old) dev_free(m, q);
  int rc;
  if ((rc = upload_vec(m, P.patch_sys, &dm.patch_sys))) return rc;
  if ((rc = upload_vec(m, P.patch_node_ptr, &dm.patch_node_ptr))) return rc;
  if ((rc = upload_vec(m, P.patch_nodes, &dm.patch_nodes))) return rc;
  if ((rc = upload_vec(m, P.patch_elem_ptr, &dm.patch_elem_ptr))) return rc;
  if ((rc = upload_vec(m, P.patch_elems, &dm.patch_elems))) return rc;
  if ((rc = upload_vec(m, P.patch_q_ptr, &dm.patch_q_ptr))) return rc;
  if ((rc = upload_vec(m, P.pq_rk, &dm.pq_rk))) return rc;
  if ((rc = upload_vec(m, P.pq_cptr, &dm.pq_cptr))) return rc;
  if ((rc = upload_vec(m, P.contrib, &dm.contrib))) return rc;
  if ((rc = upload_vec(m, P.prow_diag, &dm.prow_diag))) return rc;
  if ((rc = upload_vec(m, P.hnode_ptr, &dm.patch_hnode_ptr))) return rc;
  if ((rc = upload_vec(m, P.hnodes, &dm.patch_hnodes))) return rc;
  if ((rc = upload_vec(m, P.elnodes, &dm.patch_elnodes))) return rc;
  dm.npatch = (int)P.patch_sys.size();
  dm.max_patch_elems = P.max_elems;
  dm.max_patch_hnodes = P.max_hnodes;
  return UA_OK;
}

namespace ua {

int rebuild_patches(ua_mesh* m, PatchShape shape) {
  if (shape.cap < 1 || shape.cap > 1024 || shape.div < 0)
    return set_error(UA_ERR_INVALID, "patch shape (div %d, cap %d) out of range", shape.div, shape.cap);
  if (m->patch_shape.div == shape.div && m->patch_shape.cap == shape.cap) return UA_OK;
  UA_CUDA_TRY(cudaSetDevice(m->device));
  std::vector<int> conn, n2e_ptr, n2e;
  std::vector<double> X, Y;
  global_arrays(m, conn, X, Y, nullptr);
  node_elements(m->nod, m->nn_total, m->ne_total, conn, n2e_ptr, n2e);
  PatchPlan plan;
  int rc = build_patch_plan(m, conn, X, Y, n2e_ptr, n2e, shape, plan);
  if (rc) return rc;
  if ((rc = install_patch_plan(m, plan))) return rc;
  m->patch_shape = shape;
  return UA_OK;
}

static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int>, AsmTuning> g_tuned;

AsmTuning tuned_assembly(int device, int nod, int ndof, bool* tuned) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find({device, nod, ndof});
  if (tuned) *tuned = it != g_tuned.end();
  return it == g_tuned.end() ? AsmTuning{} : it->second;
}

void set_tuned_assembly(int device, int nod, int ndof, AsmTuning t) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[{device, nod, ndof}] = t;
}

}  // namespace ua

// detJ at the element centroid as derivVector.m:96-100 (for the orientation test of
// TestAndCorrectForInsideOutElements.m).
static double centroid_detJ(int nod, const double* xe, const double* ye) {
  double fun[kMaxNod], der[2][kMaxNod];
  shape(nod, 1.0 / 3.0, 1.0 / 3.0, fun, der);
  double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
  for (int a = 0; a < nod; ++a) {
    J11 += xe[a] * der[0][a];
    J12 += ye[a] * der[0][a];
    J21 += xe[a] * der[1][a];
    J22 += ye[a] * der[1][a];
  }
  return J11 * J22 - J12 * J21;
}

// FlipElements.m: reverse orientation.
static void flip(int nod, int* l) {
  if (nod == 3) {
    std::swap(l[1], l[2]);
  } else {
    int t[6] = {l[0], l[5], l[4], l[3], l[2], l[1]};
    for (int a = 0; a < 6; ++a) l[a] = t[a];
  }
}

extern "C" int ua_mesh_create_batch(const ua_mesh_desc* descs, int32_t count, int32_t ndof, int32_t device,
                                    ua_mesh** out) {
  if (!descs || count <= 0 || !out) return set_error(UA_ERR_INVALID, "ua_mesh_create_batch: bad arguments");
  if (ndof != 2 && ndof != 3) return set_error(UA_ERR_INVALID, "ndof must be 2 or 3");
  int nod = descs[0].nod;
  if (nod != 3 && nod != 6) return set_error(UA_ERR_INVALID, "nod must be 3 or 6 (got %d)", nod);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(UA_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= ndev) return set_error(UA_ERR_INVALID, "bad device ordinal %d", device);
  UA_CUDA_TRY(cudaSetDevice(device));

  ua_mesh* m = new ua_mesh();
  m->device = device;
  m->ndof = ndof;
  m->nod = nod;
  m->nip = quad_table(nod).nip;
  int nsys = count;
  m->sys.resize(nsys);
  // ---- validate, convert, orient -------------------------------------------------
  for (int s = 0; s < nsys; ++s) {
    const ua_mesh_desc& d = descs[s];
    if (d.nod != nod) { delete m; return set_error(UA_ERR_INVALID, "all meshes of a batch must have the same nod"); }
    if (d.nnodes <= 0 || d.nele <= 0 || !d.coordinates || !d.connectivity) {
      delete m; return set_error(UA_ERR_INVALID, "mesh %d: empty or null arrays", s);
    }
    HostSystem& hs = m->sys[s];
    hs.nn = d.nnodes; hs.ne = d.nele;
    hs.x.assign(d.coordinates, d.coordinates + d.nnodes);
    hs.y.assign(d.coordinates + d.nnodes, d.coordinates + 2 * (size_t)d.nnodes);
    hs.conn.resize((size_t)nod * d.nele);
    for (size_t i = 0; i < hs.conn.size(); ++i) {
      int v = d.connectivity[i] - d.index_base;
      if (v < 0 || v >= d.nnodes) { delete m; return set_error(UA_ERR_BAD_MESH, "mesh %d: connectivity index out of range", s); }
      hs.conn[i] = v;
    }
    for (int e = 0; e < hs.ne; ++e) {
      int l[kMaxNod]; double xe[kMaxNod], ye[kMaxNod];
      for (int a = 0; a < nod; ++a) { l[a] = hs.conn[(size_t)a * hs.ne + e]; xe[a] = hs.x[l[a]]; ye[a] = hs.y[l[a]]; }
      double dj = centroid_detJ(nod, xe, ye);
      if (!(dj != 0.0) || !std::isfinite(dj)) { delete m; return set_error(UA_ERR_BAD_MESH, "mesh %d element %d: degenerate (detJ=%g)", s, e, dj); }
      if (dj < 0) {
        flip(nod, l);
        for (int a = 0; a < nod; ++a) hs.conn[(size_t)a * hs.ne + e] = l[a];
        hs.nflipped++;
      }
    }
  }
  // ---- offsets -----------------------------------------------------------------
  m->h_node_off.assign(nsys + 1, 0);
  m->h_elem_off.assign(nsys + 1, 0);
  for (int s = 0; s < nsys; ++s) {
    m->h_node_off[s + 1] = m->h_node_off[s] + m->sys[s].nn;
    m->h_elem_off[s + 1] = m->h_elem_off[s] + m->sys[s].ne;
  }
  int NN = m->h_node_off[nsys], NE = m->h_elem_off[nsys];
  m->nn_total = NN; m->ne_total = NE;
  std::vector<int> conn, node_sys;
  std::vector<double> X, Y;
  global_arrays(m, conn, X, Y, &node_sys);
  // ---- node -> element CSR -------------------------------------------------------
  std::vector<int> n2e_ptr, n2e;
  node_elements(nod, NN, NE, conn, n2e_ptr, n2e);
  for (int g = 0; g < NN; ++g)
    if (n2e_ptr[g + 1] == n2e_ptr[g]) { delete m; return set_error(UA_ERR_BAD_MESH, "node %d belongs to no element", g); }
  // ---- node-level adjacency (sorted, includes self) ------------------------------
  std::vector<int>& nodeptr = m->h_nodeptr;
  std::vector<int>& nodecol = m->h_nodecol;
  nodeptr.assign(NN + 1, 0);
  nodecol.clear();
  {
    std::vector<int> buf;
    for (int g = 0; g < NN; ++g) {
      buf.clear();
      for (int t = n2e_ptr[g]; t < n2e_ptr[g + 1]; ++t) {
        int e = n2e[t];
        for (int a = 0; a < nod; ++a) buf.push_back(conn[(size_t)a * NE + e]);
      }
      std::sort(buf.begin(), buf.end());
      buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
      nodecol.insert(nodecol.end(), buf.begin(), buf.end());
      nodeptr[g + 1] = (int)nodecol.size();
    }
  }
  // ---- per-system dof / nnz offsets ----------------------------------------------
  m->h_dof_off.assign(nsys + 1, 0);
  m->h_knz_off.assign(nsys + 1, 0);
  m->h_nnzn.assign(nsys, 0);
  long long knz = 0;
  for (int s = 0; s < nsys; ++s) {
    int nnzn = nodeptr[m->h_node_off[s + 1]] - nodeptr[m->h_node_off[s]];
    m->h_nnzn[s] = nnzn;
    m->h_dof_off[s + 1] = m->h_dof_off[s] + ndof * m->sys[s].nn;
    knz += (long long)ndof * ndof * nnzn;
    if (knz >= (1LL << 31)) { delete m; return set_error(UA_ERR_INVALID, "tangent has more than 2^31 non-zeros"); }
    m->h_knz_off[s + 1] = (int)knz;
  }
  m->ndof_total = m->h_dof_off[nsys];
  m->nnz_total = knz;
  // ---- patches (Morton-ordered node groups within each system) --------------------
  {
    const AsmTuning t = tuned_assembly(device, nod, ndof);
    m->patch_shape = t.shape;
    m->asm_threads = t.threads;
    m->asm_regs = t.regs;
  }
  PatchPlan plan;
  {
    int prc = build_patch_plan(m, conn, X, Y, n2e_ptr, n2e, m->patch_shape, plan);
    if (prc) { delete m; return prc; }
  }
  // ---- upload ----------------------------------------------------------------------
  UA_CUDA_TRY(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  DevMesh& dm = m->dm;
  dm.nsys = nsys; dm.nn = NN; dm.ne = NE; dm.nod = nod; dm.nip = m->nip; dm.ndof = ndof;
  int rc = UA_OK;
  std::vector<int> knz_off(m->h_knz_off.begin(), m->h_knz_off.end());
  if ((rc = upload_vec(m, conn, &dm.conn))) goto fail;
  if ((rc = upload_vec(m, X, &dm.x))) goto fail;
  if ((rc = upload_vec(m, Y, &dm.y))) goto fail;
  if ((rc = upload_vec(m, nodeptr, &dm.nodeptr))) goto fail;
  if ((rc = upload_vec(m, nodecol, &dm.nodecol))) goto fail;
  if ((rc = upload_vec(m, node_sys, &dm.node_sys))) goto fail;
  if ((rc = upload_vec(m, m->h_node_off, &dm.sys_node_off))) goto fail;
  if ((rc = upload_vec(m, m->h_dof_off, &dm.sys_dof_off))) goto fail;
  if ((rc = upload_vec(m, knz_off, &dm.sys_knz_off))) goto fail;
  if ((rc = upload_vec(m, m->h_nnzn, &dm.sys_nnzn))) goto fail;
  if ((rc = install_patch_plan(m, plan))) goto fail;
#ifdef UA_BOUNDS_CHECK
  {
    const std::vector<unsigned long long> zero(1, 0ULL);
    if ((rc = upload_vec(m, zero, (const unsigned long long**)&dm.dbg))) goto fail;
  }
#else
  dm.dbg = nullptr;
#endif
  *out = m;
  return UA_OK;
fail:
  dev_free_all(m);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return rc;
}

// The first bounds violation a kernel of this handle recorded (bounds-checked build only).
extern "C" int ua_debug_bounds(const ua_mesh* m, int32_t* enabled, int32_t* site, int64_t* index) {
  if (!m || !enabled || !site || !index) return set_error(UA_ERR_INVALID, "ua_debug_bounds: null argument");
  *site = 0;
  *index = 0;
#ifdef UA_BOUNDS_CHECK
  *enabled = 1;
  unsigned long long v = 0;
  UA_CUDA_TRY(cudaSetDevice(m->device));
  UA_CUDA_TRY(cudaStreamSynchronize(m->stream));
  UA_CUDA_TRY(cudaMemcpy(&v, m->dm.dbg, sizeof(v), cudaMemcpyDeviceToHost));
  *site = (int32_t)(v >> 48);
  *index = (int64_t)(v & 0xffffffffffffULL);
#else
  *enabled = 0;
#endif
  return UA_OK;
}
