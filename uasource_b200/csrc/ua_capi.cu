// Small C-ABI entry points: version, errors, mesh queries.
#include <cstdio>
#include "ua_internal.h"

namespace ua {
const char* last_error_message();
}

extern "C" const char* ua_version(void) { return "libuassa 0.1 (sm_100a)"; }

extern "C" const char* ua_last_error(void) { return ua::last_error_message(); }

extern "C" int ua_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

extern "C" int ua_mesh_create(const ua_mesh_desc* desc, int32_t ndof, int32_t device, ua_mesh** out) {
  return ua_mesh_create_batch(desc, 1, ndof, device, out);
}

// Structural pattern of system `sys` in its own dof numbering (CSR, sorted columns).
extern "C" int ua_mesh_pattern(const ua_mesh* m, int32_t sys, int64_t* nnz, int64_t* rowptr, int64_t* colind) {
  if (!m || sys < 0 || sys >= m->dm.nsys || !nnz) return ua::set_error(UA_ERR_INVALID, "ua_mesh_pattern: bad arguments");
  const int nd = m->ndof;
  const int no = m->h_node_off[sys], nn = m->sys[sys].nn;
  const int nb = m->h_nodeptr[no];
  const long long nnzn = m->h_nodeptr[no + nn] - nb;
  *nnz = (long long)nd * nd * nnzn;
  if (!rowptr && !colind) return UA_OK;
  for (int c = 0; c < nd; ++c)
    for (int i = 0; i < nn; ++i) {
      const int g = no + i;
      const int np0 = m->h_nodeptr[g], deg = m->h_nodeptr[g + 1] - np0;
      const long long start = (long long)c * nd * nnzn + (long long)nd * (np0 - nb);
      if (rowptr) rowptr[c * nn + i] = start;
      if (colind)
        for (int b = 0; b < nd; ++b)
          for (int k = 0; k < deg; ++k) colind[start + b * deg + k] = (long long)b * nn + (m->h_nodecol[np0 + k] - no);
    }
  if (rowptr) rowptr[(long long)nd * nn] = *nnz;
  return UA_OK;
}

extern "C" int ua_mesh_info(const ua_mesh* m, int32_t sys, int32_t* nsys, int32_t* nnodes, int32_t* nele,
                            int64_t* device_bytes) {
  if (!m) return ua::set_error(UA_ERR_INVALID, "null mesh");
  if (nsys) *nsys = m->dm.nsys;
  if (sys >= 0 && sys < m->dm.nsys) {
    if (nnodes) *nnodes = m->sys[sys].nn;
    if (nele) *nele = m->sys[sys].ne;
  }
  if (device_bytes) *device_bytes = (int64_t)m->device_bytes;
  return UA_OK;
}

extern "C" int ua_mesh_flipped(const ua_mesh* m, int32_t* nflipped) {
  if (!m || !nflipped) return ua::set_error(UA_ERR_INVALID, "null argument");
  int n = 0;
  for (auto& s : m->sys) n += s.nflipped;
  *nflipped = n;
  return UA_OK;
}

extern "C" int ua_struct_sizes(int64_t* sizes, int32_t n) {
  const int64_t all[7] = {(int64_t)sizeof(ua_mesh_desc), (int64_t)sizeof(ua_params), (int64_t)sizeof(ua_fields),
                          (int64_t)sizeof(ua_bcs), (int64_t)sizeof(ua_newton_iter), (int64_t)sizeof(ua_newton_report),
                          (int64_t)sizeof(ua_tune_report)};
  if (!sizes || n < 0 || n > 7) return ua::set_error(UA_ERR_INVALID, "ua_struct_sizes: bad arguments");
  for (int i = 0; i < n; ++i) sizes[i] = all[i];
  return UA_OK;
}
