/*
 * Shared helpers of the MEX gateways: read Úa's MATLAB structs (CtrlVar, MUA,
 * F, BCs) by field name and marshal them into the plain-pointer C-ABI of
 * libuassa (include/ua_ssa.h).  Builds with `mex` (MATLAB) or
 * `mkoctfile --mex` (GNU Octave):
 *
 *   mex -I../include uvMatrixAssemblySSTREAM_mex.c -L../uasource_b200 -luassa
 *
 * The device-resident mesh handle persists across calls (static storage,
 * mexLock) and is rebuilt only when MUA.coordinates/connectivity change; it is
 * freed at exit (mexAtExit).  All mx* calls run on MATLAB's interpreter thread.
 */
#ifndef UA_MEX_COMMON_H
#define UA_MEX_COMMON_H

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"
#include "ua_ssa.h"

/* one resident handle per dof count: [0] uv (ndof 2), [1] uvh (ndof 3) */
static ua_mesh* g_meshes[2] = {NULL, NULL};
static uint64_t g_mesh_keys[2] = {0, 0};
static int g_locked = 0;

static inline void ua_mex_cleanup(void) {
    int k;
    for (k = 0; k < 2; ++k) {
        if (g_meshes[k]) ua_mesh_destroy(g_meshes[k]);
        g_meshes[k] = NULL;
        g_mesh_keys[k] = 0;
    }
}

/* FNV-1a over the raw bytes of the mesh arrays: detects a changed MUA. */
static inline uint64_t ua_mex_hash(const void* p, size_t n, uint64_t h) {
    const unsigned char* b = (const unsigned char*)p;
    size_t i;
    for (i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ULL;
    return h;
}

static inline void ua_mex_fail(int rc) {
    const char* id = "Ua:mex:Error";
    if (rc == UA_ERR_NAN_INPUT) id = "uvMatrixAssembly:NaN";
    else if (rc == UA_ERR_NO_DEVICE) id = "Ua:mex:NoDevice";
    else if (rc == UA_ERR_OOM) id = "Ua:mex:OutOfMemory";
    mexErrMsgIdAndTxt(id, "%s", ua_last_error());
}

static inline const mxArray* ua_mex_field(const mxArray* s, const char* name, int required) {
    const mxArray* f = (s && mxIsStruct(s)) ? mxGetField(s, 0, name) : NULL;
    if (!f && required) mexErrMsgIdAndTxt("Ua:mex:MissingField", "missing field %s", name);
    return f;
}

static inline double ua_mex_scalar(const mxArray* s, const char* name, double dflt) {
    const mxArray* f = ua_mex_field(s, name, 0);
    if (!f || mxIsEmpty(f)) return dflt;
    return mxGetScalar(f);
}

/* CtrlVar -> ua_params (fields named as in Ua2D_DefaultParameters.m). */
static inline void ua_mex_params(const mxArray* C, ua_params* p) {
    const mxArray* f;
    ua_params_default(p);
    p->kH = ua_mex_scalar(C, "kH", p->kH);
    p->Hh0 = ua_mex_scalar(C, "Hh0", p->Hh0);
    p->SpeedZero = ua_mex_scalar(C, "SpeedZero", p->SpeedZero);
    p->EpsZero = ua_mex_scalar(C, "EpsZero", p->EpsZero);
    p->etaZero = ua_mex_scalar(C, "etaZero", p->etaZero);
    p->Czero = ua_mex_scalar(C, "Czero", p->Czero);
    p->Cmin = ua_mex_scalar(C, "Cmin", p->Cmin);
    p->AGlenmin = ua_mex_scalar(C, "AGlenmin", p->AGlenmin);
    p->Picard = (int32_t)ua_mex_scalar(C, "Picard", p->Picard);
    p->NRviscosity = ua_mex_scalar(C, "NRviscosity", p->NRviscosity);
    p->NRitmax = (int32_t)ua_mex_scalar(C, "NRitmax", p->NRitmax);
    p->NRitmin = (int32_t)ua_mex_scalar(C, "NRitmin", p->NRitmin);
    p->NewtonAcceptRatio = ua_mex_scalar(C, "NewtonAcceptRatio", p->NewtonAcceptRatio);
    p->BacktrackingGammaMin = ua_mex_scalar(C, "BacktrackingGammaMin", p->BacktrackingGammaMin);
    p->LineSearchAllowedToUseExtrapolation =
        (int32_t)ua_mex_scalar(C, "LineSearchAllowedToUseExtrapolation", p->LineSearchAllowedToUseExtrapolation);
    p->BackTrackBeta = ua_mex_scalar(C, "BackTrackBeta", p->BackTrackBeta);
    p->BackTrackMaxIterations = (int32_t)ua_mex_scalar(C, "BackTrackMaxIterations", p->BackTrackMaxIterations);
    p->BackTrackGuardLower = ua_mex_scalar(C, "BackTrackGuardLower", p->BackTrackGuardLower);
    p->BackTrackGuardUpper = ua_mex_scalar(C, "BackTrackGuardUpper", p->BackTrackGuardUpper);
    p->uvExitBackTrackingStepLength = ua_mex_scalar(C, "uvExitBackTrackingStepLength", p->uvExitBackTrackingStepLength);
    p->ModifiedNRuvIntervalCriterion =
        (int32_t)ua_mex_scalar(C, "ModifiedNRuvIntervalCriterion", p->ModifiedNRuvIntervalCriterion);
    p->ModifiedNRuvReductionCriterion =
        ua_mex_scalar(C, "ModifiedNRuvReductionCriterion", p->ModifiedNRuvReductionCriterion);
    {
        const char* pairs[4] = {"uvDesiredWorkAndForceTolerances", "uvDesiredWorkOrForceTolerances",
                                "uvAcceptableWorkAndForceTolerances", "uvAcceptableWorkOrForceTolerances"};
        double* dst[4] = {p->uvDesiredWorkAndForceTolerances, p->uvDesiredWorkOrForceTolerances,
                          p->uvAcceptableWorkAndForceTolerances, p->uvAcceptableWorkOrForceTolerances};
        int k;
        for (k = 0; k < 4; ++k) {
            f = ua_mex_field(C, pairs[k], 0);
            if (f && mxGetNumberOfElements(f) == 2) {
                dst[k][0] = mxGetPr(f)[0];
                dst[k][1] = mxGetPr(f)[1];
            }
        }
    }
    /* uvh: CtrlVar.theta, CtrlVar.SUPG.beta0, CtrlVar.uvh.SUPG.{tau,tauMultiplier} and the uvh
     * tolerances (Ua2D_DefaultParameters.m:376-377, :494-505, :551-555) */
    p->theta = ua_mex_scalar(C, "theta", p->theta);
    {
        const mxArray* sg = ua_mex_field(C, "SUPG", 0);
        const mxArray* uvh = ua_mex_field(C, "uvh", 0);
        const mxArray* us = uvh ? ua_mex_field(uvh, "SUPG", 0) : NULL;
        if (sg) p->SUPG_beta0 = ua_mex_scalar(sg, "beta0", p->SUPG_beta0);
        if (us) {
            const mxArray* t = ua_mex_field(us, "tau", 0);
            p->uvh_SUPG_tauMultiplier = ua_mex_scalar(us, "tauMultiplier", p->uvh_SUPG_tauMultiplier);
            if (t && mxIsChar(t)) {
                char* name = mxArrayToString(t);
                if (name) {
                    if (!strcmp(name, "taus")) p->uvh_SUPG_tau = 0;
                    else if (!strcmp(name, "taut")) p->uvh_SUPG_tau = 1;
                    else if (!strcmp(name, "tau1")) p->uvh_SUPG_tau = 2;
                    else if (!strcmp(name, "tau2")) p->uvh_SUPG_tau = 3;
                    mxFree(name);
                }
            }
        }
        /* a MATLAB string object is not readable through the C API: numeric override */
        p->uvh_SUPG_tau = (int32_t)ua_mex_scalar(C, "GPUuvhSUPGtau", p->uvh_SUPG_tau);
    }
    p->uvhExitBackTrackingStepLength =
        ua_mex_scalar(C, "uvhExitBackTrackingStepLength", p->uvhExitBackTrackingStepLength);
    {
        const char* pairs[4] = {"uvhDesiredWorkAndForceTolerances", "uvhDesiredWorkOrForceTolerances",
                                "uvhAcceptableWorkAndForceTolerances", "uvhAcceptableWorkOrForceTolerances"};
        double* dst[4] = {p->uvhDesiredWorkAndForceTolerances, p->uvhDesiredWorkOrForceTolerances,
                          p->uvhAcceptableWorkAndForceTolerances, p->uvhAcceptableWorkOrForceTolerances};
        int k;
        for (k = 0; k < 4; ++k) {
            const mxArray* f = ua_mex_field(C, pairs[k], 0);
            if (f && mxGetNumberOfElements(f) == 2) {
                dst[k][0] = mxGetPr(f)[0];
                dst[k][1] = mxGetPr(f)[1];
            }
        }
    }
    /* CtrlVar.SlidingLaw as a char array (a MATLAB string object is not readable through the C
     * API: pass char(CtrlVar.SlidingLaw), or the numeric GPUSlidingLaw = UA_SLIDING_*) */
    {
        static const char* laws[14] = {"Weertman", "W", "Budd", "W-N0", "Tsai", "minCW-N0", "Coulomb", "C",
                                       "Cornford", "rpCW-N0", "Umbi", "rCW-N0", "Joughin", "rCW-V0"};
        static const int codes[14] = {UA_SLIDING_WEERTMAN, UA_SLIDING_WEERTMAN, UA_SLIDING_BUDD, UA_SLIDING_BUDD,
                                      UA_SLIDING_TSAI, UA_SLIDING_TSAI, UA_SLIDING_COULOMB, UA_SLIDING_COULOMB,
                                      UA_SLIDING_CORNFORD, UA_SLIDING_CORNFORD, UA_SLIDING_UMBI, UA_SLIDING_UMBI,
                                      UA_SLIDING_JOUGHIN, UA_SLIDING_JOUGHIN};
        const mxArray* t = ua_mex_field(C, "SlidingLaw", 0);
        if (t && mxIsChar(t)) {
            char* name = mxArrayToString(t);
            int k, found = 0;
            for (k = 0; name && k < 14; ++k)
                if (!strcmp(name, laws[k])) { p->SlidingLaw = codes[k]; found = 1; }
            if (name) mxFree(name);
            if (!found) mexErrMsgIdAndTxt("BasalDrag:CaseNotFound", "what sliding law?");
        }
        p->SlidingLaw = (int32_t)ua_mex_scalar(C, "GPUSlidingLaw", p->SlidingLaw);
    }
    p->Nzero = ua_mex_scalar(C, "Nzero", p->Nzero);
    /* the minimum-thickness active set of uvh.m:64-212 (Ua2D_DefaultParameters.m:1479-1500) */
    p->ThicknessConstraints = (int32_t)ua_mex_scalar(C, "ThicknessConstraints", p->ThicknessConstraints);
    p->ThickMin = ua_mex_scalar(C, "ThickMin", p->ThickMin);
    p->ThicknessConstraintsItMax = (int32_t)ua_mex_scalar(C, "ThicknessConstraintsItMax", p->ThicknessConstraintsItMax);
    p->MaxNumberOfNewlyIntroducedActiveThicknessConstraints = (int32_t)ua_mex_scalar(
        C, "MaxNumberOfNewlyIntroducedActiveThicknessConstraints", p->MaxNumberOfNewlyIntroducedActiveThicknessConstraints);
    p->MinNumberOfNewlyIntroducedActiveThicknessConstraints = (int32_t)ua_mex_scalar(
        C, "MinNumberOfNewlyIntroducedActiveThicknessConstraints", p->MinNumberOfNewlyIntroducedActiveThicknessConstraints);
    p->IncludeMelangeModelPhysics =
        (int32_t)ua_mex_scalar(C, "IncludeMelangeModelPhysics", p->IncludeMelangeModelPhysics);
    /* the GPU form selected by a CtrlVar.UseGPU-style switch (0=FP64, 1=mixed) */
    p->precision = (int32_t)ua_mex_scalar(C, "GPUPrecision", p->precision);
    p->krylov_rtol = ua_mex_scalar(C, "GPUKrylovTol", p->krylov_rtol);
    p->krylov_precond = (int32_t)ua_mex_scalar(C, "GPUPreconditioner", p->krylov_precond);
    p->krylov_adaptive = (int32_t)ua_mex_scalar(C, "GPUKrylovAdaptive", p->krylov_adaptive);
}

/* MUA -> cached device mesh with ndof dofs per node (2: uv, 3: uvh), rebuilt
 * when coordinates/connectivity change. */
static inline ua_mesh* ua_mex_mesh_ndof(const mxArray* MUA, int ndof) {
    const mxArray* co = ua_mex_field(MUA, "coordinates", 1);
    const mxArray* cn = ua_mex_field(MUA, "connectivity", 1);
    size_t nn = mxGetM(co), ne = mxGetM(cn), nod = mxGetN(cn), i;
    uint64_t key = 1469598103934665603ULL;
    int32_t* conn;
    ua_mesh_desc d;
    int rc;
    if (mxGetN(co) != 2 || !mxIsDouble(co) || !mxIsDouble(cn))
        mexErrMsgIdAndTxt("Ua:mex:BadMUA", "MUA.coordinates must be Nnodes x 2 double, connectivity double");
    const int slot = ndof == 3 ? 1 : 0;
    key = ua_mex_hash(mxGetPr(co), nn * 2 * sizeof(double), key);
    key = ua_mex_hash(mxGetPr(cn), ne * nod * sizeof(double), key);
    if (g_meshes[slot] && key == g_mesh_keys[slot]) return g_meshes[slot];
    if (g_meshes[slot]) ua_mesh_destroy(g_meshes[slot]);
    g_meshes[slot] = NULL;
    conn = (int32_t*)mxMalloc(ne * nod * sizeof(int32_t));
    for (i = 0; i < ne * nod; ++i) conn[i] = (int32_t)mxGetPr(cn)[i];
    d.nnodes = (int32_t)nn;
    d.nele = (int32_t)ne;
    d.nod = (int32_t)nod;
    d.index_base = 1;
    d.coordinates = mxGetPr(co);
    d.connectivity = conn;
    rc = ua_mesh_create(&d, ndof, 0, &g_meshes[slot]);
    mxFree(conn);
    if (rc != UA_OK) {
        g_meshes[slot] = NULL;
        mexErrMsgIdAndTxt(rc == UA_ERR_BAD_MESH ? "Ua:TestAndCorrectForInsideOutElements:InsideOutelements"
                                                : "Ua:mex:MeshCreate",
                          "%s", ua_last_error());
    }
    g_mesh_keys[slot] = key;
    if (!g_locked) {
        mexLock();
        mexAtExit(ua_mex_cleanup);
        g_locked = 1;
    }
    return g_meshes[slot];
}

static inline ua_mesh* ua_mex_mesh(const mxArray* MUA) { return ua_mex_mesh_ndof(MUA, 2); }

/* A nodal field: Nn-vector, or a scalar expanded as uv.m:34-40 does for m and n. */
static inline const double* ua_mex_nodal(const mxArray* F, const char* name, size_t nn, double** owned) {
    const mxArray* f = ua_mex_field(F, name, 1);
    size_t k = mxGetNumberOfElements(f), i;
    *owned = NULL;
    if (k == nn) return mxGetPr(f);
    if (k == 1) {
        *owned = (double*)mxMalloc(nn * sizeof(double));
        for (i = 0; i < nn; ++i) (*owned)[i] = mxGetScalar(f);
        return *owned;
    }
    mexErrMsgIdAndTxt("Ua:mex:BadField", "F.%s must have Nnodes elements", name);
    return NULL;
}

/* The sliding-law and melange fields of F present and non-empty (F.q, F.muk, F.V0, F.uo, F.vo,
 * F.Co, F.mo, F.ua, F.va, F.Ca, F.ma); scalars are expanded.  own[11] receives the expanded
 * copies (free them with mxFree). */
static inline void ua_mex_drag_fields(const mxArray* F, size_t nn, ua_fields* f, double** own) {
    static const char* names[11] = {"q", "muk", "V0", "uo", "vo", "Co", "mo", "ua", "va", "Ca", "ma"};
    const double** dst[11];
    int k;
    dst[0] = &f->q; dst[1] = &f->muk; dst[2] = &f->V0; dst[3] = &f->uo; dst[4] = &f->vo; dst[5] = &f->Co;
    dst[6] = &f->mo; dst[7] = &f->ua; dst[8] = &f->va; dst[9] = &f->Ca; dst[10] = &f->ma;
    for (k = 0; k < 11; ++k) {
        const mxArray* a = ua_mex_field(F, names[k], 0);
        own[k] = NULL;
        *dst[k] = NULL;
        if (a && !mxIsEmpty(a)) *dst[k] = ua_mex_nodal(F, names[k], nn, &own[k]);
    }
}

/* The constraint matrix L (nc x ncols sparse, one or two entries per row, rows of unit length;
 * ScaleL.m) of the BCs b, as AssembleLuvSSTREAM.m / AssembleLuvhSSTREAM.m build it, via
 * ua_constraint_matrix. */
static inline mxArray* ua_mex_constraint_L(ua_mesh* m, const ua_bcs* b, int32_t ncols) {
    int32_t nc = 0, k, e;
    int32_t* dof;
    double* val;
    mwIndex *jc, *ir, *cnt;
    double* pr;
    mxArray* L;
    int rc = ua_constraint_matrix(m, b, &nc, NULL, NULL, NULL);
    if (rc != UA_OK) ua_mex_fail(rc);
    dof = (int32_t*)mxMalloc((nc > 0 ? 2 * nc : 2) * sizeof(int32_t));
    val = (double*)mxMalloc((nc > 0 ? 2 * nc : 2) * sizeof(double));
    rc = ua_constraint_matrix(m, b, &nc, dof, val, NULL);
    if (rc != UA_OK) ua_mex_fail(rc);
    L = mxCreateSparse(nc, ncols, nc > 0 ? 2 * nc : 1, mxREAL);
    jc = mxGetJc(L); ir = mxGetIr(L); pr = mxGetPr(L);
    cnt = (mwIndex*)mxCalloc(ncols + 1, sizeof(mwIndex));
    for (e = 0; e < 2 * nc; ++e)
        if (dof[e] >= 0) cnt[dof[e] + 1]++;
    for (k = 0; k < ncols; ++k) cnt[k + 1] += cnt[k];
    for (k = 0; k <= ncols; ++k) jc[k] = cnt[k];
    for (e = 0; e < 2 * nc; ++e) {  /* rows in increasing order, so each column's rows come out sorted */
        if (dof[e] < 0) continue;
        ir[cnt[dof[e]]] = (mwIndex)(e / 2);
        pr[cnt[dof[e]]] = val[e];
        cnt[dof[e]]++;
    }
    mxFree(cnt); mxFree(dof); mxFree(val);
    return L;
}

/* dadh of uvhMatrixAssembly.m:152-158: F1.dasdh + F1.dabdh when
 * CtrlVar.MassBalanceGeometryFeedback is 3, else none (NULL = zero). */
static inline const double* ua_mex_dadh(const mxArray* C, const mxArray* F1, size_t nn, double** owned) {
    const mxArray *a = ua_mex_field(F1, "dasdh", 0), *b = ua_mex_field(F1, "dabdh", 0);
    size_t i;
    *owned = NULL;
    if ((int)ua_mex_scalar(C, "MassBalanceGeometryFeedback", 0) != 3) return NULL;
    *owned = (double*)mxCalloc(nn, sizeof(double));
    if (a && mxGetNumberOfElements(a) == nn) for (i = 0; i < nn; ++i) (*owned)[i] += mxGetPr(a)[i];
    if (b && mxGetNumberOfElements(b) == nn) for (i = 0; i < nn; ++i) (*owned)[i] += mxGetPr(b)[i];
    return *owned;
}

/* BCs node lists (double, 1-based) -> int32 arrays owned by the caller. */
static inline int32_t* ua_mex_nodes(const mxArray* B, const char* name, int32_t* n) {
    const mxArray* f = ua_mex_field(B, name, 0);
    size_t k = f ? mxGetNumberOfElements(f) : 0, i;
    int32_t* out;
    *n = (int32_t)k;
    if (!k) return NULL;
    out = (int32_t*)mxMalloc(k * sizeof(int32_t));
    for (i = 0; i < k; ++i) out[i] = (int32_t)mxGetPr(f)[i];
    return out;
}

/* The values that go with n nodes: NULL (all zero) when the field is missing or empty, else
 * exactly n of them. */
static inline const double* ua_mex_values(const mxArray* B, const char* name, int32_t n) {
    const mxArray* f = ua_mex_field(B, name, 0);
    if (!f || mxIsEmpty(f)) return NULL;
    if ((int64_t)mxGetNumberOfElements(f) != n)
        mexErrMsgIdAndTxt("Ua:mex:BCs", "%s has %d entries for %d nodes", name, (int)mxGetNumberOfElements(f), n);
    return mxGetPr(f);
}

/* The mesh's 1-based BC lists.  The library takes 0-based indices for
 * index_base handles created from MATLAB too, so shift here. */
static inline void ua_mex_bcs(const mxArray* B, ua_bcs* b) {
    int32_t i, n_ub = 0, n_vb = 0;
    memset(b, 0, sizeof(*b));
    if (!B || !mxIsStruct(B)) return;
    b->ufixed_node = ua_mex_nodes(B, "ubFixedNode", &b->n_ufixed);
    b->ufixed_value = ua_mex_values(B, "ubFixedValue", b->n_ufixed);
    b->vfixed_node = ua_mex_nodes(B, "vbFixedNode", &b->n_vfixed);
    b->vfixed_value = ua_mex_values(B, "vbFixedValue", b->n_vfixed);
    b->utied_a = ua_mex_nodes(B, "ubTiedNodeA", &b->n_utied);
    b->utied_b = ua_mex_nodes(B, "ubTiedNodeB", &n_ub);
    b->vtied_a = ua_mex_nodes(B, "vbTiedNodeA", &b->n_vtied);
    b->vtied_b = ua_mex_nodes(B, "vbTiedNodeB", &n_vb);
    if (n_ub != b->n_utied || n_vb != b->n_vtied)  /* CreateLuv.m pairs A(k) with B(k) */
        mexErrMsgIdAndTxt("Ua:mex:BCs", "ubTiedNodeA/B and vbTiedNodeA/B must have equal lengths");
    for (i = 0; i < b->n_ufixed; ++i) ((int32_t*)b->ufixed_node)[i] -= 1;
    for (i = 0; i < b->n_vfixed; ++i) ((int32_t*)b->vfixed_node)[i] -= 1;
    for (i = 0; i < b->n_utied; ++i) { ((int32_t*)b->utied_a)[i] -= 1; ((int32_t*)b->utied_b)[i] -= 1; }
    for (i = 0; i < b->n_vtied; ++i) { ((int32_t*)b->vtied_a)[i] -= 1; ((int32_t*)b->vtied_b)[i] -= 1; }
    b->hfixed_node = ua_mex_nodes(B, "hFixedNode", &b->n_hfixed);
    b->hfixed_value = ua_mex_values(B, "hFixedValue", b->n_hfixed);
    b->normal_node = ua_mex_nodes(B, "ubvbFixedNormalNode", &b->n_normal);
    b->normal_value = ua_mex_values(B, "ubvbFixedNormalValue", b->n_normal);
    for (i = 0; i < b->n_normal; ++i) ((int32_t*)b->normal_node)[i] -= 1;
    for (i = 0; i < b->n_hfixed; ++i) ((int32_t*)b->hfixed_node)[i] -= 1;
    b->hpos_node = ua_mex_nodes(B, "hPosNode", &b->n_hpos);  /* the active set carried from the last step */
    for (i = 0; i < b->n_hpos; ++i) ((int32_t*)b->hpos_node)[i] -= 1;
}

/* CSR values on the structural pattern -> MATLAB sparse (CSC, sorted rows, no
 * explicit zeros).  The uv pattern and values are symmetric, so the CSR arrays
 * are read as CSC. */
static inline mxArray* ua_mex_sparse(ua_mesh* m, int32_t n, const double* vals) {
    int64_t nnz = 0, j, k, out = 0;
    int64_t *rp, *ci;
    mxArray* S;
    mwIndex *jc, *ir;
    double* pr;
    ua_mesh_pattern(m, 0, &nnz, NULL, NULL);
    rp = (int64_t*)mxMalloc((n + 1) * sizeof(int64_t));
    ci = (int64_t*)mxMalloc(nnz * sizeof(int64_t));
    ua_mesh_pattern(m, 0, &nnz, rp, ci);
    for (k = 0; k < nnz; ++k) out += vals[k] != 0.0;
    S = mxCreateSparse(n, n, out > 0 ? out : 1, mxREAL);
    jc = mxGetJc(S); ir = mxGetIr(S); pr = mxGetPr(S);
    out = 0;
    for (j = 0; j < n; ++j) {
        jc[j] = (mwIndex)out;
        for (k = rp[j]; k < rp[j + 1]; ++k)
            if (vals[k] != 0.0) { ir[out] = (mwIndex)ci[k]; pr[out] = vals[k]; ++out; }
    }
    jc[n] = (mwIndex)out;
    mxFree(rp); mxFree(ci);
    return S;
}

/* CSR values of an unsymmetric tangent (uvh) on the structural pattern ->
 * MATLAB sparse: a column-count pass, then the transpose (CSC, sorted rows,
 * no explicit zeros). */
static inline mxArray* ua_mex_sparse_unsym(ua_mesh* m, int32_t n, const double* vals) {
    int64_t nnz = 0, i, k, out = 0;
    int64_t *rp, *ci;
    mwIndex *jc, *ir, *next;
    mxArray* S;
    double* pr;
    ua_mesh_pattern(m, 0, &nnz, NULL, NULL);
    rp = (int64_t*)mxMalloc((n + 1) * sizeof(int64_t));
    ci = (int64_t*)mxMalloc(nnz * sizeof(int64_t));
    ua_mesh_pattern(m, 0, &nnz, rp, ci);
    for (k = 0; k < nnz; ++k) out += vals[k] != 0.0;
    S = mxCreateSparse(n, n, out > 0 ? out : 1, mxREAL);
    jc = mxGetJc(S); ir = mxGetIr(S); pr = mxGetPr(S);
    next = (mwIndex*)mxCalloc(n + 1, sizeof(mwIndex));
    for (i = 0; i < n; ++i)
        for (k = rp[i]; k < rp[i + 1]; ++k)
            if (vals[k] != 0.0) next[ci[k] + 1]++;
    for (i = 0; i < n; ++i) next[i + 1] += next[i];
    for (i = 0; i <= n; ++i) jc[i] = next[i];
    for (i = 0; i < n; ++i)  /* rows in increasing order: each column's rows come out sorted */
        for (k = rp[i]; k < rp[i + 1]; ++k)
            if (vals[k] != 0.0) { ir[next[ci[k]]] = (mwIndex)i; pr[next[ci[k]]] = vals[k]; next[ci[k]]++; }
    mxFree(next); mxFree(rp); mxFree(ci);
    return S;
}

/* A dense vector as an n x 1 sparse (MATLAB's Tint-Fext is sparse-typed). */
static inline mxArray* ua_mex_sparse_vector(int32_t n, const double* v) {
    int32_t i, nz = 0;
    mxArray* S;
    mwIndex *jc, *ir;
    double* pr;
    for (i = 0; i < n; ++i) nz += v[i] != 0.0;
    S = mxCreateSparse(n, 1, nz > 0 ? nz : 1, mxREAL);
    jc = mxGetJc(S); ir = mxGetIr(S); pr = mxGetPr(S);
    jc[0] = 0;
    nz = 0;
    for (i = 0; i < n; ++i)
        if (v[i] != 0.0) { ir[nz] = (mwIndex)i; pr[nz] = v[i]; ++nz; }
    jc[1] = (mwIndex)nz;
    return S;
}

#endif
