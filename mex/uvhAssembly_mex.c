/*
 * [R,K] = uvhAssembly_mex(CtrlVar,MUA,F0,F1)
 *
 * Drop-in for the assembly of uvhAssembly.m:1 -> uvhMatrixAssembly.m:6-585
 * (integration points uvhAssemblyIntPointImplicitSUPG.m:10-531, nodal loop
 * uvhNodalLoopSSTREAM.m:1-229).  F0 holds the state at t (h, ub, vb, as, ab),
 * F1 the values at t+dt (h, ub, vb, as, ab; dasdh + dabdh when
 * CtrlVar.MassBalanceGeometryFeedback is 3) and the
 * time-independent fields; the time step is CtrlVar.dt.  Honors
 * CtrlVar.uvhMatrixAssembly.ZeroFields and .Ronly.  R is 3Nn x 1
 * sparse-typed, K the unsymmetric 3Nn x 3Nn sparse tangent ([] when Ronly).
 */
#include "ua_mex_common.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    const mxArray *C, *MUA, *F0, *F1;
    ua_params p;
    ua_fields f;
    ua_mesh* m;
    int Ronly = 0, Zero = 0, mode, rc, k;
    int32_t nn, neq;
    int64_t nnz = 0;
    double *R, *K = NULL, *own[14];
    double* own_drag[11];
    const char* names[8] = {"h", "S", "B", "rho", "AGlen", "n", "C", "m"};
    const double* src[8];

    if (nrhs != 4) mexErrMsgIdAndTxt("Ua:mex:nargin", "uvhAssembly_mex(CtrlVar,MUA,F0,F1)");
    C = prhs[0]; MUA = prhs[1]; F0 = prhs[2]; F1 = prhs[3];
    ua_mex_params(C, &p);
    {
        const mxArray* a = ua_mex_field(C, "uvhMatrixAssembly", 0);
        Ronly = a ? (int)ua_mex_scalar(a, "Ronly", 0) : 0;
        Zero = a ? (int)ua_mex_scalar(a, "ZeroFields", 0) : 0;
    }
    m = ua_mex_mesh_ndof(MUA, 3);
    nn = (int32_t)mxGetM(ua_mex_field(MUA, "coordinates", 1));
    neq = 3 * nn;
    memset(&f, 0, sizeof(f));
    memset(own, 0, sizeof(own));
    f.location = UA_HOST;
    for (k = 0; k < 8; ++k) src[k] = ua_mex_nodal(F1, names[k], nn, &own[k]);
    f.h = src[0]; f.S = src[1]; f.B = src[2]; f.rho = src[3];
    f.AGlen = src[4]; f.n = src[5]; f.C = src[6]; f.m = src[7];
    ua_mex_drag_fields(F1, nn, &f, own_drag);
    f.ub = mxGetPr(ua_mex_field(F1, "ub", 1));
    f.vb = mxGetPr(ua_mex_field(F1, "vb", 1));
    f.h1 = (double*)src[0];
    f.h0 = ua_mex_nodal(F0, "h", nn, &own[8]);
    f.u0 = mxGetPr(ua_mex_field(F0, "ub", 1));
    f.v0 = mxGetPr(ua_mex_field(F0, "vb", 1));
    f.as0 = ua_mex_nodal(F0, "as", nn, &own[9]);
    f.ab0 = ua_mex_nodal(F0, "ab", nn, &own[10]);
    f.as1 = ua_mex_nodal(F1, "as", nn, &own[11]);
    f.ab1 = ua_mex_nodal(F1, "ab", nn, &own[12]);
    f.dadh = ua_mex_dadh(C, F1, nn, &own[13]);
    f.rhow = ua_mex_scalar(F1, "rhow", 1030.0);
    f.g = ua_mex_scalar(F1, "g", 9.81 / 1000);
    f.alpha = ua_mex_scalar(F1, "alpha", 0.0);
    f.dt = ua_mex_scalar(C, "dt", 1.0);
    mode = Zero ? UA_ASM_ZERO_R : (Ronly ? UA_ASM_R : UA_ASM_RK);
    R = (double*)mxMalloc(neq * sizeof(double));
    if (mode == UA_ASM_RK) {
        ua_mesh_pattern(m, 0, &nnz, NULL, NULL);
        K = (double*)mxMalloc(nnz * sizeof(double));
    }
    rc = ua_uvh_assemble(m, &p, &f, mode, R, K, NULL, NULL);
    for (k = 0; k < 14; ++k) if (own[k]) mxFree(own[k]);
    for (k = 0; k < 11; ++k) if (own_drag[k]) mxFree(own_drag[k]);
    if (rc != UA_OK) ua_mex_fail(rc);
    plhs[0] = ua_mex_sparse_vector(neq, R);
    if (nlhs > 1) plhs[1] = K ? ua_mex_sparse_unsym(m, neq, K) : mxCreateDoubleMatrix(0, 0, mxREAL);
    mxFree(R);
    if (K) mxFree(K);
}
