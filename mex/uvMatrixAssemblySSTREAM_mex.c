/*
 * [Ruv,Kuv,Tint,Fext] = uvMatrixAssemblySSTREAM_mex(CtrlVar,MUA,F,BCs)
 *
 * Drop-in for uvMatrixAssemblySSTREAM.m:6 (called from uvMatrixAssembly.m:77
 * in the "sstream" case).  Honors CtrlVar.uvMatrixAssembly.Ronly and
 * CtrlVar.uvAssembly.ZeroFields (uvMatrixAssemblySSTREAM.m:17-28).  Ruv, Tint
 * and Fext are 2Nn x 1 sparse (as MATLAB's sparse-typed Tint-Fext); Kuv is
 * 2Nn x 2Nn sparse, symmetrised, exact zeros dropped.  Kuv is [] when Ronly.
 */
#include "ua_mex_common.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    const mxArray *C, *MUA, *F, *B;
    ua_params p;
    ua_fields f;
    ua_bcs b;
    ua_mesh* m;
    int Ronly = 0, Zero = 0, mode, rc;
    int32_t nn, neq;
    int64_t nnz = 0;
    double *R, *K = NULL, *T = NULL, *Fx = NULL, *own[8];
    const char* names[8] = {"h", "S", "B", "rho", "AGlen", "n", "C", "m"};
    const double* src[8];
    double* own_drag[11];
    int k;

    if (nrhs != 4) mexErrMsgIdAndTxt("Ua:mex:nargin", "uvMatrixAssemblySSTREAM_mex(CtrlVar,MUA,F,BCs)");
    C = prhs[0]; MUA = prhs[1]; F = prhs[2]; B = prhs[3];
    ua_mex_params(C, &p);
    {
        const mxArray* a = ua_mex_field(C, "uvMatrixAssembly", 0);
        const mxArray* z = ua_mex_field(C, "uvAssembly", 0);
        Ronly = a ? (int)ua_mex_scalar(a, "Ronly", 0) : 0;
        Zero = z ? (int)ua_mex_scalar(z, "ZeroFields", 0) : 0;
    }
    m = ua_mex_mesh(MUA);
    nn = (int32_t)mxGetM(ua_mex_field(MUA, "coordinates", 1));
    neq = 2 * nn;
    memset(&f, 0, sizeof(f));
    f.location = UA_HOST;
    for (k = 0; k < 8; ++k) src[k] = ua_mex_nodal(F, names[k], nn, &own[k]);
    f.h = src[0]; f.S = src[1]; f.B = src[2]; f.rho = src[3];
    f.AGlen = src[4]; f.n = src[5]; f.C = src[6]; f.m = src[7];
    ua_mex_drag_fields(F, nn, &f, own_drag);
    f.ub = mxGetPr(ua_mex_field(F, "ub", 1));
    f.vb = mxGetPr(ua_mex_field(F, "vb", 1));
    f.rhow = ua_mex_scalar(F, "rhow", 1030.0);
    f.g = ua_mex_scalar(F, "g", 9.81 / 1000);
    f.alpha = ua_mex_scalar(F, "alpha", 0.0);
    ua_mex_bcs(B, &b);
    mode = Zero ? UA_ASM_ZERO_R : (Ronly ? UA_ASM_R : UA_ASM_RK);
    R = (double*)mxMalloc(neq * sizeof(double));
    if (nlhs > 2) T = (double*)mxMalloc(neq * sizeof(double));
    if (nlhs > 3) Fx = (double*)mxMalloc(neq * sizeof(double));
    if (mode == UA_ASM_RK) {
        ua_mesh_pattern(m, 0, &nnz, NULL, NULL);
        K = (double*)mxMalloc(nnz * sizeof(double));
    }
    rc = ua_uv_assemble(m, &p, &f, &b, mode, R, K, T, Fx);
    for (k = 0; k < 8; ++k) if (own[k]) mxFree(own[k]);
    for (k = 0; k < 11; ++k) if (own_drag[k]) mxFree(own_drag[k]);
    if (rc != UA_OK) ua_mex_fail(rc);
    plhs[0] = ua_mex_sparse_vector(neq, R);
    if (nlhs > 1) plhs[1] = K ? ua_mex_sparse(m, neq, K) : mxCreateDoubleMatrix(0, 0, mxREAL);
    if (nlhs > 2) plhs[2] = ua_mex_sparse_vector(neq, T);
    if (nlhs > 3) plhs[3] = ua_mex_sparse_vector(neq, Fx);
    mxFree(R);
    if (K) mxFree(K);
    if (T) mxFree(T);
    if (Fx) mxFree(Fx);
}
