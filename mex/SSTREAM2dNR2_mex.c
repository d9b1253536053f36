/*
 * [ub,vb,lubvb,Kuv,Ruv,info,Lubvb] = SSTREAM2dNR2_mex(CtrlVar,MUA,BCs,F,l)
 *
 * Drop-in for the Newton solve SSTREAM2dNR2.m:3 (called from uv.m:104),
 * including the reset-and-retry of uv.m:107-112.  `l` is the l.ubvb vector
 * (may be []).  `info` is a struct with the RunInfo.Forward fields
 * uvConverged, uvIterations, uvResidual, uvBackTrackSteps, rForce and rWork.
 * Lubvb is the constraint matrix L of the BCs (nc x 2Nn sparse), the
 * reference's last output.
 */
#include "ua_mex_common.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    const mxArray *C, *MUA, *B, *F, *L;
    ua_params p;
    ua_fields f;
    ua_bcs b;
    ua_mesh* m;
    ua_newton_report rep;
    ua_newton_iter recs[256];
    int32_t nn, nc = 0;
    int64_t nnz = 0;
    double *ub, *vb, *lam, *K = NULL, *R = NULL, *own[8];
    const char* names[8] = {"h", "S", "B", "rho", "AGlen", "n", "C", "m"};
    const double* src[8];
    double* own_drag[11];
    int k, rc;

    if (nrhs < 4) mexErrMsgIdAndTxt("Ua:mex:nargin", "SSTREAM2dNR2_mex(CtrlVar,MUA,BCs,F,l)");
    C = prhs[0]; MUA = prhs[1]; B = prhs[2]; F = prhs[3]; L = nrhs > 4 ? prhs[4] : NULL;
    ua_mex_params(C, &p);
    m = ua_mex_mesh(MUA);
    nn = (int32_t)mxGetM(ua_mex_field(MUA, "coordinates", 1));
    memset(&f, 0, sizeof(f));
    f.location = UA_HOST;
    for (k = 0; k < 8; ++k) src[k] = ua_mex_nodal(F, names[k], nn, &own[k]);
    f.h = src[0]; f.S = src[1]; f.B = src[2]; f.rho = src[3];
    f.AGlen = src[4]; f.n = src[5]; f.C = src[6]; f.m = src[7];
    ua_mex_drag_fields(F, nn, &f, own_drag);
    plhs[0] = mxCreateDoubleMatrix(nn, 1, mxREAL);
    plhs[1] = mxCreateDoubleMatrix(nn, 1, mxREAL);
    ub = mxGetPr(plhs[0]); vb = mxGetPr(plhs[1]);
    memcpy(ub, mxGetPr(ua_mex_field(F, "ub", 1)), nn * sizeof(double));
    memcpy(vb, mxGetPr(ua_mex_field(F, "vb", 1)), nn * sizeof(double));
    f.ub = ub; f.vb = vb;
    f.rhow = ua_mex_scalar(F, "rhow", 1030.0);
    f.g = ua_mex_scalar(F, "g", 9.81 / 1000);
    f.alpha = ua_mex_scalar(F, "alpha", 0.0);
    ua_mex_bcs(B, &b);
    ua_constraint_count(m, &b, 2, &nc);
    lam = (double*)mxCalloc(nc > 0 ? nc : 1, sizeof(double));
    if (L && (int32_t)mxGetNumberOfElements(L) == nc && nc > 0) memcpy(lam, mxGetPr(L), nc * sizeof(double));
    memset(&rep, 0, sizeof(rep));
    rep.iters = recs;
    rep.iters_capacity = 256;
    if (nlhs > 3) {
        ua_mesh_pattern(m, 0, &nnz, NULL, NULL);
        K = (double*)mxMalloc(nnz * sizeof(double));
        R = (double*)mxMalloc(2 * nn * sizeof(double));
    }
    rc = ua_uv_newton(m, &p, &f, &b, lam, nc, &rep, K, R);
    for (k = 0; k < 8; ++k) if (own[k]) mxFree(own[k]);
    for (k = 0; k < 11; ++k) if (own_drag[k]) mxFree(own_drag[k]);
    if (rc != UA_OK && rc != UA_ERR_NOT_CONVERGED) ua_mex_fail(rc);
    if (nlhs > 2) {
        plhs[2] = mxCreateDoubleMatrix(nc, 1, mxREAL);
        if (nc) memcpy(mxGetPr(plhs[2]), lam, nc * sizeof(double));
    }
    if (nlhs > 3) plhs[3] = ua_mex_sparse(m, 2 * nn, K);
    if (nlhs > 4) plhs[4] = ua_mex_sparse_vector(2 * nn, R);
    if (nlhs > 5) {
        const char* fn[6] = {"uvConverged", "uvIterations", "uvResidual", "uvBackTrackSteps", "rForce", "rWork"};
        mxArray* s = mxCreateStructMatrix(1, 1, 6, fn);
        mxSetField(s, 0, "uvConverged", mxCreateDoubleScalar(rep.converged));
        mxSetField(s, 0, "uvIterations", mxCreateDoubleScalar(rep.iterations));
        mxSetField(s, 0, "uvResidual", mxCreateDoubleScalar(rep.r));
        mxSetField(s, 0, "uvBackTrackSteps", mxCreateDoubleScalar(rep.backtrack_steps));
        mxSetField(s, 0, "rForce", mxCreateDoubleScalar(rep.rForce));
        mxSetField(s, 0, "rWork", mxCreateDoubleScalar(rep.rWork));
        plhs[5] = s;
    }
    if (nlhs > 6) plhs[6] = ua_mex_constraint_L(m, &b, 2 * nn);
    mxFree(lam);
    if (K) mxFree(K);
    if (R) mxFree(R);
}
