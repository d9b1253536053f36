/*
 * [ub,vb,h,luvh,info] = SSTREAM_TransientImplicit_mex(CtrlVar,MUA,BCs1,F0,F1,l1)
 *
 * Drop-in for the implicit uvh step uvh.m:5-222 -> uvh2D.m:20 ->
 * SSTREAM_TransientImplicit.m:6-717, with the minimum-thickness active set of
 * uvh.m:64-212 when CtrlVar.ThicknessConstraints is 1 (BCs1.hPosNode, 1-based,
 * the set carried from the previous step).  F0: state at t; F1: start values at
 * t+dt and the time-independent fields; CtrlVar.dt the time step.  l1 is
 * [l.ubvb; l.h] (may be []).  info carries uvhConverged, uvhIterations, the last
 * residual and backtracking steps, and with the active set hPosNode (the final
 * set, 1-based: BCs1.hPosNode for the next step), activeSetIterations,
 * activeSetConverged and activeSetCyclical.
 */
#include "ua_mex_common.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    const mxArray *C, *MUA, *B, *F0, *F1, *L;
    ua_params p;
    ua_fields f;
    ua_bcs b;
    ua_mesh* m;
    ua_newton_report rep;
    ua_newton_iter recs[256];
    int32_t nn, nc = 0;
    double *ub, *vb, *h, *lam, *own[14];
    int32_t* hpos;
    const char* names[8] = {"h", "S", "B", "rho", "AGlen", "n", "C", "m"};
    const double* src[8];
    double* own_drag[11];
    int k, rc;

    if (nrhs < 5) mexErrMsgIdAndTxt("Ua:mex:nargin", "SSTREAM_TransientImplicit_mex(CtrlVar,MUA,BCs1,F0,F1,l1)");
    C = prhs[0]; MUA = prhs[1]; B = prhs[2]; F0 = prhs[3]; F1 = prhs[4]; L = nrhs > 5 ? prhs[5] : NULL;
    ua_mex_params(C, &p);
    p.precision = UA_PREC_FP64;  /* the uvh step runs in FP64 */
    m = ua_mex_mesh_ndof(MUA, 3);
    nn = (int32_t)mxGetM(ua_mex_field(MUA, "coordinates", 1));
    memset(&f, 0, sizeof(f));
    memset(own, 0, sizeof(own));
    f.location = UA_HOST;
    for (k = 0; k < 8; ++k) src[k] = ua_mex_nodal(F1, names[k], nn, &own[k]);
    f.h = src[0]; f.S = src[1]; f.B = src[2]; f.rho = src[3];
    f.AGlen = src[4]; f.n = src[5]; f.C = src[6]; f.m = src[7];
    ua_mex_drag_fields(F1, nn, &f, own_drag);
    plhs[0] = mxCreateDoubleMatrix(nn, 1, mxREAL);
    plhs[1] = mxCreateDoubleMatrix(nn, 1, mxREAL);
    plhs[2] = mxCreateDoubleMatrix(nn, 1, mxREAL);
    ub = mxGetPr(plhs[0]); vb = mxGetPr(plhs[1]); h = mxGetPr(plhs[2]);
    memcpy(ub, mxGetPr(ua_mex_field(F1, "ub", 1)), nn * sizeof(double));
    memcpy(vb, mxGetPr(ua_mex_field(F1, "vb", 1)), nn * sizeof(double));
    memcpy(h, src[0], nn * sizeof(double));
    f.ub = ub; f.vb = vb; f.h1 = h;
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
    ua_mex_bcs(B, &b);
    ua_constraint_count(m, &b, 3, &nc);
    lam = (double*)mxCalloc(nc > 0 ? nc : 1, sizeof(double));
    if (L && (int32_t)mxGetNumberOfElements(L) == nc && nc > 0) memcpy(lam, mxGetPr(L), nc * sizeof(double));
    memset(&rep, 0, sizeof(rep));
    rep.iters = recs;
    rep.iters_capacity = 256;
    hpos = (int32_t*)mxCalloc(nn > 0 ? nn : 1, sizeof(int32_t));
    rep.hpos_node = hpos;
    rep.hpos_capacity = nn;
    rc = ua_uvh_newton(m, &p, &f, &b, lam, nc, &rep);
    for (k = 0; k < 14; ++k) if (own[k]) mxFree(own[k]);
    for (k = 0; k < 11; ++k) if (own_drag[k]) mxFree(own_drag[k]);
    if (rc != UA_OK && rc != UA_ERR_NOT_CONVERGED) ua_mex_fail(rc);
    if (nlhs > 3) {
        plhs[3] = mxCreateDoubleMatrix(nc, 1, mxREAL);
        if (nc) memcpy(mxGetPr(plhs[3]), lam, nc * sizeof(double));
    }
    if (nlhs > 4) {
        const char* fn[10] = {"uvhConverged", "uvhIterations", "uvhResidual", "uvhBackTrackSteps", "rForce", "rWork",
                              "hPosNode", "activeSetIterations", "activeSetConverged", "activeSetCyclical"};
        mxArray* s = mxCreateStructMatrix(1, 1, p.ThicknessConstraints ? 10 : 6, fn);
        mxSetField(s, 0, "uvhConverged", mxCreateDoubleScalar(rep.converged));
        mxSetField(s, 0, "uvhIterations", mxCreateDoubleScalar(rep.iterations));
        mxSetField(s, 0, "uvhResidual", mxCreateDoubleScalar(rep.r));
        mxSetField(s, 0, "uvhBackTrackSteps", mxCreateDoubleScalar(rep.backtrack_steps));
        mxSetField(s, 0, "rForce", mxCreateDoubleScalar(rep.rForce));
        mxSetField(s, 0, "rWork", mxCreateDoubleScalar(rep.rWork));
        if (p.ThicknessConstraints) {
            mxArray* hp = mxCreateDoubleMatrix(rep.n_hpos, 1, mxREAL);
            for (k = 0; k < rep.n_hpos; ++k) mxGetPr(hp)[k] = (double)hpos[k] + 1.0;
            mxSetField(s, 0, "hPosNode", hp);
            mxSetField(s, 0, "activeSetIterations", mxCreateDoubleScalar(rep.active_set_iterations));
            mxSetField(s, 0, "activeSetConverged", mxCreateDoubleScalar(rep.active_set_converged));
            mxSetField(s, 0, "activeSetCyclical", mxCreateDoubleScalar(rep.active_set_cyclical));
        }
        plhs[4] = s;
    }
    mxFree(hpos);
    mxFree(lam);
}
