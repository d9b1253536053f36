/*
 * ua_ssa.h — C-ABI of the B200 SSA (SSTREAM) Newton library (libuassa.so).
 *
 * Drop-in boundary for Úa's shallow-shelf hot path.  Each entry point names
 * the reference MATLAB function it replaces (paths relative to the Úa source
 * tree).  The MEX gateways under mex/ marshal MATLAB structs into these
 * plain-pointer calls; Python binds the same symbols with ctypes.
 *
 * Conventions
 *  - All arrays are caller-owned.  Host pointers unless a struct says
 *    otherwise (ua_fields.location).  The library owns all device memory.
 *  - Node and element indices follow ua_mesh_desc.index_base (1 for MATLAB).
 *  - Connectivity is Nele x nod, column-major (MATLAB layout): entry (e,a) is
 *    connectivity[a*Nele + e].  Coordinates are Nnodes x 2 column-major.
 *  - Degrees of freedom are ordered as in Úa: [u(1..Nn); v(1..Nn); h(1..Nn)].
 *  - The tangent is returned on the structural pattern of the mesh (every
 *    pair of nodes sharing an element), CSR with sorted columns; for the uv
 *    system CSR == CSC because the pattern is symmetric.  ua_mesh_pattern()
 *    gives the pattern.  MATLAB's sparse() drops exact zeros; the MEX gateway
 *    does the same when it builds the mxArray.
 *  - Status: 0 = OK, negative = error (UA_ERR_*).  ua_last_error() returns a
 *    message for the last failing call on the calling thread.
 *  - Thread safety: one handle per thread; calls on one handle are serialised
 *    on the handle's CUDA stream.
 */
#ifndef UA_SSA_H
#define UA_SSA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UA_OK                 0
#define UA_ERR_INVALID       -1   /* bad argument / size */
#define UA_ERR_NAN_INPUT     -2   /* uvMatrixAssembly:NaN, SSTREAM2dNR2.m:42-66 */
#define UA_ERR_NOT_CONVERGED -3   /* RunInfo.Forward.uvConverged=0 */
#define UA_ERR_OOM           -4   /* device allocation failed / admission */
#define UA_ERR_TIMEOUT       -5   /* bounded device wait expired */
#define UA_ERR_BAD_MESH      -6   /* degenerate element (detJ==0) or bad index */
#define UA_ERR_CUDA          -7   /* CUDA runtime error */
#define UA_ERR_KRYLOV        -8   /* Krylov breakdown / iteration cap */
#define UA_ERR_NO_DEVICE     -9   /* no CUDA device or extension unusable */

/* Precision forms. */
#define UA_PREC_FP64   0   /* all FP64 (the plain form) */
#define UA_PREC_MIXED  1   /* FP32 element tangents + FP32 PCG with FP64 reductions */

/* preconditioners of the inner uv solve */
#define UA_PC_JACOBI 0   /* point Jacobi */
#define UA_PC_AMG    1   /* aggregation AMG V(1,1) cycle, l1-Jacobi smoother (default) */

/* inner solvers of the unsymmetric uvh system (both constrained, preconditioned by AMG on the
   velocity block and a block lower-triangular thickness step, or point Jacobi) */
#define UA_KRYLOV_GMRES    0   /* restarted GMRES(m), right-preconditioned (default) */
#define UA_KRYLOV_BICGSTAB 1   /* BiCGStab with restarts on breakdown */

/* CtrlVar.SlidingLaw (Ua2D_DefaultParameters.m:171-172, BasalDrag.m:184-272). */
#define UA_SLIDING_WEERTMAN 0   /* "Weertman", "W" (default) */
#define UA_SLIDING_BUDD     1   /* "Budd", "W-N0": uses F.q */
#define UA_SLIDING_TSAI     2   /* "Tsai", "minCW-N0": uses F.muk */
#define UA_SLIDING_COULOMB  3   /* "Coulomb", "C": uses F.muk */
#define UA_SLIDING_CORNFORD 4   /* "Cornford", "rpCW-N0": uses F.muk */
#define UA_SLIDING_UMBI     5   /* "Umbi", "rCW-N0": uses F.muk */
#define UA_SLIDING_JOUGHIN  6   /* "Joughin", "rCW-V0": uses F.V0 */

/* Assembly modes of uvMatrixAssembly (uvMatrixAssemblySSTREAM.m:17-28). */
#define UA_ASM_R      0   /* CtrlVar.uvMatrixAssembly.Ronly=true */
#define UA_ASM_RK     1   /* R and K */
#define UA_ASM_ZERO_R 2   /* CtrlVar.uvAssembly.ZeroFields=true, Ronly */

/* Field location. */
#define UA_HOST   0
#define UA_DEVICE 1

typedef struct ua_mesh ua_mesh;   /* opaque device-resident mesh (MUA) */

/* One mesh: MUA.coordinates / MUA.connectivity (CreateMUA.m:31-98). */
typedef struct ua_mesh_desc {
    int32_t nnodes;
    int32_t nele;
    int32_t nod;                 /* 3 (P1) or 6 (P2) */
    int32_t index_base;          /* 1 for MATLAB, 0 for C/Python */
    const double*  coordinates;  /* nnodes x 2, column-major */
    const int32_t* connectivity; /* nele x nod, column-major */
} ua_mesh_desc;

/* CtrlVar fields that change hot-path arithmetic (defaults from
 * Ua2D_DefaultParameters.m; ua_params_default() fills them). */
typedef struct ua_params {
    double kH, Hh0;                               /* :2288, :2295 */
    double SpeedZero, EpsZero, etaZero;           /* :412, :413, :415 */
    double Czero, Cmin, AGlenmin;                 /* :441, :456-460, :463 */
    int32_t Picard;                               /* :593 */
    double NRviscosity;                           /* :594 */
    int32_t NRitmax, NRitmin;                     /* :597, :600 */
    double NewtonAcceptRatio;                     /* :601 */
    double BacktrackingGammaMin;                  /* :604 */
    int32_t LineSearchAllowedToUseExtrapolation;  /* :603 */
    double BackTrackBeta;                         /* :616 */
    int32_t BackTrackMaxIterations;               /* :617 */
    int32_t BackTrackMaxExtrapolations;           /* :618 */
    double BackTrackExtrapolationRatio;           /* :619 */
    double BackTrackMinXfrac;                     /* :620 */
    int32_t BackTrackMaxFuncSame;                 /* :621 */
    double BackTrackGuardLower, BackTrackGuardUpper; /* :625-626 */
    double NLtol;                                 /* BackTracking.m:125-127 */
    double uvDesiredWorkAndForceTolerances[2];    /* :508 */
    double uvDesiredWorkOrForceTolerances[2];     /* :509 */
    double uvExitBackTrackingStepLength;          /* :510 */
    double uvAcceptableWorkAndForceTolerances[2]; /* :511 */
    double uvAcceptableWorkOrForceTolerances[2];  /* :512 */
    int32_t ModifiedNRuvIntervalCriterion;        /* :582 */
    double ModifiedNRuvReductionCriterion;        /* :583 */
    /* uvh */
    double theta, SUPG_beta0, uvh_SUPG_tauMultiplier; /* :377, :376, :555 */
    int32_t uvh_SUPG_tau;                         /* 0=taus (:551), 1=taut, 2=tau1, 3=tau2 */
    double uvhDesiredWorkAndForceTolerances[2];   /* :496 */
    double uvhDesiredWorkOrForceTolerances[2];    /* :498 */
    double uvhExitBackTrackingStepLength;         /* :502 */
    double uvhAcceptableWorkAndForceTolerances[2];/* :504 */
    double uvhAcceptableWorkOrForceTolerances[2]; /* :505 */
    /* inner Krylov solve (replaces ABfgPreEliminate.m:110 decomposition) */
    double krylov_rtol;        /* relative residual of the preconditioned solve */
    int32_t krylov_maxit;
    int32_t precision;         /* UA_PREC_* */
    int32_t patch_nodes;       /* nodes per assembly patch (one CTA each): 0 = the schedule ua_autotune chose
                                  for this device, element type and dof count, else the default shape
                                  (clamp(Nnodes/600, 16, 128) per system); > 0 = that many */
    int32_t verbose;           /* per-iteration log line to stderr */
    int32_t profile;           /* 1: time assembly and SpMV launches with CUDA events */
    int32_t krylov_adaptive;   /* 1: inner tolerance eta_k = clamp(c*sqrt(rForce_k), krylov_rtol, max)
                                  (inexact Newton forcing term); 0: krylov_rtol every iteration */
    int32_t krylov_precond;    /* UA_PC_*: preconditioner of the uv inner PCG; for uvh, UA_PC_AMG selects
                                  the block preconditioner (AMG V-cycle on the velocity block, l1-Jacobi
                                  sweeps on the thickness block) and UA_PC_JACOBI point Jacobi */
    int32_t spmv_lanes;        /* lanes per row of the uv PCG/AMG row products: 0 = by element type
                                  (1 for P1, 2 for P2), else 1, 2, 4, 8, 16 or 32 */
    int32_t asm_threads;       /* CTA size of the P1 uv assembly: 0 = the tuned one (ua_autotune), else 256;
                                  or 128 or 256 */
    int32_t asm_regs;          /* register budget of the P1 uv assembly kernel (occupancy against spills):
                                  0 = the tuned one, else 128; or 128, 96 (128-thread CTAs only) or 80 */
    int32_t uvh_krylov;        /* UA_KRYLOV_*: inner solver of the unsymmetric uvh system */
    int32_t krylov_restart;    /* GMRES restart length m (uvh) */
    double krylov_eta_c, krylov_eta_max;  /* uv forcing term eta = clamp(c*sqrt(rForce), krylov_rtol, max) */
    int32_t precond_bf16;      /* mixed precision: 1 = the AMG V-cycle's finest-level passes read a BF16
                                  copy of the tangent (the PCG operator stays FP32) */
    int32_t amg_smoothed;      /* 1 = smoothed-aggregation prolongators (default), 0 = plain aggregation;
                                  fixed by a handle's first AMG solve */
    int32_t krylov_full_grid;  /* 0 = the AMG-preconditioned PCG launches only the row and node blocks of
                                  systems still iterating (device-compacted lists, default); 1 = every
                                  block of the batch (same results) */
    int32_t amg_P_refresh;     /* smoothed aggregation: recompute each system's prolongators P on the
                                  first Newton step of its solve and then every amg_P_refresh-th step
                                  (0 = by precision: every step in FP64, every fourth in the mixed form;
                                  1 = every step); the coarse operators P'KP always use the current
                                  tangent */
    int32_t uvh_h_sweeps;      /* uvh block preconditioner: l1-Jacobi sweeps on the thickness block K_hh
                                  (0 = default 8) */
    int32_t krylov_sell;       /* 1 = the AMG-preconditioned uv PCG runs its SpMV and the V-cycle's
                                  finest-level passes on node-sliced (sliced ELL) copies of the tangent,
                                  both rows of a node per thread (default); 0 = CSR row kernels */
    int32_t SlidingLaw;        /* UA_SLIDING_* (:171) */
    double Nzero;              /* lower value of the effective pressure (:445) */
    int32_t IncludeMelangeModelPhysics;  /* ocean and atmosphere drag on floating ice (BasalDrag.m:275-343);
                                            needs F.uo, vo, Co, mo, ua, va, Ca, ma */
    /* active-set minimum-thickness constraints of the implicit uvh step (uvh.m:64-212) */
    int32_t ThicknessConstraints;        /* :1478 (1 = active-set method, the default) */
    double ThickMin;                     /* :1469 */
    int32_t ThicknessConstraintsItMax;   /* :1479 */
    int32_t MaxNumberOfNewlyIntroducedActiveThicknessConstraints;  /* :1500 */
    int32_t MinNumberOfNewlyIntroducedActiveThicknessConstraints;  /* :1502 */
} ua_params;

/* Nodal fields F (UaFields.m).  Scalars rhow, g, alpha are F.rhow, F.g, F.alpha. */
typedef struct ua_fields {
    int32_t location;          /* UA_HOST or UA_DEVICE (device pointers on the handle's device) */
    const double *h, *S, *B, *rho, *AGlen, *n, *C, *m;
    double *ub, *vb;           /* in: start / current velocities, out (newton): solution */
    double rhow, g, alpha;
    /* uvh only (SSTREAM_TransientImplicit.m): state at t0 and mass balance */
    const double *h0, *u0, *v0, *as0, *ab0, *as1, *ab1, *dadh;
    double *h1;                /* in: start thickness, out: solution */
    double dt;
    /* sliding-law fields (UaFields.m; NULL where the law does not use them): Budd exponent q,
       Coulomb friction coefficient muk, Joughin speed V0 */
    const double *q, *muk, *V0;
    /* melange: ocean velocity, drag and exponent; atmosphere the same (IncludeMelangeModelPhysics) */
    const double *uo, *vo, *Co, *mo, *ua, *va, *Ca, *ma;
    /* uv Newton (ua_uv_newton, ua_uv_newton_batch): where the solution goes, same location as
       the inputs; NULL = into ub, vb.  With both set, ub and vb are read only (the start
       velocities).  The uvh calls ignore them. */
    double *ub_out, *vb_out;
} ua_fields;

/* Boundary conditions (BCs2MLC.m, CreateLuv.m).  Index base as the mesh.  Fixed nodes, ties
 * (u_A - u_B = 0) and fixed normal velocities become rows of L scaled to unit length (ScaleL.m);
 * the rows must have disjoint support (every dof in at most one constraint), as
 * ABfgPreEliminate.m requires, else UA_ERR_INVALID.  Ties and normal velocities are taken by the
 * uv solves with the AMG preconditioner. */
typedef struct ua_bcs {
    int32_t n_ufixed; const int32_t* ufixed_node; const double* ufixed_value;
    int32_t n_vfixed; const int32_t* vfixed_node; const double* vfixed_value;
    int32_t n_utied;  const int32_t* utied_a; const int32_t* utied_b;
    int32_t n_vtied;  const int32_t* vtied_a; const int32_t* vtied_b;
    int32_t n_hfixed; const int32_t* hfixed_node; const double* hfixed_value;
    int32_t n_hpos; const int32_t* hpos_node;  /* BCs.hPosNode: the active minimum-thickness set on entry
                                                  (the previous step's, may be empty) */
    /* BCs.ubvbFixedNormalNode/Value: Nx u + Ny v = -value with the boundary's nodal normals
       (CreateLuv.m:62-72, CalcEdgeAndNodalNormals.m; uv solves) */
    int32_t n_normal; const int32_t* normal_node; const double* normal_value;
} ua_bcs;

/* One Newton iteration (the SSTREAM2dNR2.m:386-387 log line). */
typedef struct ua_newton_iter {
    int32_t iteration, iarm, krylov_its, direction; /* direction 0=full Newton, 1=backtracked */
    double gamma, r0, r, rForce, rWork;
} ua_newton_iter;

/* RunInfo.Forward subset (UaRunInfo.m:42-98) plus timing. */
typedef struct ua_newton_report {
    int32_t converged;          /* uvConverged */
    int32_t iterations;         /* uvIterations */
    int32_t backtrack_steps;    /* uvBackTrackSteps (last iteration's iarm) */
    int32_t krylov_its_total;
    int32_t cauchy_fallbacks;   /* times rLineminUa.m:96 would continue with the M-Cauchy step */
    int32_t retried;            /* uv.m:107-112 reset-and-retry happened */
    double r, rForce, rWork;    /* uvResidual (= r) */
    double assembly_ms, solve_ms, total_ms;  /* host wall clock of the phases */
    double device_ms;           /* CUDA-event time on the handle's stream, whole call */
    double kasmK_ms, kasmR_ms, kspmv_ms;     /* summed launch durations (profile=1) */
    int32_t kasmK_n, kasmR_n, kspmv_n;       /* launches timed */
    double kamgR_ms, kamgP_ms;  /* fine-level AMG restriction / prolongation+smoothing (profile=1) */
    int32_t kamgR_n, kamgP_n;
    double kwork_nnz[5], kwork_rows[5];  /* per timed class (asmK, asmR, spmv, amgR, amgP): tangent
                                            non-zeros and dof rows of the systems each timed launch
                                            processed, summed over the launches (profile=1) */
    int32_t gpu_launches;       /* kernels launched by the library during the call */
    int32_t n_iter_records;     /* entries filled in iters (<= iters_capacity) */
    int32_t iters_capacity;
    ua_newton_iter* iters;      /* caller-owned, may be NULL */
    /* Newton updates (SSTREAM2dNR2.m:367-369, SSTREAM_TransientImplicit.m:478-483): caller-owned,
     * may be NULL.  Record k (the k-th entry of iters) receives the accepted update of that
     * iteration, gamma*[du; dv; dl] for uv and gamma*[du; dv; dh; dl] for uvh (Úa dof order, then
     * the Lagrange multipliers), at updates + k*update_stride.  update_stride >= ndof*Nnodes + nl,
     * else the call returns UA_ERR_INVALID.  Filled for the first iters_capacity iterations. */
    double* updates;
    int64_t update_stride;
    /* uvh active set (RunInfo.Forward.uvhActiveSet*, uvh.m:205-207) */
    int32_t active_set_iterations;   /* uvhActiveSetIterations */
    int32_t active_set_cyclical;     /* uvhActiveSetCyclical */
    int32_t active_set_converged;    /* ActiveSetConverged (0 when ThicknessConstraintsItMax was reached) */
    int32_t n_hpos;                  /* uvhActiveSetConstraints: the size of the final active set */
    int32_t hpos_capacity;           /* capacity of hpos_node */
    int32_t* hpos_node;              /* caller-owned, may be NULL: the final BCs1.hPosNode (0-based) */
    /* profile=1, uv solves: the AMG numeric set-ups with the node-slice fills, and the whole
       Krylov iterations (SpMV, V-cycles, vector updates, reductions), summed launch-range times */
    double ksetup_ms, kkrylov_ms;
    int32_t ksetup_n, kkrylov_n;
} ua_newton_report;

/* --------------------------------------------------------------------- */

/* Library version string and device check. */
const char* ua_version(void);
const char* ua_last_error(void);
int ua_device_count(void);

/* ABI check for foreign bindings: sizes (bytes) of ua_mesh_desc, ua_params,
 * ua_fields, ua_bcs, ua_newton_iter, ua_newton_report, ua_tune_report, in that order (n <= 7).
 * No counterpart in the reference; it needs no GPU. */
int ua_struct_sizes(int64_t* sizes, int32_t n);

/* Fill CtrlVar defaults (Ua2D_DefaultParameters.m lines cited in ua_params). */
void ua_params_default(ua_params* p);

/* MUA setup: CreateMUA.m:31-98 (element orientation check as
 * TestAndCorrectForInsideOutElements.m, quadrature per QuadratureRuleDegree.m)
 * plus the symbolic CSR pattern, node patches and the element-to-CSR
 * contribution map used by the deterministic segmented-sum scatter.
 * ndof = 2 (uv) or 3 (uvh).  device = CUDA ordinal. */
int ua_mesh_create(const ua_mesh_desc* desc, int32_t ndof, int32_t device, ua_mesh** out);

/* Batched form: several independent meshes in one handle (one system each);
 * every stage of the Newton solve runs for all systems in the same launches. */
int ua_mesh_create_batch(const ua_mesh_desc* descs, int32_t count, int32_t ndof, int32_t device,
                         ua_mesh** out);
void ua_mesh_destroy(ua_mesh* m);

/* Structural pattern of the ndof-block tangent of system `sys`:
 * nnz, row pointer (nrows+1) and column indices (0-based, sorted).
 * Pass NULL arrays to query nnz only. */
int ua_mesh_pattern(const ua_mesh* m, int32_t sys, int64_t* nnz, int64_t* rowptr, int64_t* colind);

/* Number of systems, nodes and elements of system `sys`; device bytes held. */
int ua_mesh_info(const ua_mesh* m, int32_t sys, int32_t* nsys, int32_t* nnodes, int32_t* nele,
                 int64_t* device_bytes);

/* Elements flipped by the inside-out correction (0 when all had detJ>0). */
int ua_mesh_flipped(const ua_mesh* m, int32_t* nflipped);

/* uvMatrixAssembly (uvMatrixAssembly.m:5, uvMatrixAssemblySSTREAM.m:6-553)
 * for system 0 of a single-mesh handle.  mode = UA_ASM_*.
 * R: 2*Nnodes (Tint-Fext, uvMatrixAssemblySSTREAM.m:483-488);
 * K: nnz values on the structural pattern, symmetrised as (K+K.')/2
 * (uvMatrixAssemblySSTREAM.m:530-531); NULL for mode R. Tint/Fext optional. */
int ua_uv_assemble(ua_mesh* m, const ua_params* p, const ua_fields* F, const ua_bcs* bcs,
                   int32_t mode, double* R, double* Kvals, double* Tint, double* Fext);

/* Assembly autotuner.  Times the tangent+residual uv assembly of the handle's systems at the
 * fields F (nF = 1 or one per system) for each candidate schedule, reps launches each: patch
 * shapes pn = clamp(nn/div, 16, cap) nodes per patch (div = 0: cap nodes) and, for P1, CTAs of
 * 256 or 128 threads with register budgets of 128, 96 (128 threads) or 80 per thread.  The
 * fastest becomes the handle's schedule and the process-wide tuned schedule of (device, nod,
 * ndof), which handles then use when patch_nodes, asm_threads and asm_regs are 0.
 * K and R are bit-identical under every schedule.  Needs an ndof=2 handle. */
#define UA_TUNE_MAX 48
typedef struct {
    int32_t n_candidates;
    int32_t div[UA_TUNE_MAX], cap[UA_TUNE_MAX], threads[UA_TUNE_MAX], regs[UA_TUNE_MAX];
    double ms[UA_TUNE_MAX];    /* mean time of one assembly launch per candidate */
    int32_t chosen;            /* index of the fastest */
    double default_ms;         /* candidate 0: the default schedule */
} ua_tune_report;
int ua_autotune(ua_mesh* m, const ua_params* p, const ua_fields* F, int32_t nF, int32_t reps,
                ua_tune_report* rep);

/* Whole uv Newton solve: SSTREAM2dNR2.m:3-431 with the reset-and-retry of
 * uv.m:107-112.  F->ub/F->vb: start values in, solution out.  lubvb: Lagrange
 * multipliers l.ubvb (length = number of constraints), in/out, may be NULL.
 * Kvals/R (optional): the last tangent and residual, as returned by SSTREAM2dNR2. */
int ua_uv_newton(ua_mesh* m, const ua_params* p, ua_fields* F, const ua_bcs* bcs,
                 double* lubvb, int32_t nl, ua_newton_report* rep, double* Kvals, double* R);

/* Batched uv Newton: fields[i], bcs[i], reports[i] for system i of a batch
 * handle.  All systems advance together; converged ones stop contributing. */
int ua_uv_newton_batch(ua_mesh* m, const ua_params* p, ua_fields* fields, const ua_bcs* bcs,
                       ua_newton_report* reports);

/* uvhAssembly (uvhAssembly.m:1 -> uvhMatrixAssembly.m:6-585, integration
 * points uvhAssemblyIntPointImplicitSUPG.m:10-531, nodal loop
 * uvhNodalLoopSSTREAM.m:1-229) for a single-mesh ndof=3 handle.  Level 1 is
 * F->ub, F->vb, F->h1 (u, v, h at t+dt); level 0 is F->h0, u0, v0, as0, ab0;
 * F->as1, ab1, dadh (NULL = 0) the mass balance; F->dt the time step.
 * mode UA_ASM_ZERO_R is CtrlVar.uvhMatrixAssembly.ZeroFields.  R: 3*Nnodes;
 * K: the unsymmetric tangent on the structural pattern (9 blocks per node pair). */
int ua_uvh_assemble(ua_mesh* m, const ua_params* p, const ua_fields* F, int32_t mode,
                    double* R, double* Kvals, double* Tint, double* Fext);

/* Implicit uvh step: uvh.m:5-222 -> uvh2D.m:20 -> SSTREAM_TransientImplicit.m:6-717.  With
 * p->ThicknessConstraints the step runs inside the active-set loop of uvh.m:64-212
 * (ActiveSetInitialisation.m, ActiveSetUpdate.m): nodes with h < ThickMin are fixed at ThickMin,
 * constraints whose mass-flux reaction -Reactions.h/(rho dt) is negative are released
 * (CalculateReactions.m: Reactions.h = M \ Lh' l.h), until the set is unchanged, cyclical or
 * ThicknessConstraintsItMax iterations have run; bcs->hpos_node is the set on entry and
 * rep->hpos_node receives the final one.  A step that does not converge is reported as
 * UA_ERR_NOT_CONVERGED (the reference's time-step reduction of uvh2NotConvergent.m is the
 * caller's).  F->ub, vb, h1: start
 * values in, solution out.  luvh: [l.ubvb; l.h] in/out (may be NULL).  The
 * inner solve on the constrained unsymmetric system is restarted GMRES(m)
 * (m = krylov_restart) or BiCGStab (uvh_krylov), right-preconditioned by the
 * block preconditioner selected with krylov_precond. */
int ua_uvh_newton(ua_mesh* m, const ua_params* p, ua_fields* F, const ua_bcs* bcs,
                  double* luvh, int32_t nl, ua_newton_report* rep);

/* Batched implicit uvh step: fields[i], bcs[i], reports[i] per system. */
int ua_uvh_newton_batch(ua_mesh* m, const ua_params* p, ua_fields* fields, const ua_bcs* bcs,
                        ua_newton_report* reports);

/* Serving (continuous batching of uv solves over the systems of a batch
 * handle, used as slots).  No single reference counterpart: each slot runs
 * SSTREAM2dNR2.m:3-431 (with the retry of uv.m:107-112) and requests join
 * between Newton iterations while other slots iterate.
 *   ua_serve_setup : BCs of every slot (bcs[i] for slot i), once.
 *   ua_serve_begin : admit count requests into free slots sys[k] with fields
 *                    F[k] (start velocities = warm start).
 *   ua_serve_step  : one Newton iteration of every active slot; finished[i]=1
 *                    for slots whose solve ended in this step; *nactive = busy slots.
 *   ua_serve_result: solution and report of a finished slot.
 *   ua_serve_cancel: between steps, drop active slots sys[k] from the iteration (they are free
 *                    again; the other slots' results are unchanged bit for bit). */
int ua_serve_setup(ua_mesh* m, const ua_params* p, const ua_bcs* bcs);
int ua_serve_begin(ua_mesh* m, const ua_params* p, int32_t count, const int32_t* sys, const ua_fields* F);
int ua_serve_step(ua_mesh* m, const ua_params* p, int32_t* finished, int32_t* nactive);
int ua_serve_result(ua_mesh* m, int32_t sys, double* ub, double* vb, ua_newton_report* rep);
int ua_serve_cancel(ua_mesh* m, int32_t count, const int32_t* sys);

/* Velocity data of the misfit (Meas in Misfit.m:38-66 with CtrlVar.Inverse.Measurements "-uv-"):
 * measured surface velocities and their standard errors uErr = sqrt(diag(Meas.usCov)),
 * vErr = sqrt(diag(Meas.vsCov)); Nnodes each, in the memory space of the fields (ua_fields.location). */
typedef struct ua_measurements {
    const double *us, *vs, *usErr, *vsErr;
} ua_measurements;

#define UA_ADJ_LOGC      1   /* gradient with respect to log10(C) (CtrlVar.Inverse.InvertFor "-logC-") */
#define UA_ADJ_PREMUL_M  2   /* CtrlVar.Inverse.AdjointGradientPreMultiplier "M": (M/Area)\dIdC */

/* Adjoint gradient of the velocity misfit with respect to C at the solved state F->ub, F->vb of
 * a single-mesh uv handle (Misfit.m:38-260, the adjoint branch for "-uv-" data; dIdCq.m:1-163;
 * ApplyAdjointGradientPreMultiplier.m; MassMatrix2D1dof.m):
 *   I = (r_u' M r_u + r_v' M r_v)/2/Area with r = (u - us)./uErr and M the consistent mass matrix;
 *   [K L'; L 0][lambda; mu] = [dI/d(u,v); c] with K the uv tangent at the state and L, c the
 *   adjoint BCs (solveKApeSymmetric; here the constrained AMG-PCG to p->krylov_rtol);
 *   dIdC_I = int dFuvdC (u lambda_u + v lambda_v) N_I (BasalDrag.m:80-160 for the sliding law),
 *   then log(10) C .* dIdC (UA_ADJ_LOGC) and (M/Area)\dIdC (UA_ADJ_PREMUL_M).
 * Outputs are caller-owned host arrays, each may be NULL: I, dIduv (2Nn), lambda (2Nn, the
 * adjoint velocities [uAdjoint; vAdjoint]), dIdC (Nn); krylov_its the PCG iterations.  Runs in
 * FP64 whatever p->precision says.  The Coulomb law has no C-gradient in the reference and is
 * refused with UA_ERR_INVALID. */
int ua_uv_adjoint_dIdC(ua_mesh* m, const ua_params* p, const ua_fields* F, const ua_bcs* bcs_adjoint,
                       const ua_measurements* meas, int32_t flags, double* I, double* dIduv, double* lambda,
                       double* dIdC, int32_t* krylov_its);

/* The bounds-checked debug build (libuassa_debug.so, `make debug`): every kernel that gathers
 * through the connectivity, the patch element lists, the contribution lists or the node-slice
 * columns checks the index against its range; the first violation is recorded (site: 1 patch
 * element id, 2 element node id, 3 contribution element, 4 tangent index, 5 residual row, 6 node-
 * slice column) and the access is skipped.  enabled = 0 in the release build. */
int ua_debug_bounds(const ua_mesh* m, int32_t* enabled, int32_t* site, int64_t* index);

/* Free and total device memory (admission by free HBM). */
int ua_mem_info(int32_t device, int64_t* free_bytes, int64_t* total_bytes);

/* Number of rows of the constraint matrix L built from bcs (CreateLuv.m). */
int ua_constraint_count(const ua_mesh* m, const ua_bcs* bcs, int32_t ndof, int32_t* nc);

/* The constraint matrix L and right-hand side c of the BCs of a single-mesh handle
 * (AssembleLuvSSTREAM.m:2-40 -> BCs2MLC.m:19-29, CreateLuv.m:28-76, ScaleL.m:28-33; createLh.m
 * for fixed h on an ndof=3 handle).  Row k has at most two non-zeros: L(k, dof[2k]) = val[2k]
 * and, for ties and normal velocities, L(k, dof[2k+1]) = val[2k+1] (dof[2k+1] = -1 and
 * val[2k+1] = 0 for a one-entry row); dofs are 0-based in Úa order, rows scaled to unit length,
 * c(k) = rhs[k].  Rows in the order of the Lagrange multipliers: u ties, v ties, fixed u nodes
 * increasing, fixed v nodes, fixed normal velocities, fixed h nodes as given.  This is the L that
 * SSTREAM2dNR2.m:3 returns as Lubvb.  dof and val hold 2*nc entries; arrays may be NULL to
 * query *nc only. */
int ua_constraint_matrix(const ua_mesh* m, const ua_bcs* bcs, int32_t* nc, int32_t* dof, double* val,
                         double* rhs);

/* solveKApeSymmetric (solveKApeSymmetric.m:71-113) -> ABfgPreEliminate
 * (ABfgPreEliminate.m:29-160) for an SPD block A given in CSR on the host:
 * [A L'; L 0][x;y] = [f;g] with L given in CSR (nl rows, at most one non-zero
 * per column, rows with orthogonal support).  Solved with projected PCG on
 * the device.  x0/y0 are ignored (the reference ignores them too). */
int ua_solve_kape_symmetric(int32_t n, const int64_t* Arowptr, const int64_t* Acol, const double* Aval,
                            int32_t nl, const int64_t* Lrowptr, const int64_t* Lcol, const double* Lval,
                            const double* f, const double* g, double* x, double* y,
                            double rtol, int32_t maxit, int32_t* its, int32_t device);

/* Allocation-free variant of ua_solve_kape_symmetric.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory (a MEX
 * working on gpuArray data, where MATLAB owns the device allocator; a plugin
 * in a host application that forbids cudaMalloc on its solve path).  Every
 * array argument is a device pointer on `device` (CSR of A with int32 indices,
 * L as one (dof, value) pair per constraint row).  Temporaries live in a
 * library-owned static device array of about 8.5 MB that each device keeps
 * until exit; n <= UA_NOALLOC_MAX_ROWS and nl <= UA_NOALLOC_MAX_CONSTRAINTS,
 * larger sizes return UA_ERR_INVALID.  The array is shared by all calls on a
 * device, so overlapping calls race; the first call on a device looks up the
 * array's address and should come before any stream capture.  Work runs on
 * cudaStreamPerThread and the call returns after it completes; it is not
 * ordered after work on the caller's streams, so every write to the inputs
 * must be complete before the call (a stream or device synchronize).  The CSR
 * of A is checked on the device before any product reads it: a column outside
 * [0,n), a negative or decreasing row pointer or an empty matrix returns
 * UA_ERR_INVALID.  Arowptr[n] must equal the length of Acol and Aval. */
#define UA_NOALLOC_MAX_ROWS 131072
#define UA_NOALLOC_MAX_CONSTRAINTS 16384
int ua_solve_kape_symmetric_noalloc(int32_t n, const int32_t* Arowptr, const int32_t* Acol, const double* Aval,
                                    int32_t nl, const int32_t* Ldof, const double* Lval,
                                    const double* f, const double* g, double* x, double* y,
                                    double rtol, int32_t maxit, int32_t* its, int32_t device);

#ifdef __cplusplus
}
#endif
#endif /* UA_SSA_H */
