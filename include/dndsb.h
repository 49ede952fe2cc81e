/*
 * dndsb.h -- C-ABI of the B200 implementation of DNDSR's implicit residual
 * path: variational reconstruction (VR), Euler/NS right-hand side, local time
 * step and LU-SGS.
 *
 * Plain C: opaque handles, host pointers for setup data, caller-owned DEVICE
 * pointers for all state arrays, an optional cudaStream_t passed as void*,
 * and an int status on every call (0 = OK, < 0 = DNDSB_E_*).  No call aborts
 * or traps; dndsb_last_error() returns a message for the last failure of the
 * calling thread.
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the reference project root):
 *   CFV::VariationalReconstruction<dim>  src/CFV/VariationalReconstruction.hpp
 *   Euler::EulerEvaluator<model>         src/Euler/EulerEvaluator.hpp
 *
 * Array layouts (row-major):
 *   u, rhs, uInc          [nCell][nVars]
 *   uRec                  [nCell][R][nVars], R = NDOF - 1 (reference tURec rows)
 *   dt, dTau, jdiag       [nCell]
 *   matrixAAInvB          [nCell][nf+1][R][R] (block 0 = A^-1, 1+k = A^-1 B_k)
 *   vectorAInvB           [nCell][nf][R]
 */
#ifndef DNDSB_H
#define DNDSB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define DNDSB_OK 0
#define DNDSB_E_BADARG (-1)
#define DNDSB_E_CUDA (-2)
#define DNDSB_E_NONFINITE (-3)
#define DNDSB_E_NONPHYSICAL (-4) /* density or pressure <= 0 seen in a kernel */
#define DNDSB_E_UNSUPPORTED (-5)
#define DNDSB_E_DIVERGED (-6)
#define DNDSB_E_TIMEOUT (-7)

/* element kinds */
#define DNDSB_ELEM_LINE2 0
#define DNDSB_ELEM_TRI3 1
#define DNDSB_ELEM_QUAD4 2
#define DNDSB_ELEM_TET4 3
#define DNDSB_ELEM_HEX8 4

/* Riemann solver codes: src/Euler/Gas.hpp:61-96 RiemannSolverType */
#define DNDSB_RS_ROE 1
#define DNDSB_RS_HLLC 2
#define DNDSB_RS_HLLEP 3
#define DNDSB_RS_HLLEP_V1 21
#define DNDSB_RS_ROE_M1 11 /* ... DNDSB_RS_ROE_M8 = 18 */

typedef struct dndsb_mesh dndsb_mesh;
typedef struct dndsb_vr dndsb_vr;
typedef struct dndsb_eval dndsb_eval;

/* src/CFV/VRSettings.hpp:32-211 (fields of the same names) */
typedef struct dndsb_vr_settings
{
    int maxOrder, intOrder;
    double jacobiRelax;
    int SORInstead;
    int anisotropicLengths;  /* baseSettings.anisotropicLengths */
    int scaleType;           /* functionalSettings.scaleType: 0 MeanAACBB, 1 BaryDiff */
    double scaleMultiplier;
    int dirWeightScheme;     /* 0 Factorial, 1 HQM_OPT, 999 ManualDirWeight */
    double manualDirWeights[4];
    int geomWeightScheme;    /* 0 GWNone, 1 HQM_SD, 2 SD_Power */
    double geomWeightBias, geomWeightPower, geomWeightPower1, geomWeightPower2;
    double bcWeight;
} dndsb_vr_settings;

/* src/Euler/EulerEvaluatorSettings.hpp:40-330 (fields of the same names) */
typedef struct dndsb_euler_settings
{
    int nVars;
    int rsType; /* riemannSolverType */
    double rsFixScale, rsIncFScale;
    double gamma, Rgas, muGas, prGas, TRef, CSutherland; /* idealGasProperty */
    int muModel;
    int ignoreVis; /* RHS_Ignore_Viscosity flag of EvaluateRHS */
    int rsMeanValueEig; /* 1: Roe_M1..Roe_M5 take their eigenvalues, entropy fix and Roe normal velocity
                           along the face's mean normal (the batched flux, EulerEvaluator_EvaluateDt.hxx:1259-1270,
                           Gas.hpp:1272-1408); derivatives with respect to node coordinates then unsupported */
} dndsb_euler_settings;

/* ---- mesh (replaces Geom::UnstructuredMesh as input; src/Geom/Mesh/Mesh.hpp) ----
 * cell2face rows list each cell's faces; face2cell[f][1] = -1 on a boundary
 * face; a face's node order makes its normal point out of face2cell[f][0];
 * facePShift[f] maps points seen from side 0 into side 1's frame (periodic
 * translation, zero elsewhere).  All pointers are host pointers. */
int dndsb_mesh_create(dndsb_mesh **out, int dim, int cellType, int faceType, int64_t nNode, const double *coords, int64_t nCell,
                      int nvert, const int64_t *cell2node, const double *cellShift, int64_t nFace, int nfv, const int64_t *face2node,
                      const double *faceShift, const int64_t *face2cell, const int32_t *faceZone, const double *facePShift, int nf,
                      const int64_t *cell2face);
int dndsb_mesh_destroy(dndsb_mesh *m);
/* multicolour ordering used by the SGS sweeps (greedy, first fit in cell order) */
int dndsb_mesh_colors(const dndsb_mesh *m, int *nColor, int32_t *cellColorHost /* [nCell] or NULL */);

/* ---- variational reconstruction: VariationalReconstruction.hpp:108-1114 ---- */
int dndsb_vr_create(dndsb_vr **out, dndsb_mesh *mesh, const dndsb_vr_settings *s);
int dndsb_vr_destroy(dndsb_vr *vr);
/* ConstructMetrics(), VariationalReconstruction.cpp:10-43 */
int dndsb_vr_construct_metrics(dndsb_vr *vr);
/* ConstructBaseAndWeight(id2faceDircWeight), VariationalReconstruction.cpp:56-498;
 * the callback becomes a table bcDirWeight[zone][4] (NULL = all 1) */
int dndsb_vr_construct_base_and_weight(dndsb_vr *vr, const double *bcDirWeight, int nZone);
/* ConstructRecCoeff(), VariationalReconstruction.cpp:507-872 */
int dndsb_vr_construct_rec_coeff(dndsb_vr *vr);
/* out4 = {NDOF, R, Gauss points per face, Gauss points per cell} */
int dndsb_vr_sizes(const dndsb_vr *vr, int64_t *out4);
/* copies a named device array to host ("volume", "cellBary", "faceArea",
 * "matrixAAInvB", "vectorAInvB", ...); *len receives the element count */
int dndsb_vr_get_array(const dndsb_vr *vr, const char *name, double *hostOut, int64_t cap, int64_t *len);
/* DoReconstructionIter(uRec, uRecNew, u, FBoundary, putIntoNew, recordInc, uRecIsZero),
 * VariationalReconstruction_Reconstruction.hxx:485-615 (Jacobi sweep).
 * putIntoNew = 0 swaps the contents of uRec and uRecNew afterwards, like the reference.
 * precision: 0 FP64 coefficients, 1 FP32 coefficients (FP64 state and accumulation).
 * With SORInstead (VRSettings.hpp:43; the reference's default) and without recordInc the sweep is the
 * reference's in-place SOR (:534-611): uRec is updated in place colour by colour (equal to the reference's
 * sequential sweep on a mesh numbered colour by colour), a boundary face's term taken from the cell's
 * partially updated row as the reference's in-place update reads it; putIntoNew = 1 then swaps the contents
 * so that the result is in uRecNew; FP64 coefficients only.  The sweep derivatives below are those of the
 * Jacobi sweep, as the reference's DoReconstructionIterDiff. */
int dndsb_vr_do_reconstruction_iter(dndsb_vr *vr, double *uRec, double *uRecNew, const double *u, int nVars, int putIntoNew,
                                    int recordInc, int uRecIsZero, int precision, void *stream);

/* Boundary condition codes, Euler/EulerBC.hpp:35-48 EulerBCType */
#define DNDSB_BC_FAR 1
#define DNDSB_BC_WALL 2
#define DNDSB_BC_WALL_INVIS 3
#define DNDSB_BC_WALL_ISOTHERMAL 4
#define DNDSB_BC_OUT 5
#define DNDSB_BC_OUTP 6
#define DNDSB_BC_IN 7
#define DNDSB_BC_SYM 9
/* The FBoundary argument of DoReconstructionIter as a table: per face zone (the mesh's faceZone
 * values index it; zones of interior faces may hold 0) the boundary type and its value row
 * (far-field / inflow state, or the wall temperature in entry 0), nVars values per zone.  Ghost
 * values follow EulerEvaluator::generateBoundaryValue (EulerEvaluator_EvaluateDt.hxx:1743-2468).
 * A mesh with boundary faces needs this table before its first sweep. */
int dndsb_vr_set_boundary(dndsb_vr *vr, int nZone, const int32_t *type, const double *value, int nVars, double gamma, double Rgas);

/* Derivatives of one DoReconstructionIter Jacobi sweep uRecNew = S(uRec, u) (putIntoNew, FP64
 * coefficients), including the boundary term GetBoundaryRHS and its linearisation (the
 * reference's DoReconstructionIterDiff / GetBoundaryRHSDiff, _Reconstruction.hxx:99-176,617-670):
 * vjp: cot [nCell][R][nVars] -> vRec = (dS/duRec)^T cot, vU = (dS/du)^T cot
 * jvp: (dRec, du) -> dRecNew = dS/duRec dRec + dS/du du */
int dndsb_vr_iter_vjp(dndsb_vr *vr, const double *cot, const double *uRec, const double *u, int nVars, double *vRec, double *vU, void *stream);
int dndsb_vr_iter_jvp(dndsb_vr *vr, const double *dRec, const double *du, const double *uRec, const double *u, int nVars, double *dRecNew,
                      void *stream);
/* Derivatives of the same sweep with respect to the mesh node coordinates X [nNode][3] (uRec and u
 * held fixed): the cell metrics and basis moments (FiniteVolume.cpp:22-648,
 * VariationalReconstruction.cpp:56-498), the face weights and A^-1 B / A^-1 b (:507-872) and the
 * boundary term are recomputed per cell in dual numbers.  vjp: cot [nCell][R][5] -> dX = (dS/dX)^T cot;
 * jvp: dX -> dRecNew = dS/dX dX.  5 variables; VR degree 1-2 in 3-D, 1-3 in 2-D.  The first call
 * builds the per-cell node patches (a device-to-host copy of the topology, then device buffers). */
int dndsb_vr_iter_vjp_coords(dndsb_vr *vr, const double *cot, const double *uRec, const double *u, int nVars, double *dX, void *stream);
int dndsb_vr_iter_jvp_coords(dndsb_vr *vr, const double *dX, const double *uRec, const double *u, int nVars, double *dRecNew, void *stream);

/* ---- Euler evaluator: EulerEvaluator.hpp:76-1980 ---- */
int dndsb_eval_create(dndsb_eval **out, dndsb_vr *vr, const dndsb_euler_settings *s);
int dndsb_eval_destroy(dndsb_eval *ev);
/* The evaluator's BoundaryHandler (Euler/EulerBC.hpp): the same per-zone table as
 * dndsb_vr_set_boundary, with nVars, gamma and Rgas of the evaluator; it also becomes the
 * reconstruction's FBoundary (EulerSolver.hxx:163-175). */
int dndsb_eval_set_bc(dndsb_eval *ev, int nZone, const int32_t *type, const double *value);
/* The SA model's wall distance dWall (EulerEvaluator.hpp dWall, one value per cell Gauss point,
 * [nCell][nGc] in the order of the reconstruction's cell quadrature, host array).  Needed before the
 * first RHS of a 6-variable (NS_SA) evaluator. */
int dndsb_eval_set_wall_distance(dndsb_eval *ev, const double *dHost);
/* InitializeUDOF special initialisers, EulerEvaluator.hxx:1039-1143:
 * kind 2 = isentropic vortex of strength chi, 3 = Taylor-Green vortex (M0 = 0.1) */
int dndsb_eval_initialize_udof(dndsb_eval *ev, int kind, double chi, double *u, void *stream);
/* EvaluateDt(dt, u, uRec, CFL, dtMinall, MaxDt, UseLocaldt, t), EulerEvaluator_EvaluateDt.hxx:840-1048.
 * dtMinHost receives the global minimum (one host synchronisation); with useLocalDt and dtMinHost NULL
 * the call only launches. */
int dndsb_eval_evaluate_dt(dndsb_eval *ev, const double *u, double CFL, double MaxDt, int useLocalDt, double *dt, double *dtMinHost,
                           void *stream);
/* EvaluateRHS(rhs, JSource, u, uRecUnlim, uRec, ...), EulerEvaluator_EvaluateRHS.hxx:55-818
 * (no limiter: uRecUnlim == uRec).  The NS source is zero; with 6 variables (NS_SA) the SA source
 * is integrated at the cell Gauss points and JSource (the source Jacobian diagonal) is kept for
 * the next lusgs_matrix_init. */
int dndsb_eval_evaluate_rhs(dndsb_eval *ev, double *rhs, const double *u, const double *uRec, void *stream);
/* The full EvaluateRHS(rhs, JSource, u, uRecUnlim, uRec, uRecBeta, cellRHSAlpha, onlyOnHalfAlpha, t, flags),
 * EulerEvaluator.hpp:399-409 / EulerEvaluator_EvaluateRHS.hxx:55-818: point values from uRec (the limited
 * reconstruction), gradients of the viscous flux and of the SA source from uRecUnlim (may be the same
 * array); the SA source and JSource are scaled by cellRHSAlpha [nCell] (NULL = 1, :790); JSource
 * [nCell][nVars] (may be NULL) receives the source Jacobian diagonal (zero for 5 variables).  uRecBeta,
 * onlyOnHalfAlpha and t are accepted and, as in the reference's body, not read (the supported boundary
 * types are time independent).  flags: the reference's RHS_* bits (EulerEvaluator.hpp:370-378) below;
 * the direct second-order reconstruction bits are rejected with DNDSB_E_UNSUPPORTED.  Unless
 * RHS_Dont_Update_Integration is set, the wall-flux integral (:599-607, minus the summed face fluxes of
 * BCWall, BCWallIsothermal and, when muGas < 1e-99, BCWallInvis faces) is kept as "fluxWallSum"
 * (dndsb_eval_get_array). */
#define DNDSB_RHS_IGNORE_VISCOSITY (1ull << 0)
#define DNDSB_RHS_DONT_UPDATE_INTEGRATION (1ull << 1)
#define DNDSB_RHS_DONT_RECORD_BND_FLUX (1ull << 2)
int dndsb_eval_evaluate_rhs_full(dndsb_eval *ev, double *rhs, double *JSource, const double *u, const double *uRecUnlim, const double *uRec,
                                 const double *uRecBeta, const double *cellRHSAlpha, int onlyOnHalfAlpha, double t, uint64_t flags,
                                 void *stream);
/* Error reporting of EvaluateRHS (no reference counterpart: the reference asserts inside its loops).
 * By default each EvaluateRHS reads its device error word back and synchronises its stream, so that
 * it returns DNDSB_E_NONPHYSICAL / DNDSB_E_NONFINITE itself.  With set_deferred_errors(ev, 1) it only
 * launches: its kernels OR their findings into a deferred word, which check_errors reads, clears and
 * reports (one synchronisation, e.g. once per pseudo-iteration where a residual norm is read anyway). */
int dndsb_eval_set_deferred_errors(dndsb_eval *ev, int deferred);
int dndsb_eval_check_errors(dndsb_eval *ev, void *stream);
/* LUSGSMatrixInit(JDiag, JSource, dTau, dt, alphaDiag, u, uRec, 0, t), EulerEvaluator.hxx:37-159.  With the
 * scalar Jacobian jdiag holds one value per cell for 5 variables, and nVars values per cell for the SA model
 * (the shared diagonal plus alphaDiag times JSource of the last RHS); in block mode (dndsb_eval_set_jacobian_mode)
 * the block layout.  The Roe Jacobian needs u: dndsb_eval_lusgs_matrix_init_full. */
int dndsb_eval_lusgs_matrix_init(dndsb_eval *ev, const double *dTau, double dt, double alphaDiag, double *jdiag, void *stream);
/* EulerEvaluatorSettings useScalarJacobian / useRoeJacobian (EulerEvaluatorSettings.hpp:53-54, mutually
 * exclusive; an evaluator starts with useScalarJacobian).  With useScalarJacobian = 0 JDiag is block diagonal
 * (JacobianDiagBlock block mode, EulerJacobian.hpp:42-240): every jdiag argument of the LU-SGS operators
 * below (matrix_init, update_sgs, update_lusgs_*, matrix_vec) is then [nCell][2][nVars][nVars], the
 * row-major block and its inverse (GetInvert), and dndsb_eval_solve_linear uses the same blocks.  Without
 * the Roe term the block is the scalar diagonal.  With useRoeJacobian (EulerEvaluator.hxx:58-131) EvaluateDt
 * sets lambdaFace0/123/4 to the convective speed, EvaluateRHS records the face integrals of the Riemann
 * solver's eigenvalues (EvaluateRHS.hxx:527-545), the diagonal block sums (alphaDiag/2)(A_f/V) times the Roe
 * dissipation matrix plus lambdaVis I over the faces (boundary faces also the linearised ghost) plus
 * 1/dTau + 1/dt, and the neighbour increments take the Roe form (fluxJacobian0_Right_Times_du,
 * EulerEvaluator.hpp:1100-1158).  The transposed operators (lusgs_matrix_vec_t, update_sgs_t) take the
 * scalar Jacobian only. */
int dndsb_eval_set_jacobian_mode(dndsb_eval *ev, int useScalarJacobian, int useRoeJacobian);
/* LUSGSMatrixInit(JDiag, JSource, dTau, dt, alphaDiag, u, uRec, jacobianCode, t), EulerEvaluator.hxx:37-159, in
 * every Jacobian mode: u is read by the Roe term (NULL allowed otherwise), uRec and t by neither branch;
 * jacobianCode must be 0.  A singular block gives DNDSB_E_NONFINITE (one host synchronisation in block mode). */
int dndsb_eval_lusgs_matrix_init_full(dndsb_eval *ev, const double *dTau, double dt, double alphaDiag, const double *u, const double *uRec,
                                      int jacobianCode, double t, double *jdiag, void *stream);
/* The local LU (jacobiCode 2), kept inside the evaluator, in every Jacobian mode (with the scalar Jacobian its
 * diagonal blocks are the scalar diagonal, JDiag.getValue, and the neighbour blocks the scalar flux increment):
 * to_jacobian_lu = LUSGSMatrixToJacobianLU (EulerEvaluator.hxx:290-359) with JacobianLocalLU::InPlaceDecompose
 * (Solver/Direct.hpp:312-405) for iluCode 0 (the face-neighbour pattern, no fill): a block ILU(0) factored colour
 * by colour, which is the reference's natural-order factorisation on a mesh numbered colour by colour
 * (dndsb_mesh_colors).  solve_jacobian_lu = LUSGSMatrixSolveJacobianLU (:838-927): uIncNew = (LU)^-1 (rhs - A uInc)
 * + uInc, or (LU)^-1 rhs with uIncIsZero; sumIncHost [nVars] (may be NULL) the column sums of |(LU)^-1 (...)|. */
int dndsb_eval_lusgs_matrix_to_jacobian_lu(dndsb_eval *ev, double alphaDiag, const double *u, const double *jdiag, void *stream);
int dndsb_eval_lusgs_matrix_solve_jacobian_lu(dndsb_eval *ev, double alphaDiag, const double *rhs, const double *u, const double *uInc,
                                              double *uIncNew, const double *jdiag, int uIncIsZero, double *sumIncHost, void *stream);
/* UpdateSGS(alphaDiag, t, rhs, u, uInc, uIncNew, JDiag, forward, gsUpdate, sumInc, uIncIsZero),
 * EulerEvaluator.hxx:550-693, swept colour by colour; sumIncHost [nVars] may be NULL */
int dndsb_eval_update_sgs(dndsb_eval *ev, double alphaDiag, const double *rhs, const double *u, const double *uInc, double *uIncNew,
                          const double *jdiag, int forward, int gsUpdate, int uIncIsZero, double *sumIncHost, void *stream);
/* UpdateLUSGSForward / UpdateLUSGSBackward(alphaDiag, t, rhs, u, uInc, JDiag, uIncNew),
 * EulerEvaluator.hxx:376-529: forward uIncNew_i = D_i^-1 (rhs_i - sum over neighbours j < i of
 * (alphaDiag/2)(A_f/V_i) dF(u_j; uInc_j)); backward uIncNew_i += D_i^-1 (- the same sum over j > i).
 * uInc may be the same array as uIncNew, as the reference's callers pass it: the sweep then runs
 * colour by colour in place, which equals the reference's sequential sweep on a mesh numbered
 * colour by colour (dndsb_mesh_colors).  With distinct arrays every cell is independent. */
int dndsb_eval_update_lusgs_forward(dndsb_eval *ev, double alphaDiag, const double *rhs, const double *u, const double *uInc,
                                    const double *jdiag, double *uIncNew, void *stream);
int dndsb_eval_update_lusgs_backward(dndsb_eval *ev, double alphaDiag, const double *rhs, const double *u, const double *uInc,
                                     const double *jdiag, double *uIncNew, void *stream);
/* FixUMaxFilter(u), EulerEvaluator.hpp:591 / EulerEvaluator.hxx:1318-1323: the reference returns
 * without touching u; kept so that callers of the reference's sequence port unchanged. */
int dndsb_eval_fix_umax_filter(dndsb_eval *ev, double *u, void *stream);
/* LUSGSMatrixVec(alphaDiag, t, u, uInc, JDiag, AuInc), EulerEvaluator.hxx:175-274 */
int dndsb_eval_lusgs_matrix_vec(dndsb_eval *ev, double alphaDiag, const double *u, const double *uInc, const double *jdiag,
                                double *AuInc, void *stream);
/* WBAP_C limiter of the reconstruction (EulerSolver.hxx:455-556: smoothIndicatorProcedure 0,
 * limiterProcedure 1, limiterBiwayAlter 0, normWBAP false); 3-D meshes, VR degree 1-2, 5 or 6 variables.
 * smooth_indicator: DoCalculateSmoothIndicator(si, uRec, u, {0, I4})
 *   (VariationalReconstruction_LimiterProcedure.hxx:40-108), si [nCell].
 * limiter_wbap_c: DoLimiterWBAP_C(u, uRec, uRecNew, ..., si, ifAll, FM, FMI, putIntoNew = true)
 *   (VariationalReconstruction_LimiterProcedure.hxx:188-334) with the characteristic projections FM/FMI
 *   of EulerSolver.hxx:466-505 (the evaluator's gamma); cells with si < smoothThreshold are copied unless
 *   ifAll.  The first call builds matrixSecondary (VariationalReconstruction.cpp:840-866) on the device. */
int dndsb_vr_smooth_indicator(dndsb_vr *vr, const double *u, const double *uRec, int nVars, double *si, void *stream);
int dndsb_eval_limiter_wbap_c(dndsb_eval *ev, const double *u, const double *uRec, const double *si, double *uRecNew, double smoothThreshold,
                              double nStd, int ifAll, void *stream);

/* Positivity-preserving increment limiting of the implicit update (EulerSolver.hxx:696-738).
 * refRho, refP: the reference's refUPrim(0), refUPrim(I4) (far-field density and pressure), which set
 * the floors rhoEps = 1e-11 refRho, pEps = 1e-11 refP.  A state for which the reference asserts returns
 * DNDSB_E_NONPHYSICAL.  Each call synchronises its stream to return its counts.
 * cell_rhs_alpha: EvaluateCellRHSAlpha(u, uRec, uRecBeta, res, cellRHSAlpha, nLim, alphaMin, relax,
 *   compress, flag) (EulerEvaluator.hxx:1938-2062; uRec and uRecBeta are not read there): alpha [nCell]
 *   with u + alpha res inside the relaxed floors; flag 1 = MIN_IF_NOT_ONE, 2 = MIN_ALL; compressPower is
 *   the settings' uRecAlphaCompressPower.  nLimHost, alphaMinHost may be NULL.
 * cell_rhs_alpha_expansion: EvaluateCellRHSAlphaExpansion (EulerEvaluator.hxx:2064-2140).
 * add_fixed_increment: AddFixedIncrement(cx, cxInc, alpha) (EulerEvaluator.hpp:1795-1857),
 *   u += CompressInc(u, alpha inc); alphaFixMinHost (may be NULL) = the smallest density-increment ratio. */
int dndsb_eval_cell_rhs_alpha(dndsb_eval *ev, const double *u, const double *res, double *alpha, double refRho, double refP, double relax,
                              int compress, double compressPower, int ppEpsIsRelaxed, int flag, int64_t *nLimHost, double *alphaMinHost,
                              void *stream);
int dndsb_eval_cell_rhs_alpha_expansion(dndsb_eval *ev, const double *u, const double *res, double *alpha, double refRho, double refP,
                                        double alphaMin, void *stream);
int dndsb_eval_add_fixed_increment(dndsb_eval *ev, double *u, const double *inc, double alpha, double refRho, double refP, int ppEpsIsRelaxed,
                                   double *alphaFixMinHost, void *stream);

/* Derivatives of EvaluateRHS (EulerEvaluator_EvaluateRHS.hxx:55-818) with respect to the cell
 * means u and the reconstruction uRec, at the deltaLambdaCell of the last evaluate_dt (held
 * fixed): vjp: w [nCell][nVars] -> du = (dR/du)^T w, duRec = (dR/duRec)^T w; jvp: (du, duRec) -> dRhs.
 * Euler and Navier-Stokes (5 variables) through the inviscid, viscous and boundary fluxes; the SA
 * model (6 variables: SA convective and diffusion fluxes, eddy viscosity, source term) and boundary
 * zones with a viscous flux on 3-D meshes at VR degree 1-2.  Gauss-point states are recomputed, not
 * stored.  The reference has no hand-written adjoint of this path (its Python package differentiates
 * nothing). */
int dndsb_eval_rhs_vjp(dndsb_eval *ev, const double *w, const double *u, const double *uRec, double *du, double *duRec, void *stream);
int dndsb_eval_rhs_jvp(dndsb_eval *ev, const double *du, const double *duRec, const double *u, const double *uRec, double *dRhs, void *stream);
/* Gradient of the wall-flux integral along dirHost [nVars] (host array): J = dir . fluxWallSum, the
 * integral EvaluateRHS records (EulerEvaluator_EvaluateRHS.hxx:599-607: minus the face fluxes of the
 * BCWall / BCWallIsothermal faces, and of BCWallInvis faces when muGas < 1e-99).  dir = (0, 1, 0, 0, 0 ...)
 * gives the x force on the walls: pressure and skin friction, with the SA eddy viscosity for 6 variables.
 * du [nCell][nVars], duRec [nCell][R][nVars] receive dJ/du, dJ/duRec (deltaLambdaCell held fixed).
 * 3-D meshes, VR degree 1-2. */
int dndsb_eval_wall_flux_vjp(dndsb_eval *ev, const double *dirHost, const double *u, const double *uRec, double *du, double *duRec,
                             void *stream);
/* Derivatives of EvaluateRHS with respect to the mesh node coordinates X [nNode][3] (u, uRec and
 * deltaLambdaCell held fixed; geometry, basis and face points, normals and Jacobians recomputed per
 * cell in dual numbers): vjp: w [nCell][5] -> dX = (dR/dX)^T w; jvp: dX -> dRhs.  Inviscid
 * (ignoreVis) 5-variable models; VR degree 1-2 in 3-D, 1-3 in 2-D. */
int dndsb_eval_rhs_vjp_coords(dndsb_eval *ev, const double *w, const double *u, const double *uRec, double *dX, void *stream);
int dndsb_eval_rhs_jvp_coords(dndsb_eval *ev, const double *dX, const double *u, const double *uRec, double *dRhs, void *stream);
/* Both at once, sharing the per-cell recomputation: dX = (dR/dX)^T w + (dS/dX)^T cot, S the VR sweep of the
 * evaluator's reconstruction (the coupled residual's coordinate VJP). */
int dndsb_eval_residual_vjp_coords(dndsb_eval *ev, const double *w, const double *cot, const double *u, const double *uRec, double *dX,
                                   void *stream);

/* Adjoint building blocks (no reference counterpart; they transpose the operators above).
 * lusgs_matrix_vec_t: ATy = A^T y for the operator A of dndsb_eval_lusgs_matrix_vec (same lambdaFace,
 * jdiag and alphaDiag).  update_sgs_t: one Gauss-Seidel sweep on A^T y = b, colour by colour (forward:
 * colours ascending, new values of earlier colours when gsUpdate), y and yNew distinct; a forward then
 * a backward sweep is the symmetric Gauss-Seidel preconditioner of A^T.  precision 0: b, y, yNew are
 * double; 1: float (the FP32 preconditioner; the operator is applied in FP64 from the FP64 state). */
int dndsb_eval_lusgs_matrix_vec_t(dndsb_eval *ev, double alphaDiag, const double *u, const double *y, const double *jdiag, double *ATy,
                                  void *stream);
int dndsb_eval_update_sgs_t(dndsb_eval *ev, double alphaDiag, const void *b, const double *u, const void *y, void *yNew,
                            const double *jdiag, int forward, int gsUpdate, int precision, void *stream);
/* Pressure force along dir[3] on the boundary faces of zone:
 *   J = sum_f sum_g |J|_g w_g p(U_L(x_g)) (n_g . dir),  U_L = u + phi . uRec of the face's cell,
 * returned in *Jhost; dJdu [nCell][nVars] and dJduRec [nCell][R][nVars] (device, either may be NULL)
 * receive its gradient, zero away from the zone. */
int dndsb_eval_pressure_force(dndsb_eval *ev, int zone, const double *dir, const double *u, const double *uRec, double *Jhost, double *dJdu,
                              double *dJduRec, void *stream);
/* Derivative of the same objective with respect to the mesh node coordinates X [nNode][3] (u and uRec
 * held fixed): the cell's basis and the face points, normals and Jacobians differentiated.  With the
 * adjoint (psi, lam) of the coupled residual, the shape gradient is
 * dJ/dX = dJdX - dndsb_eval_rhs_vjp_coords(psi) - dndsb_vr_iter_vjp_coords(lam). */
int dndsb_eval_pressure_force_coords(dndsb_eval *ev, int zone, const double *dir, const double *u, const double *uRec, double *dJdX, void *stream);

/* Linear-solver controls, EulerSolver.hpp linearSolverControl (fields of the same names) plus the
 * precision of the solve.  meanScale: the GMRES dot weights of EulerSolver.hxx:1518-1540
 * (dot(a, b) = sum a_v b_v / (meanScale_v + 1e-200)^2); entries <= 0 count as 1. */
typedef struct dndsb_linear_settings
{
    int gmresCode;   /* 0 LU-SGS pairs, 1 GMRES from zero, 2 LU-SGS pairs then GMRES */
    int jacobiCode;  /* 1 Gauss-Seidel sweeps (multicolour), 0 Jacobi sweeps, 2 the local LU (block ILU(0), two
                        defect-correction steps per doPrecondition) */
    int sgsIter;     /* extra SGS pairs (also inside the GMRES preconditioner) */
    int nGmresSpace; /* Krylov subspace size, 1..32 */
    int nGmresIter;  /* restart cycles */
    int precision;   /* 0 FP64, 1 FP32 (preconditioner and Krylov vectors; dots accumulate in FP64) */
    int useGraph;    /* 1: capture the fixed kernel sequence once and replay it */
    double meanScale[8];
} dndsb_linear_settings;
/* EulerSolver::solveLinear + doPrecondition (EulerSolver.hxx:1407-1579, 1605-1658) with
 * LUSGSMatrixInit (EulerEvaluator.hxx:37-159) and GMRES_LeftPreconditioned::solve
 * (Solver/Linear.hpp:46-133) in one call: xInc = M^-1 rhs, for the scalar-diagonal LU-SGS
 * operator at state u, pseudo time step dTau, physical step dt and alphaDiag.  Uses the face
 * eigenvalues of the last dndsb_eval_evaluate_dt.  xInc is overwritten (the solve starts from
 * zero, as the reference's fsolve does).  No host synchronisation. */
int dndsb_eval_solve_linear(dndsb_eval *ev, const dndsb_linear_settings *ls, double alphaDiag, const double *dTau, double dt,
                            const double *u, const double *rhs, double *xInc, void *stream);
/* EvaluateNorm(res, rhs, P, volWise), EulerEvaluator.hxx:1394-1439; P = 1, 2 or >= 3 (max norm) */
int dndsb_eval_evaluate_norm(dndsb_eval *ev, const double *x, int P, int volWise, double *resHost, void *stream);
/* named evaluator arrays to host: "lambdaFace", "lambdaFaceC", "lambdaFaceVis", "deltaLambdaCell" */
int dndsb_eval_get_array(const dndsb_eval *ev, const char *name, double *hostOut, int64_t cap, int64_t *len);
/* sets deltaLambdaCell (normally produced by EvaluateDt) from a device array [nCell] */
int dndsb_eval_set_delta_lambda(dndsb_eval *ev, const double *deltaLambdaCell, void *stream);

/* Allocation-free EvaluateRHS.  No counterpart in the reference: it exists
 * for callers that must not allocate device memory when they evaluate a
 * residual (for example a program whose GPU memory belongs to its own pool
 * allocator, or a latency-critical loop that cannot take the synchronisation
 * of cudaMalloc/cudaFree).  The per-face flux scratch lives in a static device
 * array of DNDSB_NOALLOC_SCRATCH_DOUBLES doubles (8 MiB, held by every GPU
 * that loads the library until exit); meshes with nFace * nVars above that
 * are rejected with DNDSB_E_UNSUPPORTED.  The first call on a device looks up
 * the array's address (cudaGetSymbolAddress) and should come before any
 * stream capture.  Like dndsb_eval_evaluate_rhs, each call reads the error
 * word back and synchronises its stream before it returns (unless the
 * evaluator defers its error reports).  All calls on a device share the array: calls whose
 * kernels overlap on the GPU race and must be serialised by the caller.
 * Results equal dndsb_eval_evaluate_rhs. */
#define DNDSB_NOALLOC_SCRATCH_DOUBLES (1 << 20)
int dndsb_eval_evaluate_rhs_noalloc(dndsb_eval *ev, double *rhs, const double *u, const double *uRec, void *stream);

/* Device Krylov primitives for a caller-driven, right-preconditioned restarted GMRES whose operator and
 * preconditioner are applied outside the library (the adjoint and tangent solves of the coupled
 * residual; no reference counterpart, the reference's GMRES_LeftPreconditioned::solve,
 * Solver/Linear.hpp:46-133, takes its operator as a callback).  The same one-launch deterministic
 * reductions as dndsb_eval_solve_linear's GMRES, FP64 accumulation; no call synchronises.
 * precision 0: double vectors, 1: float vectors.  V: k + 1 columns (1 <= k <= 32) of
 * dndsb_krylov_ld(n) elements, 16-byte aligned, zero beyond n; H: k columns of k + 1 doubles;
 * colScale: k + 1 doubles (the normalising factors of the stored, unnormalised columns);
 * gsc: 8 + k doubles ([1] beta, [2] valid columns, [8 ...] least-squares y); work:
 * dndsb_krylov_work_bytes() bytes, zero-filled before its first use.  One cycle: start, then for
 * j = 0 .. k-1 the caller writes A M (colScale[j] V_j) into column j + 1 and calls arnoldi, then
 * update gives the correction t = V y to which the caller applies M. */
int64_t dndsb_krylov_ld(int64_t n);
size_t dndsb_krylov_work_bytes(void);
/* beta = |r| (gsc[1]); column 0 = r / beta */
int dndsb_krylov_start(int precision, int64_t n, int k, const void *r, void *V, double *gsc, double *colScale, void *work, void *stream);
/* orthogonalises column j + 1 against columns 0..j (classical Gram-Schmidt: H column j, colScale[j + 1];
 * a breakdown drops the column), then solves the least squares on j + 1 columns: y in gsc, *res = its
 * residual norm (device) */
int dndsb_krylov_arnoldi(int precision, int64_t n, int j, int k, void *V, double *H, double *colScale, double *gsc, double *res, void *work,
                         void *stream);
/* x += sum_i y_i colScale_i V_i over the columns of the last least squares */
int dndsb_krylov_update(int precision, int64_t n, int k, const void *V, const double *gsc, const double *colScale, void *x, void *stream);

const char *dndsb_last_error(void);
int dndsb_version(void);

#ifdef __cplusplus
}
#endif
#endif
