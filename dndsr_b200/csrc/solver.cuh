// Device-resident state of one mesh + variational reconstruction + Euler
// evaluator, and the launch functions the C-ABI layer calls.
//
// Layout in HBM (all arrays structure-of-arrays, 64-bit reals unless noted):
//   cell rows   : vol, smooth ratio [nCell]; bary, cent, scale [nCell][3];
//                 cellJDet [nCell][nGc]; cellPP [nCell][nGc][3];
//                 baseMoment [nCell][NDOF]
//   face rows   : area [nFace]; meanNorm, cent, pshift [nFace][3];
//                 faceJDet [nFace][nGf]; facePP, faceNorm [nFace][nGf][3];
//                 faceWeight [nFace][P+1]; faceL [nFace]
//   VR matrices : AAInvB [nCell][nf+1][R][R] (block 0 = A^-1, block 1+k = A^-1 B_k)
//                 AInvb  [nCell][nf][R]; FP32 copies for the mixed-precision path
//   state       : u [nCell][nv], uRec [nCell][R][nv] (caller-owned device buffers)
#pragma once
#include "core.cuh"
#include <vector>

namespace dndsb
{
// error classes returned by every C-ABI entry point (also in include/dndsb.h)
enum Status : int
{
    ST_OK = 0,
    ST_BADARG = -1,
    ST_CUDA = -2,
    ST_NONFINITE = -3,
    ST_NONPHYSICAL = -4,
    ST_UNSUPPORTED = -5,
    ST_DIVERGED = -6,
    ST_TIMEOUT = -7,
};

// device error word bits (set by kernels, read back by the host)
enum DevErr : int
{
    DE_NONFINITE = 1,
    DE_NONPHYSICAL = 2,
    DE_SINGULAR = 4,
};

struct MeshD
{
    int dim = 0, cellType = 0, faceType = 0, nvert = 0, nfv = 0, nf = 0;
    int64_t nNode = 0, nCell = 0, nFace = 0;
    real *coords = nullptr;     // [nNode][3]
    int32_t *cell2node = nullptr; // [nCell][nvert]
    real *cellShift = nullptr;  // [nCell][nvert][3]
    int32_t *face2node = nullptr; // [nFace][nfv]
    real *faceShift = nullptr;  // [nFace][nfv][3]
    int32_t *face2cell = nullptr; // [nFace][2], -1 on boundary side 1
    int32_t *faceZone = nullptr;  // [nFace]
    real *facePShift = nullptr; // [nFace][3]
    int32_t *cell2face = nullptr; // [nCell][nf], packed (face << 1) | side
    int32_t *cellNbr = nullptr;   // [nCell][nf], neighbour cell or -1
    int32_t *nbrSlot = nullptr;   // [nCell][nf], slot of the same face in the neighbour's row (-1 on boundaries)
    // multicolour ordering for Gauss-Seidel type sweeps
    int nColor = 0;
    int32_t *colorCells = nullptr; // cells grouped by colour
    int32_t *cellColor = nullptr;  // colour of each cell
    std::vector<int64_t> colorStart; // host copy, size nColor + 1
    // boundary faces (face2cell side 1 = -1) and the cells that own them
    int64_t nBndFace = 0, nBndCell = 0;
    int32_t *bndFace = nullptr, *bndCell = nullptr;
};

// per-zone boundary table: the FBoundary of the VR sweep and the ghost states
// of the RHS (Euler/EulerBC.hpp types, EulerEvaluator_EvaluateDt.hxx:1743-2468)
enum BCType : int
{
    BC_FAR = 1,
    BC_WALL = 2,
    BC_WALL_INVIS = 3,
    BC_WALL_ISOTHERMAL = 4,
    BC_OUT = 5,
    BC_OUTP = 6,
    BC_IN = 7,
    BC_SYM = 9,
};
struct BoundaryD
{
    int nZone = 0;
    int32_t *type = nullptr; // [nZone], 0 for zones without a boundary condition
    real *val = nullptr;     // [nZone][8]: far-field / inflow state, or wall temperature
    real gamma = 1.4, Rgas = 1;
    bool viscFree = true;    // host: every used boundary zone carries no viscous flux (far-field, outflow, slip wall, symmetry)
};

struct VRSettingsD
{
    int maxOrder = 1, intOrder = 1;
    real jacobiRelax = 1;
    int SORInstead = 0;
    int anisotropicLengths = 0;
    int scaleType = 1; // 0 MeanAACBB, 1 BaryDiff
    real scaleMultiplier = 1;
    int dirWeightScheme = 0; // 0 Factorial, 1 HQM_OPT, 999 manual
    real manualDirWeights[4] = {1, 1, 0.5, 1. / 6};
    int geomWeightScheme = 0; // 0 none, 1 HQM_SD, 2 SD_Power
    real geomWeightBias = 0, geomWeightPower = 0.5, geomWeightPower1 = 0, geomWeightPower2 = 0;
    real bcWeight = 1;
};

struct GeomD
{
    int nGc = 0, nGf = 0;
    real *vol = nullptr, *cellBary = nullptr, *cellCent = nullptr, *cellScale = nullptr, *cellJDet = nullptr, *cellPP = nullptr,
         *smoothRatio = nullptr;
    real *faceArea = nullptr, *faceCent = nullptr, *faceJDet = nullptr, *facePP = nullptr, *faceNorm = nullptr, *faceMeanNorm = nullptr;
    real *cellQw = nullptr, *faceQw = nullptr; // quadrature weights of the cell / face rule at intOrder
    real *hMax = nullptr; // [nCell] largest extent along the inertia principal axes (GetCellMaxLenScale)
};

struct VRD
{
    VRSettingsD s;
    int P = 1, NDOF = 1, R = 0;
    real *baseMoment = nullptr, *faceWeight = nullptr, *faceL = nullptr;
    real *AAInvB = nullptr, *AInvb = nullptr, *matA = nullptr;
    float *AAInvB32 = nullptr, *AInvb32 = nullptr;
    // the sweep's coefficients packed per cell as [nf][R][R+1] (row i of A^-1 B_k, then (A^-1 b_k)_i):
    // one contiguous, 16-byte aligned range per cell, staged into shared memory by bulk async copies
    real *sweepCoef = nullptr;
    float *sweepCoef32 = nullptr;
    BoundaryD bnd;           // boundary values for the BC faces of the sweep
};

struct EulerSettingsD
{
    int nVars = 5;
    int rsType = RS_Roe;
    real rsFixScale = 1, rsIncFScale = 1;
    real gamma = 1.4, Rgas = 1, muGas = 1, prGas = 0.72, TRef = 273.15, CSutherland = 110.4;
    int muModel = 1;
    int ignoreVis = 0;
    int rsMeanValueEig = 0; // Roe_M1..M5 with the eigenvalues along the face's mean normal (Gas.hpp:1272-1408)
    real kT = 0, iPr = 0; // host-derived: gamma / ((gamma - 1) cp) (T = p kT / rho), 1 / prGas
    real cp() const { return Rgas * gamma / (gamma - 1); }
    void derive() { kT = gamma / ((gamma - 1) * cp()), iPr = 1.0 / prGas; }
};

struct EvalD
{
    EulerSettingsD s;
    real *lambdaFace = nullptr, *lambdaFaceC = nullptr, *lambdaFaceVis = nullptr, *lambdaConv = nullptr, *deltaLambdaFace = nullptr;
    real *deltaLambdaCell = nullptr;
    real *faceFlux = nullptr; // scratch [nFace][nv]
    real *facePt = nullptr;   // [nGf][nFace][7]: point, unit normal, |J| w (layout of the tuned face kernel)
    real *cellPar = nullptr;  // [nCell][6]: centre, 1/L
    real *redBuf = nullptr;   // scratch for reductions
    real *adjBuf = nullptr;   // scratch of the derivative kernels [nFace][2][(R+1) nv], allocated on first use
    size_t adjBufLen = 0;     // its length in reals
    real *dWall = nullptr;    // SA: wall distance at the cell Gauss points [nCell][nGc]
    real *jSource = nullptr;  // SA: source-term Jacobian diagonal of the last RHS [nCell][nv]
    real *fluxWall = nullptr; // wall-flux integral of the last RHS [8] (EvaluateRHS.hxx:599-607 fluxWallSum)
    real *objDir = nullptr;   // [8] direction of the wall-flux objective of dndsb_eval_wall_flux_vjp
    int *errWord = nullptr;   // device error word
    int *errDeferred = nullptr; // error word of EvaluateRHS in deferred mode (read and cleared on request)
    bool deferErr = false;    // EvaluateRHS skips its per-call read-back of the error word
    // useScalarJacobian / useRoeJacobian (EulerEvaluatorSettings.hpp:53-54): 0 scalar diagonal, 1 block diagonal,
    // 2 block diagonal with the Roe term (roejac.cuh); a block jdiag is [nCell][2][nv][nv] (block, inverse)
    int jacMode = 0;
    // EulerEvaluator.hpp:187-189, allocated for jacMode 2 as one [3][nFace] range: the convective speed after
    // EvaluateDt, the face integrals of the Riemann eigenvalues divided by the area after EvaluateRHS
    real *lambdaFace0 = nullptr, *lambdaFace123 = nullptr, *lambdaFace4 = nullptr;
    // the local LU of LUSGSMatrixToJacobianLU (allocated on first use): slot blocks L / U [nCell][nf][nv][nv],
    // inverted pivots [nCell][nv][nv]
    real *luOff = nullptr, *luDinv = nullptr;
    real *luDiag = nullptr; // with the scalar Jacobian: its diagonal as blocks [nCell][nv][nv] (JDiag.getValue)
};

// EvaluateRHS flags (EulerEvaluator.hpp:370-378 RHS_* values)
constexpr unsigned RHSF_IGNORE_VISCOSITY = 1u << 0;
constexpr unsigned RHSF_DONT_UPDATE_INTEGRATION = 1u << 1;
constexpr unsigned RHSF_DONT_RECORD_BND_FLUX = 1u << 2;

// ---- setup (setup.cu) ----
int geom_construct(const MeshD &m, const VRSettingsD &s, GeomD &g, cudaStream_t st);
int vr_construct_base_and_weight(const MeshD &m, const GeomD &g, VRD &vr, const real *bcDirWeightHost, int nZone, cudaStream_t st);
int vr_construct_rec_coeff(const MeshD &m, const GeomD &g, VRD &vr, int *errWord, cudaStream_t st);

// ---- hot path (hotpath.cu) ----
int vr_iter(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *uRec, real *uRecNew, const real *u, int recordInc,
            int uRecIsZero, int useFP32, cudaStream_t st);
int eval_dt(const MeshD &m, const GeomD &g, EvalD &ev, const real *u, real CFL, real MaxDt, int useLocalDt, real *dt, real *dtMin,
            cudaStream_t st);
int eval_rhs(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *u, const real *uRec, real *rhs, real *faceFlux,
             cudaStream_t st);
// EvaluateRHS(rhs, JSource, u, uRecUnlim, uRec, uRecBeta, cellRHSAlpha, onlyOnHalfAlpha, t, flags):
// uRecG = uRecUnlim (gradients), uRec (point values), alpha = cellRHSAlpha (nullptr: 1), flags RHSF_*,
// jSourceOut [nCell][nv] (may be nullptr)
int eval_rhs_ex(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *u, const real *uRecG, const real *uRec,
                const real *alpha, unsigned flags, real *rhs, real *faceFlux, real *jSourceOut, cudaStream_t st);
int lusgs_init(const MeshD &m, const GeomD &g, EvalD &ev, const real *dTau, real dt, real alphaDiag, real *jdiag, cudaStream_t st);
int update_sgs(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *rhs, const real *u, const real *uInc,
               real *uIncNew, const real *jdiag, int forward, int gsUpdate, int uIncIsZero, real *sumIncHost, cudaStream_t st);
int lusgs_matvec(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *u, const real *uInc, const real *jdiag,
                 real *AuInc, cudaStream_t st);
// UpdateLUSGSForward / UpdateLUSGSBackward; uInc may equal uIncNew (in-place sweep over the colours)
int update_lusgs(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *rhs, const real *u, const real *uInc,
                 real *uIncNew, const real *jdiag, int forward, cudaStream_t st);
int init_field(const MeshD &m, const GeomD &g, const EvalD &ev, int kind, real chi, real *u, cudaStream_t st);
// block-mode LU-SGS operators (roejac.cu): jd [nCell][2][nv][nv]; the Roe term with ev.jacMode == 2
int lusgs_init_block(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *dTau, real dt, real alphaDiag, const real *u,
                     real *jd, cudaStream_t st);
int update_sgs_block(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *rhs, const real *u, const real *uInc, real *uIncNew,
                     const real *jd, int forward, int gsUpdate, int uIncIsZero, real *sumIncHost, cudaStream_t st);
int update_lusgs_block(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *rhs, const real *u, const real *uInc,
                       real *uIncNew, const real *jd, int forward, cudaStream_t st);
int lusgs_matvec_block(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *u, const real *uInc, const real *jd, real *AuInc,
                       cudaStream_t st);
// LUSGSMatrixToJacobianLU + decomposition (block ILU(0), colour by colour) into ev.luOff / ev.luDinv, and
// LUSGSMatrixSolveJacobianLU with it (roejac.cu); jd in the layout of the evaluator's Jacobian mode
int jacobian_lu(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *u, const real *jd, cudaStream_t st);
int solve_jacobian_lu(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *rhs, const real *u, const real *uInc, real *uIncNew,
                      const real *jd, int uIncIsZero, real *sumIncHost, cudaStream_t st);
// viscous part of the residual derivatives (adjoint_visc.cu): added to the inviscid face
// cotangents [nFace][2][(R+1) nv] / face flux derivatives [nFace][nv] before their gathers
int rhs_vjp_visc(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *w, const real *u, const real *uRec, real *faceAdj,
                 cudaStream_t st);
int rhs_jvp_visc(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *du, const real *duRec, const real *u,
                 const real *uRec, real *ffd, cudaStream_t st);
// reverse-mode interior-face derivative of the Roe-family fluxes (adjoint_roe.cu); *viscDone: the viscous
// flux's share was included (the Gauss-point-parallel kernel of plain Roe and HLLE+)
int roe_scheme_of(int rsType);
// the Gauss-point-parallel interior-face VJP of plain Roe (hllep false) or HLLE+ with the viscous flux
// (adjoint_fast.cu); ST_UNSUPPORTED outside its instantiations
int rhs_vjp_interior_fast(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, bool hllep, const real *w, const real *u,
                          const real *uRec, real *faceAdj, cudaStream_t st);
// the same for the SA model (adjoint_fast_sa.cu): 6 variables, plain Roe with the viscous flux, 3-D, VR degree 1-2
int rhs_vjp_interior_fast_sa(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *w, const real *u, const real *uRec,
                             real *faceAdj, cudaStream_t st);
int rhs_vjp_roe_interior(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *w, const real *u, const real *uRec,
                         real *faceAdj, cudaStream_t st, bool *viscDone);
// adjoint building blocks (adjoint_ops.cu)
int lusgs_matvec_t(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const real *u, const real *y, const real *jdiag, real *ATy,
                   cudaStream_t st);
int update_sgs_t(const MeshD &m, const GeomD &g, EvalD &ev, real alphaDiag, const void *b, const real *u, const void *y, void *yNew,
                 const real *jdiag, int forward, int gsUpdate, int fp32, cudaStream_t st);
int pressure_force(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, int zone, const real *dir, const real *u, const real *uRec,
                   real *Jhost, real *gU, real *gRec, cudaStream_t st);
int vr_swap(int64_t n, real *a, real *b, cudaStream_t st);
// tuned kernels (fast.cu); ST_UNSUPPORTED means "use the generic kernel"
int fast_geometry(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, cudaStream_t st);
int rhs_face_fast(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *u, const real *uRec, real *ff, cudaStream_t st);
int vr_iter_fast(const MeshD &m, const VRD &vr, int nv, const real *uRec, real *uRecNew, const real *u, int recordInc, int uRecIsZero,
                 int useFP32, cudaStream_t st);
int reduce_norm(int64_t n, int ncol, const real *x, const real *w, int op, int powP, real *redBuf, real *outHost, cudaStream_t st);
constexpr int kRedBlocks = 592;                  // 4 x 148 SMs
constexpr int kRedBufLen = kRedBlocks * 8 + 64; // partials of the deterministic reductions + final values
constexpr int kRedBufLenK = kRedBlocks * 33;    // partials of the Krylov reductions (up to 33 columns)
// column reduction of x [n][ncol] (op 0 sum of |x|^powP * w, 1 min, 2 max); returns the device address of the ncol results
real *reduce_cols(int op, int64_t n, int ncol, const real *x, const real *w, int powP, real *redBuf, cudaStream_t st);

// ---- boundary faces (bc.cu) ----
// adds relax A^-1 BCC (GetBoundaryRHS) of every boundary cell to uRecNew
int vr_iter_bc(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *uRec, real *uRecNew, const real *u, int recordInc,
               int uRecIsZero, int useFP32, cudaStream_t st);
// DoReconstructionIter with SORInstead: one in-place sweep of uRec, colour by colour (5 or 6 variables, FP64 coefficients)
int vr_iter_sor(const MeshD &m, const GeomD &g, const VRD &vr, int nv, real *uRec, const real *u, cudaStream_t st);
// writes the face flux of every boundary face
// uRecG: the reconstruction of the inner gradients (uRecUnlim)
int rhs_bc(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *u, const real *uRec, const real *uRecG, real *ff,
           cudaStream_t st);

// ---- derivatives (adjoint.cu): VJP / JVP of EvaluateRHS and of one VR Jacobi sweep ----
// deltaLambdaCell (the entropy-fix scale of the last EvaluateDt) is held fixed, as between the
// reference's EvaluateDt and EvaluateRHS calls
// ---- WBAP_C limiter (limiter.cu; 3-D, VR degree 1-2) ----
int lim_secondary_build(const MeshD &m, const GeomD &g, const VRD &vr, real **sec, int *errWord, cudaStream_t st);
// faceTerm: [nFace][4] scratch, allocated on first use
int smooth_indicator(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *u, const real *uRec, real **faceTerm, real *si,
                     cudaStream_t st);
int limiter_wbap_c(const MeshD &m, const GeomD &g, const VRD &vr, const real *sec, int nv, real gamma, const real *u, const real *uRec,
                   const real *si, real *uRecNew, real threshold, real nStd, int ifAll, cudaStream_t st);

// ---- positivity-preserving increment limiting (positivity.cu) ----
int cell_rhs_alpha(const MeshD &m, EvalD &ev, const real *u, const real *res, real *alpha, real refRho, real refP, real relax, int compress,
                   real compressPower, int ppEpsIsRelaxed, int flag, int64_t *nLim, real *alphaMin, cudaStream_t st);
int cell_rhs_alpha_expansion(const MeshD &m, EvalD &ev, const real *u, const real *res, real *alpha, real refRho, real refP, real alphaMin,
                             cudaStream_t st);
int add_fixed_increment(const MeshD &m, EvalD &ev, real *u, const real *inc, real alpha, real refRho, real refP, int ppEpsIsRelaxed,
                        real *alphaFixMin, cudaStream_t st);

// ---- derivatives with respect to the node coordinates (adjoint_geom.cu) ----
struct CoordAdjWs
{
    int maxSlot = 0;
    int32_t *patch = nullptr;                 // [nCell][maxSlot] patch nodes of each cell, -1 padded
    int64_t *start = nullptr, *ent = nullptr; // node -> (cell, slot) entries, CSR in entry order
    real *share = nullptr;                    // [nCell][maxSlot][3]
    real *lanes = nullptr;                    // [nCell][10 + NDOF][1 + 3 nvert] cell geometry and its vertex derivatives
    bool noLanes = false;                     // no memory for the lanes: geometry recomputed per use
};
int coords_ws_build(const MeshD &m, CoordAdjWs &ws);
void coords_ws_free(CoordAdjWs &ws);
// s == nullptr: the VR sweep only (w unused); otherwise EvaluateRHS (w) and/or the sweep (cot)
int coords_vjp(const MeshD &m, const GeomD &g, const VRD &vr, const EulerSettingsD *s, const real *dLamCell, CoordAdjWs &ws, const real *w,
               const real *cot, const real *u, const real *uRec, real *dX, int *errWord, cudaStream_t st);
int coords_jvp(const MeshD &m, const GeomD &g, const VRD &vr, const EulerSettingsD *s, const real *dLamCell, CoordAdjWs &ws, const real *dX,
               const real *u, const real *uRec, real *dRhs, real *dRec, int *errWord, cudaStream_t st);
// d/dX of the pressure force of one boundary zone along dir (pressure_force's objective)
int pressure_force_coords(const MeshD &m, const GeomD &g, const VRD &vr, real gamma, int zone, const real *dir, const real *u, const real *uRec,
                          CoordAdjWs &ws, real *dX, cudaStream_t st);
int rhs_vjp(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *w, const real *u, const real *uRec, real *du, real *duRec,
            cudaStream_t st);
int rhs_jvp(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *du, const real *duRec, const real *u, const real *uRec,
            real *dRhs, cudaStream_t st);
int vr_vjp(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *v, const real *uRec, const real *u, real *vRec, real *vU,
           cudaStream_t st);
int vr_jvp(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *dRec, const real *du, const real *uRec, const real *u,
           real *dRecNew, cudaStream_t st);
// forward-mode derivatives for the SA model and viscous boundary zones (adjoint_generic.cu; 3-D, VR degree 1-2);
// rhs_vjp_generic with objDir != nullptr: the gradient of the wall-flux integral along objDir [nVars]
int rhs_vjp_generic(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *w, const real *objDir, const real *u, const real *uRec,
                    real *du, real *duRec, cudaStream_t st);
int rhs_jvp_generic(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *du, const real *duRec, const real *u, const real *uRec,
                    real *dRhs, cudaStream_t st);
int vr_vjp_generic(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *v, const real *uRec, const real *u, real *vRec, real *vU,
                   cudaStream_t st);
int vr_jvp_generic(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *dRec, const real *du, const real *uRec, const real *u,
                   real *dRecNew, cudaStream_t st);

// ---- native linear solve (linsolve.cu) and its Krylov reductions (reduce.cu) ----
struct LinSettings
{
    int gmresCode = 0;   // 0 LU-SGS pairs, 1 GMRES from zero, 2 LU-SGS pairs then GMRES
    int jacobiCode = 1;  // 1 Gauss-Seidel sweeps, 0 Jacobi sweeps, 2 block ILU(0) (block Jacobian only)
    int sgsIter = 0;     // extra SGS pairs
    int nGmresSpace = 5; // Krylov subspace size (<= 32)
    int nGmresIter = 1;  // restarts
    int precision = 0;   // 0 FP64, 1 FP32
    int useGraph = 1;    // capture the solve once and replay it
    real scale2[8] = {1, 1, 1, 1, 1, 1, 1, 1}; // per-variable weights of the GMRES dot (meanScaleInv^2)
};
struct LinWs;
// bnd: the boundary table (the ghost states of the Roe-term diagonal blocks)
int linear_solve(const MeshD &m, const GeomD &g, const BoundaryD &bnd, EvalD &ev, LinWs *&ws, const LinSettings &ls, real alphaDiag,
                 const real *dTau, real dt, const real *u, const real *rhs, real *xInc, cudaStream_t st);
void linws_free(LinWs *w);
// prec 0: double vectors, 1: float vectors; nv 5 or 6; FP64 accumulation, deterministic
// Krylov basis columns are ld apart: ld = n rounded up to a multiple of 4, storage 16-byte aligned, pad zero
inline int64_t krylov_ld(int64_t n) { return (n + 3) & ~(int64_t)3; }
// Each is one launch: the last block to finish reduces the per-block partials (cnt: a zeroed device counter
// the kernels share; it is reset after each use).  colScale (may be null): normalising factors of the
// basis columns, which are stored unnormalised.
void krylov_mdot(int prec, int64_t n, int64_t ld, int nv, int ncol, const void *V, const void *w, const real *s2, real *red, real *out,
                 const real *colScale, unsigned *cnt, cudaStream_t st);
// w -= V (h colScale); *outNorm = |w|; with gsc (GMRES scalars) also *scaleNext = 1 / |w| or 0 at a breakdown
void krylov_maxpy_norm(int prec, int64_t n, int64_t ld, int nv, int ncol, const void *V, const real *h, const real *colScale, void *w,
                       const real *s2, real *red, real *outNorm, unsigned *cnt, real *gsc, int j, real *scaleNext, cudaStream_t st);
void krylov_norm(int prec, int64_t n, int nv, const void *x, const real *s2, real *red, real *outNorm, unsigned *cnt, cudaStream_t st);
void krylov_diff_norm(int prec, int64_t n, int nv, const void *x, const void *y, const real *s2, real *red, real *outNorm, unsigned *cnt,
                      cudaStream_t st);
// A caller-driven Arnoldi process (linsolve.cu): V holds k + 1 columns krylov_ld(n) apart (zero beyond n),
// H k columns of k + 1, gsc the GMRES scalars ([0] breakdown scale, [1] beta, [2] valid columns, [8...] y),
// work krylov_work_bytes() bytes zeroed before the first use.
// start: beta = |r|, V0 = r / beta.  arnoldi: column j + 1 of V holds the operator applied to column j; it is
// orthogonalised (H column j, colScale[j + 1]) and the least squares on j + 1 columns solved (y, *res = its
// residual norm).  update: x += sum_i y_i colScale_i V_i.
size_t krylov_work_bytes();
int krylov_start(int prec, int64_t n, int k, const void *r, void *V, real *gsc, real *colScale, void *work, cudaStream_t st);
int krylov_arnoldi(int prec, int64_t n, int j, int k, void *V, real *H, real *colScale, real *gsc, real *res, void *work, cudaStream_t st);
int krylov_update(int prec, int64_t n, int k, const void *V, const real *gsc, const real *colScale, void *x, cudaStream_t st);
} // namespace dndsb
