// Derivatives of the residual path for the configurations the specialised kernels of adjoint.cu,
// adjoint_roe.cu and adjoint_visc.cu do not cover: the SA model (6 variables: the SA convective and
// diffusion fluxes, the eddy viscosity in the viscous flux, the source term) and boundary zones with
// a viscous flux (no-slip and isothermal walls, inflow, pressure outflow), for 5 or 6 variables.
//
// Forward mode throughout.  Per face Gauss point the integrand of EvaluateRHS (EvaluateRHS.hxx:224-525:
// F(UL, UR; ULm, URm) minus the viscous flux of the compact gradient) is evaluated in dual numbers
// with 2 NV seeds per pass: the two point states, the two cell means, then the two point gradients
// along each axis; on a boundary face the ghost states are formed inside the pass (the point state
// and the cell mean are seeded together).  The pass results are contracted with the face cotangent
// and carried through the reconstruction basis to (u, uRec) of both cells; the per-face cotangents
// are gathered per cell in a fixed order, as in the specialised kernels.  The SA source is
// differentiated per cell Gauss point in four passes (the point state, then the gradient along each
// axis).  The JVPs are the same computations with one seed.  The entropy-fix scale deltaLambdaCell
// is held fixed.  One Jacobi sweep of the reconstruction and its boundary term are differentiated as
// in adjoint.cu, for NV variables.
#include "solver.cuh"

namespace dndsb
{
namespace gen
{
// launchers, instantiated in adjoint_generic_p{1,2}n{5,6}.cu
template <int DIM, int P, int NV>
int vjp_dp(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *w, const real *objDir, const real *u, const real *uRec,
           real *du, real *duRec, cudaStream_t st);
template <int DIM, int P, int NV>
int jvp_dp(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *du, const real *duRec, const real *u, const real *uRec,
           real *dRhs, cudaStream_t st);
template <int DIM, int P, int NV>
int vr_vjp_dp_g(const MeshD &m, const GeomD &g, const VRD &vr, const real *v, const real *uRec, const real *u, real *vRec, real *vU,
                cudaStream_t st);
template <int DIM, int P, int NV>
int vr_jvp_dp_g(const MeshD &m, const GeomD &g, const VRD &vr, const real *dRec, const real *du, const real *uRec, const real *u,
                real *dNew, cudaStream_t st);
} // namespace gen

namespace
{
using gen::jvp_dp;
using gen::vjp_dp;
using gen::vr_jvp_dp_g;
using gen::vr_vjp_dp_g;

int ensure_adj_g(const MeshD &m, const VRD &vr, EvalD &ev, int nv)
{
    size_t need = (size_t)m.nFace * 2 * (vr.R + 1) * nv;
    if (ev.adjBuf && ev.adjBufLen >= need)
        return ST_OK;
    dev_free(ev.adjBuf);
    ev.adjBuf = nullptr;
    if (dev_alloc((void **)&ev.adjBuf, sizeof(real) * need) != cudaSuccess)
        return ST_CUDA;
    ev.adjBufLen = need;
    return ST_OK;
}

int finish(cudaStream_t st, int *err)
{
    int e = 0;
    d2h(&e, err, sizeof(int), st);
    if (dev_sync(st) != cudaSuccess || last_error() != cudaSuccess)
        return ST_CUDA;
    return e ? ST_NONPHYSICAL : ST_OK;
}

// 3-D meshes, VR degree 1-2
#define DNDSB_G_DISPATCH(FN, NVV, ...)                                              \
    do                                                                               \
    {                                                                                \
        if (vr.P > 2 || m.dim != 3)                                                  \
            return ST_UNSUPPORTED;                                                   \
        return vr.P == 1 ? FN<3, 1, NVV>(__VA_ARGS__) : FN<3, 2, NVV>(__VA_ARGS__); \
    } while (0)

} // namespace

// objDir == nullptr: (dR/du)^T w, (dR/duRec)^T w; otherwise the gradient of the wall-flux integral along objDir
int rhs_vjp_generic(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *w, const real *objDir, const real *u, const real *uRec,
                    real *du, real *duRec, cudaStream_t st)
{
    const int nv = ev.s.nVars;
    if ((nv != 5 && nv != 6) || (nv == 6 && !ev.dWall))
        return ST_UNSUPPORTED;
    if (ensure_adj_g(m, vr, ev, nv) != ST_OK)
        return ST_CUDA;
    dev_zero(ev.errWord, sizeof(int), st);
    auto run = [&]() -> int
    {
        if (nv == 5)
            DNDSB_G_DISPATCH(vjp_dp, 5, m, g, vr, ev, w, objDir, u, uRec, du, duRec, st);
        DNDSB_G_DISPATCH(vjp_dp, 6, m, g, vr, ev, w, objDir, u, uRec, du, duRec, st);
    };
    int rc = run();
    if (rc != ST_OK)
        return rc;
    return finish(st, ev.errWord);
}

int rhs_jvp_generic(const MeshD &m, const GeomD &g, const VRD &vr, EvalD &ev, const real *du, const real *duRec, const real *u, const real *uRec,
                    real *dRhs, cudaStream_t st)
{
    const int nv = ev.s.nVars;
    if ((nv != 5 && nv != 6) || (nv == 6 && !ev.dWall))
        return ST_UNSUPPORTED;
    if (ensure_adj_g(m, vr, ev, nv) != ST_OK)
        return ST_CUDA;
    dev_zero(ev.errWord, sizeof(int), st);
    auto run = [&]() -> int
    {
        if (nv == 5)
            DNDSB_G_DISPATCH(jvp_dp, 5, m, g, vr, ev, du, duRec, u, uRec, dRhs, st);
        DNDSB_G_DISPATCH(jvp_dp, 6, m, g, vr, ev, du, duRec, u, uRec, dRhs, st);
    };
    int rc = run();
    if (rc != ST_OK)
        return rc;
    return finish(st, ev.errWord);
}

int vr_vjp_generic(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *v, const real *uRec, const real *u, real *vRec, real *vU,
                   cudaStream_t st)
{
    if (nv != 6)
        return ST_UNSUPPORTED;
    auto run = [&]() -> int { DNDSB_G_DISPATCH(vr_vjp_dp_g, 6, m, g, vr, v, uRec, u, vRec, vU, st); };
    int rc = run();
    if (rc != ST_OK)
        return rc;
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}

int vr_jvp_generic(const MeshD &m, const GeomD &g, const VRD &vr, int nv, const real *dRec, const real *du, const real *uRec, const real *u,
                   real *dRecNew, cudaStream_t st)
{
    if (nv != 6)
        return ST_UNSUPPORTED;
    auto run = [&]() -> int { DNDSB_G_DISPATCH(vr_jvp_dp_g, 6, m, g, vr, dRec, du, uRec, u, dRecNew, st); };
    int rc = run();
    if (rc != ST_OK)
        return rc;
    return last_error() == cudaSuccess ? ST_OK : ST_CUDA;
}
} // namespace dndsb
