// Instantiation unit of the Gauss-point-parallel interior-face VJP for the SA model (adjoint_fast.cuh): 6
// variables, plain Roe with the compact viscous flux, 3-D meshes at VR degree 1-2.
#include "adjoint_fast.cuh"

namespace dndsb
{
// ST_UNSUPPORTED when no instantiation covers the configuration (the caller then uses the forward-mode kernels)
int rhs_vjp_interior_fast_sa(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, const real *w, const real *u, const real *uRec,
                             real *faceAdj, cudaStream_t st)
{
    constexpr int NV = 6;
    if (!ev.facePt || ev.s.nVars != NV || ev.s.rsType != RS_Roe || ev.s.ignoreVis || m.dim != 3 || vr.P < 1 || vr.P > 2)
        return ST_UNSUPPORTED;
    if (vr.P == 1)
        return dispatch_vjp_ng<3, 1, NV>(m, g, vr, ev, false, true, w, u, uRec, faceAdj, st);
    return dispatch_vjp_ng<3, 2, NV>(m, g, vr, ev, false, true, w, u, uRec, faceAdj, st);
}
} // namespace dndsb
