// Instantiation unit of the Gauss-point-parallel interior-face VJP for 5 variables (adjoint_fast.cuh).
#include "adjoint_fast.cuh"

namespace dndsb
{
// ST_UNSUPPORTED when no instantiation covers the configuration (the caller then uses the per-face kernels)
int rhs_vjp_interior_fast(const MeshD &m, const GeomD &g, const VRD &vr, const EvalD &ev, bool hllep, const real *w, const real *u,
                          const real *uRec, real *faceAdj, cudaStream_t st)
{
    constexpr int NV = 5;
    if (!ev.facePt || ev.s.nVars != NV || vr.P < 1 || vr.P > 3)
        return ST_UNSUPPORTED;
    const bool visc = !ev.s.ignoreVis;
    if (m.dim == 2)
    {
        if (vr.P == 1)
            return dispatch_vjp_ng<2, 1, NV>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
        if (vr.P == 2)
            return dispatch_vjp_ng<2, 2, NV>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
        return dispatch_vjp_ng<2, 3, NV>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
    }
    if (vr.P == 1)
        return dispatch_vjp_ng<3, 1, NV>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
    if (vr.P == 2)
        return dispatch_vjp_ng<3, 2, NV>(m, g, vr, ev, hllep, visc, w, u, uRec, faceAdj, st);
    return ST_UNSUPPORTED;
}
} // namespace dndsb
