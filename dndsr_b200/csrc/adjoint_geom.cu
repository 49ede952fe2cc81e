// Node-coordinate derivatives of the residual path: host side (patches, gather, dispatch) and the
// 3-D instantiations (VR degree 1 and 2) of the per-cell recomputation in adjoint_geom.cuh.
#include "adjoint_geom.cuh"

#include <vector>

namespace dndsb
{
extern template void coords_vjp_launch<2>(const MeshD &, const GeomD &, const VRD &, const EulerSettingsD &, const real *, const real *,
                                          const real *, const real *, const real *, const CoordAdjWs &, int *, cudaStream_t);
extern template void pressure_force_coords_launch<2>(const MeshD &, const GeomD &, const VRD &, real, int, const real *, const real *,
                                                     const real *, const CoordAdjWs &, cudaStream_t);
extern template void coords_jvp_launch<2>(const MeshD &, const GeomD &, const VRD &, const EulerSettingsD &, const real *, const real *,
                                   const real *, const real *, real *, real *, int *, const real *, cudaStream_t);
extern template void coords_lanes_launch<2>(const MeshD &, const GeomD &, const VRD &, real *, cudaStream_t);

namespace
{
// dX[n] = sum of the shares of node n, in (cell, slot) order
DNDSB_GLOBAL void k_node_gather(int64_t nNode, const int64_t *__restrict__ start, const int64_t *__restrict__ ent, const real *__restrict__ share,
                                real *__restrict__ dX)
{
    DNDSB_KERNEL_LOOP(n, nNode)
    {
        real a[3] = {0, 0, 0};
        for (int64_t e = start[n]; e < start[n + 1]; e++)
            for (int d = 0; d < 3; d++)
                a[d] += share[ent[e] * 3 + d];
        for (int d = 0; d < 3; d++)
            dX[n * 3 + d] = a[d];
    }
}

bool geo_supported(const MeshD &m, const VRD &vr) { return m.nvert <= kGeoMaxVert && vr.P >= 1 && (m.dim == 2 ? vr.P <= 3 : vr.P <= 2); }

int geo_status(cudaStream_t st, int *errWord)
{
    if (last_error() != cudaSuccess)
        return ST_CUDA;
    int e = 0;
    d2h(&e, errWord, sizeof(int), st);
    if (dev_sync(st) != cudaSuccess)
        return ST_CUDA;
    return (e & DE_NONPHYSICAL) ? ST_NONPHYSICAL : ST_OK;
}
} // namespace

// the patch of every cell (its nodes, then its face neighbours' nodes, first occurrence kept) and
// the node-to-share map of the gather; built once per mesh from the device topology
int coords_ws_build(const MeshD &m, CoordAdjWs &ws)
{
    if (ws.patch)
        return ST_OK;
    std::vector<int32_t> c2n((size_t)m.nCell * m.nvert), nbr((size_t)m.nCell * m.nf);
    if (cudaMemcpy(c2n.data(), m.cell2node, sizeof(int32_t) * c2n.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(nbr.data(), m.cellNbr, sizeof(int32_t) * nbr.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        return ST_CUDA;
    const int cap = m.nvert * (m.nf + 1);
    std::vector<int32_t> lists((size_t)m.nCell * cap);
    std::vector<int> cnt(m.nCell);
    int maxSlot = 1;
    for (int64_t c = 0; c < m.nCell; c++)
    {
        int32_t *L = &lists[(size_t)c * cap];
        int n = 0;
        auto add = [&](int64_t cell)
        {
            for (int v = 0; v < m.nvert; v++)
            {
                int32_t nd = c2n[(size_t)cell * m.nvert + v];
                bool seen = false;
                for (int i = 0; i < n && !seen; i++)
                    seen = L[i] == nd;
                if (!seen)
                    L[n++] = nd;
            }
        };
        add(c);
        for (int k = 0; k < m.nf; k++)
            if (nbr[(size_t)c * m.nf + k] >= 0)
                add(nbr[(size_t)c * m.nf + k]);
        cnt[c] = n;
        maxSlot = n > maxSlot ? n : maxSlot;
    }
    std::vector<int32_t> patch((size_t)m.nCell * maxSlot, -1);
    std::vector<int64_t> start(m.nNode + 1, 0);
    for (int64_t c = 0; c < m.nCell; c++)
        for (int i = 0; i < cnt[c]; i++)
        {
            int32_t nd = lists[(size_t)c * cap + i];
            patch[(size_t)c * maxSlot + i] = nd;
            start[nd + 1]++;
        }
    for (int64_t n = 0; n < m.nNode; n++)
        start[n + 1] += start[n];
    std::vector<int64_t> fill(start.begin(), start.end() - 1), ent(start[m.nNode]);
    for (int64_t e = 0; e < (int64_t)patch.size(); e++)
        if (patch[e] >= 0)
            ent[fill[patch[e]]++] = e;
    if (dev_alloc((void **)&ws.patch, sizeof(int32_t) * patch.size()) != cudaSuccess ||
        dev_alloc((void **)&ws.start, sizeof(int64_t) * start.size()) != cudaSuccess ||
        dev_alloc((void **)&ws.ent, sizeof(int64_t) * ent.size()) != cudaSuccess ||
        dev_alloc((void **)&ws.share, sizeof(real) * 3 * patch.size()) != cudaSuccess ||
        cudaMemcpy(ws.patch, patch.data(), sizeof(int32_t) * patch.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(ws.start, start.data(), sizeof(int64_t) * start.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(ws.ent, ent.data(), sizeof(int64_t) * ent.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    {
        coords_ws_free(ws);
        return ST_CUDA;
    }
    ws.maxSlot = maxSlot;
    return ST_OK;
}

// the cell geometry lanes (value and derivatives with respect to the cell's own vertices); without
// the memory for them the kernels recompute the geometry of each cell they need
void coords_lanes_build(const MeshD &m, const GeomD &g, const VRD &vr, CoordAdjWs &ws, cudaStream_t st)
{
    if (ws.lanes || ws.noLanes)
        return;
    const size_t n = (size_t)m.nCell * (10 + vr.NDOF) * (1 + 3 * m.nvert);
    if (dev_alloc((void **)&ws.lanes, sizeof(real) * n) != cudaSuccess)
    {
        (void)last_error();
        ws.lanes = nullptr, ws.noLanes = true;
        return;
    }
    if (m.dim == 2)
        coords_lanes_launch<2>(m, g, vr, ws.lanes, st);
    else
        coords_lanes_launch<3>(m, g, vr, ws.lanes, st);
}

void coords_ws_free(CoordAdjWs &ws)
{
    dev_free(ws.patch), dev_free(ws.start), dev_free(ws.ent), dev_free(ws.share), dev_free(ws.lanes);
    ws = CoordAdjWs();
}

int coords_vjp(const MeshD &m, const GeomD &g, const VRD &vr, const EulerSettingsD *s, const real *dLamCell, CoordAdjWs &ws, const real *w,
               const real *cot, const real *u, const real *uRec, real *dX, int *errWord, cudaStream_t st)
{
    if (!geo_supported(m, vr) || (s && (s->nVars != 5 || !s->ignoreVis)))
        return ST_UNSUPPORTED;
    int rc = coords_ws_build(m, ws);
    if (rc != ST_OK)
        return rc;
    coords_lanes_build(m, g, vr, ws, st);
    const EulerSettingsD es = s ? *s : EulerSettingsD();
    dev_zero(errWord, sizeof(int), st);
    if (m.dim == 2)
        coords_vjp_launch<2>(m, g, vr, es, dLamCell, u, uRec, w, cot, ws, errWord, st);
    else
        coords_vjp_launch<3>(m, g, vr, es, dLamCell, u, uRec, w, cot, ws, errWord, st);
    DNDSB_LAUNCH(k_node_gather, m.nNode, 256, st, m.nNode, ws.start, ws.ent, ws.share, dX);
    return geo_status(st, errWord);
}

int pressure_force_coords(const MeshD &m, const GeomD &g, const VRD &vr, real gamma, int zone, const real *dir, const real *u, const real *uRec,
                          CoordAdjWs &ws, real *dX, cudaStream_t st)
{
    if (!geo_supported(m, vr))
        return ST_UNSUPPORTED;
    int rc = coords_ws_build(m, ws);
    if (rc != ST_OK)
        return rc;
    dev_zero(ws.share, sizeof(real) * 3 * m.nCell * ws.maxSlot, st);
    if (m.dim == 2)
        pressure_force_coords_launch<2>(m, g, vr, gamma, zone, dir, u, uRec, ws, st);
    else
        pressure_force_coords_launch<3>(m, g, vr, gamma, zone, dir, u, uRec, ws, st);
    DNDSB_LAUNCH(k_node_gather, m.nNode, 256, st, m.nNode, ws.start, ws.ent, ws.share, dX);
    if (last_error() != cudaSuccess || dev_sync(st) != cudaSuccess)
        return ST_CUDA;
    return ST_OK;
}

int coords_jvp(const MeshD &m, const GeomD &g, const VRD &vr, const EulerSettingsD *s, const real *dLamCell, CoordAdjWs &ws, const real *dX,
               const real *u, const real *uRec, real *dRhs, real *dRec, int *errWord, cudaStream_t st)
{
    if (!geo_supported(m, vr) || (s && (s->nVars != 5 || !s->ignoreVis)))
        return ST_UNSUPPORTED;
    coords_lanes_build(m, g, vr, ws, st);
    const EulerSettingsD es = s ? *s : EulerSettingsD();
    dev_zero(errWord, sizeof(int), st);
    if (m.dim == 2)
        coords_jvp_launch<2>(m, g, vr, es, dLamCell, dX, u, uRec, dRhs, dRec, errWord, ws.lanes, st);
    else
        coords_jvp_launch<3>(m, g, vr, es, dLamCell, dX, u, uRec, dRhs, dRec, errWord, ws.lanes, st);
    return geo_status(st, errWord);
}
} // namespace dndsb
