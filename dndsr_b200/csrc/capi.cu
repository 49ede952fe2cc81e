// C-ABI entry points (include/dndsb.h): argument checks, host-side topology
// preparation (packed cell-to-face rows, neighbour lists, multicolouring),
// device allocation of the handle-owned arrays, and dispatch to the kernels.
#include "../../include/dndsb.h"
#include "solver.cuh"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace dndsb;

struct dndsb_mesh
{
    MeshD d;
    std::vector<int32_t> cellColorHost;
    std::vector<int32_t> bndZoneHost; // zones of the boundary faces, for checking boundary tables
    int64_t nBndFace = 0;
};

struct dndsb_vr
{
    dndsb_mesh *mesh = nullptr;
    GeomD g;
    VRD vr;
    CoordAdjWs coordWs; // node-coordinate derivatives: patches and shares, built on first use
    real *limSec = nullptr; // WBAP limiter: matrixSecondary per interior face [nFace][2][R][R], built on first use
    real *siFace = nullptr; // smooth indicator: per-face terms [nFace][4], allocated on first use
    int *errWord = nullptr;
    bool metrics = false, base = false, coeff = false;
    int bndNVars = 0; // number of variables of the boundary table's values
};

struct dndsb_eval
{
    dndsb_vr *vr = nullptr;
    EvalD e;
    LinWs *lin = nullptr; // workspace of dndsb_eval_solve_linear
};

namespace
{
thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

int cuda_fail(const char *where)
{
    cudaError_t e = cudaGetLastError();
    return fail(DNDSB_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

template <class T>
int upload(T **dst, const T *src, int64_t n)
{
    if (dev_alloc((void **)dst, sizeof(T) * n) != cudaSuccess)
        return ST_CUDA;
    if (n > 0 && cudaMemcpy(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice) != cudaSuccess)
        return ST_CUDA;
    return ST_OK;
}

int status_msg(int rc, const char *where)
{
    if (rc == ST_OK)
        return DNDSB_OK;
    if (rc == ST_CUDA)
        return cuda_fail(where);
    if (rc == ST_NONPHYSICAL)
        return fail(rc, std::string(where) + ": non-physical state (density or pressure <= 0)");
    if (rc == ST_NONFINITE)
        return fail(rc, std::string(where) + ": non-finite value or singular matrix");
    if (rc == ST_UNSUPPORTED)
        return fail(rc, std::string(where) + ": configuration not supported");
    return fail(rc, std::string(where) + ": error");
}

cudaStream_t S(void *s) { return (cudaStream_t)s; }

// the batched mean-value Roe flux (rsMeanValueEig with Roe_M1..M5, Gas.hpp:1272-1408)
bool mean_value_roe(const EulerSettingsD &s) { return s.rsMeanValueEig && s.rsType >= RS_Roe_M1 && s.rsType <= RS_Roe_M1 + 4; }
} // namespace

namespace dndsb
{
const MeshD &mesh_of(const dndsb_eval *e) { return e->vr->mesh->d; }
const GeomD &geom_of(const dndsb_eval *e) { return e->vr->g; }
const VRD &vr_of(const dndsb_eval *e) { return e->vr->vr; }
bool vr_ready(const dndsb_eval *e) { return e->vr->coeff; }
EvalD &eval_of(dndsb_eval *e) { return e->e; }
int set_error(int code, const std::string &msg) { return fail(code, msg); }
} // namespace dndsb

namespace
{

bool device_ok()
{
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}
} // namespace

extern "C"
{
    const char *dndsb_last_error(void) { return g_err.c_str(); }
    int dndsb_version(void) { return 1; }

    int dndsb_mesh_create(dndsb_mesh **out, int dim, int cellType, int faceType, int64_t nNode, const double *coords, int64_t nCell,
                          int nvert, const int64_t *cell2node, const double *cellShift, int64_t nFace, int nfv, const int64_t *face2node,
                          const double *faceShift, const int64_t *face2cell, const int32_t *faceZone, const double *facePShift, int nf,
                          const int64_t *cell2face)
    {
        if (!out || !coords || !cell2node || !cellShift || !face2node || !faceShift || !face2cell || !faceZone || !facePShift || !cell2face)
            return fail(DNDSB_E_BADARG, "dndsb_mesh_create: null argument");
        if ((dim != 2 && dim != 3) || nCell <= 0 || nFace <= 0 || nf <= 0 || nf > 6 || nvert > 8 || nfv > 4)
            return fail(DNDSB_E_BADARG, "dndsb_mesh_create: bad sizes");
        if (nCell >= (1LL << 30) || nFace >= (1LL << 30) || nNode >= (1LL << 31))
            return fail(DNDSB_E_UNSUPPORTED, "dndsb_mesh_create: mesh too large for 32-bit device indices");
        if (!device_ok())
            return fail(DNDSB_E_CUDA, "dndsb_mesh_create: no CUDA device");
        auto *m = new dndsb_mesh();
        MeshD &d = m->d;
        d.dim = dim, d.cellType = cellType, d.faceType = faceType, d.nvert = nvert, d.nfv = nfv, d.nf = nf;
        d.nNode = nNode, d.nCell = nCell, d.nFace = nFace;
        std::vector<int32_t> c2n(nCell * nvert), f2n(nFace * nfv), f2c(nFace * 2), c2f(nCell * nf), nbr(nCell * nf);
        for (int64_t i = 0; i < nCell * nvert; i++)
        {
            if (cell2node[i] < 0 || cell2node[i] >= nNode)
            {
                delete m;
                return fail(DNDSB_E_BADARG, "dndsb_mesh_create: cell2node out of range");
            }
            c2n[i] = (int32_t)cell2node[i];
        }
        for (int64_t i = 0; i < nFace * nfv; i++)
            f2n[i] = (int32_t)face2node[i];
        for (int64_t f = 0; f < nFace; f++)
        {
            f2c[f * 2] = (int32_t)face2cell[f * 2];
            f2c[f * 2 + 1] = (int32_t)face2cell[f * 2 + 1];
            if (f2c[f * 2] < 0 || f2c[f * 2] >= nCell || f2c[f * 2 + 1] >= nCell)
            {
                delete m;
                return fail(DNDSB_E_BADARG, "dndsb_mesh_create: face2cell out of range");
            }
            if (f2c[f * 2 + 1] < 0)
                m->nBndFace++;
        }
        for (int64_t c = 0; c < nCell; c++)
            for (int k = 0; k < nf; k++)
            {
                int64_t f = cell2face[c * nf + k];
                if (f < 0 || f >= nFace || (face2cell[f * 2] != c && face2cell[f * 2 + 1] != c))
                {
                    delete m;
                    return fail(DNDSB_E_BADARG, "dndsb_mesh_create: cell2face inconsistent with face2cell");
                }
                int side = face2cell[f * 2] == c ? 0 : 1;
                c2f[c * nf + k] = (int32_t)((f << 1) | side);
                nbr[c * nf + k] = f2c[f * 2 + 1 - side];
            }
        // slot of each face in the neighbour's row (for transposed sweeps gathered per cell)
        std::vector<int32_t> slot(nCell * nf, -1);
        for (int64_t c = 0; c < nCell; c++)
            for (int k = 0; k < nf; k++)
            {
                int o = nbr[c * nf + k];
                if (o < 0)
                    continue;
                int64_t f = cell2face[c * nf + k];
                int side = face2cell[f * 2] == c ? 0 : 1;
                for (int j = 0; j < nf; j++)
                    if (cell2face[(int64_t)o * nf + j] == f && (o != c || (c2f[(int64_t)o * nf + j] & 1) != side))
                        slot[c * nf + k] = j;
            }
        // greedy multicolouring, first fit in cell order: on a mesh numbered
        // colour by colour this reproduces the numbering's own classes, and the
        // colour-ordered sweep equals the sequential sweep of the reference
        std::vector<int32_t> color(nCell, -1);
        int nColor = 0;
        for (int64_t c = 0; c < nCell; c++)
        {
            uint64_t used = 0;
            for (int k = 0; k < nf; k++)
            {
                int o = nbr[c * nf + k];
                if (o >= 0 && o != c && color[o] >= 0 && color[o] < 64)
                    used |= 1ULL << color[o];
            }
            int col = 0;
            while (col < 64 && (used >> col & 1ULL))
                col++;
            color[c] = col;
            nColor = std::max(nColor, col + 1);
        }
        std::vector<int64_t> start(nColor + 1, 0);
        for (int64_t c = 0; c < nCell; c++)
            start[color[c] + 1]++;
        for (int i = 0; i < nColor; i++)
            start[i + 1] += start[i];
        std::vector<int32_t> cells(nCell);
        std::vector<int64_t> pos(start.begin(), start.end() - 1);
        for (int64_t c = 0; c < nCell; c++)
            cells[pos[color[c]]++] = (int32_t)c;
        d.nColor = nColor;
        d.colorStart = start;
        // boundary faces and the cells that own them (in face / cell order)
        std::vector<int32_t> bFace, bCell;
        std::vector<char> isB(nCell, 0);
        for (int64_t f = 0; f < nFace; f++)
            if (f2c[f * 2 + 1] < 0)
                bFace.push_back((int32_t)f), isB[f2c[f * 2]] = 1;
        for (int64_t c = 0; c < nCell; c++)
            if (isB[c])
                bCell.push_back((int32_t)c);
        d.nBndFace = (int64_t)bFace.size(), d.nBndCell = (int64_t)bCell.size();
        for (int32_t f : bFace)
            m->bndZoneHost.push_back(faceZone[f]);
        m->cellColorHost = color;
        int rc = 0;
        rc |= upload(&d.coords, coords, nNode * 3);
        rc |= upload(&d.cell2node, c2n.data(), nCell * nvert);
        rc |= upload(&d.cellShift, cellShift, nCell * nvert * 3);
        rc |= upload(&d.face2node, f2n.data(), nFace * nfv);
        rc |= upload(&d.faceShift, faceShift, nFace * nfv * 3);
        rc |= upload(&d.face2cell, f2c.data(), nFace * 2);
        rc |= upload(&d.faceZone, faceZone, nFace);
        rc |= upload(&d.facePShift, facePShift, nFace * 3);
        rc |= upload(&d.cell2face, c2f.data(), nCell * nf);
        rc |= upload(&d.cellNbr, nbr.data(), nCell * nf);
        rc |= upload(&d.nbrSlot, slot.data(), nCell * nf);
        rc |= upload(&d.colorCells, cells.data(), nCell);
        rc |= upload(&d.cellColor, color.data(), nCell);
        if (!bFace.empty())
        {
            rc |= upload(&d.bndFace, bFace.data(), (int64_t)bFace.size());
            rc |= upload(&d.bndCell, bCell.data(), (int64_t)bCell.size());
        }
        if (rc)
        {
            dndsb_mesh_destroy(m);
            return cuda_fail("dndsb_mesh_create");
        }
        *out = m;
        return DNDSB_OK;
    }

    int dndsb_mesh_destroy(dndsb_mesh *m)
    {
        if (!m)
            return DNDSB_OK;
        MeshD &d = m->d;
        for (void *p : {(void *)d.coords, (void *)d.cell2node, (void *)d.cellShift, (void *)d.face2node, (void *)d.faceShift, (void *)d.face2cell,
                        (void *)d.faceZone, (void *)d.facePShift, (void *)d.cell2face, (void *)d.cellNbr, (void *)d.nbrSlot, (void *)d.colorCells, (void *)d.cellColor,
                        (void *)d.bndFace, (void *)d.bndCell})
            dev_free(p);
        delete m;
        return DNDSB_OK;
    }

    int dndsb_mesh_colors(const dndsb_mesh *m, int *nColor, int32_t *cellColorHost)
    {
        if (!m || !nColor)
            return fail(DNDSB_E_BADARG, "dndsb_mesh_colors: null argument");
        *nColor = m->d.nColor;
        if (cellColorHost)
            std::memcpy(cellColorHost, m->cellColorHost.data(), sizeof(int32_t) * m->d.nCell);
        return DNDSB_OK;
    }

    int dndsb_vr_create(dndsb_vr **out, dndsb_mesh *mesh, const dndsb_vr_settings *s)
    {
        if (!out || !mesh || !s)
            return fail(DNDSB_E_BADARG, "dndsb_vr_create: null argument");
        if (s->maxOrder < 1 || s->maxOrder > 3 || s->intOrder < 0 || s->intOrder > 6)
            return fail(DNDSB_E_UNSUPPORTED, "dndsb_vr_create: maxOrder must be 1..3 and intOrder 0..6");
        auto *v = new dndsb_vr();
        v->mesh = mesh;
        VRSettingsD &d = v->vr.s;
        d.maxOrder = s->maxOrder, d.intOrder = s->intOrder, d.jacobiRelax = s->jacobiRelax, d.SORInstead = s->SORInstead;
        d.anisotropicLengths = s->anisotropicLengths, d.scaleType = s->scaleType, d.scaleMultiplier = s->scaleMultiplier;
        d.dirWeightScheme = s->dirWeightScheme;
        for (int i = 0; i < 4; i++)
            d.manualDirWeights[i] = s->manualDirWeights[i];
        d.geomWeightScheme = s->geomWeightScheme, d.geomWeightBias = s->geomWeightBias, d.geomWeightPower = s->geomWeightPower;
        d.geomWeightPower1 = s->geomWeightPower1, d.geomWeightPower2 = s->geomWeightPower2, d.bcWeight = s->bcWeight;
        if (dev_alloc((void **)&v->errWord, sizeof(int)) != cudaSuccess)
        {
            delete v;
            return cuda_fail("dndsb_vr_create");
        }
        *out = v;
        return DNDSB_OK;
    }

    int dndsb_vr_destroy(dndsb_vr *v)
    {
        if (!v)
            return DNDSB_OK;
        GeomD &g = v->g;
        for (void *p : {(void *)g.vol, (void *)g.cellBary, (void *)g.cellCent, (void *)g.cellScale, (void *)g.cellJDet, (void *)g.cellPP,
                        (void *)g.smoothRatio, (void *)g.faceArea, (void *)g.faceCent, (void *)g.faceJDet, (void *)g.facePP, (void *)g.faceNorm,
                        (void *)g.faceMeanNorm, (void *)g.cellQw, (void *)g.faceQw, (void *)g.hMax, (void *)v->vr.baseMoment, (void *)v->vr.faceWeight,
                        (void *)v->vr.faceL, (void *)v->vr.AAInvB, (void *)v->vr.AInvb, (void *)v->vr.matA, (void *)v->vr.AAInvB32,
                        (void *)v->vr.AInvb32, (void *)v->vr.sweepCoef, (void *)v->vr.sweepCoef32, (void *)v->errWord, (void *)v->vr.bnd.type, (void *)v->vr.bnd.val})
            dev_free(p);
        coords_ws_free(v->coordWs);
        dev_free(v->limSec);
        dev_free(v->siFace);
        delete v;
        return DNDSB_OK;
    }

    int dndsb_vr_construct_metrics(dndsb_vr *v)
    {
        if (!v)
            return fail(DNDSB_E_BADARG, "dndsb_vr_construct_metrics: null");
        int rc = geom_construct(v->mesh->d, v->vr.s, v->g, 0);
        v->metrics = rc == ST_OK;
        return status_msg(rc, "dndsb_vr_construct_metrics");
    }

    int dndsb_vr_construct_base_and_weight(dndsb_vr *v, const double *bcDirWeight, int nZone)
    {
        if (!v || !v->metrics)
            return fail(DNDSB_E_BADARG, "dndsb_vr_construct_base_and_weight: call construct_metrics first");
        int rc = vr_construct_base_and_weight(v->mesh->d, v->g, v->vr, bcDirWeight, nZone, 0);
        v->base = rc == ST_OK;
        return status_msg(rc, "dndsb_vr_construct_base_and_weight");
    }

    int dndsb_vr_construct_rec_coeff(dndsb_vr *v)
    {
        if (!v || !v->base)
            return fail(DNDSB_E_BADARG, "dndsb_vr_construct_rec_coeff: call construct_base_and_weight first");
        int rc = vr_construct_rec_coeff(v->mesh->d, v->g, v->vr, v->errWord, 0);
        v->coeff = rc == ST_OK;
        return status_msg(rc, "dndsb_vr_construct_rec_coeff");
    }

    int dndsb_vr_sizes(const dndsb_vr *v, int64_t *out4)
    {
        if (!v || !out4)
            return fail(DNDSB_E_BADARG, "dndsb_vr_sizes: null");
        out4[0] = v->vr.NDOF, out4[1] = v->vr.R, out4[2] = v->g.nGf, out4[3] = v->g.nGc;
        return DNDSB_OK;
    }

    int dndsb_vr_get_array(const dndsb_vr *v, const char *name, double *hostOut, int64_t cap, int64_t *len)
    {
        if (!v || !name)
            return fail(DNDSB_E_BADARG, "dndsb_vr_get_array: null");
        const MeshD &m = v->mesh->d;
        const GeomD &g = v->g;
        const VRD &r = v->vr;
        std::string n(name);
        const double *src = nullptr;
        int64_t cnt = 0;
        int R = r.R;
        if (n == "volume") src = g.vol, cnt = m.nCell;
        else if (n == "cellBary") src = g.cellBary, cnt = m.nCell * 3;
        else if (n == "cellCent") src = g.cellCent, cnt = m.nCell * 3;
        else if (n == "cellHBox") src = g.cellScale, cnt = m.nCell * 3;
        else if (n == "cellJDet") src = g.cellJDet, cnt = m.nCell * g.nGc;
        else if (n == "cellPP") src = g.cellPP, cnt = m.nCell * g.nGc * 3;
        else if (n == "smoothRatio") src = g.smoothRatio, cnt = m.nCell;
        else if (n == "cellHMax") src = g.hMax, cnt = m.nCell;
        else if (n == "faceArea") src = g.faceArea, cnt = m.nFace;
        else if (n == "faceCent") src = g.faceCent, cnt = m.nFace * 3;
        else if (n == "faceJDet") src = g.faceJDet, cnt = m.nFace * g.nGf;
        else if (n == "facePP") src = g.facePP, cnt = m.nFace * g.nGf * 3;
        else if (n == "faceNorm") src = g.faceNorm, cnt = m.nFace * g.nGf * 3;
        else if (n == "faceMeanNorm") src = g.faceMeanNorm, cnt = m.nFace * 3;
        else if (n == "baseMoment") src = r.baseMoment, cnt = m.nCell * r.NDOF;
        else if (n == "faceWeight") src = r.faceWeight, cnt = m.nFace * (r.P + 1);
        else if (n == "faceL") src = r.faceL, cnt = m.nFace;
        else if (n == "matrixAAInvB") src = r.AAInvB, cnt = m.nCell * (m.nf + 1) * R * R;
        else if (n == "vectorAInvB") src = r.AInvb, cnt = m.nCell * m.nf * R;
        else if (n == "matrixA") src = r.matA, cnt = m.nCell * R * R;
        else
            return fail(DNDSB_E_BADARG, "dndsb_vr_get_array: unknown name " + n);
        if (!src)
            return fail(DNDSB_E_BADARG, "dndsb_vr_get_array: array not constructed yet: " + n);
        if (len)
            *len = cnt;
        if (hostOut)
        {
            if (cap < cnt)
                return fail(DNDSB_E_BADARG, "dndsb_vr_get_array: buffer too small");
            if (cudaMemcpy(hostOut, src, sizeof(double) * cnt, cudaMemcpyDeviceToHost) != cudaSuccess)
                return cuda_fail("dndsb_vr_get_array");
        }
        return DNDSB_OK;
    }

    int dndsb_vr_do_reconstruction_iter(dndsb_vr *v, double *uRec, double *uRecNew, const double *u, int nVars, int putIntoNew,
                                        int recordInc, int uRecIsZero, int precision, void *stream)
    {
        if (!v || !uRec || !uRecNew || !u)
            return fail(DNDSB_E_BADARG, "dndsb_vr_do_reconstruction_iter: null argument");
        if (!v->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_vr_do_reconstruction_iter: call construct_rec_coeff first");
        if (recordInc && !putIntoNew)
            return fail(DNDSB_E_BADARG, "dndsb_vr_do_reconstruction_iter: recordInc needs putIntoNew"); // _Reconstruction.hxx:502
        if (uRec == uRecNew)
            return fail(DNDSB_E_BADARG, "dndsb_vr_do_reconstruction_iter: uRec and uRecNew must differ");
        if (v->mesh->nBndFace > 0 && v->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_vr_do_reconstruction_iter: the mesh has boundary faces; set their boundary table first");
        if (v->vr.bnd.nZone > 0 && nVars != v->bndNVars)
            return fail(DNDSB_E_BADARG, "dndsb_vr_do_reconstruction_iter: nVars differs from the boundary table's");
        if (v->vr.s.SORInstead && !recordInc) // _Reconstruction.hxx:534-611: in place on uRec, then swapped into uRecNew with putIntoNew
        {
            if (precision != 0)
                return fail(DNDSB_E_UNSUPPORTED, "dndsb_vr_do_reconstruction_iter: the SOR sweep takes FP64 coefficients");
            int rc = vr_iter_sor(v->mesh->d, v->g, v->vr, nVars, uRec, u, S(stream));
            if (rc == ST_OK && putIntoNew)
                rc = vr_swap(v->mesh->d.nCell * v->vr.R * nVars, uRec, uRecNew, S(stream));
            return status_msg(rc, "dndsb_vr_do_reconstruction_iter");
        }
        int rc = vr_iter(v->mesh->d, v->g, v->vr, nVars, uRec, uRecNew, u, recordInc, uRecIsZero, precision, S(stream));
        if (rc == ST_OK && !putIntoNew && !recordInc)
            rc = vr_swap(v->mesh->d.nCell * v->vr.R * nVars, uRec, uRecNew, S(stream));
        return status_msg(rc, "dndsb_vr_do_reconstruction_iter");
    }

    int dndsb_vr_set_boundary(dndsb_vr *v, int nZone, const int32_t *type, const double *value, int nVars, double gamma, double Rgas)
    {
        if (!v || nZone < 0 || (nZone > 0 && (!type || !value)) || nVars < 1 || nVars > 8 || !(gamma > 1) || !(Rgas > 0))
            return fail(DNDSB_E_BADARG, "dndsb_vr_set_boundary: bad argument");
        const dndsb_mesh *m = v->mesh;
        for (int z = 0; z < nZone; z++)
        {
            int t = type[z];
            if (t != 0 && t != BC_FAR && t != BC_WALL && t != BC_WALL_INVIS && t != BC_WALL_ISOTHERMAL && t != BC_OUT && t != BC_OUTP &&
                t != BC_IN && t != BC_SYM)
                return fail(DNDSB_E_UNSUPPORTED, "dndsb_vr_set_boundary: boundary type " + std::to_string(t) + " is not available");
        }
        for (int32_t z : m->bndZoneHost) // every boundary face needs a zone with a boundary type
            if (z < 0 || z >= nZone || type[z] == 0)
                return fail(DNDSB_E_BADARG, "dndsb_vr_set_boundary: boundary zone " + std::to_string(z) + " has no boundary type");
        std::vector<double> val(std::max(nZone, 1) * 8, 0.0);
        for (int z = 0; z < nZone; z++)
            for (int i = 0; i < nVars; i++)
                val[z * 8 + i] = value[z * nVars + i];
        BoundaryD &b = v->vr.bnd;
        dev_free(b.type);
        dev_free(b.val);
        b.type = nullptr, b.val = nullptr, b.nZone = 0;
        std::vector<int32_t> ty(type, type + nZone);
        if (nZone > 0 && (upload(&b.type, ty.data(), nZone) || upload(&b.val, val.data(), (int64_t)nZone * 8)))
            return cuda_fail("dndsb_vr_set_boundary");
        b.nZone = nZone, b.gamma = gamma, b.Rgas = Rgas;
        b.viscFree = true;
        for (int32_t z : m->bndZoneHost)
            b.viscFree = b.viscFree && (type[z] == BC_FAR || type[z] == BC_OUT || type[z] == BC_WALL_INVIS || type[z] == BC_SYM);
        v->bndNVars = nVars;
        return DNDSB_OK;
    }

    int dndsb_vr_iter_vjp(dndsb_vr *v, const double *cot, const double *uRec, const double *u, int nVars, double *vRec, double *vU, void *stream)
    {
        if (!v || !cot || !uRec || !u || !vRec || !vU)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_vjp: null argument");
        if (!v->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_vjp: call construct_rec_coeff first");
        if (v->mesh->nBndFace > 0 && v->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_vjp: the mesh has boundary faces; set their boundary table first");
        return status_msg(vr_vjp(v->mesh->d, v->g, v->vr, nVars, cot, uRec, u, vRec, vU, S(stream)), "dndsb_vr_iter_vjp");
    }

    int dndsb_vr_iter_vjp_coords(dndsb_vr *v, const double *cot, const double *uRec, const double *u, int nVars, double *dX, void *stream)
    {
        if (!v || !cot || !uRec || !u || !dX)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_vjp_coords: null argument");
        if (!v->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_vjp_coords: call construct_rec_coeff first");
        if (v->mesh->nBndFace > 0 && v->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_vjp_coords: the mesh has boundary faces; set their boundary table first");
        if (nVars != 5)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_vjp_coords: needs nVars = 5");
        int rc = coords_vjp(v->mesh->d, v->g, v->vr, nullptr, nullptr, v->coordWs, nullptr, cot, u, uRec, dX, v->errWord, S(stream));
        if (rc == ST_UNSUPPORTED)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_vjp_coords: VR degree 1-2 in 3-D, 1-3 in 2-D");
        return status_msg(rc, "dndsb_vr_iter_vjp_coords");
    }

    int dndsb_vr_iter_jvp_coords(dndsb_vr *v, const double *dX, const double *uRec, const double *u, int nVars, double *dRecNew, void *stream)
    {
        if (!v || !dX || !uRec || !u || !dRecNew)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_jvp_coords: null argument");
        if (!v->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_jvp_coords: call construct_rec_coeff first");
        if (v->mesh->nBndFace > 0 && v->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_jvp_coords: the mesh has boundary faces; set their boundary table first");
        if (nVars != 5)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_jvp_coords: needs nVars = 5");
        int rc = coords_jvp(v->mesh->d, v->g, v->vr, nullptr, nullptr, v->coordWs, dX, u, uRec, nullptr, dRecNew, v->errWord, S(stream));
        if (rc == ST_UNSUPPORTED)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_jvp_coords: VR degree 1-2 in 3-D, 1-3 in 2-D");
        return status_msg(rc, "dndsb_vr_iter_jvp_coords");
    }

    int dndsb_vr_iter_jvp(dndsb_vr *v, const double *dRec, const double *du, const double *uRec, const double *u, int nVars, double *dRecNew,
                          void *stream)
    {
        if (!v || !dRec || !du || !uRec || !u || !dRecNew)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_jvp: null argument");
        if (!v->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_jvp: call construct_rec_coeff first");
        if (v->mesh->nBndFace > 0 && v->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_vr_iter_jvp: the mesh has boundary faces; set their boundary table first");
        return status_msg(vr_jvp(v->mesh->d, v->g, v->vr, nVars, dRec, du, uRec, u, dRecNew, S(stream)), "dndsb_vr_iter_jvp");
    }

    int dndsb_eval_create(dndsb_eval **out, dndsb_vr *vr, const dndsb_euler_settings *s)
    {
        if (!out || !vr || !s)
            return fail(DNDSB_E_BADARG, "dndsb_eval_create: null argument");
        if (s->nVars != 5 && s->nVars != 6)
            return fail(DNDSB_E_UNSUPPORTED, "dndsb_eval_create: nVars must be 5 (NS) or 6 (NS_SA)");
        auto *e = new dndsb_eval();
        e->vr = vr;
        EulerSettingsD &d = e->e.s;
        d.nVars = s->nVars, d.rsType = s->rsType, d.rsFixScale = s->rsFixScale, d.rsIncFScale = s->rsIncFScale;
        d.gamma = s->gamma, d.Rgas = s->Rgas, d.muGas = s->muGas, d.prGas = s->prGas, d.TRef = s->TRef, d.CSutherland = s->CSutherland;
        d.muModel = s->muModel, d.ignoreVis = s->ignoreVis;
        d.rsMeanValueEig = s->rsMeanValueEig;
        d.derive();
        const MeshD &m = vr->mesh->d;
        int rc = 0;
        rc |= dev_alloc((void **)&e->e.lambdaFace, sizeof(real) * m.nFace);
        rc |= dev_alloc((void **)&e->e.lambdaFaceC, sizeof(real) * m.nFace);
        rc |= dev_alloc((void **)&e->e.lambdaFaceVis, sizeof(real) * m.nFace);
        rc |= dev_alloc((void **)&e->e.lambdaConv, sizeof(real) * m.nFace);
        rc |= dev_alloc((void **)&e->e.deltaLambdaFace, sizeof(real) * m.nFace);
        rc |= dev_alloc((void **)&e->e.deltaLambdaCell, sizeof(real) * m.nCell);
        rc |= dev_alloc((void **)&e->e.faceFlux, sizeof(real) * std::max(m.nFace, m.nCell) * s->nVars);
        rc |= dev_alloc((void **)&e->e.redBuf, sizeof(real) * kRedBufLen);
        rc |= dev_alloc((void **)&e->e.errWord, sizeof(int));
        rc |= dev_alloc((void **)&e->e.errDeferred, sizeof(int));
        rc |= dev_alloc((void **)&e->e.fluxWall, sizeof(real) * 8);
        rc |= dev_alloc((void **)&e->e.objDir, sizeof(real) * 8);
        if (s->nVars == 6)
            rc |= dev_alloc((void **)&e->e.jSource, sizeof(real) * m.nCell * 6);
        if (rc)
        {
            dndsb_eval_destroy(e);
            return cuda_fail("dndsb_eval_create");
        }
        if (e->e.jSource)
            cudaMemset(e->e.jSource, 0, sizeof(real) * m.nCell * 6);
        if (fast_geometry(m, vr->g, vr->vr, e->e, 0) != ST_OK)
        {
            dndsb_eval_destroy(e);
            return cuda_fail("dndsb_eval_create");
        }
        cudaMemset(e->e.deltaLambdaCell, 0, sizeof(real) * m.nCell);
        cudaMemset(e->e.lambdaFace, 0, sizeof(real) * m.nFace);
        cudaMemset(e->e.lambdaConv, 0, sizeof(real) * m.nFace);
        cudaMemset(e->e.errDeferred, 0, sizeof(int));
        cudaMemset(e->e.fluxWall, 0, sizeof(real) * 8);
        *out = e;
        return DNDSB_OK;
    }

    int dndsb_eval_set_bc(dndsb_eval *e, int nZone, const int32_t *type, const double *value)
    {
        if (!e)
            return fail(DNDSB_E_BADARG, "dndsb_eval_set_bc: null argument");
        int rc = dndsb_vr_set_boundary(e->vr, nZone, type, value, e->e.s.nVars, e->e.s.gamma, e->e.s.Rgas);
        if (rc != DNDSB_OK)
            return rc;
        return DNDSB_OK;
    }

    int dndsb_eval_set_wall_distance(dndsb_eval *e, const double *dHost)
    {
        if (!e || !dHost)
            return fail(DNDSB_E_BADARG, "dndsb_eval_set_wall_distance: null argument");
        const MeshD &m = e->vr->mesh->d;
        int64_t n = m.nCell * (int64_t)e->vr->g.nGc;
        if (n <= 0)
            return fail(DNDSB_E_BADARG, "dndsb_eval_set_wall_distance: construct the reconstruction first");
        dev_free(e->e.dWall);
        e->e.dWall = nullptr;
        if (upload(&e->e.dWall, dHost, n))
            return cuda_fail("dndsb_eval_set_wall_distance");
        return DNDSB_OK;
    }

    int dndsb_eval_destroy(dndsb_eval *e)
    {
        if (!e)
            return DNDSB_OK;
        for (void *p : {(void *)e->e.lambdaFace, (void *)e->e.lambdaFaceC, (void *)e->e.lambdaFaceVis, (void *)e->e.lambdaConv,
                        (void *)e->e.deltaLambdaFace, (void *)e->e.deltaLambdaCell, (void *)e->e.faceFlux, (void *)e->e.redBuf, (void *)e->e.errWord,
                        (void *)e->e.facePt, (void *)e->e.cellPar, (void *)e->e.adjBuf, (void *)e->e.dWall, (void *)e->e.jSource,
                        (void *)e->e.errDeferred, (void *)e->e.fluxWall, (void *)e->e.objDir, (void *)e->e.lambdaFace0, (void *)e->e.luOff,
                        (void *)e->e.luDinv, (void *)e->e.luDiag})
            dev_free(p);
        linws_free(e->lin);
        delete e;
        return DNDSB_OK;
    }

    int dndsb_eval_initialize_udof(dndsb_eval *e, int kind, double chi, double *u, void *stream)
    {
        if (!e || !u || (kind != 2 && kind != 3))
            return fail(DNDSB_E_BADARG, "dndsb_eval_initialize_udof: bad argument");
        return status_msg(init_field(e->vr->mesh->d, e->vr->g, e->e, kind, chi, u, S(stream)), "dndsb_eval_initialize_udof");
    }

    int dndsb_eval_evaluate_dt(dndsb_eval *e, const double *u, double CFL, double MaxDt, int useLocalDt, double *dt, double *dtMinHost,
                               void *stream)
    {
        if (!e || !u || !dt)
            return fail(DNDSB_E_BADARG, "dndsb_eval_evaluate_dt: null argument");
        return status_msg(eval_dt(e->vr->mesh->d, e->vr->g, e->e, u, CFL, MaxDt, useLocalDt, dt, dtMinHost, S(stream)),
                          "dndsb_eval_evaluate_dt");
    }

    int dndsb_eval_evaluate_rhs(dndsb_eval *e, double *rhs, const double *u, const double *uRec, void *stream)
    {
        if (!e || !rhs || !u || !uRec)
            return fail(DNDSB_E_BADARG, "dndsb_eval_evaluate_rhs: null argument");
        if (!e->vr->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_eval_evaluate_rhs: VR not constructed");
        if (e->vr->mesh->nBndFace > 0 && e->vr->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_eval_evaluate_rhs: the mesh has boundary faces; call dndsb_eval_set_bc first");
        if (e->e.s.nVars == 6 && !e->e.dWall)
            return fail(DNDSB_E_BADARG, "dndsb_eval_evaluate_rhs: the SA model needs the wall distance (dndsb_eval_set_wall_distance)");
        return status_msg(eval_rhs(e->vr->mesh->d, e->vr->g, e->vr->vr, e->e, u, uRec, rhs, nullptr, S(stream)), "dndsb_eval_evaluate_rhs");
    }

    int dndsb_eval_evaluate_rhs_full(dndsb_eval *e, double *rhs, double *JSource, const double *u, const double *uRecUnlim, const double *uRec,
                                     const double *uRecBeta, const double *cellRHSAlpha, int onlyOnHalfAlpha, double t, uint64_t flags,
                                     void *stream)
    {
        (void)uRecBeta, (void)onlyOnHalfAlpha, (void)t; // not read by the reference's EvaluateRHS body either
        if (!e || !rhs || !u || !uRecUnlim || !uRec)
            return fail(DNDSB_E_BADARG, "dndsb_eval_evaluate_rhs_full: null argument");
        if (!e->vr->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_eval_evaluate_rhs_full: VR not constructed");
        if (e->vr->mesh->nBndFace > 0 && e->vr->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_eval_evaluate_rhs_full: the mesh has boundary faces; call dndsb_eval_set_bc first");
        if (e->e.s.nVars == 6 && !e->e.dWall)
            return fail(DNDSB_E_BADARG, "dndsb_eval_evaluate_rhs_full: the SA model needs the wall distance (dndsb_eval_set_wall_distance)");
        const uint64_t known = DNDSB_RHS_IGNORE_VISCOSITY | DNDSB_RHS_DONT_UPDATE_INTEGRATION | DNDSB_RHS_DONT_RECORD_BND_FLUX;
        if (flags & ~known)
            return fail(DNDSB_E_UNSUPPORTED, "dndsb_eval_evaluate_rhs_full: the direct second-order reconstruction flags are not supported");
        return status_msg(eval_rhs_ex(e->vr->mesh->d, e->vr->g, e->vr->vr, e->e, u, uRecUnlim, uRec, cellRHSAlpha, (unsigned)flags, rhs, nullptr,
                                      JSource, S(stream)),
                          "dndsb_eval_evaluate_rhs_full");
    }

    int dndsb_eval_set_deferred_errors(dndsb_eval *e, int deferred)
    {
        if (!e)
            return fail(DNDSB_E_BADARG, "dndsb_eval_set_deferred_errors: null argument");
        e->e.deferErr = deferred != 0;
        return DNDSB_OK;
    }

    int dndsb_eval_check_errors(dndsb_eval *e, void *stream)
    {
        if (!e)
            return fail(DNDSB_E_BADARG, "dndsb_eval_check_errors: null argument");
        int w = 0;
        d2h(&w, e->e.errDeferred, sizeof(int), S(stream));
        dev_zero(e->e.errDeferred, sizeof(int), S(stream));
        if (dev_sync(S(stream)) != cudaSuccess)
            return cuda_fail("dndsb_eval_check_errors");
        if (w & DE_NONPHYSICAL)
            return status_msg(ST_NONPHYSICAL, "dndsb_eval_check_errors");
        if (w & DE_NONFINITE)
            return status_msg(ST_NONFINITE, "dndsb_eval_check_errors");
        return DNDSB_OK;
    }

    int dndsb_eval_rhs_vjp(dndsb_eval *e, const double *w, const double *u, const double *uRec, double *du, double *duRec, void *stream)
    {
        if (!e || !w || !u || !uRec || !du || !duRec)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_vjp: null argument");
        if (!e->vr->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_vjp: VR not constructed");
        if (e->vr->mesh->nBndFace > 0 && e->vr->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_vjp: the mesh has boundary faces; call dndsb_eval_set_bc first");
        if (e->e.s.nVars == 6 && !e->e.dWall)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_vjp: the SA model needs the wall distance (dndsb_eval_set_wall_distance)");
        int rc = rhs_vjp(e->vr->mesh->d, e->vr->g, e->vr->vr, e->e, w, u, uRec, du, duRec, S(stream));
        if (rc == ST_UNSUPPORTED)
            return fail(rc, "dndsb_eval_rhs_vjp: the SA model and viscous boundary zones are differentiated on 3-D meshes at VR degree 1-2");
        return status_msg(rc, "dndsb_eval_rhs_vjp");
    }

    int dndsb_eval_wall_flux_vjp(dndsb_eval *e, const double *dirHost, const double *u, const double *uRec, double *du, double *duRec,
                                 void *stream)
    {
        if (!e || !dirHost || !u || !uRec || !du || !duRec)
            return fail(DNDSB_E_BADARG, "dndsb_eval_wall_flux_vjp: null argument");
        if (!e->vr->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_eval_wall_flux_vjp: VR not constructed");
        if (e->vr->mesh->nBndFace == 0 || e->vr->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_eval_wall_flux_vjp: the mesh has no boundary table");
        if (e->e.s.nVars == 6 && !e->e.dWall)
            return fail(DNDSB_E_BADARG, "dndsb_eval_wall_flux_vjp: the SA model needs the wall distance (dndsb_eval_set_wall_distance)");
        h2d(e->e.objDir, dirHost, sizeof(real) * e->e.s.nVars, S(stream));
        int rc = rhs_vjp_generic(e->vr->mesh->d, e->vr->g, e->vr->vr, e->e, nullptr, e->e.objDir, u, uRec, du, duRec, S(stream));
        if (rc == ST_UNSUPPORTED)
            return fail(rc, "dndsb_eval_wall_flux_vjp: needs a 3-D mesh and VR degree 1-2");
        return status_msg(rc, "dndsb_eval_wall_flux_vjp");
    }

    int dndsb_eval_rhs_vjp_coords(dndsb_eval *e, const double *w, const double *u, const double *uRec, double *dX, void *stream)
    {
        if (!e || !w || !u || !uRec || !dX)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_vjp_coords: null argument");
        if (!e->vr->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_vjp_coords: VR not constructed");
        if (e->vr->mesh->nBndFace > 0 && e->vr->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_vjp_coords: the mesh has boundary faces; call dndsb_eval_set_bc first");
        if (mean_value_roe(e->e.s))
            return fail(DNDSB_E_UNSUPPORTED, "dndsb_eval_rhs_vjp_coords: rsMeanValueEig with Roe_M1..M5 is differentiated with respect to the state only");
        dndsb_vr *v = e->vr;
        int rc = coords_vjp(v->mesh->d, v->g, v->vr, &e->e.s, e->e.deltaLambdaCell, v->coordWs, w, nullptr, u, uRec, dX, e->e.errWord, S(stream));
        if (rc == ST_UNSUPPORTED)
            return fail(rc, "dndsb_eval_rhs_vjp_coords: needs nVars = 5, ignoreVis, and VR degree 1-2 in 3-D, 1-3 in 2-D");
        return status_msg(rc, "dndsb_eval_rhs_vjp_coords");
    }

    int dndsb_eval_residual_vjp_coords(dndsb_eval *e, const double *w, const double *cot, const double *u, const double *uRec, double *dX,
                                       void *stream)
    {
        if (!e || !w || !cot || !u || !uRec || !dX)
            return fail(DNDSB_E_BADARG, "dndsb_eval_residual_vjp_coords: null argument");
        if (!e->vr->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_eval_residual_vjp_coords: VR not constructed");
        if (e->vr->mesh->nBndFace > 0 && e->vr->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_eval_residual_vjp_coords: the mesh has boundary faces; call dndsb_eval_set_bc first");
        if (mean_value_roe(e->e.s))
            return fail(DNDSB_E_UNSUPPORTED, "dndsb_eval_residual_vjp_coords: rsMeanValueEig with Roe_M1..M5 is differentiated with respect to the state only");
        dndsb_vr *v = e->vr;
        int rc = coords_vjp(v->mesh->d, v->g, v->vr, &e->e.s, e->e.deltaLambdaCell, v->coordWs, w, cot, u, uRec, dX, e->e.errWord, S(stream));
        if (rc == ST_UNSUPPORTED)
            return fail(rc, "dndsb_eval_residual_vjp_coords: needs nVars = 5, ignoreVis, and VR degree 1-2 in 3-D, 1-3 in 2-D");
        return status_msg(rc, "dndsb_eval_residual_vjp_coords");
    }

    int dndsb_eval_rhs_jvp_coords(dndsb_eval *e, const double *dX, const double *u, const double *uRec, double *dRhs, void *stream)
    {
        if (!e || !dX || !u || !uRec || !dRhs)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_jvp_coords: null argument");
        if (!e->vr->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_jvp_coords: VR not constructed");
        if (e->vr->mesh->nBndFace > 0 && e->vr->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_jvp_coords: the mesh has boundary faces; call dndsb_eval_set_bc first");
        if (mean_value_roe(e->e.s))
            return fail(DNDSB_E_UNSUPPORTED, "dndsb_eval_rhs_jvp_coords: rsMeanValueEig with Roe_M1..M5 is differentiated with respect to the state only");
        dndsb_vr *v = e->vr;
        int rc = coords_jvp(v->mesh->d, v->g, v->vr, &e->e.s, e->e.deltaLambdaCell, v->coordWs, dX, u, uRec, dRhs, nullptr, e->e.errWord, S(stream));
        if (rc == ST_UNSUPPORTED)
            return fail(rc, "dndsb_eval_rhs_jvp_coords: needs nVars = 5, ignoreVis, and VR degree 1-2 in 3-D, 1-3 in 2-D");
        return status_msg(rc, "dndsb_eval_rhs_jvp_coords");
    }

    int dndsb_eval_rhs_jvp(dndsb_eval *e, const double *du, const double *duRec, const double *u, const double *uRec, double *dRhs, void *stream)
    {
        if (!e || !du || !duRec || !u || !uRec || !dRhs)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_jvp: null argument");
        if (!e->vr->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_jvp: VR not constructed");
        if (e->vr->mesh->nBndFace > 0 && e->vr->vr.bnd.nZone == 0)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_jvp: the mesh has boundary faces; call dndsb_eval_set_bc first");
        if (e->e.s.nVars == 6 && !e->e.dWall)
            return fail(DNDSB_E_BADARG, "dndsb_eval_rhs_jvp: the SA model needs the wall distance (dndsb_eval_set_wall_distance)");
        int rc = rhs_jvp(e->vr->mesh->d, e->vr->g, e->vr->vr, e->e, du, duRec, u, uRec, dRhs, S(stream));
        if (rc == ST_UNSUPPORTED)
            return fail(rc, "dndsb_eval_rhs_jvp: the SA model and viscous boundary zones are differentiated on 3-D meshes at VR degree 1-2");
        return status_msg(rc, "dndsb_eval_rhs_jvp");
    }

    int dndsb_eval_set_jacobian_mode(dndsb_eval *e, int useScalarJacobian, int useRoeJacobian)
    {
        if (!e)
            return fail(DNDSB_E_BADARG, "dndsb_eval_set_jacobian_mode: null argument");
        if (useScalarJacobian && useRoeJacobian) // EulerEvaluatorSettings.hpp:416-417
            return fail(DNDSB_E_BADARG, "dndsb_eval_set_jacobian_mode: useScalarJacobian and useRoeJacobian are mutually exclusive");
        if (useRoeJacobian && !e->e.lambdaFace0)
        {
            const MeshD &m = e->vr->mesh->d;
            if (dev_alloc((void **)&e->e.lambdaFace0, sizeof(real) * 3 * m.nFace) != cudaSuccess)
                return cuda_fail("dndsb_eval_set_jacobian_mode");
            e->e.lambdaFace123 = e->e.lambdaFace0 + m.nFace, e->e.lambdaFace4 = e->e.lambdaFace0 + 2 * m.nFace;
            // the convective speed of the last EvaluateDt until the next EvaluateRHS records the eigenvalues
            for (real *l : {e->e.lambdaFace0, e->e.lambdaFace123, e->e.lambdaFace4})
                if (cudaMemcpy(l, e->e.lambdaConv, sizeof(real) * m.nFace, cudaMemcpyDeviceToDevice) != cudaSuccess)
                    return cuda_fail("dndsb_eval_set_jacobian_mode");
        }
        e->e.jacMode = useRoeJacobian ? 2 : (useScalarJacobian ? 0 : 1);
        return DNDSB_OK;
    }

    int dndsb_eval_lusgs_matrix_init(dndsb_eval *e, const double *dTau, double dt, double alphaDiag, double *jdiag, void *stream)
    {
        if (!e || !dTau || !jdiag)
            return fail(DNDSB_E_BADARG, "dndsb_eval_lusgs_matrix_init: null argument");
        if (e->e.jacMode == 2)
            return fail(DNDSB_E_BADARG, "dndsb_eval_lusgs_matrix_init: the Roe Jacobian needs u: use dndsb_eval_lusgs_matrix_init_full");
        if (e->e.jacMode == 1)
            return dndsb_eval_lusgs_matrix_init_full(e, dTau, dt, alphaDiag, nullptr, nullptr, 0, 0.0, jdiag, stream);
        return status_msg(lusgs_init(e->vr->mesh->d, e->vr->g, e->e, dTau, dt, alphaDiag, jdiag, S(stream)), "dndsb_eval_lusgs_matrix_init");
    }

    int dndsb_eval_lusgs_matrix_init_full(dndsb_eval *e, const double *dTau, double dt, double alphaDiag, const double *u, const double *uRec,
                                          int jacobianCode, double t, double *jdiag, void *stream)
    {
        (void)uRec, (void)t; // read by neither the scalar nor the block branch of the reference (EulerEvaluator.hxx:37-159)
        if (!e || !dTau || !jdiag || (e->e.jacMode == 2 && !u))
            return fail(DNDSB_E_BADARG, "dndsb_eval_lusgs_matrix_init_full: null argument");
        if (jacobianCode != 0) // EulerEvaluator.hxx:49
            return fail(DNDSB_E_BADARG, "dndsb_eval_lusgs_matrix_init_full: jacobianCode must be 0");
        const MeshD &m = e->vr->mesh->d;
        if (e->e.jacMode == 0)
            return status_msg(lusgs_init(m, e->vr->g, e->e, dTau, dt, alphaDiag, jdiag, S(stream)), "dndsb_eval_lusgs_matrix_init_full");
        if (e->e.jacMode == 2 && m.nBndFace > 0 && !e->vr->vr.bnd.type)
            return fail(DNDSB_E_BADARG, "dndsb_eval_lusgs_matrix_init_full: set the boundary table first");
        int rc = lusgs_init_block(m, e->vr->g, e->vr->vr, e->e, dTau, dt, alphaDiag, u, jdiag, S(stream));
        if (rc == ST_NONFINITE)
            return fail(DNDSB_E_NONFINITE, "dndsb_eval_lusgs_matrix_init_full: singular or non-finite diagonal block");
        return status_msg(rc, "dndsb_eval_lusgs_matrix_init_full");
    }

    int dndsb_eval_lusgs_matrix_to_jacobian_lu(dndsb_eval *e, double alphaDiag, const double *u, const double *jdiag, void *stream)
    {
        if (!e || !u || !jdiag)
            return fail(DNDSB_E_BADARG, "dndsb_eval_lusgs_matrix_to_jacobian_lu: null argument");
        int rc = jacobian_lu(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, u, jdiag, S(stream));
        if (rc == ST_NONFINITE)
            return fail(DNDSB_E_NONFINITE, "dndsb_eval_lusgs_matrix_to_jacobian_lu: singular pivot block");
        return status_msg(rc, "dndsb_eval_lusgs_matrix_to_jacobian_lu");
    }

    int dndsb_eval_lusgs_matrix_solve_jacobian_lu(dndsb_eval *e, double alphaDiag, const double *rhs, const double *u, const double *uInc,
                                                  double *uIncNew, const double *jdiag, int uIncIsZero, double *sumIncHost, void *stream)
    {
        if (!e || !rhs || !u || !uInc || !uIncNew || !jdiag)
            return fail(DNDSB_E_BADARG, "dndsb_eval_lusgs_matrix_solve_jacobian_lu: null argument");
        if (uInc == uIncNew || rhs == uIncNew) // EulerEvaluator.hxx:919
            return fail(DNDSB_E_BADARG, "dndsb_eval_lusgs_matrix_solve_jacobian_lu: uIncNew must differ from uInc and rhs");
        if (!e->e.luOff)
            return fail(DNDSB_E_BADARG, "dndsb_eval_lusgs_matrix_solve_jacobian_lu: build the local LU first (lusgs_matrix_to_jacobian_lu)");
        return status_msg(solve_jacobian_lu(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, rhs, u, uInc, uIncNew, jdiag, uIncIsZero, sumIncHost,
                                            S(stream)),
                          "dndsb_eval_lusgs_matrix_solve_jacobian_lu");
    }

    int dndsb_eval_update_sgs(dndsb_eval *e, double alphaDiag, const double *rhs, const double *u, const double *uInc, double *uIncNew,
                              const double *jdiag, int forward, int gsUpdate, int uIncIsZero, double *sumIncHost, void *stream)
    {
        if (!e || !rhs || !u || !uInc || !uIncNew || !jdiag)
            return fail(DNDSB_E_BADARG, "dndsb_eval_update_sgs: null argument");
        if (uInc == uIncNew)
            return fail(DNDSB_E_BADARG, "dndsb_eval_update_sgs: uInc and uIncNew must differ"); // EulerEvaluator.hxx:563
        if (e->e.jacMode)
            return status_msg(update_sgs_block(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, rhs, u, uInc, uIncNew, jdiag, forward, gsUpdate,
                                               uIncIsZero, sumIncHost, S(stream)),
                              "dndsb_eval_update_sgs");
        return status_msg(update_sgs(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, rhs, u, uInc, uIncNew, jdiag, forward, gsUpdate, uIncIsZero,
                                     sumIncHost, S(stream)),
                          "dndsb_eval_update_sgs");
    }

    int dndsb_eval_update_lusgs_forward(dndsb_eval *e, double alphaDiag, const double *rhs, const double *u, const double *uInc,
                                        const double *jdiag, double *uIncNew, void *stream)
    {
        if (!e || !rhs || !u || !uInc || !jdiag || !uIncNew)
            return fail(DNDSB_E_BADARG, "dndsb_eval_update_lusgs_forward: null argument");
        if (e->e.jacMode)
            return status_msg(update_lusgs_block(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, rhs, u, uInc, uIncNew, jdiag, 1, S(stream)),
                              "dndsb_eval_update_lusgs_forward");
        return status_msg(update_lusgs(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, rhs, u, uInc, uIncNew, jdiag, 1, S(stream)),
                          "dndsb_eval_update_lusgs_forward");
    }

    int dndsb_eval_update_lusgs_backward(dndsb_eval *e, double alphaDiag, const double *rhs, const double *u, const double *uInc,
                                         const double *jdiag, double *uIncNew, void *stream)
    {
        if (!e || !rhs || !u || !uInc || !jdiag || !uIncNew)
            return fail(DNDSB_E_BADARG, "dndsb_eval_update_lusgs_backward: null argument");
        if (e->e.jacMode)
            return status_msg(update_lusgs_block(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, rhs, u, uInc, uIncNew, jdiag, 0, S(stream)),
                              "dndsb_eval_update_lusgs_backward");
        return status_msg(update_lusgs(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, rhs, u, uInc, uIncNew, jdiag, 0, S(stream)),
                          "dndsb_eval_update_lusgs_backward");
    }

    int dndsb_eval_fix_umax_filter(dndsb_eval *e, double *u, void *stream)
    {
        (void)stream;
        if (!e || !u)
            return fail(DNDSB_E_BADARG, "dndsb_eval_fix_umax_filter: null argument");
        return DNDSB_OK; // EulerEvaluator.hxx:1318-1323 returns before touching u
    }

    int dndsb_eval_lusgs_matrix_vec(dndsb_eval *e, double alphaDiag, const double *u, const double *uInc, const double *jdiag,
                                    double *AuInc, void *stream)
    {
        if (!e || !u || !uInc || !jdiag || !AuInc)
            return fail(DNDSB_E_BADARG, "dndsb_eval_lusgs_matrix_vec: null argument");
        if (e->e.jacMode)
            return status_msg(lusgs_matvec_block(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, u, uInc, jdiag, AuInc, S(stream)),
                              "dndsb_eval_lusgs_matrix_vec");
        return status_msg(lusgs_matvec(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, u, uInc, jdiag, AuInc, S(stream)),
                          "dndsb_eval_lusgs_matrix_vec");
    }

    int dndsb_eval_lusgs_matrix_vec_t(dndsb_eval *e, double alphaDiag, const double *u, const double *y, const double *jdiag, double *ATy,
                                      void *stream)
    {
        if (!e || !u || !y || !jdiag || !ATy || y == ATy)
            return fail(DNDSB_E_BADARG, "dndsb_eval_lusgs_matrix_vec_t: null or aliased argument");
        if (e->e.jacMode)
            return fail(DNDSB_E_UNSUPPORTED, "dndsb_eval_lusgs_matrix_vec_t: the transposed operators take the scalar Jacobian");
        return status_msg(lusgs_matvec_t(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, u, y, jdiag, ATy, S(stream)),
                          "dndsb_eval_lusgs_matrix_vec_t");
    }

    int dndsb_eval_update_sgs_t(dndsb_eval *e, double alphaDiag, const void *b, const double *u, const void *y, void *yNew,
                                const double *jdiag, int forward, int gsUpdate, int precision, void *stream)
    {
        if (!e || !b || !u || !y || !yNew || !jdiag || precision < 0 || precision > 1)
            return fail(DNDSB_E_BADARG, "dndsb_eval_update_sgs_t: null argument or bad precision");
        if (y == yNew)
            return fail(DNDSB_E_BADARG, "dndsb_eval_update_sgs_t: y and yNew must differ");
        if (e->e.jacMode)
            return fail(DNDSB_E_UNSUPPORTED, "dndsb_eval_update_sgs_t: the transposed operators take the scalar Jacobian");
        return status_msg(update_sgs_t(e->vr->mesh->d, e->vr->g, e->e, alphaDiag, b, u, y, yNew, jdiag, forward, gsUpdate, precision, S(stream)),
                          "dndsb_eval_update_sgs_t");
    }

    int dndsb_vr_smooth_indicator(dndsb_vr *v, const double *u, const double *uRec, int nVars, double *si, void *stream)
    {
        if (!v || !u || !uRec || !si)
            return fail(DNDSB_E_BADARG, "dndsb_vr_smooth_indicator: null argument");
        if (!v->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_vr_smooth_indicator: call construct_rec_coeff first");
        int rc = smooth_indicator(v->mesh->d, v->g, v->vr, nVars, u, uRec, &v->siFace, si, S(stream));
        if (rc == ST_UNSUPPORTED)
            return fail(DNDSB_E_BADARG, "dndsb_vr_smooth_indicator: 3-D meshes, VR degree 1-2, 5 or 6 variables");
        return status_msg(rc, "dndsb_vr_smooth_indicator");
    }

    int dndsb_eval_limiter_wbap_c(dndsb_eval *e, const double *u, const double *uRec, const double *si, double *uRecNew, double smoothThreshold,
                                  double nStd, int ifAll, void *stream)
    {
        if (!e || !u || !uRec || !si || !uRecNew || uRec == uRecNew)
            return fail(DNDSB_E_BADARG, "dndsb_eval_limiter_wbap_c: null argument, or uRecNew aliases uRec");
        dndsb_vr *v = e->vr;
        if (!v->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_eval_limiter_wbap_c: VR not constructed");
        int rc = lim_secondary_build(v->mesh->d, v->g, v->vr, &v->limSec, v->errWord, S(stream));
        if (rc == ST_OK)
            rc = limiter_wbap_c(v->mesh->d, v->g, v->vr, v->limSec, e->e.s.nVars, e->e.s.gamma, u, uRec, si, uRecNew, smoothThreshold, nStd, ifAll,
                                S(stream));
        if (rc == ST_UNSUPPORTED)
            return fail(DNDSB_E_BADARG, "dndsb_eval_limiter_wbap_c: 3-D meshes, VR degree 1-2, 5 or 6 variables");
        if (rc == ST_NONFINITE)
            return fail(rc, "dndsb_eval_limiter_wbap_c: a face-centre derivative basis is singular");
        return status_msg(rc, "dndsb_eval_limiter_wbap_c");
    }

    int dndsb_eval_cell_rhs_alpha(dndsb_eval *e, const double *u, const double *res, double *alpha, double refRho, double refP, double relax,
                                  int compress, double compressPower, int ppEpsIsRelaxed, int flag, int64_t *nLimHost, double *alphaMinHost,
                                  void *stream)
    {
        if (!e || !u || !res || !alpha)
            return fail(DNDSB_E_BADARG, "dndsb_eval_cell_rhs_alpha: null argument");
        if (!(refRho > 0 && refP > 0))
            return fail(DNDSB_E_BADARG, "dndsb_eval_cell_rhs_alpha: refRho and refP must be positive");
        if (ppEpsIsRelaxed && !(relax < 1))
            return fail(DNDSB_E_BADARG, "dndsb_eval_cell_rhs_alpha: relaxed floors need relax < 1");
        int rc = cell_rhs_alpha(e->vr->mesh->d, e->e, u, res, alpha, refRho, refP, relax, compress, compressPower, ppEpsIsRelaxed, flag, nLimHost,
                                alphaMinHost, S(stream));
        return status_msg(rc, "dndsb_eval_cell_rhs_alpha");
    }

    int dndsb_eval_cell_rhs_alpha_expansion(dndsb_eval *e, const double *u, const double *res, double *alpha, double refRho, double refP,
                                            double alphaMin, void *stream)
    {
        if (!e || !u || !res || !alpha)
            return fail(DNDSB_E_BADARG, "dndsb_eval_cell_rhs_alpha_expansion: null argument");
        return status_msg(cell_rhs_alpha_expansion(e->vr->mesh->d, e->e, u, res, alpha, refRho, refP, alphaMin, S(stream)),
                          "dndsb_eval_cell_rhs_alpha_expansion");
    }

    int dndsb_eval_add_fixed_increment(dndsb_eval *e, double *u, const double *inc, double alpha, double refRho, double refP, int ppEpsIsRelaxed,
                                       double *alphaFixMinHost, void *stream)
    {
        if (!e || !u || !inc)
            return fail(DNDSB_E_BADARG, "dndsb_eval_add_fixed_increment: null argument");
        if (!(refRho > 0 && refP > 0))
            return fail(DNDSB_E_BADARG, "dndsb_eval_add_fixed_increment: refRho and refP must be positive");
        return status_msg(add_fixed_increment(e->vr->mesh->d, e->e, u, inc, alpha, refRho, refP, ppEpsIsRelaxed, alphaFixMinHost, S(stream)),
                          "dndsb_eval_add_fixed_increment");
    }

    int dndsb_eval_pressure_force_coords(dndsb_eval *e, int zone, const double *dir, const double *u, const double *uRec, double *dJdX,
                                         void *stream)
    {
        if (!e || !dir || !u || !uRec || !dJdX)
            return fail(DNDSB_E_BADARG, "dndsb_eval_pressure_force_coords: null argument");
        if (!e->vr->coeff)
            return fail(DNDSB_E_BADARG, "dndsb_eval_pressure_force_coords: VR not constructed");
        if (e->e.s.nVars != 5)
            return fail(DNDSB_E_BADARG, "dndsb_eval_pressure_force_coords: needs nVars = 5");
        dndsb_vr *v = e->vr;
        int rc = pressure_force_coords(v->mesh->d, v->g, v->vr, e->e.s.gamma, zone, dir, u, uRec, v->coordWs, dJdX, S(stream));
        if (rc == ST_UNSUPPORTED)
            return fail(DNDSB_E_BADARG, "dndsb_eval_pressure_force_coords: VR degree 1-2 in 3-D, 1-3 in 2-D");
        return status_msg(rc, "dndsb_eval_pressure_force_coords");
    }

    int dndsb_eval_pressure_force(dndsb_eval *e, int zone, const double *dir, const double *u, const double *uRec, double *Jhost, double *dJdu,
                                  double *dJduRec, void *stream)
    {
        if (!e || !dir || !u || !uRec || !Jhost)
            return fail(DNDSB_E_BADARG, "dndsb_eval_pressure_force: null argument");
        return status_msg(pressure_force(e->vr->mesh->d, e->vr->g, e->vr->vr, e->e, zone, dir, u, uRec, Jhost, dJdu, dJduRec, S(stream)),
                          "dndsb_eval_pressure_force");
    }

    int dndsb_eval_solve_linear(dndsb_eval *e, const dndsb_linear_settings *ls, double alphaDiag, const double *dTau, double dt,
                                const double *u, const double *rhs, double *xInc, void *stream)
    {
        if (!e || !ls || !dTau || !u || !rhs || !xInc)
            return fail(DNDSB_E_BADARG, "dndsb_eval_solve_linear: null argument");
        LinSettings s;
        s.gmresCode = ls->gmresCode, s.jacobiCode = ls->jacobiCode, s.sgsIter = ls->sgsIter;
        s.nGmresSpace = ls->nGmresSpace, s.nGmresIter = ls->nGmresIter, s.precision = ls->precision, s.useGraph = ls->useGraph;
        for (int v = 0; v < 8; v++)
        {
            double ms = ls->meanScale[v] > 0 ? ls->meanScale[v] : 1.0;
            double inv = 1.0 / (ms + 1e-200);
            s.scale2[v] = inv * inv;
        }
        int rc = linear_solve(e->vr->mesh->d, e->vr->g, e->vr->vr.bnd, e->e, e->lin, s, alphaDiag, dTau, dt, u, rhs, xInc, S(stream));
        if (rc == ST_BADARG)
            return fail(DNDSB_E_BADARG, "dndsb_eval_solve_linear: gmresCode 0..2, jacobiCode 0..2, nGmresSpace 1..32, precision 0..1");
        return status_msg(rc, "dndsb_eval_solve_linear");
    }

    int64_t dndsb_krylov_ld(int64_t n) { return krylov_ld(n); }
    size_t dndsb_krylov_work_bytes(void) { return krylov_work_bytes(); }

    int dndsb_krylov_start(int precision, int64_t n, int k, const void *r, void *V, double *gsc, double *colScale, void *work, void *stream)
    {
        if (!r || !V || !gsc || !colScale || !work)
            return fail(DNDSB_E_BADARG, "dndsb_krylov_start: null argument");
        int rc = krylov_start(precision, n, k, r, V, gsc, colScale, work, S(stream));
        if (rc == ST_BADARG)
            return fail(DNDSB_E_BADARG, "dndsb_krylov_start: n > 0, 1 <= k <= 32, precision 0..1");
        return status_msg(rc, "dndsb_krylov_start");
    }

    int dndsb_krylov_arnoldi(int precision, int64_t n, int j, int k, void *V, double *H, double *colScale, double *gsc, double *res, void *work,
                             void *stream)
    {
        if (!V || !H || !colScale || !gsc || !work)
            return fail(DNDSB_E_BADARG, "dndsb_krylov_arnoldi: null argument");
        int rc = krylov_arnoldi(precision, n, j, k, V, H, colScale, gsc, res, work, S(stream));
        if (rc == ST_BADARG)
            return fail(DNDSB_E_BADARG, "dndsb_krylov_arnoldi: n > 0, 1 <= k <= 32, 0 <= j < k, precision 0..1");
        return status_msg(rc, "dndsb_krylov_arnoldi");
    }

    int dndsb_krylov_update(int precision, int64_t n, int k, const void *V, const double *gsc, const double *colScale, void *x, void *stream)
    {
        if (!V || !gsc || !colScale || !x)
            return fail(DNDSB_E_BADARG, "dndsb_krylov_update: null argument");
        int rc = krylov_update(precision, n, k, V, gsc, colScale, x, S(stream));
        if (rc == ST_BADARG)
            return fail(DNDSB_E_BADARG, "dndsb_krylov_update: n > 0, 1 <= k <= 32, precision 0..1");
        return status_msg(rc, "dndsb_krylov_update");
    }

    int dndsb_eval_evaluate_norm(dndsb_eval *e, const double *x, int P, int volWise, double *resHost, void *stream)
    {
        if (!e || !x || !resHost || P < 1)
            return fail(DNDSB_E_BADARG, "dndsb_eval_evaluate_norm: bad argument");
        const MeshD &m = e->vr->mesh->d;
        int nv = e->e.s.nVars;
        int rc;
        if (P < 3)
        {
            rc = reduce_norm(m.nCell, nv, x, volWise ? e->vr->g.vol : nullptr, 0, P, e->e.redBuf, resHost, S(stream));
            if (rc == ST_OK)
                for (int v = 0; v < nv; v++)
                    resHost[v] = P == 1 ? resHost[v] : std::sqrt(resHost[v]);
        }
        else
            rc = reduce_norm(m.nCell, nv, x, nullptr, 2, 1, e->e.redBuf, resHost, S(stream));
        return status_msg(rc, "dndsb_eval_evaluate_norm");
    }

    int dndsb_eval_get_array(const dndsb_eval *e, const char *name, double *hostOut, int64_t cap, int64_t *len)
    {
        if (!e || !name)
            return fail(DNDSB_E_BADARG, "dndsb_eval_get_array: null");
        const MeshD &m = e->vr->mesh->d;
        std::string n(name);
        const double *src = nullptr;
        int64_t cnt = 0;
        if (n == "lambdaFace") src = e->e.lambdaFace, cnt = m.nFace;
        else if (n == "lambdaFaceC") src = e->e.lambdaFaceC, cnt = m.nFace;
        else if (n == "lambdaFaceVis") src = e->e.lambdaFaceVis, cnt = m.nFace;
        else if (n == "deltaLambdaCell") src = e->e.deltaLambdaCell, cnt = m.nCell;
        else if (n == "faceFlux") src = e->e.faceFlux, cnt = m.nFace * e->e.s.nVars;
        else if (n == "jSource" && e->e.jSource) src = e->e.jSource, cnt = m.nCell * e->e.s.nVars;
        else if (n == "fluxWallSum") src = e->e.fluxWall, cnt = e->e.s.nVars;
        else if (n == "lambdaFace0" && e->e.lambdaFace0) src = e->e.lambdaFace0, cnt = m.nFace;
        else if (n == "lambdaFace123" && e->e.lambdaFace0) src = e->e.lambdaFace123, cnt = m.nFace;
        else if (n == "lambdaFace4" && e->e.lambdaFace0) src = e->e.lambdaFace4, cnt = m.nFace;
        else
            return fail(DNDSB_E_BADARG, "dndsb_eval_get_array: unknown name " + n);
        if (len)
            *len = cnt;
        if (hostOut)
        {
            if (cap < cnt)
                return fail(DNDSB_E_BADARG, "dndsb_eval_get_array: buffer too small");
            if (cudaMemcpy(hostOut, src, sizeof(double) * cnt, cudaMemcpyDeviceToHost) != cudaSuccess)
                return cuda_fail("dndsb_eval_get_array");
        }
        return DNDSB_OK;
    }

    int dndsb_eval_set_delta_lambda(dndsb_eval *e, const double *dl, void *stream)
    {
        if (!e || !dl)
            return fail(DNDSB_E_BADARG, "dndsb_eval_set_delta_lambda: null");
        if (cudaMemcpyAsync(e->e.deltaLambdaCell, dl, sizeof(double) * e->vr->mesh->d.nCell, cudaMemcpyDeviceToDevice, S(stream)) !=
            cudaSuccess)
            return cuda_fail("dndsb_eval_set_delta_lambda");
        return DNDSB_OK;
    }
}
