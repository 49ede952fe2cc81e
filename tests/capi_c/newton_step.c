/* A plain C host program against include/dndsb.h: the reference's one-Newton-step sequence
 * (test/cpp/Euler/test_EulerEvaluator.cpp:120-226) written the way a C or C++ caller of the
 * library would write it.  The mesh comes from a binary file (written by the test that builds
 * and runs this program); the program prints the volume-weighted L1 norm of the density
 * residual and the L2 norm of the increment, and writes the residual to a file.
 *
 * usage: newton_step <mesh.bin> <rhs.out> <riemann code> <rsMeanValueEig> <CFL> <maxOrder> <intOrder>
 *                    <dirWeightScheme> <geomWeightScheme> <init: 2 = vortex chi 10.0828, 0 = state file> [u.bin]
 */
#include <cuda_runtime_api.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "../../include/dndsb.h"

#define CK(x)                                                                          \
    do                                                                                 \
    {                                                                                  \
        int rc_ = (x);                                                                 \
        if (rc_ != DNDSB_OK)                                                           \
        {                                                                              \
            fprintf(stderr, "%s failed: %d %s\n", #x, rc_, dndsb_last_error());        \
            return 1;                                                                  \
        }                                                                              \
    } while (0)

static void *read_block(FILE *f, size_t bytes)
{
    void *p = malloc(bytes ? bytes : 1);
    if (bytes && fread(p, 1, bytes, f) != bytes)
    {
        free(p);
        return NULL;
    }
    return p;
}

int main(int argc, char **argv)
{
    if (argc < 11)
    {
        fprintf(stderr, "usage: %s mesh.bin rhs.out rs mve CFL maxOrder intOrder dirW geomW init [u.bin]\n", argv[0]);
        return 2;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f)
        return 2;
    int64_t hdr[10]; /* dim, cellType, faceType, nNode, nCell, nvert, nFace, nfv, nf, unused */
    if (fread(hdr, sizeof(int64_t), 10, f) != 10)
        return 2;
    int dim = (int)hdr[0], cellType = (int)hdr[1], faceType = (int)hdr[2], nvert = (int)hdr[5], nfv = (int)hdr[7], nf = (int)hdr[8];
    int64_t nNode = hdr[3], nCell = hdr[4], nFace = hdr[6];
    double *coords = read_block(f, sizeof(double) * nNode * 3);
    int64_t *c2n = read_block(f, sizeof(int64_t) * nCell * nvert);
    double *cshift = read_block(f, sizeof(double) * nCell * nvert * 3);
    int64_t *f2n = read_block(f, sizeof(int64_t) * nFace * nfv);
    double *fshift = read_block(f, sizeof(double) * nFace * nfv * 3);
    int64_t *f2c = read_block(f, sizeof(int64_t) * nFace * 2);
    int32_t *fzone = read_block(f, sizeof(int32_t) * nFace);
    double *fpshift = read_block(f, sizeof(double) * nFace * 3);
    int64_t *c2f = read_block(f, sizeof(int64_t) * nCell * nf);
    fclose(f);
    if (!coords || !c2n || !cshift || !f2n || !fshift || !f2c || !fzone || !fpshift || !c2f)
        return 2;

    dndsb_mesh *mesh = NULL;
    CK(dndsb_mesh_create(&mesh, dim, cellType, faceType, nNode, coords, nCell, nvert, c2n, cshift, nFace, nfv, f2n, fshift, f2c, fzone,
                         fpshift, nf, c2f));
    dndsb_vr_settings vs = {0};
    vs.maxOrder = atoi(argv[6]), vs.intOrder = atoi(argv[7]), vs.jacobiRelax = 1.0, vs.scaleType = 1, vs.scaleMultiplier = 1.0;
    vs.dirWeightScheme = atoi(argv[8]), vs.geomWeightScheme = atoi(argv[9]), vs.geomWeightBias = vs.geomWeightScheme ? 1.0 : 0.0;
    vs.geomWeightPower = 0.5, vs.bcWeight = 1.0;
    vs.manualDirWeights[0] = 1, vs.manualDirWeights[1] = 1, vs.manualDirWeights[2] = 0.5, vs.manualDirWeights[3] = 1.0 / 6;
    dndsb_vr *vr = NULL;
    CK(dndsb_vr_create(&vr, mesh, &vs));
    CK(dndsb_vr_construct_metrics(vr));
    CK(dndsb_vr_construct_base_and_weight(vr, NULL, 0));
    CK(dndsb_vr_construct_rec_coeff(vr));
    int64_t sz[4];
    CK(dndsb_vr_sizes(vr, sz));
    int64_t R = sz[1];

    dndsb_euler_settings es = {0};
    es.nVars = 5, es.rsType = atoi(argv[3]), es.rsMeanValueEig = atoi(argv[4]), es.rsFixScale = 1, es.rsIncFScale = 1;
    es.gamma = 1.4, es.Rgas = 289.0, es.muGas = 1e-200, es.prGas = 0.72, es.TRef = 273.15, es.CSutherland = 110.4, es.muModel = 1;
    dndsb_eval *ev = NULL;
    CK(dndsb_eval_create(&ev, vr, &es));

    size_t nu = sizeof(double) * nCell * 5;
    double *u, *uRec, *rhs, *dTau, *jd, *xinc, *xincNew;
    if (cudaMalloc((void **)&u, nu) || cudaMalloc((void **)&uRec, nu * R) || cudaMalloc((void **)&rhs, nu) ||
        cudaMalloc((void **)&dTau, sizeof(double) * nCell) || cudaMalloc((void **)&jd, sizeof(double) * nCell) ||
        cudaMalloc((void **)&xinc, nu) || cudaMalloc((void **)&xincNew, nu))
        return 3;
    cudaMemset(uRec, 0, nu * R);
    cudaMemset(xinc, 0, nu);
    cudaMemset(xincNew, 0, nu);
    if (atoi(argv[10]) == 2)
        CK(dndsb_eval_initialize_udof(ev, 2, 10.0828, u, NULL));
    else
    {
        FILE *fu = fopen(argv[11], "rb");
        double *uh = fu ? read_block(fu, nu) : NULL;
        if (!uh)
            return 2;
        fclose(fu);
        cudaMemcpy(u, uh, nu, cudaMemcpyHostToDevice);
        free(uh);
    }
    CK(dndsb_eval_fix_umax_filter(ev, u, NULL));
    double dtMin = 0;
    CK(dndsb_eval_evaluate_dt(ev, u, atof(argv[5]), 1e100, 1, dTau, &dtMin, NULL));
    CK(dndsb_eval_evaluate_rhs(ev, rhs, u, uRec, NULL));
    double l1[5], l2[5];
    CK(dndsb_eval_evaluate_norm(ev, rhs, 1, 1, l1, NULL));
    CK(dndsb_eval_lusgs_matrix_init(ev, dTau, 1e100, 1.0, jd, NULL));
    CK(dndsb_eval_update_lusgs_forward(ev, 1.0, rhs, u, xinc, jd, xincNew, NULL));
    CK(dndsb_eval_update_lusgs_backward(ev, 1.0, rhs, u, xinc, jd, xincNew, NULL));
    CK(dndsb_eval_evaluate_norm(ev, xincNew, 2, 0, l2, NULL));
    double inc = 0;
    for (int v = 0; v < 5; v++)
        inc += l2[v] * l2[v];
    printf("rhsDensityL1 %.12e incL2 %.12e\n", l1[0], sqrt(inc));

    double *h = malloc(nu);
    cudaMemcpy(h, rhs, nu, cudaMemcpyDeviceToHost);
    FILE *fo = fopen(argv[2], "wb");
    if (!fo || fwrite(h, 1, nu, fo) != nu)
        return 4;
    fclose(fo);
    free(h);
    cudaFree(u), cudaFree(uRec), cudaFree(rhs), cudaFree(dTau), cudaFree(jd), cudaFree(xinc), cudaFree(xincNew);
    CK(dndsb_eval_destroy(ev));
    CK(dndsb_vr_destroy(vr));
    CK(dndsb_mesh_destroy(mesh));
    free(coords), free(c2n), free(cshift), free(f2n), free(fshift), free(f2c), free(fzone), free(fpshift), free(c2f);
    return 0;
}
