// Transposed flux-increment Jacobian shared by the adjoint kernels.
#pragma once
#include "solver.cuh"

namespace dndsb
{
// out = (J(U; n) - lambda I)^T y, J(U; n) the Jacobian of the physical flux through n (Gas.hpp:390-397,
// increment form Gas.hpp:462-513): the reverse sweep of the flux-increment statements
template <int NV>
DNDSB_D void flux_jac_du_t(const real *U, const real *n, const real *y, real lam, real gamma, real *out)
{
    real ir = 1.0 / U[0];
    real v[3] = {U[1] * ir, U[2] * ir, U[3] * ir};
    real p, a2, H;
    gas_thermal(U[4], U[0], dot3(v, v), gamma, p, a2, H);
    real vn = dot3(v, n);
    for (int j = 0; j < NV; j++)
        out[j] = -lam * y[j] + (j >= 1 ? vn * y[j] : 0.0);
    real bvn = 0, bp = 0;
    for (int d = 0; d < 3; d++)
    {
        out[1 + d] += n[d] * y[0];
        bvn += U[1 + d] * y[1 + d];
        bp += n[d] * y[1 + d];
    }
    bp += vn * y[4];
    bvn += (U[4] + p) * y[4];
    for (int j = 5; j < NV; j++)
        bvn += U[j] * y[j];
    out[4] += (gamma - 1) * bp;
    for (int d = 0; d < 3; d++)
    {
        real bv = n[d] * bvn - 0.5 * (gamma - 1) * U[1 + d] * bp;
        out[1 + d] += -0.5 * (gamma - 1) * v[d] * bp + ir * bv;
        out[0] += -U[1 + d] * ir * ir * bv;
    }
}

} // namespace dndsb
