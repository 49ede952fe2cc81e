// Evaluation of the VR basis of one cell at a physical point.
// VariationalReconstruction.hpp:319-368 FDiffBaseValue (localOrientation = false):
// offsets from the cell centre (first-order quadrature point) are scaled by
// the cell's axis-aligned half box (isotropic: its largest component), and
// row 0 has the cell-mean moment removed so every basis has zero mean.
#pragma once
#include "core.cuh"

namespace dndsb
{
template <int DIM>
DNDSB_HD void cell_lengths(const real *hbox, bool aniso, real L[3])
{
    L[0] = hbox[0], L[1] = hbox[1], L[2] = hbox[2];
    if (!aniso)
    {
        if (DIM == 2)
            L[0] = L[1] = dmax(L[0], L[1]);
        else
            L[0] = L[1] = L[2] = dmax(dmax(L[0], L[1]), L[2]);
    }
}

// T[rows][NDOF]; row 0 minus the moments when `moment` is not null
template <int DIM, int NDOF>
DNDSB_HD void cell_basis(const real *cent, const real *hbox, const real *moment, bool aniso, const real *p, int rows, real *T)
{
    real L[3];
    cell_lengths<DIM>(hbox, aniso, L);
    real x = (p[0] - cent[0]) / L[0], y = (p[1] - cent[1]) / L[1], z = DIM == 3 ? (p[2] - cent[2]) / L[2] : 0.0;
    basis_table<DIM, NDOF>(T, rows, x, y, z, L);
    if (moment)
        for (int k = 0; k < NDOF; k++)
            T[k] -= moment[k];
}

template <int DIM>
constexpr int ndof_of(int P)
{
    return DIM == 2 ? (P == 0 ? 1 : P == 1 ? 3 : P == 2 ? 6 : 10) : (P == 0 ? 1 : P == 1 ? 4 : P == 2 ? 10 : 20);
}
} // namespace dndsb
