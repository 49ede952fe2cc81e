// Evaluation of the VR basis of one cell at a physical point.
// VariationalReconstruction.hpp:319-368 FDiffBaseValue (localOrientation = false):
// offsets from the cell centre (first-order quadrature point) are scaled by
// the cell's axis-aligned half box (isotropic: its largest component), and
// row 0 has the cell-mean moment removed so every basis has zero mean.
#pragma once
#include "core.cuh"

namespace dndsb
{
template <int DIM, typename S>
DNDSB_HD void cell_lengths(const S *hbox, bool aniso, S L[3])
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

template <typename S>
struct NoDeduce
{
    using type = S;
};

// T[rows][NDOF]; row 0 minus the moments when `moment` is not null.  S is real, or dual numbers
// for derivatives with respect to the node coordinates.
template <int DIM, int NDOF, typename S>
DNDSB_HD void cell_basis(const S *cent, const S *hbox, const typename NoDeduce<S>::type *moment, bool aniso, const S *p, int rows, S *T)
{
    S L[3];
    cell_lengths<DIM>(hbox, aniso, L);
    S x = (p[0] - cent[0]) / L[0], y = (p[1] - cent[1]) / L[1], z = 0.0;
    if (DIM == 3)
        z = (p[2] - cent[2]) / L[2];
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

// Gauss-Jordan inverse with partial pivoting; false if singular
template <int N>
DNDSB_HD bool invert_gj(real *A, real *Ai)
{
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++)
            Ai[i * N + j] = i == j ? 1.0 : 0.0;
    for (int c = 0; c < N; c++)
    {
        int piv = c;
        for (int r = c + 1; r < N; r++)
            if (fabs(A[r * N + c]) > fabs(A[piv * N + c]))
                piv = r;
        if (A[piv * N + c] == 0)
            return false;
        if (piv != c)
            for (int j = 0; j < N; j++)
            {
                real t = A[piv * N + j];
                A[piv * N + j] = A[c * N + j], A[c * N + j] = t;
                t = Ai[piv * N + j];
                Ai[piv * N + j] = Ai[c * N + j], Ai[c * N + j] = t;
            }
        real id = 1.0 / A[c * N + c];
        for (int j = 0; j < N; j++)
            A[c * N + j] *= id, Ai[c * N + j] *= id;
        for (int r = 0; r < N; r++)
            if (r != c)
            {
                real fct = A[r * N + c];
                if (fct != 0)
                    for (int j = 0; j < N; j++)
                        A[r * N + j] -= fct * A[c * N + j], Ai[r * N + j] -= fct * Ai[c * N + j];
            }
    }
    return true;
}
} // namespace dndsb
