// Block ILU(0) of the implicit operator: JacobianLocalLU's InPlaceDecompose and Solve (Solver/Direct.hpp:312-405,
// 487-540) for iluCode 0 (the face-neighbour pattern, no fill), run colour by colour.  A row's lower neighbours
// are those of lower rank (rank = position in colour order, or the colour); cells of one colour are never
// adjacent, so every row of a colour depends only on rows of earlier colours and a colour is factored (or
// solved) in one launch.  On a mesh numbered colour by colour this is the reference's natural-order
// factorisation.
//
// Storage per row r: off [r][NF][NV][NV] (slot blocks of A, then L for lower and U for upper neighbours) and
// dinv [r][NV][NV] (the inverted pivots).  nbr [r][NF] holds the neighbour row of each slot (-1: none).
#pragma once
#include "roejac.cuh"

namespace dndsb
{
namespace ilu
{
template <int NV>
DNDSB_HD void mul_sub(const real *A, const real *B, real *C) // C -= A B (row-major NV x NV)
{
    for (int i = 0; i < NV; i++)
        for (int j = 0; j < NV; j++)
        {
            real acc = 0;
            for (int l = 0; l < NV; l++)
                acc += A[i * NV + l] * B[l * NV + j];
            C[i * NV + j] -= acc;
        }
}

template <int NF>
DNDSB_HD int slot_of(const int32_t *nbr, int64_t r, int64_t target)
{
    for (int s = 0; s < NF; s++)
        if (nbr[r * NF + s] == target)
            return s;
    return -1;
}

template <typename T, int NV>
DNDSB_HD void load(const T *src, real *dst)
{
    for (int i = 0; i < NV * NV; i++)
        dst[i] = (real)src[i];
}

// one row of the factorisation: A (the operator's slot blocks), D (the diagonal block), both of row r
template <typename T, int NV, int NF>
DNDSB_HD bool factor_row(int64_t r, const int32_t *nbr, const int32_t *rank, const T *A, const T *D, T *off, T *dinv)
{
    constexpr int NN = NV * NV;
    auto rk = [&](int64_t x) { return rank ? (int64_t)rank[x] : x; };
    const int64_t rr = rk(r);
    int low[NF], nLow = 0, upp[NF], nUpp = 0;
    for (int k = 0; k < NF; k++)
    {
        int64_t q = nbr[r * NF + k];
        if (q < 0 || q == r)
            continue;
        if (rk(q) < rr)
        {
            // insertion in ascending rank: the order of the reference's sorted lower row
            int a = nLow++;
            while (a > 0 && rk(nbr[r * NF + low[a - 1]]) > rk(q))
                low[a] = low[a - 1], a--;
            low[a] = k;
        }
        else
            upp[nUpp++] = k;
    }
    real L[NF * NN];
    for (int a = 0; a < nLow; a++)
    {
        int64_t j = nbr[r * NF + low[a]];
        real *Lij = L + a * NN;
        load<T, NV>(A + (r * NF + low[a]) * NN, Lij);
        for (int b = 0; b < a; b++)
        {
            int64_t k = nbr[r * NF + low[b]];
            int s = slot_of<NF>(nbr, k, j);
            if (s >= 0)
            {
                real Ukj[NN];
                load<T, NV>(off + (k * NF + s) * NN, Ukj);
                mul_sub<NV>(L + b * NN, Ukj, Lij);
            }
        }
        real Dj[NN], t[NN];
        load<T, NV>(dinv + j * NN, Dj);
        for (int i = 0; i < NN; i++)
            t[i] = 0;
        mul_sub<NV>(Lij, Dj, t);
        for (int i = 0; i < NN; i++)
            Lij[i] = -t[i];
    }
    real Di[NN], Dinv[NN];
    load<T, NV>(D, Di);
    for (int b = 0; b < nLow; b++)
    {
        int64_t k = nbr[r * NF + low[b]];
        int s = slot_of<NF>(nbr, k, r);
        if (s >= 0)
        {
            real Uki[NN];
            load<T, NV>(off + (k * NF + s) * NN, Uki);
            mul_sub<NV>(L + b * NN, Uki, Di);
        }
    }
    bool ok = roej::block_inv<NV>(Di, Dinv);
    for (int i = 0; i < NN; i++)
        dinv[r * NN + i] = ok ? (T)Dinv[i] : T(0);
    for (int a = 0; a < nUpp; a++)
    {
        int64_t j = nbr[r * NF + upp[a]];
        real Uij[NN];
        load<T, NV>(A + (r * NF + upp[a]) * NN, Uij);
        for (int b = 0; b < nLow; b++)
        {
            int64_t k = nbr[r * NF + low[b]];
            int s = slot_of<NF>(nbr, k, j);
            if (s >= 0)
            {
                real Ukj[NN];
                load<T, NV>(off + (k * NF + s) * NN, Ukj);
                mul_sub<NV>(L + b * NN, Ukj, Uij);
            }
        }
        for (int i = 0; i < NN; i++)
            off[(r * NF + upp[a]) * NN + i] = (T)Uij[i];
    }
    for (int a = 0; a < nLow; a++)
        for (int i = 0; i < NN; i++)
            off[(r * NF + low[a]) * NN + i] = (T)L[a * NN + i];
    // slots without a neighbour (boundary faces) and a row's periodic image of itself carry nothing
    for (int k = 0; k < NF; k++)
    {
        int64_t q = nbr[r * NF + k];
        if (q < 0 || q == r)
            for (int i = 0; i < NN; i++)
                off[(r * NF + k) * NN + i] = T(0);
    }
    return ok;
}

// rows: the rows of one colour (nullptr: the contiguous range [beg, end)); dStride: elements between diagonal blocks
template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_ilu_factor(int64_t beg, int64_t end, const int32_t *__restrict__ rows, const int32_t *__restrict__ nbr,
                               const int32_t *__restrict__ rank, const T *A, const T *__restrict__ D, int64_t dStride, T *off, T *dinv,
                               int *err) // A may be off (factored in place)
{
    DNDSB_KERNEL_LOOP(ii, end - beg)
    {
        int64_t r = rows ? (int64_t)rows[beg + ii] : beg + ii;
        if (!factor_row<T, NV, NF>(r, nbr, rank, A, D + r * dStride, off, dinv))
            atomicOr(err, (int)DE_SINGULAR);
    }
}

// forward: y_r = b_r - sum over lower slots of L y_q;  backward: x_r = dinv_r (y_r - sum over upper slots of U x_q),
// in place on x (= y)
template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_ilu_lower(int64_t beg, int64_t end, const int32_t *__restrict__ rows, const int32_t *__restrict__ nbr,
                              const int32_t *__restrict__ rank, const T *__restrict__ off, const T *b, T *x) // b may be x
{
    DNDSB_KERNEL_LOOP(ii, end - beg)
    {
        int64_t r = rows ? (int64_t)rows[beg + ii] : beg + ii;
        int64_t rr = rank ? (int64_t)rank[r] : r;
        T acc[NV];
        for (int v = 0; v < NV; v++)
            acc[v] = b[r * NV + v];
#pragma unroll
        for (int k = 0; k < NF; k++)
        {
            int64_t q = nbr[r * NF + k];
            if (q < 0 || q == r || (rank ? (int64_t)rank[q] : q) >= rr)
                continue;
            const T *L = off + (r * NF + k) * NV * NV;
            for (int i = 0; i < NV; i++)
            {
                T s = 0;
                for (int l = 0; l < NV; l++)
                    s += L[i * NV + l] * x[q * NV + l];
                acc[i] -= s;
            }
        }
        for (int v = 0; v < NV; v++)
            x[r * NV + v] = acc[v];
    }
}

template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_ilu_upper(int64_t beg, int64_t end, const int32_t *__restrict__ rows, const int32_t *__restrict__ nbr,
                              const int32_t *__restrict__ rank, const T *__restrict__ off, const T *__restrict__ dinv, T *x)
{
    DNDSB_KERNEL_LOOP(ii, end - beg)
    {
        int64_t r = rows ? (int64_t)rows[beg + ii] : beg + ii;
        int64_t rr = rank ? (int64_t)rank[r] : r;
        T acc[NV], y[NV];
        for (int v = 0; v < NV; v++)
            acc[v] = x[r * NV + v];
#pragma unroll
        for (int k = 0; k < NF; k++)
        {
            int64_t q = nbr[r * NF + k];
            if (q < 0 || q == r || (rank ? (int64_t)rank[q] : q) <= rr)
                continue;
            const T *U = off + (r * NF + k) * NV * NV;
            for (int i = 0; i < NV; i++)
            {
                T s = 0;
                for (int l = 0; l < NV; l++)
                    s += U[i * NV + l] * x[q * NV + l];
                acc[i] -= s;
            }
        }
        roej::block_mul<NV>(dinv + r * NV * NV, acc, y);
        for (int v = 0; v < NV; v++)
            x[r * NV + v] = y[v];
    }
}
} // namespace ilu
} // namespace dndsb
