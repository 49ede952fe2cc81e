// Block ILU(0) of the implicit operator: JacobianLocalLU's InPlaceDecompose and Solve (Solver/Direct.hpp:312-405,
// 487-540) for iluCode 0 (the face-neighbour pattern, no fill), run colour by colour.  A row's lower neighbours
// are those of lower rank (rank = position in colour order, or the colour); cells of one colour are never
// adjacent, so every row of a colour depends only on rows of earlier colours and a colour is factored (or
// solved) in one launch.  On a mesh numbered colour by colour this is the reference's natural-order
// factorisation.
//
// Storage: off holds per row r and slot k the block of A (then L for lower and U for upper neighbours), dinv the
// inverted pivots, D the diagonal blocks of A.  BlockLay places element e of row r (E elements per row) in tiles
// of 2^s rows: rows of a tile innermost, so that the 32 threads of a warp read one element of 32 consecutive rows
// as one contiguous 256-byte line and a warp's rows share one contiguous range; s = 0 is rows outermost
// ([row][E]).  nbr [r][NF] holds the neighbour row of each slot (-1: none).
#pragma once
#include "roejac.cuh"

namespace dndsb
{
namespace ilu
{
struct BlockLay
{
    int64_t E; // elements per row
    int s;     // log2 of the rows per tile
    DNDSB_HD int64_t at(int64_t r, int64_t e) const { return ((((r >> s) * E) + e) << s) + (r & ((int64_t(1) << s) - 1)); }
};
// rows allocated for a tiled layout of n rows
inline int64_t padded_rows(int64_t n, int s) { return ((n + (int64_t(1) << s) - 1) >> s) << s; }

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

// the block of elements e0 .. e0 + NV NV - 1 of row r
template <typename T, int NV>
DNDSB_HD void load(const T *src, BlockLay L, int64_t r, int e0, real *dst)
{
    for (int i = 0; i < NV * NV; i++)
        dst[i] = (real)src[L.at(r, e0 + i)];
}
template <typename T, int NV>
DNDSB_HD void store(const real *v, T *dst, BlockLay L, int64_t r, int e0)
{
    for (int i = 0; i < NV * NV; i++)
        dst[L.at(r, e0 + i)] = (T)v[i];
}

// one row of the factorisation: A (the operator's slot blocks) and D (diagonal blocks) in, off / dinv out.
// cnbr (may be nullptr): compact slot order for the factors — slot j < cnlow[r] holds the j-th lower neighbour in
// ascending rank, the upper neighbours follow, cnbr [r][NF] their rows (-1 after the last); the triangular solves
// then read the lower (or upper) blocks of a row from consecutive slots, so the threads of a warp load the same
// slots.  Without it the factors keep the operator's slot order.
template <typename T, int NV, int NF>
DNDSB_HD bool factor_row(int64_t r, const int32_t *nbr, const int32_t *rank, const T *A, const T *D, BlockLay offL, BlockLay dL, BlockLay DL,
                         T *off, T *dinv, int32_t *cnbr = nullptr, int32_t *cnlow = nullptr)
{
    constexpr int NN = NV * NV;
    const int32_t *fnbr = cnbr ? cnbr : nbr; // the slot lists of the factored rows
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
        load<T, NV>(A, offL, r, low[a] * NN, Lij);
        for (int b = 0; b < a; b++)
        {
            int64_t k = nbr[r * NF + low[b]];
            int s = slot_of<NF>(fnbr, k, j);
            if (s >= 0)
            {
                real Ukj[NN];
                load<T, NV>(off, offL, k, s * NN, Ukj);
                mul_sub<NV>(L + b * NN, Ukj, Lij);
            }
        }
        real Dj[NN], t[NN];
        load<T, NV>(dinv, dL, j, 0, Dj);
        for (int i = 0; i < NN; i++)
            t[i] = 0;
        mul_sub<NV>(Lij, Dj, t);
        for (int i = 0; i < NN; i++)
            Lij[i] = -t[i];
    }
    real Di[NN], Dinv[NN];
    load<T, NV>(D, DL, r, 0, Di);
    for (int b = 0; b < nLow; b++)
    {
        int64_t k = nbr[r * NF + low[b]];
        int s = slot_of<NF>(fnbr, k, r);
        if (s >= 0)
        {
            real Uki[NN];
            load<T, NV>(off, offL, k, s * NN, Uki);
            mul_sub<NV>(L + b * NN, Uki, Di);
        }
    }
    bool ok = roej::block_inv<NV>(Di, Dinv);
    if (!ok)
        for (int i = 0; i < NN; i++)
            Dinv[i] = 0;
    store<T, NV>(Dinv, dinv, dL, r, 0);
    for (int a = 0; a < nUpp; a++)
    {
        int64_t j = nbr[r * NF + upp[a]];
        real Uij[NN];
        load<T, NV>(A, offL, r, upp[a] * NN, Uij);
        for (int b = 0; b < nLow; b++)
        {
            int64_t k = nbr[r * NF + low[b]];
            int s = slot_of<NF>(fnbr, k, j);
            if (s >= 0)
            {
                real Ukj[NN];
                load<T, NV>(off, offL, k, s * NN, Ukj);
                mul_sub<NV>(L + b * NN, Ukj, Uij);
            }
        }
        store<T, NV>(Uij, off, offL, r, (cnbr ? nLow + a : upp[a]) * NN);
    }
    for (int a = 0; a < nLow; a++)
        store<T, NV>(L + a * NN, off, offL, r, (cnbr ? a : low[a]) * NN);
    real zero[NN];
    for (int i = 0; i < NN; i++)
        zero[i] = 0;
    if (cnbr)
    {
        for (int j = 0; j < NF; j++)
            cnbr[r * NF + j] = j < nLow ? nbr[r * NF + low[j]] : (j < nLow + nUpp ? nbr[r * NF + upp[j - nLow]] : -1);
        cnlow[r] = nLow;
        for (int j = nLow + nUpp; j < NF; j++)
            store<T, NV>(zero, off, offL, r, j * NN);
        return ok;
    }
    // slots without a neighbour (boundary faces) and a row's periodic image of itself carry nothing
    for (int k = 0; k < NF; k++)
    {
        int64_t q = nbr[r * NF + k];
        if (q < 0 || q == r)
            store<T, NV>(zero, off, offL, r, k * NN);
    }
    return ok;
}

// rows: the rows of one colour (nullptr: the contiguous range [beg, end))
template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_ilu_factor(int64_t beg, int64_t end, const int32_t *__restrict__ rows, const int32_t *__restrict__ nbr,
                               const int32_t *__restrict__ rank, const T *A, const T *__restrict__ D, BlockLay offL, BlockLay dL, BlockLay DL,
                               T *off, T *dinv, int *err, int32_t *cnbr, int32_t *cnlow) // A may be off (factored in place)
{
    DNDSB_KERNEL_LOOP(ii, end - beg)
    {
        int64_t r = rows ? (int64_t)rows[beg + ii] : beg + ii;
        if (!factor_row<T, NV, NF>(r, nbr, rank, A, D, offL, dL, DL, off, dinv, cnbr, cnlow))
            atomicOr(err, (int)DE_SINGULAR);
    }
}

// the triangular solves on compact factors (cnbr / cnlow of factor_row), rows [beg, end) of one colour:
// forward y_r = b_r - sum_{j < nLow} L_j y_q; backward x_r = dinv_r (y_r - sum_{j >= nLow} U_j x_q), in place
template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_ilu_lower_c(int64_t beg, int64_t end, const int32_t *__restrict__ cnbr, const int32_t *__restrict__ cnlow,
                                const T *__restrict__ off, BlockLay offL, const T *b, T *x) // b may be x
{
    constexpr int NN = NV * NV;
    DNDSB_KERNEL_LOOP(ii, end - beg)
    {
        int64_t r = beg + ii;
        T acc[NV];
        for (int v = 0; v < NV; v++)
            acc[v] = b[r * NV + v];
        const int nl = cnlow[r];
#pragma unroll
        for (int j = 0; j < NF; j++)
        {
            if (j >= nl)
                break;
            int64_t q = cnbr[r * NF + j];
            T xq[NV];
            for (int l = 0; l < NV; l++)
                xq[l] = x[q * NV + l];
            for (int i = 0; i < NV; i++)
            {
                T s = 0;
                for (int l = 0; l < NV; l++)
                    s += off[offL.at(r, j * NN + i * NV + l)] * xq[l];
                acc[i] -= s;
            }
        }
        for (int v = 0; v < NV; v++)
            x[r * NV + v] = acc[v];
    }
}

template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_ilu_upper_c(int64_t beg, int64_t end, const int32_t *__restrict__ cnbr, const int32_t *__restrict__ cnlow,
                                const T *__restrict__ off, BlockLay offL, const T *__restrict__ dinv, BlockLay dL, T *x)
{
    constexpr int NN = NV * NV;
    DNDSB_KERNEL_LOOP(ii, end - beg)
    {
        int64_t r = beg + ii;
        T acc[NV];
        for (int v = 0; v < NV; v++)
            acc[v] = x[r * NV + v];
        const int nl = cnlow[r];
#pragma unroll
        for (int j = 0; j < NF; j++)
        {
            if (j < nl)
                continue;
            int64_t q = cnbr[r * NF + j];
            if (q < 0)
                break;
            T xq[NV];
            for (int l = 0; l < NV; l++)
                xq[l] = x[q * NV + l];
            for (int i = 0; i < NV; i++)
            {
                T s = 0;
                for (int l = 0; l < NV; l++)
                    s += off[offL.at(r, j * NN + i * NV + l)] * xq[l];
                acc[i] -= s;
            }
        }
        for (int i = 0; i < NV; i++)
        {
            T s = 0;
            for (int l = 0; l < NV; l++)
                s += dinv[dL.at(r, i * NV + l)] * acc[l];
            x[r * NV + i] = s;
        }
    }
}

// forward: y_r = b_r - sum over lower slots of L y_q;  backward: x_r = dinv_r (y_r - sum over upper slots of U x_q),
// in place on x (= y)
template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_ilu_lower(int64_t beg, int64_t end, const int32_t *__restrict__ rows, const int32_t *__restrict__ nbr,
                              const int32_t *__restrict__ rank, const T *__restrict__ off, BlockLay offL, const T *b, T *x) // b may be x
{
    constexpr int NN = NV * NV;
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
            T xq[NV];
            for (int l = 0; l < NV; l++)
                xq[l] = x[q * NV + l];
            for (int i = 0; i < NV; i++)
            {
                T s = 0;
                for (int l = 0; l < NV; l++)
                    s += off[offL.at(r, k * NN + i * NV + l)] * xq[l];
                acc[i] -= s;
            }
        }
        for (int v = 0; v < NV; v++)
            x[r * NV + v] = acc[v];
    }
}

template <typename T, int NV, int NF>
DNDSB_GLOBAL void k_ilu_upper(int64_t beg, int64_t end, const int32_t *__restrict__ rows, const int32_t *__restrict__ nbr,
                              const int32_t *__restrict__ rank, const T *__restrict__ off, BlockLay offL, const T *__restrict__ dinv, BlockLay dL,
                              T *x)
{
    constexpr int NN = NV * NV;
    DNDSB_KERNEL_LOOP(ii, end - beg)
    {
        int64_t r = rows ? (int64_t)rows[beg + ii] : beg + ii;
        int64_t rr = rank ? (int64_t)rank[r] : r;
        T acc[NV];
        for (int v = 0; v < NV; v++)
            acc[v] = x[r * NV + v];
#pragma unroll
        for (int k = 0; k < NF; k++)
        {
            int64_t q = nbr[r * NF + k];
            if (q < 0 || q == r || (rank ? (int64_t)rank[q] : q) <= rr)
                continue;
            T xq[NV];
            for (int l = 0; l < NV; l++)
                xq[l] = x[q * NV + l];
            for (int i = 0; i < NV; i++)
            {
                T s = 0;
                for (int l = 0; l < NV; l++)
                    s += off[offL.at(r, k * NN + i * NV + l)] * xq[l];
                acc[i] -= s;
            }
        }
        for (int i = 0; i < NV; i++)
        {
            T s = 0;
            for (int l = 0; l < NV; l++)
                s += dinv[dL.at(r, i * NV + l)] * acc[l];
            x[r * NV + i] = s;
        }
    }
}
} // namespace ilu
} // namespace dndsb
