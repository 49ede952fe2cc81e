// Deterministic column reductions (sum / min / max) over cell rows: a fixed
// partition into kRedBlocks chunks, a fixed shared-memory tree per chunk and
// a single-block final pass, so results do not depend on scheduling.
#include "solver.cuh"

namespace dndsb
{
namespace
{
constexpr int kRedBlock = 256;

// deterministic reductions: fixed block partition, fixed shared-memory tree

template <int OP /*0 sum, 1 min, 2 max*/>
DNDSB_D real red_op(real a, real b) { return OP == 0 ? a + b : OP == 1 ? dmin(a, b) : dmax(a, b); }

template <int OP>
DNDSB_GLOBAL void k_reduce_cols(int64_t n, int ncol, const real *__restrict__ x, const real *__restrict__ w, int powP, real *partial)
{
    // partial[block][col] over rows [chunk) ; x is [n][ncol], optional row weight w
    __shared__ real sh[kRedBlock];
    real init = OP == 0 ? 0.0 : OP == 1 ? kVeryLarge : -kVeryLarge;
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t b0 = blockIdx.x * chunk, b1 = b0 + chunk < n ? b0 + chunk : n;
    for (int col = 0; col < ncol; col++)
    {
        real a = init;
        for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x)
        {
            real xv = x[i * ncol + col];
            xv = powP == 1 ? fabs(xv) : powP == 2 ? xv * xv : xv;
            real val = xv * (w ? w[i] : 1.0);
            a = red_op<OP>(a, val);
        }
        sh[threadIdx.x] = a;
        __syncthreads();
        for (int st = blockDim.x / 2; st > 0; st >>= 1)
        {
            if (threadIdx.x < st)
                sh[threadIdx.x] = red_op<OP>(sh[threadIdx.x], sh[threadIdx.x + st]);
            __syncthreads();
        }
        if (threadIdx.x == 0)
            partial[blockIdx.x * ncol + col] = sh[0];
        __syncthreads();
    }
}

template <int OP>
DNDSB_GLOBAL void k_reduce_final(int nb, int ncol, const real *__restrict__ partial, real *out)
{
    __shared__ real sh[kRedBlock];
    real init = OP == 0 ? 0.0 : OP == 1 ? kVeryLarge : -kVeryLarge;
    for (int col = 0; col < ncol; col++)
    {
        real a = init;
        for (int i = threadIdx.x; i < nb; i += blockDim.x)
            a = red_op<OP>(a, partial[i * ncol + col]);
        sh[threadIdx.x] = a;
        __syncthreads();
        for (int st = blockDim.x / 2; st > 0; st >>= 1)
        {
            if (threadIdx.x < st)
                sh[threadIdx.x] = red_op<OP>(sh[threadIdx.x], sh[threadIdx.x + st]);
            __syncthreads();
        }
        if (threadIdx.x == 0)
            out[col] = sh[0];
        __syncthreads();
    }
}

} // namespace

real *reduce_cols(int op, int64_t n, int ncol, const real *x, const real *w, int powP, real *redBuf, cudaStream_t st)
{
    real *out = redBuf + kRedBlocks * 8;
    if (op == 0)
    {
        k_reduce_cols<0><<<kRedBlocks, kRedBlock, 0, st>>>(n, ncol, x, w, powP, redBuf);
        k_reduce_final<0><<<1, kRedBlock, 0, st>>>(kRedBlocks, ncol, redBuf, out);
    }
    else if (op == 1)
    {
        k_reduce_cols<1><<<kRedBlocks, kRedBlock, 0, st>>>(n, ncol, x, w, powP, redBuf);
        k_reduce_final<1><<<1, kRedBlock, 0, st>>>(kRedBlocks, ncol, redBuf, out);
    }
    else
    {
        k_reduce_cols<2><<<kRedBlocks, kRedBlock, 0, st>>>(n, ncol, x, w, powP, redBuf);
        k_reduce_final<2><<<1, kRedBlock, 0, st>>>(kRedBlocks, ncol, redBuf, out);
    }
    return out;
}
// ---------------------------------------------------------------------------
// Krylov reductions for the native GMRES (weighted dots, Gram-Schmidt).
// Vectors are flat [n] arrays of T whose element i carries the variable
// weight s2[i % NV]; sums accumulate in FP64 over the same fixed partition.
// ---------------------------------------------------------------------------
namespace
{
DNDSB_D void block_sum4(real (*sh)[kRedBlock], real a0, real a1, real a2, real a3)
{
    sh[0][threadIdx.x] = a0, sh[1][threadIdx.x] = a1, sh[2][threadIdx.x] = a2, sh[3][threadIdx.x] = a3;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1)
    {
        if (threadIdx.x < st)
            for (int q = 0; q < 4; q++)
                sh[q][threadIdx.x] += sh[q][threadIdx.x + st];
        __syncthreads();
    }
}

// Quads of 4 consecutive elements, loaded as one 16-byte (float) or two 16-byte (double) loads.
template <typename T>
struct Quad;
template <>
struct Quad<float>
{
    using raw = float4;
    static DNDSB_D raw load_raw(const float *p) { return *(const float4 *)p; }
    static DNDSB_D real dot(const raw &v, const real (&w)[4]) { return (real)v.x * w[0] + (real)v.y * w[1] + (real)v.z * w[2] + (real)v.w * w[3]; }
    static DNDSB_D void load(const float *p, real (&o)[4])
    {
        float4 v = *(const float4 *)p;
        o[0] = v.x, o[1] = v.y, o[2] = v.z, o[3] = v.w;
    }
    // stores x rounded to float and returns the stored values
    static DNDSB_D void store(float *p, const real (&x)[4], real (&r)[4])
    {
        float4 v = make_float4((float)x[0], (float)x[1], (float)x[2], (float)x[3]);
        *(float4 *)p = v;
        r[0] = v.x, r[1] = v.y, r[2] = v.z, r[3] = v.w;
    }
};
template <>
struct Quad<double>
{
    struct raw
    {
        double2 a, b;
    };
    static DNDSB_D raw load_raw(const double *p) { return raw{((const double2 *)p)[0], ((const double2 *)p)[1]}; }
    static DNDSB_D real dot(const raw &v, const real (&w)[4]) { return v.a.x * w[0] + v.a.y * w[1] + v.b.x * w[2] + v.b.y * w[3]; }
    static DNDSB_D void load(const double *p, real (&o)[4])
    {
        double2 a = ((const double2 *)p)[0], b = ((const double2 *)p)[1];
        o[0] = a.x, o[1] = a.y, o[2] = b.x, o[3] = b.y;
    }
    static DNDSB_D void store(double *p, const real (&x)[4], real (&r)[4])
    {
        ((double2 *)p)[0] = make_double2(x[0], x[1]);
        ((double2 *)p)[1] = make_double2(x[2], x[3]);
        r[0] = x[0], r[1] = x[1], r[2] = x[2], r[3] = x[3];
    }
};

// sum over the block in a fixed order: xor-shuffle tree inside each warp (lane 0's value is
// used), then the warps in index order by one thread; valid in thread 0 (and for column k in
// thread k of the multi-column form below)
DNDSB_D real warp_sum(real x)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

constexpr int kKG = 8; // columns per pass of the multi-dot

// Called by every block after it has written its partials [block][ncol]: the block that arrives last
// (a ticket on *cnt, which it resets for the next launch) sums them per column in a fixed order (lanes
// over a fixed stride of the blocks, then a fixed xor tree, lane 0's value), the order the separate
// final pass used, so the result does not depend on which block finishes last.  out[col] = the sum
// (its square root with takeSqrt) times colScale[col] (when given).  Returns true in that block
// (uniformly over its threads).
DNDSB_D bool last_block_final(int ncol, const real *partial, real *out, const real *colScale, int takeSqrt, unsigned *cnt)
{
    __shared__ unsigned ticket;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        ticket = atomicAdd(cnt, 1u);
    __syncthreads();
    if (ticket != gridDim.x - 1)
        return false;
    __threadfence();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int col = wid; col < ncol; col += nw)
    {
        real a = 0;
        for (int i = lane; i < (int)gridDim.x; i += 32)
            a += __ldcg(partial + (int64_t)i * ncol + col);
        a = warp_sum(a);
        if (lane == 0)
        {
            real r = takeSqrt ? sqrt(a) : a;
            out[col] = colScale ? r * colScale[col] : r;
        }
    }
    if (threadIdx.x == 0)
        *cnt = 0;
    __syncthreads();
    return true;
}

// partial[block][col] = sum_i V[col][i] w[i] s2[i % NV] over the block's chunk of quads.  Columns are
// ld apart (ld a multiple of 4, the pad beyond n zero); all columns of a pass share one read of w.
// out[col] = partial sums reduced by the last block, times colScale[col] (the basis columns are stored
// unnormalised; colScale holds their normalising factors)
template <typename T, int NV>
DNDSB_GLOBAL void __launch_bounds__(kRedBlock, 4) k_kmdot(int64_t n, int64_t ld, int ncol, const T *__restrict__ V, const T *__restrict__ w,
                                                       const real *__restrict__ s2, real *partial, real *out, const real *colScale,
                                                       unsigned *cnt)
{
    __shared__ real sh[kKG][kRedBlock / 32];
    __shared__ real ss[8];
    if (threadIdx.x < NV)
        ss[threadIdx.x] = s2[threadIdx.x];
    __syncthreads();
    const int64_t nq = (n + 3) >> 2, cq = (nq + gridDim.x - 1) / gridDim.x;
    const int64_t q0 = blockIdx.x * cq, q1 = q0 + cq < nq ? q0 + cq : nq;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int c0 = 0; c0 < ncol; c0 += kKG)
    {
        real a[kKG];
#pragma unroll
        for (int k = 0; k < kKG; k++)
            a[k] = 0;
        // r = (4 q) % NV, advanced incrementally with q
        const int dr = (int)((4 * (int64_t)blockDim.x) % NV);
        int r = (int)((4 * (q0 + threadIdx.x)) % NV);
        const T *Vc = V + (int64_t)c0 * ld;
        for (int64_t q = q0 + threadIdx.x; q < q1; q += blockDim.x)
        {
            real wv[4];
            Quad<T>::load(w + 4 * q, wv);
#pragma unroll
            for (int e = 0; e < 4; e++)
                wv[e] *= ss[r + e < NV ? r + e : r + e - NV];
            r += dr;
            r = r >= NV ? r - NV : r;
            const T *pv = Vc + 4 * q;
            if (c0 + kKG <= ncol)
            {
                // a full group: every load issued (in its storage type) before the first use
                typename Quad<T>::raw v[kKG];
#pragma unroll
                for (int k = 0; k < kKG; k++)
                    v[k] = Quad<T>::load_raw(pv + k * ld);
#pragma unroll
                for (int k = 0; k < kKG; k++)
                    a[k] += Quad<T>::dot(v[k], wv);
            }
            else
            {
#pragma unroll
                for (int k = 0; k < kKG; k++)
                    if (c0 + k < ncol)
                    {
                        real v[4];
                        Quad<T>::load(pv + k * ld, v);
                        a[k] += v[0] * wv[0] + v[1] * wv[1] + v[2] * wv[2] + v[3] * wv[3];
                    }
            }
        }
#pragma unroll
        for (int k = 0; k < kKG; k++)
        {
            real x = warp_sum(a[k]);
            if (lane == 0)
                sh[k][wid] = x;
        }
        __syncthreads();
        if (threadIdx.x < kKG && c0 + (int)threadIdx.x < ncol)
        {
            real t = 0;
            for (int q = 0; q < nw; q++)
                t += sh[threadIdx.x][q];
            partial[blockIdx.x * ncol + c0 + threadIdx.x] = t;
        }
        __syncthreads();
    }
    last_block_final(ncol, partial, out, colScale, 0, cnt);
}

// w -= sum_c h[c] colScale[c] V[c] (columns subtracted in index order); the last block writes
// *outNorm = sqrt(sum_i w_i^2 s2[i % NV]) of the stored w.  w is column ncol of the same basis (not read
// through V).  With gsc (the GMRES scalars: [0] scale, [2] valid columns) it also sets the normalising
// factor of the new column, *scaleNext = 1 / norm, or 0 at a breakdown (norm <= 1e-32 scale), which it
// records in gsc[2] = j (GMRES_LeftPreconditioned::solve, Linear.hpp:100-108).
template <typename T, int NV>
DNDSB_GLOBAL void __launch_bounds__(kRedBlock, 4) k_kmaxpy_norm(int64_t n, int64_t ld, int ncol, const T *__restrict__ V, const real *__restrict__ h,
                                                             const real *__restrict__ colScale, T *w, const real *__restrict__ s2, real *partial,
                                                             real *outNorm, unsigned *cnt, real *gsc, int j, real *scaleNext)
{
    __shared__ real hs[32];
    __shared__ real ss[8];
    __shared__ real sh[kRedBlock / 32];
    if (threadIdx.x < ncol)
        hs[threadIdx.x] = h[threadIdx.x] * (colScale ? colScale[threadIdx.x] : 1.0);
    if (threadIdx.x < NV)
        ss[threadIdx.x] = s2[threadIdx.x];
    __syncthreads();
    const int64_t nq = (n + 3) >> 2, cq = (nq + gridDim.x - 1) / gridDim.x;
    const int64_t q0 = blockIdx.x * cq, q1 = q0 + cq < nq ? q0 + cq : nq;
    real a = 0;
    const int dr = (int)((4 * (int64_t)blockDim.x) % NV);
    int r = (int)((4 * (q0 + threadIdx.x)) % NV);
    for (int64_t q = q0 + threadIdx.x; q < q1; q += blockDim.x)
    {
        real x[4];
        Quad<T>::load(w + 4 * q, x);
        int c = 0;
        for (; c + 4 <= ncol; c += 4)
        {
            real v[4][4];
#pragma unroll
            for (int k = 0; k < 4; k++)
                Quad<T>::load(V + (int64_t)(c + k) * ld + 4 * q, v[k]);
#pragma unroll
            for (int k = 0; k < 4; k++)
            {
                const real hc = hs[c + k];
#pragma unroll
                for (int e = 0; e < 4; e++)
                    x[e] -= hc * v[k][e];
            }
        }
        for (; c < ncol; c++)
        {
            real v[4];
            Quad<T>::load(V + (int64_t)c * ld + 4 * q, v);
            const real hc = hs[c];
#pragma unroll
            for (int e = 0; e < 4; e++)
                x[e] -= hc * v[e];
        }
        real xr[4];
        Quad<T>::store(w + 4 * q, x, xr);
#pragma unroll
        for (int e = 0; e < 4; e++)
            a += xr[e] * xr[e] * ss[r + e < NV ? r + e : r + e - NV];
        r += dr;
        r = r >= NV ? r - NV : r;
    }
    const real x = warp_sum(a);
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        real t = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++)
            t += sh[q];
        partial[blockIdx.x] = t;
    }
    if (last_block_final(1, partial, outNorm, nullptr, 1, cnt) && gsc && threadIdx.x == 0)
    {
        real hn = *outNorm;
        bool broken = !(hn > gsc[0] * 1e-32) || gsc[2] <= j;
        *scaleNext = broken ? 0.0 : 1.0 / hn;
        if (broken && gsc[2] > j)
            gsc[2] = j;
    }
}

// partial[block] = sum_i x_i^2 s2[i % NV] (any length, any alignment)
template <typename T, int NV>
DNDSB_GLOBAL void k_knorm2(int64_t n, const T *__restrict__ x, const real *__restrict__ s2, real *partial, real *outNorm, unsigned *cnt)
{
    __shared__ real sh[4][kRedBlock];
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t b0 = blockIdx.x * chunk, b1 = b0 + chunk < n ? b0 + chunk : n;
    real a = 0;
    for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x)
    {
        real d = (real)x[i];
        a += d * d * s2[i % NV];
    }
    block_sum4(sh, a, 0, 0, 0);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = sh[0][0];
    last_block_final(1, partial, outNorm, nullptr, 1, cnt);
}

// partial[block] = sum_i (a_i - b_i)^2 s2[i % NV]
template <typename T, int NV>
DNDSB_GLOBAL void k_kdiff_norm(int64_t n, const T *__restrict__ x, const T *__restrict__ y, const real *__restrict__ s2, real *partial,
                               real *outNorm, unsigned *cnt)
{
    __shared__ real sh[4][kRedBlock];
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t b0 = blockIdx.x * chunk, b1 = b0 + chunk < n ? b0 + chunk : n;
    real a = 0;
    for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x)
    {
        real d = (real)x[i] - (real)y[i];
        a += d * d * s2[i % NV];
    }
    block_sum4(sh, a, 0, 0, 0);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = sh[0][0];
    last_block_final(1, partial, outNorm, nullptr, 1, cnt);
}

template <typename T, int NV>
void kmdot(int64_t n, int64_t ld, int ncol, const void *V, const void *w, const real *s2, real *red, real *out, const real *colScale,
           unsigned *cnt, cudaStream_t st)
{
    k_kmdot<T, NV><<<kRedBlocks, kRedBlock, 0, st>>>(n, ld, ncol, (const T *)V, (const T *)w, s2, red, out, colScale, cnt);
}

template <typename T, int NV>
void kmaxpy(int64_t n, int64_t ld, int ncol, const void *V, const real *h, const real *colScale, void *w, const real *s2, real *red,
            real *outNorm, unsigned *cnt, real *gsc, int j, real *scaleNext, cudaStream_t st)
{
    k_kmaxpy_norm<T, NV><<<kRedBlocks, kRedBlock, 0, st>>>(n, ld, ncol, (const T *)V, h, colScale, (T *)w, s2, red, outNorm, cnt, gsc, j,
                                                           scaleNext);
}

template <typename T, int NV>
void knorm(int64_t n, const void *x, const real *s2, real *red, real *outNorm, unsigned *cnt, cudaStream_t st)
{
    k_knorm2<T, NV><<<kRedBlocks, kRedBlock, 0, st>>>(n, (const T *)x, s2, red, outNorm, cnt);
}

template <typename T, int NV>
void kdiff(int64_t n, const void *x, const void *y, const real *s2, real *red, real *outNorm, unsigned *cnt, cudaStream_t st)
{
    k_kdiff_norm<T, NV><<<kRedBlocks, kRedBlock, 0, st>>>(n, (const T *)x, (const T *)y, s2, red, outNorm, cnt);
}

#define DNDSB_KDISPATCH(FN, ...)                      \
    do                                                \
    {                                                 \
        if (prec == 0 && nv == 5)                     \
            FN<double, 5>(__VA_ARGS__);               \
        else if (prec == 0)                           \
            FN<double, 6>(__VA_ARGS__);               \
        else if (nv == 5)                             \
            FN<float, 5>(__VA_ARGS__);                \
        else                                          \
            FN<float, 6>(__VA_ARGS__);                \
    } while (0)
} // namespace

// V: ncol columns ld apart (ld a multiple of 4, 16-byte aligned, zero beyond n); w: a column of the same storage
void krylov_mdot(int prec, int64_t n, int64_t ld, int nv, int ncol, const void *V, const void *w, const real *s2, real *red, real *out,
                 const real *colScale, unsigned *cnt, cudaStream_t st)
{
    DNDSB_KDISPATCH(kmdot, n, ld, ncol, V, w, s2, red, out, colScale, cnt, st);
}

void krylov_maxpy_norm(int prec, int64_t n, int64_t ld, int nv, int ncol, const void *V, const real *h, const real *colScale, void *w,
                       const real *s2, real *red, real *outNorm, unsigned *cnt, real *gsc, int j, real *scaleNext, cudaStream_t st)
{
    DNDSB_KDISPATCH(kmaxpy, n, ld, ncol, V, h, colScale, w, s2, red, outNorm, cnt, gsc, j, scaleNext, st);
}

void krylov_norm(int prec, int64_t n, int nv, const void *x, const real *s2, real *red, real *outNorm, unsigned *cnt, cudaStream_t st)
{
    DNDSB_KDISPATCH(knorm, n, x, s2, red, outNorm, cnt, st);
}

void krylov_diff_norm(int prec, int64_t n, int nv, const void *x, const void *y, const real *s2, real *red, real *outNorm, unsigned *cnt,
                      cudaStream_t st)
{
    DNDSB_KDISPATCH(kdiff, n, x, y, s2, red, outNorm, cnt, st);
}
} // namespace dndsb
