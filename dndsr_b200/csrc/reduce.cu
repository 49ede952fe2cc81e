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

// partial[block][col] = sum_i V[col][i] * w[i] * s2[i % NV] over the block's chunk
template <typename T, int NV>
DNDSB_GLOBAL void k_kmdot(int64_t n, int ncol, const T *__restrict__ V, const T *__restrict__ w, const real *__restrict__ s2, real *partial)
{
    __shared__ real sh[4][kRedBlock];
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t b0 = blockIdx.x * chunk, b1 = b0 + chunk < n ? b0 + chunk : n;
    for (int c0 = 0; c0 < ncol; c0 += 4)
    {
        real a[4] = {0, 0, 0, 0};
        for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x)
        {
            real wi = (real)w[i] * s2[i % NV];
            for (int q = 0; q < 4; q++)
                if (c0 + q < ncol)
                    a[q] += (real)V[(int64_t)(c0 + q) * n + i] * wi;
        }
        block_sum4(sh, a[0], a[1], a[2], a[3]);
        if (threadIdx.x == 0)
            for (int q = 0; q < 4 && c0 + q < ncol; q++)
                partial[blockIdx.x * ncol + c0 + q] = sh[q][0];
        __syncthreads();
    }
}

// w -= sum_c h[c] V[c]; partial[block] = sum_i w_i^2 s2[i % NV] of the stored w
template <typename T, int NV>
DNDSB_GLOBAL void k_kmaxpy_norm(int64_t n, int ncol, const T *__restrict__ V, const real *__restrict__ h, T *w, const real *__restrict__ s2,
                                real *partial)
{
    __shared__ real sh[4][kRedBlock];
    __shared__ real hs[33];
    if (threadIdx.x < ncol)
        hs[threadIdx.x] = h[threadIdx.x];
    __syncthreads();
    int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    int64_t b0 = blockIdx.x * chunk, b1 = b0 + chunk < n ? b0 + chunk : n;
    real a = 0;
    for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x)
    {
        real x = (real)w[i];
        for (int c = 0; c < ncol; c++)
            x -= hs[c] * (real)V[(int64_t)c * n + i];
        T xt = (T)x;
        w[i] = xt;
        a += (real)xt * (real)xt * s2[i % NV];
    }
    block_sum4(sh, a, 0, 0, 0);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = sh[0][0];
}

// partial[block] = sum_i (a_i - b_i)^2 s2[i % NV]
template <typename T, int NV>
DNDSB_GLOBAL void k_kdiff_norm(int64_t n, const T *__restrict__ x, const T *__restrict__ y, const real *__restrict__ s2, real *partial)
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
}

// out[col] = sum over blocks (fixed tree), optionally its square root
DNDSB_GLOBAL void k_kfinal(int nb, int ncol, const real *__restrict__ partial, real *out, int takeSqrt)
{
    __shared__ real sh[kRedBlock];
    for (int col = 0; col < ncol; col++)
    {
        real a = 0;
        for (int i = threadIdx.x; i < nb; i += blockDim.x)
            a += partial[i * ncol + col];
        sh[threadIdx.x] = a;
        __syncthreads();
        for (int st = blockDim.x / 2; st > 0; st >>= 1)
        {
            if (threadIdx.x < st)
                sh[threadIdx.x] += sh[threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            out[col] = takeSqrt ? sqrt(sh[0]) : sh[0];
        __syncthreads();
    }
}

template <typename T, int NV>
void kmdot(int64_t n, int ncol, const void *V, const void *w, const real *s2, real *red, real *out, cudaStream_t st)
{
    k_kmdot<T, NV><<<kRedBlocks, kRedBlock, 0, st>>>(n, ncol, (const T *)V, (const T *)w, s2, red);
    k_kfinal<<<1, kRedBlock, 0, st>>>(kRedBlocks, ncol, red, out, 0);
}

template <typename T, int NV>
void kmaxpy(int64_t n, int ncol, const void *V, const real *h, void *w, const real *s2, real *red, real *outNorm, cudaStream_t st)
{
    k_kmaxpy_norm<T, NV><<<kRedBlocks, kRedBlock, 0, st>>>(n, ncol, (const T *)V, h, (T *)w, s2, red);
    k_kfinal<<<1, kRedBlock, 0, st>>>(kRedBlocks, 1, red, outNorm, 1);
}

template <typename T, int NV>
void kdiff(int64_t n, const void *x, const void *y, const real *s2, real *red, real *outNorm, cudaStream_t st)
{
    k_kdiff_norm<T, NV><<<kRedBlocks, kRedBlock, 0, st>>>(n, (const T *)x, (const T *)y, s2, red);
    k_kfinal<<<1, kRedBlock, 0, st>>>(kRedBlocks, 1, red, outNorm, 1);
}

DNDSB_GLOBAL void k_ksqrt(real *x)
{
    if (threadIdx.x == 0)
        *x = sqrt(*x);
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

void krylov_mdot(int prec, int64_t n, int nv, int ncol, const void *V, const void *w, const real *s2, real *red, real *out, cudaStream_t st)
{
    DNDSB_KDISPATCH(kmdot, n, ncol, V, w, s2, red, out, st);
}

void krylov_maxpy_norm(int prec, int64_t n, int nv, int ncol, const void *V, const real *h, void *w, const real *s2, real *red, real *outNorm,
                       cudaStream_t st)
{
    DNDSB_KDISPATCH(kmaxpy, n, ncol, V, h, w, s2, red, outNorm, st);
}

void krylov_norm(int prec, int64_t n, int nv, const void *x, const real *s2, real *red, real *outNorm, cudaStream_t st)
{
    // |x| = sqrt(x . x): the dot with itself, then the root on the device
    DNDSB_KDISPATCH(kmdot, n, 1, x, x, s2, red, outNorm, st);
    k_ksqrt<<<1, 1, 0, st>>>(outNorm);
}

void krylov_diff_norm(int prec, int64_t n, int nv, const void *x, const void *y, const real *s2, real *red, real *outNorm, cudaStream_t st)
{
    DNDSB_KDISPATCH(kdiff, n, x, y, s2, red, outNorm, st);
}
} // namespace dndsb
