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
} // namespace dndsb
