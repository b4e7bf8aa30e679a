// Pixel-likelihood terms from a Cholesky factor, FP64 (batched).
//
// For C = L L^T:  chi2 = x^T C^-1 x = |L^-1 x|^2 and ln|C| = 2 sum ln L_ii.
// The reference forms C^-1 explicitly and runs a second Cholesky for the
// log-determinant (picslike/picslike.py:643-664, cosmocore/basics/
// linalg.py:430-474); both numbers follow from the one factor.
//
// One CTA per (problem, map): blocked forward substitution, 32 rows at a
// time - warp 0 solves the 32 x 32 diagonal block with shuffles, then all
// warps apply the panel to the rows below (one warp per row, coalesced reads
// of L).
#include "cf_common.cuh"

namespace {

constexpr int NT = 256;

__global__ void __launch_bounds__(NT) k_chi2(int n, const double* L, long lda, long sL, const double* X,
                                             long ldx, long sX, int nrhs, double* z_work, double* chi2)
{
    const int b = blockIdx.x / nrhs, m = blockIdx.x % nrhs;
    L += (long)b * sL;
    X += (long)b * sX;
    double* z = z_work + (long)blockIdx.x * n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < n; i += NT) z[i] = X[(long)i * ldx + m];
    __syncthreads();
    for (int b0 = 0; b0 < n; b0 += 32) {
        const int kb = n - b0 < 32 ? n - b0 : 32;
        if (warp == 0) {
            // lane i holds row b0 + i of the diagonal block (independent loads)
            double lrow[32];
#pragma unroll
            for (int k = 0; k < 32; ++k) lrow[k] = (lane < kb && k < kb) ? L[(long)(b0 + lane) * lda + b0 + k] : 1.0;
            double zi = lane < kb ? z[b0 + lane] : 0.0;
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                if (r < kb) {
                    if (lane == r) zi /= lrow[r];
                    const double zr = __shfl_sync(0xffffffffu, zi, r);
                    if (lane > r) zi -= lrow[r] * zr;
                }
            }
            if (lane < kb) z[b0 + lane] = zi;
        }
        __syncthreads();
        // rows below: 8 coalesced row loads in flight per warp, then the reductions
        const double zl = lane < kb ? z[b0 + lane] : 0.0;
        for (int r0 = b0 + kb + warp * 8; r0 < n; r0 += (NT / 32) * 8) {
            double v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i)
                v[i] = (r0 + i < n && lane < kb) ? L[(long)(r0 + i) * lda + b0 + lane] * zl : 0.0;
#pragma unroll
            for (int i = 0; i < 8; ++i)
                for (int o = 16; o; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
            if (lane == 0)
#pragma unroll
                for (int i = 0; i < 8; ++i)
                    if (r0 + i < n) z[r0 + i] -= v[i];
        }
        __syncthreads();
    }
    double s = 0.0;
    for (int i = tid; i < n; i += NT) s += z[i] * z[i];
    __shared__ double red[NT / 32];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < NT / 32; ++w) t += red[w];
        chi2[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(NT) k_logdet(int n, const double* L, long lda, long sL, double* logdet)
{
    L += (long)blockIdx.x * sL;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) s += log(L[(long)i * lda + i]);
    __shared__ double red[NT / 32];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < NT / 32; ++w) t += red[w];
        logdet[blockIdx.x] = 2.0 * t;
    }
}

}  // namespace

// chi2[b * nrhs + m] = |L_b^-1 x_{b,m}|^2, logdet[b] = 2 sum ln (L_b)_ii.
// z_work holds batch * nrhs * n doubles.  strideX = 0 shares X across the batch.
extern "C" int cf_chi2_logdet(int n, const double* L, long lda, long strideL, int batch, const double* X,
                              long ldx, long strideX, int nrhs, double* z_work, double* chi2,
                              double* logdet, void* stream)
{
    if (n <= 0 || batch < 1 || nrhs < 0 || !L) return CF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (nrhs > 0) {
        if (!X || !z_work || !chi2) return CF_ERR_ARG;
        k_chi2<<<batch * nrhs, NT, 0, st>>>(n, L, lda, strideL, X, ldx, strideX, nrhs, z_work, chi2);
        CF_CHECK_LAUNCH();
    }
    if (logdet) {
        k_logdet<<<batch, NT, 0, st>>>(n, L, lda, strideL, logdet);
        CF_CHECK_LAUNCH();
    }
    return CF_OK;
}
