// Pixel-likelihood terms from a Cholesky factor, FP64 (batched).
//
// For C = L L^T:  chi2 = x^T C^-1 x = |L^-1 x|^2 and ln|C| = 2 sum ln L_ii.
// The reference forms C^-1 explicitly and runs a second Cholesky for the
// log-determinant (picslike/picslike.py:643-664, cosmocore/basics/
// linalg.py:430-474); both numbers follow from the one factor.
//
// One CTA per (problem, map), z = L^-1 x in shared memory (global scratch for
// n above the shared-memory limit).  Blocked forward substitution, 32 rows at a
// time: warp 0 solves the 32 x 32 diagonal block (lane = row, registers and
// shuffles, reciprocal pivots), then every thread takes one row below it and
// subtracts its 32-column segment of L times the block's z (one 256-byte row
// segment per thread, 16 loads in flight, no reductions).
#include "cf_common.cuh"
#include "tri_solve.cuh"

namespace {

constexpr int NT = 256;
constexpr int SMEM_MAX_N = 24576;  // z in shared memory up to 192 KB

template <bool VEC>
__global__ void __launch_bounds__(NT, 2) k_chi2(int n, const double* L, long lda, long sL, const double* X,
                                             long ldx, long sX, int nrhs, double* z_work, double* chi2)
{
    extern __shared__ double zsh[];
    const int b = blockIdx.x / nrhs, m = blockIdx.x % nrhs;
    L += (long)b * sL;
    X += (long)b * sX;
    double* z = z_work ? z_work + (long)blockIdx.x * n : zsh;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < n; i += NT) z[i] = X[(long)i * ldx + m];
    __syncthreads();
    for (int b0 = 0; b0 < n; b0 += 32) {
        const int kb = n - b0 < 32 ? n - b0 : 32;
        if (warp == 0) cf_tri::diag_forward(L, lda, b0, kb, z, lane);
        __syncthreads();
        for (int r = b0 + kb + tid; r < n; r += NT) z[r] -= cf_tri::seg_dot<VEC>(L + (long)r * lda + b0, z + b0, kb);
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

// The same chi2 with the factor's 64 x 64 diagonal-block inverses D (block j
// at D + j 64^2, row-major with row stride kb_j): 64-row blocks, each
// diagonal solve one block-times-vector product (no dependent chain), then
// the rows below take the block's 64-wide segment (z in shared memory).
template <bool VEC>
__global__ void __launch_bounds__(NT, 4) k_chi2_dinv(int n, const double* L, long lda, long sL, const double* D,
                                                     long sD, const double* X, long ldx, long sX, int nrhs,
                                                     double* chi2)
{
    extern __shared__ double zsh[];
    double* z = zsh;
    double* zb = zsh + n;
    const int b = blockIdx.x / nrhs, m = blockIdx.x % nrhs;
    L += (long)b * sL;
    D += (long)b * sD;
    X += (long)b * sX;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < n; i += NT) z[i] = X[(long)i * ldx + m];
    __syncthreads();
    for (int b0 = 0, blk = 0; b0 < n; b0 += 64, ++blk) {
        const int kb = n - b0 < 64 ? n - b0 : 64;
        cf_tri::block_matvec<double, false>(D + (long)blk * 64 * 64, kb, z + b0, zb, tid);
        __syncthreads();
        if (tid < kb) z[b0 + tid] = zb[tid];
        __syncthreads();
        for (int r = b0 + kb + tid; r < n; r += NT)
            z[r] -= cf_tri::seg_dot64<VEC>(L + (long)r * lda + b0, z + b0, kb);
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
// z_work holds batch * nrhs * n doubles (read only for n > 24576; may be NULL below).  strideX = 0 shares X across the batch.
extern "C" int cf_chi2_logdet(int n, const double* L, long lda, long strideL, int batch, const double* X,
                              long ldx, long strideX, int nrhs, double* z_work, double* chi2,
                              double* logdet, void* stream)
{
    if (n <= 0 || batch < 1 || nrhs < 0 || !L) return CF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (nrhs > 0) {
        if (!X || !chi2 || (n > SMEM_MAX_N && !z_work)) return CF_ERR_ARG;
        const bool vec = ((uintptr_t)L & 15) == 0 && (lda & 1) == 0 && (batch == 1 || (strideL & 1) == 0);
        const bool sh = n <= SMEM_MAX_N;
        const int smem = sh ? n * (int)sizeof(double) : 0;
        auto kern = vec ? k_chi2<true> : k_chi2<false>;
        static std::atomic<int> attr[2][CF_MAX_DEVICES];
        if (int rc = cf_smem_optin(kern, SMEM_MAX_N * (int)sizeof(double), attr[vec])) return rc;
        kern<<<batch * nrhs, NT, smem, st>>>(n, L, lda, strideL, X, ldx, strideX, nrhs, sh ? nullptr : z_work, chi2);
        CF_CHECK_LAUNCH();
    }
    if (logdet) {
        k_logdet<<<batch, NT, 0, st>>>(n, L, lda, strideL, logdet);
        CF_CHECK_LAUNCH();
    }
    return CF_OK;
}

// cf_chi2_logdet with the factor's diagonal-block inverses as cf_potrf leaves
// them in its workspace (Dinv = the workspace, strideD = cf_potrf_dinv_stride(n)
// doubles between problems): 64-row blocks solved by block-times-vector
// products instead of dependent substitution chains.  n <= 24576 (the solve
// vector in shared memory).
extern "C" int cf_chi2_logdet_dinv(int n, const double* L, long lda, long strideL, const double* Dinv, long strideD,
                                   int batch, const double* X, long ldx, long strideX, int nrhs, double* chi2,
                                   double* logdet, void* stream)
{
    if (n <= 0 || batch < 1 || nrhs < 0 || !L) return CF_ERR_ARG;
    if (n > SMEM_MAX_N - 64) return CF_ERR_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    if (nrhs > 0) {
        if (!X || !chi2 || !Dinv) return CF_ERR_ARG;
        const bool vec = ((uintptr_t)L & 15) == 0 && (lda & 1) == 0 && (batch == 1 || (strideL & 1) == 0);
        const int smem = (n + 64) * (int)sizeof(double);
        auto kern = vec ? k_chi2_dinv<true> : k_chi2_dinv<false>;
        static std::atomic<int> attr[2][CF_MAX_DEVICES];
        if (int rc = cf_smem_optin(kern, SMEM_MAX_N * (int)sizeof(double), attr[vec])) return rc;
        kern<<<batch * nrhs, NT, smem, st>>>(n, L, lda, strideL, Dinv, strideD, X, ldx, strideX, nrhs, chi2);
        CF_CHECK_LAUNCH();
    }
    if (logdet) {
        k_logdet<<<batch, NT, 0, st>>>(n, L, lda, strideL, logdet);
        CF_CHECK_LAUNCH();
    }
    return CF_OK;
}
