// MLP emulator kernels: dense layers with BF16 weights and FP32 accumulation,
// SiLU activations, their backward passes, MSE loss and Adam.
//
// The emulator (5 -> 256 -> 256 -> 256 -> 1) predicts -2 Delta lnL of the
// pixel likelihood; it has no counterpart in the reference.  Batches are at
// most a few thousand rows and layers 256 wide, so every kernel here is
// latency-bound; they are written as one tiled SIMT product with three operand
// layouts and fused epilogues, and the training step is meant to be captured
// in a CUDA graph by the host.
//
//   forward       Z = A W^T + b,  A' = silu(Z)          (A: M x K, W: N x K bf16)
//   backward data dZ_prev = (dZ W) * silu'(Z_prev)       (dZ: M x N, W: N x K bf16)
//   backward wgt  dW = dZ^T A_prev,  db = sum_rows dZ    (reduction over the batch)
#include <cuda_bf16.h>

#include "cf_common.cuh"

namespace {

constexpr int TM = 64, TN = 64, TK = 16, TT = 256;

__device__ __forceinline__ float sigmoidf_(float z) { return 1.0f / (1.0f + expf(-z)); }

enum { EPI_FWD = 0, EPI_BWD_DATA = 1, EPI_STORE = 2 };

// C[m, n] = sum_k A(m, k) B(k, n).
//   A_KC: A(m, k) = A[m * lda + k] (else A[k * lda + m]); FP32.
//   B_KC: B(k, n) = B[n * ldb + k] (else B[k * ldb + n]); BT = float or bf16.
// 64 x 64 tile, 256 threads with 4 x 4 outputs each.
template <bool A_KC, bool B_KC, typename BT, int EPI>
__global__ void __launch_bounds__(TT) k_dense(int M, int N, int K, const float* __restrict__ A, long lda,
                                              const BT* __restrict__ B, long ldb, const float* __restrict__ bias,
                                              int act, const float* __restrict__ Zprev, long ldzp, float* Zout,
                                              float* Cout, long ldc)
{
    __shared__ float As[TK][TM + 4];
    __shared__ float Bs[TK][TN + 4];
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += TK) {
        // 64 x 16 of each operand: 1024 elements, 4 per thread
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = u * TT + tid;
            int mm, kk;
            if (A_KC) {
                mm = e / TK;
                kk = e % TK;
            } else {
                kk = e / TM;
                mm = e % TM;
            }
            const int gm = m0 + mm, gk = k0 + kk;
            As[kk][mm] = (gm < M && gk < K) ? (A_KC ? A[(long)gm * lda + gk] : A[(long)gk * lda + gm]) : 0.0f;
            int nn, kb;
            if (B_KC) {
                nn = e / TK;
                kb = e % TK;
            } else {
                kb = e / TN;
                nn = e % TN;
            }
            const int gn = n0 + nn, gkb = k0 + kb;
            float bv = 0.0f;
            if (gn < N && gkb < K) {
                const BT x = B_KC ? B[(long)gn * ldb + gkb] : B[(long)gkb * ldb + gn];
                bv = (float)x;
            }
            Bs[kb][nn] = bv;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < TK; ++k) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[k][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[k][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            float v = acc[i][j];
            if (EPI == EPI_FWD) {
                v += bias ? bias[n] : 0.0f;
                if (Zout) Zout[(long)m * ldc + n] = v;
                if (act) v = v * sigmoidf_(v);
            } else if (EPI == EPI_BWD_DATA) {
                const float z = Zprev[(long)m * ldzp + n];
                const float s = sigmoidf_(z);
                v *= s * (1.0f + z * (1.0f - s));
            }
            Cout[(long)m * ldc + n] = v;
        }
    }
}

// db[n] = sum_m dZ[m, n]
__global__ void k_colsum(int M, int N, const float* dZ, long ld, float* db)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.0f;
    for (int m = 0; m < M; ++m) s += dZ[(long)m * ld + n];
    db[n] = s;
}

// Mean squared error over the batch: loss = sum w_m (y_m - t_m)^2 / sum w_m and
// dy_m = 2 w_m (y_m - t_m) / sum w_m (w = NULL: unit weights).  One CTA.
__global__ void k_mse(int M, const float* y, const float* t, const float* w, float* dy, float* loss)
{
    __shared__ float red[2][32];
    float s = 0.0f, sw = 0.0f;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        const float wm = w ? w[m] : 1.0f;
        const float d = y[m] - t[m];
        s += wm * d * d;
        sw += wm;
    }
    for (int o = 16; o; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        sw += __shfl_xor_sync(0xffffffffu, sw, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = s;
        red[1][threadIdx.x >> 5] = sw;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = blockDim.x >> 5;
        s = threadIdx.x < nw ? red[0][threadIdx.x] : 0.0f;
        sw = threadIdx.x < nw ? red[1][threadIdx.x] : 0.0f;
        for (int o = 16; o; o >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, o);
            sw += __shfl_xor_sync(0xffffffffu, sw, o);
        }
        if (threadIdx.x == 0) {
            red[0][0] = s;
            red[1][0] = sw;
        }
    }
    __syncthreads();
    const float tot = red[1][0];
    if (threadIdx.x == 0 && loss) *loss = red[0][0] / tot;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        const float wm = w ? w[m] : 1.0f;
        dy[m] = 2.0f * wm * (y[m] - t[m]) / tot;
    }
}

// Adam on FP32 master parameters; writes the BF16 working copy.
//   m = b1 m + (1 - b1) g;  v = b2 v + (1 - b2) g^2;
//   p -= lr m_hat / (sqrt(v_hat) + eps),  m_hat = m / (1 - b1^t), v_hat = v / (1 - b2^t),
// with t read from the device counter *step (so a captured step replays).
__global__ void k_adam(long count, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                       float eps, const int* step, __nv_bfloat16* p16)
{
    const float t = (float)*step;
    const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);
    const float lr_t = lr * sqrtf(c2) / c1, eps_t = eps * sqrtf(c2);
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr_t * mi / (sqrtf(vi) + eps_t);
        p[i] = pi;
        if (p16) p16[i] = __float2bfloat16_rn(pi);
    }
}

__global__ void k_increment(int* c) { *c += 1; }

__global__ void k_to_bf16(long count, const float* x, __nv_bfloat16* y)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16_rn(x[i]);
}

inline dim3 grid_for(int M, int N) { return dim3(cf_cdiv(N, TN), cf_cdiv(M, TM)); }

}  // namespace

// Z = A W^T + b and out = silu(Z) (act = 1) or Z (act = 0).
//   A: M x K FP32 (row stride lda); W: N x K BF16 (row stride K); b: N FP32 or NULL;
//   Z (may be NULL) and out: M x N FP32, row stride ldo.
extern "C" int cf_mlp_dense_fwd(int M, int N, int K, const float* A, long lda, const void* W, const float* b,
                                int act, float* Z, float* out, long ldo, void* stream)
{
    if (M <= 0 || N <= 0 || K <= 0 || !A || !W || !out) return CF_ERR_ARG;
    k_dense<true, true, __nv_bfloat16, EPI_FWD><<<grid_for(M, N), TT, 0, (cudaStream_t)stream>>>(
        M, N, K, A, lda, (const __nv_bfloat16*)W, K, b, act, nullptr, 0, Z, out, ldo);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// dZ_prev = (dZ W) * silu'(Z_prev): dZ M x N FP32 (row stride N), W N x K BF16,
// Z_prev and dZ_prev M x K FP32 (row stride K).
extern "C" int cf_mlp_dense_bwd_data(int M, int N, int K, const float* dZ, const void* W, const float* Zprev,
                                     float* dZprev, void* stream)
{
    if (M <= 0 || N <= 0 || K <= 0 || !dZ || !W || !Zprev || !dZprev) return CF_ERR_ARG;
    k_dense<true, false, __nv_bfloat16, EPI_BWD_DATA><<<grid_for(M, K), TT, 0, (cudaStream_t)stream>>>(
        M, K, N, dZ, N, (const __nv_bfloat16*)W, K, nullptr, 0, Zprev, K, nullptr, dZprev, K);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// dW = dZ^T A_prev (N x K FP32) and db = column sums of dZ (N), over M rows.
//   dZ: M x N FP32 (row stride N); A_prev: M x K FP32 (row stride lda).
extern "C" int cf_mlp_dense_bwd_weight(int M, int N, int K, const float* dZ, const float* Aprev, long lda,
                                       float* dW, float* db, void* stream)
{
    if (M <= 0 || N <= 0 || K <= 0 || !dZ || !Aprev || !dW) return CF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    k_dense<false, false, float, EPI_STORE><<<grid_for(N, K), TT, 0, st>>>(N, K, M, dZ, N, Aprev, lda, nullptr, 0,
                                                                           nullptr, 0, nullptr, dW, K);
    CF_CHECK_LAUNCH();
    if (db) {
        k_colsum<<<cf_cdiv(N, 128), 128, 0, st>>>(M, N, dZ, N, db);
        CF_CHECK_LAUNCH();
    }
    return CF_OK;
}

// Weighted MSE of predictions y against targets t (w may be NULL), its gradient
// dy, and the loss value into *loss (device float, may be NULL).
extern "C" int cf_mlp_mse(int M, const float* y, const float* t, const float* w, float* dy, float* loss,
                          void* stream)
{
    if (M <= 0 || !y || !t || !dy) return CF_ERR_ARG;
    k_mse<<<1, 1024, 0, (cudaStream_t)stream>>>(M, y, t, w, dy, loss);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// One Adam step over `count` parameters (FP32 master p, moments m, v, gradient
// g).  *step (device int) is incremented first and gives t for the bias
// corrections.  p16 (may be NULL) receives the BF16 copy of p.
extern "C" int cf_mlp_adam(long count, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                           float eps, int* step, void* p16, void* stream)
{
    if (count <= 0 || !p || !g || !m || !v || !step) return CF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    k_increment<<<1, 1, 0, st>>>(step);
    CF_CHECK_LAUNCH();
    long blocks = (count + 255) / 256;
    if (blocks > 1184) blocks = 1184;
    k_adam<<<(unsigned)blocks, 256, 0, st>>>(count, p, g, m, v, lr, b1, b2, eps, step, (__nv_bfloat16*)p16);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// y = bf16(x) for `count` values.
extern "C" int cf_to_bf16(long count, const float* x, void* y, void* stream)
{
    if (count <= 0 || !x || !y) return CF_ERR_ARG;
    long blocks = (count + 255) / 256;
    if (blocks > 1184) blocks = 1184;
    k_to_bf16<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(count, x, (__nv_bfloat16*)y);
    CF_CHECK_LAUNCH();
    return CF_OK;
}
