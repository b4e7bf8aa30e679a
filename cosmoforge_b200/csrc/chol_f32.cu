// Mixed-precision pixel likelihood: FP32 batched Cholesky, FP64-refined chi2.
//
// The reference evaluates -2 lnL = x^T C^-1 x + ln|C| per parameter point with
// an FP64 inverse and a second FP64 Cholesky for the determinant
// (picslike/picslike.py:568-664, cosmocore/basics/linalg.py:362-474).  Here
// the factor is computed in FP32 and the solve is refined in FP64:
//
//   L L^T = C (FP32, blocked right-looking, 64-wide panels; the trailing
//           updates are FP32 SIMT GEMMs),
//   w = L^-1 x,  v = L^-T w               (FP64 arithmetic on the FP32 factor)
//   chi2 = 2 w.w - v^T C v                (C in FP64)
//
// The last line is x^T z_1 for one step of iterative refinement
// z_1 = z_0 + (L L^T)^-1 (x - C z_0) from z_0 = v, so the chi2 error is second
// order in the factor's backward error.  ln|C| = 2 sum ln L_ii carries the
// factor's first-order error.
#include "cf_common.cuh"
#include "potrf_diag.cuh"
#include "tri_solve.cuh"

#include "tc_sgemm.cuh"

namespace {

constexpr int NB = cf_diag::NB;

using cf_diag::k_potrf_diag_inv;

// Panels of 64 columns factored per pass before one trailing update (K = 64
// per panel): 2 or 4.
constexpr int MAX_GROUP = 4;
int g_potrf_f32_group = 4;

// Product kernel of the FP32 factor's panel solves and trailing updates:
// 1 = BF16x6 split products on the tensor cores (tc_sgemm.cu, default),
// 0 = the FP32 SIMT kernel below.
int g_potrf_f32_tensor = 1;

// FP32 SIMT GEMM, both operands K-contiguous (the "NT" form):
//   C[M x N] = alpha A[M x K] B[N x K]^T + beta C, batch on blockIdx.z.
// 128 x 128 tile, BK 16, 256 threads with 8 x 8 outputs each (two 4 x 4
// quadrants 64 rows / columns apart so shared-memory reads are broadcast-free
// float4s).  The next k-tile is fetched into registers while the current one
// is consumed.  lower_only: skip tiles strictly above the diagonal.
constexpr int SBM = 128, SBK = 16, SNT = 256, SPAD = 4;

__global__ void __launch_bounds__(SNT, 2) k_sgemm_nt(int M, int N, int K, float alpha, const float* A, long lda,
                                                  long sA, const float* B, long ldb, long sB, float beta, float* C,
                                                  long ldc, long sC, int lower_only)
{
    __shared__ __align__(16) float As[2][SBK][SBM + SPAD];
    __shared__ __align__(16) float Bs[2][SBK][SBM + SPAD];
    const int tile_m = blockIdx.y * SBM, tile_n = blockIdx.x * SBM;
    if (lower_only && tile_n > tile_m + SBM - 1) return;
    A += (long)blockIdx.z * sA;
    B += (long)blockIdx.z * sB;
    C += (long)blockIdx.z * sC;
    const int tid = threadIdx.x;
    // loader: thread -> (row lr, k half lk)
    const int lr = tid >> 1, lk = (tid & 1) * 8;
    const int ty = tid >> 4, tx = tid & 15;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
    float ra[8], rb[8];
    auto fetch = [&](int k0) {
        const int ga = tile_m + lr, gb = tile_n + lr;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int gk = k0 + lk + u;
            ra[u] = (ga < M && gk < K) ? A[(long)ga * lda + gk] : 0.0f;
            rb[u] = (gb < N && gk < K) ? B[(long)gb * ldb + gk] : 0.0f;
        }
    };
    auto stash = [&](int s) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            As[s][lk + u][lr] = ra[u];
            Bs[s][lk + u][lr] = rb[u];
        }
    };
    const int KT = (K + SBK - 1) / SBK;
    fetch(0);
    stash(0);
    __syncthreads();
    for (int kt = 0; kt < KT; ++kt) {
        const int s = kt & 1;
        if (kt + 1 < KT) fetch((kt + 1) * SBK);
#pragma unroll
        for (int k = 0; k < SBK; ++k) {
            const float4 a0 = *reinterpret_cast<const float4*>(&As[s][k][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[s][k][64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[s][k][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[s][k][64 + tx * 4]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        if (kt + 1 < KT) stash(s ^ 1);
        __syncthreads();
    }
    // reads of C first (independent loads, one latency), then 16-byte stores
    // when the row stride and base allow it
    const bool vec = ((ldc & 3) == 0) && ((((uintptr_t)C) & 15) == 0);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int r = tile_m + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int c = tile_n + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
            float v = alpha * acc[i][j];
            if (beta != 0.0f && r < M && c < N) v += beta * C[(long)r * ldc + c];
            acc[i][j] = v;
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int r = tile_m + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
        if (r >= M) continue;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int c0 = tile_n + h * 64 + tx * 4;
            float* pc = C + (long)r * ldc + c0;
            if (vec && c0 + 4 <= N) {
                *reinterpret_cast<float4*>(pc) =
                    make_float4(acc[i][h * 4], acc[i][h * 4 + 1], acc[i][h * 4 + 2], acc[i][h * 4 + 3]);
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (c0 + j < N) pc[j] = acc[i][h * 4 + j];
            }
        }
    }
}

int sgemm_nt_simt(int M, int N, int K, float alpha, const float* A, long lda, long sA, const float* B, long ldb,
                  long sB, float beta, float* C, long ldc, long sC, int batch, int lower_only, cudaStream_t st)
{
    if (M <= 0 || N <= 0) return CF_OK;
    dim3 grid(cf_cdiv(N, SBM), cf_cdiv(M, SBM), batch);
    k_sgemm_nt<<<grid, SNT, 0, st>>>(M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, lower_only);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

__global__ void k_copy2d_f32(int R, int Ccols, const float* src, long lds, long ss, float* dst, long ldd, long sd);

// The factor's work panel W (n rows x 2 NB columns per problem): FP32 for the
// SIMT kernel, or, for the tensor cores, the three BF16 split planes of the
// FP32 panel (split once, where the panel is solved, instead of in every
// output tile that reads it).  `ws` floats per problem hold either form.
struct Panel {
    float* f;
    long ws;
    int n;
    static constexpr int LD = MAX_GROUP * NB;  // columns: the panels of one pass
    __nv_bfloat16* planes() const { return reinterpret_cast<__nv_bfloat16*>(f); }
    long plane_stride() const { return (long)n * LD; }
};

// Panel solve: W[r0.., c0..c0+kb) = A21 Dinv^T (M x kb, K = kb), written to W
// and into the matrix at A21 in one pass (tensor cores: W as split planes), or
// by the SIMT GEMM and a copy.
int panel_solve(int M, int kb, float* a21, long lda, long sA, const float* D, const Panel& W, int r0, int c0,
                int batch, int* info, cudaStream_t st)
{
    if (g_potrf_f32_tensor) {
        const cf_sg::Opnd a{a21, lda, sA, 0}, d{D, kb, W.ws, 0};
        const cf_sg::Out o{nullptr, 0, 0, a21, lda, sA, W.planes() + (long)r0 * Panel::LD + c0, Panel::LD, 2 * W.ws,
                           W.plane_stride()};
        return cf_sg::sgemm(M, kb, kb, 1.0f, a, d, 0.0f, o, false, batch, 0, info, st);
    }
    float* w = W.f + (long)r0 * Panel::LD + c0;
    int rc = sgemm_nt_simt(M, kb, kb, 1.0f, a21, lda, sA, D, kb, W.ws, 0.0f, w, Panel::LD, W.ws, batch, 0, st);
    if (rc) return rc;
    k_copy2d_f32<<<dim3(cf_cdiv(kb, 32), cf_cdiv(M, 8), batch), dim3(32, 8), 0, st>>>(M, kb, w, Panel::LD, W.ws, a21,
                                                                                      lda, sA);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// C -= W[ra.., 0:K) W[rb.., 0:K)^T (M x N), lower_only as in the GEMMs.
int panel_update(int M, int N, int K, const Panel& W, int ra, int rb, float* C, long ldc, long sC, int batch,
                 int lower_only, int* info, cudaStream_t st)
{
    if (g_potrf_f32_tensor) {
        const cf_sg::Opnd a{W.planes() + (long)ra * Panel::LD, Panel::LD, 2 * W.ws, W.plane_stride()};
        const cf_sg::Opnd b{W.planes() + (long)rb * Panel::LD, Panel::LD, 2 * W.ws, W.plane_stride()};
        const cf_sg::Out o{C, ldc, sC, nullptr, 0, 0, nullptr, 0, 0, 0};
        return cf_sg::sgemm(M, N, K, -1.0f, a, b, 1.0f, o, true, batch, lower_only, info, st);
    }
    const float* wa = W.f + (long)ra * Panel::LD;
    const float* wb = W.f + (long)rb * Panel::LD;
    return sgemm_nt_simt(M, N, K, -1.0f, wa, Panel::LD, W.ws, wb, Panel::LD, W.ws, 1.0f, C, ldc, sC, batch,
                         lower_only, st);
}

__global__ void k_copy2d_f32(int R, int Ccols, const float* src, long lds, long ss, float* dst, long ldd, long sd)
{
    src += blockIdx.z * ss;
    dst += blockIdx.z * sd;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r < R && c < Ccols) dst[(long)r * ldd + c] = src[(long)r * lds + c];
}

// Z = a X + c_b W in FP64 and Z32 = (float) Z, per batch entry b.
__global__ void k_axpby_f32(long count, double a, const double* X, long sX, double c, const double* cvec,
                            const double* W, long sW, double* Z, long sZ, float* Z32, long sZ32)
{
    const int b = blockIdx.y;
    const double cb = cvec ? cvec[b] : c;
    X += b * sX;
    W += b * sW;
    if (Z) Z += b * sZ;
    Z32 += b * sZ32;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < count; e += (long)gridDim.x * blockDim.x) {
        const double v = a * X[e] + cb * W[e];
        if (Z) Z[e] = v;
        Z32[e] = (float)v;
    }
}

constexpr int CNT = 256;

// One CTA per (problem b, map m): w = L^-1 x, v = L^-T w (FP64 arithmetic on
// the FP32 factor, both vectors in shared memory), then
// chi2 = 2 w.w - v^T C v with C read from its FP64 lower triangle.  Both
// solves run over 32-row blocks (cf_tri): warp 0 solves the diagonal block,
// then the CTA applies the block's 32-wide segments - forward, one row
// segment of L per thread below the block; backward, one column of the block
// row per thread to its left, while the threads on rows at or below the block
// add that block's 32 columns of the lower triangle of C to v^T C v (every v
// they need is final by then), so C is read once, in row segments.
template <bool VL, bool VC, typename TC>
__global__ void __launch_bounds__(CNT, 2) k_chi2_refined(int n, const float* L, long lda, long sL, const TC* C,
                                                         long ldc, long sC, const double* X, long ldx, long sX,
                                                         int nrhs, double* chi2)
{
    extern __shared__ double sh[];
    double* w = sh;
    double* v = sh + n;
    const int b = blockIdx.x / nrhs, m = blockIdx.x % nrhs;
    L += (long)b * sL;
    C += (long)b * sC;
    X += (long)b * sX;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __shared__ double red[CNT / 32];
    for (int i = tid; i < n; i += CNT) w[i] = X[(long)i * ldx + m];
    __syncthreads();
    for (int b0 = 0; b0 < n; b0 += 32) {
        const int kb = n - b0 < 32 ? n - b0 : 32;
        if (warp == 0) cf_tri::diag_forward(L, lda, b0, kb, w, lane);
        __syncthreads();
        for (int r = b0 + kb + tid; r < n; r += CNT) w[r] -= cf_tri::seg_dot<VL>(L + (long)r * lda + b0, w + b0, kb);
        __syncthreads();
    }
    double s = 0.0;
    for (int i = tid; i < n; i += CNT) {
        v[i] = w[i];
        s += 2.0 * w[i] * w[i];
    }
    __syncthreads();
    double qf = 0.0;  // this thread's share of v^T C v
    for (int b0 = ((n - 1) / 32) * 32; b0 >= 0; b0 -= 32) {
        const int kb = n - b0 < 32 ? n - b0 : 32;
        if (warp == 0) cf_tri::diag_backward(L, lda, b0, kb, v, lane);
        __syncthreads();
        for (int q = tid; q < n; q += CNT) {
            if (q < b0) {
                v[q] -= cf_tri::col_dot(L, lda, b0, q, v + b0, kb);
            } else if (q >= b0 + kb) {
                qf += 2.0 * v[q] * cf_tri::seg_dot<VC>(C + (long)q * ldc + b0, v + b0, kb);
            } else {
                const TC* cr = C + (long)q * ldc;
                double t = (double)cr[q] * v[q];
                for (int c = b0; c < q; ++c) t += 2.0 * (double)cr[c] * v[c];
                qf += v[q] * t;
            }
        }
        __syncthreads();
    }
    s -= qf;
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int q = 0; q < CNT / 32; ++q) t += red[q];
        chi2[blockIdx.x] = t;
    }
}

// k_chi2_refined with the FP32 factor's diagonal-block inverses D: 64-row
// blocks, each diagonal solve a block-times-vector product (forward with D,
// backward with D^T), the rows below / columns left of the block and the
// quadratic-form strip as in k_chi2_refined.
template <bool VL, bool VC, typename TC>
__global__ void __launch_bounds__(CNT, 4) k_chi2_refined_dinv(int n, const float* L, long lda, long sL,
                                                              const float* D, long sD, const TC* C, long ldc,
                                                              long sC, const double* X, long ldx, long sX, int nrhs,
                                                              double* chi2)
{
    extern __shared__ double sh[];
    double* w = sh;
    double* v = sh + n;
    double* tb = sh + 2 * n;  // 64 doubles: a block's solution before it replaces the right-hand side
    const int b = blockIdx.x / nrhs, m = blockIdx.x % nrhs;
    L += (long)b * sL;
    D += (long)b * sD;
    C += (long)b * sC;
    X += (long)b * sX;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __shared__ double red[CNT / 32];
    for (int i = tid; i < n; i += CNT) w[i] = X[(long)i * ldx + m];
    __syncthreads();
    const int nb64 = (n + 63) / 64;
    for (int blk = 0; blk < nb64; ++blk) {
        const int b0 = blk * 64, kb = n - b0 < 64 ? n - b0 : 64;
        cf_tri::block_matvec<float, false>(D + (long)blk * 64 * 64, kb, w + b0, tb, tid);
        __syncthreads();
        if (tid < kb) w[b0 + tid] = tb[tid];
        __syncthreads();
        for (int r = b0 + kb + tid; r < n; r += CNT) w[r] -= cf_tri::seg_dot64<VL>(L + (long)r * lda + b0, w + b0, kb);
        __syncthreads();
    }
    double s = 0.0;
    for (int i = tid; i < n; i += CNT) {
        v[i] = w[i];
        s += 2.0 * w[i] * w[i];
    }
    __syncthreads();
    double qf = 0.0;  // this thread's share of v^T C v
    for (int blk = nb64 - 1; blk >= 0; --blk) {
        const int b0 = blk * 64, kb = n - b0 < 64 ? n - b0 : 64;
        cf_tri::block_matvec<float, true>(D + (long)blk * 64 * 64, kb, v + b0, tb, tid);
        __syncthreads();
        if (tid < kb) v[b0 + tid] = tb[tid];
        __syncthreads();
        for (int q = tid; q < n; q += CNT) {
            if (q < b0) {
                v[q] -= cf_tri::col_dot64(L, lda, b0, q, v + b0, kb);
            } else if (q >= b0 + kb) {
                qf += 2.0 * v[q] * cf_tri::seg_dot64<VC>(C + (long)q * ldc + b0, v + b0, kb);
            } else {
                const TC* cr = C + (long)q * ldc;
                double t = (double)cr[q] * v[q];
                for (int c = b0; c < q; ++c) t += 2.0 * (double)cr[c] * v[c];
                qf += v[q] * t;
            }
        }
        __syncthreads();
    }
    s -= qf;
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int q = 0; q < CNT / 32; ++q) t += red[q];
        chi2[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(CNT) k_logdet_f32(int n, const float* L, long lda, long sL, double* logdet)
{
    L += (long)blockIdx.x * sL;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += CNT) s += log((double)L[(long)i * lda + i]);
    __shared__ double red[CNT / 32];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < CNT / 32; ++q) t += red[q];
        logdet[blockIdx.x] = 2.0 * t;
    }
}

// floats per problem: every diagonal-block inverse (kept for the chi2 solves)
// and the work panel (FP32, or three BF16 planes of it: 3 n LD / 2 floats)
inline int nblk(int n) { return (n + NB - 1) / NB; }
inline size_t potrf_f32_dinv(int n) { return (size_t)nblk(n) * NB * NB; }
inline size_t potrf_f32_ws(int n) { return potrf_f32_dinv(n) + (size_t)3 * n * Panel::LD / 2; }

}  // namespace

// Product kernel of cf_potrf_f32: 1 = BF16x6 tensor cores (default), 0 = FP32
// SIMT.  Returns the previous setting.
extern "C" int cf_potrf_f32_set_tensor(int on)
{
    const int prev = g_potrf_f32_tensor;
    g_potrf_f32_tensor = on ? 1 : 0;
    return prev;
}

// Panels per pass of cf_potrf_f32 (2 or 4: one trailing update per 128 or 256
// columns).  Returns the previous setting.
extern "C" int cf_potrf_f32_set_group(int panels)
{
    const int prev = g_potrf_f32_group;
    if (panels == 2 || panels == 4) g_potrf_f32_group = panels;
    return prev;
}

// Floats between consecutive problems' diagonal-block inverses in the
// cf_potrf_f32 workspace (block j of problem z at work + z stride + j 64^2).
extern "C" size_t cf_potrf_f32_dinv_stride(int n) { return potrf_f32_ws(n); }

extern "C" size_t cf_potrf_f32_workspace(int n, int batch) { return potrf_f32_ws(n) * sizeof(float) * (size_t)batch; }

// Blocked FP32 Cholesky in place (lower factor), batched: per 64-wide panel the
// diagonal block is factored and inverted by one CTA and L21 = A21 L11^-T is a
// GEMM; panels go in passes of four (cf_potrf_f32_set_group) so the trailing
// update A22 -= L21 L21^T runs once per 256 columns.  The GEMMs are BF16x6 split products on the tensor cores
// unless cf_potrf_f32_set_tensor(0) selects the SIMT kernel: each panel solve
// writes its panel into the matrix (FP32) and into the work panel as three
// BF16 split planes, which the updates then copy straight into shared memory.
// info: int[batch] zeroed by the caller; k > 0 is the first bad pivot, -3 a
// tensor-core wait that ran out.
extern "C" int cf_potrf_f32(int n, float* A, long lda, long strideA, int batch, void* work, int* info, void* stream)
{
    if (n <= 0 || batch < 1 || !A || !work || lda < n) return CF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const long ws = (long)potrf_f32_ws(n);
    float* Dall = (float*)work;  // [batch][blocks][NB][NB]: block j's inverse at j NB^2
    const Panel W{Dall + potrf_f32_dinv(n), ws, n};
    constexpr size_t DSM = cf_diag::smem_bytes<float>();
    const int G = g_potrf_f32_group;
    // Passes of G panels.  W row r holds matrix row k0 + NB + r (the rows
    // below the pass's first diagonal block); panel j's columns are W columns
    // j NB ..  Panel j is first brought up to date with the pass's earlier
    // panels (K = j NB), then factored and solved; one trailing update of
    // K = G NB follows the pass, so the trailing matrix is read and written
    // once per G NB columns.
    for (int k0 = 0; k0 < n; k0 += G * NB) {
        int kdone = 0;
        bool last = false;
        for (int jp = 0; jp < G; ++jp) {
            const int kj = k0 + jp * NB;
            const int kbj = n - kj < NB ? n - kj : NB;
            if (jp > 0) {
                int rc = panel_update(n - kj, kbj, kdone, W, (jp - 1) * NB, (jp - 1) * NB,
                                      A + (long)kj * lda + kj, lda, strideA, batch, 0, info, st);
                if (rc) return rc;
            }
            float* D = Dall + (long)(kj / NB) * NB * NB;
            k_potrf_diag_inv<float><<<batch, cf_diag::NTHREADS, DSM, st>>>(A, lda, strideA, kj, kbj, D, ws, info);
            CF_CHECK_LAUNCH();
            const int rest = n - kj - kbj;
            if (rest <= 0) {
                last = true;
                break;
            }
            int rc = panel_solve(rest, kbj, A + (long)(kj + kbj) * lda + kj, lda, strideA, D, W, jp * NB, jp * NB,
                                 batch, info, st);
            if (rc) return rc;
            kdone += kbj;
        }
        if (last) break;
        // trailing update with the pass's panels, lower tiles
        const int t0 = k0 + G * NB;
        int rc = panel_update(n - t0, n - t0, kdone, W, (G - 1) * NB, (G - 1) * NB, A + (long)t0 * (lda + 1), lda,
                              strideA, batch, 1, info, st);
        if (rc) return rc;
    }
    return CF_OK;
}

// Z_b = a X_b + c_b W_b in FP64 (Z may be NULL) and its FP32 copy Z32_b
// (c_b = cvec[b] if cvec else c; strideW = 0 shares W).  The noise addition
// C = S + s N of picslike/picslike.py:301-319 producing both precisions.
extern "C" int cf_axpby_f32(long count, double a, const double* X, long strideX, double c, const double* cvec,
                            const double* W, long strideW, double* Z, long strideZ, float* Z32, long strideZ32,
                            int batch, void* stream)
{
    if (count <= 0 || batch < 1 || !X || !W || !Z32) return CF_ERR_ARG;
    long blocks = (count + 255) / 256;
    if (blocks > 1184) blocks = 1184;
    k_axpby_f32<<<dim3((unsigned)blocks, batch), 256, 0, (cudaStream_t)stream>>>(count, a, X, strideX, c, cvec, W,
                                                                                 strideW, Z, strideZ, Z32,
                                                                                 strideZ32);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

namespace {
template <typename TC>
int chi2_mixed(int n, const float* L, long lda, long strideL, const TC* C, long ldc, long strideC, int batch,
               const double* X, long ldx, long strideX, int nrhs, double* chi2, double* logdet, cudaStream_t st,
               const float* Dinv = nullptr, long strideD = 0)
{
    if (n <= 0 || batch < 1 || nrhs < 0 || !L) return CF_ERR_ARG;
    if (n > 12288 - 32) return CF_ERR_UNSUPPORTED;
    if (nrhs > 0) {
        if (!X || !C || !chi2) return CF_ERR_ARG;
        const size_t smem = (2 * (size_t)n + 64) * sizeof(double);
        constexpr long VW = 16 / sizeof(TC);  // elements per 16-byte vector
        const bool vl = ((uintptr_t)L & 15) == 0 && (lda & 3) == 0 && (batch == 1 || (strideL & 3) == 0);
        const bool vc = ((uintptr_t)C & 15) == 0 && (ldc % VW) == 0 && (batch == 1 || (strideC % VW) == 0);
        if (Dinv) {
            auto kern = vl ? (vc ? k_chi2_refined_dinv<true, true, TC> : k_chi2_refined_dinv<true, false, TC>)
                           : (vc ? k_chi2_refined_dinv<false, true, TC> : k_chi2_refined_dinv<false, false, TC>);
            static std::atomic<int> attr[4][CF_MAX_DEVICES];
            int rc = cf_smem_optin(kern, 2 * 12288 * (int)sizeof(double), attr[2 * vl + vc]);
            if (rc) return rc;
            kern<<<batch * nrhs, CNT, smem, st>>>(n, L, lda, strideL, Dinv, strideD, C, ldc, strideC, X, ldx,
                                                  strideX, nrhs, chi2);
        } else {
            auto kern = vl ? (vc ? k_chi2_refined<true, true, TC> : k_chi2_refined<true, false, TC>)
                           : (vc ? k_chi2_refined<false, true, TC> : k_chi2_refined<false, false, TC>);
            static std::atomic<int> attr[4][CF_MAX_DEVICES];
            int rc = cf_smem_optin(kern, 2 * 12288 * (int)sizeof(double), attr[2 * vl + vc]);
            if (rc) return rc;
            kern<<<batch * nrhs, CNT, smem, st>>>(n, L, lda, strideL, C, ldc, strideC, X, ldx, strideX, nrhs, chi2);
        }
        CF_CHECK_LAUNCH();
    }
    if (logdet) {
        k_logdet_f32<<<batch, CNT, 0, st>>>(n, L, lda, strideL, logdet);
        CF_CHECK_LAUNCH();
    }
    return CF_OK;
}
}  // namespace

// chi2[b nrhs + m] = 2 |L_b^-1 x|^2 - v^T C_b v with v = (L_b L_b^T)^-1 x (one
// FP64 refinement step on the FP32 factor L_b of C_b), logdet[b] = 2 sum ln
// (L_b)_ii.  C: FP64 matrices (lower triangle read); X: n x nrhs (ldx),
// strideX = 0 shares it.  n <= 12288 (two FP64 vectors in shared memory).
extern "C" int cf_chi2_logdet_mixed(int n, const float* L, long lda, long strideL, const double* C, long ldc,
                                    long strideC, int batch, const double* X, long ldx, long strideX, int nrhs,
                                    double* chi2, double* logdet, void* stream)
{
    return chi2_mixed<double>(n, L, lda, strideL, C, ldc, strideC, batch, X, ldx, strideX, nrhs, chi2, logdet,
                              (cudaStream_t)stream);
}

// The same with C in FP32 (the matrices the FP32 factor was computed from, as
// the tensor-core build writes them); the refinement arithmetic stays FP64.
extern "C" int cf_chi2_logdet_mixed_c32(int n, const float* L, long lda, long strideL, const float* C, long ldc,
                                        long strideC, int batch, const double* X, long ldx, long strideX, int nrhs,
                                        double* chi2, double* logdet, void* stream)
{
    return chi2_mixed<float>(n, L, lda, strideL, C, ldc, strideC, batch, X, ldx, strideX, nrhs, chi2, logdet,
                             (cudaStream_t)stream);
}

// cf_chi2_logdet_mixed / cf_chi2_logdet_mixed_c32 with the FP32 factor's
// diagonal-block inverses as cf_potrf_f32 leaves them in its workspace (Dinv =
// the workspace, strideD = cf_potrf_f32_dinv_stride(n) floats between
// problems): 64-row blocks, each diagonal solve a block-times-vector product.
extern "C" int cf_chi2_logdet_mixed_dinv(int n, const float* L, long lda, long strideL, const float* Dinv,
                                         long strideD, const double* C, long ldc, long strideC, int batch,
                                         const double* X, long ldx, long strideX, int nrhs, double* chi2,
                                         double* logdet, void* stream)
{
    if (!Dinv) return CF_ERR_ARG;
    return chi2_mixed<double>(n, L, lda, strideL, C, ldc, strideC, batch, X, ldx, strideX, nrhs, chi2, logdet,
                              (cudaStream_t)stream, Dinv, strideD);
}

extern "C" int cf_chi2_logdet_mixed_c32_dinv(int n, const float* L, long lda, long strideL, const float* Dinv,
                                             long strideD, const float* C, long ldc, long strideC, int batch,
                                             const double* X, long ldx, long strideX, int nrhs, double* chi2,
                                             double* logdet, void* stream)
{
    if (!Dinv) return CF_ERR_ARG;
    return chi2_mixed<float>(n, L, lda, strideL, C, ldc, strideC, batch, X, ldx, strideX, nrhs, chi2, logdet,
                             (cudaStream_t)stream, Dinv, strideD);
}
