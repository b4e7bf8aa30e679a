// Plain FP64 GEMM on the FP64 tensor pipe (DMMA, mma.sync m8n8k4 f64).
//
// C = alpha * op(A) op(B) + beta * C, row-major operands, optional batch
// (blockIdx.z with element strides) and an optional second, transposed copy
// of the result (CT = C^T), which the Fisher path uses to store A_b and A_b^T
// from one pass.  This is the plain-FP64 path: the trailing updates of the
// blocked Cholesky, the triangular-solve updates, A_b = C^-1 dC_b, Y = C^-1 X.
//
// Tile 128 x 128 x 16, 8 warps (each 64 x 32 = 8 x 4 DMMA tiles), 3-stage
// cp.async pipeline.  Shared tiles keep the global orientation of each
// operand, padded so that fragment reads are bank-conflict free in both
// orientations.
#include "cf_common.cuh"

namespace {

constexpr int BM = 128, BN = 128, BK = 16, NT = 256, STAGES = 3;
constexpr int PADK = BK + 4;    // row stride of a [m][k] tile
constexpr int PADMN = BM + 4;   // row stride of a [k][m] tile

template <bool T>
struct TileShape {  // T: tile stored [k][mn] (stride PADMN), else [mn][k] (stride PADK)
    static constexpr int elems = T ? BK * PADMN : BM * PADK;
};

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    int sz = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(src), "r"(sz));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Load a BM(or BN) x BK tile of an operand into shared memory.
// TRANS == false: operand rows are the M (or N) index, columns the K index
//                 (global element (mn, k) at p[mn * ld + k]); stored [mn][k].
// TRANS == true : operand rows are K, columns M/N (element at p[k * ld + mn]);
//                 stored [k][mn].
template <bool TRANS>
__device__ __forceinline__ void load_tile(double* s, const double* p, long ld, int mn0, int k0,
                                          int MN, int K, int tid)
{
    if (!TRANS) {
#pragma unroll
        for (int it = 0; it < (BM * BK) / NT; ++it) {
            int e = it * NT + tid;
            int r = e / BK, c = e % BK;
            int gm = mn0 + r, gk = k0 + c;
            bool v = gm < MN && gk < K;
            const double* src = v ? p + (long)gm * ld + gk : p;
            cp_async8(s + r * PADK + c, src, v);
        }
    } else {
#pragma unroll
        for (int it = 0; it < (BM * BK) / NT; ++it) {
            int e = it * NT + tid;
            int r = e / BM, c = e % BM;
            int gk = k0 + r, gm = mn0 + c;
            bool v = gm < MN && gk < K;
            const double* src = v ? p + (long)gk * ld + gm : p;
            cp_async8(s + r * PADMN + c, src, v);
        }
    }
}

template <bool TRANS>
__device__ __forceinline__ double frag(const double* s, int mn, int k)
{
    return TRANS ? s[k * PADMN + mn] : s[mn * PADK + k];
}

template <bool AT, bool BT>
__global__ void __launch_bounds__(NT) k_dgemm(int M, int N, int K, double alpha, const double* A,
                                              long lda, long sA, const double* B, long ldb, long sB,
                                              double beta, double* C, long ldc, long sC, double* CT,
                                              long ldct, long sCT, float* C32, long ldc32, long sC32,
                                              int lower_only)
{
    extern __shared__ double smem[];
    // B stored [n][k] when BT (operand given N x K), else [k][n]
    constexpr bool A_KMN = AT;      // A tile orientation: [k][m]
    constexpr bool B_KMN = !BT;     // B tile orientation: [k][n]
    constexpr int SA = TileShape<A_KMN>::elems, SB = TileShape<B_KMN>::elems;
    double* sAbuf = smem;
    double* sBbuf = smem + STAGES * SA;

    const int tile_m = blockIdx.y * BM, tile_n = blockIdx.x * BN;
    if ((lower_only & 1) && tile_n > tile_m + BM - 1) return;
    // bit 3: batch entry z is row z of a symmetric block whose columns past
    // z are not needed (tiles starting right of it are skipped)
    if ((lower_only & 8) && tile_n > (int)blockIdx.z) return;
    const long bz = blockIdx.z;
    A += bz * sA;
    B += bz * sB;
    C += bz * sC;
    if (CT) CT += bz * sCT;
    if (C32) C32 += bz * sC32;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;

    double acc[8][4][2];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    int KT = (K + BK - 1) / BK;
    // lower_only bit 1: op(A) is upper triangular (op(A) = Y^T with Y lower
    // triangular, as in Y^T Y), so the K sum of a tile starts at its first row;
    // bit 2: op(A) is lower triangular, so it ends after its last row
    const int kt0 = (lower_only & 2) ? tile_m / BK : 0;
    if (lower_only & 4) {
        const int kend = (tile_m + BM + BK - 1) / BK;
        KT = kend < KT ? kend : KT;
    }
    auto issue = [&](int kt, int st) {
        if (kt < KT) {
            load_tile<A_KMN>(sAbuf + st * SA, A, lda, tile_m, kt * BK, M, K, tid);
            load_tile<B_KMN>(sBbuf + st * SB, B, ldb, tile_n, kt * BK, N, K, tid);
        }
        cp_commit();
    };
    for (int s = 0; s < STAGES - 1; ++s) issue(kt0 + s, s);

    for (int kt = kt0; kt < KT; ++kt) {
        cp_wait<STAGES - 2>();
        __syncthreads();
        issue(kt + STAGES - 1, (kt - kt0 + STAGES - 1) % STAGES);
        const double* a_s = sAbuf + ((kt - kt0) % STAGES) * SA;
        const double* b_s = sBbuf + ((kt - kt0) % STAGES) * SB;
#pragma unroll
        for (int ks = 0; ks < BK; ks += 4) {
            double af[8], bf[4];
            const int kk = ks + (lane & 3);
#pragma unroll
            for (int mi = 0; mi < 8; ++mi) af[mi] = frag<A_KMN>(a_s, wm + mi * 8 + (lane >> 2), kk);
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) bf[ni] = frag<B_KMN>(b_s, wn + ni * 8 + (lane >> 2), kk);
#pragma unroll
            for (int mi = 0; mi < 8; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) dmma(acc[mi][ni][0], acc[mi][ni][1], af[mi], bf[ni]);
        }
    }
    cp_wait<0>();

    // All reads of C first (independent loads, one latency), then the stores.
#pragma unroll
    for (int mi = 0; mi < 8; ++mi) {
        const int r = tile_m + wm + mi * 8 + (lane >> 2);
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = tile_n + wn + ni * 8 + (lane & 3) * 2 + h;
                double v = alpha * acc[mi][ni][h];
                if (beta != 0.0 && r < M && c < N) v += beta * C[(long)r * ldc + c];
                acc[mi][ni][h] = v;
            }
        }
    }
#pragma unroll
    for (int mi = 0; mi < 8; ++mi) {
        const int r = tile_m + wm + mi * 8 + (lane >> 2);
        if (r >= M) continue;
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = tile_n + wn + ni * 8 + (lane & 3) * 2 + h;
                if (c >= N) continue;
                const double v = acc[mi][ni][h];
                C[(long)r * ldc + c] = v;
                if (CT) CT[(long)c * ldct + r] = v;
                if (C32) C32[(long)r * ldc32 + c] = (float)v;
            }
        }
    }
}

template <bool AT, bool BT>
int launch(int M, int N, int K, double alpha, const double* A, long lda, long sA, const double* B,
           long ldb, long sB, double beta, double* C, long ldc, long sC, double* CT, long ldct,
           long sCT, float* C32, long ldc32, long sC32, int batch, int lower_only, cudaStream_t st)
{
    constexpr int SA = TileShape<AT>::elems, SB = TileShape<!BT>::elems;
    const size_t smem = (size_t)STAGES * (SA + SB) * sizeof(double);
    static std::atomic<int> attr[CF_MAX_DEVICES];
    if (int rc = cf_smem_optin(k_dgemm<AT, BT>, (int)smem, attr)) return rc;
    dim3 grid(cf_cdiv(N, BN), cf_cdiv(M, BM), batch);
    k_dgemm<AT, BT><<<grid, NT, smem, st>>>(M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC,
                                            CT, ldct, sCT, C32, ldc32, sC32, lower_only);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

}  // namespace

namespace {
int dgemm(int transa, int transb, int M, int N, int K, double alpha, const double* A, long lda, long strideA,
          const double* B, long ldb, long strideB, double beta, double* C, long ldc, long strideC, double* CT,
          long ldct, long strideCT, float* C32, long ldc32, long strideC32, int batch, int lower_only,
          cudaStream_t st)
{
    if (M < 0 || N < 0 || K < 0 || batch < 1 || !C) return CF_ERR_ARG;
    if (M == 0 || N == 0) return CF_OK;
    if (!transa && !transb)
        return launch<false, false>(M, N, K, alpha, A, lda, strideA, B, ldb, strideB, beta, C, ldc, strideC, CT,
                                    ldct, strideCT, C32, ldc32, strideC32, batch, lower_only, st);
    if (!transa && transb)
        return launch<false, true>(M, N, K, alpha, A, lda, strideA, B, ldb, strideB, beta, C, ldc, strideC, CT,
                                   ldct, strideCT, C32, ldc32, strideC32, batch, lower_only, st);
    if (transa && !transb)
        return launch<true, false>(M, N, K, alpha, A, lda, strideA, B, ldb, strideB, beta, C, ldc, strideC, CT,
                                   ldct, strideCT, C32, ldc32, strideC32, batch, lower_only, st);
    return launch<true, true>(M, N, K, alpha, A, lda, strideA, B, ldb, strideB, beta, C, ldc, strideC, CT, ldct,
                              strideCT, C32, ldc32, strideC32, batch, lower_only, st);
}
}  // namespace

// transa / transb: 0 = operand given in its own orientation (A: M x K,
// B: K x N), 1 = given transposed (A as K x M, B as N x K).
extern "C" int cf_dgemm(int transa, int transb, int M, int N, int K, double alpha, const double* A,
                        long lda, long strideA, const double* B, long ldb, long strideB, double beta,
                        double* C, long ldc, long strideC, double* CT, long ldct, long strideCT,
                        int batch, int lower_only, void* stream)
{
    return dgemm(transa, transb, M, N, K, alpha, A, lda, strideA, B, ldb, strideB, beta, C, ldc, strideC, CT, ldct,
                 strideCT, nullptr, 0, 0, batch, lower_only, (cudaStream_t)stream);
}

// cf_dgemm with a rounded FP32 copy of the result (C32, row stride ldc32,
// batch stride strideC32) written from the same epilogue instead of CT.
extern "C" int cf_dgemm_f32copy(int transa, int transb, int M, int N, int K, double alpha, const double* A,
                                long lda, long strideA, const double* B, long ldb, long strideB, double beta,
                                double* C, long ldc, long strideC, float* C32, long ldc32, long strideC32,
                                int batch, int lower_only, void* stream)
{
    return dgemm(transa, transb, M, N, K, alpha, A, lda, strideA, B, ldb, strideB, beta, C, ldc, strideC, nullptr,
                 0, 0, C32, ldc32, strideC32, batch, lower_only, (cudaStream_t)stream);
}
