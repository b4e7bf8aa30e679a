// Blocked FP64 Cholesky, triangular inverse and SPD inverse (batched).
//
// Restates the reference's matrix_inverse_symm (cosmocore/basics/linalg.py:
// 152-219): Jacobi scaling D M D with D = diag(|M_ii|^-1/2), Cholesky, inverse
// from the factor, unscaling D (.) D.  The factorisation is right-looking with
// 64-wide panels: one CTA factors the diagonal block and inverts its factor
// (potrf_diag.cuh), the panel below is a DMMA GEMM against that inverse, and
// the trailing update is a lower-only DMMA GEMM.  The inverse solves L Y = I block row by block row (an in-place
// triangular solve per diagonal block plus a DMMA GEMM update), then forms
// C^-1 = Y^T Y with one lower-only GEMM.  Per-problem status `info` follows
// LAPACK: 0 = success, k > 0 = the leading minor of order k is not positive.
#include "cf_common.cuh"
#include "potrf_diag.cuh"

#include <mutex>

extern "C" int cf_dgemm(int transa, int transb, int M, int N, int K, double alpha, const double* A,
                        long lda, long strideA, const double* B, long ldb, long strideB, double beta,
                        double* C, long ldc, long strideC, double* CT, long ldct, long strideCT,
                        int batch, int lower_only, void* stream);

namespace {

constexpr int NB = cf_diag::NB;

using cf_diag::k_potrf_diag_inv;

// Batched 2D copy: dst[r * ldd + c] = src[r * lds + c], r < R, c < C.
__global__ void k_copy2d(int R, int C, const double* src, long lds, long ss, double* dst, long ldd, long sd)
{
    src += blockIdx.z * ss;
    dst += blockIdx.z * sd;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r < R && c < C) dst[(long)r * ldd + c] = src[(long)r * lds + c];
}

__global__ void k_diag_scale(const double* A, long lda, long sA, int n, double* d, long sd)
{
    A += blockIdx.y * sA;
    d += blockIdx.y * sd;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double v = fabs(A[(long)i * lda + i]);
        if (v == 0.0) v = 1.0;
        d[i] = 1.0 / sqrt(v);
    }
}

// A[r, c] *= d[r] d[c] (lower triangle only when lower != 0).
__global__ void k_scale_sym(double* A, long lda, long sA, int n, const double* d, long sd, int lower)
{
    A += blockIdx.z * sA;
    d += blockIdx.z * sd;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r < n && c < n && (!lower || c <= r)) A[(long)r * lda + c] *= d[r] * d[c];
}

// Full symmetric result from the lower triangle, with the Jacobi unscaling.
__global__ void k_unscale_mirror(double* A, long lda, long sA, int n, const double* d, long sd)
{
    A += blockIdx.z * sA;
    d += blockIdx.z * sd;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r < n && c < r) {
        double v = A[(long)r * lda + c] * d[r] * d[c];
        A[(long)r * lda + c] = v;
        A[(long)c * lda + r] = v;
    } else if (r < n && c == r) {
        A[(long)r * lda + c] *= d[r] * d[r];
    }
}

}  // namespace

namespace {
inline int nblocks(int n) { return (n + NB - 1) / NB; }
// doubles of potrf workspace per problem: every diagonal-block inverse + one
// double-width panel (two 64-column panels side by side)
inline size_t potrf_ws(int n) { return (size_t)nblocks(n) * NB * NB + (size_t)n * 2 * NB; }
// A single matrix above this order is factored with a look-ahead (a second
// panel buffer, the bulk of each trailing update on a second stream).
constexpr int LOOKAHEAD_MIN_N = 1024;
inline bool use_lookahead(int n, int batch) { return batch == 1 && n > LOOKAHEAD_MIN_N; }
inline size_t potrf_ws_total(int n, int batch)
{
    return potrf_ws(n) * (size_t)batch + (use_lookahead(n, batch) ? (size_t)n * 2 * NB : 0);
}

// Per-device side stream (highest priority: it carries the factorisation's
// critical path) and the events of the look-ahead fork / join.  The mutex
// keeps one caller's event records from interleaving with another's.
struct Lookahead {
    std::mutex mu;
    bool ready = false;
    cudaStream_t chain = nullptr;
    cudaEvent_t fork = nullptr, panel = nullptr, bulk = nullptr, join = nullptr;
};
Lookahead g_la[CF_MAX_DEVICES];

int lookahead_state(Lookahead** out)
{
    int dev = -1;
    CF_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= CF_MAX_DEVICES) return CF_ERR_UNSUPPORTED;
    Lookahead& la = g_la[dev];
    *out = &la;
    return CF_OK;
}

int lookahead_init(Lookahead& la)
{
    if (la.ready) return CF_OK;
    int least = 0, greatest = 0;
    CF_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CF_CHECK(cudaStreamCreateWithPriority(&la.chain, cudaStreamNonBlocking, greatest));
    for (cudaEvent_t* e : {&la.fork, &la.panel, &la.bulk, &la.join})
        CF_CHECK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    la.ready = true;
    return CF_OK;
}
}  // namespace

extern "C" size_t cf_potrf_workspace(int n, int batch) { return potrf_ws_total(n, batch) * sizeof(double); }

// Doubles between consecutive problems' diagonal-block inverses in the potrf
// workspace (block j of a problem at work + z stride + j 64^2).
extern "C" size_t cf_potrf_dinv_stride(int n) { return potrf_ws(n); }

namespace {
// One 128-column step of the factorisation up to the trailing update: factor
// the two diagonal blocks (keeping their inverses), solve both panels into W
// and write them back.  Returns the K = 128 panel W2 the trailing update
// A22 -= W2 W2^T needs through *w2 (nullptr when no trailing matrix is left).
int potrf_step(int n, int k0, double* A, long lda, long strideA, int batch, double* Dinv, int blk, double* W,
               long ws, int* info, cudaStream_t st, const double** w2, int* rest2_out)
{
    constexpr size_t DIAG_SMEM = cf_diag::smem_bytes<double>();
    constexpr int LDW = 2 * NB;
    void* stream = (void*)st;
    *w2 = nullptr;
    *rest2_out = 0;
    const int kb1 = n - k0 < NB ? n - k0 : NB;
    double* D1 = Dinv + (long)blk * NB * NB;
    k_potrf_diag_inv<double><<<batch, cf_diag::NTHREADS, DIAG_SMEM, st>>>(A, lda, strideA, k0, kb1, D1, ws, info);
    CF_CHECK_LAUNCH();
    const int rest1 = n - k0 - kb1;
    if (rest1 <= 0) return CF_OK;
    double* a21_1 = A + (long)(k0 + kb1) * lda + k0;
    // T1 = A21 L11^-T into W[:, 0:kb1]
    int rc = cf_dgemm(0, 1, rest1, kb1, kb1, 1.0, a21_1, lda, strideA, D1, kb1, ws, 0.0, W, LDW, ws, nullptr, 0, 0,
                      batch, 0, stream);
    if (rc) return rc;
    const int kb2 = rest1 < NB ? rest1 : NB;
    // panel 2's columns, every row below panel 1: A -= T1 T1[0:kb2]^T
    rc = cf_dgemm(0, 1, rest1, kb2, kb1, -1.0, W, LDW, ws, W, LDW, ws, 1.0, a21_1 + kb1, lda, strideA, nullptr, 0, 0,
                  batch, 0, stream);
    if (rc) return rc;
    k_copy2d<<<dim3(cf_cdiv(kb1, 32), cf_cdiv(rest1, 8), batch), dim3(32, 8), 0, st>>>(rest1, kb1, W, LDW, ws, a21_1,
                                                                                      lda, strideA);
    CF_CHECK_LAUNCH();
    const int k1 = k0 + kb1;
    double* D2 = Dinv + (long)(blk + 1) * NB * NB;
    k_potrf_diag_inv<double><<<batch, cf_diag::NTHREADS, DIAG_SMEM, st>>>(A, lda, strideA, k1, kb2, D2, ws, info);
    CF_CHECK_LAUNCH();
    const int rest2 = rest1 - kb2;
    if (rest2 <= 0) return CF_OK;
    double* a21_2 = A + (long)(k1 + kb2) * lda + k1;
    double* W2 = W + (long)kb2 * LDW;  // rows of W at and below the trailing matrix
    // T2 = A21_2 L22^-T into W[kb2:, kb1:kb1+kb2]
    rc = cf_dgemm(0, 1, rest2, kb2, kb2, 1.0, a21_2, lda, strideA, D2, kb2, ws, 0.0, W2 + kb1, LDW, ws, nullptr, 0, 0,
                  batch, 0, stream);
    if (rc) return rc;
    k_copy2d<<<dim3(cf_cdiv(kb2, 32), cf_cdiv(rest2, 8), batch), dim3(32, 8), 0, st>>>(rest2, kb2, W2 + kb1, LDW, ws,
                                                                                      a21_2, lda, strideA);
    CF_CHECK_LAUNCH();
    *w2 = W2;
    *rest2_out = rest2;
    return CF_OK;
}
}  // namespace

// Right-looking blocked Cholesky: per 64-wide panel, the diagonal block is
// factored (and inverted) by one CTA and the panel below is L21 = A21 L11^-T
// (DMMA GEMM against the inverted block); panels go in pairs so that the
// trailing update A22 -= L21 L21^T (lower-only DMMA GEMM) runs once per 128
// columns.  `work` holds cf_potrf_workspace(n, batch) bytes and keeps every
// L11^-1 for cf_trtri_lower.
//
// A single matrix of order above 1024 is factored with a look-ahead: the
// next step's 128 columns of each trailing update go first, on a
// high-priority side stream that carries the whole critical path (diagonal
// blocks, panels, those columns), while the rest of the update (the bulk of
// the FLOPs) runs on the caller's stream; two panel buffers alternate so a
// step's panels never overwrite the ones the previous bulk update still
// reads.  The side stream forks from and joins the caller's stream through
// events, so the routine stays stream-ordered and capturable.
extern "C" int cf_potrf(int n, double* A, long lda, long strideA, int batch, void* work, int* info, void* stream)
{
    if (n <= 0 || batch < 1 || !A || !work) return CF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    constexpr size_t DIAG_SMEM = cf_diag::smem_bytes<double>();
    static std::atomic<int> attr[CF_MAX_DEVICES];
    if (int rc0 = cf_smem_optin(k_potrf_diag_inv<double>, (int)DIAG_SMEM, attr)) return rc0;
    const long ws = (long)potrf_ws(n);
    double* Dinv = (double*)work;                   // [batch][nblocks][NB][NB]
    double* W = Dinv + (long)nblocks(n) * NB * NB;  // [batch][n][2 NB] (same stride ws)
    constexpr int LDW = 2 * NB;
    if (!use_lookahead(n, batch)) {
        int blk = 0;
        for (int k0 = 0; k0 < n; k0 += 2 * NB, blk += 2) {
            const double* W2 = nullptr;
            int rest2 = 0;
            int rc = potrf_step(n, k0, A, lda, strideA, batch, Dinv, blk, W, ws, info, st, &W2, &rest2);
            if (rc) return rc;
            if (!W2) break;
            double* a22 = A + (long)(k0 + 2 * NB) * (lda + 1);
            rc = cf_dgemm(0, 1, rest2, rest2, 2 * NB, -1.0, W2, LDW, ws, W2, LDW, ws, 1.0, a22, lda, strideA, nullptr,
                          0, 0, batch, 1, stream);
            if (rc) return rc;
        }
        return CF_OK;
    }
    Lookahead* la = nullptr;
    if (int rc = lookahead_state(&la)) return rc;
    std::lock_guard<std::mutex> lock(la->mu);
    if (int rc = lookahead_init(*la)) return rc;
    cudaStream_t ch = la->chain;
    double* Wbuf[2] = {W, W + (long)n * LDW};  // the second buffer follows the first problem's workspace
    CF_CHECK(cudaEventRecord(la->fork, st));
    CF_CHECK(cudaStreamWaitEvent(ch, la->fork, 0));
    int rc = CF_OK;
    bool bulk_pending = false;
    int blk = 0;
    for (int k0 = 0, it = 0; k0 < n && rc == CF_OK; k0 += 2 * NB, blk += 2, ++it) {
        const double* W2 = nullptr;
        int rest2 = 0;
        rc = potrf_step(n, k0, A, lda, strideA, 1, Dinv, blk, Wbuf[it & 1], ws, info, ch, &W2, &rest2);
        if (rc || !W2) break;
        // every earlier update of the next step's columns is done before they are updated again
        if (bulk_pending) {
            if (cudaStreamWaitEvent(ch, la->bulk, 0) != cudaSuccess) {
                rc = CF_ERR_CUDA;
                break;
            }
        }
        double* a22 = A + (long)(k0 + 2 * NB) * (lda + 1);
        const int nn = rest2 < 2 * NB ? rest2 : 2 * NB;
        // the next step's columns, every row below: critical path
        rc = cf_dgemm(0, 1, rest2, nn, 2 * NB, -1.0, W2, LDW, 0, W2, LDW, 0, 1.0, a22, lda, 0, nullptr, 0, 0, 1, 1,
                      (void*)ch);
        if (rc) break;
        const int rest3 = rest2 - nn;
        if (rest3 > 0) {
            // the rest of the trailing matrix on the caller's stream
            if (cudaEventRecord(la->panel, ch) != cudaSuccess || cudaStreamWaitEvent(st, la->panel, 0) != cudaSuccess) {
                rc = CF_ERR_CUDA;
                break;
            }
            const double* w3 = W2 + (long)nn * LDW;
            rc = cf_dgemm(0, 1, rest3, rest3, 2 * NB, -1.0, w3, LDW, 0, w3, LDW, 0, 1.0, a22 + (long)nn * (lda + 1),
                          lda, 0, nullptr, 0, 0, 1, 1, stream);
            if (rc) break;
            if (cudaEventRecord(la->bulk, st) != cudaSuccess) {
                rc = CF_ERR_CUDA;
                break;
            }
            bulk_pending = true;
        } else {
            bulk_pending = false;
        }
    }
    // join: the caller's stream waits for the side stream's last work (on every path)
    const cudaError_t e1 = cudaEventRecord(la->join, ch);
    const cudaError_t e2 = cudaStreamWaitEvent(st, la->join, 0);
    if (rc) return rc;
    if (e1 != cudaSuccess || e2 != cudaSuccess) return CF_ERR_CUDA;
    return CF_OK;
}

namespace {
// dst[r * ld + c] = v for r < R, c < C; batch (or pair) z advances dst by sd.
__global__ void k_fill2d(int R, int C, double* dst, long ld, long sd, double v)
{
    dst += blockIdx.z * sd;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r < R && c < C) dst[(long)r * ld + c] = v;
}

// Y's diagonal 64-blocks <- the inverses cf_potrf left in `work`
// (block b: kb x kb row-major at Dinv + b NB^2); grid (blocks, batch).
__global__ void k_place_diag_inv(const double* Dinv, long sD, int n, double* Y, long ldy, long sY)
{
    const int blk = blockIdx.x;
    Y += blockIdx.y * sY;
    Dinv += blockIdx.y * sD + (long)blk * NB * NB;
    const int k0 = blk * NB, kb = n - k0 < NB ? n - k0 : NB;
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) {
        const int r = e / kb, c = e - (e / kb) * kb;
        Y[(long)(k0 + r) * ldy + k0 + c] = Dinv[r * kb + c];
    }
}

// One merge step for `np` pairs of adjacent diagonal blocks (sizes s and s2)
// whose inverses Y11, Y22 are in place: Y21 = -Y22 L21 Y11.  The first pair's
// leading block starts at row / column c0; pairs are 2 s apart.  T^T =
// Y11^T L21^T is staged in the (still zero) upper block of the pair and
// cleared afterwards, so Y stays lower triangular.
int merge_pairs(int s, int s2, int np, long c0, const double* L, long lda, long sL, double* Y, long ldy, long sY,
                int batch, cudaStream_t st, void* stream)
{
    const long r0 = c0 + s;
    const long pL = 2L * s * (lda + 1), pY = 2L * s * (ldy + 1);
    // batch over pairs for one problem, or over problems pair by pair
    const int outer = batch == 1 ? 1 : np;
    const int inner = batch == 1 ? np : batch;
    const long iL = batch == 1 ? pL : sL, iY = batch == 1 ? pY : sY;
    for (int o = 0; o < outer; ++o) {
        const double* l21 = L + (r0 + (long)o * 2 * s) * lda + c0 + (long)o * 2 * s;
        double* y11 = Y + (c0 + (long)o * 2 * s) * (ldy + 1);
        double* y22 = Y + (r0 + (long)o * 2 * s) * (ldy + 1);
        double* tt = y11 + s;            // upper block (rows of block 1, columns of block 2)
        double* y21 = y22 - s;           // lower block (rows of block 2, columns of block 1)
        int rc = cf_dgemm(1, 1, s, s2, s, 1.0, y11, ldy, iY, l21, lda, iL, 0.0, tt, ldy, iY, nullptr, 0, 0, inner,
                          2, stream);
        if (rc) return rc;
        rc = cf_dgemm(0, 1, s2, s, s2, -1.0, y22, ldy, iY, tt, ldy, iY, 0.0, y21, ldy, iY, nullptr, 0, 0, inner, 4,
                      stream);
        if (rc) return rc;
        k_fill2d<<<dim3(cf_cdiv(s2, 32), cf_cdiv(s, 8), inner), dim3(32, 8), 0, st>>>(s, s2, tt, ldy, iY, 0.0);
        CF_CHECK_LAUNCH();
    }
    return CF_OK;
}
}  // namespace

// Y = L^-1 for the lower factor of cf_potrf, using the diagonal-block
// inverses it left in `work`: the 64-blocks are placed on Y's diagonal, then
// adjacent blocks are merged pairwise, level by level (64, 128, 256, ...):
// [[Y11, 0], [Y21, Y22]] with Y21 = -Y22 L21 Y11.  Every merge of a level is
// independent, so a level is two batched DMMA GEMMs that skip the triangular
// zeros of Y11 and Y22 (log2(n / 64) levels instead of n / 64 dependent
// block steps).
extern "C" int cf_trtri_lower(int n, const double* L, long lda, long strideL, double* Y, long ldy, long strideY,
                              int batch, void* work, void* stream)
{
    if (n <= 0 || batch < 1 || !L || !Y || !work) return CF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const long ws = (long)potrf_ws(n);
    const double* Dinv = (const double*)work;
    k_fill2d<<<dim3(cf_cdiv(n, 32), cf_cdiv(n, 8), batch), dim3(32, 8), 0, st>>>(n, n, Y, ldy, strideY, 0.0);
    CF_CHECK_LAUNCH();
    k_place_diag_inv<<<dim3(nblocks(n), batch), 256, 0, st>>>(Dinv, ws, n, Y, ldy, strideY);
    CF_CHECK_LAUNCH();
    for (long s = NB; s < n; s *= 2) {
        const int nfull = (int)(n / s), rem = (int)(n % s);
        if (nfull / 2 > 0) {
            int rc = merge_pairs((int)s, (int)s, nfull / 2, 0, L, lda, strideL, Y, ldy, strideY, batch, st, stream);
            if (rc) return rc;
        }
        if ((nfull & 1) && rem > 0) {  // the last full block with the partial one after it
            int rc = merge_pairs((int)s, rem, 1, (long)(nfull - 1) * s, L, lda, strideL, Y, ldy, strideY, batch, st,
                                 stream);
            if (rc) return rc;
        }
    }
    return CF_OK;
}

extern "C" size_t cf_spd_inverse_workspace(int n, int batch)
{
    return (((size_t)n * n + (size_t)n) * (size_t)batch + potrf_ws_total(n, batch)) * sizeof(double);
}

// In place inverse of symmetric positive-definite matrices (row-major,
// n x n, batch of them `strideA` doubles apart).  `work` must hold
// cf_spd_inverse_workspace(n, batch) bytes; `info` one int per problem,
// zeroed by the caller.
extern "C" int cf_spd_inverse(int n, double* A, long lda, long strideA, int batch, void* work, int* info,
                              void* stream)
{
    if (n <= 0 || batch < 1 || !A || !work) return CF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    double* Y = (double*)work;
    const long sY = (long)n * n;
    double* d = Y + sY * batch;
    double* pw = d + (long)n * batch;
    dim3 b2(32, 8);
    dim3 g2(cf_cdiv(n, 32), cf_cdiv(n, 8), batch);
    k_diag_scale<<<dim3(cf_cdiv(n, 256), batch), 256, 0, st>>>(A, lda, strideA, n, d, n);
    CF_CHECK_LAUNCH();
    k_scale_sym<<<g2, b2, 0, st>>>(A, lda, strideA, n, d, n, 1);
    CF_CHECK_LAUNCH();
    int rc = cf_potrf(n, A, lda, strideA, batch, pw, info, stream);
    if (rc) return rc;
    rc = cf_trtri_lower(n, A, lda, strideA, Y, n, sY, batch, pw, stream);
    if (rc) return rc;
    // C^-1 = Y^T Y; Y is lower triangular, so (Y^T Y)[r, c] sums k >= max(r, c)
    rc = cf_dgemm(1, 0, n, n, n, 1.0, Y, n, sY, Y, n, sY, 0.0, A, lda, strideA, nullptr, 0, 0, batch, 3, stream);
    if (rc) return rc;
    k_unscale_mirror<<<g2, b2, 0, st>>>(A, lda, strideA, n, d, n);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of cf_spd_inverse for callers that must not
// allocate device memory where they need the inverse: allocator hooks,
// plugins whose host application owns the memory pool and forbids allocations
// after start-up, integrations that must not fragment a pool they do not own.
// It launches kernels, so it is not for use inside a host callback, where CUDA
// calls are not permitted.  Its workspace (L^-1, the Jacobi scale factors, the
// diagonal-block inverses and one panel) lives in this file-scope array: a
// device allocates it when this module is first used there (lazy module
// loading) and holds it until the process exits, 1.25 M doubles = 10.0 MB.
#define CF_SPD_STATIC_MAX_N 1024
static __device__ __align__(256) double g_spd_static_scratch[(size_t)CF_SPD_STATIC_MAX_N * CF_SPD_STATIC_MAX_N +
                                                             CF_SPD_STATIC_MAX_N +
                                                             (size_t)((CF_SPD_STATIC_MAX_N + NB - 1) / NB) * NB * NB +
                                                             (size_t)CF_SPD_STATIC_MAX_N * 2 * NB];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
double* g_static_ptr[kMaxDevices] = {};

// Device address of the scratch array for the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device with that device current and cached.
int static_scratch(double** out)
{
    int dev = -1;
    CF_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return CF_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (g_static_ptr[dev] == nullptr) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_spd_static_scratch);
        if (e != cudaSuccess || p == nullptr) {
            (void)cudaGetLastError();  // do not leave the error for an unrelated later launch check
            return CF_ERR_CUDA;
        }
        g_static_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_static_ptr[dev];
    return CF_OK;
}
}  // namespace

extern "C" int cf_spd_inverse_static_max_n(void) { return CF_SPD_STATIC_MAX_N; }

// Same result as cf_spd_inverse(n, A, lda, n*n, 1, work, info, stream) with no
// caller workspace and no allocation.  The first call on a device looks up the
// scratch address and sets kernel attributes: make it at start-up, outside
// the no-allocation context and before any stream capture.  All calls share one
// scratch array: calls whose work overlaps on the GPU (different streams or
// host threads on the same device) race.  Every scratch element the routine
// reads is written by it first, so stale contents from a previous call do not
// matter; *info is set to 0 on the stream before the factorisation.
extern "C" int cf_spd_inverse_static(int n, double* A, long lda, int* info, void* stream)
{
    if (n <= 0 || !A || !info || lda < n) return CF_ERR_ARG;
    if (n > CF_SPD_STATIC_MAX_N) return CF_ERR_TOO_LARGE;
    double* work = nullptr;
    int rc = static_scratch(&work);
    if (rc) return rc;
    CF_CHECK(cudaMemsetAsync(info, 0, sizeof(int), (cudaStream_t)stream));
    return cf_spd_inverse(n, A, lda, (long)n * n, 1, work, info, stream);
}
