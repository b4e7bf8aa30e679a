// Blocked FP64 Cholesky, triangular inverse and SPD inverse (batched).
//
// Restates the reference's matrix_inverse_symm (cosmocore/basics/linalg.py:
// 152-219): Jacobi scaling D M D with D = diag(|M_ii|^-1/2), Cholesky, inverse
// from the factor, unscaling D (.) D.  The factorisation is right-looking with
// 64-wide panels: one CTA factors the diagonal block, a row-parallel kernel
// solves the panel below it, and the trailing update is a lower-only DMMA
// GEMM.  The inverse solves L Y = I block row by block row (an in-place
// triangular solve per diagonal block plus a DMMA GEMM update), then forms
// C^-1 = Y^T Y with one lower-only GEMM.  Per-problem status `info` follows
// LAPACK: 0 = success, k > 0 = the leading minor of order k is not positive.
#include "cf_common.cuh"

#include <mutex>

extern "C" int cf_dgemm(int transa, int transb, int M, int N, int K, double alpha, const double* A,
                        long lda, long strideA, const double* B, long ldb, long strideB, double beta,
                        double* C, long ldc, long strideC, double* CT, long ldct, long strideCT,
                        int batch, int lower_only, void* stream);

namespace {

constexpr int NB = 64;
constexpr int LDS = NB + 1;

// Factor the kb x kb diagonal block at (k0, k0) of each batch matrix in place.
__global__ void __launch_bounds__(256) k_potrf_diag(double* A, long lda, long sA, int k0, int kb, int* info)
{
    __shared__ double S[NB * LDS];
    __shared__ int bad;
    A += blockIdx.x * sA;
    const int tid = threadIdx.x;
    for (int e = tid; e < kb * kb; e += blockDim.x) {
        int r = e / kb, c = e % kb;
        S[r * LDS + c] = (c <= r) ? A[(long)(k0 + r) * lda + k0 + c] : 0.0;
    }
    if (tid == 0) bad = 0;
    __syncthreads();
    for (int j = 0; j < kb; ++j) {
        if (tid == 0) {
            double d = S[j * LDS + j];
            if (!(d > 0.0)) {  // also catches NaN
                if (!bad) bad = k0 + j + 1;
                d = 1.0;
            }
            S[j * LDS + j] = sqrt(d);
        }
        __syncthreads();
        const double piv = S[j * LDS + j];
        for (int r = j + 1 + tid; r < kb; r += blockDim.x) S[r * LDS + j] /= piv;
        __syncthreads();
        const int m = kb - j - 1;
        for (int e = tid; e < m * m; e += blockDim.x) {
            int r = j + 1 + e / m, c = j + 1 + e % m;
            if (c <= r) S[r * LDS + c] -= S[r * LDS + j] * S[c * LDS + j];
        }
        __syncthreads();
    }
    for (int e = tid; e < kb * kb; e += blockDim.x) {
        int r = e / kb, c = e % kb;
        A[(long)(k0 + r) * lda + k0 + c] = (c <= r) ? S[r * LDS + c] : 0.0;
    }
    if (tid == 0 && bad && info && info[blockIdx.x] == 0) info[blockIdx.x] = bad;
}

// Panel below the diagonal block: A21 <- A21 L11^-T (one thread per row).
__global__ void __launch_bounds__(NB) k_trsm_panel(double* A, long lda, long sA, int k0, int kb, int n)
{
    extern __shared__ double dsm[];
    double* Ls = dsm;
    double* Xs = dsm + NB * LDS;
    A += blockIdx.y * sA;
    const int tid = threadIdx.x;
    const int r0 = k0 + kb + blockIdx.x * NB;
    for (int e = tid; e < kb * kb; e += NB) {
        int r = e / kb, c = e % kb;
        Ls[r * LDS + c] = A[(long)(k0 + r) * lda + k0 + c];
    }
    for (int e = tid; e < NB * kb; e += NB) {
        int r = e / kb, c = e % kb;
        Xs[r * LDS + c] = (r0 + r < n) ? A[(long)(r0 + r) * lda + k0 + c] : 0.0;
    }
    __syncthreads();
    if (r0 + tid < n) {
        double* x = Xs + tid * LDS;
        for (int c = 0; c < kb; ++c) {
            double s = x[c];
            for (int t = 0; t < c; ++t) s -= x[t] * Ls[c * LDS + t];
            x[c] = s / Ls[c * LDS + c];
        }
    }
    __syncthreads();
    for (int e = tid; e < NB * kb; e += NB) {
        int r = e / kb, c = e % kb;
        if (r0 + r < n) A[(long)(r0 + r) * lda + k0 + c] = Xs[r * LDS + c];
    }
}

// In place Y[k0:k0+kb, 0:ncols] <- L11^-1 Y[k0:k0+kb, 0:ncols] (one thread per column).
__global__ void __launch_bounds__(NB) k_trsm_left(const double* L, long lda, long sL, int k0, int kb,
                                                  double* Y, long ldy, long sY, int ncols)
{
    extern __shared__ double dsm[];
    double* Ls = dsm;
    double* Xs = dsm + NB * LDS;
    L += blockIdx.y * sL;
    Y += blockIdx.y * sY;
    const int tid = threadIdx.x;
    const int c0 = blockIdx.x * NB;
    for (int e = tid; e < kb * kb; e += NB) {
        int r = e / kb, c = e % kb;
        Ls[r * LDS + c] = L[(long)(k0 + r) * lda + k0 + c];
    }
    for (int e = tid; e < kb * NB; e += NB) {
        int r = e / NB, c = e % NB;
        Xs[r * LDS + c] = (c0 + c < ncols) ? Y[(long)(k0 + r) * ldy + c0 + c] : 0.0;
    }
    __syncthreads();
    for (int r = 0; r < kb; ++r) {
        double s = Xs[r * LDS + tid];
        for (int t = 0; t < r; ++t) s -= Ls[r * LDS + t] * Xs[t * LDS + tid];
        Xs[r * LDS + tid] = s / Ls[r * LDS + r];
    }
    __syncthreads();
    for (int e = tid; e < kb * NB; e += NB) {
        int r = e / NB, c = e % NB;
        if (c0 + c < ncols) Y[(long)(k0 + r) * ldy + c0 + c] = Xs[r * LDS + c];
    }
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

__global__ void k_set_identity(double* Y, long ldy, long sY, int n)
{
    Y += blockIdx.z * sY;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    int r = blockIdx.y * blockDim.y + threadIdx.y;
    if (r < n && c < n) Y[(long)r * ldy + c] = (r == c) ? 1.0 : 0.0;
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

constexpr size_t TRSM_SMEM = 2 * NB * LDS * sizeof(double);

int set_trsm_attrs()
{
    static bool done = false;
    if (!done) {
        CF_CHECK(cudaFuncSetAttribute(k_trsm_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRSM_SMEM));
        CF_CHECK(cudaFuncSetAttribute(k_trsm_left, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRSM_SMEM));
        done = true;
    }
    return CF_OK;
}

}  // namespace

extern "C" int cf_potrf(int n, double* A, long lda, long strideA, int batch, int* info, void* stream)
{
    if (n <= 0 || batch < 1 || !A) return CF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (int rc = set_trsm_attrs()) return rc;
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int kb = n - k0 < NB ? n - k0 : NB;
        k_potrf_diag<<<batch, 256, 0, st>>>(A, lda, strideA, k0, kb, info);
        CF_CHECK_LAUNCH();
        const int rest = n - k0 - kb;
        if (rest > 0) {
            k_trsm_panel<<<dim3(cf_cdiv(rest, NB), batch), NB, TRSM_SMEM, st>>>(A, lda, strideA, k0, kb, n);
            CF_CHECK_LAUNCH();
            double* a21 = A + (long)(k0 + kb) * lda + k0;
            int rc = cf_dgemm(0, 1, rest, rest, kb, -1.0, a21, lda, strideA, a21, lda, strideA, 1.0,
                              a21 + kb, lda, strideA, nullptr, 0, 0, batch, 1, stream);
            if (rc) return rc;
        }
    }
    return CF_OK;
}

// Y = L^-1 for a lower factor L (both n x n, row-major).
extern "C" int cf_trtri_lower(int n, const double* L, long lda, long strideL, double* Y, long ldy,
                              long strideY, int batch, void* stream)
{
    if (n <= 0 || batch < 1 || !L || !Y) return CF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (int rc = set_trsm_attrs()) return rc;
    dim3 b2(32, 8);
    k_set_identity<<<dim3(cf_cdiv(n, 32), cf_cdiv(n, 8), batch), b2, 0, st>>>(Y, ldy, strideY, n);
    CF_CHECK_LAUNCH();
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int kb = n - k0 < NB ? n - k0 : NB;
        const int ncols = k0 + kb;
        k_trsm_left<<<dim3(cf_cdiv(ncols, NB), batch), NB, TRSM_SMEM, st>>>(L, lda, strideL, k0, kb, Y, ldy,
                                                                    strideY, ncols);
        CF_CHECK_LAUNCH();
        const int rest = n - k0 - kb;
        if (rest > 0) {
            int rc = cf_dgemm(0, 0, rest, ncols, kb, -1.0, L + (long)(k0 + kb) * lda + k0, lda,
                              strideL, Y + (long)k0 * ldy, ldy, strideY, 1.0,
                              Y + (long)(k0 + kb) * ldy, ldy, strideY, nullptr, 0, 0, batch, 0, stream);
            if (rc) return rc;
        }
    }
    return CF_OK;
}

extern "C" size_t cf_spd_inverse_workspace(int n, int batch)
{
    return ((size_t)n * n + (size_t)n) * sizeof(double) * (size_t)batch;
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
    dim3 b2(32, 8);
    dim3 g2(cf_cdiv(n, 32), cf_cdiv(n, 8), batch);
    k_diag_scale<<<dim3(cf_cdiv(n, 256), batch), 256, 0, st>>>(A, lda, strideA, n, d, n);
    CF_CHECK_LAUNCH();
    k_scale_sym<<<g2, b2, 0, st>>>(A, lda, strideA, n, d, n, 1);
    CF_CHECK_LAUNCH();
    int rc = cf_potrf(n, A, lda, strideA, batch, info, stream);
    if (rc) return rc;
    rc = cf_trtri_lower(n, A, lda, strideA, Y, n, sY, batch, stream);
    if (rc) return rc;
    rc = cf_dgemm(1, 0, n, n, n, 1.0, Y, n, sY, Y, n, sY, 0.0, A, lda, strideA, nullptr, 0, 0, batch, 1,
                  stream);
    if (rc) return rc;
    k_unscale_mirror<<<g2, b2, 0, st>>>(A, lda, strideA, n, d, n);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of cf_spd_inverse for callers that cannot allocate
// device memory: code running inside a host callback or a custom allocator's
// own hooks, plugins whose host forbids cudaMalloc after start-up, or
// integrations that must not fragment a pool they do not own.  Its workspace
// (L^-1 and the Jacobi scale factors) lives in this file-scope array, which
// every GPU that loads the library holds until the process exits:
// (1024^2 + 1024) doubles = 8.4 MB per device.
#define CF_SPD_STATIC_MAX_N 1024
static __device__ __align__(256) double g_spd_static_scratch[(size_t)CF_SPD_STATIC_MAX_N * CF_SPD_STATIC_MAX_N +
                                                             CF_SPD_STATIC_MAX_N];

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
        if (e != cudaSuccess || p == nullptr) return CF_ERR_CUDA;
        g_static_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_static_ptr[dev];
    return CF_OK;
}
}  // namespace

extern "C" int cf_spd_inverse_static_max_n(void) { return CF_SPD_STATIC_MAX_N; }

// Same result as cf_spd_inverse(n, A, lda, n*n, 1, work, info, stream) with no
// caller workspace and no allocation.  The first call on a device looks up the
// scratch address (make it before any stream capture).  All calls share one
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
