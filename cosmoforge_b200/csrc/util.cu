// Small elementwise helpers for the device path.
#include "cf_common.cuh"

namespace {

// Z_b = a X_b + c W   (W shared across the batch when sW == 0)
__global__ void k_axpby(long count, double a, const double* X, long sX, double c, const double* cvec,
                        const double* W, long sW, double* Z, long sZ)
{
    const long b = blockIdx.y;
    const double cb = cvec ? cvec[b] : c;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
        double v = a * X[b * sX + i];
        if (W) v += cb * W[b * sW + i];
        Z[b * sZ + i] = v;
    }
}

// B[c, r] = A[r, c] for an R x C row-major tile walk through shared memory.
__global__ void k_transpose(int R, int C, const double* A, long lda, double* B, long ldb)
{
    __shared__ double t[32][33];
    int c = blockIdx.x * 32 + threadIdx.x;
    int r = blockIdx.y * 32 + threadIdx.y;
    for (int k = 0; k < 32; k += 8)
        if (r + k < R && c < C) t[threadIdx.y + k][threadIdx.x] = A[(long)(r + k) * lda + c];
    __syncthreads();
    c = blockIdx.y * 32 + threadIdx.x;
    r = blockIdx.x * 32 + threadIdx.y;
    for (int k = 0; k < 32; k += 8)
        if (r + k < C && c < R) B[(long)(r + k) * ldb + c] = t[threadIdx.x][threadIdx.y + k];
}

}  // namespace

// Z_b = a X_b + c_b W_b with c_b = cvec[b] when cvec is given, else c.
extern "C" int cf_axpby(long count, double a, const double* X, long strideX, double c, const double* cvec,
                        const double* W, long strideW, double* Z, long strideZ, int batch, void* stream)
{
    if (count <= 0 || batch < 1 || !X || !Z) return CF_ERR_ARG;
    long blocks = (count + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_axpby<<<dim3((unsigned)blocks, batch), 256, 0, (cudaStream_t)stream>>>(count, a, X, strideX, c, cvec,
                                                                             W, strideW, Z, strideZ);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

extern "C" int cf_transpose(int R, int C, const double* A, long lda, double* B, long ldb, void* stream)
{
    if (R <= 0 || C <= 0 || !A || !B) return CF_ERR_ARG;
    k_transpose<<<dim3(cf_cdiv(C, 32), cf_cdiv(R, 32)), dim3(32, 8), 0, (cudaStream_t)stream>>>(R, C, A, lda,
                                                                                              B, ldb);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

unsigned long long g_cf_launch_count = 0;

extern "C" unsigned long long cf_launch_count(void) { return g_cf_launch_count; }

extern "C" int cf_version(void) { return 1; }

#include <cuda_bf16.h>

namespace {

// out[p][r][c] = p-th BF16 split plane of X[r][c] (cf_bf16_plane)
__global__ void k_split_bf16(int R, int C, const double* X, long ldx, int planes, __nv_bfloat16* out, long ldo,
                             long plane_stride)
{
    const long total = (long)R * C;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long r = e / C, c = e % C;
        double x = X[r * ldx + c];
        for (int p = 0; p < planes; ++p) out[p * plane_stride + r * ldo + c] = cf_bf16_plane(x);
    }
}

}  // namespace

// BF16 split planes of an R x C FP64 matrix (row stride ldx) into `planes`
// planes of row stride ldo, `plane_stride` elements apart.
extern "C" int cf_split_bf16(int R, int C, const double* X, long ldx, int planes, void* out, long ldo,
                             long plane_stride, void* stream)
{
    if (R <= 0 || C <= 0 || !X || !out || planes < 1 || planes > 3) return CF_ERR_ARG;
    long blocks = ((long)R * C + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_split_bf16<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(R, C, X, ldx, planes, (__nv_bfloat16*)out,
                                                                     ldo, plane_stride);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

namespace {

// out[p][q][i][j] = p-th BF16 split plane of x_q[i] * y_q[j]  (i < m, j < n)
__global__ void k_outer_planes(int m, int n, int nvec, const double* x, const double* y, long ldv, int planes,
                               __nv_bfloat16* out, long ld, long q_stride, long plane_stride)
{
    const long per = (long)m * n, total = (long)nvec * per;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long q = e / per, rem = e % per;
        const long i = rem / n, j = rem % n;
        double v = x[i * ldv + q] * y[j * ldv + q];
        for (int p = 0; p < planes; ++p) out[p * plane_stride + q * q_stride + i * ld + j] = cf_bf16_plane(v);
    }
}

}  // namespace

// BF16 split planes of the outer products x_q y_q^T, q < nvec (x: m x nvec,
// y: n x nvec, both with row stride ldv), into out[p][q] (m x n, row stride
// ld, q_stride / plane_stride elements apart).
extern "C" int cf_outer_planes_rect(int m, int n, int nvec, const double* x, const double* y, long ldv, int planes,
                                    void* out, long ld, long q_stride, long plane_stride, void* stream)
{
    if (m <= 0 || n <= 0 || nvec <= 0 || !x || !y || !out || planes < 1 || planes > 3) return CF_ERR_ARG;
    long blocks = ((long)nvec * m * n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_outer_planes<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(m, n, nvec, x, y, ldv, planes,
                                                                       (__nv_bfloat16*)out, ld, q_stride,
                                                                       plane_stride);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// The square case (m = n).
extern "C" int cf_outer_planes(int n, int nvec, const double* x, const double* y, long ldv, int planes, void* out,
                               long ld, long q_stride, long plane_stride, void* stream)
{
    return cf_outer_planes_rect(n, n, nvec, x, y, ldv, planes, out, ld, q_stride, plane_stride, stream);
}
