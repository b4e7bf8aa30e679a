// Quadratic forms of many maps against the derivative blocks of one spectrum.
//
// With W = D^T Y (one GEMM per spectrum: D stacks the bins' derivative
// blocks, Y = C^-1 X holds the maps in its columns),
//   q[m, p0 + b] += scale sum_{j < J} W[b * rows_per_bin + j, m] Y[yoff + j, m],
// i.e. q_b(m) = 1/2 y_m^T dC_b y_m of qube/spectra.py:1124-1186 for every map
// m at once.  One thread per (bin, map, chunk of rows), eight rows (sixteen
// loads) in flight per step: both reads coalesce across maps; the rows of a
// bin are split over enough CTAs to fill the GPU
// (W is read once from HBM, the Y rows of a chunk stay in L2 across bins), and
// the partial sums meet in q by FP64 atomics.
#include "cf_common.cuh"

namespace {

template <typename WT>
__global__ void k_qform(int nb, int J, long rows_per_bin, const WT* W, long ldW, const double* Y, long ldY, long yoff,
                        int nmaps, double scale, double* q, long ldq, int p0, int jchunk)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    const int j0 = blockIdx.z * jchunk;
    const int j1 = J < j0 + jchunk ? J : j0 + jchunk;
    if (m >= nmaps || b >= nb || j0 >= j1) return;
    const WT* w = W + (long)b * rows_per_bin * ldW + m;
    const double* y = Y + yoff * ldY + m;
    // eight rows per step, all sixteen loads issued before the products
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    int j = j0;
    for (; j + 7 < j1; j += 8) {
        WT wv[8];
        double yv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            wv[u] = w[(long)(j + u) * ldW];
            yv[u] = y[(long)(j + u) * ldY];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) acc[u & 3] += (double)wv[u] * yv[u];
    }
    for (; j < j1; ++j) acc[0] += (double)w[(long)j * ldW] * y[(long)j * ldY];
    atomicAdd(q + (long)m * ldq + p0 + b, scale * ((acc[0] + acc[1]) + (acc[2] + acc[3])));
}

template <typename WT>
int launch(int nb, int J, long rpb, const WT* W, long ldW, const double* Y, long ldY, long yoff, int nmaps,
           double scale, double* q, long ldq, int p0, void* stream)
{
    if (nb <= 0 || J <= 0 || nmaps <= 0 || !W || !Y || !q) return CF_ERR_ARG;
    // about 16 resident 128-thread CTAs on each of 148 SMs, chunks of >= 64 rows
    const long base = (long)cf_cdiv(nmaps, 128) * nb;
    long splits = (148L * 16 + base - 1) / base;
    const long max_splits = (J + 63) / 64;
    if (splits > max_splits) splits = max_splits;
    if (splits < 1) splits = 1;
    if (splits > 65535) splits = 65535;
    const int jchunk = (int)((J + splits - 1) / splits);
    k_qform<WT><<<dim3(cf_cdiv(nmaps, 128), nb, (unsigned)splits), 128, 0, (cudaStream_t)stream>>>(
        nb, J, rpb, W, ldW, Y, ldY, yoff, nmaps, scale, q, ldq, p0, jchunk);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

}  // namespace

// FP64 W (plain path).
extern "C" int cf_qform_reduce_f64(int nb, int J, long rows_per_bin, const double* W, long ldW, const double* Y,
                                   long ldY, long yoff, int nmaps, double scale, double* q, long ldq, int p0,
                                   void* stream)
{
    return launch<double>(nb, J, rows_per_bin, W, ldW, Y, ldY, yoff, nmaps, scale, q, ldq, p0, stream);
}

// FP32 W (the split-product GEMM's output in the mixed path).
extern "C" int cf_qform_reduce_f32(int nb, int J, long rows_per_bin, const float* W, long ldW, const double* Y,
                                   long ldY, long yoff, int nmaps, double scale, double* q, long ldq, int p0,
                                   void* stream)
{
    return launch<float>(nb, J, rows_per_bin, W, ldW, Y, ldY, yoff, nmaps, scale, q, ldq, p0, stream);
}
