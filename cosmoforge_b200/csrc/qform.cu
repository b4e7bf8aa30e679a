// Quadratic forms of many maps against the derivative blocks of one spectrum.
//
// With W = D^T Y (one GEMM per spectrum: D stacks the bins' derivative
// blocks, Y = C^-1 X holds the maps in its columns),
//   q[m, p0 + b] += scale sum_{j < J} W[b * rows_per_bin + j, m] Y[yoff + j, m],
// i.e. q_b(m) = 1/2 y_m^T dC_b y_m of qube/spectra.py:1124-1186 for every map
// m at once.  One thread per (bin, map): both reads coalesce across maps.
#include "cf_common.cuh"

namespace {

template <typename WT>
__global__ void k_qform(int nb, int J, long rows_per_bin, const WT* W, long ldW, const double* Y, long ldY, long yoff,
                        int nmaps, double scale, double* q, long ldq, int p0)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (m >= nmaps || b >= nb) return;
    const WT* w = W + (long)b * rows_per_bin * ldW + m;
    const double* y = Y + yoff * ldY + m;
    double acc = 0.0;
    for (int j = 0; j < J; ++j) acc += (double)w[(long)j * ldW] * y[(long)j * ldY];
    q[(long)m * ldq + p0 + b] += scale * acc;
}

template <typename WT>
int launch(int nb, int J, long rpb, const WT* W, long ldW, const double* Y, long ldY, long yoff, int nmaps,
           double scale, double* q, long ldq, int p0, void* stream)
{
    if (nb <= 0 || J <= 0 || nmaps <= 0 || !W || !Y || !q) return CF_ERR_ARG;
    k_qform<WT><<<dim3(cf_cdiv(nmaps, 128), nb), 128, 0, (cudaStream_t)stream>>>(nb, J, rpb, W, ldW, Y, ldY, yoff,
                                                                                 nmaps, scale, q, ldq, p0);
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
