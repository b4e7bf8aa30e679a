// Fisher traces and QML quadratic forms, FP64.
//
// Fisher (qube/fisher.py:557-607, cosmocore/basics/linalg.py:66-98):
//   F_pq = 1/2 Tr(A_p A_q) = 1/2 sum_{k,l} A_p[k,l] A_q[l,k].
// With A_p stored per column segment and A_q^T stored alongside, every
// segment pair (s, t) is one dense contraction over the flattened (k, l)
// plane:  F[p, q] += scale * sum_{k < K1, l < K2} X_p[k, l] Y_q[k, l],
// where X_p[k, l] = X[p * sXp + k * ldX + l] and likewise for Y.  This is a
// GEMM with M = #p, N = #q and a huge K = K1 * K2, run split-K on the DMMA
// pipe; each CTA reduces its K share in FP64 and adds it into F.
//
// QML (qube/spectra.py:1124-1186): for the derivative blocks D_p of one
// spectrum,  bias_p = 1/2 mult sum_{r,c} M[r,c] D_p[r,c]  with
// M = C^-1 N C^-1, and q_p^m = 1/2 mult sum_{r,c} y_r^m D_p[r,c] y_c^m with
// y = C^-1 x; mult = 2 for a cross block whose mirror is not stored.
#include "cf_common.cuh"

namespace {

constexpr int TBM = 64, TBN = 64, TBK = 16, TNT = 128, TST = 3, TPAD = TBK + 4;

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(src), "r"(valid ? 8 : 0));
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

__global__ void __launch_bounds__(TNT) k_trace_f64(int P1, int P2, int K1, int K2, const double* X,
                                                   long sXp, long ldX, const double* Y, long sYq, long ldY,
                                                   double scale, double* F, long ldF, long p_off,
                                                   long q_off, int sym)
{
    extern __shared__ __align__(16) double tsm[];
    double (*sX)[TBM * TPAD] = reinterpret_cast<double (*)[TBM * TPAD]>(tsm);
    double (*sY)[TBN * TPAD] = reinterpret_cast<double (*)[TBN * TPAD]>(tsm + TST * TBM * TPAD);
    const int p0 = blockIdx.y * TBM, q0 = blockIdx.z * TBN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int nl = (K2 + TBK - 1) / TBK;
    const long T = (long)K1 * nl;
    const long t_begin = T * blockIdx.x / gridDim.x, t_end = T * (blockIdx.x + 1) / gridDim.x;

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    auto issue = [&](long t, int st) {
        if (t < t_end) {
            const int k = (int)(t / nl), l0 = (int)(t % nl) * TBK;
#pragma unroll
            for (int it = 0; it < (TBM * TBK) / TNT; ++it) {
                int e = it * TNT + tid;
                int r = e / TBK, c = e % TBK;
                bool vx = (p0 + r < P1) && (l0 + c < K2);
                const double* src = vx ? X + (long)(p0 + r) * sXp + (long)k * ldX + l0 + c : X;
                cp_async8(&sX[st][r * TPAD + c], src, vx);
                bool vy = (q0 + r < P2) && (l0 + c < K2);
                const double* srcy = vy ? Y + (long)(q0 + r) * sYq + (long)k * ldY + l0 + c : Y;
                cp_async8(&sY[st][r * TPAD + c], srcy, vy);
            }
        }
        cp_commit();
    };
    for (int s = 0; s < TST - 1; ++s) issue(t_begin + s, s);
    int st = 0;
    for (long t = t_begin; t < t_end; ++t) {
        cp_wait<TST - 2>();
        __syncthreads();
        issue(t + TST - 1, (int)((t - t_begin + TST - 1) % TST));
        const double* xs = sX[st];
        const double* ys = sY[st];
#pragma unroll
        for (int ks = 0; ks < TBK; ks += 4) {
            const int kk = ks + (lane & 3);
            double af[4], bf[4];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) af[mi] = xs[(wm + mi * 8 + (lane >> 2)) * TPAD + kk];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) bf[ni] = ys[(wn + ni * 8 + (lane >> 2)) * TPAD + kk];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) dmma(acc[mi][ni][0], acc[mi][ni][1], af[mi], bf[ni]);
        }
        st = (st + 1) % TST;
    }
    cp_wait<0>();
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
        const int p = p0 + wm + mi * 8 + (lane >> 2);
        if (p >= P1) continue;
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int q = q0 + wn + ni * 8 + (lane & 3) * 2 + h;
                if (q >= P2) continue;
                const double v = scale * acc[mi][ni][h];
                atomicAdd(F + (p_off + p) * ldF + q_off + q, v);
                if (sym) atomicAdd(F + (q_off + q) * ldF + p_off + p, v);
            }
    }
}

// QML reductions over one derivative chunk.  CTA = (row band of 8 rows,
// group of up to QP params).  Accumulates bias[p] and q[m * ldq + p].
constexpr int QP = 8, QM = 4, QROWS = 8, QNT = 256;

__global__ void __launch_bounds__(QNT) k_qml_reduce(int P, int R, int Ccols, const double* D, long ldD,
                                                    long sDp, const double* M, long ldM, long mro,
                                                    long mco, const double* Yv, long ldY, int nsims,
                                                    long yro, long yco, double scale, double* bias,
                                                    double* q, long ldq)
{
    const int pg = blockIdx.y * QP;
    const int r0 = blockIdx.x * QROWS;
    const int tid = threadIdx.x;
    double ab[QP], aq[QP][QM];
#pragma unroll
    for (int i = 0; i < QP; ++i) {
        ab[i] = 0.0;
#pragma unroll
        for (int m = 0; m < QM; ++m) aq[i][m] = 0.0;
    }
    const int nm = nsims < QM ? nsims : QM;
    for (int rr = 0; rr < QROWS; ++rr) {
        const int r = r0 + rr;
        if (r >= R) break;
        double yr[QM];
#pragma unroll
        for (int m = 0; m < QM; ++m) yr[m] = (m < nm && Yv) ? Yv[(yro + r) * ldY + m] : 0.0;
        for (int c = tid; c < Ccols; c += QNT) {
            const double mv = M ? M[(mro + r) * ldM + mco + c] : 0.0;
            double yy[QM];
#pragma unroll
            for (int m = 0; m < QM; ++m) yy[m] = (m < nm && Yv) ? yr[m] * Yv[(yco + c) * ldY + m] : 0.0;
#pragma unroll
            for (int i = 0; i < QP; ++i) {
                if (pg + i < P) {
                    const double d = D[(long)r * ldD + (long)(pg + i) * sDp + c];
                    ab[i] = fma(mv, d, ab[i]);
#pragma unroll
                    for (int m = 0; m < QM; ++m) aq[i][m] = fma(yy[m], d, aq[i][m]);
                }
            }
        }
    }
    __shared__ double red[QNT / 32][QP * (QM + 1)];
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int i = 0; i < QP; ++i) {
        double v = ab[i];
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][i * (QM + 1)] = v;
#pragma unroll
        for (int m = 0; m < QM; ++m) {
            double w = aq[i][m];
            for (int o = 16; o; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
            if (lane == 0) red[warp][i * (QM + 1) + 1 + m] = w;
        }
    }
    __syncthreads();
    if (tid < QP * (QM + 1)) {
        double s = 0.0;
        for (int w = 0; w < QNT / 32; ++w) s += red[w][tid];
        const int i = tid / (QM + 1), m = tid % (QM + 1);
        if (pg + i < P) {
            if (m == 0) {
                if (bias && M) atomicAdd(bias + pg + i, scale * s);
            } else if (m - 1 < nm && q) {
                atomicAdd(q + (long)(m - 1) * ldq + pg + i, scale * s);
            }
        }
    }
}

}  // namespace

extern "C" int cf_trace_contract_f64(int P1, int P2, int K1, int K2, const double* X, long sXp, long ldX,
                                     const double* Y, long sYq, long ldY, double scale, double* F,
                                     long ldF, long p_off, long q_off, int sym, int splits, void* stream)
{
    if (P1 <= 0 || P2 <= 0 || K1 <= 0 || K2 <= 0 || !X || !Y || !F) return CF_ERR_ARG;
    long T = (long)K1 * ((K2 + TBK - 1) / TBK);
    if (splits <= 0) splits = 148 * 4;
    if (splits > T) splits = (int)T;
    dim3 grid(splits, cf_cdiv(P1, TBM), cf_cdiv(P2, TBN));
    const size_t smem = (size_t)TST * (TBM + TBN) * TPAD * sizeof(double);
    static std::atomic<int> attr[CF_MAX_DEVICES];
    if (int rc = cf_smem_optin(k_trace_f64, (int)smem, attr)) return rc;
    k_trace_f64<<<grid, TNT, smem, (cudaStream_t)stream>>>(P1, P2, K1, K2, X, sXp, ldX, Y, sYq, ldY, scale,
                                                        F, ldF, p_off, q_off, sym);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

extern "C" int cf_qml_reduce_f64(int P, int R, int Ccols, const double* D, long ldD, long sDp,
                                 const double* M, long ldM, long mro, long mco, const double* Y, long ldY,
                                 int nsims, long yro, long yco, double scale, double* bias, double* q,
                                 long ldq, void* stream)
{
    if (P <= 0 || R <= 0 || Ccols <= 0 || !D) return CF_ERR_ARG;
    if (nsims > QM && Y) return CF_ERR_UNSUPPORTED;
    dim3 grid(cf_cdiv(R, QROWS), cf_cdiv(P, QP));
    k_qml_reduce<<<grid, QNT, 0, (cudaStream_t)stream>>>(P, R, Ccols, D, ldD, sDp, M, ldM, mro, mco, Y,
                                                         ldY, nsims, yro, yco, scale, bias, q, ldq);
    CF_CHECK_LAUNCH();
    return CF_OK;
}
