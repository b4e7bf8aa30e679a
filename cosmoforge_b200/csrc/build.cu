// Fused pixel-pair builder for the signal covariance S and the binned
// derivatives dC_b (FP64 recurrences on the CUDA cores).
//
// One thread owns one pixel pair (row pixel j of field b, column pixel i of
// field a).  It forms x = r_j . r_i, runs the spin-0 / spin-2 / spin-0x2
// recurrences over l once, and accumulates the l-weighted sums of every
// output "bin" as l advances; when a bin closes its value is written.  The
// signal matrix is the one-bin case (weights = beam-smoothed C_l); a chunk
// of binned derivatives of one spectrum is the many-bin case (weights
// w_l b_l^2 inside each bin), so one recurrence pass serves every bin.
//
// Arithmetic follows the reference kernels
//   legendre_00/22/02      cosmocore/basics/legendre.py:9-149
//   get_rotation_angle     cosmocore/basics/geometry.py:15-110
//   _compute_00/22/02      cosmocore/signal_kernels.py:164-387
// Reduce mode (cf_build_block_reduce) writes nothing to HBM: every entry
// of every bin is consumed where it is formed, against W[r, c] (the noise
// bias, W = C^-1 N C^-1) and y_r y_c (quadratic forms of up to four maps),
// with one warp reduction per closed bin into per-CTA shared sums.
//
// The pair argument and the rotation angles are evaluated with explicit
// round-to-nearest operations in the reference's order (no fused
// multiply-add), because the angle of nearly collinear pairs is an ill-
// conditioned function of these products; the recurrences themselves are
// well conditioned and use FMA.
#include <cuda_bf16.h>

#include "cf_common.cuh"

namespace {

enum { K00A = 0, K00X = 1, K22A = 2, K02 = 3 };
constexpr int MAXL = 512;
constexpr int BX = 32, BY = 8;

struct BuildArgs {
    int kind, mode;  // mode < 0: signal (all tables); else derivative spectrum mode
    int na, nb;      // pixels of column field a and row field b
    const double* va;  // SoA pointings x[na], y[na], z[na]
    const double* vb;
    int lmax;
    const double* t0;
    const double* t1;
    const double* t2;
    const int* bin_of;  // [lmax+1] bin index or -1; nullptr: one bin over all l
    double* out;
    long ld, row_off, col_off, bin_stride;
    double* outT;
    long ldT, rowT_off, colT_off, binT_stride;
    long tstride;   // batch stride of the l tables
    long ostride;   // batch stride of out and outT
    int planes;     // 0: FP64 output; 1..3: BF16 split planes of the FP64 value
    long plane_stride, planeT_stride;
    int full;       // compute every pair of an auto block (no mirror writes)
    int trans;      // threads walk (col pixel, row pixel) and write only the transposed entry
    // reduce mode
    const double* W;  // symmetric n x n weight (bias) or nullptr
    long ldW;
    const double* Yv;  // n x nv maps (row stride ldY) or nullptr
    long ldY;
    int nv;
    long gro, gco;    // global row / column of the block's entry (0, 0)
    double* rbias;    // rbias[b] += scale * sum W . dC_b
    double* rq;       // rq[m * ldq + b] += scale * sum y_m y_m^T . dC_b
    long ldq;
    double scale;
    int nbins;
};

constexpr int RED_MAXB = 128, RED_QM = 4, RED_NP = 4;

// Per-pair weights of the (up to four) entries a thread emits per bin:
// f * W[r, c] and f * y_r y_c with f = 2 for entries written with a mirror.
struct RedWeights {
    double wb[RED_NP];
    double wq[RED_NP][RED_QM];
    __device__ __forceinline__ void set(const BuildArgs& a, int k, long r, long c, double f, bool transposed_read)
    {
        const long gr = a.gro + r, gc = a.gco + c;
        // W symmetric: read the orientation whose column follows threadIdx.x
        wb[k] = a.W ? f * (transposed_read ? a.W[gc * a.ldW + gr] : a.W[gr * a.ldW + gc]) : 0.0;
#pragma unroll
        for (int m = 0; m < RED_QM; ++m)
            wq[k][m] = (m < a.nv) ? f * a.Yv[gr * a.ldY + m] * a.Yv[gc * a.ldY + m] : 0.0;
    }
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int k = 0; k < RED_NP; ++k) {
            wb[k] = 0.0;
#pragma unroll
            for (int m = 0; m < RED_QM; ++m) wq[k][m] = 0.0;
        }
    }
};

// Sum over the warp of v . weights for bin b, added to the CTA's shared sums.
__device__ __forceinline__ void red_emit(const BuildArgs& a, const RedWeights& w, const double* v, int np, int b,
                                         double* s_red)
{
    double cb = 0.0, cq[RED_QM];
#pragma unroll
    for (int m = 0; m < RED_QM; ++m) cq[m] = 0.0;
    for (int k = 0; k < np; ++k) {
        cb = fma(v[k], w.wb[k], cb);
#pragma unroll
        for (int m = 0; m < RED_QM; ++m) cq[m] = fma(v[k], w.wq[k][m], cq[m]);
    }
    const bool want_b = a.W != nullptr;
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        if (want_b) cb += __shfl_xor_sync(0xffffffffu, cb, o);
#pragma unroll
        for (int m = 0; m < RED_QM; ++m)
            if (m < a.nv) cq[m] += __shfl_xor_sync(0xffffffffu, cq[m], o);
    }
    static_assert(BX == 32, "a warp is one row of the CTA");
    if (threadIdx.x == 0) {
        double* dst = s_red + b * (1 + RED_QM);
        if (want_b) atomicAdd(dst, cb);
#pragma unroll
        for (int m = 0; m < RED_QM; ++m)
            if (m < a.nv) atomicAdd(dst + 1 + m, cq[m]);
    }
}

__device__ __forceinline__ void rotation_angle(double r1x, double r1y, double r1z, double r2x,
                                               double r2y, double r2z, double& a12, double& a21)
{
    double x = __dsub_rn(__dmul_rn(r1y, r2z), __dmul_rn(r1z, r2y));
    double y = __dsub_rn(__dmul_rn(r1z, r2x), __dmul_rn(r1x, r2z));
    double z = __dsub_rn(__dmul_rn(r1x, r2y), __dmul_rn(r1y, r2x));
    double mod = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
    if (mod < 1e-8) {
        a12 = 0.0;
        a21 = 0.0;
        return;
    }
    x = __ddiv_rn(x, mod);
    y = __ddiv_rn(y, mod);
    z = __ddiv_rn(z, mod);
    const double eps = CF_PI / 180.0 / 3600.0 / 100.0;
    // projection of r onto the tangent plane: z_hat x r = (-r_y, r_x, 0), normalised
    double p1x = -r1y, p1y = r1x;
    double nm1 = __dsqrt_rn(__dadd_rn(__dmul_rn(p1x, p1x), __dmul_rn(p1y, p1y)));
    if (nm1 < 1e-8) {
        p1x = __dadd_rn(p1x, eps);
        nm1 = __dsqrt_rn(__dadd_rn(__dmul_rn(p1x, p1x), __dmul_rn(p1y, p1y)));
    }
    double p2x = -r2y, p2y = r2x;
    double nm2 = __dsqrt_rn(__dadd_rn(__dmul_rn(p2x, p2x), __dmul_rn(p2y, p2y)));
    if (nm2 < 1e-8) {
        p2x = __dadd_rn(p2x, eps);
        nm2 = __dsqrt_rn(__dadd_rn(__dmul_rn(p2x, p2x), __dmul_rn(p2y, p2y)));
    }
    p1x = __ddiv_rn(p1x, nm1);
    p1y = __ddiv_rn(p1y, nm1);
    p2x = __ddiv_rn(p2x, nm2);
    p2y = __ddiv_rn(p2y, nm2);
    double d1 = __dadd_rn(__dmul_rn(x, p1x), __dmul_rn(y, p1y));
    d1 = d1 > 1.0 ? 1.0 : (d1 < -1.0 ? -1.0 : d1);
    a12 = __dmul_rn(__dmul_rn(2.0, acos(d1)), z > 0.0 ? 1.0 : -1.0);
    double d2 = __dadd_rn(__dmul_rn(-x, p2x), __dmul_rn(-y, p2y));
    d2 = d2 > 1.0 ? 1.0 : (d2 < -1.0 ? -1.0 : d2);
    a21 = __dmul_rn(__dmul_rn(2.0, acos(d2)), -z > 0.0 ? 1.0 : -1.0);
}

struct Emitter {
    const BuildArgs& a;
    // write block entry (r, c) of bin `bin` and its mirror (c, r)
    long base;
    __device__ Emitter(const BuildArgs& args, long b) : a(args), base(b) {}
    __device__ __forceinline__ void put(long r, long c, int bin, double v, bool mirror) const
    {
        const long i = base + (a.row_off + r) * a.ld + a.col_off + bin * a.bin_stride + c;
        const long iT = base + (a.rowT_off + c) * a.ldT + a.colT_off + bin * a.binT_stride + r;
        const bool prim = !a.trans;
        mirror = a.trans || (mirror && !a.full);
        if (a.planes == 0) {
            if (prim) a.out[i] = v;
            if (mirror) a.outT[iT] = v;
            return;
        }
        __nv_bfloat16* o = reinterpret_cast<__nv_bfloat16*>(a.out);
        __nv_bfloat16* oT = reinterpret_cast<__nv_bfloat16*>(a.outT);
        double x = v;
        for (int p = 0; p < a.planes; ++p) {
            const __nv_bfloat16 h = cf_bf16_plane(x);
            if (prim) o[p * a.plane_stride + i] = h;
            if (mirror) oT[p * a.planeT_stride + iT] = h;
        }
    }
};

template <bool RED>
__global__ void __launch_bounds__(BX* BY) k_build(BuildArgs a)
{
    __shared__ double s_red[RED ? RED_MAXB * (1 + RED_QM) : 1];
    __shared__ double s_c[5][MAXL + 1];
    __shared__ double s_al[MAXL + 1], s_be[MAXL + 1];
    __shared__ int s_bin[MAXL + 1];
    __shared__ unsigned char s_emit[MAXL + 1];

    const int L = a.lmax;
    const int tid = threadIdx.y * BX + threadIdx.x;
    for (int l = tid; l <= L; l += BX * BY) {
        const double dl = (double)l;
        const long tb = (long)blockIdx.z * a.tstride;
        double w0 = a.t0 ? a.t0[tb + l] : 0.0;
        double w1 = a.t1 ? a.t1[tb + l] : 0.0;
        double w2 = a.t2 ? a.t2[tb + l] : 0.0;
        for (int k = 0; k < 5; ++k) s_c[k][l] = 0.0;
        s_al[l] = 0.0;
        s_be[l] = 0.0;
        if (a.kind == K00A || a.kind == K00X) {
            s_c[0][l] = w0 * ((2.0 * dl + 1.0) / (4.0 * CF_PI));
            if (l >= 3) {
                s_al[l] = (2.0 * dl - 1.0) / dl;
                s_be[l] = (dl - 1.0) / dl;
            }
        } else if (l >= 2) {
            double q = (dl + 2.0) * (dl + 1.0) * dl * (dl - 1.0);
            if (l >= 3) {
                s_al[l] = (2.0 * dl - 1.0) / (dl - 2.0);
                s_be[l] = (dl + 1.0) / (dl - 2.0);
            }
            if (a.kind == K22A) {
                double nrm = (2.0 * dl + 1.0) / (4.0 * CF_PI) * (1.0 / q);
                // QQ += c0 f1 + c1 f2 ; UU += c2 f1 + c3 f2 ; QU += c4 (f1 + f2)
                if (a.mode < 0) {
                    s_c[0][l] = w0 * nrm;
                    s_c[1][l] = -w1 * nrm;
                    s_c[2][l] = w1 * nrm;
                    s_c[3][l] = -w0 * nrm;
                    s_c[4][l] = w2 * nrm;
                } else if (a.mode == 0) {  // EE
                    s_c[0][l] = w0 * nrm;
                    s_c[3][l] = -w0 * nrm;
                } else if (a.mode == 1) {  // BB
                    s_c[1][l] = -w0 * nrm;
                    s_c[2][l] = w0 * nrm;
                } else {  // EB
                    s_c[4][l] = w0 * nrm;
                }
            } else {  // K02: tq = -sum c_TE p, tu = -sum c_TB p
                double nrm = (2.0 * dl + 1.0) / (4.0 * CF_PI) * sqrt(1.0 / q);
                if (a.mode < 0) {
                    s_c[0][l] = -w0 * nrm;
                    s_c[1][l] = -w1 * nrm;
                } else if (a.mode == 0) {
                    s_c[0][l] = -w0 * nrm;
                } else {
                    s_c[1][l] = -w0 * nrm;
                }
            }
        }
        s_bin[l] = a.bin_of ? a.bin_of[l] : 0;
    }
    if (RED)
        for (int k = tid; k < RED_MAXB * (1 + RED_QM); k += BX * BY) s_red[k] = 0.0;
    __syncthreads();
    for (int l = tid; l <= L; l += BX * BY) {
        int b = s_bin[l];
        s_emit[l] = (b >= 0) && (l == L || s_bin[l + 1] != b);
    }
    __syncthreads();

    // column pixel i (field a), row pixel j (field b); the transposed launch
    // walks j along threadIdx.x so that its (transposed) writes coalesce
    int i = a.trans ? blockIdx.y * BY + threadIdx.y : blockIdx.x * BX + threadIdx.x;
    int j = a.trans ? blockIdx.x * BX + threadIdx.x : blockIdx.y * BY + threadIdx.y;
    const bool autob = (a.kind == K00A || a.kind == K22A);
    const bool live = i < a.na && j < a.nb && !(autob && !a.full && j < i);
    if (!RED) {
        if (!live) return;
    } else {
        // warps reduce every closed bin: threads without a pair of their own
        // run a zero-weight stand-in (pixel 0 with itself) unless the whole
        // CTA has none
        if (!__syncthreads_or(live)) return;
        if (!live) i = j = 0;
    }
    RedWeights rw;
    double rv[RED_NP];

    const double r2x = a.va[i], r2y = a.va[a.na + i], r2z = a.va[2 * a.na + i];
    const double r1x = a.vb[j], r1y = a.vb[a.nb + j], r1z = a.vb[2 * a.nb + j];
    const bool diag = autob && (i == j);
    const double x =
        diag ? 1.0 : __dadd_rn(__dadd_rn(__dmul_rn(r1x, r2x), __dmul_rn(r1y, r2y)), __dmul_rn(r1z, r2z));
    Emitter em(a, (long)blockIdx.z * a.ostride);

    if (a.kind == K00A || a.kind == K00X) {
        if (RED) {
            if (live) rw.set(a, 0, j, i, diag ? 1.0 : 2.0, false);
            else rw.zero();
        }
        double acc = 0.0;
        double pm2 = 0.0, pm1 = 0.0;  // P_{l-2}, P_{l-1}
        for (int l = 0; l <= L; ++l) {
            double p;
            if (l == 0) p = 1.0;
            else if (l == 1) p = x;
            else if (l == 2) p = 1.5 * x * x - 0.5;
            else p = s_al[l] * x * pm1 - s_be[l] * pm2;
            pm2 = pm1;
            pm1 = p;
            acc = fma(s_c[0][l], p, acc);
            if (s_emit[l]) {
                if (RED) {
                    rv[0] = acc;
                    red_emit(a, rw, rv, 1, s_bin[l], s_red);
                } else {
                    em.put(j, i, s_bin[l], acc, !diag);
                }
                acc = 0.0;
            }
        }
    } else {
        double c1 = 1.0, s1 = 0.0, c2 = 1.0, s2 = 0.0;
        if (!diag) {
            double a1, a2;
            rotation_angle(r1x, r1y, r1z, r2x, r2y, r2z, a1, a2);
            double sa, ca;
            sincos(a1, &sa, &ca);
            c1 = ca;
            s1 = sa;
            if (a.kind == K22A) {
                sincos(a2, &sa, &ca);
                c2 = ca;
                s2 = -sa;
                s1 = -s1;
            }
        }

        if (a.kind == K22A) {
            const long n = a.na;
            if (RED) {
                if (!live) {
                    rw.zero();
                } else if (diag) {
                    rw.set(a, 0, j, i, 1.0, false);
                    rw.set(a, 1, j + n, i + n, 1.0, false);
                    rw.set(a, 2, j + n, i, 2.0, false);
                    rw.wb[3] = 0.0;
                    for (int m = 0; m < RED_QM; ++m) rw.wq[3][m] = 0.0;
                } else {
                    rw.set(a, 0, j, i, 2.0, false);
                    rw.set(a, 1, j + n, i + n, 2.0, false);
                    rw.set(a, 2, j + n, i, 2.0, false);
                    rw.set(a, 3, i + n, j, 2.0, true);
                }
            }
            const double x2 = x * x;
            double qq = 0.0, uu = 0.0, qu = 0.0;
            double pm2 = 0.0, pm1 = 3.0;  // p_1 = 0, p_2 = 3
            double dl = 2.0;
            const double c1c2 = c1 * c2, s1s2 = s1 * s2, c1s2 = c1 * s2, s1c2 = s1 * c2;
            for (int l = 2; l <= L; ++l, dl += 1.0) {
                double p, f1, f2;
                if (l == 2) {
                    p = 3.0;
                    f1 = 6.0 * (1.0 + x2);
                    f2 = -12.0 * x;
                } else {
                    p = s_al[l] * x * pm1 - s_be[l] * pm2;
                    f1 = -((2.0 * dl - 8.0) + dl * (dl - 1.0) * (1.0 - x2)) * p + (2.0 * dl + 4.0) * x * pm1;
                    f2 = 4.0 * (-(dl - 1.0) * x * p + (dl + 2.0) * pm1);
                    pm2 = pm1;
                    pm1 = p;
                }
                qq = fma(s_c[0][l], f1, fma(s_c[1][l], f2, qq));
                uu = fma(s_c[2][l], f1, fma(s_c[3][l], f2, uu));
                qu = fma(s_c[4][l], f1 + f2, qu);
                if (s_emit[l]) {
                    const int b = s_bin[l];
                    double vqq = qq * c1c2 + uu * s1s2 + qu * (c1s2 + s1c2);
                    double vuu = qq * s1s2 + uu * c1c2 - qu * (c1s2 + s1c2);
                    double vuq = -qq * s1c2 + uu * c1s2 + qu * (c1c2 - s1s2);
                    double vqu = -qq * c1s2 + uu * s1c2 + qu * (c1c2 - s1s2);
                    if (RED) {
                        if (diag) {
                            rv[0] = qq;
                            rv[1] = uu;
                            rv[2] = qu;
                            rv[3] = 0.0;
                        } else {
                            rv[0] = vqq;
                            rv[1] = vuu;
                            rv[2] = vuq;
                            rv[3] = vqu;
                        }
                        red_emit(a, rw, rv, 4, b, s_red);
                    } else if (diag) {
                        em.put(j, i, b, qq, false);
                        em.put(j + n, i + n, b, uu, false);
                        em.put(j + n, i, b, qu, true);
                        if (a.full) em.put(j, i + n, b, qu, false);
                    } else if (a.full) {  // this pair owns its entries in rows j and j + n
                        em.put(j, i, b, vqq, false);
                        em.put(j + n, i + n, b, vuu, false);
                        em.put(j + n, i, b, vuq, false);
                        em.put(j, i + n, b, vqu, false);
                    } else {
                        em.put(j, i, b, vqq, true);
                        em.put(j + n, i + n, b, vuu, true);
                        em.put(j + n, i, b, vuq, true);
                        em.put(i + n, j, b, vqu, true);
                    }
                    qq = uu = qu = 0.0;
                }
            }
        } else {
            // K02: rows = P field b [Q | U], cols = T field a
            const long npb = a.nb;
            if (RED) {
                if (live) {
                    rw.set(a, 0, j, i, 2.0, false);
                    rw.set(a, 1, j + npb, i, 2.0, false);
                } else {
                    rw.zero();
                }
            }
            const double x2 = x * x;
            double tq = 0.0, tu = 0.0;
            double pm2 = 0.0, pm1 = 3.0 * (1.0 - x2);
            for (int l = 2; l <= L; ++l) {
                double p;
                if (l == 2) {
                    p = pm1;
                } else {
                    p = s_al[l] * x * pm1 - s_be[l] * pm2;
                    pm2 = pm1;
                    pm1 = p;
                }
                tq = fma(s_c[0][l], p, tq);
                tu = fma(s_c[1][l], p, tu);
                if (s_emit[l]) {
                    const int b = s_bin[l];
                    if (RED) {
                        rv[0] = tq * c1 - tu * s1;
                        rv[1] = tq * s1 + tu * c1;
                        red_emit(a, rw, rv, 2, b, s_red);
                    } else {
                        em.put(j, i, b, tq * c1 - tu * s1, true);
                        em.put(j + npb, i, b, tq * s1 + tu * c1, true);
                    }
                    tq = tu = 0.0;
                }
            }
        }
    }
    if (RED) {
        __syncthreads();
        for (int k = tid; k < a.nbins * (1 + RED_QM); k += BX * BY) {
            const int b = k / (1 + RED_QM), m = k % (1 + RED_QM);
            const double v = s_red[k];
            if (v == 0.0) continue;
            if (m == 0) {
                if (a.rbias) atomicAdd(a.rbias + b, a.scale * v);
            } else if (m - 1 < a.nv) {
                atomicAdd(a.rq + (long)(m - 1) * a.ldq + b, a.scale * v);
            }
        }
    }
}

}  // namespace

extern "C" int cf_build_block_planes(int kind, int mode, int na, const double* va, int nb, const double* vb,
                                     int lmax, const double* t0, const double* t1, const double* t2,
                                     const int* bin_of, void* out, long ld, long row_off, long col_off,
                                     long bin_stride, void* outT, long ldT, long rowT_off, long colT_off,
                                     long binT_stride, int batch, long tstride, long ostride, int planes,
                                     long plane_stride, long planeT_stride, int flags, void* stream);

extern "C" int cf_build_block(int kind, int mode, int na, const double* va, int nb, const double* vb,
                              int lmax, const double* t0, const double* t1, const double* t2,
                              const int* bin_of, double* out, long ld, long row_off, long col_off,
                              long bin_stride, double* outT, long ldT, long rowT_off, long colT_off,
                              long binT_stride, int batch, long tstride, long ostride, void* stream)
{
    return cf_build_block_planes(kind, mode, na, va, nb, vb, lmax, t0, t1, t2, bin_of, out, ld, row_off, col_off,
                                 bin_stride, outT, ldT, rowT_off, colT_off, binT_stride, batch, tstride, ostride,
                                 0, 0, 0, 0, stream);
}

// As cf_build_block, with `planes` >= 1 writing BF16 split planes (out/outT
// are then __nv_bfloat16 arrays, planes `plane_stride` / `planeT_stride`
// elements apart) instead of FP64.  flags bit 0 (auto blocks): every entry
// of the block is computed from its own pixel pair and written once, no
// mirror writes (symmetric entries then agree to rounding, not bit for bit);
// bit 1 (cross blocks): write only the transposed block outT, threads
// walking the row field fastest so the writes coalesce.
extern "C" int cf_build_block_planes(int kind, int mode, int na, const double* va, int nb, const double* vb,
                                     int lmax, const double* t0, const double* t1, const double* t2,
                                     const int* bin_of, void* out, long ld, long row_off, long col_off,
                                     long bin_stride, void* outT, long ldT, long rowT_off, long colT_off,
                                     long binT_stride, int batch, long tstride, long ostride, int planes,
                                     long plane_stride, long planeT_stride, int flags, void* stream)
{
    if (kind < K00A || kind > K02 || na <= 0 || nb <= 0 || lmax < 0 || lmax > MAXL || !va || !vb ||
        !out || !outT || !t0)
        return CF_ERR_ARG;
    if ((kind == K00A || kind == K22A) && (na != nb || va != vb)) return CF_ERR_ARG;
    if (batch < 1) return CF_ERR_ARG;
    if (planes < 0 || planes > 3) return CF_ERR_ARG;
    const int full = flags & 1, trans = (flags >> 1) & 1;
    if (trans && (kind == K00A || kind == K22A)) return CF_ERR_ARG;
    BuildArgs a{kind, mode, na, nb, va, vb, lmax, t0, t1, t2, bin_of, (double*)out, ld, row_off, col_off,
                bin_stride, (double*)outT, ldT, rowT_off, colT_off, binT_stride, tstride, ostride, planes,
                plane_stride, planeT_stride, full, trans,
                nullptr, 0, nullptr, 0, 0, 0, 0, nullptr, nullptr, 0, 0.0, 0};
    dim3 block(BX, BY);
    dim3 grid(trans ? cf_cdiv(nb, BX) : cf_cdiv(na, BX), trans ? cf_cdiv(na, BY) : cf_cdiv(nb, BY), batch);
    k_build<false><<<grid, block, 0, (cudaStream_t)stream>>>(a);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// Build-and-reduce: the derivative entries of every bin of one block are
// consumed where they are formed, nothing is written but the sums
//   bias[b]         += scale * sum_{r,c} W[gro + r, gco + c] dC_b[r, c]
//   q[m * ldq + b]  += scale * sum_{r,c} y_m[gro + r] y_m[gco + c] dC_b[r, c]
// over the whole block and its mirror (auto blocks: both triangles; cross
// blocks: the block and its transpose, so scale 1/2 gives the reference's
// 1/2 Tr and 1/2 y^T dC_b y over the full matrix).  W symmetric (n x n, row
// stride ldW) or NULL; Y: n x nv maps (nv <= 4, row stride ldY) or NULL.
// Same recurrences and arithmetic as cf_build_block; bins <= 128.
extern "C" int cf_build_block_reduce(int kind, int mode, int na, const double* va, int nb, const double* vb,
                                     int lmax, const double* t0, const double* t1, const double* t2,
                                     const int* bin_of, int nbins, const double* W, long ldW, const double* Y,
                                     long ldY, int nv, long gro, long gco, double scale, double* bias, double* q,
                                     long ldq, void* stream)
{
    if (kind < K00A || kind > K02 || na <= 0 || nb <= 0 || lmax < 0 || lmax > MAXL || !va || !vb || !t0)
        return CF_ERR_ARG;
    if ((kind == K00A || kind == K22A) && (na != nb || va != vb)) return CF_ERR_ARG;
    if (nbins < 1 || nbins > RED_MAXB || nv < 0 || nv > RED_QM || gro < 0 || gco < 0) return CF_ERR_ARG;
    if ((W && (!bias || ldW <= 0)) || (nv > 0 && (!Y || !q || ldY < nv || ldq < nbins))) return CF_ERR_ARG;
    if (!W && nv == 0) return CF_OK;
    BuildArgs a{kind, mode, na, nb, va, vb, lmax, t0, t1, t2, bin_of, nullptr, 0, 0, 0, 0, nullptr, 0, 0, 0, 0,
                0, 0, 0, 0, 0, 0, 0,
                W, ldW, nv ? Y : nullptr, ldY, nv, gro, gco, W ? bias : nullptr, nv ? q : nullptr, ldq, scale, nbins};
    dim3 block(BX, BY);
    dim3 grid(cf_cdiv(na, BX), cf_cdiv(nb, BY), 1);
    k_build<true><<<grid, block, 0, (cudaStream_t)stream>>>(a);
    CF_CHECK_LAUNCH();
    return CF_OK;
}
