// Diagonal block of the blocked Cholesky: factor a kb x kb SPD block
// (kb <= 64) in place and form the inverse of its factor, one CTA per batch
// matrix, for FP64 and FP32.
//
// The block is factored right-looking in 16-column panels:
//   (a) warp 0 factors the panel's 16 x 16 diagonal tile, left-looking (lane i
//       holds row i in registers; column k's entries are independent dot
//       products with row k read from shared memory; one shuffle and one
//       reciprocal square root per pivot, l_kk = d rsqrt(d));
//   (b) every row below the tile is solved against it by one thread
//       (x_k = a_k / l_kk, then a_j -= x_k l_jk for the later columns j);
//   (c) the trailing lower triangle takes the rank-16 update, 3 x 3 entries
//       per thread.
// Three barriers per panel instead of one per column.  The inverse X = L^-1 is
// formed by 16-row block rows: a spare warp inverts each diagonal tile by
// forward substitution (lane c = column c) while the rows below it are solved
// in step (b), then block row I takes
// X_I = T_I^-1 (-sum_{K<I} L_IK X_K) with T_I^-1 the tile inverse (four
// independent partial sums per dot product, to shorten the dependent chains).
//
// Per-problem status follows LAPACK: info = k0 + j + 1 for the first
// non-positive (or NaN) pivot j of this block, left unchanged when the
// problem already holds an earlier failure.  A failed pivot is replaced by 1
// so the kernel completes with finite work.
#pragma once
#include "cf_common.cuh"

namespace cf_diag {

constexpr int NB = 64;
constexpr int LDS = NB + 1;
constexpr int PW = 16;
constexpr int NTHREADS = 256;

template <typename T>
constexpr size_t smem_bytes() { return (size_t)(2 * NB * LDS + PW * NB) * sizeof(T); }

template <typename T>
__global__ void __launch_bounds__(NTHREADS) k_potrf_diag_inv(T* A, long lda, long sA, int k0, int kb, T* Dinv,
                                                             long sD, int* info)
{
    extern __shared__ __align__(16) unsigned char diag_smem[];
    T* S = reinterpret_cast<T*>(diag_smem);  // the block, then L (lower, zeros above)
    T* X = S + NB * LDS;                     // L^-1
    T* Tb = X + NB * LDS;                    // PW x NB scratch of the block-row products
    __shared__ T rdg[NB];                    // reciprocal pivots 1 / l_jj
    __shared__ int bad;
    const int b = blockIdx.x;
    A += (long)b * sA;
    Dinv += (long)b * sD;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned FULL = 0xffffffffu;

    // load the lower triangle (columns fastest: coalesced; every load in
    // flight before the first store), zero the rest
    {
        const int c = tid & 63;
        T v[NB / (NTHREADS / 64)];
#pragma unroll
        for (int i = 0; i < NB / (NTHREADS / 64); ++i) {
            const int r = (tid >> 6) + i * (NTHREADS / 64);
            v[i] = (r < kb && c <= r) ? A[(long)(k0 + r) * lda + k0 + c] : T(0);
        }
#pragma unroll
        for (int i = 0; i < NB / (NTHREADS / 64); ++i) {
            const int r = (tid >> 6) + i * (NTHREADS / 64);
            S[r * LDS + c] = v[i];
            X[r * LDS + c] = T(0);
        }
    }
    if (tid == 0) bad = 0;
    __syncthreads();

    // Inverse of the factored diagonal tile at t0 (one warp, lane c = column c,
    // forward substitution): X[t0 + r][t0 + c] for c <= r.  The tile and its
    // reciprocal pivots are final once step (a) of its panel is done.
    auto tile_inverse = [&](int t0) {
        const int tw = kb - t0 < PW ? kb - t0 : PW;
        const int c = lane;
        if (c < tw) {
            T x[PW];
#pragma unroll
            for (int r = 0; r < PW; ++r) {
                T acc = (r == c) ? T(1) : T(0);
#pragma unroll
                for (int mm = 0; mm < r; ++mm)
                    if (mm >= c) acc -= S[(t0 + r) * LDS + t0 + mm] * x[mm];
                x[r] = (r >= c && r < tw) ? acc * rdg[t0 + (r < tw ? r : 0)] : T(0);
            }
#pragma unroll
            for (int r = 0; r < PW; ++r)
                if (r < tw && r >= c) X[(t0 + r) * LDS + t0 + c] = x[r];
        }
    };
    constexpr int SPARE = NTHREADS / 32 - 1;  // idle in step (b): m <= 48 rows
    int p_last = 0;
    for (int p = 0; p < kb; p += PW) {
        const int pw = kb - p < PW ? kb - p : PW;
        p_last = p;
        // (a) the pw x pw diagonal tile, warp 0, lane i = row p + i, left-looking
        // (Crout): at column k every lane forms its entry as an independent dot
        // product of its own row of L with row k of L (broadcast reads of the
        // tile in shared memory), so a pivot costs one shuffle and one
        // reciprocal square root on the critical path
        if (warp == 0) {
            T r[PW];
#pragma unroll
            for (int j = 0; j < PW; ++j) r[j] = (lane < pw && j <= lane) ? S[(p + lane) * LDS + p + j] : T(0);
            T* Sp = S + p * LDS + p;
#pragma unroll
            for (int k = 0; k < PW; ++k) {
                if (k < pw) {
                    T acc0 = r[k], acc1 = T(0);
#pragma unroll
                    for (int m = 0; m < k; ++m) {
                        const T lkm = Sp[k * LDS + m];
                        if (m & 1)
                            acc1 -= r[m] * lkm;
                        else
                            acc0 -= r[m] * lkm;
                    }
                    const T sv = acc0 + acc1;
                    T d = __shfl_sync(FULL, sv, k);
                    if (!(d > T(0))) {  // also catches NaN
                        if (lane == 0 && bad == 0) bad = k0 + p + k + 1;
                        d = T(1);
                    }
                    const T rl = rsqrt(d);
                    if (lane == k)
                        r[k] = d * rl;
                    else if (lane > k)
                        r[k] = sv * rl;
                    if (lane == 0) rdg[p + k] = rl;
                    if (lane >= k && lane < pw) Sp[lane * LDS + k] = r[k];
                    __syncwarp();
                }
            }
        }
        __syncthreads();
        const int q = p + pw;  // first row / column of the trailing block
        const int m = kb - q;
        if (m <= 0) break;
        // (b) rows below the tile: L[i][p:p+pw] = A[i][p:p+pw] L_tile^-T;
        // meanwhile the spare warp inverts the tile (step A of the inverse)
        if (warp == SPARE) tile_inverse(p);
        if (tid < m) {
            const int i = q + tid;
            T a[PW];
#pragma unroll
            for (int j = 0; j < PW; ++j) a[j] = (j < pw) ? S[i * LDS + p + j] : T(0);
#pragma unroll
            for (int k = 0; k < PW; ++k) {
                if (k < pw) {
                    a[k] *= rdg[p + k];
#pragma unroll
                    for (int j = k + 1; j < PW; ++j)
                        if (j < pw) a[j] -= a[k] * S[(p + j) * LDS + p + k];
                }
            }
#pragma unroll
            for (int j = 0; j < PW; ++j)
                if (j < pw) S[i * LDS + p + j] = a[j];
        }
        __syncthreads();
        // (c) trailing update S[i][j] -= sum_k L[i][p+k] L[j][p+k], q <= j <= i < kb
        {
            const int ti = tid >> 4, tj = tid & 15;
            T acc[3][3];
#pragma unroll
            for (int u = 0; u < 3; ++u)
#pragma unroll
                for (int v = 0; v < 3; ++v) acc[u][v] = T(0);
            for (int k = 0; k < pw; ++k) {
                T li[3], lj[3];
#pragma unroll
                for (int u = 0; u < 3; ++u) {
                    const int i = q + ti + 16 * u, j = q + tj + 16 * u;
                    li[u] = i < kb ? S[i * LDS + p + k] : T(0);
                    lj[u] = j < kb ? S[j * LDS + p + k] : T(0);
                }
#pragma unroll
                for (int u = 0; u < 3; ++u)
#pragma unroll
                    for (int v = 0; v < 3; ++v) acc[u][v] += li[u] * lj[v];
            }
#pragma unroll
            for (int u = 0; u < 3; ++u)
#pragma unroll
                for (int v = 0; v < 3; ++v) {
                    const int i = q + ti + 16 * u, j = q + tj + 16 * v;
                    if (i < kb && j <= i) S[i * LDS + j] -= acc[u][v];
                }
        }
        __syncthreads();
    }

    // write L back (zeros above the diagonal)
    {
        const int c = tid & 63;
        for (int r = tid >> 6; r < kb; r += NTHREADS / 64)
            if (c < kb) A[(long)(k0 + r) * lda + k0 + c] = (c <= r) ? S[r * LDS + c] : T(0);
    }

    // X = L^-1.  Step A: every tile but the last was inverted during step (b)
    // of its panel; the last one now
    if (warp == SPARE) tile_inverse(p_last);
    __syncthreads();
    // Step B: block rows I = 1, 2, 3: Tb = -sum_{m < 16 I} L[16I + r][m] X[m][c],
    // then X[16I + r][c] = sum_{j <= r} X_II[r][j] Tb[j][c] for c < 16 I
    for (int I0 = PW; I0 < kb; I0 += PW) {
        const int rows = kb - I0 < PW ? kb - I0 : PW;
        for (int e = tid; e < PW * I0; e += NTHREADS) {
            const int r = e / I0, c = e - (e / I0) * I0;
            T acc[4] = {T(0), T(0), T(0), T(0)};  // four independent chains over mm
            if (r < rows) {
                const T* lr = S + (I0 + r) * LDS;
                int mm = c;
                for (; mm + 3 < I0; mm += 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc[u] -= lr[mm + u] * X[(mm + u) * LDS + c];
                }
                for (; mm < I0; ++mm) acc[0] -= lr[mm] * X[mm * LDS + c];
            }
            Tb[r * NB + c] = (acc[0] + acc[1]) + (acc[2] + acc[3]);
        }
        __syncthreads();
        for (int e = tid; e < PW * I0; e += NTHREADS) {
            const int r = e / I0, c = e - (e / I0) * I0;
            if (r < rows) {
                const T* xr = X + (I0 + r) * LDS + I0;
                T acc[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
                for (int j = 0; j < PW; ++j)
                    if (j <= r) acc[j & 3] += xr[j] * Tb[j * NB + c];
                X[(I0 + r) * LDS + c] = (acc[0] + acc[1]) + (acc[2] + acc[3]);
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < kb * kb; e += NTHREADS) {
        const int r = e / kb, c = e - (e / kb) * kb;
        Dinv[r * kb + c] = X[r * LDS + c];
    }
    if (tid == 0 && bad && info && info[b] == 0) info[b] = bad;
}

}  // namespace cf_diag
