// Pieces of the blocked triangular solves of the likelihood's chi2 kernels
// (FP64 arithmetic on an FP64 or FP32 row-major lower Cholesky factor L).
//
// A solve runs over 32-row blocks: warp 0 solves the 32 x 32 diagonal block
// in registers (lane = row for L z = x, lane = column for L^T v = w, one
// shuffle per step, reciprocal pivots), then every thread of the CTA applies
// one 32-wide segment of L to the rest of the vector.  With the inverses of
// the factor's 64 x 64 diagonal blocks at hand (both Cholesky kernels keep
// them) a solve runs over 64-row blocks instead, each diagonal solve one
// parallel block-times-vector product (block_matvec).  The vector lives in
// shared memory; the segments are read with vector loads (a thread's 32
// elements of one row are contiguous), all of them in flight at once.
#pragma once

#include "cf_common.cuh"

namespace cf_tri {

// Forward solve of the diagonal block rows b0 .. b0 + kb - 1 (call from one warp).
template <typename T>
__device__ __forceinline__ void diag_forward(const T* L, long lda, int b0, int kb, double* z, int lane)
{
    double lrow[32];
    const T* row = L + (long)(b0 + lane) * lda + b0;
#pragma unroll
    for (int k = 0; k < 32; ++k) lrow[k] = (lane < kb && k < lane) ? (double)row[k] : 0.0;
    const double rinv = lane < kb ? 1.0 / (double)row[lane] : 0.0;
    double zi = lane < kb ? z[b0 + lane] : 0.0;
#pragma unroll
    for (int r = 0; r < 32; ++r) {
        if (r < kb) {
            if (lane == r) zi *= rinv;
            const double zr = __shfl_sync(0xffffffffu, zi, r);
            if (lane > r) zi -= lrow[r] * zr;
        }
    }
    if (lane < kb) z[b0 + lane] = zi;
}

// Backward solve L_bb^T v_b = v_b of the diagonal block rows b0 .. b0 + kb - 1
// (call from one warp; lane i holds column i of the block).
template <typename T>
__device__ __forceinline__ void diag_backward(const T* L, long lda, int b0, int kb, double* v, int lane)
{
    double lcol[32];
    const T* col = L + (long)b0 * lda + b0 + lane;
#pragma unroll
    for (int k = 0; k < 32; ++k) lcol[k] = (lane < kb && k > lane && k < kb) ? (double)col[(long)k * lda] : 0.0;
    const double rinv = lane < kb ? 1.0 / (double)col[(long)lane * lda] : 0.0;
    double vi = lane < kb ? v[b0 + lane] : 0.0;
#pragma unroll
    for (int r = 31; r >= 0; --r) {
        if (r < kb) {
            if (lane == r) vi *= rinv;
            const double vr = __shfl_sync(0xffffffffu, vi, r);
            if (lane < r) vi -= lcol[r] * vr;
        }
    }
    if (lane < kb) v[b0 + lane] = vi;
}

// sum_k row[k] zb[k] over one row segment of kb <= 32 elements; VEC: the
// segment starts on a 16-byte boundary (vector loads when kb == 32).
template <bool VEC>
__device__ __forceinline__ double seg_dot(const double* row, const double* zb, int kb)
{
    double acc = 0.0;
    if (VEC && kb == 32) {
        double2 q[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) q[j] = reinterpret_cast<const double2*>(row)[j];
#pragma unroll
        for (int j = 0; j < 16; ++j) acc += q[j].x * zb[2 * j] + q[j].y * zb[2 * j + 1];
    } else {
        for (int k = 0; k < kb; ++k) acc += row[k] * zb[k];
    }
    return acc;
}

template <bool VEC>
__device__ __forceinline__ double seg_dot(const float* row, const double* zb, int kb)
{
    double acc = 0.0;
    if (VEC && kb == 32) {
        float4 q[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) q[j] = reinterpret_cast<const float4*>(row)[j];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            acc += (double)q[j].x * zb[4 * j] + (double)q[j].y * zb[4 * j + 1] + (double)q[j].z * zb[4 * j + 2] +
                   (double)q[j].w * zb[4 * j + 3];
    } else {
        for (int k = 0; k < kb; ++k) acc += (double)row[k] * zb[k];
    }
    return acc;
}

// sum_k L[b0 + k, i] vb[k], k < kb: column i of the block row (one element per
// row, the warp's lanes on consecutive columns).
template <typename T>
__device__ __forceinline__ double col_dot(const T* L, long lda, int b0, int i, const double* vb, int kb)
{
    const T* c = L + (long)b0 * lda + i;
    double acc = 0.0;
    if (kb == 32) {
        T q[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) q[k] = c[(long)k * lda];
#pragma unroll
        for (int k = 0; k < 32; ++k) acc += (double)q[k] * vb[k];
    } else {
        for (int k = 0; k < kb; ++k) acc += (double)c[(long)k * lda] * vb[k];
    }
    return acc;
}

// out[r] = sum_c D[r kb + c] v[c] (TRANS: D[c kb + r]) for r < kb <= 64: a
// 64 x 64 block (row-major, row stride kb) times a vector, 256 threads, four
// per output row (16 columns each, combined by shuffles).
template <typename T, bool TRANS>
__device__ __forceinline__ void block_matvec(const T* D, int kb, const double* v, double* out, int tid)
{
    const int r = tid >> 2, p = tid & 3;
    double acc = 0.0;
    if (r < kb) {
#pragma unroll 4
        for (int c = p * 16; c < p * 16 + 16; ++c)
            if (c < kb) acc += (double)(TRANS ? D[(long)c * kb + r] : D[(long)r * kb + c]) * v[c];
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    if (r < kb && p == 0) out[r] = acc;
}

// Row segment of up to 64 elements (two halves of 32).
template <bool VEC, typename T>
__device__ __forceinline__ double seg_dot64(const T* row, const double* zb, int kb)
{
    if (kb <= 32) return seg_dot<VEC>(row, zb, kb);
    return seg_dot<VEC>(row, zb, 32) + seg_dot<VEC>(row + 32, zb + 32, kb - 32);
}

// Column of a block row of up to 64 rows (two halves of 32).
template <typename T>
__device__ __forceinline__ double col_dot64(const T* L, long lda, int b0, int i, const double* vb, int kb)
{
    if (kb <= 32) return col_dot(L, lda, b0, i, vb, kb);
    return col_dot(L, lda, b0, i, vb, 32) + col_dot(L, lda, b0 + 32, i, vb + 32, kb - 32);
}

}  // namespace cf_tri
