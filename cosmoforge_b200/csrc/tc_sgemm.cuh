// Internal interface of the tensor-core FP32 GEMM (tc_sgemm.cu) for the FP32
// Cholesky (chol_f32.cu): operands and outputs either FP32 or three BF16
// split planes.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace cf_sg {

// An operand, row-major with K contiguous: FP32, or the three BF16 split
// planes of an FP32 matrix (x = x0 + x1 + x2), `ps` elements apart.  `sz`:
// elements between batch entries.
struct Opnd {
    const void* p;
    long ld, sz, ps;
};

// Destinations of alpha A B^T + beta C: FP32 C (read when beta != 0) and/or
// the three BF16 split planes of the result (Cp, row stride ldcp, plane
// stride cp_ps); C2 gets the same FP32 values.  Any pointer may be NULL.
struct Out {
    float* C;
    long ldc, sC;
    float* C2;
    long ldc2, sC2;
    __nv_bfloat16* Cp;
    long ldcp, sCp, cp_ps;
};

// C_z = alpha A_z B_z^T + beta C_z on the tensor cores (six BF16 products).
// planes_in: A and B are split planes, copied into shared memory in 16-byte
// pieces (bases 16-byte aligned; ld, ps, sz multiples of 8 elements; any K);
// else FP32, split in the kernel.  Planes out (o.Cp) need FP32 operands.
// lower_only bit 0 skips output tiles strictly above the diagonal; info[z]
// (optional) is set to -3 when a bounded wait of problem z ran out.
int sgemm(int M, int N, int K, float alpha, const Opnd& A, const Opnd& B, float beta, const Out& o, bool planes_in,
          int batch, int lower_only, int* info, cudaStream_t st);

}  // namespace cf_sg
