// FP32 GEMM C = alpha A B^T + beta C on the tcgen05 tensor cores with BF16
// split products (sm_100a), for the likelihood's FP32 Cholesky.
//
// Each operand is split in registers into three BF16 planes,
// a = a0 + a1 + a2 (a0 = bf16(a), a1 = bf16(a - a0), a2 = bf16(a - a0 - a1)),
// and C += sum over the six plane pairs (0,0), (0,1), (1,0), (0,2), (1,1),
// (2,0) (kind::f16 MMAs, FP32 accumulation in TMEM): about 24 significant
// bits per product, the FP32 factor's own rounding level, at tensor-core
// rate instead of the SIMT pipe's.  The leading product (0,0) and the five
// corrections go to two TMEM accumulators, added in the epilogue, so the
// small terms are not summed into the large one inside the tensor core.
// Both operands are K-contiguous ("NT"), as the blocked Cholesky's panel
// solves and trailing updates use them; batch on blockIdx.z.
//
// One 128 x BN output tile per CTA (256 threads).  K runs in chunks of 64
// (one 128-byte BF16 row per operand row and plane).  Every thread holds its
// share of a chunk in registers (float4 loads, two 256-byte row segments per
// warp), splits it and stores the planes in the 128-byte swizzled K-major
// layout the MMA descriptors describe; thread 0 issues the 24 MMAs of the
// chunk and commits them to the stage's mbarrier, and the threads go on to
// load chunk c + 1 while those MMAs run.  One stage (two CTAs per SM) or two
// (one CTA per SM).  The epilogue reads both accumulators with tcgen05.ld
// (thread = output row), turns each warp's 32 x 32 pieces around in shared
// memory and writes alpha (acc0 + acc1) + beta C in coalesced row segments;
// a warp's 32 C segments are all in flight at once, the first piece's before
// the last MMA wait.  Every barrier wait is bounded; a wait that runs out
// makes the CTA drain its MMAs, free its TMEM and set info[z] = -3.
#include <cuda_bf16.h>

#include "cf_common.cuh"
#include "tc_sgemm.cuh"

namespace {

constexpr int BM = 128, KC = 64, NT = 256, PLANES = 3;
constexpr uint32_t A_BYTES = BM * KC * 2;  // one BF16 plane of the A chunk (16 KB)
constexpr unsigned long long DRAIN_NS = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(200000u)
        : "memory");
    return ok != 0;
}

// Non-blocking probe of a barrier phase (no suspend hint).
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Wait bounded in time; false when the bound ran out.  Bounds under 1 ms
// probe without suspending (try_wait may sleep up to its hint) and read the
// clock on every probe, so a bound of 0 gives up at the first unsatisfied one.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long wait_ns)
{
    const unsigned long long t0 = now_ns();
    const bool tight = wait_ns < 1000000ull;
    for (unsigned i = 0;; ++i) {
        if (tight ? mbar_test(bar, parity) : mbar_try(bar, parity)) return true;
        if ((tight || (i & 255) == 255) && now_ns() - t0 >= wait_ns) return false;
    }
}

// K-major operand rows of 128 bytes, 128-byte swizzle: 8-row atoms 1024 B apart.
__device__ __forceinline__ uint64_t smem_desc(const void* tile)
{
    const uint64_t addr = smem_u32(tile);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;         // start address
    d |= (uint64_t)(16 >> 4) << 16;       // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;     // stride byte offset: 8 rows of 128 B
    d |= (uint64_t)1 << 46;               // descriptor version (sm100)
    d |= (uint64_t)2 << 61;               // SWIZZLE_128B
    return d;
}

template <int BN>
__device__ __forceinline__ uint32_t instr_desc_bf16()
{
    // D = F32, A = B = BF16, both K-major, M = 128, N = BN.
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Byte offset of element (r, k), k < 64, in a 128-byte-swizzled K-major BF16 tile.
__device__ __forceinline__ uint32_t swz(int r, int k)
{
    return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((((k >> 3) ^ (r & 7)) << 4) | ((k & 7) << 1)));
}

// rows x 64 chunk of a K-contiguous FP32 operand (row r0.., column k0..) in
// registers: thread tid holds float4 i at row (i NT + tid) / 16, columns
// 4 ((i NT + tid) % 16) ..  + 3, so a warp reads two 256-byte row segments.
// VEC: rows start on 16-byte boundaries (ld, base and batch stride multiples
// of 4 floats), float4 loads; otherwise (or at the K edge) scalar loads.
template <int ROWS, bool VEC>
__device__ __forceinline__ void load_operand(const float* X, long ld, int r0, int nrows, int k0, int K,
                                             float4 (&v)[ROWS / 16], int tid)
{
#pragma unroll
    for (int i = 0; i < ROWS / 16; ++i) {
        const int e = i * NT + tid, r = e >> 4, k = (e & 15) * 4;
        const int gr = r0 + r, gk = k0 + k;
        const float* p = X + (long)gr * ld + gk;
        if (VEC && gr < nrows && gk + 3 < K) {
            v[i] = *reinterpret_cast<const float4*>(p);
        } else {
            v[i].x = (gr < nrows && gk < K) ? p[0] : 0.0f;
            v[i].y = (gr < nrows && gk + 1 < K) ? p[1] : 0.0f;
            v[i].z = (gr < nrows && gk + 2 < K) ? p[2] : 0.0f;
            v[i].w = (gr < nrows && gk + 3 < K) ? p[3] : 0.0f;
        }
    }
}

__device__ __forceinline__ void split3(float x, __nv_bfloat16& p0, __nv_bfloat16& p1, __nv_bfloat16& p2)
{
    p0 = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(p0);
    p1 = __float2bfloat16_rn(r1);
    p2 = __float2bfloat16_rn(r1 - __bfloat162float(p1));
}

// The registers of load_operand as three BF16 planes `plane` bytes apart, in
// the 128-byte-swizzled K-major layout (4 consecutive k share one 8-byte word).
template <int ROWS>
__device__ __forceinline__ void store_operand(const float4 (&v)[ROWS / 16], uint8_t* dst, uint32_t plane, int tid)
{
#pragma unroll
    for (int i = 0; i < ROWS / 16; ++i) {
        const int e = i * NT + tid, r = e >> 4, k = (e & 15) * 4;
        __nv_bfloat16 a[3][4];
        split3(v[i].x, a[0][0], a[1][0], a[2][0]);
        split3(v[i].y, a[0][1], a[1][1], a[2][1]);
        split3(v[i].z, a[0][2], a[1][2], a[2][2]);
        split3(v[i].w, a[0][3], a[1][3], a[2][3]);
        const uint32_t o = swz(r, k);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            uint2 w;
            w.x = (uint32_t)__bfloat16_as_ushort(a[q][0]) | ((uint32_t)__bfloat16_as_ushort(a[q][1]) << 16);
            w.y = (uint32_t)__bfloat16_as_ushort(a[q][2]) | ((uint32_t)__bfloat16_as_ushort(a[q][3]) << 16);
            *reinterpret_cast<uint2*>(dst + q * plane + o) = w;
        }
    }
}

// 16-byte pieces of a rows x 64 chunk of three BF16 planes (row r0.., column
// k0..) into the swizzled stage with cp.async; pieces past the rows or K are
// zero-filled (a piece that straddles K copies only its leading elements).
template <int ROWS>
__device__ __forceinline__ void copy_planes(const __nv_bfloat16* X, long ld, long ps, int r0, int nrows, int k0, int K,
                                            uint8_t* dst, uint32_t plane_bytes, int tid)
{
    constexpr int PIECES = PLANES * ROWS * 8;
#pragma unroll
    for (int i = 0; i < PIECES / NT; ++i) {
        const int e = i * NT + tid;
        const int pl = e / (ROWS * 8), rem = e - pl * (ROWS * 8), r = rem >> 3, j = rem & 7;
        const int gr = r0 + r, gk = k0 + j * 8;
        const int left = gr < nrows ? K - gk : 0;
        const int bytes = left >= 8 ? 16 : (left > 0 ? 2 * left : 0);
        const __nv_bfloat16* src = bytes ? X + (long)pl * ps + (long)gr * ld + gk : X;
        const uint32_t d = smem_u32(dst + pl * plane_bytes + (r >> 3) * 1024 + (r & 7) * 128 + ((j ^ (r & 7)) << 4));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
    }
}

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// PI: operands are BF16 split planes (cp.async into the stage), else FP32
// (registers, split in the kernel).  PO: the result also goes out as split
// planes.
template <int BN, int STAGES, bool VEC, bool PI, bool PO>
__global__ void __launch_bounds__(NT, STAGES == 1 ? 2 : 1) k_sgemm_bf16x6(int M, int N, int K, float alpha,
                                                                          cf_sg::Opnd A, cf_sg::Opnd B, float beta,
                                                                          cf_sg::Out o, int lower_only,
                                                                          unsigned long long wait_ns, int* info)
{
    constexpr uint32_t B_BYTES = BN * KC * 2;
    constexpr uint32_t STAGE = PLANES * (A_BYTES + B_BYTES);
    constexpr uint32_t TMEM_COLS = 2 * BN;  // leading product | corrections
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    __shared__ uint64_t done[2];
    __shared__ uint64_t drain;
    __shared__ uint32_t tmem_slot;

    const int tile_m = blockIdx.y * BM, tile_n = blockIdx.x * BN;
    if ((lower_only & 1) && tile_n > tile_m + BM - 1) return;  // whole CTA, before any allocation
    const long z = blockIdx.z;
    float* C = o.C ? o.C + z * o.sC : nullptr;
    float* C2 = o.C2 ? o.C2 + z * o.sC2 : nullptr;
    __nv_bfloat16* Cp = o.Cp ? o.Cp + z * o.sCp : nullptr;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nch = (K + KC - 1) / KC;
    const float* Af = PI ? nullptr : (const float*)A.p + z * A.sz;
    const float* Bf = PI ? nullptr : (const float*)B.p + z * B.sz;
    const __nv_bfloat16* Ap = PI ? (const __nv_bfloat16*)A.p + z * A.sz : nullptr;
    const __nv_bfloat16* Bp = PI ? (const __nv_bfloat16*)B.p + z * B.sz : nullptr;
    // the first chunks' operands are in flight while the barriers and TMEM are set up
    float4 ra[PI ? 1 : BM / 16], rb[PI ? 1 : BN / 16];
    if constexpr (PI) {
#pragma unroll
        for (int c = 0; c < STAGES; ++c) {  // one copy group per chunk, in order
            if (c < nch) {
                copy_planes<BM>(Ap, A.ld, A.ps, tile_m, M, c * KC, K, smem + c * STAGE, A_BYTES, tid);
                copy_planes<BN>(Bp, B.ld, B.ps, tile_n, N, c * KC, K, smem + c * STAGE + PLANES * A_BYTES, B_BYTES,
                                tid);
            }
            cp_commit();
        }
    } else if (nch > 0) {
        load_operand<BM, VEC>(Af, A.ld, tile_m, M, 0, K, ra, tid);
        load_operand<BN, VEC>(Bf, B.ld, tile_n, N, 0, K, rb, tid);
    }
    if (tid == 0) {
        mbar_init(&done[0], 1);
        mbar_init(&done[1], 1);
        mbar_init(&drain, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = instr_desc_bf16<BN>();

    bool aborted = false;
    for (int c = 0; c < nch; ++c) {
        const int s = c % STAGES;
        uint8_t* sa = smem + s * STAGE;  // A planes 0, 1, 2, then B planes 0, 1, 2
        uint8_t* sb = sa + PLANES * A_BYTES;
        if constexpr (PI) {
            cp_wait<STAGES - 1>();  // chunk c's group has landed
        } else {
            // the MMAs of chunk c - STAGES read this stage: wait for them before overwriting it
            bool ok = c < STAGES || mbar_wait(&done[s], (uint32_t)(((c - STAGES) / STAGES) & 1), wait_ns);
            if (__syncthreads_or(!ok)) {
                aborted = true;
                break;
            }
            store_operand<BM>(ra, sa, A_BYTES, tid);
            store_operand<BN>(rb, sb, B_BYTES, tid);
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            constexpr int TA[6] = {0, 0, 1, 0, 1, 2}, TB[6] = {0, 1, 0, 2, 1, 0};
#pragma unroll
            for (int t = 0; t < 6; ++t) {
                const uint64_t da = smem_desc(sa + TA[t] * A_BYTES), db = smem_desc(sb + TB[t] * B_BYTES);
                const uint32_t dst = tmem + (t > 0 ? (uint32_t)BN : 0u);
                const bool fresh = c == 0 && t <= 1;  // first write of each accumulator
#pragma unroll
                for (int k = 0; k < KC / 16; ++k) {  // 16 BF16 = 32 B per MMA: advance the start address
                    const uint64_t off = (uint64_t)((k * 32) >> 4);
                    umma_bf16(dst, da + off, db + off, idesc, (fresh && k == 0) ? 0u : 1u);
                }
            }
            umma_commit(&done[s]);
        }
        if constexpr (PI) {
            // refill this stage with chunk c + STAGES once chunk c's MMAs are done with it
            if (c + STAGES < nch) {
                const bool ok = mbar_wait(&done[s], (uint32_t)((c / STAGES) & 1), wait_ns);
                if (__syncthreads_or(!ok)) {
                    aborted = true;
                    break;
                }
                copy_planes<BM>(Ap, A.ld, A.ps, tile_m, M, (c + STAGES) * KC, K, sa, A_BYTES, tid);
                copy_planes<BN>(Bp, B.ld, B.ps, tile_n, N, (c + STAGES) * KC, K, sb, B_BYTES, tid);
            }
            cp_commit();
        } else if (c + 1 < nch) {
            // the next chunk's loads overlap this chunk's MMAs
            load_operand<BM, VEC>(Af, A.ld, tile_m, M, (c + 1) * KC, K, ra, tid);
            load_operand<BN, VEC>(Bf, B.ld, tile_n, N, (c + 1) * KC, K, rb, tid);
        }
    }
    if constexpr (PI) cp_wait<0>();  // no copy into the stages outlives the loop
    // Thread = output row in TMEM; each warp turns its 32 x 32 pieces around in
    // shared memory so that C is read and written in 128-byte row segments.
    // The C segments of the warp's first piece are read before the last wait.
    const int quad = warp & 3;  // a warp reads TMEM lanes 32 (warp % 4) .. + 31
    const int col = lane;
    float cv[32];
    auto load_c = [&](int g) {
        const int c = tile_n + g * 32 + col;
#pragma unroll
        for (int r = 0; r < 32; ++r) {
            const int row = tile_m + quad * 32 + r;
            cv[r] = (beta != 0.0f && C && row < M && c < N) ? C[(long)row * o.ldc + c] : 0.0f;
        }
    };
    const int g0 = warp >> 2;
    if (!aborted) load_c(g0);
    bool ok = !aborted;
    if (ok && nch > 0) {
        const int cl = nch - 1;
        ok = mbar_wait(&done[cl % STAGES], (uint32_t)((cl / STAGES) & 1), wait_ns);
    }
    if (__syncthreads_or(!ok)) {
        // drain: every MMA issued has completed before TMEM is freed
        if (tid == 0) {
            umma_commit(&drain);
            const unsigned long long t0 = now_ns();
            while (!mbar_try(&drain, 0) && now_ns() - t0 < DRAIN_NS) {
            }
        }
        if (tid == 0 && info) atomicCAS(info + z, 0, CF_ERR_TIMEOUT);
    } else if (nch > 0) {
        // the operand stages are free now: every MMA has completed
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t lane_addr = tmem + ((uint32_t)(quad * 32) << 16);
        float* T = reinterpret_cast<float*>(smem) + warp * 32 * 33;
#pragma unroll 1
        for (int g = g0; g < BN / 32; g += NT / 128) {  // the two warps of a quadrant split the columns
            if (g != g0) load_c(g);
            {
                uint32_t v[32];
                tmem_ld32(lane_addr + (uint32_t)(g * 32), v);
#pragma unroll
                for (int j = 0; j < 32; ++j) T[lane * 33 + j] = __uint_as_float(v[j]);
                tmem_ld32(lane_addr + (uint32_t)(BN + g * 32), v);
#pragma unroll
                for (int j = 0; j < 32; ++j) T[lane * 33 + j] += __uint_as_float(v[j]);
            }
            __syncwarp();
            const int c = tile_n + g * 32 + col;
#pragma unroll
            for (int r = 0; r < 32; ++r) {
                const int row = tile_m + quad * 32 + r;
                if (row < M && c < N) {
                    const float out = alpha * T[r * 33 + col] + beta * cv[r];
                    if (C) C[(long)row * o.ldc + c] = out;
                    if (C2) C2[(long)row * o.ldc2 + c] = out;
                    if constexpr (PO) {
                        __nv_bfloat16 h0, h1, h2;
                        split3(out, h0, h1, h2);
                        __nv_bfloat16* q = Cp + (long)row * o.ldcp + c;
                        q[0] = h0;
                        q[o.cp_ps] = h1;
                        q[2 * o.cp_ps] = h2;
                    }
                }
            }
            __syncwarp();
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

unsigned long long g_sgemm_wait_ns = DRAIN_NS;
// Operand stages: 2 (double buffer, one CTA per SM) or 1 (two CTAs per SM
// overlap each other's loads and MMAs).
int g_sgemm_stages = 1;

template <int BN, int STAGES, bool VEC, bool PI, bool PO>
int launch_t(int M, int N, int K, float alpha, const cf_sg::Opnd& A, const cf_sg::Opnd& B, float beta,
             const cf_sg::Out& o, int batch, int lower_only, int* info, cudaStream_t st)
{
    constexpr size_t smem = 1024 + STAGES * (size_t)PLANES * (A_BYTES + (size_t)BN * KC * 2);
    static_assert(smem <= 232448, "shared memory exceeds 227 KB");
    static std::atomic<int> attr[CF_MAX_DEVICES];
    if (int rc = cf_smem_optin(k_sgemm_bf16x6<BN, STAGES, VEC, PI, PO>, (int)smem, attr)) return rc;
    dim3 grid(cf_cdiv(N, BN), cf_cdiv(M, BM), batch);
    k_sgemm_bf16x6<BN, STAGES, VEC, PI, PO><<<grid, NT, smem, st>>>(M, N, K, alpha, A, B, beta, o, lower_only,
                                                                    g_sgemm_wait_ns, info);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

inline bool aligned16(const void* p, long ld, long stride, int batch, int per16)
{
    return ((uintptr_t)p & 15) == 0 && (ld % per16) == 0 && (batch == 1 || (stride % per16) == 0);
}

template <int BN, int STAGES>
int launch(int M, int N, int K, float alpha, const cf_sg::Opnd& A, const cf_sg::Opnd& B, float beta,
           const cf_sg::Out& o, bool pi, int batch, int lower_only, int* info, cudaStream_t st)
{
    if (pi) {
        if (o.Cp) return CF_ERR_UNSUPPORTED;
        return launch_t<BN, STAGES, false, true, false>(M, N, K, alpha, A, B, beta, o, batch, lower_only, info, st);
    }
    const bool vec = aligned16(A.p, A.ld, A.sz, batch, 4) && aligned16(B.p, B.ld, B.sz, batch, 4);
    if (o.Cp)
        return vec ? launch_t<BN, STAGES, true, false, true>(M, N, K, alpha, A, B, beta, o, batch, lower_only, info,
                                                             st)
                   : launch_t<BN, STAGES, false, false, true>(M, N, K, alpha, A, B, beta, o, batch, lower_only, info,
                                                              st);
    return vec ? launch_t<BN, STAGES, true, false, false>(M, N, K, alpha, A, B, beta, o, batch, lower_only, info, st)
               : launch_t<BN, STAGES, false, false, false>(M, N, K, alpha, A, B, beta, o, batch, lower_only, info,
                                                           st);
}

}  // namespace

namespace cf_sg {
int sgemm(int M, int N, int K, float alpha, const Opnd& A, const Opnd& B, float beta, const Out& o, bool planes_in,
          int batch, int lower_only, int* info, cudaStream_t st)
{
    if (M < 0 || N < 0 || K < 0 || batch < 1 || (!o.C && !o.C2 && !o.Cp) || (K > 0 && (!A.p || !B.p)))
        return CF_ERR_ARG;
    if (beta != 0.0f && !o.C) return CF_ERR_ARG;
    if (M == 0 || N == 0) return CF_OK;
    if (planes_in && !(aligned16(A.p, A.ld, A.sz, batch, 8) && aligned16(B.p, B.ld, B.sz, batch, 8) &&
                       A.ps % 8 == 0 && B.ps % 8 == 0))
        return CF_ERR_ARG;
    if (g_sgemm_stages == 2) {
        if (N <= 64) return launch<64, 2>(M, N, K, alpha, A, B, beta, o, planes_in, batch, lower_only, info, st);
        return launch<128, 2>(M, N, K, alpha, A, B, beta, o, planes_in, batch, lower_only, info, st);
    }
    if (N <= 64) return launch<64, 1>(M, N, K, alpha, A, B, beta, o, planes_in, batch, lower_only, info, st);
    return launch<128, 1>(M, N, K, alpha, A, B, beta, o, planes_in, batch, lower_only, info, st);
}
}  // namespace cf_sg

// C_z = alpha A_z B_z^T + beta C_z (FP32, row-major, K contiguous in A and B;
// z < batch with element strides sA, sB, sC) with six BF16 split products on
// the tensor cores.  lower_only bit 0 skips output tiles strictly above the diagonal.
// info (optional, int[batch]): set to -3 for a problem whose tile saw a wait
// run out (left alone when non-zero).
extern "C" int cf_sgemm_bf16x6(int M, int N, int K, float alpha, const float* A, long lda, long sA, const float* B,
                               long ldb, long sB, float beta, float* C, long ldc, long sC, int batch, int lower_only,
                               int* info, void* stream)
{
    if (!C) return CF_ERR_ARG;
    const cf_sg::Opnd a{A, lda, sA, 0}, b{B, ldb, sB, 0};
    const cf_sg::Out o{C, ldc, sC, nullptr, 0, 0, nullptr, 0, 0, 0};
    return cf_sg::sgemm(M, N, K, alpha, a, b, beta, o, false, batch, lower_only, info, (cudaStream_t)stream);
}

// Operand stages of cf_sgemm_bf16x6: 1 (default; two CTAs per SM) or 2 (one
// CTA per SM, double-buffered).  Returns the previous setting.
extern "C" int cf_sgemm_bf16x6_set_stages(int stages)
{
    const int prev = g_sgemm_stages;
    if (stages == 1 || stages == 2) g_sgemm_stages = stages;
    return prev;
}

// Bound of the barrier waits of cf_sgemm_bf16x6, in ns (ns < 0: the default
// 2 s; 0: give up at the first unsatisfied try).  Returns the previous bound.
extern "C" long long cf_sgemm_bf16x6_set_wait_limit(long long ns)
{
    const long long prev = (long long)g_sgemm_wait_ns;
    g_sgemm_wait_ns = ns < 0 ? DRAIN_NS : (unsigned long long)ns;
    return prev;
}
