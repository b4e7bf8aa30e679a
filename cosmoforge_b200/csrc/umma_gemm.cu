// Split-precision GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   C[M, N] = sum_t A_{a(t)}[M, K] . B_{b(t)}[N, K]^T        (FP32 accumulation in TMEM)
//
// A_s / B_s are BF16 "split planes" of FP64 operands: x = x_0 + x_1 (+ x_2)
// with x_0 = bf16(x), x_1 = bf16(x - x_0), ...  The product list selects
// which plane pairs are multiplied: BF16x3 = {(0,0), (0,1), (1,0)} keeps ~16
// significant bits, BF16x6 adds {(0,2), (1,1), (2,0)} for ~24.  Both operands
// are K-major (row-major with K contiguous).
//
// Structure (one 128 x BN output tile per CTA, 6 warps):
//   warp 0   TMA producer: 128B-swizzled boxes of A and B into a STAGES-deep
//            shared-memory ring, completion counted on per-stage mbarriers;
//   warp 1   allocates the TMEM accumulator and issues tcgen05.mma from one
//            thread; tcgen05.commit releases each stage and finally signals
//            the epilogue;
//   warps 2-5  epilogue: tcgen05.ld of the accumulator (one TMEM lane per
//            output row), then either BF16 split planes of the result (row-
//            major and/or transposed) or FP32.
// Every wait on an mbarrier is bounded; on timeout the CTA records an error,
// drains, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <type_traits>

#include "cf_common.cuh"

namespace {

constexpr int BM = 128, BK = 64, NTHREADS = 320;  // producer, MMA, 8 epilogue warps
constexpr int EPI_WARPS = 8;
constexpr unsigned long long WAIT_NS = 2000000000ull;  // 2 s bound on any single wait
constexpr int MAX_TERMS = 6;

struct Terms {
    int n;
    int a[MAX_TERMS];
    int b[MAX_TERMS];
};

// Trace mode: the K index runs over the (k, l) plane, k < K1, l < K2, and
// the CTA's share of it is blockIdx.z of gridDim.z; the result is scaled and
// added into an FP64 matrix F at (p_off + row, q_off + col) (and its mirror).
struct TraceArgs {
    int K1, K2;
    double* F;
    long ldF, p_off, q_off;
    int sym;
    double scale;
    const int* row_map;  // optional: F row of output row p (instead of p_off + p)
    const int* col_map;  // optional: F column of output column q
};

struct EpiArgs {
    __nv_bfloat16* X;   // [planes][M][ldx]
    long ldx, x_plane;
    int x_planes;
    __nv_bfloat16* XT;  // [planes][N][ldxt]
    long ldxt, xt_plane;
    float* Cf;          // [M][ldc] fp32
    long ldc;
    int M, N;
    // Scattered FP32 output (col_stride > 0 instead of Cf's row-major form):
    // element (row, col) goes to Cs[col col_stride + (row / fold) fold_ld +
    // row % fold] (fold = 0: + row), and to Cs2 likewise when given.
    float* Cs;
    float* Cs2;
    long col_stride;
    int fold;
    long fold_ld;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
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

// Wait bounded in time (wait_ns; the clock is read every 256 tries, or on
// every try for bounds under 1 ms); false (and the abort flag raised) when it
// runs out.  A bound of 0 gives up at the first unsatisfied try.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                          unsigned long long wait_ns)
{
    const unsigned long long t0 = now_ns();
    const bool tight = wait_ns < 1000000ull;  // probe without suspending (try_wait may sleep up to its hint)
    for (unsigned i = 0;; ++i) {
        if (tight ? mbar_test(bar, parity) : mbar_try(bar, parity)) return true;
        if (*abort_flag) return false;
        if ((tight || (i & 255) == 255) && now_ns() - t0 >= wait_ns) break;
    }
    *abort_flag = 1;
    return false;
}

// Wait bounded in time that ignores the abort flag: drains work already issued.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity)
{
    const unsigned long long t0 = now_ns();
    for (unsigned i = 0;; ++i) {
        if (mbar_try(bar, parity)) return;
        if ((i & 255) == 255 && now_ns() - t0 > WAIT_NS) return;
    }
}

__device__ __forceinline__ void tma_load_3d(const CUtensorMap* map, uint64_t* bar, void* dst, int c0, int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];\n"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(const CUtensorMap* map, uint64_t* bar, void* dst, int c0, int c1, int c2,
                                            int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], [%2];\n"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

// Shared-memory matrix descriptor, K-major rows of BKT BF16: BKT = 64 is the
// 128B swizzle (8-row atoms 1024 B apart), BKT = 32 the 64B swizzle (512 B).
template <int BKT>
__device__ __forceinline__ uint64_t smem_desc(const void* tile)
{
    static_assert(BKT == 64 || BKT == 32, "k-tile of 64 or 32 BF16");
    const uint64_t addr = smem_u32(tile);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;                  // start address
    d |= (uint64_t)(16 >> 4) << 16;                // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)((8 * BKT * 2) >> 4) << 32;     // stride byte offset: 8 rows
    d |= (uint64_t)1 << 46;                        // descriptor version (sm100)
    d |= (uint64_t)(BKT == 64 ? 2 : 4) << 61;      // SWIZZLE_128B / SWIZZLE_64B
    return d;
}

template <int BN, int MM = BM>
__device__ __forceinline__ uint32_t instr_desc()
{
    // D = F32, A = B = BF16, both K-major, M = MM (128, or 256 for a CTA pair), N = BN.
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(MM >> 4) << 24);
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

// --- CTA pairs (cta_group::2): one 256 x BN tile per pair of SMs ---
__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// Address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t at_rank(const void* p, uint32_t rank)
{
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(smem_u32(p)), "r"(rank));
    return out;
}
__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void umma_bf16_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                               uint32_t accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// Arrive on the barrier at this offset in both CTAs of the pair once the MMAs issued so far are done.
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar)
{
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;\n" ::"r"(
            smem_u32(bar)),
        "h"((uint16_t)3)
        : "memory");
}
// A TMA load into this CTA's shared memory whose bytes are counted on the
// pair leader's barrier (mbar: a shared::cluster address); no multicast.
__device__ __forceinline__ void tma_load_3d_pair(const CUtensorMap* map, uint32_t mbar, void* dst, int c0, int c1,
                                                 int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];\n"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(mbar), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}
__device__ __forceinline__ void tma_load_4d_pair(const CUtensorMap* map, uint32_t mbar, void* dst, int c0, int c1,
                                                 int c2, int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], [%2];\n"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(mbar), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t mbar)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(mbar) : "memory");
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

template <int BN, int STAGES, bool TRACE, int KC, int PLS, int BKT, bool SPLIT, int CG = 1>
__global__ void __launch_bounds__(NTHREADS, 1)
    k_umma_gemm(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int K,
                int n_split, Terms terms, EpiArgs epi, TraceArgs tr, int group_m, unsigned long long wait_ns,
                int* err)
{
    // Persistent: each CTA walks output tiles blockIdx.x, +gridDim.x, ...; the
    // shared-memory ring, TMEM and all mbarrier phases carry over between
    // tiles, so the epilogue of one tile overlaps the MMAs of the next.
    // Partial sums are promoted out of TMEM every KC k-tiles: the MMA thread
    // alternates between two TMEM accumulators while the epilogue warps add the
    // finished one into registers (FP32 for GEMM outputs, FP64 for the Fisher
    // traces), so no FP32 tensor-core accumulator sees more than 4 KC steps.
    // Two epilogue warps share each TMEM lane quadrant, each owning half of the
    // BN columns.
    // PLS > 1: one pipeline stage holds planes 0..PLS-1 of both operands' k-tile
    // and the MMA thread issues every product term from it (each plane is read
    // from memory once); PLS == 1: terms are walked one after the other.
    // SPLIT (with PLS > 1, term 0 the leading product of planes (0, 0)): the two
    // TMEM accumulators hold term 0 and the sum of the correction terms of the
    // same chunk instead of alternating, so the small corrections are not added
    // into the large leading sum inside the tensor core; the MMA thread waits
    // for the epilogue to read both before it starts the next chunk.
    // CG == 2: a CTA pair (cluster of two) computes a 256 x BN tile with
    // tcgen05.mma.cta_group::2 issued by the leader (rank 0); each CTA loads
    // its own 128 rows of A and half of the BN rows of B, the loads of both
    // are counted on the leader's barriers, MMA completions are multicast to
    // both CTAs' barriers and each CTA's epilogue drains its own TMEM half
    // (rows 128 rank ..) and reports to the leader.
    static_assert(CG == 1 || (CG == 2 && PLS > 1), "CTA pairs: all-planes forms only");
    using AccT = typename std::conditional<TRACE, double, float>::type;
    constexpr int HALF = BN / 2;
    constexpr int BNL = BN / CG;  // rows of B held by this CTA
    constexpr uint32_t A_BYTES = BM * BKT * 2, B_BYTES = BNL * BKT * 2;
    // stages per promotion chunk: KC k-tiles of 64
    constexpr int CH = PLS > 1 ? KC * (64 / BKT) : KC;
    static_assert(!SPLIT || PLS > 1, "split accumulators need all planes per stage");
    constexpr uint32_t A_STAGE = PLS * A_BYTES, B_STAGE = PLS * B_BYTES;
    constexpr uint32_t TMEM_COLS = 2 * BN <= 64 ? 64 : (2 * BN <= 128 ? 128 : (2 * BN <= 256 ? 256 : 512));
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = smem;
    uint8_t* sB = smem + STAGES * A_STAGE;
    uint64_t* full = (uint64_t*)(sB + STAGES * B_STAGE);
    uint64_t* empty = full + STAGES;
    uint64_t* accf = empty + STAGES;  // [2] accumulator ready
    uint64_t* acce = accf + 2;        // [2] accumulator drained
    uint64_t* dbar = acce + 2;        // MMA drain on abort
    uint32_t* tmem_slot = (uint32_t*)(dbar + 1);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = CG == 2 ? cluster_rank() : 0u;
    const bool leader = rank == 0;
    const long t_first = CG == 2 ? (long)(blockIdx.x >> 1) : (long)blockIdx.x;
    const long t_step = CG == 2 ? (long)(gridDim.x >> 1) : (long)gridDim.x;
    const int n_mt = (epi.M + BM * CG - 1) / (BM * CG), n_nt = (epi.N + BN - 1) / BN;
    const long n_tiles = (long)n_mt * n_nt * n_split;
    const int nl = TRACE ? (tr.K2 + BKT - 1) / BKT : 1;
    const long kt_total = TRACE ? (long)tr.K1 * nl : (long)((K + BKT - 1) / BKT);
    // Tile order: groups of group_m row tiles, the column tiles walked inside
    // a group, so the CTAs running at one time share a few A row panels
    // (L2-resident across the sweep) instead of touching every one of them.
    auto coords = [&](long tile, int& m0, int& n0, long& t_lo, int& kt) {
        const long per_z = (long)n_mt * n_nt;
        const int z = (int)(tile / per_z);
        const long t_in = tile % per_z;
        const int gm_full = group_m < n_mt ? group_m : n_mt;
        const int g = (int)(t_in / ((long)gm_full * n_nt));
        const int gm = min(gm_full, n_mt - g * gm_full);
        const long within = t_in - (long)g * gm_full * n_nt;
        const int mt = g * gm_full + (int)(within % gm);
        const int nt = (int)(within / gm);
        m0 = mt * BM * CG + (int)rank * BM;  // this CTA's rows
        n0 = nt * BN;
        t_lo = kt_total * z / n_split;
        kt = (int)(kt_total * (z + 1) / n_split - t_lo);
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&accf[0], 1);
        mbar_init(&accf[1], 1);
        mbar_init(&acce[0], EPI_WARPS * CG);  // a pair's leader hears both CTAs' epilogues
        mbar_init(&acce[1], EPI_WARPS * CG);
        mbar_init(dbar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 1) {
        if constexpr (CG == 2) {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                             smem_u32(tmem_slot)),
                         "r"(TMEM_COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n");
        } else {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                             smem_u32(tmem_slot)),
                         "r"(TMEM_COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    // a pair's barriers (initialised above) are signalled by the other CTA from here on
    if constexpr (CG == 2) cluster_sync();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            long g = 0;
            bool stop = false;
            for (long tile = t_first; tile < n_tiles && !stop; tile += t_step) {
                int m0, n0, kt;
                long t_lo;
                coords(tile, m0, n0, t_lo, kt);
                const int iters = PLS > 1 ? kt : terms.n * kt;
                for (int it = 0; it < iters; ++it, ++g) {
                    const int s = (int)(g % STAGES);
                    const long r = g / STAGES;
                    if (r > 0 && !mbar_wait(&empty[s], (uint32_t)((r - 1) & 1), abort_flag, wait_ns)) {
                        stop = true;
                        break;
                    }
                    // windows of KC k-tiles, term by term inside a window: every
                    // accumulator chunk holds one product term, and all terms reuse the
                    // window's planes from L2
                    int t = 0;
                    long ktile = t_lo + it;
                    if (PLS == 1) {
                        const int w = it / (KC * terms.n), rem = it % (KC * terms.n);
                        const int wlen = min(KC, kt - w * KC);
                        t = rem / wlen;
                        ktile = t_lo + (long)w * KC + rem % wlen;
                    }
                    // a pair's leader expects both CTAs' bytes on its barrier
                    if (leader) mbar_expect_tx(&full[s], CG * (A_STAGE + B_STAGE));
#pragma unroll
                    for (int pl = 0; pl < PLS; ++pl) {
                        const int pa = PLS > 1 ? pl : terms.a[t], pb = PLS > 1 ? pl : terms.b[t];
                        uint8_t* da = sA + s * A_STAGE + pl * A_BYTES;
                        uint8_t* db = sB + s * B_STAGE + pl * B_BYTES;
                        if (TRACE) {
                            const int k = (int)(ktile / nl), l0 = (int)(ktile % nl) * BKT;
                            if constexpr (CG == 2) {
                                const uint32_t fb = at_rank(&full[s], 0);
                                tma_load_4d_pair(&mapA, fb, da, l0, k, m0, pa);
                                tma_load_4d_pair(&mapB, fb, db, l0, k, n0 + (int)rank * BNL, pb);
                            } else {
                                tma_load_4d(&mapA, &full[s], da, l0, k, m0, pa);
                                tma_load_4d(&mapB, &full[s], db, l0, k, n0, pb);
                            }
                        } else {
                            const int kk = (int)ktile * BKT;
                            if constexpr (CG == 2) {
                                const uint32_t fb = at_rank(&full[s], 0);
                                tma_load_3d_pair(&mapA, fb, da, kk, m0, pa);
                                tma_load_3d_pair(&mapB, fb, db, kk, n0 + (int)rank * BNL, pb);
                            } else {
                                tma_load_3d(&mapA, &full[s], da, kk, m0, pa);
                                tma_load_3d(&mapB, &full[s], db, kk, n0, pb);
                            }
                        }
                    }
                }
            }
            // drain: every issued copy lands before the CTA may exit (a pair's leader
            // sees both CTAs' copies complete; the other waits at the final cluster barrier)
            if (leader)
                for (long q = (g > STAGES ? g - STAGES : 0); q < g; ++q)
                    mbar_drain(&full[q % STAGES], (uint32_t)((q / STAGES) & 1));
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = instr_desc<BN, BM * CG>();
            bool aborted = false;
            long g = 0, gc = 0;
            for (long tile = t_first; tile < n_tiles && !aborted && (CG == 1 || leader); tile += t_step) {
                int m0, n0, kt;
                long t_lo;
                coords(tile, m0, n0, t_lo, kt);
                const int iters = PLS > 1 ? kt : terms.n * kt;
                int buf = 0;
                for (int it = 0; it < iters; ++it, ++g) {
                    // chunk boundaries: every KC iterations (PLS > 1), or at the end of
                    // each (window, term) run of min(KC, k-tiles left) iterations
                    int pos = it % CH, clen = CH;
                    if (PLS == 1) {
                        const int w = it / (KC * terms.n), rem = it % (KC * terms.n);
                        clen = min(KC, kt - w * KC);
                        pos = rem % clen;
                    }
                    const bool first = pos == 0;
                    if (first) {
                        if (SPLIT) {  // both accumulators drained by the epilogue
                            if (gc >= 1 && !mbar_wait(&acce[0], (uint32_t)((gc - 1) & 1), abort_flag, wait_ns)) {
                                aborted = true;
                                break;
                            }
                        } else {
                            buf = (int)(gc & 1);
                            const long u = gc >> 1;
                            if (u >= 1 && !mbar_wait(&acce[buf], (uint32_t)((u - 1) & 1), abort_flag, wait_ns)) {
                                aborted = true;
                                break;
                            }
                        }
                    }
                    const int s = (int)(g % STAGES);
                    if (!mbar_wait(&full[s], (uint32_t)((g / STAGES) & 1), abort_flag, wait_ns)) {
                        aborted = true;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    const int nt = PLS > 1 ? terms.n : 1;
                    for (int t = 0; t < nt; ++t) {
                        const int pa = PLS > 1 ? terms.a[t] : 0, pb = PLS > 1 ? terms.b[t] : 0;
                        const uint64_t ad = smem_desc<BKT>(sA + s * A_STAGE + pa * A_BYTES);
                        const uint64_t bd = smem_desc<BKT>(sB + s * B_STAGE + pb * B_BYTES);
                        // SPLIT: term 0 into columns [0, BN), the others into [BN, 2 BN)
                        const uint32_t dst = tmem + (uint32_t)((SPLIT ? (t > 0) : buf) * BN);
                        const bool fresh = first && (SPLIT ? t <= 1 : t == 0);
#pragma unroll
                        for (int k = 0; k < BKT / 16; ++k) {  // 16 BF16 = 32 B per MMA; advance the start address
                            if constexpr (CG == 2)
                                umma_bf16_pair(dst, ad + (uint64_t)((k * 32) >> 4), bd + (uint64_t)((k * 32) >> 4),
                                               idesc, (fresh && k == 0) ? 0u : 1u);
                            else
                                umma_bf16(dst, ad + (uint64_t)((k * 32) >> 4), bd + (uint64_t)((k * 32) >> 4), idesc,
                                          (fresh && k == 0) ? 0u : 1u);
                        }
                    }
                    if constexpr (CG == 2)
                        umma_commit_pair(&empty[s]);
                    else
                        umma_commit(&empty[s]);
                    if (pos == clen - 1 || it == iters - 1) {
                        if constexpr (CG == 2)
                            umma_commit_pair(&accf[SPLIT ? 0 : buf]);
                        else
                            umma_commit(&accf[SPLIT ? 0 : buf]);
                        ++gc;
                    }
                }
            }
            if (aborted) {  // MMAs already issued finish before TMEM is freed
                if constexpr (CG == 2)
                    umma_commit_pair(dbar);
                else
                    umma_commit(dbar);
                mbar_drain(dbar, 0);
            }
        }
    } else {
        // epilogue warps 2..9: TMEM lanes 32 * (warp % 4) .. + 31 (one output row
        // per thread), columns [half * BN/2, half * BN/2 + BN/2)
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const uint32_t lane_addr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * HALF);
        long gc = 0;
        bool ok = true;
        for (long tile = t_first; tile < n_tiles && ok; tile += t_step) {
            int m0, n0, kt;
            long t_lo;
            coords(tile, m0, n0, t_lo, kt);
            const int iters = PLS > 1 ? kt : terms.n * kt;
            const int nchunks = PLS > 1 ? (iters + CH - 1) / CH : ((kt + KC - 1) / KC) * terms.n;
            AccT acc[HALF];
#pragma unroll
            for (int j = 0; j < HALF; ++j) acc[j] = AccT(0);
            for (int c = 0; c < nchunks; ++c, ++gc) {
                const int buf = SPLIT ? 0 : (int)(gc & 1);
                const uint32_t par = SPLIT ? (uint32_t)(gc & 1) : (uint32_t)((gc >> 1) & 1);
                if (!mbar_wait(&accf[buf], par, abort_flag, wait_ns)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
                for (int gi = 0; gi < HALF / 32; ++gi) {
                    uint32_t v[32];
                    tmem_ld32(lane_addr + (uint32_t)(buf * BN + gi * 32), v);
#pragma unroll
                    for (int j = 0; j < 32; ++j) acc[gi * 32 + j] += (AccT)__uint_as_float(v[j]);
                    if (SPLIT && terms.n > 1) {  // the correction terms' partial sum
                        tmem_ld32(lane_addr + (uint32_t)(BN + gi * 32), v);
#pragma unroll
                        for (int j = 0; j < 32; ++j) acc[gi * 32 + j] += (AccT)__uint_as_float(v[j]);
                    }
                }
                asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    if (CG == 2 && !leader)
                        mbar_arrive_remote(at_rank(&acce[buf], 0));
                    else
                        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&acce[buf])) : "memory");
                }
            }
            const int row = m0 + quad * 32 + lane;
            if (!ok || *abort_flag || iters == 0 || row >= epi.M) continue;
            if (TRACE) {
#pragma unroll
                for (int j = 0; j < HALF; ++j) {
                    const int col = n0 + half * HALF + j;
                    if (col < epi.N) {
                        const double val = tr.scale * (double)acc[j];
                        const long fr = tr.row_map ? (long)tr.row_map[row] : tr.p_off + row;
                        const long fc = tr.col_map ? (long)tr.col_map[col] : tr.q_off + col;
                        atomicAdd(tr.F + fr * tr.ldF + fc, val);
                        if (tr.sym) atomicAdd(tr.F + fc * tr.ldF + fr, val);
                    }
                }
            } else {
                // Row-major planes in 16-byte stores of 8 columns; the transposed
                // planes column by column (32 lanes = 32 consecutive rows).
                const int cbase = n0 + half * HALF;
                if (epi.Cs) {
                    // scattered FP32: one column at a time, the warp's 32 rows consecutive
                    const long roff = epi.fold ? (long)(row / epi.fold) * epi.fold_ld + row % epi.fold : (long)row;
#pragma unroll
                    for (int j = 0; j < HALF; ++j) {
                        if (cbase + j < epi.N) {
                            const long o = (long)(cbase + j) * epi.col_stride + roff;
                            epi.Cs[o] = (float)acc[j];
                            if (epi.Cs2) epi.Cs2[o] = (float)acc[j];
                        }
                    }
                    continue;
                }
#pragma unroll
                for (int j0 = 0; j0 < HALF; j0 += 8) {
                    float x[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) x[u] = (float)acc[j0 + u];
                    if (epi.Cf) {
#pragma unroll
                        for (int u = 0; u < 8; ++u)
                            if (cbase + j0 + u < epi.N) epi.Cf[(long)row * epi.ldc + cbase + j0 + u] = x[u];
                    }
                    for (int p = 0; p < epi.x_planes && (epi.X || epi.XT); ++p) {
                        __nv_bfloat16 h[8];
#pragma unroll
                        for (int u = 0; u < 8; ++u) {
                            h[u] = __float2bfloat16_rn(x[u]);
                            x[u] -= __bfloat162float(h[u]);
                        }
                        if (epi.X) {
                            __nv_bfloat16* dst = epi.X + p * epi.x_plane + (long)row * epi.ldx + cbase + j0;
                            if (cbase + j0 + 8 <= epi.N) {
                                uint4 w;
                                w.x = (uint32_t)__bfloat16_as_ushort(h[0]) | ((uint32_t)__bfloat16_as_ushort(h[1]) << 16);
                                w.y = (uint32_t)__bfloat16_as_ushort(h[2]) | ((uint32_t)__bfloat16_as_ushort(h[3]) << 16);
                                w.z = (uint32_t)__bfloat16_as_ushort(h[4]) | ((uint32_t)__bfloat16_as_ushort(h[5]) << 16);
                                w.w = (uint32_t)__bfloat16_as_ushort(h[6]) | ((uint32_t)__bfloat16_as_ushort(h[7]) << 16);
                                *reinterpret_cast<uint4*>(dst) = w;
                            } else {
                                for (int u = 0; u < 8; ++u)
                                    if (cbase + j0 + u < epi.N) dst[u] = h[u];
                            }
                        }
                        if (epi.XT) {
#pragma unroll
                            for (int u = 0; u < 8; ++u)
                                if (cbase + j0 + u < epi.N)
                                    epi.XT[p * epi.xt_plane + (long)(cbase + j0 + u) * epi.ldxt + row] = h[u];
                        }
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if constexpr (CG == 2) {
        // neither CTA leaves (or frees its TMEM) while the pair's MMAs or copies may touch it
        cluster_sync();
        if (warp == 1)
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS));
    } else if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS));
    }
    if (threadIdx.x == 0 && *abort_flag && err) atomicExch(err, 1);
}

// --- host: tensor maps through the driver entry point (no link-time libcuda) ---
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        fn = (EncodeTiledFn)p;
    }
    return fn;
}

// 3D bf16 map: dims (K, rows, planes), row stride ld elements, plane stride ps elements;
// box (bk, box_rows, 1): bk = 64 with 128B swizzle, bk = 32 with 64B swizzle.
int make_map(CUtensorMap* map, const void* base, long K, long rows, long ld, int planes, long ps, int box_rows,
             int bk = BK)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return CF_ERR_CUDA;
    if (((uintptr_t)base & 15) || (ld * 2) % 16 || (ps * 2) % 16) return CF_ERR_ARG;
    cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)planes};
    cuuint64_t strides[2] = {(cuuint64_t)ld * 2, (cuuint64_t)(ps > 0 ? ps : ld * rows) * 2};
    cuuint32_t box[3] = {(cuuint32_t)bk, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, bk == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? CF_OK : CF_ERR_ARG;
}

// 4D bf16 map for the trace mode: dims (l: K2, k: K1, row: rows, plane), strides
// ldk (between k), ldr (between rows), ps (between planes), box (64, 1, box_rows, 1).
int make_map4(CUtensorMap* map, const void* base, long K2, long K1, long rows, int planes, long ldk, long ldr,
              long ps, int box_rows)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return CF_ERR_CUDA;
    if (((uintptr_t)base & 15) || (ldk * 2) % 16 || (ldr * 2) % 16 || (ps * 2) % 16) return CF_ERR_ARG;
    cuuint64_t dims[4] = {(cuuint64_t)K2, (cuuint64_t)K1, (cuuint64_t)rows, (cuuint64_t)planes};
    cuuint64_t strides[3] = {(cuuint64_t)ldk * 2, (cuuint64_t)ldr * 2, (cuuint64_t)(ps > 0 ? ps : 16) * 2};
    cuuint32_t box[4] = {(cuuint32_t)BK, 1, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? CF_OK : CF_ERR_ARG;
}

// Promotion interval (k-tiles of 64 per FP32 accumulator): 1, 2, 4, 8, 16 or 32.
int g_promote_kc = 16;
// Trace mode on CTA pairs (256-row output tiles, each CTA holding half of the
// B rows of a 128-column tile) when both operands carry two or three planes.
int g_trace_pairs = 1;
// Row tiles per group of the persistent tile order.
int g_group_m = 16;
// Bound of the kernels' waits on pipeline barriers (drains of issued work keep WAIT_NS).
unsigned long long g_wait_ns = WAIT_NS;

template <int BN, int STAGES, bool TRACE, int KC, int PLS = 1, int BKT = BK, bool SPLIT = false, int CG = 1>
int launch_gemm_kc(const CUtensorMap& ma, const CUtensorMap& mb, int M, int N, int K, const Terms& t,
                   const EpiArgs& e, const TraceArgs& tr, int splits, int* err, cudaStream_t st)
{
    constexpr size_t RING = (size_t)STAGES * PLS * (BM * BKT * 2 + (BN / CG) * BKT * 2);
    const size_t smem = 1024 + RING + 256;
    static_assert(1024 + RING + 256 <= 232448, "shared memory ring exceeds 227 KB");
    auto kern = k_umma_gemm<BN, STAGES, TRACE, KC, PLS, BKT, SPLIT, CG>;
    static std::atomic<int> attr[CF_MAX_DEVICES];
    if (int rc = cf_smem_optin(kern, (int)smem, attr)) return rc;
    int dev = 0, sms = 0;
    CF_CHECK(cudaGetDevice(&dev));
    CF_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long tiles = (long)cf_cdiv(M, BM * CG) * cf_cdiv(N, BN) * splits;
    if constexpr (CG == 2) {
        // clusters of two CTAs on neighbouring SMs, one output tile per pair at a time
        const int np = (int)(tiles < sms / 2 ? tiles : sms / 2);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2 * np);
        cfg.blockDim = dim3(NTHREADS);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 2;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        CF_CHECK(cudaLaunchKernelEx(&cfg, kern, ma, mb, K, splits, t, e, tr, g_group_m, g_wait_ns, err));
        return CF_OK;
    }
    const int grid = (int)(tiles < sms ? tiles : sms);
    kern<<<grid, NTHREADS, smem, st>>>(ma, mb, K, splits, t, e, tr, g_group_m, g_wait_ns, err);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// GEMM mode: 1 = all planes of a 32-wide k-slice per stage with split
// accumulators where the planes allow it, 2 = all three planes of a 64-wide
// k-tile per stage on CTA pairs (256-row tiles, 2 stages of 96 KB per CTA),
// 0 = 64-wide k-tiles term by term.
int g_all_planes = 1;

template <int BN, int STAGES, bool TRACE, int PLS = 1, int BKT = BK, bool SPLIT = false, int CG = 1>
int launch_gemm(const CUtensorMap& ma, const CUtensorMap& mb, int M, int N, int K, const Terms& t,
                const EpiArgs& e, const TraceArgs& tr, int splits, int* err, cudaStream_t st)
{
    switch (g_promote_kc) {
        case 1:
            return launch_gemm_kc<BN, STAGES, TRACE, 1, PLS, BKT, SPLIT, CG>(ma, mb, M, N, K, t, e, tr, splits,
                                                                                   err, st);
        case 2:
            return launch_gemm_kc<BN, STAGES, TRACE, 2, PLS, BKT, SPLIT, CG>(ma, mb, M, N, K, t, e, tr, splits,
                                                                                   err, st);
        case 8:
            return launch_gemm_kc<BN, STAGES, TRACE, 8, PLS, BKT, SPLIT, CG>(ma, mb, M, N, K, t, e, tr, splits,
                                                                                   err, st);
        case 16:
            return launch_gemm_kc<BN, STAGES, TRACE, 16, PLS, BKT, SPLIT, CG>(ma, mb, M, N, K, t, e, tr,
                                                                                    splits, err, st);
        case 32:
            return launch_gemm_kc<BN, STAGES, TRACE, 32, PLS, BKT, SPLIT, CG>(ma, mb, M, N, K, t, e, tr,
                                                                                    splits, err, st);
        default:
            return launch_gemm_kc<BN, STAGES, TRACE, 4, PLS, BKT, SPLIT, CG>(ma, mb, M, N, K, t, e, tr, splits,
                                                                                   err, st);
    }
}

}  // namespace

int cf_umma_trace_impl(int P1, int P2, int K1, int K2, int nterms, const int* ta, const int* tb, const void* X,
                       long sXp, long ldX, long x_ps, int x_planes, const void* Y, long sYq, long ldY, long y_ps,
                       int y_planes, double scale, double* F, long ldF, long p_off, long q_off, int sym,
                       const int* row_map, const int* col_map, int splits, int* err, void* stream);

// Set the promotion interval of the tensor-core kernels (k-tiles of 64 summed
// in one FP32 TMEM accumulator before the partial is promoted): 1, 2, 4,
// 8, 16 (default) or 32.  Returns the previous value.
// Trace contractions on CTA pairs (1, default) or one CTA per output tile (0);
// returns the previous setting.
extern "C" int cf_umma_set_trace_pairs(int on)
{
    const int prev = g_trace_pairs;
    g_trace_pairs = on ? 1 : 0;
    return prev;
}

extern "C" int cf_umma_set_promotion(int kc)
{
    const int prev = g_promote_kc;
    if (kc == 1 || kc == 2 || kc == 4 || kc == 8 || kc == 16 || kc == 32) g_promote_kc = kc;
    return prev;
}

// Bound of every wait of the tcgen05 kernels on a pipeline barrier, in ns
// (ns < 0 restores the default 2 s; 0 gives up at the first unsatisfied
// try).  A wait that runs out aborts the launch: the CTA drains the copies and
// MMAs it issued (those drains keep the 2 s bound), frees its TMEM and sets the
// caller's error flag.  Returns the previous bound.
extern "C" long long cf_umma_set_wait_limit(long long ns)
{
    const long long prev = (long long)g_wait_ns;
    g_wait_ns = ns < 0 ? WAIT_NS : (unsigned long long)ns;
    return prev;
}

// CF_ERR_TIMEOUT when the device error flag of a tcgen05 launch is set (a
// wait ran out), else CF_OK; synchronises `stream` to read it.
extern "C" int cf_umma_status(const int* err, void* stream)
{
    if (!err) return CF_ERR_ARG;
    int h = 0;
    CF_CHECK(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CF_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
    return h ? CF_ERR_TIMEOUT : CF_OK;
}

// Row tiles per group of the persistent tile order (>= 1); returns the previous value.
extern "C" int cf_umma_set_group(int group_m)
{
    const int prev = g_group_m;
    if (group_m >= 1) g_group_m = group_m;
    return prev;
}

// Select the GEMM form (1 = all planes per stage, 2 = all planes on CTA
// pairs, 0 = term by term); returns the previous one.
extern "C" int cf_umma_set_all_planes(int on)
{
    const int prev = g_all_planes;
    g_all_planes = (on == 0 || on == 1 || on == 2) ? on : 1;
    return prev;
}

namespace {
int gemm_bf16(int M, int N, int K, int nterms, const int* ta, const int* tb, const void* A, long lda, long a_ps,
              int a_planes, const void* B, long ldb, long b_ps, int b_planes, const EpiArgs& e, int* err,
              cudaStream_t st)
{
    if (M <= 0 || N <= 0 || K <= 0 || nterms < 1 || nterms > MAX_TERMS || !A || !B) return CF_ERR_ARG;
    Terms t{};
    t.n = nterms;
    for (int i = 0; i < nterms; ++i) {
        if (ta[i] < 0 || ta[i] >= a_planes || tb[i] < 0 || tb[i] >= b_planes) return CF_ERR_ARG;
        t.a[i] = ta[i];
        t.b[i] = tb[i];
    }
    TraceArgs tr{};
    CUtensorMap ma, mb;
    // All planes of a 32-wide k-slice in one stage (each plane read once per
    // k-slice instead of once per term), the leading term (0, 0) accumulated
    // apart from the corrections; otherwise 64-wide k-tiles walked term by term.
    const int pls = a_planes == b_planes ? a_planes : 0;
    bool all_planes = g_all_planes && (pls == 2 || pls == 3) && t.a[0] == 0 && t.b[0] == 0;
    for (int i = 1; i < nterms && all_planes; ++i) all_planes = !(t.a[i] == 0 && t.b[i] == 0);
    if (all_planes) {
        // form 2: three planes of 64-wide k-tiles on CTA pairs (each CTA holds
        // half of B's 256 rows; 2 stages of 96 KB per CTA)
        if (g_all_planes == 2 && pls == 3) {
            int rc = make_map(&ma, A, K, M, lda, a_planes, a_ps, BM, 64);
            if (rc) return rc;
            rc = make_map(&mb, B, K, N, ldb, b_planes, b_ps, 128, 64);
            if (rc) return rc;
            return launch_gemm<256, 2, false, 3, 64, true, 2>(ma, mb, M, N, K, t, e, tr, 1, err, st);
        }
        int rc = make_map(&ma, A, K, M, lda, a_planes, a_ps, BM, 32);
        if (rc) return rc;
        rc = make_map(&mb, B, K, N, ldb, b_planes, b_ps, 256, 32);
        if (rc) return rc;
        if (pls == 3) return launch_gemm<256, 3, false, 3, 32, true>(ma, mb, M, N, K, t, e, tr, 1, err, st);
        return launch_gemm<256, 4, false, 2, 32, true>(ma, mb, M, N, K, t, e, tr, 1, err, st);
    }
    int rc = make_map(&ma, A, K, M, lda, a_planes, a_ps, BM);
    if (rc) return rc;
    rc = make_map(&mb, B, K, N, ldb, b_planes, b_ps, 256);
    if (rc) return rc;
    return launch_gemm<256, 4, false>(ma, mb, M, N, K, t, e, tr, 1, err, st);
}
}  // namespace

// C = sum_t A_{ta[t]} B_{tb[t]}^T with BF16 split planes, FP32 accumulation.
//   A: planes of M x K (row stride lda, plane stride a_ps), B: planes of N x K.
//   Outputs (any may be NULL): X = C as x_planes BF16 split planes (M x N,
//   ldx, plane stride x_ps); XT = C^T likewise (N x M, ldxt, xt_ps);
//   Cf = C in FP32 (M x N, ldc).  err: device int set to 1 if a wait ran out.
extern "C" int cf_umma_gemm_bf16(int M, int N, int K, int nterms, const int* ta, const int* tb, const void* A,
                                 long lda, long a_ps, int a_planes, const void* B, long ldb, long b_ps,
                                 int b_planes, void* X, long ldx, long x_ps, int x_planes, void* XT, long ldxt,
                                 long xt_ps, float* Cf, long ldc, int* err, void* stream)
{
    if ((X || XT) && (x_planes < 1 || x_planes > 3)) return CF_ERR_ARG;
    EpiArgs e{(__nv_bfloat16*)X, ldx, x_ps, x_planes, (__nv_bfloat16*)XT, ldxt, xt_ps, Cf, ldc, M, N,
              nullptr, nullptr, 0, 0, 0};
    return gemm_bf16(M, N, K, nterms, ta, tb, A, lda, a_ps, a_planes, B, ldb, b_ps, b_planes, e, err,
                     (cudaStream_t)stream);
}

// The same product written in FP32 to scattered addresses: element (row, col)
// of C goes to Cs[col col_stride + (row / fold) fold_ld + row % fold] (fold =
// 0: Cs[col col_stride + row]) and, when Cs2 is given, to the same offset of
// Cs2.  Lanes of a warp hold consecutive rows, so each column's segment of a
// tile is one coalesced store.  Used with rows = the entries of a block
// region of the covariance (fold = region width, fold_ld = the matrix's row
// stride) and columns = parameter points (col_stride = one matrix) to write
// C(theta) for a batch of points straight into its FP32 matrices.
extern "C" int cf_umma_gemm_bf16_scatter(int M, int N, int K, int nterms, const int* ta, const int* tb,
                                         const void* A, long lda, long a_ps, int a_planes, const void* B, long ldb,
                                         long b_ps, int b_planes, float* Cs, float* Cs2, long col_stride, int fold,
                                         long fold_ld, int* err, void* stream)
{
    if (!Cs || col_stride <= 0 || fold < 0) return CF_ERR_ARG;
    EpiArgs e{nullptr, 0, 0, 0, nullptr, 0, 0, nullptr, 0, M, N, Cs, Cs2, col_stride, fold, fold_ld};
    return gemm_bf16(M, N, K, nterms, ta, tb, A, lda, a_ps, a_planes, B, ldb, b_ps, b_planes, e, err,
                     (cudaStream_t)stream);
}

// Fisher contraction on the tensor cores:
//   F[(p_off+p) ldF + q_off+q] += scale sum_t sum_{k<K1, l<K2} X_{ta[t]}[p, k, l] Y_{tb[t]}[q, k, l]
// X_s[p, k, l] = X[s*x_ps + p*sXp + k*ldX + l] (BF16 planes), Y likewise; the
// mirror entry too when sym.  F (FP64) accumulates partial sums of `splits`
// CTAs per output tile with atomics; zero it first.
extern "C" int cf_umma_trace_bf16_mapped(int P1, int P2, int K1, int K2, int nterms, const int* ta,
                                         const int* tb, const void* X, long sXp, long ldX, long x_ps, int x_planes,
                                         const void* Y, long sYq, long ldY, long y_ps, int y_planes, double scale,
                                         double* F, long ldF, const int* row_map, const int* col_map, int sym,
                                         int splits, int* err, void* stream);

extern "C" int cf_umma_trace_bf16(int P1, int P2, int K1, int K2, int nterms, const int* ta, const int* tb,
                                  const void* X, long sXp, long ldX, long x_ps, int x_planes, const void* Y,
                                  long sYq, long ldY, long y_ps, int y_planes, double scale, double* F, long ldF,
                                  long p_off, long q_off, int sym, int splits, int* err, void* stream)
{
    return cf_umma_trace_impl(P1, P2, K1, K2, nterms, ta, tb, X, sXp, ldX, x_ps, x_planes, Y, sYq, ldY, y_ps,
                              y_planes, scale, F, ldF, p_off, q_off, sym, nullptr, nullptr, splits, err, stream);
}

// As cf_umma_trace_bf16, with output row p going to F row row_map[p] and column
// q to F column col_map[q] (device int arrays), and the mirror entry too when sym.
extern "C" int cf_umma_trace_bf16_mapped(int P1, int P2, int K1, int K2, int nterms, const int* ta,
                                         const int* tb, const void* X, long sXp, long ldX, long x_ps, int x_planes,
                                         const void* Y, long sYq, long ldY, long y_ps, int y_planes, double scale,
                                         double* F, long ldF, const int* row_map, const int* col_map, int sym,
                                         int splits, int* err, void* stream)
{
    if (!row_map || !col_map) return CF_ERR_ARG;
    return cf_umma_trace_impl(P1, P2, K1, K2, nterms, ta, tb, X, sXp, ldX, x_ps, x_planes, Y, sYq, ldY, y_ps,
                              y_planes, scale, F, ldF, 0, 0, sym, row_map, col_map, splits, err, stream);
}

int cf_umma_trace_impl(int P1, int P2, int K1, int K2, int nterms, const int* ta, const int* tb, const void* X,
                       long sXp, long ldX, long x_ps, int x_planes, const void* Y, long sYq, long ldY, long y_ps,
                       int y_planes, double scale, double* F, long ldF, long p_off, long q_off, int sym,
                       const int* row_map, const int* col_map, int splits, int* err, void* stream)
{
    if (P1 <= 0 || P2 <= 0 || K1 <= 0 || K2 <= 0 || nterms < 1 || nterms > MAX_TERMS || !X || !Y || !F)
        return CF_ERR_ARG;
    Terms t{};
    t.n = nterms;
    for (int i = 0; i < nterms; ++i) {
        if (ta[i] < 0 || ta[i] >= x_planes || tb[i] < 0 || tb[i] >= y_planes) return CF_ERR_ARG;
        t.a[i] = ta[i];
        t.b[i] = tb[i];
    }
    CUtensorMap ma, mb;
    // every plane of a k-tile in one stage when both operands carry the same planes
    const int pls = (x_planes == y_planes) ? x_planes : 1;
    const bool narrow = P2 <= 64;
    const bool pairs = g_trace_pairs && !narrow && P1 > BM && (pls == 2 || pls == 3);
    int rc = make_map4(&ma, X, K2, K1, P1, x_planes, ldX, sXp, x_ps, BM);
    if (rc) return rc;
    rc = make_map4(&mb, Y, K2, K1, P2, y_planes, ldY, sYq, y_ps, narrow ? 64 : (pairs ? 64 : 128));
    if (rc) return rc;
    const long tiles = (long)K1 * ((K2 + BK - 1) / BK);
    const int out_tiles = cf_cdiv(P1, pairs ? 2 * BM : BM) * cf_cdiv(P2, narrow ? 64 : 128);
    if (splits <= 0) splits = (148 * 2 + out_tiles - 1) / out_tiles;
    if (splits > tiles) splits = (int)tiles;
    EpiArgs e{};
    e.M = P1;
    e.N = P2;
    TraceArgs tr{K1, K2, F, ldF, p_off, q_off, sym, scale, row_map, col_map};
    cudaStream_t st = (cudaStream_t)stream;
    if (pairs) {
        if (pls == 3) return launch_gemm_kc<128, 3, true, 4, 3, BK, false, 2>(ma, mb, P1, P2, 0, t, e, tr, splits, err, st);
        return launch_gemm_kc<128, 4, true, 4, 2, BK, false, 2>(ma, mb, P1, P2, 0, t, e, tr, splits, err, st);
    }
    if (narrow) {
        if (pls == 3) return launch_gemm_kc<64, 3, true, 4, 3>(ma, mb, P1, P2, 0, t, e, tr, splits, err, st);
        if (pls == 2) return launch_gemm_kc<64, 4, true, 4, 2>(ma, mb, P1, P2, 0, t, e, tr, splits, err, st);
        return launch_gemm<64, 8, true>(ma, mb, P1, P2, 0, t, e, tr, splits, err, st);
    }
    if (pls == 3) return launch_gemm_kc<128, 2, true, 4, 3>(ma, mb, P1, P2, 0, t, e, tr, splits, err, st);
    if (pls == 2) return launch_gemm_kc<128, 3, true, 4, 2>(ma, mb, P1, P2, 0, t, e, tr, splits, err, st);
    return launch_gemm<128, 6, true>(ma, mb, P1, P2, 0, t, e, tr, splits, err, st);
}
