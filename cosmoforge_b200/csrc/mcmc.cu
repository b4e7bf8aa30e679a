// Delayed-acceptance Metropolis over parameter points (one thread per chain).
//
// Stage 1 screens a Gaussian proposal theta' = theta + L xi with the emulator
// lnL~: accept with probability min(1, exp(lnL~(theta') - lnL~(theta))).  A
// proposal that passes becomes "pending" and is decided in stage 2 by the
// exact likelihood: accept with probability
//   min(1, exp([lnL(theta') - lnL(theta)] - [lnL~(theta') - lnL~(theta)])),
// which keeps the exact posterior as the chain's stationary distribution
// (Christen & Fox, J. Comput. Graph. Stat. 14 (2005) 795).  Proposals outside
// the prior box are rejected at once.  Every completed step appends the
// chain's current point to its record samples[c][step][:].
//
// No counterpart in the reference (which has no sampler).
#include <cuda_bf16.h>

#include "cf_common.cuh"

namespace {

__device__ __forceinline__ void record(int c, int D, const double* theta, int* steps, double* samples, int max_steps)
{
    const int s = steps[c];
    if (s < max_steps)
        for (int i = 0; i < D; ++i) samples[((long)c * max_steps + s) * D + i] = theta[c * D + i];
    steps[c] = s + 1;
}

// active[c]: 0 idle (pending or finished), 1 proposal inside the box, 2 outside.
__global__ void k_propose(int C, int D, const double* theta, const int* pending, const int* steps, int max_steps,
                          const double* Lp, const double* xi, const double* lo, const double* hi, double* theta_p,
                          float* xin, int* active)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    int act = (!pending[c] && steps[c] < max_steps) ? 1 : 0;
    if (act) {
        for (int i = 0; i < D; ++i) {
            double v = theta[c * D + i];
            for (int j = 0; j <= i; ++j) v += Lp[i * D + j] * xi[c * D + j];
            theta_p[c * D + i] = v;
            if (v < lo[i] || v > hi[i]) act = 2;
            xin[c * D + i] = (float)(2.0 * (v - lo[i]) / (hi[i] - lo[i]) - 1.0);
        }
    }
    active[c] = act;
}

__global__ void k_stage1(int C, int D, const int* active, const float* y, double mu, double sigma, const double* u,
                         const double* theta, double* ltil, double* ltil_p, int* pending, int* steps,
                         double* samples, int max_steps, int* n_stage1)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C || active[c] == 0) return;
    if (active[c] == 1) {
        const double lp = -0.5 * (mu + sigma * (double)y[c]);
        ltil_p[c] = lp;
        if (log(u[c]) < lp - ltil[c]) {
            pending[c] = 1;
            n_stage1[c] += 1;
            return;
        }
    }
    record(c, D, theta, steps, samples, max_steps);
}

__global__ void k_stage2(int C, int D, const double* lexact_p, double* lexact, double* ltil, const double* ltil_p,
                         const double* u, double* theta, const double* theta_p, int* pending, int* steps,
                         double* samples, int max_steps, int* n_exact, int* n_accept)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C || !pending[c]) return;
    n_exact[c] += 1;
    const double lr = (lexact_p[c] - lexact[c]) - (ltil_p[c] - ltil[c]);
    if (log(u[c]) < lr) {
        for (int i = 0; i < D; ++i) theta[c * D + i] = theta_p[c * D + i];
        lexact[c] = lexact_p[c];
        ltil[c] = ltil_p[c];
        n_accept[c] += 1;
    }
    record(c, D, theta, steps, samples, max_steps);
    pending[c] = 0;
}

// Plain Metropolis with the exact likelihood: every active proposal is decided
// by exp(lnL(theta') - lnL(theta)).
__global__ void k_mh_accept(int C, int D, const int* active, const double* lexact_p, double* lexact, const double* u,
                            double* theta, const double* theta_p, int* steps, double* samples, int max_steps,
                            int* n_exact, int* n_accept)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C || active[c] == 0) return;
    if (active[c] == 1) {
        n_exact[c] += 1;
        if (log(u[c]) < lexact_p[c] - lexact[c]) {
            for (int i = 0; i < D; ++i) theta[c * D + i] = theta_p[c * D + i];
            lexact[c] = lexact_p[c];
            n_accept[c] += 1;
        }
    }
    record(c, D, theta, steps, samples, max_steps);
}

// Emulator sub-chain (two-level delayed acceptance): one Metropolis step on
// the emulator posterior for every chain whose proposal lies in the box.
__global__ void k_sub_accept(int C, int D, const int* active, const float* y, double mu, double sigma,
                             const double* u, const double* theta_p, double* theta_s, double* ltil_s,
                             int* n_sub_accept)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C || active[c] != 1) return;
    const double lp = -0.5 * (mu + sigma * (double)y[c]);
    if (log(u[c]) < lp - ltil_s[c]) {
        for (int i = 0; i < D; ++i) theta_s[c * D + i] = theta_p[c * D + i];
        ltil_s[c] = lp;
        n_sub_accept[c] += 1;
    }
}

// The sub-chain's end point theta_s is the exact chain's proposal: accept
// with min(1, exp([lnL(theta_s) - lnL(theta)] - [lnL~(theta_s) - lnL~(theta)])).
// Either way the next sub-chain starts from the exact chain's point.
__global__ void k_sub_final(int C, int D, const double* lexact_p, double* lexact, double* ltil, double* ltil_s,
                            const double* u, double* theta, double* theta_s, int* steps, double* samples,
                            int max_steps, int* n_exact, int* n_accept)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    if (steps[c] < max_steps) {
        n_exact[c] += 1;
        const double lr = (lexact_p[c] - lexact[c]) - (ltil_s[c] - ltil[c]);
        if (log(u[c]) < lr) {
            for (int i = 0; i < D; ++i) theta[c * D + i] = theta_s[c * D + i];
            lexact[c] = lexact_p[c];
            ltil[c] = ltil_s[c];
            n_accept[c] += 1;
        }
        record(c, D, theta, steps, samples, max_steps);
    }
    for (int i = 0; i < D; ++i) theta_s[c * D + i] = theta[c * D + i];
    ltil_s[c] = ltil[c];
}

// ---- fused emulator sub-chain: one CTA per chain, J steps in one launch ----
//
// The emulator is the MLP (D -> 256 -> ... -> 256 -> 1, SiLU, BF16 weight
// matrices, FP32 biases and accumulation) of the training kernels, read from
// its flat parameter vector (per layer: W row-major out x in, then b).  Each
// of the 8 warps of a CTA produces 32 outputs of a 256 x 256 layer: a lane
// reads 8 consecutive weights of a row (16 B, the warp reads a whole row at
// once) against its 8 inputs, and a 31-shuffle reduce-scatter leaves row
// 32 w + l's sum in lane l.  Weights stream from L2 (256 KB for two hidden
// layers); a step costs a few microseconds, so a sub-chain of tens of steps
// is small beside one batched exact evaluation.
constexpr int SC_H = 256;

__device__ __forceinline__ float sc_silu(float z) { return z * (1.0f / (1.0f + expf(-z))); }

__device__ __forceinline__ void bf16x8(const uint4& q, float* w)
{
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 f = __bfloat1622float2(h[i]);
        w[2 * i] = f.x;
        w[2 * i + 1] = f.y;
    }
}

// Standardised emulator output at the normalised input x (shared, D values);
// valid in thread 0.  All threads of the CTA call it.
__device__ float sc_mlp(const float* x, int D, int n_hidden, const __nv_bfloat16* __restrict__ w16,
                        const float* __restrict__ w32, float* h0, float* h1, float* red)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    long off = 0;
    {
        float z = w32[off + (long)SC_H * D + t];
        for (int k = 0; k < D; ++k) z = fmaf(__bfloat162float(w16[off + (long)t * D + k]), x[k], z);
        h0[t] = sc_silu(z);
        off += (long)SC_H * D + SC_H;
    }
    __syncthreads();
    float* hin = h0;
    float* hout = h1;
    for (int l = 1; l < n_hidden; ++l) {
        float hv[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) hv[i] = hin[lane * 8 + i];
        float v[32];
        const __nv_bfloat16* W = w16 + off + (long)(warp * 32) * SC_H + lane * 8;
#pragma unroll
        for (int r = 0; r < 32; ++r) {
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(W + (long)r * SC_H));
            float w[8];
            bf16x8(q, w);
            float a = 0.0f;
#pragma unroll
            for (int i = 0; i < 8; ++i) a = fmaf(w[i], hv[i], a);
            v[r] = a;
        }
        // reduce-scatter: after the stage of width s, v[i] holds row (lane's
        // higher bits) * 2s + i summed over the lanes that differ in bits >= s
#pragma unroll
        for (int s = 16; s >= 1; s >>= 1) {
            const bool hi_half = (lane & s) != 0;
#pragma unroll
            for (int i = 0; i < s; ++i) {
                const float send = hi_half ? v[i] : v[i + s];
                const float keep = hi_half ? v[i + s] : v[i];
                v[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
            }
        }
        const int row = warp * 32 + lane;
        hout[row] = sc_silu(v[0] + w32[off + (long)SC_H * SC_H + row]);
        off += (long)SC_H * SC_H + SC_H;
        __syncthreads();
        float* tmp = hin;
        hin = hout;
        hout = tmp;
    }
    float p = __bfloat162float(w16[off + t]) * hin[t];
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) p += __shfl_xor_sync(0xffffffffu, p, s);
    if (lane == 0) red[warp] = p;
    __syncthreads();
    float y = 0.0f;
    if (t == 0) {
        y = w32[off + SC_H];
        for (int w = 0; w < SC_H / 32; ++w) y += red[w];
    }
    return y;
}

// Chain c = blockIdx.x: lnL~ at theta (into ltil), then J Metropolis steps on
// the emulator posterior from theta with proposals Lp xi[j][c] and uniforms
// u[j][c]; the end point into theta_s / ltil_s, accepted moves into n_sub.
// Finished chains (steps >= max_steps) only copy theta to theta_s.
__global__ void __launch_bounds__(SC_H) k_subchain(int C, int D, int J, int n_hidden, const double* theta,
                                                   const int* steps, int max_steps, const double* Lp,
                                                   const double* xi, const double* u, const double* lo,
                                                   const double* hi, const __nv_bfloat16* w16, const float* w32,
                                                   double mu, double sigma, double* theta_s, double* ltil,
                                                   double* ltil_s, int* n_sub)
{
    __shared__ double th[16], tp[16];
    __shared__ float x[16], h0[SC_H], h1[SC_H], red[SC_H / 32];
    __shared__ int inside;
    const int c = blockIdx.x, t = threadIdx.x;
    if (steps[c] >= max_steps) {
        if (t < D) theta_s[c * D + t] = theta[c * D + t];
        return;
    }
    if (t < D) {
        th[t] = theta[c * D + t];
        x[t] = (float)(2.0 * (th[t] - lo[t]) / (hi[t] - lo[t]) - 1.0);
    }
    __syncthreads();
    float y = sc_mlp(x, D, n_hidden, w16, w32, h0, h1, red);
    double lt = -0.5 * (mu + sigma * (double)y);
    int nacc = 0;
    if (t == 0) ltil[c] = lt;
    for (int j = 0; j < J; ++j) {
        if (t == 0) {
            const double* xj = xi + ((long)j * C + c) * D;
            int in = 1;
            for (int i = 0; i < D; ++i) {
                double v = th[i];
                for (int k = 0; k <= i; ++k) v += Lp[i * D + k] * xj[k];
                tp[i] = v;
                if (v < lo[i] || v > hi[i]) in = 0;
                x[i] = (float)(2.0 * (v - lo[i]) / (hi[i] - lo[i]) - 1.0);
            }
            inside = in;
        }
        __syncthreads();
        if (inside) {
            y = sc_mlp(x, D, n_hidden, w16, w32, h0, h1, red);
            if (t == 0) {
                const double lp = -0.5 * (mu + sigma * (double)y);
                if (log(u[(long)j * C + c]) < lp - lt) {
                    for (int i = 0; i < D; ++i) th[i] = tp[i];
                    lt = lp;
                    ++nacc;
                }
            }
        }
        __syncthreads();
    }
    if (t < D) theta_s[c * D + t] = th[t];
    if (t == 0) {
        ltil_s[c] = lt;
        n_sub[c] += nacc;
    }
}

inline unsigned blocks(int C) { return (unsigned)((C + 127) / 128); }

}  // namespace

// Stage-0 proposal for every chain that is neither pending nor finished:
// theta_p = theta + Lp xi (Lp: D x D lower, row-major; xi: C x D standard
// normals), xin = theta_p mapped from the box [lo, hi] to [-1, 1] (FP32, the
// emulator's input), active[c] = 0 idle / 1 inside / 2 outside the box.
extern "C" int cf_mcmc_propose(int C, int D, const double* theta, const int* pending, const int* steps, int max_steps,
                               const double* Lp, const double* xi, const double* lo, const double* hi,
                               double* theta_p, float* xin, int* active, void* stream)
{
    if (C <= 0 || D <= 0 || D > 16) return CF_ERR_ARG;
    k_propose<<<blocks(C), 128, 0, (cudaStream_t)stream>>>(C, D, theta, pending, steps, max_steps, Lp, xi, lo, hi,
                                                            theta_p, xin, active);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// Stage 1: emulator output y (standardised -2 lnL: lnL~ = -(mu + sigma y) / 2)
// against the current lnL~; u: C uniforms.  Passing chains become pending,
// the others complete a (rejected) step.
extern "C" int cf_mcmc_stage1(int C, int D, const int* active, const float* y, double mu, double sigma,
                              const double* u, const double* theta, double* ltil, double* ltil_p, int* pending,
                              int* steps, double* samples, int max_steps, int* n_stage1, void* stream)
{
    if (C <= 0 || D <= 0) return CF_ERR_ARG;
    k_stage1<<<blocks(C), 128, 0, (cudaStream_t)stream>>>(C, D, active, y, mu, sigma, u, theta, ltil, ltil_p,
                                                           pending, steps, samples, max_steps, n_stage1);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// Stage 2: exact lnL of the pending proposals (lexact_p) decides; every
// pending chain completes a step.
extern "C" int cf_mcmc_stage2(int C, int D, const double* lexact_p, double* lexact, double* ltil,
                              const double* ltil_p, const double* u, double* theta, const double* theta_p,
                              int* pending, int* steps, double* samples, int max_steps, int* n_exact,
                              int* n_accept, void* stream)
{
    if (C <= 0 || D <= 0) return CF_ERR_ARG;
    k_stage2<<<blocks(C), 128, 0, (cudaStream_t)stream>>>(C, D, lexact_p, lexact, ltil, ltil_p, u, theta, theta_p,
                                                           pending, steps, samples, max_steps, n_exact, n_accept);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// Plain exact-likelihood Metropolis acceptance for the active chains.
extern "C" int cf_mcmc_mh_accept(int C, int D, const int* active, const double* lexact_p, double* lexact,
                                 const double* u, double* theta, const double* theta_p, int* steps, double* samples,
                                 int max_steps, int* n_exact, int* n_accept, void* stream)
{
    if (C <= 0 || D <= 0) return CF_ERR_ARG;
    k_mh_accept<<<blocks(C), 128, 0, (cudaStream_t)stream>>>(C, D, active, lexact_p, lexact, u, theta, theta_p,
                                                              steps, samples, max_steps, n_exact, n_accept);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// One emulator sub-chain step: chains with active == 1 move theta_s to
// theta_p with probability min(1, exp(lnL~(theta_p) - ltil_s)).
extern "C" int cf_mcmc_sub_accept(int C, int D, const int* active, const float* y, double mu, double sigma,
                                  const double* u, const double* theta_p, double* theta_s, double* ltil_s,
                                  int* n_sub_accept, void* stream)
{
    if (C <= 0 || D <= 0) return CF_ERR_ARG;
    k_sub_accept<<<blocks(C), 128, 0, (cudaStream_t)stream>>>(C, D, active, y, mu, sigma, u, theta_p, theta_s,
                                                               ltil_s, n_sub_accept);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// Exact-likelihood decision on the sub-chains' end points (lexact_p) for
// every unfinished chain; resets theta_s / ltil_s to the chain's point.
extern "C" int cf_mcmc_sub_final(int C, int D, const double* lexact_p, double* lexact, double* ltil,
                                 double* ltil_s, const double* u, double* theta, double* theta_s, int* steps,
                                 double* samples, int max_steps, int* n_exact, int* n_accept, void* stream)
{
    if (C <= 0 || D <= 0) return CF_ERR_ARG;
    k_sub_final<<<blocks(C), 128, 0, (cudaStream_t)stream>>>(C, D, lexact_p, lexact, ltil, ltil_s, u, theta,
                                                              theta_s, steps, samples, max_steps, n_exact,
                                                              n_accept);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// Fused emulator sub-chains (one CTA per chain, J Metropolis steps on the
// emulator posterior, the emulator's value at theta recomputed first so every
// lnL~ of a round comes from the same code).  w16 / w32: the emulator's flat
// parameter vector as BF16 (weight matrices read) and FP32 (biases read);
// sizes D -> 256 x n_hidden -> 1.  xi: J x C x D normals, u: J x C uniforms.
extern "C" int cf_mcmc_subchain(int C, int D, int J, int n_hidden, const double* theta, const int* steps,
                                int max_steps, const double* Lp, const double* xi, const double* u, const double* lo,
                                const double* hi, const void* w16, const float* w32, double mu, double sigma,
                                double* theta_s, double* ltil, double* ltil_s, int* n_sub, void* stream)
{
    if (C <= 0 || D <= 0 || D > 16 || J < 0 || n_hidden < 1 || n_hidden > 8) return CF_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(w16) & 15) != 0) return CF_ERR_ARG;
    k_subchain<<<C, SC_H, 0, (cudaStream_t)stream>>>(C, D, J, n_hidden, theta, steps, max_steps, Lp, xi, u, lo, hi,
                                                     (const __nv_bfloat16*)w16, w32, mu, sigma, theta_s, ltil,
                                                     ltil_s, n_sub);
    CF_CHECK_LAUNCH();
    return CF_OK;
}
