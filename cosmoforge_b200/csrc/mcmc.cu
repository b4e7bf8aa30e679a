// Delayed-acceptance Metropolis over parameter points (one thread per chain).
//
// Stage 1 screens a Gaussian proposal theta' = theta + L xi with the emulator
// lnL~: accept with probability min(1, exp(lnL~(theta') - lnL~(theta))).  A
// proposal that passes becomes "pending" and is judged in stage 2 with the
// exact likelihood: accept with probability
//   min(1, exp([lnL(theta') - lnL(theta)] - [lnL~(theta') - lnL~(theta)])),
// which keeps the exact posterior as the chain's stationary distribution
// (Christen & Fox, J. Comput. Graph. Stat. 14 (2005) 795).  Proposals outside
// the prior box are rejected at once.  Every completed step appends the
// chain's current point to its record samples[c][step][:].
//
// No counterpart in the reference (which has no sampler).
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

// Plain Metropolis with the exact likelihood: every active proposal is judged
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
