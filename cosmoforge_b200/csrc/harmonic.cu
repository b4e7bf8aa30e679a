// Harmonic-basis estimator: the real harmonic operator V and the
// contractions that give F, the noise bias and q from G = V C^-1 V^T,
// Z N Z^T (Z = V C^-1) and z = Z x.
//
// Reference: cosmocore/basis/harmonic_basis.py:20-180 (V), the sparse Fisher
// of the harmonic basis (qube/fisher.py:416-500, 575-583) and the harmonic
// quadratic forms.  The derivative of the covariance with respect to one
// multipole of one spectrum is, by the addition theorem,
//   dC/dC_l = t_l (V_(u,l)^T V_(v,l) [+ V_(v,l)^T V_(u,l) for u != v])
// where (u, v) are the spectrum's components (T of a spin-0 field, E or B of
// a spin-2 field) and V_(c,l) the 2l + 1 rows of component c at multipole l.
// So, with the binned weights t_(s,l) of parameter p = s nb + b,
//   F_pp' = 1/2 sum_{l in b, l' in b'} t t' sum_{(u,v),(a,b)} <G_(v,l)(a,l'), G_(u,l)(b,l')>,
//   b_p   = 1/2 sum_{l in b} t f sum_m (Z N Z^T)_(u,l,m)(v,l,m),
//   q_p   = 1/2 sum_{l in b} t f sum_m z_(u,l,m) z_(v,l,m)   (f = 2 for u != v).
// Rows of V: component-major, then multipole, then m = 0 and (cos m, sin m)
// pairs, so a component's multipole is 2l + 1 contiguous rows.
#include "cf_common.cuh"

namespace {

constexpr int HMAXL = 255;

// ---- V ---------------------------------------------------------------------
// One thread per (pixel, m).  Spin 0: fully normalised associated Legendre
// functions with the Condon-Shortley phase, sqrt(2) cos / sin (m phi) for
// m > 0.  Spin 2: Wigner small-d d^l_{m,+-2} (closed form at the first degree,
// three-term recurrence in l above it), D+ = d_{m,-2} + d_{m,2},
// D- = d_{m,-2} - d_{m,2}, E and B rows over the [Q | U] columns; the rows
// carry the overall sign that makes V^T V reproduce the pixel-space 02 / 22
// kernels of the signal builder.
__device__ double d_first(int j, int mp, int m, double ch, double sh)
{
    // explicit sum of d^j_{mp,m}; at j = max(|mp|, |m|) one term survives
    double out = 0.0;
    const double lnorm = 0.5 * (lgamma(j + mp + 1.0) + lgamma(j - mp + 1.0) + lgamma(j + m + 1.0) +
                                lgamma(j - m + 1.0));
    for (int k = 0; k <= 2 * j; ++k) {
        const int a = j + m - k, b = k, c = mp - m + k, d = j - mp - k;
        if (a < 0 || b < 0 || c < 0 || d < 0) continue;
        const double coef = exp(lnorm - lgamma(a + 1.0) - lgamma(b + 1.0) - lgamma(c + 1.0) - lgamma(d + 1.0));
        const double sgn = ((mp - m + k) & 1) ? -1.0 : 1.0;
        out += sgn * coef * pow(ch, (double)(2 * j + m - mp - 2 * k)) * pow(sh, (double)(mp - m + 2 * k));
    }
    return out;
}

__global__ void k_harm_V(int spin, int is_b, int npix, const double* vec, int lmin, int lmax, double* V, long ldV,
                         long row0, long col0, double sign)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (i >= npix || m > lmax) return;
    const double x = vec[i], y = vec[npix + i];
    double z = vec[2 * npix + i];
    z = z > 1.0 ? 1.0 : (z < -1.0 ? -1.0 : z);
    const double st = sqrt(fmax(0.0, 1.0 - z * z));
    const double phi = atan2(y, x);
    double sm, cm;
    sincos(m * phi, &sm, &cm);
    const double r2 = sqrt(2.0);
    const double inv4pi = 1.0 / (4.0 * CF_PI);
    auto row = [&](int ell, int local) { return row0 + (long)ell * ell - (long)lmin * lmin + local; };

    if (spin == 0) {
        // sectoral P_mm, then the l recurrence for this m (unnormalised by
        // sqrt((2l+1)/4pi) until written)
        double pmm = 1.0;
        for (int k = 1; k <= m; ++k) pmm *= -st * sqrt((2.0 * k - 1.0) / (2.0 * k));
        double p2 = 0.0, p1 = 0.0;
        for (int ell = m; ell <= lmax; ++ell) {
            double p;
            if (ell == m) {
                p = pmm;
            } else if (m == 0) {  // Legendre polynomials
                p = ell == 1 ? z : ((2.0 * ell - 1.0) * z * p1 - (ell - 1.0) * p2) / ell;
            } else if (ell == m + 1) {
                p = z * sqrt(2.0 * m + 1.0) * p1;
            } else {
                const double d = (double)ell * ell - (double)m * m;
                p = ((2.0 * ell - 1.0) / sqrt(d)) * z * p1 - sqrt(((ell - 1.0) * (ell - 1.0) - (double)m * m) / d) * p2;
            }
            p2 = p1;
            p1 = p;
            if (ell < lmin) continue;
            const double v = p * sqrt((2.0 * ell + 1.0) * inv4pi);
            if (m == 0) {
                V[row(ell, 0) * ldV + col0 + i] = v;
            } else {
                V[row(ell, 2 * m - 1) * ldV + col0 + i] = r2 * v * cm;
                V[row(ell, 2 * m) * ldV + col0 + i] = r2 * v * sm;
            }
        }
        return;
    }

    const double th = acos(z);
    const double ch = cos(0.5 * th), sh = sin(0.5 * th);
    const int j0 = m > 2 ? m : 2;
    if (j0 > lmax) return;
    double dp1 = d_first(j0, m, 2, ch, sh), dp2 = 0.0;   // d^l_{m,2}
    double dm1 = d_first(j0, m, -2, ch, sh), dm2 = 0.0;  // d^l_{m,-2}
    const long qc = col0 + i, uc = col0 + npix + i;
    for (int ell = j0; ell <= lmax; ++ell) {
        if (ell > j0) {
            const double j = ell;
            const double c = (j - 1.0) * sqrt((j * j - (double)m * m) * (j * j - 4.0));
            const double bq = fmax(((j - 1.0) * (j - 1.0) - (double)m * m) * ((j - 1.0) * (j - 1.0) - 4.0), 0.0);
            const double b = j * sqrt(bq);
            const double ap = (2.0 * j - 1.0) * (j * (j - 1.0) * z - 2.0 * m);
            const double am = (2.0 * j - 1.0) * (j * (j - 1.0) * z + 2.0 * m);
            const double np = (ap * dp1 - b * dp2) / c;
            const double nm = (am * dm1 - b * dm2) / c;
            dp2 = dp1;
            dp1 = np;
            dm2 = dm1;
            dm1 = nm;
        }
        if (ell < lmin) continue;
        const double sc = sign * sqrt((2.0 * ell + 1.0) * inv4pi) * 0.5;
        const double Dp = dm1 + dp1, Dm = dm1 - dp1;
        if (m == 0) {
            const long r = row(ell, 0);
            V[r * ldV + qc] = is_b ? 0.0 : sc * Dp;
            V[r * ldV + uc] = is_b ? sc * Dp : 0.0;
            continue;
        }
        const double s2 = sc * r2;
        const long rc = row(ell, 2 * m - 1), rs = row(ell, 2 * m);
        if (!is_b) {
            V[rc * ldV + qc] = s2 * Dp * cm;
            V[rc * ldV + uc] = s2 * Dm * sm;
            V[rs * ldV + qc] = s2 * Dp * sm;
            V[rs * ldV + uc] = -s2 * Dm * cm;
        } else {
            V[rc * ldV + qc] = -s2 * Dm * sm;
            V[rc * ldV + uc] = s2 * Dp * cm;
            V[rs * ldV + qc] = s2 * Dm * cm;
            V[rs * ldV + uc] = s2 * Dp * sm;
        }
    }
}

// ---- Lambda V: rows of V mixed across components with the spectra ---------
// LV[(u,l,m), j] = sum_v lam[u][v][l] V[(v,l,m), j]; rowinfo[r] = (u, l).
__global__ void k_harm_lambda(long r0, long nr, long ncol, int nc, const int* rowinfo, const long* off,
                              const double* lam, int Lp, const double* V, long ldV, double* LV, long ldL)
{
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long r = r0 + blockIdx.y;
    if (j >= ncol || blockIdx.y >= nr) return;
    const int u = rowinfo[2 * r], ell = rowinfo[2 * r + 1];
    const long local = r - off[u * Lp + ell];
    double acc = 0.0;
    for (int v = 0; v < nc; ++v) {
        const double c = lam[((long)u * nc + v) * Lp + ell];
        if (c != 0.0) acc = fma(c, V[(off[v * Lp + ell] + local) * ldV + j], acc);
    }
    LV[r * ldL + j] = acc;
}

// ---- Fisher from G ----------------------------------------------------------
// CTA (l1, l2): every entry (i, j) of the (2 l1 + 1) x (2 l2 + 1) index square
// is read from the NC^2 component sub-blocks of G once; all products of two of
// them are summed (K_{ab} = sum_ij g_a g_b, a <= b), and the spectrum pairs are
// assembled from K into F with the weights of both multipoles.
template <int NC>
__global__ void __launch_bounds__(256) k_harm_fisher(int lmin, int Lp, const double* G, long ldG, const long* off,
                                                     int nspec, const int* su, const int* sv, const double* tab,
                                                     const int* bin, int nb, double* F, long ldF)
{
    constexpr int NP = NC * NC;
    constexpr int NK = NP * (NP + 1) / 2;
    const int l1 = lmin + blockIdx.x, l2 = lmin + blockIdx.y;
    const int n1 = 2 * l1 + 1, n2 = 2 * l2 + 1;
    double acc[NK];
#pragma unroll
    for (int k = 0; k < NK; ++k) acc[k] = 0.0;
    long ro[NC], co[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        ro[c] = off[c * Lp + l1];
        co[c] = off[c * Lp + l2];
    }
    for (int e = threadIdx.x; e < n1 * n2; e += blockDim.x) {
        const int i = e / n2, j = e % n2;
        double g[NP];
#pragma unroll
        for (int p = 0; p < NC; ++p)
#pragma unroll
            for (int q = 0; q < NC; ++q) g[p * NC + q] = G[(ro[p] + i) * ldG + co[q] + j];
        int k = 0;
#pragma unroll
        for (int a = 0; a < NP; ++a)
#pragma unroll
            for (int b = a; b < NP; ++b) {
                acc[k] = fma(g[a], g[b], acc[k]);
                ++k;
            }
    }
    __shared__ double red[8][NK];
    __shared__ double K[NK];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        double v = acc[k];
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < NK; k += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][k];
        K[k] = s;
    }
    __syncthreads();
    auto kidx = [&](int a, int b) {
        if (a > b) {
            const int t = a;
            a = b;
            b = t;
        }
        return a * NP - a * (a - 1) / 2 + (b - a);
    };
    for (int t = threadIdx.x; t < nspec * nspec; t += blockDim.x) {
        const int s1 = t / nspec, s2 = t % nspec;
        const int b1 = bin[s1 * Lp + l1], b2 = bin[s2 * Lp + l2];
        if (b1 < 0 || b2 < 0) continue;
        const double w = tab[s1 * Lp + l1] * tab[s2 * Lp + l2];
        if (w == 0.0) continue;
        const int u1 = su[s1], v1 = sv[s1], u2 = su[s2], v2 = sv[s2];
        double sum = 0.0;
        // pairs (u, v) of spectrum 1 and (a, b) of spectrum 2: K[(v a), (u b)]
        const int nx = (u1 == v1) ? 1 : 2, ny = (u2 == v2) ? 1 : 2;
        for (int x = 0; x < nx; ++x) {
            const int u = x ? v1 : u1, v = x ? u1 : v1;
            for (int y = 0; y < ny; ++y) {
                const int a = y ? v2 : u2, b = y ? u2 : v2;
                sum += K[kidx(v * NC + a, u * NC + b)];
            }
        }
        atomicAdd(F + (long)(s1 * nb + b1) * ldF + s2 * nb + b2, 0.5 * w * sum);
    }
}

// ---- bias and q ---------------------------------------------------------------
// CTA (s, l): sum over the 2l + 1 rows m of A[(u,l,m), k] B[(v,l,m), k]
// (plus the swapped pair for cross spectra) over the columns k (summed into
// out[p]) or per column (out[k * ldo + p]); scaled by t_(s,l) / 2.
__global__ void __launch_bounds__(256) k_harm_pair(int lmin, int Lp, const double* A, long ldA, const double* B,
                                                   long ldB, long ncol, int per_col, const long* off, const int* su,
                                                   const int* sv, const double* tab, const int* bin, int nb,
                                                   double* out, long ldo)
{
    const int s = blockIdx.x, ell = lmin + blockIdx.y;
    const int b = bin[s * Lp + ell];
    const double t = tab[s * Lp + ell];
    if (b < 0 || t == 0.0) return;
    const int u = su[s], v = sv[s];
    const long ru = off[u * Lp + ell], rv = off[v * Lp + ell];
    const int nr = 2 * ell + 1;
    const int p = s * nb + b;
    if (per_col) {
        for (long k = threadIdx.x; k < ncol; k += blockDim.x) {
            double acc = 0.0;
            for (int m = 0; m < nr; ++m) {
                acc = fma(A[(ru + m) * ldA + k], B[(rv + m) * ldB + k], acc);
                if (u != v) acc = fma(A[(rv + m) * ldA + k], B[(ru + m) * ldB + k], acc);
            }
            atomicAdd(out + k * ldo + p, 0.5 * t * acc);
        }
        return;
    }
    double acc = 0.0;
    for (long e = threadIdx.x; e < (long)nr * ncol; e += blockDim.x) {
        const long m = e / ncol, k = e % ncol;
        acc = fma(A[(ru + m) * ldA + k], B[(rv + m) * ldB + k], acc);
        if (u != v) acc = fma(A[(rv + m) * ldA + k], B[(ru + m) * ldB + k], acc);
    }
    __shared__ double red[8];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += red[w];
        atomicAdd(out + p, 0.5 * t * sum);
    }
}

}  // namespace

// Rows [row0, row0 + (lmax+1)^2 - lmin^2) of V (row stride ldV) for one
// component over columns col0.. of its field: spin 0 (T) or the E (is_b 0) /
// B (is_b 1) part of a spin-2 field over its [Q | U] columns.  vec: SoA
// pointings x[npix] y[npix] z[npix].  Replaces harmonic_basis.py:20-180
// (row order: multipole-major, m = 0 then cos / sin pairs).
extern "C" int cf_harmonic_operator(int spin, int is_b, int npix, const double* vec, int lmin, int lmax, double* V,
                                    long ldV, long row0, long col0, void* stream)
{
    if ((spin != 0 && spin != 2) || npix <= 0 || !vec || !V || lmin < 0 || lmax < lmin || lmax > HMAXL)
        return CF_ERR_ARG;
    if (spin == 2 && lmin < 2) return CF_ERR_ARG;
    dim3 grid(cf_cdiv(npix, 128), lmax + 1);
    k_harm_V<<<grid, 128, 0, (cudaStream_t)stream>>>(spin, is_b, npix, vec, lmin, lmax, V, ldV, row0, col0,
                                                      spin == 2 ? -1.0 : 1.0);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// LV = Lambda V (see k_harm_lambda): nm rows, ncol columns; rowinfo int[2 nm]
// (component, multipole) per row; off long[nc Lp] row offset of (c, l); lam
// double[nc nc Lp] (symmetric in the components).
extern "C" int cf_harmonic_lambda(long nm, long ncol, int nc, int lmin, const int* rowinfo, const long* off,
                                  const double* lam, int Lp, const double* V, long ldV, double* LV, long ldL,
                                  void* stream)
{
    if (nm <= 0 || ncol <= 0 || nc <= 0 || lmin < 0 || !V || !LV || !rowinfo || !off || !lam) return CF_ERR_ARG;
    for (long r0 = 0; r0 < nm; r0 += 65535) {
        const long nr = nm - r0 < 65535 ? nm - r0 : 65535;
        dim3 grid(cf_cdiv(ncol, 256), (unsigned)nr);
        k_harm_lambda<<<grid, 256, 0, (cudaStream_t)stream>>>(r0, nr, ncol, nc, rowinfo, off, lam, Lp, V, ldV, LV,
                                                              ldL);
        CF_CHECK_LAUNCH();
    }
    return CF_OK;
}

// F (nspec nb x nspec nb, row stride ldF, accumulated) from G = V C^-1 V^T
// (nm x nm, row stride ldG); nc <= 3 components; off long[nc Lp]; su / sv
// int[nspec] the spectrum components; tab / bin [nspec Lp] the binned weights
// and bin of each multipole (-1 outside the bins).
extern "C" int cf_harmonic_fisher(int nc, int lmin, int lmax, int Lp, const double* G, long ldG, const long* off,
                                  int nspec, const int* su, const int* sv, const double* tab, const int* bin, int nb,
                                  double* F, long ldF, void* stream)
{
    if (nc < 1 || nc > 3 || lmin < 0 || lmax < lmin || lmax >= Lp || !G || !F || nspec <= 0) return CF_ERR_ARG;
    dim3 grid(lmax - lmin + 1, lmax - lmin + 1);
    cudaStream_t st = (cudaStream_t)stream;
    if (nc == 1)
        k_harm_fisher<1><<<grid, 256, 0, st>>>(lmin, Lp, G, ldG, off, nspec, su, sv, tab, bin, nb, F, ldF);
    else if (nc == 2)
        k_harm_fisher<2><<<grid, 256, 0, st>>>(lmin, Lp, G, ldG, off, nspec, su, sv, tab, bin, nb, F, ldF);
    else
        k_harm_fisher<3><<<grid, 256, 0, st>>>(lmin, Lp, G, ldG, off, nspec, su, sv, tab, bin, nb, F, ldF);
    CF_CHECK_LAUNCH();
    return CF_OK;
}

// out[p] (per_col 0) or out[k ldo + p] (per_col 1) += 1/2 t_(s,l) sum_m
// A_(u,l,m) . B_(v,l,m) (+ swapped for cross spectra) over the multipoles of
// each parameter's bin: with A = Z N, B = Z the raw noise bias, with
// A = B = z = Z X the raw quadratic forms of the maps' columns.
extern "C" int cf_harmonic_pair(int lmin, int lmax, int Lp, const double* A, long ldA, const double* B, long ldB,
                                long ncol, int per_col, const long* off, int nspec, const int* su, const int* sv,
                                const double* tab, const int* bin, int nb, double* out, long ldo, void* stream)
{
    if (lmin < 0 || lmax < lmin || lmax >= Lp || !A || !B || !out || ncol <= 0 || nspec <= 0) return CF_ERR_ARG;
    dim3 grid(nspec, lmax - lmin + 1);
    k_harm_pair<<<grid, 256, 0, (cudaStream_t)stream>>>(lmin, Lp, A, ldA, B, ldB, ncol, per_col, off, su, sv, tab,
                                                         bin, nb, out, ldo);
    CF_CHECK_LAUNCH();
    return CF_OK;
}
