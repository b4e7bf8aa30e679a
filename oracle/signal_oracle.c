/*
 * CPU oracle (test infrastructure, not product code): restatement of the
 * reference's pixel-space signal / derivative kernels in plain C.
 *
 * Only the tests, the smoke check and the CPU-baseline leg of the benchmark
 * may load this library; the device path never does.
 *
 * Follows, operation by operation (compiled with -ffp-contract=off so no
 * multiply-add is fused, as in the reference's Numba code):
 *   legendre_00 / legendre_22 / legendre_02   cosmocore/basics/legendre.py:9-149
 *   _project_and_norm / get_rotation_angle     cosmocore/basics/geometry.py:15-110
 *   compute_00/22/02_contribution + _compute_* cosmocore/signal_kernels.py:164-387
 *   _copy_lower_to_upper                       cosmocore/basics/linalg.py:101-120
 * A binned derivative dC_b is the same block formula with the spectrum's
 * C_l replaced by the bin weights w_l b_l^2 (cosmocore/basis/pixel.py:802-950).
 *
 * Matrices are row-major with leading dimension ld; block writers fill the
 * lower triangle (row >= col) of the full matrix, as the reference does, and
 * orc_mirror_lower copies it to the upper triangle.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846

static void leg00(double x, int lmax, double *p)
{
    p[0] = 1.0;
    if (lmax >= 1) p[1] = x;
    if (lmax >= 2) p[2] = 1.5 * x * x - 0.5;
    for (int l = 3; l <= lmax; ++l)
        p[l] = ((double)(2 * l - 1) * x * p[l - 1] - (double)(l - 1) * p[l - 2]) / (double)l;
    for (int l = 0; l <= lmax; ++l)
        p[l] *= (double)(2 * l + 1) / (4.0 * ORC_PI);
}

static void leg22(double x, int lmax, double *p, double *f1, double *f2)
{
    for (int l = 0; l <= lmax; ++l) { p[l] = 0.0; f1[l] = 0.0; f2[l] = 0.0; }
    if (lmax >= 2) {
        p[2] = 3.0;
        f1[2] = 6.0 * (1.0 + x * x);
        f2[2] = -12.0 * x;
    }
    for (int l = 3; l <= lmax; ++l) {
        p[l] = (x * (double)(2 * l - 1) * p[l - 1] - (double)(l + 1) * p[l - 2]) / (double)(l - 2);
        f1[l] = -((double)(2 * l - 8) + (double)(l * (l - 1)) * (1.0 - x * x)) * p[l]
                + (double)(2 * l + 4) * x * p[l - 1];
        f2[l] = 4.0 * ((double)(-(l - 1)) * x * p[l] + (double)(l + 2) * p[l - 1]);
    }
    for (int l = 2; l <= lmax; ++l) {
        double factor2 = 1.0 / (double)((l + 2) * (l + 1) * l * (l - 1));
        double norm = (double)(2 * l + 1) / (4.0 * ORC_PI) * factor2;
        p[l] *= norm;
        f1[l] *= norm;
        f2[l] *= norm;
    }
}

static void leg02(double x, int lmax, double *p)
{
    for (int l = 0; l <= lmax; ++l) p[l] = 0.0;
    if (lmax >= 2) p[2] = 3.0 * (1.0 - x * x);
    for (int l = 3; l <= lmax; ++l)
        p[l] = (x * (double)(2 * l - 1) * p[l - 1] - (double)(l + 1) * p[l - 2]) / (double)(l - 2);
    for (int l = 2; l <= lmax; ++l) {
        double factor = sqrt(1.0 / (double)((l + 2) * (l + 1) * l * (l - 1)));
        p[l] *= (double)(2 * l + 1) / (4.0 * ORC_PI) * factor;
    }
}

static void project_and_norm(double vx, double vy, double *ox, double *oy)
{
    const double eps = ORC_PI / 180.0 / 3600.0 / 100.0;
    double px = 0.0 * 0.0 - 1.0 * vy; /* z-axis cross v: (0*vz - 1*vy, 1*vx - 0*vz) */
    double py = 1.0 * vx - 0.0 * 0.0;
    double nm = sqrt(px * px + py * py);
    if (nm < 1e-8) {
        px += eps;
        nm = sqrt(px * px + py * py);
    }
    *ox = px / nm;
    *oy = py / nm;
}

static void rotation_angle(const double *r1, const double *r2, double *a12, double *a21)
{
    double x = r1[1] * r2[2] - r1[2] * r2[1];
    double y = r1[2] * r2[0] - r1[0] * r2[2];
    double z = r1[0] * r2[1] - r1[1] * r2[0];
    double mod = sqrt(x * x + y * y + z * z);
    if (mod < 1e-8) { *a12 = 0.0; *a21 = 0.0; return; }
    x /= mod; y /= mod; z /= mod;
    double r1x, r1y, r2x, r2y;
    project_and_norm(r1[0], r1[1], &r1x, &r1y);
    project_and_norm(r2[0], r2[1], &r2x, &r2y);
    double d1 = x * r1x + y * r1y;
    if (d1 > 1.0) d1 = 1.0; else if (d1 < -1.0) d1 = -1.0;
    double s1 = z > 0.0 ? 1.0 : -1.0;
    *a12 = 2.0 * acos(d1) * s1;
    x = -x; y = -y; z = -z;
    double d2 = x * r2x + y * r2y;
    if (d2 > 1.0) d2 = 1.0; else if (d2 < -1.0) d2 = -1.0;
    double s2 = z > 0.0 ? 1.0 : -1.0;
    *a21 = 2.0 * acos(d2) * s2;
}

static inline double dot3(const double *a, const double *b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* Spin-0 auto block of one field at offset `off`: S[off+j, off+i], j >= i. */
void orc_block_00_auto(int n, const double *v, int lmax, const double *cl,
                       double *S, long ld, long off)
{
    double *p0 = malloc(sizeof(double) * (lmax + 1));
    leg00(1.0, lmax, p0);
    double diag = 0.0;
    for (int l = 0; l <= lmax; ++l) diag += cl[l] * p0[l];
    for (int i = 0; i < n; ++i) S[(off + i) * ld + off + i] = diag;
    free(p0);
#pragma omp parallel
    {
        double *p = malloc(sizeof(double) * (lmax + 1));
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < n; ++i) {
            for (int j = i + 1; j < n; ++j) {
                leg00(dot3(v + 3 * j, v + 3 * i), lmax, p);
                double val = 0.0;
                for (int l = 0; l <= lmax; ++l) val += cl[l] * p[l];
                S[(off + j) * ld + off + i] = val;
            }
        }
        free(p);
    }
}

/* Spin-0 cross block between field a (cols, offset off_a) and field b
 * (rows, offset off_b > off_a): S[off_b+j, off_a+i] for all i, j. */
void orc_block_00_cross(int na, const double *va, int nb, const double *vb, int lmax,
                        const double *cl, double *S, long ld, long off_a, long off_b)
{
#pragma omp parallel
    {
        double *p = malloc(sizeof(double) * (lmax + 1));
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < na; ++i) {
            for (int j = 0; j < nb; ++j) {
                leg00(dot3(vb + 3 * j, va + 3 * i), lmax, p);
                double val = 0.0;
                for (int l = 0; l <= lmax; ++l) val += cl[l] * p[l];
                S[(off_b + j) * ld + off_a + i] = val;
            }
        }
        free(p);
    }
}

/* Spin-2 auto block of one field (rows/cols [Q | U] at offset off). */
void orc_block_22_auto(int n, const double *v, int lmax, const double *c11,
                       const double *c22, const double *c12, double *S, long ld, long off)
{
    {
        double *p = malloc(sizeof(double) * (lmax + 1) * 3);
        double *f1 = p + (lmax + 1), *f2 = f1 + (lmax + 1);
        leg22(1.0, lmax, p, f1, f2);
        double qq = 0.0, uu = 0.0, qu = 0.0;
        for (int l = 2; l <= lmax; ++l) {
            qq += c11[l] * f1[l] - c22[l] * f2[l];
            uu += c22[l] * f1[l] - c11[l] * f2[l];
            qu += (f1[l] + f2[l]) * c12[l];
        }
        for (int i = 0; i < n; ++i) {
            S[(off + i) * ld + off + i] = qq;
            S[(off + i + n) * ld + off + i] = qu;
            S[(off + i + n) * ld + off + i + n] = uu;
        }
        free(p);
    }
#pragma omp parallel
    {
        double *p = malloc(sizeof(double) * (lmax + 1) * 3);
        double *f1 = p + (lmax + 1), *f2 = f1 + (lmax + 1);
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < n; ++i) {
            for (int j = i + 1; j < n; ++j) {
                leg22(dot3(v + 3 * j, v + 3 * i), lmax, p, f1, f2);
                double qq = 0.0, uu = 0.0, qu = 0.0;
                for (int l = 2; l <= lmax; ++l) {
                    qq += c11[l] * f1[l] - c22[l] * f2[l];
                    uu += c22[l] * f1[l] - c11[l] * f2[l];
                    qu += (f1[l] + f2[l]) * c12[l];
                }
                double a1, a2;
                rotation_angle(v + 3 * j, v + 3 * i, &a1, &a2);
                double cos1 = cos(a1), cos2 = cos(a2);
                double sin1 = -sin(a1), sin2 = -sin(a2);
                double c1c2 = cos1 * cos2, s1s2 = sin1 * sin2;
                double c1s2 = cos1 * sin2, s1c2 = sin1 * cos2;
                S[(off + j) * ld + off + i] = qq * c1c2 + uu * s1s2 + qu * (c1s2 + s1c2);
                S[(off + j + n) * ld + off + i + n] = qq * s1s2 + uu * c1c2 - qu * (c1s2 + s1c2);
                S[(off + j + n) * ld + off + i] = -qq * s1c2 + uu * c1s2 + qu * (c1c2 - s1s2);
                S[(off + i + n) * ld + off + j] = -qq * c1s2 + uu * s1c2 + qu * (c1c2 - s1s2);
            }
        }
        free(p);
    }
}

/* Spin-0 x spin-2 block: rows = P field [Q | U] at off_p, cols = T field at off_t. */
void orc_block_02(int nt, const double *vt, int np, const double *vp, int lmax,
                  const double *c12, const double *c13, double *S, long ld, long off_t, long off_p)
{
#pragma omp parallel
    {
        double *p = malloc(sizeof(double) * (lmax + 1));
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < nt; ++i) {
            for (int j = 0; j < np; ++j) {
                leg02(dot3(vp + 3 * j, vt + 3 * i), lmax, p);
                double tq = 0.0, tu = 0.0;
                for (int l = 2; l <= lmax; ++l) {
                    tq -= c12[l] * p[l];
                    tu -= c13[l] * p[l];
                }
                double a1, a2;
                rotation_angle(vp + 3 * j, vt + 3 * i, &a1, &a2);
                double cos1 = cos(a1), sin1 = sin(a1);
                S[(off_p + j) * ld + off_t + i] = tq * cos1 - tu * sin1;
                S[(off_p + j + np) * ld + off_t + i] = tq * sin1 + tu * cos1;
            }
        }
        free(p);
    }
}

/* Copy the lower triangle onto the upper triangle of an n x n block at (off, off). */
void orc_mirror_lower(long n, double *S, long ld)
{
#pragma omp parallel for schedule(dynamic, 16)
    for (long i = 0; i < n; ++i)
        for (long j = 0; j < i; ++j) S[j * ld + i] = S[i * ld + j];
}

/* Rotation angles of one pair, exposed for unit tests. */
void orc_rotation_angle(const double *r1, const double *r2, double *out2)
{
    rotation_angle(r1, r2, &out2[0], &out2[1]);
}

void orc_legendre(int kind, double x, int lmax, double *out)
{
    if (kind == 0) leg00(x, lmax, out);
    else if (kind == 2) leg02(x, lmax, out);
    else leg22(x, lmax, out, out + lmax + 1, out + 2 * (lmax + 1));
}
