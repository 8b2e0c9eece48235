/*
 * bmc_oracle.c -- CPU oracle of the BMC-JAX forward model in C, float64, OpenMP over chains.
 * TEST INFRASTRUCTURE and the timed CPU baseline: never linked into the product.
 *
 * A restatement of the reference's float64 path, written from its source:
 *   system matrix A, C        simulation/matrix.py:83-295 (same entry layout, same lineshapes 25-81)
 *   time step                 simulation/expm.py:86-112: expm([A C; 0 0] dt) [M; 1], with the
 *                             matrix exponential of the library path (jax.scipy.linalg.expm, x64):
 *                             the [13/13] Pade approximant with scaling and squaring, theta_13 =
 *                             5.371920351148152 (Higham, SIAM J. Matrix Anal. Appl. 26, 2005),
 *                             Pade coefficients from their closed form, LU with partial pivoting
 *   event scan                simulation/simulate.py:22-132 (dt > 1e-9, spoilers, ADC reset, last_M)
 * The params layout is the C ABI's (include/bmc_b200.h): [13 + 5 n_cest][n_voxels].
 * Build: oracle/build.py (gcc -O3 -fopenmp -shared).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXN 24

static double pade13_b[14];

static void pade_coefficients(void) {
    /* b_j = (2m - j)! m! / ((2m)! j! (m - j)!), m = 13 */
    const int m = 13;
    for (int j = 0; j <= m; ++j)
        pade13_b[j] = exp(lgamma(2.0 * m - j + 1) + lgamma(m + 1.0) - lgamma(2.0 * m + 1) - lgamma(j + 1.0) -
                          lgamma(m - j + 1.0));
    /* scale to integers as usually tabulated (a common factor does not change the approximant) */
    const double s = 1.0 / pade13_b[13];
    for (int j = 0; j <= m; ++j) pade13_b[j] = nearbyint(pade13_b[j] * s);
}

static void matmul(int n, const double* A, const double* B, double* C) {
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += A[i * n + k] * B[k * n + j];
            C[i * n + j] = s;
        }
}

/* solve Q X = P in place (P overwritten by X), LU with partial pivoting */
static void lu_solve(int n, double* Q, double* P) {
    for (int c = 0; c < n; ++c) {
        int piv = c;
        double best = fabs(Q[c * n + c]);
        for (int r = c + 1; r < n; ++r)
            if (fabs(Q[r * n + c]) > best) { best = fabs(Q[r * n + c]); piv = r; }
        if (piv != c) {
            for (int k = 0; k < n; ++k) {
                double t = Q[c * n + k]; Q[c * n + k] = Q[piv * n + k]; Q[piv * n + k] = t;
                t = P[c * n + k]; P[c * n + k] = P[piv * n + k]; P[piv * n + k] = t;
            }
        }
        for (int r = c + 1; r < n; ++r) {
            const double f = Q[r * n + c] / Q[c * n + c];
            if (f == 0.0) continue;
            for (int k = c; k < n; ++k) Q[r * n + k] -= f * Q[c * n + k];
            for (int k = 0; k < n; ++k) P[r * n + k] -= f * P[c * n + k];
        }
    }
    for (int c = n - 1; c >= 0; --c) {
        for (int k = 0; k < n; ++k) {
            double s = P[c * n + k];
            for (int j = c + 1; j < n; ++j) s -= Q[c * n + j] * P[j * n + k];
            P[c * n + k] = s / Q[c * n + c];
        }
    }
}

/* E = expm(X), n x n */
static void expm13(int n, const double* X, double* E) {
    double A[MAXN * MAXN], A2[MAXN * MAXN], A4[MAXN * MAXN], A6[MAXN * MAXN], U[MAXN * MAXN],
        V[MAXN * MAXN], T[MAXN * MAXN], W[MAXN * MAXN];
    double norm = 0.0;
    for (int j = 0; j < n; ++j) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += fabs(X[i * n + j]);
        if (s > norm) norm = s;
    }
    int sq = 0;
    if (norm > 5.371920351148152) sq = (int)ceil(log2(norm / 5.371920351148152));
    const double sc = ldexp(1.0, -sq);
    const int nn = n * n;
    for (int i = 0; i < nn; ++i) A[i] = X[i] * sc;
    matmul(n, A, A, A2);
    matmul(n, A2, A2, A4);
    matmul(n, A4, A2, A6);
    const double* b = pade13_b;
    for (int i = 0; i < nn; ++i) T[i] = b[13] * A6[i] + b[11] * A4[i] + b[9] * A2[i];
    matmul(n, A6, T, W);
    for (int i = 0; i < nn; ++i) W[i] += b[7] * A6[i] + b[5] * A4[i] + b[3] * A2[i];
    for (int i = 0; i < n; ++i) W[i * n + i] += b[1];
    matmul(n, A, W, U);
    for (int i = 0; i < nn; ++i) T[i] = b[12] * A6[i] + b[10] * A4[i] + b[8] * A2[i];
    matmul(n, A6, T, V);
    for (int i = 0; i < nn; ++i) V[i] += b[6] * A6[i] + b[4] * A4[i] + b[2] * A2[i];
    for (int i = 0; i < n; ++i) V[i * n + i] += b[0];
    for (int i = 0; i < nn; ++i) {
        const double u = U[i], v = V[i];
        T[i] = v - u;              /* Q */
        E[i] = v + u;              /* P */
    }
    lu_solve(n, T, E);
    for (int s = 0; s < sq; ++s) {
        matmul(n, E, E, W);
        memcpy(E, W, sizeof(double) * nn);
    }
}

static double sl_direct(double delta, double t2) {
    double acc = 0.0;
    for (int i = 0; i <= 100; ++i) {
        const double u = 0.01 * i;
        double q = fabs(3.0 * u * u - 1.0);
        if (q < 1e-6) q = 1e-6;
        const double arg = delta * t2 / q;
        acc += sqrt(2.0 / M_PI) * t2 / q * exp(-2.0 * arg * arg);
    }
    return acc * M_PI * 0.01;
}

static double super_lorentzian(double delta, double t2, double w0) {
    if (fabs(delta) >= w0) return sl_direct(delta, t2);
    const double p0 = -300.0 - w0, p1 = -100.0 - w0, p2 = 100.0 + w0, p3 = 300.0 + w0;
    const double y0 = sl_direct(p0, t2), y1 = sl_direct(p1, t2), y2 = sl_direct(p2, t2), y3 = sl_direct(p3, t2);
    const double d0 = 30.0 * (y1 - y0), d1 = 30.0 * (y3 - y2);
    const double c = fabs((delta - p1 + 1.0) / (p2 - p1 + 1.0));
    const double c2 = c * c, c3 = c2 * c;
    return (2 * c3 - 3 * c2 + 1) * y1 + (-2 * c3 + 3 * c2) * y2 + (c3 - 2 * c2 + c) * d0 + (c3 - c2) * d1;
}

/* augmented generator X = [A C; 0 0] dt for one voxel (params column v of an nv-wide table) */
static void generator(int nc, const double* P, int nv, int v, double amp, double phase, double freq, double dt,
                      double* X) {
#define F(r) P[(size_t)(r) * nv + v]
    const int n = 1 + nc, N = 3 * n + 1, NA = N + 1;
    const int MK = 3 + 5 * nc;
    const double r1w = F(0), r2w = F(1);
    const double kmt = F(MK), fmt = F(MK + 1), dwmt = F(MK + 2), r1mt = F(MK + 3), r2mt = F(MK + 4);
    const int ls = (int)F(MK + 5);
    const double b0 = F(MK + 6), gam = F(MK + 7), b0i = F(MK + 8), rb1 = F(MK + 9);
    const double w1 = 2.0 * M_PI * amp * rb1, w1x = w1 * cos(phase), w1y = w1 * sin(phase);
    const double larmor = gam * 1e6 * b0, dw0 = larmor * b0i * 1e-6;
    const double eff = 2.0 * M_PI * freq - dw0;
    const double offmt = eff - dwmt * 1e-6 * larmor;
    double g = 0.0;
    if (fmt > 1e-9) {
        const int l = ls < 0 ? 0 : (ls > 2 ? 2 : ls);
        const double t2 = 1.0 / r2mt;
        if (l == 1) g = t2 / (1.0 + (offmt * t2) * (offmt * t2));
        else if (l == 2) g = super_lorentzian(offmt, t2, larmor * 1e-6);
    }
    const double wmt = fmt > 1e-9 ? w1 * w1 * g : 0.0;
    memset(X, 0, sizeof(double) * NA * NA);
#define A(i, j) X[(i) * NA + (j)]
    const int xw = 0, yw = n, zw = 2 * n, zm = 3 * n;
    double ksum = 0.0;
    for (int i = 0; i < nc; ++i) ksum += F(3 + i) * F(3 + nc + i);
    const double kwmt = kmt * fmt;
    A(xw, xw) = -r2w - ksum; A(xw, yw) = eff; A(xw, zw) = -w1y;
    A(yw, yw) = -r2w - ksum; A(yw, xw) = -eff; A(yw, zw) = w1x;
    A(zw, zw) = -r1w - ksum - kwmt; A(zw, yw) = -w1x; A(zw, xw) = w1y;
    for (int i = 0; i < nc; ++i) {
        const double k = F(3 + i), f = F(3 + nc + i), dw = F(3 + 2 * nc + i), r1 = F(3 + 3 * nc + i),
                     r2 = F(3 + 4 * nc + i);
        const double kwc = k * f, offc = dw * 1e-6 * larmor - eff;
        const int xc = 1 + i, yc = n + 1 + i, zc = 2 * n + 1 + i;
        A(xc, xc) = -r2 - k; A(xc, yc) = -offc; A(xc, zc) = -w1y;
        A(yc, yc) = -r2 - k; A(yc, xc) = offc; A(yc, zc) = w1x;
        A(zc, zc) = -r1 - k; A(zc, xc) = w1y; A(zc, yc) = -w1x;
        A(xw, xc) = k; A(yw, yc) = k; A(zw, zc) = k;
        A(xc, xw) = kwc; A(yc, yw) = kwc; A(zc, zw) = kwc;
        A(zc, N) = r1 * f;
    }
    A(zm, zm) = -r1mt - kmt - wmt; A(zm, zw) = kwmt; A(zw, zm) = kmt;
    A(zw, N) = r1w; A(zm, N) = r1mt * fmt;
    for (int i = 0; i < NA * NA; ++i) X[i] *= dt;
#undef A
#undef F
}

/* one chain: last_M of voxel v at offset o */
static void chain(int nc, const double* P, int nv, int v, int n_ev, const int* type, const double* dt,
                  const double* amp, const double* phase, const double* freq, const double* m0, double* last) {
    const int n = 1 + nc, N = 3 * n + 1, NA = N + 1;
    double M[MAXN], X[MAXN * MAXN], E[MAXN * MAXN];
    memcpy(M, m0, sizeof(double) * N);
    int pending = 0;
    for (int e = 0; e < n_ev; ++e) {
        if (pending) { memcpy(M, m0, sizeof(double) * N); pending = 0; }
        if (dt[e] > 1e-9) {
            generator(nc, P, nv, v, amp[e], phase[e], freq[e], dt[e], X);
            expm13(NA, X, E);
            double Mn[MAXN];
            for (int i = 0; i < N; ++i) {
                double s = E[i * NA + N];
                for (int j = 0; j < N; ++j) s += E[i * NA + j] * M[j];
                Mn[i] = s;
            }
            memcpy(M, Mn, sizeof(double) * N);
        }
        if (type[e] == 2 || type[e] == 4)
            for (int i = 0; i < 2 * n; ++i) M[i] = 0.0;
        if (type[e] == 3 && e + 1 < n_ev) pending = 1;
    }
    memcpy(last, M, sizeof(double) * N);
}

/* Z[v][o] = last_M[mz] for every chain; threads <= 0: all cores. Returns 0. */
int oracle_simulate(int n_vox, int n_off, int n_ev, int nc, const double* params, const int* type,
                    const double* dt, const double* amp, const double* phase, const double* freq,
                    const double* m0, int mz, double* out, int threads) {
    pade_coefficients();
    const int N = 3 * (1 + nc) + 1;
    const long total = (long)n_vox * n_off;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (long c = 0; c < total; ++c) {
        const int v = (int)(c / n_off), o = (int)(c % n_off);
        const size_t r = (size_t)o * n_ev;
        double last[MAXN];
        chain(nc, params, n_vox, v, n_ev, type + r, dt + r, amp + r, phase + r, freq + r, m0 + (size_t)v * N, last);
        out[c] = last[mz];
    }
    return 0;
}

int oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
