// bmc_joint.cuh -- the normal equations and the damped step of a joint fit whose samples have their own
// points (uneven batches), on the device.
//
// BMC-JAX's joint LM (fitting/joint.py:149-162) solves (H + lam (diag H + 1e-9 I)) d = -g with
// H = J^T J, g = J^T r over every free value of every sample, densely. With per-sample values and at
// most one value shared by every sample, H is an arrowhead: one P_loc x P_loc block per sample plus a
// shared column. The same linear system is solved here by eliminating each sample's block (one thread
// per sample, Gaussian elimination with partial pivoting in float64), summing the shared column's
// Schur complement in a fixed order (one block, deterministic), and back-substituting.
#pragma once
#include <cuda_runtime.h>

namespace bmc {

constexpr int kMaxJointP = 9;  // local values + the shared one

// per sample v: H[v] = sum over its chains c of J[:, c] J[:, c]^T, g[v] = J r, cost[v] = r^T r;
// chains of sample v are seg[v] .. seg[v+1]-1 of the canonical order; J is [P][n_chains]
__global__ void normal_segments_kernel(int n_vox, int P, long long n_chains, const long long* __restrict__ seg,
                                       const double* __restrict__ J, const double* __restrict__ r,
                                       double* __restrict__ H, double* __restrict__ g, double* __restrict__ cost) {
    const int warp = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= n_vox) return;
    double h[kMaxJointP * (kMaxJointP + 1) / 2], gv[kMaxJointP], c = 0.0;
#pragma unroll
    for (int i = 0; i < kMaxJointP * (kMaxJointP + 1) / 2; ++i) h[i] = 0.0;
#pragma unroll
    for (int i = 0; i < kMaxJointP; ++i) gv[i] = 0.0;
    for (long long ch = seg[warp] + lane; ch < seg[warp + 1]; ch += 32) {
        double j[kMaxJointP];
#pragma unroll
        for (int p = 0; p < kMaxJointP; ++p) j[p] = p < P ? J[(size_t)p * n_chains + ch] : 0.0;
        const double rc = r[ch];
        c = fma(rc, rc, c);
        int k = 0;
#pragma unroll
        for (int p = 0; p < kMaxJointP; ++p) {
            gv[p] = fma(j[p], rc, gv[p]);
#pragma unroll
            for (int q = 0; q <= p; ++q) {
                h[k] = fma(j[p], j[q], h[k]);
                ++k;
            }
        }
    }
    // warp sums, then lane 0 writes the symmetric block
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
#pragma unroll
    for (int p = 0; p < kMaxJointP; ++p)
        for (int o = 16; o > 0; o >>= 1) gv[p] += __shfl_xor_sync(0xffffffffu, gv[p], o);
#pragma unroll
    for (int i = 0; i < kMaxJointP * (kMaxJointP + 1) / 2; ++i)
        for (int o = 16; o > 0; o >>= 1) h[i] += __shfl_xor_sync(0xffffffffu, h[i], o);
    if (lane == 0) {
        double* Hv = H + (size_t)warp * P * P;
        int k = 0;
#pragma unroll
        for (int p = 0; p < kMaxJointP; ++p) {
#pragma unroll
            for (int q = 0; q <= p; ++q, ++k) {
                if (p < P && q < P) {
                    Hv[p * P + q] = h[k];
                    Hv[q * P + p] = h[k];
                }
            }
            if (p < P) g[(size_t)warp * P + p] = gv[p];
        }
        cost[warp] = c;
    }
}

// Solve A x = b (n <= kMaxJointP - 1, two right-hand sides) by Gaussian elimination with partial pivoting.
// Every index is static after unrolling (rows are swapped by compare-and-swap), so A stays in registers.
__host__ __device__ inline void solve2(double (&A)[kMaxJointP - 1][kMaxJointP - 1], double (&b1)[kMaxJointP - 1],
                                       double (&b2)[kMaxJointP - 1], int n) {
    constexpr int M = kMaxJointP - 1;
#pragma unroll
    for (int k = 0; k < M; ++k) {
        if (k < n) {
            int piv = k;
            double best = fabs(A[k][k]);
#pragma unroll
            for (int i = 0; i < M; ++i)
                if (i > k && i < n && fabs(A[i][k]) > best) {
                    best = fabs(A[i][k]);
                    piv = i;
                }
#pragma unroll
            for (int i = 0; i < M; ++i) {
                if (i > k && i == piv) {
#pragma unroll
                    for (int j = 0; j < M; ++j) {
                        const double t = A[k][j];
                        A[k][j] = A[i][j];
                        A[i][j] = t;
                    }
                    double t = b1[k]; b1[k] = b1[i]; b1[i] = t;
                    t = b2[k]; b2[k] = b2[i]; b2[i] = t;
                }
            }
            const double inv = 1.0 / A[k][k];
#pragma unroll
            for (int i = 0; i < M; ++i) {
                if (i > k && i < n) {
                    const double f = A[i][k] * inv;
#pragma unroll
                    for (int j = 0; j < M; ++j)
                        if (j >= k) A[i][j] = fma(-f, A[k][j], A[i][j]);
                    b1[i] = fma(-f, b1[k], b1[i]);
                    b2[i] = fma(-f, b2[k], b2[i]);
                }
            }
        }
    }
#pragma unroll
    for (int kk = 0; kk < M; ++kk) {
        const int k = M - 1 - kk;
        if (k < n) {
            double s1 = b1[k], s2 = b2[k];
#pragma unroll
            for (int j = 0; j < M; ++j)
                if (j > k && j < n) {
                    s1 = fma(-A[k][j], b1[j], s1);
                    s2 = fma(-A[k][j], b2[j], s2);
                }
            b1[k] = s1 / A[k][k];
            b2[k] = s2 / A[k][k];
        }
    }
}

// Per sample: eliminate the local block. H[v] is P x P with P = PL + S (the shared value last when S = 1);
// free[v][j] (1 free, 0 held) for the local values. Writes w = A^-1 g_p and Y = A^-1 h_ps (Y zero when
// S = 0) and the sample's terms of the shared Schur complement: red = (h_ss, h_ps^T Y, h_ps^T w, g_s).
__host__ __device__ inline void schur_eliminate_one(int v, int n_vox, int PL, int S, const double* H, const double* g,
                                                   const double* free, double lam_in, const double* d_lam,
                                                   double* Y, double* w, double* red) {
    const double lam = d_lam ? *d_lam : lam_in;
    constexpr int M = kMaxJointP - 1;
    const int P = PL + S;
    const double* Hv = H + (size_t)v * P * P;
    const double* gv = g + (size_t)v * P;
    double A[M][M], by[M], bw[M], fr[M];
#pragma unroll
    for (int j = 0; j < M; ++j) fr[j] = j < PL ? (free ? free[(size_t)v * PL + j] : 1.0) : 0.0;
#pragma unroll
    for (int j = 0; j < M; ++j) {
        by[j] = (j < PL && S) ? fr[j] * Hv[j * P + PL] : 0.0;
        bw[j] = j < PL ? fr[j] * gv[j] : 0.0;
#pragma unroll
        for (int k = 0; k < M; ++k) A[j][k] = (j < PL && k < PL) ? fr[j] * fr[k] * Hv[j * P + k] : 0.0;
        if (j < PL) A[j][j] += fr[j] * lam * (Hv[j * P + j] + 1e-9) + (1.0 - fr[j]);
    }
    solve2(A, by, bw, PL);
    double sy = 0.0, tw = 0.0;
#pragma unroll
    for (int j = 0; j < M; ++j) {
        if (j < PL) {
            Y[(size_t)v * PL + j] = by[j];
            w[(size_t)v * PL + j] = bw[j];
            if (S) {
                const double hps = fr[j] * Hv[j * P + PL];
                sy = fma(hps, by[j], sy);
                tw = fma(hps, bw[j], tw);
            }
        }
    }
    red[v] = S ? Hv[PL * P + PL] : 0.0;
    red[(size_t)n_vox + v] = sy;
    red[2 * (size_t)n_vox + v] = tw;
    red[3 * (size_t)n_vox + v] = S ? gv[PL] : 0.0;
}

__global__ void schur_eliminate_kernel(int n_vox, int PL, int S, const double* __restrict__ H,
                                       const double* __restrict__ g, const double* __restrict__ free, double lam,
                                       const double* __restrict__ d_lam,
                                       double* __restrict__ Y, double* __restrict__ w, double* __restrict__ red) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n_vox) schur_eliminate_one(v, n_vox, PL, S, H, g, free, lam, d_lam, Y, w, red);
}

// one block: the four Schur sums of a batch -- sum h_ss, sum h_ps^T Y, sum h_ps^T w, sum g_s -- in a
// fixed order (deterministic); a sharded fit adds the batches' sums across ranks before the shared step
__global__ void schur_sum_kernel(int n_vox, const double* __restrict__ red, double* __restrict__ sums) {
    __shared__ double sm[4][1024];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int v = threadIdx.x; v < n_vox; v += blockDim.x)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] += red[(size_t)q * n_vox + v];
#pragma unroll
    for (int q = 0; q < 4; ++q) sm[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
#pragma unroll
            for (int q = 0; q < 4; ++q) sm[q][threadIdx.x] += sm[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 4) sums[threadIdx.x] = sm[threadIdx.x][0];
}

// the shared step ds = -(sum g_s - sum h_ps^T w) / (H_ss + lam (H_ss + 1e-9) - sum h_ps^T Y), H_ss = sum h_ss
__global__ void schur_shared_kernel(int S, const double* __restrict__ sums, double lam_in,
                                    const double* __restrict__ d_lam, double* __restrict__ ds) {
    const double lam = d_lam ? *d_lam : lam_in;
    if (threadIdx.x == 0) {
        const double hss = sums[0], sy = sums[1], tw = sums[2], gs = sums[3];
        ds[0] = S ? -(gs - tw) / (hss + lam * (hss + 1e-9) - sy) : 0.0;
    }
}

// d_p = -(w + Y ds) per sample
__global__ void schur_back_kernel(int n_vox, int PL, const double* __restrict__ Y, const double* __restrict__ w,
                                  const double* __restrict__ ds, double* __restrict__ d) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)n_vox * PL) return;
    d[i] = -(w[i] + Y[i] * ds[0]);
}

}  // namespace bmc
