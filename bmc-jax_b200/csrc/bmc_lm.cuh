// bmc_lm.cuh -- device side of the bounded Levenberg-Marquardt fit (float64 throughout).
//
// One LM iteration of BMC-JAX fitting/lm.py:43-61 for every voxel:
//   r = Z(x) - z_meas, c = r.r, J = dZ/dx (times `free`), g = J^T r, H = J^T J,
//   A = H + lam (diag(H) + 1e-9 I) (+ diag(1 - free)), delta = solve(A, -g), x' = clip(x + delta),
//   c' = |Z(x') - z_meas|^2, accept if c' < c: lam *= 0.5, else lam *= 3.
// The parameter write-back follows fitting/params.py:100-112 (plain values) and, for the modes of
// fit_joint, fitting/joint.py:120-138 (value / factor / add, m_start rebuilt from the pools).
#pragma once
#include "bmc_kernels.cuh"

namespace bmc {

struct SlotSpec {
    int P;
    int field_row[kMaxT];   // >= 0 params row, -2 spread width, -3 m_start
    int mode[kMaxT];        // 0 value, 1 factor, 2 add
    double scale[kMaxT];
    double lo[kMaxT], hi[kMaxT];
};

// x (scaled) -> the params, start state, spread width and tangent seeds the chain kernel reads
template <int NC>
__global__ void lm_params_kernel(int n_vox, const SlotSpec sp, const double* __restrict__ base,
                                 const double* __restrict__ m0, const double* __restrict__ sigma0,
                                 const double* __restrict__ x, const double* __restrict__ freem,
                                 double* __restrict__ px, double* __restrict__ m0x, double* __restrict__ sigx,
                                 double* __restrict__ seed, double* __restrict__ dm0) {
    using L = Layout<NC>;
    constexpr int N = L::N;
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_vox) return;
    for (int r = 0; r < L::NF; ++r) px[(size_t)r * n_vox + v] = base[(size_t)r * n_vox + v];
    if (sigx) sigx[v] = sigma0 ? sigma0[v] : 0.0;
    int mslot = -1;
    double sd[kMaxT];
    for (int p = 0; p < sp.P; ++p) {
        const int fr = sp.field_row[p];
        const bool fre = freem == nullptr || freem[(size_t)v * sp.P + p] != 0.0;
        const double xp = x[(size_t)v * sp.P + p] * sp.scale[p];
        sd[p] = 0.0;
        if (fr >= 0) {
            const double old = px[(size_t)fr * n_vox + v];
            if (fre) {
                px[(size_t)fr * n_vox + v] = sp.mode[p] == 0 ? xp : (sp.mode[p] == 1 ? old * xp : old + xp);
                sd[p] = sp.mode[p] == 1 ? old * sp.scale[p] : sp.scale[p];
            }
        } else if (fr == -2) {
            if (fre) {
                if (sigx) sigx[v] = xp;
                sd[p] = sp.scale[p];
            }
        } else if (fr == -3) {
            mslot = p;
        }
    }
    // start state: initial_state(params) * m (value), or m0 * m (factor)   (joint.py:134-138)
    const double* m0v = m0 + (size_t)v * N;
    double* mo = m0x + (size_t)v * N;
    bool mfree = false;
    double mval = 1.0;
    if (mslot >= 0) {
        mfree = freem == nullptr || freem[(size_t)v * sp.P + mslot] != 0.0;
        mval = x[(size_t)v * sp.P + mslot] * sp.scale[mslot];
    }
    double ist[N];
    for (int q = 0; q < N; ++q) ist[q] = 0.0;
    ist[L::izw] = px[(size_t)L::WF * n_vox + v];
    for (int i = 0; i < NC; ++i) ist[L::izc(i)] = px[(size_t)(L::CF + i) * n_vox + v];
    ist[L::izm] = px[(size_t)L::MF * n_vox + v];
    const bool rebuild = mfree && sp.mode[mslot] == 0;
    for (int q = 0; q < N; ++q) mo[q] = !mfree ? m0v[q] : (rebuild ? ist[q] * mval : m0v[q] * mval);
    if (seed) {
        for (int p = 0; p < sp.P; ++p) seed[(size_t)p * n_vox + v] = sd[p];
    }
    if (dm0) {
        for (int p = 0; p < sp.P; ++p) {
            double* d = dm0 + ((size_t)p * n_vox + v) * N;
            for (int q = 0; q < N; ++q) d[q] = 0.0;
            if (!mfree) continue;
            if (p == mslot) {
                for (int q = 0; q < N; ++q) d[q] = (rebuild ? ist[q] : m0v[q]) * sp.scale[p];
            } else if (rebuild && sp.field_row[p] >= 0) {
                const int fr = sp.field_row[p];
                int q = -1;
                if (fr == L::WF) q = L::izw;
                else if (fr == L::MF) q = L::izm;
                else if (fr >= L::CF && fr < L::CF + NC) q = L::izc(fr - L::CF);
                if (q >= 0) d[q] = mval * sd[p];
            }
        }
    }
}

// warp-per-voxel sums over the residual points: c, g = J^T r, H = J^T J (J columns times free)
__device__ __forceinline__ void normal_sums(int lane, int v, int n_vox, int n_off, int skip, int P,
                                            const double* __restrict__ z, const double* __restrict__ zm,
                                            const double* __restrict__ J, const double* fr,
                                            double& c, double* g, double* H) {
    const int npts = n_off - skip;
    c = 0.0;
    for (int p = 0; p < P; ++p) {
        g[p] = 0.0;
        for (int q = 0; q < P; ++q) H[p * kMaxT + q] = 0.0;
    }
    for (int i = lane; i < npts; i += 32) {
        const double r = z[(size_t)v * n_off + skip + i] - zm[(size_t)v * npts + i];
        c = fma(r, r, c);
        double jr[kMaxT];
        for (int p = 0; p < P; ++p) jr[p] = J ? J[((size_t)p * n_vox + v) * n_off + skip + i] * fr[p] : 0.0;
        for (int p = 0; p < P; ++p) {
            g[p] = fma(jr[p], r, g[p]);
            for (int q = 0; q <= p; ++q) H[p * kMaxT + q] = fma(jr[p], jr[q], H[p * kMaxT + q]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_xor_sync(kFull, c, o);
        for (int p = 0; p < P; ++p) {
            g[p] += __shfl_xor_sync(kFull, g[p], o);
            for (int q = 0; q <= p; ++q) H[p * kMaxT + q] += __shfl_xor_sync(kFull, H[p * kMaxT + q], o);
        }
    }
    for (int p = 0; p < P; ++p)
        for (int q = p + 1; q < P; ++q) H[p * kMaxT + q] = H[q * kMaxT + p];
}

// solve A d = b (P x P, partial pivoting); A and b are overwritten
__device__ __forceinline__ void gauss_solve(int P, double* A, double* b) {
    for (int c = 0; c < P; ++c) {
        int piv = c;
        double best = fabs(A[c * kMaxT + c]);
        for (int r = c + 1; r < P; ++r) {
            const double a = fabs(A[r * kMaxT + c]);
            if (a > best) { best = a; piv = r; }
        }
        if (piv != c) {
            for (int k = 0; k < P; ++k) {
                const double t = A[c * kMaxT + k]; A[c * kMaxT + k] = A[piv * kMaxT + k]; A[piv * kMaxT + k] = t;
            }
            const double t = b[c]; b[c] = b[piv]; b[piv] = t;
        }
        const double inv = 1.0 / A[c * kMaxT + c];
        for (int r = c + 1; r < P; ++r) {
            const double f = A[r * kMaxT + c] * inv;
            for (int k = c; k < P; ++k) A[r * kMaxT + k] -= f * A[c * kMaxT + k];
            b[r] -= f * b[c];
        }
    }
    for (int c = P - 1; c >= 0; --c) {
        double s = b[c];
        for (int k = c + 1; k < P; ++k) s -= A[c * kMaxT + k] * b[k];
        b[c] = s / A[c * kMaxT + c];
    }
}

// normal equations, the damped solve and the clipped trial point
__global__ void lm_solve_kernel(int n_vox, int n_off, int skip, const SlotSpec sp, const double* __restrict__ z,
                                const double* __restrict__ zm, const double* __restrict__ J,
                                const double* __restrict__ freem, const double* __restrict__ x,
                                const double* __restrict__ lam, double* __restrict__ cost, double* __restrict__ xt) {
    const int lane = threadIdx.x & 31;
    const int v = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (v >= n_vox) return;
    const int P = sp.P;
    double fr[kMaxT];
    for (int p = 0; p < P; ++p) fr[p] = freem ? freem[(size_t)v * P + p] : 1.0;
    double c, g[kMaxT], H[kMaxT * kMaxT];
    normal_sums(lane, v, n_vox, n_off, skip, P, z, zm, J, fr, c, g, H);
    if (lane != 0) return;
    cost[v] = c;
    const double l = lam[v];
    double A[kMaxT * kMaxT], b[kMaxT];
    for (int p = 0; p < P; ++p) {
        for (int q = 0; q < P; ++q) A[p * kMaxT + q] = H[p * kMaxT + q];
        A[p * kMaxT + p] += l * (H[p * kMaxT + p] + 1e-9);
        if (freem) A[p * kMaxT + p] += 1.0 - fr[p];
        b[p] = -g[p];
    }
    gauss_solve(P, A, b);
    for (int p = 0; p < P; ++p) {
        const double xn = x[(size_t)v * P + p] + b[p];
        xt[(size_t)v * P + p] = fmin(fmax(xn, sp.lo[p]), sp.hi[p]);
    }
}

// accept or reject every voxel's trial point
__global__ void lm_accept_kernel(int n_vox, int n_off, int skip, int P, int it, int n_iter,
                                 const double* __restrict__ zt, const double* __restrict__ zm,
                                 const double* __restrict__ cost, const double* __restrict__ xt,
                                 double* __restrict__ x, double* __restrict__ lam, int* __restrict__ need,
                                 double* __restrict__ cost_traj, double* __restrict__ x_traj) {
    const int lane = threadIdx.x & 31;
    const int v = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (v >= n_vox) return;
    const int npts = n_off - skip;
    double cn = 0.0;
    for (int i = lane; i < npts; i += 32) {
        const double r = zt[(size_t)v * n_off + skip + i] - zm[(size_t)v * npts + i];
        cn = fma(r, r, cn);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cn += __shfl_xor_sync(kFull, cn, o);
    if (lane != 0) return;
    const bool better = cn < cost[v];
    if (better) {
        for (int p = 0; p < P; ++p) x[(size_t)v * P + p] = xt[(size_t)v * P + p];
    }
    lam[v] = better ? lam[v] * 0.5 : lam[v] * 3.0;
    need[v] = better ? 1 : 0;
    if (cost_traj) cost_traj[(size_t)v * n_iter + it] = better ? cn : cost[v];
    if (x_traj) {
        for (int p = 0; p < P; ++p) x_traj[((size_t)v * n_iter + it) * P + p] = x[(size_t)v * P + p];
    }
}

// per-sample H, g, c for a coupled joint fit
__global__ void normal_blocks_kernel(int n_vox, int n_pts, int P, const double* __restrict__ r,
                                     const double* __restrict__ J, double* __restrict__ Hout,
                                     double* __restrict__ gout, double* __restrict__ cout) {
    const int lane = threadIdx.x & 31;
    const int v = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (v >= n_vox) return;
    double c = 0.0, g[kMaxT], H[kMaxT * kMaxT];
    for (int p = 0; p < P; ++p) {
        g[p] = 0.0;
        for (int q = 0; q < P; ++q) H[p * kMaxT + q] = 0.0;
    }
    for (int i = lane; i < n_pts; i += 32) {
        const double rr = r[(size_t)v * n_pts + i];
        c = fma(rr, rr, c);
        double jr[kMaxT];
        for (int p = 0; p < P; ++p) jr[p] = J[((size_t)p * n_vox + v) * n_pts + i];
        for (int p = 0; p < P; ++p) {
            g[p] = fma(jr[p], rr, g[p]);
            for (int q = 0; q <= p; ++q) H[p * kMaxT + q] = fma(jr[p], jr[q], H[p * kMaxT + q]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_xor_sync(kFull, c, o);
        for (int p = 0; p < P; ++p) {
            g[p] += __shfl_xor_sync(kFull, g[p], o);
            for (int q = 0; q <= p; ++q) H[p * kMaxT + q] += __shfl_xor_sync(kFull, H[p * kMaxT + q], o);
        }
    }
    if (lane != 0) return;
    cout[v] = c;
    for (int p = 0; p < P; ++p) {
        gout[(size_t)v * P + p] = g[p];
        for (int q = 0; q < P; ++q)
            Hout[((size_t)v * P + p) * P + q] = q <= p ? H[p * kMaxT + q] : H[q * kMaxT + p];
    }
}

}  // namespace bmc
