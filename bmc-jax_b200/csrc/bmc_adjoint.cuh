// bmc_adjoint.cuh -- every tangent of a single-event chain in one pass (reverse mode through the dense path).
//
// A chain whose state evolves in one event only (a CW saturation block followed by its readout: the
// Z-spectra and B1 ladders the reference fits, sequences/saturation.py:16-62) ends at
//     z = lam^T exp(X) v,   X = [A C; 0 0] dt,  v = [M0; 1],  lam = e_mz,
// and its tangent in direction p is (Frechet derivative L of the exponential)
//     dz_p = lam^T L(X, dX_p) v + lam^T exp(X) dv_p = tr(dX_p H) + (exp(X)^T lam) . dv_p,
//     H = L(X, v lam^T) = int_0^1 exp((1 - s) X) v lam^T exp(s X) ds.
// H does not depend on p, so one Frechet derivative in the rank-one direction v lam^T serves every
// tangent, where forward mode (the chain kernel's dual numbers, jax.jacfwd in fitting/lm.py:39) carries
// one direction dX_p per tangent through the whole exponential.
//
// exp(X) and H come together from the dual scaling and squaring of X + eps E, E = v lam^T: the Horner
// recurrence of exp(X / 2^s) with the tangent direction E / 2^s, then s squarings of the pair
// [T, H] -> [T T, T H + H T] (exp(2Y + 2 eps F) = exp(Y + eps F)^2). A group of lanes takes one chain,
// lane j < N holding column j of T and of H. T's last row is e_N^T (the augmented row) and is not
// stored; H's is (E has a last row: v_N lam^T = lam^T). The augmented column of T, phi = T[0:N, N], is
// kept apart in shared memory, lane i updating row i (phi <- T phi + phi), and the augmented column
// of H is never formed: it enters column j < N only through T[N][j] = 0, and no tangent reads it. So
// a chain takes N lanes, not N + 1: with four CEST pools (N = 16) two chains share a warp.
//
// The tangent coefficient sets dX_p = [dA_p dC_p; 0 0] dt come from the chain kernel's own coefficient
// code with a one-direction dual number, lane p of the group computing set p; lane i then forms
// row i of dX_p times column i of H (the sparse operator applied to that column, entry i), and the
// group's sum is tr(dX_p H).
#pragma once
#include "bmc_kernels.cuh"

namespace bmc {

// lanes per chain: the state columns, rounded up to a divisor of the warp
template <int NC>
struct AdjGroup {
    static constexpr int N = Layout<NC>::N;
    static constexpr int GS = N <= 4 ? 4 : (N <= 8 ? 8 : (N <= 16 ? 16 : 32));
    static constexpr int G = 32 / GS;
    // N = 16 (four CEST pools): the squarings on the FP64 tensor cores (mma.sync m8n8k4, 2 x 2 tiles of
    // 8 x 8), the warp taking its two chains in turn. Column stride 20 (4 mod 16 doubles): the 32 lanes
    // of a fragment load, (row, col) = (g, t) or (t, g) with g < 8, t < 4, hit each 8-byte bank twice.
    // Otherwise the lanes' own FMAs, odd stride (H's columns have N + 1 rows).
    static constexpr bool kMma = N == 16;
    static constexpr int LD = kMma ? 20 : ((N + 1) | 1);
    static constexpr int PHI_LANE = N < GS ? N : 0;    // the lane that forms phi's Horner recurrence
};

// D += A B for one 8x8x4 tile (row-major A, column-major B; lane l holds A[l / 4][l % 4], B[l % 4][l / 4]
// and D[l / 4][2 (l % 4) + 0, 1])
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

template <int NC>
struct AdjSlotBody {
    static constexpr int N = Layout<NC>::N;
    static constexpr int LD = AdjGroup<NC>::LD;
    using K = StepCoef<NC, Dn<double, 0>>;
    K coef;                                   // the owner's coefficients times h = dt / 2^s
    double cw, cm, cc[NC > 0 ? NC : 1];       // ... and its constant column C h
    double T[N * LD];                         // column-major: column j at [j * LD], rows 0 .. N - 1
    double H[N * LD];                         // rows 0 .. N
    double phi[2][N];                         // T's augmented column, one buffer read while the other is written
    double v[N + 1];                          // [M0; 1]
    K dk[kMaxT];                              // per tangent: the coefficients' derivative times dt
    double dcw[kMaxT], dcm[kMaxT], dcc[kMaxT][NC > 0 ? NC : 1];   // ... and C's
    double res[kMaxT + 1];                    // the group's sums: tangents, then z
    EvRec<double> rec;
    double g0, gd[3], scale;                  // the owner's MT lineshape and its partial derivatives in
                                              // (offset, T2, bridge width); 2^-s
    int s, vox;
};

template <int NC>
struct AdjSlot : AdjSlotBody<NC> {
    static constexpr size_t kBody = sizeof(AdjSlotBody<NC>);
    static constexpr size_t kTarget = (128 / AdjGroup<NC>::G) % 128;
    static constexpr size_t kPad = (kTarget + 128 - kBody % 128) % 128;
    char pad[kPad == 0 ? 128 : kPad];
};

constexpr int kAdjWarps = 4;

template <int GS>
__device__ __forceinline__ double group_sum(double x) {
#pragma unroll
    for (int o = GS / 2; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
    return x;
}

// Rows whose chains the adjoint kernel can take: exactly one event with dt > 1e-9, an RF block or a delay,
// and besides it no spoiler or gradient (they would act on M0 or on the evolved state) and no readout
// after it that resets the state before the row ends. row_ev[o] = that event, or -1; *all_ok is cleared
// when a row is not such a row.
__global__ void adjoint_rows_kernel(const EvRec<double>* __restrict__ rec, int n_off, int n_ev, int reset_after_adc,
                                    int* __restrict__ row_ev, int* __restrict__ all_ok) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n_off) return;
    int e_star = -1, moving = 0;
    bool ok = true;
    for (int e = 0; e < n_ev; ++e) {
        const EvRec<double> r = rec[(size_t)e * n_off + o];
        const int type = (int)r.type;
        if (r.dt > 1e-9) {
            ++moving;
            e_star = e;
            ok = ok && (type == EV_RF || type == EV_DELAY);
        } else {
            ok = ok && type != EV_GRADIENT && type != EV_SPOILER;
            if (type == EV_ADC && moving > 0 && reset_after_adc && e + 1 < n_ev) ok = false;
        }
    }
    ok = ok && moving == 1;
    row_ev[o] = ok ? e_star : -1;
    if (!ok) atomicAnd(all_ok, 0);
}

template <int NC>
struct Adjoint {
    using D0 = Dn<double, 0>;
    using D1 = Dn<double, 1>;
    using C0 = Chain<NC, double, 0>;
    using C1 = Chain<NC, double, 1>;
    using S = State<NC, D0>;
    using K = StepCoef<NC, D0>;
    using SL = AdjSlot<NC>;
    static constexpr int N = Layout<NC>::N;
    static constexpr int GS = AdjGroup<NC>::GS;
    static constexpr int G = AdjGroup<NC>::G;
    static constexpr int LD = AdjGroup<NC>::LD;

    static __device__ __forceinline__ double get(const S& x, int q) {
        double r = 0.0;
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (i == q) r = C0::at(const_cast<S&>(x), i).v;
        return r;
    }

    // y = X_s x + C_s c (rows 0 .. N - 1), X_s the slot's scaled coefficients
    static __device__ __forceinline__ void op(const SL* sl, const S& x, double c, S& y) {
        C0::template matvec<false>(sl->coef, x, y);
        y.zw.v = fma(sl->cw, c, y.zw.v);
        y.zm.v = fma(sl->cm, c, y.zm.v);
#pragma unroll
        for (int i = 0; i < NC; ++i) y.zc[i].v = fma(sl->cc[i], c, y.zc[i].v);
    }

    // entry i of dX_p x + dC_p c: the tangent coefficient set p applied to a column
    static __device__ __forceinline__ double dop_row(const SL* sl, int p, const S& x, double c, int i) {
        S y;
        C0::template matvec<false>(sl->dk[p], x, y);
        y.zw.v = fma(sl->dcw[p], c, y.zw.v);
        y.zm.v = fma(sl->dcm[p], c, y.zm.v);
#pragma unroll
        for (int k = 0; k < NC; ++k) y.zc[k].v = fma(sl->dcc[p][k], c, y.zc[k].v);
        return get(y, i);
    }

    // Lane p of the group: the derivative of the owner's coefficients (and constant column) along tangent p,
    // times dt, into the slot.
    static __device__ void tangent_set(const ChainArgs& a, SL* sl, int node, int p) {
        ChainConst<NC, D1> cp;
        C1::load_const(a, sl->vox, node, cp, p);
        const EvRec<double>& rec = sl->rec;
        // the lineshape's derivative by the chain rule through its three arguments (their partials were
        // formed once per chain, by the chain's own thread)
        D1 g = dconst<double, 1>(sl->g0);
        if (cp.mt_on && cp.ls != 0 && rec.w1 != 0.0) {
            const D1 offmt = (rec.wf - cp.dw0) - cp.dwmt;
            g.d[0] = fma(sl->gd[0], offmt.d[0], fma(sl->gd[1], cp.t2mt.d[0], sl->gd[2] * cp.w0sl.d[0]));
        }
        StepCoef<NC, D1> sp;
        C1::event_coef(cp, rec, g, sp);
        const double dt = rec.dt;
        K& d = sl->dk[p];
        d.Rw2.v = dt * sp.Rw2.d[0];
        d.Rw1.v = dt * sp.Rw1.d[0];
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            d.k[i].v = dt * sp.k[i].d[0];
            d.kwc[i].v = dt * sp.kwc[i].d[0];
            d.Rc2[i].v = dt * sp.Rc2[i].d[0];
            d.Rc1[i].v = dt * sp.Rc1[i].d[0];
            d.offc[i].v = dt * sp.offc[i].d[0];
            sl->dcc[p][i] = dt * cp.cc[i].d[0];
        }
        d.offw.v = dt * sp.offw.d[0];
        d.w1x.v = dt * sp.w1x.d[0];
        d.w1y.v = dt * sp.w1y.d[0];
        d.kmt.v = dt * sp.kmt.d[0];
        d.kwmt.v = dt * sp.kwmt.d[0];
        d.Rm1W.v = dt * sp.Rm1W.d[0];
        sl->dcw[p] = dt * cp.cw.d[0];
        sl->dcm[p] = dt * cp.cm.d[0];
    }

    static __device__ __forceinline__ void unit(S& x, int j) {
#pragma unroll
        for (int q = 0; q < N; ++q) C0::at(x, q).v = q == j ? 1.0 : 0.0;
    }

    // One squaring of a slot's pair, in place, by the whole warp (N = 16):
    //   T <- T T,  H[0:N] <- T H[0:N] + H[0:N] T + phi h^T,  h <- h + h T,  phi <- T phi + phi
    // (h = H's augmented row). The rank-one term is a fifth k-step whose A column is phi and whose B row is
    // h; lanes 0-15 form h, lanes 16-31 phi. Everything is read before the warp synchronises and writes.
    template <bool kTan>
    static __device__ __forceinline__ void mma_square(SL* sl, int lane) {
        static_assert(N == 16, "tiles of 8 x 8 over a 16 x 16 matrix");
        const int g = lane >> 2, t = lane & 3;
        double* T = sl->T;
        double* H = sl->H;
        double* ph = sl->phi[0];
        double aT[2][4], bT[4][2], cT[2][2][2];
#pragma unroll
        for (int I = 0; I < 2; ++I)
#pragma unroll
            for (int K = 0; K < 4; ++K) aT[I][K] = T[(4 * K + t) * LD + 8 * I + g];
#pragma unroll
        for (int K = 0; K < 4; ++K)
#pragma unroll
            for (int J = 0; J < 2; ++J) bT[K][J] = T[(8 * J + g) * LD + 4 * K + t];
#pragma unroll
        for (int I = 0; I < 2; ++I)
#pragma unroll
            for (int J = 0; J < 2; ++J) {
                cT[I][J][0] = 0.0;
                cT[I][J][1] = 0.0;
#pragma unroll
                for (int K = 0; K < 4; ++K) dmma(cT[I][J][0], cT[I][J][1], aT[I][K], bT[K][J]);
            }
        double cH[2][2][2];
        if constexpr (kTan) {
            double aH[2][4], bH[4][2], aP[2], bP[2];
#pragma unroll
            for (int I = 0; I < 2; ++I) {
#pragma unroll
                for (int K = 0; K < 4; ++K) aH[I][K] = H[(4 * K + t) * LD + 8 * I + g];
                aP[I] = t == 0 ? ph[8 * I + g] : 0.0;
            }
#pragma unroll
            for (int J = 0; J < 2; ++J) {
#pragma unroll
                for (int K = 0; K < 4; ++K) bH[K][J] = H[(8 * J + g) * LD + 4 * K + t];
                bP[J] = t == 0 ? H[(8 * J + g) * LD + N] : 0.0;
            }
#pragma unroll
            for (int I = 0; I < 2; ++I)
#pragma unroll
                for (int J = 0; J < 2; ++J) {
                    cH[I][J][0] = 0.0;
                    cH[I][J][1] = 0.0;
#pragma unroll
                    for (int K = 0; K < 4; ++K) {
                        dmma(cH[I][J][0], cH[I][J][1], aT[I][K], bH[K][J]);
                        dmma(cH[I][J][0], cH[I][J][1], aH[I][K], bT[K][J]);
                    }
                    dmma(cH[I][J][0], cH[I][J][1], aP[I], bP[J]);
                }
        }
        // h (lanes 0-15, one column each) and phi (lanes 16-31, one row each)
        double vec = 0.0;
        if (lane < N) {
            if constexpr (kTan) {
                vec = H[lane * LD + N];
#pragma unroll
                for (int l = 0; l < N; ++l) vec = fma(H[l * LD + N], T[lane * LD + l], vec);
            }
        } else {
            const int i = lane - N;
            vec = ph[i];
#pragma unroll
            for (int l = 0; l < N; ++l) vec = fma(T[l * LD + i], ph[l], vec);
        }
        __syncwarp();
#pragma unroll
        for (int I = 0; I < 2; ++I)
#pragma unroll
            for (int J = 0; J < 2; ++J)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    T[(8 * J + 2 * t + e) * LD + 8 * I + g] = cT[I][J][e];
                    if constexpr (kTan) H[(8 * J + 2 * t + e) * LD + 8 * I + g] = cH[I][J][e];
                }
        if (lane < N) {
            if constexpr (kTan) H[lane * LD + N] = vec;
        } else {
            ph[lane - N] = vec;
        }
        __syncwarp();
    }
};

// kTan false: z only (the same layout and arithmetic without H), for the LM's trial points. Blocks per SM
// the register allocation aims at (a build may set BMC_ADJ_PRIMAL_BLOCKS for a sweep).
#ifndef BMC_ADJ_PRIMAL_BLOCKS
#define BMC_ADJ_PRIMAL_BLOCKS 2
#endif
template <int NC, bool kTan>
__global__ void __launch_bounds__(32 * kAdjWarps, kTan ? 2 : BMC_ADJ_PRIMAL_BLOCKS)
adjoint_kernel(const ChainArgs a, const int* __restrict__ row_ev, int n_tan, const __grid_constant__ TaylorTable tt) {
    using A = Adjoint<NC>;
    using D0 = Dn<double, 0>;
    using C0 = Chain<NC, double, 0>;
    using S = State<NC, D0>;
    using SL = AdjSlot<NC>;
    constexpr int N = A::N, GS = A::GS, G = A::G, LD = A::LD, PHI_LANE = AdjGroup<NC>::PHI_LANE;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SL* slots = reinterpret_cast<SL*>(smem_raw) + (threadIdx.x >> 5) * G;
    const int lane = threadIdx.x & 31, grp = lane / GS, gl = lane % GS;

    const long long nch = (long long)a.n_vox * a.n_off;
    long long ci = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = ci < nch;
    if (!valid) ci = nch - 1;
    if (a.order) ci = a.order[ci];
    const int v = (int)(ci / a.n_off), o = (int)(ci % a.n_off);
    const bool act = valid && (a.active == nullptr || a.active[v] != 0);
    if (__all_sync(kFull, !act)) return;
    const size_t ch = (size_t)v * a.n_off + o;
    const EvRec<double> rec = reinterpret_cast<const EvRec<double>*>(a.ev)[(size_t)row_ev[o] * a.n_off + o];
    unsigned wk1 = 0, wk2 = 0;

    for (int node = 0; node < a.n_nodes; ++node) {
        // this chain's event: coefficients, norm, squarings
        int s = 0;
        Dn<double, 3> g3 = dconst<double, 3>(0.0);
        ChainConst<NC, D0> cc;
        C0::load_const(a, v, node, cc);
        if (!kTan && cc.mt_on && cc.ls != 0 && rec.w1 != 0.0) {
            const D0 offmt = (rec.wf - cc.dw0) - cc.dwmt;
            g3.v = (cc.ls == 1 ? lorentzian<double, 0>(offmt, cc.t2mt)
                               : super_lorentzian<double, 0>(offmt, cc.t2mt, cc.w0sl)).v;
        } else if (kTan && cc.mt_on && cc.ls != 0 && rec.w1 != 0.0) {
            Dn<double, 3> off3 = dconst<double, 3>(((rec.wf - cc.dw0) - cc.dwmt).v);
            Dn<double, 3> t23 = dconst<double, 3>(cc.t2mt.v), w03 = dconst<double, 3>(cc.w0sl.v);
            off3.d[0] = 1.0;
            t23.d[1] = 1.0;
            w03.d[2] = 1.0;
            g3 = cc.ls == 1 ? lorentzian<double, 3>(off3, t23) : super_lorentzian<double, 3>(off3, t23, w03);
        }
        const double g0 = g3.v;
        StepCoef<NC, D0> sc;
        C0::event_coef(cc, rec, dconst<double, 0>(g0), sc);
        double nu = rec.dt * C0::coef_norm(sc, cc);
        if (!(nu < INFINITY)) {
            if (act) atomicOr(a.status, 1);
            nu = 0.0;
        }
        if (nu > tt.dense_theta) s = (int)ceil(log2(nu / tt.dense_theta));
        bool capped = false;   // more squarings than the cap: this chain's results become NaN
        if (s > 200) {
            s = 200;
            capped = true;
            if (act) atomicOr(a.status, 2);
        }
        const double h = ldexp(rec.dt, -s);

        unsigned need = __ballot_sync(kFull, act);
        while (need) {
            int my_slot = -1, grp_owner = -1;
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int c = need ? __ffs(need) - 1 : -1;
                if (need) need &= need - 1;
                if (c == lane) my_slot = g;
                if (g == grp) grp_owner = c;
            }
            if (my_slot >= 0) {
                SL* sl = &slots[my_slot];
                StepCoef<NC, D0> scs = sc;
                C0::scale_coef(scs, h);
                sl->coef = scs;
                sl->cw = h * cc.cw.v;
                sl->cm = h * cc.cm.v;
#pragma unroll
                for (int i = 0; i < NC; ++i) sl->cc[i] = h * cc.cc[i].v;
                const double* m0 = a.m0 + (size_t)v * N;
#pragma unroll
                for (int q = 0; q < N; ++q) sl->v[q] = m0[q];
                sl->v[N] = 1.0;
                sl->rec = rec;
                sl->g0 = g0;
                sl->gd[0] = g3.d[0];
                sl->gd[1] = g3.d[1];
                sl->gd[2] = g3.d[2];
                sl->scale = ldexp(1.0, -s);
                sl->s = s;
                sl->vox = v;
                if (a.work) {
                    wk1 += unsigned((N + 1) * tt.dense_m);
                    wk2 += unsigned(s);
                }
            }
            __syncwarp();
            SL* sl = &slots[grp];
            const bool have = grp_owner >= 0;
            if constexpr (kTan) {
                if (have)
                    for (int p = gl; p < n_tan; p += GS) A::tangent_set(a, sl, node, p);
            }
            const bool work = have && gl < N;
            const int s_g = have ? sl->s : 0;
            const int smax = (int)__reduce_max_sync(kFull, (unsigned)s_g);
            // column gl of exp(X / 2^s) and of its derivative along E / 2^s: Horner, T = I + X T / k
            S cv, cd;
            double cdN = 0.0;
            A::unit(cv, gl);
            A::unit(cd, -1);
            if (work) {
                const double e2 = sl->scale;
                for (int k = tt.dense_m; k >= 1; --k) {
                    S yv;
                    C0::template matvec<false>(sl->coef, cv, yv);
                    const double ik = tt.inv_k[k];
                    if constexpr (kTan) {
                        S yd;
                        A::op(sl, cd, cdN, yd);
                        const double dot = e2 * A::get(cv, a.mz);     // (E / 2^s) column: v (lam . col) / 2^s
#pragma unroll
                        for (int q = 0; q < N; ++q) C0::at(cd, q).v = ik * fma(dot, sl->v[q], C0::at(yd, q).v);
                        cdN = ik * dot;
                    }
#pragma unroll
                    for (int q = 0; q < N; ++q) C0::at(cv, q).v = (q == gl ? 1.0 : 0.0) + ik * C0::at(yv, q).v;
                }
            }
            // the augmented column: [phi; 1] <- e_N + X [phi; 1] / k
            if (have && gl == PHI_LANE) {
                S ph;
                A::unit(ph, -1);
                for (int k = tt.dense_m; k >= 1; --k) {
                    S y;
                    A::op(sl, ph, 1.0, y);
                    const double ik = tt.inv_k[k];
#pragma unroll
                    for (int q = 0; q < N; ++q) C0::at(ph, q).v = ik * C0::at(y, q).v;
                }
#pragma unroll
                for (int q = 0; q < N; ++q) sl->phi[0][q] = C0::at(ph, q).v;
            }
            __syncwarp();
            // s squarings: [T, H] <- [T T, T H + H T], phi <- T phi + phi
            if constexpr (AdjGroup<NC>::kMma) {
                if (work) {
#pragma unroll
                    for (int i = 0; i < N; ++i) {
                        sl->T[gl * LD + i] = C0::at(cv, i).v;
                        if constexpr (kTan) sl->H[gl * LD + i] = C0::at(cd, i).v;
                    }
                    if constexpr (kTan) sl->H[gl * LD + N] = cdN;
                }
                __syncwarp();
                for (int q = 0; q < smax; ++q) {
#pragma unroll
                    for (int c = 0; c < G; ++c) {
                        const int s_c = __shfl_sync(kFull, s_g, c * GS);
                        if (q < s_c) A::template mma_square<kTan>(&slots[c], lane);
                    }
                }
                if (work) {
#pragma unroll
                    for (int i = 0; i < N; ++i) {
                        C0::at(cv, i).v = sl->T[gl * LD + i];
                        if constexpr (kTan) C0::at(cd, i).v = sl->H[gl * LD + i];
                    }
                    if constexpr (kTan) cdN = sl->H[gl * LD + N];
                }
            } else {
                for (int q = 0; q < smax; ++q) {
                    const bool sq = work && q < s_g;
                    if (sq) {
#pragma unroll
                        for (int i = 0; i < N; ++i) {
                            sl->T[gl * LD + i] = C0::at(cv, i).v;
                            if constexpr (kTan) sl->H[gl * LD + i] = C0::at(cd, i).v;
                        }
                        if constexpr (kTan) sl->H[gl * LD + N] = cdN;
                    }
                    __syncwarp();
                    if (sq) {
                        const double* ph = sl->phi[q & 1];
                        S nv, nd;
                        double ndN = cdN, pj = ph[gl];
#pragma unroll
                        for (int i = 0; i < N; ++i) {
                            C0::at(nv, i).v = 0.0;
                            if constexpr (kTan) C0::at(nd, i).v = ph[i] * cdN;
                        }
#pragma unroll
                        for (int l = 0; l < N; ++l) {
                            const double wv = C0::at(cv, l).v;
#pragma unroll
                            for (int i = 0; i < N; ++i) {
                                const double t = sl->T[l * LD + i];
                                C0::at(nv, i).v = fma(t, wv, C0::at(nv, i).v);
                                if constexpr (kTan)
                                    C0::at(nd, i).v = fma(t, C0::at(cd, l).v, fma(sl->H[l * LD + i], wv, C0::at(nd, i).v));
                            }
                            if constexpr (kTan) ndN = fma(sl->H[l * LD + N], wv, ndN);
                            pj = fma(sl->T[l * LD + gl], ph[l], pj);
                        }
                        sl->phi[(q + 1) & 1][gl] = pj;
                        cv = nv;
                        if constexpr (kTan) {
                            cd = nd;
                            cdN = ndN;
                        }
                    }
                    __syncwarp();
                }
            }
            // z = sum_j (exp(X)^T lam)_j v_j (phi[mz] for j = N), and per tangent
            // tr(dX_p H) + (exp(X)^T lam) . dv_p
            const double u = work ? A::get(cv, a.mz) : 0.0;
            const double zsum = group_sum<GS>(work ? u * sl->v[gl] : 0.0);
            for (int p = 0; p < (kTan ? n_tan : 0); ++p) {
                double gp = 0.0;
                if (work) {
                    gp = A::dop_row(sl, p, cd, cdN, gl);
                    if (a.dm0) gp = fma(u, a.dm0[((size_t)p * a.n_vox + sl->vox) * N + gl], gp);
                }
                gp = group_sum<GS>(gp);
                if (have && gl == 0) sl->res[p] = gp;
            }
            if (have && gl == 0) sl->res[kMaxT] = zsum + sl->phi[AdjGroup<NC>::kMma ? 0 : (s_g & 1)][a.mz];
            __syncwarp();
            if (my_slot >= 0) {
                const SL* ms = &slots[my_slot];
                const double wgt = a.n_nodes > 1 ? a.w[node] : 1.0;
                const double z = capped ? NAN : ms->res[kMaxT];
                a.out[ch] = (node ? a.out[ch] : 0.0) + wgt * z;
                for (int p = 0; p < (kTan ? n_tan : 0); ++p) {
                    double* jp = a.jout + ((size_t)p * a.n_vox + v) * a.n_off + o;
                    *jp = (node ? *jp : 0.0) + wgt * (capped ? NAN : ms->res[p]);
                }
            }
            __syncwarp();
        }
    }
    if (a.work) {
#pragma unroll
        for (int q = 1; q < 3; ++q) {
            unsigned long long x = act ? (unsigned long long)(q == 1 ? wk1 : wk2) : 0ull;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(kFull, x, off);
            if (lane == 0 && x) atomicAdd(a.work + q, x);
        }
    }
}

}  // namespace bmc
