// bmc_adjoint_block.cuh -- every tangent of an uneven batch's repeated-block rows in one pass (reverse mode).
//
// A row whose evolving events are one block of L <= kAdjL events repeated r times (a train of block pulses
// and gaps followed by the readout: the uneven configuration's rows; r = 1 covers a single pass) ends at
//     z = lam^T P^r v,   P = E_{L-1} ... E_0,  E_i = exp(X_i),  v = [M0; 1],  lam = e_mz.
// Its tangent along p is
//     dz_p = tr(dP_p W) + (P^r)^T lam . dv_p,   W = sum_{k<r} P^k v lam^T P^{r-1-k},
//     tr(dP_p W) = sum_i tr(dE_{i,p} W_i) = sum_i tr(dX_{i,p} G_i),
//     W_i = (E_{i-1} ... E_0) W (E_{L-1} ... E_{i+1}),  G_i = L(X_i, W_i)
// (tr(L(X, E) W) = tr(E L(X, W)) for the Frechet derivative L). W comes from the adjoint states
// b_m = (P^T)^m lam and the forward states a_k = P^k v: W = sum_k a_k b_{r-1-k}^T, lane j accumulating its
// column from its own entries of the b_m. Each G_i is one dual scaling and squaring of X_i in the dense
// direction W_i, shared by every tangent; forward mode (the chain kernel's block path with dual numbers)
// carries each tangent through the block's exponentials and its r applications instead.
//
// Layout as on the chain kernel's dense path: a group of GS lanes per chain, lane j <= N holding column j of
// the matrix at hand (the augmented column N included); matrices in shared memory, column-major, all
// N + 1 rows stored.
#pragma once
#include "bmc_adjoint.cuh"

namespace bmc {

constexpr int kAdjL = 2;      // block events the kernel takes
constexpr int kAdjMaxR = 64;  // block repeats it takes

// kTan false (the primal passes): the tangent-only members shrink to one element, so that the slot
// leaves shared memory for more resident blocks
template <int NC, bool kTan = true>
struct AdjBlkSlotBody {
    static constexpr int N = Layout<NC>::N;
    static constexpr int NA = N + 1;
    static constexpr int LD = DenseGroup<NC>::LD;
    using K = StepCoef<NC, Dn<double, 0>>;
    K coef[kAdjL];                            // each event's coefficients times h_i = dt_i / 2^s_i
    double C[NC + 2];                         // the constant column (water z, MT z, CEST z), unscaled
    double E[kAdjL][NA * LD];                 // the events' propagators
    double P[NA * LD];                        // the block propagator; then T of the Frechet squarings
    double A[kTan ? NA * LD : 1];             // W and its right products
    double B[kTan ? NA * LD : 1];             // W_i; then H of the Frechet squarings
    double vec[2][NA];
    K dk[kAdjL][kTan ? kMaxT : 1];            // per event and tangent: d(coefficients) * dt_i
    double dC[kTan ? kMaxT : 1][NC + 2];      // per tangent: d(constant column), unscaled
    double res[kMaxT + 1];
    EvRec<double> rec[kAdjL];
    double g0[kAdjL], gd[kAdjL][3], h[kAdjL], scale[kAdjL];
    int s[kAdjL], moves[kAdjL];
    int L, r, vox;
};

template <int NC, bool kTan = true>
struct AdjBlkSlot : AdjBlkSlotBody<NC, kTan> {
    static constexpr size_t kBody = sizeof(AdjBlkSlotBody<NC, kTan>);
    static constexpr size_t kTarget = (128 / DenseGroup<NC>::G) % 128;
    static constexpr size_t kPad = (kTarget + 128 - kBody % 128) % 128;
    char pad[kPad == 0 ? 128 : kPad];
};

constexpr int kAdjBlkWarps = 4;

// Rows the block kernel can take, one thread per row of one table: the evolving events (dt > 1e-9) are
// exactly the repeated block found by block_scan_kernel (seg), or, with no block, lie in one window of at
// most kAdjL events taken once; the block's events are RF blocks or delays; no spoiler or gradient
// anywhere; no readout that resets the state before the row ends. out[row] = (first, L, r, 1) or zero;
// *all_ok is cleared when a row does not qualify.
__global__ void adjoint_block_rows_kernel(const EvRec<double>* __restrict__ rec, int n_rows, int n_ev, int stride,
                                          const int4* __restrict__ seg, int reset_after_adc,
                                          int4* __restrict__ out, int* __restrict__ all_ok) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n_rows) return;
    const int4 b = seg ? seg[o] : make_int4(0, 0, 0, 0);
    int first = -1, last = -1, moving = 0;
    bool ok = true;
    for (int e = 0; e < n_ev; ++e) {
        const EvRec<double> x = rec[(size_t)e * stride + o];
        const int type = (int)x.type;
        ok = ok && type != EV_GRADIENT && type != EV_SPOILER;
        if (x.dt > 1e-9) {
            ok = ok && (type == EV_RF || type == EV_DELAY);
            if (first < 0) first = e;
            last = e;
            ++moving;
        } else if (type == EV_ADC && moving > 0 && reset_after_adc && e + 1 < n_ev) {
            ok = false;
        }
    }
    int4 res = make_int4(0, 0, 0, 0);
    if (ok && moving > 0) {
        if (b.z >= 2) {
            // the block must hold every evolving event
            ok = first >= b.x && last < b.x + b.y * b.z && b.y <= kAdjL && b.z <= kAdjMaxR;
            res = make_int4(b.x, b.y, b.z, 1);
        } else {
            ok = last - first + 1 <= kAdjL;
            res = make_int4(first, last - first + 1, 1, 1);
        }
    } else {
        ok = false;
    }
    out[o] = ok ? res : make_int4(0, 0, 0, 0);
    if (!ok) atomicAnd(all_ok, 0);
}

template <int NC, bool kTan = true>
struct AdjBlk {
    using D0 = Dn<double, 0>;
    using D1 = Dn<double, 1>;
    using C0 = Chain<NC, double, 0>;
    using C1 = Chain<NC, double, 1>;
    using S = State<NC, D0>;
    using K = StepCoef<NC, D0>;
    using SL = AdjBlkSlot<NC, kTan>;
    static constexpr int N = Layout<NC>::N;
    static constexpr int NA = N + 1;
    static constexpr int GS = DenseGroup<NC>::GS;
    static constexpr int G = DenseGroup<NC>::G;
    static constexpr int LD = DenseGroup<NC>::LD;

    static __device__ __forceinline__ double get(const S& x, int q) {
        double r = 0.0;
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (i == q) r = C0::at(const_cast<S&>(x), i).v;
        return r;
    }
    static __device__ __forceinline__ void unit(S& x, int j) {
#pragma unroll
        for (int q = 0; q < N; ++q) C0::at(x, q).v = q == j ? 1.0 : 0.0;
    }
    // y = X_i,s x + C h_i c (rows 0 .. N - 1)
    static __device__ __forceinline__ void op(const SL* sl, int i, const S& x, double c, S& y) {
        C0::template matvec<false>(sl->coef[i], x, y);
        const double hc = sl->h[i] * c;
        y.zw.v = fma(sl->C[0], hc, y.zw.v);
        y.zm.v = fma(sl->C[1], hc, y.zm.v);
#pragma unroll
        for (int k = 0; k < NC; ++k) y.zc[k].v = fma(sl->C[2 + k], hc, y.zc[k].v);
    }
    // entry q of dX_{i,p} [x; c] (dk already times dt_i; dC unscaled)
    static __device__ __forceinline__ double dop_row(const SL* sl, int i, int p, const S& x, double c, int q) {
        S y;
        C0::template matvec<false>(sl->dk[i][p], x, y);
        const double dc = sl->rec[i].dt * c;
        y.zw.v = fma(sl->dC[p][0], dc, y.zw.v);
        y.zm.v = fma(sl->dC[p][1], dc, y.zm.v);
#pragma unroll
        for (int k = 0; k < NC; ++k) y.zc[k].v = fma(sl->dC[p][2 + k], dc, y.zc[k].v);
        return get(y, q);
    }
    // x (rows 0 .. N) <- M x, M an (N+1) x (N+1) column-major matrix in shared memory
    static __device__ __forceinline__ void mat_vec(const double* M, double (&x)[NA]) {
        double y[NA];
#pragma unroll
        for (int q = 0; q < NA; ++q) y[q] = 0.0;
#pragma unroll
        for (int l = 0; l < NA; ++l) {
            const double w = x[l];
#pragma unroll
            for (int q = 0; q < NA; ++q) y[q] = fma(M[l * LD + q], w, y[q]);
        }
#pragma unroll
        for (int q = 0; q < NA; ++q) x[q] = y[q];
    }
    static __device__ __forceinline__ void load_col(const double* M, int j, double (&x)[NA]) {
#pragma unroll
        for (int q = 0; q < NA; ++q) x[q] = M[j * LD + q];
    }
    static __device__ __forceinline__ void store_col(double* M, int j, const double (&x)[NA]) {
#pragma unroll
        for (int q = 0; q < NA; ++q) M[j * LD + q] = x[q];
    }

    // Lane task (i, p): the derivative of event i's coefficients along tangent p, times dt_i, and (i == 0)
    // the constant column's derivative.
    static __device__ void tangent_set(const ChainArgs& a, SL* sl, int node, int i, int p) {
        ChainConst<NC, D1> cp;
        C1::load_const(a, sl->vox, node, cp, p);
        const EvRec<double>& rec = sl->rec[i];
        D1 g = dconst<double, 1>(sl->g0[i]);
        if (cp.mt_on && cp.ls != 0 && rec.w1 != 0.0) {
            const D1 offmt = (rec.wf - cp.dw0) - cp.dwmt;
            g.d[0] = fma(sl->gd[i][0], offmt.d[0], fma(sl->gd[i][1], cp.t2mt.d[0], sl->gd[i][2] * cp.w0sl.d[0]));
        }
        StepCoef<NC, D1> sp;
        C1::event_coef(cp, rec, g, sp);
        const double dt = rec.dt;
        K& d = sl->dk[i][p];
        d.Rw2.v = dt * sp.Rw2.d[0];
        d.Rw1.v = dt * sp.Rw1.d[0];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            d.k[k].v = dt * sp.k[k].d[0];
            d.kwc[k].v = dt * sp.kwc[k].d[0];
            d.Rc2[k].v = dt * sp.Rc2[k].d[0];
            d.Rc1[k].v = dt * sp.Rc1[k].d[0];
            d.offc[k].v = dt * sp.offc[k].d[0];
        }
        d.offw.v = dt * sp.offw.d[0];
        d.w1x.v = dt * sp.w1x.d[0];
        d.w1y.v = dt * sp.w1y.d[0];
        d.kmt.v = dt * sp.kmt.d[0];
        d.kwmt.v = dt * sp.kwmt.d[0];
        d.Rm1W.v = dt * sp.Rm1W.d[0];
        if (i == 0) {
            sl->dC[p][0] = cp.cw.d[0];
            sl->dC[p][1] = cp.cm.d[0];
#pragma unroll
            for (int k = 0; k < NC; ++k) sl->dC[p][2 + k] = cp.cc[k].d[0];
        }
    }

    // column gl of exp(X_i) into E[i] (T kept in the slot's P during the squarings)
    static __device__ void exp_event(SL* sl, int i, int gl, bool work, int s_g, int smax, const TaylorTable& tt) {
        const double caug = gl == N ? 1.0 : 0.0;
        S cv;
        unit(cv, gl);
        if (work) {
            for (int k = tt.dense_m; k >= 1; --k) {
                S y;
                op(sl, i, cv, caug, y);
                const double ik = tt.inv_k[k];
#pragma unroll
                for (int q = 0; q < N; ++q) C0::at(cv, q).v = (q == gl ? 1.0 : 0.0) + ik * C0::at(y, q).v;
            }
        }
        double* T = sl->P;
        for (int q = 0; q < smax; ++q) {
            const bool sq = work && q < s_g;
            if (sq) {
#pragma unroll
                for (int r = 0; r < N; ++r) T[gl * LD + r] = C0::at(cv, r).v;
            }
            __syncwarp();
            if (sq) {
                // the lane's own column is read back from shared memory, so that the l loop need not index
                // registers and can stay partly rolled
                S nv;
#pragma unroll
                for (int r = 0; r < N; ++r) C0::at(nv, r).v = caug * T[N * LD + r];
#pragma unroll 4
                for (int l = 0; l < N; ++l) {
                    const double w = T[gl * LD + l];
#pragma unroll
                    for (int r = 0; r < N; ++r) C0::at(nv, r).v = fma(T[l * LD + r], w, C0::at(nv, r).v);
                }
                cv = nv;
            }
            __syncwarp();
        }
        if (work) {
            double* Ei = sl->E[i];
#pragma unroll
            for (int r = 0; r < N; ++r) Ei[gl * LD + r] = C0::at(cv, r).v;
            Ei[gl * LD + N] = caug;
        }
    }

    // G_i = L(X_i, W_i) (W_i in the slot's B): column gl into (cd, cdN); T and H in P and B
    static __device__ void frechet_event(SL* sl, int i, int gl, bool work, int s_g, int smax, const TaylorTable& tt,
                                         S& cd, double& cdN) {
        const double caug = gl == N ? 1.0 : 0.0;
        S cv;
        unit(cv, gl);
        unit(cd, -1);
        cdN = 0.0;
        if (work) {
            const double e2 = sl->scale[i];
            const double* W = sl->B;
            // this lane's current column, stored where the squarings' T will go (free until then): the
            // dense product with W_i reads its multipliers back from there, so that its l loop stays rolled
            // (fully unrolled, that product's 17 x 17 loads spilled registers)
            double* col = sl->P + gl * LD;
            for (int k = tt.dense_m; k >= 1; --k) {
                const double ik = tt.inv_k[k];
#pragma unroll
                for (int q = 0; q < N; ++q) col[q] = C0::at(cv, q).v;
                // tangent column first, from the current cv: cd <- (X_s cd + (W_i / 2^s) [cv; caug]) / k
                {
                    S yd;
                    op(sl, i, cd, cdN, yd);
                    double wn = e2 * W[N * LD + N] * caug;
#pragma unroll
                    for (int q = 0; q < N; ++q) C0::at(yd, q).v = fma(e2 * W[N * LD + q], caug, C0::at(yd, q).v);
#pragma unroll 2
                    for (int l = 0; l < N; ++l) {
                        const double x = e2 * col[l];
#pragma unroll
                        for (int q = 0; q < N; ++q) C0::at(yd, q).v = fma(W[l * LD + q], x, C0::at(yd, q).v);
                        wn = fma(W[l * LD + N], x, wn);
                    }
#pragma unroll
                    for (int q = 0; q < N; ++q) C0::at(cd, q).v = ik * C0::at(yd, q).v;
                    cdN = ik * wn;
                }
                // then the primal column: cv <- e_gl + X_s [cv; caug] / k
                S yv;
                op(sl, i, cv, caug, yv);
#pragma unroll
                for (int q = 0; q < N; ++q) C0::at(cv, q).v = (q == gl ? 1.0 : 0.0) + ik * C0::at(yv, q).v;
            }
        }
        __syncwarp();   // W_i is read by every lane before the squarings overwrite B
        double* T = sl->P;
        double* H = sl->B;
        for (int q = 0; q < smax; ++q) {
            const bool sq = work && q < s_g;
            if (sq) {
#pragma unroll
                for (int r = 0; r < N; ++r) {
                    T[gl * LD + r] = C0::at(cv, r).v;
                    H[gl * LD + r] = C0::at(cd, r).v;
                }
                H[gl * LD + N] = cdN;
            }
            __syncwarp();
            if (sq) {
                S nv, nd;
                double ndN = cdN;
#pragma unroll
                for (int r = 0; r < N; ++r) {
                    const double t_aug = T[N * LD + r], h_aug = H[N * LD + r];
                    C0::at(nv, r).v = caug * t_aug;
                    C0::at(nd, r).v = fma(t_aug, cdN, caug * h_aug);
                }
                ndN = fma(caug, H[N * LD + N], ndN);
#pragma unroll 2
                for (int l = 0; l < N; ++l) {
                    const double wv = T[gl * LD + l], wd = H[gl * LD + l];   // this lane's column, as stored
#pragma unroll
                    for (int r = 0; r < N; ++r) {
                        const double t = T[l * LD + r];
                        C0::at(nv, r).v = fma(t, wv, C0::at(nv, r).v);
                        C0::at(nd, r).v = fma(t, wd, fma(H[l * LD + r], wv, C0::at(nd, r).v));
                    }
                    ndN = fma(H[l * LD + N], wv, ndN);
                }
                cv = nv;
                cd = nd;
                cdN = ndN;
            }
            __syncwarp();
        }
    }
};

// kTan false: z only (phases A, B and D without W), for the plan's primal passes, with a smaller slot and
// registers capped for BMC_ADJ_BLK_PRIMAL_BLOCKS resident blocks (a build may set it for a sweep)
#ifndef BMC_ADJ_BLK_PRIMAL_BLOCKS
#define BMC_ADJ_BLK_PRIMAL_BLOCKS 3
#endif
template <int NC, bool kTan>
__global__ void __launch_bounds__(32 * kAdjBlkWarps, kTan ? 2 : BMC_ADJ_BLK_PRIMAL_BLOCKS)
adjoint_block_kernel(const ChainArgs a, const int4* __restrict__ blk, int n_tan, const __grid_constant__ TaylorTable tt) {
    using AB = AdjBlk<NC, kTan>;
    using D0 = Dn<double, 0>;
    using C0 = Chain<NC, double, 0>;
    using S = State<NC, D0>;
    using SL = AdjBlkSlot<NC, kTan>;
    constexpr int N = AB::N, NA = AB::NA, GS = AB::GS, G = AB::G, LD = AB::LD;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SL* slots = reinterpret_cast<SL*>(smem_raw) + (threadIdx.x >> 5) * G;
    const int lane = threadIdx.x & 31, grp = lane / GS, gl = lane % GS;

    const long long nch = a.n_chains;
    long long ci = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = ci < nch;
    if (!valid) ci = nch - 1;
    if (a.order) ci = a.order[ci];
    const int2 vm = a.chain_map[ci];
    const int v = vm.x, o = vm.y;
    const int t = a.vox_table[v];
    const EvRec<double>* ev = reinterpret_cast<const EvRec<double>*>(a.ev) + a.tab_base[t];
    const int stride = a.tab_noff[t];
    const int4 b = blk[a.tab_row0[t] + o];
    const bool act = valid && (a.active == nullptr || a.active[v] != 0);
    if (__all_sync(kFull, !act)) return;
    const size_t ch = (size_t)ci;
    unsigned wk1 = 0, wk2 = 0;
    double bh[kAdjMaxR];   // this lane's entries of the adjoint states b_0 .. b_{r-1}

    for (int node = 0; node < a.n_nodes; ++node) {
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
            bool capped = false;
            if (my_slot >= 0) {
                // the owner: its block's events, coefficients and squarings into the slot
                SL* sl = &slots[my_slot];
                ChainConst<NC, D0> cc;
                C0::load_const(a, v, node, cc);
                sl->C[0] = cc.cw.v;
                sl->C[1] = cc.cm.v;
#pragma unroll
                for (int k = 0; k < NC; ++k) sl->C[2 + k] = cc.cc[k].v;
                sl->L = b.y;
                sl->r = b.z;
                sl->vox = v;
                for (int i = 0; i < kAdjL; ++i) {
                    const bool in = i < b.y;
                    const EvRec<double> rec = in ? ev[(size_t)(b.x + i) * stride + o] : EvRec<double>{};
                    const bool moves = in && rec.dt > 1e-9;
                    sl->rec[i] = rec;
                    sl->moves[i] = moves ? 1 : 0;
                    int s = 0;
                    Dn<double, 3> g3 = dconst<double, 3>(0.0);
                    if (moves) {
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
                            g3 = cc.ls == 1 ? lorentzian<double, 3>(off3, t23)
                                            : super_lorentzian<double, 3>(off3, t23, w03);
                        }
                        StepCoef<NC, D0> sc;
                        C0::event_coef(cc, rec, dconst<double, 0>(g3.v), sc);
                        double nu = rec.dt * C0::coef_norm(sc, cc);
                        if (!(nu < INFINITY)) {
                            atomicOr(a.status, 1);
                            nu = 0.0;
                        }
                        if (nu > tt.dense_theta) s = (int)ceil(log2(nu / tt.dense_theta));
                        if (s > 200) {
                            s = 200;
                            capped = true;
                            atomicOr(a.status, 2);
                        }
                        const double h = ldexp(rec.dt, -s);
                        C0::scale_coef(sc, h);
                        sl->coef[i] = sc;
                        sl->h[i] = h;
                        sl->scale[i] = ldexp(1.0, -s);
                        if (a.work) {
                            // the exponential (and with tangents its Frechet derivative)
                            wk1 += unsigned((kTan ? 2 : 1) * NA * tt.dense_m);
                            wk2 += unsigned((kTan ? 2 : 1) * s);
                        }
                    }
                    sl->s[i] = s;
                    sl->g0[i] = g3.v;
                    sl->gd[i][0] = g3.d[0];
                    sl->gd[i][1] = g3.d[1];
                    sl->gd[i][2] = g3.d[2];
                }
            }
            __syncwarp();
            SL* sl = &slots[grp];
            const bool have = grp_owner >= 0;
            const bool work = have && gl < NA;
            const int L = have ? sl->L : 0, r = have ? sl->r : 0;
            const int Lmax = (int)__reduce_max_sync(kFull, (unsigned)L);
            const int rmax = (int)__reduce_max_sync(kFull, (unsigned)r);
            // tangent coefficient sets: lane task q = (event, tangent)
            if constexpr (kTan) {
                if (have)
                    for (int q = gl; q < L * n_tan; q += GS) AB::tangent_set(a, sl, node, q / n_tan, q % n_tan);
            }
            // A: the events' propagators
            for (int i = 0; i < Lmax; ++i) {
                const bool mv = have && i < L && sl->moves[i];
                const int s_g = mv ? sl->s[i] : 0;
                const int smax = (int)__reduce_max_sync(kFull, (unsigned)s_g);
                AB::exp_event(sl, i, gl, work && mv, s_g, smax, tt);
            }
            __syncwarp();
            // B: the block propagator P = E_{L-1} ... E_0, column gl (an event that does not move is the identity)
            double x[NA];
#pragma unroll
            for (int q = 0; q < NA; ++q) x[q] = q == gl ? 1.0 : 0.0;
            if (work)
                for (int i = 0; i < L; ++i)
                    if (sl->moves[i]) AB::mat_vec(sl->E[i], x);
            if (work) AB::store_col(sl->P, gl, x);
            __syncwarp();
            double b_r = 0.0;
            if constexpr (kTan) {
                // C: adjoint states b_{m+1} = P^T b_m from b_0 = lam, b_m in vec[m & 1]; lane gl keeps its entries
                // (x = P[:, gl])
                if (work) sl->vec[0][gl] = gl == a.mz ? 1.0 : 0.0;
                __syncwarp();
                for (int m = 0; m < rmax; ++m) {
                    double bn = 0.0;
                    if (work && m < r) {
                        const double* bv = sl->vec[m & 1];
                        bh[m] = bv[gl];
#pragma unroll
                        for (int l = 0; l < NA; ++l) bn = fma(x[l], bv[l], bn);
                    }
                    __syncwarp();
                    if (work && m < r) sl->vec[(m + 1) & 1][gl] = bn;
                    __syncwarp();
                }
                b_r = work ? sl->vec[r & 1][gl] : 0.0;
                __syncwarp();
            }
            // D: forward states a_{k+1} = P a_k from a_0 = [M0; 1], a_k in vec[k & 1]; lane gl accumulates
            // column gl of W
            if (work) {
                const double* m0 = a.m0 + (size_t)sl->vox * N;
                sl->vec[0][gl] = gl < N ? m0[gl] : 1.0;
            }
            __syncwarp();
            double w[NA];
#pragma unroll
            for (int q = 0; q < NA; ++q) w[q] = 0.0;
            for (int k = 0; k < rmax; ++k) {
                double an = 0.0;
                if (work && k < r) {
                    const double* av = sl->vec[k & 1];
                    if constexpr (kTan) {
                        const double bj = bh[r - 1 - k];
#pragma unroll
                        for (int q = 0; q < NA; ++q) w[q] = fma(av[q], bj, w[q]);
                    }
#pragma unroll
                    for (int l = 0; l < NA; ++l) an = fma(sl->P[l * LD + gl], av[l], an);
                }
                __syncwarp();
                if (work && k < r) sl->vec[(k + 1) & 1][gl] = an;
                __syncwarp();
            }
            const double z = have ? sl->vec[r & 1][a.mz] : 0.0;
            double gacc[kMaxT];
#pragma unroll
            for (int p = 0; p < kMaxT; ++p) gacc[p] = 0.0;
            if constexpr (kTan) {
                if (work) AB::store_col(sl->A, gl, w);
                __syncwarp();
                // E: per event, from the last: W_i = (E_{i-1} ... E_0) R_i with R_i = W E_{L-1} ... E_{i+1} (in A),
                // then G_i = L(X_i, W_i) and the contractions
                for (int i = Lmax - 1; i >= 0; --i) {
                    const bool mv = have && i < L && sl->moves[i];
                    if (work && mv) {
                        AB::load_col(sl->A, gl, x);
                        for (int q = 0; q < i; ++q)
                            if (sl->moves[q]) AB::mat_vec(sl->E[q], x);
                        AB::store_col(sl->B, gl, x);
                    }
                    __syncwarp();
                    const int s_g = mv ? sl->s[i] : 0;
                    const int smax = (int)__reduce_max_sync(kFull, (unsigned)s_g);
                    S cd;
                    double cdN;
                    AB::frechet_event(sl, i, gl, work && mv, s_g, smax, tt, cd, cdN);
                    if (work && mv && gl < N) {
#pragma unroll
                        for (int p = 0; p < kMaxT; ++p)
                            if (p < n_tan) gacc[p] += AB::dop_row(sl, i, p, cd, cdN, gl);
                    }
                    // R_{i-1} = R_i E_i: column gl is R_i E_i[:, gl]
                    if (i > 0) {
                        double y[NA];
                        if (work && mv) {
#pragma unroll
                            for (int q = 0; q < NA; ++q) y[q] = 0.0;
                            const double* Ei = sl->E[i];
#pragma unroll
                            for (int l = 0; l < NA; ++l) {
                                const double e = Ei[gl * LD + l];
#pragma unroll
                                for (int q = 0; q < NA; ++q) y[q] = fma(sl->A[l * LD + q], e, y[q]);
                            }
                        }
                        __syncwarp();
                        if (work && mv) AB::store_col(sl->A, gl, y);
                        __syncwarp();
                    }
                }
                // the start state's tangents: (P^r)^T lam . dv_p
                if (work && gl < N && a.dm0) {
#pragma unroll
                    for (int p = 0; p < kMaxT; ++p)
                        if (p < n_tan) gacc[p] = fma(b_r, a.dm0[((size_t)p * a.n_vox + sl->vox) * N + gl], gacc[p]);
                }
            }
#pragma unroll
            for (int p = 0; p < kMaxT; ++p) {
                const double gs = group_sum<GS>(p < n_tan ? gacc[p] : 0.0);
                if (have && gl == 0 && p < n_tan) sl->res[p] = gs;
            }
            if (have && gl == 0) sl->res[kMaxT] = z;
            __syncwarp();
            if (my_slot >= 0) {
                const SL* ms = &slots[my_slot];
                const double wgt = a.n_nodes > 1 ? a.w[node] : 1.0;
                a.out[ch] = (node ? a.out[ch] : 0.0) + wgt * (capped ? NAN : ms->res[kMaxT]);
                for (int p = 0; p < n_tan; ++p) {
                    double* jp = a.jout + (size_t)p * a.n_chains + ch;
                    *jp = (node ? *jp : 0.0) + wgt * (capped ? NAN : ms->res[p]);
                }
            }
            __syncwarp();
        }
    }
    if (a.work) {
#pragma unroll
        for (int q = 1; q < 3; ++q) {
            unsigned long long y = act ? (unsigned long long)(q == 1 ? wk1 : wk2) : 0ull;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) y += __shfl_xor_sync(kFull, y, off);
            if (lane == 0 && y) atomicAdd(a.work + q, y);
        }
    }
}

}  // namespace bmc
