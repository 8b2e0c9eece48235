// bmc_kernels.cuh -- the chain kernel, its dense long-event path, and the event preprocessing.
#pragma once
#include <type_traits>

#include "bmc_chain.cuh"

namespace bmc {

constexpr unsigned kFull = 0xffffffffu;

template <typename R>
__device__ __forceinline__ R warp_max(R x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(kFull, x, o));
    return x;
}

// ------------------------------------------------------------------------------------------------
// dense path: a warp exponentiates one chain's generator at a time, lane j owning column j
// ------------------------------------------------------------------------------------------------
// For an event whose generator X = [A C; 0 0] dt has a large norm (a long delay or CW block), the
// Taylor action would need ~||X|| sub-steps. Instead the warp forms exp(X) by scaling and squaring:
// exp(X / 2^s) by a degree-m Horner recurrence (each column by the sparse operator, in registers),
// then s squarings through shared memory, then the matrix-vector product with [M; 1].

// the norm above which an event inside a repeated block is exponentiated densely (a short event acts on
// the block propagator's columns by the truncated Taylor series instead)
constexpr double kBlockDenseNorm = 4.0;

// lanes per chain in the dense path: one column per lane, so a warp works on 32 / GS chains at once
template <int NC>
struct DenseGroup {
    static constexpr int NA = Layout<NC>::NA;
    static constexpr int GS = NA <= 8 ? 8 : (NA <= 16 ? 16 : 32);
    static constexpr int G = 32 / GS;
    // column stride of the matrix in shared memory, odd: the lanes of a group store and read their
    // columns (and rows) at element strides that fall on distinct banks
    static constexpr int LD = NA | 1;
};

// Warps per block and the blocks per SM the register allocation aims at, per instantiation (the forward
// kernels' count measured; a build may set BMC_FWD_MIN_BLOCKS for a sweep).
#ifndef BMC_FWD_MIN_BLOCKS
#define BMC_FWD_MIN_BLOCKS 3
#endif
template <int NC, int NT>
struct ChainLaunch {
    static constexpr int kWarps = 4;
    static constexpr int kMinBlocks = NT == 0 ? BMC_FWD_MIN_BLOCKS : 2;
};

template <int NC, typename R, int NT>
struct DenseSlotBody {
    using D = Dn<R, NT>;
    static constexpr int NA = Layout<NC>::NA;
    StepCoef<NC, D> coef;           // the owner chain's coefficients, scaled by dt / 2^s
    D cw, cm, cc[NC > 0 ? NC : 1];  // ... and its constant column C, likewise scaled
    D mat[NA * DenseGroup<NC>::LD]; // column-major: column j at [j * LD]
    D vec[NA];                      // the owner's [M; 1]
    D out[NA];
    int s;
    int ns, m, kind, r;             // repeated blocks: the event's Taylor sub-steps and degree, its kind
                                    // (bit 0 dense, bit 1 Taylor, bit 2 spoil), the block's repeats
};

// A warp's G slots are read together (each group reads the same element of its own slot), so they are
// padded to start 128 / G bytes apart modulo the 128-byte bank row: the G addresses of such a read fall
// on different banks.
template <int NC, typename R, int NT>
struct DenseSlot : DenseSlotBody<NC, R, NT> {
    static constexpr size_t kBody = sizeof(DenseSlotBody<NC, R, NT>);
    static constexpr size_t kTarget = (128 / DenseGroup<NC>::G) % 128;
    static constexpr size_t kPad = (kTarget + 128 - kBody % 128) % 128;
    char pad[kPad == 0 ? 128 : kPad];
};

template <int NC, typename R, int NT>
struct DenseSmem {
    DenseSlot<NC, R, NT> slot[DenseGroup<NC>::G];
};

template <typename RD, typename RS, int NT>
__device__ __forceinline__ Dn<RD, NT> cvt_dn(const Dn<RS, NT>& a) {
    Dn<RD, NT> r;
    r.v = RD(a.v);
    if constexpr (NT > 0) {
#pragma unroll
        for (int t = 0; t < NT; ++t) r.d[t] = RD(a.d[t]);
    }
    return r;
}

template <int NC, typename R, int NT>
struct Dense {
    template <typename RS>
    static __device__ __forceinline__ Dn<R, NT> cvt(const Dn<RS, NT>& a) { return cvt_dn<R, RS, NT>(a); }

    using D = Dn<R, NT>;
    using C = Chain<NC, R, NT>;
    using L = Layout<NC>;
    static constexpr int N = L::N;
    static constexpr int NA = L::NA;
    using SM = DenseSmem<NC, R, NT>;

    using SL = DenseSlot<NC, R, NT>;
    static constexpr int GS = DenseGroup<NC>::GS;
    static constexpr int G = DenseGroup<NC>::G;
    static constexpr int LD = DenseGroup<NC>::LD;

    // y = X_A v + C * caug: one column of X times a column of the matrix being built
    static __device__ __forceinline__ void matvec_aug(const SL* sl, const State<NC, D>& v, R caug,
                                                      State<NC, D>& y) {
        C::template matvec<false>(sl->coef, v, y);
        if (caug != R(0)) {
            y.zw = y.zw + caug * sl->cw;
            y.zm = y.zm + caug * sl->cm;
#pragma unroll
            for (int i = 0; i < NC; ++i) y.zc[i] = y.zc[i] + caug * sl->cc[i];
        }
    }

    static __device__ __forceinline__ void unit(State<NC, D>& col, int j) {
        const D z = dconst<R, NT>(R(0));
        col.xw = z; col.yw = z; col.zw = z; col.zm = z;
#pragma unroll
        for (int i = 0; i < NC; ++i) { col.xc[i] = z; col.yc[i] = z; col.zc[i] = z; }
#pragma unroll
        for (int q = 0; q < N; ++q)
            if (q == j) C::at(col, q) = dconst<R, NT>(R(1));
    }

    // Column gl of exp(X) into `col`, X the slot's coefficients and constant column (already scaled by
    // dt / 2^s): the degree-m Horner recurrence T = I + X T / k, k = m .. 1, then s squarings through the
    // slot's matrix (column j of T T is sum_l T[:, l] T[l][j]). Every lane of the warp calls it (the
    // squarings synchronise the warp, up to the warp's largest count smax); lanes with `work` compute.
    static __device__ __forceinline__ void exp_column(SL* sl, int gl, bool work, int s, int smax, State<NC, D>& col,
                                                      const TaylorTable& tt) {
        const R caug = (gl == N) ? R(1) : R(0);
        unit(col, gl);
        if (work) {
            for (int k = tt.dense_m; k >= 1; --k) {
                State<NC, D> y;
                matvec_aug(sl, col, caug, y);
                C::scal_state(y, R(tt.inv_k[k]));
                State<NC, D> e;
                unit(e, gl);
                C::axpy_state(e, y);
                col = e;
            }
        }
        for (int q = 0; q < smax; ++q) {
            const bool sq = work && q < s;
            if (sq) {
#pragma unroll
                for (int i = 0; i < N; ++i) sl->mat[gl * LD + i] = C::at(col, i);
                sl->mat[gl * LD + N] = dconst<R, NT>(caug);
            }
            __syncwarp();
            if (sq) {
                State<NC, D> nc;
                unit(nc, -1);
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    const D w = C::at(col, l);
#pragma unroll
                    for (int i = 0; i < N; ++i) C::at(nc, i) = dfma(sl->mat[l * LD + i], w, C::at(nc, i));
                }
                if (caug != R(0)) {           // the augmented column also picks up T[:, aug]
#pragma unroll
                    for (int i = 0; i < N; ++i) C::at(nc, i) = C::at(nc, i) + sl->mat[N * LD + i];
                }
                col = nc;
            }
            __syncwarp();
        }
    }

    // Every lane whose `evolve` is set gets its state advanced by exp(X) [M; 1]. The warp takes up to
    // G of those chains at a time: chain g of a round is done by lanes g GS .. g GS + NA - 1, lane
    // g GS + j owning column j.
    template <typename CC>
    static __device__ __noinline__ void event(SM* sm, int lane, bool evolve, const StepCoef<NC, D>& sc, const CC& cst,
                                              R dt, R nu, State<NC, D>& M, const TaylorTable& tt, int* status,
                                              bool count, unsigned& wh, unsigned& ws) {
        const int grp = lane / GS, gl = lane % GS;
        unsigned need = __ballot_sync(kFull, evolve);
        while (need) {
            int my_slot = -1, grp_owner = -1;
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int c = need ? __ffs(need) - 1 : -1;
                if (need) need &= need - 1;
                if (c == lane) my_slot = g;
                if (g == grp) grp_owner = c;
            }
            bool capped = false;   // more squarings needed than the cap: this chain's state becomes NaN
            if (my_slot >= 0) {
                SL* sl = &sm->slot[my_slot];
                int s = 0;
                if (nu > R(tt.dense_theta)) s = (int)ceil(log2(double(nu) / tt.dense_theta));
                if (s > 200) {
                    s = 200;
                    capped = true;
                    atomicOr(status, 2);
                }
                StepCoef<NC, D> scs = sc;
                const R h = R(ldexp(double(dt), -s));
                C::scale_coef(scs, h);
                sl->coef = scs;
                sl->cw = dconst<R, NT>(h) * cvt(cst.cw);
                sl->cm = dconst<R, NT>(h) * cvt(cst.cm);
#pragma unroll
                for (int i = 0; i < NC; ++i) sl->cc[i] = dconst<R, NT>(h) * cvt(cst.cc[i]);
                sl->s = s;
                if (count) {
                    wh += unsigned(NA * tt.dense_m);
                    ws += unsigned(s);
                }
#pragma unroll
                for (int q = 0; q < N; ++q) sl->vec[q] = C::at(M, q);
                sl->vec[N] = dconst<R, NT>(R(1));
            }
            __syncwarp();
            SL* sl = &sm->slot[grp];
            const bool work = grp_owner >= 0 && gl < NA;
            const int s = grp_owner >= 0 ? sl->s : 0;
            const int smax = (int)__reduce_max_sync(kFull, (unsigned)s);
            State<NC, D> col;
            exp_column(sl, gl, work, s, smax, col, tt);
            // M <- T [M; 1]
            if (work) {
#pragma unroll
                for (int i = 0; i < N; ++i) sl->mat[gl * LD + i] = C::at(col, i);
            }
            __syncwarp();
            if (grp_owner >= 0 && gl < N) {
                D acc = dconst<R, NT>(R(0));
                for (int j = 0; j < NA; ++j) acc = dfma(sl->mat[j * LD + gl], sl->vec[j], acc);
                sl->out[gl] = acc;
            }
            __syncwarp();
            if (my_slot >= 0) {
#pragma unroll
                for (int q = 0; q < N; ++q)
                    C::at(M, q) = capped ? dconst<R, NT>(R(NAN)) : sm->slot[my_slot].out[q];
            }
            __syncwarp();
        }
    }

    // Propagator reuse for a repeated block of events. Every lane whose `start` is set advances its state
    // through r repeats of the L events of its own row that begin at event `first` (records
    // row[e * stride]): its group builds the block's augmented propagator P = E_L ... E_1 one event at a
    // time, lane j holding column j of P -- an event of norm above kBlockDenseNorm is exponentiated densely
    // (exp_column) and multiplied in, a shorter one acts on every column by the truncated Taylor series
    // (the degree and sub-steps of the table's tolerance), a spoiler or gradient zeroes the transverse
    // rows -- and then applies P r times to [M; 1]. Each chain uses only its own row and parameters, so
    // its result does not depend on the chains that share its warp. The work counts follow the dense
    // path's units: Horner column products, squarings (one more per dense event for the product with P)
    // and Taylor terms (every column's, plus one per application of P).
    static __device__ __noinline__ void block(SM* sm, int lane, bool start, const EvRec<R>* row, int stride,
                                              int first, int L, int r, const ChainConst<NC, D>& cc,
                                              State<NC, D>& M, const TaylorTable& tt, int* status, bool count,
                                              unsigned& wt, unsigned& wh, unsigned& ws) {
        const int grp = lane / GS, gl = lane % GS;
        const R thm = R(tt.theta[tt.m_max]);
        unsigned need = __ballot_sync(kFull, start);
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
            const int Lw = (int)__reduce_max_sync(kFull, (unsigned)(my_slot >= 0 ? L : 0));
            const int rw = (int)__reduce_max_sync(kFull, (unsigned)(my_slot >= 0 ? r : 0));
            SL* sl = &sm->slot[grp];
            const bool work = grp_owner >= 0 && gl < NA;
            const R pa = (gl == N) ? R(1) : R(0);          // P's augmented row entry in this column
            State<NC, D> P;
            unit(P, gl);
            for (int k = 0; k < Lw; ++k) {
                if (my_slot >= 0) {                          // the owner prepares its event k
                    SL* so = &sm->slot[my_slot];
                    int kind = 0;
                    if (k < L) {
                        const EvRec<R> rec = row[(size_t)(first + k) * stride];
                        if (rec.dt > R(1e-9)) {
                            D g = dconst<R, NT>(R(0));
                            if (cc.mt_on && cc.ls != 0 && rec.w1 != R(0)) {
                                const D offmt = (rec.wf - cc.dw0) - cc.dwmt;
                                g = cc.ls == 1 ? lorentzian<R, NT>(offmt, cc.t2mt)
                                               : super_lorentzian<R, NT>(offmt, cc.t2mt, cc.w0sl);
                            }
                            StepCoef<NC, D> sc;
                            C::event_coef(cc, rec, g, sc);
                            R nu = rec.dt * C::coef_norm(sc, cc);
                            if (!(nu < R(INFINITY))) {
                                atomicOr(status, 1);
                                nu = R(0);
                            }
                            R h;
                            if (nu > R(kBlockDenseNorm)) {
                                int s = (int)ceil(log2(double(nu) / tt.dense_theta));
                                if (s > 200) {
                                    s = 200;
                                    capped = true;
                                    atomicOr(status, 2);
                                }
                                so->s = s;
                                h = R(ldexp(double(rec.dt), -s));
                                kind = 1;
                                if (count) {
                                    wh += unsigned(NA * tt.dense_m);
                                    ws += unsigned(s + 1);
                                }
                            } else {
                                const int ns = nu > thm ? (int)ceil(nu / thm) : 1;
                                const R per = ns == 1 ? nu : nu / R(ns);
                                int m = 1;
                                while (m < tt.m_max && R(tt.theta[m]) < per) ++m;
                                so->s = 0;
                                so->ns = ns;
                                so->m = m;
                                h = ns == 1 ? rec.dt : rec.dt / R(ns);
                                kind = 2;
                                if (count) wt += unsigned(NA * ns * m);
                            }
                            C::scale_coef(sc, h);
                            so->coef = sc;
                            so->cw = dconst<R, NT>(h) * cc.cw;
                            so->cm = dconst<R, NT>(h) * cc.cm;
#pragma unroll
                            for (int i = 0; i < NC; ++i) so->cc[i] = dconst<R, NT>(h) * cc.cc[i];
                        }
                        const int type = (int)rec.type;
                        if (type == EV_GRADIENT || type == EV_SPOILER) kind |= 4;
                    }
                    so->kind = kind;
                }
                __syncwarp();
                const int kd = grp_owner >= 0 ? sl->kind : 0;
                const bool dense = work && (kd & 1);
                if (__any_sync(kFull, dense)) {
                    const int s = dense ? sl->s : 0;
                    const int smax = (int)__reduce_max_sync(kFull, (unsigned)s);
                    State<NC, D> T;
                    exp_column(sl, gl, dense, s, smax, T, tt);
                    if (dense) {
#pragma unroll
                        for (int i = 0; i < N; ++i) sl->mat[gl * LD + i] = C::at(T, i);
                    }
                    __syncwarp();
                    if (dense) {                             // column gl of T [P; pa]
                        State<NC, D> np;
                        unit(np, -1);
#pragma unroll
                        for (int l = 0; l < N; ++l) {
                            const D w = C::at(P, l);
#pragma unroll
                            for (int i = 0; i < N; ++i) C::at(np, i) = dfma(sl->mat[l * LD + i], w, C::at(np, i));
                        }
                        if (pa != R(0)) {
#pragma unroll
                            for (int i = 0; i < N; ++i) C::at(np, i) = C::at(np, i) + sl->mat[N * LD + i];
                        }
                        P = np;
                    }
                }
                if (work && (kd & 2)) {                      // P <- exp(X)^ns P, column by column
                    const int ns = sl->ns, m = sl->m;
                    for (int j = 0; j < ns; ++j) {
                        State<NC, D> term = P;
                        R ca = pa;
                        for (int q = 1; q <= m; ++q) {
                            State<NC, D> y;
                            matvec_aug(sl, term, ca, y);
                            C::scal_state(y, R(tt.inv_k[q]));
                            term = y;
                            ca = R(0);
                            C::axpy_state(P, term);
                        }
                    }
                }
                if (work && (kd & 4)) C::spoil(P);
                __syncwarp();
            }
            // M <- P^r [M; 1]
            if (work) {
#pragma unroll
                for (int i = 0; i < N; ++i) sl->mat[gl * LD + i] = C::at(P, i);
            }
            if (my_slot >= 0) {
                SL* so = &sm->slot[my_slot];
#pragma unroll
                for (int q = 0; q < N; ++q) so->vec[q] = C::at(M, q);
                so->vec[N] = dconst<R, NT>(R(1));
                so->r = r;
                if (count) wt += unsigned(r);
            }
            __syncwarp();
            const int rr = grp_owner >= 0 ? sl->r : 0;
            for (int q = 0; q < rw; ++q) {
                const bool app = grp_owner >= 0 && gl < N && q < rr;
                D acc = dconst<R, NT>(R(0));
                if (app) {
                    for (int j = 0; j < NA; ++j) acc = dfma(sl->mat[j * LD + gl], sl->vec[j], acc);
                }
                __syncwarp();
                if (app) sl->vec[gl] = acc;
                __syncwarp();
            }
            if (my_slot >= 0) {
#pragma unroll
                for (int q = 0; q < N; ++q)
                    C::at(M, q) = capped ? dconst<R, NT>(R(NAN)) : sm->slot[my_slot].vec[q];
            }
            __syncwarp();
        }
    }
};

// the precision of the dense path: float64 always (its squarings amplify rounding by 2^s)
template <typename R>
struct DenseReal { using type = double; };

// elementwise precision change of a struct made only of Dn<RS, NT> members (StepCoef, State)
template <typename RS, typename RD, int NT, typename A, typename B>
__device__ __forceinline__ void convert_flat(const A& a, B& b) {
    constexpr int n = sizeof(A) / sizeof(Dn<RS, NT>);
    static_assert(sizeof(B) / sizeof(Dn<RD, NT>) == n, "layouts differ");
    const Dn<RS, NT>* pa = reinterpret_cast<const Dn<RS, NT>*>(&a);
    Dn<RD, NT>* pb = reinterpret_cast<Dn<RD, NT>*>(&b);
#pragma unroll
    for (int i = 0; i < n; ++i) {
        pb[i].v = RD(pa[i].v);
        if constexpr (NT > 0) {
#pragma unroll
            for (int t = 0; t < NT; ++t) pb[i].d[t] = RD(pa[i].d[t]);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// the chain kernel
// ------------------------------------------------------------------------------------------------
// COUNT: the launch adds its work counts to a.work (the measurement entry points); the other launches
// carry no counters at all.
template <int NC, typename R, int NT, bool UNEVEN = false, bool COUNT = false>
__global__ void __launch_bounds__(32 * ChainLaunch<NC, NT>::kWarps, ChainLaunch<NC, NT>::kMinBlocks)
chain_kernel(const ChainArgs a, const __grid_constant__ TaylorTable tt) {
    using D = Dn<R, NT>;
    using C = Chain<NC, R, NT>;
    using RD = typename DenseReal<R>::type;
    using SM = DenseSmem<NC, RD, NT>;
    constexpr int N = Layout<NC>::N;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    SM* dsm = reinterpret_cast<SM*>(smem_raw) + (threadIdx.x >> 5);

    // chains in offset-fastest order: neighbouring lanes are neighbouring offsets of one voxel, so a
    // warp shares parameters and its chains need similar Taylor orders
    const long long nch = UNEVEN ? a.n_chains : (long long)a.n_vox * a.n_off;
    long long ci = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = ci < nch;
    if (!valid) ci = nch - 1;
    if (a.order) ci = a.order[ci];                     // chains sorted by estimated cost (see cost_kernel)
    int v, o;
    const EvRec<R>* __restrict__ ev = reinterpret_cast<const EvRec<R>*>(a.ev);
    int stride = a.n_off, n_ev_own = a.n_ev, n_ev_loop = a.n_ev;
    int seg_row;
    if constexpr (UNEVEN) {
        // this chain's table: its records, row stride and length; the warp runs to its longest table
        const int2 vm = a.chain_map[ci];
        v = vm.x;
        o = vm.y;
        const int t = a.vox_table[v];
        ev += a.tab_base[t];
        stride = a.tab_noff[t];
        n_ev_own = a.tab_nev[t];
        n_ev_loop = (int)__reduce_max_sync(kFull, (unsigned)n_ev_own);
        seg_row = a.tab_row0 ? a.tab_row0[t] + o : 0;
    } else {
        v = (int)(ci / a.n_off);
        o = (int)(ci % a.n_off);
        seg_row = o;
    }
    // this chain's repeated block (float64 kernels; not with a trajectory, whose every event is kept)
    int4 blk = make_int4(0, 0, 0, 0);
    if constexpr (std::is_same<R, RD>::value) {
        if (a.seg && !a.traj) blk = a.seg[seg_row];
    }
    const bool use_blk = blk.z >= 2;
    const R dswitch = R(a.dense_switch > 0.0 ? a.dense_switch : tt.dense_switch);
    const int blk_end = use_blk ? blk.x + blk.z * blk.y : 0;
    const bool act = valid && (a.active == nullptr || a.active[v] != 0);
    if (__all_sync(kFull, !act)) return;

    const size_t ch = UNEVEN ? (size_t)ci : (size_t)v * a.n_off + o;
    unsigned wk0 = 0, wk1 = 0, wk2 = 0, wk3 = 0, wk4 = 0;   // this chain's work counts (each < 2^32 per launch)
    constexpr bool count = COUNT;
    ChainConst<NC, D>& cc =
        reinterpret_cast<ChainConst<NC, D>*>(smem_raw + ChainLaunch<NC, NT>::kWarps * sizeof(SM))[threadIdx.x];
    for (int node = 0; node < a.n_nodes; ++node) {
        {
            ChainConst<NC, D> tmp;
            C::load_const(a, v, node, tmp);
            cc = tmp;
        }
        State<NC, D> M;
        C::load_m0(a, v, M);
        bool reset_pending = false;
        R gkey = R(NAN);
        // The Taylor degree of the last event: the next event's search starts there (consecutive events
        // of a chain need similar degrees), a table read or two from the constant bank.
        int m_prev = 1;
        const R thm = R(tt.theta[tt.m_max]);
        const bool mt_ls = cc.mt_on && cc.ls != 0;
        D gval = dconst<R, NT>(R(0));
        // the frequency-dependent base of the norm bound, kept while the events' frequency stays fkey
        R fkey = R(NAN);
        typename C::NormBase nb{R(0), R(0)};
        for (int e = 0; e < n_ev_loop; ++e) {
            // past the end of its own table a lane sees an empty DELAY: no evolution, spoiler or readout
            const bool in = !UNEVEN || e < n_ev_own;
            EvRec<R> rec;
            if (in) {
                rec = ev[(size_t)e * stride + o];
            } else {
                rec.dt = R(0); rec.w1 = R(0); rec.c = R(1); rec.s = R(0); rec.wf = R(0); rec.type = R(EV_DELAY);
            }
            if (reset_pending) {                                   // the ADC reset of the previous event
                C::load_m0(a, v, M);
                reset_pending = false;
            }
            // a repeated block: all its events at once at its first event, none of them afterwards
            if constexpr (std::is_same<R, RD>::value) {
                const bool bstart = use_blk && act && in && e == blk.x;
                if (__any_sync(kFull, bstart))
                    Dense<NC, R, NT>::block(dsm, lane, bstart, ev + o, stride, blk.x, blk.y, blk.z, cc, M, tt, a.status,
                                            count, wk0, wk1, wk2);
            }
            const bool skip = use_blk && e >= blk.x && e < blk_end;
            const int type = skip ? EV_DELAY : (int)rec.type;
            const bool evolve = act && !skip && rec.dt > R(1e-9);
            if (__any_sync(kFull, evolve)) {
                D g = dconst<R, NT>(R(0));
                if (mt_ls && rec.w1 != R(0)) {
                    if (rec.wf != gkey) {
                        gkey = rec.wf;
                        const D offmt = (rec.wf - cc.dw0) - cc.dwmt;
                        gval = cc.ls == 1 ? lorentzian<R, NT>(offmt, cc.t2mt)
                                          : super_lorentzian<R, NT>(offmt, cc.t2mt, cc.w0sl);
                    }
                    g = gval;
                }
                D w1x, w1y, Rm1W;
                C::rf_coef(cc, rec, g, w1x, w1y, Rm1W);
                if (rec.wf != fkey) {
                    StepCoef<NC, D> s0;
                    C::event_coef(cc, rec, g, s0);
                    nb = C::norm_base(s0, cc);
                    fkey = rec.wf;
                }
                R nu = evolve ? rec.dt * C::rf_norm(nb, w1x.v, w1y.v, Rm1W.v) : R(0);
                if (!(nu < R(INFINITY))) {                          // NaN or inf: flag, let NaN propagate
                    if (evolve) atomicOr(a.status, 1);
                    nu = R(0);
                }
                // this chain's own choice: dense scaling and squaring for a large norm, else the
                // Taylor action with the fewest terms whose tail bound meets the tolerance
                const bool dense_own = evolve && nu > dswitch;
                if (__any_sync(kFull, dense_own)) {
                    StepCoef<NC, D> sc;                            // unscaled: the dense path scales by dt / 2^s
                    C::event_coef(cc, rec, g, sc);
                    if constexpr (std::is_same<R, RD>::value) {
                        Dense<NC, R, NT>::event(dsm, lane, dense_own, sc, cc, rec.dt, nu, M, tt, a.status, count, wk1, wk2);
                    } else {
                        StepCoef<NC, Dn<RD, NT>> scd;
                        State<NC, Dn<RD, NT>> Md;
                        convert_flat<R, RD, NT>(sc, scd);
                        convert_flat<R, RD, NT>(M, Md);
                        Dense<NC, RD, NT>::event(dsm, lane, dense_own, scd, cc, RD(rec.dt), RD(nu), Md, tt, a.status,
                                                 count, wk1, wk2);
                        convert_flat<RD, R, NT>(Md, M);
                    }
                }
                const bool tay = evolve && !dense_own;
                int m_own = 0, ns_own = 0;
                if (tay) {
                    ns_own = nu > thm ? (int)ceil(nu / thm) : 1;
                    const R per = ns_own == 1 ? nu : nu / R(ns_own);
                    // the smallest degree whose theta covers `per` (theta increases with m), searched from
                    // the previous event's degree: consecutive events of a chain need similar degrees, so
                    // this takes a step or two where a search from 1 takes m
                    int m = m_prev;
                    while (m < tt.m_max && R(tt.theta[m]) < per) ++m;
                    while (m > 1 && R(tt.theta[m - 1]) >= per) --m;
                    m_prev = m;
                    m_own = m;
                }
                const int ns_w = __reduce_max_sync(kFull, (unsigned)ns_own);
                const int m_w = __reduce_max_sync(kFull, (unsigned)m_own);
                if (ns_w > 0) {
                    const R h = tay ? (ns_own == 1 ? rec.dt : rec.dt / R(ns_own)) : R(0);
                    const int passes = C::taylor_apply(cc, rec, g, h, ns_w, m_w, ns_own, m_own, M, tt);
                    if (count && tay) {
                        wk0 += unsigned(ns_own * m_own);
                        // of those, the terms formed in float32 (all of them in the float32 kernel)
                        const int k32 = std::is_same<R, float>::value ? 1 : (NT == 0 ? tt.f32_from[m_own] : m_own + 1);
                        wk4 += unsigned(ns_own * (m_own + 1 - k32));
                    }
                    if (count) wk3 += unsigned(passes * m_w);
                }
            }
            if (type == EV_GRADIENT || type == EV_SPOILER) C::spoil(M);
            if (a.traj != nullptr && act && in) {
                double* tp = a.traj + (ch * a.n_ev + e) * N;
#pragma unroll
                for (int q = 0; q < N; ++q) tp[q] = double(C::at(M, q).v);
            }
            if (type == EV_ADC && a.reset_after_adc) reset_pending = (e + 1 < n_ev_own);
        }
        // last_M of this isochromat, weighted into the spread mean (written by the chain's own thread)
        if (act) {
            const R wgt = a.n_nodes > 1 ? R(a.w[node]) : R(1);
            if (a.mz >= 0) {
                D z = dconst<R, NT>(R(0));
#pragma unroll
                for (int q = 0; q < N; ++q)
                    if (q == a.mz) z = C::at(M, q);
                a.out[ch] = (node ? a.out[ch] : 0.0) + double(wgt * z.v);
                if constexpr (NT > 0) {
                    if (a.jout) {
#pragma unroll
                        for (int t = 0; t < NT; ++t) {
                            double* jp = UNEVEN ? a.jout + (size_t)(a.t0 + t) * a.n_chains + ch
                                                : a.jout + ((size_t)(a.t0 + t) * a.n_vox + v) * a.n_off + o;
                            *jp = (node ? *jp : 0.0) + double(wgt * z.d[t]);
                        }
                    }
                }
            } else {
#pragma unroll
                for (int q = 0; q < N; ++q)
                    a.out[ch * N + q] = (node ? a.out[ch * N + q] : 0.0) + double(wgt * C::at(M, q).v);
            }
        }
    }
    if constexpr (COUNT) {
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const unsigned wq = q == 0 ? wk0 : (q == 1 ? wk1 : (q == 2 ? wk2 : (q == 3 ? wk3 : wk4)));
            unsigned long long x = act ? (unsigned long long)wq : 0ull;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(kFull, x, off);
            if (lane == 0 && x) atomicAdd(a.work + q, x);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// cost estimate of every chain: the norm of its first RF event's generator (what sets its Taylor
// order), so that chains of equal order can share a warp
// ------------------------------------------------------------------------------------------------
template <int NC, typename R, bool UNEVEN = false>
__global__ void __launch_bounds__(128) cost_kernel(const ChainArgs a, float* __restrict__ key,
                                                   int* __restrict__ idx) {
    using C = Chain<NC, R, 0>;
    using D = Dn<R, 0>;
    const long long nch = UNEVEN ? a.n_chains : (long long)a.n_vox * a.n_off;
    const long long ci = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= nch) return;
    const EvRec<R>* __restrict__ ev = reinterpret_cast<const EvRec<R>*>(a.ev);
    int v, o, stride = a.n_off, n_ev = a.n_ev;
    if constexpr (UNEVEN) {
        const int2 vm = a.chain_map[ci];
        v = vm.x;
        o = vm.y;
        const int t = a.vox_table[v];
        ev += a.tab_base[t];
        stride = a.tab_noff[t];
        n_ev = a.tab_nev[t];
    } else {
        v = (int)(ci / a.n_off);
        o = (int)(ci % a.n_off);
    }
    float cost = 0.f;
    for (int e = 0; e < n_ev; ++e) {
        const EvRec<R> rec = ev[(size_t)e * stride + o];
        if ((int)rec.type != EV_RF || !(rec.dt > R(1e-9))) continue;
        ChainConst<NC, D> cc;
        C::load_const(a, v, 0, cc);
        StepCoef<NC, D> sc;
        C::event_coef(cc, rec, dconst<R, 0>(R(0)), sc);
        cost = float(rec.dt * C::coef_norm(sc, cc));
        break;
    }
    key[ci] = cost;
    idx[ci] = (int)ci;
}

// ------------------------------------------------------------------------------------------------
// repeated blocks: for every row of a table, the run of r >= 2 identical copies of a block of
// L <= kBlockMaxL events that saves the most events, among the blocks that hold no readout, evolve the
// state, and either hold an event of at least kBlockMinDt (exponentiated densely, the work the reuse
// saves) or repeat so often (r >= kBlockMinRepeats) that the per-column work of short events pays;
// (0, 0, 0) where there is none. One thread per row.
// ------------------------------------------------------------------------------------------------
constexpr int kBlockMaxL = 8;
constexpr double kBlockMinDt = 1e-3;
constexpr int kBlockMinRepeats = 48;

template <typename R>
__device__ __forceinline__ bool same_rec(const EvRec<R>& x, const EvRec<R>& y) {
    return x.dt == y.dt && x.w1 == y.w1 && x.c == y.c && x.s == y.s && x.wf == y.wf && x.type == y.type;
}

// One thread per (row, block length): kBlockScanRows rows of kBlockMaxL threads per block. Each thread
// walks its row for its own L (the candidates at increasing start, the first largest saving kept);
// the row's first thread then takes the largest saving over L = 1 .. kBlockMaxL in that order, so ties
// go to the shortest block and then the earliest start.
constexpr int kBlockScanRows = 16;
constexpr int kBlockScanThreads = kBlockScanRows * kBlockMaxL;

template <typename R>
__global__ void __launch_bounds__(kBlockScanThreads) block_scan_kernel(const EvRec<R>* __restrict__ ev, int n_rows,
                                                                       int n_ev, int stride, int4* __restrict__ seg) {
    __shared__ long long sv[kBlockScanThreads];
    __shared__ int4 sb[kBlockScanThreads];
    const int tid = threadIdx.x;
    const int o = blockIdx.x * kBlockScanRows + tid / kBlockMaxL;
    const int L = tid % kBlockMaxL + 1;
    int4 best = make_int4(0, 0, 0, 0);
    long long best_save = 0;
    if (o < n_rows) {
        const EvRec<R>* row = ev + o;
        int a = 0;
        while (a + 2 * L <= n_ev) {
            int r = 1;
            while (a + (r + 1) * L <= n_ev) {
                bool eq = true;
                for (int j = 0; j < L && eq; ++j)
                    eq = same_rec(row[(size_t)(a + j) * stride], row[(size_t)(a + r * L + j) * stride]);
                if (!eq) break;
                ++r;
            }
            if (r < 2) {
                ++a;
                continue;
            }
            bool adc = false, moves = false, long_ev = false;
            for (int j = 0; j < L; ++j) {
                const EvRec<R> x = row[(size_t)(a + j) * stride];
                adc |= (int)x.type == EV_ADC;
                moves |= x.dt > R(1e-9);
                long_ev |= x.dt >= R(kBlockMinDt);
            }
            const long long save = (long long)(r - 1) * L;
            if (!adc && moves && (long_ev || r >= kBlockMinRepeats) && save > best_save) {
                best = make_int4(a, L, r, 0);
                best_save = save;
            }
            a += r * L;
        }
    }
    sv[tid] = best_save;
    sb[tid] = best;
    __syncthreads();
    if (o < n_rows && L == 1) {
        long long bs = 0;
        int4 bb = make_int4(0, 0, 0, 0);
        for (int l = 0; l < kBlockMaxL; ++l)
            if (sv[tid + l] > bs) {
                bs = sv[tid + l];
                bb = sb[tid + l];
            }
        seg[o] = bb;
    }
}

// ------------------------------------------------------------------------------------------------
// event preprocessing: the reference table [n_off][n_ev] -> records [n_ev][n_off]
// ------------------------------------------------------------------------------------------------
template <typename R>
__global__ void prep_events_kernel(int n_off, int n_ev, const int32_t* __restrict__ type, const double* __restrict__ dt,
                                   const double* __restrict__ amp, const double* __restrict__ phase,
                                   const double* __restrict__ freq, EvRec<R>* __restrict__ out) {
    const size_t n = (size_t)n_off * n_ev;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t o = i / n_ev, e = i % n_ev;
        EvRec<R> r;
        r.dt = R(dt[i]);
        r.w1 = R(6.283185307179586 * amp[i]);
        double s, c;
        sincos(phase[i], &s, &c);
        r.c = R(c);
        r.s = R(s);
        r.wf = R(6.283185307179586 * freq[i]);
        r.type = R(type[i]);
        out[e * n_off + o] = r;
    }
}

}  // namespace bmc
