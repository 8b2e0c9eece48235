// bmc_design.cuh -- second-order tangents for protocol design: Z, its parameter tangents, and the
// derivative of both along one design direction, in one pass per chain.
//
// BMC-JAX optimises a protocol by differentiating the Cramer-Rao bound with respect to the design
// vector through jax.jacfwd of the model (design/optimize.py:43-113, design/crlb.py): a derivative of
// the Jacobian. Here every scalar of the chain is an HD (value and design derivative, bmc_device.cuh)
// and every state entry a Dn<HD, NT>, so one pass gives z, dz/dx_t, dz/dd and d^2 z/(dx_t dd) as exact
// derivatives of the computed approximation. The inputs move along the design direction together:
// the event table (dt, rf_amp, rf_phase, rf_freq, per unit of the setting), the parameters and the start
// state.
//
// One thread per chain, in launch order (the problems are small: a few truths times the rows of a
// protocol). An event evolves by the chain kernel's truncated-Taylor action (Chain::taylor_apply, warp
// synchronous) or, where its norm is above the dense threshold (long CW blocks), by a scaling and
// squaring that the thread does alone: the columns of exp(X h) by Taylor polynomials, s squarings, one
// product with [M; 1]. Its matrices live in a global scratch, entry-major with the chains adjacent.
#pragma once
#include "bmc_chain.cuh"

namespace bmc {

struct DesignArgs {
    const EvRec<double>* ev_dir;   // [n_ev][n_off]: d(dt), d(w1), d(cos phase), d(sin phase), d(wf) per unit
    const double* m0_dir;          // [n_vox][N] or null
    double* dz;                    // [n_vox][n_off]
    double* djz;                   // [P][n_vox][n_off]
    double* scratch;               // 2 N^2 + N Dn<HD, 1> per chain, entry-major: Phi, Phi^2, psi
};

// the design direction of an event table as records: [n_ev][n_off] from the reference layout [n_off][n_ev]
// (d(dt), 2 pi d(rf_amp), -sin(phase) d(phase), cos(phase) d(phase), 2 pi d(rf_freq)); null arrays are 0
__global__ void prep_dir_kernel(int n_off, int n_ev, const double* __restrict__ phase, const double* __restrict__ ddt,
                                const double* __restrict__ damp, const double* __restrict__ dphase,
                                const double* __restrict__ dfreq, EvRec<double>* __restrict__ out) {
    const size_t n = (size_t)n_off * n_ev;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t o = i / n_ev, e = i % n_ev;
        double s, c;
        sincos(phase[i], &s, &c);
        const double dp = dphase ? dphase[i] : 0.0;
        EvRec<double> r;
        r.dt = ddt ? ddt[i] : 0.0;
        r.w1 = damp ? 6.283185307179586 * damp[i] : 0.0;
        r.c = -s * dp;
        r.s = c * dp;
        r.wf = dfreq ? 6.283185307179586 * dfreq[i] : 0.0;
        r.type = 0.0;
        out[e * n_off + o] = r;
    }
}

template <int NC, int NT>
struct DesignChain {
    using D = Dn<HD, NT>;
    using C = Chain<NC, HD, NT>;
    using St = State<NC, D>;
    static constexpr int N = Layout<NC>::N;
    // entry i of a state in the reference's order (x of water and of each CEST pool, then y, then z, MT z last)
    static __device__ __forceinline__ D& el(St& s, int i) { return C::at(s, i); }

    // entry e of one of the chain's matrices: [e][chain]
    struct Mat {
        D* base;
        long long stride;
        __device__ __forceinline__ D& operator[](int e) const { return base[(long long)e * stride]; }
    };

    // M <- exp(X dt) [M; 1] = [Phi psi; 0 1]^(2^s) [M; 1], X h with h = dt / 2^s of norm <= dense_theta
    // (not inlined: its frame and the Taylor path's then share the thread's stack)
    static __device__ __noinline__ void dense_event(const ChainConst<NC, D>& cc, const EvRec<HD>& rec, D g, HD nu, St& M,
                                       const TaylorTable& tt, Mat phi, Mat phi2, Mat psi) {
        int s = 0;
        if (nu.v > tt.dense_theta) s = (int)ceil(log2(nu.v / tt.dense_theta));
        if (s > 200) s = 200;
        const HD h = rec.dt * HD(ldexp(1.0, -s));
        StepCoef<NC, D> sc;
        C::event_coef(cc, rec, g, sc);
        C::scale_coef(sc, h);
        const D zero = dconst<HD, NT>(HD(0.0));
        // column j < N of Phi = exp(A h), and psi = the first N entries of exp(X h) [0; 1]
        for (int j = 0; j <= N; ++j) {
            St term, acc, nt;
            for (int i = 0; i < N; ++i) el(term, i) = zero;
            if (j < N) {
                el(term, j) = dconst<HD, NT>(HD(1.0));
                acc = term;
                C::template matvec<false>(sc, term, nt);
            } else {
                for (int i = 0; i < N; ++i) el(acc, i) = zero;
                C::template matvec<true>(sc, term, nt, &cc, h);        // X [0; 1] = [C h; 0]
            }
            term = nt;
            C::axpy_state(acc, term);
            for (int k = 2; k <= tt.dense_m; ++k) {
                C::template matvec<false>(sc, term, nt);
                term = nt;
                C::scal_state(term, HD(tt.inv_k[k]));
                C::axpy_state(acc, term);
            }
            for (int i = 0; i < N; ++i) {
                if (j < N) phi[i * N + j] = el(acc, i);
                else psi[i] = el(acc, i);
            }
        }
        // [Phi psi; 0 1]^2 = [Phi^2, Phi psi + psi; 0 1]
        for (int q = 0; q < s; ++q) {
            D t[N];
            for (int i = 0; i < N; ++i) t[i] = psi[i];
            for (int i = 0; i < N; ++i) {
                D a = t[i];
                for (int k = 0; k < N; ++k) a = dfma(phi[i * N + k], t[k], a);
                psi[i] = a;
            }
            for (int i = 0; i < N; ++i) {
                for (int j = 0; j < N; ++j) {
                    D a = zero;
                    for (int k = 0; k < N; ++k) a = dfma(phi[i * N + k], phi[k * N + j], a);
                    phi2[i * N + j] = a;
                }
            }
            const Mat x = phi;
            phi = phi2;
            phi2 = x;
        }
        D old[N];
        for (int i = 0; i < N; ++i) old[i] = el(M, i);
        for (int i = 0; i < N; ++i) {
            D a = psi[i];
            for (int k = 0; k < N; ++k) a = dfma(phi[i * N + k], old[k], a);
            el(M, i) = a;
        }
    }

    // the event's norm bound (its value only) and the MT saturation g (not inlined, for the stack)
    static __device__ __noinline__ double event_norm(const ChainConst<NC, D>& cc, const EvRec<HD>& rec, bool mt_ls,
                                                     D& g) {
        g = dconst<HD, NT>(HD(0.0));
        if (mt_ls && rec.w1.v != 0.0) {
            const D offmt = (rec.wf - cc.dw0) - cc.dwmt;
            g = cc.ls == 1 ? lorentzian<HD, NT>(offmt, cc.t2mt) : super_lorentzian<HD, NT>(offmt, cc.t2mt, cc.w0sl);
        }
        StepCoef<NC, D> s0;
        C::event_coef(cc, rec, g, s0);
        return (rec.dt * C::coef_norm(s0, cc)).v;
    }

    static __device__ void load_m0(const ChainArgs& a, const DesignArgs& d, int v, St& M) {
#pragma unroll
        for (int q = 0; q < N; ++q) C::at(M, q) = dconst<HD, NT>(lift<HD>(a.m0, d.m0_dir, (size_t)v * N + q));
    }
};

// One thread per chain (voxel-major in launch order); tangents a.t0 .. a.t0 + NT - 1 of the set.
template <int NC, int NT>
__global__ void __launch_bounds__(128) design_kernel(const ChainArgs a, const DesignArgs d,
                                                     const TaylorTable* __restrict__ ttab) {
    using DC = DesignChain<NC, NT>;
    using D = Dn<HD, NT>;
    using C = Chain<NC, HD, NT>;
    constexpr int N = Layout<NC>::N;
    const TaylorTable& tt = *ttab;
    const long long nch = (long long)a.n_vox * a.n_off;
    long long ci = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = ci < nch;
    if (!valid) ci = nch - 1;
    if (__all_sync(kFull, !valid)) return;
    const int v = (int)(ci / a.n_off), o = (int)(ci % a.n_off);
    const EvRec<double>* __restrict__ ev = reinterpret_cast<const EvRec<double>*>(a.ev);
    const long long per = (long long)N * N;
    typename DC::Mat phi{reinterpret_cast<D*>(d.scratch) + ci, nch};
    typename DC::Mat phi2{phi.base + per * nch, nch};
    typename DC::Mat psi{phi2.base + per * nch, nch};

    ChainConst<NC, D> cc;
    C::load_const(a, v, 0, cc);
    State<NC, D> M;
    DC::load_m0(a, d, v, M);
    bool reset_pending = false;
    const bool mt_ls = cc.mt_on && cc.ls != 0;
    const HD thm = HD(tt.theta[tt.m_max]);
    for (int e = 0; e < a.n_ev; ++e) {
        const size_t ri = (size_t)e * a.n_off + o;
        const EvRec<double> b = ev[ri];
        const EvRec<double> db = d.ev_dir ? d.ev_dir[ri] : EvRec<double>{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        EvRec<HD> rec;
        rec.dt = HD(b.dt, db.dt);
        rec.w1 = HD(b.w1, db.w1);
        rec.c = HD(b.c, db.c);
        rec.s = HD(b.s, db.s);
        rec.wf = HD(b.wf, db.wf);
        rec.type = HD(b.type);
        if (reset_pending) {
            DC::load_m0(a, d, v, M);
            reset_pending = false;
        }
        const int type = (int)b.type;
        const bool evolve = valid && b.dt > 1e-9;
        if (__any_sync(kFull, evolve)) {
            D g;
            HD nu = HD(DC::event_norm(cc, rec, mt_ls, g));
            if (!evolve) nu = HD(0.0);
            if (!(nu.v < INFINITY)) {
                if (evolve) atomicOr(a.status, 1);
                nu = HD(0.0);
            }
            const bool dense = evolve && nu.v > tt.dense_switch;
            if (dense) DC::dense_event(cc, rec, g, nu, M, tt, phi, phi2, psi);
            const bool tay = evolve && !dense;
            int m_own = 0, ns_own = 0;
            if (tay) {
                ns_own = nu.v > thm.v ? (int)ceil(nu.v / thm.v) : 1;
                const double pr = ns_own == 1 ? nu.v : nu.v / ns_own;
                int m = 1;
                while (m < tt.m_max && tt.theta[m] < pr) ++m;
                m_own = m;
            }
            const int ns_w = __reduce_max_sync(kFull, (unsigned)ns_own);
            const int m_w = __reduce_max_sync(kFull, (unsigned)m_own);
            if (ns_w > 0) {
                const HD h = tay ? (ns_own == 1 ? rec.dt : rec.dt / HD(double(ns_own))) : HD(0.0);
                C::taylor_apply(cc, rec, g, h, ns_w, m_w, ns_own, m_own, M, tt);
            }
        }
        if (type == EV_GRADIENT || type == EV_SPOILER) C::spoil(M);
        if (type == EV_ADC && a.reset_after_adc) reset_pending = (e + 1 < a.n_ev);
    }
    if (!valid) return;
    D z = dconst<HD, NT>(HD(0.0));
#pragma unroll
    for (int q = 0; q < N; ++q)
        if (q == a.mz) z = C::at(M, q);
    const size_t ch = (size_t)v * a.n_off + o;
    if (a.t0 == 0) {
        a.out[ch] = z.v.v;
        d.dz[ch] = z.v.e;
    }
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const size_t jo = ((size_t)(a.t0 + t) * a.n_vox + v) * a.n_off + o;
        a.jout[jo] = z.d[t].v;
        d.djz[jo] = z.d[t].e;
    }
}

}  // namespace bmc
