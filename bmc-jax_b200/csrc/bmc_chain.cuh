// bmc_chain.cuh -- the chain kernel: one thread per (voxel, offset), the whole event table.
//
// Semantics follow BMC-JAX simulation/simulate.py:22-132 exactly:
//   * an event evolves the state only if dt > 1e-9 (simulate.py:51);
//   * GRADIENT and SPOILER zero the x and y entries of water and every CEST pool (simulate.py:55-72);
//   * last_M is the state after every event; after an ADC the running state returns to M0
//     (simulate.py:105-114); the result is last_M after the final event (simulate.py:128-132).
// The time step is exp([A C; 0 0] h)^s [M; 1]; see bmc_device.cuh for how it is evaluated.
#pragma once
#include <type_traits>

#include "bmc_device.cuh"
#include "bmc_tail32.cuh"

namespace bmc {

constexpr int kMaxNodes = 64;
constexpr int kMaxT = 8;
constexpr int kTaylorMMax = 40;

// Truncated-Taylor tables, filled by the host (bmc_capi.cu) for the precision in use:
// theta[m] = the largest ||X|| for which the degree-m tail bound stays under the tolerance.
struct TaylorTable {
    double theta[kTaylorMMax + 1];
    double inv_fact[kTaylorMMax + 1];   // 1 / k!
    double inv_k[kTaylorMMax + 1];      // 1 / k
    int m_max;             // short path: degree cap
    double dense_theta;    // dense path: ||X / 2^s|| <= dense_theta ...
    int dense_m;           // ... with this Horner degree
    double dense_switch;   // warps whose largest ||X|| exceeds this take the dense path
    // float64 kernels: for a chain of Taylor degree m, the terms from f32_from[m] on are below the
    // table's float32 threshold of the state (theta[m]^k / k! <= 1e-6 for BMC_F64, 0.3 for BMC_MIXED)
    // and are formed in float32 (> m: none)
    int f32_from[kTaylorMMax + 1];
    float inv_fact_f[kTaylorMMax + 1];  // 1 / k! in float32
};

struct ChainArgs {
    int n_vox, n_off, n_ev, n_fields;
    int mz;                    // state index written; < 0: whole state
    int reset_after_adc;
    int n_nodes;               // spread isochromats (1 = none)
    double u[kMaxNodes], w[kMaxNodes];
    const double* params;      // [n_fields][n_vox]
    const double* params_dir;  // [n_fields][n_vox] or null: the design direction of params (design kernel)
    const void* ev;            // EvRec<R>[n_ev][n_off]
    const double* m0;          // [n_vox][N]
    const double* sigma;       // [n_vox] spread width [Hz] or null
    // tangents handled by this launch: global tangent indices t0 .. t0 + NT - 1
    int t0;
    int field_row[kMaxT];
    const double* seed;        // [P][n_vox]
    const double* dm0;         // [P][n_vox][N] or null
    const int* active;         // [n_vox] or null: voxels with 0 are skipped
    const int* order;          // [n_vox * n_off] or null: the chain each thread takes, in launch order
    double* out;               // [n_vox][n_off] (mz >= 0) or [n_vox][n_off][N]
    double* jout;              // [P][n_vox][n_off] or null
    double* traj;              // [n_vox][n_off][n_ev][N] or null: the state after every event
    int* status;               // error flags (bit 0: non-finite norm)
    unsigned long long* work;  // null, or [5]: useful Taylor terms, dense Horner column products,
                               // dense squarings, Taylor terms executed (warp maximum), and of the
                               // useful Taylor terms those formed in float32
    // uneven batches (chain_kernel<..., true>): every voxel has its own event table
    long long n_chains;        // chains of the launch (canonical order: voxel-major, then row)
    const int2* chain_map;     // [n_chains]: (voxel, row of its table)
    const int* vox_table;      // [n_vox]: table of each voxel
    const long long* tab_base; // [n_tables]: first record of each table in `ev`
    const int* tab_noff;       // [n_tables]: rows (records per event) of each table
    const int* tab_nev;        // [n_tables]: events of each table
    // repeated blocks (propagator reuse): per row (a, L, r, 0), the r copies of the L events from event a
    // on are applied as one propagator; r < 2: none. Uniform tables: row o; uneven: tab_row0[t] + o.
    const int4* seg;           // null: no reuse
    const int* tab_row0;       // [n_tables]: first row of each table in `seg` (uneven batches)
    double dense_switch;       // > 0: the norm above which an event takes the dense path (else the table's)
};

template <int NC>
struct Layout {
    static constexpr int N = 3 * NC + 4;        // state size, reference layout
    static constexpr int NA = N + 1;            // augmented
    static constexpr int NF = 13 + 5 * NC;      // params rows
    // params rows (SimParams order, CEST fields expanded)
    static constexpr int WR1 = 0, WR2 = 1, WF = 2, CK = 3, CF = 3 + NC, CDW = 3 + 2 * NC, CR1 = 3 + 3 * NC,
                         CR2 = 3 + 4 * NC, MK = 3 + 5 * NC, MF = MK + 1, MDW = MK + 2, MR1 = MK + 3, MR2 = MK + 4,
                         MLS = MK + 5, B0 = MK + 6, GAM = MK + 7, B0I = MK + 8, RB1 = MK + 9;
    // reference state indices
    static constexpr int ixw = 0, iyw = NC + 1, izw = 2 * (NC + 1), izm = 3 * (NC + 1);
    static __device__ __forceinline__ int ixc(int i) { return 1 + i; }
    static __device__ __forceinline__ int iyc(int i) { return NC + 2 + i; }
    static __device__ __forceinline__ int izc(int i) { return 2 * NC + 3 + i; }
};

template <int NC, typename R, int NT>
struct Chain {
    using D = Dn<R, NT>;
    using L = Layout<NC>;
    static constexpr int N = L::N;
    static constexpr int NA = L::NA;

    // ---------------------------------------------------------------------------------------------
    // parameters -> per-chain constants (matrix.py:99-173), with tangents seeded per field row
    // ---------------------------------------------------------------------------------------------
    // tangents t0 .. t0 + NT - 1 of the launch's set (a.t0 in the chain kernel; the adjoint kernel seeds
    // one tangent per lane)
    static __device__ __forceinline__ D field(const ChainArgs& a, int row, int v, int t0) {
        D r = dconst<R, NT>(lift<R>(a.params, a.params_dir, (size_t)row * a.n_vox + v));
        if constexpr (NT > 0) {
#pragma unroll
            for (int t = 0; t < NT; ++t)
                if (a.field_row[t0 + t] == row) r.d[t] = R(a.seed[(size_t)(t0 + t) * a.n_vox + v]);
        }
        return r;
    }

    static __device__ void load_const(const ChainArgs& a, int v, int node, ChainConst<NC, D>& cc) {
        load_const(a, v, node, cc, a.t0);
    }

    static __device__ void load_const(const ChainArgs& a, int v, int node, ChainConst<NC, D>& cc, int t0) {
        const D r1w = field(a, L::WR1, v, t0), r2w = field(a, L::WR2, v, t0);
        const D b0 = field(a, L::B0, v, t0), gam = field(a, L::GAM, v, t0);
        D b0i = field(a, L::B0I, v, t0);
        const D larmor = R(1e6) * (gam * b0);
        if (a.n_nodes > 1 || a.sigma) {
            // isochromat `node`: b0_inhom + sigma u / (gamma b0 / 2 pi)   (spread.py:101-104)
            D sig = dconst<R, NT>(a.sigma ? R(a.sigma[v]) : R(0));
            if constexpr (NT > 0) {
#pragma unroll
                for (int t = 0; t < NT; ++t)
                    if (a.field_row[t0 + t] == -2) sig.d[t] = R(a.seed[(size_t)(t0 + t) * a.n_vox + v]);
            }
            const D hzpp = R(1.0 / 6.283185307179586) * (gam * b0);
            b0i = b0i + (R(a.u[node]) * sig) / hzpp;
        }
        cc.dw0 = R(1e-6) * (larmor * b0i);
        D ksum = dconst<R, NT>(R(0));
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            const D k = field(a, L::CK + i, v, t0), f = field(a, L::CF + i, v, t0);
            const D r1 = field(a, L::CR1 + i, v, t0), r2 = field(a, L::CR2 + i, v, t0);
            const D dw = field(a, L::CDW + i, v, t0);
            cc.k[i] = k;
            cc.kwc[i] = k * f;
            ksum = ksum + cc.kwc[i];
            cc.Rc2[i] = r2 + k;
            cc.Rc1[i] = r1 + k;
            cc.cc[i] = r1 * f;
            cc.offc0[i] = R(1e-6) * (dw * larmor);
        }
        const D kmt = field(a, L::MK, v, t0), fmt = field(a, L::MF, v, t0), r1mt = field(a, L::MR1, v, t0);
        const D r2mt = field(a, L::MR2, v, t0), dwmt = field(a, L::MDW, v, t0);
        cc.kmt = kmt;
        cc.kwmt = kmt * fmt;
        cc.Rm1 = r1mt + kmt;
        cc.cm = r1mt * fmt;
        cc.Rw2 = r2w + ksum;
        cc.Rw1 = (r1w + ksum) + cc.kwmt;
        cc.cw = r1w;
        cc.relb1 = field(a, L::RB1, v, t0);
        cc.dwmt = R(1e-6) * (dwmt * larmor);
        cc.t2mt = dconst<R, NT>(R(1)) / r2mt;
        cc.w0sl = R(1e-6) * larmor;
        int ls = (int)a.params[(size_t)L::MLS * a.n_vox + v];
        cc.ls = ls < 0 ? 0 : (ls > 2 ? 2 : ls);
        cc.mt_on = fmt.v > R(1e-9);
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            const double f = a.params[(size_t)(L::CF + i) * a.n_vox + v];
            cc.sf[i] = f > 1e-30 ? sqrt(f) : 1.0;
        }
        const double fm = a.params[(size_t)L::MF * a.n_vox + v];
        cc.sfm = fm > 1e-30 ? sqrt(fm) : 1.0;
    }

    // ---------------------------------------------------------------------------------------------
    // one event's coefficients (unscaled) and the infinity norm of its generator times dt
    // ---------------------------------------------------------------------------------------------
    static __device__ __forceinline__ void event_coef(const ChainConst<NC, D>& cc, const EvRec<R>& e, D g_mt,
                                                      StepCoef<NC, D>& sc) {
        const D offw = e.wf - cc.dw0;                                  // matrix.py:162
        const D w1 = e.w1 * cc.relb1;                                  // matrix.py:121
        sc.offw = offw;
        sc.w1x = e.c * w1;
        sc.w1y = e.s * w1;
        sc.Rw2 = cc.Rw2;
        sc.Rw1 = cc.Rw1;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            sc.k[i] = cc.k[i];
            sc.kwc[i] = cc.kwc[i];
            sc.Rc2[i] = cc.Rc2[i];
            sc.Rc1[i] = cc.Rc1[i];
            sc.offc[i] = cc.offc0[i] - offw;                           // matrix.py:166
        }
        sc.kmt = cc.kmt;
        sc.kwmt = cc.kwmt;
        sc.Rm1W = cc.Rm1 + (w1 * w1) * g_mt;                           // matrix.py:210, 283
    }

    // sqrt(a^2 + b^2) <= max + (sqrt(2) - 1) min, within 8.3%
    static __device__ __forceinline__ R hyp(R a, R b) { return fmax(a, b) + R(0.41421357) * fmin(a, b); }
    // sqrt(a^2 + b^2), rounded; the callers scale their result by (1 + kNormSlack) to keep a bound
    static __device__ __forceinline__ R blk(R a, R b) { return sqrt(fma(a, a, b * b)); }
    static constexpr double kNormSlack = std::is_same<R, float>::value ? 1e-6 : 1e-14;

    // An upper bound of ||D^-1 A D|| in the norm max_b ||v_b||_2 / d_b over blocks b = (x, y) pairs and
    // z entries, with d = sqrt(f) per pool. The similarity balances the exchange terms (detailed
    // balance: k f one way, k the other, so k sqrt(f) both ways) and each precession-relaxation block
    // counts sqrt(R^2 + w^2) instead of R + w (exactly in the part a chain keeps across events, through
    // the bound `hyp` for the RF term, which changes every event). Being an induced norm, it bounds
    // ||X^k|| and so the Taylor tail; the truncation error of water's entries stays below tol times
    // max(|M_w|, |M_c| / sqrt(f_c), 1).
    //
    // Every water and CEST row carries the RF term w1 once, so the bound is max(rows + w1, mt): `rows`
    // (those rows without w1) and the MT row's constant depend on the event's frequency, not on its RF
    // amplitude or phase, and a chain keeps them while its frequency stays the same (`NormBase`).
    struct NormBase {
        R rows;   // max over the water and CEST rows of their w1-free sums
        R mt_c;   // the MT row without |R1 + k + w1^2 g|
    };

    static __device__ __forceinline__ NormBase norm_base(const StepCoef<NC, D>& s, const ChainConst<NC, D>& cc) {
        // the constant column C enters through the augmented row: |C_i| / d_i
        R ex = R(0);
#pragma unroll
        for (int i = 0; i < NC; ++i) ex += fabs(s.k[i].v) * R(cc.sf[i]);
        const R km = fabs(s.kmt.v) * R(cc.sfm);
        R m = blk(s.Rw2.v, s.offw.v) + ex;
        m = fmax(m, fabs(s.Rw1.v) + ex + km + fabs(R(cc.cw.v)));
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            const R b = fabs(s.k[i].v) * R(cc.sf[i]);
            m = fmax(m, blk(s.Rc2[i].v, s.offc[i].v) + b);
            m = fmax(m, fabs(s.Rc1[i].v) + b + fabs(R(cc.cc[i].v)) / R(cc.sf[i]));
        }
        return {m * R(1 + kNormSlack), (km + fabs(R(cc.cm.v)) / R(cc.sfm)) * R(1 + kNormSlack)};
    }

    static __device__ __forceinline__ R rf_norm(const NormBase& b, R w1x, R w1y, R Rm1W) {
        return fmax(b.rows + hyp(fabs(w1x), fabs(w1y)), fabs(Rm1W) + b.mt_c);
    }

    static __device__ __forceinline__ R coef_norm(const StepCoef<NC, D>& s, const ChainConst<NC, D>& cc) {
        return rf_norm(norm_base(s, cc), s.w1x.v, s.w1y.v, s.Rm1W.v);
    }

    // the RF entries of an event's coefficients, unscaled, computed as event_coef computes them
    static __device__ __forceinline__ void rf_coef(const ChainConst<NC, D>& cc, const EvRec<R>& e, D g_mt, D& w1x,
                                                   D& w1y, D& Rm1W) {
        const D w1 = e.w1 * cc.relb1;
        w1x = e.c * w1;
        w1y = e.s * w1;
        Rm1W = cc.Rm1 + (w1 * w1) * g_mt;
    }

    static __device__ __forceinline__ void scale_coef(StepCoef<NC, D>& s, R h) {
        s.Rw2 = h * s.Rw2; s.Rw1 = h * s.Rw1;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            s.k[i] = h * s.k[i]; s.kwc[i] = h * s.kwc[i]; s.Rc2[i] = h * s.Rc2[i];
            s.Rc1[i] = h * s.Rc1[i]; s.offc[i] = h * s.offc[i];
        }
        s.offw = h * s.offw; s.w1x = h * s.w1x; s.w1y = h * s.w1y;
        s.kmt = h * s.kmt; s.kwmt = h * s.kwmt; s.Rm1W = h * s.Rm1W;
    }

    // y = X v (+ C h when WithC): the sparse Bloch-McConnell operator (matrix.py:238-293)
    template <bool WithC>
    static __device__ __forceinline__ void matvec(const StepCoef<NC, D>& s, const State<NC, D>& v, State<NC, D>& y,
                                                  const ChainConst<NC, D>* cst = nullptr, R h = R(0)) {
        // water rows: own terms and the pools' exchange terms in two partial sums (shorter dependency
        // chains), pool rows: four terms each
        D xw = dfma(s.offw, v.yw, -(s.Rw2 * v.xw));
        xw = xw - s.w1y * v.zw;
        D yw = dfma(s.w1x, v.zw, -(s.Rw2 * v.yw));
        yw = yw - s.offw * v.xw;
        D zw = dfma(s.w1y, v.xw, -(s.Rw1 * v.zw));
        zw = zw - s.w1x * v.yw;
        D zm = dfma(s.kwmt, v.zw, -(s.Rm1W * v.zm));
        if constexpr (WithC) {                     // the constant column C h, rebuilt here: it is needed
            zw = dfma(cst->cw, dconst<R, NT>(h), zw);   // by the first term of a sub-step only
            zm = dfma(cst->cm, dconst<R, NT>(h), zm);
        }
        D px = dconst<R, NT>(R(0)), py = px, pz = s.kmt * v.zm;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            px = dfma(s.k[i], v.xc[i], px);
            py = dfma(s.k[i], v.yc[i], py);
            pz = dfma(s.k[i], v.zc[i], pz);
            D xc = dfma(s.kwc[i], v.xw, -(s.Rc2[i] * v.xc[i]));
            xc = xc - s.offc[i] * v.yc[i];
            xc = xc - s.w1y * v.zc[i];
            D yc = dfma(s.kwc[i], v.yw, -(s.Rc2[i] * v.yc[i]));
            yc = dfma(s.offc[i], v.xc[i], yc);
            yc = dfma(s.w1x, v.zc[i], yc);
            D zc = dfma(s.kwc[i], v.zw, -(s.Rc1[i] * v.zc[i]));
            zc = dfma(s.w1y, v.xc[i], zc);
            zc = zc - s.w1x * v.yc[i];
            if constexpr (WithC) zc = dfma(cst->cc[i], dconst<R, NT>(h), zc);
            y.xc[i] = xc;
            y.yc[i] = yc;
            y.zc[i] = zc;
        }
        y.xw = xw + px;
        y.yw = yw + py;
        y.zw = zw + pz;
        y.zm = zm;
    }

    static __device__ __forceinline__ void axpy_state(State<NC, D>& acc, const State<NC, D>& t) {
        acc.xw = acc.xw + t.xw; acc.yw = acc.yw + t.yw; acc.zw = acc.zw + t.zw; acc.zm = acc.zm + t.zm;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            acc.xc[i] = acc.xc[i] + t.xc[i]; acc.yc[i] = acc.yc[i] + t.yc[i]; acc.zc[i] = acc.zc[i] + t.zc[i];
        }
    }
    static __device__ __forceinline__ void scal_state(State<NC, D>& t, R a) {
        t.xw = a * t.xw; t.yw = a * t.yw; t.zw = a * t.zw; t.zm = a * t.zm;
#pragma unroll
        for (int i = 0; i < NC; ++i) { t.xc[i] = a * t.xc[i]; t.yc[i] = a * t.yc[i]; t.zc[i] = a * t.zc[i]; }
    }

    // acc += a * t, entry by entry
    static __device__ __forceinline__ void fma_state(State<NC, D>& acc, R a, const State<NC, D>& t) {
        acc.xw = dfma(dconst<R, NT>(a), t.xw, acc.xw); acc.yw = dfma(dconst<R, NT>(a), t.yw, acc.yw);
        acc.zw = dfma(dconst<R, NT>(a), t.zw, acc.zw); acc.zm = dfma(dconst<R, NT>(a), t.zm, acc.zm);
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            acc.xc[i] = dfma(dconst<R, NT>(a), t.xc[i], acc.xc[i]);
            acc.yc[i] = dfma(dconst<R, NT>(a), t.yc[i], acc.yc[i]);
            acc.zc[i] = dfma(dconst<R, NT>(a), t.zc[i], acc.zc[i]);
        }
    }

    // exp(X)^s [M; 1] by s sub-steps of the degree-m Taylor polynomial, X = [A C; 0 0] h: the
    // unnormalised powers p_k = X^k [M; 1] are accumulated with weights 1/k!, so each term is one sparse
    // operator product and one fused multiply-add per state entry. The coefficients (scaled by h) are
    // formed at each sub-step, so that they are not held in registers across the rest of the event.
    // The loops run to the warp's largest (s, m); each chain uses only its own (ns_own, m_own), so a
    // chain's result never depends on which chains share its warp.
    //
    // In the float64 kernel without tangents, the terms of a chain from tt.f32_from[m_own] on (each below
    // 1e-6 of the state, in the balanced norm of coef_norm) are formed in float32 and summed in a float32
    // accumulator that is added to M once per sub-step: their rounding, a few units of 2^-24 of terms
    // below 1e-6, is at most ~2e-13 of the state per event, the order of the truncation tolerance.
    // The switch point is the chain's own: where the lanes of a warp disagree on it, the sub-step runs
    // once per distinct switch point, each lane adding its terms only in its own pass (weight 0 in the
    // others), so the result stays independent of the chains that share the warp. Cost-sorted warps
    // almost always agree (one pass). Returns the number of passes over all sub-steps.
    static __device__ __forceinline__ int taylor_apply(const ChainConst<NC, D>& cst, const EvRec<R>& rec, D g_mt,
                                                       R h, int ns_w, int m_w, int ns_own, int m_own,
                                                       State<NC, D>& M, const TaylorTable& tt) {
        constexpr bool kMixed = std::is_same<R, double>::value && NT == 0;
        // The terms are added to M as they are formed (later terms derive from `term`, not from M), so no
        // separate accumulator is held; a lane past its own sub-steps or degree adds with weight 0.
        // fma(1, t, M) rounds like M + t and fma(0, t, M) is M: the result is that of summing apart.
        int passes = 0;
#pragma unroll 1
        for (int j = 0; j < ns_w; ++j) {
            const bool on = j < ns_own;
            // this lane's switch point (0: no sub-step of its own here); lanes still to be served
            const int k32_own = on ? (kMixed ? tt.f32_from[m_own] : m_w + 1) : 0;
            unsigned pend = __ballot_sync(0xffffffffu, k32_own != 0);
#pragma unroll 1
            do {
                const int k32 = __shfl_sync(0xffffffffu, k32_own, __ffs(pend) - 1);
                const bool member = k32_own == k32;
                pend &= ~__ballot_sync(0xffffffffu, member);
                ++passes;
                const int m_on = member ? m_own : 0;
                StepCoef<NC, D> s;
                event_coef(cst, rec, g_mt, s);
                scale_coef(s, h);
                State<NC, D> term;
                matvec<true>(s, M, term, &cst, h);
                fma_state(M, member ? R(1) : R(0), term);
                int k = 2;
#pragma unroll 1
                for (; k <= m_w && k < k32; ++k) {
                    State<NC, D> nt;
                    matvec<false>(s, term, nt);
                    term = nt;
                    fma_state(M, k <= m_on ? R(tt.inv_fact[k]) : R(0), term);
                }
                if constexpr (kMixed) {
                    if (k <= m_w) {
                        // paired float32 instructions over the CEST pools (bmc_tail32.cuh)
                        using T32 = Tail32<NC>;
                        typename T32::Coef s32;
                        typename T32::St t32, a32;
                        T32::coef(s, s32);
                        T32::state(term, t32);
                        T32::zero(a32);
#pragma unroll 1
                        for (; k <= m_w; ++k) {
                            typename T32::St n32;
                            T32::matvec(s32, t32, n32);
                            t32 = n32;
                            T32::fma_acc(a32, k <= m_on ? tt.inv_fact_f[k] : 0.f, t32);
                        }
                        T32::add_to(M, a32);
                    }
                }
            } while (pend);
        }
        return passes;
    }

    // elementwise precision changes between structs made only of Dn<., 0> members (StepCoef, State)
    template <typename A, typename B>
    static __device__ __forceinline__ void to_float(const A& a, B& b) {
        constexpr int n = sizeof(A) / sizeof(double);
        static_assert(sizeof(B) == n * sizeof(float), "layouts differ");
        const double* pa = reinterpret_cast<const double*>(&a);
        float* pb = reinterpret_cast<float*>(&b);
#pragma unroll
        for (int i = 0; i < n; ++i) pb[i] = float(pa[i]);
    }
    template <typename B>
    static __device__ __forceinline__ void zero_state(B& b) {
        constexpr int n = sizeof(B) / sizeof(float);
        float* pb = reinterpret_cast<float*>(&b);
#pragma unroll
        for (int i = 0; i < n; ++i) pb[i] = 0.f;
    }
    template <typename B>
    static __device__ __forceinline__ void add_float(State<NC, D>& M, const B& a) {
        constexpr int n = sizeof(B) / sizeof(float);
        static_assert(sizeof(State<NC, D>) == n * sizeof(double), "layouts differ");
        double* pm = reinterpret_cast<double*>(&M);
        const float* pa = reinterpret_cast<const float*>(&a);
#pragma unroll
        for (int i = 0; i < n; ++i) pm[i] = pm[i] + double(pa[i]);
    }

    static __device__ __forceinline__ void spoil(State<NC, D>& M) {
        const D z = dconst<R, NT>(R(0));
        M.xw = z; M.yw = z;
#pragma unroll
        for (int i = 0; i < NC; ++i) { M.xc[i] = z; M.yc[i] = z; }
    }

    static __device__ __forceinline__ D& at(State<NC, D>& M, int ref_index) {
        // reference index -> member (used only outside hot loops)
        if (ref_index == L::ixw) return M.xw;
        if (ref_index == L::iyw) return M.yw;
        if (ref_index == L::izw) return M.zw;
        if (ref_index == L::izm) return M.zm;
        if (ref_index <= NC) return M.xc[ref_index - 1];
        if (ref_index <= 2 * NC + 1) return M.yc[ref_index - NC - 2];
        return M.zc[ref_index - 2 * NC - 3];
    }

    static __device__ void load_m0(const ChainArgs& a, int v, State<NC, D>& M) {
        const double* m0 = a.m0 + (size_t)v * N;
#pragma unroll
        for (int q = 0; q < N; ++q) {
            D x = dconst<R, NT>(R(m0[q]));
            if constexpr (NT > 0) {
                if (a.dm0) {
#pragma unroll
                    for (int t = 0; t < NT; ++t) x.d[t] = R(a.dm0[((size_t)(a.t0 + t) * a.n_vox + v) * N + q]);
                }
            }
            at(M, q) = x;
        }
    }
};

}  // namespace bmc
