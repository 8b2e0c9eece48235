// bmc_tail32.cuh -- the float32 Taylor tail with paired FMAs (sm_100 fma.rn.f32x2).
//
// In the float64 and mixed kernels the later Taylor terms of a sub-step are formed in float32 (they are
// small against the state) and summed in a float32 accumulator. Those terms are most of the kernel's
// instructions, so they use B200's paired float32 instructions: the CEST pools go in pairs (pool 2p in
// .x, pool 2p + 1 in .y), and every term of their rows is elementwise over the pair -- the water entries
// enter as broadcast pairs -- so one __ffma2_rn does the work of two fmaf. The water rows sum their pool
// contributions pairwise and add the two halves. Each half of a paired instruction rounds as fmaf does;
// only the order of some sums differs from a scalar evaluation.
#pragma once
#include "bmc_device.cuh"

namespace bmc {

template <int NC>
struct Tail32 {
    static constexpr int NP = NC / 2;          // pool pairs
    static constexpr bool ODD = (NC & 1) != 0; // the last pool, unpaired
    static constexpr int NPA = NP > 0 ? NP : 1;

    // one sub-step's scaled coefficients; the minus signs of the operator folded in
    struct Coef {
        float2 k[NPA], kwc[NPA], nRc2[NPA], nRc1[NPA], offc[NPA], noffc[NPA];
        float ko, kwco, nRc2o, nRc1o, offco;
        float nRw2, nRw1, offw, noffw, w1x, w1y, nw1x, nw1y, kmt, kwmt, nRm1W;
        float2 w1x2, w1y2, nw1x2, nw1y2;
    };
    // a term or the accumulator
    struct St {
        float xw, yw, zw, zm;
        float2 xc[NPA], yc[NPA], zc[NPA];
        float xco, yco, zco;
    };

    static __device__ __forceinline__ float2 pair(float a, float b) { return make_float2(a, b); }
    static __device__ __forceinline__ float2 bcast(float a) { return make_float2(a, a); }

    // the float64 scaled coefficients rounded to float32 (each entry rounded once)
    template <typename K>
    static __device__ __forceinline__ void coef(const K& s, Coef& c) {
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int a = 2 * p, b = 2 * p + 1;
            c.k[p] = pair(float(s.k[a].v), float(s.k[b].v));
            c.kwc[p] = pair(float(s.kwc[a].v), float(s.kwc[b].v));
            c.nRc2[p] = pair(-float(s.Rc2[a].v), -float(s.Rc2[b].v));
            c.nRc1[p] = pair(-float(s.Rc1[a].v), -float(s.Rc1[b].v));
            c.offc[p] = pair(float(s.offc[a].v), float(s.offc[b].v));
            c.noffc[p] = pair(-float(s.offc[a].v), -float(s.offc[b].v));
        }
        if constexpr (ODD) {
            c.ko = float(s.k[NC - 1].v);
            c.kwco = float(s.kwc[NC - 1].v);
            c.nRc2o = -float(s.Rc2[NC - 1].v);
            c.nRc1o = -float(s.Rc1[NC - 1].v);
            c.offco = float(s.offc[NC - 1].v);
        }
        c.nRw2 = -float(s.Rw2.v);
        c.nRw1 = -float(s.Rw1.v);
        c.offw = float(s.offw.v);
        c.noffw = -c.offw;
        c.w1x = float(s.w1x.v);
        c.w1y = float(s.w1y.v);
        c.nw1x = -c.w1x;
        c.nw1y = -c.w1y;
        c.kmt = float(s.kmt.v);
        c.kwmt = float(s.kwmt.v);
        c.nRm1W = -float(s.Rm1W.v);
        c.w1x2 = bcast(c.w1x);
        c.w1y2 = bcast(c.w1y);
        c.nw1x2 = bcast(c.nw1x);
        c.nw1y2 = bcast(c.nw1y);
    }

    // a float64 state (State<NC, Dn<double, 0>>) rounded to float32
    template <typename S64>
    static __device__ __forceinline__ void state(const S64& t, St& f) {
        f.xw = float(t.xw.v);
        f.yw = float(t.yw.v);
        f.zw = float(t.zw.v);
        f.zm = float(t.zm.v);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            f.xc[p] = pair(float(t.xc[2 * p].v), float(t.xc[2 * p + 1].v));
            f.yc[p] = pair(float(t.yc[2 * p].v), float(t.yc[2 * p + 1].v));
            f.zc[p] = pair(float(t.zc[2 * p].v), float(t.zc[2 * p + 1].v));
        }
        if constexpr (ODD) {
            f.xco = float(t.xc[NC - 1].v);
            f.yco = float(t.yc[NC - 1].v);
            f.zco = float(t.zc[NC - 1].v);
        }
    }

    static __device__ __forceinline__ void zero(St& f) {
        f.xw = f.yw = f.zw = f.zm = 0.f;
#pragma unroll
        for (int p = 0; p < NP; ++p) f.xc[p] = f.yc[p] = f.zc[p] = bcast(0.f);
        if constexpr (ODD) f.xco = f.yco = f.zco = 0.f;
    }

    // y = X v: the sparse Bloch-McConnell operator (the scalar kernel's matvec, rows regrouped)
    static __device__ __forceinline__ void matvec(const Coef& c, const St& v, St& y) {
        const float2 XW = bcast(v.xw), YW = bcast(v.yw), ZW = bcast(v.zw);
        float2 sx = bcast(0.f), sy = bcast(0.f), sz = bcast(0.f);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const float2 xc = v.xc[p], yc = v.yc[p], zc = v.zc[p];
            // xc' = kwc xw - Rc2 xc - offc yc - w1y zc;  yc' = kwc yw - Rc2 yc + offc xc + w1x zc;
            // zc' = kwc zw - Rc1 zc + w1y xc - w1x yc
            y.xc[p] = __ffma2_rn(c.kwc[p], XW, __ffma2_rn(c.nRc2[p], xc, __ffma2_rn(c.noffc[p], yc, __fmul2_rn(c.nw1y2, zc))));
            y.yc[p] = __ffma2_rn(c.kwc[p], YW, __ffma2_rn(c.nRc2[p], yc, __ffma2_rn(c.offc[p], xc, __fmul2_rn(c.w1x2, zc))));
            y.zc[p] = __ffma2_rn(c.kwc[p], ZW, __ffma2_rn(c.nRc1[p], zc, __ffma2_rn(c.w1y2, xc, __fmul2_rn(c.nw1x2, yc))));
            // the water rows' exchange terms, pairwise
            sx = __ffma2_rn(c.k[p], xc, sx);
            sy = __ffma2_rn(c.k[p], yc, sy);
            sz = __ffma2_rn(c.k[p], zc, sz);
        }
        float ex = sx.x + sx.y, ey = sy.x + sy.y, ez = sz.x + sz.y;
        if constexpr (ODD) {
            const float xc = v.xco, yc = v.yco, zc = v.zco;
            y.xco = fmaf(c.kwco, v.xw, fmaf(c.nRc2o, xc, fmaf(-c.offco, yc, c.nw1y * zc)));
            y.yco = fmaf(c.kwco, v.yw, fmaf(c.nRc2o, yc, fmaf(c.offco, xc, c.w1x * zc)));
            y.zco = fmaf(c.kwco, v.zw, fmaf(c.nRc1o, zc, fmaf(c.w1y, xc, c.nw1x * yc)));
            ex = fmaf(c.ko, xc, ex);
            ey = fmaf(c.ko, yc, ey);
            ez = fmaf(c.ko, zc, ez);
        }
        // xw' = offw yw - Rw2 xw - w1y zw + sum k xc;  yw' = w1x zw - Rw2 yw - offw xw + sum k yc;
        // zw' = w1y xw - Rw1 zw - w1x yw + kmt zm + sum k zc;  zm' = kwmt zw - Rm1W zm
        y.xw = fmaf(c.offw, v.yw, fmaf(c.nRw2, v.xw, fmaf(c.nw1y, v.zw, ex)));
        y.yw = fmaf(c.w1x, v.zw, fmaf(c.nRw2, v.yw, fmaf(c.noffw, v.xw, ey)));
        y.zw = fmaf(c.w1y, v.xw, fmaf(c.nRw1, v.zw, fmaf(c.nw1x, v.yw, fmaf(c.kmt, v.zm, ez))));
        y.zm = fmaf(c.kwmt, v.zw, c.nRm1W * v.zm);
    }

    // a += w t
    static __device__ __forceinline__ void fma_acc(St& a, float w, const St& t) {
        const float2 W = bcast(w);
        a.xw = fmaf(w, t.xw, a.xw);
        a.yw = fmaf(w, t.yw, a.yw);
        a.zw = fmaf(w, t.zw, a.zw);
        a.zm = fmaf(w, t.zm, a.zm);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            a.xc[p] = __ffma2_rn(W, t.xc[p], a.xc[p]);
            a.yc[p] = __ffma2_rn(W, t.yc[p], a.yc[p]);
            a.zc[p] = __ffma2_rn(W, t.zc[p], a.zc[p]);
        }
        if constexpr (ODD) {
            a.xco = fmaf(w, t.xco, a.xco);
            a.yco = fmaf(w, t.yco, a.yco);
            a.zco = fmaf(w, t.zco, a.zco);
        }
    }

    // M += a, in float64
    template <typename S64>
    static __device__ __forceinline__ void add_to(S64& M, const St& a) {
        M.xw.v += double(a.xw);
        M.yw.v += double(a.yw);
        M.zw.v += double(a.zw);
        M.zm.v += double(a.zm);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            M.xc[2 * p].v += double(a.xc[p].x);
            M.xc[2 * p + 1].v += double(a.xc[p].y);
            M.yc[2 * p].v += double(a.yc[p].x);
            M.yc[2 * p + 1].v += double(a.yc[p].y);
            M.zc[2 * p].v += double(a.zc[p].x);
            M.zc[2 * p + 1].v += double(a.zc[p].y);
        }
        if constexpr (ODD) {
            M.xc[NC - 1].v += double(a.xco);
            M.yc[NC - 1].v += double(a.yco);
            M.zc[NC - 1].v += double(a.zco);
        }
    }
};

}  // namespace bmc
