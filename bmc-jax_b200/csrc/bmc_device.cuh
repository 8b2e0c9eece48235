// bmc_device.cuh -- device building blocks of the Bloch-McConnell propagation (sm_100a).
//
// One thread owns one chain: a (voxel, offset) pair whose state is carried through the event
// table. The system matrix A of BMC-JAX (simulation/matrix.py:83-295) is never stored: it is a
// sparse, block-structured operator determined by ~10 + 6 n_cest coefficients, and the time step
// exp([A C; 0 0] dt) [M; 1] is applied as a truncated Taylor series of matrix-vector products
// with that operator (the action of the exponential, Al-Mohy & Higham, SIAM J. Sci. Comput. 33,
// 2011), scaled into s sub-steps. Events whose exponential has a large norm (long delays, long CW
// blocks) take a dense scaling-and-squaring path (bmc_kernels.cuh, Dense) instead.
//
// Forward-mode tangents ride along as dual numbers `Dn<R, NT>`: every coefficient and every state
// entry carries NT directional derivatives, so the tangent of Z is the exact derivative of the
// computed approximation, like jax.jacfwd of the reference's expm (fitting/lm.py:39).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace bmc {

// ------------------------------------------------------------------------------------------------
// dual numbers: value plus NT directional derivatives
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void sincos_(double x, double* s, double* c) { sincos(x, s, c); }
__device__ __forceinline__ void sincos_(float x, float* s, float* c) { sincosf(x, s, c); }

template <typename R, int NT>
struct Dn {
    R v;
    R d[NT];
};
template <typename R>
struct Dn<R, 0> {
    R v;
};

template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> dconst(R a) {
    Dn<R, NT> r;
    r.v = a;
    if constexpr (NT > 0) {
#pragma unroll
        for (int t = 0; t < NT; ++t) r.d[t] = R(0);
    }
    return r;
}

#define DN_LOOP(body)                                           \
    if constexpr (NT > 0) {                                     \
        _Pragma("unroll") for (int t = 0; t < NT; ++t) { body; } \
    }

template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> operator+(Dn<R, NT> a, Dn<R, NT> b) {
    Dn<R, NT> r;
    r.v = a.v + b.v;
    DN_LOOP(r.d[t] = a.d[t] + b.d[t]);
    return r;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> operator-(Dn<R, NT> a, Dn<R, NT> b) {
    Dn<R, NT> r;
    r.v = a.v - b.v;
    DN_LOOP(r.d[t] = a.d[t] - b.d[t]);
    return r;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> operator-(Dn<R, NT> a) {
    Dn<R, NT> r;
    r.v = -a.v;
    DN_LOOP(r.d[t] = -a.d[t]);
    return r;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> operator*(Dn<R, NT> a, Dn<R, NT> b) {
    Dn<R, NT> r;
    r.v = a.v * b.v;
    DN_LOOP(r.d[t] = fma(a.v, b.d[t], a.d[t] * b.v));
    return r;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> operator*(R a, Dn<R, NT> b) {
    Dn<R, NT> r;
    r.v = a * b.v;
    DN_LOOP(r.d[t] = a * b.d[t]);
    return r;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> operator+(Dn<R, NT> a, R b) {
    Dn<R, NT> r = a;
    r.v = a.v + b;
    return r;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> operator-(Dn<R, NT> a, R b) {
    Dn<R, NT> r = a;
    r.v = a.v - b;
    return r;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> operator-(R a, Dn<R, NT> b) {
    Dn<R, NT> r;
    r.v = a - b.v;
    DN_LOOP(r.d[t] = -b.d[t]);
    return r;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> operator+(R a, Dn<R, NT> b) {
    return b + a;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> operator*(Dn<R, NT> a, R b) {
    return b * a;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> operator/(Dn<R, NT> a, Dn<R, NT> b) {
    const R inv = R(1) / b.v;
    Dn<R, NT> r;
    r.v = a.v * inv;
    DN_LOOP(r.d[t] = (a.d[t] - r.v * b.d[t]) * inv);
    return r;
}
// a*b + c with the value part as one fused multiply-add
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> dfma(Dn<R, NT> a, Dn<R, NT> b, Dn<R, NT> c) {
    Dn<R, NT> r;
    r.v = fma(a.v, b.v, c.v);
    DN_LOOP(r.d[t] = fma(a.v, b.d[t], fma(a.d[t], b.v, c.d[t])));
    return r;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> dexp(Dn<R, NT> a) {
    Dn<R, NT> r;
    r.v = exp(a.v);
    DN_LOOP(r.d[t] = r.v * a.d[t]);
    return r;
}
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> dcos(Dn<R, NT> a) {
    Dn<R, NT> r;
    R s, c;
    sincos_(a.v, &s, &c);
    r.v = c;
    DN_LOOP(r.d[t] = -s * a.d[t]);
    return r;
}
// |x| continued with the sign of the value (the derivative jax takes for abs away from 0)
template <typename R, int NT>
__device__ __forceinline__ Dn<R, NT> dabs(Dn<R, NT> a) {
    return a.v >= R(0) ? a : -a;
}

// ------------------------------------------------------------------------------------------------
// HD: a float64 value with its derivative along one direction of the inputs (a design setting that
// moves the event table, the parameters and the start state together). Used as the scalar of the dual
// numbers, Dn<HD, NT> carries a quantity, its NT parameter tangents, and the derivative of each along
// the design direction: the mixed second derivatives of forward mode over forward mode. Values are
// computed exactly as in float64 (division and square root included), so the value parts of a
// Dn<HD, NT> computation are those of the Dn<double, NT> one. Comparisons look at the value only.
// ------------------------------------------------------------------------------------------------
// the global math functions stay visible beside HD's overloads below
using ::exp;
using ::fabs;
using ::fma;
using ::fmax;
using ::fmin;
using ::sqrt;

struct HD {
    double v, e;
    HD() = default;
    __host__ __device__ constexpr HD(double x) : v(x), e(0.0) {}
    __host__ __device__ constexpr HD(double x, double dx) : v(x), e(dx) {}
};
__device__ __forceinline__ HD operator+(HD a, HD b) { return HD(a.v + b.v, a.e + b.e); }
__device__ __forceinline__ HD operator-(HD a, HD b) { return HD(a.v - b.v, a.e - b.e); }
__device__ __forceinline__ HD operator-(HD a) { return HD(-a.v, -a.e); }
__device__ __forceinline__ HD operator*(HD a, HD b) { return HD(a.v * b.v, fma(a.v, b.e, a.e * b.v)); }
__device__ __forceinline__ HD operator/(HD a, HD b) {
    const double q = a.v / b.v;
    return HD(q, (a.e - q * b.e) / b.v);
}
__device__ __forceinline__ HD& operator+=(HD& a, HD b) { return a = a + b; }
__device__ __forceinline__ HD fma(HD a, HD b, HD c) {
    return HD(fma(a.v, b.v, c.v), fma(a.v, b.e, fma(a.e, b.v, c.e)));
}
__device__ __forceinline__ HD fabs(HD a) { return a.v < 0.0 ? -a : a; }
__device__ __forceinline__ HD fmax(HD a, HD b) { return (a.v >= b.v || b.v != b.v) ? a : b; }
__device__ __forceinline__ HD fmin(HD a, HD b) { return (a.v <= b.v || b.v != b.v) ? a : b; }
__device__ __forceinline__ HD sqrt(HD a) {
    const double r = sqrt(a.v);
    return HD(r, r > 0.0 ? a.e / (2.0 * r) : 0.0);
}
__device__ __forceinline__ HD exp(HD a) {
    const double r = exp(a.v);
    return HD(r, r * a.e);
}
__device__ __forceinline__ bool operator<(HD a, HD b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(HD a, HD b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(HD a, HD b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(HD a, HD b) { return a.v >= b.v; }
__device__ __forceinline__ bool operator==(HD a, HD b) { return a.v == b.v; }
__device__ __forceinline__ bool operator!=(HD a, HD b) { return a.v != b.v; }

// element i of an input array as the scalar R: with HD, its design derivative from `dir` (null = 0)
template <typename R>
__device__ __forceinline__ R lift(const double* x, const double* dir, size_t i) {
    return R(x[i]);
}
template <>
__device__ __forceinline__ HD lift<HD>(const double* x, const double* dir, size_t i) {
    return HD(x[i], dir ? dir[i] : 0.0);
}


// ------------------------------------------------------------------------------------------------
// event records: the shared event table, preprocessed once per call (bmc_prep_events)
// ------------------------------------------------------------------------------------------------
// Event types, BMC-JAX simulation/events.py:12-18.
enum : int { EV_DELAY = 0, EV_RF = 1, EV_GRADIENT = 2, EV_ADC = 3, EV_SPOILER = 4 };

template <typename R>
struct __align__(16) EvRec {
    R dt;      // duration [s]
    R w1;      // 2 pi rf_amp [rad/s], before rel_b1
    R c, s;    // cos, sin of rf_phase
    R wf;      // 2 pi rf_freq [rad/s]
    R type;    // event type, as a number
};

// ------------------------------------------------------------------------------------------------
// per-chain constants (everything of A and C that does not change from event to event)
// ------------------------------------------------------------------------------------------------
template <int NC, typename S>
struct ChainConst {
    S Rw2, Rw1, cw;                 // water: r2 + sum k f, r1 + sum k f + k_mt f_mt, C = r1
    S k[NC > 0 ? NC : 1];           // CEST -> water exchange k
    S kwc[NC > 0 ? NC : 1];         // water -> CEST k f
    S Rc2[NC > 0 ? NC : 1];         // r2 + k
    S Rc1[NC > 0 ? NC : 1];         // r1 + k
    S cc[NC > 0 ? NC : 1];          // C = r1 f
    S offc0[NC > 0 ? NC : 1];       // CEST resonance [rad/s]
    S kmt, kwmt, Rm1, cm;           // MT: k, k f, r1 + k, C = r1 f
    S dw0;                          // B0 offset [rad/s]
    S relb1;
    S dwmt;                         // MT resonance [rad/s]
    S t2mt;                         // 1 / r2_mt
    S w0sl;                         // larmor * 1e-6: the super-Lorentzian bridge half width
    int ls;                         // 0 none, 1 Lorentzian, 2 super-Lorentzian
    bool mt_on;                     // f_mt > 1e-9 (matrix.py:203-213)
    // balancing scales d = sqrt(f) of each CEST pool and of MT (1 where f is 0), for the norm only
    double sf[NC > 0 ? NC : 1];
    double sfm;
};

// the coefficients of one event, scaled by the sub-step h
// (the constant column C is not here: it is rebuilt from ChainConst where the first term needs it)
template <int NC, typename S>
struct StepCoef {
    S Rw2, Rw1;
    S k[NC > 0 ? NC : 1], kwc[NC > 0 ? NC : 1], Rc2[NC > 0 ? NC : 1], Rc1[NC > 0 ? NC : 1];
    S offc[NC > 0 ? NC : 1];
    S offw, w1x, w1y;
    S kmt, kwmt, Rm1W;
};

template <int NC, typename V>
struct State {
    V xw, yw, zw;
    V xc[NC > 0 ? NC : 1], yc[NC > 0 ? NC : 1], zc[NC > 0 ? NC : 1];
    V zm;
};

// ------------------------------------------------------------------------------------------------
// MT lineshapes, BMC-JAX simulation/matrix.py:25-81
// ------------------------------------------------------------------------------------------------
template <typename R, int NT>
__device__ Dn<R, NT> sl_direct(Dn<R, NT> delta, Dn<R, NT> t2) {
    // sum over u = 0, 0.01, ..., 1 of sqrt(2/pi) t2/|3u^2-1| exp(-2 (delta t2/|3u^2-1|)^2), times pi du
    Dn<R, NT> acc = dconst<R, NT>(R(0));
    const Dn<R, NT> dt2 = delta * t2;
    for (int i = 0; i <= 100; ++i) {
        const R u = R(0.01) * R(i);
        R q = fabs(R(3) * u * u - R(1));
        q = q > R(1e-6) ? q : R(1e-6);
        const R iq = R(1) / q;
        const Dn<R, NT> arg = iq * dt2;
        const Dn<R, NT> e = dexp(R(-2) * (arg * arg));
        acc = acc + iq * e;
    }
    return R(0.7978845608028654 * 3.141592653589793 * 0.01) * (t2 * acc);
}

template <typename R, int NT>
__device__ Dn<R, NT> super_lorentzian(Dn<R, NT> delta, Dn<R, NT> t2, Dn<R, NT> w0) {
    if (fabs(delta.v) >= w0.v) return sl_direct<R, NT>(delta, t2);
    const Dn<R, NT> p0 = -w0 - R(300), p1 = -w0 - R(100);
    const Dn<R, NT> p2 = w0 + R(100), p3 = w0 + R(300);
    const Dn<R, NT> y0 = sl_direct<R, NT>(p0, t2), y1 = sl_direct<R, NT>(p1, t2);
    const Dn<R, NT> y2 = sl_direct<R, NT>(p2, t2), y3 = sl_direct<R, NT>(p3, t2);
    const Dn<R, NT> d0 = R(30) * (y1 - y0), d1 = R(30) * (y3 - y2);
    const Dn<R, NT> c = dabs((delta - p1 + R(1)) / (p2 - p1 + R(1)));
    const Dn<R, NT> c2 = c * c, c3 = c2 * c;
    const Dn<R, NT> h0 = R(2) * c3 - R(3) * c2 + R(1);
    const Dn<R, NT> h1 = R(3) * c2 - R(2) * c3;
    const Dn<R, NT> h2 = c3 - R(2) * c2 + c;
    const Dn<R, NT> h3 = c3 - c2;
    return h0 * y1 + h1 * y2 + h2 * d0 + h3 * d1;
}

template <typename R, int NT>
__device__ Dn<R, NT> lorentzian(Dn<R, NT> delta, Dn<R, NT> t2) {
    const Dn<R, NT> x = delta * t2;
    return t2 / (x * x + R(1));
}

}  // namespace bmc
