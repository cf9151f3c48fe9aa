// Device arithmetic of the recurrence runner: df64 double-words, complex numbers, the four
// kernel kinds, the executors of ops 2-11 and the external wavefunctions of op 12.
//
// Every operation follows the reference runner's arithmetic in its order of evaluation
// (runner/recurrence_runner.cu:70-542, legend convert/CONVENTIONS.md:52-98) so that, built with
// -fmad=false, the f64 kind reproduces the reference's f64 kernel bit for bit. The formulas are
// those of the legend; the evaluation order (left to right, complex products as
// (ac - bd, ad + bc)) is what fixes the bits.
#pragma once
#include <stdint.h>

namespace pacuda {

// ---- df64 (Joldes, Muller, Popescu, ACM TOMS 44(2) 2017: Alg. 6, 12, 17) --------------------
struct D {
    float hi, lo;
};
__device__ __forceinline__ D dmake(float h, float l) { D z; z.hi = h; z.lo = l; return z; }

__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    s = __fadd_rn(a, b);
    float bv = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bv)), __fsub_rn(b, bv));
}
__device__ __forceinline__ void fast_two_sum(float a, float b, float &s, float &e) {
    s = __fadd_rn(a, b);
    e = __fsub_rn(b, __fsub_rn(s, a));
}
__device__ __forceinline__ D operator+(D x, D y) {
    float sh, sl, th, tl, vh, vl;
    two_sum(x.hi, y.hi, sh, sl);
    two_sum(x.lo, y.lo, th, tl);
    fast_two_sum(sh, __fadd_rn(sl, th), vh, vl);
    D z;
    fast_two_sum(vh, __fadd_rn(tl, vl), z.hi, z.lo);
    return z;
}
__device__ __forceinline__ D operator-(D x) { return dmake(-x.hi, -x.lo); }
__device__ __forceinline__ D operator-(D x, D y) { return x + (-y); }
__device__ __forceinline__ D operator*(D x, D y) {
    float ch = __fmul_rn(x.hi, y.hi);
    float cl1 = __fmaf_rn(x.hi, y.hi, -ch);
    float tl0 = __fmul_rn(x.lo, y.lo);
    float tl1 = __fmaf_rn(x.hi, y.lo, tl0);
    float cl2 = __fmaf_rn(x.lo, y.hi, tl1);
    D z;
    fast_two_sum(ch, __fadd_rn(cl1, cl2), z.hi, z.lo);
    return z;
}
__device__ __forceinline__ D operator/(D x, D y) {
    float th = __fdiv_rn(x.hi, y.hi);
    float rh = __fmul_rn(y.hi, th);
    float rl1 = __fmaf_rn(y.hi, th, -rh);
    float rl3 = __fmaf_rn(y.lo, th, rl1);
    float r_hi, r_lo;
    fast_two_sum(rh, rl3, r_hi, r_lo);
    float pi_h = __fsub_rn(x.hi, r_hi);
    float delta = __fadd_rn(pi_h, __fsub_rn(x.lo, r_lo));
    D z;
    fast_two_sum(th, __fdiv_rn(delta, y.hi), z.hi, z.lo);
    return z;
}

template <class T> struct is_f64 {
    static constexpr bool value = false;
};
template <> struct is_f64<double> {
    static constexpr bool value = true;
};

// formula constants (0, +-1, 2): exact in every type
template <class R> __device__ __forceinline__ R konst(double x);
template <> __device__ __forceinline__ double konst<double>(double x) { return x; }
template <> __device__ __forceinline__ float konst<float>(double x) { return (float)x; }
template <> __device__ __forceinline__ D konst<D>(double x) { return dmake((float)x, 0.0f); }

// f64 into a kind's layout (the reference's upload conversions)
template <class R> __device__ __forceinline__ R narrow(double x);
template <> __device__ __forceinline__ double narrow<double>(double x) { return x; }
template <> __device__ __forceinline__ float narrow<float>(double x) { return __double2float_rn(x); }
template <> __device__ __forceinline__ D narrow<D>(double x) {
    float hi = __double2float_rn(x);
    return dmake(hi, __double2float_rn(x - (double)hi));
}
// a kind's value as f64 (the reference's download conversions: hi + lo in double)
__device__ __forceinline__ double widen64(double x) { return x; }
__device__ __forceinline__ double widen64(float x) { return (double)x; }
__device__ __forceinline__ double widen64(D x) { return (double)x.hi + (double)x.lo; }

// ---- complex --------------------------------------------------------------------------------
template <class R> struct Cx {
    R re, im;
};
template <class R> __device__ __forceinline__ Cx<R> cx(R re, R im) { Cx<R> c; c.re = re; c.im = im; return c; }
template <class R> __device__ __forceinline__ Cx<R> operator+(Cx<R> a, Cx<R> b) { return cx(a.re + b.re, a.im + b.im); }
template <class R> __device__ __forceinline__ Cx<R> operator-(Cx<R> a, Cx<R> b) { return cx(a.re - b.re, a.im - b.im); }
template <class R> __device__ __forceinline__ Cx<R> operator-(Cx<R> a) { return cx(-a.re, -a.im); }
template <class R> __device__ __forceinline__ Cx<R> operator*(Cx<R> a, Cx<R> b) {
    return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <class R> __device__ __forceinline__ Cx<R> times_i(Cx<R> a) { return cx(-a.im, a.re); }
template <class R> __device__ __forceinline__ Cx<R> scaled(Cx<R> a, R s) { return cx(a.re * s, a.im * s); }

// ---- kinds: values R, denominators Den, amplitudes Amp; constants C (f64 or df64 pairs) -------
// (reference: recurrence_runner.cu:178-223)
template <class R_, class Den_, class Amp_, class Const_> struct Kind {
    typedef R_ R;
    typedef Den_ Den;
    typedef Amp_ Amp;
    typedef Const_ Const;
};
typedef Kind<double, double, double, double> KindF64;
typedef Kind<D, D, D, D> KindDF64;
typedef Kind<float, D, D, D> KindMixed;
typedef Kind<float, double, D, D> KindMixed64;

// a stored constant as R: a float reads the high word of a df64 pair
__device__ __forceinline__ double as_real(double s, double *) { return s; }
__device__ __forceinline__ D as_real(D s, D *) { return s; }
__device__ __forceinline__ float as_real(D s, float *) { return s.hi; }
template <class R, class S> __device__ __forceinline__ R cast(S s) { return as_real(s, (R *)nullptr); }
// a form component as R, for numerators
__device__ __forceinline__ double form_real(double q, double *) { return q; }
__device__ __forceinline__ D form_real(D q, D *) { return q; }
__device__ __forceinline__ float form_real(double q, float *) { return __double2float_rn(q); }
__device__ __forceinline__ float form_real(D q, float *) { return q.hi; }
template <class R, class Den> __device__ __forceinline__ R form_as(Den q) { return form_real(q, (R *)nullptr); }
// a denominator value as R (rounded once for the f32 kinds)
__device__ __forceinline__ double den_real(double x, double *) { return x; }
__device__ __forceinline__ D den_real(D x, D *) { return x; }
__device__ __forceinline__ float den_real(double x, float *) { return __double2float_rn(x); }
__device__ __forceinline__ float den_real(D x, float *) { return __fadd_rn(x.hi, x.lo); }
// an R value into the amplitude accumulator
__device__ __forceinline__ D amp_of(float x, D *) { return dmake(x, 0.0f); }
__device__ __forceinline__ D amp_of(D x, D *) { return x; }
__device__ __forceinline__ double amp_of(double x, double *) { return x; }

// ---- executors (recurrence_runner.cu:225-330; CONVENTIONS.md:71-92) ---------------------------
template <class R> __device__ __forceinline__ Cx<R> mdot(const Cx<R> *l, const Cx<R> *r) {
    return ((l[0] * r[0] - l[1] * r[1]) - l[2] * r[2]) - l[3] * r[3];
}
template <class R> __device__ __forceinline__ Cx<R> mdot_real(const Cx<R> *l, const R *q) {
    return ((scaled(l[0], q[0]) - scaled(l[1], q[1])) - scaled(l[2], q[2])) - scaled(l[3], q[3]);
}

template <int OP> struct Shape {
    static constexpr int c0 = OP == 4 ? 6 : (OP == 5 || OP == 6) ? 4 : 2;
    static constexpr int c1 = 4;
    static constexpr int cd = (OP == 4 || OP == 6) ? 4 : OP == 5 ? 6 : 2;
};

// o = the contribution's value before the scale (weyl_vector_a/b, tensor_vector, vector_wedge,
// three_vector)
template <int OP, class R>
__device__ __forceinline__ void contribution(const Cx<R> *l, const Cx<R> *r, const R *u, const R *v, Cx<R> *o) {
    if (OP == 2) {
        o[0] = ((-times_i(l[0] * r[3]) - times_i(l[1] * r[1])) + l[1] * r[2]) + times_i(l[0] * r[0]);
        o[1] = ((-(l[0] * r[2]) - times_i(l[0] * r[1])) + times_i(l[1] * r[0])) + times_i(l[1] * r[3]);
    } else if (OP == 3) {
        o[0] = ((-(l[1] * r[2]) + times_i(l[0] * r[0])) + times_i(l[0] * r[3])) + times_i(l[1] * r[1]);
        o[1] = ((-times_i(l[1] * r[3]) + l[0] * r[2]) + times_i(l[0] * r[1])) + times_i(l[1] * r[0]);
    } else if (OP == 4) {
        o[0] = (l[0] * r[1] + l[1] * r[2]) + l[2] * r[3];
        o[1] = (l[0] * r[0] + l[3] * r[2]) + l[4] * r[3];
        o[2] = (l[1] * r[0] - l[3] * r[1]) + l[5] * r[3];
        o[3] = (l[2] * r[0] - l[4] * r[1]) - l[5] * r[2];
    } else if (OP == 5) {
        o[0] = l[0] * r[1] - l[1] * r[0];
        o[1] = l[0] * r[2] - l[2] * r[0];
        o[2] = l[0] * r[3] - l[3] * r[0];
        o[3] = l[1] * r[2] - l[2] * r[1];
        o[4] = l[1] * r[3] - l[3] * r[1];
        o[5] = l[2] * r[3] - l[3] * r[2];
    } else {
        Cx<R> lr = mdot(l, r), lv = mdot_real(l, v), ru = mdot_real(r, u);
#pragma unroll
        for (int k = 0; k < 4; k++)
            o[k] = scaled(lr, u[k] - v[k]) + scaled(lv * r[k] - ru * l[k], konst<R>(2.0));
    }
}

// ops 7-9: the propagator applied to c (2 or 4 components) into o
template <int OP, class R>
__device__ __forceinline__ void propagator(const Cx<R> *c, const R *p, R reciprocal, Cx<R> f, Cx<R> *o) {
    if (OP == 9) {
        Cx<R> s = scaled(f * cx(konst<R>(0.0), konst<R>(-1.0)), reciprocal);
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = c[k] * s;
        return;
    }
    Cx<R> s = scaled(f, reciprocal), a, b;
    if (OP == 7) {
        a = ((-times_i(scaled(c[0], p[3])) - times_i(scaled(c[1], p[1]))) + scaled(c[1], p[2])) + times_i(scaled(c[0], p[0]));
        b = ((-scaled(c[0], p[2]) - times_i(scaled(c[0], p[1]))) + times_i(scaled(c[1], p[0]))) + times_i(scaled(c[1], p[3]));
    } else {
        a = ((-scaled(c[1], p[2]) + times_i(scaled(c[0], p[0]))) + times_i(scaled(c[0], p[3]))) + times_i(scaled(c[1], p[1]));
        b = ((-times_i(scaled(c[1], p[3])) + scaled(c[0], p[2])) + times_i(scaled(c[0], p[1]))) + times_i(scaled(c[1], p[0]));
    }
    o[0] = a * s;
    o[1] = b * s;
}

// op 10: factor x value
template <class R> __device__ __forceinline__ Cx<R> times_factor(R fr, R fi, Cx<R> v) {
    return cx(fr * v.re - fi * v.im, fr * v.im + fi * v.re);
}

// op 11, one component: (l r)(component factor x row factor)
template <class R>
__device__ __forceinline__ Cx<R> closure_term(Cx<R> l, Cx<R> r, R cr, R ci, R fr, R fi) {
    R sr = cr * fr - ci * fi, si = cr * fi + ci * fr;
    R pr = l.re * r.re - l.im * r.im, pi = l.re * r.im + l.im * r.re;
    return cx(pr * sr - pi * si, pr * si + pi * sr);
}

// ---- external wavefunctions, f64 (recurrence_runner.cu:337-542; CONVENTIONS.md:52-61) ---------
typedef Cx<double> W;
__device__ __forceinline__ W w64(double re, double im) { return cx(re, im); }

// the massless Weyl pair (s, b) of a particle (anti = false) or antiparticle, for either energy
// sign; `s == 0` selects the collinear form of b
__device__ __forceinline__ void weyl_pair(const double *m, int h, bool anti, W &a, W &b) {
    double e = m[0], px = m[1], py = m[2], pz = m[3];
    if (e > 0.0) {
        double s = (px == 0.0 && py == 0.0 && pz < 0.0) ? 0.0 : sqrt(fmax(e + pz, 0.0));
        if (anti && !(px == 0.0 && py == 0.0 && pz < 0.0)) s = -s;
        a = w64(s, 0.0);
        if (s == 0.0) b = w64(-(double)h * sqrt(2.0 * e), 0.0);
        else b = anti ? w64(-(double)h * px / s, py / s) : w64((double)h * px / s, -py / s);
        return;
    }
    double s = (px == 0.0 && py == 0.0 && pz > 0.0) ? 0.0 : sqrt(fmax(-(e + pz), 0.0));
    if (!anti && !(px == 0.0 && py == 0.0 && pz > 0.0)) s = -s;
    a = w64(s, 0.0);
    if (s == 0.0) b = w64(-(double)h * sqrt(2.0 * fabs(e)), 0.0);
    else b = anti ? w64((double)h * (-px) / s, -py / s) : w64(-(double)h * (-px) / s, py / s);
}

__device__ __forceinline__ void weyl_source(const double *m, int h, int ch, bool anti, W *o) {
    W a, b;
    weyl_pair(m, h, anti, a, b);
    bool pos = m[0] > 0.0;
    W z = w64(0.0, 0.0);
    // (h, ch) combinations that keep the spinor nonzero, and its component order
    bool first = pos ? (h == 1 && ch == 1) : (h == -1 && ch == 1);
    bool second = pos ? (h == -1 && ch == -1) : (h == 1 && ch == -1);
    if (!first && !second) { o[0] = z; o[1] = z; return; }
    bool ab = anti ? second : first;  // the particle's first case and the antiparticle's second are (a, b)
    if (ab) { o[0] = a; o[1] = b; } else { o[0] = b; o[1] = a; }
}

__device__ __forceinline__ void dirac_massless(const double *m, int h, bool anti, W *o) {
    W a, b, z = w64(0.0, 0.0);
    weyl_pair(m, h, anti, a, b);
    bool pos = m[0] > 0.0;
    if (!anti) {
        if (pos ? h == 1 : -h == 1) { o[0] = a; o[1] = b; o[2] = z; o[3] = z; }
        else { o[0] = z; o[1] = z; o[2] = b; o[3] = a; }
    } else {
        if (pos ? -h == 1 : h == 1) { o[0] = z; o[1] = z; o[2] = a; o[3] = b; }
        else { o[0] = b; o[1] = a; o[2] = z; o[3] = z; }
    }
}

static __device__ __noinline__ void dirac_source(const double *m, int h, double mass, bool anti, W *o) {
    if (fabs(mass) < 1.0e-8) { dirac_massless(m, h, anti, o); return; }
    double e = m[0], px = m[1], py = m[2], pz = m[3];
    int n = anti ? (e > 0.0 ? -1 : 1) : (e > 0.0 ? 1 : -1);
    int nh = n * h;
    double k = fabs(sqrt(px * px + py * py + pz * pz));
    double om1 = sqrt(fabs(e) + k);
    double om[2] = {om1, mass / om1};
    double f1 = (double)(1 + n + (1 - n) * nh) * 0.5;
    double f2 = (double)(1 + n - (1 - n) * nh) * 0.5;
    int ip = (3 + nh) / 2 - 1, im = (3 - nh) / 2 - 1;
    double g[2] = {f1 * om[ip], f2 * om[im]};
    double tx = e > 0.0 ? px : -px, ty = e > 0.0 ? py : -py, tz = e > 0.0 ? pz : -pz;
    double r = fmax(k + tz, 0.0);
    W chi[2];
    chi[0] = k == 0.0 ? w64(1.0, 0.0) : w64(sqrt(r * 0.5 / k), 0.0);
    if (r == 0.0 || k == 0.0) chi[1] = w64(-(double)nh, 0.0);
    else {
        double den = sqrt(2.0 * k * r);
        chi[1] = w64((double)nh * tx / den, (anti ? ty : -ty) / den);
    }
    double first = anti ? g[0] : g[1], second = anti ? g[1] : g[0];
    o[0] = w64(chi[im].re * first, chi[im].im * first);
    o[1] = w64(chi[ip].re * first, chi[ip].im * first);
    o[2] = w64(chi[im].re * second, chi[im].im * second);
    o[3] = w64(chi[ip].re * second, chi[ip].im * second);
}

__device__ __forceinline__ double sign_of(double value, double source) { return copysign(fabs(value), source); }

static __device__ __noinline__ void gluon_source(const double *m, int h, W *o) {
    double e = m[0], px = m[1], py = m[2], pz = m[3];
    double sqh = sqrt(0.5);
    bool pos = e > 0.0;
    double hel = pos ? (double)h : (double)(-h), pp = pos ? e : -e;
    double pt = sqrt(px * px + py * py);
    W w3 = w64(hel * pt / pp * sqh, 0.0), w1, w2;
    if (pt != 0.0) {
        if (pos) {
            double pzpt = pz / (pp * pt) * sqh * hel;
            w1 = w64(-px * pzpt, -py / pt * sqh);
            w2 = w64(-py * pzpt, px / pt * sqh);
        } else {
            double pzpt = -pz / (pp * pt) * sqh * hel;
            w1 = w64(px * pzpt, py / pt * sqh);
            w2 = w64(py * pzpt, -px / pt * sqh);
        }
    } else {
        w1 = w64(-hel * sqh, 0.0);
        w2 = w64(0.0, pos ? sign_of(sqh, pz) : -sign_of(sqh, pz));
    }
    o[0] = w64(0.0, 0.0); o[1] = w1; o[2] = w2; o[3] = w3;
}

static __device__ __noinline__ void massive_vector_source(const double *m0, int h, double mass, W *o) {
    double m[4] = {m0[0], m0[1], m0[2], m0[3]};
    if (m[0] < 0.0) {
        for (int k = 0; k < 4; k++) m[k] = -m[k];
        h = -h;
    }
    double e = m[0], px = m[1], py = m[2], pz = m[3];
    double sqh = sqrt(0.5), hel = (double)h, nsv = (double)abs(h);
    double pt2 = px * px + py * py;
    double pp = fmin(e, sqrt(pt2 + pz * pz));
    double pt = fmin(pp, sqrt(pt2));
    double hel0 = 1.0 - fabs(hel);
    if (pp == 0.0) {
        o[0] = w64(0.0, 0.0); o[1] = w64(-hel * sqh, 0.0); o[2] = w64(0.0, nsv * sqh); o[3] = w64(hel0, 0.0);
        return;
    }
    double emp = e / (mass * pp);
    W w0 = w64(hel0 * pp / mass, 0.0);
    W w3 = w64(hel0 * pz * emp + hel * pt / pp * sqh, 0.0);
    W w1, w2;
    if (pt != 0.0) {
        double pzpt = pz / (pp * pt) * sqh * hel;
        w1 = w64(hel0 * px * emp - px * pzpt, -nsv * py / pt * sqh);
        w2 = w64(hel0 * py * emp - py * pzpt, nsv * px / pt * sqh);
    } else {
        w1 = w64(-hel * sqh, 0.0);
        w2 = w64(0.0, nsv * sign_of(sqh, pz));
    }
    o[0] = w0; o[1] = w1; o[2] = w2; o[3] = w3;
}

// the wavefunction of a 10-bit template code (family | orientation << 3 | (h + 2) << 5 |
// (ch + 1) << 8); returns its component count
__device__ __forceinline__ int source_values(uint32_t code, double mass, const double *p, W *o) {
    int family = code & 7, orientation = (code >> 3) & 3;
    int h = (int)((code >> 5) & 7) - 2, ch = (int)((code >> 8) & 3) - 1;
    if (family == 0) { o[0] = w64(1.0, 0.0); return 1; }
    if (family == 1) { weyl_source(p, h, ch, orientation != 0, o); return 2; }
    if (family == 2) { dirac_source(p, h, mass, orientation == 1, o); return 4; }
    if (mass == 0.0) gluon_source(p, h, o);
    else massive_vector_source(p, h, mass, o);
    return 4;
}

__host__ __device__ __forceinline__ int source_components(uint32_t code) {
    int family = code & 7;
    return family == 0 ? 1 : family == 1 ? 2 : 4;
}

}  // namespace pacuda
