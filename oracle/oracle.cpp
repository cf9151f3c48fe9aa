// The CPU oracle of pacuda's recurrence runner. TEST INFRASTRUCTURE ONLY: tests/, smoke() and
// bench.py's CPU baseline call it as the checker; the product library never does.
//
// A restatement, in plain C++, of the arithmetic of the reference runner
// runner/recurrence_runner.cu (file:line citations below). Every floating-point operation of
// the f64 path is the reference's, in the reference's order, without contraction
// (-ffp-contract=off), so that it equals the reference's f64 kernel (built -fmad=false) bit for
// bit. The df64 / mixed / mixed64 paths restate the reference's other three kernels the same
// way, with the double-word algorithms of Joldes, Muller and Popescu (ACM TOMS 44(2), 2017).
//
// The arena is the caller's arrays (plane-major, `stride` points per plane). Points are run in
// tiles of 64 (each row over the tile's points in turn), the tiles spread over OpenMP threads.
#include "oracle.h"

#include <omp.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <unordered_map>
#include <vector>

namespace {

// ---- df64: a double-word value (hi, lo) of two floats ---------------------------------------
// Algorithms 6 (AccurateDWPlusDW), 12 (DWTimesDW3) and 17 (DWDivDW2, with DWTimesFP3) of
// Joldes, Muller, Popescu; as used by runner/recurrence_runner.cu:70-126.
struct D {
    float hi, lo;
};

inline void exact_sum(float a, float b, float &s, float &e) {  // Knuth's 2Sum
    s = a + b;
    float bv = s - a;
    e = (a - (s - bv)) + (b - bv);
}
inline void fast_exact_sum(float a, float b, float &s, float &e) {  // Dekker's Fast2Sum
    s = a + b;
    e = b - (s - a);
}
inline D dw_add(D x, D y) {
    float sh, sl, th, tl, vh, vl;
    exact_sum(x.hi, y.hi, sh, sl);
    exact_sum(x.lo, y.lo, th, tl);
    fast_exact_sum(sh, sl + th, vh, vl);
    D z;
    fast_exact_sum(vh, tl + vl, z.hi, z.lo);
    return z;
}
inline D dw_neg(D x) { return D{-x.hi, -x.lo}; }
inline D dw_mul(D x, D y) {
    float ch = x.hi * y.hi;
    float cl1 = fmaf(x.hi, y.hi, -ch);
    float tl0 = x.lo * y.lo;
    float tl1 = fmaf(x.hi, y.lo, tl0);
    float cl2 = fmaf(x.lo, y.hi, tl1);
    D z;
    fast_exact_sum(ch, cl1 + cl2, z.hi, z.lo);
    return z;
}
inline D dw_div(D x, D y) {
    float th = x.hi / y.hi;
    float rh = y.hi * th;
    float rl1 = fmaf(y.hi, th, -rh);
    float rl3 = fmaf(y.lo, th, rl1);
    float r_hi, r_lo;
    fast_exact_sum(rh, rl3, r_hi, r_lo);
    float pi_h = x.hi - r_hi;
    float delta = pi_h + (x.lo - r_lo);
    D z;
    fast_exact_sum(th, delta / y.hi, z.hi, z.lo);
    return z;
}

// ---- scalar operations per real type ---------------------------------------------------------
inline double radd(double a, double b) { return a + b; }
inline double rsub(double a, double b) { return a - b; }
inline double rmul(double a, double b) { return a * b; }
inline double rdiv(double a, double b) { return a / b; }
inline double rneg(double a) { return -a; }
inline float radd(float a, float b) { return a + b; }
inline float rsub(float a, float b) { return a - b; }
inline float rmul(float a, float b) { return a * b; }
inline float rdiv(float a, float b) { return a / b; }
inline float rneg(float a) { return -a; }
inline D radd(D a, D b) { return dw_add(a, b); }
inline D rsub(D a, D b) { return dw_add(a, dw_neg(b)); }  // x - y = x + (-y)
inline D rmul(D a, D b) { return dw_mul(a, b); }
inline D rdiv(D a, D b) { return dw_div(a, b); }
inline D rneg(D a) { return dw_neg(a); }

// a formula constant (0, +-1, 2): exact in every type
template <class R> inline R rconst(double x);
template <> inline double rconst<double>(double x) { return x; }
template <> inline float rconst<float>(double x) { return (float)x; }
template <> inline D rconst<D>(double x) { return D{(float)x, 0.0f}; }

// f64 into a type's layout, as the uploads convert (to_df64_planes, f64_to_f32_planes;
// recurrence_runner.cu:546-552, :840-869)
template <class R> inline R narrow(double x);
template <> inline double narrow<double>(double x) { return x; }
template <> inline float narrow<float>(double x) { return (float)x; }
template <> inline D narrow<D>(double x) {
    float hi = (float)x;
    return D{hi, (float)(x - (double)hi)};
}
// a type's value as f64, as the downloads convert (to_f64_planes, f32_to_f64_planes :871-880)
inline double widen64(double x) { return x; }
inline double widen64(float x) { return (double)x; }
inline double widen64(D x) { return (double)x.hi + (double)x.lo; }

// ---- complex numbers ---------------------------------------------------------------------------
template <class R> struct Cx {
    R re, im;
};
template <class R> inline Cx<R> cx(R re, R im) { return Cx<R>{re, im}; }
template <class R> inline Cx<R> cadd(Cx<R> a, Cx<R> b) { return cx(radd(a.re, b.re), radd(a.im, b.im)); }
template <class R> inline Cx<R> csub(Cx<R> a, Cx<R> b) { return cx(rsub(a.re, b.re), rsub(a.im, b.im)); }
template <class R> inline Cx<R> cneg(Cx<R> a) { return cx(rneg(a.re), rneg(a.im)); }
template <class R> inline Cx<R> cmul(Cx<R> a, Cx<R> b) {
    return cx(rsub(rmul(a.re, b.re), rmul(a.im, b.im)), radd(rmul(a.re, b.im), rmul(a.im, b.re)));
}
template <class R> inline Cx<R> cmul_i(Cx<R> a) { return cx(rneg(a.im), a.re); }
template <class R> inline Cx<R> cmul_real(Cx<R> a, R s) { return cx(rmul(a.re, s), rmul(a.im, s)); }

// ---- kinds: value, denominator and amplitude types (recurrence_runner.cu:178-190) -------------
template <class R_, class Den_, class Amp_> struct Kind {
    typedef R_ R;
    typedef Den_ Den;
    typedef Amp_ Amp;
};
typedef Kind<double, double, double> KF64;
typedef Kind<D, D, D> KDF64;
typedef Kind<float, D, D> KMixed;
typedef Kind<float, double, D> KMixed64;

// a stored constant (f64 for the f64 kernel, df64 otherwise) read as R: a float reads the high
// word of the df64 pair (ldr<float>, :150-152)
inline double as_r(double s, double *) { return s; }
inline D as_r(D s, D *) { return s; }
inline float as_r(D s, float *) { return s.hi; }
template <class R, class S> inline R load_as(S s) { return as_r(s, (R *)nullptr); }

// a momentum-form component as R for numerators (ld_form, :200-209)
inline double form_as(double q, double *) { return q; }
inline D form_as(D q, D *) { return q; }
inline float form_as(double q, float *) { return (float)q; }
inline float form_as(D q, float *) { return q.hi; }
template <class R, class Den> inline R ld_form(Den q) { return form_as(q, (R *)nullptr); }

// a denominator as R (ToReal, :212-218): unchanged, or rounded once to f32
inline double to_real(double x, double *) { return x; }
inline D to_real(D x, D *) { return x; }
inline float to_real(double x, float *) { return (float)x; }
inline float to_real(D x, float *) { return x.hi + x.lo; }

// an f32 into the amplitude accumulator (widen, :221-223)
inline D to_amp(float x, D *) { return D{x, 0.0f}; }
inline D to_amp(D x, D *) { return x; }
inline double to_amp(double x, double *) { return x; }

// ---- the executors' arithmetic (recurrence_runner.cu:225-330) ---------------------------------
template <class R> inline Cx<R> minkowski_dot(const Cx<R> *l, const Cx<R> *r) {
    return csub(csub(csub(cmul(l[0], r[0]), cmul(l[1], r[1])), cmul(l[2], r[2])), cmul(l[3], r[3]));
}
template <class R> inline Cx<R> minkowski_real_dot(const Cx<R> *l, const R *q) {
    return csub(csub(csub(cmul_real(l[0], q[0]), cmul_real(l[1], q[1])), cmul_real(l[2], q[2])),
                cmul_real(l[3], q[3]));
}

inline void shape_of(int op, int *c0, int *c1, int *cd) {  // :232-242
    *c0 = op == 4 ? 6 : (op == 5 || op == 6) ? 4 : 2;
    *c1 = 4;
    *cd = (op == 4 || op == 6) ? 4 : op == 5 ? 6 : 2;
}

// The legend of convert/CONVENTIONS.md:74-78, evaluated in the reference's order (:245-282).
template <class R>
void contribution_values(int op, const Cx<R> *l, const Cx<R> *r, const R *q0, const R *q1, Cx<R> *o) {
    if (op == 2) {
        o[0] = cadd(cadd(csub(cneg(cmul_i(cmul(l[0], r[3]))), cmul_i(cmul(l[1], r[1]))), cmul(l[1], r[2])),
                    cmul_i(cmul(l[0], r[0])));
        o[1] = cadd(cadd(csub(cneg(cmul(l[0], r[2])), cmul_i(cmul(l[0], r[1]))), cmul_i(cmul(l[1], r[0]))),
                    cmul_i(cmul(l[1], r[3])));
    } else if (op == 3) {
        o[0] = cadd(cadd(cadd(cneg(cmul(l[1], r[2])), cmul_i(cmul(l[0], r[0]))), cmul_i(cmul(l[0], r[3]))),
                    cmul_i(cmul(l[1], r[1])));
        o[1] = cadd(cadd(cadd(cneg(cmul_i(cmul(l[1], r[3]))), cmul(l[0], r[2])), cmul_i(cmul(l[0], r[1]))),
                    cmul_i(cmul(l[1], r[0])));
    } else if (op == 4) {
        o[0] = cadd(cadd(cmul(l[0], r[1]), cmul(l[1], r[2])), cmul(l[2], r[3]));
        o[1] = cadd(cadd(cmul(l[0], r[0]), cmul(l[3], r[2])), cmul(l[4], r[3]));
        o[2] = cadd(csub(cmul(l[1], r[0]), cmul(l[3], r[1])), cmul(l[5], r[3]));
        o[3] = csub(csub(cmul(l[2], r[0]), cmul(l[4], r[1])), cmul(l[5], r[2]));
    } else if (op == 5) {
        o[0] = csub(cmul(l[0], r[1]), cmul(l[1], r[0]));
        o[1] = csub(cmul(l[0], r[2]), cmul(l[2], r[0]));
        o[2] = csub(cmul(l[0], r[3]), cmul(l[3], r[0]));
        o[3] = csub(cmul(l[1], r[2]), cmul(l[2], r[1]));
        o[4] = csub(cmul(l[1], r[3]), cmul(l[3], r[1]));
        o[5] = csub(cmul(l[2], r[3]), cmul(l[3], r[2]));
    } else {  // 6: (l.r)(u - v) + 2((l.v) r - (r.u) l)
        Cx<R> lr = minkowski_dot(l, r);
        Cx<R> lv = minkowski_real_dot(l, q1);
        Cx<R> ru = minkowski_real_dot(r, q0);
        for (int k = 0; k < 4; k++) {
            Cx<R> momentum_term = cmul_real(lr, rsub(q0[k], q1[k]));
            Cx<R> current_term = cmul_real(csub(cmul(lv, r[k]), cmul(ru, l[k])), rconst<R>(2.0));
            o[k] = cadd(momentum_term, current_term);
        }
    }
}

// ops 7-9 (:285-314; CONVENTIONS.md:83-86)
template <class R>
int propagator_values(int op, const Cx<R> *c, const R *p, R reciprocal, Cx<R> row_factor, Cx<R> *o) {
    if (op == 9) {
        Cx<R> scale = cmul_real(cmul(row_factor, cx(rconst<R>(0.0), rconst<R>(-1.0))), reciprocal);
        for (int k = 0; k < 4; k++) o[k] = cmul(c[k], scale);
        return 4;
    }
    Cx<R> scale = cmul_real(row_factor, reciprocal);
    Cx<R> o0, o1;
    if (op == 7) {
        o0 = cadd(cadd(csub(cneg(cmul_i(cmul_real(c[0], p[3]))), cmul_i(cmul_real(c[1], p[1]))),
                       cmul_real(c[1], p[2])),
                  cmul_i(cmul_real(c[0], p[0])));
        o1 = cadd(cadd(csub(cneg(cmul_real(c[0], p[2])), cmul_i(cmul_real(c[0], p[1]))),
                       cmul_i(cmul_real(c[1], p[0]))),
                  cmul_i(cmul_real(c[1], p[3])));
    } else {
        o0 = cadd(cadd(cadd(cneg(cmul_real(c[1], p[2])), cmul_i(cmul_real(c[0], p[0]))),
                       cmul_i(cmul_real(c[0], p[3]))),
                  cmul_i(cmul_real(c[1], p[1])));
        o1 = cadd(cadd(cadd(cneg(cmul_i(cmul_real(c[1], p[3]))), cmul_real(c[0], p[2])),
                       cmul_i(cmul_real(c[0], p[1]))),
                  cmul_i(cmul_real(c[1], p[0])));
    }
    o[0] = cmul(o0, scale);
    o[1] = cmul(o1, scale);
    return 2;
}

// op 10 (:316-319): factor x value
template <class R> inline Cx<R> identity_value(R fr, R fi, Cx<R> v) {
    return cx(rsub(rmul(fr, v.re), rmul(fi, v.im)), radd(rmul(fr, v.im), rmul(fi, v.re)));
}

// op 11, one component (:321-330)
template <class R> inline Cx<R> closure_increment(Cx<R> l, Cx<R> r, R cr, R ci, R rfr, R rfi) {
    R scale_re = rsub(rmul(cr, rfr), rmul(ci, rfi));
    R scale_im = radd(rmul(cr, rfi), rmul(ci, rfr));
    R product_re = rsub(rmul(l.re, r.re), rmul(l.im, r.im));
    R product_im = radd(rmul(l.re, r.im), rmul(l.im, r.re));
    return cx(rsub(rmul(product_re, scale_re), rmul(product_im, scale_im)),
              radd(rmul(product_re, scale_im), rmul(product_im, scale_re)));
}

// ---- external wavefunctions, f64 (recurrence_runner.cu:337-542; CONVENTIONS.md:52-61) ---------
typedef Cx<double> W;
inline W w64(double re, double im) { return W{re, im}; }
inline double sign_of(double value, double sign_source) { return std::copysign(std::fabs(value), sign_source); }

void quark_weyl(const double *m, int h, int ch, W *o) {  // :346-365
    double e = m[0], px = m[1], py = m[2], pz = m[3];
    if (e > 0.0) {
        double s = (px == 0.0 && py == 0.0 && pz < 0.0) ? 0.0 : std::sqrt(std::fmax(e + pz, 0.0));
        W a = w64(s, 0.0);
        W b = s == 0.0 ? w64(-(double)h * std::sqrt(2.0 * e), 0.0) : w64((double)h * px / s, -py / s);
        if (h == 1 && ch == 1) { o[0] = a; o[1] = b; return; }
        if (h == -1 && ch == -1) { o[0] = b; o[1] = a; return; }
        o[0] = w64(0.0, 0.0); o[1] = w64(0.0, 0.0);
        return;
    }
    double s = (px == 0.0 && py == 0.0 && pz > 0.0) ? 0.0 : -std::sqrt(std::fmax(-(e + pz), 0.0));
    W a = w64(s, 0.0);
    W b = s == 0.0 ? w64(-(double)h * std::sqrt(2.0 * std::fabs(e)), 0.0) : w64(-(double)h * (-px) / s, py / s);
    if (h == -1 && ch == 1) { o[0] = a; o[1] = b; }
    else if (h == 1 && ch == -1) { o[0] = b; o[1] = a; }
    else { o[0] = w64(0.0, 0.0); o[1] = w64(0.0, 0.0); }
}

void antiquark_weyl(const double *m, int h, int ch, W *o) {  // :367-386
    double e = m[0], px = m[1], py = m[2], pz = m[3];
    if (e > 0.0) {
        double s = (px == 0.0 && py == 0.0 && pz < 0.0) ? 0.0 : -std::sqrt(std::fmax(e + pz, 0.0));
        W a = w64(s, 0.0);
        W b = s == 0.0 ? w64(-(double)h * std::sqrt(2.0 * e), 0.0) : w64(-(double)h * px / s, py / s);
        if (h == 1 && ch == 1) { o[0] = b; o[1] = a; return; }
        if (h == -1 && ch == -1) { o[0] = a; o[1] = b; return; }
        o[0] = w64(0.0, 0.0); o[1] = w64(0.0, 0.0);
        return;
    }
    double s = (px == 0.0 && py == 0.0 && pz > 0.0) ? 0.0 : std::sqrt(std::fmax(-(e + pz), 0.0));
    W a = w64(s, 0.0);
    W b = s == 0.0 ? w64(-(double)h * std::sqrt(2.0 * std::fabs(e)), 0.0) : w64((double)h * (-px) / s, -py / s);
    if (h == -1 && ch == 1) { o[0] = b; o[1] = a; }
    else if (h == 1 && ch == -1) { o[0] = a; o[1] = b; }
    else { o[0] = w64(0.0, 0.0); o[1] = w64(0.0, 0.0); }
}

void quark_dirac(const double *m, int h, W *o) {  // :388-406
    double e = m[0], px = m[1], py = m[2], pz = m[3];
    W z = w64(0.0, 0.0);
    if (e > 0.0) {
        double s = (px == 0.0 && py == 0.0 && pz < 0.0) ? 0.0 : std::sqrt(std::fmax(e + pz, 0.0));
        W a = w64(s, 0.0);
        W b = s == 0.0 ? w64(-(double)h * std::sqrt(2.0 * e), 0.0) : w64((double)h * px / s, -py / s);
        if (h == 1) { o[0] = a; o[1] = b; o[2] = z; o[3] = z; return; }
        o[0] = z; o[1] = z; o[2] = b; o[3] = a;
        return;
    }
    double s = (px == 0.0 && py == 0.0 && pz > 0.0) ? 0.0 : -std::sqrt(std::fmax(-(e + pz), 0.0));
    W a = w64(s, 0.0);
    W b = s == 0.0 ? w64(-(double)h * std::sqrt(2.0 * std::fabs(e)), 0.0) : w64(-(double)h * (-px) / s, py / s);
    if (-h == 1) { o[0] = a; o[1] = b; o[2] = z; o[3] = z; }
    else { o[0] = z; o[1] = z; o[2] = b; o[3] = a; }
}

void antiquark_dirac(const double *m, int h, W *o) {  // :408-426
    double e = m[0], px = m[1], py = m[2], pz = m[3];
    W z = w64(0.0, 0.0);
    if (e > 0.0) {
        double s = (px == 0.0 && py == 0.0 && pz < 0.0) ? 0.0 : -std::sqrt(std::fmax(e + pz, 0.0));
        W a = w64(s, 0.0);
        W b = s == 0.0 ? w64(-(double)h * std::sqrt(2.0 * e), 0.0) : w64(-(double)h * px / s, py / s);
        if (-h == 1) { o[0] = z; o[1] = z; o[2] = a; o[3] = b; return; }
        o[0] = b; o[1] = a; o[2] = z; o[3] = z;
        return;
    }
    double s = (px == 0.0 && py == 0.0 && pz > 0.0) ? 0.0 : std::sqrt(std::fmax(-(e + pz), 0.0));
    W a = w64(s, 0.0);
    W b = s == 0.0 ? w64(-(double)h * std::sqrt(2.0 * std::fabs(e)), 0.0) : w64((double)h * (-px) / s, -py / s);
    if (h == 1) { o[0] = z; o[1] = z; o[2] = a; o[3] = b; }
    else { o[0] = b; o[1] = a; o[2] = z; o[3] = z; }
}

void dirac_massive(const double *m, int h, double mass, bool anti, W *o) {  // :428-461
    if (std::fabs(mass) < 1.0e-8) {
        if (anti) antiquark_dirac(m, h, o);
        else quark_dirac(m, h, o);
        return;
    }
    double e = m[0], px = m[1], py = m[2], pz = m[3];
    int n = anti ? (e > 0.0 ? -1 : 1) : (e > 0.0 ? 1 : -1);
    int nh = n * h;
    double k = std::fabs(std::sqrt(px * px + py * py + pz * pz));
    double om1 = std::sqrt(std::fabs(e) + k);
    double om[2] = {om1, mass / om1};
    double f1 = (double)(1 + n + (1 - n) * nh) * 0.5;
    double f2 = (double)(1 + n - (1 - n) * nh) * 0.5;
    int ip = (3 + nh) / 2 - 1, im = (3 - nh) / 2 - 1;
    double g[2] = {f1 * om[ip], f2 * om[im]};
    double tx = e > 0.0 ? px : -px, ty = e > 0.0 ? py : -py, tz = e > 0.0 ? pz : -pz;
    double r = std::fmax(k + tz, 0.0);
    W chi[2];
    chi[0] = k == 0.0 ? w64(1.0, 0.0) : w64(std::sqrt(r * 0.5 / k), 0.0);
    if (r == 0.0 || k == 0.0) chi[1] = w64(-(double)nh, 0.0);
    else {
        double den = std::sqrt(2.0 * k * r);
        chi[1] = w64((double)nh * tx / den, (anti ? ty : -ty) / den);
    }
    double first = anti ? g[0] : g[1], second = anti ? g[1] : g[0];
    o[0] = w64(chi[im].re * first, chi[im].im * first);
    o[1] = w64(chi[ip].re * first, chi[ip].im * first);
    o[2] = w64(chi[im].re * second, chi[im].im * second);
    o[3] = w64(chi[ip].re * second, chi[ip].im * second);
}

void gluon(const double *m, int h, W *o) {  // :463-494
    double e = m[0], px = m[1], py = m[2], pz = m[3];
    double sqh = std::sqrt(0.5);
    if (e > 0.0) {
        double hel = (double)h, pp = e;
        double pt = std::sqrt(px * px + py * py);
        W w3 = w64(hel * pt / pp * sqh, 0.0), w1, w2;
        if (pt != 0.0) {
            double pzpt = pz / (pp * pt) * sqh * hel;
            w1 = w64(-px * pzpt, -py / pt * sqh);
            w2 = w64(-py * pzpt, px / pt * sqh);
        } else {
            w1 = w64(-hel * sqh, 0.0);
            w2 = w64(0.0, sign_of(sqh, pz));
        }
        o[0] = w64(0.0, 0.0); o[1] = w1; o[2] = w2; o[3] = w3;
        return;
    }
    double hel = (double)(-h), pp = -e;
    double pt = std::sqrt(px * px + py * py);
    W w3 = w64(hel * pt / pp * sqh, 0.0), w1, w2;
    if (pt != 0.0) {
        double pzpt = -pz / (pp * pt) * sqh * hel;
        w1 = w64(px * pzpt, py / pt * sqh);
        w2 = w64(py * pzpt, -px / pt * sqh);
    } else {
        w1 = w64(-hel * sqh, 0.0);
        w2 = w64(0.0, -sign_of(sqh, pz));
    }
    o[0] = w64(0.0, 0.0); o[1] = w1; o[2] = w2; o[3] = w3;
}

void massive_vector(const double *m0, int h, double mass, W *o) {  // :496-526
    double m[4] = {m0[0], m0[1], m0[2], m0[3]};
    if (m[0] < 0.0) {
        for (int k = 0; k < 4; k++) m[k] = -m[k];
        h = -h;
    }
    double e = m[0], px = m[1], py = m[2], pz = m[3];
    double sqh = std::sqrt(0.5);
    double hel = (double)h;
    double nsv = (double)std::abs(h);
    double pt2 = px * px + py * py;
    double pp = std::fmin(e, std::sqrt(pt2 + pz * pz));
    double pt = std::fmin(pp, std::sqrt(pt2));
    double hel0 = 1.0 - std::fabs(hel);
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

// the wavefunction of a template code; its component count (:529-542)
int source_values(uint32_t code, double mass, const double *p, W *o) {
    int family = code & 7, orientation = (code >> 3) & 3;
    int h = (int)((code >> 5) & 7) - 2, ch = (int)((code >> 8) & 3) - 1;
    if (family == 0) { o[0] = w64(1.0, 0.0); return 1; }
    if (family == 1) {
        if (orientation == 0) quark_weyl(p, h, ch, o);
        else antiquark_weyl(p, h, ch, o);
        return 2;
    }
    if (family == 2) { dirac_massive(p, h, mass, orientation == 1, o); return 4; }
    if (mass == 0.0) gluon(p, h, o);
    else massive_vector(p, h, mass, o);
    return 4;
}

// ---- the plan: decode, sort, program (recurrence_runner.cu:913-1054) --------------------------
struct Row {
    int op;
    uint32_t f[8];
    std::vector<uint32_t> data;
};

bool decode(const uint64_t *words, uint32_t count, const uint8_t *width, std::vector<Row> &rows) {
    rows.clear();
    for (uint32_t n = 0; n < count; n++) {
        uint64_t w = words[n];
        if ((w & 15) == 14) {  // a binding and its data words
            Row r{};
            r.op = 14;
            r.f[0] = (uint32_t)(w >> 4) & 0xffff;
            r.f[1] = (uint32_t)(w >> 20) & 0xff;
            r.f[2] = (uint32_t)(w >> 28) & 0xff;
            r.f[3] = (uint32_t)(w >> 36) & 1;
            uint32_t codes = r.f[1] + r.f[2];
            for (uint32_t k = 0; k < codes; k++) {
                uint64_t d = n + 1 + k / 2 < count ? words[n + 1 + k / 2] : 0;
                r.data.push_back((uint32_t)(k % 2 ? d >> 32 : d));
            }
            n += (codes + 1) / 2;
            rows.push_back(r);
            continue;
        }
        bool wide = false;
        auto take = [&](int bits) {  // the low `bits` bits, then shift them out
            if (bits > 32) { wide = true; return 0u; }
            uint32_t v = (uint32_t)(w & ((1ull << bits) - 1));
            w >>= bits;
            return v;
        };
        Row r{};
        r.op = (int)take(4);
        const int P = width[W_P], A = width[W_A], F = width[W_F], X = width[W_X], S = width[W_S], K = width[W_K];
        int fields[8] = {0}, nf = 0;
        if (r.op == 1) { fields[0] = P; fields[1] = P; nf = 2; }
        else if (r.op >= 2 && r.op <= 6) { int f[8] = {1, S, P, P, P, F, F, X}; std::copy(f, f + 8, fields); nf = 8; }
        else if (r.op >= 7 && r.op <= 9) { fields[0] = P; fields[1] = F; fields[2] = X; nf = 3; }
        else if (r.op == 10) { fields[0] = P; fields[1] = K; fields[2] = X; nf = 3; }
        else if (r.op == 11) { int f[6] = {P, P, A, X, X, K}; std::copy(f, f + 6, fields); nf = 6; }
        else if (r.op == 12) { int f[5] = {P, F, X, S, 10}; std::copy(f, f + 5, fields); nf = 5; }
        else if (r.op == 13) { int f[7] = {1, P, P, P, F, F, X}; std::copy(f, f + 7, fields); nf = 7; }
        else return false;  // ops 0 and 15 are not in the format
        for (int k = 0; k < nf; k++) r.f[k] = take(fields[k]);
        if (wide) return false;  // fields are at most 32 bits
        rows.push_back(r);
    }
    return true;
}

void sort_contribution_runs(std::vector<Row> &rows) {  // :980-1007
    size_t n = 0;
    while (n < rows.size()) {
        if (rows[n].op < 2 || rows[n].op > 6) { n++; continue; }
        size_t end = n;
        while (end < rows.size() && rows[end].op >= 2 && rows[end].op <= 6) end++;
        std::unordered_map<uint32_t, uint32_t> dst_base;
        bool safe = true;
        for (size_t k = n; k < end && safe; k++) {
            int c0, c1, cd;
            shape_of(rows[k].op, &c0, &c1, &cd);
            for (int q = 0; q < cd; q++) {
                auto it = dst_base.emplace(rows[k].f[4] + q, rows[k].f[4]);
                if (it.first->second != rows[k].f[4]) safe = false;
            }
        }
        for (size_t k = n; k < end && safe; k++) {
            int c0, c1, cd;
            shape_of(rows[k].op, &c0, &c1, &cd);
            for (int q = 0; q < c0 && safe; q++) safe = !dst_base.count(rows[k].f[2] + q);
            for (int q = 0; q < c1 && safe; q++) safe = !dst_base.count(rows[k].f[3] + q);
        }
        if (safe)
            std::stable_sort(rows.begin() + n, rows.begin() + end,
                             [](const Row &x, const Row &y) { return x.f[4] < y.f[4]; });
        n = end;
    }
}

enum { K_CLEAR = 1, K_CONTRIB, K_PROP, K_IDENTITY, K_CLOSURE, K_SOURCE };
enum { F_INIT = 1, F_FIRST = 2, F_LAST = 4 };
struct Op {
    int kind, op, flags;
    uint32_t w[8];
};

// the instructions of the rows; false for a row this runner cannot run
bool program(const std::vector<Row> &rows, std::vector<Op> &ops, uint32_t *sources) {
    ops.clear();
    for (size_t n = 0; n < rows.size(); n++) {
        const Row &r = rows[n];
        if (r.op == 13 || r.op == 14) return false;  // no symjit kernels (:1141-1145)
        Op o{};
        o.op = r.op;
        if (r.op >= 2 && r.op <= 6) {
            bool first = n == 0 || rows[n - 1].op < 2 || rows[n - 1].op > 6 || rows[n - 1].f[4] != r.f[4];
            bool last = n + 1 == rows.size() || rows[n + 1].op < 2 || rows[n + 1].op > 6 || rows[n + 1].f[4] != r.f[4];
            o.kind = K_CONTRIB;
            o.flags = (r.f[0] ? F_INIT : 0) | (first ? F_FIRST : 0) | (last ? F_LAST : 0);
            for (int k = 1; k < 8; k++) o.w[k] = r.f[k];
        } else {
            o.kind = r.op == 1 ? K_CLEAR : r.op <= 9 ? K_PROP : r.op == 10 ? K_IDENTITY : r.op == 11 ? K_CLOSURE : K_SOURCE;
            for (int k = 0; k < 7; k++) o.w[k + 1] = r.f[k];
        }
        ops.push_back(o);
    }
    uint32_t s = 0;
    while (s < ops.size() && ops[s].kind == K_SOURCE) s++;
    for (size_t n = s; n < ops.size(); n++)
        if (ops[n].kind == K_SOURCE) return false;  // a source after other rows (:1167-1171)
    *sources = s;
    return true;
}

// every plane, form, scale and factor a program names is inside the call's tables
bool in_bounds(const std::vector<Op> &ops, const pacman_recurrence_call *c) {
    uint64_t P = c->current_planes, A = c->amplitude_planes, F = c->momentum_planes / 4, S = c->scale_count,
             X = c->factor_count;
    auto range = [](uint64_t first, uint64_t n, uint64_t limit) { return first + n <= limit; };
    for (const Op &o : ops) {
        const uint32_t *w = o.w;
        int c0, c1, cd;
        switch (o.kind) {
        case K_CLEAR: if (!range(w[1], w[2], P)) return false; break;
        case K_CONTRIB:
            shape_of(o.op, &c0, &c1, &cd);
            if (!range(w[2], c0, P) || !range(w[3], c1, P) || !range(w[4], cd, P) || w[1] >= S || w[7] >= X) return false;
            if (o.op == 6 && (w[5] >= F || w[6] >= F)) return false;
            break;
        case K_PROP:
            if (!range(w[1], o.op == 9 ? 4 : 2, P) || w[2] >= F || w[3] >= X) return false;
            break;
        case K_IDENTITY: if (!range(w[1], w[2], P) || w[3] >= X) return false; break;
        case K_CLOSURE:
            if (!range(w[1], w[6], P) || !range(w[2], w[6], P) || w[3] >= A || w[4] >= X || !range(w[5], w[6], X))
                return false;
            break;
        case K_SOURCE: if (!range(w[1], 4, P) || w[2] >= F || w[3] >= X || w[4] >= S) return false; break;
        }
    }
    return true;
}

// ---- the interpreter over tiles of points --------------------------------------------------
constexpr size_t TILE = 64;

template <class K, class SC> struct State {
    typedef typename K::R R;
    typedef typename K::Den Den;
    typedef typename K::Amp Amp;
    R *cre, *cim;
    Amp *are, *aim;
    const Den *mom;     // forms in the kernel's layout
    const SC *sre, *sim, *fre, *fim;  // constants: double (f64) or df64
    size_t ld;
};

template <class K, class SC>
void run_tile(const State<K, SC> &s, const std::vector<Op> &ops, uint32_t first_op, size_t i0, size_t i1) {
    typedef typename K::R R;
    typedef typename K::Den Den;
    typedef typename K::Amp Amp;
    typedef Cx<R> C;
    static thread_local std::vector<C> acc_store;
    acc_store.assign(6 * TILE, C{rconst<R>(0.0), rconst<R>(0.0)});
    C *acc = acc_store.data();
    auto cur = [&](uint32_t plane, size_t i) { return C{s.cre[plane * s.ld + i], s.cim[plane * s.ld + i]}; };
    auto put = [&](uint32_t plane, size_t i, C v) { s.cre[plane * s.ld + i] = v.re; s.cim[plane * s.ld + i] = v.im; };
    for (size_t n = first_op; n < ops.size(); n++) {
        const Op &o = ops[n];
        const uint32_t *w = o.w;
        for (size_t i = i0; i < i1; i++) {
            C *a = acc + 6 * (i - i0);
            if (o.kind == K_CONTRIB) {
                int c0, c1, cd;
                shape_of(o.op, &c0, &c1, &cd);
                C scale = cmul(C{load_as<R>(s.sre[w[1]]), load_as<R>(s.sim[w[1]])},
                               C{load_as<R>(s.fre[w[7]]), load_as<R>(s.fim[w[7]])});
                C l[6], r[4], v[6];
                R q0[4], q1[4];
                for (int k = 0; k < c0; k++) l[k] = cur(w[2] + k, i);
                for (int k = 0; k < c1; k++) r[k] = cur(w[3] + k, i);
                if (o.op == 6)
                    for (int k = 0; k < 4; k++) {
                        q0[k] = ld_form<R, Den>(s.mom[(w[5] * 4 + k) * s.ld + i]);
                        q1[k] = ld_form<R, Den>(s.mom[(w[6] * 4 + k) * s.ld + i]);
                    }
                contribution_values(o.op, l, r, q0, q1, v);
                for (int k = 0; k < cd; k++) {
                    C c = cmul(v[k], scale);
                    if (!(o.flags & F_FIRST)) a[k] = cadd(a[k], c);
                    else if (o.flags & F_INIT) a[k] = c;
                    else a[k] = cadd(cur(w[4] + k, i), c);
                }
                if (o.flags & F_LAST)
                    for (int k = 0; k < cd; k++) put(w[4] + k, i, a[k]);
            } else if (o.kind == K_CLEAR) {
                for (uint32_t k = 0; k < w[2]; k++) put(w[1] + k, i, C{rconst<R>(0.0), rconst<R>(0.0)});
            } else if (o.kind == K_PROP) {
                int m = o.op == 9 ? 4 : 2;
                R p[4];
                Den q[4];
                for (int k = 0; k < 4; k++) {
                    q[k] = s.mom[(w[2] * 4 + k) * s.ld + i];
                    p[k] = ld_form<R, Den>(q[k]);
                }
                Den norm = rsub(rsub(rsub(rmul(q[0], q[0]), rmul(q[1], q[1])), rmul(q[2], q[2])), rmul(q[3], q[3]));
                R reciprocal = to_real(rdiv(rconst<Den>(1.0), norm), (R *)nullptr);
                C c[4], v[4];
                for (int k = 0; k < m; k++) c[k] = cur(w[1] + k, i);
                propagator_values(o.op, c, p, reciprocal, C{load_as<R>(s.fre[w[3]]), load_as<R>(s.fim[w[3]])}, v);
                for (int k = 0; k < m; k++) put(w[1] + k, i, v[k]);
            } else if (o.kind == K_IDENTITY) {
                R fr = load_as<R>(s.fre[w[3]]), fi = load_as<R>(s.fim[w[3]]);
                for (uint32_t k = 0; k < w[2]; k++) put(w[1] + k, i, identity_value(fr, fi, cur(w[1] + k, i)));
            } else if (o.kind == K_CLOSURE) {
                R rfr = load_as<R>(s.fre[w[4]]), rfi = load_as<R>(s.fim[w[4]]);
                size_t at = w[3] * s.ld + i;
                Amp dr = s.are[at], di = s.aim[at];
                for (uint32_t k = 0; k < w[6]; k++) {
                    C v = closure_increment(cur(w[1] + k, i), cur(w[2] + k, i), load_as<R>(s.fre[w[5] + k]),
                                            load_as<R>(s.fim[w[5] + k]), rfr, rfi);
                    dr = radd(dr, to_amp(v.re, (Amp *)nullptr));
                    di = radd(di, to_amp(v.im, (Amp *)nullptr));
                }
                s.are[at] = dr;
                s.aim[at] = di;
            }
        }
    }
}

int status_invalid() { return PACMAN_RECURRENCE_INVALID; }

template <class K, class SC>
int run_kind(const pacman_recurrence_call *c, const std::vector<Op> &ops, uint32_t sources,
             const std::vector<double> &forms, int threads) {
    typedef typename K::R R;
    typedef typename K::Den Den;
    typedef typename K::Amp Amp;
    size_t ld = c->stride, points = c->points;
    size_t cur_n = (size_t)c->current_planes * ld, amp_n = (size_t)c->amplitude_planes * ld;
    // the arena in the kernel's layout (the f64 kernel works in the caller's arrays)
    std::vector<R> cre_v, cim_v;
    std::vector<Amp> are_v, aim_v;
    std::vector<Den> mom_v;
    std::vector<SC> small(2 * ((size_t)c->scale_count + c->factor_count) + 1);
    R *cre;
    R *cim;
    Amp *are;
    Amp *aim;
    const Den *mom;
    constexpr bool f64 = sizeof(R) == 8 && sizeof(Amp) == 8 && sizeof(SC) == 8 && std::is_same<R, double>::value;
    if constexpr (f64) {
        cre = (R *)c->current_re; cim = (R *)c->current_im; are = (Amp *)c->amplitude_re; aim = (Amp *)c->amplitude_im;
        mom = (const Den *)forms.data();
    } else {
        cre_v.resize(cur_n); cim_v.resize(cur_n); are_v.resize(amp_n); aim_v.resize(amp_n);
        for (size_t k = 0; k < cur_n; k++) { cre_v[k] = narrow<R>(c->current_re[k]); cim_v[k] = narrow<R>(c->current_im[k]); }
        for (size_t k = 0; k < amp_n; k++) { are_v[k] = narrow<Amp>(c->amplitude_re[k]); aim_v[k] = narrow<Amp>(c->amplitude_im[k]); }
        cre = cre_v.data(); cim = cim_v.data(); are = are_v.data(); aim = aim_v.data();
        mom_v.resize(forms.size());
        for (size_t k = 0; k < forms.size(); k++) mom_v[k] = narrow<Den>(forms[k]);
        mom = mom_v.data();
    }
    SC *sre = small.data(), *sim = sre + c->scale_count, *fre = sim + c->scale_count, *fim = fre + c->factor_count;
    for (uint32_t k = 0; k < c->scale_count; k++) { sre[k] = narrow<SC>(c->scale_re[k]); sim[k] = narrow<SC>(c->scale_im[k]); }
    for (uint32_t k = 0; k < c->factor_count; k++) { fre[k] = narrow<SC>(c->factor_re[k]); fim[k] = narrow<SC>(c->factor_im[k]); }
    // the sources: f64, from the f64 forms, scales and factors, narrowed into the layout (:769-785)
    for (uint32_t n = 0; n < sources; n++) {
        const uint32_t *w = ops[n].w;
        for (size_t i = 0; i < points; i++) {
            double p[4];
            for (int k = 0; k < 4; k++) p[k] = forms[(w[2] * 4 + k) * ld + i];
            double fr = c->factor_re[w[3]], fi = c->factor_im[w[3]], mass = c->scale_re[w[4]];
            W v[4];
            int m = source_values(w[5], mass, p, v);
            for (int k = 0; k < m; k++) {
                double sr = fr * v[k].re - fi * v[k].im, si = fr * v[k].im + fi * v[k].re;
                cre[(w[1] + k) * ld + i] = narrow<R>(sr);
                cim[(w[1] + k) * ld + i] = narrow<R>(si);
            }
        }
    }
    State<K, SC> s{cre, cim, are, aim, mom, sre, sim, fre, fim, ld};
    long tiles = (long)((points + TILE - 1) / TILE);
    int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (long t = 0; t < tiles; t++) {
        size_t i0 = (size_t)t * TILE, i1 = std::min(points, i0 + TILE);
        run_tile<K, SC>(s, ops, sources, i0, i1);
    }
    if constexpr (!f64) {
        for (size_t p = 0; p < c->current_planes; p++)
            for (size_t i = 0; i < points; i++) {
                c->current_re[p * ld + i] = widen64(cre[p * ld + i]);
                c->current_im[p * ld + i] = widen64(cim[p * ld + i]);
            }
        for (size_t p = 0; p < c->amplitude_planes; p++)
            for (size_t i = 0; i < points; i++) {
                c->amplitude_re[p * ld + i] = widen64(are[p * ld + i]);
                c->amplitude_im[p * ld + i] = widen64(aim[p * ld + i]);
            }
    }
    return PACMAN_RECURRENCE_OK;
}

}  // namespace

extern "C" int oracle_decode(const uint64_t *words, uint32_t count, const uint8_t *width, int sort,
                             uint32_t *out, uint32_t capacity) {
    std::vector<Row> rows;
    if (!words || !width || !decode(words, count, width, rows)) return -1;
    if (sort) sort_contribution_runs(rows);
    if (out) {
        for (size_t n = 0; n < rows.size() && n < capacity; n++) {
            out[9 * n] = (uint32_t)rows[n].op;
            for (int k = 0; k < 8; k++) out[9 * n + 1 + k] = rows[n].f[k];
        }
    }
    return (int)rows.size();
}

extern "C" int oracle_run(const pacman_recurrence_call *in, int kernel, int sort, int threads) {
    const size_t v1 = offsetof(pacman_recurrence_call, zero_amplitude);
    const size_t v2 = offsetof(pacman_recurrence_call, external_momenta);
    if (!in || in->abi_version != PACMAN_RECURRENCE_ABI ||
        (in->struct_size != sizeof(pacman_recurrence_call) && in->struct_size != v1 && in->struct_size != v2))
        return PACMAN_RECURRENCE_INVALID;
    pacman_recurrence_call call;
    memset(&call, 0, sizeof call);
    memcpy(&call, in, in->struct_size);
    const pacman_recurrence_call *c = &call;
    if (c->points == 0 || c->points > c->stride || !c->words || (c->zero_amplitude_runs && !c->zero_amplitude))
        return PACMAN_RECURRENCE_INVALID;
    if (kernel < 0 || kernel > 3) return PACMAN_RECURRENCE_INVALID;
    size_t ld = c->stride, points = c->points;
    uint32_t form_count = c->momentum_planes / 4;
    std::vector<double> forms((size_t)c->momentum_planes * ld + 1, 0.0);
    if (c->flags & PACMAN_RECURRENCE_FORMS_ON_DEVICE) {
        if (!c->external_momenta || !c->form_terms || (c->term_count && (!c->term_slots || !c->term_coefficients)))
            return PACMAN_RECURRENCE_INVALID;
        for (uint32_t f = 0; f < form_count; f++)
            if (c->form_terms[2 * f] > c->term_count || c->form_terms[2 * f + 1] > c->term_count - c->form_terms[2 * f])
                return PACMAN_RECURRENCE_INVALID;
        for (uint32_t t = 0; t < c->term_count; t++)
            if (c->term_slots[t] >= c->external_count) return PACMAN_RECURRENCE_INVALID;
        // fill_forms (:747-764): 0.0 + c0 p + c1 p + ..., in term order
        for (uint32_t f = 0; f < form_count; f++) {
            uint32_t first = c->form_terms[2 * f], n = c->form_terms[2 * f + 1];
            for (int k = 0; k < 4; k++)
                for (size_t i = 0; i < points; i++) {
                    double v = 0.0;
                    for (uint32_t t = 0; t < n; t++) {
                        double term = c->term_coefficients[first + t] *
                                      c->external_momenta[((size_t)c->term_slots[first + t] * 4 + k) * points + i];
                        v = t == 0 ? 0.0 + term : v + term;
                    }
                    forms[(f * 4 + k) * ld + i] = v;
                }
        }
    } else if (c->momentum_planes) {
        if (!c->momenta) return PACMAN_RECURRENCE_INVALID;
        for (size_t p = 0; p < c->momentum_planes; p++)
            for (size_t i = 0; i < points; i++) forms[p * ld + i] = c->momenta[p * ld + i];
    }
    if ((c->scale_count && (!c->scale_re || !c->scale_im)) || (c->factor_count && (!c->factor_re || !c->factor_im)))
        return PACMAN_RECURRENCE_INVALID;
    for (uint32_t r = 0; r < c->zero_amplitude_runs; r++) {
        uint32_t first = c->zero_amplitude[2 * r], n = c->zero_amplitude[2 * r + 1];
        if (first > c->amplitude_planes || n > c->amplitude_planes - first) return PACMAN_RECURRENCE_INVALID;
        for (uint32_t p = first; p < first + n; p++)
            for (size_t i = 0; i < points; i++) c->amplitude_re[p * ld + i] = c->amplitude_im[p * ld + i] = 0.0;
    }
    std::vector<Row> rows;
    if (!decode(c->words, c->word_count, c->width, rows)) return PACMAN_RECURRENCE_INVALID;
    if (sort) sort_contribution_runs(rows);
    std::vector<Op> ops;
    uint32_t sources = 0;
    if (!program(rows, ops, &sources)) return PACMAN_RECURRENCE_DEVICE_ERROR;
    if (!in_bounds(ops, c)) return PACMAN_RECURRENCE_INVALID;
    if ((c->current_planes && (!c->current_re || !c->current_im)) ||
        (c->amplitude_planes && (!c->amplitude_re || !c->amplitude_im)))
        return PACMAN_RECURRENCE_INVALID;
    switch (kernel) {
    case PACMAN_RECURRENCE_KERNEL_F64: return run_kind<KF64, double>(c, ops, sources, forms, threads);
    case PACMAN_RECURRENCE_KERNEL_MIXED: return run_kind<KMixed, D>(c, ops, sources, forms, threads);
    case PACMAN_RECURRENCE_KERNEL_MIXED64: return run_kind<KMixed64, D>(c, ops, sources, forms, threads);
    default: return run_kind<KDF64, D>(c, ops, sources, forms, threads);
    }
}

// ---- reductions (recurrence_runner.cu:1496-1572) ---------------------------------------------
namespace {
inline double lc_term(double w, double re, double im) { return w * std::fma(re, re, im * im); }
}

extern "C" int oracle_reduce(const pacman_recurrence_reduce *r, const double *are, const double *aim, uint32_t stride) {
    if (!r || (r->count && (!r->planes || !r->weights)) || !r->output) return PACMAN_RECURRENCE_INVALID;
    for (uint32_t i = 0; i < r->points; i++) {
        double acc = r->output[i];
        for (uint32_t k = 0; k < r->count; k++) {
            size_t at = (size_t)r->planes[k] * stride + i;
            acc = acc + lc_term(r->weights[k], are[at], aim[at]);
        }
        r->output[i] = acc;
    }
    return PACMAN_RECURRENCE_OK;
}

extern "C" int oracle_reduce_resolved(const pacman_recurrence_reduce_resolved *r, const double *are,
                                      const double *aim, uint32_t stride) {
    if (!r || !r->offsets || !r->output || r->outputs == 0) return PACMAN_RECURRENCE_INVALID;
    bool zero = r->flags & PACMAN_RECURRENCE_OUTPUT_ZERO;
    for (uint32_t o = 0; o < r->outputs; o++)
        for (uint32_t i = 0; i < r->points; i++) {
            size_t out = (size_t)o * r->output_stride + (size_t)i * r->point_stride;
            double acc = zero ? 0.0 : r->output[out];
            for (uint32_t k = r->offsets[o]; k < r->offsets[o + 1]; k++) {
                size_t at = (size_t)r->planes[k] * stride + i;
                acc = acc + lc_term(r->weights[k], are[at], aim[at]);
            }
            r->output[out] = acc;
        }
    return PACMAN_RECURRENCE_OK;
}

extern "C" int oracle_reduce_sample(const pacman_recurrence_reduce_sample *r, const double *are, const double *aim,
                                    uint32_t stride) {
    if (!r || !r->offsets || !r->helicity || !r->random || !r->total || !r->chosen || r->outputs == 0)
        return PACMAN_RECURRENCE_INVALID;
    bool factor = r->numerator != r->denominator;
    for (uint32_t i = 0; i < r->points; i++) {
        double s = r->scale ? r->scale[i] : 1.0;
        auto value = [&](uint32_t o) {
            double acc = 0.0;
            for (uint32_t k = r->offsets[o]; k < r->offsets[o + 1]; k++) {
                size_t at = (size_t)r->planes[k] * stride + i;
                acc = acc + lc_term(r->weights[k], are[at], aim[at]);
            }
            if (factor) acc = acc * r->numerator / r->denominator;
            if (s != 1.0) acc = acc * s;
            return acc;
        };
        double t = 0.0;
        for (uint32_t o = 0; o < r->outputs; o++) t = t + value(o);
        double target = r->random[i] * t, cumulative = 0.0;
        uint32_t pick = 0;
        for (uint32_t o = 0; o < r->outputs; o++) {
            double v = value(o);
            if (v <= 0.0) continue;
            pick = r->helicity[o];
            cumulative = cumulative + v;
            if (cumulative > target) break;
        }
        r->total[i] = t;
        r->chosen[i] = pick;
    }
    return PACMAN_RECURRENCE_OK;
}

extern "C" int oracle_sources(const uint32_t *codes, const double *masses, const double *momenta, uint32_t count,
                              double *out_re, double *out_im) {
    for (uint32_t i = 0; i < count; i++) {
        W v[4] = {w64(0.0, 0.0), w64(0.0, 0.0), w64(0.0, 0.0), w64(0.0, 0.0)};
        source_values(codes[i], masses[i], momenta + 4 * (size_t)i, v);
        for (int k = 0; k < 4; k++) {
            out_re[4 * (size_t)i + k] = v[k].re;
            out_im[4 * (size_t)i + k] = v[k].im;
        }
    }
    return PACMAN_RECURRENCE_OK;
}
