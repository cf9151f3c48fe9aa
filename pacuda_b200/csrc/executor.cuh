// The fused plan kernel over the global arena: one thread per phase-space point runs the whole
// plan (forms, sources, rows, closures) in the order of the instruction stream.
#pragma once
#include <stdint.h>

#include "arith.cuh"
#include "program.h"

namespace pacuda {

struct RunArgs {
    void *cre, *cim;      // current arena in the kind's layout (plane-major, stride ld)
    void *are, *aim;      // amplitude arena (f64 or df64 pairs)
    double *mom;          // momentum forms: f64 planes, turned into the kind's Den layout in place
    size_t ld;
    uint32_t points;
    const double *s64;    // f64 constants: scale re [scales], scale im, then ...
    const double *f64;    // ... factor re [factors], factor im
    const double *kconst; // the same constants in the kind's layout (8 bytes each)
    uint32_t scales, factors, forms;
    bool den_is_f64;
    // forms from external momenta (null: the forms were uploaded)
    const double *external, *coefficients;
    const uint32_t *form_terms, *term_slots;
};

__device__ __forceinline__ Ins load_ins(const Ins *p, uint32_t n) {
    const uint4 *q = reinterpret_cast<const uint4 *>(p + n);
    uint4 x = __ldg(q), y = __ldg(q + 1);
    Ins o;
    o.head = x.x; o.a = x.y; o.b = x.z; o.c = x.w;
    o.f = y.x; o.s = y.y; o.x = y.z; o.y = y.w;
    return o;
}

// per-point views of the arenas
template <class K> struct PointView {
    typedef typename K::R R;
    typedef typename K::Den Den;
    typedef typename K::Amp Amp;
    typedef typename K::Const Const;
    R *cre, *cim;
    Amp *are, *aim;
    const Den *mom;
    const Const *sre, *sim, *fre, *fim;
    size_t ld, i;
    __device__ __forceinline__ Cx<R> cur(uint32_t plane) const { return cx(cre[plane * ld + i], cim[plane * ld + i]); }
    __device__ __forceinline__ void put(uint32_t plane, Cx<R> v) const {
        cre[plane * ld + i] = v.re;
        cim[plane * ld + i] = v.im;
    }
    __device__ __forceinline__ Den form(uint32_t f, int k) const { return mom[(f * 4 + k) * ld + i]; }
    __device__ __forceinline__ Cx<R> scale(uint32_t s) const { return cx(cast<R>(sre[s]), cast<R>(sim[s])); }
    __device__ __forceinline__ Cx<R> factor(uint32_t x) const { return cx(cast<R>(fre[x]), cast<R>(fim[x])); }
    __device__ __forceinline__ void amp(uint32_t a, Amp &re, Amp &im) const {
        re = are[a * ld + i];
        im = aim[a * ld + i];
    }
    __device__ __forceinline__ void put_amp(uint32_t a, Amp re, Amp im) const {
        are[a * ld + i] = re;
        aim[a * ld + i] = im;
    }
    // the global arena is the storage: nothing to write back
    __device__ __forceinline__ void writeback(uint32_t, const Cx<R> *, int) const {}
    // (its schedules keep amplitudes: no closure stores a reduction term)
    template <class A> __device__ __forceinline__ void put_term(uint32_t, A, A) const {}
};

template <class K, int OP, class V>
__device__ __forceinline__ void exec_contribution(const V &v, const Ins &o, Cx<typename K::R> *acc) {
    typedef typename K::R R;
    constexpr int c0 = Shape<OP>::c0, c1 = Shape<OP>::c1, cd = Shape<OP>::cd;
    const uint32_t flags = ins_flags(o);
    Cx<R> scale = v.scale(o.s) * v.factor(o.x);
    Cx<R> l[c0], r[c1], val[cd];
    R q0[4], q1[4];
#pragma unroll
    for (int k = 0; k < c0; k++) l[k] = v.cur(o.a + k);
#pragma unroll
    for (int k = 0; k < c1; k++) r[k] = v.cur(o.b + k);
    if (OP == 6) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            q0[k] = form_as<R>(v.form(o.f & 0xffff, k));
            q1[k] = form_as<R>(v.form(o.f >> 16, k));
        }
    }
    contribution<OP>(l, r, q0, q1, val);
    if (!(flags & F_FIRST)) {
#pragma unroll
        for (int k = 0; k < cd; k++) acc[k] = acc[k] + val[k] * scale;
    } else if (flags & F_INIT) {
#pragma unroll
        for (int k = 0; k < cd; k++) acc[k] = val[k] * scale;
    } else {
#pragma unroll
        for (int k = 0; k < cd; k++) acc[k] = v.cur(o.c + k) + val[k] * scale;
    }
    if (flags & F_LAST) {
        if (!(flags & 32))  // else the sums stay in registers for the task's closures
#pragma unroll
            for (int k = 0; k < cd; k++) v.put(o.c + k, acc[k]);
        if (flags & 8) v.writeback(o.y, acc, cd);
    }
}

template <class K, int OP, class V>
__device__ __forceinline__ void exec_propagator(const V &v, const Ins &o) {
    typedef typename K::R R;
    typedef typename K::Den Den;
    constexpr int m = OP == 9 ? 4 : 2;
    Den q[4];
    R p[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        q[k] = v.form(o.f, k);
        p[k] = form_as<R>(q[k]);
    }
    Den norm = ((q[0] * q[0] - q[1] * q[1]) - q[2] * q[2]) - q[3] * q[3];
    R reciprocal = den_real(konst<Den>(1.0) / norm, (R *)nullptr);
    Cx<R> c[4], out[4];
#pragma unroll
    for (int k = 0; k < m; k++) c[k] = v.cur(o.a + k);
    propagator<OP>(c, p, reciprocal, v.factor(o.x), out);
#pragma unroll
    for (int k = 0; k < m; k++) v.put(o.a + k, out[k]);
    if (ins_flags(o) & 8) v.writeback(o.y, out, m);
}

template <class K, class V>
__device__ __forceinline__ void exec_closure(const V &v, const Ins &o, const Cx<typename K::R> *acc) {
    typedef typename K::R R;
    typedef typename K::Amp Amp;
    Cx<R> f = v.factor(o.x);
    Amp dr, di;
    const bool term = ins_flags(o) & 64;  // F_TERM: the amplitude's only closure, from zero
    if (term) {
        dr = konst<Amp>(0.0);
        di = konst<Amp>(0.0);
    } else {
        v.amp(o.c, dr, di);
    }
    if (ins_flags(o) & 16) {
        // parent 0 is the task's sums (at most 6 components): indices known at compile time keep
        // the sums in registers
#pragma unroll
        for (int k = 0; k < 6; k++) {
            if ((uint32_t)k >= o.s) break;
            Cx<R> t = closure_term(acc[k], v.cur(o.b + k), cast<R>(v.fre[o.y + k]), cast<R>(v.fim[o.y + k]), f.re, f.im);
            dr = dr + amp_of(t.re, (Amp *)nullptr);
            di = di + amp_of(t.im, (Amp *)nullptr);
        }
    } else {
        for (uint32_t k = 0; k < o.s; k++) {
            Cx<R> t = closure_term(v.cur(o.a + k), v.cur(o.b + k), cast<R>(v.fre[o.y + k]), cast<R>(v.fim[o.y + k]), f.re,
                                   f.im);
            dr = dr + amp_of(t.re, (Amp *)nullptr);
            di = di + amp_of(t.im, (Amp *)nullptr);
        }
    }
    if (!term) v.put_amp(o.c, dr, di);
    else if (o.c != 0xffff) v.put_term(o.c, dr, di);
}

// identity (op 10) and clear (op 1) over `o.b` components
template <class K, class V>
__device__ __forceinline__ void exec_identity(const V &v, const Ins &o) {
    typedef typename K::R R;
    Cx<R> f = v.factor(o.x);
    for (uint32_t k = 0; k < o.b; k++) {
        Cx<R> x = times_factor(f.re, f.im, v.cur(o.a + k));
        v.put(o.a + k, x);
        if (ins_flags(o) & 8) v.writeback(o.y + k, &x, 1);
    }
}
template <class K, class V>
__device__ __forceinline__ void exec_clear(const V &v, const Ins &o) {
    typedef typename K::R R;
    Cx<R> z = cx(konst<R>(0.0), konst<R>(0.0));
    for (uint32_t k = 0; k < o.b; k++) {
        v.put(o.a + k, z);
        if (ins_flags(o) & 8) v.writeback(o.y + k, &z, 1);
    }
}

// one row of any kind but a source, its sum kept in `acc` across a destination's run
template <class K, class V>
__device__ __forceinline__ void exec_row(const V &v, const Ins &o, Cx<typename K::R> *acc) {
    // one jump on kind | op << 4 (the program holds no other pairs)
    switch (o.head & 0xff) {
    case K_CONTRIB | 2 << 4: exec_contribution<K, 2>(v, o, acc); break;
    case K_CONTRIB | 3 << 4: exec_contribution<K, 3>(v, o, acc); break;
    case K_CONTRIB | 4 << 4: exec_contribution<K, 4>(v, o, acc); break;
    case K_CONTRIB | 5 << 4: exec_contribution<K, 5>(v, o, acc); break;
    case K_CONTRIB | 6 << 4: exec_contribution<K, 6>(v, o, acc); break;
    case K_PROP | 7 << 4: exec_propagator<K, 7>(v, o); break;
    case K_PROP | 8 << 4: exec_propagator<K, 8>(v, o); break;
    case K_PROP | 9 << 4: exec_propagator<K, 9>(v, o); break;
    case K_CLOSURE | 11 << 4: exec_closure<K>(v, o, acc); break;
    case K_IDENTITY | 10 << 4: exec_identity<K>(v, o); break;
    case K_CLEAR | 1 << 4: exec_clear<K>(v, o); break;
    default: break;
    }
}

// forms (f64) of point i from the external momenta: 0.0 + c0 p + c1 p + ..., in term order
// (reference: recurrence_runner.cu:747-764)
__device__ __forceinline__ void fill_forms(const RunArgs &a, size_t i) {
    for (uint32_t f = 0; f < a.forms; f++) {
        uint32_t first = a.form_terms[2 * f], n = a.form_terms[2 * f + 1];
        for (int k = 0; k < 4; k++) {
            double v = 0.0;
            for (uint32_t t = 0; t < n; t++) {
                double term = __dmul_rn(a.coefficients[first + t],
                                        a.external[((size_t)a.term_slots[first + t] * 4 + k) * a.points + i]);
                v = t == 0 ? __dadd_rn(0.0, term) : __dadd_rn(v, term);
            }
            a.mom[(f * 4 + k) * a.ld + i] = v;
        }
    }
}

// the sources (f64, from the f64 forms and constants), narrowed into the current layout
// (reference: recurrence_runner.cu:769-785)
template <class R>
__device__ __forceinline__ void run_sources(const Ins *ins, uint32_t sources, const RunArgs &a, R *cre, R *cim,
                                            size_t i) {
    for (uint32_t n = 0; n < sources; n++) {
        Ins o = load_ins(ins, n);
        double p[4];
        for (int k = 0; k < 4; k++) p[k] = a.mom[(o.f * 4 + k) * a.ld + i];
        double fr = a.f64[o.x], fi = a.f64[a.factors + o.x], mass = a.s64[o.s];
        W w[4];
        int m = source_values(o.y, mass, p, w);
        for (int k = 0; k < m; k++) {
            double sr = fr * w[k].re - fi * w[k].im, si = fr * w[k].im + fi * w[k].re;
            cre[(o.a + k) * a.ld + i] = narrow<R>(sr);
            cim[(o.a + k) * a.ld + i] = narrow<R>(si);
        }
    }
}

template <class K>
__global__ void __launch_bounds__(256) run_plan(const Ins *__restrict__ ins, uint32_t count, uint32_t sources,
                                                RunArgs a) {
    typedef typename K::R R;
    typedef typename K::Den Den;
    typedef typename K::Amp Amp;
    typedef typename K::Const Const;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.points) return;
    if (a.external) fill_forms(a, i);
    R *cre = (R *)a.cre, *cim = (R *)a.cim;
    run_sources<R>(ins, sources, a, cre, cim, i);
    if (!a.den_is_f64) {
        // the forms into df64 pairs in place (each thread its own point)
        for (uint32_t p = 0; p < 4 * a.forms; p++) {
            size_t at = p * a.ld + i;
            reinterpret_cast<D *>(a.mom)[at] = narrow<D>(a.mom[at]);
        }
    }
    PointView<K> v;
    v.cre = cre;
    v.cim = cim;
    v.are = (Amp *)a.are;
    v.aim = (Amp *)a.aim;
    v.mom = (const Den *)a.mom;
    v.sre = (const Const *)a.kconst;
    v.sim = v.sre + a.scales;
    v.fre = v.sim + a.scales;
    v.fim = v.fre + a.factors;
    v.ld = a.ld;
    v.i = i;
    Cx<R> acc[6];
#pragma unroll
    for (int k = 0; k < 6; k++) acc[k] = cx(konst<R>(0.0), konst<R>(0.0));
    for (uint32_t n = sources; n < count; n++) exec_row<K>(v, load_ins(ins, n), acc);
}

}  // namespace pacuda
