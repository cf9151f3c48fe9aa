// The on-chip executor: a persistent kernel whose warps take groups of points; each point's
// currents, amplitudes and forms live in shared-memory slots (schedule.h), the lanes of a point
// run the tasks of one dataflow level at a time, and nothing but the external momenta comes in
// and the outputs go out (in the C ABI's mode also the arena's live-in planes in and its written
// planes out).
//
// A warp holds P points (P a power of two) and gives each L = 32 / P lanes. Shared memory per
// warp: [slot][P] currents (re, im), [amplitude slot][P] amplitudes, [form * 4 + k][P] forms.
#pragma once
#include <stdint.h>

#include "arith.cuh"
#include "executor.cuh"
#include "program.h"

namespace pacuda {

struct TiledPlan {
    // the schedule
    const Ins *ins;
    const uint32_t *task_first;
    const uint32_t *level_first;
    uint32_t levels;
    uint32_t cur_slots, amp_slots, forms;
    uint32_t log_p;               // P = 1 << log_p points per warp
    uint32_t warp_bytes;          // shared memory of one warp
    // constants: f64 (sources), the kind's layout (rows)
    const double *s64, *f64;
    const void *kconst;
    uint32_t scales, factors;
    // forms from external momenta (source-major planes of `points` values per point)
    const uint32_t *form_terms, *term_slots;
    const double *coefficients;
    // the resolved reduction (batch mode): outputs, offsets into (slot, weight) pairs
    const uint32_t *red_offsets, *red_slots;
    const double *red_weights;
    uint32_t outputs;
    // the C ABI's mode: live-in current planes, the amplitude slots' planes
    const uint32_t *loads;
    uint32_t nloads;
    const uint32_t *amp_planes;
};

// one launch: plans (a batch) and, per plan, its points
struct TiledLaunch {
    const TiledPlan *plans;
    uint32_t nplans;
    const unsigned long long *item_first;  // nplans + 1 prefix sums of work items (point groups)
    const double *const *external;         // per plan: source-major planes [(leg * 4 + k) * count + i]
    const uint32_t *count;                 // per plan: its points
    double *const *output;                 // per plan: [point][outputs] (batch mode)
    unsigned long long *counter;           // work-item counter (zeroed before the launch)
    // the C ABI's mode (one plan): the arenas in the kind's layout, stride ld
    bool abi;
    void *cre, *cim, *are, *aim;
    const double *mom;                     // uploaded forms (f64 planes), or null
    size_t ld;
};

template <class K> struct SlotView {
    typedef typename K::R R;
    typedef typename K::Den Den;
    typedef typename K::Amp Amp;
    typedef typename K::Const Const;
    R *cre, *cim;
    Amp *are, *aim;
    const Den *mom;
    const Const *sre, *sim, *fre, *fim;
    uint32_t log_p, pw;
    // write-back to the global arena (the C ABI's mode), else null
    R *gre, *gim;
    size_t ld, point;
    __device__ __forceinline__ uint32_t at(uint32_t slot) const { return (slot << log_p) + pw; }
    __device__ __forceinline__ Cx<R> cur(uint32_t slot) const { return cx(cre[at(slot)], cim[at(slot)]); }
    __device__ __forceinline__ void put(uint32_t slot, Cx<R> v) const {
        cre[at(slot)] = v.re;
        cim[at(slot)] = v.im;
    }
    __device__ __forceinline__ Den form(uint32_t f, int k) const { return mom[at(f * 4 + k)]; }
    __device__ __forceinline__ Cx<R> scale(uint32_t s) const { return cx(cast<R>(sre[s]), cast<R>(sim[s])); }
    __device__ __forceinline__ Cx<R> factor(uint32_t x) const { return cx(cast<R>(fre[x]), cast<R>(fim[x])); }
    __device__ __forceinline__ void amp(uint32_t a, Amp &re, Amp &im) const {
        re = are[at(a)];
        im = aim[at(a)];
    }
    __device__ __forceinline__ void put_amp(uint32_t a, Amp re, Amp im) const {
        are[at(a)] = re;
        aim[at(a)] = im;
    }
    __device__ __forceinline__ void writeback(uint32_t plane, const Cx<R> *v, int n) const {
        if (!gre) return;
        for (int k = 0; k < n; k++) {
            gre[(plane + k) * ld + point] = v[k].re;
            gim[(plane + k) * ld + point] = v[k].im;
        }
    }
};

__device__ __forceinline__ double to_f64_value(double x) { return x; }
__device__ __forceinline__ double to_f64_value(D x) { return __dadd_rn((double)x.hi, (double)x.lo); }

template <class K>
__global__ void __launch_bounds__(512, 1) run_tiled(TiledLaunch L) {
    typedef typename K::R R;
    typedef typename K::Den Den;
    typedef typename K::Amp Amp;
    typedef typename K::Const Const;
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t max_bytes = 0;
    for (uint32_t k = 0; k < L.nplans; k++) max_bytes = max(max_bytes, L.plans[k].warp_bytes);
    unsigned char *base = smem + (size_t)warp * max_bytes;
    const unsigned long long total = L.item_first[L.nplans];
    while (true) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(L.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= total) break;
        uint32_t k = 0;
        while (item >= L.item_first[k + 1]) k++;
        const TiledPlan &p = L.plans[k];
        const uint32_t log_p = p.log_p, lanes = 32u >> log_p;
        const uint32_t pw = lane / lanes, tl = lane % lanes;
        const uint32_t count = L.count[k];
        const size_t first = (size_t)(item - L.item_first[k]) << log_p;
        const bool valid = first + pw < count;
        const size_t point = valid ? first + pw : count - 1;  // padding lanes redo the last point, unwritten
        SlotView<K> v;
        v.cre = (R *)base;
        v.cim = v.cre + ((size_t)p.cur_slots << log_p);
        v.are = (Amp *)(v.cim + ((size_t)p.cur_slots << log_p));
        v.aim = v.are + ((size_t)p.amp_slots << log_p);
        double *forms64 = (double *)(v.aim + ((size_t)p.amp_slots << log_p));
        v.mom = (const Den *)forms64;
        v.sre = (const Const *)p.kconst;
        v.sim = v.sre + p.scales;
        v.fre = v.sim + p.scales;
        v.fim = v.fre + p.factors;
        v.log_p = log_p;
        v.pw = pw;
        v.gre = (L.abi && valid) ? (R *)L.cre : nullptr;
        v.gim = (R *)L.cim;
        v.ld = L.ld;
        v.point = point;
        // forms, f64: from the external momenta (0.0 + c0 p + c1 p + ..., in term order), or the
        // uploaded planes
        for (uint32_t q = tl; q < 4 * p.forms; q += lanes) {
            uint32_t f = q >> 2, c = q & 3;
            double val;
            if (L.mom) {
                val = L.mom[(size_t)q * L.ld + point];
            } else {
                uint32_t t0 = __ldg(p.form_terms + 2 * f), n = __ldg(p.form_terms + 2 * f + 1);
                const double *ext = L.external[k];
                val = 0.0;
                for (uint32_t t = 0; t < n; t++) {
                    double term = __dmul_rn(__ldg(p.coefficients + t0 + t),
                                            ext[((size_t)__ldg(p.term_slots + t0 + t) * 4 + c) * count + point]);
                    val = t == 0 ? __dadd_rn(0.0, term) : __dadd_rn(val, term);
                }
            }
            forms64[(q << log_p) + pw] = val;
        }
        // the C ABI's mode: live-in currents and every amplitude from the global arena
        if (L.abi) {
            for (uint32_t j = 0; j < p.nloads; j++) {
                uint32_t plane = __ldg(p.loads + 3 * j), slot = __ldg(p.loads + 3 * j + 1), n = __ldg(p.loads + 3 * j + 2);
                for (uint32_t c = tl; c < n; c += lanes) {
                    v.cre[((slot + c) << log_p) + pw] = ((const R *)L.cre)[(plane + c) * L.ld + point];
                    v.cim[((slot + c) << log_p) + pw] = ((const R *)L.cim)[(plane + c) * L.ld + point];
                }
            }
            for (uint32_t a = tl; a < p.amp_slots; a += lanes) {
                uint32_t plane = __ldg(p.amp_planes + a);
                v.are[(a << log_p) + pw] = ((const Amp *)L.are)[plane * L.ld + point];
                v.aim[(a << log_p) + pw] = ((const Amp *)L.aim)[plane * L.ld + point];
            }
        } else {
            for (uint32_t a = tl; a < p.amp_slots; a += lanes) {
                v.are[(a << log_p) + pw] = konst<Amp>(0.0);
                v.aim[(a << log_p) + pw] = konst<Amp>(0.0);
            }
        }
        __syncwarp();
        for (uint32_t lv = 0; lv < p.levels; lv++) {
            uint32_t t0 = __ldg(p.level_first + lv), t1 = __ldg(p.level_first + lv + 1);
            for (uint32_t t = t0 + tl; t < t1; t += lanes) {
                uint32_t i0 = __ldg(p.task_first + t), i1 = __ldg(p.task_first + t + 1);
                if (lv == 0) {
                    // sources: f64 wavefunctions from the f64 forms and constants, narrowed
                    for (uint32_t n = i0; n < i1; n++) {
                        Ins o = load_ins(p.ins, n);
                        double mom[4];
                        for (int c = 0; c < 4; c++) mom[c] = forms64[((o.f * 4 + c) << log_p) + pw];
                        double fr = __ldg(p.f64 + o.x), fi = __ldg(p.f64 + p.factors + o.x), mass = __ldg(p.s64 + o.s);
                        W w[4];
                        int m = source_values(o.y, mass, mom, w);
                        Cx<R> vals[4];
                        for (int c = 0; c < m; c++) {
                            double sr = fr * w[c].re - fi * w[c].im, si = fr * w[c].im + fi * w[c].re;
                            vals[c] = cx(narrow<R>(sr), narrow<R>(si));
                            v.put(o.a + c, vals[c]);
                        }
                        if (ins_flags(o) & 8) v.writeback(o.c, vals, m);
                    }
                } else {
                    Cx<R> acc[6];
#pragma unroll
                    for (int c = 0; c < 6; c++) acc[c] = cx(konst<R>(0.0), konst<R>(0.0));
                    for (uint32_t n = i0; n < i1; n++) exec_row<K>(v, load_ins(p.ins, n), acc);
                }
            }
            __syncwarp();
            if (lv == 0 && sizeof(Den) == 8 && !is_f64<Den>::value) {
                // the forms into df64 pairs, in place
                for (uint32_t q = tl; q < 4 * p.forms; q += lanes) {
                    uint32_t at = (q << log_p) + pw;
                    reinterpret_cast<D *>(forms64)[at] = narrow<D>(forms64[at]);
                }
                __syncwarp();
            }
        }
        if (L.abi) {
            if (valid)
                for (uint32_t a = tl; a < p.amp_slots; a += lanes) {
                    uint32_t plane = __ldg(p.amp_planes + a);
                    ((Amp *)L.are)[plane * L.ld + point] = v.are[(a << log_p) + pw];
                    ((Amp *)L.aim)[plane * L.ld + point] = v.aim[(a << log_p) + pw];
                }
        } else if (valid) {
            // the resolved reduction from zero: out[point][o] = 0 + w fma(re, re, im im) + ...
            double *out = L.output[k] + point * p.outputs;
            for (uint32_t o = tl; o < p.outputs; o += lanes) {
                double acc = 0.0;
                for (uint32_t j = __ldg(p.red_offsets + o), e = __ldg(p.red_offsets + o + 1); j < e; j++) {
                    uint32_t s = __ldg(p.red_slots + j);
                    double re = 0.0, im = 0.0;
                    if (s != ~0u) {
                        re = to_f64_value(v.are[(s << log_p) + pw]);
                        im = to_f64_value(v.aim[(s << log_p) + pw]);
                    }
                    acc = __dadd_rn(acc, __dmul_rn(__ldg(p.red_weights + j), __fma_rn(re, re, __dmul_rn(im, im))));
                }
                out[o] = acc;
            }
        }
        __syncwarp();
    }
}

}  // namespace pacuda
