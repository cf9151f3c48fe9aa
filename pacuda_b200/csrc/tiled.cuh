// The on-chip executor: a persistent kernel whose blocks take groups of points; each point's
// currents, amplitudes and forms live in shared-memory slots (schedule.h), a point's lanes run
// the tasks of one dataflow level at a time, and nothing but the external momenta comes in and
// the outputs go out (in the C ABI's mode also the arena's live-in planes in and its written
// planes out).
//
// A block runs P points at once (1 .. 32). A lane of all P points is a group of P adjacent
// threads of one warp (floor(32 / P) groups per warp, the warp's other threads idle), so each
// point has G = warps * floor(32 / P) lanes. The P threads of a group run the same task on
// consecutive points: their instruction fetches are one broadcast, their shared-memory values
// ([slot][P], interleaved) are contiguous, and their global stores cover P consecutive points of
// a plane. All points take the same lane order, so a block's points move through the levels
// together and meet at the block's barrier. A block takes one work item at a time: one plan's
// next P points. An SM runs 1 to 16 such blocks (each with its share of the warps and shared
// memory), which reach their barriers at different times; batch blocks of 1 and 8 points run a
// copy of the levels with that count built in (run_levels over SlotView<K, ABI, NP>).
#pragma once
#include <stdint.h>

#include "arith.cuh"
#include "executor.cuh"
#include "program.h"

namespace pacuda {

struct TiledPlan {
    // the schedule (instructions in the 16-byte form: pack_ins)
    const uint4 *ins;
    const uint32_t *task_first;   // per task, its instructions (tasks + 1 entries)
    const uint32_t *order;        // per level position, its task's (first, end) instructions; lane = position % G
    const uint32_t *level_first;  // levels + 1 entries into order
    uint32_t levels;
    uint32_t cur_slots, amp_slots, forms;
    uint32_t terms;               // reduction terms kept instead of amplitudes (batch mode), or 0
    uint32_t points;              // P points per block
    uint32_t lanes;               // G lanes per point: warps * floor(32 / P)
    uint32_t point_bytes;         // shared memory of one point
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
    const unsigned long long *item_first;  // nplans + 1 prefix sums of work items (a block's points)
    const double *const *external;         // per plan: source-major planes [(leg * 4 + k) * count + i]
    const uint32_t *count;                 // per plan: its points
    double *const *output;                 // per plan: [point][outputs] (batch mode)
    unsigned long long *counter;           // work-item counter (zeroed before the launch)
    // the C ABI's mode (one plan): the arenas in the kind's layout, stride ld
    bool abi;
    void *cre, *cim, *are, *aim;
    const double *mom;                     // uploaded forms (f64 planes), or null
    size_t ld;
    uint32_t const_bytes;                  // shared memory kept for a plan's constants
};

// The on-chip executor's 16-byte instruction: kind | op << 4 | flags << 8 | form 0 << 16 |
// form 1 << 24, then (a, b), (c, s), (x, y) as 16-bit pairs. Every field of a plan whose points fit
// shared memory fits (slots and constant indices below 65536, forms below 256); the host checks.
__device__ __forceinline__ Ins unpack_ins(uint4 w) {
    Ins o;
    o.head = w.x & 0xffff;
    o.f = ((w.x >> 16) & 0xff) | (w.x >> 24) << 16;
    o.a = w.y & 0xffff;
    o.b = w.y >> 16;
    o.c = w.z & 0xffff;
    o.s = w.z >> 16;
    o.x = w.w & 0xffff;
    o.y = w.w >> 16;
    return o;
}

// a hint: the line holding `p` into L1 (no register waits for it)
__device__ __forceinline__ void prefetch_l1(const void *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// a complex value as shared memory holds it: (re, im) side by side, one 8- or 16-byte access
template <class R> struct alignas(2 * sizeof(R)) Pair {
    R re, im;
};

__device__ __forceinline__ double to_f64_value(double x) { return x; }
__device__ __forceinline__ double to_f64_value(D x) { return __dadd_rn((double)x.hi, (double)x.lo); }

// the C ABI's mode: where an item's points write their planes back (thread 0 sets it per item;
// in shared memory so that no lane holds these in registers through its tasks)
struct AbiItem {
    void *cre, *cim;
    size_t ld;
    unsigned long long first;  // the item's first point
    uint32_t count;            // the plan's points
};
static __shared__ AbiItem abi_item;

// NP: the block's points when known at compile time (0: np at run time); with NP a slot's
// address is a shift of its index and its components' addresses constant offsets from it
template <class K, bool ABI, int NP = 0> struct SlotView {
    typedef typename K::R R;
    typedef typename K::Den Den;
    typedef typename K::Amp Amp;
    typedef typename K::Const Const;
    Pair<R> *cur_;        // [slot][points of the region]
    Pair<Amp> *amp_;      // [amplitude slot][points of the region]
    double *term_;        // [reduction term][points] (a schedule that keeps terms)
    const double *tw;     // the reduction's weights
    const Den *mom;
    const Const *sre, *sim, *fre, *fim;  // the plan's constants, in shared memory
    uint32_t np, pw;      // the block's points (interleaved) and this thread's
    static constexpr int kPoints = NP;
    __device__ __forceinline__ uint32_t at(uint32_t slot) const { return NP ? slot * NP + pw : slot * np + pw; }
    // the same view with the addressing of N points per block (valid when np == N)
    template <int N> __device__ __forceinline__ SlotView<K, ABI, N> with_points() const {
        SlotView<K, ABI, N> o;
        o.cur_ = cur_;
        o.amp_ = amp_;
        o.term_ = term_;
        o.tw = tw;
        o.mom = mom;
        o.sre = sre;
        o.sim = sim;
        o.fre = fre;
        o.fim = fim;
        o.np = N;
        o.pw = pw;
        return o;
    }
    __device__ __forceinline__ Cx<R> cur(uint32_t slot) const {
        Pair<R> v = cur_[at(slot)];
        return cx(v.re, v.im);
    }
    __device__ __forceinline__ void put(uint32_t slot, Cx<R> v) const {
        Pair<R> x;
        x.re = v.re;
        x.im = v.im;
        cur_[at(slot)] = x;
    }
    __device__ __forceinline__ Den form(uint32_t f, int k) const { return mom[at(f * 4 + k)]; }
    __device__ __forceinline__ Cx<R> scale(uint32_t s) const { return cx(cast<R>(sre[s]), cast<R>(sim[s])); }
    __device__ __forceinline__ Cx<R> factor(uint32_t x) const { return cx(cast<R>(fre[x]), cast<R>(fim[x])); }
    __device__ __forceinline__ void amp(uint32_t a, Amp &re, Amp &im) const {
        Pair<Amp> v = amp_[at(a)];
        re = v.re;
        im = v.im;
    }
    // a reduction term: weight x fma(re, re, im x im), the resolved reduction's arithmetic
    __device__ __forceinline__ void put_term(uint32_t t, Amp re, Amp im) const {
        double r = to_f64_value(re), i = to_f64_value(im);
        term_[at(t)] = __dmul_rn(__ldg(tw + t), __fma_rn(r, r, __dmul_rn(i, i)));
    }
    __device__ __forceinline__ void put_amp(uint32_t a, Amp re, Amp im) const {
        Pair<Amp> x;
        x.re = re;
        x.im = im;
        amp_[at(a)] = x;
    }
    __device__ __forceinline__ void writeback(uint32_t plane, const Cx<R> *v, int n) const {
        if (ABI) {
            const unsigned long long point = abi_item.first + pw;
            if (point < abi_item.count) {
                R *re = (R *)abi_item.cre, *im = (R *)abi_item.cim;
                const size_t ld = abi_item.ld;
                for (int k = 0; k < n; k++) {
                    re[(plane + k) * ld + point] = v[k].re;
                    im[(plane + k) * ld + point] = v[k].im;
                }
            }
        }
    }
};


// the levels of one item: level 0's sources, then each level's tasks in the lane order, a block
// barrier after each level (views of a compile-time point count address slots without products)
template <class K, class V>
__device__ __forceinline__ void run_levels(const V &v, const TiledPlan &p, double *forms64, uint32_t tl, bool active) {
    typedef typename K::R R;
    typedef typename K::Den Den;
    const uint32_t lanes = p.lanes, levels = p.levels;
    const uint4 *ins = p.ins;
    const uint2 *order = reinterpret_cast<const uint2 *>(p.order);
    for (uint32_t lv = 0; lv < levels; lv++) {
        const uint32_t j0 = __ldg(p.level_first + lv), j1 = active ? __ldg(p.level_first + lv + 1) : 0;
        if (lv == 0) {
            for (uint32_t j = j0 + tl; j < j1; j += lanes) {
                uint2 r = __ldg(order + j);
                // sources: f64 wavefunctions from the f64 forms and constants, narrowed
                for (uint32_t n = r.x; n < r.y; n++) {
                    Ins o = unpack_ins(__ldg(ins + n));
                    double mom[4];
                    for (int c = 0; c < 4; c++) mom[c] = forms64[v.at(o.f * 4 + c)];
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
            }
        } else {
            // the next task's range is fetched while a task runs
            // (the order arrays end with a lane count's worth of padding and the instructions
            // with one padding instruction, so these fetches need no bounds test). In blocks of one
            // point every lane fetches its own instructions, and five blocks' shared memory leaves
            // L1 little room for them: once a task's first row has run, the next task's range has
            // arrived, and that task's first and last instruction lines are prefetched into L1
            // while the rest of this one runs.
            uint32_t j = j0 + tl;
            uint2 r = j < j1 ? __ldg(order + j) : make_uint2(0, 0);
            while (j < j1) {
                uint2 cur = r;
                j += lanes;
                r = __ldg(order + j);
                if (cur.x == cur.y) continue;
                Cx<R> acc[6];
#pragma unroll
                for (int c = 0; c < 6; c++) acc[c] = cx(konst<R>(0.0), konst<R>(0.0));
                // each next instruction is fetched while its predecessor runs
                uint4 next = __ldg(ins + cur.x);
                for (uint32_t n = cur.x; n < cur.y; n++) {
                    const uint4 now = next;
                    next = __ldg(ins + n + 1);
                    exec_row<K>(v, unpack_ins(now), acc);
                    if (V::kPoints == 1 && n == cur.x) {
                        prefetch_l1(ins + r.x);
                        prefetch_l1(ins + (r.y > r.x ? r.y - 1 : r.x));
                    }
                }
            }
        }
        __syncthreads();
        if (lv == 0 && !is_f64<Den>::value) {
            // the forms into df64 pairs, in place
            if (active)
                for (uint32_t q = tl; q < 4 * p.forms; q += lanes) {
                    uint32_t at = v.at(q);
                    reinterpret_cast<D *>(forms64)[at] = narrow<D>(forms64[at]);
                }
            __syncthreads();
        }
    }
}

// ABI: the C ABI's mode (arena in and out) or a batch's (outputs only)
template <class K, bool ABI>
__global__ void __launch_bounds__(512, 1) run_tiled(TiledLaunch L) {
    typedef typename K::R R;
    typedef typename K::Den Den;
    typedef typename K::Amp Amp;
    typedef typename K::Const Const;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ unsigned long long next_item;
    const unsigned long long total = L.item_first[L.nplans];
    while (true) {
        if (threadIdx.x == 0) next_item = atomicAdd(L.counter, 1ull);
        __syncthreads();
        const unsigned long long item = next_item;
        if (item >= total) break;
        uint32_t k = 0;
        while (item >= L.item_first[k + 1]) k++;
        const TiledPlan &p = L.plans[k];
        const uint32_t np = p.points, lanes = p.lanes;
        if (ABI && threadIdx.x == 0) {
            abi_item.cre = L.cre;
            abi_item.cim = L.cim;
            abi_item.ld = L.ld;
            abi_item.first = (item - L.item_first[k]) * np;
            abi_item.count = L.count[k];
        }
        // the plan's constants (the kind's layout) into shared memory
        Const *consts = (Const *)smem;
        const uint32_t nconst = 2 * (p.scales + p.factors);
        for (uint32_t c = threadIdx.x; c < nconst; c += blockDim.x) consts[c] = ((const Const *)p.kconst)[c];
        // this thread: lane tl of point pw; the threads of no group only meet the barriers
        const uint32_t groups = 32 / np, x = threadIdx.x & 31, q = x / np, pw = x - q * np;
        const uint32_t tl = (threadIdx.x >> 5) * groups + q;
        const bool active = q < groups;
        SlotView<K, ABI> v;
        v.cur_ = (Pair<R> *)(smem + L.const_bytes);
        v.amp_ = (Pair<Amp> *)(v.cur_ + (size_t)p.cur_slots * np);
        v.term_ = (double *)(v.amp_ + (size_t)p.amp_slots * np);
        v.tw = p.red_weights;
        double *forms64 = v.term_ + (size_t)p.terms * np;
        v.mom = (const Den *)forms64;
        v.sre = consts;
        v.sim = v.sre + p.scales;
        v.fre = v.sim + p.scales;
        v.fim = v.fre + p.factors;
        v.np = np;
        v.pw = pw;
        if (active) {
            const uint32_t count = L.count[k];
            const size_t mine = (size_t)(item - L.item_first[k]) * np + pw;
            const size_t point = mine < count ? mine : count - 1;  // padding points redo the last point, unwritten
            // forms, f64: from the external momenta (0.0 + c0 p + c1 p + ..., in term order), or
            // the uploaded planes
            for (uint32_t q = tl; q < 4 * p.forms; q += lanes) {
                uint32_t f = q >> 2, c = q & 3;
                double val;
                if (ABI && L.mom) {
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
                forms64[q * np + pw] = val;
            }
            // the C ABI's mode: live-in currents and every amplitude from the global arena
            if (ABI) {
                for (uint32_t j = 0; j < p.nloads; j++) {
                    uint32_t plane = __ldg(p.loads + 3 * j), slot = __ldg(p.loads + 3 * j + 1), n = __ldg(p.loads + 3 * j + 2);
                    for (uint32_t c = tl; c < n; c += lanes)
                        v.put(slot + c, cx(((const R *)L.cre)[(plane + c) * L.ld + point],
                                           ((const R *)L.cim)[(plane + c) * L.ld + point]));
                }
                for (uint32_t a = tl; a < p.amp_slots; a += lanes) {
                    uint32_t plane = __ldg(p.amp_planes + a);
                    v.put_amp(a, ((const Amp *)L.are)[plane * L.ld + point], ((const Amp *)L.aim)[plane * L.ld + point]);
                }
            } else {
                for (uint32_t a = tl; a < p.amp_slots; a += lanes) v.put_amp(a, konst<Amp>(0.0), konst<Amp>(0.0));
                // a term whose amplitude no closure makes: the term of a zero amplitude
                for (uint32_t t = tl; t < p.terms; t += lanes) v.put_term(t, konst<Amp>(0.0), konst<Amp>(0.0));
            }
        }
        __syncthreads();  // the constants, forms and live-in values are in
        // batches of one point per block (six-leg plans, gg>ggg) and of eight (the 5-leg quark
        // plans at two blocks per SM) run a copy of the levels with that count built in; in the C
        // ABI's kernel more copies of the levels cost registers
        if (!ABI && np == 1)
            run_levels<K>(v.template with_points<1>(), p, forms64, tl, active);
        else if (!ABI && np == 8)
            run_levels<K>(v.template with_points<8>(), p, forms64, tl, active);
        else
            run_levels<K>(v, p, forms64, tl, active);
        if (ABI) {
            // (the point again from the item: nothing of it stays in registers through the levels)
            const unsigned long long at = abi_item.first + pw;
            if (active && at < abi_item.count)
                for (uint32_t a = tl; a < p.amp_slots; a += lanes) {
                    uint32_t plane = __ldg(p.amp_planes + a);
                    Amp re, im;
                    v.amp(a, re, im);
                    ((Amp *)L.are)[plane * L.ld + at] = re;
                    ((Amp *)L.aim)[plane * L.ld + at] = im;
                }
        } else if (active && (size_t)(item - L.item_first[k]) * np + pw < L.count[k]) {
            // the resolved reduction from zero: out[point][o] = 0 + w fma(re, re, im im) + ...
            const size_t point = (size_t)(item - L.item_first[k]) * np + pw;
            double *out = L.output[k] + point * p.outputs;
            for (uint32_t o = tl; p.terms && o < p.outputs; o += lanes) {
                double acc = 0.0;
                for (uint32_t j = __ldg(p.red_offsets + o), e = __ldg(p.red_offsets + o + 1); j < e; j++)
                    acc = __dadd_rn(acc, v.term_[v.at(j)]);
                out[o] = acc;
            }
            for (uint32_t o = tl; !p.terms && o < p.outputs; o += lanes) {
                double acc = 0.0;
                for (uint32_t j = __ldg(p.red_offsets + o), e = __ldg(p.red_offsets + o + 1); j < e; j++) {
                    uint32_t s = __ldg(p.red_slots + j);
                    double re = 0.0, im = 0.0;
                    if (s != ~0u) {
                        Amp ar, ai;
                        v.amp(s, ar, ai);
                        re = to_f64_value(ar);
                        im = to_f64_value(ai);
                    }
                    acc = __dadd_rn(acc, __dmul_rn(__ldg(p.red_weights + j), __fma_rn(re, re, __dmul_rn(im, im))));
                }
                out[o] = acc;
            }
        }
        __syncthreads();  // the block's shared memory is free for the next item
    }
}

}  // namespace pacuda
