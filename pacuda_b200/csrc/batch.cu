// The batched, device-resident entry points (include/pacuda_b200.h): plans compiled once,
// batches of plans evaluated in one persistent launch of the on-chip executor.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "../../include/pacuda_b200.h"
#include "tiled.cuh"
#include "tiled_host.h"

using namespace pacuda;

namespace {

const char *const kTag = "pacuda-b200";

bool failed(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return false;
    fprintf(stderr, "%s: %s: %s\n", kTag, what, cudaGetErrorString(e));
    return true;
}

template <class T> bool to_device(T **dst, const T *src, size_t n) {
    if (failed(cudaMalloc((void **)dst, std::max<size_t>(1, n) * sizeof(T)), "allocation")) return false;
    return n == 0 || !failed(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice), "copy");
}

int device_sms() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

}  // namespace

struct pacuda_b200_plan {
    int kernel = PACMAN_RECURRENCE_KERNEL_F64;
    Program prog;
    TiledDevice tiled;
    uint32_t forms = 0, scales = 0, factors = 0, outputs = 0;
    double *consts = nullptr;  // f64 scales re, im, factors re, im; then the kind's layout
    uint32_t *terms = nullptr;  // form_terms (2 per form), then term_slots
    double *coefficients = nullptr;
    uint32_t *red_offsets = nullptr, *red_slots = nullptr;
    double *red_weights = nullptr;
    uint32_t points = 1;      // points per block (a point has the block's threads / points lanes)
    size_t point_bytes = 0;
    bool fixed = false;
};

// The plans of one launch: those that run with the same blocks per SM.
struct LaunchGroup {
    std::vector<uint32_t> plans;  // indices into the batch's plans
    int blocks = 1, threads = 0;
    size_t smem = 0, const_bytes = 0;
    size_t at = 0;                // its section of the descriptor block
};

struct pacuda_b200_batch {
    std::vector<pacuda_b200_plan *> plans;
    std::vector<const double *> external;
    std::vector<uint32_t> count;
    std::vector<double *> output;
    std::vector<uint32_t> points;      // per plan: its points per block in this batch's launch
    std::vector<int> plan_blocks;      // per plan: its blocks per SM (0: the batch's)
    int blocks = 1;                    // the batch's blocks per SM (tiled_host.h kBlockChoices); 0: automatic
    // one launch per group; the descriptor block holds a section per group:
    // TiledPlan[n] | item_first[n + 1] | external[n] | output[n] | count[n] | counter
    std::vector<LaunchGroup> groups;
    unsigned char *host = nullptr, *device = nullptr;
    size_t bytes = 0;
    int sms = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t copied = nullptr;  // recorded after each run's descriptor copy
};

namespace {

void fill_plan(const pacuda_b200_plan *p, TiledPlan &d, uint32_t points, int blocks = 1) {
    memset(&d, 0, sizeof d);
    describe(p->tiled, p->forms, points, p->point_bytes, d, blocks);
    d.s64 = p->consts;
    d.f64 = p->consts + 2 * p->scales;
    d.kconst = p->consts + 2 * (p->scales + p->factors);
    d.scales = p->scales;
    d.factors = p->factors;
    d.form_terms = p->terms;
    d.term_slots = p->terms + 2 * p->forms;
    d.coefficients = p->coefficients;
    d.red_offsets = p->red_offsets;
    d.red_slots = p->red_slots;
    d.red_weights = p->red_weights;
    d.outputs = p->outputs;
}

struct Offsets {
    size_t plans, items, external, output, count, counter, total;
};
Offsets layout(size_t n) {
    Offsets o;
    o.plans = 0;
    o.items = (o.plans + n * sizeof(TiledPlan) + 15) / 16 * 16;
    o.external = (o.items + (n + 1) * 8 + 15) / 16 * 16;
    o.output = o.external + n * 8;
    o.count = o.output + n * 8;
    o.counter = (o.count + n * 4 + 15) / 16 * 16;
    o.total = o.counter + 16;
    return o;
}

// blocks per SM chosen without timing (tiled_auto_blocks)
int auto_blocks(const pacuda_b200_plan *p) {
    return tiled_auto_blocks(p->kernel, p->point_bytes, tiled_const_bytes(p->scales, p->factors));
}

// The groups and the host block from the batch's current choices: each group's shared memory and
// warps, each plan's points per block. The block is allocated again only when its size changes.
bool prepare(pacuda_b200_batch *b) {
    const size_t n = b->plans.size();
    const int kernel = b->plans[0]->kernel;
    b->plan_blocks.resize(n, 0);
    b->groups.clear();
    for (size_t k = 0; k < n; k++) {
        int blocks = b->plan_blocks[k] ? b->plan_blocks[k] : b->blocks ? b->blocks : auto_blocks(b->plans[k]);
        size_t g = 0;
        while (g < b->groups.size() && b->groups[g].blocks != blocks) g++;
        if (g == b->groups.size()) {
            b->groups.emplace_back();
            b->groups.back().blocks = blocks;
        }
        b->groups[g].plans.push_back((uint32_t)k);
    }
    size_t bytes = 0;
    for (LaunchGroup &g : b->groups) {
        g.at = bytes;
        bytes += layout(g.plans.size()).total;
    }
    if (!b->host || bytes != b->bytes) {
        cudaFreeHost(b->host);
        cudaFree(b->device);
        b->host = nullptr;
        b->device = nullptr;
        b->bytes = bytes;
        if (failed(cudaMallocHost((void **)&b->host, b->bytes), "pinned descriptors") ||
            failed(cudaMalloc((void **)&b->device, b->bytes), "descriptors"))
            return false;
    }
    memset(b->host, 0, b->bytes);
    b->points.assign(n, 0);
    for (LaunchGroup &g : b->groups) {
        const size_t m = g.plans.size();
        Offsets o = layout(m);
        unsigned char *base = b->host + g.at;
        TiledPlan *plans = (TiledPlan *)(base + o.plans);
        unsigned long long *items = (unsigned long long *)(base + o.items);
        g.threads = tiled_threads(kernel, g.blocks);
        g.const_bytes = 0;
        for (uint32_t k : g.plans)
            g.const_bytes = std::max(g.const_bytes, tiled_const_bytes(b->plans[k]->scales, b->plans[k]->factors));
        size_t room = tiled_max_smem(kernel, g.blocks);
        if (room <= g.const_bytes) {
            fprintf(stderr, "%s: the plans' constants do not fit a block's shared memory\n", kTag);
            return false;
        }
        size_t max_smem = room - g.const_bytes;
        g.smem = 0;
        items[0] = 0;
        for (size_t j = 0; j < m; j++) {
            const uint32_t k = g.plans[j];
            pacuda_b200_plan *p = b->plans[k];
            uint32_t most = tiled_max_points(p->point_bytes, g.threads, max_smem);
            if (!most || p->tiled.threads != tiled_threads(kernel)) {
                fprintf(stderr, "%s: a plan's point does not fit a block's shared memory\n", kTag);
                return false;
            }
            // the plan's choice where it fits this launch, else the default for it
            uint32_t per = tiled_points_fit(p->points, p->point_bytes, g.threads, max_smem)
                               ? p->points
                               : tiled_default_points(p->point_bytes, g.threads, max_smem);
            b->points[k] = per;
            fill_plan(p, plans[j], per, g.blocks);
            g.smem = std::max<size_t>(g.smem, (size_t)per * p->point_bytes);
            items[j + 1] = items[j] + (b->count[k] + per - 1) / per;
            ((const double **)(base + o.external))[j] = b->external[k];
            ((double **)(base + o.output))[j] = b->output[k];
            ((uint32_t *)(base + o.count))[j] = b->count[k];
        }
        g.smem += g.const_bytes;
    }
    return true;
}

TiledLaunch launch_args(const pacuda_b200_batch *b, const LaunchGroup &g) {
    const size_t m = g.plans.size();
    Offsets o = layout(m);
    unsigned char *base = b->device + g.at;
    TiledLaunch L;
    memset(&L, 0, sizeof L);
    L.plans = (const TiledPlan *)(base + o.plans);
    L.nplans = (uint32_t)m;
    L.item_first = (const unsigned long long *)(base + o.items);
    L.external = (const double *const *)(base + o.external);
    L.output = (double *const *)(base + o.output);
    L.count = (const uint32_t *)(base + o.count);
    L.counter = (unsigned long long *)(base + o.counter);
    L.abi = false;
    L.const_bytes = (uint32_t)g.const_bytes;
    return L;
}

int launch(pacuda_b200_batch *b, cudaStream_t s) {
    if (failed(cudaMemcpyAsync(b->device, b->host, b->bytes, cudaMemcpyHostToDevice, s), "descriptors"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    // (not while capturing: the graph's copy reads the block when it is replayed)
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &capturing);
    if (capturing == cudaStreamCaptureStatusNone && b->copied && failed(cudaEventRecord(b->copied, s), "event"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    for (const LaunchGroup &g : b->groups)
        if (!launch_tiled(b->plans[0]->kernel, launch_args(b, g), g.threads, g.smem, b->sms * g.blocks, s) ||
            failed(cudaGetLastError(), "launch"))
            return PACMAN_RECURRENCE_DEVICE_ERROR;
    return PACMAN_RECURRENCE_OK;
}

// the shared memory a block has for one plan's points
size_t point_smem(const pacuda_b200_plan *p) {
    return tiled_max_smem(p->kernel) - tiled_const_bytes(p->scales, p->factors);
}

// the default points per block (tiled_default_points)
uint32_t default_points(const pacuda_b200_plan *p) {
    uint32_t np = tiled_default_points(p->point_bytes, tiled_threads(p->kernel), point_smem(p));
    return np ? np : 1u;
}

}  // namespace

extern "C" pacuda_b200_plan *pacuda_b200_plan_create(const pacman_recurrence_call *c, const uint32_t *offsets,
                                                     const uint32_t *planes, const double *weights, uint32_t outputs,
                                                     uint32_t kernel) {
    if (!c || c->abi_version != PACMAN_RECURRENCE_ABI || c->struct_size != sizeof(pacman_recurrence_call) ||
        !c->words || (kernel > PACMAN_RECURRENCE_KERNEL_MIXED64 && kernel != PACUDA_B200_KERNEL_F64_FMA) || !offsets || (offsets[outputs] && (!planes || !weights)) ||
        (c->scale_count && (!c->scale_re || !c->scale_im)) || (c->factor_count && (!c->factor_re || !c->factor_im)) ||
        !c->form_terms || (c->term_count && (!c->term_slots || !c->term_coefficients))) {
        fprintf(stderr, "%s: plan_create: an invalid call description\n", kTag);
        return nullptr;
    }
    uint32_t forms = c->momentum_planes / 4;
    for (uint32_t f = 0; f < forms; f++)
        if (c->form_terms[2 * f] > c->term_count || c->form_terms[2 * f + 1] > c->term_count - c->form_terms[2 * f]) {
            fprintf(stderr, "%s: plan_create: a form's terms outside the term table\n", kTag);
            return nullptr;
        }
    for (uint32_t t = 0; t < c->term_count; t++)
        if (c->term_slots[t] >= c->external_count) {
            fprintf(stderr, "%s: plan_create: a term names a leg outside the external momenta\n", kTag);
            return nullptr;
        }
    for (uint32_t o = 0; o < outputs; o++)
        if (offsets[o] > offsets[o + 1]) return nullptr;
    for (uint32_t k = 0; k < offsets[outputs]; k++)
        if (planes[k] >= c->amplitude_planes) {
            fprintf(stderr, "%s: plan_create: a reduction plane outside the amplitudes\n", kTag);
            return nullptr;
        }
    auto *p = new pacuda_b200_plan();
    p->kernel = (int)kernel;
    Limits lim{c->current_planes, c->amplitude_planes, forms, c->scale_count, c->factor_count};
    BuildError e = build_program(c->words, c->word_count, c->width, true, lim, p->prog);
    if (e.status) {
        fprintf(stderr, "%s: plan_create: %s\n", kTag, e.message.c_str());
        delete p;
        return nullptr;
    }
    if (!p->prog.reads_before_write.empty()) {
        fprintf(stderr, "%s: plan_create: the plan reads %zu current planes before writing them\n", kTag,
                p->prog.reads_before_write.size());
        delete p;
        return nullptr;
    }
    if (!build_schedule(p->prog, c->current_planes, c->amplitude_planes, p->tiled.host)) {
        fprintf(stderr, "%s: plan_create: %s\n", kTag, p->tiled.host.why.c_str());
        delete p;
        return nullptr;
    }
    // the plan only reduces its amplitudes: where it can, keep each amplitude's term instead
    use_terms(p->tiled.host, offsets, planes, outputs, c->amplitude_planes);
    p->forms = forms;
    p->scales = c->scale_count;
    p->factors = c->factor_count;
    p->outputs = outputs;
    // constants: f64, then the kind's layout (df64 pairs unless f64)
    size_t nc = 2 * ((size_t)c->scale_count + c->factor_count);
    std::vector<double> k(2 * nc + 1, 0.0);
    for (uint32_t i = 0; i < c->scale_count; i++) { k[i] = c->scale_re[i]; k[c->scale_count + i] = c->scale_im[i]; }
    double *f = k.data() + 2 * c->scale_count;
    for (uint32_t i = 0; i < c->factor_count; i++) { f[i] = c->factor_re[i]; f[c->factor_count + i] = c->factor_im[i]; }
    for (size_t i = 0; i < nc; i++) {
        if (kernel == PACMAN_RECURRENCE_KERNEL_F64 || kernel == PACUDA_B200_KERNEL_F64_FMA) {
            k[nc + i] = k[i];
        } else {
            float hi = (float)k[i], lo = (float)(k[i] - (double)hi);
            memcpy(&k[nc + i], &hi, 4);
            memcpy((char *)&k[nc + i] + 4, &lo, 4);
        }
    }
    std::vector<uint32_t> terms(c->form_terms, c->form_terms + 2 * forms);
    terms.insert(terms.end(), c->term_slots, c->term_slots + c->term_count);
    std::vector<uint32_t> slots(offsets[outputs]);
    for (uint32_t j = 0; j < offsets[outputs]; j++) slots[j] = p->tiled.host.amp_slot_of[planes[j]];
    bool ok = to_device(&p->consts, k.data(), k.size()) && to_device(&p->terms, terms.data(), terms.size()) &&
              to_device(&p->coefficients, c->term_coefficients, c->term_count) &&
              to_device(&p->red_offsets, offsets, (size_t)outputs + 1) &&
              to_device(&p->red_slots, slots.data(), slots.size()) &&
              to_device(&p->red_weights, weights, offsets[outputs]) && upload_schedule(p->tiled, tiled_threads(p->kernel), 0) &&
              !failed(cudaDeviceSynchronize(), "plan upload");
    if (!ok) {
        if (!p->tiled.host.why.empty()) fprintf(stderr, "%s: plan_create: %s\n", kTag, p->tiled.host.why.c_str());
        pacuda_b200_plan_destroy(p);
        return nullptr;
    }
    p->point_bytes = tiled_point_bytes(p->tiled.host, forms, p->kernel);
    p->points = default_points(p);
    return p;
}

extern "C" void pacuda_b200_plan_destroy(pacuda_b200_plan *p) {
    if (!p) return;
    p->tiled.release();
    cudaFree(p->consts);
    cudaFree(p->terms);
    cudaFree(p->coefficients);
    cudaFree(p->red_offsets);
    cudaFree(p->red_slots);
    cudaFree(p->red_weights);
    delete p;
}

extern "C" uint64_t pacuda_b200_plan_flops(const pacuda_b200_plan *p) { return p ? p->prog.flops : 0; }

extern "C" int pacuda_b200_plan_set_lanes_per_point(pacuda_b200_plan *p, uint32_t lanes) {
    if (!p) return PACMAN_RECURRENCE_INVALID;
    if (lanes == 0) {
        p->fixed = false;
        p->points = default_points(p);
        return PACMAN_RECURRENCE_OK;
    }
    int threads = tiled_threads(p->kernel);
    // the most points per block whose lanes are still at least `lanes`
    uint32_t points = 0;
    for (uint32_t np = 1; np <= kMaxPoints; np++)
        if (tiled_lanes(np, threads) >= lanes) points = np;
    if (!tiled_points_fit(points, p->point_bytes, threads, point_smem(p))) return PACMAN_RECURRENCE_INVALID;
    p->points = points;
    p->fixed = true;
    return PACMAN_RECURRENCE_OK;
}

extern "C" uint32_t pacuda_b200_plan_lanes_per_point(const pacuda_b200_plan *p) {
    return p ? tiled_lanes(p->points, p->tiled.threads) : 0;
}

extern "C" pacuda_b200_batch *pacuda_b200_batch_create(pacuda_b200_plan *const *plans, uint32_t nplans,
                                                       const double *const *external, const uint32_t *count,
                                                       double *const *output) {
    if (!plans || !nplans || !external || !count || !output) return nullptr;
    for (uint32_t k = 0; k < nplans; k++)
        if (!plans[k] || plans[k]->kernel != plans[0]->kernel || !count[k] || !external[k] || !output[k]) {
            fprintf(stderr, "%s: batch_create: plan %u: a missing plan, array or point count, or another kernel kind\n",
                    kTag, k);
            return nullptr;
        }
    auto *b = new pacuda_b200_batch();
    b->plans.assign(plans, plans + nplans);
    b->external.assign(external, external + nplans);
    b->count.assign(count, count + nplans);
    b->output.assign(output, output + nplans);
    b->sms = device_sms();
    if (failed(cudaEventCreateWithFlags(&b->copied, cudaEventDisableTiming), "event") || !prepare(b)) {
        pacuda_b200_batch_destroy(b);
        return nullptr;
    }
    return b;
}

extern "C" int pacuda_b200_batch_update(pacuda_b200_batch *b, const double *const *external, const uint32_t *count,
                                        double *const *output) {
    if (!b || !external || !count || !output) return PACMAN_RECURRENCE_INVALID;
    for (size_t k = 0; k < b->plans.size(); k++)
        if (!count[k] || !external[k] || !output[k]) {
            fprintf(stderr, "%s: batch_update: plan %zu: a missing array or point count\n", kTag, k);
            return PACMAN_RECURRENCE_INVALID;
        }
    // the previous launch's copy of the descriptors must have left the pinned block
    if (failed(cudaEventSynchronize(b->copied), "batch_update")) return PACMAN_RECURRENCE_DEVICE_ERROR;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
    }
    size_t n = b->plans.size();
    b->external.assign(external, external + n);
    b->count.assign(count, count + n);
    b->output.assign(output, output + n);
    return prepare(b) ? PACMAN_RECURRENCE_OK : PACMAN_RECURRENCE_DEVICE_ERROR;
}

extern "C" int pacuda_b200_batch_run(pacuda_b200_batch *b, void *stream) {
    if (!b) return PACMAN_RECURRENCE_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    if (b->exec) return failed(cudaGraphLaunch(b->exec, s), "graph") ? PACMAN_RECURRENCE_DEVICE_ERROR : PACMAN_RECURRENCE_OK;
    return launch(b, s);
}

extern "C" int pacuda_b200_batch_capture(pacuda_b200_batch *b, void *stream) {
    if (!b) return PACMAN_RECURRENCE_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    // the legacy default stream cannot be captured: capture on a stream of the batch's own (the
    // graph is launched later on whatever stream a run names)
    cudaStream_t own = nullptr;
    if (s == nullptr || s == cudaStreamLegacy) {
        if (failed(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking), "capture stream")) return PACMAN_RECURRENCE_DEVICE_ERROR;
        s = own;
    }
    int status = PACMAN_RECURRENCE_OK;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
    }
    if (failed(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture")) {
        status = PACMAN_RECURRENCE_DEVICE_ERROR;
    } else {
        int st = launch(b, s);
        cudaError_t e = cudaStreamEndCapture(s, &b->graph);
        if (st != PACMAN_RECURRENCE_OK || failed(e, "capture") ||
            failed(cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiation"))
            status = PACMAN_RECURRENCE_DEVICE_ERROR;
    }
    if (own) cudaStreamDestroy(own);
    return status;
}

extern "C" int pacuda_b200_batch_tune(pacuda_b200_batch *b, void *stream) {
    if (!b) return PACMAN_RECURRENCE_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    // one plan alone at `points` per block and `blocks` per SM: the best of three launches, in ms
    // (or a negative time when it does not fit)
    auto time_plan = [&](size_t k, uint32_t points, int blocks) -> float {
        pacuda_b200_plan *p = b->plans[k], *one[1] = {p};
        const double *ext[1] = {b->external[k]};
        double *out[1] = {b->output[k]};
        uint32_t n = b->count[k], keep = p->points;
        p->points = points;
        pacuda_b200_batch *tb = pacuda_b200_batch_create(one, 1, ext, &n, out);
        float ms = -1.0f;
        if (tb) {
            tb->blocks = blocks;
            bool ok = prepare(tb) && tb->points[0] == points && launch(tb, s) == PACMAN_RECURRENCE_OK;
            for (int rep = 0; ok && rep < 3; rep++) {
                cudaEventRecord(t0, s);
                ok = launch(tb, s) == PACMAN_RECURRENCE_OK;
                cudaEventRecord(t1, s);
                cudaEventSynchronize(t1);
                float m = 0;
                cudaEventElapsedTime(&m, t0, t1);
                ms = rep == 0 ? m : std::min(ms, m);
            }
            if (!ok) ms = -1.0f;
            pacuda_b200_batch_destroy(tb);
        }
        p->points = keep;
        return ms;
    };
    // per plan: its fastest points per block (from the most that fit down to half of them:
    // fewer leave more of a block's lanes idle at the levels' barriers) for each blocks-per-SM
    // choice, and the fastest pair; plans of the same blocks per SM share a launch
    const int kernel = b->plans[0]->kernel;
    for (size_t k = 0; k < b->plans.size(); k++) {
        pacuda_b200_plan *p = b->plans[k];
        size_t cb = tiled_const_bytes(p->scales, p->factors);
        float best = -1.0f;
        uint32_t best_points = p->points;
        int best_blocks = 0;
        for (int blocks : kBlockChoices) {
            int threads = tiled_threads(kernel, blocks);
            size_t room = tiled_max_smem(kernel, blocks);
            uint32_t most = room > cb ? tiled_max_points(p->point_bytes, threads, room - cb) : 0;
            for (uint32_t points = most; points >= 1 && 2 * points >= most; points--) {
                if (p->fixed && points != p->points) continue;
                float ms = time_plan(k, points, blocks);
                if (ms >= 0.0f && (best < 0.0f || ms < best)) {
                    best = ms;
                    best_points = points;
                    best_blocks = blocks;
                }
            }
        }
        if (best >= 0.0f) {
            p->points = best_points;
            b->plan_blocks[k] = best_blocks;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
    }
    return prepare(b) ? PACMAN_RECURRENCE_OK : PACMAN_RECURRENCE_DEVICE_ERROR;
}

extern "C" uint32_t pacuda_b200_batch_launches(const pacuda_b200_batch *b) { return b ? (uint32_t)b->groups.size() : 0; }

extern "C" int pacuda_b200_batch_set_blocks_per_sm(pacuda_b200_batch *b, uint32_t blocks) {
    if (!b || (blocks && !tiled_blocks_valid((int)blocks))) return PACMAN_RECURRENCE_INVALID;
    if (failed(cudaEventSynchronize(b->copied), "batch")) return PACMAN_RECURRENCE_DEVICE_ERROR;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
    }
    int before = b->blocks;
    std::vector<int> before_plans = b->plan_blocks;
    b->blocks = (int)blocks;
    std::fill(b->plan_blocks.begin(), b->plan_blocks.end(), 0);  // every plan the same
    if (!prepare(b)) {
        b->blocks = before;
        b->plan_blocks = before_plans;
        prepare(b);
        return PACMAN_RECURRENCE_INVALID;
    }
    return PACMAN_RECURRENCE_OK;
}

extern "C" uint32_t pacuda_b200_batch_blocks_per_sm(const pacuda_b200_batch *b) { return b ? (uint32_t)b->blocks : 0; }

extern "C" int pacuda_b200_batch_set_plan_blocks_per_sm(pacuda_b200_batch *b, uint32_t plan, uint32_t blocks) {
    if (!b || plan >= b->plans.size() || (blocks && !tiled_blocks_valid((int)blocks))) return PACMAN_RECURRENCE_INVALID;
    if (failed(cudaEventSynchronize(b->copied), "batch")) return PACMAN_RECURRENCE_DEVICE_ERROR;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
    }
    int before = b->plan_blocks[plan];
    b->plan_blocks[plan] = (int)blocks;
    if (!prepare(b)) {
        b->plan_blocks[plan] = before;
        prepare(b);
        return PACMAN_RECURRENCE_INVALID;
    }
    return PACMAN_RECURRENCE_OK;
}

extern "C" uint32_t pacuda_b200_batch_plan_blocks_per_sm(const pacuda_b200_batch *b, uint32_t plan) {
    if (!b || plan >= b->plan_blocks.size()) return 0;
    for (const LaunchGroup &g : b->groups)
        for (uint32_t k : g.plans)
            if (k == plan) return (uint32_t)g.blocks;
    return 0;
}

extern "C" uint32_t pacuda_b200_batch_lanes_per_point(const pacuda_b200_batch *b, uint32_t plan) {
    if (!b || plan >= b->points.size() || !b->points[plan]) return 0;
    for (const LaunchGroup &g : b->groups)
        for (uint32_t k : g.plans)
            if (k == plan) return tiled_lanes(b->points[plan], g.threads);
    return 0;
}

extern "C" void pacuda_b200_batch_destroy(pacuda_b200_batch *b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->copied) {
        cudaEventSynchronize(b->copied);
        cudaEventDestroy(b->copied);
    }
    cudaFreeHost(b->host);
    cudaFree(b->device);
    delete b;
}

// ---------------------------------------------------------------------------------------------
// Evaluation without allocation (pacuda_b200_run_static).
//
// pacuda_b200_batch_create allocates a pinned and a device descriptor block. Some callers cannot
// allocate when they evaluate: an integrand callback that runs inside a host framework which owns
// the device's memory pool (an allocation there bypasses the pool, can fail once the pool has
// taken the device's memory, and stalls the device while the driver maps it), or a caller that is
// recording the surrounding work into a CUDA graph, where a cudaMalloc is no stream operation at
// all. For them this entry point keeps the descriptors of one launch and its work-item counter in
// a fixed array of this library in device memory. It allocates nothing; the plans' own arrays were
// allocated when they were created.
//
// Limits: at most PACUDA_B200_STATIC_MAX_PLANS plans per call (more are INVALID). The array is one
// per device: calls on one device must not overlap (the second call's setup would overwrite the
// first's descriptors and counter while the first runs), so issue them on one stream or order
// them with events.

namespace {

constexpr uint32_t kStaticPlans = PACUDA_B200_STATIC_MAX_PLANS;
constexpr int kStaticDevices = 64;

// the launch's descriptors; the setup kernel receives them as its parameter (under 4 KB)
struct StaticBlock {
    TiledPlan plans[kStaticPlans];
    unsigned long long items[kStaticPlans + 1];
    const double *external[kStaticPlans];
    double *output[kStaticPlans];
    uint32_t count[kStaticPlans];
};
constexpr size_t kStaticCounter = (sizeof(StaticBlock) + 255) / 256 * 256;
constexpr size_t kStaticBytes = 4096;
static_assert(kStaticCounter + sizeof(unsigned long long) <= kStaticBytes, "the static scratch is too small");
static_assert(sizeof(StaticBlock) <= 4000, "the descriptors exceed a kernel parameter");

// the scratch: StaticBlock at 0; the work-item counter at kStaticCounter, which must be zero when
// the executor starts (the setup kernel of every call zeroes it); nothing else needs a start value
__device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

__global__ void static_setup(StaticBlock block, unsigned char *scratch) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *(StaticBlock *)scratch = block;
        *(unsigned long long *)(scratch + kStaticCounter) = 0;
    }
}

std::mutex g_static_mutex;

// the driver's context id of the calling thread's current context, or 0 when it cannot be read
// (cuCtxGetId through the runtime's entry-point table: this library links no driver library)
unsigned long long current_context_id() {
    typedef int (*CtxGetCurrent)(void **);
    typedef int (*CtxGetId)(void *, unsigned long long *);
    static CtxGetCurrent get_current = nullptr;
    static CtxGetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        looked_up = true;
        void *f = nullptr, *g = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &g, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
            get_current = (CtxGetCurrent)f;
            get_id = (CtxGetId)g;
        }
        cudaGetLastError();
    }
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

struct StaticAddress {
    unsigned long long context = 0;  // the context the address belongs to (0: none)
    void *address = nullptr;
};
StaticAddress g_static_address[kStaticDevices];

// the scratch's address on the current device. It is looked up (cudaGetSymbolAddress, which may
// load this library's device code) on the first call in each context of a device, so again after
// a device reset or under another context on the same device; later calls compare the context
// id and read the cache. Where the context id cannot be read, it is looked up on every call.
unsigned char *static_scratch() {
    int dev = -1;
    if (failed(cudaGetDevice(&dev), "current device")) return nullptr;
    if (dev < 0 || dev >= kStaticDevices) {
        fprintf(stderr, "%s: run_static: device %d beyond the %d this entry point serves\n", kTag, dev, kStaticDevices);
        return nullptr;
    }
    // 0 until the thread has a current context (the symbol lookup below makes the runtime's one
    // current, so only a thread's first call looks up the address for that reason)
    const unsigned long long context = current_context_id();
    std::lock_guard<std::mutex> lock(g_static_mutex);
    StaticAddress &c = g_static_address[dev];
    if (!context || c.context != context || !c.address) {
        void *address = nullptr;
        if (failed(cudaGetSymbolAddress(&address, g_static_scratch), "static scratch address") || !address)
            return nullptr;
        c.context = context;
        c.address = address;
    }
    return (unsigned char *)c.address;
}

}  // namespace

extern "C" int pacuda_b200_run_static(pacuda_b200_plan *const *plans, uint32_t nplans, const double *const *external,
                                      const uint32_t *count, double *const *output, void *stream) {
    if (nplans == 0 || nplans > kStaticPlans) {
        fprintf(stderr, "%s: run_static: %u plans; this entry point takes 1 to %u\n", kTag, nplans, kStaticPlans);
        return PACMAN_RECURRENCE_INVALID;
    }
    if (!plans || !external || !count || !output) return PACMAN_RECURRENCE_INVALID;
    for (uint32_t k = 0; k < nplans; k++)
        if (!plans[k] || plans[k]->kernel != plans[0]->kernel || !count[k] || !external[k] || !output[k]) {
            fprintf(stderr, "%s: run_static: plan %u: a missing plan, array or point count, or another kernel kind\n",
                    kTag, k);
            return PACMAN_RECURRENCE_INVALID;
        }
    unsigned char *scratch = static_scratch();
    if (!scratch) return PACMAN_RECURRENCE_DEVICE_ERROR;
    // the launch's shape as a batch of these plans has it; the plans' own choices are not changed
    int kernel = plans[0]->kernel;
    int threads = tiled_threads(kernel);
    size_t const_bytes = 0;
    for (uint32_t k = 0; k < nplans; k++)
        const_bytes = std::max(const_bytes, tiled_const_bytes(plans[k]->scales, plans[k]->factors));
    // the shared memory a block may have, less the plan constants every block holds (checked
    // before anything is queued)
    const size_t room = tiled_max_smem(kernel);
    if (room == 0) return PACMAN_RECURRENCE_DEVICE_ERROR;
    if (room <= const_bytes) {
        fprintf(stderr, "%s: run_static: the plans' constants (%zu bytes) fill a block's shared memory\n", kTag,
                const_bytes);
        return PACMAN_RECURRENCE_INVALID;
    }
    const size_t max_smem = room - const_bytes;
    StaticBlock block;
    memset(&block, 0, sizeof block);
    size_t smem = 0;
    for (uint32_t k = 0; k < nplans; k++) {
        const pacuda_b200_plan *p = plans[k];
        uint32_t most = tiled_max_points(p->point_bytes, threads, max_smem);
        if (!most || p->tiled.threads != threads) {
            fprintf(stderr, "%s: run_static: a plan's point does not fit a block's shared memory\n", kTag);
            return PACMAN_RECURRENCE_INVALID;
        }
        uint32_t per = tiled_points_fit(p->points, p->point_bytes, threads, max_smem)
                           ? p->points
                           : tiled_default_points(p->point_bytes, threads, max_smem);
        fill_plan(p, block.plans[k], per);
        smem = std::max<size_t>(smem, (size_t)per * p->point_bytes);
        block.items[k + 1] = block.items[k] + (count[k] + per - 1) / per;
        block.external[k] = external[k];
        block.output[k] = output[k];
        block.count[k] = count[k];
    }
    smem += const_bytes;
    cudaStream_t s = (cudaStream_t)stream;
    static_setup<<<1, 32, 0, s>>>(block, scratch);
    if (failed(cudaGetLastError(), "run_static setup")) return PACMAN_RECURRENCE_DEVICE_ERROR;
    const StaticBlock *d = (const StaticBlock *)scratch;
    TiledLaunch L;
    memset(&L, 0, sizeof L);
    L.plans = d->plans;
    L.nplans = nplans;
    L.item_first = d->items;
    L.external = d->external;
    L.output = d->output;
    L.count = d->count;
    L.counter = (unsigned long long *)(scratch + kStaticCounter);
    L.abi = false;
    L.const_bytes = (uint32_t)const_bytes;
    if (!launch_tiled(kernel, L, threads, smem, device_sms(), s) || failed(cudaGetLastError(), "run_static launch"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    return PACMAN_RECURRENCE_OK;
}
