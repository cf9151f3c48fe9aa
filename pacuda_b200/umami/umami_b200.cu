// The UMAMI library of one subprocess on the B200 runner (include/umami.h): the reference's
// umami/umami_pacuda.c behind the same nine functions, the same inputs and outputs and the same
// `.pacuda` file, evaluated the B200 way.
//
// At initialisation every (process, colour) plan of the file is compiled once for the on-chip
// executor (pacuda_b200_plan_create, with the colour's resolved reduction over the helicities
// that have planes). A call then
//   1. selects each event's contributions from its channel and flavour (the provider's tables),
//      and groups them by (process, colour, leg permutation), events in order within a group;
//   2. copies the events' momenta to the device once, as the caller lays them out (row
//      n * k + leg for component k of a leg, one value per event), and each item's inputs;
//   3. gathers every group's external momenta on the device (the permutation and the process's
//      crossing applied: external leg l = sign_l x input leg permutation[crossing_l]);
//   4. evaluates every group in one run of the batched executor (a persistent launch per
//      blocks-per-SM choice), each point's helicity values reduced in the kernel from its
//      amplitudes (pacuda_b200_batch_*);
//   5. finishes each item on the device (the process-group factor, the alpha_s scale, then the
//      helicity sum, a fixed helicity's value, or the helicity drawn in proportion to its value,
//      with the reference's arithmetic in its order: recurrence_runner.cu:1532-1572) and copies
//      back one value per item (and the draw);
//   6. combines each event's contributions on the host as the reference does.
// Steps 1-5 run per chunk of events (kChunkParts), the host's steps for the next chunk while the
// device runs the previous one.
// The values equal the reference library's bit for bit: the same f64 arithmetic in the same
// order, from the same resolved reduction.
//
// Built once per subprocess with its provider header (pacuda_b200/umami/build.py), as the
// reference's library is (umami/build.sh).
#include <cuda_runtime.h>
#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/pacuda_b200.h"
#include "../../include/umami.h"
#include "../../include/umami_provider.h"
#include "pacuda_reader.h"

#ifndef UMAMI_PROVIDER_HEADER
#error "build with -DUMAMI_PROVIDER_HEADER='\"provider.h\"' (the subprocess's provider tables)"
#endif
#include UMAMI_PROVIDER_HEADER

#define UMAMI_EXPORT extern "C" __attribute__((visibility("default")))

using pacuda::PacudaColour;
using pacuda::PacudaFile;
using pacuda::PacudaProcess;

namespace {

const char *const kTag = "pacuda-b200 umami";
constexpr int kMaxLegs = 16;
// A call's events are evaluated in up to kChunks chunks of at least kChunkEvents: the host builds
// a chunk's items while the device evaluates the previous chunk. A full call's chunks take these
// shares (of kChunkWhole) of its events: a short first chunk, so that the device starts early,
// then growing ones (each chunk's host passes and copy end before the device has evaluated the
// previous chunk: on B200 the passes take about half the evaluation's time per event), and a short
// last one, so that the host's last combining is short. (Measured on B200, p p -> 3 jets, 2^20
// events: 18.6 ms per call, against 19.4 ms for four chunks of 1/8, 3/8, 3/8, 1/8.)
constexpr int kChunks = 5;
constexpr size_t kChunkEvents = 1 << 16;
constexpr size_t kChunkWhole = 64;
constexpr size_t kChunkParts[kChunks + 1] = {0, 4, 12, 28, 56, 64};

bool cuda_failed(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return false;
    fprintf(stderr, "%s: %s: %s\n", kTag, what, cudaGetErrorString(e));
    return true;
}

// a device array that only grows
template <class T> struct DeviceArray {
    T *p = nullptr;
    size_t capacity = 0;
    bool reserve(size_t n) {
        if (n <= capacity) return true;
        cudaFree(p);
        p = nullptr;
        capacity = 0;
        if (cuda_failed(cudaMalloc((void **)&p, std::max<size_t>(n, 1) * sizeof(T)), "device buffer")) return false;
        capacity = n;
        return true;
    }
    void release() {
        cudaFree(p);
        p = nullptr;
        capacity = 0;
    }
};

// a pinned host array that only grows
template <class T> struct PinnedArray {
    T *p = nullptr;
    size_t capacity = 0;
    bool reserve(size_t n) {
        if (n <= capacity) return true;
        cudaFreeHost(p);
        p = nullptr;
        capacity = 0;
        if (cuda_failed(cudaMallocHost((void **)&p, std::max<size_t>(n, 1) * sizeof(T)), "pinned buffer")) return false;
        capacity = n;
        return true;
    }
    void release() {
        cudaFreeHost(p);
        p = nullptr;
        capacity = 0;
    }
};

// One group of items (its class's plan over its events): the gather of its external momenta,
// external[(l * 4 + k) * points + q] = sign[l] * momenta[(legs * k + leg[l]) * events + event[q]],
// and where its helicity values go.
struct Group {
    unsigned long long external;  // offset of the group's planes in the external buffer
    unsigned long long first;     // its first item (items are grouped, events in order within)
    unsigned long long values;    // offset of its values ([point][live]) in the value buffer
    uint32_t points, legs;
    uint32_t live, helicities;    // outputs with planes, and all the process's helicities
    uint32_t live_at;             // offset of the colour's live helicities in the helicity table
    uint32_t factor;              // 1: times numerator / denominator (the process-group factor)
    double numerator, denominator;
    uint32_t leg[kMaxLegs];
    double sign[kMaxLegs];
};

// One item's inputs, in group order.
struct ItemIn {
    uint32_t event;    // relative to the call's first event
    int32_t helicity;  // a fixed helicity's runtime index (or -1)
    double scale;      // (alpha_s / alpha_s at conversion) ^ QCD power
    double random;     // the helicity's random number (sampling)
};

enum Mode : int { MODE_SUM = 0, MODE_HELICITY = 1, MODE_SAMPLE = 2 };

__device__ __forceinline__ uint32_t group_of(const Group *groups, uint32_t ngroups, unsigned long long item) {
    uint32_t lo = 0, hi = ngroups;  // the last group whose first item is <= item
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) / 2;
        if (groups[mid].first <= item) lo = mid; else hi = mid;
    }
    return lo;
}

// `bad` is set when any of the n values is not finite
__global__ void check_finite(const double *values, size_t n, int *bad) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (!isfinite(values[i])) *bad = 1;
}

// the external momenta of every group
__global__ void gather_groups(const Group *groups, const double *momenta, size_t events, const ItemIn *items,
                              double *external) {
    const Group &g = groups[blockIdx.y];
    const size_t n = (size_t)g.points * g.legs * 4;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        size_t q = i % g.points, lk = i / g.points;
        uint32_t l = (uint32_t)(lk >> 2), k = (uint32_t)(lk & 3);
        double v = momenta[((size_t)g.legs * k + g.leg[l]) * events + items[g.first + q].event];
        external[g.external + i] = g.sign[l] * v;
    }
}

// Each item's result from its helicity values, with the reference's arithmetic in its order: every
// value times numerator / denominator, times the scale; then the sum over all the helicities (the
// ones without planes as 0.0), the value of one helicity, or the sampling's total and draw
// (recurrence_runner.cu:1532-1572).
__global__ void finish_items(const Group *groups, uint32_t ngroups, const ItemIn *items, unsigned long long nitems,
                             const double *values, const uint32_t *live_helicity, int mode, double *value_out,
                             uint32_t *chosen_out) {
    for (unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; j < nitems;
         j += (unsigned long long)gridDim.x * blockDim.x) {
        const Group &g = groups[group_of(groups, ngroups, j)];
        const ItemIn it = items[j];
        const double *v = values + g.values + (j - g.first) * (g.live ? g.live : 1);
        const uint32_t *lh = live_helicity + g.live_at;
        auto value = [&](uint32_t o) {
            double x = v[o];
            if (g.factor) x = __ddiv_rn(__dmul_rn(x, g.numerator), g.denominator);
            if (it.scale != 1.0) x = __dmul_rn(x, it.scale);
            return x;
        };
        if (mode == MODE_SUM) {
            double sum = 0.0;
            uint32_t o = 0;
            for (uint32_t h = 0; h < g.helicities; h++) {
                double x = 0.0;
                if (o < g.live && lh[o] == h) x = value(o++);
                sum = __dadd_rn(sum, x);
            }
            value_out[j] = sum;
        } else if (mode == MODE_HELICITY) {
            double x = 0.0;
            for (uint32_t o = 0; o < g.live; o++)
                if (lh[o] == (uint32_t)it.helicity) x = value(o);
            value_out[j] = x;
        } else {
            double total = 0.0;
            for (uint32_t o = 0; o < g.live; o++) total = __dadd_rn(total, value(o));
            double target = __dmul_rn(it.random, total), cumulative = 0.0;
            uint32_t pick = 0;
            for (uint32_t o = 0; o < g.live; o++) {
                double x = value(o);
                if (x <= 0.0) continue;
                pick = lh[o];
                cumulative = __dadd_rn(cumulative, x);
                if (cumulative > target) break;
            }
            value_out[j] = total;
            chosen_out[j] = pick;
        }
    }
}

struct Colour {
    const PacudaColour *c = nullptr;
    pacuda_b200_plan *plan = nullptr;
    uint32_t live = 0;     // outputs of the plan (the helicities with planes)
    uint32_t live_at = 0;  // its live helicities' offset in the instance's helicity table
};

// contributions that evaluate alike: one (process, colour id, leg permutation)
struct Class {
    const UmamiContribution *entry = nullptr;  // the first contribution of the class
    const Colour *colour = nullptr;
};

struct Instance {
    PacudaFile file;
    std::vector<int> process;       // per provider process: its file process, or -1
    std::vector<double> alpha_s;    // per provider process
    std::vector<std::vector<Colour>> colours;  // [file process][colour]
    std::vector<Class> classes;
    std::vector<std::vector<std::vector<uint32_t>>> class_of;  // [channel][flavour][contribution]
    cudaStream_t stream = nullptr, copies = nullptr;  // compute; and the copies in
    cudaEvent_t arrived[kChunks] = {nullptr};         // a chunk's inputs are on the device
    cudaEvent_t done[kChunks] = {nullptr};            // a chunk's results are on the host
    DeviceArray<uint32_t> live_helicity;  // every colour's live helicities
    // the call's buffers
    DeviceArray<double> momenta, external, values, value_out;
    DeviceArray<uint32_t> chosen_out;
    DeviceArray<ItemIn> items;
    DeviceArray<Group> groups;
    DeviceArray<int> bad;
    PinnedArray<ItemIn> host_items;
    PinnedArray<Group> host_groups;
    PinnedArray<double> host_value;
    PinnedArray<uint32_t> host_chosen;
    PinnedArray<int> host_bad;
    // per chunk: the batch of the last call's groups (re-pointed while their plans repeat)
    pacuda_b200_batch *batch[kChunks] = {nullptr};
    std::vector<pacuda_b200_plan *> batch_plans[kChunks];
    // the host's per-call arrays, kept between calls: per event its channel << 16 | flavour, per
    // event-ordered item its place among the items
    std::vector<uint32_t> selection, at;
};

bool const supported_inputs[UMAMI_INPUT_KEY_COUNT] = {
    /* UMAMI_IN_MOMENTA */ true, /* UMAMI_IN_ALPHA_S */ UMAMI_HAS_ALPHA_S, /* UMAMI_IN_FLAVOR_INDEX */ true,
    false, /* UMAMI_IN_RANDOM_HELICITY */ true, false, /* UMAMI_IN_HELICITY_INDEX */ true, false,
    /* UMAMI_IN_CHANNEL_INDEX */ true};
bool const required_inputs[UMAMI_INPUT_KEY_COUNT] = {/* UMAMI_IN_MOMENTA */ true};
bool const supported_outputs[UMAMI_OUTPUT_KEY_COUNT] = {
    /* UMAMI_OUT_MATRIX_ELEMENT */ true, false, /* UMAMI_OUT_COLOR_INDEX */ UMAMI_HAS_COLOR_FLOW,
    /* UMAMI_OUT_HELICITY_INDEX */ true};

const UmamiParameter *parameter(size_t process, const char *name) {
    const UmamiProcess &entry = umami_provider.processes[process];
    for (size_t i = 0; i < entry.parameter_count; ++i)
        if (strcmp(entry.parameters[i].name, name) == 0) return &entry.parameters[i];
    return nullptr;
}

// a model parameter's value at conversion: the file's, else the provider's default
void converted_value(const PacudaProcess *p, const UmamiParameter *entry, double *re, double *im) {
    *re = entry->real;
    *im = entry->imaginary;
    if (!p) return;
    for (size_t k = 0; k < p->parameter_names.size(); k++)
        if (p->parameter_names[k] == entry->name) {
            *re = p->parameter_re[k];
            *im = p->parameter_im[k];
        }
}

const PacudaProcess *process_of(const Instance *in, size_t provider_process) {
    int f = in->process[provider_process];
    return f < 0 ? nullptr : &in->file.processes[f];
}

const Colour *colour_of(const Instance *in, const UmamiContribution *c) {
    int f = in->process[c->process_index];
    if (f < 0) return nullptr;
    for (const Colour &col : in->colours[f])
        if (col.c->id == c->color_id) return &col;
    return nullptr;
}

bool alpha_named(const PacudaProcess *p, const char *name) {
    return p && !p->alpha_s_name.empty() && p->alpha_s_name == name;
}

void free_instance(Instance *in) {
    if (!in) return;
    if (in->stream) cudaStreamSynchronize(in->stream);
    if (in->copies) cudaStreamSynchronize(in->copies);
    for (int c = 0; c < kChunks; c++) {
        pacuda_b200_batch_destroy(in->batch[c]);
        if (in->arrived[c]) cudaEventDestroy(in->arrived[c]);
        if (in->done[c]) cudaEventDestroy(in->done[c]);
    }
    for (auto &v : in->colours)
        for (Colour &c : v) pacuda_b200_plan_destroy(c.plan);
    in->live_helicity.release();
    in->momenta.release();
    in->external.release();
    in->values.release();
    in->value_out.release();
    in->chosen_out.release();
    in->items.release();
    in->groups.release();
    in->bad.release();
    in->host_items.release();
    in->host_groups.release();
    in->host_value.release();
    in->host_chosen.release();
    in->host_bad.release();
    if (in->stream) cudaStreamDestroy(in->stream);
    if (in->copies) cudaStreamDestroy(in->copies);
    delete in;
}

// alike when they share the process, the colour id and the leg permutation
bool same_evaluation(const UmamiContribution *x, const UmamiContribution *y) {
    return x->process_index == y->process_index && strcmp(x->color_id, y->color_id) == 0 &&
           memcmp(x->permutation, y->permutation, umami_provider.particle_count * sizeof(size_t)) == 0;
}

// One chunk of a call: its events, its items (grouped by class) and where its data go.
struct Chunk {
    size_t e0 = 0, e1 = 0;           // its events, relative to the call's first
    size_t item0 = 0, items = 0;     // its items among the call's
    size_t external = 0, values = 0; // its places in the external-momentum and value buffers
    std::vector<uint32_t> first;     // per class: its first item (relative to item0); classes + 1
};

// Queues one chunk: its momenta and items in on the copy stream, then on the compute stream
// its gather, ONE batched launch over its classes with items, its finishing pass and its results
// out. `group0`: its place in the group buffers (kChunks regions of one group per class).
UmamiStatus launch_chunk(Instance *in, int slot, const Chunk &ch, const double *momenta, size_t stride,
                         size_t offset, int mode) {
    const size_t n = umami_provider.particle_count, events = ch.e1 - ch.e0, group0 = slot * in->classes.size();
    std::vector<pacuda_b200_plan *> plans;
    std::vector<uint32_t> points;
    std::vector<const double *> ext_p;
    std::vector<double *> out_p;
    size_t ext = ch.external, vals = ch.values, groups = 0;
    double *dev_mom = in->momenta.p + 4 * n * ch.e0;
    for (size_t c = 0; c < in->classes.size(); c++) {
        uint32_t m = ch.first[c + 1] - ch.first[c];
        if (!m) continue;
        const Class &cls = in->classes[c];
        const PacudaProcess *p = process_of(in, cls.entry->process_index);
        Group &G = in->host_groups.p[group0 + groups++];
        memset(&G, 0, sizeof G);
        G.external = ext;
        G.first = ch.first[c];
        G.values = vals;
        G.points = m;
        G.legs = (uint32_t)n;
        G.live = cls.colour->live;
        G.helicities = p->helicities;
        G.live_at = cls.colour->live_at;
        G.factor = p->numerator != p->denominator;
        G.numerator = (double)p->numerator;
        G.denominator = (double)p->denominator;
        for (size_t l = 0; l < n; l++) {
            size_t source = p->crossing_leg.empty() ? l : p->crossing_leg[l];
            G.leg[l] = (uint32_t)cls.entry->permutation[source];
            G.sign[l] = p->crossing_leg.empty() ? 1.0 : p->crossing_sign[l];
        }
        plans.push_back(cls.colour->plan);
        points.push_back(m);
        ext_p.push_back(in->external.p + ext);
        out_p.push_back(in->values.p + vals);
        ext += 4 * n * m;
        vals += (size_t)std::max<uint32_t>(G.live, 1) * m;
    }
    ItemIn *items = in->items.p + ch.item0;
    Group *dev_groups = in->groups.p + group0;
    if (cuda_failed(cudaMemcpy2DAsync(dev_mom, events * sizeof(double), momenta + offset + ch.e0,
                                      stride * sizeof(double), events * sizeof(double), 4 * n,
                                      cudaMemcpyHostToDevice, in->copies),
                    "momenta") ||
        (check_finite<<<(unsigned)std::min<size_t>((4 * n * events + 255) / 256, 1024), 256, 0, in->copies>>>(
             dev_mom, 4 * n * events, in->bad.p),
         cuda_failed(cudaGetLastError(), "check")) ||
        cuda_failed(cudaMemcpyAsync(items, in->host_items.p + ch.item0, ch.items * sizeof(ItemIn),
                                    cudaMemcpyHostToDevice, in->copies),
                    "items") ||
        cuda_failed(cudaMemcpyAsync(dev_groups, in->host_groups.p + group0, groups * sizeof(Group),
                                    cudaMemcpyHostToDevice, in->copies),
                    "groups") ||
        cuda_failed(cudaEventRecord(in->arrived[slot], in->copies), "event") ||
        cuda_failed(cudaStreamWaitEvent(in->stream, in->arrived[slot], 0), "event"))
        return UMAMI_ERROR;
    cudaStream_t s = in->stream;
    uint32_t most = *std::max_element(points.begin(), points.end());
    dim3 grid((unsigned)std::min<size_t>((4 * n * most + 255) / 256, 2048), (unsigned)groups);
    gather_groups<<<grid, 256, 0, s>>>(dev_groups, dev_mom, events, items, in->external.p);
    if (cuda_failed(cudaGetLastError(), "gather")) return UMAMI_ERROR;
    pacuda_b200_batch *&batch = in->batch[slot];
    if (batch && in->batch_plans[slot] == plans) {
        if (pacuda_b200_batch_update(batch, ext_p.data(), points.data(), out_p.data()) != PACMAN_RECURRENCE_OK)
            return UMAMI_ERROR;
    } else {
        if (batch) {
            cudaStreamSynchronize(s);
            pacuda_b200_batch_destroy(batch);
        }
        batch = pacuda_b200_batch_create(plans.data(), (uint32_t)groups, ext_p.data(), points.data(), out_p.data());
        in->batch_plans[slot] = batch ? plans : std::vector<pacuda_b200_plan *>();
        if (!batch) return UMAMI_ERROR;
        // several independent blocks per SM, chosen per plan (one waits at a level's barrier while
        // the others run); else the batch keeps one
        pacuda_b200_batch_set_blocks_per_sm(batch, 0);
    }
    if (pacuda_b200_batch_run(batch, s) != PACMAN_RECURRENCE_OK) return UMAMI_ERROR;
    unsigned blocks = (unsigned)std::min<size_t>((ch.items + 255) / 256, 4096);
    finish_items<<<blocks, 256, 0, s>>>(dev_groups, (uint32_t)groups, items, ch.items, in->values.p,
                                        in->live_helicity.p, mode, in->value_out.p + ch.item0,
                                        in->chosen_out.p + ch.item0);
    if (cuda_failed(cudaGetLastError(), "finish") ||
        cuda_failed(cudaMemcpyAsync(in->host_value.p + ch.item0, in->value_out.p + ch.item0, ch.items * sizeof(double),
                                    cudaMemcpyDeviceToHost, s),
                    "values") ||
        (mode == MODE_SAMPLE &&
         cuda_failed(cudaMemcpyAsync(in->host_chosen.p + ch.item0, in->chosen_out.p + ch.item0,
                                     ch.items * sizeof(uint32_t), cudaMemcpyDeviceToHost, s),
                     "draws")))
        return UMAMI_ERROR;
    return UMAMI_SUCCESS;
}

}  // namespace

UMAMI_EXPORT UmamiStatus umami_get_meta(UmamiMetaKey key, void *result) {
    if (result == nullptr) return UMAMI_ERROR;
    switch (key) {
    case UMAMI_META_DEVICE: *(UmamiDevice *)result = UMAMI_DEVICE_CPU; break;  // host inputs and outputs
    case UMAMI_META_PARTICLE_COUNT: *(int *)result = (int)umami_provider.particle_count; break;
    case UMAMI_META_HELICITY_COUNT: *(int *)result = (int)umami_provider.helicity_count; break;
    case UMAMI_META_COLOR_COUNT:
        if (!UMAMI_HAS_COLOR_FLOW) return UMAMI_ERROR_UNSUPPORTED_META;
        *(int *)result = (int)umami_provider.color_count;
        break;
    case UMAMI_META_MASSES:
        memcpy(result, umami_provider.masses, umami_provider.particle_count * sizeof(double));
        break;
    default: return UMAMI_ERROR_UNSUPPORTED_META;
    }
    return UMAMI_SUCCESS;
}

UMAMI_EXPORT UmamiStatus umami_supported_inputs(bool const **supported, int *count) {
    if (supported == nullptr || count == nullptr) return UMAMI_ERROR;
    *supported = supported_inputs;
    *count = UMAMI_INPUT_KEY_COUNT;
    return UMAMI_SUCCESS;
}

UMAMI_EXPORT UmamiStatus umami_required_inputs(bool const **required, int *count) {
    if (required == nullptr || count == nullptr) return UMAMI_ERROR;
    *required = required_inputs;
    *count = UMAMI_INPUT_KEY_COUNT;
    return UMAMI_SUCCESS;
}

UMAMI_EXPORT UmamiStatus umami_supported_outputs(bool const **supported, int *count) {
    if (supported == nullptr || count == nullptr) return UMAMI_ERROR;
    *supported = supported_outputs;
    *count = UMAMI_OUTPUT_KEY_COUNT;
    return UMAMI_SUCCESS;
}

UMAMI_EXPORT UmamiStatus umami_free(UmamiHandle handle) {
    free_instance((Instance *)handle);
    return UMAMI_SUCCESS;
}

// `param_card_path`: the artifact's directory; the plans are read from `<directory>.pacuda`
UMAMI_EXPORT UmamiStatus umami_initialize(UmamiHandle *handle, char const *param_card_path) {
    if (handle == nullptr) return UMAMI_ERROR;
    *handle = nullptr;
    struct stat info;
    if (param_card_path == nullptr || param_card_path[0] != '/' || stat(param_card_path, &info) != 0 ||
        !S_ISDIR(info.st_mode) || umami_provider.process_count == 0 || umami_provider.particle_count > kMaxLegs)
        return UMAMI_ERROR;
    std::string path(param_card_path);
    while (path.size() > 1 && path.back() == '/') path.pop_back();
    path += ".pacuda";
    Instance *in = new Instance();
    std::string why;
    if (!pacuda::read_pacuda(path.c_str(), in->file, why)) {
        fprintf(stderr, "%s: %s\n", kTag, why.c_str());
        free_instance(in);
        return UMAMI_ERROR;
    }
    const PacudaFile &f = in->file;
    if (!f.symjit_sha256.empty()) {
        // a file whose plans need generated (symjit) kernels: this runner has none
        fprintf(stderr, "%s: %s: the plans need %zu generated kernels, which this runner does not have\n", kTag,
                path.c_str(), f.symjit_sha256.size());
        free_instance(in);
        return UMAMI_ERROR;
    }
    bool streams = !cuda_failed(cudaStreamCreateWithFlags(&in->stream, cudaStreamNonBlocking), "stream") &&
                   !cuda_failed(cudaStreamCreateWithFlags(&in->copies, cudaStreamNonBlocking), "stream");
    for (int c = 0; streams && c < kChunks; c++)
        streams = !cuda_failed(cudaEventCreateWithFlags(&in->arrived[c], cudaEventDisableTiming), "event") &&
                  !cuda_failed(cudaEventCreateWithFlags(&in->done[c], cudaEventDisableTiming), "event");
    if (f.kernel > PACMAN_RECURRENCE_KERNEL_MIXED64 || !streams) {
        fprintf(stderr, "%s: kernel kind %u\n", kTag, f.kernel);
        free_instance(in);
        return UMAMI_ERROR;
    }
    // the provider's processes in the file
    in->process.assign(umami_provider.process_count, -1);
    in->alpha_s.assign(umami_provider.process_count, 0.0);
    for (size_t i = 0; i < umami_provider.process_count; i++) {
        const UmamiProcess &entry = umami_provider.processes[i];
        for (size_t k = 0; k < f.processes.size(); k++)
            if (f.processes[k].key == entry.key) in->process[i] = (int)k;
        const PacudaProcess *p = process_of(in, i);
        if (p && (p->legs != umami_provider.particle_count || p->helicities != entry.helicity_count)) {
            fprintf(stderr, "%s: process %s: %u legs and %u helicities in the file, %zu and %zu in the provider\n",
                    kTag, entry.key, p->legs, p->helicities, umami_provider.particle_count, entry.helicity_count);
            free_instance(in);
            return UMAMI_ERROR;
        }
        if (p) in->alpha_s[i] = p->alpha_s;
    }
    // every colour of the file's processes compiled once; their live helicities in one table
    in->colours.resize(f.processes.size());
    std::vector<uint32_t> helicity_table;
    for (size_t k = 0; k < f.processes.size(); k++)
        for (const PacudaColour &c : f.processes[k].colours) {
            Colour col;
            col.c = &c;
            col.live = (uint32_t)c.live_helicity.size();
            col.live_at = (uint32_t)helicity_table.size();
            helicity_table.insert(helicity_table.end(), c.live_helicity.begin(), c.live_helicity.end());
            // the plan as a runner call describes it (the words, widths, planes, constants, forms)
            pacman_recurrence_call call;
            memset(&call, 0, sizeof call);
            call.abi_version = PACMAN_RECURRENCE_ABI;
            call.struct_size = sizeof call;
            call.words = c.words.data();
            call.words_key = pacuda::program_key(c);
            call.word_count = (uint32_t)c.words.size();
            memcpy(call.width, c.width, 8);
            call.scale_re = c.scale_re.data();
            call.scale_im = c.scale_im.data();
            call.factor_re = c.factor_re.data();
            call.factor_im = c.factor_im.data();
            call.current_planes = c.current_planes;
            call.amplitude_planes = c.amplitude_planes;
            call.momentum_planes = c.momentum_planes;
            call.scale_count = (uint32_t)c.scale_re.size();
            call.factor_count = (uint32_t)c.factor_re.size();
            call.external_count = c.external_count;
            call.term_count = (uint32_t)c.term_slots.size();
            call.form_terms = c.form_terms.data();
            call.term_slots = c.term_slots.data();
            call.term_coefficients = c.term_coefficients.data();
            // the reduction over the helicities with planes (an empty plan reduces one zero output)
            static const uint32_t none[2] = {0, 0};
            col.plan = pacuda_b200_plan_create(&call, col.live ? c.live_offsets.data() : none, c.planes.data(),
                                               c.weights.data(), std::max<uint32_t>(col.live, 1), f.kernel);
            if (!col.plan) {
                fprintf(stderr, "%s: process %s, colour %s: the plan does not compile\n", kTag,
                        f.processes[k].key.c_str(), c.id.c_str());
                in->colours[k].push_back(col);
                free_instance(in);
                return UMAMI_ERROR;
            }
            in->colours[k].push_back(col);
        }
    if (!in->live_helicity.reserve(std::max<size_t>(helicity_table.size(), 1)) ||
        cuda_failed(cudaMemcpy(in->live_helicity.p, helicity_table.data(), helicity_table.size() * sizeof(uint32_t),
                               cudaMemcpyHostToDevice),
                    "helicity table")) {
        free_instance(in);
        return UMAMI_ERROR;
    }
    // every contribution's process and colour in the file, and its class
    in->class_of.resize(umami_provider.channel_count);
    for (size_t ch = 0; ch < umami_provider.channel_count; ch++) {
        in->class_of[ch].resize(umami_provider.channels[ch].flavour_count);
        for (size_t fl = 0; fl < umami_provider.channels[ch].flavour_count; fl++) {
            const UmamiFlavour &flavour = umami_provider.channels[ch].flavours[fl];
            for (size_t j = 0; j < flavour.contribution_count; j++) {
                const UmamiContribution *entry = &flavour.contributions[j];
                if (!process_of(in, entry->process_index) || !colour_of(in, entry)) {
                    fprintf(stderr, "%s: process %s, colour %s: not in the file\n", kTag,
                            umami_provider.processes[entry->process_index].key, entry->color_id);
                    free_instance(in);
                    return UMAMI_ERROR;
                }
                for (size_t l = 0; l < umami_provider.particle_count; l++)
                    if (entry->permutation[l] >= umami_provider.particle_count) {
                        free_instance(in);
                        return UMAMI_ERROR;
                    }
                uint32_t c = 0;
                while (c < in->classes.size() && !same_evaluation(in->classes[c].entry, entry)) c++;
                if (c == in->classes.size()) in->classes.push_back(Class{entry, colour_of(in, entry)});
                in->class_of[ch][fl].push_back(c);
            }
        }
    }
    *handle = in;
    return UMAMI_SUCCESS;
}

UMAMI_EXPORT UmamiStatus umami_get_parameter(UmamiHandle handle, char const *name, double *real, double *imaginary) {
    if (handle == nullptr || name == nullptr || real == nullptr) return UMAMI_ERROR;
    Instance *in = (Instance *)handle;
    for (size_t i = 0; i < umami_provider.process_count; ++i) {
        const UmamiParameter *entry = parameter(i, name);
        if (entry == nullptr) continue;
        if (entry->is_complex && imaginary == nullptr) return UMAMI_ERROR;
        const PacudaProcess *p = process_of(in, i);
        bool alpha = alpha_named(p, name);
        double re, im;
        converted_value(p, entry, &re, &im);
        *real = alpha ? in->alpha_s[i] : re;
        if (imaginary != nullptr) *imaginary = alpha ? 0.0 : im;
        return UMAMI_SUCCESS;
    }
    return UMAMI_ERROR;
}

// alpha_s: any value (|M|^2 scales with its power); another mutable parameter: only its value at
// conversion (the file's couplings were computed from it)
UMAMI_EXPORT UmamiStatus umami_set_parameter(UmamiHandle handle, char const *name, double real, double imaginary) {
    if (handle == nullptr || name == nullptr || !isfinite(real)) return UMAMI_ERROR;
    Instance *in = (Instance *)handle;
    bool found = false;
    for (size_t i = 0; i < umami_provider.process_count; ++i) {
        const UmamiParameter *entry = parameter(i, name);
        if (entry == nullptr) continue;
        found = true;
        if (!entry->is_mutable || (entry->is_complex && !isfinite(imaginary))) return UMAMI_ERROR;
        const PacudaProcess *p = process_of(in, i);
        if (alpha_named(p, name)) {
            if (!(real >= 0.0)) return UMAMI_ERROR;
            continue;
        }
        double re, im;
        converted_value(p, entry, &re, &im);
        if (real != re || (entry->is_complex && imaginary != im)) {
            fprintf(stderr, "%s: %s = %.17g: the file was converted with %.17g; convert it again with this value\n",
                    kTag, name, real, re);
            return UMAMI_ERROR;
        }
    }
    if (!found) return UMAMI_ERROR;
    for (size_t i = 0; i < umami_provider.process_count; ++i)
        if (alpha_named(process_of(in, i), name)) in->alpha_s[i] = real;
    return UMAMI_SUCCESS;
}

UMAMI_EXPORT UmamiStatus umami_matrix_element(UmamiHandle handle, size_t count, size_t stride, size_t offset,
                                              size_t input_count, UmamiInputKey const *input_keys,
                                              void const *const *inputs, size_t output_count,
                                              UmamiOutputKey const *output_keys, void *const *outputs) {
    if (handle == nullptr || offset > stride || count > stride - offset ||
        (input_count && (input_keys == nullptr || inputs == nullptr)) ||
        (output_count && (output_keys == nullptr || outputs == nullptr)) ||
        (stride && umami_provider.particle_count > SIZE_MAX / stride / 4) || count > UINT32_MAX)
        return UMAMI_ERROR;
    void const *in_[UMAMI_INPUT_KEY_COUNT] = {nullptr};
    void *out_[UMAMI_OUTPUT_KEY_COUNT] = {nullptr};
    for (size_t i = 0; i < input_count; ++i) {
        int key = input_keys[i];
        if (key < 0 || key >= UMAMI_INPUT_KEY_COUNT || !supported_inputs[key]) return UMAMI_ERROR_UNSUPPORTED_INPUT;
        if (inputs[i] == nullptr || in_[key] != nullptr) return UMAMI_ERROR;
        in_[key] = inputs[i];
    }
    for (size_t i = 0; i < output_count; ++i) {
        int key = output_keys[i];
        if (key < 0 || key >= UMAMI_OUTPUT_KEY_COUNT || !supported_outputs[key]) return UMAMI_ERROR_UNSUPPORTED_OUTPUT;
        if (outputs[i] == nullptr || out_[key] != nullptr) return UMAMI_ERROR;
        out_[key] = outputs[i];
    }
    if (count == 0) return UMAMI_SUCCESS;
    if (in_[UMAMI_IN_MOMENTA] == nullptr) return UMAMI_ERROR_MISSING_INPUT;
    Instance *in = (Instance *)handle;
    const double *momenta = (const double *)in_[UMAMI_IN_MOMENTA];
    const unsigned *channel_in = (const unsigned *)in_[UMAMI_IN_CHANNEL_INDEX];
    const int *flavour_in = (const int *)in_[UMAMI_IN_FLAVOR_INDEX];
    const double *random_in = (const double *)in_[UMAMI_IN_RANDOM_HELICITY];
    const int *helicity_in = (const int *)in_[UMAMI_IN_HELICITY_INDEX];
    const double *alpha_in = (const double *)in_[UMAMI_IN_ALPHA_S];
    const int mode = helicity_in ? MODE_HELICITY : out_[UMAMI_OUT_HELICITY_INDEX] ? MODE_SAMPLE : MODE_SUM;

    // The call in chunks of events. Per chunk the host checks its events (as the reference checks
    // them), groups its items by class and queues its device work, then goes on with the next
    // chunk while the device runs; a chunk's events are combined as soon as its results are back.
    // Nothing reaches the caller's outputs until every chunk has been checked and every momentum
    // found finite, as in the reference (which checks all inputs before it evaluates).
    const size_t n = umami_provider.particle_count, nclasses = in->classes.size();
    const size_t nchunks = std::min<size_t>(kChunks, std::max<size_t>(1, count / kChunkEvents));
    // every buffer at its largest for this call, before anything is queued
    size_t most_items = 0, most_values = 1;
    for (size_t c = 0; c < umami_provider.channel_count; c++)
        for (size_t f = 0; f < umami_provider.channels[c].flavour_count; f++)
            most_items = std::max(most_items, umami_provider.channels[c].flavours[f].contribution_count);
    for (const Class &cls : in->classes) most_values = std::max<size_t>(most_values, cls.colour->live);
    const size_t cap = count * most_items;
    if (!in->momenta.reserve(4 * n * count) || !in->items.reserve(cap) || !in->value_out.reserve(cap) ||
        !in->chosen_out.reserve(cap) || !in->host_items.reserve(cap) || !in->host_value.reserve(cap) ||
        !in->host_chosen.reserve(cap) || !in->bad.reserve(1) || !in->host_bad.reserve(1) ||
        !in->groups.reserve(kChunks * nclasses) || !in->host_groups.reserve(kChunks * nclasses) ||
        !in->external.reserve(4 * n * cap) || !in->values.reserve(most_values * cap))
        return UMAMI_ERROR;
    auto drain = [&]() {  // queued copies read the caller's memory: they end before the call returns
        bool ok = !cuda_failed(cudaStreamSynchronize(in->stream), "evaluation");
        return !cuda_failed(cudaStreamSynchronize(in->copies), "copies") && ok;
    };
    in->host_bad.p[0] = 0;
    if (cuda_failed(cudaMemcpyAsync(in->bad.p, in->host_bad.p, sizeof(int), cudaMemcpyHostToDevice, in->copies),
                    "flag"))
        return drain(), UMAMI_ERROR;
    std::vector<Chunk> chunks(nchunks);
    if (in->selection.size() < count) in->selection.resize(count);
    if (in->at.size() < cap) in->at.resize(cap);
    uint32_t *selection = in->selection.data();  // per event: channel << 16 | flavour
    uint32_t *at = in->at.data();                // per event-ordered item: its place among the items
    size_t items_so_far = 0, ext = 0, vals = 0;
    for (size_t c = 0; c < nchunks; c++) {
        Chunk &ch = chunks[c];
        ch.e0 = nchunks == kChunks ? count * kChunkParts[c] / kChunkWhole : count * c / nchunks;
        ch.e1 = nchunks == kChunks ? count * kChunkParts[c + 1] / kChunkWhole : count * (c + 1) / nchunks;
        ch.item0 = items_so_far;
        ch.first.assign(nclasses + 1, 0);
        // its events' selections and its item count per class
        for (size_t e = ch.e0; e < ch.e1; ++e) {
            size_t event = offset + e;
            size_t channel = channel_in ? channel_in[event] : 0;
            int flavour = flavour_in ? flavour_in[event] : 0;
            if (channel >= umami_provider.channel_count || flavour < 0 ||
                (size_t)flavour >= umami_provider.channels[channel].flavour_count)
                return drain(), UMAMI_ERROR;
            const UmamiFlavour &sel = umami_provider.channels[channel].flavours[flavour];
            if (sel.contribution_count == 0 || channel > 0xffff || flavour > 0xffff) return drain(), UMAMI_ERROR;
            double random = random_in ? random_in[event] : 0.5;
            if (!isfinite(random) || random < 0.0 || random >= 1.0) return drain(), UMAMI_ERROR;
            if (helicity_in) {
                int label = helicity_in[event];
                if (label < 0 || (size_t)label >= umami_provider.exported_helicity_count) return drain(), UMAMI_ERROR;
            } else if (out_[UMAMI_OUT_HELICITY_INDEX] && sel.contribution_count != 1) {
                return drain(), UMAMI_ERROR_UNSUPPORTED_OUTPUT;
            }
            for (size_t j = 0; j < sel.contribution_count; ++j) {
                const UmamiContribution *entry = &sel.contributions[j];
                if (alpha_in) {
                    double a = alpha_in[event];
                    if (!isfinite(a) || a < 0.0) return drain(), UMAMI_ERROR;
                    if (process_of(in, entry->process_index)->alpha_s_name.empty())
                        return drain(), UMAMI_ERROR_UNSUPPORTED_INPUT;
                }
                ch.first[in->class_of[channel][flavour][j] + 1]++;
            }
            items_so_far += sel.contribution_count;
            selection[e] = (uint32_t)channel << 16 | (uint32_t)flavour;
        }
        ch.items = items_so_far - ch.item0;
        ch.external = ext;
        ch.values = vals;
        for (size_t k = 0; k < nclasses; k++) {
            size_t m = ch.first[k + 1];
            ext += 4 * n * m;
            vals += (size_t)std::max<uint32_t>(in->classes[k].colour->live, 1) * m;
            ch.first[k + 1] += ch.first[k];
        }
        // its items grouped by class, events in order within a class (a counting sort)
        std::vector<uint32_t> next(ch.first.begin(), ch.first.end() - 1);
        for (size_t e = ch.e0, k = ch.item0; e < ch.e1; ++e) {
            size_t event = offset + e, channel = selection[e] >> 16, flavour = selection[e] & 0xffff;
            const UmamiFlavour &sel = umami_provider.channels[channel].flavours[flavour];
            for (size_t j = 0; j < sel.contribution_count; ++j, ++k) {
                const UmamiContribution *entry = &sel.contributions[j];
                const PacudaProcess *p = process_of(in, entry->process_index);
                double a = alpha_in ? alpha_in[event] : in->alpha_s[entry->process_index];
                double scale = 1.0;
                if (!p->alpha_s_name.empty() && a != p->alpha_s) scale = pow(a / p->alpha_s, p->qcd_power);
                uint32_t place = next[in->class_of[channel][flavour][j]]++;
                at[k] = (uint32_t)ch.item0 + place;
                ItemIn &it = in->host_items.p[ch.item0 + place];
                it.event = (uint32_t)(e - ch.e0);
                it.helicity = helicity_in ? entry->helicity_runtime[helicity_in[event]] : -1;
                it.scale = scale;
                it.random = random_in ? random_in[event] : 0.5;
            }
        }
        if (launch_chunk(in, (int)c, ch, momenta, stride, offset, mode) != UMAMI_SUCCESS ||
            cuda_failed(cudaEventRecord(in->done[c], in->stream), "event"))
            return drain(), UMAMI_ERROR;
    }
    // every momentum's check is on the copy stream, well ahead of the evaluation: the call's
    // verdict on them comes before any output is written (as the reference checks them all first)
    if (cuda_failed(cudaMemcpyAsync(in->host_bad.p, in->bad.p, sizeof(int), cudaMemcpyDeviceToHost, in->copies),
                    "flag") ||
        cuda_failed(cudaStreamSynchronize(in->copies), "copies"))
        return drain(), UMAMI_ERROR;
    if (in->host_bad.p[0]) return drain(), UMAMI_ERROR;  // a momentum that is not finite

    // the events combined as the reference does, chunk by chunk as the results come back, into
    // the outputs; the first event whose |M|^2 is not finite ends the call (the events before it
    // are written)
    double *me_out = (double *)out_[UMAMI_OUT_MATRIX_ELEMENT];
    int *hel_out = (int *)out_[UMAMI_OUT_HELICITY_INDEX], *col_out = (int *)out_[UMAMI_OUT_COLOR_INDEX];
    for (size_t c = 0; c < nchunks; c++) {
        if (cuda_failed(cudaEventSynchronize(in->done[c]), "evaluation")) return drain(), UMAMI_ERROR;
        const Chunk &ch = chunks[c];
        const double *value = in->host_value.p;
        for (size_t e = ch.e0, k = ch.item0; e < ch.e1; ++e) {
            size_t event = offset + e;
            const UmamiFlavour &sel = umami_provider.channels[selection[e] >> 16].flavours[selection[e] & 0xffff];
            const UmamiContribution *head = &sel.contributions[0];
            int label = 0;
            double total = 0.0;
            if (mode == MODE_HELICITY) {
                label = helicity_in[event];
                for (size_t j = 0; j < sel.contribution_count; ++j) {
                    const UmamiContribution *entry = &sel.contributions[j];
                    if (entry->helicity_runtime[label] < 0) continue;
                    total += entry->factor * value[at[k + j]];
                }
            } else if (mode == MODE_SAMPLE) {
                total = value[at[k]];
                label = head->helicity_export[in->host_chosen.p[at[k]]];
                total *= head->factor;
            } else {
                for (size_t j = 0; j < sel.contribution_count; ++j)
                    total += sel.contributions[j].factor * value[at[k + j]];
            }
            k += sel.contribution_count;
            if (!isfinite(total)) return drain(), UMAMI_ERROR;
            if (me_out) me_out[event] = total;
            if (hel_out) hel_out[event] = label;
            if (col_out) col_out[event] = (int)head->color_index;
        }
    }
    if (!drain()) return UMAMI_ERROR;
    return UMAMI_SUCCESS;
}
