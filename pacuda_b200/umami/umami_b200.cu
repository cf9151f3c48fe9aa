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
//      n * k + leg for component k of a leg, one value per event);
//   3. gathers every group's external momenta on the device (the permutation and the process's
//      crossing applied: external leg l = sign_l x input leg permutation[crossing_l]);
//   4. evaluates every group in ONE persistent launch of the batched executor, each point's
//      helicity values reduced in the kernel from its amplitudes (pacuda_b200_batch_*);
//   5. copies the helicity values back and combines the events on the host exactly as the
//      reference does: the process-group factor, the alpha_s scale, then a fixed helicity, the
//      helicity sum, or the helicity drawn in proportion to its value (the arithmetic and order
//      of the reference's reduce_sample, recurrence_runner.cu:1532-1572).
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

// one group's gather: external[(l * 4 + k) * points + q] = sign[l] * momenta[(legs * k + leg[l]) * events + event[q]]
struct Gather {
    unsigned long long external;  // offset of the group's planes in the external buffer
    unsigned long long first;     // offset of its events in the event list
    uint32_t points, legs;
    uint32_t leg[kMaxLegs];
    double sign[kMaxLegs];
};

__global__ void gather_groups(const Gather *groups, uint32_t ngroups, const double *momenta, size_t events,
                              const uint32_t *event, double *external) {
    const Gather &g = groups[blockIdx.y];
    (void)ngroups;
    const size_t n = (size_t)g.points * g.legs * 4;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        size_t q = i % g.points, lk = i / g.points;
        uint32_t l = (uint32_t)(lk >> 2), k = (uint32_t)(lk & 3);
        double v = momenta[((size_t)g.legs * k + g.leg[l]) * events + event[g.first + q]];
        external[g.external + i] = g.sign[l] * v;
    }
}

struct Colour {
    const PacudaColour *c = nullptr;
    pacuda_b200_plan *plan = nullptr;
    uint32_t live = 0;  // outputs of the plan (the helicities with planes)
};

struct Instance {
    PacudaFile file;
    std::vector<int> process;       // per provider process: its file process, or -1
    std::vector<double> alpha_s;    // per provider process
    std::vector<std::vector<Colour>> colours;  // [file process][colour]
    cudaStream_t stream = nullptr;
    // the call's device and host buffers
    DeviceArray<double> momenta, external, values;
    DeviceArray<uint32_t> events;
    DeviceArray<Gather> gathers;
    PinnedArray<double> host_values;
    PinnedArray<uint32_t> host_events;
    PinnedArray<Gather> host_gathers;
    // the batch of the last call's groups (reused while the groups' plans repeat)
    pacuda_b200_batch *batch = nullptr;
    std::vector<pacuda_b200_plan *> batch_plans;
};

// One evaluation: an event's contribution.
struct Item {
    size_t event;
    const UmamiContribution *contribution;
    double scale;   // (alpha_s / alpha_s at conversion) ^ QCD power
    double random;  // the helicity's random number
    size_t values;  // its helicity values, offset into the call's value list (not sampling)
    double total;   // sampling: the sum of the helicity values and the helicity drawn
    uint32_t chosen;
    size_t index;   // its position among the event-ordered items
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
    pacuda_b200_batch_destroy(in->batch);
    for (auto &v : in->colours)
        for (Colour &c : v) pacuda_b200_plan_destroy(c.plan);
    in->momenta.release();
    in->external.release();
    in->values.release();
    in->events.release();
    in->gathers.release();
    in->host_values.release();
    in->host_events.release();
    in->host_gathers.release();
    if (in->stream) cudaStreamDestroy(in->stream);
    delete in;
}

// items alike when they share the process, the colour id and the leg permutation
int compare_evaluation(const UmamiContribution *x, const UmamiContribution *y) {
    if (x == y) return 0;
    if (x->process_index != y->process_index) return x->process_index < y->process_index ? -1 : 1;
    int c = strcmp(x->color_id, y->color_id);
    if (c != 0) return c;
    return memcmp(x->permutation, y->permutation, umami_provider.particle_count * sizeof(size_t));
}

// The helicity values of every group of `sorted` (groups: [first, end) ranges), in one batched
// launch: values of group g's point q at group_values[g] + q * live.
UmamiStatus evaluate_groups(Instance *in, const std::vector<Item> &sorted, const std::vector<size_t> &bounds,
                            const double *momenta, size_t stride, size_t offset, size_t count,
                            std::vector<size_t> &group_values) {
    const size_t n = umami_provider.particle_count, groups = bounds.size() - 1;
    // 2. the events' momenta, as the caller lays them out, rows offset .. offset + count
    if (!in->momenta.reserve(4 * n * count)) return UMAMI_ERROR;
    if (cuda_failed(cudaMemcpy2DAsync(in->momenta.p, count * sizeof(double), momenta + offset, stride * sizeof(double),
                                      count * sizeof(double), 4 * n, cudaMemcpyHostToDevice, in->stream),
                    "momenta"))
        return UMAMI_ERROR;
    // 3. the groups' gathers and their points' events
    if (!in->host_gathers.reserve(groups) || !in->host_events.reserve(sorted.size()) ||
        !in->gathers.reserve(groups) || !in->events.reserve(sorted.size()))
        return UMAMI_ERROR;
    std::vector<pacuda_b200_plan *> plans(groups);
    std::vector<uint32_t> points(groups);
    size_t ext = 0, vals = 0;
    group_values.assign(groups, 0);
    std::vector<size_t> ext_at(groups);
    for (size_t g = 0; g < groups; g++) {
        const Item &first = sorted[bounds[g]];
        const UmamiContribution *entry = first.contribution;
        const PacudaProcess *p = process_of(in, entry->process_index);
        const Colour *col = colour_of(in, entry);
        Gather &G = in->host_gathers.p[g];
        memset(&G, 0, sizeof G);
        G.external = ext;
        G.first = bounds[g];
        G.points = (uint32_t)(bounds[g + 1] - bounds[g]);
        G.legs = (uint32_t)n;
        for (size_t l = 0; l < n; l++) {
            size_t source = p->crossing_leg.empty() ? l : p->crossing_leg[l];
            G.leg[l] = (uint32_t)entry->permutation[source];
            G.sign[l] = p->crossing_leg.empty() ? 1.0 : p->crossing_sign[l];
        }
        plans[g] = col->plan;
        points[g] = G.points;
        ext_at[g] = ext;
        group_values[g] = vals;
        ext += 4 * n * G.points;
        vals += (size_t)std::max<uint32_t>(col->live, 1) * G.points;
    }
    for (size_t j = 0; j < sorted.size(); j++) in->host_events.p[j] = (uint32_t)(sorted[j].event - offset);
    if (!in->external.reserve(ext) || !in->values.reserve(vals) || !in->host_values.reserve(vals)) return UMAMI_ERROR;
    if (cuda_failed(cudaMemcpyAsync(in->gathers.p, in->host_gathers.p, groups * sizeof(Gather), cudaMemcpyHostToDevice,
                                    in->stream),
                    "gathers") ||
        cuda_failed(cudaMemcpyAsync(in->events.p, in->host_events.p, sorted.size() * sizeof(uint32_t),
                                    cudaMemcpyHostToDevice, in->stream),
                    "events"))
        return UMAMI_ERROR;
    uint32_t most = *std::max_element(points.begin(), points.end());
    dim3 grid((unsigned)std::min<size_t>((4 * n * most + 255) / 256, 4096), (unsigned)groups);
    gather_groups<<<grid, 256, 0, in->stream>>>(in->gathers.p, (uint32_t)groups, in->momenta.p, count, in->events.p,
                                                in->external.p);
    if (cuda_failed(cudaGetLastError(), "gather")) return UMAMI_ERROR;
    // 4. one launch over every group (the batch of the previous call re-pointed when its plans repeat)
    std::vector<const double *> ext_p(groups);
    std::vector<double *> out_p(groups);
    for (size_t g = 0; g < groups; g++) {
        ext_p[g] = in->external.p + ext_at[g];
        out_p[g] = in->values.p + group_values[g];
    }
    if (in->batch && in->batch_plans == plans) {
        if (pacuda_b200_batch_update(in->batch, ext_p.data(), points.data(), out_p.data()) != PACMAN_RECURRENCE_OK)
            return UMAMI_ERROR;
    } else {
        if (in->batch) {
            cudaStreamSynchronize(in->stream);
            pacuda_b200_batch_destroy(in->batch);
        }
        in->batch = pacuda_b200_batch_create(plans.data(), (uint32_t)groups, ext_p.data(), points.data(), out_p.data());
        in->batch_plans = in->batch ? plans : std::vector<pacuda_b200_plan *>();
        if (!in->batch) return UMAMI_ERROR;
    }
    if (pacuda_b200_batch_run(in->batch, in->stream) != PACMAN_RECURRENCE_OK) return UMAMI_ERROR;
    // 5. the helicity values back
    if (cuda_failed(cudaMemcpyAsync(in->host_values.p, in->values.p, vals * sizeof(double), cudaMemcpyDeviceToHost,
                                    in->stream),
                    "values") ||
        cuda_failed(cudaStreamSynchronize(in->stream), "evaluation"))
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
    if (f.kernel > PACMAN_RECURRENCE_KERNEL_MIXED64 ||
        cuda_failed(cudaStreamCreateWithFlags(&in->stream, cudaStreamNonBlocking), "stream")) {
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
    // every colour of the file's processes compiled once
    in->colours.resize(f.processes.size());
    for (size_t k = 0; k < f.processes.size(); k++)
        for (const PacudaColour &c : f.processes[k].colours) {
            Colour col;
            col.c = &c;
            col.live = (uint32_t)c.live_helicity.size();
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
    // every contribution's process and colour in the file
    for (size_t ch = 0; ch < umami_provider.channel_count; ch++)
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
    const size_t n = umami_provider.particle_count;
    auto selection_of = [&](size_t event) -> const UmamiFlavour * {
        size_t channel = channel_in ? channel_in[event] : 0;
        int flavour = flavour_in ? flavour_in[event] : 0;
        if (channel >= umami_provider.channel_count || flavour < 0 ||
            (size_t)flavour >= umami_provider.channels[channel].flavour_count)
            return nullptr;
        return &umami_provider.channels[channel].flavours[flavour];
    };

    // 1. the items: every event's contributions, in event order
    bool sample = !helicity_in && out_[UMAMI_OUT_HELICITY_INDEX];
    std::vector<Item> items;
    size_t value_count = 0;
    for (size_t event = offset; event < offset + count; ++event) {
        const UmamiFlavour *selection = selection_of(event);
        if (!selection || selection->contribution_count == 0) return UMAMI_ERROR;
        double random = random_in ? random_in[event] : 0.5;
        if (!isfinite(random) || random < 0.0 || random >= 1.0) return UMAMI_ERROR;
        if (helicity_in) {
            int label = helicity_in[event];
            if (label < 0 || (size_t)label >= umami_provider.exported_helicity_count) return UMAMI_ERROR;
        } else if (out_[UMAMI_OUT_HELICITY_INDEX] && selection->contribution_count != 1) {
            return UMAMI_ERROR_UNSUPPORTED_OUTPUT;
        }
        for (size_t l = 0; l < n; l++)
            for (size_t k = 0; k < 4; k++)
                if (!isfinite(momenta[event + stride * (n * k + l)])) return UMAMI_ERROR;
        for (size_t j = 0; j < selection->contribution_count; ++j) {
            const UmamiContribution *entry = &selection->contributions[j];
            const PacudaProcess *p = process_of(in, entry->process_index);
            double a = in->alpha_s[entry->process_index];
            if (alpha_in) {
                a = alpha_in[event];
                if (!isfinite(a) || a < 0.0) return UMAMI_ERROR;
                if (p->alpha_s_name.empty()) return UMAMI_ERROR_UNSUPPORTED_INPUT;
            }
            double scale = 1.0;
            if (!p->alpha_s_name.empty() && a != p->alpha_s) scale = pow(a / p->alpha_s, p->qcd_power);
            Item it{event, entry, scale, random, value_count, 0.0, 0, items.size()};
            items.push_back(it);
            if (!sample) value_count += p->helicities;
        }
    }
    // the groups: items by (process, colour, permutation), events in order within each
    std::vector<Item> sorted(items);
    std::stable_sort(sorted.begin(), sorted.end(), [](const Item &x, const Item &y) {
        return compare_evaluation(x.contribution, y.contribution) < 0;
    });
    std::vector<size_t> bounds{0};
    for (size_t j = 1; j < sorted.size(); j++)
        if (compare_evaluation(sorted[j].contribution, sorted[j - 1].contribution) != 0) bounds.push_back(j);
    bounds.push_back(sorted.size());
    std::vector<size_t> group_values;
    UmamiStatus status = evaluate_groups(in, sorted, bounds, momenta, stride, offset, count, group_values);
    if (status != UMAMI_SUCCESS) return status;

    // each item's helicity values (or its draw), from its group's reduced values
    std::vector<double> values(std::max<size_t>(value_count, 1), 0.0);
    for (size_t g = 0; g + 1 < bounds.size(); g++) {
        const UmamiContribution *entry = sorted[bounds[g]].contribution;
        const PacudaProcess *p = process_of(in, entry->process_index);
        const Colour *col = colour_of(in, entry);
        const PacudaColour &c = *col->c;
        const size_t live = col->live;
        const bool factor = p->numerator != p->denominator;
        for (size_t j = bounds[g]; j < bounds[g + 1]; j++) {
            Item &item = sorted[j];
            const double *v = in->host_values.p + group_values[g] + (j - bounds[g]) * std::max<size_t>(live, 1);
            if (sample) {
                // the helicity drawn in proportion to its value, as the reference's device sampling
                auto value = [&](size_t o) {
                    double acc = v[o];
                    if (factor) acc = acc * (double)p->numerator / (double)p->denominator;
                    if (item.scale != 1.0) acc = acc * item.scale;
                    return acc;
                };
                double t = 0.0;
                for (size_t o = 0; o < live; o++) t = t + value(o);
                double target = item.random * t, cumulative = 0.0;
                uint32_t pick = 0;
                for (size_t o = 0; o < live; o++) {
                    double x = value(o);
                    if (x <= 0.0) continue;
                    pick = c.live_helicity[o];
                    cumulative = cumulative + x;
                    if (cumulative > target) break;
                }
                item.total = live ? t : 0.0;
                item.chosen = live ? pick : 0;
                items[item.index].total = item.total;
                items[item.index].chosen = item.chosen;
                continue;
            }
            double *dst = values.data() + item.values;
            for (size_t k = 0; k < live; k++) {
                double x = v[k];
                if (factor) x = x * (double)p->numerator / (double)p->denominator;
                if (item.scale != 1.0) x *= item.scale;
                dst[c.live_helicity[k]] = x;
            }
        }
    }

    // the events, combined as the reference does
    size_t k = 0;
    for (size_t event = offset; event < offset + count; ++event) {
        const UmamiFlavour *selection = selection_of(event);
        const UmamiContribution *first = &selection->contributions[0];
        int label = 0;
        double total = 0.0;
        if (helicity_in) {
            label = helicity_in[event];
            for (size_t j = 0; j < selection->contribution_count; ++j) {
                const UmamiContribution *entry = &selection->contributions[j];
                if (entry->helicity_runtime[label] < 0) continue;
                total += entry->factor * values[items[k + j].values + entry->helicity_runtime[label]];
            }
        } else if (out_[UMAMI_OUT_HELICITY_INDEX]) {
            total = items[k].total;
            label = first->helicity_export[items[k].chosen];
            total *= first->factor;
        } else {
            for (size_t j = 0; j < selection->contribution_count; ++j) {
                const UmamiContribution *entry = &selection->contributions[j];
                size_t h = process_of(in, entry->process_index)->helicities;
                const double *v = values.data() + items[k + j].values;
                double value = 0.0;
                for (size_t hel = 0; hel < h; ++hel) value += v[hel];
                total += entry->factor * value;
            }
        }
        k += selection->contribution_count;
        if (!isfinite(total)) return UMAMI_ERROR;
        if (out_[UMAMI_OUT_MATRIX_ELEMENT]) ((double *)out_[UMAMI_OUT_MATRIX_ELEMENT])[event] = total;
        if (out_[UMAMI_OUT_HELICITY_INDEX]) ((int *)out_[UMAMI_OUT_HELICITY_INDEX])[event] = label;
        if (out_[UMAMI_OUT_COLOR_INDEX]) ((int *)out_[UMAMI_OUT_COLOR_INDEX])[event] = (int)first->color_index;
    }
    return UMAMI_SUCCESS;
}
