// pacuda-b200 recurrence runner: the C ABI of librecurrence.so (include/pacman_recurrence.h) on
// B200 (sm_100a).
//
// One call runs a plan over a tile of phase-space points. The device work of a call is one
// fused kernel per plan run: the momentum forms from the external momenta, the external
// wavefunctions (op 12), the rows, and the closures into the amplitude arena; the reductions
// (LC diagonal, resolved per helicity, helicity sampling) are one kernel each. All copies and
// kernels of a call go on one stream that the call synchronises once at its end.
//
// The device state is the reference's (runner/recurrence_runner.cu:886-910): one process-wide
// current arena and amplitude arena, plane-major with the call's stride, that persist between
// calls; only the runs a call names are copied; an arena that has to grow loses its contents.
// Programs are compiled once per nonzero words_key. Calls are serialised by one lock, and a run
// that keeps its amplitudes holds the lock until the same thread's reduction (:1725-1755).
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "../../include/pacman_recurrence.h"
#include "../../include/pacuda_b200.h"
#include "arith.cuh"
#include "executor.cuh"
#include "program.h"
#include "tiled.cuh"
#include "tiled_host.h"

using namespace pacuda;

namespace {

const char *const kTag = "pacman recurrence runner (pacuda-b200)";

bool failed(cudaError_t e, const char *step) {
    if (e == cudaSuccess) return false;
    fprintf(stderr, "%s: %s: %s\n", kTag, step, cudaGetErrorString(e));
    return true;
}

// ---- conversions between the f64 transfer layout and a kind's layout -------------------------

// n planes of `points` values (plane stride `ld`), f64 -> the layout in place (df64) or into
// `dst` (mixed: f32 planes)
template <class T>
__global__ void to_layout_planes(const double *src, T *dst, size_t planes, size_t ld, size_t points) {
    size_t total = planes * points;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        size_t at = k / points * ld + k % points;
        double x = src[at];
        dst[at] = narrow<T>(x);
    }
}
template <class T>
__global__ void to_f64_planes(const T *src, double *dst, size_t planes, size_t ld, size_t points) {
    size_t total = planes * points;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        size_t at = k / points * ld + k % points;
        dst[at] = widen64(src[at]);
    }
}

unsigned grid_for(size_t n, unsigned block) { return (unsigned)std::min<size_t>(8192, (n + block - 1) / block); }

// ---- reductions (reference: recurrence_runner.cu:1489-1572) ----------------------------------
__device__ __forceinline__ double as_f64(double x) { return x; }
__device__ __forceinline__ double as_f64(D x) { return __dadd_rn((double)x.hi, (double)x.lo); }
__device__ __forceinline__ double lc_term(double w, double re, double im) {
    return __dmul_rn(w, __fma_rn(re, re, __dmul_rn(im, im)));
}

template <class A>
__global__ void reduce_kernel(const A *are, const A *aim, size_t ld, const uint32_t *planes, const double *weights,
                              uint32_t count, double *output, uint32_t points) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= points) return;
    double acc = output[i];
    for (uint32_t k = 0; k < count; k++) {
        size_t at = (size_t)__ldg(planes + k) * ld + i;
        acc = __dadd_rn(acc, lc_term(__ldg(weights + k), as_f64(are[at]), as_f64(aim[at])));
    }
    output[i] = acc;
}

// one thread per point, all outputs in turn: output o at out[o * os + i * ps]
template <class A>
__global__ void reduce_resolved_kernel(const A *are, const A *aim, size_t ld, const uint32_t *planes,
                                       const double *weights, const uint32_t *offsets, uint32_t outputs,
                                       double *out, uint32_t points, size_t os, size_t ps, bool zero) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= points) return;
    for (uint32_t o = 0; o < outputs; o++) {
        size_t at_out = o * os + i * ps;
        double acc = zero ? 0.0 : out[at_out];
        for (uint32_t k = __ldg(offsets + o), end = __ldg(offsets + o + 1); k < end; k++) {
            size_t at = (size_t)__ldg(planes + k) * ld + i;
            acc = __dadd_rn(acc, lc_term(__ldg(weights + k), as_f64(are[at]), as_f64(aim[at])));
        }
        out[at_out] = acc;
    }
}

template <class A>
__device__ __forceinline__ double sample_value(const A *are, const A *aim, size_t ld, const uint32_t *planes,
                                               const double *weights, uint32_t first, uint32_t end, size_t i,
                                               bool factor, double num, double den, double scale) {
    double acc = 0.0;
    for (uint32_t k = first; k < end; k++) {
        size_t at = (size_t)__ldg(planes + k) * ld + i;
        acc = __dadd_rn(acc, lc_term(__ldg(weights + k), as_f64(are[at]), as_f64(aim[at])));
    }
    if (factor) acc = __ddiv_rn(__dmul_rn(acc, num), den);
    if (scale != 1.0) acc = __dmul_rn(acc, scale);
    return acc;
}

template <class A>
__global__ void reduce_sample_kernel(const A *are, const A *aim, size_t ld, const uint32_t *planes,
                                     const double *weights, const uint32_t *offsets, const uint32_t *helicity,
                                     uint32_t outputs, uint32_t points, const double *random, const double *scale,
                                     bool factor, double num, double den, double *total, uint32_t *chosen) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= points) return;
    double s = scale ? scale[i] : 1.0;
    double t = 0.0;
    for (uint32_t o = 0; o < outputs; o++)
        t = __dadd_rn(t, sample_value(are, aim, ld, planes, weights, __ldg(offsets + o), __ldg(offsets + o + 1), i,
                                      factor, num, den, s));
    double target = __dmul_rn(random[i], t), cumulative = 0.0;
    uint32_t pick = 0;
    for (uint32_t o = 0; o < outputs; o++) {
        double v = sample_value(are, aim, ld, planes, weights, __ldg(offsets + o), __ldg(offsets + o + 1), i, factor,
                                num, den, s);
        if (v <= 0.0) continue;
        pick = __ldg(helicity + o);
        cumulative = __dadd_rn(cumulative, v);
        if (cumulative > target) break;
    }
    total[i] = t;
    chosen[i] = pick;
}

__global__ void test_sources_kernel(const uint32_t *codes, const double *masses, const double *momenta,
                                    uint32_t count, double *out_re, double *out_im) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    W v[4] = {w64(0.0, 0.0), w64(0.0, 0.0), w64(0.0, 0.0), w64(0.0, 0.0)};
    double p[4] = {momenta[4 * (size_t)i], momenta[4 * (size_t)i + 1], momenta[4 * (size_t)i + 2],
                   momenta[4 * (size_t)i + 3]};
    source_values(codes[i], masses[i], p, v);
    for (int k = 0; k < 4; k++) {
        out_re[4 * (size_t)i + k] = v[k].re;
        out_im[4 * (size_t)i + k] = v[k].im;
    }
}

// ---- device state ------------------------------------------------------------------------------

struct Buffer {
    void *p = nullptr;
    size_t bytes = 0;
    // at least `n` bytes; a grown buffer loses its contents
    bool reserve(size_t n, const char *what) {
        if (n <= bytes) return true;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (failed(cudaMalloc(&p, std::max<size_t>(n, 16)), what)) return false;
        bytes = std::max<size_t>(n, 16);
        return true;
    }
    template <class T> T *as() const { return (T *)p; }
};

struct DeviceProgram {
    Program host;
    Ins *ins = nullptr;
    // the on-chip executor's schedule: 0 not built yet, 1 built, -1 none
    int tiled_state = 0;
    TiledDevice tiled;
};

enum { KERNEL_DF64 = PACMAN_RECURRENCE_KERNEL_DF64, KERNEL_F64 = PACMAN_RECURRENCE_KERNEL_F64,
       KERNEL_MIXED = PACMAN_RECURRENCE_KERNEL_MIXED, KERNEL_MIXED64 = PACMAN_RECURRENCE_KERNEL_MIXED64 };

struct Options {
    int kernel = KERNEL_DF64;  // the reference's default
    int block = 0;             // 0: the runner's choice
    bool sort = true;
    int executor = PACUDA_B200_EXECUTOR_AUTO;
    uint32_t lanes_per_point = 0;
};

struct Device {
    cudaStream_t stream = nullptr;
    int sms = 0;
    // arenas: currents (8 bytes per value: f64 or df64; mixed keeps f32 planes in fcur and uses
    // cur for transfers), amplitudes (8 bytes: f64 or df64), forms, staging for downloads
    Buffer cre, cim, fcre, fcim, are, aim, mom, stage;
    size_t cur_values = 0, amp_values = 0;  // the arenas' valid sizes (values)
    Buffer external, terms, consts;
    // the on-chip executor's launch descriptors (pinned host and device copies)
    unsigned char *launch_host = nullptr;
    Buffer launch_dev;
    // kept amplitudes (for one reduction)
    bool kept = false;
    int kept_kernel = KERNEL_F64;
    size_t kept_stride = 0, kept_points = 0, kept_planes = 0;
    Buffer rplanes, rweights, roffsets, rhelicity, routput, rrandom, rscale, rtotal, rchosen;
    std::unordered_map<uint64_t, DeviceProgram> programs;
    DeviceProgram scratch;
    // statistics
    bool stats = false;
    uint64_t calls = 0, points = 0, copies = 0, bytes = 0, reductions = 0;
    double seconds = 0;
};

Device dev;
Options current;
bool runs_started = false;

double now() {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + t.tv_nsec * 1e-9;
}

void print_stats() {
    if (!dev.stats || dev.calls == 0) return;
    fprintf(stderr, "%s: %llu calls, %llu points, %llu reductions, %llu copies (%.1f MB), %.3f s (%.2f us/point)\n",
            kTag, (unsigned long long)dev.calls, (unsigned long long)dev.points, (unsigned long long)dev.reductions,
            (unsigned long long)dev.copies, dev.bytes / 1e6, dev.seconds,
            dev.points ? dev.seconds * 1e6 / dev.points : 0.0);
}

bool initialize() {
    if (dev.stream) return true;
    if (failed(cudaStreamCreateWithFlags(&dev.stream, cudaStreamNonBlocking), "stream")) return false;
    int d = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&dev.sms, cudaDevAttrMultiProcessorCount, d);
    atexit(print_stats);
    return true;
}

// ---- copies ----------------------------------------------------------------------------------

bool copy_planes(void *dst, const void *src, size_t n, size_t ld, size_t points, cudaMemcpyKind kind) {
    if (n == 0) return true;
    size_t pitch = ld * sizeof(double);
    if (failed(cudaMemcpy2DAsync(dst, pitch, src, pitch, points * sizeof(double), n, kind, dev.stream), "copy"))
        return false;
    dev.copies++;
    dev.bytes += n * points * sizeof(double);
    return true;
}

// the run list's planes must lie in the arena (the reference reports a bad run as a device error,
// recurrence_runner.cu:1096)
bool runs_valid(const uint32_t *runs, uint32_t count, uint32_t planes) {
    for (uint32_t r = 0; r < count; r++) {
        uint32_t first = runs[2 * r], n = runs[2 * r + 1];
        if (first > planes || n > planes - first) return false;
    }
    return true;
}

template <class T> bool convert_in(const double *src, T *dst, const uint32_t *runs, uint32_t count, size_t ld,
                                   size_t points) {
    for (uint32_t r = 0; r < count; r++) {
        size_t off = (size_t)runs[2 * r] * ld, n = runs[2 * r + 1];
        if (n == 0) continue;
        to_layout_planes<T><<<grid_for(n * points, 256), 256, 0, dev.stream>>>(src + off, dst + off, n, ld, points);
    }
    return !failed(cudaGetLastError(), "conversion");
}

template <class T> bool convert_out(const T *src, double *dst, const uint32_t *runs, uint32_t count, size_t ld,
                                    size_t points) {
    for (uint32_t r = 0; r < count; r++) {
        size_t off = (size_t)runs[2 * r] * ld, n = runs[2 * r + 1];
        if (n == 0) continue;
        to_f64_planes<T><<<grid_for(n * points, 256), 256, 0, dev.stream>>>(src + off, dst + off, n, ld, points);
    }
    return !failed(cudaGetLastError(), "conversion");
}

// the runs of a device f64 arena (or staging) back to the host
bool download_runs(const double *dre, const double *dim, double *hre, double *him, const uint32_t *runs,
                   uint32_t count, size_t ld, size_t points) {
    for (uint32_t r = 0; r < count; r++) {
        size_t off = (size_t)runs[2 * r] * ld, n = runs[2 * r + 1];
        if (!copy_planes(hre + off, dre + off, n, ld, points, cudaMemcpyDeviceToHost) ||
            !copy_planes(him + off, dim + off, n, ld, points, cudaMemcpyDeviceToHost))
            return false;
    }
    return true;
}

bool upload_runs(double *dre, double *dim, const double *hre, const double *him, const uint32_t *runs,
                 uint32_t count, size_t ld, size_t points) {
    for (uint32_t r = 0; r < count; r++) {
        size_t off = (size_t)runs[2 * r] * ld, n = runs[2 * r + 1];
        if (!copy_planes(dre + off, hre + off, n, ld, points, cudaMemcpyHostToDevice) ||
            !copy_planes(dim + off, him + off, n, ld, points, cudaMemcpyHostToDevice))
            return false;
    }
    return true;
}

// ---- programs ----------------------------------------------------------------------------------

const DeviceProgram *prepare(const pacman_recurrence_call *c, int *status) {
    Limits lim{c->current_planes, c->amplitude_planes, c->momentum_planes / 4u, c->scale_count, c->factor_count};
    if (c->words_key) {
        auto it = dev.programs.find(c->words_key);
        if (it != dev.programs.end()) {
            // a cached program is reused by a call with other tables only if they hold it
            if (fits(it->second.host, lim)) return &it->second;
            fprintf(stderr, "%s: the program of this key names planes outside this call's tables\n", kTag);
            *status = PACMAN_RECURRENCE_INVALID;
            return nullptr;
        }
    }
    DeviceProgram p;
    BuildError e = build_program(c->words, c->word_count, c->width, current.sort, lim, p.host);
    if (e.status) {
        fprintf(stderr, "%s: %s\n", kTag, e.message.c_str());
        *status = e.status;
        return nullptr;
    }
    size_t bytes = std::max<size_t>(1, p.host.ins.size()) * sizeof(Ins);
    if (failed(cudaMalloc((void **)&p.ins, bytes), "program") ||
        failed(cudaMemcpyAsync(p.ins, p.host.ins.data(), p.host.ins.size() * sizeof(Ins), cudaMemcpyHostToDevice,
                               dev.stream), "program")) {
        *status = PACMAN_RECURRENCE_DEVICE_ERROR;
        return nullptr;
    }
    if (c->words_key) {
        // a cached program is only valid for the tables it was checked against: a later call
        // with the same key and smaller tables is checked again
        return &(dev.programs[c->words_key] = std::move(p));
    }
    if (dev.scratch.ins) {
        cudaStreamSynchronize(dev.stream);
        cudaFree(dev.scratch.ins);
    }
    dev.scratch = std::move(p);
    return &dev.scratch;
}

template <class K>
bool launch_plan(const DeviceProgram &p, const RunArgs &a, unsigned block) {
    unsigned grid = (unsigned)((a.points + block - 1) / block);
    run_plan<K><<<grid, block, 0, dev.stream>>>(p.ins, (uint32_t)p.host.ins.size(), p.host.sources, a);
    return !failed(cudaGetLastError(), "launch");
}

// ---- the on-chip executor in the C ABI's mode ------------------------------------------------

// 1 launched, 0 not applicable (the global-arena executor runs), 2 refused, -1 device error
int onchip_launch(DeviceProgram *prog, const pacman_recurrence_call *c, const RunArgs &a, bool forms_on_device,
                  int kernel) {
    if (current.executor == PACUDA_B200_EXECUTOR_ARENA) return 0;
    uint32_t forms = c->momentum_planes / 4;
    if (prog->tiled_state == 0) {
        prog->tiled_state = -1;
        if (build_schedule(prog->host, c->current_planes, c->amplitude_planes, prog->tiled.host) &&
            upload_schedule(prog->tiled, tiled_threads(kernel), dev.stream))
            prog->tiled_state = 1;
    }
    // the lanes per point: as configured, else the default points per block; one block per SM (the
    // arena write-back of a block's interleaved points is coalesced over them: several blocks of
    // fewer points measured 19 % slower for gg>ggg through this path)
    int threads = prog->tiled_state == 1 ? tiled_threads(kernel) : 0;
    size_t pb = prog->tiled_state == 1 ? tiled_point_bytes(prog->tiled.host, forms, kernel) : 0;
    size_t cb = tiled_const_bytes(c->scale_count, c->factor_count);
    size_t room = threads ? tiled_max_smem(kernel) - cb : 0;
    uint32_t np = threads && prog->tiled.threads == threads ? tiled_default_points(pb, threads, room) : 0;
    if (np && current.lanes_per_point) {
        uint32_t want = 0;  // the most points per block whose lanes are at least the configured count
        for (uint32_t n = 1; n <= kMaxPoints; n++)
            if (tiled_lanes(n, threads) >= current.lanes_per_point) want = n;
        np = tiled_points_fit(want, pb, threads, room) ? want : 0;
    }
    if (!np) return current.executor == PACUDA_B200_EXECUTOR_ONCHIP ? 2 : 0;
    size_t smem = cb + (size_t)np * pb;
    // descriptors: TiledPlan | item_first[2] | external[1] | count[1] | counter
    const size_t o_items = (sizeof(TiledPlan) + 15) / 16 * 16, o_ext = o_items + 16, o_count = o_ext + 8,
                 o_counter = (o_count + 4 + 15) / 16 * 16, total = o_counter + 16;
    if (!dev.launch_host && failed(cudaMallocHost((void **)&dev.launch_host, total), "descriptors")) return -1;
    if (!dev.launch_dev.reserve(total, "descriptors")) return -1;
    memset(dev.launch_host, 0, total);
    TiledPlan &p = *(TiledPlan *)dev.launch_host;
    describe(prog->tiled, forms, np, pb, p);
    p.s64 = a.s64;
    p.f64 = a.f64;
    p.kconst = a.kconst;
    p.scales = a.scales;
    p.factors = a.factors;
    p.form_terms = a.form_terms;
    p.term_slots = a.term_slots;
    p.coefficients = a.coefficients;
    unsigned long long *items = (unsigned long long *)(dev.launch_host + o_items);
    items[0] = 0;
    uint32_t per = np;
    items[1] = (a.points + per - 1) / per;
    *(const double **)(dev.launch_host + o_ext) = a.external;
    *(uint32_t *)(dev.launch_host + o_count) = a.points;
    if (failed(cudaMemcpyAsync(dev.launch_dev.p, dev.launch_host, total, cudaMemcpyHostToDevice, dev.stream),
               "descriptors"))
        return -1;
    unsigned char *d = dev.launch_dev.as<unsigned char>();
    TiledLaunch L;
    memset(&L, 0, sizeof L);
    L.plans = (const TiledPlan *)d;
    L.nplans = 1;
    L.item_first = (const unsigned long long *)(d + o_items);
    L.external = (const double *const *)(d + o_ext);
    L.count = (const uint32_t *)(d + o_count);
    L.counter = (unsigned long long *)(d + o_counter);
    L.abi = true;
    L.cre = a.cre;
    L.cim = a.cim;
    L.are = a.are;
    L.aim = a.aim;
    L.mom = forms_on_device ? nullptr : a.mom;
    L.ld = a.ld;
    L.const_bytes = (uint32_t)cb;
    if (!launch_tiled(kernel, L, threads, smem, dev.sms, dev.stream) || failed(cudaGetLastError(), "launch")) return -1;
    // the host descriptors are read by the copy: wait for it before a later call rewrites them
    return failed(cudaStreamSynchronize(dev.stream), "descriptors") ? -1 : 1;
}

// ---- the run ---------------------------------------------------------------------------------

int run_locked(const pacman_recurrence_call *in) {
    runs_started = true;
    if (!initialize()) return PACMAN_RECURRENCE_DEVICE_ERROR;
    const size_t v1 = offsetof(pacman_recurrence_call, zero_amplitude);
    const size_t v2 = offsetof(pacman_recurrence_call, external_momenta);
    if (!in || in->abi_version != PACMAN_RECURRENCE_ABI ||
        (in->struct_size != sizeof(pacman_recurrence_call) && in->struct_size != v1 && in->struct_size != v2))
        return PACMAN_RECURRENCE_INVALID;
    pacman_recurrence_call full;
    memset(&full, 0, sizeof full);
    memcpy(&full, in, in->struct_size);
    const pacman_recurrence_call *c = &full;
    if (c->points == 0 || c->points > c->stride || !c->words || (c->zero_amplitude_runs && !c->zero_amplitude))
        return PACMAN_RECURRENCE_INVALID;
    if ((c->scale_count && (!c->scale_re || !c->scale_im)) || (c->factor_count && (!c->factor_re || !c->factor_im)) ||
        (c->upload_current_runs && (!c->upload_current || !c->current_re || !c->current_im)) ||
        (c->download_current_runs && (!c->download_current || !c->current_re || !c->current_im)) ||
        (c->upload_amplitude_runs && (!c->upload_amplitude || !c->amplitude_re || !c->amplitude_im)) ||
        (c->download_amplitude_runs && (!c->download_amplitude || !c->amplitude_re || !c->amplitude_im)))
        return PACMAN_RECURRENCE_INVALID;
    dev.kept = false;
    const int kernel = current.kernel;
    const bool keep = c->flags & PACMAN_RECURRENCE_KEEP_AMPLITUDES;
    const bool forms_on_device = c->flags & PACMAN_RECURRENCE_FORMS_ON_DEVICE;
    double start = dev.stats ? now() : 0;
    const size_t ld = c->stride, points = c->points;
    const uint32_t form_count = c->momentum_planes / 4;
    if (forms_on_device) {
        if (!c->external_momenta || !c->form_terms || (c->term_count && (!c->term_slots || !c->term_coefficients)))
            return PACMAN_RECURRENCE_INVALID;
        for (uint32_t f = 0; f < form_count; f++)
            if (c->form_terms[2 * f] > c->term_count || c->form_terms[2 * f + 1] > c->term_count - c->form_terms[2 * f])
                return PACMAN_RECURRENCE_INVALID;
        for (uint32_t t = 0; t < c->term_count; t++)
            if (c->term_slots[t] >= c->external_count) return PACMAN_RECURRENCE_INVALID;
    } else if (c->momentum_planes && !c->momenta) {
        return PACMAN_RECURRENCE_INVALID;
    }
    for (uint32_t r = 0; r < c->zero_amplitude_runs; r++) {
        uint32_t first = c->zero_amplitude[2 * r], n = c->zero_amplitude[2 * r + 1];
        if (first > c->amplitude_planes || n > c->amplitude_planes - first) return PACMAN_RECURRENCE_INVALID;
    }
    if (!runs_valid(c->upload_current, c->upload_current_runs, c->current_planes) ||
        !runs_valid(c->download_current, c->download_current_runs, c->current_planes) ||
        !runs_valid(c->upload_amplitude, c->upload_amplitude_runs, c->amplitude_planes) ||
        !runs_valid(c->download_amplitude, c->download_amplitude_runs, c->amplitude_planes))
        return PACMAN_RECURRENCE_DEVICE_ERROR;

    // the arenas (a grown arena loses its contents: the caller uploads what the words read)
    size_t cur_n = (size_t)c->current_planes * ld, amp_n = (size_t)c->amplitude_planes * ld;
    bool mixed = kernel == KERNEL_MIXED || kernel == KERNEL_MIXED64;
    if (!dev.cre.reserve(cur_n * 8, "current arena") || !dev.cim.reserve(cur_n * 8, "current arena") ||
        !dev.are.reserve(amp_n * 8, "amplitudes") || !dev.aim.reserve(amp_n * 8, "amplitudes") ||
        (mixed && (!dev.fcre.reserve(cur_n * 4, "current arena (f32)") ||
                   !dev.fcim.reserve(cur_n * 4, "current arena (f32)"))) ||
        !dev.mom.reserve((size_t)c->momentum_planes * ld * 8, "momenta") ||
        !dev.stage.reserve(std::max(cur_n, amp_n) * 8 * 2, "staging"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;

    // constants: f64 (sources) and the kind's layout (df64 pairs for every kernel but f64)
    size_t nconst = 2 * ((size_t)c->scale_count + c->factor_count);
    std::vector<double> consts(2 * nconst + 2);
    double *c64 = consts.data();
    for (uint32_t k = 0; k < c->scale_count; k++) { c64[k] = c->scale_re[k]; c64[c->scale_count + k] = c->scale_im[k]; }
    double *f64p = c64 + 2 * c->scale_count;
    for (uint32_t k = 0; k < c->factor_count; k++) { f64p[k] = c->factor_re[k]; f64p[c->factor_count + k] = c->factor_im[k]; }
    double *kc = c64 + nconst;
    for (size_t k = 0; k < nconst; k++) {
        if (kernel == KERNEL_F64) {
            kc[k] = c64[k];
        } else {
            float hi = (float)c64[k];
            float lo = (float)(c64[k] - (double)hi);
            memcpy(&kc[k], &hi, 4);
            memcpy((char *)&kc[k] + 4, &lo, 4);
        }
    }
    if (!dev.consts.reserve(consts.size() * 8, "constants") ||
        failed(cudaMemcpyAsync(dev.consts.p, consts.data(), consts.size() * 8, cudaMemcpyHostToDevice, dev.stream),
               "constants"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;

    // momentum forms: uploaded planes, or the external momenta and the term table
    if (forms_on_device) {
        size_t ext_n = (size_t)c->external_count * 4 * points;
        size_t tbytes = (2 * (size_t)form_count + c->term_count) * 4 + (size_t)c->term_count * 8 + 16;
        if (!dev.external.reserve(ext_n * 8, "external momenta") || !dev.terms.reserve(tbytes, "form terms"))
            return PACMAN_RECURRENCE_DEVICE_ERROR;
        std::vector<char> t(tbytes, 0);
        memcpy(t.data(), c->term_coefficients, (size_t)c->term_count * 8);
        memcpy(t.data() + (size_t)c->term_count * 8, c->form_terms, 2 * (size_t)form_count * 4);
        memcpy(t.data() + (size_t)c->term_count * 8 + 2 * (size_t)form_count * 4, c->term_slots, (size_t)c->term_count * 4);
        if (failed(cudaMemcpyAsync(dev.external.p, c->external_momenta, ext_n * 8, cudaMemcpyHostToDevice, dev.stream),
                   "external momenta") ||
            failed(cudaMemcpyAsync(dev.terms.p, t.data(), tbytes, cudaMemcpyHostToDevice, dev.stream), "form terms"))
            return PACMAN_RECURRENCE_DEVICE_ERROR;
        dev.copies++;
        dev.bytes += ext_n * 8;
    } else if (c->momentum_planes &&
               !copy_planes(dev.mom.p, c->momenta, c->momentum_planes, ld, points, cudaMemcpyHostToDevice)) {
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    }

    // uploads (f64) and their conversion into the kind's layout; zeroed amplitude runs
    if (!upload_runs(dev.cre.as<double>(), dev.cim.as<double>(), c->current_re, c->current_im, c->upload_current,
                     c->upload_current_runs, ld, points) ||
        !upload_runs(dev.are.as<double>(), dev.aim.as<double>(), c->amplitude_re, c->amplitude_im,
                     c->upload_amplitude, c->upload_amplitude_runs, ld, points))
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    for (uint32_t r = 0; r < c->zero_amplitude_runs; r++) {
        size_t off = (size_t)c->zero_amplitude[2 * r] * ld, n = c->zero_amplitude[2 * r + 1];
        if (n && (failed(cudaMemset2DAsync(dev.are.as<double>() + off, ld * 8, 0, points * 8, n, dev.stream), "zero") ||
                  failed(cudaMemset2DAsync(dev.aim.as<double>() + off, ld * 8, 0, points * 8, n, dev.stream), "zero")))
            return PACMAN_RECURRENCE_DEVICE_ERROR;
    }
    int status = PACMAN_RECURRENCE_DEVICE_ERROR;
    const DeviceProgram *prog = prepare(c, &status);
    if (!prog) return status;
    if (kernel != KERNEL_F64) {
        bool ok = true;
        if (kernel == KERNEL_DF64) {
            ok = convert_in<D>(dev.cre.as<double>(), dev.cre.as<D>(), c->upload_current, c->upload_current_runs, ld, points) &&
                 convert_in<D>(dev.cim.as<double>(), dev.cim.as<D>(), c->upload_current, c->upload_current_runs, ld, points);
        } else {
            ok = convert_in<float>(dev.cre.as<double>(), dev.fcre.as<float>(), c->upload_current, c->upload_current_runs, ld, points) &&
                 convert_in<float>(dev.cim.as<double>(), dev.fcim.as<float>(), c->upload_current, c->upload_current_runs, ld, points);
        }
        ok = ok && convert_in<D>(dev.are.as<double>(), dev.are.as<D>(), c->upload_amplitude, c->upload_amplitude_runs, ld, points) &&
             convert_in<D>(dev.aim.as<double>(), dev.aim.as<D>(), c->upload_amplitude, c->upload_amplitude_runs, ld, points);
        if (!ok) return PACMAN_RECURRENCE_DEVICE_ERROR;
    }

    RunArgs a{};
    a.cre = mixed ? dev.fcre.p : dev.cre.p;
    a.cim = mixed ? dev.fcim.p : dev.cim.p;
    a.are = dev.are.p;
    a.aim = dev.aim.p;
    a.mom = dev.mom.as<double>();
    a.ld = ld;
    a.points = (uint32_t)points;
    a.s64 = dev.consts.as<double>();
    a.f64 = a.s64 + 2 * c->scale_count;
    a.kconst = a.s64 + nconst;
    a.scales = c->scale_count;
    a.factors = c->factor_count;
    a.forms = form_count;
    a.den_is_f64 = kernel == KERNEL_F64 || kernel == KERNEL_MIXED64;
    if (forms_on_device) {
        a.external = dev.external.as<double>();
        a.coefficients = dev.terms.as<double>();
        a.form_terms = (const uint32_t *)(a.coefficients + c->term_count);
        a.term_slots = a.form_terms + 2 * form_count;
    }
    unsigned block = current.block ? (unsigned)current.block : 128u;
    bool launched = false;
    int onchip = onchip_launch(const_cast<DeviceProgram *>(prog), c, a, forms_on_device, kernel);
    if (onchip < 0) return PACMAN_RECURRENCE_DEVICE_ERROR;
    if (onchip == 2) return PACMAN_RECURRENCE_INVALID;
    if (onchip == 1) launched = true;
    else switch (kernel) {
    case KERNEL_F64: launched = launch_plan<KindF64>(*prog, a, block); break;
    case KERNEL_MIXED: launched = launch_plan<KindMixed>(*prog, a, block); break;
    case KERNEL_MIXED64: launched = launch_plan<KindMixed64>(*prog, a, block); break;
    default: launched = launch_plan<KindDF64>(*prog, a, block); break;
    }
    if (!launched) return PACMAN_RECURRENCE_DEVICE_ERROR;

    // downloads: amplitudes (unless kept) and currents, as f64
    uint32_t amp_runs = keep ? 0 : c->download_amplitude_runs;
    double *sre = dev.stage.as<double>(), *sim = sre + std::max(cur_n, amp_n);
    if (amp_runs) {
        const double *srcre = dev.are.as<double>(), *srcim = dev.aim.as<double>();
        if (kernel != KERNEL_F64) {
            if (!convert_out<D>(dev.are.as<D>(), sre, c->download_amplitude, amp_runs, ld, points) ||
                !convert_out<D>(dev.aim.as<D>(), sim, c->download_amplitude, amp_runs, ld, points))
                return PACMAN_RECURRENCE_DEVICE_ERROR;
            srcre = sre;
            srcim = sim;
        }
        if (!download_runs(srcre, srcim, c->amplitude_re, c->amplitude_im, c->download_amplitude, amp_runs, ld, points))
            return PACMAN_RECURRENCE_DEVICE_ERROR;
    }
    if (c->download_current_runs) {
        if (amp_runs && failed(cudaStreamSynchronize(dev.stream), "kernel")) return PACMAN_RECURRENCE_DEVICE_ERROR;
        const double *srcre = dev.cre.as<double>(), *srcim = dev.cim.as<double>();
        bool ok = true;
        if (kernel == KERNEL_DF64) {
            ok = convert_out<D>(dev.cre.as<D>(), sre, c->download_current, c->download_current_runs, ld, points) &&
                 convert_out<D>(dev.cim.as<D>(), sim, c->download_current, c->download_current_runs, ld, points);
            srcre = sre;
            srcim = sim;
        } else if (mixed) {
            ok = convert_out<float>(dev.fcre.as<float>(), sre, c->download_current, c->download_current_runs, ld, points) &&
                 convert_out<float>(dev.fcim.as<float>(), sim, c->download_current, c->download_current_runs, ld, points);
            srcre = sre;
            srcim = sim;
        }
        if (!ok || !download_runs(srcre, srcim, c->current_re, c->current_im, c->download_current,
                                  c->download_current_runs, ld, points))
            return PACMAN_RECURRENCE_DEVICE_ERROR;
    }
    if (failed(cudaStreamSynchronize(dev.stream), "kernel")) return PACMAN_RECURRENCE_DEVICE_ERROR;
    if (keep) {
        dev.kept = true;
        dev.kept_kernel = kernel;
        dev.kept_stride = ld;
        dev.kept_points = points;
        dev.kept_planes = c->amplitude_planes;
    }
    dev.calls++;
    dev.points += points;
    if (dev.stats) dev.seconds += now() - start;
    return PACMAN_RECURRENCE_OK;
}

// ---- reductions --------------------------------------------------------------------------------

bool upload_table(Buffer &b, const void *src, size_t bytes, const char *what) {
    if (!b.reserve(std::max<size_t>(bytes, 16), what)) return false;
    return bytes == 0 || !failed(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, dev.stream), what);
}

bool check_reduction_tables(const uint32_t *offsets, uint32_t outputs, const uint32_t *planes, const double *weights,
                            uint32_t *count) {
    *count = offsets[outputs];
    if (offsets[0] != 0 || (*count && (!planes || !weights))) return false;
    for (uint32_t o = 0; o < outputs; o++)
        if (offsets[o] > offsets[o + 1]) return false;
    for (uint32_t k = 0; k < *count; k++)
        if (planes[k] >= dev.kept_planes) return false;
    return true;
}

int reduce_resolved_locked(const pacman_recurrence_reduce_resolved *r) {
    if (!initialize()) return PACMAN_RECURRENCE_DEVICE_ERROR;
    if (!r || r->abi_version != PACMAN_RECURRENCE_ABI || r->struct_size != sizeof(pacman_recurrence_reduce_resolved) ||
        !r->offsets || !r->output || r->outputs == 0 || r->outputs > 65535)
        return PACMAN_RECURRENCE_INVALID;
    if (!dev.kept || r->points != dev.kept_points) return PACMAN_RECURRENCE_INVALID;
    uint32_t count = 0;
    if (!check_reduction_tables(r->offsets, r->outputs, r->planes, r->weights, &count)) return PACMAN_RECURRENCE_INVALID;
    if (r->points == 0) return PACMAN_RECURRENCE_OK;
    double start = dev.stats ? now() : 0;
    size_t span = (size_t)(r->outputs - 1) * r->output_stride + (size_t)(r->points - 1) * r->point_stride + 1;
    bool zero = r->flags & PACMAN_RECURRENCE_OUTPUT_ZERO;
    if (!upload_table(dev.rplanes, r->planes, count * 4, "reduction") ||
        !upload_table(dev.rweights, r->weights, count * 8, "reduction") ||
        !upload_table(dev.roffsets, r->offsets, (r->outputs + 1) * 4, "reduction") ||
        !dev.routput.reserve(span * 8, "reduction"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    if (!zero && failed(cudaMemcpyAsync(dev.routput.p, r->output, span * 8, cudaMemcpyHostToDevice, dev.stream), "reduction"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    unsigned block = 128, grid = (r->points + block - 1) / block;
    if (dev.kept_kernel == KERNEL_F64)
        reduce_resolved_kernel<double><<<grid, block, 0, dev.stream>>>(
            dev.are.as<double>(), dev.aim.as<double>(), dev.kept_stride, dev.rplanes.as<uint32_t>(),
            dev.rweights.as<double>(), dev.roffsets.as<uint32_t>(), r->outputs, dev.routput.as<double>(), r->points,
            r->output_stride, r->point_stride, zero);
    else
        reduce_resolved_kernel<D><<<grid, block, 0, dev.stream>>>(
            dev.are.as<D>(), dev.aim.as<D>(), dev.kept_stride, dev.rplanes.as<uint32_t>(), dev.rweights.as<double>(),
            dev.roffsets.as<uint32_t>(), r->outputs, dev.routput.as<double>(), r->points, r->output_stride,
            r->point_stride, zero);
    if (failed(cudaGetLastError(), "reduction") ||
        failed(cudaMemcpyAsync(r->output, dev.routput.p, span * 8, cudaMemcpyDeviceToHost, dev.stream), "reduction") ||
        failed(cudaStreamSynchronize(dev.stream), "reduction"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    dev.copies += zero ? 1 : 2;
    dev.bytes += (zero ? 1 : 2) * span * 8;
    dev.reductions++;
    if (dev.stats) dev.seconds += now() - start;
    return PACMAN_RECURRENCE_OK;
}

int reduce_sample_locked(const pacman_recurrence_reduce_sample *r) {
    if (!initialize()) return PACMAN_RECURRENCE_DEVICE_ERROR;
    if (!r || r->abi_version != PACMAN_RECURRENCE_ABI || r->struct_size != sizeof(pacman_recurrence_reduce_sample) ||
        !r->offsets || !r->helicity || !r->random || !r->total || !r->chosen || r->outputs == 0)
        return PACMAN_RECURRENCE_INVALID;
    if (!dev.kept || r->points != dev.kept_points) return PACMAN_RECURRENCE_INVALID;
    uint32_t count = 0;
    if (!check_reduction_tables(r->offsets, r->outputs, r->planes, r->weights, &count)) return PACMAN_RECURRENCE_INVALID;
    if (r->points == 0) return PACMAN_RECURRENCE_OK;
    double start = dev.stats ? now() : 0;
    size_t n = r->points;
    if (!upload_table(dev.rplanes, r->planes, count * 4, "sampling") ||
        !upload_table(dev.rweights, r->weights, count * 8, "sampling") ||
        !upload_table(dev.roffsets, r->offsets, (r->outputs + 1) * 4, "sampling") ||
        !upload_table(dev.rhelicity, r->helicity, r->outputs * 4, "sampling") ||
        !upload_table(dev.rrandom, r->random, n * 8, "sampling") ||
        (r->scale && !upload_table(dev.rscale, r->scale, n * 8, "sampling")) ||
        !dev.rtotal.reserve(n * 8, "sampling") || !dev.rchosen.reserve(n * 4, "sampling"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    bool factor = r->numerator != r->denominator;
    unsigned block = 128, grid = (unsigned)((n + block - 1) / block);
    const double *scale = r->scale ? dev.rscale.as<double>() : nullptr;
    if (dev.kept_kernel == KERNEL_F64)
        reduce_sample_kernel<double><<<grid, block, 0, dev.stream>>>(
            dev.are.as<double>(), dev.aim.as<double>(), dev.kept_stride, dev.rplanes.as<uint32_t>(),
            dev.rweights.as<double>(), dev.roffsets.as<uint32_t>(), dev.rhelicity.as<uint32_t>(), r->outputs, r->points,
            dev.rrandom.as<double>(), scale, factor, r->numerator, r->denominator, dev.rtotal.as<double>(),
            dev.rchosen.as<uint32_t>());
    else
        reduce_sample_kernel<D><<<grid, block, 0, dev.stream>>>(
            dev.are.as<D>(), dev.aim.as<D>(), dev.kept_stride, dev.rplanes.as<uint32_t>(), dev.rweights.as<double>(),
            dev.roffsets.as<uint32_t>(), dev.rhelicity.as<uint32_t>(), r->outputs, r->points, dev.rrandom.as<double>(),
            scale, factor, r->numerator, r->denominator, dev.rtotal.as<double>(), dev.rchosen.as<uint32_t>());
    if (failed(cudaGetLastError(), "sampling") ||
        failed(cudaMemcpyAsync(r->total, dev.rtotal.p, n * 8, cudaMemcpyDeviceToHost, dev.stream), "sampling") ||
        failed(cudaMemcpyAsync(r->chosen, dev.rchosen.p, n * 4, cudaMemcpyDeviceToHost, dev.stream), "sampling") ||
        failed(cudaStreamSynchronize(dev.stream), "sampling"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    dev.copies += r->scale ? 4 : 3;
    dev.bytes += n * (8 * (r->scale ? 3 : 2) + 4);
    dev.reductions++;
    if (dev.stats) dev.seconds += now() - start;
    return PACMAN_RECURRENCE_OK;
}

int reduce_locked(const pacman_recurrence_reduce *r) {
    if (!initialize()) return PACMAN_RECURRENCE_DEVICE_ERROR;
    if (!r || r->abi_version != PACMAN_RECURRENCE_ABI || r->struct_size != sizeof(pacman_recurrence_reduce) ||
        (r->count && (!r->planes || !r->weights)) || !r->output)
        return PACMAN_RECURRENCE_INVALID;
    if (!dev.kept || r->points != dev.kept_points) return PACMAN_RECURRENCE_INVALID;
    for (uint32_t k = 0; k < r->count; k++)
        if (r->planes[k] >= dev.kept_planes) return PACMAN_RECURRENCE_INVALID;
    if (r->points == 0) return PACMAN_RECURRENCE_OK;
    double start = dev.stats ? now() : 0;
    size_t bytes = (size_t)r->points * 8;
    if (!upload_table(dev.rplanes, r->planes, r->count * 4, "reduction") ||
        !upload_table(dev.rweights, r->weights, r->count * 8, "reduction") ||
        !upload_table(dev.routput, r->output, bytes, "reduction"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    unsigned block = 128, grid = (r->points + block - 1) / block;
    if (dev.kept_kernel == KERNEL_F64)
        reduce_kernel<double><<<grid, block, 0, dev.stream>>>(dev.are.as<double>(), dev.aim.as<double>(), dev.kept_stride,
                                                              dev.rplanes.as<uint32_t>(), dev.rweights.as<double>(),
                                                              r->count, dev.routput.as<double>(), r->points);
    else
        reduce_kernel<D><<<grid, block, 0, dev.stream>>>(dev.are.as<D>(), dev.aim.as<D>(), dev.kept_stride,
                                                         dev.rplanes.as<uint32_t>(), dev.rweights.as<double>(), r->count,
                                                         dev.routput.as<double>(), r->points);
    if (failed(cudaGetLastError(), "reduction") ||
        failed(cudaMemcpyAsync(r->output, dev.routput.p, bytes, cudaMemcpyDeviceToHost, dev.stream), "reduction") ||
        failed(cudaStreamSynchronize(dev.stream), "reduction"))
        return PACMAN_RECURRENCE_DEVICE_ERROR;
    dev.copies += 2;
    dev.bytes += 2 * bytes;
    dev.reductions++;
    if (dev.stats) dev.seconds += now() - start;
    return PACMAN_RECURRENCE_OK;
}

// ---- the lock (reference: recurrence_runner.cu:1725-1748) ------------------------------------
std::mutex runner_lock;
thread_local bool holding_lock = false;

void acquire() {
    if (!holding_lock) {
        runner_lock.lock();
        holding_lock = true;
    }
}
void release() {
    if (holding_lock) {
        holding_lock = false;
        runner_lock.unlock();
    }
}

}  // namespace

extern "C" int pacman_recurrence_v1_run(const pacman_recurrence_call *call) {
    acquire();
    int status = run_locked(call);
    if (!(status == PACMAN_RECURRENCE_OK && dev.kept)) release();
    return status;
}

extern "C" int pacman_recurrence_v1_reduce_resolved(const pacman_recurrence_reduce_resolved *r) {
    acquire();
    int status = reduce_resolved_locked(r);
    release();
    return status;
}

extern "C" int pacman_recurrence_v1_reduce_sample(const pacman_recurrence_reduce_sample *r) {
    acquire();
    int status = reduce_sample_locked(r);
    release();
    return status;
}

extern "C" int pacman_recurrence_v1_reduce(const pacman_recurrence_reduce *r) {
    acquire();
    int status = reduce_locked(r);
    release();
    return status;
}

extern "C" int pacman_recurrence_v1_configure(const pacman_recurrence_options *o) {
    if (!o || o->abi_version != PACMAN_RECURRENCE_ABI || o->struct_size < sizeof(pacman_recurrence_options))
        return PACMAN_RECURRENCE_INVALID;
    if (o->kernel > PACMAN_RECURRENCE_KERNEL_MIXED64 || (o->block && (o->block < 32 || o->block > 1024)))
        return PACMAN_RECURRENCE_INVALID;
    acquire();
    int status = PACMAN_RECURRENCE_OK;
    Options n;
    n.kernel = (int)o->kernel;
    n.block = (int)o->block;
    n.sort = !o->no_sort;
    if (o->struct_size >= sizeof(pacuda_b200_options)) {
        const pacuda_b200_options *x = (const pacuda_b200_options *)o;
        if (x->executor > PACUDA_B200_EXECUTOR_ONCHIP || x->lanes_per_point > 512) {
            release();
            return PACMAN_RECURRENCE_INVALID;
        }
        n.executor = (int)x->executor;
        n.lanes_per_point = x->lanes_per_point;
    }
    bool same = n.kernel == current.kernel && n.block == current.block && n.sort == current.sort &&
                n.executor == current.executor && n.lanes_per_point == current.lanes_per_point;
    if (runs_started && !same) {
        fprintf(stderr, "%s: another configuration after the first run\n", kTag);
        status = PACMAN_RECURRENCE_INVALID;
    } else {
        current = n;
        dev.stats = dev.stats || o->stats != 0;
    }
    release();
    return status;
}

extern "C" uint32_t pacman_recurrence_v1_capabilities(void) {
    return PACMAN_RECURRENCE_CAP_SOURCES | PACMAN_RECURRENCE_CAP_FORMS;
}

extern "C" int pacman_recurrence_v1_symjit_kernel(const char *sha256_hex) {
    (void)sha256_hex;
    return -1;  // this runner is built without generated symjit kernels
}

extern "C" void *pacman_recurrence_v1_host_alloc(size_t bytes) {
    void *p = nullptr;
    if (cudaMallocHost(&p, bytes ? bytes : 1) != cudaSuccess) return nullptr;
    return p;
}

extern "C" void pacman_recurrence_v1_host_free(void *p) {
    if (p) cudaFreeHost(p);
}

extern "C" int pacman_recurrence_v1_test_sources(const uint32_t *codes, const double *masses, const double *momenta,
                                                 uint32_t count, double *out_re, double *out_im) {
    if (count == 0) return PACMAN_RECURRENCE_OK;
    if (!codes || !masses || !momenta || !out_re || !out_im) return PACMAN_RECURRENCE_INVALID;
    acquire();
    int status = PACMAN_RECURRENCE_OK;
    if (!initialize()) status = PACMAN_RECURRENCE_DEVICE_ERROR;
    uint32_t *dc = nullptr;
    double *dm = nullptr, *dp = nullptr, *dre = nullptr, *dim = nullptr;
    if (status == PACMAN_RECURRENCE_OK) {
        bool ok = !failed(cudaMalloc((void **)&dc, count * 4), "test") && !failed(cudaMalloc((void **)&dm, count * 8), "test") &&
                  !failed(cudaMalloc((void **)&dp, 32 * (size_t)count), "test") &&
                  !failed(cudaMalloc((void **)&dre, 32 * (size_t)count), "test") &&
                  !failed(cudaMalloc((void **)&dim, 32 * (size_t)count), "test") &&
                  !failed(cudaMemcpyAsync(dc, codes, count * 4, cudaMemcpyHostToDevice, dev.stream), "test") &&
                  !failed(cudaMemcpyAsync(dm, masses, count * 8, cudaMemcpyHostToDevice, dev.stream), "test") &&
                  !failed(cudaMemcpyAsync(dp, momenta, 32 * (size_t)count, cudaMemcpyHostToDevice, dev.stream), "test");
        if (ok) {
            test_sources_kernel<<<(count + 127) / 128, 128, 0, dev.stream>>>(dc, dm, dp, count, dre, dim);
            ok = !failed(cudaGetLastError(), "test") &&
                 !failed(cudaMemcpyAsync(out_re, dre, 32 * (size_t)count, cudaMemcpyDeviceToHost, dev.stream), "test") &&
                 !failed(cudaMemcpyAsync(out_im, dim, 32 * (size_t)count, cudaMemcpyDeviceToHost, dev.stream), "test") &&
                 !failed(cudaStreamSynchronize(dev.stream), "test");
        }
        if (!ok) status = PACMAN_RECURRENCE_DEVICE_ERROR;
    }
    cudaFree(dc); cudaFree(dm); cudaFree(dp); cudaFree(dre); cudaFree(dim);
    release();
    return status;
}
