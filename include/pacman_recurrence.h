/* pacuda-b200: the recurrence runner's C ABI, version 1.
 *
 * This header declares the boundary that pacuda's librecurrence.so exports, so that a caller
 * built against the reference (UMAMI's umami/umami_pacuda.c, the converter's
 * convert/src/replay.rs FFI mirror, RustiCol's pacman hook, runner/rectest.c) links or dlopens
 * this library unchanged. The struct layouts, enum values and entry-point signatures are the
 * reference's (runner/pacman_recurrence.h:11-150) field for field, because they are the binary
 * interface; the semantics each entry point keeps are stated beside it.
 *
 * Arenas are plane-major: plane p of an arena of stride S holds its points at [p * S + i].
 * A run list is an array of (first plane, plane count) pairs.
 */
#ifndef PACMAN_RECURRENCE_H
#define PACMAN_RECURRENCE_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define PACMAN_RECURRENCE_ABI 1

/* The field widths of a plan's 64-bit row words, indices into `width[8]`
 * (reference: runner/pacman_recurrence.h:13). P current plane, A amplitude plane, F momentum
 * form, X exact factor, S executor slot (scale), K small component count. */
enum { W_P, W_A, W_F, W_X, W_S, W_K, W_COUNT };

/* One plan run over `points` phase-space points (reference: runner/pacman_recurrence.h:18-51).
 * A caller may pass a struct that ends before `zero_amplitude` or before `external_momenta`
 * (struct_size says which); the missing fields read as 0. */
typedef struct {
    uint32_t abi_version;
    uint32_t struct_size;
    const uint64_t *words;
    uint64_t words_key;            /* nonzero: the words never change under this key (cached) */
    uint32_t word_count;
    uint8_t width[8];              /* W_P .. W_K */
    double *current_re, *current_im;
    double *amplitude_re, *amplitude_im;
    const double *momenta;         /* momentum_planes planes, four per form */
    const double *scale_re, *scale_im;
    const double *factor_re, *factor_im;
    const uint32_t *upload_current, *upload_amplitude, *download_amplitude, *download_current;
    uint32_t current_planes, amplitude_planes, momentum_planes, scale_count, factor_count;
    uint32_t upload_current_runs, upload_amplitude_runs, download_amplitude_runs,
        download_current_runs;
    uint32_t stride, points;
    /* second revision */
    const uint32_t *zero_amplitude;  /* amplitude runs zeroed on the device, not uploaded */
    uint32_t zero_amplitude_runs;
    uint32_t flags;                  /* PACMAN_RECURRENCE_KEEP_AMPLITUDES | _FORMS_ON_DEVICE */
    /* third revision: with PACMAN_RECURRENCE_FORMS_ON_DEVICE the forms are built on the device,
     * form f component k = 0.0 + c_0 p(s_0, k) + c_1 p(s_1, k) + ... over the form's terms
     * form_terms[2f] .. form_terms[2f] + form_terms[2f+1] of (term_slots, term_coefficients),
     * with p(s, k) = external_momenta[(s * 4 + k) * points + i] */
    const double *external_momenta;
    uint32_t external_count;
    uint32_t term_count;
    const uint32_t *form_terms;
    const uint32_t *term_slots;
    const double *term_coefficients;
} pacman_recurrence_call;

#define PACMAN_RECURRENCE_KEEP_AMPLITUDES 1u
#define PACMAN_RECURRENCE_FORMS_ON_DEVICE 2u

/* The LC diagonal reduction of a kept run (reference: runner/pacman_recurrence.h:58-69):
 * output[i] += weights[k] * fma(re, re, im * im) for k = 0 .. count-1 in order, (re, im) the
 * kept amplitude plane planes[k] at point i. */
typedef struct {
    uint32_t abi_version;
    uint32_t struct_size;
    const uint32_t *planes;
    const double *weights;
    double *output;
    uint32_t count, points;
} pacman_recurrence_reduce;

enum {
    PACMAN_RECURRENCE_OK = 0,
    PACMAN_RECURRENCE_INVALID = 2,
    PACMAN_RECURRENCE_DEVICE_ERROR = 3,
};

/* The resolved reduction of a kept run, one output per helicity (reference:
 * runner/pacman_recurrence.h:77-95): output[o * output_stride + i * point_stride] +=
 * weights[k] * fma(re, re, im * im) for k = offsets[o] .. offsets[o+1]-1 in order. With
 * PACMAN_RECURRENCE_OUTPUT_ZERO the output starts from zero and is not read. */
typedef struct {
    uint32_t abi_version;
    uint32_t struct_size;
    const uint32_t *planes;
    const double *weights;
    const uint32_t *offsets;  /* outputs + 1 entries */
    double *output;
    uint32_t outputs, points, output_stride, point_stride;
    uint32_t flags;
} pacman_recurrence_reduce_resolved;
#define PACMAN_RECURRENCE_OUTPUT_ZERO 1u

/* Helicity sampling of a kept run (reference: runner/pacman_recurrence.h:97-118): per point
 * the outputs' values v (each from zero, times numerator/denominator when they differ, times
 * scale[i] when given and not 1), total = 0 + v[0] + v[1] + ..., and `chosen` the helicity of
 * the output where the running sum of the positive v first exceeds random[i] * total. */
typedef struct {
    uint32_t abi_version;
    uint32_t struct_size;
    const uint32_t *planes;
    const double *weights;
    const uint32_t *offsets;   /* outputs + 1 entries */
    const uint32_t *helicity;  /* per output, the helicity `chosen` reports */
    uint32_t outputs, points;
    const double *random;      /* per point, in [0, 1) */
    const double *scale;       /* per point, or NULL */
    double numerator, denominator;
    double *total;             /* per point */
    uint32_t *chosen;          /* per point */
} pacman_recurrence_reduce_sample;

/* reference: runner/pacman_recurrence.h:120 */
int pacman_recurrence_v1_run(const pacman_recurrence_call *call);
/* reference: runner/pacman_recurrence.h:121 */
int pacman_recurrence_v1_reduce_resolved(const pacman_recurrence_reduce_resolved *reduce);
/* reference: runner/pacman_recurrence.h:122 */
int pacman_recurrence_v1_reduce_sample(const pacman_recurrence_reduce_sample *sample);
/* Pinned host memory, or NULL (reference: runner/pacman_recurrence.h:124-125) */
void *pacman_recurrence_v1_host_alloc(size_t bytes);
void pacman_recurrence_v1_host_free(void *p);
/* reference: runner/pacman_recurrence.h:126 */
int pacman_recurrence_v1_reduce(const pacman_recurrence_reduce *reduce);

#define PACMAN_RECURRENCE_CAP_SOURCES 1u
#define PACMAN_RECURRENCE_CAP_FORMS 2u

/* The runner's configuration, set before the first run (afterwards only the same one again)
 * (reference: runner/pacman_recurrence.h:131-145). A larger struct_size is accepted. */
typedef struct {
    uint32_t abi_version;
    uint32_t struct_size;
    uint32_t kernel;       /* PACMAN_RECURRENCE_KERNEL_* */
    uint32_t block;        /* threads per block, 32..1024 (0: the runner's choice) */
    uint32_t no_sort;      /* 1: keep the contribution rows in plan order */
    uint32_t stats;        /* 1: print statistics at exit */
} pacman_recurrence_options;
enum {
    PACMAN_RECURRENCE_KERNEL_DF64 = 0,
    PACMAN_RECURRENCE_KERNEL_F64 = 1,
    PACMAN_RECURRENCE_KERNEL_MIXED = 2,
    PACMAN_RECURRENCE_KERNEL_MIXED64 = 3,
};
int pacman_recurrence_v1_configure(const pacman_recurrence_options *options);

#define PACMAN_RECURRENCE_CAP_SYMJIT 4u
/* reference: runner/pacman_recurrence.h:148 */
uint32_t pacman_recurrence_v1_capabilities(void);
/* The index of the generated symjit kernel with this SHA-256, or -1 (this build has none)
 * (reference: runner/pacman_recurrence.h:150). */
int pacman_recurrence_v1_symjit_kernel(const char *sha256_hex);

/* Test entry point: the external wavefunctions of `count` (template code, mass, momentum)
 * items, four components each (reference: runner/recurrence_runner.cu:1811-1834). */
int pacman_recurrence_v1_test_sources(const uint32_t *codes, const double *masses,
                                      const double *momenta, uint32_t count, double *out_re,
                                      double *out_im);

#ifdef __cplusplus
}
#endif
#endif
