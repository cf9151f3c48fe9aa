/* The UMAMI matrix-element interface, as far as this library implements it.
 *
 * UMAMI is the interface through which an event generator (madspace, MadNIS) asks a subprocess's
 * library for |M|^2 of a batch of events. Its header belongs to the matrix-element artifact and is
 * not part of the reference; this restates only what the reference's library implements
 * (umami/umami_pacuda.c:401-752) and what its drivers pass (tests/compare_umami.py,
 * tests/drive_umami.py): the nine functions, and the key values 0 (momenta), 1 (alpha_s),
 * 2 (flavour index), 4 (helicity random number), 6 (helicity index), 8 (channel index) for inputs,
 * 0 (|M|^2), 2 (colour index), 3 (helicity index) for outputs, and 3 (the helicity count) for
 * metadata. Status 0 is success; the other values here are this library's. */
#ifndef PACUDA_B200_UMAMI_H
#define PACUDA_B200_UMAMI_H
#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void *UmamiHandle;

typedef enum {
    UMAMI_SUCCESS = 0,
    UMAMI_ERROR = 1,
    UMAMI_ERROR_UNSUPPORTED_INPUT = 2,
    UMAMI_ERROR_UNSUPPORTED_OUTPUT = 3,
    UMAMI_ERROR_UNSUPPORTED_META = 4,
    UMAMI_ERROR_MISSING_INPUT = 5,
} UmamiStatus;

typedef enum {
    UMAMI_META_DEVICE = 0,          /* UmamiDevice: where the inputs and outputs live */
    UMAMI_META_PARTICLE_COUNT = 1,  /* int */
    UMAMI_META_MASSES = 2,          /* double[particle count] */
    UMAMI_META_HELICITY_COUNT = 3,  /* int */
    UMAMI_META_COLOR_COUNT = 4,     /* int (artifacts with colour flows only) */
} UmamiMetaKey;

typedef enum { UMAMI_DEVICE_CPU = 0, UMAMI_DEVICE_CUDA = 1 } UmamiDevice;

/* Inputs are arrays indexed by event; the momenta: component k of particle `leg` of an event at
 * momenta[event + stride * (particle_count * k + leg)]. */
typedef enum {
    UMAMI_IN_MOMENTA = 0,          /* double */
    UMAMI_IN_ALPHA_S = 1,          /* double */
    UMAMI_IN_FLAVOR_INDEX = 2,     /* int */
    UMAMI_IN_RANDOM_HELICITY = 4,  /* double in [0, 1) */
    UMAMI_IN_HELICITY_INDEX = 6,   /* int: a fixed helicity */
    UMAMI_IN_CHANNEL_INDEX = 8,    /* unsigned int */
    UMAMI_INPUT_KEY_COUNT = 9      /* 3, 5 and 7 are keys this library does not take */
} UmamiInputKey;

typedef enum {
    UMAMI_OUT_MATRIX_ELEMENT = 0,  /* double */
    UMAMI_OUT_COLOR_INDEX = 2,     /* int */
    UMAMI_OUT_HELICITY_INDEX = 3,  /* int: the sampled helicity */
    UMAMI_OUTPUT_KEY_COUNT = 4     /* 1 is a key this library does not give */
} UmamiOutputKey;

UmamiStatus umami_get_meta(UmamiMetaKey key, void *result);
UmamiStatus umami_supported_inputs(bool const **supported, int *count);
UmamiStatus umami_required_inputs(bool const **required, int *count);
UmamiStatus umami_supported_outputs(bool const **supported, int *count);
/* param_card_path: the artifact's directory (absolute); the plans are read from <directory>.pacuda */
UmamiStatus umami_initialize(UmamiHandle *handle, char const *param_card_path);
UmamiStatus umami_free(UmamiHandle handle);
UmamiStatus umami_get_parameter(UmamiHandle handle, char const *name, double *real, double *imaginary);
UmamiStatus umami_set_parameter(UmamiHandle handle, char const *name, double real, double imaginary);
/* |M|^2 (and the colour and helicity indices) of events offset .. offset + count - 1 */
UmamiStatus umami_matrix_element(UmamiHandle handle, size_t count, size_t stride, size_t offset, size_t input_count,
                                 UmamiInputKey const *input_keys, void const *const *inputs, size_t output_count,
                                 UmamiOutputKey const *output_keys, void *const *outputs);

#ifdef __cplusplus
}
#endif
#endif
