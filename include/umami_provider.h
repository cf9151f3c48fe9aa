/* The provider tables of one subprocess's UMAMI library: its particles, its processes (the
 * .pacuda file's processes, matched by key, with their model parameters), and per channel and
 * flavour the contributions whose values make an event's |M|^2.
 *
 * The reference compiles its library once per subprocess against the artifact's generated
 * provider header (umami/build.sh; umami/umami_pacuda.c:40-43, which reads the fields below). That
 * header is not part of the reference, so this is this library's form of the same tables: a
 * provider header defines `static const UmamiProvider umami_provider` and the macros
 * UMAMI_HAS_ALPHA_S and UMAMI_HAS_COLOR_FLOW, and the library is built with
 * -DUMAMI_PROVIDER_HEADER='"that header"' (pacuda_b200/umami/build.py). */
#ifndef PACUDA_B200_UMAMI_PROVIDER_H
#define PACUDA_B200_UMAMI_PROVIDER_H
#include <stdbool.h>
#include <stddef.h>

typedef struct {
    const char *name;
    double real, imaginary;  /* the artifact's default value */
    bool is_complex;
    bool is_mutable;         /* may be set (alpha_s to any value; others only to the file's) */
} UmamiParameter;

typedef struct {
    const char *key;  /* the .pacuda process key */
    size_t helicity_count;
    size_t parameter_count;
    const UmamiParameter *parameters;
} UmamiProcess;

/* One evaluation of an event: process `process_index`'s plan of colour `color_id`, its leg l fed
 * the event's input leg permutation[l], times `factor`. helicity_runtime[label] is the process's
 * helicity of an exported label (or -1), helicity_export[h] the label of its helicity h. */
typedef struct {
    size_t process_index;
    const char *color_id;
    const size_t *permutation;
    double factor;
    const int *helicity_runtime;
    const int *helicity_export;
    size_t color_index;
} UmamiContribution;

typedef struct {
    size_t contribution_count;
    const UmamiContribution *contributions;
} UmamiFlavour;

typedef struct {
    size_t flavour_count;
    const UmamiFlavour *flavours;
} UmamiChannel;

typedef struct {
    size_t particle_count, helicity_count, exported_helicity_count, color_count;
    const double *masses;
    size_t process_count;
    const UmamiProcess *processes;
    size_t channel_count;
    const UmamiChannel *channels;
} UmamiProvider;

#endif
