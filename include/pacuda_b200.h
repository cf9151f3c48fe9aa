/* pacuda-b200: the batched, device-resident entry points of the recurrence runner.
 *
 * These have no counterpart in the reference (runner/pacman_recurrence.h): they are this
 * library's B200 interface for callers that keep their phase-space points on the GPU. A plan is
 * compiled once (its words and tables as a pacman_recurrence_call describes them, and its
 * resolved reduction); a batch evaluates several plans, each on its own points, in one
 * persistent kernel launch, and can be captured in a CUDA graph. Inputs and outputs are device
 * arrays: per plan the external momenta as source-major planes [(leg * 4 + k) * count + i], the
 * outputs as [point][output] (the resolved reduction from zero, OUTPUT_ZERO semantics).
 * Statuses are the PACMAN_RECURRENCE_* codes. */
#ifndef PACUDA_B200_H
#define PACUDA_B200_H
#include <stddef.h>
#include <stdint.h>

#include "pacman_recurrence.h"
#ifdef __cplusplus
extern "C" {
#endif

/* pacman_recurrence_v1_configure accepts this larger options struct (struct_size = its size): the
 * reference's fields, then the executor of runs (0: the on-chip executor when a block of the
 * plan's points fits shared memory, else the global-arena one; 1: always the global-arena executor;
 * 2: the on-chip executor, or INVALID at run time when it does not fit) and the on-chip
 * executor's lanes per point (0: automatic; as pacuda_b200_plan_set_lanes_per_point). A runner
 * given the reference's struct keeps the
 * defaults. */
typedef struct {
    pacman_recurrence_options base;
    uint32_t executor;
    uint32_t lanes_per_point;
} pacuda_b200_options;
enum { PACUDA_B200_EXECUTOR_AUTO = 0, PACUDA_B200_EXECUTOR_ARENA = 1, PACUDA_B200_EXECUTOR_ONCHIP = 2 };

typedef struct pacuda_b200_plan pacuda_b200_plan;
typedef struct pacuda_b200_batch pacuda_b200_batch;

/* A kernel kind of this API beside the reference's four (PACMAN_RECURRENCE_KERNEL_*): the f64
 * arithmetic with each product and the sum it feeds fused into one multiply-add (one rounding
 * instead of two). Not bit for bit the reference's f64 kernel; within about 1e-13 of it. */
#define PACUDA_B200_KERNEL_F64_FMA 4

/* Compiles the plan of `call` (its words, widths, plane counts, scales, factors and form terms;
 * its arrays and runs are not used) with the reduction (offsets[outputs + 1], planes, weights)
 * for the kernel kind `kernel` (PACMAN_RECURRENCE_KERNEL_* or PACUDA_B200_KERNEL_F64_FMA). NULL
 * on error, with a message on stderr. The plan may read no current plane before writing it (its
 * inputs are its sources). */
pacuda_b200_plan *pacuda_b200_plan_create(const pacman_recurrence_call *call, const uint32_t *offsets,
                                          const uint32_t *planes, const double *weights, uint32_t outputs,
                                          uint32_t kernel);
void pacuda_b200_plan_destroy(pacuda_b200_plan *plan);
/* the plan's algorithmic flops per point (fixed per-op counts) */
uint64_t pacuda_b200_plan_flops(const pacuda_b200_plan *plan);
/* the lanes that run one point's tasks: a block runs P of the plan's points at once (1 .. 32),
 * each with warps * floor(32 / P) lanes; this picks the largest P whose lanes are at least
 * `lanes` (pacuda_b200_plan_lanes_per_point returns the lanes it gives); 0 for the tuned or
 * default choice (of the point counts whose shared memory fits, the one that leaves the fewest
 * threads idle, the larger on ties); INVALID when P points do not fit */
int pacuda_b200_plan_set_lanes_per_point(pacuda_b200_plan *plan, uint32_t lanes);
uint32_t pacuda_b200_plan_lanes_per_point(const pacuda_b200_plan *plan);

/* A batch of `nplans` plans (all of one kernel kind); plan k on count[k] points. */
pacuda_b200_batch *pacuda_b200_batch_create(pacuda_b200_plan *const *plans, uint32_t nplans,
                                            const double *const *external, const uint32_t *count,
                                            double *const *output);
/* Points the batch's plans at other arrays and point counts (as batch_create takes them), without
 * allocating; a captured graph is dropped (capture again to replay). Waits for the previous run's
 * copy of the launch descriptors, not for its kernel: the caller orders its use of the old arrays. */
int pacuda_b200_batch_update(pacuda_b200_batch *batch, const double *const *external, const uint32_t *count,
                             double *const *output);
/* Times each plan's lanes-per-point choices on its own points, with 1, 2, 3, 4, 5, 8 and 16 blocks
 * per SM (those its points fit), and
 * keeps each plan's fastest pair; plans of the same blocks per SM share one launch (a run is then
 * one launch per blocks-per-SM choice in use, one after the other on the stream). */
int pacuda_b200_batch_tune(pacuda_b200_batch *batch, void *stream);
/* One persistent launch over every plan's points, on `stream` (a cudaStream_t; NULL: default). */
int pacuda_b200_batch_run(pacuda_b200_batch *batch, void *stream);
/* Captures the launch into a CUDA graph on `stream`; later runs replay it. */
int pacuda_b200_batch_capture(pacuda_b200_batch *batch, void *stream);
/* Blocks per SM of every plan's launch: 1 (one block of all the warps the registers allow), or 2, 3,
 * 4, 5, 8 or 16 independent blocks of floor(warps / blocks) warps each that share the SM's warps and
 * shared memory (while one waits at a level's barrier the others run); 0: chosen per plan without
 * timing (four for a plan of at most four points per 16-warp block, else two). Replaces the tuner's
 * per-plan choices. INVALID for another count or when the plans' points do not fit. A new batch
 * has 1. */
int pacuda_b200_batch_set_blocks_per_sm(pacuda_b200_batch *batch, uint32_t blocks);
uint32_t pacuda_b200_batch_blocks_per_sm(const pacuda_b200_batch *batch);
/* the blocks per SM plan k runs with (its own choice, else the batch's); setting 0 returns it to
 * the batch's. INVALID when its points do not fit. */
int pacuda_b200_batch_set_plan_blocks_per_sm(pacuda_b200_batch *batch, uint32_t plan, uint32_t blocks);
uint32_t pacuda_b200_batch_plan_blocks_per_sm(const pacuda_b200_batch *batch, uint32_t plan);
/* the lanes per point plan k runs with in this batch's launch (its own choice where that fits the
 * launch's blocks, else the default for them), or 0 */
uint32_t pacuda_b200_batch_lanes_per_point(const pacuda_b200_batch *batch, uint32_t plan);
/* kernel launches of one run (one per blocks-per-SM choice in use) */
uint32_t pacuda_b200_batch_launches(const pacuda_b200_batch *batch);
void pacuda_b200_batch_destroy(pacuda_b200_batch *batch);

/* Evaluates plans as a batch of them would, without a batch object and without allocating
 * anything: the launch's descriptors and its work-item counter live in a fixed array of this
 * library in device memory (one per device), which a small setup kernel fills and zeroes on
 * `stream` before the executor's launch (2 kernel launches). No counterpart in the reference.
 * For callers that cannot allocate device or pinned memory when they evaluate.
 * Limits: 1 to PACUDA_B200_STATIC_MAX_PLANS plans, else INVALID (with a message on stderr). Calls
 * on one device must not overlap in time (they share the array): use one stream, or order them.
 * The first call in each context of a device (so the first on each device, and the first after a
 * device reset), with that device current, looks up the array's address (which may load the
 * library's device code); make it before capturing any stream on that device. The launch is one
 * block per SM (a batch may run several), each plan with its own points per block when the
 * launch's shared memory allows: the same values as a batch, not always its speed. */
#define PACUDA_B200_STATIC_MAX_PLANS 8
int pacuda_b200_run_static(pacuda_b200_plan *const *plans, uint32_t nplans, const double *const *external,
                           const uint32_t *count, double *const *output, void *stream);

/* The rotated-momentum stability check's device steps (no counterpart in the reference).
 * rotate: source-major momenta [(leg * 4 + k) * n + i] of n points with every leg's spatial part
 * turned by the row-major 3x3 `rotation` (host array), energies kept, into `out`.
 * compare: the helicity sums over `parts` output arrays a[k] and b[k] ([i][outputs[k]] each; the
 * pointer arrays and `outputs` in device memory); a point whose sums differ by more than `tol`
 * relative, or are not finite, is appended (in no particular order) to index[], *count (zeroed by
 * the caller) counting them.
 * gather: the momenta of points index[0 .. *count) into `out` (source-major with stride *count);
 * scatter: their outputs src[j][outputs] back into dst[index[j]][outputs]; both launch for up to
 * `capacity` points and read the count on the device. */
int pacuda_b200_rotate(const double *external, uint32_t legs, uint32_t n, const double *rotation, double *out,
                       void *stream);
int pacuda_b200_compare(const double *const *a, const double *const *b, const uint32_t *outputs, uint32_t parts,
                        uint32_t n, double tol, uint32_t *index, uint32_t *count, void *stream);
int pacuda_b200_gather(const double *external, uint32_t legs, uint32_t n, const uint32_t *index, const uint32_t *count,
                       uint32_t capacity, double *out, void *stream);
int pacuda_b200_scatter(const double *src, uint32_t outputs, const uint32_t *index, const uint32_t *count,
                        uint32_t capacity, double *dst, void *stream);

/* Measurement: launches blocks x threads threads that each run 8 independent chains of
 * `iterations` f64 fused multiply-adds (2 flops each) on `stream`; the caller times it. `sink`
 * is a device array of at least *blocks doubles (never written in practice). */
int pacuda_b200_measure_fp64(double *sink, uint32_t iterations, uint32_t *blocks, uint32_t *threads, void *stream);

#ifdef __cplusplus
}
#endif
#endif
