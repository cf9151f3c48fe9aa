/* The CPU oracle of the recurrence runner: TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference runner's arithmetic (runner/recurrence_runner.cu),
 * used by tests/, by __graft_entry__.smoke() and by bench.py's CPU baseline as the checker and
 * the timed CPU port. The product library (pacuda_b200/librecurrence.so) never links or calls
 * it. Built with -O2 -ffp-contract=off so that its f64 path performs the reference's f64
 * operations one by one, without contraction.
 *
 * Pinning: the oracle's f64 results are compared bit for bit with the reference runner built
 * from its own sources (oracle/_ref/librecurrence.so) on the GPU box, and its sources with the
 * reference's legend (tests/check_sources.py, golden vectors in tests/golden/).
 */
#ifndef PACUDA_ORACLE_H
#define PACUDA_ORACLE_H
#include "../include/pacman_recurrence.h"
#ifdef __cplusplus
extern "C" {
#endif

/* One plan run with the caller's arrays as the whole arena: current_re/current_im hold
 * current_planes planes of `stride` (every plane, read and written in place), amplitude_re /
 * amplitude_im likewise; the upload/download run lists are not used (the arrays are the
 * device state). zero_amplitude runs are cleared; forms come from `momenta` or, with
 * PACMAN_RECURRENCE_FORMS_ON_DEVICE, from the external momenta. `kernel` is a
 * PACMAN_RECURRENCE_KERNEL_* value; non-f64 kernels convert the arrays into their layout on
 * entry and back on exit, as the reference's uploads and downloads do. `threads` <= 0: all.
 * Returns a PACMAN_RECURRENCE_* status. */
int oracle_run(const pacman_recurrence_call *call, int kernel, int sort, int threads);

/* The reductions of a kept run, on the caller's f64 amplitude arrays (stride `stride`). */
int oracle_reduce(const pacman_recurrence_reduce *r, const double *amplitude_re,
                  const double *amplitude_im, uint32_t stride);
int oracle_reduce_resolved(const pacman_recurrence_reduce_resolved *r, const double *amplitude_re,
                           const double *amplitude_im, uint32_t stride);
int oracle_reduce_sample(const pacman_recurrence_reduce_sample *r, const double *amplitude_re,
                         const double *amplitude_im, uint32_t stride);

/* The external wavefunctions (4 components per item, unused ones 0). */
int oracle_sources(const uint32_t *codes, const double *masses, const double *momenta,
                   uint32_t count, double *out_re, double *out_im);

/* The decoded rows of a plan, 9 u32 per row (op, then its 8 fields in word order); op 14 rows
 * carry kernel, inputs, pairs, direct. Returns the row count (rows may be NULL to count), or
 * -1 on a malformed plan. With sort != 0 the contribution runs are sorted as the runner does. */
int oracle_decode(const uint64_t *words, uint32_t count, const uint8_t *width, int sort,
                  uint32_t *rows, uint32_t capacity);

#ifdef __cplusplus
}
#endif
#endif
