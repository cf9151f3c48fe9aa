/* The surrogate of |M|^2: a small network trained on points the recurrence evaluates, used as the
 * first stage of two-stage unweighting (libsurrogate.so). No counterpart in the reference: its
 * runner has no learned part.
 *
 * The network: inputs x (up to 64 features, the phase-space unit-cube numbers and a subprocess
 * one-hot), four hidden layers of width 256 with SiLU, one output:
 *   h1 = silu(W1 x + b1), h2 = silu(W2 h1 + b2), h3 = silu(W3 h2 + b3), h4 = silu(W4 h3 + b4),
 *   out = w5 . h4 + b5,
 * silu(z) = z (1 + tanh(z / 2)) / 2. BF16 weights and activations in the tensor-core products
 * (tcgen05.mma, FP32 accumulation in tensor memory); FP32 master weights, biases, the output
 * layer and the Adam state. The training loss is the mean squared error of out against targets y.
 *
 * Parameters, as one FP32 vector (pacuda_sg_param_count values), in this order: W1 [256][64]
 * (row = output, column = input feature; columns at or beyond the network's input count stay 0),
 * b1 [256], W2 [256][256], b2, W3, b3, W4, b4, w5 [256], b5 [1].
 *
 * Device pointers throughout; `stream` is a cudaStream_t (NULL: the legacy default stream).
 * Status: 0 OK, 2 INVALID (bad arguments, with a message on stderr), 3 DEVICE_ERROR (a CUDA call
 * failed or a kernel's bounded wait gave up; the network should then be destroyed). */
#ifndef PACUDA_SURROGATE_H
#define PACUDA_SURROGATE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pacuda_sg_net pacuda_sg_net;

#define PACUDA_SG_WIDTH 256
#define PACUDA_SG_MAX_INPUTS 64

/* the FP32 parameter count of a network */
size_t pacuda_sg_param_count(void);

/* A network with `inputs` (1 .. 64) features, its weights drawn from `seed` (uniform in
 * +-sqrt(6 / fan_in) for W, zero biases), training workspace for batches of up to `max_batch`
 * points (a multiple of 128). NULL on failure. */
pacuda_sg_net *pacuda_sg_create(uint32_t inputs, uint32_t max_batch, uint64_t seed);
void pacuda_sg_destroy(pacuda_sg_net *net);

/* Copies `params` (host, pacuda_sg_param_count FP32 values) into the network, or its parameters
 * out to `params`; setting resets the Adam state. */
int pacuda_sg_set_params(pacuda_sg_net *net, const float *params);
int pacuda_sg_get_params(const pacuda_sg_net *net, float *params);

/* The gradient of the loss mean((out - y)^2) over `batch` points (a multiple of 128, at most
 * max_batch) with respect to every parameter, into `grad` (device, param order) and the loss into
 * `loss` (device, one float). x: device FP32 [batch][inputs]; y: device FP32 [batch]. */
int pacuda_sg_gradients(pacuda_sg_net *net, const float *x, const float *y, uint32_t batch, float *grad, float *loss,
                        void *stream);

/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8, learning rate `lr`) on the gradient of one
 * batch, as pacuda_sg_gradients computes it; the loss of the batch (before the step) is added to
 * `loss_sum` (device, one float) when it is not NULL. */
int pacuda_sg_train_step(pacuda_sg_net *net, const float *x, const float *y, uint32_t batch, float lr, float *loss_sum,
                         void *stream);

/* One Adam step (as pacuda_sg_train_step takes it) on a gradient the caller supplies (device,
 * param order): data-parallel training averages pacuda_sg_gradients over the ranks' shards (one
 * all-reduce of pacuda_sg_param_count floats) and applies the mean on every rank. */
int pacuda_sg_apply_gradients(pacuda_sg_net *net, const float *grad, float lr, void *stream);

/* out[i] for `count` points of x (device FP32 [count][inputs]) with the fused inference kernel
 * (all layers of a tile of 128 points in one block, weights streamed through shared memory). */
int pacuda_sg_forward(const pacuda_sg_net *net, const float *x, uint32_t count, float *out, void *stream);

/* the error flag of the network's kernels: 0 none, else the code of the first bounded wait that
 * gave up; -1 when it cannot be read */
int pacuda_sg_error(const pacuda_sg_net *net);

/* ---- two-stage unweighting of massless 2 -> 3 and 2 -> 4 at fixed sqrt(s) ----
 *
 * `final_state` is the number of final-state partons N, 3 or 4. Candidate i of a stream with seed
 * S has 3N - 2 uniforms from a xorshift64 stream started at splitmix64(S ^ (i * 0xD1B54A32D192ED03))
 * | 1: the 3N - 4 phase-space numbers x, then the two accept/reject uniforms (u5 and u6 for N = 3,
 * u8 and u9 for N = 4). Legs 0 and 1 are the beams.
 * N = 3 (sequential two-body decays, importance-sampled): s23 = s sigma(16 (2 x1 - 1)) with sigma
 * the logistic function; leg 2 (p1) in the centre-of-mass frame with |p1| = (s - s23) / (2 sqrt(s)),
 * cos(theta) = tanh(5.5 (2 x2 - 1)), phi = 2 pi x3; legs 3 and 4 back to back in the rest frame of
 * P - p1, cos(theta) = tanh(7 (2 x4 - 1)), phi = 2 pi x5, boosted. Its phase-space weight (the
 * density of the unit cube) J = s (1 - sigma) / (128 pi^3) x 32 sigma (1 - sigma) x
 * 5.5 (1 - cos^2 theta1) x 7 (1 - cos^2 theta2).
 * N = 4: s_Q = s sigma(16 (2 x1 - 1)), s_R = s_Q sigma(16 (2 x4 - 1)); leg 2 as above (x2, x3) with
 * |p1| = (s - s_Q) / (2 sqrt(s)); leg 3 in the rest frame of Q = P - p1 with |p| = (s_Q - s_R) /
 * (2 sqrt(s_Q)), cos(theta) = tanh(7 (2 x5 - 1)), phi = 2 pi x6; legs 4 and 5 back to back in the
 * rest frame of R = Q - p2, cos(theta) = tanh(7 (2 x7 - 1)), phi = 2 pi x8, boosted to Q's frame
 * and then with leg 3 to the lab. J = s s_Q (1 - sigma1) (1 - sigma2) / (2048 pi^5) x
 * 32 sigma1 (1 - sigma1) x 32 sigma2 (1 - sigma2) x 5.5 (1 - cos^2 theta1) x 7 (1 - cos^2 theta2) x
 * 7 (1 - cos^2 theta3).
 * The network's inputs: the 3N - 4 numbers x, then a one-hot of the subprocess (`family`), zeros
 * after. */
#define PACUDA_UW_MAX_SEGMENTS 8

typedef struct pacuda_uw_cuts {
    double pt_min, eta_max, dr_min; /* pT > pt_min, |eta| < eta_max, pairwise Delta R > dr_min (legs 2 .. N + 1) */
} pacuda_uw_cuts;

/* candidates first .. first + count - 1: the indices of those inside the cuts, appended in no
 * particular order to index[] (at most `capacity`; *counter, which the caller zeroes, counts them
 * all) */
int pacuda_uw_candidates(uint64_t seed, uint64_t first, uint32_t count, uint32_t final_state, double sqrt_s,
                         const pacuda_uw_cuts *cuts, uint64_t *index, uint32_t capacity, unsigned long long *counter,
                         void *stream);

/* Several subprocesses' candidate lists in one launch (each segment as pacuda_uw_candidates takes
 * it; at most PACUDA_UW_MAX_SEGMENTS, every index array holding `capacity` entries). */
typedef struct pacuda_uw_candidate_segment {
    uint64_t seed, first;
    uint32_t count;
    uint64_t *index;
    unsigned long long *counter;
} pacuda_uw_candidate_segment;
int pacuda_uw_candidates_segments(const pacuda_uw_candidate_segment *segments, uint32_t segment_count,
                                  uint32_t final_state, double sqrt_s, const pacuda_uw_cuts *cuts, uint32_t capacity,
                                  void *stream);

/* the points of candidates index[0 .. n): momenta as the runner reads them (source-major,
 * [(leg * 4 + k) * n + i]), the network's inputs [i][input_count] and J (each output may be NULL) */
int pacuda_uw_points(uint64_t seed, const uint64_t *index, uint32_t n, uint32_t final_state, double sqrt_s,
                     double *momenta, float *inputs, uint32_t input_count, uint32_t family, double *jac, void *stream);

/* Stage 1 in one launch of the fused inference kernel: for the candidates index[0 .. count) of
 * subprocess `family` (inside the cuts, as pacuda_uw_candidates lists them), the network's inputs
 * and the surrogate s = exp(mu + sigma out), the network's estimate of the candidate's weight
 * w = |M|^2 J; a candidate is kept when (its first decision uniform) s_max < s. Kept candidates' indices and s are appended
 * in no particular order (at most `capacity`); *counter (zeroed by the caller) counts the kept
 * ones, also beyond the capacity. */
int pacuda_uw_stage1(const pacuda_sg_net *net, uint64_t seed, const uint64_t *index, uint32_t count,
                     uint32_t final_state, uint32_t family, double mu, double sigma, double s_max, uint64_t *kept_index,
                     double *kept_s, uint32_t capacity, unsigned long long *counter, void *stream);

/* Several subprocesses' first stages in one launch: segment k is stage 1 of its own candidates
 * (seed, index[0 .. count), family, s_max) into its own outputs (kept_index, kept_s, *kept_count,
 * which the caller zeroes); every output array holds `capacity` entries. At most
 * PACUDA_UW_MAX_SEGMENTS segments. */
typedef struct pacuda_uw_segment {
    uint64_t seed;
    const uint64_t *index;
    uint32_t count, family;
    double s_max;
    uint64_t *kept_index;
    double *kept_s;
    unsigned long long *kept_count;
} pacuda_uw_segment;
int pacuda_uw_stage1_segments(const pacuda_sg_net *net, const pacuda_uw_segment *segments, uint32_t segment_count,
                              uint32_t final_state, double mu, double sigma, uint32_t capacity, void *stream);

/* The decision on points whose exact |M|^2 the runner evaluated (outputs [i][helicities], summed):
 * w = |M|^2 J. Plain unweighting (s == NULL): kept when (the first decision uniform) w_max < w,
 * weight max(1, w / w_max). Second stage (s = the first stage's values): r = w / s, kept when (the
 * second decision uniform) r_max < r, weight max(1, s / s_max) max(1, r / r_max). keep (0/1),
 * weight and me (= |M|^2) may be NULL. */
int pacuda_uw_decide(uint64_t seed, const uint64_t *index, uint32_t n, uint32_t final_state, const double *outputs,
                     uint32_t helicities, const double *jac, const double *s, double w_max, double s_max,
                     double r_max, uint8_t *keep, double *weight, double *me, void *stream);

/* Blocks per SM of the fused inference kernel (pacuda_sg_forward, the first stage): 2 (the
 * default; two blocks whose products and epilogues overlap, a 2-stage weight ring each) or 1 (one
 * block with a 9-stage weight ring); INVALID otherwise. Applies to later launches in the process. */
int pacuda_sg_set_inference_blocks(uint32_t blocks);

/* kernel launches made by the last call of each entry point (0 for none) */
uint32_t pacuda_sg_last_launches(void);

#ifdef __cplusplus
}
#endif

#endif
