// The rotated-momentum stability check's device steps (include/pacuda_b200.h): momenta turned by
// a rotation, the comparison of two evaluations' helicity sums with a compact list of the points
// that fail it, and the gather / scatter that re-evaluate those points in f64 and put their
// outputs in place. No counterpart in the reference (its runner has no such check).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/pacman_recurrence.h"
#include "../../include/pacuda_b200.h"

namespace {

struct Rotation {
    double r[9];
};

// every leg's spatial components turned by r (row-major 3x3), energies kept; source-major
// momenta [(leg * 4 + k) * n + i]
__global__ void rotate_kernel(const double *ext, uint32_t legs, uint32_t n, Rotation rot, double *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (uint32_t l = 0; l < legs; l++) {
        const double *p = ext + (size_t)l * 4 * n;
        double *q = out + (size_t)l * 4 * n;
        const double e = p[i], x = p[n + i], y = p[2 * (size_t)n + i], z = p[3 * (size_t)n + i];
        q[i] = e;
        q[n + i] = rot.r[0] * x + rot.r[1] * y + rot.r[2] * z;
        q[2 * (size_t)n + i] = rot.r[3] * x + rot.r[4] * y + rot.r[5] * z;
        q[3 * (size_t)n + i] = rot.r[6] * x + rot.r[7] * y + rot.r[8] * z;
    }
}

// the helicity sums of parts a[k] and b[k] (outputs [i][outputs[k]] each, summed over the parts);
// a point whose sums differ by more than tol relative, or are not finite, is appended to `index`
__global__ void compare_kernel(const double *const *a, const double *const *b, const uint32_t *outputs, uint32_t parts,
                               uint32_t n, double tol, uint32_t *index, uint32_t *count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = false;
    if (i < n) {
        double sa = 0.0, sb = 0.0;
        for (uint32_t k = 0; k < parts; k++)
            for (uint32_t h = 0; h < outputs[k]; h++) {
                sa += a[k][(size_t)i * outputs[k] + h];
                sb += b[k][(size_t)i * outputs[k] + h];
            }
        const double d = fabs(sa - sb), m = fabs(sa);
        bad = !(d <= tol * m) || !isfinite(sa) || !isfinite(sb);
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, bad);
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == 0 && ballot) base = atomicAdd(count, (uint32_t)__popc(ballot));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (bad) index[base + __popc(ballot & ((1u << lane) - 1u))] = i;
}

// momenta of the listed points (source-major, stride m) from those of all n points
__global__ void gather_kernel(const double *ext, uint32_t legs, uint32_t n, const uint32_t *index, const uint32_t *count,
                              double *out) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x, m = *count;
    if (j >= m) return;
    const uint32_t i = index[j];
    for (uint32_t c = 0; c < 4 * legs; c++) out[(size_t)c * m + j] = ext[(size_t)c * n + i];
}

// outputs of the listed points ([j][outputs]) put in their places ([i][outputs])
__global__ void scatter_kernel(const double *src, uint32_t outputs, const uint32_t *index, const uint32_t *count,
                               double *dst) {
    const uint32_t j = blockIdx.x, m = *count;
    if (j >= m) return;
    const uint32_t i = index[j];
    for (uint32_t h = threadIdx.x; h < outputs; h += blockDim.x) dst[(size_t)i * outputs + h] = src[(size_t)j * outputs + h];
}

bool failed(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return false;
    fprintf(stderr, "pacuda b200: %s: %s\n", what, cudaGetErrorString(e));
    return true;
}

}  // namespace

extern "C" int pacuda_b200_rotate(const double *external, uint32_t legs, uint32_t n, const double *rotation,
                                  double *out, void *stream) {
    if (!external || !out || !rotation || legs == 0) return PACMAN_RECURRENCE_INVALID;
    if (n == 0) return PACMAN_RECURRENCE_OK;
    Rotation r;
    for (int k = 0; k < 9; k++) r.r[k] = rotation[k];
    rotate_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(external, legs, n, r, out);
    return failed("rotate") ? PACMAN_RECURRENCE_DEVICE_ERROR : PACMAN_RECURRENCE_OK;
}

extern "C" int pacuda_b200_compare(const double *const *a, const double *const *b, const uint32_t *outputs,
                                   uint32_t parts, uint32_t n, double tol, uint32_t *index, uint32_t *count,
                                   void *stream) {
    if (!a || !b || !outputs || !index || !count || parts == 0) return PACMAN_RECURRENCE_INVALID;
    if (n == 0) return PACMAN_RECURRENCE_OK;
    compare_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(a, b, outputs, parts, n, tol, index, count);
    return failed("compare") ? PACMAN_RECURRENCE_DEVICE_ERROR : PACMAN_RECURRENCE_OK;
}

extern "C" int pacuda_b200_gather(const double *external, uint32_t legs, uint32_t n, const uint32_t *index,
                                  const uint32_t *count, uint32_t capacity, double *out, void *stream) {
    if (!external || !index || !count || !out || legs == 0) return PACMAN_RECURRENCE_INVALID;
    if (capacity == 0) return PACMAN_RECURRENCE_OK;
    gather_kernel<<<(capacity + 255) / 256, 256, 0, (cudaStream_t)stream>>>(external, legs, n, index, count, out);
    return failed("gather") ? PACMAN_RECURRENCE_DEVICE_ERROR : PACMAN_RECURRENCE_OK;
}

extern "C" int pacuda_b200_scatter(const double *src, uint32_t outputs, const uint32_t *index, const uint32_t *count,
                                   uint32_t capacity, double *dst, void *stream) {
    if (!src || !index || !count || !dst || outputs == 0) return PACMAN_RECURRENCE_INVALID;
    if (capacity == 0) return PACMAN_RECURRENCE_OK;
    scatter_kernel<<<capacity, 64, 0, (cudaStream_t)stream>>>(src, outputs, index, count, dst);
    return failed("scatter") ? PACMAN_RECURRENCE_DEVICE_ERROR : PACMAN_RECURRENCE_OK;
}
