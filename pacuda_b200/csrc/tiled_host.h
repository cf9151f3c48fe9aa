// Host helpers of the on-chip executor: a schedule's device copy, its shared-memory footprint,
// the warps that fit, and the launch.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "schedule.h"

namespace pacuda {

struct TiledPlan;
struct TiledLaunch;

struct TiledDevice {
    Schedule host;
    Ins *ins = nullptr;
    uint32_t *task_first = nullptr, *loads = nullptr, *amp_planes = nullptr;
    // per lanes-per-point exponent 0 .. 9: the tasks' order and its level boundaries
    uint32_t *order[10] = {nullptr}, *level_first[10] = {nullptr};
    uint32_t levels = 0;
    bool ok = false;
    void release();
};

// bytes of shared memory a block needs for one plan's constants (scales and factors, re and im)
size_t tiled_const_bytes(uint32_t scales, uint32_t factors);

// the schedule's arrays on the device
bool upload_schedule(TiledDevice &t, cudaStream_t stream);

// bytes of shared memory one point needs (kernel: PACMAN_RECURRENCE_KERNEL_*), 16-aligned
size_t tiled_point_bytes(const Schedule &s, uint32_t forms, int kernel);

// the block's threads (as the kernel's registers allow, at most 512) and its largest shared memory
int tiled_threads(int kernel);
size_t tiled_max_smem(int kernel);

// the smallest lanes-per-point exponent whose block of points fits shared memory, or -1
int tiled_min_log_lanes(size_t point_bytes, int threads, size_t max_smem);

// fills the schedule fields of a plan descriptor
void describe(const TiledDevice &t, uint32_t forms, uint32_t log_lanes, size_t point_bytes, TiledPlan &p);

// launches the persistent kernel (one block per SM) with `smem` bytes of shared memory
bool launch_tiled(int kernel, const TiledLaunch &args, int threads, size_t smem, int sms, cudaStream_t stream);

}  // namespace pacuda
