// Host helpers of the on-chip executor: a schedule's device copy, its shared-memory footprint,
// the warps that fit, and the launch.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "schedule.h"

namespace pacuda {

struct TiledPlan;
struct TiledLaunch;

// lanes per point: 1, 2, 4, 8, 16 (several points per warp), then every multiple of 32 up to 512
// (a point over several warps); choice c indexes that sequence
constexpr int kLaneChoices = 21;
inline uint32_t lanes_of_choice(int c) { return c < 5 ? 1u << c : 32u * (uint32_t)(c - 4); }
inline int lane_choice(uint32_t lanes) {
    if (lanes == 0 || lanes > 512) return -1;
    if (lanes < 32) return (lanes & (lanes - 1)) ? -1 : __builtin_ctz(lanes);
    return lanes % 32 ? -1 : 4 + (int)(lanes / 32);
}

struct TiledDevice {
    Schedule host;
    Ins *ins = nullptr;
    uint32_t *task_first = nullptr, *loads = nullptr, *amp_planes = nullptr;
    // per lane choice: the tasks' order and its level boundaries
    uint32_t *order[kLaneChoices] = {nullptr}, *level_first[kLaneChoices] = {nullptr};
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

// whether a block of `threads` runs points of `lanes` lanes within `max_smem` bytes: its
// threads / lanes points fit, and at most 15 of them span several warps (named barriers 1 .. 15)
bool tiled_lanes_fit(uint32_t lanes, size_t point_bytes, int threads, size_t max_smem);
// the fewest lanes per point that fit, or 0
uint32_t tiled_min_lanes(size_t point_bytes, int threads, size_t max_smem);

// fills the schedule fields of a plan descriptor
void describe(const TiledDevice &t, uint32_t forms, uint32_t lanes, size_t point_bytes, TiledPlan &p);

// launches the persistent kernel (one block per SM) with `smem` bytes of shared memory
bool launch_tiled(int kernel, const TiledLaunch &args, int threads, size_t smem, int sms, cudaStream_t stream);

}  // namespace pacuda
