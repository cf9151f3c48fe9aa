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
    uint32_t *task_first = nullptr, *level_first = nullptr, *loads = nullptr, *amp_planes = nullptr;
    bool ok = false;
    void release();
};

// the schedule's arrays on the device
bool upload_schedule(TiledDevice &t, cudaStream_t stream);

// bytes of shared memory one warp needs for P = 1 << log_p points (kernel: PACMAN_RECURRENCE_KERNEL_*)
size_t tiled_warp_bytes(const Schedule &s, uint32_t forms, int kernel, uint32_t log_p);

// the warps per block the kernel can run with this much shared memory per warp (0: none fit)
int tiled_warps(int kernel, size_t warp_bytes);

// fills the schedule fields of a plan descriptor
void describe(const TiledDevice &t, uint32_t forms, uint32_t log_p, size_t warp_bytes, TiledPlan &p);

// launches the persistent kernel: `launch` points to device memory holding the TiledLaunch
bool launch_tiled(int kernel, const TiledLaunch &args, int warps, size_t warp_bytes, int sms, cudaStream_t stream);

}  // namespace pacuda
