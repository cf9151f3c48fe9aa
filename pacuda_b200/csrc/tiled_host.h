// Host helpers of the on-chip executor: a schedule's device copy, its shared-memory footprint,
// the warps that fit, and the launch.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "schedule.h"

namespace pacuda {

struct TiledPlan;
struct TiledLaunch;

// points per block: 1 .. kMaxPoints; a point then has warps * floor(32 / P) lanes (a lane of all
// P points is P adjacent threads of one warp)
constexpr uint32_t kMaxPoints = 32;
// blocks per SM: 1 (one block of all the warps the registers allow) or several independent blocks
// that share those warps and reach their barriers at different times; a block of b per SM has
// floor(warps / b) warps, so 3 and 5 leave one warp unused (16 warps: 5 x 3 = 15)
constexpr int kBlockChoices[] = {1, 2, 3, 4, 5, 8, 16};
inline bool tiled_blocks_valid(int blocks) {
    for (int b : kBlockChoices)
        if (b == blocks) return true;
    return false;
}
// the threads of a block with `blocks` per SM when one block per SM has `threads`
inline int tiled_block_threads(int threads, int blocks) {
    int warps = threads / 32 / (blocks > 0 ? blocks : 1);
    return 32 * (warps > 0 ? warps : 1);
}
inline uint32_t tiled_lanes(uint32_t points, int threads) { return (uint32_t)(threads / 32) * (32 / points); }
// a point has at most 16 warps x 32 lanes
constexpr uint32_t kMaxLanes = 512;

struct TiledDevice {
    Schedule host;
    uint4 *ins = nullptr;  // the schedule's instructions, packed (pack_ins)
    uint32_t *task_first = nullptr, *loads = nullptr, *amp_planes = nullptr;
    // per lane count G (of every blocks-per-SM choice and points per block): the lane order for G
    // lanes and its level boundaries, concatenated (offsets in 32-bit words, index G)
    uint32_t *orders = nullptr, *level_firsts = nullptr;
    size_t order_at[kMaxLanes + 1] = {0}, level_at[kMaxLanes + 1] = {0};
    int threads = 0;  // the threads of one block per SM (tiled_block_threads for several)
    uint32_t levels = 0;
    bool ok = false;
    void release();
};

// bytes of shared memory a block needs for one plan's constants (scales and factors, re and im)
size_t tiled_const_bytes(uint32_t scales, uint32_t factors);

// an instruction in the on-chip executor's 16-byte form (tiled.cuh unpack_ins); false when a field
// does not fit it
bool pack_ins(const Ins &i, uint4 &w);

// the schedule's arrays on the device, with the lane orders of every points-per-block count for
// blocks of `threads`; false (with the reason in t.host.why) when an instruction does not pack
bool upload_schedule(TiledDevice &t, int threads, cudaStream_t stream);

// bytes of shared memory one point needs (kernel: PACMAN_RECURRENCE_KERNEL_*), 16-aligned
size_t tiled_point_bytes(const Schedule &s, uint32_t forms, int kernel);

// a block's threads with `blocks` blocks per SM (as the kernel's registers allow, at most 512 per
// SM) and its largest dynamic shared memory
int tiled_threads(int kernel, int blocks = 1);
size_t tiled_max_smem(int kernel, int blocks = 1);

// whether a block of `threads` runs `points` points within `max_smem` bytes
bool tiled_points_fit(uint32_t points, size_t point_bytes, int threads, size_t max_smem);
// the most points per block that fit, or 0
uint32_t tiled_max_points(size_t point_bytes, int threads, size_t max_smem);
// Blocks per SM chosen without timing for points of `point_bytes` and constants of `const_bytes`:
// four (their points run on fewer, independent warps: 4 each) when at most four points fit a
// block of all the warps, else two; fewer when the points do not fit. (Measured on B200: gg>ggg,
// 4 points per 16 warps, gains 5 % at four blocks over two; five blocks' shared memory leaves L1
// too little room for its instruction stream since the spread slot layout; qg>qgg, 16 points,
// loses 14 % at four.)
int tiled_auto_blocks(int kernel, size_t point_bytes, size_t const_bytes);

// the default points per block: of those that fit, the count that leaves the fewest threads of a
// warp without a lane (P * floor(32 / P) largest), the larger on ties; 0 when none fits
uint32_t tiled_default_points(size_t point_bytes, int threads, size_t max_smem);

// fills the schedule fields of a plan descriptor for `points` points per block, `blocks` per SM
void describe(const TiledDevice &t, uint32_t forms, uint32_t points, size_t point_bytes, TiledPlan &p, int blocks = 1);

// launches the persistent kernel (`grid` blocks: the SMs times the blocks per SM) with `smem` bytes
// of shared memory
bool launch_tiled(int kernel, const TiledLaunch &args, int threads, size_t smem, int grid, cudaStream_t stream);

}  // namespace pacuda
