// Host helpers of the on-chip executor (tiled_host.h).
#include <stdio.h>

#include <algorithm>

#include "../../include/pacman_recurrence.h"
#include "tiled.cuh"
#include "tiled_host.h"

namespace pacuda {

namespace {
template <class T> bool put(T **dst, const std::vector<T> &v, cudaStream_t s) {
    size_t bytes = std::max<size_t>(1, v.size()) * sizeof(T);
    if (cudaMalloc((void **)dst, bytes) != cudaSuccess) return false;
    return v.empty() || cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s) == cudaSuccess;
}

template <class K> const void *kernel_of(bool abi) {
    return abi ? (const void *)run_tiled<K, true> : (const void *)run_tiled<K, false>;
}

const void *kernel_for(int kernel, bool abi = false) {
    switch (kernel) {
    case PACMAN_RECURRENCE_KERNEL_F64: return kernel_of<KindF64>(abi);
    case PACMAN_RECURRENCE_KERNEL_MIXED: return kernel_of<KindMixed>(abi);
    case PACMAN_RECURRENCE_KERNEL_MIXED64: return kernel_of<KindMixed64>(abi);
    default: return kernel_of<KindDF64>(abi);
    }
}
}  // namespace

void TiledDevice::release() {
    cudaFree(ins);
    cudaFree(task_first);
    cudaFree(loads);
    cudaFree(amp_planes);
    for (int k = 0; k < kLaneChoices; k++) {
        cudaFree(order[k]);
        cudaFree(level_first[k]);
        order[k] = level_first[k] = nullptr;
    }
    ins = nullptr;
    task_first = loads = amp_planes = nullptr;
    ok = false;
}

bool upload_schedule(TiledDevice &t, cudaStream_t s) {
    t.ok = put(&t.ins, t.host.ins, s) && put(&t.task_first, t.host.task_first, s) && put(&t.loads, t.host.loads, s) &&
           put(&t.amp_planes, t.host.amp_planes, s);
    t.levels = (uint32_t)t.host.level_first.size() - 1;
    for (int k = 0; t.ok && k < kLaneChoices; k++) {
        std::vector<uint32_t> order, lf, ranges;
        lane_order(t.host, lanes_of_choice(k), order, lf);
        // each position holds its task's instruction range (first, end); (0, 0) for none
        ranges.reserve(2 * order.size());
        for (uint32_t task : order) {
            ranges.push_back(task == ~0u ? 0 : t.host.task_first[task]);
            ranges.push_back(task == ~0u ? 0 : t.host.task_first[task + 1]);
        }
        t.ok = put(&t.order[k], ranges, s) && put(&t.level_first[k], lf, s);
    }
    // the host vectors must outlive the asynchronous copies
    cudaStreamSynchronize(s);
    return t.ok;
}

size_t tiled_const_bytes(uint32_t scales, uint32_t factors) { return ((2 * (size_t)scales + 2 * factors) * 8 + 15) / 16 * 16; }

size_t tiled_point_bytes(const Schedule &s, uint32_t forms, int kernel) {
    size_t value = kernel == PACMAN_RECURRENCE_KERNEL_MIXED || kernel == PACMAN_RECURRENCE_KERNEL_MIXED64 ? 4 : 8;
    size_t per_point = 2 * value * s.cur_slots + 2 * 8 * s.amp_slots + 8 * 4 * (size_t)forms;
    return (per_point + 15) / 16 * 16;
}

int tiled_threads(int kernel) {
    cudaFuncAttributes attr, abi;
    if (cudaFuncGetAttributes(&attr, kernel_for(kernel, false)) != cudaSuccess ||
        cudaFuncGetAttributes(&abi, kernel_for(kernel, true)) != cudaSuccess)
        return 0;
    attr.numRegs = std::max(attr.numRegs, abi.numRegs);
    attr.maxThreadsPerBlock = std::min(attr.maxThreadsPerBlock, abi.maxThreadsPerBlock);
    int dev = 0, regs = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&regs, cudaDevAttrMaxRegistersPerBlock, dev);
    int per_warp = ((attr.numRegs * 32 + 255) / 256) * 256;
    int warps = per_warp ? regs / per_warp : 16;
    warps = std::min(warps, attr.maxThreadsPerBlock / 32);
    // a power of two of warps: points (and their barriers) tile the block evenly
    int w = 1;
    while (2 * w <= std::min(warps, 16)) w *= 2;
    return 32 * w;
}

size_t tiled_max_smem(int kernel) {
    cudaFuncAttributes attr, abi;
    if (cudaFuncGetAttributes(&attr, kernel_for(kernel, false)) != cudaSuccess ||
        cudaFuncGetAttributes(&abi, kernel_for(kernel, true)) != cudaSuccess)
        return 0;
    attr.sharedSizeBytes = std::max(attr.sharedSizeBytes, abi.sharedSizeBytes);
    int dev = 0, smem = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return (size_t)smem - attr.sharedSizeBytes;
}

bool tiled_lanes_fit(uint32_t lanes, size_t point_bytes, int threads, size_t max_smem) {
    if (lane_choice(lanes) < 0 || threads <= 0 || lanes > (uint32_t)threads) return false;
    // lanes < 32: a warp's 32 / L points; lanes >= 32: one point per L / 32 warps
    uint32_t per = (uint32_t)threads / lanes;
    if (lanes > 32 && per > 15) return false;
    return (size_t)per * point_bytes <= max_smem;
}

uint32_t tiled_min_lanes(size_t point_bytes, int threads, size_t max_smem) {
    for (int c = 0; c < kLaneChoices; c++)
        if (tiled_lanes_fit(lanes_of_choice(c), point_bytes, threads, max_smem)) return lanes_of_choice(c);
    return 0;
}

void describe(const TiledDevice &t, uint32_t forms, uint32_t lanes, size_t point_bytes, TiledPlan &p) {
    int choice = lane_choice(lanes);
    p.ins = t.ins;
    p.task_first = t.task_first;
    p.order = t.order[choice];
    p.level_first = t.level_first[choice];
    p.levels = t.levels;
    p.cur_slots = t.host.cur_slots;
    p.amp_slots = t.host.amp_slots;
    p.forms = forms;
    p.lanes = lanes;
    p.log_lanes = lanes < 32 ? (uint32_t)choice : 5;
    p.point_bytes = (uint32_t)point_bytes;
    p.loads = t.loads;
    p.nloads = (uint32_t)t.host.loads.size() / 3;
    p.amp_planes = t.amp_planes;
}

bool launch_tiled(int kernel, const TiledLaunch &args, int threads, size_t smem, int sms, cudaStream_t stream) {
    const void *fn = kernel_for(kernel, args.abi);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return false;
    void *params[] = {(void *)&args};
    return cudaLaunchKernel(fn, dim3(sms), dim3(threads), params, smem, stream) == cudaSuccess;
}

}  // namespace pacuda
