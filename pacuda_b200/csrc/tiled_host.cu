// Host helpers of the on-chip executor (tiled_host.h).
#include <stdio.h>

#include <algorithm>

#include "../../include/pacman_recurrence.h"
#include "../../include/pacuda_b200.h"
#include "tiled.cuh"
#include "tiled_host.h"

namespace pacuda {

namespace {
template <class T> bool put(T **dst, const std::vector<T> &v, cudaStream_t s) {
    size_t bytes = std::max<size_t>(1, v.size()) * sizeof(T);
    if (cudaMalloc((void **)dst, bytes) != cudaSuccess) return false;
    return v.empty() || cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s) == cudaSuccess;
}

}  // namespace

// the f64 kind with contracted multiply-adds (tiled_fma.cu, compiled with -fmad=true)
const void *tiled_fma_kernel(bool abi);

namespace {

template <class K> const void *kernel_of(bool abi) {
    return abi ? (const void *)run_tiled<K, true> : (const void *)run_tiled<K, false>;
}

const void *kernel_for(int kernel, bool abi = false) {
    switch (kernel) {
    case PACMAN_RECURRENCE_KERNEL_F64: return kernel_of<KindF64>(abi);
    case PACUDA_B200_KERNEL_F64_FMA: return tiled_fma_kernel(abi);
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
    cudaFree(orders);
    cudaFree(level_firsts);
    ins = nullptr;
    task_first = loads = amp_planes = orders = level_firsts = nullptr;
    ok = false;
}

bool pack_ins(const Ins &i, uint4 &w) {
    // (a closure's f records its global amplitude plane for the host; the executor reads its slot)
    uint32_t f = ins_kind(i) == K_CLOSURE ? 0 : i.f, f0 = f & 0xffff, f1 = f >> 16;
    if (ins_flags(i) > 255 || f0 > 255 || f1 > 255 || i.a > 0xffff || i.b > 0xffff || i.c > 0xffff || i.s > 0xffff ||
        i.x > 0xffff || i.y > 0xffff)
        return false;
    w.x = (i.head & 0xffff) | f0 << 16 | f1 << 24;
    w.y = i.a | i.b << 16;
    w.z = i.c | i.s << 16;
    w.w = i.x | i.y << 16;
    return true;
}

bool upload_schedule(TiledDevice &t, int threads, cudaStream_t s) {
    std::vector<uint4> packed(t.host.ins.size());
    for (size_t n = 0; n < packed.size(); n++)
        if (!pack_ins(t.host.ins[n], packed[n])) {
            t.host.why = "an instruction's field does not fit the on-chip executor's 16-byte form";
            t.ok = false;
            return false;
        }
    packed.push_back(make_uint4(0, 0, 0, 0));  // read (not run) by the prefetch after a task's last row
    t.ok = threads > 0 && put(&t.ins, packed, s) && put(&t.task_first, t.host.task_first, s) &&
           put(&t.loads, t.host.loads, s) && put(&t.amp_planes, t.host.amp_planes, s);
    t.levels = (uint32_t)t.host.level_first.size() - 1;
    t.threads = threads;
    std::vector<uint32_t> ranges, firsts;
    // one order per distinct lane count: blocks of b per SM with P points give
    // tiled_lanes(P, tiled_block_threads(threads, b)) lanes, and many pairs give the same count
    std::vector<bool> made(kMaxLanes + 1, false);
    for (int b : kBlockChoices)
        for (uint32_t np = 1; t.ok && np <= kMaxPoints; np++) {
            uint32_t lanes = tiled_lanes(np, tiled_block_threads(threads, b));
            if (lanes == 0 || lanes > kMaxLanes || made[lanes]) continue;
            made[lanes] = true;
            std::vector<uint32_t> order, lf;
            lane_order(t.host, lanes, order, lf);
            // each position holds its task's instruction range (first, end); (0, 0) for none
            t.order_at[lanes] = ranges.size();
            t.level_at[lanes] = firsts.size();
            for (uint32_t task : order) {
                ranges.push_back(task == ~0u ? 0 : t.host.task_first[task]);
                ranges.push_back(task == ~0u ? 0 : t.host.task_first[task + 1]);
            }
            firsts.insert(firsts.end(), lf.begin(), lf.end());
        }
    // the executor fetches the next position of a lane before testing it against the level's end:
    // up to a lane count past the last one
    ranges.insert(ranges.end(), 2 * kMaxLanes, 0);
    t.ok = t.ok && put(&t.orders, ranges, s) && put(&t.level_firsts, firsts, s);
    // the host vectors must outlive the asynchronous copies
    cudaStreamSynchronize(s);
    return t.ok;
}

size_t tiled_const_bytes(uint32_t scales, uint32_t factors) { return ((2 * (size_t)scales + 2 * factors) * 8 + 15) / 16 * 16; }

size_t tiled_point_bytes(const Schedule &s, uint32_t forms, int kernel) {
    size_t value = kernel == PACMAN_RECURRENCE_KERNEL_MIXED || kernel == PACMAN_RECURRENCE_KERNEL_MIXED64 ? 4 : 8;
    size_t per_point = 2 * value * s.cur_slots + 2 * 8 * s.amp_slots + 8 * (size_t)s.terms + 8 * 4 * (size_t)forms;
    return (per_point + 15) / 16 * 16;
}

int tiled_threads(int kernel, int blocks) {
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
    warps = std::max(1, std::min(warps, 16));
    return tiled_block_threads(32 * warps, blocks);
}

size_t tiled_max_smem(int kernel, int blocks) {
    cudaFuncAttributes attr, abi;
    if (cudaFuncGetAttributes(&attr, kernel_for(kernel, false)) != cudaSuccess ||
        cudaFuncGetAttributes(&abi, kernel_for(kernel, true)) != cudaSuccess)
        return 0;
    attr.sharedSizeBytes = std::max(attr.sharedSizeBytes, abi.sharedSizeBytes);
    int dev = 0, smem = 0, per_sm = 0, reserved = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    // with several blocks per SM each gets its share of the SM's shared memory
    size_t limit = blocks > 1 ? std::min<size_t>(smem, (size_t)(per_sm - blocks * reserved) / blocks) : (size_t)smem;
    return limit > attr.sharedSizeBytes ? limit - attr.sharedSizeBytes : 0;
}

bool tiled_points_fit(uint32_t points, size_t point_bytes, int threads, size_t max_smem) {
    return points >= 1 && points <= kMaxPoints && threads >= 32 && (size_t)points * point_bytes <= max_smem;
}

uint32_t tiled_max_points(size_t point_bytes, int threads, size_t max_smem) {
    for (uint32_t np = kMaxPoints; np >= 1; np--)
        if (tiled_points_fit(np, point_bytes, threads, max_smem)) return np;
    return 0;
}

int tiled_auto_blocks(int kernel, size_t point_bytes, size_t const_bytes) {
    auto most = [&](int blocks) {
        size_t room = tiled_max_smem(kernel, blocks);
        return room > const_bytes ? tiled_max_points(point_bytes, tiled_threads(kernel, blocks), room - const_bytes) : 0u;
    };
    size_t room1 = tiled_max_smem(kernel, 1);
    uint32_t one = room1 > const_bytes ? tiled_default_points(point_bytes, tiled_threads(kernel, 1), room1 - const_bytes) : 0;
    // the choices to try, most blocks first
    static const int few[] = {4, 2};
    const int *first = one && one <= 4 ? few : few + 1;
    for (const int *b = first; b != few + 2; b++)
        if (most(*b)) return *b;
    return 1;
}

uint32_t tiled_default_points(size_t point_bytes, int threads, size_t max_smem) {
    uint32_t best = 0;
    for (uint32_t np = 1; np <= kMaxPoints; np++)
        if (tiled_points_fit(np, point_bytes, threads, max_smem) && (!best || np * (32 / np) >= best * (32 / best)))
            best = np;
    return best;
}

void describe(const TiledDevice &t, uint32_t forms, uint32_t points, size_t point_bytes, TiledPlan &p, int blocks) {
    p.ins = t.ins;
    p.task_first = t.task_first;
    const uint32_t lanes = tiled_lanes(points, tiled_block_threads(t.threads, blocks));
    p.order = t.orders + t.order_at[lanes];
    p.level_first = t.level_firsts + t.level_at[lanes];
    p.levels = t.levels;
    p.cur_slots = t.host.cur_slots;
    p.amp_slots = t.host.amp_slots;
    p.terms = t.host.terms;
    p.forms = forms;
    p.points = points;
    p.lanes = lanes;
    p.point_bytes = (uint32_t)point_bytes;
    p.loads = t.loads;
    p.nloads = (uint32_t)t.host.loads.size() / 3;
    p.amp_planes = t.amp_planes;
}

bool launch_tiled(int kernel, const TiledLaunch &args, int threads, size_t smem, int grid, cudaStream_t stream) {
    const void *fn = kernel_for(kernel, args.abi);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return false;
    void *params[] = {(void *)&args};
    return cudaLaunchKernel(fn, dim3(grid), dim3(threads), params, smem, stream) == cudaSuccess;
}

}  // namespace pacuda
