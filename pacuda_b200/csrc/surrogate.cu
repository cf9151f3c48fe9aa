// The surrogate network's kernels (include/pacuda_surrogate.h): BF16 tensor-core products on
// tcgen05 with FP32 accumulators in tensor memory, operands streamed into shared memory by bulk
// copies, training by hand-written forward/backward/Adam kernels, and a fused inference kernel.
//
// Data in global memory are kept as "tile images" (umma.cuh): an A image (the M side of a
// product) is row tiles of 128 rows, each as K/64 tiles of 128 x 64 BF16 values, 16 KB each; a B
// image (the N side) is one row tile of N rows (64 or 256) as K/64 tiles of N x 64 values. One
// bulk copy moves one tile into shared memory in the layout the tensor cores read.
//
// Training (one batch of B points, B a multiple of 128):
//   forward   H_l = silu(Z_l), Z_l = H_{l-1} W_l^T + b_l     A = H_{l-1} image, B = W_l image
//   layer 4   out = w5 . bf16(h4) + b5, dout = 2 (out - y) / B, dZ4 = dout w5 silu'(z4) in the epilogue
//   backward  dZ_{l-1} = (dZ_l W_l) silu'(Z_{l-1})               A = dZ_l image, B = W_l^T image
//             dW_l = dZ_l^T H_{l-1} (split over the batch)       A = dZ_l^T image, B = H_{l-1}^T image
// Every product is C = A B^T with both operands K-major, so one kernel serves all of them; the
// epilogues write the transposed images the later products need.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <cmath>
#include <vector>

#include "../../include/pacuda_surrogate.h"
#include "phase.cuh"
#include "umma.cuh"

using namespace pacuda::umma;

namespace {

constexpr int WIDTH = PACUDA_SG_WIDTH;  // hidden width
constexpr int IN = PACUDA_SG_MAX_INPUTS;  // the first layer's K (inputs padded with zeros)
constexpr uint32_t TILE_A = 128 * 128;    // bytes of a 128-row x 64 BF16 tile
constexpr long long WAIT_CYCLES = 2000000000LL;  // a bounded wait gives up after about a second

// parameter offsets (FP32 vector)
constexpr size_t P_W1 = 0, P_B1 = P_W1 + (size_t)WIDTH * IN, P_W2 = P_B1 + WIDTH, P_B2 = P_W2 + (size_t)WIDTH * WIDTH,
                 P_W3 = P_B2 + WIDTH, P_B3 = P_W3 + (size_t)WIDTH * WIDTH, P_W4 = P_B3 + WIDTH,
                 P_B4 = P_W4 + (size_t)WIDTH * WIDTH, P_W5 = P_B4 + WIDTH, P_B5 = P_W5 + WIDTH, P_COUNT = P_B5 + 1;
__host__ __device__ constexpr size_t bias_at(int layer) {
    return layer == 0 ? P_B1 : layer == 1 ? P_B2 : layer == 2 ? P_B3 : layer == 3 ? P_B4 : P_B5;
}

// the forward weight images: W1 (1 tile of 256 x 64), W2..W4 (4 tiles each), contiguous
constexpr size_t WIMG_L1 = 0, WIMG_L2 = WIMG_L1 + 1 * 256 * 128, WIMG_L3 = WIMG_L2 + 4 * 256 * 128,
                 WIMG_L4 = WIMG_L3 + 4 * 256 * 128, WIMG_BYTES = WIMG_L4 + 4 * 256 * 128;
__host__ __device__ constexpr size_t wimg_at(int layer) {
    return layer == 0 ? WIMG_L1 : layer == 1 ? WIMG_L2 : layer == 2 ? WIMG_L3 : WIMG_L4;
}

enum Epi { EPI_PARTIAL, EPI_HIDDEN, EPI_LAST, EPI_BACK };
enum Status { ST_OK = 0, ST_INVALID = 2, ST_DEVICE = 3 };

// ---- arithmetic shared by every kernel --------------------------------------------------------

__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// silu(z) = z (1 + tanh(z / 2)) / 2 = hz + hz tanh(hz) with hz = z / 2 (one MUFU, one FMA)
__device__ __forceinline__ float silu_of_half(float hz) { return fmaf(hz, tanh_fast(hz), hz); }
__device__ __forceinline__ float silu(float z) { return silu_of_half(0.5f * z); }
__device__ __forceinline__ float silu_grad(float z) {
    const float s = 0.5f + 0.5f * tanh_fast(0.5f * z);
    return s * (1.0f + z * (1.0f - s));
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
// byte offset of element (r, k) in an A image whose row tiles hold `kt` tiles of 64 values of K
__device__ __forceinline__ size_t a_img(uint32_t r, uint32_t k, uint32_t kt) {
    return ((size_t)(r >> 7) * kt + (k >> 6)) * TILE_A + sw128_offset(r & 127u, k & 63u);
}
// byte offset of element (r, k) in a B image of `rows` rows
__device__ __forceinline__ size_t b_img(uint32_t r, uint32_t k, uint32_t rows) {
    return (size_t)(k >> 6) * rows * 128u + sw128_offset(r, k & 63u);
}

// lane j of the warp gets the sum over the warp's lanes of v[j] (v is consumed)
__device__ __forceinline__ float warp_column_sum(float (&v)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        const bool upper = (lane & off) != 0;
#pragma unroll
        for (int j = 0; j < off; j++) {
            const float send = upper ? v[j] : v[j + off];
            const float keep = upper ? v[j + off] : v[j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
    }
    return v[0];
}

__device__ __forceinline__ void flag_error(int *error, int code, volatile int *abort_flag) {
    if (error) atomicCAS(error, 0, code);
    *abort_flag = 1;
}

// ---- the product kernel --------------------------------------------------------------------------

struct GemmArgs {
    const uint8_t *a;  // A image
    const uint8_t *b;  // B image (N rows)
    uint32_t k_tiles;  // tiles of K this block multiplies (its split)
    uint32_t a_kt;     // tiles of K per row tile of the whole A image
    // EPI_PARTIAL: partial[(split * M + m) * N + n]
    float *partial;
    uint32_t m_rows;   // M
    // hidden layers
    const float *bias;
    uint8_t *h_img;    // next A image (K = 256)
    uint8_t *ht_img;   // H^T as a B image of 256 rows, K = batch
    __nv_bfloat16 *z;  // [batch][256]
    // backward
    const __nv_bfloat16 *zprev;  // [batch][256]
    uint8_t *dz_img;   // dZ as an A image (K = 256)
    uint8_t *dzt_img;  // dZ^T as an A image of 256 rows (K = batch)
    float *db_partial;      // [block][256]
    // layer 4
    const float *w5, *b5, *y;
    float inv_batch;
    float *dw5_partial;     // [block][256]
    float *scalar_partial;  // [block][2]: sum dout, sum (out - y)^2
    uint32_t batch;
    int *error;
};

template <int N>
struct GemmShape {
    static constexpr uint32_t A_BYTES = TILE_A, B_BYTES = N * 128u, STAGE = A_BYTES + B_BYTES;
    static constexpr int STAGES = N == 256 ? 4 : 6;
    static constexpr uint32_t SMEM = STAGES * STAGE + 1024;  // + alignment of the first tile
};

// column sums of the block's 128 rows for the 32 columns of chunk c: warp sums into `part`
__device__ __forceinline__ void column_chunk(float (&v)[32], float (*part)[WIDTH], int c) {
    const float s = warp_column_sum(v);
    part[threadIdx.x >> 5][32 * c + (threadIdx.x & 31)] = s;
}

template <int N, int EPI>
__global__ void __launch_bounds__(128, 1) gemm_kernel(GemmArgs g) {
    using S = GemmShape<N>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full[S::STAGES], empty[S::STAGES], done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    __shared__ float part_a[4][WIDTH], part_b[4][WIDTH];
    __shared__ float scal[4][2];
    const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
    uint8_t *smem = smem_raw + pad;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t mt = blockIdx.x, split = blockIdx.y;
    constexpr uint32_t COLS = N < 32 ? 32 : N;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S::STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(&tmem_base, COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const uint8_t *a_base = g.a + ((size_t)mt * g.a_kt + (size_t)split * g.k_tiles) * S::A_BYTES;
    const uint8_t *b_base = g.b + (size_t)split * g.k_tiles * S::B_BYTES;

    if (warp == 0 && lane == 0) {
        // producer: the tiles of A and B into the stage ring
        uint32_t issued = 0;
        for (uint32_t i = 0; i < g.k_tiles && !abort_flag; i++) {
            const int s = i % S::STAGES;
            if (i >= (uint32_t)S::STAGES && !mbar_wait(&empty[s], ((i / S::STAGES) - 1) & 1, WAIT_CYCLES)) {
                flag_error(g.error, 101, &abort_flag);
                break;
            }
            uint8_t *st = smem + (size_t)s * S::STAGE;
            mbar_expect_tx(&full[s], S::STAGE);
            bulk_load(st, a_base + (size_t)i * S::A_BYTES, S::A_BYTES, &full[s]);
            bulk_load(st + S::A_BYTES, b_base + (size_t)i * S::B_BYTES, S::B_BYTES, &full[s]);
            issued = i + 1;
        }
        // the copies still in flight end before the block does
        for (uint32_t i = issued > (uint32_t)S::STAGES ? issued - S::STAGES : 0; i < issued; i++)
            if (!mbar_wait(&full[i % S::STAGES], (i / S::STAGES) & 1, WAIT_CYCLES)) flag_error(g.error, 102, &abort_flag);
    } else if (warp == 1 && lane == 0) {
        // the MMA issuer: 4 steps of K = 16 per tile
        constexpr uint32_t idesc = idesc_bf16(128, N);
        for (uint32_t i = 0; i < g.k_tiles && !abort_flag; i++) {
            const int s = i % S::STAGES;
            if (!mbar_wait(&full[s], (i / S::STAGES) & 1, WAIT_CYCLES)) {
                flag_error(g.error, 103, &abort_flag);
                break;
            }
            tc_fence_after();
            const uint32_t a_addr = smem_u32(smem + (size_t)s * S::STAGE), b_addr = a_addr + S::A_BYTES;
#pragma unroll
            for (uint32_t k = 0; k < 4; k++)
                mma_bf16(tmem, sw128_desc(a_addr + 32 * k), sw128_desc(b_addr + 32 * k), idesc, (i | k) != 0);
            mma_commit(&empty[s]);
        }
        mma_commit(&done);
    }
    __syncwarp();
    // warp-uniform from here on: the tensor-memory loads below are .sync.aligned
    bool ready = mbar_wait(&done, 0, WAIT_CYCLES);
    tc_fence_after();
    if (!ready) flag_error(g.error, 104, &abort_flag);
    ready = __all_sync(0xffffffffu, ready && !abort_flag);

    const uint32_t r = 32 * warp + lane;  // this thread's row of the tile (its tensor-memory lane)
    const uint32_t m = mt * 128 + r;
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
    if (ready) {
        float v[32];
        if (EPI == EPI_PARTIAL) {
            float *dst = g.partial + ((size_t)split * g.m_rows + m) * N;
            for (int c = 0; c < N / 32; c++) {
                tmem_load32(lane_addr + 32 * c, v);
                float4 *d4 = reinterpret_cast<float4 *>(dst + 32 * c);
#pragma unroll
                for (int q = 0; q < 8; q++) d4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
        } else if (EPI == EPI_HIDDEN) {
            for (int c = 0; c < WIDTH / 32; c++) {
                tmem_load32(lane_addr + 32 * c, v);
                uint32_t ph[16], pz[16];
#pragma unroll
                for (int j = 0; j < 32; j += 2) {
                    const float z0 = v[j] + g.bias[32 * c + j], z1 = v[j + 1] + g.bias[32 * c + j + 1];
                    pz[j / 2] = pack_bf16(z0, z1);
                    ph[j / 2] = pack_bf16(silu(z0), silu(z1));
                }
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    *reinterpret_cast<uint4 *>(g.h_img + a_img(m, 32 * c + 8 * q, 4)) =
                        make_uint4(ph[4 * q], ph[4 * q + 1], ph[4 * q + 2], ph[4 * q + 3]);
                    reinterpret_cast<uint4 *>(g.z + (size_t)m * WIDTH + 32 * c)[q] =
                        make_uint4(pz[4 * q], pz[4 * q + 1], pz[4 * q + 2], pz[4 * q + 3]);
                }
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    const uint32_t w = ph[j / 2];
                    const uint16_t bits = (uint16_t)(j & 1 ? w >> 16 : w & 0xffff);
                    *reinterpret_cast<uint16_t *>(g.ht_img + b_img(32 * c + j, m, WIDTH)) = bits;
                }
            }
        } else {
            // EPI_LAST and EPI_BACK: dZ, its transpose and the column sums
            float dout = 0.0f, err = 0.0f;
            if (EPI == EPI_LAST) {
                float out = 0.0f;
                for (int c = 0; c < WIDTH / 32; c++) {
                    tmem_load32(lane_addr + 32 * c, v);
#pragma unroll
                    for (int j = 0; j < 32; j++) out += bf16_round(silu(v[j] + g.bias[32 * c + j])) * g.w5[32 * c + j];
                }
                out += g.b5[0];
                err = out - g.y[m];
                dout = 2.0f * err * g.inv_batch;
            }
            const uint32_t batch_kt = g.batch / 64;
            for (int c = 0; c < WIDTH / 32; c++) {
                tmem_load32(lane_addr + 32 * c, v);
                float dz[32], hw[32];
                if (EPI == EPI_LAST) {
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        const int n = 32 * c + j;
                        const float z = v[j] + g.bias[n];
                        hw[j] = dout * bf16_round(silu(z));
                        dz[j] = dout * g.w5[n] * silu_grad(z);
                    }
                } else {
                    const uint4 *zp = reinterpret_cast<const uint4 *>(g.zprev + (size_t)m * WIDTH + 32 * c);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const uint4 w = zp[q];
                        const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            const float lo = __uint_as_float(ws[e] << 16), hi = __uint_as_float(ws[e] & 0xffff0000u);
                            dz[8 * q + 2 * e] = v[8 * q + 2 * e] * silu_grad(lo);
                            dz[8 * q + 2 * e + 1] = v[8 * q + 2 * e + 1] * silu_grad(hi);
                        }
                    }
                }
                uint32_t pd[16];
#pragma unroll
                for (int j = 0; j < 32; j += 2) pd[j / 2] = pack_bf16(dz[j], dz[j + 1]);
#pragma unroll
                for (int q = 0; q < 4; q++)
                    *reinterpret_cast<uint4 *>(g.dz_img + a_img(m, 32 * c + 8 * q, 4)) =
                        make_uint4(pd[4 * q], pd[4 * q + 1], pd[4 * q + 2], pd[4 * q + 3]);
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    const uint32_t w = pd[j / 2];
                    const uint16_t bits = (uint16_t)(j & 1 ? w >> 16 : w & 0xffff);
                    *reinterpret_cast<uint16_t *>(g.dzt_img + a_img(32 * c + j, m, batch_kt)) = bits;
                }
                column_chunk(dz, part_a, c);
                if (EPI == EPI_LAST) column_chunk(hw, part_b, c);
            }
            if (EPI == EPI_LAST) {
                float a = dout, b = err * err;
#pragma unroll
                for (int off = 16; off >= 1; off >>= 1) {
                    a += __shfl_xor_sync(0xffffffffu, a, off);
                    b += __shfl_xor_sync(0xffffffffu, b, off);
                }
                if (lane == 0) {
                    scal[warp][0] = a;
                    scal[warp][1] = b;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if ((EPI == EPI_LAST || EPI == EPI_BACK) && !abort_flag) {
        for (int n = threadIdx.x; n < WIDTH; n += 128) {
            g.db_partial[(size_t)blockIdx.x * WIDTH + n] = part_a[0][n] + part_a[1][n] + part_a[2][n] + part_a[3][n];
            if (EPI == EPI_LAST)
                g.dw5_partial[(size_t)blockIdx.x * WIDTH + n] = part_b[0][n] + part_b[1][n] + part_b[2][n] + part_b[3][n];
        }
        if (EPI == EPI_LAST && threadIdx.x < 2)
            g.scalar_partial[2 * blockIdx.x + threadIdx.x] =
                scal[0][threadIdx.x] + scal[1][threadIdx.x] + scal[2][threadIdx.x] + scal[3][threadIdx.x];
    }
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, COLS);
}

// ---- inputs into images ------------------------------------------------------------------------

// x [batch][inputs] FP32 -> X as an A image (K = 64, zero padded) and X^T as a B image of 64 rows
// (K = batch); one thread per (point, 8 features)
__global__ void inputs_kernel(const float *x, uint32_t inputs, uint32_t batch, uint8_t *x_img, uint8_t *xt_img) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= batch * (IN / 8)) return;
    const uint32_t m = t / (IN / 8), k0 = 8 * (t % (IN / 8));
    uint32_t p[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const uint32_t k = k0 + 2 * e;
        const float lo = k < inputs ? x[(size_t)m * inputs + k] : 0.0f;
        const float hi = k + 1 < inputs ? x[(size_t)m * inputs + k + 1] : 0.0f;
        p[e] = pack_bf16(lo, hi);
    }
    *reinterpret_cast<uint4 *>(x_img + a_img(m, k0, 1)) = make_uint4(p[0], p[1], p[2], p[3]);
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const uint16_t bits = (uint16_t)(j & 1 ? p[j / 2] >> 16 : p[j / 2] & 0xffff);
        *reinterpret_cast<uint16_t *>(xt_img + b_img(k0 + j, m, IN)) = bits;
    }
}

// ---- parameters into weight images -----------------------------------------------------------

// one thread per weight of W1..W4: its BF16 value into the forward image (rows = outputs, K =
// inputs) and, for W2..W4, the transposed image (rows = inputs, K = outputs) the backward reads
__global__ void images_kernel(const float *params, uint8_t *wimg, uint8_t *wtimg) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t first = WIDTH * IN, per = WIDTH * WIDTH;
    if (t >= first + 3 * per) return;
    uint32_t layer, o, i;
    float w;
    if (t < first) {
        layer = 0;
        o = t / IN;
        i = t % IN;
        w = params[P_W1 + t];
    } else {
        const uint32_t u = t - first;
        layer = 1 + u / per;
        o = (u % per) / WIDTH;
        i = u % WIDTH;
        w = params[(layer == 1 ? P_W2 : layer == 2 ? P_W3 : P_W4) + (u % per)];
    }
    const __nv_bfloat16 b = __float2bfloat16_rn(w);
    const size_t at = wimg_at((int)layer);
    *reinterpret_cast<__nv_bfloat16 *>(wimg + at + b_img(o, i, WIDTH)) = b;
    if (layer > 0)
        *reinterpret_cast<__nv_bfloat16 *>(wtimg + (size_t)(layer - 1) * 4 * 256 * 128 + b_img(i, o, WIDTH)) = b;
}

// ---- gradients and Adam ----------------------------------------------------------------------------

struct GradArgs {
    const float *dw[4];   // partials [splits][256][fan_in]
    uint32_t splits;
    const float *db[4];   // [blocks][256]
    uint32_t blocks;
    const float *dw5;     // [blocks][256]
    const float *scalars; // [blocks][2]
    float *grad;          // param order
    float *loss;          // one float (set), or null
    float *loss_sum;      // one float (added), or null
};

// one thread per parameter: the sum of its partials (in a fixed order: the result does not depend
// on the launch)
__global__ void grad_kernel(GradArgs a) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P_COUNT) return;
    float s = 0.0f;
    if (t < P_B1) {
        for (uint32_t k = 0; k < a.splits; k++) s += a.dw[0][(size_t)k * WIDTH * IN + t];
    } else if (t >= P_W2 && t < P_B4 && (t - P_W2) % (WIDTH * WIDTH + WIDTH) < WIDTH * WIDTH) {
        const uint32_t l = (uint32_t)((t - P_W2) / (WIDTH * WIDTH + WIDTH)), e = (uint32_t)((t - P_W2) % (WIDTH * WIDTH + WIDTH));
        for (uint32_t k = 0; k < a.splits; k++) s += a.dw[l + 1][(size_t)k * WIDTH * WIDTH + e];
    } else if (t < P_W5) {
        // a bias of layers 1..4 (they follow their layer's weights)
        const uint32_t layer = t < P_W2 ? 0 : t < P_W3 ? 1 : t < P_W4 ? 2 : 3;
        const uint32_t n = (uint32_t)(t - (layer == 0 ? P_B1 : layer == 1 ? P_B2 : layer == 2 ? P_B3 : P_B4));
        for (uint32_t k = 0; k < a.blocks; k++) s += a.db[layer][(size_t)k * WIDTH + n];
    } else if (t < P_B5) {
        for (uint32_t k = 0; k < a.blocks; k++) s += a.dw5[(size_t)k * WIDTH + (t - P_W5)];
    } else {
        float l = 0.0f;
        for (uint32_t k = 0; k < a.blocks; k++) {
            s += a.scalars[2 * k];
            l += a.scalars[2 * k + 1];
        }
        if (a.loss) *a.loss = l;
        if (a.loss_sum) *a.loss_sum += l;
    }
    a.grad[t] = s;
}

__global__ void adam_kernel(float *params, float *m1, float *m2, const float *grad, float lr, float c1, float c2,
                            uint32_t inputs) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P_COUNT) return;
    if (t < P_B1 && (t % IN) >= inputs) return;  // the padding columns of W1 stay zero
    const float g = grad[t];
    const float a = 0.9f * m1[t] + 0.1f * g, b = 0.999f * m2[t] + 0.001f * g * g;
    m1[t] = a;
    m2[t] = b;
    params[t] -= lr * (a * c1) / (sqrtf(b * c2) + 1e-8f);
}

// ---- fused inference ------------------------------------------------------------------------------
//
// One block per 128 points at a time (persistent, two blocks per SM so that one block's products
// run while the other's epilogue does): warps 0-7 build the inputs and run the epilogues (thread
// (w, lane) owns point r = 32 (w % 4) + lane, tensor-memory lane r, and the column half w / 4),
// warp 8 streams the weight images through a ring of two 16 KB stages (tiles of 128 rows x 64
// values: chunk (k tile, half) of each layer), warp 9 issues the products (M = 128, N = 128 per
// half) into 256 FP32 columns of tensor memory. The activations stay in one 64 KB A tile set,
// overwritten in place by each epilogue once the layer's products have completed. The biases and
// the output layer's weights sit in shared memory.

constexpr int FWD_EPI_THREADS = 256;
constexpr int FWD_THREADS = FWD_EPI_THREADS + 64;
constexpr uint32_t FWD_CHUNK = 128 * 128;  // 16 KB
// the weight ring's stages for one or two blocks per SM (the shared memory left beside the 64 KB of
// activations), and the dynamic shared memory of a block
template <int CTAS> struct FwdShape {
    static constexpr int STAGES = CTAS == 1 ? 9 : 2;
    static constexpr uint32_t SMEM = 4 * TILE_A + STAGES * FWD_CHUNK + 1024;
};
constexpr int FWD_CHUNKS = 2 + 3 * 8;  // per tile: layer 1 (1 k tile x 2 halves), layers 2-4 (4 x 2)
constexpr int FWD_PARAMS = 5 * WIDTH + 1;  // b1..b4, w5, b5

struct ForwardArgs {
    const uint8_t *wimg;
    const float *params;
    const float *x;
    uint32_t inputs, count, tiles;
    float *out;
    int *error;
    // candidates (stage 1 of two-stage unweighting): segments of candidates, one per subprocess;
    // tile t belongs to the segment whose tiles [tile_first, next tile_first) hold it
    pacuda_uw_segment seg[PACUDA_UW_MAX_SEGMENTS];
    uint32_t tile_first[PACUDA_UW_MAX_SEGMENTS + 1];
    uint32_t segments;
    double mu, sigma;  // s = exp(mu + sigma out); kept when (first decision uniform) s_max < s
    uint32_t capacity;
    uint32_t numbers;  // the candidates' phase-space numbers: 5 (2 -> 3) or 8 (2 -> 4)
};

// the segment of tile t (segments are few: a linear scan)
__device__ __forceinline__ uint32_t segment_of(const ForwardArgs &g, uint32_t t) {
    uint32_t k = 0;
    while (k + 1 < g.segments && t >= g.tile_first[k + 1]) k++;
    return k;
}

enum { FWD_FROM_X = 0, FWD_CANDIDATES = 1 };

// chunk c of a tile's stream: its layer, k tile and half
__device__ __forceinline__ void fwd_chunk(int c, int &layer, int &kt, int &half) {
    if (c < 2) {
        layer = 0;
        kt = 0;
        half = c;
    } else {
        layer = 1 + (c - 2) / 8;
        kt = ((c - 2) % 8) / 2;
        half = (c - 2) % 2;
    }
}

template <int MODE, int CTAS>
__global__ void __launch_bounds__(FWD_THREADS, CTAS) forward_kernel(ForwardArgs g) {
    constexpr int FWD_STAGES = FwdShape<CTAS>::STAGES;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full[FWD_STAGES], empty[FWD_STAGES], act_ready, acc_ready, dot_ready;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    __shared__ __align__(16) float prm[FWD_PARAMS];
    __shared__ float dot_hi[128];
    const uint32_t pad = (1024u - (smem_u32(smem_raw) & 1023u)) & 1023u;
    uint8_t *act = smem_raw + pad;         // 4 A tiles: the activations (K = 256)
    uint8_t *ring = act + 4 * TILE_A;      // weight chunks
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t my_tiles = blockIdx.x < g.tiles ? (g.tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < FWD_STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&act_ready, FWD_EPI_THREADS);
        mbar_init(&acc_ready, 1);
        mbar_init(&dot_ready, FWD_EPI_THREADS / 2);
        abort_flag = 0;
        fence_mbar_init();
    }
    // b1..b4 halved (the epilogue computes z / 2 = acc / 2 + b / 2 in one FMA), then w5 and b5
    // (P_W5, P_B5 follow each other)
    for (int i = threadIdx.x; i < FWD_PARAMS; i += FWD_THREADS)
        prm[i] = i < 4 * WIDTH ? 0.5f * g.params[bias_at(i / WIDTH) + i % WIDTH] : g.params[P_W5 + (i - 4 * WIDTH)];
    if (warp == 0) tmem_alloc(&tmem_base, 256);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    if (warp == 8) {
        if (lane == 0) {
            const uint32_t total = my_tiles * FWD_CHUNKS;
            uint32_t issued = 0;
            for (uint32_t i = 0; i < total && !abort_flag; i++) {
                const int s = i % FWD_STAGES;
                if (i >= (uint32_t)FWD_STAGES && !mbar_wait(&empty[s], ((i / FWD_STAGES) - 1) & 1, WAIT_CYCLES)) {
                    flag_error(g.error, 201, &abort_flag);
                    break;
                }
                int layer, kt, half;
                fwd_chunk(i % FWD_CHUNKS, layer, kt, half);
                const size_t at = wimg_at(layer) + (size_t)kt * 256 * 128 + (size_t)half * FWD_CHUNK;
                mbar_expect_tx(&full[s], FWD_CHUNK);
                bulk_load(ring + (size_t)s * FWD_CHUNK, g.wimg + at, FWD_CHUNK, &full[s]);
                issued = i + 1;
            }
            for (uint32_t i = issued > (uint32_t)FWD_STAGES ? issued - FWD_STAGES : 0; i < issued; i++)
                if (!mbar_wait(&full[i % FWD_STAGES], (i / FWD_STAGES) & 1, WAIT_CYCLES))
                    flag_error(g.error, 202, &abort_flag);
        }
    } else if (warp == 9) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(128, 128);
            uint32_t chunk = 0, acts = 0;
            const uint32_t act_addr = smem_u32(act), ring_addr = smem_u32(ring);
            for (uint32_t t = 0; t < my_tiles && !abort_flag; t++) {
                for (int layer = 0; layer < 4 && !abort_flag; layer++) {
                    if (!mbar_wait(&act_ready, acts & 1, WAIT_CYCLES)) {
                        flag_error(g.error, 203, &abort_flag);
                        break;
                    }
                    acts++;
                    tc_fence_after();
                    const int n_chunks = layer == 0 ? 2 : 8;
                    for (int c = 0; c < n_chunks; c++, chunk++) {
                        const int s = chunk % FWD_STAGES;
                        if (!mbar_wait(&full[s], (chunk / FWD_STAGES) & 1, WAIT_CYCLES)) {
                            flag_error(g.error, 204, &abort_flag);
                            break;
                        }
                        tc_fence_after();
                        const int kt = layer == 0 ? 0 : c / 2, half = layer == 0 ? c : c % 2;
                        const uint32_t a_addr = act_addr + kt * TILE_A, b_addr = ring_addr + s * FWD_CHUNK;
#pragma unroll
                        for (uint32_t k = 0; k < 4; k++)
                            mma_bf16(tmem + 128 * half, sw128_desc(a_addr + 32 * k), sw128_desc(b_addr + 32 * k), idesc,
                                     (kt | k) != 0);
                        mma_commit(&empty[s]);
                    }
                    mma_commit(&acc_ready);
                }
            }
        }
    } else {
        // warps 0-7: inputs, epilogues, outputs; this thread: row r, columns [128 h, 128 h + 128)
        const uint32_t r = 32 * (warp & 3) + lane, h = warp >> 2;
        const uint32_t lane_addr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
        uint32_t accs = 0, dots = 0;
        for (uint32_t t = 0; t < my_tiles && !__any_sync(0xffffffffu, abort_flag != 0); t++) {
            const uint32_t tile = blockIdx.x + t * gridDim.x;
            // candidates: the tile's segment and the point's place in it
            const uint32_t sg = MODE == FWD_CANDIDATES ? segment_of(g, tile) : 0;
            const uint32_t m = MODE == FWD_CANDIDATES ? (tile - g.tile_first[sg]) * 128 + r : tile * 128 + r;
            const uint32_t m_count = MODE == FWD_CANDIDATES ? g.seg[sg].count : g.count;
            // the inputs: features [32 h, 32 h + 32) of row r of A tile 0 (K = 64)
            uint32_t p[16];
            double u_keep = 1.0;
            uint64_t cand = 0;
            if (MODE == FWD_FROM_X) {
#pragma unroll
                for (int e = 0; e < 16; e++) {
                    const uint32_t k = 32 * h + 2 * e;
                    const float lo = (m < g.count && k < g.inputs) ? g.x[(size_t)m * g.inputs + k] : 0.0f;
                    const float hi = (m < g.count && k + 1 < g.inputs) ? g.x[(size_t)m * g.inputs + k + 1] : 0.0f;
                    p[e] = pack_bf16(lo, hi);
                }
            } else {
                // the candidate's phase-space numbers and the subprocess one-hot (the listed candidates
                // are inside the cuts)
                constexpr int MAXU = pacuda::phase::MAX_UNIFORMS;
                double u[MAXU];
#pragma unroll
                for (int k = 0; k < MAXU; k++) u[k] = 0.0;
                const uint32_t nx = g.numbers;
                if (m < m_count) {
                    cand = g.seg[sg].index[m];
                    if (nx == 8) {
                        pacuda::phase::uniforms(g.seg[sg].seed, cand, u);
                    } else {
                        double v[pacuda::phase::Space<3>::UNIFORMS];
                        pacuda::phase::uniforms(g.seg[sg].seed, cand, v);
#pragma unroll
                        for (int k = 0; k < pacuda::phase::Space<3>::UNIFORMS; k++) u[k] = v[k];
                    }
                }
                u_keep = nx == 8 ? u[8] : u[5];
                const bool real = m < m_count;
                const uint32_t family = g.seg[sg].family;
                float f[32];  // this half's 32 features (constant indices only)
#pragma unroll
                for (int k = 0; k < 32; k++) f[k] = 0.0f;
                if (h == 0 && real) {
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        if ((uint32_t)k < nx) f[k] = (float)u[k];
                }
#pragma unroll
                for (int k = 0; k < 32; k++)
                    if (real && 32 * h + k == nx + family) f[k] = 1.0f;
#pragma unroll
                for (int e = 0; e < 16; e++) p[e] = pack_bf16(f[2 * e], f[2 * e + 1]);
            }
#pragma unroll
            for (int q = 0; q < 4; q++)
                *reinterpret_cast<uint4 *>(act + sw128_offset(r, 32 * h + 8 * q)) =
                    make_uint4(p[4 * q], p[4 * q + 1], p[4 * q + 2], p[4 * q + 3]);
            fence_async_shared();
            tc_fence_before();
            mbar_arrive(&act_ready);
            float out = 0.0f;
            bool done = true;
            for (int layer = 0; layer < 4; layer++) {
                const bool got = __all_sync(0xffffffffu, mbar_wait(&acc_ready, accs & 1, WAIT_CYCLES));
                if (!got) {
                    flag_error(g.error, 205, &abort_flag);
                    done = false;
                    break;
                }
                accs++;
                tc_fence_after();
                const float *bias = prm + layer * WIDTH;  // halved biases (the epilogue works on z / 2)
                // this half's 128 columns in eight pieces of 16, each piece's tensor-memory load
                // issued before the previous piece is computed (its latency hidden behind the math)
                uint32_t buf[2][16];
                tmem_load16_async(lane_addr + 128 * h, buf[0]);
#pragma unroll
                for (int piece = 0; piece < 8; piece++) {
                    uint32_t(&cur)[16] = buf[piece & 1];
                    tmem_wait16(cur);
                    if (piece + 1 < 8) tmem_load16_async(lane_addr + 128 * h + 16 * (piece + 1), buf[(piece + 1) & 1]);
                    const int col = 128 * h + 16 * piece;
                    const float4 *b4 = reinterpret_cast<const float4 *>(bias + col);
                    float bb[16];
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float4 t4 = b4[q];
                        bb[4 * q] = t4.x;
                        bb[4 * q + 1] = t4.y;
                        bb[4 * q + 2] = t4.z;
                        bb[4 * q + 3] = t4.w;
                    }
                    if (layer < 3) {
                        uint32_t ph[8];
#pragma unroll
                        for (int j = 0; j < 16; j += 2)
                            ph[j / 2] = pack_bf16(silu_of_half(fmaf(__uint_as_float(cur[j]), 0.5f, bb[j])),
                                                  silu_of_half(fmaf(__uint_as_float(cur[j + 1]), 0.5f, bb[j + 1])));
#pragma unroll
                        for (int q = 0; q < 2; q++)
                            *reinterpret_cast<uint4 *>(act + (col / 64) * TILE_A + sw128_offset(r, col % 64 + 8 * q)) =
                                make_uint4(ph[4 * q], ph[4 * q + 1], ph[4 * q + 2], ph[4 * q + 3]);
                    } else {
                        const float *w5 = prm + 4 * WIDTH + col;
#pragma unroll
                        for (int j = 0; j < 16; j++)
                            out = fmaf(bf16_round(silu_of_half(fmaf(__uint_as_float(cur[j]), 0.5f, bb[j]))), w5[j], out);
                    }
                }
                if (layer < 3) {
                    fence_async_shared();
                    tc_fence_before();
                    mbar_arrive(&act_ready);
                }
            }
            // the two column halves' dot products meet in shared memory: the upper half's threads
            // write theirs and arrive; the lower half's wait (bounded) and finish the point. The
            // next write of dot_hi comes after this tile's reads: it needs the next tile's inputs,
            // which the lower half writes after them.
            if (h == 1) {
                dot_hi[r] = out;
                mbar_arrive(&dot_ready);
                continue;
            }
            const bool have = __all_sync(0xffffffffu, mbar_wait(&dot_ready, dots & 1, WAIT_CYCLES));
            dots++;
            if (!have) {
                flag_error(g.error, 206, &abort_flag);
                continue;
            }
            if (!done) continue;
            out += dot_hi[r] + prm[5 * WIDTH];
            if (MODE == FWD_FROM_X) {
                if (m < g.count) g.out[m] = out;
            } else {
                // stage 1: s = exp(mu + sigma out), the network's estimate of the weight w = |M|^2 J;
                // kept when u5 s_max < s (warp-aggregated appends)
                const pacuda_uw_segment &sgm = g.seg[sg];
                const bool real = m < m_count;
                const double sv = real ? exp(g.mu + g.sigma * (double)out) : 0.0;
                const bool keep = real && u_keep * sgm.s_max < sv;
                const unsigned ballot = __ballot_sync(0xffffffffu, keep);
                unsigned long long base = 0;
                if (lane == 0 && ballot) base = atomicAdd(sgm.kept_count, (unsigned long long)__popc(ballot));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (keep) {
                    const unsigned long long slot = base + __popc(ballot & ((1u << lane) - 1u));
                    if (slot < g.capacity) {
                        sgm.kept_index[slot] = cand;
                        sgm.kept_s[slot] = sv;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, 256);
}

// ---- host ---------------------------------------------------------------------------------------

const char *kTag = "pacuda surrogate";
thread_local uint32_t g_last_launches = 0;

bool failed(cudaError_t e, const char *step) {
    if (e == cudaSuccess) return false;
    fprintf(stderr, "%s: %s: %s\n", kTag, step, cudaGetErrorString(e));
    return true;
}

template <int N, int EPI>
bool launch_gemm(const GemmArgs &g, uint32_t m_tiles, uint32_t splits, cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        if (failed(cudaFuncSetAttribute(gemm_kernel<N, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        GemmShape<N>::SMEM),
                   "product kernel attributes"))
            return false;
        configured = true;
    }
    gemm_kernel<N, EPI><<<dim3(m_tiles, splits), 128, GemmShape<N>::SMEM, s>>>(g);
    g_last_launches++;
    return !failed(cudaGetLastError(), "product kernel launch");
}

// blocks per SM of the inference kernel: 2 (two blocks, a 2-stage weight ring each) or 1 (one
// block, a 9-stage ring)
int g_forward_blocks = 2;

template <int MODE, int CTAS>
bool launch_forward_shape(const ForwardArgs &g, cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        if (failed(cudaFuncSetAttribute(forward_kernel<MODE, CTAS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        FwdShape<CTAS>::SMEM),
                   "inference kernel attributes"))
            return false;
        configured = true;
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t grid = std::min<uint32_t>(g.tiles, (uint32_t)CTAS * (uint32_t)sms);
    forward_kernel<MODE, CTAS><<<grid, FWD_THREADS, FwdShape<CTAS>::SMEM, s>>>(g);
    g_last_launches++;
    return !failed(cudaGetLastError(), "inference launch");
}

template <int MODE>
bool launch_forward(const ForwardArgs &g, cudaStream_t s) {
    return g_forward_blocks == 1 ? launch_forward_shape<MODE, 1>(g, s) : launch_forward_shape<MODE, 2>(g, s);
}

}  // namespace

struct pacuda_sg_net {
    uint32_t inputs = 0, max_batch = 0;
    uint64_t step = 0;
    float *params = nullptr, *m1 = nullptr, *m2 = nullptr, *grad = nullptr, *loss = nullptr;
    uint8_t *wimg = nullptr, *wtimg = nullptr;
    // workspace for a batch
    uint8_t *x_img = nullptr, *xt_img = nullptr, *h_img[3] = {}, *ht_img[3] = {}, *dz_img[2] = {}, *dzt_img = nullptr;
    __nv_bfloat16 *z[3] = {};
    float *dw_part[4] = {}, *db_part[4] = {}, *dw5_part = nullptr, *scal_part = nullptr;
    int *error = nullptr;
    std::vector<void *> owned;
};

namespace {

template <class T>
bool dalloc(pacuda_sg_net *n, T **p, size_t bytes) {
    void *q = nullptr;
    if (failed(cudaMalloc(&q, bytes ? bytes : 16), "allocation")) return false;
    n->owned.push_back(q);
    *p = (T *)q;
    return true;
}

// splits of the batch for the weight gradients: 4 tiles of K (256 points) per block when they divide
uint32_t split_tiles(uint32_t batch) { return (batch / 64) % 4 == 0 ? 4 : 2; }

int refresh_images(pacuda_sg_net *n, cudaStream_t s) {
    const uint32_t count = WIDTH * IN + 3 * WIDTH * WIDTH;
    images_kernel<<<(count + 255) / 256, 256, 0, s>>>(n->params, n->wimg, n->wtimg);
    g_last_launches++;
    return failed(cudaGetLastError(), "weight images") ? ST_DEVICE : ST_OK;
}

}  // namespace

// ---- the C ABI -------------------------------------------------------------------------------------

extern "C" size_t pacuda_sg_param_count(void) { return P_COUNT; }

extern "C" uint32_t pacuda_sg_last_launches(void) { return g_last_launches; }

extern "C" int pacuda_sg_set_inference_blocks(uint32_t blocks) {
    if (blocks != 1 && blocks != 2) return ST_INVALID;
    g_forward_blocks = (int)blocks;
    return ST_OK;
}

extern "C" void pacuda_sg_destroy(pacuda_sg_net *n) {
    if (!n) return;
    for (void *p : n->owned) cudaFree(p);
    delete n;
}

extern "C" pacuda_sg_net *pacuda_sg_create(uint32_t inputs, uint32_t max_batch, uint64_t seed) {
    if (inputs == 0 || inputs > IN || max_batch == 0 || max_batch % 128) {
        fprintf(stderr, "%s: create: %u inputs (1..%d), batches of %u points (a multiple of 128)\n", kTag, inputs, IN,
                max_batch);
        return nullptr;
    }
    pacuda_sg_net *n = new pacuda_sg_net;
    n->inputs = inputs;
    n->max_batch = max_batch;
    const size_t B = max_batch, blocks = B / 128, splits = B / 64 / 2;
    bool ok = dalloc(n, &n->params, P_COUNT * 4) && dalloc(n, &n->m1, P_COUNT * 4) && dalloc(n, &n->m2, P_COUNT * 4) &&
              dalloc(n, &n->grad, P_COUNT * 4) && dalloc(n, &n->loss, 16) && dalloc(n, &n->error, 16) &&
              dalloc(n, &n->wimg, WIMG_BYTES) && dalloc(n, &n->wtimg, 3 * 4 * 256 * 128) &&
              dalloc(n, &n->x_img, B * IN * 2) && dalloc(n, &n->xt_img, B * IN * 2) && dalloc(n, &n->dzt_img, B * WIDTH * 2) &&
              dalloc(n, &n->dw5_part, blocks * WIDTH * 4) && dalloc(n, &n->scal_part, blocks * 2 * 4);
    for (int l = 0; ok && l < 3; l++)
        ok = dalloc(n, &n->h_img[l], B * WIDTH * 2) && dalloc(n, &n->ht_img[l], B * WIDTH * 2) &&
             dalloc(n, &n->z[l], B * WIDTH * 2);
    for (int l = 0; ok && l < 2; l++) ok = dalloc(n, &n->dz_img[l], B * WIDTH * 2);
    for (int l = 0; ok && l < 4; l++)
        ok = dalloc(n, &n->dw_part[l], splits * WIDTH * (l == 0 ? IN : WIDTH) * 4) && dalloc(n, &n->db_part[l], blocks * WIDTH * 4);
    if (!ok) {
        pacuda_sg_destroy(n);
        return nullptr;
    }
    // weights uniform in +-sqrt(6 / fan_in) from a splitmix64 stream, biases zero
    std::vector<float> p(P_COUNT, 0.0f);
    uint64_t state = seed;
    auto next = [&]() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return ((z >> 11) + 0.5) / 9007199254740992.0;
    };
    for (int l = 0; l < 5; l++) {
        const size_t at = l == 0 ? P_W1 : l == 1 ? P_W2 : l == 2 ? P_W3 : l == 3 ? P_W4 : P_W5;
        const uint32_t rows = l == 4 ? 1 : WIDTH, fan = l == 0 ? inputs : WIDTH, cols = l == 0 ? IN : WIDTH;
        const double a = std::sqrt(6.0 / fan);
        for (uint32_t o = 0; o < rows; o++)
            for (uint32_t i = 0; i < fan; i++) p[at + (size_t)o * cols + i] = (float)((2.0 * next() - 1.0) * a);
    }
    if (pacuda_sg_set_params(n, p.data()) != ST_OK) {
        pacuda_sg_destroy(n);
        return nullptr;
    }
    return n;
}

extern "C" int pacuda_sg_set_params(pacuda_sg_net *n, const float *params) {
    g_last_launches = 0;
    if (!n || !params) return ST_INVALID;
    std::vector<float> p(params, params + P_COUNT);
    for (uint32_t o = 0; o < WIDTH; o++)
        for (uint32_t i = n->inputs; i < IN; i++) p[P_W1 + (size_t)o * IN + i] = 0.0f;
    if (failed(cudaMemcpy(n->params, p.data(), P_COUNT * 4, cudaMemcpyHostToDevice), "parameters") ||
        failed(cudaMemset(n->m1, 0, P_COUNT * 4), "moments") || failed(cudaMemset(n->m2, 0, P_COUNT * 4), "moments") ||
        failed(cudaMemset(n->error, 0, 16), "error flag") || failed(cudaMemset(n->wimg, 0, WIMG_BYTES), "images"))
        return ST_DEVICE;
    n->step = 0;
    if (refresh_images(n, 0) != ST_OK || failed(cudaDeviceSynchronize(), "images")) return ST_DEVICE;
    return ST_OK;
}

extern "C" int pacuda_sg_get_params(const pacuda_sg_net *n, float *params) {
    if (!n || !params) return ST_INVALID;
    return failed(cudaMemcpy(params, n->params, P_COUNT * 4, cudaMemcpyDeviceToHost), "parameters") ? ST_DEVICE : ST_OK;
}

namespace {

// the forward and backward products of one batch and the reduction of their partials into the
// gradient (param order) and the loss
int gradients(pacuda_sg_net *n, const float *x, const float *y, uint32_t batch, float *grad, float *loss,
              float *loss_sum, cudaStream_t s) {
    if (!n || !x || !y || !grad || batch == 0 || batch % 128 || batch > n->max_batch) {
        fprintf(stderr, "%s: a batch of %u points (a multiple of 128, at most %u)\n", kTag, batch, n ? n->max_batch : 0);
        return ST_INVALID;
    }
    const uint32_t blocks = batch / 128, st = split_tiles(batch), splits = batch / 64 / st, kt = batch / 64;
    inputs_kernel<<<(batch * (IN / 8) + 255) / 256, 256, 0, s>>>(x, n->inputs, batch, n->x_img, n->xt_img);
    g_last_launches++;
    if (failed(cudaGetLastError(), "inputs")) return ST_DEVICE;
    GemmArgs g;
    memset(&g, 0, sizeof g);
    g.batch = batch;
    g.error = n->error;
    g.inv_batch = 1.0f / (float)batch;
    // forward, layers 1-3
    for (int l = 0; l < 3; l++) {
        g.a = l == 0 ? n->x_img : n->h_img[l - 1];
        g.a_kt = g.k_tiles = l == 0 ? 1 : 4;
        g.b = n->wimg + wimg_at(l);
        g.bias = n->params + bias_at(l);
        g.h_img = n->h_img[l];
        g.ht_img = n->ht_img[l];
        g.z = n->z[l];
        if (!launch_gemm<256, EPI_HIDDEN>(g, blocks, 1, s)) return ST_DEVICE;
    }
    // layer 4 and the output layer: dZ4
    g.a = n->h_img[2];
    g.a_kt = g.k_tiles = 4;
    g.b = n->wimg + wimg_at(3);
    g.bias = n->params + P_B4;
    g.w5 = n->params + P_W5;
    g.b5 = n->params + P_B5;
    g.y = y;
    g.dz_img = n->dz_img[0];
    g.dzt_img = n->dzt_img;
    g.db_partial = n->db_part[3];
    g.dw5_partial = n->dw5_part;
    g.scalar_partial = n->scal_part;
    if (!launch_gemm<256, EPI_LAST>(g, blocks, 1, s)) return ST_DEVICE;
    // backward: layer l = 4, 3, 2 (index 3, 2, 1): dW_l, then dZ_{l-1}
    int cur = 0;
    for (int l = 3; l >= 1; l--) {
        GemmArgs w;
        memset(&w, 0, sizeof w);
        w.error = n->error;
        w.a = n->dzt_img;
        w.a_kt = kt;
        w.k_tiles = st;
        w.b = n->ht_img[l - 1];
        w.partial = n->dw_part[l];
        w.m_rows = WIDTH;
        if (!launch_gemm<256, EPI_PARTIAL>(w, 2, splits, s)) return ST_DEVICE;
        GemmArgs d;
        memset(&d, 0, sizeof d);
        d.error = n->error;
        d.batch = batch;
        d.a = n->dz_img[cur];
        d.a_kt = d.k_tiles = 4;
        d.b = n->wtimg + (size_t)(l - 1) * 4 * 256 * 128;
        d.zprev = n->z[l - 1];
        d.dz_img = n->dz_img[cur ^ 1];
        d.dzt_img = n->dzt_img;
        d.db_partial = n->db_part[l - 1];
        if (!launch_gemm<256, EPI_BACK>(d, blocks, 1, s)) return ST_DEVICE;
        cur ^= 1;
    }
    // dW1 = dZ1^T X
    {
        GemmArgs w;
        memset(&w, 0, sizeof w);
        w.error = n->error;
        w.a = n->dzt_img;
        w.a_kt = kt;
        w.k_tiles = st;
        w.b = n->xt_img;
        w.partial = n->dw_part[0];
        w.m_rows = WIDTH;
        if (!launch_gemm<64, EPI_PARTIAL>(w, 2, splits, s)) return ST_DEVICE;
    }
    GradArgs a;
    for (int l = 0; l < 4; l++) {
        a.dw[l] = n->dw_part[l];
        a.db[l] = n->db_part[l];
    }
    a.splits = splits;
    a.blocks = blocks;
    a.dw5 = n->dw5_part;
    a.scalars = n->scal_part;
    a.grad = grad;
    a.loss = loss;
    a.loss_sum = loss_sum;
    grad_kernel<<<(unsigned)((P_COUNT + 255) / 256), 256, 0, s>>>(a);
    g_last_launches++;
    return failed(cudaGetLastError(), "gradient reduction") ? ST_DEVICE : ST_OK;
}

}  // namespace

extern "C" int pacuda_sg_gradients(pacuda_sg_net *n, const float *x, const float *y, uint32_t batch, float *grad,
                                   float *loss, void *stream) {
    g_last_launches = 0;
    return gradients(n, x, y, batch, grad, loss, nullptr, (cudaStream_t)stream);
}

namespace {

// one Adam step on the gradient `grad` (param order, device) and the weight images
int adam_step(pacuda_sg_net *n, const float *grad, float lr, cudaStream_t s) {
    n->step++;
    const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, (double)n->step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow(0.999, (double)n->step)));
    adam_kernel<<<(unsigned)((P_COUNT + 255) / 256), 256, 0, s>>>(n->params, n->m1, n->m2, grad, lr, c1, c2, n->inputs);
    g_last_launches++;
    if (failed(cudaGetLastError(), "adam")) return ST_DEVICE;
    return refresh_images(n, s);
}

}  // namespace

extern "C" int pacuda_sg_apply_gradients(pacuda_sg_net *n, const float *grad, float lr, void *stream) {
    g_last_launches = 0;
    if (!n || !grad) return ST_INVALID;
    return adam_step(n, grad, lr, (cudaStream_t)stream);
}

extern "C" int pacuda_sg_train_step(pacuda_sg_net *n, const float *x, const float *y, uint32_t batch, float lr,
                                    float *loss_sum, void *stream) {
    g_last_launches = 0;
    cudaStream_t s = (cudaStream_t)stream;
    int st = gradients(n, x, y, batch, n ? n->grad : nullptr, nullptr, loss_sum, s);
    if (st != ST_OK) return st;
    return adam_step(n, n->grad, lr, s);
}

extern "C" int pacuda_sg_forward(const pacuda_sg_net *n, const float *x, uint32_t count, float *out, void *stream) {
    g_last_launches = 0;
    if (!n || !x || !out || count == 0) return ST_INVALID;
    ForwardArgs g;
    memset(&g, 0, sizeof g);
    g.wimg = n->wimg;
    g.params = n->params;
    g.x = x;
    g.inputs = n->inputs;
    g.count = count;
    g.tiles = (count + 127) / 128;
    g.out = out;
    g.error = n->error;
    return launch_forward<FWD_FROM_X>(g, (cudaStream_t)stream) ? ST_OK : ST_DEVICE;
}

// the error flag of the network's kernels (0: none), for tests and callers that check after a run
extern "C" int pacuda_sg_error(const pacuda_sg_net *n) {
    int e = 0;
    if (!n || failed(cudaMemcpy(&e, n->error, sizeof e, cudaMemcpyDeviceToHost), "error flag")) return -1;
    return e;
}

// ---- two-stage unweighting ------------------------------------------------------------------------

namespace {

using pacuda::phase::Cuts;
using pacuda::phase::Map;
using pacuda::phase::Space;

// The candidates first .. first + count - 1 of one stream: the indices of those inside the cuts,
// appended (unordered, warp-aggregated) to index[] while below `capacity`; *count_out counts all
// of them. A block takes LIST_ROUNDS x 256 consecutive candidates (candidate k of the block in
// round k / 256 on thread k % 256): each thread gives its candidates the f32 first look
// (phase.cuh surely_fails32), the ones it cannot drop are gathered in shared memory, and then the
// block's threads take those through the f64 map and cuts, which decide; gathering several rounds
// keeps the f64 pass's warps full. (Blocks of 256 threads: the kernels below are launched so.)
constexpr uint32_t LIST_ROUNDS = 16, LIST_BLOCK = 256 * LIST_ROUNDS;

template <int N>
__device__ __forceinline__ void list_block(uint64_t seed, uint64_t first, uint32_t count, double sqrt_s,
                                           const Cuts &cuts, uint64_t *index, uint32_t capacity,
                                           unsigned long long *count_out, uint32_t block_first) {
    constexpr int F = N, L = Space<N>::LEGS;
    __shared__ uint64_t maybe[LIST_BLOCK];
    __shared__ uint32_t n_maybe;
    if (threadIdx.x == 0) n_maybe = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (uint32_t r = 0; r < LIST_ROUNDS; r++) {
        const uint64_t i = (uint64_t)block_first + r * 256 + threadIdx.x;
        bool check = false;
        if (i < count) {
            float u[Space<N>::NUMBERS], q[F][3];
            pacuda::phase::uniforms32(seed, first + i, u);
            pacuda::phase::final32(u, sqrt_s, q);
            check = !pacuda::phase::surely_fails32(q, sqrt_s, cuts);
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, check);
        uint32_t base = 0;
        if (lane == 0 && ballot) base = atomicAdd(&n_maybe, (uint32_t)__popc(ballot));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (check) maybe[base + __popc(ballot & ((1u << lane) - 1u))] = first + i;
    }
    __syncthreads();
    const uint32_t m = n_maybe;
    for (uint32_t at = 0; at < m; at += 256) {
        if (at + threadIdx.x >= ((m + 31u) & ~31u)) break;  // whole warps past the last gathered candidate
        bool pass = false;
        uint64_t cand = 0;
        if (at + threadIdx.x < m) {
            cand = maybe[at + threadIdx.x];
            double u[Space<N>::UNIFORMS], p[L][4];
            pacuda::phase::uniforms(seed, cand, u);
            Map<N>::momenta(u, sqrt_s, p);
            pass = pacuda::phase::passes(p, cuts);
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, pass);
        unsigned long long base = 0;
        if (lane == 0 && ballot) base = atomicAdd(count_out, (unsigned long long)__popc(ballot));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (pass) {
            const unsigned long long slot = base + __popc(ballot & ((1u << lane) - 1u));
            if (slot < capacity) index[slot] = cand;
        }
    }
}

template <int N>
__global__ void __launch_bounds__(256) candidates_kernel(uint64_t seed, uint64_t first, uint32_t count, double sqrt_s,
                                                         Cuts cuts, uint64_t *index, uint32_t capacity,
                                                         unsigned long long *count_out) {
    list_block<N>(seed, first, count, sqrt_s, cuts, index, capacity, count_out, blockIdx.x * LIST_BLOCK);
}

// several subprocesses' candidates in one launch: block b lists segment k's candidates when
// block_first[k] <= b < block_first[k + 1]
struct CandidateSegments {
    pacuda_uw_candidate_segment seg[PACUDA_UW_MAX_SEGMENTS];
    uint32_t block_first[PACUDA_UW_MAX_SEGMENTS + 1];
    uint32_t segments;
};

template <int N>
__global__ void __launch_bounds__(256) candidate_segments_kernel(CandidateSegments c, double sqrt_s, Cuts cuts,
                                                                 uint32_t capacity) {
    uint32_t k = 0;
    while (k + 1 < c.segments && blockIdx.x >= c.block_first[k + 1]) k++;
    const pacuda_uw_candidate_segment &sg = c.seg[k];
    list_block<N>(sg.seed, sg.first, sg.count, sqrt_s, cuts, sg.index, capacity, sg.counter,
                  (blockIdx.x - c.block_first[k]) * LIST_BLOCK);
}

// the points of candidates index[0..n): source-major momenta [(leg * 4 + k) * n + i] for the
// runner, the network's inputs [i][inputs] (the phase-space numbers, then the family's one-hot)
// and the map's weight
template <int N>
__global__ void points_kernel(uint64_t seed, const uint64_t *index, uint32_t n, double sqrt_s, double *momenta,
                              float *inputs_out, uint32_t inputs, uint32_t family, double *jac) {
    constexpr int X = Space<N>::NUMBERS, L = Space<N>::LEGS;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double u[Space<N>::UNIFORMS], p[L][4];
    pacuda::phase::uniforms(seed, index[i], u);
    const double j = Map<N>::momenta(u, sqrt_s, p);
    if (momenta)
        for (int leg = 0; leg < L; leg++)
            for (int k = 0; k < 4; k++) momenta[(size_t)(leg * 4 + k) * n + i] = p[leg][k];
    if (inputs_out)
        for (uint32_t f = 0; f < inputs; f++)
            inputs_out[(size_t)i * inputs + f] = f < (uint32_t)X ? (float)u[f] : (f == X + family ? 1.0f : 0.0f);
    if (jac) jac[i] = j;
}

// |M|^2 = the sum of the runner's helicity outputs, w = |M|^2 J, and the accept/reject decision
// (u_a, u_b: the candidate's two decision uniforms, after its phase-space numbers):
// plain (s == null): kept when u_a w_max < w, weight max(1, w / w_max);
// second stage: r = w / s, kept when u_b r_max < r, weight max(1, s / s_max) max(1, r / r_max)
template <int N>
__global__ void decide_kernel(uint64_t seed, const uint64_t *index, uint32_t n, const double *outputs, uint32_t helicities,
                              const double *jac, const double *s, double w_max, double s_max, double r_max, uint8_t *keep,
                              double *weight, double *me) {
    constexpr int X = Space<N>::NUMBERS;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double m2 = 0.0;
    for (uint32_t h = 0; h < helicities; h++) m2 += outputs[(size_t)i * helicities + h];
    const double w = m2 * jac[i];
    double u[Space<N>::UNIFORMS];
    pacuda::phase::uniforms(seed, index[i], u);
    bool k;
    double wt;
    if (!s) {
        k = u[X] * w_max < w;
        wt = k ? fmax(1.0, w / w_max) : 0.0;
    } else {
        const double r = w / s[i];
        k = u[X + 1] * r_max < r;
        wt = k ? fmax(1.0, s[i] / s_max) * fmax(1.0, r / r_max) : 0.0;
    }
    if (keep) keep[i] = k;
    if (weight) weight[i] = wt;
    if (me) me[i] = m2;
}

bool final_state_valid(uint32_t n) { return n == 3 || n == 4; }

}  // namespace

extern "C" int pacuda_uw_candidates(uint64_t seed, uint64_t first, uint32_t count, uint32_t final_state, double sqrt_s,
                                    const pacuda_uw_cuts *cuts, uint64_t *index, uint32_t capacity,
                                    unsigned long long *counter, void *stream) {
    g_last_launches = 0;
    if (!cuts || !index || !counter || count == 0 || !(sqrt_s > 0) || !final_state_valid(final_state)) return ST_INVALID;
    Cuts c{cuts->pt_min, cuts->eta_max, cuts->dr_min};
    const dim3 grid((count + LIST_BLOCK - 1) / LIST_BLOCK);
    if (final_state == 4)
        candidates_kernel<4><<<grid, 256, 0, (cudaStream_t)stream>>>(seed, first, count, sqrt_s, c, index, capacity, counter);
    else
        candidates_kernel<3><<<grid, 256, 0, (cudaStream_t)stream>>>(seed, first, count, sqrt_s, c, index, capacity, counter);
    g_last_launches++;
    return failed(cudaGetLastError(), "candidates") ? ST_DEVICE : ST_OK;
}

extern "C" int pacuda_uw_candidates_segments(const pacuda_uw_candidate_segment *segs, uint32_t segments,
                                             uint32_t final_state, double sqrt_s, const pacuda_uw_cuts *cuts,
                                             uint32_t capacity, void *stream) {
    g_last_launches = 0;
    if (!segs || !cuts || segments == 0 || segments > PACUDA_UW_MAX_SEGMENTS || !(sqrt_s > 0) ||
        !final_state_valid(final_state))
        return ST_INVALID;
    CandidateSegments c;
    memset(&c, 0, sizeof c);
    uint32_t blocks = 0;
    for (uint32_t k = 0; k < segments; k++) {
        if ((segs[k].count && !segs[k].index) || !segs[k].counter) return ST_INVALID;
        c.seg[k] = segs[k];
        c.block_first[k] = blocks;
        blocks += (segs[k].count + LIST_BLOCK - 1) / LIST_BLOCK;
    }
    c.block_first[segments] = blocks;
    c.segments = segments;
    if (blocks == 0) return ST_OK;
    const Cuts cc{cuts->pt_min, cuts->eta_max, cuts->dr_min};
    if (final_state == 4)
        candidate_segments_kernel<4><<<blocks, 256, 0, (cudaStream_t)stream>>>(c, sqrt_s, cc, capacity);
    else
        candidate_segments_kernel<3><<<blocks, 256, 0, (cudaStream_t)stream>>>(c, sqrt_s, cc, capacity);
    g_last_launches++;
    return failed(cudaGetLastError(), "candidates") ? ST_DEVICE : ST_OK;
}

extern "C" int pacuda_uw_points(uint64_t seed, const uint64_t *index, uint32_t n, uint32_t final_state, double sqrt_s,
                                double *momenta, float *inputs, uint32_t input_count, uint32_t family, double *jac,
                                void *stream) {
    g_last_launches = 0;
    const uint32_t x = 3 * final_state - 4;
    if (!index || n == 0 || !(sqrt_s > 0) || !final_state_valid(final_state) ||
        (inputs && (input_count < x || input_count > IN || x + family >= input_count)))
        return ST_INVALID;
    const dim3 grid((n + 127) / 128);
    if (final_state == 4)
        points_kernel<4><<<grid, 128, 0, (cudaStream_t)stream>>>(seed, index, n, sqrt_s, momenta, inputs, input_count,
                                                                  family, jac);
    else
        points_kernel<3><<<grid, 128, 0, (cudaStream_t)stream>>>(seed, index, n, sqrt_s, momenta, inputs, input_count,
                                                                  family, jac);
    g_last_launches++;
    return failed(cudaGetLastError(), "points") ? ST_DEVICE : ST_OK;
}

extern "C" int pacuda_uw_decide(uint64_t seed, const uint64_t *index, uint32_t n, uint32_t final_state,
                                const double *outputs, uint32_t helicities, const double *jac, const double *s,
                                double w_max, double s_max, double r_max, uint8_t *keep, double *weight, double *me,
                                void *stream) {
    g_last_launches = 0;
    if (!index || !outputs || !jac || helicities == 0 || !final_state_valid(final_state)) return ST_INVALID;
    if (n == 0) return ST_OK;
    const dim3 grid((n + 127) / 128);
    if (final_state == 4)
        decide_kernel<4><<<grid, 128, 0, (cudaStream_t)stream>>>(seed, index, n, outputs, helicities, jac, s, w_max,
                                                                  s_max, r_max, keep, weight, me);
    else
        decide_kernel<3><<<grid, 128, 0, (cudaStream_t)stream>>>(seed, index, n, outputs, helicities, jac, s, w_max,
                                                                  s_max, r_max, keep, weight, me);
    g_last_launches++;
    return failed(cudaGetLastError(), "decide") ? ST_DEVICE : ST_OK;
}

extern "C" int pacuda_uw_stage1_segments(const pacuda_sg_net *n, const pacuda_uw_segment *segs, uint32_t segments,
                                         uint32_t final_state, double mu, double sigma, uint32_t capacity,
                                         void *stream) {
    g_last_launches = 0;
    if (!n || !segs || segments == 0 || segments > PACUDA_UW_MAX_SEGMENTS || !final_state_valid(final_state)) {
        fprintf(stderr, "%s: stage 1: 1 to %d segments of 3 or 4 final-state partons\n", kTag, PACUDA_UW_MAX_SEGMENTS);
        return ST_INVALID;
    }
    const uint32_t x = 3 * final_state - 4;
    ForwardArgs g;
    memset(&g, 0, sizeof g);
    uint32_t tiles = 0;
    for (uint32_t k = 0; k < segments; k++) {
        const pacuda_uw_segment &sg = segs[k];
        if ((sg.count && !sg.index) || !sg.kept_index || !sg.kept_s || !sg.kept_count || x + sg.family >= n->inputs) {
            fprintf(stderr, "%s: stage 1: segment %u: a missing array or a family beyond the inputs\n", kTag, k);
            return ST_INVALID;
        }
        g.seg[k] = sg;
        g.tile_first[k] = tiles;
        tiles += (sg.count + 127) / 128;
    }
    g.tile_first[segments] = tiles;
    if (tiles == 0) return ST_OK;
    g.segments = segments;
    g.wimg = n->wimg;
    g.params = n->params;
    g.inputs = n->inputs;
    g.tiles = tiles;
    g.error = n->error;
    g.mu = mu;
    g.sigma = sigma;
    g.capacity = capacity;
    g.numbers = x;
    return launch_forward<FWD_CANDIDATES>(g, (cudaStream_t)stream) ? ST_OK : ST_DEVICE;
}

extern "C" int pacuda_uw_stage1(const pacuda_sg_net *n, uint64_t seed, const uint64_t *index, uint32_t count,
                                uint32_t final_state, uint32_t family, double mu, double sigma, double s_max,
                                uint64_t *kept_index, double *kept_s, uint32_t capacity, unsigned long long *counter,
                                void *stream) {
    pacuda_uw_segment sg;
    sg.seed = seed;
    sg.index = index;
    sg.count = count;
    sg.family = family;
    sg.s_max = s_max;
    sg.kept_index = kept_index;
    sg.kept_s = kept_s;
    sg.kept_count = counter;
    if (!index) return ST_INVALID;
    return pacuda_uw_stage1_segments(n, &sg, 1, final_state, mu, sigma, capacity, stream);
}
