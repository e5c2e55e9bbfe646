// Learned warm start: a per-pixel MLP on the 5th-generation tensor cores.
//
// Network: 32 inputs (30 used) -> 64 -> 64 -> 64 (GELU) -> 32 outputs (20
// used at five layers, sigmoid). Weights and activations are BF16, products
// accumulate in FP32 in tensor memory. Inputs of a pixel: the 27 RGB values of
// its clamped 3x3 neighbourhood and log(1/256 + c) of its own colour. Outputs:
// the solver's start x = [alpha_0..alpha_{L-1}, rgb_0..rgb_{L-1}] (4L values).
//
// B200 mapping. One CTA of 128 threads owns a tile of 128 pixels (samples);
// thread t owns row t, which is TMEM lane t. Every GEMM is one
// tcgen05.mma.cta_group::1.kind::f16 chain issued by a single thread:
//   forward      Z = H W^T      M=128 (samples)  N=out  K=in   A K-major, B K-major
//   backward     dH = dZ W      M=128 (samples)  N=in   K=out  A K-major, B MN-major
//   weights      dW += dZ^T H   M=64  (outputs)  N=in   K=128  A MN-major, B MN-major
// Operands sit in shared memory in the canonical no-swizzle layout of 8x8
// BF16 core matrices (128 bytes each, K fastest inside a core matrix), so one
// activation tile serves as a K-major operand (forward) and as an MN-major
// operand (weight gradient) without a transposed copy. Completion is tracked
// with tcgen05.commit on an mbarrier; every wait is bounded and sets an error
// flag instead of spinning forever. Accumulators are read with
// tcgen05.ld.32x32b (warp w reads lanes 32w..32w+31).
#include <cuda_bf16.h>

#include "solver_dispatch.hpp"

namespace unb {
namespace mlp {

constexpr int kIn = 32, kHidden = 64, kOut = 32, kTile = 128;

// ------------------------------------------------------------- PTX helpers --
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Element index of (row r, column k) in a rows x K tile made of 8x8 core
// matrices: core (r/8, k/8) at ((r/8)*(K/8) + k/8) * 64 elements, row r%8 at
// 8 elements (16 bytes) inside it.
__device__ __forceinline__ int cidx(int r, int k, int K) {
    return ((((r >> 3) * (K >> 3)) + (k >> 3)) << 6) + ((r & 7) << 3) + (k & 7);
}

// Shared-memory matrix descriptor, no swizzle (start, leading and stride byte
// offsets in 16-byte units; descriptor version 1).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16 with BF16 A/B and FP32 D.
__host__ __device__ constexpr uint32_t idesc(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(id), "r"(acc));
}

__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait for the mbarrier phase `parity` to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t it = 0; it < (1u << 24); ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Make generic-proxy shared-memory writes and TMEM reads of all threads
// visible to the next tensor-core operation issued after the barrier.
__device__ __forceinline__ void sync_for_mma() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t tmem_alloc(uint32_t* slot, uint32_t cols) {
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                     "r"(cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return *slot;
}

__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t cols) {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * __expf(-0.5f * x * x);
}
__device__ __forceinline__ float sigmoid(float x) { return 1.0f / (1.0f + __expf(-x)); }

// ----------------------------------------------------------- shared tiles --
// Weights: W1 64x32, W2 64x64, W3 64x64, W4 32x64 (out x in), each in the
// core-matrix layout with K = in.
struct WeightTiles {
    __nv_bfloat16 w1[kHidden * kIn], w2[kHidden * kHidden], w3[kHidden * kHidden], w4[kOut * kHidden];
    float b1[kHidden], b2[kHidden], b3[kHidden], b4[kOut];
};

__device__ void load_weights(WeightTiles& s, const MlpDevice& p) {
    for (int i = threadIdx.x; i < kHidden * kIn; i += blockDim.x) s.w1[cidx(i / kIn, i % kIn, kIn)] = p.w[0][i];
    for (int i = threadIdx.x; i < kHidden * kHidden; i += blockDim.x) {
        s.w2[cidx(i / kHidden, i % kHidden, kHidden)] = p.w[1][i];
        s.w3[cidx(i / kHidden, i % kHidden, kHidden)] = p.w[2][i];
    }
    for (int i = threadIdx.x; i < kOut * kHidden; i += blockDim.x) s.w4[cidx(i / kHidden, i % kHidden, kHidden)] = p.w[3][i];
    for (int i = threadIdx.x; i < kHidden; i += blockDim.x) { s.b1[i] = p.b[0][i]; s.b2[i] = p.b[1][i]; s.b3[i] = p.b[2][i]; }
    for (int i = threadIdx.x; i < kOut; i += blockDim.x) s.b4[i] = p.b[3][i];
}

// K-major operand (rows x K tile) for K step ks: LBO = 128 B between the two
// K chunks, SBO = (K/8)*128 B between 8-row groups.
__device__ __forceinline__ uint64_t kmajor(const void* tile, int K, int ks) {
    return sdesc(smem_u32(tile) + uint32_t(ks) * 256u, 128u, uint32_t(K / 8) * 128u);
}
// The same rows x K tile read MN-major along its rows, for K step ks over
// rows (16 rows per step): 8-element MN groups are the tile's K chunks
// (SBO = 128 B), 8-row K groups are its row groups (LBO = (K/8)*128 B).
__device__ __forceinline__ uint64_t mnmajor(const void* tile, int K, int ks) {
    return sdesc(smem_u32(tile) + uint32_t(ks) * 2u * uint32_t(K / 8) * 128u, uint32_t(K / 8) * 128u, 128u);
}

// Features of pixel i of a w x h packed RGB image.
__device__ __forceinline__ void features(const double* image, int w, int h, int64_t i, float* f) {
    const int y = int(i / w), x = int(i % w);
    int k = 0;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            const int yy = min(max(y + dy, 0), h - 1), xx = min(max(x + dx, 0), w - 1);
            const double* p = image + 3 * (int64_t(yy) * w + xx);
            f[k++] = float(p[0]); f[k++] = float(p[1]); f[k++] = float(p[2]);
        }
    const double* c = image + 3 * i;
#pragma unroll
    for (int r = 0; r < 3; ++r) f[k++] = __logf(float(c[r]) + (1.0f / 256.0f));
    f[30] = 0.0f; f[31] = 0.0f;
}

struct Forward {
    __nv_bfloat16 h0[kTile * kIn], h1[kTile * kHidden], h2[kTile * kHidden], h3[kTile * kHidden];
};

// Z = H W^T for a layer: M=128, N=n, K=k; accumulate into TMEM column `col`.
__device__ __forceinline__ void gemm_forward(uint32_t tmem, int col, const void* h, const void* w, int n, int k) {
    if (threadIdx.x == 0) {
        const uint32_t id = idesc(kTile, n, false, false);
        for (int ks = 0; ks < k / 16; ++ks) mma(tmem + col, kmajor(h, k, ks), kmajor(w, k, ks), id, ks > 0);
    }
}

// ------------------------------------------------------------------ kernels --
// Inference: x0 for every pixel (n x 4L floats, pixel-major).
__global__ void __launch_bounds__(128, 1) infer_kernel(MlpDevice p, const double* image, int w, int h, int L,
                                                      float* out, int32_t* error) {
    extern __shared__ __align__(128) unsigned char smem[];
    WeightTiles& W = *reinterpret_cast<WeightTiles*>(smem);
    Forward& F = *reinterpret_cast<Forward*>(smem + ((sizeof(WeightTiles) + 127) / 128) * 128);
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int t = threadIdx.x, warp = t >> 5;
    load_weights(W, p);
    if (t == 0) mbar_init(&bar);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const uint32_t tmem = tmem_alloc(&tmem_slot, 64);
    const uint32_t lane_base = tmem + (uint32_t(32 * warp) << 16);
    uint32_t phase = 0;
    bool ok = true;
    const int64_t n = int64_t(w) * h;
    const int64_t tiles = (n + kTile - 1) / kTile;
    for (int64_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const int64_t i = tile * kTile + t;
        float f[kIn];
        if (i < n) features(image, w, h, i, f);
        else for (int k = 0; k < kIn; ++k) f[k] = 0.0f;
        for (int k = 0; k < kIn; ++k) F.h0[cidx(t, k, kIn)] = __float2bfloat16(f[k]);
        const void* hin[3] = {F.h0, F.h1, F.h2};
        __nv_bfloat16* hout[3] = {F.h1, F.h2, F.h3};
        const void* wt[3] = {W.w1, W.w2, W.w3};
        const float* bs[3] = {W.b1, W.b2, W.b3};
        for (int layer = 0; layer < 3 && ok; ++layer) {
            sync_for_mma();
            gemm_forward(tmem, 0, hin[layer], wt[layer], kHidden, layer == 0 ? kIn : kHidden);
            if (t == 0) commit(&bar);
            ok = mbar_wait(&bar, phase);
            phase ^= 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int c = 0; c < kHidden; c += 16) {
                float z[16];
                tmem_ld16(lane_base + c, z);
                for (int j = 0; j < 16; ++j) hout[layer][cidx(t, c + j, kHidden)] = __float2bfloat16(gelu(z[j] + bs[layer][c + j]));
            }
        }
        if (!ok) break;
        sync_for_mma();
        gemm_forward(tmem, 0, F.h3, W.w4, kOut, kHidden);
        if (t == 0) commit(&bar);
        ok = mbar_wait(&bar, phase);
        phase ^= 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        float z[kOut];
        tmem_ld16(lane_base, z);
        tmem_ld16(lane_base + 16, z + 16);
        if (i < n)
            for (int k = 0; k < 4 * L; ++k) out[i * (4 * L) + k] = sigmoid(z[k] + W.b4[k]);
    }
    if (!ok && t == 0) atomicExch(error, 1);
    tmem_free(tmem, 64);
}

// One training pass over `count` samples (features fp32 [count][32],
// targets fp32 [count][outs]): loss = mean over samples and outputs of
// (sigmoid(z) - target)^2. Accumulates dW (fp32, out x in row-major) and db
// into `grad` with atomics; adds the loss sum into grad->loss.
struct TrainTiles {
    Forward f;
    float gz1[kTile * kHidden], gz2[kTile * kHidden], gz3[kTile * kHidden];   // GELU'(Z), row-major [sample][unit]
    __nv_bfloat16 dz[kTile * kHidden];                                         // dZ of the current layer
    float db[4][kHidden];
};

__global__ void __launch_bounds__(128, 1) train_kernel(MlpDevice p, const float* feats, const float* targets,
                                                      int count, int outs, MlpGrad g, int32_t* error) {
    extern __shared__ __align__(128) unsigned char smem[];
    WeightTiles& W = *reinterpret_cast<WeightTiles*>(smem);
    TrainTiles& S = *reinterpret_cast<TrainTiles*>(smem + ((sizeof(WeightTiles) + 127) / 128) * 128);
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    load_weights(W, p);
    for (int i = t; i < 4 * kHidden; i += blockDim.x) S.db[i / kHidden][i % kHidden] = 0.0f;
    for (int i = t; i < kTile * kHidden; i += blockDim.x) S.dz[i] = __float2bfloat16(0.0f);
    if (t == 0) mbar_init(&bar);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    // TMEM columns: [0,64) forward Z / backward dH; [64,96) dW1; [128,192)
    // dW2; [192,256) dW3; [256,320) dW4. dW tiles are M=64: row r lives in
    // lane 32*(r/16) + r%16.
    const uint32_t tmem = tmem_alloc(&tmem_slot, 512);
    const uint32_t lane_base = tmem + (uint32_t(32 * warp) << 16);
    const int dw_col[4] = {64, 128, 192, 256};
    uint32_t phase = 0;
    bool ok = true, first = true;
    float loss = 0.0f;
    const int tiles = (count + kTile - 1) / kTile;
    for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const int i = tile * kTile + t;
        const bool valid = i < count;
        // ---- forward, keeping H (bf16) and GELU'(Z)
        for (int k = 0; k < kIn; ++k) S.f.h0[cidx(t, k, kIn)] = __float2bfloat16(valid ? feats[int64_t(i) * kIn + k] : 0.0f);
        const void* hin[3] = {S.f.h0, S.f.h1, S.f.h2};
        __nv_bfloat16* hout[3] = {S.f.h1, S.f.h2, S.f.h3};
        float* gz[3] = {S.gz1, S.gz2, S.gz3};
        const void* wt[4] = {W.w1, W.w2, W.w3, W.w4};
        const float* bs[3] = {W.b1, W.b2, W.b3};
        for (int layer = 0; layer < 3 && ok; ++layer) {
            sync_for_mma();
            gemm_forward(tmem, 0, hin[layer], wt[layer], kHidden, layer == 0 ? kIn : kHidden);
            if (t == 0) commit(&bar);
            ok = mbar_wait(&bar, phase);
            phase ^= 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int c = 0; c < kHidden; c += 16) {
                float z[16];
                tmem_ld16(lane_base + c, z);
                for (int j = 0; j < 16; ++j) {
                    const float a = z[j] + bs[layer][c + j];
                    // Padded sample rows carry zeros through the whole pass.
                    hout[layer][cidx(t, c + j, kHidden)] = __float2bfloat16(valid ? gelu(a) : 0.0f);
                    gz[layer][t * kHidden + c + j] = valid ? gelu_grad(a) : 0.0f;
                }
            }
        }
        if (!ok) break;
        sync_for_mma();
        gemm_forward(tmem, 0, S.f.h3, W.w4, kOut, kHidden);
        if (t == 0) commit(&bar);
        ok = mbar_wait(&bar, phase);
        phase ^= 1;
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        {
            float z[kOut];
            tmem_ld16(lane_base, z);
            tmem_ld16(lane_base + 16, z + 16);
            const float scale = 2.0f / (float(count) * float(outs));
            for (int k = 0; k < kHidden; ++k) {
                float d = 0.0f;
                if (valid && k < outs) {
                    const float y = sigmoid(z[k] + W.b4[k]);
                    const float e = y - targets[int64_t(i) * outs + k];
                    loss += e * e;
                    d = scale * e * y * (1.0f - y);
                }
                S.dz[cidx(t, k, kHidden)] = __float2bfloat16(d);
                if (k < kOut) atomicAdd(&S.db[3][k], d);
            }
        }
        // ---- backward: layer 4 (dZ4 = S.dz, 64 columns, 20 used), then 3, 2, 1
        const void* hprev[4] = {S.f.h0, S.f.h1, S.f.h2, S.f.h3};
        for (int layer = 3; layer >= 0 && ok; --layer) {
            const int in = layer == 0 ? kIn : kHidden;
            const int out = layer == 3 ? kOut : kHidden;
            sync_for_mma();
            if (t == 0) {
                // dW += dZ^T H: M=64 (units, dz tile read MN-major), N=in, K=128 samples.
                const uint32_t idw = idesc(64, in, true, true);
                for (int ks = 0; ks < kTile / 16; ++ks)
                    mma(tmem + dw_col[layer], mnmajor(S.dz, kHidden, ks), mnmajor(hprev[layer], in, ks), idw,
                        (!first || ks > 0) ? 1u : 0u);
                if (layer > 0) {
                    // dH = dZ W: M=128, N=in, K=out (weights read MN-major).
                    const uint32_t idh = idesc(kTile, in, false, true);
                    for (int ks = 0; ks < out / 16; ++ks)
                        mma(tmem, kmajor(S.dz, kHidden, ks), mnmajor(wt[layer], in, ks), idh, ks > 0);
                }
                commit(&bar);
            }
            ok = mbar_wait(&bar, phase);
            phase ^= 1;
            if (!ok || layer == 0) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int c = 0; c < kHidden; c += 16) {
                float dh[16];
                tmem_ld16(lane_base + c, dh);
                for (int j = 0; j < 16; ++j) {
                    const float d = dh[j] * gz[layer - 1][t * kHidden + c + j];
                    S.dz[cidx(t, c + j, kHidden)] = __float2bfloat16(d);
                    atomicAdd(&S.db[layer - 1][c + j], d);
                }
            }
        }
        first = false;
    }
    // ---- flush dW and db accumulated by this CTA
    sync_for_mma();
    if (ok && !first) {
        const int rows_per_warp = 16;
        for (int layer = 0; layer < 4; ++layer) {
            const int in = layer == 0 ? kIn : kHidden;
            const int out = layer == 3 ? kOut : kHidden;
            for (int c = 0; c < in; c += 16) {
                float v[16];
                tmem_ld16(lane_base + dw_col[layer] + c, v);
                if (lane < rows_per_warp) {
                    const int r = warp * rows_per_warp + lane;   // dW row (unit)
                    if (r < out)
                        for (int j = 0; j < 16; ++j) atomicAdd(&g.w[layer][r * in + c + j], v[j]);
                }
            }
        }
    }
    __syncthreads();
    for (int i = t; i < 3 * kHidden + kOut; i += blockDim.x) {
        const int layer = i < 3 * kHidden ? i / kHidden : 3;
        const int u = i < 3 * kHidden ? i % kHidden : i - 3 * kHidden;
        atomicAdd(&g.b[layer][u], S.db[layer][u]);
    }
    for (int off = 16; off > 0; off >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, off);
    if (lane == 0) atomicAdd(g.loss, loss);
    if (!ok && t == 0) atomicExch(error, 1);
    tmem_free(tmem, 512);
}

// Adam on the FP32 master weights; refreshes the BF16 copies and clears the
// gradient. Parameter blocks: 4 weight matrices then 4 bias vectors.
__global__ void adam_kernel(MlpMaster m, MlpGrad g, MlpDevice p, float lr, float b1, float b2, float eps, int step) {
    const float c1 = 1.0f - __powf(b1, float(step)), c2 = 1.0f - __powf(b2, float(step));
    const int sizes[8] = {kHidden * kIn, kHidden * kHidden, kHidden * kHidden, kOut * kHidden,
                          kHidden, kHidden, kHidden, kOut};
    for (int blk = 0; blk < 8; ++blk) {
        float* w = blk < 4 ? m.w[blk] : m.b[blk - 4];
        float* gr = blk < 4 ? g.w[blk] : g.b[blk - 4];
        float* mm = blk < 4 ? m.mw[blk] : m.mb[blk - 4];
        float* vv = blk < 4 ? m.vw[blk] : m.vb[blk - 4];
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < sizes[blk]; i += gridDim.x * blockDim.x) {
            const float gi = gr[i];
            mm[i] = b1 * mm[i] + (1.0f - b1) * gi;
            vv[i] = b2 * vv[i] + (1.0f - b2) * gi * gi;
            w[i] -= lr * (mm[i] / c1) / (sqrtf(vv[i] / c2) + eps);
            gr[i] = 0.0f;
            if (blk < 4) const_cast<__nv_bfloat16*>(p.w[blk])[i] = __float2bfloat16(w[i]);
        }
    }
}

// Training features of the pixels of an image (n x 32 floats).
__global__ void features_kernel(const double* image, int w, int h, float* feats) {
    const int64_t n = int64_t(w) * h;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        float f[kIn];
        features(image, w, h, i, f);
        for (int k = 0; k < kIn; ++k) feats[i * kIn + k] = f[k];
    }
}

size_t infer_smem() { return ((sizeof(WeightTiles) + 127) / 128) * 128 + sizeof(Forward); }
size_t train_smem() { return ((sizeof(WeightTiles) + 127) / 128) * 128 + sizeof(TrainTiles); }

}  // namespace mlp

cudaError_t launch_mlp_infer(const MlpDevice& p, const double* image, int w, int h, int L, float* out,
                             int32_t* error, int sms, cudaStream_t s) {
    const size_t smem = mlp::infer_smem();
    cudaError_t e = cudaFuncSetAttribute(mlp::infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    const int64_t tiles = (int64_t(w) * h + mlp::kTile - 1) / mlp::kTile;
    const int grid = int(tiles < sms ? tiles : sms);
    mlp::infer_kernel<<<grid, 128, smem, s>>>(p, image, w, h, L, out, error);
    return cudaGetLastError();
}

cudaError_t launch_mlp_features(const double* image, int w, int h, float* feats, cudaStream_t s) {
    mlp::features_kernel<<<148 * 4, 256, 0, s>>>(image, w, h, feats);
    return cudaGetLastError();
}

cudaError_t launch_mlp_train(const MlpDevice& p, const float* feats, const float* targets, int count, int outs,
                             const MlpGrad& g, int32_t* error, int sms, cudaStream_t s) {
    const size_t smem = mlp::train_smem();
    cudaError_t e = cudaFuncSetAttribute(mlp::train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    const int tiles = (count + mlp::kTile - 1) / mlp::kTile;
    const int grid = tiles < sms ? tiles : sms;
    mlp::train_kernel<<<grid, 128, smem, s>>>(p, feats, targets, count, outs, g, error);
    return cudaGetLastError();
}

cudaError_t launch_mlp_adam(const MlpMaster& m, const MlpGrad& g, const MlpDevice& p, float lr, int step,
                            cudaStream_t s) {
    mlp::adam_kernel<<<8, 256, 0, s>>>(m, g, p, lr, 0.9f, 0.999f, 1e-8f, step);
    return cudaGetLastError();
}

}  // namespace unb
