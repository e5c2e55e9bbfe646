// Training data for the warm-start MLP: solver outputs as targets, and
// seeded minibatch sampling from the pool of (features, targets) rows.
#include "solver_dispatch.hpp"

namespace unb {
namespace {

// Packed [l][i][RGBA] first pass -> pixel-major x = [alpha_l..., rgb_l...].
__global__ void gather_targets(const double* packed, int64_t n, int L, float* targets) {
    const int outs = 4 * L;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        for (int l = 0; l < L; ++l) {
            const double* p = packed + (int64_t(l) * n + i) * 4;
            targets[i * outs + l] = float(p[3]);
            for (int c = 0; c < 3; ++c) targets[i * outs + L + 3 * l + c] = float(p[c]);
        }
    }
}

__device__ __forceinline__ uint64_t mix(uint64_t x) {   // splitmix64 finalizer
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__global__ void sample_batch(const float* feats, const float* targets, int64_t pool, int outs, int batch,
                             uint64_t seed, float* bfeats, float* btargets) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= batch) return;
    const int64_t src = int64_t(mix(seed * 0x100000001B3ull + uint64_t(j)) % uint64_t(pool));
    for (int k = 0; k < kMlpIn; ++k) bfeats[int64_t(j) * kMlpIn + k] = feats[src * kMlpIn + k];
    for (int k = 0; k < outs; ++k) btargets[int64_t(j) * outs + k] = targets[src * outs + k];
}

}  // namespace

cudaError_t launch_gather_targets(const double* packed, int64_t n, int L, float* targets, cudaStream_t s) {
    gather_targets<<<148 * 4, 256, 0, s>>>(packed, n, L, targets);
    return cudaGetLastError();
}

cudaError_t launch_sample_batch(const float* feats, const float* targets, int64_t pool, int outs, int batch,
                                uint64_t seed, float* bfeats, float* btargets, cudaStream_t s) {
    sample_batch<<<(batch + 255) / 256, 256, 0, s>>>(feats, targets, pool, outs, batch, seed, bfeats, btargets);
    return cudaGetLastError();
}

}  // namespace unb
