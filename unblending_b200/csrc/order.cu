// Work-queue order of a solve launch: the pixels grouped by colour.
//
// A quad's path through the method (which actions it takes, how many
// line-search trials, how many outer steps) depends on the pixel's target
// colour; in the first pass it is a function of that colour alone. The
// lockstep kernel runs every action that any quad of a warp needs, with the
// other quads waiting, so a warp whose eight pixels have similar colours
// wastes fewer trips. The queue therefore hands out pixels in a Morton
// (Z-curve) order of their RGB quantized to `bits` bits a channel (4 to 7,
// about one cell per pixel for the launch's pixel count):
// consecutive queue indices, which the quads of a warp pull at about the same
// time, are pixels of nearby colours. Each pixel's solve reads only its own
// inputs, so the order changes the speed and never the results.
//
// A counting sort over the 2^(3*bits) colour cells: count, exclusive scan
// (two kernels), scatter. Within a cell the scatter's atomics decide the
// order.
#include <algorithm>

#include "solver_dispatch.hpp"

namespace unb {

namespace {

constexpr int kMinOrderBits = 4, kMaxOrderBits = 7;

// The pixels being ordered: queue index k is pixel first + k of `image`,
// or (a batched group) queue index k of `jobs`, in the image whose offset is
// the last one <= k.
struct OrderSource {
    const double* image;
    int first;
    const BatchJob* jobs;
    int job_count;
    // The RGB of queue index k, and the value the order stores for it.
    __device__ __forceinline__ const double* rgb(int k, int32_t& value) const {
        if (!jobs) {
            value = first + k;
            return image + 3 * size_t(value);
        }
        int lo = 0, hi = job_count - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].offset <= int64_t(k)) lo = mid; else hi = mid - 1;
        }
        value = k;
        return jobs[lo].image + 3 * size_t(int64_t(k) - jobs[lo].offset);
    }
};

// Cell of a pixel: the bits of the three quantized channels interleaved
// (bit b of channel c at bit 3b + c). NaN and negative values fall in level 0,
// values >= 1 in the top level.
__device__ __forceinline__ uint32_t colour_cell(const double* rgb, int bits) {
    uint32_t key = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double v = rgb[c];
        const uint32_t q = v >= 0.0 ? (v < 1.0 ? uint32_t(v * double(1 << bits)) : (1u << bits) - 1u) : 0u;
#pragma unroll
        for (int b = 0; b < kMaxOrderBits; ++b)
            if (b < bits) key |= ((q >> b) & 1u) << (3 * b + c);
    }
    return key;
}

__global__ void order_count(const OrderSource src, int count, int bits, uint32_t* __restrict__ cells) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        int32_t value;
        atomicAdd(&cells[colour_cell(src.rgb(k, value), bits)], 1u);
    }
}

// Exclusive prefix sum of the cell counts, in place, in chunks of
// kScanChunk cells (one block each): order_chunk_sums adds up each chunk,
// order_chunk_scan adds the chunks before its own and scans its chunk.
constexpr int kScanChunk = 4096, kScanThreads = 256, kScanPer = kScanChunk / kScanThreads;
static_assert(kScanPer == 16, "each scan thread owns four uint4 of cells");

__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* warp_totals) {
    v = __reduce_add_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0) warp_totals[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t t = 0;
#pragma unroll
    for (int w = 0; w < kScanThreads / 32; ++w) t += warp_totals[w];
    __syncthreads();
    return t;
}

__global__ void __launch_bounds__(kScanThreads) order_chunk_sums(const uint32_t* __restrict__ cells,
                                                                 uint32_t* __restrict__ sums) {
    __shared__ uint32_t warp_totals[kScanThreads / 32];
    const uint32_t* c = cells + size_t(blockIdx.x) * kScanChunk;
    uint32_t v = 0;
    for (int k = threadIdx.x; k < kScanChunk; k += kScanThreads) v += c[k];
    const uint32_t t = block_sum(v, warp_totals);
    if (threadIdx.x == 0) sums[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kScanThreads) order_chunk_scan(uint32_t* __restrict__ cells,
                                                                 const uint32_t* __restrict__ sums) {
    __shared__ uint32_t warp_totals[kScanThreads / 32];
    uint32_t before = 0;
    for (int k = threadIdx.x; k < int(blockIdx.x); k += kScanThreads) before += sums[k];
    const uint32_t carry = block_sum(before, warp_totals);
    // This thread's kScanPer consecutive cells (64 bytes, aligned).
    uint4* mine = reinterpret_cast<uint4*>(cells + size_t(blockIdx.x) * kScanChunk + size_t(threadIdx.x) * kScanPer);
    uint4 v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = mine[q];
    uint32_t own = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) own += v[q].x + v[q].y + v[q].z + v[q].w;
    // Exclusive prefix of the threads' totals over the block.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = own;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += u;
    }
    if (lane == 31) warp_totals[warp] = inc;
    __syncthreads();
    uint32_t run = carry + inc - own;
    for (int w = 0; w < warp; ++w) run += warp_totals[w];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint4 o;
        o.x = run; run += v[q].x;
        o.y = run; run += v[q].y;
        o.z = run; run += v[q].z;
        o.w = run; run += v[q].w;
        mine[q] = o;
    }
}

__global__ void order_scatter(const OrderSource src, int count, int bits, uint32_t* __restrict__ cells,
                              int32_t* __restrict__ order) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        int32_t value;
        const double* rgb = src.rgb(k, value);
        order[atomicAdd(&cells[colour_cell(rgb, bits)], 1u)] = value;
    }
}

// Bits a channel for `count` pixels: the fewest with at least one cell per
// pixel, within [kMinOrderBits, kMaxOrderBits].
int order_bits(int count) {
    int bits = kMinOrderBits;
    while (bits < kMaxOrderBits && (int64_t(1) << (3 * bits)) < int64_t(count)) ++bits;
    return bits;
}

}  // namespace

// The cells, then one chunk sum per kScanChunk cells.
size_t order_cells(int count) {
    const size_t cells = size_t(1) << (3 * order_bits(count));
    return cells + cells / kScanChunk;
}

namespace {
cudaError_t launch_order(const OrderSource& src, int count, uint32_t* cells, int32_t* order, int sms, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const int bits = order_bits(count);
    const int cell_count = 1 << (3 * bits);
    cudaError_t e = cudaMemsetAsync(cells, 0, sizeof(uint32_t) * size_t(cell_count), s);
    if (e != cudaSuccess) return e;
    const int threads = 256;
    const int blocks = std::min((count + threads - 1) / threads, 8 * sms);
    const int chunks = cell_count / kScanChunk;
    uint32_t* sums = cells + cell_count;
    order_count<<<blocks, threads, 0, s>>>(src, count, bits, cells);
    order_chunk_sums<<<chunks, kScanThreads, 0, s>>>(cells, sums);
    order_chunk_scan<<<chunks, kScanThreads, 0, s>>>(cells, sums);
    order_scatter<<<blocks, threads, 0, s>>>(src, count, bits, cells, order);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_pixel_order(const double* image, int first, int count, uint32_t* cells, int32_t* order, int sms,
                               cudaStream_t s) {
    return launch_order(OrderSource{image, first, nullptr, 0}, count, cells, order, sms, s);
}

cudaError_t launch_group_order(const BatchJob* jobs, int job_count, int total, uint32_t* cells, int32_t* order,
                               int sms, cudaStream_t s) {
    return launch_order(OrderSource{nullptr, 0, jobs, job_count}, total, cells, order, sms, s);
}

}  // namespace unb
