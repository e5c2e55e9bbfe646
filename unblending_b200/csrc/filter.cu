// Guided-filter refinement targets on the GPU, accumulated in FP64.
//
// Computes, for every filtered channel p (the L first-pass alphas, plus the
// background RGB when smoothing) with the RGB image I as guidance, the
// He et al. colour guided filter of the reference (image_processing.cpp:214-273,
// the O(n) twin in refinement/guided_filter.cuh:14-45 and
// streaming_guided_filter.cuh:34-60):
//     a = (cov(I) + eps Id)^-1 cov(I, p),  b = mean(p) - a . mean(I),
//     q = box(b) + box(a) . I,  target = clip(q, 0, 1)
// with clamp-to-edge (2r+1)^2 mean filters, then the alpha normalization of
// unblending.cpp:311-333 (all-Plus: divide by the alpha sum; all-SourceOver:
// require alpha_0 == 1 within 1e-5).
//
// Layout: planes of n doubles, row-major pixels. Each mean filter is two
// passes (rows, then columns), O(1) per pixel for any radius, as the
// reference's GPU filter is (row prefix scans, guided_filter.cuh:49-66):
//   * rows: one CTA per image row; each plane of the row is prefix-summed
//     across the CTA in shared memory (FP64; padding keeps the threads'
//     chunk scans free of bank conflicts) and the
//     window sums are prefix differences, read and written with coalesced
//     accesses. The first box's
//     planes (I, I I^T, p, I p) are formed from the image and the first pass
//     inside this kernel instead of being packed to memory first.
//   * columns: one thread per (plane, column, segment of rows) with a
//     sliding window down its segment, so that a warp reads 32 adjacent
//     doubles per step and the grid has enough warps to cover the latency.
// All sums stay in FP64: E[I^2] - E[I]^2 cancels.
#include "solver_dispatch.hpp"

namespace unb {
namespace {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Threads of a row-pass CTA: 128 at 64 registers gives eight CTAs per SM,
// so the rows of a 1024-high image run in one wave of 148 x 8 CTAs.
constexpr int kRowThreads = 128;
// Widest row the prefix pass keeps in shared memory (at most 102 KiB of
// doubles with the padding below); wider images take the one-thread-per-row
// sliding pass.
constexpr int kRowPrefixMaxWidth = 12288;

// Shared-memory slot of row element x in the prefix pass: thread t scans
// elements [t*chunk, (t+1)*chunk), so the lanes of a warp are `chunk`
// doubles apart, and an even chunk puts them in the same banks (16-way at
// chunk 8, the 1024-wide image). One pad double after every 2^sh values,
// 2^sh the lowest set bit of an even chunk, makes the distance between lanes
// odd (chunk + chunk / 2^sh = m (2^sh + 1), m odd), so a warp's 32 doubles
// fall on 16 distinct bank pairs: two wavefronts, the minimum for 8-byte
// words. An odd chunk is conflict-free unpadded (sh = 31). Contiguous reads
// of 32 values take at most three wavefronts.
__host__ __device__ __forceinline__ int row_chunk(int w) { return (w + kRowThreads - 1) / kRowThreads; }
__host__ __device__ __forceinline__ int row_pad_shift(int w) {
    const int c = row_chunk(w);
    if (c & 1) return 31;
    int sh = 0;
    while (((c >> sh) & 1) == 0) ++sh;
    return sh;
}
__host__ __device__ __forceinline__ int padx(int x, int sh) { return x + (x >> sh); }
constexpr int kColSegment = 128;   // rows per thread of the column pass

// Channel value p_c of pixel i: first-pass alpha of layer c (c < L), else the
// background colour channel c - L.
__device__ __forceinline__ double channel(const double* first, size_t n, int L, int c, size_t i) {
    return c < L ? first[(size_t(c) * n + i) * 4 + 3] : first[i * 4 + (c - L)];
}

// planes: [0..2] I, [3..8] I_r I_r, I_r I_g, I_r I_b, I_g I_g, I_g I_b, I_b I_b,
// then per channel c: [9+4c] p, [9+4c+1..3] I_r p, I_g p, I_b p.
__global__ void pack_planes(const double* image, const double* first, double* planes, size_t n, int L, int channels) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double r = image[3 * i], g = image[3 * i + 1], b = image[3 * i + 2];
        planes[i] = r; planes[n + i] = g; planes[2 * n + i] = b;
        planes[3 * n + i] = r * r; planes[4 * n + i] = r * g; planes[5 * n + i] = r * b;
        planes[6 * n + i] = g * g; planes[7 * n + i] = g * b; planes[8 * n + i] = b * b;
        for (int c = 0; c < channels; ++c) {
            const double p = channel(first, n, L, c, i);
            double* o = planes + (9 + 4 * size_t(c)) * n;
            o[i] = p; o[n + i] = r * p; o[2 * n + i] = g * p; o[3 * n + i] = b * p;
        }
    }
}

// Value of packed plane k (the layout of pack_planes) at pixel i.
__device__ __forceinline__ double packed_value(const double* image, const double* first, size_t n, int L, int k,
                                               size_t i) {
    if (k < 3) return image[3 * i + k];
    if (k < 9) {
        // I_r I_r, I_r I_g, I_r I_b, I_g I_g, I_g I_b, I_b I_b
        const int a = k < 6 ? 0 : (k < 8 ? 1 : 2);
        const int b = k < 6 ? k - 3 : (k < 8 ? k - 5 : 2);
        return image[3 * i + a] * image[3 * i + b];
    }
    const int c = (k - 9) >> 2, m = (k - 9) & 3;
    const double p = channel(first, n, L, c, i);
    return m == 0 ? p : image[3 * i + (m - 1)] * p;
}

// Clamp-to-edge window mean along rows by prefix sums, one CTA per row:
// for each plane the row's values go to shared memory, are prefix-summed
// across the CTA (each thread scans its chunk, the chunk totals are scanned
// by shuffles), and out[x] = (S[min(x+r, w-1)] - S[x-r-1] + clamped copies of
// the end values) / (2r+1). PACKED: plane k of the input is packed plane k,
// formed from the image and the first pass.
template <bool PACKED>
__global__ void __launch_bounds__(kRowThreads, 8)
box_rows_prefix(const double* in, const double* image, const double* first, double* out, int w, int h, int planes,
                int L, int r) {
    extern __shared__ double sm_row[];   // w prefix values (padded), then one total per warp
    const int sh = row_pad_shift(w);
    double* warp_total = sm_row + padx(w - 1, sh) + 1;
    const int y = blockIdx.x;
    const size_t n = size_t(w) * h, row0 = size_t(y) * w;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const int chunk = row_chunk(w);
    const int x0 = min(w, t * chunk), x1 = min(w, x0 + chunk);
    const double norm = double(2 * r + 1);
    for (int k = 0; k < planes; ++k) {
        const double* src = PACKED ? nullptr : in + size_t(k) * n + row0;
        // Coalesced load of the row into shared memory.
        for (int x = t; x < w; x += kRowThreads)
            sm_row[padx(x, sh)] = PACKED ? packed_value(image, first, n, L, k, row0 + x) : src[x];
        __syncthreads();
        // Inclusive scan: this thread's chunk, then the chunk totals.
        double s = 0.0;
        for (int x = x0; x < x1; ++x) { s += sm_row[padx(x, sh)]; sm_row[padx(x, sh)] = s; }
        double incl = s;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        if (lane == 31) warp_total[wid] = incl;
        __syncthreads();
        double carry = incl - s;   // exclusive prefix of this thread within its warp
        for (int q = 0; q < wid; ++q) carry += warp_total[q];
        for (int x = x0; x < x1; ++x) sm_row[padx(x, sh)] += carry;
        __syncthreads();
        // Window sums: prefix differences plus the clamped copies of the end
        // values (read again from their source, exactly).
        const double first_v = PACKED ? packed_value(image, first, n, L, k, row0) : src[0];
        const double last_v = PACKED ? packed_value(image, first, n, L, k, row0 + w - 1) : src[w - 1];
        double* dst = out + size_t(k) * n + row0;
        for (int x = t; x < w; x += kRowThreads) {
            const int hi = min(x + r, w - 1), lo = x - r - 1;
            double sum = sm_row[padx(hi, sh)] - (lo >= 0 ? sm_row[padx(lo, sh)] : 0.0);
            if (x - r < 0) sum += double(r - x) * first_v;
            if (x + r > w - 1) sum += double(x + r - (w - 1)) * last_v;
            dst[x] = sum / norm;
        }
        __syncthreads();
    }
}

// Clamp-to-edge window mean along columns: one thread per (plane, column,
// segment of kColSegment rows), sliding down its segment; the first window
// is summed in full. Threads of a warp take adjacent columns.
__global__ void box_cols_segments(const double* in, double* out, int w, int h, int planes, int r) {
    const int segs = (h + kColSegment - 1) / kColSegment;
    const size_t job = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (job >= size_t(planes) * segs * w) return;
    const int x = int(job % w);
    const size_t rest = job / w;
    const int s = int(rest % segs), p = int(rest / segs);
    const double* col = in + size_t(p) * w * h + x;
    double* o = out + size_t(p) * w * h + x;
    const int y0 = s * kColSegment, y1 = min(h, y0 + kColSegment);
    const double norm = double(2 * r + 1);
    double sum = 0.0;
    for (int j = y0 - r; j <= y0 + r; ++j) sum += col[size_t(clampi(j, 0, h - 1)) * w];
    for (int y = y0; y < y1; ++y) {
        o[size_t(y) * w] = sum / norm;
        sum += col[size_t(clampi(y + r + 1, 0, h - 1)) * w] - col[size_t(clampi(y - r, 0, h - 1)) * w];
    }
}

// Sliding mean along rows: one thread per (plane, row) (rows wider than the
// prefix pass holds).
__global__ void box_rows(const double* in, double* out, int w, int h, int planes, int r) {
    const int job = blockIdx.x * blockDim.x + threadIdx.x;
    if (job >= planes * h) return;
    const double* row = in + size_t(job) * w;
    double* o = out + size_t(job) * w;
    const double norm = double(2 * r + 1);
    double sum = double(r + 1) * row[0];
    const int hi = r < w - 1 ? r : w - 1;
    for (int x = 1; x <= hi; ++x) sum += row[x];
    if (r >= w) sum += double(r - w + 1) * row[w - 1];
    for (int x = 0; x < w; ++x) {
        o[x] = sum / norm;
        sum += row[clampi(x + r + 1, 0, w - 1)] - row[clampi(x - r, 0, w - 1)];
    }
}

// Per pixel: (cov(I) + eps Id)^-1 by cofactors, then a and b of every
// channel. coef planes per channel c: [4c] b, [4c+1..3] a_r, a_g, a_b.
__global__ void coefficients(const double* mean, double* coef, size_t n, int channels, double eps) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double r = mean[i], g = mean[n + i], b = mean[2 * n + i];
        const double a = mean[3 * n + i] - r * r + eps, d = mean[4 * n + i] - r * g, e = mean[5 * n + i] - r * b;
        const double f = mean[6 * n + i] - g * g + eps, hh = mean[7 * n + i] - g * b, ii = mean[8 * n + i] - b * b + eps;
        const double A = f * ii - hh * hh, B = e * hh - d * ii, C = d * hh - e * f;
        const double D = a * ii - e * e, E = d * e - a * hh, F = a * f - d * d;
        const double det = a * A + d * B + e * C;
        const double i0 = A / det, i1 = B / det, i2 = C / det, i4 = D / det, i5 = E / det, i8 = F / det;
        for (int c = 0; c < channels; ++c) {
            const double* m = mean + (9 + 4 * size_t(c)) * n;
            const double mp = m[i];
            const double x = m[n + i] - r * mp, y = m[2 * n + i] - g * mp, z = m[3 * n + i] - b * mp;
            const double ar = i0 * x + i1 * y + i2 * z;
            const double ag = i1 * x + i4 * y + i5 * z;
            const double ab = i2 * x + i5 * y + i8 * z;
            double* o = coef + 4 * size_t(c) * n;
            o[i] = mp - ar * r - ag * g - ab * b;
            o[n + i] = ar; o[2 * n + i] = ag; o[3 * n + i] = ab;
        }
    }
}

// q = box(b) + box(a) . I, clip, normalize; write alpha and background targets.
__global__ void finish_targets(const double* image, const double* first, const double* mcoef, double* targets,
                               int32_t* status, size_t n, int L, int channels, int smooth, int plus, int identity) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double I[3] = {image[3 * i], image[3 * i + 1], image[3 * i + 2]};
        double sum = 0.0;
        int32_t code = 0;
        for (int c = 0; c < channels; ++c) {
            double q;
            if (identity) {
                q = channel(first, n, L, c, i);
            } else {
                const double* m = mcoef + 4 * size_t(c) * n;
                q = m[i];
                for (int k = 0; k < 3; ++k) q += m[(k + 1) * n + i] * I[k];
            }
            q = q < 0.0 ? 0.0 : (q > 1.0 ? 1.0 : q);
            targets[size_t(c) * n + i] = q;
            if (c < L) sum += q;
            if (c == 0) code = (!plus && fabs(q - 1.0) >= 1e-5) ? 2 : 0;
        }
        if (plus) {
            if (sum > 0.0) for (int l = 0; l < L; ++l) targets[size_t(l) * n + i] = targets[size_t(l) * n + i] / sum;
            else code = 1;
        }
        if (!smooth) for (int k = 0; k < 3; ++k) targets[size_t(L + k) * n + i] = first[i * 4 + k];
        status[i] = code;
    }
}

// Window means of `planes` planes: rows (prefix pass, or the sliding pass
// for very wide rows) into tmp, then columns into out. With `image`, the
// input planes are the packed planes of the first box, formed on the fly
// (the sliding row pass needs them in memory: pack_planes writes them to
// `in` first).
cudaError_t box(const double* in, const double* image, const double* first, int L, int channels, double* tmp,
                double* out, int w, int h, int planes, int r, cudaStream_t s) {
    if (w <= kRowPrefixMaxWidth) {
        const size_t smem = (size_t(padx(w - 1, row_pad_shift(w))) + 1 + kRowThreads / 32) * sizeof(double);
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(image ? box_rows_prefix<true> : box_rows_prefix<false>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            if (e != cudaSuccess) return e;
        }
        if (image) box_rows_prefix<true><<<h, kRowThreads, smem, s>>>(nullptr, image, first, tmp, w, h, planes, L, r);
        else box_rows_prefix<false><<<h, kRowThreads, smem, s>>>(in, nullptr, nullptr, tmp, w, h, planes, L, r);
    } else {
        const int threads = 128;
        if (image) {
            int grid = int((size_t(w) * h + 255) / 256);
            if (grid > 148 * 32) grid = 148 * 32;
            pack_planes<<<grid, 256, 0, s>>>(image, first, const_cast<double*>(in), size_t(w) * h, L, channels);
        }
        box_rows<<<(planes * h + threads - 1) / threads, threads, 0, s>>>(in, tmp, w, h, planes, r);
    }
    const int segs = (h + kColSegment - 1) / kColSegment;
    const size_t jobs = size_t(planes) * segs * w;
    const int threads = 256;
    box_cols_segments<<<unsigned((jobs + threads - 1) / threads), threads, 0, s>>>(tmp, out, w, h, planes, r);
    return cudaGetLastError();
}

}  // namespace

int filter_launches(int width, int radius) {
    if (radius == 0) return 1;
    return width <= kRowPrefixMaxWidth ? 6 : 7;
}

size_t filter_scratch_doubles(int width, int height, int layers, int smooth) {
    const size_t n = size_t(width) * height;
    const size_t channels = size_t(layers) + (smooth ? 3 : 0);
    const size_t packed = 9 + 4 * channels, coef = 4 * channels;
    return n * (3 * packed + coef);
}

cudaError_t launch_filter(const FilterArgs& a, cudaStream_t s) {
    const int w = a.width, h = a.height, L = a.layers;
    const size_t n = size_t(w) * h;
    const int channels = L + (a.smooth ? 3 : 0);
    const int packed = 9 + 4 * channels, ncoef = 4 * channels;
    // scratch: planes | tmp | means (packed planes each) | coef (ncoef planes).
    // The second mean filter runs coef -> planes (row pass) -> tmp.
    double* planes = a.scratch;
    double* tmp = planes + size_t(packed) * n;
    double* means = tmp + size_t(packed) * n;
    double* coef = means + size_t(packed) * n;
    double* mcoef = tmp;
    const int threads = 256;
    int grid = int((n + threads - 1) / threads);
    if (grid > 148 * 32) grid = 148 * 32;
    const int identity = a.radius == 0;
    if (!identity) {
        cudaError_t e = box(planes, a.image, a.first, L, channels, tmp, means, w, h, packed, a.radius, s);
        if (e != cudaSuccess) return e;
        coefficients<<<grid, threads, 0, s>>>(means, coef, n, channels, a.eps);
        e = box(coef, nullptr, nullptr, L, channels, planes, mcoef, w, h, ncoef, a.radius, s);
        if (e != cudaSuccess) return e;
    }
    finish_targets<<<grid, threads, 0, s>>>(a.image, a.first, mcoef, a.targets, a.status, n, L, channels, a.smooth,
                                            a.plus, identity);
    return cudaGetLastError();
}

}  // namespace unb
