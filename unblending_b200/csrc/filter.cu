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
// sliding-window passes (rows, then columns), O(1) per pixel for any radius.
// The row pass gives each thread one row (its reads stream through L1); the
// column pass gives each thread one column so a warp reads 32 adjacent
// doubles per row step. All sums stay in FP64: E[I^2] - E[I]^2 cancels.
#include "solver_dispatch.hpp"

namespace unb {
namespace {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

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

// Sliding mean along rows: one thread per (plane, row).
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

// Sliding mean along columns: one thread per (plane, column).
__global__ void box_cols(const double* in, double* out, int w, int h, int planes, int r) {
    const int job = blockIdx.x * blockDim.x + threadIdx.x;
    if (job >= planes * w) return;
    const int p = job / w, x = job % w;
    const double* col = in + size_t(p) * w * h + x;
    double* o = out + size_t(p) * w * h + x;
    const double norm = double(2 * r + 1);
    double sum = double(r + 1) * col[0];
    const int hi = r < h - 1 ? r : h - 1;
    for (int y = 1; y <= hi; ++y) sum += col[size_t(y) * w];
    if (r >= h) sum += double(r - h + 1) * col[size_t(h - 1) * w];
    for (int y = 0; y < h; ++y) {
        o[size_t(y) * w] = sum / norm;
        sum += col[size_t(clampi(y + r + 1, 0, h - 1)) * w] - col[size_t(clampi(y - r, 0, h - 1)) * w];
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

void box(const double* in, double* tmp, double* out, int w, int h, int planes, int r, cudaStream_t s) {
    const int threads = 128;
    box_rows<<<(planes * h + threads - 1) / threads, threads, 0, s>>>(in, tmp, w, h, planes, r);
    box_cols<<<(planes * w + threads - 1) / threads, threads, 0, s>>>(tmp, out, w, h, planes, r);
}

}  // namespace

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
        pack_planes<<<grid, threads, 0, s>>>(a.image, a.first, planes, n, L, channels);
        box(planes, tmp, means, w, h, packed, a.radius, s);
        coefficients<<<grid, threads, 0, s>>>(means, coef, n, channels, a.eps);
        box(coef, planes, mcoef, w, h, ncoef, a.radius, s);
    }
    finish_targets<<<grid, threads, 0, s>>>(a.image, a.first, mcoef, a.targets, a.status, n, L, channels, a.smooth,
                                            a.plus, identity);
    return cudaGetLastError();
}

}  // namespace unb
