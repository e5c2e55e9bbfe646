// C ABI of the B200 unblending path: validation, device context, and the
// orchestration of upload -> (filter) -> solve -> FP64 check/re-solve ->
// download on one CUDA stream.
//
// Mirrors the reference's C layer (sdk/unblending_c.cpp:23-110) and the
// argument checks of its buffer API (unblending.cpp:505-534,590-604):
// same validation order, same error codes, output written only on success.
#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/unblending.h"
#include "../../include/unblending_b200.h"
#include "solver_dispatch.hpp"

namespace {

using namespace unb;

struct CudaFailure : std::runtime_error {
    cudaError_t code;
    explicit CudaFailure(cudaError_t c) : std::runtime_error(cudaGetErrorString(c)), code(c) {}
};
struct SolverFailure : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void ck(cudaError_t e) {
    if (e == cudaSuccess) return;
    if (e == cudaErrorMemoryAllocation) { cudaGetLastError(); throw std::bad_alloc(); }
    throw CudaFailure(e);
}

thread_local int64_t t_launches = 0;

// NVTX range over a host-side scope (a public call, or the enqueueing of one
// stage of a pass), seen by Nsight tools; without a tool attached it costs a
// null check.
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

// Grow-only device allocation.
struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    Buffer() = default;
    Buffer(const Buffer&) = delete;
    Buffer& operator=(const Buffer&) = delete;
    ~Buffer() { if (ptr) cudaFree(ptr); }
    template <class T> T* get(size_t count) {
        const size_t want = std::max<size_t>(count * sizeof(T), 256);
        if (want > bytes) {
            if (ptr) cudaFree(ptr);
            ptr = nullptr; bytes = 0;
            ck(cudaMalloc(&ptr, want));
            bytes = want;
        }
        return static_cast<T*>(ptr);
    }
};

// A batched first pass captured as a CUDA graph, with the device tables and
// scratch it refers to; replayed while the same job list comes back.
struct BatchPlan {
    std::vector<unsigned char> key;
    cudaGraphExec_t exec = nullptr;
    std::vector<std::unique_ptr<Buffer>> buffers;
    std::vector<int32_t*> counts;   // per group: [0] misses, [1] failures
    int64_t pixels = 0;
    int launches = 0;
    BatchPlan() = default;
    BatchPlan(const BatchPlan&) = delete;
    BatchPlan& operator=(const BatchPlan&) = delete;
    ~BatchPlan() { if (exec) cudaGraphExecDestroy(exec); }
    template <class T> T* alloc(size_t count) {
        buffers.push_back(std::make_unique<Buffer>());
        return buffers.back()->get<T>(count);
    }
};

// ------------------------------------------------------------ host copies --
// The host-buffer entry points copy the caller's image and first pass up and
// the results down. Page-locked host memory (cudaHostAlloc, cudaHostRegister)
// goes to the copy engine directly. From pageable memory (a plain heap
// buffer, as the reference's CLI passes) the driver would stage each copy
// through small page-locked buffers of its own, one host thread at a time,
// at a fraction of the host link's rate; such copies go instead through a
// ring of page-locked chunks owned by the device context (Staging), each
// chunk filled or drained by several host threads (CopyPool) while the copy
// engine moves the previous ones.

// Host threads that split one memcpy with the caller. One process-wide pool,
// never destroyed (its threads sleep on a condition variable and end with
// the process); concurrent calls take turns.
class CopyPool {
public:
    static CopyPool& get() {
        static CopyPool* pool = new CopyPool(helpers());
        return *pool;
    }
    void copy(void* dst, const void* src, size_t bytes) {
        std::lock_guard<std::mutex> call(call_mutex_);
        const int parts = int(threads_.size()) + 1;
        if (parts == 1 || bytes < (size_t(1) << 20)) { std::memcpy(dst, src, bytes); return; }
        {
            std::lock_guard<std::mutex> l(m_);
            job_ = Job{static_cast<char*>(dst), static_cast<const char*>(src), bytes, parts};
            pending_ = parts - 1;
            ++generation_;
        }
        wake_.notify_all();
        run_part(job_, 0);   // the caller's share
        std::unique_lock<std::mutex> l(m_);
        done_.wait(l, [this] { return pending_ == 0; });
    }

private:
    struct Job {
        char* dst = nullptr;
        const char* src = nullptr;
        size_t bytes = 0;
        int parts = 1;
    };
    // Helpers besides the caller: half the hardware threads, at most 7.
    static int helpers() {
        const unsigned hw = std::thread::hardware_concurrency();
        return int(std::min<unsigned>(7, hw > 2 ? hw / 2 - 1 : 0));
    }
    // Part k of j.parts, on 64-byte boundaries.
    static void run_part(const Job& j, int k) {
        const size_t per = (j.bytes / size_t(j.parts) + 63) & ~size_t(63);
        const size_t b = std::min(j.bytes, per * size_t(k)), e = std::min(j.bytes, b + per);
        if (e > b) std::memcpy(j.dst + b, j.src + b, e - b);
    }
    explicit CopyPool(int n) {
        for (int i = 0; i < n; ++i) threads_.emplace_back([this, i] { loop(i + 1); });
    }
    void loop(int part) {
        uint64_t seen = 0;
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> l(m_);
                wake_.wait(l, [&] { return generation_ != seen; });
                seen = generation_;
                j = job_;
            }
            run_part(j, part);
            std::lock_guard<std::mutex> l(m_);
            if (--pending_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> threads_;
    std::mutex call_mutex_, m_;
    std::condition_variable wake_, done_;
    Job job_;
    int pending_ = 0;
    uint64_t generation_ = 0;
};

// Page-locked chunks of a device context for copies of pageable buffers
// (allocated on the first such copy), and per chunk the event of the last
// copy that used it.
struct Staging {
    static constexpr size_t kChunk = size_t(8) << 20;
    static constexpr int kSlots = 4;
    unsigned char* ring = nullptr;
    cudaEvent_t done[kSlots] = {};
    Staging() = default;
    Staging(const Staging&) = delete;
    Staging& operator=(const Staging&) = delete;
    ~Staging() {
        if (ring) cudaFreeHost(ring);
        for (auto e : done)
            if (e) cudaEventDestroy(e);
    }
    unsigned char* chunk(size_t k) const { return ring + (k % kSlots) * kChunk; }
    cudaEvent_t& event(size_t k) { return done[k % kSlots]; }
    // False when the chunks cannot be had (page-locked memory is a limited
    // resource): the copy then goes to the driver directly.
    bool ensure() {
        if (ring) return true;
        for (auto& e : done)
            if (!e && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
                e = nullptr;
                cudaGetLastError();
                return false;
            }
        void* p = nullptr;
        if (cudaHostAlloc(&p, kChunk * kSlots, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        ring = static_cast<unsigned char*>(p);
        return true;
    }
};

// True for host memory the copy engine can read directly.
bool page_locked(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

// One per CUDA device: a stream, the solver's scratch, and timing events.
// Calls on the same device are serialized by `mutex`.
struct Context {
    std::unique_ptr<BatchPlan> plan;
    std::map<std::pair<int, int>, std::pair<int, int>> tuned;   // (L, precision) -> (variant, threads)
    int device = 0, sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[6] = {};
    std::mutex mutex;
    Buffer image, first, out, targets, fstatus, scratch, list_a, list_b, small, status, counters, history;
    Buffer order, order_cells;               // work-queue order of a pass (order.cu) and its counting-sort cells
    Buffer defer_list, defer_state;          // pixels deferred by an FP64 solve launch and their state
    Buffer warm, mlp_w, mlp_b;               // warm-start network on the device
    Staging staging;                         // page-locked chunks for pageable caller buffers
    std::vector<float> mlp_uploaded;         // parameters currently in mlp_w / mlp_b
    // Concurrent branches of a batched pass (one per layer-count group) and
    // the events that fork them from and join them to the call's stream.
    cudaStream_t branch[kMaxLayers] = {};
    cudaEvent_t join[kMaxLayers] = {};
    cudaEvent_t fork = nullptr;
    explicit Context(int dev) : device(dev) {
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        ck(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        for (auto& e : ev) ck(cudaEventCreate(&e));
    }
};

// Copies `bytes` of the caller's host buffer `src` to device memory `dst` on
// stream `s`. Returns once `src` may be reused (its pageable contents are in
// the staging chunks or on the device).
void upload(Context& c, void* dst, const void* src, size_t bytes, cudaStream_t s) {
    Staging& g = c.staging;
    if (bytes < Staging::kChunk || page_locked(src) || !g.ensure()) {
        ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return;
    }
    for (size_t off = 0, k = 0; off < bytes; off += Staging::kChunk, ++k) {
        const size_t len = std::min(Staging::kChunk, bytes - off);
        ck(cudaEventSynchronize(g.event(k)));   // the chunk's previous copy is done
        CopyPool::get().copy(g.chunk(k), static_cast<const unsigned char*>(src) + off, len);
        ck(cudaMemcpyAsync(static_cast<unsigned char*>(dst) + off, g.chunk(k), len, cudaMemcpyHostToDevice, s));
        ck(cudaEventRecord(g.event(k), s));
    }
}

// Copies `bytes` of device memory `src` to the caller's host buffer `dst`
// after the work already on stream `s`. Pageable `dst`: returns when `dst`
// holds them. Page-locked `dst`: returns once the copy is enqueued.
void download(Context& c, void* dst, const void* src, size_t bytes, cudaStream_t s) {
    Staging& g = c.staging;
    if (bytes < Staging::kChunk || page_locked(dst) || !g.ensure()) {
        ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        return;
    }
    const size_t chunks = (bytes + Staging::kChunk - 1) / Staging::kChunk;
    auto enqueue = [&](size_t k) {
        const size_t off = k * Staging::kChunk, len = std::min(Staging::kChunk, bytes - off);
        ck(cudaEventSynchronize(g.event(k)));   // the chunk's previous copy is done
        ck(cudaMemcpyAsync(g.chunk(k), static_cast<const unsigned char*>(src) + off, len, cudaMemcpyDeviceToHost, s));
        ck(cudaEventRecord(g.event(k), s));
    };
    for (size_t k = 0; k < std::min<size_t>(chunks, Staging::kSlots); ++k) enqueue(k);
    for (size_t k = 0; k < chunks; ++k) {
        const size_t off = k * Staging::kChunk, len = std::min(Staging::kChunk, bytes - off);
        ck(cudaEventSynchronize(g.event(k)));
        CopyPool::get().copy(static_cast<unsigned char*>(dst) + off, g.chunk(k), len);
        if (k + Staging::kSlots < chunks) enqueue(k + Staging::kSlots);
    }
}

Context& context() {
    static std::mutex registry_mutex;
    static std::map<int, std::unique_ptr<Context>> registry;
    int dev = 0;
    ck(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(registry_mutex);
    auto& slot = registry[dev];
    if (!slot) slot = std::make_unique<Context>(dev);
    return *slot;
}

// ------------------------------------------------------------- validation --
struct Spec {
    int width = 0, height = 0, layers = 0;
    size_t pixels = 0, required = 0, row_stride = 0;
    bool opaque = true, smooth = false, strict = false, plus = false, source_over = true;
};

bool symmetric_pd(const double* p) {
    // Symmetric within 1e-12 relative (Frobenius), then a Cholesky pivot test
    // (sdk/unblending_c.cpp:39-41: isApprox(transpose, 1e-12) and LLT success).
    double diff = 0, norm = 0;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            const double d = p[3 * r + c] - p[3 * c + r];
            diff += d * d;
            norm += p[3 * r + c] * p[3 * r + c];
        }
    if (!(diff <= 1e-24 * norm)) return false;
    const double l00 = p[0];
    if (!(l00 > 0)) return false;
    const double a = std::sqrt(l00), l10 = p[3] / a, l20 = p[6] / a;
    const double d1 = p[4] - l10 * l10;
    if (!(d1 > 0)) return false;
    const double b = std::sqrt(d1), l21 = (p[7] - l20 * l10) / b;
    const double d2 = p[8] - l20 * l20 - l21 * l21;
    return d2 > 0;
}

int32_t validate(const unblending_rgb_view* image, const unblending_layer* layers, size_t layer_count,
                 const unblending_options* options, const double* output, size_t output_capacity, bool refine,
                 const double* first, size_t first_size, Spec& s, bool device_mode) {
    constexpr int max_int = std::numeric_limits<int>::max();
    if (!image || !layers || !layer_count || layer_count > size_t(max_int) / 4 || image->width <= 0 ||
        image->height <= 0 || image->width > max_int / image->height)
        return UNBLENDING_INVALID_ARGUMENT;
    const size_t pixels = size_t(image->width) * size_t(image->height);
    if (pixels > (std::numeric_limits<size_t>::max() / sizeof(double)) / 4 / layer_count)
        return UNBLENDING_INVALID_ARGUMENT;
    const size_t required = 4 * pixels * layer_count;
    if (!device_mode && output_capacity < required) return UNBLENDING_BUFFER_TOO_SMALL;
    if (!output) return UNBLENDING_INVALID_ARGUMENT;

    const unblending_options defaults = UNBLENDING_OPTIONS_INIT;
    if (!options) options = &defaults;
    if (options->struct_size < sizeof(unblending_options) ||
        (options->opaque_background != 0 && options->opaque_background != 1) ||
        (options->smooth_background != 0 && options->smooth_background != 1) || options->target_concurrency < 0)
        return UNBLENDING_INVALID_ARGUMENT;
    if (options->backend != UNBLENDING_BACKEND_AUTO && options->backend != UNBLENDING_BACKEND_CUDA)
        return UNBLENDING_INVALID_ARGUMENT;   // unknown backend, or CPU: no CPU path in this library

    for (size_t l = 0; l < layer_count; ++l) {
        const auto& L = layers[l];
        if (L.blend_mode < UNBLENDING_NORMAL || L.blend_mode > UNBLENDING_LINEAR_DODGE) return UNBLENDING_INVALID_ARGUMENT;
        for (double v : L.mean) if (!std::isfinite(v)) return UNBLENDING_INVALID_ARGUMENT;
        for (double v : L.precision) if (!std::isfinite(v)) return UNBLENDING_INVALID_ARGUMENT;
        if (!symmetric_pd(L.precision)) return UNBLENDING_INVALID_ARGUMENT;
    }

    // Buffer API checks (unblending.cpp:508-534).
    if (!image->data) return UNBLENDING_INVALID_ARGUMENT;
    const size_t row_size = 3 * size_t(image->width);
    size_t stride = image->row_stride ? image->row_stride : row_size;
    if (!device_mode) {
        if (stride < row_size || image->size < row_size ||
            size_t(image->height - 1) > (image->size - row_size) / stride)
            return UNBLENDING_INVALID_ARGUMENT;
    } else {
        stride = row_size;
    }
    if (layer_count > size_t(kMaxLayers)) return UNBLENDING_INVALID_ARGUMENT;   // compiled layer counts
    if (pixels > size_t(max_int)) return UNBLENDING_INVALID_ARGUMENT;

    s.width = image->width; s.height = image->height; s.layers = int(layer_count);
    s.pixels = pixels; s.required = required; s.row_stride = stride;
    s.opaque = options->opaque_background != 0;
    s.smooth = options->smooth_background != 0;
    s.strict = options->backend == UNBLENDING_BACKEND_CUDA;
    s.plus = true; s.source_over = true;
    for (size_t l = 0; l < layer_count; ++l) {
        const auto& L = layers[l];
        s.plus &= L.comp_x == 2 && L.comp_y == 1 && L.comp_z == 1;
        s.source_over &= L.comp_x == 1 && L.comp_y == 1 && L.comp_z == 1;
    }
    if (refine) {
        // unblending.cpp:597-604
        if (!first || (!device_mode && first_size != required)) return UNBLENDING_INVALID_ARGUMENT;
        if (s.smooth && !s.opaque) return UNBLENDING_INVALID_ARGUMENT;
        if (!s.plus && !s.source_over) return UNBLENDING_INVALID_ARGUMENT;
    } else {
        s.smooth = false;   // smoothing applies to refinement only
    }
    return UNBLENDING_OK;
}

int32_t resolve_solver(const unblending_solver_options* in, unblending_solver_options& out) {
    const unblending_solver_options defaults = UNBLENDING_SOLVER_OPTIONS_INIT;
    out = defaults;
    if (!in) return UNBLENDING_OK;
    // Callers built before pixel_order was added pass the shorter layout; the
    // fields they do not have keep their defaults.
    if (in->struct_size < offsetof(unblending_solver_options, pixel_order)) return UNBLENDING_INVALID_ARGUMENT;
    std::memcpy(&out, in, std::min<size_t>(in->struct_size, sizeof(unblending_solver_options)));
    out.struct_size = sizeof(unblending_solver_options);
    if ((out.precision != UNBLENDING_PRECISION_FP32 && out.precision != UNBLENDING_PRECISION_FP64) ||
        out.starts < 1 || out.starts > 3 || !(out.epsilon > 0) || !std::isfinite(out.epsilon) || out.inner < 1 ||
        out.outer < 1 || !(out.inner_tolerance > 0) || !(out.outer_tolerance > 0) ||
        (out.resolve_misses != 0 && out.resolve_misses != 1) ||
        (out.threads_per_block != 0 && (out.threads_per_block % 32 != 0 || out.threads_per_block < 32 ||
                                        out.threads_per_block > 128)) ||
        out.kernel_variant < -1 || out.kernel_variant >= kFp32Variants || out.fp64_variant < -1 ||
        out.fp64_variant >= kFp64Variants || out.fp32_outer < 0 || out.gradient_quorum < 0 ||
        out.gradient_quorum > 8 || out.frozen_stop < 0 || (out.pixel_order != 0 && out.pixel_order != 1) ||
        out.defer_outer < 0)
        return UNBLENDING_INVALID_ARGUMENT;
    return UNBLENDING_OK;
}

// FP32 kernel variant measured on B200 (FP32 solve of the first pass /
// refinement, ms; 1024x1024, 5 layers | 6 layers with colour noise): history
// in shared memory, registers capped for 4 blocks per SM 56.6 / 62.7 |
// 133 / 116; capped for 5 blocks 54.1 / 73.6 | 158 / 181; capped for 4 blocks
// with the evaluation rolled over the layers 54.3 / 48.6 | 130 / 101.
// The refinement (pinned alphas) runs three lanes per pixel (variant 5):
// 48.8 -> 44.6 ms.
int default_fp32_variant(int L, bool refine) { (void)L; return refine ? 5 : 3; }

// FP64 kernel variant measured on B200 (1024x1024, 5 layers; re-solve of the
// FP32 misses, first pass / refinement, ms): shared history uncapped 91 / 130;
// global history with x, g, d and the evaluation's per-layer intermediates in
// shared memory (evaluation rolled over the layers), capped for 3 blocks:
// 59 / 83 (FP64 solve of every pixel: 282 / 238, against 342 / 324 uncapped).
// The refinement as 2 with three lanes per pixel (variant 5): re-solve 78.6 ->
// 66.2 ms, FP64 solve of every pixel 221 -> 191 ms.
// First passes with the cold values in the global array too (variant 3, a
// smaller shared slice for 4 blocks per SM): re-solve 60.6 -> 53.0 ms, FP64 solve
// of every pixel 292 -> 248 ms (for the refinement it gains nothing).
// The refinement with the bookkeeping rolled over the layers (variant 6; its
// smaller instruction footprint cut instruction-fetch stalls from 3.6 to 1.4
// cycles per issue): 106.5 -> 102.5 ms. The first pass keeps variant 3 (its
// rolled form ran 145 against 139 ms: more instructions, and loads of its
// global cold values no longer issued together). The refinement of 6 with its
// cold values in the global array too (variant 7, 4 blocks per SM instead of
// 3): 94.7 -> 94.0 ms with the colour-ordered queue.
int default_fp64_variant(bool refine) { return refine ? 7 : 3; }
int fp64_variant(const unblending_solver_options& so, bool refine) {
    return so.fp64_variant >= 0 ? so.fp64_variant : default_fp64_variant(refine);
}

// Bytes of a global-memory L-BFGS history array for L layers and values of
// `elem` bytes, sized for kGlobalHistoryBlocksPerSm blocks on every SM.
size_t history_lanes(int sms) { return size_t(kGlobalHistoryBlocksPerSm) * sms * kSliceStride; }
// (the history, then the cold values of the variants that keep them there,
// then the three-lane refinement's pinned-alpha gradient at x).
size_t history_bytes(int L, size_t elem, int sms) { return history_lanes(sms) * (2 * kHistory + 4) * L * elem; }

// Points `a` at a history array when the kernel variant keeps its history in
// global memory.
void attach_history(SolveArgs& a, void* array, bool fp64, int variant, int sms) {
    if (!variant_global_history(fp64, variant)) return;
    a.history = array;
    a.history_lanes = int(history_lanes(sms));
}

SolverControls controls(const unblending_solver_options& so) {
    SolverControls c;
    c.inner = so.inner; c.outer = so.outer; c.starts = so.starts;
    c.inner_tolerance = so.inner_tolerance; c.outer_tolerance = so.outer_tolerance;
    c.gradient_quorum = so.gradient_quorum;
    // Waiting for a quorum at the direction step pays in the FP64 solve of
    // every pixel (1024x1024, 5 layers: 211 -> 191 ms first pass, 203 -> 177
    // refinement) but not in the FP32 solve (50 -> 52 ms) or in the FP64
    // re-solve of the FP32 misses (44 -> 45 ms).
    c.direction_quorum = so.precision == UNBLENDING_PRECISION_FP64 ? 3 : 0;
    // FP64 solves stop a pixel once frozen_stop consecutive outer steps moved
    // neither its point nor its best point. Oracle traces of every pixel of
    // eleven images (1024x1024 five-layer, 4096-size six-layer crop, six of
    // the uneven batch, dodge/burn/soft-light stacks; both passes): with 4 such
    // steps no pixel's best point moved afterwards, so the outputs equal the
    // full schedule's, while 11-39 % of the outer steps were left out (all of
    // them steps of pixels that end unsolved, at ~66 evaluations a step). The
    // FP32 solve never freezes that way before its cap.
    c.frozen_stop = so.precision == UNBLENDING_PRECISION_FP64 ? so.frozen_stop : 0;
    return c;
}

// Controls of the FP64 re-solve behind the FP32 solve: the method's own, with
// the frozen stop (controls() sets it for the FP64 precision solve too).
SolverControls resolve_controls(const unblending_solver_options& so) {
    SolverControls c = controls(so);
    c.frozen_stop = so.frozen_stop;
    return c;
}

// Controls of the FP32 solve. When its misses are re-solved in FP64, the FP32
// solve stops after fp32_outer outer steps: a pixel still unsolved by then
// mostly never converges (92% of those run to the outer cap and fail, at
// ~1050 evaluations each against ~100 for a converging pixel), and every
// pixel stopped unconverged, whatever its best point, goes to the FP64
// re-solve, which gives it the reference method's own result. Measured on
// 1024x1024, 5 layers (ms of FP32 solve + FP64 re-solve, both passes): cap 9
// 183.7, 10 184.2, 11 187.4, 12 192.1.
SolverControls fp32_controls(const unblending_solver_options& so) {
    SolverControls c = controls(so);
    if (so.resolve_misses && so.fp32_outer > 0 && so.fp32_outer < c.outer) {
        c.outer = so.fp32_outer;
        c.cap_is_miss = 1;
    }
    return c;
}

template <class T> Models<T> make_models(const unblending_layer* layers, int L) {
    Models<T> m{};
    for (int l = 0; l < L; ++l) {
        for (int r = 0; r < 3; ++r) m.mean[l][r] = T(layers[l].mean[r]);
        for (int k = 0; k < 9; ++k) m.prec[l][k] = T(layers[l].precision[k]);
        m.mode[l] = layers[l].blend_mode;
        m.X[l] = layers[l].comp_x; m.Y[l] = layers[l].comp_y; m.Z[l] = layers[l].comp_z;
        set_blend_table(m, l, layers[l].blend_mode);
    }
    return m;
}

// ------------------------------------------------------- warm-start MLP --
constexpr int kMlpSizes[4][2] = {{kMlpHidden, kMlpIn}, {kMlpHidden, kMlpHidden}, {kMlpHidden, kMlpHidden},
                                 {kMlpOut, kMlpHidden}};

const float* mlp_weight(const unblending_mlp& m, int k) { return k == 0 ? m.w1 : k == 1 ? m.w2 : k == 2 ? m.w3 : m.w4; }
const float* mlp_bias(const unblending_mlp& m, int k) { return k == 0 ? m.b1 : k == 1 ? m.b2 : k == 2 ? m.b3 : m.b4; }
float* mlp_weight(unblending_mlp& m, int k) { return k == 0 ? m.w1 : k == 1 ? m.w2 : k == 2 ? m.w3 : m.w4; }
float* mlp_bias(unblending_mlp& m, int k) { return k == 0 ? m.b1 : k == 1 ? m.b2 : k == 2 ? m.b3 : m.b4; }

size_t mlp_weight_count() {
    size_t s = 0;
    for (auto& d : kMlpSizes) s += size_t(d[0]) * d[1];
    return s;
}
size_t mlp_bias_count() { return 3 * kMlpHidden + kMlpOut; }

bool mlp_valid(const unblending_mlp* m, int L) {
    if (!m || m->struct_size < sizeof(unblending_mlp) || m->layer_count != L) return false;
    for (int k = 0; k < 4; ++k) {
        for (int i = 0; i < kMlpSizes[k][0] * kMlpSizes[k][1]; ++i) if (!std::isfinite(mlp_weight(*m, k)[i])) return false;
        for (int i = 0; i < kMlpSizes[k][0]; ++i) if (!std::isfinite(mlp_bias(*m, k)[i])) return false;
    }
    return true;
}

// Device copy of a network (BF16 weights, FP32 biases), uploaded when it
// differs from the one already on this device.
MlpDevice upload_model(Context& c, const unblending_mlp& m, cudaStream_t s) {
    __nv_bfloat16* w = c.mlp_w.get<__nv_bfloat16>(mlp_weight_count());
    float* b = c.mlp_b.get<float>(mlp_bias_count());
    std::vector<float> flat;
    flat.reserve(mlp_weight_count() + mlp_bias_count());
    for (int k = 0; k < 4; ++k) flat.insert(flat.end(), mlp_weight(m, k), mlp_weight(m, k) + kMlpSizes[k][0] * kMlpSizes[k][1]);
    for (int k = 0; k < 4; ++k) flat.insert(flat.end(), mlp_bias(m, k), mlp_bias(m, k) + kMlpSizes[k][0]);
    if (flat != c.mlp_uploaded) {
        std::vector<__nv_bfloat16> wb(mlp_weight_count());
        for (size_t i = 0; i < wb.size(); ++i) wb[i] = __float2bfloat16(flat[i]);
        ck(cudaMemcpyAsync(w, wb.data(), wb.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice, s));
        ck(cudaMemcpyAsync(b, flat.data() + mlp_weight_count(), mlp_bias_count() * sizeof(float),
                           cudaMemcpyHostToDevice, s));
        ck(cudaStreamSynchronize(s));   // host staging vectors go out of scope
        c.mlp_uploaded = std::move(flat);
    }
    MlpDevice d;
    size_t off = 0, boff = 0;
    for (int k = 0; k < 4; ++k) {
        d.w[k] = w + off; off += size_t(kMlpSizes[k][0]) * kMlpSizes[k][1];
        d.b[k] = b + boff; boff += kMlpSizes[k][0];
    }
    return d;
}

// --------------------------------------------------------------- a pass --
struct PassIO {
    const double* image = nullptr;   // device, packed RGB
    const double* first = nullptr;   // device, refinement
    double* out = nullptr;           // device
    int32_t* status = nullptr;       // device, per pixel (context buffer when the caller passes none)
    uint32_t* counters = nullptr;    // device or null
    int first_pixel = 0, pixel_count = -1;   // the pixels solved (rows of the image); -1: all
};

struct PassResult {
    int32_t* small = nullptr;   // device: [0] misses, [1] failures after re-solve, [2] normalization failures
    unsigned long long* tally = nullptr;   // device: SolveArgs::tally of the FP64 solves, then of the FP32 solve
    int radius = 0;
};

// Totals of a pass's evaluations (PassResult::tally) into the stats.
void put_tally(unblending_stats* st, const unsigned long long* t) {
    st->fp64_values = int64_t(t[0]); st->fp64_gradients = int64_t(t[1]);
    st->fp32_values = int64_t(t[2]); st->fp32_gradients = int64_t(t[3]);
}

// Enqueues one pass on `s`. Events ev[0..3] bracket filter / solve / re-solve.
PassResult enqueue_pass(Context& c, const Spec& sp, bool refine, const unblending_layer* layers,
                        const unblending_solver_options& so, const PassIO& io, cudaStream_t s) {
    PassResult R;
    const int L = sp.layers;
    const size_t n = sp.pixels;
    // Words [0, 4) queue heads, [4, 8) counts, then 4 tally totals (64-bit):
    // FP64 values, FP64 gradients, FP32 values, FP32 gradients.
    uint32_t* queues = c.small.get<uint32_t>(8 + 8);
    int32_t* counts = reinterpret_cast<int32_t*>(queues + 4);
    R.small = counts;
    R.tally = reinterpret_cast<unsigned long long*>(queues + 8);
    ck(cudaMemsetAsync(queues, 0, (8 + 8) * sizeof(uint32_t), s));

    ck(cudaEventRecord(c.ev[0], s));
    double* targets = nullptr;
    int32_t* fstatus = nullptr;
    if (refine) {
        R.radius = so.radius >= 0 ? so.radius : 60 * std::min(sp.width, sp.height) / 1000;
        FilterArgs f;
        f.width = sp.width; f.height = sp.height; f.layers = L; f.radius = R.radius; f.eps = so.epsilon;
        f.opaque = sp.opaque; f.smooth = sp.smooth; f.plus = sp.plus;
        f.image = io.image; f.first = io.first;
        targets = c.targets.get<double>((size_t(L) + 3) * n);
        fstatus = c.fstatus.get<int32_t>(n);
        f.targets = targets; f.status = fstatus;
        f.scratch = R.radius > 0 ? c.scratch.get<double>(filter_scratch_doubles(sp.width, sp.height, L, sp.smooth)) : nullptr;
        const Range range("guided filter");
        ck(launch_filter(f, s));
        t_launches += filter_launches(sp.width, R.radius);
    }
    ck(cudaEventRecord(c.ev[1], s));

    const SolverControls ctl = controls(so), ctl32 = fp32_controls(so), ctl_re = resolve_controls(so);
    SolveArgs a;
    a.n = int(n);
    a.first_pixel = io.first_pixel; a.pixel_count = io.pixel_count;
    a.image = io.image; a.first = io.first; a.targets = targets; a.out = io.out;
    a.status = io.status; a.counters = io.counters;
    a.input_status = fstatus; a.input_failed = counts + 2;
    a.opaque = sp.opaque; a.smooth = sp.smooth;
    a.queue = queues;
    a.miss_list = c.list_a.get<int32_t>(n);
    a.miss_count = counts + 0;
    a.tally = R.tally;
    if (so.pixel_order) {
        // The solve hands out its pixels grouped by colour (order.cu).
        const int count = io.pixel_count >= 0 ? io.pixel_count : int(n);
        int32_t* order = c.order.get<int32_t>(size_t(count));
        uint32_t* cells = c.order_cells.get<uint32_t>(order_cells(count));
        const Range range("queue order");
        ck(launch_pixel_order(io.image, io.first_pixel, count, cells, order, c.sms, s));
        t_launches += 4;
        a.order = order;
    }
    if (!refine && so.warm_start) {
        // Learned start point for every pixel, then the solve from it.
        const MlpDevice dev = upload_model(c, *so.warm_start, s);
        float* warm = c.warm.get<float>(size_t(4) * L * n);
        ck(launch_mlp_infer(dev, io.image, sp.width, sp.height, L, warm, counts + 3, c.sms, s));
        ++t_launches;
        a.warm = warm;
    }
    const int threads = so.threads_per_block ? so.threads_per_block : 128;
    // One history array serves the FP32 solve and the FP64 re-solve (they run
    // one after the other on the stream).
    void* history = c.history.get<unsigned char>(history_bytes(L, sizeof(double), c.sms));
    if (so.precision == UNBLENDING_PRECISION_FP64) {
        attach_history(a, history, true, fp64_variant(so, refine), c.sms);
        const Range range(refine ? "refinement solve (fp64)" : "first-pass solve (fp64)");
        const int solved = io.pixel_count >= 0 ? io.pixel_count : int(n);
        if (so.defer_outer > 0 && solved > 0 && variant_defers(fp64_variant(so, refine), refine)) {
            // Pixels still unsolved at outer step defer_outer leave this
            // launch (up to a quarter of its pixels; the rest carry on) ...
            a.defer_outer = so.defer_outer;
            a.defer_capacity = std::max(1, solved / 4);
            a.defer_list = c.defer_list.get<int32_t>(size_t(a.defer_capacity));
            a.defer_count = reinterpret_cast<int32_t*>(queues + 3);
            a.defer_state = c.defer_state.get<double>(size_t(a.defer_capacity) * 4 * size_t(defer_words(L)));
        }
        ck(launch_solve_fp64(L, refine, fp64_variant(so, refine), make_models<double>(layers, L), ctl, a, threads,
                             c.sms, s));
        ++t_launches;
        if (a.defer_outer > 0) {
            // ... and are resumed together by the next launch (queue 2), from
            // the state they left with: each pixel takes the same steps.
            SolveArgs d = a;
            d.defer_outer = 0;
            d.resume = 1;
            d.list = a.defer_list; d.list_count = a.defer_count; d.list_limit = a.defer_capacity;
            d.order = nullptr;
            d.queue = queues + 2;
            d.input_status = nullptr; d.input_failed = nullptr;
            ck(launch_solve_fp64(L, refine, fp64_variant(so, refine), make_models<double>(layers, L), ctl, d, threads,
                                 c.sms, s));
            ++t_launches;
            a.defer_outer = 0;
        }
        ck(cudaEventRecord(c.ev[2], s));
        if (a.warm) {
            // Pixels that the learned start leaves unsolved get the plain
            // solve from the reference's start.
            SolveArgs b = a;
            b.list = a.miss_list; b.list_count = counts + 0;
            b.miss_list = c.list_b.get<int32_t>(n); b.miss_count = counts + 1;
            b.queue = queues + 1;
            b.input_status = nullptr; b.input_failed = nullptr;
            b.warm = nullptr;
            ck(launch_solve_fp64(L, refine, fp64_variant(so, refine), make_models<double>(layers, L), ctl, b, threads,
                                 c.sms, s));
            ++t_launches;
        } else {
            ck(cudaMemcpyAsync(counts + 1, counts + 0, sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
        }
    } else {
        const int variant = so.kernel_variant >= 0 ? so.kernel_variant : default_fp32_variant(L, refine);
        attach_history(a, history, false, variant, c.sms);
        a.tally = R.tally + 2;
        const Range range(refine ? "refinement solve (fp32 + fp64 re-solve)" : "first-pass solve (fp32 + fp64 re-solve)");
        ck(launch_solve_fp32(L, refine, variant, make_models<float>(layers, L), ctl32, a, threads, c.sms, s));
        ++t_launches;
        ck(cudaEventRecord(c.ev[2], s));
        if (so.resolve_misses) {
            // Misses of a learned start first fall back to the plain FP32
            // solve from the reference's start (queue 2, its misses counted in
            // slot 3 of the queue words); what that misses, and the plain
            // solve's own misses, get the FP64 re-solve from the reference's
            // start.
            int32_t* list_a = a.miss_list;
            int32_t* list_b = c.list_b.get<int32_t>(n);
            int32_t* fp64_list = list_a;
            int32_t* fp64_count = counts + 0;
            int32_t* fp64_misses = list_b;
            if (a.warm) {
                SolveArgs w = a;
                w.list = list_a; w.list_count = counts + 0;
                w.miss_list = list_b; w.miss_count = reinterpret_cast<int32_t*>(queues + 3);
                w.queue = queues + 2;
                w.input_status = nullptr; w.input_failed = nullptr;
                w.warm = nullptr;
                ck(launch_solve_fp32(L, refine, variant, make_models<float>(layers, L), ctl32, w, threads, c.sms, s));
                ++t_launches;
                fp64_list = list_b; fp64_count = w.miss_count; fp64_misses = list_a;
            }
            SolveArgs b = a;
            b.list = fp64_list; b.list_count = fp64_count;
            b.miss_list = fp64_misses;
            b.miss_count = counts + 1;
            b.queue = queues + 1;
            b.input_status = nullptr; b.input_failed = nullptr;
            b.warm = nullptr;   // the reference's (cold) start
            b.history = nullptr; b.history_lanes = 0;
            b.tally = R.tally;
            attach_history(b, history, true, fp64_variant(so, refine), c.sms);
            ck(launch_solve_fp64(L, refine, fp64_variant(so, refine), make_models<double>(layers, L), ctl_re, b,
                                 threads, c.sms, s));
            ++t_launches;
        } else {
            ck(cudaMemcpyAsync(counts + 1, counts + 0, sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
        }
    }
    ck(cudaEventRecord(c.ev[3], s));
    return R;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    return cudaEventElapsedTime(&ms, a, b) == cudaSuccess ? ms : 0.f;
}

// Host-side fault injection (no GPU fault): UNBLENDING_FAULT=alloc makes the
// call fail as a device allocation does (ck's std::bad_alloc),
// UNBLENDING_FAULT=launch as a failed kernel launch does (ck's CudaFailure),
// before its first CUDA call; the call then returns UNBLENDING_OUT_OF_MEMORY /
// UNBLENDING_CUDA_ERROR without touching the device or the caller's output
// (sdk/unblending_c.cpp:87-91 maps exceptions to these codes).
void injected_fault() {
    const char* f = std::getenv("UNBLENDING_FAULT");
    if (!f) return;
    if (std::strcmp(f, "alloc") == 0) throw std::bad_alloc();
    if (std::strcmp(f, "launch") == 0) throw CudaFailure(cudaErrorLaunchFailure);
}

template <class F> int32_t guarded(F&& f) {
    try {
        injected_fault();
        return f();
    } catch (const std::bad_alloc&) { return UNBLENDING_OUT_OF_MEMORY; }
    catch (const CudaFailure& e) { cudaGetLastError(); return UNBLENDING_CUDA_ERROR; }
    catch (const SolverFailure&) { return UNBLENDING_CUDA_ERROR; }
    catch (const std::invalid_argument&) { return UNBLENDING_INVALID_ARGUMENT; }
    catch (const std::length_error&) { return UNBLENDING_INVALID_ARGUMENT; }
    catch (...) { return UNBLENDING_SOLVER_ERROR; }
}

// Host-buffer call: upload, pass, check, download.
int32_t host_call(const unblending_rgb_view* image, const unblending_layer* layers, size_t layer_count,
                  const double* first, size_t first_size, const unblending_options* options,
                  const unblending_solver_options* solver, double* output, size_t output_capacity, int32_t* status,
                  uint32_t* counters, unblending_stats* stats, bool refine) {
    t_launches = 0;
    const Range range(refine ? "unblending_refine" : "unblending_unmix");
    Spec sp;
    int32_t rc = validate(image, layers, layer_count, options, output, output_capacity, refine, first, first_size, sp,
                          false);
    if (rc != UNBLENDING_OK) return rc;
    unblending_solver_options so;
    if ((rc = resolve_solver(solver, so)) != UNBLENDING_OK) return rc;
    if (stats && stats->struct_size < sizeof(unblending_stats)) return UNBLENDING_INVALID_ARGUMENT;
    if (refine) so.warm_start = nullptr;   // the learned start seeds the first pass only
    if (so.warm_start && !mlp_valid(so.warm_start, sp.layers)) return UNBLENDING_INVALID_ARGUMENT;
    return guarded([&]() -> int32_t {
        Context& c = context();
        std::lock_guard<std::mutex> lock(c.mutex);
        cudaStream_t s = c.stream;
        const size_t n = sp.pixels, L = size_t(sp.layers);
        PassIO io;
        double* d_image = c.image.get<double>(3 * n);
        cudaEvent_t t0, t1;
        ck(cudaEventCreate(&t0)); ck(cudaEventCreate(&t1));
        struct EvGuard { cudaEvent_t a, b; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); } } guard{t0, t1};
        ck(cudaEventRecord(t0, s));
        const size_t row = 3 * size_t(sp.width);
        if (sp.row_stride == row)
            upload(c, d_image, image->data, 3 * n * sizeof(double), s);
        else
            ck(cudaMemcpy2DAsync(d_image, row * sizeof(double), image->data, sp.row_stride * sizeof(double),
                                 row * sizeof(double), size_t(sp.height), cudaMemcpyHostToDevice, s));
        io.image = d_image;
        if (refine) {
            double* d_first = c.first.get<double>(4 * L * n);
            upload(c, d_first, first, 4 * L * n * sizeof(double), s);
            io.first = d_first;
        }
        io.out = c.out.get<double>(4 * L * n);
        io.status = c.status.get<int32_t>(n);
        io.counters = counters ? c.counters.get<uint32_t>(5 * n) : nullptr;
        PassResult R = enqueue_pass(c, sp, refine, layers, so, io, s);
        int32_t counts[3] = {0, 0, 0};
        unsigned long long tally[4] = {};
        ck(cudaMemcpyAsync(counts, R.small, sizeof(counts), cudaMemcpyDeviceToHost, s));
        ck(cudaMemcpyAsync(tally, R.tally, sizeof(tally), cudaMemcpyDeviceToHost, s));
        ck(cudaStreamSynchronize(s));
        if (sp.strict && (counts[1] > 0 || counts[2] > 0)) throw SolverFailure("pixels miss the feasibility tolerance");
        ck(cudaEventRecord(c.ev[4], s));
        download(c, output, io.out, 4 * L * n * sizeof(double), s);
        if (status) download(c, status, io.status, n * sizeof(int32_t), s);
        if (counters) download(c, counters, io.counters, 5 * n * sizeof(uint32_t), s);
        ck(cudaEventRecord(t1, s));
        ck(cudaStreamSynchronize(s));
        ck(cudaGetLastError());
        if (stats) {
            stats->radius = R.radius;
            stats->pixels = int64_t(n);
            stats->misses = counts[0];
            stats->failed = counts[1];
            stats->normalization_failed = counts[2];
            stats->ms_upload = elapsed(t0, c.ev[0]);
            stats->ms_filter = elapsed(c.ev[0], c.ev[1]);
            stats->ms_solve = elapsed(c.ev[1], c.ev[2]);
            stats->ms_resolve = elapsed(c.ev[2], c.ev[3]);
            stats->ms_download = elapsed(c.ev[4], t1);
            stats->ms_total = elapsed(t0, t1);
            put_tally(stats, tally);
        }
        return UNBLENDING_OK;
    });
}

int32_t device_call(int32_t width, int32_t height, const double* image, const unblending_layer* layers,
                    size_t layer_count, const double* first, const unblending_options* options,
                    const unblending_solver_options* solver, double* output, int32_t* status, uint32_t* counters,
                    void* stream, unblending_stats* stats, bool refine, int32_t row_begin = 0,
                    int32_t row_end = -1) {
    t_launches = 0;
    unblending_rgb_view view{image, 0, width, height, 0};
    const Range range(refine ? "unblending_refine_device" : "unblending_unmix_device");
    Spec sp;
    int32_t rc = validate(&view, layers, layer_count, options, output, 0, refine, first, 0, sp, true);
    if (rc != UNBLENDING_OK) return rc;
    if (row_end < 0) row_end = height;
    if (row_begin < 0 || row_begin > row_end || row_end > height) return UNBLENDING_INVALID_ARGUMENT;
    unblending_solver_options so;
    if ((rc = resolve_solver(solver, so)) != UNBLENDING_OK) return rc;
    if (stats && stats->struct_size < sizeof(unblending_stats)) return UNBLENDING_INVALID_ARGUMENT;
    if (refine) so.warm_start = nullptr;   // the learned start seeds the first pass only
    if (so.warm_start && !mlp_valid(so.warm_start, sp.layers)) return UNBLENDING_INVALID_ARGUMENT;
    return guarded([&]() -> int32_t {
        Context& c = context();
        std::lock_guard<std::mutex> lock(c.mutex);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c.stream;
        PassIO io;
        io.image = image; io.first = first; io.out = output;
        if (refine && first == output && so.precision == UNBLENDING_PRECISION_FP32 && so.resolve_misses) {
            // The FP64 re-solve reads the first pass of pixels the FP32 solve
            // has already overwritten: keep a private copy.
            double* copy = c.first.get<double>(4 * size_t(sp.layers) * sp.pixels);
            ck(cudaMemcpyAsync(copy, first, 4 * size_t(sp.layers) * sp.pixels * sizeof(double),
                               cudaMemcpyDeviceToDevice, s));
            io.first = copy;
        }
        io.status = status ? status : c.status.get<int32_t>(sp.pixels);
        io.counters = counters;
        io.first_pixel = row_begin * width;
        io.pixel_count = (row_end - row_begin) * width;
        PassResult R = enqueue_pass(c, sp, refine, layers, so, io, s);
        if (stats) {
            int32_t counts[3] = {0, 0, 0};
            unsigned long long tally[4] = {};
            ck(cudaMemcpyAsync(counts, R.small, sizeof(counts), cudaMemcpyDeviceToHost, s));
            ck(cudaMemcpyAsync(tally, R.tally, sizeof(tally), cudaMemcpyDeviceToHost, s));
            ck(cudaStreamSynchronize(s));
            stats->radius = R.radius;
            stats->pixels = int64_t(row_end - row_begin) * width;
            stats->misses = counts[0];
            stats->failed = counts[1];
            stats->normalization_failed = counts[2];
            stats->ms_upload = 0;
            stats->ms_filter = elapsed(c.ev[0], c.ev[1]);
            stats->ms_solve = elapsed(c.ev[1], c.ev[2]);
            stats->ms_resolve = elapsed(c.ev[2], c.ev[3]);
            stats->ms_download = 0;
            stats->ms_total = elapsed(c.ev[0], c.ev[3]);
            put_tally(stats, tally);
            if (sp.strict && (counts[1] > 0 || counts[2] > 0)) throw SolverFailure("pixels miss the feasibility tolerance");
        }
        ck(cudaPeekAtLastError());
        return UNBLENDING_OK;
    });
}

}  // namespace

extern "C" {

uint32_t unblending_abi_version(void) { return UNBLENDING_ABI_VERSION; }

int32_t unblending_unmix(const unblending_rgb_view* image, const unblending_layer* layers, size_t layer_count,
                         const unblending_options* options, double* output, size_t output_capacity) {
    return host_call(image, layers, layer_count, nullptr, 0, options, nullptr, output, output_capacity, nullptr,
                     nullptr, nullptr, false);
}

int32_t unblending_refine(const unblending_rgb_view* image, const unblending_layer* layers, size_t layer_count,
                          const double* first_pass, size_t first_pass_size, const unblending_options* options,
                          double* output, size_t output_capacity) {
    return host_call(image, layers, layer_count, first_pass, first_pass_size, options, nullptr, output,
                     output_capacity, nullptr, nullptr, nullptr, true);
}

int32_t unblending_unmix_ex(const unblending_rgb_view* image, const unblending_layer* layers, size_t layer_count,
                            const unblending_options* options, const unblending_solver_options* solver,
                            double* output, size_t output_capacity, int32_t* status, uint32_t* counters,
                            unblending_stats* stats) {
    return host_call(image, layers, layer_count, nullptr, 0, options, solver, output, output_capacity, status,
                     counters, stats, false);
}

int32_t unblending_refine_ex(const unblending_rgb_view* image, const unblending_layer* layers, size_t layer_count,
                             const double* first_pass, size_t first_pass_size, const unblending_options* options,
                             const unblending_solver_options* solver, double* output, size_t output_capacity,
                             int32_t* status, uint32_t* counters, unblending_stats* stats) {
    return host_call(image, layers, layer_count, first_pass, first_pass_size, options, solver, output,
                     output_capacity, status, counters, stats, true);
}

int32_t unblending_unmix_device(int32_t width, int32_t height, const double* image, const unblending_layer* layers,
                                size_t layer_count, const unblending_options* options,
                                const unblending_solver_options* solver, double* output, int32_t* status,
                                uint32_t* counters, void* stream, unblending_stats* stats) {
    return device_call(width, height, image, layers, layer_count, nullptr, options, solver, output, status, counters,
                       stream, stats, false);
}

int32_t unblending_refine_device(int32_t width, int32_t height, const double* image, const unblending_layer* layers,
                                 size_t layer_count, const double* first_pass, const unblending_options* options,
                                 const unblending_solver_options* solver, double* output, int32_t* status,
                                 uint32_t* counters, void* stream, unblending_stats* stats) {
    return device_call(width, height, image, layers, layer_count, first_pass, options, solver, output, status,
                       counters, stream, stats, true);
}

int32_t unblending_unmix_device_rows(int32_t width, int32_t height, const double* image,
                                     const unblending_layer* layers, size_t layer_count,
                                     const unblending_options* options, const unblending_solver_options* solver,
                                     double* output, int32_t* status, uint32_t* counters, int32_t row_begin,
                                     int32_t row_end, void* stream, unblending_stats* stats) {
    if (row_end < 0) return UNBLENDING_INVALID_ARGUMENT;   // (device_call reads -1 as "every row")
    return device_call(width, height, image, layers, layer_count, nullptr, options, solver, output, status, counters,
                       stream, stats, false, row_begin, row_end);
}

int32_t unblending_refine_device_rows(int32_t width, int32_t height, const double* image,
                                      const unblending_layer* layers, size_t layer_count, const double* first_pass,
                                      const unblending_options* options, const unblending_solver_options* solver,
                                      double* output, int32_t* status, uint32_t* counters, int32_t row_begin,
                                      int32_t row_end, void* stream, unblending_stats* stats) {
    if (row_end < 0) return UNBLENDING_INVALID_ARGUMENT;   // (device_call reads -1 as "every row")
    return device_call(width, height, image, layers, layer_count, first_pass, options, solver, output, status,
                       counters, stream, stats, true, row_begin, row_end);
}

int64_t unblending_last_launch_count(void) { return t_launches; }

int32_t unblending_unmix_batch_device(const unblending_image_job* jobs, int32_t count, const unblending_options* options,
                                      const unblending_solver_options* solver, void* stream, unblending_stats* stats) {
    t_launches = 0;
    const Range range("unblending_unmix_batch_device");
    if (!jobs || count < 1) return UNBLENDING_INVALID_ARGUMENT;
    if (stats && stats->struct_size < sizeof(unblending_stats)) return UNBLENDING_INVALID_ARGUMENT;
    unblending_solver_options so;
    int32_t rc = resolve_solver(solver, so);
    if (rc != UNBLENDING_OK) return rc;
    std::vector<Spec> specs(count);
    std::map<int, std::vector<int>> groups;   // layer count -> jobs
    std::map<int, const unblending_mlp*> group_model;
    for (int k = 0; k < count; ++k) {
        const auto& J = jobs[k];
        unblending_rgb_view view{J.image, 0, J.width, J.height, 0};
        if (J.layer_count < 1) return UNBLENDING_INVALID_ARGUMENT;
        rc = validate(&view, J.layers, size_t(J.layer_count), options, J.output, 0, false, nullptr, 0, specs[k], true);
        if (rc != UNBLENDING_OK) return rc;
        if (J.warm_start) {
            if (!mlp_valid(J.warm_start, J.layer_count)) return UNBLENDING_INVALID_ARGUMENT;
            auto it = group_model.find(J.layer_count);
            // One network per layer count within a batch.
            if (it != group_model.end() && it->second != J.warm_start) return UNBLENDING_INVALID_ARGUMENT;
            group_model[J.layer_count] = J.warm_start;
        }
        groups[J.layer_count].push_back(k);
    }
    // Plan key: everything the captured graph depends on.
    std::vector<unsigned char> key;
    auto put = [&](const void* p, size_t bytes) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        key.insert(key.end(), b, b + bytes);
    };
    put(&count, sizeof(count));
    put(&stream, sizeof(stream));
    put(&so, offsetof(unblending_solver_options, warm_start));
    put(&so.fp64_variant, sizeof(so.fp64_variant)); put(&so.fp32_outer, sizeof(so.fp32_outer));
    put(&so.gradient_quorum, sizeof(so.gradient_quorum));
    put(&so.frozen_stop, sizeof(so.frozen_stop));
    put(&so.pixel_order, sizeof(so.pixel_order));
    put(&so.defer_outer, sizeof(so.defer_outer));
    for (int k = 0; k < count; ++k) {
        const auto& J = jobs[k];
        put(&J.width, sizeof(J.width)); put(&J.height, sizeof(J.height));
        put(&J.image, sizeof(J.image)); put(&J.output, sizeof(J.output)); put(&J.status, sizeof(J.status));
        put(&J.layer_count, sizeof(J.layer_count));
        put(J.layers, sizeof(unblending_layer) * size_t(J.layer_count));
        const bool warm = J.warm_start != nullptr;
        put(&warm, sizeof(warm));
        if (warm) put(J.warm_start, sizeof(unblending_mlp));
    }
    return guarded([&]() -> int32_t {
        Context& c = context();
        std::lock_guard<std::mutex> lock(c.mutex);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c.stream;
        if (!c.plan || c.plan->key != key) {
            c.plan.reset();
            auto plan = std::make_unique<BatchPlan>();
            plan->key = key;
            const SolverControls ctl = controls(so), ctl32 = fp32_controls(so), ctl_re = resolve_controls(so);
            struct Group {
                int L;
                SolveArgs fp, mid, re;   // first solve (warm where given), FP32 re-solve of its misses from
                                         // the reference start (groups with a learned start), FP64 re-solve
                uint32_t* queues;
                int32_t* counts;
                std::vector<std::pair<int, float*>> infer;   // job, warm slice
                MlpDevice net;
                int variant = 0, threads = 128;
                int64_t total = 0;
                int32_t* order = nullptr;   // colour order of the group's queue (pixel_order)
                uint32_t* order_cells = nullptr;
            };
            std::vector<Group> gs;
            for (auto& [L, members] : groups) {
                Group G;
                G.L = L;
                std::vector<BatchJob> table, cold;
                std::vector<Models<float>> m32;
                std::vector<Models<double>> m64;
                int64_t off = 0;
                const unblending_mlp* net = group_model.count(L) ? group_model[L] : nullptr;
                float* warm = nullptr;
                int64_t total = 0;
                for (int k : members) total += int64_t(specs[k].pixels);
                G.total = total;
                if (net) warm = plan->alloc<float>(size_t(total) * 4 * L);
                for (int k : members) {
                    const auto& J = jobs[k];
                    BatchJob b;
                    b.image = J.image; b.out = J.output; b.status = J.status;
                    b.offset = off; b.n = int64_t(specs[k].pixels); b.model = int32_t(table.size());
                    b.warm = nullptr;
                    cold.push_back(b);
                    if (J.warm_start) {
                        b.warm = warm + off * 4 * L;
                        G.infer.emplace_back(k, const_cast<float*>(b.warm));
                    }
                    table.push_back(b);
                    m32.push_back(make_models<float>(J.layers, L));
                    m64.push_back(make_models<double>(J.layers, L));
                    off += b.n;
                }
                if (net) {
                    // The group's own device copy of its network (the graph keeps referring to it).
                    const MlpDevice shared = upload_model(c, *net, s);
                    __nv_bfloat16* w = plan->alloc<__nv_bfloat16>(mlp_weight_count());
                    float* bb = plan->alloc<float>(mlp_bias_count());
                    ck(cudaMemcpyAsync(w, shared.w[0], mlp_weight_count() * sizeof(__nv_bfloat16),
                                       cudaMemcpyDeviceToDevice, s));
                    ck(cudaMemcpyAsync(bb, shared.b[0], mlp_bias_count() * sizeof(float), cudaMemcpyDeviceToDevice, s));
                    for (int q = 0; q < 4; ++q) {
                        G.net.w[q] = w + (shared.w[q] - shared.w[0]);
                        G.net.b[q] = bb + (shared.b[q] - shared.b[0]);
                    }
                }
                BatchJob* d_table = plan->alloc<BatchJob>(2 * table.size());
                Models<float>* d_m32 = plan->alloc<Models<float>>(m32.size());
                Models<double>* d_m64 = plan->alloc<Models<double>>(m64.size());
                ck(cudaMemcpyAsync(d_table, table.data(), table.size() * sizeof(BatchJob), cudaMemcpyHostToDevice, s));
                ck(cudaMemcpyAsync(d_table + table.size(), cold.data(), cold.size() * sizeof(BatchJob),
                                   cudaMemcpyHostToDevice, s));
                ck(cudaMemcpyAsync(d_m32, m32.data(), m32.size() * sizeof(Models<float>), cudaMemcpyHostToDevice, s));
                ck(cudaMemcpyAsync(d_m64, m64.data(), m64.size() * sizeof(Models<double>), cudaMemcpyHostToDevice, s));
                ck(cudaStreamSynchronize(s));   // host tables go out of scope
                G.queues = plan->alloc<uint32_t>(8);
                G.counts = reinterpret_cast<int32_t*>(G.queues + 4);
                int32_t* lists = plan->alloc<int32_t>(2 * size_t(total));
                if (so.pixel_order) {
                    G.order = plan->alloc<int32_t>(size_t(total));
                    G.order_cells = plan->alloc<uint32_t>(order_cells(int(total)));
                }
                SolveArgs& a = G.fp;
                a.n = int(total);
                a.jobs = d_table; a.job_count = int(table.size());
                a.opaque = specs[members[0]].opaque; a.smooth = 0;
                a.queue = G.queues;
                a.miss_list = lists; a.miss_count = G.counts + 0;
                a.order = G.order;
                SolveArgs& b = G.re;
                b = a;
                b.order = nullptr;
                b.jobs = d_table + table.size();
                b.models = d_m64;
                b.list = lists; b.list_count = G.counts + 0;
                b.miss_list = lists + total; b.miss_count = G.counts + 1;
                b.queue = G.queues + 1;
                if (!G.infer.empty() && so.precision != UNBLENDING_PRECISION_FP64) {
                    // As the single-image pass: the learned start's misses get the
                    // plain FP32 solve first (cold jobs of the group repeat theirs,
                    // with the same result), its misses the FP64 re-solve.
                    SolveArgs& w = G.mid;
                    w = a;
                    w.order = nullptr;
                    w.jobs = d_table + table.size();
                    w.models = d_m32;
                    w.list = lists; w.list_count = G.counts + 0;
                    w.miss_list = lists + total; w.miss_count = reinterpret_cast<int32_t*>(G.queues + 3);
                    w.queue = G.queues + 2;
                    b.list = lists + total; b.list_count = w.miss_count;
                    b.miss_list = lists;
                }
                a.models = so.precision == UNBLENDING_PRECISION_FP64 ? static_cast<const void*>(d_m64) : d_m32;
                // FP64: the solve's misses are the group's failures, unless a
                // learned start leaves them to the plain solve (G.re, as the
                // single-image pass does).
                if (so.precision == UNBLENDING_PRECISION_FP64 && G.infer.empty()) a.miss_count = G.counts + 1;
                plan->counts.push_back(G.counts);
                plan->pixels += total;
                void* history = plan->alloc<unsigned char>(history_bytes(L, sizeof(double), c.sms));
                // Autotuner: time each FP32 kernel variant / block size on a
                // sample of this group's pixels spread over its images.
                const auto tkey = std::make_pair(L, so.precision);
                if (so.precision == UNBLENDING_PRECISION_FP32 && so.threads_per_block == 0 && so.kernel_variant < 0) {
                    if (!c.tuned.count(tkey)) {
                        const int S = int(std::min<int64_t>(total, 8192));
                        std::vector<int32_t> sample(S);
                        for (int q = 0; q < S; ++q) sample[q] = int32_t(int64_t(q) * total / S);
                        int32_t* d_sample = plan->alloc<int32_t>(S);
                        int32_t* d_count = plan->alloc<int32_t>(1);
                        ck(cudaMemcpyAsync(d_sample, sample.data(), S * sizeof(int32_t), cudaMemcpyHostToDevice, s));
                        ck(cudaMemcpyAsync(d_count, &S, sizeof(int32_t), cudaMemcpyHostToDevice, s));
                        const std::pair<int, int> candidates[4] = {{3, 128}, {1, 128}, {2, 128}, {3, 64}};
                        float best_ms = 1e30f;
                        std::pair<int, int> best = candidates[0];
                        for (const auto& cand : candidates) {
                            SolveArgs t = a;
                            t.jobs = d_table + table.size();   // reference start: the network has not run yet
                            t.list = d_sample; t.list_count = d_count;
                            t.miss_list = nullptr; t.status = nullptr;
                            attach_history(t, history, false, cand.first, c.sms);
                            ck(cudaMemsetAsync(G.queues, 0, 8 * sizeof(uint32_t), s));
                            ck(cudaEventRecord(c.ev[4], s));
                            ck(launch_solve_batch_fp32(L, cand.first, ctl32, t, cand.second, c.sms, s));
                            ck(cudaEventRecord(c.ev[5], s));
                            ck(cudaEventSynchronize(c.ev[5]));
                            const float ms = elapsed(c.ev[4], c.ev[5]);
                            if (ms < best_ms) { best_ms = ms; best = cand; }
                        }
                        c.tuned[tkey] = best;
                    }
                    G.variant = c.tuned[tkey].first;
                    G.threads = c.tuned[tkey].second;
                } else {
                    G.variant = so.kernel_variant >= 0 ? so.kernel_variant : default_fp32_variant(L, false);
                    G.threads = so.threads_per_block ? so.threads_per_block : 128;
                }
                if (so.precision == UNBLENDING_PRECISION_FP64) attach_history(a, history, true, fp64_variant(so, false), c.sms);
                else attach_history(a, history, false, G.variant, c.sms);
                attach_history(G.mid, history, false, G.variant, c.sms);
                attach_history(b, history, true, fp64_variant(so, false), c.sms);
                gs.push_back(G);
            }
            // Capture every group's work into one graph, each group on its own
            // branch: the groups' persistent launches run back to back on the
            // GPU, the next group's blocks filling the SMs that the previous
            // group's tail frees. (One kernel over all layer counts was built
            // and measured twice: with every solver inlined, its single
            // register allocation spilled 0.6-1.6 KB of stack per thread; with
            // each count's solver out of line, it ran 4.45 against 6.52 Mpx/s
            // on a 64-image batch, its one shared-memory size set by the
            // largest layer count holding every group's occupancy down.)
            if (!c.fork) {
                ck(cudaEventCreateWithFlags(&c.fork, cudaEventDisableTiming));
                for (int q = 0; q < kMaxLayers; ++q) {
                    ck(cudaStreamCreateWithFlags(&c.branch[q], cudaStreamNonBlocking));
                    ck(cudaEventCreateWithFlags(&c.join[q], cudaEventDisableTiming));
                }
            }
            cudaGraph_t graph = nullptr;
            ck(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
            int launches = 0;
            try {
                ck(cudaEventRecord(c.fork, s));
                for (size_t gi = 0; gi < gs.size(); ++gi) {
                    auto& G = gs[gi];
                    cudaStream_t s = c.branch[gi];   // this group's branch (shadows the call's stream)
                    ck(cudaStreamWaitEvent(s, c.fork, 0));
                    ck(cudaMemsetAsync(G.queues, 0, 8 * sizeof(uint32_t), s));
                    if (G.order) {
                        // The group's queue grouped by colour (order.cu).
                        ck(launch_group_order(G.fp.jobs, G.fp.job_count, int(G.total), G.order_cells, G.order, c.sms,
                                              s));
                        launches += 4;
                    }
                    for (auto& [k, w] : G.infer) {
                        ck(launch_mlp_infer(G.net, jobs[k].image, jobs[k].width, jobs[k].height, G.L, w, G.counts + 3,
                                            c.sms, s));
                        ++launches;
                    }
                    if (so.precision == UNBLENDING_PRECISION_FP64) {
                        ck(launch_solve_batch_fp64(G.L, fp64_variant(so, false), ctl, G.fp, 128, c.sms, s));
                        ++launches;
                        if (!G.infer.empty()) {
                            ck(launch_solve_batch_fp64(G.L, fp64_variant(so, false), ctl, G.re, 128, c.sms, s));
                            ++launches;
                        }
                    } else {
                        ck(launch_solve_batch_fp32(G.L, G.variant, ctl32, G.fp, G.threads, c.sms, s));
                        ++launches;
                        if (so.resolve_misses && !G.infer.empty()) {
                            ck(launch_solve_batch_fp32(G.L, G.variant, ctl32, G.mid, G.threads, c.sms, s));
                            ++launches;
                        }
                        if (so.resolve_misses) {
                            ck(launch_solve_batch_fp64(G.L, fp64_variant(so, false), ctl_re, G.re, 128, c.sms, s));
                            ++launches;
                        } else {
                            ck(cudaMemcpyAsync(G.counts + 1, G.counts, sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
                        }
                    }
                    ck(cudaEventRecord(c.join[gi], s));
                }
                for (size_t gi = 0; gi < gs.size(); ++gi) ck(cudaStreamWaitEvent(s, c.join[gi], 0));
            } catch (...) {
                cudaStreamEndCapture(s, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            ck(cudaStreamEndCapture(s, &graph));
            cudaError_t e = cudaGraphInstantiate(&plan->exec, graph, 0);
            cudaGraphDestroy(graph);
            ck(e);
            plan->launches = launches;
            c.plan = std::move(plan);
        }
        BatchPlan& P = *c.plan;
        ck(cudaEventRecord(c.ev[0], s));
        ck(cudaGraphLaunch(P.exec, s));
        ck(cudaEventRecord(c.ev[1], s));
        t_launches = P.launches;
        if (stats) {
            int64_t misses = 0, failed = 0;
            for (int32_t* cnt : P.counts) {
                int32_t h[2];
                ck(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s));
                ck(cudaStreamSynchronize(s));
                misses += h[0]; failed += h[1];
            }
            *stats = unblending_stats{};
            stats->struct_size = sizeof(unblending_stats);
            stats->pixels = P.pixels;
            stats->misses = misses; stats->failed = failed;
            stats->ms_solve = elapsed(c.ev[0], c.ev[1]);
            stats->ms_total = stats->ms_solve;
        }
        ck(cudaPeekAtLastError());
        return UNBLENDING_OK;
    });
}

int32_t unblending_mlp_predict_device(const unblending_mlp* model, int32_t width, int32_t height, const double* image,
                                      float* out, void* stream) {
    t_launches = 0;
    if (!model || !image || !out || width <= 0 || height <= 0 || width > std::numeric_limits<int>::max() / height)
        return UNBLENDING_INVALID_ARGUMENT;
    if (model->layer_count < 1 || model->layer_count > kMaxLayers || !mlp_valid(model, model->layer_count))
        return UNBLENDING_INVALID_ARGUMENT;
    return guarded([&]() -> int32_t {
        Context& c = context();
        std::lock_guard<std::mutex> lock(c.mutex);
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c.stream;
        const MlpDevice dev = upload_model(c, *model, s);
        int32_t* err = c.small.get<int32_t>(8) + 7;
        ck(cudaMemsetAsync(err, 0, sizeof(int32_t), s));
        ck(launch_mlp_infer(dev, image, width, height, model->layer_count, out, err, c.sms, s));
        ++t_launches;
        int32_t failed = 0;
        ck(cudaMemcpyAsync(&failed, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        ck(cudaStreamSynchronize(s));
        if (failed) throw CudaFailure(cudaErrorLaunchTimeout);
        return UNBLENDING_OK;
    });
}

int32_t unblending_mlp_loss_grad_device(const unblending_mlp* model, int32_t count, const float* features,
                                        const float* targets, unblending_mlp* gradient) {
    t_launches = 0;
    if (!model || !features || !targets || !gradient || count < 1 || gradient->struct_size < sizeof(unblending_mlp))
        return UNBLENDING_INVALID_ARGUMENT;
    if (model->layer_count < 1 || model->layer_count > kMaxLayers || !mlp_valid(model, model->layer_count))
        return UNBLENDING_INVALID_ARGUMENT;
    const int outs = 4 * model->layer_count;
    return guarded([&]() -> int32_t {
        Context& c = context();
        std::lock_guard<std::mutex> lock(c.mutex);
        cudaStream_t s = c.stream;
        const MlpDevice dev = upload_model(c, *model, s);
        const size_t nw = mlp_weight_count(), nb = mlp_bias_count(), np = nw + nb;
        Buffer grad_b;
        float* grad = grad_b.get<float>(np + 1);
        ck(cudaMemsetAsync(grad, 0, (np + 1) * sizeof(float), s));
        MlpGrad g;
        size_t o = 0, ob = nw;
        for (int k = 0; k < 4; ++k) {
            g.w[k] = grad + o; o += size_t(kMlpSizes[k][0]) * kMlpSizes[k][1];
            g.b[k] = grad + ob; ob += kMlpSizes[k][0];
        }
        g.loss = grad + np;
        int32_t* err = c.small.get<int32_t>(8) + 7;
        ck(cudaMemsetAsync(err, 0, sizeof(int32_t), s));
        ck(launch_mlp_train(dev, features, targets, count, outs, g, err, c.sms, s));
        ++t_launches;
        std::vector<float> out(np + 1);
        int32_t failed = 0;
        ck(cudaMemcpyAsync(out.data(), grad, (np + 1) * sizeof(float), cudaMemcpyDeviceToHost, s));
        ck(cudaMemcpyAsync(&failed, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        ck(cudaStreamSynchronize(s));
        if (failed) throw CudaFailure(cudaErrorLaunchTimeout);
        gradient->layer_count = model->layer_count;
        o = 0;
        for (int k = 0; k < 4; ++k) {
            const size_t sz = size_t(kMlpSizes[k][0]) * kMlpSizes[k][1];
            std::copy(out.begin() + o, out.begin() + o + sz, mlp_weight(*gradient, k));
            o += sz;
        }
        for (int k = 0; k < 4; ++k) {
            std::copy(out.begin() + o, out.begin() + o + kMlpSizes[k][0], mlp_bias(*gradient, k));
            o += kMlpSizes[k][0];
        }
        gradient->loss = out[np] / float(size_t(count) * outs);
        gradient->steps = 0;
        return UNBLENDING_OK;
    });
}

int32_t unblending_mlp_train_device(int32_t count, const int32_t* widths, const int32_t* heights,
                                    const double* const* images, const unblending_layer* layers, size_t layer_count,
                                    const unblending_options* options, const unblending_solver_options* solver,
                                    const unblending_mlp_options* mlp_options, unblending_mlp* model) {
    t_launches = 0;
    if (count <= 0 || !widths || !heights || !images || !model || model->struct_size < sizeof(unblending_mlp))
        return UNBLENDING_INVALID_ARGUMENT;
    const unblending_mlp_options mdef = UNBLENDING_MLP_OPTIONS_INIT;
    const unblending_mlp_options mo = mlp_options ? *mlp_options : mdef;
    if ((mlp_options && mlp_options->struct_size < sizeof(unblending_mlp_options)) || mo.batch < 128 ||
        mo.batch > (1 << 20) || mo.steps < 1 || !(mo.learning_rate > 0))
        return UNBLENDING_INVALID_ARGUMENT;
    unblending_solver_options so;
    int32_t rc = resolve_solver(solver, so);
    if (rc != UNBLENDING_OK) return rc;
    so.warm_start = nullptr;   // targets come from the reference's start
    std::vector<Spec> specs(count);
    size_t pool = 0, largest = 0;
    for (int k = 0; k < count; ++k) {
        unblending_rgb_view view{images[k], 0, widths[k], heights[k], 0};
        rc = validate(&view, layers, layer_count, options, images[k], 0, false, nullptr, 0, specs[k], true);
        if (rc != UNBLENDING_OK) return rc;
        pool += specs[k].pixels;
        largest = std::max(largest, specs[k].pixels);
    }
    const int L = int(layer_count), outs = 4 * L;
    return guarded([&]() -> int32_t {
        Context& c = context();
        std::lock_guard<std::mutex> lock(c.mutex);
        cudaStream_t s = c.stream;
        // Pool of (features, targets): the first pass of every image.
        Buffer feats_b, targets_b, packed_b, bf_b, bt_b, master_b, grad_b, wdev_b;
        float* feats = feats_b.get<float>(pool * kMlpIn);
        float* targets = targets_b.get<float>(pool * outs);
        double* packed = packed_b.get<double>(largest * outs);
        size_t off = 0;
        for (int k = 0; k < count; ++k) {
            const Spec& sp = specs[k];
            ck(launch_mlp_features(images[k], sp.width, sp.height, feats + off * kMlpIn, s));
            PassIO io;
            io.image = images[k];
            io.out = packed;
            io.status = c.status.get<int32_t>(sp.pixels);
            enqueue_pass(c, sp, false, layers, so, io, s);
            ck(launch_gather_targets(packed, int64_t(sp.pixels), L, targets + off * outs, s));
            off += sp.pixels;
        }
        // Parameters: FP32 masters + Adam moments, BF16 copies, gradients.
        const size_t nw = mlp_weight_count(), nb = mlp_bias_count(), np = nw + nb;
        float* master = master_b.get<float>(3 * np);   // params | m | v
        float* grad = grad_b.get<float>(np + 1);       // dW | db | loss
        __nv_bfloat16* wdev = wdev_b.get<__nv_bfloat16>(nw);
        std::vector<float> init(3 * np, 0.0f);
        {
            // He-uniform for the GELU layers, Glorot-uniform for the output;
            // rows of the output layer beyond 4L stay zero.
            uint64_t st = mo.seed * 0x9E3779B97F4A7C15ull + 1;
            auto uni = [&]() {
                st ^= st << 13; st ^= st >> 7; st ^= st << 17;
                return double(st >> 11) * (1.0 / 9007199254740992.0);
            };
            size_t o = 0;
            for (int k = 0; k < 4; ++k) {
                const int rows = kMlpSizes[k][0], cols = kMlpSizes[k][1];
                const int fan_in = k == 0 ? 30 : cols;
                const double bound = k < 3 ? std::sqrt(6.0 / fan_in) : std::sqrt(6.0 / (fan_in + outs));
                for (int r = 0; r < rows; ++r)
                    for (int q = 0; q < cols; ++q)
                        init[o + size_t(r) * cols + q] = (k == 3 && r >= outs) ? 0.0f : float((2 * uni() - 1) * bound);
                o += size_t(rows) * cols;
            }
        }
        std::vector<__nv_bfloat16> wb(nw);
        for (size_t i = 0; i < nw; ++i) wb[i] = __float2bfloat16(init[i]);
        ck(cudaMemcpyAsync(master, init.data(), init.size() * sizeof(float), cudaMemcpyHostToDevice, s));
        ck(cudaMemcpyAsync(wdev, wb.data(), nw * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice, s));
        ck(cudaMemsetAsync(grad, 0, (np + 1) * sizeof(float), s));
        MlpDevice dev;
        MlpMaster mm;
        MlpGrad g;
        {
            size_t o = 0, ob = nw;
            for (int k = 0; k < 4; ++k) {
                const size_t sz = size_t(kMlpSizes[k][0]) * kMlpSizes[k][1];
                dev.w[k] = wdev + o;
                mm.w[k] = master + o; mm.mw[k] = master + np + o; mm.vw[k] = master + 2 * np + o;
                g.w[k] = grad + o;
                o += sz;
                dev.b[k] = master + ob;
                mm.b[k] = master + ob; mm.mb[k] = master + np + ob; mm.vb[k] = master + 2 * np + ob;
                g.b[k] = grad + ob;
                ob += kMlpSizes[k][0];
            }
            g.loss = grad + np;
        }
        float* bfeats = bf_b.get<float>(size_t(mo.batch) * kMlpIn);
        float* btargets = bt_b.get<float>(size_t(mo.batch) * outs);
        int32_t* err = c.small.get<int32_t>(8) + 7;
        ck(cudaMemsetAsync(err, 0, sizeof(int32_t), s));
        float loss = 0.0f;
        for (int step = 1; step <= mo.steps; ++step) {
            ck(launch_sample_batch(feats, targets, int64_t(pool), outs, mo.batch, mo.seed * 1000003ull + step, bfeats,
                                   btargets, s));
            if (step == mo.steps) ck(cudaMemsetAsync(g.loss, 0, sizeof(float), s));
            ck(launch_mlp_train(dev, bfeats, btargets, mo.batch, outs, g, err, c.sms, s));
            if (step == mo.steps) ck(cudaMemcpyAsync(&loss, g.loss, sizeof(float), cudaMemcpyDeviceToHost, s));
            ck(launch_mlp_adam(mm, g, dev, mo.learning_rate, step, s));
            t_launches += 3;
        }
        std::vector<float> out(np);
        int32_t failed = 0;
        ck(cudaMemcpyAsync(out.data(), master, np * sizeof(float), cudaMemcpyDeviceToHost, s));
        ck(cudaMemcpyAsync(&failed, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        ck(cudaStreamSynchronize(s));
        if (failed) throw CudaFailure(cudaErrorLaunchTimeout);
        model->layer_count = L;
        size_t o = 0;
        for (int k = 0; k < 4; ++k) {
            const size_t sz = size_t(kMlpSizes[k][0]) * kMlpSizes[k][1];
            std::copy(out.begin() + o, out.begin() + o + sz, mlp_weight(*model, k));
            o += sz;
        }
        for (int k = 0; k < 4; ++k) {
            std::copy(out.begin() + o, out.begin() + o + kMlpSizes[k][0], mlp_bias(*model, k));
            o += kMlpSizes[k][0];
        }
        model->loss = loss / float(size_t(mo.batch) * outs);
        model->steps = mo.steps;
        return UNBLENDING_OK;
    });
}

// First pass without any allocation: the solve's scratch (queue heads, miss
// counters, miss lists) comes from the fixed array of noalloc.cu, and the
// work runs on the caller's stream with no library stream or event.
int32_t unblending_unmix_device_noalloc(int32_t width, int32_t height, const double* image,
                                        const unblending_layer* layers, size_t layer_count,
                                        const unblending_options* options, const unblending_solver_options* solver,
                                        double* output, int32_t* status, void* stream) {
    t_launches = 0;
    unblending_rgb_view view{image, 0, width, height, 0};
    Spec sp;
    int32_t rc = validate(&view, layers, layer_count, options, output, 0, false, nullptr, 0, sp, true);
    if (rc != UNBLENDING_OK) return rc;
    unblending_solver_options so;
    if ((rc = resolve_solver(solver, so)) != UNBLENDING_OK) return rc;
    if (sp.pixels > noalloc_max_pixels()) return UNBLENDING_INVALID_ARGUMENT;   // checked before any CUDA call
    // The learned start needs device buffers of its own (network, predictions):
    // refused here rather than silently ignored.
    if (so.warm_start) return UNBLENDING_INVALID_ARGUMENT;
    return guarded([&]() -> int32_t {
        void* base = nullptr;
        size_t bytes = 0, max_pixels = 0;
        ck(noalloc_scratch(&base, &bytes, &max_pixels));
        if (sp.pixels > max_pixels) return UNBLENDING_INVALID_ARGUMENT;
        int dev = 0, sms = 0;
        ck(cudaGetDevice(&dev));
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int L = sp.layers;
        const size_t n = sp.pixels;
        // Layout: [0,32) queue heads, [32,64) counters, [256, ...) two lists.
        uint32_t* queues = static_cast<uint32_t*>(base);
        int32_t* counts = reinterpret_cast<int32_t*>(static_cast<unsigned char*>(base) + 32);
        int32_t* list_a = reinterpret_cast<int32_t*>(static_cast<unsigned char*>(base) + 256);
        int32_t* list_b = list_a + n;
        // The array keeps the previous call's contents: the queue heads and
        // counters must start at zero; the lists are written before they are read.
        ck(cudaMemsetAsync(base, 0, 64, s));
        const SolverControls ctl = controls(so), ctl32 = fp32_controls(so), ctl_re = resolve_controls(so);
        SolveArgs a;
        a.n = int(n);
        a.image = image; a.out = output; a.status = status;
        a.opaque = sp.opaque; a.smooth = 0;
        a.queue = queues;
        a.miss_list = list_a;
        a.miss_count = counts + 0;
        const int threads = so.threads_per_block ? so.threads_per_block : 128;
        // Kernel variants that keep their history in global memory would need
        // an array: this entry point runs their shared-memory counterparts
        // (same results).
        const int v64 = variant_global_history(true, fp64_variant(so, false)) ? 0 : fp64_variant(so, false);
        if (so.precision == UNBLENDING_PRECISION_FP64) {
            ck(launch_solve_fp64(L, false, v64, make_models<double>(layers, L), ctl, a, threads, sms, s));
            ++t_launches;
        } else {
            int variant = so.kernel_variant >= 0 ? so.kernel_variant : default_fp32_variant(L, false);
            if (variant_global_history(false, variant)) variant = 3;
            ck(launch_solve_fp32(L, false, variant, make_models<float>(layers, L), ctl32, a, threads, sms, s));
            ++t_launches;
            if (so.resolve_misses) {
                SolveArgs b = a;
                b.list = list_a; b.list_count = counts + 0;
                b.miss_list = list_b; b.miss_count = counts + 1;
                b.queue = queues + 1;
                ck(launch_solve_fp64(L, false, v64, make_models<double>(layers, L), ctl_re, b, threads, sms, s));
                ++t_launches;
            }
        }
        ck(cudaPeekAtLastError());
        return UNBLENDING_OK;
    });
}

}  // extern "C"
