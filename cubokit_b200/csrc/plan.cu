// Host side of the engine: the C ABI of include/cubo_ptycho.h, input validation, the scan tables, device buffers and
// the per-iteration launch sequence.  Runs on the caller's thread; all device work goes to the context's stream.
#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>
#include <type_traits>
#include <unordered_map>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/cubo_ptycho.h"
#include "engine.h"

using namespace cubo;

struct cubo_ptycho_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    bool timing = false;           // CUDA events around each preprocessing kernel launch
    double prepare_ms = 0.0;       // their device time, summed
    long long prepare_launches = 0;
    // page-locked host staging for the object and probe transfers (grown on demand, freed with the context): copies
    // from it run at full link speed and its pages are already mapped
    void *pinned = nullptr;
    size_t pinned_bytes = 0;
};

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kSide128 = 128;

// --------------------------------------------------------------------------------------------- device buffers

// Freed device blocks kept per device for reuse while a context of the library is alive on that device: a plan's
// multi-GB buffers cost milliseconds to map and unmap (cudaMalloc / cudaFree), which a call that creates and destroys a
// plan pays each time.  A block is kept only after the device has synchronised (what cudaFree does anyway), so no
// queued work still uses it; a request takes the smallest kept block of at least its size and at most 25 % larger;
// a failed cudaMalloc empties the cache and tries again; the last context destroyed on a device empties its cache.
class BlockCache {
  public:
    static BlockCache &get() {
        static BlockCache c;
        return c;
    }
    cudaError_t allocate(void **ptr, size_t *bytes, size_t want, int device) {
        {
            std::lock_guard<std::mutex> lock(m_);
            auto &blocks = free_[slot(device)];
            auto it = blocks.lower_bound(want);
            if (it != blocks.end() && it->first <= want + want / 4) {
                *ptr = it->second;
                *bytes = it->first;
                held_[slot(device)] -= it->first;
                blocks.erase(it);
                return cudaSuccess;
            }
        }
        cudaError_t e = cudaMalloc(ptr, want);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            flush(device);
            e = cudaMalloc(ptr, want);
        }
        if (e == cudaSuccess) *bytes = want;
        else *ptr = nullptr;
        return e;
    }
    void release(void *ptr, size_t bytes, int device) {
        int current = device;
        cudaGetDevice(&current);
        if (current != device) cudaSetDevice(device);
        cudaDeviceSynchronize();
        bool keep = false;
        {
            std::lock_guard<std::mutex> lock(m_);
            if (contexts_[slot(device)] > 0 && held_[slot(device)] + bytes <= kCap) {
                free_[slot(device)].emplace(bytes, ptr);
                held_[slot(device)] += bytes;
                keep = true;
            }
        }
        if (!keep) cudaFree(ptr);
        if (current != device) cudaSetDevice(current);
    }
    void context_created(int device) {
        std::lock_guard<std::mutex> lock(m_);
        contexts_[slot(device)]++;
    }
    void context_destroyed(int device) {
        bool last = false;
        {
            std::lock_guard<std::mutex> lock(m_);
            last = --contexts_[slot(device)] <= 0;
        }
        if (last) flush(device);
    }
    void flush(int device) {
        std::multimap<size_t, void *> blocks;
        {
            std::lock_guard<std::mutex> lock(m_);
            blocks.swap(free_[slot(device)]);
            held_[slot(device)] = 0;
        }
        for (auto &b : blocks) cudaFree(b.second);
    }

  private:
    static constexpr int kDevices = 64;
    static constexpr size_t kCap = 64ull << 30;  // bytes kept at most per device
    static int slot(int device) { return device >= 0 && device < kDevices ? device : 0; }
    std::mutex m_;
    std::multimap<size_t, void *> free_[kDevices];
    size_t held_[kDevices] = {};
    int contexts_[kDevices] = {};
};

struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    int device = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    ~DeviceBuffer() { release(); }
    void release() {
        if (ptr) BlockCache::get().release(ptr, bytes, device);
        ptr = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t b) {
        release();
        if (b == 0) b = 16;
        cudaGetDevice(&device);
        return BlockCache::get().allocate(&ptr, &bytes, b, device);
    }
    template <typename X> X *as() const { return static_cast<X *>(ptr); }
};

struct Failure {
    int status;
    std::string message;
};

[[noreturn]] void fail(int status, const std::string &message) { throw Failure{status, message}; }

void check(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return;
    cudaGetLastError();  // clear a sticky launch error flag where possible
    const int status = (e == cudaErrorMemoryAllocation) ? CUBO_PTYCHO_OUT_OF_MEMORY : CUBO_PTYCHO_CUDA_ERROR;
    fail(status, std::string(what) + ": " + cudaGetErrorString(e));
}

std::vector<double2> twiddles(int L) {
    std::vector<double2> t(L);
    for (int k = 0; k < L; k++) {
        const double a = -2.0 * kPi * (double)k / (double)L;
        t[k] = make_double2(std::cos(a), std::sin(a));
    }
    return t;
}

// Copies v into b, reusing b's memory when it is large enough (no cudaFree, which waits for the device, when tables are
// rebuilt between iterations).
template <typename X>
void upload(DeviceBuffer &b, const std::vector<X> &v, cudaStream_t s) {
    if (b.ptr == nullptr || b.bytes < v.size() * sizeof(X)) check(b.alloc(v.size() * sizeof(X)), "cudaMalloc");
    if (!v.empty()) check(cudaMemcpyAsync(b.ptr, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice, s), "upload");
}

bool finite_positive(double v) { return std::isfinite(v) && v > 0; }

// bf16 bits of a double: rounded to float, then to bf16 (nearest, ties to even) on the float's bits.
uint16_t bf16_round(double v) {
    const float f = (float)v;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}
double bf16_to_double(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return (double)f;
}

}  // namespace

// The context's page-locked staging buffer of at least `bytes` (its contents are not kept when it grows).
void *pinned_staging(cubo_ptycho_context *ctx, size_t bytes) {
    if (ctx->pinned_bytes < bytes) {
        if (ctx->pinned) cudaFreeHost(ctx->pinned);
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
        check(cudaHostAlloc(&ctx->pinned, bytes, cudaHostAllocDefault), "cudaHostAlloc staging");
        ctx->pinned_bytes = bytes;
    }
    return ctx->pinned;
}

// ------------------------------------------------------------------------------------------------ the plan

struct cubo_ptycho_plan {
    cubo_ptycho_context *ctx = nullptr;
    int R = 0, C = 0, OR = 0, OC = 0, P = 0, n = 0;
    long long objects = 0;
    cubo_ptycho_params params{};
    std::vector<unsigned char> mask;
    double divisor = 0;
    bool fp64 = false;
    int classes = 1;        // shift classes; class 0 is the zero shift
    int groups = 1;         // probe-gather position groups
    int tiles_x = 0, tiles = 0;
    int tile_w = kTileW, tile_h = kTileH;  // object-gather tile
    int probe_blocks = 0;
    bool fast = false;      // 128 x 128 FP32 register-resident position pass
    bool bf16 = false;      // 128 x 128 split-BF16 tensor-core position pass
    bool global64 = false;  // FP64 position pass through global memory (the plane does not fit shared memory)
    bool global32 = false;  // FP32 position pass through global memory (global32.cu)
    // split-BF16: an iteration runs band by band (position pass, object gather, probe gather of one band of
    // band_size positions at a time) so that a band's residuals stay in L2 between the pass and the gathers
    bool banded = false;
    int band_size = 0, bands = 0;
    // in a batch: this plan's generic position pass / its object and probe gathers run in the batch's grouped
    // (persistent, every item at once) launches instead of its own
    bool grouped_pass = false, grouped_gathers = false;
    std::vector<int> band_tile_offsets;  // [bands + 1]: band b's object-gather tiles are band_tiles[offsets[b] ..]
    bool plane128 = false;  // FP64 128 x 128 planes: FFT, pointwise step and inverse FFT in one clustered launch
    int plane_cluster = 2;  // CTAs per plane of that launch
    int states = 1;         // probe states (the mixed-state engine; 1 = single slice)
    int slices = 1;         // object slices (the multislice engine)
    bool multislice = false;        // the multislice engine (its iteration, even with one slice)
    bool identical_slices = false;  // multislice: every slice replaced by their mean after each update
    bool orthogonalize = false;     // mixed state: orthogonalise the states after every iteration
    bool zero_pixel_infinite = true; // mixed state: an exactly zero far-field pixel adds an infinite error term
    int sms = 148;
    long long error_count = 0;  // residual partials summed by the error kernel
    bool tape_valid = false;    // dpsi holds the residuals of the current state (forward ran, nothing changed since)
    long long iterations_done = 0;
    long long errors_capacity = 0;
    long long launches = 0;
    Radices rad_rows{}, rad_columns{};
    // position correction (FP64 form): positions on the device ([rows | columns]), their start, limits in pixels
    bool correct_positions = false;
    double limit_update = 0, limit_total = 0;
    double initial_mean_row = 0, initial_mean_column = 0;
    bool scan_stale = false;             // positions moved since the scan tables were built
    int correction_chunk = 1;            // positions per exit-wave batch
    std::vector<double> positions_given; // [rows | columns] as supplied

    // timing
    bool timing = false;
    struct Timed { int kind; cudaEvent_t a, b; };
    std::vector<Timed> pending;
    std::vector<cudaEvent_t> event_pool;
    std::vector<double> kind_ms;
    std::vector<long long> kind_launches;

    // device memory
    DeviceBuffer amplitudes, rr, cc, cls, tile_start, tile_list;
    DeviceBuffer object, grad_o, weight_o, tile_max;
    DeviceBuffer dpsi, error, errors, iteration;
    DeviceBuffer probe64, scratch64, spectrum64, shifted, shift_tmp64, ramps_r64, ramps_c64;
    DeviceBuffer partial_grad, partial_weight, grad_p64, weight_p64, probe_block_max;
    DeviceBuffer maxes, sums, aperture64, mask_dev, error_scratch, loss_slot;
    DeviceBuffer tw_r, tw_c, tw_r64, tw_c64;
    DeviceBuffer c_planes, fault;
    DeviceBuffer positions64, initial64, object_before, far64, position_bad, fractions64;
    DeviceBuffer gram64, mixing64, ortho64;
    DeviceBuffer waves64, props64, ident, slice_max;  // multislice: entering waves, propagators, identity classes
    DeviceBuffer prop_factors64;  // multislice, 128 x 128 planes: per gap the row and the column factor (128 + 128)
    DeviceBuffer mixed_factors64;  // mixed state, 128 x 128 planes: the projection's factor per position and pixel
    DeviceBuffer tile_counts;          // position correction: candidate counts per tile, rebuilt on the device
    DeviceBuffer band_tiles, dpsi_band;  // banded iterations: tiles per band, the residuals of one band
    DeviceBuffer shard_loss, shard_counter;  // sharded iterations: this plan's summed squared error, its reduce counter
    long long tile_capacity = 0;       // entries the candidate list holds

    ~cubo_ptycho_plan() {
        for (auto &t : pending) { event_pool.push_back(t.a); event_pool.push_back(t.b); }
        for (auto e : event_pool) cudaEventDestroy(e);
    }
};

namespace {

enum Kind { kPositionPass, kObjectGather, kProbeGather, kProbeReduce, kMaxReduce, kObjectUpdate, kProbeSide,
            kErrorReduce, kShiftTable, kPositionCorrection, kBackPropagation, kKinds };
const char *kKindNames[kKinds] = {"position_pass", "object_gather", "probe_gather", "probe_reduce", "max_reduce",
                                  "object_update", "probe_update_constraints", "error_reduce", "shift_table",
                                  "position_correction", "back_propagation"};

cudaEvent_t take_event(cubo_ptycho_plan *p) {
    if (!p->event_pool.empty()) {
        cudaEvent_t e = p->event_pool.back();
        p->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    check(cudaEventCreate(&e), "cudaEventCreate");
    return e;
}

// Runs `launch` (which enqueues `count` kernels) and accounts for it.
template <typename F>
void timed(cubo_ptycho_plan *p, Kind kind, int count, F &&launch) {
    cudaStream_t s = p->ctx->stream;
    cudaEvent_t a = nullptr, b = nullptr;
    if (p->timing) {
        a = take_event(p);
        b = take_event(p);
        check(cudaEventRecord(a, s), "cudaEventRecord");
    }
    check(launch(), kKindNames[kind]);
    p->launches += count;
    if (p->timing) {
        check(cudaEventRecord(b, s), "cudaEventRecord");
        p->pending.push_back({kind, a, b});
        p->kind_launches[kind] += count;
    }
}

void collect_timing(cubo_ptycho_plan *p) {
    if (p->pending.empty()) return;
    check(cudaStreamSynchronize(p->ctx->stream), "cudaStreamSynchronize");
    for (auto &t : p->pending) {
        float ms = 0;
        check(cudaEventElapsedTime(&ms, t.a, t.b), "cudaEventElapsedTime");
        p->kind_ms[t.kind] += ms;
        p->event_pool.push_back(t.a);
        p->event_pool.push_back(t.b);
    }
    p->pending.clear();
}

// PtychographyPositionCorrection.pixelDistances (Ptychography.swift:74-84): the two limits in pixels, or a refusal.
void position_limits(const cubo_ptycho_params *pp, double *update, double *total) {
    if (!std::isfinite(pp->position_step_size)) fail(CUBO_PTYCHO_INVALID_INPUT, "position step");
    double scale = 1.0;
    if (pp->has_max_position_update_distance || pp->has_max_position_total_distance) {
        const double r = pp->position_row_sampling, c = pp->position_column_sampling;
        if (!(std::isfinite(r) && r > 0 && std::isfinite(c) && c > 0))
            fail(CUBO_PTYCHO_INVALID_INPUT, "position correction needs both samplings with a distance");
        scale = std::sqrt(r * r + c * c);
    }
    const double inf = std::numeric_limits<double>::infinity();
    for (int k = 0; k < 2; k++) {
        const bool has = k == 0 ? pp->has_max_position_update_distance : pp->has_max_position_total_distance;
        const double d = k == 0 ? pp->max_position_update_distance : pp->max_position_total_distance;
        if (has && !(std::isfinite(d) && d > 0)) fail(CUBO_PTYCHO_INVALID_INPUT, "position distance");
    }
    *update = (pp->has_max_position_update_distance ? pp->max_position_update_distance : inf) / scale;
    *total = (pp->has_max_position_total_distance ? pp->max_position_total_distance : inf) / scale;
}

// Ptychography.swift:236-264: the refusals of the reference (position correction only on the Double path: here the
// FP64 form).
void validate(const cubo_ptycho_problem *pr, const cubo_ptycho_params *pp, double *divisor_out) {
    if (!pr || !pp) fail(CUBO_PTYCHO_INVALID_INPUT, "null problem or params");
    if (pp->has_position_correction) {
        if (pp->form != CUBO_PTYCHO_FORM_FP64)
            fail(CUBO_PTYCHO_INVALID_INPUT, "position correction runs in the FP64 form (the reference's Double path)");
        double u, t;
        position_limits(pp, &u, &t);
    }
    if (!(pr->rows > 1 && pr->columns > 1 && pr->object_rows > 1 && pr->object_columns > 1))
        fail(CUBO_PTYCHO_INVALID_INPUT, "array dimensions must exceed 1");
    const long long n = (long long)pr->rows * pr->columns;
    if (!(pr->count > 0)) fail(CUBO_PTYCHO_INVALID_INPUT, "no positions");
    if ((long long)pr->count * n > (1LL << 40)) fail(CUBO_PTYCHO_INVALID_INPUT, "too many samples");
    if (!pr->amplitudes || !pr->position_rows || !pr->position_columns) fail(CUBO_PTYCHO_INVALID_INPUT, "null input");
    if (!(pp->iterations >= 0 && finite_positive(pp->step_size))) fail(CUBO_PTYCHO_INVALID_INPUT, "iterations or step");
    if (!(std::isfinite(pp->normalization_minimum) && pp->normalization_minimum >= 0 && pp->normalization_minimum <= 1))
        fail(CUBO_PTYCHO_INVALID_INPUT, "normalization minimum");
    const double limit = (double)(INT64_MAX / 4);
    for (int i = 0; i < pr->count; i++) {
        const double r = pr->position_rows[i], c = pr->position_columns[i];
        if (!(std::isfinite(r) && std::isfinite(c) && std::fabs(r) < limit && std::fabs(c) < limit))
            fail(CUBO_PTYCHO_INVALID_INPUT, "position");
    }
    const double rad = pp->probe_amplitude_relative_radius, wid = pp->probe_amplitude_relative_width;
    if (!(std::isfinite(rad) && rad >= 0 && rad <= 0.5 && std::isfinite(wid) && wid > 0 && wid <= 0.5))
        fail(CUBO_PTYCHO_INVALID_INPUT, "probe amplitude constraint parameters");
    if (!(pr->object_rows >= pr->rows && pr->object_columns >= pr->columns))
        fail(CUBO_PTYCHO_INVALID_INPUT, "object smaller than probe");
    // the amplitudes themselves (finite, non-negative) and their energy are checked on the device once uploaded
    double d = 1.0;
    if (pp->error_normalization == CUBO_PTYCHO_ERRORS_MEAN_INTENSITY) {
        d = pp->mean_intensity * (double)pr->count;
        if (!finite_positive(d)) fail(CUBO_PTYCHO_INVALID_INPUT, "error normalisation divisor");
    }
    if (pp->form < CUBO_PTYCHO_FORM_FP32 || pp->form > CUBO_PTYCHO_FORM_FP64) fail(CUBO_PTYCHO_INVALID_INPUT, "form");
    if (pp->gather_tile < 0 || pp->gather_tile > 3) fail(CUBO_PTYCHO_INVALID_INPUT, "gather tile");
    if (pp->pass_shape < 0 || pp->pass_shape > 3) fail(CUBO_PTYCHO_INVALID_INPUT, "position-pass shape");
    if (pp->variant < CUBO_PTYCHO_VARIANT_AUTO || pp->variant > CUBO_PTYCHO_VARIANT_GLOBAL)
        fail(CUBO_PTYCHO_INVALID_INPUT, "variant");
    *divisor_out = d;
}

long long wrap_ll(long long v, long long m) {
    long long r = v % m;
    return r < 0 ? r + m : r;
}

// Scan tables from positions (host, count each): ties-to-even centres (Ptychography.swift:301), wrapped; shift classes
// by exact fraction, with their phase ramps; the object-gather candidate lists.  Run at plan creation and, with
// position correction, whenever the positions have moved.
void build_scan(cubo_ptycho_plan *p, const double *rows_in, const double *columns_in) {
    cudaStream_t s = p->ctx->stream;
    const int R = p->R, C = p->C, n = p->n, P = p->P;
    std::vector<int> rr(P), cc(P), cls(P);
    struct PairHash {
        size_t operator()(const std::pair<uint64_t, uint64_t> &k) const {
            return std::hash<uint64_t>()(k.first * 0x9E3779B97F4A7C15ull ^ k.second);
        }
    };
    std::unordered_map<std::pair<uint64_t, uint64_t>, int, PairHash> class_of;
    class_of.reserve((size_t)P);
    std::vector<std::pair<double, double>> fractions;  // classes 1..
    for (int i = 0; i < P; i++) {
        const double r = rows_in[i], c = columns_in[i];
        const double rn = std::nearbyint(r), cn = std::nearbyint(c);
        const double dr = r - rn, dc = c - cn;
        rr[i] = (int)wrap_ll((long long)rn, p->OR);
        cc[i] = (int)wrap_ll((long long)cn, p->OC);
        if (p->correct_positions) {  // positions move every iteration: one class each, as the device rebuilds them
            fractions.push_back({dr, dc});
            cls[i] = dr == 0 && dc == 0 ? 0 : i + 1;
            continue;
        }
        if (dr == 0 && dc == 0) { cls[i] = 0; continue; }
        uint64_t kr, kc;
        std::memcpy(&kr, &dr, 8);
        std::memcpy(&kc, &dc, 8);
        auto key = std::make_pair(kr, kc);
        auto it = class_of.find(key);
        if (it == class_of.end()) {
            fractions.push_back({dr, dc});
            it = class_of.emplace(key, (int)fractions.size()).first;
        }
        cls[i] = it->second;
    }
    p->classes = 1 + (int)fractions.size();
    upload(p->rr, rr, s);
    upload(p->cc, cc, s);
    upload(p->cls, cls, s);
    // ---- object-gather candidate lists: for each tile, the positions whose window touches it, ascending
    // tiles wide along x, the residual's contiguous axis; the square default wastes the fewest lanes on windows that
    // reach only part of a tile (at a 128 x 128 detector and a 4-pixel step ~80 % of a tile's candidate slots hold a
    // pixel of the window, against ~75 % for 32 x 8) and measured fastest at 128 x 128 in every form
    const int choice = p->params.gather_tile;
    const int wide = choice == 1 ? 32 : choice == 3 ? 64 : choice == 2 ? 16 : kTileW;
    const int narrow = kGatherThreads / wide;
    p->tile_w = wide;
    p->tile_h = narrow;
    p->tiles_x = (p->OC + p->tile_w - 1) / p->tile_w;
    const int tiles_y = (p->OR + p->tile_h - 1) / p->tile_h;
    p->tiles = p->tiles_x * tiles_y;
    {
        // counted and listed on the device from the wrapped centres (one warp per tile, positions ascending)
        if (p->tile_start.bytes < (size_t)(p->tiles + 1) * sizeof(int))
            check(p->tile_start.alloc((size_t)(p->tiles + 1) * sizeof(int)), "cudaMalloc");
        check(launch_tile_lists(p->rr.as<int>(), p->cc.as<int>(), P, R, C, p->OR, p->OC, p->tile_w, p->tile_h, p->tiles_x,
                                p->tiles, p->tile_start.as<int>(), nullptr, nullptr, 0, s), "count candidates");
        std::vector<int> counts(p->tiles + 1, 0);
        check(cudaMemcpyAsync(counts.data(), p->tile_start.ptr, (size_t)p->tiles * sizeof(int), cudaMemcpyDeviceToHost, s),
              "download counts");
        check(cudaStreamSynchronize(s), "count candidates");
        long long total = 0;
        for (int t = 0; t < p->tiles; t++) {  // exclusive sums
            const int c = counts[t];
            counts[t] = (int)total;
            total += c;
        }
        if (total > INT32_MAX) fail(CUBO_PTYCHO_UNSUPPORTED, "object-gather candidate lists exceed 2^31 entries");
        counts[p->tiles] = (int)total;
        upload(p->tile_start, counts, s);
        // with position correction the lists are rebuilt on the device: room for every window's largest tile count
        const long long capacity =
            p->correct_positions ? std::max<long long>(total, (long long)P * (R / p->tile_h + 3) * (C / p->tile_w + 3))
                                 : total;
        if (p->tile_list.bytes < (size_t)std::max<long long>(capacity, 1) * sizeof(int))
            check(p->tile_list.alloc((size_t)std::max<long long>(capacity, 1) * sizeof(int)), "cudaMalloc");
        p->tile_capacity = std::max<long long>(capacity, 1);
        check(launch_tile_lists(p->rr.as<int>(), p->cc.as<int>(), P, R, C, p->OR, p->OC, p->tile_w, p->tile_h, p->tiles_x,
                                p->tiles, nullptr, p->tile_start.as<int>(), p->tile_list.as<int>(),
                                (int)std::min<long long>(p->tile_capacity, INT32_MAX), s), "list candidates");
    }
    const size_t shifted_bytes = (size_t)p->states * p->classes * n * (p->fp64 ? sizeof(double2) : sizeof(float2));
    if (p->shifted.bytes < shifted_bytes) check(p->shifted.alloc(shifted_bytes), "cudaMalloc");
    const int frac = p->classes - 1;
    if (frac > 0) {
        if (p->shift_tmp64.bytes < (size_t)frac * n * sizeof(double2))
            check(p->shift_tmp64.alloc((size_t)frac * n * sizeof(double2)), "cudaMalloc shift table");
        if (p->ramps_r64.bytes < (size_t)frac * R * sizeof(double2))
            check(p->ramps_r64.alloc((size_t)frac * R * sizeof(double2)), "cudaMalloc");
        if (p->ramps_c64.bytes < (size_t)frac * C * sizeof(double2))
            check(p->ramps_c64.alloc((size_t)frac * C * sizeof(double2)), "cudaMalloc");
        std::vector<double2> fr((size_t)frac);
        for (int f = 0; f < frac; f++) fr[f] = make_double2(fractions[f].first, fractions[f].second);
        upload(p->fractions64, fr, s);  // the ramps themselves are computed on the device (Ptychography.swift:304-311)
        check(launch_ramp_table(p->fractions64.as<double2>(), frac, R, C, p->ramps_r64.as<double2>(),
                                p->ramps_c64.as<double2>(), s), "shift ramps");
    }
}

// Bands of an iteration run band by band (split-BF16): band b holds positions [b band_size, (b + 1) band_size).  Lists
// per band the object-gather tiles with a candidate inside it (ascending), and every tile without candidates in band 0,
// which writes their zero sums and maxima.
void build_band_tiles(cubo_ptycho_plan *p) {
    cudaStream_t s = p->ctx->stream;
    std::vector<int> starts(p->tiles + 1), list;
    check(cudaMemcpyAsync(starts.data(), p->tile_start.ptr, starts.size() * sizeof(int), cudaMemcpyDeviceToHost, s),
          "download candidate lists");
    check(cudaStreamSynchronize(s), "download candidate lists");
    list.resize(std::max(1, starts[p->tiles]));
    check(cudaMemcpyAsync(list.data(), p->tile_list.ptr, (size_t)starts[p->tiles] * sizeof(int), cudaMemcpyDeviceToHost,
                          s), "download candidate lists");
    check(cudaStreamSynchronize(s), "download candidate lists");
    std::vector<std::vector<int>> per_band(p->bands);
    for (int t = 0; t < p->tiles; t++) {
        if (starts[t] == starts[t + 1]) { per_band[0].push_back(t); continue; }
        int last = -1;
        for (int i = starts[t]; i < starts[t + 1]; i++) {  // candidates ascending: their bands too
            const int b = list[i] / p->band_size;
            if (b != last) { per_band[b].push_back(t); last = b; }
        }
    }
    p->band_tile_offsets.assign(p->bands + 1, 0);
    std::vector<int> flat;
    for (int b = 0; b < p->bands; b++) {
        std::sort(per_band[b].begin(), per_band[b].end());
        flat.insert(flat.end(), per_band[b].begin(), per_band[b].end());
        p->band_tile_offsets[b + 1] = (int)flat.size();
    }
    if (flat.empty()) flat.push_back(0);
    upload(p->band_tiles, flat, s);
}

// The residuals of every position, for the paths that keep them (the adjoint pair, sharded iterations): allocated at
// plan creation, or on first use by a banded plan.
template <typename T>
void ensure_dpsi(cubo_ptycho_plan *p) {
    const size_t bytes = (size_t)p->states * p->P * p->n * sizeof(C2<T>);
    if (p->dpsi.bytes < bytes) check(p->dpsi.alloc(bytes), "cudaMalloc dpsi");
}

template <typename T>
void build_plan(cubo_ptycho_plan *p, const cubo_ptycho_problem *pr) {
    cudaStream_t s = p->ctx->stream;
    const int R = p->R, C = p->C, n = p->n, P = p->P;
    build_scan(p, pr->position_rows, pr->position_columns);
    // ---- amplitudes (Float32, [position][row][column]; the 128 x 128 kernel's register order when it runs)
    check(p->amplitudes.alloc((size_t)P * n * sizeof(float)), "cudaMalloc amplitudes");
    check(cudaMemcpyAsync(p->amplitudes.ptr, pr->amplitudes, (size_t)P * n * sizeof(float),
                          pr->amplitudes_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s),
          "upload amplitudes");
    {
        // every amplitude finite and non-negative, and sum A^2 (Ptychography.swift:247-259), in the supplied order
        DeviceBuffer scratch, bad;
        check(scratch.alloc((size_t)amplitude_check_scratch() * sizeof(double)), "cudaMalloc");
        check(bad.alloc(sizeof(int)), "cudaMalloc");
        check(cudaMemsetAsync(bad.ptr, 0, sizeof(int), s), "memset");
        check(launch_amplitude_check(p->amplitudes.as<float>(), (long long)P * n, scratch.as<double>(), bad.as<int>(), s),
              "amplitude check");
        double energy = 0;
        int any_bad = 0;
        check(cudaMemcpyAsync(&energy, scratch.as<double>() + amplitude_check_scratch() - 1, sizeof(double),
                              cudaMemcpyDeviceToHost, s), "download");
        check(cudaMemcpyAsync(&any_bad, bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, s), "download");
        check(cudaStreamSynchronize(s), "amplitude check");
        if (any_bad) fail(CUBO_PTYCHO_INVALID_INPUT, "amplitude not finite and non-negative");
        if (p->params.error_normalization != CUBO_PTYCHO_ERRORS_MEAN_INTENSITY) {
            if (!finite_positive(energy)) fail(CUBO_PTYCHO_INVALID_INPUT, "error normalisation divisor");
            p->divisor = energy;
        }
    }
    if (p->fast || p->bf16) {
        DeviceBuffer permuted;
        check(permuted.alloc((size_t)P * n * sizeof(float)), "cudaMalloc amplitudes");
        if (p->fast) check(launch_permute_amplitudes(p->amplitudes.as<float>(), permuted.as<float>(), P, s), "permute amplitudes");
        else check(launch_permute_bf16_amplitudes(p->amplitudes.as<float>(), permuted.as<float>(), P, s), "permute amplitudes");
        check(cudaStreamSynchronize(s), "permute amplitudes");
        std::swap(p->amplitudes.ptr, permuted.ptr);
        std::swap(p->amplitudes.bytes, permuted.bytes);
        std::swap(p->amplitudes.device, permuted.device);
    }
    // ---- state and work buffers
    check(p->object.alloc((size_t)p->slices * p->objects * sizeof(C2<T>)), "cudaMalloc object");
    check(p->grad_o.alloc((size_t)p->slices * p->objects * sizeof(C2<T>)), "cudaMalloc");
    check(p->weight_o.alloc((size_t)p->slices * p->objects * sizeof(T)), "cudaMalloc");
    check(p->tile_max.alloc((size_t)p->slices * p->tiles * sizeof(double)), "cudaMalloc");
    if (p->multislice) {
        check(p->waves64.alloc((size_t)(p->slices - 1) * P * n * sizeof(double2)), "cudaMalloc entering waves");
        check(p->slice_max.alloc((size_t)p->slices * sizeof(double)), "cudaMalloc");
        std::vector<int> ident(P);
        for (int i = 0; i < P; i++) ident[i] = i;
        upload(p->ident, ident, s);
    }
    if (p->banded) {
        // one band's residuals; the residuals of every position (the adjoint pair's tape, sharded iterations) are
        // allocated when first needed
        check(p->dpsi_band.alloc((size_t)p->band_size * n * sizeof(C2<T>)), "cudaMalloc band residuals");
        build_band_tiles(p);
    } else {
        check(p->dpsi.alloc((size_t)p->states * P * n * sizeof(C2<T>)), "cudaMalloc dpsi");
    }
    p->error_count = p->fast     ? (long long)P * fast128_partials_per_position()
                     : p->bf16     ? (long long)P * bf16_partials_per_position()
                     : p->global32 ? (long long)P * global32_partials_per_position(p->R, p->C)
                                   : P;
    if (p->fast || p->plane128) {
        check(p->fault.alloc(sizeof(int)), "cudaMalloc");
        check(cudaMemsetAsync(p->fault.ptr, 0, sizeof(int), s), "memset");
    }
    if (p->bf16) {
        // the real factor C of the 128-point DFT matrix (row 0 = 1, row 1 = cos(pi k), rows 2j, 2j + 1 = cos, sin of
        // 2 pi j k / 128) and C_sigma (its columns in the kernel's stage-4 order), split into bf16 hi + lo in FP64:
        // planes C hi, C lo, C_sigma hi, C_sigma lo, [m][k]
        auto c_value = [&](int m, int k) -> double {
            if (m == 0) return 1.0;
            if (m == 1) return (k & 1) ? -1.0 : 1.0;
            const double a = 2.0 * kPi * (double)(((m >> 1) * k) % R) / (double)R;
            return (m & 1) ? std::sin(a) : std::cos(a);
        };
        std::vector<uint16_t> planes(4 * (size_t)n);
        for (int m = 0; m < R; m++)
            for (int k = 0; k < C; k++) {
                const double v[2] = {c_value(m, k), c_value(m, bf16_sigma(k))};
                for (int part = 0; part < 2; part++) {
                    const uint16_t hi = bf16_round(v[part]);
                    const uint16_t lo = bf16_round(v[part] - bf16_to_double(hi));
                    planes[(size_t)(2 * part) * n + m * C + k] = hi;
                    planes[(size_t)(2 * part + 1) * n + m * C + k] = lo;
                }
            }
        upload(p->c_planes, planes, s);
        check(p->fault.alloc(sizeof(int)), "cudaMalloc");
        check(cudaMemsetAsync(p->fault.ptr, 0, sizeof(int), s), "memset");
    }
    check(p->error.alloc((size_t)p->error_count * sizeof(double)), "cudaMalloc");
    check(p->iteration.alloc(sizeof(int)), "cudaMalloc");
    check(cudaMemsetAsync(p->iteration.ptr, 0, sizeof(int), s), "memset");
    check(p->probe64.alloc((size_t)p->states * n * sizeof(double2)), "cudaMalloc");
    if (p->states > 1) {
        check(p->gram64.alloc((size_t)p->states * p->states * sizeof(double2)), "cudaMalloc");
        check(p->mixing64.alloc((size_t)p->states * p->states * sizeof(double2)), "cudaMalloc");
        check(p->ortho64.alloc((size_t)p->states * n * sizeof(double2)), "cudaMalloc");
    }
    check(p->scratch64.alloc((size_t)n * sizeof(double2)), "cudaMalloc");
    check(p->spectrum64.alloc((size_t)n * sizeof(double2)), "cudaMalloc");
    // probe-gather groups: one wave of CTAs on a 148-SM part (the kernel's resident CTAs per SM times 148, over the
    // pixel blocks: a second, partly filled wave left most SMs waiting on a few); a function of the problem and the
    // kernel's build only, so the summation order (and the result) does not depend on the device
    const int kblocks = (n + 255) / 256;
    p->groups = std::max(1, std::min(P, 148 * probe_gather_resident_ctas<T>() / kblocks));
    if (p->fast) p->groups = std::min(P, fast128_ctas());  // the position pass writes one partial per CTA
    check(p->partial_grad.alloc((size_t)p->groups * n * sizeof(C2<T>)), "cudaMalloc");
    check(p->partial_weight.alloc((size_t)p->groups * n * sizeof(T)), "cudaMalloc");
    check(p->grad_p64.alloc((size_t)p->states * n * sizeof(double2)), "cudaMalloc");
    check(p->weight_p64.alloc((size_t)n * sizeof(double)), "cudaMalloc");
    p->probe_blocks = kblocks;
    check(p->probe_block_max.alloc((size_t)kblocks * sizeof(double)), "cudaMalloc");
    check(p->maxes.alloc(4 * sizeof(double)), "cudaMalloc");
    check(p->error_scratch.alloc((size_t)error_reduce_scratch() * sizeof(double)), "cudaMalloc");
    check(p->loss_slot.alloc(2 * sizeof(double)), "cudaMalloc");  // [0] the loss, [1] an int counter
    check(p->sums.alloc(8 * sizeof(double)), "cudaMalloc");
    check(p->aperture64.alloc((size_t)n * sizeof(double)), "cudaMalloc");
    if (!p->mask.empty()) upload(p->mask_dev, p->mask, s);
    // ---- twiddles
    const std::vector<double2> tr = twiddles(R), tc = twiddles(C);
    upload(p->tw_r64, tr, s);
    upload(p->tw_c64, tc, s);
    std::vector<C2<T>> trt(R), tct(C);
    for (int i = 0; i < R; i++) trt[i] = mk<T>((T)tr[i].x, (T)tr[i].y);
    for (int i = 0; i < C; i++) tct[i] = mk<T>((T)tc[i].x, (T)tc[i].y);
    upload(p->tw_r, trt, s);
    upload(p->tw_c, tct, s);
    p->rad_rows = factor_length(R);
    p->rad_columns = factor_length(C);
}

Fft2Plan64 fft64(const cubo_ptycho_plan *p) {
    return Fft2Plan64{p->R, p->C, p->rad_rows, p->rad_columns, p->tw_r64.as<double2>(), p->tw_c64.as<double2>()};
}

// After a synchronize: a device wait that ran out (split-BF16 kernel) turns into CUBO_PTYCHO_DEVICE_TIMEOUT.
void check_fault(cubo_ptycho_plan *p) {
    if (!p->bf16 && !p->fast && !p->plane128) return;
    int f = 0;
    check(cudaMemcpy(&f, p->fault.ptr, sizeof(int), cudaMemcpyDeviceToHost), "read fault flag");
    if (f) {
        cudaMemset(p->fault.ptr, 0, sizeof(int));
        fail(CUBO_PTYCHO_DEVICE_TIMEOUT, "a device-side completion wait ran out");
    }
}

void ensure_errors(cubo_ptycho_plan *p, long long needed) {
    if (needed <= p->errors_capacity) return;
    long long cap = std::max<long long>(needed, std::max<long long>(64, 2 * p->errors_capacity));
    DeviceBuffer fresh;
    check(fresh.alloc((size_t)cap * sizeof(double)), "cudaMalloc errors");
    if (p->iterations_done > 0)
        check(cudaMemcpyAsync(fresh.ptr, p->errors.ptr, (size_t)p->iterations_done * sizeof(double),
                              cudaMemcpyDeviceToDevice, p->ctx->stream), "copy errors");
    check(cudaStreamSynchronize(p->ctx->stream), "cudaStreamSynchronize");
    std::swap(p->errors.ptr, fresh.ptr);
    std::swap(p->errors.bytes, fresh.bytes);
    std::swap(p->errors.device, fresh.device);
    p->errors_capacity = cap;
}

// A clustered 128 x 128 plane launch (FP64) over every position: the fields every use shares.
Plane128Args plane_args(const cubo_ptycho_plan *p, int mode) {
    Plane128Args a{};
    a.mode = mode; a.first = 0; a.count = p->P; a.in_kind = kInputByPosition;
    a.scan = ScanTables{p->rr.as<int>(), p->cc.as<int>(), p->cls.as<int>()};
    a.object_rows = p->OR; a.object_columns = p->OC; a.pointwise = kPointwiseNone; a.scale = 1.0 / p->n;
    a.amplitudes = p->amplitudes.as<float>(); a.error = p->error.as<double>(); a.inv_n = 1.0 / p->n;
    a.tw = p->tw_r64.as<double2>(); a.out_stride = 1; a.out_offset = 0; a.fault = p->fault.as<int>();
    a.ahead = p->sms / 2;  // the clusters resident at once (Q / 2 CTAs per SM, Q per cluster)
    return a;
}

void enqueue_plane(cubo_ptycho_plan *p, Kind kind, const Plane128Args &a) {
    timed(p, kind, 1, [&] { return launch_plane128(a, p->plane_cluster, p->ctx->stream); });
}

// The full plane launch of every position: `in` (by class or by position) times the object patch (conjugated), FFT,
// the propagator factors x 1/n (project == false) or the modulus projection with the error (project == true),
// inverse FFT, into `out`.
void enqueue_plane128(cubo_ptycho_plan *p, Kind kind, const double2 *in, bool by_class, const double2 *object,
                      bool conj_object, bool project, const double2 *prop_factors, bool conj_prop, double2 *out) {
    Plane128Args a = plane_args(p, kPlaneFull);
    a.in = in; a.in_kind = by_class ? kInputByClass : kInputByPosition; a.object = object;
    a.conj_object = conj_object ? 1 : 0; a.pointwise = project ? kPointwiseProjection : kPointwiseFactors;
    a.prop_rows = prop_factors; a.prop_columns = prop_factors ? prop_factors + 128 : nullptr; a.prop_stride = 0;
    a.conj_prop = conj_prop ? 1 : 0; a.out = out;
    enqueue_plane(p, kind, a);
}

// The shift table of probe state `st`.
template <typename T>
void enqueue_shift_table_state(cubo_ptycho_plan *p, int st) {
    cudaStream_t s = p->ctx->stream;
    const int n = p->n, frac = p->classes - 1;
    const double2 *probe = p->probe64.as<double2>() + (size_t)st * n;
    C2<T> *table = p->shifted.as<C2<T>>() + (size_t)st * p->classes * n;
    timed(p, kShiftTable, 1, [&] { return launch_convert<T>(probe, table, n, s); });
    if (frac == 0) return;
    if constexpr (std::is_same<T, double>::value) {
        if (p->plane128) {  // classes 1 .. frac: the probe's spectrum x the class's ramps, inverse FFT, one launch
            timed(p, kShiftTable, 2, [&] {
                cudaError_t e = cudaMemcpyAsync(p->spectrum64.ptr, probe, (size_t)n * sizeof(double2),
                                                cudaMemcpyDeviceToDevice, s);
                if (e == cudaSuccess) e = launch_fft2_f64(fft64(p), p->spectrum64.as<double2>(), 1, false, s);
                return e;
            });
            Plane128Args a = plane_args(p, kPlaneInverse);
            a.first = 1; a.count = frac; a.in = p->spectrum64.as<double2>(); a.in_kind = kInputSingle;
            a.pointwise = kPointwiseFactors; a.prop_rows = p->ramps_r64.as<double2>();
            a.prop_columns = p->ramps_c64.as<double2>(); a.prop_stride = kSide128; a.out = table;
            enqueue_plane(p, kShiftTable, a);
            return;
        }
    }
    timed(p, kShiftTable, 2 + 1 + 2 + 1 + 1, [&] {
        cudaError_t e = cudaMemcpyAsync(p->spectrum64.ptr, probe, (size_t)n * sizeof(double2),
                                        cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = launch_fft2_f64(fft64(p), p->spectrum64.as<double2>(), 1, false, s);
        if (e == cudaSuccess)
            e = launch_shift_ramps(p->spectrum64.as<double2>(), p->ramps_r64.as<double2>(), p->ramps_c64.as<double2>(),
                                   p->R, p->C, frac, p->shift_tmp64.as<double2>(), s);
        if (e == cudaSuccess) e = launch_fft2_f64(fft64(p), p->shift_tmp64.as<double2>(), frac, true, s);
        if (e == cudaSuccess) e = launch_scale_f64(p->shift_tmp64.as<double2>(), frac * n, 1.0 / n, s);
        if (e == cudaSuccess)
            e = launch_convert<T>(p->shift_tmp64.as<double2>(), table + n, (long long)frac * n, s);
        return e;
    });
}

// The shifted-probe table for the current probe: class 0 is the probe itself, classes 1.. its Fourier shifts (one
// table per probe state, [state][class][pixel]).
template <typename T>
void enqueue_shift_table(cubo_ptycho_plan *p) {
    for (int st = 0; st < p->states; st++) enqueue_shift_table_state<T>(p, st);
}

// Probe update and constraints, FP64 (Ptychography.swift:383-395).  With several probe states
// (PtychographyEngines.swift:212-244): every state takes its own gradient with the shared normalisation; the centre of
// mass of state 0 shifts every state; the aperture constrains state 0; the amplitude constraint and the support apply
// to every state; then the orthogonalisation.
void enqueue_probe_side(cubo_ptycho_plan *p) {
    cudaStream_t s = p->ctx->stream;
    const cubo_ptycho_params &pp = p->params;
    const int n = p->n, S = p->states;
    double2 *probes = p->probe64.as<double2>(), *x = p->scratch64.as<double2>();
    double *sums = p->sums.as<double>();
    if (!pp.fix_probe) {
        for (int st = 0; st < S; st++)
            timed(p, kProbeSide, 1, [&] {
                return launch_probe_update(probes + (size_t)st * n, p->grad_p64.as<double2>() + (size_t)st * n,
                                           p->weight_p64.as<double>(), n, p->maxes.as<double>() + 1, pp.step_size,
                                           pp.normalization_minimum, s);
            });
        if (pp.fix_probe_center_of_mass) {  // PtychographyConstraints.swift:34-37: the centre of mass of state 0
            timed(p, kProbeSide, 1, [&] { return launch_probe_moments(probes, p->R, p->C, sums, s); });
            for (int st = 0; st < S; st++) {
                double2 *probe = probes + (size_t)st * n;
                timed(p, kProbeSide, 6, [&] {
                    cudaError_t e = cudaMemcpyAsync(x, probe, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, s);
                    if (e == cudaSuccess) e = launch_fft2_f64(fft64(p), x, 1, false, s);
                    if (e == cudaSuccess) e = launch_com_ramp(x, p->R, p->C, sums, s);
                    if (e == cudaSuccess) e = launch_fft2_f64(fft64(p), x, 1, true, s);
                    if (e == cudaSuccess) e = launch_scale_f64(x, n, 1.0 / n, s);
                    if (e == cudaSuccess) e = launch_commit_if_valid(probe, x, n, sums, s);
                    return e;
                });
            }
        }
        if (pp.fix_probe_aperture) {  // PtychographyConstraints.swift:59-71, state 0
            double2 *probe = probes;
            timed(p, kProbeSide, 8, [&] {
                cudaError_t e = launch_energy(probe, n, sums + 3, s);
                if (e == cudaSuccess) e = cudaMemcpyAsync(x, probe, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, s);
                if (e == cudaSuccess) e = launch_fft2_f64(fft64(p), x, 1, false, s);
                if (e == cudaSuccess) e = launch_aperture_phase(x, p->aperture64.as<double>(), n, s);
                if (e == cudaSuccess) e = launch_fft2_f64(fft64(p), x, 1, true, s);
                if (e == cudaSuccess) e = launch_scale_f64(x, n, 1.0 / n, s);
                if (e == cudaSuccess) e = launch_energy(x, n, sums + 4, s);
                if (e == cudaSuccess) e = launch_renormalise(probe, x, n, sums + 3, sums + 4, s);
                return e;
            });
        }
        if (pp.constrain_probe_amplitude) {  // PtychographyConstraints.swift:40-55, every state
            for (int st = 0; st < S; st++) {
                double2 *probe = probes + (size_t)st * n;
                timed(p, kProbeSide, 4, [&] {
                    cudaError_t e = launch_energy(probe, n, sums + 3, s);
                    if (e == cudaSuccess)
                        e = launch_amplitude_mask(probe, p->R, p->C, pp.probe_amplitude_relative_radius,
                                                  pp.probe_amplitude_relative_width, s);
                    if (e == cudaSuccess) e = launch_energy(probe, n, sums + 4, s);
                    if (e == cudaSuccess) e = launch_renormalise(probe, probe, n, sums + 3, sums + 4, s);
                    return e;
                });
            }
        }
    }
    if (!p->mask.empty())  // Ptychography.swift:395, not gated on fixProbe
        for (int st = 0; st < S; st++)
            timed(p, kProbeSide, 1, [&] {
                return launch_support_mask(probes + (size_t)st * n, p->mask_dev.as<unsigned char>(), n, s);
            });
    if (p->orthogonalize && S > 1)  // PtychographyEngines.swift:250-253, not gated on fixProbe
        timed(p, kProbeSide, 4, [&] {
            return launch_orthogonalize(probes, S, n, p->gram64.as<double2>(), p->mixing64.as<double2>(),
                                        p->ortho64.as<double2>(), s);
        });
}

// Shifted probes, then the position pass over every position: residuals (dpsi) and per-position squared errors.
// The generic position pass's arguments over every position of the plan.
template <typename T>
PositionPassArgs<T> position_pass_args(cubo_ptycho_plan *p) {
    const int n = p->n;
    PositionPassArgs<T> pa{};
    pa.rows = p->R; pa.columns = p->C; pa.object_rows = p->OR; pa.object_columns = p->OC; pa.n = n;
    pa.first = 0; pa.count = p->P; pa.scan = ScanTables{p->rr.as<int>(), p->cc.as<int>(), p->cls.as<int>()};
    pa.shifted = p->shifted.as<C2<T>>(); pa.object = p->object.as<C2<T>>();
    pa.amplitudes = p->amplitudes.as<float>(); pa.dpsi = p->dpsi.as<C2<T>>(); pa.error = p->error.as<double>();
    pa.tw_rows = p->tw_r.as<C2<T>>(); pa.tw_columns = p->tw_c.as<C2<T>>();
    pa.rad_rows = p->rad_rows; pa.rad_columns = p->rad_columns; pa.inv_n = (T)(1.0 / n);
    return pa;
}

template <typename T>
void enqueue_position_pass(cubo_ptycho_plan *p) {
    cudaStream_t s = p->ctx->stream;
    ensure_dpsi<T>(p);
    const int n = p->n;
    const ScanTables scan{p->rr.as<int>(), p->cc.as<int>(), p->cls.as<int>()};
    enqueue_shift_table<T>(p);
    const PositionPassArgs<T> pa = position_pass_args<T>(p);
    if (p->bf16) {
        Bf16Args ba{};
        ba.object_rows = p->OR; ba.object_columns = p->OC; ba.first = 0; ba.count = p->P; ba.scan = scan;
        ba.shifted = p->shifted.as<float2>(); ba.object = p->object.as<float2>();
        ba.amplitudes = p->amplitudes.as<float>(); ba.dpsi = p->dpsi.as<float2>(); ba.dpsi_first = 0;
        ba.error = p->error.as<double>();
        ba.c_planes = p->c_planes.as<uint16_t>(); ba.fault = p->fault.as<int>();
        timed(p, kPositionPass, 1, [&] { return launch_bf16(ba, p->sms, s); });
    } else if (p->fast) {
        Fast128Args fa{};
        fa.object_rows = p->OR; fa.object_columns = p->OC; fa.first = 0; fa.count = p->P; fa.scan = scan;
        fa.shifted = p->shifted.as<float2>(); fa.object = p->object.as<float2>();
        fa.amplitudes = p->amplitudes.as<float>(); fa.dpsi = p->dpsi.as<float2>(); fa.dpsi_first = 0;
        fa.accumulate = 0; fa.error = p->error.as<double>();
        fa.tw128 = p->tw_r.as<float2>();
        fa.partial_grad = p->partial_grad.as<float2>(); fa.partial_weight = p->partial_weight.as<float>();
        fa.fault = p->fault.as<int>();
        timed(p, kPositionPass, 1, [&] { return launch_fast128(fa, p->sms, s); });
    } else if (p->states > 1 && p->plane128) {
        if constexpr (std::is_same<T, double>::value) {  // every state's far field, the summed projection, inverses
            for (int st = 0; st < p->states; st++) {
                Plane128Args a = plane_args(p, kPlaneForward);
                a.in = p->shifted.as<double2>() + (size_t)st * p->classes * n; a.in_kind = kInputByClass;
                a.object = p->object.as<double2>(); a.out = p->dpsi.as<double2>() + (size_t)st * p->P * n;
                enqueue_plane(p, kPositionPass, a);
            }
            timed(p, kPositionPass, 1, [&] {
                return launch_mixed_factors(p->dpsi.as<double2>(), p->amplitudes.as<float>(), p->P, p->states, n,
                                            p->zero_pixel_infinite, p->error.as<double>(),
                                            p->mixed_factors64.as<double>(), s);
            });
            for (int st = 0; st < p->states; st++) {  // each state's residual: its far field x the common factor
                Plane128Args a = plane_args(p, kPlaneInverse);
                a.in = p->dpsi.as<double2>() + (size_t)st * p->P * n; a.out = const_cast<double2 *>(a.in);
                a.pointwise = kPointwiseFactorPlane; a.factors = p->mixed_factors64.as<double>();
                enqueue_plane(p, kPositionPass, a);
            }
        }
    } else if (p->states > 1) {
        if constexpr (std::is_same<T, double>::value) {
            MixedPassArgs ma{};
            ma.rows = p->R; ma.columns = p->C; ma.object_rows = p->OR; ma.object_columns = p->OC; ma.count = p->P;
            ma.states = p->states; ma.scan = scan; ma.shifted = p->shifted.as<double2>();
            ma.shifted_state_stride = (long long)p->classes * n; ma.object = p->object.as<double2>();
            ma.amplitudes = p->amplitudes.as<float>(); ma.dpsi = p->dpsi.as<double2>(); ma.error = p->error.as<double>();
            ma.zero_pixel_infinite = p->zero_pixel_infinite ? 1 : 0;
            int count = 0;
            timed(p, kPositionPass, 0, [&] { return launch_mixed_position_pass(ma, fft64(p), &count, s); });
            p->launches += count;
            if (p->timing) p->kind_launches[kPositionPass] += count;
        }
    } else if (p->plane128) {
        if constexpr (std::is_same<T, double>::value)
            enqueue_plane128(p, kPositionPass, p->shifted.as<double2>(), true, p->object.as<double2>(), false, true,
                             nullptr, false, p->dpsi.as<double2>());
    } else if (p->global64) {
        int count = 0;
        if constexpr (std::is_same<T, double>::value) {
            timed(p, kPositionPass, 0, [&] { return launch_position_pass_global(pa, fft64(p), &count, s); });
            p->launches += count;
            if (p->timing) p->kind_launches[kPositionPass] += count;
        }
    } else if (p->global32) {
        int count = 0;
        if constexpr (std::is_same<T, float>::value) {
            timed(p, kPositionPass, 0, [&] { return launch_position_pass_global32(pa, &count, s); });
            p->launches += count;
            if (p->timing) p->kind_launches[kPositionPass] += count;
        }
    } else if (!p->grouped_pass) {
        timed(p, kPositionPass, 1, [&] { return launch_position_pass<T>(pa, p->params.pass_shape, s); });
    }
}

// Object and probe gradient sums from dpsi: grad_o / weight_o (object), grad_p64 / weight_p64 (probe), maxima.
// The object gather's arguments over every tile and candidate of the plan.
template <typename T>
ObjectGatherArgs<T> object_gather_args(cubo_ptycho_plan *p) {
    const int n = p->n;
    ObjectGatherArgs<T> ga{};
    ga.rows = p->R; ga.columns = p->C; ga.object_rows = p->OR; ga.object_columns = p->OC; ga.n = n;
    ga.tiles_x = p->tiles_x; ga.tile_w = p->tile_w; ga.tile_h = p->tile_h; ga.tile_start = p->tile_start.as<int>(); ga.tile_list = p->tile_list.as<int>();
    ga.scan = ScanTables{p->rr.as<int>(), p->cc.as<int>(), p->cls.as<int>()};
    ga.shifted = p->shifted.as<C2<T>>(); ga.dpsi = p->dpsi.as<C2<T>>();
    ga.grad = p->grad_o.as<C2<T>>(); ga.weight = p->weight_o.as<T>(); ga.tile_max = p->tile_max.as<double>();
    ga.states = p->states;
    ga.dpsi_state_stride = (long long)p->P * n;
    ga.shifted_state_stride = (long long)p->classes * n;
    return ga;
}

// The probe gather's arguments over every position of the plan (probe state 0).
template <typename T>
ProbeGatherArgs<T> probe_gather_args(cubo_ptycho_plan *p) {
    ProbeGatherArgs<T> pg{};
    pg.rows = p->R; pg.columns = p->C; pg.object_rows = p->OR; pg.object_columns = p->OC; pg.n = p->n;
    pg.count = p->P; pg.groups = p->groups; pg.scan = ScanTables{p->rr.as<int>(), p->cc.as<int>(), p->cls.as<int>()};
    pg.object = p->object.as<C2<T>>(); pg.dpsi = p->dpsi.as<C2<T>>();
    pg.partial_grad = p->partial_grad.as<C2<T>>(); pg.partial_weight = p->partial_weight.as<T>();
    return pg;
}

template <typename T>
void enqueue_gathers(cubo_ptycho_plan *p) {
    cudaStream_t s = p->ctx->stream;
    ensure_dpsi<T>(p);
    const int n = p->n;
    const ObjectGatherArgs<T> ga = object_gather_args<T>(p);
    if (!p->grouped_gathers) timed(p, kObjectGather, 1, [&] { return launch_object_gather<T>(ga, p->tiles, s); });

    ProbeGatherArgs<T> pg = probe_gather_args<T>(p);
    for (int st = 0; st < p->states; st++) {  // each probe state's gradient from its own residuals
        pg.dpsi = p->dpsi.as<C2<T>>() + (size_t)st * p->P * n;
        if (!p->fast && !p->grouped_gathers)  // the 128 x 128 FP32 position pass already wrote per-CTA probe partials
            timed(p, kProbeGather, 1, [&] { return launch_probe_gather<T>(pg, s); });
        timed(p, kProbeReduce, 1, [&] {
            return launch_probe_reduce<T>(p->partial_grad.as<C2<T>>(), p->partial_weight.as<T>(), p->groups, n,
                                          p->grad_p64.as<double2>() + (size_t)st * n, p->weight_p64.as<double>(),
                                          p->probe_block_max.as<double>(), s);
        });
    }
    timed(p, kMaxReduce, 2, [&] {
        cudaError_t e = launch_max_reduce(p->tile_max.as<double>(), p->tiles, p->maxes.as<double>(), s);
        if (e == cudaSuccess) e = launch_max_reduce(p->probe_block_max.as<double>(), p->probe_blocks, p->maxes.as<double>() + 1, s);
        return e;
    });
}

// The position pass and both gathers band by band (the split-BF16 and the FP32 128 x 128 passes): each band's
// residuals are written into one band-sized buffer and read back by its object and probe gathers while they are still
// in L2; the gathers continue every sum from where the previous band left it, in the same candidate order, so the
// object gradient equals the unbanded gather's bit for bit.  The FP32 pass keeps its per-CTA probe partials across the
// bands (with bands of whole multiples of its 148 CTAs each CTA still sums its positions in the same order: the probe
// gradient is the unbanded one too); the split-BF16 form's probe gather groups each band's positions.  Then the probe
// partials' FP64 reduction and the maxima, as enqueue_gathers.
void enqueue_banded_pass_and_gathers(cubo_ptycho_plan *p) {
    cudaStream_t s = p->ctx->stream;
    const int n = p->n;
    const ScanTables scan{p->rr.as<int>(), p->cc.as<int>(), p->cls.as<int>()};
    enqueue_shift_table<float>(p);
    Fast128Args fa{};  // the FP32 128 x 128 pass: the probe-gradient partials accumulate in the pass, per CTA
    fa.object_rows = p->OR; fa.object_columns = p->OC; fa.scan = scan;
    fa.shifted = p->shifted.as<float2>(); fa.object = p->object.as<float2>();
    fa.amplitudes = p->amplitudes.as<float>(); fa.dpsi = p->dpsi_band.as<float2>(); fa.error = p->error.as<double>();
    fa.tw128 = p->tw_r.as<float2>();
    fa.partial_grad = p->partial_grad.as<float2>(); fa.partial_weight = p->partial_weight.as<float>();
    fa.fault = p->fault.as<int>();
    Bf16Args ba{};
    ba.object_rows = p->OR; ba.object_columns = p->OC; ba.scan = scan;
    ba.shifted = p->shifted.as<float2>(); ba.object = p->object.as<float2>();
    ba.amplitudes = p->amplitudes.as<float>(); ba.dpsi = p->dpsi_band.as<float2>(); ba.error = p->error.as<double>();
    ba.c_planes = p->c_planes.as<uint16_t>(); ba.fault = p->fault.as<int>();
    ObjectGatherArgs<float> ga{};
    ga.rows = p->R; ga.columns = p->C; ga.object_rows = p->OR; ga.object_columns = p->OC; ga.n = n;
    ga.tiles_x = p->tiles_x; ga.tile_w = p->tile_w; ga.tile_h = p->tile_h;
    ga.tile_start = p->tile_start.as<int>(); ga.tile_list = p->tile_list.as<int>();
    ga.scan = scan; ga.shifted = p->shifted.as<float2>(); ga.dpsi = p->dpsi_band.as<float2>();
    ga.grad = p->grad_o.as<float2>(); ga.weight = p->weight_o.as<float>(); ga.tile_max = p->tile_max.as<double>();
    ProbeGatherArgs<float> pg{};
    pg.rows = p->R; pg.columns = p->C; pg.object_rows = p->OR; pg.object_columns = p->OC; pg.n = n;
    pg.groups = p->groups; pg.scan = scan; pg.object = p->object.as<float2>(); pg.dpsi = p->dpsi_band.as<float2>();
    pg.partial_grad = p->partial_grad.as<float2>(); pg.partial_weight = p->partial_weight.as<float>();
    for (int b = 0; b < p->bands; b++) {
        const int first = b * p->band_size, count = std::min(p->band_size, p->P - first);
        if (p->bf16) {
            ba.first = first; ba.count = count; ba.dpsi_first = first;
            timed(p, kPositionPass, 1, [&] { return launch_bf16(ba, p->sms, s); });
        } else {
            fa.first = first; fa.count = count; fa.dpsi_first = first; fa.accumulate = b > 0 ? 1 : 0;
            timed(p, kPositionPass, 1, [&] { return launch_fast128(fa, p->sms, s); });
        }
        const int tiles = p->band_tile_offsets[b + 1] - p->band_tile_offsets[b];
        ga.band_tiles = p->band_tiles.as<int>() + p->band_tile_offsets[b];
        ga.band_first = first; ga.band_end = first + count;
        if (tiles > 0) timed(p, kObjectGather, 1, [&] { return launch_object_gather<float>(ga, tiles, s); });
        pg.first = first; pg.count = count; pg.accumulate = b > 0 ? 1 : 0;
        if (p->bf16) timed(p, kProbeGather, 1, [&] { return launch_probe_gather<float>(pg, s); });
    }
    timed(p, kProbeReduce, 1, [&] {
        return launch_probe_reduce<float>(p->partial_grad.as<float2>(), p->partial_weight.as<float>(), p->groups, n,
                                          p->grad_p64.as<double2>(), p->weight_p64.as<double>(),
                                          p->probe_block_max.as<double>(), s);
    });
    timed(p, kMaxReduce, 2, [&] {
        cudaError_t e = launch_max_reduce(p->tile_max.as<double>(), p->tiles, p->maxes.as<double>(), s);
        if (e == cudaSuccess) e = launch_max_reduce(p->probe_block_max.as<double>(), p->probe_blocks, p->maxes.as<double>() + 1, s);
        return e;
    });
}

// Position correction after the object update, before the amplitude cap (Ptychography.swift:371-377): the exit waves
// of a chunk of positions with the object before and after the update, their far fields, the per-position solve.
void enqueue_position_correction(cubo_ptycho_plan *p) {
    cudaStream_t s = p->ctx->stream;
    const ScanTables scan{p->rr.as<int>(), p->cc.as<int>(), p->cls.as<int>()};
    for (int first = 0; first < p->P; first += p->correction_chunk) {
        const int m = std::min(p->correction_chunk, p->P - first);
        if (p->plane128) {
            // the forward model's far field and the updated object's one row further (two forward plane launches),
            // then the one column further with the solve of every position in the same launch
            for (int v = 0; v < 3; v++) {
                Plane128Args a = plane_args(p, kPlaneForward);
                a.first = first; a.count = m; a.in = p->shifted.as<double2>(); a.in_kind = kInputByClass;
                a.object = v == 0 ? p->object_before.as<double2>() : p->object.as<double2>();
                a.object_row_offset = v == 1 ? 1 : 0; a.object_column_offset = v == 2 ? 1 : 0;
                a.out = p->far64.as<double2>(); a.out_stride = 2; a.out_offset = v - 2LL * first;
                if (v == 2) {
                    a.pointwise = kPointwiseSolve; a.out_offset = 0; a.far = p->far64.as<double2>();
                    a.positions = p->positions64.as<double>(); a.initial = p->initial64.as<double>();
                    a.position_count = p->P; a.position_step_size = p->params.position_step_size;
                    a.limit_update = p->limit_update; a.limit_total = p->limit_total;
                    a.position_bad = p->position_bad.as<int>();
                }
                enqueue_plane(p, kPositionCorrection, a);
            }
            continue;
        }
        timed(p, kPositionCorrection, 3, [&] {
            cudaError_t e = launch_position_exit_waves(p->shifted.as<double2>(), scan, p->object_before.as<double2>(),
                                                       p->object.as<double2>(), first, m, p->R, p->C, p->OR, p->OC,
                                                       p->far64.as<double2>(), s);
            if (e == cudaSuccess) e = launch_fft2_f64(fft64(p), p->far64.as<double2>(), 3 * m, false, s);
            if (e == cudaSuccess)
                e = launch_position_solve(p->far64.as<double2>(), p->amplitudes.as<float>(), first, m, p->n,
                                          p->positions64.as<double>(), p->initial64.as<double>(), p->P,
                                          p->params.position_step_size, p->limit_update, p->limit_total,
                                          p->position_bad.as<int>(), s);
            return e;
        });
    }
}

// The rest of an iteration once the gradient sums are in: updates, constraints, position correction, error.
template <typename T>
void enqueue_iteration_tail(cubo_ptycho_plan *p) {
    cudaStream_t s = p->ctx->stream;
    const cubo_ptycho_params &pp = p->params;
    const bool correct = std::is_same<T, double>::value && p->correct_positions;
    if (correct)
        check(cudaMemcpyAsync(p->object_before.ptr, p->object.ptr, (size_t)p->objects * sizeof(double2),
                              cudaMemcpyDeviceToDevice, s), "copy object");
    // the mixed-state engine always applies the threshold (PtychographyEngines.swift:209)
    const bool threshold = p->states > 1 || pp.constrain_object_amplitude;
    const int cap = !correct && threshold ? 1 : 0, pure = !correct && pp.pure_phase_object ? 1 : 0;
    timed(p, kObjectUpdate, 1, [&] {
        return launch_object_update<T>(p->object.as<C2<T>>(), p->grad_o.as<C2<T>>(), p->weight_o.as<T>(),
                                       (int)p->objects, p->maxes.as<double>(), pp.step_size, pp.normalization_minimum,
                                       cap, pure, s);
    });
    if (correct) {
        enqueue_position_correction(p);
        if (pp.constrain_object_amplitude || pp.pure_phase_object)
            timed(p, kObjectUpdate, 1, [&] {
                return launch_object_cap<T>(p->object.as<C2<T>>(), (int)p->objects, pp.pure_phase_object ? 1 : 0, s);
            });
        p->scan_stale = true;
    }
    enqueue_probe_side(p);
    if (correct && pp.constrain_positions_center_of_mass)  // Ptychography.swift:398-401
        timed(p, kPositionCorrection, 1, [&] {
            return launch_position_center(p->positions64.as<double>(), p->P, p->initial_mean_row,
                                          p->initial_mean_column, s);
        });
    timed(p, kErrorReduce, 2, [&] {
        return launch_error_reduce(p->error.as<double>(), p->error_count, p->divisor, p->errors.as<double>(),
                                   p->iteration.as<int>(), p->error_scratch.as<double>(), s);
    });
}

template <typename T>
void enqueue_iteration(cubo_ptycho_plan *p) {
    if (p->banded) {
        enqueue_banded_pass_and_gathers(p);
    } else {
        enqueue_position_pass<T>(p);
        enqueue_gathers<T>(p);
    }
    enqueue_iteration_tail<T>(p);
}

// One multislice iteration (MultislicePtychography.reconstruct, PtychographyEngines.swift:495-585), FP64.  The object
// holds the slices [slice][row][column]; waves64 the waves entering slices 1 .. L-1 ([slice - 1][position][pixel]; the
// wave entering slice 0 is the shifted probe, read from the shift table); dpsi the exit wave of the last slice, then
// its residual chi, then chi carried back through the slices.
void enqueue_multislice_iteration(cubo_ptycho_plan *p) {
    cudaStream_t s = p->ctx->stream;
    const cubo_ptycho_params &pp = p->params;
    const int n = p->n, P = p->P, L = p->slices;
    const long long plane = p->objects, planes = (long long)P * n;
    const double inv_n = 1.0 / n;
    const ScanTables scan{p->rr.as<int>(), p->cc.as<int>(), p->cls.as<int>()};
    const ScanTables own{p->rr.as<int>(), p->cc.as<int>(), p->ident.as<int>()};  // class p = position p
    double2 *obj = p->object.as<double2>(), *chi = p->dpsi.as<double2>(), *waves = p->waves64.as<double2>();
    const double2 *shifted = p->shifted.as<double2>(), *props = p->props64.as<double2>();
    const double2 *factors = p->prop_factors64.as<double2>();
    const Fft2Plan64 f = fft64(p);
    enqueue_shift_table<double>(p);
    if (p->plane128) {  // forward and detector, one plane launch per slice
        for (int sl = 0; sl < L; sl++) {
            const double2 *in = sl == 0 ? shifted : waves + (size_t)(sl - 1) * planes;
            const bool last = sl == L - 1;
            enqueue_plane128(p, kPositionPass, in, sl == 0, obj + (size_t)sl * plane, false, last,
                             last ? nullptr : factors + (size_t)sl * 256, false, last ? chi : waves + (size_t)sl * planes);
        }
    } else {
    // forward (:503-515): exit_s = wave_s x O_s; wave_{s+1} = IFFT(FFT(exit_s) x prop_s / n)
    timed(p, kPositionPass, 6 * (L - 1) + 1, [&] {
        cudaError_t e = cudaSuccess;
        for (int sl = 0; sl < L && e == cudaSuccess; sl++) {
            const bool last = sl == L - 1;
            double2 *target = last ? chi : waves + (size_t)sl * planes;
            if (sl == 0)
                e = launch_patch_multiply(shifted, true, obj, false, scan, 0, P, p->R, p->C, p->OR, p->OC, target, s);
            else
                e = launch_patch_multiply(waves + (size_t)(sl - 1) * planes, false, obj + (size_t)sl * plane, false,
                                          scan, 0, P, p->R, p->C, p->OR, p->OC, target, s);
            if (last) break;
            if (e == cudaSuccess) e = launch_fft2_f64(f, target, P, false, s);
            if (e == cudaSuccess) e = launch_spectrum_multiply(target, P, n, props + (size_t)sl * n, false, inv_n, s);
            if (e == cudaSuccess) e = launch_fft2_f64(f, target, P, true, s);
        }
        return e;
    });
    // detector (:516-524): the projection of the last exit wave's far field, chi its inverse transform
    PositionPassArgs<double> pa{};
    pa.rows = p->R; pa.columns = p->C; pa.object_rows = p->OR; pa.object_columns = p->OC; pa.n = n;
    pa.first = 0; pa.count = P; pa.scan = scan; pa.amplitudes = p->amplitudes.as<float>(); pa.dpsi = chi;
    pa.error = p->error.as<double>(); pa.inv_n = inv_n;
    timed(p, kPositionPass, 5, [&] {
        cudaError_t e = launch_fft2_f64(f, chi, P, false, s);
        if (e == cudaSuccess) e = launch_project_global(pa, s);
        if (e == cudaSuccess) e = launch_fft2_f64(f, chi, P, true, s);
        return e;
    });
    }
    // backward (:526-545): slice s's gradient from its entering wave and chi, chi x conj(O_s) carried back one slice;
    // at slice 0 the probe gradient from conj(O_0) chi
    ObjectGatherArgs<double> ga{};
    ga.rows = p->R; ga.columns = p->C; ga.object_rows = p->OR; ga.object_columns = p->OC; ga.n = n;
    ga.tiles_x = p->tiles_x; ga.tile_w = p->tile_w; ga.tile_h = p->tile_h;
    ga.tile_start = p->tile_start.as<int>(); ga.tile_list = p->tile_list.as<int>(); ga.dpsi = chi;
    for (int sl = L - 1; sl >= 0; sl--) {
        ga.scan = sl == 0 ? scan : own;
        ga.shifted = sl == 0 ? shifted : waves + (size_t)(sl - 1) * planes;
        ga.grad = p->grad_o.as<double2>() + (size_t)sl * plane;
        ga.weight = p->weight_o.as<double>() + (size_t)sl * plane;
        ga.tile_max = p->tile_max.as<double>() + (size_t)sl * p->tiles;
        timed(p, kObjectGather, 1, [&] { return launch_object_gather<double>(ga, p->tiles, s); });
        if (sl == 0) break;
        if (p->plane128) {
            enqueue_plane128(p, kBackPropagation, chi, false, obj + (size_t)sl * plane, true, false,
                             factors + (size_t)(sl - 1) * 256, true, chi);
            continue;
        }
        timed(p, kBackPropagation, 6, [&] {
            cudaError_t e = launch_patch_multiply(chi, false, obj + (size_t)sl * plane, true, scan, 0, P, p->R, p->C,
                                                  p->OR, p->OC, chi, s);
            if (e == cudaSuccess) e = launch_fft2_f64(f, chi, P, false, s);
            if (e == cudaSuccess) e = launch_spectrum_multiply(chi, P, n, props + (size_t)(sl - 1) * n, true, inv_n, s);
            if (e == cudaSuccess) e = launch_fft2_f64(f, chi, P, true, s);
            return e;
        });
    }
    ProbeGatherArgs<double> pg{};
    pg.rows = p->R; pg.columns = p->C; pg.object_rows = p->OR; pg.object_columns = p->OC; pg.n = n;
    pg.count = P; pg.groups = p->groups; pg.scan = scan; pg.object = obj; pg.dpsi = chi;
    pg.partial_grad = p->partial_grad.as<double2>(); pg.partial_weight = p->partial_weight.as<double>();
    timed(p, kProbeGather, 1, [&] { return launch_probe_gather<double>(pg, s); });
    timed(p, kProbeReduce, 1, [&] {
        return launch_probe_reduce<double>(pg.partial_grad, pg.partial_weight, p->groups, n, p->grad_p64.as<double2>(),
                                           p->weight_p64.as<double>(), p->probe_block_max.as<double>(), s);
    });
    timed(p, kMaxReduce, L + 1, [&] {
        cudaError_t e = cudaSuccess;
        for (int sl = 0; sl < L && e == cudaSuccess; sl++)
            e = launch_max_reduce(p->tile_max.as<double>() + (size_t)sl * p->tiles, p->tiles,
                                  p->slice_max.as<double>() + sl, s);
        if (e == cudaSuccess)
            e = launch_max_reduce(p->probe_block_max.as<double>(), p->probe_blocks, p->maxes.as<double>() + 1, s);
        return e;
    });
    // updates (:547-572): each slice with its own maximum weight; identical slices averaged before the threshold,
    // which always applies
    const bool identical = p->identical_slices;
    timed(p, kObjectUpdate, L + (identical ? 2 : 0), [&] {
        cudaError_t e = cudaSuccess;
        for (int sl = 0; sl < L && e == cudaSuccess; sl++)
            e = launch_object_update<double>(obj + (size_t)sl * plane, p->grad_o.as<double2>() + (size_t)sl * plane,
                                             p->weight_o.as<double>() + (size_t)sl * plane, (int)plane,
                                             p->slice_max.as<double>() + sl, pp.step_size, pp.normalization_minimum,
                                             identical ? 0 : 1, !identical && pp.pure_phase_object ? 1 : 0, s);
        if (identical && e == cudaSuccess) e = launch_average_slices(obj, L, plane, s);
        if (identical && e == cudaSuccess)
            e = launch_object_cap<double>(obj, (int)(L * plane), pp.pure_phase_object ? 1 : 0, s);
        return e;
    });
    enqueue_probe_side(p);
    timed(p, kErrorReduce, 2, [&] {
        return launch_error_reduce(p->error.as<double>(), p->error_count, p->divisor, p->errors.as<double>(),
                                   p->iteration.as<int>(), p->error_scratch.as<double>(), s);
    });
}

// A sharded iteration's first half (the plan holds one band of the positions): shifted probes, the position pass and the
// gathers leave this band's object and probe gradient sums and weights, and its summed squared error in shard_loss, for
// the caller to sum over the bands (Ptychography.swift:298-359, split at the accumulations).
template <typename T>
void enqueue_shard_gradients(cubo_ptycho_plan *p) {
    cudaStream_t s = p->ctx->stream;
    enqueue_position_pass<T>(p);
    enqueue_gathers<T>(p);
    check(cudaMemsetAsync(p->shard_counter.ptr, 0, sizeof(int), s), "memset");
    timed(p, kErrorReduce, 2, [&] {
        return launch_error_reduce(p->error.as<double>(), p->error_count, 1.0, p->shard_loss.as<double>(),
                                   p->shard_counter.as<int>(), p->error_scratch.as<double>(), s);
    });
}

// Its second half, once the gradient sums and weights hold every band's: the maxima of the summed weights, then the
// object and probe updates with their constraints, as one iteration does (Ptychography.swift:360-399).
template <typename T>
void enqueue_shard_update(cubo_ptycho_plan *p) {
    cudaStream_t s = p->ctx->stream;
    const cubo_ptycho_params &pp = p->params;
    timed(p, kMaxReduce, 2, [&] {
        cudaError_t e = launch_max_values<T>(p->weight_o.as<T>(), p->objects, p->maxes.as<double>(), s);
        if (e == cudaSuccess) e = launch_max_values<double>(p->weight_p64.as<double>(), p->n, p->maxes.as<double>() + 1, s);
        return e;
    });
    const bool threshold = p->states > 1 || pp.constrain_object_amplitude;
    timed(p, kObjectUpdate, 1, [&] {
        return launch_object_update<T>(p->object.as<C2<T>>(), p->grad_o.as<C2<T>>(), p->weight_o.as<T>(),
                                       (int)p->objects, p->maxes.as<double>(), pp.step_size, pp.normalization_minimum,
                                       threshold ? 1 : 0, pp.pure_phase_object ? 1 : 0, s);
    });
    enqueue_probe_side(p);
}

// The positions on the device after position correction: [rows | columns].
std::vector<double> download_positions(cubo_ptycho_plan *p) {
    std::vector<double> v((size_t)2 * p->P);
    int bad = 0;
    check(cudaMemcpyAsync(v.data(), p->positions64.ptr, v.size() * sizeof(double), cudaMemcpyDeviceToHost, p->ctx->stream),
          "download positions");
    check(cudaMemcpyAsync(&bad, p->position_bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, p->ctx->stream), "download");
    check(cudaStreamSynchronize(p->ctx->stream), "position correction");
    if (bad & 2) fail(CUBO_PTYCHO_CUDA_ERROR, "object-gather candidate lists outgrew their capacity");
    if (bad) fail(CUBO_PTYCHO_INVALID_INPUT, "a corrected position left the representable range");
    return v;
}

// Scan tables for the positions position correction moved (the next iteration's forward model uses them), built on the
// device without waiting: centres and one shift class per position, their phase ramps, the candidate lists (counted,
// scanned and listed in a fixed order, so the lists equal the host's).
void refresh_scan(cubo_ptycho_plan *p) {
    if (!p->correct_positions || !p->scan_stale) return;
    cudaStream_t s = p->ctx->stream;
    const int P = p->P;
    if (p->tile_counts.bytes < (size_t)p->tiles * sizeof(int))
        check(p->tile_counts.alloc((size_t)p->tiles * sizeof(int)), "cudaMalloc");
    timed(p, kPositionCorrection, 5, [&] {
        cudaError_t e = launch_scan_tables(p->positions64.as<double>(), P, p->OR, p->OC, p->rr.as<int>(),
                                           p->cc.as<int>(), p->cls.as<int>(), p->fractions64.as<double2>(), s);
        if (e == cudaSuccess)
            e = launch_ramp_table(p->fractions64.as<double2>(), P, p->R, p->C, p->ramps_r64.as<double2>(),
                                  p->ramps_c64.as<double2>(), s);
        if (e == cudaSuccess)
            e = launch_tile_lists(p->rr.as<int>(), p->cc.as<int>(), P, p->R, p->C, p->OR, p->OC, p->tile_w, p->tile_h,
                                  p->tiles_x, p->tiles, p->tile_counts.as<int>(), nullptr, nullptr, 0, s);
        if (e == cudaSuccess)
            e = launch_exclusive_scan(p->tile_counts.as<int>(), p->tiles, p->tile_start.as<int>(), p->tile_capacity,
                                      p->position_bad.as<int>(), s);
        if (e == cudaSuccess)
            e = launch_tile_lists(p->rr.as<int>(), p->cc.as<int>(), P, p->R, p->C, p->OR, p->OC, p->tile_w, p->tile_h,
                                  p->tiles_x, p->tiles, nullptr, p->tile_start.as<int>(), p->tile_list.as<int>(),
                                  (int)std::min<long long>(p->tile_capacity, INT32_MAX), s);
        return e;
    });
    p->scan_stale = false;
}

void enqueue_iterations(cubo_ptycho_plan *p, int iterations) {
    ensure_errors(p, p->iterations_done + iterations);
    if (iterations > 0) p->tape_valid = false;
    for (int i = 0; i < iterations; i++) {
        refresh_scan(p);
        if (p->multislice) enqueue_multislice_iteration(p);
        else if (p->fp64) enqueue_iteration<double>(p);
        else enqueue_iteration<float>(p);
        p->iterations_done++;
    }
}

}  // namespace

// ------------------------------------------------------------------------------------------------ C ABI

namespace {
int run_guarded(cubo_ptycho_context *ctx, const std::function<void()> &body) {
    if (!ctx) return CUBO_PTYCHO_INVALID_INPUT;
    try {
        cudaError_t e = cudaSetDevice(ctx->device);
        if (e != cudaSuccess) fail(CUBO_PTYCHO_CUDA_ERROR, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
        body();
        ctx->last_error.clear();
        return CUBO_PTYCHO_OK;
    } catch (const Failure &f) {
        ctx->last_error = f.message;
        return f.status;
    } catch (const std::bad_alloc &) {
        ctx->last_error = "host out of memory";
        return CUBO_PTYCHO_OUT_OF_MEMORY;
    }
}
}  // namespace

extern "C" {

void cubo_ptycho_params_default(cubo_ptycho_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->iterations = 8;
    p->step_size = 0.5;
    p->normalization_minimum = 1;
    p->constrain_object_amplitude = 1;
    p->probe_amplitude_relative_radius = 0.5;
    p->probe_amplitude_relative_width = 0.05;
    p->error_normalization = CUBO_PTYCHO_ERRORS_SUPPLIED_AMPLITUDE_ENERGY;
    p->form = CUBO_PTYCHO_FORM_FP32;
    p->position_step_size = 0.5;  // PtychographyPositionCorrection defaults (Ptychography.swift:68-69)
    p->position_row_sampling = std::numeric_limits<double>::quiet_NaN();
    p->position_column_sampling = std::numeric_limits<double>::quiet_NaN();
}

int cubo_ptycho_create(int device, cubo_ptycho_context **out) {
    if (!out) return CUBO_PTYCHO_INVALID_INPUT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return CUBO_PTYCHO_NO_DEVICE;
    }
    if (device < 0 || device >= count) return CUBO_PTYCHO_INVALID_INPUT;
    auto *ctx = new (std::nothrow) cubo_ptycho_context();
    if (!ctx) return CUBO_PTYCHO_OUT_OF_MEMORY;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return CUBO_PTYCHO_CUDA_ERROR;
    }
    BlockCache::get().context_created(device);
    *out = ctx;
    return CUBO_PTYCHO_OK;
}

int cubo_ptycho_destroy(cubo_ptycho_context *ctx) {
    if (!ctx) return CUBO_PTYCHO_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
    BlockCache::get().context_destroyed(ctx->device);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    delete ctx;
    return CUBO_PTYCHO_OK;
}

const char *cubo_ptycho_last_error(const cubo_ptycho_context *ctx) {
    return ctx ? ctx->last_error.c_str() : "no context";
}

void *cubo_ptycho_stream(cubo_ptycho_context *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int cubo_ptycho_synchronize(cubo_ptycho_context *ctx) {
    return run_guarded(ctx, [&] { check(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize"); });
}

}  // extern "C"

namespace {
// cubo_ptycho_plan_create, and the mixed-state engine's plan when `mixed` is given.
// MultislicePtychography.propagators (PtychographyEngines.swift:427-442): per thickness dz the Fresnel kernel
// exp(-i pi lambda dz (kr^2 + kc^2)), k = fftfreq / sampling, [thickness][row][column].
std::vector<double2> fresnel_propagators(int rows, int columns, double row_sampling, double column_sampling,
                                         double wavelength, int count, const double *thicknesses) {
    const bool ok = rows > 1 && columns > 1 && std::isfinite(row_sampling) && row_sampling > 0 &&
                    std::isfinite(column_sampling) && column_sampling > 0 && std::isfinite(wavelength) &&
                    wavelength > 0 && count > 0 && thicknesses != nullptr;
    if (!ok) fail(CUBO_PTYCHO_INVALID_INPUT, "propagators: sides above 1, positive finite samplings and wavelength, "
                                             "at least one thickness");
    for (int i = 0; i < count; i++)
        if (!std::isfinite(thicknesses[i])) fail(CUBO_PTYCHO_INVALID_INPUT, "propagators: thickness not finite");
    const size_t n = (size_t)rows * columns;
    std::vector<double2> out((size_t)count * n);
    for (int i = 0; i < count; i++)
        for (int r = 0; r < rows; r++) {
            const double kr = frequency(r, rows) / row_sampling;
            for (int c = 0; c < columns; c++) {
                const double kc = frequency(c, columns) / column_sampling;
                const double phase = -kPi * wavelength * thicknesses[i] * (kr * kr + kc * kc);
                out[(size_t)i * n + (size_t)r * columns + c] = make_double2(std::cos(phase), std::sin(phase));
            }
        }
    return out;
}

// The same kernels as separable factors: exp(-i pi lambda dz kr^2) per row frequency and exp(-i pi lambda dz kc^2)
// per column frequency, [thickness][rows + columns]; their product is the propagator.
std::vector<double2> fresnel_factors(int rows, int columns, double row_sampling, double column_sampling,
                                     double wavelength, int count, const double *thicknesses) {
    std::vector<double2> out((size_t)count * (rows + columns));
    for (int i = 0; i < count; i++) {
        double2 *f = out.data() + (size_t)i * (rows + columns);
        for (int r = 0; r < rows; r++) {
            const double kr = frequency(r, rows) / row_sampling;
            const double phase = -kPi * wavelength * thicknesses[i] * (kr * kr);
            f[r] = make_double2(std::cos(phase), std::sin(phase));
        }
        for (int c = 0; c < columns; c++) {
            const double kc = frequency(c, columns) / column_sampling;
            const double phase = -kPi * wavelength * thicknesses[i] * (kc * kc);
            f[rows + c] = make_double2(std::cos(phase), std::sin(phase));
        }
    }
    return out;
}

int create_plan(cubo_ptycho_context *ctx, const cubo_ptycho_problem *pr, const cubo_ptycho_params *pp,
                const cubo_ptycho_mixed_params *mixed, const cubo_ptycho_multislice_params *multi,
                cubo_ptycho_plan **out) {
    if (!out) return CUBO_PTYCHO_INVALID_INPUT;
    *out = nullptr;
    std::unique_ptr<cubo_ptycho_plan> plan;
    const int status = run_guarded(ctx, [&] {
        double divisor = 0;
        validate(pr, pp, &divisor);
        if (mixed) {  // PtychographyEngines.swift:159-166; the engine is the reference's Double one
            if (!(mixed->states >= 1 && mixed->states <= kMaxStates))
                fail(CUBO_PTYCHO_INVALID_INPUT, "probe states: 1 to " + std::to_string(kMaxStates));
            if (pp->form != CUBO_PTYCHO_FORM_FP64)
                fail(CUBO_PTYCHO_INVALID_INPUT, "the mixed-state engine runs in the FP64 form (the reference's is Double)");
            if (pp->has_position_correction) fail(CUBO_PTYCHO_INVALID_INPUT, "no position correction in mixed state");
            if (mixed->zero_pixel_error != CUBO_PTYCHO_ZERO_PIXEL_REFERENCE &&
                mixed->zero_pixel_error != CUBO_PTYCHO_ZERO_PIXEL_FINITE)
                fail(CUBO_PTYCHO_INVALID_INPUT, "zero-pixel error mode");
            if (!line_fft_supported(pr->rows, pr->columns))
                fail(CUBO_PTYCHO_UNSUPPORTED, "detector sides above the line transform's 4096");
        }
        std::vector<double2> props;
        if (multi) {  // PtychographyEngines.swift:471-480; the engine is the reference's Double one
            if (mixed) fail(CUBO_PTYCHO_INVALID_INPUT, "one engine per plan");
            if (!(multi->slices >= 1 && multi->slices <= 1024))
                fail(CUBO_PTYCHO_INVALID_INPUT, "object slices: 1 to 1024");
            if (multi->slices > 1 && !multi->slice_thicknesses)
                fail(CUBO_PTYCHO_INVALID_INPUT, "slice thicknesses: one per gap between slices");
            if (pp->form != CUBO_PTYCHO_FORM_FP64)
                fail(CUBO_PTYCHO_INVALID_INPUT, "the multislice engine runs in the FP64 form (the reference's is Double)");
            if (pp->has_position_correction) fail(CUBO_PTYCHO_INVALID_INPUT, "no position correction in multislice");
            const double zero = 0.0;  // one slice: the propagator of a zero thickness, validated but never applied
            props = fresnel_propagators(pr->rows, pr->columns, multi->row_sampling, multi->column_sampling,
                                        multi->wavelength, std::max(1, multi->slices - 1),
                                        multi->slices > 1 ? multi->slice_thicknesses : &zero);
            if (!line_fft_supported(pr->rows, pr->columns))
                fail(CUBO_PTYCHO_UNSUPPORTED, "detector sides above the line transform's 4096");
        }
        plan.reset(new cubo_ptycho_plan());
        cubo_ptycho_plan *p = plan.get();
        p->ctx = ctx;
        p->R = pr->rows; p->C = pr->columns; p->OR = pr->object_rows; p->OC = pr->object_columns; p->P = pr->count;
        p->n = p->R * p->C;
        if (mixed) {
            p->states = mixed->states;
            p->orthogonalize = mixed->orthogonalize_probes != 0;
            p->zero_pixel_infinite = mixed->zero_pixel_error == CUBO_PTYCHO_ZERO_PIXEL_REFERENCE;
        }
        if (multi) {
            p->slices = multi->slices;
            p->multislice = true;
            p->identical_slices = multi->identical_slices != 0;
        }
        p->objects = (long long)p->OR * p->OC;
        p->params = *pp;
        if (pp->probe_support_mask) p->mask.assign(pp->probe_support_mask, pp->probe_support_mask + p->n);
        for (auto &m : p->mask) m = m ? 1 : 0;
        p->params.probe_support_mask = nullptr;
        p->divisor = divisor;
        p->fp64 = pp->form == CUBO_PTYCHO_FORM_FP64;
        if (pp->form == CUBO_PTYCHO_FORM_SPLIT_BF16 && !bf16_applicable(p->R, p->C))
            fail(CUBO_PTYCHO_UNSUPPORTED, "the split-BF16 tensor-core form needs a 128 x 128 detector");
        int optin = 0;
        check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device), "attribute");
        const bool smem_pass = position_pass_supported(p->n, p->fp64) &&
                               position_pass_smem(p->n, p->R, p->C, p->fp64) <= (size_t)optin;
        // FP64 planes too large for one CTA go through global memory (any size the line transform takes)
        p->global64 = p->fp64 && (!smem_pass || pp->variant == CUBO_PTYCHO_VARIANT_GLOBAL || p->states > 1 ||
                                  p->multislice);
        // 128 x 128 FP64 planes: the clustered plane launches (not with the generic variant)
        p->plane128 = p->global64 && p->R == 128 && p->C == 128 && pp->variant != CUBO_PTYCHO_VARIANT_GENERIC;
        if (p->plane128) {
            check(configure_plane128(), "configure plane transform");
            p->plane_cluster = plane128_cluster();
        }
        // FP32 planes too large for one CTA (or any size with the global variant): rows and columns through global memory
        p->global32 = !p->fp64 && pp->form != CUBO_PTYCHO_FORM_SPLIT_BF16 &&
                      (!smem_pass || pp->variant == CUBO_PTYCHO_VARIANT_GLOBAL) && global32_applicable(p->R, p->C);
        if (p->global32) check(configure_global32(), "configure global-memory FP32 pass");
        if (!smem_pass && !(p->global64 && line_fft_supported(p->R, p->C)) && !p->global32)
            fail(CUBO_PTYCHO_UNSUPPORTED, "detector of " + std::to_string(p->n) + " pixels exceeds the shared-memory "
                                              "transform of this form");
        check(configure_kernels(), "configure kernels");
        check(configure_fft_lines(), "configure line transforms");
        p->bf16 = pp->form == CUBO_PTYCHO_FORM_SPLIT_BF16;
        if (p->bf16) check(configure_bf16(), "configure split-BF16 kernel");
        p->fast = !p->fp64 && !p->bf16 && !p->global32 && pp->variant != CUBO_PTYCHO_VARIANT_GENERIC &&
                  fast128_applicable(p->R, p->C);
        if (p->fast) check(configure_fast128(), "configure 128 x 128 kernel");
        check(cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, ctx->device), "attribute");
        if (p->bf16 || p->fast) {
            // CUBO_PTYCHO_BAND_POSITIONS = k > 0 runs the iteration in bands of k positions (their residuals in one
            // band-sized buffer, read back by the band's gathers while still in L2); unset or 0: one pass over every
            // position.  Bands of 444 positions (three waves of the pass, 57 MB of residuals) measured 19.4 ms per
            // iteration at the 256^2-scan, 128^2-detector workload against 12.3 ms in one pass: each band's launches
            // cost more than the L2 reads save (the pass ~30 us more per launch than its share of one pass, the
            // gathers twice as long per position on band-sized grids), so one pass is the default.
            long long size = p->P;
            if (const char *env = std::getenv("CUBO_PTYCHO_BAND_POSITIONS")) {
                const long long v = std::atoll(env);
                if (v > 0) size = v;
            }
            p->band_size = (int)std::max<long long>(1, std::min<long long>(size, p->P));
            p->bands = (p->P + p->band_size - 1) / p->band_size;
            p->banded = p->bands > 1;
        }
        p->kind_ms.assign(kKinds, 0.0);
        p->kind_launches.assign(kKinds, 0);
        p->correct_positions = pp->has_position_correction != 0;  // before the scan tables: one class per position
        if (p->fp64) build_plan<double>(p, pr);
        else build_plan<float>(p, pr);
        if (p->plane128 && p->states > 1)
            check(p->mixed_factors64.alloc((size_t)p->P * p->n * sizeof(double)), "cudaMalloc mixed-state factors");
        if (p->multislice && p->slices > 1) {
            upload(p->props64, props, ctx->stream);
            if (p->plane128)
                upload(p->prop_factors64,
                       fresnel_factors(p->R, p->C, multi->row_sampling, multi->column_sampling, multi->wavelength,
                                       p->slices - 1, multi->slice_thicknesses),
                       ctx->stream);
        }
        p->positions_given.resize((size_t)2 * p->P);
        std::copy(pr->position_rows, pr->position_rows + p->P, p->positions_given.begin());
        std::copy(pr->position_columns, pr->position_columns + p->P, p->positions_given.begin() + p->P);
        if (pp->has_position_correction) {
            p->correct_positions = true;
            position_limits(pp, &p->limit_update, &p->limit_total);
            double mr = 0, mc = 0;  // Ptychography.swift:270, summed in order
            for (int i = 0; i < p->P; i++) {
                mr += pr->position_rows[i];
                mc += pr->position_columns[i];
            }
            p->initial_mean_row = mr / (double)p->P;
            p->initial_mean_column = mc / (double)p->P;
            upload(p->positions64, p->positions_given, ctx->stream);
            upload(p->initial64, p->positions_given, ctx->stream);
            check(p->object_before.alloc((size_t)p->objects * sizeof(double2)), "cudaMalloc");
            check(p->position_bad.alloc(sizeof(int)), "cudaMalloc");
            check(cudaMemsetAsync(p->position_bad.ptr, 0, sizeof(int), ctx->stream), "memset");
            // far fields per position, FP64 (three; two with the clustered plane launches, which solve with the
            // third on chip): chunks of at most 1 GiB (2 GiB)
            const size_t per_position = (size_t)(p->plane128 ? 2 : 3) * p->n * sizeof(double2);
            const size_t budget = p->plane128 ? (2ull << 30) : (1ull << 30);
            p->correction_chunk = (int)std::max<size_t>(1, std::min<size_t>(p->P, budget / per_position));
            check(p->far64.alloc((size_t)p->correction_chunk * per_position), "cudaMalloc");
        }
        check(cudaStreamSynchronize(ctx->stream), "plan upload");
    });
    if (status == CUBO_PTYCHO_OK) *out = plan.release();
    return status;
}
}  // namespace

extern "C" {

int cubo_ptycho_plan_create(cubo_ptycho_context *ctx, const cubo_ptycho_problem *pr, const cubo_ptycho_params *pp,
                            cubo_ptycho_plan **out) {
    return create_plan(ctx, pr, pp, nullptr, nullptr, out);
}

void cubo_ptycho_mixed_params_default(cubo_ptycho_mixed_params *m) {
    if (!m) return;
    m->states = 1;
    m->orthogonalize_probes = 1;
    m->zero_pixel_error = CUBO_PTYCHO_ZERO_PIXEL_REFERENCE;
}

int cubo_ptycho_mixed_plan_create(cubo_ptycho_context *ctx, const cubo_ptycho_problem *pr,
                                  const cubo_ptycho_params *pp, const cubo_ptycho_mixed_params *mixed,
                                  cubo_ptycho_plan **out) {
    if (!mixed) return CUBO_PTYCHO_INVALID_INPUT;
    return create_plan(ctx, pr, pp, mixed, nullptr, out);
}

int cubo_ptycho_orthogonalize(cubo_ptycho_context *ctx, int states, int rows, int columns, double *re, double *im) {
    return run_guarded(ctx, [&] {  // MixedstatePtychography.orthogonalize (PtychographyEngines.swift:265-269)
        if (!re || !im) fail(CUBO_PTYCHO_INVALID_INPUT, "null probes");
        if (!(states >= 1 && states <= kMaxStates && rows > 1 && columns > 1 && (long long)rows * columns <= (1 << 26)))
            fail(CUBO_PTYCHO_INVALID_INPUT, "shape");
        const size_t n = (size_t)rows * columns, total = (size_t)states * n;
        std::vector<double2> v(total);
        for (size_t k = 0; k < total; k++) {
            if (!std::isfinite(re[k]) || !std::isfinite(im[k])) fail(CUBO_PTYCHO_INVALID_INPUT, "probe not finite");
            v[k] = make_double2(re[k], im[k]);
        }
        if (states == 1) return;
        cudaStream_t s = ctx->stream;
        DeviceBuffer probes, gram, mixing, scratch;
        upload(probes, v, s);
        check(gram.alloc((size_t)states * states * sizeof(double2)), "cudaMalloc");
        check(mixing.alloc((size_t)states * states * sizeof(double2)), "cudaMalloc");
        check(scratch.alloc(total * sizeof(double2)), "cudaMalloc");
        check(launch_orthogonalize(probes.as<double2>(), states, (int)n, gram.as<double2>(), mixing.as<double2>(),
                                   scratch.as<double2>(), s), "orthogonalize");
        check(cudaMemcpyAsync(v.data(), probes.ptr, total * sizeof(double2), cudaMemcpyDeviceToHost, s), "download");
        check(cudaStreamSynchronize(s), "orthogonalize");
        for (size_t k = 0; k < total; k++) {
            re[k] = v[k].x;
            im[k] = v[k].y;
        }
    });
}

int cubo_ptycho_mixed_reconstruct(cubo_ptycho_context *ctx, const cubo_ptycho_problem *pr,
                                  const cubo_ptycho_params *pp, const cubo_ptycho_mixed_params *mixed, double *ore,
                                  double *oim, double *pre, double *pim, double *errors) {
    if (!ctx) return CUBO_PTYCHO_INVALID_INPUT;
    if (!mixed || !ore || !oim || !pre || !pim || (pp && pp->iterations > 0 && !errors)) {
        ctx->last_error = "null input or output";
        return CUBO_PTYCHO_INVALID_INPUT;
    }
    cubo_ptycho_plan *plan = nullptr;
    int status = create_plan(ctx, pr, pp, mixed, nullptr, &plan);
    if (status != CUBO_PTYCHO_OK) return status;
    status = cubo_ptycho_plan_set_state(plan, ore, oim, pre, pim);
    if (status == CUBO_PTYCHO_OK) status = cubo_ptycho_plan_iterate(plan, pp->iterations, errors);
    if (status == CUBO_PTYCHO_OK) status = cubo_ptycho_plan_get_state(plan, ore, oim, pre, pim);
    const std::string message = ctx->last_error;
    cubo_ptycho_plan_destroy(plan);
    ctx->last_error = message;
    return status;
}

int cubo_ptycho_propagators(int rows, int columns, double row_sampling, double column_sampling, double wavelength,
                            int count, const double *thicknesses, double *re, double *im) {
    if (!re || !im) return CUBO_PTYCHO_INVALID_INPUT;
    try {
        const std::vector<double2> v =
            fresnel_propagators(rows, columns, row_sampling, column_sampling, wavelength, count, thicknesses);
        for (size_t k = 0; k < v.size(); k++) {
            re[k] = v[k].x;
            im[k] = v[k].y;
        }
    } catch (const Failure &f) {
        return f.status;
    } catch (const std::bad_alloc &) {
        return CUBO_PTYCHO_OUT_OF_MEMORY;
    }
    return CUBO_PTYCHO_OK;
}

int cubo_ptycho_multislice_plan_create(cubo_ptycho_context *ctx, const cubo_ptycho_problem *pr,
                                       const cubo_ptycho_params *pp, const cubo_ptycho_multislice_params *multi,
                                       cubo_ptycho_plan **out) {
    if (!multi) {
        if (out) *out = nullptr;
        return CUBO_PTYCHO_INVALID_INPUT;
    }
    return create_plan(ctx, pr, pp, nullptr, multi, out);
}

int cubo_ptycho_multislice_reconstruct(cubo_ptycho_context *ctx, const cubo_ptycho_problem *pr,
                                       const cubo_ptycho_params *pp, const cubo_ptycho_multislice_params *multi,
                                       double *ore, double *oim, double *pre, double *pim, double *errors) {
    if (!ctx) return CUBO_PTYCHO_INVALID_INPUT;
    if (!multi || !ore || !oim || !pre || !pim || (pp && pp->iterations > 0 && !errors)) {
        ctx->last_error = "null input or output";
        return CUBO_PTYCHO_INVALID_INPUT;
    }
    cubo_ptycho_plan *plan = nullptr;
    int status = create_plan(ctx, pr, pp, nullptr, multi, &plan);
    if (status != CUBO_PTYCHO_OK) return status;
    status = cubo_ptycho_plan_set_state(plan, ore, oim, pre, pim);
    if (status == CUBO_PTYCHO_OK) status = cubo_ptycho_plan_iterate(plan, pp->iterations, errors);
    if (status == CUBO_PTYCHO_OK) status = cubo_ptycho_plan_get_state(plan, ore, oim, pre, pim);
    const std::string message = ctx->last_error;
    cubo_ptycho_plan_destroy(plan);
    ctx->last_error = message;
    return status;
}

int cubo_ptycho_plan_destroy(cubo_ptycho_plan *plan) {
    if (!plan) return CUBO_PTYCHO_OK;
    cudaSetDevice(plan->ctx->device);
    cudaStreamSynchronize(plan->ctx->stream);
    delete plan;
    return CUBO_PTYCHO_OK;
}

int cubo_ptycho_plan_set_state(cubo_ptycho_plan *p, const double *ore, const double *oim, const double *pre,
                               const double *pim) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        if (!ore || !oim || !pre || !pim) fail(CUBO_PTYCHO_INVALID_INPUT, "null state");
        const long long object_values = (long long)p->slices * p->objects;  // every slice, [slice][row][column]
        for (long long j = 0; j < object_values; j++)
            if (!std::isfinite(ore[j]) || !std::isfinite(oim[j])) fail(CUBO_PTYCHO_INVALID_INPUT, "object not finite");
        const size_t probe_values = (size_t)p->states * p->n;  // every probe state, [state][row][column]
        for (size_t k = 0; k < probe_values; k++)
            if (!std::isfinite(pre[k]) || !std::isfinite(pim[k])) fail(CUBO_PTYCHO_INVALID_INPUT, "probe not finite");
        cudaStream_t s = p->ctx->stream;
        p->tape_valid = false;
        // through the context's pinned staging buffer: the probe (complex128), then the object in the plan's type
        const size_t object_bytes = (size_t)object_values * (p->fp64 ? sizeof(double2) : sizeof(float2));
        uint8_t *stage = static_cast<uint8_t *>(pinned_staging(p->ctx, probe_values * sizeof(double2) + object_bytes));
        double2 *probe = reinterpret_cast<double2 *>(stage);
        for (size_t k = 0; k < probe_values; k++) probe[k] = make_double2(pre[k], pim[k]);
        if (p->fp64) {
            double2 *o = reinterpret_cast<double2 *>(stage + probe_values * sizeof(double2));
            for (long long j = 0; j < object_values; j++) o[j] = make_double2(ore[j], oim[j]);
        } else {
            float2 *o = reinterpret_cast<float2 *>(stage + probe_values * sizeof(double2));
            for (long long j = 0; j < p->objects; j++) o[j] = make_float2((float)ore[j], (float)oim[j]);
        }
        check(cudaMemcpyAsync(p->probe64.ptr, probe, probe_values * sizeof(double2), cudaMemcpyHostToDevice, s),
              "upload probe");
        check(cudaMemcpyAsync(p->object.ptr, stage + probe_values * sizeof(double2), object_bytes,
                              cudaMemcpyHostToDevice, s), "upload object");
        check(cudaStreamSynchronize(s), "sync");
        // the initial Fourier amplitude for fixProbeAperture (PtychographyConstraints.swift:79-83)
        if (p->params.fix_probe_aperture) {
            check(cudaMemcpyAsync(p->scratch64.ptr, p->probe64.ptr, (size_t)p->n * sizeof(double2), cudaMemcpyDeviceToDevice, s), "copy");
            check(launch_fft2_f64(fft64(p), p->scratch64.as<double2>(), 1, false, s), "fft");
            check(launch_magnitude(p->scratch64.as<double2>(), p->aperture64.as<double>(), p->n, s), "magnitude");
            check(cudaStreamSynchronize(s), "sync");
        }
    });
}

int cubo_ptycho_plan_get_state(cubo_ptycho_plan *p, double *ore, double *oim, double *pre, double *pim) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        cudaStream_t s = p->ctx->stream;
        const size_t probe_values = (size_t)p->states * p->n;
        const size_t object_values = p->fp64 ? (size_t)p->slices * p->objects : (size_t)p->objects;
        const size_t object_bytes = object_values * (p->fp64 ? sizeof(double2) : sizeof(float2));
        uint8_t *stage = static_cast<uint8_t *>(pinned_staging(p->ctx, probe_values * sizeof(double2) + object_bytes));
        const double2 *probe = reinterpret_cast<const double2 *>(stage);
        check(cudaMemcpyAsync(stage, p->probe64.ptr, probe_values * sizeof(double2), cudaMemcpyDeviceToHost, s),
              "download probe");
        check(cudaMemcpyAsync(stage + probe_values * sizeof(double2), p->object.ptr, object_bytes,
                              cudaMemcpyDeviceToHost, s), "download object");
        check(cudaStreamSynchronize(s), "sync");
        if (p->fp64) {
            const double2 *o = reinterpret_cast<const double2 *>(stage + probe_values * sizeof(double2));
            for (size_t j = 0; j < object_values; j++) { if (ore) ore[j] = o[j].x; if (oim) oim[j] = o[j].y; }
        } else {
            const float2 *o = reinterpret_cast<const float2 *>(stage + probe_values * sizeof(double2));
            for (size_t j = 0; j < object_values; j++) { if (ore) ore[j] = o[j].x; if (oim) oim[j] = o[j].y; }
        }
        for (size_t k = 0; k < probe_values; k++) { if (pre) pre[k] = probe[k].x; if (pim) pim[k] = probe[k].y; }
    });
}

int cubo_ptycho_plan_get_positions(cubo_ptycho_plan *p, double *rows, double *columns) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        if (!rows || !columns) fail(CUBO_PTYCHO_INVALID_INPUT, "null output");
        const std::vector<double> v = p->correct_positions ? download_positions(p) : p->positions_given;
        std::copy(v.begin(), v.begin() + p->P, rows);
        std::copy(v.begin() + p->P, v.end(), columns);
    });
}

int cubo_ptycho_plan_enqueue(cubo_ptycho_plan *p, int iterations) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        if (iterations < 0) fail(CUBO_PTYCHO_INVALID_INPUT, "iterations");
        enqueue_iterations(p, iterations);
    });
}

int cubo_ptycho_plan_errors(cubo_ptycho_plan *p, int count, double *errors) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        if (count < 0 || count > p->iterations_done || (count > 0 && !errors)) fail(CUBO_PTYCHO_INVALID_INPUT, "count");
        check(cudaStreamSynchronize(p->ctx->stream), "sync");
        check_fault(p);
        if (count > 0)
            check(cudaMemcpy(errors, p->errors.as<double>() + (p->iterations_done - count), (size_t)count * sizeof(double),
                             cudaMemcpyDeviceToHost), "download errors");
    });
}

int cubo_ptycho_plan_enqueue_gradients(cubo_ptycho_plan *p) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        if (p->multislice || p->correct_positions)
            fail(CUBO_PTYCHO_UNSUPPORTED, "sharded iterations: single-slice and mixed-state plans without position correction");
        if (!p->shard_loss.ptr) {
            check(p->shard_loss.alloc(sizeof(double)), "cudaMalloc");
            check(p->shard_counter.alloc(sizeof(int)), "cudaMalloc");
        }
        p->tape_valid = false;
        if (p->fp64) enqueue_shard_gradients<double>(p);
        else enqueue_shard_gradients<float>(p);
    });
}

int cubo_ptycho_plan_gradient_buffers(cubo_ptycho_plan *p, void **grad_object, void **weight_object, void **grad_probe,
                                      void **weight_probe, void **loss, int *real_bytes) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        if (!p->shard_loss.ptr) fail(CUBO_PTYCHO_INVALID_INPUT, "no gradients enqueued on this plan yet");
        if (grad_object) *grad_object = p->grad_o.ptr;
        if (weight_object) *weight_object = p->weight_o.ptr;
        if (grad_probe) *grad_probe = p->grad_p64.ptr;
        if (weight_probe) *weight_probe = p->weight_p64.ptr;
        if (loss) *loss = p->shard_loss.ptr;
        if (real_bytes) *real_bytes = p->fp64 ? 8 : 4;
    });
}

int cubo_ptycho_plan_apply_gradients(cubo_ptycho_plan *p) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        if (!p->shard_loss.ptr) fail(CUBO_PTYCHO_INVALID_INPUT, "no gradients enqueued on this plan yet");
        if (p->fp64) enqueue_shard_update<double>(p);
        else enqueue_shard_update<float>(p);
    });
}

int cubo_ptycho_plan_iterate(cubo_ptycho_plan *p, int iterations, double *errors) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    int cancelled = 0;
    const int status = run_guarded(p->ctx, [&] {
        if (iterations < 0) fail(CUBO_PTYCHO_INVALID_INPUT, "iterations");
        const long long start = p->iterations_done;
        ensure_errors(p, start + iterations);
        for (int i = 0; i < iterations; i++) {
            if (p->params.cancel && *p->params.cancel) { cancelled = 1; break; }  // Ptychography.swift:281
            enqueue_iterations(p, 1);
            if (p->params.progress) {
                check(cudaStreamSynchronize(p->ctx->stream), "sync");
                p->params.progress(i + 1, iterations, p->params.progress_user);  // Ptychography.swift:401
            }
        }
        check(cudaStreamSynchronize(p->ctx->stream), "sync");
        check_fault(p);
        if (p->correct_positions) download_positions(p);  // a position out of range fails the call, as it throws
        if (!cancelled && errors && iterations > 0)
            check(cudaMemcpy(errors, p->errors.as<double>() + start, (size_t)iterations * sizeof(double),
                             cudaMemcpyDeviceToHost), "download errors");
    });
    if (status == CUBO_PTYCHO_OK && cancelled) {
        p->ctx->last_error = "cancelled";
        return CUBO_PTYCHO_CANCELLED;
    }
    return status;
}

int cubo_ptycho_reconstruct(cubo_ptycho_context *ctx, const cubo_ptycho_problem *pr, const cubo_ptycho_params *pp,
                            double *ore, double *oim, double *pre, double *pim, double *errors) {
    if (!ctx) return CUBO_PTYCHO_INVALID_INPUT;
    if (!ore || !oim || !pre || !pim || (pp && pp->iterations > 0 && !errors)) {
        ctx->last_error = "null output";
        return CUBO_PTYCHO_INVALID_INPUT;
    }
    cubo_ptycho_plan *plan = nullptr;
    int status = cubo_ptycho_plan_create(ctx, pr, pp, &plan);
    if (status != CUBO_PTYCHO_OK) return status;
    status = cubo_ptycho_plan_set_state(plan, ore, oim, pre, pim);
    if (status == CUBO_PTYCHO_OK) status = cubo_ptycho_plan_iterate(plan, pp->iterations, errors);
    if (status == CUBO_PTYCHO_OK) status = cubo_ptycho_plan_get_state(plan, ore, oim, pre, pim);
    if (status == CUBO_PTYCHO_OK && pp->position_rows_out && pp->position_columns_out)
        status = cubo_ptycho_plan_get_positions(plan, pp->position_rows_out, pp->position_columns_out);
    const std::string message = ctx->last_error;
    cubo_ptycho_plan_destroy(plan);
    ctx->last_error = message;
    return status;
}

}  // extern "C"

namespace {
template <typename T>
void enqueue_forward(cubo_ptycho_plan *p) {
    refresh_scan(p);
    enqueue_position_pass<T>(p);
    check(cudaMemsetAsync(p->loss_slot.ptr, 0, 2 * sizeof(double), p->ctx->stream), "memset");
    timed(p, kErrorReduce, 2, [&] {
        return launch_error_reduce(p->error.as<double>(), p->error_count, 1.0, p->loss_slot.as<double>(),
                                   reinterpret_cast<int *>(p->loss_slot.as<double>() + 1), p->error_scratch.as<double>(),
                                   p->ctx->stream);
    });
}

template <typename T>
void download_object_gradient(cubo_ptycho_plan *p, double scale, double *re, double *im) {
    std::vector<C2<T>> g((size_t)p->objects);
    check(cudaMemcpyAsync(g.data(), p->grad_o.ptr, g.size() * sizeof(C2<T>), cudaMemcpyDeviceToHost, p->ctx->stream),
          "download gradient");
    check(cudaStreamSynchronize(p->ctx->stream), "sync");
    for (long long j = 0; j < p->objects; j++) {
        if (re) re[j] = scale * (double)g[j].x;
        if (im) im[j] = scale * (double)g[j].y;
    }
}
}  // namespace

extern "C" {

int cubo_ptycho_plan_forward(cubo_ptycho_plan *p, double *loss) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        if (p->states > 1 || p->multislice) fail(CUBO_PTYCHO_UNSUPPORTED, "the adjoint pair is single-slice only");
        if (p->fp64) enqueue_forward<double>(p);
        else enqueue_forward<float>(p);
        p->tape_valid = true;
        double l = 0;
        check(cudaMemcpyAsync(&l, p->loss_slot.ptr, sizeof(double), cudaMemcpyDeviceToHost, p->ctx->stream), "loss");
        check(cudaStreamSynchronize(p->ctx->stream), "sync");
        check_fault(p);
        if (loss) *loss = l;
    });
}

int cubo_ptycho_plan_backward(cubo_ptycho_plan *p, int recompute, double *loss, double *gore, double *goim,
                              double *gpre, double *gpim) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        if (p->states > 1 || p->multislice) fail(CUBO_PTYCHO_UNSUPPORTED, "the adjoint pair is single-slice only");
        if (recompute || !p->tape_valid) {
            if (p->fp64) enqueue_forward<double>(p);
            else enqueue_forward<float>(p);
            p->tape_valid = true;
        }
        if (p->fp64) enqueue_gathers<double>(p);
        else enqueue_gathers<float>(p);
        // dL/dRe + i dL/dIm = -2 n * (sum of conj(.) dpsi): dpsi carries the inverse transform's 1/n
        const double scale = -2.0 * (double)p->n;
        if (p->fp64) download_object_gradient<double>(p, scale, gore, goim);
        else download_object_gradient<float>(p, scale, gore, goim);
        std::vector<double2> gp(p->n);
        double l = 0;
        check(cudaMemcpyAsync(gp.data(), p->grad_p64.ptr, (size_t)p->n * sizeof(double2), cudaMemcpyDeviceToHost,
                              p->ctx->stream), "download gradient");
        check(cudaMemcpyAsync(&l, p->loss_slot.ptr, sizeof(double), cudaMemcpyDeviceToHost, p->ctx->stream), "loss");
        check(cudaStreamSynchronize(p->ctx->stream), "sync");
        check_fault(p);
        for (int k = 0; k < p->n; k++) {
            if (gpre) gpre[k] = scale * gp[k].x;
            if (gpim) gpim[k] = scale * gp[k].y;
        }
        if (loss) *loss = l;
    });
}

int cubo_ptycho_plan_set_timing(cubo_ptycho_plan *p, int enabled) {
    if (!p) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        collect_timing(p);
        p->timing = enabled != 0;
        std::fill(p->kind_ms.begin(), p->kind_ms.end(), 0.0);
        std::fill(p->kind_launches.begin(), p->kind_launches.end(), 0);
    });
}

int cubo_ptycho_plan_kernel_stats(cubo_ptycho_plan *p, int capacity, const char **names, double *ms,
                                  long long *launches, int *count) {
    if (!p || !count) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(p->ctx, [&] {
        collect_timing(p);
        int filled = 0;
        for (int k = 0; k < kKinds && filled < capacity; k++) {
            if (names) names[filled] = kKindNames[k];
            if (ms) ms[filled] = p->kind_ms[k];
            if (launches) launches[filled] = p->kind_launches[k];
            filled++;
        }
        *count = filled;
    });
}

long long cubo_ptycho_plan_launch_count(const cubo_ptycho_plan *p) { return p ? p->launches : -1; }

}  // extern "C"

struct cubo_ptycho_batch {
    cubo_ptycho_context *ctx = nullptr;
    std::vector<cubo_ptycho_plan *> plans;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<void *> captured_errors;  // the error buffers the graph was captured with
    long long launches_per_iteration = 0;
    // Grouped launches: the generic position passes of every item with the same square compile-time-plan detector,
    // form and CTA shape in one persistent launch; the object gathers (and, but for the FP32 128 x 128 items, which sum
    // their probe gradient in the pass, the probe gathers) of every item of a form in one each.  Each group holds one
    // argument structure per item and the items' unit offsets in device memory.
    struct Group {
        int wave = 0;  // the wave of items it belongs to
        int kind = 0;  // 0 position pass, 1 object gather, 2 probe gather
        bool fp64 = false;
        int N = 0, shape = 0;
        std::vector<cubo_ptycho_plan *> plans;
        std::vector<int> prefix;
        DeviceBuffer args, offsets;
    };
    std::vector<std::unique_ptr<Group>> groups;  // DeviceBuffer does not move: held by pointer
    bool grouping = true;  // CUBO_PTYCHO_BATCH_GROUPED=0: every item launches its own kernels (for comparison)
    // Items run in waves, in batch order, whose residuals together take at most wave_bytes (an item larger than that is
    // a wave of its own): a wave's passes, then its gathers.  Default: one wave of every item.  Waves of ~96 MB (to
    // keep a wave's residuals in L2 for its gathers) grouped almost nothing on the 64-reconstruction batch and measured
    // 64.2 ms per iteration against 57.8 ms in one wave and 61.3 ms with every item launching its own kernels.
    size_t wave_bytes = SIZE_MAX;
    std::vector<int> wave_of;  // per plan
    ~cubo_ptycho_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto *p : plans) delete p;
    }
};

namespace {

template <typename T>
void upload_group_args(cubo_ptycho_batch::Group &g, cudaStream_t s) {
    if (g.kind == 0) {
        std::vector<PositionPassArgs<T>> v;
        for (auto *p : g.plans) v.push_back(position_pass_args<T>(p));
        upload(g.args, v, s);
    } else if (g.kind == 1) {
        std::vector<ObjectGatherArgs<T>> v;
        for (auto *p : g.plans) v.push_back(object_gather_args<T>(p));
        upload(g.args, v, s);
    } else {
        std::vector<ProbeGatherArgs<T>> v;
        for (auto *p : g.plans) v.push_back(probe_gather_args<T>(p));
        upload(g.args, v, s);
    }
    upload(g.offsets, g.prefix, s);
}

// Sorts the batch's plans into groups (before a capture: the argument tables hold the plans' current buffers).
void build_groups(cubo_ptycho_batch *b) {
    cudaStream_t s = b->ctx->stream;
    b->groups.clear();
    for (auto *p : b->plans) p->grouped_pass = p->grouped_gathers = false;
    // waves: consecutive items whose residuals together fit the budget (without grouping, one item each)
    b->wave_of.assign(b->plans.size(), 0);
    {
        int wave = 0;
        size_t bytes = 0;
        for (size_t i = 0; i < b->plans.size(); i++) {
            const cubo_ptycho_plan *p = b->plans[i];
            const size_t r = (size_t)p->states * p->P * p->n * (p->fp64 ? sizeof(double2) : sizeof(float2));
            if (i > 0 && (bytes + r > b->wave_bytes || !b->grouping)) { wave++; bytes = 0; }
            bytes += r;
            b->wave_of[i] = wave;
        }
    }
    if (!b->grouping) return;
    std::map<std::tuple<int, int, int, int, int>, size_t> index;  // (wave, kind, fp64, N, shape) -> group
    size_t item = 0;
    auto add = [&](int kind, cubo_ptycho_plan *p, int N, int shape, int units) {
        const auto key = std::make_tuple(b->wave_of[item], kind, p->fp64 ? 1 : 0, N, shape);
        auto it = index.find(key);
        if (it == index.end()) {
            it = index.emplace(key, b->groups.size()).first;
            b->groups.emplace_back(new cubo_ptycho_batch::Group());
            auto &ng = *b->groups.back();
            ng.wave = b->wave_of[item];
            ng.kind = kind;
            ng.fp64 = p->fp64;
            ng.N = N;
            ng.shape = shape;
            ng.prefix.push_back(0);
        }
        auto &g = *b->groups[it->second];
        g.plans.push_back(p);
        g.prefix.push_back(g.prefix.back() + units);
    };
    for (item = 0; item < b->plans.size(); item++) {
        cubo_ptycho_plan *p = b->plans[item];
        if (p->states != 1 || p->multislice || p->banded || p->correct_positions) continue;
        if (p->fp64) ensure_dpsi<double>(p);
        else ensure_dpsi<float>(p);
        const bool generic_pass = p->fp64 ? !p->global64 && !p->plane128 : !p->fast && !p->bf16 && !p->global32;
        if (generic_pass && position_pass_groupable(p->R, p->C, p->fp64)) {
            add(0, p, p->R, p->params.pass_shape, p->P);
            p->grouped_pass = true;
        }
        add(1, p, 0, 0, p->tiles);
        if (!p->fast) add(2, p, 0, 0, ((p->n + 255) / 256) * p->groups);
        p->grouped_gathers = true;
    }
    for (auto &g : b->groups) {
        if (g->fp64) upload_group_args<double>(*g, s);
        else upload_group_args<float>(*g, s);
    }
}

template <typename T>
cudaError_t launch_group(const cubo_ptycho_batch::Group &g, cudaStream_t s) {
    const int items = (int)g.plans.size(), total = g.prefix.back();
    if (g.kind == 0)
        return launch_position_pass_grouped<T>(g.args.as<PositionPassArgs<T>>(), g.offsets.as<int>(), items, total,
                                               g.N, g.shape, s);
    if (g.kind == 1)
        return launch_object_gather_grouped<T>(g.args.as<ObjectGatherArgs<T>>(), g.offsets.as<int>(), items, total, s);
    return launch_probe_gather_grouped<T>(g.args.as<ProbeGatherArgs<T>>(), g.offsets.as<int>(), items, total, s);
}

// Captures one iteration of every plan of the batch into a graph (again when an error buffer moved), wave by wave: the
// wave's shifted probes and own position passes, its grouped passes, its grouped gathers, then its items' own gathers,
// reductions, updates, constraints and error.
void capture_batch(cubo_ptycho_batch *b) {
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    cudaStream_t s = b->ctx->stream;
    build_groups(b);
    check(cudaStreamSynchronize(s), "batch groups");
    long long before = 0;
    for (auto *p : b->plans) before += p->launches;
    check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
        const int waves = b->plans.empty() ? 0 : b->wave_of.back() + 1;
        for (int w = 0; w < waves; w++) {
            for (size_t i = 0; i < b->plans.size(); i++) {
                if (b->wave_of[i] != w) continue;
                cubo_ptycho_plan *p = b->plans[i];
                if (p->banded) enqueue_banded_pass_and_gathers(p);
                else if (p->fp64) enqueue_position_pass<double>(p);
                else enqueue_position_pass<float>(p);
            }
            for (int kind = 0; kind < 3; kind++)  // the wave's passes before any of its gathers
                for (const auto &g : b->groups)
                    if (g->wave == w && g->kind == kind)
                        check(g->fp64 ? launch_group<double>(*g, s) : launch_group<float>(*g, s), "grouped launch");
            for (size_t i = 0; i < b->plans.size(); i++) {
                if (b->wave_of[i] != w) continue;
                cubo_ptycho_plan *p = b->plans[i];
                if (p->fp64) {
                    if (!p->banded) enqueue_gathers<double>(p);
                    enqueue_iteration_tail<double>(p);
                } else {
                    if (!p->banded) enqueue_gathers<float>(p);
                    enqueue_iteration_tail<float>(p);
                }
            }
        }
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    check(cudaStreamEndCapture(s, &b->graph), "cudaStreamEndCapture");
    check(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate");
    long long after = 0;
    for (auto *p : b->plans) after += p->launches;
    b->launches_per_iteration = after - before + (long long)b->groups.size();
    b->captured_errors.clear();
    for (auto *p : b->plans) b->captured_errors.push_back(p->errors.ptr);
}

}  // namespace

extern "C" {

int cubo_ptycho_batch_create(cubo_ptycho_context *ctx, int count, const cubo_ptycho_problem *problems,
                             const cubo_ptycho_params *params, cubo_ptycho_batch **out) {
    if (!ctx || !out || count < 1 || !problems || !params) return CUBO_PTYCHO_INVALID_INPUT;
    *out = nullptr;
    auto *b = new (std::nothrow) cubo_ptycho_batch();
    if (!b) return CUBO_PTYCHO_OUT_OF_MEMORY;
    b->ctx = ctx;
    if (const char *env = std::getenv("CUBO_PTYCHO_BATCH_GROUPED")) b->grouping = std::atoi(env) != 0;
    if (const char *env = std::getenv("CUBO_PTYCHO_BATCH_WAVE_MB")) {
        const long long mb = std::atoll(env);
        if (mb > 0) b->wave_bytes = (size_t)mb << 20;
    }
    for (int i = 0; i < count; i++) {
        if (params[i].has_position_correction) {  // the positions it moves are read back between iterations
            delete b;
            ctx->last_error = "reconstruction " + std::to_string(i) + ": position correction is not available in a "
                              "graph-replayed batch";
            return CUBO_PTYCHO_INVALID_INPUT;
        }
        cubo_ptycho_plan *p = nullptr;
        const int st = cubo_ptycho_plan_create(ctx, &problems[i], &params[i], &p);
        if (st != CUBO_PTYCHO_OK) {
            const std::string msg = "reconstruction " + std::to_string(i) + ": " + ctx->last_error;
            delete b;
            ctx->last_error = msg;
            return st;
        }
        b->plans.push_back(p);
    }
    *out = b;
    return CUBO_PTYCHO_OK;
}

int cubo_ptycho_batch_destroy(cubo_ptycho_batch *b) {
    if (!b) return CUBO_PTYCHO_OK;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    delete b;
    return CUBO_PTYCHO_OK;
}

int cubo_ptycho_batch_set_state(cubo_ptycho_batch *b, int index, const double *ore, const double *oim,
                                const double *pre, const double *pim) {
    if (!b || index < 0 || index >= (int)b->plans.size()) return CUBO_PTYCHO_INVALID_INPUT;
    return cubo_ptycho_plan_set_state(b->plans[index], ore, oim, pre, pim);
}

int cubo_ptycho_batch_get_state(cubo_ptycho_batch *b, int index, double *ore, double *oim, double *pre, double *pim) {
    if (!b || index < 0 || index >= (int)b->plans.size()) return CUBO_PTYCHO_INVALID_INPUT;
    return cubo_ptycho_plan_get_state(b->plans[index], ore, oim, pre, pim);
}

int cubo_ptycho_batch_errors(cubo_ptycho_batch *b, int index, int count, double *errors) {
    if (!b || index < 0 || index >= (int)b->plans.size()) return CUBO_PTYCHO_INVALID_INPUT;
    return cubo_ptycho_plan_errors(b->plans[index], count, errors);
}

long long cubo_ptycho_batch_launches_per_iteration(const cubo_ptycho_batch *b) {
    return b ? b->launches_per_iteration : -1;
}

int cubo_ptycho_batch_run(cubo_ptycho_batch *b, int iterations, int synchronize) {
    if (!b) return CUBO_PTYCHO_INVALID_INPUT;
    return run_guarded(b->ctx, [&] {
        if (iterations < 0) fail(CUBO_PTYCHO_INVALID_INPUT, "iterations");
        for (auto *p : b->plans) {
            if (p->timing) fail(CUBO_PTYCHO_INVALID_INPUT, "timing is on for a plan of the batch");
            ensure_errors(p, p->iterations_done + iterations);
        }
        bool stale = !b->exec || b->captured_errors.size() != b->plans.size();
        for (size_t i = 0; !stale && i < b->plans.size(); i++) stale = b->captured_errors[i] != b->plans[i]->errors.ptr;
        if (stale) capture_batch(b);
        for (int it = 0; it < iterations; it++) check(cudaGraphLaunch(b->exec, b->ctx->stream), "cudaGraphLaunch");
        for (auto *p : b->plans) {
            p->iterations_done += iterations;
            p->tape_valid = false;
        }
        if (synchronize) {
            check(cudaStreamSynchronize(b->ctx->stream), "sync");
            for (auto *p : b->plans) check_fault(p);
        }
    });
}

namespace {
// PtychographyPreparation.amplitudes(from:origins:shift:) (PtychographyPreparation.swift:142-183); `on_device`: cube and
// amplitudes are device pointers.  Host data moves in chunks of at most 256 MB, alternating between two streams so that
// one chunk's upload overlaps the previous chunk's download; the per-pattern sums are kept for all patterns and summed
// once at the end in a fixed order, so the result does not depend on the chunking.
void prepare_amplitudes(cubo_ptycho_context *ctx, int count, int rows, int columns, const float *cube,
                        const double *origin_rows, const double *origin_columns, int shift, float *amplitudes,
                        double *mean_intensity, double *clipped_mean_intensity, bool on_device) {
    // PtychographyPreparation.swift:148-159
    if (!(count > 0 && rows > 1 && columns > 1)) fail(CUBO_PTYCHO_INVALID_INPUT, "cube shape");
    const long long n = (long long)rows * columns;
    if ((long long)count * n > (1LL << 40)) fail(CUBO_PTYCHO_INVALID_INPUT, "too many samples");
    if (!cube || !origin_rows || !origin_columns || !amplitudes || !mean_intensity || !clipped_mean_intensity)
        fail(CUBO_PTYCHO_INVALID_INPUT, "null input");
    if (shift != CUBO_PTYCHO_SHIFT_BILINEAR && shift != CUBO_PTYCHO_SHIFT_CUBIC_SPLINE) fail(CUBO_PTYCHO_INVALID_INPUT, "shift");
    for (int i = 0; i < count; i++)
        if (!(std::isfinite(origin_rows[i]) && std::fabs(origin_rows[i]) < 1e9 && std::isfinite(origin_columns[i]) &&
              std::fabs(origin_columns[i]) < 1e9))
            fail(CUBO_PTYCHO_INVALID_INPUT, "origin");
    int optin = 0, sms = 0;
    check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device), "attribute");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device), "attribute");
    const bool cubic = shift == CUBO_PTYCHO_SHIFT_CUBIC_SPLINE;
    const size_t smem_limit = (size_t)optin - 1024;
    if (n > (1LL << 30) || (cubic && (prepare_smem(rows, columns, true, false) > smem_limit ||
                                      std::max(rows, columns) > prepare_max_line())))
        fail(CUBO_PTYCHO_UNSUPPORTED, "pattern of " + std::to_string(n) + " pixels exceeds one CTA's shared memory");
    check(configure_prepare(), "configure preprocessing");
    const int ctas = sms;  // CTAs of 1024 threads, one per SM
    cudaStream_t s0 = ctx->stream;
    DeviceBuffer sums, scratch, bad, dorig;
    check(sums.alloc((size_t)prepare_sums_per_pattern() * count * sizeof(double)), "cudaMalloc");
    check(scratch.alloc((size_t)prepare_scratch_doubles() * sizeof(double)), "cudaMalloc");
    check(bad.alloc(sizeof(int)), "cudaMalloc");
    check(cudaMemsetAsync(bad.ptr, 0, sizeof(int), s0), "memset");
    // Swift :301-306, :321-328: the whole part floor(origin) (wrapped into the pattern) and the fraction
    // origin - floor(origin), which is exact
    std::vector<PatternShift> shifts((size_t)count);
    for (int i = 0; i < count; i++) {
        const double fr = std::floor(origin_rows[i]), fc = std::floor(origin_columns[i]);
        const long long wr = (long long)fr % rows, wc = (long long)fc % columns;
        shifts[i] = PatternShift{origin_rows[i] - fr, origin_columns[i] - fc, (int)(wr < 0 ? wr + rows : wr),
                                 (int)(wc < 0 ? wc + columns : wc)};
    }
    upload(dorig, shifts, s0);
    const PatternShift *dshift = dorig.as<PatternShift>();
    // with timing on, one event pair around each kernel launch (on its stream), read after the final synchronize
    struct EventPair {
        cudaEvent_t start = nullptr, stop = nullptr;
    };
    std::vector<EventPair> timed;
    struct ReleaseEvents {
        std::vector<EventPair> &v;
        ~ReleaseEvents() {
            for (auto &e : v) {
                if (e.start) cudaEventDestroy(e.start);
                if (e.stop) cudaEventDestroy(e.stop);
            }
        }
    } release_events{timed};
    auto timed_launch = [&](cudaStream_t st, const std::function<cudaError_t()> &launch) {
        if (!ctx->timing) return check(launch(), "preprocess");
        timed.emplace_back();
        check(cudaEventCreate(&timed.back().start), "cudaEventCreate");
        check(cudaEventCreate(&timed.back().stop), "cudaEventCreate");
        check(cudaEventRecord(timed.back().start, st), "cudaEventRecord");
        check(launch(), "preprocess");
        check(cudaEventRecord(timed.back().stop, st), "cudaEventRecord");
    };
    if (on_device) {
        timed_launch(s0, [&] {
            return launch_prepare(cube, count, rows, columns, dshift, cubic, amplitudes, sums.as<double>(),
                                  bad.as<int>(), ctas, smem_limit, s0);
        });
    } else {
        const long long chunk = std::max<long long>(1, std::min<long long>(count, (256LL << 20) / (n * 4)));
        cudaStream_t s1 = nullptr;
        cudaEvent_t ready = nullptr, done[2] = {nullptr, nullptr};
        check(cudaStreamCreateWithFlags(&s1, cudaStreamNonBlocking), "cudaStreamCreate");
        struct Release {
            cudaStream_t &s; cudaEvent_t &a, &b0, &b1;
            ~Release() { if (a) cudaEventDestroy(a); if (b0) cudaEventDestroy(b0); if (b1) cudaEventDestroy(b1); if (s) cudaStreamDestroy(s); }
        } release{s1, ready, done[0], done[1]};
        check(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "cudaEventCreate");
        check(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming), "cudaEventCreate");
        check(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming), "cudaEventCreate");
        check(cudaEventRecord(ready, s0), "cudaEventRecord");  // origins uploaded, flag cleared
        check(cudaStreamWaitEvent(s1, ready, 0), "cudaStreamWaitEvent");
        DeviceBuffer in[2], out[2];
        for (int b = 0; b < 2; b++) {
            check(in[b].alloc((size_t)(chunk * n) * sizeof(float)), "cudaMalloc");
            check(out[b].alloc((size_t)(chunk * n) * sizeof(float)), "cudaMalloc");
        }
        int slot = 0;
        for (long long first = 0; first < count; first += chunk, slot ^= 1) {
            const int c = (int)std::min<long long>(chunk, count - first);
            cudaStream_t st = slot ? s1 : s0;
            check(cudaMemcpyAsync(in[slot].ptr, cube + first * n, (size_t)(c * n) * sizeof(float), cudaMemcpyHostToDevice,
                                  st), "upload cube");
            timed_launch(st, [&] {
                return launch_prepare(in[slot].as<float>(), c, rows, columns, dshift + first, cubic,
                                      out[slot].as<float>(), sums.as<double>() + (size_t)prepare_sums_per_pattern() * first,
                                      bad.as<int>(), ctas, smem_limit, st);
            });
            check(cudaMemcpyAsync(amplitudes + first * n, out[slot].ptr, (size_t)(c * n) * sizeof(float),
                                  cudaMemcpyDeviceToHost, st), "download amplitudes");
        }
        check(cudaEventRecord(done[1], s1), "cudaEventRecord");
        check(cudaStreamWaitEvent(s0, done[1], 0), "cudaStreamWaitEvent");
        check(cudaStreamSynchronize(s1), "preprocess");
    }
    check(launch_prepare_means(sums.as<double>(), count, scratch.as<double>(), s0), "mean intensities");
    double means[2] = {0, 0};
    int any_bad = 0;
    check(cudaMemcpyAsync(means, scratch.as<double>() + prepare_scratch_doubles() - 2, sizeof(means),
                          cudaMemcpyDeviceToHost, s0), "download");
    check(cudaMemcpyAsync(&any_bad, bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, s0), "download");
    check(cudaStreamSynchronize(s0), "preprocess");
    for (auto &e : timed) {
        float ms = 0.0f;
        check(cudaEventElapsedTime(&ms, e.start, e.stop), "cudaEventElapsedTime");
        ctx->prepare_ms += ms;
        ctx->prepare_launches += 1;
    }
    if (any_bad) fail(CUBO_PTYCHO_INVALID_INPUT, "cube value not finite");
    *mean_intensity = means[0];
    *clipped_mean_intensity = means[1];
}
}  // namespace

int cubo_ptycho_prepare_amplitudes(cubo_ptycho_context *ctx, int count, int rows, int columns, const float *cube,
                                   const double *origin_rows, const double *origin_columns, int shift, float *amplitudes,
                                   double *mean_intensity, double *clipped_mean_intensity) {
    return run_guarded(ctx, [&] {
        prepare_amplitudes(ctx, count, rows, columns, cube, origin_rows, origin_columns, shift, amplitudes, mean_intensity,
                           clipped_mean_intensity, false);
    });
}

int cubo_ptycho_prepare_amplitudes_device(cubo_ptycho_context *ctx, int count, int rows, int columns,
                                          const float *cube_device, const double *origin_rows,
                                          const double *origin_columns, int shift, float *amplitudes_device,
                                          double *mean_intensity, double *clipped_mean_intensity) {
    return run_guarded(ctx, [&] {
        prepare_amplitudes(ctx, count, rows, columns, cube_device, origin_rows, origin_columns, shift, amplitudes_device,
                           mean_intensity, clipped_mean_intensity, true);
    });
}

int cubo_ptycho_measure_peaks(cubo_ptycho_context *ctx, double *fp32_tflops, double *fp64_tflops) {
    return run_guarded(ctx, [&] {
        if (!fp32_tflops || !fp64_tflops) fail(CUBO_PTYCHO_INVALID_INPUT, "null output");
        int sms = 0;
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device), "attribute");
        check(measure_fma_peaks(ctx->stream, sms, fp32_tflops, fp64_tflops), "FMA peaks");
    });
}

int cubo_ptycho_set_timing(cubo_ptycho_context *ctx, int enabled) {
    if (!ctx) return CUBO_PTYCHO_INVALID_INPUT;
    ctx->timing = enabled != 0;
    ctx->prepare_ms = 0.0;
    ctx->prepare_launches = 0;
    return CUBO_PTYCHO_OK;
}

int cubo_ptycho_prepare_kernel_stats(cubo_ptycho_context *ctx, double *ms, long long *launches) {
    if (!ctx || !ms || !launches) return CUBO_PTYCHO_INVALID_INPUT;
    *ms = ctx->prepare_ms;
    *launches = ctx->prepare_launches;
    return CUBO_PTYCHO_OK;
}

int cubo_ptycho_probe_build(cubo_ptycho_context *ctx, int rows, int columns, double row_sampling, double column_sampling,
                            double wavelength, double cutoff, double rolloff, double defocus, double astigmatism,
                            double astigmatism_angle, double spherical_aberration, int term_count, const double *terms,
                            double *re, double *im) {
    return run_guarded(ctx, [&] {
        // Ptychography.swift:147-153
        if (!(rows > 1 && columns > 1) || !re || !im) fail(CUBO_PTYCHO_INVALID_INPUT, "probe shape");
        const double pos[4] = {row_sampling, column_sampling, wavelength, cutoff};
        for (double v : pos) if (!finite_positive(v)) fail(CUBO_PTYCHO_INVALID_INPUT, "probe sampling");
        if (!(std::isfinite(rolloff) && rolloff >= 0)) fail(CUBO_PTYCHO_INVALID_INPUT, "rolloff");
        if (!(std::isfinite(defocus) && std::isfinite(astigmatism) && std::isfinite(astigmatism_angle) &&
              std::isfinite(spherical_aberration)))
            fail(CUBO_PTYCHO_INVALID_INPUT, "aberrations");
        if (term_count < 0 || (term_count > 0 && !terms)) fail(CUBO_PTYCHO_INVALID_INPUT, "terms");
        for (int t = 0; t < term_count; t++) {  // PtychographyAberrationTerm.isValid, Ptychography.swift:123-125
            const double nr = terms[4 * t], mr = terms[4 * t + 1], sine = terms[4 * t + 2], c = terms[4 * t + 3];
            if (!(std::isfinite(c) && nr >= 1 && nr <= 64 && mr >= 0 && (sine == 0 || mr > 0)))
                fail(CUBO_PTYCHO_INVALID_INPUT, "aberration term");
        }
        const int n = rows * columns;
        cudaStream_t s = ctx->stream;
        check(configure_fft_lines(), "configure line transforms");
        DeviceBuffer field, dterms, twr, twc, sum;
        check(field.alloc((size_t)n * sizeof(double2)), "cudaMalloc");
        check(sum.alloc(sizeof(double)), "cudaMalloc");
        std::vector<double> tv(terms ? terms : nullptr, terms ? terms + 4 * term_count : nullptr);
        upload(dterms, tv, s);
        upload(twr, twiddles(rows), s);
        upload(twc, twiddles(columns), s);
        Fft2Plan64 f{rows, columns, factor_length(rows), factor_length(columns), twr.as<double2>(), twc.as<double2>()};
        check(launch_probe_spectrum(field.as<double2>(), rows, columns, row_sampling, column_sampling, wavelength, cutoff,
                                    rolloff, defocus, astigmatism, astigmatism_angle, spherical_aberration, term_count,
                                    dterms.as<double>(), s), "probe spectrum");
        check(launch_fft2_f64(f, field.as<double2>(), 1, true, s), "probe transform");
        check(launch_scale_f64(field.as<double2>(), n, 1.0 / n, s), "scale");
        check(launch_energy(field.as<double2>(), n, sum.as<double>(), s), "energy");
        double energy = 0;
        check(cudaMemcpyAsync(&energy, sum.ptr, sizeof(double), cudaMemcpyDeviceToHost, s), "download");
        std::vector<double2> out(n);
        check(cudaMemcpyAsync(out.data(), field.ptr, (size_t)n * sizeof(double2), cudaMemcpyDeviceToHost, s), "download");
        check(cudaStreamSynchronize(s), "sync");
        const double norm = std::sqrt(energy);
        if (!finite_positive(norm)) fail(CUBO_PTYCHO_INVALID_INPUT, "probe without intensity");
        for (int k = 0; k < n; k++) { re[k] = out[k].x / norm; im[k] = out[k].y / norm; }
    });
}

}  // extern "C"
