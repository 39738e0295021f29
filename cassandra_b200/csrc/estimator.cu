// Pattern-based score estimators (Pattern/Evaluator.h) on the device, and
// the reference's estimator file format (IO/Binary.cpp).
//
// A ScoreEstimator expands each pattern's dense (symmetry-shared) weights
// into one table of 3^k floats per variation of the pattern
// (Pattern/Evaluator.cpp:11-29):
//     table_i[FastIndex(c, variation_i)] = dense[Indices(c)[i]]
// for every configuration c of variation_i's squares, and evaluates a
// position as the FP32 sum, in variation order, of table_i[FastIndex(pos,
// variation_i)] (:48-54).  A MultiStageScoreEstimator holds one estimator
// per stage of stage_size empty counts (:77-88).  Here the tables of all
// stages live in one device array; expansion, evaluation of a batch and
// ScoreEstimator::Weights (:56-73) are kernels.  Evaluation sums in the
// reference's order, so scores are bitwise those of the reference.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "indexer.cuh"
#include "internal.cuh"
#include "patterns.h"

namespace cas {
namespace {

constexpr int kMaxSlots = 256;  // expanded tables of one estimator (patterns x variations)

// Stages(stage_size), Pattern/Evaluator.cpp:6-9.
int stages_of(int stage_size) { return static_cast<int>(std::ceil(65.0 / stage_size)); }

// One expanded table: its variation's squares in FastIndex digit order (the
// set bits of the mask, lowest first) and its first float in a stage.
struct Slot {
    int64_t toff;
    int nsq;
    int pattern;
    uint8_t sq[kMaxSquares];
};

void mask_squares(uint64_t m, Slot& s)
{
    s.nsq = 0;
    for (int b = 0; b < 64; b++)
        if ((m >> b) & 1u) s.sq[s.nsq++] = static_cast<uint8_t>(b);
}

// The position whose cells on the squares sq are the ternary digits of e
// (digit 1: player, 2: opponent), lowest digit on sq[0].
__device__ __forceinline__ void decode_config(const uint8_t* sq, int n, uint32_t e, uint64_t& p, uint64_t& o)
{
    p = 0;
    o = 0;
    for (int i = 0; i < n; i++) {
        const uint32_t d = e % 3u;
        e /= 3u;
        if (d == 1u) p |= uint64_t(1) << sq[i];
        if (d == 2u) o |= uint64_t(1) << sq[i];
    }
}

__device__ __forceinline__ int slot_of(const int64_t* toff, int nslots, int64_t t)
{
    int lo = 0, hi = nslots - 1;  // largest s with toff[s] <= t
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (toff[mid] <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// tables[st][toff_s + e] = dense[st][Indices(c)[i]] for every stage st, table
// s (variation i of its pattern) and configuration index e.
__global__ void expand_kernel(const Slot* __restrict__ slots, const int64_t* __restrict__ toff, int nslots,
                              const Instance* __restrict__ inst, const uint32_t* __restrict__ itables,
                              const float* __restrict__ dense, int64_t W, int64_t T, int stages,
                              float* __restrict__ out)
{
    const int64_t total = static_cast<int64_t>(stages) * T;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t st = i / T, t = i - st * T;
        const int s = slot_of(toff, nslots, t);
        uint64_t p, o;
        decode_config(slots[s].sq, slots[s].nsq, static_cast<uint32_t>(t - toff[s]), p, o);
        const uint32_t idx = eval_slot(inst[s], itables, static_cast<uint32_t>(p), static_cast<uint32_t>(p >> 32),
                                       static_cast<uint32_t>(o), static_cast<uint32_t>(o >> 32));
        out[i] = dense[st * W + idx];
    }
}

// MultiStageScoreEstimator::Eval of a batch: stage = empty count /
// stage_size, then the FP32 sum over the tables in order.  A record with a
// square of both players (not a position: its FastIndex would leave the
// table) or whose stage has no estimator scores NaN.
__global__ void __launch_bounds__(256) eval_kernel(const Slot* __restrict__ slots, int nslots,
                                                    const float* __restrict__ tables, int64_t T, int stage_size,
                                                    int stages, const ulonglong2* __restrict__ pos, int64_t n,
                                                    float* __restrict__ out)
{
    __shared__ Slot s_slots[kMaxSlots];
    for (int s = threadIdx.x; s < nslots; s += blockDim.x) s_slots[s] = slots[s];
    __syncthreads();
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const ulonglong2 po = pos[r];
        const uint64_t p = po.x, o = po.y;
        const int empty = 64 - __popcll(p | o);
        const int st = empty / stage_size;
        if (st >= stages || (p & o) != 0) {  // no such stage, or not a position (a square of both players)
            out[r] = __int_as_float(0x7fc00000);
            continue;
        }
        const float* tb = tables + static_cast<int64_t>(st) * T;
        const uint32_t plo = static_cast<uint32_t>(p), phi = static_cast<uint32_t>(p >> 32);
        const uint32_t olo = static_cast<uint32_t>(o), ohi = static_cast<uint32_t>(o >> 32);
        float sum = 0.0f;
        for (int s = 0; s < nslots; s++) {
            const Slot& sl = s_slots[s];
            sum += __ldg(tb + sl.toff + digits(sl.sq, sl.nsq, plo, phi, olo, ohi));
        }
        out[r] = sum;
    }
}

// ScoreEstimator::Weights (Pattern/Evaluator.cpp:56-73) of one stage: for
// every configuration c of a pattern's squares, dense[Index(c)] = first
// table[FastIndex(c, pattern)]; when several configurations share a dense
// index the reference keeps the last one it enumerates (Configurations:
// player bits major, opponent bits minor, Pattern/Helpers.cpp:86-101).  Pass
// 1 records that configuration's rank per dense index, pass 2 writes it.
__global__ void weights_rank_kernel(const Slot* __restrict__ pslots, const int64_t* __restrict__ poff, int npat,
                                    const Instance* __restrict__ inst0, const uint32_t* __restrict__ itables,
                                    uint32_t* __restrict__ best, const float* __restrict__ table, int pass,
                                    const int64_t* __restrict__ first_toff, float* __restrict__ dense)
{
    const int64_t total = poff[npat];
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int j = slot_of(poff, npat, i);
        const Slot& sl = pslots[j];
        const uint32_t e = static_cast<uint32_t>(i - poff[j]);
        uint64_t p, o;
        decode_config(sl.sq, sl.nsq, e, p, o);
        // the configuration's rank in the reference's enumeration
        uint32_t pe = 0, oe = 0, x = e;
        for (int k = 0; k < sl.nsq; k++) {
            const uint32_t d = x % 3u;
            x /= 3u;
            if (d == 1u) pe |= 1u << k;
            if (d == 2u) oe |= 1u << k;
        }
        const uint32_t rank = ((pe << sl.nsq) | oe) + 1u;
        const uint32_t idx = eval_slot(inst0[j], itables, static_cast<uint32_t>(p), static_cast<uint32_t>(p >> 32),
                                       static_cast<uint32_t>(o), static_cast<uint32_t>(o >> 32));
        if (pass == 0)
            atomicMax(best + idx, rank);
        else if (best[idx] == rank)
            dense[idx] = table[first_toff[j] + e];
    }
}

}  // namespace
}  // namespace cas

using namespace cas;

// The device estimator: the pattern recipes (reference index mode) of the
// input masks, the square lists of every variation, and the tables of every
// stage.
struct cas_estimator {
    int device = -1;
    int stage_size = 1;
    int stages = 0;
    int64_t W = 0;                  // dense weights per stage
    int64_t T = 0;                  // table floats per stage
    PatternSet ps;                  // recipes of the input masks (expansion)
    PatternSet ps_stored;           // recipes of the stored patterns (Weights)
    std::vector<uint64_t> stored;   // Pattern(): CreateIndexer's pattern per mask
    std::vector<Slot> slots;
    std::vector<int64_t> toff;      // nslots + 1
    Slot* d_slots = nullptr;
    int64_t* d_toff = nullptr;
    Instance* d_inst = nullptr;
    uint32_t* d_itables = nullptr;
    float* d_tables = nullptr;      // [stages][T]
    // Weights(): per pattern its stored squares, configuration offsets, the
    // slot-0 recipe of the stored pattern and its first table's offset
    Slot* d_pslots = nullptr;
    int64_t* d_poff = nullptr;
    Instance* d_inst0 = nullptr;
    uint32_t* d_itables0 = nullptr;
    int64_t* d_first = nullptr;
    int64_t pconfigs = 0;
};

namespace {

void free_estimator(cas_estimator* e)
{
    if (!e) return;
    for (const void* p : {(const void*)e->d_slots, (const void*)e->d_toff, (const void*)e->d_inst,
                          (const void*)e->d_itables, (const void*)e->d_tables, (const void*)e->d_pslots,
                          (const void*)e->d_poff, (const void*)e->d_inst0, (const void*)e->d_itables0,
                          (const void*)e->d_first})
        dfree(p);
    delete e;
}

template <typename V>
cas_status upload(V** dst, const std::vector<V>& v)
{
    CAS_CUDA(dmalloc(dst, sizeof(V) * std::max<size_t>(1, v.size())));
    if (!v.empty()) CAS_CUDA(cudaMemcpy(*dst, v.data(), sizeof(V) * v.size(), cudaMemcpyHostToDevice));
    return CAS_OK;
}

unsigned grid_of(int64_t n) { return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 8LL * sm_count()))); }

// --- the file format (IO/Binary.h:33-69): arithmetic values raw, vectors as
// a size_t count then the elements; ScoreEstimator = Pattern(), Weights();
// MultiStageScoreEstimator = int stage_size, Pattern(), vector of
// ScoreEstimator; AccuracyModel = vector<float>; PatternBasedEstimator =
// score, accuracy (IO/Binary.cpp:3-58).

struct Writer {
    FILE* f;
    bool ok = true;
    template <typename T>
    void put(const T& v) { ok = ok && std::fwrite(&v, sizeof v, 1, f) == 1; }
    template <typename T>
    void put_vec(const T* v, uint64_t n)
    {
        put<uint64_t>(n);
        if (n) ok = ok && std::fwrite(v, sizeof(T), n, f) == n;
    }
};

struct Reader {
    FILE* f;
    bool ok = true;
    template <typename T>
    T get()
    {
        T v{};
        ok = ok && std::fread(&v, sizeof v, 1, f) == 1;
        return v;
    }
    template <typename T>
    std::vector<T> get_vec(uint64_t limit)
    {
        const uint64_t n = get<uint64_t>();
        std::vector<T> v;
        if (!ok || n > limit) {
            ok = false;
            return v;
        }
        v.resize(n);
        if (n) ok = ok && std::fread(v.data(), sizeof(T), n, f) == n;
        return v;
    }
};

struct EstimatorFile {
    int stage_size = 0;
    std::vector<uint64_t> pattern;
    std::vector<std::vector<float>> weights;  // per stage
    std::vector<float> accuracy;
};

constexpr uint64_t kMaxFileCount = uint64_t(1) << 32;

cas_status read_file(const char* path, EstimatorFile& ef)
{
    FILE* f = std::fopen(path, "rb");
    CAS_REQUIRE(f, CAS_ERR_INVALID_ARGUMENT, std::string("estimator file: cannot open ") + path);
    Reader r{f};
    ef.stage_size = r.get<int32_t>();
    ef.pattern = r.get_vec<uint64_t>(1024);
    const uint64_t n = r.ok ? r.get<uint64_t>() : 0;
    if (r.ok && n > 1024) r.ok = false;
    for (uint64_t s = 0; r.ok && s < n; s++) {
        const std::vector<uint64_t> sp = r.get_vec<uint64_t>(1024);
        if (r.ok && sp != ef.pattern) {
            std::fclose(f);
            set_error("estimator file: a stage's patterns differ from the estimator's");
            return CAS_ERR_INVALID_ARGUMENT;
        }
        ef.weights.push_back(r.get_vec<float>(kMaxFileCount));
    }
    if (r.ok) ef.accuracy = r.get_vec<float>(1024);
    std::fclose(f);
    CAS_REQUIRE(r.ok, CAS_ERR_INVALID_ARGUMENT, std::string("estimator file: truncated or malformed: ") + path);
    CAS_REQUIRE(ef.stage_size > 0 && !ef.pattern.empty(), CAS_ERR_INVALID_ARGUMENT,
                "estimator file: bad stage size or no patterns");
    for (const auto& w : ef.weights)
        CAS_REQUIRE(w.size() == ef.weights.front().size(), CAS_ERR_INVALID_ARGUMENT,
                    "estimator file: stages of different sizes");
    return CAS_OK;
}

}  // namespace

extern "C" {

CAS_API int cas_estimator_stages(int stage_size) { return stage_size > 0 ? stages_of(stage_size) : 0; }

CAS_API cas_status cas_estimator_save(const char* path, int stage_size, const uint64_t* masks, int n_masks,
                                      const float* h_weights, const float* accuracy, int n_accuracy)
{
    CAS_REQUIRE(path && masks && n_masks > 0 && stage_size > 0 && h_weights && (n_accuracy == 0 || accuracy) &&
                    n_accuracy >= 0,
                CAS_ERR_INVALID_ARGUMENT, "cas_estimator_save: bad argument");
    PatternSet ps;
    std::string err;
    CAS_REQUIRE(build_pattern_set(masks, n_masks, CAS_INDEX_REFERENCE, ps, err), CAS_ERR_PATTERN,
                "cas_estimator_save: " + err);
    std::vector<uint64_t> stored;
    for (const IndexerInfo& in : ps.indexers) stored.push_back(in.stored_pattern);
    const int stages = stages_of(stage_size);
    FILE* f = std::fopen(path, "wb");
    CAS_REQUIRE(f, CAS_ERR_INVALID_ARGUMENT, std::string("cas_estimator_save: cannot create ") + path);
    Writer w{f};
    w.put<int32_t>(stage_size);
    w.put_vec(stored.data(), stored.size());
    w.put<uint64_t>(static_cast<uint64_t>(stages));
    for (int s = 0; s < stages; s++) {
        w.put_vec(stored.data(), stored.size());
        w.put_vec(h_weights + static_cast<int64_t>(s) * ps.cols, static_cast<uint64_t>(ps.cols));
    }
    w.put_vec(accuracy, static_cast<uint64_t>(n_accuracy));
    const bool closed = std::fclose(f) == 0;
    CAS_REQUIRE(w.ok && closed, CAS_ERR_INVALID_ARGUMENT, std::string("cas_estimator_save: write failed: ") + path);
    return CAS_OK;
}

CAS_API cas_status cas_estimator_file_info(const char* path, int* stage_size, int* n_masks, int* stages,
                                           int64_t* weights_per_stage, int* n_accuracy)
{
    CAS_REQUIRE(path, CAS_ERR_INVALID_ARGUMENT, "cas_estimator_file_info: null path");
    EstimatorFile ef;
    CAS_TRY(read_file(path, ef));
    if (stage_size) *stage_size = ef.stage_size;
    if (n_masks) *n_masks = static_cast<int>(ef.pattern.size());
    if (stages) *stages = static_cast<int>(ef.weights.size());
    if (weights_per_stage) *weights_per_stage = ef.weights.empty() ? 0 : static_cast<int64_t>(ef.weights[0].size());
    if (n_accuracy) *n_accuracy = static_cast<int>(ef.accuracy.size());
    return CAS_OK;
}

CAS_API cas_status cas_estimator_file_read(const char* path, uint64_t* h_masks, float* h_weights, float* h_accuracy)
{
    CAS_REQUIRE(path, CAS_ERR_INVALID_ARGUMENT, "cas_estimator_file_read: null path");
    EstimatorFile ef;
    CAS_TRY(read_file(path, ef));
    if (h_masks) std::memcpy(h_masks, ef.pattern.data(), sizeof(uint64_t) * ef.pattern.size());
    if (h_weights)
        for (size_t s = 0; s < ef.weights.size(); s++)
            std::memcpy(h_weights + s * ef.weights[s].size(), ef.weights[s].data(), sizeof(float) * ef.weights[s].size());
    if (h_accuracy && !ef.accuracy.empty())
        std::memcpy(h_accuracy, ef.accuracy.data(), sizeof(float) * ef.accuracy.size());
    return CAS_OK;
}

CAS_API cas_status cas_estimator_create(const uint64_t* masks, int n_masks, int stage_size, const float* d_weights,
                                        void* stream, cas_estimator** out)
{
    CAS_REQUIRE(out && masks && n_masks > 0 && stage_size > 0 && d_weights, CAS_ERR_INVALID_ARGUMENT,
                "cas_estimator_create: bad argument");
    *out = nullptr;
    CAS_TRY(require_device());
    std::unique_ptr<cas_estimator, void (*)(cas_estimator*)> e(new (std::nothrow) cas_estimator, free_estimator);
    CAS_REQUIRE(e, CAS_ERR_OUT_OF_MEMORY, "cas_estimator_create: out of host memory");
    std::string err;
    CAS_REQUIRE(build_pattern_set(masks, n_masks, CAS_INDEX_REFERENCE, e->ps, err), CAS_ERR_PATTERN,
                "cas_estimator_create: " + err);
    for (const IndexerInfo& in : e->ps.indexers) e->stored.push_back(in.stored_pattern);
    CAS_REQUIRE(build_pattern_set(e->stored.data(), n_masks, CAS_INDEX_REFERENCE, e->ps_stored, err),
                CAS_ERR_PATTERN, "cas_estimator_create: " + err);
    CAS_REQUIRE(e->ps_stored.cols == e->ps.cols, CAS_ERR_PATTERN,
                "cas_estimator_create: the stored patterns index another weight space");
    const int nslots = static_cast<int>(e->ps.variations.size());
    CAS_REQUIRE(nslots <= kMaxSlots && static_cast<int>(e->ps.instances.size()) == nslots, CAS_ERR_PATTERN,
                "cas_estimator_create: more than 256 pattern variations");
    CAS_CUDA(cudaGetDevice(&e->device));
    e->stage_size = stage_size;
    e->stages = stages_of(stage_size);
    e->W = e->ps.cols;
    int64_t t = 0;
    for (int s = 0; s < nslots; s++) {
        Slot sl{};
        mask_squares(e->ps.variations[s], sl);
        CAS_REQUIRE(sl.nsq <= 16, CAS_ERR_PATTERN, "cas_estimator_create: a variation with more than 16 squares");
        sl.toff = t;
        sl.pattern = e->ps.slot_indexer[s];
        e->slots.push_back(sl);
        e->toff.push_back(t);
        int64_t sz = 1;
        for (int k = 0; k < sl.nsq; k++) sz *= 3;
        t += sz;
    }
    e->toff.push_back(t);
    e->T = t;
    // Weights(): per pattern the stored pattern's squares and recipe
    std::vector<Slot> pslots;
    std::vector<int64_t> poff, first;
    std::vector<Instance> inst0;
    int64_t pc = 0;
    for (int j = 0; j < n_masks; j++) {
        Slot sl{};
        mask_squares(e->stored[j], sl);
        pslots.push_back(sl);
        poff.push_back(pc);
        int64_t sz = 1;
        for (int k = 0; k < sl.nsq; k++) sz *= 3;
        pc += sz;
        int s0 = 0;  // first slot of the estimator's pattern j (its variation 0)
        while (s0 < nslots && e->ps.slot_indexer[s0] != j) s0++;
        first.push_back(e->toff[s0]);
        int r0 = 0;
        while (r0 < static_cast<int>(e->ps_stored.instances.size()) && e->ps_stored.slot_indexer[r0] != j) r0++;
        inst0.push_back(e->ps_stored.instances[r0]);
    }
    poff.push_back(pc);
    e->pconfigs = pc;
    CAS_TRY(upload(&e->d_slots, e->slots));
    CAS_TRY(upload(&e->d_toff, e->toff));
    CAS_TRY(upload(&e->d_inst, e->ps.instances));
    CAS_TRY(upload(&e->d_itables, e->ps.tables));
    CAS_TRY(upload(&e->d_pslots, pslots));
    CAS_TRY(upload(&e->d_poff, poff));
    CAS_TRY(upload(&e->d_inst0, inst0));
    CAS_TRY(upload(&e->d_itables0, e->ps_stored.tables));
    CAS_TRY(upload(&e->d_first, first));
    const int64_t total = static_cast<int64_t>(e->stages) * e->T;
    CAS_CUDA(dmalloc(&e->d_tables, sizeof(float) * std::max<int64_t>(total, 1)));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    { expand_kernel<<<grid_of(total), 256, 0, s>>>(e->d_slots, e->d_toff, nslots, e->d_inst, e->d_itables, d_weights,
                                                   e->W, e->T, e->stages, e->d_tables); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    *out = e.release();
    return CAS_OK;
}

CAS_API void cas_estimator_destroy(cas_estimator* e)
{
    if (!e) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (e->device >= 0 && cur != e->device) cudaSetDevice(e->device);
    free_estimator(e);
    if (cur >= 0) cudaSetDevice(cur);
}

CAS_API cas_status cas_estimator_info(const cas_estimator* e, int* stage_size, int* stages, int* n_masks,
                                      int64_t* weights_per_stage, int64_t* table_floats_per_stage)
{
    CAS_REQUIRE(e, CAS_ERR_INVALID_ARGUMENT, "cas_estimator_info: null estimator");
    if (stage_size) *stage_size = e->stage_size;
    if (stages) *stages = e->stages;
    if (n_masks) *n_masks = static_cast<int>(e->stored.size());
    if (weights_per_stage) *weights_per_stage = e->W;
    if (table_floats_per_stage) *table_floats_per_stage = e->T;
    return CAS_OK;
}

CAS_API cas_status cas_estimator_patterns(const cas_estimator* e, uint64_t* h_out)
{
    CAS_REQUIRE(e && h_out, CAS_ERR_INVALID_ARGUMENT, "cas_estimator_patterns: null argument");
    std::memcpy(h_out, e->stored.data(), sizeof(uint64_t) * e->stored.size());
    return CAS_OK;
}

CAS_API cas_status cas_estimator_tables(const cas_estimator* e, int stage, float* d_out, void* stream)
{
    CAS_REQUIRE(e && d_out && stage >= 0 && stage < e->stages, CAS_ERR_INVALID_ARGUMENT,
                "cas_estimator_tables: bad argument");
    CAS_CUDA(cudaMemcpyAsync(d_out, e->d_tables + static_cast<int64_t>(stage) * e->T, sizeof(float) * e->T,
                             cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)));
    return CAS_OK;
}

CAS_API cas_status cas_estimator_eval(const cas_estimator* e, const uint64_t* d_positions, int64_t n, float* d_scores,
                                      void* stream)
{
    CAS_REQUIRE(e && n >= 0 && (n == 0 || (d_positions && d_scores)), CAS_ERR_INVALID_ARGUMENT,
                "cas_estimator_eval: bad argument");
    CAS_REQUIRE((reinterpret_cast<uintptr_t>(d_positions) & 15) == 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_estimator_eval: position records must be 16-byte aligned");
    if (n == 0) return CAS_OK;
    { eval_kernel<<<grid_of(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        e->d_slots, static_cast<int>(e->slots.size()), e->d_tables, e->T, e->stage_size, e->stages,
        reinterpret_cast<const ulonglong2*>(d_positions), n, d_scores); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

CAS_API cas_status cas_estimator_weights(const cas_estimator* e, int stage, float* d_out, void* stream)
{
    CAS_REQUIRE(e && d_out && stage >= 0 && stage < e->stages, CAS_ERR_INVALID_ARGUMENT,
                "cas_estimator_weights: bad argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t* best = nullptr;
    CAS_CUDA(dmalloc(&best, sizeof(uint32_t) * std::max<int64_t>(e->W, 1)));
    CAS_CUDA(cudaMemsetAsync(best, 0, sizeof(uint32_t) * e->W, s));
    CAS_CUDA(cudaMemsetAsync(d_out, 0, sizeof(float) * e->W, s));
    const float* table = e->d_tables + static_cast<int64_t>(stage) * e->T;
    const int npat = static_cast<int>(e->stored.size());
    for (int pass = 0; pass < 2; pass++) {
        { weights_rank_kernel<<<grid_of(e->pconfigs), 256, 0, s>>>(e->d_pslots, e->d_poff, npat, e->d_inst0,
                                                                   e->d_itables0, best, table, pass, e->d_first,
                                                                   d_out); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
    }
    dfree(best);
    return CAS_OK;
}

}  // extern "C"
