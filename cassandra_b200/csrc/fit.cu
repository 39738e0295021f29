// FitWeights (PatternFit/PatternFit.cpp:7-39) end to end on the device, and
// the seeded synthetic data generator.
#include <algorithm>
#include <cmath>
#include <vector>

#include "board.cuh"
#include "common.cuh"
#include "fast.cuh"
#include "internal.cuh"

namespace cas {
namespace {

__global__ void generate_positions_kernel(uint64_t seed, int64_t n, int min_e, int max_e, ulonglong2* __restrict__ out,
                                          unsigned int* __restrict__ failures)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        uint64_t p, o;
        if (!random_play_position(seed, static_cast<uint64_t>(i), min_e, max_e, p, o)) atomicAdd(failures, 1u);
        out[i] = make_ulonglong2(p, o);
    }
}

// w*_c ~ N(0, sigma^2) by Box-Muller on the counter stream (seed, c).
__global__ void true_weights_kernel(uint64_t seed, int64_t cols, double sigma, double* __restrict__ w)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        Stream rng(seed ^ 0x5EED0F3EC7ED1ULL, static_cast<uint64_t>(c));
        const double u1 = rng.unit(), u2 = rng.unit();
        w[c] = sigma * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    }
}

// b_r = clamp(2 rint(((A w*)_r + e_r) / 2), -64, 64), e_r ~ N(0, noise^2);
// aw holds (A w*)_r, computed on whichever layout the CSR has.
__global__ void targets_kernel(const double* __restrict__ aw, int64_t rows, uint64_t seed, double noise,
                               int64_t first_row, double* __restrict__ b)
{
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < rows;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        Stream rng(seed ^ 0xB0A5EDD15EA5EULL, static_cast<uint64_t>(first_row + r));
        const double u1 = rng.unit(), u2 = rng.unit();
        const double e = noise * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
        b[r] = fmin(64.0, fmax(-64.0, 2.0 * rint((aw[r] + e) * 0.5)));
    }
}

__global__ void f32_to_f64_kernel(const float* __restrict__ in, int64_t n, double* __restrict__ out)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<double>(in[i]);
}

__global__ void f64_to_f32_kernel(const double* __restrict__ in, int64_t n, float* __restrict__ out)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<float>(in[i]);
}

unsigned grid(int64_t n)
{
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, sm_count() * 16LL)));
}

}  // namespace
}  // namespace cas

using namespace cas;

extern "C" {

CAS_API cas_status cas_generate_positions(uint64_t seed, int64_t n, int min_empties, int max_empties,
                                          uint64_t* d_out, void* stream)
{
    CAS_REQUIRE(n >= 0 && (n == 0 || d_out), CAS_ERR_INVALID_ARGUMENT, "cas_generate_positions: bad argument");
    CAS_REQUIRE(0 <= min_empties && min_empties <= max_empties && max_empties <= 60, CAS_ERR_INVALID_ARGUMENT,
                "cas_generate_positions: empty counts must satisfy 0 <= min <= max <= 60");
    CAS_REQUIRE((reinterpret_cast<uintptr_t>(d_out) & 15) == 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_generate_positions: output must be 16-byte aligned");
    CAS_TRY(require_device());
    if (n == 0) return CAS_OK;
    auto s = static_cast<cudaStream_t>(stream);
    unsigned int* fails = nullptr;
    CAS_CUDA(cudaMallocAsync(&fails, sizeof(unsigned int), s));
    CAS_CUDA(cudaMemsetAsync(fails, 0, sizeof(unsigned int), s));
    { generate_positions_kernel<<<grid(n), 256, 0, s>>>(seed, n, min_empties, max_empties,
                                                      reinterpret_cast<ulonglong2*>(d_out), fails); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    unsigned int h = 0;
    CAS_CUDA(cudaMemcpyAsync(&h, fails, sizeof h, cudaMemcpyDeviceToHost, s));
    CAS_CUDA(cudaStreamSynchronize(s));
    cudaFreeAsync(fails, s);
    CAS_REQUIRE(h == 0, CAS_ERR_INVALID_ARGUMENT, "cas_generate_positions: target empty count unreachable");
    return CAS_OK;
}

CAS_API cas_status cas_generate_positions_host(uint64_t seed, int64_t first, int64_t n, int min_empties,
                                               int max_empties, uint64_t* h_out)
{
    CAS_REQUIRE(n >= 0 && first >= 0 && (n == 0 || h_out), CAS_ERR_INVALID_ARGUMENT,
                "cas_generate_positions_host: bad argument");
    CAS_REQUIRE(0 <= min_empties && min_empties <= max_empties && max_empties <= 60, CAS_ERR_INVALID_ARGUMENT,
                "cas_generate_positions_host: empty counts must satisfy 0 <= min <= max <= 60");
    bool ok = true;
#pragma omp parallel for schedule(static) reduction(&& : ok)
    for (int64_t i = 0; i < n; i++) {
        uint64_t p, o;
        ok = random_play_position(seed, static_cast<uint64_t>(first + i), min_empties, max_empties, p, o) && ok;
        h_out[2 * i] = p;
        h_out[2 * i + 1] = o;
    }
    CAS_REQUIRE(ok, CAS_ERR_INVALID_ARGUMENT, "cas_generate_positions_host: target empty count unreachable");
    return CAS_OK;
}

CAS_API cas_status cas_generate_targets(const cas_csr* a, uint64_t seed, double w_sigma, double noise_sigma,
                                        double* d_b, double* d_w_true, void* stream)
{
    return cas_generate_targets_rows(a, seed, w_sigma, noise_sigma, 0, d_b, d_w_true, stream);
}

CAS_API cas_status cas_generate_targets_rows(const cas_csr* a, uint64_t seed, double w_sigma, double noise_sigma,
                                             int64_t first_row, double* d_b, double* d_w_true, void* stream)
{
    CAS_REQUIRE(a && (d_b || a->rows == 0) && first_row >= 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_generate_targets: bad argument");
    auto s = static_cast<cudaStream_t>(stream);
    double* w = d_w_true;
    if (!w) CAS_CUDA(cudaMallocAsync(&w, sizeof(double) * std::max<int64_t>(a->cols, 1), s));
    { true_weights_kernel<<<grid(a->cols), 256, 0, s>>>(seed, a->cols, w_sigma, w); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    if (a->rows) {
        // A w* into d_b first (FP64 product on the CSR's layout), then noise and rounding in place
        CAS_TRY(cas_spmv(a, CAS_F64, w, d_b, stream));
        { targets_kernel<<<grid(a->rows), 256, 0, s>>>(d_b, a->rows, seed, noise_sigma, first_row, d_b); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
    }
    if (!d_w_true) cudaFreeAsync(w, s);
    return CAS_OK;
}

namespace {
// FitWeights on device buffers.  chunks (may be null): the positions are
// still arriving in row chunks (the build indexes each behind its copy);
// scores_ready (may be null): the solve waits for it before reading the
// scores.
cas_status fit_weights_device(const cas_patterns* p, const uint64_t* d_positions, const double* d_scores, int64_t rows,
                              const cas_solve_opts* o, double* d_weights, cas_solve_report* rep, cudaStream_t s,
                              const PositionChunks* chunks, cudaEvent_t scores_ready)
{
    cudaEvent_t e0, e1;
    CAS_CUDA(cudaEventCreate(&e0));
    CAS_CUDA(cudaEventCreate(&e1));
    CAS_CUDA(cudaEventRecord(e0, s));
    // The mixed solver runs on the blocked layout, the plain FP64 path on the
    // reference's row layout; only the layout the solve uses is built.
    int layouts = CAS_LAYOUT_ROWS;
    if (o->precision == CAS_MIXED && fast_supported(pattern_set(p))) layouts = CAS_LAYOUT_BLOCKED;
    cas_csr* a = nullptr;
    cas_status st = csr_from_positions(p, d_positions, rows, layouts, s, &a, chunks);
    if (st != CAS_OK) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return st;
    }
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float setup_ms = 0;
    cudaEventElapsedTime(&setup_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (scores_ready) {
        const cudaError_t e = cudaStreamWaitEvent(s, scores_ready, 0);
        if (e != cudaSuccess) {
            cas_csr_destroy(a);
            CAS_CUDA(e);
        }
    }
    st = cas_solve(a, o, d_scores, d_weights, rep, s);
    if (rep) rep->setup_seconds = setup_ms * 1e-3;
    cas_csr_destroy(a);
    return st;
}
}  // namespace

CAS_API cas_status cas_fit_weights_device(const cas_patterns* p, const uint64_t* d_positions, const double* d_scores,
                                          int64_t rows, const cas_solve_opts* o, double* d_weights,
                                          cas_solve_report* rep, void* stream)
{
    cas::NvtxRange nvtx_range("cas_fit_weights_device");
    CAS_REQUIRE(p && o && d_weights, CAS_ERR_INVALID_ARGUMENT, "cas_fit_weights_device: null argument");
    CAS_REQUIRE(rows >= 0 && (rows == 0 || (d_positions && d_scores)), CAS_ERR_INVALID_ARGUMENT,
                "cas_fit_weights_device: bad rows or buffers");
    return fit_weights_device(p, d_positions, d_scores, rows, o, d_weights, rep, static_cast<cudaStream_t>(stream),
                              nullptr, nullptr);
}

CAS_API cas_status cas_fit_weights(const uint64_t* masks, int n_masks, cas_index_mode mode,
                                   const uint64_t* h_positions, const float* h_scores, int64_t rows,
                                   const cas_solve_opts* o, float* h_weights, cas_solve_report* rep)
{
    cas::NvtxRange nvtx_range("cas_fit_weights");
    CAS_REQUIRE(masks && o && h_weights && rows >= 0, CAS_ERR_INVALID_ARGUMENT, "cas_fit_weights: bad argument");
    CAS_REQUIRE(rows == 0 || (h_positions && h_scores), CAS_ERR_INVALID_ARGUMENT, "cas_fit_weights: null input");
    CAS_TRY(require_device());
    cas_patterns* p = nullptr;
    CAS_TRY(cas_patterns_create(masks, n_masks, mode, &p));
    const int64_t cols = cas_patterns_cols(p);
    cudaStream_t s = nullptr;
    CAS_CUDA(cudaStreamCreate(&s));
    uint64_t* d_pos = nullptr;
    float* d_s32 = nullptr;
    double *d_s = nullptr, *d_w = nullptr;
    float* d_w32 = nullptr;
    cas_status st = CAS_OK;
    auto fail = [&](cudaError_t e) {
        set_error(std::string("cas_fit_weights: ") + cudaGetErrorString(e));
        st = e == cudaErrorMemoryAllocation ? CAS_ERR_OUT_OF_MEMORY : CAS_ERR_CUDA;
    };
    // The inputs go up on a copy stream: the positions in kInputChunks row
    // chunks, each indexed as soon as it has landed (while the next one is
    // copied), then the scores, converted to FP64 there and waited for by the
    // solve only.
    constexpr int kInputChunks = 8;
    cudaStream_t cs = nullptr;
    cudaEvent_t ready[kInputChunks] = {};
    cudaEvent_t scores_ready = nullptr;
    int64_t row_end[kInputChunks];
    cudaError_t e = dmalloc(&d_pos, 16 * std::max<int64_t>(rows, 1));
    if (e == cudaSuccess) e = dmalloc(&d_s32, sizeof(float) * std::max<int64_t>(rows, 1));
    if (e == cudaSuccess) e = dmalloc(&d_s, sizeof(double) * std::max<int64_t>(rows, 1));
    if (e == cudaSuccess) e = dmalloc(&d_w, sizeof(double) * std::max<int64_t>(cols, 1));
    if (e == cudaSuccess) e = dmalloc(&d_w32, sizeof(float) * std::max<int64_t>(cols, 1));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    for (int c = 0; c < kInputChunks && e == cudaSuccess; c++) {
        const int64_t r0 = rows * c / kInputChunks, r1 = rows * (c + 1) / kInputChunks;
        row_end[c] = r1;
        e = cudaEventCreateWithFlags(&ready[c], cudaEventDisableTiming);
        if (e == cudaSuccess && r1 > r0)
            e = cudaMemcpyAsync(d_pos + 2 * r0, h_positions + 2 * r0, 16 * (r1 - r0), cudaMemcpyHostToDevice, cs);
        if (e == cudaSuccess) e = cudaEventRecord(ready[c], cs);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&scores_ready, cudaEventDisableTiming);
    if (e == cudaSuccess && rows) e = cudaMemcpyAsync(d_s32, h_scores, sizeof(float) * rows, cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess && rows) {
        { f32_to_f64_kernel<<<grid(rows), 256, 0, cs>>>(d_s32, rows, d_s); cas::count_launch(); }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(scores_ready, cs);
    if (e != cudaSuccess) fail(e);
    if (st == CAS_OK) {
        const PositionChunks chunks{kInputChunks, row_end, ready};
        st = fit_weights_device(p, d_pos, d_s, rows, o, d_w, rep, s, &chunks, scores_ready);
    }
    if (st == CAS_OK || st == CAS_ERR_NOT_CONVERGED) {
        { f64_to_f32_kernel<<<grid(cols), 256, 0, s>>>(d_w, cols, d_w32); cas::count_launch(); }
        e = cudaMemcpyAsync(h_weights, d_w32, sizeof(float) * cols, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) fail(e);
    }
    cudaStreamSynchronize(s);
    if (cs) {
        cudaStreamSynchronize(cs);
        cudaStreamDestroy(cs);
    }
    for (cudaEvent_t ev : ready)
        if (ev) cudaEventDestroy(ev);
    if (scores_ready) cudaEventDestroy(scores_ready);
    dfree(d_pos);
    dfree(d_s32);
    dfree(d_s);
    dfree(d_w);
    dfree(d_w32);
    cudaStreamDestroy(s);
    cas_patterns_destroy(p);
    return st;
}

namespace {
// The per-stage fits by LSQR or LSMR: one CSR (the layout a single fit of
// that precision uses) and one solver per stage, each on its own stream,
// run to tolerance together -- the host steps the unfinished solvers in
// turn, so that one stage's chunk of iterations runs while another's state
// is read.  A stage without rows gets zero weights.  Each stage's result is
// the single fit's of that stage.
cas_status batched_least_squares(const cas_patterns* p, const uint64_t* d_positions, const double* d_scores,
                                 const int64_t* h_rows, int problems, const cas_solve_opts* o, double* d_weights,
                                 cas_solve_report* reports, cudaStream_t s)
{
    const int64_t cols = cas_patterns_cols(p);
    const int layouts =
        (o->precision == CAS_MIXED && fast_supported(pattern_set(p))) ? CAS_LAYOUT_BLOCKED : CAS_LAYOUT_ROWS;
    std::vector<cudaStream_t> streams(problems, nullptr);
    std::vector<cas_csr*> csrs(problems, nullptr);
    std::vector<cas_solver*> solvers(problems, nullptr);
    std::vector<cas_status> sts(problems, CAS_OK);
    std::vector<cas_solve_report> reps(problems, cas_solve_report{});
    cudaEvent_t ready = nullptr, e0 = nullptr, e1 = nullptr;
    cas_status st = CAS_OK;
    auto cuda = [&](cudaError_t e) {
        if (e != cudaSuccess && st == CAS_OK) {
            set_error(std::string("batched least squares: ") + cudaGetErrorString(e));
            st = e == cudaErrorMemoryAllocation ? CAS_ERR_OUT_OF_MEMORY : CAS_ERR_CUDA;
        }
    };
    cuda(cudaEventCreate(&ready));
    cuda(cudaEventCreate(&e0));
    cuda(cudaEventCreate(&e1));
    if (st == CAS_OK) cuda(cudaEventRecord(ready, s));  // the inputs are written on s
    if (st == CAS_OK) cuda(cudaEventRecord(e0, s));
    int64_t row0 = 0;
    for (int q = 0; q < problems && st == CAS_OK; q++) {
        const int64_t rq = std::max<int64_t>(h_rows[q], 0);
        if (rq == 0) {
            cuda(cudaMemsetAsync(d_weights + q * cols, 0, sizeof(double) * cols, s));
            continue;
        }
        cuda(cudaStreamCreateWithFlags(&streams[q], cudaStreamNonBlocking));
        if (st == CAS_OK) cuda(cudaStreamWaitEvent(streams[q], ready, 0));
        if (st == CAS_OK) st = cas_csr_from_positions_layout(p, d_positions + 2 * row0, rq, layouts, streams[q], &csrs[q]);
        if (st == CAS_OK) st = cas_solver_create(csrs[q], o, d_scores + row0, nullptr, streams[q], &solvers[q]);
        row0 += rq;
    }
    // set-up time: from the first build to the last solver's set-up
    float setup_ms = 0;
    for (int q = 0; q < problems && st == CAS_OK; q++)
        if (streams[q]) {
            cuda(cudaEventRecord(e1, streams[q]));
            if (st == CAS_OK) cuda(cudaStreamWaitEvent(s, e1, 0));
        }
    if (st == CAS_OK) cuda(cudaEventRecord(e1, s));
    if (st == CAS_OK) cuda(cudaEventSynchronize(e1));
    if (st == CAS_OK) cuda(cudaEventElapsedTime(&setup_ms, e0, e1));
    if (st == CAS_OK) st = solvers_run_all(solvers.data(), problems, reps.data(), sts.data());
    for (int q = 0; q < problems && st == CAS_OK; q++) {
        if (!solvers[q]) continue;
        if (sts[q] == CAS_OK || sts[q] == CAS_ERR_NOT_CONVERGED) st = cas_solver_x(solvers[q], d_weights + q * cols);
    }
    for (int q = 0; q < problems; q++)
        if (streams[q]) cuda(cudaStreamSynchronize(streams[q]));
    for (int q = 0; q < problems; q++) {
        if (solvers[q]) cas_solver_destroy(solvers[q]);
        if (csrs[q]) cas_csr_destroy(csrs[q]);
        if (streams[q]) cudaStreamDestroy(streams[q]);
    }
    if (ready) cudaEventDestroy(ready);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (reports)
        for (int q = 0; q < problems; q++) {
            reports[q] = reps[q];
            reports[q].setup_seconds = setup_ms * 1e-3;
        }
    if (st != CAS_OK) return st;
    for (int q = 0; q < problems; q++)
        if (sts[q] != CAS_OK) return sts[q];  // the first stage that did not converge
    return CAS_OK;
}
}  // namespace

CAS_API cas_status cas_fit_weights_batched_device(const cas_patterns* p, const uint64_t* d_positions,
                                                  const double* d_scores, const int64_t* h_problem_rows,
                                                  int problems, const cas_solve_opts* o, double* d_weights,
                                                  cas_solve_report* reports, void* stream)
{
    cas::NvtxRange nvtx_range("cas_fit_weights_batched_device");
    CAS_REQUIRE(p && o && d_weights && h_problem_rows, CAS_ERR_INVALID_ARGUMENT,
                "cas_fit_weights_batched_device: null argument");
    auto s = static_cast<cudaStream_t>(stream);
    if (o->method == CAS_LSQR || o->method == CAS_LSMR)
        return batched_least_squares(p, d_positions, d_scores, h_problem_rows, problems, o, d_weights, reports, s);
    cudaEvent_t e0, e1;
    CAS_CUDA(cudaEventCreate(&e0));
    CAS_CUDA(cudaEventCreate(&e1));
    CAS_CUDA(cudaEventRecord(e0, s));
    cas_csr* a = nullptr;
    cas_status st = cas_csr_from_positions_batched(p, d_positions, h_problem_rows, problems, stream, &a);
    if (st != CAS_OK) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return st;
    }
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float setup_ms = 0;
    cudaEventElapsedTime(&setup_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st = cas_solve_batched(a, o, d_scores, d_weights, reports, stream);
    if (reports)
        for (int q = 0; q < problems; q++) reports[q].setup_seconds = setup_ms * 1e-3;
    cas_csr_destroy(a);
    return st;
}

CAS_API cas_status cas_fit_weights_batched(const uint64_t* masks, int n_masks, cas_index_mode mode,
                                           const uint64_t* h_positions, const float* h_scores,
                                           const int64_t* h_problem_rows, int problems, const cas_solve_opts* o,
                                           float* h_weights, cas_solve_report* reports)
{
    cas::NvtxRange nvtx_range("cas_fit_weights_batched");
    CAS_REQUIRE(masks && o && h_weights && h_problem_rows && problems >= 1, CAS_ERR_INVALID_ARGUMENT,
                "cas_fit_weights_batched: bad argument");
    int64_t rows = 0;
    for (int q = 0; q < problems; q++) rows += std::max<int64_t>(h_problem_rows[q], 0);
    CAS_REQUIRE(rows == 0 || (h_positions && h_scores), CAS_ERR_INVALID_ARGUMENT,
                "cas_fit_weights_batched: null input");
    CAS_TRY(require_device());
    cas_patterns* p = nullptr;
    CAS_TRY(cas_patterns_create(masks, n_masks, mode, &p));
    const int64_t cols = cas_patterns_cols(p) * problems;
    cudaStream_t s = nullptr;
    CAS_CUDA(cudaStreamCreate(&s));
    uint64_t* d_pos = nullptr;
    float* d_s32 = nullptr;
    double *d_s = nullptr, *d_w = nullptr;
    float* d_w32 = nullptr;
    cas_status st = CAS_OK;
    auto fail = [&](cudaError_t e) {
        set_error(std::string("cas_fit_weights_batched: ") + cudaGetErrorString(e));
        st = e == cudaErrorMemoryAllocation ? CAS_ERR_OUT_OF_MEMORY : CAS_ERR_CUDA;
    };
    cudaError_t e = dmalloc(&d_pos, 16 * std::max<int64_t>(rows, 1));
    if (e == cudaSuccess) e = dmalloc(&d_s32, sizeof(float) * std::max<int64_t>(rows, 1));
    if (e == cudaSuccess) e = dmalloc(&d_s, sizeof(double) * std::max<int64_t>(rows, 1));
    if (e == cudaSuccess) e = dmalloc(&d_w, sizeof(double) * std::max<int64_t>(cols, 1));
    if (e == cudaSuccess) e = dmalloc(&d_w32, sizeof(float) * std::max<int64_t>(cols, 1));
    if (e == cudaSuccess && rows) e = cudaMemcpyAsync(d_pos, h_positions, 16 * rows, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && rows) e = cudaMemcpyAsync(d_s32, h_scores, sizeof(float) * rows, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) fail(e);
    if (st == CAS_OK) {
        { f32_to_f64_kernel<<<grid(rows), 256, 0, s>>>(d_s32, rows, d_s); cas::count_launch(); }
        st = cas_fit_weights_batched_device(p, d_pos, d_s, h_problem_rows, problems, o, d_w, reports, s);
    }
    if (st == CAS_OK || st == CAS_ERR_NOT_CONVERGED) {
        { f64_to_f32_kernel<<<grid(cols), 256, 0, s>>>(d_w, cols, d_w32); cas::count_launch(); }
        e = cudaMemcpyAsync(h_weights, d_w32, sizeof(float) * cols, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) fail(e);
    }
    cudaStreamSynchronize(s);
    dfree(d_pos);
    dfree(d_s32);
    dfree(d_s);
    dfree(d_w);
    dfree(d_w32);
    cudaStreamDestroy(s);
    cas_patterns_destroy(p);
    return st;
}

}  // extern "C"
