// Batched Jacobi-PCG: the independent per-stage fits of the reference's
// training loop (PatternFit/PatternFit.cpp:53-84 fits one estimator per
// empty-count stage, one after another) solved together.
//
// The batch is one block-diagonal CSR in the blocked layout (problem q owns
// its rows and the columns [q * P, (q + 1) * P)), built by
// cas_csr_from_positions_batched.  Each problem runs its own PCG
// (Math/Solver.h:78-117) with its own alpha, beta, residual and stopping
// test: the products cover all problems in one launch each, and the vector
// steps run on a (CTAs per problem) x (problems) grid whose reductions stay
// inside one problem.  A problem that reaches the tolerance is retired: its
// flag in pdone makes every later kernel skip its blocks, work items and
// columns, so the cost of an iteration shrinks as problems converge.
// Iterations are captured once as a CUDA graph chunk and replayed.
//
// Precision follows the single solver: mixed = FP32 products and FP32
// gather copy of p, FP64 vectors and compensated FP64 scalars, residual
// replaced by the FP64 true residual every refine_every iterations; plain =
// FP64 products.  Converged problems are verified with the FP64 true
// residual and resumed (with a restarted search direction) if it is above
// the tolerance.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "fast.cuh"
#include "internal.cuh"

namespace cas {
namespace {

constexpr int kBVecThreads = 256;
constexpr int kBRedThreads = 512;

// Per-problem scalar slots (stride kBSlots) and flags (stride kBFlags).
enum BSlot { bRz = 0, bPap, bAlpha, bBeta, bRr, bBn2, bRes, bTol, bTrue, kBSlots };
enum BFlag { bStatus = 0, bIter, bRefine, kBFlags };

struct BDev {
    double* scal;   // [nprob][kBSlots]
    int* flags;     // [nprob][kBFlags]
    int* pdone;     // [nprob] retired problems
    int* ndone;     // number of retired problems
    int* alldone;   // 1 once every problem is retired (products return at entry)
    int nprob;
};

__device__ __forceinline__ bool retired(const BDev& d, int q) { return *(volatile const int*)(d.pdone + q) != 0; }

template <bool COMP>
__device__ __forceinline__ void bacc(Comp& c, double x)
{
    if (COMP)
        c.add(x);
    else
        c.s += x;
}

// Partial (s, c) of one CTA into part[2 * (q * nbx + bx)].
template <bool COMP>
__device__ void bwrite(double* part, int q, int nbx, Comp v, double* smem)
{
    const Comp r = block_sum_comp<kBVecThreads>(v, smem);
    if (threadIdx.x == 0) {
        part[2 * (q * nbx + blockIdx.x)] = r.s;
        part[2 * (q * nbx + blockIdx.x) + 1] = COMP ? r.c : 0.0;
    }
}

// Sum of n partial pairs from part, by one block.
template <bool COMP>
__device__ double bsum(const double* part, int n, double* smem)
{
    Comp acc;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        if (COMP) {
            acc.add(part[2 * i]);
            acc.add(part[2 * i + 1]);
        } else {
            acc.s += part[2 * i];
        }
    }
    if (COMP) return block_sum_comp<kBRedThreads>(acc, smem).value();
    return block_sum<kBRedThreads>(acc.s, smem);
}

// ||A'q||^2 per problem from the product partials (T = partial type).
template <typename T>
__global__ void __launch_bounds__(kBVecThreads) bnorm_kernel(FastCols fc, const T* __restrict__ partial, int nbx,
                                                             double* __restrict__ part, BDev d, int skip_retired)
{
    __shared__ double smem[64];
    const int q = blockIdx.y;
    if (skip_retired && retired(d, q)) return;
    const int64_t P = fc.g.pcols, base = q * P;
    Comp acc;
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < P;
         c += static_cast<int64_t>(nbx) * blockDim.x) {
        const double v = fast_col_sum<T>(fc, partial, base + c);
        acc.add(v * v);
    }
    bwrite<true>(part, q, nbx, acc, smem);
}

__global__ void __launch_bounds__(kBRedThreads) bstore_kernel(const double* __restrict__ part, int nbx, BDev d,
                                                              int slot, int skip_retired)
{
    __shared__ double smem[64];
    const int q = blockIdx.x;
    if (skip_retired && retired(d, q)) return;
    const double v = bsum<true>(part + 2 * q * nbx, nbx, smem);
    if (threadIdx.x == 0) d.scal[q * kBSlots + slot] = v;
}

// r = A'(b - A x) from the FP64 product, z = D r; p = z on (re)start.
// Partials of r.z and r.r per (problem, CTA).
template <bool COMP, typename G>
__global__ void __launch_bounds__(kBVecThreads) bresidual_kernel(FastCols fc, const double* __restrict__ partial,
                                                                 double* __restrict__ r, double* __restrict__ z,
                                                                 double* __restrict__ p, G* __restrict__ pg,
                                                                 const double* __restrict__ dinv, int nbx,
                                                                 double* __restrict__ part_rz,
                                                                 double* __restrict__ part_rr, int restart, BDev d)
{
    __shared__ double smem[64];
    const int q = blockIdx.y;
    if (retired(d, q)) return;
    const int64_t P = fc.g.pcols, base = q * P;
    Comp rz, rr;
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < P;
         c += static_cast<int64_t>(nbx) * blockDim.x) {
        const int64_t i = base + c;
        const double rc = fast_col_sum<double>(fc, partial, i);
        const double zc = dinv[i] * rc;
        r[i] = rc;
        z[i] = zc;
        if (restart) {
            p[i] = zc;
            if (pg) pg[i] = static_cast<G>(zc);
        }
        bacc<COMP>(rz, rc * zc);
        bacc<COMP>(rr, rc * rc);
    }
    bwrite<COMP>(part_rz, q, nbx, rz, smem);
    bwrite<COMP>(part_rr, q, nbx, rr, smem);
}

// alpha = rz / p'A'Ap per problem; p'A'Ap = sum of the A p norm partials of
// the problem's blocks.  Breakdown when p'A'Ap <= 0 with rz > 0.
template <bool COMP>
__global__ void __launch_bounds__(kBRedThreads) balpha_kernel(FastGeometry g, const double* __restrict__ part_q, BDev d)
{
    __shared__ double smem[64];
    const int q = blockIdx.x;
    if (retired(d, q)) return;
    const int b0 = g.pblk0[q], nb = g.pblk0[q + 1] - g.pblk0[q];
    const double pap = bsum<COMP>(part_q + 2 * b0, nb, smem);
    if (threadIdx.x == 0) {
        double* sc = d.scal + q * kBSlots;
        sc[bPap] = pap;
        const double rz = sc[bRz];
        if (!(pap > 0) || !isfinite(pap)) {
            sc[bAlpha] = 0;
            if (rz > 0 || !isfinite(pap)) d.flags[q * kBFlags + bStatus] = CAS_ERR_BREAKDOWN;
            d.pdone[q] = 1;
            if (atomicAdd(d.ndone, 1) + 1 == d.nprob) *d.alldone = 1;
        } else {
            sc[bAlpha] = rz / pap;
        }
    }
}

// x += alpha p; r -= alpha A'A p; z = D r; partials of r.z, r.r.
template <bool COMP, typename T>
__global__ void __launch_bounds__(kBVecThreads) bupdate_kernel(FastCols fc, const T* __restrict__ partial,
                                                               double* __restrict__ x, double* __restrict__ r,
                                                               double* __restrict__ z, const double* __restrict__ p,
                                                               const double* __restrict__ dinv, int nbx,
                                                               double* __restrict__ part_rz,
                                                               double* __restrict__ part_rr, BDev d)
{
    __shared__ double smem[64];
    const int q = blockIdx.y;
    if (retired(d, q)) return;
    const double alpha = d.scal[q * kBSlots + bAlpha];
    const int64_t P = fc.g.pcols, base = q * P;
    Comp rz, rr;
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < P;
         c += static_cast<int64_t>(nbx) * blockDim.x) {
        const int64_t i = base + c;
        const double s = fast_col_sum<T>(fc, partial, i);
        x[i] += alpha * p[i];
        const double rc = r[i] - alpha * s;
        const double zc = dinv[i] * rc;
        r[i] = rc;
        z[i] = zc;
        bacc<COMP>(rz, rc * zc);
        bacc<COMP>(rr, rc * rc);
    }
    bwrite<COMP>(part_rz, q, nbx, rz, smem);
    bwrite<COMP>(part_rr, q, nbx, rr, smem);
}

// rz_new, rr -> beta, relative residual, retirement.  replace != 0: residual
// replacement (r.z replaced, beta and the iteration count left alone).
template <bool COMP>
__global__ void __launch_bounds__(kBRedThreads) bbeta_kernel(const double* __restrict__ part_rz,
                                                             const double* __restrict__ part_rr, int nbx, BDev d,
                                                             int replace)
{
    __shared__ double smem[64];
    const int q = blockIdx.x;
    if (retired(d, q)) return;
    const double rz_new = bsum<COMP>(part_rz + 2 * q * nbx, nbx, smem);
    const double rr = bsum<COMP>(part_rr + 2 * q * nbx, nbx, smem);
    if (threadIdx.x == 0) {
        double* sc = d.scal + q * kBSlots;
        int* fl = d.flags + q * kBFlags;
        const double rz = sc[bRz];
        const double bn2 = sc[bBn2];
        const double res = bn2 > 0 ? sqrt(rr / bn2) : sqrt(rr);
        if (!replace) {
            sc[bBeta] = rz != 0 ? rz_new / rz : 0.0;
            fl[bIter] += 1;
        } else {
            fl[bRefine] += 1;
        }
        sc[bRz] = rz_new;
        sc[bRr] = rr;
        sc[bRes] = res;
        bool stop = false;
        if (!isfinite(rz_new) || !isfinite(rr)) {
            fl[bStatus] = CAS_ERR_BREAKDOWN;
            stop = true;
        } else if (rr == 0 || (sc[bTol] > 0 && res <= sc[bTol])) {
            stop = true;
        }
        if (stop) {
            d.pdone[q] = 1;
            if (atomicAdd(d.ndone, 1) + 1 == d.nprob) *d.alldone = 1;
        }
    }
}

// p = z + beta p (and the gather copy).
template <typename G>
__global__ void __launch_bounds__(kBVecThreads) bdirection_kernel(int64_t P, int nbx, const double* __restrict__ z,
                                                                  double* __restrict__ p, G* __restrict__ pg, BDev d)
{
    const int q = blockIdx.y;
    if (retired(d, q)) return;
    const double beta = d.scal[q * kBSlots + bBeta];
    const int64_t base = q * P;
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < P;
         c += static_cast<int64_t>(nbx) * blockDim.x) {
        const int64_t i = base + c;
        const double v = z[i] + beta * p[i];
        p[i] = v;
        if (pg) pg[i] = static_cast<G>(v);
    }
}

// Jacobi scaling of the batch (DiagonalPreconditioner, Math/Solver.h:25-38).
__global__ void bprecond_kernel(const uint64_t* __restrict__ diag, int64_t n, int jacobi, double* __restrict__ dinv)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double v = 1.0;
        if (jacobi) {
            v = 1.0 / static_cast<double>(diag[c]);
            if (!(isfinite(v) && fabs(v) >= 2.2250738585072014e-308)) v = 1.0;
        }
        dinv[c] = v;
    }
}

struct BatchSolver {
    const cas_csr* A = nullptr;
    const FastLayout* f = nullptr;
    cas_solve_opts o{};
    cudaStream_t s = nullptr;
    bool own_stream = false;
    bool mixed = false;
    int B = 0, nbx = 1;
    int64_t P = 0, C = 0, R = 0;
    double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *dinv = nullptr;
    float* pg32 = nullptr;
    void* q = nullptr;
    double* q64 = nullptr;
    const double* b = nullptr;
    double *part_q = nullptr, *part_a = nullptr, *part_b = nullptr;
    double* scal = nullptr;
    int* flags = nullptr;  // [B][kBFlags] then pdone[B], ndone, alldone
    std::vector<double> h_scal;
    std::vector<int> h_flags;
    cudaGraphExec_t graph = nullptr;
    int graph_len = 0, graph_phase = -1;
    long long graph_kernels = 0;
    int launched = 0;

    BDev dev() const
    {
        BDev d;
        d.scal = scal;
        d.flags = flags;
        d.pdone = flags + B * kBFlags;
        d.ndone = d.pdone + B;
        d.alldone = d.ndone + 1;
        d.nprob = B;
        return d;
    }
    int nflags() const { return B * kBFlags + B + 2; }
    dim3 vgrid() const { return dim3(static_cast<unsigned>(nbx), static_cast<unsigned>(B)); }

    ~BatchSolver()
    {
        if (graph) cudaGraphExecDestroy(graph);
        if (own_stream) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
        for (void* ptr : {(void*)x, (void*)r, (void*)z, (void*)p, (void*)dinv, (void*)pg32, q, (void*)q64,
                          (void*)part_q, (void*)part_a, (void*)part_b, (void*)scal, (void*)flags})
            cudaFree(ptr);
    }

    // A'(b - A x) in FP64 into the t64 partials; retired problems skipped
    // when `gate`.
    cas_status residual_products(bool gate)
    {
        const BDev d = dev();
        CAS_TRY((fast_spmv<double, double>(*f, x, q64, b, nullptr, part_q, gate ? d.alldone : nullptr, 2, s, nullptr,
                                           gate ? d.pdone : nullptr)));
        return fast_spmv_t_partials<double>(*f, q64, gate ? d.alldone : nullptr, s, gate ? d.pdone : nullptr);
    }

    // Residual replacement (restart: p = z too) for the active problems.
    template <bool COMP>
    cas_status refine(bool restart, bool gate)
    {
        CAS_TRY(residual_products(gate));
        const BDev d = dev();
        const FastCols fc = fast_cols<double>(*f);
        const double* t64 = static_cast<const double*>(f->t64.partial);
        if (mixed)
            { bresidual_kernel<COMP, float><<<vgrid(), kBVecThreads, 0, s>>>(fc, t64, r, z, p, pg32, dinv, nbx, part_a,
                                                                        part_b, restart ? 1 : 0, d); cas::count_launch(); }
        else
            { bresidual_kernel<COMP, double><<<vgrid(), kBVecThreads, 0, s>>>(fc, t64, r, z, p, nullptr, dinv, nbx,
                                                                         part_a, part_b, restart ? 1 : 0, d); cas::count_launch(); }
        { bbeta_kernel<COMP><<<B, kBRedThreads, 0, s>>>(part_a, part_b, nbx, d, 1); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }

    template <bool COMP, typename T>
    cas_status iteration()
    {
        const BDev d = dev();
        const T* pgather = std::is_same<T, float>::value ? reinterpret_cast<const T*>(pg32) : reinterpret_cast<const T*>(p);
        CAS_TRY((fast_spmv<T, T>(*f, pgather, static_cast<T*>(q), nullptr, nullptr, part_q, d.alldone, 0, s, nullptr,
                                 d.pdone)));
        CAS_TRY(fast_spmv_t_partials<T>(*f, static_cast<const T*>(q), d.alldone, s, d.pdone));
        { balpha_kernel<COMP><<<B, kBRedThreads, 0, s>>>(f->g, part_q, d); cas::count_launch(); }
        const FastCols fc = fast_cols<T>(*f);
        { bupdate_kernel<COMP, T><<<vgrid(), kBVecThreads, 0, s>>>(fc, static_cast<const T*>(sizeof(T) == 4 ? f->t32.partial
                                                                                                        : f->t64.partial),
                                                                  x, r, z, p, dinv, nbx, part_a, part_b, d); cas::count_launch(); }
        { bbeta_kernel<COMP><<<B, kBRedThreads, 0, s>>>(part_a, part_b, nbx, d, 0); cas::count_launch(); }
        if (mixed)
            { bdirection_kernel<float><<<vgrid(), kBVecThreads, 0, s>>>(P, nbx, z, p, pg32, d); cas::count_launch(); }
        else
            { bdirection_kernel<double><<<vgrid(), kBVecThreads, 0, s>>>(P, nbx, z, p, nullptr, d); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }

    cas_status issue_iteration(int global_index)
    {
        if (mixed) {
            CAS_TRY((iteration<true, float>()));
            if (o.refine_every > 0 && (global_index + 1) % o.refine_every == 0) CAS_TRY(refine<true>(false, true));
        } else {
            CAS_TRY((iteration<false, double>()));
        }
        return CAS_OK;
    }

    cas_status issue_chunk(int first, int n)
    {
        const int period = (mixed && o.refine_every > 0) ? o.refine_every : 1;
        const int phase = first % period;
        if (n > 1) {
            if (!graph || graph_len != n || graph_phase != phase) {
                if (graph) {
                    cudaGraphExecDestroy(graph);
                    graph = nullptr;
                }
                cudaGraph_t g = nullptr;
                CAS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                cas_status st = CAS_OK;
                const long long before = launch_count();
                for (int i = 0; i < n && st == CAS_OK; i++) st = issue_iteration(first + i);
                graph_kernels = launch_count() - before;
                count_launch(-graph_kernels);  // captured, not launched
                cudaError_t e = cudaStreamEndCapture(s, &g);
                if (st != CAS_OK) {
                    if (g) cudaGraphDestroy(g);
                    return st;
                }
                CAS_CUDA(e);
                e = cudaGraphInstantiate(&graph, g, 0);
                cudaGraphDestroy(g);
                CAS_CUDA(e);
                graph_len = n;
                graph_phase = phase;
            }
            CAS_CUDA(cudaGraphLaunch(graph, s));
            count_launch(graph_kernels);
        } else {
            for (int i = 0; i < n; i++) CAS_TRY(issue_iteration(first + i));
        }
        launched += n;
        return CAS_OK;
    }

    cas_status read_state()
    {
        CAS_CUDA(cudaMemcpyAsync(h_scal.data(), scal, sizeof(double) * h_scal.size(), cudaMemcpyDeviceToHost, s));
        CAS_CUDA(cudaMemcpyAsync(h_flags.data(), flags, sizeof(int) * h_flags.size(), cudaMemcpyDeviceToHost, s));
        CAS_CUDA(cudaStreamSynchronize(s));
        return CAS_OK;
    }

    // ||A'(b - A x)||^2 of every problem into slot bTrue (all problems).
    cas_status true_residuals()
    {
        CAS_TRY(residual_products(false));
        const BDev d = dev();
        { bnorm_kernel<double><<<vgrid(), kBVecThreads, 0, s>>>(fast_cols<double>(*f), static_cast<const double*>(f->t64.partial),
                                                                nbx, part_a, d, 0); cas::count_launch(); }
        { bstore_kernel<<<B, kBRedThreads, 0, s>>>(part_a, nbx, d, bTrue, 0); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        return read_state();
    }

    double rel_true(int qq) const
    {
        const double bn2 = h_scal[qq * kBSlots + bBn2], t = h_scal[qq * kBSlots + bTrue];
        return bn2 > 0 ? std::sqrt(t / bn2) : std::sqrt(t);
    }

    cas_status init(const double* d_b, void* stream)
    {
        f = A->fast;
        B = f->g.nprob;
        P = f->g.pcols;
        C = f->g.cols;
        R = f->g.rows;
        b = d_b;
        mixed = o.precision == CAS_MIXED;
        nbx = static_cast<int>(std::max<int64_t>(
            1, std::min<int64_t>((P + kBVecThreads - 1) / kBVecThreads, (4LL * sm_count() + B - 1) / B)));
        if (stream) {
            s = static_cast<cudaStream_t>(stream);
        } else {
            CAS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            own_stream = true;
        }
        const size_t cb = sizeof(double) * std::max<int64_t>(C, 1), rb = sizeof(double) * std::max<int64_t>(R, 1);
        for (double** ptr : {&x, &r, &z, &p, &dinv}) CAS_CUDA(cudaMalloc(ptr, cb));
        if (mixed) CAS_CUDA(cudaMalloc(&pg32, sizeof(float) * std::max<int64_t>(C, 1)));
        CAS_CUDA(cudaMalloc(&q, mixed ? sizeof(float) * std::max<int64_t>(R, 1) : rb));
        CAS_CUDA(cudaMalloc(&q64, rb));
        CAS_CUDA(cudaMalloc(&part_q, sizeof(double) * 2 * std::max<int64_t>(f->g.nblocks, 1)));
        CAS_CUDA(cudaMalloc(&part_a, sizeof(double) * 2 * B * nbx));
        CAS_CUDA(cudaMalloc(&part_b, sizeof(double) * 2 * B * nbx));
        CAS_CUDA(cudaMalloc(&scal, sizeof(double) * B * kBSlots));
        h_scal.assign(static_cast<size_t>(B) * kBSlots, 0.0);
        CAS_CUDA(cudaMalloc(&flags, sizeof(int) * nflags()));
        h_flags.assign(static_cast<size_t>(nflags()), 0);
        CAS_CUDA(cudaMemsetAsync(scal, 0, sizeof(double) * B * kBSlots, s));
        CAS_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * nflags(), s));
        for (int qq = 0; qq < B; qq++) h_scal[qq * kBSlots + bTol] = o.tol;
        CAS_CUDA(cudaMemcpyAsync(scal, h_scal.data(), sizeof(double) * h_scal.size(), cudaMemcpyHostToDevice, s));
        CAS_CUDA(cudaMemsetAsync(x, 0, cb, s));
        { bprecond_kernel<<<static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((C + 255) / 256, 4LL * sm_count()))), 256, 0, s>>>(
            A->diag_int, C, o.jacobi ? 1 : 0, dinv); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        const BDev d = dev();
        // ||A'b||^2 per problem
        CAS_TRY(fast_spmv_t_partials<double>(*f, b, nullptr, s, nullptr));
        { bnorm_kernel<double><<<vgrid(), kBVecThreads, 0, s>>>(fast_cols<double>(*f), static_cast<const double*>(f->t64.partial),
                                                                nbx, part_a, d, 0); cas::count_launch(); }
        { bstore_kernel<<<B, kBRedThreads, 0, s>>>(part_a, nbx, d, bBn2, 0); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        // r = A'b, z = D r, p = z (x = 0)
        if (mixed)
            CAS_TRY(refine<true>(true, false));
        else
            CAS_TRY(refine<false>(true, false));
        CAS_TRY(read_state());
        // the initial residual counted as a refinement: reset the counters
        for (int qq = 0; qq < B; qq++) h_flags[qq * kBFlags + bRefine] = 0;
        CAS_CUDA(cudaMemcpyAsync(flags, h_flags.data(), sizeof(int) * B * kBFlags, cudaMemcpyHostToDevice, s));
        CAS_CUDA(cudaStreamSynchronize(s));
        return CAS_OK;
    }

    cas_status run(cas_solve_report* reports, double* d_x_out)
    {
        cudaEvent_t e0, e1;
        CAS_CUDA(cudaEventCreate(&e0));
        CAS_CUDA(cudaEventCreate(&e1));
        CAS_CUDA(cudaEventRecord(e0, s));
        const int chunk = o.check_every > 0 ? o.check_every : 50;
        cas_status st = CAS_OK;
        int extra_checks = 0;
        bool verified = false;
        while (true) {
            CAS_TRY(read_state());
            const int* pd = h_flags.data() + B * kBFlags;
            for (int qq = 0; qq < B; qq++)
                if (h_flags[qq * kBFlags + bStatus] != 0 && st == CAS_OK)
                    st = static_cast<cas_status>(h_flags[qq * kBFlags + bStatus]);
            if (st != CAS_OK) break;
            const bool all = h_flags[B * kBFlags + B + 1] != 0;
            if (all || launched >= o.max_iterations) {
                // verify the retired problems with the FP64 true residual
                CAS_TRY(true_residuals());
                verified = true;
                if (o.tol <= 0 || launched >= o.max_iterations) break;
                std::vector<int> resume;
                for (int qq = 0; qq < B; qq++)
                    if (pd[qq] && rel_true(qq) > o.tol) resume.push_back(qq);
                if (resume.empty()) break;
                if (++extra_checks > 20) {
                    st = CAS_ERR_NOT_CONVERGED;
                    break;
                }
                // the recursive residual drifted: resume those problems with the
                // FP64 residual and a restarted direction
                std::vector<int> pdh(pd, pd + B);
                int nd = 0;
                for (int qq : resume) pdh[qq] = 0;
                for (int qq = 0; qq < B; qq++) nd += pdh[qq];
                std::vector<int> tail(pdh);
                tail.push_back(nd);
                tail.push_back(0);
                CAS_CUDA(cudaMemcpyAsync(flags + B * kBFlags, tail.data(), sizeof(int) * (B + 2),
                                         cudaMemcpyHostToDevice, s));
                if (mixed)
                    CAS_TRY(refine<true>(true, true));
                else
                    CAS_TRY(refine<false>(true, true));
                CAS_CUDA(cudaStreamSynchronize(s));  // the host vector above must outlive the copy
                verified = false;
                continue;
            }
            const int n = std::min(chunk, o.max_iterations - launched);
            CAS_TRY(issue_chunk(launched, n));
        }
        if (!verified && st == CAS_OK) CAS_TRY(true_residuals());
        CAS_CUDA(cudaEventRecord(e1, s));
        CAS_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        CAS_TRY(read_state());
        bool all_ok = true;
        for (int qq = 0; qq < B; qq++) {
            const double rel = rel_true(qq);
            if (o.tol > 0 && !(rel <= o.tol)) all_ok = false;
            if (reports) {
                cas_solve_report& rp = reports[qq];
                rp.iterations = h_flags[qq * kBFlags + bIter];
                rp.refinements = h_flags[qq * kBFlags + bRefine];
                rp.rel_residual = rel;
                rp.residuum = h_scal[qq * kBSlots + bRr];
                rp.seconds = ms * 1e-3;
                rp.setup_seconds = 0;
            }
        }
        if (d_x_out && C) CAS_CUDA(cudaMemcpyAsync(d_x_out, x, sizeof(double) * C, cudaMemcpyDeviceToDevice, s));
        CAS_CUDA(cudaStreamSynchronize(s));
        if (st == CAS_OK && !all_ok) st = CAS_ERR_NOT_CONVERGED;
        if (st == CAS_ERR_NOT_CONVERGED) set_error("batched solve: some problems did not reach the tolerance");
        if (st == CAS_ERR_BREAKDOWN) set_error("batched solve: breakdown (p'A'Ap <= 0 or non-finite scalar)");
        return st;
    }
};

}  // namespace
}  // namespace cas

using namespace cas;

extern "C" {

CAS_API cas_status cas_solve_batched(const cas_csr* a, const cas_solve_opts* o, const double* d_b, double* d_x,
                                     cas_solve_report* reports, void* stream)
{
    CAS_REQUIRE(a && o && (a->rows == 0 || d_b) && (a->cols == 0 || d_x), CAS_ERR_INVALID_ARGUMENT,
                "cas_solve_batched: null argument");
    CAS_REQUIRE(a->fast, CAS_ERR_INVALID_ARGUMENT,
                "cas_solve_batched: needs the blocked layout (cas_csr_from_positions_batched)");
    CAS_REQUIRE(o->method == CAS_PCG || o->method == CAS_CG, CAS_ERR_INVALID_ARGUMENT,
                "cas_solve_batched: PCG or CG only");
    CAS_REQUIRE(o->precision == CAS_PLAIN_FP64 || o->precision == CAS_MIXED, CAS_ERR_INVALID_ARGUMENT,
                "cas_solve_batched: unknown precision");
    CAS_REQUIRE(o->max_iterations >= 0 && o->tol >= 0, CAS_ERR_INVALID_ARGUMENT, "cas_solve_batched: bad options");
    CAS_TRY(require_device());
    BatchSolver bs;
    bs.A = a;
    bs.o = *o;
    if (o->method == CAS_CG) bs.o.jacobi = 0;
    CAS_TRY(bs.init(d_b, stream));
    return bs.run(reports, d_x);
}

}  // extern "C"
