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
enum BSlot { bRz = 0, bPap, bAlpha, bBeta, bRr, bBn2, bRes, bTol, bTrue, bRrRef, kBSlots };
enum BFlag { bStatus = 0, bIter, bRefine, bRestart, bIterRef, kBFlags };

// A replacement that finds the recursive residual off by more than this
// (relative) restarts the problem's search direction (as in the single
// solver: the FP32 product errors have reached p).
constexpr double kBRestartDeviation = 0.1;

// Residual replacements of the mixed solver are scheduled per problem as in
// the single solver: after a drop of kBReplaceDrop since the last one, after
// refine_every iterations, or when the recursive residual meets the
// tolerance (a problem retires on its true residual only).
constexpr double kBReplaceDrop = 1e-4;

struct BDev {
    double* scal;   // [nprob][kBSlots]
    int* flags;     // [nprob][kBFlags]
    int* pdone;     // [nprob] retired problems
    int* ndone;     // number of retired problems
    int* alldone;   // 1 once every problem is retired (products return at entry)
    int* pskip;     // [nprob] no residual replacement due (retired problems included)
    int* nneed;     // problems with a replacement due this iteration
    int* skipall;   // 1 while no problem has a replacement due
    int* fin;       // CTAs of the step's beta kernel that have finished (reset by the last)
    int* nbody;     // graph replacement steps run (each due iteration adds one)
    int nprob;
};

__device__ __forceinline__ bool retired(const BDev& d, int q) { return *(volatile const int*)(d.pdone + q) != 0; }

__device__ __forceinline__ void retire(const BDev& d, int q)
{
    d.pdone[q] = 1;
    d.pskip[q] = 1;
    if (atomicAdd(d.ndone, 1) + 1 == d.nprob) *d.alldone = 1;
}

template <bool COMP>
__device__ __forceinline__ void bacc(Comp& c, double x)
{
    if (COMP)
        c.add(x);
    else
        c.s += x;
}

// The problems a vector step works on (FastActive), in problem order: the
// CTAs of the step's 1D grid are dealt round-robin over them (CTA i serves
// list slot i % n as its (i / n)-th CTA), so a lone remaining problem gets
// the whole grid and 60 problems about 10 CTAs each.  Partials live at
// part[q][rank]; a reduction over problem q sums the ranks its slot had.
// The same list tells the products which problems' blocks and items run.
using ActiveList = FastActive;

struct Slot {
    int q, rank, ranks;  // problem, CTA rank within it, CTAs serving it
};

__device__ __forceinline__ bool cta_slot(const ActiveList* al, Slot& sl)
{
    const int n = al->n;
    if (n == 0) return false;
    const int a = static_cast<int>(blockIdx.x) % n;
    sl.q = al->list[a];
    sl.rank = static_cast<int>(blockIdx.x) / n;
    sl.ranks = (static_cast<int>(gridDim.x) - a + n - 1) / n;
    return true;
}

// CTAs that served problem q in a step over G CTAs (0 if q is not listed).
__device__ __forceinline__ int ranks_of(const ActiveList* al, int q, int G)
{
    const int n = al->n, a = al->pos[q];
    return (n == 0 || a < 0) ? 0 : (G - a + n - 1) / n;
}

// Rebuilds the list of problems not retired (one warp per 32 problems:
// threads 0..63 of the calling CTA; every thread of it must call).
__device__ void compact_active(const int* __restrict__ pdone, int nprob, ActiveList* al, int* base)
{
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const bool act = t < nprob && !*(volatile const int*)(pdone + t);
    unsigned m = 0;
    if (t < 64) m = __ballot_sync(0xffffffffu, act);
    if (t < 64 && lane == 0) base[w + 1] = __popc(m);
    if (t == 0) base[0] = 0;
    __syncthreads();
    if (t < nprob) {
        const int before = (w == 0 ? 0 : base[1]) + __popc(m & ((1u << lane) - 1));
        al->pos[t] = act ? before : -1;
        if (act) al->list[before] = t;
    }
    if (t == 0) al->n = base[1] + base[2];
}

__global__ void bcompact_kernel(const int* __restrict__ pdone, int nprob, ActiveList* al)
{
    __shared__ int base[3];
    compact_active(pdone, nprob, al, base);
}

// Partial (s, c) of one CTA into part[2 * (q * G + rank)].
template <bool COMP>
__device__ void bwrite(double* part, const Slot& sl, Comp v, double* smem)
{
    const Comp r = block_sum_comp<kBVecThreads>(v, smem);
    if (threadIdx.x == 0) {
        const int64_t i = static_cast<int64_t>(sl.q) * gridDim.x + sl.rank;
        part[2 * i] = r.s;
        part[2 * i + 1] = COMP ? r.c : 0.0;
    }
}

// Sum of n partial pairs from part, by one block of THREADS threads (valid
// in thread 0).
template <bool COMP, int THREADS = kBRedThreads>
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
    if (COMP) return block_sum_comp<THREADS>(acc, smem).value();
    return block_sum<THREADS>(acc.s, smem);
}

// ||A'q||^2 per listed problem from the product partials (T = partial type).
template <typename T>
__global__ void __launch_bounds__(kBVecThreads) bnorm_kernel(FastCols fc, const T* __restrict__ partial,
                                                             double* __restrict__ part, const ActiveList* al)
{
    __shared__ double smem[64];
    Slot sl;
    if (!cta_slot(al, sl)) return;
    const int64_t P = fc.g.pcols, base = sl.q * P;
    Comp acc;
    for (int64_t c = static_cast<int64_t>(sl.rank) * blockDim.x + threadIdx.x; c < P;
         c += static_cast<int64_t>(sl.ranks) * blockDim.x) {
        const double v = fast_col_sum<T>(fc, partial, base + c);
        acc.add(v * v);
    }
    bwrite<true>(part, sl, acc, smem);
}

__global__ void __launch_bounds__(kBRedThreads) bstore_kernel(const double* __restrict__ part, int G,
                                                              const ActiveList* al, BDev d, int slot)
{
    __shared__ double smem[64];
    const int q = blockIdx.x;
    const int k = ranks_of(al, q, G);
    if (k == 0) return;
    const double v = bsum<true>(part + 2 * static_cast<int64_t>(q) * G, k, smem);
    if (threadIdx.x == 0) d.scal[q * kBSlots + slot] = v;
}

// r = A'(b - A x) from the FP64 product, z = D r; p = z on (re)start.
// Partials of r.z and r.r per (problem, CTA), and (part_dev not null) of
// ||r_rec - r||^2 against the recursive residual being replaced.
template <bool COMP, typename G>
__global__ void __launch_bounds__(kBVecThreads) bresidual_kernel(FastCols fc, const double* __restrict__ partial,
                                                                 double* __restrict__ r, double* __restrict__ z,
                                                                 double* __restrict__ p, G* __restrict__ pg,
                                                                 const double* __restrict__ dinv,
                                                                 const ActiveList* al,
                                                                 double* __restrict__ part_rz,
                                                                 double* __restrict__ part_rr, int restart, BDev d,
                                                                 double* __restrict__ part_dev,
                                                                 const int* __restrict__ qgate)
{
    __shared__ double smem[64];
    Slot sl;
    if (!cta_slot(al, sl) || *(volatile const int*)(qgate + sl.q)) return;
    const int q = sl.q;
    const int64_t P = fc.g.pcols, base = q * P;
    Comp rz, rr, dev;
    for (int64_t c = static_cast<int64_t>(sl.rank) * blockDim.x + threadIdx.x; c < P;
         c += static_cast<int64_t>(sl.ranks) * blockDim.x) {
        const int64_t i = base + c;
        const double rc = fast_col_sum<double>(fc, partial, i);
        const double zc = dinv[i] * rc;
        if (part_dev) {
            const double dd = r[i] - rc;
            bacc<COMP>(dev, dd * dd);
        }
        r[i] = rc;
        z[i] = zc;
        if (restart) {
            p[i] = zc;
            if (pg) pg[i] = static_cast<G>(zc);
        }
        bacc<COMP>(rz, rc * zc);
        bacc<COMP>(rr, rc * rc);
    }
    bwrite<COMP>(part_rz, sl, rz, smem);
    bwrite<COMP>(part_rr, sl, rr, smem);
    if (part_dev) bwrite<COMP>(part_dev, sl, dev, smem);
}

// p = z (and the gather copy) for the problems whose replacement set bRestart.
template <typename G>
__global__ void __launch_bounds__(kBVecThreads) brestart_kernel(int64_t P, const ActiveList* al,
                                                                const double* __restrict__ z, double* __restrict__ p,
                                                                G* __restrict__ pg, BDev d)
{
    Slot sl;
    if (!cta_slot(al, sl)) return;
    const int q = sl.q;
    if (retired(d, q) || !*(volatile const int*)(d.flags + q * kBFlags + bRestart)) return;
    const int64_t base = q * P;
    for (int64_t c = static_cast<int64_t>(sl.rank) * blockDim.x + threadIdx.x; c < P;
         c += static_cast<int64_t>(sl.ranks) * blockDim.x) {
        p[base + c] = z[base + c];
        if (pg) pg[base + c] = static_cast<G>(z[base + c]);
    }
}

// alpha = rz / p'A'Ap per problem, then x += alpha p; r -= alpha A'A p;
// z = D r; partials of r.z, r.r.  p'A'Ap is the sum of the A p norm
// partials of the problem's blocks (kAxSplitMax per block), summed by every
// CTA of the problem in the same order, so all of them get the same alpha;
// the problem's first CTA stores it.  p'A'Ap <= 0 means p lies in the null
// space of A (a rank-deficient problem, or the residual at rounding level):
// the problem retires and the FP64 true residual decides between converged
// and a restart from it; a non-finite p'A'Ap is a breakdown.
template <bool COMP, typename T>
__global__ void __launch_bounds__(kBVecThreads) bupdate_kernel(FastCols fc, const T* __restrict__ partial,
                                                               double* __restrict__ x, double* __restrict__ r,
                                                               double* __restrict__ z, const double* __restrict__ p,
                                                               const double* __restrict__ dinv,
                                                               const ActiveList* al,
                                                               const double* __restrict__ part_q,
                                                               double* __restrict__ part_rz,
                                                               double* __restrict__ part_rr, BDev d)
{
    __shared__ double smem[64];
    __shared__ double s_pap;
    Slot sl;
    if (!cta_slot(al, sl) || retired(d, sl.q)) return;
    const int q = sl.q;
    const int b0 = fc.g.pblk0[q], nb = fc.g.pblk0[q + 1] - fc.g.pblk0[q];
    const double pap_sum = bsum<COMP, kBVecThreads>(part_q + 2 * static_cast<int64_t>(b0) * kAxSplitMax,
                                                    nb * kAxSplitMax, smem);
    if (threadIdx.x == 0) s_pap = pap_sum;
    __syncthreads();
    const double pap = s_pap;
    double* sc = d.scal + q * kBSlots;
    const bool ok = pap > 0 && isfinite(pap);
    if (sl.rank == 0 && threadIdx.x == 0) {
        sc[bPap] = pap;
        sc[bAlpha] = ok ? sc[bRz] / pap : 0.0;
        if (!ok) {
            if (!isfinite(pap)) d.flags[q * kBFlags + bStatus] = CAS_ERR_BREAKDOWN;
            retire(d, q);
        }
    }
    if (!ok) return;
    const double alpha = sc[bRz] / pap;
    const int64_t P = fc.g.pcols, base = q * P;
    Comp rz, rr;
    for (int64_t c = static_cast<int64_t>(sl.rank) * blockDim.x + threadIdx.x; c < P;
         c += static_cast<int64_t>(sl.ranks) * blockDim.x) {
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
    bwrite<COMP>(part_rz, sl, rz, smem);
    bwrite<COMP>(part_rr, sl, rr, smem);
}

// rz_new, rr -> beta, relative residual, retirement.  replace != 0: residual
// replacement (r.z replaced, beta and the iteration count left alone).
//
// With next (the step's beta kernel), the last CTA to finish also prepares
// the next steps: the whole-launch gate of this iteration's replacement
// step (skipall, set while no problem has one due; the count of due
// problems reset), with use_cond the condition of the replacement step's
// graph node and the count of such steps run (nbody), and the list of
// problems still active for the next iteration.
template <bool COMP>
__global__ void __launch_bounds__(kBRedThreads) bbeta_kernel(const double* __restrict__ part_rz,
                                                             const double* __restrict__ part_rr, int G,
                                                             const ActiveList* al, BDev d, int replace,
                                                             const double* __restrict__ part_dev,
                                                             const int* __restrict__ qgate, int plan_refine,
                                                             ActiveList* next, int use_cond,
                                                             cudaGraphConditionalHandle cond)
{
    __shared__ double smem[64];
    __shared__ int s_last;
    __shared__ int base[3];
    const int q = blockIdx.x;
    const int k = ranks_of(al, q, G);
    if (!*(volatile const int*)(qgate + q) && k != 0) {
        const int64_t o = 2 * static_cast<int64_t>(q) * G;
        const double rz_new = bsum<COMP>(part_rz + o, k, smem);
        const double rr = bsum<COMP>(part_rr + o, k, smem);
        const double dev2 = part_dev ? bsum<COMP>(part_dev + o, k, smem) : 0.0;
        if (threadIdx.x == 0) {
            double* sc = d.scal + q * kBSlots;
            int* fl = d.flags + q * kBFlags;
            if (part_dev) fl[bRestart] = dev2 > kBRestartDeviation * kBRestartDeviation * rr ? 1 : 0;
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
            if (replace) {
                sc[bRrRef] = rr;
                fl[bIterRef] = fl[bIter];
            }
            const bool met = rr == 0 || (sc[bTol] > 0 && res <= sc[bTol]);
            if (!isfinite(rz_new) || !isfinite(rr)) {
                fl[bStatus] = CAS_ERR_BREAKDOWN;
                retire(d, q);
            } else if (!replace && plan_refine > 0) {
                fl[bRestart] = 0;
                const bool due = met || rr <= kBReplaceDrop * kBReplaceDrop * sc[bRrRef] ||
                                 fl[bIter] - fl[bIterRef] >= plan_refine;
                d.pskip[q] = due ? 0 : 1;
                if (due) atomicAdd(d.nneed, 1);
            } else if (met) {
                retire(d, q);
            }
        }
    }
    if (!next) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();  // this CTA's flags before its count
        s_last = atomicAdd(d.fin, 1) == static_cast<int>(gridDim.x) - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) {
        *d.fin = 0;
        if (plan_refine > 0) {
            const int skip = (*(volatile int*)d.alldone || atomicAdd(d.nneed, 0) == 0) ? 1 : 0;
            *d.skipall = skip;
            *d.nneed = 0;
            if (use_cond) {
                cudaGraphSetConditional(cond, skip ? 0u : 1u);
                if (!skip) *d.nbody += 1;
            }
        }
    }
    compact_active(d.pdone, d.nprob, next, base);
}

// p = z + beta p (and the gather copy).
template <typename G>
__global__ void __launch_bounds__(kBVecThreads) bdirection_kernel(int64_t P, const ActiveList* al,
                                                                  const double* __restrict__ z, double* __restrict__ p,
                                                                  G* __restrict__ pg, BDev d)
{
    Slot sl;
    if (!cta_slot(al, sl) || retired(d, sl.q)) return;
    const int q = sl.q;
    const double beta = d.scal[q * kBSlots + bBeta];
    const int64_t base = q * P;
    for (int64_t c = static_cast<int64_t>(sl.rank) * blockDim.x + threadIdx.x; c < P;
         c += static_cast<int64_t>(sl.ranks) * blockDim.x) {
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
    int B = 0, G = 1;  // problems; CTAs of a vector step
    int64_t P = 0, C = 0, R = 0;
    double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *dinv = nullptr;
    float* pg32 = nullptr;
    void* q = nullptr;
    double* q64 = nullptr;
    const double* b = nullptr;
    double *part_q = nullptr, *part_a = nullptr, *part_b = nullptr, *part_c = nullptr;
    double* scal = nullptr;
    int* flags = nullptr;  // [B][kBFlags] then pdone[B], ndone, alldone, pskip[B], nneed, skipall, fin, nbody
    ActiveList* act = nullptr;  // problems not retired (rebuilt every iteration)
    ActiveList* all = nullptr;  // every problem
    std::vector<double> h_scal;
    std::vector<int> h_flags;
    cudaGraphExec_t graph = nullptr;
    int graph_len = 0, graph_phase = -1;
    long long graph_kernels = 0;
    cudaStream_t s2 = nullptr;     // captures the bodies of the replacement steps' graph nodes
    long long body_kernels = 0;    // kernels of one replacement step
    int nbody_seen = 0;            // replacement steps already counted
    int launched = 0;

    BDev dev() const
    {
        BDev d;
        d.scal = scal;
        d.flags = flags;
        d.pdone = flags + B * kBFlags;
        d.ndone = d.pdone + B;
        d.alldone = d.ndone + 1;
        d.pskip = d.alldone + 1;
        d.nneed = d.pskip + B;
        d.skipall = d.nneed + 1;
        d.fin = d.skipall + 1;
        d.nbody = d.fin + 1;
        d.nprob = B;
        return d;
    }
    int nflags() const { return B * kBFlags + B + 2 + B + 2 + 2; }
    int nbody_index() const { return nflags() - 1; }
    dim3 vgrid() const { return dim3(static_cast<unsigned>(G)); }

    ~BatchSolver()
    {
        if (graph) cudaGraphExecDestroy(graph);
        if (own_stream) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
        if (s2) cudaStreamDestroy(s2);
        for (void* ptr : {(void*)x, (void*)r, (void*)z, (void*)p, (void*)dinv, (void*)pg32, q, (void*)q64,
                          (void*)part_q, (void*)part_a, (void*)part_b, (void*)part_c, (void*)scal,
                          (void*)flags, (void*)act, (void*)all})
            dfree(ptr);
    }

    // How a residual replacement selects its problems.
    enum class Sel { All, Active, Due };

    // A'(b - A x) in FP64 into the t64 partials, for all problems, the
    // active ones, or those with a replacement due.
    // (Sel::Active rebuilds the active list first: the host resumed problems.)
    cas_status residual_products(Sel sel)
    {
        const BDev d = dev();
        int* whole = sel == Sel::All ? nullptr : (sel == Sel::Active ? d.alldone : d.skipall);
        const int* per = sel == Sel::All ? nullptr : (sel == Sel::Active ? d.pdone : d.pskip);
        if (sel == Sel::Active) { bcompact_kernel<<<1, 64, 0, s>>>(d.pdone, B, act); cas::count_launch(); }
        const ActiveList* al = sel == Sel::All ? all : act;
        CAS_TRY((fast_spmv<double, double>(*f, x, q64, b, nullptr, part_q, whole, 2, s, nullptr, per, al)));
        return fast_spmv_t_partials<double>(*f, q64, whole, s, per, al);
    }

    // Residual replacement (restart: p = z too) for the active problems.
    // Residual replacement.  Sel::All / Sel::Active (set-up, resumption):
    // r, z and p = z restart.  Sel::Due (the in-graph step of the mixed
    // solver, every iteration, gated by the beta kernel's schedule): measures
    // the recursive residual's drift and restarts the direction of the
    // problems whose drift exceeds kBRestartDeviation; retires the problems
    // whose true residual meets the tolerance.
    // reuse_atb (set-up): x is zero and the FP64 partials hold A'b, which is
    // then the residual A'(b - A x) itself.
    template <bool COMP>
    cas_status refine(Sel sel, bool reuse_atb = false)
    {
        if (!reuse_atb) CAS_TRY(residual_products(sel));
        const BDev d = dev();
        const FastCols fc = fast_cols<double>(*f);
        const double* t64 = static_cast<const double*>(f->t64.partial);
        const bool restart = sel != Sel::Due;
        double* pdev = restart ? nullptr : part_c;
        const int* qgate = sel == Sel::Due ? d.pskip : d.pdone;
        // Sel::All works on every problem; the others on the active list
        const ActiveList* al = sel == Sel::All ? all : act;
        if (mixed)
            { bresidual_kernel<COMP, float><<<vgrid(), kBVecThreads, 0, s>>>(fc, t64, r, z, p, pg32, dinv, al, part_a,
                                                                        part_b, restart ? 1 : 0, d, pdev, qgate); cas::count_launch(); }
        else
            { bresidual_kernel<COMP, double><<<vgrid(), kBVecThreads, 0, s>>>(fc, t64, r, z, p, nullptr, dinv, al,
                                                                         part_a, part_b, restart ? 1 : 0, d, pdev,
                                                                         qgate); cas::count_launch(); }
        { bbeta_kernel<COMP><<<B, kBRedThreads, 0, s>>>(part_a, part_b, G, al, d, 1, pdev, qgate, 0, nullptr, 0, 0); cas::count_launch(); }
        if (pdev) {
            if (mixed)
                { brestart_kernel<float><<<vgrid(), kBVecThreads, 0, s>>>(P, al, z, p, pg32, d); cas::count_launch(); }
            else
                { brestart_kernel<double><<<vgrid(), kBVecThreads, 0, s>>>(P, al, z, p, nullptr, d); cas::count_launch(); }
        }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }

    // One iteration.  The active list was rebuilt by the previous
    // iteration's beta kernel (or by the set-up / resumption); a problem
    // retired since then is still listed and skipped by every kernel.  The
    // beta kernel plans this iteration's replacement step and, with
    // use_cond, sets the condition of its graph node.
    template <bool COMP, typename T>
    cas_status iteration(int use_cond, cudaGraphConditionalHandle cond)
    {
        const BDev d = dev();
        const T* pgather = std::is_same<T, float>::value ? reinterpret_cast<const T*>(pg32) : reinterpret_cast<const T*>(p);
        CAS_TRY((fast_spmv<T, T>(*f, pgather, static_cast<T*>(q), nullptr, nullptr, part_q, d.alldone, 0, s, nullptr,
                                 d.pdone, act)));
        CAS_TRY(fast_spmv_t_partials<T>(*f, static_cast<const T*>(q), d.alldone, s, d.pdone, act));
        const FastCols fc = fast_cols<T>(*f);
        { bupdate_kernel<COMP, T><<<vgrid(), kBVecThreads, 0, s>>>(fc, static_cast<const T*>(sizeof(T) == 4 ? f->t32.partial
                                                                                                        : f->t64.partial),
                                                                  x, r, z, p, dinv, act, part_q, part_a, part_b, d); cas::count_launch(); }
        { bbeta_kernel<COMP><<<B, kBRedThreads, 0, s>>>(part_a, part_b, G, act, d, 0, nullptr, d.pdone,
                                                       mixed ? std::max(o.refine_every, 1) : 0, act, use_cond,
                                                       cond); cas::count_launch(); }
        if (mixed)
            { bdirection_kernel<float><<<vgrid(), kBVecThreads, 0, s>>>(P, act, z, p, pg32, d); cas::count_launch(); }
        else
            { bdirection_kernel<double><<<vgrid(), kBVecThreads, 0, s>>>(P, act, z, p, nullptr, d); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }

    // The mixed solver's replacement step of an iteration being captured:
    // a conditional graph node whose body (captured on s2) runs only when
    // the beta kernel found a replacement due.  Kernels of the body are
    // counted when they run (nbody).
    cas_status capture_replacement(cudaGraphConditionalHandle h)
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        CAS_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd));
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeIf;
        np.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        CAS_CUDA(cudaGraphAddNode(&node, cg, deps, nd, &np));
        cudaGraph_t body = np.conditional.phGraph_out[0];
        CAS_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
        CAS_CUDA(cudaStreamBeginCaptureToGraph(s2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        std::swap(s, s2);
        const long long before = launch_count();
        const cas_status st = refine<true>(Sel::Due);
        body_kernels = launch_count() - before;
        count_launch(-body_kernels);  // counted when the body runs
        std::swap(s, s2);
        cudaGraph_t out = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s2, &out);
        CAS_TRY(st);
        CAS_CUDA(e);
        return CAS_OK;
    }

    cas_status issue_iteration(bool capturing)
    {
        if (mixed) {
            if (capturing) {
                cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
                cudaGraph_t cg = nullptr;
                CAS_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, nullptr, nullptr));
                cudaGraphConditionalHandle h = 0;
                CAS_CUDA(cudaGraphConditionalHandleCreate(&h, cg, 0, cudaGraphCondAssignDefault));
                CAS_TRY((iteration<true, float>(1, h)));
                CAS_TRY(capture_replacement(h));
            } else {
                CAS_TRY((iteration<true, float>(0, 0)));
                CAS_TRY(refine<true>(Sel::Due));  // runs only for problems the beta kernel scheduled
            }
        } else {
            CAS_TRY((iteration<false, double>(0, 0)));
        }
        return CAS_OK;
    }

    cas_status issue_chunk(int n)
    {
        const int phase = 0;  // every iteration is the same graph segment
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
                for (int i = 0; i < n && st == CAS_OK; i++) st = issue_iteration(true);
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
            for (int i = 0; i < n; i++) CAS_TRY(issue_iteration(false));
        }
        launched += n;
        return CAS_OK;
    }

    cas_status read_state()
    {
        CAS_CUDA(cudaMemcpyAsync(h_scal.data(), scal, sizeof(double) * h_scal.size(), cudaMemcpyDeviceToHost, s));
        CAS_CUDA(cudaMemcpyAsync(h_flags.data(), flags, sizeof(int) * h_flags.size(), cudaMemcpyDeviceToHost, s));
        CAS_CUDA(cudaStreamSynchronize(s));
        const int nb = h_flags[nbody_index()];
        if (nb > nbody_seen) count_launch(static_cast<long long>(nb - nbody_seen) * body_kernels);
        nbody_seen = nb;
        return CAS_OK;
    }

    // ||A'(b - A x)||^2 of every problem into slot bTrue (all problems).
    cas_status true_residuals()
    {
        CAS_TRY(residual_products(Sel::All));
        const BDev d = dev();
        { bnorm_kernel<double><<<vgrid(), kBVecThreads, 0, s>>>(fast_cols<double>(*f), static_cast<const double*>(f->t64.partial),
                                                                part_a, all); cas::count_launch(); }
        { bstore_kernel<<<B, kBRedThreads, 0, s>>>(part_a, G, all, d, bTrue); cas::count_launch(); }
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
        G = 4 * sm_count();
        if (stream) {
            s = static_cast<cudaStream_t>(stream);
        } else {
            CAS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            own_stream = true;
        }
        if (mixed) CAS_CUDA(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
        const size_t cb = sizeof(double) * std::max<int64_t>(C, 1), rb = sizeof(double) * std::max<int64_t>(R, 1);
        for (double** ptr : {&x, &r, &z, &p, &dinv}) CAS_CUDA(dmalloc(ptr, cb));
        if (mixed) CAS_CUDA(dmalloc(&pg32, sizeof(float) * std::max<int64_t>(C, 1)));
        CAS_CUDA(dmalloc(&q, mixed ? sizeof(float) * std::max<int64_t>(R, 1) : rb));
        CAS_CUDA(dmalloc(&q64, rb));
        CAS_CUDA(dmalloc(&part_q, sizeof(double) * 2 * kAxSplitMax * std::max<int64_t>(f->g.nblocks, 1)));
        CAS_CUDA(dmalloc(&part_a, sizeof(double) * 2 * B * G));
        CAS_CUDA(dmalloc(&part_b, sizeof(double) * 2 * B * G));
        CAS_CUDA(dmalloc(&part_c, sizeof(double) * 2 * B * G));
        CAS_CUDA(dmalloc(&act, sizeof(ActiveList)));
        CAS_CUDA(dmalloc(&all, sizeof(ActiveList)));
        {
            ActiveList h{};
            h.n = B;
            for (int qq = 0; qq < kMaxProblems; qq++) {
                h.list[qq] = qq < B ? qq : 0;
                h.pos[qq] = qq < B ? qq : -1;
            }
            CAS_CUDA(cudaMemcpy(all, &h, sizeof h, cudaMemcpyHostToDevice));
            CAS_CUDA(cudaMemcpy(act, &h, sizeof h, cudaMemcpyHostToDevice));
        }
        CAS_CUDA(dmalloc(&scal, sizeof(double) * B * kBSlots));
        h_scal.assign(static_cast<size_t>(B) * kBSlots, 0.0);
        CAS_CUDA(dmalloc(&flags, sizeof(int) * nflags()));
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
                                                                part_a, all); cas::count_launch(); }
        { bstore_kernel<<<B, kBRedThreads, 0, s>>>(part_a, G, all, d, bBn2); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        // r = A'b (the partials just summed), z = D r, p = z (x = 0); no
        // replacement due yet
        if (mixed)
            CAS_TRY(refine<true>(Sel::All, true));
        else
            CAS_TRY(refine<false>(Sel::All, true));
        CAS_TRY(read_state());
        // the initial residual counted as a refinement: reset the counters;
        // no replacement is due before the first iteration's schedule
        for (int qq = 0; qq < B; qq++) h_flags[qq * kBFlags + bRefine] = 0;
        for (int qq = 0; qq < B; qq++) h_flags[B * kBFlags + B + 2 + qq] = 1;
        h_flags[B * kBFlags + B + 2 + B + 1] = 1;
        CAS_CUDA(cudaMemcpyAsync(flags, h_flags.data(), sizeof(int) * nflags(), cudaMemcpyHostToDevice, s));
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
                tail.insert(tail.end(), pdh.begin(), pdh.end());  // pskip: retired ones stay skipped
                tail.push_back(0);
                tail.push_back(1);
                CAS_CUDA(cudaMemcpyAsync(flags + B * kBFlags, tail.data(), sizeof(int) * (2 * B + 4),
                                         cudaMemcpyHostToDevice, s));
                if (mixed)
                    CAS_TRY(refine<true>(Sel::Active));
                else
                    CAS_TRY(refine<false>(Sel::Active));
                CAS_CUDA(cudaStreamSynchronize(s));  // the host vector above must outlive the copy
                verified = false;
                continue;
            }
            const int n = std::min(chunk, o.max_iterations - launched);
            CAS_TRY(issue_chunk(n));
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
    cas::NvtxRange nvtx_range("cas_solve_batched");
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
