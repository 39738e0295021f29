// Iterative solvers on the device: Jacobi-PCG on the normal equations
// (Math/Solver.h:78-117, driven as in PatternFit/PatternFit.cpp:29-32), CG
// (P = I, Math/Solver.h:40-76) and LSQR (Math/Solver.h:128-182).
//
// All solver state and every scalar (alpha, beta, r.z, norms) lives on the
// device, so an iteration is a fixed sequence of kernel launches with no
// host round trip; `check_every` iterations are captured once as a CUDA graph
// and replayed.  After convergence every kernel returns at entry (device
// flag), so the tail of a chunk costs only launch latency.
//
// Precision modes:
//   CAS_PLAIN_FP64  FP64 vectors, FP64 sparse products, plain FP64 sums.
//   CAS_MIXED       FP32 gather vectors (p for A p, q = A p for A' q) — exact
//                   for A's 0/1 entries up to the rounding of the vectors —
//                   FP64 accumulation inside the products, FP64 compensated
//                   (Neumaier) dots and norms, and every refine_every
//                   iterations the true normal-equation residual
//                   A'(b - A x) recomputed in FP64 and substituted for the
//                   recursive one (residual replacement, search direction
//                   kept).
#include <algorithm>
#include <cmath>
#include <vector>
#include <cstring>

#include "common.cuh"
#include "fast.cuh"
#include "internal.cuh"

namespace cas {

namespace {

constexpr int kVecThreads = 256;
constexpr int kRedThreads = 1024;

// Device scalar slots.
enum Slot {
    kRz = 0,      // r.z
    kPap = 1,     // p.A'A p = ||A p||^2
    kAlpha = 2,
    kBeta = 3,
    kRr = 4,      // r.r (Residuum of PCG)
    kBn2 = 5,     // ||A'b||^2
    kRes = 6,     // sqrt(rr / bn2), recursive
    kTol = 7,
    // LSQR
    kLAlpha = 8, kLBeta = 9, kPhiBar = 10, kRhoBar = 11, kPhiRho = 12, kThetaRho = 13, kInvBeta = 14,
    kArNorm = 15,  // |phi_bar * alpha * c| estimate of ||A'r||
    kTrue = 16,    // ||A'(b - A x)||^2 of the last true-residual evaluation
    kRrRef = 17,   // r.r right after the last residual replacement (mixed PCG)
    // LSMR (shares kLAlpha, kLBeta, kInvBeta with LSQR)
    kMAlphaBar = 18, kZetaBar = 19, kCBar = 20, kSBar = 21, kMRho = 22, kMRhoBar = 23,
    kFHbar = 24, kFX = 25, kFH = 26,  // coefficients of the h_bar, x, h updates
    kArn0 = 27,   // LSQR/LSMR: recursive ||A'r|| estimate at the last (re)start
    kBn2S = 28,   // LSQR/LSMR with column scaling: ||S A'b||^2 (denominator of the recursive estimate)
    kSlots = 29
};
// kPending: LSQR met its tolerance in the last step; the step's x/w update
// still has to run, so kDone is raised by the next step's first kernel.
// kRestart: the last residual replacement found the recursive residual off
// by more than kRestartDeviation (relative): the search direction restarts.
// kSkip: no residual replacement is due this iteration (mixed PCG), or no
// restart from the FP64 residual (mixed LSQR/LSMR); the replacement or
// restart step of every iteration returns at entry while it is set.
// kIterRef: iteration count at the last replacement.
enum Flag {
    kDone = 0, kStatus = 1, kIter = 2, kRefine = 3, kPending = 4, kRestart = 5, kSkip = 6, kIterRef = 7,
    kVerified = 8,  // the tolerance was met by a freshly computed FP64 true residual
    kFlags = 9
};

// Reliable updating of the mixed solver: when the recursive residual has
// drifted this far from the FP64 true residual that replaces it, the FP32
// product errors it carries (components outside the range of A'A) have
// reached the search direction too; the direction restarts as p = z.
// Below it, the replacement keeps the direction (a restart would discard
// the Krylov space built so far).
constexpr double kRestartDeviation = 0.1;

// Reliable updating: the mixed PCG replaces its recursive residual by the
// FP64 true residual as soon as the recursive one has dropped by this factor
// since the last replacement (so it never reaches the noise floor of the
// FP32 products, where CG would start fitting that noise), after
// refine_every iterations at the latest, and whenever it meets the
// tolerance (convergence is declared on the true residual only).
constexpr double kReplaceDrop = 1e-4;

// Mixed LSQR/LSMR restart from the FP64 residual b - A x (an outer
// refinement step on the least-squares correction) once the recursive
// estimate of ||A'r|| has dropped by this factor since the last (re)start:
// well above the relative accuracy the FP32 products leave a cycle, so a
// cycle never iterates on noise, and few enough restarts that little of
// the Krylov space is thrown away.
constexpr double kLsqrRestartDrop = 1e-4;
// A host check at a chunk boundary that finds the true residual this many
// times above the mixed cycle's recursive estimate restarts the cycle: the
// cycle has reached the floor its FP32 products leave (on the unscaled
// systems the two agree within 2x until then, measured).
constexpr double kLsqrDrift = 4.0;

__device__ __forceinline__ bool gated(const int* gate) { return gate && *(volatile const int*)gate != 0; }

struct Dev {
    double* scal;
    int* flags;
};

__device__ __forceinline__ bool finished(const int* flags) { return *(volatile const int*)flags != 0; }

// Sum of n (s, c) partial pairs in a fixed order by one block.
template <bool COMP>
__device__ double reduce_partials(const double* part, int n, double* smem)
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
    if (COMP) return block_sum_comp<kRedThreads>(acc, smem).value();
    return block_sum<kRedThreads>(acc.s, smem);
}

template <bool COMP>
__device__ void write_partial(double* part, Comp v, double* smem)
{
    if (COMP) {
        Comp r = block_sum_comp<kVecThreads>(v, smem);
        if (threadIdx.x == 0) {
            part[2 * blockIdx.x] = r.s;
            part[2 * blockIdx.x + 1] = r.c;
        }
    } else {
        double r = block_sum<kVecThreads>(v.s, smem);
        if (threadIdx.x == 0) {
            part[2 * blockIdx.x] = r;
            part[2 * blockIdx.x + 1] = 0;
        }
    }
}

template <bool COMP>
__device__ __forceinline__ void acc_add(Comp& c, double x)
{
    if (COMP)
        c.add(x);
    else
        c.s += x;
}

// ---------------------------------------------------------------------------
// Products with fused reductions.
// ---------------------------------------------------------------------------

// q = A p (+ optionally q -= coef * q_old for LSQR), partial ||q||^2.
// mode 0: q = A p.  mode 1 (LSQR): q = A p - scal[coef_slot] * q (in place).
// mode 2 (residual): q = b - A p, FP64 (b given).
template <typename T, typename Q, bool COMP, int MODE>
__global__ void __launch_bounds__(kVecThreads) spmv_norm_kernel(const uint32_t* __restrict__ idx, int64_t rows, int k,
                                                                 const T* __restrict__ p, Q* __restrict__ q,
                                                                 const double* __restrict__ b,
                                                                 double* __restrict__ part, Dev dv, int coef_slot,
                                                                 const int* __restrict__ gate)
{
    __shared__ double smem[64];
    if (gated(gate)) return;
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    const double coef = MODE == 1 ? dv.scal[coef_slot] : 0.0;
    Comp mine;
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows;
         r += warps) {
        const uint32_t* row = idx + r * k;
        double acc = 0;
        for (int j = lane; j < k; j += 32) acc += static_cast<double>(__ldg(p + __ldg(row + j)));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            if (MODE == 1) acc -= coef * static_cast<double>(q[r]);
            if (MODE == 2) acc = (b ? b[r] : 0.0) - acc;
            q[r] = static_cast<Q>(acc);
            const double qq = static_cast<double>(static_cast<Q>(acc));
            acc_add<COMP>(mine, qq * qq);
        }
    }
    write_partial<COMP>(part, mine, smem);
}

// Partial sums of A' q per work unit (deterministic, FP64 accumulation).
template <typename Q>
__global__ void __launch_bounds__(kVecThreads) spmv_t_units_flag_kernel(CsrView a, const Q* __restrict__ q,
                                                                        double* __restrict__ partial,
                                                                        const int* __restrict__ gate)
{
    if (gated(gate)) return;
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t u = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); u < a.units;
         u += warps) {
        const int32_t c = a.unit_col[u];
        const int64_t begin = a.col_ptr[c] + static_cast<int64_t>(u - a.unit_ptr[c]) * kUnit;
        const int64_t end = min(a.col_ptr[c + 1], begin + kUnit);
        double acc = 0;
        for (int64_t e = begin + lane; e < end; e += 32) acc += static_cast<double>(__ldg(q + __ldg(a.row_idx + e)));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) partial[u] = acc;
    }
}

__device__ __forceinline__ double unit_sum(const CsrView& a, const double* partial, int64_t c)
{
    double acc = 0;
    for (uint32_t u = a.unit_ptr[c]; u < a.unit_ptr[c + 1]; u++) acc += partial[u];
    return acc;
}

// Column c of the last A'q product, whichever layout computed it:
// kind 0 sums the rows layout's work-unit partials, kind 1/2 the blocked
// layout's FP32/FP64 item partials; kind -1 means "no product" (0).
struct ColSum {
    int kind = -1;
    CsrView a;
    const double* unit_partial = nullptr;
    FastCols fc;
    const float* p32 = nullptr;
    const double* p64 = nullptr;
    __device__ __forceinline__ double operator()(int64_t c) const
    {
        if (kind == 1) return fast_col_sum<float>(fc, p32, c);
        if (kind == 2) return fast_col_sum<double>(fc, p64, c);
        if (kind == 0) return unit_sum(a, unit_partial, c);
        return 0.0;
    }
};

// ---------------------------------------------------------------------------
// PCG vector steps.
// ---------------------------------------------------------------------------

// alpha = rz / pAp (single block).  Breakdown when pAp is not finite.
template <bool COMP>
__global__ void __launch_bounds__(kRedThreads) pcg_alpha_kernel(const double* __restrict__ part, int n, Dev dv)
{
    __shared__ double smem[64];
    if (finished(dv.flags)) return;
    const double pap = reduce_partials<COMP>(part, n, smem);
    if (threadIdx.x == 0) {
        const double rz = dv.scal[kRz];
        dv.scal[kPap] = pap;
        if (!isfinite(pap)) {
            dv.scal[kAlpha] = 0;
            dv.flags[kStatus] = CAS_ERR_BREAKDOWN;
            dv.flags[kDone] = 1;
            dv.flags[kSkip] = 1;
        } else if (!(pap > 0)) {
            // p has no component outside the null space of A: the normal
            // equations are solved as far as the products resolve them (a
            // rank-deficient A, or the residual at rounding level).  Stop;
            // the FP64 true residual decides between converged and a
            // restart from it.
            dv.scal[kAlpha] = 0;
            dv.flags[kDone] = 1;
            dv.flags[kSkip] = 1;
        } else {
            dv.scal[kAlpha] = rz / pap;
        }
    }
}

// s = A'A p (from unit partials); x += alpha p; r -= alpha s; z = d r;
// partials of r.z and r.r.
template <bool COMP>
__global__ void __launch_bounds__(kVecThreads) pcg_update_kernel(ColSum cs,
                                                                 double* __restrict__ x, double* __restrict__ r,
                                                                 double* __restrict__ z, const double* __restrict__ p,
                                                                 const double* __restrict__ d,
                                                                 double* __restrict__ part_rz,
                                                                 double* __restrict__ part_rr, Dev dv)
{
    __shared__ double smem[64];
    if (finished(dv.flags)) return;
    const double alpha = dv.scal[kAlpha];
    Comp rz, rr;
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cs.a.cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double s = cs(c);
        x[c] += alpha * p[c];
        const double rc = r[c] - alpha * s;
        const double zc = d[c] * rc;
        r[c] = rc;
        z[c] = zc;
        acc_add<COMP>(rz, rc * zc);
        acc_add<COMP>(rr, rc * rc);
    }
    write_partial<COMP>(part_rz, rz, smem);
    write_partial<COMP>(part_rr, rr, smem);
}

// rz_new, rr -> beta, residual, convergence (single block).
// replace != 0: residual-replacement step; r.z is replaced but beta and the
// iteration count are left alone.
// part_dev (replacement only, may be null): partials of ||r_rec - r_true||^2;
// sets kRestart when the deviation exceeds kRestartDeviation.
// plan_refine > 0 (mixed PCG, not a replacement): the tolerance test moves to
// the replacement step, which this kernel schedules through kSkip (drop by
// kReplaceDrop, plan_refine iterations, or tolerance met).
template <bool COMP>
__global__ void __launch_bounds__(kRedThreads) pcg_beta_kernel(const double* __restrict__ part_rz,
                                                               const double* __restrict__ part_rr, int n, Dev dv,
                                                               int replace, const int* __restrict__ gate,
                                                               const double* __restrict__ part_dev, int plan_refine)
{
    __shared__ double smem[64];
    if (gated(gate)) return;
    const double rz_new = reduce_partials<COMP>(part_rz, n, smem);
    const double rr = reduce_partials<COMP>(part_rr, n, smem);
    const double dev2 = part_dev ? reduce_partials<COMP>(part_dev, n, smem) : 0.0;
    if (threadIdx.x == 0) {
        if (part_dev) dv.flags[kRestart] = dev2 > kRestartDeviation * kRestartDeviation * rr ? 1 : 0;
        const double rz = dv.scal[kRz];
        const double bn2 = dv.scal[kBn2];
        const double res = bn2 > 0 ? sqrt(rr / bn2) : sqrt(rr);
        if (!replace) {
            dv.scal[kBeta] = rz != 0 ? rz_new / rz : 0.0;
            dv.flags[kIter] += 1;
        } else {
            dv.flags[kRefine] += 1;
        }
        dv.scal[kRz] = rz_new;
        dv.scal[kRr] = rr;
        dv.scal[kRes] = res;
        const bool met = dv.scal[kTol] > 0 && res <= dv.scal[kTol];
        if (replace) {
            dv.scal[kRrRef] = rr;
            dv.flags[kIterRef] = dv.flags[kIter];
        }
        if (!isfinite(rz_new) || !isfinite(rr)) {
            dv.flags[kStatus] = CAS_ERR_BREAKDOWN;
            dv.flags[kDone] = 1;
            dv.flags[kSkip] = 1;
        } else if (!replace && plan_refine > 0) {
            dv.flags[kRestart] = 0;
            const bool due = met || rr <= kReplaceDrop * kReplaceDrop * dv.scal[kRrRef] ||
                             dv.flags[kIter] - dv.flags[kIterRef] >= plan_refine;
            dv.flags[kSkip] = due ? 0 : 1;
        } else if (met) {
            dv.flags[kDone] = 1;
            dv.flags[kSkip] = 1;
            if (replace) dv.flags[kVerified] = 1;
        }
    }
}

// p = z + beta p (and the FP32 gather copy).
template <typename T>
__global__ void __launch_bounds__(kVecThreads) pcg_direction_kernel(int64_t n, const double* __restrict__ z,
                                                                    double* __restrict__ p, T* __restrict__ pg,
                                                                    Dev dv)
{
    if (finished(dv.flags)) return;
    const double beta = dv.scal[kBeta];
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double v = z[c] + beta * p[c];
        p[c] = v;
        if (pg) pg[c] = static_cast<T>(v);
    }
}

// p = z (and the gather copy) when the last replacement set kRestart.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) pcg_restart_kernel(int64_t n, const double* __restrict__ z,
                                                                  double* __restrict__ p, T* __restrict__ pg, Dev dv)
{
    if (finished(dv.flags) || !*(volatile const int*)(dv.flags + kRestart)) return;
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        p[c] = z[c];
        if (pg) pg[c] = static_cast<T>(z[c]);
    }
}

// r = A'(b - A x) from unit partials; z = d r; partials of r.z and r.r, and
// (part_dev not null) of ||r_old - r||^2 against the recursive residual it
// replaces.  Also initialises p = z (init != 0) and ||A'b||^2 (bn != 0,
// x = 0).
template <bool COMP, typename T>
__global__ void __launch_bounds__(kVecThreads) pcg_residual_kernel(ColSum cs,
                                                                   double* __restrict__ r, double* __restrict__ z,
                                                                   double* __restrict__ p, T* __restrict__ pg,
                                                                   const double* __restrict__ d,
                                                                   double* __restrict__ part_rz,
                                                                   double* __restrict__ part_rr, int init, Dev dv,
                                                                   const int* __restrict__ gate,
                                                                   const double* __restrict__ bn,
                                                                   double* __restrict__ part_dev)
{
    __shared__ double smem[64];
    if (gated(gate)) return;
    Comp rz, rr, dev;
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cs.a.cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double rc = (bn ? bn[c] : 0.0) + cs(c);
        const double zc = d[c] * rc;
        if (part_dev) {
            const double dd = r[c] - rc;
            acc_add<COMP>(dev, dd * dd);
        }
        r[c] = rc;
        z[c] = zc;
        if (init) {
            p[c] = zc;
            if (pg) pg[c] = static_cast<T>(zc);
        }
        acc_add<COMP>(rz, rc * zc);
        acc_add<COMP>(rr, rc * rc);
    }
    write_partial<COMP>(part_rz, rz, smem);
    write_partial<COMP>(part_rr, rr, smem);
    if (part_dev) write_partial<COMP>(part_dev, dev, smem);
}

// DiagonalPreconditioner (Math/Solver.h:25-38): d = 1/diag(A'A), entries that
// are not normal (inf from an empty column) become 1.  mode 0: d = 1;
// mode 2: the LSQR/LSMR column scale d = diag(A'A)^-1/2, 1 for an empty
// column.
__global__ void precond_kernel(const uint64_t* __restrict__ diag, int64_t n, int mode, double* __restrict__ d)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double v = 1.0;
        if (mode) {
            const double dg = static_cast<double>(diag[c]);
            v = 1.0 / (mode == 2 ? sqrt(dg) : dg);
            if (!(isfinite(v) && fabs(v) >= 2.2250738585072014e-308)) v = 1.0;  // not std::isnormal
        }
        d[c] = v;
    }
}

// A caller's DiagonalPreconditioner (Math/Solver.h:25-38): d = the given
// entries, those that are not normal replaced by 1.
// out = in rounded to FP32 (the gather copy of a rows-length vector).
__global__ void to_f32_kernel(const double* __restrict__ in, int64_t n, float* __restrict__ out)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[i] = static_cast<float>(in[i]);
}

__global__ void user_precond_kernel(const double* __restrict__ in, int64_t n, double* __restrict__ d)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double v = in[c];
        d[c] = (isfinite(v) && fabs(v) >= 2.2250738585072014e-308) ? v : 1.0;
    }
}

template <typename T>
__global__ void cast_kernel(int64_t n, const double* __restrict__ in, T* __restrict__ out)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[c] = static_cast<T>(in[c]);
}

// ||v||^2 partials of v = bn + (A' q from unit partials); partial may be
// null (v = bn), bn may be null (v = A' q).  Used for ||A'b||^2 and ||A'r||^2.
// sc (may be null) scales v column by column first (||S A'b||^2).
template <bool COMP>
__global__ void __launch_bounds__(kVecThreads) norm_units_kernel(ColSum cs,
                                                                 double* __restrict__ out, double* __restrict__ part,
                                                                 const double* __restrict__ bn,
                                                                 const double* __restrict__ sc = nullptr)
{
    __shared__ double smem[64];
    Comp acc;
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cs.a.cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double v = ((bn ? bn[c] : 0.0) + cs(c)) * (sc ? sc[c] : 1.0);
        if (out) out[c] = v;
        acc_add<COMP>(acc, v * v);
    }
    write_partial<COMP>(part, acc, smem);
}

template <bool COMP>
__global__ void __launch_bounds__(kRedThreads) store_sum_kernel(const double* __restrict__ part, int n,
                                                                double* __restrict__ dst)
{
    __shared__ double smem[64];
    const double v = reduce_partials<COMP>(part, n, smem);
    if (threadIdx.x == 0) *dst = v;
}

// ---------------------------------------------------------------------------
// LSQR steps (Math/Solver.h:139-177) with deferred normalisation: u and v
// are stored unnormalised (u_hat, v_hat) next to their scale 1/beta, 1/alpha
// held as device scalars, so no separate scaling pass is needed.
// ---------------------------------------------------------------------------

// Column scale of an LSQR/LSMR solve on A S (null: unscaled).
__device__ __forceinline__ double col_scale(const double* sc, int64_t c) { return sc ? sc[c] : 1.0; }

// The kernels of an LSQR/LSMR step return at entry once the solver is done
// (init 0 and 2) and, for the restart step, while *gate is set; init 1 is
// the set-up and always runs.
__device__ __forceinline__ bool lsqr_skip(const Dev& dv, int init, const int* gate)
{
    return (init != 1 && finished(dv.flags)) || gated(gate);
}

// v_hat = (1/beta) S A' u_hat - beta v  (v = v_hat_prev / alpha_prev);
// partial ||v_hat||^2.  init: v_hat = (1/beta) S A' u_hat.
template <bool COMP, typename T>
__global__ void __launch_bounds__(kVecThreads) lsqr_v_kernel(ColSum cs,
                                                             double* __restrict__ v, double* __restrict__ part,
                                                             Dev dv, int init, const int* __restrict__ gate,
                                                             const double* __restrict__ sc)
{
    __shared__ double smem[64];
    if (lsqr_skip(dv, init, gate)) return;
    const double inv_beta = dv.scal[kInvBeta];
    const double beta = dv.scal[kLBeta];
    const double inv_alpha_prev = dv.scal[kLAlpha] != 0 ? 1.0 / dv.scal[kLAlpha] : 0.0;
    Comp acc;
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cs.a.cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double val = inv_beta * col_scale(sc, c) * cs(c);
        if (!init) val -= beta * (v[c] * inv_alpha_prev);
        v[c] = val;
        acc_add<COMP>(acc, val * val);
    }
    write_partial<COMP>(part, acc, smem);
}

// beta = ||u_hat|| (u_hat = A S v - alpha u, alpha u = alpha/beta_prev u_hat_prev
// folded into the SpMV's coefficient slot).  Single block.
template <bool COMP>
__global__ void __launch_bounds__(kRedThreads) lsqr_beta_kernel(const double* __restrict__ part, int n, Dev dv,
                                                                int init, const int* __restrict__ gate)
{
    __shared__ double smem[64];
    if (lsqr_skip(dv, init, gate)) return;
    const double s = reduce_partials<COMP>(part, n, smem);
    if (threadIdx.x == 0) {
        const double beta = sqrt(s);
        dv.scal[kLBeta] = beta;
        dv.scal[kInvBeta] = beta > 0 ? 1.0 / beta : 0.0;
        if (init) dv.scal[kPhiBar] = beta;  // phi_bar = beta (Math/Solver.h:149)
        if (init == 2) dv.flags[kRefine] += 1;  // restart from the true residual
    }
}

// Relative recursive residual of an LSQR/LSMR step (against ||S A'b|| when
// the columns are scaled, the norm the recursion estimates), the tolerance
// test and, with plan (mixed solves), the restart test: a restart is
// scheduled (kSkip cleared) when the estimate has dropped by
// kLsqrRestartDrop since the last (re)start and the tolerance is not met.
__device__ __forceinline__ void lsqr_step_tests(Dev dv, double arn, int plan, bool scaled)
{
    dv.scal[kArNorm] = arn;
    dv.flags[kIter] += 1;
    const double bn2 = dv.scal[scaled ? kBn2S : kBn2];
    const double res = bn2 > 0 ? arn / sqrt(bn2) : arn;
    dv.scal[kRes] = res;
    const bool met = dv.scal[kTol] > 0 && res <= dv.scal[kTol];
    if (met) dv.flags[kPending] = 1;
    if (plan && !met && arn <= kLsqrRestartDrop * dv.scal[kArn0]) dv.flags[kSkip] = 0;
}

// alpha = ||v_hat||; Givens step; scalars for the x/w update.  Single block.
template <bool COMP>
__global__ void __launch_bounds__(kRedThreads) lsqr_alpha_kernel(const double* __restrict__ part, int n, Dev dv,
                                                                 int init, const int* __restrict__ gate, int plan,
                                                                 int scaled)
{
    __shared__ double smem[64];
    if (lsqr_skip(dv, init, gate)) return;
    const double s = reduce_partials<COMP>(part, n, smem);
    if (threadIdx.x == 0) {
        const double alpha = sqrt(s);
        if (init) {
            dv.scal[kLAlpha] = alpha;
            dv.scal[kRhoBar] = alpha;  // rho_bar = alpha (Math/Solver.h:150)
            dv.scal[kArNorm] = alpha * dv.scal[kLBeta];
            dv.scal[kArn0] = alpha * dv.scal[kLBeta];
            return;
        }
        const double beta = dv.scal[kLBeta];
        const double rho_bar = dv.scal[kRhoBar], phi_bar = dv.scal[kPhiBar];
        const double rho = sqrt(rho_bar * rho_bar + beta * beta);
        if (!(rho > 0) || !isfinite(rho)) {
            dv.scal[kPhiRho] = 0;
            dv.scal[kThetaRho] = 0;
            dv.flags[kDone] = 1;
            if (!isfinite(rho)) dv.flags[kStatus] = CAS_ERR_BREAKDOWN;
            return;
        }
        const double c = rho_bar / rho, sn = beta / rho;
        const double theta = sn * alpha;
        const double phi = c * phi_bar;
        dv.scal[kRhoBar] = -c * alpha;
        dv.scal[kPhiBar] = sn * phi_bar;
        dv.scal[kPhiRho] = phi / rho;
        dv.scal[kThetaRho] = theta / rho;
        dv.scal[kLAlpha] = alpha;
        // ||A'r_k|| = phi_bar_{k+1} * alpha_{k+1} * |c_k| (Paige & Saunders 1982)
        lsqr_step_tests(dv, fabs(sn * phi_bar * alpha * c), plan, scaled != 0);
    }
}

// x += (phi/rho) S w; w = v - (theta/rho) w; gather copy vg = S v (v
// normalised).
template <typename T>
__global__ void __launch_bounds__(kVecThreads) lsqr_xw_kernel(int64_t n, double* __restrict__ x,
                                                              double* __restrict__ w, const double* __restrict__ v,
                                                              T* __restrict__ vg, Dev dv, int init,
                                                              const int* __restrict__ gate,
                                                              const double* __restrict__ sc)
{
    if (lsqr_skip(dv, init, gate)) return;
    const double inv_alpha = dv.scal[kLAlpha] != 0 ? 1.0 / dv.scal[kLAlpha] : 0.0;
    const double phi_rho = dv.scal[kPhiRho], theta_rho = dv.scal[kThetaRho];
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double vn = v[c] * inv_alpha;
        const double scale = col_scale(sc, c);
        if (init) {
            w[c] = vn;
        } else {
            x[c] += phi_rho * scale * w[c];
            w[c] = vn - theta_rho * w[c];
        }
        vg[c] = static_cast<T>(scale * vn);
    }
}

// u_hat in FP32 after a restart of the mixed solver computed it in FP64.
__global__ void __launch_bounds__(kVecThreads) lsqr_round_u_kernel(int64_t n, const double* __restrict__ u,
                                                                   float* __restrict__ uf, Dev dv,
                                                                   const int* __restrict__ gate)
{
    if (finished(dv.flags) || gated(gate)) return;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        uf[i] = static_cast<float>(u[i]);
}

// ---------------------------------------------------------------------------
// LSMR steps (Math/Solver.h:222-287): the same bidiagonalisation as LSQR
// (u_hat, v_hat with deferred normalisation), then three Givens rotations
// on scalars and the h_bar, x, h updates.
// ---------------------------------------------------------------------------

// signum and GivensRotation (Math/Solver.h:184-220, the sym_ortho form of
// scipy's lsqr.py): c, s, r with the signs of the reference.
__device__ __forceinline__ double signum(double v) { return v < 0 ? -1.0 : (v > 0 ? 1.0 : 0.0); }
__device__ __forceinline__ void givens(double a, double b, double& c, double& s, double& r)
{
    if (b == 0) {
        c = signum(a);
        s = 0;
        r = fabs(a);
    } else if (a == 0) {
        c = 0;
        s = signum(b);
        r = fabs(b);
    } else if (fabs(b) > fabs(a)) {
        const double tau = a / b;
        s = signum(b) / sqrt(1 + tau * tau);
        c = s * tau;
        r = b / s;
    } else {
        const double tau = b / a;
        c = signum(a) / sqrt(1 + tau * tau);
        s = c * tau;
        r = a / c;
    }
}

// alpha = ||v_hat||, then the rotations of one LSMR step and the update
// coefficients; |zeta_bar| estimates ||A'r|| (the stopping test's
// recursive residual).  init: the constructor's scalars (:236-251).  A
// zero rho or rho_bar means the bidiagonalisation ended (the solution is
// exact): the solver stops.  Single block.
template <bool COMP>
__global__ void __launch_bounds__(kRedThreads) lsmr_alpha_kernel(const double* __restrict__ part, int n, Dev dv,
                                                                 int init, const int* __restrict__ gate, int plan,
                                                                 int scaled)
{
    __shared__ double smem[64];
    if (lsqr_skip(dv, init, gate)) return;
    const double sum = reduce_partials<COMP>(part, n, smem);
    if (threadIdx.x != 0) return;
    const double alpha = sqrt(sum);
    double* sc = dv.scal;
    const double beta = sc[kLBeta];
    if (init) {
        sc[kLAlpha] = alpha;
        sc[kMAlphaBar] = alpha;
        sc[kZetaBar] = alpha * beta;
        sc[kMRho] = 1;
        sc[kMRhoBar] = 1;
        sc[kCBar] = 1;
        sc[kSBar] = 0;
        sc[kArNorm] = alpha * beta;
        sc[kArn0] = alpha * beta;
        return;
    }
    const double rho_old = sc[kMRho], rho_bar_old = sc[kMRhoBar];
    double c_hat, s_hat, alpha_hat;
    givens(sc[kMAlphaBar], 0.0, c_hat, s_hat, alpha_hat);
    double c, s, rho;
    givens(alpha_hat, beta, c, s, rho);
    const double theta_new = s * alpha;
    const double theta_bar = sc[kSBar] * rho;
    double c_bar, s_bar, rho_bar;
    givens(sc[kCBar] * rho, theta_new, c_bar, s_bar, rho_bar);
    const double zeta = c_bar * sc[kZetaBar];
    const double zeta_bar = -s_bar * sc[kZetaBar];
    if (!(rho != 0 && rho_bar != 0 && rho_old != 0 && rho_bar_old != 0) || !isfinite(rho) || !isfinite(rho_bar)) {
        sc[kFHbar] = sc[kFX] = sc[kFH] = 0;
        dv.flags[kDone] = 1;
        if (!isfinite(rho) || !isfinite(rho_bar)) dv.flags[kStatus] = CAS_ERR_BREAKDOWN;
        return;
    }
    sc[kMAlphaBar] = c * alpha;
    sc[kMRho] = rho;
    sc[kMRhoBar] = rho_bar;
    sc[kCBar] = c_bar;
    sc[kSBar] = s_bar;
    sc[kZetaBar] = zeta_bar;
    sc[kFHbar] = theta_bar * rho / rho_old / rho_bar_old;
    sc[kFX] = zeta / rho / rho_bar;
    sc[kFH] = theta_new / rho;
    sc[kLAlpha] = alpha;
    lsqr_step_tests(dv, fabs(zeta_bar), plan, scaled != 0);
}

// h_bar = h - f_hbar h_bar; x += f_x S h_bar; h = v - f_h h (v normalised);
// gather copy vg = S v.  init: h = v, h_bar = 0.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) lsmr_update_kernel(int64_t n, double* __restrict__ x,
                                                                  double* __restrict__ h, double* __restrict__ hbar,
                                                                  const double* __restrict__ v, T* __restrict__ vg,
                                                                  Dev dv, int init, const int* __restrict__ gate,
                                                                  const double* __restrict__ sc)
{
    if (lsqr_skip(dv, init, gate)) return;
    const double inv_alpha = dv.scal[kLAlpha] != 0 ? 1.0 / dv.scal[kLAlpha] : 0.0;
    const double f_hbar = dv.scal[kFHbar], f_x = dv.scal[kFX], f_h = dv.scal[kFH];
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < n;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const double vn = v[c] * inv_alpha;
        const double scale = col_scale(sc, c);
        if (init) {
            h[c] = vn;
            hbar[c] = 0;
        } else {
            const double hb = h[c] - f_hbar * hbar[c];
            hbar[c] = hb;
            x[c] += f_x * scale * hb;
            h[c] = vn - f_h * h[c];
        }
        vg[c] = static_cast<T>(scale * vn);
    }
}

// coefficient of the u recursion: alpha / beta_prev (u_hat holds beta_prev u).
// First kernel of an LSQR step: a tolerance met by the previous step stops
// the solver here, after that step's x/w update has run.  It also closes
// the gate of the step's restart, which the step's alpha kernel may open.
__global__ void lsqr_coef_kernel(Dev dv, int slot)
{
    dv.flags[kSkip] = 1;
    if (finished(dv.flags)) return;
    if (dv.flags[kPending]) {
        dv.flags[kDone] = 1;
        return;
    }
    dv.scal[slot] = dv.scal[kLAlpha] * dv.scal[kInvBeta];
}

unsigned vec_grid(int64_t n)
{
    const int64_t want = (n + kVecThreads - 1) / kVecThreads;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(want, static_cast<int64_t>(sm_count()) * 4)));
}
unsigned row_grid(int64_t rows)
{
    const int64_t want = (rows + 7) / 8;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(want, static_cast<int64_t>(sm_count()) * 16)));
}

}  // namespace

// ---------------------------------------------------------------------------
// Solver object.
// ---------------------------------------------------------------------------
struct SolverImpl {
    const cas_csr* A = nullptr;
    CsrView a;
    const FastLayout* fast = nullptr;
    cas_solve_opts o{};
    // LSQR and LSMR: the bidiagonalisation methods on min ||Ax - b||
    bool least_squares() const { return o.method == CAS_LSQR || o.method == CAS_LSMR; }
    // LSQR/LSMR on A S, S = diag(A'A)^-1/2 held in d
    bool scaled() const { return least_squares() && o.scale_columns != 0; }
    const double* col_scale() const { return scaled() ? d : nullptr; }
    cudaStream_t s = nullptr;
    int device = 0;
    bool mixed = false;
    bool fast32 = false;  // FP32 products on the blocked layout
    bool fast64 = false;  // FP64 products on the blocked layout
    int64_t C = 0, R = 0;
    // C-length FP64 vectors
    double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *d = nullptr, *w = nullptr, *v = nullptr;
    float* pg32 = nullptr;   // FP32 gather copy (mixed)
    // R-length
    void* q = nullptr;        // A p: float (mixed) or double (plain)
    double* q64 = nullptr;    // FP64 residual b - A x (refinement / true residual)
    const double* b = nullptr;   // rows-length targets (null with a normal RHS)
    const double* bn = nullptr;  // cols-length normal-equation RHS A'b (PCG/CG only)
    const double* user_d = nullptr;  // a caller's diagonal preconditioner (PCG only; read at set-up)
    double* b_own = nullptr;
    double* partial = nullptr;  // unit partials of the rows layout
    double *part_q = nullptr, *part_a = nullptr, *part_b = nullptr, *part_c = nullptr;
    int n_row_blocks = 0, n_vec_blocks = 0, n_q_parts = 0;
    double* scal = nullptr;
    int* flags = nullptr;
    double* host_scal = nullptr;  // pinned mirror
    int* host_flags = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_len = 0;
    long long graph_kernels = 0;
    int launched = 0;  // iterations issued (including no-op tail)
    bool own_stream = false;  // graphs cannot be captured on the legacy default stream
    Dev dv() const { return Dev{scal, flags}; }

    ~SolverImpl()
    {
        if (graph) cudaGraphExecDestroy(graph);
        if (own_stream) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
        for (void* ptr : {(void*)x, (void*)r, (void*)z, (void*)p, (void*)d, (void*)w, (void*)v, (void*)pg32, q,
                          (void*)q64, (void*)b_own, (void*)partial, (void*)part_q, (void*)part_a, (void*)part_b, (void*)part_c,
                          (void*)scal, (void*)flags})
            dfree(ptr);
        hfree(host_scal);
        hfree(host_flags);
    }

    // Column sums of the last A'q of precision T.
    template <typename T>
    ColSum colsum() const
    {
        ColSum cs;
        cs.a = a;
        const bool use_fast = sizeof(T) == 4 ? fast32 : fast64;
        if (use_fast) {
            cs.kind = sizeof(T) == 4 ? 1 : 2;
            cs.fc = fast_cols<T>(*fast);
            cs.p32 = static_cast<const float*>(fast->t32.partial);
            cs.p64 = static_cast<const double*>(fast->t64.partial);
        } else {
            cs.kind = 0;
            cs.unit_partial = partial;
        }
        return cs;
    }

    // Device flag words that let graph-captured kernels return at entry:
    // done() once the solver has converged, skip() while no residual
    // replacement is due.
    const int* done() const { return flags + kDone; }
    const int* skip() const { return flags + kSkip; }

    // q = A g (mode 0), A g - scal[coef_slot] q (1), rhs - A g (2), with
    // partials of ||q||^2 in part_q (count in n_q_parts).  The kernels
    // return at entry while *gate != 0 (gate may be null).
    template <bool COMP, typename G, typename Q>
    cas_status product(const G* g, Q* qq, int mode, const double* rhs, int coef_slot, const int* gate)
    {
        const bool use_fast = sizeof(G) == 4 ? fast32 : fast64;
        if (use_fast) {
            return fast_spmv<G, Q>(*fast, g, qq, rhs, scal + coef_slot, part_q, const_cast<int*>(gate), mode, s,
                                   &n_q_parts);
        }
        n_q_parts = n_row_blocks;
        const Dev D = dv();
        if (mode == 0)
            { spmv_norm_kernel<G, Q, COMP, 0><<<n_row_blocks, kVecThreads, 0, s>>>(a.idx, R, a.k, g, qq, rhs, part_q, D,
                                                                               coef_slot, gate); cas::count_launch(); }
        else if (mode == 1)
            { spmv_norm_kernel<G, Q, COMP, 1><<<n_row_blocks, kVecThreads, 0, s>>>(a.idx, R, a.k, g, qq, rhs, part_q, D,
                                                                               coef_slot, gate); cas::count_launch(); }
        else
            { spmv_norm_kernel<G, Q, COMP, 2><<<n_row_blocks, kVecThreads, 0, s>>>(a.idx, R, a.k, g, qq, rhs, part_q, D,
                                                                               coef_slot, gate); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }

    // Partials of A' q (summed later through colsum<Q>()).
    template <typename Q>
    cas_status product_t(const Q* qq, const int* gate)
    {
        const bool use_fast = sizeof(Q) == 4 ? fast32 : fast64;
        if (use_fast) return fast_spmv_t_partials<Q>(*fast, qq, const_cast<int*>(gate), s);
        { spmv_t_units_flag_kernel<Q><<<row_grid(a.units), kVecThreads, 0, s>>>(a, qq, partial, gate); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }

    template <bool COMP, typename T>
    cas_status issue_pcg_iteration()
    {
        const Dev D = dv();
        const T* pgather = std::is_same<T, float>::value ? reinterpret_cast<const T*>(pg32) : reinterpret_cast<const T*>(p);
        CAS_TRY((product<COMP, T, T>(pgather, static_cast<T*>(q), 0, nullptr, 0, done())));
        CAS_TRY(product_t<T>(static_cast<const T*>(q), done()));
        { pcg_alpha_kernel<COMP><<<1, kRedThreads, 0, s>>>(part_q, n_q_parts, D); cas::count_launch(); }
        { pcg_update_kernel<COMP><<<n_vec_blocks, kVecThreads, 0, s>>>(colsum<T>(), x, r, z, p, d, part_a, part_b, D); cas::count_launch(); }
        { pcg_beta_kernel<COMP><<<1, kRedThreads, 0, s>>>(part_a, part_b, n_vec_blocks, D, 0, done(), nullptr,
                                                          mixed ? std::max(o.refine_every, 1) : 0); cas::count_launch(); }
        { pcg_direction_kernel<T><<<n_vec_blocks, kVecThreads, 0, s>>>(
            C, z, p, std::is_same<T, float>::value ? reinterpret_cast<T*>(pg32) : nullptr, D); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }

    // Residual replacement: r = A'(b - A x) (or b' - A'A x) in FP64, z = d r,
    // r.z, r.r.  restart: also p = z (set-up, resumption after a failed
    // verification).  Otherwise this is the in-graph step of the mixed PCG:
    // gated by kSkip, it measures the recursive residual's drift, restarts
    // the direction when the drift exceeds kRestartDeviation and declares
    // convergence on the true residual.
    template <bool COMP>
    // reuse_atb: x is zero and the partials of the last transposed product
    // are those of A'b (the set-up's), so A'(b - A x) = A'b is read from them
    // instead of recomputed; FP32 ones when atb32 (the mixed set-up).
    cas_status issue_pcg_refine(bool restart, bool reuse_atb = false, bool atb32 = false)
    {
        const Dev D = dv();
        const int* gate = restart ? nullptr : skip();
        if (!reuse_atb) {
            CAS_TRY((product<COMP, double, double>(x, q64, 2, b, 0, gate)));
            CAS_TRY(product_t<double>(q64, gate));
        }
        double* pdev = restart ? nullptr : part_c;
        if (mixed)
            { pcg_residual_kernel<COMP, float><<<n_vec_blocks, kVecThreads, 0, s>>>(
                  atb32 ? colsum<float>() : colsum<double>(), r, z, p, pg32, d,
                                                                                part_a, part_b, restart ? 1 : 0, D,
                                                                                gate, bn, pdev); cas::count_launch(); }
        else
            { pcg_residual_kernel<COMP, double><<<n_vec_blocks, kVecThreads, 0, s>>>(colsum<double>(), r, z, p, nullptr, d,
                                                                                 part_a, part_b, restart ? 1 : 0, D,
                                                                                 gate, bn, pdev); cas::count_launch(); }
        { pcg_beta_kernel<COMP><<<1, kRedThreads, 0, s>>>(part_a, part_b, n_vec_blocks, D, 1, gate, pdev, 0); cas::count_launch(); }
        if (!restart) {
            if (mixed)
                { pcg_restart_kernel<float><<<n_vec_blocks, kVecThreads, 0, s>>>(C, z, p, pg32, D); cas::count_launch(); }
            else
                { pcg_restart_kernel<double><<<n_vec_blocks, kVecThreads, 0, s>>>(C, z, p, nullptr, D); cas::count_launch(); }
        }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }

    template <bool COMP, typename T>
    cas_status issue_lsqr_iteration()
    {
        const Dev D = dv();
        T* vg = reinterpret_cast<T*>(std::is_same<T, float>::value ? (void*)pg32 : (void*)p);
        const double* sc = col_scale();
        const int plan = mixed ? 1 : 0;
        const int sd = scaled() ? 1 : 0;
        // u_hat = A S v - (alpha / beta_prev) u_hat_prev
        { lsqr_coef_kernel<<<1, 1, 0, s>>>(D, kPap); cas::count_launch(); }
        CAS_TRY((product<COMP, T, T>(vg, static_cast<T*>(q), 1, nullptr, kPap, done())));
        { lsqr_beta_kernel<COMP><<<1, kRedThreads, 0, s>>>(part_q, n_q_parts, D, 0, nullptr); cas::count_launch(); }
        // v_hat = (1/beta) S A' u_hat - beta v
        CAS_TRY(product_t<T>(static_cast<const T*>(q), done()));
        { lsqr_v_kernel<COMP, T><<<n_vec_blocks, kVecThreads, 0, s>>>(colsum<T>(), v, part_a, D, 0, nullptr, sc); cas::count_launch(); }
        if (o.method == CAS_LSMR) {
            // LSMR: h in w, h_bar in z
            { lsmr_alpha_kernel<COMP><<<1, kRedThreads, 0, s>>>(part_a, n_vec_blocks, D, 0, nullptr, plan, sd); cas::count_launch(); }
            { lsmr_update_kernel<T><<<n_vec_blocks, kVecThreads, 0, s>>>(C, x, w, z, v, vg, D, 0, nullptr, sc); cas::count_launch(); }
        } else {
            { lsqr_alpha_kernel<COMP><<<1, kRedThreads, 0, s>>>(part_a, n_vec_blocks, D, 0, nullptr, plan, sd); cas::count_launch(); }
            { lsqr_xw_kernel<T><<<n_vec_blocks, kVecThreads, 0, s>>>(C, x, w, v, vg, D, 0, nullptr, sc); cas::count_launch(); }
        }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }

    // LSQR/LSMR (re)start from the current x (Math/Solver.h:139-151 with
    // b - A x for b): beta u = b - A x ; alpha v = S A'u ; w = v ; phi_bar =
    // beta ; rho_bar = alpha.  mode 1 = set-up, 2 = the restart step of a
    // mixed iteration inside a graph chunk (runs only when the step's alpha
    // kernel opened the kSkip gate), 3 = a restart issued by the host.
    // The mixed solver computes u and S A'u in FP64 (u is the least-squares
    // residual, large next to A'u once the solve has progressed, so FP32
    // would bury A'u under its own rounding) and keeps an FP32 copy of u_hat
    // for the following steps: a restart is one outer refinement step on the
    // least-squares correction.
    cas_status issue_lsqr_start(int mode) { return mixed ? issue_lsqr_start_t<true>(mode) : issue_lsqr_start_t<false>(mode); }

    template <bool COMP>
    cas_status issue_lsqr_start_t(int mode)
    {
        const Dev D = dv();
        const int* gate = mode == 2 ? skip() : nullptr;
        const int init = mode == 1 ? 1 : 2;
        const double* sc = col_scale();
        const int sd = scaled() ? 1 : 0;
        CAS_TRY((product<COMP, double, double>(x, q64, 2, b, 0, gate)));
        { lsqr_beta_kernel<COMP><<<1, kRedThreads, 0, s>>>(part_q, n_q_parts, D, init, gate); cas::count_launch(); }
        CAS_TRY(product_t<double>(q64, gate));
        { lsqr_v_kernel<COMP, double><<<n_vec_blocks, kVecThreads, 0, s>>>(colsum<double>(), v, part_a, D, init, gate, sc); cas::count_launch(); }
        if (mixed) {
            { lsqr_round_u_kernel<<<row_grid(R), kVecThreads, 0, s>>>(R, q64, static_cast<float*>(q), D, gate); cas::count_launch(); }
        } else {
            CAS_CUDA(cudaMemcpyAsync(q, q64, sizeof(double) * R, cudaMemcpyDeviceToDevice, s));
        }
        if (o.method == CAS_LSMR) {
            { lsmr_alpha_kernel<COMP><<<1, kRedThreads, 0, s>>>(part_a, n_vec_blocks, D, init, gate, 0, sd); cas::count_launch(); }
            if (mixed)
                { lsmr_update_kernel<float><<<n_vec_blocks, kVecThreads, 0, s>>>(C, x, w, z, v, pg32, D, init, gate, sc); cas::count_launch(); }
            else
                { lsmr_update_kernel<double><<<n_vec_blocks, kVecThreads, 0, s>>>(C, x, w, z, v, p, D, init, gate, sc); cas::count_launch(); }
        } else {
            { lsqr_alpha_kernel<COMP><<<1, kRedThreads, 0, s>>>(part_a, n_vec_blocks, D, init, gate, 0, sd); cas::count_launch(); }
            if (mixed)
                { lsqr_xw_kernel<float><<<n_vec_blocks, kVecThreads, 0, s>>>(C, x, w, v, pg32, D, init, gate, sc); cas::count_launch(); }
            else
                { lsqr_xw_kernel<double><<<n_vec_blocks, kVecThreads, 0, s>>>(C, x, w, v, p, D, init, gate, sc); cas::count_launch(); }
        }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }

    cas_status issue_iteration(int global_index)
    {
        const bool lsqr = o.method == CAS_LSQR || o.method == CAS_LSMR;
        if (lsqr) {
            if (mixed) {
                CAS_TRY((issue_lsqr_iteration<true, float>()));
                CAS_TRY(issue_lsqr_start(2));  // runs only when the step's alpha kernel scheduled it
            } else {
                CAS_TRY((issue_lsqr_iteration<false, double>()));
            }
            return CAS_OK;
        }
        if (mixed) {
            CAS_TRY((issue_pcg_iteration<true, float>()));
            CAS_TRY(issue_pcg_refine<true>(false));  // runs only when the beta kernel scheduled it
        } else {
            CAS_TRY((issue_pcg_iteration<false, double>()));
        }
        return CAS_OK;
    }

    // Issues n iterations starting at global index `first`, through a cached
    // CUDA graph when the chunk shape allows.
    cas_status issue_chunk(int first, int n)
    {
        if (n > 1) {
            if (!graph || graph_len != n) {
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
            }
            CAS_CUDA(cudaGraphLaunch(graph, s));
            count_launch(graph_kernels);
        } else {
            for (int i = 0; i < n; i++) CAS_TRY(issue_iteration(first + i));
        }
        launched += n;
        return CAS_OK;
    }

    // The device buffers that hold an iteration's state, in checkpoint order
    // (vectors, the rows-length products LSQR/LSMR keep their u in, device
    // scalars and flags); the partial sums are scratch and not included.
    std::vector<std::pair<void*, size_t>> state_buffers() const
    {
        const size_t cb = sizeof(double) * std::max<int64_t>(C, 1), rb8 = sizeof(double) * std::max<int64_t>(R, 1);
        std::vector<std::pair<void*, size_t>> v_;
        for (double* ptr : {x, r, z, p, d, w, v}) v_.push_back({ptr, cb});
        if (mixed) v_.push_back({pg32, sizeof(float) * std::max<int64_t>(C, 1)});
        v_.push_back({q, mixed ? sizeof(float) * std::max<int64_t>(R, 1) : rb8});
        v_.push_back({q64, rb8});
        v_.push_back({scal, sizeof(double) * kSlots});
        v_.push_back({flags, sizeof(int) * kFlags});
        return v_;
    }

    cas_status read_state()
    {
        CAS_CUDA(cudaMemcpyAsync(host_scal, scal, sizeof(double) * kSlots, cudaMemcpyDeviceToHost, s));
        CAS_CUDA(cudaMemcpyAsync(host_flags, flags, sizeof(int) * kFlags, cudaMemcpyDeviceToHost, s));
        CAS_CUDA(cudaStreamSynchronize(s));
        return CAS_OK;
    }

    // ||A'(b - A x)|| / ||A'b|| in FP64 (does not touch solver state).
    cas_status true_residual(double* out)
    {
        CAS_TRY((product<true, double, double>(x, q64, 2, b, 0, nullptr)));
        CAS_TRY(product_t<double>(q64, nullptr));
        { norm_units_kernel<true><<<n_vec_blocks, kVecThreads, 0, s>>>(colsum<double>(), nullptr, part_a, bn); cas::count_launch(); }
        { store_sum_kernel<true><<<1, kRedThreads, 0, s>>>(part_a, n_vec_blocks, scal + kTrue); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        double h[kSlots];
        CAS_CUDA(cudaMemcpyAsync(h, scal, sizeof(double) * kSlots, cudaMemcpyDeviceToHost, s));
        CAS_CUDA(cudaStreamSynchronize(s));
        const double num = h[kTrue];
        const double bn2 = h[kBn2];
        *out = bn2 > 0 ? std::sqrt(num / bn2) : std::sqrt(num);
        return CAS_OK;
    }

    cas_status init(const double* x0)
    {
        C = a.cols;
        R = a.rows;
        mixed = o.precision == CAS_MIXED;
        fast = A->fast;
        const bool rows_layout = (A->layouts & CAS_LAYOUT_ROWS) != 0;
        fast32 = fast && (mixed || !rows_layout);
        fast64 = fast && (mixed || !rows_layout);
        n_row_blocks = static_cast<int>(row_grid(R));
        n_vec_blocks = static_cast<int>(vec_grid(C));
        // norm partials: one per row CTA (rows layout) or per (block, row
        // split) (blocked)
        const int q_parts = std::max({n_row_blocks, sm_count(),
                                      fast ? static_cast<int>(fast->g.nblocks * fast_ax_splits(fast->g.nblocks)) : 0});
        const size_t cb = sizeof(double) * std::max<int64_t>(C, 1), rb8 = sizeof(double) * std::max<int64_t>(R, 1);
        for (double** ptr : {&x, &r, &z, &p, &d, &w, &v}) CAS_CUDA(dmalloc(ptr, cb));
        if (mixed) CAS_CUDA(dmalloc(&pg32, sizeof(float) * std::max<int64_t>(C, 1)));
        CAS_CUDA(dmalloc(&q, mixed ? sizeof(float) * std::max<int64_t>(R, 1) : rb8));
        CAS_CUDA(dmalloc(&q64, rb8));
        if (rows_layout) CAS_CUDA(dmalloc(&partial, sizeof(double) * std::max<int64_t>(a.units, 1)));
        CAS_CUDA(dmalloc(&part_q, sizeof(double) * 2 * q_parts));
        CAS_CUDA(dmalloc(&part_a, sizeof(double) * 2 * std::max(n_vec_blocks, q_parts)));
        CAS_CUDA(dmalloc(&part_b, sizeof(double) * 2 * n_vec_blocks));
        CAS_CUDA(dmalloc(&part_c, sizeof(double) * 2 * n_vec_blocks));
        CAS_CUDA(dmalloc(&scal, sizeof(double) * kSlots));
        CAS_CUDA(dmalloc(&flags, sizeof(int) * kFlags));
        CAS_CUDA(hmalloc(&host_scal, sizeof(double) * kSlots));
        CAS_CUDA(hmalloc(&host_flags, sizeof(int) * kFlags));
        CAS_CUDA(cudaMemsetAsync(scal, 0, sizeof(double) * kSlots, s));
        CAS_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * kFlags, s));
        const double tol = o.tol;
        CAS_CUDA(cudaMemcpyAsync(scal + kTol, &tol, sizeof tol, cudaMemcpyHostToDevice, s));
        if (x0)
            CAS_CUDA(cudaMemcpyAsync(x, x0, cb, cudaMemcpyDeviceToDevice, s));
        else
            CAS_CUDA(cudaMemsetAsync(x, 0, cb, s));
        CAS_CUDA(cudaMemsetAsync(w, 0, cb, s));
        CAS_CUDA(cudaMemsetAsync(v, 0, cb, s));
        const int pmode = (o.method == CAS_PCG && o.jacobi) ? 1 : (scaled() ? 2 : 0);
        if (user_d)
            { user_precond_kernel<<<vec_grid(C), kVecThreads, 0, s>>>(user_d, C, d); cas::count_launch(); }
        else
            { precond_kernel<<<vec_grid(C), kVecThreads, 0, s>>>(a.diag_int, C, pmode, d); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        const Dev D = dv();

        // ||A'b||^2 (denominator of the relative residual).  The mixed PCG
        // from x0 = 0 forms A'b with its FP32 products: its first residual
        // then carries FP32 rounding like every recursive residual of that
        // solver, and the FP64 replacements and the final FP64 check decide
        // convergence.
        const bool atb32 = !bn && !x0 && mixed && fast32 && !least_squares();
        if (bn) {
            ColSum none;
            none.a = a;
            { norm_units_kernel<true><<<n_vec_blocks, kVecThreads, 0, s>>>(none, nullptr, part_a, bn); cas::count_launch(); }
        } else if (atb32) {
            { to_f32_kernel<<<row_grid(R), kVecThreads, 0, s>>>(b, R, static_cast<float*>(q)); cas::count_launch(); }
            CAS_TRY(product_t<float>(static_cast<const float*>(q), nullptr));
            { norm_units_kernel<true><<<n_vec_blocks, kVecThreads, 0, s>>>(colsum<float>(), nullptr, part_a, nullptr); cas::count_launch(); }
        } else {
            CAS_TRY(product_t<double>(b, nullptr));
            { norm_units_kernel<true><<<n_vec_blocks, kVecThreads, 0, s>>>(colsum<double>(), nullptr, part_a, nullptr); cas::count_launch(); }
        }
        { store_sum_kernel<true><<<1, kRedThreads, 0, s>>>(part_a, n_vec_blocks, scal + kBn2); cas::count_launch(); }
        if (scaled()) {
            // ||S A'b||^2: the norm the scaled recursion's residual estimate is relative to
            { norm_units_kernel<true><<<n_vec_blocks, kVecThreads, 0, s>>>(colsum<double>(), nullptr, part_a, nullptr, d); cas::count_launch(); }
            { store_sum_kernel<true><<<1, kRedThreads, 0, s>>>(part_a, n_vec_blocks, scal + kBn2S); cas::count_launch(); }
        }
        CAS_CHECK_LAUNCH();

        if (least_squares()) {
            CAS_TRY(issue_lsqr_start(1));
        } else {
            // from x0 = 0 the first residual is A'b, whose partials the norm
            // above has just read
            const bool reuse_atb = !x0 && !bn;
            if (mixed) CAS_TRY(issue_pcg_refine<true>(true, reuse_atb, atb32));
            else CAS_TRY(issue_pcg_refine<false>(true, reuse_atb));
        }
        CAS_TRY(read_state());
        // the initial residual replacement counted as a refinement; reset
        int zero = 0;
        CAS_CUDA(cudaMemcpyAsync(flags + kRefine, &zero, sizeof zero, cudaMemcpyHostToDevice, s));
        if (host_flags[kStatus] != 0) {
            set_error("solver setup: non-finite right-hand side");
            return static_cast<cas_status>(host_flags[kStatus]);
        }
        return CAS_OK;
    }
};

}  // namespace cas

using namespace cas;

struct cas_solver {
    SolverImpl impl;
};

namespace {
cas_status validate_opts(const cas_solve_opts* o)
{
    CAS_REQUIRE(o, CAS_ERR_INVALID_ARGUMENT, "null solver options");
    CAS_REQUIRE(o->method == CAS_PCG || o->method == CAS_LSQR || o->method == CAS_CG || o->method == CAS_LSMR,
                CAS_ERR_INVALID_ARGUMENT, "unknown solver method");
    CAS_REQUIRE(o->precision == CAS_PLAIN_FP64 || o->precision == CAS_MIXED, CAS_ERR_INVALID_ARGUMENT,
                "unknown precision mode");
    CAS_REQUIRE(o->max_iterations >= 0 && o->check_every >= 0 && o->refine_every >= 0, CAS_ERR_INVALID_ARGUMENT,
                "negative iteration counts in solver options");
    CAS_REQUIRE(o->scale_columns == 0 || o->scale_columns == 1, CAS_ERR_INVALID_ARGUMENT,
                "scale_columns must be 0 or 1");
    return CAS_OK;
}
}  // namespace

extern "C" {

CAS_API void cas_solve_opts_default(cas_solve_opts* o)
{
    if (!o) return;
    o->method = CAS_PCG;
    o->precision = CAS_PLAIN_FP64;
    o->tol = 1e-8;
    o->max_iterations = 20000;
    o->refine_every = 50;
    o->check_every = 50;
    o->jacobi = 1;
    o->scale_columns = 0;
}

}  // extern "C"

namespace {
cas_status create_solver(const cas_csr* a, const cas_solve_opts* o, const double* d_b, const double* d_bn,
                         const double* d_x0, void* stream, cas_solver** out, const double* d_diag = nullptr)
{
    CAS_TRY(validate_opts(o));
    *out = nullptr;
    CAS_TRY(require_device());
    auto* sv = new (std::nothrow) cas_solver;
    CAS_REQUIRE(sv, CAS_ERR_OUT_OF_MEMORY, "cas_solver_create: out of host memory");
    SolverImpl& m = sv->impl;
    m.A = a;
    m.a = a->view();
    m.o = *o;
    m.s = static_cast<cudaStream_t>(stream);
    if (m.s == nullptr) {
        // a blocking stream orders itself with the legacy default stream
        if (cudaStreamCreate(&m.s) != cudaSuccess) {
            delete sv;
            set_error("cas_solver_create: cannot create a stream");
            return CAS_ERR_CUDA;
        }
        m.own_stream = true;
    }
    m.b = d_b;
    if (d_bn) {
        // the normal-equation right-hand side is copied (cols doubles)
        if (dmalloc(&m.b_own, sizeof(double) * std::max<int64_t>(a->cols, 1)) != cudaSuccess ||
            cudaMemcpyAsync(m.b_own, d_bn, sizeof(double) * a->cols, cudaMemcpyDeviceToDevice, m.s) != cudaSuccess) {
            delete sv;
            set_error("cas_solver_create_normal: cannot copy the right-hand side");
            return CAS_ERR_CUDA;
        }
        m.bn = m.b_own;
    }
    cudaGetDevice(&m.device);
    m.user_d = d_diag;
    cas_status st = m.init(d_x0);
    m.user_d = nullptr;  // copied into the solver's d at set-up
    if (st != CAS_OK) {
        delete sv;
        return st;
    }
    *out = sv;
    return CAS_OK;
}
}  // namespace

extern "C" {

CAS_API cas_status cas_solver_create(const cas_csr* a, const cas_solve_opts* o, const double* d_b,
                                     const double* d_x0, void* stream, cas_solver** out)
{
    CAS_REQUIRE(a && out, CAS_ERR_INVALID_ARGUMENT, "cas_solver_create: null argument");
    CAS_REQUIRE(d_b || a->rows == 0, CAS_ERR_INVALID_ARGUMENT, "cas_solver_create: null right-hand side");
    return create_solver(a, o, d_b, nullptr, d_x0, stream, out);
}

CAS_API cas_status cas_solver_create_normal(const cas_csr* a, const cas_solve_opts* o, const double* d_normal_b,
                                            const double* d_x0, void* stream, cas_solver** out)
{
    CAS_REQUIRE(a && out, CAS_ERR_INVALID_ARGUMENT, "cas_solver_create_normal: null argument");
    CAS_REQUIRE(d_normal_b || a->cols == 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_solver_create_normal: null right-hand side");
    CAS_REQUIRE(o && o->method != CAS_LSQR && o->method != CAS_LSMR, CAS_ERR_INVALID_ARGUMENT,
                "cas_solver_create_normal: LSQR and LSMR need the rows-length right-hand side");
    return create_solver(a, o, nullptr, d_normal_b, d_x0, stream, out);
}

CAS_API cas_status cas_solver_create_normal_diag(const cas_csr* a, const cas_solve_opts* o, const double* d_normal_b,
                                                 const double* d_diag, const double* d_x0, void* stream,
                                                 cas_solver** out)
{
    CAS_REQUIRE(a && out, CAS_ERR_INVALID_ARGUMENT, "cas_solver_create_normal_diag: null argument");
    CAS_REQUIRE((d_normal_b && d_diag) || a->cols == 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_solver_create_normal_diag: null right-hand side or preconditioner");
    CAS_REQUIRE(o && o->method == CAS_PCG, CAS_ERR_INVALID_ARGUMENT,
                "cas_solver_create_normal_diag: the diagonal preconditioner is a PCG argument");
    return create_solver(a, o, nullptr, d_normal_b, d_x0, stream, out, d_diag);
}

CAS_API void cas_solver_destroy(cas_solver* s) { delete s; }

namespace {
// Header of a solver checkpoint (cas_solver_save_state).
struct StateHeader {
    uint64_t magic;
    uint32_t version;
    int32_t method, precision, scaled;
    int64_t cols, rows;
    uint64_t bytes;  // the whole checkpoint, header included
};
constexpr uint64_t kStateMagic = 0x5453564c4f534143ull;  // "CASOLVST"
constexpr uint32_t kStateVersion = 1;

StateHeader state_header(const SolverImpl& m)
{
    StateHeader h{};
    h.magic = kStateMagic;
    h.version = kStateVersion;
    h.method = m.o.method;
    h.precision = m.o.precision;
    h.scaled = m.scaled() ? 1 : 0;
    h.cols = m.C;
    h.rows = m.R;
    h.bytes = sizeof(StateHeader);
    for (const auto& b : m.state_buffers()) h.bytes += b.second;
    return h;
}
}  // namespace

CAS_API cas_status cas_solver_state_size(const cas_solver* sv, size_t* bytes)
{
    CAS_REQUIRE(sv && bytes, CAS_ERR_INVALID_ARGUMENT, "cas_solver_state_size: null argument");
    *bytes = state_header(sv->impl).bytes;
    return CAS_OK;
}

CAS_API cas_status cas_solver_save_state(cas_solver* sv, void* h_buf, size_t bytes)
{
    CAS_REQUIRE(sv && h_buf, CAS_ERR_INVALID_ARGUMENT, "cas_solver_save_state: null argument");
    SolverImpl& m = sv->impl;
    const StateHeader h = state_header(m);
    CAS_REQUIRE(bytes >= h.bytes, CAS_ERR_INVALID_ARGUMENT, "cas_solver_save_state: buffer smaller than cas_solver_state_size");
    char* out = static_cast<char*>(h_buf);
    std::memcpy(out, &h, sizeof h);
    size_t off = sizeof h;
    for (const auto& b : m.state_buffers()) {
        CAS_CUDA(cudaMemcpyAsync(out + off, b.first, b.second, cudaMemcpyDeviceToHost, m.s));
        off += b.second;
    }
    CAS_CUDA(cudaStreamSynchronize(m.s));
    return CAS_OK;
}

CAS_API cas_status cas_solver_load_state(cas_solver* sv, const void* h_buf, size_t bytes)
{
    CAS_REQUIRE(sv && h_buf, CAS_ERR_INVALID_ARGUMENT, "cas_solver_load_state: null argument");
    SolverImpl& m = sv->impl;
    CAS_REQUIRE(bytes >= sizeof(StateHeader), CAS_ERR_INVALID_ARGUMENT, "cas_solver_load_state: buffer too small");
    StateHeader h;
    std::memcpy(&h, h_buf, sizeof h);
    const StateHeader want = state_header(m);
    CAS_REQUIRE(h.magic == kStateMagic && h.version == kStateVersion, CAS_ERR_INVALID_ARGUMENT,
                "cas_solver_load_state: not a solver checkpoint of this version");
    CAS_REQUIRE(h.method == want.method && h.precision == want.precision && h.scaled == want.scaled &&
                    h.cols == want.cols && h.rows == want.rows && h.bytes == want.bytes && bytes >= h.bytes,
                CAS_ERR_INVALID_ARGUMENT,
                "cas_solver_load_state: the checkpoint was saved by a solver of another method, precision, "
                "column scaling or matrix shape");
    const char* in = static_cast<const char*>(h_buf);
    size_t off = sizeof h;
    for (const auto& b : m.state_buffers()) {
        CAS_CUDA(cudaMemcpyAsync(b.first, in + off, b.second, cudaMemcpyHostToDevice, m.s));
        off += b.second;
    }
    CAS_TRY(m.read_state());  // also waits for the copies: the caller may free its buffer
    return CAS_OK;
}

CAS_API cas_status cas_solver_iterate(cas_solver* sv, int n)
{
    CAS_REQUIRE(sv && n >= 0, CAS_ERR_INVALID_ARGUMENT, "cas_solver_iterate: bad argument");
    SolverImpl& m = sv->impl;
    const int chunk = m.o.check_every > 0 ? m.o.check_every : n;
    int done = 0;
    while (done < n) {
        const int c = std::min(chunk, n - done);
        CAS_TRY(m.issue_chunk(m.launched, c));
        done += c;
    }
    CAS_TRY(m.read_state());
    return m.host_flags[kStatus] != 0 ? static_cast<cas_status>(m.host_flags[kStatus]) : CAS_OK;
}

CAS_API cas_status cas_solver_residuum(cas_solver* sv, double* h_out)
{
    CAS_REQUIRE(sv && h_out, CAS_ERR_INVALID_ARGUMENT, "cas_solver_residuum: null argument");
    CAS_TRY(sv->impl.read_state());
    *h_out = sv->impl.o.method == CAS_LSQR ? sv->impl.host_scal[kPhiBar]
                                           : (sv->impl.o.method == CAS_LSMR ? 0.0 : sv->impl.host_scal[kRr]);
    return CAS_OK;
}

CAS_API cas_status cas_solver_x(cas_solver* sv, double* d_out)
{
    CAS_REQUIRE(sv && (d_out || sv->impl.C == 0), CAS_ERR_INVALID_ARGUMENT, "cas_solver_x: null argument");
    SolverImpl& m = sv->impl;
    if (m.C) CAS_CUDA(cudaMemcpyAsync(d_out, m.x, sizeof(double) * m.C, cudaMemcpyDeviceToDevice, m.s));
    return CAS_OK;
}

CAS_API cas_status cas_solver_rel_residual(cas_solver* sv, double* h_out)
{
    CAS_REQUIRE(sv && h_out, CAS_ERR_INVALID_ARGUMENT, "cas_solver_rel_residual: null argument");
    return sv->impl.true_residual(h_out);
}

CAS_API int cas_solver_iterations(const cas_solver* sv)
{
    if (!sv) return -1;
    auto& m = const_cast<cas_solver*>(sv)->impl;
    if (m.read_state() != CAS_OK) return -1;
    return m.host_flags[kIter];
}

}  // extern "C"

namespace cas {
// The host side of one solve to tolerance, as a sequence of steps: each
// step reads the device state once, takes the decisions of a chunk
// boundary (convergence on the FP64 true residual, restarts and
// replacements requested by the host) and issues the next chunk of
// iterations without waiting for it.  cas_solver_run steps one solver; the
// batched LSQR/LSMR fit steps several, each on its own stream, in turn, so
// that one solver's chunk runs while the host reads another's state.
struct RunLoop {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double rel = 0;
    int extra_checks = 0;
    cas_status st = CAS_OK;
    bool finished = false;
    float ms = 0;
};

cas_status run_begin(SolverImpl& m, RunLoop& L)
{
    CAS_CUDA(cudaEventCreate(&L.e0));
    CAS_CUDA(cudaEventCreate(&L.e1));
    CAS_CUDA(cudaEventRecord(L.e0, m.s));
    return CAS_OK;
}

cas_status run_step(SolverImpl& m, RunLoop& L)
{
    const int chunk = m.o.check_every > 0 ? m.o.check_every : 50;
    CAS_TRY(m.read_state());
    const int it = m.host_flags[kIter];
    if (m.host_flags[kStatus] != 0) {
        L.st = static_cast<cas_status>(m.host_flags[kStatus]);
        L.finished = true;
        return CAS_OK;
    }
    const bool done = m.host_flags[kDone] || m.host_flags[kPending];
    if (m.least_squares() && m.o.tol > 0 && !done && it > 0) {
        // LSQR's recursive residual estimates lose their meaning once the
        // bidiagonalisation loses orthogonality, and iterating past
        // convergence can diverge (the reference's LSQR has no stopping
        // test), so its stopping test is the true FP64 residual, checked
        // at every chunk boundary.
        CAS_TRY(m.true_residual(&L.rel));
        if (L.rel <= m.o.tol) {
            L.finished = true;
            return CAS_OK;
        }
        // The mixed solver's cycle has drifted: its estimate is more than
        // kLsqrDrift times below the true residual (the FP32 products'
        // noise floor reached before the restart drop): restart now.
        if (m.mixed && m.host_scal[kRes] * kLsqrDrift < L.rel && !m.scaled()) CAS_TRY(m.issue_lsqr_start(3));
    }
    if (done) {
        if (m.host_flags[kVerified] && !m.least_squares()) {
            // a residual replacement met the tolerance on the FP64 true residual
            L.rel = m.host_scal[kRes];
            L.finished = true;
            return CAS_OK;
        }
        // verify with the true FP64 residual
        CAS_TRY(m.true_residual(&L.rel));
        if (m.o.tol <= 0 || L.rel <= m.o.tol || it >= m.o.max_iterations) {
            L.finished = true;
            return CAS_OK;
        }
        if (L.extra_checks > 20) {
            L.st = CAS_ERR_NOT_CONVERGED;
            L.finished = true;
            return CAS_OK;
        }
        // recursive residual drifted: replace it and continue
        L.extra_checks++;
        static const int zero = 0;
        CAS_CUDA(cudaMemcpyAsync(m.flags + kDone, &zero, sizeof zero, cudaMemcpyHostToDevice, m.s));
        CAS_CUDA(cudaMemcpyAsync(m.flags + kPending, &zero, sizeof zero, cudaMemcpyHostToDevice, m.s));
        if (m.least_squares() && m.mixed) {
            // the mixed cycle's estimate met the tolerance but the FP64
            // residual did not: restart from it
            CAS_TRY(m.issue_lsqr_start(3));
        } else if (m.least_squares()) {
            // LSQR / LSMR have no residual to replace: tighten the recursive target
            double t = m.host_scal[kTol] * 0.5;
            CAS_CUDA(cudaMemcpyAsync(m.scal + kTol, &t, sizeof t, cudaMemcpyHostToDevice, m.s));
        } else if (m.mixed) {
            // the converged step skipped p = z + beta p: restart p = z
            CAS_TRY(m.issue_pcg_refine<true>(true));
        } else {
            CAS_TRY(m.issue_pcg_refine<false>(true));
        }
        return CAS_OK;  // the next step reads the state again
    }
    if (it >= m.o.max_iterations) {
        CAS_TRY(m.true_residual(&L.rel));
        if (m.o.tol > 0 && L.rel > m.o.tol) L.st = CAS_ERR_NOT_CONVERGED;
        L.finished = true;
        return CAS_OK;
    }
    const int n = std::min(chunk, m.o.max_iterations - it);
    CAS_TRY(m.issue_chunk(m.launched, n));
    return CAS_OK;
}

// Ends a solve: its device time, the report, the status.
cas_status run_end(SolverImpl& m, RunLoop& L, cas_solve_report* rep)
{
    CAS_CUDA(cudaEventRecord(L.e1, m.s));
    CAS_CUDA(cudaEventSynchronize(L.e1));
    cudaEventElapsedTime(&L.ms, L.e0, L.e1);
    cudaEventDestroy(L.e0);
    cudaEventDestroy(L.e1);
    L.e0 = L.e1 = nullptr;
    CAS_TRY(m.read_state());
    if (rep) {
        rep->iterations = m.host_flags[kIter];
        rep->refinements = m.host_flags[kRefine];
        rep->rel_residual = L.rel;
        rep->residuum = m.o.method == CAS_LSQR ? m.host_scal[kPhiBar] : (m.o.method == CAS_LSMR ? 0.0 : m.host_scal[kRr]);
        rep->seconds = L.ms * 1e-3;
        rep->setup_seconds = 0;
    }
    if (L.st == CAS_ERR_NOT_CONVERGED) set_error("solver did not reach the tolerance within max_iterations");
    if (L.st == CAS_ERR_BREAKDOWN) set_error("solver breakdown (p'A'Ap <= 0 or non-finite scalar)");
    return L.st;
}

void run_abandon(RunLoop& L)
{
    if (L.e0) cudaEventDestroy(L.e0);
    if (L.e1) cudaEventDestroy(L.e1);
    L.e0 = L.e1 = nullptr;
}
}  // namespace cas

extern "C" {

CAS_API cas_status cas_solver_run(cas_solver* sv, cas_solve_report* rep)
{
    cas::NvtxRange nvtx_range("cas_solver_run");
    CAS_REQUIRE(sv, CAS_ERR_INVALID_ARGUMENT, "cas_solver_run: null solver");
    SolverImpl& m = sv->impl;
    RunLoop L;
    cas_status st = run_begin(m, L);
    while (st == CAS_OK && !L.finished) st = run_step(m, L);
    if (st != CAS_OK) {
        run_abandon(L);
        return st;
    }
    return run_end(m, L, rep);
}

}  // extern "C"

namespace cas {
// Several solvers to tolerance at once, each on its own stream (the batched
// LSQR/LSMR fit): the host steps the unfinished ones in turn.  Returns the
// first error of a CUDA call; per-solver statuses go to sts.
cas_status solvers_run_all(cas_solver* const* svs, int n, cas_solve_report* reps, cas_status* sts)
{
    std::vector<RunLoop> loops(n);
    for (int i = 0; i < n; i++) {
        sts[i] = CAS_OK;
        if (svs[i]) CAS_TRY(run_begin(svs[i]->impl, loops[i]));
    }
    cas_status err = CAS_OK;
    for (bool any = true; any && err == CAS_OK;) {
        any = false;
        for (int i = 0; i < n && err == CAS_OK; i++) {
            if (!svs[i] || loops[i].finished) continue;
            err = run_step(svs[i]->impl, loops[i]);
            any = true;
        }
    }
    for (int i = 0; i < n; i++) {
        if (!svs[i]) continue;
        if (err != CAS_OK) {
            run_abandon(loops[i]);
            continue;
        }
        sts[i] = run_end(svs[i]->impl, loops[i], reps ? &reps[i] : nullptr);
    }
    return err;
}
}  // namespace cas

extern "C" {

CAS_API cas_status cas_solve(const cas_csr* a, const cas_solve_opts* o, const double* d_b, double* d_x,
                             cas_solve_report* rep, void* stream)
{
    cas_solver* sv = nullptr;
    CAS_TRY(cas_solver_create(a, o, d_b, nullptr, stream, &sv));
    cas_status st = cas_solver_run(sv, rep);
    if (st == CAS_OK || st == CAS_ERR_NOT_CONVERGED) {
        cas_status s2 = cas_solver_x(sv, d_x);
        if (s2 != CAS_OK) st = s2;
        cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    }
    cas_solver_destroy(sv);
    return st;
}

}  // extern "C"
