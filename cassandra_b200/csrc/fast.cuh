// The blocked layout of a pattern CSR and its products (fast.cu).
//
// Rows are cut into blocks of kBlockRows.  Inside a block the entries of each
// pattern (indexer) are stored together:
//
//   A16  uint16  [block][pattern][row][slot]   local column of every entry
//   G32  uint32  [block][pattern][entry]       (local column << 16) |
//                                              (row in block << 2) | end,
//                                              sorted by column then row (the
//                                              transposed copy); end marks the
//                                              last entry of each column
//
// G32 is stored in rounds of kRound entries: the sorted order is cut into
// rounds from each group's start (every group starts on a round boundary),
// and inside a round the 32 consecutive entries a lane reduces (lane L:
// entries 32L .. 32L+31) lie in 8 rows of 512 bytes, one 16-byte word per
// lane and row, so that a warp reads a round with 8 coalesced loads.
// round_phys() maps an entry's position in the sorted order to its place.
//
// Both copies group a block's entries by pattern, so that a CTA touches one
// pattern's columns at a time.  A x stages that
// pattern's slice of x in shared memory and gathers from there; A'y stages
// the block's slice of y in shared memory and reduces the column-sorted
// entries of one column chunk into a shared-memory accumulator.  Local
// columns must fit 16 bits (index space per pattern <= 65536).
#pragma once
#include <cstdint>

#include "internal.cuh"

namespace cas {

constexpr int kBlockRows = 16384;        // rows per block (and per A'y tile)
constexpr int kRound = 1024;             // G32 entries of one A'y round (32 lanes x 32)
constexpr int kLaneRun = kRound / 32;    // consecutive entries a lane reduces per round
constexpr int kFastThreads = 1024;       // threads of the A'y kernel
constexpr int kAxThreads = 1024;         // threads of the A x kernel
constexpr int kAxRows = kBlockRows / kAxThreads;  // rows per thread in A x
constexpr int kAxAhead = 3;              // index loads in flight per thread in A x
constexpr int kChunkCols = 8192;         // column chunk of the A'y accumulators
constexpr int kSubCols = 1024;           // column sub-chunk: the finest split of an A'y item
constexpr int kSubPerChunk = kChunkCols / kSubCols;
constexpr int kEvalRedMax = 4096;        // CTAs of each reduction of an evaluator training step
constexpr int kAxSplitMax = 32;          // most CTAs sharing one block's rows in A x
constexpr int kAxDirectRows = kAxThreads / 2;  // rows of a unit that gathers x without staging (one thread a row)
static_assert(kBlockRows / kAxSplitMax <= kAxDirectRows, "a block split kAxSplitMax ways must fit the direct path");
constexpr int kAtySplitMax = 16;         // most CTAs sharing one A'y item's columns
constexpr int kMaxFastPatterns = 32;
constexpr int kTable32 = 57344;          // x entries staged per pattern, FP32
constexpr int kTable64 = 28672;          // x entries staged per pattern, FP64

constexpr int kMaxProblems = 64;         // independent fits in one batched layout

// Per-pattern geometry, passed to kernels by value.
//
// A layout may hold several independent problems (a batch of fits over the
// same patterns): problem q owns rows [prow0[q], prow0[q+1]) and blocks
// [pblk0[q], pblk0[q+1]) -- blocks never straddle problems, so a problem's
// last block may be partial -- and columns [q * pcols, (q + 1) * pcols).
// The matrix is block diagonal.  A single fit is the case nprob == 1.
struct FastGeometry {
    int npat = 0;
    int k = 0;                           // entries per row (sum of slots)
    int64_t rows = 0, cols = 0;          // cols = nprob * pcols
    int64_t nblocks = 0;
    int slot0[kMaxFastPatterns];
    int slots[kMaxFastPatterns];
    int64_t off[kMaxFastPatterns];       // column offset of the pattern inside a problem
    int space[kMaxFastPatterns];         // columns of the pattern
    int chunk0[kMaxFastPatterns];        // first global chunk of the pattern
    int nchunks = 0;
    int nprob = 1;
    int64_t pcols = 0;                   // columns per problem
    int64_t prow0[kMaxProblems + 1];     // first row of each problem
    int pblk0[kMaxProblems + 1];         // first block of each problem

    __host__ __device__ int prob_of_block(int64_t b) const
    {
        int lo = 0, hi = nprob - 1;  // largest q with pblk0[q] <= b
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pblk0[mid] <= b)
                lo = mid;
            else
                hi = mid - 1;
        }
        return lo;
    }
    __host__ __device__ int prob_of_row(int64_t r) const
    {
        int lo = 0, hi = nprob - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prow0[mid] <= r)
                lo = mid;
            else
                hi = mid - 1;
        }
        return lo;
    }
    __host__ __device__ int64_t block_row0(int64_t b) const
    {
        const int q = prob_of_block(b);
        return prow0[q] + (b - pblk0[q]) * kBlockRows;
    }
    __host__ __device__ int64_t block_rows(int64_t b) const
    {
        const int q = prob_of_block(b);
        const int64_t r = prow0[q + 1] - (prow0[q] + (b - pblk0[q]) * kBlockRows);
        return r < kBlockRows ? r : kBlockRows;
    }
    // First column of the problem that owns block b.
    __host__ __device__ int64_t col_base(int64_t b) const { return prob_of_block(b) * pcols; }
    // Block and row inside the block of row r.
    __host__ __device__ void locate_row(int64_t r, int64_t& b, int64_t& rb) const
    {
        const int q = prob_of_row(r);
        const int64_t local = r - prow0[q];
        b = pblk0[q] + local / kBlockRows;
        rb = local - (local / kBlockRows) * kBlockRows;
    }
    // Rows of a block rounded up to kRound, so that every (block, pattern)
    // segment starts on a G32 round (and on a 16-byte boundary).
    __host__ __device__ int64_t padded_rows(int64_t b) const
    {
        return (block_rows(b) + kRound - 1) & ~int64_t(kRound - 1);
    }
    // Element offset of (block, pattern) in A16 / G32.
    __host__ __device__ int64_t seg(int64_t b, int p) const
    {
        return b * int64_t(kBlockRows) * k + padded_rows(b) * slot0[p];
    }
    __host__ __device__ int64_t seg_len(int64_t b, int p) const { return block_rows(b) * slots[p]; }
    __host__ __device__ int64_t total_elems() const
    {
        return nblocks == 0 ? 0 : (nblocks - 1) * int64_t(kBlockRows) * k + padded_rows(nblocks - 1) * k;
    }
};

// Place in G32 of the entry at position i of the sorted order (i counted
// from any round boundary): offset o = 32 L + 4 q + j inside the round goes
// to 128 q + 4 L + j.
__host__ __device__ __forceinline__ uint32_t round_phys(uint32_t i)
{
    return (i & ~uint32_t(kRound - 1)) | ((i & 0x1Cu) << 5) | ((i & 0x3E0u) >> 3) | (i & 3u);
}
static_assert(kRound == 1024 && kLaneRun == 32, "round_phys assumes 32 lanes x 32 entries");

// The problems a batched step works on (those not retired), in problem
// order, rebuilt on the device before each iteration.  Given to the
// products, it lets a few remaining small problems still fill the GPU: A x
// and A'y split their work units (a block's rows, an item's columns) over
// more CTAs the fewer units the listed problems have.
struct FastActive {
    int n;
    int list[kMaxProblems];
    int pos[kMaxProblems];  // slot of each problem in list, -1 if absent
};

// Work list of one A'y variant.  Columns are grouped into "super-chunks":
// sets of column pieces (whole 8192-column chunks of one pattern, or a
// pattern's last partial chunk) packed into one shared-memory accumulator of
// per_sc chunks, so several narrow patterns share one pass over a block's y
// slice.  An item is (super-chunk, block range); every item writes the
// partial sums of its super-chunk's columns, and a column's value is the sum
// of its super-chunk's items in item order.
struct FastTranspose {
    int per_sc = 1;        // accumulator capacity in chunks
    bool range_major = false;  // single fits: items run block range by block range (y slices shared in L2)
    int items_per_sm = 2;  // work items per SM the entries are balanced over
    bool pack = true;      // super-chunks may hold pieces of several patterns
    bool persistent = false;  // one CTA per SM taking items from a counter (else one CTA per item)
    int nsc = 0;
    int npieces = 0;
    int nitems = 0;
    int64_t max_item_entries = 0;  // most G32 entries any item reduces
    int* sc_piece0 = nullptr;  // [nsc + 1] first piece of each super-chunk
    int* sc_width = nullptr;   // [nsc] accumulator columns in use
    int* piece_pat = nullptr;  // [npieces] pattern of the piece
    int* piece_ch0 = nullptr;  // [npieces] first global chunk
    int* piece_ch1 = nullptr;  // [npieces] one past the last global chunk (same pattern)
    int* piece_acc = nullptr;  // [npieces] accumulator offset of the piece's first column
    int* chunk_sc = nullptr;   // [nchunks] super-chunk of every chunk
    int* chunk_acc = nullptr;  // [nchunks] accumulator offset of the chunk's first column
    int* item_sc = nullptr;    // [nitems]
    int* item_b0 = nullptr;    // [nitems]
    int* item_b1 = nullptr;    // [nitems]
    int64_t* item_part = nullptr;  // [nitems] offset of the item's partials
    int* sc_item0 = nullptr;       // [nprob * nsc + 1] first entry of each (problem, super-chunk) in sc_part
    int64_t* sc_part = nullptr;    // [nitems] partial offsets of the items, listed super-chunk by super-chunk
                                   // (block ranges in order): the order the column sums add them in
    void* partial = nullptr;       // float or double partials
    int* ctr = nullptr;            // [2] work counter and finished CTAs of the persistent schedule (reset by the kernel)
    void* meta = nullptr;          // one device block holding every array above except partial
};

// One measured A'y schedule of the build-time autotuner.
struct FastTuneEntry {
    int per_sc;
    int range_major;
    int items_per_sm;
    int pack;
    int persistent;
    float ms;  // mean time of one FP32 A'y (partials + column sums) on this layout
};
constexpr int kMaxTune = 12;

struct FastLayout {
    FastGeometry g;
    FastTuneEntry tune[kMaxTune];      // candidates timed at build (empty: default schedule)
    int ntune = 0;
    int tune_cached = 0;               // schedule taken from the per-process cache
    uint16_t* a16 = nullptr;
    uint32_t* g32 = nullptr;
    uint32_t* sub_start = nullptr;     // [nblocks][nchunks * kSubPerChunk] absolute index in G32 of the
                                       // first entry of every column sub-chunk (a chunk starts at its first)
    FastTranspose t32, t64;            // A'y work lists of the solvers (FP32, FP64)
    FastTranspose tb;                  // one item per (block, chunk): adjoints over block ranges
    float* eval_partial = nullptr;     // [blocks][cols] partials of the last adjoint
    float* eval_dscore = nullptr;      // [blocks * kBlockRows] loss gradient of a training step's rows
    int64_t eval_blocks = 0;           // blocks the two buffers above hold
    bool eval_captured = false;        // a CUDA graph captured a call that uses them: they never move again
    double* eval_red = nullptr;        // [2 * kEvalRedMax] per-CTA loss partials of a training step
    int* eval_ctr = nullptr;           // last-CTA counter of the training step's epilogue
};

// Hyperparameters of one training step of the evaluator (Adam as
// torch.optim.Adam without weight decay; mean Huber loss plus l2 ||w||^2).
struct EvalAdam {
    float lr, beta1, beta2, eps, l2, delta;
};

// Device view used by the column reductions of the solver.
struct FastCols {
    FastGeometry g;
    int nsc;                 // super-chunks per problem
    const int* chunk_sc;
    const int* chunk_acc;
    const int* sc_item0;
    const int64_t* sc_part;
};

// Builds the blocked layout from positions (indexes them itself).  Returns
// CAS_ERR_INVALID_ARGUMENT without touching `out` if the pattern set does
// not fit the layout (a pattern wider than 16-bit columns, too many patterns
// or a slot count other than 1, 2, 4, 8).
// prob_rows (host, nprob entries) splits the rows into independent problems
// (a batch of fits, in row order); null with nprob == 1 is a single fit.
// chunks (may be null): positions still arriving, indexed chunk by chunk.
cas_status fast_build(const DevicePatterns& dp, const PatternSet& ps, const uint64_t* d_pos, int64_t rows,
                      const int64_t* prob_rows, int nprob, uint64_t* diag_int, FastLayout& out, cudaStream_t s,
                      const PositionChunks* chunks = nullptr);
bool fast_supported(const PatternSet& ps);
void fast_free(FastLayout& f);

// y = A x on the blocked layout; also writes partials of ||y||^2, one per
// (block, row split) (part may be null; *n_parts = their number).  mode 0:
// y = A x; 1: y = A x - coef * y (coef read from *coef); 2: y = b - A x (b
// may be null: y = -A x).  done_flag set: nothing runs; pdone[q] set: the
// rows of problem q are skipped (their partials are 0).
//
// Without act a block's rows are split over ax_splits(nblocks) CTAs and the
// partials are laid out [block][split].  With act only the listed problems'
// blocks run, split by a factor the kernel derives from the listed blocks,
// and the partials are laid out [block][kAxSplitMax] (splits not used are 0):
// problem q's partials are the 2 * kAxSplitMax * (pblk0[q+1] - pblk0[q])
// doubles from part + 2 * kAxSplitMax * pblk0[q].
template <typename T, typename Y>
cas_status fast_spmv(const FastLayout& f, const T* x, Y* y, const double* b, const double* coef, double* part,
                     int* done_flag, int mode, cudaStream_t s, int* n_parts, const int* pdone = nullptr,
                     const FastActive* act = nullptr);
// Row splits per block of A x without an active list.
int fast_ax_splits(int64_t nblocks);

// Partials of A' y on the blocked layout (FP32: float partials, FP64:
// double partials; a null y stands for a vector of ones); columns are
// summed by fast_col_sum().  Items of
// problems whose pdone flag is set are skipped.  An item's columns may be
// split over several CTAs (column sub-chunks), each writing its columns of
// the item's partials, so the partial layout does not depend on the split.
// With act only the listed problems' items run (one CTA per SM taking
// units from the work counter).
template <typename T>
cas_status fast_spmv_t_partials(const FastLayout& f, const T* y, int* done_flag, cudaStream_t s,
                                const int* pdone = nullptr, const FastActive* act = nullptr);

template <typename T>
FastCols fast_cols(const FastLayout& f);

template <typename T>
__device__ __forceinline__ double fast_col_sum(const FastCols& fc, const T* partial, int64_t c)
{
    int64_t q = 0;
    if (fc.g.nprob > 1) {
        q = c / fc.g.pcols;
        c -= q * fc.g.pcols;
    }
    int p = 0;
    while (p + 1 < fc.g.npat && fc.g.off[p + 1] <= c) p++;
    const int local = static_cast<int>(c - fc.g.off[p]);
    const int ch = fc.g.chunk0[p] + local / kChunkCols;
    const int sc = static_cast<int>(q) * fc.nsc + fc.chunk_sc[ch];
    const int pos = fc.chunk_acc[ch] + local % kChunkCols;
    double acc = 0;
    // unrolled so that the partials' loads are issued ahead of the adds,
    // which keep their order
#pragma unroll 8
    for (int it = fc.sc_item0[sc]; it < fc.sc_item0[sc + 1]; it++) acc += static_cast<double>(partial[fc.sc_part[it] + pos]);
    return acc;
}

// Jacobi diagonal diag(A'A) as integers (deterministic), written over diag:
// the column counts from the FP32 A'y of a vector of ones (exact while every
// item holds fewer than 2^24 entries, else counted from G32 directly) plus
// the share of rows that hold a column more than once.  Needs the FP32 work
// list.
cas_status fast_diag(const FastLayout& f, uint64_t* diag, cudaStream_t s);

// Evaluator forward over rows [row0, row1) (FP32 scores) and its adjoint
// grad = A' g over the rows of blocks [b0, b1) (deterministic; grad has cols
// entries and is overwritten).
cas_status fast_eval_forward(const FastLayout& f, int64_t row0, int64_t row1, const float* w, float* score,
                             cudaStream_t s);
cas_status fast_eval_backward(FastLayout& f, int64_t b0, int64_t b1, const float* g, float* grad, cudaStream_t s);
// One training step on rows [row0, row1) (block bounds; row1 may be the last
// row): three kernels — forward with the Huber loss and its gradient, the
// adjoint's partials, and the epilogue with the L2 term and Adam (w, m, v
// updated; *step advanced; the step's loss added to *loss_sum).
cas_status fast_eval_adam_step(FastLayout& f, int64_t row0, int64_t row1, const float* target, float* w, float* m,
                               float* v, int64_t* step, double* loss_sum, const EvalAdam& o, cudaStream_t s);

// Full A'y into a dense vector (standalone product).
template <typename T>
cas_status fast_spmv_t(const FastLayout& f, const T* y, T* x, cudaStream_t s);

}  // namespace cas
