/*
 * cassandra_b200 — C ABI of the B200 pattern-evaluator fitting path.
 *
 * The path: batches of Reversi positions -> ternary pattern indices under the
 * board symmetries (Pattern/Indexer.cpp) -> a fixed-width CSR matrix with
 * implicit 1.0 entries (Math/MatrixCSR.h) and a sort-built transposed copy ->
 * Jacobi-PCG on the normal equations and LSQR (Math/Solver.h), as driven by
 * FitWeights (PatternFit/PatternFit.cpp:7-39).
 *
 * Conventions
 *  - Every entry point returns a cas_status; CAS_OK is 0.  A failing call
 *    leaves a message retrievable with cas_last_error() on the same thread.
 *    No C++ exception crosses this boundary.
 *  - Pointers prefixed d_ are device pointers (CUDA global memory of the
 *    current device); h_ are host pointers.  Both are borrowed for the call
 *    (device pointers until the stream work completes).
 *  - `stream` is a cudaStream_t passed as void*; NULL means the legacy
 *    default stream.  Calls on one handle must be serialised by the caller.
 *  - Positions are 16-byte records {uint64 P, uint64 O}: P = discs of the
 *    side to move, O = opponent, bit 63 = A1 ... bit 0 = H8
 *    (Board/Position.h:11-33, Board/Field.h:7-18).
 *  - Handles own their device memory; destroy functions accept NULL.
 *  - There is no CPU fallback: without a usable CUDA device the compute
 *    entry points return CAS_ERR_NO_DEVICE.
 */
#ifndef CASSANDRA_B200_H
#define CASSANDRA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CAS_API __attribute__((visibility("default")))

typedef enum cas_status {
    CAS_OK = 0,
    CAS_ERR_SIZE_MISMATCH = 1,    /* "Size mismatch." (Math/MatrixCSR.cpp:51-52, Math/Solver.h:91-93) */
    CAS_ERR_INVALID_ARGUMENT = 2, /* null pointer, negative size, bad enum */
    CAS_ERR_PATTERN = 3,          /* mask unusable (empty, >16 squares, index space > 2^32) */
    CAS_ERR_CUDA = 4,             /* CUDA runtime error (message has the details) */
    CAS_ERR_OUT_OF_MEMORY = 5,
    CAS_ERR_NO_DEVICE = 6,        /* no usable CUDA device */
    CAS_ERR_BREAKDOWN = 7,        /* solver breakdown: p'A'Ap <= 0, or a non-finite scalar */
    CAS_ERR_NOT_CONVERGED = 8     /* tolerance not reached within max_iterations */
} cas_status;

/* Name of a status code ("CAS_OK", ...).  Never NULL. */
CAS_API const char* cas_status_name(cas_status s);

/* Copies the calling thread's last error message (NUL-terminated, truncated
 * to cap) and returns its full length. */
CAS_API size_t cas_last_error(char* buf, size_t cap);

/* ABI version: major * 10000 + minor * 100 + patch. */
CAS_API int cas_version(void);

/* Number of kernels this library has launched in this process (kernels of a
 * replayed CUDA graph count at every replay).  Used to report launches. */
CAS_API long long cas_kernel_launches(void);

/* No counterpart in the reference (memory of the library's own objects).
 * Layouts, solvers and the one-shot fits take device and pinned host memory
 * from a per-device cache that keeps freed blocks for the next object of a
 * similar size (the training loop fits the same shapes repeatedly), up to a
 * quarter of the device's memory.  A cached block is reused only after the
 * work that used it has finished, as with cudaFree.
 * cas_cached_memory: bytes held in the cache now (free, not in use).
 * cas_release_cached_memory: returns every cached block to the driver. */
CAS_API size_t cas_cached_memory(void);
CAS_API void cas_release_cached_memory(void);

/* ------------------------------------------------------------------------ */
/* Pattern sets: GroupIndexer (Pattern/Indexer.h:29-40)                      */
/* ------------------------------------------------------------------------ */

typedef enum cas_index_mode {
    /* Bit-exact with GroupIndexer::InsertIndices (Pattern/Indexer.cpp:413-422):
     * each mask goes through CreateIndexer (:319-365) and is collapsed by its
     * symmetry stabiliser. */
    CAS_INDEX_REFERENCE = 0,
    /* The A_Indexer recipe (Pattern/Indexer.cpp:31-41) for every mask: 8
     * instances (id, C, D, H, V, H.C, H.D, H.V), 3^k columns per mask, column
     * offsets the running sum of 3^k. */
    CAS_INDEX_EXPANDED = 1
} cas_index_mode;

typedef struct cas_patterns cas_patterns;

/* Replaces GroupIndexer(std::vector<uint64_t>) (Pattern/Indexer.cpp:382-392).
 * Masks use the repo's bit order (bit 0 = H8). */
CAS_API cas_status cas_patterns_create(const uint64_t* masks, int n, cas_index_mode mode, cas_patterns** out);
CAS_API void cas_patterns_destroy(cas_patterns* p);
/* GroupIndexer::index_space_size (Pattern/Indexer.h:33). */
CAS_API int64_t cas_patterns_cols(const cas_patterns* p);
/* Variations().size(): entries per CSR row (PatternFit/PatternFit.cpp:14). */
CAS_API int cas_patterns_nnz_per_row(const cas_patterns* p);
/* GroupIndexer::Variations() (Pattern/Indexer.cpp:394-403): writes
 * nnz_per_row masks. */
CAS_API cas_status cas_patterns_variations(const cas_patterns* p, uint64_t* h_out);
/* Per-mask indexer facts for mask i: the pattern CreateIndexer stores
 * (Pattern/Indexer.cpp:353-360 may flip it), symmetry_group_order,
 * index_space_size and the column offset of its block. */
CAS_API cas_status cas_patterns_indexer(const cas_patterns* p, int i, uint64_t* stored_pattern, int* order,
                                        int64_t* space, int64_t* offset);

/* Indexer kernel: writes nnz_per_row uint32 column indices per position,
 * row-major, exactly as GroupIndexer::InsertIndices fills MatrixCSR::Row(i)
 * (PatternFit/PatternFit.cpp:18-21). */
CAS_API cas_status cas_index(const cas_patterns* p, const uint64_t* d_positions, int64_t n, uint32_t* d_out,
                             void* stream);

/* ------------------------------------------------------------------------ */
/* Matrices: MatrixCSR (Math/MatrixCSR.h:11-33)                              */
/* ------------------------------------------------------------------------ */

typedef enum cas_dtype { CAS_F32 = 0, CAS_F64 = 1 } cas_dtype;

typedef struct cas_csr cas_csr;

/* Index d_positions and build the device-resident CSR plus its transposed
 * copy and the column statistics (replaces PatternFit/PatternFit.cpp:12-21).
 * Builds both layouts below (BLOCKED only when the pattern set fits it). */
CAS_API cas_status cas_csr_from_positions(const cas_patterns* p, const uint64_t* d_positions, int64_t rows,
                                          void* stream, cas_csr** out);
/* Device layouts of a CSR.  ROWS is the reference's row-major structure
 * (uint32 indices, rows * nnz_per_row) plus its transposed copy sorted by
 * (column, row).  BLOCKED stores each pattern's entries per 16384-row block
 * as 16-bit local columns, plus a per-block column-sorted copy; its products
 * stage their gather vectors in shared memory (the fast path of the mixed
 * solver).  BLOCKED needs every pattern's index space <= 65536. */
typedef enum cas_layout { CAS_LAYOUT_ROWS = 1, CAS_LAYOUT_BLOCKED = 2 } cas_layout;

/* As cas_csr_from_positions, building only the layouts in `layouts` (a mask
 * of cas_layout).  Products use BLOCKED when present. */
CAS_API cas_status cas_csr_from_positions_layout(const cas_patterns* p, const uint64_t* d_positions, int64_t rows,
                                                 int layouts, void* stream, cas_csr** out);
/* Mask of the layouts a CSR holds. */
CAS_API int cas_csr_layouts(const cas_csr* a);

/* Build from existing row-major indices (MatrixCSR(K, rows, cols) filled via
 * Row(i), Math/MatrixCSR.cpp:5-19).  The indices are copied. */
CAS_API cas_status cas_csr_from_indices(const uint32_t* d_indices, int nnz_per_row, int64_t rows, int64_t cols,
                                        void* stream, cas_csr** out);
CAS_API void cas_csr_destroy(cas_csr* a);
CAS_API int64_t cas_csr_rows(const cas_csr* a);
CAS_API int64_t cas_csr_cols(const cas_csr* a);
CAS_API int cas_csr_nnz_per_row(const cas_csr* a);
/* Device pointer to the rows * nnz_per_row row-major column indices (NULL
 * when the CSR has no ROWS layout). */
CAS_API const uint32_t* cas_csr_indices(const cas_csr* a);
/* Device pointers to the transposed copy: col_ptr (cols + 1 int64) and the
 * row index of every entry, sorted by (column, row). */
CAS_API cas_status cas_csr_transposed(const cas_csr* a, const int64_t** d_col_ptr, const uint32_t** d_row_idx);

/* No counterpart in the reference: the schedules of the FP32 transposed
 * product on the BLOCKED layout that the build-time autotuner timed for this
 * matrix (accumulator width in 8192-column chunks per work item, work items
 * run block range by block range so that concurrent items share y slices
 * through L2 or balanced by entries super-chunk by super-chunk, work items
 * per SM, accumulators shared by several patterns, persistent CTAs taking
 * items from a counter; mean milliseconds per product), and the schedule in
 * use.  Returns
 * the number of timed schedules written (at most max): 0 when the schedule
 * came from the per-process cache of an earlier build of the same shape, from
 * the CAS_ATY_SCHEDULE environment variable, or is the default of layouts
 * under 64 blocks; -1 without a blocked layout. */
typedef struct cas_schedule {
    int chunks_per_item;
    int range_major; /* items run block range by block range (super-chunks share y slices through L2) */
    int items_per_sm;
    int pack;
    int persistent;
    float ms;
} cas_schedule;
CAS_API int cas_csr_schedules(const cas_csr* a, cas_schedule* out, int max, cas_schedule* in_use);

/* y = A x (operator*(const MatrixCSR&, const Vector&), Math/MatrixCSR.cpp:49-65).
 * x has cols entries, y rows entries, both of dtype. */
CAS_API cas_status cas_spmv(const cas_csr* a, cas_dtype dtype, const void* d_x, void* d_y, void* stream);
/* x = A' y (operator*(const Vector&, const MatrixCSR&), Math/MatrixCSR.cpp:67-87),
 * computed over the transposed copy: deterministic, no atomics. */
CAS_API cas_status cas_spmv_t(const cas_csr* a, cas_dtype dtype, const void* d_y, void* d_x, void* stream);
/* 1 / diag(A'A) with a duplicate of multiplicity m counting m^2
 * (JacobiPreconditionerOfATA, Math/MatrixCSR.cpp:21-47); empty columns give inf.
 * diag(A'A) is exact integers, counted when the matrix is built: on the
 * blocked layout from the FP32 transposed product of a vector of ones (exact
 * while every work item holds fewer than 2^24 entries) plus the repeated
 * (column, row) pairs, else directly from the sorted copy; the environment
 * variable CAS_DIAG_FROM_G32=1 selects the direct count for every build. */
CAS_API cas_status cas_jacobi(const cas_csr* a, cas_dtype dtype, void* d_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Differentiable evaluator: score = A w and its adjoint                     */
/* ------------------------------------------------------------------------ */

/* Rows per block of the BLOCKED layout (16384); minibatches of the evaluator
 * are whole blocks. */
CAS_API int64_t cas_block_rows(void);
/* Forward of the pattern evaluator on rows [row0, row1): score[i] = sum of
 * w over the row's columns, FP32 (ScoreEstimator::Eval of every position,
 * Pattern/Evaluator.cpp:48-54, for the CSR's index mode).  Needs BLOCKED. */
CAS_API cas_status cas_eval_forward(const cas_csr* a, int64_t row0, int64_t row1, const float* d_w, float* d_score,
                                    void* stream);
/* Adjoint: grad = A_rows' g for the rows [row0, row1) (block boundaries; row1
 * may be the last row); g has row1 - row0 entries, grad cols entries
 * (overwritten).  Computed on the per-block column-sorted copy:
 * deterministic, no atomics.  Needs BLOCKED. */
CAS_API cas_status cas_eval_backward(const cas_csr* a, int64_t row0, int64_t row1, const float* d_g, float* d_grad,
                                     void* stream);

/* One training step of the evaluator on a minibatch.  The reference fits
 * pattern weights by least squares only; this is the training form of its
 * score (Pattern/Evaluator.cpp:48-54 over the minibatch's rows) with the
 * objective mean Huber(score - target; delta) + l2 ||w||^2 and the update of
 * torch.optim.Adam (betas, eps; no weight decay). */
typedef struct cas_adam_opts {
    float lr, beta1, beta2, eps; /* Adam */
    float l2, delta;             /* L2 weight and Huber threshold of the objective */
} cas_adam_opts;
/* Rows [row0, row1) (block boundaries as for cas_eval_backward); d_target has
 * row1 - row0 entries; d_w, d_m, d_v (cols entries: weights and Adam
 * moments) are updated in place; *d_step (the Adam step count) is advanced;
 * the step's loss (weights before the update) is added to *d_loss_sum.  Three
 * kernels on `stream`, no host synchronisation and no allocation after the
 * first call of the largest minibatch, so it can be captured in a CUDA graph;
 * deterministic (fixed reduction orders, integer counters only).  The scratch
 * it (and cas_eval_backward) uses belongs to the CSR and grows when a call
 * spans more blocks than any call before.  Once a call has been captured
 * into a CUDA graph that scratch never moves: a later call (captured or not)
 * that would grow it returns CAS_ERR_INVALID_ARGUMENT, and so does a call
 * that would grow it while being captured.  The loss reduction and its
 * last-CTA counter are also one per CSR: calls on one CSR must be serialised
 * (one stream, or graphs replayed one after another); overlapping calls on
 * different streams corrupt each other's loss and counter. */
CAS_API cas_status cas_eval_adam_step(const cas_csr* a, int64_t row0, int64_t row1, const float* d_target,
                                      float* d_w, float* d_m, float* d_v, int64_t* d_step, double* d_loss_sum,
                                      const cas_adam_opts* opts, void* stream);

/* ------------------------------------------------------------------------ */
/* Solvers: PCG, LSQR, CG (Math/Solver.h)                                    */
/* ------------------------------------------------------------------------ */

typedef enum cas_method {
    CAS_PCG = 0,  /* Jacobi-PCG on A'A x = A'b (Math/Solver.h:78-117 as FitWeights calls it) */
    CAS_LSQR = 1, /* LSQR on min ||Ax - b|| (Math/Solver.h:128-182) */
    CAS_CG = 2,   /* PCG with the identity preconditioner (Math/Solver.h:40-76) */
    CAS_LSMR = 3  /* LSMR on min ||Ax - b|| (Math/Solver.h:222-287); its Residuum() is 0, as there */
} cas_method;

typedef enum cas_precision {
    /* FP64 vectors, FP64 products: the plain method. */
    CAS_PLAIN_FP64 = 0,
    /* FP32 sparse products and FP32 gather vectors (exact for the 0/1 entries
     * of A); FP64 accumulation, FP64 compensated dots/norms/scalars; the true
     * FP64 residual is recomputed every refine_every iterations. */
    CAS_MIXED = 1
} cas_precision;

typedef struct cas_solve_opts {
    cas_method method;
    cas_precision precision;
    double tol;         /* stop when ||A'(b-Ax)|| / ||A'b|| <= tol; <= 0: run max_iterations */
    int max_iterations;
    int refine_every;   /* CAS_MIXED PCG: most iterations between true-residual replacements (50).
                           CAS_MIXED LSQR/LSMR restart from the FP64 residual when their
                           recursive estimate of ||A'r|| has dropped 1e4-fold since the last
                           (re)start, or when a host check finds it off the true residual. */
    int check_every;    /* iterations per host-side convergence check (graph chunk) */
    int jacobi;         /* PCG: 1 = Jacobi preconditioner (FitWeights), 0 = none */
    int scale_columns;  /* LSQR/LSMR: 1 = iterate on A S with S = diag(A'A)^-1/2 (empty columns
                           scaled by 1) and return x = S y; 0 = the reference's unscaled
                           method (Math/Solver.h:128-287), the default.  Ignored by PCG/CG. */
} cas_solve_opts;

typedef struct cas_solve_report {
    int iterations;          /* iterations performed */
    int refinements;         /* true-residual recomputations performed */
    double rel_residual;     /* final ||A'(b-Ax)|| / ||A'b||, recomputed in FP64 */
    double residuum;         /* IterativeSolver::Residuum(): PCG r.r, LSQR phi_bar */
    double seconds;          /* device time of the solve (CUDA events) */
    double setup_seconds;    /* device time of indexing/CSR build (fit calls only) */
} cas_solve_report;

/* tol 1e-8, max_iterations 20000, refine_every 50, check_every 50, jacobi 1, PCG, FP64. */
CAS_API void cas_solve_opts_default(cas_solve_opts* o);

typedef struct cas_solver cas_solver;

/* Stateful solver mirroring IterativeSolver (Math/Solver.h:9-16).  For PCG
 * the system is A'A x = A'b with b the rows-length target vector, exactly
 * PCG(transposed(A) * A, P, x0, transposed(A) * b) of PatternFit.cpp:31.
 * d_x0 may be NULL (x0 = 0).  A must outlive the solver. */
CAS_API cas_status cas_solver_create(const cas_csr* a, const cas_solve_opts* o, const double* d_b,
                                     const double* d_x0, void* stream, cas_solver** out);
/* The same solver given the normal-equation right-hand side b' = A'b (cols
 * doubles, copied) instead of b: PCG(transposed(A) * A, P, x0, b') exactly as
 * the reference's caller writes it (PatternFit/PatternFit.cpp:31).  PCG and CG
 * only; residuals are then b' - A'A x. */
CAS_API cas_status cas_solver_create_normal(const cas_csr* a, const cas_solve_opts* o, const double* d_normal_b,
                                            const double* d_x0, void* stream, cas_solver** out);
/* PCG given the normal-equation right-hand side and an explicit diagonal
 * preconditioner d (cols doubles, copied; entries that are not normal act as
 * 1): PCG(transposed(A) * A, DiagonalPreconditioner(d), x0, b') with any
 * DiagonalPreconditioner, not only JacobiPreconditionerOfATA
 * (Math/Solver.h:25-38, :78-117).  o->method must be CAS_PCG; o->jacobi is
 * ignored. */
CAS_API cas_status cas_solver_create_normal_diag(const cas_csr* a, const cas_solve_opts* o, const double* d_normal_b,
                                                 const double* d_diag, const double* d_x0, void* stream,
                                                 cas_solver** out);
CAS_API void cas_solver_destroy(cas_solver* s);
/* IterativeSolver::Iterate(n). */
CAS_API cas_status cas_solver_iterate(cas_solver* s, int n);
/* IterativeSolver::Residuum(): PCG r.r of the recursive residual, LSQR phi_bar. */
CAS_API cas_status cas_solver_residuum(cas_solver* s, double* h_out);
/* IterativeSolver::X(): cols doubles into device memory. */
CAS_API cas_status cas_solver_x(cas_solver* s, double* d_out);
/* ||A'(b - Ax)|| / ||A'b|| of the current iterate, in FP64. */
CAS_API cas_status cas_solver_rel_residual(cas_solver* s, double* h_out);
/* Iterate until opts.tol or opts.max_iterations; fills the report. */
CAS_API cas_status cas_solver_run(cas_solver* s, cas_solve_report* rep);
CAS_API int cas_solver_iterations(const cas_solver* s);

/* Checkpoint and resume of an iterative solve (no counterpart in the
 * reference, whose solvers keep their state in host Vectors for one run):
 * the solver's device state -- the iterate, residual, preconditioned
 * residual and direction vectors, the bidiagonalisation vectors of
 * LSQR/LSMR (rows-length u included), the device scalars and flags -- as
 * one host byte buffer of cas_solver_state_size bytes (a header, then the
 * buffers).  A checkpoint loads into a solver created with the same method,
 * precision, column scaling and matrix shape (checked:
 * CAS_ERR_INVALID_ARGUMENT otherwise) on the same matrix and right-hand side
 * (not checked).  Iterating on from a loaded checkpoint gives bitwise the
 * iterates the saved solver would have produced, provided the products
 * run the same kernels: in one process, or, for FP32 products on the
 * blocked layout, with the same A'y schedule (CAS_ATY_SCHEDULE).  Both
 * calls synchronise the solver's stream. */
CAS_API cas_status cas_solver_state_size(const cas_solver* s, size_t* bytes);
CAS_API cas_status cas_solver_save_state(cas_solver* s, void* h_buf, size_t bytes);
CAS_API cas_status cas_solver_load_state(cas_solver* s, const void* h_buf, size_t bytes);

/* ------------------------------------------------------------------------ */
/* Batched fits: one problem per empty-count stage                           */
/* ------------------------------------------------------------------------ */

/* The independent per-stage fits of the training loop
 * (PatternFit/PatternFit.cpp:53-84 builds and fits one estimator per
 * empty-count stage, one after another; Pattern/Evaluator.cpp:77-88 keeps one
 * per stage) as one block-diagonal matrix in the BLOCKED layout: problem q is
 * rows [sum of h_problem_rows[0..q)) ...) of d_positions and owns columns
 * [q * C, (q + 1) * C), C = cas_patterns_cols(p).  1 to 64 problems; any
 * problem may be empty.  cas_spmv / cas_spmv_t / cas_jacobi work on it as on
 * any CSR (the products of the block-diagonal matrix). */
CAS_API cas_status cas_csr_from_positions_batched(const cas_patterns* p, const uint64_t* d_positions,
                                                  const int64_t* h_problem_rows, int problems, void* stream,
                                                  cas_csr** out);
/* Number of problems of a CSR (1 for a single fit); h_row0 (problems + 1
 * entries, may be null) receives each problem's first row and the total. */
CAS_API int cas_csr_problems(const cas_csr* a, int64_t* h_row0);
/* Solves every problem of a batched CSR with its own Jacobi-PCG (or CG)
 * (Math/Solver.h:78-117 per problem: own alpha, beta, residual and stopping
 * test) in one run: the products of an iteration cover all problems in one
 * launch each, problems that reach opts.tol are retired and skipped, and
 * iterations are replayed as CUDA graph chunks of opts.check_every.  d_b has
 * the rows of all problems, d_x receives problems * C weights; reports (may
 * be null) receives one report per problem (FP64 true relative residual).
 * Returns CAS_ERR_NOT_CONVERGED if any problem missed the tolerance. */
CAS_API cas_status cas_solve_batched(const cas_csr* a, const cas_solve_opts* o, const double* d_b, double* d_x,
                                     cas_solve_report* reports, void* stream);

/* One-shot solve: create, run, copy x, destroy. */
CAS_API cas_status cas_solve(const cas_csr* a, const cas_solve_opts* o, const double* d_b, double* d_x,
                             cas_solve_report* rep, void* stream);

/* ------------------------------------------------------------------------ */
/* FitWeights (PatternFit/PatternFit.cpp:7-39)                               */
/* ------------------------------------------------------------------------ */

/* Host buffers in, host weights out (cols floats); every step (upload,
 * indexing, CSR build, Jacobi, solve, download) runs on the device. */
CAS_API cas_status cas_fit_weights(const uint64_t* masks, int n_masks, cas_index_mode mode,
                                   const uint64_t* h_positions, const float* h_scores, int64_t rows,
                                   const cas_solve_opts* o, float* h_weights, cas_solve_report* rep);
/* Device-resident variant: scores and weights are FP64 device vectors. */
CAS_API cas_status cas_fit_weights_device(const cas_patterns* p, const uint64_t* d_positions, const double* d_scores,
                                          int64_t rows, const cas_solve_opts* o, double* d_weights,
                                          cas_solve_report* rep, void* stream);

/* The per-stage fits of the training loop (PatternFit/PatternFit.cpp:53-84:
 * one FitWeights per empty-count stage, one after another) as one batched
 * solve: problem q is the next h_problem_rows[q] positions and scores;
 * weights out are problems * cols floats (problem-major), reports one per
 * problem.  PCG and CG: one block-diagonal layout and one batched solve
 * (cas_csr_from_positions_batched + cas_solve_batched).  LSQR and LSMR: one
 * CSR and one solver per problem, each on its own stream, all run to
 * tolerance together (the host steps them in turn); each problem's result
 * is its single fit's.  A problem without rows gets zero weights.  The
 * first problem that did not converge sets the returned status. */
CAS_API cas_status cas_fit_weights_batched(const uint64_t* masks, int n_masks, cas_index_mode mode,
                                           const uint64_t* h_positions, const float* h_scores,
                                           const int64_t* h_problem_rows, int problems, const cas_solve_opts* o,
                                           float* h_weights, cas_solve_report* reports);
/* Device-resident variant: scores and weights are FP64 device vectors. */
CAS_API cas_status cas_fit_weights_batched_device(const cas_patterns* p, const uint64_t* d_positions,
                                                  const double* d_scores, const int64_t* h_problem_rows,
                                                  int problems, const cas_solve_opts* o, double* d_weights,
                                                  cas_solve_report* reports, void* stream);

/* ------------------------------------------------------------------------ */
/* Synthetic data (seeded, deterministic, identical on host and device)      */
/* ------------------------------------------------------------------------ */

/* Positions reached by uniform random legal play from the start position
 * (RandomPlayer semantics, Game/Player.cpp:3-16; passes are played, games
 * that end before the target are discarded and replayed).  The empty count
 * of position i is drawn uniformly from [min_empties, max_empties]. */
CAS_API cas_status cas_generate_positions(uint64_t seed, int64_t n, int min_empties, int max_empties,
                                          uint64_t* d_out, void* stream);
/* Same generator on the host CPU (for fixtures and cross-checks). */
CAS_API cas_status cas_generate_positions_host(uint64_t seed, int64_t first, int64_t n, int min_empties,
                                               int max_empties, uint64_t* h_out);
/* Targets b = clamp(2*rint((A w* + e)/2), -64, 64) with w* ~ N(0, w_sigma^2)
 * per column and e ~ N(0, noise_sigma^2) per row, seeded.  Optionally
 * returns w* (cols doubles, may be NULL). */
CAS_API cas_status cas_generate_targets(const cas_csr* a, uint64_t seed, double w_sigma, double noise_sigma,
                                        double* d_b, double* d_w_true, void* stream);
/* The same targets for a block of rows of a larger system: row r of `a` is
 * row first_row + r of the whole system (its noise is drawn from that row's
 * stream), so ranks that each hold a block of rows generate the whole
 * system's targets between them.  first_row = 0 is cas_generate_targets. */
CAS_API cas_status cas_generate_targets_rows(const cas_csr* a, uint64_t seed, double w_sigma, double noise_sigma,
                                             int64_t first_row, double* d_b, double* d_w_true, void* stream);

/* ------------------------------------------------------------------------ */
/* Pattern-based score estimators (Pattern/Evaluator.h, IO/Binary.cpp)       */
/* ------------------------------------------------------------------------ */

/* Stages(stage_size) (Pattern/Evaluator.cpp:6-9): ceil(65 / stage_size). */
CAS_API int cas_estimator_stages(int stage_size);
/* Save(PatternBasedEstimator) (IO/Binary.cpp:46-63) of the estimator whose
 * stage s (s < cas_estimator_stages(stage_size)) holds the dense weights
 * h_weights + s * C, C = the reference-mode column count of masks (the
 * layout FitWeights fits, PatternFit/PatternFit.cpp:7-39), and whose
 * accuracy model has the n_accuracy parameters (the reference's default
 * model has 5, Pattern/Evaluator.h AccuracyModel).  The bytes are those the
 * reference writes for ScoreEstimator(masks, weights) stages: the stored
 * patterns of CreateIndexer and ScoreEstimator::Weights(), size_t counts,
 * native byte order. */
CAS_API cas_status cas_estimator_save(const char* path, int stage_size, const uint64_t* masks, int n_masks,
                                      const float* h_weights, const float* accuracy, int n_accuracy);
/* LoadPatternBasedEstimator (IO/Binary.cpp:65-68), in two calls: the sizes,
 * then the stored patterns (n_masks), the weights of every stage (stages *
 * weights_per_stage floats) and the accuracy parameters (any pointer may be
 * NULL).  Files whose stages hold other patterns than the estimator are
 * rejected. */
CAS_API cas_status cas_estimator_file_info(const char* path, int* stage_size, int* n_masks, int* stages,
                                           int64_t* weights_per_stage, int* n_accuracy);
CAS_API cas_status cas_estimator_file_read(const char* path, uint64_t* h_masks, float* h_weights, float* h_accuracy);

/* A MultiStageScoreEstimator on the device (Pattern/Evaluator.cpp:11-29,
 * 77-83): d_weights holds cas_estimator_stages(stage_size) stages of dense
 * weights (C floats each, as above); every stage is expanded into one table
 * of 3^k floats per variation of every pattern, by a kernel. */
typedef struct cas_estimator cas_estimator;
CAS_API cas_status cas_estimator_create(const uint64_t* masks, int n_masks, int stage_size, const float* d_weights,
                                        void* stream, cas_estimator** out);
CAS_API void cas_estimator_destroy(cas_estimator* e);
CAS_API cas_status cas_estimator_info(const cas_estimator* e, int* stage_size, int* stages, int* n_masks,
                                      int64_t* weights_per_stage, int64_t* table_floats_per_stage);
/* Pattern(): CreateIndexer's stored pattern of every mask. */
CAS_API cas_status cas_estimator_patterns(const cas_estimator* e, uint64_t* h_out);
/* The expanded tables of one stage (table_floats_per_stage floats, variation
 * order). */
CAS_API cas_status cas_estimator_tables(const cas_estimator* e, int stage, float* d_out, void* stream);
/* MultiStageScoreEstimator::Eval (Pattern/Evaluator.cpp:48-54, 85-88) of n
 * positions ({P, O} uint64 pairs, 16-byte aligned): the FP32 sum in the
 * reference's order, bitwise its result.  A record with a square of both
 * players (not a position) scores NaN. */
CAS_API cas_status cas_estimator_eval(const cas_estimator* e, const uint64_t* d_positions, int64_t n, float* d_scores,
                                      void* stream);
/* ScoreEstimator::Weights() (Pattern/Evaluator.cpp:56-73) of one stage: C
 * dense floats. */
CAS_API cas_status cas_estimator_weights(const cas_estimator* e, int stage, float* d_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Training-data ingestion                                                   */
/* ------------------------------------------------------------------------ */

/* Binary '<QQb' records (NeuralNetwork/NeuralNetwork.py:21-29): 17 bytes
 * each, P and O little-endian uint64 then an int8 score, no header.  Reads up
 * to max_records into h_positions ({P, O} pairs) and h_scores; with both
 * NULL only counts the whole records of the file.  A trailing partial record
 * is not read (the reference's reader stops there). */
CAS_API cas_status cas_read_records(const char* path, uint64_t* h_positions, int8_t* h_scores, int64_t max_records,
                                    int64_t* n_records);
/* Text lines of ScoredPosition (LoadScoredPositionFile, IO/File.cpp:16-24;
 * ScoredPosition::FromString, Game/ScoredPosition.cpp:3-8): 64 board
 * characters, the side to move in column 65, the score (sign, digits,
 * halved, int8 as Score keeps it) from column 69.  Same calling convention
 * as cas_read_records; a line that is not a scored position is an error
 * naming the line. */
CAS_API cas_status cas_read_scored_positions(const char* path, uint64_t* h_positions, int8_t* h_scores,
                                             int64_t max_records, int64_t* n_records);

/* ------------------------------------------------------------------------ */
/* Allocation-free product                                                   */
/* ------------------------------------------------------------------------ */

/* No counterpart in the reference.  y = A x and *d_norm2 = ||y||^2, in FP64,
 * over caller-owned row-major indices (rows * nnz_per_row uint32 column
 * indices, each < cols) — the product and the norm the PCG step needs —
 * without allocating any device memory.  For callers that cannot let the
 * library allocate: device memory owned by another allocator or held to a
 * fixed budget, or a code path where cudaMalloc/cudaFree may not run because
 * they synchronise the device.  The per-CTA
 * partial sums live in a fixed 128 KB device array inside the library
 * (resident on every GPU that loads it until exit), which caps rows at
 * cas_spmv_norm_noalloc_max_rows() = 16,777,216; larger inputs are rejected
 * with CAS_ERR_INVALID_ARGUMENT.  The first call on a device looks up that
 * array's device address (no allocation); make it before any stream capture.
 * The lookup assumes the primary context and is not redone after
 * cudaDeviceReset.  Calls share the array: calls that overlap on the GPU race
 * and must be serialised by the caller.  The call is asynchronous, so an index
 * >= cols cannot be reported as a status: it is never read through, and it
 * makes its row's y and *d_norm2 NaN.  The result does not depend on the GPU
 * model (fixed 2048 rows per CTA). */
CAS_API int64_t cas_spmv_norm_noalloc_max_rows(void);
CAS_API cas_status cas_spmv_norm_noalloc(const uint32_t* d_indices, int nnz_per_row, int64_t rows, int64_t cols,
                                         const double* d_x, double* d_y, double* d_norm2, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CASSANDRA_B200_H */
