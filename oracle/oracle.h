/*
 * Parity oracle (test infrastructure only): a plain-C, FP64 restatement of the
 * reference's fitting path, used by tests/ and by bench.py's CPU baseline to
 * check the CUDA library.  Nothing in the shipped library calls it.
 *
 * Pinned against the reference itself: tests/test_oracle.py compares every
 * function below with the reference sources compiled by oracle/Makefile
 * (oracle/_ref) and with the golden vectors committed under tests/golden/.
 */
#ifndef CAS_ORACLE_H
#define CAS_ORACLE_H
#include <stdint.h>

/* Board/BitBoard.cpp:4-84: 0 codiagonal, 1 diagonal, 2 horizontal, 3 vertical */
uint64_t or_flip(int which, uint64_t b);
/* Pattern/Helpers.cpp:44-47 */
uint32_t or_fast_index(uint64_t p, uint64_t o, uint64_t mask);

/* GroupIndexer (Pattern/Indexer.cpp:382-422), mode 0 = reference
 * (CreateIndexer per mask), mode 1 = expanded (A_Indexer recipe per mask).
 * Returns 0 on success; writes cols and entries per row. */
int or_group_info(const uint64_t* masks, int n, int mode, int64_t* cols, int* k);
/* Fills rows * k indices, row-major (PatternFit/PatternFit.cpp:18-21). */
int or_group_index(const uint64_t* masks, int n, int mode, const uint64_t* po, int64_t rows, uint32_t* out);

/* Math/MatrixCSR.cpp in FP64: y = A x, x = A'y, d = 1/diag(A'A) */
void or_spmv(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* x, double* y);
void or_spmv_t(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* y, double* x);
void or_jacobi(int k, int64_t rows, int64_t cols, const uint32_t* idx, double* d);

/* ||A'(b - Ax)|| / ||A'b|| */
double or_normal_residual(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, const double* x);

/* Math/Solver.h:78-117 (jacobi = 1: DiagonalPreconditioner of
 * JacobiPreconditionerOfATA; 0: identity, i.e. CG) on A'A x = A'b from x0 = 0,
 * FP64.  Runs `iterations` steps, or until the relative normal-equation
 * residual is <= tol when tol > 0 (checked every check_every steps).
 * Returns the steps taken; writes x and Residuum() (r.r). */
int or_pcg(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int jacobi, int iterations,
           double tol, int check_every, double* x, double* residuum);
/* Math/Solver.h:128-182 from x0 = 0, FP64; writes x and Residuum() (phi_bar). */
int or_lsmr(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int iterations, double tol,
            int check_every, double* x, double* zeta_bar);
int or_lsqr(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int iterations, double tol,
            int check_every, double* x, double* residuum);
/* The same two methods on A S with S = diag(A'A)^-1/2 (1 for an empty
 * column) when scale != 0, returning x = S y: column scaling, which the
 * reference does not have. */
int or_lsqr_scaled(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int scale,
                   int iterations, double tol, int check_every, double* x, double* residuum);
int or_lsmr_scaled(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int scale,
                   int iterations, double tol, int check_every, double* x, double* zeta_bar);

/* The library's seeded random-play positions {P, O} (index first .. first+n)
 * and targets b = clamp(2 rint((A w* + e) / 2), -64, 64), w* ~ N(0, w_sigma^2),
 * e ~ N(0, noise_sigma^2), from the same counter-based streams, for a process
 * that must not load the CUDA library.  0 on success. */
int or_generate_positions(uint64_t seed, int64_t first, int64_t n, int min_e, int max_e, uint64_t* po);
void or_generate_targets(int k, int64_t rows, int64_t cols, const uint32_t* idx, uint64_t seed, double w_sigma,
                         double noise_sigma, double* b, double* w_true);

#endif
