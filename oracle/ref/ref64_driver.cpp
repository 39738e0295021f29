// Test infrastructure only: the reference's Math/ sources (Vector.cpp,
// MatrixCSR.cpp, MatrixProxy.h, Solver.h) compiled where they lie with the
// scalar type retyped from float to double by a macro, so that the tests and
// the CPU baseline have an FP64 run of the reference's own PCG and LSQR.  The
// reference ships only the FP32 build, whose attainable residual is far above
// 1e-8.  The sources on disk are not modified; this file only wraps them.
//
// All standard headers that the reference includes are included first, so
// that the macro below touches only the reference's own code.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <functional>
#include <iostream>
#include <memory>
#include <numeric>
#include <omp.h>
#include <span>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#define float double
#include "Math/Vector.cpp"
#include "Math/MatrixCSR.cpp"
#include "Math/MatrixProxy.h"
#include "Math/Solver.h"
#undef float

namespace {
MatrixCSR make_csr(int k, int64_t rows, int64_t cols, const uint32_t* idx)
{
    MatrixCSR m(static_cast<size_t>(k), static_cast<size_t>(rows), static_cast<size_t>(cols));
    for (int64_t r = 0; r < rows; r++) std::memcpy(m.Row(r).data(), idx + r * k, sizeof(uint32_t) * k);
    return m;
}

// ||A'(b - A x)|| / ||A'b||, evaluated with the reference's own FP64 products.
double normal_residual(const MatrixCSR& m, const Vector& b, const Vector& x)
{
    Vector atb = b * m;
    Vector r = b - m * x;
    Vector atr = r * m;
    double d = norm(atb);
    return d > 0 ? norm(atr) / d : norm(atr);
}
}  // namespace

extern "C" {

// Math/MatrixCSR.cpp:49-65 in FP64
void ref64_spmv(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* x, double* y)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector r = m * Vector(x, x + cols);
    std::memcpy(y, r.data(), sizeof(double) * rows);
}

// Math/MatrixCSR.cpp:67-87 in FP64
void ref64_spmv_t(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* y, double* x)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector r = Vector(y, y + rows) * m;
    std::memcpy(x, r.data(), sizeof(double) * cols);
}

// Math/MatrixCSR.cpp:21-47 in FP64
void ref64_jacobi(int k, int64_t rows, int64_t cols, const uint32_t* idx, double* d)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector r = JacobiPreconditionerOfATA(m);
    std::memcpy(d, r.data(), sizeof(double) * cols);
}

// FitWeights' solve (PatternFit/PatternFit.cpp:24-32) in FP64.  Runs until the
// relative normal-equation residual is <= tol (checked every check_every
// iterations with the reference's products) or max_iterations is reached.
// Returns the iteration count; writes x, the final relative residual and the
// seconds spent (setup included, residual checks excluded).
int ref64_pcg(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int max_iterations,
              double tol, int check_every, double* x_out, double* rel_res, double* seconds)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector score(b, b + rows);
    double t0 = omp_get_wtime();
    double excluded = 0;
    DiagonalPreconditioner P(JacobiPreconditionerOfATA(m));
    PCG solver(transposed(m) * m, P, Vector(cols, 0.0), transposed(m) * score);
    int it = 0;
    double res = 1;
    while (it < max_iterations) {
        int n = std::min(check_every, max_iterations - it);
        solver.Iterate(n);
        it += n;
        if (tol > 0) {
            double c0 = omp_get_wtime();
            res = normal_residual(m, score, solver.X());
            excluded += omp_get_wtime() - c0;
            if (res <= tol) break;
        }
    }
    *seconds = omp_get_wtime() - t0 - excluded;
    Vector x = solver.X();
    std::memcpy(x_out, x.data(), sizeof(double) * cols);
    *rel_res = normal_residual(m, score, x);
    return it;
}

// LSQR (Math/Solver.h:128-182) in FP64, same stopping rule as ref64_pcg.
int ref64_lsqr(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int max_iterations,
               double tol, int check_every, double* x_out, double* rel_res, double* seconds)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector score(b, b + rows);
    double t0 = omp_get_wtime();
    double excluded = 0;
    LSQR solver(m, Vector(cols, 0.0), score);
    int it = 0;
    while (it < max_iterations) {
        int n = std::min(check_every, max_iterations - it);
        solver.Iterate(n);
        it += n;
        if (tol > 0) {
            double c0 = omp_get_wtime();
            double res = normal_residual(m, score, solver.X());
            excluded += omp_get_wtime() - c0;
            if (res <= tol) break;
        }
    }
    *seconds = omp_get_wtime() - t0 - excluded;
    Vector x = solver.X();
    std::memcpy(x_out, x.data(), sizeof(double) * cols);
    *rel_res = normal_residual(m, score, x);
    return it;
}

// LSMR (Math/Solver.h:222-287) in FP64, same stopping rule as ref64_pcg.
int ref64_lsmr(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int max_iterations,
               double tol, int check_every, double* x_out, double* rel_res, double* seconds)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector score(b, b + rows);
    double t0 = omp_get_wtime();
    double excluded = 0;
    LSMR solver(m, Vector(cols, 0.0), score);
    int it = 0;
    while (it < max_iterations) {
        int n = std::min(check_every, max_iterations - it);
        solver.Iterate(n);
        it += n;
        if (tol > 0) {
            double c0 = omp_get_wtime();
            double res = normal_residual(m, score, solver.X());
            excluded += omp_get_wtime() - c0;
            if (res <= tol) break;
        }
    }
    *seconds = omp_get_wtime() - t0 - excluded;
    Vector x = solver.X();
    std::memcpy(x_out, x.data(), sizeof(double) * cols);
    *rel_res = normal_residual(m, score, x);
    return it;
}

// The check of solutions computed elsewhere against the reference's own FP64
// products on one system: out[i] = ||A'(b - A x_i)|| / ||A'b|| for the n
// vectors x_i (cols doubles each, one after another), and hit[c] = 1 where
// column c has entries (JacobiPreconditionerOfATA finite).
void ref64_check(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int n, const double* xs,
                 double* out, uint8_t* hit)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector score(b, b + rows);
    for (int i = 0; i < n; i++) {
        const double* x = xs + static_cast<int64_t>(i) * cols;
        out[i] = normal_residual(m, score, Vector(x, x + cols));
    }
    if (hit) {
        Vector d = JacobiPreconditionerOfATA(m);
        for (int64_t c = 0; c < cols; c++) hit[c] = std::isfinite(d[c]) ? 1 : 0;
    }
}

// One PCG iteration's wall time in FP64 on a prebuilt system, averaged over n
// iterations (the bounded CPU-baseline sample).
double ref64_pcg_seconds_per_iteration(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b,
                                       int n)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector score(b, b + rows);
    DiagonalPreconditioner P(JacobiPreconditionerOfATA(m));
    PCG solver(transposed(m) * m, P, Vector(cols, 0.0), transposed(m) * score);
    solver.Iterate(1);
    double t0 = omp_get_wtime();
    solver.Iterate(n);
    return (omp_get_wtime() - t0) / n;
}

}  // extern "C"
