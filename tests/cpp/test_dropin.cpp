// The reference's own usage of its fitting API, compiled unchanged in shape
// against the drop-in header: MatrixCSR known answers
// (MathTest/MatrixCSR.cpp:3-55), the FitWeights sequence
// (PatternFit/PatternFit.cpp:12-38), PCG with another DiagonalPreconditioner,
// LSQR and LSMR (Math/Solver.h:78-287).
// Prints "OK <name>" per check and exits non-zero on the first failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "cassandra_b200.hpp"

using namespace cassandra_b200;

static int failures = 0;
#define EXPECT(cond, name)                                    \
    do {                                                      \
        if (cond) {                                           \
            std::printf("OK %s\n", name);                     \
        } else {                                              \
            std::printf("FAIL %s (%s:%d)\n", name, __FILE__, __LINE__); \
            failures++;                                       \
        }                                                     \
    } while (0)

static MatrixCSR CreateMatrix()
{
    // 1 1 0 0
    // 0 1 1 0
    // 0 0 0 2
    MatrixCSR m(2, 3, 4);
    m.Row(0)[0] = 0;
    m.Row(0)[1] = 1;
    m.Row(1)[0] = 1;
    m.Row(1)[1] = 2;
    m.Row(2)[0] = 3;
    m.Row(2)[1] = 3;
    return m;
}

int main()
{
    {
        MatrixCSR matrix = CreateMatrix();
        EXPECT(matrix.Rows() == 3 && matrix.Cols() == 4 && matrix.Row(0).size() == 2, "RowsAndCols");
        EXPECT((matrix * Vector({1, 2, 3, 4})) == Vector({3, 5, 8}), "MatrixVectorMultiplication");
        EXPECT((Vector({1, 2, 3}) * matrix) == Vector({1, 3, 2, 6}), "VectorMatrixMultiplication");
        EXPECT(JacobiPreconditionerOfATA(matrix) == Vector({1, 0.5, 1, 0.25}), "JacobiPreconditionerOfATA");
        bool thrown = false;
        try {
            matrix* Vector({1, 2, 3});
        } catch (const std::runtime_error& e) {
            thrown = std::string(e.what()) == "Size mismatch.";
        }
        EXPECT(thrown, "SizeMismatch");
    }
    {
        // FitWeights' sequence on a small pattern system (PatternFit/PatternFit.cpp:12-38)
        const std::vector<uint64_t> pattern{0x42FF, 0x070707, 0x1F1F, 0x8040201008040201, 0xFF00};
        const int rows = 3000;
        std::vector<uint64_t> pos(2 * rows);
        cas_generate_positions_host(5, 0, rows, 20, 40, pos.data());
        auto indexer = GroupIndexer(pattern);
        std::size_t elements_per_row = indexer.Variations().size();
        std::size_t cols = indexer.index_space_size;
        MatrixCSR matrix{elements_per_row, static_cast<std::size_t>(rows), cols};
        auto idx = indexer.Indices(pos);
        for (int i = 0; i < rows; i++)
            for (std::size_t k = 0; k < elements_per_row; k++) matrix.Row(i)[k] = idx[i * elements_per_row + k];
        Vector score(rows);
        for (int i = 0; i < rows; i++) score[i] = static_cast<float>(2 * ((i * 7919) % 33) - 32);

        Vector weights(cols, 0.0f);
        DiagonalPreconditioner P(JacobiPreconditionerOfATA(matrix));
        PCG solver(transposed(matrix) * matrix, P, weights, transposed(matrix) * score);
        const float r0 = solver.Residuum();
        solver.Iterate(10);
        Vector x = solver.X();
        EXPECT(x.size() == cols, "PCG X size");
        EXPECT(solver.Residuum() < r0, "PCG residuum decreases");
        Vector fw = FitWeights(pattern, pos, score, 10);
        float diff = 0, mx = 0;
        for (std::size_t i = 0; i < cols; i++) {
            diff = std::max(diff, std::fabs(fw[i] - x[i]));
            mx = std::max(mx, std::fabs(x[i]));
        }
        EXPECT(diff <= 1e-4f * mx, "FitWeights equals the explicit PCG sequence");
        Vector err = solver.Error();
        EXPECT(err.size() == cols, "PCG Error size");

        // A DiagonalPreconditioner other than Jacobi is honoured: with d = 1 the
        // PCG iterates are CG's (Math/Solver.h:40-76 and :78-117 with P = I).
        PCG pcg_identity(transposed(matrix) * matrix, DiagonalPreconditioner(Vector(cols, 1.0f)), weights,
                         transposed(matrix) * score);
        CG cg(transposed(matrix) * matrix, weights, transposed(matrix) * score);
        pcg_identity.Iterate(4);
        cg.Iterate(4);
        Vector xp = pcg_identity.X(), xc = cg.X();
        float dpc = 0, mpc = 0;
        for (std::size_t i = 0; i < cols; i++) {
            dpc = std::max(dpc, std::fabs(xp[i] - xc[i]));
            mpc = std::max(mpc, std::fabs(xc[i]));
        }
        EXPECT(dpc <= 1e-5f * mpc && mpc > 0, "PCG honours its DiagonalPreconditioner");
        EXPECT(std::fabs(pcg_identity.Residuum() - cg.Residuum()) <= 1e-4f * cg.Residuum(),
               "PCG with P = I has CG's residuum");
        struct Other : Preconditioner {
            Vector apply(const Vector& v) const override { return v; }
            Vector revert(const Vector& v) const override { return v; }
        };
        bool refused = false;
        try {
            PCG other(transposed(matrix) * matrix, Other{}, weights, transposed(matrix) * score);
        } catch (const std::invalid_argument&) {
            refused = true;
        }
        EXPECT(refused, "PCG refuses a preconditioner it cannot apply");

        LSQR lsqr(matrix, Vector(cols, 0.0f), score);
        lsqr.Iterate(5);
        Vector e = lsqr.Error();
        double n2 = 0, b2 = 0;
        for (int i = 0; i < rows; i++) {
            n2 += double(e[i]) * e[i];
            b2 += double(score[i]) * score[i];
        }
        EXPECT(std::fabs(std::sqrt(n2) - lsqr.Residuum()) <= 1e-3 * std::sqrt(b2), "LSQR Residuum is ||b - Ax||");

        // LSMR (Math/Solver.h:184-287): Residuum() is 0 as in the reference;
        // its residual ||b - Ax|| decreases from ||b||
        LSMR lsmr(matrix, Vector(cols, 0.0f), score);
        lsmr.Iterate(5);
        Vector el = lsmr.Error();
        double nl2 = 0;
        for (int i = 0; i < rows; i++) nl2 += double(el[i]) * el[i];
        EXPECT(lsmr.Residuum() == 0.0f, "LSMR Residuum is 0");
        EXPECT(std::sqrt(nl2) < std::sqrt(b2), "LSMR reduces ||b - Ax||");
    }
    std::printf(failures ? "FAILED %d\n" : "ALL OK\n", failures);
    return failures ? 1 : 0;
}
