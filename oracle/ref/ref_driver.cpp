// Test infrastructure only: a thin extern "C" shim over the reference's own
// sources (compiled where they lie, unmodified) so that the Python tests can
// execute the reference's indexer, CSR products and solvers as the parity
// oracle.  Nothing in the shipped library links against this file.
//
// Every function forwards to the reference symbol named in its comment; the
// only logic restated here is FitWeights (PatternFit/PatternFit.cpp:12-38),
// which the reference defines without a header and next to code that pulls in
// its game-tree search.
#include "Board/Board.h"
#include "Pattern/Helpers.h"
#include "Pattern/Indexer.h"
#include "Math/Vector.h"
#include "Math/MatrixCSR.h"
#include "Math/MatrixProxy.h"
#include "Math/Solver.h"
#include <cstdint>
#include <cstring>
#include <span>
#include <vector>

namespace {
Position pos_at(const uint64_t* po, int64_t i) { return Position(po[2 * i], po[2 * i + 1]); }

MatrixCSR make_csr(int k, int64_t rows, int64_t cols, const uint32_t* idx)
{
    MatrixCSR m(static_cast<size_t>(k), static_cast<size_t>(rows), static_cast<size_t>(cols));
    for (int64_t r = 0; r < rows; r++) {
        auto row = m.Row(r);
        std::memcpy(row.data(), idx + r * k, sizeof(uint32_t) * k);
    }
    return m;
}
}  // namespace

extern "C" {

// Board/BitBoard.cpp:4-84
uint64_t ref_flip(int which, uint64_t b)
{
    switch (which) {
        case 0: return FlippedCodiagonal(b);
        case 1: return FlippedDiagonal(b);
        case 2: return FlippedHorizontal(b);
        case 3: return FlippedVertical(b);
    }
    return 0;
}

// Pattern/Helpers.cpp:44-47
uint32_t ref_fast_index(uint64_t p, uint64_t o, uint64_t mask) { return FastIndex(Position(p, o), mask); }

// Pattern/Indexer.cpp:319-365 (class choice, stored pattern, group order, index space)
void ref_create_indexer(uint64_t mask, uint64_t* stored_pattern, int* order, int* space)
{
    auto ix = CreateIndexer(mask);
    *stored_pattern = ix->pattern;
    *order = ix->symmetry_group_order;
    *space = ix->index_space_size;
}

// Pattern/Indexer.cpp:382-392 + Variations :394-403
int ref_group_info(const uint64_t* masks, int n, int64_t* cols, uint64_t* variations_out)
{
    GroupIndexer g(std::vector<uint64_t>(masks, masks + n));
    *cols = g.index_space_size;
    auto v = g.Variations();
    if (variations_out)
        for (size_t i = 0; i < v.size(); i++) variations_out[i] = v[i];
    return static_cast<int>(v.size());
}

// Pattern/Indexer.cpp:413-422, filled row by row as PatternFit/PatternFit.cpp:18-21 does
void ref_group_index(const uint64_t* masks, int n, const uint64_t* po, int64_t rows, uint32_t* out)
{
    GroupIndexer g(std::vector<uint64_t>(masks, masks + n));
    const int k = static_cast<int>(g.Variations().size());
#pragma omp parallel for
    for (int64_t i = 0; i < rows; i++)
        g.InsertIndices(pos_at(po, i), std::span<uint32_t>(out + i * k, k));
}

// The expanded layout composed of the reference's own public functions: the
// A_Indexer recipe (Pattern/Indexer.cpp:31-41: FastIndex of the 8 flipped
// positions against the unflipped mask) for every mask, column offsets the
// running sum of 3^k.  For an asymmetric mask this is CreateIndexer itself.
void ref_expanded_index(const uint64_t* masks, int n, const uint64_t* po, int64_t rows, uint32_t* out)
{
    std::vector<uint32_t> offset(n);
    uint32_t off = 0;
    for (int m = 0; m < n; m++) {
        offset[m] = off;
        off += static_cast<uint32_t>(pown(3, std::popcount(masks[m])));
    }
    const int k = 8 * n;
#pragma omp parallel for
    for (int64_t i = 0; i < rows; i++) {
        const Position pos = pos_at(po, i);
        const Position var[8] = {pos,
                                 FlippedCodiagonal(pos),
                                 FlippedDiagonal(pos),
                                 FlippedHorizontal(pos),
                                 FlippedVertical(pos),
                                 FlippedHorizontal(FlippedCodiagonal(pos)),
                                 FlippedHorizontal(FlippedDiagonal(pos)),
                                 FlippedHorizontal(FlippedVertical(pos))};
        uint32_t* row = out + i * k;
        for (int m = 0; m < n; m++)
            for (int s = 0; s < 8; s++) row[8 * m + s] = offset[m] + FastIndex(var[s], masks[m]);
    }
}

// Pattern/Indexer.h:19 Indices() of a single CreateIndexer indexer
int ref_indexer_indices(uint64_t mask, uint64_t p, uint64_t o, uint32_t* out)
{
    auto ix = CreateIndexer(mask);
    auto v = ix->Indices(Position(p, o));
    for (size_t i = 0; i < v.size(); i++) out[i] = v[i];
    return static_cast<int>(v.size());
}

// Board/PositionGenerator.cpp:4-14
void ref_random_positions(unsigned int seed, int64_t n, uint64_t* out)
{
    RandomPositionGenerator gen(seed);
    for (int64_t i = 0; i < n; i++) {
        Position p = gen();
        out[2 * i] = p.Player();
        out[2 * i + 1] = p.Opponent();
    }
}

// Pattern/Helpers.cpp:81-102 (enumeration order of Configurations)
int64_t ref_configurations(uint64_t mask, uint64_t* out)
{
    int64_t n = 0;
    for (Position c : Configurations(mask)) {
        if (out) {
            out[2 * n] = c.Player();
            out[2 * n + 1] = c.Opponent();
        }
        n++;
    }
    return n;
}

// Board/PossibleMoves.cpp, Board/Position.cpp:84-103
uint64_t ref_possible_moves(uint64_t p, uint64_t o) { return static_cast<uint64_t>(PossibleMoves(Position(p, o))); }
void ref_play(uint64_t p, uint64_t o, int move, uint64_t* out)
{
    Position r = Play(Position(p, o), static_cast<Field>(move));
    out[0] = r.Player();
    out[1] = r.Opponent();
}

// Math/MatrixCSR.cpp:49-65
void ref_spmv(int k, int64_t rows, int64_t cols, const uint32_t* idx, const float* x, float* y)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector r = m * Vector(x, x + cols);
    std::memcpy(y, r.data(), sizeof(float) * rows);
}

// Math/MatrixCSR.cpp:67-87
void ref_spmv_t(int k, int64_t rows, int64_t cols, const uint32_t* idx, const float* y, float* x)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector r = Vector(y, y + rows) * m;
    std::memcpy(x, r.data(), sizeof(float) * cols);
}

// Math/MatrixCSR.cpp:21-47
void ref_jacobi(int k, int64_t rows, int64_t cols, const uint32_t* idx, float* d)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector r = JacobiPreconditionerOfATA(m);
    std::memcpy(d, r.data(), sizeof(float) * cols);
}

// FitWeights (PatternFit/PatternFit.cpp:12-38) on a prebuilt CSR: Jacobi-PCG on
// A'A x = A'b from x0 = 0 (Math/Solver.h:78-117).  Writes x and Residuum().
void ref_pcg(int k, int64_t rows, int64_t cols, const uint32_t* idx, const float* b, int iterations,
             float* x_out, float* residuum)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    Vector score(b, b + rows);
    Vector weights(cols, 0.0f);
    DiagonalPreconditioner P(JacobiPreconditionerOfATA(m));
    PCG solver(transposed(m) * m, P, weights, transposed(m) * score);
    solver.Iterate(iterations);
    Vector x = solver.X();
    std::memcpy(x_out, x.data(), sizeof(float) * cols);
    *residuum = solver.Residuum();
}

// LSQR (Math/Solver.h:128-182) from x0 = 0.  Writes x and Residuum() (phi_bar).
void ref_lsqr(int k, int64_t rows, int64_t cols, const uint32_t* idx, const float* b, int iterations,
              float* x_out, float* residuum)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    LSQR solver(m, Vector(cols, 0.0f), Vector(b, b + rows));
    solver.Iterate(iterations);
    Vector x = solver.X();
    std::memcpy(x_out, x.data(), sizeof(float) * cols);
    *residuum = solver.Residuum();
}

}  // extern "C"
