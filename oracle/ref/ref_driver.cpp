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
#include "Pattern/Evaluator.h"
#include "IO/Binary.h"
#include "Game/ScoredPosition.h"
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

// A MatrixCSR kept across calls (one per minibatch of the evaluator's CPU
// baseline), and the same two products on it.
void* ref_csr_new(int k, int64_t rows, int64_t cols, const uint32_t* idx)
{
    return new MatrixCSR(make_csr(k, rows, cols, idx));
}

void ref_csr_free(void* m) { delete static_cast<MatrixCSR*>(m); }

// Math/MatrixCSR.cpp:49-65
void ref_csr_mul(const void* pm, const float* x, float* y)
{
    const MatrixCSR& m = *static_cast<const MatrixCSR*>(pm);
    Vector r = m * Vector(x, x + m.Cols());
    std::memcpy(y, r.data(), sizeof(float) * m.Rows());
}

// Math/MatrixCSR.cpp:67-87
void ref_csr_tmul(const void* pm, const float* y, float* x)
{
    const MatrixCSR& m = *static_cast<const MatrixCSR*>(pm);
    Vector r = Vector(y, y + m.Rows()) * m;
    std::memcpy(x, r.data(), sizeof(float) * m.Cols());
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

// LSMR (Math/Solver.h:222-287) from x0 = 0.  Writes x; *residuum receives
// the reference's Residuum(), which is 0 for LSMR (:284).
void ref_lsmr(int k, int64_t rows, int64_t cols, const uint32_t* idx, const float* b, int iterations,
              float* x_out, float* residuum)
{
    MatrixCSR m = make_csr(k, rows, cols, idx);
    LSMR solver(m, Vector(cols, 0.0f), Vector(b, b + rows));
    solver.Iterate(iterations);
    Vector x = solver.X();
    std::memcpy(x_out, x.data(), sizeof(float) * cols);
    *residuum = solver.Residuum();
}

// ScoreEstimator(pattern, weights) (Pattern/Evaluator.cpp:11-29) and its
// Eval (:48-54) on every position.
void ref_estimator_eval(const uint64_t* masks, int n, const float* weights, int64_t n_weights, const uint64_t* po,
                        int64_t rows, float* out)
{
    ScoreEstimator se(std::vector<uint64_t>(masks, masks + n), std::span<const float>(weights, n_weights));
    for (int64_t i = 0; i < rows; i++) out[i] = se.Eval(pos_at(po, i));
}

// ScoreEstimator::Weights() (Pattern/Evaluator.cpp:56-73) of the estimator
// built from dense weights: writes n_weights floats.
void ref_estimator_weights(const uint64_t* masks, int n, const float* weights, int64_t n_weights, float* out)
{
    ScoreEstimator se(std::vector<uint64_t>(masks, masks + n), std::span<const float>(weights, n_weights));
    const std::vector<float> w = se.Weights();
    std::memcpy(out, w.data(), sizeof(float) * std::min<size_t>(w.size(), static_cast<size_t>(n_weights)));
}

// MultiStageScoreEstimator (Pattern/Evaluator.cpp:77-88) whose stage s holds
// ScoreEstimator(pattern, weights + s * n_weights); Eval of every position.
void ref_msse_eval(int stage_size, const uint64_t* masks, int n, const float* weights, int64_t n_weights,
                   const uint64_t* po, int64_t rows, float* out)
{
    std::vector<uint64_t> pattern(masks, masks + n);
    MultiStageScoreEstimator msse(stage_size, pattern);
    for (size_t s = 0; s < msse.estimators.size(); s++)
        msse.estimators[s] = ScoreEstimator(pattern, std::span<const float>(weights + s * n_weights, n_weights));
    for (int64_t i = 0; i < rows; i++) out[i] = msse.Eval(pos_at(po, i));
}

// Save(PatternBasedEstimator) (IO/Binary.cpp:46-63) of the estimator whose
// stage s holds the dense weights weights + s * n_weights.
void ref_save_estimator(const char* path, int stage_size, const uint64_t* masks, int n, const float* weights,
                        int64_t n_weights, const float* accuracy, int n_accuracy)
{
    std::vector<uint64_t> pattern(masks, masks + n);
    MultiStageScoreEstimator msse(stage_size, pattern);
    for (size_t s = 0; s < msse.estimators.size(); s++)
        msse.estimators[s] = ScoreEstimator(pattern, std::span<const float>(weights + s * n_weights, n_weights));
    PatternBasedEstimator pbe(std::move(msse), AccuracyModel(std::vector<float>(accuracy, accuracy + n_accuracy)));
    Save(pbe, std::filesystem::path(path));
}

// LoadPatternBasedEstimator (IO/Binary.cpp:65-68): stage size, stages,
// masks (up to max_masks), each stage's Weights() (up to max_weights floats
// per stage) and the accuracy parameters (up to 8).  Returns the number of
// masks.
int ref_load_estimator(const char* path, int* stage_size, int* stages, uint64_t* masks, int max_masks, float* weights,
                       int64_t max_weights, float* accuracy, int* n_accuracy)
{
    const PatternBasedEstimator pbe = LoadPatternBasedEstimator(std::filesystem::path(path));
    *stage_size = pbe.StageSize();
    *stages = pbe.Stages();
    const std::vector<uint64_t> pattern = pbe.Pattern();
    for (size_t i = 0; i < pattern.size() && static_cast<int>(i) < max_masks; i++) masks[i] = pattern[i];
    for (int s = 0; s < pbe.Stages(); s++) {
        const std::vector<float> w = pbe.score.estimators[s].Weights();
        std::memcpy(weights + s * max_weights, w.data(), sizeof(float) * std::min<size_t>(w.size(), max_weights));
    }
    const std::vector<float>& a = pbe.accuracy.ParameterValues();
    *n_accuracy = static_cast<int>(a.size());
    for (size_t i = 0; i < a.size() && i < 8; i++) accuracy[i] = a[i];
    return static_cast<int>(pattern.size());
}

// ScoredPosition::FromString (Game/ScoredPosition.cpp:3-8) of one text line:
// 0 on success, 1 if the reference throws.
int ref_parse_scored_position(const char* line, uint64_t* p, uint64_t* o, int* score)
{
    try {
        const ScoredPosition sp = ScoredPosition::FromString(std::string_view(line));
        *p = sp.pos.Player();
        *o = sp.pos.Opponent();
        *score = static_cast<int>(sp.score);
        return 0;
    } catch (...) {
        return 1;
    }
}

// to_string(ScoredPosition) (Game/ScoredPosition.cpp:20-23) into out (at
// least 80 bytes): the line the reference writes for a position and score.
void ref_format_scored_position(uint64_t p, uint64_t o, int score, char* out)
{
    const std::string s = to_string(ScoredPosition{Position(p, o), Score(score)});
    std::memcpy(out, s.c_str(), s.size() + 1);
}

}  // extern "C"
