// Pattern sets: host-side construction of the per-instance index recipes
// that the indexer kernel evaluates.
//
// Every index the reference computes is a combination of FastIndex values
// (Pattern/Helpers.cpp:44-47): FastIndex(G(pos), m) with G one of the board
// symmetries and m a (sub)mask.  Digit i of FastIndex is the state of G(pos)
// at the i-th set bit of m (LSB first), i.e. the state of pos at the square
// that G moves there.  The host therefore resolves every (G, m) pair into a
// list of source squares once, and the device evaluates
//     digits(list) = sum_i 3^i * cell(pos, list[i]),  cell = empty 0, P 1, O 2
// for each list, then combines the lists as the reference's indexer class
// does (Pattern/Indexer.cpp:17-317).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cassandra_b200.h"

namespace cas {

// Board symmetries on bitboards, bit b = square (x = b & 7, y = b >> 3).
// The mappings are those of Board/BitBoard.cpp:4-84 (pinned by
// BoardTest/BitBoard.cpp:6-24): codiagonal (x,y)->(7-y,7-x), diagonal
// (x,y)->(y,x), horizontal (x,y)->(7-x,y), vertical (x,y)->(x,7-y).
enum Flip : int { kCodiagonal = 0, kDiagonal = 1, kHorizontal = 2, kVertical = 3 };
uint64_t flipped(int which, uint64_t b);
inline uint64_t flipped_c(uint64_t b) { return flipped(kCodiagonal, b); }
inline uint64_t flipped_d(uint64_t b) { return flipped(kDiagonal, b); }
inline uint64_t flipped_h(uint64_t b) { return flipped(kHorizontal, b); }
inline uint64_t flipped_v(uint64_t b) { return flipped(kVertical, b); }

// FastIndex on the host (Pattern/Helpers.cpp:44-47), by its definition.
uint32_t fast_index(uint64_t p, uint64_t o, uint64_t mask);

// Kinds of instance recipes the kernel evaluates.
enum InstanceKind : uint8_t {
    kDirect = 0,    // A_Indexer: digits(list0)
    kPair = 1,      // V_Indexer: unordered pair {digits(list0), digits(list1)}
    kDiagPair = 2,  // D_Indexer: pair of half digits, times diag size, plus digits(list2)
    kTable = 3      // VH/DC/VHDC: dense orbit table over digits(list0)
};

constexpr int kMaxSquares = 16;

// One CSR slot's recipe.  Plain data, copied to the device verbatim.
struct Instance {
    uint8_t kind;
    uint8_t n0, n1, n2;          // lengths of the three square lists
    uint32_t offset;             // column offset of the pattern's block
    uint32_t half_size;          // kPair/kDiagPair: 3^popcount(mask & half)
    uint32_t diag_size;          // kDiagPair: 3^popcount(mask & diag)
    uint32_t table_offset;       // kTable: start of the dense table
    uint8_t sq[3][kMaxSquares];  // source squares, digit order
};
static_assert(sizeof(Instance) == 68, "Instance layout");

// Indexer facts of one input mask (mirrors CreateIndexer's result).
struct IndexerInfo {
    uint64_t input_mask;
    uint64_t stored_pattern;  // Indexer::pattern (CreateIndexer may flip it)
    int kind;                 // InstanceKind of its instances
    int order;                // symmetry_group_order
    int64_t space;            // index_space_size
    int64_t offset;           // column offset of its block
};

struct PatternSet {
    cas_index_mode mode;
    std::vector<uint64_t> masks;
    std::vector<IndexerInfo> indexers;
    std::vector<Instance> instances;     // one per CSR slot, slot order
    std::vector<uint64_t> variations;    // GroupIndexer::Variations()
    std::vector<int> slot_indexer;       // indexer of each slot
    std::vector<uint32_t> tables;        // concatenated dense tables
    int64_t cols = 0;
};

// Builds the recipes; returns false with a message on unusable masks.
bool build_pattern_set(const uint64_t* masks, int n, cas_index_mode mode, PatternSet& out, std::string& err);

// Evaluates slot `s` of a pattern set for one position on the host (used by
// the host-side checks; the device kernel does the same arithmetic).
uint32_t eval_instance_host(const PatternSet& ps, int s, uint64_t p, uint64_t o);

}  // namespace cas
