// Host-side construction of pattern sets (see patterns.h).
#include "patterns.h"

#include <algorithm>
#include <bit>
#include <cstdio>

namespace cas {

namespace {

constexpr uint64_t kLowerHalf = 0x00000000FFFFFFFFULL;      // V_Indexer half (Pattern/Indexer.cpp:61)
constexpr uint64_t kStrictLower = 0x0080C0E0F0F8FCFEULL;    // D_Indexer half (Pattern/Indexer.cpp:104)
constexpr uint64_t kDiagonalLine = 0x8040201008040201ULL;   // D_Indexer diag (Pattern/Indexer.cpp:105)

int square_after(int which, int b)
{
    const int x = b & 7, y = b >> 3;
    switch (which) {
        case kCodiagonal: return (7 - x) * 8 + (7 - y);
        case kDiagonal: return x * 8 + y;
        case kHorizontal: return y * 8 + (7 - x);
        default: return (7 - y) * 8 + x;
    }
}

uint64_t pow3(int e)
{
    uint64_t r = 1;
    while (e-- > 0) r *= 3;
    return r;
}

uint64_t pdep(uint64_t src, uint64_t mask)
{
    uint64_t r = 0;
    for (int i = 0; mask; i++, mask &= mask - 1)
        if ((src >> i) & 1) r |= mask & (0 - mask);
    return r;
}

struct Pos {
    uint64_t p, o;
};
Pos flip_pos(int which, Pos a) { return {flipped(which, a.p), flipped(which, a.o)}; }

// A transform is a list of flips applied in order (first element first).
using Transform = std::vector<int>;

uint64_t apply_transform(const Transform& g, uint64_t b)
{
    for (int f : g) b = flipped(f, b);
    return b;
}

// Source squares of FastIndex(G(pos), m): digit i reads pos at the square
// that G moves onto the i-th set bit of m.
bool source_squares(uint64_t m, const Transform& g, uint8_t* out, uint8_t& n)
{
    n = 0;
    for (uint64_t bits = m; bits; bits &= bits - 1) {
        const int s = std::countr_zero(bits);
        int src = -1;
        for (int t = 0; t < 64; t++)
            if (apply_transform(g, 1ULL << t) == (1ULL << s)) {
                src = t;
                break;
            }
        if (src < 0 || n >= kMaxSquares) return false;
        out[n++] = static_cast<uint8_t>(src);
    }
    return true;
}

Transform then(Transform g, int f)
{
    g.push_back(f);
    return g;
}

// Configurations(mask) in the reference's enumeration order
// (Pattern/Helpers.cpp:81-102): p outer, o inner, p & o == 0, deposited.
template <typename F>
void for_each_configuration(uint64_t mask, F&& f)
{
    const uint64_t size = 1ULL << std::popcount(mask);
    for (uint64_t p = 0; p < size; p++)
        for (uint64_t o = 0; o < size; o++)
            if ((p & o) == 0) f(Pos{pdep(p, mask), pdep(o, mask)});
}

// Dense orbit table of a VH/DC/VHDC pattern (Pattern/Indexer.cpp:153-178,
// 207-230, 261-293): configurations in enumeration order, each new orbit
// gets the next index.
uint32_t build_dense_table(uint64_t m, const std::vector<Transform>& orbit, std::vector<uint32_t>& table)
{
    table.assign(pow3(std::popcount(m)), 0xFFFFFFFFu);
    uint32_t index = 0;
    for_each_configuration(m, [&](Pos c) {
        if (table[fast_index(c.p, c.o, m)] != 0xFFFFFFFFu) return;
        for (const Transform& g : orbit) {
            Pos v{apply_transform(g, c.p), apply_transform(g, c.o)};
            table[fast_index(v.p, v.o, m)] = index;
        }
        index++;
    });
    return index;
}

const std::vector<Transform> kAInstances = {{}, {kCodiagonal}, {kDiagonal}, {kHorizontal}, {kVertical},
                                            {kCodiagonal, kHorizontal}, {kDiagonal, kHorizontal},
                                            {kVertical, kHorizontal}};

std::vector<uint64_t> a_variations(uint64_t m)
{
    // Pattern/Indexer.cpp:43-55 (note C(H(m)) etc.: H applied first here)
    return {m, flipped_c(m), flipped_d(m), flipped_h(m), flipped_v(m),
            flipped_c(flipped_h(m)), flipped_d(flipped_h(m)), flipped_v(flipped_h(m))};
}

}  // namespace

uint64_t flipped(int which, uint64_t b)
{
    uint64_t r = 0;
    for (; b; b &= b - 1) r |= 1ULL << square_after(which, std::countr_zero(b));
    return r;
}

uint32_t fast_index(uint64_t p, uint64_t o, uint64_t mask)
{
    uint32_t idx = 0, w = 1;
    for (; mask; mask &= mask - 1, w *= 3) {
        const uint64_t bit = mask & (0 - mask);
        idx += (p & bit) ? w : ((o & bit) ? 2 * w : 0);
    }
    return idx;
}

bool build_pattern_set(const uint64_t* masks, int n, cas_index_mode mode, PatternSet& ps, std::string& err)
{
    ps = PatternSet{};
    ps.mode = mode;
    if (n <= 0) {
        err = "pattern set needs at least one mask";
        return false;
    }
    int64_t offset = 0;
    for (int i = 0; i < n; i++) {
        const uint64_t m = masks[i];
        const int k = std::popcount(m);
        if (m == 0 || k > kMaxSquares) {
            char buf[128];
            std::snprintf(buf, sizeof buf, "mask %d (0x%016llx) has %d squares; 1..16 are supported", i,
                          static_cast<unsigned long long>(m), k);
            err = buf;
            return false;
        }
        ps.masks.push_back(m);
        IndexerInfo info{m, m, kDirect, 8, 0, offset};
        std::vector<Instance> inst;
        std::vector<uint64_t> vars;

        auto direct = [&](uint64_t mm, const Transform& g) {
            Instance s{};
            s.kind = kDirect;
            if (!source_squares(mm, g, s.sq[0], s.n0)) return false;
            inst.push_back(s);
            return true;
        };
        auto pair = [&](uint64_t mm, const Transform& g) {
            Instance s{};
            s.kind = kPair;
            s.half_size = static_cast<uint32_t>(pow3(std::popcount(mm & kLowerHalf)));
            if (!source_squares(mm & kLowerHalf, g, s.sq[0], s.n0)) return false;
            if (!source_squares(mm & kLowerHalf, then(g, kVertical), s.sq[1], s.n1)) return false;
            inst.push_back(s);
            return true;
        };
        auto diag_pair = [&](uint64_t mm, const Transform& g) {
            Instance s{};
            s.kind = kDiagPair;
            s.half_size = static_cast<uint32_t>(pow3(std::popcount(mm & kStrictLower)));
            s.diag_size = static_cast<uint32_t>(pow3(std::popcount(mm & kDiagonalLine)));
            if (!source_squares(mm & kStrictLower, g, s.sq[0], s.n0)) return false;
            if (!source_squares(mm & kStrictLower, then(g, kDiagonal), s.sq[1], s.n1)) return false;
            if (!source_squares(mm & kDiagonalLine, g, s.sq[2], s.n2)) return false;
            inst.push_back(s);
            return true;
        };
        auto table = [&](uint64_t mm, const Transform& g, uint32_t table_offset) {
            Instance s{};
            s.kind = kTable;
            s.table_offset = table_offset;
            if (!source_squares(mm, g, s.sq[0], s.n0)) return false;
            inst.push_back(s);
            return true;
        };

        bool ok = true;
        if (mode == CAS_INDEX_EXPANDED) {
            info.space = static_cast<int64_t>(pow3(k));
            for (const Transform& g : kAInstances) ok = ok && direct(m, g);
            vars = a_variations(m);
        } else {
            // CreateIndexer's classification (Pattern/Indexer.cpp:343-364).
            const bool v = flipped_v(m) == m, h = flipped_h(m) == m;
            const bool d = flipped_d(m) == m, c = flipped_c(m) == m;
            std::vector<uint32_t> dense;
            if ((v && h && d && c) || (v && h) || (d && c)) {
                std::vector<Transform> orbit, inst_g;
                if (v && h && d && c) {
                    orbit = kAInstances;
                    orbit[5] = {kHorizontal, kCodiagonal};  // var6 = C(H(config)) (Pattern/Indexer.cpp:279-281)
                    orbit[6] = {kHorizontal, kDiagonal};
                    orbit[7] = {kHorizontal, kVertical};
                    inst_g = {{}};
                    vars = {m};
                    info.order = 1;
                } else if (v && h) {
                    orbit = {{}, {kVertical}, {kHorizontal}, {kVertical, kHorizontal}};
                    inst_g = {{}, {kDiagonal}};
                    vars = {m, flipped_d(m)};
                    info.order = 2;
                } else {
                    orbit = {{}, {kDiagonal}, {kCodiagonal}, {kDiagonal, kCodiagonal}};
                    inst_g = {{}, {kVertical}};
                    vars = {m, flipped_v(m)};
                    info.order = 2;
                }
                info.kind = kTable;
                info.space = build_dense_table(m, orbit, dense);
                const uint32_t toff = static_cast<uint32_t>(ps.tables.size());
                ps.tables.insert(ps.tables.end(), dense.begin(), dense.end());
                for (const Transform& g : inst_g) ok = ok && table(m, g, toff);
            } else if (v || h) {
                const uint64_t mm = v ? m : flipped_d(m);  // h-only: V_Indexer(FlippedDiagonal(p))
                info.stored_pattern = mm;
                info.kind = kPair;
                info.order = 4;
                const int64_t hs = static_cast<int64_t>(pow3(std::popcount(mm & kLowerHalf)));
                info.space = hs * (hs + 1) / 2;
                for (const Transform& g : std::vector<Transform>{{}, {kCodiagonal}, {kDiagonal}, {kHorizontal}})
                    ok = ok && pair(mm, g);
                vars = {mm, flipped_c(mm), flipped_d(mm), flipped_h(mm)};
            } else if (d || c) {
                const uint64_t mm = d ? m : flipped_v(m);  // c-only: D_Indexer(FlippedVertical(p))
                info.stored_pattern = mm;
                info.kind = kDiagPair;
                info.order = 4;
                const int64_t hs = static_cast<int64_t>(pow3(std::popcount(mm & kStrictLower)));
                const int64_t ds = static_cast<int64_t>(pow3(std::popcount(mm & kDiagonalLine)));
                info.space = ds * hs * (hs + 1) / 2;
                for (const Transform& g : std::vector<Transform>{{}, {kCodiagonal}, {kHorizontal}, {kVertical}})
                    ok = ok && diag_pair(mm, g);
                vars = {mm, flipped_c(mm), flipped_h(mm), flipped_v(mm)};
            } else {
                info.space = static_cast<int64_t>(pow3(k));
                for (const Transform& g : kAInstances) ok = ok && direct(m, g);
                vars = a_variations(m);
            }
        }
        if (!ok) {
            err = "could not resolve the squares of a pattern instance";
            return false;
        }
        for (Instance& s : inst) s.offset = static_cast<uint32_t>(offset);
        const int idx = static_cast<int>(ps.indexers.size());
        for (size_t j = 0; j < inst.size(); j++) ps.slot_indexer.push_back(idx);
        ps.instances.insert(ps.instances.end(), inst.begin(), inst.end());
        ps.variations.insert(ps.variations.end(), vars.begin(), vars.end());
        ps.indexers.push_back(info);
        offset += info.space;
        if (offset > 0xFFFFFFFFLL) {
            err = "total index space exceeds 2^32 columns";
            return false;
        }
    }
    ps.cols = offset;
    return true;
}

uint32_t eval_instance_host(const PatternSet& ps, int s, uint64_t p, uint64_t o)
{
    const Instance& in = ps.instances[s];
    auto digits = [&](int l, int n) {
        uint32_t idx = 0;
        for (int i = n - 1; i >= 0; i--) {
            const int t = in.sq[l][i];
            idx = idx * 3 + static_cast<uint32_t>(((p >> t) & 1) + 2 * ((o >> t) & 1));
        }
        return idx;
    };
    uint32_t r = 0;
    switch (in.kind) {
        case kDirect: r = digits(0, in.n0); break;
        case kPair:
        case kDiagPair: {
            uint32_t a = digits(0, in.n0), b = digits(1, in.n1);
            if (a > b) std::swap(a, b);
            r = a * in.half_size + b - (a * (a + 1) / 2);
            if (in.kind == kDiagPair) r = r * in.diag_size + digits(2, in.n2);
            break;
        }
        default: r = ps.tables[in.table_offset + digits(0, in.n0)]; break;
    }
    return in.offset + r;
}

}  // namespace cas
