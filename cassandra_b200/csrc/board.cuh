// Board arithmetic shared by host and device code: legal-move generation,
// disc flips and the counter-based random stream of the synthetic data
// generator.  Bit b is square (x = b & 7, y = b >> 3); bit 63 = A1 and
// bit 0 = H8 as in Board/Field.h:7-18.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define CAS_HD __host__ __device__ __forceinline__
#else
#define CAS_HD inline
#endif

namespace cas {

// Position::Start() (Board/Position.cpp:24-35): X on D5/E4, O on D4/E5,
// X to move.
constexpr uint64_t kStartP = 0x0000000810000000ULL;
constexpr uint64_t kStartO = 0x0000001008000000ULL;

constexpr uint64_t kNotX0 = 0xFEFEFEFEFEFEFEFEULL;  // clears x == 0 after a +x shift
constexpr uint64_t kNotX7 = 0x7F7F7F7F7F7F7F7FULL;  // clears x == 7 after a -x shift

// One step in direction d (0..7): +x, -x, +y, -y, +x+y, -x+y, +x-y, -x-y.
CAS_HD uint64_t step(uint64_t b, int d)
{
    switch (d) {
        case 0: return (b << 1) & kNotX0;
        case 1: return (b >> 1) & kNotX7;
        case 2: return b << 8;
        case 3: return b >> 8;
        case 4: return (b << 9) & kNotX0;
        case 5: return (b << 7) & kNotX7;
        case 6: return (b >> 7) & kNotX0;
        default: return (b >> 9) & kNotX7;
    }
}

// Squares where the side to move (p) can play: an empty square from which a
// line of one or more opponent discs ends in one of p's discs.
CAS_HD uint64_t legal_moves(uint64_t p, uint64_t o)
{
    uint64_t moves = 0;
#pragma unroll
    for (int d = 0; d < 8; d++) {
        uint64_t t = step(p, d) & o;
#pragma unroll
        for (int i = 0; i < 5; i++) t |= step(t, d) & o;
        moves |= step(t, d);
    }
    return moves & ~(p | o);
}

// Opponent discs turned by playing square m.
CAS_HD uint64_t turned_discs(uint64_t p, uint64_t o, int m)
{
    uint64_t all = 0;
#pragma unroll
    for (int d = 0; d < 8; d++) {
        uint64_t line = 0, x = step(1ULL << m, d);
        while (x & o) {
            line |= x;
            x = step(x, d);
        }
        if (x & p) all |= line;
    }
    return all;
}

CAS_HD int popcount64(uint64_t x)
{
#if defined(__CUDA_ARCH__)
    return __popcll(x);
#else
    return __builtin_popcountll(x);
#endif
}

CAS_HD int lowest_square(uint64_t x)
{
#if defined(__CUDA_ARCH__)
    return __ffsll(static_cast<long long>(x)) - 1;
#else
    return __builtin_ctzll(x);
#endif
}

// SplitMix64 (Steele, Lea, Flood 2014) as a counter-based stream: the state
// is advanced by the golden-ratio increment and mixed on output.
struct Stream {
    uint64_t s;
    CAS_HD static uint64_t mix(uint64_t z)
    {
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    CAS_HD Stream(uint64_t seed, uint64_t index) : s(mix(seed ^ mix(index + 0x632BE59BD9B4E019ULL))) {}
    CAS_HD uint64_t next()
    {
        s += 0x9E3779B97F4A7C15ULL;
        return mix(s);
    }
    // Uniform integer in [0, n) by the multiply-high method on 32 random bits.
    CAS_HD uint32_t below(uint32_t n) { return static_cast<uint32_t>(((next() >> 32) * n) >> 32); }
    // Uniform double in (0, 1).
    CAS_HD double unit() { return (static_cast<double>(next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
};

// Position i of the random-play generator: empty count uniform in
// [min_e, max_e]; uniform choice among the legal moves (RandomPlayer,
// Game/Player.cpp:3-16); a side without moves passes; a game that ends
// before reaching the target is discarded and replayed from the start with
// the stream continuing.  Returns false only if max_attempts were exhausted.
CAS_HD bool random_play_position(uint64_t seed, uint64_t i, int min_e, int max_e, uint64_t& out_p, uint64_t& out_o,
                                 int max_attempts = 1 << 16)
{
    Stream rng(seed, i);
    const int target = min_e + static_cast<int>(rng.below(static_cast<uint32_t>(max_e - min_e + 1)));
    for (int attempt = 0; attempt < max_attempts; attempt++) {
        uint64_t p = kStartP, o = kStartO;
        int empties = 60;
        bool ended = false;
        while (empties > target) {
            uint64_t moves = legal_moves(p, o);
            if (moves == 0) {
                if (legal_moves(o, p) == 0) {
                    ended = true;
                    break;
                }
                const uint64_t t = p;  // pass
                p = o;
                o = t;
                continue;
            }
            uint32_t k = rng.below(static_cast<uint32_t>(popcount64(moves)));
            while (k--) moves &= moves - 1;
            const int m = lowest_square(moves);
            const uint64_t f = turned_discs(p, o, m);
            const uint64_t np = o ^ f;
            o = p ^ f ^ (1ULL << m);
            p = np;
            empties--;
        }
        if (!ended) {
            out_p = p;
            out_o = o;
            return true;
        }
    }
    out_p = kStartP;
    out_o = kStartO;
    return false;
}

}  // namespace cas
