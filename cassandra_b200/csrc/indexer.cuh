// Device evaluation of the indexer recipes built by patterns.cpp: the
// ternary digits of a square list and the per-kind combination of
// Pattern/Indexer.cpp:17-317.
#pragma once
#include <cstdint>

#include "patterns.h"

namespace cas {

__device__ __forceinline__ uint32_t digits(const uint8_t* sq, int n, uint32_t plo, uint32_t phi, uint32_t olo,
                                           uint32_t ohi)
{
    uint32_t idx = 0;
    for (int i = n - 1; i >= 0; i--) {
        const int t = sq[i];
        const uint32_t pw = t < 32 ? plo : phi, ow = t < 32 ? olo : ohi;
        const int sh = t & 31;
        idx = idx * 3 + ((pw >> sh) & 1u) + (((ow >> sh) & 1u) << 1);
    }
    return idx;
}

__device__ __forceinline__ uint32_t eval_slot(const Instance& in, const uint32_t* __restrict__ tables, uint32_t plo,
                                              uint32_t phi, uint32_t olo, uint32_t ohi)
{
    uint32_t r;
    if (in.kind == kDirect) {
        r = digits(in.sq[0], in.n0, plo, phi, olo, ohi);
    } else if (in.kind == kTable) {
        r = __ldg(tables + in.table_offset + digits(in.sq[0], in.n0, plo, phi, olo, ohi));
    } else {
        uint32_t a = digits(in.sq[0], in.n0, plo, phi, olo, ohi);
        uint32_t b = digits(in.sq[1], in.n1, plo, phi, olo, ohi);
        const uint32_t lo = min(a, b), hi = max(a, b);
        r = lo * in.half_size + hi - (lo * (lo + 1) / 2);
        if (in.kind == kDiagPair) r = r * in.diag_size + digits(in.sq[2], in.n2, plo, phi, olo, ohi);
    }
    return in.offset + r;
}

}  // namespace cas
