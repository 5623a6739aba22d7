// Device building blocks of the pair test, shared by the kernels that run it:
// column-unit layout of the PRMT selector streams, the per-row match-mask
// pools and the two Myers recurrences (two 16-bit lanes for L <= 15, one lane
// for L = 16).  Used by the graph-building kernels and by the allocation-free
// conflict count.
#pragma once

#include <cstdint>

#include "ig_internal.h"

namespace ig {
namespace myers {

// ---------------------------------------------------------------------------
// Column streams.  A column "unit" is what a thread tests against its row in
// one inner step:
//  * L <= 15: two columns, one per 16-bit lane of a 32-bit word.  Stored as 16
//    32-bit selector words, one per character position; bits 0..15 hold the
//    PRMT nibbles (2a, 2a+1, 2b, 2b+1) of the two columns' characters a, b.
//  * L = 16: one column.  Stored as 16-bit selectors (2c, 2c+1, -, -), two
//    character positions per 32-bit word.
// With P01 = Peq0 | Peq1 << 16 and P23 = Peq2 | Peq3 << 16 (the row's Myers
// match masks), __byte_perm(P01, P23, sel) returns Peq[a] | Peq[b] << 16
// (resp. Peq[c] in the low half).
// ---------------------------------------------------------------------------
template <int L>
struct Unit {
    static constexpr bool kTwo = L <= 15;
    static constexpr int kCols = kTwo ? 2 : 1;      // columns per unit
    static constexpr int kVec = kTwo ? 4 : 2;       // uint4 per unit in the stream
    static constexpr int kUsed = kTwo ? (L + 3) / 4 : 2;  // uint4 read per unit
    static constexpr int kBytes = kVec * 16;
    static constexpr int kTileUnits = kTileCols / kCols;
};


__device__ __forceinline__ uint32_t nib(uint32_t c) { return (2u * c) | ((2u * c + 1u) << 4); }

template <int L>
__device__ __forceinline__ void row_pools(uint32_t w, uint32_t &p01, uint32_t &p23)
{
    // In the two-lane layout every mask carries bit 15, the lane separator.
    constexpr uint32_t sep = Unit<L>::kTwo ? 0x8000u : 0u;
    uint32_t m0 = sep, m1 = sep, m2 = sep, m3 = sep;
#pragma unroll
    for (int k = 0; k < L; ++k) {
        const uint32_t c = (w >> (2 * k)) & 3u;
        const uint32_t bit = 1u << k;
        m0 |= (c == 0u) ? bit : 0u;
        m1 |= (c == 1u) ? bit : 0u;
        m2 |= (c == 2u) ? bit : 0u;
        m3 |= (c == 3u) ? bit : 0u;
    }
    p01 = m0 | (m1 << 16);
    p23 = m2 | (m3 << 16);
}

// Integer multiply-add with an operand the compiler cannot see as a constant,
// so it stays an IMAD on the FMA pipe instead of a shift/add on the ALU pipe
// (the ALU pipe is the one the logic operations saturate).
__device__ __forceinline__ uint32_t imad(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// Myers' bit-vector recurrence in Hyyro's formulation (global alignment: the
// horizontal delta entering row 0 is +1):
//   Xv = Eq | Mv;  Xh = (((Eq & Pv) + Pv) ^ Pv) | Eq
//   Ph = Mv | ~(Xh | Pv);  Mh = Pv & Xh;  Ph <<= 1 (+1);  Mh <<= 1
//   Pv = Mh | ~(Xv | Ph);  Mv = Ph & Xv
// and the distance read at the end of the text as L + popc(Pv) - popc(Mv) over
// the pattern rows.  The add and both shifts run as IMADs.
//
// Two-lane form (L <= 15): lane 0 = bits 0..14, lane 1 = bits 16..30, 15
// pattern rows each (rows >= L never match); bits 15 and 31 separate them.
// Invariants that keep the lanes independent:
//   Eq has both separator bits set (every Peq mask carries bit 15),
//   Pv and Mv have both separator bits clear,
//   Mh has the top row (bits 14, 30) clear -- it could only shift into a separator.
// Then the carry of (Eq&Pv)+Pv stops at bit 15 (both addends are 0 there),
// Ph has bit 15 clear (Xh has it set, Mv not), so Ph*2 + 0x00010001 injects the
// +1 boundary into row 0 of both lanes without a carry, Mh*2 brings 0 into row 0
// of lane 1, and the new Pv has bit 15 clear because Xv has it set.
template <int L>
__device__ __forceinline__ void myers_two(uint32_t p01, uint32_t p23, const uint32_t (&sel)[16], uint32_t one,
                                          uint32_t two, int lim, bool &h0, bool &h1)
{
    uint32_t pv = 0x7fff7fffu, mv = 0u;
#pragma unroll
    for (int k = 0; k < L; ++k) {
        const uint32_t eq = __byte_perm(p01, p23, sel[k]);
        const uint32_t xv = eq | mv;
        const uint32_t s = imad(eq & pv, one, pv);
        const uint32_t xh = (s ^ pv) | eq;
        const uint32_t ph = mv | ~(xh | pv);
        const uint32_t mh = pv & xh & 0xbfffbfffu;
        const uint32_t ph2 = imad(ph, two, 0x00010001u);
        const uint32_t mh2 = imad(mh, two, 0u);
        pv = mh2 | ~(xv | ph2);
        mv = ph2 & xv & 0x7fff7fffu;
    }
    constexpr uint32_t M0 = (1u << L) - 1u;
    constexpr uint32_t M1 = M0 << 16;
    h0 = (__popc(pv & M0) - __popc(mv & M0)) < lim;
    h1 = (__popc(pv & M1) - __popc(mv & M1)) < lim;
}

// One-lane form (L = 16): bits >= 16 of Eq hold other masks' bytes; carries
// and shifts only move upwards, so they never reach the pattern rows.
template <int L>
__device__ __forceinline__ bool myers_one(uint32_t p01, uint32_t p23, const uint32_t (&sel)[8], uint32_t one,
                                          uint32_t two, uint32_t hi, int lim)
{
    uint32_t pv = 0xffffffffu, mv = 0u;
#pragma unroll
    for (int k = 0; k < L; ++k) {
        const uint32_t sw = (k & 1) ? __umulhi(sel[k >> 1], hi) : sel[k >> 1];
        const uint32_t eq = __byte_perm(p01, p23, sw);
        const uint32_t xv = eq | mv;
        const uint32_t s = imad(eq & pv, one, pv);
        const uint32_t xh = (s ^ pv) | eq;
        const uint32_t ph = mv | ~(xh | pv);
        const uint32_t mh = pv & xh;
        const uint32_t ph2 = imad(ph, two, 1u);
        const uint32_t mh2 = imad(mh, two, 0u);
        pv = mh2 | ~(xv | ph2);
        mv = ph2 & xv;
    }
    constexpr uint32_t M = (L >= 32) ? 0xffffffffu : ((1u << L) - 1u);
    return (__popc(pv & M) - __popc(mv & M)) < lim;
}

}  // namespace myers
}  // namespace ig
