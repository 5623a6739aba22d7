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
__device__ __forceinline__ void myers_two_vectors(uint32_t p01, uint32_t p23, const uint32_t (&sel)[16],
                                                  uint32_t one, uint32_t two, uint32_t &pv, uint32_t &mv)
{
    pv = 0x7fff7fffu;
    mv = 0u;
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
}

// Hit flags ED < lim + L of the two columns.
template <int L>
__device__ __forceinline__ void myers_two(uint32_t p01, uint32_t p23, const uint32_t (&sel)[16], uint32_t one,
                                          uint32_t two, int lim, bool &h0, bool &h1)
{
    uint32_t pv, mv;
    myers_two_vectors<L>(p01, p23, sel, one, two, pv, mv);
    constexpr uint32_t M0 = (1u << L) - 1u;
    constexpr uint32_t M1 = M0 << 16;
    h0 = (__popc(pv & M0) - __popc(mv & M0)) < lim;
    h1 = (__popc(pv & M1) - __popc(mv & M1)) < lim;
}

// Exact distances of the two columns.
template <int L>
__device__ __forceinline__ void myers_two_dist(uint32_t p01, uint32_t p23, const uint32_t (&sel)[16], uint32_t one,
                                               uint32_t two, int &d0, int &d1)
{
    uint32_t pv, mv;
    myers_two_vectors<L>(p01, p23, sel, one, two, pv, mv);
    constexpr uint32_t M0 = (1u << L) - 1u;
    constexpr uint32_t M1 = M0 << 16;
    d0 = L + __popc(pv & M0) - __popc(mv & M0);
    d1 = L + __popc(pv & M1) - __popc(mv & M1);
}

// One-lane form (L = 16): bits >= 16 of Eq hold other masks' bytes; carries
// and shifts only move upwards, so they never reach the pattern rows.
template <int L>
__device__ __forceinline__ void myers_one_vectors(uint32_t p01, uint32_t p23, const uint32_t (&sel)[8], uint32_t one,
                                                  uint32_t two, uint32_t hi, uint32_t &pv, uint32_t &mv)
{
    pv = 0xffffffffu;
    mv = 0u;
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
}

template <int L>
__device__ __forceinline__ bool myers_one(uint32_t p01, uint32_t p23, const uint32_t (&sel)[8], uint32_t one,
                                          uint32_t two, uint32_t hi, int lim)
{
    uint32_t pv, mv;
    myers_one_vectors<L>(p01, p23, sel, one, two, hi, pv, mv);
    constexpr uint32_t M = (L >= 32) ? 0xffffffffu : ((1u << L) - 1u);
    return (__popc(pv & M) - __popc(mv & M)) < lim;
}

template <int L>
__device__ __forceinline__ int myers_one_dist(uint32_t p01, uint32_t p23, const uint32_t (&sel)[8], uint32_t one,
                                              uint32_t two, uint32_t hi)
{
    uint32_t pv, mv;
    myers_one_vectors<L>(p01, p23, sel, one, two, hi, pv, mv);
    constexpr uint32_t M = (L >= 32) ? 0xffffffffu : ((1u << L) - 1u);
    return L + __popc(pv & M) - __popc(mv & M);
}

// ---------------------------------------------------------------------------
// Banded lanes.  For a threshold k = min_ed - 1 the decision ED <= k between
// two equal-length strings only needs the diagonals |i - j| <= w, w = k/2
// (Ukkonen): a path that leaves them costs more than k.  Each column's band is
// a (2w+1)-bit vector, bit b <-> row i = j - w + b, and the recurrence is
// Myers' with the band re-aligned by one row per column:
//   D0 = (((Eq & VP) + VP) ^ VP) | Eq | VN          (carry out of the band dropped)
//   HN = VP & D0;  HP = VN | ~(D0 | VP)
//   Y  = D0 >> 1                                     (next column's alignment; 0 enters at the bottom)
//   VN = Y & HP;   VP = HN | ~(Y | HP)
// starting from VP = 1 on the band rows i >= 1 (rows <= 0 carry no delta) and
// VN = 0.  The centre bit b = w is the main diagonal: D[L][L] = L - sum_j D0_j[w].
// Many pair tests share one 32-bit word:
//  * kNib  (w <= 1, min_ed <= 4): eight 4-bit lanes, band bits 0..2, bit 3 spare
//    (two rows x four columns per thread)
//  * kByte (w <= 3, min_ed <= 8): four 8-bit lanes, band bits 0..6, bit 7 spare
// The spare bits of VP and Eq stay 0, so a lane's carry stops in its own spare
// bit; D0 is masked to the band before it is shifted.  Y is not masked: its
// spare bit may hold the next lane's bit 0, which reaches VN's spare bit only
// (HP's spare bit is always 1, so VP's stays 0) and is masked out of D0.
// Per character step kNib issues 11 ALU-pipe ops (1 PRMT, 8 LOP3, the add,
// the shift) and one IMAD (the lane counter, off the critical path) for eight
// pair tests (two rows x four columns), kByte the same for four (one row x
// four columns).  (Moving the add and the shift to the FMA pipe as IMAD /
// IMAD.HI, as an earlier form did, cut the ALU count to 9 but ran 7 % slower:
// IMAD.HI is half rate and both sit on the recurrence's critical path.)  The
// match masks of all lanes come from one PRMT on a window register W_j whose
// byte c is the band window of Peq[c] at column j (kNib: two rows' windows,
// one per nibble).  Lane counters of the centre bits (weight 2^w per byte)
// are compared with the threshold by adding 128 - 2^w (L - k) per byte and
// reading bit 7.
// ---------------------------------------------------------------------------
enum LaneMode : int { kModeFull = 0, kModeNib = 1, kModeByte = 2 };

// Column units of the banded modes: 4 columns each.  kNib: one 32-bit word
// per position (nibble l = char of column l in bits 0..15, bits 16..31 zero),
// 16 words.  kByte: 16 bits per position (nibble l = char of column l), two
// positions per word.
template <int MODE>
struct BandUnit {
    static constexpr int kCols = 4;                          // columns per unit
    static constexpr int kVec = MODE == kModeNib ? 4 : 2;    // uint4 per unit
    static constexpr int kBytes = kVec * 16;
    static constexpr int kTileCols = MODE == kModeNib ? 512 : 1024;  // columns per staged tile (8 KiB)
};

// Per-row band windows W_j, j = 0..L-1 (column j+1).
template <int L, int MODE>
__device__ __forceinline__ void band_windows(uint32_t word, int w, uint32_t (&W)[L])
{
    uint32_t pe[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int k = 0; k < L; ++k) {
        const uint32_t c = (word >> (2 * k)) & 3u;
        const uint32_t bit = 1u << k;
        pe[0] |= (c == 0u) ? bit : 0u;
        pe[1] |= (c == 1u) ? bit : 0u;
        pe[2] |= (c == 2u) ? bit : 0u;
        pe[3] |= (c == 3u) ? bit : 0u;
    }
    const uint32_t bandmask = (1u << (2 * w + 1)) - 1u;
#pragma unroll
    for (int j = 0; j < L; ++j) {
        const int sh = j - w;  // rows i = j + 1 - w + b  <->  Peq bit i - 1
        uint32_t x = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            uint32_t v = sh >= 0 ? (pe[c] >> sh) : (pe[c] << (-sh));
            x |= (v & bandmask) << (8 * c);
        }
        W[j] = x;
    }
}

struct BandConst {
    uint32_t vp0, bm, c, k;       // initial VP, band mask, centre mask, threshold constant
    uint32_t one, h16;            // opaque 1 and 2^16 (IMAD / IMAD.HI operands)
};

// Eight pair tests: two rows A, B of one thread against four columns.  W2[j]
// byte c holds row A's band window for character c in its low nibble and row
// B's in its high nibble, so one PRMT with the column selector (nibble k =
// character of column k at position j) yields all eight lanes: nibble 2k =
// (A, column k), nibble 2k+1 = (B, column k).  Hit flags at bit 8k+7 of he
// (row A) and ho (row B).
template <int L>
__device__ __forceinline__ void band_nib2(const uint32_t (&W2)[L], const uint32_t (&sel)[16], const BandConst &q,
                                          uint32_t &he, uint32_t &ho)
{
    uint32_t vp = q.vp0, vn = 0u, acc = 0u, be = 0u, bo = 0u;
#pragma unroll
    for (int j = 0; j < L; ++j) {
        const uint32_t eq = __byte_perm(W2[j], W2[j], sel[j]);
        const uint32_t sum = (eq & vp) + vp;
        const uint32_t d0 = ((sum ^ vp) | eq | vn) & q.bm;
        const uint32_t hn = vp & d0;
        const uint32_t hp = vn | ~(d0 | vp);
        acc = imad(d0 & q.c, q.one, acc);  // off the critical path: on the FMA pipe
        if ((j + 1) % 7 == 0 || j == L - 1) {  // nibble counters hold at most 7 steps of 2^w
            be = imad(acc & 0x0f0f0f0fu, q.one, be);
            bo = imad((acc >> 4) & 0x0f0f0f0fu, q.one, bo);
            acc = 0u;
        }
        const uint32_t ys = d0 >> 1;  // spare bits may pick up a neighbour's bit 0
        vn = ys & hp;
        vp = hn | ~(ys | hp);
    }
    he = (be + q.k) & 0x80808080u;
    ho = (bo + q.k) & 0x80808080u;
}

// Four pair tests (one row, four columns); hit flag of column l at bit 8l+7.
template <int L>
__device__ __forceinline__ uint32_t band_byte(const uint32_t (&W)[L], const uint32_t (&sel)[8], const BandConst &q)
{
    uint32_t vp = q.vp0, vn = 0u, acc = 0u;
#pragma unroll
    for (int j = 0; j < L; ++j) {
        const uint32_t s = (j & 1) ? __umulhi(sel[j >> 1], q.h16) : sel[j >> 1];
        const uint32_t eq = __byte_perm(W[j], W[j], s);
        const uint32_t sum = (eq & vp) + vp;
        const uint32_t d0 = ((sum ^ vp) | eq | vn) & q.bm;
        const uint32_t hn = vp & d0;
        const uint32_t hp = vn | ~(d0 | vp);
        acc = imad(d0 & q.c, q.one, acc);  // off the critical path: on the FMA pipe
        const uint32_t ys = d0 >> 1;
        vn = ys & hp;
        vp = hn | ~(ys | hp);
    }
    return imad(acc, q.one, q.k) & 0x80808080u;
}

// Per-job constants of the banded modes (host and device).
__host__ __device__ inline int band_mode(int len, int min_ed)
{
    (void)len;
    if (min_ed >= 1 && min_ed <= 4)
        return kModeNib;
    if (min_ed >= 5 && min_ed <= 8)
        return kModeByte;
    return kModeFull;
}

__host__ __device__ inline void band_constants(int len, int min_ed, int mode, int &w, uint32_t &vp0, uint32_t &bm,
                                               uint32_t &c, uint32_t &k)
{
    const int kk = min_ed - 1;
    w = kk / 2;
    const int B = 2 * w + 1;
    const uint32_t lane_bm = (1u << B) - 1u;
    const uint32_t lane_vp = lane_bm & ~((1u << w) - 1u);  // band rows i >= 1: bits w..2w
    const uint32_t rep = mode == kModeNib ? 0x11111111u : 0x01010101u;
    bm = lane_bm * rep;
    vp0 = lane_vp * rep;
    c = (1u << w) * rep;
    int thr = (1 << w) * (len - kk);
    if (thr < 0)
        thr = 0;
    k = (uint32_t)(128 - thr) * 0x01010101u;
}

}  // namespace myers
}  // namespace ig
