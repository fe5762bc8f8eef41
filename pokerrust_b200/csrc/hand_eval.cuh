// Seven-card hand values on the device (deck order: card = 13 * suit + rank, rank 0 = deuce).
#pragma once
#include <stdint.h>

namespace prb {

__device__ __forceinline__ int top_bit(uint32_t m) { return 31 - __clz(m); }

// Highest rank of a five-card run in a 13-bit rank mask (the wheel counts as five-high),
// or -1.
__device__ __forceinline__ int straight_high(uint32_t m) {
    // bit r of run5 is set when ranks r-4 .. r are all present
    uint32_t run5 = m & (m << 1) & (m << 2) & (m << 3) & (m << 4);
    if (run5) return top_bit(run5);
    const uint32_t wheel = (1u << 12) | 0xFu;  // A 2 3 4 5
    return (m & wheel) == wheel ? 3 : -1;
}

// Value of the best five-card hand among 5..7 cards: category << 20 | ranks in decreasing
// significance, 4 bits each. Larger is better; equal values are ties.
__device__ __forceinline__ uint32_t hand_value(unsigned long long cards) {
    uint32_t s[4];
#pragma unroll
    for (int k = 0; k < 4; k++) s[k] = (uint32_t)(cards >> (13 * k)) & 0x1FFFu;
    const uint32_t all = s[0] | s[1] | s[2] | s[3];
    // flushes and straight flushes
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (__popc(s[k]) >= 5) {
            const int sf = straight_high(s[k]);
            if (sf >= 0) return (8u << 20) | ((uint32_t)sf << 16);
        }
    }
    const uint32_t quads = s[0] & s[1] & s[2] & s[3];
    const uint32_t three = (s[0] & s[1] & s[2]) | (s[0] & s[1] & s[3]) | (s[0] & s[2] & s[3]) |
                           (s[1] & s[2] & s[3]);
    const uint32_t two = (s[0] & s[1]) | (s[0] & s[2]) | (s[0] & s[3]) | (s[1] & s[2]) |
                         (s[1] & s[3]) | (s[2] & s[3]);
    const uint32_t trips = three & ~quads;
    const uint32_t pairs = two & ~three;
    uint32_t v;
    if (quads) {
        const int q = top_bit(quads);
        return (7u << 20) | ((uint32_t)q << 16) | ((uint32_t)top_bit(all & ~(1u << q)) << 12);
    }
    if (trips) {
        const int t = top_bit(trips);
        const uint32_t rest = (trips & ~(1u << t)) | pairs;
        if (rest) return (6u << 20) | ((uint32_t)t << 16) | ((uint32_t)top_bit(rest) << 12);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (__popc(s[k]) >= 5) {
            uint32_t m = s[k];
            v = 5u << 20;
#pragma unroll
            for (int i = 0; i < 5; i++) {
                const int r = top_bit(m);
                v |= (uint32_t)r << (16 - 4 * i);
                m &= ~(1u << r);
            }
            return v;
        }
    }
    const int st = straight_high(all);
    if (st >= 0) return (4u << 20) | ((uint32_t)st << 16);
    if (trips) {
        const int t = top_bit(trips);
        uint32_t m = all & ~(1u << t);
        const int k1 = top_bit(m);
        m &= ~(1u << k1);
        return (3u << 20) | ((uint32_t)t << 16) | ((uint32_t)k1 << 12) | ((uint32_t)top_bit(m) << 8);
    }
    if (__popc(pairs) >= 2) {
        const int p1 = top_bit(pairs);
        const int p2 = top_bit(pairs & ~(1u << p1));
        const int k = top_bit(all & ~(1u << p1) & ~(1u << p2));
        return (2u << 20) | ((uint32_t)p1 << 16) | ((uint32_t)p2 << 12) | ((uint32_t)k << 8);
    }
    if (pairs) {
        const int p = top_bit(pairs);
        uint32_t m = all & ~(1u << p);
        v = (1u << 20) | ((uint32_t)p << 16);
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const int r = top_bit(m);
            v |= (uint32_t)r << (12 - 4 * i);
            m &= ~(1u << r);
        }
        return v;
    }
    uint32_t m = all;
    v = 0;
#pragma unroll
    for (int i = 0; i < 5; i++) {
        const int r = top_bit(m);
        v |= (uint32_t)r << (16 - 4 * i);
        m &= ~(1u << r);
    }
    return v;
}

}  // namespace prb
