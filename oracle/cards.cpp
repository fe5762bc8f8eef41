// Oracle (test infrastructure only): combinatorics and 7-card hand ranking.
//
// Colex indexing follows src/combination_map.rs:33-75 of the reference. Hand
// ranking restates the standard poker ordering that the third-party `poker`
// crate implements (called at src/evaluator.rs:46,75): straight flush > quads >
// full house > flush > straight > trips > two pair > pair > high card, ties
// broken by the ranks that make up the best five cards.
#include "oracle_internal.h"

#include <algorithm>
#include <thread>
#include <vector>

extern "C" int64_t or_choose(int n, int k) {
    // combination_map.rs:68-75
    if (k < 0 || n < k) return 0;
    int64_t r = 1;
    for (int i = 1; i <= k; i++) r = r * (n - k + i) / i;
    return r;
}

extern "C" int64_t or_colex_index(uint64_t set) {
    // combination_map.rs:33-42: sum over the c-th lowest set bit i of choose(i, c)
    int64_t res = 0;
    int c = 1;
    while (set) {
        int i = __builtin_ctzll(set);
        res += or_choose(i, c);
        set &= set - 1;
        c++;
    }
    return res;
}

extern "C" uint64_t or_pair_from_index(int index) {
    // inverse of the 2-subset colex index: index = a + b(b-1)/2, a < b
    int b = 1;
    while ((int64_t)(b + 1) * b / 2 <= index) b++;
    int a = index - b * (b - 1) / 2;
    return (1ull << a) | (1ull << b);
}

extern "C" void or_card_order(uint64_t *out) {
    // evaluator.rs:29-40: all 2-card masks sorted ascending, which is colex order
    int n = 0;
    for (int b = 1; b < 52; b++)
        for (int a = 0; a < b; a++) out[n++] = (1ull << a) | (1ull << b);
}

extern "C" void or_card_indexes(uint16_t *out) {
    // evaluator.rs:159-172: for each card, the 51 hand indexes that hold it, ascending
    uint64_t order[OR_HANDS];
    or_card_order(order);
    int fill[52] = {0};
    for (int i = 0; i < OR_HANDS; i++) {
        int c1, c2;
        or_separate(order[i], &c1, &c2);
        out[c1 * 51 + fill[c1]++] = (uint16_t)i;
        out[c2 * 51 + fill[c2]++] = (uint16_t)i;
    }
}

// Highest card rank of a five-in-a-row inside a 13-bit rank mask, or -1.
// The wheel A-2-3-4-5 counts with the five as its high card.
static int straight_high(uint32_t m) {
    for (int hi = 12; hi >= 4; hi--) {
        uint32_t w = 0x1Fu << (hi - 4);
        if ((m & w) == w) return hi;
    }
    if ((m & 0x100Fu) == 0x100Fu) return 3;
    return -1;
}

static inline uint32_t pack(int cat, const int *k, int nk) {
    uint32_t v = (uint32_t)cat << 20;
    for (int i = 0; i < nk; i++) v |= (uint32_t)k[i] << (16 - 4 * i);
    return v;
}

// Top `n` ranks of mask `m`, skipping ranks in `skip`.
static int top_ranks(uint32_t m, uint32_t skip, int n, int *out) {
    int got = 0;
    for (int r = 12; r >= 0 && got < n; r--)
        if ((m >> r & 1) && !(skip >> r & 1)) out[got++] = r;
    return got;
}

extern "C" uint32_t or_hand_value(uint64_t cards) {
    int cnt[13] = {0};
    uint32_t smask[4] = {0, 0, 0, 0};
    uint32_t rmask = 0;
    uint64_t c = cards;
    while (c) {
        int i = __builtin_ctzll(c);
        c &= c - 1;
        int r = or_rank(i), s = or_suit(i);
        cnt[r]++;
        smask[s] |= 1u << r;
        rmask |= 1u << r;
    }
    int k[5];
    int flush_suit = -1;
    for (int s = 0; s < 4; s++) {
        if (__builtin_popcount(smask[s]) >= 5) {
            flush_suit = s;
            int sh = straight_high(smask[s]);
            if (sh >= 0) {
                k[0] = sh;
                return pack(8, k, 1);
            }
        }
    }
    uint32_t quad = 0, trip = 0, pair = 0;
    for (int r = 0; r < 13; r++) {
        if (cnt[r] == 4) quad |= 1u << r;
        else if (cnt[r] == 3) trip |= 1u << r;
        else if (cnt[r] == 2) pair |= 1u << r;
    }
    if (quad) {
        int q = 31 - __builtin_clz(quad);
        k[0] = q;
        top_ranks(rmask, 1u << q, 1, k + 1);
        return pack(7, k, 2);
    }
    if (trip) {
        int t = 31 - __builtin_clz(trip);
        uint32_t rest = (trip & ~(1u << t)) | pair;
        if (rest) {
            k[0] = t;
            k[1] = 31 - __builtin_clz(rest);
            return pack(6, k, 2);
        }
    }
    if (flush_suit >= 0) {
        top_ranks(smask[flush_suit], 0, 5, k);
        return pack(5, k, 5);
    }
    int sh = straight_high(rmask);
    if (sh >= 0) {
        k[0] = sh;
        return pack(4, k, 1);
    }
    if (trip) {
        int t = 31 - __builtin_clz(trip);
        k[0] = t;
        top_ranks(rmask, 1u << t, 2, k + 1);
        return pack(3, k, 3);
    }
    if (__builtin_popcount(pair) >= 2) {
        int p1 = 31 - __builtin_clz(pair);
        int p2 = 31 - __builtin_clz(pair & ~(1u << p1));
        k[0] = p1;
        k[1] = p2;
        top_ranks(rmask, (1u << p1) | (1u << p2), 1, k + 2);
        return pack(2, k, 3);
    }
    if (pair) {
        int p = 31 - __builtin_clz(pair);
        k[0] = p;
        top_ranks(rmask, 1u << p, 3, k + 1);
        return pack(1, k, 4);
    }
    top_ranks(rmask, 0, 5, k);
    return pack(0, k, 5);
}

extern "C" void or_count_7card(int64_t *counts, int64_t *distinct, int nthreads) {
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    if (nthreads <= 0) nthreads = 1;
    // Work split over the highest card of the 7-set.
    std::vector<std::vector<int64_t>> part(nthreads, std::vector<int64_t>(9, 0));
    std::vector<std::vector<uint32_t>> seen(nthreads);
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) {
        th.emplace_back([&, t]() {
            std::vector<uint8_t> mark(1u << 24, 0);
            for (int g = 6 + t; g < 52; g += nthreads) {
                uint64_t top = 1ull << g;
                // enumerate 6-subsets of cards below g with Gosper's hack
                uint64_t s = (1ull << 6) - 1;
                uint64_t lim = 1ull << g;
                while (s < lim) {
                    uint32_t v = or_hand_value(s | top);
                    part[t][v >> 20]++;
                    mark[v] = 1;
                    uint64_t cc = s & (~s + 1), r = s + cc;
                    s = (((r ^ s) >> 2) / cc) | r;
                }
            }
            for (uint32_t v = 0; v < (1u << 24); v++)
                if (mark[v]) seen[t].push_back(v);
        });
    }
    for (auto &x : th) x.join();
    for (int i = 0; i < 9; i++) {
        counts[i] = 0;
        for (int t = 0; t < nthreads; t++) counts[i] += part[t][i];
    }
    std::vector<uint32_t> all;
    for (int t = 0; t < nthreads; t++) all.insert(all.end(), seen[t].begin(), seen[t].end());
    std::sort(all.begin(), all.end());
    *distinct = (int64_t)(std::unique(all.begin(), all.end()) - all.begin());
}
