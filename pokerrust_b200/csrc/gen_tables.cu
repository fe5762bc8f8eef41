// Hand-rank tables for every river board of a flop, built on the device.
//
// Produces, per {turn, river} slot, the packed tables the reference's host builds and
// uploads every iteration (src/evaluator.rs:55-135 builds them with the `poker` crate,
// src/cuda_interface.rs:444-475 packs them): the rank-sorted order of the 1326 hands with
// tie-group flags and per-chunk group bounds (stored inverted: entry [hand] holds the
// hand's sorted position, entry [p] keeps position p's group flag), the per-card lists
// with new-group flags, and the percentile-hand-strength bucket of every hand
// (src/evaluator.rs:243-308, u32 arithmetic). One CTA per slot; the device re-pack
// (pack_boards.cu) then derives the river kernel's layout from these.
//
// Deck order: card = 13 * suit + rank, rank 0 = deuce.
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "gen_tables.h"
#include "hand_eval.cuh"
#include "layout.h"

namespace prb {
namespace {

constexpr int kEvalLen = 1326 + 512;
constexpr int kCollLen = 52 * 51;
constexpr int NT = 256;


__global__ void __launch_bounds__(NT) gen_tables_kernel(unsigned long long flop, uint16_t *__restrict__ eval,
                                                        uint16_t *__restrict__ coll,
                                                        uint16_t *__restrict__ abstr) {
    const int slot = blockIdx.x;
    const int tid = threadIdx.x;
    uint16_t *e = eval + (size_t)slot * kEvalLen;
    uint16_t *cv = coll + (size_t)slot * kCollLen;
    uint16_t *ab = abstr + (size_t)slot * kHands;
    int p1, p2;
    hand_cards(slot, &p1, &p2);
    const unsigned long long pair = (1ull << p1) | (1ull << p2);
    if (pair & flop) {
        // slots overlapping the flop stay zero (cuda_interface.rs:449-455)
        for (int i = tid; i < kEvalLen; i += NT) e[i] = 0;
        for (int i = tid; i < kCollLen; i += NT) cv[i] = 0;
        for (int i = tid; i < kHands; i += NT) ab[i] = 0;
        return;
    }
    const unsigned long long board = flop | pair;

    __shared__ unsigned long long key[2048];
    __shared__ uint16_t result[kEvalLen];  // sorted order with flags, then the chunk tables
    __shared__ uint16_t cards_of[kHands];
    __shared__ uint32_t phs[kHands];
    __shared__ uint16_t pos_of[kHands];

    // 1. value of every hand; blocked hands take the lowest value (Eval::WORST)
    for (int h = tid; h < 2048; h += NT) {
        if (h < kHands) {
            int c1, c2;
            hand_cards(h, &c1, &c2);
            cards_of[h] = (uint16_t)(c1 | (c2 << 8));
            const unsigned long long hm = (1ull << c1) | (1ull << c2);
            const uint32_t v = (hm & board) ? 0u : 1u + hand_value(hm | board);
            key[h] = ((unsigned long long)v << 11) | (unsigned long long)h;
        } else {
            key[h] = ~0ull;
        }
    }
    __syncthreads();
    // 2. bitonic sort by (value, hand index), ascending (evaluator.rs:80)
    for (int k = 2; k <= 2048; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < 2048; i += NT) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long a = key[i], b = key[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        key[i] = b;
                        key[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    // 3. flags and chunk group bounds (evaluator.rs:81-107), per-card lists
    //    (evaluator.rs:108-130) and phs buckets (evaluator.rs:243-308); short serial walks
    if (tid == 0) {
        uint32_t prev = 0;
        int last_group = 0;
        for (int s = 0; s < kHands; s++) {
            const uint32_t v = (uint32_t)(key[s] >> 11);
            int idx = (int)(key[s] & 2047);
            pos_of[idx] = (uint16_t)s;
            if (v > prev || s == 0) {
                prev = v;
                last_group = s;
                idx |= 2048;
            }
            if (s % 6 == 0) result[1326 + s / 6] = (uint16_t)last_group;
            result[s] = (uint16_t)idx;
        }
        for (int i = 1326 + 221; i < 1326 + 256; i++) result[i] = 0;
        int next_group = kHands;
        uint32_t prevb = 0xFFFFFFFFu;
        for (int s = kHands - 1; s >= 0; s--) {
            const uint32_t v = (uint32_t)(key[s] >> 11);
            if (v < prevb) {
                prevb = v;
                next_group = s + 1;
            }
            if (s % 6 == 5 || s == kHands - 1) result[1326 + 256 + s / 6] = (uint16_t)next_group;
        }
        for (int i = 1326 + 256 + 221; i < kEvalLen; i++) result[i] = 0;
    }
    if (tid == 32) {
        // per-card lists in sorted order; bit 2048 marks a new group for that card
        uint8_t fill[52];
        uint16_t card_group[52];
        for (int c = 0; c < 52; c++) fill[c] = card_group[c] = 0;
        int current_group = 0;
        uint32_t prev = 0;
        for (int s = 0; s < kHands; s++) {
            const uint32_t v = (uint32_t)(key[s] >> 11);
            if (v > prev || s == 0) {
                prev = v;
                current_group++;
            }
            const int h = (int)(key[s] & 2047);
            const int cs[2] = {cards_of[h] & 255, cards_of[h] >> 8};
            for (int k = 0; k < 2; k++) {
                const int c = cs[k];
                uint16_t val = (uint16_t)h;
                if (current_group > card_group[c]) {
                    card_group[c] = (uint16_t)current_group;
                    val |= 2048;
                }
                cv[c * 51 + fill[c]++] = val;
            }
        }
    }
    if (tid == 64) {
        // phs with the reference's wrapping u32 arithmetic
        uint32_t coll_tot[52], coll_cur[52];
        for (int c = 0; c < 52; c++) coll_tot[c] = coll_cur[c] = 0;
        for (int h = 0; h < kHands; h++) phs[h] = 0;
        uint32_t cumulative = 0;
        int s = 0;
        while (s < kHands) {
            const uint32_t v = (uint32_t)(key[s] >> 11);
            int en = s + 1;
            while (en < kHands && (uint32_t)(key[en] >> 11) == v) en++;
            uint32_t cur = 0;
            for (int q = s; q < en; q++) {
                const int h = (int)(key[q] & 2047);
                const int c1 = cards_of[h] & 255, c2 = cards_of[h] >> 8;
                if (((1ull << c1) | (1ull << c2)) & board) continue;
                phs[h] += cumulative;
                cur += 2;
                phs[h] -= coll_tot[c1];
                coll_cur[c1] += 2;
                phs[h] -= coll_tot[c2];
                coll_cur[c2] += 2;
            }
            for (int q = s; q < en; q++) {
                const int h = (int)(key[q] & 2047);
                const int c1 = cards_of[h] & 255, c2 = cards_of[h] >> 8;
                if (((1ull << c1) | (1ull << c2)) & board) continue;
                phs[h] += cur + 1;
                phs[h] -= coll_cur[c1];
                phs[h] -= coll_cur[c2];
            }
            cumulative += cur;
            for (int q = s; q < en; q++) {
                const int h = (int)(key[q] & 2047);
                const int c1 = cards_of[h] & 255, c2 = cards_of[h] >> 8;
                coll_tot[c1] += coll_cur[c1];
                coll_cur[c1] = 0;
                coll_tot[c2] += coll_cur[c2];
                coll_cur[c2] = 0;
            }
            s = en;
        }
    }
    __syncthreads();
    // 4. packed output: eval inverted (cuda_interface.rs:458-464), buckets
    for (int h = tid; h < kHands; h += NT) {
        e[h] = (uint16_t)((result[h] & 2048) | pos_of[h]);
        ab[h] = (uint16_t)((phs[h] * 256u) / (990u * 2u));
    }
    for (int i = kHands + tid; i < kEvalLen; i += NT) e[i] = result[i];
}

}  // namespace

cudaError_t launch_gen_tables(unsigned long long flop, uint16_t *eval, uint16_t *coll, uint16_t *abstr,
                              cudaStream_t stream) {
    gen_tables_kernel<<<kSlotsPerBoard, NT, 0, stream>>>(flop, eval, coll, abstr);
    return cudaGetLastError();
}

}  // namespace prb
