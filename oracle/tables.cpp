// Oracle (test infrastructure only): per-board hand-rank tables and their GPU packing.
//
// or_board_tables restates the per-board closure of src/evaluator.rs:60-135 and the
// bucket abstraction src/evaluator.rs:243-308; or_pack_flop_tables restates
// src/cuda_interface.rs:48-102 (including the "inverse eval" permutation of :458-464).
#include "oracle_internal.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <utility>
#include <vector>

void or_parallel_for(int n, int nthreads, const std::function<void(int)> &f) {
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    if (nthreads <= 1 || n <= 1) {
        for (int i = 0; i < n; i++) f(i);
        return;
    }
    std::vector<std::thread> th;
    std::atomic_int next(0);
    for (int t = 0; t < std::min(nthreads, n); t++)
        th.emplace_back([&]() {
            for (int i; (i = next.fetch_add(1)) < n;) f(i);
        });
    for (auto &x : th) x.join();
}

// evaluator.rs:243-308, with the reference's u32 wrapping arithmetic kept.
static void phs(const uint16_t *sorted, const uint64_t *card_order, uint64_t board,
                uint16_t *out) {
    const uint32_t M = OR_BUCKETS;
    std::vector<std::vector<int>> groups;
    std::vector<int> current{sorted[0] & 2047};
    for (int i = 1; i < OR_HANDS; i++) {
        if (sorted[i] & 2048) {
            groups.push_back(current);
            current.clear();
        }
        current.push_back(sorted[i] & 2047);
    }
    groups.push_back(current);

    uint32_t collisions[52] = {0};
    uint32_t cumulative = 0;
    uint32_t result[OR_HANDS] = {0};
    for (auto &group : groups) {
        uint32_t current_cumulative = 0;
        uint32_t current_collisions[52] = {0};
        for (int index : group) {
            uint64_t cards = card_order[index];
            if (cards & board) continue;
            int c[2];
            or_separate(cards, &c[0], &c[1]);
            result[index] += cumulative;
            current_cumulative += 2;
            for (int k = 0; k < 2; k++) {
                result[index] -= collisions[c[k]];
                current_collisions[c[k]] += 2;
            }
        }
        for (int index : group) {
            uint64_t cards = card_order[index];
            if (cards & board) continue;
            int c[2];
            or_separate(cards, &c[0], &c[1]);
            result[index] += current_cumulative + 1;  // +1: inclusion-exclusion of the hand itself
            for (int k = 0; k < 2; k++) result[index] -= current_collisions[c[k]];
        }
        cumulative += current_cumulative;
        for (int i = 0; i < 52; i++) collisions[i] += current_collisions[i];
    }
    for (int i = 0; i < OR_HANDS; i++) out[i] = (uint16_t)((result[i] * M) / (990u * 2u));
}

extern "C" void or_board_tables(uint64_t board, uint16_t *result, uint16_t *coll_vec,
                                uint16_t *abstr) {
    uint64_t card_order[OR_HANDS];
    or_card_order(card_order);
    std::memset(result, 0, sizeof(uint16_t) * OR_EVAL_LEN);
    std::memset(coll_vec, 0, sizeof(uint16_t) * OR_COLL_LEN);
    // evaluator.rs:64-80: blocked hands rank as Eval::WORST (0 here, below every real
    // hand value), then sort by (value, index).
    std::vector<std::pair<uint32_t, int>> evals(OR_HANDS);
    for (int i = 0; i < OR_HANDS; i++) {
        uint32_t v = (card_order[i] & board) ? 0u : or_hand_value(card_order[i] | board);
        evals[i] = {v, i};
    }
    std::sort(evals.begin(), evals.end());
    // evaluator.rs:81-94: group-start flag 2048 and the per-chunk group starts.
    uint32_t prev_eval = 0;
    int last_group = 0;
    for (int s = 0; s < OR_HANDS; s++) {
        uint32_t eval = evals[s].first;
        int index = evals[s].second;
        if (eval > prev_eval || s == 0) {
            prev_eval = eval;
            last_group = s;
            index |= 2048;
        }
        if (s % 6 == 0) result[1326 + s / 6] = (uint16_t)last_group;
        result[s] = (uint16_t)index;
    }
    // evaluator.rs:95-107: the next group after each chunk, walking from the best hand.
    int next_group = 1326;
    uint32_t prev = 0xFFFFFFFFu;  // Eval::BEST bound
    for (int s = OR_HANDS - 1; s >= 0; s--) {
        uint32_t eval = evals[s].first;
        if (eval < prev) {
            prev = eval;
            next_group = s + 1;
        }
        if (s % 6 == 5 || s == 1325) result[1326 + 256 + s / 6] = (uint16_t)next_group;
    }
    // evaluator.rs:108-130: per-card lists in sorted order with new-group flags.
    int indexes[52] = {0};
    int card_group[52] = {0};
    int current_group = 0;
    for (int i = 0; i < OR_HANDS; i++) {
        uint16_t si = result[i];
        if (si & 2048) current_group++;
        si &= 2047;
        int c[2];
        or_separate(card_order[si], &c[0], &c[1]);
        for (int k = 0; k < 2; k++) {
            uint16_t val = si;
            if (current_group > card_group[c[k]]) {
                card_group[c[k]] = current_group;
                val |= 2048;
            }
            coll_vec[c[k] * 51 + indexes[c[k]]++] = val;
        }
    }
    phs(result, card_order, board, abstr);
}

extern "C" void or_pack_flop_tables(uint64_t flop, uint16_t *eval, uint16_t *coll,
                                    uint16_t *abstr, int nthreads) {
    // cuda_interface.rs:444-475: slot j = colex index of the 2-card set; slots that
    // overlap the flop stay zero; the eval block is stored "inverted" so that
    // eval[hand] & 2047 is the hand's sorted position and eval[p] & 2048 is the
    // group-start flag of sorted position p.
    or_parallel_for(OR_HANDS, nthreads, [&](int j) {
        uint64_t cards = or_pair_from_index(j);
        uint16_t *e = eval + (size_t)j * OR_EVAL_LEN;
        uint16_t *c = coll + (size_t)j * OR_COLL_LEN;
        uint16_t *a = abstr + (size_t)j * OR_HANDS;
        if (cards & flop) {
            std::memset(e, 0, sizeof(uint16_t) * OR_EVAL_LEN);
            std::memset(c, 0, sizeof(uint16_t) * OR_COLL_LEN);
            std::memset(a, 0, sizeof(uint16_t) * OR_HANDS);
            return;
        }
        std::vector<uint16_t> sorted(OR_EVAL_LEN);
        or_board_tables(flop | cards, sorted.data(), c, a);
        std::memcpy(e, sorted.data(), sizeof(uint16_t) * OR_EVAL_LEN);
        for (int i = 0; i < OR_HANDS; i++) {
            int h = sorted[i] & 2047;
            e[h] &= 2048;
            e[h] |= (uint16_t)i;
        }
    });
}
