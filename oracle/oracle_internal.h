// Oracle (test infrastructure only): shared internal helpers.
#ifndef POKERRUST_ORACLE_INTERNAL_H
#define POKERRUST_ORACLE_INTERNAL_H

#include "oracle.h"

#include <functional>

// evaluator.rs:234-242: the two card numbers of a hand, lower first.
static inline void or_separate(uint64_t cards, int *c1, int *c2) {
    *c1 = __builtin_ctzll(cards);
    cards &= cards - 1;
    *c2 = __builtin_ctzll(cards);
}

// Deck order of Card::generate_deck(): suit-major, card = 13 * suit + rank, rank 0 = deuce,
// suits in the order clubs, hearts, spades, diamonds (the order src/state.rs:155 lists them).
static inline int or_rank(int card) { return card % 13; }
static inline int or_suit(int card) { return card / 13; }

// Runs f(i) for i in [0, n) on up to nthreads threads (rayon's role in the reference).
void or_parallel_for(int n, int nthreads, const std::function<void(int)> &f);

// One river subgame (state.rs:377-433); the f64 form is best response only.
int or_river_one_f32(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, uint64_t board4,
                     float bet, const float *opp, float *regrets, int player, bool exploit,
                     float *out);
// The same CFR pass that also adds the updater's average-strategy sums (own = its range).
int or_river_one_f32_avg(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, uint64_t board4,
                         float bet, const float *opp, const float *own, float *regrets, float *avg,
                         int player, float *out);
int or_river_one_f64(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, uint64_t board4,
                     float bet, const double *opp, const float *regrets, int player, double *out);

#endif
