/*
 * Oracle: CPU restatement of the reference's river-subtree CFR path.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load this library, and only
 * as the checker or the timed CPU baseline. The product library
 * (pokerrust_b200/) never links, loads or calls it.
 *
 * What it restates (reference paths are relative to the pokerrust project):
 *   - colex indexing of k-subsets of 52 cards      src/combination_map.rs:33-75
 *   - hand-rank tables per 5-card board            src/evaluator.rs:22-184
 *   - percentile-hand-strength (phs) buckets       src/evaluator.rs:243-308
 *   - the GPU packing of those tables              src/cuda_interface.rs:48-102
 *   - the river subtree (28 states, 26 edges)      src/builder.rs:34-79, src/state.rs:66-217,
 *                                                  src/cuda/builder.cu:8-138
 *   - river CFR / best response, per hand, f32     src/state.rs:219-296,377-433,436-569,
 *                                                  src/strategy.rs:86-153
 *   - the full fixed-flop game and its driver      src/state.rs, src/game.rs:30-143
 *
 * The 7-card hand ranking lives in the third-party `poker` crate
 * (gustafbergmark/poker rev dc15b08056977f9e067ec06a4af8f83358b45005, v0.4.1,
 * Cargo.lock:139-141), which is not part of the reference tree. It is restated
 * here from the standard hand-ranking rules; the deck order is suit-major
 * (card = 13*suit + rank, rank 0 = deuce, suit order clubs, hearts, spades,
 * diamonds as in src/state.rs:155), so the reference flop {0,1,2} is 2c 3c 4c. A
 * rank-major deck would make that flop three deuces, and then the phs arithmetic of
 * evaluator.rs:292-305 wraps below zero on quad-deuce boards and the reference's own
 * assert at strategy.rs:114 fails; the suit-major order avoids that. Parity of ranks
 * and permutations is pinned by
 * the published 7-card category counts and equivalence-class count, not by
 * reference fixtures (the reference ships none).
 */
#ifndef POKERRUST_ORACLE_H
#define POKERRUST_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_HANDS 1326
#define OR_EVAL_LEN (1326 + 256 * 2)
#define OR_COLL_LEN (52 * 51)
#define OR_BUCKETS 256
#define OR_RIVER_EDGES 26
#define OR_RIVER_STATES 28

/* --- combinatorics (combination_map.rs) --- */
int64_t or_choose(int n, int k);
int64_t or_colex_index(uint64_t set);           /* any popcount */
uint64_t or_pair_from_index(int index);          /* 2-card colex inverse */
void or_card_order(uint64_t *out1326);           /* evaluator.rs:29-40 */
void or_card_indexes(uint16_t *out2652);         /* evaluator.rs:159-172 */

/* --- hand ranking (poker crate, restated) --- */
uint32_t or_hand_value(uint64_t cards);          /* 5..7 cards; larger is better; 0 = WORST */
/* Counts of all C(52,7) hands per category [9] and number of distinct values. */
void or_count_7card(int64_t *category_counts9, int64_t *distinct_values, int nthreads);

/* --- tables for one 5-card board (evaluator.rs:55-135) --- */
void or_board_tables(uint64_t board5, uint16_t *eval1838, uint16_t *coll2652,
                     uint16_t *abstr1326);
/* GPU packing for a flop over all 1326 {turn,river} slots (cuda_interface.rs:48-102).
 * eval: 1326*1838, coll: 1326*2652, abstr: 1326*1326. nthreads <= 0 means all cores. */
void or_pack_flop_tables(uint64_t flop, uint16_t *eval, uint16_t *coll, uint16_t *abstr,
                         int nthreads);

/* --- river subtree --- */
/* Order of the river cards within a river pass: 0 ascending (state.rs), 1 descending. The
 * same sum in another f32 rounding, for measuring the trajectory's dependence on summation
 * order. Applies to every later pass of every game and batch in the process. */
void or_set_river_order(int descending);

/* Describes the 28-state river tree in builder.cu order. For state s:
 * terminal[s] (0 NonTerminal, 1 SBWins, 2 BBWins, 3 Showdown, 4 River),
 * actor[s] (0 small, 1 big), parent[s], sb_raise[s], bb_raise[s] (bets minus the root bet),
 * nchild[s], child[s*3+k], edge[s*3+k] (edge id of action k, -1 if none). */
void or_river_tree(int *terminal, int *actor, int *parent, float *sb_off, float *bb_off,
                   int *nchild, int *child, int *edge);

/* One river evaluation per subgame, per state.rs:377-433 (CPU branch).
 * board4[n]: 4-card boards (flop + turn); bet[n]: equal bets at the river root;
 * opp_range[n*1326]: the opponent's range at the river root;
 * regrets[n*26*256]: per-edge bucket regrets (edge order of or_river_tree), updated in place
 * when calc_exploit == 0; result[n*1326]: the updating player's values.
 * player: 0 small, 1 big. tables: packed flop tables from or_pack_flop_tables.
 * Returns 0 on success, nonzero on a violated reference assertion. */
int or_river_batch(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, int n,
                   const uint64_t *board4, const float *bet, const float *opp_range,
                   float *regrets, int player, int calc_exploit, float *result, int nthreads);

/* A CFR pass that also accumulates average-strategy sums (an addition: the reference keeps
 * none): own_range[n*1326] is the updating player's range at the river root; for each of
 * its decision states avg[edge][bucket] += sum over hands of reach into the state times
 * the action probability. */
int or_river_batch_avg(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, int n,
                       const uint64_t *board4, const float *bet, const float *opp_range,
                       const float *own_range, float *regrets, float *avg, int player,
                       float *result, int nthreads);

/* Same traversal in double precision, best response only (calc_exploit semantics). */
int or_river_br_f64(uint64_t flop, const uint16_t *eval, const uint16_t *abstr, int n,
                    const uint64_t *board4, const double *bet, const double *opp_range,
                    const float *regrets, int player, double *result, int nthreads);

/* --- full fixed-flop game (builder.rs, state.rs, game.rs) --- */
void *or_game_new(uint64_t flop, int nthreads);
void or_game_free(void *game);
int or_game_num_rivers(void *game);
/* River roots in the order the builder reaches them (state.rs:114-121). */
void or_game_river_roots(void *game, uint64_t *board4, float *bet);
/* One iteration (game.rs:68-119): SB update then BB update. */
void or_game_iterate(void *game);
/* Best-response values (game.rs:120-178): sums of the SB and BB BR vectors, and
 * the reference's mb/h figure (game.rs:175). use_f64 selects an FP64 traversal. */
void or_game_exploitability(void *game, int use_f64, double *sum_sb, double *sum_bb,
                            double *mbh);
/* Copies of the river regrets (27783*26*256 for the reference flop) in river-root order. */
void or_game_river_regrets(void *game, float *out);
/* Average-strategy sums (not in the reference): the updater's reach into each of its
 * decisions times the action probability, per hand above the river and per bucket in the
 * river subgames. Enable before iterating. */
void or_game_enable_average(void *game);
/* The root's values of the last iteration's SB and BB CFR passes (2 on no iteration yet). */
int or_game_root_values(void *game, float *sb, float *bb);
/* Sums over all upper-tree regrets / average sums and all river regrets / average sums. */
void or_game_totals(void *game, double *upper_regrets, double *upper_avg, double *river_regrets,
                    double *river_avg);
/* River average sums [rivers][26][256] (2 if averages are off). */
int or_game_river_average(void *game, float *out);

#ifdef __cplusplus
}
#endif
#endif
