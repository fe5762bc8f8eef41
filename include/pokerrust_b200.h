/*
 * pokerrust_b200: C ABI of the B200 river-subtree CFR solver.
 *
 * The first seven functions are the drop-in boundary: the same unmangled symbols, argument
 * meaning and call protocol as the reference's CUDA library (src/cuda/interface.cu:9-122),
 * as its Rust FFI binds them (src/cuda_interface.rs:8-31). The C side of the reference
 * spells the 64-bit and 16-bit arguments `long` / `short`; on LP64 those are the same
 * types as uint64_t / uint16_t here, which is how the Rust side declares them.
 *
 * The pr_* functions are extensions with no counterpart in the reference: status codes,
 * device-resident entry points, state access for tests and checkpoints.
 *
 * Error convention: the reference prints CUDA errors and carries on. The drop-in symbols
 * keep that (a line on stderr) and also record a sticky status that pr_last_error()
 * returns; the pr_* functions return that status directly (0 = success).
 */
#ifndef POKERRUST_B200_H
#define POKERRUST_B200_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- drop-in boundary (src/cuda_interface.rs:8-31, src/cuda/interface.cu:9-122) ---- */

/* Replaces init_builder (interface.cu:72-85, cuda_interface.rs:9): returns a
 * library-owned builder. The reference sizes it for 63*49*9 subgames; this one grows as
 * build_river_cuda adds subgames. */
void *init_builder(void);

/* Replaces upload_c (interface.cu:87-89, cuda_interface.rs:11): copies 1326 floats (the
 * opponent range at river root `index`) into the builder's pinned staging. Safe to call
 * from many threads at once for distinct indexes, as state.rs:340-341,380-387 does. A range
 * holding a NaN, an infinity or a negative weight is not copied and sets the sticky status
 * (pr_last_error() == 2); the reference copies it unchecked. */
void upload_c(void *builder, int index, const float *v);

/* Replaces download_c (interface.cu:91-93, cuda_interface.rs:12): copies the 1326 result
 * values of river root `index` out of the staging. Thread-safe across distinct indexes. */
void download_c(void *builder, int index, float *v);

/* Replaces build_river_cuda (interface.cu:95-121, builder.cu:123-138,
 * cuda_interface.rs:13): adds one river subgame (4-card board `cards`, equal bets `bet`)
 * with zero regrets; returns its index, increasing from 0. Single-threaded init only. */
int build_river_cuda(uint64_t cards, float bet, void *builder);

/* Replaces transfer_flop_eval_cuda (interface.cu:50-68, cuda_interface.rs:14-21): takes
 * the reference's packed per-board tables for `flop` (1326 slots of 1326+512 eval, 52*51
 * collision and 1326 bucket entries, cuda_interface.rs:444-479) and returns an opaque
 * handle to device tables. Caller buffers are copied, not kept. */
void *transfer_flop_eval_cuda(uint64_t flop, const uint64_t *card_order,
                              const uint16_t *card_indexes, const uint16_t *eval,
                              const uint16_t *coll_vec, const uint16_t *abstractions);

/* Replaces free_eval_cuda (interface.cu:69-71, cuda_interface.rs:22). */
void free_eval_cuda(void *eval);

/* Replaces evaluate_cuda (interface.cu:11-49, cuda_interface.rs:24-29): synchronous. Reads
 * every subgame's opponent range from the staging, runs the river pass for
 * `updating_player` (0 small, 1 big) and overwrites the staging with the results.
 * calc_exploit = false: counterfactual values and a regret update of the updater's edges;
 * true: best-response values, regrets untouched. */
void evaluate_cuda(void *builder, void *eval, uint16_t updating_player, bool calc_exploit);

/* ---- extensions (no counterpart in the reference) ---- */

/* Sticky status of the last failing call on this process (0 = none), and its text. */
int pr_last_error(void);
const char *pr_error_string(int status);
void pr_clear_error(void);

/* evaluate_cuda with a status code. */
int pr_evaluate(void *builder, void *eval, int updating_player, int calc_exploit);

/* Device-resident pass: ranges / results are device pointers to n rows of 1328 floats
 * (n = pr_builder_count), stream is a cudaStream_t (NULL = the builder's stream).
 * Asynchronous: returns after the launch. */
int pr_evaluate_device(void *builder, void *eval, int updating_player, int calc_exploit,
                       const float *d_ranges, float *d_results, void *stream);

/* Batch forms of upload_c / download_c for rows first .. first+count-1; v holds count
 * rows of 1326 floats (the same copies the reference's caller makes one call at a time).
 * pr_upload_batch skips rows upload_c would refuse and then returns 2. */
int pr_upload_batch(void *builder, int first, int count, const float *v);
int pr_download_batch(void *builder, int first, int count, float *v);

/* Average strategies (an addition: the reference keeps none). After pr_enable_average, every
 * CFR pass of evaluate_cuda / pr_evaluate also accumulates, per river root, edge and bucket,
 * the sum over rivers and hands of the updater's reach into the state times the action's
 * probability. The updater's own range at each root is staged with pr_upload_own (same
 * contract as upload_c). pr_get_average copies the sums (count * 26 * 256 floats). */
int pr_enable_average(void *builder);
void pr_upload_own(void *builder, int index, const float *v);
int pr_get_average(void *builder, float *out);
int pr_set_average(void *builder, const float *in);

/* Number of river subgames in the builder, and the row stride (floats) of pr_* buffers. */
int pr_builder_count(void *builder);
int pr_range_stride(void);

/* Bucket regrets, count * 26 * 256 floats in the reference's edge order
 * (src/cuda/builder.cu:85-97 numbering). Host buffers; synchronous. */
int pr_get_regrets(void *builder, float *out);
int pr_set_regrets(void *builder, const float *in);

/* Releases a builder (the reference never frees it). */
void pr_free_builder(void *builder);

/* Builds the hand-rank tables of every river board of `flop` on the device (the work the
 * reference's host does in src/evaluator.rs:22-184 and packs in src/cuda_interface.rs:48-102)
 * and returns a handle usable wherever transfer_flop_eval_cuda's is; release it with
 * free_eval_cuda. Check pr_eval_status. */
void *pr_tables_build(uint64_t flop);

/* Copies a handle's tables out in the reference's packed layout (1326 slots of 1838 eval,
 * 2652 collision and 1326 bucket u16 entries); null outputs are skipped. */
int pr_tables_export(void *eval, uint16_t *eval_out, uint16_t *coll_out, uint16_t *abstr_out);

/* On-disk tables (extension; the reference only sketched a bincode dump, evaluator.rs:43-45,
 * 148-154): a versioned file with a checksum of the packed eval, collision and bucket
 * tables. pr_tables_load returns a handle like transfer_flop_eval_cuda's (release with
 * free_eval_cuda), or null if the file is missing, truncated or corrupted. */
int pr_tables_save(void *eval, const char *path);
void *pr_tables_load(const char *path);

/* Status of a table handle: 0, or the bit set of table inconsistencies found on upload. */
int pr_eval_status(void *eval);

/* Shared memory bytes the river kernel uses per CTA with these tables (0 if invalid). */
size_t pr_river_smem_bytes(void *eval, int calc_exploit, int fp64);

/* Best-response pass in double precision (the exploitability check): ranges / results are
 * host arrays of count rows of 1326 doubles; regrets are read, not changed. Synchronous. */
int pr_evaluate_br64(void *builder, void *eval, int updating_player, const double *ranges,
                     double *results);

/* The same passes on caller-owned device rows of 1328 (pr_range_stride) on `stream`
 * (null = the builder's stream), asynchronous:
 * pr_evaluate_device_own is a CFR pass that also accumulates average-strategy sums from the
 * updater's own ranges d_own (pr_enable_average first); pr_evaluate_br64_device is the
 * double-precision best response. No reference counterparts: they let a device-side upper
 * tree feed the river solver without host copies. */
int pr_evaluate_device_own(void *builder, void *eval, int updating_player, const float *d_ranges,
                           const float *d_own, float *d_results, void *stream);
int pr_evaluate_br64_device(void *builder, void *eval, int updating_player, const double *d_ranges,
                            double *d_results, void *stream);

/* ---- whole-game driver (extension): the host side of the reference's GPU build ----
 * (src/builder.rs, src/state.rs, src/strategy.rs:37-82, src/permutation_handler.rs,
 * src/game.rs) over the functions above. Tables are built on the device. */

/* Builds the fixed-flop game (preflop, the given flop, turn, river roots); nthreads <= 0
 * uses every core for the turn cards. Null on failure (see pr_last_error). */
void *pr_game_new(uint64_t flop, int nthreads);
void pr_game_free(void *game);
int pr_game_num_rivers(void *game);
/* River roots (4-card board, equal bet) in the order the game registers them. */
int pr_game_river_roots(void *game, uint64_t *boards, float *bets);
/* The game's river builder and table handle, for the functions above. */
void *pr_game_builder(void *game);
void *pr_game_tables(void *game);
/* CFR iterations (game.rs:68-119): small blind update, then big blind update. */
int pr_game_iterate(void *game, int iterations);
/* The root's counterfactual values (per colex hand, 1326 floats each) of the last
 * iteration's small-blind and big-blind CFR passes: the vectors eval_state returns at the
 * root in game.rs:68-119. 2 before the first iteration. */
int pr_game_root_values(void *game, float *sb, float *bb);
/* Where the preflop/flop/turn tree is traversed: 1 (default) on the device, level by level,
 * with each iteration replayed as one CUDA graph; 0 on the host through upload_c /
 * evaluate_cuda / download_c, the reference's protocol (game.rs:68-119). Both give the
 * same results bit for bit. Returns the previous setting, or -1 on error. */
int pr_game_set_device_tree(void *game, int on);
/* Best-response sums of both players and the reference's mb/h figure (game.rs:120-178);
 * fp64 = 1 runs the whole best response in double precision. */
int pr_game_exploitability(void *game, int fp64, double *sum_sb, double *sum_bb, double *mbh);
/* Seconds spent so far in host traversal and in device passes. */
int pr_game_timings(void *game, double *host_seconds, double *device_seconds);
/* Upper-tree regrets (pr_game_upper_regret_count floats, node order) and river regrets. */
size_t pr_game_upper_regret_count(void *game);
int pr_game_get_regrets(void *game, float *upper, float *river);
/* Replaces the upper-tree regrets and/or the river regrets (either pointer may be null; same
 * layouts as pr_game_get_regrets), e.g. to restore a state kept by the caller. Returns 2 for a
 * null game or a NaN or infinite regret in either array (nothing is changed then). */
int pr_game_set_regrets(void *game, const float *upper, const float *river);
/* Average strategies for the whole game: upper-tree sums (per hand, regret layout) and
 * river sums (per bucket, pr_get_average layout) from the next iteration on. */
int pr_game_enable_average(void *game);
int pr_game_get_average(void *game, float *upper, float *river);
/* Checkpoints: regrets (and average sums, when enabled) of the whole game in a versioned,
 * checksummed binary file; loading checks the flop and sizes. 0 = success, 3 = wrong or
 * corrupted file. */
int pr_game_save(void *game, const char *path);
int pr_game_load(void *game, const char *path);

/* ---- batched general river subgames (extension; no reference counterpart) ----
 * Many independent river subgames, each with its own 5-card board, pot, stack and bet tree,
 * solved with per-hand regrets (CFR with regrets clipped at zero, the reference's update
 * rule) by one persistent kernel fed from a device work queue; each CFR iteration is
 * replayed as one CUDA graph. Tree rules: player 0 acts first; bets of 0.5 pot (sizes bit
 * 0), 1 pot (bit 1) and all-in (bit 2), at most max_raises (1..3) bets and raises; a fold
 * loses pot/2 plus the folder's river chips, a showdown moves pot/2 plus the river chips.
 * Hands are colex indexes (1326; hands that touch the board are ignored). */
typedef struct {
    uint64_t board;     /* 5 cards, bit i = card i (13 * suit + rank) */
    float pot;          /* chips in the pot before the river, pot/2 from each player; > 0, finite */
    float stack;        /* chips behind each player; >= 0, finite */
    uint32_t sizes;     /* bet sizes enabled: bit 0 half pot, bit 1 pot, bit 2 all-in; at least
                           one, no other bits */
    int32_t max_raises; /* bets + raises on the river, 1..3 */
} pr_subgame;

/* Builds one subgame's tree on the host (16-byte nodes in pre-order; nodes_out may be null,
 * else room for 128 nodes). 0 on success, 2 if the spec is invalid. */
int pr_batch_tree(const pr_subgame *spec, void *nodes_out, int *num_nodes, int *num_edges, int *num_leaves);
/* ranges: [count][2][1326] floats (player 0, player 1), finite and non-negative. Null on
 * failure (a bad board or tree, a NaN, infinite or negative weight, an allocation). */
void *pr_batch_new(const pr_subgame *specs, int count, const float *ranges);
void pr_batch_free(void *batch);
int pr_batch_count(void *batch);
int pr_batch_shape(void *batch, int s, int *num_nodes, int *num_edges, int *num_leaves);
int pr_batch_enable_average(void *batch);
/* CFR iterations: player 0 update, then player 1. */
int pr_batch_iterate(void *batch, int iterations);
/* Average sums weighted by the iteration number (on = 1: iteration t adds t x reach x
 * strategy) or by 1 (on = 0, the default); the weight restarts at 1. */
int pr_batch_set_linear_average(void *batch, int on);
/* No counterpart in the reference. pr_batch_iterate for callers that may not allocate once
 * their solve loop runs: a process whose GPU memory is handed out by its own caching
 * allocator, or a loop on a shared GPU where a cudaMalloc / cudaFree (they synchronise the
 * device) or building a CUDA graph (pr_batch_iterate does that on its first call) would stall
 * other work. The passes are launched directly, and the work-queue scratch (queue heads and
 * queue order) sits in a fixed 256 KB device array of the library, held on every GPU that
 * loads it, so the call makes no cudaMalloc, cudaFree or other allocating call.
 * Limit: 65536 subgames per batch (status 2 beyond). The queue heads are cleared before every
 * pass; the order is rewritten on every call. The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress): make that first call before any stream
 * capture. All calls share the one array, so calls that overlap on the GPU race: issue them
 * one after another. It runs the same iteration as pr_batch_iterate (launch configuration,
 * linear averaging and average weights included), so both give the same results. */
int pr_batch_iterate_noalloc(void *batch, int iterations);
/* Per subgame: best-response sums of each player (range-weighted root values) and the
 * exploitability (br0 + br1) / 2 per unit of joint range mass, in chips; against the
 * current (use_average 0) or average strategies; fp64 = 1 in double precision. */
int pr_batch_exploitability(void *batch, int use_average, int fp64, double *br0, double *br1, double *expl);
/* Counterfactual values of `player` at the root ([count][1326], double) under the current or
 * average strategies, and their range-weighted sums (the player's subgame value). */
int pr_batch_root_values(void *batch, int player, int use_average, double *values, double *sums);
/* Adjoint pair. Forward: the subgame value V = r0^T U(sigma) r1 (player 0's expected chips
 * times the joint range mass) under the current or average strategies, double precision.
 * Backward: dV/dr0 = player 0's counterfactual values, dV/dr1 = minus player 1's
 * ([count][1326] each), and dV/dsigma(a, h) = r0(h) x value of root action a for hand h
 * ([count][8][1326]; player 0 acts at the root). Reach vectors are recomputed in the
 * backward pass, not stored per node. Null outputs are skipped. */
int pr_batch_value(void *batch, int use_average, double *V);
int pr_batch_value_grad(void *batch, int use_average, double *d_r0, double *d_r1, double *d_sigma);
/* The same backward pass with device outputs (device pointers, same layouts; null skipped),
 * for callers that use the gradients on the GPU. Synchronous. */
int pr_batch_value_grad_device(void *batch, int use_average, double *d_r0, double *d_r1, double *d_sigma);
/* Replaces subgame s's ranges ([2][1326] floats). NaNs and infinities are refused (status
 * 2); negative weights are accepted, since the value and its adjoint are bilinear in the
 * ranges (central differences step below zero); CFR on them is the caller's concern. */
int pr_batch_set_ranges(void *batch, int s, const float *r);
/* Regrets / average sums of subgame s: [edges][1326] floats, edges in tree order. */
int pr_batch_get_regrets(void *batch, int s, float *out);
int pr_batch_set_regrets(void *batch, int s, const float *in);
int pr_batch_get_average(void *batch, int s, float *out);
int pr_batch_set_average(void *batch, int s, const float *in);
/* Every subgame's regrets (which 0) or average sums (which 1) in one call: out[sum of the
 * subgames' edge counts][1326] floats, subgames in batch order, edges in tree order. */
int pr_batch_get_all(void *batch, int which, float *out);
/* Launch configuration per tree-shape class (0: up to 16 leaves, 1: more): hands per
 * thread (2, 3, 4), resident CTAs per SM, queue order (0 most work first, 1 input order). */
int pr_batch_config(void *batch, int c, int *K, int *per_sm, int *order, int *count);
int pr_batch_set_config(void *batch, int c, int K, int per_sm, int order);
/* Autotuner: times every configuration per class on the batch's first (up to) 8192
 * subgames and keeps the fastest; their solver state is restored afterwards. ms_out[2]: the
 * chosen configurations' per-pass times on those subgames. */
int pr_batch_tune(void *batch, double *ms_out);
/* Algorithmic HBM bytes of one CFR iteration (roofline numerator). */
double pr_batch_iteration_bytes(void *batch);

/* ---- turn-leaf value network (extension) ----
 * D[M][N] (f32) = A[M][K] . B[N][K]^T for bf16 A, B on the tcgen05 tensor cores (device
 * pointers; M % 128 == 0, N % bn == 0, K % 64 == 0, bn 128 or 256). Synchronous. */
int pr_gemm_bf16(const void *A, const void *B, float *D, int M, int N, int K, int bn, void *stream);
/* The same product with either operand stored MN-major: a_mn = 1 reads A from a [K][M]
 * array, b_mn = 1 reads B from a [K][N] array (the tensor cores take either layout). */
int pr_gemm_bf16_major(const void *A, const void *B, float *D, int M, int N, int K, int bn, int a_mn, int b_mn,
                       void *stream);
/* Asynchronous form; err is a device int that collects error bits of timed-out waits. */
int pr_gemm_bf16_async(const void *A, const void *B, float *D, int M, int N, int K, int bn, int *err,
                       void *stream);
/* The same BF16 product in the persistent form (no reference counterpart): one CTA per SM
 * walks the output tiles with a double-buffered tensor-memory accumulator, so each tile's
 * epilogue overlaps the next tile's main loop. D holds `splits` split-K parts [z][M][N]
 * (f32); either operand may be MN-major. Synchronous: 0, 2 for bad shapes, 1 on error. */
int pr_gemm_bf16_persistent(const void *A, const void *B, float *D, int M, int N, int K, int bn, int a_mn,
                            int b_mn, int splits, void *stream);
/* The K-major persistent product launched on `stream` without synchronising; err: a device
 * int collecting the kernel's error bits. 0, 2 (bad shapes) or 1. */
int pr_gemm_bf16_persistent_async(const void *A, const void *B, float *D, int M, int N, int K, int bn, int *err,
                                  void *stream);
/* Test support for the GEMM's bounded waits (no reference counterpart): the K-major product
 * with an mbarrier wait limit of wait_ns and, with withhold_k >= 0, one tile load of CTA
 * (0, 0) armed but never issued, so that the waits for it run out and the kernel returns
 * with its error bits set (2 = MMA wait, 1 = producer wait) instead of hanging. Returns the
 * error bits, -2 for bad shapes (K > 256 when a load is withheld), -1 on a CUDA error. */
int pr_gemm_bf16_wait_test(const void *A, const void *B, float *D, int M, int N, int K, int bn,
                           unsigned long long wait_ns, int withhold_k, void *stream);

/* The network: 2706 inputs (both ranges, the 4 turn cards as 52 0/1 values, pot / 200 and
 * stack / (10 pot)) -> 4 x 1024 GELU -> 2652 outputs (both players' counterfactual values per
 * hand over the pot). BF16 weights and activations, FP32 accumulation and master weights,
 * MSE loss, Adam. rows: the batch the buffers are sized for (a multiple of 256). Inputs and
 * outputs are device pointers: ranges [n][2][1326], boards [n] (4-card masks), scalars [n][2],
 * targets / out [n][2652]; n <= rows. */
void *pr_mlp_new(int rows, uint64_t seed);
void pr_mlp_free(void *net);
int pr_mlp_rows(void *net);
/* The GEMM form of the network's passes: 1 = the persistent form (pr_gemm_bf16_persistent,
 * 128 x 128 tiles), 0 = one CTA per tile. Both give the same results bit for bit. Returns the
 * previous setting, -1 for a null network. */
int pr_mlp_set_persistent(void *net, int on);
int pr_mlp_forward(void *net, const float *ranges, const uint64_t *boards, const float *scalars, float *out,
                   int n);
/* One step: forward, loss, backward, Adam with learning rate lr (lr = 0: gradients only).
 * loss: the batch's mean squared error before the update. */
int pr_mlp_train_step(void *net, const float *ranges, const uint64_t *boards, const float *scalars,
                      const float *targets, int n, float lr, double *loss);
/* Layer l (0..4): fan-out x fan-in of the live weights; host copies of W, b and of the last
 * step's gradients. */
int pr_mlp_layer_shape(int l, int *fan_out, int *fan_in);
int pr_mlp_get_layer(void *net, int l, float *W, float *b);
int pr_mlp_set_layer(void *net, int l, const float *W, const float *b);
int pr_mlp_get_grad(void *net, int l, float *dW, float *db);

/* ---- full fixed-flop game with general bets (extension; no reference counterpart) ----
 * Flop and turn streets with pot-fraction bets (rules in the source of pr_full_tree), a
 * chance node dealing the 49 turn cards, and at the end of the turn a river chance node whose
 * 48 river subgames (pr_subgame trees with the leaf's pot and stack) are solved by the batched
 * river solver in the same pass. CFR with regrets clipped at zero, alternating players; the
 * average strategy is the reach-weighted sum. Net-leaf mode answers the leaves with chips
 * behind by the value network instead. */
typedef struct {
    float fracs[4];     /* bet and raise sizes as pot fractions */
    int32_t nfrac;      /* 0..4 */
    int32_t allin;      /* all-in is an option */
    int32_t max_raises; /* bets + raises on the street, 0..4 */
} pr_street;
typedef struct {
    uint64_t flop;          /* 3 cards */
    float pot;              /* chips in the pot before the flop, pot/2 from each player */
    float stack;            /* chips behind each player */
    pr_street street[2];    /* flop, turn */
    uint32_t river_sizes;   /* river subgames: pr_subgame.sizes */
    int32_t river_raises;   /* river subgames: pr_subgame.max_raises */
} pr_full_spec;

/* The flop and turn nodes on the host: 48-byte nodes in pre-order and the child list (see
 * full_tree.h for the layout); null outputs are skipped. 2 if the spec is bad (a flop of
 * other than 3 cards, a pot that is not positive and finite, a negative or infinite stack,
 * fractions that are not positive and finite, street raises outside 0..4, river sizes
 * outside bits 0-2 or none, river raises outside 1..3) or the outputs are too small. */
int pr_full_tree(const pr_full_spec *spec, void *nodes_out, int max_nodes, int *num_nodes, int *num_edges,
                 int *num_leaves, int *kids_out, int max_kids);
/* ranges: [2][1326] floats (hands touching the flop are ignored). Null on failure: a bad
 * spec (as pr_full_tree), a range holding a NaN, an infinity or a negative weight, or an
 * allocation that fails. */
void *pr_full_new(const pr_full_spec *spec, const float *ranges);
void pr_full_free(void *game);
int pr_full_shape(void *game, int *num_nodes, int *num_edges, int *num_leaves, int *bet_subgames,
                  int *allin_subgames);
/* Net-leaf mode on (a pr_mlp_new network) or off (null). */
int pr_full_set_net(void *game, void *net);
/* Net leaves shifted to zero sum (on = 1): the outputs v0, v1 move by -e/2 with
 * e = r0 . v0 + r1 . v1 over the normalised leaf ranges, which true subgame values satisfy
 * with e = 0. Off by default. */
int pr_full_set_zero_sum(void *game, int on);
/* The batched solver's autotuner on both river-subgame batches; ms_out[4] (or null): the
 * chosen per-pass times of each batch's two shape classes. */
int pr_full_tune(void *game, double *ms_out);
/* Average sums weighted by the iteration number (1, the default) or uniformly (0). */
int pr_full_set_linear_average(void *game, int on);
/* One CFR half-iteration for `player`; pr_full_iterate: whole iterations (one CUDA graph each
 * without a network). */
int pr_full_pass(void *game, int player);
int pr_full_iterate(void *game, int iterations);
/* FP64 best responses to the average strategies over the whole game and the exploitability
 * (br0 + br1) / 2 per unit of joint range mass, in chips. resolve_iterations > 0 first
 * re-solves the river subgames of the leaves with chips behind from zero under the current
 * average flop and turn strategies (for net-leaf strategies, which stop at the turn). In
 * net-leaf mode this replaces those subgames' regrets and average sums; in plain mode they are
 * kept aside (a device copy of their rows) and restored, so measuring leaves the solve as it
 * was. */
int pr_full_exploitability(void *game, int resolve_iterations, double *br0, double *br1, double *expl);
/* Device state: which 0 regrets / 1 average sums [edges][1326] f32; 2 reach [nodes][2][1326],
 * 3 leaf values [leaves][1326], 4 node values [nodes][1326] (f32, last CFR pass); 5, 6, 7
 * the same in f64 from the last best response; 8 network inputs [net leaves][2][1326] and
 * 9 reach masses [net leaves][2] (f32, last net-leaf pass). pr_full_write: which 0 or 1. */
int pr_full_read(void *game, int which, void *out);
/* Zeroes every regret and average sum (flop, turn and river subgames). */
int pr_full_reset(void *game);
int pr_full_write(void *game, int which, const void *in);
/* River subgame batches (0: leaves with chips behind, 1: all-in leaves; subgame j * 48 + k is
 * river card k, in card order, of the batch's j-th leaf), their leaf node ids, and the joint
 * mass of the initial ranges. */
void *pr_full_batch(void *game, int which);
int pr_full_batch_leaves(void *game, int which, int *nodes_out);
double pr_full_joint(void *game);

#ifdef __cplusplus
}
#endif
#endif
