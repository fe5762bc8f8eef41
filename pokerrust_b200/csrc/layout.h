// Device data layout of the river solver.
//
// Board tables. The reference hands the GPU, per {turn, river} slot, the rank-sorted hand
// order as an inverse permutation with group-start flags, per-card collision lists and
// the bucket of every hand (src/cuda_interface.rs:48-102, src/cuda/evaluator.cuh:8-15).
// transfer_flop_eval_cuda keeps that interface and re-packs the tables once on the device
// into BoardPack, a layout built for the river kernel:
//   - only the 1081 hands that share no card with the five board cards ("live" hands)
//     appear; blocked hands have zero reach in every reference code path;
//   - the live hands in rank order ("global list"), each with its bucket;
//   - for each of the 47 cards not on the board, the 46 live hands holding it, in rank
//     order ("card lists"); these give the blocker corrections of a showdown;
//   - for each live hand the slots of its tie group in the global list and in its two
//     card lists, so that a showdown value is a handful of prefix-sum lookups.
#pragma once
#include <stdint.h>

namespace prb {

constexpr int kHands = 1326;
constexpr int kRangeStride = 1328;  // floats per range / result row (16-byte rows)
constexpr int kBlocked = 245;       // hands sharing a card with a 5-card board
constexpr int kLive = 1081;         // C(47, 2)
constexpr int kGSlots = 1088;       // global list slots: 1081 hands, end sentinel, padding
constexpr int kNumLists = 47;       // cards not on the board
constexpr int kLSlots = 48;         // card list slots: 46 hands, end sentinel, padding
constexpr int kListLen = 46;
constexpr int kSlotsPerBoard = 1326;  // colex index of the {turn, river} pair

constexpr uint32_t kNoBucket = 0xFFFF;
// Element words of the lists. Rank list (gelem):
//   hand (bits 0-10) | bucket (11-18) | starts a tie group (19) | tie group id (20-30)
// Card lists (celem):
//   hand (bits 0-10) | bucket (11-18) | starts a group within the list (19) | card group id (20-31)
// Padding elements carry hand kNoHand.
constexpr uint32_t kNoHand = 2047;
constexpr uint32_t kGroupStart = 1u << 19;

// Largest tie-group counts any 5-card board can have: 1081 hands in the rank list, 47 * 46
// hands in the card lists.
constexpr int kMaxGroups = kLive;
constexpr int kMaxCardGroups = kNumLists * kListLen;

struct BoardPack {
    // Per live hand in rank order (index l = sorted position - 245):
    //  x: hand | bucket << 11 | low card << 19 | high card << 25
    //  y: tie group id in the rank list
    //  z: group id of the hand in its low card's list
    //  w: group id of the hand in its high card's list
    uint4 meta[kGSlots];
    // Live hands in bucket order (then rank order): l | bucket << 16; padding entries carry
    // bucket kNoBucket. Bucket sums become segmented reductions over this order.
    uint32_t border[kGSlots];
    uint32_t gelem[kGSlots];               // rank list elements
    uint32_t celem[kNumLists * kLSlots];   // card list elements, 48 slots per list
    uint8_t list_card[64];                 // card of each card list
    int32_t num_groups;                    // tie groups in the rank list
    int32_t num_card_groups;               // groups over all card lists
    int32_t pad[2];
};

static_assert(sizeof(BoardPack) % 16 == 0, "BoardPack rows must stay 16-byte aligned");

// Per-subgame descriptor (one river root built by build_river_cuda).
struct SubgameDesc {
    unsigned long long board4;  // flop + turn
    float bet;                  // equal bets at the river root
    int pad;
};

}  // namespace prb
