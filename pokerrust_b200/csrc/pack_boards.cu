// Device-side re-pack of the reference's per-board tables into BoardPack.
//
// Input per {turn, river} slot (src/cuda_interface.rs:48-102): the "inverse eval" block
// (eval[hand] & 2047 = the hand's rank-sorted position, eval[p] & 2048 = position p starts
// a tie group; 1326 + 512 entries, the chunk tables after 1326 are not needed here) and
// the bucket of each hand. Collision lists (coll_vec) are derivable from the sort order,
// so they are rebuilt here rather than copied.
#include "device_common.cuh"
#include "layout.h"
#include "pack_boards.h"

namespace prb {

__global__ void __launch_bounds__(256) pack_boards_kernel(unsigned long long flop,
                                                          const uint16_t *__restrict__ eval,
                                                          const uint16_t *__restrict__ abstr,
                                                          BoardPack *__restrict__ packs,
                                                          int *__restrict__ err) {
    const int slot = blockIdx.x;
    const int tid = threadIdx.x;
    int c1, c2;
    hand_cards(slot, &c1, &c2);
    const unsigned long long pair = (1ull << c1) | (1ull << c2);
    BoardPack *out = packs + slot;
    if (pair & flop) return;  // slot never addressed by a river subgame of this flop
    const unsigned long long board = flop | pair;
    const uint16_t *e = eval + (size_t)slot * (1326 + 512);
    const uint16_t *a = abstr + (size_t)slot * kHands;

    __shared__ uint16_t sorted[kHands];
    __shared__ uint16_t cards_of[kHands];  // low card | high card << 8
    __shared__ unsigned int seen[kHands];
    __shared__ uint16_t gid[kLive];
    __shared__ uint16_t gstart[kLive];
    __shared__ uint32_t lo[kLive];  // group id of the hand in its low card's list
    __shared__ uint32_t hi[kLive];  // ... and in its high card's list
    __shared__ int list_groups[kNumLists];
    __shared__ uint8_t list_card[64];
    __shared__ int bad;

    if (tid == 0) bad = 0;
    for (int i = tid; i < kHands; i += blockDim.x) {
        seen[i] = 0;
        int hc1, hc2;
        hand_cards(i, &hc1, &hc2);
        cards_of[i] = (uint16_t)(hc1 | (hc2 << 8));
    }
    __syncthreads();
    for (int h = tid; h < kHands; h += blockDim.x) {
        int pos = e[h] & 2047;
        if (pos >= kHands) {
            atomicOr(&bad, 1);
            continue;
        }
        sorted[pos] = (uint16_t)h;
        atomicAdd(&seen[pos], 1u);
    }
    __syncthreads();
    for (int p = tid; p < kHands; p += blockDim.x) {
        if (seen[p] != 1) atomicOr(&bad, 2);
        int h = sorted[p];
        int hc1 = cards_of[h] & 255, hc2 = cards_of[h] >> 8;
        bool blocked = ((1ull << hc1) | (1ull << hc2)) & board;
        if (blocked != (p < kBlocked)) atomicOr(&bad, 4);  // blocked hands rank first
        if (a[h] >= 256) atomicOr(&bad, 8);                 // strategy.rs:114 bound
    }
    __syncthreads();
    if (bad) {
        if (tid == 0) atomicOr(err, bad);
        return;
    }
    if (tid == 0) {
        // tie groups of the live hands, from the group-start flags
        int g = -1, start = 0;
        for (int l = 0; l < kLive; l++) {
            if (l == 0 || (e[kBlocked + l] & 2048)) {
                g++;
                start = l;
            }
            gid[l] = (uint16_t)g;
            gstart[l] = (uint16_t)start;
        }
        out->num_groups = g + 1;
        atomicMax(err + 1, g + 1);
        int n = 0;
        for (int c = 0; c < 52; c++) {
            if (!(board >> c & 1)) list_card[n++] = (uint8_t)c;
        }
        for (; n < 64; n++) list_card[n] = 0;
    }
    __syncthreads();
    if (tid < kNumLists) {
        // groups inside one card list: hands of the list that share a tie group
        const int li = tid;
        const int card = list_card[li];
        int k = 0, ng = 0, prev = -1;
        for (int l = 0; l < kLive && k < kListLen; l++) {
            int h = sorted[kBlocked + l];
            int hc1 = cards_of[h] & 255, hc2 = cards_of[h] >> 8;
            if (hc1 == card || hc2 == card) {
                if (gid[l] != prev) ng++;
                prev = gid[l];
                k++;
            }
        }
        list_groups[li] = ng;
    }
    __syncthreads();
    if (tid < kNumLists) {
        // card list of one live card, in rank order, with its group ids
        const int li = tid;
        const int card = list_card[li];
        uint16_t pos[kListLen];
        int k = 0;
        for (int l = 0; l < kLive && k < kListLen; l++) {
            int h = sorted[kBlocked + l];
            int hc1 = cards_of[h] & 255, hc2 = cards_of[h] >> 8;
            if (hc1 == card || hc2 == card) pos[k++] = (uint16_t)l;
        }
        if (k != kListLen) atomicOr(err, 16);  // cannot happen once the checks above passed
        int base = 0;
        for (int i = 0; i < li; i++) base += list_groups[i];
        uint32_t *ce = out->celem + li * kLSlots;
        int cg = base - 1;
        for (int j = 0; j < k; j++) {
            const bool start = j == 0 || gid[pos[j]] != gid[pos[j - 1]];
            if (start) cg++;
            int l = pos[j];
            int h = sorted[kBlocked + l];
            ce[j] = (uint32_t)h | ((uint32_t)a[h] << 11) | (start ? kGroupStart : 0u) | ((uint32_t)cg << 20);
            if ((cards_of[h] & 255) == card) lo[l] = (uint32_t)cg;
            else hi[l] = (uint32_t)cg;
        }
        ce[kListLen] = kNoHand;
        ce[kListLen + 1] = kNoHand;
        if (li == kNumLists - 1) {
            out->num_card_groups = cg + 1;
            atomicMax(err + 2, cg + 1);
        }
    }
    __syncthreads();
    for (int l = tid; l < kGSlots; l += blockDim.x) {
        if (l < kLive) {
            int h = sorted[kBlocked + l];
            int hc1 = cards_of[h] & 255, hc2 = cards_of[h] >> 8;
            uint32_t x = (uint32_t)h | ((uint32_t)a[h] << 11) | ((uint32_t)hc1 << 19) |
                         ((uint32_t)hc2 << 25);
            out->meta[l] = make_uint4(x, gid[l], lo[l], hi[l]);
            out->gelem[l] = (uint32_t)h | ((uint32_t)a[h] << 11) | (gstart[l] == l ? kGroupStart : 0u) |
                            ((uint32_t)gid[l] << 20);
        } else {
            out->meta[l] = make_uint4(0, 0, 0, 0);
            out->gelem[l] = kNoHand;
        }
    }
    if (tid < 64) out->list_card[tid] = list_card[tid];
    if (tid == 64) {
        // counting sort of the live hands by bucket (stable in rank order)
        uint16_t start[257];
        for (int b = 0; b <= 256; b++) start[b] = 0;
        for (int l = 0; l < kLive; l++) start[a[sorted[kBlocked + l]] + 1]++;
        for (int b = 0; b < 256; b++) start[b + 1] += start[b];
        for (int l = 0; l < kLive; l++) {
            const int b = a[sorted[kBlocked + l]];
            out->border[start[b]++] = (uint32_t)l | ((uint32_t)b << 16);
        }
        for (int l = kLive; l < kGSlots; l++) out->border[l] = kNoBucket << 16;
    }
}

void launch_pack_boards(unsigned long long flop, const uint16_t *eval, const uint16_t *abstr,
                        BoardPack *packs, int *err, cudaStream_t stream) {
    pack_boards_kernel<<<kSlotsPerBoard, 256, 0, stream>>>(flop, eval, abstr, packs, err);
}

}  // namespace prb
