"""Shared-memory bank model of river_kernel's data-dependent gathers (river_cfr.cu), on the
oracle's board tables of the reference flop.

For sampled boards the test rebuilds what pack_boards_kernel packs (rank order, tie groups,
card lists with their group ids, phs buckets, bucket order) and replays the addresses each
warp gathers in the kernel's three phases, per river card:
- rank-list scan: warps 0-3, lane g holds rank slots 9g..9g+8; each element gathers its
  hand's range and its bucket's opponent-reach row;
- card-list scans: warps 4-15, 8 lanes per list, lane s holds slots 6s..6s+5; the same two
  gathers per element;
- output phase: warps 0-11, lane t takes bucket-order positions 3t..3t+2; each hand gathers
  its tie-group row, the card-list group rows of its two cards, its range, its reach row and
  its bucket's own-reach row, and reads its result to add to it.
Bank model: a 32-bit warp access takes as many wavefronts as the most distinct words in one
bank; a 128-bit access, per quarter warp, as many as the most distinct 16-byte chunks in one
bank group. The conflict wavefronts of an access are the ones above one per active quarter.

The reach rows in four interleaved copies (chunk k of bucket b of copy q at chunk
(b*4 + k)*4 + q; lane p of a quarter reads copy p & 3, lanes 4-7 in chunk order 1, 0, 3, 2)
make the reach-row gathers conflict-free; with one copy 80 bytes apart they are not. Run
with -s to print the table per access.
"""
import numpy as np
import pytest

from oracle import oracle as O

HANDS, LIVE, BLOCKED, BUCKETS = 1326, 1081, 245, 256


def _hand_cards():
    co = O.card_order()
    out = np.zeros((HANDS, 2), int)
    for h in range(HANDS):
        m = int(co[h])
        lo = (m & -m).bit_length() - 1
        out[h] = (lo, (m & ~(1 << lo)).bit_length() - 1)
    return out


def _pack(board5, hc):
    e, _, a = O.board_tables(board5)
    live = (e[:HANDS] & 2047)[BLOCKED:].astype(int)
    flags = (e[:HANDS] & 2048) != 0
    gid = np.cumsum(np.r_[True, flags[BLOCKED + 1:]]) - 1
    lo, hi = np.zeros(LIVE, int), np.zeros(LIVE, int)
    lists = []
    cg = -1
    for card in (c for c in range(52) if not (board5 >> c) & 1):
        pos = [l for l in range(LIVE) if card in hc[live[l]]]
        assert len(pos) == 46
        elems = []
        for j, l in enumerate(pos):
            if j == 0 or gid[pos[j]] != gid[pos[j - 1]]:
                cg += 1
            elems.append(l)
            if hc[live[l]][0] == card:
                lo[l] = cg
            else:
                hi[l] = cg
        lists.append(elems)
    b = a[live].astype(int)
    order = sorted(range(LIVE), key=lambda l: (b[l], l))
    return dict(live=live, b=b, gid=gid, lo=lo, hi=hi, lists=lists, order=order, G=int(gid[-1]) + 1, CG=cg + 1)


def _w32(addrs):
    words = {a // 4 for a in addrs if a is not None}
    if not words:
        return 0
    banks = {}
    for w in words:
        banks.setdefault(w % 32, set()).add(w)
    return max(len(s) for s in banks.values()) - 1


def _w128(addrs):
    extra = 0
    for q in range(4):
        chunks = {a // 16 for a in addrs[8 * q:8 * q + 8] if a is not None}
        if chunks:
            groups = {}
            for c in chunks:
                groups.setdefault(c % 8, set()).add(c)
            extra += max(len(s) for s in groups.values()) - 1
    return extra


def _reach(b, k, lane, replicated):
    """Byte offset of chunk k of bucket b's opponent-reach row as lane `lane` reads it."""
    if replicated:
        return 16 * (b * 16 + (k ^ ((lane >> 2) & 1)) * 4 + (lane & 3))
    return 80 * b + 16 * k


def _conflicts(P, replicated):
    """Conflict wavefronts per access kind for one river card of board pack P."""
    # byte offsets of the gathered arrays modulo 128 in the kernel's layout for the reference
    # flop (136 rank groups, 917 card-list groups); only the 128-byte phase matters
    off_r, off_out, off_vg, off_vc, off_wown = 64, 0, 80, 80, 0
    out = dict.fromkeys(["reach rows, rank-list scan", "reach rows, card-list scans", "reach rows, output phase",
                         "card-list group rows, output phase", "hand ranges and results", "tie-group and own-reach rows"], 0)
    live, b = P["live"], P["b"]
    for w in range(4):
        for i in range(9):
            slots = [(w * 32 + lane) * 9 + i for lane in range(32)]
            ls = [s if s < LIVE else None for s in slots]
            out["hand ranges and results"] += _w32([None if l is None else off_r + 4 * live[l] for l in ls])
            for k in range(4):
                out["reach rows, rank-list scan"] += _w128(
                    [None if l is None else _reach(b[l], k, lane, replicated) for lane, l in enumerate(ls)])
    for cw in range(12):
        for i in range(6):
            ls = []
            for lane in range(32):
                li, j = cw * 4 + (lane >> 3), (lane & 7) * 6 + i
                ls.append(P["lists"][li][j] if li < 47 and j < 46 else None)
            out["hand ranges and results"] += _w32([None if l is None else off_r + 4 * live[l] for l in ls])
            for k in range(4):
                out["reach rows, card-list scans"] += _w128(
                    [None if l is None else _reach(b[l], k, lane, replicated) for lane, l in enumerate(ls)])
    for w in range(12):
        for i in range(3):
            ls = [P["order"][j] if j < LIVE else None for j in ((w * 32 + lane) * 3 + i for lane in range(32))]
            for k in range(3):
                out["tie-group and own-reach rows"] += _w128(
                    [None if l is None else off_vg + 48 * P["gid"][l] + 16 * k for l in ls])
                for side in ("lo", "hi"):
                    out["card-list group rows, output phase"] += _w128(
                        [None if l is None else off_vc + 48 * P[side][l] + 16 * k for l in ls])
            out["hand ranges and results"] += _w32([None if l is None else off_r + 4 * live[l] for l in ls])
            out["hand ranges and results"] += _w32([None if l is None else off_out + 4 * live[l] for l in ls])
            for k in range(4):
                out["reach rows, output phase"] += _w128(
                    [None if l is None else _reach(b[l], k, lane, replicated) for lane, l in enumerate(ls)])
            for k in range(5):
                out["tie-group and own-reach rows"] += _w128(
                    [None if l is None else off_wown + 80 * b[l] + 16 * k for l in ls])
    return out


@pytest.fixture(scope="module")
def packs():
    hc = _hand_cards()
    rng = np.random.default_rng(0)
    turns = [c for c in range(52) if not (O.REFERENCE_FLOP >> c) & 1]
    boards = []
    for t in rng.choice(turns, 3, replace=False):
        for r in rng.choice([c for c in turns if c != t], 4, replace=False):
            boards.append(O.REFERENCE_FLOP | (1 << int(t)) | (1 << int(r)))
    return [_pack(bd, hc) for bd in boards]


def test_replicated_reach_rows_remove_their_conflicts(packs):
    one = [_conflicts(P, False) for P in packs]
    four = [_conflicts(P, True) for P in packs]
    print("\nconflict wavefronts per river card (mean of the sampled boards): one copy / four copies")
    for key in one[0]:
        a = np.mean([c[key] for c in one])
        f = np.mean([c[key] for c in four])
        print(f"  {key:38s} {a:8.1f} {f:8.1f}")
    for c1, c4 in zip(one, four):
        for key in ("reach rows, rank-list scan", "reach rows, card-list scans", "reach rows, output phase"):
            assert c4[key] == 0, (key, c4[key])
        assert c1["reach rows, card-list scans"] > 0
        # the other gathers do not depend on the reach-row layout
        for key in ("card-list group rows, output phase", "hand ranges and results", "tie-group and own-reach rows"):
            assert c1[key] == c4[key]


def test_packs_fit_the_kernel_bounds(packs):
    # the tie-group counts size shared memory: the reference flop's boards stay at the sizes
    # the kernel is laid out for (at most 1081 rank groups, 47 x 46 card-list groups)
    for P in packs:
        assert 1 <= P["G"] <= LIVE and 47 <= P["CG"] <= 47 * 46
        assert P["b"].min() >= 0 and P["b"].max() < BUCKETS
