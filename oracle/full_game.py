"""Oracle for the full fixed-flop game with general bets (flop and turn streets above river
subgames).

TEST INFRASTRUCTURE ONLY: an independent restatement, in numpy (float64), of the full-game
rules and of one CFR half-iteration or best-response sweep over the flop and turn streets.
The reference's own full game is the limit tree of src/state.rs:66-217 and
src/builder.rs:13-79; the sweeps follow its upper-tree traversal (state.rs:219-376: reach
top-down, values bottom-up, regret matching with the 1e-4 cutoff of strategy.rs:138-156,
regrets clipped at zero, chance nodes averaged over their cards), extended to pot-fraction
bets, a dealt turn and river subgames at the end of the turn. The river subgames
themselves are checked against oracle/batch.cpp (Subgame in oracle.py).

Rules restated: both players have pot/2 in before the flop and `stack` behind; player 0
acts first on each street. Not facing a bet: check or bet frac x pot-now (capped at the
chips behind; repeated or zero amounts dropped) or all-in; player 1's check ends the
street. Facing a bet: fold, call (ends the street), or raise to-call + frac x (pot after the
call) (capped) or all-in, while raises remain and more than the call is behind. A fold
loses pot/2 + the folder's chips of the street (pot = pot at the street's start). The flop
ends in a deal of the 49 turn cards; the turn ends in a leaf (the river).
"""
import numpy as np

HANDS = 1326
DECISION, FOLD, DEAL, LEAF = 0, 1, 2, 3


def hand_cards():
    """Cards (c1 < c2) of each colex hand h = c1 + c2 (c2 - 1) / 2."""
    c1 = np.zeros(HANDS, np.int64)
    c2 = np.zeros(HANDS, np.int64)
    h = 0
    for b in range(1, 52):
        for a in range(b):
            c1[h], c2[h] = a, b
            h += 1
    return c1, c2


_C1, _C2 = hand_cards()
_MASK = (np.uint64(1) << _C1.astype(np.uint64)) | (np.uint64(1) << _C2.astype(np.uint64))
# hands sharing no card
_COMPAT = ((_C1[:, None] != _C1[None, :]) & (_C1[:, None] != _C2[None, :]) &
           (_C2[:, None] != _C1[None, :]) & (_C2[:, None] != _C2[None, :])).astype(np.float64)


def blocked(cards):
    """Hands that hold any of the cards in the mask."""
    return (_MASK & np.uint64(cards)) != 0


class Tree:
    """The flop and turn streets as flat lists, pre-order."""

    def __init__(self, flop, pot, stack, streets):
        """streets: [(fracs, allin, max_raises)] for the flop and the turn."""
        self.flop = int(flop)
        self.streets = streets
        self.kind, self.actor, self.parent, self.in_edge, self.level = [], [], [], [], []
        self.stake, self.stack, self.board, self.street = [], [], [], []
        self.children, self.first_edge = [], []
        self.leaf_index = []
        self.edges = 0
        self.leaves = []
        root = self._node(DECISION, 0, -1, -1, 0, 0, self.flop)
        self._decide(root, 0, float(pot), float(stack), 0.0, 0.0, 0, 0)

    def _node(self, kind, actor, parent, in_edge, level, street, board):
        self.kind.append(kind)
        self.actor.append(actor)
        self.parent.append(parent)
        self.in_edge.append(in_edge)
        self.level.append(level)
        self.street.append(street)
        self.board.append(board)
        self.stake.append(0.0)
        self.stack.append(0.0)
        self.children.append([])
        self.first_edge.append(-1)
        self.leaf_index.append(-1)
        return len(self.kind) - 1

    def _end(self, me, street, pot, behind):
        f32 = np.float32
        if street == 1:
            self.kind[me] = LEAF
            self.stake[me] = float(f32(pot))
            self.stack[me] = float(f32(behind))
            self.leaf_index[me] = len(self.leaves)
            self.leaves.append(me)
            return
        self.kind[me] = DEAL
        for c in range(52):
            if (self.flop >> c) & 1:
                continue
            b = self.board[me] | (1 << c)
            ch = self._node(DECISION, 0, me, -1, self.level[me] + 1, 1, b)
            self.children[me].append(ch)
            self._decide(ch, 1, pot, behind, 0.0, 0.0, 0, 0)

    def _decide(self, me, street, pot, stack, c0, c1, actor, raises):
        # chip arithmetic in single precision, as the library states it
        f32 = np.float32
        fracs, allin, max_raises = self.streets[street]
        mine, theirs = (c0, c1) if actor == 0 else (c1, c0)
        behind = float(f32(f32(stack) - f32(mine)))
        owe = float(f32(f32(theirs) - f32(mine)))
        now = float(f32(f32(f32(pot) + f32(c0)) + f32(c1)))
        acts = []  # (kind, chips)

        def offer(amount, floor):
            if any(k == "bet" and a == amount for k, a in acts):
                return
            if amount > floor:
                acts.append(("bet", amount))

        if owe <= 0:
            acts.append(("check", 0.0))
            if raises < max_raises and behind > 0:
                for fr in fracs:
                    offer(min(float(f32(f32(fr) * f32(now))), behind), 0.0)
                if allin:
                    offer(behind, 0.0)
        else:
            acts.append(("fold", 0.0))
            acts.append(("call", owe))
            if raises < max_raises and behind > owe:
                for fr in fracs:
                    offer(min(float(f32(f32(owe) + f32(f32(fr) * f32(f32(now) + f32(owe))))), behind), owe)
                if allin:
                    offer(behind, owe)
        e0 = self.edges
        self.edges += len(acts)
        self.first_edge[me] = e0
        lvl = self.level[me]
        board = self.board[me]
        for a, (k, chips) in enumerate(acts):
            if k == "check" and actor == 0:
                ch = self._node(DECISION, 1, me, e0 + a, lvl + 1, street, board)
                self.children[me].append(ch)
                self._decide(ch, street, pot, stack, c0, c1, 1, raises)
            elif k == "check":
                ch = self._node(LEAF, 0, me, e0 + a, lvl + 1, street, board)
                self.children[me].append(ch)
                self._end(ch, street, float(f32(f32(f32(pot) + f32(c0)) + f32(c1))), float(f32(f32(stack) - f32(c0))))
            elif k == "bet":
                n0 = float(f32(f32(c0) + f32(chips))) if actor == 0 else c0
                n1 = float(f32(f32(c1) + f32(chips))) if actor == 1 else c1
                ch = self._node(DECISION, 1 - actor, me, e0 + a, lvl + 1, street, board)
                self.children[me].append(ch)
                self._decide(ch, street, pot, stack, n0, n1, 1 - actor, raises + 1)
            elif k == "fold":
                ch = self._node(FOLD, actor, me, e0 + a, lvl + 1, street, board)
                self.stake[ch] = float(f32(f32(f32(0.5) * f32(pot)) + f32(mine)))
                self.children[me].append(ch)
            else:  # call
                ch = self._node(LEAF, 0, me, e0 + a, lvl + 1, street, board)
                self.children[me].append(ch)
                self._end(ch, street, float(f32(f32(pot) + f32(f32(2.0) * f32(theirs)))),
                          float(f32(f32(stack) - f32(theirs))))

    def __len__(self):
        return len(self.kind)


def _strategy(src, first, n, average):
    """[n][HANDS] strategy of a decision node from its rows (regrets or average sums)."""
    rows = np.maximum(src[first:first + n].astype(np.float64), 0.0)
    s = rows.sum(axis=0)
    cut = 0.0 if average else float(np.float32(1e-4))
    uni = s <= cut
    out = np.where(uni[None, :], 1.0 / n, rows / np.where(uni, 1.0, s)[None, :])
    return out


def reach(tree, init, src, average):
    """Top-down reach [nodes][2][HANDS] (float64) from the initial ranges [2][HANDS]."""
    N = len(tree)
    R = np.zeros((N, 2, HANDS))
    R[0] = np.where(blocked(tree.flop)[None, :], 0.0, init)
    for i in range(N):
        k = tree.kind[i]
        if k == DECISION:
            n = len(tree.children[i])
            sg = _strategy(src, tree.first_edge[i], n, average)
            for a, ch in enumerate(tree.children[i]):
                R[ch] = R[i]
                R[ch, tree.actor[i]] = R[i, tree.actor[i]] * sg[a]
        elif k == DEAL:
            for ch in tree.children[i]:
                dealt = tree.board[ch] & ~tree.board[i]
                R[ch] = np.where(blocked(dealt)[None, :], 0.0, R[i])
    return R


def sweep_up(tree, R, leafV, upd, src, average, mode, regrets=None, avg=None):
    """Bottom-up values of `upd` [nodes][HANDS]; mode "cfr" also returns updated regrets and
    average sums (float64 arrays), "br" takes the maximum at upd's decisions."""
    N = len(tree)
    V = np.zeros((N, HANDS))
    reg = None if regrets is None else regrets.astype(np.float64).copy()
    av = None if avg is None else avg.astype(np.float64).copy()
    for i in range(N - 1, -1, -1):
        k = tree.kind[i]
        if k == LEAF:
            V[i] = leafV[tree.leaf_index[i]]
        elif k == FOLD:
            opp = R[i, 1 - upd]
            sign = -1.0 if tree.actor[i] == upd else 1.0
            V[i] = sign * tree.stake[i] * (_COMPAT @ opp)
        elif k == DEAL:
            acc = np.zeros(HANDS)
            for ch in tree.children[i]:
                dealt = tree.board[ch] & ~tree.board[i]
                acc += np.where(blocked(dealt), 0.0, V[ch])
            V[i] = acc / len(tree.children[i])
        else:
            kids = tree.children[i]
            n = len(kids)
            U = np.stack([V[c] for c in kids])
            if tree.actor[i] != upd:
                V[i] = U.sum(axis=0)
            elif mode == "br":
                V[i] = U.max(axis=0)
            else:
                sg = _strategy(src, tree.first_edge[i], n, average)
                V[i] = (sg * U).sum(axis=0)
                if mode == "cfr":
                    e0 = tree.first_edge[i]
                    reg[e0:e0 + n] = np.maximum(reg[e0:e0 + n] + U - V[i][None, :], 0.0)
                    if av is not None:
                        av[e0:e0 + n] += R[i, upd][None, :] * sg
    return V, reg, av


def joint(init, flop):
    """Sum over clash-free hand pairs off the flop of r0(h) r1(o)."""
    off = ~blocked(flop)
    r0 = np.where(off, init[0], 0.0).astype(np.float64)
    r1 = np.where(off, init[1], 0.0).astype(np.float64)
    return float(r0 @ _COMPAT @ r1)
