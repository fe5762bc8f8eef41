"""Python loader for the oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: the CPU restatement of the reference's river-subtree CFR path
(see oracle.h for the reference file:line each part follows). tests/, the smoke check and
the CPU-baseline legs of bench.py use it as the checker or the timed CPU baseline; the
product package never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO_PATH = os.path.join(HERE, "_build", "liboracle.so")
HANDS = 1326
EVAL_LEN = 1326 + 512
COLL_LEN = 52 * 51
EDGES = 26
BUCKETS = 256
REFERENCE_FLOP = 0b111  # cards {0, 1, 2}: the reference's fixed flop (game.rs:70-71)

_lib = None


REF_SO = os.path.join(HERE, "_ref", "libpoker_ref.so")


def reference_tree():
    """The reference checkout whose src/cuda the `ref` recipe compiles: the environment
    variable POKERRUST_REFERENCE, else the default the Makefile names; None if absent."""
    tree = os.environ.get("POKERRUST_REFERENCE")
    if not tree:
        out = subprocess.run(["make", "-s", "-C", HERE, "--no-print-directory", "print-reference"],
                             capture_output=True, text=True)
        tree = out.stdout.strip() if out.returncode == 0 else ""
    return tree if tree and os.path.isdir(os.path.join(tree, "src", "cuda")) else None


def build():
    """Compiles the oracle with its Makefile (g++) and, where the reference sources are
    present, the reference's own CUDA library into oracle/_ref (nvcc)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    tree = reference_tree()
    if tree:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE={tree}"], check=True)
    return SO_PATH


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(SO_PATH):
            build()
        L = ctypes.CDLL(SO_PATH)
        vp, u64, i32, f32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_float
        L.or_choose.restype = ctypes.c_int64
        L.or_choose.argtypes = [i32, i32]
        L.or_colex_index.restype = ctypes.c_int64
        L.or_colex_index.argtypes = [u64]
        L.or_pair_from_index.restype = u64
        L.or_pair_from_index.argtypes = [i32]
        L.or_card_order.argtypes = [vp]
        L.or_card_indexes.argtypes = [vp]
        L.or_hand_value.restype = ctypes.c_uint32
        L.or_hand_value.argtypes = [u64]
        L.or_count_7card.argtypes = [vp, vp, i32]
        L.or_board_tables.argtypes = [u64, vp, vp, vp]
        L.or_pack_flop_tables.argtypes = [u64, vp, vp, vp, i32]
        L.or_river_tree.argtypes = [vp] * 8
        L.or_set_river_order.argtypes = [i32]
        L.or_river_batch.restype = i32
        L.or_river_batch.argtypes = [u64, vp, vp, i32, vp, vp, vp, vp, i32, i32, vp, i32]
        L.or_river_batch_avg.restype = i32
        L.or_river_batch_avg.argtypes = [u64, vp, vp, i32, vp, vp, vp, vp, vp, vp, i32, vp, i32]
        L.or_river_br_f64.restype = i32
        L.or_river_br_f64.argtypes = [u64, vp, vp, i32, vp, vp, vp, vp, i32, vp, i32]
        L.or_game_new.restype = vp
        L.or_game_new.argtypes = [u64, i32]
        L.or_game_free.argtypes = [vp]
        L.or_game_num_rivers.restype = i32
        L.or_game_num_rivers.argtypes = [vp]
        L.or_game_river_roots.argtypes = [vp, vp, vp]
        L.or_game_iterate.argtypes = [vp]
        L.or_game_exploitability.argtypes = [vp, i32, vp, vp, vp]
        L.or_game_river_regrets.argtypes = [vp, vp]
        L.or_game_enable_average.argtypes = [vp]
        L.or_game_root_values.restype = i32
        L.or_game_root_values.argtypes = [vp, vp, vp]
        L.or_game_totals.argtypes = [vp, vp, vp, vp, vp]
        L.or_game_river_average.restype = i32
        L.or_game_river_average.argtypes = [vp, vp]
        L.or_bet_tree.restype = i32
        L.or_bet_tree.argtypes = [f32, f32, ctypes.c_uint32, i32] + [vp] * 7 + [i32, vp, vp, vp]
        L.or_sub_new.restype = vp
        L.or_sub_new.argtypes = [u64, f32, f32, ctypes.c_uint32, i32, vp, vp]
        L.or_sub_free.argtypes = [vp]
        L.or_sub_edges.restype = i32
        L.or_sub_edges.argtypes = [vp]
        L.or_sub_get.argtypes = [vp, i32, vp]
        L.or_sub_set.argtypes = [vp, i32, vp]
        L.or_sub_cfr_half.argtypes = [vp, i32, i32]
        L.or_sub_best_response.restype = ctypes.c_double
        L.or_sub_best_response.argtypes = [vp, i32, i32, vp]
        L.or_sub_value.restype = ctypes.c_double
        L.or_sub_value.argtypes = [vp, i32, i32, vp]
        L.or_sub_joint.restype = ctypes.c_double
        L.or_sub_joint.argtypes = [vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def card_order():
    out = np.zeros(HANDS, np.uint64)
    load().or_card_order(_p(out))
    return out


def card_indexes():
    out = np.zeros(COLL_LEN, np.uint16)
    load().or_card_indexes(_p(out))
    return out


def hand_value(cards):
    return int(load().or_hand_value(int(cards)))


def count_7card(nthreads=0):
    counts = np.zeros(9, np.int64)
    distinct = ctypes.c_int64()
    load().or_count_7card(_p(counts), ctypes.byref(distinct), nthreads)
    return counts, distinct.value


def board_tables(board5):
    e = np.zeros(EVAL_LEN, np.uint16)
    c = np.zeros(COLL_LEN, np.uint16)
    a = np.zeros(HANDS, np.uint16)
    load().or_board_tables(int(board5), _p(e), _p(c), _p(a))
    return e, c, a


def pack_flop_tables(flop=REFERENCE_FLOP, nthreads=0):
    """(eval, coll, abstr) as cuda_interface.rs:444-479 packs them for transfer_flop_eval_cuda."""
    e = np.zeros(HANDS * EVAL_LEN, np.uint16)
    c = np.zeros(HANDS * COLL_LEN, np.uint16)
    a = np.zeros(HANDS * HANDS, np.uint16)
    load().or_pack_flop_tables(int(flop), _p(e), _p(c), _p(a), nthreads)
    return e, c, a


def set_river_order(descending):
    """Visit the 48 river cards of every later river pass in descending order (True) or in
    the reference's ascending order (False): the same sums in another f32 rounding."""
    load().or_set_river_order(int(bool(descending)))


def river_tree():
    i = lambda n: np.zeros(n, np.int32)
    term, actor, parent, nchild = i(28), i(28), i(28), i(28)
    child, edge = i(84), i(84)
    sb, bb = np.zeros(28, np.float32), np.zeros(28, np.float32)
    load().or_river_tree(_p(term), _p(actor), _p(parent), _p(sb), _p(bb), _p(nchild), _p(child), _p(edge))
    return dict(terminal=term, actor=actor, parent=parent, sb_off=sb, bb_off=bb, nchild=nchild,
                child=child.reshape(28, 3), edge=edge.reshape(28, 3))


def river_batch(flop, eval_tables, abstr, board4, bet, opp_range, regrets, player, calc_exploit,
                nthreads=0):
    """One river pass per subgame (state.rs:377-433); regrets are updated in place."""
    board4 = np.ascontiguousarray(board4, np.uint64)
    bet = np.ascontiguousarray(bet, np.float32)
    opp = np.ascontiguousarray(opp_range, np.float32)
    assert regrets.dtype == np.float32 and regrets.flags.c_contiguous
    n = board4.size
    out = np.zeros((n, HANDS), np.float32)
    err = load().or_river_batch(int(flop), _p(eval_tables), _p(abstr), n, _p(board4), _p(bet), _p(opp),
                                _p(regrets), int(player), int(bool(calc_exploit)), _p(out), nthreads)
    if err:
        raise AssertionError(f"oracle river pass hit a reference assertion (code {err})")
    return out


def river_batch_avg(flop, eval_tables, abstr, board4, bet, opp_range, own_range, regrets, avg, player,
                    nthreads=0):
    """A CFR pass that also accumulates average-strategy sums into `avg` (in place)."""
    board4 = np.ascontiguousarray(board4, np.uint64)
    bet = np.ascontiguousarray(bet, np.float32)
    opp = np.ascontiguousarray(opp_range, np.float32)
    own = np.ascontiguousarray(own_range, np.float32)
    assert regrets.dtype == np.float32 and regrets.flags.c_contiguous
    assert avg.dtype == np.float32 and avg.flags.c_contiguous
    n = board4.size
    out = np.zeros((n, HANDS), np.float32)
    err = load().or_river_batch_avg(int(flop), _p(eval_tables), _p(abstr), n, _p(board4), _p(bet), _p(opp),
                                    _p(own), _p(regrets), _p(avg), int(player), _p(out), nthreads)
    if err:
        raise AssertionError(f"oracle river pass hit a reference assertion (code {err})")
    return out


def river_br_f64(flop, eval_tables, abstr, board4, bet, opp_range, regrets, player, nthreads=0):
    board4 = np.ascontiguousarray(board4, np.uint64)
    bet = np.ascontiguousarray(bet, np.float64)
    opp = np.ascontiguousarray(opp_range, np.float64)
    regrets = np.ascontiguousarray(regrets, np.float32)
    n = board4.size
    out = np.zeros((n, HANDS), np.float64)
    err = load().or_river_br_f64(int(flop), _p(eval_tables), _p(abstr), n, _p(board4), _p(bet), _p(opp),
                                 _p(regrets), int(player), _p(out), nthreads)
    if err:
        raise AssertionError(f"oracle river pass hit a reference assertion (code {err})")
    return out


class Game:
    """The full fixed-flop game of the reference on the CPU (builder.rs, state.rs, game.rs)."""

    def __init__(self, flop=REFERENCE_FLOP, nthreads=0):
        self.ptr = load().or_game_new(int(flop), nthreads)

    @property
    def num_rivers(self):
        return load().or_game_num_rivers(self.ptr)

    def river_roots(self):
        n = self.num_rivers
        b = np.zeros(n, np.uint64)
        bet = np.zeros(n, np.float32)
        load().or_game_river_roots(self.ptr, _p(b), _p(bet))
        return b, bet

    def iterate(self):
        load().or_game_iterate(self.ptr)

    def exploitability(self, use_f64=False):
        a, b, m = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        load().or_game_exploitability(self.ptr, int(bool(use_f64)), ctypes.byref(a), ctypes.byref(b),
                                      ctypes.byref(m))
        return a.value, b.value, m.value

    def river_regrets(self):
        out = np.zeros((self.num_rivers, EDGES, BUCKETS), np.float32)
        load().or_game_river_regrets(self.ptr, _p(out))
        return out

    def enable_average(self):
        load().or_game_enable_average(self.ptr)

    def root_values(self):
        """The root's values of the last iteration's SB and BB CFR passes, [2][1326] f32."""
        out = np.zeros((2, HANDS), np.float32)
        if load().or_game_root_values(self.ptr, _p(out[0]), _p(out[1])):
            raise ValueError("no iteration yet")
        return out

    def totals(self):
        """Sums of all upper regrets, upper average sums, river regrets, river average sums."""
        v = [ctypes.c_double() for _ in range(4)]
        load().or_game_totals(self.ptr, *[ctypes.byref(x) for x in v])
        return np.array([x.value for x in v])

    def river_average(self):
        out = np.zeros((self.num_rivers, EDGES, BUCKETS), np.float32)
        if load().or_game_river_average(self.ptr, _p(out)):
            raise ValueError("average sums are off")
        return out

    def __del__(self):
        try:
            if self.ptr:
                load().or_game_free(self.ptr)
        except Exception:
            pass


# ---- general river subgames (the batch solver's rules) ----

def bet_tree(pot, stack, sizes, max_raises, max_nodes=512):
    """The subgame's tree in pre-order: dict of per-node arrays and counts."""
    i = lambda: np.zeros(max_nodes, np.int32)
    kind, actor, parent, in_edge, nchild, depth = i(), i(), i(), i(), i(), i()
    stake = np.zeros(max_nodes, np.float32)
    n, e, l = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    st = load().or_bet_tree(float(pot), float(stack), int(sizes), int(max_raises), _p(kind), _p(actor),
                            _p(parent), _p(in_edge), _p(nchild), _p(stake), _p(depth), max_nodes,
                            ctypes.byref(n), ctypes.byref(e), ctypes.byref(l))
    if st:
        raise ValueError(f"or_bet_tree failed ({st})")
    k = n.value
    return dict(kind=kind[:k], actor=actor[:k], parent=parent[:k], in_edge=in_edge[:k], nchild=nchild[:k],
                stake=stake[:k], depth=depth[:k], num_edges=e.value, num_leaves=l.value)


class Subgame:
    """One general river subgame on the CPU: per-hand CFR in single precision, best
    response and strategy evaluation in double precision (colex hand order)."""

    def __init__(self, board, pot, stack, sizes, max_raises, r0, r1):
        self._r = [np.ascontiguousarray(r0, np.float32), np.ascontiguousarray(r1, np.float32)]
        self.ptr = load().or_sub_new(int(board), float(pot), float(stack), int(sizes), int(max_raises),
                                     _p(self._r[0]), _p(self._r[1]))
        if not self.ptr:
            raise ValueError("bad subgame")
        self.edges = load().or_sub_edges(self.ptr)

    def __del__(self):
        if getattr(self, "ptr", None):
            load().or_sub_free(self.ptr)
            self.ptr = None

    def _get(self, which):
        out = np.zeros((self.edges, HANDS), np.float32)
        load().or_sub_get(self.ptr, which, _p(out))
        return out

    def _set(self, which, v):
        v = np.ascontiguousarray(v, np.float32).reshape(self.edges, HANDS)
        load().or_sub_set(self.ptr, which, _p(v))

    regrets = property(lambda self: self._get(0), lambda self, v: self._set(0, v))
    average = property(lambda self: self._get(1), lambda self, v: self._set(1, v))

    def cfr_half(self, player, accumulate=False):
        load().or_sub_cfr_half(self.ptr, int(player), int(bool(accumulate)))

    def iterate(self, n=1, accumulate=False):
        for _ in range(n):
            self.cfr_half(0, accumulate)
            self.cfr_half(1, accumulate)

    def best_response(self, player, use_average=False):
        root = np.zeros(HANDS, np.float64)
        s = load().or_sub_best_response(self.ptr, int(player), int(bool(use_average)), _p(root))
        return s, root

    def value(self, player, use_average=False):
        root = np.zeros(HANDS, np.float64)
        s = load().or_sub_value(self.ptr, int(player), int(bool(use_average)), _p(root))
        return s, root

    def joint(self):
        return load().or_sub_joint(self.ptr)

    def exploitability(self, use_average=False):
        b0, _ = self.best_response(0, use_average)
        b1, _ = self.best_response(1, use_average)
        return b0, b1, (b0 + b1) / 2.0 / self.joint()
