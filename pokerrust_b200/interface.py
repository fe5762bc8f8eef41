"""Host-side mirror of the reference's Rust FFI wrapper (src/cuda_interface.rs:8-123),
over the C ABI of include/pokerrust_b200.h.

Function names, argument meaning and call order follow cuda_interface.rs:
initialize_builder / build_river at game construction, transfer_flop_eval + free_eval
around every iteration, upload_gpu / download_gpu per river root and evaluate_gpu per
half-iteration. There is no CPU fallback: loading fails loudly when the CUDA library has
not been built.
"""
import ctypes
import os

import numpy as np

from .build import SO_PATH

HANDS = 1326
RANGE_STRIDE = 1328
EDGES = 26
BUCKETS = 256

_lib = None


class SubgameSpec(ctypes.Structure):
    """pr_subgame: one general river subgame (board, pot, stack, bet sizes, raise cap)."""
    _fields_ = [("board", ctypes.c_uint64), ("pot", ctypes.c_float), ("stack", ctypes.c_float),
                ("sizes", ctypes.c_uint32), ("max_raises", ctypes.c_int32)]


SPEC_DTYPE = np.dtype([("board", "<u8"), ("pot", "<f4"), ("stack", "<f4"), ("sizes", "<u4"),
                       ("max_raises", "<i4")])


class StreetRules(ctypes.Structure):
    """pr_street: bet sizes of one street (pot fractions, all-in, raise cap)."""
    _fields_ = [("fracs", ctypes.c_float * 4), ("nfrac", ctypes.c_int32), ("allin", ctypes.c_int32),
                ("max_raises", ctypes.c_int32)]


class FullSpec(ctypes.Structure):
    """pr_full_spec: a fixed-flop game with general bets on the flop and turn and river
    subgames at the end of the turn."""
    _fields_ = [("flop", ctypes.c_uint64), ("pot", ctypes.c_float), ("stack", ctypes.c_float),
                ("street", StreetRules * 2), ("river_sizes", ctypes.c_uint32), ("river_raises", ctypes.c_int32)]


# the host tree's 48-byte nodes (full_tree.h: FNode)
FNODE_DTYPE = np.dtype([("kind", "u1"), ("actor", "u1"), ("nchild", "u1"), ("street", "u1"), ("parent", "<i4"),
                        ("in_edge", "<i4"), ("edge", "<i4"), ("kids", "<i4"), ("level", "<i4"),
                        ("stake", "<f4"), ("stack", "<f4"), ("pad", "<u4"), ("board", "<u8")], align=True)
assert FNODE_DTYPE.itemsize == 48


class PokerLibError(RuntimeError):
    pass


def lib():
    """The loaded CUDA library (pokerrust_b200/_lib/libpokerrust_b200.so)."""
    global _lib
    if _lib is None:
        if not os.path.exists(SO_PATH):
            raise PokerLibError(
                f"{SO_PATH} is missing: build it with `python -m pokerrust_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(SO_PATH)
        vp, u64, u16, f32, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint16, ctypes.c_float, ctypes.c_int
        fp = ctypes.POINTER(ctypes.c_float)
        L.init_builder.restype = vp
        L.init_builder.argtypes = []
        L.upload_c.argtypes = [vp, i32, fp]
        L.download_c.argtypes = [vp, i32, fp]
        L.build_river_cuda.restype = i32
        L.build_river_cuda.argtypes = [u64, f32, vp]
        L.transfer_flop_eval_cuda.restype = vp
        L.transfer_flop_eval_cuda.argtypes = [u64, vp, vp, vp, vp, vp]
        L.free_eval_cuda.argtypes = [vp]
        L.evaluate_cuda.argtypes = [vp, vp, u16, ctypes.c_bool]
        L.pr_last_error.restype = i32
        L.pr_error_string.restype = ctypes.c_char_p
        L.pr_error_string.argtypes = [i32]
        L.pr_evaluate.restype = i32
        L.pr_evaluate.argtypes = [vp, vp, i32, i32]
        L.pr_evaluate_device.restype = i32
        L.pr_evaluate_device.argtypes = [vp, vp, i32, i32, vp, vp, vp]
        L.pr_upload_batch.restype = i32
        L.pr_upload_batch.argtypes = [vp, i32, i32, vp]
        L.pr_download_batch.restype = i32
        L.pr_download_batch.argtypes = [vp, i32, i32, vp]
        L.pr_builder_count.restype = i32
        L.pr_builder_count.argtypes = [vp]
        L.pr_range_stride.restype = i32
        L.pr_get_regrets.restype = i32
        L.pr_get_regrets.argtypes = [vp, vp]
        L.pr_set_regrets.restype = i32
        L.pr_set_regrets.argtypes = [vp, vp]
        L.pr_free_builder.argtypes = [vp]
        L.pr_eval_status.restype = i32
        L.pr_eval_status.argtypes = [vp]
        L.pr_river_smem_bytes.restype = ctypes.c_size_t
        L.pr_river_smem_bytes.argtypes = [vp, i32, i32]
        L.pr_game_new.restype = vp
        L.pr_game_new.argtypes = [u64, i32]
        L.pr_game_free.argtypes = [vp]
        L.pr_game_num_rivers.restype = i32
        L.pr_game_num_rivers.argtypes = [vp]
        L.pr_game_river_roots.restype = i32
        L.pr_game_river_roots.argtypes = [vp, vp, vp]
        L.pr_game_builder.restype = vp
        L.pr_game_builder.argtypes = [vp]
        L.pr_game_tables.restype = vp
        L.pr_game_tables.argtypes = [vp]
        L.pr_game_iterate.restype = i32
        L.pr_game_iterate.argtypes = [vp, i32]
        L.pr_game_root_values.restype = i32
        L.pr_game_root_values.argtypes = [vp, vp, vp]
        sg = ctypes.POINTER(SubgameSpec)
        L.pr_batch_tree.restype = i32
        L.pr_batch_tree.argtypes = [sg, vp, vp, vp, vp]
        L.pr_batch_new.restype = vp
        L.pr_batch_new.argtypes = [sg, i32, vp]
        L.pr_batch_free.argtypes = [vp]
        L.pr_batch_count.restype = i32
        L.pr_batch_count.argtypes = [vp]
        L.pr_batch_shape.restype = i32
        L.pr_batch_shape.argtypes = [vp, i32, vp, vp, vp]
        L.pr_batch_enable_average.restype = i32
        L.pr_batch_enable_average.argtypes = [vp]
        L.pr_batch_iterate.restype = i32
        L.pr_batch_iterate.argtypes = [vp, i32]
        L.pr_batch_exploitability.restype = i32
        L.pr_batch_exploitability.argtypes = [vp, i32, i32, vp, vp, vp]
        L.pr_batch_root_values.restype = i32
        L.pr_batch_root_values.argtypes = [vp, i32, i32, vp, vp]
        for name in ("pr_batch_get_regrets", "pr_batch_set_regrets", "pr_batch_get_average",
                     "pr_batch_set_average"):
            getattr(L, name).restype = i32
            getattr(L, name).argtypes = [vp, i32, vp]
        L.pr_batch_config.restype = i32
        L.pr_batch_config.argtypes = [vp, i32, vp, vp, vp, vp]
        L.pr_batch_set_config.restype = i32
        L.pr_batch_set_config.argtypes = [vp, i32, i32, i32, i32]
        L.pr_batch_tune.restype = i32
        L.pr_batch_tune.argtypes = [vp, vp]
        L.pr_batch_get_all.restype = i32
        L.pr_batch_get_all.argtypes = [vp, i32, vp]
        L.pr_batch_iterate_noalloc.restype = i32
        L.pr_batch_iterate_noalloc.argtypes = [vp, i32]
        L.pr_gemm_bf16.restype = i32
        L.pr_gemm_bf16.argtypes = [vp, vp, vp, i32, i32, i32, i32, vp]
        L.pr_gemm_bf16_major.restype = i32
        L.pr_gemm_bf16_major.argtypes = [vp, vp, vp, i32, i32, i32, i32, i32, i32, vp]
        L.pr_gemm_bf16_async.restype = i32
        L.pr_gemm_bf16_async.argtypes = [vp, vp, vp, i32, i32, i32, i32, vp, vp]
        L.pr_gemm_bf16_persistent_async.restype = i32
        L.pr_gemm_bf16_persistent_async.argtypes = [vp, vp, vp, i32, i32, i32, i32, vp, vp]
        L.pr_gemm_bf16_persistent.restype = i32
        L.pr_gemm_bf16_persistent.argtypes = [vp, vp, vp, i32, i32, i32, i32, i32, i32, i32, vp]
        L.pr_gemm_bf16_wait_test.restype = i32
        L.pr_gemm_bf16_wait_test.argtypes = [vp, vp, vp, i32, i32, i32, i32, ctypes.c_uint64, i32, vp]
        L.pr_mlp_set_persistent.restype = i32
        L.pr_mlp_set_persistent.argtypes = [vp, i32]
        L.pr_mlp_new.restype = vp
        L.pr_mlp_new.argtypes = [i32, u64]
        L.pr_mlp_free.argtypes = [vp]
        L.pr_mlp_rows.restype = i32
        L.pr_mlp_rows.argtypes = [vp]
        L.pr_mlp_forward.restype = i32
        L.pr_mlp_forward.argtypes = [vp, vp, vp, vp, vp, i32]
        L.pr_mlp_train_step.restype = i32
        L.pr_mlp_train_step.argtypes = [vp, vp, vp, vp, vp, i32, f32, vp]
        L.pr_mlp_layer_shape.restype = i32
        L.pr_mlp_layer_shape.argtypes = [i32, vp, vp]
        for name in ("pr_mlp_get_layer", "pr_mlp_set_layer", "pr_mlp_get_grad"):
            getattr(L, name).restype = i32
            getattr(L, name).argtypes = [vp, i32, vp, vp]
        L.pr_batch_value.restype = i32
        L.pr_batch_value.argtypes = [vp, i32, vp]
        L.pr_batch_value_grad.restype = i32
        L.pr_batch_value_grad.argtypes = [vp, i32, vp, vp, vp]
        L.pr_batch_value_grad_device.restype = i32
        L.pr_batch_value_grad_device.argtypes = [vp, i32, vp, vp, vp]
        L.pr_batch_set_ranges.restype = i32
        L.pr_batch_set_ranges.argtypes = [vp, i32, vp]
        L.pr_batch_set_linear_average.restype = i32
        L.pr_batch_set_linear_average.argtypes = [vp, i32]
        L.pr_batch_iteration_bytes.restype = ctypes.c_double
        L.pr_batch_iteration_bytes.argtypes = [vp]
        L.pr_game_set_device_tree.restype = i32
        L.pr_game_set_device_tree.argtypes = [vp, i32]
        L.pr_evaluate_device_own.restype = i32
        L.pr_evaluate_device_own.argtypes = [vp, vp, i32, vp, vp, vp, vp]
        L.pr_evaluate_br64_device.restype = i32
        L.pr_evaluate_br64_device.argtypes = [vp, vp, i32, vp, vp, vp]
        L.pr_game_exploitability.restype = i32
        L.pr_game_exploitability.argtypes = [vp, i32, vp, vp, vp]
        L.pr_game_timings.restype = i32
        L.pr_game_timings.argtypes = [vp, vp, vp]
        L.pr_game_upper_regret_count.restype = ctypes.c_size_t
        L.pr_game_upper_regret_count.argtypes = [vp]
        L.pr_game_enable_average.restype = i32
        L.pr_game_enable_average.argtypes = [vp]
        L.pr_game_get_average.restype = i32
        L.pr_game_get_average.argtypes = [vp, vp, vp]
        L.pr_set_average.restype = i32
        L.pr_set_average.argtypes = [vp, vp]
        L.pr_game_save.restype = i32
        L.pr_game_save.argtypes = [vp, ctypes.c_char_p]
        L.pr_game_load.restype = i32
        L.pr_game_load.argtypes = [vp, ctypes.c_char_p]
        L.pr_game_get_regrets.restype = i32
        L.pr_game_get_regrets.argtypes = [vp, vp, vp]
        L.pr_game_set_regrets.restype = i32
        L.pr_game_set_regrets.argtypes = [vp, vp, vp]
        L.pr_enable_average.restype = i32
        L.pr_enable_average.argtypes = [vp]
        L.pr_upload_own.argtypes = [vp, i32, ctypes.POINTER(ctypes.c_float)]
        L.pr_get_average.restype = i32
        L.pr_get_average.argtypes = [vp, vp]
        L.pr_evaluate_br64.restype = i32
        L.pr_evaluate_br64.argtypes = [vp, vp, i32, vp, vp]
        L.pr_tables_build.restype = vp
        L.pr_tables_build.argtypes = [u64]
        L.pr_tables_export.restype = i32
        L.pr_tables_export.argtypes = [vp, vp, vp, vp]
        L.pr_tables_save.restype = i32
        L.pr_tables_save.argtypes = [vp, ctypes.c_char_p]
        L.pr_tables_load.restype = vp
        L.pr_tables_load.argtypes = [ctypes.c_char_p]
        fs = ctypes.POINTER(FullSpec)
        L.pr_full_tree.restype = i32
        L.pr_full_tree.argtypes = [fs, vp, i32, vp, vp, vp, vp, i32]
        L.pr_full_new.restype = vp
        L.pr_full_new.argtypes = [fs, vp]
        L.pr_full_free.argtypes = [vp]
        L.pr_full_shape.restype = i32
        L.pr_full_shape.argtypes = [vp, vp, vp, vp, vp, vp]
        L.pr_full_set_zero_sum.restype = i32
        L.pr_full_set_zero_sum.argtypes = [vp, i32]
        L.pr_full_set_net.restype = i32
        L.pr_full_set_net.argtypes = [vp, vp]
        L.pr_full_pass.restype = i32
        L.pr_full_pass.argtypes = [vp, i32]
        L.pr_full_iterate.restype = i32
        L.pr_full_iterate.argtypes = [vp, i32]
        L.pr_full_exploitability.restype = i32
        L.pr_full_exploitability.argtypes = [vp, i32, vp, vp, vp]
        L.pr_full_read.restype = i32
        L.pr_full_read.argtypes = [vp, i32, vp]
        L.pr_full_tune.restype = i32
        L.pr_full_tune.argtypes = [vp, vp]
        L.pr_full_set_linear_average.restype = i32
        L.pr_full_set_linear_average.argtypes = [vp, i32]
        L.pr_full_reset.restype = i32
        L.pr_full_reset.argtypes = [vp]
        L.pr_full_write.restype = i32
        L.pr_full_write.argtypes = [vp, i32, vp]
        L.pr_full_batch.restype = vp
        L.pr_full_batch.argtypes = [vp, i32]
        L.pr_full_batch_leaves.restype = i32
        L.pr_full_batch_leaves.argtypes = [vp, i32, vp]
        L.pr_full_joint.restype = ctypes.c_double
        L.pr_full_joint.argtypes = [vp]
        _lib = L
    return _lib


def _check(status, what):
    if status != 0:
        raise PokerLibError(f"{what}: {lib().pr_error_string(status).decode()} (status {status})")


def card_order():
    """The 1326 two-card hands as 52-bit masks in colex order (src/evaluator.rs:29-40)."""
    out = np.zeros(HANDS, np.uint64)
    n = 0
    for hi in range(1, 52):
        for lo in range(hi):
            out[n] = (1 << lo) | (1 << hi)
            n += 1
    return out


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def initialize_builder():
    """cuda_interface.rs:432-434."""
    p = lib().init_builder()
    if not p:
        _check(lib().pr_last_error() or 1, "init_builder")
    return p


def build_river(cards, bet, builder):
    """cuda_interface.rs:435-437: adds a river root, returns its index."""
    idx = lib().build_river_cuda(int(cards), float(bet), builder)
    if idx < 0:
        _check(lib().pr_last_error() or 2, "build_river_cuda")
    return idx


def upload_gpu(builder, index, v):
    """cuda_interface.rs:423-425."""
    v = np.ascontiguousarray(v, dtype=np.float32)
    assert v.shape == (HANDS,)
    lib().upload_c(builder, int(index), v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))


def download_gpu(builder, index):
    """cuda_interface.rs:427-431."""
    out = np.zeros(HANDS, dtype=np.float32)
    lib().download_c(builder, int(index), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    return out


def transfer_flop_eval(flop, card_order, card_indexes, eval_tables, coll_vec, abstractions):
    """cuda_interface.rs:438-492 after packing: the packed tables of all 1326 {turn, river}
    slots for `flop` (1326*1838, 1326*2652 and 1326*1326 u16) go to the device."""
    card_order = np.ascontiguousarray(card_order, dtype=np.uint64)
    card_indexes = np.ascontiguousarray(card_indexes, dtype=np.uint16)
    eval_tables = np.ascontiguousarray(eval_tables, dtype=np.uint16)
    coll_vec = np.ascontiguousarray(coll_vec, dtype=np.uint16)
    abstractions = np.ascontiguousarray(abstractions, dtype=np.uint16)
    assert card_order.size == HANDS and card_indexes.size == 52 * 51
    assert eval_tables.size == HANDS * (HANDS + 512)
    assert coll_vec.size == HANDS * 52 * 51 and abstractions.size == HANDS * HANDS
    p = lib().transfer_flop_eval_cuda(int(flop), _ptr(card_order), _ptr(card_indexes), _ptr(eval_tables),
                                      _ptr(coll_vec), _ptr(abstractions))
    st = lib().pr_eval_status(p)
    if st != 0:
        lib().free_eval_cuda(p)
        raise PokerLibError(f"transfer_flop_eval_cuda rejected the tables (bits {st})")
    return p


def build_flop_tables(flop):
    """Hand-rank tables of every river board of `flop`, generated on the device (no host
    tables needed); usable wherever transfer_flop_eval's handle is."""
    p = lib().pr_tables_build(int(flop))
    st = lib().pr_eval_status(p)
    if st != 0:
        lib().free_eval_cuda(p)
        raise PokerLibError(f"pr_tables_build failed (status {st})")
    return p


def export_tables(ptr):
    """The handle's tables in the reference's packed layout: (eval, coll, abstractions)."""
    e = np.zeros(HANDS * (HANDS + 512), np.uint16)
    c = np.zeros(HANDS * 52 * 51, np.uint16)
    a = np.zeros(HANDS * HANDS, np.uint16)
    _check(lib().pr_tables_export(ptr, _ptr(e), _ptr(c), _ptr(a)), "pr_tables_export")
    return e, c, a


def save_tables(ptr, path):
    """Writes a table handle's packed tables to a checksummed file (pr_tables_save)."""
    _check(lib().pr_tables_save(ptr, os.fsencode(path)), "pr_tables_save")


def load_tables(path):
    """Reads a table file into a device table handle (pr_tables_load)."""
    ptr = lib().pr_tables_load(os.fsencode(path))
    if not ptr:
        raise PokerLibError(f"pr_tables_load failed for {path}")
    return ptr


def free_eval(ptr):
    """cuda_interface.rs:494-498."""
    lib().free_eval_cuda(ptr)


def evaluate_gpu(builder, evaluator, updating_player, calc_exploit):
    """cuda_interface.rs:500-513; updating_player is 0 (small) or 1 (big)."""
    lib().pr_clear_error()
    lib().evaluate_cuda(builder, evaluator, int(updating_player), bool(calc_exploit))
    _check(lib().pr_last_error(), "evaluate_cuda")


class Builder:
    """Owning wrapper with batch access, for drivers and tests."""

    def __init__(self):
        self.ptr = initialize_builder()
        self.owner = True

    @classmethod
    def wrap(cls, ptr):
        """A non-owning view of a builder owned elsewhere (e.g. by a Game)."""
        b = cls.__new__(cls)
        b.ptr = ptr
        b.owner = False
        return b

    def add(self, cards, bet):
        return build_river(cards, bet, self.ptr)

    @property
    def count(self):
        return lib().pr_builder_count(self.ptr)

    def upload_all(self, ranges):
        ranges = np.ascontiguousarray(ranges, dtype=np.float32)
        assert ranges.shape == (self.count, HANDS)
        _check(lib().pr_upload_batch(self.ptr, 0, self.count, _ptr(ranges)), "pr_upload_batch")

    def download_all(self, out=None):
        """All rows of the staging ([count][1326] floats), into `out` when given (a caller that
        reuses its buffers, as the reference's Rust caller reuses its vectors)."""
        if out is None:
            out = np.zeros((self.count, HANDS), dtype=np.float32)
        assert out.shape == (self.count, HANDS) and out.dtype == np.float32 and out.flags.c_contiguous
        _check(lib().pr_download_batch(self.ptr, 0, self.count, _ptr(out)), "pr_download_batch")
        return out

    def regrets(self):
        out = np.zeros((self.count, EDGES, BUCKETS), dtype=np.float32)
        _check(lib().pr_get_regrets(self.ptr, _ptr(out)), "pr_get_regrets")
        return out

    def enable_average(self):
        _check(lib().pr_enable_average(self.ptr), "pr_enable_average")

    def upload_own_all(self, ranges):
        ranges = np.ascontiguousarray(ranges, dtype=np.float32)
        assert ranges.shape == (self.count, HANDS)
        fp = ctypes.POINTER(ctypes.c_float)
        for i in range(self.count):
            lib().pr_upload_own(self.ptr, i, ranges[i].ctypes.data_as(fp))

    def average_sums(self):
        out = np.zeros((self.count, EDGES, BUCKETS), dtype=np.float32)
        _check(lib().pr_get_average(self.ptr, _ptr(out)), "pr_get_average")
        return out

    def set_regrets(self, regrets):
        regrets = np.ascontiguousarray(regrets, dtype=np.float32)
        assert regrets.shape == (self.count, EDGES, BUCKETS)
        _check(lib().pr_set_regrets(self.ptr, _ptr(regrets)), "pr_set_regrets")

    def evaluate(self, tables, updating_player, calc_exploit=False):
        _check(lib().pr_evaluate(self.ptr, tables, int(updating_player), int(bool(calc_exploit))), "pr_evaluate")

    def best_response_f64(self, tables, updating_player, ranges):
        """Double-precision best-response values for every subgame (count x 1326)."""
        ranges = np.ascontiguousarray(ranges, dtype=np.float64)
        assert ranges.shape == (self.count, HANDS)
        out = np.zeros((self.count, HANDS), np.float64)
        _check(lib().pr_evaluate_br64(self.ptr, tables, int(updating_player), _ptr(ranges), _ptr(out)),
               "pr_evaluate_br64")
        return out

    def evaluate_device(self, tables, updating_player, calc_exploit, d_ranges, d_results, stream=None):
        _check(lib().pr_evaluate_device(self.ptr, tables, int(updating_player), int(bool(calc_exploit)),
                                        ctypes.c_void_p(d_ranges), ctypes.c_void_p(d_results),
                                        ctypes.c_void_p(stream) if stream else None),
               "pr_evaluate_device")

    def close(self):
        if self.ptr and self.owner:
            lib().pr_free_builder(self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Game:
    """The whole fixed-flop game (src/game.rs) on the device: tables generated on the GPU,
    river subgames on the GPU, and the preflop/flop/turn tree on the GPU as well
    (device_tree=True, one CUDA graph per iteration) or on the host through the reference's
    upload / evaluate / download protocol (device_tree=False)."""

    def __init__(self, flop, nthreads=0, device_tree=True):
        self.ptr = lib().pr_game_new(int(flop), int(nthreads))
        if not self.ptr:
            raise PokerLibError(f"pr_game_new failed (status {lib().pr_last_error()})")
        self.set_device_tree(device_tree)

    def set_device_tree(self, on):
        return bool(lib().pr_game_set_device_tree(self.ptr, int(bool(on))))

    @property
    def num_rivers(self):
        return lib().pr_game_num_rivers(self.ptr)

    def river_roots(self):
        n = self.num_rivers
        boards = np.zeros(n, np.uint64)
        bets = np.zeros(n, np.float32)
        _check(lib().pr_game_river_roots(self.ptr, _ptr(boards), _ptr(bets)), "pr_game_river_roots")
        return boards, bets

    @property
    def builder(self):
        return lib().pr_game_builder(self.ptr)

    @property
    def tables(self):
        return lib().pr_game_tables(self.ptr)

    def iterate(self, iterations=1):
        _check(lib().pr_game_iterate(self.ptr, int(iterations)), "pr_game_iterate")

    def root_values(self):
        """The root's values of the last iteration's SB and BB CFR passes, [2][1326] f32."""
        out = np.zeros((2, HANDS), np.float32)
        _check(lib().pr_game_root_values(self.ptr, _ptr(out[0]), _ptr(out[1])), "pr_game_root_values")
        return out

    def exploitability(self, fp64=False):
        a, b, m = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(lib().pr_game_exploitability(self.ptr, int(bool(fp64)), ctypes.byref(a), ctypes.byref(b),
                                            ctypes.byref(m)), "pr_game_exploitability")
        return a.value, b.value, m.value

    def timings(self):
        h, d = ctypes.c_double(), ctypes.c_double()
        _check(lib().pr_game_timings(self.ptr, ctypes.byref(h), ctypes.byref(d)), "pr_game_timings")
        return h.value, d.value

    def regrets(self):
        up = np.zeros(lib().pr_game_upper_regret_count(self.ptr), np.float32)
        riv = np.zeros((self.num_rivers, EDGES, BUCKETS), np.float32)
        _check(lib().pr_game_get_regrets(self.ptr, _ptr(up), _ptr(riv)), "pr_game_get_regrets")
        return up, riv

    def set_regrets(self, upper=None, river=None):
        """Replaces the upper-tree regrets and/or the river regrets (layouts of regrets())."""
        up = None if upper is None else np.ascontiguousarray(upper, dtype=np.float32)
        riv = None if river is None else np.ascontiguousarray(river, dtype=np.float32)
        if up is not None:
            assert up.shape == (lib().pr_game_upper_regret_count(self.ptr),)
        if riv is not None:
            assert riv.shape == (self.num_rivers, EDGES, BUCKETS)
        _check(lib().pr_game_set_regrets(self.ptr, None if up is None else _ptr(up),
                                         None if riv is None else _ptr(riv)), "pr_game_set_regrets")

    def enable_average(self):
        _check(lib().pr_game_enable_average(self.ptr), "pr_game_enable_average")

    def save(self, path):
        st = lib().pr_game_save(self.ptr, os.fsencode(path))
        if st:
            raise PokerLibError(f"pr_game_save failed ({st})")

    def load(self, path):
        st = lib().pr_game_load(self.ptr, os.fsencode(path))
        if st:
            raise PokerLibError(f"pr_game_load failed ({st}): wrong game, corrupted or unreadable file")

    def average_sums(self):
        up = np.zeros(lib().pr_game_upper_regret_count(self.ptr), np.float32)
        riv = np.zeros((self.num_rivers, EDGES, BUCKETS), np.float32)
        _check(lib().pr_game_get_average(self.ptr, _ptr(up), _ptr(riv)), "pr_game_get_average")
        return up, riv

    def close(self):
        if self.ptr:
            lib().pr_game_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- batched general river subgames ----

def bet_tree(pot, stack, sizes, max_raises):
    """The library's tree of one subgame: structured array of nodes (pre-order) and counts."""
    spec = SubgameSpec(0, float(pot), float(stack), int(sizes), int(max_raises))
    nodes = np.zeros(128, np.dtype([("kind", "u1"), ("actor", "u1"), ("nchild", "u1"), ("depth", "u1"),
                                    ("parent", "<u2"), ("in_edge", "<u2"), ("edge", "<u2"), ("pad", "<u2"),
                                    ("stake", "<f4")]))
    n, e, l = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib().pr_batch_tree(ctypes.byref(spec), _ptr(nodes), ctypes.byref(n), ctypes.byref(e),
                               ctypes.byref(l)), "pr_batch_tree")
    return nodes[:n.value], e.value, l.value


def random_subgames(count, seed=0, max_nodes=60):
    """Seeded general river subgames: 5 distinct board cards; pot ~ U{2..200}; stack ~
    U{pot..10 pot}; a non-empty subset of {half pot, pot, all-in} and 1-3 bets and raises,
    redrawn until the tree has at most `max_nodes` nodes; ranges U(0,1) per hand with 25 %
    zeroed, hands on the board zeroed, normalised to sum 1. Returns (specs, ranges[count][2][1326])."""
    rng = np.random.default_rng(seed)
    order = card_order()
    specs = np.zeros(count, SPEC_DTYPE)
    ranges = np.zeros((count, 2, HANDS), np.float32)
    for i in range(count):
        cards = rng.choice(52, 5, replace=False)
        board = 0
        for c in cards:
            board |= 1 << int(c)
        pot = int(rng.integers(2, 201))
        stack = int(rng.integers(pot, 10 * pot + 1))
        while True:
            sizes = int(rng.integers(1, 8))
            raises = int(rng.integers(1, 4))
            try:
                nodes, _, _ = bet_tree(pot, stack, sizes, raises)
            except PokerLibError:
                continue  # beyond the solver's tree limits
            if len(nodes) <= max_nodes:
                break
        specs[i] = (board, pot, stack, sizes, raises)
        live = (order & np.uint64(board)) == 0
        for p in range(2):
            r = rng.random(HANDS, dtype=np.float32)
            r[rng.random(HANDS) < 0.25] = 0.0
            r[~live] = 0.0
            ranges[i, p] = r / r.sum()
    return specs, ranges


class Batch:
    """Many general river subgames solved together on the device (pr_batch_*)."""

    def __init__(self, specs, ranges):
        specs = np.array(specs, SPEC_DTYPE)              # copies: set_ranges updates the batch's own
        ranges = np.array(ranges, np.float32, order="C")  # record, never the caller's arrays
        assert ranges.shape == (len(specs), 2, HANDS)
        self.count = len(specs)
        self.specs = specs
        self.ranges = ranges
        self.ptr = lib().pr_batch_new(specs.ctypes.data_as(ctypes.POINTER(SubgameSpec)), self.count,
                                      _ptr(ranges))
        if not self.ptr:
            raise PokerLibError("pr_batch_new failed (bad board or bet tree; see stderr)")

    def shape(self, s):
        n, e, l = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().pr_batch_shape(self.ptr, int(s), ctypes.byref(n), ctypes.byref(e), ctypes.byref(l)),
               "pr_batch_shape")
        return n.value, e.value, l.value

    def enable_average(self):
        _check(lib().pr_batch_enable_average(self.ptr), "pr_batch_enable_average")

    def iterate(self, iterations=1):
        _check(lib().pr_batch_iterate(self.ptr, int(iterations)), "pr_batch_iterate")

    def set_linear_average(self, on=True):
        """Average sums weighted by the iteration number (True) or by 1 (False, the default)."""
        _check(lib().pr_batch_set_linear_average(self.ptr, int(bool(on))), "pr_batch_set_linear_average")

    def iterate_noalloc(self, iterations=1):
        """pr_batch_iterate_noalloc: eager iterations with the queue scratch in a fixed device
        array (no allocation; one call at a time)."""
        _check(lib().pr_batch_iterate_noalloc(self.ptr, int(iterations)), "pr_batch_iterate_noalloc")

    def exploitability(self, use_average=False, fp64=True):
        b0 = np.zeros(self.count)
        b1 = np.zeros(self.count)
        ex = np.zeros(self.count)
        _check(lib().pr_batch_exploitability(self.ptr, int(bool(use_average)), int(bool(fp64)), _ptr(b0),
                                             _ptr(b1), _ptr(ex)), "pr_batch_exploitability")
        return b0, b1, ex

    def root_values(self, player, use_average=False):
        v = np.zeros((self.count, HANDS))
        s = np.zeros(self.count)
        _check(lib().pr_batch_root_values(self.ptr, int(player), int(bool(use_average)), _ptr(v), _ptr(s)),
               "pr_batch_root_values")
        return v, s

    def value(self, use_average=False):
        """Forward: V = r0^T U(sigma) r1 per subgame (double)."""
        v = np.zeros(self.count)
        _check(lib().pr_batch_value(self.ptr, int(bool(use_average)), _ptr(v)), "pr_batch_value")
        return v

    def value_grad(self, use_average=False):
        """Backward: (dV/dr0, dV/dr1, dV/dsigma at the root) per subgame."""
        g0 = np.zeros((self.count, HANDS))
        g1 = np.zeros((self.count, HANDS))
        gs = np.zeros((self.count, 8, HANDS))
        _check(lib().pr_batch_value_grad(self.ptr, int(bool(use_average)), _ptr(g0), _ptr(g1), _ptr(gs)),
               "pr_batch_value_grad")
        return g0, g1, gs

    def value_grad_device(self, d_r0, d_r1, d_sigma, use_average=False):
        """Backward with device outputs: torch tensors (float64, [count][1326], [count][1326],
        [count][8][1326]) or None to skip one."""
        p = lambda t: t.data_ptr() if t is not None else None
        _check(lib().pr_batch_value_grad_device(self.ptr, int(bool(use_average)), p(d_r0), p(d_r1), p(d_sigma)),
               "pr_batch_value_grad_device")

    def set_ranges(self, s, r):
        r = np.ascontiguousarray(r, np.float32).reshape(2, HANDS)
        _check(lib().pr_batch_set_ranges(self.ptr, int(s), _ptr(r)), "pr_batch_set_ranges")
        self.ranges[s] = r

    def _rows(self, name, s, data=None):
        edges = self.shape(s)[1]
        if data is None:
            out = np.zeros((edges, HANDS), np.float32)
            _check(getattr(lib(), name)(self.ptr, int(s), _ptr(out)), name)
            return out
        data = np.ascontiguousarray(data, np.float32).reshape(edges, HANDS)
        _check(getattr(lib(), name)(self.ptr, int(s), _ptr(data)), name)

    def regrets(self, s):
        return self._rows("pr_batch_get_regrets", s)

    def set_regrets(self, s, v):
        self._rows("pr_batch_set_regrets", s, v)

    def average(self, s):
        return self._rows("pr_batch_get_average", s)

    def all_rows(self, which, out=None):
        """pr_batch_get_all: every subgame's regrets (which 0) or average sums (which 1),
        [sum of edge counts][1326] f32; `out` may be a caller-owned array of that shape."""
        if out is None:
            edges = int(sum(self.shape(i)[1] for i in range(self.count)))
            out = np.zeros((edges, HANDS), np.float32)
        _check(lib().pr_batch_get_all(self.ptr, int(which), _ptr(out)), "pr_batch_get_all")
        return out

    def set_average(self, s, v):
        self._rows("pr_batch_set_average", s, v)

    def config(self, c):
        k, per, order, count = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().pr_batch_config(self.ptr, int(c), ctypes.byref(k), ctypes.byref(per), ctypes.byref(order),
                                     ctypes.byref(count)), "pr_batch_config")
        return dict(K=k.value, per_sm=per.value, order=order.value, count=count.value)

    def set_config(self, c, K, per_sm=1, order=0):
        _check(lib().pr_batch_set_config(self.ptr, int(c), int(K), int(per_sm), int(order)),
               "pr_batch_set_config")

    def tune(self):
        ms = np.zeros(2)
        _check(lib().pr_batch_tune(self.ptr, _ptr(ms)), "pr_batch_tune")
        return ms

    def iteration_bytes(self):
        return lib().pr_batch_iteration_bytes(self.ptr)

    @classmethod
    def _borrow(cls, ptr):
        """A view of a batch owned by another object (not freed by close())."""
        b = cls.__new__(cls)
        b.ptr = ptr
        b.count = lib().pr_batch_count(ptr)
        b.specs = None
        b.ranges = None
        b._borrowed = True
        return b

    def close(self):
        if self.ptr and not getattr(self, "_borrowed", False):
            lib().pr_batch_free(self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- turn-leaf value network ----

class ValueNet:
    """The turn-leaf value network (pr_mlp_*): 2706 inputs (both ranges, the 4 turn cards,
    pot / 200 and stack / (10 pot)) -> 4 x 1024 GELU -> 2652 outputs (both players'
    counterfactual values per hand over the pot), BF16 tcgen05 GEMMs with FP32 accumulation,
    trained with MSE and Adam. Inputs and targets are device tensors (torch)."""

    LAYERS = 5

    def __init__(self, rows=4096, seed=0):
        self.rows = rows
        self.ptr = lib().pr_mlp_new(int(rows), int(seed))
        if not self.ptr:
            raise PokerLibError("pr_mlp_new failed")

    @staticmethod
    def layer_shape(l):
        o, i = ctypes.c_int(), ctypes.c_int()
        _check(lib().pr_mlp_layer_shape(int(l), ctypes.byref(o), ctypes.byref(i)), "pr_mlp_layer_shape")
        return o.value, i.value

    def set_persistent(self, on=True):
        """pr_mlp_set_persistent: the persistent GEMM form (True) or one CTA per tile."""
        return lib().pr_mlp_set_persistent(self.ptr, int(bool(on)))

    def forward(self, ranges, boards, scalars, out):
        """ranges [n][2][1326] f32, boards [n] int64 (4-card masks), scalars [n][2] f32,
        out [n][2652] f32: device tensors, n <= rows."""
        n = int(boards.shape[0])
        _check(lib().pr_mlp_forward(self.ptr, ranges.data_ptr(), boards.data_ptr(), scalars.data_ptr(),
                                    out.data_ptr(), n), "pr_mlp_forward")

    def train_step(self, ranges, boards, scalars, targets, lr):
        loss = ctypes.c_double()
        n = int(boards.shape[0])
        _check(lib().pr_mlp_train_step(self.ptr, ranges.data_ptr(), boards.data_ptr(), scalars.data_ptr(),
                                       targets.data_ptr(), n, float(lr), ctypes.byref(loss)), "pr_mlp_train_step")
        return loss.value

    def layer(self, l):
        o, i = self.layer_shape(l)
        W = np.zeros((o, i), np.float32)
        b = np.zeros(o, np.float32)
        _check(lib().pr_mlp_get_layer(self.ptr, int(l), _ptr(W), _ptr(b)), "pr_mlp_get_layer")
        return W, b

    def set_layer(self, l, W, b):
        W = np.ascontiguousarray(W, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        _check(lib().pr_mlp_set_layer(self.ptr, int(l), _ptr(W), _ptr(b)), "pr_mlp_set_layer")

    def grad(self, l):
        o, i = self.layer_shape(l)
        W = np.zeros((o, i), np.float32)
        b = np.zeros(o, np.float32)
        _check(lib().pr_mlp_get_grad(self.ptr, int(l), _ptr(W), _ptr(b)), "pr_mlp_get_grad")
        return W, b

    def close(self):
        if self.ptr:
            lib().pr_mlp_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- full fixed-flop game with general bets ----

def full_spec(flop, pot, stack, flop_fracs=(0.75,), flop_allin=True, flop_raises=1, turn_fracs=(0.75,),
              turn_allin=True, turn_raises=1, river_sizes=0b011, river_raises=2):
    """A FullSpec: 3-card flop mask, pot before the flop, chips behind, per-street sizes."""
    sp = FullSpec()
    sp.flop = int(flop)
    sp.pot = float(pot)
    sp.stack = float(stack)
    for i, (fr, ai, rz) in enumerate(((flop_fracs, flop_allin, flop_raises), (turn_fracs, turn_allin, turn_raises))):
        fr = list(fr)
        assert len(fr) <= 4
        for k, f in enumerate(fr):
            sp.street[i].fracs[k] = float(f)
        sp.street[i].nfrac = len(fr)
        sp.street[i].allin = int(bool(ai))
        sp.street[i].max_raises = int(rz)
    sp.river_sizes = int(river_sizes)
    sp.river_raises = int(river_raises)
    return sp


def full_tree(spec):
    """The flop and turn nodes (FNODE_DTYPE array in pre-order), the child list, edge and
    leaf counts."""
    n, e, l = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib().pr_full_tree(ctypes.byref(spec), None, 0, ctypes.byref(n), ctypes.byref(e), ctypes.byref(l),
                              None, 0), "pr_full_tree")
    nodes = np.zeros(n.value, FNODE_DTYPE)
    kids = np.zeros(max(1, 64 * n.value), np.int32)
    _check(lib().pr_full_tree(ctypes.byref(spec), nodes.ctypes.data_as(ctypes.c_void_p), n.value, None, None,
                              None, kids.ctypes.data_as(ctypes.c_void_p), len(kids)), "pr_full_tree")
    used = 0
    for nd in nodes:
        if nd["kind"] in (0, 2):
            used = max(used, int(nd["kids"]) + int(nd["nchild"]))
    return nodes, kids[:used], e.value, l.value


class FullGame:
    """A fixed-flop game with general bets on every street, solved on the device: flop and
    turn by level-synchronous sweeps, the river by the batched river solver (pr_full_*)."""

    def __init__(self, spec, ranges):
        self.spec = spec
        ranges = np.ascontiguousarray(ranges, np.float32).reshape(2, HANDS)
        self.ptr = lib().pr_full_new(ctypes.byref(spec), _ptr(ranges))
        if not self.ptr:
            raise PokerLibError("pr_full_new failed (bad spec or allocation; see stderr)")
        n, e, l, b, a = (ctypes.c_int() for _ in range(5))
        _check(lib().pr_full_shape(self.ptr, ctypes.byref(n), ctypes.byref(e), ctypes.byref(l), ctypes.byref(b),
                                   ctypes.byref(a)), "pr_full_shape")
        self.nodes, self.edges, self.leaves = n.value, e.value, l.value
        self.bet_subgames, self.allin_subgames = b.value, a.value
        self.joint = lib().pr_full_joint(self.ptr)
        self._net = None

    def set_net(self, net):
        """Net-leaf mode with a ValueNet, or plain river subgames (None)."""
        self._net = net
        _check(lib().pr_full_set_net(self.ptr, net.ptr if net is not None else None), "pr_full_set_net")

    def set_zero_sum(self, on=True):
        """pr_full_set_zero_sum: net leaves shifted so both players' range-weighted values cancel."""
        _check(lib().pr_full_set_zero_sum(self.ptr, int(bool(on))), "pr_full_set_zero_sum")

    def tune(self):
        """Autotunes the river-subgame batches; per-pass ms of each batch's two classes."""
        ms = np.zeros(4)
        _check(lib().pr_full_tune(self.ptr, _ptr(ms)), "pr_full_tune")
        return ms

    def set_linear_average(self, on):
        """Average sums weighted by the iteration number (True, the default) or by 1."""
        _check(lib().pr_full_set_linear_average(self.ptr, int(bool(on))), "pr_full_set_linear_average")

    def half_iteration(self, player):
        _check(lib().pr_full_pass(self.ptr, int(player)), "pr_full_pass")

    def iterate(self, iterations=1):
        _check(lib().pr_full_iterate(self.ptr, int(iterations)), "pr_full_iterate")

    def exploitability(self, resolve_iterations=0):
        """(BR0, BR1, exploitability per unit of joint mass in chips), FP64."""
        b0, b1, ex = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(lib().pr_full_exploitability(self.ptr, int(resolve_iterations), ctypes.byref(b0), ctypes.byref(b1),
                                            ctypes.byref(ex)), "pr_full_exploitability")
        return b0.value, b1.value, ex.value

    def _read(self, which, shape, dtype):
        out = np.zeros(shape, dtype)
        _check(lib().pr_full_read(self.ptr, int(which), out.ctypes.data_as(ctypes.c_void_p)), "pr_full_read")
        return out

    def regrets(self):
        return self._read(0, (self.edges, HANDS), np.float32)

    def average(self):
        return self._read(1, (self.edges, HANDS), np.float32)

    def reach(self, fp64=False):
        return self._read(5 if fp64 else 2, (self.nodes, 2, HANDS), np.float64 if fp64 else np.float32)

    def leaf_values(self, fp64=False):
        return self._read(6 if fp64 else 3, (self.leaves, HANDS), np.float64 if fp64 else np.float32)

    def node_values(self, fp64=False):
        return self._read(7 if fp64 else 4, (self.nodes, HANDS), np.float64 if fp64 else np.float32)

    def net_inputs(self):
        """Normalised ranges [net leaves][2][1326] and reach masses [net leaves][2] of the last
        net-leaf pass (leaves in batch_leaves(0) order)."""
        n = self.bet_subgames // 48
        return self._read(8, (n, 2, HANDS), np.float32), self._read(9, (n, 2), np.float32)

    def _write(self, which, data):
        data = np.ascontiguousarray(data, np.float32).reshape(self.edges, HANDS)
        _check(lib().pr_full_write(self.ptr, int(which), _ptr(data)), "pr_full_write")

    def set_regrets(self, data):
        self._write(0, data)

    def reset(self):
        """Zero regrets and average sums everywhere (flop, turn, river subgames)."""
        _check(lib().pr_full_reset(self.ptr), "pr_full_reset")

    def set_average(self, data):
        self._write(1, data)

    def batch(self, which):
        """The river subgames of the leaves with chips behind (0) or all-in (1), or None. The
        batch belongs to the game: use it only while the game is open."""
        p = lib().pr_full_batch(self.ptr, int(which))
        return Batch._borrow(p) if p else None

    def batch_leaves(self, which):
        n = lib().pr_full_batch_leaves(self.ptr, int(which), None)
        out = np.zeros(max(1, n), np.int32)
        lib().pr_full_batch_leaves(self.ptr, int(which), out.ctypes.data_as(ctypes.c_void_p))
        return out[:n]

    def close(self):
        if self.ptr:
            lib().pr_full_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
