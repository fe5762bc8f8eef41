"""The C-ABI library loads and exports every symbol include/pokerrust_b200.h declares
(no GPU calls)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pokerrust_b200.h")

REFERENCE_SYMBOLS = ["init_builder", "upload_c", "download_c", "build_river_cuda",
                     "transfer_flop_eval_cuda", "free_eval_cuda", "evaluate_cuda"]


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text)


@pytest.fixture(scope="module")
def so_path():
    from pokerrust_b200.build import SO_PATH, build
    build()
    return SO_PATH


def test_header_declares_reference_boundary():
    fns = declared_functions()
    for s in REFERENCE_SYMBOLS:
        assert s in fns


def test_library_exports_every_declared_symbol(so_path):
    lib = ctypes.CDLL(so_path)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_exports_are_unmangled_c_symbols(so_path):
    out = subprocess.run(["nm", "-D", "--defined-only", so_path], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for name in declared_functions():
        assert name in exported, name


def test_static_archive_for_rust_build(so_path):
    from pokerrust_b200.build import A_PATH
    out = subprocess.run(["nm", "--defined-only", A_PATH], capture_output=True, text=True,
                         check=True).stdout
    for s in REFERENCE_SYMBOLS:
        assert re.search(rf" T {s}$", out, re.M), s


def test_error_strings_without_gpu(so_path):
    from pokerrust_b200 import lib
    assert lib().pr_error_string(0) == b"ok"
    assert lib().pr_range_stride() == 1328
    assert lib().pr_river_smem_bytes(None, 0, 0) == 0      # no tables: nothing to size


def test_null_handles_are_refused_without_gpu(so_path):
    # the entry points check their arguments before any CUDA call (inside the trace range
    # each one opens), so a null handle is refused with status 2 on a machine without a GPU
    from pokerrust_b200 import lib
    L = lib()
    assert L.pr_evaluate(None, None, 0, 0) == 2
    assert L.pr_batch_iterate(None, 1) == 2
    assert L.pr_batch_value(None, 0, None) == 2
    assert L.pr_game_iterate(None, 1) == 2
    assert L.pr_full_iterate(None, 1) == 2
    assert L.pr_mlp_forward(None, None, None, None, None, 0) == 2
    assert L.pr_game_set_regrets(None, None, None) == 2
    L.pr_clear_error()
    assert L.pr_last_error() == 0


@pytest.mark.parametrize("name", [
    "pr_batch_exploitability", "pr_batch_tune", "pr_batch_get_all", "pr_batch_set_ranges",
    "pr_batch_get_regrets", "pr_batch_set_linear_average", "pr_batch_enable_average",
    "pr_batch_iterate_noalloc", "pr_batch_value_grad", "pr_full_exploitability", "pr_full_set_zero_sum",
    "pr_full_set_net", "pr_full_tune", "pr_game_root_values", "pr_game_get_regrets", "pr_game_get_average",
    "pr_game_enable_average", "pr_game_exploitability", "pr_mlp_train_step", "pr_mlp_get_layer",
    "pr_mlp_set_layer", "pr_mlp_get_grad", "pr_get_regrets", "pr_set_regrets", "pr_upload_batch"])
def test_every_handle_entry_point_refuses_null(so_path, name):
    # null handle, null buffers, zero sizes: status 2 before any CUDA call
    from pokerrust_b200 import lib
    f = getattr(lib(), name)
    args = [0.0 if t in (ctypes.c_float, ctypes.c_double) else (None if t is ctypes.c_void_p else 0)
            for t in f.argtypes]
    assert f(*args) == 2
    lib().pr_clear_error()


def test_setters_return_minus_one_for_a_null_handle(so_path):
    from pokerrust_b200 import lib
    assert lib().pr_game_set_device_tree(None, 1) == -1
    assert lib().pr_mlp_set_persistent(None, 1) == -1
