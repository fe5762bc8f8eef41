"""B200-native river-subtree CFR for the fixed-flop limit hold'em game of pokerrust.

The CUDA library sits behind the reference's C ABI (include/pokerrust_b200.h);
`pokerrust_b200.interface` mirrors the reference's Rust FFI wrapper
(src/cuda_interface.rs) on top of it.
"""
from .interface import (  # noqa: F401
    HANDS,
    RANGE_STRIDE,
    SPEC_DTYPE,
    Batch,
    Builder,
    FullGame,
    Game,
    PokerLibError,
    ValueNet,
    bet_tree,
    random_subgames,
    build_flop_tables,
    build_river,
    card_order,
    full_spec,
    full_tree,
    download_gpu,
    evaluate_gpu,
    export_tables,
    free_eval,
    initialize_builder,
    lib,
    transfer_flop_eval,
    upload_gpu,
)
