"""What the trained turn-leaf value network gains: trained on river-solver data, its
held-out error beats the zero and training-mean predictors by a wide margin, at a small
fraction of the time of the river solves it replaces (48 river subgames per turn state)."""
import pytest

pytestmark = pytest.mark.gpu


def test_trained_network_beats_baselines():
    from pokerrust_b200 import train_value_net as T
    out = T.run(train_n=512, test_n=128, iterations=40, cheap=3, epochs=40, batch=256, lr=1e-3, seed=3)
    mse = out["test_mse"]
    assert mse["network"] < 0.6 * mse["train_mean"], mse
    assert mse["network"] < 0.5 * mse["zero"], mse
    curve = out["train"]["loss_curve"]
    assert curve[-1] < 0.5 * curve[0], curve
    t = out["seconds_per_state"]
    assert t["network"] < 0.1 * t["river_solve_3_iterations"], t
    print("\nvalue network:", mse, t)
