"""Known answers for the oracle's restatement of the callers either side of the
epoch: the post-run arrays (src/core/scenario.rs:636-690 with
src/core/data/shapes.rs:171-352), the final segmentation metrics
(src/core/algorithm/metrics.rs:226-447) and the epoch loop
run_model_based (src/core/scenario.rs:725-795).

The reference tree holds no test of these functions, so the answers here are
worked by hand from the reference code; the GPU is compared against this
oracle in tests/test_gpu_post.py and tests/test_gpu_scenario_loop.py."""

import numpy as np
import pytest

F = np.float32


def _states(rows):
    """[T, 3V] from rows of per-voxel (x, y, z) triples."""
    return np.array([np.concatenate(r) for r in rows], dtype=F)


def test_spherical_arrays_known_answers(oracle_mod):
    nan = np.nan
    X = _states([
        [(0.0, 0.0, 0.0), (nan, 0.0, 0.0)],
        [(3.0, -4.0, 0.0), (0.0, 0.0, 2.0)],
        [(-1.0, 1.0, 1.0), (0.0, 0.0, -2.0)],
        [(0.0, 4.0, 3.0), (0.0, 1.0, 0.0)],
    ])
    out, rc = oracle_mod.plotting_arrays(X, sample_rate_hz=2000.0)
    assert rc == 0
    mag = out["magnitude"]
    np.testing.assert_array_equal(mag[:, 0], F([0.0, 7.0, 3.0, 7.0]))
    assert np.isnan(mag[0, 1])
    np.testing.assert_array_equal(mag[1:, 1], F([2.0, 2.0, 1.0]))
    # acos(0 / 0) is NaN; acos(z / |.|_1) otherwise; atan2(y, x)
    assert np.isnan(out["theta"][0, 0])
    assert out["theta"][1, 1] == F(0.0) and out["theta"][2, 1] == np.arccos(F(-1.0))
    assert out["phi"][1, 0] == np.arctan2(F(-4.0), F(3.0))
    # first of equal maxima (steps 1 and 3 of voxel 0), NaN steps skipped (voxel 1, step 0)
    np.testing.assert_array_equal(out["magnitude_max"], F([7.0, 2.0]))
    assert out["phi_max"][0] == np.arctan2(F(-4.0), F(3.0))
    assert out["theta_max"][1] == F(0.0)
    # activation time = step / sample_rate * 1000 (ms)
    np.testing.assert_array_equal(out["activation_times"], F([1.0 / 2000.0 * 1000.0, 1.0 / 2000.0 * 1000.0]))


def test_spherical_all_nan_voxel_is_an_error(oracle_mod):
    X = _states([[(np.nan, 1.0, 1.0), (1.0, 0.0, 0.0)], [(1.0, np.nan, 0.0), (2.0, 0.0, 0.0)]])
    out, rc = oracle_mod.plotting_arrays(X, 1000.0)
    assert rc == -8  # argmax_skipnan: MinMaxError::EmptyInput
    assert np.isnan(out["magnitude_max"][0]) and out["magnitude_max"][1] == F(2.0)
    assert out["activation_times"][1] == F(1.0)


def _grid_case():
    """Four cells: voxel 0 (pathological, max 0.5), voxel 1 (ventricle, max 0.2),
    voxel 2 (pathological, max 1.5: never predicted), and a pathological cell without a voxel."""
    X = _states([[(0.5, 0.0, 0.0), (0.2, 0.0, 0.0), (0.0, 1.5, 0.0)],
                 [(0.25, 0.0, -0.25), (0.0, -0.1, 0.0), (0.5, 0.5, 0.5)]])
    types = np.array([6, 5, 6, 6], np.int32).reshape(2, 2, 1)
    numbers = np.array([0, 3, 6, -1], np.int32).reshape(2, 2, 1)
    return X, types, numbers


def test_final_metrics_known_answers(oracle_mod):
    X, types, numbers = _grid_case()
    r = oracle_mod.calculate_final(X, types, numbers)
    dice, iou = r["dice_score_over_threshold"], r["iou_over_threshold"]
    prec, rec = r["precision_over_threshold"], r["recall_over_threshold"]
    # i < 20: nothing predicted; 20 <= i < 50: voxel 1 only (a false positive); i >= 50: voxels 0 and 1
    np.testing.assert_array_equal(dice[:50], 0.0)
    np.testing.assert_array_equal(iou[:50], 0.0)
    np.testing.assert_array_equal(prec[:50], 0.0)
    np.testing.assert_array_equal(rec[:50], 0.0)
    np.testing.assert_array_equal(dice[50:], F(2) / F(5))
    np.testing.assert_array_equal(iou[50:], F(1) / F(4))
    np.testing.assert_array_equal(prec[50:], F(1) / F(2))
    np.testing.assert_array_equal(rec[50:], F(1) / F(3))
    # first threshold of the largest Dice score
    assert r["threshold"] == F(50) / F(100)
    assert (r["dice"], r["iou"], r["recall"], r["precision"]) == (F(0.4), F(0.25), F(1) / F(3), F(0.5))


def test_final_metrics_without_pathology(oracle_mod):
    X, types, numbers = _grid_case()
    types = np.where(types == 6, 5, types).astype(np.int32)
    r = oracle_mod.calculate_final(X, types, numbers)
    # recall is 1 without ground-truth positives; Dice 0 everywhere -> threshold 0
    np.testing.assert_array_equal(r["recall_over_threshold"], 1.0)
    np.testing.assert_array_equal(r["dice_score_over_threshold"], 0.0)
    assert r["threshold"] == 0.0 and r["recall"] == 1.0


@pytest.fixture(scope="module")
def tiny(oracle_mod):
    from conftest import oracle_forward
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=(4, 4, 3), num_steps=80, num_beats=2, patho_size=2, pulse_onset=2,
                           pulse_sigma_samples=4.0, noise_fraction=0.01, seed=5)
    return sc.attach_measurements(sc.build(spec), oracle_forward(oracle_mod))


def test_epoch_loop_schedule_and_snapshots(oracle_mod, tiny):
    o = oracle_mod.from_scenario(tiny, num_batch_slots=8)
    a = oracle_mod.algo(learning_rate=0.5)
    g0 = o.gains.copy()
    summary, losses, snaps = o.run_model_based(a, epochs=4, learning_rate_reduction_interval=2,
                                               learning_rate_reduction_factor=0.5, snapshots_interval=2,
                                               beat_orders=[[0, 1]] * 4)
    assert summary["epochs_run"] == 4 and losses.shape == (4, 3)
    assert a.learning_rate == 0.5  # restored
    # epoch 0 runs with learning rate 0: the snapshot after it holds the initial gains
    assert len(snaps["gains"]) == 2
    np.testing.assert_array_equal(snaps["gains"][0], g0)
    assert not np.array_equal(snaps["gains"][1], g0)
    assert summary["loss"] == losses[-1, 0] == o.loss_batch[o.batch_index - 1]


def test_epoch_loop_stops_on_non_normal_loss(oracle_mod, tiny):
    o = oracle_mod.from_scenario(tiny, num_batch_slots=16)
    a = oracle_mod.algo(learning_rate=1e30)
    summary, losses, _ = o.run_model_based(a, epochs=8, beat_orders=[[0, 1]] * 8)
    assert summary["epochs_run"] < 8
    assert not np.isfinite(losses[-1, 0]) and np.all(np.isfinite(losses[:-1, 0]))
