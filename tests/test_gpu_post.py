"""GPU post-run pass against the oracle, on the states the GPU computed.

Bars: magnitudes, their maxima, activation times and every final metric
(Dice, IoU, precision, recall over 101 thresholds and the summary) are
bit-identical - they are sums of absolute values, comparisons, counts and
single IEEE divisions. theta and phi come from CUDA's acosf / atan2f against
the host libm's: within 4e-6 rad (a few ulp of pi), NaN in the same places."""

import numpy as np
import pytest

from conftest import oracle_forward

pytestmark = pytest.mark.gpu

ANGLE_ATOL = 4e-6


@pytest.fixture(scope="module")
def alg():
    from cardiotrust_b200 import algorithm

    return algorithm


@pytest.fixture(scope="module")
def ctx(alg):
    c = alg.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def shell(oracle_mod):
    """Ellipsoidal shell (cells without a voxel around it), 2 beats, a pathological block."""
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=(12, 11, 10), mask="shell", shell_semi_axes=(6.0, 5.5, 5.0), shell_thickness=2.0,
                           num_steps=300, num_beats=2, patho_size=3, pulse_onset=2, pulse_sigma_samples=5.0,
                           noise_fraction=0.01, seed=4)
    return sc.attach_measurements(sc.build(spec), oracle_forward(oracle_mod))


def _angles_close(got, want):
    assert np.array_equal(np.isnan(got), np.isnan(want))
    ok = ~np.isnan(want)
    assert np.abs(got[ok].astype(np.float64) - want[ok]).max(initial=0.0) <= ANGLE_ATOL


def _check_arrays(eng, ref):
    for f in ("magnitude", "magnitude_max"):
        np.testing.assert_array_equal(eng.read(f"system_states_{f}"), ref[f], err_msg=f)
    np.testing.assert_array_equal(eng.read("activation_times"), ref["activation_times"])
    for f in ("theta", "phi", "theta_max", "phi_max"):
        _angles_close(eng.read(f"system_states_{f}"), ref[f])


def test_plotting_arrays_match_oracle(alg, ctx, oracle_mod, cuboid8):
    eng = alg.EpochEngine.from_scenario(ctx, cuboid8)
    eng.run_epoch(0)
    X = eng.read("system_states")
    eng.calculate_plotting_arrays(cuboid8.spec.sample_rate_hz)
    ref, rc = oracle_mod.plotting_arrays(X, cuboid8.spec.sample_rate_hz)
    assert rc == 0
    _check_arrays(eng, ref)
    eng.close()


def test_plotting_arrays_nan_states(alg, ctx, oracle_mod, shell):
    """NaN gains on one voxel: its states are NaN at every step (no maximum: CT_ERR_NO_MAXIMUM, as
    the reference's argmax_skipnan error), and its neighbours' states turn NaN part-way (NaN steps
    are skipped by the maximum)."""
    from cardiotrust_b200._lib import CT_ERR_NO_MAXIMUM, CtError

    eng = alg.EpochEngine.from_scenario(ctx, shell)
    g = shell.model.gains.copy()
    v = shell.num_voxels // 2
    g[3 * v: 3 * v + 3] = np.nan
    eng.write("gains", g)
    eng.simulate()
    X = eng.read("system_states")
    assert np.isnan(X[:, 3 * v]).all() and np.isnan(X).any(axis=0).sum() > 3
    with pytest.raises(CtError) as e:
        eng.calculate_plotting_arrays(shell.spec.sample_rate_hz)
    assert e.value.status == CT_ERR_NO_MAXIMUM
    ref, rc = oracle_mod.plotting_arrays(X, shell.spec.sample_rate_hz)
    assert rc == CT_ERR_NO_MAXIMUM
    _check_arrays(eng, ref)
    eng.close()


@pytest.fixture(scope="module")
def shell_front():
    """The same shell with a 120-step beat: the activation front is part-way across, so the voxels'
    maxima spread from 0 to 1 and the Dice score changes along the threshold sweep."""
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=(12, 11, 10), mask="shell", shell_semi_axes=(6.0, 5.5, 5.0), shell_thickness=2.0,
                           num_steps=120, num_beats=2, patho_size=3, pulse_onset=2, pulse_sigma_samples=5.0,
                           noise_fraction=0.01, seed=4)
    return sc.build(spec)


@pytest.mark.parametrize("case", ["as_built", "front_truth", "front_model", "nan_voxel"])
def test_final_metrics_match_oracle(alg, ctx, oracle_mod, shell, shell_front, case):
    """States of the estimated model as built (maxima all near 1), of the ground-truth and estimated
    models with the front part-way across, and of a model with one NaN voxel."""
    scn = shell_front if case.startswith("front") else shell
    eng = alg.EpochEngine.from_scenario(ctx, scn, truth=case == "front_truth")
    if case == "nan_voxel":
        g = scn.model.gains.copy()
        g[0:3] = np.nan
        eng.write("gains", g)
    eng.simulate()
    X = eng.read("system_states")
    got = eng.calculate_final(scn.types_truth, scn.numbers)
    want = oracle_mod.calculate_final(X, scn.types_truth, scn.numbers)
    for f in ("dice_score_over_threshold", "iou_over_threshold", "precision_over_threshold", "recall_over_threshold"):
        np.testing.assert_array_equal(getattr(got, f), want[f], err_msg=f)
    for f in ("threshold", "dice", "iou", "recall", "precision"):
        assert np.float32(getattr(got, f)) == np.float32(want[f]), f
    if case == "front_truth":
        assert len(np.unique(want["dice_score_over_threshold"])) > 10  # the sweep is exercised
    eng.close()


def test_final_metrics_rejects_bad_voxel_numbers(alg, ctx, shell):
    from cardiotrust_b200._lib import CT_ERR_INVALID_ARGUMENT, CtError

    eng = alg.EpochEngine.from_scenario(ctx, shell)
    bad = shell.numbers.copy()
    bad.flat[np.argmax(bad.ravel() >= 0)] = 3 * shell.num_voxels  # one past the last state
    with pytest.raises(CtError) as e:
        eng.calculate_final(shell.types_truth, bad)
    assert e.value.status == CT_ERR_INVALID_ARGUMENT
    eng.close()
