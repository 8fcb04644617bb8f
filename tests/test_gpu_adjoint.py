"""GPU adjoint mode (back-propagation through time with checkpoints) against
the float64 oracle, whose own gradient is pinned by central differences in
test_adjoint_oracle.py.

Bars: states, measurements and metrics as in the reference mode (the
forward is shared); gradients <= 1e-3 relative (norm-wise) to the float64
oracle, the stated gradient tolerance."""

import numpy as np
import pytest

from conftest import oracle_forward, rel_err

pytestmark = pytest.mark.gpu

TOL_GRAD = 1e-3
TOL_LOSS = 1e-4


@pytest.fixture(scope="module")
def alg():
    from cardiotrust_b200 import algorithm

    return algorithm


@pytest.fixture(scope="module")
def ctx(alg):
    c = alg.Context(0)
    yield c
    c.close()


def _pair(alg, oracle_mod, **kw):
    a = alg.Algorithm(**kw)
    o = oracle_mod.algo(
        optimizer=int(a.optimizer), ap_derivative=int(a.ap_derivative), freeze_gains=int(a.freeze_gains),
        freeze_delays=int(a.freeze_delays), batch_size=a.batch_size, learning_rate=a.learning_rate,
        mse_strength=a.mse_strength, maximum_regularization_strength=a.maximum_regularization_strength,
        maximum_regularization_threshold=a.maximum_regularization_threshold,
        difference_regularization_strength=a.difference_regularization_strength,
        smoothness_regularization_strength=a.smoothness_regularization_strength,
    )
    return a, o


def _check_epoch(alg, eng, o, precision, tol_grad=TOL_GRAD):
    bi = eng.run_epoch(0, grad_mode=alg.GradMode.Adjoint, precision=precision)
    assert bi == o.batch_index
    assert rel_err(eng.read("grad_gains"), o.d_gains) < tol_grad
    assert rel_err(eng.read("grad_coefs"), o.d_coefs) < tol_grad
    for f, ref in [("loss", o.loss), ("loss_batch", o.loss_batch),
                   ("loss_maximum_regularization", o.loss_maximum_regularization)]:
        assert rel_err(eng.read(f), ref) < TOL_LOSS, f


CASES = {
    # cuboid8: T = 500 -> two checkpoint segments (256 + 244 steps)
    "sgd_gains": dict(learning_rate=0.5),
    "adam_all": dict(optimizer=1, learning_rate=1e-3, freeze_delays=False, maximum_regularization_threshold=0.5),
    "coefs_only_regularised": dict(freeze_gains=True, freeze_delays=False, difference_regularization_strength=1e-3,
                                   ap_derivative=0),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_adjoint_vs_f64_oracle(alg, ctx, oracle_mod, cuboid8, case):
    kw = {k: (alg.Optimizer(v) if k == "optimizer" else alg.APDerivative(v) if k == "ap_derivative" else v)
          for k, v in CASES[case].items()}
    a, oa = _pair(alg, oracle_mod, **kw)
    eng = alg.EpochEngine.from_scenario(ctx, cuboid8, algorithm=a)
    o = oracle_mod.from_scenario(cuboid8, dtype=np.float64)
    o.run_epoch(oa, adjoint=True)
    _check_epoch(alg, eng, o, alg.Precision.Fp32)
    # the forward is the reference mode's: states of the beat bit-identical to the f32 oracle
    o32 = oracle_mod.from_scenario(cuboid8)
    o32.simulate()
    np.testing.assert_array_equal(eng.read("system_states"), o32.system_states)
    eng.close()


def test_adjoint_tensor_core_precision(alg, ctx, oracle_mod, cuboid8):
    """H^T r on tcgen05 with the 3xTF32 split feeds the adjoint: same bar."""
    a, oa = _pair(alg, oracle_mod, optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    eng = alg.EpochEngine.from_scenario(ctx, cuboid8, algorithm=a)
    o = oracle_mod.from_scenario(cuboid8, dtype=np.float64)
    o.run_epoch(oa, adjoint=True)
    _check_epoch(alg, eng, o, alg.Precision.Tf32x3)
    eng.close()


def test_adjoint_batches_beats_and_ring_growth(alg, ctx, oracle_mod):
    """3 beats, batch_size 1, T = 300 (segments of 256 and 44 steps): three updates that roll delays,
    so the adjoint ring is re-sized between epochs; gradients of the last batch and the parameters
    after every update are compared."""
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=(6, 5, 4), num_steps=300, num_beats=3, patho_size=2, patho_origin=(1, 1, 1),
                           pulse_onset=3, pulse_sigma_samples=5.0, noise_fraction=0.02, seed=9)
    scn = sc.attach_measurements(sc.build(spec), oracle_forward(oracle_mod))
    a, oa = _pair(alg, oracle_mod, batch_size=1, optimizer=alg.Optimizer.Adam, learning_rate=5e-2,
                  freeze_delays=False)
    eng = alg.EpochEngine.from_scenario(ctx, scn, num_batch_slots=6, algorithm=a)
    o = oracle_mod.from_scenario(scn, dtype=np.float64, num_batch_slots=6)
    order = np.array([1, 2, 0], np.int32)
    g0, c0 = scn.model.gains.astype(np.float64), scn.model.coefs.astype(np.float64)
    for epoch in range(2):
        bi = eng.run_epoch(3 * epoch, beat_order=order, grad_mode=alg.GradMode.Adjoint)
        o.run_epoch(oa, beat_order=order, adjoint=True)
        assert bi == o.batch_index == 3 * (epoch + 1)
        assert rel_err(eng.read("grad_gains"), o.d_gains) < TOL_GRAD
        assert rel_err(eng.read("grad_coefs"), o.d_coefs) < TOL_GRAD
        assert rel_err(eng.read("gains") - g0, o.gains - g0) < TOL_GRAD
        assert rel_err(eng.read("coefs") - c0, o.coefs - c0) < TOL_GRAD
        np.testing.assert_array_equal(eng.read("delays"), o.delays)
    eng.close()


def test_adjoint_multi_tile_ctas(alg, ctx, oracle_mod):
    """22^3 cuboid (333 tiles of 32 voxels, more than one CTA per SM holds at once): the form in which a
    CTA walks several tiles and adds its accumulators to global memory after every block of steps."""
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=(22, 22, 22), num_steps=260, num_sensors=16, patho_size=4, pulse_onset=2,
                           pulse_sigma_samples=5.0, noise_fraction=0.01, seed=2)
    scn = sc.attach_measurements(sc.build(spec), oracle_forward(oracle_mod))
    a, oa = _pair(alg, oracle_mod, optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=a)
    o = oracle_mod.from_scenario(scn, dtype=np.float64)
    o.run_epoch(oa, adjoint=True)
    _check_epoch(alg, eng, o, alg.Precision.Fp32)
    eng.close()


def test_adjoint_reference_mode_unchanged_after_adjoint(alg, ctx, oracle_mod, cuboid8):
    """An adjoint epoch followed by a reference epoch: the reference derivation still matches the oracle."""
    a, oa = _pair(alg, oracle_mod, learning_rate=0.5)
    eng = alg.EpochEngine.from_scenario(ctx, cuboid8, num_batch_slots=2, algorithm=a)
    o = oracle_mod.from_scenario(cuboid8, num_batch_slots=2)
    eng.run_epoch(0, grad_mode=alg.GradMode.Adjoint)
    o.run_epoch(oa, adjoint=True)
    eng.run_epoch(1, grad_mode=alg.GradMode.Reference)
    o.run_epoch(oa)
    assert rel_err(eng.read("grad_gains"), o.d_gains) < TOL_GRAD
    assert rel_err(eng.read("loss_batch"), o.loss_batch) < TOL_LOSS
    eng.close()
