"""GPU parity: the CUDA epoch (through the C ABI) against the CPU restatement.

Bars, written per check:
  * states x[t, s]: bit-identical (same operations in the same order);
  * derivatives given the same mapped residuals: bit-identical;
  * the measurement products (H x, H^T r) sum in a different order than
    ndarray/matrixmultiply, so everything downstream of them is compared with
    the stated tolerances: <= 1e-4 relative on states/measurements/losses,
    <= 1e-3 relative (norm-wise) on gradients and parameter updates.
"""

import numpy as np
import pytest

from conftest import max_rel_err, oracle_forward, rel_err

pytestmark = pytest.mark.gpu

TOL_MEAS = 1e-5   # H x in fp32, any summation order, vs the reference order
TOL_LOSS = 1e-4
TOL_GRAD = 1e-3


@pytest.fixture(scope="module")
def alg():
    from cardiotrust_b200 import algorithm

    return algorithm


@pytest.fixture(scope="module")
def ctx(alg):
    c = alg.Context(0)
    yield c
    c.close()


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def assert_bitwise(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    diff = bits(a) != bits(b)
    if diff.any():
        idx = np.argwhere(diff)[0]
        pytest.fail(f"{what}: {int(diff.sum())} of {a.size} elements differ; first at {tuple(idx)}: "
                    f"{a[tuple(idx)]!r} vs {b[tuple(idx)]!r}")


def algo_pair(alg, oracle_mod, **kw):
    """(GPU Algorithm, oracle Algo) with the same settings."""
    a = alg.Algorithm(**{k: v for k, v in kw.items()})
    o = oracle_mod.algo(
        optimizer=int(a.optimizer), ap_derivative=int(a.ap_derivative), freeze_gains=int(a.freeze_gains),
        freeze_delays=int(a.freeze_delays), batch_size=a.batch_size, learning_rate=a.learning_rate,
        mse_strength=a.mse_strength, maximum_regularization_strength=a.maximum_regularization_strength,
        maximum_regularization_threshold=a.maximum_regularization_threshold,
        difference_regularization_strength=a.difference_regularization_strength,
        smoothness_regularization_strength=a.smoothness_regularization_strength,
    )
    return a, o


def test_forward_states_bitwise(alg, ctx, oracle_mod, cuboid8):
    eng = alg.EpochEngine.from_scenario(ctx, cuboid8, truth=True)
    y, x = eng.simulate(with_states=True)
    o = oracle_mod.from_scenario(cuboid8, truth=True)
    y_ref = o.simulate()
    assert_bitwise(x, o.system_states, "system_states")
    assert rel_err(y, y_ref) < TOL_MEAS
    eng.close()


def test_golden_fixture(alg, ctx):
    """Committed oracle outputs (tests/golden/make_golden.py): 4^3 cuboid, 2 beats, Adam, coefficients."""
    import pathlib

    z = np.load(pathlib.Path(__file__).with_name("golden") / "cuboid4_b2.npz")
    kw = dict(zip([str(k) for k in z["algo_keys"]], z["algo"].tolist()))
    a = alg.Algorithm(optimizer=alg.Optimizer(int(kw["optimizer"])), ap_derivative=alg.APDerivative(int(kw["ap_derivative"])),
                      freeze_gains=bool(kw["freeze_gains"]), freeze_delays=bool(kw["freeze_delays"]),
                      batch_size=int(kw["batch_size"]), learning_rate=kw["learning_rate"],
                      difference_regularization_strength=kw["difference_regularization_strength"],
                      smoothness_regularization_strength=kw["smoothness_regularization_strength"])
    eng = alg.EpochEngine(ctx, gains=z["gains"], output_state_indices=z["output_state_indices"], coefs=z["coefs"],
                          delays=z["delays"], initial_delays=z["initial_delays"],
                          measurement_matrix=z["measurement_matrix"], control_matrix=z["control_matrix"],
                          control_function=z["control_function"], measurements=z["measurements_actual"],
                          algorithm=a)
    assert eng.run_epoch(0, beat_order=z["beat_order"]) == 1
    assert_bitwise(eng.read("system_states"), z["out_system_states"], "system_states (last beat)")
    assert rel_err(eng.read("measurements"), z["out_measurements"]) < TOL_MEAS
    assert rel_err(eng.read("grad_gains"), z["out_grad_gains"]) < TOL_GRAD
    assert rel_err(eng.read("grad_coefs"), z["out_grad_coefs"]) < TOL_GRAD
    g0 = z["gains"].astype(np.float64)
    assert rel_err(eng.read("gains") - g0, z["out_gains"] - g0) < TOL_GRAD
    np.testing.assert_array_equal(eng.read("delays"), z["out_delays"])
    assert rel_err(eng.read("loss"), z["out_loss"]) < TOL_LOSS
    assert rel_err(eng.read("loss_batch"), z["out_loss_batch"]) < TOL_LOSS
    avg = eng.read("average_delays")
    np.testing.assert_array_equal(np.isnan(avg), np.isnan(z["out_average_delays"]))
    eng.close()


CASES = {
    "sgd_gains": dict(learning_rate=0.5),
    "sgd_textbook_coefs": dict(learning_rate=0.5, freeze_delays=False),
    "sgd_simple_coefs": dict(learning_rate=0.5, freeze_delays=False, ap_derivative=0),
    "adam_all": dict(optimizer=1, learning_rate=1e-3, freeze_delays=False),
    "adam_regularised": dict(optimizer=1, learning_rate=1e-3, freeze_delays=False,
                             difference_regularization_strength=1e-3, smoothness_regularization_strength=1e-2,
                             maximum_regularization_threshold=0.5),
    "frozen": dict(freeze_gains=True, freeze_delays=True),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_epoch_vs_oracle(alg, ctx, oracle_mod, cuboid8, case):
    kw = CASES[case]
    kw = {k: (alg.Optimizer(v) if k == "optimizer" else alg.APDerivative(v) if k == "ap_derivative" else v)
          for k, v in kw.items()}
    a, oa = algo_pair(alg, oracle_mod, **kw)
    eng = alg.EpochEngine.from_scenario(ctx, cuboid8, num_batch_slots=2, algorithm=a)
    o = oracle_mod.from_scenario(cuboid8, num_batch_slots=2)
    g0, c0 = cuboid8.model.gains.astype(np.float64), cuboid8.model.coefs.astype(np.float64)
    for epoch in range(2):
        bi = eng.run_epoch(epoch)
        o.run_epoch(oa)
        assert bi == o.batch_index == epoch + 1
        if epoch == 0:
            assert_bitwise(eng.read("system_states"), o.system_states, "system_states")
        else:
            assert rel_err(eng.read("system_states"), o.system_states) < TOL_LOSS
        assert rel_err(eng.read("measurements"), o.measurements) < TOL_MEAS * (1 if epoch == 0 else 10)
        assert rel_err(eng.read("grad_gains"), o.d_gains) < TOL_GRAD
        assert rel_err(eng.read("grad_coefs"), o.d_coefs) < TOL_GRAD
        assert rel_err(eng.read("gains") - g0, o.gains - g0) < TOL_GRAD
        assert rel_err(eng.read("coefs") - c0, o.coefs - c0) < TOL_GRAD
        np.testing.assert_array_equal(eng.read("delays"), o.delays)
        for f, ref in [("loss", o.loss), ("loss_mse", o.loss_mse),
                       ("loss_maximum_regularization", o.loss_maximum_regularization),
                       ("loss_batch", o.loss_batch), ("loss_mse_batch", o.loss_mse_batch),
                       ("loss_maximum_regularization_batch", o.loss_maximum_regularization_batch)]:
            assert rel_err(eng.read(f), ref) < TOL_LOSS, f
        assert rel_err(eng.read("residuals"), o.residuals) < TOL_GRAD
        assert rel_err(eng.read("mapped_residuals"), o.mapped_residuals) < TOL_GRAD
        if epoch == 0:
            assert_bitwise(eng.read("maximum_regularization"), o.maximum_regularization, "maximum_regularization")
            assert_bitwise(eng.read("ap_outputs_now"), o.ap_outputs_now, "ap_outputs_now")
        assert int(eng.read("adam_step")[0]) == int(o.step[0])
    eng.close()


def test_derivatives_bitwise_given_mapped_residuals(alg, ctx, oracle_mod, cuboid8):
    """With the GPU's own H^T r fed to the CPU loop, gradients and the update agree bit for bit."""
    a, oa = algo_pair(alg, oracle_mod, optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False,
                      difference_regularization_strength=1e-3, maximum_regularization_threshold=0.5)
    eng = alg.EpochEngine.from_scenario(ctx, cuboid8, algorithm=a)
    eng.run_epoch(0)
    mr = eng.read("mapped_residuals_history")
    o = oracle_mod.from_scenario(cuboid8)
    o.mapped_residuals_override = np.ascontiguousarray(mr[None])
    o.run_epoch(oa)
    assert_bitwise(eng.read("system_states"), o.system_states, "system_states")
    assert_bitwise(eng.read("ap_outputs_now"), o.ap_outputs_now, "ap_outputs_now")
    assert_bitwise(eng.read("ap_outputs_last"), o.ap_outputs_last, "ap_outputs_last")
    assert_bitwise(eng.read("coefs_fir"), o.coefs_fir, "coefs_fir")
    assert_bitwise(eng.read("coefs_iir"), o.coefs_iir, "coefs_iir")
    assert_bitwise(eng.read("grad_gains"), o.d_gains, "grad_gains")
    assert_bitwise(eng.read("grad_coefs"), o.d_coefs, "grad_coefs")
    assert_bitwise(eng.read("gains"), o.gains, "gains after Adam")
    assert_bitwise(eng.read("coefs"), o.coefs, "coefs after Adam + roll")
    np.testing.assert_array_equal(eng.read("delays"), o.delays)
    assert_bitwise(eng.read("gains_first_moment"), o.gains_first_moment, "Adam m")
    assert_bitwise(eng.read("gains_second_moment"), o.gains_second_moment, "Adam v")
    assert_bitwise(eng.read("average_delays"), o.average_delays, "average_delays")
    eng.close()


def test_batches_and_beat_order(alg, ctx, oracle_mod):
    """3 beats, batch_size 2: an in-loop update, a derivative reset, and a final partial batch."""
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=(5, 4, 3), num_steps=80, num_beats=3, patho_size=2, patho_origin=(1, 1, 0),
                           pulse_onset=1, pulse_sigma_samples=4.0, noise_fraction=0.02, seed=5)
    scn = sc.attach_measurements(sc.build(spec), oracle_forward(oracle_mod))
    a, oa = algo_pair(alg, oracle_mod, batch_size=2, learning_rate=0.5, freeze_delays=False)
    eng = alg.EpochEngine.from_scenario(ctx, scn, num_batch_slots=4, algorithm=a)
    o = oracle_mod.from_scenario(scn, num_batch_slots=4)
    order = np.array([2, 0, 1], np.int32)
    bi = eng.run_epoch(0, beat_order=order)
    o.run_epoch(oa, beat_order=order)
    assert bi == o.batch_index == 2
    # the last beat runs after the in-loop update, whose parameters agree within the gradient tolerance
    assert rel_err(eng.read("system_states"), o.system_states) < TOL_LOSS
    assert rel_err(eng.read("measurements"), o.measurements) < 10 * TOL_MEAS
    assert rel_err(eng.read("loss_batch"), o.loss_batch) < TOL_LOSS
    g0 = scn.model.gains.astype(np.float64)
    assert rel_err(eng.read("gains") - g0, o.gains - g0) < TOL_GRAD
    assert int(eng.read("adam_step")[0]) == 3
    eng.close()


@pytest.mark.parametrize("shape,T", [((1, 1, 1), 5), ((2, 1, 1), 1), ((2, 2, 1), 2), ((3, 3, 3), 3)])
def test_edge_shapes(alg, ctx, oracle_mod, shape, T):
    """A lone voxel (no neighbours), one and two steps, a 3^3 block with T below every delay."""
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=shape, num_steps=T, num_sensors=2, patho_size=0, pulse_onset=0,
                           pulse_sigma_samples=1.0, seed=1)
    scn = sc.build(spec)
    scn.measurements = np.zeros((1, T, scn.num_sensors), np.float32)
    a, oa = algo_pair(alg, oracle_mod, learning_rate=0.5, freeze_delays=False)
    eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=a)
    o = oracle_mod.from_scenario(scn)
    eng.run_epoch(0)
    o.run_epoch(oa)
    assert_bitwise(eng.read("system_states"), o.system_states, "system_states")
    assert rel_err(eng.read("grad_gains"), o.d_gains) < TOL_GRAD
    assert rel_err(eng.read("loss_batch"), o.loss_batch) < TOL_LOSS
    eng.close()


def test_long_delays_beyond_steps(alg, ctx, oracle_mod, cuboid8):
    """Delays larger than the number of steps: every history read is the zero before t = 0."""
    d = np.where(cuboid8.model.delays > 0, 700, 0).astype(np.int32)
    from cardiotrust_b200 import scenario as sc
    import dataclasses

    model = dataclasses.replace(cuboid8.model, delays=d)
    scn = dataclasses.replace(cuboid8, model=model)
    a, oa = algo_pair(alg, oracle_mod, learning_rate=0.5)
    eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=a)
    o = oracle_mod.from_scenario(scn)
    eng.run_epoch(0)
    o.run_epoch(oa)
    assert_bitwise(eng.read("system_states"), o.system_states, "system_states")
    eng.close()


def test_invalid_inputs(alg, ctx, cuboid8):
    from cardiotrust_b200 import _lib

    m = cuboid8.model
    osi = m.output_state_indices.copy()
    osi[3, 5] = osi[3, 5] + 1 if osi[3, 5] >= 0 else 4
    with pytest.raises(_lib.CtError) as e:
        alg.EpochEngine(ctx, gains=m.gains, output_state_indices=osi, coefs=m.coefs, delays=m.delays,
                        initial_delays=m.initial_delays, measurement_matrix=cuboid8.measurement_matrix,
                        control_matrix=cuboid8.control_matrix, control_function=cuboid8.control_function)
    assert e.value.status == _lib.CT_ERR_INVALID_INDEX
    d = m.delays.copy()
    d[d > 0] = 0
    with pytest.raises(_lib.CtError) as e:
        alg.EpochEngine(ctx, gains=m.gains, output_state_indices=m.output_state_indices, coefs=m.coefs, delays=d,
                        initial_delays=m.initial_delays, measurement_matrix=cuboid8.measurement_matrix,
                        control_matrix=cuboid8.control_matrix, control_function=cuboid8.control_function)
    assert e.value.status == _lib.CT_ERR_INVALID_ARGUMENT
    eng = alg.EpochEngine.from_scenario(ctx, cuboid8, num_batch_slots=1)
    eng.run_epoch(0)
    with pytest.raises(_lib.CtError) as e:
        eng.run_epoch(1)
    assert e.value.status == _lib.CT_ERR_BATCH_INDEX
    with pytest.raises(_lib.CtError) as e:
        eng.run_epoch(0, grad_mode=7)
    assert e.value.status == _lib.CT_ERR_NOT_SUPPORTED
    with pytest.raises(_lib.CtError):
        eng.run_epoch(0, beat_order=np.array([3], np.int32))
    eng.close()


def test_reference_shaped_api(alg, ctx, oracle_mod, cuboid8):
    """run_epoch(results, &mut batch_index, data, config) over three epochs: loss_batch decreases."""
    eng = alg.EpochEngine.from_scenario(ctx, cuboid8, num_batch_slots=3)
    results = alg.Results(eng)
    bi = alg.BatchIndex(0)
    data = alg.Data(measurements=cuboid8.measurements)
    cfg = alg.Algorithm(learning_rate=0.5, epochs=3)
    for _ in range(cfg.epochs):
        alg.run_epoch(results, bi, data, cfg)
    lb = results.metrics.loss_batch
    assert bi.value == 3
    assert lb[0] > lb[1] > lb[2], lb
    eng.close()


@pytest.mark.parametrize("precision,tol_meas,tol_grad", [(1, TOL_MEAS, TOL_GRAD), (2, 5e-4, 5e-3),
                                                         (3, TOL_MEAS, TOL_GRAD)])
def test_tensor_core_precisions(alg, ctx, oracle_mod, cuboid8, precision, tol_meas, tol_grad):
    """tcgen05 measurement products: split TF32 and the sliced BF16 products keep the FP32 bars;
    one-pass TF32 has looser, stated bars (operands rounded to 10-bit mantissas)."""
    a, oa = algo_pair(alg, oracle_mod, optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    eng = alg.EpochEngine.from_scenario(ctx, cuboid8, num_batch_slots=2, algorithm=a)
    o = oracle_mod.from_scenario(cuboid8, num_batch_slots=2)
    o64 = oracle_mod.from_scenario(cuboid8, num_batch_slots=2, dtype=np.float64)
    g0 = cuboid8.model.gains.astype(np.float64)
    for epoch in range(2):
        eng.run_epoch(epoch, precision=alg.Precision(precision))
        o.run_epoch(oa)
        o64.run_epoch(oa)
        if epoch == 0:
            assert_bitwise(eng.read("system_states"), o.system_states, "system_states")
        assert rel_err(eng.read("measurements"), o64.measurements) < tol_meas * (1 if epoch == 0 else 10)
        assert rel_err(eng.read("grad_gains"), o64.d_gains) < tol_grad
        assert rel_err(eng.read("grad_coefs"), o64.d_coefs) < tol_grad
        assert rel_err(eng.read("gains") - g0, o64.gains - g0) < tol_grad
        assert rel_err(eng.read("loss_batch"), o64.loss_batch) < 10 * TOL_LOSS
    eng.close()


def test_tensor_core_shapes(alg, ctx, oracle_mod):
    """tcgen05 path on ragged shapes: T not a multiple of 128, more than 128 sensor rows (two N tiles of
    the H x product), states not a multiple of the 256-wide H^T r tile."""
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=(6, 5, 4), num_steps=203, num_sensors=50, patho_size=2, patho_origin=(2, 2, 1),
                           pulse_onset=1, pulse_sigma_samples=4.0, noise_fraction=0.01, seed=9)
    scn = sc.attach_measurements(sc.build(spec), oracle_forward(oracle_mod))
    assert scn.num_sensors == 150 and scn.num_states % 4 == 0
    a, oa = algo_pair(alg, oracle_mod, learning_rate=0.5, freeze_delays=False)
    o64 = oracle_mod.from_scenario(scn, dtype=np.float64)
    o64.run_epoch(oa)
    for precision in (alg.Precision.Fp32, alg.Precision.Tf32x3, alg.Precision.Bf16x6):
        eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=a)
        eng.run_epoch(0, precision=precision)
        assert rel_err(eng.read("measurements"), o64.measurements) < TOL_MEAS, precision
        assert rel_err(eng.read("mapped_residuals_history"), _mr_history(o64, scn)) < 1e-4, precision
        assert rel_err(eng.read("grad_gains"), o64.d_gains) < TOL_GRAD, precision
        eng.close()


def test_tensor_core_many_sensor_rows(alg, ctx, oracle_mod):
    """256 triaxial sensors (768 rows, as in the precision config): H x takes three 256-column tiles."""
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=(6, 5, 4), num_steps=140, num_sensors=256, patho_size=2, patho_origin=(2, 2, 1),
                           pulse_onset=1, pulse_sigma_samples=4.0, noise_fraction=0.01, seed=12)
    scn = sc.attach_measurements(sc.build(spec), oracle_forward(oracle_mod))
    assert scn.num_sensors == 768 and scn.num_states % 4 == 0
    a, oa = algo_pair(alg, oracle_mod, optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    o64 = oracle_mod.from_scenario(scn, dtype=np.float64)
    o64.run_epoch(oa)
    for precision in (alg.Precision.Tf32x3, alg.Precision.Tf32, alg.Precision.Bf16x6):
        eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=a)
        eng.run_epoch(0, precision=precision)
        loose = precision == alg.Precision.Tf32
        assert rel_err(eng.read("measurements"), o64.measurements) < (5e-4 if loose else TOL_MEAS), precision
        assert rel_err(eng.read("mapped_residuals_history"), _mr_history(o64, scn)) < (5e-3 if loose else 1e-4)
        assert rel_err(eng.read("grad_gains"), o64.d_gains) < (5e-3 if loose else TOL_GRAD), precision
        eng.close()


@pytest.mark.parametrize("shape", [(5, 5, 5), (7, 3, 3), (6, 5, 3)])
def test_tensor_core_state_count_not_multiple_of_4(alg, ctx, oracle_mod, shape):
    """States not a multiple of 4 (375, 189 and 270 states): the H x operand is padded to 16-byte rows
    (zero columns) and the tcgen05 products keep the FP32 bars, in both gradient modes."""
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=shape, num_steps=160, num_sensors=20, patho_size=2, patho_origin=(1, 1, 1),
                           pulse_onset=1, pulse_sigma_samples=4.0, noise_fraction=0.01, seed=13)
    scn = sc.attach_measurements(sc.build(spec), oracle_forward(oracle_mod))
    assert scn.num_states % 4 != 0
    a, oa = algo_pair(alg, oracle_mod, optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    o64 = oracle_mod.from_scenario(scn, dtype=np.float64)
    o64.run_epoch(oa)
    adj = oracle_mod.from_scenario(scn, dtype=np.float64)
    adj.run_epoch(oa, adjoint=True)
    for mode, ref in ((alg.GradMode.Reference, o64), (alg.GradMode.Adjoint, adj)):
        for precision in (alg.Precision.Tf32x3, alg.Precision.Bf16x6):
            eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=a)
            eng.run_epoch(0, grad_mode=mode, precision=precision)
            assert rel_err(eng.read("measurements"), ref.measurements) < TOL_MEAS, (mode, precision)
            assert rel_err(eng.read("grad_gains"), ref.d_gains) < TOL_GRAD, (mode, precision)
            assert rel_err(eng.read("grad_coefs"), ref.d_coefs) < TOL_GRAD, (mode, precision)
            eng.close()


def _mr_history(o64, scn):
    """H^T r of every step of the last beat, in float64, from the oracle's residuals."""
    H = scn.measurement_matrix[-1].astype(np.float64)
    r = o64.measurements[-1].astype(np.float64) - scn.measurements[-1].astype(np.float64)
    return r @ H


def test_run_epoch_host_matches_device_path(alg, ctx, cuboid8):
    """ct_run_epoch_host (model in host memory, copied in and back every epoch, one wait) gives the
    same parameters and batch-wise losses, bit for bit, as writing the fields, running ct_run_epoch
    and reading them back; over three epochs (reference, adjoint, reference gradients) the host
    arrays carry the model forward."""
    import torch

    cfg = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-2, freeze_delays=False)
    ref = alg.EpochEngine.from_scenario(ctx, cuboid8, num_batch_slots=3, algorithm=cfg)
    eng = alg.EpochEngine.from_scenario(ctx, cuboid8, num_batch_slots=3, algorithm=cfg)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    gains, coefs, delays = pin(ref.read("gains")), pin(ref.read("coefs")), pin(ref.read("delays"))
    meas = pin(cuboid8.measurements)
    loss = pin(np.zeros(eng.dims["NB"], np.float32))
    bi_ref = bi = 0
    for mode in (alg.GradMode.Reference, alg.GradMode.Adjoint, alg.GradMode.Reference):
        bi_ref = ref.run_epoch(bi_ref, beat_order=[0], grad_mode=mode, sync=True)
        bi = eng.run_epoch_host(bi, gains, coefs, delays, meas, loss, beat_order=[0], grad_mode=mode)
    assert bi == bi_ref == 3
    assert_bitwise(gains, ref.read("gains"), "gains")
    assert_bitwise(coefs, ref.read("coefs"), "coefs")
    assert np.array_equal(delays, ref.read("delays"))
    assert_bitwise(loss, ref.read("loss_batch"), "loss_batch")
    # a connected pair with delay 0 is refused before anything is copied
    bad = delays.copy()
    osi = cuboid8.model.output_state_indices
    v, n = np.argwhere(osi[0::3, 0::3] >= 0)[0]
    bad[v, n] = 0
    before = gains.copy()
    with pytest.raises(alg.CtError) as err:
        eng.run_epoch_host(bi, gains, coefs, bad, meas, loss, beat_order=[0])
    assert err.value.status == alg._lib.CT_ERR_INVALID_ARGUMENT
    assert_bitwise(gains, before, "gains after a refused call")
    ref.close()
    eng.close()
