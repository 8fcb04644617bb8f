"""Batched scenarios (one persistent launch per phase over every member, the
epoch replayed from a CUDA graph) against the same scenarios run one at a
time through ct_run_epoch with beats in index order.

The batched forward uses the same arithmetic as the single-scenario forward
and each tile writes its own step partial, so states and metrics are
bit-identical; gradients and updates in adjoint mode differ only in the
order gradient sums are added (per block instead of once per launch)."""

import numpy as np
import pytest

from conftest import oracle_forward, rel_err

pytestmark = pytest.mark.gpu


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
def members(oracle_mod):
    from cardiotrust_b200 import scenario as sc

    specs = [
        sc.ScenarioSpec(shape=(6, 5, 4), num_steps=200, num_beats=2, patho_size=2, pulse_onset=3,
                        pulse_sigma_samples=5.0, noise_fraction=0.01, seed=1),
        sc.ScenarioSpec(shape=(8, 8, 4), num_steps=300, num_beats=1, num_sensors=12, patho_size=2, pulse_onset=5,
                        pulse_sigma_samples=6.0, noise_fraction=0.01, seed=2),
        sc.ScenarioSpec(shape=(10, 9, 8), mask="shell", shell_semi_axes=(5.0, 4.5, 4.0), shell_thickness=2.0,
                        num_steps=260, num_beats=3, patho_size=2, pulse_onset=2, pulse_sigma_samples=5.0,
                        noise_fraction=0.01, seed=3),
        sc.ScenarioSpec(shape=(5, 5, 5), num_steps=150, num_beats=2, num_sensors=20, patho_size=2, pulse_onset=4,
                        pulse_sigma_samples=4.0, noise_fraction=0.01, seed=4),
    ]
    return [sc.attach_measurements(sc.build(s), oracle_forward(oracle_mod)) for s in specs]


def _engines(alg, ctx, members, algo):
    return [alg.EpochEngine.from_scenario(ctx, m, num_batch_slots=8, algorithm=algo) for m in members]


@pytest.mark.parametrize("precision", ["Fp32", "Bf16x6"])
@pytest.mark.parametrize("mode", ["reference", "adjoint"])
def test_batch_matches_single_runs(alg, ctx, members, mode, precision):
    gm = alg.GradMode.Adjoint if mode == "adjoint" else alg.GradMode.Reference
    prec = alg.Precision[precision]
    algo = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    batched = _engines(alg, ctx, members, algo)
    single = _engines(alg, ctx, members, algo)
    batch = alg.EpochBatch(ctx, batched, grad_mode=gm, precision=prec)
    for epoch in range(2):
        idx = batch.run_epoch()
        assert list(idx) == [epoch + 1] * len(members)
        for m, e in zip(members, single):
            e.run_epoch(epoch, beat_order=np.arange(m.num_beats), grad_mode=gm, precision=prec)
        for k, (b, e) in enumerate(zip(batched, single)):
            if epoch == 0:
                np.testing.assert_array_equal(b.read("system_states"), e.read("system_states"), err_msg=str(k))
                np.testing.assert_array_equal(b.read("loss"), e.read("loss"), err_msg=str(k))
            tol = 1e-6 if mode == "adjoint" else 0.0
            for f in ("grad_gains", "grad_coefs", "gains", "coefs"):
                got, want = b.read(f), e.read(f)
                if tol == 0.0:
                    np.testing.assert_array_equal(got, want, err_msg=f"{k} {f}")
                else:
                    assert rel_err(got, want) < tol, (k, f)
            np.testing.assert_array_equal(b.read("delays"), e.read("delays"))
            assert rel_err(b.read("loss_batch"), e.read("loss_batch")) < 1e-6
    info = batch.info()
    assert info["uses_graph"] and info["graph_kernels"] > 0
    batch.close()
    for e in batched + single:
        e.close()


def test_batch_tensor_core_precision(alg, ctx, members):
    """Every member on the tensor cores, including those whose state count is not a multiple of 4."""
    algo = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    assert any(m.num_states % 4 for m in members)
    batched = _engines(alg, ctx, members, algo)
    single = _engines(alg, ctx, members, algo)
    batch = alg.EpochBatch(ctx, batched, grad_mode=alg.GradMode.Adjoint, precision=alg.Precision.Tf32x3)
    batch.run_epoch()
    for m, e in zip(members, single):
        e.run_epoch(0, beat_order=np.arange(m.num_beats), grad_mode=alg.GradMode.Adjoint,
                    precision=alg.Precision.Tf32x3)
    for b, e in zip(batched, single):
        assert rel_err(b.read("grad_gains"), e.read("grad_gains")) < 1e-6
    batch.close()
    for e in batched + single:
        e.close()


def test_batch_rejects_per_batch_updates(alg, ctx, members):
    from cardiotrust_b200._lib import CtError

    a = alg.Algorithm(batch_size=1)
    engs = _engines(alg, ctx, members[:2], a)
    with pytest.raises(CtError):
        alg.EpochBatch(ctx, engs)
    for e in engs:
        e.close()


def test_batch_recaptures_after_algorithm_change(alg, ctx, members):
    algo = alg.Algorithm(optimizer=alg.Optimizer.Sgd, learning_rate=0.5)
    batched = _engines(alg, ctx, members[:2], algo)
    single = _engines(alg, ctx, members[:2], algo)
    batch = alg.EpochBatch(ctx, batched)
    batch.run_epoch()
    for m, e in zip(members[:2], single):
        e.run_epoch(0, beat_order=np.arange(m.num_beats))
    for e in batched + single:
        e.set_learning_rate(0.25)
    batch.run_epoch()
    for m, e in zip(members[:2], single):
        e.run_epoch(1, beat_order=np.arange(m.num_beats))
    for b, e in zip(batched, single):
        assert rel_err(b.read("gains"), e.read("gains")) < 1e-6
    batch.close()
    for e in batched + single:
        e.close()


def test_batch_autotune_trains_like_single_runs(alg, ctx, members):
    """The autotuner's trial epochs are real epochs: after it, every member has trained exactly as many
    epochs as its one-at-a-time twin (schedules change the order of nothing but independent work)."""
    algo = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    batched = _engines(alg, ctx, members, algo)
    single = _engines(alg, ctx, members, algo)
    batch = alg.EpochBatch(ctx, batched, grad_mode=alg.GradMode.Adjoint)
    choice = batch.autotune()
    assert choice["ckpt_steps"] in (32, 64, 128) and choice["tile_order"] in (0, 1, 2) and choice["epoch_ms"] > 0
    epochs = int(batch.batch_indices[0])
    assert epochs == 5 and all(int(i) == epochs for i in batch.batch_indices)
    batch.run_epoch()
    for m, e in zip(members, single):
        for ep in range(epochs + 1):
            e.run_epoch(ep, beat_order=np.arange(m.num_beats), grad_mode=alg.GradMode.Adjoint)
    for b, e in zip(batched, single):
        assert rel_err(b.read("gains"), e.read("gains")) < 1e-5
        assert rel_err(b.read("coefs"), e.read("coefs")) < 1e-5
        np.testing.assert_array_equal(b.read("delays"), e.read("delays"))
    batch.close()
    for e in batched + single:
        e.close()
