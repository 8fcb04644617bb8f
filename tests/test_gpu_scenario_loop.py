"""The epoch loop run_model_based (src/core/scenario.rs:725-795) on the GPU
against the oracle's restatement, and the batched loop against one-at-a-time
GPU loops.

Bars: states of the first epoch and the learning-rate-0 snapshot
bit-identical; losses <= 1e-4 and parameter changes <= 1e-3 relative (the
epoch's own bars); the early stop at the same epoch; batched members
bit-identical to their single runs in reference mode."""

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


def _scenario(oracle_mod, seed, shape=(6, 5, 4), steps=200, beats=2):
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=shape, num_steps=steps, num_beats=beats, patho_size=2, pulse_onset=3,
                           pulse_sigma_samples=5.0, noise_fraction=0.01, seed=seed)
    return sc.attach_measurements(sc.build(spec), oracle_forward(oracle_mod))


@pytest.fixture(scope="module")
def small(oracle_mod):
    return _scenario(oracle_mod, 11)


def _oracle_algo(oracle_mod, a):
    return oracle_mod.algo(optimizer=int(a.optimizer), ap_derivative=int(a.ap_derivative),
                           freeze_gains=int(a.freeze_gains), freeze_delays=int(a.freeze_delays),
                           batch_size=a.batch_size, learning_rate=a.learning_rate)


@pytest.mark.parametrize("optimizer", ["sgd", "adam"])
def test_run_model_based_matches_oracle(alg, ctx, oracle_mod, small, optimizer):
    epochs = 5
    a = alg.Algorithm(epochs=epochs, learning_rate=0.5 if optimizer == "sgd" else 2e-3,
                      optimizer=alg.Optimizer.Sgd if optimizer == "sgd" else alg.Optimizer.Adam,
                      freeze_delays=optimizer == "sgd", learning_rate_reduction_interval=2,
                      learning_rate_reduction_factor=0.5, snapshots_interval=2)
    orders = np.array([[1, 0], [0, 1], [1, 0], [0, 1], [0, 1]], np.int32)
    eng = alg.EpochEngine.from_scenario(ctx, small, num_batch_slots=2 * epochs, algorithm=a)
    summary, losses, bi = eng.run_model_based(0, beat_orders=orders)
    o = oracle_mod.from_scenario(small, num_batch_slots=2 * epochs)
    oa = _oracle_algo(oracle_mod, a)
    osum, olosses, osnaps = o.run_model_based(oa, epochs, 2, 0.5, 2, beat_orders=orders)
    assert summary["epochs_run"] == osum["epochs_run"] == epochs and bi == o.batch_index
    assert summary["snapshots"] == 3
    assert rel_err(losses, olosses) < 1e-4
    g0, c0 = small.model.gains, small.model.coefs
    assert rel_err(eng.read("gains") - g0, o.gains - g0) < 1e-3
    assert rel_err(eng.read("coefs") - c0, o.coefs - c0) < 1e-3
    np.testing.assert_array_equal(eng.read("delays"), o.delays)
    assert rel_err(eng.read("average_delays"), o.average_delays) < 1e-4
    snaps = {f: eng.read_snapshots(f) for f in ("gains", "coefs", "delays", "system_states", "measurements")}
    assert all(len(v) == 3 for v in snaps.values())
    # epoch 0 runs at learning rate 0: parameters unchanged and states bit-identical to the oracle
    np.testing.assert_array_equal(snaps["gains"][0], g0)
    np.testing.assert_array_equal(snaps["system_states"][0], osnaps["system_states"][0])
    for k in range(3):
        assert rel_err(snaps["gains"][k] - g0, osnaps["gains"][k] - g0) < 1e-3
        np.testing.assert_array_equal(snaps["delays"][k], osnaps["delays"][k])
        assert rel_err(snaps["measurements"][k], osnaps["measurements"][k]) < 1e-4
    eng.close()


def test_run_model_based_stops_like_the_oracle(alg, ctx, oracle_mod, small):
    a = alg.Algorithm(epochs=8, learning_rate=1e30)
    orders = np.tile(np.array([0, 1], np.int32), (8, 1))
    eng = alg.EpochEngine.from_scenario(ctx, small, num_batch_slots=16, algorithm=a)
    summary, losses, _ = eng.run_model_based(0, beat_orders=orders)
    o = oracle_mod.from_scenario(small, num_batch_slots=16)
    osum, olosses, _ = o.run_model_based(_oracle_algo(oracle_mod, a), 8, beat_orders=orders)
    assert summary["epochs_run"] == osum["epochs_run"] < 8
    assert not np.isfinite(summary["loss"]) and len(losses) == summary["epochs_run"]
    assert rel_err(losses[:-1], olosses[:-1]) < 1e-4
    eng.close()


def test_batched_loop_matches_single_loops(alg, ctx, oracle_mod, small):
    """Three members, the second diverges: it stops on its own and the others finish as a smaller
    batch, bit-identical to their one-at-a-time loops (reference mode, beats in index order)."""
    scns = [small, _scenario(oracle_mod, 12, shape=(5, 5, 5), steps=150, beats=1),
            _scenario(oracle_mod, 13, shape=(7, 4, 4), steps=180, beats=3)]
    epochs = 6
    lrs = [0.5, 1e30, 0.25]
    mk = lambda lr: alg.Algorithm(epochs=epochs, learning_rate=lr, learning_rate_reduction_interval=3,  # noqa: E731
                                  learning_rate_reduction_factor=0.5)
    batched = [alg.EpochEngine.from_scenario(ctx, s, num_batch_slots=3 * epochs, algorithm=mk(lr))
               for s, lr in zip(scns, lrs)]
    single = [alg.EpochEngine.from_scenario(ctx, s, num_batch_slots=3 * epochs, algorithm=mk(lr))
              for s, lr in zip(scns, lrs)]
    batch = alg.EpochBatch(ctx, batched)
    summaries, losses = batch.run_model_based(mk(1.0))
    assert summaries[1]["epochs_run"] < epochs
    assert summaries[0]["epochs_run"] == summaries[2]["epochs_run"] == epochs
    for k, (s, e) in enumerate(zip(scns, single)):
        orders = np.tile(np.arange(s.num_beats, dtype=np.int32), (epochs, 1))
        ssum, slosses, sbi = e.run_model_based(0, beat_orders=orders)
        assert ssum["epochs_run"] == summaries[k]["epochs_run"], k
        assert sbi == batch.batch_indices[k]
        n = ssum["epochs_run"]
        np.testing.assert_array_equal(losses[k, :n], slosses, err_msg=str(k))
        if k != 1:
            for f in ("gains", "coefs", "delays", "average_delays"):
                np.testing.assert_array_equal(batched[k].read(f), e.read(f), err_msg=f"{k} {f}")
    batch.close()
    for e in batched + single:
        e.close()
