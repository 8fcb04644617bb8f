"""The adjoint (back-propagation through time) restatement in the oracle,
checked against central finite differences of the stated loss in float64.

The adjoint mode has no counterpart in the reference crate; its oracle is
pinned by these finite-difference checks (eps 1e-3, 200 random parameters:
gains of connected pairs and all-pass coefficients) and by the identity of
its forward, metrics and update with the reference epoch."""

import numpy as np
import pytest

import oracle as orc
from cardiotrust_b200 import scenario as sc

from conftest import oracle_forward

FD_EPS = 1e-3


@pytest.fixture(scope="module")
def small(oracle_mod):
    spec = sc.ScenarioSpec(
        shape=(5, 4, 4), num_steps=90, num_sensors=8, patho_size=2, patho_origin=(1, 1, 1), pulse_onset=5,
        pulse_sigma_samples=4.0, noise_fraction=0.01, seed=3,
    )
    scn = sc.build(spec)
    return sc.attach_measurements(scn, oracle_forward(oracle_mod))


def _algo(**kw):
    base = dict(freeze_gains=0, freeze_delays=0, maximum_regularization_threshold=0.05, maximum_regularization_strength=0.5)
    base.update(kw)
    return orc.algo(**base)


def _fd_params(scn, count, seed, kink_rows=()):
    """Random (kind, flat index) pairs: half gains of connected (i, k), half coefficients of connected (v, n).

    Gains of the rows in ``kink_rows`` are left out: there the state is exactly
    0 while its voxel's maximum regularisation is active, where |x| has no
    derivative (the reference takes signum(0) = 1, central differences see 0)."""
    rng = np.random.default_rng(seed)
    osi = scn.model.output_state_indices
    ok = osi >= 0
    ok[list(kink_rows), :] = False
    gain_idx = np.flatnonzero(ok.reshape(-1))
    coef_idx = np.flatnonzero(osi[0::3, 0::3].reshape(-1) >= 0)
    g = rng.choice(gain_idx, count // 2, replace=False)
    c = rng.choice(coef_idx, count - count // 2, replace=False)
    return [("gains", int(i)) for i in g] + [("coefs", int(i)) for i in c]


def test_adjoint_matches_central_differences(small):
    a = _algo()
    e = orc.from_scenario(small, dtype=np.float64)
    loss0 = e.stated_loss(a, gradient=True)
    assert loss0 > 0
    grads = {"gains": e.d_gains.copy(), "coefs": e.d_coefs.copy()}
    assert np.abs(grads["gains"]).max() > 0 and np.abs(grads["coefs"]).max() > 0
    T, S = e.system_states.shape
    xs = e.system_states.reshape(T, S // 3, 3)
    active = np.abs(xs).sum(-1) > a.maximum_regularization_threshold
    kink = (xs == 0) & active[:, :, None]
    kink_rows = np.unique(np.nonzero(kink)[1] * 3 + np.nonzero(kink)[2])
    params = _fd_params(small, 200, seed=11, kink_rows=kink_rows)
    fd = np.empty(len(params))
    adj = np.empty(len(params))
    for q, (kind, idx) in enumerate(params):
        arr = getattr(e, kind).reshape(-1)
        keep = arr[idx]
        arr[idx] = keep + FD_EPS
        lp = e.stated_loss(a)
        arr[idx] = keep - FD_EPS
        lm = e.stated_loss(a)
        arr[idx] = keep
        fd[q] = (lp - lm) / (2 * FD_EPS)
        adj[q] = grads[kind].reshape(-1)[idx]
    # central differences carry O(eps^2) truncation error: compare per kind against the kind's scale
    for kind in ("gains", "coefs"):
        sel = np.array([p[0] == kind for p in params])
        scale = np.abs(adj[sel]).max()
        err = np.abs(fd[sel] - adj[sel]).max() / scale
        assert err < 1e-4, (kind, err)
    rel = np.linalg.norm(fd - adj) / np.linalg.norm(adj)
    assert rel < 1e-4, rel


def test_adjoint_difference_regularisation_term(small):
    """The difference-regularisation part of the coefficient gradient is count * diff * delta^5 per (v, n)."""
    e0 = orc.from_scenario(small, dtype=np.float64)
    e0.stated_loss(_algo(difference_regularization_strength=0.0), gradient=True)
    base = e0.d_coefs.copy()
    for deriv, counts in ((1, None), (0, "simple")):
        e = orc.from_scenario(small, dtype=np.float64)
        e.stated_loss(_algo(difference_regularization_strength=0.25, ap_derivative=deriv), gradient=True)
        T = small.num_steps
        d = small.model.delays.astype(np.float64)
        c = small.model.coefs.astype(np.float64)
        delta = small.model.initial_delays.astype(np.float64) - (d + (1 - c) / (1 + c))
        if counts is None:
            n = np.full_like(d, 9 * T)
        else:
            connected = small.model.output_state_indices[0::3, 0::3] >= 0
            n = np.where(connected, 9 * np.maximum(0, T - d), 0)
        np.testing.assert_allclose(e.d_coefs - base, n * 0.25 * delta**5, rtol=1e-9, atol=1e-12)


def test_adjoint_epoch_keeps_reference_forward_and_metrics(small):
    """run_epoch in adjoint mode: same states, measurements and metrics as the reference epoch; its
    gradients are the stated-loss gradient of the pre-update parameters."""
    a = _algo(optimizer=1, learning_rate=1e-3)
    ref = orc.from_scenario(small, dtype=np.float64)
    ref.run_epoch(a)
    adj = orc.from_scenario(small, dtype=np.float64)
    adj.run_epoch(a, adjoint=True)
    for name in ("system_states", "measurements", "loss", "loss_mse", "loss_maximum_regularization", "loss_batch"):
        np.testing.assert_array_equal(getattr(adj, name), getattr(ref, name), err_msg=name)
    g = orc.from_scenario(small, dtype=np.float64)
    g.stated_loss(a, gradient=True)
    np.testing.assert_allclose(adj.d_gains, g.d_gains, rtol=0, atol=0)
    np.testing.assert_allclose(adj.d_coefs, g.d_coefs, rtol=0, atol=0)
    assert int(adj.step[0]) == 2


def test_adjoint_instantaneous_part_is_reference_gain_derivative(small):
    """Over a single step nothing propagates through time: the adjoint gain gradient equals the
    reference's per-step gain derivative (derivation.rs:307-329)."""
    spec = sc.ScenarioSpec(shape=(3, 3, 3), num_steps=1, num_sensors=4, pulse_onset=0, pulse_sigma_samples=1.0, seed=5)
    scn = sc.build(spec)
    scn.measurements = np.random.default_rng(0).normal(size=(1, 1, 12)).astype(np.float32)
    a = _algo(freeze_delays=1)
    ref = orc.from_scenario(scn, dtype=np.float64)
    ref.run_epoch(a)
    g = orc.from_scenario(scn, dtype=np.float64)
    g.stated_loss(a, gradient=True)
    np.testing.assert_allclose(g.d_gains, ref.d_gains, rtol=1e-12, atol=1e-15)
