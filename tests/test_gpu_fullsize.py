"""The configurations at their stated sizes, through the C ABI, against the oracle.

* 20x20x20 cuboid (24,000 states), the full 2,000-step beat, 111 sensor rows, 1 % noise, Adam:
  states bit-identical to the f32 oracle, reference-mode and adjoint gradients within 1e-3 of the
  f64 oracle, for the FP32 CUDA-core and the sliced BF16 tensor-core products.
* The 64x64x48 ellipsoidal shell (47,264 voxels, 141,792 states), 111 sensor rows: the GPU adjoint
  over a 600-step beat (three segments of the 256-step checkpoint interval, recomputed between
  checkpoints) within 1e-3 of the f64 oracle's back-propagation.
* The same shell geometry on a 40-step beat: the f64 oracle's adjoint and the GPU adjoint against
  central differences (eps 1e-3) of the stated loss on 200 random parameters (gains of connected
  pairs and all-pass coefficients, up to 100 of them, drawn where the beat's gradient is not zero).
"""

import numpy as np
import pytest

from conftest import oracle_forward, rel_err

pytestmark = pytest.mark.gpu

TOL_GRAD = 1e-3
FD_EPS = 1e-3


def _noisy(scn, oracle_mod, fraction=0.01):
    t = scn.truth
    fwd = oracle_mod.OracleEpoch(t.gains, t.output_state_indices, t.coefs, t.delays, t.initial_delays,
                                 scn.measurement_matrix, scn.control_matrix, scn.control_function)
    y = fwd.simulate().astype(np.float64)
    del fwd
    rng = np.random.default_rng(scn.spec.seed + 7919)
    sigma = fraction * float(np.sqrt(np.mean(y ** 2)))
    scn.measurements = (y + rng.normal(0.0, sigma, size=y.shape)).astype(np.float32)
    return scn


@pytest.fixture(scope="module")
def alg():
    from cardiotrust_b200 import algorithm

    return algorithm


def test_cuboid20_full_beat(alg, oracle_mod):
    from cardiotrust_b200 import scenario as sc

    oracle_mod.set_threads(0)
    scn = _noisy(sc.build(sc.workload_spec("cuboid20")), oracle_mod)
    assert scn.num_states == 24000 and scn.num_steps == 2000 and scn.num_sensors == 111
    a = oracle_mod.algo(optimizer=1, learning_rate=1e-3, freeze_delays=0)
    f32 = oracle_mod.from_scenario(scn)
    f32.simulate()
    states = f32.system_states.copy()
    del f32
    ref = oracle_mod.from_scenario(scn, dtype=np.float64)
    ref.run_epoch(a)
    adj = oracle_mod.from_scenario(scn, dtype=np.float64)
    adj.stated_loss(a, gradient=True)
    ctx = alg.Context(0)
    cfg = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    for prec in (alg.Precision.Fp32, alg.Precision.Bf16x6):
        eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=cfg)
        eng.run_epoch(0, precision=prec)
        x = eng.read("system_states")
        assert np.array_equal(x.view(np.uint32), states.view(np.uint32)), prec
        assert rel_err(eng.read("measurements"), ref.measurements) < 1e-5, prec
        assert rel_err(eng.read("grad_gains"), ref.d_gains) < TOL_GRAD, prec
        assert rel_err(eng.read("grad_coefs"), ref.d_coefs) < TOL_GRAD, prec
        assert rel_err(eng.read("loss_batch"), ref.loss_batch) < 1e-4, prec
        eng.close()
        eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=cfg)
        eng.run_epoch(0, grad_mode=alg.GradMode.Adjoint, precision=prec)
        assert rel_err(eng.read("grad_gains"), adj.d_gains) < TOL_GRAD, prec
        assert rel_err(eng.read("grad_coefs"), adj.d_coefs) < TOL_GRAD, prec
        eng.close()
    ctx.close()


def test_shell_adjoint_three_checkpoint_segments(alg, oracle_mod):
    from cardiotrust_b200 import scenario as sc

    oracle_mod.set_threads(0)
    spec = sc.workload_spec("shell")
    spec.num_steps = 600
    spec.pulse_onset = 5
    scn = _noisy(sc.build(spec), oracle_mod)
    assert scn.num_states == 141792 and scn.num_sensors == 111
    a = oracle_mod.algo(optimizer=1, learning_rate=1e-3, freeze_delays=0)
    adj = oracle_mod.from_scenario(scn, dtype=np.float64)
    adj.stated_loss(a, gradient=True)
    ctx = alg.Context(0)
    cfg = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    for prec in (alg.Precision.Fp32, alg.Precision.Bf16x6):
        eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=cfg)
        eng.run_epoch(0, grad_mode=alg.GradMode.Adjoint, precision=prec)
        eg, ec = rel_err(eng.read("grad_gains"), adj.d_gains), rel_err(eng.read("grad_coefs"), adj.d_coefs)
        eng.close()
        assert eg < TOL_GRAD and ec < TOL_GRAD, (prec, eg, ec)
    ctx.close()


def test_shell_geometry_central_differences(alg, oracle_mod):
    from cardiotrust_b200 import scenario as sc

    oracle_mod.set_threads(0)
    spec = sc.workload_spec("shell")
    spec.num_steps = 40
    spec.pulse_onset = 1
    spec.pulse_sigma_samples = 3.0
    scn = _noisy(sc.build(spec), oracle_mod, fraction=0.05)
    a = oracle_mod.algo(freeze_gains=0, freeze_delays=0, maximum_regularization_threshold=0.05,
                        maximum_regularization_strength=0.5)
    e = oracle_mod.from_scenario(scn, dtype=np.float64)
    e.stated_loss(a, gradient=True)
    grads = {"gains": e.d_gains.copy(), "coefs": e.d_coefs.copy()}
    # the GPU adjoint of the same loss (FP32 products)
    ctx = alg.Context(0)
    cfg = alg.Algorithm(freeze_gains=False, freeze_delays=False, maximum_regularization_threshold=0.05,
                        maximum_regularization_strength=0.5)
    eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=cfg)
    eng.run_epoch(0, grad_mode=alg.GradMode.Adjoint, precision=alg.Precision.Fp32)
    gpu = {"gains": eng.read("grad_gains").astype(np.float64), "coefs": eng.read("grad_coefs").astype(np.float64)}
    eng.close()
    ctx.close()
    # 200 random parameters where the short beat's gradient is not zero; gains of rows whose state sits
    # on the |x| kink (exactly 0 while its voxel's regularisation is active) are left out
    T, S = e.system_states.shape
    xs = e.system_states.reshape(T, S // 3, 3)
    active = np.abs(xs).sum(-1) > a.maximum_regularization_threshold
    kink = (xs == 0) & active[:, :, None]
    kink_rows = np.unique(np.nonzero(kink)[1] * 3 + np.nonzero(kink)[2])
    rng = np.random.default_rng(17)
    osi = scn.model.output_state_indices
    ok = (osi >= 0) & (np.abs(grads["gains"]) > 1e-9 * np.abs(grads["gains"]).max())
    ok[kink_rows, :] = False
    gpool = np.flatnonzero(ok.reshape(-1))
    okc = (osi[0::3, 0::3] >= 0) & (np.abs(grads["coefs"]) > 1e-9 * np.abs(grads["coefs"]).max())
    cpool = np.flatnonzero(okc.reshape(-1))
    # the short beat reaches a few hops around the excitation: 200 parameters in all, coefficients
    # as many as have a gradient (at least 40), gains the rest
    assert len(cpool) >= 40 and len(gpool) >= 100, (len(cpool), len(gpool))
    nc = min(100, len(cpool))
    ci = rng.choice(cpool, nc, replace=False)
    gi = rng.choice(gpool, 200 - nc, replace=False)
    params = [("gains", int(i)) for i in gi] + [("coefs", int(i)) for i in ci]
    fd = np.empty(len(params))
    adj = np.empty(len(params))
    gp = np.empty(len(params))
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
        gp[q] = gpu[kind].reshape(-1)[idx]
    for kind in ("gains", "coefs"):
        sel = np.array([p[0] == kind for p in params])
        scale = np.abs(adj[sel]).max()
        assert np.abs(fd[sel] - adj[sel]).max() / scale < 1e-4, kind
        assert np.abs(fd[sel] - gp[sel]).max() / scale < 1e-3, kind
    assert np.linalg.norm(fd - adj) / np.linalg.norm(adj) < 1e-4
    assert np.linalg.norm(fd - gp) / np.linalg.norm(fd) < 1e-3
