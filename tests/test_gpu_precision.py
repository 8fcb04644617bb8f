"""Product precision on the ill-conditioned precision workload: the 64x64x48 ellipsoidal shell
(47,264 voxels, 141,792 states) with 256 triaxial sensors (768 rows) and 1 % measurement noise, so the
residuals are about 1 % of the signal.

Here the gradient is a near-cancelling sum of small residual terms. A product whose error leans one
way (the tensor core's FP32 accumulation loses low bits toward zero) biases it, while unbiased rounding
averages out. The bar is the stated gradient tolerance: every gradient within 1e-3 (norm-wise relative) of the f64
oracle, in both gradient modes, for the FP32 CUDA-core products and the sliced BF16 tensor-core products.
The beat is cut from 8,000 to 1,000 steps so that the f64 oracle (OpenMP) finishes in a few minutes; the
states stay bit-identical to the f32 oracle regardless.
"""

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL_GRAD = 1e-3
TOL_STATES = 1e-4
STEPS = 1000


def _noisy_shell(oracle_mod, steps):
    """The precision workload cut to `steps` steps, truth measurements from the f32 oracle forward plus
    1 % noise."""
    from cardiotrust_b200 import scenario as sc

    oracle_mod.set_threads(0)
    spec = sc.workload_spec("shell_precision")
    spec.num_steps = steps
    scn = sc.build(spec)
    t = scn.truth
    fwd = oracle_mod.OracleEpoch(t.gains, t.output_state_indices, t.coefs, t.delays, t.initial_delays,
                                 scn.measurement_matrix, scn.control_matrix, scn.control_function)
    y = fwd.simulate().astype(np.float64)
    del fwd
    rng = np.random.default_rng(spec.seed + 7919)
    sigma = 0.01 * float(np.sqrt(np.mean(y ** 2)))
    scn.measurements = (y + rng.normal(0.0, sigma, size=y.shape)).astype(np.float32)
    return scn


@pytest.fixture(scope="module")
def shell768(oracle_mod):
    """The precision workload cut to STEPS steps and the f64 oracle's reference-mode epoch and adjoint
    gradient from its initial parameters."""
    scn = _noisy_shell(oracle_mod, STEPS)
    a = oracle_mod.algo(optimizer=1, learning_rate=1e-3, freeze_delays=0)
    ref = oracle_mod.from_scenario(scn, dtype=np.float64)
    ref.run_epoch(a)
    out = {"system_states": ref.system_states.copy(), "measurements": ref.measurements.copy(),
           "grad_gains": ref.d_gains.copy(), "grad_coefs": ref.d_coefs.copy()}
    del ref
    adj = oracle_mod.from_scenario(scn, dtype=np.float64)
    adj.stated_loss(a, gradient=True)
    out["adjoint_grad_gains"] = adj.d_gains.copy()
    out["adjoint_grad_coefs"] = adj.d_coefs.copy()
    del adj
    f32 = oracle_mod.from_scenario(scn)
    f32.simulate()
    out["states_f32"] = f32.system_states.copy()
    return scn, out


@pytest.mark.parametrize("precision", ["Fp32", "Bf16x6", "Tf32x3"])
def test_gradients_meet_bar_on_768_row_shell(shell768, precision):
    """Every product mode the library runs here meets the bar; a TF32 mode may instead be refused by the
    library's guard (its first-beat gradients compared with the sliced products')."""
    from cardiotrust_b200 import algorithm as alg

    scn, ref = shell768
    assert scn.num_sensors == 768 and scn.num_states == 141792
    prec = alg.Precision[precision]
    ctx = alg.Context(0)
    cfg = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=cfg)
    if precision == "Tf32x3":
        from cardiotrust_b200 import _lib

        try:
            eng.run_epoch(0, beat_order=np.arange(scn.num_beats), precision=prec)
        except _lib.CtError as exc:
            assert exc.status == _lib.CT_ERR_NOT_SUPPORTED and "refused" in str(exc)
            eng.close()
            ctx.close()
            return
    else:
        eng.run_epoch(0, beat_order=np.arange(scn.num_beats), precision=prec)
    x = eng.read("system_states")
    assert np.array_equal(x.view(np.uint32), ref["states_f32"].view(np.uint32)), "states differ from the f32 oracle"
    assert rel_err(x, ref["system_states"]) < TOL_STATES
    errs = {"measurements": rel_err(eng.read("measurements"), ref["measurements"]),
            "grad_gains": rel_err(eng.read("grad_gains"), ref["grad_gains"]),
            "grad_coefs": rel_err(eng.read("grad_coefs"), ref["grad_coefs"])}
    eng.close()
    eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=cfg)
    eng.run_epoch(0, beat_order=np.arange(scn.num_beats), grad_mode=alg.GradMode.Adjoint, precision=prec)
    errs["adjoint_grad_gains"] = rel_err(eng.read("grad_gains"), ref["adjoint_grad_gains"])
    errs["adjoint_grad_coefs"] = rel_err(eng.read("grad_coefs"), ref["adjoint_grad_coefs"])
    eng.close()
    ctx.close()
    assert errs["measurements"] < 1e-5, errs
    for k in ("grad_gains", "grad_coefs", "adjoint_grad_gains", "adjoint_grad_coefs"):
        assert errs[k] < TOL_GRAD, (precision, errs)


def test_tf32x3_refused_on_short_768_row_beat(oracle_mod):
    """On a 48-step beat of the same shell the residual-driven gradient is small against the signal, and the
    TF32 split products' biased accumulation puts them ~2e-2 off: the library refuses the mode
    (CT_ERR_NOT_SUPPORTED, parameters and derivatives untouched) instead of returning those gradients."""
    from cardiotrust_b200 import _lib
    from cardiotrust_b200 import algorithm as alg

    scn = _noisy_shell(oracle_mod, 48)
    ctx = alg.Context(0)
    cfg = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-3, freeze_delays=False)
    eng = alg.EpochEngine.from_scenario(ctx, scn, algorithm=cfg)
    g0, c0 = eng.read("gains"), eng.read("coefs")
    for _ in range(2):  # the verdict is kept: the second call refuses without re-checking
        with pytest.raises(_lib.CtError) as exc:
            eng.run_epoch(0, precision=alg.Precision.Tf32x3)
        assert exc.value.status == _lib.CT_ERR_NOT_SUPPORTED
        assert "refused" in str(exc.value)
    assert np.array_equal(eng.read("gains"), g0) and np.array_equal(eng.read("coefs"), c0)
    assert not np.any(eng.read("grad_gains"))
    eng.run_epoch(0, precision=alg.Precision.Bf16x6)  # the sliced products run on the same scenario
    eng.close()
    ctx.close()
