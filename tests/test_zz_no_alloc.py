"""The allocation-free H x entry point against the scenario path's H x.

ct_predict_measurements_noalloc serves callers that must not see this library
allocate device memory (hosts that keep every device buffer in their own pool
or arena, or under a fixed budget, and callers that cannot take the implicit
synchronisation of cudaMalloc / cudaFree). It keeps its split-K partial sums in
a file-scope device array. These tests call it through the C ABI twice in a row
on caller-owned device buffers and compare both results with the predicted
measurements of ct_simulate (the existing entry point) and with an f64 product
of the same operands, within the 1e-5 relative tolerance the other H x checks
use; a second test fills the scratch array to its limit (one split of
num_steps x 128 = 2,097,152 partials) and checks the first size past it is
refused. The file name sorts last so a run that stops at the first failure has
run every other test first.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_MEAS = 1e-5


def _rel(a, b, scale):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / scale)


def test_noalloc_matches_scenario_path_twice():
    import torch

    from cardiotrust_b200 import _lib
    from cardiotrust_b200 import algorithm as alg
    from cardiotrust_b200 import scenario as sc

    spec = sc.ScenarioSpec(shape=(8, 8, 8), num_steps=300, num_beats=1, patho_size=3, patho_origin=(3, 3, 3),
                           pulse_onset=2, pulse_sigma_samples=6.0, seed=21)
    scn = sc.build(spec)
    ctx = alg.Context(0)
    eng = alg.EpochEngine.from_scenario(ctx, scn, truth=True)
    y_ref, x = eng.simulate(with_states=True)  # existing entry point: forward + H x
    eng.close()
    T, S = x.shape
    M = scn.num_sensors
    rng = np.random.default_rng(4)
    z = (y_ref[0] + rng.normal(0.0, 0.01 * float(np.abs(y_ref).max()), size=y_ref[0].shape)).astype(np.float32)

    dev = torch.device("cuda", 0)
    X = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    H = torch.from_numpy(np.ascontiguousarray(scn.measurement_matrix[0])).to(dev)
    Z = torch.from_numpy(z).to(dev)
    Y = torch.empty((T, M), dtype=torch.float32, device=dev)
    R = torch.empty((T, M), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    lib = _lib.lib()
    scale = float(np.linalg.norm(y_ref[0].astype(np.float64)))
    # predict_measurements (prediction.rs:112-130) of the same states in f64
    y64 = x.astype(np.float64) @ scn.measurement_matrix[0].astype(np.float64).T
    for call in range(2):
        Y.fill_(float("nan"))
        R.fill_(float("nan"))
        rc = lib.ct_predict_measurements_noalloc(X.data_ptr(), H.data_ptr(), Z.data_ptr(), Y.data_ptr(),
                                                 R.data_ptr(), T, S, M, ctypes.c_void_p(stream) if stream else None)
        _lib.check(rc)
        torch.cuda.synchronize(dev)
        y = Y.cpu().numpy()
        r = R.cpu().numpy()
        assert np.isfinite(y).all() and np.isfinite(r).all(), call
        assert _rel(y, y_ref[0], scale) < TOL_MEAS, call
        assert _rel(r, y_ref[0] - z, scale) < TOL_MEAS, call
        assert _rel(y, y64, scale) < TOL_MEAS, call

    # beyond the static scratch: a clear error, nothing launched
    rc = lib.ct_predict_measurements_noalloc(X.data_ptr(), H.data_ptr(), None, Y.data_ptr(), None, 40000, S, M, None)
    assert rc == _lib.CT_ERR_INVALID_ARGUMENT
    buf = ctypes.create_string_buffer(512)
    lib.ct_last_error(buf, len(buf))
    assert b"static scratch" in buf.value
    ctx.close()


def test_noalloc_at_scratch_limit():
    """num_steps x ceil64(num_sensors) exactly at the 2,097,152-float scratch (16,384 steps x 128): one
    split-K partial fills the whole array; both calls against an f64 product; 16,385 steps refused."""
    import torch

    from cardiotrust_b200 import _lib

    T, S, M = 16384, 1536, 111
    rng = np.random.default_rng(8)
    x = rng.standard_normal((T, S)).astype(np.float32)
    h = rng.standard_normal((M, S)).astype(np.float32)
    z = rng.standard_normal((T, M)).astype(np.float32)
    y64 = x.astype(np.float64) @ h.astype(np.float64).T
    dev = torch.device("cuda", 0)
    X = torch.from_numpy(x).to(dev)
    H = torch.from_numpy(h).to(dev)
    Z = torch.from_numpy(z).to(dev)
    Y = torch.empty((T, M), dtype=torch.float32, device=dev)
    R = torch.empty((T, M), dtype=torch.float32, device=dev)
    lib = _lib.lib()
    scale = float(np.linalg.norm(y64))
    for call in range(2):
        Y.fill_(float("nan"))
        R.fill_(float("nan"))
        _lib.check(lib.ct_predict_measurements_noalloc(X.data_ptr(), H.data_ptr(), Z.data_ptr(), Y.data_ptr(),
                                                       R.data_ptr(), T, S, M, None))
        torch.cuda.synchronize(dev)
        y = Y.cpu().numpy()
        r = R.cpu().numpy()
        assert np.isfinite(y).all() and np.isfinite(r).all(), call
        assert _rel(y, y64, scale) < TOL_MEAS, call
        assert _rel(r, y64 - z, scale) < TOL_MEAS, call
    rc = lib.ct_predict_measurements_noalloc(X.data_ptr(), H.data_ptr(), None, Y.data_ptr(), None, T + 1, S, M, None)
    assert rc == _lib.CT_ERR_INVALID_ARGUMENT
