"""CPU restatement of the reference estimation epoch — the parity checker.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``; never by the product package.

``oracle.cpp`` follows ``src/core/algorithm.rs:124-281`` and the step
functions it calls (file:line citations inside). :class:`OracleEpoch` owns a
Results-like set of numpy arrays for one scenario and runs epochs on them in
f32 (reference rounding) or f64.
"""

from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
_BUILD = _HERE / "_build"
_LIB_PATH = _BUILD / "liboracle.so"
_lib = None

CXXFLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math", "-std=c++17", "-shared", "-fPIC", "-fopenmp"]


def build(force: bool = False) -> pathlib.Path:
    """Compile oracle.cpp into oracle/_build/liboracle.so (g++)."""
    src = _HERE / "oracle.cpp"
    if force or not _LIB_PATH.exists() or _LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        _BUILD.mkdir(exist_ok=True)
        tmp = _LIB_PATH.with_suffix(f".{os.getpid()}.tmp")
        subprocess.check_call(["g++", *CXXFLAGS, str(src), "-o", str(tmp)])
        os.replace(tmp, _LIB_PATH)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(str(_LIB_PATH))
        _lib.oracle_from_samples_to_coef.restype = ctypes.c_float
        _lib.oracle_from_samples_to_coef.argtypes = [ctypes.c_float]
        _lib.oracle_from_coef_to_samples.restype = ctypes.c_float
        _lib.oracle_from_coef_to_samples.argtypes = [ctypes.c_float]
        _lib.oracle_set_threads.argtypes = [ctypes.c_int]
        _lib.oracle_max_threads.restype = ctypes.c_int
    return _lib


def set_threads(n: int) -> None:
    """Threads of the oracle's parallel loops, process-wide (0 = OpenMP's default, all cores). Only
    loops over independent outputs run in parallel, so every result is bit-identical for any count."""
    lib().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


class Algo(ctypes.Structure):
    """Fields of the reference ``Algorithm`` config the epoch reads (config/algorithm.rs:25-58)."""

    _fields_ = [
        ("optimizer", ctypes.c_int32),
        ("ap_derivative", ctypes.c_int32),
        ("freeze_gains", ctypes.c_int32),
        ("freeze_delays", ctypes.c_int32),
        ("batch_size", ctypes.c_int64),
        ("learning_rate", ctypes.c_float),
        ("mse_strength", ctypes.c_float),
        ("maximum_regularization_strength", ctypes.c_float),
        ("maximum_regularization_threshold", ctypes.c_float),
        ("difference_regularization_strength", ctypes.c_float),
        ("smoothness_regularization_strength", ctypes.c_float),
    ]


_P = ctypes.c_void_p
_EPOCH_FIELDS = [
    ("num_states", ctypes.c_int64),
    ("num_voxels", ctypes.c_int64),
    ("num_sensors", ctypes.c_int64),
    ("num_steps", ctypes.c_int64),
    ("num_beats", ctypes.c_int64),
    ("num_batch_slots", ctypes.c_int64),
] + [
    (name, _P)
    for name in (
        "gains output_state_indices coefs delays initial_delays measurement_matrix control_matrix "
        "control_function_values actual_measurements ap_outputs_now ap_outputs_last system_states measurements "
        "residuals average_delays d_gains d_coefs coefs_iir coefs_fir mapped_residuals maximum_regularization "
        "maximum_regularization_sum step gains_first_moment gains_second_moment coefs_first_moment "
        "coefs_second_moment loss loss_mse loss_maximum_regularization loss_batch loss_mse_batch "
        "loss_maximum_regularization_batch mapped_residuals_override mapped_residuals_history"
    ).split()
]


class _EpochStruct(ctypes.Structure):
    _fields_ = _EPOCH_FIELDS


class OracleEpoch:
    """One scenario's model + Results arrays, run by the CPU restatement.

    ``dtype`` is np.float32 (reference rounding) or np.float64.
    """

    def __init__(
        self,
        gains,
        output_state_indices,
        coefs,
        delays,
        initial_delays,
        measurement_matrix,
        control_matrix,
        control_function,
        actual_measurements=None,
        num_batch_slots: int = 1,
        dtype=np.float32,
        keep_mapped_residuals: bool = False,
    ):
        self.dtype = np.dtype(dtype)
        f = lambda a: np.ascontiguousarray(np.asarray(a), dtype=self.dtype).copy()  # noqa: E731
        i32 = lambda a: np.ascontiguousarray(np.asarray(a), dtype=np.int32).copy()  # noqa: E731
        self.gains = f(gains)
        self.output_state_indices = i32(output_state_indices)
        self.coefs = f(coefs)
        self.delays = i32(delays)
        self.initial_delays = f(initial_delays)
        self.measurement_matrix = f(measurement_matrix)
        self.control_matrix = f(control_matrix)
        self.control_function_values = f(control_function)
        B, M, S = self.measurement_matrix.shape
        T = self.control_function_values.shape[0]
        V = S // 3
        self.num_states, self.num_voxels, self.num_sensors, self.num_steps, self.num_beats = S, V, M, T, B
        if actual_measurements is None:
            actual_measurements = np.zeros((B, T, M))
        self.actual_measurements = f(actual_measurements)
        z = lambda *shape: np.zeros(shape, dtype=self.dtype)  # noqa: E731
        self.ap_outputs_now = z(S, 78)
        self.ap_outputs_last = z(S, 78)
        self.system_states = z(T, S)
        self.measurements = z(B, T, M)
        self.residuals = z(M)
        self.average_delays = np.full(V, np.nan, dtype=self.dtype)
        self.d_gains = z(S, 78)
        self.d_coefs = z(V, 26)
        self.coefs_iir = z(S, 78)
        self.coefs_fir = z(S, 78)
        self.mapped_residuals = z(S)
        self.maximum_regularization = z(S)
        self.maximum_regularization_sum = z(1)
        self.step = np.ones(1, dtype=np.int64)
        self.gains_first_moment = z(S, 78)
        self.gains_second_moment = z(S, 78)
        self.coefs_first_moment = z(V, 26)
        self.coefs_second_moment = z(V, 26)
        self.loss = z(T)
        self.loss_mse = z(T)
        self.loss_maximum_regularization = z(T)
        self.num_batch_slots = int(num_batch_slots)
        self.loss_batch = z(num_batch_slots)
        self.loss_mse_batch = z(num_batch_slots)
        self.loss_maximum_regularization_batch = z(num_batch_slots)
        self.mapped_residuals_override = None
        self.mapped_residuals_history = z(B, T, S) if keep_mapped_residuals else None
        self.batch_index = 0

    def _struct(self) -> _EpochStruct:
        s = _EpochStruct()
        for name, ctype in _EPOCH_FIELDS:
            val = getattr(self, name)
            if ctype is _P:
                setattr(s, name, None if val is None else val.ctypes.data)
            else:
                setattr(s, name, int(val))
        return s

    def run_epoch(self, algo: Algo, beat_order=None, adjoint: bool = False) -> None:
        """One call of ``run_epoch`` (algorithm.rs:124-281).

        ``adjoint=True`` replaces the reference derivation by the exact
        gradient of the stated loss (back-propagation through time); the
        forward, metrics and update are unchanged.
        """
        s = self._struct()
        order = None
        if beat_order is not None:
            order = np.ascontiguousarray(beat_order, dtype=np.int32)
        bi = ctypes.c_int64(self.batch_index)
        kind = "adjoint_" if adjoint else ""
        fn = getattr(lib(), f"oracle_run_epoch_{kind}{'f32' if self.dtype == np.float32 else 'f64'}")
        rc = fn(
            ctypes.byref(s),
            ctypes.byref(algo),
            None if order is None else order.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            ctypes.byref(bi),
        )
        if rc != 0:
            raise RuntimeError(f"oracle run_epoch failed with status {rc}")
        self.batch_index = bi.value

    def stated_loss(self, algo: Algo, gradient: bool = False) -> float:
        """Stated loss summed over beats, sum_t (mse/M)/2 |r|^2 + reg/2 sum_v relu(|x_v|_1 - thr)^2.

        With ``gradient=True`` its exact gradient (plus the reference's
        difference-regularisation term) is left in ``d_gains`` / ``d_coefs``.
        f64 only.
        """
        if self.dtype != np.float64:
            raise TypeError("stated_loss needs a float64 OracleEpoch")
        s = self._struct()
        fn = lib().oracle_adjoint_gradient_f64
        fn.restype = ctypes.c_double
        fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        return float(fn(ctypes.addressof(s), ctypes.addressof(algo), int(gradient)))

    def simulate(self) -> np.ndarray:
        """Forward of every beat (simulation.rs:129-150); returns measurements [B,T,M]."""
        s = self._struct()
        fn = lib().oracle_simulate_f32 if self.dtype == np.float32 else lib().oracle_simulate_f64
        fn(ctypes.byref(s))
        return self.measurements.copy()


    def run_model_based(self, algo: Algo, epochs: int, learning_rate_reduction_interval: int = 0,
                        learning_rate_reduction_factor: float = 0.0, snapshots_interval: int = 0,
                        beat_orders=None, adjoint: bool = False):
        """``run_model_based`` (src/core/scenario.rs:725-795): learning rate 0 in epoch 0, restored in
        epoch 1, multiplied by the factor at every multiple of the interval; the batch losses of the
        last batch after every epoch; a snapshot (results.rs:224-247) at every multiple of the
        snapshot interval; stop when the loss is not a normal number; average delays of the final
        parameters. Returns (summary dict, [epochs_run, 3] losses, snapshots dict of lists)."""
        original = np.float32(algo.learning_rate)
        lr = original
        losses = []
        snaps = {"gains": [], "coefs": [], "delays": [], "system_states": [], "measurements": []}
        summary = dict(epochs_run=0, loss=0.0, loss_mse=0.0, loss_maximum_regularization=0.0)
        for e in range(int(epochs)):
            if e == 0:
                lr = np.float32(0.0)
            elif e == 1:
                lr = original
            if learning_rate_reduction_interval != 0 and e % learning_rate_reduction_interval == 0:
                lr = np.float32(lr * np.float32(learning_rate_reduction_factor))
            algo.learning_rate = float(lr)
            self.run_epoch(algo, beat_order=None if beat_orders is None else beat_orders[e], adjoint=adjoint)
            i = self.batch_index - 1
            row = (self.loss_batch[i], self.loss_mse_batch[i], self.loss_maximum_regularization_batch[i])
            summary.update(epochs_run=e + 1, loss=float(row[0]), loss_mse=float(row[1]),
                           loss_maximum_regularization=float(row[2]))
            losses.append(row)
            if snapshots_interval != 0 and e % snapshots_interval == 0:
                snaps["gains"].append(self.gains.copy())
                snaps["coefs"].append(self.coefs.copy())
                snaps["delays"].append(self.delays.copy())
                snaps["system_states"].append(self.system_states.copy())
                snaps["measurements"].append(self.measurements.copy())
            loss = np.float32(row[0])
            if not (np.isfinite(loss) and abs(loss) >= np.finfo(np.float32).tiny):  # f32::is_normal
                break
        algo.learning_rate = float(original)
        s = self._struct()
        lib().oracle_average_delays_f32(ctypes.byref(s))
        return summary, np.array(losses, dtype=self.dtype).reshape(-1, 3), snaps


def plotting_arrays(system_states: np.ndarray, sample_rate_hz: float):
    """Estimation side of ``calculate_plotting_arrays`` (src/core/scenario.rs:636-690): spherical
    arrays [T,V], their values at each voxel's first magnitude maximum and activation times [V].
    Returns (dict of arrays, status: 0, or -8 when some voxel is NaN at every step)."""
    X = np.ascontiguousarray(system_states, dtype=np.float32)
    T, S = X.shape
    V = S // 3
    out = {k: np.empty((T, V), np.float32) for k in ("magnitude", "theta", "phi")}
    out.update({k: np.empty(V, np.float32) for k in ("magnitude_max", "theta_max", "phi_max", "activation_times")})
    fn = lib().oracle_plotting_arrays_f32
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_float] + [ctypes.c_void_p] * 7
    rc = fn(X.ctypes.data, T, S, float(sample_rate_hz), *[out[k].ctypes.data for k in (
        "magnitude", "theta", "phi", "magnitude_max", "theta_max", "phi_max", "activation_times")])
    return out, int(rc)


def calculate_final(system_states: np.ndarray, ground_truth_types: np.ndarray, voxel_numbers: np.ndarray) -> dict:
    """``metrics::calculate_final`` (src/core/algorithm/metrics.rs:226-447) and the Dice-optimal
    summary (src/core/scenario.rs:601-617), restated literally (one voxel-type prediction per
    threshold)."""
    X = np.ascontiguousarray(system_states, dtype=np.float32)
    gt = np.ascontiguousarray(ground_truth_types, dtype=np.int32)
    nums = np.ascontiguousarray(voxel_numbers, dtype=np.int32)
    out = np.empty(4 * 101 + 5, np.float32)
    fn = lib().oracle_calculate_final_f32
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_int64, ctypes.c_void_p]
    fn(X.ctypes.data, X.shape[0], X.shape[1], gt.ctypes.data, nums.ctypes.data, gt.size, out.ctypes.data)
    keys = ("threshold", "dice", "iou", "recall", "precision")
    res = dict(dice_score_over_threshold=out[0:101], iou_over_threshold=out[101:202],
               precision_over_threshold=out[202:303], recall_over_threshold=out[303:404])
    res.update({k: float(out[404 + i]) for i, k in enumerate(keys)})
    return res


def measurement_matrix(types, numbers, positions_mm, voxel_size_mm, sensor_positions_mm, sensor_orientations,
                       array_offsets_mm, num_states: int) -> np.ndarray:
    """``MeasurementMatrix::from_model_spatial_description`` (src/core/model/functional/measurement.rs:66-123),
    literal f32 loops. Returns H [B, M, S]."""
    t = np.ascontiguousarray(types, dtype=np.int32)
    nums = np.ascontiguousarray(numbers, dtype=np.int32)
    pos = np.ascontiguousarray(positions_mm, dtype=np.float32)
    sp = np.ascontiguousarray(sensor_positions_mm, dtype=np.float32)
    so = np.ascontiguousarray(sensor_orientations, dtype=np.float32)
    off = np.ascontiguousarray(array_offsets_mm, dtype=np.float32).reshape(-1, 3)
    M, B = sp.shape[0], off.shape[0]
    H = np.zeros((B, M, num_states), np.float32)
    fn = lib().oracle_measurement_matrix_f32
    fn.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64] * 3 + [ctypes.c_float] + [ctypes.c_void_p] * 3 + \
        [ctypes.c_int64] * 3 + [ctypes.c_void_p]
    nx, ny, nz = t.shape
    rc = fn(t.ctypes.data, nums.ctypes.data, pos.ctypes.data, nx, ny, nz, float(voxel_size_mm), sp.ctypes.data,
            so.ctypes.data, off.ctypes.data, M, B, num_states, H.ctypes.data)
    if rc:
        raise ValueError("a connectable voxel has no voxel number")
    return H


def connect_voxels(types, numbers, positions_mm, velocities, current_factor_in_pathology: float, num_states: int):
    """``connect_voxels`` / ``try_to_connect`` (src/core/model/functional/allpass.rs:295-494), the literal
    activation-time sweep (small grids: O(activation times x cells)). Returns (gains [S, 78],
    activation_time_ms [nx, ny, nz], NaN where never activated)."""
    t = np.ascontiguousarray(types, dtype=np.int32)
    nums = np.ascontiguousarray(numbers, dtype=np.int32)
    pos = np.ascontiguousarray(positions_mm, dtype=np.float32)
    vel = np.ascontiguousarray(velocities, dtype=np.float32)
    gains = np.zeros((num_states, 78), np.float32)
    act = np.empty(t.shape, np.float32)
    fn = lib().oracle_connect_voxels_f32
    fn.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64] * 3 + [ctypes.c_void_p, ctypes.c_float] + \
        [ctypes.c_void_p] * 2
    nx, ny, nz = t.shape
    if fn(t.ctypes.data, nums.ctypes.data, pos.ctypes.data, nx, ny, nz, vel.ctypes.data,
          float(current_factor_in_pathology), gains.ctypes.data, act.ctypes.data):
        raise ValueError("an activated voxel has no voxel number")
    return gains, act


def delay_samples(types, numbers, positions_mm, velocities, sample_rate_hz: float, num_voxels: int):
    """``calculate_delay_samples_array`` (src/core/model/functional/allpass/delay.rs:35-111) with the
    integer delays and coefficients of ``APParameters::from_model_config`` (allpass.rs:86-100).
    ``velocities``: [10] per VoxelType discriminant. Returns (samples, delays, coefs) [V, 26], or
    raises ValueError naming the first (cell, offset column) whose delay is below one sample."""
    t = np.ascontiguousarray(types, dtype=np.int32)
    nums = np.ascontiguousarray(numbers, dtype=np.int32)
    pos = np.ascontiguousarray(positions_mm, dtype=np.float32)
    vel = np.ascontiguousarray(velocities, dtype=np.float32)
    samples = np.empty((num_voxels, 26), np.float32)
    delays = np.empty((num_voxels, 26), np.int32)
    coefs = np.empty((num_voxels, 26), np.float32)
    fn = lib().oracle_delay_samples_f32
    fn.restype = ctypes.c_int64
    fn.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64] * 3 + [ctypes.c_void_p, ctypes.c_float, ctypes.c_int64] + \
        [ctypes.c_void_p] * 3
    nx, ny, nz = t.shape
    rc = fn(t.ctypes.data, nums.ctypes.data, pos.ctypes.data, nx, ny, nz, vel.ctypes.data, float(sample_rate_hz),
            num_voxels, samples.ctypes.data, delays.ctypes.data, coefs.ctypes.data)
    if rc:
        cell, col = divmod(-rc - 1, 26)
        raise ValueError(f"delay below one sample at cell {cell}, offset column {col}")
    return samples, delays, coefs


def algo(**kw) -> Algo:
    """An Algo with the reference defaults (config/algorithm.rs:59-85), overridden by ``kw``."""
    a = Algo()
    defaults = dict(
        optimizer=0,
        ap_derivative=1,
        freeze_gains=0,
        freeze_delays=1,
        batch_size=0,
        learning_rate=200.0,
        mse_strength=1.0,
        maximum_regularization_strength=1.0,
        maximum_regularization_threshold=1.01,
        difference_regularization_strength=0.0,
        smoothness_regularization_strength=0.0,
    )
    defaults.update(kw)
    for k, v in defaults.items():
        setattr(a, k, v)
    return a


def from_scenario(scn, dtype=np.float32, num_batch_slots: int = 1, truth: bool = False, **kw) -> OracleEpoch:
    """OracleEpoch over a :class:`cardiotrust_b200.scenario.Scenario` (model or truth parameters)."""
    p = scn.truth if truth else scn.model
    return OracleEpoch(
        p.gains,
        p.output_state_indices,
        p.coefs,
        p.delays,
        p.initial_delays,
        scn.measurement_matrix,
        scn.control_matrix,
        scn.control_function,
        scn.measurements,
        num_batch_slots=num_batch_slots,
        dtype=dtype,
        **kw,
    )
