"""Host-side mirror of the reference estimation API over the CUDA library.

Reference interface (paths relative to the crate root):

* ``run_epoch(results: &mut Results, batch_index: &mut usize, data: &Data,
  config: &Algorithm) -> anyhow::Result<()>``  — src/core/algorithm.rs:124-129
* ``Algorithm`` (the fields the epoch reads)   — src/core/config/algorithm.rs:25-85
* ``Results { metrics, estimations, derivatives, model }`` — src/core/scenario/results.rs:28-34
* ``Optimizer {Sgd, Adam}``                     — src/core/algorithm/refinement.rs:8-12
* ``APDerivative {Simple, Textbook}``           — src/core/config/algorithm.rs:17-21

Every call goes through ``include/cardiotrust_cuda.h``; errors surface as
:class:`~cardiotrust_b200._lib.CtError` (the counterpart of ``anyhow::Error``).
"""

from __future__ import annotations

import ctypes
import dataclasses
import enum
from types import SimpleNamespace
from typing import Optional

import numpy as np

from . import _lib
from ._lib import CtError, check, fptr, iptr, lib


class Optimizer(enum.IntEnum):
    Sgd = 0
    Adam = 1


class APDerivative(enum.IntEnum):
    Simple = 0
    Textbook = 1


class GradMode(enum.IntEnum):
    Reference = 0  # the reference's per-step derivation (derivation.rs:173-229)
    Adjoint = 1  # exact gradient of the stated loss, back-propagation through time with checkpoints


class Precision(enum.IntEnum):
    Fp32 = 0  # FP32 CUDA-core GEMMs
    Tf32x3 = 1  # tcgen05 TF32 with hi/lo operand split
    Tf32 = 2  # tcgen05 TF32, one pass
    Bf16x6 = 3  # tcgen05 BF16 on error-free 8-bit slices, exact accumulation (unbiased like FP32)


# The product mode of every call that does not name one: the sliced BF16 tensor-core products, whose
# accumulation is exact, are within the gradient target on every configuration measured and closer to
# f64 than the FP32 CUDA-core products (7x smaller H x error on the 768-row shell).
DEFAULT_PRECISION = Precision.Bf16x6


@dataclasses.dataclass
class Algorithm:
    """Algorithm config with the reference defaults (config/algorithm.rs:59-85)."""

    optimizer: Optimizer = Optimizer.Sgd
    epochs: int = 10
    batch_size: int = 0
    snapshots_interval: int = 0
    learning_rate: float = 200.0
    learning_rate_reduction_factor: float = 0.0
    learning_rate_reduction_interval: int = 0
    mse_strength: float = 1.0
    slow_down_stregth: float = 0.0  # read by nothing on the epoch path (update.rs:163-167)
    maximum_regularization_strength: float = 1.0
    maximum_regularization_threshold: float = 1.01
    difference_regularization_strength: float = 0.0
    smoothness_regularization_strength: float = 0.0
    freeze_gains: bool = False
    freeze_delays: bool = True
    ap_derivative: APDerivative = APDerivative.Textbook

    def run_config(self, grad_mode=None, precision=None) -> _lib.CtRunConfig:
        """The epoch-loop settings of run_model_based (scenario.rs:725-795)."""
        c = _lib.CtRunConfig()
        c.epochs = int(self.epochs)
        c.learning_rate_reduction_interval = int(self.learning_rate_reduction_interval)
        c.learning_rate_reduction_factor = float(self.learning_rate_reduction_factor)
        c.grad_mode = int(GradMode.Reference if grad_mode is None else grad_mode)
        c.precision = int(DEFAULT_PRECISION if precision is None else precision)
        c.snapshots_interval = int(self.snapshots_interval)
        return c

    def to_ct(self) -> _lib.CtAlgorithm:
        a = _lib.CtAlgorithm()
        a.optimizer = int(self.optimizer)
        a.ap_derivative = int(self.ap_derivative)
        a.freeze_gains = int(bool(self.freeze_gains))
        a.freeze_delays = int(bool(self.freeze_delays))
        a.batch_size = int(self.batch_size)
        a.learning_rate = float(self.learning_rate)
        a.mse_strength = float(self.mse_strength)
        a.maximum_regularization_strength = float(self.maximum_regularization_strength)
        a.maximum_regularization_threshold = float(self.maximum_regularization_threshold)
        a.difference_regularization_strength = float(self.difference_regularization_strength)
        a.smoothness_regularization_strength = float(self.smoothness_regularization_strength)
        return a


class Context:
    """A device and the stream all work is issued on (GPU::new, gpu.rs:31-64)."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        self._h = ctypes.c_void_p()
        check(lib().ct_ctx_create(int(device), ctypes.c_void_p(stream) if stream else None, ctypes.byref(self._h)))
        self.device = device

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        check(lib().ct_ctx_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def close(self) -> None:
        if self._h:
            lib().ct_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=np.float32)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=np.int32)


class EpochEngine:
    """One scenario's model, estimations, derivatives and metrics in GPU memory."""

    def __init__(
        self,
        ctx: Context,
        *,
        gains,
        output_state_indices,
        coefs,
        delays,
        initial_delays,
        measurement_matrix,
        control_matrix,
        control_function,
        measurements=None,
        num_batch_slots: int = 1,
        algorithm: Optional[Algorithm] = None,
        spatial: Optional["SpatialDescription"] = None,
    ):
        self.ctx = ctx
        self.algorithm = algorithm or Algorithm()
        if measurement_matrix is None:
            # the lead field is computed on the device from the spatial description
            if spatial is None:
                raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, "measurement_matrix or spatial is required")
            H = None
            B, M, S = spatial.num_beats, spatial.num_sensors, _f32(gains).shape[0]
        else:
            H = _f32(measurement_matrix)
            if H.ndim != 3:
                raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, "measurement_matrix must be [beats, sensors, states]")
            B, M, S = H.shape
        u = _f32(control_function)
        keep = dict(
            gains=_f32(gains),
            osi=_i32(output_state_indices),
            coefs=_f32(coefs),
            delays=_i32(delays),
            init=_f32(initial_delays),
            H=H,
            ctrl=_f32(control_matrix),
            u=u,
            meas=None if measurements is None else _f32(measurements),
        )
        V = S // 3
        expect = dict(gains=(S, 78), osi=(S, 78), coefs=(V, 26), delays=(V, 26), init=(V, 26), ctrl=(S,), u=(u.shape[0],))
        for k, shp in expect.items():
            if tuple(keep[k].shape) != shp:
                raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, f"{k} has shape {keep[k].shape}, expected {shp}")
        if keep["meas"] is not None and keep["meas"].shape != (B, u.shape[0], M):
            raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, f"measurements have shape {keep['meas'].shape}")
        d = _lib.CtScenarioDesc()
        d.num_states, d.num_sensors, d.num_steps, d.num_beats = S, M, u.shape[0], B
        d.num_batch_slots = int(num_batch_slots)
        d.gains = fptr(keep["gains"])
        d.output_state_indices = iptr(keep["osi"])
        d.coefs = fptr(keep["coefs"])
        d.delays = iptr(keep["delays"])
        d.initial_delays = fptr(keep["init"])
        d.measurement_matrix = fptr(H) if H is not None else None
        d.control_matrix = fptr(keep["ctrl"])
        d.control_function = fptr(u)
        d.measurements = fptr(keep["meas"]) if keep["meas"] is not None else None
        self._h = ctypes.c_void_p()
        ca = self.algorithm.to_ct()
        check(lib().ct_scenario_create(ctx.handle, ctypes.byref(d), ctypes.byref(ca), ctypes.byref(self._h)))
        self.dims = dict(S=S, V=V, M=M, T=u.shape[0], B=B, NB=int(num_batch_slots))
        if H is None:
            self.set_measurement_matrix(spatial)

    def set_measurement_matrix(self, spatial: "SpatialDescription") -> None:
        """The Biot-Savart measurement matrix computed on the device straight into this scenario
        (``ct_scenario_set_measurement_matrix``): no [B, M, S] host array crosses PCIe."""
        desc, _keep = spatial.to_ct()
        check(lib().ct_scenario_set_measurement_matrix(self._h, ctypes.byref(desc)))

    # -- parameters
    def set_algorithm(self, algorithm: Algorithm) -> None:
        self.algorithm = algorithm
        ca = algorithm.to_ct()
        check(lib().ct_set_algorithm(self._h, ctypes.byref(ca)))

    def set_freeze(self, freeze_gains: bool, freeze_delays: bool) -> None:
        check(lib().ct_set_freeze(self._h, int(freeze_gains), int(freeze_delays)))

    def set_learning_rate(self, lr: float) -> None:
        check(lib().ct_set_learning_rate(self._h, float(lr)))

    # -- work
    def run_epoch(self, batch_index: int = 0, beat_order=None, grad_mode=GradMode.Reference,
                  precision=DEFAULT_PRECISION, sync: bool = True) -> int:
        bi = ctypes.c_int64(int(batch_index))
        order = None if beat_order is None else _i32(beat_order)
        check(lib().ct_run_epoch(self._h, ctypes.byref(bi), None if order is None else iptr(order), int(grad_mode),
                                 int(precision)))
        if sync:
            self.sync()
        return bi.value

    def run_epoch_host(self, batch_index: int, gains: np.ndarray, coefs: np.ndarray, delays: np.ndarray,
                       measurements: Optional[np.ndarray] = None, loss_batch: Optional[np.ndarray] = None,
                       beat_order=None, grad_mode=GradMode.Reference, precision=DEFAULT_PRECISION) -> int:
        """One epoch with the model in host memory, like the reference's ``run_epoch`` updating
        ``results.model`` in place (ct_run_epoch_host): ``gains`` [S,78], ``coefs`` [V,26] and ``delays``
        [V,26] (reference order, C-contiguous; pinned for full speed) are copied in and overwritten with
        the updated parameters; ``measurements`` [B,T,M] (optional) is copied in; ``loss_batch``
        [num_batch_slots] (optional) receives the batch-wise loss. One wait, at the end."""
        D = self.dims
        for name, arr, dtype, shape in (("gains", gains, np.float32, (D["S"], 78)), ("coefs", coefs, np.float32, (D["V"], 26)),
                                        ("delays", delays, np.int32, (D["V"], 26)),
                                        ("measurements", measurements, np.float32, (D["B"], D["T"], D["M"])),
                                        ("loss_batch", loss_batch, np.float32, (D["NB"],))):
            if arr is None and name in ("measurements", "loss_batch"):
                continue
            if arr.shape != shape or arr.dtype != np.dtype(dtype) or not arr.flags.c_contiguous:
                raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, f"{name} needs a C-contiguous {np.dtype(dtype)} array of shape {shape}")
        bi = ctypes.c_int64(int(batch_index))
        order = None if beat_order is None else _i32(beat_order)
        check(lib().ct_run_epoch_host(self._h, ctypes.byref(bi), None if order is None else iptr(order), int(grad_mode),
                                      int(precision), fptr(gains), fptr(coefs), iptr(delays),
                                      None if measurements is None else fptr(measurements),
                                      None if loss_batch is None else fptr(loss_batch)))
        return bi.value

    def run_epoch_plain(self, batch_index: int = 0, beat_order=None, sync: bool = True) -> int:
        """The plain GPU form of :meth:`run_epoch` (reference gradients, FP32): one kernel launch per
        phase per step, one scenario at a time - the baseline the persistent form is measured against."""
        bi = ctypes.c_int64(int(batch_index))
        order = None if beat_order is None else _i32(beat_order)
        check(lib().ct_run_epoch_plain(self._h, ctypes.byref(bi), None if order is None else iptr(order)))
        if sync:
            self.sync()
        return bi.value

    def simulate(self, with_states: bool = False):
        D = self.dims
        y = np.empty((D["B"], D["T"], D["M"]), dtype=np.float32)
        x = np.empty((D["T"], D["S"]), dtype=np.float32) if with_states else None
        check(lib().ct_simulate(self._h, fptr(y), fptr(x) if x is not None else None))
        return (y, x) if with_states else y

    def sync(self) -> None:
        check(lib().ct_sync(self._h))

    def kernel_launches(self) -> int:
        n = ctypes.c_int64()
        check(lib().ct_kernel_launches(self._h, ctypes.byref(n)))
        return n.value

    def set_profiling(self, enable: bool) -> None:
        check(lib().ct_set_profiling(self._h, int(enable)))

    def read_profile(self) -> dict:
        """{phase: (device ms, kernel launches)} accumulated since profiling was enabled."""
        n = len(_lib.PHASES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int64 * n)()
        check(lib().ct_read_profile(self._h, ms, cnt))
        return {p: (ms[i], cnt[i]) for i, p in enumerate(_lib.PHASES)}

    def run_model_based(self, batch_index: int = 0, beat_orders=None, grad_mode=GradMode.Reference,
                        precision=DEFAULT_PRECISION, algorithm: Optional[Algorithm] = None):
        """The reference's epoch loop (scenario.rs:725-795) with this engine's algorithm settings:
        learning-rate schedule, per-epoch summary, snapshots, early stop on a non-normal loss, final
        average delays. Returns (summary dict, [epochs_run, 3] per-epoch losses, batch index)."""
        a = algorithm or self.algorithm
        cfg = a.run_config(grad_mode, precision)
        losses = np.zeros((max(int(a.epochs), 1), 3), dtype=np.float32)
        order = None
        if beat_orders is not None:
            order = _i32(beat_orders)
            if order.shape != (int(a.epochs), self.dims["B"]):
                raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, f"beat_orders must be [{a.epochs}, {self.dims['B']}]")
        bi = ctypes.c_int64(int(batch_index))
        summ = _lib.CtRunSummary()
        check(lib().ct_run_model_based(self._h, ctypes.byref(cfg), None if order is None else iptr(order),
                                       ctypes.byref(bi), fptr(losses), ctypes.byref(summ)))
        out = {f: getattr(summ, f) for f, _ in _lib.CtRunSummary._fields_}
        return out, losses[: summ.epochs_run].copy(), bi.value

    def calculate_plotting_arrays(self, sample_rate_hz: float) -> None:
        """Spherical arrays, their maxima and activation times of the last beat's states
        (scenario.rs:636-690, estimation side); read them as ``system_states_*`` / ``activation_times``."""
        check(lib().ct_calculate_plotting_arrays(self._h, float(sample_rate_hz)))

    def calculate_final(self, ground_truth_types, voxel_numbers) -> "FinalMetrics":
        """metrics::calculate_final (metrics.rs:226-447) on the last beat's states, and the summary at
        the Dice-optimal threshold (scenario.rs:601-617)."""
        t = _i32(ground_truth_types)
        n = _i32(voxel_numbers)
        if t.shape != n.shape or t.ndim != 3:
            raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, "ground truth types and voxel numbers must be the same 3-d grid")
        m = _lib.CtFinalMetrics()
        check(lib().ct_calculate_final(self._h, iptr(t), iptr(n), *t.shape, ctypes.byref(m)))
        return FinalMetrics.from_ct(m)

    def read_snapshots(self, name: str) -> np.ndarray:
        """Snapshots of the last run_model_based call: gains, coefs, delays, system_states or
        measurements, with a leading snapshot axis (Snapshots, results.rs:179-248)."""
        code, dtype, shape = _lib.SNAPSHOT_FIELDS[name]
        D = self.dims
        per = shape(D["S"], D["V"], D["M"], D["T"], D["B"])
        nbytes = ctypes.c_size_t()
        check(lib().ct_field_size(self._h, code, ctypes.byref(nbytes)))
        n = nbytes.value // (int(np.prod(per)) * np.dtype(dtype).itemsize)
        out = np.empty((n, *per), dtype=dtype)
        check(lib().ct_read_field(self._h, code, out.ctypes.data_as(ctypes.c_void_p), out.nbytes))
        return out

    # -- fields
    def read(self, name: str) -> np.ndarray:
        code, dtype, shape = _lib.FIELDS[name]
        D = self.dims
        out = np.empty(shape(D["S"], D["V"], D["M"], D["T"], D["B"], D["NB"]), dtype=dtype)
        check(lib().ct_read_field(self._h, code, out.ctypes.data_as(ctypes.c_void_p), out.nbytes))
        return out

    def read_into(self, name: str, out: np.ndarray) -> np.ndarray:
        """Read a field into a caller-owned C-contiguous array (e.g. pinned host memory)."""
        code, dtype, shape = _lib.FIELDS[name]
        D = self.dims
        want = shape(D["S"], D["V"], D["M"], D["T"], D["B"], D["NB"])
        if out.shape != want or out.dtype != np.dtype(dtype) or not out.flags.c_contiguous:
            raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, f"{name} needs a C-contiguous {dtype} array of shape {want}")
        check(lib().ct_read_field(self._h, code, out.ctypes.data_as(ctypes.c_void_p), out.nbytes))
        return out

    def write(self, name: str, value) -> None:
        code, dtype, shape = _lib.FIELDS[name]
        D = self.dims
        arr = np.ascontiguousarray(np.asarray(value), dtype=dtype)
        want = shape(D["S"], D["V"], D["M"], D["T"], D["B"], D["NB"])
        if arr.shape != want:
            raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, f"{name} has shape {arr.shape}, expected {want}")
        check(lib().ct_write_field(self._h, code, arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes))

    def close(self) -> None:
        if self._h:
            lib().ct_scenario_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @classmethod
    def from_scenario(cls, ctx: Context, scn, *, truth: bool = False, num_batch_slots: int = 1,
                      algorithm: Optional[Algorithm] = None, device_lead_field: bool = False) -> "EpochEngine":
        """An engine for a built scenario; ``device_lead_field`` computes the measurement matrix on the
        device from the scenario's geometry instead of copying ``scn.measurement_matrix``."""
        p = scn.truth if truth else scn.model
        return cls(
            ctx,
            gains=p.gains,
            output_state_indices=p.output_state_indices,
            coefs=p.coefs,
            delays=p.delays,
            initial_delays=p.initial_delays,
            measurement_matrix=None if device_lead_field else scn.measurement_matrix,
            spatial=SpatialDescription.from_scenario(scn, truth=truth) if device_lead_field else None,
            control_matrix=scn.control_matrix,
            control_function=scn.control_function,
            measurements=scn.measurements,
            num_batch_slots=num_batch_slots,
            algorithm=algorithm,
        )


# ------------------------------------------------------------------------------------------
# Model construction on the device


@dataclasses.dataclass
class SpatialDescription:
    """The parts of the reference's ``SpatialDescription`` (src/core/model/spatial.rs) and model
    config that the measurement matrix and the delay arrays are built from."""

    voxel_types: np.ndarray  # [nx,ny,nz] VoxelType discriminants
    voxel_numbers: np.ndarray  # [nx,ny,nz] state index 3v, -1 = None
    voxel_positions_mm: np.ndarray  # [nx,ny,nz,3]
    voxel_size_mm: float
    sensor_positions_mm: np.ndarray  # [M,3]
    sensor_orientations: np.ndarray  # [M,3]
    sensor_array_offsets_mm: np.ndarray  # [B,3]
    sample_rate_hz: float = 2000.0
    propagation_velocities_m_per_s: Optional[np.ndarray] = None  # [10] per VoxelType

    @property
    def num_sensors(self) -> int:
        return int(np.asarray(self.sensor_positions_mm).shape[0])

    @property
    def num_beats(self) -> int:
        return int(np.asarray(self.sensor_array_offsets_mm).reshape(-1, 3).shape[0])

    @property
    def num_voxels(self) -> int:
        t = np.asarray(self.voxel_types)
        return int(((t >= 1) & (t <= 6)).sum())

    def to_ct(self):
        """(CtSpatialDesc, arrays it points into: keep them alive while the struct is used)."""
        keep = dict(
            t=np.ascontiguousarray(self.voxel_types, dtype=np.int32),
            n=np.ascontiguousarray(self.voxel_numbers, dtype=np.int32),
            p=np.ascontiguousarray(self.voxel_positions_mm, dtype=np.float32),
            sp=np.ascontiguousarray(self.sensor_positions_mm, dtype=np.float32),
            so=np.ascontiguousarray(self.sensor_orientations, dtype=np.float32),
            off=np.ascontiguousarray(np.asarray(self.sensor_array_offsets_mm).reshape(-1, 3), dtype=np.float32),
            vel=np.ascontiguousarray(np.zeros(10) if self.propagation_velocities_m_per_s is None
                                     else self.propagation_velocities_m_per_s, dtype=np.float32),
        )
        if keep["t"].ndim != 3 or keep["n"].shape != keep["t"].shape or keep["p"].shape != keep["t"].shape + (3,):
            raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, "voxel grid arrays must be [nx,ny,nz] and [nx,ny,nz,3]")
        if keep["sp"].shape != keep["so"].shape or keep["sp"].ndim != 2 or keep["sp"].shape[1] != 3:
            raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, "sensor arrays must be [M,3]")
        if keep["vel"].shape != (10,):
            raise CtError(_lib.CT_ERR_INVALID_ARGUMENT, "propagation velocities must have 10 entries")
        d = _lib.CtSpatialDesc()
        d.nx, d.ny, d.nz = keep["t"].shape
        d.voxel_types = iptr(keep["t"])
        d.voxel_numbers = iptr(keep["n"])
        d.voxel_positions_mm = fptr(keep["p"])
        d.voxel_size_mm = float(self.voxel_size_mm)
        d.sample_rate_hz = float(self.sample_rate_hz)
        d.propagation_velocities_m_per_s = fptr(keep["vel"])
        d.num_sensors = keep["sp"].shape[0]
        d.num_beats = keep["off"].shape[0]
        d.sensor_positions_mm = fptr(keep["sp"])
        d.sensor_orientations = fptr(keep["so"])
        d.sensor_array_offsets_mm = fptr(keep["off"])
        return d, keep

    @classmethod
    def from_scenario(cls, scn, truth: bool = False) -> "SpatialDescription":
        from . import scenario as sc

        spec = scn.spec
        return cls(
            voxel_types=scn.types_truth if truth else scn.types_model,
            voxel_numbers=scn.numbers,
            voxel_positions_mm=scn.positions_mm,
            voxel_size_mm=spec.voxel_size_mm,
            sensor_positions_mm=scn.sensor_positions_mm,
            sensor_orientations=scn.sensor_orientations,
            sensor_array_offsets_mm=sc.array_offsets_mm(spec),
            sample_rate_hz=spec.sample_rate_hz,
            propagation_velocities_m_per_s=sc.velocities_by_type(spec),
        )


def measurement_matrix(ctx: Context, spatial: SpatialDescription) -> np.ndarray:
    """``MeasurementMatrix::from_model_spatial_description`` (measurement.rs:66-123) on the device:
    H [B, M, S] in reference state order."""
    desc, _keep = spatial.to_ct()
    out = np.empty((spatial.num_beats, spatial.num_sensors, 3 * spatial.num_voxels), np.float32)
    check(lib().ct_measurement_matrix(ctx.handle, ctypes.byref(desc), fptr(out), out.nbytes))
    return out


def delay_samples(ctx: Context, spatial: SpatialDescription):
    """``calculate_delay_samples_array`` (allpass/delay.rs:35-111) with the delays and coefficients of
    ``APParameters::from_model_config`` (allpass.rs:86-100), on the device.
    Returns (initial_delays f32, delays i32, coefs f32), each [V, 26]."""
    desc, _keep = spatial.to_ct()
    V = spatial.num_voxels
    samples = np.empty((V, 26), np.float32)
    delays = np.empty((V, 26), np.int32)
    coefs = np.empty((V, 26), np.float32)
    check(lib().ct_delay_samples(ctx.handle, ctypes.byref(desc), fptr(samples), iptr(delays), fptr(coefs),
                                 samples.size))
    return samples, delays, coefs


def connect_voxels(spatial: SpatialDescription, current_factor_in_pathology: float = 0.0):
    """``connect_voxels`` (allpass.rs:295-494) in the library's native host code: (gains [S, 78],
    activation_time_ms [nx, ny, nz], NaN where never activated)."""
    desc, _keep = spatial.to_ct()
    S = 3 * spatial.num_voxels
    gains = np.empty((S, 78), np.float32)
    act = np.empty(np.asarray(spatial.voxel_types).shape, np.float32)
    check(lib().ct_connect_voxels(ctypes.byref(desc), float(current_factor_in_pathology), fptr(gains), gains.nbytes,
                                  fptr(act)))
    return gains, act


def output_state_indices(spatial: SpatialDescription) -> np.ndarray:
    """``init_output_state_indicies`` (allpass.rs:212-289): [S, 78] i32, -1 = None."""
    desc, _keep = spatial.to_ct()
    out = np.empty((3 * spatial.num_voxels, 78), np.int32)
    check(lib().ct_output_state_indices(ctypes.byref(desc), iptr(out), out.nbytes))
    return out


def ap_parameters(ctx: Context, spatial: SpatialDescription, current_factor_in_pathology: float = 0.0):
    """``APParameters::from_model_config`` (allpass.rs:71-107): gains and activation times from the
    native activation-front search, the index table, and the delay arrays from the device."""
    gains, act = connect_voxels(spatial, current_factor_in_pathology)
    samples, delays, coefs = delay_samples(ctx, spatial)
    return SimpleNamespace(gains=gains, output_state_indices=output_state_indices(spatial), coefs=coefs,
                           delays=delays, initial_delays=samples, activation_time_ms=act)


# ------------------------------------------------------------------------------------------
# Reference-shaped wrappers


@dataclasses.dataclass
class Data:
    """``Data.simulation.measurements`` [beats, steps, sensors] (data.rs:13-15)."""

    measurements: np.ndarray


class EpochBatch:
    """Several :class:`EpochEngine` scenarios of one context run as one schedule per epoch.

    Per beat index, one persistent forward launch and (adjoint mode) one
    persistent adjoint launch cover the tiles of every member; the epoch is
    captured once as a CUDA graph and replayed. Members need batch_size 0;
    their beats run in index order. Destroy the batch before its members.
    """

    def __init__(self, ctx: "Context", engines, grad_mode=GradMode.Reference, precision=DEFAULT_PRECISION):
        self._ctx = ctx
        self._engines = list(engines)
        handles = (ctypes.c_void_p * len(self._engines))(*[e._h.value for e in self._engines])
        h = ctypes.c_void_p()
        check(lib().ct_batch_create(ctx.handle, handles, len(self._engines), int(grad_mode), int(precision),
                                    ctypes.byref(h)))
        self._h = h
        self.batch_indices = np.zeros(len(self._engines), dtype=np.int64)

    def run_epoch(self, sync: bool = True) -> np.ndarray:
        """One epoch of every member; returns the members' batch indices afterwards."""
        check(lib().ct_batch_run_epoch(self._h, self.batch_indices.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        if sync:
            self.sync()
        return self.batch_indices.copy()

    def sync(self) -> None:
        check(lib().ct_batch_sync(self._h))

    def info(self) -> dict:
        k = ctypes.c_int64()
        g, f, a = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().ct_batch_info(self._h, ctypes.byref(k), ctypes.byref(g), ctypes.byref(f), ctypes.byref(a)))
        return {"graph_kernels": int(k.value), "uses_graph": bool(g.value), "forward_ctas": int(f.value),
                "adjoint_ctas": int(a.value)}

    def autotune(self) -> dict:
        """Time candidate schedules on real epochs (they train) and keep the fastest; see ct_batch_autotune."""
        k, o, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(lib().ct_batch_autotune(self._h, self.batch_indices.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                      ctypes.byref(k), ctypes.byref(o), ctypes.byref(ms)))
        return {"ckpt_steps": k.value, "tile_order": o.value, "epoch_ms": ms.value}

    def run_model_based(self, algorithm: Algorithm, grad_mode=GradMode.Reference, precision=DEFAULT_PRECISION):
        """The reference's epoch loop over every member (ct_batch_run_model_based): each member follows
        its own learning rate through ``algorithm``'s schedule and stops on its own non-normal loss.
        ``grad_mode`` / ``precision`` must be the batch's. Returns (per-member summary dicts,
        [members, epochs, 3] losses; rows past a member's last epoch are NaN)."""
        cfg = algorithm.run_config(grad_mode, precision)
        n = len(self._engines)
        losses = np.full((n, max(int(algorithm.epochs), 1), 3), np.nan, dtype=np.float32)
        summ = (_lib.CtRunSummary * n)()
        check(lib().ct_batch_run_model_based(self._h, ctypes.byref(cfg),
                                             self.batch_indices.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                             fptr(losses), summ))
        out = [{f: getattr(summ[i], f) for f, _ in _lib.CtRunSummary._fields_} for i in range(n)]
        return out, losses[:, : int(algorithm.epochs)]

    def set_profiling(self, enable: bool) -> None:
        """Per-phase CUDA-event timing of batched epochs (eager launches while enabled)."""
        check(lib().ct_batch_set_profiling(self._h, int(enable)))

    def read_profile(self) -> dict:
        ms = (ctypes.c_double * len(_lib.PHASES))()
        check(lib().ct_batch_read_profile(self._h, ms))
        return {name: float(ms[i]) for i, name in enumerate(_lib.PHASES)}

    def close(self) -> None:
        if self._h:
            lib().ct_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Results:
    """``Results`` (results.rs:28-34) whose arrays live on the GPU; attribute groups read on access."""

    def __init__(self, engine: EpochEngine):
        self.engine = engine
        self._data_id = None

    def _group(self, names):
        return SimpleNamespace(**{n: self.engine.read(n) for n in names})

    @property
    def metrics(self):
        return self._group(
            ["loss", "loss_mse", "loss_maximum_regularization", "loss_batch", "loss_mse_batch",
             "loss_maximum_regularization_batch"]
        )

    @property
    def estimations(self):
        return self._group(
            ["ap_outputs_now", "ap_outputs_last", "system_states", "measurements", "residuals", "average_delays"]
        )

    @property
    def derivatives(self):
        return self._group(
            ["grad_gains", "grad_coefs", "coefs_fir", "coefs_iir", "mapped_residuals", "maximum_regularization",
             "maximum_regularization_sum", "adam_step"]
        )

    @property
    def ap_params(self):
        return self._group(["gains", "coefs", "delays"])


class BatchIndex:
    """Mutable batch cursor, the ``&mut usize`` of run_epoch."""

    def __init__(self, value: int = 0):
        self.value = int(value)


def run_epoch(results: Results, batch_index: BatchIndex, data: Data, config: Algorithm, beat_order=None) -> None:
    """One estimation epoch (algorithm.rs:124-281) on the GPU.

    ``beat_order`` fixes the beat visiting order; None uses the library's
    seeded shuffle (the reference shuffles with an unseeded generator).
    """
    eng = results.engine
    if results._data_id != id(data):
        eng.write("measurements_actual", data.measurements)
        results._data_id = id(data)
    eng.set_algorithm(config)
    batch_index.value = eng.run_epoch(batch_index.value, beat_order=beat_order)


@dataclasses.dataclass
class FinalMetrics:
    """Metrics::*_over_threshold (metrics.rs:20-37) and the Summary fields at the Dice-optimal threshold."""

    dice_score_over_threshold: np.ndarray
    iou_over_threshold: np.ndarray
    precision_over_threshold: np.ndarray
    recall_over_threshold: np.ndarray
    threshold: float
    dice: float
    iou: float
    recall: float
    precision: float

    @classmethod
    def from_ct(cls, m: _lib.CtFinalMetrics) -> "FinalMetrics":
        arr = lambda f: np.ctypeslib.as_array(getattr(m, f)).astype(np.float32).copy()  # noqa: E731
        return cls(arr("dice_score_over_threshold"), arr("iou_over_threshold"), arr("precision_over_threshold"),
                   arr("recall_over_threshold"), float(m.threshold), float(m.dice), float(m.iou), float(m.recall),
                   float(m.precision))


@dataclasses.dataclass
class Summary:
    """``Summary`` (summary.rs:25-42)."""

    loss: float = 0.0
    loss_mse: float = 0.0
    loss_maximum_regularization: float = 0.0
    dice: float = 0.0
    iou: float = 0.0
    precision: float = 0.0
    recall: float = 0.0
    threshold: float = 0.0


def run_model_based(results: Results, data: Data, config: Algorithm, beat_orders=None,
                    grad_mode=GradMode.Reference, precision=DEFAULT_PRECISION) -> Summary:
    """``run_model_based`` (scenario.rs:725-795) on the GPU: ``config.epochs`` epochs under the
    learning-rate schedule, snapshots every ``config.snapshots_interval`` epochs (read them with
    ``results.engine.read_snapshots``), early stop when the loss is not normal, then the average
    delays of the final parameters. The returned Summary carries the loss fields."""
    eng = results.engine
    if results._data_id != id(data):
        eng.write("measurements_actual", data.measurements)
        results._data_id = id(data)
    eng.set_algorithm(config)
    summ, _, bi = eng.run_model_based(0, beat_orders=beat_orders, grad_mode=grad_mode, precision=precision,
                                      algorithm=config)
    results.batch_index = bi
    results.epochs_run = summ["epochs_run"]
    return Summary(loss=summ["loss"], loss_mse=summ["loss_mse"],
                   loss_maximum_regularization=summ["loss_maximum_regularization"])


def calculate_plotting_arrays(results: Results, sample_rate_hz: float) -> None:
    """Estimation side of ``calculate_plotting_arrays`` (scenario.rs:636-690)."""
    results.engine.calculate_plotting_arrays(sample_rate_hz)


def calculate_final(results: Results, ground_truth_types, voxel_numbers, summary: Optional[Summary] = None):
    """``metrics::calculate_final`` (metrics.rs:226-242) plus the Dice-optimal summary fields
    (scenario.rs:601-617), filled into ``summary`` when given."""
    m = results.engine.calculate_final(ground_truth_types, voxel_numbers)
    if summary is not None:
        summary.threshold, summary.dice, summary.iou = m.threshold, m.dice, m.iou
        summary.recall, summary.precision = m.recall, m.precision
    return m
