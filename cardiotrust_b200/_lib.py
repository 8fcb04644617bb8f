"""ctypes binding of libcardiotrust_cuda.so (declared in include/cardiotrust_cuda.h).

Importing this module loads the in-tree shared library; a missing or stale
build raises ImportError instead of falling back to any CPU path.
"""

from __future__ import annotations

import ctypes
import pathlib

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "libcardiotrust_cuda.so"

CT_OK = 0
CT_ERR_INVALID_ARGUMENT = -1
CT_ERR_CUDA = -2
CT_ERR_OUT_OF_MEMORY = -3
CT_ERR_TIMEOUT = -4
CT_ERR_INVALID_INDEX = -5
CT_ERR_NOT_SUPPORTED = -6
CT_ERR_BATCH_INDEX = -7
CT_ERR_NO_MAXIMUM = -8
CT_THRESHOLDS = 101

CT_OPT_SGD, CT_OPT_ADAM = 0, 1
CT_AP_SIMPLE, CT_AP_TEXTBOOK = 0, 1
CT_GRAD_REFERENCE = 0
CT_PREC_FP32 = 0
CT_PREC_TF32X3 = 1
CT_PREC_TF32 = 2
CT_PREC_BF16X6 = 3

# ct_field values with (dtype, shape-builder(S, V, M, T, B, NB))
FIELDS = {
    "gains": (0, np.float32, lambda S, V, M, T, B, NB: (S, 78)),
    "coefs": (1, np.float32, lambda S, V, M, T, B, NB: (V, 26)),
    "delays": (2, np.int32, lambda S, V, M, T, B, NB: (V, 26)),
    "measurements_actual": (3, np.float32, lambda S, V, M, T, B, NB: (B, T, M)),
    "system_states": (10, np.float32, lambda S, V, M, T, B, NB: (T, S)),
    "measurements": (11, np.float32, lambda S, V, M, T, B, NB: (B, T, M)),
    "residuals": (12, np.float32, lambda S, V, M, T, B, NB: (M,)),
    "ap_outputs_now": (13, np.float32, lambda S, V, M, T, B, NB: (S, 78)),
    "ap_outputs_last": (14, np.float32, lambda S, V, M, T, B, NB: (S, 78)),
    "average_delays": (15, np.float32, lambda S, V, M, T, B, NB: (V,)),
    "grad_gains": (20, np.float32, lambda S, V, M, T, B, NB: (S, 78)),
    "grad_coefs": (21, np.float32, lambda S, V, M, T, B, NB: (V, 26)),
    "coefs_fir": (22, np.float32, lambda S, V, M, T, B, NB: (S, 78)),
    "coefs_iir": (23, np.float32, lambda S, V, M, T, B, NB: (S, 78)),
    "mapped_residuals": (24, np.float32, lambda S, V, M, T, B, NB: (S,)),
    "maximum_regularization": (25, np.float32, lambda S, V, M, T, B, NB: (S,)),
    "maximum_regularization_sum": (26, np.float32, lambda S, V, M, T, B, NB: (1,)),
    "adam_step": (27, np.int64, lambda S, V, M, T, B, NB: (1,)),
    "gains_first_moment": (28, np.float32, lambda S, V, M, T, B, NB: (S, 78)),
    "gains_second_moment": (29, np.float32, lambda S, V, M, T, B, NB: (S, 78)),
    "coefs_first_moment": (30, np.float32, lambda S, V, M, T, B, NB: (V, 26)),
    "coefs_second_moment": (31, np.float32, lambda S, V, M, T, B, NB: (V, 26)),
    "mapped_residuals_history": (32, np.float32, lambda S, V, M, T, B, NB: (T, S)),
    "loss": (40, np.float32, lambda S, V, M, T, B, NB: (T,)),
    "loss_mse": (41, np.float32, lambda S, V, M, T, B, NB: (T,)),
    "loss_maximum_regularization": (42, np.float32, lambda S, V, M, T, B, NB: (T,)),
    "loss_batch": (43, np.float32, lambda S, V, M, T, B, NB: (NB,)),
    "loss_mse_batch": (44, np.float32, lambda S, V, M, T, B, NB: (NB,)),
    "loss_maximum_regularization_batch": (45, np.float32, lambda S, V, M, T, B, NB: (NB,)),
    "system_states_magnitude": (50, np.float32, lambda S, V, M, T, B, NB: (T, V)),
    "system_states_theta": (51, np.float32, lambda S, V, M, T, B, NB: (T, V)),
    "system_states_phi": (52, np.float32, lambda S, V, M, T, B, NB: (T, V)),
    "system_states_magnitude_max": (53, np.float32, lambda S, V, M, T, B, NB: (V,)),
    "system_states_theta_max": (54, np.float32, lambda S, V, M, T, B, NB: (V,)),
    "system_states_phi_max": (55, np.float32, lambda S, V, M, T, B, NB: (V,)),
    "activation_times": (56, np.float32, lambda S, V, M, T, B, NB: (V,)),
}

# Snapshot fields: (ct_field, dtype, per-snapshot shape); the leading snapshot count comes from
# ct_field_size.
SNAPSHOT_FIELDS = {
    "gains": (60, np.float32, lambda S, V, M, T, B: (S, 78)),
    "coefs": (61, np.float32, lambda S, V, M, T, B: (V, 26)),
    "delays": (62, np.int32, lambda S, V, M, T, B: (V, 26)),
    "system_states": (63, np.float32, lambda S, V, M, T, B: (T, S)),
    "measurements": (64, np.float32, lambda S, V, M, T, B: (B, T, M)),
}

EXPORTED = [
    "ct_version",
    "ct_status_string",
    "ct_last_error",
    "ct_ctx_create",
    "ct_ctx_destroy",
    "ct_ctx_stream",
    "ct_scenario_create",
    "ct_scenario_destroy",
    "ct_scenario_dims",
    "ct_run_epoch",
    "ct_run_epoch_plain",
    "ct_run_epoch_host",
    "ct_batch_create",
    "ct_batch_destroy",
    "ct_batch_run_epoch",
    "ct_batch_sync",
    "ct_batch_info",
    "ct_batch_autotune",
    "ct_batch_set_profiling",
    "ct_batch_read_profile",
    "ct_simulate",
    "ct_set_algorithm",
    "ct_set_freeze",
    "ct_set_learning_rate",
    "ct_field_size",
    "ct_read_field",
    "ct_write_field",
    "ct_sync",
    "ct_kernel_launches",
    "ct_set_profiling",
    "ct_read_profile",
    "ct_predict_measurements_noalloc",
    "ct_run_model_based",
    "ct_batch_run_model_based",
    "ct_calculate_plotting_arrays",
    "ct_calculate_final",
    "ct_measurement_matrix",
    "ct_delay_samples",
    "ct_scenario_set_measurement_matrix",
    "ct_connect_voxels",
    "ct_output_state_indices",
]

PHASES = ["forward", "measure", "map_residuals", "derive", "step_metrics", "update"]


class CtAlgorithm(ctypes.Structure):
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


_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int32)


class CtScenarioDesc(ctypes.Structure):
    _fields_ = [
        ("num_states", ctypes.c_int64),
        ("num_sensors", ctypes.c_int64),
        ("num_steps", ctypes.c_int64),
        ("num_beats", ctypes.c_int64),
        ("num_batch_slots", ctypes.c_int64),
        ("gains", _fp),
        ("output_state_indices", _ip),
        ("coefs", _fp),
        ("delays", _ip),
        ("initial_delays", _fp),
        ("measurement_matrix", _fp),
        ("control_matrix", _fp),
        ("control_function", _fp),
        ("measurements", _fp),
    ]


class CtRunConfig(ctypes.Structure):
    _fields_ = [
        ("epochs", ctypes.c_int64),
        ("learning_rate_reduction_interval", ctypes.c_int64),
        ("learning_rate_reduction_factor", ctypes.c_float),
        ("grad_mode", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("snapshots_interval", ctypes.c_int64),
    ]


class CtRunSummary(ctypes.Structure):
    _fields_ = [
        ("epochs_run", ctypes.c_int64),
        ("snapshots", ctypes.c_int64),
        ("loss", ctypes.c_float),
        ("loss_mse", ctypes.c_float),
        ("loss_maximum_regularization", ctypes.c_float),
    ]


class CtFinalMetrics(ctypes.Structure):
    _fields_ = [
        ("dice_score_over_threshold", ctypes.c_float * CT_THRESHOLDS),
        ("iou_over_threshold", ctypes.c_float * CT_THRESHOLDS),
        ("precision_over_threshold", ctypes.c_float * CT_THRESHOLDS),
        ("recall_over_threshold", ctypes.c_float * CT_THRESHOLDS),
        ("threshold", ctypes.c_float),
        ("dice", ctypes.c_float),
        ("iou", ctypes.c_float),
        ("recall", ctypes.c_float),
        ("precision", ctypes.c_float),
    ]


class CtSpatialDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int64),
        ("ny", ctypes.c_int64),
        ("nz", ctypes.c_int64),
        ("voxel_types", _ip),
        ("voxel_numbers", _ip),
        ("voxel_positions_mm", _fp),
        ("voxel_size_mm", ctypes.c_float),
        ("sample_rate_hz", ctypes.c_float),
        ("propagation_velocities_m_per_s", _fp),
        ("num_sensors", ctypes.c_int64),
        ("num_beats", ctypes.c_int64),
        ("sensor_positions_mm", _fp),
        ("sensor_orientations", _fp),
        ("sensor_array_offsets_mm", _fp),
    ]


class CtError(RuntimeError):
    """A non-zero ct_status, with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


def load(path: pathlib.Path = LIB_PATH) -> ctypes.CDLL:
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build it with `python -m cardiotrust_b200.build` (nvcc, sm_100a); "
            "there is no CPU fallback"
        )
    lib = ctypes.CDLL(str(path))
    vp = ctypes.c_void_p
    lib.ct_version.restype = ctypes.c_int
    lib.ct_status_string.restype = ctypes.c_char_p
    lib.ct_status_string.argtypes = [ctypes.c_int]
    lib.ct_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.ct_ctx_create.argtypes = [ctypes.c_int, vp, ctypes.POINTER(vp)]
    lib.ct_ctx_destroy.argtypes = [vp]
    lib.ct_ctx_stream.argtypes = [vp, ctypes.POINTER(vp)]
    lib.ct_scenario_create.argtypes = [vp, ctypes.POINTER(CtScenarioDesc), ctypes.POINTER(CtAlgorithm), ctypes.POINTER(vp)]
    lib.ct_scenario_destroy.argtypes = [vp]
    lib.ct_scenario_dims.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int64)] * 4
    lib.ct_run_epoch.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), _ip, ctypes.c_int, ctypes.c_int]
    lib.ct_run_epoch_plain.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), _ip]
    lib.ct_run_epoch_host.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), _ip, ctypes.c_int, ctypes.c_int, _fp, _fp,
                                      _ip, _fp, _fp]
    lib.ct_batch_create.argtypes = [vp, ctypes.POINTER(vp), ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    lib.ct_batch_destroy.argtypes = [vp]
    lib.ct_batch_run_epoch.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    lib.ct_batch_sync.argtypes = [vp]
    lib.ct_batch_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.ct_batch_set_profiling.argtypes = [vp, ctypes.c_int]
    lib.ct_batch_autotune.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
    lib.ct_batch_read_profile.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    lib.ct_simulate.argtypes = [vp, _fp, _fp]
    lib.ct_set_algorithm.argtypes = [vp, ctypes.POINTER(CtAlgorithm)]
    lib.ct_set_freeze.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.ct_set_learning_rate.argtypes = [vp, ctypes.c_float]
    lib.ct_field_size.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
    lib.ct_read_field.argtypes = [vp, ctypes.c_int, vp, ctypes.c_size_t]
    lib.ct_write_field.argtypes = [vp, ctypes.c_int, vp, ctypes.c_size_t]
    lib.ct_sync.argtypes = [vp]
    lib.ct_kernel_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    lib.ct_set_profiling.argtypes = [vp, ctypes.c_int]
    lib.ct_read_profile.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]
    lib.ct_predict_measurements_noalloc.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int64, ctypes.c_int64,
                                                    ctypes.c_int64, vp]
    lib.ct_run_model_based.argtypes = [vp, ctypes.POINTER(CtRunConfig), _ip, ctypes.POINTER(ctypes.c_int64), _fp,
                                       ctypes.POINTER(CtRunSummary)]
    lib.ct_batch_run_model_based.argtypes = [vp, ctypes.POINTER(CtRunConfig), ctypes.POINTER(ctypes.c_int64), _fp,
                                             ctypes.POINTER(CtRunSummary)]
    lib.ct_calculate_plotting_arrays.argtypes = [vp, ctypes.c_float]
    lib.ct_calculate_final.argtypes = [vp, _ip, _ip, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                       ctypes.POINTER(CtFinalMetrics)]
    lib.ct_measurement_matrix.argtypes = [vp, ctypes.POINTER(CtSpatialDesc), _fp, ctypes.c_size_t]
    lib.ct_delay_samples.argtypes = [vp, ctypes.POINTER(CtSpatialDesc), _fp, _ip, _fp, ctypes.c_int64]
    lib.ct_scenario_set_measurement_matrix.argtypes = [vp, ctypes.POINTER(CtSpatialDesc)]
    lib.ct_connect_voxels.argtypes = [ctypes.POINTER(CtSpatialDesc), ctypes.c_float, _fp, ctypes.c_size_t, _fp]
    lib.ct_output_state_indices.argtypes = [ctypes.POINTER(CtSpatialDesc), _ip, ctypes.c_size_t]
    for name in EXPORTED:
        getattr(lib, name)  # AttributeError if a declared symbol is not exported
    return lib


_LIB = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB


def check(status: int) -> None:
    if status != CT_OK:
        buf = ctypes.create_string_buffer(1024)
        lib().ct_last_error(buf, len(buf))
        raise CtError(status, buf.value.decode(errors="replace") or lib().ct_status_string(status).decode())


def fptr(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)
