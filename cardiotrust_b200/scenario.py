"""Seeded synthetic scenarios for the estimation epoch.

This module builds every array the epoch consumes, from a small spec:

* the voxel grid (cuboid or ellipsoidal shell), voxel types and the C-order
  state numbering of ``src/core/model/spatial/voxels.rs:407-424``;
* ``output_state_indices`` as in ``src/core/model/functional/allpass.rs:212-289``;
* gains from the activation-front search of ``connect_voxels`` /
  ``try_to_connect`` (``allpass.rs:295-494``), with the gain and direction
  rules of ``allpass/gain.rs:9-29`` and ``allpass/direction.rs:13-22``;
* integer delays, all-pass coefficients and initial delays from a conduction
  velocity (``allpass/delay.rs:14-23,35-111``, ``allpass.rs:71-107,644-668``);
* the Biot-Savart lead field ``H[beat, sensor_row, state]``
  (``src/core/model/functional/measurement.rs:66-123``) for triaxial sensors
  whose rows cycle x, y, z (``src/core/model/spatial/sensors.rs:65-92``);
* a one-hot control matrix on the excitation voxel's x component
  (``src/core/model/functional/control.rs:43-64``) and a Gaussian-derivative
  control pulse.

Ground-truth measurements need a forward pass; :func:`attach_measurements`
takes the forward as a callable so the caller decides which engine runs it
(the CUDA library in the product path).

Index conventions (identical to the reference crate): state ``i = 3*v + a``
for voxel number ``v`` and current component ``a``; gain column
``k = 3*n + b`` for neighbour offset index ``n`` (0..25) and neighbour
component ``b``; coefficient/delay index ``(v, n)``.
"""

from __future__ import annotations

import dataclasses
import math
from typing import Callable, Optional

import numpy as np

# VoxelType discriminants, in the order of src/core/model/spatial/voxels.rs:664-676.
VT_NONE, VT_SINOATRIAL, VT_ATRIUM, VT_AV, VT_HPS, VT_VENTRICLE, VT_PATHOLOGICAL = 0, 1, 2, 3, 4, 5, 6
VT_VESSEL, VT_TORSO, VT_CHAMBER = 7, 8, 9

_CONNECTABLE = {VT_SINOATRIAL, VT_ATRIUM, VT_AV, VT_HPS, VT_VENTRICLE, VT_PATHOLOGICAL}

# is_connection_allowed(output, input), voxels.rs:707-742
_ALLOWED_INPUTS = {
    VT_SINOATRIAL: {VT_ATRIUM, VT_PATHOLOGICAL, VT_VENTRICLE},
    VT_ATRIUM: {VT_SINOATRIAL, VT_ATRIUM, VT_AV, VT_PATHOLOGICAL},
    VT_AV: {VT_ATRIUM, VT_HPS, VT_PATHOLOGICAL},
    VT_HPS: {VT_HPS, VT_AV, VT_VENTRICLE, VT_PATHOLOGICAL},
    VT_VENTRICLE: {VT_VENTRICLE, VT_HPS, VT_PATHOLOGICAL},
}

F32_EPS = np.float32(np.finfo(np.float32).eps)
# physical_constants::VACUUM_MAG_PERMEABILITY (CODATA 2018), cast to f32 as in measurement.rs:88
MU0 = np.float32(1.25663706212e-6)


def offset_to_gain_index(x: int, y: int, z: int, out_dim: int) -> Optional[int]:
    """Gain column for a neighbour offset and output component (allpass.rs:532-548)."""
    if x == 0 and y == 0 and z == 0:
        return None
    idx = out_dim + (z + 1) * 3 + (y + 1) * 9 + (x + 1) * 27
    if idx > 27 + 9 + 3:
        idx -= 3
    return idx


def gain_index_to_offset(k: int) -> Optional[tuple]:
    """Inverse of :func:`offset_to_gain_index` (allpass.rs:553-573)."""
    if k > 77:
        return None
    c = k + 3 if k >= 27 + 9 + 3 else k
    return (c // 27 % 3 - 1, c // 9 % 3 - 1, c // 3 % 3 - 1, c % 3)


def offset_to_delay_index(x: int, y: int, z: int) -> Optional[int]:
    """Coefficient/delay column for a neighbour offset (allpass.rs:578-588)."""
    if x == 0 and y == 0 and z == 0:
        return None
    idx = (z + 1) + (y + 1) * 3 + (x + 1) * 9
    if idx > 9 + 3 + 1:
        idx -= 1
    return idx


def delay_index_to_offset(n: int) -> Optional[tuple]:
    """Inverse of :func:`offset_to_delay_index` (allpass.rs:597-611)."""
    if n > 26:
        return None
    c = n + 1 if n > 9 + 3 else n
    return (c // 9 % 3 - 1, c // 3 % 3 - 1, c % 3 - 1)


def from_samples_to_coef(samples) -> np.float32:
    """Fractional delay -> all-pass coefficient, clamped (allpass.rs:640-646)."""
    s = np.float32(samples)
    frac = np.float32(math.fmod(float(s), 1.0))
    coef = np.float32((np.float32(1.0) - frac) / (np.float32(1.0) + frac))
    return np.float32(min(max(coef, np.float32(1e-4)), np.float32(1.0) - np.float32(1e-4)))


def from_coef_to_samples(coef) -> np.float32:
    """All-pass coefficient -> fractional delay in samples (allpass.rs:661-665)."""
    c = np.float32(coef)
    return np.float32((np.float32(1.0) - c) / (c + np.float32(1.0)))


# ---------------------------------------------------------------------------------------------
# spec


@dataclasses.dataclass
class ScenarioSpec:
    """What to build; the named workloads are in :func:`workload_spec`."""

    shape: tuple = (8, 8, 8)
    mask: str = "cuboid"  # "cuboid" | "shell"
    shell_semi_axes: tuple = (30.0, 25.0, 22.0)
    shell_thickness: float = 8.0
    voxel_size_mm: float = 2.5
    velocity_m_per_s: float = 0.6
    sample_rate_hz: float = 2000.0
    num_steps: int = 500
    num_beats: int = 1
    num_sensors: int = 37  # triaxial sensors -> 3 rows each
    sensor_spacing_mm: float = 20.0
    sensor_height_mm: float = 100.0
    beat_shift_mm: float = 10.0
    patho_size: int = 3
    patho_origin: Optional[tuple] = None  # None -> seeded random placement
    excitation: str = "corner"  # "corner" | "random"
    pulse_sigma_samples: float = 10.0
    pulse_onset: Optional[int] = None  # None -> seeded
    noise_fraction: float = 0.0
    seed: int = 0


@dataclasses.dataclass
class APParams:
    gains: np.ndarray  # [S,78] f32
    output_state_indices: np.ndarray  # [S,78] i32, -1 = None
    coefs: np.ndarray  # [V,26] f32
    delays: np.ndarray  # [V,26] i32
    initial_delays: np.ndarray  # [V,26] f32
    activation_time_ms: np.ndarray  # [nx,ny,nz] f32, NaN = never activated


@dataclasses.dataclass
class Scenario:
    spec: ScenarioSpec
    types_truth: np.ndarray
    types_model: np.ndarray
    numbers: np.ndarray  # [nx,ny,nz] i32, -1 = None
    positions_mm: np.ndarray  # [nx,ny,nz,3] f32
    truth: APParams
    model: APParams
    measurement_matrix: np.ndarray  # [B,M,S] f32
    control_matrix: np.ndarray  # [S] f32
    control_function: np.ndarray  # [T] f32
    sensor_positions_mm: np.ndarray
    sensor_orientations: np.ndarray
    measurements: Optional[np.ndarray] = None  # [B,T,M] f32 (ground truth + noise)

    @property
    def num_voxels(self) -> int:
        return int(self.model.coefs.shape[0])

    @property
    def num_states(self) -> int:
        return 3 * self.num_voxels

    @property
    def num_sensors(self) -> int:
        return int(self.measurement_matrix.shape[1])

    @property
    def num_steps(self) -> int:
        return int(self.control_function.shape[0])

    @property
    def num_beats(self) -> int:
        return int(self.measurement_matrix.shape[0])


# ---------------------------------------------------------------------------------------------
# geometry


def _mask(spec: ScenarioSpec) -> np.ndarray:
    nx, ny, nz = spec.shape
    if spec.mask == "cuboid":
        return np.ones((nx, ny, nz), dtype=bool)
    if spec.mask == "shell":
        a, b, c = spec.shell_semi_axes
        th = spec.shell_thickness
        x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        cx, cy, cz = (nx - 1) / 2.0, (ny - 1) / 2.0, (nz - 1) / 2.0
        r_out = ((x - cx) / a) ** 2 + ((y - cy) / b) ** 2 + ((z - cz) / c) ** 2
        r_in = ((x - cx) / (a - th)) ** 2 + ((y - cy) / (b - th)) ** 2 + ((z - cz) / (c - th)) ** 2
        return (r_out <= 1.0) & (r_in > 1.0)
    raise ValueError(f"unknown mask {spec.mask!r}")


def voxel_count(spec: ScenarioSpec) -> int:
    """Voxels of the scenario a spec builds (the mask's cells), without building it."""
    return int(_mask(spec).sum())


def _positions(shape, size_mm: float) -> np.ndarray:
    """Voxel centres: size*idx + size/2 (voxels.rs:499-527, zero heart offset)."""
    nx, ny, nz = shape
    size = np.float32(size_mm)
    half = np.float32(size_mm / 2.0)
    pos = np.zeros((nx, ny, nz, 3), dtype=np.float32)
    for d, n in enumerate((nx, ny, nz)):
        idx = np.arange(n, dtype=np.float32)
        vals = (size.astype(np.float64) * idx + half).astype(np.float32)  # fma of exact small values
        sl = [None, None, None]
        sl[d] = slice(None)
        pos[..., d] = vals[tuple(sl)]
    return pos


def _numbers(types: np.ndarray) -> np.ndarray:
    """C-order numbering of connectable voxels in steps of 3 (voxels.rs:407-424)."""
    conn = np.isin(types, list(_CONNECTABLE))
    nums = np.full(types.shape, -1, dtype=np.int64)
    flat = conn.ravel()
    nums.ravel()[flat] = np.arange(int(flat.sum()), dtype=np.int64) * 3
    return nums.astype(np.int32)


def _delay_s(p_in: np.ndarray, p_out: np.ndarray, velocity: float) -> np.float32:
    """delay.rs:14-23: |p_in - p_out| / v with the distance in metres, in f32."""
    d = ((p_in - p_out) / np.float32(1000.0)).astype(np.float32)
    sq = np.float32(0.0)
    for comp in d:
        sq = np.float32(sq + np.float32(comp * comp))
    return np.float32(np.float32(np.sqrt(sq)) / np.float32(velocity))


def _direction(p_in: np.ndarray, p_out: np.ndarray) -> np.ndarray:
    """direction.rs:13-22: (p_in - p_out) / L1 norm."""
    d = ((p_in - p_out) / np.float32(1000.0)).astype(np.float32)
    norm = np.float32(0.0)
    for comp in d:
        norm = np.float32(norm + np.float32(abs(comp)))
    return (d / norm).astype(np.float32)


def _gain(dir_in: np.ndarray, dir_out: np.ndarray) -> np.ndarray:
    """gain.rs:9-29: g[i, o] = dir_in[i] * sign(dir_out[o]) (0 where dir_out[o] ~ 0)."""
    g = np.zeros((3, 3), dtype=np.float32)
    for i in range(3):
        for o in range(3):
            c = dir_out[o]
            mult = np.float32(0.0) if abs(c) <= F32_EPS else np.float32(math.copysign(1.0, c))
            g[i, o] = np.float32(dir_in[i] * mult)
    return g


def _relative_eq(a: np.ndarray, b: float) -> np.ndarray:
    """approx::relative_eq! with default epsilon and max_relative = f32::EPSILON."""
    diff = np.abs(a - np.float32(b))
    largest = np.maximum(np.abs(a), np.float32(abs(b)))
    return (diff <= F32_EPS) | (diff <= largest * F32_EPS)


def _neighbour_table(numbers: np.ndarray) -> np.ndarray:
    """Neighbour voxel number per (voxel, offset index), -1 where absent; offsets as in delay.rs:54-73."""
    nx, ny, nz = numbers.shape
    conn = numbers >= 0
    V = int(conn.sum())
    coords = np.argwhere(conn)  # C-order == numbering order
    nbr = np.full((V, 26), -1, dtype=np.int32)
    for ox in (-1, 0, 1):
        for oy in (-1, 0, 1):
            for oz in (-1, 0, 1):
                if ox == 0 and oy == 0 and oz == 0:
                    continue
                n = offset_to_delay_index(ox, oy, oz)
                X, Y, Z = coords[:, 0] + ox, coords[:, 1] + oy, coords[:, 2] + oz
                inb = (X >= 0) & (X < nx) & (Y >= 0) & (Y < ny) & (Z >= 0) & (Z < nz)
                num = np.full(V, -1, dtype=np.int64)
                num[inb] = numbers[X[inb], Y[inb], Z[inb]]
                nbr[:, n] = np.where(num >= 0, num // 3, -1)
    return nbr


def _output_state_indices(types: np.ndarray, numbers: np.ndarray) -> np.ndarray:
    """init_output_state_indicies (allpass.rs:212-289): out[3v+a, 3n+b] = 3*nbr(v,n) + b."""
    nbr = _neighbour_table(numbers)
    V = nbr.shape[0]
    out = np.full((V, 26, 3), -1, dtype=np.int64)
    for b in range(3):
        out[:, :, b] = np.where(nbr >= 0, 3 * nbr.astype(np.int64) + b, -1)
    out = out.reshape(V, 78)
    return np.repeat(out, 3, axis=0).astype(np.int32)


def _delay_samples(types, numbers, positions, velocity, sample_rate) -> np.ndarray:
    """calculate_delay_samples_array (delay.rs:35-111) for a uniform velocity.

    Every neighbour pair with the same offset has the same distance on a
    regular grid (positions are exact multiples of the voxel size), so the
    delay is evaluated once per offset, on the first voxel that has that
    neighbour, with the f32 arithmetic of delay.rs:14-23.
    """
    nbr = _neighbour_table(numbers)
    V = nbr.shape[0]
    out = np.zeros((V, 26), dtype=np.float32)
    coords = np.argwhere(numbers >= 0)  # numbering order
    for n in range(26):
        has = nbr[:, n] >= 0
        if not has.any():
            continue
        v = int(np.argmax(has))
        ox, oy, oz = delay_index_to_offset(n)
        x, y, z = coords[v]
        samples = np.float32(_delay_s(positions[x, y, z], positions[x + ox, y + oy, z + oz], velocity)
                             * np.float32(sample_rate))
        if samples < 1.0:
            raise ValueError(f"delay below one sample: {samples}")
        out[has, n] = samples
    return out


def _connect_voxels(types, numbers, positions, velocity, current_factor_in_pathology):
    """Activation-front search of connect_voxels / try_to_connect (allpass.rs:295-494).

    The reference visits activation times in increasing order; at each time
    ``current`` it takes a snapshot of the activated voxels whose time is
    relative_eq to ``current`` and lets each of them, in C order, activate
    its not yet activated neighbours (first come, first served). Here the
    activated-but-unvisited voxels sit in a heap keyed by time, so each
    snapshot is popped instead of found by a scan of the whole grid; a
    voxel activated while a snapshot is processed waits for a later one, as
    in the reference. Distances, directions and gains depend only on the
    position difference of the pair and the output voxel's direction, and
    are cached on those keys.

    Returns (gains [S,78], activation_time_ms [nx,ny,nz]).
    """
    import heapq

    nx, ny, nz = types.shape
    S = int((numbers >= 0).sum()) * 3
    gains = np.zeros((S, 78), dtype=np.float32)
    act = np.full(types.shape, np.nan, dtype=np.float32)
    dirs = np.zeros(types.shape + (3,), dtype=np.float32)
    patho_zero = abs(current_factor_in_pathology) <= F32_EPS or abs(current_factor_in_pathology) == 0.0
    types_l = types.tolist()
    numbers_l = numbers.tolist()
    heap = []  # (time, C-order index) of activated voxels not visited yet
    for idx in np.argwhere(types == VT_SINOATRIAL):
        act[tuple(idx)] = np.float32(0.0)
        dirs[tuple(idx)] = np.array([1.0, 0.0, 0.0], dtype=np.float32)
        heapq.heappush(heap, (0.0, int(np.ravel_multi_index(tuple(idx), types.shape))))
    pair_cache = {}
    gain_cache = {}
    offsets = [(ox, oy, oz) for ox in (-1, 0, 1) for oy in (-1, 0, 1) for oz in (-1, 0, 1) if (ox, oy, oz) != (0, 0, 0)]
    col = {(ox, oy, oz): offset_to_gain_index(ox, oy, oz, 0) for (ox, oy, oz) in offsets}
    f_in = np.float32(current_factor_in_pathology)
    f_out = np.float32(np.float32(1.0) / np.float32(current_factor_in_pathology)) if not patho_zero else None
    while heap:
        current = np.float32(heap[0][0])
        tol = max(float(F32_EPS), abs(float(current)) * float(F32_EPS))
        snap = []
        while heap and (heap[0][0] - float(current)) <= tol:
            snap.append(heapq.heappop(heap)[1])
        snap.sort()  # C order, as indexed_iter
        for flat in snap:
            xo, yo, zo = np.unravel_index(flat, types.shape)
            xo, yo, zo = int(xo), int(yo), int(zo)
            t_out = act[xo, yo, zo]
            type_out = types_l[xo][yo][zo]
            if type_out not in _CONNECTABLE:
                continue
            dir_out = dirs[xo, yo, zo]
            dir_key = dir_out.tobytes()
            for ox, oy, oz in offsets:
                xi, yi, zi = xo - ox, yo - oy, zo - oz
                if not (0 <= xi < nx and 0 <= yi < ny and 0 <= zi < nz):
                    continue
                type_in = types_l[xi][yi][zi]
                if type_in not in _CONNECTABLE:
                    continue
                if not np.isnan(act[xi, yi, zi]):
                    continue
                if type_in not in _ALLOWED_INPUTS.get(type_out, set()) and type_out != VT_PATHOLOGICAL:
                    continue
                if type_in == VT_PATHOLOGICAL and patho_zero:
                    continue
                p_in = positions[xi, yi, zi]
                p_out = positions[xo, yo, zo]
                dkey = (p_in - p_out).tobytes()
                pr = pair_cache.get(dkey)
                if pr is None:
                    pr = (_delay_s(p_in, p_out, velocity), _direction(p_in, p_out))
                    pair_cache[dkey] = pr
                ds, direction = pr
                t_in = np.float32(t_out + ds)
                act[xi, yi, zi] = t_in
                dirs[xi, yi, zi] = direction
                gkey = (dkey, dir_key)
                g = gain_cache.get(gkey)
                if g is None:
                    g = _gain(direction, dir_out)
                    gain_cache[gkey] = g
                if type_in == VT_PATHOLOGICAL and type_out != VT_PATHOLOGICAL:
                    g = (g * f_in).astype(np.float32)
                if type_out == VT_PATHOLOGICAL and type_in != VT_PATHOLOGICAL:
                    g = (g * f_out).astype(np.float32)
                base = numbers_l[xi][yi][zi]
                c0 = col[(ox, oy, oz)]
                gains[base:base + 3, c0:c0 + 3] = g
                heapq.heappush(heap, (float(t_in), (xi * ny + yi) * nz + zi))
    return gains, (act * np.float32(1000.0)).astype(np.float32)


def _ap_params(types, numbers, positions, spec: ScenarioSpec, current_factor) -> APParams:
    """APParameters::from_model_config (allpass.rs:71-107)."""
    gains, act_ms = _connect_voxels(types, numbers, positions, spec.velocity_m_per_s, current_factor)
    samples = _delay_samples(types, numbers, positions, spec.velocity_m_per_s, spec.sample_rate_hz)
    delays = samples.astype(np.int64).astype(np.int32)  # from_samples_to_usize truncates
    frac = np.fmod(samples.astype(np.float32), np.float32(1.0))
    coefs = ((np.float32(1.0) - frac) / (np.float32(1.0) + frac)).astype(np.float32)
    coefs = np.clip(coefs, np.float32(1e-4), np.float32(1.0) - np.float32(1e-4)).astype(np.float32)
    osi = _output_state_indices(types, numbers)
    return APParams(
        gains=gains,
        output_state_indices=osi,
        coefs=coefs.reshape(samples.shape),
        delays=delays,
        initial_delays=samples,
        activation_time_ms=act_ms,
    )


def _sensors(spec: ScenarioSpec, positions: np.ndarray, mask: np.ndarray):
    """Planar hexagonal grid of triaxial sensors above the volume; rows cycle x, y, z."""
    pts = []
    ring = 0
    while len(pts) < spec.num_sensors:
        if ring == 0:
            pts.append((0.0, 0.0))
        else:
            # hex ring of radius `ring`, 6*ring points
            corners = [(math.cos(math.pi / 3 * c), math.sin(math.pi / 3 * c)) for c in range(7)]
            for side in range(6):
                (ax, ay), (bx, by) = corners[side], corners[side + 1]
                for j in range(ring):
                    f = j / ring
                    pts.append((ring * (ax + (bx - ax) * f), ring * (ay + (by - ay) * f)))
        ring += 1
    pts = pts[: spec.num_sensors]
    occupied = positions[mask]
    centre = occupied.mean(axis=0)
    top = occupied[:, 2].max()
    sp = []
    ori = []
    for px, py in pts:
        for d in range(3):
            sp.append(
                (centre[0] + px * spec.sensor_spacing_mm, centre[1] + py * spec.sensor_spacing_mm, top + spec.sensor_height_mm)
            )
            o = [0.0, 0.0, 0.0]
            o[d] = 1.0
            ori.append(o)
    return np.asarray(sp, dtype=np.float32), np.asarray(ori, dtype=np.float32)


def array_offsets_mm(spec: ScenarioSpec) -> np.ndarray:
    """Sensor-array offset of every beat [B, 3] (sensors.array_offsets_mm): beat b moves the array by
    b x beat_shift_mm along x."""
    off = np.zeros((spec.num_beats, 3), dtype=np.float32)
    off[:, 0] = np.arange(spec.num_beats, dtype=np.float32) * np.float32(spec.beat_shift_mm)
    return off


def velocities_by_type(spec: ScenarioSpec) -> np.ndarray:
    """Propagation velocity per VoxelType discriminant [10] (PropagationVelocitiesMPerS::get,
    config/model.rs:138-150): the spec's uniform velocity for the connectable types, 0 otherwise."""
    vel = np.zeros(10, dtype=np.float32)
    vel[VT_SINOATRIAL:VT_PATHOLOGICAL + 1] = np.float32(spec.velocity_m_per_s)
    return vel


def _measurement_matrix(spec, types, numbers, positions, s_pos, s_ori) -> np.ndarray:
    """Biot-Savart lead field per beat (measurement.rs:66-123), vectorised over voxels in f32."""
    conn = numbers >= 0
    vpos = positions[conn].astype(np.float32)  # C-order == numbering order
    vnum = numbers[conn].astype(np.int64)
    S = int(conn.sum()) * 3
    M = s_pos.shape[0]
    B = spec.num_beats
    size_m = np.float32(spec.voxel_size_mm / 1000.0)
    vol = np.float32(size_m * np.float32(size_m * size_m))
    cf = np.float32(np.float32(np.float32(MU0 * vol) / np.float32(4.0 * np.float32(math.pi))) * np.float32(1e12))
    H = np.zeros((B, M, S), dtype=np.float32)
    for beat in range(B):
        offset = array_offsets_mm(spec)[beat]
        for m in range(M):
            spos = (s_pos[m] + offset).astype(np.float32)
            o = s_ori[m]
            d = ((spos[None, :] - vpos) / np.float32(1000.0)).astype(np.float32)
            sq = ((d[:, 0] * d[:, 0]).astype(np.float32) + (d[:, 1] * d[:, 1]).astype(np.float32)).astype(np.float32)
            sq = (sq + (d[:, 2] * d[:, 2]).astype(np.float32)).astype(np.float32)
            r = np.sqrt(sq).astype(np.float32)
            r3 = (r * (r * r)).astype(np.float32)
            c0 = (np.float64(o[2]) * d[:, 1] - np.float64(o[1]) * d[:, 2]).astype(np.float32)
            c1 = (np.float64(o[0]) * d[:, 2] - np.float64(o[2]) * d[:, 0]).astype(np.float32)
            c2 = (np.float64(o[1]) * d[:, 0] - np.float64(o[0]) * d[:, 1]).astype(np.float32)
            H[beat, m, vnum + 0] = ((cf * c0).astype(np.float32) / r3).astype(np.float32)
            H[beat, m, vnum + 1] = ((cf * c1).astype(np.float32) / r3).astype(np.float32)
            H[beat, m, vnum + 2] = ((cf * c2).astype(np.float32) / r3).astype(np.float32)
    return H


def _pulse(num_steps: int, sigma: float, onset: int) -> np.ndarray:
    """Gaussian-derivative pulse with unit peak: -x exp((1 - x^2)/2), x = (t - t0)/sigma."""
    t = np.arange(num_steps, dtype=np.float64)
    t0 = onset + 3.0 * sigma
    x = (t - t0) / sigma
    u = -x * np.exp((1.0 - x * x) / 2.0)
    return u.astype(np.float32)


def build(spec: ScenarioSpec, ctx=None) -> Scenario:
    """Build a scenario (everything except the ground-truth measurements).

    With ``ctx`` (an ``algorithm.Context``) the model arrays come from the library: the
    activation-front gain search and the index table in its native host code, the delay arrays and
    the measurement matrix on the device (bit-identical to the numpy restatement used otherwise)."""
    rng = np.random.default_rng(spec.seed)
    mask = _mask(spec)
    nx, ny, nz = spec.shape
    occ = np.argwhere(mask)
    if occ.size == 0:
        raise ValueError("empty voxel mask")
    if spec.excitation == "corner":
        exc = tuple(int(c) for c in occ[0])
    else:
        exc = tuple(int(c) for c in occ[rng.integers(len(occ))])

    types_model = np.where(mask, VT_VENTRICLE, VT_NONE).astype(np.uint8)
    types_model[exc] = VT_SINOATRIAL
    types_truth = types_model.copy()
    if spec.patho_size > 0:
        ps = spec.patho_size
        if spec.patho_origin is not None:
            origin = spec.patho_origin
        else:
            # random block whose voxels are all in the mask and away from the excitation voxel
            for _ in range(1000):
                origin = tuple(int(rng.integers(0, max(1, n - ps + 1))) for n in (nx, ny, nz))
                blk = mask[origin[0] : origin[0] + ps, origin[1] : origin[1] + ps, origin[2] : origin[2] + ps]
                far = max(abs(origin[d] + ps // 2 - exc[d]) for d in range(3)) > ps
                if blk.size == ps**3 and blk.any() and far:
                    break
        blk = types_truth[origin[0] : origin[0] + ps, origin[1] : origin[1] + ps, origin[2] : origin[2] + ps]
        blk[blk == VT_VENTRICLE] = VT_PATHOLOGICAL

    numbers = _numbers(types_model)
    positions = _positions(spec.shape, spec.voxel_size_mm)
    s_pos, s_ori = _sensors(spec, positions, mask)
    if ctx is None:
        model = _ap_params(types_model, numbers, positions, spec, current_factor=0.0)
        truth = _ap_params(types_truth, numbers, positions, spec, current_factor=0.0)
        H = _measurement_matrix(spec, types_model, numbers, positions, s_pos, s_ori)
    else:
        from . import algorithm as alg

        def spatial(types):
            return alg.SpatialDescription(voxel_types=types, voxel_numbers=numbers, voxel_positions_mm=positions,
                                          voxel_size_mm=spec.voxel_size_mm, sensor_positions_mm=s_pos,
                                          sensor_orientations=s_ori, sensor_array_offsets_mm=array_offsets_mm(spec),
                                          sample_rate_hz=spec.sample_rate_hz,
                                          propagation_velocities_m_per_s=velocities_by_type(spec))

        def params(types):
            p = alg.ap_parameters(ctx, spatial(types), 0.0)
            return APParams(gains=p.gains, output_state_indices=p.output_state_indices, coefs=p.coefs,
                            delays=p.delays, initial_delays=p.initial_delays, activation_time_ms=p.activation_time_ms)

        model, truth = params(types_model), params(types_truth)
        H = alg.measurement_matrix(ctx, spatial(types_model))

    S = 3 * model.coefs.shape[0]
    control_matrix = np.zeros(S, dtype=np.float32)
    control_matrix[int(numbers[exc])] = 1.0
    onset = spec.pulse_onset if spec.pulse_onset is not None else int(rng.integers(0, max(1, spec.num_steps // 10)))
    u = _pulse(spec.num_steps, spec.pulse_sigma_samples, onset)

    return Scenario(
        spec=spec,
        types_truth=types_truth,
        types_model=types_model,
        numbers=numbers,
        positions_mm=positions,
        truth=truth,
        model=model,
        measurement_matrix=H,
        control_matrix=control_matrix,
        control_function=u,
        sensor_positions_mm=s_pos,
        sensor_orientations=s_ori,
    )


def attach_measurements(scn: Scenario, forward: Callable[..., np.ndarray]) -> Scenario:
    """Ground-truth measurements: forward of the truth model, plus seeded Gaussian noise.

    ``forward(gains, output_state_indices, coefs, delays, measurement_matrix,
    control_matrix, control_function) -> [B, T, M] f32`` runs the system
    prediction of every beat (the simulation loop of
    ``src/core/data/simulation.rs:129-150``). Noise is N(0, sigma) per sensor
    row with sigma = ``noise_fraction`` x RMS of the clean measurements.
    """
    t = scn.truth
    y = forward(
        t.gains,
        t.output_state_indices,
        t.coefs,
        t.delays,
        scn.measurement_matrix,
        scn.control_matrix,
        scn.control_function,
    ).astype(np.float32)
    if scn.spec.noise_fraction > 0:
        rng = np.random.default_rng(scn.spec.seed + 7919)
        sigma = scn.spec.noise_fraction * float(np.sqrt(np.mean(y.astype(np.float64) ** 2)))
        y = (y + rng.normal(0.0, sigma, size=y.shape)).astype(np.float32)
    scn.measurements = np.ascontiguousarray(y)
    return scn


# ---------------------------------------------------------------------------------------------
# the workloads


def workload_spec(name: str, seed: int = 0) -> ScenarioSpec:
    """Named workloads: 'cuboid8' (8^3, T=500), 'cuboid20' (20^3, T=2000),
    'shell' (64x64x48 ellipsoidal shell, T=4000), 'shell_precision' (T=8000, 256 sensors)."""
    if name == "cuboid8":
        return ScenarioSpec(shape=(8, 8, 8), num_steps=500, patho_size=3, patho_origin=(3, 3, 3), seed=seed)
    if name == "cuboid20":
        return ScenarioSpec(shape=(20, 20, 20), num_steps=2000, patho_size=5, noise_fraction=0.01, seed=seed)
    if name == "shell":
        return ScenarioSpec(shape=(64, 64, 48), mask="shell", num_steps=4000, patho_size=5, noise_fraction=0.01, seed=seed)
    if name == "shell_precision":
        return ScenarioSpec(
            shape=(64, 64, 48), mask="shell", num_steps=8000, num_sensors=256, patho_size=5, noise_fraction=0.01, seed=seed
        )
    raise ValueError(f"unknown workload {name!r}")


def batch_workload_specs(count: int = 64, seed: int = 0) -> list:
    """The batched workload: ``count`` scenarios of uneven size.

    Each draws its voxel count log-uniformly from 500 to 30,000 (even
    entries cuboids of random aspect, odd entries ellipsoidal shells scaled
    from the 64x64x48 shell), 1 to 8 beats, 1,000 to 4,000 steps, 37 to 128
    triaxial sensors, a random 3x3x3 pathological block and a random
    control-pulse onset in the first tenth of the beat. Sizes are drawn from
    ``seed``; every scenario has its own seed for the rest.
    """
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        target = float(np.exp(rng.uniform(np.log(500.0), np.log(30000.0))))
        beats = int(rng.integers(1, 9))
        steps = int(rng.integers(1000, 4001))
        sensors = int(rng.integers(37, 129))
        onset = int(rng.integers(0, steps // 10))
        if i % 2 == 0:
            a, b = (float(x) for x in rng.uniform(0.8, 1.25, size=2))
            edge = target ** (1.0 / 3.0)
            nx = max(4, int(round(edge * a)))
            ny = max(4, int(round(edge * b)))
            nz = max(4, int(round(target / (nx * ny))))
            spec = ScenarioSpec(shape=(nx, ny, nz), mask="cuboid")
        else:
            sc = (target / 47264.0) ** (1.0 / 3.0)
            shape = (max(8, int(math.ceil(64 * sc))), max(8, int(math.ceil(64 * sc))), max(6, int(math.ceil(48 * sc))))
            spec = ScenarioSpec(shape=shape, mask="shell", shell_semi_axes=(30.0 * sc, 25.0 * sc, 22.0 * sc),
                                shell_thickness=max(2.0, 8.0 * sc))
        spec.num_steps = steps
        spec.num_beats = beats
        spec.num_sensors = sensors
        spec.patho_size = 3
        spec.pulse_onset = onset
        spec.noise_fraction = 0.01
        spec.seed = seed * 1000 + i + 1
        specs.append(spec)
    return specs
