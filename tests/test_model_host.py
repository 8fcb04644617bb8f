"""The library's native host model builders against the oracle (CPU, no device work):
ct_connect_voxels (connect_voxels / try_to_connect, allpass.rs:295-494) and ct_output_state_indices
(init_output_state_indicies, allpass.rs:212-289).

Bars: gains and activation times bit-identical to the oracle's literal activation-time sweep and to
the host scenario builder (a third restatement, heap-ordered); the index table equal to the
builder's. Cases: cuboids and shells, the ground truth's pathological block with a zero and a
non-zero current factor, per-type velocities, several Sinoatrial voxels, atrial/AV/HPS types with
the reference's connection rules; the gain-row-sum invariant of src/core/model/tests.rs:8-60.
"""

import numpy as np
import pytest

from cardiotrust_b200 import scenario as sc

SPECS = {
    "cuboid8": sc.ScenarioSpec(shape=(8, 8, 8), num_steps=4),
    "shell": sc.ScenarioSpec(shape=(20, 20, 16), mask="shell", shell_semi_axes=(9.0, 8.0, 7.0), shell_thickness=3.0,
                             num_steps=4, patho_size=3, seed=2),
    "cuboid_random_sa": sc.ScenarioSpec(shape=(9, 7, 6), num_steps=4, excitation="random", seed=7),
}


@pytest.fixture(scope="module")
def alg():
    from cardiotrust_b200 import algorithm

    return algorithm


def _oracle(oracle_mod, sd, factor):
    return oracle_mod.connect_voxels(sd.voxel_types, sd.voxel_numbers, sd.voxel_positions_mm,
                                     sd.propagation_velocities_m_per_s, factor, 3 * sd.num_voxels)


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


@pytest.mark.parametrize("name", sorted(SPECS))
@pytest.mark.parametrize("truth", [False, True], ids=["model", "truth"])
def test_connect_voxels_matches_oracle_and_builder(alg, oracle_mod, name, truth):
    s = sc.build(SPECS[name])
    sd = alg.SpatialDescription.from_scenario(s, truth=truth)
    gains, act = alg.connect_voxels(sd, 0.0)
    g_o, a_o = _oracle(oracle_mod, sd, 0.0)
    assert _same(gains, g_o) and _same(act, a_o)
    p = s.truth if truth else s.model
    assert _same(gains, p.gains) and _same(act, p.activation_time_ms)
    assert np.array_equal(alg.output_state_indices(sd), p.output_state_indices)


@pytest.mark.parametrize("factor", [0.5, 2.0, 1e-3])
def test_pathology_current_factor(alg, oracle_mod, factor):
    """A non-zero factor connects the pathological block and scales gains into / out of it."""
    s = sc.build(SPECS["shell"])
    sd = alg.SpatialDescription.from_scenario(s, truth=True)
    assert (sd.voxel_types == sc.VT_PATHOLOGICAL).any()
    gains, act = alg.connect_voxels(sd, factor)
    g_o, a_o = _oracle(oracle_mod, sd, factor)
    assert _same(gains, g_o) and _same(act, a_o)
    patho = sd.voxel_types == sc.VT_PATHOLOGICAL
    assert np.all(np.isfinite(act[patho]))
    g0, a0 = alg.connect_voxels(sd, 0.0)
    assert np.all(np.isnan(a0[patho]))


def test_tissue_types_velocities_and_two_sinoatrial_voxels(alg, oracle_mod):
    """Atrium / AV / HPS / ventricle layers with their own velocities and the reference's connection
    rules (voxels.rs:707-742), two Sinoatrial voxels, and cells without a voxel."""
    s = sc.build(sc.ScenarioSpec(shape=(10, 6, 6), num_steps=4))
    types = s.types_model.copy()
    types[:3] = sc.VT_ATRIUM
    types[3] = sc.VT_AV
    types[4:6] = sc.VT_HPS
    types[6:] = sc.VT_VENTRICLE
    types[0, 0, 0] = types[0, 5, 5] = sc.VT_SINOATRIAL
    types[8, 2:4, 2:4] = sc.VT_NONE
    types[2, 1, 1] = sc.VT_PATHOLOGICAL
    numbers = np.full(types.shape, -1, np.int32)
    conn = (types >= 1) & (types <= 6)
    numbers[conn] = 3 * np.arange(int(conn.sum()), dtype=np.int32)
    vel = np.zeros(10, np.float32)
    vel[1:7] = np.array([0.8, 0.7, 0.05, 2.0, 0.6, 0.3], np.float32)
    sd = alg.SpatialDescription(voxel_types=types, voxel_numbers=numbers, voxel_positions_mm=s.positions_mm,
                                voxel_size_mm=2.5, sensor_positions_mm=s.sensor_positions_mm,
                                sensor_orientations=s.sensor_orientations,
                                sensor_array_offsets_mm=np.zeros((1, 3), np.float32),
                                propagation_velocities_m_per_s=vel)
    for factor in (0.0, 0.25):
        gains, act = alg.connect_voxels(sd, factor)
        g_o, a_o = _oracle(oracle_mod, sd, factor)
        assert _same(gains, g_o) and _same(act, a_o)
    assert act[0, 0, 0] == 0 and act[0, 5, 5] == 0
    assert np.isnan(act[8, 2, 2])  # no voxel there
    assert np.all(np.isfinite(act[conn]))  # the AV layer passes the front from atrium to HPS


def test_gain_row_sum_invariant(alg):
    """src/core/model/tests.rs:8-60: per voxel, sum of |gains| over its three rows plus the control
    matrix lies in (0.99, 3.01)."""
    s = sc.build(SPECS["shell"])
    sd = alg.SpatialDescription.from_scenario(s)
    gains, _ = alg.connect_voxels(sd, 0.0)
    V = sd.num_voxels
    sums = np.abs(gains).reshape(V, 3 * 78).sum(axis=1) + s.control_matrix.reshape(V, 3).sum(axis=1)
    assert np.all((sums > 0.99) & (sums < 3.01))


def test_invalid_numbering_and_sizes_are_rejected(alg):
    from cardiotrust_b200._lib import CT_ERR_INVALID_ARGUMENT, CtError, fptr, lib

    s = sc.build(SPECS["cuboid8"])
    sd = alg.SpatialDescription.from_scenario(s)
    nums = sd.voxel_numbers.copy()
    nums[1, 1, 1] = nums[1, 1, 2]
    sd.voxel_numbers = nums
    with pytest.raises(CtError) as e:
        alg.connect_voxels(sd, 0.0)
    assert e.value.status == CT_ERR_INVALID_ARGUMENT
    with pytest.raises(CtError):
        alg.output_state_indices(sd)
    sd = alg.SpatialDescription.from_scenario(s)
    desc, _keep = sd.to_ct()
    small = np.empty((3, 78), np.float32)
    act = np.empty(sd.voxel_types.shape, np.float32)
    import ctypes

    assert lib().ct_connect_voxels(ctypes.byref(desc), 0.0, fptr(small), small.nbytes, fptr(act)) == \
        CT_ERR_INVALID_ARGUMENT


def test_no_sinoatrial_voxel_activates_nothing(alg, oracle_mod):
    """Without a Sinoatrial voxel the reference's sweep finds no candidate at time 0 and stops: every
    activation time stays None and every gain 0."""
    s = sc.build(SPECS["cuboid8"])
    sd = alg.SpatialDescription.from_scenario(s)
    types = sd.voxel_types.copy()
    types[types == sc.VT_SINOATRIAL] = sc.VT_VENTRICLE
    sd.voxel_types = types
    gains, act = alg.connect_voxels(sd, 0.0)
    g_o, a_o = _oracle(oracle_mod, sd, 0.0)
    assert np.all(np.isnan(act)) and np.all(np.isnan(a_o))
    assert not gains.any() and not g_o.any()


def test_isolated_voxel_and_unknown_types(alg, oracle_mod):
    """A connectable voxel with no connectable neighbour is never activated; cells of non-connectable
    types (Vessel, Torso, Chamber) neither carry voxels nor pass the front."""
    types = np.full((6, 5, 4), sc.VT_VENTRICLE, np.int32)
    types[0, 0, 0] = sc.VT_SINOATRIAL
    types[3, :, :] = sc.VT_TORSO  # a wall the front cannot cross
    types[5, 4, 3] = sc.VT_VENTRICLE
    types[4, :, :] = sc.VT_CHAMBER
    types[5, :, :] = sc.VT_VESSEL
    types[5, 4, 3] = sc.VT_VENTRICLE  # isolated behind the wall
    numbers = np.full(types.shape, -1, np.int32)
    conn = (types >= 1) & (types <= 6)
    numbers[conn] = 3 * np.arange(int(conn.sum()), dtype=np.int32)
    pos = (np.stack(np.meshgrid(*[np.arange(n) for n in types.shape], indexing="ij"), axis=-1) * 2.5).astype(np.float32)
    vel = np.zeros(10, np.float32)
    vel[1:7] = 0.6
    sd = alg.SpatialDescription(voxel_types=types, voxel_numbers=numbers, voxel_positions_mm=pos, voxel_size_mm=2.5,
                                sensor_positions_mm=np.zeros((3, 3), np.float32),
                                sensor_orientations=np.eye(3, dtype=np.float32),
                                sensor_array_offsets_mm=np.zeros((1, 3), np.float32),
                                propagation_velocities_m_per_s=vel)
    gains, act = alg.connect_voxels(sd, 0.0)
    g_o, a_o = _oracle(oracle_mod, sd, 0.0)
    assert _same(gains, g_o) and _same(act, a_o)
    assert np.all(np.isfinite(act[:3])) and np.all(np.isnan(act[3:]))
    v_iso = numbers[5, 4, 3] // 3
    assert not gains[3 * v_iso:3 * v_iso + 3].any()
    osi = alg.output_state_indices(sd)
    assert np.all(osi[3 * v_iso:3 * v_iso + 3] == -1)  # no connectable neighbour at any offset


def test_spatial_description_shapes_are_checked(alg):
    """The Python mirror refuses malformed arrays before any library call."""
    from cardiotrust_b200._lib import CtError

    s = sc.build(SPECS["cuboid8"])
    good = alg.SpatialDescription.from_scenario(s)
    assert good.num_voxels == s.num_voxels and good.num_sensors == s.num_sensors and good.num_beats == 1
    for field, value in (("voxel_numbers", s.numbers[:-1]), ("voxel_positions_mm", s.positions_mm[..., :2]),
                         ("sensor_orientations", s.sensor_orientations[:-1]),
                         ("propagation_velocities_m_per_s", np.zeros(6, np.float32))):
        bad = alg.SpatialDescription.from_scenario(s)
        setattr(bad, field, value)
        with pytest.raises(CtError):
            bad.to_ct()


def test_array_offsets_and_velocities(alg):
    spec = sc.ScenarioSpec(shape=(4, 4, 4), num_beats=3, beat_shift_mm=7.5, velocity_m_per_s=0.8)
    off = sc.array_offsets_mm(spec)
    assert off.shape == (3, 3) and np.array_equal(off[:, 0], np.float32([0.0, 7.5, 15.0])) and not off[:, 1:].any()
    vel = sc.velocities_by_type(spec)
    assert vel.shape == (10,) and np.all(vel[1:7] == np.float32(0.8)) and vel[0] == 0 and not vel[7:].any()


def test_full_size_shell_matches_literal_sweep(alg, oracle_mod):
    """The 64x64x48 ellipsoidal shell of the adjoint and precision configs (47,264 voxels): the native
    search equals the literal sweep (a full grid scan per activation time, ~10 s) bit for bit."""
    s = sc.build(sc.workload_spec("shell"))
    sd = alg.SpatialDescription.from_scenario(s)
    gains, act = alg.connect_voxels(sd, 0.0)
    g_o, a_o = _oracle(oracle_mod, sd, 0.0)
    assert _same(gains, g_o) and _same(act, a_o)
    assert np.isfinite(act).sum() == sd.num_voxels
