"""Oracle restatements of the model construction: the Biot-Savart measurement matrix
(measurement.rs:66-123) and the delay arrays (allpass/delay.rs:35-111, allpass.rs:86-100).

CPU-only. Pins: the reference's calculate_delay_s known answers (delay.rs:125-153), the
Biot-Savart law in float64 for a lone voxel, and bit-equality with the host scenario builder
(an independent vectorised restatement) on cuboids and shells with several beats.
"""

import math

import numpy as np
import pytest

from cardiotrust_b200 import scenario as sc


def _grid(types, positions):
    types = np.asarray(types, dtype=np.int32)
    numbers = np.full(types.shape, -1, dtype=np.int32)
    conn = (types >= 1) & (types <= 6)
    numbers[conn] = 3 * np.arange(int(conn.sum()), dtype=np.int32)
    return types, numbers, np.asarray(positions, dtype=np.float32)


@pytest.mark.parametrize("p_out, cell, velocity, rate, expect", [
    ((2000.0, 0.0, 0.0), (1, 0, 0), 2.0, 4.0, 0.5 * 4.0),   # calculate_delay_s_1: 0.5 s
    ((4000.0, 4000.0, 0.0), (1, 1, 0), 2.0, 2.0, 2.5 * 2.0),  # calculate_delay_s_2: 2.5 s
])
def test_delay_known_answers(oracle_mod, p_out, cell, velocity, rate, expect):
    types = np.zeros((2, 2, 1), np.int32)
    types[0, 0, 0] = sc.VT_VENTRICLE
    types[cell] = sc.VT_VENTRICLE
    pos = np.zeros((2, 2, 1, 3), np.float32)
    pos[0, 0, 0] = (1000.0, 0.0, 0.0)
    pos[cell] = p_out
    t, n, p = _grid(types, pos)
    vel = np.zeros(10, np.float32)
    vel[sc.VT_VENTRICLE] = velocity
    samples, delays, coefs = oracle_mod.delay_samples(t, n, p, vel, rate, 2)
    col = sc.offset_to_delay_index(cell[0], cell[1], cell[2])
    assert samples[0, col] == np.float32(expect)
    assert delays[0, col] == int(expect)
    assert coefs[0, col] == sc.from_samples_to_coef(expect)
    # the reverse pair has the same distance; every other column has no neighbour
    back = sc.offset_to_delay_index(-cell[0], -cell[1], -cell[2])
    assert samples[1, back] == np.float32(expect)
    others = np.ones((2, 26), bool)
    others[0, col] = others[1, back] = False
    assert np.all(samples[others] == 0) and np.all(delays[others] == 0)
    assert np.all(coefs[others] == np.float32(1.0) - np.float32(1e-4))


def test_delay_below_one_sample_names_first_pair(oracle_mod):
    spec = sc.ScenarioSpec(shape=(3, 3, 3), num_steps=4)
    s = sc.build(spec)
    vel = sc.velocities_by_type(spec) * np.float32(1e4)  # far too fast: every delay < 1 sample
    with pytest.raises(ValueError, match="cell 0, offset column 13"):
        # cell (0,0,0): offsets with x = -1, y = -1 or z = -1 leave the grid; (0,0,+1) is column 13
        oracle_mod.delay_samples(s.types_model, s.numbers, s.positions_mm, vel, spec.sample_rate_hz, s.num_voxels)


def test_lead_field_lone_voxel_matches_biot_savart(oracle_mod):
    types = np.full((1, 1, 1), sc.VT_VENTRICLE, np.int32)
    pos = np.array([[[[1.0, -2.0, 3.0]]]], np.float32)
    t, n, p = _grid(types, pos)
    sp = np.array([[10.0, 20.0, 100.0], [-30.0, 5.0, 80.0]], np.float32)
    so = np.array([[0.0, 0.0, 1.0], [0.6, 0.8, 0.0]], np.float32)
    off = np.array([[0.0, 0.0, 0.0], [5.0, 0.0, 0.0]], np.float32)
    H = oracle_mod.measurement_matrix(t, n, p, 2.5, sp, so, off, 3)
    vol = (2.5e-3) ** 3
    for b in range(2):
        for m in range(2):
            d = (sp[m].astype(np.float64) + off[b] - pos[0, 0, 0]) / 1000.0
            # B . o = p . (d x o) for a current dipole p at the voxel, d = sensor - voxel
            want = 1e-7 * vol * np.cross(d, so[m].astype(np.float64)) / np.linalg.norm(d) ** 3 * 1e12
            np.testing.assert_allclose(H[b, m], want, rtol=2e-6, atol=1e-12 * np.abs(want).max())


@pytest.mark.parametrize("spec", [
    sc.ScenarioSpec(shape=(8, 8, 8), num_beats=2, num_steps=4),
    sc.ScenarioSpec(shape=(20, 20, 16), mask="shell", shell_semi_axes=(9.0, 8.0, 7.0), shell_thickness=3.0,
                    num_beats=3, num_steps=4),
], ids=["cuboid8_b2", "shell_b3"])
def test_oracle_equals_host_builder(oracle_mod, spec):
    s = sc.build(spec)
    H = oracle_mod.measurement_matrix(s.types_model, s.numbers, s.positions_mm, spec.voxel_size_mm,
                                      s.sensor_positions_mm, s.sensor_orientations, sc.array_offsets_mm(spec),
                                      s.num_states)
    assert np.array_equal(H.view(np.uint32), s.measurement_matrix.view(np.uint32))
    samples, delays, coefs = oracle_mod.delay_samples(s.types_model, s.numbers, s.positions_mm,
                                                      sc.velocities_by_type(spec), spec.sample_rate_hz, s.num_voxels)
    m = s.model
    assert np.array_equal(samples, m.initial_delays)
    assert np.array_equal(delays, m.delays)
    assert np.array_equal(coefs.view(np.uint32), m.coefs.view(np.uint32))
    # the lattice's three distances: faces, face diagonals, body diagonals (2.5 mm at 0.6 m/s, 2 kHz)
    base = 2.5e-3 / 0.6 * 2000.0
    vals = np.unique(samples[samples > 0])
    np.testing.assert_allclose(vals, [base, base * math.sqrt(2), base * math.sqrt(3)], rtol=1e-6)
