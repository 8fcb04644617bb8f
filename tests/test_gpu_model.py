"""Model construction on the device against the oracle, through the C ABI.

Bars: the measurement matrix and the delay arrays are bit-identical to the oracle's f32 loops
(measurement.rs:66-123, allpass/delay.rs:35-111) - every operation is one IEEE-rounded
add, multiply, divide or square root, or the reference's fused multiply-add, in the reference's
order; only the sign of exact zeros may differ, so values are compared with ==. An epoch of a
scenario whose matrix was computed on the device is bit-identical to one whose matrix was copied
from the host, with FP32 and tensor-core products (whose operand splits are rebuilt by the fill).
"""

import numpy as np
import pytest

from conftest import oracle_forward

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def alg():
    from cardiotrust_b200 import algorithm

    return algorithm


@pytest.fixture(scope="module")
def ctx(alg):
    c = alg.Context(0)
    yield c
    c.close()


def _specs():
    from cardiotrust_b200 import scenario as sc

    return {
        "cuboid8_b2": sc.ScenarioSpec(shape=(8, 8, 8), num_beats=2, num_steps=4),
        "shell_b3": sc.ScenarioSpec(shape=(20, 20, 16), mask="shell", shell_semi_axes=(9.0, 8.0, 7.0),
                                    shell_thickness=3.0, num_beats=3, num_steps=4, patho_size=3, seed=5),
    }


def _oracle_h(oracle_mod, sd):
    return oracle_mod.measurement_matrix(sd.voxel_types, sd.voxel_numbers, sd.voxel_positions_mm, sd.voxel_size_mm,
                                         sd.sensor_positions_mm, sd.sensor_orientations, sd.sensor_array_offsets_mm,
                                         3 * sd.num_voxels)


@pytest.mark.parametrize("name", ["cuboid8_b2", "shell_b3"])
def test_measurement_matrix_bit_identical(alg, ctx, oracle_mod, name):
    from cardiotrust_b200 import scenario as sc

    s = sc.build(_specs()[name])
    sd = alg.SpatialDescription.from_scenario(s)
    H = alg.measurement_matrix(ctx, sd)
    want = _oracle_h(oracle_mod, sd)
    assert H.shape == want.shape
    assert np.array_equal(H, want)
    assert np.array_equal(H, s.measurement_matrix)


def test_measurement_matrix_general_orientations(alg, ctx, oracle_mod):
    """Sensors tilted off the axes: the cross product's fused multiply-adds matter."""
    from cardiotrust_b200 import scenario as sc

    s = sc.build(_specs()["shell_b3"])
    rng = np.random.default_rng(11)
    ori = rng.normal(size=s.sensor_orientations.shape)
    ori = (ori / np.linalg.norm(ori, axis=1, keepdims=True)).astype(np.float32)
    sd = alg.SpatialDescription.from_scenario(s)
    sd.sensor_orientations = ori
    sd.sensor_positions_mm = (s.sensor_positions_mm + rng.normal(scale=3.0, size=ori.shape)).astype(np.float32)
    assert np.array_equal(alg.measurement_matrix(ctx, sd), _oracle_h(oracle_mod, sd))


@pytest.mark.parametrize("name", ["cuboid8_b2", "shell_b3"])
def test_delay_samples_bit_identical(alg, ctx, oracle_mod, name):
    from cardiotrust_b200 import scenario as sc

    s = sc.build(_specs()[name])
    sd = alg.SpatialDescription.from_scenario(s, truth=True)  # the pathological block has its own velocity
    vel = sd.propagation_velocities_m_per_s.copy()
    vel[sc.VT_PATHOLOGICAL] = np.float32(0.37)
    vel[sc.VT_SINOATRIAL] = np.float32(0.45)
    sd.propagation_velocities_m_per_s = vel
    samples, delays, coefs = alg.delay_samples(ctx, sd)
    w_s, w_d, w_c = oracle_mod.delay_samples(sd.voxel_types, sd.voxel_numbers, sd.voxel_positions_mm, vel,
                                             sd.sample_rate_hz, sd.num_voxels)
    assert np.array_equal(samples, w_s)
    assert np.array_equal(delays, w_d)
    assert np.array_equal(coefs.view(np.uint32), w_c.view(np.uint32))
    if name == "cuboid8_b2":
        sd0 = alg.SpatialDescription.from_scenario(s)
        s0, d0, c0 = alg.delay_samples(ctx, sd0)
        assert np.array_equal(s0, s.model.initial_delays) and np.array_equal(d0, s.model.delays)
        assert np.array_equal(c0, s.model.coefs)


def test_delay_below_one_sample_is_an_error(alg, ctx, oracle_mod):
    from cardiotrust_b200 import scenario as sc
    from cardiotrust_b200._lib import CT_ERR_INVALID_ARGUMENT, CtError

    spec = sc.ScenarioSpec(shape=(3, 3, 3), num_steps=4)
    s = sc.build(spec)
    sd = alg.SpatialDescription.from_scenario(s)
    sd.propagation_velocities_m_per_s = sd.propagation_velocities_m_per_s * np.float32(1e4)
    with pytest.raises(CtError, match=r"voxel \(0, 0, 0\), offset column 13") as e:
        alg.delay_samples(ctx, sd)
    assert e.value.status == CT_ERR_INVALID_ARGUMENT
    with pytest.raises(ValueError, match="cell 0, offset column 13"):
        oracle_mod.delay_samples(sd.voxel_types, sd.voxel_numbers, sd.voxel_positions_mm,
                                 sd.propagation_velocities_m_per_s, sd.sample_rate_hz, sd.num_voxels)


def test_invalid_grids_are_rejected(alg, ctx):
    from cardiotrust_b200 import scenario as sc
    from cardiotrust_b200._lib import CT_ERR_INVALID_ARGUMENT, CtError

    s = sc.build(sc.ScenarioSpec(shape=(3, 3, 3), num_steps=4))
    for bad in ("duplicate", "not_multiple_of_3", "missing"):
        sd = alg.SpatialDescription.from_scenario(s)
        nums = sd.voxel_numbers.copy()
        if bad == "duplicate":
            nums[0, 0, 1] = nums[0, 0, 0]
        elif bad == "not_multiple_of_3":
            nums[0, 0, 1] += 1
        else:
            nums[2, 2, 2] = -1
        sd.voxel_numbers = nums
        with pytest.raises(CtError) as e:
            alg.measurement_matrix(ctx, sd)
        assert e.value.status == CT_ERR_INVALID_ARGUMENT
        with pytest.raises(CtError):
            alg.delay_samples(ctx, sd)


def test_scenario_lead_field_on_device_gives_identical_epochs(alg, ctx, oracle_mod):
    """A 9x7x5 cuboid (945 states, not a multiple of 4: padded tensor-core operands) with 2 beats,
    created without a host matrix and filled on the device, against the same scenario copied from
    the host."""
    from cardiotrust_b200 import scenario as sc
    from cardiotrust_b200._lib import CtError

    spec = sc.ScenarioSpec(shape=(9, 7, 5), num_steps=200, num_beats=2, patho_size=3, pulse_onset=2,
                           pulse_sigma_samples=5.0, noise_fraction=0.01, seed=4)
    s = sc.attach_measurements(sc.build(spec), oracle_forward(oracle_mod))
    assert s.num_states % 4 != 0
    cfg = alg.Algorithm(optimizer=alg.Optimizer.Adam, learning_rate=1e-2, freeze_delays=False)
    for precision in (alg.Precision.Fp32, alg.Precision.Tf32x3):
        host = alg.EpochEngine.from_scenario(ctx, s, algorithm=cfg)
        dev = alg.EpochEngine.from_scenario(ctx, s, algorithm=cfg, device_lead_field=True)
        for e in (host, dev):
            e.run_epoch(0, beat_order=[1, 0], precision=precision)
        for name in ("measurements", "system_states", "grad_gains", "grad_coefs", "gains", "coefs", "loss"):
            a, b = host.read(name), dev.read(name)
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (precision, name)
        assert np.abs(dev.read("measurements")).max() > 0
        # a description of another scenario size is refused
        sd = alg.SpatialDescription.from_scenario(s)
        sd.sensor_positions_mm = sd.sensor_positions_mm[:-3]
        sd.sensor_orientations = sd.sensor_orientations[:-3]
        with pytest.raises(CtError):
            dev.set_measurement_matrix(sd)
        host.close()
        dev.close()


@pytest.mark.parametrize("name", ["cuboid8_b2", "shell_b3"])
def test_builder_on_the_library_equals_numpy_builder(alg, ctx, name):
    """scenario.build(spec, ctx): gains, index table and activation times from the native search, delay
    arrays and measurement matrix from the device - the same scenario as the numpy restatement."""
    from cardiotrust_b200 import scenario as sc

    spec = _specs()[name]
    a, b = sc.build(spec), sc.build(spec, ctx=ctx)
    assert np.array_equal(a.measurement_matrix, b.measurement_matrix)
    for p, q in ((a.model, b.model), (a.truth, b.truth)):
        for f in ("gains", "output_state_indices", "coefs", "delays", "initial_delays", "activation_time_ms"):
            x, y = getattr(p, f), getattr(q, f)
            assert x.dtype == y.dtype and x.shape == y.shape, f
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), f
