"""Regenerate tests/golden/cuboid4_b2.npz: a 4x4x4 cuboid, 2 beats, T=64, one
Adam epoch with coefficient derivatives, computed by the f32 CPU restatement.

Run from the repository root:  python tests/golden/make_golden.py
The fixture stores the scenario inputs and the oracle's outputs, so the GPU
test compares against committed bytes rather than a live CPU run.
"""

import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from cardiotrust_b200 import scenario as sc  # noqa: E402

OUT = pathlib.Path(__file__).with_name("cuboid4_b2.npz")
ALGO = dict(optimizer=1, ap_derivative=1, freeze_gains=0, freeze_delays=0, batch_size=0, learning_rate=0.01,
            difference_regularization_strength=1e-3, smoothness_regularization_strength=1e-2)
BEAT_ORDER = np.array([1, 0], dtype=np.int32)


def main():
    spec = sc.ScenarioSpec(shape=(4, 4, 4), num_steps=64, num_beats=2, patho_size=2, patho_origin=(1, 1, 1),
                           pulse_onset=2, pulse_sigma_samples=3.0, noise_fraction=0.01, seed=11)
    scn = sc.build(spec)

    def fwd(gains, osi, coefs, delays, H, ctrl, u):
        return oracle.OracleEpoch(gains, osi, coefs, delays, np.zeros_like(coefs), H, ctrl, u).simulate()

    sc.attach_measurements(scn, fwd)
    o = oracle.from_scenario(scn)
    o.run_epoch(oracle.algo(**ALGO), beat_order=BEAT_ORDER)
    m = scn.model
    np.savez_compressed(
        OUT,
        gains=m.gains, output_state_indices=m.output_state_indices, coefs=m.coefs, delays=m.delays,
        initial_delays=m.initial_delays, measurement_matrix=scn.measurement_matrix,
        control_matrix=scn.control_matrix, control_function=scn.control_function,
        measurements_actual=scn.measurements, beat_order=BEAT_ORDER,
        algo=np.array([ALGO[k] for k in sorted(ALGO)], dtype=np.float64), algo_keys=np.array(sorted(ALGO)),
        out_system_states=o.system_states, out_measurements=o.measurements, out_grad_gains=o.d_gains,
        out_grad_coefs=o.d_coefs, out_gains=o.gains, out_coefs=o.coefs, out_delays=o.delays,
        out_loss=o.loss, out_loss_mse=o.loss_mse, out_loss_maximum_regularization=o.loss_maximum_regularization,
        out_loss_batch=o.loss_batch, out_average_delays=o.average_delays,
    )
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
