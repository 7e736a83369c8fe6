"""Regenerate the golden fixtures in this folder.

``forward_no_rlc_s11.npy`` is the reference's own fixture
``tests/fixtures/golden_forward_no_rlc_s11.npy`` (rfx-fdtd 1.6.7): S11 of a
CPML-6 lumped-port run at 3..7 GHz, produced by the reference's JAX solver and
asserted by its ``tests/test_lumped_rlc_ad.py:138-152``.  It is copied as data
because the reference tree is not available where the tests run.

``oracle_<scenario>.npz`` hold the probe traces and DFT planes of the
scenarios in ``tests/scenarios.py`` computed by the CPU oracle in float32
(``*_f32``) and float64 (``*_f64``) arithmetic; they let the GPU tests check
the CUDA path without re-running the oracle.

Usage: ``python tests/golden/make_golden.py /path/to/rfx``
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main(ref_root):
    src = os.path.join(ref_root, "tests", "fixtures", "golden_forward_no_rlc_s11.npy")
    shutil.copyfile(src, os.path.join(HERE, "forward_no_rlc_s11.npy"))
    from tests.scenarios import c1_readme, medium_uniform, small_nonuniform, small_uniform
    for build in (small_uniform, small_nonuniform, c1_readme, medium_uniform):
        sc = build()
        out = {}
        for tag, dt in (("f32", np.float32), ("f64", np.float64)):
            res = sc.run_oracle(dt)
            out[f"ts_{tag}"] = res.time_series
            for q, acc in enumerate(res.dft_planes):
                out[f"dft{q}_{tag}"] = acc
        np.savez_compressed(os.path.join(HERE, f"oracle_{sc.name}.npz"), **out)
        print(sc.name, "written")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
