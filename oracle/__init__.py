"""CPU oracle for the rfx time-stepping hot path -- TEST INFRASTRUCTURE ONLY.

This package is a NumPy restatement of the reference solver's scan body
(bk-squared/rfx, rfx-fdtd 1.6.7).  It exists only to check the CUDA path:
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it, and nothing in the
``rfx_b200`` package may.  The product path never routes through it.

Pinning.  The reference cannot run in this environment (it needs JAX, which is
not installed and cannot be fetched).  The restatement is pinned instead by
(1) the reference's own golden vector ``tests/fixtures/golden_forward_no_rlc_s11.npy``
(a CPML-6 uniform scan with a lumped port, reproduced by ``oracle.port``; see
``tests/test_oracle_golden.py``), and (2) the reference's physics gates restated
on it (CPML reflection and energy decay from ``tests/test_cpml.py``, the
running DFT against a post-hoc DFT from ``tests/test_dft_probes.py``, and the
non-uniform-to-uniform reduction).  Every function cites the reference file and
line it follows.
"""

from .fdtd import (  # noqa: F401
    C0, EPS_0, MU_0,
    UniformGrid, NonUniformGrid, make_uniform_grid, make_nonuniform_grid,
    profile_to_inv_arrays, cpml_profile, build_cpml,
    gaussian_pulse, j_source_waveform, current_source_waveform,
    port_source_waveform, port_sigma,
    tangential_edge_masks, run_uniform, run_nonuniform, run_until_decay_uniform, run_until_decay_nonuniform,
    OracleResult,
    NTFF_FACES, ntff_init, ntff_phases, ntff_step,
)
from . import farfield  # noqa: F401
