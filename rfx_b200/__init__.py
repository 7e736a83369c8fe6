"""rfx_b200: B200-native time-stepping hot path of the rfx FDTD solver.

The Yee E/H leapfrog on uniform and graded grids, CPML, PEC faces and edge
masks, soft sources, point probes, running-DFT planes, Poynting-flux monitors
and the NTFF Huygens box run as hand-written
sm_100a CUDA kernels behind the C ABI of ``include/rfxb200.h``; the modules
here are the host-side mirror of the reference's Python interface for that
path (``rfx.simulation.run``, ``rfx.nonuniform.run_nonuniform``), plus the
reverse-time adjoint and the batched sweep.
"""

from .grid import Grid, NonUniformGrid, make_nonuniform_grid  # noqa: F401
from .simulation import (  # noqa: F401
    DFTPlaneProbe, FDTDState, FluxMonitor, LumpedPortSParamSpec, MaterialArrays, ProbeSpec, SimResult,
    extract_lumped_s11, flux_spectrum, init_dft_plane_probe, init_flux_monitor, run, run_until_decay,
)
from .sources import (  # noqa: F401
    GaussianPulse, LumpedPort, SourceSpec, make_current_source, make_j_source, make_port_source,
    make_source, setup_lumped_port,
)
from .nonuniform import run_nonuniform, run_nonuniform_until_decay  # noqa: F401
from .checkpoint import (  # noqa: F401
    load_plan_state, load_snapshots, load_state, save_plan_state, save_snapshots, save_state,
)
from .farfield import (  # noqa: F401
    FarFieldResult, NTFFBox, NTFFData, compute_far_field, directivity, directivity_torch, far_field,
    init_ntff_data, make_ntff_box, radiation_pattern,
)

__version__ = "0.1.0"
