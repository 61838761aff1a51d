"""B200 particle erosion: a CUDA drop-in for the bake's erosion stage.

``pgerosion.maps`` mirrors ``globe.erosion.maps`` (ErosionState,
run_iteration, step, thermal_erosion, apply_uplift, start_replay,
hold_datum) with the state on the GPU and every pass in libpgerosion.so;
``pgerosion.stage`` mirrors ``globe.erosion.run`` (run, checkpoints,
outputs).  ``pgerosion.geometry`` builds the cube-sphere tables,
``pgerosion.params`` the parameters and random streams, and
``pgerosion.synth`` the seeded synthetic worlds of the benchmarks.
"""
from . import _lib, geometry, params, synth  # noqa: F401

__version__ = "0.1.0"


def library_version() -> int:
    return int(_lib.load().pge_version())
