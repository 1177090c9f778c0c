"""Problem registry (``get_preset``) with the reference's 3D presets.

The table restates ``gpu_fem/presets.py:31-441`` (geometry, mesh counts,
supports and loads per preset name) so preset names keep meaning the same
problem; the solve path reads nothing else from a preset.
"""

from __future__ import annotations

from .problem_spec import DistributedLoad, EdgeSupport, PointLoad, PointSupport, ProblemSpec


def _cantilever(nx, ny, nz, vf=0.3):
    return ProblemSpec(Lx=2.0, Ly=1.0, Lz=0.5, nelx=nx, nely=ny, nelz=nz, volfrac=vf,
                       supports=[EdgeSupport("left", "fixed")],
                       loads=[PointLoad(x=2.0, y=0.5, z=0.25, fy=-1.0)])


def _bridge(nx, ny, nz, zs=(0.0, 0.25, 0.5), Lx=3.0, Lz=0.5):
    sup = [PointSupport(0.0, 0.0, z, "fixed") for z in zs]
    sup += [PointSupport(Lx, 0.0, z, "roller_x") for z in zs]
    return ProblemSpec(Lx=Lx, Ly=1.0, Lz=Lz, nelx=nx, nely=ny, nelz=nz, volfrac=0.3,
                       supports=sup, loads=[DistributedLoad("top", -1.0)])


def _mbb(nx, ny, nz):
    return ProblemSpec(Lx=3.0, Ly=1.0, Lz=0.5, nelx=nx, nely=ny, nelz=nz, volfrac=0.5,
                       supports=[EdgeSupport("left", "pin_x"), PointSupport(3.0, 0.0, 0.25, "pin_y")],
                       loads=[PointLoad(x=0.0, y=1.0, z=0.25, fy=-1.0)])


def _bracket(nx, ny, nz):
    return ProblemSpec(Lx=1.0, Ly=2.0, Lz=0.5, nelx=nx, nely=ny, nelz=nz, volfrac=0.3,
                       supports=[EdgeSupport("top", "fixed")],
                       loads=[PointLoad(x=1.0, y=0.0, z=0.25, fy=-0.7, fx=0.3)])


def _torsion(nx, ny, nz):
    return ProblemSpec(Lx=3.0, Ly=1.0, Lz=1.0, nelx=nx, nely=ny, nelz=nz, volfrac=0.25,
                       supports=[EdgeSupport("left", "fixed")],
                       loads=[PointLoad(3.0, 1.0, 0.5, fy=-0.5, fz=0.5),
                              PointLoad(3.0, 0.0, 0.5, fy=0.5, fz=-0.5)])


def _column(nx, ny, nz):
    return ProblemSpec(Lx=1.0, Ly=4.0, Lz=1.0, nelx=nx, nely=ny, nelz=nz, volfrac=0.20,
                       supports=[EdgeSupport("bottom", "fixed")],
                       loads=[DistributedLoad("top", -1.0)])


PRESETS_3D = {
    "cantilever_3d": _cantilever(24, 12, 6),
    "bridge_3d": _bridge(30, 10, 5),
    "mbb_3d": _mbb(30, 10, 5),
    "bracket_3d": _bracket(12, 24, 6),
    "torsion_3d": _torsion(30, 10, 10),
    "column_3d": _column(10, 40, 10),
    "cantilever_3d_large": _cantilever(40, 20, 10),
    "cantilever_3d_xlarge": _cantilever(60, 30, 15),
    "cantilever_3d_vf02": _cantilever(24, 12, 6, 0.20),
    "cantilever_3d_vf04": _cantilever(24, 12, 6, 0.40),
}

PRESETS_GPU = {
    "cantilever_gpu_medium": _cantilever(80, 40, 20),
    "cantilever_gpu_large": _cantilever(120, 60, 30),
    "cantilever_gpu_xlarge": _cantilever(160, 80, 40),
    "cantilever_gpu_xxlarge": _cantilever(200, 100, 50),
    "cantilever_gpu_2M": _cantilever(252, 126, 63),
    "cantilever_gpu_5M": _cantilever(342, 171, 86),
    "cantilever_gpu_8M": _cantilever(400, 200, 100),
    "cantilever_gpu_10M": _cantilever(430, 215, 108),
    "mbb_gpu_xlarge": _mbb(210, 70, 35),
    "mbb_gpu_xxlarge": _mbb(264, 88, 44),
    "bridge_gpu_large": _bridge(150, 50, 25, zs=(0.0, 0.125, 0.25, 0.375, 0.5)),
    "bridge_gpu_medium": _bridge(90, 30, 15),
    "bridge_gpu_xlarge": _bridge(180, 60, 30),
    "bridge_gpu_500k": _bridge(210, 70, 35),
    "bridge_gpu_1M": _bridge(264, 88, 44),
    "mbb_gpu_medium": _mbb(90, 30, 15),
    # the reference table defines mbb_gpu_large twice; the later 150x50x25 entry wins
    "mbb_gpu_large": _mbb(150, 50, 25),
    "torsion_gpu_medium": _torsion(60, 20, 20),
    "bracket_gpu_medium": _bracket(30, 60, 15),
    "column_gpu_medium": _column(20, 80, 20),
    "torsion_gpu_500k": _torsion(165, 55, 55),
    "torsion_gpu_1M": _torsion(210, 70, 70),
    "column_gpu_500k": _column(50, 200, 50),
    "column_gpu_1M": _column(63, 252, 63),
    "bracket_gpu_500k": _bracket(80, 160, 40),
    "bracket_gpu_1M": _bracket(100, 200, 50),
}

ALL_PRESETS = {**PRESETS_3D, **PRESETS_GPU}


def cantilever_spec(nelx: int, nely: int, nelz: int) -> ProblemSpec:
    """Cantilever of the reference geometry on an arbitrary grid (x=0 face clamped,
    unit downward load at the node nearest the centre of the x = Lx face)."""
    return _cantilever(nelx, nely, nelz)


def get_preset(name: str) -> ProblemSpec:
    if name not in ALL_PRESETS:
        raise KeyError(f"Unknown preset '{name}'. Available: {sorted(ALL_PRESETS.keys())}")
    return ALL_PRESETS[name]


def list_presets() -> list[str]:
    return sorted(ALL_PRESETS.keys())
