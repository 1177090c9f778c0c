"""Fixtures from the reference's published guarded SIMP trajectories.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_published_trajectories.py

Copies the reference's data/analysis_tables/guarded_adaptive_trajectories__*.csv
(its run_simp_floor_trajectory.py with --policy guarded_adaptive at the default
arguments on cantilever_gpu_medium, 64,000 elements, and bridge_gpu_medium,
40,500 elements: 40 SIMP iterations each, penal 4.5 at the start, schedule-only
controller, four-level FP64 Chebyshev GMG, FGMRES restart 300, maxiter 300,
probe 100 / r50 at 50, floors 1e-12 | 1e-3, 1e-2) as
published_guarded_trajectories_{iters,summary}.csv, and its fixed-floor
trajectories (--policy fixed_floor, floors 1e-12, 1e-3 and 1e-2 on the same two
presets; simp_floor_trajectories__{cantilever,bridge}__*.csv) as
published_fixed_floor_trajectories_{cantilever,bridge}_{iters,summary}.csv.
"""

from __future__ import annotations

import os
import shutil

HERE = os.path.dirname(os.path.abspath(__file__))


def main() -> None:
    root = os.environ.get("SIMPFEM_REFERENCE_ROOT")
    if not root:
        raise SystemExit("set SIMPFEM_REFERENCE_ROOT to a checkout of the reference project")
    tables = os.path.join(root, "data", "analysis_tables")
    for name in ("iters", "summary"):
        shutil.copyfile(os.path.join(tables, f"guarded_adaptive_trajectories__trajectory_{name}.csv"),
                        os.path.join(HERE, f"published_guarded_trajectories_{name}.csv"))
        for preset in ("cantilever", "bridge"):
            shutil.copyfile(os.path.join(tables, f"simp_floor_trajectories__{preset}__trajectory_{name}.csv"),
                            os.path.join(HERE, f"published_fixed_floor_trajectories_{preset}_{name}.csv"))
    print("wrote published_{guarded,fixed_floor}_trajectories_*.csv")


if __name__ == "__main__":
    main()
