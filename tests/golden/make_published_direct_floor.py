"""Fixtures from the reference's published direct-solve tables.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_published_direct_floor.py

Copies, from the reference's data/analysis_tables, the critical-floor table of
its run_direct_floor_atlas.py at the default arguments (cantilever_3d, seed 19,
solid probabilities 0.10-0.35, floors 1e-12-1e-3) as
published_direct_floor_critical_seed19.csv, and the seed-19 rows of its
run_direct_floor_conditioning.py table (floors 1e-12-1e-2) as
published_direct_floor_conditioning_seed19.csv.
"""

from __future__ import annotations

import csv
import os
import shutil

HERE = os.path.dirname(os.path.abspath(__file__))


def main() -> None:
    root = os.environ.get("SIMPFEM_REFERENCE_ROOT")
    if not root:
        raise SystemExit("set SIMPFEM_REFERENCE_ROOT to a checkout of the reference project")
    tables = os.path.join(root, "data", "analysis_tables")
    shutil.copyfile(os.path.join(tables, "direct_floor_atlas_seed19__direct_floor_critical.csv"),
                    os.path.join(HERE, "published_direct_floor_critical_seed19.csv"))
    with open(os.path.join(tables, "direct_floor_conditioning__direct_floor_conditioning.csv"), newline="") as f:
        rows = list(csv.DictReader(f))
    with open(os.path.join(HERE, "published_direct_floor_conditioning_seed19.csv"), "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=list(rows[0]))
        w.writeheader()
        w.writerows(r for r in rows if r["seed"] == "19")
    print("wrote published_direct_floor_{critical,conditioning}_seed19.csv")


if __name__ == "__main__":
    main()
