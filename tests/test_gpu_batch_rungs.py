"""Uneven-size states in flight together, each solved at every floor rung
(gpu_fem.batch_rungs.RungBatch): every solve guarded, rows in state order, and
the result independent of thread scheduling -- two fresh batches on the same
states give bitwise-identical rows -- and equal to the same worker assignment
run one state at a time."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MESHES = ((20, 10, 10), (24, 12, 6), (16, 8, 8))


def _rows(cuda, width, states):
    from gpu_fem.batch_rungs import RungBatch

    return RungBatch(meshes=MESHES, width=width).run(states)


def test_rung_batch_is_deterministic_and_guarded(cuda):
    from gpu_fem.batch_rungs import make_states

    states = make_states(9, meshes=MESHES)
    a = _rows(cuda, 2, states)
    b = _rows(cuda, 2, states)
    assert len(a) == 27
    assert [r["state"] for r in a] == [s for s, _, _ in states for _ in range(3)]
    assert all(r["guarded"] == 1 and r["true_rel_residual"] <= 1e-6 for r in a)
    for x, y in zip(a, b):
        assert x["iters"] == y["iters"] and x["true_rel_residual"] == y["true_rel_residual"]


def test_rung_batch_matches_one_worker_per_mesh(cuda):
    from gpu_fem.batch_rungs import make_states

    states = make_states(6, meshes=MESHES)
    a = _rows(cuda, 1, states)
    # width 1: each mesh's states go to one worker in order, as a sequential run would
    from gpu_fem.batch_rungs import RungBatch

    seq = RungBatch(meshes=MESHES, width=1)
    rows = []
    for st in states:
        rows += seq.run([st])
    for x, y in zip(a, rows):
        assert x["iters"] == y["iters"] and x["true_rel_residual"] == y["true_rel_residual"]
