"""The column grouping of the block-sparse buildMatrix (src/linearSolver.c:
186-252): a distance-3 colouring of the face-neighbour graph, host only.

* Valid: no two cells within three face-neighbour steps share a colour (the
  condition under which one residual pass yields each grouped column's
  entries in the rows of its cell and of its face neighbours exactly).
* Few: the tabu-search refinement takes the greedy colouring of an airfoil
  O-grid with an odd number of cells around (12 colours) to at most 10, and
  keeps the 8 of the 256 x 128 NACA 0012 grid, which is optimal (eight cells
  of a quad grid lie pairwise within three steps).
* Deterministic: the same colouring on every call.
"""
import os
import tempfile

import numpy as np
import pytest

import ccfd_b200 as cc
from ccfd_b200 import meshgen, workloads


def _balls(off, nb):
    n = len(off) - 1
    out = []
    for d in range(n):
        seen = {d}
        frontier = [d]
        for _ in range(3):
            nxt = []
            for c in frontier:
                for h in range(off[c], off[c + 1]):
                    e = nb[h]
                    if e >= 0 and e not in seen:
                        seen.add(e)
                        nxt.append(e)
            frontier = nxt
        seen.discard(d)
        out.append(seen)
    return out


def _check_valid(off, nb, color):
    for d, ball in enumerate(_balls(off.tolist(), nb.tolist())):
        assert all(color[e] != color[d] for e in ball), d


def _mesh(case):
    m = case.mesh()
    return m["hs_offset"], m["hs_nb"]


def test_small_meshes_valid_and_deterministic():
    with tempfile.TemporaryDirectory() as tmp:
        meshgen.naca_ogrid(0.0, 0.0, 0.12, 33, 12, r_far=5.0, h0=1e-2, wall_code=101).write_gmsh(
            os.path.join(tmp, "af.msh"))
        case = cc.CaseData.from_text(meshgen.airfoil_ini("af", implicit=True, precond=True), tmp)
    off, nb = _mesh(case)
    c0, n0 = cc.colour_cells(off, nb, budget=0)
    c1, n1 = cc.colour_cells(off, nb)
    c2, n2 = cc.colour_cells(off, nb)
    _check_valid(off, nb, c0)
    _check_valid(off, nb, c1)
    assert n1 <= n0 and c1.max() == n1 - 1 and len(np.unique(c1)) == n1
    assert n1 == n2 and np.array_equal(c1, c2)


def test_empty_and_bad_arguments():
    c, n = cc.colour_cells(np.zeros(1, np.int64), np.zeros(0, np.int64))
    assert n == 0 and len(c) == 0
    with pytest.raises(cc.CcfdError):
        cc.colour_cells(np.array([0, 1], np.int64), np.array([5], np.int64))
    # offsets must start at zero and never decrease
    with pytest.raises(cc.CcfdError):
        cc.colour_cells(np.array([0, 2, 1], np.int64), np.array([1, -1], np.int64))
    with pytest.raises(cc.CcfdError):
        cc.colour_cells(np.array([1, 2], np.int64), np.array([-1, -1], np.int64))


def test_batched_airfoil_grid_takes_at_most_ten_colours():
    spec = workloads.airfoil_specs(1)[0]
    with tempfile.TemporaryDirectory() as tmp:
        case = workloads.airfoil_case(spec, tmp, "af0")
    off, nb = _mesh(case)
    assert (spec["ni"] % 2) == 1
    _, n_greedy = cc.colour_cells(off, nb, budget=0)
    color, n = cc.colour_cells(off, nb)
    assert n_greedy == 12 and n <= 10
    _check_valid(off, nb, color)


def test_naca0012_grid_keeps_eight_colours():
    with tempfile.TemporaryDirectory() as tmp:
        meshgen.naca_ogrid(0.0, 0.0, 0.12, 256, 128, r_far=20.0, h0=1e-4, wall_code=201).write_gmsh(
            os.path.join(tmp, "af.msh"))
        case = cc.CaseData.from_text(meshgen.airfoil_ini("af", navier_stokes=True, implicit=True, precond=True),
                                     tmp)
    off, nb = _mesh(case)
    color, n = cc.colour_cells(off, nb)
    assert n == 8
    _check_valid(off, nb, color)
