"""Multi-domain .sol files (parallel runs of the reference) on the CPU: gen3d's
greedy partition, the per-domain writer (writeParallelComputationFiles) and
the ingest that merges the domains into one mesh.

* a one-domain file set is byte for byte the single-domain .sol;
* the files of 2, 3 and 4 domains (bump channel with three levels, NACA
  O-grid with two, a moving mesh's GCL records) ingest to exactly the
  canonical form of the mesh they were written from, on every level;
* the canonical form is a fixed point and keeps the discretisation: a few
  multigrid cycles of the CPU restatement agree with the original ordering
  to round-off.
"""
import filecmp

import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, host_controls, initial_state

NAMES = ["side_idx", "side_w", "side_len", "bnd_idx", "bnd_w", "node_reg", "node_ind", "volume", "wall_dist"]


def assert_same_mesh(a, b, moving=False):
    assert a.nlevels == b.nlevels
    for level in range(1, a.nlevels + 1):
        names = NAMES + (["parent", "rweight"] if level > 1 else ["coords"])
        if moving:
            names += ["side_gcl", "bnd_gcl"] + (["volume_prev", "volume_prev2"] if level == 1 else [])
        for name in names:
            x, y = a.array(level, name), b.array(level, name)
            assert x is not None and y is not None, (level, name)
            assert x.shape == y.shape and np.array_equal(x, y), (level, name)


@pytest.fixture(scope="module")
def bump():
    m = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    yield m
    m.close()


def test_partition_covers_every_node(bump):
    for nd in (2, 3, 4):
        col = bump.partition(nd)
        counts = np.bincount(col)[1:]
        assert col.min() == 1 and len(counts) == nd and counts.min() > 0
        assert counts.max() < 2.0 * counts.min()


def test_one_domain_is_the_single_domain_file(bump, tmp_path):
    single = tmp_path / "single.sol"
    bump.write_sol(single)
    bump.write_sol_domains(tmp_path / "par", tmp_path / "plotreg.reg", 1)
    assert filecmp.cmp(single, str(tmp_path / "par") + ".sol_1", shallow=False)


@pytest.mark.parametrize("nd", [2, 3, 4])
def test_domains_ingest_to_the_canonical_mesh(bump, tmp_path, nd):
    bump.write_sol_domains(tmp_path / "bump", tmp_path / "plotreg.reg", nd)
    merged = Mesh.read_sol_domains(tmp_path / "bump", tmp_path / "plotreg.reg")
    canon = bump.canonical()
    try:
        assert_same_mesh(merged, canon)
    finally:
        merged.close()
        canon.close()


def test_given_colours_and_an_o_grid(tmp_path):
    m = Mesh.naca0012(24, 8, 4, first_cell=1e-3, nlayer=6, farfield=8.0, nlevels=2)
    try:
        n = m.level(1).n_nodes
        col = (np.arange(n) % 3 + 1).astype(np.int32)  # scattered domains: many crossing sides
        m.write_sol_domains(tmp_path / "naca", tmp_path / "plotreg.reg", 3, color=col)
        merged = Mesh.read_sol_domains(tmp_path / "naca", tmp_path / "plotreg.reg")
        canon = m.canonical()
        assert_same_mesh(merged, canon)
        merged.close()
        canon.close()
    finally:
        m.close()


def test_moving_mesh_domains(tmp_path):
    m = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=2)
    try:
        x0 = m.array(1, "coords")
        xs = [x0 + t * np.array([[0.01], [0.02], [-0.015]]) * np.sin(np.pi * x0[0] / 3.0) for t in (2, 1, 0)]
        m.set_moving(*xs, 2)
        m.write_sol_domains(tmp_path / "mv", tmp_path / "plotreg.reg", 2)
        merged = Mesh.read_sol_domains(tmp_path / "mv", tmp_path / "plotreg.reg")
        canon = m.canonical()
        assert_same_mesh(merged, canon, moving=True)
        assert np.abs(merged.array(1, "side_gcl")).max() > 0
        merged.close()
        canon.close()
    finally:
        m.close()


def test_canonical_form_is_a_fixed_point_and_keeps_the_solution(bump):
    c1 = bump.canonical()
    c2 = c1.canonical()
    assert_same_mesh(c1, c2)
    ctl = host_controls(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, numberOfGridsToUse=3)
    u0 = initial_state(ctl, bump, perturb_seed=11, amplitude=0.02)
    runs = []
    for mesh in (bump, c1):
        s = Solver(ctl, mesh, backend=oracle_backend())
        s.set_state(u0)
        s.start()
        for cyc in range(1, 4):
            s.cycle(cyc)
        runs.append(s.get_state(1))
        s.close()
    # level-1 nodes keep their numbers; only the order of the sums differs
    assert np.allclose(runs[0], runs[1], rtol=1e-10, atol=1e-12)
    assert not np.array_equal(runs[0], u0)
    c1.close()
    c2.close()
