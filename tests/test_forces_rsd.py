"""The force set of writeResiduals and its residual-history output (CPU).

* forceCalcType 3 (calculateLiftAndDrag3, SolverSource/mgnsg3d_def_par.F90:
  15129-15313) in the CPU restatement, checked against a numpy restatement
  written from the Fortran: face loads scattered to the wall nodes, then the
  seven sums;
* the .rsd line (format 504) and the screen line (format 501) of
  writeResiduals (mgnsg3d_mg_par.F90:1449-1516), checked against lines
  spelled out by the Fortran edit descriptors;
* the host library's copy of the controls defaults equals the GPU
  library's.
"""
import ctypes
import math

import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import (Mesh, Solver, _abi, default_controls, host_controls, initial_state,
                          run_steady)
from flite3d_b200.mesh import cycle_line, rsd_line


def _forces3_numpy(c, mesh, p, wall_stress):
    """calculateLiftAndDrag3 from the Fortran (def_par:15150-15240, 15290-15296)."""
    xyz = mesh.array(1, "coords")
    bidx = mesh.array(1, "bnd_idx")
    bw = mesh.array(1, "bnd_w")
    reg, ind = mesh.array(1, "node_reg"), mesh.array(1, "node_ind")
    n = xyz.shape[1]
    help3 = np.zeros((3, n))
    pinf = 1.0 / (c.gamma * c.MachNumber * c.MachNumber)
    for i in range(bidx.shape[1]):
        i1, i2, face = bidx[0, i] - 1, bidx[1, i] - 1, bidx[2, i]
        if face == 1 or face == 9:
            if xyz[2, i1] > c.groundplane + 0.01 or xyz[2, i2] > c.groundplane + 0.01:
                help3[:, i1] += 4.0 * bw[:, i] * (p[i1] - pinf)
                help3[:, i2] += 4.0 * bw[:, i] * (p[i2] - pinf)
                if c.ReynoldsNumber > 0.0 and face == 1:
                    area = math.sqrt(float(np.sum(bw[:, i] ** 2)))
                    help3[:, i1] += 4.0 * wall_stress[:, i1] * area
                    help3[:, i2] += 4.0 * wall_stress[:, i2] * area
    a, b = math.radians(c.alpha), math.radians(c.beta)
    ft = np.array([math.cos(a) * math.cos(b), math.sin(b), math.sin(a)])
    fn1 = np.array([-ft[2], 0.0, ft[0]])
    fn2 = np.array([-ft[1], ft[0], 0.0])
    s = np.zeros(7)  # lift, drag, latF, latM, longMl, longMd, rollM
    for q in range(reg[0], reg[1] + 1):
        ip = ind[q - 1] - 1
        d = xyz[:, ip] - np.array(c.datum[:])
        h = help3[:, ip]
        s[0] += h @ fn1
        s[1] += h @ ft
        s[2] += h @ fn2
        s[3] += -d[0] * (h @ fn2) + d[1] * (h @ ft)
        s[4] += -d[0] * (h @ fn1)
        s[5] += d[2] * (h @ ft)
        s[6] += -d[1] * (h @ fn1) + d[2] * (h @ fn2)
    return 2.0 * s / c.referenceArea


@pytest.mark.parametrize("re", [0.0, 5000.0], ids=["inviscid", "laminar"])
def test_force_calc_type_3_matches_numpy(re):
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=2)
    c = default_controls(ReynoldsNumber=re, numberOfGridsToUse=2, fluxType=1, forceCalcType=3, alpha=2.5,
                         beta=1.0, wallsAreIsentropic=1)
    c.datum[0], c.datum[1], c.datum[2] = 1.5, 0.25, -0.1
    o = Solver(c, mesh, backend=oracle_backend())
    o.set_state(initial_state(c, mesh, perturb_seed=7, amplitude=0.05))
    o.start()
    for cyc in range(1, 4):
        o.cycle(cyc)
    f = o.forces()
    p = o.get_pressure(1)
    n = mesh.level(1).n_nodes
    ws = np.zeros((3, n))
    o.be.get_array(o._h, 1, b"wallStress", ws.ctypes.data_as(ctypes.c_void_p))
    expect = _forces3_numpy(c, mesh, p, ws)
    got = np.array([f[0], f[1], f[2], f[4], f[6], f[7], f[8]])
    np.testing.assert_allclose(got, expect, rtol=1e-11, atol=1e-14)
    assert abs(f[0]) > 1e-6 and abs(f[8]) > 1e-9
    # frictionDrag and longM stay calculateLiftAndDrag's: compare with type 1
    c1 = default_controls(ReynoldsNumber=re, numberOfGridsToUse=2, fluxType=1, forceCalcType=1, alpha=2.5,
                          beta=1.0, wallsAreIsentropic=1)
    c1.datum[0], c1.datum[1], c1.datum[2] = 1.5, 0.25, -0.1
    o1 = Solver(c1, mesh, backend=oracle_backend())
    o1.set_state(initial_state(c1, mesh, perturb_seed=7, amplitude=0.05))
    o1.start()
    for cyc in range(1, 4):
        o1.cycle(cyc)
    f1 = o1.forces()
    assert f1[3] == f[3] and f1[5] == f[5]
    assert f1[6] == f1[7] == f1[8] == 0.0


def test_force_calc_type_2_is_refused():
    mesh = Mesh.bump_channel(4, 2, 2, 0.05, nlevels=1)
    c = default_controls(ReynoldsNumber=0.0, forceCalcType=2)
    with pytest.raises(RuntimeError, match="status 2"):
        Solver(c, mesh, backend=oracle_backend())


def test_rsd_line_follows_format_504():
    forces = [0.0123456, -0.00123456, 1.5, 2.25e-3, -3.75, 10.0, 0.0, 0.0, 0.0]
    res = [1e-3, 2e-4, 3e-5, 4e-6, 5e-7]
    line = rsd_line(12, 1e-3, 1.0, forces, res)
    expect = ("     12" + "  -0.30000E+01" + "   0.12346E-01" + "  -0.12346E-02"
              + "     1.500000 " + "     0.002250 " + "    -3.750000 " + "    10.000000 "
              + "    -3.698970 " + "    -4.522879 " + "    -5.397940 " + "    -6.301030 ")
    assert line == expect
    # forceCalcType 3: longMl, longMd, rollM in place of longM and the norms
    forces3 = forces[:6] + [0.5, -0.25, 1234567.0]
    line3 = rsd_line(3, 1.0, 1.0, forces3, res, force_calc_type=3)
    assert line3 == ("      3" + "   0.00000E+00" + "   0.12346E-01" + "  -0.12346E-02"
                     + "     1.500000 " + "     0.002250 " + "    -3.750000 " + "     0.500000 "
                     + "    -0.250000 " + "*************" + " ")
    # below a 1e-15 reduction currentRes is -100 (mg_par:1474-1478)
    assert rsd_line(9, 1e-20, 1.0, forces, res)[7:21] == "  -0.43429E+02"


def test_cycle_line_follows_format_501():
    line = cycle_line(7, [2.0, 4.0, 6.0, 8.0, 10.0], [0.5, 0.25, 0.126, 1e-7, 0.0], 0.5, 0.01234567, -1.5e-5)
    expect = ("      7"
              + "   0.10000E+01 (0.50E+00) " + "   0.20000E+01 (0.25E+00) "
              + "   0.30000E+01 (0.13E+00) " + "   0.40000E+01 (0.10E-06) "
              + "   0.50000E+01 (0.00E+00) " + "  0.1235E-01" + " -0.1500E-04")
    assert line == expect


def test_run_steady_writes_the_residual_history(tmp_path):
    mesh = Mesh.bump_channel(8, 4, 4, 0.05, nlevels=2)
    c = default_controls(ReynoldsNumber=0.0, numberOfGridsToUse=2, fluxType=1)
    o = Solver(c, mesh, backend=oracle_backend())
    o.set_state(initial_state(c, mesh, perturb_seed=3))
    o.start()
    path = tmp_path / "case.rsd"
    screen = []
    hist = run_steady(o, orders=8.0, max_cycles=4, rsd=path, screen=screen.append)
    lines = path.read_text().splitlines()
    assert len(lines) == len(hist) == len(screen) == 4
    assert [int(ln[:7]) for ln in lines] == [1, 2, 3, 4]
    assert lines[0][7:21] == "   0.00000E+00"
    r = [h[1] for h in hist]
    assert float(lines[-1][7:21]) == pytest.approx(math.log10(r[-1] / r[0]), abs=1e-5)
    assert float(lines[-1][21:35]) == pytest.approx(hist[-1][2], rel=1e-4, abs=1e-12)


def test_host_controls_equal_gpu_library_controls():
    for kw in ({}, dict(MachNumber=0.8, alpha=1.25, ReynoldsNumber=6e6, fluxType=4)):
        a, b = default_controls(**kw), host_controls(**kw)
        assert bytes(a) == bytes(b)
    assert ctypes.sizeof(_abi.Controls) == len(bytes(host_controls()))
