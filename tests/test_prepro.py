"""Preprocessor (gen3d tet-path restatement) and the reference file formats."""
import numpy as np
import pytest

from flite3d_b200 import Mesh, read_rst, write_rst, read_unk, write_unk, write_res
from flite3d_b200.mesh import density_perturbation, splitmix64


def test_bump_channel_counts_config1():
    # 48x16x16 hexes, Kuhn split: 14,161 nodes, 73,728 tets, 91,472 edges
    m = Mesh.bump_channel(48, 16, 16, 0.05, nlevels=3)
    s = m.sizes(1)
    assert s["nodes"] == 49 * 17 * 17 == 14161
    assert s["sides"] == 91472
    assert m.nlevels == 3


@pytest.mark.parametrize("level", [1, 2, 3])
def test_closure_and_volume(level):
    # the reference's own self-check (def_par:14430-14568, gen3d_grid.f90:
    # 3661-3697): sum_j +-w_ij + 2 sum_b w_b = 0 per node; and the control
    # volumes tile the domain: 3 - bump area (0.05 * 0.5 * 1)
    m = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    closure, vol = m.check(level)
    assert closure < 1e-12
    assert vol == pytest.approx(2.975, rel=1e-13)


def test_boundary_first_numbering_and_register():
    m = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=2)
    for level in (1, 2):
        d = m.level(level)
        reg = m.array(level, "node_reg")
        ind = m.array(level, "node_ind")
        bidx = m.array(level, "bnd_idx")
        # boundary edges only touch boundary nodes 1..Nb
        assert bidx[:2].max() <= d.n_bnodes
        # the register tiles 1..n_normals in indicator order
        assert reg[0] == 1
        assert reg[17] == d.n_normals  # end of indicator 9 at index -3
        assert sorted(ind.tolist()) == sorted(set(ind.tolist()))


def test_outward_boundary_weights():
    # the far-field Roe flux of def_par:2258-2346 is upwind only for outward
    # boundary coefficients; the inflow plane x=0 must have w_b.x < 0
    m = Mesh.bump_channel(12, 4, 4, 0.0, nlevels=1)
    bidx = m.array(1, "bnd_idx")
    bw = m.array(1, "bnd_w")
    xyz = m.array(1, "coords")
    far = bidx[2] == 3
    x1 = xyz[0, bidx[0, far] - 1]
    inflow = x1 == 0.0
    assert np.all(bw[0, far][inflow] < 0)
    assert np.all(bw[0, far][~inflow] > 0)


def test_agglomeration_operators():
    m = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    for level in (2, 3):
        par = m.array(level, "parent")
        w = m.array(level, "rweight")
        nc = m.level(level).n_nodes
        assert par.min() >= 1 and par.max() <= nc
        # restriction of a constant is the constant: weights sum to 1 per parent
        s = np.bincount(par - 1, weights=w, minlength=nc)
        assert np.allclose(s, 1.0, atol=1e-14)
        # coarse boundary nodes hold fine boundary nodes
        nbf = m.level(level - 1).n_bnodes
        assert par[:nbf].max() <= m.level(level).n_bnodes


def test_sol_round_trip(tmp_path):
    m = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=3)
    p = tmp_path / "case.sol_1"
    m.write_sol(p)
    r = Mesh.read_sol(p)
    assert r.nlevels == m.nlevels
    for level in range(1, m.nlevels + 1):
        for name in ("side_idx", "side_w", "side_len", "bnd_idx", "bnd_w", "node_reg", "node_ind",
                     "volume", "wall_dist"):
            a, b = m.array(level, name), r.array(level, name)
            assert np.array_equal(a, b), (level, name)
        if level > 1:
            assert np.array_equal(m.array(level, "parent"), r.array(level, "parent"))
            assert np.array_equal(m.array(level, "rweight"), r.array(level, "rweight"))
    assert np.array_equal(m.array(1, "coords"), r.array(1, "coords"))


def test_sol_rejects_corrupt_record(tmp_path):
    m = Mesh.bump_channel(6, 2, 2, 0.05, nlevels=2)
    p = tmp_path / "case.sol_1"
    m.write_sol(p)
    data = bytearray(p.read_bytes())
    data[40] ^= 0x7F  # break a record marker inside the boundary block
    bad = tmp_path / "bad.sol_1"
    bad.write_bytes(bytes(data))
    with pytest.raises(RuntimeError):
        Mesh.read_sol(bad)
    bad.write_bytes(bytes(p.read_bytes()[:1000]))
    with pytest.raises(RuntimeError):
        Mesh.read_sol(bad)


def test_restart_and_result_files(tmp_path):
    n = 57
    prim = np.vstack([1 + 0.01 * np.arange(n), np.full(n, 0.9), np.zeros(n), np.full(n, 0.1),
                      np.full(n, 7.6)])
    write_rst(tmp_path / "c.rst_1", prim)
    assert np.array_equal(read_rst(tmp_path / "c.rst_1", n), prim)
    with pytest.raises(RuntimeError):
        read_rst(tmp_path / "c.rst_1", n + 1)  # "Startup file is not compatible"
    write_unk(tmp_path / "c.unk", prim)
    assert np.array_equal(read_unk(tmp_path / "c.unk", n), prim)
    # .res holds rho and u_j/rho (def_par:15331-15345)
    u = prim.copy()
    u[1:] *= prim[0]
    write_res(tmp_path / "c.res_1", u)
    back = read_unk(tmp_path / "c.res_1", n)
    assert np.allclose(back, prim, rtol=1e-15)


def test_splitmix64_known_values():
    # published first outputs of SplitMix64 seeded with 1234567
    assert splitmix64(1234567, 3).tolist() == [6457827717110365317, 3203168211198807973,
                                                9817491932198370423]
    d = density_perturbation(1000)
    assert d.min() >= -0.01 and d.max() <= 0.01


def test_plt_and_plotreg(tmp_path):
    m = Mesh.bump_channel(6, 2, 2, 0.05, nlevels=1)
    m.write_plt(tmp_path / "base.plt")
    m.write_plotreg(tmp_path / "plotreg.reg")
    raw = (tmp_path / "base.plt").read_bytes()
    head = np.frombuffer(raw[4:16], dtype=np.int32)
    assert head.tolist() == [6 * 6 * 2 * 2, 7 * 3 * 3, 2 * (2 * 6 * 2 + 2 * 6 * 2 + 2 * 2 * 2)]


def test_naca0012_generator():
    from flite3d_b200 import Mesh
    m = Mesh.naca0012(64, 24, 4, first_cell=1e-3, growth=1.2, nlayer=10, farfield=10.0, span=0.5, nlevels=3)
    d = m.level(1)
    assert d.n_nodes == 64 * 25 * 5
    closure, volume = m.check(1)
    assert closure < 1e-13
    # the O-grid's polygonal far field of 64 sides, less the section, over the span
    poly = 0.5 * 64 * 10.0 ** 2 * np.sin(2 * np.pi / 64) * 0.5
    assert abs(volume - poly) < 0.01 * poly
    ind = set(int(v) for v in m.array(1, "bnd_idx").reshape(3, -1)[2])
    assert ind == {1, 2, 3}
    wd = m.array(1, "wall_dist")
    assert wd.min() >= 0.0 and wd.max() <= 10.5


def test_makeplot_merges_domains(tmp_path):
    """makeplot scatters each domain's result columns to the global nodes of
    plotreg.reg: one domain through the mesh's own register, and two
    hand-made domains that share a node."""
    from flite3d_b200.mesh import makeplot, write_res
    from flite3d_b200 import _abi
    import ctypes
    m = Mesh.bump_channel(6, 2, 2, 0.05, nlevels=1)
    n = m.level(1).n_nodes
    rng = np.random.default_rng(0)
    u = np.abs(rng.standard_normal((5, n))) + 1.0
    m.write_plotreg(tmp_path / "plotreg.reg")
    write_res(tmp_path / "case.res_1", u)
    makeplot(tmp_path / "plotreg.reg", tmp_path / "case.res_", 5, tmp_path / "case.unk")
    merged = read_unk(tmp_path / "case.unk", n, 5)
    perm = np.zeros(n, dtype=np.int32)
    _abi.check(_abi.prepro_lib().fp_node_perm(m._h, perm.ctypes.data_as(ctypes.c_void_p)), "fp_node_perm")
    res = np.vstack([u[:1], u[1:] / u[0]])  # what the result file holds
    assert np.array_equal(merged[:, perm - 1], res)
    # two domains of 3 local nodes over 5 global ones, node 3 in both
    import struct

    def rec(f, payload):
        f.write(struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload)))
    with open(tmp_path / "two.reg", "wb") as f:
        rec(f, struct.pack("<ii", 5, 2))
        for pairs in (((1, 1), (2, 2), (3, 3)), ((1, 3), (2, 4), (3, 5))):
            rec(f, struct.pack("<i", 3))
            for a, b in pairs:
                rec(f, struct.pack("<ii", a, b))
    parts = [np.arange(1, 16, dtype=float).reshape(5, 3), 100 + np.arange(1, 16, dtype=float).reshape(5, 3)]
    for d, x in enumerate(parts, 1):
        with open(tmp_path / f"two.res_{d}", "wb") as f:
            rec(f, struct.pack("<i", 3))
            rec(f, x.tobytes())
    makeplot(tmp_path / "two.reg", tmp_path / "two.res_", 5, tmp_path / "two.unk")
    got = read_unk(tmp_path / "two.unk", 5, 5)
    want = np.zeros((5, 5))
    want[:, 0:3] = parts[0]
    want[:, 2:5] = parts[1]  # the later domain writes node 3 last
    assert np.array_equal(got, want)
