"""Host-side formats: input deck files, op files, norms, case generators."""
import os

import numpy as np

from piafs_b200 import cases, deck


def test_keyfile_roundtrip(tmp_path):
    p = tmp_path / "solver.inp"
    deck.write_keyfile(str(p), {"ndims": 2, "size": [64, 48], "dt": 0.5, "model": "navierstokes2d"})
    kv = deck.read_keyfile(str(p))
    assert kv["ndims"] == ["2"] and kv["size"] == ["64", "48"]
    assert float(kv["dt"][0]) == 0.5 and kv["model"] == ["navierstokes2d"]


def test_boundary_roundtrip(tmp_path):
    p = tmp_path / "boundary.inp"
    z = [deck.BoundaryZone("periodic", 0, 1, [0, 0, -1e99, 1e99]),
         deck.BoundaryZone("slip-wall", 1, -1, [-1e99, 1e99, 0, 0], [0.0, 0.25])]
    deck.write_boundary(str(p), z)
    back = deck.read_boundary(str(p), 2)
    assert [b.bctype for b in back] == ["periodic", "slip-wall"]
    assert back[1].face == -1 and back[1].wall_velocity == [0.0, 0.25]


def test_boundary_roundtrip_flow_zones(tmp_path):
    # zone data as InitializeBoundaries.c:106-168 reads it, 2D with 11 variables
    p = tmp_path / "boundary.inp"
    big = 1e99
    sc = [1.0, 0.005, 0, 0, 0, 0, 0]
    z = [deck.BoundaryZone("subsonic-inflow", 1, 1, [-big, big, 0, 0], values=[1.0, 0.0, 0.3] + sc),
         deck.BoundaryZone("subsonic-outflow", 1, -1, [-big, big, 0, 0], values=[0.7]),
         deck.BoundaryZone("noslip-wall", 0, 1, [0, 0, -big, big], [0.0, 0.1]),
         deck.BoundaryZone("supersonic-inflow", 0, -1, [0, 0, -big, big], values=[2.0, -1.5, 0.0, 3.0] + sc),
         deck.BoundaryZone("subsonic-ambivalent", 0, 1, [0, 0, -big, big], values=[1.0, 0.2, 0.0, 0.7]),
         deck.BoundaryZone("supersonic-outflow", 0, -1, [0, 0, -big, big]),
         deck.BoundaryZone("dirichlet", 1, 1, [-big, big, 0, 0], values=list(range(11)))]
    deck.write_boundary(str(p), z)
    back = deck.read_boundary(str(p), 2, nvars=11)
    assert [b.bctype for b in back] == [b.bctype for b in z]
    for a, b in zip(back, z):
        assert a.values == (None if b.values is None else [float(v) for v in b.values])
        assert a.wall_velocity == b.wall_velocity


def test_op_file_roundtrip(tmp_path):
    x, y = np.linspace(0, 1, 5), np.linspace(0, 2, 3)
    u = np.arange(15 * 4, dtype=np.float64).reshape(15, 4)
    p = str(tmp_path / deck.op_filename(7))
    assert p.endswith("op_00007.bin")
    deck.write_op(p, [x, y], u)
    op = deck.read_op(p)
    assert op.ndims == 2 and op.nvars == 4 and list(op.size) == [5, 3]
    assert np.array_equal(op.u, u) and np.array_equal(op.grid[1], y)


def test_rel_norms_follow_comparesolutions():
    ref = np.array([[1.0, 0.0], [3.0, 0.0]])
    u = np.array([[1.5, 1e-3], [3.0, 0.0]])
    n = deck.rel_norms(u, ref)
    # var 0: L1 = 0.25/2 ; ref L1 = 2 ; var 1: reference norm 0 -> absolute
    assert abs(n[0][0] - 0.125) < 1e-15 and abs(n[1][0] - 5e-4) < 1e-15
    assert abs(n[0][2] - 0.5 / 3.0) < 1e-15


def test_case_generators_write_complete_decks(tmp_path):
    m = cases.ns2d_photochem_beam(str(tmp_path / "c2"), N=16, NY=12, n_iter=3)
    files = set(os.listdir(tmp_path / "c2"))
    assert {"solver.inp", "boundary.inp", "physics.inp", "chemistry.inp", "imap.inp", "initial.inp"} <= files
    # dt from CFL 0.4 at t = 0 with sound speed sqrt(gamma p / rho) = 1
    assert abs(m["dt"] - 0.4 / 16) / m["dt"] < 2e-6
    g, u = deck.read_array_binary(str(tmp_path / "c2" / "initial.inp"), [16, 12], 11)
    assert abs(u[:, 3].mean() - (1 / m["gamma"]) / (m["gamma"] - 1)) < 1e-12
    assert 0.5 <= m["beam_amp"] <= 1.5
    m1 = cases.euler1d_density_wave(str(tmp_path / "c1"), N=32, n_iter=2)
    g, u = deck.read_array_binary(str(tmp_path / "c1" / "initial.inp"), [32], 3)
    assert np.allclose(u[:, 0], 1 + 0.2 * np.sin(2 * np.pi * g[0]))


def test_seeded_generators_are_deterministic(tmp_path):
    cases.ns2d_photochem_beam(str(tmp_path / "a"), N=8, n_iter=1)
    cases.ns2d_photochem_beam(str(tmp_path / "b"), N=8, n_iter=1)
    a = open(tmp_path / "a" / "initial.inp", "rb").read()
    b = open(tmp_path / "b" / "initial.inp", "rb").read()
    assert a == b
