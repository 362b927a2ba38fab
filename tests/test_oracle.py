"""The CPU oracle (oracle/piafs_oracle.c) against the reference's own outputs.

Each golden fixture is a deck plus the final solution the reference binary
wrote for it (tests/golden/make_golden.py).  The restatement follows the
reference's arithmetic order and is built with the same flags, so agreement
is required bit for bit: this pins the oracle the GPU parity tests use.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases
from oracle import oracle
from piafs_b200 import deck


@pytest.mark.parametrize("name", golden_cases(oracle_scope=True))
def test_oracle_matches_reference_bitwise(name):
    d = os.path.join(GOLDEN, name)
    case = oracle.load(d)
    u = case.run()
    ref = deck.read_op(os.path.join(d, "ref_final.bin"))
    got = case.interior(u)
    assert ref.u.shape == got.shape
    assert np.array_equal(got, ref.u), np.abs(got - ref.u).max()


def test_oracle_tridiag_matches_dense_solve():
    rng = np.random.default_rng(5)
    n, ns = 17, 5
    a = rng.uniform(-1, 1, (n, ns)); c = rng.uniform(-1, 1, (n, ns))
    b = 4 + rng.uniform(0, 1, (n, ns)); x = rng.uniform(-1, 1, (n, ns))
    a[0] = 0; c[-1] = 0
    M = [np.diag(b[:, k]) + np.diag(a[1:, k], -1) + np.diag(c[:-1, k], 1) for k in range(ns)]
    want = np.stack([np.linalg.solve(M[k], x[:, k]) for k in range(ns)], axis=1)
    A, B, Cc, X = (np.ascontiguousarray(v) for v in (a, b, c, x))
    oracle.lib().orc_tridiag(oracle._dp(A), oracle._dp(B), oracle._dp(Cc), oracle._dp(X), n, ns)
    np.testing.assert_allclose(X, want, rtol=1e-12, atol=1e-13)


def test_oracle_derives_chemistry_parameters():
    case = oracle.load(os.path.join(GOLDEN, "ns2d_chem_crweno5_llf_64x48"))
    # theta = 4.2117e-5 realises Re = 1e4; gamma and Pr follow the O2 gas
    assert abs(case.Re - 1e4) / 1e4 < 1e-5
    assert abs(case.gamma - 1.413) < 1e-12
    assert abs(case.Pr - 0.65167) < 1e-4
    assert case.P.bc_gamma == 1.4          # walls keep the physics.inp gamma


def test_oracle_conserves_mass_periodic_1d():
    case = oracle.load(os.path.join(GOLDEN, "euler1d_weno5_roe_n1024"))
    u0 = case.interior(case.u0)
    u = case.interior(case.run(nsteps=50))
    assert abs(u[:, 0].sum() - u0[:, 0].sum()) / u0[:, 0].sum() < 1e-13
