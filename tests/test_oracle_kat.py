"""The C oracle's equilibria and FD stencils against known answers produced by the
reference's own functions (tests/golden/kat_sc.npz, made by make_golden.py)."""
import os

import numpy as np
import pytest

from oracle import refsc, sc


@pytest.fixture(scope="module")
def kat(golden_dir):
    return np.load(os.path.join(golden_dir, "kat_sc.npz"))


def test_feq_matches_reference(kat):
    got = np.array([sc.feq(int(l), r, u, t, c) for l, r, u, t, c in
                    zip(kat["L"], kat["rho"], kat["u"], kat["theta"], kat["corr"])])
    np.testing.assert_allclose(got, kat["feq"], rtol=1e-13, atol=1e-16)


def test_geq_factorised_equals_reference_polynomial(kat):
    got = np.array([sc.geq(int(l), r, U, t, u) for l, r, U, t, u in
                    zip(kat["L"], kat["rho"], kat["U"], kat["theta"], kat["u"])])
    np.testing.assert_allclose(got, kat["geq"], rtol=1e-12, atol=1e-14)
    for i in range(kat["geq_all"].shape[0]):
        row = [sc.geq(l, kat["rho"][i], kat["U"][i], kat["theta"][i], kat["u"][i]) for l in range(27)]
        np.testing.assert_allclose(row, kat["geq_all"][i], rtol=1e-12, atol=1e-14)


def test_geq_moment_form(kat):
    got = np.array([sc.geq_moment(int(l), re, q, R, t) for l, re, q, R, t in
                    zip(kat["L"], kat["rhoe"], kat["q"], kat["R"], kat["theta"])])
    np.testing.assert_allclose(got, kat["geq_moment"], rtol=1e-12, atol=1e-13)


def test_gstr(kat):
    got = np.array([sc.gstr(int(l), g, d) for l, g, d in zip(kat["L"], kat["geqv"], kat["dq"])])
    np.testing.assert_array_equal(got, kat["gstr"])


@pytest.mark.parametrize("name", ["fd_central", "fd_fuw"])
def test_fd_typed(kat, name):
    fn = getattr(sc, name)
    s = kat["fd_s"]
    got = np.array([fn(s[i, 0], s[i, 1], s[i, 2], 1.0, kat["fd_vel"][i], int(kat["fd_tl"][i]), int(kat["fd_tr"][i]))
                    for i in range(len(s))])
    np.testing.assert_array_equal(got, kat[name])


def test_fd_uw(kat):
    s = kat["fd_s"]
    got = np.array([sc.fd_uw(s[i, 0], s[i, 1], s[i, 2], 1.0, kat["fd_vel"][i]) for i in range(len(s))])
    np.testing.assert_array_equal(got, kat["fd_uw"])


def test_equilibrium_moments():
    """Moments the equilibria must reproduce (mass, momentum, total energy, energy flux)."""
    rng = np.random.Generator(np.random.PCG64(7))
    CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1])
    CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1])
    CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1])
    c = np.stack([CX, CY, CZ], 1)
    for _ in range(10):
        rho, U, th = rng.uniform(0.5, 2), rng.uniform(0.1, 1), rng.uniform(0.05, 0.3)
        u = rng.uniform(-0.1, 0.1, 3)
        f = np.array([sc.feq(l, rho, u, th, np.zeros(3)) for l in range(27)])
        g = np.array([sc.geq(l, rho, U, th, u) for l in range(27)])
        E = U + 0.5 * u @ u
        H = E + th
        np.testing.assert_allclose(f.sum(), rho, rtol=1e-13)
        np.testing.assert_allclose(c.T @ f, rho * u, rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(g.sum(), rho * E, rtol=1e-13)
        np.testing.assert_allclose(c.T @ g, rho * H * u, rtol=1e-12, atol=1e-15)
        P = np.einsum("l,la,lb->ab", f, c, c)
        np.testing.assert_allclose(P, rho * th * np.eye(3) + rho * np.outer(u, u), rtol=1e-12, atol=1e-15)


@pytest.mark.skipif(not refsc.available(), reason="reference library not built here")
def test_geq_against_reference_library_live():
    rng = np.random.Generator(np.random.PCG64(11))
    for _ in range(200):
        l = int(rng.integers(0, 27))
        rho, U, th = rng.uniform(0.5, 2), rng.uniform(0.1, 2), rng.uniform(0.01, 0.5)
        u = rng.uniform(-0.3, 0.3, 3)
        assert sc.geq(l, rho, U, th, u) == pytest.approx(refsc.geq_poly(l, rho, U, th, u), rel=1e-11, abs=1e-14)
