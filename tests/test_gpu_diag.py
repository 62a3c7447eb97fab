"""lbmgpu_diagnostics through the C ABI against a numpy restatement of the reference's
OutputKeEns (src/output.cpp:212-275: sum rho|u|^2, sum rho|curl u|^2 with the wrapped
central differences, sum rho E over the fluid cells) on the downloaded state, plus the
heat-release sum and the temperature extremes; 1e-12 relative for the sums, exact for the
extremes; single component (Taylor-Green vortex) and reacting multicomponent channel."""
import numpy as np
import pytest

import lbmgpu
import mech
import workloads as W
from oracle import cases

pytestmark = pytest.mark.gpu


def _wrap(i, N):
    """output.cpp:235-249: lower neighbour wraps to N-2 below 1; only otherwise does the
    upper one wrap to 1 above N-2."""
    lo, hi = i - 1, i + 1
    low = lo < 1
    return np.where(low, N - 2, lo), np.where(~low & (hi > N - 2), 1, hi)


def keens(c, energy):
    Nx, Ny, Nz = c.shape
    I, J, K = np.nonzero(c["type"] == W.TYPE_F)
    u, v, w, rho = c["u"], c["v"], c["w"], c["rho"]
    ib, ia = _wrap(I, Nx)
    jb, ja = _wrap(J, Ny)
    kb, ka = _wrap(K, Nz)
    uy = (u[I, ja, K] - u[I, jb, K]) / 2
    uz = (u[I, J, ka] - u[I, J, kb]) / 2
    vx = (v[ia, J, K] - v[ib, J, K]) / 2
    vz = (v[I, J, ka] - v[I, J, kb]) / 2
    wx = (w[ia, J, K] - w[ib, J, K]) / 2
    wy = (w[I, ja, K] - w[I, jb, K]) / 2
    r = rho[I, J, K]
    uu = u[I, J, K] ** 2 + v[I, J, K] ** 2 + w[I, J, K] ** 2
    vort = (wy - vz) ** 2 + (uz - wx) ** 2 + (vx - uy) ** 2
    return (r * uu).sum(), (r * vort).sum(), energy[I, J, K].sum(), (I, J, K)


def _close(got, want, scale=None, tol=1e-12):
    scale = max(abs(want) if scale is None else scale, 1e-300)
    assert abs(got - want) <= tol * scale, (got, want)


def test_diagnostics_single_component():
    cells, prm = cases.tgv_sc(12, Re=10.0)
    with lbmgpu.Lattice(*cells.shape, prm["nu"], prm["R"], prm["gamma"], prm["prtl"]) as lat:
        lat.upload(cells)
        lat.init()
        lat.step(5)
        d1 = lat.diagnostics()
        d2 = lat.diagnostics()
        c = cells.copy()
        lat.download(c)
    assert d1 == d2
    cv = prm["R"] / (prm["gamma"] - 1.0)
    E = c["rho"] * (cv * c["temp"] + 0.5 * (c["u"] ** 2 + c["v"] ** 2 + c["w"] ** 2))
    ke, ens, en, idx = keens(c, E)
    assert ke > 0 and ens > 0
    _close(d1["kinetic"], ke)
    _close(d1["enstrophy"], ens)
    _close(d1["energy"], en)
    assert d1["hrr"] == 0.0
    assert d1["T_max"] == c["temp"][idx].max() and d1["T_min"] == c["temp"][idx].min()


def test_diagnostics_reacting_channel():
    m = mech.h2_air_9()
    mix, sp = W.flame_channel_mc(m, NX=16, NY=6, NZ=4)
    with lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=W.FLAME_UNITS,
                        chem=lbmgpu.CHEM_REF_EXPLICIT) as lat:
        lat.upload(mix, sp)
        lat.init()
        lat.step(3)
        d1 = lat.diagnostics()
        d2 = lat.diagnostics()
        c = mix.copy()
        s = [a.copy() for a in sp]
        lat.download(c, s)
    assert d1 == d2
    ke, ens, en, idx = keens(c, c["rhoe"])
    _close(d1["kinetic"], ke)
    _close(d1["enstrophy"], ens)
    _close(d1["energy"], en)
    hrr = c["HRR"][idx]
    assert np.abs(hrr).sum() > 0
    _close(d1["hrr"], hrr.sum(), scale=np.abs(hrr).sum())
    assert d1["T_max"] == c["temp"][idx].max() and d1["T_min"] == c["temp"][idx].min()
