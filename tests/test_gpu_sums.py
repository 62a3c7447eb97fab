"""lbmgpu_sums through the C ABI: the FP64 conserved totals over the fluid cells against
numpy sums of the downloaded state (single component: rho, rho u, rho (c_v T + |u|^2/2);
multicomponent: rho, rho u, rhoE, rho_a and the element totals), 1e-13 relative; and
bitwise reproducible from one call to the next."""
import numpy as np
import pytest

import lbmgpu
import mech
import workloads as W
from oracle import cases

pytestmark = pytest.mark.gpu


def _close(got, want, tol=1e-13):
    scale = max(abs(want), 1e-300)
    assert abs(got - want) / scale < tol, (got, want)


def test_gpu_sums_single_component():
    cells, prm = cases.tgv_sc(12, Re=10.0)
    with lbmgpu.Lattice(*cells.shape, prm["nu"], prm["R"], prm["gamma"], prm["prtl"]) as lat:
        lat.upload(cells)
        lat.init()
        lat.step(5)
        s1 = lat.sums()
        s2 = lat.sums()
        c = cells.copy()
        lat.download(c)
    assert s1 == s2
    fl = c["type"] == W.TYPE_F
    rho, u, v, w, T = (c[k][fl] for k in ("rho", "u", "v", "w", "temp"))
    cv = prm["R"] / (prm["gamma"] - 1.0)
    want = [rho.sum(), (rho * u).sum(), (rho * v).sum(), (rho * w).sum(),
            (rho * (cv * T + 0.5 * (u * u + v * v + w * w))).sum()]
    assert len(s1) == 5
    _close(s1[0], want[0])
    for k in (1, 2, 3):  # momentum sums of a vortex are near zero: compare to the mass scale
        assert abs(s1[k] - want[k]) < 1e-13 * abs(want[0])
    _close(s1[4], want[4])


def test_gpu_sums_multicomponent():
    m = mech.h2_air_9()
    mix, sp = W.flame_channel_mc(m, NX=10, NY=6, NZ=4)
    with lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=W.FLAME_UNITS,
                        chem=lbmgpu.CHEM_REF_EXPLICIT) as lat:
        lat.upload(mix, sp)
        lat.init()
        lat.step(3)
        s1 = lat.sums()
        s2 = lat.sums()
        c = mix.copy()
        s = [a.copy() for a in sp]
        lat.download(c, s)
    assert s1 == s2
    ns = len(sp)
    assert len(s1) == 5 + ns + 5
    fl = c["type"] == W.TYPE_F
    rho = c["rho"][fl]
    _close(s1[0], rho.sum())
    for k, f in ((1, "u"), (2, "v"), (3, "w")):
        assert abs(s1[k] - (rho * c[f][fl]).sum()) < 1e-13 * abs(rho.sum())
    _close(s1[4], c["rhoe"][fl].sum())
    el = np.zeros(5)
    for a in range(ns):
        ra = s[a]["rho"][fl]
        _close(s1[5 + a], ra.sum())
        el += (ra / m.W[a]).sum() * np.array([m.elements[a][e] for e in range(5)])
    for e in range(5):
        if el[e] == 0.0:
            assert s1[5 + ns + e] == 0.0
        else:
            _close(s1[5 + ns + e], el[e])
