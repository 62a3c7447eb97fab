"""GPU parity of the single-component path through the C ABI (liblbmgpu.so).

The CUDA path is compared with (a) fields produced by the reference's own solver
(tests/golden/sc_*.npz) and (b) the C oracle run on the same seeded inputs.
Tolerance: FP64 throughout; 1e-12 relative (to the field's max magnitude) for the short
runs, 1e-10 relative after 1000 steps of the 64^3 Taylor-Green vortex.
"""
import hashlib
import os

import numpy as np
import pytest

import lbmgpu
from oracle import cases, sc

pytestmark = pytest.mark.gpu
FIELDS = ["rho", "u", "v", "w", "temp", "p"]


def _cmp(got, ref, rtol, what="", scale=None):
    """max |got - ref| relative to the field's magnitude (or to `scale`: velocity
    components are measured against the largest velocity component)."""
    scale = max(np.max(np.abs(ref)) if scale is None else scale, 1e-300)
    err = np.max(np.abs(got - ref)) / scale
    assert err <= rtol, f"{what}: max |diff|/scale = {err:.3e} > {rtol}"


def _vscale(gold, cp, sel=Ellipsis):
    return max(np.max(np.abs(gold[f"{c}_{cp}"][sel])) for c in "uvw")


def _lattice(cells, params):
    Nx, Ny, Nz = cells.shape
    return lbmgpu.Lattice(Nx, Ny, Nz, params["nu"], params["R"], params["gamma"], params["prtl"])


def _gpu_run(cells, params, checkpoints, phases=False):
    lat = _lattice(cells, params)
    lat.upload(cells)
    lat.init()
    out = {}
    done = 0
    for cp in checkpoints:
        if phases:
            for _ in range(cp - done):
                lat.collide()
                lat.streaming()
                lat.tms_bc()
                lat.calculate_moment()
        else:
            lat.step(cp - done)
        done = cp
        st = lat.synchronize()
        assert st == 0, f"device status {st:#x}"
        c = cells.copy()
        lat.download(c)
        out[cp] = c
    lat.close()
    return out


CASES = {
    "sc_tgv12.npz": (lambda: cases.tgv_sc(12, Re=10.0), [1, 50]),
    "sc_channel.npz": (lambda: cases.channel_sc(), [1, 40]),
    "sc_channel_fs.npz": (lambda: cases.channel_sc(freeslip_z=True), [1, 40]),
}


@pytest.mark.parametrize("fixture", sorted(CASES))
def test_gpu_matches_reference_fixture(golden_dir, fixture):
    make, cps = CASES[fixture]
    cells, params = make()
    gold = np.load(os.path.join(golden_dir, fixture))
    assert hashlib.sha256(np.ascontiguousarray(cells).tobytes()).hexdigest() == str(gold["input_sha256"])
    res = _gpu_run(cells, params, cps)
    fl = cells["type"] == cases.TYPE_F
    idx = tuple(gold["pop_cells"].T)
    for cp in cps:
        c = res[cp]
        for f in FIELDS:
            _cmp(c[f][fl], gold[f"{f}_{cp}"][fl], 1e-12, f"{fixture} {f} step {cp}",
                 _vscale(gold, cp, fl) if f in "uvw" else None)
        for f in ("f", "g", "fpc", "gpc", "p_tensor", "rhoe"):
            _cmp(c[f][idx], gold[f"{f}_{cp}"], 1e-12, f"{fixture} {f} step {cp}")


def test_gpu_phase_calls_match_oracle():
    """The reference's per-phase call sequence through the ABI against the C oracle, with
    every population, on a non-cubic box (all boundary types)."""
    cells, params = cases.channel_sc(NX=20, NY=9, NZ=7)
    res = _gpu_run(cells, params, [3, 17], phases=True)
    a = cells.copy()
    o = sc.OracleSC(a, params["nu"], params["R"], params["gamma"], params["prtl"])
    o.init()
    o.loop(3)
    fl = cells["type"] == cases.TYPE_F

    def vs(c):
        return max(np.max(np.abs(c[k][fl])) for k in "uvw")

    for f in FIELDS + ["f", "g", "fpc", "gpc", "p_tensor", "rhoe", "energy_flux"]:
        _cmp(res[3][f][fl], a[f][fl], 1e-12, f, vs(a) if f in "uvw" else None)
    o.loop(14)
    for f in FIELDS + ["f", "g", "fpc", "gpc"]:
        _cmp(res[17][f][fl], a[f][fl], 1e-12, f, vs(a) if f in "uvw" else None)


def test_gpu_phase_order_enforced():
    cells, params = cases.tgv_sc(8, Re=10.0)
    with _lattice(cells, params) as lat:
        with pytest.raises(lbmgpu.LbmGpuError):
            lat.collide()  # nothing uploaded yet
        lat.upload(cells)
        lat.init()
        with pytest.raises(lbmgpu.LbmGpuError):
            lat.streaming()
        lat.collide()
        with pytest.raises(lbmgpu.LbmGpuError):
            lat.calculate_moment()
        with pytest.raises(lbmgpu.LbmGpuError):
            lat.download(cells.copy())  # mid-step
        lat.streaming()
        lat.tms_bc()
        lat.calculate_moment()
        lat.step(2)
        assert lat.synchronize() == 0


def test_gpu_restart_roundtrip():
    """Download mid-run, upload into a fresh handle, continue: identical to running on
    (the reference's restart: the next Collide uses the stored f and moments)."""
    cells, params = cases.channel_sc(NX=16, NY=8, NZ=6)
    a = _gpu_run(cells, params, [10])[10]
    with _lattice(cells, params) as lat:
        lat.upload(cells)
        lat.init()
        lat.step(10)
        mid = cells.copy()
        lat.download(mid)
        lat.step(7)
        end_a = cells.copy()
        lat.download(end_a)
    with _lattice(cells, params) as lat2:
        lat2.upload(mid)
        lat2.step(7)
        end_b = cells.copy()
        lat2.download(end_b)
    fl = cells["type"] == cases.TYPE_F
    for f in FIELDS:
        np.testing.assert_array_equal(a[f][fl], mid[f][fl])
    # the restarted run has the same populations; its first collision uses the stored
    # moments, as the reference's own restart does
    vsc = max(np.max(np.abs(end_a[k][fl])) for k in "uvw")
    for f in FIELDS + ["f", "g"]:
        _cmp(end_b[f][fl], end_a[f][fl], 1e-12, f, vsc if f in "uvw" else None)


def test_gpu_tgv64_1000_steps_matches_reference():
    """Config 1: 64^3 periodic TGV, Ma 0.1, Re 400, FP64, 1000 steps, against the
    reference's own fields (every 4th cell per axis) and whole-field sums."""
    cells, params = cases.tgv_sc(64)
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "sc_tgv64.npz"))
    assert hashlib.sha256(np.ascontiguousarray(cells).tobytes()).hexdigest() == str(gold["input_sha256"])
    res = _gpu_run(cells, params, [100, 1000])
    sample = (slice(1, 65, 4), slice(1, 65, 4), slice(1, 65, 4))
    fl = cells["type"] == cases.TYPE_F
    for cp in (100, 1000):
        c = res[cp]
        for f in FIELDS:
            _cmp(c[sample][f], gold[f"{f}_{cp}"], 1e-10, f"{f} step {cp}", _vscale(gold, cp) if f in "uvw" else None)
        np.testing.assert_allclose(np.sum(c["rho"][fl]), gold[f"sum_mass_{cp}"], rtol=1e-12)
        ke = 0.5 * np.sum(c["rho"][fl] * (c["u"][fl] ** 2 + c["v"][fl] ** 2 + c["w"][fl] ** 2))
        np.testing.assert_allclose(ke, gold[f"sum_ke_{cp}"], rtol=1e-10)
        np.testing.assert_allclose(np.sum(c["rhoe"][fl]), gold[f"sum_rhoe_{cp}"], rtol=1e-12)


def test_gpu_status_flags_on_injected_bad_state():
    """A state corrupted on the host before upload raises the device status bits
    (negative temperature -> tau and state flags) without any device fault."""
    cells, params = cases.tgv_sc(8, Re=10.0)
    bad = cells.copy()
    bad["temp"][4, 4, 4] = -0.5
    with _lattice(cells, params) as lat:
        lat.upload(bad)
        lat.init()
        lat.step(2)
        st = lat.synchronize()
        assert st & (lbmgpu.ST_TAU_UNSTABLE | lbmgpu.ST_NEG_STATE | lbmgpu.ST_NAN)
        assert lat.status(clear=True) == st
        assert lat.status() == 0
