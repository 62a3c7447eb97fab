"""lbmgpu_sums_noalloc is for callers that may not allocate device memory once their run
is set up: a lattice sized to fill the GPU, a monitoring loop that must not stall other
streams through cudaMalloc's device-wide synchronisation, a host whose memory pool owns
the device.  Its reduction scratch is a fixed array of the library, loaded when a handle
is created.  Checked here through the C ABI against lbmgpu_sums (handle scratch) on the
same state: identical totals, bit for bit, on two calls in a row -- so the fixed scratch
carries nothing from one call into the next -- for a single-component and a
multicomponent handle; on a fresh handle whose first reduction is the no-alloc one,
neither the handle's device bytes nor the device's free memory move across the call; and
out-of-range sizes are rejected.  Collected last, so it also runs after every other GPU
test in the same process."""
import pytest

import lbmgpu
import mech
import workloads as W
from oracle import cases

pytestmark = pytest.mark.gpu


def _two_calls_agree(lat):
    for _ in range(2):
        want = lat.sums()
        got = lat.sums_noalloc()
        assert got == want
        lat.step(1)


def test_no_alloc_sums_match_single_component():
    cells, prm = cases.tgv_sc(12, Re=10.0)
    with lbmgpu.Lattice(*cells.shape, prm["nu"], prm["R"], prm["gamma"], prm["prtl"]) as lat:
        lat.upload(cells)
        lat.init()
        lat.step(2)
        _two_calls_agree(lat)


def test_no_alloc_sums_match_multicomponent():
    m = mech.h2_air_9()
    mix, sp = W.flame_channel_mc(m, NX=10, NY=6, NZ=4)
    with lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=W.FLAME_UNITS,
                        chem=lbmgpu.CHEM_REF_EXPLICIT) as lat:
        lat.upload(mix, sp)
        lat.init()
        lat.step(2)
        _two_calls_agree(lat)


def test_no_alloc_first_call_allocates_nothing():
    import torch
    cells, prm = cases.tgv_sc(12, Re=10.0)
    with lbmgpu.Lattice(*cells.shape, prm["nu"], prm["R"], prm["gamma"], prm["prtl"]) as lat:
        lat.upload(cells)
        lat.init()
        lat.step(2)
        lat.synchronize()
        held = lat.device_bytes()
        free0, _ = torch.cuda.mem_get_info(0)
        got = lat.sums_noalloc()
        free1, _ = torch.cuda.mem_get_info(0)
        assert lat.device_bytes() == held
        assert free1 == free0
        assert lat.sums() == got


def test_no_alloc_sums_reject_sizes():
    cells, prm = cases.tgv_sc(12, Re=10.0)
    with lbmgpu.Lattice(*cells.shape, prm["nu"], prm["R"], prm["gamma"], prm["prtl"]) as lat:
        lat.upload(cells)
        for n in (4, lbmgpu.SUMS_MAX + 1):
            with pytest.raises(lbmgpu.LbmGpuError):
                lat.sums_noalloc(n)
