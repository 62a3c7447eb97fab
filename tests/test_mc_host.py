"""The device's multicomponent per-cell functions (csrc/mc_cell.cuh), built for the host,
against the reference's own multicomponent solver (fixtures from oracle/_ref/libref_mc*.so
on the Cantera-API shim).  Same inputs, FP64, tolerance 1e-12 relative."""
import os

import numpy as np
import pytest

from mc_common import GOLDEN, NS, build_host_lib, case, digest, host_run, rel


@pytest.fixture(scope="module")
def hostlib(tmp_path_factory):
    return build_host_lib(tmp_path_factory.mktemp("mchost"))


@pytest.mark.parametrize("fixture", ["mc_mix8.npz", "mc_react8.npz"])
def test_host_cells_match_reference(hostlib, fixture):
    m, mix, sp, reaction, cps = case(fixture)
    gold = np.load(os.path.join(GOLDEN, fixture))
    assert digest(mix, sp) == str(gold["input_sha256"])
    fl = (mix["type"] == 0).reshape(-1)
    for cp in cps:
        R, st = host_run(hostlib, m, mix, sp, reaction, cp)
        assert st == 0
        assert rel(R[0][fl], gold[f"rho_{cp}"].reshape(-1)[fl]) < 1e-12
        vs = max(np.abs(gold[f"{k}_{cp}"].reshape(-1)[fl]).max() for k in "uvw")
        for q, k in ((1, "u"), (2, "v"), (3, "w")):
            assert rel(R[q][fl], gold[f"{k}_{cp}"].reshape(-1)[fl], vs) < 1e-12, k
        assert rel(R[4][fl], gold[f"temp_{cp}"].reshape(-1)[fl]) < 1e-12
        assert rel(R[5][fl], gold[f"p_{cp}"].reshape(-1)[fl]) < 1e-12
        assert rel(R[6][fl], gold[f"rhoe_{cp}"].reshape(-1)[fl]) < 1e-12
        for a in range(NS):
            assert rel(R[14 + 8 * a][fl], gold[f"sp_rho_{cp}"][a].reshape(-1)[fl]) < 1e-12, a
            assert rel(R[14 + 8 * a + 7][fl], gold[f"sp_X_{cp}"][a].reshape(-1)[fl]) < 1e-12, a
        if reaction:
            assert rel(R[13][fl], gold[f"HRR_{cp}"].reshape(-1)[fl]) < 1e-10
