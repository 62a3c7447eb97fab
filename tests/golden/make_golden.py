"""Generates the golden fixtures in this directory from the reference's OWN code.

Run from the repository root (needs the reference tree, built by ``make -C oracle ref
REF=<reference tree>``):

    python tests/golden/make_golden.py --reference <reference tree>

(or with the tree in the LBM_REFERENCE environment variable).

It drives ``oracle/_ref/libref_sc.so`` -- the reference's single-component sources
compiled unchanged -- on seeded inputs and records:

* ``kat_sc.npz``           known answers of calculate_feq, calculate_geq (both forms),
                           calculate_gstr and the FD stencils on seeded random arguments;
* ``sc_tgv12.npz``         12^3 Taylor-Green vortex (Re 10), fields after 1 and 50 steps;
* ``sc_channel.npz``       24x10x8 channel with inflow/outflow/solid/adiabatic cells,
                           fields after 1 and 40 steps;
* ``sc_channel_fs.npz``    the same channel with free-slip z walls;
* ``sc_tgv64.npz``         the 64^3, Re 400, Ma 0.1 Taylor-Green vortex: fields on every
                           4th cell per axis and whole-field sums after 100 and 1000 steps;
* ``mc_mix8.npz``          8^3 periodic 9-species H2/air mixing layer (REACTION off), the
                           reference's multicomponent solver on the Cantera-API shim, fields
                           after 1 and 40 steps;
* ``mc_react8.npz``        the same with REACTION on and an 1800 K hot slab, 30 steps;
* ``mc_chan.npz``          10x6x4 reacting H2-air channel: characteristic outflow ghosts
                           (TYPE_O_C, NSCBC) at both x ends, TMS solid walls at y, periodic
                           z, an ignition kernel at mid-x; fields after 1, 2 and 20 steps;
* ``mc_inflow.npz``        10x6x6 mixing layer between a characteristic inflow (TYPE_I_C,
                           inline LODI) and outflow (TYPE_O_C), periodic y and z, REACTION
                           off; fields after 1, 2 and 20 steps.
* ``mc_flame512[_nofma].npz``  config 3's 512x8x8 reacting channel, 50 steps, and
  ``mc_inflow32[_nofma].npz``  a 32^3 slab of config 2, 20 steps (make_mc_shapes: sampled
                           cells and whole-field sums, both builds of the reference);
* ``mc_chan_nofma.npz``, ``mc_inflow_nofma.npz``  the same two cases run by the reference
                           built without floating-point contraction (-ffp-contract=off),
                           fields after 1, 2, 5, 10 and 20 steps.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import cases, refmc, refsc  # noqa: E402

sys.path.insert(0, os.path.join(ROOT, "lattice-boltzmann-method_b200"))
import mech as mechmod  # noqa: E402


def mech_path():
    """The reference's nh3.yaml (the 9-species H2/O2/N2 subset is extracted from it)."""
    ref = os.environ.get("LBM_REFERENCE")
    if "--reference" in sys.argv:
        ref = sys.argv[sys.argv.index("--reference") + 1]
    if not ref:
        raise SystemExit("make_golden.py: pass --reference <reference tree> or set LBM_REFERENCE")
    return os.path.join(ref, "src", "reaction-mech", "nh3.yaml")

MC_FIELDS = ["rho", "u", "v", "w", "temp", "p", "rhoe", "HRR"]

FIELDS = ["rho", "u", "v", "w", "temp", "p"]


def digest(cells):
    return hashlib.sha256(np.ascontiguousarray(cells).tobytes()).hexdigest()


def run_ref(cells, params, checkpoints, sample=None, pop_cells=None):
    NX, NY, NZ = [s - 2 for s in cells.shape]
    ref = refsc.RefSC(NX, NY, NZ, params["nu"], params["R"], params["gamma"], params["prtl"], cases.MIXTURE_SC)
    ref.cells[...] = cells
    ref.init()
    out = {}
    done = 0
    for cp in checkpoints:
        ref.loop(cp - done)
        done = cp
        c = ref.cells
        sel = c if sample is None else c[sample]
        for f in FIELDS:
            out[f"{f}_{cp}"] = np.ascontiguousarray(sel[f])
        fl = c["type"] == cases.TYPE_F
        out[f"sum_mass_{cp}"] = np.sum(c["rho"][fl])
        out[f"sum_ke_{cp}"] = 0.5 * np.sum(c["rho"][fl] * (c["u"][fl] ** 2 + c["v"][fl] ** 2 + c["w"][fl] ** 2))
        out[f"sum_rhoe_{cp}"] = np.sum(c["rhoe"][fl])
        if pop_cells is not None:
            idx = tuple(pop_cells.T)
            out[f"f_{cp}"] = np.ascontiguousarray(c["f"][idx])
            out[f"g_{cp}"] = np.ascontiguousarray(c["g"][idx])
            out[f"fpc_{cp}"] = np.ascontiguousarray(c["fpc"][idx])
            out[f"gpc_{cp}"] = np.ascontiguousarray(c["gpc"][idx])
            out[f"p_tensor_{cp}"] = np.ascontiguousarray(c["p_tensor"][idx])
            out[f"rhoe_{cp}"] = np.ascontiguousarray(c["rhoe"][idx])
    ref.close()
    return out


def pick_cells(cells, n, seed):
    fl = np.argwhere(cells["type"] == cases.TYPE_F)
    rng = np.random.Generator(np.random.PCG64(seed))
    return fl[rng.choice(len(fl), size=min(n, len(fl)), replace=False)]


def kat(seed=cases.SEED, n=64):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = {}
    # product-form feq and polynomial geq on physically plausible arguments
    L = rng.integers(0, 27, size=n)
    rho = rng.uniform(0.5, 2.0, size=n)
    u = rng.uniform(-0.2, 0.2, size=(n, 3))
    theta = rng.uniform(0.02, 0.4, size=n)
    corr = rng.uniform(-0.01, 0.01, size=(n, 3))
    U = rng.uniform(0.05, 2.0, size=n)
    out.update(L=L, rho=rho, u=u, theta=theta, corr=corr, U=U)
    out["feq"] = np.array([refsc.feq(int(L[i]), rho[i], u[i], theta[i], corr[i]) for i in range(n)])
    out["geq"] = np.array([refsc.geq_poly(int(L[i]), rho[i], U[i], theta[i], u[i]) for i in range(n)])
    # the whole 27-direction sets for a few states
    out["geq_all"] = np.array([[refsc.geq_poly(l, rho[i], U[i], theta[i], u[i]) for l in range(27)] for i in range(8)])
    out["feq_all"] = np.array([[refsc.feq(l, rho[i], u[i], theta[i], corr[i]) for l in range(27)] for i in range(8)])
    # moment-form geq on symmetric R
    rhoe = rng.uniform(0.5, 3.0, size=n)
    q = rng.uniform(-0.3, 0.3, size=(n, 3))
    A = rng.uniform(-0.2, 0.2, size=(n, 3, 3))
    R = np.einsum("nij,nkj->nik", A, A) + np.eye(3)[None] * rng.uniform(0.2, 1.0, size=(n, 1, 1))
    out.update(rhoe=rhoe, q=q, R=R)
    out["geq_moment"] = np.array([refsc.geq_moment(int(L[i]), rhoe[i], q[i], R[i], theta[i]) for i in range(n)])
    geqv = rng.uniform(-1, 1, size=n)
    dq = rng.uniform(-0.1, 0.1, size=(n, 3))
    out.update(geqv=geqv, dq=dq)
    out["gstr"] = np.array([refsc.gstr(int(L[i]), geqv[i], dq[i]) for i in range(n)])
    # FD stencils over every pair of neighbour types
    types = np.arange(10)
    tl, tr = np.meshgrid(types, types, indexing="ij")
    tl = tl.ravel()
    tr = tr.ravel()
    m = len(tl)
    s = rng.uniform(-1, 1, size=(m, 3))
    vel = rng.uniform(-0.1, 0.1, size=m)
    out.update(fd_tl=tl, fd_tr=tr, fd_s=s, fd_vel=vel)
    out["fd_central"] = np.array([refsc.fd_central(s[i, 0], s[i, 1], s[i, 2], 1.0, vel[i], int(tl[i]), int(tr[i]))
                                  for i in range(m)])
    out["fd_fuw"] = np.array([refsc.fd_fuw(s[i, 0], s[i, 1], s[i, 2], 1.0, vel[i], int(tl[i]), int(tr[i]))
                              for i in range(m)])
    out["fd_uw"] = np.array([refsc.fd_uw(s[i, 0], s[i, 1], s[i, 2], 1.0, vel[i]) for i in range(m)])
    return out


def run_ref_mc(mix, sp, m, checkpoints, reaction, pop_cells, variant=False):
    NX, NY, NZ = [s_ - 2 for s_ in mix.shape]
    refmc.set_threads(1 if variant == "nofma" else (os.cpu_count() or 1), reaction, variant)
    ref = refmc.RefMC(NX, NY, NZ, m, cases.FLAME_UNITS, cases.MIXTURE_MC, cases.SPECIES, reaction=reaction,
                      fast=variant)
    ref.cells[...] = mix
    for a in range(len(sp)):
        ref.species[a][...] = sp[a]
    ref.init()
    out = {}
    done = 0
    idx = tuple(pop_cells.T)
    for cp in checkpoints:
        ref.loop(cp - done)
        done = cp
        for f in MC_FIELDS:
            out[f"{f}_{cp}"] = np.ascontiguousarray(ref.cells[f])
        out[f"sp_rho_{cp}"] = np.stack([ref.species[a]["rho"] for a in range(len(sp))])
        out[f"sp_X_{cp}"] = np.stack([ref.species[a]["X"] for a in range(len(sp))])
        out[f"sp_u_{cp}"] = np.stack([ref.species[a]["u"] for a in range(len(sp))])
        out[f"sp_f_{cp}"] = np.stack([ref.species[a]["f"][idx] for a in range(len(sp))])
        out[f"sp_fpc_{cp}"] = np.stack([ref.species[a]["fpc"][idx] for a in range(len(sp))])
        out[f"g_{cp}"] = np.ascontiguousarray(ref.cells["g"][idx])
        out[f"p_tensor_{cp}"] = np.ascontiguousarray(ref.cells["p_tensor"][idx])
    ref.close()
    return out


def mc_digest(mix, sp):
    h = hashlib.sha256(np.ascontiguousarray(mix).tobytes())
    for a in sp:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    args = [a for i, a in enumerate(sys.argv[1:]) if a != "--reference" and sys.argv[i] != "--reference"]
    only = args[0] if args else "all"   # "sc", "mc", "mc_nofma", "mc_shapes", "mc_mechs" or "all"
    if only in ("all", "sc"):
        make_sc()
    if only in ("all", "mc"):
        make_mc()
    if only == "mc_nofma":
        make_mc_nofma()
    if only in ("all", "mc_shapes"):
        make_mc_shapes()
    if only in ("all", "mc_mechs"):
        make_mc_mechs()
    print("fixtures written to", HERE)


def make_sc():
    if not refsc.available():
        raise SystemExit("oracle/_ref/libref_sc.so missing: run `make -C oracle ref` first")
    refsc.set_threads(os.cpu_count() or 1)
    np.savez_compressed(os.path.join(HERE, "kat_sc.npz"), **kat())

    cells, params = cases.tgv_sc(12, Re=10.0)
    out = run_ref(cells, params, [1, 50], pop_cells=pick_cells(cells, 32, 1))
    out.update(input_sha256=digest(cells), pop_cells=pick_cells(cells, 32, 1))
    np.savez_compressed(os.path.join(HERE, "sc_tgv12.npz"), **out)

    for name, fs in (("sc_channel.npz", False), ("sc_channel_fs.npz", True)):
        cells, params = cases.channel_sc(freeslip_z=fs)
        pc = pick_cells(cells, 48, 2)
        out = run_ref(cells, params, [1, 40], pop_cells=pc)
        out.update(input_sha256=digest(cells), pop_cells=pc)
        np.savez_compressed(os.path.join(HERE, name), **out)

    cells, params = cases.tgv_sc(64)
    sample = (slice(1, 65, 4), slice(1, 65, 4), slice(1, 65, 4))
    out = run_ref(cells, params, [100, 1000], sample=sample)
    out.update(input_sha256=digest(cells))
    np.savez_compressed(os.path.join(HERE, "sc_tgv64.npz"), **out)


def make_mc():
    m = mechmod.h2_air_9()
    refmc.set_threads(os.cpu_count() or 1)
    for name, reaction, kw, cps in (("mc_mix8.npz", False, {}, [1, 40]),
                                    ("mc_react8.npz", True, {"T_hi": 1800.0}, [1, 30])):
        mix, sp = cases.mixing_layer_mc(m, N=8, **kw)
        pc = pick_cells(mix, 16, 3)
        out = run_ref_mc(mix, sp, m, cps, reaction, pc)
        out.update(input_sha256=mc_digest(mix, sp), pop_cells=pc)
        np.savez_compressed(os.path.join(HERE, name), **out)
    for name, mix_sp, reaction in (("mc_chan.npz", cases.flame_channel_mc(m, NX=10, NY=6, NZ=4), True),
                                   ("mc_inflow.npz", cases.inflow_layer_mc(m, NX=10, NY=6, NZ=6), False)):
        mix, sp = mix_sp
        pc = boundary_cells(mix, 24, 4)
        out = run_ref_mc(mix, sp, m, [1, 2, 20], reaction, pc)
        out.update(input_sha256=mc_digest(mix, sp), pop_cells=pc)
        np.savez_compressed(os.path.join(HERE, name), **out)
    make_mc_nofma()


def make_mc_mechs():
    """The reference's other mechanisms (6 species, two global steps with fractional reaction
    orders): a reacting 8^3 mixing layer, a fuel-laden 1800 K slab in air (5 % CH4 or C3H8 by
    mass), 30 steps."""
    for name, m, fuel in (("mc_ch4_react8.npz", mechmod.ch4_2s(), "CH4"),
                          ("mc_c3h8_react8.npz", mechmod.c3h8_2s(), "C3H8")):
        mix, sp = cases.mixing_layer_mc(m, N=8, T_hi=1800.0, fuel=fuel, Y_H2=0.05)
        pc = pick_cells(mix, 16, 3)
        out = run_ref_mc(mix, sp, m, [1, 30], True, pc)
        out.update(input_sha256=mc_digest(mix, sp), pop_cells=pc)
        np.savez_compressed(os.path.join(HERE, name), **out)


def make_mc_shapes():
    """Config 3's 512x8x8 reacting channel (50 steps) and a 32^3 slab of config 2 with its
    characteristic inflow and outflow (20 steps), each run by the reference built with
    floating-point contraction (the oracle) and without it (single-threaded): at every
    checkpoint the fields and species densities of 512 sampled fluid cells (256 next to a
    boundary, 256 anywhere) and the sums of rho, rhoE and each rho_a over all fluid cells."""
    m = mechmod.h2_air_9()
    for name, mix_sp, reaction, cps in (("mc_flame512", cases.flame_channel_mc(m, NX=512, NY=8, NZ=8), True,
                                         [1, 20, 50]),
                                        ("mc_inflow32", cases.inflow_layer_mc(m, NX=32, NY=32, NZ=32), False,
                                         [1, 20])):
        mix, sp = mix_sp
        t = mix["type"]
        fl = np.argwhere(t == cases.TYPE_F)
        rng = np.random.Generator(np.random.PCG64(7))
        near = np.array([bool(np.any((t[i - 1:i + 2, j - 1:j + 2, k - 1:k + 2] != cases.TYPE_F)
                                     & (t[i - 1:i + 2, j - 1:j + 2, k - 1:k + 2] != cases.TYPE_P)))
                         for (i, j, k) in fl])
        pick = np.concatenate([rng.choice(np.flatnonzero(near), 256, replace=False),
                               rng.choice(len(fl), 256, replace=False)])
        cells = fl[pick]
        idx = tuple(cells.T)
        mask = t == cases.TYPE_F
        for variant, suffix in ((False, ""), ("nofma", "_nofma")):
            NX, NY, NZ = [s_ - 2 for s_ in mix.shape]
            refmc.set_threads(1 if variant == "nofma" else (os.cpu_count() or 1), reaction, variant)
            ref = refmc.RefMC(NX, NY, NZ, m, cases.FLAME_UNITS, cases.MIXTURE_MC, cases.SPECIES, reaction=reaction,
                              fast=variant)
            ref.cells[...] = mix
            for a in range(len(sp)):
                ref.species[a][...] = sp[a]
            ref.init()
            out = {"input_sha256": mc_digest(mix, sp), "cells": cells, "checkpoints": np.array(cps)}
            done = 0
            for cp in cps:
                ref.loop(cp - done)
                done = cp
                for f in MC_FIELDS:
                    out[f"{f}_{cp}"] = np.ascontiguousarray(ref.cells[f][idx])
                out[f"sp_rho_{cp}"] = np.stack([ref.species[a]["rho"][idx] for a in range(len(sp))])
                out[f"sum_rho_{cp}"] = ref.cells["rho"][mask].sum()
                out[f"sum_rhoe_{cp}"] = ref.cells["rhoe"][mask].sum()
                out[f"sum_sp_rho_{cp}"] = np.array([ref.species[a]["rho"][mask].sum() for a in range(len(sp))])
            ref.close()
            np.savez_compressed(os.path.join(HERE, f"{name}{suffix}.npz"), **out)


def make_mc_nofma():
    """The boundary cases run by the reference built without floating-point contraction (no
    fused multiply-adds, oracle/_ref/libref_mc*_nofma.so), single-threaded."""
    m = mechmod.h2_air_9()
    for name, mix_sp, reaction in (("mc_chan_nofma.npz", cases.flame_channel_mc(m, NX=10, NY=6, NZ=4), True),
                                   ("mc_inflow_nofma.npz", cases.inflow_layer_mc(m, NX=10, NY=6, NZ=6), False)):
        mix, sp = mix_sp
        pc = boundary_cells(mix, 24, 4)
        out = run_ref_mc(mix, sp, m, [1, 2, 5, 10, 20], reaction, pc, variant="nofma")
        out.update(input_sha256=mc_digest(mix, sp), pop_cells=pc)
        np.savez_compressed(os.path.join(HERE, name), **out)


def boundary_cells(cells, n, seed):
    """Fluid cells for the population records: those next to a non-periodic ghost first."""
    t = cells["type"]
    fl = np.argwhere(t == cases.TYPE_F)
    near = []
    for (i, j, k) in fl:
        nb = t[i - 1:i + 2, j - 1:j + 2, k - 1:k + 2]
        near.append(bool(np.any((nb != cases.TYPE_F) & (nb != cases.TYPE_P))))
    near = np.array(near)
    rng = np.random.Generator(np.random.PCG64(seed))
    a = fl[near][rng.permutation(int(near.sum()))][: n // 2 + n % 2]
    b = fl[~near][rng.permutation(int((~near).sum()))][: n // 2]
    return np.concatenate([a, b])


if __name__ == "__main__":
    main()
