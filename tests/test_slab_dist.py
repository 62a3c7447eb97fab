"""Slab decomposition along x on the CPU: two (and three) gloo ranks, each holding one slab of a
multicomponent lattice (the host build of the device's per-cell functions and of the halo
pack/unpack, tests/host/mc_slab_host.cpp over csrc/halo.cuh), step phase by phase and
exchange their halo planes through torch.distributed (slab.exchange, the schedule the
multi-GPU bench runs over NCCL) -- the post-collision populations crossing each face after
the collision, the edge planes' records after the moments.  The two slabs' planes, gathered,
equal the single-domain run bit for bit (FP64), on
  * a 12^3 reacting H2/air mixing layer, periodic in x (the slabs are each other's upper and
    lower neighbours through the periodic face), cut through the H2 interface;
  * the turbulent reacting layer of config 4 at 12^3: characteristic outflow ghosts on the y
    faces (boundary cells along both slab faces), periodic x and z, turbulence.
The single-domain runs of this driver also equal the whole-step host driver the other tests
use (tests/host/mc_host.cpp)."""
import ctypes
import os
import socket
import subprocess

import numpy as np
import pytest

import mech
import slab
import workloads as W
from mc_common import CSRC, NREC, ROOT, build_host_lib, host_run, soa_state

D = ctypes.c_double
STEPS = 6


def build_slab_lib(tmpdir):
    out = os.path.join(str(tmpdir), "libmcslab.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC,
                    os.path.join(ROOT, "tests", "host", "mc_slab_host.cpp"), "-o", out], check=True)
    return out


def load(path):
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.mch_create.restype = vp
    L.mch_create.argtypes = [ctypes.c_int] * 3 + [vp, vp, ctypes.c_float, ctypes.c_float] + [ctypes.c_int] * 4 + [vp]
    for f in ("mch_collide", "mch_stream", "mch_destroy"):
        getattr(L, f).argtypes = [vp]
    L.mch_halo.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int]
    L.mch_halo_values.restype = ctypes.c_long
    L.mch_halo_values.argtypes = [ctypes.c_int]
    L.mch_record.restype = ctypes.c_uint
    L.mch_record.argtypes = [vp, vp]
    return L


def case(name):
    m = mech.h2_air_9()
    if name == "mixing":
        mix, sp = W.mixing_layer_mc(m, N=12, T_hi=1800.0)
        return m, mix, sp, W.FLAME_UNITS, 1, 5  # slab 0: planes 1..4, slab 1: 5..12 (cut in the interface)
    mix, sp = W.turbulent_layer_mc(m, N=12)
    return m, mix, sp, W.TURB_UNITS, 1, None  # the slabs of slab.partition


def lattice(L, m, mix, sp, units, chem, halo_lo=0, halo_hi=0, nx_glob=None):
    typ = np.ascontiguousarray(mix["type"].astype(np.int8).reshape(-1))
    rec0 = np.ascontiguousarray(soa_state(mix, sp))
    Nx, Ny, Nz = mix.shape
    h = L.mch_create(Nx, Ny, Nz, typ.ctypes.data, ctypes.addressof(m), units[0], units[1], chem, halo_lo, halo_hi,
                     nx_glob or Nx, rec0.ctypes.data)
    assert h
    return h


def record(L, h, shape):
    out = np.zeros((NREC, int(np.prod(shape))))
    st = L.mch_record(h, out.ctypes.data)
    return out.reshape((NREC,) + shape), st


def single_domain(path, name):
    L = load(path)
    m, mix, sp, units, chem, cut = case(name)
    h = lattice(L, m, mix, sp, units, chem)
    for _ in range(STEPS):
        L.mch_collide(h)
        L.mch_stream(h)
    R, st = record(L, h, mix.shape)
    L.mch_destroy(h)
    return R, st


def _rank_main(rank, world, port, path, name, outdir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        L = load(path)
        m, mix, sp, units, chem, cut = case(name)
        Nx = mix.shape[0]
        a, b = slab.partition(Nx - 2, world, rank) if cut is None else ((1, cut - 1) if rank == 0 else (cut, Nx - 2))
        sl = slice(a - 1, b + 2)
        lmix = np.ascontiguousarray(mix[sl])
        lsp = [np.ascontiguousarray(s_[sl]) for s_ in sp]
        h = lattice(L, m, lmix, lsp, units, chem, 1, 1, Nx)
        Ny, Nz = mix.shape[1:]

        def pack(face, what):
            buf = np.zeros(int(L.mch_halo_values(what)) * Ny * Nz)
            L.mch_halo(h, face, what, buf.ctypes.data, 1)
            return torch.from_numpy(buf)

        def unpack(face, what, t):
            L.mch_halo(h, face, what, t.numpy().ctypes.data, 0)

        comm = slab.TorchComm(dist)

        def exchange(what):
            slab.exchange(what, pack, unpack, comm, world, rank)

        for _ in range(STEPS):
            L.mch_collide(h)
            exchange(slab.POPULATIONS)  # the populations crossing each face
            L.mch_stream(h)
            exchange(slab.RECORD)  # the edge planes' records
        R, st = record(L, h, lmix.shape)
        L.mch_destroy(h)
        np.save(os.path.join(outdir, f"rank{rank}.npy"), R[:, 1:-1])
        np.save(os.path.join(outdir, f"status{rank}.npy"), np.array([st, a, b]))
    finally:
        dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.fixture(scope="module")
def slab_lib(tmp_path_factory):
    return build_slab_lib(tmp_path_factory.mktemp("mcslab"))


@pytest.mark.parametrize("name,world", [("mixing", 2), ("turbulent", 2), ("turbulent", 3)])
def test_gloo_slabs_equal_the_single_domain(slab_lib, name, world, tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(world, free_port(), slab_lib, name, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    R, st = single_domain(slab_lib, name)
    assert st == 0
    for rank in range(world):
        s, a, b = np.load(os.path.join(tmp_path, f"status{rank}.npy"))
        assert s == 0
        got = np.load(os.path.join(tmp_path, f"rank{rank}.npy"))
        want = R[:, a:b + 1]
        fl = (case(name)[1]["type"][a:b + 1] == W.TYPE_F)
        assert np.array_equal(got[:, fl], want[:, fl]), f"rank {rank}: {np.max(np.abs(got[:, fl] - want[:, fl]))}"


def test_stateful_driver_equals_the_whole_step_driver(slab_lib, tmp_path):
    """The phase-by-phase driver without halos is the whole-step host driver: same records."""
    R, st = single_domain(slab_lib, "mixing")
    m, mix, sp, units, chem, cut = case("mixing")
    assert units == W.FLAME_UNITS
    R2, st2 = host_run(build_host_lib(tmp_path), m, mix, sp, chem, STEPS)
    fl = (mix["type"] == W.TYPE_F).reshape(-1)
    assert st == 0 and st2 == 0
    assert np.array_equal(R.reshape(NREC, -1)[:, fl], R2[:, fl])
