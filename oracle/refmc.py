"""ctypes view of the reference's own MULTICOMPONENT solver compiled against the
Cantera-API shim: ``oracle/_ref/libref_mc.so`` (REACTION off) and ``libref_mcr.so``
(REACTION on).  Test infrastructure only.

Routines driven: LBM::LBM(Nx,Ny,Nz,species) (src/lbm-main.cpp:39-118), LBM::Init
(src/lbm-init.cpp:85-146), LBM::loop (src/lbm-main.cpp:149-196) and its phases.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATHS = {False: os.path.join(HERE, "_ref", "libref_mc.so"), True: os.path.join(HERE, "_ref", "libref_mcr.so")}
# the timed baseline: the same sources with the reference's optimisation flags (-O3
# -ffast-math -flto); the parity oracle above is built without -ffast-math
FAST_PATHS = {False: os.path.join(HERE, "_ref", "libref_mc_fast.so"),
              True: os.path.join(HERE, "_ref", "libref_mcr_fast.so")}
# the oracle without floating-point contraction (no fused multiply-adds)
NOFMA_PATHS = {False: os.path.join(HERE, "_ref", "libref_mc_nofma.so"),
               True: os.path.join(HERE, "_ref", "libref_mcr_nofma.so")}
_libs = {}


def _path(reaction, fast):
    if fast == "nofma":
        return NOFMA_PATHS[reaction]
    return (FAST_PATHS if fast else PATHS)[reaction]


def available(reaction=False, fast=False):
    """fast: False (the oracle), True (the reference's -O3 -ffast-math build) or "nofma"."""
    return os.path.exists(_path(reaction, fast))


def lib(reaction=False, fast=False):
    key = (reaction, fast)
    if key not in _libs:
        L = ctypes.CDLL(_path(reaction, fast))
        vp = ctypes.c_void_p
        L.ref_mc_set_mech.argtypes = [vp]
        L.ref_mc_set_units.argtypes = [ctypes.c_float, ctypes.c_float]
        L.ref_mc_layout.argtypes = [ctypes.POINTER(ctypes.c_size_t), ctypes.c_int]
        L.ref_mc_create.restype = vp
        L.ref_mc_create.argtypes = [ctypes.c_int] * 4 + [ctypes.POINTER(ctypes.c_char_p)]
        for n in ("ref_mc_destroy", "ref_mc_init"):
            getattr(L, n).argtypes = [vp]
        L.ref_mc_cells.restype = vp
        L.ref_mc_cells.argtypes = [vp]
        L.ref_mc_species.restype = vp
        L.ref_mc_species.argtypes = [vp, ctypes.c_int]
        L.ref_mc_loop.argtypes = [vp, ctypes.c_int]
        L.ref_mc_phase.argtypes = [vp, ctypes.c_int]
        L.ref_mc_set_threads.argtypes = [ctypes.c_int]
        L.ref_mc_write_restart.argtypes = [vp, ctypes.c_int]
        L.ref_mc_output_vtk.argtypes = [vp, ctypes.c_int]
        L.ref_mc_read_restart.restype = vp
        L.ref_mc_read_restart.argtypes = [ctypes.c_char_p]
        for f in ("ref_mc_nx", "ref_mc_ny", "ref_mc_nz"):
            getattr(L, f).restype = ctypes.c_int
            getattr(L, f).argtypes = [vp]
        _libs[key] = L
    return _libs[key]


def layout(reaction=False):
    out = (ctypes.c_size_t * 21)()
    lib(reaction).ref_mc_layout(out, 21)
    keys = ["size", "type", "p_tensor", "rho", "u", "v", "w", "p", "g", "gpc", "rhoe", "energy_flux", "temp", "HRR",
            "sp_size", "sp_X", "sp_rho", "sp_f", "sp_fpc", "sp_u", "sp_v"]
    return dict(zip(keys, [int(x) for x in out]))


class RefMC:
    """One reference multicomponent ``LBM`` object; `mech` is a mech.Mech table."""

    def __init__(self, NX, NY, NZ, mech, units, mix_dtype, sp_dtype, reaction=False, fast=False):
        self.L = lib(reaction, fast)
        self._mech = mech
        self.L.ref_mc_set_mech(ctypes.byref(mech))
        self.L.ref_mc_set_units(units[0], units[1])
        names = mech.species_names()
        arr = (ctypes.c_char_p * len(names))(*[n.encode() for n in names])
        self.h = self.L.ref_mc_create(NX, NY, NZ, len(names), arr)
        self._views(mech, mix_dtype, sp_dtype, (NX + 2, NY + 2, NZ + 2))

    def _views(self, mech, mix_dtype, sp_dtype, shape=None):
        names = mech.species_names()
        if shape is None:
            shape = (self.L.ref_mc_nx(self.h), self.L.ref_mc_ny(self.h), self.L.ref_mc_nz(self.h))
        self.shape = shape
        n = int(np.prod(self.shape))
        buf = (ctypes.c_char * (n * mix_dtype.itemsize)).from_address(self.L.ref_mc_cells(self.h))
        self.cells = np.frombuffer(buf, dtype=mix_dtype).reshape(self.shape)
        self.species = []
        for a in range(len(names)):
            b = (ctypes.c_char * (n * sp_dtype.itemsize)).from_address(self.L.ref_mc_species(self.h, a))
            self.species.append(np.frombuffer(b, dtype=sp_dtype).reshape(self.shape))

    def init(self):
        self.L.ref_mc_init(self.h)

    def loop(self, n):
        self.L.ref_mc_loop(self.h, n)

    def phase(self, which):
        self.L.ref_mc_phase(self.h, which)

    def write_restart(self, step):
        """The reference's write_restart: ./restart%06d.dat in the current directory."""
        self.L.ref_mc_write_restart(self.h, step)

    def output_vtk(self, nout):
        """The reference's OutputVTK: ./field%06d.vtr in the current directory."""
        self.L.ref_mc_output_vtk(self.h, nout)

    @classmethod
    def from_restart(cls, path, mech, units, mix_dtype, sp_dtype, reaction=False, fast=False):
        """A reference LBM object built by the reference's read_restart."""
        self = cls.__new__(cls)
        self.L = lib(reaction, fast)
        self._mech = mech
        self.L.ref_mc_set_mech(ctypes.byref(mech))
        self.L.ref_mc_set_units(units[0], units[1])
        self.h = self.L.ref_mc_read_restart(path.encode())
        self._views(mech, mix_dtype, sp_dtype)
        return self

    def close(self):
        if self.h:
            self.cells = None
            self.species = []
            self.L.ref_mc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_threads(n, reaction=False, fast=False):
    lib(reaction, fast).ref_mc_set_threads(n)
