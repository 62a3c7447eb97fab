"""ctypes view of ``oracle/liboracle.so`` (plain-C restatement; test infrastructure)."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)


class Grid(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int),
                ("nu", _D), ("R", _D), ("gamma", _D), ("prtl", _D), ("dt", ctypes.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        L.orc_sc_sizeof.restype = ctypes.c_size_t
        L.orc_feq.restype = _D
        L.orc_feq.argtypes = [ctypes.c_int, _D, _DP, _D, _DP]
        L.orc_geq.restype = _D
        L.orc_geq.argtypes = [ctypes.c_int, _D, _D, _D, _DP]
        L.orc_geq_moment.restype = _D
        L.orc_geq_moment.argtypes = [ctypes.c_int, _D, _DP, _DP, _D]
        L.orc_gstr.restype = _D
        L.orc_gstr.argtypes = [ctypes.c_int, _D, _DP]
        for name in ("orc_fd_central", "orc_fd_fuw"):
            fn = getattr(L, name)
            fn.restype = _D
            fn.argtypes = [_D] * 5 + [ctypes.c_int] * 2
        L.orc_fd_uw.restype = _D
        L.orc_fd_uw.argtypes = [_D] * 5
        for name in ("orc_sc_init", "orc_sc_collide", "orc_sc_streaming", "orc_sc_tms_bc", "orc_sc_moment"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.POINTER(Grid)]
        L.orc_sc_loop.argtypes = [ctypes.c_void_p, ctypes.POINTER(Grid), ctypes.c_int]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _dp(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_DP)


def feq(l, rho, u, theta, corr):
    u, pu = _dp(u)
    c, pc = _dp(corr)
    return lib().orc_feq(l, rho, pu, theta, pc)


def geq(l, rho, U, theta, v):
    v, pv = _dp(v)
    return lib().orc_geq(l, rho, U, theta, pv)


def geq_moment(l, rhoe, q, R, theta):
    q, pq = _dp(q)
    R, pR = _dp(np.asarray(R).reshape(9))
    return lib().orc_geq_moment(l, rhoe, pq, pR, theta)


def gstr(l, geqv, dq):
    dq, pd = _dp(dq)
    return lib().orc_gstr(l, geqv, pd)


def fd_central(*a):
    return lib().orc_fd_central(*a)


def fd_fuw(*a):
    return lib().orc_fd_fuw(*a)


def fd_uw(*a):
    return lib().orc_fd_uw(*a)


def set_threads(n):
    lib().orc_set_threads(n)


class OracleSC:
    """Runs the C oracle in place on an AoS cell array (numpy structured, C-contiguous)."""

    def __init__(self, cells, nu, R, gamma, prtl):
        assert cells.flags.c_contiguous and cells.dtype.itemsize == lib().orc_sc_sizeof()
        self.cells = cells
        Nx, Ny, Nz = cells.shape
        self.grid = Grid(Nx, Ny, Nz, nu, R, gamma, prtl, 1)

    def _call(self, name, *extra):
        getattr(lib(), name)(self.cells.ctypes.data, ctypes.byref(self.grid), *extra)

    def init(self):
        self._call("orc_sc_init")

    def collide(self):
        self._call("orc_sc_collide")

    def streaming(self):
        self._call("orc_sc_streaming")

    def tms_bc(self):
        self._call("orc_sc_tms_bc")

    def moment(self):
        self._call("orc_sc_moment")

    def loop(self, n):
        self._call("orc_sc_loop", n)
