"""ctypes view of ``oracle/_ref/libref_sc.so`` -- the reference's own single-component
solver compiled from its sources (recipe: ``oracle/Makefile``).

Test infrastructure only.  The library is the ground truth for the single-component
path: ``LBM::Init`` (src/lbm-init.cpp:8-82), ``LBM::loop`` (src/lbm-main.cpp:149-196)
and the equilibrium/FD helpers (src/headers/lbm.hpp:276-305, src/lbm-edf.cpp:38-164,
src/headers/FD.hpp:108-127, src/FD.cpp:5-74).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref_sc.so")

_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        L.ref_sc_layout.argtypes = [ctypes.POINTER(ctypes.c_size_t), ctypes.c_int]
        L.ref_sc_create.restype = ctypes.c_void_p
        L.ref_sc_create.argtypes = [ctypes.c_int] * 3 + [_D] * 4
        L.ref_sc_destroy.argtypes = [ctypes.c_void_p]
        L.ref_sc_cells.restype = ctypes.c_void_p
        L.ref_sc_cells.argtypes = [ctypes.c_void_p]
        L.ref_sc_init.argtypes = [ctypes.c_void_p]
        L.ref_sc_loop.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_sc_phase.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_sc_set_threads.argtypes = [ctypes.c_int]
        L.ref_sc_max_threads.restype = ctypes.c_int
        L.ref_sc_feq.restype = _D
        L.ref_sc_feq.argtypes = [ctypes.c_int, _D, _DP, _D, _DP]
        L.ref_sc_geq_poly.restype = _D
        L.ref_sc_geq_poly.argtypes = [ctypes.c_int, _D, _D, _D, _DP]
        L.ref_sc_geq_moment.restype = _D
        L.ref_sc_geq_moment.argtypes = [ctypes.c_int, _D, _DP, _DP, _D]
        L.ref_sc_gstr.restype = _D
        L.ref_sc_gstr.argtypes = [ctypes.c_int, _D, _DP]
        L.ref_sc_feq_geq.argtypes = [ctypes.c_void_p, _DP, _DP, _D, _DP, _D]
        for name in ("ref_fd_central", "ref_fd_fuw"):
            fn = getattr(L, name)
            fn.restype = _D
            fn.argtypes = [_D] * 5 + [ctypes.c_int] * 2
        L.ref_fd_uw.restype = _D
        L.ref_fd_uw.argtypes = [_D] * 5
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_DP)


def layout():
    out = (ctypes.c_size_t * 15)()
    lib().ref_sc_layout(out, 15)
    keys = ["size", "type", "f", "fpc", "p_tensor", "rho", "u", "v", "w", "p", "g", "gpc",
            "rhoe", "energy_flux", "temp"]
    return dict(zip(keys, [int(x) for x in out]))


class RefSC:
    """One reference ``LBM`` object (single component), interior size NX x NY x NZ."""

    def __init__(self, NX, NY, NZ, nu, R, gamma, prtl, dtype):
        self.h = lib().ref_sc_create(NX, NY, NZ, nu, R, gamma, prtl)
        self.shape = (NX + 2, NY + 2, NZ + 2)
        n = int(np.prod(self.shape))
        buf = (ctypes.c_char * (n * dtype.itemsize)).from_address(lib().ref_sc_cells(self.h))
        self.cells = np.frombuffer(buf, dtype=dtype).reshape(self.shape)

    def init(self):
        lib().ref_sc_init(self.h)

    def loop(self, n):
        lib().ref_sc_loop(self.h, n)

    def phase(self, which):
        lib().ref_sc_phase(self.h, which)

    def feq_geq(self, rho, vel, T):
        f = np.zeros(27)
        g = np.zeros(27)
        v = np.ascontiguousarray(vel, dtype=np.float64)
        lib().ref_sc_feq_geq(self.h, _dp(f), _dp(g), rho, _dp(v), T)
        return f, g

    def close(self):
        if self.h:
            self.cells = None
            lib().ref_sc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def feq(l, rho, u, theta, corr):
    u = np.ascontiguousarray(u, dtype=np.float64)
    c = np.ascontiguousarray(corr, dtype=np.float64)
    return lib().ref_sc_feq(l, rho, _dp(u), theta, _dp(c))


def geq_poly(l, rho, U, theta, v):
    v = np.ascontiguousarray(v, dtype=np.float64)
    return lib().ref_sc_geq_poly(l, rho, U, theta, _dp(v))


def geq_moment(l, rhoe, q, R, theta):
    q = np.ascontiguousarray(q, dtype=np.float64)
    R = np.ascontiguousarray(R, dtype=np.float64).reshape(9)
    return lib().ref_sc_geq_moment(l, rhoe, _dp(q), _dp(R), theta)


def gstr(l, geq, dq):
    dq = np.ascontiguousarray(dq, dtype=np.float64)
    return lib().ref_sc_gstr(l, geq, _dp(dq))


def fd_central(l, c, r, dx, vel, tl, tr):
    return lib().ref_fd_central(l, c, r, dx, vel, tl, tr)


def fd_fuw(l, c, r, dx, vel, tl, tr):
    return lib().ref_fd_fuw(l, c, r, dx, vel, tl, tr)


def fd_uw(s0, s1, s2, dx, vel):
    return lib().ref_fd_uw(s0, s1, s2, dx, vel)


def set_threads(n):
    lib().ref_sc_set_threads(n)


def max_threads():
    return lib().ref_sc_max_threads()
