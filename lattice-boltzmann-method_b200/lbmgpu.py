"""Python binding of liblbmgpu.so (the C ABI in include/lbmgpu.h), through ctypes.

The library is the product: every call below goes straight to the sm_100a kernels.
There is no fallback -- if the shared library or a CUDA device is missing, the calls
raise ``LbmGpuError``.

The cell arrays exchanged with the device use the reference's own cell record
(class MIXTURE, src/headers/lbm.hpp:56-88), so a state can move between this library and
the reference solver (Init, restart files, VTK output) without conversion.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbmgpu.so")
ABI_VERSION = 2

FP64, FP32 = 0, 1
ST_NAN, ST_NEG_STATE, ST_TAU_UNSTABLE = 0x1, 0x2, 0x4
KIND_COLLIDE, KIND_STREAM_MOMENT, KIND_OTHER = 0, 1, 2

# The single-component MIXTURE record (1024 bytes; offsets as laid out by g++/x86-64).
MIXTURE_SC = np.dtype({
    "names": ["type", "f", "fpc", "p_tensor", "rho", "u", "v", "w", "p", "g", "gpc", "rhoe",
              "energy_flux", "temp"],
    "formats": ["<i2", ("<f8", 27), ("<f8", 27), ("<f8", (3, 3)), "<f8", "<f8", "<f8", "<f8", "<f8",
                ("<f8", 27), ("<f8", 27), "<f8", ("<f8", 3), "<f8"],
    "offsets": [0, 8, 224, 440, 512, 520, 528, 536, 544, 552, 768, 984, 992, 1016],
    "itemsize": 1024,
})

EXPORTS = [
    "lbmgpu_create", "lbmgpu_destroy", "lbmgpu_upload", "lbmgpu_download", "lbmgpu_upload_planes",
    "lbmgpu_download_planes", "lbmgpu_set_halo", "lbmgpu_halo_bytes", "lbmgpu_halo_pack", "lbmgpu_halo_unpack",
    "lbmgpu_get_stream", "lbmgpu_write_restart", "lbmgpu_read_restart", "lbmgpu_write_vtk", "lbmgpu_vtk_fields",
    "lbmgpu_init",
    "lbmgpu_collide_species", "lbmgpu_collide", "lbmgpu_streaming", "lbmgpu_tms_bc",
    "lbmgpu_calculate_moment", "lbmgpu_step", "lbmgpu_time_steps", "lbmgpu_synchronize", "lbmgpu_status",
    "lbmgpu_profile", "lbmgpu_kernel_times", "lbmgpu_device_bytes", "lbmgpu_error_string",
    "lbmgpu_units_from_dx_dt", "lbmgpu_sums_count", "lbmgpu_sums", "lbmgpu_sums_noalloc", "lbmgpu_diagnostics",
    "lbmgpu_surrogate_collect", "lbmgpu_surrogate_load_samples", "lbmgpu_surrogate_samples",
    "lbmgpu_surrogate_augment", "lbmgpu_surrogate_train",
    "lbmgpu_surrogate_enable", "lbmgpu_surrogate_eval", "lbmgpu_surrogate_params", "lbmgpu_surrogate_stats",
    "lbmgpu_surrogate_grads",
]
SUMS_MAX = 22
HALO_POPULATIONS, HALO_RECORD = 0, 1
KERNEL_KINDS = 8
DIAG_COUNT = 6
SUR_IN, SUR_OUT, SUR_NPARAMS = 12, 10, 36046


class RestartInfo(ctypes.Structure):
    """lbmgpu_restart_info: the restart header's LBM fields."""
    _fields_ = [("dx", ctypes.c_int), ("dy", ctypes.c_int), ("dz", ctypes.c_int), ("step", ctypes.c_int),
                ("Ra", ctypes.c_double), ("permeability", ctypes.c_double)]


VTK_SI, VTK_MASSFRAC = 1, 2


class SurrogateReport(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_long), ("train_steps", ctypes.c_long), ("last_loss", ctypes.c_double),
                ("cells_predicted", ctypes.c_long), ("cells_integrated", ctypes.c_long),
                ("cells_audited", ctypes.c_long), ("audit_rel_err", ctypes.c_double),
                ("audit_max_abs_err", ctypes.c_double), ("audit_dY", ctypes.c_double), ("enabled", ctypes.c_int),
                ("collecting", ctypes.c_int)]
CHEM_OFF, CHEM_REF_EXPLICIT, CHEM_ROSENBROCK = 0, 1, 2
ST_NEWTON, ST_CHEM = 0x8, 0x10


class MixtureLayout(ctypes.Structure):
    _fields_ = [("size", ctypes.c_size_t)] + [(n, ctypes.c_long) for n in (
        "type", "f", "fpc", "p_tensor", "rho", "u", "v", "w", "p", "g", "gpc", "rhoe", "energy_flux",
        "temp", "HRR")]


class SpeciesLayout(ctypes.Structure):
    _fields_ = [("size", ctypes.c_size_t)] + [(n, ctypes.c_long) for n in ("X", "rho", "f", "fpc", "u", "v", "w")]


class Desc(ctypes.Structure):
    _fields_ = [("abi_version", ctypes.c_int), ("device", ctypes.c_int), ("Nx", ctypes.c_int),
                ("Ny", ctypes.c_int), ("Nz", ctypes.c_int), ("n_species", ctypes.c_int),
                ("precision", ctypes.c_int), ("dt_sim", ctypes.c_int), ("nu", ctypes.c_double),
                ("gas_const", ctypes.c_double), ("gamma", ctypes.c_double), ("prtl", ctypes.c_double),
                ("mix", MixtureLayout), ("spc", SpeciesLayout), ("mech", ctypes.c_void_p),
                ("units_m", ctypes.c_float), ("units_kg", ctypes.c_float), ("units_s", ctypes.c_float),
                ("units_K", ctypes.c_float), ("chem_mode", ctypes.c_int)]


class LbmGpuError(RuntimeError):
    def __init__(self, code, what):
        self.code = code
        super().__init__(f"{what}: {error_string(code)} ({code})")


# the parity build of the same sources without fused multiply-adds (tests only)
NOFMA_LIB_PATH = os.path.join(HERE, "liblbmgpu_nofma.so")
_libs = {}


def lib(path=None):
    """Loads liblbmgpu.so, or the library at `path` (raises OSError when it has not been
    built)."""
    path = path or LIB_PATH
    if path not in _libs:
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.lbmgpu_create.argtypes = [ctypes.POINTER(Desc), ctypes.POINTER(vp)]
        for name in ("lbmgpu_destroy", "lbmgpu_init", "lbmgpu_collide_species", "lbmgpu_collide",
                     "lbmgpu_streaming", "lbmgpu_tms_bc", "lbmgpu_calculate_moment", "lbmgpu_synchronize"):
            getattr(L, name).argtypes = [vp]
        L.lbmgpu_upload.argtypes = [vp, vp, vp]
        L.lbmgpu_download.argtypes = [vp, vp, vp]
        L.lbmgpu_upload_planes.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp]
        L.lbmgpu_download_planes.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp]
        L.lbmgpu_set_halo.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.lbmgpu_halo_bytes.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
        L.lbmgpu_halo_pack.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
        L.lbmgpu_halo_unpack.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
        L.lbmgpu_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.lbmgpu_write_restart.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(RestartInfo)]
        L.lbmgpu_read_restart.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(RestartInfo)]
        L.lbmgpu_write_vtk.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        L.lbmgpu_vtk_fields.argtypes = [vp, ctypes.POINTER(ctypes.c_float), ctypes.c_size_t, ctypes.c_int]
        L.lbmgpu_units_from_dx_dt.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]
        L.lbmgpu_step.argtypes = [vp, ctypes.c_int]
        L.lbmgpu_time_steps.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.lbmgpu_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32), ctypes.c_int]
        L.lbmgpu_profile.argtypes = [vp, ctypes.c_int]
        L.lbmgpu_kernel_times.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_long),
                                          ctypes.POINTER(ctypes.c_double)]
        L.lbmgpu_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
        L.lbmgpu_sums_count.argtypes = [vp]
        L.lbmgpu_sums.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
        L.lbmgpu_sums_noalloc.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
        L.lbmgpu_diagnostics.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
        fp = ctypes.POINTER(ctypes.c_float)
        L.lbmgpu_surrogate_collect.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_long]
        L.lbmgpu_surrogate_load_samples.argtypes = [vp, fp, fp, ctypes.c_long]
        L.lbmgpu_surrogate_samples.argtypes = [vp, fp, fp, ctypes.POINTER(ctypes.c_ubyte), ctypes.c_long]
        L.lbmgpu_surrogate_augment.argtypes = [vp, ctypes.c_long, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                               ctypes.c_uint]
        L.lbmgpu_surrogate_train.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint,
                                             ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.lbmgpu_surrogate_enable.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.lbmgpu_surrogate_eval.argtypes = [vp, fp, ctypes.c_long, fp]
        L.lbmgpu_surrogate_params.argtypes = [vp, fp, ctypes.c_long, ctypes.c_int]
        L.lbmgpu_surrogate_stats.argtypes = [vp, ctypes.POINTER(SurrogateReport)]
        L.lbmgpu_surrogate_grads.argtypes = [vp, fp, ctypes.c_long]
        L.lbmgpu_error_string.argtypes = [ctypes.c_int]
        L.lbmgpu_error_string.restype = ctypes.c_char_p
        _libs[path] = L
    return _libs[path]


def error_string(code):
    return lib().lbmgpu_error_string(code).decode()


def layout_of(dtype):
    """MixtureLayout (byte offsets) of a numpy structured dtype; -1 for absent fields."""
    lay = MixtureLayout()
    lay.size = dtype.itemsize
    for name, _ in MixtureLayout._fields_[1:]:
        setattr(lay, name, dtype.fields[name][1] if name in dtype.fields else -1)
    return lay


def species_layout_of(dtype):
    lay = SpeciesLayout()
    lay.size = dtype.itemsize
    for name, _ in SpeciesLayout._fields_[1:]:
        setattr(lay, name, dtype.fields[name][1])
    return lay


def units_from_dx_dt(dx, dt):
    """(m, kg, s, K) as the reference's units.set_m_kg_s(dx, dt) leaves them."""
    out = (ctypes.c_float * 4)()
    _check(lib().lbmgpu_units_from_dx_dt(dx, dt, out), "lbmgpu_units_from_dx_dt")
    return tuple(out)


def _check(rc, what):
    if rc < 0:
        raise LbmGpuError(rc, what)
    return rc


class Lattice:
    """One LBM object on one GPU: the device counterpart of the reference's ``LBM`` class.

    ``Nx, Ny, Nz`` include the ghost layer (the reference's LBM::Nx etc.).
    """

    def __init__(self, Nx, Ny, Nz, nu=0.0, gas_const=1.0, gamma=1.4, prtl=0.5, device=0,
                 precision=FP64, dtype=MIXTURE_SC, dt_sim=1, mech=None, species_dtype=None, dx_dt=None,
                 chem=CHEM_OFF, library=None):
        """Single component: nu, gas_const, gamma, prtl.  Multicomponent: `mech` (a
        mech.Mech table), `dtype`/`species_dtype` (the MIXTURE and SPECIES records) and
        `dx_dt` (the arguments of the reference's units.set_m_kg_s(dx, dt)).  `library`: the
        path of another build of the library (the tests' no-FMA parity build)."""
        self.L = lib(library)
        d = Desc()
        d.abi_version = ABI_VERSION
        d.device = device
        d.Nx, d.Ny, d.Nz = Nx, Ny, Nz
        d.precision = precision
        d.dt_sim = dt_sim
        d.nu, d.gas_const, d.gamma, d.prtl = nu, gas_const, gamma, prtl
        d.mix = layout_of(dtype)
        self.ns = 0
        if mech is not None:
            self.ns = mech.n_species
            self._mech = mech
            d.n_species = mech.n_species
            d.mech = ctypes.addressof(mech)
            d.spc = species_layout_of(species_dtype)
            d.units_m, d.units_kg, d.units_s, d.units_K = units_from_dx_dt(*dx_dt)
            d.chem_mode = chem
        self.dtype = dtype
        self.species_dtype = species_dtype
        self.shape = (Nx, Ny, Nz)
        self.h = ctypes.c_void_p()
        _check(self.L.lbmgpu_create(ctypes.byref(d), ctypes.byref(self.h)), "lbmgpu_create")

    # -- state transfer ---------------------------------------------------------------
    def _cells_ptr(self, cells, shape=None):
        shape = shape or self.shape
        if cells.dtype != self.dtype or cells.shape != shape or not cells.flags.c_contiguous:
            raise ValueError("cell array must be a C-contiguous %s array of shape %s" % (self.dtype, shape))
        return cells.ctypes.data

    def _species_ptrs(self, species, shape=None):
        shape = shape or self.shape
        if self.ns == 0:
            return None
        if species is None or len(species) != self.ns:
            raise ValueError("one species array per species is required")
        for sp in species:
            if sp.dtype != self.species_dtype or sp.shape != shape or not sp.flags.c_contiguous:
                raise ValueError("species arrays must be C-contiguous %s arrays of shape %s"
                                 % (self.species_dtype, shape))
        return (ctypes.c_void_p * self.ns)(*[sp.ctypes.data for sp in species])

    # -- restart and field output ---------------------------------------------------------
    def write_restart(self, path, info):
        """The reference's restart file of the current state (lbmgpu_write_restart)."""
        _check(self.L.lbmgpu_write_restart(self.h, str(path).encode(), ctypes.byref(info)), "lbmgpu_write_restart")

    def read_restart(self, path):
        """Loads a reference restart file (lbmgpu_read_restart); returns its RestartInfo."""
        info = RestartInfo()
        _check(self.L.lbmgpu_read_restart(self.h, str(path).encode(), ctypes.byref(info)), "lbmgpu_read_restart")
        return info

    def write_vtk(self, path, dx=1, flags=0):
        """The reference's OutputVTK file of the current state (lbmgpu_write_vtk)."""
        _check(self.L.lbmgpu_write_vtk(self.h, str(path).encode(), dx, flags), "lbmgpu_write_vtk")

    # -- slab decomposition along x ------------------------------------------------------
    def set_halo(self, lo, hi, nx_global):
        """Marks the low / high x ghost plane as a halo of the neighbouring slab
        (lbmgpu_set_halo); nx_global is the whole domain's Nx with ghosts."""
        _check(self.L.lbmgpu_set_halo(self.h, int(lo), int(hi), int(nx_global)), "lbmgpu_set_halo")

    def stream(self):
        """The handle's cudaStream_t as an integer (lbmgpu_get_stream)."""
        p = ctypes.c_void_p()
        _check(self.L.lbmgpu_get_stream(self.h, ctypes.byref(p)), "lbmgpu_get_stream")
        return p.value or 0

    def halo_bytes(self, what):
        b = ctypes.c_size_t()
        _check(self.L.lbmgpu_halo_bytes(self.h, what, ctypes.byref(b)), "lbmgpu_halo_bytes")
        return b.value

    def halo_pack(self, face, what, dev_ptr):
        """Enqueues the face's outgoing values into the device buffer at dev_ptr."""
        _check(self.L.lbmgpu_halo_pack(self.h, face, what, ctypes.c_void_p(dev_ptr)), "lbmgpu_halo_pack")

    def halo_unpack(self, face, what, dev_ptr):
        """Enqueues the face's incoming values from the device buffer at dev_ptr."""
        _check(self.L.lbmgpu_halo_unpack(self.h, face, what, ctypes.c_void_p(dev_ptr)), "lbmgpu_halo_unpack")

    def upload_planes(self, i0, cells, species):
        """Uploads the x-planes i0 .. i0 + cells.shape[0] - 1 (lbmgpu_upload_planes)."""
        shape = (cells.shape[0],) + self.shape[1:]
        _check(self.L.lbmgpu_upload_planes(self.h, i0, i0 + shape[0], self._cells_ptr(cells, shape),
                                          self._species_ptrs(species, shape)), "lbmgpu_upload_planes")

    def download_planes(self, i0, cells, species):
        """Downloads the x-planes i0 .. i0 + cells.shape[0] - 1 (lbmgpu_download_planes)."""
        shape = (cells.shape[0],) + self.shape[1:]
        _check(self.L.lbmgpu_download_planes(self.h, i0, i0 + shape[0], self._cells_ptr(cells, shape),
                                            self._species_ptrs(species, shape)), "lbmgpu_download_planes")

    def upload(self, cells, species=None):
        _check(self.L.lbmgpu_upload(self.h, self._cells_ptr(cells), self._species_ptrs(species)), "lbmgpu_upload")

    def download(self, cells, species=None):
        _check(self.L.lbmgpu_download(self.h, self._cells_ptr(cells), self._species_ptrs(species)),
               "lbmgpu_download")

    # -- the reference's phases -------------------------------------------------------
    def init(self):
        _check(self.L.lbmgpu_init(self.h), "lbmgpu_init")

    def collide_species(self):
        return self.L.lbmgpu_collide_species(self.h)

    def collide(self):
        _check(self.L.lbmgpu_collide(self.h), "lbmgpu_collide")

    def streaming(self):
        _check(self.L.lbmgpu_streaming(self.h), "lbmgpu_streaming")

    def tms_bc(self):
        _check(self.L.lbmgpu_tms_bc(self.h), "lbmgpu_tms_bc")

    def calculate_moment(self):
        _check(self.L.lbmgpu_calculate_moment(self.h), "lbmgpu_calculate_moment")

    def step(self, n=1):
        _check(self.L.lbmgpu_step(self.h, n), "lbmgpu_step")

    def time_steps(self, n):
        """Runs n steps and returns their device time in ms (CUDA events on the handle's
        stream)."""
        ms = ctypes.c_double()
        _check(self.L.lbmgpu_time_steps(self.h, n, ctypes.byref(ms)), "lbmgpu_time_steps")
        return ms.value

    def synchronize(self):
        return _check(self.L.lbmgpu_synchronize(self.h), "lbmgpu_synchronize")

    def status(self, clear=False):
        f = ctypes.c_uint32()
        _check(self.L.lbmgpu_status(self.h, ctypes.byref(f), int(clear)), "lbmgpu_status")
        return f.value

    # -- timing -------------------------------------------------------------------------
    def profile(self, enable=True):
        _check(self.L.lbmgpu_profile(self.h, int(enable)), "lbmgpu_profile")

    def kernel_times(self):
        """Per kernel kind (0 collide / population update, 1 stream+boundary+moment
        (multicomponent: the interior pull and sums), 2 other, 3 multicomponent collision
        parameters, 4 chemistry surrogate, 5 multicomponent moment solve, 6 multicomponent
        energy-flux terms, 7 stiff chemistry of every cell): launches and device ms."""
        launches = (ctypes.c_long * KERNEL_KINDS)()
        ms = (ctypes.c_double * KERNEL_KINDS)()
        _check(self.L.lbmgpu_kernel_times(self.h, KERNEL_KINDS, launches, ms), "lbmgpu_kernel_times")
        return list(launches), list(ms)

    # -- conserved sums -------------------------------------------------------------------
    def sums(self):
        """FP64 totals over the fluid cells: mass, momentum (3), total energy, then
        (multicomponent) the species masses and the H, O, N, Ar, C element totals."""
        k = self.L.lbmgpu_sums_count(self.h)
        _check(k if k < 0 else 0, "lbmgpu_sums_count")
        out = (ctypes.c_double * k)()
        _check(self.L.lbmgpu_sums(self.h, out, k), "lbmgpu_sums")
        return list(out)

    # -- chemistry surrogate (CHEM_ROSENBROCK) ------------------------------------------------
    def surrogate_collect(self, enable=True, stride=1, capacity=1 << 20):
        """While enabled, each integrator step writes the (features, targets) of every
        stride-th cell to the device sample set (capacity rows)."""
        _check(self.L.lbmgpu_surrogate_collect(self.h, int(enable), int(stride), int(capacity)),
               "lbmgpu_surrogate_collect")

    def surrogate_load_samples(self, x, y):
        """Replaces the sample set: x (n, 12) raw features, y (n, 10) raw targets."""
        import numpy as np
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        _check(self.L.lbmgpu_surrogate_load_samples(self.h, x.ctypes.data_as(fp), y.ctypes.data_as(fp), len(x)),
               "lbmgpu_surrogate_load_samples")

    def surrogate_samples(self, n=None):
        """The first n rows (all by default) of the sample set: (x (n, 12), y (n, 10), valid (n,))."""
        import numpy as np
        if n is None:
            n = self.surrogate_stats()["samples"]
        x = np.zeros((n, SUR_IN), np.float32)
        y = np.zeros((n, SUR_OUT), np.float32)
        v = np.zeros(n, np.uint8)
        fp = ctypes.POINTER(ctypes.c_float)
        _check(self.L.lbmgpu_surrogate_samples(self.h, x.ctypes.data_as(fp), y.ctypes.data_as(fp),
                                              v.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), n),
               "lbmgpu_surrogate_samples")
        return x, y, v.astype(bool)

    def surrogate_augment(self, n, span_y=1.5, span_t=0.01, y_trace=1e-3, seed=1):
        """Appends n integrator-labelled rows perturbed from random valid sample rows (mass
        fractions below y_trace by exp(U(-span_y, span_y)), T by exp(U(-span_t, span_t)))."""
        _check(self.L.lbmgpu_surrogate_augment(self.h, int(n), float(span_y), float(span_t), float(y_trace), int(seed)),
               "lbmgpu_surrogate_augment")

    def surrogate_train(self, epochs=10, batch=4096, lr=1e-3, seed=1, refit=False):
        """Adam epochs over the sample set (step size lr decaying to 0 along a half cosine);
        returns the last epoch's mean standardised loss."""
        loss = ctypes.c_double()
        _check(self.L.lbmgpu_surrogate_train(self.h, int(epochs), int(batch), float(lr), int(seed), int(refit),
                                            ctypes.byref(loss)), "lbmgpu_surrogate_train")
        return loss.value

    def surrogate_enable(self, enable=True, audit_period=100):
        _check(self.L.lbmgpu_surrogate_enable(self.h, int(enable), int(audit_period)), "lbmgpu_surrogate_enable")

    def surrogate_eval(self, x):
        """The network on raw features x (n, 12) -> raw predictions (n, 10)."""
        import numpy as np
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((len(x), SUR_OUT), np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        _check(self.L.lbmgpu_surrogate_eval(self.h, x.ctypes.data_as(fp), len(x), y.ctypes.data_as(fp)),
               "lbmgpu_surrogate_eval")
        return y

    def surrogate_params(self, values=None):
        """Gets (values None) or sets the packed parameters (SUR_NPARAMS floats)."""
        import numpy as np
        buf = np.zeros(SUR_NPARAMS, np.float32) if values is None else np.ascontiguousarray(values, np.float32).copy()
        fp = ctypes.POINTER(ctypes.c_float)
        _check(self.L.lbmgpu_surrogate_params(self.h, buf.ctypes.data_as(fp), len(buf), int(values is not None)),
               "lbmgpu_surrogate_params")
        return buf

    def surrogate_grads(self):
        """The last training minibatch's loss gradients, packed like the parameters."""
        import numpy as np
        buf = np.zeros(SUR_NPARAMS, np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        _check(self.L.lbmgpu_surrogate_grads(self.h, buf.ctypes.data_as(fp), len(buf)), "lbmgpu_surrogate_grads")
        return buf

    def surrogate_stats(self):
        r = SurrogateReport()
        _check(self.L.lbmgpu_surrogate_stats(self.h, ctypes.byref(r)), "lbmgpu_surrogate_stats")
        return {k: getattr(r, k) for k, _ in SurrogateReport._fields_}

    def diagnostics(self):
        """Device-reduced diagnostics (lattice units): dict of kinetic (sum rho|u|^2),
        enstrophy (sum rho|curl u|^2), energy (sum rho E), hrr (sum of the heat-release
        field), T_max, T_min."""
        out = (ctypes.c_double * DIAG_COUNT)()
        _check(self.L.lbmgpu_diagnostics(self.h, out, DIAG_COUNT), "lbmgpu_diagnostics")
        return dict(zip(("kinetic", "enstrophy", "energy", "hrr", "T_max", "T_min"), list(out)))

    def sums_noalloc(self, n_out=None):
        """The same totals through lbmgpu_sums_noalloc (fixed device scratch, no
        allocation); n_out defaults to the handle's count."""
        k = self.L.lbmgpu_sums_count(self.h)
        _check(k if k < 0 else 0, "lbmgpu_sums_count")
        n = k if n_out is None else n_out
        out = (ctypes.c_double * max(n, 1))()
        _check(self.L.lbmgpu_sums_noalloc(self.h, out, n), "lbmgpu_sums_noalloc")
        return list(out)[:k]

    def device_bytes(self):
        b = ctypes.c_size_t()
        _check(self.L.lbmgpu_device_bytes(self.h, ctypes.byref(b)), "lbmgpu_device_bytes")
        return b.value

    def close(self):
        if self.h:
            self.L.lbmgpu_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
