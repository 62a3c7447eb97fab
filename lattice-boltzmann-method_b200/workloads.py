"""Seeded synthetic initial states (the workloads of the parity tests and the bench).

Each state is an AoS cell array with the reference's single-component MIXTURE layout
(src/headers/lbm.hpp:56-88), the form the reference's case setups (src/setup.cpp) leave
before LBM::run: cell types and the macroscopic fields u, v, w, p, temp.  It is ready for
the device upload and for the reference solver alike.

Seeds: numpy PCG64 with seed 20261203 unless stated otherwise.  No external dataset is
involved.
"""
import math

import numpy as np

SEED = 20261203
TYPE_F, TYPE_S, TYPE_P, TYPE_A, TYPE_FS, TYPE_I, TYPE_O, TYPE_I_C, TYPE_O_C, TYPE_Q = range(10)

# Byte layout of the single-component MIXTURE record (1024 bytes).
MIXTURE_SC = np.dtype({
    "names": ["type", "f", "fpc", "p_tensor", "rho", "u", "v", "w", "p", "g", "gpc", "rhoe",
              "energy_flux", "temp"],
    "formats": ["<i2", ("<f8", 27), ("<f8", 27), ("<f8", (3, 3)), "<f8", "<f8", "<f8", "<f8", "<f8",
                ("<f8", 27), ("<f8", 27), "<f8", ("<f8", 3), "<f8"],
    "offsets": [0, 8, 224, 440, 512, 520, 528, 536, 544, 552, 768, 984, 992, 1016],
    "itemsize": 1024,
})


def blank_sc(NX, NY, NZ):
    """Cells as the reference constructor leaves them (lbm.hpp:59-83): fluid type,
    rho = 1, zero velocity, p = T = 1/3; populations zero."""
    c = np.zeros((NX + 2, NY + 2, NZ + 2), dtype=MIXTURE_SC)
    c["type"] = TYPE_F
    c["rho"] = 1.0
    c["p"] = 1.0 / 3.0
    c["temp"] = 1.0 / 3.0
    return c


def tgv_sc(N, Ma=0.1, Re=400.0, R=0.1, T0=1.0, gamma=1.4, prtl=0.71, noise=1e-3, seed=SEED,
           NY=None, NZ=None):
    """Single-component 3-D Taylor-Green vortex in a periodic box (N^3 interior cells).

    u = U sin x cos y cos z, v = -U cos x sin y cos z, w = 0 with x = 2 pi i / N over the
    reference's array index (as in the reference's TAYLOR_GREEN_3D setup, setup.cpp:94-148);
    rho = 1, T = 1 with gas constant R = 0.1, so theta = R T = 0.1; U = Ma * sqrt(gamma theta);
    nu = U (N / 2 pi) / Re; p = (p0 + rho U^2/16 (cos 2x + cos 2y)(cos 2z + 2)) (1 + xi)
    with seeded uniform xi in [-noise, noise] (the density noise reaches rho through
    Init's rho = p / (R T)).  At theta = 1/3 the reference's own single-component scheme
    diverges within 100 steps for Re >= 25 at 32^3 (and at 64^3, Re = 400); theta = 0.1 runs
    the 64^3, Re = 400, Ma = 0.1 case stably for 1000 steps.
    """
    NY = NY or N
    NZ = NZ or N
    c = blank_sc(N, NY, NZ)
    Nx, Ny, Nz = c.shape
    theta = R * T0
    U = Ma * math.sqrt(gamma * theta)
    nu = U * (N / (2.0 * math.pi)) / Re
    i, j, k = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    ghost = (i == 0) | (i == Nx - 1) | (j == 0) | (j == Ny - 1) | (k == 0) | (k == Nz - 1)
    c["type"][ghost] = TYPE_P
    x = 2.0 * math.pi * i / N
    y = 2.0 * math.pi * j / NY
    z = 2.0 * math.pi * k / NZ
    rng = np.random.Generator(np.random.PCG64(seed))
    xi = rng.uniform(-noise, noise, size=c.shape)
    fl = ~ghost
    rho0 = 1.0
    p0 = rho0 * R * T0
    c["u"][fl] = (U * np.sin(x) * np.cos(y) * np.cos(z))[fl]
    c["v"][fl] = (-U * np.cos(x) * np.sin(y) * np.cos(z))[fl]
    c["w"][fl] = 0.0
    p = (p0 + rho0 * U * U / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)) * (1.0 + xi)
    c["p"][fl] = p[fl]
    c["temp"][fl] = T0
    params = dict(nu=nu, R=R, gamma=gamma, prtl=prtl, U=U)
    return c, params


def channel_sc(NX=24, NY=10, NZ=8, u_in=0.05, R=0.1, T0=1.0, T_wall=0.9, gamma=1.4, prtl=0.71,
               nu=0.02, seed=SEED, noise=1e-3, freeslip_z=False):
    """Single-component channel exercising every single-component boundary type:
    inflow ghost (TYPE_I, prescribed u, T) at i = 0, outflow ghost (TYPE_O, prescribed p)
    at i = Nx-1, solid walls (TYPE_S, wall temperature T_wall) at j = 0 and an adiabatic
    wall (TYPE_A) at j = Ny-1; z is periodic, or free-slip (TYPE_FS) when freeslip_z.
    The interior starts at rest with seeded pressure noise."""
    c = blank_sc(NX, NY, NZ)
    Nx, Ny, Nz = c.shape
    rng = np.random.Generator(np.random.PCG64(seed))
    p0 = R * T0
    c["temp"] = T0
    c["p"] = p0 * (1.0 + rng.uniform(-noise, noise, size=c.shape))
    t = c["type"]
    if freeslip_z:
        t[:, :, 0] = TYPE_FS
        t[:, :, Nz - 1] = TYPE_FS
    else:
        t[:, :, 0] = TYPE_P
        t[:, :, Nz - 1] = TYPE_P
    t[:, 0, :] = TYPE_S
    t[:, Ny - 1, :] = TYPE_A
    t[0, :, :] = TYPE_I
    t[Nx - 1, :, :] = TYPE_O
    c["u"][0, :, :] = u_in
    c["temp"][0, :, :] = T0
    c["temp"][:, 0, :] = T_wall
    c["p"][Nx - 1, :, :] = p0
    c["u"][1:Nx - 1, 1:Ny - 1, 1:Nz - 1] = 0.0
    params = dict(nu=nu, R=R, gamma=gamma, prtl=prtl)
    return c, params


# ---------------------------------------------------------------------------------------
# Multicomponent states (MULTICOMP on): the mixture record (600 bytes) and one species
# record per species (472 bytes), src/headers/lbm.hpp:56-102.
# ---------------------------------------------------------------------------------------
MIXTURE_MC = np.dtype({
    "names": ["type", "p_tensor", "rho", "u", "v", "w", "p", "g", "gpc", "rhoe", "energy_flux", "temp", "HRR"],
    "formats": ["<i2", ("<f8", (3, 3)), "<f8", "<f8", "<f8", "<f8", "<f8", ("<f8", 27), ("<f8", 27), "<f8",
                ("<f8", 3), "<f8", "<f8"],
    "offsets": [0, 8, 80, 88, 96, 104, 112, 120, 336, 552, 560, 584, 592],
    "itemsize": 600,
})
SPECIES = np.dtype({
    "names": ["X", "rho", "f", "fpc", "u", "v", "w"],
    "formats": ["<f8", "<f8", ("<f8", 27), ("<f8", 27), "<f8", "<f8", "<f8"],
    "offsets": [0, 8, 16, 232, 448, 456, 464],
    "itemsize": 472,
})

# lattice units of the reference's flame cases (units.set_m_kg_s(20e-6, 1e-9), setup.cpp:2758):
# dx = 20 um, dt = 1 ns, temperature unit 12000 K (units.hpp:32-44)
FLAME_UNITS = (20e-6, 1e-9)
K_UNIT = 12000.0
ONE_ATM = 101325.0
SPECIES_MIN = 1e-8


def p_lattice(p_si, units=FLAME_UNITS):
    """units.p(): SI pressure to lattice units, in float arithmetic like the reference."""
    m = np.float32(units[0])
    s = np.float32(units[1])
    kg = np.float32(float(m) ** 3)
    return float(np.float32(p_si) * (m * (s * s)) / kg)


def t_lattice(T_si):
    """units.temp(): SI temperature to lattice units (float)."""
    return float(np.float32(T_si) / np.float32(K_UNIT))


def u_lattice(u_si, units=FLAME_UNITS):
    m = np.float32(units[0])
    s = np.float32(units[1])
    return float(np.float32(u_si) * s / m)


def _blank_mc(NX, NY, NZ, ns):
    shape = (NX + 2, NY + 2, NZ + 2)
    mix = np.zeros(shape, dtype=MIXTURE_MC)
    mix["type"] = TYPE_F
    mix["rho"] = 1.0
    mix["p"] = 1.0 / 3.0
    mix["temp"] = 1.0 / 3.0
    sp = [np.zeros(shape, dtype=SPECIES) for _ in range(ns)]
    return mix, sp


def mixing_layer_mc(mech, N=16, NY=None, NZ=None, Y_H2=0.03, T_lo=300.0, T_hi=1000.0, amp=0.1, width=None,
                    u_si=0.0, seed=SEED, periodic_x=True, fuel="H2"):
    """Seeded sinusoidal H2/air interface (the non-reacting mixing case): H2 (or `fuel`) mass
    fraction from 0 to Y_H2 (balance air, O2:N2 = 0.233:0.767 by mass), T from T_lo to T_hi across a
    tanh interface at x0 + A sin(2 pi y/L + phi1) sin(2 pi z/L + phi2) with random phases;
    p = 1 atm; the remaining species at mole fraction 1e-8.  With periodic_x the domain
    holds a hot H2 slab between two such interfaces (fully periodic box).  The tanh width
    defaults to max(1.5, N/8) cells: sharper 300 K -> 1000 K fronts drive the reference's own
    solver unstable within a few steps at 32^3."""
    width = max(1.5, N / 8.0) if width is None else width
    NY = NY or N
    NZ = NZ or N
    names = mech.species_names()
    ns = len(names)
    mix, sp = _blank_mc(N, NY, NZ, ns)
    Nx, Ny, Nz = mix.shape
    rng = np.random.Generator(np.random.PCG64(seed))
    ph = rng.uniform(0, 2 * np.pi, size=4)
    i, j, k = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    ghost = (i == 0) | (i == Nx - 1) | (j == 0) | (j == Ny - 1) | (k == 0) | (k == Nz - 1)
    mix["type"][ghost] = TYPE_P
    A = amp * N
    y2 = 2 * np.pi * j / NY
    z2 = 2 * np.pi * k / NZ
    x0 = 0.3 * N + A * np.sin(y2 + ph[0]) * np.sin(z2 + ph[1])
    x1 = 0.7 * N + A * np.sin(y2 + ph[2]) * np.sin(z2 + ph[3])
    if periodic_x:
        s = 0.5 * (1 + np.tanh((i - x0) / width)) * 0.5 * (1 + np.tanh((x1 - i) / width))
    else:
        s = 0.5 * (1 + np.tanh((i - x0) / width))
    W = np.array([mech.W[kk] for kk in range(ns)])
    Y = np.zeros(mix.shape + (ns,))
    Y[..., names.index(fuel)] = Y_H2 * s
    air = 1.0 - Y[..., names.index(fuel)]
    Y[..., names.index("O2")] = 0.233 * air
    Y[..., names.index("N2")] = 0.767 * air
    X = Y / W
    X /= X.sum(-1, keepdims=True)
    for a, n in enumerate(names):
        if n not in (fuel, "O2", "N2"):
            X[..., a] = SPECIES_MIN
    X[..., names.index(fuel)] = np.maximum(X[..., names.index(fuel)], SPECIES_MIN)
    X /= X.sum(-1, keepdims=True)
    fl = ~ghost
    T = T_lo + (T_hi - T_lo) * s
    mix["temp"][fl] = np.float32(T[fl] / K_UNIT).astype(np.float64)
    mix["p"][fl] = p_lattice(ONE_ATM)
    mix["u"][fl] = u_lattice(u_si)
    for a in range(ns):
        sp[a]["X"][fl] = X[..., a][fl]
    return mix, sp


def _mole_fractions(mech, Y_named):
    """Mole fractions of a composition given by mass fraction per species name (the rest
    at SPECIES_MIN mole fraction), normalised."""
    names = mech.species_names()
    ns = len(names)
    W = np.array([mech.W[k] for k in range(ns)])
    Y = np.zeros(ns)
    for n_, y in Y_named.items():
        Y[names.index(n_)] = y
    X = Y / W
    X /= X.sum()
    X = np.maximum(X, SPECIES_MIN)
    return X / X.sum()


def flame_channel_mc(mech, NX=32, NY=8, NZ=8, T_u=300.0, T_b=1800.0, T_wall=300.0, width=None, seed=SEED):
    """Reacting H2-air channel with characteristic boundaries (the shape of config 3):
    stoichiometric H2-air (X_H2 : X_O2 : X_N2 = 0.2958 : 0.1479 : 0.5563) at 1 atm and
    T_u, a tanh ignition kernel to T_b at mid-x (width max(1.5, NX/16) cells); x ends are
    TYPE_O_C ghosts (target pressure 1 atm), y walls TYPE_S at T_wall, z periodic.  A
    seeded sinusoidal ripple on the kernel position breaks the y/z symmetry."""
    width = max(1.5, NX / 16.0) if width is None else width
    names = mech.species_names()
    ns = len(names)
    mix, sp = _blank_mc(NX, NY, NZ, ns)
    Nx, Ny, Nz = mix.shape
    rng = np.random.Generator(np.random.PCG64(seed))
    ph = rng.uniform(0, 2 * np.pi, size=2)
    i, j, k = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    mix["type"][(k == 0) | (k == Nz - 1)] = TYPE_P
    mix["type"][(i == 0) | (i == Nx - 1)] = TYPE_O_C
    mix["type"][(j == 0) | (j == Ny - 1)] = TYPE_S
    W = np.array([mech.W[kk] for kk in range(ns)])
    Xu = np.full(ns, SPECIES_MIN)
    for n_, x in (("H2", 0.2958), ("O2", 0.1479), ("N2", 0.5563)):
        Xu[names.index(n_)] = x
    Xu /= Xu.sum()
    xc = 0.5 * NX + 0.05 * NX * np.sin(2 * np.pi * j / NY + ph[0]) * np.sin(2 * np.pi * k / NZ + ph[1])
    s = 0.5 * (np.tanh((i - xc + 0.125 * NX) / width) - np.tanh((i - xc - 0.125 * NX) / width))
    T = T_u + (T_b - T_u) * s
    solid = mix["type"] == TYPE_S
    T[solid] = T_wall
    gas_cells = ~solid
    mix["temp"][gas_cells] = np.float32(T[gas_cells] / K_UNIT).astype(np.float64)
    mix["temp"][solid] = t_lattice(T_wall)
    mix["p"][gas_cells] = p_lattice(ONE_ATM)
    for a in range(ns):
        sp[a]["X"][gas_cells] = Xu[a]
    del W
    return mix, sp


def inflow_layer_mc(mech, NX=32, NY=8, NZ=8, u_in_si=5.0, T_in=300.0, Y_H2=0.03, T_hot=1000.0, width=None,
                    seed=SEED):
    """H2/air mixing layer between a characteristic inflow and outflow (the shape of
    config 2): x = 0 ghosts TYPE_I_C carry the inflow target (air at T_in, u = u_in_si),
    x = NX+1 ghosts TYPE_O_C the target pressure of 1 atm, y and z periodic.  Inside, the
    seeded interface of mixing_layer_mc (H2-laden hot gas downstream of x0) advected at
    the inflow velocity."""
    width = max(1.5, NX / 8.0) if width is None else width
    mix, sp = mixing_layer_mc(mech, N=NX, NY=NY, NZ=NZ, Y_H2=Y_H2, T_lo=T_in, T_hi=T_hot, width=width,
                              u_si=u_in_si, seed=seed, periodic_x=False)
    Nx = mix.shape[0]
    ns = len(sp)
    mix["type"][0] = TYPE_I_C
    mix["type"][Nx - 1] = TYPE_O_C
    Xair = _mole_fractions(mech, {"O2": 0.233, "N2": 0.767})
    for (ii, T, X) in ((0, T_in, Xair), (Nx - 1, None, None)):
        if X is None:  # outflow ghost: the state next to it, pressure 1 atm
            mix["temp"][ii] = mix["temp"][ii - 1]
            mix["u"][ii] = mix["u"][ii - 1]
            for a in range(ns):
                sp[a]["X"][ii] = sp[a]["X"][ii - 1]
        else:
            mix["temp"][ii] = t_lattice(T)
            mix["u"][ii] = u_lattice(u_in_si)
            for a in range(ns):
                sp[a]["X"][ii] = X[a]
        mix["p"][ii] = p_lattice(ONE_ATM)
    return mix, sp


# ---------------------------------------------------------------------------------------
# Decaying turbulent reacting H2/air layer (config 4's case), generated plane range by plane
# range so that lattices whose AoS copy does not fit in host memory (83 GB at 256^3) can be
# uploaded in pieces (lbmgpu_upload_planes).
# ---------------------------------------------------------------------------------------
# units.set_m_kg_s(dx, dt) with dx = 2 um and dx / dt = 4000 m/s.  The reference's species
# equilibria are product forms in theta_a = R_a T (dt/dx)^2, so the light species bound dx/dt
# from below (theta_H of the hot side 0.77, theta_H2 0.39 at 1500 K); the sound speed then
# bounds the velocity: u' = 0.02 is Mach 0.23 in 300 K air.  At u' = 0.05 (Mach 0.58) the
# reference's scheme diverges within 60 steps at every such (dx, dt); at u' = 0.02 it runs
# 180 steps at the 256^3 case's resolution (64 cells per energy-containing wavelength).
TURB_UNITS = (2e-6, 2e-6 / 4000.0)


def turbulence_field(N, u_rms=0.02, k0=4.0, seed=SEED):
    """Seeded isotropic, solenoidal velocity field on an N^3 periodic box (lattice units):
    random-phase Fourier synthesis with the energy spectrum E(k) ~ (k/k0)^4 exp(-2 (k/k0)^2)
    (peak at k = k0), each mode's random complex amplitude projected onto the plane normal
    to its wave vector (divergence-free) and scaled to sqrt(E(k) / (4 pi k^2)); the real
    part of the inverse transform, rescaled so the rms of each component, averaged over the
    three, is u_rms.  Returns float64 arrays (u, v, w) of shape (N, N, N)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    k1 = np.fft.fftfreq(N, 1.0 / N)
    kx, ky, kz = np.meshgrid(k1, k1, k1, indexing="ij", sparse=True)
    k2 = kx * kx + ky * ky + kz * kz
    kk = np.sqrt(k2)
    E = (kk / k0) ** 4 * np.exp(-2.0 * (kk / k0) ** 2)
    amp = np.where(kk > 0, np.sqrt(E / (4.0 * np.pi * np.where(k2 > 0, k2, 1.0))), 0.0)
    a = [rng.standard_normal((N, N, N)) + 1j * rng.standard_normal((N, N, N)) for _ in range(3)]
    kd = (kx * a[0] + ky * a[1] + kz * a[2]) / np.where(k2 > 0, k2, 1.0)
    vel = []
    for c, kc in zip(a, (kx, ky, kz)):
        c -= kc * kd
        c *= amp
        vel.append(np.real(np.fft.ifftn(c)))
    del a, kd
    rms = math.sqrt(sum(float(np.mean(v * v)) for v in vel) / 3.0)
    return tuple(v * (u_rms / rms) for v in vel)


def turbulent_layer_mc(mech, N=32, i0=0, i1=None, field=None, Y_H2=0.03, T_lo=300.0, T_hi=1500.0, width=None,
                       u_rms=0.02, k0=4.0, seed=SEED, units=TURB_UNITS, x_trace=1e-6):
    """The x-planes i0 .. i1-1 (ghosts counted; default all N + 2) of a decaying turbulent
    reacting H2/air layer on an N^3 interior: H2-laden air (mass fraction Y_H2, balance air
    with O2:N2 = 0.233:0.767 by mass) at T_hi above a tanh interface in y at mid-height
    (width max(1.5, N/16) cells), air at T_lo below it, p = 1 atm, the other species at mole
    fraction x_trace (1e-6: at the 1e-8 of the other cases they sit on the reference's
    species density floor SPECIES_MIN, where its species update -- the skip rule,
    src/lbm-collision.cpp:512-513 -- makes any flow with velocity diverge within 20 steps);
    the velocity field of turbulence_field(N, u_rms, k0, seed) everywhere.
    Periodic (TYPE_P ghosts) in x and z; TYPE_O_C characteristic outflow ghosts (target
    pressure 1 atm) on both y faces, overriding the periodic ghosts at the edges.  Every
    ghost cell carries the fields of its nearest interior cell.  `field` reuses a
    turbulence_field result across plane ranges."""
    width = max(1.5, N / 16.0) if width is None else width
    i1 = N + 2 if i1 is None else i1
    if field is None:
        field = turbulence_field(N, u_rms=u_rms, k0=k0, seed=seed)
    names = mech.species_names()
    ns = len(names)
    shape = (i1 - i0, N + 2, N + 2)
    mix = np.zeros(shape, dtype=MIXTURE_MC)
    sp = [np.zeros(shape, dtype=SPECIES) for _ in range(ns)]
    mix["rho"] = 1.0
    i = np.arange(i0, i1)[:, None, None]
    j = np.arange(N + 2)[None, :, None]
    k = np.arange(N + 2)[None, None, :]
    ty = np.full(shape, TYPE_F, dtype=np.int16)
    ty[np.broadcast_to((i == 0) | (i == N + 1) | (k == 0) | (k == N + 1), shape)] = TYPE_P
    ty[np.broadcast_to((j == 0) | (j == N + 1), shape)] = TYPE_O_C
    mix["type"] = ty
    # fields of the nearest interior cell
    ic = np.clip(np.arange(i0, i1), 1, N) - 1
    jc = np.clip(np.arange(N + 2), 1, N) - 1
    sel = np.ix_(ic, jc, jc)
    for name, comp in zip(("u", "v", "w"), field):
        mix[name] = comp[sel]
    jj = np.clip(j, 1, N).astype(np.float64)
    s = 0.5 * (1.0 + np.tanh((jj - 0.5 * (N + 1)) / width))
    s = np.broadcast_to(s, shape)
    W = np.array([mech.W[q] for q in range(ns)])
    Y = np.zeros(shape + (ns,))
    Y[..., names.index("H2")] = Y_H2 * s
    air = 1.0 - Y[..., names.index("H2")]
    Y[..., names.index("O2")] = 0.233 * air
    Y[..., names.index("N2")] = 0.767 * air
    X = Y / W
    X /= X.sum(-1, keepdims=True)
    for a, n in enumerate(names):
        if n not in ("H2", "O2", "N2"):
            X[..., a] = x_trace
    X[..., names.index("H2")] = np.maximum(X[..., names.index("H2")], x_trace)
    X /= X.sum(-1, keepdims=True)
    T = T_lo + (T_hi - T_lo) * s
    mix["temp"] = np.float32(T / K_UNIT).astype(np.float64)
    mix["p"] = p_lattice(ONE_ATM, units)
    for a in range(ns):
        sp[a]["X"] = X[..., a]
    return mix, sp
