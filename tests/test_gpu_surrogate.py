"""The chemistry surrogate through the C ABI (lbmgpu_surrogate_*): the fused tensor-core
forward pass against a torch FP32 reference that rounds operands to BF16 like the device
(each feature as a BF16 value plus a BF16 remainder),
the first Adam step and the backward pass's raw gradients against torch autograd, learning a
smooth function, and the whole
collect -> train -> replace loop on the reacting fixture (audit error, exact element
conservation of the projected prediction)."""
import numpy as np
import pytest
import torch

import lbmgpu
import mech
import workloads as W
from mc_common import case

pytestmark = pytest.mark.gpu

SHAPES = [("W1", (128, 12)), ("b1", (128,)), ("W2", (128, 128)), ("b2", (128,)), ("W3", (128, 128)), ("b3", (128,)),
          ("W4", (10, 128)), ("b4", (10,)), ("x_mean", (12,)), ("x_std", (12,)), ("x_lo", (12,)), ("x_hi", (12,)),
          ("y_mean", (10,)), ("y_std", (10,))]


def unpack(buf):
    out, p = {}, 0
    for k, sh in SHAPES:
        n = int(np.prod(sh))
        out[k] = buf[p:p + n].reshape(sh).copy()
        p += n
    assert p == lbmgpu.SUR_NPARAMS
    return out


def pack(d):
    return np.concatenate([np.asarray(d[k], np.float32).reshape(-1) for k, _ in SHAPES])


def seeded_params(seed=7):
    rng = np.random.default_rng(seed)
    d = {}
    for k, sh in SHAPES[:8]:
        fan = sh[1] if len(sh) == 2 else 128
        d[k] = (rng.uniform(-1, 1, sh) * (np.sqrt(6.0 / fan) if len(sh) == 2 else 0.1)).astype(np.float32)
    d["x_mean"] = rng.normal(size=12).astype(np.float32)
    d["x_std"] = rng.uniform(0.5, 2.0, 12).astype(np.float32)
    d["x_lo"] = np.full(12, -1e9, np.float32)
    d["x_hi"] = np.full(12, 1e9, np.float32)
    d["y_mean"] = rng.normal(size=10).astype(np.float32)
    d["y_std"] = rng.uniform(0.5, 2.0, 10).astype(np.float32)
    return d


def bf16(t):
    return t.to(torch.bfloat16).to(torch.float32)


def torch_forward(d, x, round_bf16=True):
    r = bf16 if round_bf16 else (lambda t: t)
    t = lambda a: torch.tensor(a, dtype=torch.float32)  # noqa: E731
    h = (t(x) - t(d["x_mean"])) / t(d["x_std"])
    h = r(h) + r(h - r(h))  # the device's BF16 value + BF16 remainder of each feature
    for L in (1, 2, 3):
        h = r(torch.nn.functional.gelu(h @ r(t(d[f"W{L}"])).T + t(d[f"b{L}"]), approximate="tanh"))
    out = h @ r(t(d["W4"])).T + t(d["b4"])
    return out * t(d["y_std"]) + t(d["y_mean"])


def lattice():
    m, mix, sp, _, _ = case("mc_react8.npz")
    lat = lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=W.FLAME_UNITS,
                         chem=lbmgpu.CHEM_ROSENBROCK)
    return lat, m, mix, sp


def test_surrogate_forward_matches_torch_bf16_reference():
    d = seeded_params()
    x = np.random.default_rng(3).normal(size=(1000, 12)).astype(np.float32) * d["x_std"] + d["x_mean"]
    lat, *_ = lattice()
    with lat:
        lat.surrogate_params(pack(d))
        got = lat.surrogate_eval(x)
        back = unpack(lat.surrogate_params())
    for k in d:
        np.testing.assert_array_equal(back[k], d[k])
    ref = torch_forward(d, x).numpy()
    err = np.abs((got - ref) / d["y_std"]).max()  # in standardised output units
    assert err < 2e-2, err


def test_surrogate_first_adam_step_follows_torch_gradient():
    d = seeded_params(11)
    d["x_lo"][:] = 0.0
    d["x_hi"][:] = 0.0
    rng = np.random.default_rng(5)
    n = 512
    x = (rng.normal(size=(n, 12)) * d["x_std"] + d["x_mean"]).astype(np.float32)
    y = (rng.normal(size=(n, 10)) * d["y_std"] + d["y_mean"]).astype(np.float32)
    lr = 1e-3
    lat, *_ = lattice()
    with lat:
        lat.surrogate_params(pack(d))
        lat.surrogate_load_samples(x, y)
        loss = lat.surrogate_train(epochs=1, batch=n, lr=lr, seed=1, refit=False)
        new = unpack(lat.surrogate_params())
    # torch: the same standardised MSE, FP32, one gradient
    P = {k: torch.tensor(d[k], requires_grad=k[0] in "Wb") for k in d}
    h = (torch.tensor(x) - P["x_mean"]) / P["x_std"]
    for L in (1, 2, 3):
        h = torch.nn.functional.gelu(h @ P[f"W{L}"].T + P[f"b{L}"], approximate="tanh")
    out = h @ P["W4"].T + P["b4"]
    tl = ((out - (torch.tensor(y) - P["y_mean"]) / P["y_std"]) ** 2).mean()
    tl.backward()
    assert abs(loss - tl.item()) < 0.02 * tl.item()
    for k in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        g = P[k].grad.numpy()
        step = new[k] - d[k]
        # Adam's first step moves every parameter by lr against the sign of its gradient
        big = np.abs(g) > 1e-3 * np.abs(g).max()
        assert np.allclose(np.abs(step[big]), lr, rtol=0.02), k
        agree = np.sign(step) == -np.sign(g)
        assert (np.abs(g) * agree).sum() / np.abs(g).sum() > 0.99, k


def test_surrogate_backward_gradients_match_autograd():
    """The tensor-core backward pass (k_gemm_tn on tcgen05: dW = dZ^T X, dH = dZ W, GELU',
    column-summed bias gradients) against torch autograd of the same network and loss on the
    same minibatch, tensor by tensor: the device's gradients of one 512-row batch
    (lbmgpu_surrogate_grads) within 2e-2 of autograd's in the relative 2-norm, and 90 % of
    every tensor's entries within 5e-2 of autograd's largest entry of that tensor.  The
    reference rounds the weights and each layer's activations to BF16 as the device's forward
    pass does; the device also rounds the backward operands to BF16 (FP32 accumulation),
    which the tolerance covers."""
    d = seeded_params(13)
    d["x_lo"][:] = 0.0
    d["x_hi"][:] = 0.0
    rng = np.random.default_rng(17)
    n = 512
    x = (rng.normal(size=(n, 12)) * d["x_std"] + d["x_mean"]).astype(np.float32)
    y = (rng.normal(size=(n, 10)) * d["y_std"] + d["y_mean"]).astype(np.float32)
    lat, *_ = lattice()
    with lat:
        lat.surrogate_params(pack(d))
        lat.surrogate_load_samples(x, y)
        lat.surrogate_train(epochs=1, batch=n, lr=1e-6, seed=1, refit=False)
        got = unpack(lat.surrogate_grads())
    P = {k: torch.tensor(d[k], requires_grad=k[0] in "Wb") for k in d}
    h = (torch.tensor(x) - P["x_mean"]) / P["x_std"]
    h = bf16(h) + bf16(h - bf16(h))
    for L in (1, 2, 3):
        h = bf16(torch.nn.functional.gelu(h @ bf16(P[f"W{L}"]).T + P[f"b{L}"], approximate="tanh"))
    out = h @ bf16(P["W4"]).T + P["b4"]
    ((out - (torch.tensor(y) - P["y_mean"]) / P["y_std"]) ** 2).mean().backward()
    for k in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        want = P[k].grad.numpy()
        rel = np.linalg.norm(got[k] - want) / np.linalg.norm(want)
        close = np.abs(got[k] - want) <= 5e-2 * np.abs(want).max()
        print(k, f"rel {rel:.2e}", f"close {close.mean():.3f}")
        assert rel < 2e-2, (k, rel)
        assert close.mean() > 0.9, k


def test_surrogate_learns_a_smooth_map():
    rng = np.random.default_rng(9)
    n = 16384
    x = rng.uniform(-1, 1, size=(n, 12)).astype(np.float32)
    A = rng.normal(size=(12, 10)).astype(np.float32) / 3
    y = (np.sin(x @ A) + 0.3 * (x[:, :10] ** 2)).astype(np.float32)
    lat, *_ = lattice()
    with lat:
        lat.surrogate_load_samples(x[:12288], y[:12288])
        first = lat.surrogate_train(epochs=1, batch=1024, lr=3e-3, seed=2)
        last = lat.surrogate_train(epochs=40, batch=1024, lr=3e-3, seed=3)
        pred = lat.surrogate_eval(x[12288:])
    assert last < 0.05 * first, (first, last)
    rms = np.sqrt(((pred - y[12288:]) ** 2).mean(0)) / y.std(0)
    assert rms.max() < 0.25, rms


def element_totals(m, s, ns):
    return np.array([sum(s[5 + a] / m.W[a] * m.elements[a][e] for a in range(ns)) for e in range(3)])


def test_surrogate_replaces_the_integrator_on_the_reacting_fixture():
    lat, m, mix, sp = lattice()
    with lat:
        lat.upload(mix, sp)
        lat.init()
        lat.surrogate_collect(True, stride=1, capacity=mix.size * 60)
        lat.step(60)
        assert lat.synchronize() == 0
        st = lat.surrogate_stats()
        assert st["samples"] == mix.size * 60
        lat.surrogate_collect(False)
        loss = lat.surrogate_train(epochs=200, batch=1024, lr=2e-3, seed=4)
        assert loss < 0.05, loss
        # every cell audited: the integrator's result is used, the network is scored
        lat.surrogate_enable(True, audit_period=1)
        lat.step(5)
        assert lat.synchronize() == 0
        st = lat.surrogate_stats()
        assert st["cells_audited"] == 5 * int((mix["type"] == 0).sum())
        audit_err = st["audit_rel_err"]
        # the network in charge (no audit): element totals change only through transport,
        # exactly as in a step of the integrator from the same state
        c = mix.copy()
        s_ = [a.copy() for a in sp]
        lat.download(c, s_)
        e0 = element_totals(m, lat.sums(), len(sp))
        lat.surrogate_enable(True, audit_period=0)
        lat.step(1)
        assert lat.synchronize() == 0
        st = lat.surrogate_stats()
        assert st["cells_predicted"] > 0
        e_sur = element_totals(m, lat.sums(), len(sp))
        lat.upload(c, s_)
        lat.surrogate_enable(False)
        lat.step(1)
        e_int = element_totals(m, lat.sums(), len(sp))
    # the chemistry source conserves the elements exactly in both (the correction's exactness
    # is tested on the host); what moves the totals is the LBM's density floor on the trace
    # species, ~1e-9 of the totals per step in either run
    assert np.all(np.abs(e_int - e0) <= 1e-8 * np.abs(e0)), e_int - e0
    assert np.all(np.abs(e_sur - e0) <= 1e-8 * np.abs(e0)), e_sur - e0
    print("surrogate audit: relative L1 error of dY", audit_err)
    assert audit_err < 0.05, audit_err


def test_surrogate_augment_rows_are_integrator_labelled(tmp_path):
    """lbmgpu_surrogate_augment: the appended rows are perturbed states (mass fractions
    summing to 1, T within the requested factor of the source rows' range) labelled by the
    integrator -- the host build of the same ROS2 step (tests/host/mc_host.cpp, ros2_host),
    started from each row's stored features, gives the same dY and dT to the rounding of
    the FP32 feature storage."""
    import ctypes

    from mc_common import build_host_lib
    lat, m, mix, sp = lattice()
    with lat:
        lat.upload(mix, sp)
        lat.init()
        lat.surrogate_collect(True, stride=1, capacity=mix.size * 4)
        lat.step(4)
        assert lat.synchronize() == 0
        lat.surrogate_collect(False)
        n0 = lat.surrogate_stats()["samples"]
        lat.surrogate_augment(3000, span_y=1.5, span_t=0.01, y_trace=1e-3, seed=3)
        assert lat.surrogate_stats()["samples"] == n0 + 3000
        x, y, v = lat.surrogate_samples()
    src_x = x[:n0][v[:n0]]
    ax, ay = x[n0:][v[n0:]].astype(np.float64), y[n0:][v[n0:]].astype(np.float64)
    assert v[n0:].mean() > 0.99
    assert np.abs(ax[:, 2:11].sum(1) - 1.0).max() < 1e-5
    assert ax[:, 0].min() >= src_x[:, 0].min() * np.exp(-0.0101)
    assert ax[:, 0].max() <= src_x[:, 0].max() * np.exp(0.0101)
    L = build_host_lib(tmp_path)
    L.ros2_host.restype = ctypes.c_long
    L.ros2_host.argtypes = [ctypes.POINTER(mech.Mech), ctypes.c_long] + [ctypes.c_void_p] * 3 + [ctypes.c_double]
    Wk = np.array([m.W[k] for k in range(9)])
    Y = np.ascontiguousarray(ax[:, 2:11])
    T = np.ascontiguousarray(ax[:, 0])
    rho = np.ascontiguousarray(np.exp(ax[:, 1]) / (8314.46261815324 * T * (Y / Wk).sum(1)))
    Y0, T0 = Y.copy(), T.copy()
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    assert L.ros2_host(ctypes.byref(m), len(T), P(rho), P(Y), P(T), float(ax[0, 11])) == 0
    dY, dT = Y - Y0, T - T0
    err = np.abs(dY[:, :8] - ay[:, :8]).sum() / np.abs(dY[:, :8]).sum()
    assert err < 1e-4, err
    assert np.abs(dT - ay[:, 9]).max() <= 1e-4 * np.abs(dT).max() + 1e-6


def test_surrogate_gains_over_the_integrator():
    """What the trained network gains over the method without it, on a reacting channel
    (258x66x66 with ghosts, 1.1 M cells: outflow ends, TMS walls), trained on 40 integrator
    steps: from the same state, 10 steps with the surrogate (1 % audit) and 10 steps of plain
    ROS2.  The chemistry kernels (the surrogate's features, network, use of the prediction and
    integrator list, against the integrator's kernel; the transport kernel both share is not
    counted) take at most a third of the integrator's time per step, while the heat release
    integrated over cells and steps and the peak temperature stay within 1 % and 0.1 % of the
    integrator's.  (The lattice is large enough for the audited cells' integrations -- 1 % of
    the cells -- to fill the GPU, as they do at the configurations' sizes; on a lattice of a
    few hundred thousand cells their one serial integration each is a fixed latency of about
    0.2 ms that no cell count amortises.)"""
    m = mech.h2_air_9()
    mix, sp = W.flame_channel_mc(m, NX=256, NY=64, NZ=64)
    with lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=W.FLAME_UNITS,
                        chem=lbmgpu.CHEM_ROSENBROCK) as lat:
        lat.upload(mix, sp)
        lat.init()
        lat.surrogate_collect(True, stride=16, capacity=mix.size * 40 // 16 + 40)
        lat.step(40)
        assert lat.synchronize() == 0
        lat.surrogate_collect(False)
        lat.surrogate_augment(lat.surrogate_stats()["samples"] // 2, seed=5)
        lat.surrogate_train(epochs=16, batch=4096, lr=2e-3, seed=5)
        c0, s0 = mix.copy(), [a.copy() for a in sp]
        lat.download(c0, s0)
        res = {}
        for name, on in (("surrogate", True), ("plain", False)):
            lat.upload(c0, s0)
            lat.surrogate_enable(on, audit_period=100)
            lat.step(2)  # warm-up
            lat.upload(c0, s0)
            lat.profile(True)
            hrr, tpk = 0.0, 0.0
            for _ in range(10):
                lat.step(1)
                d = lat.diagnostics()
                hrr += d["hrr"]
                tpk = max(tpk, d["T_max"])
            launches, ms = lat.kernel_times()
            lat.profile(False)
            assert lat.synchronize() == 0
            res[name] = (ms[4] + ms[7], hrr, tpk)  # chemistry kernels; transport (3) is shared
    (t_s, h_s, p_s), (t_p, h_p, p_p) = res["surrogate"], res["plain"]
    print("chemistry ms per 10 steps: surrogate", t_s, "plain", t_p, "heat release", h_s, h_p)
    assert t_s * 3 <= t_p, (t_s, t_p)
    assert abs(h_s - h_p) <= 0.01 * abs(h_p), (h_s, h_p)
    assert abs(p_s - p_p) <= 1e-3 * p_p, (p_s, p_p)


def test_surrogate_online_rows_are_the_audited_integrator_states(tmp_path):
    """Collection during surrogate steps: each step appends one row per fluid cell on the
    audit stride (n % audit_period == the step's phase) -- the cells the integrator takes
    anyway, audited or outside the training box -- labelled by the integrator: the host
    build of the same ROS2 step reproduces every appended row's dY and dT to the rounding of
    the FP32 feature storage; a refresh trains on the grown set."""
    import ctypes

    from mc_common import build_host_lib
    lat, m, mix, sp = lattice()
    P = 7
    fluid = np.flatnonzero(mix["type"].reshape(-1) == 0)
    with lat:
        lat.upload(mix, sp)
        lat.init()
        lat.surrogate_collect(True, stride=1, capacity=mix.size * 10)
        lat.step(10)
        assert lat.synchronize() == 0
        lat.surrogate_collect(False)
        lat.surrogate_train(epochs=20, batch=1024, lr=2e-3, seed=9)
        n0 = lat.surrogate_stats()["samples"]
        lat.surrogate_enable(True, audit_period=P)
        per = -(-mix.size // P)
        lat.surrogate_collect(True, stride=1, capacity=n0 + 3 * per)
        lat.step(3)
        assert lat.synchronize() == 0
        st = lat.surrogate_stats()
        assert st["samples"] == n0 + 3 * per
        x, y, v = lat.surrogate_samples()
        lat.surrogate_train(epochs=1, batch=1024, lr=5e-4, seed=10)  # a refresh on the grown set
        assert lat.synchronize() == 0
    for s_ in range(3):  # every fluid cell of the step's stride wrote its row, nothing else did
        got = set(np.flatnonzero(v[n0 + s_ * per:n0 + (s_ + 1) * per]).tolist())
        assert any(got == set((fluid[fluid % P == ph] // P).tolist()) for ph in range(P)), s_
    new = np.arange(n0, n0 + 3 * per)
    ax, ay = x[new][v[new]].astype(np.float64), y[new][v[new]].astype(np.float64)
    assert len(ax) > 0
    L = build_host_lib(tmp_path)
    L.ros2_host.restype = ctypes.c_long
    L.ros2_host.argtypes = [ctypes.POINTER(mech.Mech), ctypes.c_long] + [ctypes.c_void_p] * 3 + [ctypes.c_double]
    Wk = np.array([m.W[k] for k in range(9)])
    Y = np.ascontiguousarray(ax[:, 2:11])
    T = np.ascontiguousarray(ax[:, 0])
    rho = np.ascontiguousarray(np.exp(ax[:, 1]) / (8314.46261815324 * T * (Y / Wk).sum(1)))
    Y0, T0 = Y.copy(), T.copy()
    Pp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    assert L.ros2_host(ctypes.byref(m), len(T), Pp(rho), Pp(Y), Pp(T), float(ax[0, 11])) == 0
    err = np.abs((Y - Y0)[:, :8] - ay[:, :8]).sum() / np.abs((Y - Y0)[:, :8]).sum()
    assert err < 1e-4, err
