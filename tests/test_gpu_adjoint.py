"""Adjoint of the step against central finite differences of the FP64 forward.

Both the adjoint and the finite differences run the same prescribed dt
schedule (recorded once from a nominal run), so the timestep minimum, which
the adjoint does not differentiate, is held fixed on both sides.  Parameters
are the card values of model 10 / EOS 41 (G, yield stress, hardening modulus,
Mie-Grueneisen slope s) and the impact velocity.  The autograd wrapper below
exists in the tests only.

The step is piecewise smooth: particles at the yield surface change branch,
and the nodal viscosity is |tr|-shaped at tr = 0, which is exactly where
every particle of the still-uniform part of the bar sits.  A central
difference whose step moves some particle across such a kink averages the
two one-sided slopes, so the steps below are small enough to stay on one
branch (relative 1e-6 for the parameters of a sum over all particles; the
measured error then falls to 1e-7 - 1e-9), and the initial-state check moves
positions, which keeps the uniform region uniform.
"""
import dataclasses

import numpy as np
import pytest
import torch

from mcmtop_b200 import _abi
from mcmtop_b200.deck import CM, VEL, taylor_bar
from mcmtop_b200.solver import Solver

pytestmark = pytest.mark.gpu

PREC = _abi.PREC_FP64
DX = 0.8e-3
NSTEPS = 30
EVERY = 8          # checkpoint interval (segments of 8 steps, the last one shorter)
V0 = 190.0
SLOTS = [("strinput", 0), ("strinput", 1), ("strinput", 2), ("eosinput", 1)]
REL_STEP = 1e-4    # central differences, relative step (the bar-shape loss)
REL_STEP_SUM = 1e-6   # for sums over all particles (more particles near a kink)


@pytest.fixture(scope="module")
def lib(gpu_lib):
    return gpu_lib


def deck_with(theta, v0):
    d = taylor_bar(dx=DX, velocity=v0)
    m = d.materials[0]
    for (arr, k), val in zip(SLOTS, theta):
        getattr(m, arr)[k] = val
    return d


def nominal_theta():
    m = taylor_bar(dx=DX).materials[0]
    return np.array([getattr(m, arr)[k] for arr, k in SLOTS])


@pytest.fixture(scope="module")
def dts(lib):
    s = Solver(taylor_bar(dx=DX, velocity=V0), PREC)
    out = [s.dt]
    for _ in range(NSTEPS):
        s.step_a()
        s.dt_update()
        out.append(s.dt)
        s.step_b()
        s.step_c()
    s.close()
    return np.array(out)


def run(theta, v0, dts):
    s = Solver(deck_with(theta, v0), PREC)
    s.adjoint_forward(dts, EVERY)
    st = s.download(["x", "v"])
    return s, st["x"], st["v"]


def fd(fun, theta, v0, rel=REL_STEP):
    """Central differences of fun(theta, v0) in the 4 parameters and v0."""
    out = []
    for k in range(5):
        h = rel * (theta[k] if k < 4 else v0)
        tp, tm = theta.copy(), theta.copy()
        vp, vm = v0, v0
        if k < 4:
            tp[k] += h
            tm[k] -= h
        else:
            vp, vm = v0 + h, v0 - h
        out.append((fun(tp, vp) - fun(tm, vm)) / (2 * h))
    return np.array(out)


def test_adjoint_linear_functional_matches_fd(lib, dts):
    """L = sum W.x + U.v of the final state, random W, U."""
    theta = nominal_theta()
    rng = np.random.default_rng(7)
    s, x, v = run(theta, V0, dts)
    W = rng.standard_normal(x.shape)
    U = rng.standard_normal(v.shape) * 1e2
    pb, x0b, v0b = s.adjoint_backward(W, U)
    s.close()
    grad = np.concatenate([pb[0], [-VEL * v0b[:, 2].sum()]])

    def L(t, v0):
        s2, x2, v2 = run(t, v0, dts)
        s2.close()
        return float((W * x2).sum() + (U * v2).sum())

    ref = fd(L, theta, V0, REL_STEP_SUM)
    rel = np.abs(grad - ref) / np.maximum(np.abs(ref), 1e-300)
    print("adjoint", grad, "fd", ref, "rel", rel)
    assert np.all(rel < 1e-3), (grad, ref, rel)


def test_reverse_constitutive_matches_dual_passes(lib, dts):
    """The hand-written reverse of the model-10 / EOS-41 update (adj_kind 1,
    the default for this bar) and the forward-mode dual passes (adj_kind 2)
    give the same gradients: parameters and initial-state adjoints to 1e-9
    of their largest magnitude (the two differ only in rounding)."""
    theta = nominal_theta()
    rng = np.random.default_rng(5)
    s, x, v = run(theta, V0, dts)
    W = rng.standard_normal(x.shape)
    U = rng.standard_normal(v.shape) * 1e2
    assert s.tuning()["adj_kind"] == 1
    pb1, x01, v01 = s.adjoint_backward(W, U)
    s.set_tuning(adj_kind=2)
    assert s.tuning()["adj_kind"] == 2
    pb2, x02, v02 = s.adjoint_backward(W, U)
    s.close()
    for got, ref, name in ((pb1, pb2, "parameters"), (x01, x02, "x0"), (v01, v02, "v0")):
        err = float(np.max(np.abs(got - ref))) / float(np.max(np.abs(ref)))
        print(name, "reverse vs dual:", err)
        assert err <= 1e-9, (name, err)
    assert np.all(np.abs(pb1[0]) > 0)


def test_adjoint_initial_state_gradient(lib, dts):
    """dL/dx of the initial state along one random direction against FD."""
    theta = nominal_theta()
    rng = np.random.default_rng(11)
    s, x, v = run(theta, V0, dts)
    W = rng.standard_normal(x.shape)
    U = rng.standard_normal(v.shape) * 1e2
    _, x0b, _ = s.adjoint_backward(W, U)
    s.close()
    dirx = rng.standard_normal(x.shape) * (DX * CM * 1e-2)
    base = taylor_bar(dx=DX, velocity=V0)

    def L(eps):
        s2 = Solver(base.replace(x=base.x + eps * dirx), PREC)
        s2.adjoint_forward(dts, EVERY)
        st = s2.download(["x", "v"])
        s2.close()
        return float((W * st["x"]).sum() + (U * st["v"]).sum())

    eps = 1e-3
    ref = (L(eps) - L(-eps)) / (2 * eps)
    got = float((x0b * dirx).sum())
    assert abs(got - ref) <= 1e-3 * abs(ref), (got, ref)


class BarShape(torch.autograd.Function):
    """Final bar length and footprint radius of the Taylor bar as a function
    of (G, yield, hardening, s, impact velocity), with the adjoint as backward."""

    @staticmethod
    def forward(ctx, params, dts):
        p = params.detach().cpu().numpy()
        s, x, _ = run(p[:4], float(p[4]), dts)
        z = x[:, 2]
        imax, imin = int(z.argmax()), int(z.argmin())
        base = np.nonzero(taylor_bar(dx=DX).x[:, 2] < DX * CM)[0]   # the layer that hits the wall
        r = np.hypot(x[base, 0], x[base, 1])
        kr = int(base[r.argmax()])
        ctx.state = (s, imax, imin, kr, x[kr].copy(), float(r.max()), x.shape)
        return torch.tensor([z[imax] - z[imin], r.max()], dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        s, imax, imin, kr, xk, rad, shape = ctx.state
        g = g.detach().cpu().numpy()
        xbar = np.zeros(shape)
        xbar[imax, 2] += g[0]
        xbar[imin, 2] -= g[0]
        xbar[kr, :2] += g[1] * xk[:2] / rad
        pb, _, v0b = s.adjoint_backward(xbar, None)
        s.close()
        grad = np.concatenate([pb[0], [-VEL * v0b[:, 2].sum()]])
        return torch.tensor(grad, dtype=torch.float64), None


def test_autograd_bar_shape_loss_matches_fd(lib, dts):
    theta = nominal_theta()
    p0 = np.concatenate([theta, [V0]])
    with torch.no_grad():
        nominal = BarShape.apply(torch.tensor(p0), dts)
    target = nominal * torch.tensor([0.99, 1.02], dtype=torch.float64)
    params = torch.tensor(p0, requires_grad=True)
    out = BarShape.apply(params, dts)
    loss = ((out - target) ** 2).sum()
    loss.backward()
    grad = params.grad.numpy()

    def L(t, v0):
        with torch.no_grad():
            o = BarShape.apply(torch.tensor(np.concatenate([t, [v0]])), dts)
        return float(((o - target) ** 2).sum())

    ref = fd(L, theta, V0)
    rel = np.abs(grad - ref) / np.maximum(np.abs(ref), 1e-300)
    print("adjoint", grad, "fd", ref, "rel", rel)
    assert np.all(rel < 1e-3), (grad, ref, rel)


def test_fp32_forward_adjoint_agrees_with_fp64(lib, dts):
    """The gradient along the mixed-precision forward (FP32 pair sums) against
    the one along the FP64 forward: the trajectories differ by the mixed
    step's error (about 1e-5 of each field), and so do the gradients."""
    theta = nominal_theta()
    rng = np.random.default_rng(21)
    grads = {}
    for name, prec in (("fp64", PREC), ("mixed", _abi.PREC_MIXED)):
        s = Solver(deck_with(theta, V0), prec)
        s.adjoint_forward(dts, EVERY)
        x = s.download(["x"])["x"]
        if name == "fp64":
            W = rng.standard_normal(x.shape)
        pb, _, v0b = s.adjoint_backward(W, None)
        s.close()
        grads[name] = np.concatenate([pb[0], [-VEL * v0b[:, 2].sum()]])
    rel = np.abs(grads["mixed"] - grads["fp64"]) / np.abs(grads["fp64"])
    print("fp64", grads["fp64"], "mixed", grads["mixed"], "rel", rel)
    assert np.all(rel < 1e-3), rel


def test_adjoint_rejects_unsupported(lib):
    d = taylor_bar(dx=DX)
    s = Solver(d, PREC, reorder_interval=5)
    with pytest.raises(_abi.MCMError):
        s.adjoint_forward(np.full(3, s.dt), 2)
    s.close()


def test_adjoint_regrows_storage_within_a_segment(lib, dts):
    """A segment whose neighbour table overflows is re-run from its checkpoint
    after the table has grown: same forward end state, same gradient."""
    theta = nominal_theta()
    rng = np.random.default_rng(3)
    s1, x1, v1 = run(theta, V0, dts)
    W = rng.standard_normal(x1.shape)
    pb1, x01, _ = s1.adjoint_backward(W, None)
    s1.close()
    s2 = Solver(deck_with(theta, V0), PREC)
    s2.set_tuning(nbr_stride=8)
    s2.adjoint_forward(dts, EVERY)
    st = s2.download(["x", "v"])
    assert np.array_equal(st["x"], x1) and np.array_equal(st["v"], v1)
    s2.set_tuning(nbr_stride=8)   # and once more for the backward's recomputation
    pb2, x02, _ = s2.adjoint_backward(W, None)
    s2.close()
    assert np.allclose(pb2, pb1, rtol=1e-12, atol=0.0)
    assert np.allclose(x02, x01, rtol=1e-9, atol=1e-12 * np.max(np.abs(x01)))


# ------------------------------------------------------ other models and EOS
def _schedule(deck, nsteps):
    s = Solver(deck, PREC)
    out = [s.dt]
    for _ in range(nsteps):
        s.step_a()
        s.dt_update()
        out.append(s.dt)
        s.step_b()
        s.step_c()
    s.close()
    return np.array(out)


def _linear_check(make_deck, slots, dts, rel, seed):
    """Adjoint of L = sum W.x + U.v of the final state with respect to the
    card values `slots` ((array, index, material)) against central
    differences of the FP64 forward along the same dt schedule."""
    rng = np.random.default_rng(seed)
    s = Solver(make_deck({}), PREC)
    s.adjoint_forward(dts, EVERY)
    st = s.download(["x", "v"])
    W = rng.standard_normal(st["x"].shape)
    U = rng.standard_normal(st["v"].shape) * 1e2
    pb, _, _ = s.adjoint_backward(W, U)
    s.close()
    for arr, k, m in slots:
        v0 = getattr(make_deck({}).materials[m], arr)[k]
        h = rel * abs(v0)

        def L(val):
            s2 = Solver(make_deck({(arr, k, m): val}), PREC)
            s2.adjoint_forward(dts, EVERY)
            out = s2.download(["x", "v"])
            s2.close()
            return float((W * out["x"]).sum() + (U * out["v"]).sum())

        ref = (L(v0 + h) - L(v0 - h)) / (2 * h)
        got = pb[m][3 if arr == "eosinput" else k]
        assert abs(got - ref) <= 1e-3 * abs(ref), (arr, k, got, ref)


def _with_cards(deck, changes):
    mats = []
    for m, card in enumerate(deck.materials):
        c = dataclasses.replace(card, strinput=card.strinput.copy(), eosinput=card.eosinput.copy())
        for (arr, k, mm), val in changes.items():
            if mm == m:
                getattr(c, arr)[k] = val
        mats.append(c)
    return deck.replace(materials=mats)


def test_adjoint_model10_with_dyna_grueneisen_eos(lib):
    """Model 10 with EOS 4 (MCM/mcm_eos4c.f90, mcm_eqos4.f90): G, yield stress
    and the slope s1 against central differences."""
    from test_gpu_materials import _model10_eos

    card = _model10_eos(4)
    base = taylor_bar(dx=DX, velocity=V0, material=card)

    def make(changes):
        return _with_cards(base, changes)

    dts = _schedule(base, NSTEPS)
    _linear_check(make, [("strinput", 0, 0), ("strinput", 1, 0), ("eosinput", 1, 0)], dts, REL_STEP_SUM, 31)


def test_adjoint_fluid_column(lib):
    """The null material (model 9, no viscosity) with the polynomial EOS 1,
    gravity and five ghost walls: d/d(c1) and the initial positions along a
    random direction against central differences."""
    from mcmtop_b200.deck import fluid_column

    base = fluid_column(dx=0.01, block=(0.1, 0.06, 0.2), box=(0.4, 0.06, 0.3))

    def make(changes):
        return _with_cards(base, changes)

    dts = _schedule(base, NSTEPS)
    _linear_check(make, [("eosinput", 1, 0)], dts, REL_STEP_SUM, 41)
    rng = np.random.default_rng(43)
    s = Solver(base, PREC)
    s.adjoint_forward(dts, EVERY)
    st = s.download(["x", "v"])
    W = rng.standard_normal(st["x"].shape)
    _, x0b, _ = s.adjoint_backward(W, None)
    s.close()
    dirx = rng.standard_normal(st["x"].shape) * 1e-4

    def L(eps):
        s2 = Solver(base.replace(x=base.x + eps * dirx), PREC)
        s2.adjoint_forward(dts, EVERY)
        out = s2.download(["x"])["x"]
        s2.close()
        return float((W * out).sum())

    ref = (L(1e-3) - L(-1e-3)) / 2e-3
    got = float((x0b * dirx).sum())
    assert abs(got - ref) <= 1e-3 * abs(ref), (got, ref)


def test_adjoint_rejects_models_with_carried_state(lib):
    """Models whose stress state carries between steps beyond what the reverse
    step holds (model 3's back stress, model 9 with viscosity) are rejected."""
    from test_gpu_materials import _solid

    s = Solver(taylor_bar(dx=DX, material=_solid(3)), PREC)
    with pytest.raises(_abi.MCMError):
        s.adjoint_forward(np.full(3, s.dt), 2)
    s.close()
