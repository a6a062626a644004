"""Known-answer and invariant tests of the CPU oracle (no GPU).

The reference publishes no tests or golden data, so the oracle is checked
against closed forms of the cubic B-spline (MCM/mcm_kernel.f90,
MCM/mcm_gradw.f90), first-order consistency of the mixed-corrected gradient
(MCM/mcm_corr_strain.f90), the radial return of model 10
(MCM/mcm_f3dm10.f90), the Mie-Grueneisen pressure (MCM/mcm_eos41p.f90), a
brute-force neighbour search (MCM/mcm_ll_neighbours.f90) and energy bounds.
"""
import ctypes as C
import math

import numpy as np
import pytest

from mcmtop_b200.deck import MaterialCard, taylor_bar
from oracle import pyoracle
from oracle.pyoracle import Oracle


def _w(lib, xi, xj, h):
    a = np.asarray(xi, dtype=np.float64)
    b = np.asarray(xj, dtype=np.float64)
    return lib.mcmo_kernel_w(3, a.ctypes.data_as(C.POINTER(C.c_double)), b.ctypes.data_as(C.POINTER(C.c_double)), h)


def _gw(lib, xi, xj, h):
    a = np.asarray(xi, dtype=np.float64)
    b = np.asarray(xj, dtype=np.float64)
    out = np.zeros(3)
    lib.mcmo_gradw(3, a.ctypes.data_as(C.POINTER(C.c_double)), b.ctypes.data_as(C.POINTER(C.c_double)), h,
                   out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def test_kernel_closed_form(oracle_lib):
    h = 0.7
    c1 = 1.0 / (math.pi * h ** 3)
    for z, expect in [(0.0, c1), (0.5, c1 * ((0.75 * 0.5 - 1.5) * 0.5 * 0.5 + 1)), (1.0, 0.25 * c1),
                      (1.5, c1 / 4 * 0.5 ** 3), (2.0, 0.0), (2.5, 0.0)]:
        w = _w(oracle_lib, [z * h, 0, 0], [0, 0, 0], h)
        assert w == pytest.approx(expect, rel=1e-14, abs=1e-300)
    # gradient: dW/dr * xij/r, zero at r = 0
    for z in (0.3, 0.9, 1.2, 1.9):
        r = z * h
        xi = np.array([r / math.sqrt(3)] * 3)
        g = _gw(oracle_lib, xi, [0, 0, 0], h)
        dw = c1 * (2.25 * z - 3) * z if z < 1 else -0.75 * c1 * (2 - z) ** 2
        assert np.allclose(g, dw * xi / (r * h), rtol=1e-13)
    assert np.all(_gw(oracle_lib, [1, 2, 3], [1, 2, 3], h) == 0)


def test_kernel_normalisation(oracle_lib):
    dx = 1.0
    h = 1.3 * dx
    r = np.arange(-4, 5) * dx
    s = 0.0
    for x in r:
        for y in r:
            for z in r:
                s += _w(oracle_lib, [x + 0.17, y - 0.05, z + 0.31], [0, 0, 0], h) * dx ** 3
    assert abs(s - 1.0) < 2e-3


def _block(n=8, dx=0.1, disctype=1, model10=False, seed=3, jitter=0.01):
    rng = np.random.default_rng(seed)
    g = (np.arange(n) + 0.5) * dx
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1) + rng.uniform(-jitter, jitter, (n ** 3, 3)) * dx
    if model10:
        deck = taylor_bar(dx=1.0e-3)
        mat = deck.materials[0]
    else:
        mat = MaterialCard(model=1, eos=0, rho=8.0)
        mat.strinput[0] = 1.0
        mat.strinput[1] = 0.3
    mat.h = 1.3 * dx
    mat.mass = mat.rho * n ** 3 * dx ** 3
    from mcmtop_b200.deck import Deck

    return Deck(ndim=3, disctype=disctype, tssf=0.3, tcrit_opt=1, materials=[mat], x=x, v=np.zeros_like(x),
                mat=np.ones(n ** 3, dtype=np.int32), dispbc=np.zeros(n ** 3, dtype=np.int32))


def _interior(deck, margin):
    lo, hi = deck.x.min(0), deck.x.max(0)
    return np.all((deck.x > lo + margin) & (deck.x < hi - margin), axis=1)


def test_corrected_gradient_of_linear_fields():
    """MCM/mcm_corr_strain.f90 forms grad v = sum V v_j (B^-1 g_j) with
    B(n,m) = sum V (x_j - x_i)(n) g_j(m): the result is A B B^-T for v = A x + b,
    exact where B is symmetric (regular-lattice interior), about 1% off with
    jitter.  The oracle reproduces both."""
    A = np.array([[0.3, -0.2, 0.1], [0.05, -0.4, 0.25], [-0.15, 0.2, 0.35]])
    sym = 0.5 * (A + A.T)
    skew = 0.5 * (A - A.T)
    deck = _block(disctype=1, jitter=0.0)
    deck.v = deck.x @ A.T + np.array([1.0, -2.0, 0.5])
    orc = Oracle(deck)
    orc.set_scalar("dt", 0.0)   # no half-step shift: the field is linear in the positions used
    orc.step_a()
    inner = _interior(deck, 2.7 * 0.1)
    assert inner.sum() >= 8
    assert np.max(np.abs(orc.get("rod")[inner] - sym)) < 1e-10
    assert np.max(np.abs(orc.get("spin")[inner] - skew)) < 1e-10
    deck = _block(disctype=1, jitter=0.01)
    deck.v = deck.x @ A.T
    orc = Oracle(deck)
    orc.set_scalar("dt", 0.0)
    orc.step_a()
    err = np.max(np.abs(orc.get("rod") - sym)) / np.max(np.abs(sym))
    assert 1e-6 < err < 0.05


def test_basic_gradient_interior_accuracy():
    deck = _block(n=10, disctype=0)
    A = np.array([[0.3, -0.2, 0.1], [0.05, -0.4, 0.25], [-0.15, 0.2, 0.35]])
    deck.v = deck.x @ A.T
    orc = Oracle(deck)
    orc.set_scalar("dt", 0.0)
    orc.step_a()
    rod = orc.get("rod")
    c = deck.x.mean(0)
    inner = np.all(np.abs(deck.x - c) < 0.2, axis=1)
    sym = 0.5 * (A + A.T)
    assert inner.sum() > 20
    assert np.max(np.abs(rod[inner] - sym)) < 0.05 * np.max(np.abs(sym))


def test_rigid_rotation_preserves_stress_invariants():
    deck = _block(disctype=1, jitter=0.0)
    w = np.array([0.2, -0.1, 0.3])
    deck.v = np.cross(np.broadcast_to(w, deck.x.shape), deck.x - deck.x.mean(0))
    orc = Oracle(deck)
    rng = np.random.default_rng(0)
    S = rng.normal(size=(deck.np, 3, 3))
    S = S + S.transpose(0, 2, 1)
    orc.set("sigma", S)
    # the half-step shift of MCM/mcm_strain.f90:27-31 leaves rod = dt/2 W^2 for a
    # rigid rotation; with a small dt the elastic increment is ~1e-8 of sigma
    orc.set_scalar("dt", 1.0e-3)
    orc.step_a()
    inner = _interior(deck, 2.7 * 0.1)
    out = orc.get("sigma")[inner]
    S = S[inner]
    assert np.max(np.abs(orc.get("rod")[inner])) < 1e-4
    # Q sigma Q^T (MCM/mcm_stress_rot1.f90:164-182) keeps trace and norm
    assert np.allclose(np.trace(out, axis1=1, axis2=2), np.trace(S, axis1=1, axis2=2), rtol=1e-7, atol=1e-7)
    assert np.allclose(np.linalg.norm(out, axis=(1, 2)), np.linalg.norm(S, axis=(1, 2)), rtol=1e-7)
    assert np.max(np.abs(out - S)) > 1e-5


def test_radial_return_never_exceeds_yield_surface():
    deck = taylor_bar(dx=0.8e-3)
    orc = Oracle(deck)
    orc.run(60)
    si, ei, g = orc.material_table(1)
    qs, qh = si[1], si[2]
    s = orc.get("s")
    aj2 = 0.5 * (s[:, 0, 0] ** 2 + s[:, 1, 1] ** 2 + s[:, 2, 2] ** 2) + s[:, 0, 1] ** 2 + s[:, 0, 2] ** 2 + s[:, 1, 2] ** 2
    seq = np.sqrt(3 * aj2)
    yield_now = qs + qh * orc.get("efps")
    assert np.all(seq <= yield_now * (1 + 1e-10))
    plastic = orc.get("efps") > 0
    assert plastic.sum() > 50
    # particles yielding in the last step sit on the surface
    assert np.sum(np.isclose(seq[plastic], yield_now[plastic], rtol=1e-10)) > 10


def test_mie_grueneisen_initial_pressure():
    """p(rho, e=0) of MCM/mcm_eos41p.f90:43-63 at a compressed state given by init_rhoe = 1."""
    deck = taylor_bar(dx=1.6e-3)
    rho1 = 8.93 * 1.01
    pard = np.zeros((deck.np, 4))
    pard[:, 2] = rho1
    orc = _create_with_pardata(deck, pard)
    si, ei, g = orc.material_table(1)
    cc, sl, gamma = ei[0], ei[1], ei[4]
    rho0 = deck.materials[0].rho
    mu = rho1 / rho0 - 1.0
    ao = rho0 * (cc * cc)
    bo = ao * (1.0 + 2.0 * (sl - 1.0))
    co = ao * (2.0 * (sl - 1.0) + 3.0 * ((sl - 1.0) * (sl - 1.0)))
    gam = gamma * rho0 / rho1
    f = gam * mu
    ph = ao * mu + bo * (mu * mu) + co * (mu * mu * mu)
    expect = ph * (1.0 - 0.5 * f) + rho1 * gam * 0.0
    assert orc.get("p")[0] == expect
    assert np.all(orc.get("sigma")[:, 0, 0] == -expect)


def _create_with_pardata(deck, pard):
    lib = pyoracle.load()
    o = Oracle.__new__(Oracle)
    o.lib = lib
    d = pyoracle.ODeck()
    d.ndim, d.disctype, d.nummat, d.np = deck.ndim, deck.disctype, 1, deck.np
    d.endtime, d.tssf, d.itss, d.drelax_scale = deck.endtime, deck.tssf, deck.itss, deck.drelax_scale
    d.init_v_opt, d.massopt, d.init_h_opt, d.init_rhoe = 1, 0, 0, 1
    d.tcrit_opt, d.mirr_opt = deck.tcrit_opt, deck.mirr_opt
    for k in range(6):
        d.sym_flag[k] = int(deck.sym_flag[k])
    d.krtype = 1
    m = pyoracle.OMaterial()
    c = deck.materials[0]
    m.model, m.eos, m.rho, m.mass, m.h = c.model, c.eos, c.rho, c.mass, c.h
    for i in range(48):
        m.strinput[i] = float(c.strinput[i])
    for i in range(24):
        m.eosinput[i] = float(c.eosinput[i])
    x = np.ascontiguousarray(deck.x)
    v = np.ascontiguousarray(deck.v)
    mat = np.ascontiguousarray(deck.mat)
    disp = np.ascontiguousarray(deck.dispbc)
    pd = np.ascontiguousarray(pard)
    st = C.c_int()
    o.sim = lib.mcmo_create(C.byref(d), C.byref(m), pyoracle._dp(x), pyoracle._dp(v), pyoracle._ip(mat),
                            pyoracle._ip(disp), pyoracle._dp(pd), C.byref(st))
    assert o.sim, st.value
    o.n, o.nmat = deck.np, 1
    return o


def test_neighbour_sets_match_brute_force():
    deck = taylor_bar(dx=0.8e-3, length=8e-3)
    orc = Oracle(deck)
    x = deck.x
    h = np.full(deck.np, deck.materials[0].h)
    d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    hs = (h[:, None] + h[None, :]) ** 2
    nb = (d2 < hs) & ~np.eye(deck.np, dtype=bool)
    for i in range(deck.np):
        got = np.sort(orc.nbrlist(i + 1)) - 1
        assert np.array_equal(got, np.nonzero(nb[i])[0]), i
    # symmetry of the relation
    nn = orc.get_int("nnbr")
    assert nn.sum() == nb.sum()


def test_ghosts_are_mirror_images():
    deck = taylor_bar(dx=0.8e-3, length=8e-3)
    orc = Oracle(deck)
    par, gx, gv = orc.ghosts()
    x = deck.x[par - 1]
    assert np.array_equal(gx[:, :2], x[:, :2])
    assert np.array_equal(gx[:, 2], -x[:, 2])
    assert np.all(x[:, 2] < 4 * deck.materials[0].h)


def test_initial_dt_is_cfl():
    deck = taylor_bar(dx=0.8e-3)
    orc = Oracle(deck)
    c = orc.get("c")
    vabs = orc.get("vabs")
    h = orc.get("h")
    assert orc.scalar("dt") == 0.3 * np.min(h / (c + vabs))


def test_energy_balance_bounded():
    deck = taylor_bar(dx=0.8e-3)
    orc = Oracle(deck)
    e0 = orc.scalar("totale")
    orc.run(300)
    e1 = orc.scalar("totale")
    assert abs(e1 - e0) / e0 < 0.02
    assert orc.scalar("kinetice") < 0.9 * e0


@pytest.mark.parametrize("case", ["bar", "fluid"])
def test_openmp_build_matches_serial(case):
    """The OpenMP build (the timed CPU baseline) is bitwise the serial one:
    every parallel loop writes only its own particle."""
    from mcmtop_b200.deck import fluid_column

    if case == "bar":
        deck = taylor_bar(dx=0.6e-3)
    else:
        deck = fluid_column(dx=0.01, block=(0.1, 0.06, 0.2), box=(0.4, 0.06, 0.3))
    a = Oracle(deck)
    b = Oracle(deck, openmp=True)
    for _ in range(4):
        a.step()
        b.step()
    for f in ["x", "v", "rho", "e", "p", "sigma", "q", "efps"]:
        assert np.array_equal(a.get(f), b.get(f)), f
    assert np.array_equal(a.get_int("nnbr"), b.get_int("nnbr"))


# ------------------------------------------- variable h and XSPH, restated
def _bar(**kw):
    return taylor_bar(dx=0.8e-3, length=8e-3).replace(**kw)


def test_variable_h_from_strain_rate(oracle_lib):
    # MCM/mcm_update_h.f90:27-36: h = hold (1 + tr dt / ndim) for p >= pcut; hmax their largest h
    orc = Oracle(_bar(h_opt=1))
    for _ in range(3):
        orc.step()
    h0, p0, pc0 = orc.get("h").copy(), orc.get("p").copy(), orc.get("pcut").copy()
    dt = orc.scalar("dt")
    orc.step_a()
    tr = orc.get("tracerod")
    on = p0 >= pc0
    want = np.where(on, h0 * (1.0 + tr * dt / 3.0), h0)
    assert np.array_equal(orc.get("h"), want)
    assert np.array_equal(orc.get("hold")[on], h0[on])
    assert orc.scalar("hmax") == want[on].max()
    assert not np.all(want == h0)


def test_variable_h_from_density(oracle_lib):
    # MCM/mcm_update_h.f90:38-49: h = h0 (rho0 / rho)^(1/ndim) with the density before mcm_rhoupd
    orc = Oracle(_bar(h_opt=2))
    for _ in range(3):
        orc.step()
    orc.step_a()
    rho_prev = orc.get("rhoold")            # mcm_rhoupd saves the density it starts from
    want = orc.get("h0") * np.power(orc.get("rho0") / rho_prev, 1.0 / 3.0)
    np.testing.assert_allclose(orc.get("h"), want, rtol=2e-16, atol=0)


def _w_kernel(r, h):
    c1 = 1.0 / (math.acos(-1.0) * h * h * h)
    z = r / h
    return np.where(z < 1.0, c1 * (((0.75 * z - 1.5) * z) * z + 1.0),
                    np.where(z < 2.0, (c1 / 4.0) * (2.0 - z) ** 3, 0.0))


def test_xsph_restated(oracle_lib):
    # MCM/mcm_update_velocity.f90:61-87 restated on the oracle's state: updated
    # velocities of real neighbours, ghost velocities from the ghosts' creation,
    # W with the neighbour's h, V_j = m_j / ((rho_j + rho_i) / 2), epsilon 0.1
    orc = Oracle(_bar(veloc_opt=1))
    for _ in range(3):
        orc.step()
    orc.step_a()
    orc.dt_update()
    orc.step_b()
    x, v, a = orc.get("x").copy(), orc.get("v").copy(), orc.get("a").copy()
    m, rho, h, rhoold = orc.get("mass"), orc.get("rho"), orc.get("h"), orc.get("rhoold")
    dt, dtold = orc.scalar("dt"), orc.scalar("dtold")
    gpar, gx, gv = orc.ghosts()
    vu = v + a * (0.5 * (dt + dtold))
    sv = np.zeros_like(v)
    nghost = 0
    for i in range(len(x)):
        js = orc.nbrlist(i + 1) - 1
        r = np.sqrt(((x[i] - x[js]) ** 2).sum(axis=1))
        vol = m[js] / (0.5 * (rho[js] + rho[i]))
        sv[i] = ((vol * _w_kernel(r, h[js]))[:, None] * (vu[js] - vu[i])).sum(axis=0)
        gq = orc.g_nbrlist(i + 1) - 1
        if len(gq):
            nghost += len(gq)
            pj = gpar[gq] - 1                 # a ghost carries its parent's mass, h and start-of-step rho
            r = np.sqrt(((x[i] - gx[gq]) ** 2).sum(axis=1))
            vol = m[pj] / (0.5 * (rhoold[pj] + rho[i]))
            sv[i] += ((vol * _w_kernel(r, h[pj]))[:, None] * (gv[gq] - vu[i])).sum(axis=0)
    orc.step_c()
    assert nghost > 0
    want = vu + 0.1 * sv
    np.testing.assert_allclose(orc.get("v"), want, rtol=0, atol=1e-12 * np.abs(want).max())
    assert np.abs(0.1 * sv).max() > 1e-6 * np.abs(want).max()     # the smoothing is not negligible


def test_dynamic_relaxation_restated(oracle_lib):
    # MCM/mcm_update_velocity.f90:33-44: v = drelax_scale v + a (dt + dtold) / 2
    orc = Oracle(_bar(drelax_scale=0.5))
    for _ in range(3):
        orc.step()
    orc.step_a()
    orc.dt_update()
    orc.step_b()
    v, a = orc.get("v").copy(), orc.get("a").copy()
    dtn = 0.5 * (orc.scalar("dt") + orc.scalar("dtold"))
    orc.step_c()
    assert np.array_equal(orc.get("v"), 0.5 * v + a * dtn)


def _rep_restated(orc, deck):
    """Monaghan's repulsive acceleration of MCM/mcm_rep_contact.f90:37-161,
    restated in numpy on the oracle's state (positions after the strain
    half-step round trip, the contact lists of the step's search)."""
    x, h, mass = orc.get("x"), orc.get("h"), orc.get("mass")
    mat = orc.get_int("mat")
    kc = np.asarray(deck.k_cont, dtype=np.float64)
    nc = np.asarray(deck.n_cont, dtype=np.float64)
    gpar, gx, _ = orc.ghosts()
    rep = np.zeros((deck.np, 3))
    for i in range(deck.np):
        cont = orc.contlist(i + 1)
        if cont.size == 0:
            continue
        gcont = orc.g_contlist(i + 1)
        xs = [x[j - 1] for j in cont] + [gx[g - 1] for g in gcont]
        hs = [h[j - 1] for j in cont] + [h[gpar[g - 1] - 1] for g in gcont]
        ms = [mass[j - 1] for j in cont] + [mass[gpar[g - 1] - 1] for g in gcont]
        ks = [kc[mat[j - 1] - 1] for j in cont] + [kc[mat[gpar[g - 1] - 1] - 1] for g in gcont]
        for xj, hj, mj, kj in zip(xs, hs, ms, ks):
            havg = 0.5 * (h[i] + hj)
            ratio = hj / havg
            inv_w = 1.0 / ((0.75 * ratio - 1.5) * ratio * ratio + 1.0) if ratio < 1 else 1.0 / (2.0 - ratio) ** 3
            d = x[i] - xj
            r = np.sqrt(d @ d)
            z = r / havg
            c1 = 1.0 / (np.pi * havg ** 3)
            if z < 1:
                dw = c1 * (2.25 * z - 3.0) * z
                fij = inv_w * ((0.75 * z - 1.5) * z * z + 1.0)
            elif z < 2:
                dw = -0.75 * c1 * (2.0 - z) ** 2
                fij = 0.25 * inv_w * (2.0 - z) ** 3
            else:
                dw, fij = 0.0, 0.0
            grad = dw * d / (r * havg) if r > 0 else np.zeros(3)
            rep[i] -= mj * (kc[mat[i] - 1] + kj) * fij ** nc[mat[i] - 1] * grad
    return rep


@pytest.mark.parametrize("disctype", [0, 1])
def test_repulsive_contact_restated(disctype, oracle_lib):
    # a two-material bar with contacttype 1: contact lists hold exactly the
    # other material's particles within reach, the repulsion follows the
    # formulas of mcm_rep_contact.f90, the acceleration starts from it and the
    # per-material contact forces sum mass x repulsion (disctype 0 only)
    from mcmtop_b200.deck import two_material_bar

    deck = two_material_bar(contacttype=1, disctype=disctype)
    orc = Oracle(deck)
    for _ in range(15):
        orc.step()
    orc.step_a()
    orc.dt_update()
    orc.step_b()
    x, h, mat = orc.get("x"), orc.get("h"), orc.get_int("mat")
    ncont = orc.get_int("ncont")
    assert ncont.sum() > 0
    for i in range(0, deck.np, 37):
        d2 = ((x - x[i]) ** 2).sum(axis=1)
        near = np.flatnonzero((d2 < (h + h[i]) ** 2) & (mat != mat[i])) + 1
        assert np.array_equal(np.sort(orc.contlist(i + 1)), near)
        assert not np.isin(orc.nbrlist(i + 1), near).any()
    rep = orc.get("repulsion")
    ref = _rep_restated(orc, deck)
    assert np.max(np.abs(rep - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.max(np.abs(ref)) > 0
    cf = orc.contact_forces()
    if disctype == 0:
        mass = orc.get("mass")
        for m in (1, 2):
            want = (mass[mat == m, None] * rep[mat == m]).sum(axis=0)
            assert np.allclose(cf[m - 1], want, rtol=1e-12, atol=0)
        assert cf[0, 2] < 0 < cf[1, 2]          # the halves push each other apart
    else:
        assert not cf.any()                      # mcm_corr_acceleration does not sum them
