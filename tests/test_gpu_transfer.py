"""mcm_gpu_upload / mcm_gpu_download: the host arrays in the reference's
layout ((3,np) vectors, (3,3,np) tensors, reference particle order) come back
unchanged, also after the storage has been re-sorted on the device."""
import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import taylor_bar
from mcmtop_b200.solver import Solver

pytestmark = pytest.mark.gpu

SCALARS = ["mass", "h", "hold", "rho", "rhoold", "e", "p", "c", "vabs", "efps", "pcut", "p_cut", "fail",
           "mindist", "critts", "tracerod", "etry", "einc", "capa", "h0"]


def _state(n, rng):
    st = {k: rng.uniform(0.5, 2.0, n) for k in SCALARS}
    for k in ("x", "v", "a"):
        st[k] = rng.standard_normal((n, 3))
    sig = rng.standard_normal((n, 3, 3))
    st["sigma"] = sig                      # upper and lower triangle differ (as for the cap model)
    for k in ("s", "alfa", "rod"):
        t = rng.standard_normal((n, 3, 3))
        st[k] = 0.5 * (t + t.transpose(0, 2, 1))
    q = rng.uniform(0.0, 1.0, n)
    st["q"] = q[:, None, None] * np.eye(3)[None]
    st["mat"] = np.ones(n, np.int32)
    st["dispbc"] = rng.integers(0, 8, n).astype(np.int32)
    return st


@pytest.mark.parametrize("prec", [_abi.PREC_FP64_EXACT, _abi.PREC_MIXED])
def test_upload_download_round_trip(prec, gpu_lib):
    deck = taylor_bar(dx=0.8e-3)
    sol = Solver(deck, prec)
    try:
        rng = np.random.default_rng(3)
        st = _state(sol.n, rng)
        st["x"] = deck.x.copy()            # a body the step can run on
        sol.upload(st)
        got = sol.download(list(st))
        for k, a in st.items():
            assert np.array_equal(got[k], a), k
        # another state given as the ABI's own buffers ((3,np), (3,3,np) column-major)
        st2 = _state(sol.n, rng)
        st2["x"] = deck.x.copy()
        raw = {k: np.ascontiguousarray(a.transpose(0, 2, 1) if a.ndim == 3 else a) for k, a in st2.items()}
        sol.upload(raw, fortran_layout=True)
        got = sol.download(list(st2))
        for k, a in st2.items():
            assert np.array_equal(got[k], a), k
    finally:
        sol.close()


def test_download_after_resorting(gpu_lib):
    # with a re-sort of the storage every step, arrays still come back in the reference order
    deck = taylor_bar(dx=0.8e-3)
    a = Solver(deck, _abi.PREC_MIXED, reorder_interval=1)
    b = Solver(deck, _abi.PREC_MIXED)
    try:
        ref = b.download(["mass", "x"])
        a.run(3)
        after = a.download(["mass", "x", "spin", "qold"])
        assert np.array_equal(after["mass"], ref["mass"])
        assert np.abs(after["x"] - ref["x"]).max() < 0.05
        spin = after["spin"]
        assert np.array_equal(spin, -spin.transpose(0, 2, 1))
        qo = after["qold"]
        assert np.array_equal(qo, qo[:, 0, 0][:, None, None] * np.eye(3)[None])
    finally:
        a.close()
        b.close()


def test_downloaded_neighbour_counts_follow_the_reference_order(gpu_lib):
    # the counts live per cell-order position on the device
    deck = taylor_bar(dx=0.8e-3)
    sol = Solver(deck, _abi.PREC_FP64_EXACT, reorder_interval=2)
    try:
        sol.run(5)
        nn, _, gn, _ = sol.neighbours()
        got = sol.download(["nnbr", "g_nnbr"])
        assert np.array_equal(got["nnbr"], nn) and np.array_equal(got["g_nnbr"], gn)
        assert gn.any()
    finally:
        sol.close()



def test_download_into_caller_buffers(gpu_lib):
    deck = taylor_bar(dx=0.8e-3)
    sol = Solver(deck, _abi.PREC_MIXED)
    try:
        sol.run(3)
        ref = sol.download(["x", "sigma", "rho", "mat"])
        buf = {"x": np.empty((sol.n, 3)), "sigma": np.empty((sol.n, 9)), "rho": np.empty(sol.n),
               "mat": np.empty(sol.n, np.int32)}
        sol.download_into(buf)
        assert np.array_equal(buf["x"], ref["x"]) and np.array_equal(buf["rho"], ref["rho"])
        assert np.array_equal(buf["sigma"].reshape(-1, 3, 3).transpose(0, 2, 1), ref["sigma"])
        assert np.array_equal(buf["mat"], ref["mat"])
        with pytest.raises(ValueError):
            sol.download_into({"x": np.empty((sol.n, 2))})
    finally:
        sol.close()
