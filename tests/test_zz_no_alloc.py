"""GPU test of mcm_gpu_calctotale_noalloc, the entry point for callers that
cannot allocate device memory (their device memory belongs to their own pool,
or they must keep cudaMalloc out of the time step).  It must give the same
per-material energies as the energy sums of mcm_gpu_step_b, on two calls in a
row (the calls share one scratch array).  This file sorts last so that a run
stopping at the first failure has run every other test first."""
import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import taylor_bar
from mcmtop_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _noalloc_energies(lib, state, nmat):
    import torch

    dev = torch.device("cuda", 0)
    mass = torch.tensor(state["mass"], dtype=torch.float64, device=dev)
    vabs = torch.tensor(state["vabs"], dtype=torch.float64, device=dev)
    v = torch.tensor(np.ascontiguousarray(state["v"]).ravel(), dtype=torch.float64, device=dev)
    e = torch.tensor(state["e"], dtype=torch.float64, device=dev)
    mat = torch.tensor(state["mat"], dtype=torch.int32, device=dev)
    out = torch.full((5 * nmat + 3,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    st = lib.mcm_gpu_calctotale_noalloc(mass.data_ptr(), vabs.data_ptr(), v.data_ptr(), e.data_ptr(),
                                        mat.data_ptr(), len(state["mass"]), nmat, out.data_ptr(), None)
    assert st == _abi.MCM_OK, lib.mcm_gpu_strerror(st)
    return out.cpu().numpy()


def test_noalloc_energies_match_step_b(gpu_lib):
    lib = gpu_lib
    deck = taylor_bar(dx=0.8e-3)
    sol = Solver(deck, _abi.PREC_FP64_EXACT, device=0)
    fields = ["mass", "vabs", "v", "e", "mat"]
    for call in range(2):
        for _ in range(3):
            sol.step()
        sol.step_a()
        sol.dt_update()
        ref = sol.step_b().copy()                      # energies summed inside mcm_gpu_step_b
        state = sol.download(fields)                   # the arrays that sum read (before step_c)
        got = _noalloc_energies(lib, state, sol.nmat)
        scale = np.abs(ref).max()
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - ref)) <= 1e-13 * scale, (call, got, ref)
        sol.step_c()
    sol.close()


def test_noalloc_several_materials(gpu_lib):
    # two materials: every slot of the 5*nmat+3 output against step_b's sums,
    # then with some material ids outside 1..nmat, which the call skips
    from mcmtop_b200.deck import two_material_bar

    lib = gpu_lib
    deck = two_material_bar()
    sol = Solver(deck, _abi.PREC_FP64, device=0)
    for _ in range(4):
        sol.step()
    sol.step_a()
    sol.dt_update()
    ref = sol.step_b().copy()
    state = sol.download(["mass", "vabs", "v", "e", "mat"])
    sol.close()
    got = _noalloc_energies(lib, state, 2)
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.abs(ref).max(), (got, ref)
    bad = dict(state)
    mat = state["mat"].copy()
    rng = np.random.default_rng(5)
    odd = rng.choice(len(mat), size=len(mat) // 10, replace=False)
    mat[odd[: len(odd) // 2]] = 0
    mat[odd[len(odd) // 2:]] = 3
    bad["mat"] = mat
    got = _noalloc_energies(lib, bad, 2)
    want = []
    for m in (1, 2):
        sel = mat == m
        ms, va, v = state["mass"][sel], state["vabs"][sel], state["v"][sel]
        want += [(0.5 * ms * va * va).sum(), state["e"][sel].sum(), *(ms[:, None] * np.abs(v)).sum(axis=0)]
    want += [want[0] + want[5], want[1] + want[6], want[0] + want[5] + want[1] + want[6]]
    assert np.allclose(got, want, rtol=1e-12, atol=0.0), (got, want)


def test_noalloc_rejects_too_many_materials(gpu_lib):
    st = gpu_lib.mcm_gpu_calctotale_noalloc(1, 1, 1, 1, 1, 10, _abi.MAX_MATERIALS + 1, 1, None)
    assert st == _abi.MCM_EINVAL
