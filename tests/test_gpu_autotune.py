"""TUNING_AUTOTUNE and the cache modes of the C ABI (the reference maps
them in src/common/c_api.cpp:76-107 to its autotune sweep and disk cache,
src/unified/unified_solver.cpp:403-597, 649-925): the tuned handle solves
correctly, CACHE_AUTO writes the choice to the on-disk table and a later
create takes it, NODISK and NOCACHE never touch the disk."""
import os

import pytest

from sunny_gen_eigensolver_b200 import accuracy, generators

pytestmark = pytest.mark.gpu


def _table(d):
    p = os.path.join(d, "tune_v1.tsv")
    if not os.path.exists(p):
        return {}
    out = {}
    for line in open(p):
        k, v = line.rstrip("\n").split("\t")
        out[k] = v
    return out


@pytest.mark.parametrize("n", [54, 72])
def test_autotune_cache_modes(cuda, tmp_path, monkeypatch, n):
    import torch
    from sunny_gen_eigensolver_b200 import Solver, solve
    monkeypatch.setenv("SUNNY_GENEIG_CACHE_DIR", str(tmp_path))
    H, S = generators.baseline_problems(n, 8, seed=90 + n)
    Ht, St = torch.from_numpy(H).cuda(), torch.from_numpy(S).cuda()
    with Solver(n) as s0:
        W0, _, i0 = solve(Ht, St, solver=s0)
    with Solver(n, tuning="autotune", cache="auto") as s1:
        regime = s1.regime
        assert regime in ("smem-cta", "smem-wide", "l2-slot")
        W, U, info = solve(Ht, St, solver=s1)
    assert torch.equal(info, i0)
    Wn, Un = W.cpu().numpy(), U.cpu().numpy()
    assert accuracy.eig_err_rel(H, Wn, W0.cpu().numpy()).max() <= 1e-12
    assert accuracy.residual(H, S, Wn, Un).max() <= 1e-12
    t = _table(tmp_path)
    assert len(t) == 1
    (key, cfg), = t.items()
    assert f"n={n};" in key and cfg.split(":")[0] == regime
    # a later create takes the cached choice; a malformed line is ignored
    with open(os.path.join(tmp_path, "tune_v1.tsv"), "a") as f:
        f.write("garbage line without a tab\n")
    with Solver(n, tuning="autotune", cache="auto") as s2:
        assert s2.regime == regime
    # NODISK (choice kept in this process) and NOCACHE (tuned again) write nothing
    fresh = tmp_path / "fresh"
    fresh.mkdir()
    monkeypatch.setenv("SUNNY_GENEIG_CACHE_DIR", str(fresh))
    for cache in ("nodisk", "nocache"):
        with Solver(n, tuning="autotune", cache=cache) as s:
            W, U, info = solve(Ht, St, solver=s)
        assert _table(fresh) == {}
        assert torch.equal(info, i0)
        assert accuracy.residual(H, S, W.cpu().numpy(), U.cpu().numpy()).max() <= 1e-12
