"""Uneven-size batches: plan table persistence (CPU) and, on the GPU, that one
graph replay over all size classes gives exactly the per-size launches'
results."""
import json

import numpy as np
import pytest

from sunny_gen_eigensolver_b200.batching import Plan, TuneTable, lpt_plan, mix_key


def test_lpt_plan_balances():
    p = lpt_plan({12: 1.0, 24: 2.0, 54: 5.0, 72: 4.0}, 2)
    loads = sorted(sum({12: 1.0, 24: 2.0, 54: 5.0, 72: 4.0}[n] for n in lane) for lane in p.streams)
    assert loads == [6.0, 6.0]
    assert lpt_plan({12: 1.0}, 8).streams == [[12]]


def test_table_roundtrip_atomic_and_rejects_corruption(tmp_path):
    path = tmp_path / "plans.json"
    t = TuneTable(path)
    key = mix_key({54: 1000, 12: 300}, "dev")
    t.put(key, Plan([[54], [12]]))
    assert not list(tmp_path.glob(".plans.*"))            # no temporary left behind
    t2 = TuneTable(path)
    assert t2.get(key).streams == [[54], [12]] and not t2.rejected
    path.write_text("{not json")
    t3 = TuneTable(path)
    assert t3.rejected and t3.get(key) is None
    path.write_text(json.dumps({"format": "other", "version": 1, "plans": {}}))
    assert TuneTable(path).rejected
    path.write_text(json.dumps({"format": "sunny-geneig-uneven-plans", "version": 1,
                                "plans": {key: {"streams": [["x"]]}}}))
    assert TuneTable(path).rejected
    t3.put(key, Plan([[12, 54]]))                          # a rejected table is rewritten
    assert TuneTable(path).get(key).streams == [[12, 54]]


def test_mix_key_rounds_counts():
    assert mix_key({54: 16384, 12: 60000}) == mix_key({12: 60400, 54: 16300})


def test_plan_size_configs_roundtrip_and_validation(tmp_path):
    from sunny_gen_eigensolver_b200.batching import size_configs
    path = tmp_path / "plans.json"
    key = mix_key({54: 100, 216: 10}, "dev")
    cfg = {54: {"regime": "smem-cta", "slots_per_sm": 0}, 216: {"regime": "l2-slot", "slots_per_sm": 2}}
    TuneTable(path).put(key, Plan([[216], [54]], cfg))
    got = TuneTable(path).get(key)
    assert got.configs == cfg and got.streams == [[216], [54]]
    raw = json.loads(path.read_text())
    raw["plans"][key]["configs"]["54"]["regime"] = "warp-magic"
    path.write_text(json.dumps(raw))
    assert TuneTable(path).rejected
    raw["version"] = 1                                      # tables from the previous format are ignored
    path.write_text(json.dumps(raw))
    assert TuneTable(path).rejected
    assert size_configs(54)[0]["regime"] == "smem-cta" and len(size_configs(54)) == 3
    assert all(c["regime"] == "l2-slot" for c in size_configs(216))
    assert {"regime": "smem-wide", "slots_per_sm": 0} in size_configs(72)


@pytest.mark.gpu
def test_graph_replay_matches_per_size_launches(cuda, tmp_path):
    """autotune picks a configuration per size and a stream plan; one graph
    replay then gives exactly what one launch per size with the same
    configurations gives, twice in a row, and the results meet the zhegv
    bars."""
    import torch
    from oracle import zhegv_batch
    from sunny_gen_eigensolver_b200 import accuracy, generators
    from sunny_gen_eigensolver_b200.batching import UnevenBatch
    rng = np.random.default_rng(3)
    sizes = rng.choice([12, 24, 54, 72, 108], size=300, p=[0.3, 0.2, 0.25, 0.15, 0.1])
    ub = UnevenBatch(sizes)
    inputs = {}
    for n, c in ub.counts.items():
        H, S = generators.baseline_problems(n, c, seed=n)
        inputs[n] = (H, S)
        ub.set_inputs(n, torch.from_numpy(H).cuda().transpose(-1, -2), torch.from_numpy(S).cuda().transpose(-1, -2))
    table = TuneTable(tmp_path / "plans.json")
    plan = ub.autotune(table)
    assert sorted(x for lane in plan.streams for x in lane) == sorted(ub.counts)
    assert sorted(plan.configs) == sorted(ub.counts)
    for n, cfg in plan.configs.items():
        assert ub.solvers[n].regime == cfg["regime"]
    ub.run_sequential()
    torch.cuda.synchronize()
    ref = {n: (ub.W[n].clone(), ub.U[n].clone(), ub.info[n].clone()) for n in ub.counts}
    for n in ub.counts:
        ub.W[n].zero_(); ub.U[n].zero_(); ub.info[n].fill_(-1)
    ub.replay()
    ub.replay()
    torch.cuda.synchronize()
    for n in ub.counts:
        assert torch.equal(ub.W[n], ref[n][0]) and torch.equal(ub.U[n], ref[n][1]) and torch.equal(ub.info[n], ref[n][2])
        assert bool((ub.info[n] == 0).all())
        H, S = inputs[n]
        W = ub.W[n].cpu().numpy()
        U = ub.U[n].transpose(-1, -2).cpu().numpy()
        Wr, _, _ = zhegv_batch(H, S)
        assert accuracy.eig_err_rel(H, W, Wr).max() <= 1e-12
        assert accuracy.residual(H, S, W, U).max() <= 1e-12
    # the chosen plan and configurations were persisted and are reused
    known = TuneTable(tmp_path / "plans.json").get(mix_key(ub.counts, torch.cuda.get_device_name()))
    assert known is not None and known.configs == plan.configs


def test_plan_persistent_configs_roundtrip_and_validation(tmp_path):
    path = tmp_path / "plans.json"
    key = "persistent|" + mix_key({12: 100, 216: 10}, "dev")
    pers = {216: {"regime": "l2-slot", "per_item": 1}, 12: {"regime": "smem-cta", "per_item": 16}}
    TuneTable(path).put(key, Plan([[12, 216]], persistent=pers))
    assert TuneTable(path).get(key).persistent == pers
    raw = json.loads(path.read_text())
    raw["plans"][key]["persistent"]["12"]["per_item"] = 0
    path.write_text(json.dumps(raw))
    assert TuneTable(path).rejected


@pytest.mark.gpu
def test_persistent_launch_matches_per_size_launches(cuda, tmp_path):
    """The one-launch persistent kernel over a mix of sizes in both regimes
    (smem-cta 12, 24, 54; l2-slot 72, 108) gives bit for bit what one launch
    per size gives in the same regime, twice in a row and from a captured
    graph, with a non-positive-definite problem's info code and NaN fill;
    the results meet the zhegv bars. autotune_persistent then picks a
    configuration per size, which is persisted and reused."""
    import torch
    from oracle import zhegv_batch
    from sunny_gen_eigensolver_b200 import Solver, accuracy, generators
    from sunny_gen_eigensolver_b200.batching import UnevenBatch
    rng = np.random.default_rng(4)
    sizes = rng.choice([12, 24, 54, 72, 108], size=400, p=[0.3, 0.2, 0.25, 0.15, 0.1])
    ub = UnevenBatch(sizes)
    inputs = {}
    for n, c in ub.counts.items():
        H, S = generators.baseline_problems(n, c, seed=100 + n)
        if n == 24:
            S[3] = np.eye(n)
            S[3, 5, 5] = -1.0                       # info = n + 6
        inputs[n] = (H, S)
        ub.set_inputs(n, torch.from_numpy(H).cuda().transpose(-1, -2), torch.from_numpy(S).cuda().transpose(-1, -2))
    ref = {}
    for n in ub.counts:
        with Solver(n) as s:
            s.launch(ub.H[n], ub.S[n], ub.W[n], ub.U[n], ub.info[n])
            torch.cuda.synchronize()
        ref[n] = (ub.W[n].clone(), ub.U[n].clone(), ub.info[n].clone())
    ub.persistent()
    shape = ub.uneven.shape
    assert [x[0] for x in shape] == sorted(ub.counts, reverse=True)
    assert {x[0]: x[1] for x in shape} == {n: ("smem-cta" if n <= 60 else "l2-slot") for n in ub.counts}

    def check():
        torch.cuda.synchronize()
        for n in ub.counts:
            assert torch.equal(ub.info[n], ref[n][2])
            assert torch.equal(ub.W[n].nan_to_num(7.0), ref[n][0].nan_to_num(7.0))
            assert torch.equal(ub.U[n].nan_to_num(7.0), ref[n][1].nan_to_num(7.0))
            ub.W[n].zero_(); ub.U[n].zero_(); ub.info[n].fill_(-1)

    for _ in range(2):
        ub.launch_persistent()
        check()
    ub.capture_persistent()
    ub.replay_persistent()
    check()
    ub.launch_persistent()
    torch.cuda.synchronize()
    for n in ub.counts:
        H, S = inputs[n]
        info = ub.info[n].cpu().numpy()
        Wr, _, ir = zhegv_batch(H, S)
        assert np.array_equal(info, ir)
        ok = ir == 0
        W = ub.W[n].cpu().numpy()[ok]
        U = ub.U[n].transpose(-1, -2).cpu().numpy()[ok]
        assert accuracy.eig_err_rel(H[ok], W, Wr[ok]).max() <= 1e-12
        assert accuracy.residual(H[ok], S[ok], W, U).max() <= 1e-12
    assert ref[24][2][3].item() == 24 + 6
    table = TuneTable(tmp_path / "plans.json")
    chosen = ub.autotune_persistent(table)
    assert sorted(chosen) == sorted(ub.counts)
    key = "persistent|" + mix_key(ub.counts, torch.cuda.get_device_name())
    assert TuneTable(tmp_path / "plans.json").get(key).persistent == chosen
    ub.replay_persistent()
    torch.cuda.synchronize()
    for n in ub.counts:
        assert torch.equal(ub.info[n], ref[n][2])
