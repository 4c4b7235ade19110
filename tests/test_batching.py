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


@pytest.mark.gpu
def test_graph_replay_matches_per_size_launches(cuda, tmp_path):
    import torch
    from sunny_gen_eigensolver_b200 import generators
    from sunny_gen_eigensolver_b200.batching import UnevenBatch
    rng = np.random.default_rng(3)
    sizes = rng.choice([12, 24, 54, 72, 108], size=300, p=[0.3, 0.2, 0.25, 0.15, 0.1])
    ub = UnevenBatch(sizes)
    for n, c in ub.counts.items():
        H, S = generators.baseline_problems(n, c, seed=n)
        ub.set_inputs(n, torch.from_numpy(H).cuda().transpose(-1, -2), torch.from_numpy(S).cuda().transpose(-1, -2))
    ub.run_sequential()
    torch.cuda.synchronize()
    ref = {n: (ub.W[n].clone(), ub.U[n].clone(), ub.info[n].clone()) for n in ub.counts}
    for n in ub.counts:
        ub.W[n].zero_(); ub.U[n].zero_(); ub.info[n].fill_(-1)
    table = TuneTable(tmp_path / "plans.json")
    plan = ub.autotune(table)
    assert sorted(x for lane in plan.streams for x in lane) == sorted(ub.counts)
    for n in ub.counts:
        ub.W[n].zero_(); ub.U[n].zero_(); ub.info[n].fill_(-1)
    ub.replay()
    ub.replay()
    torch.cuda.synchronize()
    for n in ub.counts:
        assert torch.equal(ub.W[n], ref[n][0]) and torch.equal(ub.U[n], ref[n][1]) and torch.equal(ub.info[n], ref[n][2])
        assert bool((ub.info[n] == 0).all())
    # the chosen plan was persisted and is reused
    assert TuneTable(tmp_path / "plans.json").get(mix_key(ub.counts, torch.cuda.get_device_name())) is not None
