"""The CPU-baseline legs of bench.py, on small inputs: the differenced
timing cancels each call's set-up and counts the units a run reports, and
the CG and explicit legs report the contract's keys with a positive rate."""
import os
import sys

import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_timed_difference_cancels_setup_and_counts_reported_units():
    import bench
    calls = []

    def run(k):
        # 5 s of set-up per call; a run stops early after 7 units (like a
        # converged CG) and reports how many it did
        done = min(k, 7)
        calls.append(k)
        return 5.0 + 0.25 * done, done

    per, units, total = bench._timed_difference(run, seconds=100.0, cap=100)   # m = 38: stops at 7
    assert calls[0] == 1 and calls[1] == 1                 # untimed warm-up, then the short run
    assert units == 6 and per == 0.25 and total == 5.0 + 0.25 * 7


def test_cpu_legs_report_the_contract_keys():
    import bench
    from oracle import fea_oracle as O
    X, el = O.hex_block(3, jitter=0.1, seed=2)
    m = O.Model(X, [O.Group("C3D8", el, 1.0, 50.0)], [], [])
    gc = 1e-3 * torch.randn(int(m.free_mask().sum()), generator=torch.Generator().manual_seed(0),
                            dtype=torch.float64)
    R, (ip, ix, v) = m.assemble(gc)
    cg = bench.cpu_cg_iteration(ip, ix.to(torch.int32), v, -R, 0.2)
    Xt, et = O.tet_block(2)
    ex = bench.cpu_explicit_step(Xt.numpy(), et.numpy(), 1e-3, 0.2)
    for line, unit in ((cg, "ms per CG iteration"), (ex, "steps/s")):
        assert set(line) == {"value", "unit", "cores", "kind", "sample"}
        assert line["unit"] == unit and line["kind"] == "port" and line["value"] > 0 and line["cores"] >= 1
