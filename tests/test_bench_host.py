"""bench.py's host-side pieces that need no GPU: the CPU baseline of the
served and batched mixes (the oracle, one solve at a time)."""
import math

import bench

CFG = dict(thetas=[0.30], sigma=-0.7131541429)


def test_serve_cpu_baseline_charges_each_request(monkeypatch):
    # a fixed block time per grid size isolates the charging rule:
    # t_block(N) x NEV x (1 + NS) blocks per iteration x the request's iterations
    class FakeStep:
        def __init__(self, w):
            assert w["nev"] == 1 and w["ns"] == 5 and w["order"] == 5
            self.n = w["n"]

        def seconds(self):
            return {2: 0.5, 3: 2.0}[self.n]

    monkeypatch.setattr(bench, "OracleBlockStep", FakeStep)
    reqs = [dict(n=2, nev=1), dict(n=2, nev=2), dict(n=3, nev=4)]
    iters = {0: 3, 1: 4, 2: 0}  # an iteration count of 0 is charged as one iteration
    out = bench.serve_cpu_baseline(CFG, reqs, iters)
    cpu_s = 0.5 * 1 * 6 * 3 + 0.5 * 2 * 6 * 4 + 2.0 * 4 * 6 * 1
    assert math.isclose(out["value"], 3 / cpu_s, rel_tol=1e-12)
    assert out["unit"] == "solves/s" and out["kind"] == "port" and out["cores"] >= 1
    assert "N=2 0.500 s" in out["sample"] and "N=3 2.000 s" in out["sample"]


def test_serve_cpu_baseline_runs_the_oracle():
    out = bench.serve_cpu_baseline(CFG, [dict(n=2, nev=1), dict(n=2, nev=2)], {0: 2, 1: 2})
    assert out["value"] > 0 and math.isfinite(out["value"])
    assert "N=2" in out["sample"] and "2 requests" in out["sample"]


def test_serve_roofline_is_the_streams_matvec_rate():
    reqs = [dict(n=3, nev=1), dict(n=4, nev=2)]
    out = bench.serve_roofline(reqs, {0: 100, 1: 40}, 2.0, 50.0)
    flops = 100 * bench.alg_flops(7) + 40 * bench.alg_flops(9)
    assert math.isclose(out["achieved"], flops / 2.0 / 1e12, rel_tol=1e-12)
    assert math.isclose(out["frac"], out["achieved"] / 50.0, rel_tol=1e-12)
    assert out["matvecs"] == 140 and out["unit"] == "TFLOP/s" and out["traffic"] is None
