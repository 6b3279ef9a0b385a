"""bench.py's reference arm on the CPU: the oracle timed on bounded samples of
the dome workload (c0), extrapolated with the oracle's recorded iteration
counts.  The line must carry the repo arm's config dict (the same keys and
values), the reference fields of the bench contract, and a sample time
inside its own steps."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


class _OneRank:
    world, rank = 1, 0

    def barrier(self):
        pass

    def max(self, x):
        return x


def test_reference_arm_line_on_the_dome():
    args = bench.parse_args(["--impl", "reference", "--workload", "c0", "--steps", "2", "--warmup", "1"])
    out = bench.run_reference(args, _OneRank())
    assert out["impl"] == "reference" and out["value"] > 0
    models = bench.make_models(args)
    cols, nodes = bench.workload_stats(models)
    assert out["config"] == bench.config_dict(args, models, cols, nodes, 1)
    assert out["cpu_baseline"]["cores"] == 1 and out["cpu_baseline"]["kind"] == "port"
    assert out["cpu_baseline"]["value"] == out["value"]
    assert out["e2e"] == {"value": out["value"], "unit": out["unit"], "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}
    assert "oracle" in out["cpu_baseline"]["sample"]
    # the extrapolation uses the oracle's own recorded counts of this workload
    rec = bench.load_counts("c0/l2rel")
    assert rec and "oracle" in rec["source"]
    assert out["ms_per_step"] < 60_000
