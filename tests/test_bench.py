"""CPU checks of bench.py's contract: the reference arm's JSON line (the FP64
C restatement timed on the host cores) and the helpers the GPU arm uses."""
from __future__ import annotations

import importlib
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    return importlib.import_module("bench")


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == "biot_savart_gint_per_s"
    assert d["unit"] == "Gint/s" and d["higher_is_better"] is True and d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["targets"] == 88803 and d["config"]["filaments"] == 175080


def test_traffic_from_committed_profile():
    """Both stream layouts have a committed capture to scale from."""
    b = _bench()
    n = 15547629240
    for chained in (False, True):
        t = b.profiled_traffic(n, chained)
        assert t is not None and 1e7 < t < 1e10, chained
        assert abs(b.profiled_traffic(2 * n, chained) - 2 * t) < 1e-6 * t


def test_workload_sizes_match_the_metric_case():
    b = _bench()
    _, fams, P, nf, nt = b.workload(1, "large")
    assert (nf, nt) == (175080, 88803)
    assert P.shape == (nt, 3, 1, 1) and len(fams) == 2
