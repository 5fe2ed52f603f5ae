"""Host-side helpers of bench.py (no GPU): the per-field relative L2 and its
area-weighted variant used in the accuracy block of the bench line."""
import numpy as np
import torch

import bench


def test_per_field_rel_and_area_weighted():
    rng = np.random.default_rng(5)
    nf, nphi, nlat = 3, 8, 6
    b = rng.standard_normal((nf, nphi, nlat))
    a = b + 1e-3 * rng.standard_normal((nf, nphi, nlat))
    w = rng.uniform(0.1, 1.0, nlat)
    r = bench._per_field_rel(torch.from_numpy(a), torch.from_numpy(b))
    ref = np.linalg.norm((a - b).reshape(nf, -1), axis=1) / np.linalg.norm(b.reshape(nf, -1), axis=1)
    assert r["fields"] == nf and np.isclose(r["max"], ref.max()) and np.isclose(r["median"], np.median(ref))
    ra = bench._per_field_rel_area(torch.from_numpy(a), torch.from_numpy(b), w)
    num = np.sqrt((((a - b) ** 2) * w).reshape(nf, -1).sum(1))
    den = np.sqrt(((b ** 2) * w).reshape(nf, -1).sum(1))
    assert np.isclose(ra["max"], (num / den).max())


def test_reference_arm_line_contract():
    """`bench.py --impl reference` (the CPU restatement timed on the host
    cores, the driver's reference arm) prints one JSON line with the headline
    metric, unit and direction of our arm, the same workload configuration,
    a cpu_baseline block and an e2e block without host-device copies."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == "GFLOP/s"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["lmax"] == 255 and d["config"]["fields"] == 64 and d["config"]["vector_pairs"] == 32
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
