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
