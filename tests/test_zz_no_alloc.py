"""sph_SH_to_spat_noalloc: the synthesis entry point that performs no device
allocation, for callers that cannot have cudaMalloc called while they run
(their own allocator holds the device memory, or an implicit synchronisation
would break their latency budget).  It must give the same grids as
sph_SH_to_spat, call after call, while reusing the library's fixed scratch
array.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _noalloc(s, spec, out):
    from sph_swe_b200 import capi

    batch = spec.numel() // s.nlm
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return capi.lib().sph_SH_to_spat_noalloc(s.h, ctypes.c_void_p(spec.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                             batch, stream)


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_first_calls_reserve_no_device_memory(gpu, precision):
    """On a fresh handle the no-allocation entry point runs before any
    allocating call, and the device's free memory is the same before and
    after two calls: neither the handle's workspace nor the library's scratch
    array is reserved by the entry point (the scratch is reserved when the
    handle is created)."""
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph
    from tests.helpers import random_spec, rel_l2

    L, batch = 127, 3
    s = Sph(L, precision=precision)
    specs = [torch.from_numpy(random_spec(L, batch, seed=700 + k)).cuda() for k in range(2)]
    outs = [torch.full((batch, s.nphi, s.nlat), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for spec, out in zip(specs, outs):
        assert _noalloc(s, spec, out) == capi.SPH_OK, capi.last_error()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, f"the no-allocation calls changed free device memory by {free0 - free1} bytes"
    tol = 1e-12 if precision == 0 else 1e-6
    for spec, out in zip(specs, outs):
        ref = s.SH_to_spat(spec).cpu().numpy()
        assert rel_l2(out.cpu().numpy(), ref) < tol


@pytest.mark.parametrize("L,batch", [(63, 7), (255, 5)])
def test_noalloc_synthesis_matches_allocating_entry_point(gpu, L, batch):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph
    from tests.helpers import random_spec, rel_l2

    s = Sph(L)
    for call in range(2):
        spec = torch.from_numpy(random_spec(L, batch, seed=100 + 10 * L + call)).cuda()
        ref = s.SH_to_spat(spec).cpu().numpy()
        out = torch.full((batch, s.nphi, s.nlat), float("nan"), dtype=torch.float64, device="cuda")
        rc = _noalloc(s, spec, out)
        assert rc == capi.SPH_OK, capi.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert rel_l2(got, ref) < 1e-12, call


def test_noalloc_rejects_batches_beyond_the_fixed_scratch(gpu):
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph

    s = Sph(255)
    spec = torch.zeros(6, s.nlm, dtype=torch.complex128, device="cuda")
    out = torch.empty(6, s.nphi, s.nlat, dtype=torch.float64, device="cuda")
    assert _noalloc(s, spec, out) == capi.SPH_ERR_ARG
    assert "at most 5 fields" in capi.last_error()


def test_noalloc_refuses_an_unreserved_tuned_workspace(gpu):
    """A mixed handle tuned to the loader-only tensor-core variant needs a
    prepared-operand buffer that only an allocating call grows: until one has
    run with that batch the no-allocation entry point refuses, afterwards it
    runs and matches."""
    from sph_swe_b200 import capi
    from sph_swe_b200.sph import Sph
    from tests.helpers import random_spec, rel_l2

    L, batch = 63, 5
    s = Sph(L, precision=capi.SPH_PREC_MIXED)
    s.tune_load({"lmax": L, "nphi": s.nphi, "kernels": [{"kind": 0, "batch": batch, "variant": 9}]})
    spec = torch.from_numpy(random_spec(L, batch, seed=321)).cuda()
    out = torch.empty(batch, s.nphi, s.nlat, dtype=torch.float64, device="cuda")
    assert _noalloc(s, spec, out) == capi.SPH_ERR_ARG
    assert "workspace" in capi.last_error()
    ref = s.SH_to_spat(spec).cpu().numpy()  # allocating call: grows the buffer
    for _ in range(2):
        out.fill_(float("nan"))
        assert _noalloc(s, spec, out) == capi.SPH_OK, capi.last_error()
        torch.cuda.synchronize()
        assert rel_l2(out.cpu().numpy(), ref) < 1e-12
