"""The allocation-free element-energy entry point (fea_energy_volume_noalloc).

Callers that cannot allocate device memory at the call — hosts whose device
memory is all reserved by their own pool allocator, or foreign-language hosts
that only pass pointers they already own — use this variant; its scratch is a
fixed array inside the library.  These tests call it through the C ABI and
compare it with the allocating entry point (fea_energy_volume) on two calls in
a row.  The file sorts last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process, where
its first call performs the per-device set-up.
"""
import ctypes as C

import pytest
import torch

from tests.helpers import fea_model

pytestmark = pytest.mark.gpu

def test_noalloc_energy_matches_allocating_entry_point(golden):
    """Bitwise equal to fea_energy_volume: both run the same kernels with the
    same summation order.  The larger C3D8 group runs first and the C3D4
    group after it, twice each, so that partials left in the shared array by
    a larger call would show in a smaller one."""
    from fea_b200 import _lib as L
    from fea_b200.plan import stream, vptr
    cases = []
    for name, kind in (("hex5", "C3D8"), ("cfg1", "C3D4")):
        g = golden(name)
        c, e, _ = fea_model(g, kind)
        c.initialize()
        P = c.assembly.plan
        mu, kappa = e.materials.parameters()
        gc = torch.from_numpy(g["state"]).cuda()
        ref = torch.zeros(1, dtype=torch.float64, device="cuda")
        P.energy_volume(0, mu, kappa, gc, ref)
        cases.append((P, mu, kappa, gc, float(ref)))
    for _ in range(2):
        for P, mu, kappa, gc, ref in cases:
            out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
            st = L.fea_energy_volume_noalloc(C.byref(P.nodes), C.byref(P.groups[0].desc), mu, kappa, vptr(gc),
                                             vptr(out), stream())
            assert st == L.FEA_OK
            torch.cuda.synchronize()
            assert float(out) == ref


def test_noalloc_energy_rejects_groups_beyond_its_limit(golden):
    from fea_b200 import _lib as L
    from fea_b200.plan import stream, vptr
    g = golden("hex5")
    c, e, _ = fea_model(g, "C3D8")
    c.initialize()
    P = c.assembly.plan
    big = L.Group.from_buffer_copy(P.groups[0].desc)
    big.ne = L.FEA_NOALLOC_MAX_ELEMS + 1          # checked before any launch
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    gc = torch.zeros(P.ndof, dtype=torch.float64, device="cuda")
    st = L.fea_energy_volume_noalloc(C.byref(P.nodes), C.byref(big), 1.0, 1.0, vptr(gc), vptr(out), stream())
    assert st == L.FEA_ETOOBIG
