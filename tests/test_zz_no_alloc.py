"""The allocation-free energy entry point (oct_elastic_energy_noalloc) against the existing
energy entry point (oct_scene_energy, elastic part).

It exists for callers that cannot allocate device memory when they need the number (a host
application whose device memory belongs to its own pool and forbids driver allocations in
its frame loop, or a real-time loop that cannot take cudaMalloc's latency and implicit
synchronisation): they pass device inputs and a device output, and the function's only
intermediate storage is a static per-device array.  The test calls it twice in a row
through the C ABI on the same state: both results match the existing entry point within the
energy tolerance of the other tests (1e-3 relative) and are bit-identical to each other
(fixed summation order), for the four materials with an energy (Hooke, StVK, NeoHooke, Stable
NeoHooke) on all five element types.  The file sorts last so a stop-at-first-failure run has already run
everything else; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu


CASES = [(O.TETRA, (8, 2, 2), 1e5), (O.HEXA, (4, 2, 2), 2e5), (O.TETRA10, (4, 2, 2), 2e5),
         (O.TETRA20, (2, 1, 1), 2e5), (O.HEXA27, (2, 1, 1), 2e5)]


@pytest.mark.parametrize("material", [O.HOOKE, O.STVK, O.NEOHOOKE, O.STABLE_NEOHOOKE])
@pytest.mark.parametrize("element,cells,young", CASES)
def test_noalloc_energy_matches_scene_energy_twice(ctx, element, cells, young, material):
    import torch
    import octopusengine_b200 as ob
    from octopusengine_b200 import capi
    X, T = O.beam_mesh(element, cells, (1.0, 0.25, 0.25))
    fixed = O.fixed_by_plane(X, (0.01, 0, 0), (-1, 0, 0))
    s = ob.Scene(ctx, element, X, T, density=1000.0, young=young, poisson=0.45, fixed_ids=fixed, iterations=10,
                 gravity=(0.0, 0.0, -9.81), material=material)
    for _ in range(10):
        s.step(0.01, 1)
    expected = s.energy()[1]
    assert abs(expected) > 0
    p = torch.tensor(s.get_position(), device="cuda")
    Xd = torch.tensor(X, device="cuda")
    Td = torch.tensor(T, device="cuda", dtype=torch.int32)
    out = torch.zeros(2, device="cuda", dtype=torch.float64)
    torch.cuda.synchronize()
    got = []
    for call in range(2):
        st = capi.lib().oct_elastic_energy_noalloc(element, material, C.c_void_p(p.data_ptr()),
                                                   C.c_void_p(Xd.data_ptr()), C.c_void_p(Td.data_ptr()), len(T),
                                                   young, 0.45, C.c_void_p(out[call:].data_ptr()), None)
        assert st == capi.OK
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for g in got:
        assert abs(g - expected) / abs(expected) < 1e-3, (g, expected)
    assert got[0] == got[1]
    s.close()


def test_noalloc_energy_rejects_oversized_meshes(ctx):
    import torch
    from octopusengine_b200 import capi
    dummy = torch.zeros(4, device="cuda")
    out = torch.zeros(1, device="cuda", dtype=torch.float64)
    st = capi.lib().oct_elastic_energy_noalloc(O.TETRA, 3, C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()),
                                               C.c_void_p(dummy.data_ptr()), (1 << 20) + 1, 1e5, 0.3,
                                               C.c_void_p(out.data_ptr()), None)
    assert st == capi.EINVAL
