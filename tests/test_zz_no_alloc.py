"""The allocation-free sums entry point (fg2_sums_noalloc), called through the C ABI.

It exists for callers that cannot call cudaMalloc -- an application whose own allocator
already holds the GPU's memory, a loop that must not allocate, or code holding a state
array without a simulation handle -- so it reduces through a static device array instead
of handle-owned partials.  Two calls in a row must agree with fg2_sim_sums (the allocating
path) within the tolerance of the sums test; the first call also sets the array up.  This
file is collected last so that a failure here stops a `-x` run only after every other test.
"""
import numpy as np
import pytest

import fg2_b200

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme,storage,n1,n2", [("hydro", "f32", 300, 260), ("hydro", "f64", 123, 77),
                                                  ("hydro-isot", "f32", 200, 333)])
def test_sums_noalloc_matches_allocating_sums(scheme, storage, n1, n2, cuda):
    import torch
    lib = fg2_b200.load_library(scheme)
    out = torch.zeros(4, dtype=torch.float64, device=cuda)  # the caller's output buffer
    with fg2_b200.Sim(n1, n2, scheme=scheme, storage=storage) as a, \
            fg2_b200.Sim(n1, n2, scheme=scheme, storage=storage) as b:
        for s, seed in ((a, 11), (b, 12)):
            s.config()
            s.init("turb" if scheme == "hydro-isot" else "kh", seed=seed)
        pitch, cell = a.layout()
        assert cell == a.nvar
        for sim in (a, b, a):  # calls in a row, on different states, reusing the static scratch
            expect = sim.sums()
            rc = lib.fg2_sums_noalloc(lib.fg2_sim_u(sim.h), n1, n2, pitch, fg2_b200.STORAGE[storage],
                                      out.data_ptr(), sim.stream)
            assert rc == 0, lib.fg2_last_error()
            torch.cuda.synchronize()
            np.testing.assert_allclose(out.cpu().numpy(), expect, rtol=1e-12, atol=1e-9)


def test_sums_noalloc_rejects_grids_beyond_the_scratch(cuda):
    import torch
    lib = fg2_b200.load_library("hydro")
    out = torch.zeros(4, dtype=torch.float64, device=cuda)
    with fg2_b200.Sim(16, 16) as s:
        pitch, _ = s.layout()
        # rejected on the host before anything is launched
        too_many = lib.fg2_sums_noalloc(lib.fg2_sim_u(s.h), 20000, 16, pitch, 0, out.data_ptr(), s.stream)
    assert too_many == -1
    assert b"exceeds the scratch limit" in lib.fg2_last_error()
