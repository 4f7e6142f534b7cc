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

MAX_ROWS = 16384  # FG2_NOALLOC_MAX_ROWS in include/fg2_b200.h


def nan_output(cuda):
    """The caller's 4-double output buffer, NaN-filled so a result that never arrived cannot
    pass, and the fill finished before the library's stream writes it."""
    import torch
    out = torch.full((4,), float("nan"), dtype=torch.float64, device=cuda)
    torch.cuda.synchronize()
    return out


def call(lib, sim, n1, n2, out, storage):
    pitch, _ = sim.layout()
    return lib.fg2_sums_noalloc(lib.fg2_sim_u(sim.h), n1, n2, pitch, fg2_b200.STORAGE[storage], out.data_ptr(),
                                sim.stream)


@pytest.mark.parametrize("scheme,storage,n1,n2,setup", [("hydro", "f32", 300, 260, "kh"), ("hydro", "f64", 123, 77, "kh"),
                                                        ("hydro-isot", "f32", 200, 333, "turb"),
                                                        ("disk", "f32", 96, 64, "smooth")])
def test_sums_noalloc_matches_allocating_sums(scheme, storage, n1, n2, setup, cuda):
    import torch
    lib = fg2_b200.load_library(scheme)
    with fg2_b200.Sim(n1, n2, scheme=scheme, storage=storage) as a, \
            fg2_b200.Sim(n1, n2, scheme=scheme, storage=storage) as b:
        for s, seed in ((a, 11), (b, 12)):
            s.config()
            s.init(setup, seed=seed)
        pitch, cell = a.layout()
        assert cell == a.nvar
        for sim in (a, b, a):  # calls in a row, on different states, reusing the static scratch
            expect = sim.sums()
            out = nan_output(cuda)
            rc = call(lib, sim, n1, n2, out, storage)
            assert rc == 0, lib.fg2_last_error()
            torch.cuda.synchronize()
            np.testing.assert_allclose(out.cpu().numpy(), expect, rtol=1e-12, atol=1e-9)


def test_sums_noalloc_allocates_nothing(cuda):
    """Once the first call has set the array up, further calls leave the device's free
    memory unchanged."""
    import torch
    lib = fg2_b200.load_library("hydro")
    with fg2_b200.Sim(256, 256) as s:
        s.config()
        s.init("kh", seed=3)
        out = nan_output(cuda)
        assert call(lib, s, 256, 256, out, "f32") == 0, lib.fg2_last_error()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        for _ in range(5):
            assert call(lib, s, 256, 256, out, "f32") == 0, lib.fg2_last_error()
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0
        np.testing.assert_allclose(out.cpu().numpy(), s.sums(), rtol=1e-12, atol=1e-9)


def test_sums_noalloc_takes_the_largest_grid_and_rejects_one_row_more(cuda):
    import torch
    lib = fg2_b200.load_library("hydro")
    with fg2_b200.Sim(MAX_ROWS + 1, 8) as s:
        s.config()
        s.init("kh", seed=5)
        x = s.download()
        out = nan_output(cuda)
        # rejected on the host before anything is launched
        assert call(lib, s, MAX_ROWS + 1, 8, out, "f32") == -1
        assert b"exceeds the scratch limit" in lib.fg2_last_error()
        # the first MAX_ROWS rows of the same array are accepted
        assert call(lib, s, MAX_ROWS, 8, out, "f32") == 0, lib.fg2_last_error()
        torch.cuda.synchronize()
    q = x[:MAX_ROWS].astype(np.float64)
    rho = np.exp(q[..., 0])
    expect = [rho.sum(), (rho * q[..., 1]).sum(), (rho * q[..., 2]).sum(),
              (rho * (np.exp(q[..., 3]) + 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2))).sum()]
    np.testing.assert_allclose(out.cpu().numpy(), expect, rtol=1e-10)
