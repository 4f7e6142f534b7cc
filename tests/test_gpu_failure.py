"""Failure detection on the GPU without a fault: every wait inside the substage kernel (on a
TMA chunk's mbarrier, and on its own copies before the CTA exits) gives up after 2 s, sets an
error bit in the status word and returns.  The test makes the waits run out on purpose (each
chunk expects more bytes than its copies deliver; the copies themselves are ordinary and in
bounds), checks that the host reports FG2_ERR_TIMEOUT, and that the context stays usable: the
next step, with normal waits, gives bitwise the state of a fresh simulation."""
import time

import numpy as np
import pytest

import fg2_b200

pytestmark = pytest.mark.gpu


def make(n1, n2):
    s = fg2_b200.Sim(n1, n2, scheme="hydro")
    s.config()
    s.init("noise", seed=3)
    return s


def test_timed_out_waits_are_reported_and_recoverable(cuda):
    dt = 1e-4
    with make(64, 96) as s, make(64, 96) as ref:
        x0 = s.download()
        s.test_stall_waits(16)
        t0 = time.monotonic()
        s.stage(0, dt)
        with pytest.raises(fg2_b200.FG2Error, match="wait gave up"):
            s.sync()
        took = time.monotonic() - t0
        # one wait on a chunk plus one per ring slot while draining, 2 s each
        assert 1.5 < took < 30.0, took

        s.test_stall_waits(0)
        s.clear_status()
        assert s.sync() == 0
        s.upload(x0)
        assert s.step(0.0, dt) == 0
        assert ref.step(0.0, dt) == 0
        assert np.array_equal(s.download(), ref.download())
