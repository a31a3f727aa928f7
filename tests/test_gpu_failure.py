"""Failure handling on the GPU without a fault: a device wait that nothing
ends runs out, records a time-out status the host reads, and the context
keeps working. Requires a GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_the_context_stays_usable():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hbp_b200 as E
    import pyoracle as O
    from scenes import make_scene
    ctx = E.Context(0)
    try:
        assert ctx.check_bounded_wait()
        assert ctx.check_bounded_wait()  # again: the probe resets its own state
        s = make_scene(96, 64, 32, 7)
        disp = ctx.run_pair(s.left, s.right, 32, E.default_params(post=1))
    finally:
        ctx.close()
    ref = O.driver_median(O.pipeline(s.left, s.right, 32)["disp"])
    assert np.array_equal(disp.view(np.uint32), ref.view(np.uint32))
