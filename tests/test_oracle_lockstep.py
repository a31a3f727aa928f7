"""The oracle's lock-step message-error mode (CPU): a shadow run that takes the
main float run's discrete decisions (candidate planes, kept slots) and carries
its own costs, beliefs and messages. In float it must repeat the run exactly
(every difference 0), which checks the replay's bookkeeping; in FP64 it gives
the message error of FP32 and FP16 storage. Neither changes the main run."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def case():
    import pyoracle as O
    from scenes import make_scene
    s = make_scene(96, 64, 32, 7)
    return O, s, O.cost_stage(s.left, s.right, 32), O.segment(O.lab(s.left))


@pytest.mark.parametrize("fp16", [False, True])
def test_float_shadow_repeats_the_run(case, fp16):
    O, s, cs, seg = case
    disp, st = O.hbp_lockstep(seg, cs["vol"], cs["wta"], 96, 64, 32, fp16_msg=fp16, shadow_fp64=False)
    ref = O.hbp(seg, cs["vol"], cs["wta"], 96, 64, 32, fp16_msg=fp16)[0]
    assert np.array_equal(disp.view(np.uint32), ref.view(np.uint32))
    assert st["values"] > 0 and st["msg_ref_max"] > 0
    if not fp16:
        assert st["msg_err_max"] == 0.0 and st["msg_raw_err_max"] == 0.0
    else:  # the FP16 rounding of the stored values, carried along by the beliefs
        assert 0.0 < st["msg_err_mean"] < 1e-3 * st["msg_ref_mean"]
        assert st["msg_err_max"] < 0.01 * st["msg_ref_max"]


def test_fp64_shadow_message_error(case):
    O, s, cs, seg = case
    d32, e32 = O.hbp_lockstep(seg, cs["vol"], cs["wta"], 96, 64, 32, fp16_msg=False)
    d16, e16 = O.hbp_lockstep(seg, cs["vol"], cs["wta"], 96, 64, 32, fp16_msg=True)
    assert np.array_equal(d32, O.hbp(seg, cs["vol"], cs["wta"], 96, 64, 32)[0])
    assert np.array_equal(d16, O.hbp(seg, cs["vol"], cs["wta"], 96, 64, 32, fp16_msg=True)[0])
    for e in (e32, e16):
        assert 0.0 < e["msg_err_mean"] < 0.05 * e["msg_ref_mean"]
        assert e["msg_err_max"] <= e["msg_ref_max"]
    # FP16 storage adds little to the float arithmetic's own error
    assert e16["msg_err_mean"] < 1.25 * e32["msg_err_mean"]

