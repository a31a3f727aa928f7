"""The profiling entry points (hbp_profile_enable / read / read_kernel /
breakdown): the data-cost figures of hbp_profile_read equal kernel 0 of
hbp_profile_read_kernel, both count timed launches with positive device
time and compulsory bytes, and the breakdown's timed launches are a subset
of all launches. Requires a GPU."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H, D, NP = 160, 120, 48, 4


def test_profile_entry_points():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hbp_b200 as E
    from scenes import make_scene

    scenes = [make_scene(W, H, D, 90 + i) for i in range(NP)]
    ctx = E.Context(0)
    try:
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        dL = [dev(s.left) for s in scenes]
        dR = [dev(s.right) for s in scenes]
        out = [torch.zeros((H, W), dtype=torch.float32, device="cuda") for _ in scenes]
        arr = lambda ts: (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])
        prm = E.default_params(post=1, msg_fp16=1)
        E._check(E.lib().hbp_set_bp_streams(ctx.h, 1))
        E._check(E.lib().hbp_profile_enable(ctx.h, 3))
        E._check(E.lib().hbp_run_batch_d(ctx.h, NP, arr(dL), arr(dR), W, H, D, C.byref(prm), arr(out), None))
        torch.cuda.synchronize()

        ms, n, b, px = C.c_double(), C.c_long(), C.c_double(), C.c_double()
        E._check(E.lib().hbp_profile_read(ctx.h, C.byref(ms), C.byref(n), C.byref(b), C.byref(px)))
        k = []
        for kern in (0, 1):
            kms, kn, kb, ku = C.c_double(), C.c_long(), C.c_double(), C.c_double()
            E._check(E.lib().hbp_profile_read_kernel(ctx.h, kern, C.byref(kms), C.byref(kn), C.byref(kb),
                                                     C.byref(ku)))
            k.append((kms.value, kn.value, kb.value, ku.value))
            assert kms.value > 0 and kn.value > 0 and kb.value > 0 and ku.value > 0
        assert (ms.value, n.value, b.value, px.value) == k[0]
        # data cost: 16 B per list position (8 B list entry, 2 x 4 volume bytes) at least
        assert k[0][2] >= 16.0 * k[0][3]

        cells = 10 * 32
        bms = (C.c_double * cells)()
        timed = (C.c_long * cells)()
        every = (C.c_long * cells)()
        E._check(E.lib().hbp_profile_breakdown(ctx.h, bms, timed, every))
        bms, timed, every = np.array(bms[:]), np.array(timed[:]), np.array(every[:])
        assert timed.sum() > 0 and np.all(timed <= every) and np.all(bms[timed == 0] == 0)
        assert bms.sum() > 0
        with pytest.raises(E.HbpError):
            E._check(E.lib().hbp_profile_read_kernel(ctx.h, 2, C.byref(ms), C.byref(n), C.byref(b), C.byref(px)))
        E._check(E.lib().hbp_profile_enable(ctx.h, 0))
    finally:
        ctx.close()
