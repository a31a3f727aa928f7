"""The BP-stream autotuner of batches (hbp_set_bp_streams, hbp_set_autotune,
hbp_autotune_table): the stream count changes no result, fixed or chosen by
the autotuner while it explores, and the autotuner's table records each
candidate count of the batch's class with exactly one chosen. Requires a
GPU."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H, D, NP = 160, 120, 48, 5


def test_stream_counts_and_autotuner_change_no_result():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hbp_b200 as E
    from scenes import make_scene

    scenes = [make_scene(W, H, D, 70 + i) for i in range(NP)]
    ctx = E.Context(0)
    try:
        prm = E.default_params(post=1)
        single = [ctx.run_pair(s.left, s.right, D, prm) for s in scenes]
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        dL = [dev(s.left) for s in scenes]
        dR = [dev(s.right) for s in scenes]
        out = [torch.zeros((H, W), dtype=torch.float32, device="cuda") for _ in scenes]
        arr = lambda ts: (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])

        def batch():
            for o in out:
                o.zero_()
            E._check(E.lib().hbp_run_batch_d(ctx.h, NP, arr(dL), arr(dR), W, H, D, C.byref(prm), arr(out), None))
            torch.cuda.synchronize()
            for a, b in zip(single, out):
                assert np.array_equal(a.view(np.uint32), b.cpu().numpy().view(np.uint32))

        def table():
            n = E.lib().hbp_autotune_table(ctx.h, None, 0)
            rows = (C.c_double * (9 * max(n, 1)))()
            assert E.lib().hbp_autotune_table(ctx.h, rows, n) == n
            return np.array(rows[:9 * n]).reshape(n, 9)

        t0 = table()  # the single pairs' class (one view, one stream)
        for s in (1, 3, 8):
            E._check(E.lib().hbp_set_bp_streams(ctx.h, s))
            batch()
        assert np.array_equal(table(), t0)  # a fixed count explores nothing

        E._check(E.lib().hbp_set_bp_streams(ctx.h, 0))
        E._check(E.lib().hbp_set_autotune(ctx.h, 1))
        # 5 views: candidates 2 and 4, two rounds each, then the choice
        for _ in range(5):
            batch()
        t = table()
        t = t[t[:, 5] == NP]
        assert sorted(t[:, 6].astype(int).tolist()) == [2, 4]
        assert np.all(t[:, :6].astype(int) == [W, H, D, 0, 1, NP])
        assert np.all(t[:, 7] > 0) and t[:, 8].sum() == 1
        chosen = t[t[:, 8] == 1][0]
        assert chosen[7] == t[:, 7].min()

        E._check(E.lib().hbp_set_autotune(ctx.h, 0))
        full = table()
        batch()
        assert np.array_equal(table(), full)
    finally:
        ctx.close()
