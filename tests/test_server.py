"""Request server (continuous batching): every result equals the single-pair
path's bit for bit, alone and in a mix of sizes running together; admission
by device footprint. GPU tests, plus argument checks that need no GPU."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hbp_b200 as E
    return E


MIX = [(160, 120, 48, 21), (96, 64, 32, 22), (450, 375, 64, 23), (320, 240, 64, 24), (160, 120, 48, 25),
       (200, 150, 40, 26)]


@pytest.mark.gpu
@pytest.mark.parametrize("fp16", [0, 1])
def test_results_alone_and_in_a_mix_equal_run_pair(gpu, fp16):
    E = gpu
    from scenes import make_scene
    scenes = [make_scene(W, H, D, seed) for W, H, D, seed in MIX]
    prm = E.default_params(post=1, msg_fp16=fp16)
    ctx = E.Context(0)
    try:
        want = [ctx.run_pair(s.left, s.right, D, prm) for s, (_, _, D, _) in zip(scenes, MIX)]
    finally:
        ctx.close()
    srv = E.Server(0, budget_bytes=16 << 30, prep_lanes=3, params=prm)
    try:
        # alone
        rid = srv.submit(scenes[2].left, scenes[2].right, MIX[2][2])
        alone, lat = srv.wait(rid)
        assert lat > 0
        assert np.array_equal(alone.view(np.uint32), want[2].view(np.uint32))
        # all at once: they join the BP of those already running
        ids = [srv.submit(s.left, s.right, D) for s, (_, _, D, _) in zip(scenes, MIX)]
        for rid, w in zip(ids, want):
            got, _ = srv.wait(rid)
            assert np.array_equal(got.view(np.uint32), w.view(np.uint32))
    finally:
        srv.close()


@pytest.mark.gpu
def test_segmentation_variant_through_the_server(gpu):
    """A server created with another SegHAC configuration (Ward linkage, 8
    neighbours, pre-blur) returns hbp_run_pair's result with the same
    parameters, bit for bit."""
    E = gpu
    from scenes import make_scene
    prm = E.default_params(post=1, msg_fp16=1, linkage=3, num_nb=8, sigma=0.7)
    s = make_scene(160, 120, 48, 31)
    ctx = E.Context(0)
    try:
        want = ctx.run_pair(s.left, s.right, 48, prm)
    finally:
        ctx.close()
    srv = E.Server(0, budget_bytes=8 << 30, prep_lanes=2, params=prm)
    try:
        got, _ = srv.wait(srv.submit(s.left, s.right, 48))
    finally:
        srv.close()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_server_rejects_a_bad_segmentation_configuration():
    """The configuration is checked when the server is created (no GPU needed)."""
    import hbp_b200 as E
    with pytest.raises(E.HbpError):
        E.Server(0, budget_bytes=1 << 30, prep_lanes=1, params=E.default_params(post=1, num_nb=6))


@pytest.mark.gpu
def test_admission_by_footprint(gpu):
    E = gpu
    from scenes import make_scene
    need = E.request_bytes(160, 120, 48)
    prm = E.default_params(post=1)
    srv = E.Server(0, budget_bytes=need + need // 2, prep_lanes=2, params=prm)  # one pair at a time
    try:
        with pytest.raises(E.HbpError) as ei:
            s = make_scene(320, 240, 64, 1)
            srv.submit(s.left, s.right, 64)
        assert ei.value.status == 3  # admission rejected: can never fit
        scenes = [make_scene(160, 120, 48, 30 + i) for i in range(4)]
        ids = [srv.submit(s.left, s.right, 48) for s in scenes]
        outs = [srv.wait(i)[0] for i in ids]
    finally:
        srv.close()
    ctx = E.Context(0)
    try:
        for s, o in zip(scenes, outs):
            assert np.array_equal(o, ctx.run_pair(s.left, s.right, 48, prm))
    finally:
        ctx.close()


def test_server_arguments_checked_without_gpu():
    import ctypes as C
    import build as engine_build
    engine_build.build()
    import hbp_b200 as E
    L = E.lib()
    h = C.c_void_p()
    assert L.hbp_server_create(0, 0, 2, None, C.byref(h)) == 1  # no budget
    assert L.hbp_server_create(0, 1 << 30, 0, None, C.byref(h)) == 1  # no lanes
    p = E.default_params(post=2)
    assert L.hbp_server_create(0, 1 << 30, 2, C.byref(p), C.byref(h)) == 1  # LR post not served
    assert E.request_bytes(720, 496, 128) > 720 * 496 * 128
    assert L.hbp_poll(None, 1) == 1


@pytest.mark.gpu
def test_device_memory_returns_after_contexts_and_servers(gpu):
    """Destroying a context or a server frees its slabs, including the slabs the
    server's pool frees to make room for a larger pair."""
    E = gpu
    import torch
    from scenes import make_scene
    small, big = make_scene(160, 120, 48, 40), make_scene(320, 240, 64, 41)
    prm = E.default_params(post=1)

    def cycle():
        ctx = E.Context(0)
        ctx.run_pair(small.left, small.right, 48, prm)
        ctx.close()
        need = E.request_bytes(320, 240, 64)
        srv = E.Server(0, budget_bytes=need + need // 2, prep_lanes=1, params=prm)
        for s, D in ((small, 48), (big, 64), (small, 48), (big, 64)):
            srv.wait(srv.submit(s.left, s.right, D))
        srv.close()

    cycle()  # the first use loads modules and creates the runtime's own state
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        cycle()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 < (64 << 20), (free0, free1)


@pytest.mark.gpu
def test_destroy_finishes_requests_still_in_preparation(gpu):
    """hbp_server_destroy right after submitting: every admitted request,
    including those a preparation lane has not yet finished (or started),
    still runs to the end and writes its disparity, equal to hbp_run_pair's."""
    E = gpu
    from scenes import make_scene
    prm = E.default_params(post=1)
    scenes = [make_scene(160, 120, 48, 50 + i) for i in range(6)]
    ctx = E.Context(0)
    try:
        want = [ctx.run_pair(s.left, s.right, 48, prm) for s in scenes]
    finally:
        ctx.close()
    srv = E.Server(0, budget_bytes=8 << 30, prep_lanes=1, params=prm)  # all fit: none is dropped
    ids = [srv.submit(s.left, s.right, 48) for s in scenes]
    outs = [srv._live[i][2] for i in ids]
    keep = dict(srv._live)  # the buffers must outlive the destroy
    srv.close()
    for o, w in zip(outs, want):
        assert np.array_equal(o.view(np.uint32), w.view(np.uint32))
    del keep


@pytest.mark.gpu
def test_small_requests_pass_a_large_one_that_does_not_fit(gpu):
    """Admission with bypass: a large pair that must wait for memory does not
    hold back the small pairs queued behind it; it still runs, with the result
    of hbp_run_pair."""
    E = gpu
    import time
    from scenes import make_scene
    prm = E.default_params(post=1)
    big = [make_scene(720, 496, 128, 60 + i) for i in range(2)]
    small = [make_scene(96, 64, 32, 70 + i) for i in range(3)]
    nb, ns = E.request_bytes(720, 496, 128), E.request_bytes(96, 64, 32)
    budget = nb + 3 * ns + ns // 2  # the second large pair waits for the first's memory
    assert 2 * nb > budget
    srv = E.Server(0, budget_bytes=budget, prep_lanes=2, params=prm)
    try:
        t0 = time.perf_counter()
        ids = [(srv.submit(b.left, b.right, 128), time.perf_counter()) for b in big]
        ids += [(srv.submit(s.left, s.right, 32), time.perf_counter()) for s in small]
        done = []
        for rid, ts in ids:
            out, lat = srv.wait(rid)
            done.append((ts - t0) * 1e3 + lat)
            if rid == ids[1][0]:
                second_big = out
    finally:
        srv.close()
    # every small pair finished before the second large one, which had to
    # wait for the first large one's memory
    assert max(done[2:]) < done[1], done
    ctx = E.Context(0)
    try:
        assert np.array_equal(second_big, ctx.run_pair(big[1].left, big[1].right, 128, prm))
    finally:
        ctx.close()
