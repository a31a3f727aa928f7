"""hbp_driver_median_noalloc_d: the driver median with its scratch in a static
device array, checked against the context entry point hbp_driver_median_d on
two calls in a row. Requires a GPU. The file name keeps it last in collection
so it also runs after every other test has used the library."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Both paths run the same float comparisons on the same values, so the
# tolerance is zero: results must be identical bit for bit.
ATOL = 0.0


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hbp_b200 as E
    return E, torch


def disparity(rng, H, W):
    d = rng.uniform(0, 120, (H, W)).astype(np.float32)
    d[rng.uniform(size=d.shape) < 0.07] = -1.0  # invalid pixels stay untouched
    return d


def test_noalloc_matches_context_path_two_calls(env):
    E, torch = env
    rng = np.random.default_rng(17)
    maps = [disparity(rng, 496, 720), disparity(rng, 375, 450)]
    ctx = E.Context(0)
    try:
        want = []
        for d in maps:
            t = torch.from_numpy(d.copy()).cuda()
            ctx.driver_median_d(t, d.shape[1], d.shape[0])
            want.append(t.cpu().numpy())
    finally:
        ctx.close()
    inputs = [torch.from_numpy(d.copy()).cuda() for d in maps]
    torch.cuda.synchronize()
    free = []
    for t, d, w in zip(inputs, maps, want):
        E.driver_median_noalloc_d(t, d.shape[1], d.shape[0])
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        got = t.cpu().numpy()
        np.testing.assert_allclose(got, w, rtol=0, atol=ATOL)
        assert not np.array_equal(got, d)  # the filter did change the map
    # the first call did the one-time setup; the second one allocated nothing
    assert free[1] == free[0]


def test_noalloc_on_side_stream(env):
    E, torch = env
    import pyoracle as O
    rng = np.random.default_rng(5)
    d = disparity(rng, 70, 90)
    t = torch.from_numpy(d.copy()).cuda()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    E.driver_median_noalloc_d(t, 90, 70, s.cuda_stream)
    s.synchronize()
    np.testing.assert_allclose(t.cpu().numpy(), O.driver_median(d), rtol=0, atol=ATOL)


def test_noalloc_rejects_oversize(env):
    E, torch = env
    t = torch.zeros(16, device="cuda")
    W, H = 2049, 1024  # 2049*1024 > HBP_NOALLOC_MAX_PIXELS; nothing is launched
    assert W * H > E.NOALLOC_MAX_PIXELS
    with pytest.raises(E.HbpError) as ei:
        E.driver_median_noalloc_d(t, W, H)
    assert ei.value.status == 1 and "HBP_NOALLOC_MAX_PIXELS" in str(ei.value)
    assert torch.count_nonzero(t).item() == 0
