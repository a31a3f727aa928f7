"""The C ABI library loads and exports every function include/hbp_b200.h
declares; host-only entry points answer without a GPU."""
import ctypes as C

import numpy as np
import pytest


@pytest.fixture(scope="module")
def lib():
    import build as engine_build  # hbp-isp_b200/build.py (incremental)
    engine_build.build()
    import hbp_b200 as E
    return E, E.lib()


def test_every_declared_symbol_is_exported(lib):
    E, L = lib
    names = E.exported_symbols_from_header()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_host_only_entry_points(lib):
    E, L = lib
    p = E.default_params()
    assert abs(p.alpha - 1000.1) < 1e-3 and abs(p.tau_smooth - 0.6) < 1e-6 and p.min_level == 2
    assert L.hbp_status_string(0) == b"ok" and L.hbp_status_string(5) == b"CUDA error"
    for code, name in E.STATUS.items():  # the binding's table is the library's
        assert L.hbp_status_string(code) == name.encode(), code
    assert E.volume_bytes(720, 496, 128) == 720 * 496 * 128
    assert E.volume_bytes(17, 5, 3) == 3 * 2 * 3 * 32  # overhanging tiles are stored whole
    h = C.c_void_p()
    assert L.hbp_ctx_create(0, -5, 0, C.byref(h)) != 0  # bad arguments rejected
    ph = (C.c_double * 4)()
    assert L.hbp_last_phase_ms(None, ph) == 1


def test_noalloc_rejects_before_touching_the_device(lib):
    E, L = lib
    with pytest.raises(E.HbpError):
        E.driver_median_noalloc_d(None, 720, 496)
    assert L.hbp_driver_median_noalloc_d(C.c_void_p(16), 0, 10, None) == 1
    assert L.hbp_driver_median_noalloc_d(C.c_void_p(16), 2049, 1024, None) == 1


def test_new_entry_points_reject_bad_arguments_on_the_host(lib):
    """The MC-CNN, AD, segmentation-variant, per-level, median and pyramid entry
    points check their arguments before any device work (no GPU needed)."""
    E, L = lib
    P = C.c_void_p
    p16 = P(16)
    INVALID = 1
    f = C.c_float
    assert L.hbp_volume_f32_bytes(720, 496, 128) == 4 * 720 * 496 * 128
    assert L.hbp_volume_f32_bytes(0, 496, 128) == 0
    # null context / pointers, tau <= 0, no output pair
    assert L.hbp_cost_f32_d(None, p16, 64, 64, 16, f(0.5), p16, p16, None, None, None) == INVALID
    assert L.hbp_cost_f32_d(p16, None, 64, 64, 16, f(0.5), p16, p16, None, None, None) == INVALID
    assert L.hbp_cost_f32_d(p16, p16, 64, 64, 16, f(0.0), p16, p16, None, None, None) == INVALID
    assert L.hbp_cost_f32_d(p16, p16, 64, 64, 16, f(0.5), None, None, None, None, None) == INVALID
    assert L.hbp_cost_f32_d(p16, p16, 64, 64, 16, f(0.5), p16, None, None, None, None) == INVALID
    assert L.hbp_cost_ad_d(None, p16, p16, 64, 64, 16, p16, p16, p16, p16, None, None, None) == INVALID
    assert L.hbp_cost_ad_d(p16, p16, p16, 64, 64, 16, None, p16, p16, p16, None, None, None) == INVALID
    assert L.hbp_infer_f32_d(None, p16, p16, 16, f(0.5), None, p16, None, None) == INVALID
    assert L.hbp_infer_levels_d(None, p16, None, p16, 16, f(25.0), None, 8, p16, None, None, None) == INVALID
    assert L.hbp_segment_cfg_d(None, p16, 64, 64, 2, 4, C.c_double(0.0), P(16), None) == INVALID
    assert L.hbp_lab_sigma_d(None, p16, 64, 64, C.c_double(1.0), p16, None) == INVALID
    assert L.hbp_weighted_median_gpu_d(None, p16, p16, p16, None, 64, 64, None) == INVALID
    assert L.hbp_patch_weights_d(None, p16, None) == INVALID
    ptrs = (P * 4)()
    assert L.hbp_pyramid_device(None, ptrs, None, None, None) == INVALID


def test_params_layout_matches_the_binding(lib):
    """The Python binding's hbp_params (the layout a ctypes binding declares)
    has the C struct's size, and the defaults are the reference's."""
    E, L = lib
    L.hbp_params_size.restype = C.c_size_t
    assert C.sizeof(E.Params) == L.hbp_params_size()
    p = E.default_params()
    assert (p.linkage, p.num_nb, p.sigma, p.msg_fp16, p.post) == (2, 4, 0.0, 0, 1)


def test_volume_layout_helper(lib):
    """volume_to_dhw inverts the Census volume layout the header states, at a
    ragged size (W and H not multiples of the tile size)."""
    E, L = lib
    W, H, D = 19, 6, 7
    rng = np.random.default_rng(3)
    dhw = rng.integers(0, 26, (D, H, W), dtype=np.uint8)
    TX = (W + 7) // 8
    buf = np.zeros(E.volume_bytes(W, H, D), np.uint8)
    for d in range(D):
        for y in range(H):
            for x in range(W):
                buf[((y // 4 * TX + x // 8) * D + d) * 32 + (y % 4) * 8 + x % 8] = dhw[d, y, x]
    assert np.array_equal(E.volume_to_dhw(buf, W, H, D), dhw.reshape(D, H * W))
