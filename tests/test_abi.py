"""The C ABI library loads and exports every function include/hbp_b200.h
declares; host-only entry points answer without a GPU."""
import ctypes as C

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
