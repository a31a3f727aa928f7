"""Python binding of the B200 HBP-ISP engine's C ABI (include/hbp_b200.h).

Host-buffer entry points take numpy arrays; the ``*_d`` stage entry points
take device tensors (torch) and pass their data pointers. The engine library
must be built (``python hbp-isp_b200/build.py``); there is no fallback: a
missing library raises ``EngineUnavailable``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("HBP_B200_LIB") or os.path.join(HERE, "lib", "libhbp_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "hbp_b200.h")

P = C.c_void_p
STATUS = {0: "ok", 1: "invalid argument", 2: "out of memory", 3: "admission rejected", 4: "no convergence",
          5: "CUDA error", 6: "timeout", 7: "not ready", 8: "internal error", 9: "cancelled"}


class EngineUnavailable(RuntimeError):
    pass


class HbpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Params(C.Structure):
    _fields_ = [("alpha", C.c_float), ("tau_smooth", C.c_float), ("min_level", C.c_int),
                ("msg_fp16", C.c_int), ("post", C.c_int), ("linkage", C.c_int), ("num_nb", C.c_int),
                ("sigma", C.c_double)]


_lib = None


def lib():
    """Load the engine library (raises EngineUnavailable if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EngineUnavailable(f"{LIB_PATH} not built; run python hbp-isp_b200/build.py")
        L = C.CDLL(LIB_PATH)
        L.hbp_last_error.restype = C.c_char_p
        L.hbp_status_string.restype = C.c_char_p
        L.hbp_ctx_stream.restype = P
        L.hbp_ctx_create.argtypes = [C.c_int, C.c_long, C.c_int, C.POINTER(P)]
        L.hbp_lab_d.argtypes = [P, P, C.c_long, P, P]
        L.hbp_request_bytes.restype = C.c_size_t
        L.hbp_server_create.argtypes = [C.c_int, C.c_size_t, C.c_int, P, C.POINTER(P)]
        L.hbp_server_destroy.argtypes = [P]
        L.hbp_submit.argtypes = [P, P, P, C.c_int, C.c_int, C.c_int, P, C.POINTER(C.c_longlong)]
        L.hbp_poll.argtypes = [P, C.c_longlong]
        L.hbp_wait.argtypes = [P, C.c_longlong, C.c_double, C.POINTER(C.c_double)]
        L.hbp_autotune_table.argtypes = [P, P, C.c_int]
        L.hbp_autotune_table.restype = C.c_int
        _lib = L
    return _lib


def exported_symbols_from_header(path: str = HEADER) -> list[str]:
    """Function names declared in the C header."""
    import re
    txt = open(path).read()
    return sorted(set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(hbp_\w+)\s*\(", txt, flags=re.M)))


def _check(st: int):
    if st != 0:
        raise HbpError(st, lib().hbp_last_error().decode())


def _p(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(P)
    # a torch tensor on the device: the engine runs on its own non-blocking
    # stream, so torch's pending work on the tensor (a fill, a copy) must
    # finish first
    import torch
    torch.cuda.current_stream(a.device).synchronize()
    return P(a.data_ptr())


def default_params(**kw) -> Params:
    p = Params()
    lib().hbp_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def volume_f32_bytes(W: int, H: int, D: int) -> int:
    """Size of the tiled float volume of the MC-CNN path."""
    f = lib().hbp_volume_f32_bytes
    f.restype = C.c_size_t
    return f(W, H, D)


def volume_f32_to_dhw(vol: np.ndarray, W: int, H: int, D: int) -> np.ndarray:
    """Tiled float volume -> [D][H*W]."""
    TX, TY = (W + 7) // 8, (H + 3) // 4
    v = np.asarray(vol, np.float32)[: TX * TY * D * 32].reshape(TY, TX, D, 4, 8)
    v = v.transpose(2, 0, 3, 1, 4).reshape(D, TY * 4, TX * 8)[:, :H, :W]
    return np.ascontiguousarray(v.reshape(D, H * W))


def volume_bytes(W: int, H: int, D: int) -> int:
    """Size of the tiled cost volume (see hbp_volume_bytes in the header)."""
    f = lib().hbp_volume_bytes
    f.restype = C.c_size_t
    return f(W, H, D)


def volume_to_dhw(buf: np.ndarray, W: int, H: int, D: int) -> np.ndarray:
    """Tiled volume bytes -> [D][H*W] (the reference's disparity-major order)."""
    TX, TY = (W + 7) // 8, (H + 3) // 4
    v = np.asarray(buf, np.uint8)[: TX * TY * D * 32].reshape(TY, TX, D, 4, 8)
    v = v.transpose(2, 0, 3, 1, 4).reshape(D, TY * 4, TX * 8)[:, :H, :W]
    return np.ascontiguousarray(v.reshape(D, H * W))


NOALLOC_MAX_PIXELS = 2097152  # HBP_NOALLOC_MAX_PIXELS of the header


def driver_median_noalloc_d(disp, W: int, H: int, stream: int | None = None):
    """hbp_driver_median_noalloc_d: in-place driver median of a device disparity
    map on the current device, no context and no device allocation; enqueued
    on ``stream`` (None = legacy default stream) and not synchronised."""
    _check(lib().hbp_driver_median_noalloc_d(_p(disp), W, H, P(stream) if stream else None))


class Context:
    """One device context (stream + device memory slab). Not thread safe."""

    def __init__(self, device: int = 0, max_pixels: int = 0, max_disp: int = 0):
        h = P()
        _check(lib().hbp_ctx_create(device, max_pixels, max_disp, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().hbp_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return lib().hbp_ctx_stream(self.h) or 0

    # ------------------------------------------------------------ whole pair
    def run_pair(self, left: np.ndarray, right: np.ndarray, D: int, params: Params | None = None,
                 want_plane: bool = False):
        left = np.ascontiguousarray(left, np.uint8)
        right = np.ascontiguousarray(right, np.uint8)
        H, W = left.shape[:2]
        disp = np.zeros((H, W), np.float32)
        plane = np.zeros((H, W, 3), np.float32) if want_plane else None
        prm = params or default_params()
        _check(lib().hbp_run_pair(self.h, _p(left), _p(right), W, H, D, C.byref(prm), _p(disp), _p(plane)))
        return (disp, plane) if want_plane else disp

    # ------------------------------------------------------------ stages (device)
    def cost_census_d(self, bgrL, bgrR, W, H, D, censusL, censusR, vol, wta, volR=None, wtaR=None):
        _check(lib().hbp_cost_census_d(self.h, _p(bgrL), _p(bgrR), W, H, D, _p(censusL), _p(censusR),
                                       _p(vol), _p(wta), _p(volR), _p(wtaR), None))

    def cost_f32_d(self, src, W, H, D, tau, vol, wta, volR=None, wtaR=None):
        _check(lib().hbp_cost_f32_d(self.h, _p(src), W, H, D, C.c_float(tau), _p(vol), _p(wta), _p(volR),
                                    _p(wtaR), None))

    def cost_ad_d(self, bgrL, bgrR, W, H, D, greyL, greyR, vol, wta, volR=None, wtaR=None):
        _check(lib().hbp_cost_ad_d(self.h, _p(bgrL), _p(bgrR), W, H, D, _p(greyL), _p(greyR), _p(vol), _p(wta),
                                   _p(volR), _p(wtaR), None))

    def infer_f32_d(self, vol, wta, D, tau, params: Params | None, disp, plane=None):
        prm = params or default_params()
        _check(lib().hbp_infer_f32_d(self.h, _p(vol), _p(wta), D, C.c_float(tau), C.byref(prm), _p(disp),
                                     _p(plane), None))

    def infer_levels_d(self, vol, volf, wta, D, tau, params: Params | None, max_levels, disp_levels,
                       plane_levels=None) -> int:
        prm = params or default_params()
        n = C.c_int(0)
        _check(lib().hbp_infer_levels_d(self.h, _p(vol), _p(volf), _p(wta), D, C.c_float(tau), C.byref(prm),
                                        max_levels, _p(disp_levels), _p(plane_levels), C.byref(n), None))
        return n.value

    def lab_d(self, bgr, n, lab4):
        _check(lib().hbp_lab_d(self.h, _p(bgr), n, _p(lab4), None))

    def crtrees_d(self, nn, N, clus) -> int:
        k = C.c_int(0)
        _check(lib().hbp_crtrees_d(self.h, _p(nn), N, _p(clus), C.byref(k), None))
        return k.value

    def segment_cfg_d(self, bgr, W, H, linkage, num_nb, sigma) -> int:
        L = C.c_int(0)
        _check(lib().hbp_segment_cfg_d(self.h, _p(bgr), W, H, linkage, num_nb, C.c_double(sigma), C.byref(L),
                                       None))
        return L.value

    def segment_target_d(self, bgr, W, H, linkage, num_nb, sigma, target_clus) -> int:
        L = C.c_int(0)
        _check(lib().hbp_segment_target_d(self.h, _p(bgr), W, H, linkage, num_nb, C.c_double(sigma), target_clus,
                                          C.byref(L), None))
        return L.value

    def segment_draw_d(self, out, fmt: int, bgr=None, level: int = -1) -> None:
        """SegHAC's picture of level `level` into device memory `out`: fmt 0
        label+1 as BGR bytes, 1 label+1 as ints, 2 the boundaries over `bgr`."""
        _check(lib().hbp_segment_draw_d(self.h, level, fmt, _p(bgr), _p(out), None))

    def segment_labels_d(self, labels, level: int = -1) -> int:
        """Every pixel's cluster after pyramid level `level` (-1: the last)
        as device ints; returns the number of clusters."""
        k = C.c_int(0)
        _check(lib().hbp_segment_labels_d(self.h, level, _p(labels), C.byref(k), None))
        return k.value

    def lab_sigma_d(self, bgr, W, H, sigma, lab4):
        _check(lib().hbp_lab_sigma_d(self.h, _p(bgr), W, H, C.c_double(sigma), _p(lab4), None))

    def segment_d(self, bgr, W, H) -> int:
        L = C.c_int(0)
        _check(lib().hbp_segment_d(self.h, _p(bgr), W, H, C.byref(L), None))
        return L.value

    def pyramid(self) -> dict:
        """The last pyramid in the reference's ISP layout (host arrays)."""
        sizes = np.zeros(2 * 64, np.int32)
        _check(lib().hbp_pyramid_levels(self.h, _p(sizes), 64))
        sizes = sizes.reshape(64, 2)
        L = int(np.count_nonzero(sizes[:, 0]))
        sizes = sizes[:L].copy()
        tn, te = int(sizes[:, 0].sum()), int(sizes[:, 1].sum())
        clus = np.zeros(tn, np.int32)
        mean = np.zeros(6 * tn, np.float32)
        bd = np.zeros((te, 2), np.int32)
        bdl = np.zeros(te, np.int32)
        _check(lib().hbp_pyramid_copy(self.h, _p(clus), _p(mean), _p(bd), _p(bdl)))
        return dict(level_sizes=sizes, clus=clus, mean=mean, bd=bd, bdl=bdl)

    def infer_d(self, vol, wta, D, params: Params | None, disp, plane=None):
        prm = params or default_params()
        _check(lib().hbp_infer_d(self.h, _p(vol), _p(wta), D, C.byref(prm), _p(disp), _p(plane), None))

    def lr_check_d(self, dispL, dispR, planeL, fail, disp_out, W, H):
        _check(lib().hbp_lr_check_d(self.h, _p(dispL), _p(dispR), _p(planeL), _p(fail), _p(disp_out), W, H, None))

    def weighted_median_d(self, bgrL, fail, plane, disp_out, W, H):
        _check(lib().hbp_weighted_median_d(self.h, _p(bgrL), _p(fail), _p(plane), _p(disp_out), W, H, None))

    def weighted_median_gpu_d(self, bgrL, fail, plane, disp_out, W, H):
        _check(lib().hbp_weighted_median_gpu_d(self.h, _p(bgrL), _p(fail), _p(plane), _p(disp_out), W, H, None))

    def check_bounded_wait(self) -> bool:
        t = C.c_int(0)
        _check(lib().hbp_check_bounded_wait(self.h, C.byref(t)))
        return bool(t.value)

    def patch_weights_d(self, wtab766):
        _check(lib().hbp_patch_weights_d(self.h, _p(wtab766), None))

    def driver_median_d(self, disp, W, H):
        _check(lib().hbp_driver_median_d(self.h, _p(disp), W, H, None))


def request_bytes(W: int, H: int, D: int) -> int:
    """Device footprint the server admits a W x H x D pair by."""
    return lib().hbp_request_bytes(W, H, D)


class Server:
    """hbp_server: continuous-batching request server on one GPU. submit()
    takes host arrays (kept referenced until wait() returns) and returns a
    request id; wait() returns (disparity, latency_ms)."""

    def __init__(self, device: int = 0, budget_bytes: int = 120 << 30, prep_lanes: int = 4,
                 params: Params | None = None):
        h = P()
        prm = params or default_params(post=1)
        _check(lib().hbp_server_create(device, budget_bytes, prep_lanes, C.byref(prm), C.byref(h)))
        self.h = h
        self._live = {}

    def submit(self, left: np.ndarray, right: np.ndarray, D: int) -> int:
        left = np.ascontiguousarray(left, np.uint8)
        right = np.ascontiguousarray(right, np.uint8)
        H, W = left.shape[:2]
        out = np.zeros((H, W), np.float32)
        rid = C.c_longlong(0)
        _check(lib().hbp_submit(self.h, _p(left), _p(right), W, H, D, _p(out), C.byref(rid)))
        self._live[rid.value] = (left, right, out)
        return rid.value

    def poll(self, rid: int) -> bool:
        st = lib().hbp_poll(self.h, rid)
        if st == 7:
            return False
        _check(st)
        return True

    def wait(self, rid: int, timeout_ms: float = -1.0):
        lat = C.c_double(0)
        st = lib().hbp_wait(self.h, rid, timeout_ms, C.byref(lat))
        if st == 6:  # still running: keep the buffers
            _check(st)
        _, _, out = self._live.pop(rid)
        _check(st)
        return out, lat.value

    def close(self):
        if self.h:
            lib().hbp_server_destroy(self.h)
            self.h = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
