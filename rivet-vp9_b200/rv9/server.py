"""The serving engine of include/rv9_server.h: many live streams on one GPU,
admitted by an HBM budget, their requests overlapping on the device.

    eng = Engine(device=0, hbm_budget=120 << 30)
    sid = eng.open_stream(1920, 1080, bit_depth=8)
    eng.submit(sid, packet, tag=7)
    for c in eng.poll(timeout_ms=100):
        c.frames        # Frame objects (packed planes)
        c.latency_ms    # submit -> frames in host memory
"""
import ctypes

from . import CFrame, DeviceError, Frame, RV9_OK, Rv9Error, _ERRORS, load_library


class CStreamSpec(ctypes.Structure):
    _fields_ = [("max_width", ctypes.c_uint32), ("max_height", ctypes.c_uint32), ("bit_depth", ctypes.c_uint32),
                ("ss_x", ctypes.c_uint32), ("ss_y", ctypes.c_uint32)]


class CCompletion(ctypes.Structure):
    _fields_ = [("stream", ctypes.c_int64), ("tag", ctypes.c_uint64), ("status", ctypes.c_int),
                ("n_frames", ctypes.c_uint32), ("submit_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("frames", CFrame * 2), ("handle", ctypes.c_void_p)]


class CEngineStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("streams_open", "streams_pending", "requests_submitted",
                                              "requests_completed", "frames_decoded", "reserved_bytes",
                                              "budget_bytes")]


EXPORTS = ("rv9_engine_create", "rv9_engine_free", "rv9_stream_reservation", "rv9_stream_open", "rv9_stream_close",
           "rv9_submit", "rv9_poll", "rv9_completion_release", "rv9_engine_get_stats")


def _bind(lib):
    if getattr(lib, "_rv9_server_bound", False):
        return lib
    vp = ctypes.c_void_p
    lib.rv9_engine_create.restype = vp
    lib.rv9_engine_create.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32]
    lib.rv9_engine_free.argtypes = [vp]
    lib.rv9_stream_reservation.restype = ctypes.c_uint64
    lib.rv9_stream_reservation.argtypes = [ctypes.POINTER(CStreamSpec)]
    lib.rv9_stream_open.argtypes = [vp, ctypes.POINTER(CStreamSpec), ctypes.POINTER(ctypes.c_int64)]
    lib.rv9_stream_close.argtypes = [vp, ctypes.c_int64]
    lib.rv9_submit.argtypes = [vp, ctypes.c_int64, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint64]
    lib.rv9_poll.restype = ctypes.c_size_t
    lib.rv9_poll.argtypes = [vp, ctypes.POINTER(CCompletion), ctypes.c_size_t, ctypes.c_int]
    lib.rv9_completion_release.argtypes = [vp, ctypes.POINTER(CCompletion)]
    lib.rv9_engine_get_stats.argtypes = [vp, ctypes.POINTER(CEngineStats)]
    lib._rv9_server_bound = True
    return lib


def spec(width, height, bit_depth=8, chroma=(1, 1)):
    return CStreamSpec(width, height, bit_depth, chroma[0], chroma[1])


def reservation(width, height, bit_depth=8, chroma=(1, 1), lib_path=None):
    """Device bytes the engine reserves for a stream of this size (no GPU
    needed)."""
    lib = _bind(load_library(lib_path))
    s = spec(width, height, bit_depth, chroma)
    return lib.rv9_stream_reservation(ctypes.byref(s))


class Completion:
    """A finished request. `frames` holds Frame objects copied out of the
    engine's pinned buffers, which go back to the stream at once."""

    def __init__(self, c, frames, md5s=None):
        self.stream, self.tag, self.status = c.stream, c.tag, c.status
        self.submit_ms, self.latency_ms = c.submit_ms, c.latency_ms
        self.n_frames = c.n_frames
        self.frames = frames
        self.md5s = md5s  # hex MD5 of each frame's packed planes, when asked for

    @property
    def ok(self):
        return self.status == RV9_OK


class Engine:
    def __init__(self, device=-1, hbm_budget=120 << 30, workers=0, lib_path=None):
        self._lib = _bind(load_library(lib_path))
        self._e = self._lib.rv9_engine_create(device, hbm_budget, workers)
        if not self._e:
            raise DeviceError(self._lib.rv9_last_global_error().decode(errors="replace"))

    def open_stream(self, width, height, bit_depth=8, chroma=(1, 1)):
        s = spec(width, height, bit_depth, chroma)
        sid = ctypes.c_int64()
        st = self._lib.rv9_stream_open(self._e, ctypes.byref(s), ctypes.byref(sid))
        if st != RV9_OK:
            raise _ERRORS.get(st, Rv9Error)(f"rv9_stream_open: status {st}")
        return sid.value

    def close_stream(self, sid):
        st = self._lib.rv9_stream_close(self._e, sid)
        if st != RV9_OK:
            raise _ERRORS.get(st, Rv9Error)(f"rv9_stream_close: status {st}")

    def submit(self, sid, packet, tag=0):
        st = self._lib.rv9_submit(self._e, sid, packet, len(packet), tag)
        if st != RV9_OK:
            raise _ERRORS.get(st, Rv9Error)(f"rv9_submit: status {st}")

    def poll(self, max_items=64, timeout_ms=0, keep_frames=True, digest=None):
        """Finished requests; with keep_frames False only their metadata is
        kept (the frames are not copied out). `digest(tag)` -> True asks for
        the MD5 of that request's frames, hashed in place in the engine's
        buffer before it is released (Completion.md5s)."""
        import hashlib
        arr = (CCompletion * max_items)()
        n = self._lib.rv9_poll(self._e, arr, max_items, timeout_ms)
        out = []
        for c in arr[:n]:
            frames = [Frame(c.frames[i]) for i in range(c.n_frames)] if keep_frames else []
            md5s = None
            if digest is not None and digest(c.tag) and c.status == RV9_OK:
                md5s = [hashlib.md5(memoryview((ctypes.c_char * c.frames[i].size).from_address(
                    ctypes.cast(c.frames[i].data, ctypes.c_void_p).value))).hexdigest() for i in range(c.n_frames)]
            out.append(Completion(c, frames, md5s))
            self._lib.rv9_completion_release(self._e, ctypes.byref(c))
        return out

    def stats(self):
        s = CEngineStats()
        self._lib.rv9_engine_get_stats(self._e, ctypes.byref(s))
        return {n: getattr(s, n) for n, _ in CEngineStats._fields_}

    def close(self):
        if getattr(self, "_e", None):
            self._lib.rv9_engine_free(self._e)
            self._e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
