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
                                              "budget_bytes", "batched_steps", "batched_frames",
                                              "device_parse_batches", "device_parsed_frames",
                                              "device_parse_wait_us", "device_parse_batch_us")]


EXPORTS = ("rv9_engine_create", "rv9_engine_create_batched", "rv9_engine_free", "rv9_stream_reservation", "rv9_stream_open", "rv9_stream_close",
           "rv9_submit", "rv9_poll", "rv9_completion_release", "rv9_engine_get_stats", "rv9_engine_set_device_parse", "rv9_engine_stream_reservation",
           "rv9_cluster_create", "rv9_cluster_set_device_parse",
           "rv9_cluster_free", "rv9_cluster_stream_open", "rv9_cluster_stream_close", "rv9_cluster_submit",
           "rv9_cluster_poll", "rv9_cluster_completion_release", "rv9_cluster_get_stats", "rv9_place_least_loaded")


def _bind(lib):
    if getattr(lib, "_rv9_server_bound", False):
        return lib
    vp = ctypes.c_void_p
    lib.rv9_engine_create.restype = vp
    lib.rv9_engine_create.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32]
    lib.rv9_engine_create_batched.restype = vp
    lib.rv9_engine_create_batched.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32]
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
    lib.rv9_engine_set_device_parse.argtypes = [vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32]
    lib.rv9_engine_stream_reservation.restype = ctypes.c_uint64
    lib.rv9_engine_stream_reservation.argtypes = [vp, ctypes.POINTER(CStreamSpec)]
    lib.rv9_cluster_set_device_parse.argtypes = [vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32]
    lib.rv9_cluster_create.restype = vp
    lib.rv9_cluster_create.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint32]
    lib.rv9_cluster_free.argtypes = [vp]
    lib.rv9_cluster_stream_open.argtypes = [vp, ctypes.POINTER(CStreamSpec), ctypes.POINTER(ctypes.c_int64),
                                            ctypes.POINTER(ctypes.c_int)]
    lib.rv9_cluster_stream_close.argtypes = [vp, ctypes.c_int64]
    lib.rv9_cluster_submit.argtypes = [vp, ctypes.c_int64, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint64]
    lib.rv9_cluster_poll.restype = ctypes.c_size_t
    lib.rv9_cluster_poll.argtypes = [vp, ctypes.POINTER(CCompletion), ctypes.c_size_t, ctypes.c_int]
    lib.rv9_cluster_completion_release.argtypes = [vp, ctypes.POINTER(CCompletion)]
    lib.rv9_cluster_get_stats.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CEngineStats)]
    lib.rv9_place_least_loaded.restype = ctypes.c_int
    lib.rv9_place_least_loaded.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                           ctypes.c_size_t, ctypes.c_uint64]
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

    def __init__(self, c, frames):
        self.stream, self.tag, self.status = c.stream, c.tag, c.status
        self.submit_ms, self.latency_ms = c.submit_ms, c.latency_ms
        self.n_frames = c.n_frames
        self.frames = frames

    @property
    def ok(self):
        return self.status == RV9_OK


class Engine:
    """A serving engine (rv9_engine). `groups` > 0 makes the batched form
    (rv9_engine_create_batched): the streams' frames reconstructed together,
    one launch per stage per step, in that many launch groups."""

    def __init__(self, device=-1, hbm_budget=120 << 30, workers=0, lib_path=None, groups=0, device_parse=False,
                 window=0, max_batches=0):
        self._lib = _bind(load_library(lib_path))
        if groups:
            self._e = self._lib.rv9_engine_create_batched(device, hbm_budget, workers, groups)
        else:
            self._e = self._lib.rv9_engine_create(device, hbm_budget, workers)
        if not self._e:
            raise DeviceError(self._lib.rv9_last_global_error().decode(errors="replace"))
        if device_parse:
            self.set_device_parse(device_parse, window, max_batches)

    def set_device_parse(self, on=True, window=0, max_batches=0):
        """rv9_engine_set_device_parse: a stream's queued requests (two or
        more) parsed on the GPU in batches of up to `window`, for the streams
        opened after the call."""
        st = self._lib.rv9_engine_set_device_parse(self._e, 1 if on else 0, window, max_batches)
        if st != RV9_OK:
            raise _ERRORS.get(st, Rv9Error)(f"rv9_engine_set_device_parse: status {st}")

    def reservation(self, width, height, bit_depth=8, chroma=(1, 1)):
        """Device bytes a stream of this size reserves in this engine
        (rv9_engine_stream_reservation)."""
        s = spec(width, height, bit_depth, chroma)
        return self._lib.rv9_engine_stream_reservation(self._e, ctypes.byref(s))

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

    def poll(self, max_items=64, timeout_ms=0, keep_frames=True):
        """Finished requests. keep_frames: True copies every request's frames
        out of the engine's buffers (Completion.frames), False none, or a
        predicate on the request's tag picks the requests whose frames are
        copied."""
        arr = (CCompletion * max_items)()
        n = self._lib.rv9_poll(self._e, arr, max_items, timeout_ms)
        out = []
        for c in arr[:n]:
            keep = keep_frames(c.tag) if callable(keep_frames) else keep_frames
            frames = [Frame(c.frames[i]) for i in range(c.n_frames)] if keep else []
            out.append(Completion(c, frames))
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


def place_least_loaded(load, budget, need, lib_path=None):
    """The cluster's placement rule (rv9_place_least_loaded), no device
    needed: the index of the device a stream of `need` bytes goes to, given
    each device's reserved bytes and budget; -1 when none could hold it."""
    lib = _bind(load_library(lib_path))
    n = len(load)
    a = (ctypes.c_uint64 * n)(*load)
    b = (ctypes.c_uint64 * n)(*budget)
    return lib.rv9_place_least_loaded(a, b, n, need)


class Cluster:
    """A serving engine per device (rv9_cluster): each stream placed whole on
    the least loaded device by reserved bytes; one poll for all devices."""

    def __init__(self, devices, hbm_budget=120 << 30, workers=0, lib_path=None):
        self._lib = _bind(load_library(lib_path))
        arr = (ctypes.c_int * len(devices))(*devices)
        self._c = self._lib.rv9_cluster_create(arr, len(devices), hbm_budget, workers)
        if not self._c:
            raise DeviceError(self._lib.rv9_last_global_error().decode(errors="replace"))
        self.n_devices = len(devices)

    def set_device_parse(self, on=True, window=0, max_batches=0):
        """rv9_cluster_set_device_parse: every device's engine parses queued
        requests on its GPU in batches (streams opened after the call)."""
        st = self._lib.rv9_cluster_set_device_parse(self._c, 1 if on else 0, window, max_batches)
        if st != RV9_OK:
            raise _ERRORS.get(st, Rv9Error)(f"rv9_cluster_set_device_parse: status {st}")

    def open_stream(self, width, height, bit_depth=8, chroma=(1, 1)):
        """Returns (stream id, device ordinal it was placed on)."""
        s = spec(width, height, bit_depth, chroma)
        sid, dev = ctypes.c_int64(), ctypes.c_int()
        st = self._lib.rv9_cluster_stream_open(self._c, ctypes.byref(s), ctypes.byref(sid), ctypes.byref(dev))
        if st != RV9_OK:
            raise _ERRORS.get(st, Rv9Error)(f"rv9_cluster_stream_open: status {st}")
        return sid.value, dev.value

    def close_stream(self, sid):
        st = self._lib.rv9_cluster_stream_close(self._c, sid)
        if st != RV9_OK:
            raise _ERRORS.get(st, Rv9Error)(f"rv9_cluster_stream_close: status {st}")

    def submit(self, sid, packet, tag=0):
        st = self._lib.rv9_cluster_submit(self._c, sid, packet, len(packet), tag)
        if st != RV9_OK:
            raise _ERRORS.get(st, Rv9Error)(f"rv9_cluster_submit: status {st}")

    def poll(self, max_items=64, timeout_ms=0, keep_frames=True):
        arr = (CCompletion * max_items)()
        n = self._lib.rv9_cluster_poll(self._c, arr, max_items, timeout_ms)
        out = []
        for c in arr[:n]:
            frames = [Frame(c.frames[i]) for i in range(c.n_frames)] if keep_frames else []
            out.append(Completion(c, frames))
            self._lib.rv9_cluster_completion_release(self._c, ctypes.byref(c))
        return out

    def stats(self, device_index):
        s = CEngineStats()
        self._lib.rv9_cluster_get_stats(self._c, device_index, ctypes.byref(s))
        return {n: getattr(s, n) for n, _ in CEngineStats._fields_}

    def close(self):
        if getattr(self, "_c", None):
            self._lib.rv9_cluster_free(self._c)
            self._c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
