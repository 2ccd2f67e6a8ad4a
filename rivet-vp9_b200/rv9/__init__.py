"""Python binding of the B200 VP9 decoder (ctypes over librv9.so).

Mirrors the reference crate's decoder API (rivet-vp9 src/decoder/mod.rs:150-216
and src/frame.rs:115-229):

    dec = rv9.Decoder()
    for packet in packets:
        frame = dec.decode(packet)        # the last frame the packet shows, or None
        frames = dec.decode_all(packet)   # every frame it shows

Errors are raised as the reference's error kinds: BitstreamError,
UnsupportedError, InvalidInputError; device failures as DeviceError.
The library runs reconstruction on the GPU only: importing works anywhere,
but Decoder() raises DeviceError when librv9.so or a usable CUDA device is
missing.
"""
import ctypes
import os

from . import containers  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "_build", "librv9.so")

RV9_OK, RV9_BITSTREAM, RV9_UNSUPPORTED, RV9_INVALID_INPUT, RV9_DEVICE = range(5)
CHROMA_NAMES = {0: "Yuv420", 1: "Yuv422", 2: "Yuv440", 3: "Yuv444"}


class Rv9Error(Exception):
    pass


class BitstreamError(Rv9Error):
    pass


class UnsupportedError(Rv9Error):
    pass


class InvalidInputError(Rv9Error):
    pass


class DeviceError(Rv9Error):
    pass


_ERRORS = {RV9_BITSTREAM: BitstreamError, RV9_UNSUPPORTED: UnsupportedError,
           RV9_INVALID_INPUT: InvalidInputError, RV9_DEVICE: DeviceError}


class CPlane(ctypes.Structure):
    _fields_ = [("offset", ctypes.c_size_t), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32)]


class CFrame(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("bit_depth", ctypes.c_uint32),
                ("chroma", ctypes.c_uint32), ("color_space", ctypes.c_uint32), ("full_range", ctypes.c_uint32),
                ("render_width", ctypes.c_uint32), ("render_height", ctypes.c_uint32),
                ("data", ctypes.POINTER(ctypes.c_uint8)), ("size", ctypes.c_size_t), ("planes", CPlane * 3)]


class CStats(ctypes.Structure):
    _fields_ = [("device_ms", ctypes.c_double), ("parse_ms", ctypes.c_double), ("frames", ctypes.c_uint64),
                ("algorithmic_bytes", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint64)]


# Every symbol include/rv9.h declares.
EXPORTS = ("rv9_decoder_new", "rv9_decoder_free", "rv9_decoder_set_threads", "rv9_decoder_set_parse_depth", "rv9_decoder_set_max_pixels",
           "rv9_decoder_frames_decoded", "rv9_last_error", "rv9_last_global_error", "rv9_decode_all",
           "rv9_decode", "rv9_frame_release", "rv9_decode_packets", "rv9_decoder_stats", "rv9_sequence_load",
           "rv9_sequence_run", "rv9_sequence_frames", "rv9_sequence_luma_samples", "rv9_sequence_algorithmic_bytes",
           "rv9_sequence_record_bytes", "rv9_sequence_free", "rv9_sequence_clone", "rv9_decoder_download_slot", "rv9_kernel_stats",
           "rv9_sequence_run_noalloc", "rv9_sequences_run", "rv9_sequences_run_batched", "rv9_sequences_autotune_batched", "rv9_decoder_autotune",
           "rv9_sequences_autotune", "rv9_decoder_set_event_mask", "rv9_decoder_threads", "rv9_decoder_set_wait_limit",
           "rv9_decoder_set_test_fault", "rv9_decoder_set_frame_sink", "rv9_decoder_frame_sink_state",
           "rv9_decoder_set_frame_digests", "rv9_decoder_frame_digests", "rv9_decoder_set_device_parse",
           "rv9_decoder_device_parse_stats")


class CTuneResult(ctypes.Structure):
    _fields_ = [("intra_ctas_per_sm_x4", ctypes.c_int32), ("inter_threads", ctypes.c_int32),
                ("best_ms", ctypes.c_double), ("default_ms", ctypes.c_double), ("inter_fork", ctypes.c_int32)]


class CKernelStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 24), ("launches", ctypes.c_uint64), ("ms", ctypes.c_double),
                ("algorithmic_bytes", ctypes.c_uint64)]

_lib = None


def load_library(path=None):
    """Loads librv9.so (the CUDA build); raises DeviceError if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise DeviceError(f"{p} is not built: run rivet-vp9_b200/build.py (the decoder has no CPU path)")
    lib = ctypes.CDLL(p)
    vp = ctypes.c_void_p
    lib.rv9_decoder_new.restype = vp
    lib.rv9_decoder_new.argtypes = [ctypes.c_int]
    lib.rv9_decoder_free.argtypes = [vp]
    lib.rv9_decoder_set_threads.argtypes = [vp, ctypes.c_uint32]
    lib.rv9_decoder_set_parse_depth.argtypes = [vp, ctypes.c_uint32]
    lib.rv9_decoder_set_max_pixels.argtypes = [vp, ctypes.c_uint64]
    lib.rv9_decoder_set_device_parse.restype = ctypes.c_int
    lib.rv9_decoder_set_device_parse.argtypes = [vp, ctypes.c_int, ctypes.c_uint32]
    lib.rv9_decoder_device_parse_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64),
                                                   ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_double)]
    lib.rv9_decoder_frames_decoded.restype = ctypes.c_uint64
    lib.rv9_decoder_frames_decoded.argtypes = [vp]
    lib.rv9_last_error.restype = ctypes.c_char_p
    lib.rv9_last_error.argtypes = [vp]
    lib.rv9_last_global_error.restype = ctypes.c_char_p
    lib.rv9_decode_all.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(CFrame), ctypes.c_size_t,
                                   ctypes.POINTER(ctypes.c_size_t)]
    lib.rv9_decode.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(CFrame),
                               ctypes.POINTER(ctypes.c_int)]
    lib.rv9_frame_release.argtypes = [ctypes.POINTER(CFrame)]
    lib.rv9_decode_packets.argtypes = [vp, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t),
                                       ctypes.c_size_t, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t),
                                       ctypes.POINTER(ctypes.c_size_t)]
    lib.rv9_decoder_stats.argtypes = [vp, ctypes.POINTER(CStats), ctypes.c_int]
    lib.rv9_sequence_load.argtypes = [vp, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t),
                                      ctypes.c_size_t, ctypes.POINTER(vp)]
    lib.rv9_sequence_run.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.rv9_sequence_run_noalloc.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_double)]
    lib.rv9_decoder_autotune.argtypes = [vp, vp, ctypes.POINTER(CTuneResult)]
    lib.rv9_sequences_autotune.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_size_t,
                                           ctypes.POINTER(CTuneResult)]
    lib.rv9_sequences_run.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_size_t, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_double)]
    lib.rv9_sequences_run_batched.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_size_t,
                                              ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.rv9_sequences_autotune_batched.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_size_t,
                                                   ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(CTuneResult)]
    for name in ("rv9_sequence_luma_samples", "rv9_sequence_algorithmic_bytes", "rv9_sequence_record_bytes"):
        getattr(lib, name).restype = ctypes.c_uint64
        getattr(lib, name).argtypes = [vp]
    lib.rv9_sequence_frames.restype = ctypes.c_uint32
    lib.rv9_sequence_frames.argtypes = [vp]
    lib.rv9_sequence_free.argtypes = [vp, vp]
    lib.rv9_sequence_clone.argtypes = [vp, vp, ctypes.POINTER(vp)]
    lib.rv9_decoder_download_slot.argtypes = [vp, ctypes.c_int, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    lib.rv9_decoder_set_event_mask.argtypes = [vp, ctypes.c_uint32]
    lib.rv9_decoder_set_frame_sink.argtypes = [vp, vp, ctypes.c_size_t]
    lib.rv9_decoder_frame_sink_state.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_size_t),
                                                 ctypes.POINTER(ctypes.c_uint64)]
    lib.rv9_decoder_set_frame_digests.argtypes = [vp, ctypes.c_size_t]
    lib.rv9_decoder_frame_digests.restype = ctypes.c_size_t
    lib.rv9_decoder_frame_digests.argtypes = [vp, vp, ctypes.c_size_t]
    lib.rv9_decoder_threads.restype = ctypes.c_uint32
    lib.rv9_decoder_threads.argtypes = [vp]
    lib.rv9_decoder_set_wait_limit.argtypes = [vp, ctypes.c_uint32]
    lib.rv9_decoder_set_test_fault.argtypes = [vp, ctypes.c_uint32]
    lib.rv9_kernel_stats.restype = ctypes.c_size_t
    lib.rv9_kernel_stats.argtypes = [vp, ctypes.POINTER(CKernelStat), ctypes.c_size_t, ctypes.c_int]
    if path is None:
        _lib = lib
    return lib


class Sequence:
    """Parsed frames whose records are resident in device memory."""

    def __init__(self, dec, handle):
        self._dec, self._h = dec, handle
        L = dec._lib
        self.frames = L.rv9_sequence_frames(handle)
        self.luma_samples = L.rv9_sequence_luma_samples(handle)
        self.algorithmic_bytes = L.rv9_sequence_algorithmic_bytes(handle)
        self.record_bytes = L.rv9_sequence_record_bytes(handle)

    def run(self, per_kernel=False, graph=False):
        """Reconstructs every frame on the device; returns the CUDA-event
        milliseconds of the run. `graph`: replay a CUDA graph of the run
        (captured on first use)."""
        ms = ctypes.c_double()
        flags = (RV9_RUN_PER_KERNEL if per_kernel else 0) | (RV9_RUN_GRAPH if graph else 0)
        st = self._dec._lib.rv9_sequence_run(self._dec._dec, self._h, flags, ctypes.byref(ms))
        if st != RV9_OK:
            _raise(self._dec._lib, self._dec._dec, st)
        return ms.value

    def run_noalloc(self):
        """run() without allocating device memory (rv9_sequence_run_noalloc):
        the wavefront scratch is a fixed 1 MiB static device array shared by
        every such call on the device (overlapping calls race), and the frame
        buffers come from the decoder's pool, which an earlier run() of this
        sequence fills. Raises InvalidInputError when either does not suffice."""
        ms = ctypes.c_double()
        st = self._dec._lib.rv9_sequence_run_noalloc(self._dec._dec, self._h, ctypes.byref(ms))
        if st != RV9_OK:
            _raise(self._dec._lib, self._dec._dec, st)
        return ms.value

    def free(self):
        if self._h:
            self._dec._lib.rv9_sequence_free(self._dec._dec, self._h)
            self._h = None


DEVICE_PARSE_SHARED = 2  # rv9_decoder_set_device_parse: host and device share a batch
RV9_RUN_PER_KERNEL = 1
RV9_RUN_GRAPH = 2


def autotune_concurrent(pairs):
    """Picks one launch shape for (decoder, sequence) pairs reconstructed
    together (rv9_sequences_autotune); returns the choice and the batch's
    times."""
    if not pairs:
        return None
    lib = pairs[0][0]._lib
    n = len(pairs)
    decs = (ctypes.c_void_p * n)(*[d._dec for d, _ in pairs])
    seqs = (ctypes.c_void_p * n)(*[s._h for _, s in pairs])
    r = CTuneResult()
    st = lib.rv9_sequences_autotune(decs, seqs, n, ctypes.byref(r))
    if st != RV9_OK:
        _raise(lib, pairs[0][0]._dec, st)
    return {"intra_ctas_per_sm_x4": r.intra_ctas_per_sm_x4, "inter_threads": r.inter_threads,
            "inter_fork": bool(r.inter_fork), "best_ms": r.best_ms, "default_ms": r.default_ms}


def run_concurrent(pairs, per_kernel=False, graph=False):
    """Reconstructs several (decoder, sequence) pairs at once, each decoder on
    its own CUDA stream (rv9_sequences_run); returns the CUDA-event
    milliseconds from the common start to the last stream's end."""
    if not pairs:
        return 0.0
    lib = pairs[0][0]._lib
    n = len(pairs)
    decs = (ctypes.c_void_p * n)(*[d._dec for d, _ in pairs])
    seqs = (ctypes.c_void_p * n)(*[s._h for _, s in pairs])
    ms = ctypes.c_double()
    flags = (RV9_RUN_PER_KERNEL if per_kernel else 0) | (RV9_RUN_GRAPH if graph else 0)
    st = lib.rv9_sequences_run(decs, seqs, n, flags, ctypes.byref(ms))
    if st != RV9_OK:
        _raise(lib, pairs[0][0]._dec, st)
    return ms.value


def run_batched(pairs, groups=1):
    """Reconstructs several (decoder, sequence) pairs with one launch per stage
    for all sequences' next frames (rv9_sequences_run_batched), the decoders
    split into `groups` groups on their own CUDA streams; returns the
    CUDA-event milliseconds of the run."""
    if not pairs:
        return 0.0
    lib = pairs[0][0]._lib
    n = len(pairs)
    decs = (ctypes.c_void_p * n)(*[d._dec for d, _ in pairs])
    seqs = (ctypes.c_void_p * n)(*[s._h for _, s in pairs])
    ms = ctypes.c_double()
    st = lib.rv9_sequences_run_batched(decs, seqs, n, int(groups), ctypes.byref(ms))
    if st != RV9_OK:
        _raise(lib, pairs[0][0]._dec, st)
    return ms.value


def autotune_batched(pairs):
    """The autotuner for run_batched (rv9_sequences_autotune_batched): the
    fastest number of groups and intra grain for these pairs; the grain is
    kept on the first decoder."""
    lib = pairs[0][0]._lib
    n = len(pairs)
    decs = (ctypes.c_void_p * n)(*[d._dec for d, _ in pairs])
    seqs = (ctypes.c_void_p * n)(*[s._h for _, s in pairs])
    groups = ctypes.c_int32()
    r = CTuneResult()
    st = lib.rv9_sequences_autotune_batched(decs, seqs, n, ctypes.byref(groups), ctypes.byref(r))
    if st != RV9_OK:
        _raise(lib, pairs[0][0]._dec, st)
    return {"groups": groups.value, "intra_ctas_per_sm_x4": r.intra_ctas_per_sm_x4, "best_ms": r.best_ms,
            "default_ms": r.default_ms}


class Plane:
    __slots__ = ("offset", "width", "height")

    def __init__(self, offset, width, height):
        self.offset, self.width, self.height = offset, width, height


class Frame:
    """A decoded frame in the reference's layout: Y, U, V packed (stride ==
    width), one byte per sample at 8 bits, little-endian uint16 above."""

    def __init__(self, c: CFrame):
        self.width, self.height, self.bit_depth = c.width, c.height, c.bit_depth
        self.chroma = CHROMA_NAMES.get(c.chroma, str(c.chroma))
        self.color_space, self.full_range = c.color_space, bool(c.full_range)
        self.render_width, self.render_height = c.render_width, c.render_height
        self.data = ctypes.string_at(c.data, c.size) if c.size else b""
        self.planes = [Plane(p.offset, p.width, p.height) for p in c.planes]

    def bytes_per_sample(self):
        return 2 if self.bit_depth > 8 else 1

    def plane(self, i):
        p = self.planes[i]
        n = p.width * p.height * self.bytes_per_sample()
        return self.data[p.offset:p.offset + n]

    def packed(self):
        return self.data


def _raise(lib, dec, st):
    msg = lib.rv9_last_error(dec).decode(errors="replace") if dec else ""
    raise _ERRORS.get(st, Rv9Error)(msg or f"status {st}")


class Decoder:
    """A VP9 decoder whose reconstruction runs on CUDA device `device`."""

    def __init__(self, device=-1, lib_path=None):
        self._lib = load_library(lib_path)
        self._dec = self._lib.rv9_decoder_new(device)
        if not self._dec:
            raise DeviceError(self._lib.rv9_last_global_error().decode(errors="replace"))

    def close(self):
        if getattr(self, "_dec", None):
            self._lib.rv9_decoder_free(self._dec)
            self._dec = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_threads(self, n):
        self._lib.rv9_decoder_set_threads(self._dec, n)

    def set_parse_depth(self, frames):
        """Frames parsed at once by decode_packets / load_sequence (0: auto)."""
        self._lib.rv9_decoder_set_parse_depth(self._dec, frames)

    def threads(self):
        """Host threads parsing uses (Decoder::threads)."""
        return self._lib.rv9_decoder_threads(self._dec)

    def set_max_pixels(self, n):
        self._lib.rv9_decoder_set_max_pixels(self._dec, n)

    def set_device_parse(self, on=True, window_frames=0):
        """Parse tiles on the GPU where the frames allow it (rv9_decoder_set_device_parse):
        decode_packets and load_sequence then take that path; results are identical.
        on=DEVICE_PARSE_SHARED splits batches of independent frames between the host's
        threads and the device."""
        mode = on if (isinstance(on, int) and not isinstance(on, bool)) else (1 if on else 0)
        st = self._lib.rv9_decoder_set_device_parse(self._dec, mode, window_frames)
        if st != 0:
            _raise(self._lib, self._dec, st)

    def device_parse_stats(self):
        """(frames the device parser took, its boolean decodes, its device milliseconds)."""
        f, b, ms = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_double(0)
        self._lib.rv9_decoder_device_parse_stats(self._dec, ctypes.byref(f), ctypes.byref(b), ctypes.byref(ms))
        return f.value, b.value, ms.value

    def set_wait_limit(self, polls):
        """Polls before a device-side wavefront wait gives up (0: default)."""
        self._lib.rv9_decoder_set_wait_limit(self._dec, polls)

    def set_test_fault(self, mask):
        """Failure injection for tests (rv9_decoder_set_test_fault): bit 0
        leaves each frame's first intra job untaken, bit 1 its first
        loop-filter row; 0 turns it off."""
        self._lib.rv9_decoder_set_test_fault(self._dec, mask)

    def frames_decoded(self):
        return self._lib.rv9_decoder_frames_decoded(self._dec)

    def decode_all(self, packet: bytes):
        cap = 16
        frames = (CFrame * cap)()
        n = ctypes.c_size_t()
        st = self._lib.rv9_decode_all(self._dec, packet, len(packet), frames, cap, ctypes.byref(n))
        if st != RV9_OK:
            _raise(self._lib, self._dec, st)
        out = []
        for i in range(min(n.value, cap)):
            out.append(Frame(frames[i]))
            self._lib.rv9_frame_release(ctypes.byref(frames[i]))
        return out

    def decode(self, packet: bytes):
        frames = self.decode_all(packet)
        return frames[-1] if frames else None

    def decode_packets(self, packets, out_buffer, out_ptr=None):
        """Decodes a sequence of packets with parsing overlapped with the
        device work; shown frames are written packed into `out_buffer` (a
        writable buffer, e.g. pinned memory). Returns (frames, bytes)."""
        n = len(packets)
        arr = (ctypes.c_char_p * n)(*packets)
        lens = (ctypes.c_size_t * n)(*[len(p) for p in packets])
        nf, nb = ctypes.c_size_t(), ctypes.c_size_t()
        if out_ptr is None:
            out_ptr = ctypes.addressof((ctypes.c_char * len(out_buffer)).from_buffer(out_buffer))
        st = self._lib.rv9_decode_packets(self._dec, arr, lens, n, out_ptr, len(out_buffer),
                                          ctypes.byref(nf), ctypes.byref(nb))
        if st != RV9_OK:
            _raise(self._lib, self._dec, st)
        return nf.value, nb.value

    def decode_packets_to(self, packets, out_ptr, cap):
        """decode_packets into `cap` bytes of memory at address `out_ptr`
        (e.g. pinned host memory). Returns (frames, bytes)."""
        n = len(packets)
        arr = (ctypes.c_char_p * n)(*packets)
        lens = (ctypes.c_size_t * n)(*[len(p) for p in packets])
        nf, nb = ctypes.c_size_t(), ctypes.c_size_t()
        st = self._lib.rv9_decode_packets(self._dec, arr, lens, n, out_ptr, cap, ctypes.byref(nf), ctypes.byref(nb))
        if st != RV9_OK:
            _raise(self._lib, self._dec, st)
        return nf.value, nb.value

    def load_sequence(self, packets):
        """Parses `packets` (one stream from its start) and keeps their records
        in device memory for run_sequence."""
        n = len(packets)
        arr = (ctypes.c_char_p * n)(*packets)
        lens = (ctypes.c_size_t * n)(*[len(p) for p in packets])
        seq = ctypes.c_void_p()
        st = self._lib.rv9_sequence_load(self._dec, arr, lens, n, ctypes.byref(seq))
        if st != RV9_OK:
            _raise(self._lib, self._dec, st)
        return Sequence(self, seq)

    def clone_sequence(self, seq):
        """A copy of `seq` (any decoder's, same device) held by this decoder."""
        out = ctypes.c_void_p()
        st = self._lib.rv9_sequence_clone(self._dec, seq._h, ctypes.byref(out))
        if st != RV9_OK:
            _raise(self._lib, self._dec, st)
        return Sequence(self, out)

    def autotune(self, seq):
        """Picks this decoder's launch shapes for the geometry of `seq`'s
        frames (rv9_decoder_autotune); returns the choice and the times."""
        r = CTuneResult()
        st = self._lib.rv9_decoder_autotune(self._dec, seq._h, ctypes.byref(r))
        if st != RV9_OK:
            _raise(self._lib, self._dec, st)
        return {"intra_ctas_per_sm_x4": r.intra_ctas_per_sm_x4, "inter_threads": r.inter_threads,
                "inter_fork": bool(r.inter_fork), "best_ms": r.best_ms, "default_ms": r.default_ms}

    def download_slot(self, slot, cap):
        buf = ctypes.create_string_buffer(cap)
        n = ctypes.c_size_t()
        st = self._lib.rv9_decoder_download_slot(self._dec, slot, buf, cap, ctypes.byref(n))
        if st != RV9_OK:
            _raise(self._lib, self._dec, st)
        return buf.raw[:n.value]

    def set_frame_sink(self, ptr, cap):
        """Every frame shown from now on is copied, packed, to `cap` bytes at
        address `ptr` (host or device memory); ptr 0 turns the sink off."""
        self._lib.rv9_decoder_set_frame_sink(self._dec, ptr or None, cap if ptr else 0)

    def set_frame_digests(self, cap_frames):
        """On-device MD5 of every frame shown from now on (up to cap_frames;
        0 turns it off)."""
        st = self._lib.rv9_decoder_set_frame_digests(self._dec, cap_frames)
        if st != RV9_OK:
            _raise(self._lib, self._dec, st)

    def frame_digests(self, cap=1 << 16):
        """The hex MD5s computed on the device so far, in show order."""
        buf = ctypes.create_string_buffer(16 * cap)
        n = self._lib.rv9_decoder_frame_digests(self._dec, buf, cap)
        return [buf.raw[16 * i:16 * i + 16].hex() for i in range(min(n, cap))]

    def frame_sink_state(self):
        """(frames, bytes, dropped) of the frame sink."""
        f, b, d = ctypes.c_uint64(), ctypes.c_size_t(), ctypes.c_uint64()
        self._lib.rv9_decoder_frame_sink_state(self._dec, ctypes.byref(f), ctypes.byref(b), ctypes.byref(d))
        return f.value, b.value, d.value

    def set_event_mask(self, names=None):
        """Kernels that per_kernel runs bracket with events (None: all)."""
        if names is None:
            mask = 0xFFFFFFFF
        else:
            order = list(self.kernel_stats().keys())
            mask = 0
            for n in names:
                mask |= 1 << order.index(n)
        self._lib.rv9_decoder_set_event_mask(self._dec, mask)

    def kernel_stats(self, reset=False):
        arr = (CKernelStat * 16)()
        n = self._lib.rv9_kernel_stats(self._dec, arr, 16, 1 if reset else 0)
        return {a.name.decode(): {"launches": a.launches, "ms": a.ms, "algorithmic_bytes": a.algorithmic_bytes}
                for a in arr[:min(n, 16)]}

    def stats(self, reset=False):
        s = CStats()
        self._lib.rv9_decoder_stats(self._dec, ctypes.byref(s), 1 if reset else 0)
        return {"device_ms": s.device_ms, "parse_ms": s.parse_ms, "frames": s.frames,
                "algorithmic_bytes": s.algorithmic_bytes, "kernel_launches": s.kernel_launches}
