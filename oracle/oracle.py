"""ORACLE — test infrastructure only (the checker, never the product).

ctypes binding of oracle/_build/liboracle.so: the CPU restatement of the
reference decoder's reconstruction (see oracle.cpp) behind the same decoder
API as the product (rv9o_* for rv9_*). Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline / reference legs use it.
"""
import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")


class CPlane(ctypes.Structure):
    _fields_ = [("offset", ctypes.c_size_t), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32)]


class CFrame(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("bit_depth", ctypes.c_uint32),
                ("chroma", ctypes.c_uint32), ("color_space", ctypes.c_uint32), ("full_range", ctypes.c_uint32),
                ("render_width", ctypes.c_uint32), ("render_height", ctypes.c_uint32),
                ("data", ctypes.POINTER(ctypes.c_uint8)), ("size", ctypes.c_size_t), ("planes", CPlane * 3)]


def build():
    """Builds liboracle.so with its Makefile (g++, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        L.rv9o_decoder_new.restype = vp
        L.rv9o_decoder_free.argtypes = [vp]
        L.rv9o_decoder_set_threads.argtypes = [vp, ctypes.c_uint32]
        L.rv9o_decoder_set_max_pixels.argtypes = [vp, ctypes.c_uint64]
        L.rv9o_decoder_frames_decoded.restype = ctypes.c_uint64
        L.rv9o_decoder_frames_decoded.argtypes = [vp]
        L.rv9o_last_error.restype = ctypes.c_char_p
        L.rv9o_last_error.argtypes = [vp]
        L.rv9o_recon_seconds.restype = ctypes.c_double
        L.rv9o_recon_seconds.argtypes = [vp]
        L.rv9o_decode_all.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(CFrame), ctypes.c_size_t,
                                      ctypes.POINTER(ctypes.c_size_t)]
        L.rv9o_frame_release.argtypes = [ctypes.POINTER(CFrame)]
        L.rv9o_decode_packets.argtypes = [vp, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t),
                                          ctypes.c_size_t, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t),
                                          ctypes.POINTER(ctypes.c_size_t)]
        for name in ("rv9o_test_itx", "rv9o_test_intra", "rv9o_test_lf"):
            getattr(L, name).restype = None
        _lib = L
    return _lib


class OracleError(Exception):
    def __init__(self, status, msg):
        super().__init__(f"status {status}: {msg}")
        self.status = status


class OracleFrame:
    def __init__(self, c):
        self.width, self.height, self.bit_depth = c.width, c.height, c.bit_depth
        self.chroma = c.chroma
        self.data = ctypes.string_at(c.data, c.size) if c.size else b""
        self.planes = [(p.offset, p.width, p.height) for p in c.planes]

    def packed(self):
        return self.data


class OracleDecoder:
    def __init__(self, threads=1):
        self._L = lib()
        self._d = self._L.rv9o_decoder_new()
        self._L.rv9o_decoder_set_threads(self._d, threads)

    def __del__(self):
        try:
            self._L.rv9o_decoder_free(self._d)
        except Exception:
            pass

    def set_max_pixels(self, pixels):
        self._L.rv9o_decoder_set_max_pixels(self._d, pixels)

    def decode_all(self, packet):
        cap = 16
        frames = (CFrame * cap)()
        n = ctypes.c_size_t()
        st = self._L.rv9o_decode_all(self._d, packet, len(packet), frames, cap, ctypes.byref(n))
        if st != 0:
            raise OracleError(st, self._L.rv9o_last_error(self._d).decode(errors="replace"))
        out = []
        for i in range(min(n.value, cap)):
            out.append(OracleFrame(frames[i]))
            self._L.rv9o_frame_release(ctypes.byref(frames[i]))
        return out

    def decode_packets(self, packets, out_buffer):
        n = len(packets)
        arr = (ctypes.c_char_p * n)(*packets)
        lens = (ctypes.c_size_t * n)(*[len(p) for p in packets])
        nf, nb = ctypes.c_size_t(), ctypes.c_size_t()
        ptr = ctypes.addressof((ctypes.c_char * len(out_buffer)).from_buffer(out_buffer))
        st = self._L.rv9o_decode_packets(self._d, arr, lens, n, ptr, len(out_buffer), ctypes.byref(nf),
                                         ctypes.byref(nb))
        if st != 0:
            raise OracleError(st, self._L.rv9o_last_error(self._d).decode(errors="replace"))
        return nf.value, nb.value

    def recon_seconds(self):
        return self._L.rv9o_recon_seconds(self._d)
