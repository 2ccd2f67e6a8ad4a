"""The stream generator's binding (librv9enc.so, host CPU): seeded synthetic
VP9 streams of the benchmark shapes (include/rv9_encoder.h)."""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
ENC_LIB = os.path.join(os.path.dirname(_HERE), "_build", "librv9enc.so")


class GenConfig(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("bit_depth", ctypes.c_uint32),
                ("ss_x", ctypes.c_uint32), ("ss_y", ctypes.c_uint32), ("frames", ctypes.c_uint32),
                ("base_q_idx", ctypes.c_int32), ("tile_cols_log2", ctypes.c_uint32),
                ("golden_interval", ctypes.c_uint32), ("seed", ctypes.c_uint32), ("pan_x", ctypes.c_int32),
                ("pan_y", ctypes.c_int32), ("rectangles", ctypes.c_uint32), ("noise", ctypes.c_uint32),
                ("threads", ctypes.c_uint32), ("color_space", ctypes.c_uint32),
                ("non_resilient", ctypes.c_uint32), ("adapt_interval", ctypes.c_uint32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ENC_LIB):
            import importlib.util
            spec = importlib.util.spec_from_file_location("rv9_build", os.path.join(os.path.dirname(_HERE), "build.py"))
            m = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(m)
            m.build_encoder()
        L = ctypes.CDLL(ENC_LIB)
        L.rv9_gen_stream.argtypes = [ctypes.POINTER(GenConfig), ctypes.c_void_p, ctypes.c_size_t,
                                     ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
        L.rv9_gen_stream.restype = ctypes.c_int
        L.rv9_gen_last_reconstruction.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        L.rv9_gen_last_reconstruction.restype = ctypes.c_size_t
        L.rv9_gen_source_frame.argtypes = [ctypes.POINTER(GenConfig), ctypes.c_uint32, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def config(width, height, frames, q, bit_depth=8, chroma=(1, 1), tile_cols_log2=0, golden_interval=8, seed=0,
           pan=(2, 1), rectangles=3, noise=8, threads=0, color_space=0, non_resilient=0, adapt_interval=0):
    c = GenConfig()
    c.width, c.height, c.bit_depth = width, height, bit_depth
    c.ss_x, c.ss_y = chroma
    c.frames, c.base_q_idx, c.tile_cols_log2 = frames, q, tile_cols_log2
    c.golden_interval, c.seed = golden_interval, seed
    c.pan_x, c.pan_y = pan
    c.rectangles, c.noise, c.threads = rectangles, noise, threads
    c.color_space = color_space  # 0: BT.709
    c.non_resilient, c.adapt_interval = non_resilient, adapt_interval
    return c


def generate(cfg):
    """Encodes cfg.frames synthetic frames; returns the list of packets."""
    L = lib()
    bps = 2 if cfg.bit_depth > 8 else 1
    cap = max(1 << 20, int(cfg.width * cfg.height * 3 * bps * cfg.frames))
    buf = ctypes.create_string_buffer(cap)
    sizes = (ctypes.c_size_t * cfg.frames)()
    total = ctypes.c_size_t()
    if L.rv9_gen_stream(ctypes.byref(cfg), buf, cap, sizes, ctypes.byref(total)) != 0:
        raise ValueError("stream generation failed (invalid configuration)")
    raw = buf.raw[:total.value]
    out, pos = [], 0
    for s in sizes:
        out.append(raw[pos:pos + s])
        pos += s
    return out


def last_reconstruction():
    """The generator's reconstruction of the last frame it encoded (packed
    like a decoded frame)."""
    L = lib()
    n = L.rv9_gen_last_reconstruction(None, 0)
    buf = ctypes.create_string_buffer(n)
    L.rv9_gen_last_reconstruction(buf, n)
    return buf.raw
