"""Small seeded streams in the shapes of the benchmark configurations, made
by the repository's stream generator (each a few frames, so that the oracle
checks them in seconds)."""
import hashlib

CASES = {
    # name: (width, height, bit_depth, chroma, frames, q, tile_cols_log2, golden_interval, noise)
    "cif_8bit_q60": (352, 288, 8, (1, 1), 6, 60, 0, 8, 8),
    "1080p_8bit_q40": (1920, 1080, 8, (1, 1), 4, 40, 2, 2, 6),
    "2160p_10bit_q30": (3840, 2160, 10, (1, 1), 3, 30, 2, 2, 24),
    "720p_12bit_444_q30": (1280, 720, 12, (0, 0), 5, 30, 2, 2, 24),
    "720p_10bit_422_q50": (1280, 720, 10, (1, 0), 4, 50, 1, 2, 12),
}

# Streams whose frames are not error-resilient: inter frames read the previous
# frame's motion vectors, and every `adapt`-th frame adapts probabilities (a
# frame the host parser keeps, between frames the device parser may take).
# name: (width, height, bit_depth, chroma, frames, q, tile_cols_log2, adapt)
LINKED = {
    "cif_8bit_linked": (352, 288, 8, (1, 1), 12, 60, 0, 4),
    "720p_8bit_linked": (1280, 720, 8, (1, 1), 9, 50, 2, 3),
    "360p_10bit_444_linked": (640, 360, 10, (0, 0), 8, 45, 0, 0),
}


def generate(name, seed=3):
    from rv9 import streams
    w, h, bd, chroma, frames, q, tcl, golden, noise = CASES[name]
    cfg = streams.config(w, h, frames, q, bit_depth=bd, chroma=chroma, tile_cols_log2=tcl, golden_interval=golden,
                         seed=seed, pan=(3, 2), rectangles=12, noise=noise)
    packets = streams.generate(cfg)
    return packets, hashlib.md5(streams.last_reconstruction()).hexdigest()


def generate_linked(name, seed=5):
    from rv9 import streams
    w, h, bd, chroma, frames, q, tcl, adapt = LINKED[name]
    cfg = streams.config(w, h, frames, q, bit_depth=bd, chroma=chroma, tile_cols_log2=tcl, golden_interval=4,
                         seed=seed, pan=(3, 2), rectangles=8, noise=8, non_resilient=1, adapt_interval=adapt)
    return streams.generate(cfg)
