"""ctypes mirrors of include/rv9_records.h for the tests."""
import ctypes


class Segmentation(ctypes.Structure):
    _fields_ = [("enabled", ctypes.c_uint8), ("update_map", ctypes.c_uint8), ("temporal_update", ctypes.c_uint8),
                ("abs_or_delta_update", ctypes.c_uint8), ("feature_enabled", (ctypes.c_uint8 * 4) * 8),
                ("feature_data", (ctypes.c_int16 * 4) * 8)]


class FrameDesc(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("mi_cols", ctypes.c_uint32),
                ("mi_rows", ctypes.c_uint32), ("sb64_cols", ctypes.c_uint32), ("sb64_rows", ctypes.c_uint32),
                ("ss_x", ctypes.c_uint8), ("ss_y", ctypes.c_uint8), ("bit_depth", ctypes.c_uint8),
                ("lossless", ctypes.c_uint8), ("legacy_uv", ctypes.c_uint8), ("frame_is_intra", ctypes.c_uint8),
                ("show_frame", ctypes.c_uint8), ("tile_cols_log2", ctypes.c_uint8), ("base_q_idx", ctypes.c_int32),
                ("delta_q_y_dc", ctypes.c_int32), ("delta_q_uv_dc", ctypes.c_int32), ("delta_q_uv_ac", ctypes.c_int32),
                ("lf_level", ctypes.c_uint8), ("lf_sharpness", ctypes.c_uint8), ("lf_delta_enabled", ctypes.c_uint8),
                ("reserved1", ctypes.c_uint8), ("lf_ref_deltas", ctypes.c_int8 * 4), ("lf_mode_deltas", ctypes.c_int8 * 2),
                ("reserved2", ctypes.c_uint8 * 2), ("seg", Segmentation), ("ref_width", ctypes.c_uint32 * 3),
                ("ref_height", ctypes.c_uint32 * 3), ("color_space", ctypes.c_uint8), ("color_range", ctypes.c_uint8),
                ("reserved3", ctypes.c_uint8 * 2), ("render_width", ctypes.c_uint32), ("render_height", ctypes.c_uint32)]


class Block(ctypes.Structure):
    _fields_ = [("mi_row", ctypes.c_uint16), ("mi_col", ctypes.c_uint16), ("mi_size", ctypes.c_uint8),
                ("flags", ctypes.c_uint8), ("tx_size", ctypes.c_uint8), ("segment_id", ctypes.c_uint8),
                ("y_mode", ctypes.c_uint8), ("uv_mode", ctypes.c_uint8), ("interp_filter", ctypes.c_uint8),
                ("coded_skip", ctypes.c_uint8), ("sub_modes", ctypes.c_uint8 * 4), ("ref_frame", ctypes.c_int8 * 2),
                ("n_tok", ctypes.c_uint16), ("tok_start", ctypes.c_uint32), ("mv", ((ctypes.c_int32 * 2) * 4) * 2)]


SS_SIZE = [[[0, 14], [14, 14]], [[1, 0], [14, 14]], [[2, 14], [0, 14]], [[3, 2], [1, 0]], [[4, 3], [14, 1]],
           [[5, 14], [3, 2]], [[6, 5], [4, 3]], [[7, 6], [14, 4]], [[8, 14], [6, 5]], [[9, 8], [7, 6]],
           [[10, 9], [14, 7]], [[11, 14], [9, 8]], [[12, 11], [10, 9]]]
MAX_TX = [0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3, 3]
N8W = [1, 1, 1, 1, 1, 2, 2, 2, 4, 4, 4, 8, 8]
N8H = [1, 1, 1, 1, 2, 1, 2, 4, 2, 4, 8, 4, 8]
SUBSIZE = [[0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12],
           [14, 14, 14, 2, 14, 14, 5, 14, 14, 8, 14, 14, 11],
           [14, 14, 14, 1, 14, 14, 4, 14, 14, 7, 14, 14, 10],
           [14, 14, 14, 0, 14, 14, 3, 14, 14, 6, 14, 14, 9]]


def random_blocks(rng, mi_rows, mi_cols, ss_x, ss_y):
    """A random partition of the frame into blocks (the partition syntax's
    shapes), each with random mode info."""
    out = []

    def valid(size):
        return size < 3 or SS_SIZE[size][ss_x][ss_y] != 14

    def block(r, c, size):
        if r >= mi_rows or c >= mi_cols:
            return
        b = Block()
        b.mi_row, b.mi_col, b.mi_size = r, c, size
        b.tx_size = int(rng.integers(0, MAX_TX[size] + 1))
        rf = int(rng.integers(0, 4))
        b.ref_frame[0], b.ref_frame[1] = rf, -1
        b.y_mode = int(rng.integers(0, 10)) if rf == 0 else int(rng.integers(10, 14))
        skip = int(rng.random() < 0.4)
        b.flags = skip | (2 if rf > 0 else 0)
        b.segment_id = int(rng.integers(0, 8))
        out.append(b)

    def part(r, c, bsize):
        if r >= mi_rows or c >= mi_cols:
            return
        half = N8W[bsize] >> 1
        choices = [p for p in range(4) if SUBSIZE[p][bsize] != 14 and valid(SUBSIZE[p][bsize])]
        p = int(rng.choice(choices))
        sub = SUBSIZE[p][bsize]
        if sub < 3 or p == 0:
            block(r, c, sub)
        elif p == 1:
            block(r, c, sub)
            block(r + half, c, sub)
        elif p == 2:
            block(r, c, sub)
            block(r, c + half, sub)
        else:
            for dr, dc in ((0, 0), (0, half), (half, 0), (half, half)):
                part(r + dr, c + dc, sub)

    for r in range(0, mi_rows, 8):
        for c in range(0, mi_cols, 8):
            part(r, c, 12)
    return out
