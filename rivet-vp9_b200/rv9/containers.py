"""Container readers for VP9 packets: IVF and a minimal WebM (Matroska) walk.

IVF follows rivet-vp9's reader (src/ivf.rs:42-100): a 32-byte file header
(header length at byte 6), then per frame a 12-byte header (little-endian
size, 64-bit timestamp). The WebM walk follows the reference's test support
(tests/common/mod.rs:12-75): descend Segment, Cluster and BlockGroup, take
the payload of every SimpleBlock and Block of the first track (no lacing),
stop at an element that overruns its parent.
"""
import struct


def ivf_packets(data: bytes):
    if len(data) < 32 or data[:4] != b"DKIF":
        raise ValueError("not an IVF file")
    header_len = struct.unpack_from("<H", data, 6)[0]
    pos = max(header_len, 32)
    out = []
    while pos + 12 <= len(data):
        size = struct.unpack_from("<I", data, pos)[0]
        if pos + 12 + size > len(data):
            raise ValueError("IVF frame runs past the end of the file")
        out.append(bytes(data[pos + 12: pos + 12 + size]))
        pos += 12 + size
    return out


def ivf_header(data: bytes):
    """(fourcc, width, height, rate, scale, frames) of an IVF file."""
    fourcc = bytes(data[8:12])
    w, h, rate, scale, frames = struct.unpack_from("<HHIII", data, 12)
    return fourcc, w, h, rate, scale, frames


def ivf_write(packets, width, height, rate=30, scale=1) -> bytes:
    out = bytearray(b"DKIF")
    out += struct.pack("<HH4sHHIII", 0, 32, b"VP90", width, height, rate, scale, len(packets))
    out += b"\0" * 4
    for i, p in enumerate(packets):
        out += struct.pack("<IQ", len(p), i)
        out += p
    return bytes(out)


def _vint(data, pos, keep_marker):
    if pos >= len(data):
        return None
    first = data[pos]
    if first == 0:
        return None
    length = 8 - first.bit_length() + 1
    if length > 8 or pos + length > len(data):
        return None
    v = first if keep_marker else first & ((1 << (8 - length)) - 1)
    for i in range(1, length):
        v = (v << 8) | data[pos + i]
    return v, length


def _walk(data, out, track):
    pos = 0
    while pos < len(data):
        r = _vint(data, pos, True)
        if r is None:
            return
        eid, il = r
        r = _vint(data, pos + il, False)
        if r is None:
            return
        size, sl = r
        start = pos + il + sl
        unknown = size == (1 << (7 * sl)) - 1
        if not unknown and start + size > len(data):
            return
        end = len(data) if unknown else start + size
        if eid in (0x18538067, 0x1F43B675, 0xA0):
            _walk(data[start:end], out, track)
        elif eid in (0xA3, 0xA1):
            b = data[start:end]
            r = _vint(b, 0, False)
            if r is not None:
                tn, tl = r
                if track[0] is None:
                    track[0] = tn
                if tn == track[0] and len(b) >= tl + 3:
                    out.append(bytes(b[tl + 3:]))
        pos = end


def webm_packets(data: bytes):
    out = []
    _walk(memoryview(data).tobytes(), out, [None])
    return out


def packets(data: bytes):
    """Packets of a file by content: IVF if it starts with DKIF, else WebM."""
    if data[:4] == b"DKIF":
        return ivf_packets(data)
    return webm_packets(data)
