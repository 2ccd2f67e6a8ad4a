"""The multi-device front end (rv9_cluster) on the GPU: with one GPU here,
two engines on device 0 stand in for two devices, so that placement spreads
the streams over both by reserved bytes; every stream's frames must be its
published MD5s whichever engine decoded it, with host parsing and with
device parsing (rv9_cluster_set_device_parse)."""
import hashlib
import os

import pytest

from conftest import VECTORS_DIR, expected_md5s, read_packets

pytestmark = pytest.mark.gpu

NAMES = ["vp90-2-02-size-130x132.webm", "vp90-2-05-resize.ivf", "vp91-2-04-yuv444.webm",
         "vp92-2-20-10bit-yuv420.webm", "vp90-2-10-show-existing-frame2.webm", "vp90-2-03-size-226x226.webm"]


@pytest.mark.parametrize("device_parse", [False, True], ids=["host_parse", "device_parse"])
def test_cluster_places_and_decodes_exactly(device_parse):
    from rv9 import server
    # Room for three streams per engine (with device parsing a stream also
    # reserves its batch's device records).
    cl = server.Cluster([0, 0], hbm_budget=(24 if device_parse else 8) << 30, workers=4)
    try:
        if device_parse:
            cl.set_device_parse(True, window=4)
        sids, placed, want = [], [], {}
        for n in NAMES:
            path = os.path.join(VECTORS_DIR, n)
            sid, dev = cl.open_stream(4096, 2176, bit_depth=12 if "12bit" in n else 10, chroma=(0, 0))
            assert dev == 0
            sids.append(sid)
            want[sid] = expected_md5s(path)
            for i, p in enumerate(read_packets(path)):
                cl.submit(sid, p, tag=i)
        # Equal reservations alternate between the two engines.
        placed = [cl.stats(i)["streams_open"] + cl.stats(i)["streams_pending"] for i in range(2)]
        assert placed == [3, 3], placed
        got = {sid: {} for sid in sids}
        total = sum(len(read_packets(os.path.join(VECTORS_DIR, n))) for n in NAMES)
        done = 0
        for _ in range(2000):
            for c in cl.poll(max_items=64, timeout_ms=50):
                assert c.ok, c.status
                got[c.stream][c.tag] = [hashlib.md5(f.packed()).hexdigest() for f in c.frames]
                done += 1
            if done == total:
                break
        assert done == total
        for sid in sids:
            md5s = [m for tag in sorted(got[sid]) for m in got[sid][tag]]
            assert md5s == want[sid]
        for sid in sids:
            cl.close_stream(sid)
    finally:
        cl.close()
