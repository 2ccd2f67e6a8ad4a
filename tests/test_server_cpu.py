"""The serving API's argument checks, on the CPU (no device needed): calls
on a null engine or cluster are refused before anything runs, and the
reservation of a stream spec is defined without an engine."""
import ctypes


def test_null_engine_and_cluster_are_refused():
    import rv9
    from rv9 import server
    lib = server._bind(rv9.load_library())
    spec = server.spec(1920, 1080)
    assert lib.rv9_engine_set_device_parse(None, 1, 8, 0) == rv9.RV9_INVALID_INPUT
    assert lib.rv9_cluster_set_device_parse(None, 1, 8, 0) == rv9.RV9_INVALID_INPUT
    assert lib.rv9_engine_stream_reservation(None, ctypes.byref(spec)) == 0
    # The plain reservation grows with the frame.
    small = lib.rv9_stream_reservation(ctypes.byref(server.spec(640, 360)))
    assert 0 < small < lib.rv9_stream_reservation(ctypes.byref(spec))
