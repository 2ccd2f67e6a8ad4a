"""Placement of streams across the GPUs of a node (rv9_cluster), on the CPU:
the placement rule against fake device lists, and a cluster that refuses to
start without a device. Each stream goes whole to one device (the least
loaded by reserved bytes among those with room), since a stream's frames
chain through its own reference slots and streams share nothing."""
import pytest

GB = 1 << 30


@pytest.fixture(scope="module")
def server():
    import rv9  # noqa: F401  (builds nothing; the library is built by conftest's users)
    from rv9 import server
    return server


def test_least_loaded_device_with_room(server):
    assert server.place_least_loaded([5 * GB, 2 * GB, 9 * GB], [10 * GB] * 3, 1 * GB) == 1
    # Ties go to the lowest index.
    assert server.place_least_loaded([3 * GB, 3 * GB], [10 * GB] * 2, 1 * GB) == 0
    # The least loaded device lacks room (smaller budget): the next one that has it.
    assert server.place_least_loaded([1 * GB, 4 * GB], [2 * GB, 10 * GB], 2 * GB) == 1


def test_no_room_now_goes_to_the_least_loaded_that_could_hold_it(server):
    # Every device is full: the stream waits on the least loaded one.
    assert server.place_least_loaded([9 * GB, 8 * GB, 9 * GB], [10 * GB] * 3, 3 * GB) == 1
    # A device whose whole budget is too small is never chosen.
    assert server.place_least_loaded([0, 8 * GB], [1 * GB, 10 * GB], 3 * GB) == 1


def test_nothing_could_hold_it(server):
    assert server.place_least_loaded([0, 0], [1 * GB, 1 * GB], 2 * GB) == -1
    assert server.place_least_loaded([], [], 1) == -1


def test_placement_sequence_balances_bytes(server):
    # The served mix's reservations placed one after another on 8 devices:
    # every device ends within one stream's reservation of the others.
    r720 = server.reservation(1280, 720)
    r1080 = server.reservation(1920, 1080)
    r2160 = server.reservation(3840, 2160, bit_depth=10)
    mix = [r720] * 13 + [r1080] * 13 + [r2160] * 6
    load = [0] * 8
    for need in mix:
        d = server.place_least_loaded(load, [120 * GB] * 8, need)
        assert d >= 0
        load[d] += need
    assert max(load) - min(load) <= max(mix)


def test_cluster_needs_a_device(server):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import rv9
    with pytest.raises(rv9.DeviceError):
        server.Cluster([0, 1])
