"""Host logic of the Eb/N0 sweep (the GPU part is the decode-summary entry
point, tested in test_gpu_summary.py)."""
from sogrand_b200.sweep import parse_points


def test_parse_points_range_and_list():
    assert parse_points("1.0:3.0:0.25") == [1.0, 1.25, 1.5, 1.75, 2.0, 2.25, 2.5, 2.75, 3.0]
    assert parse_points("2.0:2.0:0.5") == [2.0]
    assert parse_points("1.25,1.5,2") == [1.25, 1.5, 2.0]
