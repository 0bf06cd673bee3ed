"""Shape classes of batched / served LPs and the lane-target table (no GPU):
b2_shape_class buckets by nonzeros (< 4K, < 16K, < 64K, < 256K, more) and
entries per row (< 8, < 16, < 32, more); the built-in table holds a valid lane
target for every class."""
import b200pdlp as B


def test_shape_class_buckets():
    assert B.shape_class(600, 1800, 10_800) == 1 * 4 + 2       # 16-32 entries a row, 4K-16K nonzeros
    assert B.shape_class(50, 120, 480) == 0 * 4 + 1            # 8-16 a row, < 4K
    assert B.shape_class(5000, 15000, 105_000) == 3 * 4 + 2    # 64K-256K
    assert B.shape_class(500_000, 1_000_000, 8_000_000) == 4 * 4 + 2
    assert B.shape_class(100, 100, 100) == 0                   # 1 a row
    assert B.shape_class(10, 10, 10_000) == 1 * 4 + 3          # 1,000 a row, 4K-16K
    assert B.shape_class(0, 5, 0) == 0


def test_default_table_is_complete():
    t = B.default_tune_table()
    assert len(t["lane_target"]) == B.TUNE_CLASSES
    assert all(v in (4, 8, 16, 32) for v in t["lane_target"])
    assert t["lane_target"][B.shape_class(3000, 9000, 54_000)] == 32  # measured on a B200: 16+ a row, 16K-64K
