"""TEXMEX descriptor files (.fvecs / .bvecs / .ivecs) and the recall tally."""
import numpy as np
import pytest

from matching_sift_b200 import datagen, vecs


def test_fvecs_round_trip_and_slices(tmp_path):
    x = np.random.default_rng(0).random((37, 128), dtype=np.float32)
    p = tmp_path / "a.fvecs"
    vecs.write_vecs(p, x)
    assert p.stat().st_size == 37 * (4 + 128 * 4)
    np.testing.assert_array_equal(vecs.read_fvecs(p), x)
    np.testing.assert_array_equal(vecs.read_fvecs(p, count=5, start=30), x[30:35])
    assert vecs.read_fvecs(p, count=0, start=37).shape == (0, 128)
    with pytest.raises(ValueError):
        vecs.read_fvecs(p, count=8, start=30)
    with pytest.raises(ValueError):
        vecs.read_fvecs(p, dim=64)


def test_record_layout_is_dim_then_values(tmp_path):
    p = tmp_path / "b.bvecs"
    vecs.write_vecs(p, np.array([[1, 2, 3], [250, 251, 252]], dtype=np.uint8))
    raw = p.read_bytes()
    assert raw == (b"\x03\x00\x00\x00\x01\x02\x03" + b"\x03\x00\x00\x00\xfa\xfb\xfc")
    np.testing.assert_array_equal(vecs.read_bvecs(p)[1], [250, 251, 252])


def test_bad_dimension_in_a_later_record_is_reported(tmp_path):
    p = tmp_path / "c.fvecs"
    vecs.write_vecs(p, np.zeros((4, 8), np.float32))
    raw = bytearray(p.read_bytes())
    raw[2 * (4 + 32):2 * (4 + 32) + 4] = np.int32(9).tobytes()  # record 2 claims dimension 9
    p.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="record 2"):
        vecs.read_fvecs(p)
    np.testing.assert_array_equal(vecs.read_fvecs(p, count=2), np.zeros((2, 8), np.float32))


def test_truncated_file_is_rejected(tmp_path):
    p = tmp_path / "d.fvecs"
    vecs.write_vecs(p, np.ones((3, 4), np.float32))
    p.write_bytes(p.read_bytes()[:-2])
    with pytest.raises(ValueError):
        vecs.read_fvecs(p)


def test_sift_floats_convert_to_u8_exactly(tmp_path):
    q, _ = datagen.make_workload(50, 100, seed=1)
    p = tmp_path / "q.fvecs"
    vecs.write_vecs(p, q.astype(np.float32))
    np.testing.assert_array_equal(vecs.to_u8(vecs.read_fvecs(p)), q)
    with pytest.raises(ValueError):
        vecs.to_u8(np.array([[0.5]], np.float32))
    with pytest.raises(ValueError):
        vecs.to_u8(np.array([[256.0]], np.float32))
    h = vecs.scaled_half(q)
    assert h.dtype == np.float16
    np.testing.assert_array_equal(h.astype(np.float32) * 512, q.astype(np.float32))


def test_ivecs_keeps_the_first_k_ids(tmp_path):
    t = np.arange(3 * 100, dtype=np.int32).reshape(3, 100)
    p = tmp_path / "gt.ivecs"
    vecs.write_vecs(p, t)
    np.testing.assert_array_equal(vecs.read_ivecs(p, k=10), t[:, :10])
    with pytest.raises(ValueError):
        vecs.read_ivecs(p, k=101)


def test_recall_tally_counts_misses_per_rank():
    truth = np.tile(np.arange(100), (4, 1))
    # query 0: rank 0 hit; 1: at rank 5; 2: at rank 55; 3: no match (0xFFFFFFFF)
    matches = np.array([0, 5, 55, 0xFFFFFFFF], dtype=np.uint32)
    m = vecs.recall_misses(matches, truth)
    assert m[1] == 3 and m[10] == 2 and m[50] == 2 and m[60] == 1 and m[100] == 1
    assert vecs.recall_at(matches, truth, 1) == 0.25
