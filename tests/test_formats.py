"""Graph files: the BANG / DiskANN disk layout the reference's tooling writes
(scripts/bang-preprocess.py:37-72), converted on the host from its 772-byte records.
Pinned against the reference's own fixtures in data/sift10k, read in place."""
import os

import numpy as np
import pytest

from conftest import REFERENCE

GOLDEN = os.path.join(REFERENCE, "vamana", "vout", "vamana.out")
BANG = os.path.join(REFERENCE, "data", "sift10k", "test_sift10k_index_disk.bin")
META = os.path.join(REFERENCE, "data", "sift10k", "sift10k_index_disk_metadata.bin")
need_ref = pytest.mark.skipif(not (os.path.exists(GOLDEN) and os.path.exists(BANG)),
                              reason="reference fixtures not present")


def _records(path, n=10000, rec=772):
    raw = np.fromfile(path, dtype=np.uint8).reshape(n, rec)
    return raw, raw[:, 512:516].view(np.uint32)[:, 0], raw[:, 516:].view(np.uint32)


@need_ref
def test_converted_golden_graph_matches_the_bang_fixture(tmp_path):
    """The fixture holds the golden graph of a neighbouring build run: every row whose
    neighbour set agrees must come out byte for byte as the fixture has it."""
    import vann

    out = str(tmp_path / "g")
    vann.convert_graph_file(GOLDEN, 10000, 128, 64, 5000, out)
    ours, od, oa = _records(out + "_disk.bin")
    fix, fd, fa = _records(BANG)
    src, sd, sa = _records(GOLDEN)
    same_set = [i for i in range(10000)
                if sd[i] == fd[i] and np.array_equal(np.sort(sa[i, :sd[i]]), fa[i, :fd[i]])]
    assert len(same_set) >= 9990
    for i in range(10000):
        assert np.array_equal(oa[i, :od[i]], np.sort(sa[i, :sd[i]]))  # ids sorted
        assert np.array_equal(ours[i, :512], src[i, :512])             # vector unchanged
        assert np.array_equal(oa[i, od[i]:], sa[i, sd[i]:])            # unused slots unchanged
    rows_equal = [i for i in same_set if np.array_equal(ours[i], fix[i])]
    agree_pad = [i for i in same_set if np.array_equal(sa[i, sd[i]:], fa[i, fd[i]:])]
    assert rows_equal == agree_pad and len(rows_equal) >= 9990


@need_ref
def test_bang_fixture_is_a_fixed_point(tmp_path):
    """Sorted rows stay as they are: converting the fixture reproduces it exactly."""
    import vann

    out = str(tmp_path / "g")
    vann.convert_graph_file(BANG, 10000, 128, 64, 5000, out)
    assert open(out + "_disk.bin", "rb").read() == open(BANG, "rb").read()


@pytest.mark.skipif(not os.path.exists(META), reason="reference fixtures not present")
def test_metadata_layout_matches_the_fixture(tmp_path):
    import vann

    # a tiny record file with the fixture's header values (medoid 3732, D 128, R 64)
    raw = np.zeros((10000, 772), np.uint8)
    raw[:, 512:516] = np.frombuffer(np.uint32(1).tobytes(), np.uint8)  # degree 1
    path = str(tmp_path / "rec.bin")
    raw.tofile(path)
    out = str(tmp_path / "g")
    vann.convert_graph_file(path, 10000, 128, 64, 3732, out)
    assert open(out + "_disk_metadata.bin", "rb").read() == open(META, "rb").read()


def test_degree_zero_is_rejected(tmp_path):
    import vann

    raw = np.zeros((4, 4 * 16 + 4 + 4 * 8), np.uint8)
    path = str(tmp_path / "rec.bin")
    raw.tofile(path)
    with pytest.raises(vann.VannError) as e:
        vann.convert_graph_file(path, 4, 16, 8, 0, str(tmp_path / "g"))
    assert e.value.status == vann.ERR_STATE
