"""Gauge configuration files in HILA's binary format (gaugefield.h:196-271,
field_io.h:128-330).  Host-only: runs without a GPU.

The format is pinned by writing files with numpy from the reference's layout
(int64 header {394824242, NDIM, sizeof(SU<3,double>), Lx..Lt}, then dir-major
lexicographic links) and reading them back, and the other way round."""
import numpy as np
import pytest

FLAG = 394824242


def _links(dims, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((4, int(np.prod(dims)), 3, 3, 2))


def _write_numpy(path, dims, links, header=None):
    h = np.array(header if header is not None else [FLAG, 4, 144, *dims], np.int64)
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(np.ascontiguousarray(links, np.float64).tobytes())


def test_write_matches_reference_layout(hw, tmp_path):
    dims = (4, 2, 6, 4)
    U = _links(dims, 1)
    p = tmp_path / "conf.bin"
    hw.config_write(str(p), dims, U)
    raw = p.read_bytes()
    assert np.frombuffer(raw[:56], np.int64).tolist() == [FLAG, 4, 144, *dims]
    assert raw[56:] == U.tobytes()
    assert hw.config_dims(str(p)) == dims


def test_read_numpy_written_file(hw, tmp_path):
    dims = (2, 4, 4, 6)
    U = _links(dims, 2)
    p = tmp_path / "conf.bin"
    _write_numpy(p, dims, U)
    assert np.array_equal(hw.config_read(str(p)), U)
    assert np.array_equal(hw.config_read(str(p), dims), U)


def test_round_trip_generated_links(hw, tmp_path):
    dims = (4, 4, 4, 8)
    U = hw.generate_links(dims, 0.3, 11)
    p = tmp_path / "conf.bin"
    hw.config_write(str(p), dims, U)
    assert np.array_equal(hw.config_read(str(p), dims), U)


def test_periodic_replication(hw, tmp_path):
    small, big = (2, 4, 2, 4), (4, 4, 6, 8)
    U = _links(small, 3)
    p = tmp_path / "small.bin"
    _write_numpy(p, small, U)
    R = hw.config_read(str(p), big)
    Us = U.reshape(4, small[3], small[2], small[1], small[0], 3, 3, 2)
    Rb = R.reshape(4, big[3], big[2], big[1], big[0], 3, 3, 2)
    for t in range(big[3]):
        for z in range(big[2]):
            for y in range(big[1]):
                for x in range(big[0]):
                    assert np.array_equal(Rb[:, t, z, y, x], Us[:, t % small[3], z % small[2], y % small[1],
                                                               x % small[0]])


@pytest.mark.parametrize("header,msg", [
    ([FLAG + 1, 4, 144, 2, 2, 2, 2], "wrong id"),
    ([FLAG, 3, 144, 2, 2, 2, 2], "wrong dimensionality"),
    ([FLAG, 4, 72, 2, 2, 2, 2], "wrong size of field element"),
    ([FLAG, 4, 144, 3, 2, 2, 2], "incorrect lattice dimension"),
])
def test_header_errors(hw, tmp_path, header, msg):
    p = tmp_path / "bad.bin"
    _write_numpy(p, (2, 2, 2, 2), _links((2, 2, 2, 2), 4), header=header)
    with pytest.raises(hw.HilaError) as e:
        hw.config_read(str(p), (4, 4, 4, 4))
    assert msg in str(e.value)
    assert e.value.code == hw.HW_ERR_INVALID


def test_truncated_file(hw, tmp_path):
    dims = (2, 2, 2, 2)
    p = tmp_path / "short.bin"
    _write_numpy(p, dims, _links(dims, 5)[:3])
    with pytest.raises(hw.HilaError) as e:
        hw.config_read(str(p), dims)
    assert "file ends inside direction 3" in str(e.value)
