"""XAMG's binary system file (src/io/detail/reader.inl:47-177) through the C
ABI, on the CPU: u32 nrows, u32 nnz, u32 row[nrows+1], u32 col[nnz],
f64 val[nnz], then optional f64 b and x of nrows*nv values each. Files are
written here byte by byte with numpy, read back by the library, and the
library's writer must produce the same bytes."""
import numpy as np
import pytest


def numpy_file(path, row, col, val, b=None, x=None):
    with open(path, "wb") as f:
        f.write(np.array([len(row) - 1, len(col)], np.uint32).tobytes())
        f.write(np.asarray(row, np.uint32).tobytes())
        f.write(np.asarray(col, np.uint32).tobytes())
        f.write(np.asarray(val, np.float64).tobytes())
        if b is not None:
            f.write(np.asarray(b, np.float64).tobytes())
        if x is not None:
            f.write(np.asarray(x, np.float64).tobytes())


@pytest.mark.parametrize("nv", [1, 4])
@pytest.mark.parametrize("with_b,with_x", [(False, False), (True, False), (True, True)])
def test_read_system_matches_the_format(xamg, tmp_path, nv, with_b, with_x):
    row, col, val = xamg.generate_cube(5, 4, 3)
    n = len(row) - 1
    rng = np.random.default_rng(nv)
    b = rng.standard_normal(n * nv) if with_b else None
    x = rng.standard_normal(n * nv) if with_x else None
    path = tmp_path / "sys.bin"
    numpy_file(path, row, col, val, b, x)
    r, c, v, bb, xx, found = xamg.read_system(path, nv)
    assert r.tobytes() == row.tobytes() and c.tobytes() == col.tobytes()
    assert v.tobytes() == val.tobytes()
    assert found == (1 if with_b else 0) | (2 if with_x else 0)
    assert bb.tobytes() == (b.tobytes() if with_b else np.ones(n * nv).tobytes())
    assert xx.tobytes() == (x.tobytes() if with_x else np.zeros(n * nv).tobytes())
    # the writer gives the same bytes back
    out = tmp_path / "out.bin"
    xamg.write_system(out, row, col, val, nv, b, x)
    assert out.read_bytes() == path.read_bytes()


def test_read_system_rejects_bad_files(xamg, tmp_path):
    row, col, val = xamg.generate_cube(3, 3, 3)
    path = tmp_path / "short.bin"
    numpy_file(path, row, col, val)
    data = path.read_bytes()
    (tmp_path / "cut.bin").write_bytes(data[:-12])
    with pytest.raises(xamg.XamgError):
        xamg.read_system(tmp_path / "cut.bin")
    with pytest.raises(xamg.XamgError):
        xamg.read_system(tmp_path / "missing.bin")
    bad = bytearray(data)
    bad[8:12] = np.array([5], np.uint32).tobytes()  # row[0] != 0
    (tmp_path / "bad.bin").write_bytes(bytes(bad))
    with pytest.raises(xamg.XamgError):
        xamg.read_system(tmp_path / "bad.bin")
    with pytest.raises(xamg.XamgError):
        xamg.write_system(tmp_path / "w.bin", row, col, val, 1, None, np.zeros(27))
