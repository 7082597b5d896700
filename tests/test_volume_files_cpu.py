"""Reading volumes back (CPU): the viewer's .txt info parse and
Volume::loadFromBinaryFile semantics (index order, byte order, data types,
header offset, mirroring, size check)."""
import numpy as np
import pytest

from ct_b200 import CtbError, load_volume, read_volume_info
from ct_b200 import _lib as L

INFO = """vol.raw

[Image dimensions]
U resolution:\t\t256
V resolution:\t\t192

[Volume dimensions]
X size:\t\t\t\t{x}
Y size:\t\t\t\t{y}
Z size:\t\t\t\t{z}

[Data format]
Data type:\t\t\t32bit IEEE 754 float
Byte order:\t\t\t{bo}
Index order:\t\t{io}"""


def test_read_volume_info(tmp_path):
    p = tmp_path / "vol.txt"
    p.write_text(INFO.format(x=7, y=5, z=3, bo="Big endian", io="X fastest"))
    assert read_volume_info(p) == {"x": 7, "y": 5, "z": 3, "index_order": L.X_FASTEST, "byte_order": L.BIG_ENDIAN}
    p.write_text(INFO.format(x=7, y=5, z=3, bo="Little endian", io="Z fastest"))
    assert read_volume_info(p)["index_order"] == L.Z_FASTEST
    p.write_text("X size:\t4\nY size:\t4\n")
    with pytest.raises(CtbError):
        read_volume_info(p)


DTYPES = {0: "f4", 1: "f8", 2: "u1", 3: "i1", 4: "u2", 5: "i2", 6: "u4", 7: "i4"}


@pytest.mark.parametrize("dt", sorted(DTYPES))
@pytest.mark.parametrize("order", [L.X_FASTEST, L.Z_FASTEST])
@pytest.mark.parametrize("endian", [L.LITTLE_ENDIAN, L.BIG_ENDIAN])
def test_load_volume(tmp_path, dt, order, endian):
    rng = np.random.default_rng(dt * 4 + order * 2 + endian)
    X, Y, Z = 6, 5, 4
    vol = (rng.integers(0, 100, (Z, Y, X)) - (0 if DTYPES[dt][0] == "u" else 50)).astype(np.float32)
    data = vol if order == L.X_FASTEST else vol.transpose(2, 1, 0)
    code = (">" if endian == L.BIG_ENDIAN else "<") + DTYPES[dt]
    p = tmp_path / "v.raw"
    p.write_bytes(b"HDR!" + np.ascontiguousarray(data).astype(code).tobytes())
    out = load_volume(p, X, Y, Z, order, endian, dt, header_offset=4)
    assert np.array_equal(out, vol)
    out = load_volume(p, X, Y, Z, order, endian, dt, header_offset=4, mirror=(True, False, True))
    assert np.array_equal(out, vol[::-1, :, ::-1])


def test_load_volume_size_check(tmp_path):
    p = tmp_path / "v.raw"
    p.write_bytes(b"\0" * 100)
    with pytest.raises(CtbError) as e:
        load_volume(p, 5, 5, 5)
    assert "Expected filesize" in e.value.message
