"""Image files through the C ABI (host only): EDF, MHD and PGM against the headers and behaviour
the reference's tests fix (io/tests/test_EDFHandler.cpp, test_MHDHandler.cpp,
test_PGMHandler.cpp) and against its parse rules (io/EDFHandler.cpp, io/MHDHandler.cpp)."""
import numpy as np
import pytest

import elsa_b200


def _header_lines(path):
    raw = open(path, "rb").read()
    header = raw[:raw.index(b"}") + 1].decode()
    parts = header.split("\n")
    # as test_EDFHandler.cpp:44-49: drop '{', the padding and the closing '}'
    assert parts[0] == "{" and parts[-1] == "}" and parts[-2].strip() == ""
    return parts[1:-2], raw


@pytest.mark.parametrize("dims,lines", [
    ([5], ["Dim_1 = 5;", "Size = 20;", "Spacing = 1;"]),
    ([5, 10], ["Dim_1 = 5;", "Dim_2 = 10;", "Size = 200;", "Spacing = 1 1;"]),
])
def test_edf_header_golden(tmp_path, dims, lines):
    path = str(tmp_path / "a.edf")
    elsa_b200.edf_write(path, np.zeros(int(np.prod(dims)), np.float32), dims)
    parts, raw = _header_lines(path)
    assert parts[:4] == ["HeaderID = EH:000001:000000:000000;", "Image = 1;",
                         "ByteOrder = LowByteFirst;", "DataType = FloatValue;"]
    assert parts[4:] == lines
    head = raw.index(b"}") + 2
    assert head % 1024 == 0 and len(raw) == head + 4 * int(np.prod(dims))


def test_edf_round_trip(tmp_path):
    path = str(tmp_path / "b.edf")
    ones = np.ones(11 * 17, np.float32)  # test_EDFHandler.cpp:116-137
    elsa_b200.edf_write(path, ones, [11, 17])
    data, dims, spacing, kind = elsa_b200.edf_read(path)
    assert dims == [11, 17] and spacing == [1.0, 1.0] and kind == "float32"
    assert np.array_equal(data, ones)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(6 * 5 * 4).astype(np.float32)
    elsa_b200.edf_write(path, x, [6, 5, 4], [0.5, 1.0, 2.0])
    data, dims, spacing, _ = elsa_b200.edf_read(path)
    assert dims == [6, 5, 4] and spacing == [0.5, 1.0, 2.0]
    assert np.array_equal(data, x)


def _edf(tmp_path, header, payload=b""):
    path = str(tmp_path / "h.edf")
    with open(path, "wb") as f:
        f.write(header.encode() + payload)
    return path


def test_edf_reader_rules(tmp_path):
    vals = np.array([1, 2, 65535, 7, 0, 3], np.uint16)
    # quoted values, ';' inside quotes, mixed-case names, unsigned short data
    path = _edf(tmp_path, "{\n  dim_1 = 3 ;\n DIM_2=2;\r\nTitle = \"a;b\";\nByteOrder = "
                          "'LowByteFirst';\nDataType = UnsignedShort;\nSize = 12;\n}\n",
                vals.tobytes())
    data, dims, spacing, kind = elsa_b200.edf_read(path)
    assert dims == [3, 2] and kind == "uint16" and spacing == [1.0, 1.0]
    assert np.array_equal(data, vals.astype(np.float32))
    d64 = np.array([0.25, -1.5], np.float64)
    path = _edf(tmp_path, "{\nDim_1 = 2;\nDataType = DoubleValue;\nSize = 16;\nSpacing = 3;\n}\n",
                d64.tobytes())
    data, dims, spacing, kind = elsa_b200.edf_read(path)
    assert kind == "float64" and spacing == [3.0] and np.array_equal(data, d64.astype(np.float32))


@pytest.mark.parametrize("header,msg", [
    ("Dim_1 = 2;\nDataType = Float;\nSize = 8;\n}\n", "no header opening marker"),
    ("{\nDataType = Float;\nSize = 8;\n}\n", "dimension information not found"),
    ("{\nDim_1 = 2;\nSize = 8;\n}\n", "data type not found"),
    ("{\nDim_1 = 2;\nDataType = Int64;\nSize = 8;\n}\n", "invalid/unsupported data type"),
    ("{\nDim_1 = 2;\nDataType = Float;\nSize = 8;\nCompression = gzip;\n}\n",
     "compression not supported"),
    ("{\nDim_1 = 2;\nDataType = Float;\nSize = 9;\n}\n", "size inconsistency"),
    ("{\nDim_1 = 2;\nDataType = Float;\n}\n", "size inconsistency"),
    ("{\nDim_1 = 2;\nDataType = Float;\nSize = 8;\nByteOrder = HighByteFirst;\n}\n",
     "byte order"),
    ("{\nDim_1 = 2;\nDataType = Float;\nSize = 8;\nImage = 2;\n}\n", "image not set to 1"),
    ("{\nDim_1 = 2;\nDataType = Float;\nSize = 8;\nSpacing = 1 2;\n}\n", "spacing inconsistency"),
    ("{\nDim_1 = 2;\nDataType = Float;\nSize = 8;\nbroken;\n}\n", "name/value delimiter"),
    ("{\nDim_1 = two;\nDataType = Float;\nSize = 8;\n}\n", "failed to interpret"),
    ("{\nDim_1 = 2;\nDataType = SignedByte;\nSize = 2;\n}\n", "invalid/unsupported data type"),
    ("{\nDim_1 = 2;\nDataType = Float;\nSize = 8;\n}\n", "sufficient data"),
])
def test_edf_reader_errors(tmp_path, header, msg):
    path = _edf(tmp_path, header, b"\0\0\0\0" if "sufficient" in msg else
                (b"\0" * 8 if "SignedByte" not in header else b"\0\0"))
    with pytest.raises(elsa_b200.InvalidArgumentError, match=msg):
        elsa_b200.edf_read(path)
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.edf_read(str(tmp_path / "missing.edf"))


def test_mhd_round_trip_and_header(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)  # test_MHDHandler.cpp:28-41 writes test.mhd / test.raw here
    ones = np.ones(11 * 17, np.float32)
    elsa_b200.mhd_write("test.mhd", "test.raw", ones, [11, 17])
    data, dims, spacing, kind = elsa_b200.mhd_read("test.mhd")
    assert dims == [11, 17] and spacing == [1.0, 1.0] and kind == "float32"
    assert np.array_equal(data, ones)
    # vectors printed as Eigen prints them: right-aligned to the widest coefficient
    elsa_b200.mhd_write("b.mhd", "b.raw", np.zeros(50, np.float32), [5, 10], [0.5, 1.0])
    assert open("b.mhd").read().splitlines() == [
        "NDims = 2", "DimSize =  5 10", "ElementSpacing = 0.5   1", "ElementType = MET_FLOAT",
        "ElementByteOrderMSB = False", "ElementDataFile = b.raw"]
    # the data file is found relative to the meta file, from any working directory
    sub = tmp_path / "sub"
    sub.mkdir()
    monkeypatch.chdir(sub)
    data, dims, spacing, _ = elsa_b200.mhd_read(str(tmp_path / "b.mhd"))
    assert dims == [5, 10] and spacing == [0.5, 1.0]


def test_mhd_reader_rules_and_errors(tmp_path):
    vals = np.array([3, 1, 4, 1, 5, 9], np.uint16)
    (tmp_path / "d.raw").write_bytes(vals.tobytes())

    def meta(text):
        p = tmp_path / "m.mhd"
        p.write_text(text)
        return str(p)

    good = ("  ndims = 2\n\nDIMSIZE = 3 2\nElementType = met_ushort\n"
            "ElementByteOrderMSB = no\nElementSpacing = 2 0.5\nElementDataFile = d.raw\n")
    data, dims, spacing, kind = elsa_b200.mhd_read(meta(good))
    assert dims == [3, 2] and spacing == [2.0, 0.5] and kind == "uint16"
    assert np.array_equal(data, vals.astype(np.float32))
    for text, msg in [
        (good.replace("  ndims = 2\n", ""), "ndims"),
        (good.replace("= no", "= True"), "little endian"),
        (good.replace("met_ushort", "MET_INT"), "unsupported value"),
        (good.replace("ElementType = met_ushort\n", ""), "element type"),
        (good.replace("ElementDataFile = d.raw\n", ""), "element data file"),
        (good.replace("DIMSIZE = 3 2", "DimSize = 3 2 1"), "dimension size mismatch"),
        (good.replace("2 0.5", "2"), "spacing size mismatch"),
        (good + "no pair here\n", "name/value pair"),
        (good.replace("d.raw", "nothere.raw"), "can not read"),
        (good.replace("met_ushort", "MET_CHAR"), "invalid/unsupported data type"),
    ]:
        with pytest.raises(elsa_b200.InvalidArgumentError, match=msg):
            elsa_b200.mhd_read(meta(text))


def test_pgm_golden(tmp_path):
    """test_PGMHandler.cpp:27-76: a 10 x 10 image of i + 10."""
    x = (np.arange(100) + 10).astype(np.float32)
    path = str(tmp_path / "a.pgm")
    elsa_b200.pgm_write(path, x, [10, 10])
    text = open(path).read()
    lines = text.split("\n", 3)
    assert lines[:3] == ["P2", "10 10", "255"]
    body = lines[3].split(" ")
    assert body[-1] == ""
    mn, mx = np.float32(x.min()), np.float32(x.max())
    want = [str(int(np.float32(np.float32(v - mn) / np.float32(mx - mn)) * np.float32(255.0)))
            for v in x]
    assert body[:-1] == want
    # 3D data with a last dimension of 1 is a slice; other shapes are rejected
    elsa_b200.pgm_write(path, x, [10, 10, 1])
    with pytest.raises(elsa_b200.InvalidArgumentError, match="2D"):
        elsa_b200.pgm_write(path, x, [100])
    with pytest.raises(elsa_b200.InvalidArgumentError):
        elsa_b200.pgm_write(path, x, [5, 5, 4])
    # a constant image scales by 0
    elsa_b200.pgm_write(path, np.full(4, 3.0, np.float32), [2, 2])
    assert open(path).read() == "P2\n2 2\n255\n0 0 0 0 "
