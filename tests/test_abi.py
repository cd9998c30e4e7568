"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "zg_encoder.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_expected_surface():
    names = declared_functions()
    for n in ("zg_ctx_create", "zg_encode", "zg_encode_device", "zg_reply_slice", "zg_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(pkg):
    path = pkg.build.build()
    lib = ctypes.CDLL(path)
    for n in declared_functions():
        assert hasattr(lib, n), n
    assert sorted(pkg.C_ABI_FUNCTIONS) == declared_functions()


def test_too_large_blob_rejected_before_device(pkg):
    """RawData::try_from rejects len > MAX_RAW_DATA_SIZE (raw_data.rs:76-95)."""
    d = pkg.Dims(10, 10)
    try:
        pkg.RawData.try_from(bytes(d.max_raw_data_size + 1), d)
    except pkg.TooLargeBlob as e:
        assert (e.actual, e.expected_max) == (d.max_raw_data_size + 1, d.max_raw_data_size)
        assert str(e) == f"TooLargeBlob {{ actual: {d.max_raw_data_size + 1}, expected_max: {d.max_raw_data_size} }}"
    else:
        raise AssertionError("expected TooLargeBlob")
    rd = pkg.RawData.try_from(b"abc", d)
    assert rd.padded[-4:] == (3).to_bytes(4, "little") and rd.as_bytes() == b"abc"
    assert len(rd.padded) == d.max_blob_size == 32505856
    assert d.max_raw_data_size == 32505852
