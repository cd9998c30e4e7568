"""LightEncodedSlice (crates/encoder/src/encoder/light_slice.rs:11-79): the
C ABI's host conversions against the ark-serialize field order, and the
reference's round trip (encoder/blob.rs:268-280, test_light_slice) over every
slice of an oracle-encoded blob. Host code only: runs without a GPU."""
import pytest

LR, LC = 4, 5


@pytest.fixture(scope="module")
def slices(oracle):
    op = oracle.params(LR, LC, 3)
    blob = oracle.encode(op, bytes(range(200)) * 7)
    return [blob.slice(i) for i in range(3 << LR)]


def parse(s):
    """EncodedSlice fields in derive(CanonicalSerialize) order (slice.rs:15-20,
    amt/slice.rs:13-18, BlobRow encode.rs:205-212, merkle/slice.rs:12-18)."""
    C = 1 << LC
    o = 0

    def take(n):
        nonlocal o
        v = s[o:o + n]
        o += n
        return v

    f = {"index": take(8), "amt_index": take(8), "commitment": take(64), "row_index": take(8),
         "row": take(8 + 32 * C), "proof": take(8 + 128 * LR), "high": take(64), "roots": take(96),
         "path": take(8 + 32 * LR), "merkle_index": take(8), "leaf": take(32)}
    assert o == len(s)
    return f


def test_light_slice_layout_and_round_trip(pkg, slices):
    dims = pkg.Dims(LR, LC)
    for i, s in enumerate(slices):
        f = parse(s)
        light = pkg.LightEncodedSlice.from_slice(s, dims)
        exp = f["index"] + f["commitment"] + f["proof"] + f["high"] + f["roots"] + f["path"] + f["leaf"]
        assert light.data == exp and light.index == i
        assert len(light.data) == 280 + 160 * LR
        assert light.into_slice(f["row"][8:]) == s


def test_light_slice_index_checks(pkg, slices):
    dims = pkg.Dims(LR, LC)
    s = bytearray(slices[5])
    s[8:16] = (6).to_bytes(8, "little")
    with pytest.raises(RuntimeError, match=r"UnmatchedAMTIndex \{ row_index: 5, amt_index: 6 \}"):
        pkg.LightEncodedSlice.from_slice(bytes(s), dims)
    s = bytearray(slices[5])
    off = len(s) - 40
    s[off:off + 8] = (9).to_bytes(8, "little")
    with pytest.raises(RuntimeError, match=r"UnmatchedMerkleIndex \{ row_index: 5, merkle_index: 9 \}"):
        pkg.LightEncodedSlice.from_slice(bytes(s), dims)
    with pytest.raises(RuntimeError, match="length"):
        pkg.LightEncodedSlice.from_slice(slices[5][:-1], dims)
    light = pkg.LightEncodedSlice.from_slice(slices[5], dims)
    with pytest.raises(RuntimeError, match="row length"):
        light.into_slice(bytes(31))
