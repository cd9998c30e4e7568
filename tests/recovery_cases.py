"""Recovery inputs shared by the oracle tests and the GPU parity tests.

Encoded rows are codewords of a linear code over Fr, so field-linear
combinations of two encodings are encodings too; that builds the inputs whose
coset-0 rows decode to an invalid RawBlob / RawData (the error branches of
raw_blob.rs:42-58 and raw_data.rs:25-38 as reached from
crates/recovery/src/lib.rs:40).
"""
import random

from zgo import R_MOD


def split_rows(data: bytes, log_row: int, log_col: int) -> dict:
    """Encoded data (3R rows of C 32-byte elements) -> {row id: row bytes}."""
    n = 32 << log_col
    return {i: data[i * n:(i + 1) * n] for i in range(3 << log_row)}


def combine(rows_a: dict, rows_b: dict, fa: int, fb: int) -> dict:
    """fa * A + fb * B element-wise mod r (a codeword of fa*D_A + fb*D_B)."""
    out = {}
    for i, ra in rows_a.items():
        rb = rows_b[i]
        els = []
        for j in range(0, len(ra), 32):
            x = int.from_bytes(ra[j:j + 32], "little")
            y = int.from_bytes(rb[j:j + 32], "little")
            els.append(((fa * x + fb * y) % R_MOD).to_bytes(32, "little"))
        out[i] = b"".join(els)
    return out


def patterns(log_row: int) -> list:
    """Received-row sets: erasures at the ends, a whole coset, only the
    systematic rows, alternate rows, and seeded random sets of R .. 3R rows."""
    R = 1 << log_row
    pats = [
        list(range(1, 3 * R)),
        list(range(0, R)) + list(range(R + 1, 3 * R)),
        list(range(R + 1, 3 * R)),
        list(range(2 * R, 3 * R)),
        list(range(0, R)),
        list(range(1, 3 * R, 2)),
        list(range(R, 2 * R)),
    ]
    rng = random.Random(4)
    for k in (R, R + 1, 2 * R, 3 * R - 1, 3 * R):
        pats.append(sorted(rng.sample(range(3 * R), k)))
    return pats


def bad_codewords(encode, log_row: int, log_col: int) -> list:
    """(name, rows, expected) for inputs that are codewords of no valid
    RawData, or no valid input at all: `expected` is the error message, or
    the payload bytes where recovery succeeds. `encode(payload)` returns the
    encoded data bytes of a payload."""
    R, C = 1 << log_row, 1 << log_col
    max_raw = 31 * R * C - 4
    ones = split_rows(encode(b"\x01" * max_raw), log_row, log_col)
    a = split_rows(encode(b"x" * 100), log_row, log_col)
    b = split_rows(encode(b"x" * 50), log_row, log_col)
    cases = [
        # 2^248 * D: coset-0 values with a nonzero byte 31
        ("scalar", combine(ones, ones, 1 << 248, 0), "Incorrect scalar"),
        # element-wise sum of two full payloads: length field 2 * max_raw
        ("length", combine(ones, ones, 1, 1), "Incorrect length field"),
        # A - B: length 50 with bytes 50..99 still set
        ("padding", combine(a, b, 1, R_MOD - 1), "Non zero in padding range"),
    ]
    # one element of one row changed while more than R rows arrive
    bad = dict(a)
    row = bytearray(bad[R + 3])
    row[5] ^= 1
    bad[R + 3] = bytes(row)
    cases.append(("inconsistent", {i: bad[i] for i in range(0, 2 * R)}, "Inconsistent rows (degree check)"))
    # a value >= r (the reference panics in raw_slice_to_line)
    nc = dict(a)
    row = bytearray(nc[7])
    row[32 * 3:32 * 4] = b"\xff" * 32
    nc[7] = bytes(row)
    cases.append(("noncanonical", nc, "Non-canonical field element in slice"))
    # ... which the reference meets before it counts the rows
    assert R > 8
    cases.append(("noncanonical-few", {i: nc[i] for i in range(R - 1)}, "Non-canonical field element in slice"))
    # too few rows, a row id past the encoded rows, rows of the wrong length dropped
    cases.append(("few", {i: a[i] for i in range(2 * R + 2, 3 * R)}, "Not enough valid lines"))
    over = {i: a[i] for i in range(2 * R + 1, 3 * R)}
    over[3 * R] = a[0]
    cases.append(("overflow", over, "Cannot recover data: RowIdOverflow"))
    short = {i: a[i] for i in range(R)}
    short[R] = a[R][:-1]
    short[R + 1] = a[R + 1] + b"\x00"
    cases.append(("dropped", short, b"x" * 100))
    return cases
