"""Generates the golden fixtures of tests/golden/ with an independent pure-
Python restatement of the encode path:
  encode_3x5.json  an 8 x 32 blob (LOG_ROW = 3, LOG_COL = 5), plus single
                   known-answer vectors (keccak, G1 multiples, roots);
  encode_6x5.json  a 64 x 32 blob, the reference's own test setting
                   (BLOB_ROW_LOG = 6, BLOB_COL_LOG = 5 when TEST_SETTING,
                   crates/encoder/src/constants.rs:11-15), full payload.

It shares no code with oracle/ or the CUDA library: Python integers for Fr,
Fq and G1, naive O(n^2) DFTs, a pure-Python Keccak-f[1600], and params from
the scalar domain of the seeded tau (every param point is s * G1, so every
AMT output is (sum of scalar x param-scalar) * G1). The reference files each
step follows are cited inline. Run: python tests/golden/make_golden.py
"""
import hashlib
import json
import os

R_MOD = 21888242871839275222246405745257275088548364400416034343698204186575808495617
Q_MOD = 21888242871839275222246405745257275088696311157297823662689037894645226208583
G1 = (1, 2)
COSET_N = 3
# the shapes of the fixtures: (file, log_row, log_col, seed, payload)
FIXTURES = [
    ("encode_3x5.json", 3, 5, 42, bytes((i * 7 + 3) % 251 for i in range(200))),
    ("encode_6x5.json", 6, 5, 222, bytes((i * 131 + 17) % 256 for i in range(31 * 2048 - 4))),
]


# ---- Keccak-256 (tiny-keccak Keccak::v256: rate 136, pad 0x01 .. 0x80)
RC = [0x0000000000000001, 0x0000000000008082, 0x800000000000808A, 0x8000000080008000, 0x000000000000808B,
      0x0000000080000001, 0x8000000080008081, 0x8000000000008009, 0x000000000000008A, 0x0000000000000088,
      0x0000000080008009, 0x000000008000000A, 0x000000008000808B, 0x800000000000008B, 0x8000000000008089,
      0x8000000000008003, 0x8000000000008002, 0x8000000000000080, 0x000000000000800A, 0x800000008000000A,
      0x8000000080008081, 0x8000000000008080, 0x0000000080000001, 0x8000000080008008]
ROT = [[0, 36, 3, 41, 18], [1, 44, 10, 45, 2], [62, 6, 43, 15, 61], [28, 55, 25, 21, 56], [27, 20, 39, 8, 14]]
M64 = (1 << 64) - 1


def _rotl(x, n):
    return ((x << n) | (x >> (64 - n))) & M64 if n else x


def _keccak_f(a):
    for rnd in range(24):
        c = [a[x][0] ^ a[x][1] ^ a[x][2] ^ a[x][3] ^ a[x][4] for x in range(5)]
        d = [c[(x - 1) % 5] ^ _rotl(c[(x + 1) % 5], 1) for x in range(5)]
        a = [[a[x][y] ^ d[x] for y in range(5)] for x in range(5)]
        b = [[0] * 5 for _ in range(5)]
        for x in range(5):
            for y in range(5):
                b[y][(2 * x + 3 * y) % 5] = _rotl(a[x][y], ROT[x][y])
        a = [[b[x][y] ^ ((~b[(x + 1) % 5][y]) & b[(x + 2) % 5][y]) for y in range(5)] for x in range(5)]
        a[0][0] ^= RC[rnd]
    return a


def keccak256(data: bytes, pad=0x01) -> bytes:
    rate = 136
    msg = bytearray(data)
    msg.append(pad)
    while len(msg) % rate:
        msg.append(0)
    msg[-1] |= 0x80
    a = [[0] * 5 for _ in range(5)]
    for off in range(0, len(msg), rate):
        blk = msg[off:off + rate]
        for i in range(rate // 8):
            a[i % 5][i // 5] ^= int.from_bytes(blk[8 * i:8 * i + 8], "little")
        a = _keccak_f(a)
    out = b"".join(a[i % 5][i // 5].to_bytes(8, "little") for i in range(4))
    return out


# ---- G1 (y^2 = x^3 + 3) affine with None = infinity
def g1_add(p, q):
    if p is None:
        return q
    if q is None:
        return p
    if p[0] == q[0]:
        if (p[1] + q[1]) % Q_MOD == 0:
            return None
        lam = 3 * p[0] * p[0] * pow(2 * p[1], -1, Q_MOD) % Q_MOD
    else:
        lam = (q[1] - p[1]) * pow(q[0] - p[0], -1, Q_MOD) % Q_MOD
    x = (lam * lam - p[0] - q[0]) % Q_MOD
    return (x, (lam * (p[0] - x) - p[1]) % Q_MOD)


def g1_mul(k, p=G1):
    acc, base = None, p
    k %= R_MOD
    while k:
        if k & 1:
            acc = g1_add(acc, base)
        base = g1_add(base, base)
        k >>= 1
    return acc


def ser_g1(p) -> bytes:
    """ark-serialize 0.4 uncompressed affine: x || y LE, y's top byte holds
    SWFlags (bit 7: y > -y, bit 6: infinity)."""
    if p is None:
        return bytes(63) + b"\x40"
    x, y = p
    b = bytearray(x.to_bytes(32, "little") + y.to_bytes(32, "little"))
    if y > Q_MOD - y:
        b[63] |= 0x80
    return bytes(b)


def reply_commitment(p) -> bytes:  # grpc/src/service.rs:77-83
    return bytes(64) if p is None else p[0].to_bytes(32, "little") + p[1].to_bytes(32, "little")


# ---- Fr domain helpers (ark-poly Radix2EvaluationDomain semantics)
def root(log_n):
    return pow(5, (R_MOD - 1) >> log_n, R_MOD)


def dft(v, w):
    n = len(v)
    wp = [1] * n  # w^e for e < n (w has order n)
    for e in range(1, n):
        wp[e] = wp[e - 1] * w % R_MOD
    return [sum(v[j] * wp[(j * k) % n] for j in range(n)) % R_MOD for k in range(n)]


def idft(v):
    n = len(v)
    ni = pow(n, -1, R_MOD)
    return [x * ni % R_MOD for x in dft(v, pow(root(n.bit_length() - 1), -1, R_MOD))]


def bitrev(x, bits):
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


def coset_factor(log_len, idx):  # prove_params/generate.rs:128-137
    return pow(root(28), bitrev(idx, 28 - log_len), R_MOD)


def splitmix64(state):
    state = (state + 0x9E3779B97F4A7C15) & M64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return state, z ^ (z >> 31)


def tau_from_seed(seed):
    s, acc = seed, 0
    for i in range(8):
        s, w = splitmix64(s)
        acc |= w << (64 * i)
    return acc % R_MOD


# ---- params in the scalar domain (prove_params/generate.rs:139-263)
def param_scalars(tau, coset, LOG_ROW, LOG_COL):
    N = 1 << (LOG_ROW + LOG_COL)
    depth = LOG_ROW + LOG_COL
    w = pow(coset_factor(depth, coset), -1, R_MOD) if coset else 1
    tp = tau * w % R_MOD
    pw = [pow(tp, i, R_MOD) for i in range(N)]
    hs = pow(tau, (1 << (depth + 2)) - N, R_MOD)
    basis = idft(pw)
    high = [x * hs % R_MOD for x in basis]
    ninv = pow(N, -1, R_MOD)
    quot = []
    for d in range(1, LOG_ROW + 1):
        m = N >> d
        coeff = [0] * N
        for i in range(1, m + 1):
            coeff[i] = pw[m - i]
        q = [x * ninv % R_MOD for x in dft(coeff, root(depth))]
        quot.append([q[bitrev(p, depth)] for p in range(N)])
    enact = lambda v: [v[bitrev(p, depth)] for p in range(N)]
    return enact(basis), quot, enact(high)


# ---- encode (crates/amt/src/blob/encode.rs:91-200, encoder/blob.rs:32-72, merkle/blob.rs)
def encode(LOG_ROW, LOG_COL, SEED, PAYLOAD):
    ROWS, COLS = 1 << LOG_ROW, 1 << LOG_COL
    N = ROWS * COLS
    max_blob = 31 * N
    max_raw = max_blob - 4
    raw = bytearray(max_blob)
    raw[:len(PAYLOAD)] = PAYLOAD
    raw[max_raw:] = len(PAYLOAD).to_bytes(4, "little")
    blob = [int.from_bytes(raw[31 * i:31 * i + 31], "little") for i in range(N)]
    points = [0] * N
    for i in range(N):  # change_matrix_direction(LOG_COL, LOG_ROW)
        r, j = divmod(i, COLS)
        points[j * ROWS + r] = blob[i]
    coeff = idft(points)
    tau = tau_from_seed(SEED)
    cosets = []
    for c in range(COSET_N):
        g = coset_factor(LOG_ROW + LOG_COL, c) if c else 1
        ev = dft([coeff[m] * pow(g, m, R_MOD) % R_MOD for m in range(N)], root(LOG_ROW + LOG_COL))
        ri = [ev[bitrev(p, LOG_ROW + LOG_COL)] for p in range(N)]
        basis, quot, high = param_scalars(tau, c, LOG_ROW, LOG_COL)
        batch = N >> LOG_ROW
        leaves = [sum(ri[k * batch + t] * basis[k * batch + t] for t in range(batch)) % R_MOD
                  for k in range(ROWS)]
        levels = [leaves]
        while len(levels[0]) > 1:
            prev = levels[0]
            levels.insert(0, [(prev[2 * i] + prev[2 * i + 1]) % R_MOD for i in range(len(prev) // 2)])
        commitment = levels[0][0]
        commits = levels[1:]  # commitments[d] has 2^(d+1) nodes
        proofs = []
        for d in range(1, LOG_ROW + 1):
            chunk = N >> d
            proofs.append([sum(ri[k * chunk + t] * quot[d - 1][k * chunk + t] for t in range(chunk)) % R_MOD
                           for k in range(1 << d)])
        high_c = sum(ri[p] * high[p] for p in range(N)) % R_MOD
        blob_rows = [ev[j * ROWS + r] for r in range(ROWS) for j in range(COLS)]  # row-major
        cosets.append({"rows": blob_rows, "commitment": commitment, "commits": commits,
                       "proofs": proofs, "high": high_c})
    assert all(c["commitment"] == cosets[0]["commitment"] for c in cosets)
    data = [x.to_bytes(32, "little") for c in cosets for x in c["rows"]]
    layer = [keccak256(b"".join(data[8 * i:8 * i + 8])) for i in range(len(data) // 8)]
    tree = [layer]
    while len(tree[0]) > COSET_N:
        prev = tree[0]
        tree.insert(0, [keccak256(prev[2 * i] + prev[2 * i + 1]) for i in range(len(prev) // 2)])
    roots = tree[0]
    file_root = keccak256(keccak256(roots[0] + roots[1]) + roots[2])
    pt = {}

    def point(s):
        if s not in pt:
            pt[s] = g1_mul(s)
        return pt[s]

    slices = []
    u64 = lambda v: v.to_bytes(8, "little")
    for index in range(COSET_N * ROWS):
        c, local = divmod(index, ROWS)
        cs = cosets[c]
        out = bytearray()
        out += u64(index) + u64(index) + ser_g1(point(cs["commitment"]))
        out += u64(local) + u64(COLS)
        for x in cs["rows"][local * COLS:(local + 1) * COLS]:
            out += x.to_bytes(32, "little")
        rev = bitrev(local, LOG_ROW)
        out += u64(LOG_ROW)
        for d in range(LOG_ROW):
            lv = rev >> (LOG_ROW - 1 - d)
            out += ser_g1(point(cs["commits"][d][lv ^ 1])) + ser_g1(point(cs["proofs"][d][lv ^ 1]))
        out += ser_g1(point(cs["high"]))
        for rt in roots:
            out += rt
        out += u64(LOG_ROW)
        for d in range(LOG_ROW, 0, -1):
            out += tree[d][(index >> (LOG_ROW - d)) ^ 1]
        out += u64(index) + tree[LOG_ROW][index]
        slices.append(bytes(out))
    return {
        "log_row": LOG_ROW, "log_col": LOG_COL, "seed": SEED, "payload_hex": PAYLOAD.hex(),
        "tau": hex(tau),
        "erasure_commitment": reply_commitment(point(cosets[0]["commitment"])).hex(),
        "roots": [r.hex() for r in roots], "file_root": file_root.hex(),
        "encoded_data_sha256": hashlib.sha256(b"".join(data)).hexdigest(),
        "slice_sha256": [hashlib.sha256(s).hexdigest() for s in slices],
        "slice_size": len(slices[0]),
    }


def vectors():
    ks = [1, 2, 3, 0x1234567890ABCDEF, R_MOD - 1, tau_from_seed(7)]
    return {
        "keccak256": {m.hex(): keccak256(m).hex() for m in (b"", b"abc", bytes(range(200)))},
        "g1_mul": {hex(k): ser_g1(g1_mul(k)).hex() for k in ks},
        "coset_factor_16_1_eq_root_32": coset_factor(4, 1) == root(5),
        "root_of_unity_28": hex(root(28)),
    }


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    for k, (name, lr, lc, seed, payload) in enumerate(FIXTURES):
        out = {"encode": encode(lr, lc, seed, payload)}
        if k == 0:
            out["vectors"] = vectors()
        with open(os.path.join(here, name), "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)
        print("wrote", os.path.join(here, name))
