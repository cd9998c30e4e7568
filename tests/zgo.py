"""ctypes binding of the CPU oracle (oracle/, test infrastructure only).

Used by the tests, __graft_entry__.smoke() and bench.py's CPU baseline as the
checker; never by the product path.
"""
import ctypes
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "_build", "libzg_oracle.so")

_P = ctypes.c_void_p
_SZ = ctypes.c_size_t
_SIGS = {
    "zgo_num_threads": (ctypes.c_int, []),
    "zgo_set_threads": (None, [ctypes.c_int]),
    "zgo_keccak256": (None, [ctypes.c_char_p, _SZ, ctypes.c_char_p, ctypes.c_uint8]),
    "zgo_fr_ntt": (ctypes.c_int, [ctypes.c_char_p, _SZ, ctypes.c_int, _SZ, _SZ]),
    "zgo_fr_root_of_unity": (None, [ctypes.c_int, ctypes.c_char_p]),
    "zgo_fr_coset_factor": (None, [_SZ, _SZ, ctypes.c_char_p]),
    "zgo_tau_from_seed": (None, [ctypes.c_uint64, ctypes.c_char_p]),
    "zgo_fr_mul": (None, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p]),
    "zgo_g1_mul_gen": (None, [ctypes.c_char_p, ctypes.c_char_p]),
    "zgo_msm_g1": (None, [ctypes.c_char_p, ctypes.c_char_p, _SZ, ctypes.c_char_p]),
    "zgo_pairing_selftest": (ctypes.c_int, [ctypes.c_uint64]),
    "zgo_params_new": (_P, [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int]),
    "zgo_params_from_mont": (_P, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                  ctypes.POINTER(_SZ)]),
    "zgo_params_free": (None, [_P]),
    "zgo_params_mont": (_SZ, [_P, ctypes.c_int, ctypes.c_char_p, _SZ]),
    "zgo_param_points": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                        ctypes.c_int, ctypes.POINTER(ctypes.c_uint64), _SZ, ctypes.c_char_p]),
    "zgo_encode": (_P, [_P, ctypes.c_char_p, _SZ, ctypes.POINTER(ctypes.c_int)]),
    "zgo_blob_free": (None, [_P]),
    "zgo_blob_commitment": (None, [_P, ctypes.c_char_p]),
    "zgo_blob_roots": (None, [_P, ctypes.c_char_p]),
    "zgo_blob_file_root": (None, [_P, ctypes.c_char_p]),
    "zgo_blob_data": (None, [_P, ctypes.c_char_p]),
    "zgo_blob_slice": (_SZ, [_P, _SZ, ctypes.c_char_p, _SZ]),
    "zgo_blob_amt_outputs": (_SZ, [_P, ctypes.c_int, ctypes.c_char_p]),
    "zgo_amt_scalar_domain": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                             ctypes.c_char_p, ctypes.c_char_p]),
    "zgo_slice_verify": (ctypes.c_int, [_P, ctypes.c_char_p, _SZ, ctypes.c_char_p, ctypes.c_char_p,
                                        ctypes.POINTER(ctypes.c_int64)]),
    "zgo_merkle_roots": (None, [ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p]),
    "zgo_verify_params_new": (_P, [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_char_p]),
    "zgo_cpu_job_new": (_P, [_P, ctypes.c_char_p, _SZ]),
    "zgo_cpu_job_free": (None, [_P]),
    "zgo_cpu_job_step": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.POINTER(_SZ)]),
    "zgo_blob_all_slices": (_SZ, [_P, ctypes.c_char_p, _SZ]),
    "zgo_random_points": (None, [ctypes.c_uint64, _SZ, ctypes.c_char_p]),
    "zgo_recover": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64),
                                   ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(_SZ), _SZ,
                                   ctypes.c_char_p, ctypes.POINTER(_SZ), ctypes.c_char_p, _SZ]),
}

R_MOD = 21888242871839275222246405745257275088548364400416034343698204186575808495617
Q_MOD = 21888242871839275222246405745257275088696311157297823662689037894645226208583

# verifier result codes (oracle/zgo_capi.cpp)
V_OK = 0
V_UNMATCHED_AMT_INDEX = 1
V_UNMATCHED_MERKLE_INDEX = 2
V_AMT_INCORRECT_COMMITMENT = 10
V_AMT_INCORRECT_ROW_SIZE = 11
V_AMT_ROW_INDEX_OVERFLOW = 12
V_AMT_UNMATCHED_COSET_INDEX = 13
V_AMT_INCORRECT_PROOF = 14
V_MERKLE_INCORRECT_ROOT = 20
V_MERKLE_INCORRECT_SIZE = 21
V_MERKLE_ROW_INDEX_OVERFLOW = 22
V_MERKLE_INCORRECT_LOCAL_ROOT = 23
V_MERKLE_INCORRECT_PROOF = 24
V_DESERIALIZE = 30
P_UNEXPECTED_DATA_LENGTH, P_INCORRECT_POSITION, P_KZG, P_INCONSISTENT, P_LDT = range(5)


def build():
    subprocess.run(["make", "-C", ORACLE_DIR], check=True, stdout=subprocess.DEVNULL)
    return ORACLE_LIB


_LIB = None


def load():
    global _LIB
    if _LIB is None:
        build()
        L = ctypes.CDLL(ORACLE_LIB)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


class OracleParams:
    def __init__(self, L, handle, log_row, log_col, seed):
        self.L, self.h, self.log_row, self.log_col, self.seed = L, handle, log_row, log_col, seed

    def mont(self, coset):
        n = self.L.zgo_params_mont(self.h, coset, None, 0)
        buf = ctypes.create_string_buffer(n)
        self.L.zgo_params_mont(self.h, coset, buf, n)
        return buf.raw

    def __del__(self):
        try:
            self.L.zgo_params_free(self.h)
        except Exception:
            pass


class OracleBlob:
    def __init__(self, L, handle, log_row, log_col):
        self.L, self.h, self.log_row, self.log_col = L, handle, log_row, log_col

    def commitment(self):
        b = ctypes.create_string_buffer(64)
        self.L.zgo_blob_commitment(self.h, b)
        return b.raw

    def roots(self):
        b = ctypes.create_string_buffer(96)
        self.L.zgo_blob_roots(self.h, b)
        return b.raw

    def file_root(self):
        b = ctypes.create_string_buffer(32)
        self.L.zgo_blob_file_root(self.h, b)
        return b.raw

    def data(self):
        n = 3 * (1 << (self.log_row + self.log_col)) * 32
        b = ctypes.create_string_buffer(n)
        self.L.zgo_blob_data(self.h, b)
        return b.raw

    def slice(self, i):
        n = self.L.zgo_blob_slice(self.h, i, None, 0)
        b = ctypes.create_string_buffer(n)
        self.L.zgo_blob_slice(self.h, i, b, n)
        return b.raw

    def all_slices(self):
        """Every serialized slice, back to back, as one bytes object."""
        n = self.L.zgo_blob_all_slices(self.h, None, 0)
        b = ctypes.create_string_buffer(n)
        assert self.L.zgo_blob_all_slices(self.h, b, n) == n
        return b.raw

    def amt_outputs(self, coset):
        n = self.L.zgo_blob_amt_outputs(self.h, coset, None)
        b = ctypes.create_string_buffer(64 * n)
        self.L.zgo_blob_amt_outputs(self.h, coset, b)
        return b.raw

    def __del__(self):
        try:
            self.L.zgo_blob_free(self.h)
        except Exception:
            pass


class CpuJob:
    def __init__(self, L, handle):
        self.L, self.h = L, handle

    def step(self):
        """Runs one coset step; returns (coset, file_root or None, reply bytes)."""
        root = ctypes.create_string_buffer(32)
        nbytes = ctypes.c_size_t()
        c = self.L.zgo_cpu_job_step(self.h, root, ctypes.byref(nbytes))
        assert c >= 0, "payload too large"
        return c, (root.raw if c == 2 else None), nbytes.value

    def __del__(self):
        try:
            self.L.zgo_cpu_job_free(self.h)
        except Exception:
            pass


class TooLargeBlob(Exception):
    pass


class Oracle:
    def __init__(self):
        self.L = load()

    def params(self, log_row, log_col, seed, ec_domain=False):
        h = self.L.zgo_params_new(log_row, log_col, seed, 1 if ec_domain else 0)
        return OracleParams(self.L, h, log_row, log_col, seed)

    def params_from_mont(self, log_row, log_col, files):
        arr = (ctypes.c_char_p * 3)(*files)
        lens = (ctypes.c_size_t * 3)(*[len(f) for f in files])
        h = self.L.zgo_params_from_mont(log_row, log_col, arr, lens)
        assert h, "malformed params"
        return OracleParams(self.L, h, log_row, log_col, None)

    def encode(self, params, data: bytes):
        err = ctypes.c_int()
        h = self.L.zgo_encode(params.h, data, len(data), ctypes.byref(err))
        if err.value == 1:
            raise TooLargeBlob(len(data))
        return OracleBlob(self.L, h, params.log_row, params.log_col)

    def verify_params(self, log_row, log_col, seed, basis_lines: bytes):
        h = self.L.zgo_verify_params_new(log_row, log_col, seed, basis_lines)
        return OracleParams(self.L, h, log_row, log_col, seed)

    def merkle_roots(self, log_row, log_col, items: bytes):
        out = ctypes.create_string_buffer(96)
        self.L.zgo_merkle_roots(log_row, log_col, items, out)
        return out.raw

    def verify(self, params, slice_bytes, commitment, root):
        det = (ctypes.c_int64 * 4)()
        rc = self.L.zgo_slice_verify(params.h, slice_bytes, len(slice_bytes), commitment, root, det)
        return rc, list(det)

    def keccak256(self, data: bytes, pad=0x01):
        out = ctypes.create_string_buffer(32)
        self.L.zgo_keccak256(data, len(data), out, pad)
        return out.raw

    def ntt(self, data: bytes, inverse=False, coset_idx=0, coset_len=0):
        n = len(data) // 32
        buf = ctypes.create_string_buffer(data, len(data))
        rc = self.L.zgo_fr_ntt(buf, n, 1 if inverse else 0, coset_idx, coset_len)
        assert rc == 0
        return buf.raw

    def root_of_unity(self, log_n):
        out = ctypes.create_string_buffer(32)
        self.L.zgo_fr_root_of_unity(log_n, out)
        return int.from_bytes(out.raw, "little")

    def coset_factor(self, length, idx):
        out = ctypes.create_string_buffer(32)
        self.L.zgo_fr_coset_factor(length, idx, out)
        return int.from_bytes(out.raw, "little")

    def tau(self, seed):
        out = ctypes.create_string_buffer(32)
        self.L.zgo_tau_from_seed(seed, out)
        return int.from_bytes(out.raw, "little")

    def g1_mul_gen(self, k: int):
        out = ctypes.create_string_buffer(64)
        self.L.zgo_g1_mul_gen(k.to_bytes(32, "little"), out)
        return out.raw

    def msm(self, bases_mont: bytes, scalars: bytes):
        n = len(scalars) // 32
        out = ctypes.create_string_buffer(64)
        self.L.zgo_msm_g1(bases_mont, scalars, n, out)
        return out.raw

    def param_points(self, log_row, log_col, seed, coset, line, idx):
        arr = (ctypes.c_uint64 * len(idx))(*idx)
        out = ctypes.create_string_buffer(64 * len(idx))
        self.L.zgo_param_points(log_row, log_col, seed, coset, line, arr, len(idx), out)
        return out.raw

    def amt_scalar_domain(self, log_row, log_col, seed, coset, coset_rows: bytes):
        R = 1 << log_row
        out = ctypes.create_string_buffer(64 * (4 * R - 2))
        n = self.L.zgo_amt_scalar_domain(log_row, log_col, seed, coset, coset_rows, out)
        assert n == 4 * R - 2
        return out.raw

    def random_points(self, seed, n):
        out = ctypes.create_string_buffer(64 * n)
        self.L.zgo_random_points(seed, n, out)
        return out.raw

    def cpu_job(self, params, data: bytes):
        """Step-wise full-blob run of the restated CPU encode path (one coset
        per step, three steps per blob; see oracle/zgo_capi.cpp)."""
        return CpuJob(self.L, self.L.zgo_cpu_job_new(params.h, data, len(data)))

    def recover(self, log_row, log_col, rows: dict):
        ids = sorted(rows)
        n = len(ids)
        arr = (ctypes.c_uint64 * n)(*ids)
        bufs = (ctypes.c_char_p * n)(*[rows[i] for i in ids])
        lens = (ctypes.c_size_t * n)(*[len(rows[i]) for i in ids])
        out = ctypes.create_string_buffer(31 * (1 << (log_row + log_col)))
        out_len = ctypes.c_size_t()
        msg = ctypes.create_string_buffer(256)
        rc = self.L.zgo_recover(log_row, log_col, arr, bufs, lens, n, out, ctypes.byref(out_len), msg, 256)
        if rc:
            return rc, msg.value.decode()
        return 0, out.raw[:out_len.value]
