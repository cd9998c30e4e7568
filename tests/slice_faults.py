"""Corruptions of a serialized EncodedSlice and the VerifierError each must
produce: the reference's fault-injection table (gen_err_signer_map /
get_invalid_row, crates/encoder/src/encoder/blob.rs:84-229, amt/blob.rs:61-96,
merkle/blob.rs:60-106). Shared by the oracle tests and the GPU verifier tests."""
import os
import sys

import zgo

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as mg  # noqa: E402


def slice_layout(lr, lc):
    C = 1 << lc
    a = 96 + 32 * C
    h = a + 8 + 128 * lr
    m = h + 64
    t = m + 104 + 32 * lr
    return {"row": 96, "proof": a + 8, "high": h, "merkle": m, "mproof": m + 104, "leaf_index": t,
            "leaf": t + 8, "end": t + 40}


def parse_g1(b):
    if b[63] & 0x40:
        return None
    y = bytearray(b[32:])
    y[31] &= 0x3F
    return int.from_bytes(b[:32], "little"), int.from_bytes(bytes(y), "little")


def bump(h):  # H256::from_low_u64_be(H256(h).to_low_u64_be() + 1)
    return bytes(24) + ((int.from_bytes(h[24:], "big") + 1) & ((1 << 64) - 1)).to_bytes(8, "big")


def fault_cases(slices, index, log_row, log_col):
    """(corrupted bytes, code, sub, a, b, c) for slice `index` of a blob."""
    R = 1 << log_row
    lay = slice_layout(log_row, log_col)
    s = slices[index]
    coset, local = divmod(index, R)
    u64 = lambda v: v.to_bytes(8, "little")
    out = [(u64(index + 1) + s[8:], zgo.V_UNMATCHED_AMT_INDEX, 0, index + 1, index, 0)]
    if index < 3 * R - 1:
        nxt = slices[index + 1]
        out.append((s[:8] + nxt[8:lay["merkle"]] + s[lay["merkle"]:], zgo.V_UNMATCHED_AMT_INDEX, 0, index,
                    index + 1, 0))
        out.append((s[:lay["merkle"]] + nxt[lay["merkle"]:], zgo.V_UNMATCHED_MERKLE_INDEX, 0, index, index + 1, 0))
    # AMT: WrongRow
    row0 = (int.from_bytes(s[96:128], "little") + 1) % zgo.R_MOD
    out.append((s[:96] + row0.to_bytes(32, "little") + s[128:], zgo.V_AMT_INCORRECT_PROOF, zgo.P_INCONSISTENT,
                coset, local, 0))
    # AMT: WrongIndex (row.index += 1)
    out.append((s[:80] + u64(local + 1) + s[88:], zgo.V_AMT_UNMATCHED_COSET_INDEX, 0, coset, local, local + 1))
    # AMT: WrongCommitment (commitment + G1)
    bad_com = mg.ser_g1(mg.g1_add(parse_g1(s[16:80]), mg.G1))
    out.append((s[:16] + bad_com + s[80:], zgo.V_AMT_INCORRECT_COMMITMENT, 0, 0, 0, 0))
    # AMT: IncorrectHighCommitment (high + G1)
    h = lay["high"]
    bad_high = mg.ser_g1(mg.g1_add(parse_g1(s[h:h + 64]), mg.G1))
    out.append((s[:h] + bad_high + s[h + 64:], zgo.V_AMT_INCORRECT_PROOF, zgo.P_LDT, coset, local, 0))
    # Merkle: WrongIndex (leaf_index += 1)
    li = lay["leaf_index"]
    out.append((s[:li] + u64(index + 1) + s[li + 8:], zgo.V_UNMATCHED_MERKLE_INDEX, 0, index, index + 1, 0))
    # Merkle: WrongLocalRoot
    lf = lay["leaf"]
    out.append((s[:lf] + bump(s[lf:lf + 32]), zgo.V_MERKLE_INCORRECT_LOCAL_ROOT, 0, index, 0, 0))
    # Merkle: WrongProof (proof[0])
    mp = lay["mproof"]
    out.append((s[:mp] + bump(s[mp:mp + 32]) + s[mp + 32:], zgo.V_MERKLE_INCORRECT_PROOF, 0, index, 0, 0))
    # Merkle: WrongRoot (every root)
    m = lay["merkle"]
    roots = b"".join(bump(s[m + 32 * k:m + 32 * k + 32]) for k in range(3))
    out.append((s[:m] + roots + s[m + 96:], zgo.V_MERKLE_INCORRECT_ROOT, 0, 0, 0, 0))
    return out
