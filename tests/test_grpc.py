"""The gRPC drop-in (encoder.Encoder/EncodeBlob): wire format of the
reference's proto (grpc/proto/encoder.proto:5-21), the service wiring and the
error mapping (grpc/src/service.rs:47-65), on CPU with a stand-in encoder."""
import importlib
import threading

import grpc
import pytest


@pytest.fixture(scope="module")
def gs(pkg):
    return importlib.import_module(pkg.__name__ + ".grpc_service")


def test_wire_format_matches_the_proto(gs):
    # field 1 bytes (tag 0x0a), field 2 bool (tag 0x10)
    assert gs.EncodeBlobRequest(data=b"ab", require_data=True).SerializeToString() == b"\x0a\x02ab\x10\x01"
    r = gs.EncodeBlobReply(version=3, erasure_commitment=b"c", storage_root=b"r", encoded_data=b"d",
                           encoded_slice=[b"s0", b"s1"])
    assert r.SerializeToString() == (b"\x08\x03" + b"\x12\x01c" + b"\x1a\x01r" + b"\x22\x01d"
                                     + b"\x2a\x02s0" + b"\x2a\x02s1")
    back = gs.EncodeBlobReply.FromString(r.SerializeToString())
    assert list(back.encoded_slice) == [b"s0", b"s1"] and back.version == 3


class _Reply:
    def __init__(self, data, require_data):
        self.version = 0
        self.erasure_commitment = bytes(64)
        self.storage_root = data[:32].ljust(32, b"\0")
        self.encoded_data = data if require_data else b""
        self.encoded_slice = [data[::-1], data]


class _StandIn:
    """submit / wait with the package's error behaviour and no GPU."""

    def __init__(self, pkg, limit):
        self.pkg, self.limit, self.calls = pkg, limit, 0
        self.lock = threading.Lock()

    def submit(self, data, require_data):
        with self.lock:
            self.calls += 1
        if len(data) > self.limit:
            raise self.pkg.TooLargeBlob(len(data), self.limit)
        return (data, require_data)

    def wait(self, ticket):
        return _Reply(*ticket)


def test_server_round_trip_and_errors(pkg, gs):
    svc = _StandIn(pkg, limit=1000)
    server, port = gs.serve(svc, "127.0.0.1:0", workers=4)
    try:
        c = gs.Client(f"127.0.0.1:{port}")
        rep = c.encode_blob(b"hello payload", True, timeout=30)
        assert rep.version == 0 and rep.encoded_data == b"hello payload"
        assert list(rep.encoded_slice) == [b"daolyap olleh", b"hello payload"]
        assert c.encode_blob(b"x", False, timeout=30).encoded_data == b""
        with pytest.raises(grpc.RpcError) as ei:
            c.encode_blob(bytes(1001), True, timeout=30)
        assert ei.value.code() == grpc.StatusCode.UNKNOWN
        assert ei.value.details() == "TooLargeBlob { actual: 1001, expected_max: 1000 }"
        # concurrent calls, each gets its own reply
        outs = {}

        def call(i):
            outs[i] = c.encode_blob(bytes([i]) * (i + 1), True, timeout=30).encoded_data

        ts = [threading.Thread(target=call, args=(i,)) for i in range(8)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        assert all(outs[i] == bytes([i]) * (i + 1) for i in range(8))
        c.close()
    finally:
        server.stop(0)
