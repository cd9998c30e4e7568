"""gRPC EncodeBlob served by the B200 encoder: every reply equals
EncoderService::process_data's bytes and the oracle's, also under concurrent
requests; oversized payloads fail as the reference's server does."""
import importlib
import threading

import grpc
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_grpc_encode_blob_matches_process_data(gpu_pkg, oracle):
    gs = importlib.import_module(gpu_pkg.__name__ + ".grpc_service")
    params = gpu_pkg.ZgEncoderParams.from_seed(4, 6, 13)
    op = oracle.params(4, 6, 13)
    svc = gpu_pkg.EncoderService(params)
    server, port = gs.serve(svc, "127.0.0.1:0", workers=4)
    try:
        client = gs.Client(f"127.0.0.1:{port}")
        rng = np.random.default_rng(31)
        sizes = [0, 1, 777, params.dims.max_raw_data_size]
        payloads = [rng.integers(0, 256, size=n, dtype=np.uint8).tobytes() for n in sizes]
        got = [None] * len(payloads)

        def call(i):
            got[i] = client.encode_blob(payloads[i], i % 2 == 0, timeout=120)

        ts = [threading.Thread(target=call, args=(i,)) for i in range(len(payloads))]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        for i, data in enumerate(payloads):
            exp = svc.process_data(data, i % 2 == 0)
            r = got[i]
            assert r.version == exp.version == 0
            assert r.erasure_commitment == exp.erasure_commitment
            assert r.storage_root == exp.storage_root
            assert r.encoded_data == exp.encoded_data
            assert list(r.encoded_slice) == list(exp.encoded_slice)
            ob = oracle.encode(op, data)
            assert r.storage_root == ob.file_root() and r.erasure_commitment == ob.commitment()
        with pytest.raises(grpc.RpcError) as ei:
            client.encode_blob(bytes(params.dims.max_raw_data_size + 1), False, timeout=60)
        assert ei.value.code() == grpc.StatusCode.UNKNOWN
        assert ei.value.details().startswith("TooLargeBlob { actual: ")
        client.close()
    finally:
        server.stop(0)
        params.close()
