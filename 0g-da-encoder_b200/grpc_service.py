"""gRPC `encoder.Encoder/EncodeBlob` served by the B200 encoder.

The reference serves this RPC with tonic (grpc/proto/encoder.proto:5-21,
grpc/src/service.rs:47-65, grpc/src/lib.rs:11-28): one request carries the
payload and `require_data`, the reply the `EncodeBlobReply` fields, an encoder
error becomes status UNKNOWN with the error's Debug text, and messages may be
up to 1 GiB. This module serves the same service name, method, message field
numbers and error mapping, so a client of the reference talks to it
unchanged. The message classes are built at import time from a descriptor
written here (no generated code, no protoc). Requests go through the C ABI's
request pipeline (zg_submit / zg_wait): concurrent RPCs share the GPU, one
blob's copies overlapping another's compute.
"""
from concurrent import futures

import grpc
from google.protobuf import descriptor_pb2, descriptor_pool, message_factory

SERVICE = "encoder.Encoder"
METHOD = "/encoder.Encoder/EncodeBlob"
MESSAGE_SIZE_LIMIT = 1 << 30  # MESSAGE_SIZE_LIMIT, grpc/src/lib.rs:11
DEFAULT_ADDRESS = "0.0.0.0:34000"  # run/config.toml:3


def _message_classes():
    F = descriptor_pb2.FieldDescriptorProto
    fd = descriptor_pb2.FileDescriptorProto(name="encoder.proto", package="encoder", syntax="proto3")
    req = fd.message_type.add(name="EncodeBlobRequest")
    req.field.add(name="data", number=1, type=F.TYPE_BYTES, label=F.LABEL_OPTIONAL)
    req.field.add(name="require_data", number=2, type=F.TYPE_BOOL, label=F.LABEL_OPTIONAL)
    rep = fd.message_type.add(name="EncodeBlobReply")
    rep.field.add(name="version", number=1, type=F.TYPE_UINT32, label=F.LABEL_OPTIONAL)
    rep.field.add(name="erasure_commitment", number=2, type=F.TYPE_BYTES, label=F.LABEL_OPTIONAL)
    rep.field.add(name="storage_root", number=3, type=F.TYPE_BYTES, label=F.LABEL_OPTIONAL)
    rep.field.add(name="encoded_data", number=4, type=F.TYPE_BYTES, label=F.LABEL_OPTIONAL)
    rep.field.add(name="encoded_slice", number=5, type=F.TYPE_BYTES, label=F.LABEL_REPEATED)
    svc = fd.service.add(name="Encoder")
    svc.method.add(name="EncodeBlob", input_type=".encoder.EncodeBlobRequest", output_type=".encoder.EncodeBlobReply")
    pool = descriptor_pool.DescriptorPool()
    pool.Add(fd)
    return (message_factory.GetMessageClass(pool.FindMessageTypeByName("encoder.EncodeBlobRequest")),
            message_factory.GetMessageClass(pool.FindMessageTypeByName("encoder.EncodeBlobReply")))


EncodeBlobRequest, EncodeBlobReply = _message_classes()


class EncoderServicer:
    """EncoderService::encode_blob (grpc/src/service.rs:47-65). `service` is
    anything with submit(data, require_data) / wait(ticket) returning a reply
    with the EncodeBlobReply fields: the package's EncoderService."""

    def __init__(self, service):
        self.service = service

    def EncodeBlob(self, request, context):
        from . import EncoderError  # TooLargeBlob and friends
        try:
            r = self.service.wait(self.service.submit(request.data, request.require_data))
        except EncoderError as e:
            # .map_err(|e| Status::new(Code::Unknown, e)) with e = format!("{:?}", err)
            context.abort(grpc.StatusCode.UNKNOWN, str(e))
        return EncodeBlobReply(version=r.version, erasure_commitment=r.erasure_commitment,
                               storage_root=r.storage_root, encoded_data=r.encoded_data,
                               encoded_slice=list(r.encoded_slice))


def add_to_server(servicer: EncoderServicer, server: grpc.Server):
    handler = grpc.method_handlers_generic_handler(SERVICE, {
        "EncodeBlob": grpc.unary_unary_rpc_method_handler(
            servicer.EncodeBlob, request_deserializer=EncodeBlobRequest.FromString,
            response_serializer=EncodeBlobReply.SerializeToString),
    })
    server.add_generic_rpc_handlers((handler,))


def _options():
    return [("grpc.max_send_message_length", MESSAGE_SIZE_LIMIT),
            ("grpc.max_receive_message_length", MESSAGE_SIZE_LIMIT)]


def serve(service, address: str = DEFAULT_ADDRESS, workers: int = 8):
    """Start a server for `service` (run_server, grpc/src/lib.rs:13-28).
    Returns (server, port), the server started; the caller stops it
    (server.stop(grace)). Port 0 in `address` picks a free port."""
    server = grpc.server(futures.ThreadPoolExecutor(max_workers=workers), options=_options())
    add_to_server(EncoderServicer(service), server)
    port = server.add_insecure_port(address)
    if port == 0:
        raise RuntimeError(f"cannot bind {address}")
    server.start()
    return server, port


class Client:
    """EncodeBlob over a channel: Client(address).encode_blob(data, require_data)."""

    def __init__(self, address: str):
        self.channel = grpc.insecure_channel(address, options=_options())
        self.call = self.channel.unary_unary(METHOD, request_serializer=EncodeBlobRequest.SerializeToString,
                                             response_deserializer=EncodeBlobReply.FromString)

    def encode_blob(self, data: bytes, require_data: bool, timeout=None):
        return self.call(EncodeBlobRequest(data=data, require_data=require_data), timeout=timeout)

    def close(self):
        self.channel.close()
