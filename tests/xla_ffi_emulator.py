"""A stand-in for the XLA runtime side of the FFI C ABI, in ctypes: builds
the call frame XLA hands a custom-call handler (buffers, results, scalar
attributes sorted by name, execution stage) and an API table whose error,
stream and device-memory functions are Python callbacks. Used by the tests
to call libsbh_b200's XLA handlers (include/sbh_xla_ffi.h) the way XLA
would, without jax or jaxlib.

The struct layouts are those of XLA's FFI C API, version 0.1, which the
library's handlers are written against (barnes-hut_b200/csrc/sbh_xla_ffi_abi.h)."""
import ctypes
from ctypes import POINTER, c_char_p, c_int, c_int64, c_size_t, c_uint32, c_void_p

import numpy as np

DT_S32, DT_U8, DT_F32 = 4, 6, 11
ARG_BUFFER = RET_BUFFER = 1
ATTR_SCALAR = 3
STAGE_EXECUTE = 3
EXT_METADATA = 1
ERR_INVALID_ARGUMENT, ERR_RESOURCE_EXHAUSTED, ERR_INTERNAL = 3, 8, 13


class ExtBase(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("type", c_int), ("next", c_void_p)]


class ApiVersion(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("major_version", c_int),
                ("minor_version", c_int)]


class Buffer(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("dtype", c_int), ("data", c_void_p),
                ("rank", c_int64), ("dims", POINTER(c_int64))]


class Args(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("size", c_int64),
                ("types", POINTER(c_int)), ("args", POINTER(c_void_p))]


class Rets(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("size", c_int64),
                ("types", POINTER(c_int)), ("rets", POINTER(c_void_p))]


class ByteSpan(ctypes.Structure):
    _fields_ = [("ptr", c_char_p), ("len", c_size_t)]


class Scalar(ctypes.Structure):
    _fields_ = [("dtype", c_int), ("value", c_void_p)]


class Attrs(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("size", c_int64),
                ("types", POINTER(c_int)), ("names", POINTER(POINTER(ByteSpan))), ("attrs", POINTER(c_void_p))]


class CallFrame(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("api", c_void_p), ("ctx", c_void_p),
                ("stage", c_int), ("args", Args), ("rets", Rets), ("attrs", Attrs)]


class Metadata(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("api_version", ApiVersion), ("traits", c_uint32)]


class MetadataExt(ctypes.Structure):
    _fields_ = [("extension_base", ExtBase), ("metadata", POINTER(Metadata))]


class ErrorCreateArgs(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("message", c_char_p), ("errc", c_int)]


class StreamGetArgs(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("ctx", c_void_p), ("stream", c_void_p)]


class AllocArgs(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("ctx", c_void_p), ("size", c_size_t),
                ("alignment", c_size_t), ("data", c_void_p)]


class FreeArgs(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("ctx", c_void_p), ("size", c_size_t),
                ("data", c_void_p)]


ERROR_CREATE = ctypes.CFUNCTYPE(c_void_p, POINTER(ErrorCreateArgs))
STREAM_GET = ctypes.CFUNCTYPE(c_void_p, POINTER(StreamGetArgs))
ALLOC = ctypes.CFUNCTYPE(c_void_p, POINTER(AllocArgs))
FREE = ctypes.CFUNCTYPE(c_void_p, POINTER(FreeArgs))


class Api(ctypes.Structure):
    _fields_ = [("struct_size", c_size_t), ("extension_start", c_void_p), ("api_version", ApiVersion),
                ("internal_api", c_void_p), ("error_create", ERROR_CREATE), ("error_get_message", c_void_p),
                ("error_destroy", c_void_p), ("handler_register", c_void_p), ("stream_get", STREAM_GET),
                ("type_id_register", c_void_p), ("execution_context_get", c_void_p), ("state_set", c_void_p),
                ("state_get", c_void_p), ("device_memory_allocate", ALLOC), ("device_memory_free", FREE)]


class HandlerError(Exception):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code, self.message = code, message


class FakeXla:
    """The runtime half: errors, stream and (optionally) device scratch.

    stream: the CUDA stream handle the handlers receive (an int).
    allocate: callable(size) -> (device pointer, keep-alive object), or None
      for a runtime whose API table ends before XLA_FFI_DeviceMemory_Allocate
      (the handlers then take scratch from cudaMallocAsync)."""

    def __init__(self, stream: int = 0, allocate=None):
        self.stream = stream
        self.errors = {}
        self.live = {}
        self.allocations = 0
        self._allocate = allocate
        self._cb = [ERROR_CREATE(self._error_create), STREAM_GET(self._stream_get), ALLOC(self._alloc), FREE(self._free)]
        self.api = Api()
        self.api.api_version = ApiVersion(ctypes.sizeof(ApiVersion), None, 0, 1)
        self.api.error_create, self.api.stream_get = self._cb[0], self._cb[1]
        if allocate is not None:
            self.api.device_memory_allocate, self.api.device_memory_free = self._cb[2], self._cb[3]
            self.api.struct_size = ctypes.sizeof(Api)
        else:
            self.api.struct_size = Api.device_memory_allocate.offset

    def _error_create(self, a):
        key = 0x1000 + 16 * len(self.errors)
        self.errors[key] = (a.contents.errc, a.contents.message.decode())
        return key

    def _stream_get(self, a):
        a.contents.stream = self.stream
        return None

    def _alloc(self, a):
        ptr, keep = self._allocate(int(a.contents.size))
        self.live[ptr] = keep
        self.allocations += 1
        a.contents.data = ptr
        return None

    def _free(self, a):
        self.live.pop(int(a.contents.data), None)
        return None

    def call(self, fn, args, rets, attrs, stage=STAGE_EXECUTE):
        """fn: the handler (ctypes function). args / rets: (dtype code, data
        pointer, shape) triples. attrs: name -> np.int32 / np.float32 value.
        Raises HandlerError when the handler returns an error."""
        keep = []

        def buffers(items):
            out = (c_void_p * max(len(items), 1))()
            types = (c_int * max(len(items), 1))()
            for i, (dt, ptr, shape) in enumerate(items):
                dims = (c_int64 * max(len(shape), 1))(*shape)
                b = Buffer(ctypes.sizeof(Buffer), None, dt, ptr, len(shape), dims)
                keep.extend([dims, b])
                out[i] = ctypes.addressof(b)
                types[i] = ARG_BUFFER
            keep.extend([out, types])
            return types, out

        at, aa = buffers(args)
        rt, rr = buffers(rets)
        names = sorted(attrs)
        n = len(names)
        ntypes = (c_int * max(n, 1))()
        nspans = (POINTER(ByteSpan) * max(n, 1))()
        nvals = (c_void_p * max(n, 1))()
        for i, name in enumerate(names):
            v = attrs[name]
            if isinstance(v, np.int32) or isinstance(v, int):
                cv, dt = ctypes.c_int32(int(v)), DT_S32
            else:
                cv, dt = ctypes.c_float(float(v)), DT_F32
            raw = name.encode()
            span = ByteSpan(raw, len(raw))
            sc = Scalar(dt, ctypes.cast(ctypes.pointer(cv), c_void_p))
            keep.extend([cv, raw, span, sc])
            ntypes[i] = ATTR_SCALAR
            nspans[i] = ctypes.pointer(span)
            nvals[i] = ctypes.addressof(sc)
        frame = CallFrame()
        frame.struct_size = ctypes.sizeof(CallFrame)
        frame.api = ctypes.addressof(self.api)
        frame.ctx = 0x42
        frame.stage = stage
        frame.args = Args(ctypes.sizeof(Args), None, len(args), at, aa)
        frame.rets = Rets(ctypes.sizeof(Rets), None, len(rets), rt, rr)
        frame.attrs = Attrs(ctypes.sizeof(Attrs), None, n, ntypes, nspans, nvals)
        fn.restype = c_void_p
        fn.argtypes = [c_void_p]
        err = fn(ctypes.addressof(frame))
        if err:
            code, msg = self.errors[err]
            raise HandlerError(code, msg)

    @staticmethod
    def metadata(fn):
        """The registration-time metadata query: returns (major, minor, traits)."""
        md = Metadata()
        md.struct_size = ctypes.sizeof(Metadata)
        ext = MetadataExt(ExtBase(ctypes.sizeof(MetadataExt), EXT_METADATA, None), ctypes.pointer(md))
        frame = CallFrame()
        frame.struct_size = ctypes.sizeof(CallFrame)
        frame.extension_start = ctypes.addressof(ext)
        fn.restype = c_void_p
        fn.argtypes = [c_void_p]
        err = fn(ctypes.addressof(frame))
        assert not err
        return md.api_version.major_version, md.api_version.minor_version, md.traits
