"""Calling MEX functions through the MEX runtime stand-in from Python.

TEST INFRASTRUCTURE ONLY: used by ``tests/`` (the reference's own MEX kernels
as the oracle's pin, this repository's gateways as the drop-in under test)
and by ``bench.py --impl reference`` (the reference's GPU kernels timed on the
same device).  gpuArray inputs wrap CUDA torch tensors in place; host inputs
are copied in column-major order; MEX errors come back as ``MexError`` with
the identifier the function raised.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

CLASS = dict(double=6, single=7, int8=8, uint8=9, int16=10, uint16=11, int32=12, uint32=13, int64=14, uint64=15,
             logical=3, char=4, struct=2)
_NP = {6: np.float64, 7: np.float32, 8: np.int8, 9: np.uint8, 10: np.int16, 11: np.uint16, 12: np.int32,
       13: np.uint32, 14: np.int64, 15: np.uint64, 3: np.bool_}
_FROM_NP = {np.dtype(np.float64): (6, 0), np.dtype(np.float32): (7, 0), np.dtype(np.complex128): (6, 1),
            np.dtype(np.complex64): (7, 1), np.dtype(np.int32): (12, 0), np.dtype(np.uint8): (9, 0),
            np.dtype(np.uint64): (15, 0), np.dtype(np.int64): (14, 0), np.dtype(np.bool_): (3, 0)}


class MexError(RuntimeError):
    def __init__(self, identifier: str, message: str):
        super().__init__(f"{identifier}: {message}")
        self.identifier = identifier
        self.message = message


class MxArray:
    """An mxArray owned by Python (destroyed with the object unless handed to a MEX call)."""

    def __init__(self, rt: "MexRuntime", ptr: int, keep=None, owned: bool = True):
        self.rt, self.ptr, self._keep, self.owned = rt, ptr, keep, owned

    def __del__(self):
        if getattr(self, "owned", False) and self.ptr:
            self.rt.lib.mexshim_destroy(C.c_void_p(self.ptr))
            self.ptr = None

    def info(self):
        g, c, x, nd = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        dims = (C.c_size_t * 8)()
        kind = self.rt.lib.mexshim_info(C.c_void_p(self.ptr), C.byref(g), C.byref(c), C.byref(x), C.byref(nd), dims, 8)
        return dict(kind=kind, gpu=bool(g.value), cls=c.value, complex=bool(x.value),
                    dims=tuple(dims[i] for i in range(nd.value)))

    @property
    def dims(self):
        return self.info()["dims"]

    def numpy(self) -> np.ndarray:
        """A host copy in MATLAB shape (column-major data, NumPy array of the same shape)."""
        inf = self.info()
        dtype = np.dtype(_NP[inf["cls"]])
        if inf["complex"]:
            dtype = np.dtype(np.complex64 if dtype == np.float32 else np.complex128)
        n = int(np.prod(inf["dims"]))
        out = np.empty(n, dtype)
        ptr = self.rt.lib.mexshim_data(C.c_void_p(self.ptr))
        if n:
            if inf["gpu"]:
                import torch
                t = torch.as_tensor(_Cai(ptr, (n,), dtype), device="cuda")
                out[:] = t.cpu().numpy()
            else:
                C.memmove(out.ctypes.data, ptr, out.nbytes)
        return out.reshape(inf["dims"], order="F")

    def torch(self):
        """A CUDA torch view of a gpuArray, shaped like MATLAB (column-major strides); keeps this object alive."""
        import torch
        inf = self.info()
        if not inf["gpu"]:
            raise ValueError("not a gpuArray")
        dtype = np.dtype(_NP[inf["cls"]])
        if inf["complex"]:
            dtype = np.dtype(np.complex64 if dtype == np.float32 else np.complex128)
        ptr = self.rt.lib.mexshim_data(C.c_void_p(self.ptr))
        t = torch.as_tensor(_Cai(ptr, tuple(reversed(inf["dims"])), dtype, owner=self), device="cuda")
        return t.permute(*reversed(range(t.dim())))

    def field(self, name: str) -> "MxArray":
        p = self.rt.lib.mexshim_field(C.c_void_p(self.ptr), name.encode())
        if not p:
            raise KeyError(name)
        return MxArray(self.rt, p, keep=self, owned=False)

    def scalar(self) -> float:
        return float(self.numpy().ravel()[0])


class _Cai:
    def __init__(self, ptr, shape, dtype, owner=None):
        self.__cuda_array_interface__ = dict(shape=tuple(shape), typestr=np.dtype(dtype).str, data=(ptr, False),
                                             version=3, strides=None)
        self._owner = owner


class MexRuntime:
    """The stand-in runtime (oracle/_ref/libmexshim.so) and the MEX libraries loaded into it."""

    def __init__(self):
        path = _build.build_shim()
        self.lib = C.CDLL(path, mode=C.RTLD_GLOBAL)
        L = self.lib
        L.mexshim_gpu_wrap.restype = C.c_void_p
        L.mexshim_gpu_wrap.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t), C.c_int, C.c_int]
        L.mexshim_host_array.restype = C.c_void_p
        L.mexshim_host_array.argtypes = [C.c_int, C.POINTER(C.c_size_t), C.c_int, C.c_int, C.c_void_p]
        L.mexshim_string.restype = C.c_void_p
        L.mexshim_string.argtypes = [C.c_char_p]
        L.mexshim_struct.restype = C.c_void_p
        L.mexshim_struct.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_void_p)]
        L.mexshim_call.restype = C.c_int
        L.mexshim_call.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p),
                                   C.c_char_p, C.c_char_p, C.c_int]
        L.mexshim_info.restype = C.c_int
        L.mexshim_data.restype = C.c_void_p
        L.mexshim_data.argtypes = [C.c_void_p]
        L.mexshim_field.restype = C.c_void_p
        L.mexshim_field.argtypes = [C.c_void_p, C.c_char_p]
        L.mexshim_destroy.argtypes = [C.c_void_p]
        L.mexshim_live_device_bytes.restype = C.c_longlong
        L.mexshim_clear.restype = C.c_int
        self._mex = {}

    def load(self, path: str):
        """A MEX library's mexFunction."""
        if path not in self._mex:
            lib = C.CDLL(path)
            self._mex[path] = (lib, C.cast(lib.mexFunction, C.c_void_p).value)
        return self._mex[path][1]

    # -- inputs -------------------------------------------------------------
    def gpu(self, tensor, dims=None) -> MxArray:
        """A gpuArray over a CUDA tensor's memory.  ``dims`` are the MATLAB
        dimensions; the tensor's memory must be column-major for them (a
        contiguous tensor with the dimensions reversed, or its permuted view)."""
        import torch
        t = tensor
        if dims is None:
            dims = tuple(t.shape)
            if t.dim() > 1 and not t.permute(*reversed(range(t.dim()))).is_contiguous():
                raise ValueError("tensor memory is not column-major for its shape")
        if t.dtype in (torch.complex64, torch.complex128):
            cls, cplx = (7 if t.dtype == torch.complex64 else 6), 1
        else:
            cls, cplx = {torch.float32: 7, torch.float64: 6, torch.int32: 12, torch.uint8: 9,
                         torch.bool: 3}[t.dtype], 0
        d = (C.c_size_t * len(dims))(*dims)
        p = self.lib.mexshim_gpu_wrap(C.c_void_p(t.data_ptr()), len(dims), d, cls, cplx)
        return MxArray(self, p, keep=t)

    def host(self, a, cls: str | None = None) -> MxArray:
        a = np.asarray(a)
        if cls is not None:
            a = a.astype(_NP[CLASS[cls]])
        if a.dtype == np.bool_:
            a = a.astype(np.uint8)
            code, cplx = 3, 0
        else:
            code, cplx = _FROM_NP[a.dtype]
        dims = a.shape if a.ndim >= 2 else ((1, a.size) if a.ndim == 1 else (1, 1))
        data = np.asfortranarray(a.reshape(dims))
        d = (C.c_size_t * len(dims))(*dims)
        p = self.lib.mexshim_host_array(len(dims), d, code, cplx, data.ctypes.data_as(C.c_void_p))
        return MxArray(self, p)

    def logical(self, v: bool) -> MxArray:
        return self.host(np.array([[bool(v)]]))

    def string(self, s: str) -> MxArray:
        return MxArray(self, self.lib.mexshim_string(s.encode()))

    def struct(self, fields: dict) -> MxArray:
        names = list(fields)
        vals = [v if isinstance(v, MxArray) else self._auto(v) for v in fields.values()]
        for v in vals:
            v.owned = False                 # the struct owns its fields
        arr_n = (C.c_char_p * len(names))(*[n.encode() for n in names])
        arr_v = (C.c_void_p * len(vals))(*[v.ptr for v in vals])
        s = MxArray(self, self.lib.mexshim_struct(len(names), arr_n, arr_v))
        s._keep = vals
        return s

    def _auto(self, v) -> MxArray:
        if isinstance(v, str):
            return self.string(v)
        if isinstance(v, bool):
            return self.logical(v)
        if isinstance(v, dict):
            return self.struct(v)
        return self.host(np.asarray(v, np.float64) if not isinstance(v, np.ndarray) else v)

    # -- calls --------------------------------------------------------------
    def call(self, fn, nlhs: int, *args) -> list:
        """[out1, ..., out_nlhs] = fn(args...); raises MexError on a MEX error."""
        ins = [a if isinstance(a, MxArray) else self._auto(a) for a in args]
        prhs = (C.c_void_p * max(len(ins), 1))(*[a.ptr for a in ins])
        plhs = (C.c_void_p * max(nlhs, 1))()
        ident = C.create_string_buffer(2048)
        msg = C.create_string_buffer(2048)
        rc = self.lib.mexshim_call(C.c_void_p(fn), nlhs, plhs, len(ins), prhs, ident, msg, 2048)
        outs = [MxArray(self, plhs[i]) for i in range(nlhs) if plhs[i]]
        if rc:
            raise MexError(ident.value.decode(), msg.value.decode())
        return outs

    def live_device_bytes(self) -> int:
        return int(self.lib.mexshim_live_device_bytes())

    def clear(self) -> int:
        """Run the mexAtExit functions (as `clear mex`)."""
        return int(self.lib.mexshim_clear())


def reference_available() -> bool:
    return bool(_build.reference_kernels()) and len(_build.reference_kernels()) == 2


_RT = None


def runtime() -> MexRuntime:
    global _RT
    if _RT is None:
        _RT = MexRuntime()
    return _RT


def reference_kernels() -> dict:
    """mexFunction pointers of the reference's decompBlockLU and applyBlockLU (prebuilt)."""
    rt = runtime()
    return {name: rt.load(path) for name, path in _build.reference_kernels().items()}


def gateway(name: str, out_dir: str) -> int:
    """Build (into out_dir) and load one of this repository's gateways; its mexFunction."""
    src = os.path.join(_build.ROOT, "waveforminversionust_b200", "mex", name + ".c")
    out = os.path.join(out_dir, f"gw_{name}.so")
    _build.build_gateway(src, out)
    return runtime().load(out)
