"""Build a MEX gateway of magpackage_b200/mex/ with the test runtime (mx_runtime.cpp)
into a shared object and call it from Python with MATLAB argument semantics.

Arguments are numpy arrays read as MATLAB sees the reference's layouts: a C-order
(a, b) array is MATLAB's [b x a] column-major matrix, a 1-D array a column, a
Python number a 1x1 scalar, None the empty [].
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
PKG = os.path.join(ROOT, "magpackage_b200")
GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build(name: str, out_dir: str) -> str:
    """Compile magpackage_b200/mex/<name>.cpp + the runtime, linked against libmagasm.so."""
    src = os.path.join(PKG, "mex", name + ".cpp")
    so = os.path.join(str(out_dir), name + ".so")
    cmd = [GXX, "-std=c++11", "-O1", "-fPIC", "-shared", "-Wall", "-Werror", "-I" + HERE,
           "-I" + os.path.join(ROOT, "include"), src, os.path.join(HERE, "mx_runtime.cpp"),
           "-L" + PKG, "-lmagasm", "-Wl,-rpath," + PKG, "-o", so]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(out.stderr)
    return so


class GatewayError(RuntimeError):
    pass


class Gateway:
    def __init__(self, so: str):
        L = C.CDLL(so)
        L.rt_wrap.restype = C.c_void_p
        L.rt_wrap.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t]
        L.rt_call.restype = C.c_int
        L.rt_call.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p), C.c_char_p, C.c_int]
        L.rt_info.argtypes = [C.c_void_p, C.POINTER(C.c_size_t)]
        L.mxGetPr.restype = C.POINTER(C.c_double)
        L.mxGetPr.argtypes = [C.c_void_p]
        L.mxGetJc.restype = C.POINTER(C.c_uint64)
        L.mxGetJc.argtypes = [C.c_void_p]
        L.mxGetIr.restype = C.POINTER(C.c_uint64)
        L.mxGetIr.argtypes = [C.c_void_p]
        L.mxDestroyArray.argtypes = [C.c_void_p]
        self.L = L

    def _arg(self, a, keep):
        if a is None:
            return self.L.rt_wrap(None, 0, 0)
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        if a.ndim == 0:
            m, n = 1, 1
        elif a.ndim == 1:
            m, n = a.size, 1
        else:
            m, n = a.shape[-1], a.size // max(a.shape[-1], 1)
        return self.L.rt_wrap(a.ctypes.data if a.size else None, m, n)

    def _out(self, p):
        info = (C.c_size_t * 4)()
        self.L.rt_info(p, info)
        m, n, sparse, nnz = info
        if sparse:
            jc = np.ctypeslib.as_array(self.L.mxGetJc(p), (n + 1,)).copy()
            ir = np.ctypeslib.as_array(self.L.mxGetIr(p), (max(nnz, 1),))[:nnz].copy()
            pr = np.ctypeslib.as_array(self.L.mxGetPr(p), (max(nnz, 1),))[:nnz].copy()
            res = {"sparse": True, "m": m, "n": n, "jc": jc.astype(np.int64), "ir": ir.astype(np.int64), "pr": pr}
        else:
            pr = np.ctypeslib.as_array(self.L.mxGetPr(p), (m * n,)).copy() if m * n else np.zeros(0)
            res = {"sparse": False, "m": m, "n": n, "pr": pr}
        self.L.mxDestroyArray(p)
        return res

    def __call__(self, nlhs, *args):
        keep = []
        prhs = (C.c_void_p * max(len(args), 1))(*[self._arg(a, keep) for a in args])
        plhs = (C.c_void_p * 8)()
        msg = C.create_string_buffer(512)
        rc = self.L.rt_call(nlhs, plhs, len(args), prhs, msg, 512)
        for i in range(len(args)):
            self.L.mxDestroyArray(prhs[i])
        outs = [self._out(plhs[i]) for i in range(8) if plhs[i]]
        if rc != 0:
            raise GatewayError(msg.value.decode())
        return outs
