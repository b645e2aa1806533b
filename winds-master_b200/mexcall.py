"""Calling a ``mexFunction`` from Python without MATLAB.

A shared library that links ``csrc/mx_shim.cpp`` exports the mx*/mex* subset
declared in ``include/mex.h`` plus ``mxshim_call``. :class:`MexLib` builds
``mxArray`` inputs from NumPy arrays and strings, calls the library's
``mexFunction`` through ``mxshim_call`` (which turns ``mexErrMsg*`` into an
error code), and converts the outputs back to Fortran-ordered NumPy arrays.
This is how the tests call both this engine's MEX entry and the reference's
own compiled MEX source with identical arguments.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

mwSize = C.c_size_t
mxDOUBLE_CLASS = 6
mxREAL = 0


class MexError(RuntimeError):
    """A MEX error raised by ``mexErrMsgTxt`` / ``mexErrMsgIdAndTxt``."""

    def __init__(self, ident: str, message: str):
        super().__init__(f"{ident}: {message}" if ident else message)
        self.identifier = ident
        self.message = message


class MexLib:
    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.lib = C.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        L = self.lib
        L.mxCreateNumericArray.restype = C.c_void_p
        L.mxCreateNumericArray.argtypes = [mwSize, C.POINTER(mwSize), C.c_int, C.c_int]
        L.mxCreateString.restype = C.c_void_p
        L.mxCreateString.argtypes = [C.c_char_p]
        L.mxDestroyArray.argtypes = [C.c_void_p]
        L.mxGetPr.restype = C.POINTER(C.c_double)
        L.mxGetPr.argtypes = [C.c_void_p]
        L.mxGetNumberOfDimensions.restype = mwSize
        L.mxGetNumberOfDimensions.argtypes = [C.c_void_p]
        L.mxGetDimensions.restype = C.POINTER(mwSize)
        L.mxGetDimensions.argtypes = [C.c_void_p]
        L.mxGetNumberOfElements.restype = C.c_size_t
        L.mxGetNumberOfElements.argtypes = [C.c_void_p]
        L.mxshim_call.restype = C.c_int
        L.mxshim_call.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.c_int,
                                  C.POINTER(C.c_void_p), C.c_char_p, C.c_char_p, C.c_size_t]
        self.mexfn = C.cast(L.mexFunction, C.c_void_p)

    def _to_mx(self, v):
        L = self.lib
        if isinstance(v, str):
            return L.mxCreateString(v.encode())
        a = np.asarray(v, dtype=np.float64)
        if a.ndim == 0:
            a = a.reshape(1, 1)
        elif a.ndim == 1:
            a = a.reshape(1, -1)
        dims = (mwSize * a.ndim)(*a.shape)
        m = L.mxCreateNumericArray(a.ndim, dims, mxDOUBLE_CLASS, mxREAL)
        n = a.size
        if n:
            buf = np.ctypeslib.as_array(L.mxGetPr(m), shape=(n,))
            buf[:] = a.ravel(order="F")
        return m

    def _from_mx(self, m):
        L = self.lib
        nd = L.mxGetNumberOfDimensions(m)
        d = L.mxGetDimensions(m)
        shape = tuple(int(d[i]) for i in range(nd))
        n = int(np.prod(shape))
        if n == 0:
            return np.zeros(shape, order="F")
        flat = np.ctypeslib.as_array(L.mxGetPr(m), shape=(n,)).copy()
        return flat.reshape(shape, order="F")

    def call(self, nlhs: int, *args):
        L = self.lib
        prhs = (C.c_void_p * max(len(args), 1))()
        made = []
        try:
            for i, a in enumerate(args):
                prhs[i] = self._to_mx(a)
                made.append(prhs[i])
            plhs = (C.c_void_p * max(nlhs, 1))()
            eid = C.create_string_buffer(512)
            emsg = C.create_string_buffer(512)
            rc = L.mxshim_call(self.mexfn, nlhs, plhs, len(args), prhs, eid, emsg, 512)
            outs = []
            for i in range(nlhs):
                if plhs[i]:
                    if rc == 0:
                        outs.append(self._from_mx(plhs[i]))
                    L.mxDestroyArray(plhs[i])
            if rc != 0:
                raise MexError(eid.value.decode(), emsg.value.decode())
            return outs
        finally:
            for m in made:
                L.mxDestroyArray(m)
