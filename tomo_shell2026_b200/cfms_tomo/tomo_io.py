"""ctypes helpers, unit conversions and optimum picking of the reference
front-end (cfms_tomo/tomo_io.py:1-81), on the B200 library.

The pointer aliases keep the reference's names: ``Cptr1iL`` is
``POINTER(c_long)`` as in the reference (tomo_io.py:8); it is only ever used
to pass int32 numpy buffers by address, which is width-independent, so it
works unchanged on LP64 Linux where ``c_long`` is 64-bit.  Reading int32
results back goes through :func:`Cptr1iL_to_np`, which reinterprets the
address as int32 instead of trusting ``c_long``.
"""
from __future__ import annotations

import ctypes as ct
import datetime
import time

import numpy as np

Cptr1i = ct.POINTER(ct.c_short)    # int16 pixels
Cptr1iL = ct.POINTER(ct.c_long)    # element ids (int32 buffers passed by address)
Cptr1d = ct.POINTER(ct.c_float)    # float32


def np_to_Cptr1i(X):
    return X.ctypes.data_as(Cptr1i)


def np_to_Cptr1iL(X):
    return X.ctypes.data_as(Cptr1iL)


def np_to_Cptr1d(X):
    return X.ctypes.data_as(Cptr1d)


def _read(ptr, rows, ctype, dtype):
    if rows == 0 or not ptr:
        return []
    addr = ct.cast(ptr, ct.c_void_p).value
    return np.ctypeslib.as_array(ct.cast(addr, ct.POINTER(ctype)), shape=(rows,)).astype(dtype)


def Cptr1i_to_np(ptr, rows):
    return _read(ptr, rows, ct.c_int16, np.int16)


def Cptr1iL_to_np(ptr, rows):
    return _read(ptr, rows, ct.c_int32, np.int32)


def Cptr1d_to_np(ptr, rows):
    return _read(ptr, rows, ct.c_float, np.float32)


def my_FStr(float_value, precision=1):
    return "{0:.{precision}f}".format(float_value, precision=precision)


def my_toRadian(degree):
    return degree * np.pi / 180.0


def my_toDegree(radian):
    return radian * 180.0 / np.pi


FStr = np.vectorize(my_FStr)
toRadian = np.vectorize(my_toRadian)
toDegree = np.vectorize(my_toDegree)


def StartTimer(str=""):  # noqa: A002 - reference argument name
    if len(str) > 0:
        print(str)
    return time.time()


def EndTimer(start_time, filename):
    print(filename + "= ", datetime.timedelta(seconds=time.time() - start_time), " seconds \n")


def smallestN_indices(data1D, N, maintain_order=False):
    """Best / worst N indices after rounding to 0.1 (tomo_io.py:50-56):
    argsort of ``round(x * 10) * 0.1``, ascending for the best, descending
    for the worst (numpy's default quicksort, so ties keep numpy's order)."""
    rounded = np.round(np.asarray(data1D) * 10.0) * 0.1
    best = rounded.argsort()
    worst = rounded.argsort()[::-1]
    if best.size >= N:
        return best[:N], worst[:N]
    return best, worst


def findOptimals(YPR, Mss, bVerbose=False, nOptimalToFind=1):
    """(best, worst) TomoResult of the rounded-Mss ranking (tomo_io.py:59-80)."""
    from .tomo_result import TomoResult
    best_ids, worst_ids = smallestN_indices(Mss, nOptimalToFind, maintain_order=True)
    n = min(best_ids.size, nOptimalToFind)
    bests, worsts = [], []
    for i in range(n):
        b, w = best_ids[i], worst_ids[i]
        B = TomoResult([YPR[b, 0], YPR[b, 1], YPR[b, 2], 0, Mss[b], Mss[b]])
        W = TomoResult([YPR[w, 0], YPR[w, 1], YPR[w, 2], 0, Mss[w], Mss[w]])
        if bVerbose:
            B.print()
            W.print()
        bests.append(B)
        worsts.append(W)
    return bests[0], worsts[0]
