"""ctypes wrapper of the CPU oracle (libcsaw_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, to check or to time against.  The product library never
loads it.  Parity against the C-SAW reference itself is unpinned (the
reference ships no tests or golden data and its sampler is cuRAND-driven
device code); see csaw_oracle.h.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

NEIGHBOR, WALK, MDRW = 0, 1, 2
UNBIASED, DEGREE, EDGE_WEIGHT = 0, 1, 2
MAX_DEPTH = 128


class _Params(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32),
        ("bias", ctypes.c_int32),
        ("n_samples", ctypes.c_int32),
        ("frontier_size", ctypes.c_int32),
        ("depth", ctypes.c_int32),
        ("fanout", ctypes.c_int32 * MAX_DEPTH),
        ("seed", ctypes.c_uint64),
        ("sample_base", ctypes.c_int64),
        ("flags", ctypes.c_int32),
    ]


DEDUP = 1


def build():
    """Compile the oracle with its Makefile (gcc only)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libcsaw_oracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        p = ctypes.c_void_p
        L.oracle_philox4x32_10.argtypes = [p, p, p]
        L.oracle_canon_prefix.argtypes = [p, ctypes.c_int64, p]
        L.oracle_make_seeds.argtypes = [p, ctypes.c_int64, ctypes.c_int64, ctypes.c_uint64, p]
        L.oracle_make_seeds.restype = ctypes.c_int
        L.oracle_run.argtypes = [p, p, p, ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(_Params), p,
                                 p, p, p, p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
        L.oracle_run.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().oracle_philox4x32_10(_ptr(c), _ptr(k), _ptr(o))
    return o


def canon_prefix(w):
    w = np.ascontiguousarray(w, dtype=np.float32)
    P = np.zeros_like(w)
    lib().oracle_canon_prefix(_ptr(w), w.size, _ptr(P))
    return P


def make_seeds(rowptr, n, seed):
    rp = np.ascontiguousarray(rowptr, dtype=np.int64)
    out = np.zeros(n, dtype=np.int32)
    rc = lib().oracle_make_seeds(_ptr(rp), rp.size - 1, n, seed, _ptr(out))
    if rc:
        raise ValueError("oracle_make_seeds failed")
    return out


def run(rowptr, col, weight, seeds, mode, bias, n_samples, frontier_size, depth, fanout=None,
        seed=0, n_threads=1, cap=None, sample_base=0, flags=0):
    """Returns (src, dst, sample, depth) int32 arrays in oracle order."""
    rp = np.ascontiguousarray(rowptr, dtype=np.int64)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    wt = None if weight is None else np.ascontiguousarray(weight, dtype=np.float32)
    sd = np.ascontiguousarray(seeds, dtype=np.int32)
    P = _Params()
    P.mode, P.bias, P.n_samples = mode, bias, n_samples
    P.frontier_size, P.depth, P.seed = frontier_size, depth, seed
    P.sample_base = sample_base
    P.flags = flags
    fo = list(fanout or [])
    for i in range(min(depth, MAX_DEPTH)):
        P.fanout[i] = fo[i] if i < len(fo) else (fo[-1] if fo else 1)
    V = rp.size - 1
    if cap is None:
        cap = 1 << 20
    n = ctypes.c_int64(0)
    while True:
        bufs = [np.zeros(cap, dtype=np.int32) for _ in range(4)]
        rc = lib().oracle_run(_ptr(rp), _ptr(cl), _ptr(wt), V, cl.size, ctypes.byref(P), _ptr(sd),
                              *[_ptr(b) for b in bufs], cap, ctypes.byref(n), n_threads)
        if rc == 3:
            cap = n.value
            continue
        if rc != 0:
            raise ValueError(f"oracle_run failed rc={rc}")
        k = n.value
        return tuple(b[:k] for b in bufs)
