"""CPU tests of the host side: the C-ABI library loads and exports every
symbol include/csaw.h declares, argument validation that returns before any
CUDA call, generators, and host-side helpers."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "csaw.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(csaw_\w+)\s*\(", txt)))


def test_library_exports_every_header_symbol():
    import csaw
    from csaw import _lib
    L = csaw.lib()
    names = header_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.EXPORTS)
    assert b"sm_100a" in L.csaw_version()


def test_graph_create_validates_before_cuda():
    import csaw
    L = csaw.lib()
    h = ctypes.c_void_p()
    rp = np.array([0, 2, 1], dtype=np.int64)   # not monotone, rowptr[V] != E
    col = np.array([1, 0], dtype=np.int32)
    rc = L.csaw_graph_create(rp.ctypes.data_as(ctypes.c_void_p), 1, col.ctypes.data_as(ctypes.c_void_p), None, 2,
                             2, 0, ctypes.byref(h))
    assert rc == csaw.sampler._lib.ERR_INVALID
    assert b"rowptr" in L.csaw_last_error()
    rp = np.array([0, 1, 2], dtype=np.int64)
    col = np.array([5, 0], dtype=np.int32)     # col out of range
    rc = L.csaw_graph_create(rp.ctypes.data_as(ctypes.c_void_p), 1, col.ctypes.data_as(ctypes.c_void_p), None, 2,
                             2, 0, ctypes.byref(h))
    assert rc == 1 and b"col" in L.csaw_last_error()
    w = np.array([1.0, -1.0], dtype=np.float32)
    col = np.array([1, 0], dtype=np.int32)
    rc = L.csaw_graph_create(rp.ctypes.data_as(ctypes.c_void_p), 1, col.ctypes.data_as(ctypes.c_void_p),
                             w.ctypes.data_as(ctypes.c_void_p), 2, 2, 0, ctypes.byref(h))
    assert rc == 1 and b"weights" in L.csaw_last_error()


def test_sample_rejects_null_graph():
    import csaw
    L = csaw.lib()
    p = csaw.make_params(0, 0, 1, 1, 2, 2)
    n = ctypes.c_int64()
    assert L.csaw_sample(None, ctypes.byref(p), None, None, None, None, None, 0, ctypes.byref(n), None) == 1


def test_edge_bound():
    import csaw
    p = csaw.make_params("neighbor", "degree", 4000, 4, 20, 3)
    assert csaw.edge_bound(p) == 4000 * 4 * (20 + 400 + 8000)
    p = csaw.make_params("neighbor", "unbiased", 10, 1, 0, 3, fanout=[15, 10, 5])
    assert csaw.edge_bound(p) == 10 * (15 + 150 + 750)
    p = csaw.make_params("walk", "degree", 4000, 1, 1, 64)
    assert csaw.edge_bound(p) == 4000 * 64


def test_rmat_generator_is_deterministic_and_clean():
    from csaw import graphgen
    a = graphgen.rmat(10, 8, seed=4)
    b = graphgen.rmat(10, 8, seed=4)
    assert np.array_equal(a.rowptr, b.rowptr) and np.array_equal(a.col, b.col)
    assert np.array_equal(a.weight, b.weight)
    src = np.repeat(np.arange(a.n_vertices), np.diff(a.rowptr))
    assert not np.any(src == a.col)
    key = src * a.n_vertices + a.col
    assert np.unique(key).size == key.size
    # symmetric
    rkey = a.col.astype(np.int64) * a.n_vertices + src
    assert np.array_equal(np.sort(key), np.sort(rkey))
    assert a.weight.min() > 0 and a.weight.max() <= 1


def test_powerlaw_generator_shape():
    from csaw import graphgen
    g = graphgen.powerlaw_directed(n_vertices=50_000, n_edges=291_000, max_degree=460, seed=1)
    deg = np.diff(g.rowptr)
    assert g.n_edges == 291_000 and deg.max() == 460
    src = np.repeat(np.arange(g.n_vertices), deg)
    assert not np.any(src == g.col)
    key = src * g.n_vertices + g.col
    assert np.unique(key).size == key.size
    # heavy tail: log-log slope of the out-degree CCDF is roughly -(gamma - 1)
    ds = np.arange(2, 200)
    ccdf = np.array([(deg >= d).mean() for d in ds])
    slope = np.polyfit(np.log(ds), np.log(ccdf), 1)[0]
    assert -1.6 < slope < -0.6


def test_reference_file_roundtrip(tmp_path):
    from csaw import graphgen
    g = graphgen.rmat(8, 4, seed=2)
    graphgen.write_reference_format(g, tmp_path / "beg.bin", tmp_path / "csr.bin")
    h = graphgen.read_reference_format(tmp_path / "beg.bin", tmp_path / "csr.bin")
    assert np.array_equal(g.rowptr, h.rowptr) and np.array_equal(g.col, h.col)
    assert np.fromfile(tmp_path / "beg.bin", dtype=np.int64).size == g.n_vertices + 1


def test_device_rmat_generator_is_clean_on_cpu():
    """rmat_device (the torch generator used for the large synthetic graphs)
    produces a sorted CSR without self-loops or duplicates, symmetric when
    asked, with the requested weight law; run here on the CPU device."""
    from csaw import graphgen
    g = graphgen.rmat_device(11, 8, seed=4, device="cpu", weight="pareto:1.5")
    rp, col = g.rowptr, g.col
    src = np.repeat(np.arange(g.n_vertices), np.diff(rp))
    key = src * g.n_vertices + col
    assert (np.diff(key) > 0).all() and (src != col).all()
    assert np.array_equal(np.sort(col.astype(np.int64) * g.n_vertices + src), key)   # symmetric
    assert g.weight.dtype == np.float32 and g.weight.min() >= 1.0                   # Pareto, x_m = 1
    d = graphgen.rmat_device(11, 8, seed=4, device="cpu", symmetrize=False, weight="uniform")
    assert d.n_edges < g.n_edges and 0.0 < d.weight.min() and d.weight.max() <= 1.0
    again = graphgen.rmat_device(11, 8, seed=4, device="cpu", weight="pareto:1.5")
    assert np.array_equal(again.col, g.col) and np.array_equal(again.weight, g.weight)


def test_params_flags_layout():
    """The Python mirror of csaw_params carries the dedup flag where the C ABI
    expects it (size and offset of the trailing fields)."""
    import ctypes
    from csaw import _lib, make_params
    p = make_params(0, 1, 10, 2, 5, 2, seed=3, dedup=True)
    assert p.flags == _lib.PARAM_DEDUP
    assert _lib.Params.flags.offset == _lib.Params.sample_base.offset + 8
    assert ctypes.sizeof(_lib.Params) == _lib.Params.reserved.offset + 4


def test_python_constants_match_header():
    """Every CSAW_* enum value of include/csaw.h has the same value in the
    Python binding (status codes, modes, biases, schedules, flags, options)."""
    from csaw import _lib
    txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "csaw.h")).read(), flags=re.S)
    consts = re.findall(r"\bCSAW_(\w+)\s*=\s*(-?\d+)", txt)
    assert len(consts) >= 20
    for name, value in consts:
        assert hasattr(_lib, name), name
        assert getattr(_lib, name) == int(value), name


def test_stream_option_rejects_null_graph():
    """csaw_stream_graph_set_option checks its handle before any CUDA call."""
    import csaw
    from csaw import _lib
    L = csaw.lib()
    assert L.csaw_stream_graph_set_option(None, _lib.STREAM_OPT_READ_IN_PLACE, 1) == _lib.ERR_INVALID
