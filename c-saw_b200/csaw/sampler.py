"""Host-side mirror of C-SAW's sampler interface over the csaw-b200 C ABI.

C-SAW's user surface is its positional run parameters -- #samples
(n_subgraph), FrontierSize, NeighborSize, Depth/Length (mpi_main.cpp:19-28,
README.md:30) -- the api.cuh hooks, a CSR input and a per-sample edge list
output (Si, sample_class.cuh:76-90).  `Graph.sample` takes the same
parameters and returns the edge list as (src, dst, sample, depth) tensors;
`Sampler` keeps the reference's host entry point (non-stream/main.cu:196).
PyTorch only provides device buffers and the current stream here.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import (BIAS_DEGREE, BIAS_EDGE_WEIGHT, BIAS_HOOK, BIAS_UNBIASED, MODE_MDRW, MODE_NEIGHBOR,
                   MODE_WALK, SCHED_PLAIN, CsawError, check, lib)

BIAS_NAMES = {"unbiased": BIAS_UNBIASED, "degree": BIAS_DEGREE, "weight": BIAS_EDGE_WEIGHT,
              "hook": BIAS_HOOK}
MODE_NAMES = {"neighbor": MODE_NEIGHBOR, "walk": MODE_WALK, "mdrw": MODE_MDRW}


def make_params(mode, bias, n_samples, frontier_size=1, neighbor_size=1, depth=1, fanout=None, seed=0,
                schedule=SCHED_PLAIN, sample_base=0, dedup=False):
    p = _lib.Params()
    p.mode = MODE_NAMES.get(mode, mode)
    p.bias = BIAS_NAMES.get(bias, bias)
    p.schedule = schedule
    p.n_samples = n_samples
    p.frontier_size = frontier_size
    p.neighbor_size = neighbor_size
    p.depth = depth
    for i, n in enumerate(fanout or []):
        p.fanout[i] = n
    p.seed = seed
    p.sample_base = sample_base
    p.flags = _lib.PARAM_DEDUP if dedup else 0
    return p


def fanouts(p):
    return [p.fanout[i] or p.neighbor_size for i in range(p.depth)]


def edge_bound(p):
    """Largest possible number of output edges for params p."""
    if p.mode == MODE_NEIGHBOR:
        tot, lvl = 0, p.frontier_size
        for n in fanouts(p):
            lvl *= n
            tot += lvl
        return p.n_samples * tot
    return p.n_samples * p.depth


def _torch():
    import torch
    return torch


class Graph:
    """A CSR resident on the current CUDA device (csaw_graph_create).

    cdf_cache: None builds the per-vertex bias prefix cache on the first
    batched or learned biased job; True builds it for every schedule (the
    plain one included); False never builds it.
    """

    def __init__(self, csr, rowptr64=None, degree_bias=False, cdf_cache=None):
        L = lib()
        if rowptr64 is None:
            rowptr64 = csr.n_edges >= 2**31
        self.rowptr_host = csr.rowptr if rowptr64 else csr.rowptr32()
        self.csr = csr
        flags = _lib.GRAPH_DEGREE_BIAS if degree_bias else 0
        if cdf_cache is not None:
            flags |= _lib.GRAPH_CDF_CACHE if cdf_cache else _lib.GRAPH_NO_CDF_CACHE
        h = ctypes.c_void_p()
        w = None if csr.weight is None else csr.weight.ctypes.data_as(ctypes.c_void_p)
        check(L.csaw_graph_create(self.rowptr_host.ctypes.data_as(ctypes.c_void_p), int(rowptr64),
                                  csr.col.ctypes.data_as(ctypes.c_void_p), w, csr.n_vertices,
                                  csr.n_edges, flags, ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().csaw_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stats(self):
        s = _lib.Stats()
        check(lib().csaw_graph_stats(self.h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _lib.Stats._fields_}

    def set_option(self, option, value):
        check(lib().csaw_graph_set_option(self.h, option, int(value)))

    # ---- learned scheduler
    def sched_record(self, n_records):
        """Record up to n execution profiles on the next learned-schedule runs."""
        self.set_option(_lib.OPT_SCHED_RECORD, n_records)

    def sched_info(self):
        n, t, l = ctypes.c_int64(), ctypes.c_int(), ctypes.c_float()
        check(lib().csaw_sched_info(self.h, ctypes.byref(n), ctypes.byref(t), ctypes.byref(l)))
        m = ctypes.c_uint32()
        check(lib().csaw_sched_classes(self.h, ctypes.byref(m)))
        return {"records": n.value, "trained": bool(t.value), "loss": l.value, "class_mask": m.value}

    def sched_records(self, max_n=1 << 20):
        out = np.zeros(max_n, dtype=PROF_DTYPE)
        n = ctypes.c_int64()
        check(lib().csaw_sched_get_records(self.h, out.ctypes.data_as(ctypes.c_void_p), max_n, ctypes.byref(n)))
        return out[:n.value]

    def sched_train(self, epochs=300, lr=3e-3, seed=0):
        loss = ctypes.c_float()
        check(lib().csaw_sched_train(self.h, epochs, lr, seed, ctypes.byref(loss)))
        return loss.value

    def sched_model(self):
        w = np.zeros(_lib.MLP_NPARAM, dtype=np.float32)
        nrm = np.zeros(_lib.MLP_NORM, dtype=np.float32)
        check(lib().csaw_sched_get_model(self.h, w.ctypes.data_as(ctypes.c_void_p), nrm.ctypes.data_as(ctypes.c_void_p)))
        return w, nrm

    def sched_set_model(self, w, nrm):
        w = np.ascontiguousarray(w, dtype=np.float32)
        nrm = np.ascontiguousarray(nrm, dtype=np.float32)
        check(lib().csaw_sched_set_model(self.h, w.ctypes.data_as(ctypes.c_void_p), nrm.ctypes.data_as(ctypes.c_void_p)))

    def profile(self, enable=True):
        check(lib().csaw_graph_profile(self.h, int(enable)))

    def kernel_stats(self, kind):
        ms = ctypes.c_double()
        n, b, it = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib().csaw_graph_kernel_stats(self.h, _lib.KERNEL_KINDS.get(kind, kind), ctypes.byref(ms),
                                            ctypes.byref(n), ctypes.byref(b), ctypes.byref(it)))
        return {"ms": ms.value, "launches": n.value, "bytes": b.value, "items": it.value}

    def make_seeds(self, n, seed, stream=None):
        torch = _torch()
        out = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
        st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(lib().csaw_make_seeds(self.h, n, seed, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st)))
        return out[:n]

    def sample(self, params, seeds, capacity=None, out=None, with_sample=True, with_depth=True, stream=None):
        """Run one job on device seeds; returns (src, dst, sample, depth) device tensors."""
        torch = _torch()
        if capacity is None:
            capacity = edge_bound(params)
        if out is None:
            out = torch.empty((2 + with_sample + with_depth, max(capacity, 1)), dtype=torch.int32, device="cuda")
        ptrs = [ctypes.c_void_p(out[i].data_ptr()) for i in range(out.shape[0])]
        src, dst = ptrs[0], ptrs[1]
        smp = ptrs[2] if with_sample else None
        dep = ptrs[2 + with_sample] if with_depth else None
        n = ctypes.c_int64()
        st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        seeds = seeds.to(device="cuda", dtype=torch.int32).contiguous()
        check(lib().csaw_sample(self.h, ctypes.byref(params), ctypes.c_void_p(seeds.data_ptr()), src, dst, smp,
                                dep, capacity, ctypes.byref(n), ctypes.c_void_p(st)))
        k = n.value
        res = [out[0, :k], out[1, :k]]
        res.append(out[2, :k] if with_sample else None)
        res.append(out[2 + with_sample, :k] if with_depth else None)
        return tuple(res)

    def sample_noalloc(self, params, seeds, out, capacity=None, with_sample=True, with_depth=True, stream=None):
        """Neighbor sampling through csaw_sample_noalloc: the library allocates
        nothing during the call (queues live in a fixed 32 MiB device array),
        for callers that must not call cudaMalloc while sampling -- e.g. a
        serving loop whose memory was reserved up front.  `out` is the
        caller's preallocated device tensor of shape (rows, capacity)."""
        torch = _torch()
        if capacity is None:
            capacity = out.shape[1]
        ptrs = [ctypes.c_void_p(out[i].data_ptr()) for i in range(out.shape[0])]
        n = ctypes.c_int64()
        st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        check(lib().csaw_sample_noalloc(self.h, ctypes.byref(params), ctypes.c_void_p(seeds.data_ptr()), ptrs[0],
                                        ptrs[1], ptrs[2] if with_sample else None,
                                        ptrs[2 + with_sample] if with_depth else None, capacity, ctypes.byref(n),
                                        ctypes.c_void_p(st)))
        k = n.value
        return (out[0, :k], out[1, :k], out[2, :k] if with_sample else None,
                out[2 + with_sample, :k] if with_depth else None)

    def autotune(self, jobs, stream=None):
        """Times the batch under each launch shape (csaw_graph_autotune) and
        keeps the fastest; returns the chosen shape and times."""
        arr = (_lib.Job * len(jobs))()
        for j, bj in zip(arr, jobs):
            bj.fill(j)
        r = _lib.TuneResult()
        st = stream if stream is not None else _torch().cuda.current_stream().cuda_stream
        check(lib().csaw_graph_autotune(self.h, arr, len(jobs), ctypes.c_void_p(st), ctypes.byref(r)))
        return {f: getattr(r, f) for f, _ in _lib.TuneResult._fields_}

    def sample_batch(self, jobs, stream=None):
        """Run several BatchJobs together (csaw_sample_batch); returns their edge lists."""
        arr = (_lib.Job * len(jobs))()
        for j, bj in zip(arr, jobs):
            bj.fill(j)
        if stream is None and not all(b.host for b in jobs):
            stream = _torch().cuda.current_stream().cuda_stream
        check(lib().csaw_sample_batch(self.h, arr, len(jobs), ctypes.c_void_p(stream) if stream else None))
        for j, bj in zip(arr, jobs):
            bj.n = j.n_out
        return [bj.result() for bj in jobs]

    def sample_host(self, params, seeds, capacity=None, with_sample=True, with_depth=True, out=None,
                    stream=None):
        """Host seeds in, host edge list out (copies inside the call)."""
        if capacity is None:
            capacity = edge_bound(params)
        seeds = np.ascontiguousarray(seeds, dtype=np.int32)
        if out is None:
            out = np.empty((2 + with_sample + with_depth, max(capacity, 1)), dtype=np.int32)
        ptr = lambda i: out[i].ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        n = ctypes.c_int64()
        st = ctypes.c_void_p(stream) if stream is not None else None
        check(lib().csaw_sample_host(self.h, ctypes.byref(params), seeds.ctypes.data_as(ctypes.c_void_p), ptr(0),
                                     ptr(1), ptr(2) if with_sample else None,
                                     ptr(2 + with_sample) if with_depth else None, capacity, ctypes.byref(n), st))
        k = n.value
        return (out[0, :k], out[1, :k], out[2, :k] if with_sample else None,
                out[2 + with_sample, :k] if with_depth else None)


PROF_DTYPE = np.dtype([("x", np.float32, 8), ("cls", np.int32), ("cycles", np.float32)])


def mlp_grad(params, norm, records):
    """Mean loss and gradient of the scheduler MLP on `records` (PROF_DTYPE
    array), computed by the library's GPU kernel."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    norm = np.ascontiguousarray(norm, dtype=np.float32)
    records = np.ascontiguousarray(records, dtype=PROF_DTYPE)
    grad = np.zeros(_lib.MLP_NPARAM, dtype=np.float32)
    loss = ctypes.c_float()
    check(lib().csaw_mlp_grad_host(params.ctypes.data_as(ctypes.c_void_p), norm.ctypes.data_as(ctypes.c_void_p),
                                   records.ctypes.data_as(ctypes.c_void_p), len(records),
                                   grad.ctypes.data_as(ctypes.c_void_p), ctypes.byref(loss)))
    return loss.value, grad


class StreamGraph:
    """A graph whose adjacency stays in host memory and is paged to the device
    by partitions of 2^partition_bits vertices (csaw_stream_graph_create);
    slot_budget_bytes bounds the device memory for resident partitions.  The
    CSR arrays are kept referenced (they are page-locked in place)."""

    def __init__(self, csr, partition_bits=20, slot_budget_bytes=32 << 30, rowptr64=None):
        L = lib()
        if rowptr64 is None:
            rowptr64 = csr.n_edges >= 2**31
        self.rowptr_host = csr.rowptr if rowptr64 else csr.rowptr32()
        self.csr = csr
        h = ctypes.c_void_p()
        w = None if csr.weight is None else csr.weight.ctypes.data_as(ctypes.c_void_p)
        check(L.csaw_stream_graph_create(self.rowptr_host.ctypes.data_as(ctypes.c_void_p), int(rowptr64),
                                         csr.col.ctypes.data_as(ctypes.c_void_p), w, csr.n_vertices, csr.n_edges,
                                         partition_bits, slot_budget_bytes, ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().csaw_stream_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def cache(self, bias):
        """Builds the prefix cache of `bias` (csaw_stream_graph_cache): later
        jobs with that bias stream each partition's prefix instead of its
        weights and search it (the same edges)."""
        check(lib().csaw_stream_graph_cache(self.h, BIAS_NAMES.get(bias, bias)))

    def set_option(self, option, value):
        """csaw_stream_graph_set_option (e.g. _lib.STREAM_OPT_READ_IN_PLACE)."""
        check(lib().csaw_stream_graph_set_option(self.h, option, int(value)))

    def info(self):
        s = _lib.StreamInfo()
        check(lib().csaw_stream_stats(self.h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _lib.StreamInfo._fields_}

    def sample(self, params, seeds, capacity=None, out=None, with_sample=True, with_depth=True, stream=None):
        torch = _torch()
        if capacity is None:
            capacity = edge_bound(params)
        if out is None:
            out = torch.empty((2 + with_sample + with_depth, max(capacity, 1)), dtype=torch.int32, device="cuda")
        ptrs = [ctypes.c_void_p(out[i].data_ptr()) for i in range(out.shape[0])]
        n = ctypes.c_int64()
        st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        seeds = seeds.to(device="cuda", dtype=torch.int32).contiguous()
        check(lib().csaw_stream_sample(self.h, ctypes.byref(params), ctypes.c_void_p(seeds.data_ptr()), ptrs[0],
                                       ptrs[1], ptrs[2] if with_sample else None,
                                       ptrs[2 + with_sample] if with_depth else None, capacity, ctypes.byref(n),
                                       ctypes.c_void_p(st)))
        k = n.value
        return (out[0, :k], out[1, :k], out[2, :k] if with_sample else None,
                out[2 + with_sample, :k] if with_depth else None)


class BatchJob:
    """One job of Graph.sample_batch: params, seeds and output buffers (device
    tensors, or numpy arrays with host=True)."""

    def __init__(self, params, seeds, capacity=None, out=None, with_sample=True, with_depth=True, host=False):
        self.params = params
        self.capacity = edge_bound(params) if capacity is None else capacity
        self.host = host
        self.with_sample, self.with_depth = with_sample, with_depth
        rows = 2 + with_sample + with_depth
        if host:
            self.seeds = np.ascontiguousarray(seeds, dtype=np.int32)
            self.out = out if out is not None else np.empty((rows, max(self.capacity, 1)), dtype=np.int32)
        else:
            torch = _torch()
            self.seeds = seeds.to(device="cuda", dtype=torch.int32).contiguous()
            self.out = out if out is not None else torch.empty((rows, max(self.capacity, 1)), dtype=torch.int32,
                                                                 device="cuda")
        self.n = 0

    def _ptr(self, x):
        if self.host:
            return x.ctypes.data_as(ctypes.c_void_p).value
        return x.data_ptr()

    def fill(self, j):
        j.params = ctypes.pointer(self.params)
        j.seeds = self._ptr(self.seeds)
        j.out_src, j.out_dst = self._ptr(self.out[0]), self._ptr(self.out[1])
        j.out_sample = self._ptr(self.out[2]) if self.with_sample else None
        j.out_depth = self._ptr(self.out[2 + self.with_sample]) if self.with_depth else None
        j.capacity = self.capacity
        j.host_buffers = int(self.host)

    def result(self):
        k = self.n
        o = self.out
        return (o[0, :k], o[1, :k], o[2, :k] if self.with_sample else None,
                o[2 + self.with_sample, :k] if self.with_depth else None)


class Server:
    """Request loop with continuous batching on a resident Graph
    (csaw_server_*): a native worker thread admits requests as slots and the
    device budget free up and runs them concurrently; results land in host
    buffers (numpy arrays, or page-locked torch CPU tensors for a direct
    copy).  submit/wait may be called from several threads."""

    def __init__(self, graph, n_slots=8, device_budget=1 << 30, max_wait_us=2000):
        cfg = _lib.ServerConfig(n_slots, max_wait_us, device_budget)
        h = ctypes.c_void_p()
        check(lib().csaw_server_create(graph.h, ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.graph = graph
        self._live = {}

    def close(self):
        if self.h:
            lib().csaw_server_destroy(self.h)
            self.h = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _addr(x):
        if isinstance(x, np.ndarray):
            return x.ctypes.data_as(ctypes.c_void_p).value
        return x.data_ptr()

    def submit(self, params, seeds, out=None, capacity=None, with_sample=True, with_depth=True):
        """Queues one request; returns its ticket.  seeds: host int32 array
        (copied); out: (2 + with_sample + with_depth, capacity) int32 host
        buffer, kept referenced until wait() reports the ticket."""
        seeds = np.ascontiguousarray(seeds, dtype=np.int32)
        if capacity is None:
            capacity = edge_bound(params) if out is None else out.shape[1]
        rows = 2 + with_sample + with_depth
        if out is None:
            out = np.empty((rows, max(capacity, 1)), dtype=np.int32)
        ptr = [self._addr(out[i]) for i in range(rows)]
        t = ctypes.c_uint64()
        check(lib().csaw_server_submit(self.h, ctypes.byref(params), seeds.ctypes.data_as(ctypes.c_void_p), ptr[0],
                                       ptr[1], ptr[2] if with_sample else None,
                                       ptr[2 + with_sample] if with_depth else None, capacity, ctypes.byref(t)))
        self._live[t.value] = (out, with_sample, with_depth)
        return t.value

    def wait(self, ticket, timeout_us=-1):
        """(edges, latency_ms, (src, dst, sample, depth) views) once the request
        is done; None while it is pending after timeout_us.  Raises CsawError
        for a failed request."""
        n, lat = ctypes.c_int64(), ctypes.c_double()
        rc = lib().csaw_server_wait(self.h, ticket, timeout_us, ctypes.byref(n), ctypes.byref(lat))
        if rc == _lib.PENDING:
            return None
        live = self._live.pop(ticket, None)
        check(rc)
        out, ws, wd = live
        k = n.value
        res = (out[0, :k], out[1, :k], out[2, :k] if ws else None, out[2 + ws, :k] if wd else None)
        return k, lat.value, res

    def stats(self, reset=False):
        st = _lib.ServerStats()
        check(lib().csaw_server_get_stats(self.h, int(reset), ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in _lib.ServerStats._fields_}


class Arguments:
    """struct arguments of the reference (sampler.cuh:3-6)."""

    def __init__(self, sampled_edges=0, time=0.0):
        self.sampled_edges = sampled_edges
        self.time = time


def Sampler(beg, csr, n_blocks, n_threads, n_subgraph, FrontierSize, NeighborSize, Depth, args=None, rank=0):
    """Reference host entry (non-stream/main.cu:196): loads int64 beg/csr files,
    samples (FrontierSize == 1) or runs MDRW (FrontierSize > 1), returns
    Arguments(sampled_edges, time)."""
    e = ctypes.c_int()
    t = ctypes.c_double()
    check(lib().csaw_sampler_compat(str(beg).encode(), str(csr).encode(), n_blocks, n_threads, n_subgraph,
                                    FrontierSize, NeighborSize, Depth, ctypes.byref(e), ctypes.byref(t)))
    out = args if args is not None else Arguments()
    out.sampled_edges, out.time = e.value, t.value
    return out


__all__ = ["mlp_grad", "PROF_DTYPE", "Graph", "StreamGraph", "Sampler", "Arguments", "BatchJob", "make_params", "edge_bound", "CsawError"]
