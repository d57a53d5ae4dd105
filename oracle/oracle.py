"""ORACLE — test infrastructure only.

ctypes wrapper around oracle/_build/liboracle.so, the CPU restatement of the
reference's partitioning path (see oracle/oracle.h for the parity status and
the deterministic rules). Only tests/, __graft_entry__.smoke() and the CPU
baseline legs of bench.py import this module; the product never does.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_HOST = os.path.join(_HERE, "..", "gpu-heipa_b200", "host")
_SOURCES = [os.path.join(_HERE, "oracle.cpp"), os.path.join(_HOST, "initial_partition.cpp"),
            os.path.join(_HOST, "metis_kway.cpp")]


def build(force=False):
    """Compiles the oracle with g++ (OpenMP) into oracle/_build/, and the
    reference's own initial partitioner into oracle/_ref/ when the reference
    sources are present (build_ref.py)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("oracle_build_ref", os.path.join(_HERE, "build_ref.py"))
    build_ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(build_ref)
    build_ref.build_ref()
    os.makedirs(os.path.dirname(_LIB_PATH), exist_ok=True)
    if not force and os.path.exists(_LIB_PATH):
        deps = _SOURCES + [os.path.join(_HERE, "oracle.h"), os.path.join(_HOST, "metis_kway.h"),
                           os.path.join(_HOST, "initial_partition.h")]
        if os.path.getmtime(_LIB_PATH) >= max(os.path.getmtime(s) for s in deps):
            return _LIB_PATH
    cmd = ["g++", "-O3", "-std=c++17", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-o", _LIB_PATH] + _SOURCES
    subprocess.run(cmd, check=True)
    return _LIB_PATH


_lib = None

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_s32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p


def lib():
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = ctypes.CDLL(_LIB_PATH)
    c = ctypes
    sig = {
        "or_xorshift32": (c.c_uint32, [c.c_uint32]),
        "or_threads": (c.c_int, []),
        "or_murmur3_u32": (c.c_uint32, [c.c_uint32, c.c_uint32]),
        "or_gain_bucket": (c.c_uint32, [c.c_int32, c.c_int32]),
        "or_gain_bucket_float": (c.c_uint32, [c.c_int32, c.c_int32]),
        "or_graph_new": (_vp, [c.c_uint32, c.c_uint32, _vp, _vp, _vp, _vp]),
        "or_graph_free": (None, [_vp]),
        "or_graph_n": (c.c_uint32, [_vp]),
        "or_graph_m": (c.c_uint32, [_vp]),
        "or_graph_has_ew": (c.c_int, [_vp]),
        "or_graph_has_vw": (c.c_int, [_vp]),
        "or_graph_get": (None, [_vp, _vp, _vp, _vp, _vp]),
        "or_match": (c.c_uint32, [_vp, _vp]),
        "or_contract": (_vp, [_vp, _vp, c.c_uint32]),
        "or_edge_cut": (c.c_int64, [_vp, _vp]),
        "or_comm_cost": (c.c_int64, [_vp, _vp, _vp, _vp, c.c_uint32]),
        "or_distance_matrix": (None, [_vp, _vp, c.c_uint32, _vp]),
        "or_jet_new": (_vp, [_vp, c.c_uint32, c.c_int32, _vp, _vp, _vp, c.c_uint32]),
        "or_jet_free": (None, [_vp]),
        "or_jet_lp": (c.c_uint32, [_vp, c.c_uint32, _vp]),
        "or_jet_weak": (c.c_uint32, [_vp, _vp]),
        "or_jet_strong": (c.c_uint32, [_vp, _vp]),
        "or_jet_perform": (None, [_vp, _vp, c.c_uint32, _vp, _vp]),
        "or_jet_state": (None, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
        "or_jet_refine": (None, [_vp, c.c_uint32, c.c_int32, c.c_int, c.c_uint32, _vp, _vp, _vp, _vp, _vp,
                                 c.c_uint32]),
        "or_partition": (c.c_int64, [_vp, c.c_uint32, c.c_double, c.c_int, c.c_uint64, _vp]),
        "or_map_hm": (c.c_int64, [_vp, _vp, _vp, c.c_uint32, c.c_double, c.c_int, c.c_uint64, _vp]),
        "or_map_im": (c.c_int64, [_vp, _vp, _vp, c.c_uint32, c.c_double, c.c_uint64, _vp]),
        "or_lmax": (c.c_int32, [c.c_int64, c.c_uint32, c.c_double]),
        "or_set_ref_kway": (None, [_vp]),
        "or_uses_ref_kway": (c.c_int, []),
        "or_initial_kway": (None, [_vp, c.c_uint32, c.c_double, c.c_uint64, _vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    ref = ref_lib()
    if ref is not None:
        L.or_set_ref_kway(ctypes.cast(ref.ref_kway_partition, ctypes.c_void_p))
    _lib = L
    return L


_REF_PATH = os.path.join(_HERE, "_ref", "libkway_ref.so")
_ref = None


def ref_lib():
    """The reference's own initial partitioner (oracle/_ref/libkway_ref.so,
    built by build_ref.py from the reference's sources), or None."""
    global _ref
    if _ref is None and os.path.exists(_REF_PATH):
        R = ctypes.CDLL(_REF_PATH)
        R.ref_kway_partition.restype = None
        R.ref_kway_partition.argtypes = [ctypes.c_uint32, _vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_uint64, _vp]
        _ref = R
    return _ref


def uses_reference_kway():
    """True when the oracle pipelines take their initial partitions from the
    reference's own code."""
    return bool(lib().or_uses_ref_kway())


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _s32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


class Graph:
    """A CSR graph held by the oracle (copies the arrays)."""

    def __init__(self, xadj=None, adj=None, ew=None, vw=None, handle=None):
        L = lib()
        if handle is not None:
            self.h = handle
        else:
            xadj, adj = _u32(xadj), _u32(adj)
            ew, vw = _s32(ew), _s32(vw)
            n = len(xadj) - 1
            self.h = L.or_graph_new(n, len(adj), _p(xadj), _p(adj), _p(ew), _p(vw))
        self.n = L.or_graph_n(self.h)
        self.m = L.or_graph_m(self.h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_graph_free(self.h)
            self.h = None

    def arrays(self):
        L = lib()
        xadj = np.zeros(self.n + 1, np.uint32)
        adj = np.zeros(self.m, np.uint32)
        ew = np.zeros(self.m, np.int32)
        vw = np.zeros(self.n, np.int32)
        L.or_graph_get(self.h, _p(xadj), _p(adj), _p(ew), _p(vw))
        has_ew = bool(L.or_graph_has_ew(self.h))
        has_vw = bool(L.or_graph_has_vw(self.h))
        return xadj, adj, (ew if has_ew else None), (vw if has_vw else None)


def initial_kway(g, k, eps, seed):
    """The initial partition of the oracle pipelines (kway_core.h:1548-1571)."""
    part = np.zeros(g.n, np.uint32)
    lib().or_initial_kway(g.h, k, eps, seed, _p(part))
    return part


def ref_kway(xadj, adj, vw, ew, k, imbalance, seed):
    """GPU_HeiPa::ModifiedMetis::partition itself on a CSR (weights required)."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("oracle/_ref/libkway_ref.so is not built")
    xadj, adj, vw, ew = _u32(xadj), _u32(adj), _s32(vw), _s32(ew)
    part = np.zeros(len(xadj) - 1, np.uint32)
    R.ref_kway_partition(len(xadj) - 1, _p(xadj), _p(adj), _p(vw), _p(ew), int(k), float(imbalance), int(seed),
                         _p(part))
    return part


def match(g):
    mp = np.zeros(g.n, np.uint32)
    nc = lib().or_match(g.h, _p(mp))
    return mp, int(nc)


def contract(g, mapping, n_c):
    mapping = _u32(mapping)
    return Graph(handle=lib().or_contract(g.h, _p(mapping), int(n_c)))


def edge_cut(g, part):
    part = _u32(part)
    return int(lib().or_edge_cut(g.h, _p(part)))


def comm_cost(g, part, hier, dist):
    part, hier, dist = _u32(part), _u32(hier), _s32(dist)
    return int(lib().or_comm_cost(g.h, _p(part), _p(hier), _p(dist), len(hier)))


def distance_matrix(hier, dist):
    hier, dist = _u32(hier), _s32(dist)
    k = int(np.prod(hier))
    out = np.zeros(k * k, np.int32)
    lib().or_distance_matrix(_p(hier), _p(dist), len(hier), _p(out))
    return out.reshape(k, k)


def lmax(total_weight, k, eps):
    return int(lib().or_lmax(int(total_weight), int(k), float(eps)))


class Jet:
    """One level of Jet refinement state (edge cut, or J when hier is given)."""

    def __init__(self, g, k, lmax_, part, hier=None, dist=None):
        L = lib()
        self.g, self.k, self.n = g, int(k), g.n
        part = _u32(part)
        hier = None if hier is None else _u32(hier)
        dist = None if dist is None else _s32(dist)
        self.h = L.or_jet_new(g.h, self.k, int(lmax_), _p(part), _p(hier), _p(dist),
                              0 if hier is None else len(hier))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_jet_free(self.h)
            self.h = None

    def lp(self, ratio_pct):
        out = np.zeros(self.n, np.uint32)
        c = lib().or_jet_lp(self.h, int(ratio_pct), _p(out))
        return out[:c].copy()

    def weak(self):
        out = np.zeros(self.n, np.uint32)
        c = lib().or_jet_weak(self.h, _p(out))
        return out[:c].copy()

    def strong(self):
        out = np.zeros(self.n, np.uint32)
        c = lib().or_jet_strong(self.h, _p(out))
        return out[:c].copy()

    def perform(self, moves, obj):
        moves = _u32(moves)
        o = ctypes.c_int64(int(obj))
        mw = ctypes.c_int32(0)
        lib().or_jet_perform(self.h, _p(moves), len(moves), ctypes.byref(o), ctypes.byref(mw))
        return int(o.value), int(mw.value)

    def state(self):
        n, k = self.n, self.k
        st = dict(map=np.zeros(n, np.uint32), bw=np.zeros(k, np.int32), dest_part=np.zeros(n, np.uint32),
                  gain1=np.zeros(n, np.int32), lock=np.zeros(n, np.uint32), dest_cache=np.zeros(n, np.uint32),
                  gain_cache=np.zeros(n, np.int32))
        lib().or_jet_state(self.h, *[_p(st[x]) for x in
                                     ("map", "bw", "dest_part", "gain1", "lock", "dest_cache", "gain_cache")])
        return st


def jet_refine(g, k, lmax_, ultra, level, part, obj, maxw, hier=None, dist=None):
    part = _u32(part).copy()
    o = ctypes.c_int64(int(obj))
    mw = ctypes.c_int32(int(maxw))
    hier = None if hier is None else _u32(hier)
    dist = None if dist is None else _s32(dist)
    lib().or_jet_refine(g.h, int(k), int(lmax_), int(bool(ultra)), int(level), _p(part), ctypes.byref(o),
                        ctypes.byref(mw), _p(hier), _p(dist), 0 if hier is None else len(hier))
    return part, int(o.value), int(mw.value)


def partition(g, k, eps=0.03, ultra=False, seed=0):
    out = np.zeros(g.n, np.uint32)
    cut = lib().or_partition(g.h, int(k), float(eps), int(bool(ultra)), int(seed), _p(out))
    return out, int(cut)


def map_hm(g, hier, dist, eps=0.03, ultra=False, seed=0):
    hier, dist = _u32(hier), _s32(dist)
    out = np.zeros(g.n, np.uint32)
    J = lib().or_map_hm(g.h, _p(hier), _p(dist), len(hier), float(eps), int(bool(ultra)), int(seed), _p(out))
    return out, int(J)


def map_im(g, hier, dist, eps=0.03, seed=0):
    hier, dist = _u32(hier), _s32(dist)
    out = np.zeros(g.n, np.uint32)
    J = lib().or_map_im(g.h, _p(hier), _p(dist), len(hier), float(eps), int(seed), _p(out))
    return out, int(J)


def threads():
    """Host threads of the oracle's parallel loops (results do not depend on it)."""
    return int(lib().or_threads())


def xorshift32(x):
    return int(lib().or_xorshift32(int(x) & 0xFFFFFFFF))


def murmur3_u32(key, seed=0):
    return int(lib().or_murmur3_u32(int(key) & 0xFFFFFFFF, int(seed) & 0xFFFFFFFF))


def gain_bucket(gx, vwgt):
    return int(lib().or_gain_bucket(int(gx), int(vwgt)))


def gain_bucket_float(gx, vwgt):
    return int(lib().or_gain_bucket_float(int(gx), int(vwgt)))


if __name__ == "__main__":
    print(build(force=True))
