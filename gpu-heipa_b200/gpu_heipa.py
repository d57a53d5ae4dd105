"""Python binding of the partitioner's C ABI (include/gpuheipa.h).

Mirrors the reference's operator surface for this path:
  partition(graph, k, imbalance, config)           -> GPU-HeiPa (Solver::solve)
  process_map(graph, hierarchy, distance, config)  -> GPU-HeiProMap (ProMapSolver)
plus the phase kernels (match, contract, Jet) for stepping and inspection.

The CUDA library is required: importing this module raises if
lib/libgpuheipa.so is missing, and every call raises HeiPaError when the C
ABI reports a failure. There is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libgpuheipa.so")

HP_MAP_IM, HP_MAP_HM, HP_MAP_HM_ULTRA = 0, 1, 2
MAP_MODES = {"IM": HP_MAP_IM, "HM": HP_MAP_HM, "HM-ultra": HP_MAP_HM_ULTRA}
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "I/O error",
          5: "invalid graph", 6: "device error", 7: "input too large", 8: "busy"}
EDGE_CUT_NOALLOC_MAX_N = 4194304


class HeiPaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing; build it with gpu-heipa_b200/build.py")

_L = ctypes.CDLL(LIB_PATH)
_vp = ctypes.c_void_p
_u32, _u64, _i32, _i64, _dbl, _int = (ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int64,
                                      ctypes.c_double, ctypes.c_int)
_SIG = {
    "hp_ctx_create": (_int, [_int, ctypes.c_size_t, _vp]),
    "hp_ctx_destroy": (_int, [_vp]),
    "hp_last_error": (ctypes.c_char_p, [_vp]),
    "hp_arena_estimate": (ctypes.c_size_t, [_u32, _u64, _int, _int]),
    "hp_arena_peak": (ctypes.c_size_t, [_vp]),
    "hp_graph_upload": (_int, [_vp, _u32, _u64, _vp, _vp, _vp, _vp, _vp]),
    "hp_graph_free": (_int, [_vp, _vp]),
    "hp_graph_info": (_int, [_vp, _vp, _vp, _vp]),
    "hp_graph_download": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "hp_match": (_int, [_vp, _vp, _vp, _vp]),
    "hp_contract": (_int, [_vp, _vp, _vp, _u32, _vp]),
    "hp_jet_refine": (_int, [_vp, _vp, _u32, _i32, _int, _u32, _vp, _vp, _vp, _vp, _vp, _u32]),
    "hp_jet_begin": (_int, [_vp, _vp, _u32, _i32, _vp, _vp, _vp, _u32, _vp]),
    "hp_jet_lp": (_int, [_vp, _u32, _vp, _vp]),
    "hp_jet_weak": (_int, [_vp, _vp, _vp]),
    "hp_jet_strong": (_int, [_vp, _vp, _vp]),
    "hp_jet_perform": (_int, [_vp, _vp, _vp]),
    "hp_jet_state": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hp_jet_end": (_int, [_vp]),
    "hp_edge_cut": (_int, [_vp, _vp, _vp, _vp]),
    "hp_comm_cost": (_int, [_vp, _vp, _vp, _vp, _vp, _u32, _vp]),
    "hp_edge_cut_noalloc": (_int, [_u32, _u32, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hp_selftest_barrier_timeout": (_int, [ctypes.c_int, _u32, _vp, _vp]),
    "hp_coop_slot_acquire": (_int, [ctypes.c_int, ctypes.c_int]),
    "hp_initial_partition": (_int, [_u32, _vp, _vp, _vp, _vp, _u32, ctypes.c_double, ctypes.c_uint64, _vp]),
    "hp_coop_slot_release": (_int, [ctypes.c_int]),
    "hp_partition": (_int, [_vp, _u32, _u64, _vp, _vp, _vp, _vp, _u32, _dbl, _int, _u64, _vp, _vp]),
    "hp_partition_graph": (_int, [_vp, _vp, _u32, _dbl, _int, _u64, _vp, _vp]),
    "hp_map": (_int, [_vp, _u32, _u64, _vp, _vp, _vp, _vp, _vp, _vp, _u32, _dbl, _int, _u64, _vp, _vp]),
    "hp_map_graph": (_int, [_vp, _vp, _vp, _vp, _u32, _dbl, _int, _u64, _vp, _vp]),
    "hp_last_solve_stats": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "hp_last_solve_maxw": (_int, [_vp, _vp, _vp]),
    "hp_last_solve_level": (_int, [_vp, _u32, _vp, _vp]),
    "hp_tune": (_int, [_vp, ctypes.c_char_p, _i64]),
    "hp_instrument": (_int, [_vp, _int]),
    "hp_kernel_timing": (_int, [_vp, ctypes.c_char_p, _vp, _vp, _vp]),
    "hp_kernel_log": (_int, [_vp, _u64, ctypes.c_char_p, ctypes.c_size_t, _vp, _vp]),
    "hp_event_record": (_int, [_vp, _int]),
    "hp_event_elapsed": (_int, [_vp, _int, _int, _vp]),
    "hp_kernel_launches": (_u64, []),
    "hp_profile": (_int, [_vp, _int]),
    "hp_profile_entry": (_int, [_vp, _u32, ctypes.c_char_p, ctypes.c_size_t, _vp, _vp]),
    "hp_partition_batch": (_int, [_vp, _vp, _u32, _u32]),
    "hp_server_create": (_int, [_int, ctypes.c_size_t, _u32, _vp]),
    "hp_server_submit_partition": (_int, [_vp, _u32, _u64, _vp, _vp, _vp, _vp, _u32, _dbl, _int, _u64, _vp, _vp]),
    "hp_server_submit_map": (_int, [_vp, _u32, _u64, _vp, _vp, _vp, _vp, _vp, _vp, _u32, _dbl, _int, _u64, _vp,
                                    _vp]),
    "hp_server_poll": (_int, [_vp, _u64, _vp]),
    "hp_server_wait": (_int, [_vp, _u64, _vp, _vp, _vp]),
    "hp_server_last_error": (ctypes.c_char_p, [_vp]),
    "hp_server_destroy": (_int, [_vp]),
    "hp_read_metis": (_int, [ctypes.c_char_p, _vp]),
    "hp_gen_grid": (_int, [_u32, _u32, _i32, _i32, _u64, _vp]),
    "hp_gen_rmat": (_int, [_u32, _u32, _dbl, _dbl, _dbl, _i32, _i32, _u64, _int, _vp]),
    "hp_gen_rgg3d": (_int, [_u32, _dbl, _i32, _i32, _u64, _int, _vp]),
    "hp_host_graph_info": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "hp_host_graph_copy": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "hp_host_graph_free": (_int, [_vp]),
    "hp_write_metis": (_int, [ctypes.c_char_p, _u32, _u64, _vp, _vp, _vp, _vp]),
    "hp_write_partition": (_int, [ctypes.c_char_p, _vp, _u32]),
}
for _name, (_res, _args) in _SIG.items():
    _f = getattr(_L, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = tuple(_SIG)


def lib():
    return _L


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _a_u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _a_i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def _host_check(rc, what):
    if rc != 0:
        raise HeiPaError(rc, what)


class Graph:
    """A host CSR graph: xadj (n+1), adj (m directed entries), optional edge
    weights ew (m) and vertex weights vw (n); None means unit weights."""

    def __init__(self, xadj, adj, ew=None, vw=None):
        self.xadj = _a_u32(xadj)
        self.adj = _a_u32(adj)
        self.ew = _a_i32(ew)
        self.vw = _a_i32(vw)
        self.n = len(self.xadj) - 1
        self.m = len(self.adj)

    @property
    def undirected_edges(self):
        return self.m // 2

    def total_weight(self):
        return int(self.n if self.vw is None else self.vw.astype(np.int64).sum())

    @staticmethod
    def _from_handle(h):
        n, m, he, hv = _u32(), _u64(), _int(), _int()
        _L.hp_host_graph_info(h, ctypes.byref(n), ctypes.byref(m), ctypes.byref(he), ctypes.byref(hv))
        xadj = np.empty(n.value + 1, np.uint32)
        adj = np.empty(m.value, np.uint32)
        ew = np.empty(m.value, np.int32) if he.value else None
        vw = np.empty(n.value, np.int32) if hv.value else None
        _L.hp_host_graph_copy(h, _p(xadj), _p(adj), _p(ew), _p(vw))
        _L.hp_host_graph_free(h)
        return Graph(xadj, adj, ew, vw)

    @staticmethod
    def read_metis(path):
        h = _vp()
        _host_check(_L.hp_read_metis(str(path).encode(), ctypes.byref(h)), f"cannot read {path}")
        return Graph._from_handle(h)

    def write_metis(self, path):
        _host_check(_L.hp_write_metis(str(path).encode(), self.n, self.m, _p(self.xadj), _p(self.adj), _p(self.ew),
                                      _p(self.vw)), f"cannot write {path}")

    @staticmethod
    def grid(w, h, w_lo=0, w_hi=0, seed=0):
        g = _vp()
        _host_check(_L.hp_gen_grid(w, h, w_lo, w_hi, seed, ctypes.byref(g)), "grid generator failed")
        return Graph._from_handle(g)

    @staticmethod
    def rmat(scale, edge_factor, a=0.57, b=0.19, c=0.19, w_lo=1, w_hi=10, seed=0, explicit_vw=False):
        g = _vp()
        _host_check(_L.hp_gen_rmat(scale, edge_factor, a, b, c, w_lo, w_hi, seed, int(explicit_vw), ctypes.byref(g)),
                    "rmat generator failed")
        return Graph._from_handle(g)

    @staticmethod
    def rgg3d(n, mean_degree, w_lo=1, w_hi=100, seed=0, explicit_vw=True):
        g = _vp()
        _host_check(_L.hp_gen_rgg3d(n, mean_degree, w_lo, w_hi, seed, int(explicit_vw), ctypes.byref(g)),
                    "rgg generator failed")
        return Graph._from_handle(g)


class BatchItem(ctypes.Structure):
    """Mirror of hp_batch_item (include/gpuheipa.h)."""
    _fields_ = [("n", ctypes.c_uint32), ("m", ctypes.c_uint64), ("xadj", _vp), ("adj", _vp), ("ew", _vp),
                ("vw", _vp), ("k", ctypes.c_uint32), ("imbalance", ctypes.c_double), ("ultra", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("part", _vp), ("cut", ctypes.c_int64), ("status", ctypes.c_int)]


class Server:
    """Serving loop (hp_server_*): submit partitioning / mapping requests as
    they arrive; each runs as soon as a worker and device memory are free.
    The host arrays of a request are kept alive here until it is waited on."""

    def __init__(self, device=0, buffer_bytes=8 << 30, workers=8):
        self.h = _vp()
        rc = _L.hp_server_create(device, buffer_bytes, workers, ctypes.byref(self.h))
        if rc != 0:
            self.h = None
            raise HeiPaError(rc, "server creation failed")
        self._keep = {}

    def submit_partition(self, g, k, imbalance=0.03, config="default", seed=0):
        part = np.empty(g.n, np.uint32)
        rid = _u64()
        _host_check(_L.hp_server_submit_partition(self.h, g.n, g.m, _p(g.xadj), _p(g.adj), _p(g.ew), _p(g.vw), int(k),
                                                  float(imbalance), int(config == "ultra"), int(seed), _p(part),
                                                  ctypes.byref(rid)), "submit failed")
        self._keep[rid.value] = (g, part)
        return rid.value

    def submit_map(self, g, hierarchy, distance, imbalance=0.03, config="HM", seed=0):
        hier, dist = _a_u32(hierarchy), _a_i32(distance)
        part = np.empty(g.n, np.uint32)
        rid = _u64()
        _host_check(_L.hp_server_submit_map(self.h, g.n, g.m, _p(g.xadj), _p(g.adj), _p(g.ew), _p(g.vw), _p(hier),
                                            _p(dist), len(hier), float(imbalance), MAP_MODES[config], int(seed),
                                            _p(part), ctypes.byref(rid)), "submit failed")
        self._keep[rid.value] = (g, part, hier, dist)
        return rid.value

    def done(self, rid):
        d = _int()
        _L.hp_server_poll(self.h, rid, ctypes.byref(d))
        return bool(d.value)

    def wait(self, rid):
        """Returns (part, objective, latency_ms, run_ms)."""
        obj, lat, run = _i64(), _dbl(), _dbl()
        rc = _L.hp_server_wait(self.h, rid, ctypes.byref(obj), ctypes.byref(lat), ctypes.byref(run))
        keep = self._keep.pop(rid, None)
        if rc != 0:
            raise HeiPaError(rc, _L.hp_server_last_error(self.h).decode())
        return keep[1], obj.value, lat.value, run.value

    def close(self):
        if self.h:
            _L.hp_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def kernel_launches():
    """Kernels launched by this process through the library so far."""
    return int(_L.hp_kernel_launches())


DEVERR_SPIN = 8  # device error bit: a bounded wait gave up


def initial_partition(g, k, imbalance=0.03, seed=0):
    """The reference's host k-way partitioner on host graph g, rows in their
    given order (hp_initial_partition); returns the labels."""
    part = np.empty(g.n, np.uint32)
    _host_check(_L.hp_initial_partition(g.n, _p(g.xadj), _p(g.adj), _p(g.vw), _p(g.ew), int(k), float(imbalance),
                                        int(seed), _p(part)), "initial partition failed")
    return part


def coop_slot_acquire(device=0, timeout_ms=0):
    """Takes the device's cooperative-launch slot (hp_coop_slot_acquire).
    Returns False when another holder kept it for timeout_ms."""
    rc = _L.hp_coop_slot_acquire(device, int(timeout_ms))
    if rc == 8:
        return False
    _host_check(rc, "cooperative slot acquire failed")
    return True


def coop_slot_release(device=0):
    """Returns the device's cooperative-launch slot (hp_coop_slot_release)."""
    _host_check(_L.hp_coop_slot_release(device), "cooperative slot release failed")


def selftest_barrier_timeout(device=0, blocks=4):
    """Runs hp_selftest_barrier_timeout: a cooperative kernel in which one
    block never reaches the grid barrier. Returns (error bits, kernel ms)."""
    err = ctypes.c_uint32(0)
    ms = ctypes.c_double(0.0)
    rc = _L.hp_selftest_barrier_timeout(device, blocks, ctypes.byref(err), ctypes.byref(ms))
    if rc != 0:
        raise HeiPaError(rc, "barrier self-test failed")
    return err.value, ms.value


def edge_cut_noalloc(n, m, d_xadj, d_adj, d_ew, part, stream=0):
    """Edge cut of a caller-owned device CSR (integer device addresses of
    uint32 xadj[n+1], uint32 adj[m] and int32 ew[m] or None) under a host
    partition, computed without any allocation (hp_edge_cut_noalloc). `stream`
    is a cudaStream_t handle (0: the legacy default stream). Calls on one
    device share a fixed scratch area and must not overlap."""
    part = _a_u32(part)
    if len(part) != n:
        raise HeiPaError(1, "partition length differs from n")
    c = _i64()
    rc = _L.hp_edge_cut_noalloc(n, m, d_xadj, d_adj, d_ew, _p(part), stream or None, ctypes.byref(c))
    if rc == 7:
        raise HeiPaError(rc, f"n = {n} exceeds the limit of {EDGE_CUT_NOALLOC_MAX_N} vertices")
    _host_check(rc, "edge cut without allocation failed")
    return c.value


def write_partition(path, part):
    part = _a_u32(part)
    _host_check(_L.hp_write_partition(str(path).encode(), _p(part), len(part)), f"cannot write {path}")


def arena_estimate(n, m, has_ew=True, has_vw=True):
    return int(_L.hp_arena_estimate(n, m, int(has_ew), int(has_vw)))


class DeviceGraph:
    def __init__(self, ctx, handle):
        self.ctx, self.h = ctx, handle
        n, m, w = _u32(), _u64(), _i64()
        _L.hp_graph_info(handle, ctypes.byref(n), ctypes.byref(m), ctypes.byref(w))
        self.n, self.m, self.total_vw = n.value, m.value, w.value

    def free(self):
        if self.h:
            self.ctx._check(_L.hp_graph_free(self.ctx.h, self.h))
            self.h = None

    def download(self):
        xadj = np.empty(self.n + 1, np.uint32)
        adj = np.empty(self.m, np.uint32)
        ew = np.empty(self.m, np.int32)
        vw = np.empty(self.n, np.int32)
        self.ctx._check(_L.hp_graph_download(self.ctx.h, self.h, _p(xadj), _p(adj), _p(ew), _p(vw)))
        return Graph(xadj, adj, ew, vw)


class Jet:
    """One level of Jet refinement driven step by step."""

    def __init__(self, ctx, dgraph, k, lmax, part, hierarchy=None, distance=None):
        self.ctx, self.n, self.k = ctx, dgraph.n, int(k)
        part = _a_u32(part)
        hier = None if hierarchy is None else _a_u32(hierarchy)
        dist = None if distance is None else _a_i32(distance)
        h = _vp()
        ctx._check(_L.hp_jet_begin(ctx.h, dgraph.h, self.k, int(lmax), _p(part), _p(hier), _p(dist),
                                   0 if hier is None else len(hier), ctypes.byref(h)))
        self.h = h

    def _moves(self, fn, *args):
        out = np.empty(self.n, np.uint32)
        c = _u32()
        self.ctx._check(fn(self.h, *args, _p(out), ctypes.byref(c)))
        return out[:c.value].copy()

    def lp(self, ratio_pct):
        return self._moves(_L.hp_jet_lp, _u32(int(ratio_pct)))

    def weak(self):
        return self._moves(_L.hp_jet_weak)

    def strong(self):
        return self._moves(_L.hp_jet_strong)

    def perform(self, obj):
        o, mw = _i64(int(obj)), _i32(0)
        self.ctx._check(_L.hp_jet_perform(self.h, ctypes.byref(o), ctypes.byref(mw)))
        return o.value, mw.value

    def state(self):
        n, k = self.n, self.k
        st = dict(map=np.empty(n, np.uint32), bw=np.empty(k, np.int32), dest_part=np.empty(n, np.uint32),
                  gain1=np.empty(n, np.int32), lock=np.empty(n, np.uint32), dest_cache=np.empty(n, np.uint32),
                  gain_cache=np.empty(n, np.int32))
        self.ctx._check(_L.hp_jet_state(self.h, *[_p(st[x]) for x in
                                                  ("map", "bw", "dest_part", "gain1", "lock", "dest_cache",
                                                   "gain_cache")]))
        return st

    def close(self):
        if self.h:
            _L.hp_jet_end(self.h)
            self.h = None


class Context:
    """A device, a stream and a device-memory arena (LIFO like the
    reference's KokkosMemoryStack)."""

    def __init__(self, device=0, arena_bytes=1 << 30):
        h = _vp()
        rc = _L.hp_ctx_create(int(device), int(arena_bytes), ctypes.byref(h))
        if rc != 0:
            raise HeiPaError(rc, "context creation failed")
        self.h = h

    def close(self):
        if self.h:
            _L.hp_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise HeiPaError(rc, _L.hp_last_error(self.h).decode())

    def last_error(self):
        return _L.hp_last_error(self.h).decode()

    def arena_peak(self):
        return int(_L.hp_arena_peak(self.h))

    def upload(self, g):
        h = _vp()
        self._check(_L.hp_graph_upload(self.h, g.n, g.m, _p(g.xadj), _p(g.adj), _p(g.ew), _p(g.vw),
                                       ctypes.byref(h)))
        return DeviceGraph(self, h)

    def match(self, dg):
        mp = np.empty(dg.n, np.uint32)
        nc = _u32()
        self._check(_L.hp_match(self.h, dg.h, _p(mp), ctypes.byref(nc)))
        return mp, nc.value

    def contract(self, dg, mapping, n_coarse):
        mapping = _a_u32(mapping)
        h = _vp()
        self._check(_L.hp_contract(self.h, dg.h, _p(mapping), int(n_coarse), ctypes.byref(h)))
        return DeviceGraph(self, h)

    def jet_refine(self, dg, k, lmax, part, obj, maxw, ultra=False, level=0, hierarchy=None, distance=None):
        part = _a_u32(part).copy()
        o, mw = _i64(int(obj)), _i32(int(maxw))
        hier = None if hierarchy is None else _a_u32(hierarchy)
        dist = None if distance is None else _a_i32(distance)
        self._check(_L.hp_jet_refine(self.h, dg.h, int(k), int(lmax), int(bool(ultra)), int(level), _p(part),
                                     ctypes.byref(o), ctypes.byref(mw), _p(hier), _p(dist),
                                     0 if hier is None else len(hier)))
        return part, o.value, mw.value

    def jet(self, dg, k, lmax, part, hierarchy=None, distance=None):
        return Jet(self, dg, k, lmax, part, hierarchy, distance)

    def edge_cut(self, dg, part):
        part = _a_u32(part)
        c = _i64()
        self._check(_L.hp_edge_cut(self.h, dg.h, _p(part), ctypes.byref(c)))
        return c.value

    def comm_cost(self, dg, part, hierarchy, distance):
        part, hier, dist = _a_u32(part), _a_u32(hierarchy), _a_i32(distance)
        c = _i64()
        self._check(_L.hp_comm_cost(self.h, dg.h, _p(part), _p(hier), _p(dist), len(hier), ctypes.byref(c)))
        return c.value

    def partition(self, g, k, imbalance=0.03, config="default", seed=0, out=None):
        """GPU-HeiPa: host graph in, host partition out (upload and download
        included)."""
        if config not in ("default", "ultra"):
            raise ValueError("config must be 'default' or 'ultra'")
        part = np.empty(g.n, np.uint32) if out is None else out
        c = _i64()
        self._check(_L.hp_partition(self.h, g.n, g.m, _p(g.xadj), _p(g.adj), _p(g.ew), _p(g.vw), int(k),
                                    float(imbalance), int(config == "ultra"), int(seed), _p(part), ctypes.byref(c)))
        return part, c.value

    def partition_graph(self, dg, k, imbalance=0.03, config="default", seed=0, out=None):
        part = np.empty(dg.n, np.uint32) if out is None else out
        c = _i64()
        self._check(_L.hp_partition_graph(self.h, dg.h, int(k), float(imbalance), int(config == "ultra"), int(seed),
                                          _p(part), ctypes.byref(c)))
        return part, c.value

    def process_map(self, g, hierarchy, distance, imbalance=0.03, config="HM", seed=0, out=None):
        """GPU-HeiProMap: returns (mapping, J) with J over directed entries."""
        hier, dist = _a_u32(hierarchy), _a_i32(distance)
        part = np.empty(g.n, np.uint32) if out is None else out
        J = _i64()
        self._check(_L.hp_map(self.h, g.n, g.m, _p(g.xadj), _p(g.adj), _p(g.ew), _p(g.vw), _p(hier), _p(dist),
                              len(hier), float(imbalance), MAP_MODES[config], int(seed), _p(part), ctypes.byref(J)))
        return part, J.value

    def process_map_graph(self, dg, hierarchy, distance, imbalance=0.03, config="HM", seed=0, out=None):
        hier, dist = _a_u32(hierarchy), _a_i32(distance)
        part = np.empty(dg.n, np.uint32) if out is None else out
        J = _i64()
        self._check(_L.hp_map_graph(self.h, dg.h, _p(hier), _p(dist), len(hier), float(imbalance), MAP_MODES[config],
                                    int(seed), _p(part), ctypes.byref(J)))
        return part, J.value

    def partition_batch(self, graphs, ks, imbalance=0.03, config="default", seed=0, workers=8):
        """hp_partition_batch: [(part, cut)] for graphs[i] with ks[i] blocks."""
        items = (BatchItem * len(graphs))()
        parts = []
        for i, (g, k) in enumerate(zip(graphs, ks)):
            part = np.empty(g.n, np.uint32)
            parts.append(part)
            items[i] = BatchItem(g.n, g.m, _p(g.xadj), _p(g.adj), _p(g.ew), _p(g.vw), int(k), float(imbalance),
                                 int(config == "ultra"), int(seed), _p(part), 0, 0)
        self._check(_L.hp_partition_batch(self.h, items, len(graphs), workers))
        return [(parts[i], items[i].cut) for i in range(len(graphs))]

    def last_solve_stats(self):
        ms = (ctypes.c_double * 5)()
        o, lm, lv = _i64(), _i32(), _u32()
        self._check(_L.hp_last_solve_stats(self.h, ms, ctypes.byref(o), ctypes.byref(lm), ctypes.byref(lv)))
        keys = ("coarsening", "contraction", "initial_partitioning", "uncontraction", "refinement")
        im, fm = _i32(), _i32()
        self._check(_L.hp_last_solve_maxw(self.h, ctypes.byref(im), ctypes.byref(fm)))
        sizes, ln, lmm = [], _u32(), _u64()
        while _L.hp_last_solve_level(self.h, len(sizes), ctypes.byref(ln), ctypes.byref(lmm)) == 0:
            sizes.append((ln.value, lmm.value))
        return dict(phase_ms=dict(zip(keys, list(ms))), initial_obj=o.value, lmax=lm.value, levels=lv.value,
                    initial_maxw=im.value, final_maxw=fm.value, level_sizes=sizes)

    def event_record(self, slot):
        self._check(_L.hp_event_record(self.h, int(slot)))

    def event_elapsed(self, a, b):
        ms = ctypes.c_float()
        self._check(_L.hp_event_elapsed(self.h, int(a), int(b), ctypes.byref(ms)))
        return ms.value

    def profile(self, enable=True):
        """Diagnostic phase timers (synchronising)."""
        self._check(_L.hp_profile(self.h, int(enable)))

    def profile_entries(self):
        out = {}
        i = 0
        buf = ctypes.create_string_buffer(64)
        ms, cnt = ctypes.c_double(), _u64()
        while _L.hp_profile_entry(self.h, i, buf, 64, ctypes.byref(ms), ctypes.byref(cnt)) == 0:
            out[buf.value.decode()] = (ms.value, cnt.value)
            i += 1
        return out

    def tune(self, name, value):
        """hp_tune: set a size threshold between equivalent implementations."""
        self._check(_L.hp_tune(self.h, name.encode(), int(value)))

    def instrument(self, enable=True):
        self._check(_L.hp_instrument(self.h, int(enable)))

    def kernel_log(self):
        """Per-launch kernel-timer records [(name, ms, bytes)] in launch order."""
        out, i = [], 0
        buf = ctypes.create_string_buffer(64)
        ms, by = _dbl(), _dbl()
        while _L.hp_kernel_log(self.h, i, buf, 64, ctypes.byref(ms), ctypes.byref(by)) == 0:
            out.append((buf.value.decode(), ms.value, by.value))
            i += 1
        return out

    def kernel_timing(self, name):
        l, ms, b = _u64(), ctypes.c_double(), ctypes.c_double()
        self._check(_L.hp_kernel_timing(self.h, name.encode(), ctypes.byref(l), ctypes.byref(ms), ctypes.byref(b)))
        return dict(launches=l.value, ms=ms.value, bytes=b.value)


def partition(g, k, imbalance=0.03, config="default", seed=0, device=0):
    with Context(device, arena_estimate(g.n, g.m, g.ew is not None, g.vw is not None)) as ctx:
        return ctx.partition(g, k, imbalance, config, seed)


def process_map(g, hierarchy, distance, imbalance=0.03, config="HM", seed=0, device=0):
    with Context(device, arena_estimate(g.n, g.m, g.ew is not None, g.vw is not None)) as ctx:
        return ctx.process_map(g, hierarchy, distance, imbalance, config, seed)
