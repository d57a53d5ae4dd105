"""CPU checks of the C ABI boundary: the shared library loads, exports every
function include/gpuheipa.h declares, and rejects bad arguments on the host
without device work. Also checks that the product never reaches the oracle."""
import ctypes
import os
import re
import subprocess

import pytest

import gpu_heipa as H
from conftest import has_gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gpuheipa.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = _declared()
    assert len(names) >= 40
    out = subprocess.run(["nm", "-D", "--defined-only", H.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = ctypes.CDLL(H.LIB_PATH)
    for n in names:
        assert getattr(lib, n) is not None


def test_binding_covers_header():
    assert sorted(H.EXPORTED) == _declared()


def test_host_side_rejections():
    L = H.lib()
    assert L.hp_last_error(None) == b"null context"
    assert L.hp_arena_peak(None) == 0
    c = ctypes.c_int64()
    # hp_edge_cut_noalloc: null result pointer, null arrays, oversize n.
    assert L.hp_edge_cut_noalloc(4, 0, None, None, None, None, None, None) == 1
    x = (ctypes.c_uint32 * 8)()
    assert L.hp_edge_cut_noalloc(4, 0, ctypes.cast(x, ctypes.c_void_p), None, None, None, None,
                                 ctypes.byref(c)) == 1
    assert L.hp_edge_cut_noalloc(H.EDGE_CUT_NOALLOC_MAX_N + 1, 0, ctypes.cast(x, ctypes.c_void_p), None, None,
                                 ctypes.cast(x, ctypes.c_void_p), None, ctypes.byref(c)) == 7
    # Null handles on context-bound calls.
    assert L.hp_edge_cut(None, None, None, None) == 1
    assert L.hp_partition_graph(None, None, 4, 0.03, 0, 0, None, None) == 1


def test_arena_estimate_monotone():
    a = H.arena_estimate(1000, 10000)
    b = H.arena_estimate(2000, 10000)
    c = H.arena_estimate(2000, 20000)
    assert 0 < a < b < c


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_context_without_device_is_an_error():
    with pytest.raises(H.HeiPaError):
        H.Context(0, 1 << 20)


def test_product_does_not_use_oracle():
    # The package and the C ABI must not import, link or load the oracle.
    pat = re.compile(r"\boracle\b|liboracle|\bor_[a-z_]+\(")
    hits = []
    for base in (os.path.join(ROOT, "gpu-heipa_b200"), os.path.join(ROOT, "include")):
        for dirpath, dirs, files in os.walk(base):
            dirs[:] = [d for d in dirs if d not in ("_build", "lib", "bin", "__pycache__")]
            for f in files:
                if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                    path = os.path.join(dirpath, f)
                    for i, line in enumerate(open(path, errors="replace"), 1):
                        code = line.split("//")[0].split("#")[0]
                        if pat.search(code):
                            hits.append(f"{path}:{i}: {line.strip()}")
    assert not hits, hits
