"""ORACLE — test infrastructure only. Recipe that compiles the reference's own
host initial partitioner (GPU_HeiPa::ModifiedMetis, the plain-C++ headers
src/initial_partitioning/kway_partitioner/kway_*.h) from its sources where
they lie, into oracle/_ref/libkway_ref.so, without the reference's build
system and without Kokkos:

  oracle/_ref/src/initial_partitioning/kway_partitioner/*.h  symlinks to the
      reference's headers (unmodified, not copied)
  oracle/_ref/src/utility/definitions.h, oracle/_ref/src/datastructures/graph.h
      symlinks to the stand-ins in oracle/ref_shim/ (kway_core.h resolves its
      two Kokkos-bound includes, "../../utility/definitions.h" and
      "../../datastructures/graph.h", relative to the symlinked header)
  oracle/kway_ref.cpp  the C entry point, compiled with -I oracle/_ref

Outputs go only to oracle/_ref/ (git-ignored). Without a reference tree (for
example on a machine that only runs the tests) the prebuilt library is kept.
"""
import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("GPU_HEIPA_REFERENCE", "/root/reference")
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libkway_ref.so")
KWAY_DIR = os.path.join("src", "initial_partitioning", "kway_partitioner")


def _link(src, dst):
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    if os.path.islink(dst) or os.path.exists(dst):
        if os.path.islink(dst) and os.readlink(dst) == src:
            return
        os.unlink(dst)
    os.symlink(src, dst)


def build_ref(force=False):
    """Builds oracle/_ref/libkway_ref.so; returns its path, or None when neither
    the reference sources nor a prebuilt library are available."""
    headers = sorted(glob.glob(os.path.join(REF, KWAY_DIR, "kway_*.h")))
    if not headers:
        return LIB if os.path.exists(LIB) else None
    for h in headers:
        _link(h, os.path.join(OUT, KWAY_DIR, os.path.basename(h)))
    _link(os.path.join(HERE, "ref_shim", "utility", "definitions.h"),
          os.path.join(OUT, "src", "utility", "definitions.h"))
    _link(os.path.join(HERE, "ref_shim", "datastructures", "graph.h"),
          os.path.join(OUT, "src", "datastructures", "graph.h"))
    deps = headers + [os.path.join(HERE, "kway_ref.cpp")] + glob.glob(os.path.join(HERE, "ref_shim", "*", "*.h"))
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps):
        return LIB
    cmd = ["g++", "-O2", "-std=c++20", "-fPIC", "-shared", "-I" + OUT, os.path.join(HERE, "kway_ref.cpp"), "-o", LIB]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build_ref(force=True))
