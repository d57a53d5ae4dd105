"""The oracle's parallel loops give the same results on one host thread and on
all of them (CPU only). Each side runs in its own process so that
OMP_NUM_THREADS takes effect when the OpenMP runtime starts."""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

SCRIPT = r"""
import hashlib, json, sys
sys.path[:0] = [sys.argv[1], sys.argv[2], sys.argv[3]]
import numpy as np
import gpu_heipa as H
import oracle as O
from helpers import to_oracle

def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()

out = {"threads": O.threads()}
r = H.Graph.rmat(15, 16, seed=11)
g = to_oracle(r)
mp, nc = O.match(g)
out["match"] = [digest(mp), int(nc)]
c = O.contract(g, mp, nc)
out["contract"] = [digest(a) for a in c.arrays() if a is not None]
for ultra in (False, True):
    p, cut = O.partition(g, 64, 0.03, ultra, 5)
    out["partition_%d" % ultra] = [digest(p), int(cut)]
m = to_oracle(H.Graph.rgg3d(20000, 14.0, 1, 100, seed=8, explicit_vw=True))
p, J = O.map_hm(m, [2, 4, 3], [1, 10, 100], 0.03, False, 3)
out["hm"] = [digest(p), int(J)]
p, J = O.map_im(m, [2, 4, 3], [1, 10, 100], 0.03, 3)
out["im"] = [digest(p), int(J)]
print(json.dumps(out))
"""


def _run(threads):
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    else:
        env.pop("OMP_NUM_THREADS", None)
    r = subprocess.run([sys.executable, "-c", SCRIPT, os.path.join(ROOT, "gpu-heipa_b200"),
                        os.path.join(ROOT, "oracle"), HERE],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_oracle_results_do_not_depend_on_threads():
    one = _run(1)
    many = _run(4)
    assert one.pop("threads") == 1
    assert many.pop("threads") == 4
    assert one == many
