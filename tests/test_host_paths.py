"""The host symbolic analysis keeps its structures as bit rows up to a size
limit (16384 unknowns) and in sorted vectors and ordered sets beyond it (the
Min-Fill ordering has one sparse path at every size). Both representations
must give identical orderings, filled patterns, LU programs, level schedules
and stamp maps. KARAM_BITROW_MAX moves the limit, so the large-problem code
runs here on small cases in a child process and its tables are compared with
the default path's. CPU only."""
import os
import pickle
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = ("config1", "config2", "grid8", "grid12", "grid16")

DUMP = r"""
import pickle, sys
sys.path.insert(0, sys.argv[1])
import karam_b200 as K
from karam_b200 import circuits
out = {}
for name in sys.argv[3].split(","):
    nl = getattr(circuits, name)() if not name.startswith("grid") else circuits.grid_circuit(int(name[4:]))
    p = K.Problem(None, nl)
    raw, perm, tw = p.ordering()
    sched = p.lu_schedule()
    out[name] = dict(raw=raw, perm=perm, tw=tw, filled=p.filled_pattern(), prog=p.lu_program(),
                     smap=p.stamp_map(), sched=sched, info=p.info)
    p.close()
with open(sys.argv[2], "wb") as fh:
    pickle.dump(out, fh)
"""


def dump(tmp_path, tag, env_extra):
    path = tmp_path / f"{tag}.pkl"
    env = dict(os.environ, **env_extra)
    subprocess.run([sys.executable, "-c", DUMP, ROOT, str(path), ",".join(CASES)], check=True,
                   env=env, timeout=600)
    with open(path, "rb") as fh:
        return pickle.load(fh)


def same(a, b):
    if isinstance(a, dict):
        return a.keys() == b.keys() and all(same(a[k], b[k]) for k in a)
    if isinstance(a, (tuple, list)):
        return len(a) == len(b) and all(same(x, y) for x, y in zip(a, b))
    if isinstance(a, np.ndarray):
        return np.array_equal(a, b)
    return a == b


@pytest.mark.timeout(900)
def test_large_problem_host_paths_give_identical_tables(tmp_path):
    default = dump(tmp_path, "bits", {"KARAM_BITROW_MAX": ""})
    sparse = dump(tmp_path, "sets", {"KARAM_BITROW_MAX": "0"})
    for name in CASES:
        for key in default[name]:
            assert same(default[name][key], sparse[name][key]), (name, key)
