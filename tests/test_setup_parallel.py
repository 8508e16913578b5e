"""The set-up's row-parallel pair enumeration (csrc/setup/topology.cpp pairs_within_rows) and
the non-bonded repulsion list built on it (csrc/setup/parameters.cpp generate_repulsion): the
list is every non-bonded pair within 20 bohr, ordered by (i, j), whatever the number of
threads; and the set-up CN, which leaves out the partners whose term is exactly zero, against
a plain restatement of the 1600 bohr^2 threshold form (cn_calculator.cpp:115-177)."""
import os
import subprocess
import sys
from math import erf, exp, log
from pathlib import Path

import numpy as np

from curcuma_b200 import workloads
from tests.oracle_api import Oracle, BOHR_A

ROOT = Path(__file__).resolve().parent.parent
SNIPPET = """
import hashlib, numpy as np
from curcuma_b200 import workloads
from tests.oracle_api import Oracle
Z, X = workloads.water_cluster(300, 17)
o = Oracle(Z, X)
rep = o.topology(5, 2)
print(len(rep), hashlib.sha256(np.ascontiguousarray(rep, dtype=np.int64).tobytes()).hexdigest())
"""


def _run(threads):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    out = subprocess.run([sys.executable, "-c", SNIPPET], cwd=ROOT, env=env, capture_output=True, text=True,
                         check=True)
    return out.stdout.split()


def test_repulsion_list_independent_of_threads():
    assert _run(1) == _run(4)


def test_repulsion_list_is_every_nonbonded_pair_within_20_bohr():
    Z, X = workloads.water_cluster(300, 17)       # 900 atoms: the grid path
    o = Oracle(Z, X)
    rep = [tuple(p) for p in o.topology(5, 2)]
    bonded = {tuple(sorted(p)) for p in o.topology(11, 2)}
    xb = X / BOHR_A
    d2 = ((xb[:, None, :] - xb[None, :, :]) ** 2).sum(-1)
    i, j = np.nonzero(np.triu(d2 <= 400.0, 1))
    want = [(a, b) for a, b in zip(i.tolist(), j.tolist()) if (a, b) not in bonded]
    assert rep == want                             # same pairs, ordered by (i, j)


def test_setup_cn_against_plain_threshold_sum():
    Z, X = workloads.water_cluster(300, 17)
    o = Oracle(Z, X)
    xb = X / BOHR_A
    # per-atom CN radii as the set-up uses them: 4/3 Pyykko radius (Angstrom) x 1.8897259886
    pyykko = {1: 0.32, 8: 0.63}
    rc = np.array([4.0 / 3.0 * pyykko[int(z)] * 1.8897259886 for z in Z])
    want = np.zeros(len(Z))
    for a in range(len(Z)):
        d2 = ((xb - xb[a]) ** 2).sum(-1)
        js = [b for b in range(len(Z)) if b != a and d2[b] <= 1600.0]
        s = 0.0
        for b in js:                               # ascending partner order, every partner
            r = d2[b] ** 0.5
            s += 0.5 * (1.0 + erf(-7.5 * ((r - (rc[a] + rc[b])) / (rc[a] + rc[b]))))
        want[a] = log(1.0 + exp(4.4)) - log(1.0 + exp(4.4 - s))
    got = o.atom_data(1)                           # the set-up CN
    assert np.abs(got - want).max() < 1e-13
