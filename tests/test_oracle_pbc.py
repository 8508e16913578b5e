"""The oracle's periodic boundary conditions: the minimum-image convention of curcuma's CUDA
kernels (ff_methods/cuda/gfnff_kernels.cu:92-119 applyMIC and its callers), restated in
oracle/gfnff_oracle.cpp.  curcuma applies the minimum image to the displacement vectors of
the CN and its chain rule, bonds, angles, HB/XB A-H, H-B, A-B vectors, HB coordination
numbers, repulsion, Coulomb and D4 pairs, and not to torsions, inversions, ATM, BATM, the
EEQ matrix (its charges come from plain distances) or the set-up lists.  No curcuma output
for a periodic GFN-FF system exists to pin against: these tests check the restatement's
rules.

* a cell much larger than the system changes nothing (the minimum image is the plain
  difference);
* two waters whose O-H...O contact crosses a cell face: the CN of the contact atoms and the
  Coulomb, D4 and repulsion terms see the image, the plain set-up does not;
* a water box in a cell slightly larger than itself: the periodic contacts change the
  Coulomb, D4 and repulsion terms and leave torsions, inversions, ATM and BATM alone;
* moving one molecule by a lattice vector (cubic and triclinic cells) leaves the
  minimum-image terms (bonds, angles, D4, repulsion, CN) unchanged while the charges move
  (the EEQ matrix uses plain distances, as in curcuma)."""
import math

import numpy as np
import pytest

from curcuma_b200 import workloads
from tests.oracle_api import Oracle


def _box(nw=48, seed=5, gap=2.8):
    Z, X = workloads.water_cluster(nw, seed)
    L = workloads.water_box_edge(nw) + gap
    return Z, X, L


def water(o, u):
    """O at o, the first O-H bond along the unit vector u (Angstrom)."""
    r, ang = 0.9572, math.radians(104.52)
    u = np.asarray(u, float) / np.linalg.norm(u)
    w = np.cross(u, [0.0, 0.0, 1.0])
    if np.linalg.norm(w) < 1e-6:
        w = np.cross(u, [0.0, 1.0, 0.0])
    w /= np.linalg.norm(w)
    h1 = o + r * u
    h2 = o + r * (math.cos(ang) * u + math.sin(ang) * w)
    return [o, h1, h2]


def face_dimer(L=10.0, contact=1.85):
    """Water A near x = 0 with an O-H pointing along -x; water B near x = L whose O is
    `contact` Angstrom from that H through the x face (plainly ~L away)."""
    a = water(np.array([0.6, L / 2, L / 2]), [-1.0, 0.0, 0.0])
    ob = a[1] + np.array([-contact, 0.0, 0.0]) + np.array([L, 0.0, 0.0])
    b = water(ob, [0.3, 1.0, 0.2])
    return np.array([8, 1, 1, 8, 1, 1]), np.array(a + b)


def test_large_cell_is_the_isolated_system():
    Z, X, L = _box()
    T0, G0, q0, cn0 = Oracle(Z, X).engrad(X)
    T1, G1, q1, cn1 = Oracle(Z, X, unit_cell=np.eye(3) * 10 * L).engrad(X)
    for k in T0:
        assert abs(T0[k] - T1[k]) < 1e-10, k
    assert np.abs(G0 - G1).max() < 1e-10
    assert np.abs(cn0 - cn1).max() < 1e-12


def test_contact_through_a_face():
    Z, X = face_dimer()
    T0, G0, q0, cn0 = Oracle(Z, X).engrad(X)
    T1, G1, q1, cn1 = Oracle(Z, X, unit_cell=np.eye(3) * 10.0).engrad(X)
    # the H of A and the O of B count each other through the face
    assert cn1[1] - cn0[1] > 1e-7 and cn1[3] - cn0[3] > 1e-7
    assert (cn1 >= cn0 - 1e-12).all()                  # image partners only add
    for k in ("coulomb", "dispersion", "nonbonded_rep"):
        assert abs(T1[k] - T0[k]) > 1e-6, k
    assert T1["dispersion"] < T0["dispersion"]
    assert np.abs(G1[:, 0] - G0[:, 0]).max() > 1e-5   # the contact acts along x
    assert abs(G1.sum(axis=0)).max() < 1e-9           # minimum-image forces still balance


def test_periodic_contacts_in_a_water_box():
    Z, X, L = _box()
    T0, G0, q0, cn0 = Oracle(Z, X).engrad(X)
    T1, G1, q1, cn1 = Oracle(Z, X, unit_cell=np.eye(3) * L).engrad(X)
    assert (cn1 >= cn0 - 1e-12).all()
    for k in ("coulomb", "dispersion", "nonbonded_rep"):
        assert abs(T1[k] - T0[k]) > 1e-6, k
    for k in ("torsion", "inversion", "atm", "batm", "storsion"):
        assert abs(T1[k] - T0[k]) < 1e-12, k
    assert T1["dispersion"] < T0["dispersion"]       # more partners at shorter distances
    assert abs(q1.sum()) < 1e-10


@pytest.mark.parametrize("skew", [False, True], ids=["cubic", "triclinic"])
def test_lattice_translation_of_one_molecule(skew):
    Z, X, L = _box()
    cell = np.eye(3) * L
    if skew:
        cell[1] = [0.3 * L, L, 0.0]       # b tilted in the a-b plane
        cell[2] = [0.2 * L, -0.1 * L, L]
    o = Oracle(Z, X, unit_cell=cell)      # set-up at X; evaluations at X and at X2
    T1, G1, q1, cn1 = o.engrad(X)
    X2 = X.copy()
    X2[3:6] += cell[0] - cell[2]          # the second water, shifted by a - c
    T2, G2, q2, cn2 = o.engrad(X2)
    assert np.abs(cn2 - cn1).max() < 1e-12
    for k in ("bond", "angle", "dispersion", "bonded_rep", "nonbonded_rep"):
        assert abs(T2[k] - T1[k]) < 1e-10, k
    assert np.abs(q2 - q1).max() > 1e-6     # the EEQ matrix sees the plain distances


def test_singular_cell_is_refused():
    Z, X, L = _box(8, 3)
    with pytest.raises(RuntimeError):
        Oracle(Z, X, unit_cell=[[L, 0, 0], [2 * L, 0, 0], [0, 0, L]])
