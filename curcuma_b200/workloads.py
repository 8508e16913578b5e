"""Seeded synthetic structures for the GFN-FF benchmark configurations.

No public dataset is involved; every structure is generated from a seed (1000 + config
index by default):

1. ``alkane(64)``: n-C64H130, all-trans, C-C 1.54 A, C-H 1.09 A, tetrahedral angles, then
   Gaussian noise (sigma 0.05 A) on every coordinate.
2. ``water_cluster(1000)``: O placed by rejection sampling in a cube at 1.0 g/cm^3 with
   O-O >= 2.6 A; rigid waters (0.9572 A, 104.52 deg) with uniform random orientations.
   Orientations are re-drawn while an intermolecular H...H < 1.4 A or H...O < 1.5 A, so
   every water stays its own molecular fragment.
3. ``solvated_peptide(50, 1500)``: Gly50 (standard backbone geometry, phi/psi drawn from
   the beta region +-20 deg) inside 1500 waters.
4. ``conformer_batch(512)``: saturated C/N/O chains, size log-uniform in [20, 300] atoms,
   heteroatom fraction 0.15, branching probability 0.1, torsions uniform in [0, 2 pi),
   hydrogens filled to valence.
5. ``large_cluster()``: 6000 waters + 40 C20H42 at random positions and orientations,
   heavy-atom overlaps rejected at 2.0 A.

All coordinates are Angstrom; element numbers follow the periodic table.
"""
import math

import numpy as np

H, C, N, O = 1, 6, 7, 8
TET = math.radians(109.4712)
BOND = {(C, C): 1.54, (C, H): 1.09, (C, N): 1.47, (C, O): 1.43, (N, H): 1.01, (O, H): 0.96,
        (N, N): 1.45, (N, O): 1.40, (O, O): 1.48}
VALENCE = {C: 4, N: 3, O: 2}
AVOGADRO = 6.02214076e23


def bond_len(a, b):
    return BOND.get((a, b)) or BOND.get((b, a))


def place(a, b, c, r, theta, phi):
    """NeRF: position of d with |cd| = r, angle bcd = theta, dihedral abcd = phi."""
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    nn = np.linalg.norm(n)
    if nn < 1e-8:
        # colinear reference: pick any perpendicular
        t = np.array([1.0, 0.0, 0.0]) if abs(bc[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
        n = np.cross(t, bc)
        nn = np.linalg.norm(n)
    n /= nn
    m = np.cross(n, bc)
    d2 = np.array([-r * math.cos(theta), r * math.sin(theta) * math.cos(phi), r * math.sin(theta) * math.sin(phi)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


def random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


class Tree:
    """Tree-shaped molecule built atom by atom in internal coordinates."""

    def __init__(self):
        self.Z, self.X, self.parent, self.children = [], [], [], []

    def add(self, z, x, parent):
        self.Z.append(z)
        self.X.append(np.asarray(x, dtype=float))
        self.parent.append(parent)
        self.children.append([])
        if parent >= 0:
            self.children[parent].append(len(self.Z) - 1)
        return len(self.Z) - 1

    def ref_frame(self, i):
        """(xa, xb, b): new substituents of i are placed with dihedral a-b-i-new, where b
        is bonded to i and a is bonded to b."""
        b = self.parent[i] if self.parent[i] >= 0 else self.children[i][0]
        cand = ([self.parent[b]] if self.parent[b] >= 0 else []) + self.children[b]
        cand = [a for a in cand if a != i]
        xa = self.X[cand[0]] if cand else self.X[b] + np.array([0.0, 1.0, 0.3])
        return xa, self.X[b], b

    def arrays(self):
        return np.array(self.Z, dtype=np.int32), np.array(self.X)


def fill_hydrogens(t: Tree, rng=None):
    """Adds H to every heavy atom up to its valence at tetrahedral positions."""
    nheavy = len(t.Z)
    for i in range(nheavy):
        z = t.Z[i]
        if z not in VALENCE:
            continue
        nb = len(t.children[i]) + (1 if t.parent[i] >= 0 else 0)
        need = VALENCE[z] - nb
        if need <= 0:
            continue
        pa, pb, b = t.ref_frame(i)
        # dihedrals of the heavy substituents other than the frame atom b
        used = []
        for c in t.children[i]:
            if c != b:
                used.append(_dihedral(pa, pb, t.X[i], t.X[c]))
        base = used[0] if used else (rng.uniform(0, 2 * math.pi) if rng is not None else math.pi)
        slots = [base + k * 2 * math.pi / 3 for k in range(3)]
        free = [s for s in slots if all(abs(_wrap(s - u)) > 0.5 for u in used)]
        for k in range(need):
            phi = free[k % len(free)] if free else base + math.pi
            t.add(H, place(pa, pb, t.X[i], bond_len(z, H), TET, phi), i)


def _wrap(a):
    return (a + math.pi) % (2 * math.pi) - math.pi


def _dihedral(a, b, c, d):
    b0, b1, b2 = a - b, c - b, d - c
    b1n = b1 / np.linalg.norm(b1)
    v = b0 - np.dot(b0, b1n) * b1n
    w = b2 - np.dot(b2, b1n) * b1n
    x = np.dot(v, w)
    y = np.dot(np.cross(b1n, v), w)
    return math.atan2(y, x)


def alkane(nc=64, seed=1001, sigma=0.05, noise=True):
    t = Tree()
    x0 = np.zeros(3)
    t.add(C, x0, -1)
    t.add(C, x0 + np.array([bond_len(C, C), 0, 0]), 0)
    t.add(C, place(np.array([0.0, 1.0, 0.0]), t.X[0], t.X[1], bond_len(C, C), TET, math.pi), 1)
    for k in range(3, nc):
        t.add(C, place(t.X[k - 3], t.X[k - 2], t.X[k - 1], bond_len(C, C), TET, math.pi), k - 1)
    fill_hydrogens(t)
    Z, X = t.arrays()
    if noise:
        rng = np.random.default_rng(seed)
        X = X + rng.normal(scale=sigma, size=X.shape)
    return Z, X


def water_geometry():
    r, ang = 0.9572, math.radians(104.52)
    o = np.zeros(3)
    h1 = np.array([r * math.sin(ang / 2), r * math.cos(ang / 2), 0.0])
    h2 = np.array([-r * math.sin(ang / 2), r * math.cos(ang / 2), 0.0])
    com = (15.999 * o + 1.008 * (h1 + h2)) / 18.015
    return np.array([o, h1, h2]) - com


class Grid:
    """Spatial hash for the rejection tests."""

    def __init__(self, cell=3.0):
        self.cell = cell
        self.cells = {}

    def key(self, x):
        return tuple(np.floor(x / self.cell).astype(int))

    def add(self, x, z):
        self.cells.setdefault(self.key(x), []).append((x, z))

    def near(self, x, r):
        k = self.key(x)
        m = int(math.ceil(r / self.cell))
        for dx in range(-m, m + 1):
            for dy in range(-m, m + 1):
                for dz in range(-m, m + 1):
                    for item in self.cells.get((k[0] + dx, k[1] + dy, k[2] + dz), ()):
                        yield item


def _fits(grid, atoms, zs, min_heavy, min_any=1.2, min_hh=1.4, min_ho=1.5):
    for x, z in zip(atoms, zs):
        for y, zy in grid.near(x, max(min_heavy, min_hh, min_ho)):
            d = np.linalg.norm(x - y)
            if z != H and zy != H and d < min_heavy:
                return False
            if z == H and zy == H and d < min_hh:
                return False
            if (z == H) != (zy == H) and d < min_ho:
                return False
            if d < min_any:
                return False
    return True


def solvate(rng, n_water, box, grid=None, Z=None, X=None, min_oo=2.6, center=None):
    Zs = [] if Z is None else list(Z)
    Xs = [] if X is None else list(X)
    grid = grid or Grid()
    wg = water_geometry()
    placed = 0
    tries = 0
    while placed < n_water:
        tries += 1
        if tries > 2000 * n_water:
            raise RuntimeError("water placement did not converge")
        o = rng.uniform(0.0, box, size=3) if center is None else center + rng.uniform(-box / 2, box / 2, size=3)
        ok = True
        for y, zy in grid.near(o, min_oo):
            if zy != H and np.linalg.norm(o - y) < min_oo:
                ok = False
                break
        if not ok:
            continue
        for _ in range(20):
            Rm = random_rotation(rng)
            atoms = o + wg @ Rm.T
            if _fits(grid, atoms, [O, H, H], min_oo):
                break
        else:
            continue
        for x, z in zip(atoms, [O, H, H]):
            grid.add(x, z)
            Xs.append(x)
            Zs.append(z)
        placed += 1
    return np.array(Zs, dtype=np.int32), np.array(Xs), grid


def water_box_edge(n_water, density=1.0, extra_volume=0.0):
    vol = n_water * 18.015 / (AVOGADRO * density) * 1e24 + extra_volume
    return vol ** (1.0 / 3.0)


def water_cluster(n_water=1000, seed=1002):
    rng = np.random.default_rng(seed)
    Z, X, _ = solvate(rng, n_water, water_box_edge(n_water))
    return Z, X


def glycine_chain(nres=50, rng=None):
    """H-(Gly)n-OH, standard backbone geometry, phi/psi in the beta region +-20 deg."""
    t = Tree()
    phi0, psi0 = math.radians(-120.0), math.radians(130.0)
    d = math.radians(20.0)
    nN = t.add(N, np.zeros(3), -1)
    ca = t.add(C, np.array([1.458, 0.0, 0.0]), nN)
    cc = t.add(C, place(np.array([0.0, 1.0, 0.0]), t.X[nN], t.X[ca], 1.525, math.radians(111.2), math.pi), ca)
    prev = (nN, ca, cc)
    for r in range(nres):
        nN, ca, cc = prev
        psi = psi0 + rng.uniform(-d, d)
        phi = phi0 + rng.uniform(-d, d)
        # carbonyl O trans to the next N
        if r < nres - 1:
            n2 = t.add(N, place(t.X[nN], t.X[ca], t.X[cc], 1.329, math.radians(116.2), psi), cc)
            t.add(O, place(t.X[nN], t.X[ca], t.X[cc], 1.231, math.radians(120.1), psi + math.pi), cc)
            ca2 = t.add(C, place(t.X[ca], t.X[cc], t.X[n2], 1.458, math.radians(121.7), math.pi), n2)
            t.add(H, place(t.X[ca], t.X[cc], t.X[n2], 1.01, math.radians(119.0), 0.0), n2)
            c2 = t.add(C, place(t.X[cc], t.X[n2], t.X[ca2], 1.525, math.radians(111.2), phi), ca2)
            prev = (n2, ca2, c2)
        else:
            o1 = t.add(O, place(t.X[nN], t.X[ca], t.X[cc], 1.34, math.radians(112.0), psi), cc)
            t.add(O, place(t.X[nN], t.X[ca], t.X[cc], 1.21, math.radians(124.0), psi + math.pi), cc)
            t.add(H, place(t.X[ca], t.X[cc], t.X[o1], 0.97, math.radians(106.0), math.pi), o1)
    # hydrogens on CA (2 each) and the N terminus (2)
    nheavy = len(t.Z)
    for i in range(nheavy):
        z = t.Z[i]
        nb = len(t.children[i]) + (1 if t.parent[i] >= 0 else 0)
        if z == C and nb == 2:       # glycine CA
            p = t.parent[i]
            ch = [c for c in t.children[i] if t.Z[c] != H][0]
            for s in (+1, -1):
                t.add(H, place(t.X[ch], t.X[p], t.X[i], 1.09, TET, s * 2 * math.pi / 3 + _dihedral(t.X[ch], t.X[p], t.X[i], t.X[ch]) * 0), i)
        if z == N and t.parent[i] < 0:   # N terminus NH2
            ca0 = t.children[i][0]
            c0 = [c for c in t.children[ca0] if t.Z[c] == C][0]
            for phi in (math.radians(60.0), math.radians(-60.0)):
                t.add(H, place(t.X[c0], t.X[ca0], t.X[i], 1.01, TET, phi), i)
    return t.arrays()


def solvated_peptide(nres=50, n_water=1500, seed=1003):
    rng = np.random.default_rng(seed)
    Zp, Xp = glycine_chain(nres, rng)
    Xp = Xp - Xp.mean(axis=0)
    ext = np.ptp(Xp, axis=0).max()
    pep_vol = 4.0 / 3.0 * math.pi * (1.7 ** 3) * len(Zp) * 0.5
    box = max(water_box_edge(n_water, extra_volume=pep_vol), ext + 6.0)
    Xp = Xp + box / 2
    grid = Grid()
    for x, z in zip(Xp, Zp):
        grid.add(x, z)
    Z, X, _ = solvate(rng, n_water, box, grid, Zp, Xp)
    return Z, X


def random_chain(n_atoms_target, rng, hetero=0.15, branch=0.1, max_attempts=400):
    """Saturated C/N/O tree with H filled to valence; about n_atoms_target atoms.

    Heavy atoms grow with torsions uniform in [0, 2 pi); a new heavy atom is redrawn while
    it comes closer than 3.0 A to a heavy atom three or more bonds away, and a finished
    molecule is rejected while two atoms not within two bonds are closer than 1.0 A (H-H),
    1.5 A (H-heavy) or 2.0 A (heavy-heavy), so the bond graph seen by the force field is
    the constructed one."""
    for _attempt in range(max_attempts):
        t = Tree()
        t.add(C, np.zeros(3), -1)
        t.add(C, np.array([bond_len(C, C), 0.0, 0.0]), 0)
        open_sites = {0: VALENCE[C] - 1, 1: VALENCE[C] - 1}
        tip = 1

        def n_est():
            return len(t.Z) + sum(max(0, VALENCE[z] - (len(t.children[i]) + (t.parent[i] >= 0)))
                                  for i, z in enumerate(t.Z))

        def near2(i):
            s1 = set([i] + t.children[i] + ([t.parent[i]] if t.parent[i] >= 0 else []))
            s2 = set(s1)
            for a in s1:
                s2 |= set(t.children[a] + ([t.parent[a]] if t.parent[a] >= 0 else []))
            return s2

        stalled = 0
        while n_est() < n_atoms_target and stalled < 400:
            base = tip
            if rng.random() < branch:
                cands = [i for i, s_ in open_sites.items() if s_ > 1 and t.Z[i] == C]
                if cands:
                    base = cands[rng.integers(len(cands))]
            if open_sites.get(base, 0) <= 1:
                cands = [i for i, s_ in open_sites.items() if s_ > 1]
                if not cands:
                    break
                base = cands[-1]
            z = C if rng.random() >= hetero else (N if rng.random() < 0.5 else O)
            if t.Z[base] in (N, O) and z in (N, O):
                z = C
            pa, pb, fb = t.ref_frame(base)
            used = [_dihedral(pa, pb, t.X[base], t.X[c]) for c in t.children[base] if c != fb]
            if used:   # further substituents sit in the remaining tetrahedral slots
                slots = [used[0] + k * 2 * math.pi / 3 for k in (1, 2)]
                slots = [s_ for s_ in slots if all(abs(_wrap(s_ - u)) > 0.5 for u in used)]
                if not slots:
                    stalled += 1
                    continue
                phi = slots[rng.integers(len(slots))]
            else:
                phi = rng.uniform(0, 2 * math.pi)
            x = place(pa, pb, t.X[base], bond_len(t.Z[base], z), TET, phi)
            skip = near2(base)
            if any(np.linalg.norm(x - t.X[k]) < 3.0 for k in range(len(t.Z)) if k not in skip):
                stalled += 1
                continue
            i = t.add(z, x, base)
            open_sites[base] -= 1
            open_sites[i] = VALENCE[z] - 1
            tip = i if open_sites[i] > 0 else tip
        fill_hydrogens(t, rng)
        Z, X = t.arrays()
        n = len(Z)
        adj = [set() for _ in range(n)]
        for i, p_ in enumerate(t.parent):
            if p_ >= 0:
                adj[i].add(p_)
                adj[p_].add(i)
        d = np.linalg.norm(X[:, None, :] - X[None, :, :], axis=-1)
        isH = Z == H
        # minimum non-bonded separation: H-H 1.0, H-heavy 1.5, heavy-heavy 2.0 A
        dmin = np.where(isH[:, None] & isH[None, :], 1.0,
                        np.where(isH[:, None] | isH[None, :], 1.5, 2.0))
        ok = True
        for i in range(n):
            close = np.nonzero(d[i] < dmin[i])[0]
            two = set(adj[i])
            for a in adj[i]:
                two |= adj[a]
            if any(j != i and j not in two for j in close):
                ok = False
                break
        if ok:
            return Z, X
    raise RuntimeError("could not build a clash-free chain")


def conformer_batch(n_mol=512, seed=1004, lo=20, hi=300):
    rng = np.random.default_rng(seed)
    mols = []
    for _ in range(n_mol):
        target = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        mols.append(random_chain(target, rng))
    return mols


def large_cluster(n_water=6000, n_alkane=40, nc=20, seed=1005):
    rng = np.random.default_rng(seed)
    Za, Xa = alkane(nc, noise=False)
    Xa = Xa - Xa.mean(axis=0)
    alk_vol = n_alkane * (282.55 / (AVOGADRO * 0.79) * 1e24)
    box = water_box_edge(n_water, extra_volume=alk_vol)
    grid = Grid()
    Z, X = [], []
    placed = 0
    while placed < n_alkane:
        R = random_rotation(rng)
        pos = rng.uniform(0, box, size=3)
        Xn = Xa @ R.T + pos
        if _fits(grid, Xn, Za, 2.0, min_any=1.2, min_hh=1.2, min_ho=1.2):
            for x, z in zip(Xn, Za):
                grid.add(x, z)
                X.append(x)
                Z.append(z)
            placed += 1
    Z, X, _ = solvate(rng, n_water, box, grid, np.array(Z), np.array(X))
    return Z, X


CONFIGS = {
    1: ("n-C64H130 all-trans + 0.05 A noise", lambda: alkane(64, 1001)),
    2: ("1000 H2O cluster, 1.0 g/cm3", lambda: water_cluster(1000, 1002)),
    3: ("Gly50 + 1500 H2O", lambda: solvated_peptide(50, 1500, 1003)),
    5: ("6000 H2O + 40 C20H42", lambda: large_cluster(6000, 40, 20, 1005)),
}
