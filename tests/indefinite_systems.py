"""Systems whose reduced EEQ matrix is indefinite: an H2 molecule at the bond length of
curcuma's HH reference case (0.471 A) contributes one unknown with a negative diagonal (the
hydrogen hardness is negative, and at that distance the pair's Coulomb kernel exceeds the
atoms' self terms), so a chain of such H2 molecules with a few waters beside it takes the
pivoted-LU fallback.  The chain spans more than 90 bohr, so the exact-gradient mode's charge response
(a second solve with the same factor) runs too."""
import numpy as np

from curcuma_b200 import workloads


def h2_chain(n_h2=30, spacing=3.5, n_water=8, seed=3, bond=0.471):
    rng = np.random.default_rng(seed)
    Z, X = [], []
    for k in range(n_h2):
        c = np.array([k * spacing, 0.0, 0.0])
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        Z += [1, 1]
        X += [c - 0.5 * bond * u, c + 0.5 * bond * u]
    Zw, Xw = workloads.water_cluster(n_water, seed)
    Xw = Xw - Xw.mean(axis=0) + np.array([n_h2 * spacing / 2, 6.0, 0.0])
    return np.concatenate([np.array(Z), Zw]), np.concatenate([np.array(X), Xw])
