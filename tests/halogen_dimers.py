"""Halogen-bonded dimers CH3X...NH3 (X = Cl, Br, I): C-X...N linear, X...N 3.0 A, the N lone
pair towards X.  None of the reference fixtures has a halogen bond; these exercise the XB
term (ff_workspace_gfnff.cpp:1411-1524)."""
import numpy as np

CX = {17: 1.78, 35: 1.94, 53: 2.14}   # C-X bond lengths (A)


def dimer(x_el=35, x_n=3.0):
    C = np.array([0.0, 0.0, -CX[x_el]])
    H = [C + np.array([1.03 * np.cos(a), 1.03 * np.sin(a), -0.36]) for a in 2 * np.pi * np.arange(3) / 3]
    N = np.array([0.0, 0.0, x_n])
    HN = [N + np.array([0.94 * np.cos(a), 0.94 * np.sin(a), 0.38]) for a in 2 * np.pi * np.arange(3) / 3 + 0.5]
    Z = np.array([6, x_el, 1, 1, 1, 7, 1, 1, 1])
    return Z, np.array([C, [0.0, 0.0, 0.0], *H, N, *HN])
