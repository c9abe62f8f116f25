"""Tetrahedral quadrature tables (quadrature_utils.h:125-179 of the reference).

Keast 5-point rule for TET10: barycentric rows (1/4,1/4,1/4,1/4) and the
permutations with one coordinate 1/2 and three 1/6; weights
(-4/5, 9/20, 9/20, 9/20, 9/20) scaled by the unit-tet volume 1/6 (one weight is
negative).  (x, y, z) are the barycentric columns 1..3.  TET4 uses the centroid
with weight 1/6.
"""
import numpy as np

N_QP_T10_5 = 5
N_NODE_T10_10 = 10
N_QP_T4_1 = 1
N_NODE_T4_4 = 4

tet5pt_bary = np.array([
    [0.25, 0.25, 0.25, 0.25],
    [0.5, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0],
    [1.0 / 6.0, 0.5, 1.0 / 6.0, 1.0 / 6.0],
    [1.0 / 6.0, 1.0 / 6.0, 0.5, 1.0 / 6.0],
    [1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0, 0.5],
])
tet5pt_weights = np.array([-4.0 / 5.0, 9.0 / 20.0, 9.0 / 20.0, 9.0 / 20.0, 9.0 / 20.0]) * (1.0 / 6.0)
tet5pt_x = np.ascontiguousarray(tet5pt_bary[:, 1])
tet5pt_y = np.ascontiguousarray(tet5pt_bary[:, 2])
tet5pt_z = np.ascontiguousarray(tet5pt_bary[:, 3])

tet1pt_x = np.array([0.25])
tet1pt_y = np.array([0.25])
tet1pt_z = np.array([0.25])
tet1pt_weights = np.array([1.0 / 6.0])


def t10():
    return tet5pt_x, tet5pt_y, tet5pt_z, tet5pt_weights


def t4():
    return tet1pt_x, tet1pt_y, tet1pt_z, tet1pt_weights
