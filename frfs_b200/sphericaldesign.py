"""Antipodal spherical designs for the half-sphere quadrature.

The reference loads a 2M-point symmetric (antipodal) design and keeps the
first M points (frfs/solvers/dgfs/velocitymesh.py:128-135,
frfs/sphericaldesign/__init__.py:84-107).  Q depends only on the M axes
{+s, -s}, so a design is given here by one point of each antipodal pair.

Built in (closed form):
  M = 1   two poles (0, 0, +-1)
  M = 3   octahedron (a spherical 3-design)
  M = 6   icosahedron with a vertex at (0, 0, 1) and one at
          (2/sqrt(5), 0, 1/sqrt(5)): the orientation of the reference's
          12-point Womersley design, so the axes coincide with it
  M = 12  the 24 points (+-1, +-1, +-c)/|.| and permutations with
          c^2 = 3 + sqrt(10): the octahedral orbit that is an exact spherical
          5-design (the average of x^4 + y^4 + z^4 over the orbit equals the
          sphere average 3/5 exactly for this c).  The reference ships no
          24-point design (its files hold 2, 6, 12, 32, ... points), so
          M = 12 is supplied here.
Any other M: pass ``ssrule`` as a file path with 2M rows "x y z" (the
reference's file format), the first M rows are used.

The gas-mixture operator integrates over the full sphere
(frfs/solvers/dgfsbi/velocitymesh.py:158-166): ``full_sphere_design(M)``
is the M-point antipodal design, a built-in half design of M/2 points and
its antipodes, or the M rows of a design file.
"""
import os

import numpy as np


def _icosahedron_half():
    pts = [(0.0, 0.0, 1.0)]
    r, z = 2.0 / np.sqrt(5.0), 1.0 / np.sqrt(5.0)
    for k in range(5):
        ang = -2.0 * np.pi * k / 5.0
        pts.append((r * np.cos(ang), r * np.sin(ang), z))
    return np.array(pts)


def _octahedral_5design_half():
    c = np.sqrt(3.0 + np.sqrt(10.0))
    half = []
    for pos in range(3):
        others = [i for i in range(3) if i != pos]
        for s1 in (1.0, -1.0):
            for s2 in (1.0, -1.0):
                v = [0.0, 0.0, 0.0]
                v[pos], v[others[0]], v[others[1]] = c, s1, s2
                half.append(v)
    return np.array(half) / np.sqrt(2.0 + c * c)


def half_sphere_design(M, ssrule='womersley'):
    """M points, one from each antipodal pair of a 2M-point design."""
    if ssrule and os.path.isfile(str(ssrule)):
        pts = np.loadtxt(ssrule)[:, :3]
        if pts.shape[0] != 2 * M:
            raise ValueError(f'design file has {pts.shape[0]} points, need {2 * M}')
        return pts[:M].copy()
    if M == 1:
        return np.array([[0.0, 0.0, 1.0]])
    if M == 3:
        return np.eye(3)[[2, 0, 1]]
    if M == 6:
        return _icosahedron_half()
    if M == 12:
        return _octahedral_5design_half()
    raise ValueError('No suitable spherical quadrature rule found '
                     f'(built-in M in 1, 3, 6, 12; got M={M}); pass a file')


def full_sphere_design(M, ssrule='womersley'):
    """M points of an antipodal design on the whole sphere."""
    if ssrule and os.path.isfile(str(ssrule)):
        pts = np.loadtxt(ssrule)[:, :3]
        if pts.shape[0] != M:
            raise ValueError(f'design file has {pts.shape[0]} points, need {M}')
        return pts.copy()
    if M % 2:
        raise ValueError(f'built-in full-sphere designs have an even number of points (got M={M})')
    half = half_sphere_design(M // 2)
    return np.concatenate([half, -half])
