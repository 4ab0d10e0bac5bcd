"""Writes tests/golden/periodic_map.npz: the reference's full-to-reduced node map of the
periodic voxel grid (``PeriodicVoxelMap.reduced_of_full``, src/phast/solid3d/periodic.py:40-123)
for grids periodic on every axis, on some axes and on none, including one-voxel axes.

Usage: python tests/golden/make_golden_periodic_map.py <path to the reference's src directory>
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

GRIDS = [((3, 4, 5), (True, True, True)), ((3, 4, 5), (False, True, False)), ((2, 1, 3), (True, True, False)),
         ((1, 1, 1), (True, True, True)), ((4, 3, 2), (False, False, False))]


def main(src):
    from make_golden import _import_reference
    _import_reference(src)
    from phast.solid3d.model import VoxelGrid
    from phast.solid3d.periodic import PeriodicVoxelMap
    out = {}
    for n, (shape, per) in enumerate(GRIDS):
        pmap = PeriodicVoxelMap.build(VoxelGrid(shape, (0.1, 0.2, 0.3), periodic=per))
        out[f"shape_{n}"] = np.array(shape)
        out[f"periodic_{n}"] = np.array(per)
        out[f"reduced_shape_{n}"] = np.array(pmap.reduced_shape)
        out[f"rof_{n}"] = pmap.reduced_of_full.numpy()
    out["n"] = np.array([len(GRIDS)])
    np.savez(os.path.join(HERE, "periodic_map.npz"), **out)


if __name__ == "__main__":
    main(sys.argv[1])
