"""Writes tests/golden/reference_fixtures.npz from the reference's own data files.

Run where the reference checkout is present (it is not on the machines that run
the GPU tests and the benchmark, which read only the .npz written here):

    python tests/golden/make_reference_fixtures.py [REFERENCE_ROOT]

Contents (each array exactly as the reference loads it):
  leaf_mask      2D/vortex/data/leaf_mask_256_scaled.npz["mask"], uint8 256x256: the
                 obstacle of the vortex experiment (2D/vortex/lfm_midpoint_simulator.py:406,418)
  density_G_2d,  2D/shape/data/density_{G,R}_arial_scaled_shifted_0.8.npy, uint8 256x256:
  density_R_2d   initial / target density of the 2D shape experiment
                 (2D/shape/optimize_shape_G_R.py:435,442)
  density_G_3d,  3D/model/density_{G,R}_centered_1.2x_128x128.npy, float64 128x128: the
  density_R_3d   glyphs the 3D shape experiment extrudes along z (3D/optimize_shape_G_R.py:204-218)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root="/root/reference"):
    j = lambda *p: os.path.join(ref_root, *p)
    out = {
        "leaf_mask": np.load(j("2D", "vortex", "data", "leaf_mask_256_scaled.npz"))["mask"],
        "density_G_2d": np.load(j("2D", "shape", "data", "density_G_arial_scaled_shifted_0.8.npy")),
        "density_R_2d": np.load(j("2D", "shape", "data", "density_R_arial_scaled_shifted_0.8.npy")),
        "density_G_3d": np.load(j("3D", "model", "density_G_centered_1.2x_128x128.npy")),
        "density_R_3d": np.load(j("3D", "model", "density_R_centered_1.2x_128x128.npy")),
    }
    path = os.path.join(HERE, "reference_fixtures.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(*sys.argv[1:])
