"""Extract small golden fixtures from the reference's own committed outputs.

Reads (only when run, in a checkout that has the reference mounted):
  Taylor_Green_Vortex/Initial_particle_information.dat   t = 0 state of the
      100 x 100 Taylor-Green run (X Y VX VY RHO P/pressure_0), 10 decimals
  Taylor_Green_Vortex/Kinetic_energy.dat                  KE/KE0 every 100 steps
  Taylor_Green_Vortex/Maximum_velocity_magnitude.dat      max |u|/U every 100 steps
Writes tests/golden/tgv_reference.npz (every 10th particle row and the first
50 rows of both time series).  The tests never read the reference tree.

Usage: python tests/golden/make_golden.py <path of the reference checkout>
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def rows(path, ncol):
    out = []
    for line in open(path):
        t = line.split()
        if len(t) != ncol:
            continue
        try:
            out.append([float(x) for x in t])
        except ValueError:
            pass
    return np.array(out)


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the reference checkout>")
    tgv = os.path.join(sys.argv[1], "Taylor_Green_Vortex")
    init = rows(os.path.join(tgv, "Initial_particle_information.dat"), 6)
    assert init.shape == (10000, 6), init.shape
    idx = np.arange(0, 10000, 10)
    ke = rows(os.path.join(tgv, "Kinetic_energy.dat"), 2)[:50]
    vmax = rows(os.path.join(tgv, "Maximum_velocity_magnitude.dat"), 2)[:50]
    np.savez_compressed(os.path.join(HERE, "tgv_reference.npz"), init_index=idx, init_rows=init[idx],
                        kinetic_energy=ke, max_velocity=vmax)
    print("wrote", os.path.join(HERE, "tgv_reference.npz"))


if __name__ == "__main__":
    main()
