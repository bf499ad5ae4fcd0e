"""Regenerate the golden fixtures from the reference's own test data.

    python tests/golden/make_golden.py /path/to/galfast      (or GALFAST_REFERENCE=/path/to/galfast)

reads tests/os_vel2pm/result/sky.obs.txt of the reference (the output of its
postprocessing test, tests/os_vel2pm/go.sh) and writes os_vel2pm_sky_obs.npz
beside this script: the columns lb[2] absSDSSr SDSSr comp XYZ[3] radec[2]
vcyl[3] pmlb[3] as printed (XYZ in the galactocentric convention of that
file, which vcyl2pm uses internally).
"""
import os
import sys

import numpy as np


def main(ref):
    path = os.path.join(ref, "tests", "os_vel2pm", "result", "sky.obs.txt")
    rows = np.loadtxt(path)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "os_vel2pm_sky_obs.npz")
    np.savez_compressed(out, lb=rows[:, 0:2], absmag=rows[:, 2], mag=rows[:, 3], comp=rows[:, 4].astype(np.int32),
                        XYZ=rows[:, 5:8], radec=rows[:, 8:10], vcyl=rows[:, 10:13], pmlb=rows[:, 13:16])
    print("wrote", out, rows.shape)


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GALFAST_REFERENCE")
    if not src:
        sys.exit("usage: make_golden.py <galfast source tree> (or set GALFAST_REFERENCE)")
    main(src)
