"""Regenerates the golden fixtures in this directory from RUMD's own data.

The RUMD source tree ships equilibrated Kob-Andersen configurations
(``Conf/KobAndersen/*.xyz.gz``) whose particle lines carry the forces, the
per-particle potential energy and (in the newer files) the per-particle virial
that RUMD itself computed for those positions with Pot_LJ_12_6, a shifted
potential (SP) cut-off at 2.5 sigma_ij and the KA parameters.  They are the
reference's golden vectors for the pair force path.  This script parses them
(format written by src/ConfigurationWriterReader.cu:90-180; ``vir`` is w.w/2,
line 173) and stores compact ``.npz`` fixtures so that the tests do not need
the reference tree.  Two of the files are also copied unchanged into conf/
for the configuration-reader tests.

Usage:  python tests/golden/make_golden.py RUMD_SOURCE_TREE
"""
import gzip
import os
import sys

import numpy as np

FILES = [
    "N100L4.6.xyz.gz",
    "N256L6.0.xyz.gz",
    "KA_N256_L6.0_T0.50.xyz.gz",
    "N864L9.0.xyz.gz",
    "KA_N864_L9.0_T0.80.xyz.gz",
    "KA_N1000_T0.5.xyz.gz",
    "KA_N1000_T1.0.xyz.gz",
    "KA_N1000_T5.0.xyz.gz",
    "KA_N1024_T0.8.xyz.gz",
    "N1372L10.456.xyz.gz",
    "N2000L11.86.xyz.gz",
    "KA_N4096_T0.8.xyz.gz",
]


def parse(path):
    with gzip.open(path, "rt") as fh:
        n = int(fh.readline().split()[0])
        header = fh.readline().split()
        meta = {}
        for tok in header:
            if "=" in tok:
                k, v = tok.split("=", 1)
                meta[k] = v
        cols = meta["columns"].split(",")
        rows = [fh.readline().split() for _ in range(n)]
    arr = {c: np.array([r[k] for r in rows]) for k, c in enumerate(cols)}
    L = np.array([float(x) for x in meta["boxLengths"].split(",")], np.float64)
    out = {
        "L": L,
        "type": arr["type"].astype(np.int32),
        "pos": np.stack([arr[c].astype(np.float64) for c in ("x", "y", "z")], 1),
        "vel": np.stack([arr[c].astype(np.float64) for c in ("vx", "vy", "vz")], 1),
        "force": np.stack([arr[c].astype(np.float64) for c in ("fx", "fy", "fz")], 1),
        "pe": arr["pe"].astype(np.float64),
        "xi": float(meta.get("Nose-Hoover-Ps", "0")),
    }
    if "vir" in arr:
        out["vir"] = arr["vir"].astype(np.float64)
    if "imx" in arr:
        out["im"] = np.stack([arr[c].astype(np.int32) for c in ("imx", "imy", "imz")], 1)
    return out


# RUMD's own configuration files, copied unchanged for the reader tests: one
# in ioformat=1 (dt, boxLengths, Nose-Hoover-Ps) and one in ioformat=2
# (integrator=IntegratorNVT,dt,T,tau,xi and sim_box=RectangularSimulationBox,
# two types of unequal mass)
RAW = [
    ("Conf/KobAndersen", "KA_N256_L6.0_T0.50.xyz.gz"),
    ("Conf/SingleComponentLiquid", "MgCu_equil_0.051_0.055.xyz.gz"),
]


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py RUMD_SOURCE_TREE")
    root = sys.argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    for name in FILES:
        d = parse(os.path.join(root, "Conf", "KobAndersen", name))
        stem = name.replace(".xyz.gz", "")
        np.savez_compressed(os.path.join(here, f"ka_{stem}.npz"), **d)
        print(stem, len(d["type"]), "vir" in d)
    import shutil
    os.makedirs(os.path.join(here, "conf"), exist_ok=True)
    for sub, name in RAW:
        shutil.copyfile(os.path.join(root, sub, name), os.path.join(here, "conf", name))
        print("copied", name)


if __name__ == "__main__":
    main()
