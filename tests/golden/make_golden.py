"""Pack the reference's golden vectors into tests/golden/ref100.npz.

Reads, from a checkout of the reference project (default /root/reference):
  tests/XcT_ref100.in                       100-fiber input layout
  tests/config.ini                          the run configuration
  tests/reference/100_{numeric,analytic}_{gmres,direct}/{0,1}_{BVec,XVec,
      TRANSVel,ROTVel,POS,ORIENT}.ref       Fortran validate-mode outputs
The .ref files are F16.8, one value per line (fortran/fibers.f95:205-303).
The *_AMat.ref files and reference.map are not part of the reference checkout,
so A is pinned only through b, x and everything downstream of them.

Run:  python tests/golden/make_golden.py [reference_root]
"""
import configparser
import json
import os
import sys

import numpy as np

FIELDS = ["BVec", "XVec", "TRANSVel", "ROTVel", "POS", "ORIENT"]
VARIANTS = ["numeric_gmres", "numeric_direct", "analytic_gmres", "analytic_direct"]


def main(root):
    out = {}
    with open(os.path.join(root, "tests", "XcT_ref100.in")) as fh:
        n = int(fh.readline())
        rows = [list(map(float, fh.readline().split())) for _ in range(2 * n)]
    rows = np.array(rows, dtype=np.float64)
    out["positions"] = rows[0::2]
    out["orientations"] = rows[1::2]
    cfg = configparser.ConfigParser()
    cfg.read(os.path.join(root, "tests", "config.ini"))
    conf = {s: dict(cfg[s]) for s in cfg.sections()}
    out["config_json"] = np.array(json.dumps(conf))
    for v in VARIANTS:
        for t in (0, 1):
            for f in FIELDS:
                p = os.path.join(root, "tests", "reference", "100_" + v, "%d_%s.ref" % (t, f))
                out["%s/%d_%s" % (v, t, f)] = np.loadtxt(p, dtype=np.float64)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref100.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, len(out), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
