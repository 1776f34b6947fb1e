"""Pack the reference's golden vectors into tests/golden/ref100.npz.

Reads, from a checkout of the reference project (its root is a required argument):
  tests/XcT_ref100.in                       100-fiber input layout
  tests/config.ini                          the run configuration
  tests/reference/100_{numeric,analytic}_{gmres,direct}/{0,1}_{BVec,XVec,
      TRANSVel,ROTVel,POS,ORIENT}.ref       Fortran validate-mode outputs
The .ref files are F16.8, one value per line (fortran/fibers.f95:205-303).
The *_AMat.ref files and reference.map are not part of the reference checkout,
so A is pinned only through b, x and everything downstream of them.

It also writes tests/golden/ref2000_stats.json: the packing statistics of the
reference's 2000-fiber benchmark layout tests/XcT_ref2000.in (made by its
generator tools/gen2.f95), which the generator tests compare against.

Run:  python tests/golden/make_golden.py <reference_root>
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
    stats = layout_stats(os.path.join(root, "tests", "XcT_ref2000.in"))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref2000_stats.json")
    with open(dst, "w") as fh:
        json.dump(stats, fh, indent=1, sort_keys=True)
        fh.write("\n")
    print("wrote", dst)


def read_xct(path):
    with open(path) as fh:
        n = int(fh.readline())
        rows = np.array([list(map(float, fh.readline().split())) for _ in range(2 * n)], dtype=np.float64)
    return rows[0::2], rows[1::2]


def layout_stats(path):
    """Packing statistics of an XcT layout: fiber count, radius of the
    smallest origin-centred sphere holding every centre, minimum and mean
    nearest-neighbour centre distance, and the minimum segment-segment
    distance (segments centre +- orientation)."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from rigidfibers_b200.generate import layout_statistics
    pos, ori = read_xct(path)
    st = layout_statistics(pos, ori)
    st["source"] = "tests/XcT_ref2000.in of the reference (generator tools/gen2.f95, min distance 0.2)"
    return st


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference_root>")
    main(sys.argv[1])
