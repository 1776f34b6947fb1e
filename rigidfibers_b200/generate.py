"""Seeded synthetic fiber layouts.

`sphere_layout`: centres uniform in a ball of radius `radius` (cube rejection),
rejecting any centre closer than `min_distance` to an accepted one;
orientations uniform on the unit sphere (normalised standard normal).  This
stands in for the thesis' concentration-controlled scenes; the reference's
own generator (tools/gen2.f95) enforces a segment-segment distance instead.

`serving_radius`: sphere radius for a circumscribed-sphere volume fraction
phi = N (L/2)^3 / R^3 (L = 2), i.e. R = (N / phi)^(1/3).
"""
import numpy as np


def layout_seed(config_id, n):
    return 1000003 * config_id + n


def sphere_layout(n, radius, min_distance=0.2, seed=0, max_tries=200):
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = np.empty((n, 3))
    count = 0
    cell = max(min_distance, 1e-9)
    grid = {}
    tries = 0
    while count < n:
        cand = rng.uniform(-radius, radius, size=(4 * (n - count) + 16, 3))
        cand = cand[np.einsum("ij,ij->i", cand, cand) <= radius * radius]
        for c in cand:
            key = tuple(np.floor(c / cell).astype(int))
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        for idx in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                            d = pts[idx] - c
                            if d @ d < min_distance * min_distance:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                pts[count] = c
                grid.setdefault(key, []).append(count)
                count += 1
                if count == n:
                    break
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place %d fibers in radius %g" % (n, radius))
    ori = rng.standard_normal((n, 3))
    ori /= np.linalg.norm(ori, axis=1, keepdims=True)
    return pts, ori


def serving_radius(n, phi=0.01):
    return (n / phi) ** (1.0 / 3.0)
