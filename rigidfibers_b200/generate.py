"""Seeded synthetic fiber layouts.

`grown_sphere_layout`: the concentration-controlled scenes of the reference's
benchmark mode (tools/gen2.f95, called by runner/cuda_runner.py:253): fibers
(segments of length 2) are placed one by one in the outer shell
[r - 4 d, r] of a sphere whose radius r starts at d and grows by d whenever
1000 consecutive candidates are rejected; a candidate is rejected when its
segment-segment distance to any placed fiber is below d.  Orientations are a
uniform sample of the cube [-1,1]^3, normalised.  Written from the published
closest-point-between-segments construction (D. Sunday), vectorised over the
placed fibers.

`sphere_layout`: centres uniform in a ball of radius `radius` (cube rejection),
rejecting any centre closer than `min_distance` to an accepted one;
orientations uniform on the unit sphere (normalised standard normal).  This
stands in for the thesis' concentration-controlled scenes; the reference's
own generator (tools/gen2.f95) enforces a segment-segment distance instead.

`box_layout`: the same centre-distance rule with centres uniform in a cube,
the kind of layout of the reference's 2000-fiber benchmark file
tests/XcT_ref2000.in.

`serving_radius`: sphere radius for a circumscribed-sphere volume fraction
phi = N (L/2)^3 / R^3 (L = 2), i.e. R = (N / phi)^(1/3).
"""
import numpy as np


def layout_seed(config_id, n):
    return 1000003 * config_id + n


def _centre_rejection(rng, n, half, min_distance, in_ball, max_tries):
    """Centres drawn uniformly from the cube [-half, half]^3 (kept only inside
    the ball of radius `half` when in_ball), each rejected when it lies closer
    than min_distance to an accepted one (grid-bucketed neighbour search)."""
    pts = np.empty((n, 3))
    count = 0
    cell = max(min_distance, 1e-9)
    grid = {}
    tries = 0
    while count < n:
        cand = rng.uniform(-half, half, size=(4 * (n - count) + 16, 3))
        if in_ball:
            cand = cand[np.einsum("ij,ij->i", cand, cand) <= half * half]
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
            raise RuntimeError("could not place %d fibers in a domain of half-size %g" % (n, half))
    return pts


def sphere_layout(n, radius, min_distance=0.2, seed=0, max_tries=200):
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = _centre_rejection(rng, n, radius, min_distance, True, max_tries)
    ori = rng.standard_normal((n, 3))
    ori /= np.linalg.norm(ori, axis=1, keepdims=True)
    return pts, ori


def box_layout(n, half_side, min_distance=0.2, seed=0, max_tries=200):
    """Centres uniform in the cube [-half_side, half_side]^3 with the same
    centre-distance rejection as sphere_layout; orientations uniform on the
    unit sphere.  This is the kind of layout of the reference's 2000-fiber
    benchmark file tests/XcT_ref2000.in: its centres fill a cube of half side
    4.28 with minimum centre distance 0.2 (its segments come as close as
    1.6e-4, so it was not made by the segment-distance generator)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = _centre_rejection(rng, n, half_side, min_distance, False, max_tries)
    ori = rng.standard_normal((n, 3))
    ori /= np.linalg.norm(ori, axis=1, keepdims=True)
    return pts, ori


def serving_radius(n, phi=0.01):
    return (n / phi) ** (1.0 / 3.0)


def segment_distances2(p, o, P, O):
    """Squared distances between segments [p_b - o_b, p_b + o_b] (B of them,
    or one) and [P_k - O_k, P_k + O_k] (K of them): a (B, K) array (or (K,))."""
    single = np.ndim(p) == 1
    p = np.atleast_2d(p)[:, None, :]
    o = np.atleast_2d(o)[:, None, :]
    P = np.asarray(P)[None, :, :]
    O = np.asarray(O)[None, :, :]
    u = 2.0 * o
    v = 2.0 * O
    w = (p - o) - (P - O)
    a = np.sum(u * u, -1)
    b = np.sum(u * v, -1)
    c = np.sum(v * v, -1)
    d = np.sum(u * w, -1)
    e = np.sum(v * w, -1)
    a = np.broadcast_to(a, b.shape)
    den = a * c - b * b
    small = den < 1e-5
    sN = np.where(small, 0.0, b * e - c * d)
    sD = np.where(small, 1.0, den)
    tN = np.where(small, e, a * e - b * d)
    tD = np.where(small, c, den)
    lo = (~small) & (sN < 0.0)
    hi = (~small) & (sN > sD)
    sN = np.where(lo, 0.0, np.where(hi, sD, sN))
    tN = np.where(lo, e, np.where(hi, e + b, tN))
    tD = np.where(lo | hi, c, tD)
    tlo = tN < 0.0
    thi = tN > tD
    tN = np.where(tlo, 0.0, np.where(thi, tD, tN))
    s_lo_val = -d
    s_hi_val = -d + b
    sN = np.where(tlo, np.where(s_lo_val < 0.0, 0.0, np.where(s_lo_val > a, sD, s_lo_val)), sN)
    sD = np.where(tlo & (s_lo_val >= 0.0) & (s_lo_val <= a), a, sD)
    sN = np.where(thi, np.where(s_hi_val < 0.0, 0.0, np.where(s_hi_val > a, sD, s_hi_val)), sN)
    sD = np.where(thi & (s_hi_val >= 0.0) & (s_hi_val <= a), a, sD)
    sc = np.where(np.abs(sN) < 1e-5, 0.0, sN / sD)
    tc = np.where(np.abs(tN) < 1e-5, 0.0, tN / tD)
    dP = w + sc[..., None] * u - tc[..., None] * v
    out = np.sum(dP * dP, -1)
    return out[0] if single else out


def segment_distances2_pairs(p, o, P, O):
    """Squared distances between segments p_k +- o_k and P_k +- O_k, pairwise (K,)."""
    u = 2.0 * o
    v = 2.0 * O
    w = (p - o) - (P - O)
    a = np.sum(u * u, -1)
    b = np.sum(u * v, -1)
    c = np.sum(v * v, -1)
    d = np.sum(u * w, -1)
    e = np.sum(v * w, -1)
    den = a * c - b * b
    small = den < 1e-5
    sN = np.where(small, 0.0, b * e - c * d)
    sD = np.where(small, 1.0, den)
    tN = np.where(small, e, a * e - b * d)
    tD = np.where(small, c, den)
    lo = (~small) & (sN < 0.0)
    hi = (~small) & (sN > sD)
    sN = np.where(lo, 0.0, np.where(hi, sD, sN))
    tN = np.where(lo, e, np.where(hi, e + b, tN))
    tD = np.where(lo | hi, c, tD)
    tlo = tN < 0.0
    thi = tN > tD
    tN = np.where(tlo, 0.0, np.where(thi, tD, tN))
    s_lo_val = -d
    s_hi_val = -d + b
    sN = np.where(tlo, np.where(s_lo_val < 0.0, 0.0, np.where(s_lo_val > a, sD, s_lo_val)), sN)
    sD = np.where(tlo & (s_lo_val >= 0.0) & (s_lo_val <= a), a, sD)
    sN = np.where(thi, np.where(s_hi_val < 0.0, 0.0, np.where(s_hi_val > a, sD, s_hi_val)), sN)
    sD = np.where(thi & (s_hi_val >= 0.0) & (s_hi_val <= a), a, sD)
    sc = np.where(np.abs(sN) < 1e-5, 0.0, sN / sD)
    tc = np.where(np.abs(tN) < 1e-5, 0.0, tN / tD)
    dP = w + sc[:, None] * u - tc[:, None] * v
    return np.sum(dP * dP, -1)


def grown_sphere_layout(n, min_distance=0.2, seed=0, max_retries=1000, batch=64):
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = np.empty((n, 3))
    ori = np.empty((n, 3))
    radius = min_distance
    d2 = min_distance * min_distance
    for i in range(n):
        while True:
            placed = False
            tries = 0
            while tries < max_retries:
                rmin = max(0.0, radius - 4.0 * min_distance)
                c = rng.uniform(-radius, radius, (4 * batch, 3))
                r2 = np.einsum("ij,ij->i", c, c)
                c = c[(r2 > rmin * rmin) & (r2 < radius * radius)][:batch]
                if len(c) == 0:
                    continue
                t = rng.uniform(-1.0, 1.0, (len(c), 3))
                t /= np.linalg.norm(t, axis=1, keepdims=True)
                ok = np.ones(len(c), bool)
                if i > 0:
                    # only fibers whose centres are closer than 2 + d can come
                    # within d of the candidate (segments of half-length 1)
                    dc = c[:, None, :] - pos[None, :i, :]
                    bi, kj = np.nonzero(np.einsum("bkj,bkj->bk", dc, dc) < (2.0 + min_distance) ** 2)
                    if len(bi):
                        dd = segment_distances2_pairs(c[bi], t[bi], pos[kj], ori[kj])
                        bad = bi[dd < d2]
                        ok[bad] = False
                k = np.flatnonzero(ok)
                take = min(len(c), max_retries - tries)
                if len(k) and k[0] < take:
                    pos[i], ori[i] = c[k[0]], t[k[0]]
                    placed = True
                    break
                tries += take
            if placed:
                break
            radius += min_distance
    return pos, ori


def layout_statistics(pos, ori, chunk=256):
    """Packing statistics of a layout (fibers are segments centre +- orientation):
    fiber count, radius of the smallest origin-centred sphere holding every
    centre, minimum and mean nearest-neighbour centre distance, and minimum
    and mean nearest-neighbour segment-segment distance.  All pairs are
    compared, in row chunks (O(N^2) work, meant for N up to a few thousand)."""
    pos = np.asarray(pos, np.float64)
    ori = np.asarray(ori, np.float64)
    n = len(pos)
    nn_c = np.full(n, np.inf)
    nn_s = np.full(n, np.inf)
    for i0 in range(0, n, chunk):
        i1 = min(n, i0 + chunk)
        dc = pos[i0:i1, None, :] - pos[None, :, :]
        d2 = np.einsum("bkj,bkj->bk", dc, dc)
        s2 = segment_distances2(pos[i0:i1], ori[i0:i1], pos, ori)
        rows = np.arange(i1 - i0)
        d2[rows, rows + i0] = np.inf
        s2[rows, rows + i0] = np.inf
        nn_c[i0:i1] = np.sqrt(d2.min(axis=1))
        nn_s[i0:i1] = np.sqrt(np.maximum(s2.min(axis=1), 0.0))
    return {"fibers": int(n), "centre_radius": float(np.sqrt((pos * pos).sum(1)).max()),
            "min_centre_distance": float(nn_c.min()), "mean_nn_centre_distance": float(nn_c.mean()),
            "min_segment_distance": float(nn_s.min()), "mean_nn_segment_distance": float(nn_s.mean())}


def serving_requests(count=512, seed=0, n_min=16, n_max=1000, steps_min=5, steps_max=50,
                     slenderness=(0.01, 0.005)):
    """The serving ensemble: `count` independent suspensions with N drawn
    log-uniform in [n_min, n_max], slenderness from `slenderness`, and
    steps_min..steps_max time steps each.  Layouts are drawn per request by
    request_layout() (centres in a sphere of volume fraction ~1%)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ns = np.exp(rng.uniform(np.log(n_min), np.log(n_max + 1), size=count)).astype(int).clip(n_min, n_max)
    eps = rng.choice(np.asarray(slenderness, np.float64), size=count)
    steps = rng.integers(steps_min, steps_max + 1, size=count)
    return [dict(id=i, n=int(ns[i]), slenderness=float(eps[i]), nsteps=int(steps[i]), seed=int(seed) * 100003 + i)
            for i in range(count)]


def request_layout(req):
    return sphere_layout(req["n"], serving_radius(req["n"]), seed=req["seed"])
