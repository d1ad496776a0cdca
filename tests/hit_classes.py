"""Classification of hit-record differences between the FP32 device traversal and the FP64
oracle, for the hit-record parity tests.

Both sides trace the same rays (FP32 values; the oracle widens them to FP64) through the same
BVH. The bar: hit/miss and primitive id are equal, except for these documented classes, each
decided in FP64 from the triangles involved:

  tie       both primitives are hit in FP64 and their distances lie within 1 FP32 ulp of each
            other: the FP32 distance cannot order them (the reference breaks exact ties to the
            lower primitive id, src/render/bvh.cpp:274-275);
  graze     the ray passes so close to an edge of one of the two triangles that the FP32 edge
            function's rounding error bound (first order, times 2) exceeds the FP64 value: FP32
            cannot decide the side of that edge (the reference's shear test,
            src/render/intersection.cpp:108-152, evaluated with FP32 roundings);
  interval  the FP64 distance lies within the FP32 distance error of an end of the query
            interval, or below the self-intersection bound evaluated with FP32's unit roundoff
            (the rejection at src/render/intersection.cpp:143-150), so FP32 may keep or drop it.

Anything else is "unexplained", and the tests require none.
"""

from __future__ import annotations

import numpy as np

U32 = 2.0 ** -24  # FP32 unit roundoff


def _gamma(n: int, u: float) -> float:
    return n * u / (1 - n * u)


def shear_test(tri: np.ndarray, o: np.ndarray, d: np.ndarray):
    """FP64 shear-space evaluation of one triangle for one ray.

    Returns (inside, t, e, de, t_err, self_bound32): `inside` is the closed-interval edge test with
    a nonzero determinant, `t` the FP64 distance, `e` the three edge functions, `de` a first-order
    bound on the FP32 device's error in each edge function, `t_err` a bound on its FP32 distance
    error, and `self_bound32` the distance below which the FP32 test rejects the hit as a
    self-intersection.
    """
    tri = np.asarray(tri, np.float64)
    o = np.asarray(o, np.float64)
    d = np.asarray(d, np.float64)
    ad = np.abs(d)
    kz = 0 if ad[0] > ad[1] else 1
    if ad[2] > ad[kz]:
        kz = 2
    kx = 0 if kz == 2 else kz + 1
    ky = 0 if kx == 2 else kx + 1
    if d[kz] < 0:
        kx, ky = ky, kx
    sx, sy, sz = d[kx] / d[kz], d[ky] / d[kz], 1.0 / d[kz]
    t = tri - o
    tz = t[:, kz]
    px = t[:, kx] - sx * tz
    py = t[:, ky] - sy * tz
    # FP32 device: t = fl(v - o) (one rounding), s = fl(d/dz) (one), p = fma(-s, z, t) (one).
    dpx = U32 * (np.abs(t[:, kx]) + 2 * np.abs(sx * tz) + np.abs(px))
    dpy = U32 * (np.abs(t[:, ky]) + 2 * np.abs(sy * tz) + np.abs(py))
    e = np.empty(3)
    de = np.empty(3)
    for k, (i, j) in enumerate(((1, 2), (2, 0), (0, 1))):
        e[k] = px[i] * py[j] - py[i] * px[j]
        de[k] = (dpx[i] * abs(py[j]) + abs(px[i]) * dpy[j] + dpy[i] * abs(px[j])
                 + abs(py[i]) * dpx[j] + 2 * U32 * abs(e[k]))
    det = e.sum()
    inside = bool(((e >= 0).all() or (e <= 0).all()) and det != 0)
    z = tz * sz
    if det == 0:
        return False, np.inf, e, de, np.inf, 0.0
    dist = float(e @ z / det)
    # t = sum(e_k z_k) / sum(e_k): dt/de_k = (z_k - t) / det and dt/dz_k = e_k / det, with
    # |dz_k| <= 2u|z_k|, plus the roundings of the final sum and division.
    t_err = float((de @ np.abs(z - dist) + 2 * U32 * np.abs(e) @ np.abs(z)) / abs(det)
                  + 4 * U32 * abs(dist))
    # The self-intersection bound of the shear test with FP32's unit roundoff.
    g2, g3, g5 = _gamma(2, U32), _gamma(3, U32), _gamma(5, U32)
    xm, ym, zm = np.abs(px).max(), np.abs(py).max(), np.abs(z).max()
    ex, ey = g5 * (xm + zm), g5 * (ym + zm)
    eedge = 2 * (g2 * xm * ym + ey * xm + ex * ym)
    emax = np.abs(e).max()
    self_bound = float(3 * (g3 * emax * zm + eedge * zm + g3 * zm * emax) / abs(det))
    return inside, dist, e, de, t_err, self_bound


def _graze(e, de) -> bool:
    return bool(np.any(np.abs(e) <= 2 * de))


def classify(tris, o, d, tmin, tmax, prim_a, prim_b) -> str:
    """Class of one difference: prim_a and prim_b are the two sides' primitives (None = miss)."""
    info = {}
    for p in (prim_a, prim_b):
        if p is not None and p not in info:
            info[p] = shear_test(tris[p], o, d)
    if prim_a is not None and prim_b is not None and prim_a != prim_b:
        ia, ib = info[prim_a], info[prim_b]
        if ia[0] and ib[0]:
            ulp = float(np.spacing(np.float32(max(abs(ia[1]), abs(ib[1])))))
            if abs(ia[1] - ib[1]) <= ulp:
                return "tie"
    if any(_graze(v[2], v[3]) for v in info.values()):
        return "graze"
    for inside, dist, _, _, t_err, self_bound in info.values():
        if not inside:
            continue
        if abs(dist - tmax) <= t_err or abs(dist - tmin) <= t_err or dist <= self_bound + t_err:
            return "interval"
    return "unexplained"


def compare_nearest(g_prim, c_hit, c_prim, tris, origins, dirs, tmin, tmax, limit=None):
    """Counts per class over all rays whose nearest-hit records differ.

    g_prim: device primitive ids (0xFFFFFFFF = miss); c_hit/c_prim: oracle hit flags and ids.
    Returns (classes, examples) with a few unexplained rays for the failure message.
    """
    g_hit = g_prim != 0xFFFFFFFF
    c_hit = np.asarray(c_hit, bool)
    # Widen before substituting -1: NumPy casts a Python -1 to the array's uint32 otherwise.
    c_prim = np.where(c_hit, np.asarray(c_prim).astype(np.int64), -1)
    g_prim64 = np.where(g_hit, np.asarray(g_prim).astype(np.int64), -1)
    differ = np.flatnonzero((g_hit != c_hit) | (g_prim64 != c_prim))
    classes = {"tie": 0, "graze": 0, "interval": 0, "unexplained": 0}
    examples = []
    tmin = np.broadcast_to(np.asarray(tmin, np.float64), (len(g_prim),))
    tmax = np.broadcast_to(np.asarray(tmax, np.float64), (len(g_prim),))
    for i in differ:
        a = int(g_prim64[i]) if g_hit[i] else None
        b = int(c_prim[i]) if c_hit[i] else None
        cls = classify(tris, origins[i], dirs[i], float(tmin[i]), float(tmax[i]), a, b)
        classes[cls] += 1
        if cls == "unexplained" and len(examples) < 5:
            examples.append((int(i), a, b))
    return classes, examples


def compare_occlusion(g_occ, c_occ, g_nearest, c_nearest, tris, origins, dirs, tmin, tmax):
    """Counts per class over shadow segments whose occlusion differs. g_nearest/c_nearest give,
    for every segment, each side's nearest primitive in the same interval (the occluder that
    decided the difference; None where that side saw the segment clear)."""
    differ = np.flatnonzero(np.asarray(g_occ, bool) != np.asarray(c_occ, bool))
    classes = {"tie": 0, "graze": 0, "interval": 0, "unexplained": 0}
    examples = []
    for i in differ:
        p = g_nearest(i) if g_occ[i] else c_nearest(i)
        cls = classify(tris, origins[i], dirs[i], float(tmin[i]), float(tmax[i]), p, None)
        classes[cls] += 1
        if cls == "unexplained" and len(examples) < 5:
            examples.append((int(i), p))
    return classes, examples
