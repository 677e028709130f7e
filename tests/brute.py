"""Independent brute-force signed distance for the block-with-hole part, with no code
shared with the oracle's search: the unsigned distance is the least distance to its
seven trimmed faces (each in closed form: a planar region or the hole's finite wall),
the sign is point membership (inside the block and outside the hole).
Test infrastructure only."""
import numpy as np


def _seg(p, a, b):
    ab = b - a
    t = np.clip(((p - a) @ ab) / (ab @ ab), 0.0, 1.0)
    return np.linalg.norm(p - (a + t[:, None] * ab), axis=1)


def _circle(p, c, r, zaxis):
    d = p - c
    h = d @ zaxis
    inplane = d - h[:, None] * zaxis
    rho = np.linalg.norm(inplane, axis=1)
    return np.sqrt((rho - r) ** 2 + h ** 2)


def block_with_hole_sdf(p, size=(100.0, 60.0, 40.0), center=(50.0, 30.0), r=10.0):
    p = np.asarray(p, dtype=np.float64).reshape(-1, 3)
    X, Y, Z = size
    cx, cy = center
    corners = {(i, j, k): np.array([i * X, j * Y, k * Z]) for i in (0, 1) for j in (0, 1) for k in (0, 1)}
    ez = np.array([0.0, 0.0, 1.0])
    best = np.full(len(p), np.inf)

    def rect_face(axis, val, lo2, hi2, hole):
        # planar face axis = val, spanning the other two axes over [lo2, hi2]
        o = [k for k in range(3) if k != axis]
        u, v = p[:, o[0]], p[:, o[1]]
        inside = (u >= lo2[0]) & (u <= hi2[0]) & (v >= lo2[1]) & (v <= hi2[1])
        if hole:
            inside &= np.hypot(u - cx, v - cy) >= r
        dplane = np.abs(p[:, axis] - val)
        # boundary: four lines (+ the hole circle)
        pts = []
        for (a, b) in [((lo2[0], lo2[1]), (hi2[0], lo2[1])), ((hi2[0], lo2[1]), (hi2[0], hi2[1])),
                       ((hi2[0], hi2[1]), (lo2[0], hi2[1])), ((lo2[0], hi2[1]), (lo2[0], lo2[1]))]:
            A = np.zeros(3); B = np.zeros(3)
            A[axis] = B[axis] = val
            A[o[0]], A[o[1]] = a
            B[o[0]], B[o[1]] = b
            pts.append(_seg(p, A, B))
        db = np.min(pts, axis=0)
        if hole:
            db = np.minimum(db, _circle(p, np.array([cx, cy, val]), r, ez))
        return np.where(inside, dplane, db)

    best = np.minimum(best, rect_face(2, 0.0, (0, 0), (X, Y), True))
    best = np.minimum(best, rect_face(2, Z, (0, 0), (X, Y), True))
    best = np.minimum(best, rect_face(1, 0.0, (0, 0), (X, Z), False))
    best = np.minimum(best, rect_face(1, Y, (0, 0), (X, Z), False))
    best = np.minimum(best, rect_face(0, 0.0, (0, 0), (Y, Z), False))
    best = np.minimum(best, rect_face(0, X, (0, 0), (Y, Z), False))
    # the hole's wall: the finite tube
    rho = np.hypot(p[:, 0] - cx, p[:, 1] - cy)
    hz = np.clip(p[:, 2], 0.0, Z)
    best = np.minimum(best, np.sqrt((rho - r) ** 2 + (p[:, 2] - hz) ** 2))
    inside = (p[:, 0] > 0) & (p[:, 0] < X) & (p[:, 1] > 0) & (p[:, 1] < Y) & (p[:, 2] > 0) & (p[:, 2] < Z) & (rho > r)
    return np.where(inside, -best, best)
