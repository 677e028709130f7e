"""The solid description of ``include/icam_solid.h`` as ctypes structures, and a
builder that fills it.

A :class:`SolidBuilder` collects faces, edges, vertices and loop uses the way the
reference's import assembles ``Solid3`` (crates/icam-core/src/solid3.rs:597-851):
every edge is used once in each direction by its two faces (twice by one face for
a seam), loops run counterclockwise seen from outside the solid, and each use
carries its curve in the face's parameter domain (trim2.rs:40-62). ``desc()``
returns an ``IcamSolidDesc`` whose arrays stay alive as long as the builder.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

PLANE, CYLINDER, CONE, SPHERE, TORUS, NURBS = range(6)
EDGE_LINE, EDGE_ARC, EDGE_SPLINE = range(3)


class IcamFrame(C.Structure):
    _fields_ = [("o", C.c_double * 3), ("z", C.c_double * 3), ("x", C.c_double * 3)]


class IcamFaceDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("sense", C.c_int32), ("f", IcamFrame),
        ("a", C.c_double), ("b", C.c_double),
        ("du", C.c_int32), ("dv", C.c_int32), ("nsu", C.c_int32), ("nsv", C.c_int32),
        ("patch_off", C.c_int64), ("brk_off", C.c_int64),
        ("lo", C.c_double * 2), ("hi", C.c_double * 2), ("period", C.c_double * 2),
        ("first_use", C.c_int32), ("n_uses", C.c_int32),
    ]


class IcamEdgeDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("v0", C.c_int32), ("v1", C.c_int32),
        ("f0", C.c_int32), ("f1", C.c_int32),
        ("degree", C.c_int32), ("first_piece", C.c_int32), ("n_pieces", C.c_int32),
        ("pad", C.c_int32),
        ("a", C.c_double * 3), ("b", C.c_double * 3),
        ("f", IcamFrame), ("r", C.c_double), ("t0", C.c_double), ("sweep", C.c_double),
    ]


class IcamUseDesc(C.Structure):
    _fields_ = [
        ("edge", C.c_int32), ("rev", C.c_int32), ("loop", C.c_int32), ("seam", C.c_int32),
        ("first_pc", C.c_int32), ("n_pc", C.c_int32),
    ]


class IcamSolidDesc(C.Structure):
    _fields_ = [
        ("n_faces", C.c_int32), ("n_edges", C.c_int32), ("n_verts", C.c_int32), ("n_uses", C.c_int32),
        ("faces", C.POINTER(IcamFaceDesc)), ("edges", C.POINTER(IcamEdgeDesc)),
        ("verts", C.POINTER(C.c_double)), ("uses", C.POINTER(IcamUseDesc)),
        ("patches", C.POINTER(C.c_double)), ("breaks", C.POINTER(C.c_double)),
        ("cpieces", C.POINTER(C.c_double)), ("pcurves", C.POINTER(C.c_double)),
        ("n_patch_doubles", C.c_int64), ("n_break_doubles", C.c_int64),
        ("n_cpiece_doubles", C.c_int64), ("n_pcurve_doubles", C.c_int64),
        ("tol", C.c_double),
    ]


def _v(x):
    return np.asarray(x, dtype=np.float64)


def unit(x):
    x = _v(x)
    return x / np.linalg.norm(x)


class Frame:
    """Origin, unit z, unit x (made orthogonal to z); y = z x x."""

    def __init__(self, o, z, x):
        self.o = _v(o)
        self.z = unit(z)
        x = _v(x)
        x = x - self.z * float(np.dot(x, self.z))
        self.x = unit(x)
        self.y = np.cross(self.z, self.x)

    def local(self, p):
        d = _v(p) - self.o
        return np.array([d @ self.x, d @ self.y, d @ self.z])

    def world(self, l):
        return self.o + self.x * l[0] + self.y * l[1] + self.z * l[2]

    def c(self):
        f = IcamFrame()
        f.o[:] = list(self.o)
        f.z[:] = list(self.z)
        f.x[:] = list(self.x)
        return f


# ---------------------------------------------------------------- B-spline helpers

def insert_knot(p, knots, pts, x):
    """Boehm's insertion of knot x into a degree-p B-spline (homogeneous points)."""
    knots = list(knots)
    # span index k with knots[k] <= x < knots[k+1] (the last nonempty span for x at the end)
    k = None
    for i in range(len(knots) - 1):
        if knots[i] <= x < knots[i + 1]:
            k = i
    if k is None:
        k = max(i for i in range(len(knots) - 1) if knots[i] < knots[i + 1])
    new = []
    for i in range(len(pts) + 1):
        if i <= k - p:
            new.append(pts[i])
        elif i > k:
            new.append(pts[i - 1])
        else:
            a = (x - knots[i]) / (knots[i + p] - knots[i])
            new.append((1 - a) * pts[i - 1] + a * pts[i])
    knots.insert(k + 1, x)
    return knots, new


def bezier_pieces(p, knots, pts):
    """The Bezier pieces of a clamped B-spline (homogeneous rows of an array),
    by inserting every interior knot up to multiplicity p (The NURBS Book 5.6).
    Returns [(points (p+1, dim), t0, t1)]."""
    knots = list(knots)
    pts = [np.array(q, dtype=np.float64) for q in pts]
    for x in sorted(set(knots[p + 1:len(knots) - p - 1])):
        while knots.count(x) < p:
            knots, pts = insert_knot(p, knots, pts, x)
    out = []
    breaks = sorted(set(knots))
    for a, b in zip(breaks[:-1], breaks[1:]):
        last_a = max(i for i, x in enumerate(knots) if x == a)
        first = last_a - p
        out.append((np.array(pts[first:first + p + 1]), a, b))
    return out


def _extract_axis0(p, knots, pts):
    """The Bezier pieces of a clamped degree-p B-spline along axis 0 of pts (every
    other axis carried along: many curves at once), by Boehm's insertion of each
    interior knot up to multiplicity p. Returns (pieces (spans, p+1, ...), breaks)."""
    knots = [float(x) for x in knots]
    pts = np.asarray(pts, dtype=np.float64)
    for x in sorted(set(knots[p + 1:len(knots) - p - 1])):
        while knots.count(x) < p:
            k = max(i for i in range(len(knots) - 1) if knots[i] <= x < knots[i + 1])
            n = len(pts)
            i = np.arange(k - p + 1, k + 1)
            a = (x - np.asarray(knots)[i]) / (np.asarray(knots)[i + p] - np.asarray(knots)[i])
            a = a.reshape((-1,) + (1,) * (pts.ndim - 1))
            mid = (1 - a) * pts[i - 1] + a * pts[i]
            pts = np.concatenate([pts[: k - p + 1], mid, pts[k:n]], axis=0)
            knots.insert(k + 1, x)
    breaks = sorted(set(knots))
    pieces = []
    for a0 in breaks[:-1]:
        last_a = max(i for i, x in enumerate(knots) if x == a0)
        first = last_a - p
        pieces.append(pts[first:first + p + 1])
    return np.stack(pieces), np.array(breaks)


def surface_spans(du, dv, ku, kv, net_h):
    """Bezier spans of a clamped rational B-spline surface, net_h[i][j] homogeneous
    (i along u). Returns (patches (nsu, nsv, du+1, dv+1, 4), u breaks, v breaks)."""
    net_h = np.asarray(net_h, dtype=np.float64)
    # along u for every column j at once: (nsu, du+1, nv, 4)
    pu, ub = _extract_axis0(du, ku, net_h)
    # then along v for every Bezier row: axis 0 = v
    pv, vb = _extract_axis0(dv, kv, np.moveaxis(pu, 2, 0))  # (nsv, dv+1, nsu, du+1, 4)
    patches = np.ascontiguousarray(np.transpose(pv, (2, 0, 3, 1, 4)))  # (nsu, nsv, du+1, dv+1, 4)
    return patches, ub, vb


def elevate_to_cubic(pts_h):
    """A Bezier curve of degree <= 3 (homogeneous rows) raised to degree 3."""
    q = np.asarray(pts_h, dtype=np.float64)
    while len(q) < 4:
        n = len(q) - 1
        r = [q[0]]
        for i in range(1, n + 1):
            a = i / (n + 1)
            r.append(a * q[i - 1] + (1 - a) * q[i])
        r.append(q[n])
        q = np.array(r)
    return q


def line_pcurve(a, b):
    """A straight segment in (u, v) as one rational cubic piece (weights 1)."""
    a, b = _v(a), _v(b)
    return [np.array([[*(a + (b - a) * t), 1.0] for t in (0, 1 / 3, 2 / 3, 1)])]


def arc_pcurve(center, r, t0, sweep, to_uv=None):
    """A circular arc (in a plane's own 2D coordinates, or mapped affinely by
    to_uv) as rational cubic pieces: quarter arcs at most, each an exact rational
    quadratic (weights 1, cos(q/2), 1) raised to degree 3."""
    n = max(1, int(math.ceil(abs(sweep) / (math.pi / 2) - 1e-9)))
    q = sweep / n
    out = []
    c = _v(center)
    for k in range(n):
        a0 = t0 + q * k
        am = a0 + q / 2
        a1 = a0 + q
        w = math.cos(q / 2)
        p0 = c + r * np.array([math.cos(a0), math.sin(a0)])
        p1 = c + r / w * np.array([math.cos(am), math.sin(am)])
        p2 = c + r * np.array([math.cos(a1), math.sin(a1)])
        if to_uv is not None:
            p0, p1, p2 = to_uv(p0), to_uv(p1), to_uv(p2)
        h = np.array([[*p0, 1.0], [*(p1 * w), w], [*p2, 1.0]])
        out.append(elevate_to_cubic(h))
    return out


# ---------------------------------------------------------------- the builder

class SolidBuilder:
    def __init__(self, tol=1e-9):
        self.tol = tol
        self.verts = []
        self.edges = []
        self.faces = []  # dicts
        self.patches = []
        self.breaks = []
        self.cpieces = []
        self.pcurves = []
        self._keep = []
        self._desc = None

    # vertices and edges
    def vertex(self, p):
        self.verts.append(_v(p))
        return len(self.verts) - 1

    def line(self, v0, v1):
        e = IcamEdgeDesc()
        e.kind = EDGE_LINE
        e.v0, e.v1 = v0, v1
        e.f0 = e.f1 = -1
        e.a[:] = list(self.verts[v0])
        e.b[:] = list(self.verts[v1])
        self.edges.append(e)
        return len(self.edges) - 1

    def arc(self, frame: Frame, r, t0, sweep, v0, v1):
        e = IcamEdgeDesc()
        e.kind = EDGE_ARC
        e.v0, e.v1 = v0, v1
        e.f0 = e.f1 = -1
        e.f = frame.c()
        e.r, e.t0, e.sweep = r, t0, sweep
        self.edges.append(e)
        return len(self.edges) - 1

    def spline(self, pieces_h, v0, v1):
        """A rational B-spline edge as Bezier pieces (each (deg+1, 4) homogeneous)."""
        e = IcamEdgeDesc()
        e.kind = EDGE_SPLINE
        e.v0, e.v1 = v0, v1
        e.f0 = e.f1 = -1
        deg = len(pieces_h[0]) - 1
        e.degree = deg
        e.first_piece = len(self.cpieces)
        e.n_pieces = len(pieces_h)
        for p in pieces_h:
            assert len(p) == deg + 1
            self.cpieces.append(np.asarray(p, dtype=np.float64))
        self.edges.append(e)
        return len(self.edges) - 1

    # faces
    def face(self, kind, sense, frame=None, a=0.0, b=0.0, lo=(0, 0), hi=(1, 1), period=(0, 0), nurbs=None):
        f = IcamFaceDesc()
        f.kind = kind
        f.sense = sense
        if frame is not None:
            f.f = frame.c()
        f.a, f.b = a, b
        f.lo[:] = list(lo)
        f.hi[:] = list(hi)
        f.period[:] = list(period)
        if nurbs is not None:
            patches, ub, vb = nurbs
            nsu, nsv, du1, dv1, _ = patches.shape
            f.du, f.dv, f.nsu, f.nsv = du1 - 1, dv1 - 1, nsu, nsv
            f.patch_off = sum(p.size for p in self.patches)
            self.patches.append(np.ascontiguousarray(patches, dtype=np.float64).ravel())
            f.brk_off = sum(len(x) for x in self.breaks)
            self.breaks.append(np.concatenate([ub, vb]).astype(np.float64))
        self.faces.append({"desc": f, "loops": []})
        return len(self.faces) - 1

    def loop(self, face, uses):
        """uses: [(edge, rev, pcurve pieces or None for a seam)] in traversal order."""
        self.faces[face]["loops"].append(uses)

    def desc(self) -> IcamSolidDesc:
        if getattr(self, "_desc", None) is not None:
            return self._desc
        for e in self.edges:
            e.f0 = e.f1 = -1
        self.pcurves = []
        faces = (IcamFaceDesc * len(self.faces))()
        uses = []
        for fi, fd in enumerate(self.faces):
            f = fd["desc"]
            f.first_use = len(uses)
            for li, lp in enumerate(fd["loops"]):
                for (ei, rev, pcs) in lp:
                    u = IcamUseDesc()
                    u.edge, u.rev, u.loop = ei, int(rev), li
                    seam = pcs is None
                    u.seam = int(seam)
                    u.first_pc = len(self.pcurves)
                    u.n_pc = 0 if seam else len(pcs)
                    if not seam:
                        for pc in pcs:
                            pc = np.asarray(pc, dtype=np.float64)
                            assert pc.shape == (4, 3), pc.shape
                            self.pcurves.append(pc)
                    uses.append(u)
                    e = self.edges[ei]
                    if e.f0 < 0:
                        e.f0 = fi
                    elif e.f1 < 0:
                        e.f1 = fi
                    else:
                        raise ValueError(f"edge {ei} used by more than two faces")
            f.n_uses = len(uses) - f.first_use
            faces[fi] = f
        for i, e in enumerate(self.edges):
            if e.f0 < 0 or e.f1 < 0:
                raise ValueError(f"edge {i} is used by {int(e.f0 >= 0) + int(e.f1 >= 0)} faces (not a closed shell)")
        edges = (IcamEdgeDesc * len(self.edges))(*self.edges)
        uarr = (IcamUseDesc * max(1, len(uses)))(*uses)
        verts = np.ascontiguousarray(np.array(self.verts, dtype=np.float64).reshape(-1, 3))

        def cat(lst):
            if not lst:
                return np.zeros(1)
            return np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64).ravel() for x in lst]))

        patches, breaks, cpieces, pcurves = cat(self.patches), cat(self.breaks), cat(self.cpieces), cat(self.pcurves)
        self._keep = [faces, edges, uarr, verts, patches, breaks, cpieces, pcurves]
        d = IcamSolidDesc()
        d.n_faces, d.n_edges, d.n_verts, d.n_uses = len(self.faces), len(self.edges), len(self.verts), len(uses)
        d.faces = C.cast(faces, C.POINTER(IcamFaceDesc))
        d.edges = C.cast(edges, C.POINTER(IcamEdgeDesc))
        d.uses = C.cast(uarr, C.POINTER(IcamUseDesc))
        dp = C.POINTER(C.c_double)
        d.verts = verts.ctypes.data_as(dp)
        d.patches = patches.ctypes.data_as(dp)
        d.breaks = breaks.ctypes.data_as(dp)
        d.cpieces = cpieces.ctypes.data_as(dp)
        d.pcurves = pcurves.ctypes.data_as(dp)
        d.n_patch_doubles = patches.size
        d.n_break_doubles = breaks.size
        d.n_cpiece_doubles = cpieces.size
        d.n_pcurve_doubles = pcurves.size
        d.tol = self.tol
        self._desc = d
        return d
