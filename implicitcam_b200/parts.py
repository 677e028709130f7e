"""Seeded synthetic parts, built as closed B-rep solids (``solid.SolidBuilder``).

- ``can``: the reference's own test solid, a cylinder r 3 from z 0 to 5
  (crates/icam-core/src/solid3.rs:2009-2041);
- ``bump_box``: the reference's 10 x 10 box with a biquadratic B-spline top
  (solid3.rs:2092-2147);
- ``block_with_hole``: a 100 x 60 x 40 mm block minus a 20 mm through-hole along z
  at its centre (6 planes + 1 cylinder);
- ``freeform_top``: a 120 x 120 x 50 mm block whose top face is a clamped bicubic
  rational B-spline with 16 x 16 control points, heights 50 mm plus 8 seeded
  Gaussian bumps, weights in [0.8, 1.2];
- ``frustum``, ``ball``, ``ring``: a cone-sided can, a sphere and a torus, the analytic
  surface kinds the parts above lack (the sphere and torus have no edges at all);
- ``boss`` (cylinder, torus fillet, plane cap), ``countersunk_block`` (a hole with a
  cone countersink) and ``dome`` (a cylinder under a hemisphere): the analytic families
  of a batch of uneven parts;
- ``nurbs_dome``, ``nurbs_ball``: a dome and a sphere whose caps are rational B-spline
  surfaces of revolution collapsing at their poles;
- ``mold``: a 250 x 200 x 80 mm block with a pocket whose floor is 500 one-span bicubic
  rational B-spline faces joined along shared B-spline edges, and 40 filleted bosses on
  its rim.

Random numbers come from the reference checkers' xorshift64 generator
(crates/icam-check/src/exact_check.rs:45-52) seeded through splitmix64, so that
seed 0 is usable.
"""
from __future__ import annotations

import math

import numpy as np

from .solid import (
    CONE, CYLINDER, NURBS, PLANE, SPHERE, TORUS, Frame, SolidBuilder, arc_pcurve, elevate_to_cubic,
    line_pcurve, surface_spans,
)

TAU = 2.0 * math.pi
MASK = (1 << 64) - 1


class Rng:
    """xorshift64 (exact_check.rs:45-52), seeded by splitmix64(seed)."""

    def __init__(self, seed: int):
        z = (seed + 0x9E3779B97F4A7C15) & MASK
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        z ^= z >> 31
        self.s = z or 0x2545F4914F6CDD1D

    def next(self) -> int:
        x = self.s
        x ^= (x << 13) & MASK
        x ^= x >> 7
        x ^= (x << 17) & MASK
        self.s = x
        return x

    def uniform(self, a=0.0, b=1.0) -> float:
        return a + (b - a) * ((self.next() >> 11) * (1.0 / (1 << 53)))


def _pad(lo, hi, frac=0.05):
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    p = frac * (hi - lo) + 1e-9 * (np.abs(hi) + np.abs(lo)) + 1e-6
    return lo - p, hi + p


class _Plane:
    """A planar face's frame and the map of 3D edges into its (u, v)."""

    def __init__(self, frame: Frame):
        self.fr = frame

    def uv(self, p):
        return self.fr.local(p)[:2]

    def pcurve(self, b: SolidBuilder, ei, rev):
        e = b.edges[ei]
        if e.kind == 0:
            a, c = self.uv(list(e.a)), self.uv(list(e.b))
            pcs = line_pcurve(a, c)
        elif e.kind == 1:
            af = Frame(list(e.f.o), list(e.f.z), list(e.f.x))

            def to_uv(q2):
                return self.uv(af.world([q2[0], q2[1], 0.0]))

            pcs = arc_pcurve([0.0, 0.0], e.r, e.t0, e.sweep, to_uv)
        else:
            pcs = []
            deg = e.degree
            for k in range(e.n_pieces):
                p = b.cpieces[e.first_piece + k]
                hom = []
                for q in p:
                    w = q[3]
                    xyz = q[:3] / w
                    u, v = self.uv(xyz)
                    hom.append([u * w, v * w, w])
                pcs.append(elevate_to_cubic(np.array(hom)) if deg < 3 else np.array(hom))
        if rev:
            pcs = [pc[::-1].copy() for pc in pcs[::-1]]
        return pcs

    def domain(self, b: SolidBuilder, uses):
        pts = []
        for ei, rev in uses:
            for pc in self.pcurve(b, ei, rev):
                pts.extend(pc[:, :2] / pc[:, 2:3])
        pts = np.array(pts)
        return _pad(pts.min(0), pts.max(0))


def _plane_face(b: SolidBuilder, frame: Frame, sense, loops):
    """loops: [[(edge, rev), ...], ...]"""
    pl = _Plane(frame)
    lo, hi = pl.domain(b, [u for lp in loops for u in lp])
    f = b.face(PLANE, sense, frame, lo=lo, hi=hi)
    for lp in loops:
        b.loop(f, [(ei, rev, pl.pcurve(b, ei, rev)) for ei, rev in lp])
    return f


def can(r=3.0, height=5.0):
    """The reference test's can (solid3.rs:2009-2041): two planes, one cylinder,
    two circles, one seam."""
    b = SolidBuilder(tol=1e-9)
    z, x = [0, 0, 1], [1, 0, 0]
    f0 = Frame([0, 0, 0], z, x)
    f1 = Frame([0, 0, height], z, x)
    va = b.vertex([r, 0, 0])
    vb = b.vertex([r, 0, height])
    c0 = b.arc(f0, r, 0.0, TAU, va, va)
    c1 = b.arc(f1, r, 0.0, TAU, vb, vb)
    seam = b.line(va, vb)
    _plane_face(b, f0, -1, [[(c0, True)]])
    _plane_face(b, f1, +1, [[(c1, False)]])
    lo, hi = _pad([0.0, 0.0], [TAU, height])
    cyl = b.face(CYLINDER, +1, f0, a=r, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(cyl, [
        (c0, False, line_pcurve([0.0, 0.0], [TAU, 0.0])),
        (seam, False, None),
        (c1, True, line_pcurve([TAU, height], [0.0, height])),
        (seam, True, None),
    ])
    return b


def block_with_hole(size=(100.0, 60.0, 40.0), center=(50.0, 30.0), r=10.0):
    """A block [0,X]x[0,Y]x[0,Z] minus a through-hole of radius r along z."""
    X, Y, Z = size
    b = SolidBuilder(tol=1e-9)
    c = {}
    for i, x in enumerate((0.0, X)):
        for j, y in enumerate((0.0, Y)):
            for k, zz in enumerate((0.0, Z)):
                c[i, j, k] = b.vertex([x, y, zz])
    L = lambda p, q: b.line(c[p], c[q])  # noqa: E731
    eb = [L((0, 0, 0), (1, 0, 0)), L((1, 0, 0), (1, 1, 0)), L((1, 1, 0), (0, 1, 0)), L((0, 1, 0), (0, 0, 0))]
    et = [L((0, 0, 1), (1, 0, 1)), L((1, 0, 1), (1, 1, 1)), L((1, 1, 1), (0, 1, 1)), L((0, 1, 1), (0, 0, 1))]
    ev = {ij: L((*ij, 0), (*ij, 1)) for ij in ((0, 0), (1, 0), (1, 1), (0, 1))}
    cx, cy = center
    va = b.vertex([cx + r, cy, 0.0])
    vb = b.vertex([cx + r, cy, Z])
    fz0 = Frame([cx, cy, 0.0], [0, 0, 1], [1, 0, 0])
    fz1 = Frame([cx, cy, Z], [0, 0, 1], [1, 0, 0])
    c0 = b.arc(fz0, r, 0.0, TAU, va, va)
    c1 = b.arc(fz1, r, 0.0, TAU, vb, vb)
    seam = b.line(va, vb)
    # bottom (outward -z): clockwise in xy, the hole counterclockwise
    _plane_face(b, Frame([0, 0, 0], [0, 0, 1], [1, 0, 0]), -1,
                [[(eb[3], True), (eb[2], True), (eb[1], True), (eb[0], True)], [(c0, False)]])
    # top (outward +z)
    _plane_face(b, Frame([0, 0, Z], [0, 0, 1], [1, 0, 0]), +1,
                [[(et[0], False), (et[1], False), (et[2], False), (et[3], False)], [(c1, True)]])
    # front y = 0 (outward -y): local (x, z)
    _plane_face(b, Frame([0, 0, 0], [0, -1, 0], [1, 0, 0]), +1,
                [[(eb[0], False), (ev[1, 0], False), (et[0], True), (ev[0, 0], True)]])
    # right x = X (outward +x): local (y, z)
    _plane_face(b, Frame([X, 0, 0], [1, 0, 0], [0, 1, 0]), +1,
                [[(eb[1], False), (ev[1, 1], False), (et[1], True), (ev[1, 0], True)]])
    # back y = Y (outward +y): local (X - x, z)
    _plane_face(b, Frame([X, Y, 0], [0, 1, 0], [-1, 0, 0]), +1,
                [[(eb[2], False), (ev[0, 1], False), (et[2], True), (ev[1, 1], True)]])
    # left x = 0 (outward -x): local (Y - y, z)
    _plane_face(b, Frame([0, Y, 0], [-1, 0, 0], [0, -1, 0]), +1,
                [[(eb[3], False), (ev[0, 0], False), (et[3], True), (ev[0, 1], True)]])
    # the hole's wall: outward toward the axis (sense -1), (angle, height)
    lo, hi = _pad([0.0, 0.0], [TAU, Z])
    cyl = b.face(CYLINDER, -1, fz0, a=r, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(cyl, [
        (c1, False, line_pcurve([0.0, Z], [TAU, Z])),
        (seam, True, None),
        (c0, True, line_pcurve([TAU, 0.0], [0.0, 0.0])),
        (seam, False, None),
    ])
    return b


def _boundary_pieces(patches, side):
    """The Bezier pieces of a surface's boundary iso-curve, in increasing parameter:
    side 'u0', 'u1' (u fixed, along v) or 'v0', 'v1' (v fixed, along u)."""
    nsu, nsv = patches.shape[:2]
    if side == "u0":
        return [patches[0, j, 0, :, :].copy() for j in range(nsv)]
    if side == "u1":
        return [patches[nsu - 1, j, -1, :, :].copy() for j in range(nsv)]
    if side == "v0":
        return [patches[i, 0, :, 0, :].copy() for i in range(nsu)]
    return [patches[i, nsv - 1, :, -1, :].copy() for i in range(nsu)]


def _nurbs_box(b: SolidBuilder, du, dv, ku, kv, net_h, X, Y, top_sense=+1):
    """A block [0,X]x[0,Y]x[0,top] whose top face is the given clamped rational
    B-spline (u along x, v along y; its boundary iso-curves lie in the four side
    planes), four side planes and a bottom plane."""
    patches, ub, vb = surface_spans(du, dv, ku, kv, net_h)
    corner = lambda h: h[:3] / h[3]  # noqa: E731
    P = np.asarray(net_h)
    c = {}
    for i, x in enumerate((0.0, X)):
        for j, y in enumerate((0.0, Y)):
            c[i, j, 0] = b.vertex([x, y, 0.0])
            c[i, j, 1] = b.vertex(corner(P[-1 if i else 0, -1 if j else 0]))
    L = lambda p, q: b.line(c[p], c[q])  # noqa: E731
    eb = [L((0, 0, 0), (1, 0, 0)), L((1, 0, 0), (1, 1, 0)), L((1, 1, 0), (0, 1, 0)), L((0, 1, 0), (0, 0, 0))]
    ev = {ij: L((*ij, 0), (*ij, 1)) for ij in ((0, 0), (1, 0), (1, 1), (0, 1))}
    # top edges, stored in increasing surface parameter
    s_v0 = b.spline(_boundary_pieces(patches, "v0"), c[0, 0, 1], c[1, 0, 1])  # y = 0, along x
    s_u1 = b.spline(_boundary_pieces(patches, "u1"), c[1, 0, 1], c[1, 1, 1])  # x = X, along y
    s_v1 = b.spline(_boundary_pieces(patches, "v1"), c[0, 1, 1], c[1, 1, 1])  # y = Y, along x
    s_u0 = b.spline(_boundary_pieces(patches, "u0"), c[0, 0, 1], c[0, 1, 1])  # x = 0, along y
    u0, u1, v0, v1 = ub[0], ub[-1], vb[0], vb[-1]
    top = b.face(NURBS, top_sense, lo=[u0, v0], hi=[u1, v1], nurbs=(patches, ub, vb))
    b.loop(top, [
        (s_v0, False, line_pcurve([u0, v0], [u1, v0])),
        (s_u1, False, line_pcurve([u1, v0], [u1, v1])),
        (s_v1, True, line_pcurve([u1, v1], [u0, v1])),
        (s_u0, True, line_pcurve([u0, v1], [u0, v0])),
    ])
    _plane_face(b, Frame([0, 0, 0], [0, 0, 1], [1, 0, 0]), -1,
                [[(eb[3], True), (eb[2], True), (eb[1], True), (eb[0], True)]])
    _plane_face(b, Frame([0, 0, 0], [0, -1, 0], [1, 0, 0]), +1,
                [[(eb[0], False), (ev[1, 0], False), (s_v0, True), (ev[0, 0], True)]])
    _plane_face(b, Frame([X, 0, 0], [1, 0, 0], [0, 1, 0]), +1,
                [[(eb[1], False), (ev[1, 1], False), (s_u1, True), (ev[1, 0], True)]])
    _plane_face(b, Frame([X, Y, 0], [0, 1, 0], [-1, 0, 0]), +1,
                [[(eb[2], False), (ev[0, 1], False), (s_v1, False), (ev[1, 1], True)]])
    _plane_face(b, Frame([0, Y, 0], [-1, 0, 0], [0, -1, 0]), +1,
                [[(eb[3], False), (ev[0, 0], False), (s_u0, False), (ev[0, 1], True)]])
    return b


def _spline_faces(b: SolidBuilder, patches, ub, vb, cu, cv, sense=+1):
    """One B-spline surface (its Bezier spans `patches` (NU, NV, ..), breaks ub, vb) cut
    along span boundaries into faces: face (a, c) holds spans cu[a]..cu[a+1]-1 by
    cv[c]..cv[c+1]-1 (cu, cv increasing from 0 to NU, NV). Neighbouring faces share their
    vertices and iso-curve edges, so they join as the surface does. Returns the vertices
    fvx[a, c] at the cut grid and the edges eu[a, c] (u = ub[cu[a]], along v over face
    row c) and ev[a, c] (v = vb[cv[c]], along u over face column a), each stored in
    increasing parameter."""
    NU, NV = patches.shape[:2]
    FU, FV = len(cu) - 1, len(cv) - 1
    pt = lambda hh: hh[:3] / hh[3]  # noqa: E731
    fvx = {}
    for a in range(FU + 1):
        for c in range(FV + 1):
            i, j = min(cu[a], NU - 1), min(cv[c], NV - 1)
            fvx[a, c] = b.vertex(pt(patches[i, j, -1 if cu[a] == NU else 0, -1 if cv[c] == NV else 0]))
    eu, ev = {}, {}
    for a in range(FU + 1):
        for c in range(FV):
            i = cu[a]
            pieces = [(patches[i, j, 0] if i < NU else patches[NU - 1, j, -1]).copy() for j in range(cv[c], cv[c + 1])]
            eu[a, c] = b.spline(pieces, fvx[a, c], fvx[a, c + 1])
    for a in range(FU):
        for c in range(FV + 1):
            j = cv[c]
            pieces = [(patches[i, j, :, 0] if j < NV else patches[i, NV - 1, :, -1]).copy() for i in range(cu[a], cu[a + 1])]
            ev[a, c] = b.spline(pieces, fvx[a, c], fvx[a + 1, c])
    for a in range(FU):
        for c in range(FV):
            i0, i1, j0, j1 = cu[a], cu[a + 1], cv[c], cv[c + 1]
            u0, u1, v0, v1 = ub[i0], ub[i1], vb[j0], vb[j1]
            f = b.face(NURBS, sense, lo=[u0, v0], hi=[u1, v1],
                       nurbs=(patches[i0:i1, j0:j1].copy(), np.asarray(ub[i0:i1 + 1]).copy(),
                              np.asarray(vb[j0:j1 + 1]).copy()))
            b.loop(f, [
                (ev[a, c], False, line_pcurve([u0, v0], [u1, v0])),
                (eu[a + 1, c], False, line_pcurve([u1, v0], [u1, v1])),
                (ev[a, c + 1], True, line_pcurve([u1, v1], [u0, v1])),
                (eu[a, c], True, line_pcurve([u0, v1], [u0, v0])),
            ])
    return fvx, eu, ev


def _patched_box(b: SolidBuilder, du, dv, ku, kv, net_h, X, Y, cu, cv):
    """_nurbs_box with its top cut into faces along span boundaries (_spline_faces):
    a block [0,X]x[0,Y]x[0,top], the top a clamped rational B-spline of degrees (du, dv)
    cut into (len(cu) - 1) x (len(cv) - 1) faces, four side planes and a bottom plane."""
    patches, ub, vb = surface_spans(du, dv, ku, kv, net_h)
    fvx, eu, ev = _spline_faces(b, patches, ub, vb, cu, cv)
    FU, FV = len(cu) - 1, len(cv) - 1
    c = {}
    for i, x in enumerate((0.0, X)):
        for j, y in enumerate((0.0, Y)):
            c[i, j, 0] = b.vertex([x, y, 0.0])
    c[0, 0, 1], c[1, 0, 1], c[1, 1, 1], c[0, 1, 1] = fvx[0, 0], fvx[FU, 0], fvx[FU, FV], fvx[0, FV]
    L = lambda p, q: b.line(c[p], c[q])  # noqa: E731
    eb = [L((0, 0, 0), (1, 0, 0)), L((1, 0, 0), (1, 1, 0)), L((1, 1, 0), (0, 1, 0)), L((0, 1, 0), (0, 0, 0))]
    es = {ij: L((*ij, 0), (*ij, 1)) for ij in ((0, 0), (1, 0), (1, 1), (0, 1))}
    _plane_face(b, Frame([0, 0, 0], [0, 0, 1], [1, 0, 0]), -1,
                [[(eb[3], True), (eb[2], True), (eb[1], True), (eb[0], True)]])
    _plane_face(b, Frame([0, 0, 0], [0, -1, 0], [1, 0, 0]), +1,
                [[(eb[0], False), (es[1, 0], False)] + [(ev[a, 0], True) for a in reversed(range(FU))]
                 + [(es[0, 0], True)]])
    _plane_face(b, Frame([X, 0, 0], [1, 0, 0], [0, 1, 0]), +1,
                [[(eb[1], False), (es[1, 1], False)] + [(eu[FU, cc], True) for cc in reversed(range(FV))]
                 + [(es[1, 0], True)]])
    _plane_face(b, Frame([X, Y, 0], [0, 1, 0], [-1, 0, 0]), +1,
                [[(eb[2], False), (es[0, 1], False)] + [(ev[a, FV], False) for a in range(FU)] + [(es[1, 1], True)]])
    _plane_face(b, Frame([0, Y, 0], [-1, 0, 0], [0, -1, 0]), +1,
                [[(eb[3], False), (es[0, 0], False)] + [(eu[0, cc], False) for cc in range(FV)] + [(es[0, 1], True)]])
    return b


def _even_cuts(spans, faces):
    """`faces` + 1 cut indices from 0 to `spans`, as even as the spans allow."""
    faces = max(1, min(faces, spans))
    return [round(spans * k / faces) for k in range(faces + 1)]


def freeform_patches(seed=0, n=16, size=120.0, base=50.0, bumps=8, degree=3, faces=4):
    """The freeform top of freeform_top, of any degree (2 or 3; weights U[0.7, 1.3]),
    cut along its knot lines into faces x faces B-spline faces (as even as its n - degree
    spans a side allow) that join C^(degree-1) along shared B-spline edges: faces^2 + 5
    faces in all."""
    rng = Rng(seed)
    g = []
    for _ in range(bumps):
        g.append((rng.uniform(2.0, 6.0), rng.uniform(8.0, 25.0), rng.uniform(0.0, size), rng.uniform(0.0, size)))
    step = size / (n - 1)
    net = np.zeros((n, n, 4))
    for i in range(n):
        for j in range(n):
            x, y = step * i, step * j
            z = base + sum(a * math.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * s * s)) for a, s, cx, cy in g)
            w = rng.uniform(0.7, 1.3)
            net[i, j] = [x * w, y * w, z * w, w]
    spans = n - degree
    knots = [0.0] * (degree + 1) + [k / spans for k in range(1, spans)] + [1.0] * (degree + 1)
    cuts = _even_cuts(spans, faces)
    b = SolidBuilder(tol=1e-9)
    return _patched_box(b, degree, degree, knots, knots, net, size, size, cuts, cuts)


def ridge_box(fold=0.3, size=30.0, base=13.0, wave=0.0, n=7):
    """A size x size block whose top is a bicubic B-spline with a knot of full multiplicity
    at its middle in u: heights base - fold |x - size / 2| (+ wave sin(pi y / size)), so
    the top folds along x = size / 2 into a ridge, a crease inside the face (the
    reference's C0 knot line, solid3.rs:1821). n control points a side (odd, 7 or more:
    the triple knot at 1/2 needs the middle one on the ridge)."""
    if n < 7 or n % 2 == 0:
        raise ValueError("ridge_box needs an odd n of 7 or more")
    net = np.zeros((n, n, 4))
    for i in range(n):
        for j in range(n):
            x, y = size * i / (n - 1), size * j / (n - 1)
            net[i, j] = [x, y, base - fold * abs(x - size / 2) + wave * math.sin(math.pi * y / size), 1.0]
    inner = n - 7
    ku = [0.0] * 4 + [k / (inner // 2 + 1) * 0.5 for k in range(1, inner // 2 + 1)] + [0.5] * 3 + \
         [0.5 + k / (inner // 2 + 1) * 0.5 for k in range(1, inner // 2 + 1)] + [1.0] * 4
    kv = [0.0] * 4 + [k / (n - 3) for k in range(1, n - 3)] + [1.0] * 4
    return _nurbs_box(SolidBuilder(tol=1e-9), 3, 3, ku, kv, net, size, size)


def bump_box():
    """The reference test's bump box (solid3.rs:2092-2147): a 10 x 10 box whose top
    is a biquadratic B-spline over the square, z(5i, 5j) control heights zc."""
    zc = [[5.0, 5.0, 5.0], [7.0, 9.0, 5.0], [5.0, 6.0, 5.0]]
    net = np.array([[[5.0 * i, 5.0 * j, zc[i][j], 1.0] for j in range(3)] for i in range(3)])
    k = [0.0, 0.0, 0.0, 1.0, 1.0, 1.0]
    b = SolidBuilder(tol=1e-9)
    return _nurbs_box(b, 2, 2, k, k, net, 10.0, 10.0)


def bump_box_top(x, y):
    """The bump box's top height z = S(x, y) (its B-spline in closed form)."""
    zc = [[5.0, 5.0, 5.0], [7.0, 9.0, 5.0], [5.0, 6.0, 5.0]]

    def bern(t):
        return [(1 - t) ** 2, 2 * t * (1 - t), t * t]

    bu, bv = bern(x / 10.0), bern(y / 10.0)
    return sum(bu[i] * bv[j] * zc[i][j] for i in range(3) for j in range(3))


def freeform_top(seed=0, n=16, size=120.0, base=50.0, bumps=8):
    """A size x size x base block whose top is a clamped bicubic rational B-spline:
    n x n control points on a uniform grid, heights base + the sum of `bumps`
    Gaussians (amplitude U[2,6] mm, sigma U[8,25] mm, centres U[0,size]^2), weights
    U[0.8,1.2], uniform interior knots (n - 3 spans each way)."""
    rng = Rng(seed)
    g = []
    for _ in range(bumps):
        a = rng.uniform(2.0, 6.0)
        s = rng.uniform(8.0, 25.0)
        cx = rng.uniform(0.0, size)
        cy = rng.uniform(0.0, size)
        g.append((a, s, cx, cy))
    step = size / (n - 1)
    net = np.zeros((n, n, 4))
    for i in range(n):
        for j in range(n):
            x, y = step * i, step * j
            z = base + sum(a * math.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * s * s)) for a, s, cx, cy in g)
            w = rng.uniform(0.8, 1.2)
            net[i, j] = [x * w, y * w, z * w, w]
    spans = n - 3
    knots = [0.0] * 4 + [k / spans for k in range(1, spans)] + [1.0] * 4
    b = SolidBuilder(tol=1e-9)
    return _nurbs_box(b, 3, 3, knots, knots, net, size, size)


def frustum(r0=2.0, half_angle_deg=20.0, height=4.0):
    """The can with a cone for its side: radius r0 at z = 0 widening to
    r0 + height tan(angle) at z = height (two planes, one cone, two circles, one seam)."""
    b = SolidBuilder(tol=1e-9)
    ang = math.radians(half_angle_deg)
    r1 = r0 + height * math.tan(ang)
    z, x = [0, 0, 1], [1, 0, 0]
    f0 = Frame([0, 0, 0], z, x)
    f1 = Frame([0, 0, height], z, x)
    va = b.vertex([r0, 0, 0])
    vb = b.vertex([r1, 0, height])
    c0 = b.arc(f0, r0, 0.0, TAU, va, va)
    c1 = b.arc(f1, r1, 0.0, TAU, vb, vb)
    seam = b.line(va, vb)
    _plane_face(b, f0, -1, [[(c0, True)]])
    _plane_face(b, f1, +1, [[(c1, False)]])
    lo, hi = _pad([0.0, 0.0], [TAU, height])
    cone = b.face(CONE, +1, f0, a=r0, b=ang, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(cone, [
        (c0, False, line_pcurve([0.0, 0.0], [TAU, 0.0])),
        (seam, False, None),
        (c1, True, line_pcurve([TAU, height], [0.0, height])),
        (seam, True, None),
    ])
    return b


def ball(r=3.0, center=(0.0, 0.0, 0.0)):
    """A sphere: one face, no loops, no edges, no vertices."""
    b = SolidBuilder(tol=1e-9)
    b.face(SPHERE, +1, Frame(list(center), [0, 0, 1], [1, 0, 0]), a=r, lo=[0.0, -math.pi / 2],
           hi=[TAU, math.pi / 2], period=[TAU, 0.0])
    return b


def ring(major=4.0, minor=1.5):
    """A torus about z: one face, periodic both ways, no loops, no edges, no vertices."""
    b = SolidBuilder(tol=1e-9)
    b.face(TORUS, +1, Frame([0, 0, 0], [0, 0, 1], [1, 0, 0]), a=major, b=minor, lo=[0.0, -math.pi],
           hi=[TAU, math.pi], period=[TAU, TAU])
    return b


def _boss_body(b: SolidBuilder, cx, cy, z0, r, height, fillet):
    """A boss's cylinder from z0 to z0 + height - fillet, its quarter-torus fillet and its
    cap plane (radius r - fillet at z0 + height); returns its base circle at z0, whose
    face below (a disc, or a plane with the circle as a hole) is the caller's."""
    z, x = [0, 0, 1], [1, 0, 0]
    zm = height - fillet
    f0, fm, f1 = Frame([cx, cy, z0], z, x), Frame([cx, cy, z0 + zm], z, x), Frame([cx, cy, z0 + height], z, x)
    va, vm = b.vertex([cx + r, cy, z0]), b.vertex([cx + r, cy, z0 + zm])
    vt = b.vertex([cx + r - fillet, cy, z0 + height])
    c0 = b.arc(f0, r, 0.0, TAU, va, va)
    cm = b.arc(fm, r, 0.0, TAU, vm, vm)
    ct = b.arc(f1, r - fillet, 0.0, TAU, vt, vt)
    seam_c = b.line(va, vm)
    # the fillet's seam: a quarter circle in the xz plane from (r, zm) up to (r - f, height)
    seam_t = b.arc(Frame([cx + r - fillet, cy, z0 + zm], [0, -1, 0], [1, 0, 0]), fillet, 0.0, math.pi / 2, vm, vt)
    _plane_face(b, f1, +1, [[(ct, False)]])
    lo, hi = _pad([0.0, 0.0], [TAU, zm])
    cyl = b.face(CYLINDER, +1, f0, a=r, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(cyl, [
        (c0, False, line_pcurve([0.0, 0.0], [TAU, 0.0])),
        (seam_c, False, None),
        (cm, True, line_pcurve([TAU, zm], [0.0, zm])),
        (seam_c, True, None),
    ])
    lo, hi = _pad([0.0, 0.0], [TAU, math.pi / 2])
    tor = b.face(TORUS, +1, fm, a=r - fillet, b=fillet, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(tor, [
        (cm, False, line_pcurve([0.0, 0.0], [TAU, 0.0])),
        (seam_t, False, None),
        (ct, True, line_pcurve([TAU, math.pi / 2], [0.0, math.pi / 2])),
        (seam_t, True, None),
    ])
    return c0


def boss(r=3.0, height=5.0, fillet=1.0):
    """A boss: the can with its top edge rounded by a quarter-torus fillet (bottom plane,
    cylinder to height - fillet, torus of major r - fillet and minor fillet, top plane
    of radius r - fillet; three circles, two seams)."""
    b = SolidBuilder(tol=1e-9)
    c0 = _boss_body(b, 0.0, 0.0, 0.0, r, height, fillet)
    _plane_face(b, Frame([0, 0, 0], [0, 0, 1], [1, 0, 0]), -1, [[(c0, True)]])
    return b


def dome(r=3.0, height=4.0):
    """A spherical dome: a cylinder of radius r to `height` capped by the hemisphere on
    its top circle (bottom plane, cylinder, sphere; two circles, one seam). The sphere's
    one loop is its equator; its pole lies inside the face."""
    b = SolidBuilder(tol=1e-9)
    z, x = [0, 0, 1], [1, 0, 0]
    f0, f1 = Frame([0, 0, 0], z, x), Frame([0, 0, height], z, x)
    va, vb = b.vertex([r, 0, 0]), b.vertex([r, 0, height])
    c0 = b.arc(f0, r, 0.0, TAU, va, va)
    c1 = b.arc(f1, r, 0.0, TAU, vb, vb)
    seam = b.line(va, vb)
    _plane_face(b, f0, -1, [[(c0, True)]])
    lo, hi = _pad([0.0, 0.0], [TAU, height])
    cyl = b.face(CYLINDER, +1, f0, a=r, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(cyl, [
        (c0, False, line_pcurve([0.0, 0.0], [TAU, 0.0])),
        (seam, False, None),
        (c1, True, line_pcurve([TAU, height], [0.0, height])),
        (seam, True, None),
    ])
    lo, hi = _pad([0.0, 0.0], [TAU, math.pi / 2])
    sph = b.face(SPHERE, +1, f1, a=r, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(sph, [(c1, False, line_pcurve([0.0, 0.0], [TAU, 0.0]))])
    return b


def nurbs_dome(r=3.0, height=4.0, rise=None):
    """`dome` with its cap as a rational biquadratic B-spline of revolution: u the angle
    about z (four quarter arcs, knots 0..4, periodic), v the meridian from the equator
    (v = 0) to the apex (v = 1). rise None: the hemisphere (a quarter arc, the apex
    smooth); else the meridian's control points (r, height), (r / 2, height + 3 rise / 4),
    (0, height + rise), a pointed apex (a cone point). The equator is the cap's boundary
    curve (a spline edge of four rational quadratic pieces). The side v = 1 collapses to
    the apex, a pole inside the face (its one loop is the equator): the reference's pole
    feature with its fan pseudo-normal (solid3.rs:1609-1625, 1960-1986) answers the points
    whose nearest point it is."""
    s = math.sqrt(0.5)
    ring = [(1, 0, 1), (1, 1, s), (0, 1, 1), (-1, 1, s), (-1, 0, 1), (-1, -1, s), (0, -1, 1), (1, -1, s), (1, 0, 1)]
    if rise is None:
        merid = [(r, height, 1.0), (r, height + r, s), (0.0, height + r, 1.0)]
    else:
        merid = [(r, height, 1.0), (0.5 * r, height + 0.75 * rise, 1.0), (0.0, height + rise, 1.0)]
    net = np.array([[[cx * rho * wu * wv, cy * rho * wu * wv, zz * wu * wv, wu * wv] for rho, zz, wv in merid]
                    for cx, cy, wu in ring])
    ku = [0.0] * 3 + [1.0, 1.0, 2.0, 2.0, 3.0, 3.0] + [4.0] * 3
    kv = [0.0] * 3 + [1.0] * 3
    patches, ub, vb_ = surface_spans(2, 2, ku, kv, net)
    b = SolidBuilder(tol=1e-9)
    z, x = [0, 0, 1], [1, 0, 0]
    f0 = Frame([0, 0, 0], z, x)
    va, vb = b.vertex([r, 0, 0]), b.vertex([r, 0, height])
    c0 = b.arc(f0, r, 0.0, TAU, va, va)
    c1 = b.spline(_boundary_pieces(patches, "v0"), vb, vb)
    seam = b.line(va, vb)
    _plane_face(b, f0, -1, [[(c0, True)]])
    lo, hi = _pad([0.0, 0.0], [TAU, height])
    cyl = b.face(CYLINDER, +1, f0, a=r, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(cyl, [
        (c0, False, line_pcurve([0.0, 0.0], [TAU, 0.0])),
        (seam, False, None),
        (c1, True, line_pcurve([TAU, height], [0.0, height])),
        (seam, True, None),
    ])
    cap = b.face(NURBS, +1, lo=[ub[0], vb_[0]], hi=[ub[-1], vb_[-1]], period=[ub[-1] - ub[0], 0.0],
                 nurbs=(patches, ub, vb_))
    b.loop(cap, [(c1, False, line_pcurve([ub[0], 0.0], [ub[-1], 0.0]))])
    return b


def nurbs_ball(r=3.0):
    """`ball` as one rational biquadratic B-spline face of revolution with no loops: u the
    angle about z (four quarter arcs, periodic), v the meridian from the south pole
    (v = 0) to the north pole (v = 2) in two quarter arcs. Both v sides collapse to a
    point inside the face: two poles and no vertex."""
    s = math.sqrt(0.5)
    ring = [(1, 0, 1), (1, 1, s), (0, 1, 1), (-1, 1, s), (-1, 0, 1), (-1, -1, s), (0, -1, 1), (1, -1, s), (1, 0, 1)]
    merid = [(0.0, -r, 1.0), (r, -r, s), (r, 0.0, 1.0), (r, r, s), (0.0, r, 1.0)]
    net = np.array([[[cx * rho * wu * wv, cy * rho * wu * wv, zz * wu * wv, wu * wv] for rho, zz, wv in merid]
                    for cx, cy, wu in ring])
    ku = [0.0] * 3 + [1.0, 1.0, 2.0, 2.0, 3.0, 3.0] + [4.0] * 3
    kv = [0.0] * 3 + [1.0, 1.0] + [2.0] * 3
    patches, ub, vb = surface_spans(2, 2, ku, kv, net)
    b = SolidBuilder(tol=1e-9)
    b.face(NURBS, +1, lo=[ub[0], vb[0]], hi=[ub[-1], vb[-1]], period=[ub[-1] - ub[0], 0.0], nurbs=(patches, ub, vb))
    return b


def _dome_body(b: SolidBuilder, cx, cy, z0, r, height):
    """A dome standing on the plane z = z0: a cylinder of radius r to z0 + height capped by
    the hemisphere on its top circle. Returns its base circle, a hole loop for the plane."""
    z, x = [0, 0, 1], [1, 0, 0]
    f0, f1 = Frame([cx, cy, z0], z, x), Frame([cx, cy, z0 + height], z, x)
    va, vb = b.vertex([cx + r, cy, z0]), b.vertex([cx + r, cy, z0 + height])
    c0 = b.arc(f0, r, 0.0, TAU, va, va)
    c1 = b.arc(f1, r, 0.0, TAU, vb, vb)
    seam = b.line(va, vb)
    lo, hi = _pad([0.0, 0.0], [TAU, height])
    cyl = b.face(CYLINDER, +1, f0, a=r, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(cyl, [
        (c0, False, line_pcurve([0.0, 0.0], [TAU, 0.0])),
        (seam, False, None),
        (c1, True, line_pcurve([TAU, height], [0.0, height])),
        (seam, True, None),
    ])
    lo, hi = _pad([0.0, 0.0], [TAU, math.pi / 2])
    sph = b.face(SPHERE, +1, f1, a=r, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(sph, [(c1, False, line_pcurve([0.0, 0.0], [TAU, 0.0]))])
    return c0


def _plate(b: SolidBuilder, X, Y, Z, holes):
    """A plate [0,X]x[0,Y]x[0,Z] whose top face has the given hole loops (the base circles
    of bodies standing on it): bottom, four sides and the top."""
    c = {}
    for i, xx in enumerate((0.0, X)):
        for j, yy in enumerate((0.0, Y)):
            for k, zz in enumerate((0.0, Z)):
                c[i, j, k] = b.vertex([xx, yy, zz])
    L = lambda p, q: b.line(c[p], c[q])  # noqa: E731
    eb = [L((0, 0, 0), (1, 0, 0)), L((1, 0, 0), (1, 1, 0)), L((1, 1, 0), (0, 1, 0)), L((0, 1, 0), (0, 0, 0))]
    et = [L((0, 0, 1), (1, 0, 1)), L((1, 0, 1), (1, 1, 1)), L((1, 1, 1), (0, 1, 1)), L((0, 1, 1), (0, 0, 1))]
    es = {ij: L((*ij, 0), (*ij, 1)) for ij in ((0, 0), (1, 0), (1, 1), (0, 1))}
    _plane_face(b, Frame([0, 0, 0], [0, 0, 1], [1, 0, 0]), -1,
                [[(eb[3], True), (eb[2], True), (eb[1], True), (eb[0], True)]])
    _plane_face(b, Frame([0, 0, 0], [0, -1, 0], [1, 0, 0]), +1,
                [[(eb[0], False), (es[1, 0], False), (et[0], True), (es[0, 0], True)]])
    _plane_face(b, Frame([X, 0, 0], [1, 0, 0], [0, 1, 0]), +1,
                [[(eb[1], False), (es[1, 1], False), (et[1], True), (es[1, 0], True)]])
    _plane_face(b, Frame([X, Y, 0], [0, 1, 0], [-1, 0, 0]), +1,
                [[(eb[2], False), (es[0, 1], False), (et[2], True), (es[1, 1], True)]])
    _plane_face(b, Frame([0, Y, 0], [-1, 0, 0], [0, -1, 0]), +1,
                [[(eb[3], False), (es[0, 0], False), (et[3], True), (es[0, 1], True)]])
    _plane_face(b, Frame([0, 0, Z], [0, 0, 1], [1, 0, 0]), +1,
                [[(et[0], False), (et[1], False), (et[2], False), (et[3], False)]] + [[(h, True)] for h in holes])
    return b


def bodies_on_plate(seed=0, kind="boss", count=2, plate=(40.0, 30.0, 8.0)):
    """`count` bodies standing in a row on a plate: filleted bosses (kind "boss": cylinder,
    quarter-torus fillet, cap; radius U[2,5] mm, height U[3,12] mm) or domes ("dome":
    cylinder under a hemisphere; radius U[2,5] mm, cylinder height U[1,6] mm). The plate
    and its bodies are one solid: 6 + 3 count faces (bosses) or 6 + 2 count (domes)."""
    rng = Rng(seed)
    X, Y, Z = plate
    b = SolidBuilder(tol=1e-9)
    holes = []
    for k in range(count):
        cx, cy = X * (k + 0.5) / count, Y / 2
        r = min(rng.uniform(2.0, 5.0), 0.45 * min(X / count, Y))
        if kind == "boss":
            hgt = rng.uniform(3.0, 12.0)
            holes.append(_boss_body(b, cx, cy, Z, r, hgt, min(0.3 * r, 0.4 * hgt) * rng.uniform(0.5, 1.0)))
        else:
            holes.append(_dome_body(b, cx, cy, Z, r, rng.uniform(1.0, 6.0)))
    return _plate(b, X, Y, Z, holes)


def countersunk_block(size=(40.0, 30.0, 20.0), center=(20.0, 15.0), r=4.0, sink=2.0, half_angle_deg=45.0):
    """A block [0,X]x[0,Y]x[0,Z] with a through-hole of radius r along z whose top
    `sink` mm widens as a cone (the countersink) to r + sink tan(angle) at z = Z."""
    X, Y, Z = size
    ang = math.radians(half_angle_deg)
    rt = r + sink * math.tan(ang)
    zm = Z - sink
    b = SolidBuilder(tol=1e-9)
    c = {}
    for i, xx in enumerate((0.0, X)):
        for j, yy in enumerate((0.0, Y)):
            for k, zz in enumerate((0.0, Z)):
                c[i, j, k] = b.vertex([xx, yy, zz])
    L = lambda p, q: b.line(c[p], c[q])  # noqa: E731
    eb = [L((0, 0, 0), (1, 0, 0)), L((1, 0, 0), (1, 1, 0)), L((1, 1, 0), (0, 1, 0)), L((0, 1, 0), (0, 0, 0))]
    et = [L((0, 0, 1), (1, 0, 1)), L((1, 0, 1), (1, 1, 1)), L((1, 1, 1), (0, 1, 1)), L((0, 1, 1), (0, 0, 1))]
    ev = {ij: L((*ij, 0), (*ij, 1)) for ij in ((0, 0), (1, 0), (1, 1), (0, 1))}
    cx, cy = center
    va, vm, vb = b.vertex([cx + r, cy, 0.0]), b.vertex([cx + r, cy, zm]), b.vertex([cx + rt, cy, Z])
    fz0 = Frame([cx, cy, 0.0], [0, 0, 1], [1, 0, 0])
    fzm = Frame([cx, cy, zm], [0, 0, 1], [1, 0, 0])
    fz1 = Frame([cx, cy, Z], [0, 0, 1], [1, 0, 0])
    c0 = b.arc(fz0, r, 0.0, TAU, va, va)
    cm = b.arc(fzm, r, 0.0, TAU, vm, vm)
    c1 = b.arc(fz1, rt, 0.0, TAU, vb, vb)
    seam_c = b.line(va, vm)
    seam_k = b.line(vm, vb)
    _plane_face(b, Frame([0, 0, 0], [0, 0, 1], [1, 0, 0]), -1,
                [[(eb[3], True), (eb[2], True), (eb[1], True), (eb[0], True)], [(c0, False)]])
    _plane_face(b, Frame([0, 0, Z], [0, 0, 1], [1, 0, 0]), +1,
                [[(et[0], False), (et[1], False), (et[2], False), (et[3], False)], [(c1, True)]])
    _plane_face(b, Frame([0, 0, 0], [0, -1, 0], [1, 0, 0]), +1,
                [[(eb[0], False), (ev[1, 0], False), (et[0], True), (ev[0, 0], True)]])
    _plane_face(b, Frame([X, 0, 0], [1, 0, 0], [0, 1, 0]), +1,
                [[(eb[1], False), (ev[1, 1], False), (et[1], True), (ev[1, 0], True)]])
    _plane_face(b, Frame([X, Y, 0], [0, 1, 0], [-1, 0, 0]), +1,
                [[(eb[2], False), (ev[0, 1], False), (et[2], True), (ev[1, 1], True)]])
    _plane_face(b, Frame([0, Y, 0], [-1, 0, 0], [0, -1, 0]), +1,
                [[(eb[3], False), (ev[0, 0], False), (et[3], True), (ev[0, 1], True)]])
    # the hole's wall and the countersink: outward toward the axis (sense -1)
    lo, hi = _pad([0.0, 0.0], [TAU, zm])
    cyl = b.face(CYLINDER, -1, fz0, a=r, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(cyl, [
        (cm, False, line_pcurve([0.0, zm], [TAU, zm])),
        (seam_c, True, None),
        (c0, True, line_pcurve([TAU, 0.0], [0.0, 0.0])),
        (seam_c, False, None),
    ])
    lo, hi = _pad([0.0, 0.0], [TAU, sink])
    cone = b.face(CONE, -1, fzm, a=r, b=ang, lo=[0.0, lo[1]], hi=[TAU, hi[1]], period=[TAU, 0.0])
    b.loop(cone, [
        (c1, False, line_pcurve([0.0, sink], [TAU, sink])),
        (seam_k, True, None),
        (cm, True, line_pcurve([TAU, 0.0], [0.0, 0.0])),
        (seam_k, False, None),
    ])
    return b


def mold(seed=0, size=(250.0, 200.0, 80.0), rim=25.0, fu=25, fv=20, floor=40.0, bumps=10, bosses=40,
         spans=(5, 21)):
    """A mold cavity: a size block with a pocket `rim` mm in from its sides, the pocket's
    floor one clamped bicubic rational B-spline (heights floor plus `bumps` seeded
    Gaussians, amplitude U[2,8] mm, sigma U[10,40] mm; weights in [0.8, 1.2] from three
    seeded plane waves of 30-90 mm; uniform knots)
    cut along its knot lines into fu x fv faces: face column a holds m_u[a] spans, face row
    c m_v[c], each drawn from `spans`, so a face is a patch of (m_u + 3) x (m_v + 3)
    control points (8 x 8 to 24 x 24) and neighbouring faces join C2 along shared B-spline
    edges; four vertical pocket walls; and `bosses` filleted bosses (cylinder,
    quarter-torus fillet, cap; radius U[3,6] mm, height U[5,15] mm) standing on the rim.
    About 640 faces."""
    X, Y, Z = size
    ax, ay, bx, by = rim, rim, X - rim, Y - rim
    rng = Rng(seed)
    g = []
    for _ in range(bumps):
        g.append((rng.uniform(2.0, 8.0), rng.uniform(10.0, 40.0), rng.uniform(ax, bx), rng.uniform(ay, by)))
    mu = [spans[0] + int(rng.next() % (spans[1] - spans[0] + 1)) for _ in range(fu)]
    mv = [spans[0] + int(rng.next() % (spans[1] - spans[0] + 1)) for _ in range(fv)]
    su, sv = sum(mu), sum(mv)
    nu, nv = su + 3, sv + 3
    xs = ax + (bx - ax) * np.arange(nu) / (nu - 1)
    ys = ay + (by - ay) * np.arange(nv) / (nv - 1)
    XX, YY = np.meshgrid(xs, ys, indexing="ij")
    zz = floor + sum(a * np.exp(-((XX - cx) ** 2 + (YY - cy) ** 2) / (2 * s * s)) for a, s, cx, cy in g)
    # weights in [0.8, 1.2] from a seeded field over the floor (three plane waves of 30 to
    # 90 mm), not drawn a control point at a time: on a net of control points a fraction
    # of a millimetre apart, independent weights would ripple the surface at that scale
    waves = [(rng.uniform(30.0, 90.0), rng.uniform(0.0, TAU), rng.uniform(0.0, TAU)) for _ in range(3)]
    w = 1.0 + 0.2 / 3.0 * sum(np.cos(TAU / L * (XX * math.cos(a) + YY * math.sin(a)) + ph) for L, a, ph in waves)
    net = np.stack([XX * w, YY * w, zz * w, w], -1)
    ku = [0.0] * 4 + [k / su for k in range(1, su)] + [1.0] * 4
    kv = [0.0] * 4 + [k / sv for k in range(1, sv)] + [1.0] * 4
    patches, ub, vb = surface_spans(3, 3, ku, kv, net)
    b = SolidBuilder(tol=1e-9)
    cu = [int(x) for x in np.concatenate([[0], np.cumsum(mu)])]
    cv = [int(x) for x in np.concatenate([[0], np.cumsum(mv)])]
    fvx, eu, ev = _spline_faces(b, patches, ub, vb, cu, cv)
    # the block's corners, the rim's corners at the top and the pocket walls' vertical edges
    cb = {}
    for i, xx in enumerate((0.0, X)):
        for j, yy in enumerate((0.0, Y)):
            for k, zz in enumerate((0.0, Z)):
                cb[i, j, k] = b.vertex([xx, yy, zz])
    L = lambda p, q: b.line(cb[p], cb[q])  # noqa: E731
    eb = [L((0, 0, 0), (1, 0, 0)), L((1, 0, 0), (1, 1, 0)), L((1, 1, 0), (0, 1, 0)), L((0, 1, 0), (0, 0, 0))]
    et = [L((0, 0, 1), (1, 0, 1)), L((1, 0, 1), (1, 1, 1)), L((1, 1, 1), (0, 1, 1)), L((0, 1, 1), (0, 0, 1))]
    es = {ij: L((*ij, 0), (*ij, 1)) for ij in ((0, 0), (1, 0), (1, 1), (0, 1))}
    rv = {(0, 0): b.vertex([ax, ay, Z]), (1, 0): b.vertex([bx, ay, Z]), (1, 1): b.vertex([bx, by, Z]),
          (0, 1): b.vertex([ax, by, Z])}
    fc = {(0, 0): fvx[0, 0], (1, 0): fvx[fu, 0], (1, 1): fvx[fu, fv], (0, 1): fvx[0, fv]}
    rl = [b.line(rv[0, 0], rv[1, 0]), b.line(rv[1, 0], rv[1, 1]), b.line(rv[1, 1], rv[0, 1]), b.line(rv[0, 1], rv[0, 0])]
    wv = {ij: b.line(fc[ij], rv[ij]) for ij in fc}  # up from the floor's corners
    # outer block: bottom and four sides
    _plane_face(b, Frame([0, 0, 0], [0, 0, 1], [1, 0, 0]), -1,
                [[(eb[3], True), (eb[2], True), (eb[1], True), (eb[0], True)]])
    _plane_face(b, Frame([0, 0, 0], [0, -1, 0], [1, 0, 0]), +1,
                [[(eb[0], False), (es[1, 0], False), (et[0], True), (es[0, 0], True)]])
    _plane_face(b, Frame([X, 0, 0], [1, 0, 0], [0, 1, 0]), +1,
                [[(eb[1], False), (es[1, 1], False), (et[1], True), (es[1, 0], True)]])
    _plane_face(b, Frame([X, Y, 0], [0, 1, 0], [-1, 0, 0]), +1,
                [[(eb[2], False), (es[0, 1], False), (et[2], True), (es[1, 1], True)]])
    _plane_face(b, Frame([0, Y, 0], [-1, 0, 0], [0, -1, 0]), +1,
                [[(eb[3], False), (es[0, 0], False), (et[3], True), (es[0, 1], True)]])
    # the pocket's walls, outward into the pocket: each runs along the floor's boundary
    # edges, up a corner, back along the rim, down the other corner (counterclockwise seen
    # from the pocket)
    front = [(ev[a, 0], True) for a in reversed(range(fu))]  # y = ay, x from bx to ax
    _plane_face(b, Frame([bx, ay, 0], [0, 1, 0], [-1, 0, 0]), +1,
                [front + [(wv[0, 0], False), (rl[0], False), (wv[1, 0], True)]])
    right = [(eu[fu, c], True) for c in reversed(range(fv))]  # x = bx, y from by to ay
    _plane_face(b, Frame([bx, by, 0], [-1, 0, 0], [0, -1, 0]), +1,
                [right + [(wv[1, 0], False), (rl[1], False), (wv[1, 1], True)]])
    back = [(ev[a, fv], False) for a in range(fu)]  # y = by, x from ax to bx
    _plane_face(b, Frame([ax, by, 0], [0, -1, 0], [1, 0, 0]), +1,
                [back + [(wv[1, 1], False), (rl[2], False), (wv[0, 1], True)]])
    left = [(eu[0, c], False) for c in range(fv)]  # x = ax, y from ay to by
    _plane_face(b, Frame([ax, ay, 0], [1, 0, 0], [0, 1, 0]), +1,
                [left + [(wv[0, 1], False), (rl[3], False), (wv[0, 0], True)]])
    # bosses on the rim's centre line, evenly spaced by arc length
    half = rim / 2
    px, py = X - rim, Y - rim  # the centre line's rectangle sides
    per = 2 * (px + py)
    holes = []
    for k in range(bosses):
        t = (k + 0.5) * per / bosses
        if t < px:
            cx, cy = half + t, half
        elif t < px + py:
            cx, cy = X - half, half + (t - px)
        elif t < 2 * px + py:
            cx, cy = X - half - (t - px - py), Y - half
        else:
            cx, cy = half, Y - half - (t - 2 * px - py)
        r = rng.uniform(3.0, 6.0)
        hgt = rng.uniform(5.0, 15.0)
        fil = min(0.3 * r, 0.4 * hgt) * rng.uniform(0.5, 1.0)
        holes.append([(_boss_body(b, cx, cy, Z, r, hgt, fil), True)])
    # the top: the block's outline, the pocket's rim as a hole, the bosses' bases as holes
    _plane_face(b, Frame([0, 0, Z], [0, 0, 1], [1, 0, 0]), +1,
                [[(et[0], False), (et[1], False), (et[2], False), (et[3], False)],
                 [(rl[3], True), (rl[2], True), (rl[1], True), (rl[0], True)]] + holes)
    return b


CONFIGS = {
    "can": can,
    "bump_box": bump_box,
    "block_with_hole": block_with_hole,
    "freeform_top": freeform_top,
}
