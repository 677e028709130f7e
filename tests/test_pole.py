"""Poles: a B-spline face whose domain side collapses on to one point inside the face
(parts.nurbs_dome: a cap of revolution whose meridians meet at the apex; the reference's
pole feature, crates/icam-core/src/solid3.rs:1609-1625, 1960-1986, and the Creases rule of
surface3.rs:579-591).

CPU: with a pointed apex, the oracle's distances equal the closed form (the distance in the
meridian plane to the profile: bottom, wall and the quadratic meridian), above the apex
where the pole is the nearest point and everywhere around it; with the hemisphere, they
equal the analytic dome's; a sphere made of one such face with a pole at each end and no
loops equals the analytic ball; the pack takes the faces. B200: the library's points equal the
closed form (pointed apex) and agree with the oracle with equal signs, and its levels are
the oracle's (the map identical, i16 words within one step, no sign flip).

Where a point lies a hair outside the pointed apex's normal cone its nearest point is on
the cap within ~1e-3 mm of the apex, where the surface's u-tangent all but vanishes and is
known only to the rounding of nearly equal control points: the reference's critical-point
test (surface3.rs:565-572) rejects the nearest point there, the search has already lowered
its bound to that distance, and the pole answers, up to ~1e-7 mm farther. The oracle keeps
that behaviour (such points are a sliver of the cone's edge: the tests hold nearly every
point to 1e-12 and every point to the bake's 1e-7 of the diagonal); the library
scales that test's allowance on sub-patches beside a pole and finds the nearest point.
"""
import numpy as np
import pytest

from implicitcam_b200 import part_gpu, parts

R, H, RISE = 3.0, 4.0, 2.0


def profile_distance(p):
    """Signed distance to the pointed dome by its symmetry: in the meridian half-plane
    (rho, z), to the bottom segment, the wall and the quadratic Bezier meridian
    (r, H), (r / 2, H + 3 rise / 4), (0, H + rise), negative inside."""
    rho, z = np.hypot(p[:, 0], p[:, 1]), p[:, 2]
    q = np.stack([rho, z], 1)
    P0, P1, P2 = np.array([R, H]), np.array([0.5 * R, H + 0.75 * RISE]), np.array([0.0, H + RISE])
    t = np.linspace(0.0, 1.0, 4001)
    C = ((1 - t) ** 2)[:, None] * P0 + (2 * t * (1 - t))[:, None] * P1 + (t ** 2)[:, None] * P2
    tt = t[np.argmin(((q[:, None, :] - C[None]) ** 2).sum(2), 1)]
    for _ in range(30):  # Newton on the squared distance, kept in [0, 1]
        c = ((1 - tt) ** 2)[:, None] * P0 + (2 * tt * (1 - tt))[:, None] * P1 + (tt ** 2)[:, None] * P2
        dc = (2 * (1 - tt))[:, None] * (P1 - P0) + (2 * tt)[:, None] * (P2 - P1)
        ddc = 2 * (P2 - 2 * P1 + P0)
        g = ((c - q) * dc).sum(1)
        hh = (dc * dc).sum(1) + ((c - q) * ddc).sum(1)
        tt = np.clip(tt - g / hh, 0.0, 1.0)
    c = ((1 - tt) ** 2)[:, None] * P0 + (2 * tt * (1 - tt))[:, None] * P1 + (tt ** 2)[:, None] * P2
    d = np.hypot(*(c - q).T)
    d = np.minimum(d, np.hypot(rho - R, z - np.clip(z, 0.0, H)))  # the wall
    d = np.minimum(d, np.hypot(rho - np.minimum(rho, R), z))  # the bottom
    # inside: under the meridian (rho(t) = r (1 - t^2 / 2 - ... ) is monotone: solve it)
    a, b, c0 = P0[0] - 2 * P1[0] + P2[0], 2 * (P1[0] - P0[0]), P0[0] - rho
    tr = np.where(np.abs(a) > 0, (-b - np.sqrt(np.maximum(b * b - 4 * a * c0, 0.0))) / (2 * a if a else 1.0), -c0 / b)
    tr = np.where((tr < 0) | (tr > 1), (-b + np.sqrt(np.maximum(b * b - 4 * a * c0, 0.0))) / (2 * a if a else 1.0), tr)
    zc = (1 - tr) ** 2 * P0[1] + 2 * tr * (1 - tr) * P1[1] + tr ** 2 * P2[1]
    inside = (z > 0) & (rho < R) & ((z < H) | (z < zc))
    return np.where(inside, -d, d)


def test_pointed_apex_is_the_closed_form(oracle_mod):
    o = oracle_mod.Oracle(parts.nurbs_dome(R, H, rise=RISE))
    rng = np.random.default_rng(0)
    apex = np.array([0.0, 0.0, H + RISE])
    # above the apex, inside its normal cone (the pole nearest), and all around the part
    up = apex + np.stack([rng.uniform(-0.4, 0.4, 1500), rng.uniform(-0.4, 0.4, 1500), rng.uniform(0.05, 2.0, 1500)], 1)
    near = apex + rng.normal(0.0, 0.4, (1500, 3))
    wide = rng.uniform([-5, -5, -2], [5, 5, 9], (1500, 3))
    p = np.concatenate([up, near, wide])
    d = o.sdf(p)[0]
    ref = profile_distance(p)
    err = np.abs(d - ref)
    assert (err < 1e-12).mean() > 0.99
    assert err.max() < 1e-7 * np.linalg.norm([2 * R, 2 * R, H + RISE])
    assert (np.sign(d) == np.sign(ref)).all()
    at_pole = np.linalg.norm(p - apex, axis=1) - np.abs(d) < 1e-12
    assert at_pole.sum() > 300  # the pole is the nearest point of many of them


def test_round_apex_is_the_analytic_dome(oracle_mod):
    a = oracle_mod.Oracle(parts.dome(R, H))
    n = oracle_mod.Oracle(parts.nurbs_dome(R, H))
    rng = np.random.default_rng(1)
    p = np.concatenate([rng.normal([0, 0, H + R], 0.5, (2000, 3)), rng.uniform([-5, -5, -2], [5, 5, 9], (2000, 3))])
    p = p[np.hypot(p[:, 0], p[:, 1]) > 1e-3]  # off the axis (on it the reference's search runs to its cap)
    da, dn = a.sdf(p), n.sdf(p)
    assert np.abs(da[0] - dn[0]).max() < 1e-11
    assert (np.sign(da[0]) == np.sign(dn[0])).all()
    assert not dn[4].any()


def test_two_poles_are_the_ball(oracle_mod):
    """A sphere as one B-spline face with no loops collapsing at both poles."""
    a = oracle_mod.Oracle(parts.ball(R))
    n = oracle_mod.Oracle(parts.nurbs_ball(R))
    rng = np.random.default_rng(2)
    p = np.concatenate([rng.uniform(-5, 5, (2000, 3)), np.array([0, 0, R]) + rng.normal(0, 0.3, (1000, 3)),
                        np.array([0, 0, -R]) + rng.normal(0, 0.3, (1000, 3))])
    p = p[np.hypot(p[:, 0], p[:, 1]) > 1e-3]
    da, dn = a.sdf(p), n.sdf(p)
    assert np.abs(da[0] - dn[0]).max() < 1e-11
    assert (np.sign(da[0]) == np.sign(dn[0])).all()
    assert not dn[4].any()


def test_a_pole_face_packs():
    """The pack takes a face with a pole (the point feature and the never-cleared sides)
    before any device work; on a machine without a GPU the call then fails for want of
    one, not for the pole."""
    for solid in (parts.nurbs_dome(R, H), parts.nurbs_dome(R, H, rise=RISE), parts.nurbs_ball(R)):
        try:
            part_gpu.PartGpu(solid).close()
        except part_gpu.IcamError as e:
            assert "no normal" not in str(e) and "B-spline" not in str(e)


def _oracle_level(o, h, lo, nb, clamp):
    om, idx, _ = o.decide(h, lo, nb, clamp)
    idx = np.sort(idx)
    m = om.copy()
    atlas = []
    if len(idx):
        firsts = np.stack([lo[0] + 8 * h * (idx % nb[0]), lo[1] + 8 * h * ((idx // nb[0]) % nb[1]),
                           lo[2] + 8 * h * (idx // (nb[0] * nb[1]))], 1)
        _, _, kind, words = o.bricks(firsts, h, clamp)
        for j, bi in enumerate(idx):
            m[bi] = part_gpu.AIR if kind[j] == 1 else (part_gpu.SOLID if kind[j] == 2 else len(atlas))
            if kind[j] == 0:
                atlas.append(words[j])
    return m, np.array(atlas, dtype=np.uint32).reshape(-1, 365)


@pytest.mark.gpu
def test_two_poles_on_the_gpu(oracle_mod):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    g = part_gpu.PartGpu(parts.nurbs_ball(R), need=1.0)
    try:
        rng = np.random.default_rng(4)
        p = np.concatenate([rng.uniform(-5, 5, (4000, 3)), np.array([0, 0, R]) + rng.normal(0, 0.3, (2000, 3)),
                            np.array([0, 0, -R]) + rng.normal(0, 0.3, (2000, 3))])
        p = p[np.hypot(p[:, 0], p[:, 1]) > 0.05]
        v, f = g.points(p)
        assert (f == 0).all()
        assert np.abs(v - (np.linalg.norm(p, axis=1) - R)).max() < 1e-9 * 2 * R * np.sqrt(3)
    finally:
        g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("rise", [RISE, None])
def test_poles_on_the_gpu(oracle_mod, rise):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    b = parts.nurbs_dome(R, H, rise=rise)
    o = oracle_mod.Oracle(b)
    lo, hi = map(np.asarray, o.bbox())
    diag = float(np.linalg.norm(hi - lo))
    h, clamp = 0.1, 0.5
    g = part_gpu.PartGpu(b, need=clamp + 4 * h * np.sqrt(3))
    try:
        rng = np.random.default_rng(3)
        top = H + (R if rise is None else rise)
        p = np.concatenate([np.array([0.0, 0.0, top]) + rng.normal(0.0, 0.5, (8000, 3)),
                            rng.uniform([-5, -5, -2], [5, 5, top + 2], (8000, 3))])
        # off the axis: on it, under a round apex, the pole is as near as the cap's foot
        # and both searches run to their budgets
        p = p[np.hypot(p[:, 0], p[:, 1]) > (0.05 if rise is None else 1e-3)]
        v, f = g.points(p)
        d = o.sdf(p)[0]
        assert (f == 0).all()
        if rise is not None:
            assert np.abs(v - profile_distance(p)).max() < 1e-9 * diag
        err = np.abs(v - d)
        assert (err < 1e-9 * diag).mean() > 0.99
        assert err.max() < 1e-7 * diag
        assert (np.sign(v[np.abs(d) > 1e-9]) == np.sign(d[np.abs(d) > 1e-9])).all()
        # a level whose nodes keep off the axis (0.0371 from it at least)
        l2 = lo - clamp - 0.0371
        nb = np.ceil((hi - l2 + clamp) / (8 * h)).astype(np.int64)
        m0, oa = _oracle_level(o, h, l2, nb, clamp)
        qo = part_gpu.unpack_atlas(oa).astype(np.int64)
        for prec in (part_gpu.FP64, part_gpu.MIXED):
            m, a, st = g.level(h, l2, nb, clamp, precision=prec)
            assert st["nodes_undecided"] == 0
            assert (m == m0).all() and a.shape == oa.shape
            qg = part_gpu.unpack_atlas(a).astype(np.int64)
            assert np.abs(qg - qo).max() <= 1
            assert not ((qg > 0) & (qo < 0)).any() and not ((qg < 0) & (qo > 0)).any()
            if prec == part_gpu.FP64:
                assert (qg == qo).mean() > 0.999
    finally:
        g.close()
