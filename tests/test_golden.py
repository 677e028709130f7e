"""The oracle against the committed golden vectors (tests/golden/, made from the
reference tests' closed forms and brute force by make_golden.py). CPU only."""
import os

import numpy as np

from implicitcam_b200 import parts

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def test_can_golden(oracle_mod):
    g = load("can")
    d, _, _, _, unsure, _ = oracle_mod.Oracle(parts.can()).sdf(g["points"])
    assert not unsure.any()
    assert np.abs(d - g["sdf"]).max() < 1e-9  # solid3.rs:2066


def test_bump_box_golden(oracle_mod):
    g = load("bump_box")
    d, _, _, _, unsure, _ = oracle_mod.Oracle(parts.bump_box()).sdf(g["points"])
    assert not unsure.any()
    assert ((d < 0) == g["inside"]).all()
    assert (np.abs(d) <= g["dense"] + 1e-9).all()
    assert (np.abs(d) >= g["dense"] - float(g["h"])).all()


def test_block_with_hole_golden(oracle_mod):
    g = load("block_with_hole")
    d, _, _, _, unsure, _ = oracle_mod.Oracle(parts.block_with_hole()).sdf(g["points"])
    assert not unsure.any()
    assert np.abs(d - g["sdf"]).max() < 1e-9
    assert (np.sign(d) == np.sign(g["sdf"])).all()


def test_oracle_level_of_the_block(oracle_mod):
    """The oracle's bake on its own: brick map entries agree with the centre's sign,
    every read brick straddles or nears the surface (partcache.rs:301-313)."""
    o = oracle_mod.Oracle(parts.block_with_hole())
    h, lo, nb = 1.0, np.array([-2.0, -2.0, -2.0]), np.array([13, 8, 6])
    clamp = h * np.sqrt(3)
    m, idx, dc = o.decide(h, lo, nb, clamp)
    r = 0.5 * np.sqrt(3) * (8 * h + 2 * clamp)
    assert (np.abs(dc) <= r + clamp + 1e-9).all()
    cen = np.stack([np.arange(m.size) % nb[0], (np.arange(m.size) // nb[0]) % nb[1], np.arange(m.size) // (nb[0] * nb[1])], 1)
    c = lo + 8 * h * cen + 4 * h
    air = m == oracle_mod.AIR
    d = o.sdf(c[air | (m == oracle_mod.SOLID)])[0]
    assert ((d > 0) == air[air | (m == oracle_mod.SOLID)]).all()
