"""The library's double-precision point query run on the CPU.

The search of the k_points kernel (field.cuh: the tree walk, the per-feature evaluators,
the sub-patch branch and bound with its pole rules) is written as __host__ __device__
functions; `host_field.cu` builds it for the host over a pack made by the library's own
builder. Here it answers random points of every part family, creases and poles included,
and must agree with the oracle (the reference's search restated) within 1e-9 of the
part's diagonal with the same signs, every point decided. This checks the device
algorithm itself without a GPU; the B200 tests check the kernels.

Near a pointed pole the oracle keeps the reference's search, which can return the pole up
to ~1e-7 mm farther than the cap's true foot at the edge of the pole's normal cone (the
library finds the foot); there the bar is 1e-7 of the diagonal for every point and 1e-9
for nearly all.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from implicitcam_b200 import parts

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    out = str(tmp_path_factory.mktemp("host_field") / "libhost_field.so")
    csrc = os.path.join(ROOT, "implicitcam_b200", "csrc")
    # the device code is not run: PTX for one architecture keeps the build to seconds
    cmd = [nvcc, "-Xcompiler", "-fPIC", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=compute_100a",
           "-shared", "-o", out, os.path.join(HERE, "host_field.cu"), os.path.join(csrc, "pack_build.cpp"),
           os.path.join(csrc, "host_geom.cpp")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    lib = C.CDLL(out)
    lib.host_points.restype = C.c_int
    lib.host_points.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_long, C.c_double, C.c_void_p, C.c_void_p,
                                C.c_char_p, C.c_size_t]
    return lib


def host_points(lib, solid, p, need=2.0, cap=np.inf):
    desc = solid.desc()
    p = np.ascontiguousarray(p, dtype=np.float64)
    v = np.zeros(len(p))
    f = np.zeros(len(p), np.int32)
    err = C.create_string_buffer(512)
    rc = lib.host_points(C.addressof(desc), need, p.ctypes.data, len(p), cap, v.ctypes.data, f.ctypes.data, err,
                         512)
    assert rc == 0, err.value
    return v, f


CASES = {
    "can": lambda: parts.can(),
    "block_with_hole": lambda: parts.block_with_hole(),
    "bump_box": lambda: parts.bump_box(),
    "freeform_top": lambda: parts.freeform_top(seed=3, n=8, size=40.0, base=20.0, bumps=4),
    "countersunk_block": lambda: parts.countersunk_block(),
    "bosses_on_plate": lambda: parts.bodies_on_plate(seed=2, kind="boss", count=2, plate=(24.0, 12.0, 4.0)),
    "domes_on_plate": lambda: parts.bodies_on_plate(seed=2, kind="dome", count=2, plate=(24.0, 12.0, 4.0)),
    "freeform_patches": lambda: parts.freeform_patches(seed=11, n=14, size=40.0, base=15.0, bumps=5, degree=2,
                                                       faces=6),
    "ridge": lambda: parts.ridge_box(fold=0.3, size=30.0, base=13.0, wave=1.5, n=9),
    "round_pole": lambda: parts.nurbs_dome(3.0, 4.0),
    "pointed_pole": lambda: parts.nurbs_dome(3.0, 4.0, rise=2.0),
    "two_poles": lambda: parts.nurbs_ball(3.0),
}


@pytest.mark.parametrize("name", list(CASES))
def test_device_search_on_the_host(oracle_mod, host_lib, name):
    solid = CASES[name]()
    o = oracle_mod.Oracle(solid)
    lo, hi = map(np.asarray, o.bbox())
    diag = float(np.linalg.norm(hi - lo))
    rng = np.random.default_rng(len(name))
    p = rng.uniform(lo - 2.0, hi + 2.0, (1500, 3))
    if "pole" in name:  # off the axis of revolution (on it the searches run to their budgets)
        p = np.concatenate([p, rng.normal([0.0, 0.0, hi[2]], 0.5, (1500, 3))])
        p = p[np.hypot(p[:, 0], p[:, 1]) > 0.05]
    v, f = host_points(host_lib, solid, p)
    d = o.sdf(p)[0]
    assert (f == 0).all()
    err = np.abs(v - d)
    if name == "pointed_pole":
        assert (err < 1e-9 * diag).mean() > 0.99 and err.max() < 1e-7 * diag
    else:
        assert err.max() < 1e-9 * diag
    sure = np.abs(d) > 1e-9
    assert (np.sign(v[sure]) == np.sign(d[sure])).all()


@pytest.mark.parametrize("name", ["block_with_hole", "freeform_top", "ridge", "pointed_pole"])
def test_capped_reads_on_the_host(oracle_mod, host_lib, name):
    """A read capped at 1 mm (the decision's and the brick lists' reads): exact with flag
    0 within the cap, the cap with flag 1 past it (gpu.wgsl:1909-1921)."""
    solid = CASES[name]()
    o = oracle_mod.Oracle(solid)
    lo, hi = map(np.asarray, o.bbox())
    diag = float(np.linalg.norm(hi - lo))
    rng = np.random.default_rng(9)
    p = rng.uniform(lo - 2.0, hi + 2.0, (1500, 3))
    if "pole" in name:
        p = p[np.hypot(p[:, 0], p[:, 1]) > 0.05]
    cap = 1.0
    v, f = host_points(host_lib, solid, p, cap=cap)
    d = o.sdf(p)[0]
    inner, outer = np.abs(d) < cap - 1e-9, np.abs(d) > cap + 1e-9
    assert inner.sum() > 50 and outer.sum() > 50
    assert (f[inner] == 0).all() and np.abs(v[inner] - d[inner]).max() < 1e-7 * diag
    assert (f[outer] == 1).all() and (v[outer] == cap).all()
