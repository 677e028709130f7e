"""The CUDA library as a C ABI, without a GPU: it loads, exports every entry point
include/icam_cuda.h declares, checks its arguments, and fails loudly (an error code
and message, never a CPU path) when no device is there."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from implicitcam_b200 import build, part_gpu, parts

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "icam_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(icam_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return C.CDLL(part_gpu.LIB)


def test_exports_every_declared_entry_point(lib):
    names = declared()
    assert len(names) >= 12, names
    for n in names:
        assert hasattr(lib, n), n


def test_solid_descriptions_are_closed_shells():
    for name, make in parts.CONFIGS.items():
        b = make()
        d = b.desc()
        assert d.n_faces > 0 and d.n_edges > 0 and d.n_verts > 0, name
        # every edge used by two faces (twice by one for a seam)
        for i in range(d.n_edges):
            e = d.edges[i]
            assert e.f0 >= 0 and e.f1 >= 0, (name, i)


def test_bad_arguments_are_refused(lib):
    L = part_gpu.lib()
    err = C.create_string_buffer(256)
    h = C.c_void_p()
    assert L.icam_pack_create(None, None, C.byref(h), err, 256) == 1
    assert b"null" in err.value
    assert L.icam_pack_info(None, None) == 1


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="a GPU is present")
def test_no_gpu_fails_loudly():
    with pytest.raises(part_gpu.IcamError) as e:
        part_gpu.PartGpu(parts.block_with_hole())
    assert "cuda" in str(e.value).lower()


def test_rust_binding_names_match_the_header():
    """The Rust extern block of the integration guide binds exactly the header's entry points."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    rust = sorted(set(re.findall(r"pub fn (icam_\w+)\(", text)))
    assert rust == declared()


def test_a_creased_bspline_face_is_refused():
    """A B-spline face with a C0 crease along an interior knot line (a triple knot of a
    cubic whose control heights fold there) is refused when packed, before any device
    work: the pack has no knot-line features (Exact::c0_line), so it must not bake such
    a face with the crease's nearest points missing. The same top without the fold packs."""
    import numpy as np

    from implicitcam_b200 import part_gpu, parts
    from implicitcam_b200.solid import SolidBuilder

    def top(fold):
        n, size = 7, 30.0
        net = np.zeros((n, n, 4))
        for i in range(n):
            for j in range(n):
                x, y = size * i / (n - 1), size * j / (n - 1)
                z = 10.0 + (fold * abs(x - size / 2) if fold else 0.02 * x * y / size)
                net[i, j] = [x, y, z, 1.0]
        knots = [0.0] * 4 + [0.5] * 3 + [1.0] * 4
        return parts._nurbs_box(SolidBuilder(tol=1e-9), 3, 3, knots, knots, net, size, size)

    with pytest.raises(part_gpu.IcamError, match="crease"):
        part_gpu.PartGpu(top(0.3))
    # the unfolded top passes the check (it may then fail only for want of a GPU)
    try:
        part_gpu.PartGpu(top(0.0)).close()
    except part_gpu.IcamError as e:
        assert "crease" not in str(e) and "pole" not in str(e)
