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


def test_a_creased_bspline_face_packs():
    """A B-spline face creased along an interior knot line (a triple knot of a cubic whose
    control heights fold there) passes the pack's checks before any device work: the
    crease becomes the face's own edge (its pieces along the knot line, the spans either
    side for its sign). On a machine without a GPU the call then fails for want of one,
    not for the crease."""
    try:
        part_gpu.PartGpu(parts.ridge_box(fold=0.3)).close()
    except part_gpu.IcamError as e:
        assert "crease" not in str(e) and "pole" not in str(e)
