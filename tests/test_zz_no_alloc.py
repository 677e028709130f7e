"""icam_bricks_static, the brick read that allocates nothing, against icam_bricks.

Some callers cannot allocate while they read bricks: a machining simulation that
reserved the GPU's memory for its stock model up front, or a loop between its own
stream-ordered kernels that cannot take cudaFree's device-wide wait. For them the
library reads bricks through one fixed device array. These tests call it through the
C ABI, two calls in a row on different bricks, each compared with icam_bricks on the
same bricks: the double values within 1e-9 of the part's box diagonal (1e-7 for the
mixed kernels), the flags and the float pairs equal. The second call checks that the
shared device array carries nothing over from the first. Runs alone in a fresh
process as well as after the other GPU tests (its file name sorts last).
"""
import ctypes as C

import numpy as np
import pytest

from implicitcam_b200 import part_gpu, parts

pytestmark = pytest.mark.gpu

TOL = {part_gpu.FP64: 1e-9, part_gpu.MIXED: 1e-7, part_gpu.MIXED_LEARNED: 1e-7}  # x diagonal
MAX_BRICKS = 256  # ICAM_STATIC_BRICKS


@pytest.fixture(scope="module")
def part(oracle_mod):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    b = parts.block_with_hole()
    g = part_gpu.PartGpu(b)
    lo, hi = oracle_mod.Oracle(b).bbox()
    L = part_gpu.lib()
    f = L.icam_bricks_static
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_void_p,
                  C.c_char_p, C.c_size_t]
    yield g, f, np.asarray(lo, float), np.asarray(hi, float)
    g.close()


def first_nodes(lo, hi, h, offset, count):
    """count bricks of cell side h on a grid over the part's box, shifted by offset."""
    lo2 = lo - 2 * h + offset
    nb = np.maximum(1, np.ceil((hi - lo2 + 2 * h) / (8 * h))).astype(int)
    ijk = np.stack(np.meshgrid(*[np.arange(k) for k in nb], indexing="ij"), -1).reshape(-1, 3)
    firsts = lo2 + ijk * 8 * h
    step = max(1, len(firsts) // count)
    return np.ascontiguousarray(firsts[::step][:count])


def call_static(f, g, firsts, h, clamp, precision, want_vals=True, want_d=True):
    n = len(firsts)
    vals = np.full((n, 729, 2), np.nan, np.float32)
    d = np.full((n, 729), np.nan)
    err = C.create_string_buffer(256)
    rc = f(g.h, firsts.ctypes.data, n, h, clamp, precision, vals.ctypes.data if want_vals else None,
           d.ctypes.data if want_d else None, err, 256)
    assert rc == 0, err.value
    return vals, d


def check_against_icam_bricks(g, f, firsts, h, clamp, precision, diag):
    vals_s, d_s = call_static(f, g, firsts, h, clamp, precision)
    vals_r, d_r = g.bricks(firsts, h, clamp, precision=precision)
    assert np.array_equal(vals_s[:, :, 1], vals_r[:, :, 1])
    assert (vals_s[:, :, 1] != 2).all()
    assert np.abs(d_s - d_r).max() <= TOL[precision] * diag
    assert np.abs(vals_s[:, :, 0] - vals_r[:, :, 0]).max() <= TOL[precision] * diag + 1e-6 * clamp


def test_two_calls_match_icam_bricks(part):
    g, f, lo, hi = part
    diag = float(np.linalg.norm(hi - lo))
    cases = [
        (first_nodes(lo, hi, 0.5, 0.0, 200), 0.5, 0.5 * np.sqrt(3), part_gpu.FP64),
        (first_nodes(lo, hi, 0.25, 0.37, MAX_BRICKS), 0.25, 2.0, part_gpu.MIXED),
    ]
    for firsts, h, clamp, precision in cases:
        check_against_icam_bricks(g, f, firsts, h, clamp, precision, diag)


def test_one_output_at_a_time(part):
    """values_out alone and d_out alone: the other one is not written."""
    g, f, lo, hi = part
    firsts = first_nodes(lo, hi, 0.5, 0.11, 64)
    h, clamp = 0.5, 0.5 * np.sqrt(3)
    vals_r, d_r = g.bricks(firsts, h, clamp)
    vals_s, d_s = call_static(f, g, firsts, h, clamp, part_gpu.FP64, want_d=False)
    assert np.isnan(d_s).all()
    assert np.array_equal(vals_s, vals_r)
    vals_s, d_s = call_static(f, g, firsts, h, clamp, part_gpu.FP64, want_vals=False)
    assert np.isnan(vals_s).all()
    assert np.array_equal(d_s, d_r)
    err = C.create_string_buffer(256)
    assert f(g.h, None, 0, h, clamp, part_gpu.FP64, None, None, err, 256) == 0  # no bricks: nothing to do


def test_learned_needs_the_seed_network_then_matches(oracle_mod):
    """ICAM_MIXED_LEARNED: refused before the pack's seed network is trained, as
    icam_bricks refuses it; after training, two calls in a row agree with icam_bricks."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    b = parts.freeform_top(seed=0)
    g = part_gpu.PartGpu(b)
    L = part_gpu.lib()
    f = L.icam_bricks_static
    lo, hi = (np.asarray(x, float) for x in oracle_mod.Oracle(b).bbox())
    diag = float(np.linalg.norm(hi - lo))
    firsts = first_nodes(lo + [0, 0, 45], hi, 0.5, 0.0, 128)  # bricks about the B-spline top
    err = C.create_string_buffer(256)
    rc = f(g.h, firsts.ctypes.data, len(firsts), 0.5, 2.0, part_gpu.MIXED_LEARNED, None, None, err, 256)
    assert rc == 1 and b"seed network" in err.value  # ICAM_ERR_ARG
    with pytest.raises(part_gpu.IcamError):
        g.bricks(firsts, 0.5, 2.0, precision=part_gpu.MIXED_LEARNED)
    g.seednet_train(300, batch=1024, seed=1)
    check_against_icam_bricks(g, f, firsts, 0.5, 2.0, part_gpu.MIXED_LEARNED, diag)
    check_against_icam_bricks(g, f, first_nodes(lo + [0, 0, 45], hi, 0.25, 0.13, MAX_BRICKS), 0.25, 2.0,
                              part_gpu.MIXED_LEARNED, diag)
    g.close()


def test_too_many_bricks_is_refused(part):
    g, f, lo, hi = part
    firsts = np.zeros((MAX_BRICKS + 1, 3))
    err = C.create_string_buffer(256)
    rc = f(g.h, firsts.ctypes.data, len(firsts), 0.5, 1.0, part_gpu.FP64, None, None, err, 256)
    assert rc == 7  # ICAM_ERR_ROOM
    assert b"257 bricks asked, at most 256" in err.value
