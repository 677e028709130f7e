"""Python binding of the C ABI (include/icam_cuda.h), mirroring the reference's GPU
host for the part field, ``PartGpu`` (crates/icam-sim/src/partgpu.rs), and the level
bake of ``PartCache`` (crates/icam-sim/src/partcache.rs).

Every call runs the CUDA library ``libicam_cuda.so`` built in this package; there is
no CPU path. A missing library or GPU raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .solid import IcamSolidDesc

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libicam_cuda.so")

FP64, MIXED, MIXED_LEARNED = 0, 1, 2
AIR, SOLID, WORDS = 0xFFFFFFFF, 0xFFFFFFFE, 365
READ = 0xFFFFFFF0  # a brick the box decision leaves to be read

_lib = None


class IcamPackOptions(C.Structure):
    _fields_ = [("device", C.c_int), ("need", C.c_double)]


class IcamBakeStats(C.Structure):
    _fields_ = [
        ("boxes_read", C.c_int64), ("bricks_read", C.c_int64), ("bricks_words", C.c_int64),
        ("nodes_exact", C.c_int64), ("nodes_far", C.c_int64), ("nodes_undecided", C.c_int64),
        ("pairs", C.c_int64), ("fallback_nodes", C.c_int64), ("kernel_launches", C.c_int64),
        ("ms_decide", C.c_double), ("ms_cull", C.c_double), ("ms_nodes", C.c_double), ("ms_post", C.c_double),
        ("census", C.c_int64 * 5), ("bricks_settled", C.c_int64), ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64),
        ("nodes_double", C.c_int64), ("centres_double", C.c_int64), ("newton_solves", C.c_int64),
        ("newton_evals", C.c_int64),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "census"}
        d["census"] = list(self.census)
        return d


class IcamBatchLevel(C.Structure):
    _fields_ = [("h", C.c_double), ("lo", C.c_double * 3), ("nb", C.c_int64 * 3), ("clamp", C.c_double),
                ("origin", C.c_double * 3), ("has_origin", C.c_int32), ("pad", C.c_int32)]


class IcamBatchPart(C.Structure):
    _fields_ = [("d_map", C.c_void_p), ("d_atlas", C.c_void_p), ("n_slots", C.c_size_t), ("bricks_read", C.c_int64)]


class IcamBatchStats(C.Structure):
    _fields_ = [("parts", C.c_int64), ("boxes_read", C.c_int64), ("bricks_read", C.c_int64),
                ("bricks_words", C.c_int64), ("nodes_exact", C.c_int64), ("nodes_undecided", C.c_int64),
                ("kernel_launches", C.c_int64), ("warps", C.c_int32), ("graph_replayed", C.c_int32),
                ("tune_ms", C.c_double * 3), ("ms_decide", C.c_double), ("ms_bricks", C.c_double),
                ("bricks_settled", C.c_int64)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "tune_ms"}
        d["tune_ms"] = list(self.tune_ms)
        return d


def lib():
    """The CUDA library, loaded once (raises when it is missing: build it with
    ``python -m implicitcam_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"{LIB} is missing: build it with `python -m implicitcam_b200.build`")
        L = C.CDLL(LIB)
        vp, sz = C.c_void_p, C.c_size_t
        L.icam_pack_create.restype = C.c_int
        L.icam_pack_create.argtypes = [vp, vp, C.POINTER(vp), C.c_char_p, sz]
        L.icam_pack_destroy.argtypes = [vp]
        L.icam_pack_info.argtypes = [vp, vp]
        L.icam_last_error.restype = C.c_char_p
        L.icam_last_error.argtypes = [vp]
        L.icam_points.argtypes = [vp, vp, sz, C.c_double, C.c_int, C.c_int, vp, vp]
        L.icam_bricks.argtypes = [vp, vp, sz, C.c_double, C.c_double, C.c_int, vp, vp]
        L.icam_bake_level.argtypes = [vp, C.c_double, vp, vp, C.c_double, vp, C.c_int, vp, vp, sz, C.POINTER(sz), vp]
        L.icam_level_read.argtypes = [vp, vp, sz, vp, sz]
        L.icam_decide_level.argtypes = [vp, C.c_double, vp, vp, C.c_double, vp, C.c_int, vp, vp, vp, sz,
                                        C.POINTER(sz), vp]
        L.icam_bake_level_device.argtypes = [vp, C.c_double, vp, vp, C.c_double, vp, C.c_int, C.POINTER(vp),
                                             C.POINTER(vp), C.POINTER(sz), vp]
        L.icam_list.argtypes = [vp, vp, C.c_double, C.c_double, vp, sz, C.POINTER(sz)]
        L.icam_warm.argtypes = [vp, C.c_double]
        L.icam_pack_stream.restype = vp
        L.icam_pack_stream.argtypes = [vp]
        L.icam_probe_fma.argtypes = [vp, C.c_int, C.POINTER(C.c_double)]
        u64, d = C.c_uint64, C.c_double
        L.icam_seednet_samples.argtypes = [vp, sz, u64, d, vp, vp]
        L.icam_seednet_params.argtypes = [vp, vp, vp, C.POINTER(sz)]
        L.icam_seednet_grad.argtypes = [vp, vp, vp, sz, vp, C.POINTER(d)]
        L.icam_seednet_train.argtypes = [vp, C.c_int64, C.c_int64, u64, d, d, vp]
        L.icam_seednet_ab.argtypes = [vp, sz, u64, d, vp]
        L.icam_pack_box.argtypes = [vp, vp, vp]
        L.icam_batch_create.argtypes = [vp, sz, C.POINTER(vp), C.c_char_p, sz]
        L.icam_batch_destroy.argtypes = [vp]
        L.icam_batch_bake.argtypes = [vp, vp, C.c_int, vp, vp]
        L.icam_batch_read.argtypes = [vp, vp, sz, vp, vp, sz]
        L.icam_batch_last_error.restype = C.c_char_p
        L.icam_batch_last_error.argtypes = [vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class IcamError(RuntimeError):
    pass


class PartGpu:
    """The part packed on one GPU (PartGpu::new, partgpu.rs:132)."""

    def __init__(self, solid, need: float = 2.0, device: int = 0):
        desc = solid.desc() if hasattr(solid, "desc") else solid
        assert isinstance(desc, IcamSolidDesc)
        self._solid = solid
        self._desc = desc
        self.device = device
        opt = IcamPackOptions(device, need)
        h = C.c_void_p()
        err = C.create_string_buffer(1024)
        rc = lib().icam_pack_create(C.byref(desc), C.byref(opt), C.byref(h), err, 1024)
        if rc != 0:
            raise IcamError(f"icam_pack_create: {rc}: {err.value.decode()}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().icam_pack_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except TypeError:  # interpreter shutdown: the module's globals are gone
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise IcamError(f"{what}: {rc}: {lib().icam_last_error(self.h).decode()}")

    def box(self):
        """The solid's box (lo, hi)."""
        lo, hi = np.zeros(3), np.zeros(3)
        self._check(lib().icam_pack_box(self.h, _p(lo), _p(hi)), "icam_pack_box")
        return lo, hi

    def info(self):
        c = np.zeros(7, np.int64)
        lib().icam_pack_info(self.h, _p(c))
        return dict(zip(["faces", "edges", "verts", "subs", "pieces", "cells", "bvh"], c.tolist()))

    def points(self, xyz, clamp=np.inf, capped=False, precision=FP64):
        """Signed distance of points: (value, flag) with flag 0 exact, 1 a bound past
        the clamp, 2 undecided (PartGpu::points_scatter(_capped), partgpu.rs:243-264)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        n = len(xyz)
        v = np.zeros(n)
        f = np.zeros(n, np.int8)
        self._check(lib().icam_points(self.h, _p(xyz), n, float(clamp), int(capped), precision, _p(v), _p(f)),
                    "icam_points")
        return v, f

    def bricks(self, firsts, h, clamp, precision=FP64):
        """Every node of each brick (PartGpu::bricks, partgpu.rs:227): float pairs
        (value, flag) as the reference returns them, and the double values."""
        firsts = np.ascontiguousarray(firsts, dtype=np.float64).reshape(-1, 3)
        n = len(firsts)
        vals = np.zeros((n, 729, 2), np.float32)
        d = np.zeros((n, 729))
        self._check(lib().icam_bricks(self.h, _p(firsts), n, float(h), float(clamp), precision, _p(vals), _p(d)),
                    "icam_bricks")
        return vals, d

    def level(self, h, lo, nb, clamp=None, origin=None, precision=FP64, atlas=True):
        """One level of the brick cache (PartCache::level, partcache.rs:433):
        (map, atlas (slots x 365 words), stats)."""
        lo = np.ascontiguousarray(lo, dtype=np.float64)
        nb = np.ascontiguousarray(nb, dtype=np.int64)
        clamp = h * np.sqrt(3.0) if clamp is None else clamp
        org = None if origin is None else np.ascontiguousarray(origin, dtype=np.float64)
        m = np.zeros(int(np.prod(nb)), np.uint32)
        ns = C.c_size_t()
        st = IcamBakeStats()
        # one bake for the map and the slot count, then the atlas sized to it read back
        self._check(lib().icam_bake_level(self.h, float(h), _p(lo), _p(nb), float(clamp), _p(org), precision, _p(m),
                                          None, 0, C.byref(ns), C.byref(st)), "icam_bake_level")
        if not atlas:
            return m, None, st.as_dict()
        a = np.zeros((ns.value, WORDS), np.uint32)
        self._check(lib().icam_level_read(self.h, None, 0, _p(a), a.size), "icam_level_read")
        return m, a, st.as_dict()

    def decide(self, h, lo, nb, clamp=None, origin=None, precision=FP64):
        """The level's box decision alone (PartCache::decide, partcache.rs:226-331):
        (map with READ at the bricks to read, their indices in brick order, their
        centres' distances, stats)."""
        lo = np.ascontiguousarray(lo, dtype=np.float64)
        nb = np.ascontiguousarray(nb, dtype=np.int64)
        clamp = h * np.sqrt(3.0) if clamp is None else clamp
        org = None if origin is None else np.ascontiguousarray(origin, dtype=np.float64)
        total = int(np.prod(nb))
        m = np.zeros(total, np.uint32)
        idx = np.zeros(total, np.int64)
        dc = np.zeros(total)
        n = C.c_size_t()
        st = IcamBakeStats()
        self._check(lib().icam_decide_level(self.h, float(h), _p(lo), _p(nb), float(clamp), _p(org), precision, _p(m),
                                            _p(idx), _p(dc), total, C.byref(n), C.byref(st)), "icam_decide_level")
        return m, idx[: n.value].copy(), dc[: n.value].copy(), st.as_dict()

    def level_read(self, map_entries, slots):
        """The last level baked on this pack, read back without baking again: (map, atlas)."""
        m = np.zeros(int(map_entries), np.uint32)
        a = np.zeros((int(slots), WORDS), np.uint32)
        self._check(lib().icam_level_read(self.h, _p(m), m.size, _p(a), a.size), "icam_level_read")
        return m, a

    def level_into(self, h, lo, nb, clamp, map_out, atlas_out, origin=None, precision=FP64):
        """The bake with its map and atlas written into caller buffers (numpy arrays or
        host torch tensors, pinned for fast copies): (slots, stats)."""
        lo = np.ascontiguousarray(lo, dtype=np.float64)
        nb = np.ascontiguousarray(nb, dtype=np.int64)
        org = None if origin is None else np.ascontiguousarray(origin, dtype=np.float64)

        def ptr(x):
            return C.c_void_p(x.data_ptr()) if hasattr(x, "data_ptr") else _p(x)

        def words(x):
            return x.numel() if hasattr(x, "numel") else x.size

        ns = C.c_size_t()
        st = IcamBakeStats()
        self._check(lib().icam_bake_level(self.h, float(h), _p(lo), _p(nb), float(clamp), _p(org), precision,
                                          ptr(map_out), ptr(atlas_out), words(atlas_out), C.byref(ns), C.byref(st)),
                    "icam_bake_level")
        return ns.value, st.as_dict()

    def level_torch(self, h, lo, nb, clamp=None, origin=None, precision=FP64):
        """The bake read into torch tensors on the pack's device (one bake, then one
        device-to-device read): (map int32 (the u32 entries), atlas int32 slots x 365)."""
        import torch

        lo = np.ascontiguousarray(lo, dtype=np.float64)
        nb = np.ascontiguousarray(nb, dtype=np.int64)
        clamp = h * np.sqrt(3.0) if clamp is None else clamp
        org = None if origin is None else np.ascontiguousarray(origin, dtype=np.float64)
        ns = C.c_size_t()
        st = IcamBakeStats()
        self._check(lib().icam_bake_level(self.h, float(h), _p(lo), _p(nb), float(clamp), _p(org), precision, None,
                                          None, 0, C.byref(ns), C.byref(st)), "icam_bake_level")
        dev = torch.device("cuda", self.device)
        m = torch.empty(int(np.prod(nb)), dtype=torch.int32, device=dev)
        a = torch.empty((ns.value, WORDS), dtype=torch.int32, device=dev)
        self._check(lib().icam_level_read(self.h, C.c_void_p(m.data_ptr()), m.numel(),
                                          C.c_void_p(a.data_ptr()) if ns.value else None, a.numel()),
                    "icam_level_read")
        return m, a

    def level_device(self, h, lo, nb, clamp=None, origin=None, precision=FP64):
        """The same bake with its results left on the device: (map ptr, atlas ptr, slots, stats)."""
        lo = np.ascontiguousarray(lo, dtype=np.float64)
        nb = np.ascontiguousarray(nb, dtype=np.int64)
        clamp = h * np.sqrt(3.0) if clamp is None else clamp
        org = None if origin is None else np.ascontiguousarray(origin, dtype=np.float64)
        dm, da, ns = C.c_void_p(), C.c_void_p(), C.c_size_t()
        st = IcamBakeStats()
        self._check(lib().icam_bake_level_device(self.h, float(h), _p(lo), _p(nb), float(clamp), _p(org), precision,
                                                 C.byref(dm), C.byref(da), C.byref(ns), C.byref(st)),
                    "icam_bake_level_device")
        return dm.value, da.value, ns.value, st.as_dict()

    def list(self, c, r, d):
        """Candidate codes (kind << 28 | index) within reach (PartGpu::list, partgpu.rs:220)."""
        c = np.ascontiguousarray(c, dtype=np.float64)
        out = np.zeros(1 << 16, np.uint32)
        n = C.c_size_t()
        self._check(lib().icam_list(self.h, _p(c), float(r), float(d), _p(out), out.size, C.byref(n)), "icam_list")
        return out[: min(n.value, out.size)].copy()

    def stream(self):
        """The pack's CUDA stream handle (cudaStream_t as an int)."""
        return lib().icam_pack_stream(self.h)

    def probe_fma(self, precision=FP64):
        """Measured FMA throughput of the device (FLOP/s) in double or single precision."""
        f = C.c_double()
        self._check(lib().icam_probe_fma(self.h, precision, C.byref(f)), "icam_probe_fma")
        return f.value

    def warm(self, secs):
        self._check(lib().icam_warm(self.h, float(secs)), "icam_warm")

    # ---- the seed network (no counterpart in the reference; see include/icam_cuda.h)

    def seednet_samples(self, n, seed=0, need=2.0):
        """n training pairs from the exact evaluator: inputs (n x 32) and targets
        (n x 4: s, t, d / L, 1)."""
        x = np.zeros((n, 32), np.float32)
        y = np.zeros((n, 4), np.float32)
        self._check(lib().icam_seednet_samples(self.h, n, seed, float(need), _p(x), _p(y)), "icam_seednet_samples")
        return x, y

    def seednet_params(self, set_to=None):
        """The FP32 parameter vector (after setting it to `set_to` when given)."""
        n = C.c_size_t()
        lib().icam_seednet_params(self.h, None, None, C.byref(n))
        out = np.zeros(n.value, np.float32)
        src = None if set_to is None else np.ascontiguousarray(set_to, dtype=np.float32)
        self._check(lib().icam_seednet_params(self.h, _p(out), _p(src), C.byref(n)), "icam_seednet_params")
        return out

    def seednet_grad(self, x, y):
        """Gradient of the mean loss over pairs (x, y) at the current parameters, and the loss."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = np.zeros(len(self.seednet_params()), np.float32)
        loss = C.c_double()
        self._check(lib().icam_seednet_grad(self.h, _p(x), _p(y), len(x), _p(g), C.byref(loss)), "icam_seednet_grad")
        return g, loss.value

    def seednet_train(self, steps, batch=4096, seed=0, need=2.0, lr=1e-3):
        """Trains on fresh pairs; the loss of every step."""
        loss = np.zeros(max(steps, 1), np.float32)
        self._check(lib().icam_seednet_train(self.h, steps, batch, seed, float(need), float(lr), _p(loss)),
                    "icam_seednet_train")
        return loss[:steps]

    def seednet_ab(self, n, seed=1, need=2.0):
        """The net's Newton starts against the centre start on n fresh pairs."""
        st = np.zeros(8)
        self._check(lib().icam_seednet_ab(self.h, n, seed, float(need), _p(st)), "icam_seednet_ab")
        keys = ["pairs", "mean_iters_net", "mean_iters_centre", "p99_iters_net", "p99_iters_centre",
                "fallback_rate", "pairs_differing", "max_diff_over_L"]
        return dict(zip(keys, st.tolist()))


def unpack_atlas(atlas):
    """The i16 node values of each slot (729 a brick, x fastest)."""
    a = np.asarray(atlas, dtype=np.uint32).reshape(-1, WORDS)
    lo = (a & 0xFFFF).astype(np.uint16).view(np.int16)
    hi = (a >> 16).astype(np.uint16).view(np.int16)
    q = np.empty((len(a), 730), np.int16)
    q[:, 0::2] = lo
    q[:, 1::2] = hi
    return q[:, :729]


class Batch:
    """Many parts baked together (icam_batch_*, include/icam_cuda.h): all parts' box
    decisions in one launch a box size, all parts' bricks in one launch of the brick
    kernel, the rest replayed as a CUDA graph. A part may appear more than once (e.g. at
    two resolutions). No counterpart in the reference."""

    def __init__(self, parts):
        self.parts = list(parts)
        arr = (C.c_void_p * len(self.parts))(*[p.h for p in self.parts])
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        rc = lib().icam_batch_create(arr, len(self.parts), C.byref(h), err, 512)
        if rc != 0:
            raise IcamError(f"icam_batch_create: {rc}: {err.value.decode()}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().icam_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def bake(self, levels, precision=FP64, read=True):
        """levels: per part (h, lo, nb, clamp[, origin]). Returns the stats and, with
        read, every part's (map, atlas) in host memory."""
        n = len(self.parts)
        lv = (IcamBatchLevel * n)()
        for i, L in enumerate(levels):
            h, lo, nb, clamp = L[:4]
            origin = L[4] if len(L) > 4 else None
            lv[i].h, lv[i].clamp = float(h), float(clamp)
            for k in range(3):
                lv[i].lo[k], lv[i].nb[k] = float(lo[k]), int(nb[k])
                lv[i].origin[k] = float(origin[k]) if origin is not None else 0.0
            lv[i].has_origin = int(origin is not None)
        out = (IcamBatchPart * n)()
        st = IcamBatchStats()
        rc = lib().icam_batch_bake(self.h, lv, precision, out, C.byref(st))
        if rc != 0:
            raise IcamError(f"icam_batch_bake: {rc}: {lib().icam_batch_last_error(self.h).decode()}")
        res = []
        if read:
            for i, L in enumerate(levels):
                m = np.zeros(int(np.prod(L[2])), np.uint32)
                a = np.zeros(max(out[i].n_slots, 1) * WORDS, np.uint32)
                rc = lib().icam_batch_read(self.h, C.byref(out[i]), len(m), _p(m), _p(a), len(a))
                if rc != 0:
                    raise IcamError(f"icam_batch_read: {rc}: {lib().icam_batch_last_error(self.h).decode()}")
                res.append((m, a[: out[i].n_slots * WORDS].reshape(-1, WORDS)))
        return st.as_dict(), res
