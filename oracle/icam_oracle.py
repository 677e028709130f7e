"""ctypes binding of the f64 CPU oracle (liboracle.so, built by ``make`` here).

TEST INFRASTRUCTURE ONLY: the oracle is the checker the CUDA library is compared
against. Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` load it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

AIR = 0xFFFFFFFF
SOLID = 0xFFFFFFFE
READ = 0xFFFFFFF0

_lib = None


def build(quiet=True):
    subprocess.run(["make", "-C", HERE], check=True, capture_output=quiet)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        dp = C.POINTER(C.c_double)
        L.oracle_new.restype = C.c_void_p
        L.oracle_new.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_bbox.argtypes = [C.c_void_p, dp, dp]
        L.oracle_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.oracle_sdf.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_double, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.oracle_candidates.restype = C.c_int
        L.oracle_candidates.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_int, C.c_void_p]
        L.oracle_decide.restype = C.c_int64
        L.oracle_decide.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_int,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
        L.oracle_decide_rule.restype = C.c_int64
        L.oracle_decide_rule.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                         C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
        L.oracle_bricks.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_int,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    """The exact evaluator over a solid description (``solid.SolidBuilder``)."""

    def __init__(self, builder, threads=None):
        self._builder = builder
        self._desc = builder.desc()
        err = C.create_string_buffer(512)
        self.h = lib().oracle_new(C.byref(self._desc), err, 512)
        if not self.h:
            raise ValueError(err.value.decode())
        self.threads = threads or os.cpu_count() or 1

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_free(self.h)
            self.h = None

    def bbox(self):
        lo, hi = np.zeros(3), np.zeros(3)
        dp = C.POINTER(C.c_double)
        lib().oracle_bbox(self.h, lo.ctypes.data_as(dp), hi.ctypes.data_as(dp))
        return lo, hi

    def sdf(self, pts, bound=np.inf, threads=None):
        """(d, q, feature kind (0 face, 1 edge, 2 vertex), feature id, unsure, pops)."""
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        n = len(pts)
        d = np.zeros(n)
        q = np.zeros((n, 3))
        kind = np.zeros(n, np.int32)
        fid = np.zeros(n, np.int32)
        unsure = np.zeros(n, np.uint8)
        pops = np.zeros(n, np.int32)
        lib().oracle_sdf(self.h, _p(pts), n, float(bound), _p(d), _p(q), _p(kind), _p(fid), _p(unsure), _p(pops),
                         threads or self.threads)
        return d, q, kind, fid, unsure.astype(bool), pops

    def candidates(self, c, r, d):
        c = np.ascontiguousarray(c, dtype=np.float64)
        out = np.zeros(4096, np.int32)
        kinds = np.zeros(4096, np.int32)
        n = lib().oracle_candidates(self.h, _p(c), float(r), float(d), _p(out), 4096, _p(kinds))
        return out[:n].copy(), kinds[:n].copy()

    def decide(self, h, lo, nb, clamp, origin=None, threads=None, tight=False):
        """The level's brick map and the bricks to read (partcache.rs:226-331).

        tight=True bounds each box by its own nodes' half diagonal rather than that of
        the box grown by the clamp (the rule the library's bakes use)."""
        lo = np.ascontiguousarray(lo, dtype=np.float64)
        nb = np.ascontiguousarray(nb, dtype=np.int64)
        origin = lo + h if origin is None else np.ascontiguousarray(origin, dtype=np.float64)
        total = int(np.prod(nb))
        m = np.zeros(total, np.uint32)
        cap = total
        idx = np.zeros(cap, np.int64)
        dc = np.zeros(cap)
        n = lib().oracle_decide_rule(self.h, float(h), _p(lo), _p(nb), float(clamp), _p(origin),
                                     threads or self.threads, int(bool(tight)), _p(m), _p(idx), _p(dc), cap)
        return m, idx[:n].copy(), dc[:n].copy()

    def bricks(self, firsts, h, clamp, threads=None):
        """exact_brick for each first node: (values before quantisation, i16 values,
        packed kind (0 words, 1 air, 2 solid), words)."""
        firsts = np.ascontiguousarray(firsts, dtype=np.float64).reshape(-1, 3)
        n = len(firsts)
        f = np.zeros((n, 729))
        q = np.zeros((n, 729), np.int16)
        kind = np.zeros(n, np.int32)
        words = np.zeros((n, 365), np.uint32)
        lib().oracle_bricks(self.h, _p(firsts), n, float(h), float(clamp), threads or self.threads, _p(f), _p(q),
                            _p(kind), _p(words))
        return f, q, kind, words
