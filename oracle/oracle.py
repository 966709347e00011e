"""ctypes bindings for the CPU checkers — TEST INFRASTRUCTURE ONLY.

`Oracle` wraps liboracle.so (the project's CPU restatement, fmm_oracle.c) and
`RefLib` wraps _ref/libref.so (the reference rezucch1/nbody-FMM compiled from
its own sources by oracle/Makefile).  Only tests/, the smoke entry and
bench.py's CPU-baseline leg import this module; the product never does.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")

_d = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)
_u64 = ctypes.POINTER(ctypes.c_uint64)
_u32 = ctypes.POINTER(ctypes.c_uint32)


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _f64(a, cols=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
        L = ctypes.CDLL(path)
        L.orc_tree_build.restype = ctypes.c_void_p
        L.orc_tree_build.argtypes = [ctypes.c_int, ctypes.c_int64, _d, ctypes.c_uint]
        L.orc_tree_free.argtypes = [ctypes.c_void_p]
        L.orc_tree_depth.argtypes = [ctypes.c_void_p]
        L.orc_tree_box.argtypes = [ctypes.c_void_p, _d, _d]
        L.orc_tree_level_size.restype = ctypes.c_int64
        L.orc_tree_level_size.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_tree_level_keys.restype = ctypes.c_int64
        L.orc_tree_level_keys.argtypes = [ctypes.c_void_p, ctypes.c_int, _u64]
        L.orc_tree_leaves.restype = ctypes.c_int64
        L.orc_tree_leaves.argtypes = [ctypes.c_void_p, _u64, _i64, _i64]
        L.orc_tree_npairs.restype = ctypes.c_int64
        L.orc_tree_npairs.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_tree_pairs.restype = ctypes.c_int64
        L.orc_tree_pairs.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _u64, _u64]
        L.orc_morton_encode.restype = ctypes.c_uint64
        L.orc_morton_encode.argtypes = [_u32, ctypes.c_int]
        L.orc_morton_decode.argtypes = [ctypes.c_uint64, ctypes.c_int, _u32]
        L.orc_direct.argtypes = [ctypes.c_int, ctypes.c_int64, _d, _d, ctypes.c_double, ctypes.c_int64, _i64, _d, _d]
        L.orc_naive_ref.argtypes = [ctypes.c_int, ctypes.c_int64, _d, _d, _d]
        L.orc_fmm.argtypes = [ctypes.c_int, ctypes.c_int64, _d, _d, ctypes.c_uint, ctypes.c_uint, ctypes.c_int, _d, _d]
        L.orc_fmm_ex.argtypes = [ctypes.c_int, ctypes.c_int64, _d, _d, ctypes.c_uint, ctypes.c_uint, ctypes.c_int,
                                 ctypes.c_double, ctypes.c_int64, _d, _d]
        L.orc_fmm_adaptive.argtypes = [ctypes.c_int, ctypes.c_int64, _d, _d, ctypes.c_uint, ctypes.c_uint,
                                       ctypes.c_uint, ctypes.c_double, ctypes.c_int64, ctypes.c_int64, _d, _d]
        L.orc_adaptive_flags.restype = ctypes.c_int64
        L.orc_adaptive_flags.argtypes = [ctypes.c_int, ctypes.c_int64, _d, ctypes.c_uint, ctypes.c_uint, ctypes.c_int64,
                                         ctypes.c_void_p]
        for f in ("orc_regular_scaled", "orc_irregular_scaled", "orc_regular_racah", "orc_irregular_racah"):
            getattr(L, f).argtypes = [ctypes.c_uint, _d, _d]
        L.orc_p2m_3d.argtypes = [ctypes.c_uint, ctypes.c_int64, _d, _d, _d, _d]
        self.L = L

    # ---- tree
    def tree(self, pos, threshold, with_pairs=True):
        pos = _f64(pos)
        n, dim = pos.shape
        h = self.L.orc_tree_build(dim, n, _p(pos, _d), threshold)
        if not h:
            raise ValueError("orc_tree_build rejected the input")
        try:
            D = self.L.orc_tree_depth(h)
            lo = np.zeros(3)
            hi = np.zeros(3)
            self.L.orc_tree_box(h, _p(lo, _d), _p(hi, _d))
            nl = self.L.orc_tree_level_size(h, D)
            keys = np.zeros(nl, np.uint64)
            start = np.zeros(nl + 1, np.int64)
            perm = np.zeros(n, np.int64)
            self.L.orc_tree_leaves(h, _p(keys, _u64), _p(start, _i64), _p(perm, _i64))
            levels = []
            pairs = []
            for d in range(D + 1):
                m = self.L.orc_tree_level_size(h, d)
                k = np.zeros(m, np.uint64)
                self.L.orc_tree_level_keys(h, d, _p(k, _u64))
                levels.append(k)
                pl = []
                for kind in ((0, 1) if with_pairs else ()):
                    c = self.L.orc_tree_npairs(h, d, kind)
                    tk = np.zeros(max(c, 1), np.uint64)
                    sk = np.zeros(max(c, 1), np.uint64)
                    self.L.orc_tree_pairs(h, d, kind, _p(tk, _u64), _p(sk, _u64))
                    pl.append((tk[:c], sk[:c]))
                pairs.append(pl)
            return dict(depth=D, lo=lo[:dim], hi=hi[:dim], leaf_keys=keys, leaf_start=start, perm=perm,
                        level_keys=levels, pairs=pairs)
        finally:
            self.L.orc_tree_free(h)

    def morton_encode(self, coords):
        c = np.ascontiguousarray(coords, dtype=np.uint32)
        return int(self.L.orc_morton_encode(_p(c, _u32), len(c)))

    def morton_decode(self, code, dim):
        c = np.zeros(3, np.uint32)
        self.L.orc_morton_decode(ctypes.c_uint64(code), dim, _p(c, _u32))
        return c[:dim]

    # ---- forces (grad = acceleration / G)
    def direct(self, pos, mass, eps2=0.0, targets=None, want_pot=False):
        pos = _f64(pos)
        mass = _f64(mass)
        n, dim = pos.shape
        t = None if targets is None else np.ascontiguousarray(targets, dtype=np.int64)
        nt = n if t is None else len(t)
        g = np.zeros((nt, dim))
        pot = np.zeros(nt) if want_pot else None
        self.L.orc_direct(dim, n, _p(pos, _d), _p(mass, _d), eps2, nt, _p(t, _i64), _p(g, _d), _p(pot, _d))
        return (g, pot) if want_pot else g

    def naive_ref(self, pos, mass):
        pos = _f64(pos)
        mass = _f64(mass)
        n, dim = pos.shape
        g = np.zeros((n, dim))
        self.L.orc_naive_ref(dim, n, _p(pos, _d), _p(mass, _d), _p(g, _d))
        return g

    def fmm(self, pos, mass, p, threshold, centre_mode=0, want_pot=False, eps2=0.0, direct_max=0):
        """FMM force pass (grad = acceleration / G).  direct_max > 0 sums
        interaction pairs with n_t * n_s <= direct_max directly."""
        pos = _f64(pos)
        mass = _f64(mass)
        n, dim = pos.shape
        g = np.zeros((n, dim))
        pot = np.zeros(n) if want_pot else None
        rc = self.L.orc_fmm_ex(dim, n, _p(pos, _d), _p(mass, _d), p, threshold, centre_mode, eps2, direct_max,
                               _p(g, _d), _p(pot, _d))
        if rc != 0:
            raise ValueError("orc_fmm failed")
        return (g, pot) if want_pot else g

    def fmm_adaptive(self, pos, mass, p, threshold, aleaf=None, want_pot=False, eps2=0.0, direct_max=0,
                     w_direct_max=0):
        """FMM with adaptive targets on the uniform tree (3D and 2D): targets stop at
        cells of at most `aleaf` (default: threshold) particles and sum their
        colleagues' particles directly, larger colleagues through their
        children's multipoles where far enough (orc_fmm_adaptive)."""
        pos = _f64(pos)
        mass = _f64(mass)
        n, dim = pos.shape
        g = np.zeros((n, dim))
        pot = np.zeros(n) if want_pot else None
        rc = self.L.orc_fmm_adaptive(dim, n, _p(pos, _d), _p(mass, _d), p, threshold,
                                     threshold if aleaf is None else aleaf, eps2, direct_max, w_direct_max,
                                     _p(g, _d), _p(pot, _d))
        if rc != 0:
            raise ValueError("orc_fmm_adaptive failed")
        return (g, pot) if want_pot else g

    def adaptive_flags(self, pos, threshold, aleaf):
        """orc_fmm_adaptive's per-cell flags, one uint8 array per level in
        the order of tree()['level_keys']: bit 0 active target, bit 1
        adaptive leaf (orc_adaptive_flags)."""
        pos = _f64(pos)
        n, dim = pos.shape
        total = self.L.orc_adaptive_flags(dim, n, _p(pos, _d), threshold, aleaf, 0, None)
        if total < 0:
            raise ValueError("orc_adaptive_flags rejected the input")
        flags = np.zeros(total, np.uint8)
        self.L.orc_adaptive_flags(dim, n, _p(pos, _d), threshold, aleaf, total, flags.ctypes.data_as(ctypes.c_void_p))
        sizes = [len(k) for k in self.tree(pos, threshold)["level_keys"]]
        return np.split(flags, np.cumsum(sizes)[:-1])

    # ---- harmonics
    def _harm(self, fn, p, r, size):
        out = np.zeros(size)
        r = np.ascontiguousarray(r, dtype=np.float64)
        getattr(self.L, fn)(p, _p(r, _d), _p(out, _d))
        return out

    def regular_scaled(self, p, r):
        o = self._harm("orc_regular_scaled", p, r, (p + 1) * (p + 2))
        return o[0::2] + 1j * o[1::2]

    def irregular_scaled(self, p, r):
        o = self._harm("orc_irregular_scaled", p, r, (p + 1) * (p + 2))
        return o[0::2] + 1j * o[1::2]

    def regular_racah(self, p, r):
        return self._harm("orc_regular_racah", p, r, (p + 1) ** 2)

    def irregular_racah(self, p, r):
        return self._harm("orc_irregular_racah", p, r, (p + 1) ** 2)

    def p2m_3d(self, p, pos, mass, centre):
        pos = _f64(pos)
        mass = _f64(mass)
        c = _f64(centre)
        out = np.zeros((p + 1) * (p + 2))
        self.L.orc_p2m_3d(p, len(mass), _p(pos, _d), _p(mass, _d), _p(c, _d), _p(out, _d))
        return out[0::2] + 1j * out[1::2]


class RefLib:
    """The reference implementation itself (built from its sources)."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference sources exist")
        L = ctypes.CDLL(path)
        L.ref_set_params.argtypes = [ctypes.c_uint, ctypes.c_uint]
        L.ref_grav_const.restype = ctypes.c_double
        for f in ("ref_fmm", "ref_naive"):
            getattr(L, f).argtypes = [ctypes.c_int, ctypes.c_int64, _d, _d, _d]
        L.ref_se_steps.argtypes = [ctypes.c_int, ctypes.c_int64, _d, _d, _d, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.ref_tree_build.argtypes = [ctypes.c_int, ctypes.c_int64, _d, _d]
        L.ref_tree_level_size.restype = ctypes.c_int64
        L.ref_tree_level_size.argtypes = [ctypes.c_int]
        L.ref_tree_leaves.restype = ctypes.c_int64
        L.ref_tree_leaves.argtypes = [_u64, _i64, _i64]
        L.ref_tree_level_keys.restype = ctypes.c_int64
        L.ref_tree_level_keys.argtypes = [ctypes.c_int, _u64]
        L.ref_tree_npairs.restype = ctypes.c_int64
        L.ref_tree_npairs.argtypes = [ctypes.c_int, ctypes.c_int]
        L.ref_tree_pairs.restype = ctypes.c_int64
        L.ref_tree_pairs.argtypes = [ctypes.c_int, ctypes.c_int, _u64, _u64]
        L.ref_p2m_3d.argtypes = [ctypes.c_uint, ctypes.c_int64, _d, _d, _d, _d]
        L.ref_regular_3d.argtypes = [ctypes.c_uint, _d, _d]
        L.ref_irregular_3d.argtypes = [ctypes.c_uint, _d, _d]
        self.L = L
        self.G = L.ref_grav_const()

    def fmm(self, pos, mass, p, threshold):
        """FMM::update; returns grad = acceleration / G."""
        pos = _f64(pos)
        mass = _f64(mass)
        n, dim = pos.shape
        acc = np.zeros((n, dim))
        self.L.ref_set_params(p, threshold)
        self.L.ref_fmm(dim, n, _p(pos, _d), _p(mass, _d), _p(acc, _d))
        return acc / self.G

    def naive(self, pos, mass):
        pos = _f64(pos)
        mass = _f64(mass)
        n, dim = pos.shape
        acc = np.zeros((n, dim))
        self.L.ref_naive(dim, n, _p(pos, _d), _p(mass, _d), _p(acc, _d))
        return acc / self.G

    def se_steps(self, pos, vel, mass, dt, steps, use_fmm, p=2, threshold=20):
        pos = np.array(pos, dtype=np.float64, order="C")
        vel = np.array(vel, dtype=np.float64, order="C")
        mass = _f64(mass)
        n, dim = pos.shape
        self.L.ref_set_params(p, threshold)
        self.L.ref_se_steps(dim, n, _p(pos, _d), _p(vel, _d), _p(mass, _d), dt, steps, int(use_fmm))
        return pos, vel

    def tree(self, pos, threshold):
        pos = _f64(pos)
        n, dim = pos.shape
        mass = np.ones(n)
        self.L.ref_set_params(2, threshold)
        D = self.L.ref_tree_build(dim, n, _p(pos, _d), _p(mass, _d))
        nl = self.L.ref_tree_level_size(D)
        keys = np.zeros(nl, np.uint64)
        start = np.zeros(nl + 1, np.int64)
        perm = np.zeros(n, np.int64)
        self.L.ref_tree_leaves(_p(keys, _u64), _p(start, _i64), _p(perm, _i64))
        levels, pairs = [], []
        for d in range(D + 1):
            m = self.L.ref_tree_level_size(d)
            k = np.zeros(m, np.uint64)
            self.L.ref_tree_level_keys(d, _p(k, _u64))
            levels.append(k)
            pl = []
            for kind in (0, 1):
                c = self.L.ref_tree_npairs(d, kind)
                tk = np.zeros(max(c, 1), np.uint64)
                sk = np.zeros(max(c, 1), np.uint64)
                self.L.ref_tree_pairs(d, kind, _p(tk, _u64), _p(sk, _u64))
                pl.append((tk[:c], sk[:c]))
            pairs.append(pl)
        self.L.ref_tree_free()
        return dict(depth=D, leaf_keys=keys, leaf_start=start, perm=perm, level_keys=levels, pairs=pairs)

    def p2m_3d(self, p, pos, mass, centre):
        pos = _f64(pos)
        mass = _f64(mass)
        c = _f64(centre)
        out = np.zeros(2 * p * p + 4 * p + 1)
        self.L.ref_p2m_3d(p, len(mass), _p(pos, _d), _p(mass, _d), _p(c, _d), _p(out, _d))
        return out

    def regular_3d(self, p, r):
        out = np.zeros((p + 1) ** 2)
        r = _f64(r)
        self.L.ref_regular_3d(p, _p(r, _d), _p(out, _d))
        return out

    def irregular_3d(self, p, r):
        out = np.zeros((p + 1) ** 2)
        r = _f64(r)
        self.L.ref_irregular_3d(p, _p(r, _d), _p(out, _d))
        return out


def glibc_rand_sequence(seed, count):
    """glibc srand(seed)/rand() values, as the reference's tests draw them."""
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(seed)
    libc.rand.restype = ctypes.c_int
    return np.array([libc.rand() for _ in range(count)], dtype=np.float64)


RAND_MAX = 2147483647
