"""Python binding of libfmmgpu.so (the C ABI in include/fmm_gpu.h).

`Context` mirrors the reference's update-method interface for the force
pass: `evaluate` is FMM::update (src/system_updaters/FMM.cpp:9-12) on plain
arrays, `direct` is NaiveUpdate::update (naive_update.cpp:9-35) in FP64,
`integrate` is QuadratureMethod::integrate (quadrature_method.hpp:24) with
the state kept on the GPU, and `tree` exports Tree::init_tree's structure
(tree.cpp:15-91).  Accelerations are G * grad exactly as
Particle::compute_new_accelaration stores them (particle.cpp:16-21).

The library must be built (`make -C nbody-fmm_b200`); there is no CPU
fallback: importing works without it, but creating a Context raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libfmmgpu.so")

FMM_OK = 0
FMM_ERR_INVALID_ARGUMENT = -1
FMM_ERR_CUDA = -2
FMM_ERR_OUT_OF_MEMORY = -3
FMM_ERR_NONFINITE_INPUT = -4
FMM_ERR_NONFINITE_OUTPUT = -5
FMM_ERR_UNSUPPORTED = -6
FMM_ERR_TIMEOUT = -7
FMM_ERR_NO_DEVICE = -8
FMM_ERR_TOO_LARGE = -10
FMM_ERR_IO = -11
FMM_NOALLOC_MAX_TARGETS = 262144

FMM_M2L_FP32 = 0
FMM_M2L_TC = 1
FMM_ORDER_FIXED = 0
FMM_ORDER_GEOMETRIC = 1
FMM_ORDER_LEARNED = 2
FMM_ORDER_NPARAM = 7312
FMM_ORDER_NFEAT = 32
FMM_ORDER_NOUT = 9
ORDER_MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "order_model.npy")
FMM_SOFT_PLUMMER = 0
FMM_SOFT_NAIVE_REF = 1
FMM_INT_SYMPLECTIC_EULER = 0
FMM_INT_RK4 = 1

# Every symbol include/fmm_gpu.h declares.
EXPORTED = (
    "fmm_strerror", "fmm_version", "fmm_config_default", "fmm_create", "fmm_destroy", "fmm_evaluate",
    "fmm_evaluate_device", "fmm_synchronize", "fmm_direct", "fmm_direct_device", "fmm_integrate",
    "fmm_tree_build", "fmm_tree_depth", "fmm_tree_level_size", "fmm_tree_level_keys", "fmm_tree_leaves",
    "fmm_tree_pairs", "fmm_tree_adaptive_flags", "fmm_last_stats", "fmm_launch_count", "fmm_direct_noalloc",
    "fmm_order_set_model",
    "fmm_order_get_model", "fmm_order_collect", "fmm_order_train", "fmm_order_forward_grad", "fmm_autotune",
    "fmm_evaluate_batched", "fmm_frames_open", "fmm_frames_write", "fmm_frames_write_device", "fmm_frames_flush",
    "fmm_frames_close", "fmm_integrate_frames",
)


class FmmConfig(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32), ("p", ctypes.c_int32), ("leaf_cap", ctypes.c_int32), ("m2l_mode", ctypes.c_int32),
        ("eps2", ctypes.c_double), ("G", ctypes.c_double), ("device", ctypes.c_int32),
        ("direct_max", ctypes.c_int32), ("order_mode", ctypes.c_int32), ("order_margin", ctypes.c_int32),
        ("order_tol", ctypes.c_float), ("judge_samples", ctypes.c_int32), ("judge_budget", ctypes.c_float),
        ("judge_every", ctypes.c_int32), ("adaptive_leaf", ctypes.c_int32), ("p2p_chunk", ctypes.c_int32),
        ("m2l_run", ctypes.c_int32),
    ]


class FmmStats(ctypes.Structure):
    _fields_ = [
        ("depth", ctypes.c_int32), ("n_levels", ctypes.c_int32), ("n_leaves", ctypes.c_int64),
        ("n_cells", ctypes.c_int64), ("m2l_pairs", ctypes.c_int64), ("p2p_pairs", ctypes.c_int64),
        ("ms_tree", ctypes.c_double), ("ms_upward", ctypes.c_double), ("ms_m2l", ctypes.c_double),
        ("ms_downward", ctypes.c_double), ("ms_p2p", ctypes.c_double), ("ms_total", ctypes.c_double),
        ("m2l_tiles", ctypes.c_int64), ("ms_far_direct", ctypes.c_double),
        ("far_direct_pairs", ctypes.c_int64), ("direct_max", ctypes.c_int64), ("judge_rel_l2", ctypes.c_double),
        ("order_fallbacks", ctypes.c_int64), ("m2l_width_sum", ctypes.c_int64), ("reserved", ctypes.c_double * 7),
    ]


class FmmTuneResult(ctypes.Structure):
    _fields_ = [("n_candidates", ctypes.c_int32), ("best", ctypes.c_int32), ("leaf_cap", ctypes.c_int32 * 16),
                ("direct_max", ctypes.c_int32 * 16), ("ms", ctypes.c_double * 16),
                ("adaptive_leaf", ctypes.c_int32 * 16), ("p2p_chunk", ctypes.c_int32 * 16),
                ("m2l_run", ctypes.c_int32 * 16)]


FMM_TUNE_LEAF = 1
FMM_TUNE_ADAPTIVE = 2
FMM_TUNE_KERNELS = 4


class FmmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} (code {code})")
        self.code = code


_d = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)
_u64 = ctypes.POINTER(ctypes.c_uint64)
_vp = ctypes.c_void_p
_lib = None


def load_library(path=LIB_PATH):
    """Loads libfmmgpu.so and declares its prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FmmError(FMM_ERR_NO_DEVICE, f"{path} is missing: build it with `make -C nbody-fmm_b200`")
    L = ctypes.CDLL(path)
    L.fmm_strerror.restype = ctypes.c_char_p
    L.fmm_strerror.argtypes = [ctypes.c_int]
    L.fmm_version.restype = ctypes.c_char_p
    L.fmm_config_default.argtypes = [ctypes.POINTER(FmmConfig)]
    L.fmm_create.argtypes = [ctypes.POINTER(FmmConfig), ctypes.POINTER(_vp)]
    L.fmm_destroy.argtypes = [_vp]
    L.fmm_evaluate.argtypes = [_vp, ctypes.c_int64, _d, _d, _d, _d]
    L.fmm_evaluate_device.argtypes = [_vp, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp]
    L.fmm_synchronize.argtypes = [_vp]
    L.fmm_direct.argtypes = [_vp, ctypes.c_int64, _d, _d, ctypes.c_int64, _i64, ctypes.c_int32, _d, _d]
    L.fmm_direct_device.argtypes = [_vp, ctypes.c_int64, _vp, _vp, ctypes.c_int64, _vp, ctypes.c_int32, _vp, _vp, _vp]
    L.fmm_integrate.argtypes = [_vp, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_int64, _d, _d, _d, _d]
    L.fmm_tree_build.argtypes = [_vp, ctypes.c_int64, _d]
    L.fmm_tree_depth.argtypes = [_vp, ctypes.POINTER(ctypes.c_int32)]
    L.fmm_tree_level_size.argtypes = [_vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]
    L.fmm_tree_level_keys.argtypes = [_vp, ctypes.c_int32, _u64]
    L.fmm_tree_leaves.argtypes = [_vp, _u64, _i64, _i64]
    L.fmm_tree_pairs.argtypes = [_vp, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64), _u64, _u64]
    L.fmm_tree_adaptive_flags.argtypes = [_vp, ctypes.c_int32, ctypes.c_void_p]
    L.fmm_last_stats.argtypes = [_vp, ctypes.POINTER(FmmStats)]
    L.fmm_launch_count.restype = ctypes.c_int64
    L.fmm_launch_count.argtypes = [_vp]
    L.fmm_direct_noalloc.argtypes = [ctypes.c_int32, ctypes.c_int64, _vp, _vp, ctypes.c_int64, _vp, ctypes.c_int32,
                                     ctypes.c_double, ctypes.c_double, _vp, _vp, _vp]
    _f = ctypes.POINTER(ctypes.c_float)
    L.fmm_order_set_model.argtypes = [_vp, _f, ctypes.c_int32]
    L.fmm_order_get_model.argtypes = [_vp, _f, ctypes.c_int32]
    L.fmm_order_collect.argtypes = [_vp, ctypes.c_int64, _vp, _vp, ctypes.c_int32, ctypes.c_uint64, _vp, _vp, _vp]
    L.fmm_order_train.argtypes = [_vp, _vp, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, _f]
    L.fmm_order_forward_grad.argtypes = [_vp, _vp, ctypes.c_int32, _vp, _vp, _vp, _vp, _vp]
    L.fmm_autotune.argtypes = [_vp, ctypes.c_int64, _vp, _vp, ctypes.c_int32, ctypes.POINTER(FmmTuneResult), _vp]
    L.fmm_evaluate_batched.argtypes = [_vp, ctypes.c_int32, _i64, _vp, _vp, _vp, _vp, ctypes.c_int32]
    L.fmm_frames_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(_vp)]
    L.fmm_frames_write.argtypes = [_vp, ctypes.c_int64, _d, _d, _d, _d, ctypes.c_int32, ctypes.c_double]
    L.fmm_frames_write_device.argtypes = [_vp, ctypes.c_int64, _vp, _vp, _vp, _vp, ctypes.c_int32, ctypes.c_double,
                                          _vp]
    L.fmm_frames_flush.argtypes = [_vp]
    L.fmm_frames_close.argtypes = [_vp]
    L.fmm_integrate_frames.argtypes = [_vp, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_int64, _d, _d,
                                       _d, _d, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double]
    _lib = L
    return L


def _check(rc):
    if rc != FMM_OK:
        raise FmmError(rc, _lib.fmm_strerror(rc).decode())


def _p(a, t=_d):
    return None if a is None else a.ctypes.data_as(t)


class Frames:
    """Frame output of a simulation loop (fmm_frames_*): per step the
    reference exporter's datasets (position, velocity, acceleration as
    n x 3 FP64, 2D padded with z = 0; weight as n) in `<dir>/<base>_<step:05>.bin`
    and the XDMF time-series index `<dir>/<base>.xmf`, rewritten per frame."""

    def __init__(self, directory, base="particles", dim=3):
        L = load_library()
        self._h = _vp()
        _check(L.fmm_frames_open(os.fsencode(directory), base.encode(), dim, ctypes.byref(self._h)))
        self.dim = dim

    def write(self, pos, vel, mass, step, time, acc=None):
        """A frame from host arrays (n x dim, n x dim, n; acc optional),
        written before the call returns."""
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        acc = None if acc is None else np.ascontiguousarray(acc, dtype=np.float64)
        _check(_lib.fmm_frames_write(self._h, len(mass), _p(pos), _p(vel), _p(acc), _p(mass), step, time))

    def write_device(self, n, pos_ptr, vel_ptr, mass_ptr, step, time, acc_ptr=None, stream=None):
        """A frame from device arrays: their copy is enqueued on `stream`
        (an int handle) and the file is written by a writer thread."""
        _check(_lib.fmm_frames_write_device(self._h, n, pos_ptr, vel_ptr, acc_ptr, mass_ptr, step, time, stream))

    def flush(self):
        _check(_lib.fmm_frames_flush(self._h))

    def close(self):
        if self._h:
            h, self._h = self._h, _vp()
            _check(_lib.fmm_frames_close(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def direct_noalloc(dim, n, pos_ptr, mass_ptr, acc_ptr, pot_ptr=None, ntargets=0, targets_ptr=None,
                   soft_mode=FMM_SOFT_PLUMMER, eps2=0.0, G=1.0, stream=None):
    """FP64 direct sum on the current GPU into caller-owned device buffers,
    without any device allocation and without a Context (fmm_direct_noalloc).
    For callers that cannot allocate device memory when they need forces; at
    most FMM_NOALLOC_MAX_TARGETS targets; concurrent calls on one GPU race
    on the library's fixed scratch.  Enqueued on `stream` (an int handle)."""
    L = load_library()
    _check(L.fmm_direct_noalloc(dim, n, pos_ptr, mass_ptr, ntargets, targets_ptr, soft_mode, eps2, G, acc_ptr,
                                pot_ptr, stream))


class Context:
    """One FMM force evaluator on one GPU (fmm_create / fmm_destroy)."""

    def __init__(self, dim=3, p=8, leaf_cap=64, m2l_mode=FMM_M2L_FP32, eps2=0.0, G=1.0, device=0, direct_max=-1,
                 order_mode=FMM_ORDER_FIXED, order_margin=1, order_tol=2e-6, judge_samples=0, judge_budget=1e-6,
                 judge_every=1, order_model=None, adaptive_leaf=0, p2p_chunk=0, m2l_run=0):
        L = load_library()
        cfg = FmmConfig()
        _check(L.fmm_config_default(ctypes.byref(cfg)))
        cfg.dim, cfg.p, cfg.leaf_cap, cfg.m2l_mode = dim, p, leaf_cap, m2l_mode
        cfg.eps2, cfg.G, cfg.device, cfg.direct_max = eps2, G, device, direct_max
        cfg.order_mode, cfg.order_margin = order_mode, order_margin
        cfg.order_tol, cfg.judge_samples, cfg.judge_budget = order_tol, judge_samples, judge_budget
        cfg.judge_every = judge_every
        cfg.adaptive_leaf = adaptive_leaf
        cfg.p2p_chunk, cfg.m2l_run = p2p_chunk, m2l_run
        h = _vp()
        _check(L.fmm_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.dim = dim
        self.cfg = cfg
        if order_model is None and order_mode == FMM_ORDER_LEARNED and os.path.exists(ORDER_MODEL_PATH):
            order_model = np.load(ORDER_MODEL_PATH)
        if order_model is not None:
            self.set_order_model(order_model)

    def close(self):
        if getattr(self, "_h", None):
            _lib.fmm_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _arrays(self, pos, mass):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        if pos.ndim != 2 or pos.shape[1] != self.dim or mass.shape != (pos.shape[0],):
            raise FmmError(FMM_ERR_INVALID_ARGUMENT, "pos must be (n, dim) and mass (n,)")
        return pos, mass

    def evaluate(self, pos, mass, want_pot=False, out=None, out_pot=None):
        """One force pass (host buffers): returns acc (n, dim) [, pot (n,)].
        `out` / `out_pot` may be preallocated (e.g. pinned) C-contiguous float64 arrays."""
        pos, mass = self._arrays(pos, mass)
        n = pos.shape[0]
        acc = out if out is not None else np.zeros((n, self.dim))
        if acc.shape != (n, self.dim) or acc.dtype != np.float64 or not acc.flags.c_contiguous:
            raise FmmError(FMM_ERR_INVALID_ARGUMENT, "out must be a C-contiguous (n, dim) float64 array")
        pot = (out_pot if out_pot is not None else np.zeros(n)) if want_pot else None
        _check(_lib.fmm_evaluate(self._h, n, _p(pos), _p(mass), _p(acc), _p(pot)))
        return (acc, pot) if want_pot else acc

    def evaluate_device(self, n, pos_ptr, mass_ptr, acc_ptr, pot_ptr=None, stream=None):
        """One force pass on device pointers (ints), enqueued on `stream`."""
        _check(_lib.fmm_evaluate_device(self._h, n, pos_ptr, mass_ptr, acc_ptr, pot_ptr, stream))

    def synchronize(self):
        _check(_lib.fmm_synchronize(self._h))

    def direct(self, pos, mass, targets=None, soft_mode=FMM_SOFT_PLUMMER, want_pot=False):
        """FP64 direct sum on the GPU (acc = G * grad) for `targets` (all if None)."""
        pos, mass = self._arrays(pos, mass)
        n = pos.shape[0]
        t = None if targets is None else np.ascontiguousarray(targets, dtype=np.int64)
        nt = n if t is None else len(t)
        acc = np.zeros((nt, self.dim))
        pot = np.zeros(nt) if want_pot else None
        _check(_lib.fmm_direct(self._h, n, _p(pos), _p(mass), nt, _p(t, _i64), soft_mode, _p(acc), _p(pot)))
        return (acc, pot) if want_pot else acc

    def direct_device(self, n, pos_ptr, mass_ptr, ntargets, targets_ptr, acc_ptr, pot_ptr=None,
                      soft_mode=FMM_SOFT_PLUMMER, stream=None):
        _check(_lib.fmm_direct_device(self._h, n, pos_ptr, mass_ptr, ntargets, targets_ptr, soft_mode, acc_ptr,
                                      pot_ptr, stream))

    def integrate(self, method, dt, steps, pos, vel, mass, frames=None, every=1, step0=0, t0=0.0):
        """Advances (pos, vel) by `steps` steps; returns new pos, vel and the
        last acc.  With `frames` (a Frames), a frame of the state is written
        before every `every`-th step (fmm_integrate_frames)."""
        pos, mass = self._arrays(pos, mass)
        pos = pos.copy()
        vel = np.array(vel, dtype=np.float64, order="C", copy=True)
        acc = np.zeros_like(pos)
        if frames is None:
            _check(_lib.fmm_integrate(self._h, method, dt, steps, pos.shape[0], _p(pos), _p(vel), _p(mass), _p(acc)))
        else:
            _check(_lib.fmm_integrate_frames(self._h, method, dt, steps, pos.shape[0], _p(pos), _p(vel), _p(mass),
                                             _p(acc), frames._h, every, step0, t0))
        return pos, vel, acc

    def tree(self, pos, with_pairs=True):
        """Builds the tree of `pos` and returns it in the oracle's dict layout."""
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        n = pos.shape[0]
        _check(_lib.fmm_tree_build(self._h, n, _p(pos)))
        D = ctypes.c_int32()
        _check(_lib.fmm_tree_depth(self._h, ctypes.byref(D)))
        D = D.value
        cnt = ctypes.c_int64()
        _check(_lib.fmm_tree_level_size(self._h, D, ctypes.byref(cnt)))
        nl = cnt.value
        keys = np.zeros(nl, np.uint64)
        start = np.zeros(nl + 1, np.int64)
        perm = np.zeros(n, np.int64)
        _check(_lib.fmm_tree_leaves(self._h, _p(keys, _u64), _p(start, _i64), _p(perm, _i64)))
        levels, pairs = [], []
        for d in range(D + 1):
            _check(_lib.fmm_tree_level_size(self._h, d, ctypes.byref(cnt)))
            k = np.zeros(cnt.value, np.uint64)
            _check(_lib.fmm_tree_level_keys(self._h, d, _p(k, _u64)))
            levels.append(k)
            pl = []
            if with_pairs:
                for kind in (0, 1):
                    c = ctypes.c_int64()
                    _check(_lib.fmm_tree_pairs(self._h, d, kind, ctypes.byref(c), None, None))
                    tk = np.zeros(max(c.value, 1), np.uint64)
                    sk = np.zeros(max(c.value, 1), np.uint64)
                    _check(_lib.fmm_tree_pairs(self._h, d, kind, ctypes.byref(c), _p(tk, _u64), _p(sk, _u64)))
                    pl.append((tk[: c.value], sk[: c.value]))
            pairs.append(pl)
        return dict(depth=D, leaf_keys=keys, leaf_start=start, perm=perm, level_keys=levels, pairs=pairs)

    def adaptive_flags(self, adaptive_leaf):
        """The adaptive-target flags of the tree last built by tree(), one
        uint8 array per level in the order of its level_keys (bit 0 target,
        bit 1 adaptive leaf; fmm_tree_adaptive_flags)."""
        sizes = []
        cnt = ctypes.c_int64()
        D = ctypes.c_int32()
        _check(_lib.fmm_tree_depth(self._h, ctypes.byref(D)))
        for d in range(D.value + 1):
            _check(_lib.fmm_tree_level_size(self._h, d, ctypes.byref(cnt)))
            sizes.append(cnt.value)
        flags = np.zeros(sum(sizes), np.uint8)
        _check(_lib.fmm_tree_adaptive_flags(self._h, adaptive_leaf, flags.ctypes.data_as(ctypes.c_void_p)))
        return np.split(flags, np.cumsum(sizes)[:-1])

    def stats(self):
        s = FmmStats()
        _check(_lib.fmm_last_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in FmmStats._fields_ if k != "reserved"}

    def launch_count(self):
        return int(_lib.fmm_launch_count(self._h))

    def evaluate_batched(self, offsets, pos_ptr, mass_ptr, acc_ptr, pot_ptr=None, workers=0):
        """Independent systems stored one after another in device arrays
        (fmm_evaluate_batched); offsets: nsys + 1 int64 values from 0."""
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        _check(_lib.fmm_evaluate_batched(self._h, len(offsets) - 1, _p(offsets, _i64), pos_ptr, mass_ptr, acc_ptr,
                                         pot_ptr, workers))

    def autotune(self, n, pos_ptr, mass_ptr, tune_leaf=False, stream=None, tune_adaptive=False,
                 tune_kernels=False):
        """Times candidate direct-pair thresholds (and leaf capacities,
        adaptive-target thresholds and kernel shapes) on the given system and
        keeps the fastest (fmm_autotune).  Returns the candidates as a list of
        dicts and the chosen one."""
        r = FmmTuneResult()
        flags = ((FMM_TUNE_LEAF if tune_leaf else 0) | (FMM_TUNE_ADAPTIVE if tune_adaptive else 0) |
                 (FMM_TUNE_KERNELS if tune_kernels else 0))
        _check(_lib.fmm_autotune(self._h, n, pos_ptr, mass_ptr, flags, ctypes.byref(r), stream))
        cands = [{"leaf_cap": r.leaf_cap[i], "direct_max": r.direct_max[i], "adaptive_leaf": r.adaptive_leaf[i],
                  "p2p_chunk": r.p2p_chunk[i], "m2l_run": r.m2l_run[i], "ms": r.ms[i]}
                 for i in range(r.n_candidates)]
        best = cands[r.best]
        self.cfg.leaf_cap, self.cfg.direct_max = best["leaf_cap"], best["direct_max"]
        self.cfg.adaptive_leaf = best["adaptive_leaf"]
        self.cfg.p2p_chunk, self.cfg.m2l_run = best["p2p_chunk"], best["m2l_run"]
        return cands, best

    # ---- learned pair orders
    def set_order_model(self, params):
        """Loads the order MLP (FMM_ORDER_NPARAM floats, fmm_order_set_model)."""
        params = np.ascontiguousarray(params, dtype=np.float32).ravel()
        _check(_lib.fmm_order_set_model(self._h, _p(params, ctypes.POINTER(ctypes.c_float)), params.size))

    def get_order_model(self):
        out = np.zeros(FMM_ORDER_NPARAM, np.float32)
        _check(_lib.fmm_order_get_model(self._h, _p(out, ctypes.POINTER(ctypes.c_float)), out.size))
        return out

    def order_collect(self, n, pos_ptr, mass_ptr, ntiles, seed, feat_ptr, labels_ptr, stream=None):
        """One fixed-order evaluation that writes the features and FP64
        truncation-error labels of ntiles sampled M2L tiles into device
        buffers (fmm_order_collect)."""
        _check(_lib.fmm_order_collect(self._h, n, pos_ptr, mass_ptr, ntiles, seed, feat_ptr, labels_ptr, stream))

    def order_train(self, feat_ptr, labels_ptr, n, epochs, batch=8192, lr=1e-3):
        """Trains the loaded model in place on device data; returns the mean
        loss of every epoch (fmm_order_train)."""
        loss = np.zeros(epochs, np.float32)
        _check(_lib.fmm_order_train(self._h, feat_ptr, labels_ptr, n, epochs, batch, lr,
                                    _p(loss, ctypes.POINTER(ctypes.c_float))))
        return loss


def order_forward_grad(feat_ptr, labels_ptr, n, params_ptr, pred_ptr, grad_ptr, loss_ptr, stream=None):
    """Predictions, mean squared error and its parameter gradient on device
    buffers (fmm_order_forward_grad)."""
    load_library()
    _check(_lib.fmm_order_forward_grad(feat_ptr, labels_ptr, n, params_ptr, pred_ptr, grad_ptr, loss_ptr, stream))


def order_init_params(seed=0):
    """He-initialised MLP parameters in the library's flat layout (the rows
    of W3 and b3 beyond the nine outputs are zero)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(FMM_ORDER_NPARAM, np.float32)
    nf, nh = FMM_ORDER_NFEAT, 64
    w1, b1 = 0, nh * nf
    w2, b2 = b1 + nh, b1 + nh + nh * nh
    w3, b3 = b2 + nh, b2 + nh + 16 * nh
    p[w1:b1] = rng.normal(0.0, np.sqrt(2.0 / nf), nh * nf)
    p[w2:b2] = rng.normal(0.0, np.sqrt(2.0 / nh), nh * nh)
    p[w3:w3 + FMM_ORDER_NOUT * nh] = rng.normal(0.0, np.sqrt(1.0 / nh), FMM_ORDER_NOUT * nh)
    return p
