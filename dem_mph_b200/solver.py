"""Python binding of libdmph.so through its C ABI (include/dmph.h).

The library is loaded from this package directory (built in-tree by
dem_mph_b200.build); there is no fallback: if it is missing or no CUDA device
is present the calls fail loudly.
"""
import ctypes as C
import os
import struct

import numpy as np

from . import abi
from .abi import Params, Info, FIELDS

CHECKPOINT_USER_MAX = 4096  # DMPH_CHECKPOINT_USER_MAX

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdmph.so")

_lib = None


def lib():
    """Load libdmph.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("dem_mph_b200/libdmph.so is not built: run python -m dem_mph_b200.build")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.dmph_params_default.argtypes = [vp]
        L.dmph_read_data_file.argtypes = [C.c_char_p, vp]
        L.dmph_read_grid_file.argtypes = [C.c_char_p, vp, C.POINTER(C.c_int), vp, vp, vp]
        L.dmph_write_prof_file.argtypes = [C.c_char_p, vp, C.c_int, vp, vp, vp]
        L.dmph_io_last_message.restype = C.c_char_p
        L.dmph_create.argtypes = [vp, C.c_int, vp, vp, vp, C.POINTER(vp)]
        L.dmph_step.argtypes = [vp, C.c_int]
        L.dmph_step_timed.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
        L.dmph_get_state.argtypes = [vp, vp, vp, vp, vp]
        L.dmph_step_begin.argtypes = [vp, C.POINTER(C.c_double)]
        L.dmph_step_finish.argtypes = [vp, C.c_int]
        L.dmph_get_rows.argtypes = [vp, C.c_int, vp, vp, vp]
        L.dmph_set_rows.argtypes = [vp, C.c_int, vp, vp, vp]
        L.dmph_set_state.argtypes = [vp, vp, vp]
        L.dmph_get_field.argtypes = [vp, C.c_int, vp]
        L.dmph_get_info.argtypes = [vp, vp]
        L.dmph_get_neighbor_list.argtypes = [vp, vp, vp, C.c_int64]
        L.dmph_get_global_sums.argtypes = [vp, vp]
        L.dmph_get_list_stats.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
        L.dmph_set_bodies.argtypes = [vp, C.c_int, vp, vp]
        L.dmph_get_rebuild_stats.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.dmph_checkpoint_write.argtypes = [vp, C.c_char_p, vp, C.c_int]
        L.dmph_checkpoint_open.argtypes = [C.c_char_p, C.POINTER(vp), vp, C.c_int, C.POINTER(C.c_int)]
        L.dmph_get_bodies.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
        L.dmph_set_profiling.argtypes = [vp, C.c_int]
        L.dmph_set_graph.argtypes = [vp, C.c_int]
        L.dmph_set_pair_mode.argtypes = [vp, C.c_int]
        L.dmph_get_phase_times.argtypes = [vp, vp, vp, C.c_int]
        L.dmph_autotune.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), vp, vp]
        L.dmph_set_variants.argtypes = [vp, C.c_int, C.c_int]
        L.dmph_autotune_list_build.argtypes = [vp, C.c_int, C.POINTER(C.c_int), vp]
        L.dmph_ensemble_create.argtypes = [vp, C.c_int, C.POINTER(vp)]
        L.dmph_ensemble_step.argtypes = [vp, C.c_int]
        L.dmph_ensemble_step_timed.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
        L.dmph_ensemble_autotune.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), vp, vp]
        L.dmph_ensemble_set_graph.argtypes = [vp, C.c_int]
        L.dmph_ensemble_info.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.dmph_ensemble_set_profiling.argtypes = [vp, C.c_int]
        L.dmph_ensemble_get_phase_times.argtypes = [vp, vp, vp, C.c_int]
        L.dmph_ensemble_last_error.argtypes = [vp]
        L.dmph_ensemble_last_error.restype = C.c_char_p
        L.dmph_ensemble_destroy.argtypes = [vp]
        L.dmph_surrogate_params_default.argtypes = [vp]
        L.dmph_surrogate_enable.argtypes = [vp, vp]
        L.dmph_surrogate_collect.argtypes = [vp, C.c_int]
        L.dmph_surrogate_train.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
        L.dmph_surrogate_advance.argtypes = [vp, C.c_int]
        L.dmph_surrogate_get_stats.argtypes = [vp, vp]
        L.dmph_surrogate_get_weights.argtypes = [vp, vp, C.c_int]
        L.dmph_surrogate_set_weights.argtypes = [vp, vp, C.c_int]
        L.dmph_mlp_forward.argtypes = [vp, vp, C.c_int, vp]
        L.dmph_mlp_forward_layers.argtypes = [vp, vp, C.c_int, vp]
        L.dmph_surrogate_get_samples.argtypes = [vp, vp, vp, C.c_int, C.POINTER(C.c_int)]
        L.dmph_surrogate_add_samples.argtypes = [vp, vp, vp, C.c_int]
        L.dmph_mlp_forward_timed.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float)]
        L.dmph_mlp_gradient.argtypes = [vp, vp, vp, C.c_int, vp, C.POINTER(C.c_float)]
        L.dmph_surrogate_features.argtypes = [vp, vp, C.POINTER(C.c_int)]
        L.dmph_write_bodies_file.argtypes = [C.c_char_p, C.c_int, C.c_int, vp, vp]
        L.dmph_read_bodies_file.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), vp, vp]
        L.dmph_bodies_from_contacts.argtypes = [vp, C.c_int, vp, vp, vp, C.POINTER(C.c_int), vp, C.c_int]
        L.dmph_bodies_last_message.restype = C.c_char_p
        L.dmph_destroy.argtypes = [vp]
        L.dmph_last_error.argtypes = [vp]
        L.dmph_last_error.restype = C.c_char_p
        L.dmph_version.restype = C.c_char_p
        _lib = L
    return _lib


def write_bodies(path, body_of_row, body_density):
    """Write a body sidecar file (dmph_write_bodies_file)."""
    b = np.ascontiguousarray(body_of_row, dtype=np.int32)
    rho = np.ascontiguousarray(body_density, dtype=np.float64)
    rc = lib().dmph_write_bodies_file(path.encode(), len(rho), len(b), _ptr(b), _ptr(rho))
    if rc != 0:
        raise DmphError(rc, lib().dmph_bodies_last_message().decode())


def read_bodies(path):
    """(body_of_row, body_density) of a body sidecar file (dmph_read_bodies_file)."""
    L = lib()
    nb, nr = C.c_int(), C.c_int()
    rc = L.dmph_read_bodies_file(path.encode(), C.byref(nb), C.byref(nr), None, None)
    if rc != 0:
        raise DmphError(rc, L.dmph_bodies_last_message().decode())
    b = np.empty(nr.value, np.int32)
    rho = np.empty(nb.value, np.float64)
    rc = L.dmph_read_bodies_file(path.encode(), C.byref(nb), C.byref(nr), _ptr(b), _ptr(rho))
    if rc != 0:
        raise DmphError(rc, L.dmph_bodies_last_message().decode())
    return b, rho


def bodies_from_contacts(params, typ, x):
    """(body_of_row, body_density): the solid particles connected by contact
    at 1.01 dx, numbered by first row (dmph_bodies_from_contacts)."""
    t = np.ascontiguousarray(typ, dtype=np.int32)
    xx = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
    b = np.empty(len(t), np.int32)
    rho = np.empty(len(t), np.float64)
    nb = C.c_int()
    rc = lib().dmph_bodies_from_contacts(C.byref(params), len(t), _ptr(t), _ptr(xx), _ptr(b), C.byref(nb),
                                         _ptr(rho), len(t))
    if rc != 0:
        raise DmphError(rc, lib().dmph_bodies_last_message().decode())
    return b, rho[:nb.value].copy()


PASS_VARIANTS = 5  # DMPH_PASS_VARIANTS (stencil passes)
LIST_VARIANTS = 4  # DMPH_LIST_VARIANTS (Verlet-list passes, the FP32 default)
BUILD_VARIANTS = 3  # DMPH_BUILD_VARIANTS (FP32 list build)


class DmphError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("dmph error %d: %s" % (code, msg))
        self.code = code


def _ptr(a):
    return a.ctypes.data if a is not None else None


class Solver:
    """One solver context on the current CUDA device."""

    def __init__(self, params, typ, x, v):
        L = lib()
        self.params = params.copy()
        self._typ = np.ascontiguousarray(typ, dtype=np.int32)
        xx = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        vv = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
        self.n = len(self._typ)
        h = C.c_void_p()
        rc = L.dmph_create(C.byref(self.params), self.n, _ptr(self._typ), _ptr(xx), _ptr(vv), C.byref(h))
        if rc != 0:
            raise DmphError(rc, L.dmph_last_error(None).decode())
        self._h = h

    def _check(self, rc):
        if rc != 0:
            raise DmphError(rc, lib().dmph_last_error(self._h).decode())

    def checkpoint(self, path, user=b""):
        """write a checkpoint for an exact resume (dmph_checkpoint_write);
        `user`: up to CHECKPOINT_USER_MAX bytes of the caller's own"""
        u = bytes(user)
        self._check(lib().dmph_checkpoint_write(self._h, os.fsencode(path), u if u else None, len(u)))

    @classmethod
    def open_checkpoint(cls, path):
        """(Solver, user bytes) from a checkpoint file (dmph_checkpoint_open):
        stepping it gives the bits the writing context would have given"""
        L = lib()
        h = C.c_void_p()
        ubuf = C.create_string_buffer(CHECKPOINT_USER_MAX)
        nu = C.c_int()
        rc = L.dmph_checkpoint_open(os.fsencode(path), C.byref(h), ubuf, CHECKPOINT_USER_MAX, C.byref(nu))
        if rc != 0:
            raise DmphError(rc, L.dmph_last_error(None).decode())
        self = cls.__new__(cls)
        self._h = h
        # the creation parameters and the types by row, from the file's head
        with open(path, "rb") as f:
            head = f.read(40)
            pbytes, hbytes = struct.unpack_from("<II", head, 12)
            nrows, nbodies, _, ubytes = struct.unpack_from("<iiii", head, 24)
            self.params = Params.from_buffer_copy(f.read(pbytes))
            f.seek(hbytes + ubytes, 1)
            self._typ = np.frombuffer(f.read(4 * nrows), np.int32).copy()
        self.n = nrows
        if nbodies > 0:
            self.nbodies = nbodies
        return self, ubuf.raw[:nu.value]

    def step(self, n=1):
        self._check(lib().dmph_step(self._h, n))

    def step_timed(self, n=1):
        ms = C.c_float()
        self._check(lib().dmph_step_timed(self._h, n, C.byref(ms)))
        return ms.value

    def step_begin(self):
        """drift part of one step; the largest squared displacement since the
        last rebuild (dmph_step_begin)"""
        m2 = C.c_double()
        self._check(lib().dmph_step_begin(self._h, C.byref(m2)))
        return m2.value

    def step_finish(self, rebuild):
        self._check(lib().dmph_step_finish(self._h, 1 if rebuild else 0))

    def get_rows(self, rows):
        """(x[k,3], v[k,3]) of input rows"""
        r = np.ascontiguousarray(rows, dtype=np.int32)
        x = np.empty((len(r), 3))
        v = np.empty((len(r), 3))
        self._check(lib().dmph_get_rows(self._h, len(r), _ptr(r), _ptr(x), _ptr(v)))
        return x, v

    def set_rows(self, rows, x, v):
        r = np.ascontiguousarray(rows, dtype=np.int32)
        xx = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        vv = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
        self._check(lib().dmph_set_rows(self._h, len(r), _ptr(r), _ptr(xx), _ptr(vv)))

    def state(self, out=None):
        """(type, x[N,3], v[N,3], orig_id) in the current sorted order.  `out`
        may give the four arrays to fill (e.g. page-locked host buffers, which
        the copies then reach at full link speed)."""
        if out is None:
            out = (np.empty(self.n, np.int32), np.empty((self.n, 3), np.float64),
                   np.empty((self.n, 3), np.float64), np.empty(self.n, np.int32))
        t, x, v, o = out
        for a, dt, shape in ((t, np.int32, (self.n,)), (x, np.float64, (self.n, 3)),
                             (v, np.float64, (self.n, 3)), (o, np.int32, (self.n,))):
            if a.dtype != dt or a.shape != shape or not a.flags.c_contiguous:
                raise ValueError("state(out=...) wants C-contiguous %s arrays of shape %s" % (np.dtype(dt), shape))
        self._check(lib().dmph_get_state(self._h, _ptr(t), _ptr(x), _ptr(v), _ptr(o)))
        return t, x, v, o

    def set_state(self, x=None, v=None):
        xx = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
        vv = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        self._check(lib().dmph_set_state(self._h, _ptr(xx), _ptr(vv)))

    def field(self, name):
        fid, dt, comps = FIELDS[name]
        out = np.empty(self.n * comps, dtype=dt)
        self._check(lib().dmph_get_field(self._h, fid, _ptr(out)))
        return out.reshape(-1, 3) if comps == 3 else out

    def info(self):
        inf = Info()
        self._check(lib().dmph_get_info(self._h, C.byref(inf)))
        return inf

    def rebuild_stats(self):
        """(rebuild triggers, full rebuilds with cell sort and lists) since
        creation (dmph_get_rebuild_stats; equal without list reuse)"""
        a, b = C.c_int64(), C.c_int64()
        self._check(lib().dmph_get_rebuild_stats(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def neighbor_list(self):
        ptr = np.empty(self.n + 1, np.int64)
        self._check(lib().dmph_get_neighbor_list(self._h, _ptr(ptr), None, 0))
        ind = np.empty(max(int(ptr[-1]), 1), np.int32)
        self._check(lib().dmph_get_neighbor_list(self._h, _ptr(ptr), _ptr(ind), int(ptr[-1])))
        return ptr, ind[:int(ptr[-1])]

    def global_sums(self):
        """FP64 sums over fluid and debris (dmph_get_global_sums): dict with
        mass, momentum (3), kinetic and potential energy"""
        out = np.zeros(6)
        self._check(lib().dmph_get_global_sums(self._h, _ptr(out)))
        return {"mass": out[0], "momentum": out[1:4].copy(), "kinetic": out[4], "potential": out[5]}

    def list_stats(self, with_overflow=False):
        """(entries walked by pass A, entries walked by pass B) of the current
        Verlet lists (dmph_get_list_stats), plus the overflow flag when asked;
        zeros in stencil mode"""
        a, b, o = C.c_int64(0), C.c_int64(0), C.c_int32(0)
        self._check(lib().dmph_get_list_stats(self._h, C.byref(a), C.byref(b), C.byref(o)))
        return (a.value, b.value, bool(o.value)) if with_overflow else (a.value, b.value)

    def set_bodies(self, body_of_row, body_density):
        """Make debris bodies rigid (see dmph_set_bodies): body_of_row[r] is the
        body of input row r (-1 none), body_density[b] its density."""
        b = np.ascontiguousarray(body_of_row, dtype=np.int32)
        rho = np.ascontiguousarray(body_density, dtype=np.float64)
        self._check(lib().dmph_set_bodies(self._h, len(rho), _ptr(b), _ptr(rho)))
        self.nbodies = len(rho)

    def bodies(self):
        """dict of body arrays: X, V, L (B,3), q (B,4), M (B,), F, T (B,3)"""
        B = getattr(self, "nbodies", 0)
        out = {k: np.zeros((B, 3)) for k in ("X", "V", "L", "F", "T")}
        out["q"] = np.zeros((B, 4))
        out["M"] = np.zeros(B)
        self._check(lib().dmph_get_bodies(self._h, _ptr(out["X"]), _ptr(out["V"]), _ptr(out["q"]), _ptr(out["L"]),
                                          _ptr(out["M"]), _ptr(out["F"]), _ptr(out["T"])))
        return out

    PHASES = ("drift", "rebuild", "pass_a", "pass_b", "dem", "bodies", "list_build")

    def set_pair_mode(self, mode):
        """"stencil" or "list" (dmph_set_pair_mode; FP32 split build)"""
        self._check(lib().dmph_set_pair_mode(self._h, {"stencil": 0, "list": 1}[mode]))

    def set_graph(self, on=True):
        """replay each step as one CUDA graph (see dmph_set_graph)"""
        self._check(lib().dmph_set_graph(self._h, 1 if on else 0))

    def autotune(self):
        """choose the fastest launch variants of the FP32 pair passes on the
        current state (dmph_autotune); returns (variant_a, variant_b, ms_a, ms_b)"""
        a, b = C.c_int(), C.c_int()
        ma = np.zeros(PASS_VARIANTS, np.float32)
        mb = np.zeros(PASS_VARIANTS, np.float32)
        self._check(lib().dmph_autotune(self._h, C.byref(a), C.byref(b), _ptr(ma), _ptr(mb)))
        return a.value, b.value, ma, mb

    def autotune_list_build(self, steps_per_variant=10):
        """(chosen variant, mean list-build ms per variant) of the FP32 list
        build's launch variants, timed over real rebuilds while stepping
        (dmph_autotune_list_build; advances 3 x steps_per_variant steps)."""
        v = C.c_int()
        ms = np.zeros(BUILD_VARIANTS, np.float32)
        self._check(lib().dmph_autotune_list_build(self._h, steps_per_variant, C.byref(v), _ptr(ms)))
        return v.value, ms

    def set_variants(self, variant_a, variant_b):
        self._check(lib().dmph_set_variants(self._h, variant_a, variant_b))

    # ---------------------------------------------------------- surrogate
    def enable_surrogate(self, **kw):
        """attach the learned K-step surrogate (dmph_surrogate_enable); keyword
        arguments override fields of dmph_surrogate_params_default"""
        sp = abi.SurrogateParams()
        lib().dmph_surrogate_params_default(C.byref(sp))
        for k, v in kw.items():
            if not hasattr(sp, k):
                raise KeyError(k)
            setattr(sp, k, v)
        self._check(lib().dmph_surrogate_enable(self._h, C.byref(sp)))
        self.surrogate_params = sp

    def surrogate_collect(self, nblocks):
        self._check(lib().dmph_surrogate_collect(self._h, nblocks))

    def surrogate_train(self, iters):
        loss = C.c_float()
        self._check(lib().dmph_surrogate_train(self._h, iters, C.byref(loss)))
        return loss.value

    def surrogate_advance(self, nblocks):
        self._check(lib().dmph_surrogate_advance(self._h, nblocks))

    def surrogate_stats(self):
        st = abi.SurrogateStats()
        self._check(lib().dmph_surrogate_get_stats(self._h, C.byref(st)))
        return st.as_dict()

    def surrogate_weights(self):
        n = lib().dmph_surrogate_get_weights(self._h, None, 0)
        if n < 0:
            self._check(n)
        w = np.zeros(n, np.float32)
        self._check(lib().dmph_surrogate_get_weights(self._h, _ptr(w), n))
        return w

    def set_surrogate_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(lib().dmph_surrogate_set_weights(self._h, _ptr(w), len(w)))

    def mlp_forward(self, X, layers=False):
        """the surrogate network on host rows (dmph_mlp_forward: the fused
        kernel; layers=True: one GEMM per layer, dmph_mlp_forward_layers)"""
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, abi.MLP_IN)
        Y = np.zeros((len(X), abi.MLP_OUT), np.float32)
        fn = lib().dmph_mlp_forward_layers if layers else lib().dmph_mlp_forward
        self._check(fn(self._h, _ptr(X), len(X), _ptr(Y)))
        return Y

    def surrogate_samples(self, capacity):
        """(X [rows, 64], T [rows, 16]) of the training pool, oldest first
        (dmph_surrogate_get_samples)"""
        X = np.zeros((capacity, abi.MLP_IN), np.float32)
        T = np.zeros((capacity, abi.MLP_OUT), np.float32)
        rows = C.c_int()
        self._check(lib().dmph_surrogate_get_samples(self._h, _ptr(X), _ptr(T), capacity, C.byref(rows)))
        return X[:rows.value], T[:rows.value]

    def surrogate_add_samples(self, X, T):
        """append rows to the training pool (dmph_surrogate_add_samples)"""
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, abi.MLP_IN)
        T = np.ascontiguousarray(T, dtype=np.float32).reshape(-1, abi.MLP_OUT)
        self._check(lib().dmph_surrogate_add_samples(self._h, _ptr(X), _ptr(T), len(X)))

    def mlp_forward_ms(self, n, reps=20, layers=False):
        """device ms of one forward pass over n rows of the surrogate's
        current features (dmph_mlp_forward_timed)"""
        ms = C.c_float()
        self._check(lib().dmph_mlp_forward_timed(self._h, n, reps, 1 if layers else 0, C.byref(ms)))
        return ms.value

    def mlp_gradient(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, abi.MLP_IN)
        T = np.ascontiguousarray(T, dtype=np.float32).reshape(-1, abi.MLP_OUT)
        g = np.zeros(len(self.surrogate_weights()), np.float32)
        loss = C.c_float()
        self._check(lib().dmph_mlp_gradient(self._h, _ptr(X), _ptr(T), len(X), _ptr(g), C.byref(loss)))
        return g, loss.value

    def surrogate_features(self):
        F = np.zeros((self.n, abi.MLP_FEATURES), np.float32)
        rows = C.c_int()
        self._check(lib().dmph_surrogate_features(self._h, _ptr(F), C.byref(rows)))
        return F[:rows.value]

    def set_profiling(self, on=True):
        self._check(lib().dmph_set_profiling(self._h, 1 if on else 0))

    def phase_times(self):
        """{phase: (total_ms, count)} accumulated since set_profiling(True)"""
        ms = np.zeros(len(self.PHASES), np.float64)
        n = np.zeros(len(self.PHASES), np.int64)
        self._check(lib().dmph_get_phase_times(self._h, _ptr(ms), _ptr(n), len(self.PHASES)))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(self.PHASES)}

    def close(self):
        if getattr(self, "_h", None):
            lib().dmph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Ensemble:
    """Independent FP32 scenes advanced together (dmph_ensemble_*): the pair
    passes of all scenes run as one persistent launch each, a whole ensemble
    step is one CUDA graph.  Keeps references to its solvers; step the scenes
    only through the ensemble while it exists."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        hs = (C.c_void_p * len(self.solvers))(*[s._h.value for s in self.solvers])
        h = C.c_void_p()
        rc = lib().dmph_ensemble_create(hs, len(self.solvers), C.byref(h))
        if rc != 0:
            raise DmphError(rc, "dmph_ensemble_create rejected the scenes")
        self._h = h

    def _check(self, rc):
        if rc != 0:
            raise DmphError(rc, lib().dmph_ensemble_last_error(self._h).decode())

    def step(self, n=1):
        self._check(lib().dmph_ensemble_step(self._h, n))

    def step_timed(self, n=1):
        ms = C.c_float()
        self._check(lib().dmph_ensemble_step_timed(self._h, n, C.byref(ms)))
        return ms.value

    def autotune(self):
        a, b = C.c_int(), C.c_int()
        ma = np.zeros(PASS_VARIANTS, np.float32)
        mb = np.zeros(PASS_VARIANTS, np.float32)
        self._check(lib().dmph_ensemble_autotune(self._h, C.byref(a), C.byref(b), _ptr(ma), _ptr(mb)))
        return a.value, b.value, ma, mb

    def set_pair_mode(self, mode):
        """"stencil" or "list" (dmph_set_pair_mode; FP32 split build)"""
        self._check(lib().dmph_set_pair_mode(self._h, {"stencil": 0, "list": 1}[mode]))

    def set_graph(self, on=True):
        self._check(lib().dmph_ensemble_set_graph(self._h, 1 if on else 0))

    def set_profiling(self, on=True):
        """CUDA events around the ensemble passes (dmph_ensemble_set_profiling)"""
        self._check(lib().dmph_ensemble_set_profiling(self._h, 1 if on else 0))

    def phase_times(self):
        """{phase: (total ms, launches)} of the timed phases (pass_a, pass_b)"""
        ms = np.zeros(7)
        n = np.zeros(7, np.int64)
        self._check(lib().dmph_ensemble_get_phase_times(self._h, _ptr(ms), _ptr(n), 7))
        return {name: (float(ms[k]), int(n[k])) for k, name in ((2, "pass_a"), (3, "pass_b")) if n[k] > 0}

    def info(self):
        n, s = C.c_int64(), C.c_int64()
        self._check(lib().dmph_ensemble_info(self._h, C.byref(n), C.byref(s)))
        return {"kernel_launches": n.value, "steps": s.value}

    def close(self):
        if getattr(self, "_h", None):
            lib().dmph_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_data_file(path):
    """dem.data -> Params through the library's own reader (dmph_read_data_file)."""
    p = abi.Params()
    lib().dmph_params_default(C.byref(p))
    rc = lib().dmph_read_data_file(path.encode(), C.byref(p))
    if rc != 0:
        raise DmphError(rc, lib().dmph_io_last_message().decode())
    return p


def read_grid_file(path, params):
    """.grid/.prof -> (type, x, v) through dmph_read_grid_file; fills the header into params."""
    n = C.c_int(0)
    rc = lib().dmph_read_grid_file(path.encode(), C.byref(params), C.byref(n), None, None, None)
    if rc != 0:
        raise DmphError(rc, lib().dmph_io_last_message().decode())
    t = np.empty(n.value, np.int32)
    x = np.empty((n.value, 3), np.float64)
    v = np.empty((n.value, 3), np.float64)
    rc = lib().dmph_read_grid_file(path.encode(), C.byref(params), C.byref(n), _ptr(t), _ptr(x), _ptr(v))
    if rc != 0:
        raise DmphError(rc, lib().dmph_io_last_message().decode())
    return t, x, v
