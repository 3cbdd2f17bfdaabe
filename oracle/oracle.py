"""ctypes wrapper of liboracle.so, the CPU restatement of the reference step.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, never by the dem_mph_b200 package.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None

INT_FIELDS = {"ParticleIndex", "Property", "NeighborCount", "FluidNeighborCount",
              "SolidNeighborCount", "CellIndex", "CellParticle", "NeighborInd",
              "CellFluidParticleBegin", "CellFluidParticleEnd", "CellSolidParticleBegin",
              "CellSolidParticleEnd", "CellWallParticleBegin", "CellWallParticleEnd"}
VEC_FIELDS = {"Position", "Velocity", "Force", "GravityCenter", "NeighborCalculatedPosition"}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("oracle/liboracle.so is not built (make -C oracle oracle)")
        L = C.CDLL(LIB_PATH)
        L.dmph_oracle_create.restype = C.c_void_p
        L.dmph_oracle_create.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.dmph_oracle_step.argtypes = [C.c_void_p, C.c_int]
        L.dmph_oracle_size.restype = C.c_long
        L.dmph_oracle_size.argtypes = [C.c_void_p, C.c_char_p]
        L.dmph_oracle_get.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        L.dmph_oracle_scalar.restype = C.c_double
        L.dmph_oracle_scalar.argtypes = [C.c_void_p, C.c_char_p]
        L.dmph_oracle_destroy.argtypes = [C.c_void_p]
        L.dmph_oracle_set_bodies.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.dmph_oracle_get_bodies.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        L.dmph_oracle_pressure_force.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.dmph_oracle_step_begin.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.dmph_oracle_step_finish.argtypes = [C.c_void_p, C.c_int]
        L.dmph_oracle_rows.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.dmph_oracle_cell_sort.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.mlp_oracle_param_count.restype = C.c_int
        L.mlp_oracle_forward.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.mlp_oracle_grad.restype = C.c_double
        L.mlp_oracle_grad.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        _lib = L
    return _lib


class Oracle:
    """FP64 CPU restatement of the reference solver on one scene."""

    def __init__(self, params, typ, x, v):
        L = lib()
        self._typ = np.ascontiguousarray(typ, dtype=np.int32)
        xx = np.ascontiguousarray(x, dtype=np.float64)
        vv = np.ascontiguousarray(v, dtype=np.float64)
        self.n = len(self._typ)
        self._h = L.dmph_oracle_create(C.byref(params), self.n, self._typ.ctypes.data,
                                       xx.ctypes.data, vv.ctypes.data)
        if not self._h:
            raise ValueError("dmph_oracle_create rejected the scene")

    def step(self, n=1):
        rc = lib().dmph_oracle_step(self._h, n)
        if rc != 0:
            raise RuntimeError("dmph_oracle_step failed (%d)" % rc)

    def step_begin(self):
        """drift, walls, wrap, force reset; returns the largest squared
        displacement since the last rebuild"""
        m2 = C.c_double()
        lib().dmph_oracle_step_begin(self._h, C.byref(m2))
        return m2.value

    def step_finish(self, rebuild):
        lib().dmph_oracle_step_finish(self._h, 1 if rebuild else 0)

    def get_rows(self, rows):
        r = np.ascontiguousarray(rows, dtype=np.int32)
        x = np.empty((len(r), 3))
        v = np.empty((len(r), 3))
        if lib().dmph_oracle_rows(self._h, len(r), r.ctypes.data, x.ctypes.data, v.ctypes.data, 0) != 0:
            raise ValueError("row out of range")
        return x, v

    def set_rows(self, rows, x, v):
        r = np.ascontiguousarray(rows, dtype=np.int32)
        xx = np.ascontiguousarray(x, dtype=np.float64)
        vv = np.ascontiguousarray(v, dtype=np.float64)
        if lib().dmph_oracle_rows(self._h, len(r), r.ctypes.data, xx.ctypes.data, vv.ctypes.data, 1) != 0:
            raise ValueError("row out of range")

    def get(self, name):
        L = lib()
        size = L.dmph_oracle_size(self._h, name.encode())
        if size < 0:
            raise KeyError(name)
        if name == "NeighborPtr":
            out = np.empty(size, dtype=np.int64)
        elif name in INT_FIELDS:
            out = np.empty(size, dtype=np.int32)
        else:
            out = np.empty(size, dtype=np.float64)
        L.dmph_oracle_get(self._h, name.encode(), out.ctypes.data)
        if name in VEC_FIELDS:
            out = out.reshape(-1, 3)
        return out

    def set_bodies(self, body_of_row, body_density):
        b = np.ascontiguousarray(body_of_row, dtype=np.int32)
        rho = np.ascontiguousarray(body_density, dtype=np.float64)
        rc = lib().dmph_oracle_set_bodies(self._h, len(rho), b.ctypes.data, rho.ctypes.data)
        if rc != 0:
            raise ValueError("dmph_oracle_set_bodies rejected the bodies")
        self.nbodies = len(rho)

    def bodies(self):
        B = getattr(self, "nbodies", 0)
        out = {k: np.zeros((B, 3)) for k in ("X", "V", "L")}
        out["q"] = np.zeros((B, 4))
        out["M"] = np.zeros(B)
        lib().dmph_oracle_get_bodies(self._h, out["X"].ctypes.data, out["V"].ctypes.data, out["q"].ctypes.data,
                                     out["L"].ctypes.data, out["M"].ctypes.data)
        return out

    def pressure_force(self, pressure):
        """pressure-gradient force [N,3] of the given pressure field on the
        current positions and neighbour lists"""
        P = np.ascontiguousarray(pressure, dtype=np.float64)
        if P.shape != (self.n,):
            raise ValueError("pressure_force wants %d pressures" % self.n)
        F = np.zeros((self.n, 3))
        lib().dmph_oracle_pressure_force(self._h, P.ctypes.data, F.ctypes.data)
        return F

    def scalar(self, name):
        return lib().dmph_oracle_scalar(self._h, name.encode())

    def close(self):
        if self._h:
            lib().dmph_oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cell_sort(params, typ, x):
    """(sorted keys, permutation) of the reference's cell sort of the given
    particles alone (dmph_oracle_cell_sort)"""
    t = np.ascontiguousarray(typ, dtype=np.int32)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    key = np.empty(len(t), np.int32)
    perm = np.empty(len(t), np.int32)
    rc = lib().dmph_oracle_cell_sort(C.byref(params), len(t), t.ctypes.data, xx.ctypes.data, key.ctypes.data,
                                     perm.ctypes.data)
    if rc != 0:
        raise ValueError("dmph_oracle_cell_sort rejected the input (%d)" % rc)
    return key, perm


def mlp_forward(params, X):
    """CPU restatement of the surrogate MLP (oracle/dmph_mlp_oracle.c): X n x 64 -> n x 16"""
    P = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.zeros((len(X), 16), np.float32)
    lib().mlp_oracle_forward(P.ctypes.data, len(X), X.ctypes.data, Y.ctypes.data)
    return Y


def mlp_grad(params, X, T, n_valid=6):
    """(gradient, loss) of the mean squared error over the first n_valid outputs"""
    P = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    G = np.zeros(lib().mlp_oracle_param_count(), np.float32)
    loss = lib().mlp_oracle_grad(P.ctypes.data, len(X), X.ctypes.data, T.ctypes.data, n_valid, G.ctypes.data)
    return G, loss


def read_ref_dump(d):
    """Read one step directory written by oracle/_ref/ref_dump*."""
    out = {}
    for fn in os.listdir(d):
        base, ext = os.path.splitext(fn)
        path = os.path.join(d, fn)
        if ext == ".f64":
            a = np.fromfile(path, dtype=np.float64)
            out[base] = a.reshape(-1, 3) if base in VEC_FIELDS else a
        elif ext == ".i32":
            out[base] = np.fromfile(path, dtype=np.int32)
        elif ext == ".i64":
            out[base] = np.fromfile(path, dtype=np.int64)
        elif fn == "meta.txt":
            meta = {}
            for line in open(path):
                k, *vals = line.split()
                meta[k] = [float(s) for s in vals] if len(vals) > 1 else float(vals[0])
            out["meta"] = meta
    return out
