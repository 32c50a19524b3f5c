"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

liboracle_axj.so is the line-faithful C restatement of the reference's hot path in
axj_oracle.c. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
use it, as the checker; the product (axisymmetricjet_b200 / libaxj.so) never does.
Parity status: unpinned against reference outputs (see axj_oracle.c's header).
"""
import ctypes as C
import os
import subprocess

import numpy as np

from axisymmetricjet_b200._ffi import AxjBcRecord, AxjParams, AxjPatch, dptr, patch_array, patches_to_tuples, \
    record_array

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}
# "plain": the oracle proper (no FMA contraction); "fma": the same source with FMA
# contraction, only used to calibrate how far two correct FP64 builds drift apart.
_VARIANTS = {"plain": "liboracle_axj.so", "fma": "liboracle_axj_fma.so"}


def build(variant="plain"):
    subprocess.run(["make", "-s", "-C", _HERE, _VARIANTS[variant]], check=True)


def load(variant="plain"):
    if variant in _LIBS:
        return _LIBS[variant]
    path = os.path.join(_HERE, _VARIANTS[variant])
    if not os.path.exists(path):
        build(variant)
    lib = C.CDLL(path)
    dp = C.POINTER(C.c_double)
    i64 = C.c_int64
    v = C.c_void_p
    sig = {
        "axo_create": (v, [C.POINTER(AxjParams), i64, i64, dp, dp, dp, C.POINTER(AxjPatch), i64]),
        "axo_destroy": (None, [v]),
        "axo_set_state": (C.c_int, [v, dp, dp, i64, C.c_double]),
        "axo_get_state": (C.c_int, [v, dp]),
        "axo_get_time": (None, [v, C.POINTER(i64), dp, dp]),
        "axo_compute_dt": (C.c_int, [v, dp]),
        "axo_rk4_step": (C.c_int, [v, C.c_double]),
        "axo_rhs": (C.c_int, [v, dp, dp]),
        "axo_deriv1": (C.c_int, [v, dp, i64, dp]),
        "axo_deriv2": (C.c_int, [v, dp, i64, dp, dp]),
        "axo_deriv2comp": (C.c_int, [v, dp, i64, dp]),
        "axo_tgfilter": (C.c_int, [v, dp, i64, i64, dp]),
        "axo_sensor": (C.c_int, [v, dp, dp, dp, dp]),
        "axo_tables": (None, [v, dp, dp, dp]),
        "axo_metrics": (None, [v, dp, dp, dp, dp]),
        "axo_set_decomposition": (C.c_int, [v, i64, i64]),
        "axo_block_T": (None, [v, dp]),
        "axo_point_maps": (None, [v, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "axo_patches_from_records": (C.c_int, [C.POINTER(AxjBcRecord), i64, i64, i64, C.POINTER(AxjPatch),
                                               C.POINTER(i64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIBS[variant] = lib
    return lib


def patches_from_records(records, Nz, Nr):
    lib = load()
    rec = record_array(records)
    out = (AxjPatch * max(len(records), 1))()
    n = C.c_int64(0)
    lib.axo_patches_from_records(rec, len(records), Nz, Nr, out, C.byref(n))
    return patches_to_tuples(out, n.value)


class Oracle:
    """Same method names and array conventions as axisymmetricjet_b200.AxiJetSolver."""

    def __init__(self, params, zvec, rvec, ibval, patches, variant="plain"):
        self.lib = load(variant)
        zvec = np.ascontiguousarray(zvec, dtype=np.float64)
        rvec = np.ascontiguousarray(rvec, dtype=np.float64)
        ibval = np.ascontiguousarray(ibval, dtype=np.float64)
        self.Nr, self.Nz = zvec.shape
        self.params = params
        pa = patch_array(patches)
        self.h = self.lib.axo_create(C.byref(params), self.Nz, self.Nr, dptr(zvec), dptr(rvec), dptr(ibval), pa,
                                     len(patches))
        if not self.h:
            raise ValueError("oracle: grid too small")

    def close(self):
        if self.h:
            self.lib.axo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _field(self):
        return np.empty((self.Nr, self.Nz), dtype=np.float64)

    def set_state(self, pv, pv_target, iteration=0, time=0.0):
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        tg = np.ascontiguousarray(pv_target, dtype=np.float64)
        self.lib.axo_set_state(self.h, dptr(pv), dptr(tg), int(iteration), float(time))

    def get_state(self):
        out = np.empty((5, self.Nr, self.Nz), dtype=np.float64)
        self.lib.axo_get_state(self.h, dptr(out))
        return out

    def get_time(self):
        it, t, ts = C.c_int64(0), C.c_double(0.0), C.c_double(0.0)
        self.lib.axo_get_time(self.h, C.byref(it), C.byref(t), C.byref(ts))
        return it.value, t.value

    def stale_T(self):
        it, t, ts = C.c_int64(0), C.c_double(0.0), C.c_double(0.0)
        self.lib.axo_get_time(self.h, C.byref(it), C.byref(t), C.byref(ts))
        return ts.value

    def set_decomposition(self, dims_z, dims_r):
        """Replica of the reference run on a dims_z x dims_r process grid (ModDecomp.f90):
        block-local sensor edges and first rows, the in-place z filter restarted at block
        starts, per-block stale T and top-sponge denominator. Resets the blocks' T to 0."""
        rc = self.lib.axo_set_decomposition(self.h, int(dims_z), int(dims_r))
        if rc != 0:
            raise ValueError(f"oracle: decomposition {dims_z} x {dims_r} rejected (status {rc})")
        self.dims = (int(dims_z), int(dims_r))

    def point_maps(self):
        """zrow, rrow, blank, nfaceops, faceop_ids per point (see axo_point_maps); needs a
        state (set_state) for the recorded pass of the bc loop."""
        out = {k: np.zeros((self.Nr, self.Nz), dtype=np.uint8) for k in ("zrow", "rrow", "blank", "nfaceops")}
        out["faceop_ids"] = np.zeros((self.Nr, self.Nz), dtype=np.uint64)
        self.lib.axo_point_maps(self.h, out["zrow"].ctypes.data, out["rrow"].ctypes.data, out["blank"].ctypes.data,
                                out["nfaceops"].ctypes.data, out["faceop_ids"].ctypes.data)
        return out

    def block_T(self):
        """The module scalar T of every block, as [dims_r, dims_z]."""
        dz, dr = getattr(self, "dims", (1, 1))
        out = np.empty(dz * dr)
        self.lib.axo_block_T(self.h, dptr(out))
        return out.reshape(dr, dz)

    def compute_time_step(self):
        d = C.c_double(0.0)
        rc = self.lib.axo_compute_dt(self.h, C.byref(d))
        if rc != 0:
            raise RuntimeError(f"oracle ComputeTimeStep status {rc}")
        return d.value

    def rk4(self, delt):
        self.lib.axo_rk4_step(self.h, float(delt))

    def run(self, nsteps):
        d = 0.0
        for _ in range(nsteps):
            d = self.compute_time_step()
            self.rk4(d)
        return d

    def compute_rhs(self, pv):
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        out = np.empty_like(pv)
        self.lib.axo_rhs(self.h, dptr(pv), dptr(out))
        return out

    def deriv1(self, var, dirn):
        out = self._field()
        self.lib.axo_deriv1(self.h, dptr(np.ascontiguousarray(var, dtype=np.float64)), int(dirn), dptr(out))
        return out

    def deriv2(self, var, dirn, first):
        out = self._field()
        self.lib.axo_deriv2(self.h, dptr(np.ascontiguousarray(var, dtype=np.float64)), int(dirn),
                            dptr(np.ascontiguousarray(first, dtype=np.float64)), dptr(out))
        return out

    def deriv2comp(self, var, dirn):
        out = self._field()
        self.lib.axo_deriv2comp(self.h, dptr(np.ascontiguousarray(var, dtype=np.float64)), int(dirn), dptr(out))
        return out

    def tgfilter(self, var, dirn, out, inplace=False):
        out = np.array(out, dtype=np.float64, order="C", copy=True)
        v = None if inplace else dptr(np.ascontiguousarray(var, dtype=np.float64))
        self.lib.axo_tgfilter(self.h, v, int(dirn), int(bool(inplace)), dptr(out))
        return out

    def sensor(self, pv):
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        mu, beta, kappa = self._field(), self._field(), self._field()
        self.lib.axo_sensor(self.h, dptr(pv), dptr(mu), dptr(beta), dptr(kappa))
        return mu, beta, kappa

    def tables(self):
        s1, s2, tg = np.empty((9, 6)), np.empty((9, 6)), np.empty((9, 11))
        self.lib.axo_tables(self.h, dptr(s1), dptr(s2), dptr(tg))
        return s1, s2, tg

    def metrics(self):
        a, b, c, d = self._field(), self._field(), self._field(), self._field()
        self.lib.axo_metrics(self.h, dptr(a), dptr(b), dptr(c), dptr(d))
        return a, b, c, d
