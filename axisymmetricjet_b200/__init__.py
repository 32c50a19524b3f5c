"""B200 per-step hot path of the axisymmetric compressible jet solver (nataraj2/AxisymmetricJet).

The compute path is libaxj.so (hand-written sm_100a CUDA behind the C-ABI in
include/axj.h). This module is the host-side mirror of the reference's call
interface for that path -- ComputeTimeStep / RK4 / ComputeRHS and the operator
routines -- over ctypes. There is no CPU fallback: if the library or a CUDA
device is missing, every call raises.

Array convention: a field is a numpy float64 array of shape (Nr, Nz) (z fastest,
the reference's column-major (Nz, Nr) layout); a solution pv is (5, Nr, Nz)
holding rho, V_r, V_theta, V_z, T (pv(Nz,Nr,1,5) of ModuleVariables.f90:39).
"""
import ctypes as C
import os

import numpy as np

from ._ffi import (AXJ_OK, STATUS, AxjBatchTuning, AxjBcRecord, AxjMlp, AxjParams, AxjPatch, AxjTrainCfg,
                   default_params, default_train_cfg, dptr, patch_array, patches_to_tuples, record_array)

__all__ = ["AxiJetSolver", "AxjBatch", "AxjError", "AxjMlp", "default_params", "default_train_cfg", "load_library",
           "read_bc_file", "patches_from_records", "operator_tables", "point_maps", "prep_maps", "library_path", "mlp_init"]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def library_path():
    return os.path.join(_HERE, "libaxj.so")


class AxjError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def load_library():
    """Load the in-tree libaxj.so (built by axisymmetricjet_b200.build). Raises if absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m axisymmetricjet_b200.build` "
                           "(there is no CPU fallback)")
    lib = C.CDLL(path)
    dp = C.POINTER(C.c_double)
    fp = C.POINTER(C.c_float)
    i64 = C.c_int64
    h = C.c_void_p
    sig = {
        "axj_default_params": (None, [C.POINTER(AxjParams)]),
        "axj_create": (C.c_int, [C.POINTER(AxjParams), i64, i64, dp, dp, dp, C.POINTER(AxjPatch), i64,
                                 C.POINTER(h)]),
        "axj_set_state": (C.c_int, [h, dp, dp, i64, C.c_double]),
        "axj_get_state": (C.c_int, [h, dp]),
        "axj_get_time": (C.c_int, [h, C.POINTER(i64), dp]),
        "axj_compute_dt": (C.c_int, [h, dp]),
        "axj_rk4_step": (C.c_int, [h, C.c_double]),
        "axj_run": (C.c_int, [h, i64, i64, C.c_void_p, C.c_void_p, dp]),
        "axj_run_timed": (C.c_int, [h, i64, dp]),
        "axj_profile_steps": (C.c_int, [h, i64, dp, C.POINTER(i64)]),
        "axj_rhs": (C.c_int, [h, dp, dp]),
        "axj_deriv1": (C.c_int, [h, dp, i64, dp]),
        "axj_deriv2": (C.c_int, [h, dp, i64, dp, dp]),
        "axj_tgfilter": (C.c_int, [h, dp, i64, i64, dp]),
        "axj_sensor": (C.c_int, [h, dp, dp, dp, dp]),
        "axj_last_error": (C.c_char_p, [h]),
        "axj_set_wait_limit": (C.c_int, [h, i64]),
        "axj_destroy": (None, [h]),
        "axj_read_bc_file": (C.c_int, [C.c_char_p, C.POINTER(AxjBcRecord), i64, C.POINTER(i64)]),
        "axj_operator_tables": (C.c_int, [dp, dp, dp]),
        "axj_prep_maps": (C.c_int, [C.POINTER(AxjPatch), i64, i64, i64, dp, i64, C.c_void_p, C.c_void_p, i64,
                                    C.POINTER(i64), C.c_void_p, i64, C.c_void_p, C.c_void_p]),
        "axj_point_maps": (C.c_int, [C.POINTER(AxjPatch), i64, i64, i64, dp, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]),
        "axj_patches_from_records": (C.c_int, [C.POINTER(AxjBcRecord), i64, i64, i64, C.POINTER(AxjPatch),
                                               C.POINTER(i64)]),
        "axj_version": (C.c_char_p, []),
        "axj_mu_of_T": (C.c_double, [C.c_double]),
        "axj_default_train_cfg": (None, [C.POINTER(AxjTrainCfg)]),
        "axj_mlp_init": (None, [C.POINTER(AxjMlp), i64]),
        "axj_mlp_set": (C.c_int, [h, C.POINTER(AxjMlp)]),
        "axj_mlp_get": (C.c_int, [h, C.POINTER(AxjMlp)]),
        "axj_dataset_reserve": (C.c_int, [h, i64]),
        "axj_dataset_add": (C.c_int, [h]),
        "axj_dataset_size": (C.c_int, [h, C.POINTER(i64)]),
        "axj_mlp_train": (C.c_int, [h, C.POINTER(AxjTrainCfg), fp]),
        "axj_dataset_sample": (C.c_int, [h, i64, i64, i64, fp, fp]),
        "axj_mlp_grad": (C.c_int, [h, fp, fp, i64, C.POINTER(AxjMlp), fp]),
        "axj_mlp_features": (C.c_int, [h, dp, fp]),
        "axj_mlp_predict": (C.c_int, [h, dp, dp, dp]),
        "axj_learned_stats": (C.c_int, [h, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)]),
        "axj_batch_default_tuning": (None, [C.POINTER(AxjBatchTuning)]),
        "axj_batch_create": (C.c_int, [C.POINTER(h), i64, C.POINTER(h)]),
        "axj_batch_run": (C.c_int, [h, i64]),
        "axj_batch_run_timed": (C.c_int, [h, i64, dp]),
        "axj_batch_set_tuning": (C.c_int, [h, C.POINTER(AxjBatchTuning)]),
        "axj_batch_get_tuning": (C.c_int, [h, C.POINTER(AxjBatchTuning)]),
        "axj_batch_autotune": (C.c_int, [h, i64, C.POINTER(AxjBatchTuning), dp, C.POINTER(i64)]),
        "axj_batch_last_error": (C.c_char_p, [h]),
        "axj_batch_destroy": (None, [h]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


OUTPUT_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_int64, C.c_double, C.POINTER(C.c_double))


def _check(lib, h, rc):
    if rc != AXJ_OK:
        msg = lib.axj_last_error(h)
        raise AxjError(rc, msg.decode() if msg else "")


def operator_tables():
    """(SBP1 [9, 6], SBP2 [9, 6], TGfilt [9, 11]) as the device kernels use them
    (ModOperator.f90:5-121)."""
    lib = load_library()
    s1, s2, tg = np.empty((9, 6)), np.empty((9, 6)), np.empty((9, 11))
    _check(lib, None, lib.axj_operator_tables(dptr(s1), dptr(s2), dptr(tg)))
    return s1, s2, tg


def point_maps(patches, Nz, Nr, ibval):
    """The per-point stencil rows and face operations the device descriptors encode
    (CreateAllPatches, ModPatch.f90:214-242; the BoundaryConditions loop, ModBC.f90:25-274):
    dict of zrow, rrow, blank, nfaceops (uint8) and faceop_ids (uint64: 1-based patch
    numbers, one per byte), each (Nr, Nz)."""
    lib = load_library()
    ib = np.ascontiguousarray(ibval, dtype=np.float64)
    pa = patch_array(patches)
    out = {k: np.zeros((Nr, Nz), dtype=np.uint8) for k in ("zrow", "rrow", "blank", "nfaceops")}
    out["faceop_ids"] = np.zeros((Nr, Nz), dtype=np.uint64)
    _check(lib, None, lib.axj_point_maps(pa, len(patches), Nz, Nr, dptr(ib), out["zrow"].ctypes.data,
                                         out["rrow"].ctypes.data, out["blank"].ctypes.data,
                                         out["nfaceops"].ctypes.data, out["faceop_ids"].ctypes.data))
    return out


def prep_maps(patches, Nz, Nr, ibval, algorithm=0):
    """The descriptors (Nr rows of pitch P = Nz rounded up to 32), face list, tile lists
    and stale-T point that axj_create builds: algorithm 0 the host path, 1 the device
    path's per-row / per-tile functions run on the host, 2 the device path."""
    lib = load_library()
    ib = np.ascontiguousarray(ibval, dtype=np.float64)
    pa = patch_array(patches)
    P = (Nz + 31) // 32 * 32
    desc = np.zeros((Nr, P), dtype=np.uint32)
    nf = C.c_int64(0)
    counts = np.zeros(4, dtype=np.int64)
    stale = np.zeros(2, dtype=np.int64)
    ntile_cap = 2 * ((Nz + 31) // 32) * (Nr // 8 + 2)
    faces = np.zeros(1 << 20, dtype=np.int32)
    tiles = np.zeros((ntile_cap, 2), dtype=np.int32)
    _check(lib, None, lib.axj_prep_maps(pa, len(patches), Nz, Nr, dptr(ib), int(algorithm), desc.ctypes.data,
                                        faces.ctypes.data, faces.size, C.byref(nf), tiles.ctypes.data, ntile_cap,
                                        counts.ctypes.data, stale.ctypes.data))
    lists, n = [], 0
    for c in counts:
        lists.append(tiles[n:n + c].copy())
        n += c
    return {"desc": desc, "faces": faces[:nf.value].copy(), "tiles": lists, "stale": tuple(int(v) for v in stale)}


def read_bc_file(path):
    """Rows of a bc file (ModPatch.f90:30-63) as (bc, bc_dir, istart, iend, jstart, jend) tuples."""
    lib = load_library()
    n = C.c_int64(0)
    _check(lib, None, lib.axj_read_bc_file(path.encode(), None, 0, C.byref(n)))
    arr = (AxjBcRecord * max(n.value, 1))()
    _check(lib, None, lib.axj_read_bc_file(path.encode(), arr, n.value, C.byref(n)))
    return [(arr[k].bc, arr[k].bc_dir, arr[k].istart, arr[k].iend, arr[k].jstart, arr[k].jend)
            for k in range(n.value)]


def patches_from_records(records, Nz, Nr):
    """PatchCreation for one block holding the whole grid (ModPatch.f90:117-309)."""
    lib = load_library()
    rec = record_array(records)
    out = (AxjPatch * max(len(records), 1))()
    n = C.c_int64(0)
    _check(lib, None, lib.axj_patches_from_records(rec, len(records), Nz, Nr, out, C.byref(n)))
    return patches_to_tuples(out, n.value)


class AxiJetSolver:
    """One device-resident block of the jet solver.

    Mirrors the reference's per-step interface: compute_time_step() is
    ComputeTimeStep (ModInputOutput.f90:389-438), rk4(delt) is RK4
    (ModRungeKutta.f90:5-171), compute_rhs(pv) is AssignValues + ComputeRHS
    (ModRHS.f90:5-258); deriv1/deriv2/tgfilter/sensor are the operator routines.
    """

    def __init__(self, params, zvec, rvec, ibval, patches):
        self.lib = load_library()
        zvec = np.ascontiguousarray(zvec, dtype=np.float64)
        rvec = np.ascontiguousarray(rvec, dtype=np.float64)
        ibval = np.ascontiguousarray(ibval, dtype=np.float64)
        self.Nr, self.Nz = zvec.shape
        assert rvec.shape == zvec.shape and ibval.shape == zvec.shape
        self.params = params
        pa = patch_array(patches)
        h = C.c_void_p()
        rc = self.lib.axj_create(C.byref(params), self.Nz, self.Nr, dptr(zvec), dptr(rvec), dptr(ibval), pa,
                                 len(patches), C.byref(h))
        _check(self.lib, None, rc)
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.axj_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _chk(self, rc):
        _check(self.lib, self.h, rc)

    def _field(self):
        return np.empty((self.Nr, self.Nz), dtype=np.float64)

    def set_state(self, pv, pv_target, iteration=0, time=0.0):
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        tg = np.ascontiguousarray(pv_target, dtype=np.float64)
        assert pv.shape == (5, self.Nr, self.Nz) and tg.shape == pv.shape
        self._chk(self.lib.axj_set_state(self.h, dptr(pv), dptr(tg), int(iteration), float(time)))

    def get_state(self, out=None):
        if out is None:
            out = np.empty((5, self.Nr, self.Nz), dtype=np.float64)
        self._chk(self.lib.axj_get_state(self.h, dptr(out)))
        return out

    def get_time(self):
        it = C.c_int64(0)
        t = C.c_double(0.0)
        self._chk(self.lib.axj_get_time(self.h, C.byref(it), C.byref(t)))
        return it.value, t.value

    def compute_time_step(self):
        d = C.c_double(0.0)
        self._chk(self.lib.axj_compute_dt(self.h, C.byref(d)))
        return d.value

    def rk4(self, delt):
        self._chk(self.lib.axj_rk4_step(self.h, float(delt)))

    def set_wait_limit(self, tries):
        """Poll limit of the kernels' bounded TMA waits on this handle's device (< 0: the
        default; 0: every wait gives up at once and the step reports AXJ_ERR_TIMEOUT)."""
        self._chk(self.lib.axj_set_wait_limit(self.h, int(tries)))

    def run(self, nsteps, out_every=0, callback=None):
        """nsteps x (ComputeTimeStep + RK4) on the device; returns the last dt."""
        cb = None
        if callback is not None and out_every > 0:
            n = 5 * self.Nr * self.Nz
            shape = (5, self.Nr, self.Nz)

            def _cb(user, iteration, time, pv):
                arr = np.ctypeslib.as_array(pv, shape=(n,)).reshape(shape).copy()
                callback(iteration, time, arr)

            cb = OUTPUT_CB(_cb)
        d = C.c_double(0.0)
        self._chk(self.lib.axj_run(self.h, int(nsteps), int(out_every), C.cast(cb, C.c_void_p) if cb else None,
                                   None, C.byref(d)))
        return d.value

    def run_timed(self, nsteps):
        """nsteps graph-replayed steps; returns their device time in ms (CUDA events)."""
        ms = C.c_double(0.0)
        self._chk(self.lib.axj_run_timed(self.h, int(nsteps), C.byref(ms)))
        return ms.value

    def profile_steps(self, nsteps):
        """nsteps eager steps with CUDA events around each launch group.
        Returns ({dt, sensor, stage, step}: ms summed, {dt, sensor, stage}: launches)."""
        ms = (C.c_double * 4)()
        nl = (C.c_int64 * 3)()
        self._chk(self.lib.axj_profile_steps(self.h, int(nsteps), ms, nl))
        keys = ("dt", "sensor", "stage", "step")
        return dict(zip(keys, list(ms))), dict(zip(keys[:3], list(nl)))

    def compute_rhs(self, pv):
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        out = np.empty_like(pv)
        self._chk(self.lib.axj_rhs(self.h, dptr(pv), dptr(out)))
        return out

    def deriv1(self, var, dirn):
        var = np.ascontiguousarray(var, dtype=np.float64)
        out = self._field()
        self._chk(self.lib.axj_deriv1(self.h, dptr(var), int(dirn), dptr(out)))
        return out

    def deriv2(self, var, dirn, first):
        var = np.ascontiguousarray(var, dtype=np.float64)
        first = np.ascontiguousarray(first, dtype=np.float64)
        out = self._field()
        self._chk(self.lib.axj_deriv2(self.h, dptr(var), int(dirn), dptr(first), dptr(out)))
        return out

    def tgfilter(self, var, dirn, out, inplace=False):
        out = np.array(out, dtype=np.float64, order="C", copy=True)
        v = None if inplace else dptr(np.ascontiguousarray(var, dtype=np.float64))
        self._chk(self.lib.axj_tgfilter(self.h, v, int(dirn), int(bool(inplace)), dptr(out)))
        return out

    def sensor(self, pv):
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        mu, beta, kappa = self._field(), self._field(), self._field()
        self._chk(self.lib.axj_sensor(self.h, dptr(pv), dptr(mu), dptr(beta), dptr(kappa)))
        return mu, beta, kappa

    # ---- learned sensor ----
    def mlp_set(self, model):
        """Install a model: an AxjMlp or a dict of its fields (see AxjMlp.to_dict)."""
        m = model if isinstance(model, AxjMlp) else AxjMlp.from_dict(model)
        self._chk(self.lib.axj_mlp_set(self.h, C.byref(m)))

    def mlp_get(self):
        m = AxjMlp()
        self._chk(self.lib.axj_mlp_get(self.h, C.byref(m)))
        return m.to_dict()

    def dataset_reserve(self, nsnapshots):
        self._chk(self.lib.axj_dataset_reserve(self.h, int(nsnapshots)))

    def dataset_add(self):
        self._chk(self.lib.axj_dataset_add(self.h))

    def dataset_size(self):
        n = C.c_int64(0)
        self._chk(self.lib.axj_dataset_size(self.h, C.byref(n)))
        return n.value

    def mlp_train(self, cfg=None, **overrides):
        """Adam training on the device; returns the per-step batch losses."""
        cfg = cfg if cfg is not None else default_train_cfg(**overrides)
        loss = np.zeros(max(int(cfg.steps), 1), dtype=np.float32)
        self._chk(self.lib.axj_mlp_train(self.h, C.byref(cfg), _fptr(loss)))
        return loss[:int(cfg.steps)]

    def dataset_sample(self, batch, seed, step):
        X = np.zeros((int(batch), 100), dtype=np.float32)
        T = np.zeros((int(batch), 2), dtype=np.float32)
        self._chk(self.lib.axj_dataset_sample(self.h, int(batch), int(seed), int(step), _fptr(X), _fptr(T)))
        return X, T

    def mlp_grad(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        g = AxjMlp()
        loss = np.zeros(1, dtype=np.float32)
        self._chk(self.lib.axj_mlp_grad(self.h, _fptr(X), _fptr(T), X.shape[0], C.byref(g), _fptr(loss)))
        d = g.to_dict()
        for k in ("feat_mean", "feat_scale", "out_scale"):
            d.pop(k)
        return d, float(loss[0])

    def mlp_features(self, pv):
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        out = np.zeros((4, self.Nr, self.Nz), dtype=np.float32)
        self._chk(self.lib.axj_mlp_features(self.h, dptr(pv), _fptr(out)))
        return out

    def mlp_predict(self, pv):
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        b, k = self._field(), self._field()
        self._chk(self.lib.axj_mlp_predict(self.h, dptr(pv), dptr(b), dptr(k)))
        return b, k

    def learned_stats(self):
        a, b, c = C.c_int64(0), C.c_int64(0), C.c_int64(0)
        self._chk(self.lib.axj_learned_stats(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return {"judged_outputs": a.value, "fallbacks": b.value, "judges": c.value}


class AxjBatch:
    """Many AxiJetSolver instances advanced together (axj_batch_*): every kernel of the
    step runs once for all instances, the step is graph-captured. The solvers keep their
    state; close the batch before them."""

    def __init__(self, solvers):
        self.lib = load_library()
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s.h for s in self.solvers])
        b = C.c_void_p()
        rc = self.lib.axj_batch_create(arr, len(self.solvers), C.byref(b))
        if rc != AXJ_OK:
            raise AxjError(rc, self.lib.axj_batch_last_error(None).decode())
        self.b = b

    def _chk(self, rc):
        if rc != AXJ_OK:
            raise AxjError(rc, self.lib.axj_batch_last_error(self.b).decode())

    def run(self, nsteps):
        self._chk(self.lib.axj_batch_run(self.b, int(nsteps)))

    def run_timed(self, nsteps):
        ms = C.c_double(0.0)
        self._chk(self.lib.axj_batch_run_timed(self.b, int(nsteps), C.byref(ms)))
        return ms.value

    def tuning(self):
        t = AxjBatchTuning()
        self._chk(self.lib.axj_batch_get_tuning(self.b, C.byref(t)))
        return t.to_dict()

    def set_tuning(self, **kw):
        t = AxjBatchTuning()
        self._chk(self.lib.axj_batch_get_tuning(self.b, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, int(v))
        self._chk(self.lib.axj_batch_set_tuning(self.b, C.byref(t)))

    def autotune(self, steps_per_trial=5):
        """Time every candidate tuning, keep the fastest; returns (chosen, trial times in ms)."""
        t = AxjBatchTuning()
        ms = (C.c_double * 32)()
        n = C.c_int64(0)
        self._chk(self.lib.axj_batch_autotune(self.b, int(steps_per_trial), C.byref(t), ms, C.byref(n)))
        return t.to_dict(), list(ms)[:n.value]

    def close(self):
        if getattr(self, "b", None):
            self.lib.axj_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fptr(a):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_float))


def mlp_init(seed):
    """axj_mlp_init: the seeded initial model as a dict of float32 arrays."""
    m = AxjMlp()
    load_library().axj_mlp_init(C.byref(m), int(seed))
    return m.to_dict()
