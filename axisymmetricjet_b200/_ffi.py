"""ctypes mirror of include/axj.h: the POD structs and status codes of the C-ABI."""
import ctypes as C

import numpy as np

AXJ_OK = 0
STATUS = {
    0: "AXJ_OK",
    1: "AXJ_ERR_ARG",
    2: "AXJ_ERR_CUDA",
    3: "AXJ_ERR_NONFINITE",
    4: "AXJ_ERR_DT_BLOWUP",
    5: "AXJ_ERR_TIMEOUT",
    6: "AXJ_ERR_BADPATCH",
    7: "AXJ_ERR_BADGRID",
    8: "AXJ_ERR_NOMEM",
    9: "AXJ_ERR_NODEVICE",
    10: "AXJ_ERR_UNSUPPORTED",
}

# boundary-condition codes (ModuleVariables.f90:112-117)
AXIS, SAT_FARFIELD, NSCBC_NONREFLECTING, SAT_NOSLIP_WALL, NSCBC_NOSLIP_WALL, SPONGE = 90, 91, 92, 93, 94, 95


class AxjParams(C.Structure):
    _fields_ = [
        ("gam", C.c_double),
        ("Re", C.c_double),
        ("Pr", C.c_double),
        ("CFL", C.c_double),
        ("sponge_start_top", C.c_double),
        ("sponge_A_top", C.c_double),
        ("sponge_end_left", C.c_double),
        ("sponge_A_left", C.c_double),
        ("C_mu", C.c_double),
        ("C_beta", C.c_double),
        ("C_kappa", C.c_double),
        ("forcing_alpha", C.c_double),
        ("forcing_z0", C.c_double),
        ("forcing_r0", C.c_double),
        ("forcing_lz", C.c_double),
        ("forcing_lr", C.c_double),
        ("forcing_mat", C.c_double * 25),
        ("do_viscous_terms", C.c_int64),
        ("shock_capturing", C.c_int64),
        ("control_forcing", C.c_int64),
        ("dt_mode", C.c_int64),
        ("precision", C.c_int64),
        ("sensor", C.c_int64),
        ("judge_every", C.c_int64),
        ("judge_threshold", C.c_double),
        ("device", C.c_int64),
        ("harmonic_amp", C.c_double),
        ("harmonic_st", C.c_double),
        ("harmonic_uj", C.c_double),
        ("patch_prep", C.c_int64),
        ("stage_rows", C.c_int64),
        ("judge_stages", C.c_int64),
        ("reserved", C.c_int64 * 1),
    ]


class AxjPatch(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("i_start", "i_end", "j_start", "j_end", "bc", "bc_dir")]


class AxjBcRecord(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("bc", "bc_dir", "istart", "iend", "jstart", "jend")]


MLP_CH, MLP_IN, MLP_HID, MLP_OUT = 4, 100, 64, 2


class AxjMlp(C.Structure):
    _fields_ = [
        ("w1", C.c_float * (MLP_HID * MLP_IN)),
        ("b1", C.c_float * MLP_HID),
        ("w2", C.c_float * (MLP_HID * MLP_HID)),
        ("b2", C.c_float * MLP_HID),
        ("w3", C.c_float * (MLP_OUT * MLP_HID)),
        ("b3", C.c_float * MLP_OUT),
        ("feat_mean", C.c_float * MLP_CH),
        ("feat_scale", C.c_float * MLP_CH),
        ("out_scale", C.c_float * MLP_OUT),
    ]
    SHAPES = {"w1": (MLP_HID, MLP_IN), "b1": (MLP_HID,), "w2": (MLP_HID, MLP_HID), "b2": (MLP_HID,),
              "w3": (MLP_OUT, MLP_HID), "b3": (MLP_OUT,), "feat_mean": (MLP_CH,), "feat_scale": (MLP_CH,),
              "out_scale": (MLP_OUT,)}

    def to_dict(self):
        """float32 numpy copies of every field, weights as (out, in) matrices."""
        return {k: np.ctypeslib.as_array(getattr(self, k)).reshape(shp).astype(np.float32).copy()
                for k, shp in self.SHAPES.items()}

    @classmethod
    def from_dict(cls, d):
        m = cls()
        for k, shp in cls.SHAPES.items():
            arr = np.ascontiguousarray(np.asarray(d[k], dtype=np.float32).reshape(-1))
            assert arr.size == int(np.prod(shp)), k
            C.memmove(getattr(m, k), arr.ctypes.data, arr.nbytes)
        return m


class AxjTrainCfg(C.Structure):
    _fields_ = [
        ("steps", C.c_int64),
        ("batch", C.c_int64),
        ("lr", C.c_double),
        ("beta1", C.c_double),
        ("beta2", C.c_double),
        ("eps", C.c_double),
        ("seed", C.c_int64),
        ("fit_normalization", C.c_int64),
        ("reserved", C.c_int64 * 6),
    ]


def default_train_cfg(**overrides):
    """The defaults of axj_default_train_cfg: 2000 Adam steps, batch 65536, lr 1e-3."""
    c = AxjTrainCfg()
    c.steps, c.batch, c.lr, c.beta1, c.beta2, c.eps, c.seed, c.fit_normalization = \
        2000, 65536, 1e-3, 0.9, 0.999, 1e-8, 1, 1
    for k, v in overrides.items():
        setattr(c, k, v)
    return c


class AxjBatchTuning(C.Structure):
    _fields_ = [("tile_order", C.c_int64), ("stage_ctas_per_sm", C.c_int64), ("sensor_ctas_per_sm", C.c_int64),
                ("stage_rows", C.c_int64), ("general_ctas_per_sm", C.c_int64), ("general_serial", C.c_int64),
                ("reserved", C.c_int64 * 2)]

    def to_dict(self):
        return {"tile_order": self.tile_order, "stage_ctas_per_sm": self.stage_ctas_per_sm,
                "sensor_ctas_per_sm": self.sensor_ctas_per_sm, "stage_rows": self.stage_rows,
                "general_ctas_per_sm": self.general_ctas_per_sm, "general_serial": self.general_serial}


def default_params(**overrides):
    """The reference defaults of ModuleVariables.f90:4-188 (same as axj_default_params)."""
    p = AxjParams()
    p.gam, p.Re, p.Pr, p.CFL = 1.4, 1000.0, 0.72, 0.5
    p.sponge_start_top, p.sponge_A_top = 12.5, 0.5
    p.sponge_end_left, p.sponge_A_left = 6.0, 5.0
    p.C_mu = p.C_beta = p.C_kappa = 0.0
    p.forcing_alpha, p.forcing_lz, p.forcing_lr = 6.0, 1.0, 1.0
    p.do_viscous_terms, p.shock_capturing, p.control_forcing = 1, 0, 0
    p.dt_mode, p.precision, p.sensor = 0, 0, 0
    p.judge_every, p.judge_threshold = 50, 0.1
    for k, v in overrides.items():
        if k == "forcing_mat":
            arr = np.asarray(v, dtype=np.float64).reshape(25)
            for q in range(25):
                p.forcing_mat[q] = float(arr[q])
        else:
            setattr(p, k, v)
    return p


def patch_array(patches):
    """list of (i_start, i_end, j_start, j_end, bc, bc_dir) -> ctypes array."""
    arr = (AxjPatch * max(len(patches), 1))()
    for k, p in enumerate(patches):
        for n, v in zip(("i_start", "i_end", "j_start", "j_end", "bc", "bc_dir"), p):
            setattr(arr[k], n, int(v))
    return arr


def record_array(records):
    """list of (bc, bc_dir, istart, iend, jstart, jend) -> ctypes array."""
    arr = (AxjBcRecord * max(len(records), 1))()
    for k, r in enumerate(records):
        for n, v in zip(("bc", "bc_dir", "istart", "iend", "jstart", "jend"), r):
            setattr(arr[k], n, int(v))
    return arr


def patches_to_tuples(arr, n):
    return [(arr[k].i_start, arr[k].i_end, arr[k].j_start, arr[k].j_end, arr[k].bc, arr[k].bc_dir) for k in range(n)]


def dptr(a):
    """Pointer to a C-contiguous float64 numpy array."""
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "expected a C-contiguous float64 array"
    return a.ctypes.data_as(C.POINTER(C.c_double))
