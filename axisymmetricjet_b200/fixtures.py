"""Synthetic jet cases: grid, iblank, initial condition, target and bc records.

The reference ships no grid, restart or target file (only bc_4400x640_nozzle.dat),
so cases are generated from their published shapes:

* jet512x128  -- plain method, small: Nz=512 x Nr=128, z uniform on [0, 30D],
  r_j = 10D sinh(3 j/(Nr-1))/sinh(3), gamma=1.4, Pr=0.72, Re=1000, M_j=0.9,
  shock capturing off, 100 RK4 steps.
* jet4400x640 -- production size: Nz=4400 x Nr=640, z on [0, 60D], r to 15D,
  M_j=1.5, Re=5000, shock capturing on, 1000 RK4 steps.
* small test cases of the same construction, and a nozzle case with a blanked
  lip and no-slip wall patches laid out like the reference's own nozzle bc file
  (bc_4400x640_nozzle.dat, WriteMeshAndSoln/write_soln_file.f90:223-257).
* the case of the reference's own generator (WriteMeshAndSoln/write_soln_file.f90):
  its stretched 250 x 50 grid, blanked lip, bc file and initial condition, restated
  operation for operation (writemesh_case).

Initial condition: V_z = U_j/2 (1 + tanh((0.5D - r)/(2*0.05D))), V_r = V_theta = 0,
T from Crocco-Busemann (write_soln_file.f90:68-72), rho = 1/T (p = rho T = 1), plus a
seeded Gaussian perturbation of amplitude 1e-3 U_j on V_r and V_z where |r-0.5D| < 0.2D.
The target (pv_target) is the unperturbed profile.
"""
import math

import numpy as np

from ._ffi import AXIS, NSCBC_NONREFLECTING, NSCBC_NOSLIP_WALL, SAT_FARFIELD, SAT_NOSLIP_WALL, default_params

# Artificial-diffusivity coefficients used when shock capturing is on. The reference
# ships C_mu = C_beta = C_kappa = 0 (ModuleVariables.f90:164); these are the
# Kawai-Lele-type values.
SC_COEFFS = dict(C_mu=0.002, C_beta=1.75, C_kappa=0.01)

JET_RECORDS = [
    (SAT_FARFIELD, 1, 1, 1, 1, -1),           # inflow z = 0
    (NSCBC_NONREFLECTING, -1, -1, -1, 1, -1),  # outflow z = z_max
    (NSCBC_NONREFLECTING, -2, 1, -1, -1, -1),  # top r = r_max
    (AXIS, 2, 1, -1, 1, 1),                    # axis r = 0
]


def grid(Nz, Nr, zmax, rmax):
    z = zmax * np.arange(Nz, dtype=np.float64) / (Nz - 1)
    r = rmax * np.sinh(3.0 * np.arange(Nr, dtype=np.float64) / (Nr - 1)) / np.sinh(3.0)
    zvec = np.ascontiguousarray(np.broadcast_to(z[None, :], (Nr, Nz)))
    rvec = np.ascontiguousarray(np.broadcast_to(r[:, None], (Nr, Nz)))
    return z, r, zvec, rvec


def jet_profile(r, Mj, Tj_Tinf=1.0, gam=1.4):
    """(rho, V_z, T) of the tanh jet with Crocco-Busemann temperature."""
    Uj = Mj * np.sqrt(Tj_Tinf)
    ut = 0.5 * (1.0 + np.tanh((0.5 - r) / (2.0 * 0.05)))
    T_Tj = 0.5 * (gam - 1.0) * ut * (1.0 - ut) * Mj ** 2 + ut + (1.0 - ut) / Tj_Tinf
    T = Tj_Tinf * T_Tj
    return 1.0 / T, Uj * ut, T, Uj


def initial_condition(r, Nz, Mj, seed=12345, amp=1e-3, Tj_Tinf=1.0, gam=1.4):
    Nr = r.shape[0]
    rho, Vz, T, Uj = jet_profile(r, Mj, Tj_Tinf, gam)
    tgt = np.zeros((5, Nr, Nz))
    tgt[0] = rho[:, None]
    tgt[3] = Vz[:, None]
    tgt[4] = T[:, None]
    pv = tgt.copy()
    rng = np.random.default_rng(seed)
    mask = (np.abs(r - 0.5) < 0.2)[:, None]
    pv[1] += amp * Uj * rng.standard_normal((Nr, Nz)) * mask
    pv[3] += amp * Uj * rng.standard_normal((Nr, Nz)) * mask
    return np.ascontiguousarray(pv), np.ascontiguousarray(tgt)


def make_case(Nz, Nr, zmax, rmax, Mj, Re, sc=False, seed=12345, records=None, ibval=None, **pkw):
    z, r, zvec, rvec = grid(Nz, Nr, zmax, rmax)
    kw = dict(Re=float(Re))
    if sc:
        kw.update(shock_capturing=1, **SC_COEFFS)
    kw.update(pkw)
    params = default_params(**kw)
    pv, tgt = initial_condition(r, Nz, Mj, seed=seed)
    if ibval is None:
        ibval = np.ones((Nr, Nz))
    return dict(Nz=Nz, Nr=Nr, z=z, r=r, zvec=zvec, rvec=rvec, ibval=np.ascontiguousarray(ibval),
                records=list(records or JET_RECORDS), params=params, pv=pv, target=tgt, Mj=Mj)


def nozzle_records(iw, jb, jt, wall=NSCBC_NOSLIP_WALL):
    """A nozzle lip from z = 0 to i = iw between rows jb and jt (1-based), with the
    record order of the reference's nozzle bc file."""
    return [
        (SAT_FARFIELD, 1, 1, 1, 1, jb),
        (wall, -2, 1, iw, jb, jb),
        (wall, 1, iw, iw, jb, jt),
        (wall, 2, 1, iw, jt, jt),
        (SAT_FARFIELD, 1, 1, 1, jt, -1),
        (NSCBC_NONREFLECTING, -2, 1, -1, -1, -1),
        (NSCBC_NONREFLECTING, -1, -1, -1, 1, -1),
        (AXIS, 2, 1, -1, 1, 1),
    ]


def nozzle_case(Nz=96, Nr=64, zmax=30.0, rmax=15.0, Mj=0.9, Re=1000.0, iw=20, jb=24, jt=28, wall=NSCBC_NOSLIP_WALL,
                sc=False, seed=12345, **pkw):
    ib = np.ones((Nr, Nz))
    ib[jb:jt - 1, :iw - 1] = 0.0  # rows jb+1..jt-1, columns 1..iw-1 (1-based) are inside the lip
    return make_case(Nz, Nr, zmax, rmax, Mj, Re, sc=sc, seed=seed, records=nozzle_records(iw, jb, jt, wall),
                     ibval=ib, **pkw)


def _stretched(i, n, delta, pos, cmin, cmax):
    """compute_coord_val (WriteMeshAndSoln/write_soln_file.f90:95-115): a tanh-stretched
    coordinate clustered at cmin + pos. xi = float(i)/float(n) is a default-REAL (single
    precision) division and 1.0 - xi a single-precision difference, as in the Fortran;
    the rest is double precision."""
    f32 = np.float32
    pos1 = pos / (cmax - cmin)
    xi = f32(i) / f32(n)
    u1 = math.tanh(delta * float(f32(1.0) - xi)) * (1.0 - pos1)
    u2 = (2.0 - math.tanh(delta * float(xi))) * pos1
    fac = 1.0 - ((u1 + u2) - pos1)
    return cmin + fac * (cmax - cmin)


def writemesh_grid(nx=150, ny=50, n_wall_zone=100):
    """create_AxiJet_CartGrid (write_soln_file.f90:117-213): the z coordinate of the
    first nx columns up to the first one beyond z = 11 (ipos2), a second stretching from
    11 to 15 over the wall zone from ipos2 on, the r coordinate, and iblank = 0 inside
    the nozzle lip (1 < r < 1.05, z < 6). Returns (z, r, iblank[Nr, Nz]) with 1-based
    quantities of the Fortran turned into 0-based arrays."""
    Nz = nx + n_wall_zone
    z = np.zeros(Nz)
    ipos2 = None
    for i in range(1, nx + 1):
        xval = _stretched(i, nx, 3.0, 6.0, 0.0, 15.0)
        if xval > 11.0:
            ipos2 = i
            break
        z[i - 1] = xval
    if ipos2 is None:
        raise ValueError("the first stretching never passes z = 11")
    for i in range(ipos2, Nz + 1):
        z[i - 1] = _stretched(i - ipos2, Nz - ipos2, 2.0, 3.0, 11.0, 15.0)
    r = np.array([_stretched(j, ny, 6.0, 1.0, 0.0, 15.0) for j in range(1, ny + 1)])
    lip = (r[:, None] > 1.0) & (r[:, None] < 1.05) & (z[None, :] < 6.0)
    iblank = np.where(lip, 0.0, 1.0)
    return z, r, iblank


def writemesh_records(z, r):
    """The bc file written by create_AxiJet_CartGrid (write_soln_file.f90:219-257):
    jbottom = the last row at or below r = 1, jtop = the first row at or above r = 1.05,
    iright = the first column at or beyond z = 6 (all 1-based), no-slip NSCBC walls
    around the lip and at the outflow, a non-reflecting top and the axis."""
    jbottom = int(np.nonzero(r > 1.0)[0][0])          # first 1-based j with r > 1, minus 1
    jtop = int(np.nonzero(r < 1.05)[0][-1]) + 2       # last 1-based j with r < 1.05, plus 1
    iright = int(np.nonzero(z < 6.0)[0][-1]) + 2      # last 1-based i with z < 6, plus 1
    return [
        (SAT_FARFIELD, 1, 1, 1, 1, jbottom),
        (NSCBC_NOSLIP_WALL, -2, 1, iright, jbottom, jbottom),
        (NSCBC_NOSLIP_WALL, 1, iright, iright, jbottom, jtop),
        (NSCBC_NOSLIP_WALL, 2, 1, iright, jtop, jtop),
        (SAT_FARFIELD, 1, 1, 1, jtop, -1),
        (NSCBC_NONREFLECTING, -2, 1, -1, -1, -1),
        (NSCBC_NOSLIP_WALL, -1, -1, -1, 1, -1),
        (AXIS, 2, 1, -1, 1, 1),
    ]


def write_bc_file(path, records):
    """A bc file in the layout create_AxiJet_CartGrid writes (write_soln_file.f90:248-257):
    per row grid, bc, dir, istart, iend, jstart, jend, kstart, kend as '(9(I0,2X))'."""
    with open(path, "w") as f:
        for bc, d, i0, i1, j0, j1 in records:
            f.write("".join("%d  " % v for v in (1, bc, d, i0, i1, j0, j1, 1, 1)) + "\n")


def writemesh_solution(z, r, Mj=0.8, Tj_Tinf=0.6, gam=1.4):
    """The initial condition of write_soln_file.f90:36-90 as pv[5, Nr, Nz]: a tanh jet
    of radius 1 (theta = 0.1, a default-REAL literal stored in a double), decaying as
    (z - 5)**-1.5 beyond z = 6, zero velocity beyond r = 1, density from the
    Crocco-Busemann relation and T = 1/rho."""
    theta = float(np.float32(0.1))
    Uj = Mj * math.pow(Tj_Tinf, 0.5)
    Nz, Nr = z.shape[0], r.shape[0]
    # libm tanh and pow per value, as the Fortran calls them
    u = np.array([0.5 * (1.0 - math.tanh(1.0 / (4.0 * theta) * (rj - 1.0 / rj))) for rj in r])
    u = 2.0 * u - 1.0
    uu = np.broadcast_to(u[:, None], (Nr, Nz)).copy()
    decay = np.array([math.pow(zi - 6.0 + 1.0, 1.5) if zi > 6.0 else 1.0 for zi in z])
    far = z > 6.0
    uu[:, far] = uu[:, far] / decay[far][None, :]
    uu[r > 1.0, :] = 0.0
    term1 = 0.5 * (gam - 1.0) * uu * (1.0 - uu) * (Mj * Mj)
    term3 = (1.0 / Tj_Tinf) * (1.0 - uu)
    rho = (1.0 / ((term1 + uu) + term3)) / Tj_Tinf
    pv = np.zeros((5, Nr, Nz))
    pv[0] = rho
    pv[3] = uu * Uj
    pv[4] = 1.0 / rho
    return pv


def writemesh_case(sc=False, **pkw):
    """The case WriteMeshAndSoln generates (write_soln_file.f90:1-265): the 250 x 50
    stretched grid with the blanked nozzle lip, its bc file and its initial condition,
    which is also the target (the reference reads the one solution file for both).
    pkw go to the parameters (reference defaults otherwise)."""
    z, r, ib = writemesh_grid()
    Nz, Nr = z.shape[0], r.shape[0]
    kw = dict(pkw)
    if sc:
        kw = dict(shock_capturing=1, **SC_COEFFS, **kw)
    pv = writemesh_solution(z, r)
    return dict(Nz=Nz, Nr=Nr, z=z, r=r,
                zvec=np.ascontiguousarray(np.broadcast_to(z[None, :], (Nr, Nz))),
                rvec=np.ascontiguousarray(np.broadcast_to(r[:, None], (Nr, Nz))),
                ibval=np.ascontiguousarray(ib), records=writemesh_records(z, r), params=default_params(**kw),
                pv=np.ascontiguousarray(pv), target=pv.copy(), Mj=0.8)


CASES = {
    "jet512x128": dict(Nz=512, Nr=128, zmax=30.0, rmax=10.0, Mj=0.9, Re=1000.0, sc=False),
    "jet4400x640": dict(Nz=4400, Nr=640, zmax=60.0, rmax=15.0, Mj=1.5, Re=5000.0, sc=True),
    "jet96x64": dict(Nz=96, Nr=64, zmax=30.0, rmax=15.0, Mj=0.9, Re=1000.0, sc=False),
    "jet96x64sc": dict(Nz=96, Nr=64, zmax=30.0, rmax=15.0, Mj=1.5, Re=5000.0, sc=True),
    # profiling case: the production physics on fewer z points (state 52 MB, larger than L2
    # once the RK work buffers are counted, about 0.8 GB on the device)
    "jet2048x640": dict(Nz=2048, Nr=640, zmax=60.0, rmax=15.0, Mj=1.5, Re=5000.0, sc=True),
}


def case(name, **kw):
    spec = dict(CASES[name])
    spec.update(kw)
    return make_case(**spec)


def batch_instances(n=64, seed=2024, nz_range=(256, 2048), nr_range=(96, 384), mach_range=(0.9, 1.5),
                    re_range=(1000.0, 5000.0), amp_frac=(0.0, 0.02), st_range=(0.2, 0.6), **pkw):
    """Cases of uneven independent jets for a batch: Nz and Nr drawn uniformly from
    their ranges and rounded to multiples of 32, Mach and Re uniform, and an
    azimuthal-mode-0 harmonic inflow forcing (control_forcing = 2) in the shear layer
    near the inflow with amplitude uniform in amp_frac * U_j and Strouhal number in
    st_range. Every case has the small plain case's construction (z on [0, 30D], r to
    10D, tanh profile, seeded perturbation) with shock capturing on; pkw go to the
    parameters of every case (e.g. precision, sensor)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        Nz = int(np.clip(32 * np.round(rng.uniform(*nz_range) / 32), 32, None))
        Nr = int(np.clip(32 * np.round(rng.uniform(*nr_range) / 32), 32, None))
        Mj = float(rng.uniform(*mach_range))
        Re = float(rng.uniform(*re_range))
        Uj = Mj  # T_j = T_inf = 1
        amp = float(rng.uniform(*amp_frac)) * Uj
        st = float(rng.uniform(*st_range))
        c = make_case(Nz, Nr, 30.0, 10.0, Mj, Re, sc=True, seed=seed + k, control_forcing=2, forcing_z0=1.0,
                      forcing_r0=0.5, forcing_lz=0.5, forcing_lr=0.2, harmonic_amp=amp, harmonic_st=st,
                      harmonic_uj=Uj, **pkw)
        c.update(Re=Re, amp=amp, St=st)
        out.append(c)
    return out
