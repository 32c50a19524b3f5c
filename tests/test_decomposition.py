"""The oracle's replica of a decomposed reference run (ModDecomp.f90: a dims_z x dims_r
process grid with halo exchanges). The device path is the single block (dims = (1, 1));
these tests pin where, and only where, a decomposed reference run departs from it:
nowhere without shock capturing and with the physical dt; through the per-rank stale T
in the reference dt; through the block-local sensor edges and first rows and the
restarted in-place z filter with shock capturing."""
import math

import numpy as np
import pytest

from axisymmetricjet_b200 import fixtures
from axisymmetricjet_b200._ffi import NSCBC_NOSLIP_WALL


def oracle(oracle_mod, c, dims=None):
    o = oracle_mod.Oracle(c["params"], c["zvec"], c["rvec"], c["ibval"],
                          oracle_mod.patches_from_records(c["records"], c["Nz"], c["Nr"]))
    if dims is not None:
        o.set_decomposition(*dims)
    o.set_state(c["pv"], c["target"])
    return o


@pytest.mark.parametrize("dims", [(2, 2), (3, 1), (1, 2)])
def test_plain_physical_dt_run_is_decomposition_independent(oracle_mod, dims):
    """Without shock capturing and with the local-T dt, every operator reads freshly
    exchanged halos: a decomposed run equals the single block bit for bit."""
    c = fixtures.case("jet96x64", dt_mode=1)
    a, b = oracle(oracle_mod, c), oracle(oracle_mod, c, dims)
    for _ in range(4):
        da, db = a.compute_time_step(), b.compute_time_step()
        assert da == db
        a.rk4(da)
        b.rk4(db)
    assert np.array_equal(a.get_state(), b.get_state())


def _dt_with_T(o, c, Ts, i_lo, i_hi, j_lo, j_hi):
    """ComputeTimeStep (ModInputOutput.f90:389-438) over one block with the scalar Ts,
    from the state: mu = kappa = T**0.666, beta = 0.6 mu, lambda = beta - 2/3 mu."""
    pv = o.get_state()
    dxidz, detadr, _, _ = o.metrics()
    Re, Pr, CFL = c["params"].Re, c["params"].Pr, c["params"].CFL
    best = math.inf
    for j in range(j_lo, j_hi):
        for i in range(i_lo, i_hi):
            Vr, Vz, T = pv[1, j, i], pv[3, j, i], pv[4, j, i]
            mu = math.pow(T, 0.666)
            lam = 0.6 * mu - (2.0 / 3.0) * mu
            dx, dr = dxidz[j, i], detadr[j, i]
            inv = abs(Vz * dx + Vr * dr) + math.sqrt(Ts) * math.sqrt(dx * dx + dr * dr)
            visc = 2.0 * max(mu / Re, lam / Re, mu / (Re * Pr)) * (abs(dx) + abs(dr)) ** 2
            best = min(best, CFL / (inv + visc))
    return best


def _blocks(N, d):
    """0-based [lo, hi) of each block: N // d points, the last block the rest
    (ModDecomp.f90:35-105)."""
    w = N // d
    return [(b * w, N if b == d - 1 else (b + 1) * w) for b in range(d)]


def test_reference_dt_takes_the_min_over_ranks_of_their_stale_T(oracle_mod):
    """The stale module scalar T is per rank: the last face point its own bc loop
    visited, or the last point of its RHS loops; dt is the MIN over ranks. 2 x 8 blocks
    of 48 x 8 points: the axis-side ranks end their inflow face at row 8, in the shear
    layer, where T differs from the ambient value the single block ends with."""
    c = fixtures.case("jet96x64")
    dims = (2, 8)
    a, b = oracle(oracle_mod, c), oracle(oracle_mod, c, dims)
    for _ in range(1):  # before the first RHS every rank's T is 0
        d = a.compute_time_step()
        assert b.compute_time_step() == d
        a.rk4(d)
        b.rk4(d)
    assert np.array_equal(a.get_state(), b.get_state())
    Tb = b.block_T()
    # the top-right rank visits the top face last, at (Nz, Nr), as the single block does
    assert Tb[-1, -1] == a.stale_T()
    assert Tb[0, 0] != a.stale_T()
    zb, rb = _blocks(c["Nz"], dims[0]), _blocks(c["Nr"], dims[1])
    want = min(_dt_with_T(b, c, Tb[q, p], zb[p][0], zb[p][1], rb[q][0], rb[q][1])
               for q in range(dims[1]) for p in range(dims[0]))
    got = b.compute_time_step()
    assert abs(got - want) <= 1e-14 * want, (got, want)
    single = a.compute_time_step()
    assert got != single


def test_sensor_departs_only_near_the_block_boundary_in_z(oracle_mod):
    """dims_z = 2 (boundary between columns 48 and 49, 1-based): one-sided deltaz at
    both block edges and the in-place z filter restarted at column 49 from the left
    block's unfiltered values. Columns up to 43 keep the single block's values (their
    9-point windows reach column 47 at most)."""
    c = fixtures.case("jet96x64sc")
    a, b = oracle(oracle_mod, c), oracle(oracle_mod, c, (2, 1))
    sa, sb = a.sensor(c["pv"]), b.sensor(c["pv"])
    for fa, fb in zip(sa, sb):
        assert np.array_equal(fa[:, :43], fb[:, :43])
    assert any(not np.array_equal(fa[:, 43:52], fb[:, 43:52]) for fa, fb in zip(sa, sb))


def test_sensor_departs_only_near_the_block_boundary_in_r(oracle_mod):
    """dims_r = 2 (boundary between rows 32 and 33): the upper block's first row takes
    the axis form of the dilatation and S22, deltar is one-sided at both block edges; the
    fourth differences (reach 4) and the r filter (reach 4) spread it to rows 25..40.
    Rows up to 24 and from 41 on keep the single block's values."""
    c = fixtures.case("jet96x64sc")
    a, b = oracle(oracle_mod, c), oracle(oracle_mod, c, (1, 2))
    sa, sb = a.sensor(c["pv"]), b.sensor(c["pv"])
    for fa, fb in zip(sa, sb):
        assert np.array_equal(fa[:24], fb[:24])
        assert np.array_equal(fa[41:], fb[41:])
    assert any(not np.array_equal(fa[24:41], fb[24:41]) for fa, fb in zip(sa, sb))


def test_decomposed_shock_capturing_run_stays_close(oracle_mod):
    """A 2 x 2 run with shock capturing departs from the single block (the device
    path) only by the block-boundary effects: small, but not zero."""
    c = fixtures.case("jet96x64sc", dt_mode=1)
    a, b = oracle(oracle_mod, c), oracle(oracle_mod, c, (2, 2))
    for _ in range(5):
        d = a.compute_time_step()
        a.rk4(d)
        b.rk4(d)
    sa, sb = a.get_state(), b.get_state()
    rel = [np.linalg.norm(sa[k] - sb[k]) / np.linalg.norm(sa[k]) for k in (0, 3, 4)]
    assert 0.0 < max(rel) < 1e-6, rel


def test_rejected_decompositions(oracle_mod):
    c = fixtures.nozzle_case(wall=NSCBC_NOSLIP_WALL)  # 96 x 64, lip face strip at i = 20..23
    o = oracle(oracle_mod, c)
    with pytest.raises(ValueError):
        o.set_decomposition(13, 1)  # blocks of 7 columns
    with pytest.raises(ValueError):
        o.set_decomposition(9, 1)   # blocks of 10: a boundary at column 21 splits the strip
    o.set_decomposition(4, 2)       # boundaries at 25, 49, 73 and row 33: accepted
