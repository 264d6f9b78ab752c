"""Known-answer tests of the device stages, from the inputs and expectations
of the reference's own self-checks (src/benchmark.cpp:39-677): synthetic
states whose result is known in closed form, independent of the oracle.

1 halo fingerprint (:39-104): interior prim carries the block id, ghosts
  -999; after exchange_bc every ghost layer at an interface-window centre
  carries the neighbour's id.
2 unit-cube metrics (:109-165): x = i, y = j, z = k gives vol == 1 (device).
3 physical BC logic (:170-297): no-slip wall negates the mirrored velocity,
  zeroes it on the face and flags ghost 3 with a negative density; slip wall
  reflects the normal velocity; far field flags ghost 3.
4 state update (:302-382): uniform state; c, T = M^2 gamma p / rho,
  Sutherland mu, Q.
5 time step (:387-494): metrics diag 10, vol 1e-3, rho = p = 1, mu = 0.1,
  Re = 1000, cfl = 1: dt = cfl / (3 (c 10 + 2 mu 100 / (Re rho vol))) / vol.
6 viscous exactness (:499-593): u = y^2, metrics diag 0.01, vol 1e-3,
  mu = 0.1, Re = 1000: dq(x-momentum) at the block centre = -2.0e-7.
7 interface averaging (:598-677): vol = 1, dq = block id + 1000; the
  interface face centre holds the mean of the two blocks.
"""
import math

import numpy as np
import pytest

from orion_b200 import cases, solver

pytestmark = pytest.mark.gpu
NG = cases.NG


def _centre(b):
    return NG + (b.idim - 1) // 2, NG + (b.jdim - 1) // 2, NG + (b.kdim - 1) // 2


def test_kat1_halo_fingerprint():
    case = cases.small_case("kat1", dims=(33, 25, 23), split=(2, 2, 1))
    fs = solver.FlowFieldSet(case)
    for n, b in enumerate(case.blocks):
        nx, ny, nz = b.padded
        prim = np.full((6, nz, ny, nx), -999.0)
        k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        inner = (slice(NG, NG + b.kdim), slice(NG, NG + b.jdim), slice(NG, NG + b.idim))
        prim[0][inner] = n
        prim[1][inner] = 0.0
        prim[2][inner] = i[inner]
        prim[3][inner] = j[inner]
        prim[4][inner] = k[inner]
        prim[5][inner] = 1.0
        fs.upload(n, "prim", prim)
    solver.HaloExchanger().exchange_bc(None, fs)
    checked = 0
    for n, b in enumerate(case.blocks):
        p = fs.download(n, "prim")
        ic, jc, kc = _centre(b)
        for face, reg in zip(cases.FACES, b.regions):
            if reg.bctype != cases.BC_INTERFACE:
                continue
            for layer in (1, 2, 3):
                at = {"imin": (kc, jc, NG - layer), "imax": (kc, jc, NG + b.idim - 1 + layer),
                      "jmin": (kc, NG - layer, ic), "jmax": (kc, NG + b.jdim - 1 + layer, ic),
                      "kmin": (NG - layer, jc, ic), "kmax": (NG + b.kdim - 1 + layer, jc, ic)}[face]
                assert abs(p[0][at] - (reg.nbt - 1)) <= 0.1, (n, face, layer, p[0][at])
                checked += 1
    assert checked == 4 * 2 * 3  # four blocks, two interfaces each, three layers
    fs.close()


def test_kat2_unit_cube_metrics_on_device():
    ni, nj, nk = 13, 12, 12
    k, j, i = np.meshgrid(np.arange(nk), np.arange(nj), np.arange(ni), indexing="ij")
    blk = cases.Block(ni, nj, nk, i.astype(np.float64), j.astype(np.float64), k.astype(np.float64))
    case = cases.Case("kat2", [blk], cases.FlowParams())
    fs = solver.FlowFieldSet(case, init=False)
    vol = fs.download(0, "vol")
    assert np.max(np.abs(vol[NG:-NG, NG:-NG, NG:-NG] - 1.0)) <= 1e-12
    fs.close()


def test_kat3_physical_bc_logic():
    # no-slip (adiabatic) wall on jmin, far field on imin
    case = cases.small_case("kat3v", dims=(33, 25, 23), noise_seed=3)
    b = case.blocks[0]
    ic, jc, kc = _centre(b)
    fs = solver.FlowFieldSet(case)
    before = fs.download(0, "prim")
    solver.apply_physical_bc(None, fs)
    p = fs.download(0, "prim")
    for d in (1, 2, 3):
        assert np.array_equal(p[1:4, kc, NG - d, ic], -before[1:4, kc, NG + d, ic])
    assert p[0, kc, NG - 3, ic] < 0 and p[0, kc, NG - 1, ic] > 0
    assert np.all(p[1:4, kc, NG, ic] == 0.0)
    assert p[0, kc, jc, NG - 3] < 0  # far-field ghost 3 flagged
    fs.close()

    # slip wall (Euler, no wall-normal averaging)
    case = cases.small_case("kat3i", dims=(33, 25, 23), noise_seed=4, nvis=0, method=0)
    fs = solver.FlowFieldSet(case)
    before = fs.download(0, "prim")
    met = fs.download(0, "metrics")
    solver.apply_physical_bc(None, fs)
    p = fs.download(0, "prim")
    m = met[3:6, kc, NG, ic]  # eta metrics at the wall point
    nrm = m / max(math.sqrt(float(m[0] * m[0] + m[1] * m[1] + m[2] * m[2])), 1e-30)
    for d in (1, 2, 3):
        vi = before[1:4, kc, NG + d, ic]
        vn = vi[0] * nrm[0] + vi[1] * nrm[1] + vi[2] * nrm[2]
        assert np.allclose(p[1:4, kc, NG - d, ic], vi - 2.0 * vn * nrm, rtol=0, atol=1e-13)
        sign = -1.0 if d == 3 else 1.0
        assert p[0, kc, NG - d, ic] == sign * before[0, kc, NG + d, ic]
        assert p[4, kc, NG - d, ic] == before[4, kc, NG + d, ic]
    fs.close()


def test_kat4_state_update():
    case = cases.small_case("kat4", dims=(25, 17, 13), moo=0.5)
    b = case.blocks[0]
    nx, ny, nz = b.padded
    prim = np.empty((6, nz, ny, nx))
    prim[0], prim[1], prim[2], prim[3], prim[4], prim[5] = 1.0, 10.0, 20.0, 30.0, 1.0e5, 1.0
    fs = solver.FlowFieldSet(case)
    fs.upload(0, "prim", prim)
    solver.StateUpdater.update_flow_states(fs)
    ic, jc, kc = _centre(b)
    g, p = case.params.gamma, case.params
    a2 = g * 1.0e5 / 1.0
    t = (p.moo * p.moo) * a2
    mu = t * math.sqrt(t) * (1.0 + p.visc) / (t + p.visc)
    assert fs.download(0, "c")[kc, jc, ic] == pytest.approx(math.sqrt(a2), rel=1e-14)
    assert fs.download(0, "prim")[5, kc, jc, ic] == pytest.approx(t, rel=1e-14)
    assert fs.download(0, "mu")[kc, jc, ic] == pytest.approx(mu, rel=1e-14)
    q = fs.download(0, "q")[:, kc, jc, ic]
    expect = [1.0, 10.0, 20.0, 30.0, 1.0e5 / (g - 1.0) + 0.5 * 1.0 * (100.0 + 400.0 + 900.0)]
    assert np.allclose(q, expect, rtol=1e-14, atol=0)
    fs.close()


def test_kat5_time_step():
    case = cases.small_case("kat5", dims=(25, 17, 13), reynolds=1000.0, cfl=1.0)
    b = case.blocks[0]
    nx, ny, nz = b.padded
    fs = solver.FlowFieldSet(case)
    met = np.zeros((9, nz, ny, nx))
    met[0] = met[4] = met[8] = 10.0
    fs.upload(0, "metrics", met)
    fs.upload(0, "vol", np.full((nz, ny, nx), 1e-3))
    prim = np.zeros((6, nz, ny, nx))
    prim[0] = prim[4] = prim[5] = 1.0
    fs.upload(0, "prim", prim)
    c = math.sqrt(case.params.gamma)
    fs.upload(0, "c", np.full((nz, ny, nx), c))
    fs.upload(0, "mu", np.full((nz, ny, nx), 0.1))
    phydtime = solver.TimeIntegrator.calculate_time_step(fs)
    dt_phys = 1.0 / (3.0 * (c * 10.0 + 2.0 * 0.1 * 100.0 / (1000.0 * 1.0 * 1e-3)))
    dt = fs.download(0, "dt")[NG:-NG, NG:-NG, NG:-NG]
    assert np.allclose(dt, dt_phys / 1e-3, rtol=1e-13, atol=0)
    assert phydtime == pytest.approx(dt_phys, rel=1e-13)
    fs.close()


def test_kat6_viscous_exactness():
    """u = y^2 on the grid that metrics diag 0.01 and vol 1e-3 describe (spacing
    0.1): tau_xy = 2 mu y, its eta-face flux 0.01 tau_xy differences to
    2e-4 per index, so dq(x-momentum) = -2e-4 / Re = -2e-7.  The stencils are
    exact on a quadratic; the xi and zeta fluxes of x-momentum vanish."""
    case = cases.small_case("kat6", dims=(25, 25, 25), reynolds=1000.0)
    b = case.blocks[0]
    nx, ny, nz = b.padded
    fs = solver.FlowFieldSet(case)
    met = np.zeros((9, nz, ny, nx))
    met[0] = met[4] = met[8] = 0.01
    fs.upload(0, "metrics", met)
    fs.upload(0, "vol", np.full((nz, ny, nx), 1e-3))
    _, j, _ = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    prim = np.zeros((6, nz, ny, nx))
    prim[0] = prim[4] = prim[5] = 1.0
    prim[1] = (0.1 * (j - NG)) ** 2
    fs.upload(0, "prim", prim)
    fs.upload(0, "mu", np.full((nz, ny, nx), 0.1))
    fs.upload(0, "dq", np.zeros((5, nz, ny, nx)))
    solver.FluxComputer.compute_viscous_rhs(fs)
    ic, jc, kc = _centre(b)
    got = fs.download(0, "dq")[1, kc, jc, ic]
    assert abs(got - (-2.0e-7)) <= 1e-10
    assert got == pytest.approx(-2.0e-7, rel=1e-8)
    fs.close()


def test_kat7_interface_averaging():
    case = cases.small_case("kat7", dims=(33, 25, 23), split=(2, 1, 1))
    fs = solver.FlowFieldSet(case)
    for n, b in enumerate(case.blocks):
        nx, ny, nz = b.padded
        fs.upload(n, "vol", np.ones((nz, ny, nx)))
        fs.upload(n, "dq", np.full((5, nz, ny, nx), 1000.0 + n))
    solver.HaloExchanger().average_interface_residuals(None, fs)
    b0, b1 = case.blocks
    _, jc, kc = _centre(b0)
    assert np.all(fs.download(0, "dq")[:, kc, jc, NG + b0.idim - 1] == 1000.5)
    assert np.all(fs.download(1, "dq")[:, kc, jc, NG] == 1000.5)
    # away from the interface nothing moves
    assert np.all(fs.download(0, "dq")[:, kc, jc, NG] == 1000.0)
    fs.close()
