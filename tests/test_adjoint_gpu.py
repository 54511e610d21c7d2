"""Adjoint of the RK4 Biot-Savart step (tc_rk4_adjoint) on the GPU.

Checked against (1) an FP64 reference gradient: the same RK4 map written in
torch on the CPU and differentiated by torch.autograd (small grids), and
(2) centred finite differences (eps = 1e-6) of J through the GPU forward
step, on seeded entries: vorticities and tangent-plane position
perturbations (renormalised to the sphere), and (3) centred finite differences
taken through the reference's own BVERK4 (its Fortran source run by oracle/f90,
committed as tests/golden/ref_fd_rh4_l1.npz). The adjoint is wrapped in a
torch.autograd.Function here, in the test harness only.
"""
import math

import numpy as np
import pytest
import torch

from thesiscode_b200 import _native as N
from thesiscode_b200 import configs
from thesiscode_b200.panel_velocity import Context

pytestmark = pytest.mark.gpu


def adjoint(ctx, xA, zA, aA, dt, nsteps, ckpt, functional=N.TC_J_ENSTROPHY, probe=0):
    J = np.zeros(1)
    gz = np.zeros_like(zA)
    gx = np.zeros_like(xA)
    N.call("tc_rk4_adjoint", ctx.handle, N.dptr(np.ascontiguousarray(xA)), N.dptr(np.ascontiguousarray(zA)),
           N.dptr(np.ascontiguousarray(aA)), xA.shape[0], dt, nsteps, ckpt, functional, probe,
           N.dptr(J), N.dptr(gz), N.dptr(gx))
    return J[0], gz, gx


class EnstrophyAfterRK4(torch.autograd.Function):
    """J = sum zeta(T)^2 A through the library's forward and adjoint (test harness only)."""

    @staticmethod
    def forward(ctx_, x, z, area, lib_ctx, dt, nsteps, ckpt):
        J, gz, gx = adjoint(lib_ctx, x.detach().numpy(), z.detach().numpy(), area.numpy(), dt, nsteps, ckpt)
        ctx_.save_for_backward(torch.from_numpy(gx), torch.from_numpy(gz))
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx_, g):
        gx, gz = ctx_.saved_tensors
        return g * gx, g * gz, None, None, None, None, None


def torch_rk4_state(x, z, area, omega, d2, dt, nsteps):
    """The RK4 map of the active panels in torch FP64 (test harness): (x(T), zeta(T))."""
    n = x.shape[0]
    eye = torch.eye(n, dtype=torch.float64)

    def rhs(x, z):
        D = 1.0 + d2 - x @ x.T
        W = (z * area)[None, :] / (D + eye) * (1.0 - eye)
        S = W @ x
        u = -torch.cross(x, S, dim=1) / (4.0 * np.pi)
        return u, -2.0 * omega * u[:, 2]

    for _ in range(nsteps):
        k1x, k1z = rhs(x, z)
        k1x, k1z = dt * k1x, dt * k1z
        k2x, k2z = rhs(x + 0.5 * k1x, z + 0.5 * k1z)
        k2x, k2z = dt * k2x, dt * k2z
        k3x, k3z = rhs(x + 0.5 * k2x, z + 0.5 * k2z)
        k3x, k3z = dt * k3x, dt * k3z
        k4x, k4z = rhs(x + k3x, z + k3z)
        k4x, k4z = dt * k4x, dt * k4z
        x = x + k1x / 6 + k2x / 3 + k3x / 3 + k4x / 6
        z = z + k1z / 6 + k2z / 3 + k3z / 3 + k4z / 6
    return x, z


def torch_rk4_enstrophy(x, z, area, omega, d2, dt, nsteps, probe=None):
    n = x.shape[0]
    eye = torch.eye(n, dtype=torch.float64)

    def rhs(x, z):
        D = 1.0 + d2 - x @ x.T
        W = (z * area)[None, :] / (D + eye) * (1.0 - eye)
        S = W @ x
        u = -torch.cross(x, S, dim=1) / (4.0 * np.pi)
        return u, -2.0 * omega * u[:, 2]

    for _ in range(nsteps):
        k1x, k1z = rhs(x, z)
        k1x, k1z = dt * k1x, dt * k1z
        k2x, k2z = rhs(x + 0.5 * k1x, z + 0.5 * k1z)
        k2x, k2z = dt * k2x, dt * k2z
        k3x, k3z = rhs(x + 0.5 * k2x, z + 0.5 * k2z)
        k3x, k3z = dt * k3x, dt * k3z
        k4x, k4z = rhs(x + k3x, z + k3z)
        k4x, k4z = dt * k4x, dt * k4z
        x = x + k1x / 6 + k2x / 3 + k3x / 3 + k4x / 6
        z = z + k1z / 6 + k2z / 3 + k3z / 3 + k4z / 6
    return (z * z * area).sum() if probe is None else z[probe]


def jet(level):
    return configs.jet(level=level, delta=0.02, dt=0.005, steps=20)


@pytest.mark.parametrize("level", [2, 3])
def test_adjoint_matches_torch_autograd_fp64(gpu, level):
    # a Gaussian vortex: not zonally symmetric, so u_z != 0 and dJ/dx is not roundoff-sized;
    # level 3 (1,280 panels) is the largest the dense torch reference handles in seconds
    w = configs.gaussian(level=level, delta=0.02, dt=0.01)
    ctx = Context(0, "fp64")
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    nsteps, ckpt = 6, 4  # a partial last segment too
    x = torch.tensor(w.xA, requires_grad=True)
    z = torch.tensor(w.zetaA, requires_grad=True)
    area = torch.tensor(w.areaA)
    Jt = torch_rk4_enstrophy(x, z, area, w.omega, w.deltas[0] ** 2, w.dt, nsteps)
    Jt.backward()
    x2 = torch.tensor(w.xA, requires_grad=True)
    z2 = torch.tensor(w.zetaA, requires_grad=True)
    Jl = EnstrophyAfterRK4.apply(x2, z2, area, ctx, w.dt, nsteps, ckpt)
    Jl.backward()
    assert abs(Jl.item() - Jt.item()) <= 1e-12 * abs(Jt.item())
    gz_ref, gx_ref = z.grad.numpy(), x.grad.numpy()
    scale = np.abs(gz_ref).max()
    assert np.abs(z2.grad.numpy() - gz_ref).max() <= 1e-10 * scale
    # sum zeta^2 A is an invariant of the semi-discrete flow (dJ/dt = -4 Omega sum G_j u_z,j = 0 by
    # the antisymmetry of the pair term), so dJ/dx is only RK4-truncation sized: compare absolutely
    assert np.abs(x2.grad.numpy() - gx_ref).max() <= 1e-10 * scale
    ctx.close()


def test_adjoint_probe_gradient_matches_torch_autograd_fp64(gpu):
    """J = zeta_p(T): its position gradient is O(1), a full check of the position adjoint."""
    w = configs.gaussian(level=2, delta=0.02, dt=0.01)
    ctx = Context(0, "fp64")
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    nsteps, ckpt, p = 6, 4, 41
    x = torch.tensor(w.xA, requires_grad=True)
    z = torch.tensor(w.zetaA, requires_grad=True)
    Jt = torch_rk4_enstrophy(x, z, torch.tensor(w.areaA), w.omega, w.deltas[0] ** 2, w.dt, nsteps, probe=p)
    Jt.backward()
    J, gz, gx = adjoint(ctx, w.xA, w.zetaA, w.areaA, w.dt, nsteps, ckpt, N.TC_J_PROBE, p)
    assert abs(J - Jt.item()) <= 1e-12 * abs(Jt.item())
    assert np.abs(gx).max() > 1e-3
    assert np.abs(gx - x.grad.numpy()).max() <= 1e-10 * np.abs(gx).max()
    assert np.abs(gz - z.grad.numpy()).max() <= 1e-10 * np.abs(gz).max()
    ctx.close()


@pytest.mark.parametrize("level", [4, 6])
def test_adjoint_matches_centred_fd(gpu, level):
    """32 seeded entries (seed 33), eps = 1e-6, jet (delta 0.02), 20 steps of dt 0.005, checkpoint
    every 5; at level 6 (81,920 panels) this is the adjoint benchmark configuration itself.
    Error measure: |FD - adjoint| / max over all gradient entries <= 1e-6 (for J = sum zeta^2 A the
    position entries are RK4-truncation sized; J(+) - J(-) is summed termwise with exact rounding, so
    the FD's own rounding noise stays well below the bound). The position
    adjoint is then checked by FD through the probe functional J = zeta_p(T), whose position
    gradient is O(1)."""
    w = jet(level)
    ctx = Context(0, "fp64")
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    nsteps, ckpt, eps = 20, 5, 1e-6
    J, gz, gx = adjoint(ctx, w.xA, w.zetaA, w.areaA, w.dt, nsteps, ckpt)

    def final(x, z):
        x, z = x.copy(), z.copy()
        ctx.rk4_step(x, z, w.areaA, np.zeros((0, 3)), np.zeros((0, 3)), w.dt, nsteps)
        return z

    def J_of(x, z):
        return math.fsum(final(x, z) ** 2 * w.areaA)

    def J_diff(xp, zp, xm, zm):
        # J(+) - J(-) as one exactly rounded sum of the termwise differences: rounding J ~ 12
        # (level 6) itself would leave ulp(J) / (2 eps) ~ 1e-9 of noise, near the bound
        fp, fm = final(xp, zp), final(xm, zm)
        return math.fsum((fp - fm) * (fp + fm) * w.areaA)

    def tangent_pair(j, t):
        xp, xm = w.xA.copy(), w.xA.copy()
        xp[j] = (w.xA[j] + eps * t) / np.linalg.norm(w.xA[j] + eps * t)
        xm[j] = (w.xA[j] - eps * t) / np.linalg.norm(w.xA[j] - eps * t)
        return xp, xm

    def tangent(rng, j):
        t = rng.standard_normal(3)
        t -= t.dot(w.xA[j]) * w.xA[j]
        return t / np.linalg.norm(t)

    assert abs(J_of(w.xA, w.zetaA) - J) <= 1e-12 * abs(J)
    rng = np.random.default_rng(33)
    picks = rng.choice(w.nA, 32, replace=False)
    scale = max(np.abs(gz).max(), np.abs(gx).max())
    for m, j in enumerate(picks):
        if m % 2 == 0:  # vorticity entry
            zp, zm = w.zetaA.copy(), w.zetaA.copy()
            zp[j] += eps
            zm[j] -= eps
            fd = J_diff(w.xA, zp, w.xA, zm) / (2 * eps)
            assert abs(fd - gz[j]) <= 1e-6 * scale, (j, fd, gz[j])
        else:  # position entry along a tangent direction, renormalised
            t = tangent(rng, j)
            xp, xm = tangent_pair(j, t)
            fd = J_diff(xp, w.zetaA, xm, w.zetaA) / (2 * eps)
            assert abs(fd - gx[j].dot(t)) <= 1e-6 * scale, (j, fd, gx[j].dot(t))
    # position adjoint through the probe functional
    p = int(picks[0])
    Jp, gzp, gxp = adjoint(ctx, w.xA, w.zetaA, w.areaA, w.dt, nsteps, ckpt, N.TC_J_PROBE, p)
    near = np.argsort(np.linalg.norm(w.xA - w.xA[p], axis=1))[:8]  # the panels that move zeta_p most
    for j in near:
        t = tangent(rng, j)
        xp, xm = tangent_pair(j, t)
        fd = (final(xp, w.zetaA)[p] - final(xm, w.zetaA)[p]) / (2 * eps)
        assert abs(fd - gxp[j].dot(t)) <= 1e-6 * np.abs(gxp).max(), (j, fd, gxp[j].dot(t))
    ctx.close()


def test_adjoint_probe_functional_and_errors(gpu):
    w = jet(2)
    ctx = Context(0, "fp64")
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    J, gz, gx = adjoint(ctx, w.xA, w.zetaA, w.areaA, w.dt, 3, 2, N.TC_J_PROBE, 17)
    x, z = w.xA.copy(), w.zetaA.copy()
    ctx.rk4_step(x, z, w.areaA, np.zeros((0, 3)), np.zeros((0, 3)), w.dt, 3)
    assert J == z[17]
    eps = 1e-6
    zp, zm = w.zetaA.copy(), w.zetaA.copy()
    zp[17] += eps
    zm[17] -= eps
    vals = []
    for zz in (zp, zm):
        x, z = w.xA.copy(), zz.copy()
        ctx.rk4_step(x, z, w.areaA, np.zeros((0, 3)), np.zeros((0, 3)), w.dt, 3)
        vals.append(z[17])
    assert abs((vals[0] - vals[1]) / (2 * eps) - gz[17]) <= 1e-6
    with pytest.raises(N.TcError):
        adjoint(ctx, w.xA, w.zetaA, w.areaA, w.dt, 3, 0)  # checkpoint interval 0
    c32 = Context(0, "fp32c")
    with pytest.raises(N.TcError) as e:
        adjoint(c32, w.xA, w.zetaA, w.areaA, w.dt, 3, 2)
    assert e.value.status == N.TC_ERR_STATE
    c32.close()
    ctx.close()


def test_trajectory_vjp_matches_torch_autograd_fp64(gpu):
    """tc_rk4_vjp with seeded random cotangents on both x(T) and zeta(T) against
    torch.autograd.grad of the same RK4 map with those grad_outputs."""
    w = configs.gaussian(level=2, delta=0.02, dt=0.01)
    ctx = Context(0, "fp64")
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    nsteps, ckpt = 5, 2
    rng = np.random.default_rng(8)
    gTx = rng.standard_normal((w.nA, 3))
    gTz = rng.standard_normal(w.nA)
    x = torch.tensor(w.xA, requires_grad=True)
    z = torch.tensor(w.zetaA, requires_grad=True)
    xT, zT = torch_rk4_state(x, z, torch.tensor(w.areaA), w.omega, w.deltas[0] ** 2, w.dt, nsteps)
    gx_ref, gz_ref = torch.autograd.grad((xT, zT), (x, z), (torch.tensor(gTx), torch.tensor(gTz)))
    J_ref = float((xT.detach() * torch.tensor(gTx)).sum() + (zT.detach() * torch.tensor(gTz)).sum())
    J, gz, gx = np.zeros(1), np.zeros(w.nA), np.zeros((w.nA, 3))
    N.call("tc_rk4_vjp", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, w.dt, nsteps,
           ckpt, N.dptr(gTx), N.dptr(gTz), N.dptr(J), N.dptr(gz), N.dptr(gx))
    assert abs(J[0] - J_ref) <= 1e-12 * abs(J_ref)
    assert np.abs(gx - gx_ref.numpy()).max() <= 1e-10 * np.abs(gx_ref.numpy()).max()
    assert np.abs(gz - gz_ref.numpy()).max() <= 1e-10 * np.abs(gz_ref.numpy()).max()
    # the zeta-only cotangent equals the enstrophy adjoint's seed 2 zeta A: same gradient
    Jz, gz2, gx2 = np.zeros(1), np.zeros(w.nA), np.zeros((w.nA, 3))
    zfin = w.zetaA.copy()
    xfin = w.xA.copy()
    ctx.rk4_step(xfin, zfin, w.areaA, np.zeros((0, 3)), np.zeros((0, 3)), w.dt, nsteps)
    seed = 2.0 * zfin * w.areaA
    N.call("tc_rk4_vjp", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, w.dt, nsteps,
           ckpt, None, N.dptr(seed), N.dptr(Jz), N.dptr(gz2), N.dptr(gx2))
    Je, gze, gxe = adjoint(ctx, w.xA, w.zetaA, w.areaA, w.dt, nsteps, ckpt)
    assert np.abs(gz2 - gze).max() <= 1e-12 * np.abs(gze).max()
    assert np.abs(gx2 - gxe).max() <= 1e-12 * np.abs(gze).max()
    with pytest.raises(N.TcError):
        N.call("tc_rk4_vjp", ctx.handle, N.dptr(w.xA), N.dptr(w.zetaA), N.dptr(w.areaA), w.nA, w.dt,
               nsteps, ckpt, None, None, N.dptr(Jz), N.dptr(gz2), N.dptr(gx2))
    ctx.close()


def test_every_vjp_mode_gives_the_same_gradient(gpu):
    """The eight ways of visiting the pairs in a stage's vector-Jacobian product (two passes,
    fused column reductions, row passes with one to three rows per thread and one or two Newton
    steps) agree to rounding."""
    w = configs.gaussian(level=3, delta=0.02, dt=0.01)
    ctx = Context(0, "fp64")
    ctx.set_omega(w.omega)
    ctx.set_deltas(*w.deltas)
    res = {}
    for mode in range(8):
        N.call("tc_set_adjoint_mode", ctx.handle, mode)
        res[mode] = adjoint(ctx, w.xA, w.zetaA, w.areaA, w.dt, 4, 2, N.TC_J_PROBE, 100)
    ref = res[0]
    scale = max(np.abs(ref[1]).max(), np.abs(ref[2]).max())
    for mode, (J, gz, gx) in res.items():
        assert J == ref[0]
        assert max(np.abs(gz - ref[1]).max(), np.abs(gx - ref[2]).max()) <= 1e-12 * scale, mode
    with pytest.raises(N.TcError):
        N.call("tc_set_adjoint_mode", ctx.handle, 8)
    ctx.close()


def test_adjoint_is_the_gradient_of_the_reference_map(gpu):
    """Centred finite differences taken through the reference's own BVERK4 (its Fortran source run
    by oracle/f90: PanelVelocityParallel.f90:435-658, level 1, Rossby-Haurwitz initial condition,
    delta 0, three steps of dt 0.01; tests/golden/ref_fd_rh4_l1.npz) against the library's
    adjoint of the same J = sum zeta(T)^2 A: 8 vorticity and 8 tangent-position entries, within
    1e-6 of the largest gradient entry; J itself to 1e-12."""
    from pathlib import Path

    f = dict(np.load(Path(__file__).resolve().parent / "golden" / "ref_fd_rh4_l1.npz"))
    xA, zA, aA = f["xA"], f["zetaA"], f["areaA"]
    eps, dt, nsteps = float(f["eps"]), float(f["dt"]), int(f["steps"])
    ctx = Context(0, "fp64")
    ctx.set_omega(2 * np.pi)
    ctx.set_deltas(0.0, 0.0, 0.05)
    J, gz, gx = adjoint(ctx, xA, zA, aA, dt, nsteps, 2)
    ctx.close()
    assert abs(J - math.fsum(f["zeta_final"] ** 2 * aA)) <= 1e-12 * abs(J)
    scale = max(np.abs(gz).max(), np.abs(gx).max())
    for m, j in enumerate(f["picks"]):
        fp, fm = f["zeta_plus"][m], f["zeta_minus"][m]
        fd = math.fsum((fp - fm) * (fp + fm) * aA) / (2 * eps)
        g = gz[j] if m % 2 == 0 else gx[j].dot(f["tangents"][m])
        assert abs(fd - g) <= 1e-6 * scale, (m, j, fd, g)
