"""Molecular dynamics on the device (velocity Verlet + SETTLE) through the C ABI.

1. The first steps against an independent host integrator: the same velocity Verlet
   (VelocityVerlet.java:73-120) with oracle forces, positions constrained by iterative
   SHAKE and velocities by solving the RATTLE conditions with numpy.  SETTLE is the
   analytical solution of the same constraint equations, so positions agree to rounding.
2. NVE: 200 steps of 1 fs for 216 rigid waters keep every O-H and H-H distance and
   conserve the total energy (the reference's DynamicsNVETest checks conservation the
   same way).
"""
import math

import numpy as np
import pytest

from forcefieldx_b200.energy import ForceFieldEnergy
from forcefieldx_b200.system import WATER_648, water_box, water_params
from oracle import binding as ob

pytestmark = pytest.mark.gpu

KCAL = 418.4                      # Constants.KCAL_TO_GRAM_ANG2_PER_PS2
ROH, THETA = 0.9572, math.radians(104.52)
RHH = 2.0 * ROH * math.sin(THETA / 2.0)
MO, MH = 15.999, 1.008


def _system(seed=4):
    s = water_box(WATER_648["n_side"], WATER_648["edge"], seed=seed)
    p = water_params(WATER_648["edge"], pme_grid=WATER_648["grid"])
    n = s.n_atoms
    mass = np.where(np.arange(n) % 3 == 0, MO, MH)
    settle = np.arange(n).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    kT = 0.0019872041 * 300.0
    vel = rng.normal(size=(n, 3)) * np.sqrt(kT * KCAL / mass)[:, None]
    return s, p, mass, settle, vel


def _shake(x0, x, mass, settle, tol=1e-13):
    """Iterative SHAKE on the three sides of every molecule (constraint forces along the
    prior sides)."""
    x = x.copy()
    pairs = [(0, 1, ROH), (0, 2, ROH), (1, 2, RHH)]
    for _ in range(500):
        worst = 0.0
        for a, b, d in pairs:
            ia, ib = settle[:, a], settle[:, b]
            r = x[ib] - x[ia]
            r0 = x0[ib] - x0[ia]
            diff = (r * r).sum(1) - d * d
            worst = max(worst, np.abs(diff).max() / (d * d))
            inva, invb = 1.0 / mass[ia], 1.0 / mass[ib]
            g = diff / (2.0 * (r * r0).sum(1) * (inva + invb))
            x[ia] += (g * inva)[:, None] * r0
            x[ib] -= (g * invb)[:, None] * r0
        if worst < tol:
            return x
    raise AssertionError("SHAKE did not converge")


def _rattle(x, v, mass, settle):
    v = v.copy()
    A, B, C = settle[:, 0], settle[:, 1], settle[:, 2]
    e = [x[B] - x[A], x[C] - x[B], x[A] - x[C]]
    e = [u / np.linalg.norm(u, axis=1)[:, None] for u in e]
    for w in range(settle.shape[0]):
        ia, ib, ic = A[w], B[w], C[w]
        eab, ebc, eca = e[0][w], e[1][w], e[2][w]
        iA, iB, iC = 1 / mass[ia], 1 / mass[ib], 1 / mass[ic]
        # Columns: response of the three side velocities to unit impulses t_AB, t_BC, t_CA.
        K = np.zeros((3, 3))
        for j, (p_, q_, u) in enumerate([(ia, ib, eab), (ib, ic, ebc), (ic, ia, eca)]):
            dv = {ia: np.zeros(3), ib: np.zeros(3), ic: np.zeros(3)}
            dv[p_] -= u / mass[p_]
            dv[q_] += u / mass[q_]
            K[0, j] = (dv[ib] - dv[ia]) @ eab
            K[1, j] = (dv[ic] - dv[ib]) @ ebc
            K[2, j] = (dv[ia] - dv[ic]) @ eca
        rhs = -np.array([(v[ib] - v[ia]) @ eab, (v[ic] - v[ib]) @ ebc, (v[ia] - v[ic]) @ eca])
        t = np.linalg.solve(K, rhs)
        v[ia] += iA * (-t[0] * eab + t[2] * eca)
        v[ib] += iB * (t[0] * eab - t[1] * ebc)
        v[ic] += iC * (t[1] * ebc - t[2] * eca)
    return v


def test_md_matches_host_integrator():
    s, p, mass, settle, vel = _system()
    dt, steps = 0.001, 3
    with ForceFieldEnergy(s, p) as ffe:
        ffe.md_setup(mass, settle, ROH, RHH)
        xg, vg, epg, ekg = ffe.md_run(s.xyz, vel, dt, steps)
    x, v = s.xyz.copy(), vel.copy()
    a = -KCAL * ob.energy(s, p, xyz=x)["grad"] / mass[:, None]
    for _ in range(steps):
        x0 = x.copy()
        v = v + 0.5 * dt * a
        x = _shake(x0, x + dt * v, mass, settle)
        v = (x - x0) / dt
        a = -KCAL * ob.energy(s, p, xyz=x)["grad"] / mass[:, None]
        v = _rattle(x, v + 0.5 * dt * a, mass, settle)
    assert np.abs(xg - x).max() < 1e-9, np.abs(xg - x).max()
    assert np.abs(vg - v).max() < 1e-6, np.abs(vg - v).max()


def test_md_nve_conserves_energy_and_geometry():
    s, p, mass, settle, vel = _system(seed=9)
    with ForceFieldEnergy(s, p) as ffe:
        ffe.md_setup(mass, settle, ROH, RHH)
        x, v, ep, ek = ffe.md_run(s.xyz, vel, 0.001, 200)
    roh = np.linalg.norm(x[settle[:, 1]] - x[settle[:, 0]], axis=1)
    roh2 = np.linalg.norm(x[settle[:, 2]] - x[settle[:, 0]], axis=1)
    rhh = np.linalg.norm(x[settle[:, 2]] - x[settle[:, 1]], axis=1)
    assert np.abs(roh - ROH).max() < 1e-9 and np.abs(roh2 - ROH).max() < 1e-9
    assert np.abs(rhh - RHH).max() < 1e-9
    # Relative velocities along the sides vanish.
    e = x[settle[:, 1]] - x[settle[:, 0]]
    vrel = ((v[settle[:, 1]] - v[settle[:, 0]]) * e).sum(1) / np.linalg.norm(e, axis=1)
    assert np.abs(vrel).max() < 1e-9
    etot = ep + ek
    drift = np.abs(etot - etot[0]).max()
    print(f"NVE 200 x 1 fs: E0={etot[0]:.4f} max|E-E0|={drift:.4f} kcal/mol, mean KE={ek.mean():.2f}")
    assert drift < 1e-3 * ek.mean() * 10, drift


def test_aspc_predictor_cuts_iterations_and_keeps_the_solution():
    """Along a smooth path of configurations the ASPC guess (after six stored solves)
    lowers the PCG iteration count; every result still agrees with the oracle's solve
    from the direct dipoles to the convergence tolerance."""
    s, p, mass, settle, vel = _system(seed=2)
    with ForceFieldEnergy(s, p) as ffe:
        ffe.md_setup(mass, settle, ROH, RHH)
        path = [s.xyz]
        x, v = s.xyz, vel
        for _ in range(9):
            x, v, _, _ = ffe.md_run(x, v, 0.001, 1)
            path.append(x)
    iters = {}
    for aspc in (False, True):
        with ForceFieldEnergy(s, p) as ffe:
            ffe.set_scf_predictor(aspc)
            iters[aspc] = []
            for k, x in enumerate(path):
                e, g = ffe.energy_and_gradient(x)
                iters[aspc].append(int(ffe.count("scf_iter")))
                if aspc and k >= 6:
                    ref = ob.energy(s, p, xyz=x)
                    assert abs(ffe.terms[2] - ref["terms"][2]) < 1e-6 * abs(ref["terms"][2])
                    assert float(np.sqrt(np.mean((g - ref["grad"]) ** 2))) < 1e-4
    print("PCG iterations without / with ASPC:", iters[False], iters[True])
    assert iters[True][:6] == iters[False][:6]
    assert sum(iters[True][6:]) < sum(iters[False][6:])
