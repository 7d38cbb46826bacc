"""Central finite differences of the oracle energy (GradientUtils.testGradient,
modules/potential/src/main/java/ffx/potential/utils/GradientUtils.java:78-206:
step 1e-5 A, per-atom tolerance 1e-2 kcal/mol/A)."""
import numpy as np

from forcefieldx_b200.system import water_box, water_params
from oracle import binding as ob


def test_oracle_fd_gradient_water():
    s = water_box(6, 18.643, seed=11)
    p = water_params(18.643, vdw_cutoff=7.0, ewald_cutoff=7.0, pme_grid=(20, 20, 20))
    r = ob.energy(s, p)
    assert r["status"] == 0
    rng = np.random.default_rng(3)
    h = 1.0e-5
    for atom in rng.choice(s.n_atoms, 5, replace=False):
        for d in range(3):
            x = s.xyz.copy()
            x[atom, d] += h
            ep = ob.energy(s, p, xyz=x, gradient=False)["terms"][9]
            x[atom, d] -= 2 * h
            em = ob.energy(s, p, xyz=x, gradient=False)["terms"][9]
            assert abs((ep - em) / (2 * h) - r["grad"][atom, d]) < 1.0e-2
