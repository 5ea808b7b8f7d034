"""Why BiCGSTAB parity is asserted on tightly converged fields: the
reference's own trajectory amplifies ulp-level differences (measured here
with the bit-faithful oracle, CPU only)."""
import numpy as np

from oracle import oracle as O
from tests.golden import make_golden as MG


def test_bicgstab_amplifies_ulp_perturbations_but_converged_fields_agree():
    w = MG.solve_case()
    g = O.Grid(*w.shape, *w.d, w.k0)
    G = O.green(g)
    e = O.incident(g, w.theta, w.phi, w.psi)
    x0, s0, _ = O.solve(g, G, w.eps, w.flags, e, "bicgstab", 1e-8)
    shifts = []
    for seed in range(3):
        rng = np.random.default_rng(seed)
        ep = e * (1 + 1e-16 * rng.standard_normal(e.shape))
        assert np.abs(ep - e).max() < 5e-16 * np.abs(e).max()  # one ulp in re and im
        _, s, _ = O.solve(g, G, w.eps, w.flags, ep, "bicgstab", 1e-8)
        shifts.append(s - s0)
    assert max(abs(s) for s in shifts) >= 2   # the step count is not stable to +-1
    # ... but tightly converged fields agree to the tolerance
    xa, _, _ = O.solve(g, G, w.eps, w.flags, e, "bicgstab", 1e-12)
    rng = np.random.default_rng(0)
    xb, _, _ = O.solve(g, G, w.eps, w.flags, e * (1 + 1e-16 * rng.standard_normal(e.shape)), "bicgstab", 1e-12)
    assert np.linalg.norm(xa - xb) / np.linalg.norm(xa) < 1e-11
