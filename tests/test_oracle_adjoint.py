"""The hand-written oracle adjoint against central finite differences of the oracle forward (CPU)."""
import numpy as np

from oracle import adjoint as oa
from oracle import extras as ox
from oracle import graph as og


def test_oracle_adjoint_matches_finite_differences():
    rng = np.random.default_rng(0)
    pts = rng.uniform(0, 1, (300, 2))
    g = og.build_graph(pts, n0=30, k=6)
    bins, vals = ox.matern_kernel(p=1, variance=1.0, cutoff=0.3, r_min=1e-4, r_max=3, n_bins=200, jitter=1e-4)
    xi, gv, gl = rng.standard_normal(300), rng.standard_normal(300), 0.7
    gx, gvals = oa.generate_vjp(g, (bins, vals), xi, gv, gl)
    h = 1e-6
    for _ in range(3):
        dx = rng.standard_normal(300)
        dv = rng.standard_normal(200) * 1e-2
        fp = oa.loss(g, (bins, vals + h * dv), xi + h * dx, gv, gl)
        fm = oa.loss(g, (bins, vals - h * dv), xi - h * dx, gv, gl)
        fd = (fp - fm) / (2 * h)
        assert abs(fd - (gx @ dx + gvals @ dv)) <= 1e-6 * abs(fd)
