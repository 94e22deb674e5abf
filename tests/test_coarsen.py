"""Coarse-graining for the closure's training data (CPU): a smooth velocity field survives
it to the interpolation error, the corrected coarse divergence equals the area-weighted
mean of the fine divergence, the correction leaves the coarse vorticity alone, and h is
averaged with the fine cell areas."""
import numpy as np

from dmplex_b200 import closure_pipeline as cp
from dmplex_b200.coarsen import CoarseGrainer, relative_vorticity_matrix


def _normal(g, field):
    return np.einsum("ij,ij->i", field(g.edge_points), g.edge_normals)


def _solid(x):
    return np.cross(np.array([0.3, -0.2, 1.0]), x)


def _potential(x):  # tangential gradient of a . x
    a = np.array([1.0, 0.5, -0.3])
    return a - (x @ a)[:, None] * x


def test_coarse_graining_smooth_fields():
    from dmplex_b200 import model_tables
    gf, gc = cp._grid(5), cp._grid(3)
    c = CoarseGrainer(gf, gc)
    Z = relative_vorticity_matrix(model_tables(gc, pv_flux="trisk", kinetic_energy="cell"))
    for field in (_solid, _potential):
        yf = np.r_[_normal(gf, field), np.ones(gf.nc)]
        plain, fixed = c(yf, divergence_fix=False), c(yf)
        exact = _normal(gc, field)
        uc = fixed[:gc.ne]
        assert np.linalg.norm(uc - exact) <= 5e-3 * np.linalg.norm(exact)
        # coarse divergence = area-weighted mean of the fine divergence, less its global
        # area-weighted mean
        target = c.Rh @ (c.Df @ yf[:gf.ne])
        target -= (gc.cell_areas @ target) / gc.cell_areas.sum()
        mism = c.Dc @ uc - target
        scale = max(np.abs(target).max(), np.abs(c.Dc @ exact).max(), np.abs(exact).max() / gc.dual_lengths.max())
        assert np.abs(mism).max() <= 1e-9 * scale
        # the correction is curl-free: vorticity unchanged
        dz = Z @ (uc - plain[:gc.ne])
        assert np.abs(dz).max() <= 1e-10 * max(np.abs(Z @ plain[:gc.ne]).max(), np.abs(Z @ exact).max())
        assert np.allclose(fixed[gc.ne:], 1.0, rtol=0, atol=1e-14)
    # h: area weights sum to one per coarse cell and every fine cell has one owner
    assert np.allclose(np.asarray(c.Rh.sum(axis=1)).ravel(), 1.0, atol=1e-14)
    assert np.array_equal(np.diff(c.Rh.tocsc().indptr), np.ones(gf.nc, dtype=np.int64))
