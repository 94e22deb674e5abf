"""Coarse-graining of a fine-mesh state onto a coarser hexagon mesh (no reference
counterpart; it produces the closure's training data and its error reference).

  h: area-weighted average of the fine cells whose generator lies nearest to the coarse
     generator (each fine cell belongs to exactly one coarse cell).
  u: the normal component n_e . v of the fine velocity rebuilt at the fine generators by
     Perot's formula v_i = (1/A_i) sum_e s_{e,i} l_e u_e (x_e - x_i), inverse-distance
     averaged over the 3 generators nearest the coarse edge point; then the curl-free
     correction G phi (G the TRiSK gradient (phi_r - phi_l) / d_e, whose discrete curl is
     zero, so the vorticity is untouched) for which the coarse divergence equals the
     area-weighted mean of the fine divergence (less its area-weighted global mean, which
     a coarse divergence cannot have; it is zero up to the cells' area mismatch). Interpolation alone leaves a divergence
     made mostly of noise at the scale of the coarse cells; the correction removes it.

The maps are linear: sparse matrices built once, and the symmetric positive semidefinite
system for phi, A D G = -S^T diag(l/d) S (S the signed cell incidence of the edges), solved
by conjugate gradients. The state is [u; h] in file numbering, as everywhere else.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.spatial import cKDTree


class CoarseGrainer:
    def __init__(self, fine, coarse, neighbours: int = 3):
        self.fine, self.coarse = fine, coarse
        # cells: fine cell -> nearest coarse generator
        owner = cKDTree(coarse.centers).query(fine.centers)[1]
        A = fine.cell_areas
        tot = np.bincount(owner, weights=A, minlength=coarse.nc)
        self.Rh = sp.csr_matrix((A / tot[owner], (owner, np.arange(fine.nc))), shape=(coarse.nc, fine.nc))
        self._torch = None
        # Perot reconstruction at the fine generators: V (3 nc_f x ne_f)
        cw = fine.cell_edges.shape[1]
        ce = fine.cell_edges - 1
        s = fine.cell_signs
        x = fine.centers
        rows, cols, vals = [], [], []
        for k in range(cw):
            e = ce[:, k]
            w = s[:, k] * fine.primal_lengths[e] / A
            d = fine.edge_points[e] - x
            d -= np.einsum("ij,ij->i", d, x)[:, None] * x  # tangent part
            for comp in range(3):
                rows.append(3 * np.arange(fine.nc) + comp)
                cols.append(e)
                vals.append(w * d[:, comp])
        V = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(3 * fine.nc, fine.ne))
        # coarse edge: inverse-distance average of the nearest fine generators, projected
        dist, idx = cKDTree(fine.centers).query(coarse.edge_points, k=neighbours)
        wts = 1.0 / np.maximum(dist, 1e-12)
        wts /= wts.sum(axis=1, keepdims=True)
        n = coarse.edge_normals
        rows, cols, vals = [], [], []
        for j in range(neighbours):
            for comp in range(3):
                rows.append(np.arange(coarse.ne))
                cols.append(3 * idx[:, j] + comp)
                vals.append(wts[:, j] * n[:, comp])
        P = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(coarse.ne, 3 * fine.nc))
        self.Ru = (P @ V).tocsr()
        # divergence correction: D = A^-1 S^T diag(l), G = -diag(1/d) S, A D G = -K
        c = coarse
        self.Df, self.Dc = _divergence_from_grid(fine), _divergence_from_grid(c)
        ec = c.edge_cells - 1
        S = sp.csr_matrix((np.r_[np.ones(c.ne), -np.ones(c.ne)],
                           (np.r_[np.arange(c.ne), np.arange(c.ne)], np.r_[ec[:, 0], ec[:, 1]])),
                          shape=(c.ne, c.nc))
        self.G = (-sp.diags(1.0 / c.dual_lengths) @ S).tocsr()
        self.K = (S.T @ sp.diags(c.primal_lengths / c.dual_lengths) @ S).tocsr()

    def __call__(self, y_fine: np.ndarray, divergence_fix: bool = True) -> np.ndarray:
        f, c = self.fine, self.coarse
        u_f = y_fine[:f.ne]
        u = self.Ru @ u_f
        if divergence_fix:
            r = self.Rh @ (self.Df @ u_f) - self.Dc @ u
            r -= (c.cell_areas @ r) / c.cell_areas.sum()  # sum A D u = 0 for every u
            b = c.cell_areas * r
            b -= b.mean()
            phi = _cg_numpy(self.K, b)
            u = u - self.G @ phi  # D G (-phi) = -A^-1 K (-phi) = A^-1 b
        return np.concatenate([u, self.Rh @ y_fine[f.ne:]])

    def torch_apply(self, Yf, divergence_fix: bool = True, iters: int = 4000, rtol: float = 1e-11):
        """Columns of Yf (fine states, (ne_f + nc_f) x k, CUDA float64) -> coarse states."""
        import torch
        if self._torch is None:
            def t(m):
                m = m.tocsr()
                return torch.sparse_csr_tensor(torch.from_numpy(m.indptr), torch.from_numpy(m.indices),
                                               torch.from_numpy(m.data), size=m.shape, dtype=torch.float64,
                                               device=Yf.device)
            self._torch = {"Ru": t(self.Ru), "Rh": t(self.Rh), "Df": t(self.Df), "Dc": t(self.Dc),
                           "G": t(self.G), "K": t(self.K),
                           "A": torch.from_numpy(self.coarse.cell_areas).to(Yf.device)}
        T = self._torch
        ne = self.fine.ne
        u = T["Ru"] @ Yf[:ne]
        if divergence_fix:
            A = T["A"][:, None]
            r = T["Rh"] @ (T["Df"] @ Yf[:ne]) - T["Dc"] @ u
            r = r - (A * r).sum(0, keepdim=True) / A.sum()
            b = A * r
            b = b - b.mean(0, keepdim=True)
            phi = _cg_torch(lambda p: T["K"] @ p, b, iters, rtol)
            u = u - T["G"] @ phi
        return torch.cat([u, T["Rh"] @ Yf[ne:]], dim=0)


def _divergence_from_grid(g) -> sp.csr_matrix:
    """(D F)_i = sum_k s_{k,i} l_e F_e / A_i over the cell's edges (TRiSKShallowWater.jl:112)."""
    ce = g.cell_edges - 1
    nc, cw = ce.shape
    vals = g.cell_signs * g.primal_lengths[ce] / g.cell_areas[:, None]
    rows = np.repeat(np.arange(nc), cw)
    return sp.csr_matrix((vals.ravel(), (rows, ce.ravel())), shape=(nc, g.ne))


def _cg_numpy(K, b, iters: int = 4000, rtol: float = 1e-11):
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rs = r @ r
    rs0 = max(rs, 1e-300)
    for _ in range(iters):
        Ap = K @ p
        alpha = rs / max(p @ Ap, 1e-300)
        x += alpha * p
        r -= alpha * Ap
        rs_new = r @ r
        if np.sqrt(rs_new / rs0) < rtol:
            break
        p = r + (rs_new / max(rs, 1e-300)) * p
        rs = rs_new
    return x


def _cg_torch(apply, b, iters, rtol):
    """Batched conjugate gradients for a symmetric positive semidefinite operator on the
    columns of b (each column's right side orthogonal to the null space)."""
    x = b.new_zeros(b.shape)
    r = b.clone()
    p = r.clone()
    rs = (r * r).sum(0)
    rs0 = rs.clone().clamp_min(1e-300)
    for _ in range(iters):
        Ap = apply(p)
        alpha = rs / (p * Ap).sum(0).clamp_min(1e-300)
        x += alpha * p
        r -= alpha * Ap
        rs_new = (r * r).sum(0)
        if float((rs_new / rs0).max().sqrt()) < rtol:
            break
        p = r + (rs_new / rs.clamp_min(1e-300)) * p
        rs = rs_new
    return x


def divergence_matrix(coeffs: dict) -> sp.csr_matrix:
    """D with (D F)_i = sum_k divergence[i, k] F[cell_edges[i, k]] (the continuity equation
    is dh/dt = -D F, TRiSKShallowWater.jl:298-305)."""
    ce = coeffs["cell_edges"] - 1
    nc, cw = ce.shape
    rows = np.repeat(np.arange(nc), cw)
    return sp.csr_matrix((coeffs["divergence"].ravel(), (rows, ce.ravel())), shape=(nc, coeffs["ne"]))


def relative_vorticity_matrix(coeffs: dict) -> sp.csr_matrix:
    """zeta_v = sum_k curl[v, k] u[vertex_edges[v, k]] (TRiSKShallowWater.jl:421-426)."""
    ve = coeffs["vertex_edges"] - 1
    nv, vw = ve.shape
    rows = np.repeat(np.arange(nv), vw)
    return sp.csr_matrix((coeffs["curl"].ravel(), (rows, ve.ravel())), shape=(nv, coeffs["ne"]))


def edge_geometry(grid) -> np.ndarray:
    """The closure's 7 geometry inputs per edge (file order): l_e, d_e, the two generator
    distances, the edge point's z, and the z components of the normal and the tangent."""
    x, n = grid.edge_points, grid.edge_normals
    tangent = np.cross(x, n)
    return np.ascontiguousarray(np.stack([grid.primal_lengths, grid.dual_lengths, grid.cell_distances[:, 0],
                                          grid.cell_distances[:, 1], x[:, 2], n[:, 2], tangent[:, 2]],
                                         axis=1).astype(np.float32))
