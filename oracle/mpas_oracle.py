"""CPU oracle of the MPAS-Gassmann horizontal operators (test infrastructure, never shipped).

A numpy restatement of dmplex.jl's `slow_tendencies!` for flat ground and of the kernels it
launches, vectorised over entities and levels with every per-entity sum in the reference's
order (numpy does not contract to FMA):

    slow_tendencies!(m, ys, pressure)  src/Nonhydrostatic/MPAS/Gassmann/Stepping.jl:22-56
    diagnose_kernel!                   src/Nonhydrostatic/MPAS/Operators.jl:6-15
    vertex_kinetic_kernel!             Operators.jl:18-25
    cell_from_vertex_kernel!           Operators.jl:28-35
    w_kinetic_kernel!                  Operators.jl:38-41
    eta_kernel!                        Operators.jl:44-52
    edge_density_kernel!               Operators.jl:55-63
    w_tendency_vi_kernel!              Operators.jl:69-86
    vertex_pv_kernel!                  Operators.jl:88-102
    edge_pv_kernel!                    Operators.jl:104-115
    w_tendency_kernel!                 Operators.jl:118-133
    edge_w, vn_tendency_kernel!        src/Nonhydrostatic/MPAS/Gassmann/Tendencies.jl:4-12,38-75
    concorr_cell_kernel!               Operators.jl:136-145
    Rd, Cpd, Cvd, P0                   src/Nonhydrostatic/Common/Constants.jl:12-14

Fields are numpy arrays (nlev, n) / (nlev + 1, n): the memory of the reference's (n, nlev)
column-major arrays. ``MpasOracleC`` runs the same restatement in C with OpenMP
(oracle/mpas_oracle.c), bit for bit the same, for the timed CPU baseline. Tables are those of dmplex_b200.mpas.mpas_tables ((entity, k), 1-based;
``trisk`` and ``trisk_index`` edge-first as in the reference). Pinned by the reference's
own operator test (test/extruded.jl:54-106) in tests/test_mpas.py.
"""
from __future__ import annotations

import math

import numpy as np

_POW = np.frompyfunc(math.pow, 2, 1)

RD = 287.0
CPD = 1004.0
CVD = CPD - RD
P0 = 100000.0


class MpasOracle:
    def __init__(self, t: dict):
        self.t = t
        self.nc, self.ne, self.nv, self.nlev = t["nc"], t["ne"], t["nv"], t["nlev"]
        self.ce = t["cell_edges"] - 1
        self.ec = t["edge_cells"] - 1
        self.ev = t["edge_vertices"] - 1
        self.ve = t["vertex_edges"] - 1
        self.vc = t["vertex_cells"] - 1
        self.ti = t["trisk_index"].astype(np.int64) - 1            # (ne, nt, 3)
        self.vk = t.get("vk_weights") is not None
        if self.vk:
            self.kcv = t["vk_cell_vertices"] - 1

    # -- Operators.jl ------------------------------------------------------------------
    def diagnose(self, vn, rho, rhotheta):
        t = self.t
        K = np.zeros((self.nlev, self.nc))
        for j in range(self.ce.shape[1]):
            v = vn[:, self.ce[:, j]]
            K = K + t["kinetic"][:, j] * (v * v)
        theta = rhotheta / rho
        # the C library's pow, element by element (numpy's own vectorized pow differs from it
        # in the last bit for a few percent of the values)
        exner = _POW(RD * rhotheta / P0, RD / CVD).astype(np.float64)
        return theta, exner, K

    def vertex_kinetic(self, vn):
        Kv = np.zeros((self.nlev, self.nv))
        for j in range(self.ve.shape[1]):
            v = vn[:, self.ve[:, j]]
            Kv = Kv + self.t["vk_weights"][:, j] * (v * v)
        return Kv

    def cell_from_vertex(self, K, Kv):
        s = np.zeros_like(K)
        for j in range(self.kcv.shape[1]):
            s = s + self.t["vk_kites"][:, j] * Kv[:, self.kcv[:, j]]
        return K + s

    def w_kinetic(self, K, w):
        t = self.t
        dz, dzh = t["dz_cells"], t["dzh_cells"]
        return K + (dzh[:-1] * (w[:-1] * w[:-1]) + dzh[1:] * (w[1:] * w[1:])) / (4 * dz)

    def eta(self, vn, w):
        t = self.t
        l, r = self.ec[:, 0], self.ec[:, 1]
        out = np.zeros((self.nlev + 1, self.ne))
        j = slice(1, self.nlev)
        out[j] = (vn[1:] - vn[:-1]) / t["dzh_edges"][j] - (w[j][:, r] - w[j][:, l]) * t["inverse_dual"]
        return out

    def edge_density(self, vn, rho):
        ew = self.t["edge_weight"]
        r = ew[:, 0] * rho[:, self.ec[:, 0]] + ew[:, 1] * rho[:, self.ec[:, 1]]
        return r, r * vn

    def w_tendency_vi(self, eta, vn, rhoe, K, massweighted):
        t = self.t
        tw = np.zeros((self.nlev + 1, self.nc))
        wl = t["wlow"][1:self.nlev]
        s = np.zeros((self.nlev - 1, self.nc))
        for n in range(self.ce.shape[1]):
            e = self.ce[:, n]
            if massweighted:
                rl, ru = rhoe[:-1][:, e], rhoe[1:][:, e]
            else:
                rl = ru = np.ones((self.nlev - 1, self.nc))
            s = s + t["inner"][:, n] * eta[1:self.nlev][:, e] * (rl * vn[:-1][:, e] + ru * vn[1:][:, e]) / (
                2 * (wl * rl + (1 - wl) * ru))
        tw[1:self.nlev] = s - (K[1:] - K[:-1]) / t["dzh_cells"][1:self.nlev]
        return tw

    def vertex_pv(self, vn, rho):
        t = self.t
        z = np.zeros((self.nlev, self.nv))
        h = np.zeros((self.nlev, self.nv))
        for j in range(self.ve.shape[1]):
            z = z + t["curl"][:, j] * vn[:, self.ve[:, j]]
        for j in range(self.vc.shape[1]):
            h = h + t["vertex_weight"][:, j] * rho[:, self.vc[:, j]]
        return (z + t["coriolis"]) / h, z, h

    def edge_pv(self, qv, zv, rv):
        t = self.t
        v1, v2 = self.ev[:, 0], self.ev[:, 1]
        if t["iap_pv"]:
            rh = t["rhombus"]
            z = rh[:, 0] * zv[:, v1] + rh[:, 1] * zv[:, v2]
            h = rh[:, 0] * rv[:, v1] + rh[:, 1] * rv[:, v2]
            return (z + t["edge_coriolis"]) / h
        return (qv[:, v1] + qv[:, v2]) / 2

    def w_tendency(self, w, vn):
        t = self.t
        tw = np.zeros((self.nlev + 1, self.nc))
        s = np.zeros((self.nlev - 1, self.nc))
        for n in range(self.ce.shape[1]):
            e = self.ce[:, n]
            v = (vn[:-1][:, e] + vn[1:][:, e]) / 2
            l, r = self.ec[e, 0], self.ec[e, 1]
            wj = w[1:self.nlev]
            s = s + 2 * t["kinetic"][:, n] * v * (wj[:, r] - wj[:, l]) * t["inverse_dual"][e]
        dz = t["dz_cells"]
        wi = w[1:self.nlev]
        tw[1:self.nlev] = -s - wi * (w[2:] - w[:-2]) / (dz[:-1] + dz[1:])
        return tw

    def concorr_cell(self, vn, ddxn):
        s = np.zeros((self.nlev, self.nc))
        for n in range(self.ce.shape[1]):
            e = self.ce[:, n]
            s = s + self.t["inner"][:, n] * vn[:, e] * ddxn[:, e]
        return s

    # -- Tendencies.jl -----------------------------------------------------------------
    def _edge_w(self, w, rho, j, mw):
        """w~ at interface j (0-based, 1..nlev-1) of every edge."""
        t = self.t
        ew, wlow = t["edge_weight"], t["wlow"]
        l, r = self.ec[:, 0], self.ec[:, 1]
        if mw:
            hl = wlow[j][l] * rho[j - 1][l] + (1 - wlow[j][l]) * rho[j][l]
            hr = wlow[j][r] * rho[j - 1][r] + (1 - wlow[j][r]) * rho[j][r]
        else:
            hl = hr = np.ones(self.ne)
        M = ew[:, 0] * hl * w[j][l] + ew[:, 1] * hr * w[j][r]
        return M / (ew[:, 0] * hl + ew[:, 1] * hr)

    def vn_tendency(self, vn, Fs, w, rho, theta, exner, K, qe, eta, pressure):
        t = self.t
        nlev = self.nlev
        l, r = self.ec[:, 0], self.ec[:, 1]
        ew, invd = t["edge_weight"], t["inverse_dual"]
        s = np.zeros((nlev, self.ne))
        for j in range(self.ti.shape[1]):
            a, b, c = self.ti[:, j, 0], self.ti[:, j, 1], self.ti[:, j, 2]
            s = s + t["trisk"][:, j] * Fs[:, a] * (qe[:, b] + qe[:, c])
        te = ew[:, 0] * theta[:, l] + ew[:, 1] * theta[:, r]
        out = s - invd * (K[:, r] - K[:, l])
        if pressure > 0:
            dpi = (exner[:, r] - exner[:, l]) * invd
            out = out - pressure * (CPD * te * dpi)
        dz, dzh = t["dz_edges"], t["dzh_edges"]
        if t["vertical"] > 0:
            mw = t["vertical"] == 2
            W = np.zeros((nlev + 1, self.ne))
            for j in range(1, nlev):
                W[j] = self._edge_w(w, rho, j, mw)
            res = np.empty_like(out)
            for k in range(nlev):
                Wl = W[k] if k > 0 else 0.0
                Wu = W[k + 1] if k < nlev - 1 else 0.0
                res[k] = out[k] - (dzh[k] * eta[k] * Wl + dzh[k + 1] * eta[k + 1] * Wu) / (2 * dz[k])
            return res
        res = np.empty_like(out)
        for k in range(nlev):
            we = (w[k][l] + w[k][r] + w[k + 1][l] + w[k + 1][r]) / 4
            vlow = (vn[k - 1] + vn[k]) / 2 if k > 0 else vn[k]
            vup = (vn[k] + vn[k + 1]) / 2 if k < nlev - 1 else vn[k]
            res[k] = out[k] - we * (vup - vlow) / dz[k]
        return res

    def slow_tendencies(self, vn, w, rho, rhotheta, pressure=1.0) -> dict:
        """The work arrays slow_tendencies! fills, for flat ground (Stepping.jl:22-56)."""
        t = self.t
        theta, exner, K = self.diagnose(vn, rho, rhotheta)
        out = {"theta": theta, "exner": exner}
        if self.vk:
            Kv = self.vertex_kinetic(vn)
            K = self.cell_from_vertex(K, Kv)
            out["Kv"] = Kv
        qv, zv, rv = self.vertex_pv(vn, rho)
        qe = self.edge_pv(qv, zv, rv)
        rhoe, Fs = self.edge_density(vn, rho)
        eta = np.zeros((self.nlev + 1, self.ne))
        if t["vertical"] > 0:
            if not t["five_band"]:
                K = self.w_kinetic(K, w)
            eta = self.eta(vn, w)
            tw = self.w_tendency_vi(eta, vn, rhoe, K, t["vertical"] == 2)
            if t["five_band"]:
                K = self.w_kinetic(K, w)
        else:
            tw = self.w_tendency(w, vn)
        tvn = self.vn_tendency(vn, Fs, w, rho, theta, exner, K, qe, eta, pressure)
        out.update(K=K, qv=qv, zetav=zv, rhov=rv, qe=qe, rhoe=rhoe, Fs=Fs, eta=eta, tw=tw, tvn=tvn)
        return out


_TABLE_INDEX = ("cell_edges", "edge_cells", "edge_vertices", "vertex_edges", "vertex_cells", "vk_cell_vertices")
_TABLE_REAL = ("kinetic", "inner", "vk_kites", "edge_weight", "rhombus", "inverse_dual", "edge_coriolis", "curl",
               "vertex_weight", "vk_weights", "coriolis", "trisk", "dz_cells", "dzh_cells", "wlow", "dz_edges",
               "dzh_edges")
_FIELDS_OUT = ("theta", "exner", "K", "Kv", "qv", "zetav", "rhov", "qe", "rhoe", "Fs", "eta", "tvn", "tw", "Kh")


def _c_structs():
    import ctypes as C
    p = C.c_void_p

    class Tables(C.Structure):
        _fields_ = ([(n, C.c_int64) for n in ("nc", "ne", "nv", "nlev")]
                    + [(n, C.c_int32) for n in ("cw", "vw", "nt", "vk", "iap_pv", "vertical", "five_band", "reserved")]
                    + [(n, p) for n in _TABLE_INDEX + _TABLE_REAL + ("trisk_index",)])

    class Fields(C.Structure):
        _fields_ = [(n, p) for n in ("vn", "w", "rho", "rt", "theta", "exner", "K", "Kv", "qv", "zv", "rv", "qe",
                                     "rhoe", "Fs", "eta", "tvn", "tw", "Kh")]
    return Tables, Fields


class MpasOracleC:
    """slow_tendencies of MpasOracle in C with OpenMP on ``threads`` host threads."""

    def __init__(self, t: dict, threads: int = 1):
        import ctypes as C
        from oracle.oracle import _lib
        self.lib = _lib
        Tables, Fields = _c_structs()
        if _lib.mpas_oracle_tables_size() != C.sizeof(Tables) or _lib.mpas_oracle_fields_size() != C.sizeof(Fields):
            raise RuntimeError("oracle struct layout mismatch")
        self._Fields = Fields
        s = Tables()
        s.nc, s.ne, s.nv, s.nlev = t["nc"], t["ne"], t["nv"], t["nlev"]
        s.cw, s.vw, s.nt = t["cell_edges"].shape[1], t["vertex_edges"].shape[1], t["trisk"].shape[1]
        s.vk = int(t.get("vk_weights") is not None)
        s.iap_pv, s.vertical, s.five_band = int(bool(t["iap_pv"])), int(t["vertical"]), int(bool(t["five_band"]))
        self._keep = []
        for name in _TABLE_INDEX + _TABLE_REAL + ("trisk_index",):
            a = t.get(name)
            if a is None:
                continue
            dt = np.int64 if name in _TABLE_INDEX else (np.int32 if name == "trisk_index" else np.float64)
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            setattr(s, name, a.ctypes.data)
        self._s = s
        self.nc, self.ne, self.nv, self.nlev = t["nc"], t["ne"], t["nv"], t["nlev"]
        self.vk = bool(s.vk)
        self.threads = int(threads)

    def slow_tendencies(self, vn, w, rho, rhotheta, pressure=1.0) -> dict:
        import ctypes as C
        nc, ne, nv, nl = self.nc, self.ne, self.nv, self.nlev
        shapes = {"theta": (nl, nc), "exner": (nl, nc), "K": (nl, nc), "Kv": (nl, nv), "qv": (nl, nv),
                  "zetav": (nl, nv), "rhov": (nl, nv), "qe": (nl, ne), "rhoe": (nl, ne), "Fs": (nl, ne),
                  "eta": (nl + 1, ne), "tvn": (nl, ne), "tw": (nl + 1, nc), "Kh": (nl, nc)}
        out = {k: np.zeros(v) for k, v in shapes.items()}
        ins = [np.ascontiguousarray(x, dtype=np.float64) for x in (vn, w, rho, rhotheta)]
        f = self._Fields()
        for name, a in zip(("vn", "w", "rho", "rt"), ins):
            setattr(f, name, a.ctypes.data)
        for name, key in (("theta", "theta"), ("exner", "exner"), ("K", "K"), ("Kv", "Kv"), ("qv", "qv"),
                          ("zv", "zetav"), ("rv", "rhov"), ("qe", "qe"), ("rhoe", "rhoe"), ("Fs", "Fs"),
                          ("eta", "eta"), ("tvn", "tvn"), ("tw", "tw"), ("Kh", "Kh")):
            setattr(f, name, out[key].ctypes.data)
        self.lib.mpas_oracle_set_threads(self.threads)
        self.lib.mpas_oracle_slow_tendencies(C.byref(self._s), C.byref(f), C.c_double(pressure))
        del out["Kh"]
        if not self.vk:
            del out["Kv"]
        return out
