"""FP64 discrete adjoint of the oracle time step (the adjoint oracle).

TEST INFRASTRUCTURE ONLY: imported by tests/, never by the product package.

The reference has no adjoint, so this is the only check of the library's
gradients besides finite differences. It differentiates the oracle's own
discrete step exactly:

* L_F and L_B, the stage right-hand sides without the source (interface
  coupling included), are linear in the state. Each is assembled as a sparse
  matrix by probing ``orc_rhs`` with coloured unit vectors: every output of the
  stencil depends on inputs at most 3 cells away in x and in the global row,
  so inputs of one field on a 7 x 7 lattice never share an output.
* The post-step interface filter is assembled the same way from ``orc_filter``.
* One step (reference src/pml_fs_kernels.cu:765-868, oracle ``step``) is
      k1 = L_d0 Y1 (+ src), Y1 = U;   Y2 = M(U + c0 k1);  acc = U + w0 k1
      k2 = L_d1 Y2;                   Y3 = M(U + c1 k2);  acc += w1 k2
      k3 = L_d0 Y3;                   Y4 = M(U + c2 k3);  acc += w2 k3
      k4 = L_d1 Y4;                   U' = F(M(acc + c3 k4) + (1 - M) U)
  with M the cells a stage updates, so its transpose is
      mu = F^T lam;  kb4 = c3 M mu;             Yb4 = L_d1^T kb4
      kb3 = M(w2 mu + c2 Yb4);                  Yb3 = L_d0^T kb3
      kb2 = M(w1 mu + c1 Yb3);                  Yb2 = L_d1^T kb2
      kb1 = M(w0 mu + c0 Yb2);                  Yb1 = L_d0^T kb1
      lam_prev = mu + M(Yb4 + Yb3 + Yb2) + Yb1
* The stage RHS is linear in each material coefficient of the output cell, so
  its derivative is the RHS evaluated with that coefficient set to 1 and every
  other one off (stiffness 0, density +inf: the oracle divides by rho), and
  the gradient of a coefficient is the sum over steps and stages of
  kb_s . L_d,m(Y_s) over the main fields of its cell, plus, on the interface
  row, the other medium's main fields of the same column (the coupling mixes
  them).
"""
from __future__ import annotations

import copy
import ctypes

import numpy as np
import scipy.sparse as sp

from . import pyoracle

# Field order of an oracle set (mfdm_oracle.cpp enum Field).
FIELDS = ["fvx", "fvz", "fp", "svx", "svz", "ssx", "ssz", "ssxz",
          "fxvx", "fxvz", "fxex", "fxez", "sxvx", "sxvz", "sxex", "sxez",
          "szvx", "szvz", "szex", "szez", "fzvx", "fzvz", "fzex", "fzez"]
FLUID = [f.startswith("f") for f in FIELDS]
MAIN = {"fluid": [0, 1, 2], "solid": [3, 4, 5, 6, 7]}
# coefficient -> (medium, basis arrays)
COEFS = ["K", "rf", "C11", "C13", "C33", "C55", "rs"]
MEDIUM = {"K": "fluid", "rf": "fluid", "C11": "solid", "C13": "solid", "C33": "solid",
          "C55": "solid", "rs": "solid"}

_dp = ctypes.POINTER(ctypes.c_double)


def _lib():
    lib = pyoracle.lib()
    if not hasattr(lib, "_adj_ready"):
        lib.orc_set_len.restype = ctypes.c_longlong
        lib.orc_set_len.argtypes = [ctypes.c_void_p]
        lib.orc_rhs.restype = ctypes.c_int
        lib.orc_rhs.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        lib.orc_filter.restype = ctypes.c_int
        lib.orc_filter.argtypes = [ctypes.c_void_p, _dp]
        lib.orc_get_state.restype = ctypes.c_int
        lib.orc_get_state.argtypes = [ctypes.c_void_p, _dp]
        lib.orc_set_state.restype = ctypes.c_int
        lib.orc_set_state.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int]
        lib.orc_step_save.restype = ctypes.c_int
        lib.orc_step_save.argtypes = [ctypes.c_void_p, _dp]
        lib._adj_ready = True
    return lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class _Handle:
    def __init__(self, model, precision=64, round_inputs=False):
        m, self._keep = pyoracle._model_struct(model, 0, round_inputs)
        self.h = _lib().orc_create(ctypes.byref(m), int(precision))
        if not self.h:
            raise RuntimeError("oracle create failed")
        self.n = int(_lib().orc_set_len(self.h))

    def rhs(self, d: int, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros(self.n)
        if _lib().orc_rhs(self.h, int(d), _p(x), _p(out)) != 0:
            raise RuntimeError("orc_rhs failed")
        return out

    def filter(self, x: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(x, dtype=np.float64).copy()
        if _lib().orc_filter(self.h, _p(y)) != 0:
            raise RuntimeError("orc_filter failed")
        return y

    def close(self):
        if self.h:
            _lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Layout:
    """Offsets of the packed oracle set and the global row of each array row."""

    def __init__(self, nx, nzf, nzs):
        self.nx, self.nzf, self.nzs = nx, nzf, nzs
        self.rows = [nzf if fl else nzs for fl in FLUID]
        self.g0 = [0 if fl else nzf - 1 for fl in FLUID]
        self.off = np.concatenate([[0], np.cumsum([r * nx for r in self.rows])]).astype(np.int64)
        self.n = int(self.off[-1])
        field = np.zeros(self.n, np.int64)
        for f in range(len(FIELDS)):
            field[self.off[f]:self.off[f + 1]] = f
        self.field = field
        loc = np.arange(self.n) - self.off[field]
        self.row = loc // nx
        self.col = loc % nx
        self.grow = self.row + np.asarray(self.g0)[field]

    def index(self, f, r, c):
        return self.off[f] + np.asarray(r) * self.nx + np.asarray(c)


def _lattice_offset(target, have):
    """Offset in [-3, 3] from `have` to the nearest value congruent to `target` mod 7."""
    return (np.mod(target - have, 7) + 3) % 7 - 3


def probe_operator(apply, lay: Layout, fields=None, radius_check=True):
    """Sparse matrix of the linear map `apply` (packed set -> packed set) by
    probing every input field on a 7 x 7 lattice of (global row, column)."""
    rows_i, cols_j, vals = [], [], []
    fields = range(len(FIELDS)) if fields is None else fields
    for f in fields:
        sel = np.arange(lay.off[f], lay.off[f + 1])
        for cz in range(7):
            for cx in range(7):
                pick = sel[(np.mod(lay.grow[sel], 7) == cz) & (np.mod(lay.col[sel], 7) == cx)]
                if pick.size == 0:
                    continue
                e = np.zeros(lay.n)
                e[pick] = 1.0
                out = apply(e)
                i = np.nonzero(out)[0]
                if i.size == 0:
                    continue
                gr = lay.grow[i] + _lattice_offset(cz, lay.grow[i])
                gc = lay.col[i] + _lattice_offset(cx, lay.col[i])
                r = gr - lay.g0[f]
                ok = (r >= 0) & (r < lay.rows[f]) & (gc >= 0) & (gc < lay.nx)
                if radius_check and not np.all(ok):
                    raise AssertionError(f"probe of field {FIELDS[f]} reached beyond radius 3")
                j = lay.index(f, r[ok], gc[ok])
                rows_i.append(i[ok])
                cols_j.append(j)
                vals.append(out[i[ok]])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows_i), np.concatenate(cols_j))),
                         shape=(lay.n, lay.n))


def _basis_model(model, coef):
    """Copy of `model` whose stage RHS is the derivative with respect to one
    material coefficient: that coefficient 1, stiffness 0, density +inf."""
    m = copy.deepcopy(model)
    fl = {k: np.asarray(v, dtype=np.float64).copy() for k, v in model.fluid.items()}
    so = {k: np.asarray(v, dtype=np.float64).copy() for k, v in model.solid.items()}
    fl["K"][:] = 0.0
    fl["rho"][:] = np.inf
    for k in ("C11", "C13", "C33", "C55"):
        so[k][:] = 0.0
    so["rho"][:] = np.inf
    if coef == "K":
        fl["K"][:] = 1.0
    elif coef == "rf":
        fl["rho"][:] = 1.0
    elif coef == "rs":
        so["rho"][:] = 1.0
    else:
        so[coef][:] = 1.0
    m.fluid, m.solid = fl, so
    return m


class OracleAdjoint:
    """FP64 forward, adjoint and gradient of the oracle step for one model (shot 0)."""

    def __init__(self, model, round_inputs=False):
        self.model = model
        self.round_inputs = round_inputs
        self.h = _Handle(model, 64, round_inputs)
        self.lay = Layout(model.nx, model.nz_f, model.nz_s)
        assert self.lay.n == self.h.n
        self.L = [probe_operator(lambda x, d=d: self.h.rhs(d, x), self.lay) for d in (0, 1)]
        self.F = self._filter_matrix()
        self.basis = {c: _Handle(_basis_model(model, c), 64, round_inputs) for c in COEFS}
        self.mask = self._stage_mask()
        dt = float(np.float32(model.dt))
        self.c = [dt / 2, dt / 2, dt, dt / 6]
        self.w = [dt / 6, dt / 3, dt / 3]
        self.gap = pyoracle.record_gap(model.dt)
        nx, lay = model.nx, self.lay
        cols = np.arange(nx)
        self.rec_idx = [lay.index(3, 0, cols), lay.index(4, 0, cols),
                        lay.index(2, model.nz_f - 1, cols)]  # svx, svz, fp

    def _filter_matrix(self):
        lay, nx, nzf = self.lay, self.lay.nx, self.lay.nzf
        iface = [(0, nzf - 1), (1, nzf - 1), (2, nzf - 1), (3, 0), (4, 0), (5, 0), (6, 0), (7, 0)]
        cols = np.arange(3, nx - 3)
        filt = np.concatenate([lay.index(f, r, cols) for f, r in iface])
        # F = identity off the filtered cells + the filter's own map into them
        keep = np.ones(lay.n)
        keep[filt] = 0.0
        rows_i, cols_j, vals = [], [], []
        for f, r in iface:
            for cx in range(7):
                cc = np.arange(nx)[np.arange(nx) % 7 == cx]
                e = np.zeros(lay.n)
                src = lay.index(f, r, cc)
                e[src] = 1.0
                out = self.h.filter(e)
                i = filt[out[filt] != 0.0]
                gc = lay.col[i] + _lattice_offset(cx, lay.col[i])
                ok = (gc >= 0) & (gc < nx)
                assert np.all(ok)
                rows_i.append(i)
                cols_j.append(lay.index(f, r, gc))
                vals.append(out[i])
        part = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows_i), np.concatenate(cols_j))),
                             shape=(lay.n, lay.n))
        return sp.diags(keep).tocsr() + part

    def _stage_mask(self):
        """Cells a stage updates (the oracle's live cells): every cell of the
        state fields, only the strip cells of the ADE fields."""
        lay, npd, nx = self.lay, self.model.npd, self.model.nx
        nzs, cpml = self.model.nz_s, getattr(self.model, "boundary_type", 2) == 1
        m = np.zeros(lay.n)
        f, r, c = lay.field, lay.row, lay.col
        main = f <= 7
        xstrip = (f >= 8) & (f <= 15) & (((c >= 3) & (c < 3 + npd)) | ((c >= nx - 3 - npd) & (c < nx - 3)))
        zstrip = (f >= 16) & (f <= 19) & (r >= nzs - 3 - npd)
        ftop = (f >= 20) & cpml & (r >= 3) & (r <= npd + 2)
        m[main | xstrip | zstrip | ftop] = 1.0
        return m

    # ---- forward -------------------------------------------------------------
    def forward(self, nsteps, save=True):
        """Runs from rest; returns records [ns][3][nx] (svx, svz, fp) and the
        stage inputs of every step (list of 4 packed sets) when `save`."""
        h = self.h
        n = self.lay.n
        zero = np.zeros(n)
        _lib().orc_set_state(h.h, _p(zero), 0)
        ns = -(-nsteps // self.gap)
        rec = np.zeros((ns, 3, self.model.nx))
        ys = []
        buf = np.zeros(4 * n)
        st = np.zeros(n)
        for it in range(nsteps):
            if _lib().orc_step_save(h.h, _p(buf)) != 0:
                raise RuntimeError("orc_step_save failed")
            if save:
                ys.append(buf.reshape(4, n).copy())
            if it % self.gap == 0:
                _lib().orc_get_state(h.h, _p(st))
                for q in range(3):
                    rec[it // self.gap, q] = st[self.rec_idx[q]]
        return rec, ys

    # ---- adjoint -------------------------------------------------------------
    def _grad_stage(self, g, d, kb, y):
        lay, nx, nzf = self.lay, self.model.nx, self.model.nz_f
        for cname, hb in self.basis.items():
            gm = hb.rhs(d, y) * kb
            med = MEDIUM[cname]
            own = MAIN[med]
            other = MAIN["solid" if med == "fluid" else "fluid"]
            acc = sum(gm[lay.off[f]:lay.off[f + 1]].reshape(lay.rows[f], nx) for f in own)
            # the coupling carries this medium's coefficient into the other
            # medium's interface row
            if med == "fluid":
                acc[nzf - 1] += sum(gm[lay.off[f]:lay.off[f] + nx] for f in other)
            else:
                acc[0] += sum(gm[lay.index(f, nzf - 1, 0):lay.index(f, nzf - 1, 0) + nx]
                              for f in other)
            g[cname] += acc

    def gradient(self, nsteps, residual, ys):
        """Gradients of sum_n residual[n] . rec[n] with respect to the seven
        coefficient arrays, given the stage inputs `ys` of the forward run."""
        lay, M = self.lay, self.mask
        c0, c1, c2, c3 = self.c
        w0, w1, w2 = self.w
        g = {cname: np.zeros((self.model.nz_f if MEDIUM[cname] == "fluid" else self.model.nz_s,
                              self.model.nx)) for cname in COEFS}
        lam = np.zeros(lay.n)
        LT = [L.T.tocsr() for L in self.L]
        FT = self.F.T.tocsr()
        for n in range(nsteps - 1, -1, -1):
            if n % self.gap == 0:
                for q in range(3):
                    lam[self.rec_idx[q]] += residual[n // self.gap, q]
            d0 = 1 if (n & 1) else 0
            d1 = 1 - d0
            mu = FT @ lam
            a = M * mu
            kb = c3 * a
            self._grad_stage(g, d1, kb, ys[n][3])
            y = LT[d1] @ kb
            new = mu + M * y
            kb = M * (w2 * a + c2 * y)
            self._grad_stage(g, d0, kb, ys[n][2])
            y = LT[d0] @ kb
            new += M * y
            kb = M * (w1 * a + c1 * y)
            self._grad_stage(g, d1, kb, ys[n][1])
            y = LT[d1] @ kb
            new += M * y
            kb = M * (w0 * a + c0 * y)
            self._grad_stage(g, d0, kb, ys[n][0])
            y = LT[d0] @ kb
            new += y
            lam = new
        return g

    def close(self):
        self.h.close()
        for hb in self.basis.values():
            hb.close()


# ---- parameterisation: vp, vs, rho ----------------------------------------------

def params_of(model):
    """(vp, vs, rho) of the solid and (vp, rho) of the fluid, FP64, from C11, C55, rho, K."""
    rs = np.asarray(model.solid["rho"], np.float64)
    vp = np.sqrt(np.asarray(model.solid["C11"], np.float64) / rs)
    vs = np.sqrt(np.asarray(model.solid["C55"], np.float64) / rs)
    rf = np.asarray(model.fluid["rho"], np.float64)
    vpf = np.sqrt(np.asarray(model.fluid["K"], np.float64) / rf)
    return {"vp": vp, "vs": vs, "rho": rs, "vp_f": vpf, "rho_f": rf}


def with_params(model, p):
    """Copy of `model` with isotropic coefficients built from the parameters."""
    m = copy.deepcopy(model)
    vp, vs, rho = p["vp"], p["vs"], p["rho"]
    mu = rho * vs ** 2
    lam = rho * (vp ** 2 - 2.0 * vs ** 2)
    m.solid = {"C11": lam + 2 * mu, "C13": lam, "C33": lam + 2 * mu, "C55": mu, "rho": rho.copy()}
    m.fluid = {"K": p["rho_f"] * p["vp_f"] ** 2, "rho": p["rho_f"].copy()}
    return m


def chain_rule(gc, p):
    """Coefficient gradients (C11, C13, C33, C55, rs = 1/rho_s, K, rf = 1/rho_f)
    to (vp, vs, rho) of the solid and (vp, rho) of the fluid."""
    vp, vs, rho = p["vp"], p["vs"], p["rho"]
    gsum = gc["C11"] + gc["C33"] + gc["C13"]
    out = {"vp": 2 * rho * vp * gsum,
           "vs": 2 * rho * vs * (gc["C55"] - 2 * gc["C13"]),
           "rho": vp ** 2 * gsum - 2 * vs ** 2 * gc["C13"] + vs ** 2 * gc["C55"] - gc["rs"] / rho ** 2}
    vpf, rf = p["vp_f"], p["rho_f"]
    out["vp_f"] = 2 * rf * vpf * gc["K"]
    out["rho_f"] = vpf ** 2 * gc["K"] - gc["rf"] / rf ** 2
    return out


def misfit(rec, obs):
    """L2 misfit on the pressure and velocity records, and its residual."""
    r = rec - obs
    return 0.5 * float(np.sum(r * r)), r
