"""Multi-material SIMP law, FP64 numpy (oracle; test infrastructure only).

Restates PenalizedMultiMaterial (MaterialModels.py:102-235) on an n_el x n_mat design:

  forward   (MaterialModels.py:146-178): c = clip(rho, void, 1), a = c^p, b = 1 - a,
            E = max(void, sum_m E_m a_m prod_{k != m} b_k);
            plain: E = clip(rho @ E_mat, void, 1)
  backward  (MaterialModels.py:180-205): dE/drho_j = p c_j^(p-1) (E_j prod_{k != j} b_k
            - sum_{m != j} E_m a_m prod_{k != m, j} b_k)   (the sum before its clip)
  con       (MaterialModels.py:207-218): without rho_mat, per material
            sum_e rho_em dg_e / vol <= mass_m; with rho_mat, one mass test
            sum_e (rho_e . rho_mat) dg_e / vol <= mass shared by every material
  ocP       (MaterialModels.py:220-228): rho sqrt(-df / dg) with NaN -> 0 (df > 0), all
            ones * 1e-3 when that is zero everywhere
  init      (MaterialModels.py:230-232): ones (n_el, n_mat)

The pinned values are the fixtures that tests/golden/make_golden.py generates by running
the reference class itself (multimaterial.npz).
"""
import numpy as np


class MultiMaterialLaw:
    def __init__(self, n_material=2, mass=((0.25,), (0.25,)), E_mat=((1.0,), (0.5,)), rho_mat=None, void=1e-6,
                 penalty=3.0):
        self.n = int(n_material)
        self.E_mat = np.asarray(E_mat, dtype=np.float64).reshape(-1)
        self.rho_mat = None if rho_mat is None else np.asarray(rho_mat, dtype=np.float64).reshape(-1)
        self.mass = np.asarray(mass, dtype=np.float64).reshape(-1)
        if self.rho_mat is not None:
            self.mass = self.mass[:1]
        self.void = float(void)
        self.penalty = float(penalty)

    def forward(self, rho, plain=False):
        rho = np.asarray(rho, dtype=np.float64).reshape(-1, self.n)
        if plain:
            return np.clip(rho @ self.E_mat, self.void, 1.0)
        c = np.clip(rho, self.void, 1.0)
        a = c ** self.penalty
        b = 1.0 - a
        E = np.zeros(rho.shape[0])
        for m in range(self.n):
            t = a[:, m].copy()
            for k in range(self.n):
                if k != m:
                    t *= b[:, k]
            E += t * self.E_mat[m]
        return np.maximum(E, self.void)

    def backward(self, rho):
        rho = np.asarray(rho, dtype=np.float64).reshape(-1, self.n)
        c = np.clip(rho, self.void, 1.0)
        a = c ** self.penalty
        b = 1.0 - a
        out = np.zeros_like(c)
        for j in range(self.n):
            dj = self.penalty * c[:, j] ** (self.penalty - 1.0)
            g = np.zeros(c.shape[0])
            for i in range(self.n):
                t = np.ones(c.shape[0])
                for k in range(self.n):
                    if k != j:
                        t *= a[:, k] if k == i else b[:, k]
                g += (dj if i == j else -dj) * t * self.E_mat[i]
            out[:, j] = g
        return out

    def con(self, rho, dg, vol):
        rho = np.asarray(rho, dtype=np.float64).reshape(-1, self.n)
        dg = np.asarray(dg, dtype=np.float64).reshape(-1, 1)
        if self.rho_mat is None:
            V = (rho * dg).sum(axis=0)
            return (V / vol - self.mass) <= 0
        V = ((rho * dg) @ self.rho_mat).sum()
        return np.ones(self.n, dtype=bool) * bool(V / vol <= self.mass[0])

    def ocp(self, df, dg, rho):
        rho = np.asarray(rho, dtype=np.float64).reshape(-1, self.n)
        df = np.asarray(df, dtype=np.float64).reshape(-1, self.n)
        dg = np.asarray(dg, dtype=np.float64).reshape(-1, 1)
        with np.errstate(invalid="ignore"):
            ocP = rho * np.nan_to_num(np.sqrt(-df / dg), nan=0)
        if np.abs(ocP).sum() == 0:
            ocP = np.ones_like(ocP) * 1e-3
        return ocP
