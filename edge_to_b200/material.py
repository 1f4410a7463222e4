"""SIMP material law, drop-in for SingleMaterial (MaterialModels.py:3-99).

Works on torch tensors (the GPU arrays of this package) and on numpy arrays; the
``np=`` keyword of the reference is accepted and ignored.  The "void" bound is a clip,
E = clip(rho^p, void, 1), not Emin + rho^p (E0 - Emin): E0 lives in the element matrix.
"""
import numpy as np
import torch


def _clip(x, lo, hi):
    if isinstance(x, torch.Tensor):
        return torch.clamp(x, lo, hi)
    return np.clip(x, lo, hi)


class MaterialModel:
    def __init__(self, E=1.0, nu=0.33, n_sets=1):
        self.E = E
        self.nu = nu
        self.n_sets = n_sets

    def __call__(self, rho, iteration, **kwargs):
        return self.__forward__(rho, iteration, **kwargs)

    def evaluate_constraint(self, rho, dg, vol, **kwargs):
        return self.__con__(rho, dg, vol, **kwargs)

    def ocP(self, df, dg, rho, **kwargs):
        return self.__ocP__(df, dg, rho, **kwargs)

    def base_properties(self):
        return {"E": self.E, "nu": self.nu, "n_sets": self.n_sets}

    def grad(self, rho, iteration, **kwargs):
        return self.__backward__(rho, iteration, **kwargs)

    def is_terminal(self, iteration):
        return True

    def init_desvars(self, nel, **kwargs):
        return self.__initvars__(nel, **kwargs)


class SingleMaterial(MaterialModel):
    def __init__(self, E=1.0, nu=0.33, void=1e-6, penalty=3.0, volume_fraction=0.25, penalty_schedule=None):
        super().__init__(E=E, nu=nu, n_sets=1)
        self.void = void
        self.penalty = penalty
        self.volume_fraction = volume_fraction
        self.penalty_schedule = penalty_schedule

    def current_penalty(self, iteration):
        if self.penalty_schedule is not None:
            return self.penalty_schedule(self.penalty, iteration)
        return self.penalty

    def __forward__(self, rho, iteration, plain=False, np=None):
        if plain:
            return _clip(rho, self.void, 1.0)
        return _clip(rho ** self.current_penalty(iteration), self.void, 1.0)

    def __backward__(self, rho, iteration, np=None):
        pen = self.current_penalty(iteration)
        return pen * _clip(rho, self.void, 1.0) ** (pen - 1)

    def __con__(self, rho, dg, vol, np=None):
        if isinstance(rho, torch.Tensor):
            dgs = torch.as_tensor(dg, dtype=rho.dtype, device=rho.device).squeeze()
            V = (rho.squeeze() * dgs).sum()
            return torch.tensor([bool(V / vol <= self.volume_fraction)], device=rho.device)
        V = (rho.squeeze() * np_squeeze(dg)).sum()
        return __import__("numpy").array([V / vol <= self.volume_fraction])

    def __ocP__(self, df, dg, rho, np=None):
        if isinstance(rho, torch.Tensor):
            dgs = torch.as_tensor(dg, dtype=rho.dtype, device=rho.device).reshape(-1, 1)
            ocP = rho * torch.nan_to_num(torch.sqrt(torch.clamp(-df / dgs, min=0)), nan=0.0)
            if torch.abs(ocP).sum() == 0:
                ocP = torch.ones_like(ocP) * 1e-3
            return ocP
        import numpy as _np
        ocP = rho * _np.nan_to_num(_np.sqrt(_np.maximum(-df / _np.asarray(dg).reshape(-1, 1), 0)), nan=0)
        if _np.abs(ocP).sum() == 0:
            ocP = _np.ones_like(ocP) * 1e-3
        return ocP

    def __initvars__(self, nel, np=None, dtype=None):
        return torch.ones(nel, dtype=torch.float64, device="cuda")

    def is_terminal(self, iteration):
        if self.penalty_schedule is not None:
            return self.penalty_schedule(self.penalty, iteration) == self.penalty
        return True


def np_squeeze(x):
    return np.asarray(x).squeeze()


def _dev(x):
    """FP64 CUDA tensor of x (numpy arrays are copied to the device)."""
    return torch.as_tensor(x, dtype=torch.float64).to("cuda")



class PenalizedMultiMaterial(MaterialModel):
    """Multi-material SIMP law, drop-in for PenalizedMultiMaterial (MaterialModels.py:102-235).

    The design is n_el x n_material (row-major, as in the reference).  With c = clip(rho,
    void, 1), a = c^p and b = 1 - a, the Young's modulus is E = max(void, sum_m E_m a_m
    prod_{k != m} b_k) and ``grad`` its derivative before the clip; ``plain=True`` gives
    clip(rho @ E_mat, void, 1).  Both run in the CUDA kernel behind edge_mm_law (up to 8
    materials).  The mass constraint is per material (``mass`` has one row per material) or,
    with ``rho_mat``, one shared test sum_e (rho_e . rho_mat) A_e / V <= mass.  ``__call__``
    returns E as an (n_el, 1) array like the reference; CuTopOpt flattens it.
    """

    def __init__(self, E=1.0, nu=0.33, n_material=2, mass=np.array([[0.25], [0.25]]),
                 E_mat=np.array([[1.0], [0.5]]), rho_mat=None, void=1e-6, penalty=3.0, penalty_schedule=None):
        super().__init__(E=E, nu=nu, n_sets=n_material)
        self.n_material = n_material
        self.mass = np.asarray(mass)
        self.E_mat = np.asarray(E_mat)
        self.rho_mat = None if rho_mat is None else np.asarray(rho_mat)
        self.void = void
        self.penalty = penalty
        self.penalty_schedule = penalty_schedule
        if self.E_mat.shape[0] != self.n_material:
            raise ValueError("E_mat must have the same number of materials as n_material")
        if not 1 <= self.n_material <= 8:
            raise ValueError("n_material must be between 1 and 8")
        if self.rho_mat is not None:
            if self.rho_mat.shape[0] != self.n_material:
                raise ValueError("rho_mat must have the same number of materials as n_material")
            if self.mass.shape[0] != 1:
                raise ValueError("if rho_mat is not None, mass must have only one value")
            self.mass = self.mass.flatten()[0]
        elif self.mass.shape[0] != self.n_material:
            raise ValueError("Mass and E_mat must have the same number of materials")

    def current_penalty(self, iteration):
        if self.penalty_schedule is not None:
            return self.penalty_schedule(self.penalty, iteration)
        return self.penalty

    def _law(self, rho, iteration, plain, want_grad):
        from . import _lib
        was_np = isinstance(rho, np.ndarray)
        r = torch.as_tensor(rho, dtype=torch.float64).to("cuda").reshape(-1, self.n_material).contiguous()
        n_el = r.shape[0]
        E = torch.empty(n_el, dtype=torch.float64, device="cuda")
        dE = torch.empty(n_el, self.n_material, dtype=torch.float64, device="cuda") if want_grad else None
        _lib.call("edge_mm_law", n_el, self.n_material, _lib.ptr(r),
                  _lib.double_array(self.E_mat.reshape(-1).astype(np.float64).tolist()), float(self.void),
                  float(self.current_penalty(iteration)), 1 if plain else 0, _lib.ptr(E),
                  _lib.ptr(dE) if want_grad else None, _lib.stream_ptr())
        out = dE if want_grad else E.reshape(-1, 1)
        return out.cpu().numpy() if was_np else out

    def __forward__(self, rho, iteration, plain=False, np=None):
        return self._law(rho, iteration, plain, False)

    def __backward__(self, rho, iteration, np=None):
        return self._law(rho, iteration, False, True)

    def __con__(self, rho, dg, vol, np=None):
        rho = _dev(rho)
        dgs = _dev(dg).reshape(-1, 1)
        r = rho.reshape(-1, self.n_material)
        if self.rho_mat is None:
            V = (r * dgs).sum(dim=0)
            mass = torch.as_tensor(self.mass.reshape(-1), dtype=rho.dtype, device=rho.device)
            return (V / vol - mass) <= 0
        rm = torch.as_tensor(self.rho_mat.reshape(-1), dtype=rho.dtype, device=rho.device)
        V = ((r * dgs) @ rm).sum()
        ok = bool(V / vol <= float(self.mass))
        return torch.full((self.n_material,), ok, dtype=torch.bool, device=rho.device)

    def __ocP__(self, df, dg, rho, np=None):
        was_np = not isinstance(rho, torch.Tensor)
        rho, df = _dev(rho), _dev(df)
        dgs = _dev(dg).reshape(-1, 1)
        ocP = rho * torch.nan_to_num(torch.sqrt(-df / dgs), nan=0.0)
        if torch.abs(ocP).sum() == 0:
            ocP = torch.ones_like(ocP) * 1e-3
        return ocP.cpu().numpy() if was_np else ocP

    def __initvars__(self, nel, np=None, dtype=None):
        return torch.ones(nel, self.n_material, dtype=torch.float64, device="cuda")

    def is_terminal(self, iteration):
        if self.penalty_schedule is not None:
            return self.penalty_schedule(self.penalty, iteration) == self.penalty
        return True
