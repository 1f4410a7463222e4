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
