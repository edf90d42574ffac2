"""Eddy-viscosity SGS model selection (wmles/sgs.py:14-50).

``make_sgs(name, **kw)`` returns a descriptor; the model itself is evaluated per cell in
the CUDA stage kernel from the Green-Gauss velocity gradient g[i, j] = du_i/dx_j and the
filter width delta = V^(1/3):

* smagorinsky(Cs=0.16): nu_t = (Cs delta)^2 sqrt(2 S:S)                      (sgs.py:14-18)
* wale(Cw=0.325):       nu_t = (Cw delta)^2 (Sd:Sd)^1.5 / ((S:S)^2.5 + (Sd:Sd)^1.25 + 1e-30)
                                                                              (sgs.py:21-30)
* vreman(Cs=0.17):      nu_t = 2.5 Cs^2 sqrt(max(B_beta, 0) / (g:g + 1e-30))  (sgs.py:33-42)
* None / "none":        implicit LES, mu_t = 0                                 (sgs.py:46-47)
and mu_t = rho nu_t.
"""
from dataclasses import dataclass

SGS_IDS = {"none": 0, "smagorinsky": 1, "wale": 2, "vreman": 3}
_DEFAULTS = {"smagorinsky": ("Cs", 0.16), "wale": ("Cw", 0.325), "vreman": ("Cs", 0.17)}


@dataclass(frozen=True)
class SGSModel:
    name: str
    coeff: float

    @property
    def model_id(self):
        return SGS_IDS[self.name]


def make_sgs(name="vreman", **kw):
    if isinstance(name, SGSModel):
        return name
    if name in (None, "none"):
        return SGSModel("none", 0.0)
    if name not in _DEFAULTS:
        raise KeyError(name)
    key, default = _DEFAULTS[name]
    extra = set(kw) - {key}
    if extra:
        raise TypeError(f"{name}() got unexpected keyword arguments {sorted(extra)}")
    return SGSModel(name, float(kw.get(key, default)))
