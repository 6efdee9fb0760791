"""The FP64 oracle run on torch tensors, for torch.autograd.

TEST INFRASTRUCTURE. ``torch_oracle_module()`` executes the source of
``oracle/microphysics.py`` with its ``np`` bound to a small dispatcher that
sends every array call of the step to torch (float64, CPU). The result is a
torch transcription of the microphysics step, operation for operation the
same program as the numpy oracle (which is pinned to the reference's own
source), that torch.autograd can differentiate.

The set-up constants (``setupm``, ``set_timestep``) are not differentiated:
``TorchOracle`` takes them from a numpy ``OracleMicrophysics`` and runs only
the step on torch tensors.

Forward-mode AD (``torch.autograd.forward_ad``) differentiates this program
as written: ``jvp_per_input`` gives J dx for one direction per input field.
Reverse mode does not run on it: the level sweeps write rows of arrays in
place, which the backward pass cannot replay (torch raises), and the
reference's masked divisions (``W(dqh > 0, x / dqh, 0)`` and the like) would
turn the zero cotangent of an unselected branch into 0 * inf = NaN.
"""
import contextlib
import importlib.util
import os
import sys
import types

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F64 = torch.float64


def _t(x):
    return x if isinstance(x, torch.Tensor) else torch.as_tensor(x, dtype=F64)


def _any_tensor(*xs):
    return any(isinstance(x, torch.Tensor) for x in xs)


class _TorchNumpy(types.SimpleNamespace):
    """The numpy names the oracle's step uses, dispatched to torch when an
    argument is a tensor (array constructors always build tensors)."""

    float64 = np.float64

    @staticmethod
    def _dtype(dtype):
        if dtype is bool or dtype is np.bool_:
            return torch.bool
        return F64

    def where(self, c, a, b):
        if not _any_tensor(c, a, b):
            return np.where(c, a, b)
        return torch.where(_t(c) if not isinstance(c, torch.Tensor) else c, _t(a), _t(b))

    # min, max and abs as selections: the same values as numpy's, and at a
    # tie the derivative of the first argument (|x| at 0: that of x), the
    # branch convention of the hand-written adjoints and of the dual numbers
    # (torch.minimum/maximum would split a tie's derivative in halves)
    def minimum(self, a, b):
        if not _any_tensor(a, b):
            return np.minimum(a, b)
        a, b = _t(a), _t(b)
        return torch.where(a <= b, a, b)

    def maximum(self, a, b):
        if not _any_tensor(a, b):
            return np.maximum(a, b)
        a, b = _t(a), _t(b)
        return torch.where(a >= b, a, b)

    def exp(self, x):
        return torch.exp(x) if isinstance(x, torch.Tensor) else np.exp(x)

    def log(self, x):
        return torch.log(x) if isinstance(x, torch.Tensor) else np.log(x)

    def sqrt(self, x):
        return torch.sqrt(x) if isinstance(x, torch.Tensor) else np.sqrt(x)

    def abs(self, x):
        return torch.where(x >= 0.0, x, -x) if isinstance(x, torch.Tensor) else np.abs(x)

    def arctan(self, x):
        return np.arctan(x)

    def array(self, x, *a, **k):
        return np.array(x, *a, **k)

    def asarray(self, x, dtype=None):
        if isinstance(x, torch.Tensor):
            return x.to(F64)
        return np.asarray(x, dtype=dtype)

    def broadcast_to(self, x, shape):
        return torch.broadcast_to(_t(x), tuple(shape))

    def zeros(self, shape, dtype=None):
        return torch.zeros(tuple(np.atleast_1d(shape)), dtype=self._dtype(dtype))

    def empty(self, shape, dtype=None):
        return torch.zeros(tuple(np.atleast_1d(shape)), dtype=self._dtype(dtype))

    def ones(self, shape, dtype=None):
        return torch.ones(tuple(np.atleast_1d(shape)), dtype=self._dtype(dtype))

    def full(self, shape, value, dtype=None):
        return torch.full(tuple(np.atleast_1d(shape)), float(value), dtype=self._dtype(dtype))

    @staticmethod
    def errstate(**_):
        return contextlib.nullcontext()


def _install_tensor_copy():
    # the oracle copies arrays with ``a.copy()``; on a tensor that is clone()
    if not hasattr(torch.Tensor, "copy"):
        torch.Tensor.copy = torch.Tensor.clone


_MODULE = None


def torch_oracle_module():
    """``oracle/microphysics.py`` executed with torch behind ``np``."""
    global _MODULE
    if _MODULE is not None:
        return _MODULE
    _install_tensor_copy()
    path = os.path.join(ROOT, "oracle", "microphysics.py")
    src = open(path).read()
    marker = "import numpy as np\n"
    assert src.count(marker) == 1
    src = src.replace(marker, "np = __torch_numpy__\n")
    spec = importlib.util.spec_from_loader("oracle_torch_microphysics", loader=None)
    mod = importlib.util.module_from_spec(spec)
    mod.__dict__["__torch_numpy__"] = _TorchNumpy()
    mod.__file__ = path
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    exec(compile(src, path, "exec"), mod.__dict__)
    _MODULE = mod
    return mod


class TorchOracle:
    """One microphysics step of the oracle on torch FP64 tensors.

    ``state`` maps the MicrophysicsState names to (L, n) tensors (``land``
    (n,)); ``qaz`` is the (L, n) accumulator at the step's start. Returns the
    step's outputs as a dict: the ten tendencies (from zero), ``wmp``,
    ``qaz`` and the four surface totals."""

    def __init__(self, cfg, ncol, nlev, area, timestep):
        from oracle.microphysics import OracleMicrophysics

        ref = OracleMicrophysics(cfg, ncol, nlev, area)
        ref._set_timestep(float(timestep))
        mod = torch_oracle_module()
        self.obj = mod.OracleMicrophysics.__new__(mod.OracleMicrophysics)
        self.obj.__dict__.update(ref.__dict__)
        self.obj.area = torch.as_tensor(np.asarray(area, dtype=np.float64).reshape(ncol))
        self.timestep = float(timestep)

    def __call__(self, state, qaz):
        s = {k: v.clone() for k, v in state.items()}
        for t in ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt"):
            s[t] = torch.zeros_like(state["pt"])
        self.obj.qaz = qaz.clone()
        pr = self.obj(s, self.timestep)
        out = {t: s[t] for t in ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt")}
        out["wmp"] = s["wmp"]
        out["qaz"] = self.obj.qaz
        out.update(pr)
        return out


STATE = ("pt", "qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qcld", "ua", "va", "delprsi", "delz",
         "wmp", "qaz")
OUTPUTS = ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt", "wmp", "qaz",
           "rain", "snow", "ice", "graupel")


def jvp_per_input(cfg, timestep, X, land, area, DX):
    """Forward-mode derivatives of one step, one direction per input field.

    X, DX: (14, L, n) arrays, rows in ``STATE`` order (the 13 state fields,
    then the accumulator); land, area: (n,). All 14 directions go through one
    forward-mode pass: the columns are independent, so the state is repeated
    14 times along the column axis and copy f carries direction DX[f] on
    input f alone. Returns (Y, T): Y[o] the outputs ((L, n) or (n,)), T[o][f]
    the tangent of output o along DX[f]."""
    import torch.autograd.forward_ad as fwAD

    nf, L, n = X.shape
    assert nf == len(STATE)
    Xr = np.tile(X, (1, 1, nf))
    Tr = np.zeros_like(Xr)
    for f in range(nf):
        Tr[f, :, f * n:(f + 1) * n] = DX[f]
    oracle = TorchOracle(cfg, nf * n, L, np.tile(area, nf), timestep)
    with fwAD.dual_level():
        state = {name: fwAD.make_dual(torch.as_tensor(Xr[i]), torch.as_tensor(Tr[i]))
                 for i, name in enumerate(STATE[:-1])}
        state["land"] = torch.as_tensor(np.tile(np.asarray(land, dtype=np.float64), nf))
        qaz = fwAD.make_dual(torch.as_tensor(Xr[-1]), torch.as_tensor(Tr[-1]))
        out = oracle(state, qaz)
        Y, T = {}, {}
        for o in OUTPUTS:
            primal, tangent = fwAD.unpack_dual(out[o])
            primal = primal.detach().numpy()
            tangent = np.zeros_like(primal) if tangent is None else tangent.detach().numpy()
            Y[o] = primal[..., :n].copy()
            T[o] = [tangent[..., f * n:(f + 1) * n].copy() for f in range(nf)]
    return Y, T
