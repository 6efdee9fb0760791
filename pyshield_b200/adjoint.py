"""Adjoint of the microphysics step: vector-Jacobian products on the GPU.

pySHiELD has no adjoint. This module differentiates one
``Microphysics.__call__`` (``pySHiELD/stencils/microphysics.py:1981-2263``)
with the hand-written FP64 reverse kernel behind ``shield_mp_step_vjp``:

* ``step_vjp(mp, state, land, cot, timestep)``: the VJP of one step;
* ``MicrophysicsStep``: a ``torch.autograd.Function`` computing the step's
  outputs from its 14 inputs, whose backward is ``step_vjp``;
* ``rollout(mp, state, land, timestep, nsteps)``: a window of steps, each
  followed by the state update of ``update_physics_state_with_tendencies``
  (``pySHiELD/stencils/physics.py:151-194``). Autograd keeps only each
  step's input fields (per-step checkpointing); the adjoint kernel
  recomputes everything inside a step from them.

The inputs are the 13 state fields of ``MicrophysicsState`` and ``qaz``,
the persistent cloud-fraction accumulator (the reference's never-reset
``self._qaz``, ``microphysics.py:1674``): it carries from step to step, so
a window of steps is differentiated through it too. Fields are
``(nx, ny, nz)`` float64 CUDA tensors (any strides; level k = 0 at the
model top), the surface totals ``(nx, ny)``. The forward runs the plain
FP64 step with fresh zero tendencies, so its outputs are the step's
increments, the updated wmp and the updated accumulator (the handle's own
accumulator is set from the input and left at the output).
"""

import ctypes

from ._lib import (
    MP_STATE_FIELDS,
    MP_TENDENCY_FIELDS,
    SHIELD_MP_PLAIN,
    ShieldMpCotangents,
    ShieldMpFields,
    ShieldMpGradients,
    check,
    load,
)
from .microphysics import _current_stream
from .quantity import field2d, field3d

# pt qvapor qliquid qrain qice qsnow qgraupel qcld ua va delprsi delz wmp, and the accumulator
STATE = MP_STATE_FIELDS + ("qaz",)
OUT3 = MP_TENDENCY_FIELDS + ("wmp", "qaz")
OUT2 = ("rain", "snow", "ice", "graupel")
OUTPUTS = OUT3 + OUT2
# the fields update_physics_state_with_tendencies advances, with their tendency
ADVANCED = (("qvapor", "qv_dt"), ("qliquid", "ql_dt"), ("qrain", "qr_dt"), ("qice", "qi_dt"), ("qsnow", "qs_dt"),
            ("qgraupel", "qg_dt"), ("qcld", "qa_dt"), ("pt", "pt_dt"), ("ua", "udt"), ("va", "vdt"))


def _empty3(like):
    import torch

    nx, ny, nz = like.shape
    return torch.zeros((nz, ny, nx), dtype=torch.float64, device=like.device).permute(2, 1, 0)


def _check_state(mp, state):
    if len(state) != len(STATE):
        raise ValueError(f"expected the {len(STATE)} fields {STATE}")
    for name, t in zip(STATE, state):
        if tuple(t.shape) != (mp.nx, mp.ny, mp.nz):
            raise ValueError(f"{name}: shape {tuple(t.shape)} is not the domain {(mp.nx, mp.ny, mp.nz)}")


def _state_fields(mp, state, land):
    F = ShieldMpFields()
    ext = (mp.nx, mp.ny, mp.nz)
    for name, t in zip(MP_STATE_FIELDS, state):
        setattr(F, name, field3d(t, ext))
    F.land = field2d(land, (mp.nx, mp.ny))
    return F


def step_forward(mp, state, land, timestep, stream=None, tendencies=None):
    """Outputs of one step from the 14 inputs: the ten increments, the
    updated wmp and accumulator, and the four surface totals (mm/day).

    ``tendencies`` (dict of tendency name -> field, missing ones zero): the
    incoming tendencies the step adds its increments to, which the outputs
    then include; with ``de_ice`` the step reads ``qi_dt`` and rewrites
    ``qi_dt``, ``qs_dt``, qice and qsnow (state copies are used here)."""
    import torch

    _check_state(mp, state)
    mp.set_qaz(state[-1].permute(2, 1, 0).contiguous())
    F = _state_fields(mp, state, land)
    w_out = _empty3(state[0])
    w_out.copy_(state[STATE.index("wmp")])
    F.wmp = field3d(w_out, (mp.nx, mp.ny, mp.nz))
    tend = [_empty3(state[0]) for _ in MP_TENDENCY_FIELDS]
    for name, t in zip(MP_TENDENCY_FIELDS, tend):
        if tendencies is not None and tendencies.get(name) is not None:
            t.copy_(tendencies[name])
        setattr(F, name, field3d(t, (mp.nx, mp.ny, mp.nz)))
    if tendencies is not None:
        # de_ice writes the step's input qi and qs in place
        keep_q = []
        for name in ("qice", "qsnow"):
            q = _empty3(state[0])
            q.copy_(state[STATE.index(name)])
            keep_q.append(q)
            setattr(F, name, field3d(q, (mp.nx, mp.ny, mp.nz)))
    pr = torch.zeros((4, mp.ny, mp.nx), dtype=torch.float64, device=state[0].device)
    base, plane = pr.data_ptr(), mp.nx * mp.ny * 8
    F.rain, F.snow, F.ice, F.graupel = base, base + plane, base + 2 * plane, base + 3 * plane
    rc = load().shield_mp_step(mp._handle, ctypes.byref(F), float(timestep), SHIELD_MP_PLAIN,
                               ctypes.c_void_p(_current_stream(stream)))
    check(rc, mp._handle, "shield_mp_step")
    qaz = mp.get_qaz().permute(2, 1, 0)
    return tuple(tend) + (w_out, qaz) + tuple(pr[i].t() for i in range(4))


def step_vjp(mp, state, land, cot, timestep, stream=None, tendencies=None):
    """Input adjoints (14 fields, ``STATE`` order) of one step at ``state``
    for the output cotangents ``cot`` (``OUTPUTS`` order; None = zero).
    ``tendencies``: the incoming tendencies of the forward (``step_forward``);
    only de_ice reads one (``qi_dt``)."""
    _check_state(mp, state)
    if len(cot) != len(OUTPUTS):
        raise ValueError(f"expected {len(OUTPUTS)} cotangents {OUTPUTS}")
    ext = (mp.nx, mp.ny, mp.nz)
    F = _state_fields(mp, state, land)
    if tendencies is not None and tendencies.get("qi_dt") is not None:
        F.qi_dt = field3d(tendencies["qi_dt"], ext)
    C = ShieldMpCotangents()
    keep = []
    for name, c in zip(OUT3, cot[: len(OUT3)]):
        if c is None:
            continue  # a null field is a zero cotangent
        keep.append(c)
        setattr(C, name, field3d(c, ext))
    for name, c in zip(OUT2, cot[len(OUT3):]):
        if c is None:
            setattr(C, name, None)
            continue
        cc = c.t().contiguous()  # (ny, nx): column j * nx + i
        keep.append(cc)
        setattr(C, name, cc.data_ptr())
    G = ShieldMpGradients()
    grads = [_empty3(state[0]) for _ in STATE]
    for name, g in zip(STATE, grads):
        setattr(G, name, field3d(g, ext))
    rc = load().shield_mp_step_vjp(mp._handle, ctypes.byref(F), ctypes.byref(C), ctypes.byref(G), float(timestep),
                                   ctypes.c_void_p(_current_stream(stream)))
    check(rc, mp._handle, "shield_mp_step_vjp")
    del keep
    return tuple(grads)


try:
    import torch

    class MicrophysicsStep(torch.autograd.Function):
        """``outputs = MicrophysicsStep.apply(mp, timestep, land, *state)``:
        the 16 outputs (``OUTPUTS``) of one step of ``mp`` from its 14
        inputs (``STATE``); differentiable in every input."""

        @staticmethod
        def forward(ctx, mp, timestep, land, *state):
            outs = step_forward(mp, state, land, timestep)
            ctx.mp = mp
            ctx.timestep = timestep
            ctx.land = land
            ctx.save_for_backward(*state)
            return outs

        @staticmethod
        def backward(ctx, *gouts):
            state = ctx.saved_tensors
            grads = step_vjp(ctx.mp, state, ctx.land, gouts, ctx.timestep)
            return (None, None, None) + grads

except ImportError:  # pragma: no cover
    MicrophysicsStep = None


def step(mp, state, land, timestep):
    """Differentiable step: dict of the outputs from a dict of the inputs."""
    outs = MicrophysicsStep.apply(mp, timestep, land, *[state[n] for n in STATE])
    return dict(zip(OUTPUTS, outs))


def rollout(mp, state, land, timestep, nsteps):
    """``nsteps`` steps, each followed by X <- X + dt X_dt for the fields of
    ``ADVANCED``, and wmp, qaz <- the step's (delprsi, delz unchanged).
    Returns the final state dict and the list of per-step output dicts."""
    cur = dict(state)
    history = []
    for _ in range(nsteps):
        out = step(mp, cur, land, timestep)
        nxt = dict(cur)
        for x, xdt in ADVANCED:
            nxt[x] = cur[x] + out[xdt] * timestep
        nxt["wmp"] = out["wmp"]
        nxt["qaz"] = out["qaz"]
        history.append(out)
        cur = nxt
    return cur, history
