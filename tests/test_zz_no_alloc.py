"""The allocation-free step (shield_mp_step_noalloc) against the handle step.

shield_mp_step_noalloc serves hosts that may not allocate device memory: it
keeps the step's cloud-fraction accumulator in a fixed array inside the
library instead of a handle's buffer. Its results must match shield_mp_step's
on the same inputs, call after call. The second call matters: with do_qa
off, the qa_dt of a step depends on the accumulator the previous step left.

This file is collected last, so it runs both after the rest of the GPU suite
and (run on its own) as the first user of the array in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from golden_io import MP_TENDENCIES
from mp_helpers import TOL_PLAIN, assert_close, device_state, floors, read_state

FIELDS = MP_TENDENCIES + ("wmp", "qice", "qsnow", "rain", "snow", "ice", "graupel")


def _fields(ms, nx, ny, nz, precip):
    from pyshield_b200 import _lib
    from pyshield_b200.quantity import field2d, field3d

    F = _lib.ShieldMpFields()
    for name in _lib.MP_STATE_FIELDS + _lib.MP_TENDENCY_FIELDS:
        setattr(F, name, field3d(getattr(ms, name), (nx, ny, nz)))
    F.land = field2d(ms.land, (nx, ny))
    base, plane = precip.data_ptr(), nx * ny * 8
    F.rain, F.snow, F.ice, F.graupel = base, base + plane, base + 2 * plane, base + 3 * plane
    return F


def _last_error(lib):
    buf = ctypes.create_string_buffer(512)
    lib.shield_last_error(buf, 512)
    return buf.value.decode()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_noalloc_matches_handle_step(precision):
    import torch

    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200._lib import SHIELD_MP_MIXED, SHIELD_MP_PLAIN, load, make_config
    from pyshield_b200.inputs import make_state
    from pyshield_b200.microphysics import Microphysics
    from pyshield_b200.quantity import field2d

    nx, ny, nz, dt = 24, 16, 79, 225.0
    cfg = PhysicsConfig(dt_atmos=dt, mp_time=dt / 2, do_qa=False)
    state, area = make_state(nx * ny, nz, seed=11, n_cube=nx, sat_fraction=0.3)

    # the existing entry point, through its handle
    ms_h, sf, qf, gd = device_state(state, area, nx, ny)
    mp = Microphysics(sf, qf, gd, cfg, precision=precision)
    # the allocation-free entry point, on its own copy of the same state
    ms_n, _, _, gd_n = device_state(state, area, nx, ny)
    lib = load()
    c = make_config(cfg)
    precip = torch.zeros((4, ny, nx), dtype=torch.float64, device="cuda")
    F = _fields(ms_n, nx, ny, nz, precip)
    area2 = field2d(gd_n.area, (nx, ny))
    mode = SHIELD_MP_MIXED if precision == "mixed" else SHIELD_MP_PLAIN
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    for step in range(2):
        mp(ms_h, dt)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.shield_mp_step_noalloc(ctypes.byref(c), nx, ny, nz, area2, ctypes.byref(F), dt, mode, int(step == 0), stream)
        assert rc == 0, _last_error(lib)
        torch.cuda.synchronize()
        if step > 0:
            # after the first call's set-up, a call takes no device memory
            assert torch.cuda.mem_get_info()[0] == free_before

        ref = read_state(ms_h, nx, ny, nz)
        got = read_state(ms_n, nx, ny, nz)
        for i, p in enumerate(("rain", "snow", "ice", "graupel")):
            ref[p] = getattr(mp, p).t().contiguous().cpu().numpy().reshape(-1)
            got[p] = precip[i].contiguous().cpu().numpy().reshape(-1)
        assert np.any(ref["qa_dt"] != 0.0)
        assert_close(got, ref, FIELDS, TOL_PLAIN, ctx=f"noalloc/{precision}/call{step}", fl=floors(state, ref, dt))


def test_noalloc_rejects_oversized_domain():
    """A domain beyond the fixed scratch fails with SHIELD_ELAYOUT and a
    message naming the limit, before any device work."""
    from pyshield_b200 import _lib
    from pyshield_b200._config import PhysicsConfig

    lib = _lib.load()
    c = _lib.make_config(PhysicsConfig())
    F = _lib.ShieldMpFields()
    area = _lib.ShieldField2D()
    nx, ny, nz = 512, 64, 79  # 2.59 M cells > 2^21
    rc = lib.shield_mp_step_noalloc(ctypes.byref(c), nx, ny, nz, area, ctypes.byref(F), 225.0, 0, 1, None)
    assert rc == -2
    msg = _last_error(lib)
    assert "2097152" in msg and "shield_mp_step" in msg
