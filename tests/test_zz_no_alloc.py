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
from mp_helpers import TOL_PLAIN, assert_close, device_state, gpu_floors as floors, read_state

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


def _noalloc_call(lib, c, nx, ny, nz, area2, F, dt, mode, first, stream):
    rc = lib.shield_mp_step_noalloc(ctypes.byref(c), nx, ny, nz, area2, ctypes.byref(F), dt, mode, int(first), stream)
    assert rc == 0, _last_error(lib)


def _compare(mp, ms_h, ms_n, precip, nx, ny, nz, state, dt, ctx):
    ref = read_state(ms_h, nx, ny, nz)
    got = read_state(ms_n, nx, ny, nz)
    for i, p in enumerate(("rain", "snow", "ice", "graupel")):
        ref[p] = getattr(mp, p).t().contiguous().cpu().numpy().reshape(-1)
        got[p] = precip[i].contiguous().cpu().numpy().reshape(-1)
    assert np.any(ref["qa_dt"] != 0.0)
    assert_close(got, ref, FIELDS, TOL_PLAIN, ctx=ctx, fl=floors(state, ref, dt))


def _pair(nx, ny, nz, dt, seed, precision):
    """A handle step and the allocation-free step's arguments on two copies
    of the same state."""
    import torch

    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200._lib import SHIELD_MP_MIXED, SHIELD_MP_PLAIN, load, make_config
    from pyshield_b200.inputs import make_state
    from pyshield_b200.microphysics import Microphysics
    from pyshield_b200.quantity import field2d

    cfg = PhysicsConfig(dt_atmos=dt, mp_time=dt / 2, do_qa=False)
    state, area = make_state(nx * ny, nz, seed=seed, n_cube=nx, sat_fraction=0.3)
    # the existing entry point, through its handle
    ms_h, sf, qf, gd = device_state(state, area, nx, ny)
    mp = Microphysics(sf, qf, gd, cfg, precision=precision)
    # the allocation-free entry point, on its own copy of the same state
    ms_n, _, _, gd_n = device_state(state, area, nx, ny)
    precip = torch.zeros((4, ny, nx), dtype=torch.float64, device="cuda")
    F = _fields(ms_n, nx, ny, nz, precip)
    area2 = field2d(gd_n.area, (nx, ny))
    mode = SHIELD_MP_MIXED if precision == "mixed" else SHIELD_MP_PLAIN
    return load(), make_config(cfg), state, mp, ms_h, ms_n, precip, F, area2, mode


@pytest.mark.gpu
@pytest.mark.parametrize("nz", [79, 127])
@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_noalloc_matches_handle_step(precision, nz):
    """Two calls in a row against the handle step (the second reads the
    accumulator the first left in the library's array)."""
    import torch

    nx, ny, dt = 24, 16, 225.0
    lib, c, state, mp, ms_h, ms_n, precip, F, area2, mode = _pair(nx, ny, nz, dt, 11, precision)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for step in range(2):
        mp(ms_h, dt)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _noalloc_call(lib, c, nx, ny, nz, area2, F, dt, mode, step == 0, stream)
        torch.cuda.synchronize()
        if step > 0:
            # after the first call's set-up, a call takes no device memory
            assert torch.cuda.mem_get_info()[0] == free_before
        _compare(mp, ms_h, ms_n, precip, nx, ny, nz, state, dt, f"noalloc/{precision}/L{nz}/call{step}")
    bad = ctypes.c_int64(0)
    assert lib.shield_mp_check_noalloc(nx, ctypes.byref(bad), stream) == 0, _last_error(lib)
    assert bad.value == -1


@pytest.mark.gpu
def test_noalloc_first_step_after_larger_domain():
    """A larger domain's calls leave its accumulator in the shared array; a
    smaller domain's first_step call must then start from zero, exactly as a
    fresh handle does."""
    import torch

    dt = 225.0
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib, c, _, _, _, _, _, Fb, area_b, mode = _pair(40, 30, 79, dt, 5, "plain")
    for step in range(2):
        _noalloc_call(lib, c, 40, 30, 79, area_b, Fb, dt, mode, step == 0, stream)
    nx, ny, nz = 12, 10, 79
    lib, c, state, mp, ms_h, ms_n, precip, F, area2, mode = _pair(nx, ny, nz, dt, 6, "plain")
    for step in range(2):
        mp(ms_h, dt)
        _noalloc_call(lib, c, nx, ny, nz, area2, F, dt, mode, step == 0, stream)
        torch.cuda.synchronize()
        _compare(mp, ms_h, ms_n, precip, nx, ny, nz, state, dt, f"noalloc/after-larger/call{step}")


@pytest.mark.gpu
def test_noalloc_reports_nonfinite_column():
    """A NaN planted on the host in one column's input is reported by
    shield_mp_check_noalloc with that column, and the record is cleared."""
    import torch

    nx, ny, nz, dt = 12, 6, 79, 225.0
    lib, c, _, _, _, ms_n, _, F, area2, mode = _pair(nx, ny, nz, dt, 3, "plain")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    i, j = 7, 2
    ms_n.pt.view[i, j, 30] = float("nan")
    _noalloc_call(lib, c, nx, ny, nz, area2, F, dt, mode, True, stream)
    bad = ctypes.c_int64(0)
    assert lib.shield_mp_check_noalloc(nx, ctypes.byref(bad), stream) == -4
    assert bad.value == i + nx * j
    assert f"i = {i}, j = {j}" in _last_error(lib)
    assert lib.shield_mp_check_noalloc(nx, ctypes.byref(bad), stream) == 0
    assert bad.value == -1


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
