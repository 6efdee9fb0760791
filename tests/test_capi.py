"""The C-ABI library: exports, host-side constants, behaviour without a GPU.
No compute call runs here."""
import ctypes
import os
import re

import numpy as np
import pytest

from pyshield_b200 import _lib
from pyshield_b200._config import PhysicsConfig

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "shield_mp.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^int\s+(shield_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.EXPORTS)


def test_config_struct_matches_header_field_order():
    src = open(HEADER).read()
    body = src[src.index("typedef struct {") : src.index("} ShieldMpConfig;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        m = re.match(r"(?:typedef struct \{)?\s*(double|int)\s+(.*)", decl, flags=re.S)
        if m:
            names += [x.strip() for x in m.group(2).split(",")]
    assert names == [n for n, _ in _lib._CFG_FIELDS]


@pytest.mark.parametrize("dt", [150.0, 180.0, 225.0, 450.0, 600.0])
@pytest.mark.parametrize("over", [{}, dict(fast_sat_adj=False, c_paut=0.55, rthresh=1e-5, tice=273.15)])
def test_host_constants_match_oracle(dt, over):
    """setupm / _set_timestep computed in C++ agree with the oracle's numpy
    restatement (which is bit-exact with the reference)."""
    from oracle.microphysics import set_timestep, setupm
    from pyshield_b200 import constants as C

    cfg = PhysicsConfig(dt_atmos=dt, **over)
    lib = _lib.load()
    buf = (ctypes.c_double * 400)()
    n = _lib.check(lib.shield_mp_setup_constants(ctypes.byref(_lib.make_config(cfg)), dt, buf, 400))
    got = np.array(buf[:n])
    K = setupm(cfg)
    T = set_timestep(cfg, dt)
    expect = list(C.packed())
    expect += [K[k] for k in ("c_air", "c_vap", "d0_vap", "lv00", "cpaut", "so3", "zs", "log_10", "tice0", "t_wfr")]
    expect += [K["fac_rc"], K["cracs"], K["csacr"], K["cgacr"], K["cgacs"]]
    expect += [K[f"acco_{i}{j}"] for i in range(3) for j in range(4)]
    expect += [K["csacw"], K["csaci"], K["cgacw"], K["cgaci"], K["cracw"]]
    expect += [K[f"cssub_{i}"] for i in range(5)] + [K[f"crevp_{i}"] for i in range(5)]
    expect += [K["cgfr_0"], K["cgfr_1"]] + [K[f"csmlt_{i}"] for i in range(5)] + [K[f"cgmlt_{i}"] for i in range(5)]
    expect += [K["ces0"]]
    iqs_lo = C.E00 * np.exp((C.D2ICE * np.log(1.0 - 160.0 / C.TICE) - C.LI2 * 160.0 / (C.T_SAT_MIN * C.TICE)) / C.RVGAS)
    expect += [iqs_lo, dt, T["rdt"], T["dts"], T["dt_rain"], T["rdts"], T["dt_evap"]]
    expect += [T["fac_i2s"], T["fac_g2v"], T["fac_v2g"], T["fac_imlt"], T["fac_l2v"]]
    expect = np.array(expect)
    assert got.shape == expect.shape
    # libm and numpy may differ in the last place of exp/log/pow; the five
    # fac_* = 1 - exp(-x) (the last entries) amplify that by 1 / fac, so they
    # are held to two ulps of 1 in absolute terms
    nfac = 5
    np.testing.assert_allclose(got[:-nfac], expect[:-nfac], rtol=4e-16, atol=0.0)
    np.testing.assert_allclose(got[-nfac:], expect[-nfac:], rtol=0.0, atol=4.5e-16)
    # the physical constants are plain arithmetic: identical
    np.testing.assert_array_equal(got[: len(C.packed())], np.array(C.packed()))


def test_bad_timestep_is_rejected():
    lib = _lib.load()
    buf = (ctypes.c_double * 400)()
    cfg = _lib.make_config(PhysicsConfig(dt_atmos=150.0))
    assert lib.shield_mp_setup_constants(ctypes.byref(cfg), 0.0, buf, 400) == -1
    assert "timestep" in _lib.last_error()
    assert lib.shield_mp_setup_constants(ctypes.byref(cfg), float("nan"), buf, 400) == -1


def test_create_without_a_gpu_fails_loudly():
    """No CUDA device here: creating a handle must fail with an error code and
    a message, never fall back to the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = ctypes.c_void_p()
    area = _lib.ShieldField2D(ctypes.c_void_p(16), 1, 1)
    rc = lib.shield_mp_create(ctypes.byref(_lib.make_config(PhysicsConfig(dt_atmos=150.0))), 4, 4, 10, area, ctypes.byref(h))
    assert rc == -3
    assert _lib.last_error()
    from pyshield_b200.grid import GridIndexing, StencilFactory
    from pyshield_b200.microphysics import Microphysics

    with pytest.raises(Exception):
        Microphysics(StencilFactory(GridIndexing(4, 4, 10)), None, None, PhysicsConfig(dt_atmos=150.0))


def test_argument_checks_on_the_cpu():
    lib = _lib.load()
    h = ctypes.c_void_p()
    area = _lib.ShieldField2D(ctypes.c_void_p(16), 1, 1)
    cfg = _lib.make_config(PhysicsConfig(dt_atmos=150.0))
    assert lib.shield_mp_create(ctypes.byref(cfg), 4, 4, 300, area, ctypes.byref(h)) == -2  # too many levels
    assert lib.shield_mp_create(ctypes.byref(cfg), 0, 4, 10, area, ctypes.byref(h)) == -1
    cfg_ppm = _lib.make_config(PhysicsConfig(dt_atmos=150.0, use_ppm=True))
    assert lib.shield_mp_create(ctypes.byref(cfg_ppm), 4, 4, 10, area, ctypes.byref(h)) == -1
    assert "use_ppm" in _lib.last_error()
    assert lib.shield_mp_step(None, None, 150.0, 0, None) == -1
    assert lib.shield_update_physics_state(0, 1, 1, None, None, None, 1.0, None) == -1


def test_ctypes_structs_match_the_header(tmp_path):
    """The ctypes mirrors of the header's structs have the C sizes and field
    offsets (a mismatch would hand the kernels shifted pointers)."""
    import ctypes
    import subprocess

    from pyshield_b200 import _lib

    checks = {
        "ShieldMpFields": (_lib.ShieldMpFields, ["land", "rain", "graupel"]),
        "ShieldMpCotangents": (_lib.ShieldMpCotangents, ["qaz", "rain"]),
        "ShieldMpGradients": (_lib.ShieldMpGradients, ["qaz"]),
        "ShieldMpMember": (_lib.ShieldMpMember, ["nx", "timestep", "area"]),
        "ShieldPhysicsFields": (_lib.ShieldPhysicsFields, ["wmp", "vdt"]),
        "ShieldEdgePlan": (_lib.ShieldEdgePlan, ["r"]),
        "ShieldDwindGeometry": (_lib.ShieldDwindGeometry, ["edge_vect_s", "edge_stride"]),
        "ShieldDwindTile": (_lib.ShieldDwindTile, ["dt5", "plan", "geometry", "u", "v_dt"]),
        "ShieldMpConfig": (_lib.ShieldMpConfig, ["clin"]),
    }
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "shield_mp.h"', "int main(void) {"]
    for name, (_, fields) in checks.items():
        src.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for f in fields:
            src.append(f'  printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    src.append("  return 0;\n}")
    c = tmp_path / "sizes.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "sizes"
    r = subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(c), "-o", str(exe)], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for name, (cls, fields) in checks.items():
        assert int(got[name]) == ctypes.sizeof(cls), name
        for f in fields:
            assert int(got[f"{name}.{f}"]) == getattr(cls, f).offset, f"{name}.{f}"
