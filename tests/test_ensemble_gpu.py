"""Ensembles of uneven members in one persistent launch.

The batched step must give each member exactly what its own Microphysics
step gives (same kernel body, same constants): bit for bit in the FP64 form,
for every launch shape the autotuner may pick, and through CUDA-graph
replay."""
import numpy as np
import pytest

from golden_io import MP_TENDENCIES
from mp_helpers import device_state, read_state

pytestmark = pytest.mark.gpu

MEMBERS = ((12, 6, 150.0), (24, 12, 225.0), (8, 6, 180.0), (36, 6, 120.0))  # (nx, ny, dt)
L = 79


def _states(seed0, nlev=L):
    from pyshield_b200.inputs import make_state

    out = []
    for m, (nx, ny, dt) in enumerate(MEMBERS):
        st, area = make_state(nx * ny, nlev, seed=seed0 + m, n_cube=max(nx, ny), ts_offset=(-1.0) ** m * 2.0)
        out.append((st, area, nx, ny, dt))
    return out


def _single(cfg, members, nsteps, precision, nlev=L):
    from pyshield_b200.microphysics import Microphysics

    res = []
    for st, area, nx, ny, dt in members:
        ms, sf, qf, gd = device_state(st, area, nx, ny)
        mp = Microphysics(sf, qf, gd, cfg, precision=precision)
        for _ in range(nsteps):
            mp(ms, dt)
        o = read_state(ms, nx, ny, nlev)
        o["rain"] = mp.rain.cpu().numpy()
        o["qaz"] = mp.get_qaz().cpu().numpy()
        res.append(o)
    return res


def _ensemble(cfg, members, precision):
    from pyshield_b200.ensemble import MicrophysicsEnsemble

    built = [device_state(st, area, nx, ny) for st, area, nx, ny, dt in members]
    ens = MicrophysicsEnsemble(cfg, [b[0] for b in built], [b[3].area for b in built], [m[4] for m in members],
                               precision=precision)
    return ens, built


def _read(ens, built, members, nlev=L):
    res = []
    for m, ((ms, _, _, _), (st, area, nx, ny, dt)) in enumerate(zip(built, members)):
        o = read_state(ms, nx, ny, nlev)
        o["rain"] = ens.precip(m)[0].cpu().numpy()
        o["qaz"] = ens.qaz(m).cpu().numpy()
        res.append(o)
    return res


@pytest.mark.parametrize("shape,nlev", [((2, 4), L), ((4, 2), L), ((6, 1), L), ((8, 1), L), ((8, 2), L),
                                        ((1, 4), 127), ((4, 1), 127), ((2, 2), 127), ((1, 4), 90), ((4, 1), 90)])
def test_batched_plain_equals_members_bitwise(shape, nlev):
    import torch

    from pyshield_b200._config import PhysicsConfig

    cfg = PhysicsConfig(dt_atmos=150.0)
    members = _states(100, nlev)
    ref = _single(cfg, members, 1, "plain", nlev)
    ens, built = _ensemble(cfg, members, "plain")
    ens.step(*shape)
    torch.cuda.synchronize()
    got = _read(ens, built, members, nlev)
    for m, (a, b) in enumerate(zip(got, ref)):
        for f in MP_TENDENCIES + ("wmp", "rain", "qaz"):
            np.testing.assert_array_equal(a[f], b[f], err_msg=f"member {m} field {f} shape {shape}")


def test_graph_replay_and_autotune():
    import torch

    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.ensemble import launch_shapes

    cfg = PhysicsConfig(dt_atmos=150.0)
    members = _states(200)
    ref = _single(cfg, members, 3, "plain")
    ens, built = _ensemble(cfg, members, "plain")
    ens.tuned = (2, 2)
    ens.capture()  # runs one warm step outside the graph
    ens.replay()
    ens.replay()
    torch.cuda.synchronize()
    got = _read(ens, built, members)
    for m, (a, b) in enumerate(zip(got, ref)):
        for f in MP_TENDENCIES + ("wmp", "qaz"):
            np.testing.assert_array_equal(a[f], b[f], err_msg=f"member {m} field {f}")
    tuned, timings = ens.autotune(reps=1)
    assert tuned in timings and all(v > 0 for v in timings.values())
    assert set(timings) == set(launch_shapes(L))


def test_batched_mixed_matches_members():
    import torch

    from pyshield_b200._config import PhysicsConfig

    cfg = PhysicsConfig(dt_atmos=150.0)
    members = _states(300)
    ref = _single(cfg, members, 1, "mixed")
    ens, built = _ensemble(cfg, members, "mixed")
    ens.step(2, 2)
    torch.cuda.synchronize()
    got = _read(ens, built, members)
    for m, (a, b) in enumerate(zip(got, ref)):
        for f in MP_TENDENCIES + ("wmp",):
            scale = max(float(np.max(np.abs(b[f]))), 1e-300)
            assert float(np.max(np.abs(a[f] - b[f]))) <= 1e-9 * scale, (m, f)
