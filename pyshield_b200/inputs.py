"""Seeded synthetic microphysics states (there is no public dataset for this path).

One generator serves every workload. The per-point distributions are:

* surface pressure ``ps ~ U(980, 1030) hPa``, on hybrid levels whose interface
  pressures are ``p = PTOP + (ps - PTOP) * s**1.7`` with ``s = k / L``
  (this project's choice: pySHiELD ships no ak/bk table);
* temperature on a 6.5 K/km lapse rate from ``Ts ~ U(280, 302) K`` down to a
  215 K tropopause, plus ``N(0, 1.5) K`` noise;
* ``qv = RH * qsat`` with ``RH ~ U(0.3, 1.05)`` per point; optionally a
  fraction of columns at ``RH ~ U(0.98, 1.02)`` to sit on the
  saturation-adjustment thresholds;
* cloud water ``qc ~ logU(1e-7, 2e-3)`` where ``RH > 0.9`` and ``T > 253 K``;
  rain ``qr ~ logU(1e-7, 1e-3)`` below the freezing level; cloud ice, snow and
  graupel ``~ logU(1e-8, 5e-4)`` above it; zero elsewhere;
* cloud fraction 1 where total condensate exceeds 1e-6, else 0;
* ``delz < 0`` from hydrostatic balance; ``wmp ~ N(0, 1) m/s``;
  ``ua, va ~ N(0, 10) m/s``; land mask ``~ Bernoulli(0.3)``;
* cell area ``4 pi R^2 / (6 N^2)`` for a CN cubed sphere;
* all ten tendencies zero (``prepare_microphysics`` zeroes them before the
  microphysics call, ``pySHiELD/stencils/physics.py:133-143``).

Arrays are returned in the (L, n) level-major layout with k = 0 at the model
top.
"""

import numpy as np

from . import constants as C

PTOP = 100.0  # Pa; model-top pressure of the synthetic hybrid grid
RADIUS = 6.3712e6  # m

STATE_FIELDS = (
    "pt", "qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qcld",
    "ua", "va", "delprsi", "delz", "wmp",
)
TENDENCY_FIELDS = (
    "pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt",
    "udt", "vdt",
)


def _qsat_liquid(t, p):
    """Saturation specific humidity over water (Clausius-Clapeyron form of
    the microphysics' own ``wqs1`` vapour pressure), used only to build RH."""
    es = C.E00 * np.exp(
        (C.DC_VAP * np.log(t / C.TICE) + C.LV0 * (t - C.TICE) / (t * C.TICE)) / C.RVGAS
    )
    return C.EPS * es / np.maximum(p - (1.0 - C.EPS) * es, 1.0)


def _logu(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size))


def cube_area(n_cube):
    """Mean cell area of a C``n_cube`` cubed sphere [m^2]."""
    return 4.0 * np.pi * RADIUS ** 2 / (6.0 * n_cube * n_cube)


def make_state(ncol, nlev, seed=0, n_cube=None, ts_offset=0.0, sat_fraction=0.0):
    """Return ``(state, area)``: a dict of (L, n) / (n,) float64 arrays keyed
    by MicrophysicsState attribute names (tendencies included, zeroed), and
    the (n,) cell-area array."""
    rng = np.random.default_rng(seed)
    L, n = nlev, ncol
    ps = rng.uniform(980.0e2, 1030.0e2, n)
    s = (np.arange(L + 1, dtype=np.float64) / L) ** 1.7
    p_if = PTOP + (ps[None, :] - PTOP) * s[:, None]  # (L+1, n), top -> surface
    delp = p_if[1:] - p_if[:-1]
    p_mid = 0.5 * (p_if[1:] + p_if[:-1])
    ts = rng.uniform(280.0, 302.0, n) + ts_offset
    noise = rng.normal(0.0, 1.5, (L, n))
    # integrate heights upward from the surface with the lapse-rate profile
    t = np.empty((L, n))
    dz = np.empty((L, n))
    z_bot = np.zeros(n)
    for k in range(L - 1, -1, -1):
        t_guess = np.maximum(215.0, ts - 6.5e-3 * z_bot)
        h = C.RDGAS * t_guess / C.GRAV * np.log(p_if[k + 1] / p_if[k])
        t[k] = np.maximum(215.0, ts - 6.5e-3 * (z_bot + 0.5 * h)) + noise[k]
        dz[k] = C.RDGAS * t[k] / C.GRAV * np.log(p_if[k + 1] / p_if[k])
        z_bot = z_bot + dz[k]
    rh = rng.uniform(0.3, 1.05, (L, n))
    if sat_fraction > 0.0:
        sat_cols = rng.random(n) < sat_fraction
        rh[:, sat_cols] = rng.uniform(0.98, 1.02, (L, int(sat_cols.sum())))
    qv = rh * _qsat_liquid(t, p_mid)
    qv = np.minimum(qv, 0.05)
    warm = t > C.TICE
    qc = np.where((rh > 0.9) & (t > 253.0), _logu(rng, 1e-7, 2e-3, (L, n)), 0.0)
    qr = np.where(warm, _logu(rng, 1e-7, 1e-3, (L, n)), 0.0)
    qi = np.where(~warm, _logu(rng, 1e-8, 5e-4, (L, n)), 0.0)
    qs = np.where(~warm, _logu(rng, 1e-8, 5e-4, (L, n)), 0.0)
    qg = np.where(~warm, _logu(rng, 1e-8, 5e-4, (L, n)), 0.0)
    cond = qc + qr + qi + qs + qg
    qa = np.where(cond > 1e-6, 1.0, 0.0)
    tv = t * (1.0 + C.ZVIR * qv)
    delz = -(C.RDGAS * tv / C.GRAV) * np.log(p_if[1:] / p_if[:-1])
    state = {
        "pt": t,
        "qvapor": qv,
        "qliquid": qc,
        "qrain": qr,
        "qice": qi,
        "qsnow": qs,
        "qgraupel": qg,
        "qcld": qa,
        "ua": rng.normal(0.0, 10.0, (L, n)),
        "va": rng.normal(0.0, 10.0, (L, n)),
        "delprsi": delp,
        "delz": delz,
        "wmp": rng.normal(0.0, 1.0, (L, n)),
        "land": (rng.random(n) < 0.3).astype(np.float64),
    }
    for name in TENDENCY_FIELDS:
        state[name] = np.zeros((L, n))
    if n_cube is None:
        n_cube = max(1, int(round(np.sqrt(n / 6.0))))
    area = np.full(n, cube_area(n_cube))
    return state, area


def copy_state(state):
    return {k: np.array(v, copy=True) for k, v in state.items()}


PHYSICS_3D = (
    "qvapor", "qliquid", "qice", "qrain", "qsnow", "qgraupel", "qo3mr", "qsgs_tke", "qcld", "pt", "delp", "delz",
    "ua", "va", "w", "omga", "physics_updated_specific_humidity", "physics_updated_qliquid", "physics_updated_qice",
    "physics_updated_qrain", "physics_updated_qsnow", "physics_updated_qgraupel", "physics_updated_cloud_fraction",
    "physics_updated_pt", "physics_updated_ua", "physics_updated_va", "delprsi", "phii", "phil", "dz", "wmp", "prsi",
    "prsik",
)
PHYSICS_INTERFACE = ("phii", "prsi", "prsik")


def make_physics_state(nx, ny, nlev, seed=0, halo=3, sat_fraction=0.2):
    """A ``PhysicsState``'s storages for the physics driver: a dict of
    NDSL-layout arrays (nx + 2 halo + 1, ny + 2 halo + 1, nlev + 1) keyed by
    the PhysicsState field names (``land`` 2-D), plus the ten tendencies of
    ``physics_state.microphysics`` under their own names, and the (n,) cell
    area.

    The compute domain holds a ``make_state`` column set (``delp`` is its
    pressure thickness). ``qo3mr ~ U(1e-8, 1e-5)``, ``qsgs_tke ~ U(0, 2)``,
    ``w ~ U(-1, 1)``, ``omga ~ U(-2, 2) Pa/s``. The halo points and the extra
    level hold plausible random values (the full-domain stencils read the
    halo), interface pressure and geopotential there are monotone profiles,
    and every output field and tendency starts from random values (the
    steps overwrite what the reference overwrites)."""
    rng = np.random.default_rng(seed)
    h, L = halo, nlev
    n = nx * ny
    state, area = make_state(n, L, seed=seed, n_cube=nx, sat_fraction=sat_fraction)
    shape = (nx + 2 * h + 1, ny + 2 * h + 1, L + 1)
    ci, cj = slice(h, h + nx), slice(h, h + ny)

    def put(arr_ln, lo, hi):
        a = rng.uniform(lo, hi, shape)
        if arr_ln is not None:
            a[ci, cj, :L] = arr_ln.reshape(L, ny, nx).transpose(2, 1, 0)
        return a

    st = {}
    for q in ("qvapor", "qliquid", "qice", "qrain", "qsnow", "qgraupel", "qcld"):
        st[q] = put(state[q], 0.0, 1e-3)
    st["qo3mr"] = put(None, 1e-8, 1e-5)
    st["qsgs_tke"] = put(None, 0.0, 2.0)
    st["pt"] = put(state["pt"], 200.0, 300.0)
    st["delp"] = put(state["delprsi"], 100.0, 2000.0)
    st["delz"] = put(state["delz"], -800.0, -50.0)
    st["ua"] = put(state["ua"], -30.0, 30.0)
    st["va"] = put(state["va"], -30.0, 30.0)
    st["w"] = put(None, -1.0, 1.0)
    st["omga"] = put(None, -2.0, 2.0)
    for nm in PHYSICS_3D:
        if nm.startswith("physics_updated") or nm in ("delprsi", "phil", "dz", "wmp", "prsik"):
            st[nm] = put(None, -1.0, 1.0)
    st["prsi"] = np.cumsum(rng.uniform(100.0, 2000.0, shape), axis=2) + PTOP
    st["phii"] = np.cumsum(rng.uniform(100.0, 3000.0, shape)[..., ::-1], axis=2)[..., ::-1] - 100.0
    land = np.zeros(shape[:2])
    land[ci, cj] = state["land"].reshape(ny, nx).T
    st["land"] = land
    for t in TENDENCY_FIELDS:
        st[t] = rng.uniform(-1.0, 1.0, shape)
    return st, area
