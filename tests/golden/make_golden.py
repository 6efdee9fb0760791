"""Generate golden fixtures by running the reference's own pySHiELD source.

Usage (in a container where the pySHiELD source tree is available)::

    python tests/golden/make_golden.py [--reference /path/to/pySHiELD-checkout]

gt4py and NDSL are not installable here, so ``gtshim/`` provides the names
the reference imports, and its ``_gtexec`` module executes the stencil
definitions with GT4Py's numpy-backend semantics. Everything that runs is the
reference's code: ``Microphysics.__init__`` / ``setupm`` / ``__call__``, the
stencils ``fields_init``, ``warm_rain``, ``sedimentation``, ``icloud``,
``fields_update`` and the pointwise functions of ``microphysics_funcs.py``,
plus the coupling stencils of ``physics.py``, ``update_atmos_state.py`` and
``fv_update_phys.py``.

Inputs come from ``pyshield_b200.inputs.make_state`` plus per-case
perturbations that reach the rarer branches (negative species for
``fix_negative``, temperatures below ``T_MIN``, pressures below ``P_MIN``,
non-zero incoming tendencies). Each case is written to ``<case>.npz`` next to
this script; the tests compare the oracle against these files bit for bit,
and the CUDA kernels against the oracle.
"""

import argparse
import dataclasses
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

MP_OUT = ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt")


def _setup_paths(reference):
    sys.path.insert(0, os.path.join(HERE, "gtshim"))
    sys.path.insert(0, REPO)
    sys.path.insert(0, reference)


def mp_cases():
    """(name, nx, ny, L, dt, nsteps, config overrides, perturbation) tuples."""
    return [
        ("mp_default", 6, 4, 24, 150.0, 2, {}, "none"),
        ("mp_substeps", 5, 3, 20, 450.0, 1, {}, "stress"),
        (
            "mp_flags_a",
            4,
            4,
            18,
            225.0,
            2,
            dict(
                do_qa=True,
                fast_sat_adj=False,
                z_slope_ice=False,
                z_slope_liq=False,
                do_sedi_heat=True,
                hydrostatic=True,
                de_ice=True,
                sedi_transport=False,
            ),
            "stress",
        ),
        (
            "mp_flags_b",
            4,
            3,
            16,
            180.0,
            1,
            dict(
                irain_f=1,
                const_vi=True,
                const_vs=True,
                const_vg=True,
                const_vr=True,
                vi_fac=0.3333333333333333,
                vg_fac=2.0,
                vr_fac=4.0,
                rad_snow=False,
                rad_rain=False,
                do_sedi_heat=True,
                fix_negative=False,
            ),
            "none",
        ),
        ("mp_prog_ccn_off_ice", 3, 3, 12, 150.0, 1, dict(vi_fac=1.0e-6), "stress"),
    ]


def perturb(state, kind, seed):
    """Push some points into the rarer branches of the scheme."""
    if kind == "none":
        return
    rng = np.random.default_rng(seed + 1000)
    L, n = state["pt"].shape
    # negative species for fix_negative (fields_init :202-276)
    for name in ("qice", "qsnow", "qgraupel", "qrain", "qliquid"):
        m = rng.random((L, n)) < 0.04
        state[name][m] = -rng.uniform(1e-9, 2e-6, int(m.sum()))
    # a negative vapour run near the surface and the top
    m = rng.random(n) < 0.3
    state["qvapor"][L - 1, m] = -1e-7
    state["qvapor"][L - 3, m] = -5e-8
    state["qvapor"][2, m] = -1e-8
    # very cold tops (T < T_MIN) and thin top layers (p1 < P_MIN)
    state["pt"][0, : n // 2] = 170.0
    state["delprsi"][0, : n // 3] = 20.0
    # non-zero incoming tendencies (they are accumulated)
    for name in MP_OUT:
        state[name][...] = rng.normal(0.0, 1e-6, (L, n))
    state["qi_dt"][...] = rng.normal(0.0, 1e-7, (L, n))


def to_storage(arr_ln, nx, ny, h=3):
    """(L, n) -> NDSL storage (nx+2h+1, ny+2h+1, L+1), column c = j*nx + i."""
    L = arr_ln.shape[0]
    out = np.zeros((nx + 2 * h + 1, ny + 2 * h + 1, L + 1))
    out[h : h + nx, h : h + ny, :L] = arr_ln.reshape(L, ny, nx).transpose(2, 1, 0)
    return out


def to_storage2d(arr_n, nx, ny, h=3):
    out = np.zeros((nx + 2 * h + 1, ny + 2 * h + 1))
    out[h : h + nx, h : h + ny] = arr_n.reshape(ny, nx).T
    return out


def from_storage(st, nx, ny, L, h=3):
    return st[h : h + nx, h : h + ny, :L].transpose(2, 1, 0).reshape(L, nx * ny).copy()


def run_mp_case(name, nx, ny, L, dt, nsteps, overrides, kind):
    import pySHiELD
    from ndsl.dsl.stencil import GridIndexing, StencilFactory
    from ndsl.grid import GridData
    from ndsl.initialization.allocator import QuantityFactory
    from ndsl.quantity import Quantity
    from pySHiELD.stencils.microphysics import Microphysics, MicrophysicsState

    from pyshield_b200._config import PhysicsConfig as OurConfig
    from pyshield_b200.inputs import make_state

    n = nx * ny
    seed = abs(hash(name)) % (2 ** 31)
    seed = sum(ord(c) for c in name)
    state, area = make_state(n, L, seed=seed, n_cube=nx)
    perturb(state, kind, seed)
    inputs = {k: v.copy() for k, v in state.items()}

    cfg_kwargs = dict(dt_atmos=dt, npx=nx + 1, npy=ny + 1, npz=L)
    cfg_kwargs.update(overrides)
    ref_cfg = pySHiELD.PhysicsConfig(**cfg_kwargs)
    gi = GridIndexing(nx, ny, L)
    sf = StencilFactory(gi)
    qf = QuantityFactory(nx, ny, L)
    dims3 = ["x", "y", "z"]

    def q3(a):
        return Quantity(to_storage(a, nx, ny), dims3, "", origin=(3, 3, 0), extent=(nx, ny, L))

    area_q = Quantity(to_storage2d(area, nx, ny), ["x", "y"], "m^2", origin=(3, 3), extent=(nx, ny))
    grid_data = GridData(area=area_q)
    mp = Microphysics(sf, qf, grid_data, ref_cfg)

    fields3 = {
        k: q3(state[k])
        for k in ("pt", "qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qcld", "ua", "va", "delprsi", "delz", "wmp")
    }
    zeros = qf.zeros(dims3, "")
    land_q = Quantity(to_storage2d(state["land"], nx, ny), ["x", "y"], "", origin=(3, 3), extent=(nx, ny))
    ms = MicrophysicsState(
        pt=fields3["pt"],
        qvapor=fields3["qvapor"],
        qliquid=fields3["qliquid"],
        qrain=fields3["qrain"],
        qice=fields3["qice"],
        qsnow=fields3["qsnow"],
        qgraupel=fields3["qgraupel"],
        qcld=fields3["qcld"],
        ua=fields3["ua"],
        va=fields3["va"],
        delp=qf.zeros(dims3, ""),
        delz=fields3["delz"],
        omga=qf.zeros(dims3, ""),
        delprsi=fields3["delprsi"],
        wmp=fields3["wmp"],
        dz=qf.zeros(dims3, ""),
        tendency=zeros,
        land=land_q,
    )
    for t in MP_OUT:
        getattr(ms, t).data[...] = to_storage(state[t], nx, ny)

    out = {}
    for step in range(nsteps):
        mp(ms, timestep=dt)
        for t in MP_OUT:
            out[f"s{step}_{t}"] = from_storage(getattr(ms, t).data, nx, ny, L)
        for f in ("wmp", "qice", "qsnow"):
            out[f"s{step}_{f}"] = from_storage(getattr(ms, f).data, nx, ny, L)
        for p, attr in (("rain", "_rain"), ("snow", "_snow"), ("ice", "_ice"), ("graupel", "_graupel")):
            out[f"s{step}_{p}"] = from_storage(getattr(mp, attr).data, nx, ny, L)[0]
        out[f"s{step}_qaz"] = from_storage(mp._qaz.data, nx, ny, L)

    our_fields = {f.name for f in dataclasses.fields(OurConfig)}
    meta = {
        "name": name,
        "nx": nx,
        "ny": ny,
        "L": L,
        "dt": dt,
        "nsteps": nsteps,
        "config": {k: v for k, v in cfg_kwargs.items() if k in our_fields},
        "kind": kind,
    }
    arrays = {f"in_{k}": v for k, v in inputs.items()}
    arrays["in_area"] = area
    arrays.update(out)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=json.dumps(meta), **arrays)
    return meta


def coupling_cases():
    return [("cpl_small", 5, 4, 16, 225.0, 0), ("cpl_stress", 4, 3, 12, 150.0, 1)]


def run_coupling_case(name, nx, ny, L, dt, stress):
    """Coupling stencils on one synthetic state, each run on its own inputs:
    update_physics_state_with_tendencies (physics.py:151-194),
    fill_gfs_delp (update_atmos_state.py:21-37),
    prepare_tendencies_and_update_tracers (update_atmos_state.py:40-92),
    moist_cv and update_pressure_and_surface_winds (fv_update_phys.py:32-75).
    The domains are those the reference constructs them with."""
    import pySHiELD.stencils.physics as phys
    import pySHiELD.update.fv_update_phys as fvp
    import pySHiELD.update.update_atmos_state as uas
    from ndsl.dsl.stencil import GridIndexing, StencilFactory

    import pyshield_b200.constants as C

    rng = np.random.default_rng(sum(ord(c) for c in name))
    h = 3
    gi = GridIndexing(nx, ny, L)
    sf = StencilFactory(gi)
    shape = gi.domain_full(add=(1, 1, 1))
    qn = ("qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel")
    out = {}

    def rnd(lo, hi):
        return rng.uniform(lo, hi, shape)

    # --- update_physics_state_with_tendencies
    names_in = qn + ("qcld", "pt", "ua", "va")
    arrs = {}
    for nm in names_in:
        arrs[nm] = rnd(0.0, 1e-3) if nm.startswith("q") else rnd(-20.0, 300.0)
    tnd = {t: rng.normal(0.0, 1e-5, shape) for t in MP_OUT}
    upd = {f"u_{nm}": np.zeros(shape) for nm in names_in}
    st = sf.from_origin_domain(phys.update_physics_state_with_tendencies, origin=gi.origin_compute(), domain=gi.domain_compute())
    st(
        arrs["qvapor"], arrs["qliquid"], arrs["qrain"], arrs["qice"], arrs["qsnow"], arrs["qgraupel"],
        arrs["qcld"], arrs["pt"], arrs["ua"], arrs["va"],
        tnd["qv_dt"], tnd["ql_dt"], tnd["qr_dt"], tnd["qi_dt"], tnd["qs_dt"], tnd["qg_dt"], tnd["qa_dt"], tnd["pt_dt"], tnd["udt"], tnd["vdt"],
        upd["u_qvapor"], upd["u_qliquid"], upd["u_qrain"], upd["u_qice"], upd["u_qsnow"], upd["u_qgraupel"],
        upd["u_qcld"], upd["u_pt"], upd["u_ua"], upd["u_va"], dt,
    )
    for nm in names_in:
        out[f"upd_in_{nm}"] = arrs[nm]
        out[f"upd_out_{nm}"] = upd[f"u_{nm}"]
    for t in MP_OUT:
        out[f"upd_in_{t}"] = tnd[t]

    # --- fill_gfs_delp on the full (halo) domain with L+1 levels
    delp = rnd(50.0, 2000.0)
    q = rnd(-2e-9, 5e-3)
    if stress:
        q[..., 3:7] = rng.uniform(-1e-6, 2e-9, q[..., 3:7].shape)
    out["fill_in_delp"] = delp.copy()
    out["fill_in_q"] = q.copy()
    st = sf.from_origin_domain(uas.fill_gfs_delp, origin=gi.origin_full(), domain=gi.domain_full(add=(0, 0, 1)))
    st(delp, q, 1.0e-9)
    out["fill_out_q"] = q

    # --- prepare_tendencies_and_update_tracers
    p = {}
    for nm in ("u_dt", "v_dt", "pt_dt"):
        p[nm] = rng.normal(0.0, 1e-4, shape)
    for nm in ("u_t1", "v_t1", "u_t0", "v_t0"):
        p[nm] = rnd(-30.0, 30.0)
    p["pu_pt"] = rnd(200.0, 300.0)
    p["pt_t0"] = rnd(200.0, 300.0)
    for nm in qn:
        p[f"pu_{nm}"] = rnd(0.0, 2e-3)
        p[f"{nm}_t0"] = rnd(0.0, 2e-3)
    prsi = np.cumsum(rnd(50.0, 2000.0), axis=2)
    p["prsi"] = prsi
    p["delp"] = rnd(50.0, 2000.0)
    for k, v in p.items():
        out[f"prep_in_{k}"] = v.copy()
    st = sf.from_origin_domain(
        uas.prepare_tendencies_and_update_tracers, origin=gi.origin_compute(), domain=gi.domain_compute(add=(0, 0, 1))
    )
    st(
        p["u_dt"], p["v_dt"], p["pt_dt"], p["u_t1"], p["v_t1"], p["pu_pt"],
        p["pu_qvapor"], p["pu_qliquid"], p["pu_qrain"], p["pu_qsnow"], p["pu_qice"], p["pu_qgraupel"],
        p["u_t0"], p["v_t0"], p["pt_t0"],
        p["qvapor_t0"], p["qliquid_t0"], p["qrain_t0"], p["qsnow_t0"], p["qice_t0"], p["qgraupel_t0"],
        p["prsi"], p["delp"], 1.0 / dt,
    )
    for k in ("u_dt", "v_dt", "pt_dt", "delp") + tuple(f"{nm}_t0" for nm in qn):
        out[f"prep_out_{k}"] = p[k]

    # --- moist_cv + update_pressure_and_surface_winds
    m = {nm: rnd(0.0, 2e-3) for nm in qn}
    m["pt"] = rnd(200.0, 300.0)
    m["t_dt"] = rng.normal(0.0, 1e-4, shape)
    for k, v in m.items():
        out[f"mcv_in_{k}"] = v.copy()
    st = sf.from_origin_domain(fvp.moist_cv, origin=gi.origin_compute(), domain=gi.domain_compute(add=(0, 0, 1)))
    st(m["qvapor"], m["qliquid"], m["qrain"], m["qsnow"], m["qice"], m["qgraupel"], m["pt"], m["t_dt"], C.CP_AIR, dt)
    out["mcv_out_pt"] = m["pt"]
    out["mcv_out_t_dt"] = m["t_dt"]

    pe = np.zeros(shape)
    pe[..., 0] = 100.0
    pdelp = rnd(50.0, 2000.0)
    ua = rnd(-30.0, 30.0)
    va = rnd(-30.0, 30.0)
    peln = np.zeros(shape)
    pk = np.zeros(shape)
    ps = np.zeros(shape[:2])
    us = np.zeros(shape[:2])
    vs = np.zeros(shape[:2])
    for k, v in (("pe", pe), ("delp", pdelp), ("ua", ua), ("va", va)):
        out[f"ups_in_{k}"] = v.copy()
    st = sf.from_origin_domain(
        fvp.update_pressure_and_surface_winds, origin=gi.origin_compute(), domain=gi.domain_compute(add=(0, 0, 1))
    )
    st(pe, pdelp, peln, pk, C.KAPPA, ua, va, ps, us, vs)
    for k, v in (("pe", pe), ("peln", peln), ("pk", pk), ("ps", ps), ("u_srf", us), ("v_srf", vs)):
        out[f"ups_out_{k}"] = v
    meta = {"name": name, "nx": nx, "ny": ny, "L": L, "dt": dt, "halo": h}
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=json.dumps(meta), **out)
    return meta


def run_coupling_chain(name, nx, ny, L, dt, seed):
    """The column part of UpdateAtmosphereState.__call__ with dycore_only=False
    and apply_tendencies=True (update_atmos_state.py:301-349,
    fv_update_phys.py:170-186) on one consistent state: fill_gfs_delp on the
    physics-updated vapour, prepare_tendencies_and_update_tracers, moist_cv
    and update_pressure_and_surface_winds, each on the domain the reference
    builds it with."""
    import pySHiELD.update.fv_update_phys as fvp
    import pySHiELD.update.update_atmos_state as uas
    from ndsl.dsl.stencil import GridIndexing, StencilFactory

    import pyshield_b200.constants as C

    rng = np.random.default_rng(seed)
    gi = GridIndexing(nx, ny, L)
    sf = StencilFactory(gi)
    shape = gi.domain_full(add=(1, 1, 1))

    def rnd(lo, hi):
        return rng.uniform(lo, hi, shape)

    f = {}
    for nm in ("u_dt", "v_dt", "pt_dt"):
        f[nm] = rng.normal(0.0, 1e-4, shape)
    f["pu_ua"] = rnd(-30.0, 30.0)
    f["pu_va"] = rnd(-30.0, 30.0)
    f["pu_pt"] = rnd(200.0, 300.0)
    for nm in ("qvapor", "qliquid", "qrain", "qsnow", "qice", "qgraupel"):
        f["pu_" + nm] = rnd(0.0, 2e-3)
        f["dy_" + nm] = rnd(0.0, 2e-3)
    # a few small / negative vapour values for fill_gfs_delp
    m = rng.random(shape) < 0.05
    f["pu_qvapor"][m] = rng.uniform(-2e-6, 2e-9, int(m.sum()))
    f["ph_ua"] = rnd(-30.0, 30.0)
    f["ph_va"] = rnd(-30.0, 30.0)
    f["ph_pt"] = rnd(200.0, 300.0)
    f["prsi"] = np.cumsum(rnd(50.0, 2000.0), axis=2)
    f["dy_delp"] = rnd(50.0, 2000.0)
    f["dy_pt"] = rnd(200.0, 300.0)
    f["pe"] = np.zeros(shape)
    f["pe"][..., 0] = 100.0
    f["peln"] = np.zeros(shape)
    f["pk"] = np.zeros(shape)
    f["dy_ua"] = rnd(-30.0, 30.0)
    f["dy_va"] = rnd(-30.0, 30.0)
    out = {f"in_{k}": v.copy() for k, v in f.items()}
    ps = np.zeros(shape[:2])
    us = np.zeros(shape[:2])
    vs = np.zeros(shape[:2])
    fill = sf.from_origin_domain(uas.fill_gfs_delp, origin=gi.origin_full(), domain=gi.domain_full(add=(0, 0, 1)))
    prep = sf.from_origin_domain(
        uas.prepare_tendencies_and_update_tracers, origin=gi.origin_compute(), domain=gi.domain_compute(add=(0, 0, 1))
    )
    mcv = sf.from_origin_domain(fvp.moist_cv, origin=gi.origin_compute(), domain=gi.domain_compute(add=(0, 0, 1)))
    ups = sf.from_origin_domain(
        fvp.update_pressure_and_surface_winds, origin=gi.origin_compute(), domain=gi.domain_compute(add=(0, 0, 1))
    )
    fill(f["dy_delp"], f["pu_qvapor"], 1.0e-9)
    prep(
        f["u_dt"], f["v_dt"], f["pt_dt"], f["pu_ua"], f["pu_va"], f["pu_pt"],
        f["pu_qvapor"], f["pu_qliquid"], f["pu_qrain"], f["pu_qsnow"], f["pu_qice"], f["pu_qgraupel"],
        f["ph_ua"], f["ph_va"], f["ph_pt"],
        f["dy_qvapor"], f["dy_qliquid"], f["dy_qrain"], f["dy_qsnow"], f["dy_qice"], f["dy_qgraupel"],
        f["prsi"], f["dy_delp"], 1.0 / dt,
    )
    mcv(f["dy_qvapor"], f["dy_qliquid"], f["dy_qrain"], f["dy_qsnow"], f["dy_qice"], f["dy_qgraupel"], f["dy_pt"], f["pt_dt"], C.CP_AIR, dt)
    ups(f["pe"], f["dy_delp"], f["peln"], f["pk"], C.KAPPA, f["dy_ua"], f["dy_va"], ps, us, vs)
    for k, v in f.items():
        out[f"out_{k}"] = v
    out["out_ps"] = ps
    out["out_u_srf"] = us
    out["out_v_srf"] = vs
    meta = {"name": name, "nx": nx, "ny": ny, "L": L, "dt": dt, "halo": 3}
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=json.dumps(meta), **out)
    return meta


D2P_FIELDS = ("qvapor", "qliquid", "qrain", "qsnow", "qice", "qgraupel", "qo3mr", "qsgs_tke", "qcld", "pt", "delp",
              "delz", "ua", "va", "w", "omga")


def run_dycore_to_physics_case(name, nx, ny, L, seed):
    """pySHiELD's ``DycoreToPhysics.__call__`` (update_atmos_state.py:145-232)
    without the dry convective adjustment: the 16-field copy on the
    interface-extended compute domain, levels 0 .. nz - 1."""
    from ndsl.dsl.stencil import GridIndexing, StencilFactory
    from ndsl.initialization.allocator import QuantityFactory
    from pyFV3 import DynamicalCoreConfig
    from pySHiELD.update.update_atmos_state import DycoreToPhysics

    rng = np.random.default_rng(seed)
    shape = (nx + 7, ny + 7, L + 1)
    dy = {f: rng.uniform(-1.0, 1.0, shape) for f in D2P_FIELDS}
    ph = {f: rng.uniform(-1.0, 1.0, shape) for f in D2P_FIELDS}
    out = {f"in_dycore_{f}": v.copy() for f, v in dy.items()}
    out.update({f"in_physics_{f}": v.copy() for f, v in ph.items()})

    class _State:
        pass

    ds, ps = _State(), _State()
    for f in D2P_FIELDS:
        setattr(ds, f, dy[f])
        setattr(ps, f, ph[f])
    gi = GridIndexing(nx, ny, L)
    d2p = DycoreToPhysics(StencilFactory(gi), QuantityFactory(nx, ny, L), DynamicalCoreConfig(), False, False)
    d2p(ds, ps)
    out.update({f"out_physics_{f}": ph[f] for f in D2P_FIELDS})
    meta = {"name": name, "nx": nx, "ny": ny, "L": L, "halo": 3}
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=json.dumps(meta), **out)
    return meta


DWIND_GEOM = ("vlon1", "vlon2", "vlon3", "vlat1", "vlat2", "vlat3", "es1_1", "es1_2", "es1_3", "ew2_1", "ew2_2",
              "ew2_3", "edge_vect_w", "edge_vect_e")


def dwind_cases():
    """(name, subtile nx, ny, L, layout, rank, dt_atmos, grid_type)."""
    return [
        ("dwind_tile", 8, 7, 5, (1, 1), 0, 225.0, 0),
        ("dwind_sub0", 6, 6, 4, (2, 2), 0, 150.0, 0),
        ("dwind_sub3", 6, 6, 4, (2, 2), 3, 150.0, 0),
        ("dwind_periodic", 6, 5, 4, (1, 1), 0, 180.0, 4),
    ]


def run_dwind_case(name, nx, ny, L, layout, rank, dt, grid_type):
    """pySHiELD's AGrid2DGridPhysics.__call__ (update_dwind_phys.py:490-701)
    on one rank's subtile: the prep, the wind-tendency reset, the cube-edge
    corrections of the rank's tile edges, and the D-grid wind update (or the
    doubly periodic update for grid_type > 3)."""
    from types import SimpleNamespace

    from ndsl.comm.partitioner import TilePartitioner
    from ndsl.dsl.stencil import GridIndexing, StencilFactory
    from ndsl.initialization.allocator import QuantityFactory
    from pySHiELD.update.update_dwind_phys import AGrid2DGridPhysics

    rng = np.random.default_rng(sum(ord(c) for c in name))
    h = 3
    part = TilePartitioner(layout)
    sy, sx = part.subtile_index(rank)
    edges = (sy == 0, sy == layout[1] - 1, sx == 0, sx == layout[0] - 1)
    gi = GridIndexing(nx, ny, L, h, edges=edges)
    shape = (nx + 2 * h + 1, ny + 2 * h + 1, L + 1)
    npx, npy = nx * layout[0] + 1, ny * layout[1] + 1
    geom = {k: rng.uniform(-1.0, 1.0, shape[:2]) for k in DWIND_GEOM}
    geom["edge_vect_s"] = rng.uniform(0.0, 1.0, shape[0])
    geom["edge_vect_n"] = rng.uniform(0.0, 1.0, shape[0])
    grid_info = SimpleNamespace(grid_type=grid_type, **geom)
    namelist = SimpleNamespace(dt_atmos=dt, npx=npx, npy=npy, layout=layout)
    fields = {k: rng.uniform(-5.0, 5.0, shape) for k in ("u", "v", "u_dt", "v_dt")}
    out = {f"in_{k}": v.copy() for k, v in fields.items()}
    out.update({f"geom_{k}": v for k, v in geom.items()})
    a2d = AGrid2DGridPhysics(StencilFactory(gi), QuantityFactory(nx, ny, L), part, rank, namelist, grid_info)
    a2d(fields["u"], fields["v"], fields["u_dt"], fields["v_dt"])
    out.update({f"out_{k}": v for k, v in fields.items()})
    meta = {"name": name, "nx": nx, "ny": ny, "L": L, "halo": h, "layout": list(layout), "rank": rank,
            "subtile_index": [int(sy), int(sx)], "edges": [bool(e) for e in edges], "npx": npx, "npy": npy, "dt": dt,
            "grid_type": grid_type}
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=json.dumps(meta), **out)
    return meta


def physics_cases():
    """(name, nx, ny, L, dt, seed, config overrides)."""
    return [
        ("phys_default", 4, 3, 14, 150.0, 41, {}),
        ("phys_substeps", 3, 4, 12, 225.0, 42, dict(mp_time=150.0, do_qa=True)),
    ]


def run_physics_case(name, nx, ny, L, dt, seed, overrides):
    """pySHiELD's ``Physics.__call__`` (physics.py:276-366) end to end:
    atmos_phys_driver_statein, get_prs_fv3, get_phi_fv3, prepare_microphysics,
    the microphysics step and update_physics_state_with_tendencies, on a
    ``PhysicsState`` of NDSL-layout storages (halo 3, nz + 1 levels) from
    ``pyshield_b200.inputs.make_physics_state``."""
    import pySHiELD
    from ndsl.dsl.stencil import GridIndexing, StencilFactory
    from ndsl.grid import GridData
    from ndsl.initialization.allocator import QuantityFactory
    from ndsl.quantity import Quantity
    from pySHiELD.physics_state import PhysicsState
    from pySHiELD.stencils.physics import Physics

    from pyshield_b200.inputs import PHYSICS_3D, PHYSICS_INTERFACE, PTOP, make_physics_state

    h = 3
    st, area = make_physics_state(nx, ny, L, seed=seed, halo=h)
    inputs = {k: v.copy() for k, v in st.items()}
    cfg_kwargs = dict(dt_atmos=dt, npx=nx + 1, npy=ny + 1, npz=L)
    cfg_kwargs.update(overrides)
    ref_cfg = pySHiELD.PhysicsConfig(**cfg_kwargs)
    gi = GridIndexing(nx, ny, L)
    sf = StencilFactory(gi)
    qf = QuantityFactory(nx, ny, L)
    area_q = Quantity(to_storage2d(area, nx, ny), ["x", "y"], "m^2", origin=(h, h), extent=(nx, ny))
    grid_data = GridData(area=area_q, ptop=PTOP)
    phys = Physics(sf, qf, grid_data, ref_cfg)
    quantities = {}
    for nm in PHYSICS_3D:
        dims = ["x", "y", "z_interface" if nm in PHYSICS_INTERFACE else "z"]
        quantities[nm] = Quantity(st[nm], dims, "", origin=(h, h, 0), extent=(nx, ny, L + 1 if nm in PHYSICS_INTERFACE else L))
    quantities["land"] = Quantity(st["land"], ["x", "y"], "", origin=(h, h), extent=(nx, ny))
    ps = PhysicsState(**quantities, quantity_factory=qf, schemes=ref_cfg.schemes)
    for t in MP_OUT:
        getattr(ps.microphysics, t).data[...] = st[t]
    phys(ps, dt)

    out = {f"in_{k}": v for k, v in inputs.items()}
    for nm in PHYSICS_3D:
        out[f"out_{nm}"] = ps.__dict__[nm].data
    for t in MP_OUT:
        out[f"out_{t}"] = getattr(ps.microphysics, t).data
    out["out__prsik"] = phys._prsik.data
    out["out__dm3d"] = phys._dm3d.data
    out["out__del_gz"] = phys._del_gz.data
    mp = phys._microphysics
    for p, attr in (("rain", "_rain"), ("snow", "_snow"), ("ice", "_ice"), ("graupel", "_graupel")):
        out[f"out_{p}"] = from_storage(getattr(mp, attr).data, nx, ny, L)[0]
    out["in_area"] = area
    meta = {"name": name, "nx": nx, "ny": ny, "L": L, "dt": dt, "halo": h, "ptop": PTOP,
            "config": {k: v for k, v in cfg_kwargs.items()}}
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=json.dumps(meta), **out)
    return meta


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PYSHIELD_REFERENCE"),
                    help="checkout of pySHiELD (the directory holding the pySHiELD package); "
                         "or set PYSHIELD_REFERENCE")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference <pySHiELD checkout> or set PYSHIELD_REFERENCE")
    _setup_paths(args.reference)
    for case in mp_cases():
        if args.only and args.only != case[0]:
            continue
        meta = run_mp_case(*case)
        print("wrote", meta["name"])
    for case in coupling_cases():
        if args.only and args.only != case[0]:
            continue
        meta = run_coupling_case(*case)
        print("wrote", meta["name"])
    for case in (("cpl_chain", 6, 5, 20, 225.0, 7),):
        if args.only and args.only != case[0]:
            continue
        meta = run_coupling_chain(*case)
        print("wrote", meta["name"])
    for case in physics_cases():
        if args.only and args.only != case[0]:
            continue
        meta = run_physics_case(*case)
        print("wrote", meta["name"])
    for case in dwind_cases():
        if args.only and args.only != case[0]:
            continue
        meta = run_dwind_case(*case)
        print("wrote", meta["name"])
    for case in (("d2p_copy", 5, 4, 10, 61),):
        if args.only and args.only != case[0]:
            continue
        meta = run_dycore_to_physics_case(*case)
        print("wrote", meta["name"])


if __name__ == "__main__":
    main()
