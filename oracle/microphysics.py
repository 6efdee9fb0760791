"""CPU oracle: FP64 numpy restatement of pySHiELD's GFDL microphysics step.

TEST INFRASTRUCTURE ONLY. Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg may import this module, and only as the
checker (or as the timed CPU stand-in for the reference's numpy backend).
The product path (``pyshield_b200``) never calls it.

What it restates (paths within the pySHiELD project):

* ``pySHiELD/stencils/microphysics.py:27-276``   fields_init
* ``pySHiELD/stencils/microphysics.py:280-653``  warm_rain
* ``pySHiELD/stencils/microphysics.py:657-1217`` sedimentation
* ``pySHiELD/stencils/microphysics.py:1220-1449`` icloud
* ``pySHiELD/stencils/microphysics.py:1452-1553`` fields_update
* ``pySHiELD/stencils/microphysics.py:1806-1979`` setupm / _set_timestep
* ``pySHiELD/stencils/microphysics.py:1981-2263`` the call sequence
* ``pySHiELD/functions/microphysics_funcs.py:1-1260`` pointwise functions

GT4Py execution semantics are reproduced explicitly: a PARALLEL block runs
each statement over its whole interval before the next statement; FORWARD and
BACKWARD blocks run level by level with all statements of a level in order,
so ``[0, 0, -1]`` / ``[0, 0, +1]`` reads see values already updated in the
sweep. Conditionals become masks; a temporary assigned under a condition keeps
its previous value elsewhere. Every arithmetic expression is written with the
same operand order as the reference, so that numpy evaluates the same
sequence of IEEE operations.

Array layout: 3-D fields are ``(L, n)`` arrays (level-major, k = 0 at the
model top, k = L-1 at the surface); 2-D fields are ``(n,)``.

Parity pin: ``tests/golden/make_golden.py`` runs the reference's own stencil
source through a GT4Py-semantics numpy executor and the golden fixtures it
writes are compared bit-for-bit with this oracle by
``tests/test_oracle_golden.py``.
"""

import numpy as np
import numpy as _np  # the integer flag words stay host numpy whatever backs np

from pyshield_b200 import constants as C

# --- microphysics_funcs.py:7-42 (numeric table, kept identical) -------------
VCONS = 6.6280504
VCONG = 87.2382675
NORMS = 942477796.076938
NORMG = 5026548245.74367
VCONR = 2503.23638966667
NORMR = 25132741228.7183
THR = 1.0e-8
THI = 1.0e-8
THG = 1.0e-8
THS = 1.0e-8
AA = -4.14122e-5
BB = -0.00538922
CC = -0.0516344
DD_FS = 0.00216078
EE = 1.9714
VR_MIN = 1.0e-3
VF_MIN = 1.0e-5
P_MIN = 100.0
DT_FR = 8.0
SFCRHO = 1.2
RHOS = 1.0e2
RHOG = 4.0e2
RHOR = 1.0e3
DZ_MIN_FLIP = 1.0e-2
QCMIN = 1.0e-12
QRMIN = 1.0e-8
QVMIN = 1.0e-20

W = np.where
mn = np.minimum
mx = np.maximum


def _flag_bits(mask, bit):
    """The int32 word ``bit`` where the column mask is set, else 0 (the
    column flags are integers and never differentiated)."""
    m = mask.detach().cpu().numpy() if hasattr(mask, "detach") else mask
    return _np.where(_np.asarray(m, dtype=bool), bit, 0).astype(_np.int32)


def _first_level(mask):
    """Index of the first level where the (L, n) mask is set, per column."""
    m = mask.detach().cpu().numpy() if hasattr(mask, "detach") else mask
    return _np.argmax(_np.asarray(m, dtype=bool), axis=0).astype(_np.int32)


def dim(x, y):
    """microphysics_funcs.py:45-49"""
    diff = x - y
    return W(diff > 0.0, diff, 0.0)


# --- saturation specific humidity: microphysics_funcs.py:52-145 -------------
def wqs1(ta, den):
    return (
        C.E00
        * np.exp(
            (C.DC_VAP * np.log(ta / C.TICE) + C.LV0 * (ta - C.TICE) / (ta * C.TICE))
            / C.RVGAS
        )
    ) / (C.RVGAS * ta * den)


def wqs2(ta, den):
    tmp = wqs1(ta, den)
    return tmp, tmp * (C.DC_VAP + C.LV0 / ta) / (C.RVGAS * ta)


def iqs1(ta, den):
    ice_hi = (
        C.E00
        * np.exp(
            (C.D2ICE * np.log(ta / C.TICE) + C.LI2 * (ta - C.TICE) / (ta * C.TICE))
            / C.RVGAS
        )
    ) / (C.RVGAS * ta * den)
    ice_lo = (
        C.E00
        * np.exp(
            (
                C.D2ICE * np.log(1.0 - 160.0 / C.TICE)
                - C.LI2 * 160.0 / (C.T_SAT_MIN * C.TICE)
            )
            / C.RVGAS
        )
    ) / (C.RVGAS * C.T_SAT_MIN * den)
    liq = wqs1(ta, den)
    liq_cap = wqs1(C.TICE + 102.0 + 0.0 * ta, den)
    return W(
        ta < C.TICE,
        W(ta >= C.T_SAT_MIN, ice_hi, ice_lo),
        W(ta <= C.TICE + 102.0, liq, liq_cap),
    )


def iqs2(ta, den):
    tmp = iqs1(ta, den)
    d_ice_hi = tmp * (C.D2ICE + C.LI2 / ta) / (C.RVGAS * ta)
    d_ice_lo = (
        tmp * (C.D2ICE + C.LI2 / C.T_SAT_MIN) / (C.RVGAS * C.T_SAT_MIN)
    )
    d_liq = tmp * (C.DC_VAP + C.LV0 / ta) / (C.RVGAS * ta)
    d_liq_cap = (
        tmp
        * (C.DC_VAP + C.LV0 / (C.TICE + 102.0))
        / (C.RVGAS * (C.TICE + 102.0))
    )
    dtmp = W(
        ta < C.TICE,
        W(ta >= C.T_SAT_MIN, d_ice_hi, d_ice_lo),
        W(ta <= C.TICE + 102.0, d_liq, d_liq_cap),
    )
    return tmp, dtmp


# --- microphysics_funcs.py:148-179 -------------------------------------------
def acr3d(v1, v2, q1, q2, c, cac_ik, cac_i1k, cac_i2k, rho):
    t1 = np.sqrt(q1 * rho)
    s1 = np.sqrt(q2 * rho)
    s2 = np.sqrt(s1)
    return (
        c * np.abs(v1 - v2) * q1 * s2 * (cac_ik * t1 + cac_i1k * np.sqrt(t1) * s2 + cac_i2k * s1)
    )


def smlt(tc, dqs, qsrho, psacw, psacr, c_0, c_1, c_2, c_3, c_4, rho, rhofac):
    return (c_0 * tc / rho - c_1 * dqs) * (
        c_2 * np.sqrt(qsrho) + c_3 * qsrho ** 0.65625 * np.sqrt(rhofac)
    ) + c_4 * tc * (psacw + psacr)


def gmlt(tc, dqs, qgrho, pgacw, pgacr, c_0, c_1, c_2, c_3, c_4, rho):
    return (c_0 * tc / rho - c_1 * dqs) * (
        c_2 * np.sqrt(qgrho) + c_3 * qgrho ** 0.6875 / rho ** 0.25
    ) + c_4 * tc * (pgacw + pgacr)


# --- setup: microphysics.py:1806-1979 ----------------------------------------
def setupm(cfg):
    """Process constants of ``Microphysics.setupm`` (microphysics.py:1813-1953)."""
    gam263 = 1.456943
    gam275 = 1.608355
    gam290 = 1.827363
    gam325 = 2.54925
    gam350 = 3.323363
    gam380 = 4.694155
    rnzs = 3.0e6
    rnzr = 8.0e6
    rnzg = 4.0e6
    acc = np.array([5.0, 2.0, 0.5])
    pie = 4.0 * np.arctan(1.0)
    fac_rc = (4.0 / 3.0) * pie * RHOR * cfg.rthresh ** 3
    vdifu = 2.11e-5
    tcond = 2.36e-2
    visk = 1.259e-5
    hlts = 2.8336e6
    hltc = 2.5e6
    hltf = 3.336e5
    ch2o = 4.1855e3
    pisq = pie * pie
    scm3 = (visk / vdifu) ** (1.0 / 3.0)
    cracs = pisq * rnzr * rnzs * RHOS
    csacr = pisq * rnzr * rnzs * RHOR
    cgacr = pisq * rnzr * rnzg * RHOR
    cgacs = pisq * rnzg * rnzs * RHOS
    cgacs = cgacs * cfg.c_pgacs
    act = np.empty(8)
    act[0] = pie * rnzs * RHOS
    act[1] = pie * rnzr * RHOR
    act[5] = pie * rnzg * RHOG
    act[2] = act[1]
    act[3] = act[0]
    act[4] = act[1]
    act[6] = act[0]
    act[7] = act[5]
    acco = np.empty((3, 4))
    for i in range(3):
        for k in range(4):
            acco[i, k] = acc[i] / (
                act[2 * k] ** ((6 - i) * 0.25) * act[2 * k + 1] ** ((i + 1) * 0.25)
            )
    gcon = 40.74 * np.sqrt(SFCRHO)
    csacw = pie * rnzs * cfg.clin * gam325 / (4.0 * act[0] ** 0.8125)
    craci = pie * rnzr * cfg.alin * gam380 / (4.0 * act[1] ** 0.95)
    csaci = csacw * cfg.c_psaci
    cgacw = pie * rnzg * gam350 * gcon / (4.0 * act[5] ** 0.875)
    cgaci = cgacw * 0.05
    cracw = craci
    cracw = cfg.c_cracw * cracw
    k = {}
    k["cssub_0"] = 2.0 * pie * vdifu * tcond * C.RVGAS * rnzs
    k["cssub_1"] = 0.78 / np.sqrt(act[0])
    k["cssub_2"] = (
        0.31 * scm3 * gam263 * np.sqrt(cfg.clin / visk) / act[0] ** 0.65625
    )
    k["cssub_3"] = tcond * C.RVGAS
    k["cssub_4"] = (hlts ** 2) * vdifu
    cgsub_1 = 0.78 / np.sqrt(act[5])
    cgsub_2 = 0.31 * scm3 * gam275 * np.sqrt(gcon / visk) / act[5] ** 0.6875
    k["crevp_0"] = 2.0 * pie * vdifu * tcond * C.RVGAS * rnzr
    k["crevp_1"] = 0.78 / np.sqrt(act[1])
    k["crevp_2"] = (
        0.31 * scm3 * gam290 * np.sqrt(cfg.alin / visk) / act[1] ** 0.725
    )
    k["crevp_3"] = k["cssub_3"]
    k["crevp_4"] = hltc ** 2 * vdifu
    k["cgfr_0"] = 20.0e2 * pisq * rnzr * RHOR / act[1] ** 1.75
    k["cgfr_1"] = 0.66
    k["csmlt_0"] = 2.0 * pie * tcond * rnzs / hltf
    k["csmlt_1"] = 2.0 * pie * vdifu * rnzs * hltc / hltf
    k["csmlt_2"] = k["cssub_1"]
    k["csmlt_3"] = k["cssub_2"]
    k["csmlt_4"] = ch2o / hltf
    k["cgmlt_0"] = 2.0 * pie * tcond * rnzg / hltf
    k["cgmlt_1"] = 2.0 * pie * vdifu * rnzg * hltc / hltf
    k["cgmlt_2"] = cgsub_1
    k["cgmlt_3"] = cgsub_2
    k["cgmlt_4"] = ch2o / hltf
    es0 = 6.107799961e2
    k["fac_rc"] = fac_rc
    k["cracs"] = cracs
    k["csacr"] = csacr
    k["cgacr"] = cgacr
    k["cgacs"] = cgacs
    for i in range(3):
        for j in range(4):
            k[f"acco_{i}{j}"] = acco[i, j]
    k["csacw"] = csacw
    k["csaci"] = csaci
    k["cgacw"] = cgacw
    k["cgaci"] = cgaci
    k["cracw"] = cracw
    k["ces0"] = C.EPS * es0
    # gfdl_cloud_microphys_init (microphysics.py:1806-1811), __init__ (:1643-1658)
    k["log_10"] = np.log(10.0)
    k["tice0"] = cfg.tice - 0.01
    k["t_wfr"] = cfg.tice - 40.0
    k["c_air"] = C.CP_AIR
    k["c_vap"] = C.CP_VAP
    k["d0_vap"] = k["c_vap"] - C.C_LIQ
    k["lv00"] = C.HLV - k["d0_vap"] * C.TICE
    k["cpaut"] = cfg.c_paut * 0.104 * C.GRAV / 1.717e-5
    k["so3"] = 7.0 / 3.0
    k["zs"] = 0.0
    return {name: float(v) for name, v in k.items()}


def set_timestep(cfg, timestep):
    """``Microphysics._set_timestep`` (microphysics.py:1964-1979)."""
    mpdt = min(timestep, cfg.mp_time)
    rdt = 1.0 / timestep
    ntimes = int(round(timestep / mpdt))
    dts = timestep / ntimes
    dt_rain = dts * 0.5
    rdts = 1.0 / dts
    dt_evap = 0.5 * dts if cfg.fast_sat_adj else dts
    return {
        "mpdt": mpdt,
        "rdt": rdt,
        "ntimes": ntimes,
        "dts": dts,
        "dt_rain": dt_rain,
        "rdts": rdts,
        "dt_evap": dt_evap,
        "fac_i2s": float(1.0 - np.exp(-dts / cfg.tau_i2s)),
        "fac_g2v": float(1.0 - np.exp(-dts / cfg.tau_g2v)),
        "fac_v2g": float(1.0 - np.exp(-dts / cfg.tau_v2g)),
        "fac_imlt": float(1.0 - np.exp(-0.5 * dts / cfg.tau_imlt)),
        "fac_l2v": float(1.0 - np.exp(-dt_evap / cfg.tau_l2v)),
    }


class _K:
    """Attribute bag of config flags + setupm + timestep scalars."""

    def __init__(self, cfg, setup, ts):
        self.cfg = cfg
        self.__dict__.update(setup)
        self.__dict__.update(ts)
        self.do_sedi_w = False if cfg.hydrostatic else cfg.do_sedi_w
        self.use_ccn = False if cfg.prog_ccn else True


def _column_any(cond):
    """GT4Py ``no_fall`` idiom (microphysics.py:349-368): 0 everywhere in a
    column if ``cond`` holds at any level, else 1. Returns the 2-D flag
    broadcast to (L, n)."""
    L = cond.shape[0]
    no_fall = np.empty(cond.shape)
    no_fall[0] = W(cond[0], 0.0, 1.0)
    for k in range(1, L):
        no_fall[k] = W(no_fall[k - 1] == 1.0, W(cond[k], 0.0, 1.0), 0.0)
    for k in range(L - 2, -1, -1):
        no_fall[k] = W(no_fall[k + 1] == 0.0, no_fall[k + 1], no_fall[k])
    return no_fall


def _ze_column(dz1, zs):
    """BACKWARD height sweep (microphysics.py:756-765 / 373-380)."""
    L = dz1.shape[0]
    ze = np.empty(dz1.shape)
    ze[L - 1] = zs - dz1[L - 1]
    for k in range(L - 2, -1, -1):
        ze[k] = ze[k + 1] - dz1[k]
    return ze


def _dz_from_ze(ze, zs):
    dz = np.empty(ze.shape)
    dz[:-1] = ze[:-1] - ze[1:]
    dz[-1] = ze[-1] - zs
    return dz


def _implicit_fall(m, q, dz, dd, dp1):
    """Implicit upwind fall of one species, use_ppm=False
    (microphysics.py:454-490 for rain; :839-876 ice; :970-1007 snow;
    :1103-1140 graupel). Returns (q_mass, qm, m1_flux, surface_flux) with
    updates applied only where ``m`` (the no_fall == 0 mask) is set."""
    L = q.shape[0]
    qmass = W(m, q * dp1, q)
    qm = np.zeros(q.shape)
    qm[0] = W(m[0], qmass[0] / (dz[0] + dd[0]), qm[0])
    for k in range(1, L):
        qm[k] = W(m[k], (qmass[k] + dd[k - 1] * qm[k - 1]) / (dz[k] + dd[k]), qm[k])
    qm = W(m, qm * dz, qm)
    flux = np.zeros(q.shape)
    flux[0] = W(m[0], qmass[0] - qm[0], flux[0])
    for k in range(1, L):
        flux[k] = W(m[k], flux[k - 1] + qmass[k] - qm[k], flux[k])
    sfc = flux[L - 1]
    return qmass, qm, flux, sfc


def _w_transport(m, w, dm, flux, vt):
    """Vertical-velocity transport (microphysics.py:492-515 and repeats)."""
    wn = w.copy()
    wn[0] = W(m[0], (dm[0] * w[0] + flux[0] * vt[0]) / (dm[0] - flux[0]), w[0])
    wn[1:] = W(
        m[1:],
        (dm[1:] * w[1:] - flux[:-1] * vt[:-1] + flux[1:] * vt[1:])
        / (dm[1:] + flux[:-1] - flux[1:]),
        w[1:],
    )
    return wn


def _sedi_heat(m, tz, dz1, dp1, qv, ql, qr, qi, qs, qg, flux, c_cond):
    """Implicit heating by falling condensate (microphysics.py:516-557 with
    C_LIQ; :1176-1217 with C_ICE)."""
    L = tz.shape[0]
    dgz = -0.5 * C.GRAV * dz1
    cvn = dp1 * (
        C.CV_AIR + qv * C.CV_VAP + (qr + ql) * C.C_LIQ + (qi + qs + qg) * C.C_ICE
    )
    tz = tz.copy()
    tmp = cvn[0] + flux[0] * c_cond
    tz[0] = W(m[0], tz[0] + flux[0] * dgz[0] / tmp, tz[0])
    for k in range(1, L):
        tz[k] = W(
            m[k],
            (
                (cvn[k] + c_cond * (flux[k] - flux[k - 1])) * tz[k]
                + flux[k - 1] * c_cond * tz[k - 1]
                + dgz[k] * (flux[k - 1] + flux[k])
            )
            / (cvn[k] + c_cond * flux[k]),
            tz[k],
        )
    return tz


# --- microphysics_funcs.py:182-265 -------------------------------------------
def revap_racc(m, dt, K, h_var, qg, qi, ql, qr, qs, qv, tz, den, denfac):
    c_air, c_vap = K.c_air, K.c_vap
    a = m & (tz > K.t_wfr) & (qr > QRMIN)
    lhl = K.lv00 + K.d0_vap * tz
    q_liq = ql + qr
    q_sol = qi + qs + qg
    cvm = c_air + qv * c_vap + q_liq * C.C_LIQ + q_sol * C.C_ICE
    lcpk = lhl / cvm
    tin = tz - lcpk * ql
    qpz = qv + ql
    qsat, dqsdt = wqs2(tin, den)
    dqh = mx(ql, h_var * mx(qpz, QCMIN))
    dqh = mn(dqh, 0.2 * qpz)
    dqv = qsat - qv
    q_minus = qpz - dqh
    q_plus = qpz + dqh
    b = a & (dqv > QVMIN) & (qsat > q_minus)
    dq = W(qsat > q_plus, qsat - qpz, 0.25 * (q_minus - qsat) ** 2 / dqh)
    qden = qr * den
    t2 = tin * tin
    evap = (
        K.crevp_0
        * t2
        * dq
        * (K.crevp_1 * np.sqrt(qden) + K.crevp_2 * np.exp(0.725 * np.log(qden)))
        / (K.crevp_3 * t2 + K.crevp_4 * qsat * den)
    )
    evap = mn(qr, mn(dt * evap, dqv / (1.0 + lcpk * dqsdt)))
    qr = W(b, qr - evap, qr)
    qv = W(b, qv + evap, qv)
    q_liq = W(b, q_liq - evap, q_liq)
    cvm = W(b, c_air + qv * c_vap + q_liq * C.C_LIQ + q_sol * C.C_ICE, cvm)
    tz = W(b, tz - evap * lhl / cvm, tz)
    c = a & (qr > QRMIN) & (ql > 1.0e-6) & (qsat < q_minus)
    sink = dt * denfac * K.cracw * np.exp(0.95 * np.log(qr * den))
    sink = sink / (1.0 + sink) * ql
    ql = W(c, ql - sink, ql)
    qr = W(c, qr + sink, qr)
    return qg, qi, ql, qr, qs, qv, tz


# --- microphysics_funcs.py:268-372 -------------------------------------------
def fall_speed(K, qg, qi, ql, qs, tk, den):
    cfg = K.cfg
    rhof = np.sqrt(mn(10.0, SFCRHO / den))
    if cfg.const_vi:
        vti = np.full(qi.shape, cfg.vi_fac)
    else:
        vi0 = 0.01 * cfg.vi_fac
        tc = tk - cfg.tice
        vti = (
            (3.0 + np.log(qi * den) / K.log_10) * (tc * (AA * tc + BB) + CC)
            + DD_FS * tc
            + EE
        )
        vti = vi0 * np.exp(K.log_10 * vti) * 0.8
        vti = mn(cfg.vi_max, mx(VF_MIN, vti))
        vti = W(qi < THI, VF_MIN, vti)
    if cfg.const_vs:
        vts = np.full(qs.shape, cfg.vs_fac)
    else:
        vts = cfg.vs_fac * VCONS * rhof * np.exp(0.0625 * np.log(qs * den / NORMS))
        vts = mn(cfg.vs_max, mx(VF_MIN, vts))
        vts = W(qs < THS, VF_MIN, vts)
    if cfg.const_vg:
        vtg = np.full(qg.shape, cfg.vg_fac)
    else:
        vtg = cfg.vg_fac * VCONG * rhof * np.sqrt(np.sqrt(np.sqrt(qg * den / NORMG)))
        vtg = mn(cfg.vg_max, mx(VF_MIN, vtg))
        vtg = W(qg < THG, VF_MIN, vtg)
    return vtg, vti, vts


def compute_rain_fspeed(K, no_fall, qrz, den):
    cfg = K.cfg
    if cfg.const_vr:
        v = np.full(qrz.shape, cfg.vr_fac)
    else:
        qden = qrz * den
        v = (
            cfg.vr_fac
            * VCONR
            * np.sqrt(mn(10.0, SFCRHO / den))
            * np.exp(0.2 * np.log(qden / NORMR))
        )
        v = mn(cfg.vr_max, mx(VR_MIN, v))
        v = W(qrz < THR, VR_MIN, v)
    vtrz = W(no_fall == 1.0, VF_MIN, v)
    r1 = np.zeros(qrz.shape)
    return vtrz, r1


# --- microphysics_funcs.py:375-428 -------------------------------------------
def autoconv_no_subgrid_var(K, qlz, qrz, tz, den, ccn, c_praut):
    qc0 = K.fac_rc * ccn
    qc = qc0 if K.use_ccn else qc0 / den
    dq = qlz - qc
    a = (tz > K.t_wfr) & (dq > 0.0)
    sink = mn(dq, K.dt_rain * c_praut * den * np.exp(K.so3 * np.log(qlz)))
    return W(a, qlz - sink, qlz), W(a, qrz + sink, qrz)


def autoconv_subgrid_var(K, qlz, qrz, tz, den, ccn, c_praut, dl):
    qc0 = K.fac_rc * ccn
    a = tz > K.t_wfr + DT_FR
    dl = mn(mx(1.0e-6, dl), 0.5 * qlz)
    qc = qc0 if K.use_ccn else qc0 / den
    dq = 0.5 * (qlz + dl - qc)
    b = a & (dq > 0.0)
    sink = mn(1.0, dq / dl) * K.dt_rain * c_praut * den * np.exp(K.so3 * np.log(qlz))
    return W(b, qlz - sink, qlz), W(b, qrz + sink, qrz)


def _cvm(K, qv, q_liq, q_sol):
    return K.c_air + qv * K.c_vap + q_liq * C.C_LIQ + q_sol * C.C_ICE


# --- microphysics_funcs.py:431-850 -------------------------------------------
def subgrid_z_proc(K, h_var, rh_adj, rh_rain, qaz, qgz, qiz, qlz, qrz, qsz, qvz, tz, den, denfac, p1):
    cfg = K.cfg
    tice, t_wfr, t_sub = cfg.tice, K.t_wfr, cfg.t_sub
    lv00, d0_vap = K.lv00, K.d0_vap
    lhl = lv00 + d0_vap * tz
    lhi = C.LI00 + C.DC_ICE * tz
    q_liq = qlz + qrz
    q_sol = qiz + qsz + qgz
    cvm = _cvm(K, qvz, q_liq, q_sol)
    lcpk = lhl / cvm
    icpk = lhi / cvm
    tcpk = lcpk + icpk
    tcp3 = lcpk + icpk * mn(1.0, dim(tice, tz) / (tice - t_wfr))

    act = p1 >= P_MIN
    # T < T_MIN: instant deposition (:488-499)
    a = act & (tz < C.T_MIN)
    sink = dim(1.0e-7, qvz)
    qvz = W(a, qvz - sink, qvz)
    qiz = W(a, qiz + sink, qiz)
    q_sol = W(a, q_sol + sink, q_sol)
    cvm = W(a, _cvm(K, qvz, q_liq, q_sol), cvm)
    tz = W(a, tz + sink * (lhl + lhi) / cvm, tz)
    if not cfg.do_qa:
        qaz = W(a, qaz + 1.0, qaz)

    e = act & ~a  # the else branch of ``tz < T_MIN``
    lhl = W(e, lv00 + d0_vap * tz, lhl)
    lhi = W(e, C.LI00 + C.DC_ICE * tz, lhi)
    lcpk = W(e, lhl / cvm, lcpk)
    icpk = W(e, lhi / cvm, icpk)
    tcpk = W(e, lcpk + icpk, tcpk)
    tcp3 = W(e, lcpk + icpk * mn(1.0, dim(tice, tz) / (tice - t_wfr)), tcp3)
    qpz = qvz + qlz + qiz
    tin = tz - (lhl * (qlz + qiz) + lhi * qiz) / (
        K.c_air + qpz * K.c_vap + qrz * C.C_LIQ + (qsz + qgz) * C.C_ICE
    )
    warm = tin > t_sub + 6.0
    rh = qpz / iqs1(tin, den)
    dry = e & warm & (rh < rh_adj)
    tz = W(dry, tin, tz)
    qvz = W(dry, qpz, qvz)
    qlz = W(dry, 0.0, qlz)
    qiz = W(dry, 0.0, qiz)

    g = e & ((warm & (rh >= rh_adj)) | ~warm)
    # cloud water <-> vapour adjustment (:531-554)
    qsw, dwsdt = wqs2(tz, den)
    dq0 = qsw - qvz
    factor = mn(1.0, K.fac_l2v * (10.0 * dq0 / qsw))
    evap = W(
        dq0 > 0.0,
        mn(qlz, factor * dq0 / (1.0 + tcp3 * dwsdt)),
        dq0 / (1.0 + tcp3 * dwsdt),
    )
    qvz = W(g, qvz + evap, qvz)
    qlz = W(g, qlz - evap, qlz)
    q_liq = W(g, q_liq - evap, q_liq)
    cvm = W(g, _cvm(K, qvz, q_liq, q_sol), cvm)
    tz = W(g, tz - evap * lhl / cvm, tz)
    lhi = W(g, C.LI00 + C.DC_ICE * tz, lhi)
    icpk = W(g, lhi / cvm, icpk)
    # forced freezing below t_wfr (:560-575)
    dtmp = t_wfr - tz
    h = g & (dtmp > 0.0) & (qlz > QCMIN)
    sink = mn(qlz, mn(qlz * dtmp * 0.125, dtmp / icpk))
    qlz = W(h, qlz - sink, qlz)
    qiz = W(h, qiz + sink, qiz)
    q_liq = W(h, q_liq - sink, q_liq)
    q_sol = W(h, q_sol + sink, q_sol)
    cvm = W(h, _cvm(K, qvz, q_liq, q_sol), cvm)
    tz = W(h, tz + sink * lhi / cvm, tz)
    lhi = W(g, C.LI00 + C.DC_ICE * tz, lhi)
    icpk = W(g, lhi / cvm, icpk)
    # Bigg mechanism (:581-605)
    if cfg.fast_sat_adj:
        dt_pisub = 0.5 * K.dts
    else:
        dt_pisub = K.dts
        tc = tice - tz
        h = g & (qlz > QRMIN) & (tc > 0.0)
        sink = 3.3333e-10 * K.dts * (np.exp(0.66 * tc) - 1.0) * den * qlz * qlz
        sink = mn(qlz, mn(tc / icpk, sink))
        qlz = W(h, qlz - sink, qlz)
        qiz = W(h, qiz + sink, qiz)
        q_liq = W(h, q_liq - sink, q_liq)
        q_sol = W(h, q_sol + sink, q_sol)
        cvm = W(h, _cvm(K, qvz, q_liq, q_sol), cvm)
        tz = W(h, tz + sink * lhi / cvm, tz)

    def upd_lat(lhl, lhi, lcpk, icpk, tcpk):
        lhl = W(g, lv00 + d0_vap * tz, lhl)
        lhi = W(g, C.LI00 + C.DC_ICE * tz, lhi)
        lcpk = W(g, lhl / cvm, lcpk)
        icpk = W(g, lhi / cvm, icpk)
        tcpk = W(g, lcpk + icpk, tcpk)
        return lhl, lhi, lcpk, icpk, tcpk

    lhl, lhi, lcpk, icpk, tcpk = upd_lat(lhl, lhi, lcpk, icpk, tcpk)
    # ice deposition / sublimation (:614-661)
    h = g & (tz < tice)
    qsi, dqsdt = iqs2(tz, den)
    dq = qvz - qsi
    sink = dq / (1.0 + tcpk * dqsdt)
    pidep = W(
        qiz > QRMIN,
        dt_pisub
        * dq
        * 349138.78
        * np.exp(0.875 * np.log(qiz * den))
        / (qsi * den * C.LAT2 / (0.0243 * C.RVGAS * tz ** 2) + 4.42478e4),
        0.0,
    )
    tmp = tice - tz
    qi_crt = cfg.qi_gen * mn(cfg.qi_lim, 0.1 * tmp) / den
    sink_dep = mn(sink, mn(mx(qi_crt - qiz, pidep), tmp / tcpk))
    pidep_sub = pidep * mn(1.0, dim(tz, t_sub) * 0.2)
    sink_sub = mx(pidep_sub, mx(sink, -qiz))
    sink = W(dq > 0.0, sink_dep, sink_sub)
    qvz = W(h, qvz - sink, qvz)
    qiz = W(h, qiz + sink, qiz)
    q_sol = W(h, q_sol + sink, q_sol)
    cvm = W(h, _cvm(K, qvz, q_liq, q_sol), cvm)
    tz = W(h, tz + sink * (lhl + lhi) / cvm, tz)
    lhl, lhi, lcpk, icpk, tcpk = upd_lat(lhl, lhi, lcpk, icpk, tcpk)
    # snow sublimation / deposition (:670-706)
    h = g & (qsz > QRMIN)
    qsi, dqsdt = iqs2(tz, den)
    qden = qsz * den
    tmp = np.exp(0.65625 * np.log(qden))
    tsq = tz * tz
    dq = (qsi - qvz) / (1.0 + tcpk * dqsdt)
    pssub = (
        K.cssub_0
        * tsq
        * (K.cssub_1 * np.sqrt(qden) + K.cssub_2 * tmp * np.sqrt(denfac))
        / (K.cssub_3 * tsq + K.cssub_4 * qsi * den)
    )
    pssub = (qsi - qvz) * K.dts * pssub
    pssub = W(
        pssub > 0.0,
        mn(pssub * mn(1.0, dim(tz, t_sub) * 0.2), qsz),
        W(tz > tice, 0.0, mx(pssub, mx(dq, (tz - tice) / tcpk))),
    )
    qsz = W(h, qsz - pssub, qsz)
    qvz = W(h, qvz + pssub, qvz)
    q_sol = W(h, q_sol - pssub, q_sol)
    cvm = W(h, _cvm(K, qvz, q_liq, q_sol), cvm)
    tz = W(h, tz - pssub * (lhl + lhi) / cvm, tz)
    lhl, lhi, lcpk, icpk, tcpk = upd_lat(lhl, lhi, lcpk, icpk, tcpk)
    # graupel sublimation / deposition (:715-746)
    h = g & (qgz > QRMIN)
    qsi, dqsdt = iqs2(tz, den)
    dq = (qvz - qsi) / (1.0 + tcpk * dqsdt)
    pgsub = (qvz / qsi - 1.0) * qgz
    pgsub = W(
        pgsub > 0.0,
        W(
            tz > tice,
            0.0,
            mn(mn(K.fac_v2g * pgsub, 0.2 * dq), mn(qlz + qrz, (tice - tz) / tcpk)),
        ),
        mx(K.fac_g2v * pgsub, dq) * mn(1.0, dim(tz, t_sub) * 0.1),
    )
    qgz = W(h, qgz + pgsub, qgz)
    qvz = W(h, qvz - pgsub, qvz)
    q_sol = W(h, q_sol + pgsub, q_sol)
    cvm = W(h, _cvm(K, qvz, q_liq, q_sol), cvm)
    tz = W(h, tz + pgsub * (lhl + lhi) / cvm, tz)
    # minimum evaporation of rain (:751-769)
    lhl = W(g, lv00 + d0_vap * tz, lhl)
    lcpk = W(g, lhl / cvm, lcpk)
    h = g & (qrz > QCMIN)
    qsw, dqsdt = wqs2(tz, den)
    sink = mn(qrz, dim(rh_rain * qsw, qvz) / (1.0 + lcpk * dqsdt))
    qvz = W(h, qvz + sink, qvz)
    qrz = W(h, qrz - sink, qrz)
    q_liq = W(h, q_liq - sink, q_liq)
    cvm = W(h, _cvm(K, qvz, q_liq, q_sol), cvm)
    tz = W(h, tz - sink * lhl / cvm, tz)
    # cloud fraction (:774-848)
    lhl = W(g, lv00 + d0_vap * tz, lhl)
    cvm = W(g, K.c_air + (qvz + q_liq + q_sol) * K.c_vap, cvm)
    lcpk = W(g, lhl / cvm, lcpk)
    if not cfg.do_qa:
        q_sol = qiz + qsz if cfg.rad_snow else qiz
        q_liq = qlz + qrz if cfg.rad_rain else qlz
        q_cond = q_liq + q_sol
        qpz = qvz + q_cond
        tin = tz - (lcpk * q_cond + icpk * q_sol)
        qsi = iqs1(tin, den)
        qsw = wqs1(tin, den)
        rqi = W(q_cond > 3.0e-6, q_sol / q_cond, (tice - tin) / (tice - t_wfr))
        qmix = rqi * qsi + (1.0 - rqi) * qsw
        qstar = W(tin <= t_wfr, qsi, W(tin >= tice, qsw, qmix))
        dq = mx(QCMIN, h_var * qpz)
        q_plus = qpz + dq
        q_minus = qpz - dq
        h = g & (qpz > QRMIN)
        full = h & (qstar < q_minus)
        part = h & ~(qstar < q_minus) & (qstar < q_plus) & (q_cond > cfg.qc_crt)
        qaz = W(full, qaz + 1.0, W(part, qaz + (q_plus - qstar) / (dq + dq), qaz))
    return qaz, qgz, qiz, qlz, qrz, qsz, qvz, tz


# --- microphysics_funcs.py:853-1260 ------------------------------------------
def icloud_main(K, h_var, rh_adj, rh_rain, qaz, qgz, qiz, qlz, qrz, qsz, qvz, tz, den, denfac, vtgz, vtrz, vtsz, p1, di, q_liq, q_sol, cvm):
    cfg = K.cfg
    tice, dts, rdts = cfg.tice, K.dts, K.rdts
    lhi = C.LI00 + C.DC_ICE * tz
    icpk = lhi / cvm
    act = p1 >= P_MIN
    pgacr = np.zeros(tz.shape)
    pgacw = np.zeros(tz.shape)
    tc = tz - tice
    warm = act & (tc >= 0.0)
    cold = act & ~(tc >= 0.0)

    # --- melting branch (:938-1052)
    dqs0 = K.ces0 / p1 - qvz
    a = warm & (qsz > QCMIN)
    factor = denfac * K.csacw * np.exp(0.8125 * np.log(qsz * den))
    psacw = W(qlz > QRMIN, factor / (1.0 + dts * factor) * qlz, 0.0)
    r = qrz > QRMIN
    psacr = W(
        r,
        mn(acr3d(vtsz, vtrz, qrz, qsz, K.csacr, K.acco_01, K.acco_11, K.acco_21, den), qrz * rdts),
        0.0,
    )
    pracs = W(r, acr3d(vtrz, vtsz, qsz, qrz, K.cracs, K.acco_00, K.acco_10, K.acco_20, den), 0.0)
    psmlt = mx(
        0.0,
        smlt(tc, dqs0, qsz * den, psacw, psacr, K.csmlt_0, K.csmlt_1, K.csmlt_2, K.csmlt_3, K.csmlt_4, den, denfac),
    )
    sink = mn(qsz, mn(dts * (psmlt + pracs), tc / icpk))
    qsz = W(a, qsz - sink, qsz)
    tmp = mn(sink, dim(cfg.qs_mlt, qlz))
    qlz = W(a, qlz + tmp, qlz)
    qrz = W(a, qrz + sink - tmp, qrz)
    q_liq = W(a, q_liq + sink, q_liq)
    q_sol = W(a, q_sol - sink, q_sol)
    cvm = W(a, _cvm(K, qvz, q_liq, q_sol), cvm)
    tz = W(a, tz - sink * lhi / cvm, tz)
    tc = W(a, tz - tice, tc)
    lhi = W(warm, C.LI00 + C.DC_ICE * tz, lhi)
    icpk = W(warm, lhi / cvm, icpk)
    a = warm & (qgz > QCMIN) & (tc > 0.0)
    pgacr = W(
        a & (qrz > QRMIN),
        mn(acr3d(vtgz, vtrz, qrz, qgz, K.cgacr, K.acco_02, K.acco_12, K.acco_22, den), rdts * qrz),
        pgacr,
    )
    qden = qgz * den
    factor = K.cgacw * qden / np.sqrt(den * np.sqrt(np.sqrt(qden)))
    pgacw = W(a & (qlz > QRMIN), factor / (1.0 + dts * factor) * qlz, pgacw)
    pgmlt = dts * gmlt(tc, dqs0, qden, pgacw, pgacr, K.cgmlt_0, K.cgmlt_1, K.cgmlt_2, K.cgmlt_3, K.cgmlt_4, den)
    pgmlt = mn(mx(0.0, pgmlt), mn(qgz, tc / icpk))
    qgz = W(a, qgz - pgmlt, qgz)
    qrz = W(a, qrz + pgmlt, qrz)
    q_liq = W(a, q_liq + pgmlt, q_liq)
    q_sol = W(a, q_sol - pgmlt, q_sol)
    cvm = W(a, _cvm(K, qvz, q_liq, q_sol), cvm)
    tz = W(a, tz - pgmlt * lhi / cvm, tz)

    # --- cold branch (:1054-1227)
    a = cold & (qiz > 3.0e-7)
    factor = dts * denfac * K.csaci * np.exp(0.05 * tc + 0.8125 * np.log(qsz * den))
    psaci = W(qsz > 1.0e-7, factor / (1.0 + factor) * qiz, 0.0)
    qim = cfg.qi0_crt / den
    tmp = K.fac_i2s if cfg.const_vi else K.fac_i2s * np.exp(0.025 * tc)
    di = W(a, mx(di, QRMIN), di)
    q_plus = qiz + di
    dq = W(qim > (qiz - di), (0.25 * (q_plus - qim) ** 2) / di, qiz - qim)
    psaut = W(q_plus > (qim + QRMIN), tmp * dq, 0.0)
    sink = mn(0.75 * qiz, psaci + psaut)
    qiz = W(a, qiz - sink, qiz)
    qsz = W(a, qsz + sink, qsz)
    b = a & (qgz > 1.0e-6)
    factor = dts * K.cgaci * np.sqrt(den) * qgz
    pgaci = factor / (1.0 + factor) * qiz
    qiz = W(b, qiz - pgaci, qiz)
    qgz = W(b, qgz + pgaci, qgz)

    tc = W(cold, tz - tice, tc)
    a = cold & (qrz > 1e-7) & (tc < 0.0)
    psacr = W(
        qsz > 1.0e-7,
        dts * acr3d(vtsz, vtrz, qrz, qsz, K.csacr, K.acco_01, K.acco_11, K.acco_21, den),
        0.0,
    )
    pgfr = dts * K.cgfr_0 / den * (np.exp(-K.cgfr_1 * tc) - 1.0) * np.exp(1.75 * np.log(qrz * den))
    sink = psacr + pgfr
    factor = mn(sink, mn(qrz, -tc / icpk)) / mx(sink, QRMIN)
    psacr = factor * psacr
    pgfr = factor * pgfr
    sink = psacr + pgfr
    qrz = W(a, qrz - sink, qrz)
    qsz = W(a, qsz + psacr, qsz)
    qgz = W(a, qgz + pgfr, qgz)
    q_liq = W(a, q_liq - sink, q_liq)
    q_sol = W(a, q_sol + sink, q_sol)
    cvm = W(a, _cvm(K, qvz, q_liq, q_sol), cvm)
    tz = W(a, tz + sink * lhi / cvm, tz)
    lhi = W(cold, C.LI00 + C.DC_ICE * tz, lhi)
    icpk = W(cold, lhi / cvm, icpk)

    a = cold & (qsz > 1.0e-7)
    sink = W(
        qgz > QRMIN,
        dts * acr3d(vtgz, vtsz, qsz, qgz, K.cgacs, K.acco_03, K.acco_13, K.acco_23, den),
        0.0,
    )
    qsm = cfg.qs0_crt / den
    factor = dts * 1.0e-3 * np.exp(0.09 * (tz - tice))
    sink = W(qsz > qsm, sink + factor / (1.0 + factor) * (qsz - qsm), sink)
    sink = mn(qsz, sink)
    qsz = W(a, qsz - sink, qsz)
    qgz = W(a, qgz + sink, qgz)

    a = cold & (qgz > 1.0e-7) & (tz < K.tice0)
    qden = qgz * den
    factor = dts * K.cgacw * qden / np.sqrt(den * np.sqrt(np.sqrt(qden)))
    pgacw_c = W(qlz > 1.0e-6, factor / (1.0 + factor) * qlz, 0.0)
    pgacr_c = W(
        qrz > 1.0e-6,
        mn(dts * acr3d(vtgz, vtrz, qrz, qgz, K.cgacr, K.acco_02, K.acco_12, K.acco_22, den), qrz),
        0.0,
    )
    sink = pgacr_c + pgacw_c
    factor = mn(sink, dim(tice, tz) / icpk) / mx(sink, QRMIN)
    pgacr_c = factor * pgacr_c
    pgacw_c = factor * pgacw_c
    sink = pgacr_c + pgacw_c
    qgz = W(a, qgz + sink, qgz)
    qrz = W(a, qrz - pgacr_c, qrz)
    qlz = W(a, qlz - pgacw_c, qlz)
    q_liq = W(a, q_liq - sink, q_liq)
    q_sol = W(a, q_sol + sink, q_sol)
    cvm = W(a, _cvm(K, qvz, q_liq, q_sol), cvm)
    tz = W(a, tz + sink * lhi / cvm, tz)

    return subgrid_z_proc(K, h_var, rh_adj, rh_rain, qaz, qgz, qiz, qlz, qrz, qsz, qvz, tz, den, denfac, p1)


def _slope(q, zslope):
    """Monotone vertical slope ``dl``/``di`` (microphysics.py:595-620 and
    1341-1367). Returns the limited slope before the h_var floor, or None
    when the slope option is off."""
    if not zslope:
        return None
    L = q.shape[0]
    dq = np.zeros(q.shape)
    dq[1:] = 0.5 * (q[1:] - q[:-1])
    d = np.zeros(q.shape)
    if L > 2:
        a = dq[1:-1]
        b = dq[2:]
        d_in = 0.5 * mn(np.abs(a + b), 0.5 * q[1:-1])
        d_in = W(a * b <= 0.0, W(a > 0.0, mn(d_in, mn(a, -b)), 0.0), d_in)
        d[1:-1] = d_in
    d[0] = 0.0
    d[L - 1] = 0.0
    return d


class OracleMicrophysics:
    """``Microphysics`` (microphysics.py:1623-2263) on numpy arrays.

    ``qaz`` is the reference's persistent scratch Quantity (``self._qaz``,
    zero at construction and never reset, :1674); it lives on this object
    across calls in the same way.
    """

    def __init__(self, cfg, ncol, nlev, area):
        self.cfg = cfg
        self.n = ncol
        self.L = nlev
        self.area = np.asarray(area, dtype=np.float64).reshape(ncol)
        self.setup = setupm(cfg)
        self.timestep = None
        self.qaz = np.zeros((nlev, ncol))
        self._set_timestep(float(cfg.dt_atmos))
        # the column branch flags of the last call, (ntimes, ncol) int32, in
        # the bit layout of the library's shield_mp_step_flags: bit 0/1 rain
        # falls in the first/second warm_rain pass, bit 2/3/4 ice/snow/
        # graupel fall (no_fall == 0, :349-368, :773-1168), bits 16-23 the
        # first level with stop_k == 1 (:706-724)
        self.flags = None

    def _set_timestep(self, timestep):
        self.ts = set_timestep(self.cfg, timestep)
        self.timestep = timestep

    def __call__(self, state, timestep):
        """Advance one step. ``state`` maps MicrophysicsState attribute names
        to arrays ((L, n) for 3-D, (n,) for ``land``); tendencies are
        accumulated in place, ``wmp`` (and ``qice``/``qsnow`` with de_ice)
        are updated in place. Returns the surface precipitation totals
        (mm/day) as a dict of (n,) arrays: rain, snow, ice, graupel."""
        if timestep != self.timestep:
            self._set_timestep(timestep)
        with np.errstate(all="ignore"):
            return self._step(state, float(timestep))

    def _step(self, s, timestep):
        cfg = self.cfg
        K = _K(cfg, self.setup, self.ts)
        L, n = self.L, self.n
        c_air, c_vap = K.c_air, K.c_vap
        land = s["land"].reshape(n)
        area = self.area
        rdt = K.rdt
        zs = K.zs

        # ---------------- fields_init (microphysics.py:27-276) ----------------
        qi = s["qice"]
        qs = s["qsnow"]
        if cfg.de_ice:
            qi_dt = s["qi_dt"]
            qs_dt = s["qs_dt"]
            qio = qi - timestep * qi_dt
            qin = mx(qio, cfg.qi0_max)
            m = qi > qin
            qs_new = W(m, qs + qi - qin, qs)
            qi_new = W(m, qin, qi)
            dqi = (qin - qio) * rdt
            qs_dt[...] = W(m, qs_dt + qi_dt - dqi, qs_dt)
            qi_dt[...] = W(m, dqi, qi_dt)
            qi[...] = qi_new
            qs[...] = qs_new
        qiz = qi.copy()
        qsz = qs.copy()
        t0 = s["pt"].copy()
        tz = t0.copy()
        dp1 = s["delprsi"].copy()
        dp0 = dp1.copy()
        qvz = s["qvapor"].copy()
        qlz = s["qliquid"].copy()
        qrz = s["qrain"].copy()
        qgz = s["qgraupel"].copy()
        dp1 = dp1 * (1.0 - qvz)
        omq = dp0 / dp1
        qvz = qvz * omq
        qlz = qlz * omq
        qrz = qrz * omq
        qiz = qiz * omq
        qsz = qsz * omq
        qgz = qgz * omq
        qa0 = s["qcld"].copy()
        dz0 = s["delz"].copy()
        den0 = -dp1 / (C.GRAV * dz0)
        p1 = den0 * C.RDGAS * t0
        qv0, ql0, qr0, qi0, qs0, qg0 = qvz, qlz, qrz, qiz, qsz, qgz
        m1 = np.zeros((L, n))
        u0 = s["ua"].copy()
        v0 = s["va"].copy()
        u1 = u0.copy()
        v1 = v0.copy()
        if cfg.prog_ccn:
            ccn = np.zeros((L, n)) * 1.0e6  # self._qn is always zero
            c_praut = K.cpaut * (ccn * RHOR) ** (-1.0 / 3.0)
        else:
            ccn = np.broadcast_to((cfg.ccn_l * land + cfg.ccn_o * (1.0 - land)) * 1.0e6, (L, n)).copy()
            if K.use_ccn:
                ccn[L - 1] = ccn[L - 1] * C.RDGAS * tz[L - 1] / p1[L - 1]
                for k in range(L - 2, -1, -1):
                    ccn[k] = ccn[k + 1]
            c_praut = K.cpaut * (ccn * RHOR) ** (-1.0 / 3.0)
        s_leng = np.sqrt(np.sqrt(area * 1.0e-10))
        t_land = cfg.dw_land * s_leng
        t_ocean = cfg.dw_ocean * s_leng
        h_var = t_land * land + t_ocean * (1.0 - land)
        h_var = mn(0.2, mx(0.01, h_var))
        rh_adj = 1.0 - h_var - cfg.rh_inc
        rh_rain = mx(0.35, rh_adj - cfg.rh_inr)
        h_var = np.broadcast_to(h_var, (L, n))
        rh_adj = np.broadcast_to(rh_adj, (L, n))
        rh_rain = np.broadcast_to(rh_rain, (L, n))
        if cfg.fix_negative:
            cvm = c_air + qvz * c_vap + (qrz + qlz) * C.C_LIQ + (qiz + qsz + qgz) * C.C_ICE
            lcpk = (K.lv00 + K.d0_vap * tz) / cvm
            icpk = (C.LI00 + C.DC_ICE * tz) / cvm
            m = qiz < 0.0
            qsz = W(m, qsz + qiz, qsz)
            qiz = W(m, 0.0, qiz)
            m = qsz < 0.0
            qgz = W(m, qgz + qsz, qgz)
            qsz = W(m, 0.0, qsz)
            m = qgz < 0.0
            qrz = W(m, qrz + qgz, qrz)
            tz = W(m, tz - qgz * icpk, tz)
            qgz = W(m, 0.0, qgz)
            m = qrz < 0.0
            qlz = W(m, qlz + qrz, qlz)
            qrz = W(m, 0.0, qrz)
            m = qlz < 0.0
            qvz = W(m, qvz + qlz, qvz)
            tz = W(m, tz - qlz * lcpk, tz)
            qlz = W(m, 0.0, qlz)
            qvz = qvz.copy()
            for k in range(1, L):
                qvz[k] = W(qvz[k - 1] < 0.0, qvz[k] + qvz[k - 1] * dp1[k - 1] / dp1[k], qvz[k])
            qvz[: L - 1] = W(qvz[: L - 1] < 0.0, 0.0, qvz[: L - 1])
            flag = (qvz[L - 1] < 0.0) & (qvz[L - 2] > 0.0)
            dq = mn(-qvz[L - 1] * dp1[L - 1], qvz[L - 2] * dp1[L - 2])
            qvz[L - 2] = W(flag, qvz[L - 2] - dq / dp1[L - 2], qvz[L - 2])
            qvz[L - 1] = W(flag, qvz[L - 1] + dq / dp1[L - 1], qvz[L - 1])

        rain = np.zeros(n)
        snow = np.zeros(n)
        ice = np.zeros(n)
        graupel = np.zeros(n)
        w = s["wmp"]
        wz = w.copy()
        qaz = self.qaz
        den = np.zeros((L, n))
        denfac = np.zeros((L, n))
        dz1 = np.zeros((L, n))
        m1_sol = np.zeros((L, n))

        def warm_rain(is_first, qgz, qiz, qlz, qrz, qsz, qvz, tz, den, denfac, dz1, wz, m1, m1_sol, rain):
            """microphysics.py:280-653"""
            if is_first:
                dz1 = dz0 * tz / t0
                den = den0 * dz0 / dz1
                denfac = np.sqrt(SFCRHO / den)
            dt5 = 0.5 * K.dt_rain
            m1_rain = np.zeros((L, n))
            no_fall = _column_any(qrz > QRMIN)
            vtrz, r1 = compute_rain_fspeed(K, no_fall, qrz, den)
            fall = no_fall == 0.0
            flags[-1] |= _flag_bits(fall[0], 1 if is_first else 2)
            ze = _ze_column(dz1, zs)
            qgz, qiz, qlz, qrz, qsz, qvz, tz = revap_racc(
                fall, dt5, K, h_var, qgz, qiz, qlz, qrz, qsz, qvz, tz, den, denfac
            )
            if K.do_sedi_w:
                dm = dp1 * (1.0 + qvz + qlz + qrz + qiz + qsz + qgz)
            dz = _dz_from_ze(ze, zs)
            dd = K.dt_rain * vtrz
            qmass, qm, m1_rain_f, sfc = _implicit_fall(fall, qrz, dz, dd, dp1)
            m1_rain = W(fall, m1_rain_f, m1_rain)
            r1 = W(fall, np.broadcast_to(sfc, (L, n)), r1)
            qrz = W(fall, qm / dp1, qmass)
            if K.do_sedi_w:
                wz = _w_transport(fall, wz, dm, m1_rain, vtrz)
            if cfg.do_sedi_heat:
                tz = _sedi_heat(fall, tz, dz1, dp1, qvz, qlz, qrz, qiz, qsz, qgz, m1_rain, C.C_LIQ)
            qgz, qiz, qlz, qrz, qsz, qvz, tz = revap_racc(
                fall, dt5, K, h_var, qgz, qiz, qlz, qrz, qsz, qvz, tz, den, denfac
            )
            if cfg.irain_f != 0:
                qlz, qrz = autoconv_no_subgrid_var(K, qlz, qrz, tz, den, ccn, c_praut)
            else:
                dl = _slope(qlz, cfg.z_slope_liq)
                if dl is not None:
                    dl = mx(dl, mx(QVMIN, h_var * qlz))
                else:
                    dl = mx(QVMIN, h_var * qlz)
                qlz, qrz = autoconv_subgrid_var(K, qlz, qrz, tz, den, ccn, c_praut, dl)
            rain = rain + r1[0]
            if is_first:
                m1 = m1 + m1_rain
            else:
                m1 = m1 + m1_rain + m1_sol
            return qgz, qiz, qlz, qrz, qsz, qvz, tz, den, denfac, dz1, wz, m1, vtrz, rain

        def sedimentation(qgz, qiz, qlz, qrz, qsz, qvz, tz, wz, graupel, ice, rain, snow):
            """microphysics.py:657-1217"""
            vtgz, vtiz, vtsz = fall_speed(K, qgz, qiz, qlz, qsz, tz, den)
            m1_sol = np.zeros((L, n))
            lhi = C.LI00 + C.DC_ICE * tz
            q_liq = qlz + qrz
            q_sol = qiz + qsz + qgz
            cvm = c_air + qvz * c_vap + q_liq * C.C_LIQ + q_sol * C.C_ICE
            icpk = lhi / cvm
            # significant melting level (:706-724)
            stop_k = np.empty((L, n))
            stop_k[0] = W(tz[0] > cfg.tice, 1.0, 0.0)
            for k in range(1, L - 1):
                stop_k[k] = W(stop_k[k - 1] == 0.0, W(tz[k] > cfg.tice, 1.0, 0.0), 1.0)
            stop_k[L - 1] = 1.0
            flags[-1] |= _first_level(stop_k == 1.0) << 16
            tc = tz - cfg.tice
            a = (stop_k == 1.0) & (qiz > QCMIN) & (tc > 0.0)
            sink = mn(qiz, K.fac_imlt * tc / icpk)
            tmp = mn(sink, dim(cfg.ql_mlt, qlz))
            qlz = W(a, qlz + tmp, qlz)
            qrz = W(a, qrz + sink - tmp, qrz)
            qiz = W(a, qiz - sink, qiz)
            q_liq = W(a, q_liq + sink, q_liq)
            q_sol = W(a, q_sol - sink, q_sol)
            cvm = W(a, c_air + qvz * c_vap + q_liq * C.C_LIQ + q_sol * C.C_ICE, cvm)
            tz = W(a, tz - sink * lhi / cvm, tz)
            ze = _ze_column(dz1, zs)
            dz = _dz_from_ze(ze, zs)

            # ice (:773-900)
            no_fall = _column_any(qiz > QRMIN)
            fall = (cfg.vi_fac >= 1.0e-5) & (no_fall == 0.0)
            i1 = np.zeros(n)
            flags[-1] |= _flag_bits(fall[0], 4)
            if K.do_sedi_w:
                dm = dp1 * (1.0 + qvz + qlz + qrz + qiz + qsz + qgz)
            dd = K.dts * vtiz
            qmass, qm, flux, sfc = _implicit_fall(fall, qiz, dz, dd, dp1)
            m1_sol = W(fall, flux, m1_sol)
            i1 = W(fall[0], sfc, i1)
            qiz = W(fall, qm / dp1, qmass)
            if K.do_sedi_w:
                wz = _w_transport(fall, wz, dm, m1_sol, vtiz)

            # snow (:902-1035)
            no_fall = _column_any(qsz > QRMIN)
            fall = no_fall == 0.0
            s1 = np.zeros(n)
            flags[-1] |= _flag_bits(fall[0], 8)
            if K.do_sedi_w:
                dm = dp1 * (1.0 + qvz + qlz + qrz + qiz + qsz + qgz)
            dd = K.dts * vtsz
            qmass, qm, m1_tf, sfc = _implicit_fall(fall, qsz, dz, dd, dp1)
            s1 = W(fall[0], sfc, s1)
            qsz = W(fall, qm / dp1, qmass)
            m1_sol = W(fall, m1_sol + m1_tf, m1_sol)
            if K.do_sedi_w:
                wz = _w_transport(fall, wz, dm, m1_tf, vtsz)

            # graupel (:1037-1168)
            no_fall = _column_any(qgz > QRMIN)
            fall = no_fall == 0.0
            g1 = np.zeros(n)
            flags[-1] |= _flag_bits(fall[0], 16)
            if K.do_sedi_w:
                dm = dp1 * (1.0 + qvz + qlz + qrz + qiz + qsz + qgz)
            dd = K.dts * vtgz
            qmass, qm, m1_tf, sfc = _implicit_fall(fall, qgz, dz, dd, dp1)
            g1 = W(fall[0], sfc, g1)
            qgz = W(fall, qm / dp1, qmass)
            m1_sol = W(fall, m1_sol + m1_tf, m1_sol)
            if K.do_sedi_w:
                wz = _w_transport(fall, wz, dm, m1_tf, vtgz)

            rain = rain + 0.0
            snow = snow + s1
            graupel = graupel + g1
            ice = ice + i1
            if cfg.do_sedi_heat:
                tz = _sedi_heat(
                    np.ones((L, n), dtype=bool), tz, dz1, dp1, qvz, qlz, qrz, qiz, qsz, qgz, m1_sol, C.C_ICE
                )
            return qgz, qiz, qlz, qrz, qsz, qvz, tz, wz, vtgz, vtsz, m1_sol, graupel, ice, rain, snow

        def icloud(qaz, qgz, qiz, qlz, qrz, qsz, qvz, tz, vtgz, vtrz, vtsz):
            """microphysics.py:1220-1449"""
            lhi = C.LI00 + C.DC_ICE * tz
            q_liq = qlz + qrz
            q_sol = qiz + qsz + qgz
            cvm = c_air + qvz * c_vap + q_liq * C.C_LIQ + q_sol * C.C_ICE
            icpk = lhi / cvm
            a = (tz > cfg.tice) & (qiz > QCMIN)
            melt = mn(qiz, K.fac_imlt * (tz - cfg.tice) / icpk)
            tmp = mn(melt, dim(cfg.ql_mlt, qlz))
            b = ~a & (tz < K.t_wfr) & (qlz > QCMIN)
            dtmp = K.t_wfr - tz
            factor = mn(1.0, dtmp / DT_FR)
            sink = mn(qlz * factor, dtmp / icpk)
            qi_crt = cfg.qi_gen * mn(cfg.qi_lim, 0.1 * (cfg.tice - tz)) / den
            tmp2 = mn(sink, dim(qi_crt, qiz))
            qlz_n = W(a, qlz + tmp, W(b, qlz - sink, qlz))
            qrz = W(a, qrz + melt - tmp, qrz)
            qsz = W(b, qsz + sink - tmp2, qsz)
            qiz = W(a, qiz - melt, W(b, qiz + tmp2, qiz))
            qlz = qlz_n
            q_liq = W(a, q_liq + melt, W(b, q_liq - sink, q_liq))
            q_sol = W(a, q_sol - melt, W(b, q_sol + sink, q_sol))
            cvm = W(a | b, c_air + qvz * c_vap + q_liq * C.C_LIQ + q_sol * C.C_ICE, cvm)
            tz = W(a, tz - melt * lhi / cvm, W(b, tz + sink * lhi / cvm, tz))
            di = _slope(qiz, cfg.z_slope_ice)
            if di is not None:
                di = mx(di, mx(QVMIN, h_var * qiz))
            else:
                di = mx(QVMIN, h_var * qiz)
            return icloud_main(
                K, h_var, rh_adj, rh_rain, qaz, qgz, qiz, qlz, qrz, qsz, qvz, tz,
                den, denfac, vtgz, vtrz, vtsz, p1, di, q_liq, q_sol, cvm,
            )

        flags = []
        for _ in range(K.ntimes):
            flags.append(_np.zeros(n, dtype=_np.int32))
            (qgz, qiz, qlz, qrz, qsz, qvz, tz, den, denfac, dz1, wz, m1, vtrz, rain) = warm_rain(
                True, qgz, qiz, qlz, qrz, qsz, qvz, tz, den, denfac, dz1, wz, m1, m1_sol, rain
            )
            (qgz, qiz, qlz, qrz, qsz, qvz, tz, wz, vtgz, vtsz, m1_sol, graupel, ice, rain, snow) = sedimentation(
                qgz, qiz, qlz, qrz, qsz, qvz, tz, wz, graupel, ice, rain, snow
            )
            (qgz, qiz, qlz, qrz, qsz, qvz, tz, den, denfac, dz1, wz, m1, vtrz, rain) = warm_rain(
                False, qgz, qiz, qlz, qrz, qsz, qvz, tz, den, denfac, dz1, wz, m1, m1_sol, rain
            )
            qaz, qgz, qiz, qlz, qrz, qsz, qvz, tz = icloud(
                qaz, qgz, qiz, qlz, qrz, qsz, qvz, tz, vtgz, vtrz, vtsz
            )
        self.qaz = qaz
        self.flags = _np.stack(flags)
        if K.do_sedi_w:
            w[...] = wz

        # ---------------- fields_update (microphysics.py:1452-1553) ----------
        if cfg.sedi_transport:
            for k in range(1, L):
                u1[k] = (dp0[k] * u1[k] + m1[k - 1] * u1[k - 1]) / (dp0[k] + m1[k - 1])
                v1[k] = (dp0[k] * v1[k] + m1[k - 1] * v1[k - 1]) / (dp0[k] + m1[k - 1])
            s["udt"][1:] = s["udt"][1:] + (u1[1:] - u0[1:]) * rdt
            s["vdt"][1:] = s["vdt"][1:] + (v1[1:] - v0[1:]) * rdt
        omq = dp1 / dp0
        s["qv_dt"][...] = s["qv_dt"] + rdt * (qvz - qv0) * omq
        s["ql_dt"][...] = s["ql_dt"] + rdt * (qlz - ql0) * omq
        s["qr_dt"][...] = s["qr_dt"] + rdt * (qrz - qr0) * omq
        s["qi_dt"][...] = s["qi_dt"] + rdt * (qiz - qi0) * omq
        s["qs_dt"][...] = s["qs_dt"] + rdt * (qsz - qs0) * omq
        s["qg_dt"][...] = s["qg_dt"] + rdt * (qgz - qg0) * omq
        cvm = c_air + qvz * c_vap + (qrz + qlz) * C.C_LIQ + (qiz + qsz + qgz) * C.C_ICE
        s["pt_dt"][...] = s["pt_dt"] + rdt * (tz - t0) * cvm / C.CP_AIR
        if cfg.do_qa:
            s["qa_dt"][...] = 0.0
        else:
            s["qa_dt"][...] = s["qa_dt"] + rdt * (qaz / K.ntimes - qa0)
        convt = 86400.0 * rdt * C.RGRAV
        return {
            "rain": rain * convt,
            "snow": snow * convt,
            "ice": ice * convt,
            "graupel": graupel * convt,
        }
