"""CPU oracle for the A-grid to D-grid wind update of the physics tendencies.

TEST INFRASTRUCTURE ONLY (see ``oracle/microphysics.py``).

Restates ``AGrid2DGridPhysics`` (``pySHiELD/update/update_dwind_phys.py``):
the stencils of :12-161 and the sequence and domains of ``__init__`` /
``__call__`` (:171-701), on full storages (k on the last axis). The edge
regions follow the constructor's arithmetic, including its asymmetries
(``global_is < im2`` on the north edge against ``<=`` on the south edge;
the upper south stencil runs whenever ``global_ie > im2``).
"""

import numpy as np


def edge_plan(nx, ny, n_halo, npx, npy, layout, subtile_index, edges):
    """The edge regions of update_dwind_phys.py:214-440 in local storage
    indices. ``edges``: (south, north, west, east). Returns a dict of lists
    of (line, lo, hi, direction) with ``line`` the fixed index (i for the
    west/east lines, j for south/north), [lo, hi) the range along the edge
    and ``direction`` +1 (the region reads its neighbour above) or -1."""
    south, north, west, east = edges
    h = n_halo
    isc, iec, jsc, jec = h, h + nx - 1, h, h + ny - 1
    im2 = int((npx - 1) / 2) + 2
    jm2 = int((npy - 1) / 2) + 2
    wx = int((npx - 1) / layout[0])
    wy = int((npy - 1) / layout[1])
    sy, sx = subtile_index
    g_is, g_js = isc + sx * wx, jsc + sy * wy
    g_ie, g_je = iec + sx * wx, jec + sy * wy

    def loc_y(jg):
        return jg - sy * wy

    def loc_x(ig):
        return ig - sx * wx

    shape0, shape1 = nx + 2 * h + 1, ny + 2 * h + 1
    plan = {"west": [], "east": [], "south": [], "north": []}
    for name, on, i_line in (("west", west, h), ("east", east, shape0 - h - 1)):
        if not on:
            continue
        je_lower = loc_y(min(jm2, g_je))
        lower_n = je_lower - jsc + 1
        upper = None
        if g_je > jm2:
            js_upper = loc_y(max(jm2 + 1, g_js))
            upper_n = jec - js_upper + 1
            if upper_n > 0:
                upper = (i_line, js_upper, js_upper + upper_n, -1)
        lower = (i_line, h, h + lower_n, +1) if (g_js <= jm2 and lower_n > 0) else None
        # order of __call__: lower edge stencil, upper edge stencil + copy, lower copy
        plan[name] = [r for r in (lower, upper) if r is not None]
    for name, on, j_line in (("south", south, h), ("north", north, shape1 - h - 1)):
        if not on:
            continue
        ie_lower = loc_x(min(im2, g_ie))
        lower_n = ie_lower - isc + 1
        if name == "south":
            lower_ok = g_is <= im2 and lower_n > 0
            upper_ok = g_ie > im2
        else:
            lower_ok = g_is < im2 and lower_n > 0
            upper_ok = g_ie >= im2
        upper = None
        if upper_ok:
            is_upper = loc_x(max(im2 + 1, g_is))
            upper_n = iec - is_upper + 1
            if name == "south" or upper_n > 0:
                upper = (j_line, is_upper, is_upper + upper_n, -1)
        lower = (j_line, h, h + lower_n, +1) if lower_ok else None
        plan[name] = [r for r in (lower, upper) if r is not None]
    return plan


def agrid_to_dgrid(u, v, u_dt, v_dt, g, nx, ny, npz, n_halo, dt5, plan):
    """In place on u, v, u_dt, v_dt (storages (I, J, K)). ``g`` maps the
    geometry names (vlon1..3, vlat1..3, es1_1..3, ew2_1..3: (I, J);
    edge_vect_w, edge_vect_e: (I, J); edge_vect_s, edge_vect_n: (I,))."""
    h = n_halo
    ks = slice(0, npz)
    # update_dwind_prep_stencil on origin (h - 1, h - 1), domain (nx + 2, ny + 2)
    pi, pj = slice(h - 1, h + nx + 1), slice(h - 1, h + ny + 1)
    v3 = []
    for m in (1, 2, 3):
        v3.append(u_dt[..., ks] * g[f"vlon{m}"][..., None] + v_dt[..., ks] * g[f"vlat{m}"][..., None])
    ue, ve = [], []
    for m in range(3):
        a = np.full(u.shape[:2] + (npz,), np.nan)
        b = np.full(u.shape[:2] + (npz,), np.nan)
        a[pi, pj] = v3[m][h - 1 : h + nx + 1, h - 2 : h + ny] + v3[m][pi, pj]
        b[pi, pj] = v3[m][h - 2 : h + nx, h - 1 : h + ny + 1] + v3[m][pi, pj]
        ue.append(a)
        ve.append(b)
    # set_winds_zero on the same domain
    u_dt[pi, pj, ks] = 0.0
    v_dt[pi, pj, ks] = 0.0
    # y edges on ve (west, east): vt = e * ve[j +- 1] + (1 - e) * ve, then copied back
    for name in ("west", "east"):
        ev = g[f"edge_vect_{name[0]}"]
        vts = []
        for i_line, lo, hi, d in plan[name]:
            js = slice(lo, hi)
            e = ev[i_line, js][:, None]
            vts.append((i_line, js, [e * ve[m][i_line, lo + d : hi + d] + (1.0 - e) * ve[m][i_line, js] for m in range(3)]))
        for i_line, js, vt in vts[::-1]:  # the upper copy runs before the lower one
            for m in range(3):
                ve[m][i_line, js] = vt[m]
    # x edges on ue (south, north)
    for name in ("south", "north"):
        ev = g[f"edge_vect_{name[0]}"]
        uts = []
        for j_line, lo, hi, d in plan[name]:
            isl = slice(lo, hi)
            e = ev[isl][:, None]
            uts.append((j_line, isl, [e * ue[m][lo + d : hi + d, j_line] + (1.0 - e) * ue[m][isl, j_line] for m in range(3)]))
        for j_line, isl, ut in uts[::-1]:
            for m in range(3):
                ue[m][isl, j_line] = ut[m]
    # update_uwind_stencil on (nx, ny + 1), update_vwind_stencil on (nx + 1, ny)
    ui, uj = slice(h, h + nx), slice(h, h + ny + 1)
    u[ui, uj, ks] = u[ui, uj, ks] + dt5 * (
        ue[0][ui, uj] * g["es1_1"][ui, uj, None] + ue[1][ui, uj] * g["es1_2"][ui, uj, None]
        + ue[2][ui, uj] * g["es1_3"][ui, uj, None]
    )
    vi, vj = slice(h, h + nx + 1), slice(h, h + ny)
    v[vi, vj, ks] = v[vi, vj, ks] + dt5 * (
        ve[0][vi, vj] * g["ew2_1"][vi, vj, None] + ve[1][vi, vj] * g["ew2_2"][vi, vj, None]
        + ve[2][vi, vj] * g["ew2_3"][vi, vj, None]
    )


def doubly_periodic(u, v, u_dt, v_dt, nx, ny, npz, n_halo, dt5):
    """doubly_periodic_wind_update (update_dwind_phys.py:153-161) on the
    compute domain."""
    h = n_halo
    ci, cj, ks = slice(h, h + nx), slice(h, h + ny), slice(0, npz)
    u[ci, cj, ks] = u[ci, cj, ks] + dt5 * (u_dt[ci, h - 1 : h + ny - 1, ks] + u_dt[ci, cj, ks])
    v[ci, cj, ks] = v[ci, cj, ks] + dt5 * (v_dt[h - 1 : h + nx - 1, cj, ks] + v_dt[ci, cj, ks])
