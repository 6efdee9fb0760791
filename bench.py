"""Benchmark of the GFDL microphysics step (column-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--levels 79] [--form plain|mixed]

Workload: C96 (6 x 96 x 96 = 55,296 columns) x 79 levels, one
``Microphysics.__call__`` of 180 s per step, on a seeded synthetic state
(no public dataset exists for this path; the distributions are those of
``pyshield_b200.inputs``). The arrays are NDSL-layout storages (halo 3,
i-fastest), as a GT4Py GPU backend would hand them over. One step moves
1.26 GB, far more than the 126 MB L2, so no L2 flush is needed between
steps.

Reported (one JSON line, rank 0):
  value      column-steps/s over all ranks, inputs resident in HBM, timed with
             CUDA events on the launching stream (max over ranks);
  e2e        the same metric through the public API with host buffers: every
             step's inputs copied from pinned host memory to the device and
             its outputs copied back, inside the timed region (the copies run
             on their own streams and overlap the neighbouring steps'
             compute, see HostPipeline);
  roofline   HBM roofline of the dominant kernel: algorithmic bytes
             (36 fields x L x 8 B + 48 B per column-step) per launch / mean
             launch time, against the measured copy bandwidth;
  cpu_baseline  the FP64 numpy oracle (the restatement of the reference's numpy
             backend) on the host cores, on a bounded sample of columns.

--impl reference times that CPU implementation on the workload's metric
(each step a bounded sample of the columns, all host cores).
Multi-GPU: one process per GPU under torchrun; the columns are independent,
so every rank advances its own C96 domain (weak scaling, no collective on
the data path); the timing is the max over ranks.
"""

import argparse
import json
import multiprocessing as mp_
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

N_CUBE = 96
DT = 180.0
HALO = 3


# DRAM bytes (read + write) per algorithmic byte of the step kernel, from an
# ncu capture of the C48 L79 workload (dram__bytes_read.sum +
# dram__bytes_write.sum = 239.38 + 88.32 MB for 315.19 MB of algorithmic
# traffic; the extra writes are register spills that reach DRAM); the
# kernel streams each field once, so the ratio carries over to C96.
NCU_TRAFFIC_RATIO = (239.381248 + 88.321024) / 315.19

# FP64 flops per column-step of the plain step kernel (2 per DFMA, 1 per
# DADD or DMUL, thread-level counts of predicated-on instructions), from an
# ncu capture of the C48 launch divided by its columns; by level count.
FP64_FLOPS_PER_COLUMN_STEP = {79: (2 * 1419707201 + 566933197 + 677884763) / 13824}


def algorithmic_bytes_per_column_step(nlev):
    """Reads: 13 state fields, 10 tendencies (accumulated) and the persistent
    cloud-fraction accumulator; writes: 10 tendencies, wmp and the
    accumulator (36 fields x L x 8 B); per column: land, area read and four
    precipitation totals written (48 B)."""
    return 36 * nlev * 8 + 48


# ------------------------------------------------------------ CPU baseline
def _oracle_worker(conn, n, nlev, seed):
    """One host process of OracleDomain: owns ``n`` columns of the domain
    (its own seeded state) and advances them by one step per request. The
    state copy for the next step is made before the request arrives, so the
    timed step is the oracle's work alone."""
    sys.path.insert(0, REPO)
    from oracle.microphysics import OracleMicrophysics
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.inputs import copy_state, make_state

    state, area = make_state(n, nlev, seed=seed, n_cube=N_CUBE)
    m = OracleMicrophysics(PhysicsConfig(dt_atmos=DT), n, nlev, area)
    nxt = copy_state(state)
    conn.send("ready")
    while conn.recv() is not None:
        t0 = time.perf_counter()
        m(nxt, DT)
        dt = time.perf_counter() - t0
        conn.send(dt)
        nxt = copy_state(state)
    conn.close()


class OracleDomain:
    """The FP64 numpy oracle advancing a whole domain of ``ncol`` columns per
    step, the columns split into ``cores`` contiguous slices, one persistent
    host process each (spawned, so it may start before or after CUDA is
    initialised). ``step()`` returns the wall time of one whole-domain step:
    from the request to the last slice's reply."""

    def __init__(self, ncol, nlev, cores):
        ctx = mp_.get_context("spawn")
        base, extra = divmod(ncol, cores)
        self.sizes = [base + (1 if i < extra else 0) for i in range(cores)]
        self.ncol, self.nlev, self.cores = ncol, nlev, cores
        self.conns, self.procs = [], []
        for i, n in enumerate(self.sizes):
            a, b = ctx.Pipe()
            p = ctx.Process(target=_oracle_worker, args=(b, n, nlev, 100 + i), daemon=True)
            p.start()
            self.conns.append(a)
            self.procs.append(p)
        for c in self.conns:
            assert c.recv() == "ready"

    def step(self):
        t0 = time.perf_counter()
        for c in self.conns:
            c.send(1)
        for c in self.conns:
            c.recv()
        return time.perf_counter() - t0

    def close(self):
        for c in self.conns:
            c.send(None)
        for p in self.procs:
            p.join(timeout=30)


def cpu_baseline(domain, steps, warmup=1):
    """Whole-domain steps of the oracle: returns (column-steps/s, seconds per
    step, sample description)."""
    for _ in range(warmup):
        domain.step()
    t = sum(domain.step() for _ in range(steps))
    per = t / steps
    sample = (f"{steps} whole-domain step(s) of {domain.ncol} columns x {domain.nlev} levels (dt {DT:g} s), "
              f"columns split over {domain.cores} host processes, numpy FP64 oracle")
    return domain.ncol / per, per, sample


# ------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock samples every 20 ms from a reader thread, each with its
    host time, so that the samples of a short timed region can be picked out:
    ``start()`` waits for the first sample (nvidia-smi takes a moment to come
    up), ``mark()`` brackets the timed region, ``stop()`` summarises the samples
    inside it (the nearest ones if the region was shorter than the interval)."""

    FIELDS = (
        "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
        "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
        "clocks_event_reasons.sw_power_cap"
    )
    INTERVAL_MS = 20

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.window = [None, None]
        self.thread = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line))

    def start(self, wait_s=5.0):
        import threading

        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.INTERVAL_MS)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
            )
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        t_end = time.monotonic() + wait_s
        while not self.lines and time.monotonic() < t_end and self.proc.poll() is None:
            time.sleep(0.01)

    def mark(self, which):
        self.window[0 if which == "begin" else 1] = time.monotonic()

    @staticmethod
    def _parse(line):
        parts = [p.strip() for p in line.split(",")]
        if len(parts) < 7:
            return None
        try:
            return float(parts[0]), float(parts[1]), parts[3:7]
        except ValueError:
            return None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            self.proc.wait()
        if self.thread is not None:
            self.thread.join(timeout=5)
        rows = [(t, r) for t, r in ((t, self._parse(x)) for t, x in self.lines) if r is not None]
        t0, t1 = self.window
        inside = rows
        if t0 is not None and t1 is not None:
            # a sample printed within one interval after the region still
            # describes it
            inside = [x for x in rows if t0 <= x[0] <= t1 + self.INTERVAL_MS / 1000.0]
            if not inside and rows:
                mid = 0.5 * (t0 + t1)
                inside = sorted(rows, key=lambda x: abs(x[0] - mid))[:2]
        sm = [r[0] for _, r in inside]
        smax = [r[1] for _, r in inside]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for _, r in inside:
            for name, v in zip(names, r[2]):
                if v.lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "samples": len(sm),
            "samples_total": len(rows),
            "interval_ms": self.INTERVAL_MS,
            "reasons": sorted(reasons),
        }


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def fp64_peak(reps=5):
    """Measured FP64 throughput of this GPU (TFLOP/s): CUDA-event time of the
    FP64 probe (libshield_probe.so; independent DFMA chains on every SM, 2
    flops per DFMA), the mean of ``reps`` launches after a warm-up, with
    nothing changed on the GPU."""
    import ctypes

    import torch

    from pyshield_b200.build import PROBE_LIB

    lib = ctypes.CDLL(PROBE_LIB)
    lib.shield_probe_dfma.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                      ctypes.c_void_p]
    nsm = lib.shield_probe_sm_count()
    bps, iters = 8, 20000
    out = torch.empty(nsm * bps, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    flops = ctypes.c_double()

    def launch():
        rc = lib.shield_probe_dfma(ctypes.c_void_p(out.data_ptr()), bps, iters, ctypes.byref(flops),
                                   ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, f"FP64 probe launch failed ({rc})"

    launch()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        launch()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    return flops.value / (ms / 1000.0) / 1e12


# ------------------------------------------------------------ GPU arm
def build_state(nlev, device, seed, n_cube=N_CUBE, sat_fraction=0.0):
    """Synthetic C96 state as NDSL-layout torch storages on ``device``."""
    import numpy as np
    import torch

    from pyshield_b200.grid import GridData, GridIndexing, QuantityFactory, StencilFactory
    from pyshield_b200.inputs import make_state
    from pyshield_b200.microphysics import MicrophysicsState
    from pyshield_b200.quantity import Quantity

    nx, ny = n_cube, 6 * n_cube  # the six tiles side by side
    n = nx * ny
    state, area = make_state(n, nlev, seed=seed, n_cube=n_cube, sat_fraction=sat_fraction)
    gi = GridIndexing(nx, ny, nlev, HALO)
    qf = QuantityFactory(gi, device=device)
    host = {}

    def put(name, arr_ln):
        q = qf.zeros(["x", "y", "z"], "")
        v = q.view  # (nx, ny, nlev) view of i-fastest storage
        src = torch.from_numpy(np.ascontiguousarray(arr_ln.reshape(nlev, ny, nx)))
        v.copy_(src.permute(2, 1, 0).to(device))
        host[name] = src
        return q

    qs = {k: put(k, v) for k, v in state.items() if k != "land"}
    land = qf.zeros(["x", "y"], "")
    land.view.copy_(torch.from_numpy(state["land"].reshape(ny, nx).T.copy()).to(device))
    area_q = qf.zeros(["x", "y"], "")
    area_q.view.copy_(torch.from_numpy(area.reshape(ny, nx).T.copy()).to(device))
    tend = qf.zeros(["x", "y", "z"], "")
    ms = MicrophysicsState(
        qs["pt"], qs["qvapor"], qs["qliquid"], qs["qrain"], qs["qice"], qs["qsnow"], qs["qgraupel"], qs["qcld"],
        qs["ua"], qs["va"], qf.zeros(["x", "y", "z"], ""), qs["delz"], qf.zeros(["x", "y", "z"], ""), qs["delprsi"],
        qs["wmp"], qf.zeros(["x", "y", "z"], ""), tend, land,
    )
    for t in ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt"):
        setattr(ms, t, qs[t])
    return ms, StencilFactory(gi), qf, GridData(area_q), host, land, (nx, ny, n)


def run_adjoint(nsteps_window=8, reps=5, n_cube=96, nlev=79, dt=150.0, window=True):
    """Adjoint cost at C96 L79 (C48 without the window beside it): the device
    time of one VJP of the step (shield_mp_step_vjp) against one forward step,
    and of an nsteps window (forward steps with the state update, then the
    backward through torch.autograd with per-step checkpointing) against the
    window's forward alone. Each timing is the mean of ``reps`` runs after a
    warm-up."""
    import torch

    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.adjoint import OUTPUTS, STATE, rollout, step_forward, step_vjp
    from pyshield_b200.microphysics import Microphysics

    device = torch.device("cuda", torch.cuda.current_device())
    ms, sf, qf, gd, host, land, (nx, ny, n) = build_state(nlev, device, seed=77, n_cube=n_cube)
    mp = Microphysics(sf, qf, gd, PhysicsConfig(dt_atmos=int(dt)))
    x = [getattr(ms, f).view.clone() for f in STATE[:-1]]
    x.append(torch.zeros((nx, ny, nlev), dtype=torch.float64, device=device))
    lnd = land.view.clone()
    y = step_forward(mp, x, lnd, dt)
    g = torch.Generator(device=device).manual_seed(1)

    def cotangent(v):
        # a cotangent in its output's own layout (i fastest, as the step writes them)
        t = torch.randn(tuple(reversed(v.shape)), generator=g, device=device, dtype=torch.float64)
        return t.permute(*reversed(range(v.dim())))

    ybar = [cotangent(v) for v in y]
    stream = torch.cuda.current_stream()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    fwd_ms = timed(lambda: mp(ms, dt))
    vjp_ms = timed(lambda: step_vjp(mp, x, lnd, ybar, dt))
    res = {
        "workload": f"GFDL microphysics step, C{n_cube} ({n} columns) x L{nlev}, dt {dt:g} s, FP64",
        "forward_ms": fwd_ms,
        "vjp_ms": vjp_ms,
        "vjp_over_forward": vjp_ms / fwd_ms,
    }
    if not window:
        return res

    def window_forward():
        with torch.no_grad():
            rollout(mp, dict(zip(STATE, x)), lnd, dt, nsteps_window)

    def window_backward():
        xs = [t.clone().requires_grad_(True) for t in x]
        final, _ = rollout(mp, dict(zip(STATE, xs)), lnd, dt, nsteps_window)
        loss = sum(final[f].sum() for f in STATE)
        torch.autograd.grad(loss, xs)

    wf_ms = timed(window_forward)
    wb_ms = timed(window_backward)
    res.update({
        "window_steps": nsteps_window,
        "window_forward_ms": wf_ms,
        "window_forward_and_backward_ms": wb_ms,
        "window_backward_over_forward": (wb_ms - wf_ms) / wf_ms,
        "note": "device time (CUDA events); the window keeps each step's inputs and recomputes inside the step",
    })
    return res


E2E_IN = ("pt", "qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qcld", "ua", "va", "delprsi", "delz",
          "wmp")
# The tendencies start every step at zero: Physics.__call__'s
# prepare_microphysics zeroes them on the device before the microphysics
# (physics.py:133-143), so a host never uploads them.
E2E_ZERO = ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt")
E2E_OUT = ("pt_dt", "qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt", "qa_dt", "udt", "vdt", "wmp")


class HostPipeline:
    """The step driven from host memory, as a host that keeps its state on
    the CPU would drive it.

    Every step uploads its 13 state fields and the land mask from pinned host
    memory (one contiguous DMA, fields in the host's (k, j, i) array order),
    scatters them into the device storages, zeroes the 10 tendencies on the
    device (as the physics driver does before the microphysics), calls
    ``mp(ms, dt)`` (the public API), gathers the 11 result fields and the 4
    precipitation totals into one device buffer and downloads it into pinned
    host memory (one DMA).

    Uploads and downloads run on their own streams with two staging buffers
    each way, so step s+1's upload and step s-1's download overlap step s's
    compute; the PCIe link carries both directions at once."""

    def __init__(self, ms, mp, land, host, dims, device):
        import torch

        nx, ny, nz = dims
        self.ms, self.mp, self.land, self.dims = ms, mp, land, dims
        self.plane, self.p2 = nz * ny * nx, ny * nx
        n_in = len(E2E_IN) * self.plane + self.p2
        n_out = len(E2E_OUT) * self.plane + 4 * self.p2
        h_in = torch.empty(n_in, dtype=torch.float64).pin_memory()
        for i, f in enumerate(E2E_IN):
            h_in[i * self.plane:(i + 1) * self.plane].copy_(host[f].reshape(-1))
        h_in[len(E2E_IN) * self.plane:].copy_(land.view.t().reshape(-1).cpu())
        self.h_in = h_in
        self.h_out = [torch.empty(n_out, dtype=torch.float64).pin_memory() for _ in range(2)]
        self.d_in = [torch.empty(n_in, dtype=torch.float64, device=device) for _ in range(2)]
        self.d_out = [torch.empty(n_out, dtype=torch.float64, device=device) for _ in range(2)]
        self.h2d_bytes, self.d2h_bytes = n_in * 8, n_out * 8
        self.up, self.down = torch.cuda.Stream(device), torch.cuda.Stream(device)

    def _field(self, buf, i):
        nx, ny, nz = self.dims
        return buf[i * self.plane:(i + 1) * self.plane].view(nz, ny, nx).permute(2, 1, 0)

    def run(self, steps):
        """Run ``steps`` host-to-host steps; return their device time (ms) from
        the first upload to the last download."""
        import torch

        nx, ny, nz = self.dims
        comp = torch.cuda.current_stream()
        ev = lambda: torch.cuda.Event()  # noqa: E731
        up_done, scat_done = [ev(), ev()], [ev(), ev()]
        gath_done, down_done = [ev(), ev()], [ev(), ev()]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(comp)
        self.up.wait_event(e0)
        self.down.wait_event(e0)
        for s in range(steps):
            b = s % 2
            with torch.cuda.stream(self.up):
                if s >= 2:
                    self.up.wait_event(scat_done[b])
                self.d_in[b].copy_(self.h_in, non_blocking=True)
                up_done[b].record(self.up)
            comp.wait_event(up_done[b])
            for i, f in enumerate(E2E_IN):
                getattr(self.ms, f).view.copy_(self._field(self.d_in[b], i))
            self.land.view.copy_(self.d_in[b][len(E2E_IN) * self.plane:].view(ny, nx).t())
            scat_done[b].record(comp)
            for t in E2E_ZERO:
                getattr(self.ms, t).data.zero_()
            self.mp(self.ms, DT)
            if s >= 2:
                comp.wait_event(down_done[b])
            for i, f in enumerate(E2E_OUT):
                self._field(self.d_out[b], i).copy_(getattr(self.ms, f).view)
            self.d_out[b][len(E2E_OUT) * self.plane:].view(4, ny, nx).copy_(self.mp._precip)
            gath_done[b].record(comp)
            with torch.cuda.stream(self.down):
                self.down.wait_event(gath_done[b])
                self.h_out[b].copy_(self.d_out[b], non_blocking=True)
                down_done[b].record(self.down)
        for b in range(min(steps, 2)):
            comp.wait_event(down_done[b])
        e1.record(comp)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def link_only(self, steps):
        """The link's own time for ``steps`` steps' copies, no compute: the
        same uploads and downloads on their two streams at once, then each
        direction alone. Returns ms per step (both, upload, download)."""
        import torch

        comp = torch.cuda.current_stream()

        def timed(up, down):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(comp)
            self.up.wait_event(e0)
            self.down.wait_event(e0)
            for s in range(steps):
                b = s % 2
                if up:
                    with torch.cuda.stream(self.up):
                        self.d_in[b].copy_(self.h_in, non_blocking=True)
                if down:
                    with torch.cuda.stream(self.down):
                        self.h_out[b].copy_(self.d_out[b], non_blocking=True)
            ue, de = torch.cuda.Event(), torch.cuda.Event()
            ue.record(self.up)
            de.record(self.down)
            comp.wait_event(ue)
            comp.wait_event(de)
            e1.record(comp)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / steps

        return timed(True, True), timed(True, False), timed(False, True)


def link_record(r):
    """The e2e step against the link: the per-step copies alone (both
    directions at once, as the pipeline runs them; each direction alone)."""
    if not r.get("link"):
        return None
    both, up, down = r["link"]
    e2e_step = r["e2e_ms"] / r["e2e_steps"]
    return {"copies_alone_ms_per_step": both, "e2e_ms_per_step": e2e_step, "frac": both / e2e_step,
            "h2d_alone_gbs": r["h2d"] / (up * 1e6), "d2h_alone_gbs": r["d2h"] / (down * 1e6),
            "both_gbs": (r["h2d"] + r["d2h"]) / (both * 1e6),
            "note": "device time (CUDA events) of the pipeline's own pinned copies without the step: the link's "
                    "bound on the host-to-host rate"}


def prestep_bytes(nx, ny, nz, h=HALO):
    """Algorithmic HBM bytes of one shield_physics_prestep launch: each field
    that statein, get_prs_fv3, get_phi_fv3 and prepare_microphysics read is
    read once and each they write is written once. A compute column reads
    delp and the 7 tracers on nz + 1 levels and delz, qsgs_tke, pt, omga on
    nz; it writes phii, prsi, prsik, the 7 tracers and delp on nz + 1 levels
    and qsgs_tke, dm, delprsi, del_gz, phil, dz, wmp and the 10 tendencies on
    nz. A halo column reads prsi, phii (nz + 1) and pt, qvapor (nz) and
    writes phii (nz + 1), delprsi, del_gz and phil (nz)."""
    L, L1 = nz, nz + 1
    ncomp = nx * ny
    nhalo = (nx + 2 * h) * (ny + 2 * h) - ncomp
    return 8 * (ncomp * (19 * L1 + 21 * L) + nhalo * (3 * L1 + 5 * L))


def run_physics(n_cube=N_CUBE, nlev=79, dt=DT, reps=5):
    """pySHiELD's Physics.__call__ at CN x nlev: the fused driver pre-step
    kernel, the microphysics step and the state update. Every step starts
    from the same storages (restored outside the timed region, as a model
    hands the physics a fresh dycore state each step); each call is timed
    with CUDA events, and the pre-step launch alone likewise."""
    import numpy as np
    import torch

    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.grid import GridData, GridIndexing, QuantityFactory, StencilFactory
    from pyshield_b200.inputs import PHYSICS_3D, PHYSICS_INTERFACE, PTOP, TENDENCY_FIELDS, make_physics_state
    from pyshield_b200.physics import Physics, PhysicsState
    from pyshield_b200.quantity import Quantity

    nx, ny = n_cube, 6 * n_cube
    st, area = make_physics_state(nx, ny, nlev, seed=99, halo=HALO)

    def dev3(a):
        return torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).cuda().permute(2, 1, 0)

    def dev2(a):
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()

    gi = GridIndexing(nx, ny, nlev, HALO)
    qf = QuantityFactory(gi)
    q = {}
    for nm in PHYSICS_3D:
        dims = ("x", "y", "z_interface" if nm in PHYSICS_INTERFACE else "z")
        q[nm] = Quantity(dev3(st[nm]), dims, "", (HALO, HALO, 0), (nx, ny, nlev + 1 if nm in PHYSICS_INTERFACE else nlev))
    q["land"] = Quantity(dev2(st["land"]), ("x", "y"), "", (HALO, HALO), (nx, ny))
    cfg = PhysicsConfig(dt_atmos=int(dt))
    ps = PhysicsState(**q, quantity_factory=qf, schemes=cfg.schemes)
    area_st = np.zeros(st["land"].shape)
    area_st[HALO:HALO + nx, HALO:HALO + ny] = area.reshape(ny, nx).T
    phys = Physics(StencilFactory(gi), qf, GridData(Quantity(dev2(area_st), ("x", "y"), "m^2", (HALO, HALO), (nx, ny)), PTOP), cfg)
    pristine = {nm: q[nm].data.clone() for nm in PHYSICS_3D}
    pristine.update({t: dev3(st[t]) for t in TENDENCY_FIELDS})
    del st

    def restore():
        for nm in PHYSICS_3D:
            q[nm].data.copy_(pristine[nm])
        for t in TENDENCY_FIELDS:
            getattr(ps.microphysics, t).data.copy_(pristine[t])

    stream = torch.cuda.current_stream()

    def timed(fn):
        total = 0.0
        for r in range(reps + 1):
            restore()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            if r > 0:  # the first call warms up
                total += e0.elapsed_time(e1)
        return total / reps

    full_ms = timed(lambda: phys(ps, dt))
    pre_ms = timed(lambda: phys.prestep(ps))
    nbytes = prestep_bytes(nx, ny, nlev)
    peak, peak_kind = peaks()
    achieved = nbytes / (pre_ms / 1000.0) / 1e9
    ncol = nx * ny
    # DycoreToPhysics then Physics, as two calls and with the copy fused into
    # the pre-step launch (a dycore state of the copy's 16 fields)
    import types

    from pyshield_b200.coupling import D2P_FIELDS, DycoreToPhysics

    dyc = types.SimpleNamespace(**{f: Quantity(q[f].data.clone(), ("x", "y", "z"), "", (HALO, HALO, 0),
                                               (nx, ny, nlev)) for f in D2P_FIELDS})
    d2p = DycoreToPhysics(StencilFactory(gi), qf, None, False, False)

    def copy_then_physics():
        d2p(dyc, ps)
        phys(ps, dt)

    sep_ms = timed(copy_then_physics)
    fused_ms = timed(lambda: phys(ps, dt, dycore_state=dyc))
    sep_pre_ms = timed(lambda: (d2p(dyc, ps), phys.prestep(ps)))
    fused_pre_ms = timed(lambda: phys.prestep(ps, dycore_state=dyc))
    return {
        "workload": f"Physics.__call__ (driver pre-steps, microphysics, state update), C{n_cube} ({ncol} columns) "
                    f"x L{nlev}, dt {dt:g} s, FP64",
        "ms_per_step": full_ms,
        "column_steps_per_s": ncol / (full_ms / 1000.0),
        "prestep_ms": pre_ms,
        "prestep_roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "bytes_per_launch": nbytes,
                             "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"},
        "gpu_launches_per_step": 3,
        "with_dycore_copy": {
            "copy_then_physics_ms": sep_ms, "fused_ms": fused_ms,
            "copy_then_prestep_ms": sep_pre_ms, "fused_prestep_ms": fused_pre_ms,
            "note": "DycoreToPhysics.__call__ then Physics.__call__, against Physics.__call__(dycore_state=...) "
                    "with the copy inside the pre-step launch (bit-identical results)"},
        "note": "device time (CUDA events), mean of the timed calls; the storages are restored before each call",
    }


def coupling_bytes(nx, ny, nz, h=HALO):
    """Algorithmic HBM bytes of one shield_update_atmos_state launch with
    apply_tendencies, each field read once and written once: fill_gfs_delp
    reads delp and reads and writes the vapour on nz levels of every column
    of the full domain; a compute column reads 22 more fields (the three
    tendencies, physics-updated winds, temperature and five condensates, the
    physics winds and temperature, six dycore tracers, prsi and the dycore
    temperature) and writes 14 (the three tendencies, delp, six tracers,
    temperature, pe, peln, pk), on nz + 1 levels."""
    nk = nz + 1
    ncomp = nx * ny
    nfull = (nx + 2 * h) * (ny + 2 * h)
    return 8 * (nfull * 3 * (nk - 1) + ncomp * 36 * nk)


def run_coupling(n_cube=N_CUBE, nlev=79, dt=DT, reps=5):
    """UpdateAtmosphereState.__call__ (fill_gfs_delp, prepare_tendencies_and_
    update_tracers, moist_cv, update_pressure_and_surface_winds; one kernel)
    at CN x nlev on random storages of plausible magnitudes; every call
    starts from the same storages (restored outside the timed region)."""
    import types

    import numpy as np
    import torch

    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.coupling import UpdateAtmosphereState
    from pyshield_b200.grid import GridIndexing, StencilFactory
    from pyshield_b200.quantity import Quantity

    nx, ny = n_cube, 6 * n_cube
    shape = (nx + 2 * HALO + 1, ny + 2 * HALO + 1, nlev + 1)
    rng = np.random.default_rng(5)

    def dev(a):
        if a.ndim == 2:
            return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()
        return torch.from_numpy(np.ascontiguousarray(a.transpose(2, 1, 0))).cuda().permute(2, 1, 0)

    def q(a):
        ext = (nx, ny, nlev) if a.ndim == 3 else (nx, ny)
        org = (HALO, HALO, 0) if a.ndim == 3 else (HALO, HALO)
        return Quantity(dev(a), ("x", "y", "z")[: a.ndim], "", org, ext)

    def rnd(lo, hi):
        return rng.uniform(lo, hi, shape)

    f = {}
    for nm in ("u_dt", "v_dt", "pt_dt"):
        f[nm] = rng.normal(0.0, 1e-4, shape)
    for nm in ("pu_ua", "pu_va", "ph_ua", "ph_va", "dy_ua", "dy_va"):
        f[nm] = rnd(-30.0, 30.0)
    for nm in ("pu_pt", "ph_pt", "dy_pt"):
        f[nm] = rnd(200.0, 300.0)
    for nm in ("qvapor", "qliquid", "qrain", "qsnow", "qice", "qgraupel"):
        f["pu_" + nm] = rnd(0.0, 2e-3)
        f["dy_" + nm] = rnd(0.0, 2e-3)
    f["prsi"] = np.cumsum(rnd(50.0, 2000.0), axis=2)
    f["dy_delp"] = rnd(50.0, 2000.0)
    f["pe"] = np.zeros(shape)
    f["pe"][..., 0] = 100.0
    f["peln"] = np.zeros(shape)
    f["pk"] = np.zeros(shape)
    Q = {k: q(v) for k, v in f.items()}
    pristine = {k: v.data.clone() for k, v in Q.items()}
    del f
    d = types.SimpleNamespace(
        qvapor=Q["dy_qvapor"], qliquid=Q["dy_qliquid"], qrain=Q["dy_qrain"], qsnow=Q["dy_qsnow"],
        qice=Q["dy_qice"], qgraupel=Q["dy_qgraupel"], delp=Q["dy_delp"], pt=Q["dy_pt"], pe=Q["pe"],
        peln=Q["peln"], pk=Q["pk"], ua=Q["dy_ua"], va=Q["dy_va"], ps=q(np.zeros(shape[:2])),
    )
    p = types.SimpleNamespace(
        physics_updated_ua=Q["pu_ua"], physics_updated_va=Q["pu_va"], physics_updated_pt=Q["pu_pt"],
        physics_updated_specific_humidity=Q["pu_qvapor"], physics_updated_qliquid=Q["pu_qliquid"],
        physics_updated_qrain=Q["pu_qrain"], physics_updated_qsnow=Q["pu_qsnow"], physics_updated_qice=Q["pu_qice"],
        physics_updated_qgraupel=Q["pu_qgraupel"], ua=Q["ph_ua"], va=Q["ph_va"], pt=Q["ph_pt"], prsi=Q["prsi"],
    )
    uas = UpdateAtmosphereState(StencilFactory(GridIndexing(nx, ny, nlev, HALO)), None, PhysicsConfig(dt_atmos=int(dt)))
    stream = torch.cuda.current_stream()
    total = 0.0
    for r in range(reps + 1):
        for k, v in Q.items():
            v.data.copy_(pristine[k])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        uas(d, p, Q["u_dt"], Q["v_dt"], Q["pt_dt"], dt)
        e1.record(stream)
        torch.cuda.synchronize()
        if r > 0:
            total += e0.elapsed_time(e1)
    ms = total / reps
    nbytes = coupling_bytes(nx, ny, nlev)
    peak, peak_kind = peaks()
    achieved = nbytes / (ms / 1000.0) / 1e9
    return {
        "workload": f"UpdateAtmosphereState.__call__ column stencils, C{n_cube} ({nx * ny} columns) x L{nlev}, FP64",
        "ms_per_step": ms,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "bytes_per_launch": nbytes,
                     "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"},
        "note": "device time (CUDA events), mean of the timed calls; the storages are restored before each call",
    }


def d2p_bytes(nx, ny, nz):
    """Algorithmic HBM bytes of one shield_copy_dycore_to_physics launch: 16
    fields read and written on the compute domain plus one interface point
    in x and y, levels 0 .. nz - 1."""
    return 8 * 2 * 16 * (nx + 1) * (ny + 1) * nz


def run_d2p(n_cube=N_CUBE, nlev=79, reps=5):
    """DycoreToPhysics.__call__'s copy at CN x nlev (all six tiles side by
    side), CUDA events around each call."""
    import torch

    from pyshield_b200.coupling import D2P_FIELDS, DycoreToPhysics
    from pyshield_b200.grid import GridIndexing, QuantityFactory, StencilFactory
    from pyshield_b200.quantity import Quantity

    nx, ny = n_cube, 6 * n_cube
    shape = (nlev + 1, ny + 2 * HALO + 1, nx + 2 * HALO + 1)
    gen = torch.Generator(device="cuda").manual_seed(7)

    class State:
        pass

    ds, ps = State(), State()
    for f in D2P_FIELDS:
        for st in (ds, ps):
            t = torch.rand(shape, dtype=torch.float64, device="cuda", generator=gen).permute(2, 1, 0)
            setattr(st, f, Quantity(t, ("x", "y", "z"), "", (HALO, HALO, 0), (nx, ny, nlev)))
    gi = GridIndexing(nx, ny, nlev, HALO)
    d2p = DycoreToPhysics(StencilFactory(gi), QuantityFactory(gi), None, False, False)
    stream = torch.cuda.current_stream()
    d2p(ds, ps)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        d2p(ds, ps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    nbytes = d2p_bytes(nx, ny, nlev)
    peak, peak_kind = peaks()
    achieved = nbytes / (ms / 1000.0) / 1e9
    return {
        "workload": f"DycoreToPhysics.__call__ copy of 16 fields, C{n_cube} ({nx * ny} columns) x L{nlev}, FP64",
        "ms_per_step": ms,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "bytes_per_launch": nbytes,
                     "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"},
        "note": "device time (CUDA events), mean of back-to-back calls; 2.3 GB of storages, more than L2",
    }


def dwind_bytes(nx, ny, nz):
    """Algorithmic HBM bytes of one shield_agrid_to_dgrid call on a tile
    whose four edges are cube edges: the tendencies read where the u and v
    points average them (nx ny + 2 nx + 2 ny points each), u read and written
    on nx x (ny + 1), v on (nx + 1) x ny, both tendencies zeroed on the prep
    domain (nx + 2) x (ny + 2), at nz levels; and the 2-D geometry: six
    vector components on the tendencies' points, three on each wind's."""
    nt = nx * ny + 2 * nx + 2 * ny
    nu, nv, nz0 = nx * (ny + 1), (nx + 1) * ny, (nx + 2) * (ny + 2)
    return 8 * (nz * (2 * nt + 2 * nu + 2 * nv + 2 * nz0) + 6 * nt + 3 * nu + 3 * nv)


def run_dwind(n_cube=N_CUBE, nlev=79, dt=DT, reps=10):
    """AGrid2DGridPhysics.__call__ on the six CN tiles (each its own storages
    and a whole-tile edge plan, as six ranks of a 1 x 1 layout would run it).
    The six calls are captured in one CUDA graph and the replays timed with
    CUDA events: a call moves about 48 MB, a few microseconds of device
    time, so launched from Python the time would be the host's."""
    import types

    import torch

    from pyshield_b200.dwind import AGrid2DGridPhysics
    from pyshield_b200.grid import GridIndexing, StencilFactory
    from pyshield_b200.quantity import Quantity

    nx = ny = n_cube
    h = HALO
    gen = torch.Generator(device="cuda").manual_seed(11)

    def field3(lo, hi):
        t = torch.rand((nlev + 1, ny + 2 * h + 1, nx + 2 * h + 1), dtype=torch.float64, device="cuda",
                       generator=gen) * (hi - lo) + lo
        return Quantity(t.permute(2, 1, 0), ("x", "y", "z"), "", (h, h, 0), (nx, ny, nlev))

    def field2(lo, hi):
        t = torch.rand((ny + 2 * h + 1, nx + 2 * h + 1), dtype=torch.float64, device="cuda", generator=gen)
        return (t * (hi - lo) + lo).t()

    names2 = ("vlon1", "vlon2", "vlon3", "vlat1", "vlat2", "vlat3", "es1_1", "es1_2", "es1_3", "ew2_1", "ew2_2",
              "ew2_3")
    tiles = []
    for _ in range(6):
        gi = GridIndexing(nx, ny, nlev, h)
        gi.south_edge = gi.north_edge = gi.west_edge = gi.east_edge = True
        geom = {n: field2(-1.0, 1.0) for n in names2}
        geom["edge_vect_w"] = field2(0.0, 1.0)
        geom["edge_vect_e"] = field2(0.0, 1.0)
        geom["edge_vect_s"] = torch.rand(nx + 2 * h + 1, dtype=torch.float64, device="cuda", generator=gen)
        geom["edge_vect_n"] = torch.rand(nx + 2 * h + 1, dtype=torch.float64, device="cuda", generator=gen)
        grid_info = types.SimpleNamespace(grid_type=0, **geom)
        part = types.SimpleNamespace(subtile_index=lambda rank: (0, 0))
        namelist = types.SimpleNamespace(dt_atmos=dt, npx=nx + 1, npy=ny + 1, layout=(1, 1))
        a2d = AGrid2DGridPhysics(StencilFactory(gi), None, part, 0, namelist, grid_info)
        q = {k: field3(-30.0, 30.0) for k in ("u", "v")}
        q.update({k: field3(-1e-3, 1e-3) for k in ("u_dt", "v_dt")})
        tiles.append((a2d, q, geom))
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for a2d, q, _ in tiles:
            a2d(q["u"], q["v"], q["u_dt"], q["v_dt"])
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for a2d, q, _ in tiles:
            a2d(q["u"], q["v"], q["u_dt"], q["v_dt"])
    graph.replay()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        graph.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del graph
    # the six tiles in one call (agrid_to_dgrid_tiles: two launches), also replayed from a graph
    from pyshield_b200.dwind import agrid_to_dgrid_tiles

    calls = [(a2d, q["u"], q["v"], q["u_dt"], q["v_dt"]) for a2d, q, _ in tiles]
    with torch.cuda.stream(side):
        agrid_to_dgrid_tiles(calls)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        agrid_to_dgrid_tiles(calls)
    graph.replay()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        graph.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_tiles = e0.elapsed_time(e1) / reps
    del graph
    nbytes = 6 * dwind_bytes(nx, ny, nlev)
    peak, peak_kind = peaks()
    achieved = nbytes / (ms_tiles / 1000.0) / 1e9
    return {
        "workload": f"AGrid2DGridPhysics.__call__ on the six C{n_cube} tiles ({nx} x {ny} x L{nlev} each, "
                    "whole-tile edge plan), FP64",
        "ms_per_step": ms_tiles,
        "launches_per_step": 2,
        "separate_calls_ms": ms,
        "separate_calls_launches": 12,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "bytes_per_launch": nbytes,
                     "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"},
        "note": "device time (CUDA events) of CUDA-graph replays: the six tiles in one agrid_to_dgrid_tiles call "
                "(two launches), and as six AGrid2DGridPhysics calls (two launches each); the six tiles' "
                "storages, 290 MB, are more than L2",
    }


MIXED_ERROR_FIELDS = (("T", "pt_dt", "pt"), ("qv", "qv_dt", "qvapor"), ("qc", "ql_dt", "qliquid"),
                      ("qr", "qr_dt", "qrain"), ("qi", "qi_dt", "qice"), ("qs", "qs_dt", "qsnow"),
                      ("qg", "qg_dt", "qgraupel"))


def run_c384_mixed(nlev=79, dt=150.0, nsteps=5, n_cube=384):
    """The mixed form against the plain FP64 form at C384: 6 x 384 x 384 =
    884,736 columns x L79, 5 steps of 150 s, 10 % of the columns at RH
    U(0.98, 1.02). Each form runs its own 5-step rollout from the same state
    (tendencies zeroed before each step, the state advanced by them after).
    Reported per field: max |mixed - plain| / max |plain| and the rms of
    |mixed - plain| / max |plain|, for the first step (identical inputs) and
    the worst step, of the tendencies of T, qv, qc, qr, qi, qs, qg and of the
    four surface totals; the same after 5 steps for the state itself; the
    mixed form's column water budget; and the device time per step of both
    forms (CUDA events around each step)."""
    import torch

    from pyshield_b200 import constants as C
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.coupling import update_physics_state_with_tendencies
    from pyshield_b200.microphysics import Microphysics

    device = torch.device("cuda", torch.cuda.current_device())
    cfg = PhysicsConfig(dt_atmos=dt)
    runs = {}
    for form in ("plain", "mixed"):
        ms, sf, qf, gd, host, land, (nx, ny, n) = build_state(nlev, device, seed=384, n_cube=n_cube,
                                                              sat_fraction=0.1)
        host.clear()
        runs[form] = (ms, Microphysics(sf, qf, gd, cfg, precision=form))
    names = MIXED_ERROR_FIELDS
    upd = (("qvapor", "qv_dt"), ("qliquid", "ql_dt"), ("qrain", "qr_dt"), ("qice", "qi_dt"), ("qsnow", "qs_dt"),
           ("qgraupel", "qg_dt"), ("qcld", "qa_dt"), ("pt", "pt_dt"), ("ua", "udt"), ("va", "vdt"))
    stream = torch.cuda.current_stream()
    ms_step = {"plain": [], "mixed": []}
    err = {}
    water = None

    def rel(a, b):
        sc = float(b.abs().max())
        d = (a - b).abs()
        sc = sc if sc > 0 else 1.0
        return float(d.max()) / sc, float(d.pow(2).mean().sqrt()) / sc

    for step in range(nsteps):
        for form, (ms, mp) in runs.items():
            for _, t in upd:
                getattr(ms, t).data.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            mp(ms, dt)
            e1.record(stream)
            torch.cuda.synchronize()
            ms_step[form].append(e0.elapsed_time(e1))
        (mp_p_state, mp_p), (mp_m_state, mp_m) = runs["plain"], runs["mixed"]
        for label, tnd, _ in names:
            e = rel(getattr(mp_m_state, tnd).view, getattr(mp_p_state, tnd).view)
            w = err.setdefault(label, {"first_step": e, "worst_step": e})
            w["worst_step"] = (max(w["worst_step"][0], e[0]), max(w["worst_step"][1], e[1]))
        for p in ("rain", "snow", "ice", "graupel"):
            e = rel(getattr(mp_m, p), getattr(mp_p, p))
            w = err.setdefault(p, {"first_step": e, "worst_step": e})
            w["worst_step"] = (max(w["worst_step"][0], e[0]), max(w["worst_step"][1], e[1]))
        if step == 0:
            # column water budget of the mixed step: the tendencies' column
            # integral plus the surface fluxes, relative to the column water
            ms = mp_m_state
            dp = ms.delprsi.view
            qdt = sum(getattr(ms, t).view for t in ("qv_dt", "ql_dt", "qr_dt", "qi_dt", "qs_dt", "qg_dt"))
            wdt = (qdt * dp).sum(2) * C.RGRAV
            pr = (mp_m.rain + mp_m.snow + mp_m.ice + mp_m.graupel) / 86400.0
            col = sum(getattr(ms, f).view for f in ("qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel"))
            colw = (col * dp).sum(2) * C.RGRAV / dt
            water = float(((wdt + pr).abs() / colw).max())
        for form, (ms, mp) in runs.items():
            st = [getattr(ms, x) for x, _ in upd]
            update_physics_state_with_tendencies(*st, *[getattr(ms, t) for _, t in upd], *st, dt)
    torch.cuda.synchronize()
    state_err = {label: rel(getattr(runs["mixed"][0], f).view, getattr(runs["plain"][0], f).view)
                 for label, _, f in names}
    plain_ms = sum(ms_step["plain"]) / nsteps
    mixed_ms = sum(ms_step["mixed"]) / nsteps
    n = 6 * n_cube * n_cube
    out = {
        "workload": f"GFDL microphysics step, C{n_cube} ({n} columns) x L{nlev}, {nsteps} steps of {dt:g} s, "
                    "10 % of columns at RH U(0.98, 1.02)",
        "plain_ms_per_step": plain_ms,
        "mixed_ms_per_step": mixed_ms,
        "mixed_speedup": plain_ms / mixed_ms,
        "plain_column_steps_per_s": n / (plain_ms / 1000.0),
        "mixed_column_steps_per_s": n / (mixed_ms / 1000.0),
        "tendency_error_vs_plain": {k: {"first_step_max": v["first_step"][0], "first_step_rms": v["first_step"][1],
                                        "worst_step_max": v["worst_step"][0], "worst_step_rms": v["worst_step"][1]}
                                    for k, v in err.items()},
        "state_error_after_steps": {k: {"max": v[0], "rms": v[1]} for k, v in state_err.items()},
        "mixed_water_budget_max_rel": water,
        "note": "errors relative to max |plain| of each field; tendencies for T..qg (pt_dt..qg_dt), surface "
                "totals in mm/day; device time (CUDA events) per step",
    }
    runs.clear()
    torch.cuda.empty_cache()
    return out


def max_over_ranks(values, world, device):
    """Each rank's device-measured times -> their maximum over all ranks (the
    slowest replica sets the job's time). One all-reduce; every rank calls it
    at the same point."""
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def whole_job_rate(world, columns_per_rank, steps, total_ms):
    """Column-steps/s of the whole job: every replica advances its own
    columns ``steps`` times; the time is the max over ranks."""
    return world * columns_per_rank * steps / (total_ms / 1000.0)


def run_ours(args, rank, world, local_rank):
    import torch

    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.microphysics import Microphysics

    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    nlev = args.levels
    # this rank's slice of the job's domain: its own seeded C-N state
    start, _ = rank_columns(rank, world, 6 * args.ncube * args.ncube)
    ms, sf, qf, gd, host, land, (nx, ny, n) = build_state(nlev, device, seed=1234 + start // (6 * args.ncube ** 2),
                                                          n_cube=args.ncube)
    cfg = PhysicsConfig(dt_atmos=DT)
    mp = Microphysics(sf, qf, gd, cfg, precision=args.form)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    clocks = ClockSampler(local_rank)
    clocks.start()
    for _ in range(args.warmup):
        mp(ms, DT)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    clocks.mark("begin")
    t_start.record(stream)
    for s in range(args.steps):
        ev[s][0].record(stream)
        mp(ms, DT)
        ev[s][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    clocks.mark("end")
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = t_start.elapsed_time(t_end)
    launch_ms = [a.elapsed_time(b) for a, b in ev]
    mean_launch_ms = sum(launch_ms) / len(launch_ms)

    # ---- end to end through the public API with pinned host buffers
    # the pipeline's first upload and last download are not overlapped: 16 steps amortise them as a run would
    e2e_steps = max(4, min(args.steps, 16))
    if args.no_e2e:
        total_ms, _, mean_launch_ms = max_over_ranks([total_ms, 0.0, mean_launch_ms], world, device)
        return {"n": n, "nlev": nlev, "total_ms": total_ms, "mean_launch_ms": mean_launch_ms, "e2e_ms": 0.0,
                "e2e_steps": 0, "h2d": 0, "d2h": 0, "clocks": clk, "mixed_ms": 0.0}
    pipe = HostPipeline(ms, mp, land, host, (nx, ny, nlev), device)
    pipe.run(2)  # warm-up: allocations, first-copy set-up
    torch.cuda.synchronize()
    barrier()
    e2e_ms = pipe.run(e2e_steps)
    barrier()
    h2d, d2h = pipe.h2d_bytes, pipe.d2h_bytes
    link = pipe.link_only(e2e_steps)

    # the mixed form on the same state, for the FP64-vs-mixed comparison
    mixed_ms = 0.0
    if args.form == "plain" and not args.no_mixed:
        mpm = Microphysics(sf, qf, gd, cfg, precision="mixed")
        for _ in range(args.warmup):
            mpm(ms, DT)
        torch.cuda.synchronize()
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        for _ in range(args.steps):
            mpm(ms, DT)
        m1.record(stream)
        torch.cuda.synchronize()
        mixed_ms = m0.elapsed_time(m1) / args.steps

    total_ms, e2e_ms, mean_launch_ms, mixed_ms = max_over_ranks([total_ms, e2e_ms, mean_launch_ms, mixed_ms], world, device)
    return {
        "mixed_ms": mixed_ms,
        "n": n,
        "nlev": nlev,
        "total_ms": total_ms,
        "mean_launch_ms": mean_launch_ms,
        "e2e_ms": e2e_ms,
        "e2e_steps": e2e_steps,
        "h2d": h2d,
        "d2h": d2h,
        "link": link,
        "clocks": clk,
    }


def run_ensemble(args):
    """The ensemble workload on its own (``--ensemble``): one JSON line."""
    emit(measure_ensemble(args.members, args.levels, args.steps))


def measure_ensemble(nm, levels, steps):
    """``nm`` members of sizes C24/C48/C96 (6 N^2 columns, the six tiles side
    by side), dt ~ U(120, 225) s, per-member Ts offset N(0, 3) K and seed.
    Times ``nm`` sequential launches (one Microphysics per member, FP64 and
    mixed) against one batched launch of the whole ensemble (autotuned
    launch shape, replayed from a CUDA graph); mean of ``steps`` runs after
    a warm-up, CUDA events."""
    import numpy as np
    import torch

    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.ensemble import MicrophysicsEnsemble
    from pyshield_b200.microphysics import Microphysics

    rng = np.random.default_rng(4)
    sizes = rng.choice([24, 48, 96], nm)
    dts = rng.uniform(120.0, 225.0, nm)
    offs = rng.normal(0.0, 3.0, nm)
    cfg = PhysicsConfig(dt_atmos=150.0)
    built = []
    for m in range(nm):
        ms, sf, qf, gd, host, land, (nx, ny, n) = build_state(levels, torch.device("cuda", torch.cuda.current_device()),
                                                             seed=7000 + m, n_cube=int(sizes[m]))
        host.clear()
        ms.pt.view.add_(float(offs[m]))
        built.append((ms, sf, qf, gd, n))
    total_cols = sum(b[4] for b in built)
    stream = torch.cuda.current_stream()

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    for form in ("plain", "mixed"):
        mps = [Microphysics(b[1], b[2], b[3], cfg, precision=form) for b in built]

        def sequential():
            for mp_, b, dt in zip(mps, built, dts):
                mp_(b[0], float(dt))

        out[f"sequential_{form}_ms"] = timed(sequential, steps)
        del mps
    for form in ("mixed", "plain"):
        ens = MicrophysicsEnsemble(cfg, [b[0] for b in built], [b[3].area for b in built], [float(d) for d in dts],
                                   precision=form)
        tuned, timings = ens.autotune(reps=1)
        ens.capture()
        out[f"batched_{form}_ms"] = timed(ens.replay, steps)
        out[f"autotune_{form}"] = {f"{g}x{b}": round(ms, 3) for (g, b), ms in timings.items()}
        out[f"tuned_{form}"] = f"{tuned[0]} columns/block, {tuned[1]} blocks/SM"
        ens.graph = None
        del ens
    rec = {
        "metric": "GFDL MP column-steps/s, ensemble",
        "workload": f"{nm} members, sizes C24/C48/C96 ({int((sizes == 24).sum())}/{int((sizes == 48).sum())}/"
                    f"{int((sizes == 96).sum())}), {total_cols} columns x L{levels}, dt U(120,225) s",
        "unit": "column-steps/s",
        "steps": steps,
    }
    for k, v in list(out.items()):
        if k.endswith("_ms"):
            rec[k.replace("_ms", "_column_steps_per_s")] = total_cols / (v / 1000.0)
        rec[k] = v
    rec["batched_mixed_vs_sequential_plain"] = out["sequential_plain_ms"] / out["batched_mixed_ms"]
    rec["batched_mixed_vs_sequential_mixed"] = out["sequential_mixed_ms"] / out["batched_mixed_ms"]
    del built
    torch.cuda.empty_cache()
    return rec


def emit(rec):
    print(json.dumps(rec), flush=True)


def self_launch(n):
    """``bench.py --gpus N`` started as a single process: start the N ranks
    (one process per GPU) through torch.distributed.run with the same
    arguments on a free local port, and return their exit status."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def rank_columns(rank, world, ncol):
    """Columns [start, stop) of the whole job's domain that rank ``rank``
    advances: the job is ``world`` C-N domains side by side (weak scaling),
    rank r owning the r-th. Ranks share no column and need no exchange."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return rank * ncol, (rank + 1) * ncol


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--levels", type=int, default=79)
    ap.add_argument("--form", default="plain", choices=["plain", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-cost measurement (C96 and C48)")
    ap.add_argument("--no-physics", action="store_true", help="skip the Physics.__call__ measurement")
    ap.add_argument("--no-coupling", action="store_true",
                    help="skip the UpdateAtmosphereState, DycoreToPhysics and AGrid2DGridPhysics measurements")
    ap.add_argument("--no-c384", action="store_true", help="skip the C384 mixed-against-plain comparison")
    ap.add_argument("--ncube", type=int, default=N_CUBE, help="cube size N of the CN workload (default 96)")
    ap.add_argument("--ensemble", action="store_true", help="run the ensemble workload instead")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the ensemble measurement of the default line")
    ap.add_argument("--members", type=int, default=64)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    if args.ensemble:
        run_ensemble(args)
        return
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(self_launch(args.gpus))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    cores = os.cpu_count() or 1
    nlev = args.levels
    ncol = 6 * args.ncube * args.ncube
    config = {
        "workload": f"GFDL microphysics step, C{args.ncube} ({ncol} columns) x L{nlev}, dt {DT:g} s",
        "columns_per_gpu": ncol,
        "levels": nlev,
        "dt_s": DT,
        "form": args.form,
        "layout": "NDSL storage, halo 3, i-fastest",
        "l2": f"no flush: {algorithmic_bytes_per_column_step(nlev) * ncol / 1e9:.3g} GB moved per step, > 126 MB L2",
        "parallelism": f"{world} GPUs, one C{args.ncube} domain each (rank r owns columns r*{ncol} .. (r+1)*{ncol}-1)"
                       if world > 1 else "1 GPU",
    }
    metric = "GFDL MP column-steps/s"

    # the oracle's worker processes start before any CUDA use
    domain = None
    want_cpu = (args.impl == "reference" or not args.no_cpu_baseline) and rank == 0 and world == 1
    if args.impl == "reference" and rank == 0:
        want_cpu = True
    if want_cpu:
        domain = OracleDomain(ncol, nlev, cores)

    if args.impl == "reference":
        if rank != 0:
            return
        # the driver's W warm-up steps, then K timed whole-domain steps
        value, per, sample = cpu_baseline(domain, args.steps, warmup=args.warmup)
        domain.close()
        rec = {
            "impl": "reference",
            "metric": metric,
            "value": value,
            "unit": "column-steps/s",
            "n_gpus": args.gpus,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": 1000.0 * per,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": config,
            "cpu_baseline": {"value": value, "unit": "column-steps/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "column-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference (GT4Py/NDSL) cannot be installed here; this times the FP64 numpy oracle that "
                    "restates the reference's numpy backend bit for bit, whole-domain steps on every host core"
                    + ("; only rank 0 runs it" if world > 1 else ""),
        }
        emit(rec)
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    r = run_ours(args, rank, world, local_rank)
    steps = args.steps
    value = whole_job_rate(world, r["n"], steps, r["total_ms"])
    bytes_launch = algorithmic_bytes_per_column_step(nlev) * r["n"]
    achieved = bytes_launch / (r["mean_launch_ms"] / 1000.0) / 1e9
    peak, peak_kind = peaks()
    e2e_value = whole_job_rate(world, r["n"], r["e2e_steps"], r["e2e_ms"]) if r["e2e_ms"] > 0 else None

    cpu = None
    if want_cpu:
        v, per, sample = cpu_baseline(domain, 3, warmup=1)
        domain.close()
        one = OracleDomain(3456, nlev, 1)
        v1, _, _ = cpu_baseline(one, 1, warmup=0)
        one.close()
        cpu = {"value": v, "unit": "column-steps/s", "cores": cores, "kind": "port",
               "sample": sample + f"; {1000.0 * per:.0f} ms per step; one process alone on 3456 columns: "
                                  f"{v1:.4g} column-steps/s"}
    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint and args.form == "plain":
        adjoint = run_adjoint(n_cube=96)
        adjoint["c48"] = run_adjoint(n_cube=48, window=False)
    physics = (run_physics(n_cube=args.ncube, nlev=nlev)
               if (rank == 0 and world == 1 and not args.no_physics and args.form == "plain") else None)
    coupling = (run_coupling(n_cube=args.ncube, nlev=nlev)
                if (rank == 0 and world == 1 and not args.no_coupling and args.form == "plain") else None)
    # the ensemble of 64 members C24/C48/C96 at L79: sequential launches
    # against one batched, graph-replayed launch
    ensemble = (measure_ensemble(args.members, 79, 3)
                if (rank == 0 and world == 1 and not args.no_ensemble and args.form == "plain") else None)
    fp64 = None
    if rank == 0:
        peak64 = fp64_peak()
        fp64 = {"bound": "fp64", "peak": peak64, "unit": "TFLOP/s",
                "peak_source": "measured: FP64 probe (independent DFMA chains on every SM, CUDA events)"}
        if FP64_FLOPS_PER_COLUMN_STEP.get(nlev) and args.form == "plain":
            ach = FP64_FLOPS_PER_COLUMN_STEP[nlev] * r["n"] / (r["mean_launch_ms"] / 1000.0) / 1e12
            fp64.update({"achieved": ach, "frac": ach / peak64,
                         "flops_per_column_step": FP64_FLOPS_PER_COLUMN_STEP[nlev],
                         "flops_source": "ncu smsp__sass_thread_inst_executed_op_{dfma,dadd,dmul}_pred_on.sum "
                                         "(2 flops per DFMA) of the C48 launch, per column"})
    c384 = (run_c384_mixed(nlev=79)
            if (rank == 0 and world == 1 and not args.no_c384 and args.form == "plain" and nlev == 79) else None)
    d2p = dwind = None
    if rank == 0 and world == 1 and not args.no_coupling and args.form == "plain":
        d2p = run_d2p(n_cube=args.ncube, nlev=nlev)
        dwind = run_dwind(n_cube=args.ncube, nlev=nlev)

    if rank == 0:
        rec = {
            "metric": metric,
            "value": value,
            "unit": "column-steps/s",
            "n_gpus": world,
            "steps": steps,
            "warmup": args.warmup,
            "ms_per_step": r["total_ms"] / steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.form == "plain" else "f32+f64",
            "data": "synthetic",
            "config": config,
            "e2e": ({"value": e2e_value, "unit": "column-steps/s", "h2d_bytes_per_step": r["h2d"],
                     "d2h_bytes_per_step": r["d2h"],
                     "note": "pinned host buffers through Microphysics.__call__: uploads the 13 state fields and "
                             "land, zeroes the 10 tendencies on the device (the physics driver's "
                             "prepare_microphysics), downloads the 10 tendencies, wmp and 4 surface totals",
                     "link": link_record(r)}
                    if e2e_value else None),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": NCU_TRAFFIC_RATIO * bytes_launch if nlev == 79 and args.form == "plain" else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the C48 L79 launch, "
                                           "scaled by columns to this launch",
                         "peak_source": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)",
                         "bytes_per_launch": bytes_launch},
            "roofline_fp64": fp64,
            "cpu_baseline": cpu,
            "gpu_launches": steps,
            "mixed": ({"value": world * r["n"] / (r["mixed_ms"] / 1000.0), "unit": "column-steps/s",
                       "ms_per_step": r["mixed_ms"], "speedup_vs_fp64": r["total_ms"] / steps / r["mixed_ms"],
                       "dtype": "f32 process rates + f64 saturation adjustment, fall and budgets"}
                      if r["mixed_ms"] > 0 else None),
            "clocks": r["clocks"],
            "adjoint": adjoint,
            "physics": physics,
            "coupling": coupling,
            "dycore_to_physics": d2p,
            "agrid_to_dgrid": dwind,
            "c384_mixed": c384,
            "ensemble": ensemble,
        }
        emit(rec)

    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
