"""bench.py's end-to-end leg computes what a direct step computes.

HostPipeline uploads every step's state fields from pinned host memory,
zeroes the tendencies on the device, steps, and downloads the results, with
the copies on their own streams overlapping the neighbouring steps. Every
step re-uploads the same inputs, so each download must equal the result of
one step on the device-resident state.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_host_pipeline_downloads_match_direct_step():
    import torch

    import bench
    from pyshield_b200._config import PhysicsConfig
    from pyshield_b200.microphysics import Microphysics

    dev = torch.device("cuda", 0)
    nlev = 79
    # the direct path: every step restores the initial inputs on the device
    # and steps; the handle's cloud-fraction accumulator carries over, as it
    # does in the pipeline
    ms, sf, qf, gd, host, land, (nx, ny, n) = bench.build_state(nlev, dev, seed=5, n_cube=12)
    mp = Microphysics(sf, qf, gd, PhysicsConfig(dt_atmos=bench.DT))
    steps = 5
    ref = {}
    for s in range(steps):
        for f in bench.E2E_IN:
            getattr(ms, f).view.copy_(host[f].permute(2, 1, 0).to(dev))
        for t in bench.E2E_ZERO:
            getattr(ms, t).data.zero_()
        mp(ms, bench.DT)
        ref[s % 2] = ({f: getattr(ms, f).view.permute(2, 1, 0).contiguous().cpu().numpy() for f in bench.E2E_OUT},
                      mp._precip.cpu().numpy())

    # the pipeline on another state built from the same seed
    ms2, sf2, qf2, gd2, host2, land2, _ = bench.build_state(nlev, dev, seed=5, n_cube=12)
    mp2 = Microphysics(sf2, qf2, gd2, PhysicsConfig(dt_atmos=bench.DT))
    pipe = bench.HostPipeline(ms2, mp2, land2, host2, (nx, ny, nlev), dev)
    assert pipe.run(steps) > 0.0
    plane = nx * ny * nlev
    for b in range(2):
        out = pipe.h_out[b].numpy()
        for i, f in enumerate(bench.E2E_OUT):
            got = out[i * plane:(i + 1) * plane].reshape(nlev, ny, nx)
            np.testing.assert_array_equal(got, ref[b][0][f], err_msg=f)
        got_p = out[len(bench.E2E_OUT) * plane:].reshape(4, ny, nx)
        np.testing.assert_array_equal(got_p, ref[b][1])
    assert pipe.h2d_bytes == (len(bench.E2E_IN) * plane + nx * ny) * 8
    assert pipe.d2h_bytes == (len(bench.E2E_OUT) * plane + 4 * nx * ny) * 8
