"""SinglePulse.inject on the GPU: the injection kernel against the host add_to_timestream arithmetic
(bitwise, all three storage dtypes, pulses straddling both chunk edges), and an end-to-end check
that a pulse injected into noise comes out of the dedisperser and the toy grouper as an event at
the injected DM and arrival time (pirate_frb/tests/test_pulse_injection.py does the analogous
check on its int4 frames)."""

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["float32", "float16", "bfloat16"])
def test_inject_matches_host(pb2lib, dtype):
    import torch
    from pirate_b200 import simpulse as sp
    tdt = getattr(torch, dtype)
    nfreq, nt = 64, 512
    edges = np.linspace(400.0, 800.0, nfreq + 1)
    p = sp.SinglePulse(dm=60.0, sm=0.02, intrinsic_width=2e-3, spectral_index=-0.5, undispersed_arrival_time_sec=0.1,
                       time_sample_ms=1.0, snr=40.0, freq_edges_MHz=edges, freq_variances=np.ones(nfreq))
    assert p.it_end - p.it_start > 300
    rng = np.random.default_rng(3)
    for chunk_it0 in (p.it_start - 100, p.it_start + 150, p.it_end - 50):
        x = torch.from_numpy(rng.standard_normal((nfreq, nt)).astype(np.float32)).to(tdt)
        g = x.cuda()
        p.inject(g, chunk_it0, weight=1.5)
        torch.cuda.synchronize()
        # host: out = round(out + 1.5 * value), one fp32 multiply and one fp32 add
        want = x.to(torch.float32).numpy().copy()
        for f in range(nfreq):
            for k in range(p.freq_nt[f]):
                t = p.freq_it0[f] + k - chunk_it0
                if 0 <= t < nt:
                    want[f, t] = np.float32(want[f, t] + np.float32(np.float32(1.5) * p.sparse_data[p.freq_sd_off[f] + k]))
        want = torch.from_numpy(want).to(tdt)
        bits = torch.int32 if dtype == "float32" else torch.int16
        assert torch.equal(g.cpu().view(bits), want.view(bits)), chunk_it0


def test_injected_pulse_is_detected(pb2lib):
    import torch
    from pirate_b200 import simpulse as sp
    from pirate_b200.grouper import ToyGrouper
    cfg = H.toy_config(rank=8, nfreq=300, nt=512, dtype="float32", beams_per_gpu=2, beams_per_batch=2,
                       primary_trees=[dict(num_early_triggers=0, max_width=16, dm_downsampling=0, time_downsampling=0,
                                           wt_dm_downsampling=16, wt_time_downsampling=16)])
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    dd = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
    dd.allocate()
    dd.fill_analytic_weights(np.ones(plan.nfreq))
    grouper = ToyGrouper(dd, plan, snr_threshold=9.0)
    dm, uat, snr = 6.0, 1.1, 30.0
    pulse = sp.SinglePulse(dm=dm, sm=0.0, intrinsic_width=2e-3, spectral_index=0.0, undispersed_arrival_time_sec=uat,
                           time_sample_ms=1.0, snr=snr, freq_edges_MHz=sp.config_freq_edges(plan.config),
                           freq_variances=np.ones(plan.nfreq))
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    events = []
    for ichunk in range(5):
        with dd.get_input() as x:
            x.copy_(torch.randn(x.shape, generator=gen, device=x.device, dtype=torch.float32))
            pulse.inject(x[1], ichunk * plan.nt_in)
        ev, _ = grouper.process_chunk(ichunk)
        events += list(ev)
    assert events, "no event"
    assert all(e["ibeam"] == 1 for e in events), events          # nothing in the noise-only beam
    best = max(events, key=lambda e: e["snr"])
    assert 0.6 * snr < best["snr"] < 1.2 * snr, best
    assert abs(best["dm"] - dm) < 0.1 * dm, best
    t_lowest = (uat + sp.dispersion_delay(dm, plan.config.to_dict()["zone_freq_edges"][0])) * 1e3
    assert abs(best["time_samples"] - t_lowest) < 8, (best, t_lowest)
