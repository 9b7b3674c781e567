"""Simulated FRB pulses (pirate's simpulse.SinglePulse, src_lib/simpulse.cpp): the C++ construction
(own radix-2 FFT) against the numpy restatement in the oracle (numpy's FFT), the SNR normalization,
the pulse's arrival times, pirate's upsampling self-consistency test
(pirate_frb/simpulse/test_pulse_upsampling.py) and the sparse-representation invariants of pirate's
test_pulse_invariants (pirate_frb/tests/test_pulse_injection.py)."""

import numpy as np
import pytest

import oracle as O


def _sp():
    from pirate_b200 import simpulse
    return simpulse


def _edges(rng, nfreq, lo, hi, irregular=True):
    if not irregular:
        return np.linspace(lo, hi, nfreq + 1)
    df = rng.uniform(0.2, 1.8, nfreq)
    return lo + (hi - lo) * np.concatenate([[0.0], np.cumsum(df)]) / df.sum()


CASES = [
    dict(dm=50.0, sm=0.0, intrinsic_width=1e-3, spectral_index=0.0, undispersed_arrival_time_sec=0.2,
         time_sample_ms=1.0, snr=20.0),
    dict(dm=300.0, sm=2.0, intrinsic_width=3e-4, spectral_index=-1.5, undispersed_arrival_time_sec=-0.5,
         time_sample_ms=0.983, snr=12.0),
    dict(dm=0.0, sm=0.5, intrinsic_width=0.0, spectral_index=2.0, undispersed_arrival_time_sec=1.0,
         time_sample_ms=2.0, snr=50.0),
    dict(dm=1200.0, sm=0.1, intrinsic_width=5e-3, spectral_index=0.7, undispersed_arrival_time_sec=0.0,
         time_sample_ms=1.0, snr=8.0, subband_freq_lo_MHz=520.0, subband_freq_hi_MHz=610.0),
]


@pytest.mark.parametrize("k", range(len(CASES)))
def test_matches_numpy_restatement(pb2lib, k):
    rng = np.random.default_rng(k)
    edges = _edges(rng, 64, 400.0, 800.0, irregular=(k % 2 == 0))
    var = rng.uniform(0.5, 2.0, 64)
    p = _sp().SinglePulse(freq_edges_MHz=edges, freq_variances=var, **CASES[k])
    it0, nt, off, data, a, b = O.single_pulse(freq_edges_MHz=edges, freq_variances=var, **CASES[k])
    assert np.array_equal(p.freq_it0, it0) and np.array_equal(p.freq_nt, nt) and np.array_equal(p.freq_sd_off, off)
    assert (p.it_start, p.it_end) == (a, b)
    np.testing.assert_allclose(p.sparse_data, data, rtol=2e-5, atol=2e-6 * np.abs(data).max())
    # matched-filter normalization: sum(value^2 / variance) = snr^2
    ch = np.repeat(np.arange(64), p.freq_nt)
    e = np.sum(p.sparse_data.astype(np.float64) ** 2 / var[ch])
    assert e == pytest.approx(CASES[k]["snr"] ** 2, rel=1e-5)


def test_dispersion_and_scattering(pb2lib):
    sp = _sp()
    assert sp.dispersion_delay(100.0, 400.0) == pytest.approx(1e-3 * 4.148808e6 * 100.0 / 400.0 ** 2, rel=1e-15)
    assert sp.scattering_time(2.0, 500.0) == pytest.approx(2e-3 * 16.0, rel=1e-15)
    with pytest.raises(RuntimeError):
        sp.dispersion_delay(-1.0, 400.0)
    with pytest.raises(RuntimeError):
        sp.scattering_time(1.0, 0.0)


def test_arrival_times(pb2lib):
    """A narrow, unscattered pulse sits, in every channel, at the undispersed arrival time plus the
    channel's mean dispersion delay (centroid within a quarter sample)."""
    sp = _sp()
    edges = np.linspace(400.0, 800.0, 257)
    p = sp.SinglePulse(dm=500.0, sm=0.0, intrinsic_width=2e-3, spectral_index=0.0, undispersed_arrival_time_sec=0.3,
                       time_sample_ms=1.0, snr=30.0, freq_edges_MHz=edges, freq_variances=np.ones(256))
    for f in range(0, 256, 17):
        v = p.sparse_data[p.freq_sd_off[f]:p.freq_sd_off[f] + p.freq_nt[f]].astype(np.float64)
        t = (p.freq_it0[f] + np.arange(v.size) + 0.5) * 1e-3
        cen = np.sum(v * t) / np.sum(v)
        want = 0.3 + 0.5 * (sp.dispersion_delay(500.0, edges[f]) + sp.dispersion_delay(500.0, edges[f + 1]))
        assert abs(cen - want) < 0.25e-3, (f, cen, want)


def _downsample(arr, nf, nt):
    F, T = arr.shape
    return arr.reshape(nf, F // nf, nt, T // nt).sum(axis=(1, 3))


@pytest.mark.parametrize("nupfreq,nupsample", [(1, 2), (2, 1), (2, 2), (3, 4)])
def test_upsampling_self_consistency(pb2lib, nupfreq, nupsample):
    """pirate_frb/simpulse/test_pulse_upsampling.py: a pulse simulated on a finer grid, summed back
    onto the coarse grid, has the coarse pulse's shape (correlation above 0.995)."""
    sp = _sp()
    rng = np.random.default_rng(100 * nupfreq + nupsample)
    nfreq, lo = 300, 500.0
    hi = lo * 1.6
    tsamp = 2e-3
    diag = nfreq * tsamp / (sp.dispersion_delay(1.0, lo) - sp.dispersion_delay(1.0, hi))
    dm = rng.uniform(0.5, 2.0) * diag
    sm = 0.3 * tsamp / sp.scattering_time(1.0, 0.5 * (lo + hi))
    kw = dict(dm=dm, sm=sm, intrinsic_width=1.5 * tsamp, spectral_index=rng.uniform(-1, 1), snr=30.0)
    uat = -sp.dispersion_delay(dm, hi) + 10 * tsamp
    coarse = _edges(rng, nfreq, lo, hi)
    fine = np.concatenate([np.linspace(coarse[i], coarse[i + 1], nupfreq + 1)[:-1] for i in range(nfreq)] + [coarse[-1:]])
    p0 = sp.SinglePulse(freq_edges_MHz=coarse, freq_variances=np.ones(nfreq), time_sample_ms=1e3 * tsamp,
                        undispersed_arrival_time_sec=uat, **kw)
    p1 = sp.SinglePulse(freq_edges_MHz=fine, freq_variances=np.ones(nfreq * nupfreq),
                        time_sample_ms=1e3 * tsamp / nupsample, undispersed_arrival_time_sec=uat, **kw)
    assert p0.it_start >= 0 and p1.it_start >= 0
    nt = max(p0.it_end, -(-p1.it_end // nupsample)) + 8
    a0 = np.zeros((nfreq, nt), np.float32)
    p0.add_to_timestream(a0, 0)
    a1 = np.zeros((nfreq * nupfreq, nt * nupsample), np.float32)
    p1.add_to_timestream(a1, 0)
    a1 = _downsample(a1, nfreq, nt)
    r = np.sum(a0 * a1) / np.sqrt(np.sum(a0 * a0) * np.sum(a1 * a1))
    assert r > 0.995, r


def test_invariants_shift_and_span(pb2lib):
    sp = _sp()
    edges = np.linspace(400.0, 800.0, 65)
    kw = dict(dm=200.0, sm=0.05, intrinsic_width=1e-3, spectral_index=0.0, time_sample_ms=1.0, snr=15.0,
              freq_edges_MHz=edges, freq_variances=np.ones(64))
    p = sp.SinglePulse(undispersed_arrival_time_sec=-1.5, **kw)      # arrival extends to t < 0
    assert p.it_start < 0 < p.it_end
    assert (p.it_start <= p.freq_it0).all() and (p.freq_it0 + p.freq_nt <= p.it_end).all()
    assert np.array_equal(p.freq_sd_off, np.concatenate([[0], np.cumsum(p.freq_nt)[:-1]]))
    q = sp.SinglePulse(undispersed_arrival_time_sec=-1.5 + 0.037, **kw)   # 37 whole samples later
    assert np.array_equal(q.freq_it0, p.freq_it0 + 37) and np.allclose(q.sparse_data, p.sparse_data, rtol=1e-5)
    d0 = p.sparse_data.copy()
    p.shift_samples(37)
    assert np.array_equal(q.freq_it0, p.freq_it0) and (q.it_start, q.it_end) == (p.it_start, p.it_end)
    assert np.array_equal(p.sparse_data, d0)
    assert p.undispersed_arrival_time_sec == pytest.approx(-1.5 + 0.037)
    out = np.zeros((64, p.it_end - p.it_start), np.float32)
    p.add_to_timestream(out, p.it_start, weight=2.0)
    assert np.sum(out) == pytest.approx(2.0 * np.sum(p.sparse_data.astype(np.float64)), rel=1e-5)
    with pytest.raises(RuntimeError, match="does not cover"):
        p.add_to_timestream(np.zeros((64, p.it_end - p.it_start - 1), np.float32), p.it_start)
    with pytest.raises(RuntimeError, match="does not cover"):
        p.add_to_timestream(np.zeros((64, p.it_end - p.it_start), np.float32), p.it_start + 1)


def test_subband_and_errors(pb2lib):
    sp = _sp()
    edges = np.linspace(400.0, 800.0, 41)
    kw = dict(dm=100.0, sm=0.0, intrinsic_width=1e-3, spectral_index=0.0, undispersed_arrival_time_sec=0.1,
              time_sample_ms=1.0, snr=10.0, freq_edges_MHz=edges, freq_variances=np.ones(40))
    p = sp.SinglePulse(subband_freq_lo_MHz=500.0, subband_freq_hi_MHz=600.0, **kw)
    on = (edges[1:] > 500.0) & (edges[:-1] < 600.0)
    assert (p.freq_nt[on] > 0).all() and (p.freq_nt[~on] == 0).all() and (p.freq_it0[~on] == p.it_start).all()
    bad = [dict(kw, subband_freq_lo_MHz=900.0, subband_freq_hi_MHz=1000.0),
           dict(kw, dm=0.0, intrinsic_width=0.0),
           dict(kw, internal_nt=100),
           dict(kw, freq_variances=np.zeros(40)),
           dict(kw, freq_edges_MHz=edges[::-1].copy()),
           dict(kw, time_sample_ms=-1.0)]
    for b in bad:
        with pytest.raises(RuntimeError):
            sp.SinglePulse(**b)


def test_matches_pirate_simpulse(pb2lib):
    """Against pirate's own SinglePulse (src_lib/simpulse.cpp compiled unmodified in oracle/_ref, MKL's
    complex-to-real DFT supplied by oracle/ksgpu_shim/mkl_dfti.h), committed by
    tests/golden/make_ref_golden.py: the same sample ranges exactly, and the same float32 samples to
    within 1e-6 of the pulse's peak (they agree bit for bit when generated)."""
    import json
    import os
    import helpers as H
    fix = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pirate_ref_fixtures.npz"))
    meta = json.loads(bytes(fix["meta_json"]).decode())
    sp_mod = _sp()
    for pc in H.pulse_fixture_cases():
        m = meta[pc["name"]]
        sp = sp_mod.SinglePulse(freq_edges_MHz=pc["edges"], freq_variances=pc["var"], **pc["params"])
        assert (sp.it_start, sp.it_end) == (m["it_start"], m["it_end"]), pc["name"]
        for k in ("freq_it0", "freq_nt", "freq_sd_off"):
            assert np.array_equal(getattr(sp, k), fix["%s/%s" % (pc["name"], k)]), (pc["name"], k)
        ref = fix["%s/sparse_data" % pc["name"]]
        assert sp.sparse_data.shape == ref.shape
        err = np.abs(sp.sparse_data.astype(np.float64) - ref).max()
        assert err <= 1e-6 * np.abs(ref).max(), (pc["name"], err)
