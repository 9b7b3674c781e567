"""Analytic peak-finding variances (pirate's PfAvarApproximation, include/pirate/PfVariance.hpp:86-120)
against pirate's own python implementation (pirate_frb/slow_avar/PfVariance.py:465-640) through the
golden fixtures of tests/golden/make_avar_golden.py, plus properties the model has exactly."""

import json
import os

import numpy as np
import pytest

import helpers as H

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "avar_golden.npz")


def _golden():
    return np.load(GOLDEN)


def _case_names():
    return sorted({k.split("/")[0] for k in _golden().files} - {"full_r16"})


def _plan(pb, cfg):
    return pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))


@pytest.mark.parametrize("name", _case_names())
def test_matches_pirate_python(pb2lib, name):
    """Same shapes; values equal to pirate's python to 1e-12 relative (the sums run in a different
    order; pirate's own C++-vs-python test allows 1e-9, pirate_frb/fast_avar/test_fast_avar.py:20)."""
    g = _golden()
    cfg = json.loads(bytes(g[name + "/config"]).decode())
    plan = _plan(pb2lib, cfg)
    a = pb2lib.PfAvarApproximation(plan, g[name + "/freq_variances"])
    assert a.ntrees == plan.ntrees and a.nfreq == plan.nfreq
    for i in range(plan.ntrees):
        want = g["%s/tree%d" % (name, i)]
        got = a.tree_variance[i]
        t = plan.trees[i]
        assert got.shape == want.shape == (t.nsubbands, t.ndm_wt, t.nprofiles)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)


def test_full_size_matches_pirate_python(pb2lib):
    """The benchmark's rank-16 plan (16384 channels, 5 primary trees): every 13th variance of each
    tree equal to pirate's python to 1e-12 relative. The per-channel variances are regenerated from
    the fixture's seed (numpy's PCG64 stream is stable across numpy versions)."""
    g = _golden()
    cfg = json.loads(bytes(g["full_r16/config"]).decode())
    plan = _plan(pb2lib, cfg)
    fv = np.random.default_rng(7).uniform(0.5, 1.5, plan.nfreq)
    a = pb2lib.PfAvarApproximation(plan, fv)
    for i in range(plan.ntrees):
        np.testing.assert_allclose(a.tree_variance[i].ravel()[::13], g["full_r16/tree%d_strided" % i], rtol=1e-12, atol=0)


def test_linear_in_freq_variances(pb2lib):
    """Variances are linear in the per-channel input variances."""
    plan = _plan(pb2lib, H.toy_config(rank=8, nfreq=300, nt=512))
    rng = np.random.default_rng(3)
    v1 = rng.uniform(0.1, 2.0, plan.nfreq)
    v2 = rng.uniform(0.1, 2.0, plan.nfreq)
    a1 = pb2lib.PfAvarApproximation(plan, v1).tree_variance
    a2 = pb2lib.PfAvarApproximation(plan, v2).tree_variance
    a12 = pb2lib.PfAvarApproximation(plan, v1 + v2).tree_variance
    a3 = pb2lib.PfAvarApproximation(plan, 4.0 * v1).tree_variance
    for i in range(plan.ntrees):
        np.testing.assert_allclose(a12[i], a1[i] + a2[i], rtol=1e-13)
        assert np.array_equal(a3[i], 4.0 * a1[i])     # scaling by a power of two is exact


def test_one_channel_per_tree_channel(pb2lib):
    """With wt_dm_downsampling = 2^rank the variances come from level 0 of the tree: single tree
    channels, no delays. Each input channel then contributes (overlap)^2 * A_p(0), so the profile
    dependence is exactly the kernels' zero-lag autocorrelations A_p(0)."""
    cfg = H.toy_config(rank=5, nfreq=40, nt=256, subbands=[1], primary_trees=[
        dict(num_early_triggers=0, max_width=8, dm_downsampling=0, time_downsampling=0,
             wt_dm_downsampling=32, wt_time_downsampling=16)])
    plan = _plan(pb2lib, cfg)
    v = pb2lib.PfAvarApproximation(plan, np.ones(plan.nfreq)).tree_variance[0]
    A0 = np.array([1.0, 2, 1.5, 2.5, 4, 3, 5, 8, 6, 10])    # zero-lag autocorrelations of the 10 profiles
    assert v.shape == (1, 1, 10)
    np.testing.assert_allclose(v[0, 0] / v[0, 0, 0], A0, rtol=1e-14)


@pytest.mark.parametrize("bad", ["short", "zero", "negative", "nan"])
def test_rejects_bad_freq_variances(pb2lib, bad):
    plan = _plan(pb2lib, H.toy_config(rank=6, nfreq=100, nt=256))
    fv = np.ones(plan.nfreq)
    if bad == "short":
        fv = fv[:-1]
    elif bad == "zero":
        fv[7] = 0.0
    elif bad == "negative":
        fv[0] = -1.0
    else:
        fv[50] = np.nan
    with pytest.raises(RuntimeError, match="freq_variances"):
        pb2lib.PfAvarApproximation(plan, fv)


def test_tree_subbands(pb2lib):
    """plan.trees[i].n_to_flo / n_to_fhi: the subbands' peak-finding band ranges."""
    import oracle as O
    cfg = H.toy_config(rank=8, nfreq=300, nt=512, subbands=[2, 2, 1])
    plan = _plan(pb2lib, cfg)
    full = O.subbands([2, 2, 1])
    t0 = plan.trees[0]
    assert t0.n_to_flo == full["n_to_flo"] and t0.n_to_fhi == full["n_to_fhi"]
    for t in plan.trees:
        assert len(t.n_to_flo) == len(t.n_to_fhi) == t.nsubbands
        assert all(0 <= lo < hi <= 2 ** t.pf_rank for lo, hi in zip(t.n_to_flo, t.n_to_fhi))
