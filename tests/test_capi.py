"""CPU tests of the C ABI (include/pirate_b200.h): the shared library loads, exports every function
the header declares, and its host-only entry points (config, plan) behave like pirate's
DedispersionConfig / DedispersionPlan, including their error behaviour. No compute calls: these run
without a GPU."""

import ctypes
import os
import re

import pytest

import helpers as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pirate_b200.h")


def _declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    names = re.findall(r"\b(pb2_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_symbols_exported(pb2lib):
    names = _declared_functions()
    assert len(names) >= 30, names
    L = ctypes.CDLL(pb2lib.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, "declared in pirate_b200.h but not exported: %s" % missing


def test_version_and_no_error(pb2lib):
    L = pb2lib.lib()
    assert L.pb2_version().decode()
    assert isinstance(L.pb2_last_error().decode(), str)


def _config_handle(pb2lib, text):
    L = pb2lib.lib()
    h = ctypes.c_void_p()
    rc = L.pb2_config_from_yaml_string(text.encode(), ctypes.byref(h))
    return rc, h


def test_config_yaml_round_trip(pb2lib):
    cfg = pb2lib.DedispersionConfig.from_dict(H.toy_config())
    y1 = cfg.to_yaml_string()
    cfg2 = pb2lib.DedispersionConfig.from_yaml_string(y1)
    assert cfg2.to_yaml_string() == y1
    d = cfg2.to_dict()
    assert d["toplevel_tree_rank"] == 8
    assert d["frequency_subband_counts"] == [2, 2, 1]
    assert len(d["primary_trees"]) == 2


def test_config_errors_are_reported(pb2lib):
    L = pb2lib.lib()
    good = pb2lib.DedispersionConfig.from_dict(H.toy_config()).to_yaml_string()
    # unknown key
    rc, h = _config_handle(pb2lib, good + "no_such_key: 3\n")
    assert rc != 0 and not h.value
    assert "no_such_key" in L.pb2_last_error().decode()
    # tree rank too small for the subband counts / invalid value
    bad = good.replace("toplevel_tree_rank: 8", "toplevel_tree_rank: 0")
    rc, h = _config_handle(pb2lib, bad)
    assert rc != 0 and L.pb2_last_error().decode()
    # malformed document
    rc, h = _config_handle(pb2lib, "zone_nfreq: [1, 2\n")
    assert rc != 0 and L.pb2_last_error().decode()
    # null output pointer
    assert L.pb2_config_from_yaml_string(good.encode(), None) != 0


def test_config_frequency_delay_maps(pb2lib):
    cfg = pb2lib.DedispersionConfig.from_dict(H.toy_config(rank=8))
    L = pb2lib.lib()
    f = ctypes.c_double()
    d = ctypes.c_double()
    # the delay map is monotone: top of the band has zero delay, bottom has delay 2^rank
    assert L.pb2_config_frequency_to_delay(cfg._h, ctypes.c_double(800.0), ctypes.byref(d)) == 0
    assert abs(d.value) < 1e-9
    assert L.pb2_config_frequency_to_delay(cfg._h, ctypes.c_double(400.0), ctypes.byref(d)) == 0
    assert abs(d.value - 256.0) < 1e-6
    assert L.pb2_config_delay_to_frequency(cfg._h, ctypes.c_double(128.0), ctypes.byref(f)) == 0
    assert L.pb2_config_frequency_to_delay(cfg._h, f, ctypes.byref(d)) == 0
    assert abs(d.value - 128.0) < 1e-6
    cm = (ctypes.c_double * 257)()
    assert L.pb2_config_channel_map(cfg._h, cm, 257) == 0
    vals = list(cm)
    assert all(b >= a for a, b in zip(vals, vals[1:])) or all(b <= a for a, b in zip(vals, vals[1:]))
    # wrong length is an error, not an overrun
    assert L.pb2_config_channel_map(cfg._h, cm, 100) != 0


def test_plan_trees_and_errors(pb2lib):
    L = pb2lib.lib()
    cfg = pb2lib.DedispersionConfig.from_dict(H.toy_config())
    plan = pb2lib.DedispersionPlan(cfg)
    n = ctypes.c_long()
    assert L.pb2_plan_ntrees(plan._h, ctypes.byref(n)) == 0
    assert n.value == len(plan.trees) >= 2
    info = pb2lib._TreeInfo()
    assert L.pb2_plan_tree_info(plan._h, n.value, ctypes.byref(info)) != 0   # out of range
    assert "itree" in L.pb2_last_error().decode() or L.pb2_last_error().decode()
    for t in plan.trees:
        assert t.ndm_out * t.dm_downsampling == 2 ** (t.amb_rank + t.dd_rank)
        assert t.nt_out * t.time_downsampling == t.nt_ds
        assert t.nprofiles == 1 + 3 * (t.max_width.bit_length() - 1)
    y = plan.to_yaml_string()
    assert "trees" in y or "tree" in y
    # a plan from a null config is an error
    h = ctypes.c_void_p()
    assert L.pb2_plan_create(None, ctypes.byref(h)) != 0


def test_plan_rejects_bad_downsampling(pb2lib):
    d = H.toy_config()
    d["primary_trees"][0]["dm_downsampling"] = 2   # must be 0 or 2^pf_rank
    cfg = pb2lib.DedispersionConfig.from_dict(d)
    with pytest.raises(Exception) as e:
        pb2lib.DedispersionPlan(cfg)
    assert "dm_downsampling" in str(e.value)


def test_new_entry_points_validate_arguments(pb2lib):
    """Argument checks of the analytic-weight, grouper and pulse entry points run before any device
    work, so they report errors (status != 0 and a message) without a GPU."""
    import numpy as np
    L = pb2lib.lib()
    from pirate_b200 import simpulse
    simpulse._sigs()
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(H.toy_config(rank=6, nfreq=100, nt=256)))
    vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)

    def fails(rc, word):
        msg = L.pb2_last_error().decode()
        assert rc != 0 and word in msg, msg

    # PfAvarApproximation: wrong tree count, wrong output length, null pointers
    fv = np.ones(plan.nfreq)
    outs = [np.zeros(t.nsubbands * t.ndm_wt * t.nprofiles) for t in plan.trees]
    ptrs = (dp * plan.ntrees)(*[o.ctypes.data_as(dp) for o in outs])
    lens = (ctypes.c_long * plan.ntrees)(*[o.size for o in outs])
    assert L.pb2_plan_pf_variances(plan._h, fv.ctypes.data_as(dp), fv.size, ptrs, lens, plan.ntrees) == 0
    fails(L.pb2_plan_pf_variances(plan._h, fv.ctypes.data_as(dp), fv.size, ptrs, lens, plan.ntrees + 1), "ntrees")
    lens[0] += 1
    fails(L.pb2_plan_pf_variances(plan._h, fv.ctypes.data_as(dp), fv.size, ptrs, lens, plan.ntrees), "out[0]")
    fails(L.pb2_plan_pf_variances(plan._h, None, fv.size, ptrs, lens, plan.ntrees), "null")
    fails(L.pb2_dd_fill_analytic_weights(None, fv.ctypes.data_as(dp), fv.size), "null")
    fails(L.pb2_plan_tree_subbands(plan._h, 0, (ctypes.c_long * 9)(), (ctypes.c_long * 9)(), 9), "subbands")
    # batch decoders: empty input
    z = np.zeros(1, np.int64)
    fails(L.pb2_plan_decode_argmax_batch(plan._h, 0, z.ctypes.data, *[z.ctypes.data] * 3, *[z.ctypes.data] * 5), "nonempty")
    # beam peaks: null outputs, bad tree count, bad dtype
    o = pb2lib._Outputs()
    buf = np.zeros(64, np.float32)
    fails(L.pb2_beam_peaks(None, *[buf.ctypes.data] * 5, None), "null")
    o.ntrees = 0
    fails(L.pb2_beam_peaks(ctypes.byref(o), *[buf.ctypes.data] * 5, None), "ntrees")
    o.ntrees, o.nbeams, o.dtype = 1, 1, 7
    o.ndm_out[0], o.nt_out[0] = 2, 2
    o.out_max[0] = o.out_argmax[0] = buf.ctypes.data
    fails(L.pb2_beam_peaks(ctypes.byref(o), *[buf.ctypes.data] * 5, None), "dtype")
    # pulses: invalid parameters are refused at creation; a null chunk at injection
    edges = np.linspace(400.0, 800.0, 11)
    var = np.ones(10)
    p = simpulse._PulseParams(-1.0, 0.0, 1e-3, 0.0, 0.1, 1.0, 10.0, 0.0, 1e9, 1024)
    h = ctypes.c_void_p()
    fails(L.pb2_pulse_create(ctypes.byref(p), edges.ctypes.data, var.ctypes.data, 10, ctypes.byref(h)), "dm")
    p.dm = 50.0
    assert L.pb2_pulse_create(ctypes.byref(p), edges.ctypes.data, var.ctypes.data, 10, ctypes.byref(h)) == 0
    fails(L.pb2_pulse_inject(h, None, 0, 10, 256, 256, 0, 1.0, None), "null")
    fails(L.pb2_pulse_add_to_timestream(h, buf.ctypes.data, 9, 4, 4, 0, 1.0), "row per channel")
    L.pb2_pulse_destroy(h)
    # the timing loop: null arguments, and a dedisperser that was never allocated (no device work)
    rtb = np.zeros(8)
    fails(L.pb2_dd_time(None, 8, rtb.ctypes.data_as(dp)), "null")
    dd = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
    fails(L.pb2_dd_time(dd._h, 8, None), "null")
    fails(L.pb2_dd_time(dd._h, 8, rtb.ctypes.data_as(dp)), "allocate")


def test_kernel_launches_per_batch(pb2lib):
    """Launch count per (chunk, batch), from the plan alone (no GPU needed): gridding, one stage-1
    launch per primary tree, one stage-2 grid per run of consecutive output trees that share a stage-2
    kernel (same dd rank and staggered-subband flag), one peak-finding launch per output tree."""
    prim = [dict(num_early_triggers=0, max_width=32, dm_downsampling=0, time_downsampling=0,
                 wt_dm_downsampling=64, wt_time_downsampling=64) for _ in range(5)]
    cfg = H.toy_config(rank=16, nfreq=16384, nt=2048, dtype="float16", subbands=[0, 0, 0, 0, 1], beams_per_gpu=4,
                       beams_per_batch=4, primary_trees=prim)
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    dd = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
    # the benchmark's plan: its five output trees share one stage-2 kernel (dd rank 8, no staggered pairs)
    assert plan.ntrees == 5 and {t.dd_rank for t in plan.trees} == {8}
    assert dd.kernels_per_batch() == 1 + 5 + 1 + 5
    # plans with early triggers and subbands: between one stage-2 grid and one per output tree
    for case in ([2, 2, 1], [1, 1, 1], [0, 1]):
        cfg = H.toy_config(rank=9, nfreq=300, nt=256, subbands=case)
        plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
        n = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1).kernels_per_batch()
        npri = len(cfg["primary_trees"])
        assert 1 + npri + 1 + plan.ntrees <= n <= 1 + npri + 2 * plan.ntrees, (case, n)
