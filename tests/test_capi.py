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
