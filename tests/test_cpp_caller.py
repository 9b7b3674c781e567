"""The C++ and pybind11 surfaces (include/pirate_b200.hpp, pirate_b200._pirate_b200_pybind), which
mirror pirate's C++ GpuDedisperser and its pybind11 module over the C ABI: a compiled C++ caller and
the pybind11 module read the same plan as the ctypes mirror (CPU), and on the GPU the C++ caller's
float32 outputs equal the fp32 oracle bit for bit."""

import os
import subprocess

import numpy as np
import pytest

import helpers as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dd_cpp.cpp")


def _build(tmp_path):
    exe = str(tmp_path / "dd_cpp")
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", SRC,
           "-o", exe, "-L", os.path.join(ROOT, "pirate_b200"), "-lpirate_b200", "-L/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath," + os.path.join(ROOT, "pirate_b200")]
    subprocess.check_call(cmd)
    return exe


def _cfg():
    return H.case_config(H.PARITY_CASES[1])


def _yaml(pb, cfg, tmp_path):
    p = tmp_path / "cfg.yml"
    p.write_text(pb.DedispersionConfig.from_dict(cfg).to_yaml_string())
    return str(p)


def test_cpp_caller_reads_plan(pb2lib, tmp_path):
    exe = _build(tmp_path)
    cfg = _cfg()
    out = subprocess.check_output([exe, _yaml(pb2lib, cfg, tmp_path), "--plan"], text=True).split("\n")
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    assert out[0] == "ntrees %d" % plan.ntrees
    for i, t in enumerate(plan.trees):
        assert out[1 + i].split()[1:] == [str(v) for v in (t.primary_tree_index, t.early_trigger_level, t.ndm_out, t.nt_out,
                                                           t.nprofiles, t.Dcore)]


def test_pybind_module_reads_plan(pb2lib, tmp_path):
    from pirate_b200 import _pirate_b200_pybind as pyb
    cfg = _cfg()
    c = pyb.DedispersionConfig.from_yaml(_yaml(pb2lib, cfg, tmp_path))
    plan = pyb.DedispersionPlan(c)
    ref = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    assert plan.ntrees == ref.ntrees
    for a, b in zip(plan.trees, ref.trees):
        assert (a.ndm_out, a.nt_out, a.nprofiles, a.Dcore, a.nmultiplets) == (b.ndm_out, b.nt_out, b.nprofiles, b.Dcore, b.nmultiplets)
    assert plan.decode_argmax(0x00010000, 0, 1, 2) == tuple(ref.decode_argmax(0x00010000, 0, 1, 2))
    with pytest.raises(RuntimeError):
        pyb.DedispersionConfig.from_yaml_string("toplevel_tree_rank: [")


@pytest.mark.gpu
def test_cpp_caller_matches_oracle(pb2lib, tmp_path):
    exe = _build(tmp_path)
    cfg = _cfg()
    nb = cfg["beams_per_gpu"] // cfg["beams_per_batch"]
    nchunks = 3
    xs = H.make_inputs(cfg, nchunks, seed=31)
    orc, _ = H.run_oracle(cfg, [], [])
    ws = H.make_weights(orc, seed=31)
    _, ores = H.run_oracle(cfg, xs, ws, 1, 32)
    (tmp_path / "in.bin").write_bytes(b"".join(np.ascontiguousarray(x, np.float32).tobytes() for x in xs))
    (tmp_path / "wt.bin").write_bytes(b"".join(np.ascontiguousarray(w, np.float32).tobytes() for w in ws))
    subprocess.check_call([exe, _yaml(pb2lib, cfg, tmp_path), str(len(xs)), str(tmp_path / "in.bin"),
                           str(tmp_path / "wt.bin"), str(tmp_path / "out.bin")])
    raw = (tmp_path / "out.bin").read_bytes()
    o = 0
    for seq in range(nchunks * nb):
        for i in range(orc.ntrees):
            n = int(np.prod(orc.out_shape(i)))
            m = np.frombuffer(raw, np.float32, n, o).reshape(orc.out_shape(i))
            o += 4 * n
            a = np.frombuffer(raw, np.uint32, n, o).reshape(orc.out_shape(i))
            o += 4 * n
            assert np.array_equal(m.astype(np.float64), ores[seq][0][i]), (seq, i)
            assert np.array_equal(a, ores[seq][1][i]), (seq, i)
