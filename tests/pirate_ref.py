"""ctypes front end of oracle/_ref/libpirate_ref.so: pirate's OWN reference CPU dedisperser
(src_lib/ReferenceDedisperser.cpp and the files it uses), compiled unmodified from pirate's source tree
by 'make -C oracle ref PIRATE_SRC=...' against the ksgpu / yaml-cpp stand-ins in oracle/ksgpu_shim.

Test infrastructure only. It pins the restated oracle (oracle/refdd.cpp, tests/oracle.py) and, through
the committed fixtures of tests/golden/make_ref_golden.py, the CUDA path to pirate's own arithmetic.
The library exists only where pirate's sources were available to build it; tests that need it skip
otherwise, and the committed fixtures carry its outputs everywhere else.
"""

import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "_ref", "libpirate_ref.so")

TREE_INFO_KEYS = ["ipri", "et_level", "amb_rank", "dd_rank", "nt_ds", "ndm_out", "nt_out", "ndm_wt",
                  "nt_wt", "nprofiles", "N", "M", "Dcore", "max_width", "pf_rank", "time_ds"]

_lib = None
c_long_p = ctypes.POINTER(ctypes.c_long)
c_double_p = ctypes.POINTER(ctypes.c_double)
vp = ctypes.c_void_p


def build(pirate_src):
    """Compiles pirate's reference sources from 'pirate_src' into oracle/_ref (make -C oracle ref)."""
    subprocess.check_call(["make", "-s", "-j8", "-C", ORACLE_DIR, "ref", "PIRATE_SRC=" + os.path.abspath(pirate_src)])


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref is not built (make -C oracle ref PIRATE_SRC=<pirate source tree>)")
        L = ctypes.CDLL(LIB_PATH)
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_create.restype = vp
        L.ref_create.argtypes = [ctypes.c_int, c_long_p, c_double_p, ctypes.c_double, ctypes.c_long, ctypes.c_long,
                                 ctypes.c_long, ctypes.c_int, c_long_p, ctypes.c_int, c_long_p, ctypes.c_long,
                                 ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_int]
        L.ref_destroy.argtypes = [vp]
        L.ref_ntrees.restype = ctypes.c_long
        L.ref_ntrees.argtypes = [vp]
        L.ref_tree_info.argtypes = [vp, ctypes.c_long, c_long_p]
        L.ref_dedisperse.argtypes = [vp, ctypes.c_long, ctypes.c_long, vp, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                     ctypes.POINTER(vp)]
        L.ref_eval_tokens.argtypes = [vp, ctypes.c_long, vp, vp, vp]
        L.ref_self_tests.argtypes = [ctypes.c_long]
        _lib = L
    return _lib


def _err():
    return lib().ref_last_error().decode()


def _longs(v):
    return (ctypes.c_long * max(len(v), 1))(*[int(x) for x in v])


def self_tests(niter):
    """pirate's ReferenceTree::test_basics, ReferenceTree::test_subbands, ReferenceLagbuf::test_random."""
    if lib().ref_self_tests(int(niter)) != 0:
        raise RuntimeError("pirate reference self-test failed: " + _err())


class PirateReferenceDedisperser:
    """pirate's ReferenceDedisperser (sophistication 0, 1 or 2) on a config dict of the form used by
    tests/helpers.toy_config, with every tree's Dcore = min(time_downsampling, dcore_max)."""

    def __init__(self, cfg, sophistication=1, dcore_max=8, tree_domain=False):
        L = lib()
        zn, ze, sb = cfg["zone_nfreq"], cfg["zone_freq_edges"], cfg["frequency_subband_counts"]
        pts = []
        for p in cfg["primary_trees"]:
            pts += [p["num_early_triggers"], p["max_width"], p.get("dm_downsampling", 0),
                    p.get("time_downsampling", 0), p["wt_dm_downsampling"], p["wt_time_downsampling"]]
        nbits = {"float32": 32, "float16": 16, "bfloat16": 16}[cfg["dtype"]]
        zed = (ctypes.c_double * len(ze))(*ze)
        h = L.ref_create(len(zn), _longs(zn), zed, float(cfg["time_sample_ms"]), int(cfg["toplevel_tree_rank"]),
                         int(cfg["time_samples_per_chunk"]), nbits, len(sb), _longs(sb), len(cfg["primary_trees"]),
                         _longs(pts), int(cfg["beams_per_gpu"]), int(cfg["beams_per_batch"]), int(dcore_max),
                         int(sophistication), int(bool(tree_domain)))
        if not h:
            raise RuntimeError("pirate reference: " + _err())
        self.h = h
        self.B = int(cfg["beams_per_batch"])
        self.nbatches = int(cfg["beams_per_gpu"]) // self.B
        self.ntrees = L.ref_ntrees(h)
        self.trees = []
        for i in range(self.ntrees):
            info = (ctypes.c_long * 16)()
            if L.ref_tree_info(h, i, info) != 0:
                raise RuntimeError(_err())
            self.trees.append(dict(zip(TREE_INFO_KEYS, list(info))))
        self.seq = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_destroy(self.h)
            self.h = None

    def out_shape(self, i):
        t = self.trees[i]
        return (self.B, t["ndm_out"], t["nt_out"])

    def dedisperse(self, x, weights):
        """Next (chunk, batch) in seq_id order: ichunk = seq // nbatches, ibatch = seq % nbatches.
        Returns (out_max list (float32), out_argmax list (uint32))."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        wts = [np.ascontiguousarray(w, dtype=np.float32) for w in weights]
        omax = [np.zeros(self.out_shape(i), dtype=np.float32) for i in range(self.ntrees)]
        oarg = [np.zeros(self.out_shape(i), dtype=np.uint32) for i in range(self.ntrees)]
        n = self.ntrees
        wp = (vp * n)(*[w.ctypes.data for w in wts])
        mp = (vp * n)(*[a.ctypes.data for a in omax])
        ap = (vp * n)(*[a.ctypes.data for a in oarg])
        ichunk, ibatch = divmod(self.seq, self.nbatches)
        if lib().ref_dedisperse(self.h, ichunk, ibatch, x.ctypes.data, wp, mp, ap) != 0:
            raise RuntimeError("pirate reference: " + _err())
        self.seq += 1
        self._last_wts = wts
        return omax, oarg

    def eval_tokens(self, itree, tokens):
        tokens = np.ascontiguousarray(tokens, dtype=np.uint32)
        out = np.zeros(self.out_shape(itree), dtype=np.float32)
        if lib().ref_eval_tokens(self.h, int(itree), tokens.ctypes.data, self._last_wts[itree].ctypes.data,
                                 out.ctypes.data) != 0:
            raise RuntimeError("pirate reference eval_tokens: " + _err())
        return out


class PiratePulse:
    """pirate's simpulse.SinglePulse (src_lib/simpulse.cpp), with MKL's complex-to-real DFT supplied by
    oracle/ksgpu_shim/mkl_dfti.h. Exposes it_start, it_end, freq_it0, freq_nt, freq_sd_off, sparse_data."""

    def __init__(self, dm, sm, intrinsic_width, spectral_index, undispersed_arrival_time_sec, time_sample_ms, snr,
                 freq_edges_MHz, freq_variances, subband_freq_lo_MHz=0.0, subband_freq_hi_MHz=1.0e9, internal_nt=1024):
        L = lib()
        if not getattr(L, "_pulse_sigs", False):
            L.ref_pulse_create.restype = vp
            L.ref_pulse_create.argtypes = [c_double_p, ctypes.c_long, vp, vp, ctypes.c_long]
            L.ref_pulse_destroy.argtypes = [vp]
            L.ref_pulse_range.argtypes = [vp, c_long_p]
            L.ref_pulse_sparse.argtypes = [vp, vp, vp, vp, vp]
            L.ref_pulse_add_to_timestream.argtypes = [vp, vp, ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_float]
            L._pulse_sigs = True
        edges = np.ascontiguousarray(freq_edges_MHz, dtype=np.float64)
        var = np.ascontiguousarray(freq_variances, dtype=np.float64)
        p = (ctypes.c_double * 9)(dm, sm, intrinsic_width, spectral_index, undispersed_arrival_time_sec,
                                  time_sample_ms, snr, subband_freq_lo_MHz, subband_freq_hi_MHz)
        h = L.ref_pulse_create(p, int(internal_nt), edges.ctypes.data, var.ctypes.data, var.size)
        if not h:
            raise RuntimeError("pirate SinglePulse: " + _err())
        self.h = h
        self.nfreq = var.size
        r = (ctypes.c_long * 3)()
        L.ref_pulse_range(h, r)
        self.it_start, self.it_end = r[0], r[1]
        self.freq_it0 = np.zeros(self.nfreq, np.int64)
        self.freq_nt = np.zeros(self.nfreq, np.int64)
        self.freq_sd_off = np.zeros(self.nfreq, np.int64)
        self.sparse_data = np.zeros(r[2], np.float32)
        if L.ref_pulse_sparse(h, self.freq_it0.ctypes.data, self.freq_nt.ctypes.data, self.freq_sd_off.ctypes.data,
                              self.sparse_data.ctypes.data) != 0:
            raise RuntimeError(_err())

    def add_to_timestream(self, out, out_it0, weight=1.0):
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.ndim == 2
        if lib().ref_pulse_add_to_timestream(self.h, out.ctypes.data, out.shape[0], out.shape[1], int(out_it0),
                                             float(weight)) != 0:
            raise RuntimeError("pirate SinglePulse.add_to_timestream: " + _err())

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_pulse_destroy(self.h)
            self.h = None
