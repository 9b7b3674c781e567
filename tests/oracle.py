"""ctypes front end of the CPU oracle (oracle/refdd.cpp).

Test infrastructure only: the oracle restates pirate's CPU reference dedisperser
(src_lib/ReferenceDedisperser.cpp, ReferenceTree.cpp, ReferenceLagbuf.cpp,
ReferenceLaggedDownsamplingKernel.cpp, PeakFindingKernel.cpp) and is used as the
checker for the CUDA path, never as part of it.
"""

import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "liborc.so")

_lib = None

c_long_p = ctypes.POINTER(ctypes.c_long)
c_double_p = ctypes.POINTER(ctypes.c_double)


def build():
    src = os.path.join(ORACLE_DIR, "refdd.cpp")
    if (not os.path.exists(LIB_PATH)) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR, "liborc.so"])


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, c_long_p, c_double_p, ctypes.c_double, ctypes.c_long,
                                 ctypes.c_long, ctypes.c_long, ctypes.c_int, c_long_p, ctypes.c_int,
                                 c_long_p, ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_int,
                                 ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_ntrees.restype = ctypes.c_long
        L.orc_ntrees.argtypes = [ctypes.c_void_p]
        L.orc_tree_info.argtypes = [ctypes.c_void_p, ctypes.c_long, c_long_p]
        L.orc_channel_map.argtypes = [ctypes.c_void_p, c_double_p]
        L.orc_dedisperse.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p,
                                     ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                                     ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
        L.orc_eval_tokens.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]
        L.orc_gridded.argtypes = [ctypes.c_void_p, c_double_p]
        L.orc_pf_input.argtypes = [ctypes.c_void_p, ctypes.c_long, c_double_p]
        L.orc_test_tree_basics.restype = ctypes.c_double
        L.orc_test_tree_basics.argtypes = [ctypes.c_uint64] + [ctypes.c_long] * 6 + [ctypes.c_int]
        L.orc_test_tree_subbands.restype = ctypes.c_double
        L.orc_test_tree_subbands.argtypes = [ctypes.c_uint64, ctypes.c_int, c_long_p] + [ctypes.c_long] * 6 + [ctypes.c_int]
        L.orc_test_lagbuf.restype = ctypes.c_double
        L.orc_test_lagbuf.argtypes = [ctypes.c_uint64] + [ctypes.c_long] * 4
        L.orc_subbands.argtypes = [ctypes.c_int, c_long_p, c_long_p, c_long_p, c_long_p, c_long_p, c_long_p]
        L.orc_restrict_subbands.argtypes = [ctypes.c_int, c_long_p, ctypes.c_long, ctypes.c_long, c_long_p]
        L.orc_dequantize.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                                     ctypes.c_long, ctypes.c_long]
        L.orc_half_to_float_c.restype = ctypes.c_float
        L.orc_half_to_float_c.argtypes = [ctypes.c_uint16]
        _lib = L
    return _lib


def _err():
    return lib().orc_last_error().decode()


def _longs(v):
    a = (ctypes.c_long * max(len(v), 1))(*[int(x) for x in v])
    return a


TREE_INFO_KEYS = ["ipri", "et_level", "amb_rank", "dd_rank", "nt_ds", "ndm_out", "nt_out", "ndm_wt",
                  "nt_wt", "nprofiles", "N", "M", "Dcore", "max_width", "pf_rank", "time_ds"]


class OracleDedisperser:
    """ReferenceDedisperser restated on the CPU (sophistication 0 or 1, fp32 or fp64)."""

    def __init__(self, cfg, sophistication=1, real_bits=32, dcore_max=8):
        L = lib()
        zn = cfg["zone_nfreq"]
        ze = cfg["zone_freq_edges"]
        sb = cfg["frequency_subband_counts"]
        pts = []
        for p in cfg["primary_trees"]:
            pts += [p["num_early_triggers"], p["max_width"], p.get("dm_downsampling", 0),
                    p.get("time_downsampling", 0), p["wt_dm_downsampling"], p["wt_time_downsampling"]]
        nbits = {"float32": 32, "float16": 16, "bfloat16": 16}[cfg["dtype"]]
        zed = (ctypes.c_double * len(ze))(*ze)
        h = L.orc_create(len(zn), _longs(zn), zed, float(cfg["time_sample_ms"]), int(cfg["toplevel_tree_rank"]),
                         int(cfg["time_samples_per_chunk"]), nbits, len(sb), _longs(sb),
                         len(cfg["primary_trees"]), _longs(pts), int(cfg["beams_per_gpu"]),
                         int(cfg["beams_per_batch"]), int(dcore_max), int(sophistication), int(real_bits))
        if not h:
            raise RuntimeError("oracle: " + _err())
        self.h = h
        self.cfg = cfg
        self.B = int(cfg["beams_per_batch"])
        self.nfreq = int(sum(zn))
        self.nt_in = int(cfg["time_samples_per_chunk"])
        self.rank = int(cfg["toplevel_tree_rank"])
        self.ntrees = L.orc_ntrees(h)
        self.trees = []
        for i in range(self.ntrees):
            info = (ctypes.c_long * 16)()
            L.orc_tree_info(h, i, info)
            self.trees.append(dict(zip(TREE_INFO_KEYS, list(info))))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def channel_map(self):
        out = np.zeros(2 ** self.rank + 1, dtype=np.float64)
        lib().orc_channel_map(self.h, out.ctypes.data_as(c_double_p))
        return out

    def wt_shape(self, i):
        t = self.trees[i]
        return (self.B, t["ndm_wt"], t["nt_wt"], t["nprofiles"], t["N"])

    def out_shape(self, i):
        t = self.trees[i]
        return (self.B, t["ndm_out"], t["nt_out"])

    def dedisperse(self, ibatch, x, weights, tree_domain=False):
        """x: float32 (B, nfreq, nt_in), or with tree_domain (B, 2^toplevel_tree_rank, nt_in) already
        gridded (ReferenceDedisperser's tree_domain_input); weights: list of float32 arrays of
        wt_shape(i). Returns (out_max list (float64), out_argmax list (uint32))."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        assert x.shape == (self.B, (1 << self.rank) if tree_domain else self.nfreq, self.nt_in)
        wts = [np.ascontiguousarray(w, dtype=np.float32) for w in weights]
        omax = [np.zeros(self.out_shape(i), dtype=np.float64) for i in range(self.ntrees)]
        oarg = [np.zeros(self.out_shape(i), dtype=np.uint32) for i in range(self.ntrees)]
        n = self.ntrees
        wp = (ctypes.c_void_p * n)(*[w.ctypes.data for w in wts])
        mp = (ctypes.c_void_p * n)(*[a.ctypes.data for a in omax])
        ap = (ctypes.c_void_p * n)(*[a.ctypes.data for a in oarg])
        rc = lib().orc_dedisperse(self.h, int(ibatch), x.ctypes.data, wp, mp, ap, int(bool(tree_domain)))
        if rc != 0:
            raise RuntimeError("oracle: " + _err())
        self._last_wts = wts
        return omax, oarg

    def eval_tokens(self, itree, tokens, wt=None):
        """Re-evaluates the trial selected by each token (last dedisperse() call)."""
        tokens = np.ascontiguousarray(tokens, dtype=np.uint32)
        wt = self._last_wts[itree] if wt is None else np.ascontiguousarray(wt, dtype=np.float32)
        out = np.zeros(self.out_shape(itree), dtype=np.float64)
        rc = lib().orc_eval_tokens(self.h, int(itree), tokens.ctypes.data, wt.ctypes.data, out.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle eval_tokens: bad token")
        return out

    def gridded(self):
        out = np.zeros((self.B, 2 ** self.rank, self.nt_in), dtype=np.float64)
        lib().orc_gridded(self.h, out.ctypes.data_as(c_double_p))
        return out

    def pf_input(self, itree):
        t = self.trees[itree]
        out = np.zeros((self.B, t["ndm_out"], t["M"], t["nt_ds"]), dtype=np.float64)
        lib().orc_pf_input(self.h, int(itree), out.ctypes.data_as(c_double_p))
        return out


def test_tree_basics(seed, N, B, T, S, amb, dd, real_bits=32):
    r = lib().orc_test_tree_basics(seed, N, B, T, S, amb, dd, real_bits)
    if r < 0:
        raise RuntimeError(_err())
    return r


def test_tree_subbands(seed, counts, nchunks, B, T, S, amb, dd, real_bits=32):
    r = lib().orc_test_tree_subbands(seed, len(counts), _longs(counts), nchunks, B, T, S, amb, dd, real_bits)
    if r < 0:
        raise RuntimeError(_err())
    return r


def test_lagbuf(seed, nrows, nchunks, ntime, maxlag):
    r = lib().orc_test_lagbuf(seed, nrows, nchunks, ntime, maxlag)
    if r < 0:
        raise RuntimeError(_err())
    return r


def subbands(counts):
    NM = (ctypes.c_long * 2)()
    L = lib()
    if L.orc_subbands(len(counts), _longs(counts), NM, None, None, None, None) != 0:
        raise RuntimeError(_err())
    N, M = NM[0], NM[1]
    m_to_n = (ctypes.c_long * M)()
    m_to_d = (ctypes.c_long * M)()
    flo = (ctypes.c_long * N)()
    fhi = (ctypes.c_long * N)()
    L.orc_subbands(len(counts), _longs(counts), NM, m_to_n, m_to_d, flo, fhi)
    return dict(N=N, M=M, m_to_n=list(m_to_n), m_to_d=list(m_to_d), n_to_flo=list(flo), n_to_fhi=list(fhi))


def restrict_subbands(counts, et_level, new_pf_rank):
    out = (ctypes.c_long * 8)()
    n = lib().orc_restrict_subbands(len(counts), _longs(counts), et_level, new_pf_rank, out)
    if n < 0:
        raise RuntimeError(_err())
    return list(out[:n])


def bare_weights(shape, nprofiles):
    """Unit-variance ('bare kernel') weights 1/sqrt(sum of squared kernel taps) per profile
    (PeakFindingKernelParams::fill_host_weights with empty variances, PeakFindingKernel.cu:606)."""
    var = [1.0]
    L = (nprofiles - 1) // 3
    for l in range(L):
        var += [2.0 ** (l + 1), 1.5 * 2.0 ** l, 2.5 * 2.0 ** l]
    w = (1.0 / np.sqrt(np.array(var, dtype=np.float64))).astype(np.float32)
    out = np.empty(shape, dtype=np.float32)
    out[...] = w[None, None, None, :, None]
    return out


def random_weights(shape, rng):
    """Sparse random weights in the spirit of fill_host_weights(randomize=True)."""
    B, D, T, P, N = shape
    p0 = rng.uniform(0.01, 1.1, size=(B, D, T, 1, 1))
    r = rng.uniform(0, 1, size=shape)
    x = rng.uniform(0, 1, size=shape)
    return np.where(r < p0, x, 0.0).astype(np.float32)


def dequantize(data_u8, scales_offsets_f16, nbeams, nfreq, ntime):
    """ReferenceDequantizationKernel::apply (src_lib/GpuDequantizationKernel.cu:326-380), fp32 output.
    data_u8: (nbeams, nfreq, ntime // 2) uint8, two int4 samples per byte (low nibble first);
    scales_offsets_f16: (nbeams, nfreq, ntime // 256, 2) float16 (scale, offset)."""
    d = np.ascontiguousarray(data_u8, dtype=np.uint8)
    so = np.ascontiguousarray(scales_offsets_f16, dtype=np.float16)
    out = np.empty((nbeams, nfreq, ntime), np.float32)
    if lib().orc_dequantize(d.ctypes.data, so.ctypes.data, out.ctypes.data, nbeams, nfreq, ntime) != 0:
        raise RuntimeError(_err())
    return out


def random_quantized(rng, nbeams, nfreq, ntime, missing=0.01):
    """Seeded int4 data (two samples per byte, a fraction 'missing' of -8 sentinels) and fp16
    (scale, offset) pairs: scales in [0, 1], offsets in [-1, 1], as pirate's test
    (src_lib/GpuDequantizationKernel.cu:508-515)."""
    v = rng.integers(-7, 8, size=(nbeams, nfreq, ntime))
    v[rng.random(v.shape) < missing] = -8
    nib = (v & 0xf).astype(np.uint8)
    data = (nib[..., 0::2] | (nib[..., 1::2] << 4)).astype(np.uint8)
    so = np.empty((nbeams, nfreq, ntime // 256, 2), np.float16)
    so[..., 0] = rng.uniform(0.0, 1.0, so.shape[:-1])
    so[..., 1] = rng.uniform(-1.0, 1.0, so.shape[:-1])
    return data, so


# -------------------------------------------------------------------------------------------------
# Simulated pulses: numpy restatement of pirate's SinglePulse constructor (src_lib/simpulse.cpp:131-320),
# with numpy's FFT for the synthesis.

K_DM = 4.148808e6            # ms MHz^2 per pc cm^-3 (include/pirate/constants.hpp:49)


def single_pulse(dm, sm, intrinsic_width, spectral_index, undispersed_arrival_time_sec, time_sample_ms, snr,
                 freq_edges_MHz, freq_variances, subband_freq_lo_MHz=0.0, subband_freq_hi_MHz=1.0e9, internal_nt=1024):
    """Returns (freq_it0, freq_nt, freq_sd_off, sparse_data float32, it_start, it_end)."""
    edges = np.asarray(freq_edges_MHz, np.float64)
    var = np.asarray(freq_variances, np.float64)
    nfreq, N = edges.size - 1, int(internal_nt)
    dt = 1.0e-3 * time_sample_ms
    nu0 = 0.5 * (edges[0] + edges[-1])
    it0 = np.zeros(nfreq, np.int64)
    nt = np.zeros(nfreq, np.int64)
    off = np.zeros(nfreq, np.int64)
    vals, snr_sq, total = [], 0.0, 0

    def cum_at(cum, s):
        if s < 1.0e-10:
            return 0.0
        if s > N - 1.0e-10:
            return cum[N]
        i = int(s)
        return (1.0 - (s - i)) * cum[i] + (s - i) * cum[i + 1]

    for f in range(nfreq):
        lo, hi = edges[f], edges[f + 1]
        off[f] = total
        if hi <= subband_freq_lo_MHz or lo >= subband_freq_hi_MHz:
            continue
        nuc = 0.5 * (lo + hi)
        d0 = 1.0e-3 * K_DM * dm / hi ** 2
        d1 = 1.0e-3 * K_DM * dm / lo ** 2
        dmw = d1 - d0
        ts = 1.0e-3 * sm / (nuc / 1000.0) ** 4
        t0 = d0 - 0.1 * dmw - 4.0 * intrinsic_width - ts
        t1 = d1 + 0.1 * dmw + 4.0 * intrinsic_width + 10.0 * ts
        tcen = 0.5 * (d0 + d1) - (t0 + (t1 - t0) / (2.0 * N))
        om = (np.pi / (t1 - t0)) * np.arange(N + 1)
        x = 0.5 * dmw * om
        sinc = np.where(x * x > 1.0e-100, np.sin(x) / np.where(x == 0, 1.0, x), 1.0)
        z = np.exp(-0.5 * (intrinsic_width * om) ** 2) * sinc / (1.0 + 1j * ts * om) * np.exp(-1j * tcen * om)
        z[0] = z[0].real
        z[N] = z[N].real
        prof = np.fft.irfft(z, n=2 * N) * (2 * N)
        cum = np.concatenate([[0.0], np.cumsum(np.maximum(prof[:N], 0.0))])
        cum = cum / cum[N]
        pt0, pt1 = undispersed_arrival_time_sec + t0, undispersed_arrival_time_sec + t1
        i0, i1 = int(np.floor(pt0 / dt)), int(np.ceil(pt1 / dt))
        it0[f], nt[f] = i0, i1 - i0
        total += i1 - i0
        amp = (nuc / nu0) ** spectral_index / dt
        for it in range(i0, i1):
            a = cum_at(cum, N * (it * dt - pt0) / (t1 - t0))
            b = cum_at(cum, N * ((it + 1) * dt - pt0) / (t1 - t0))
            v = amp * (b - a)
            vals.append(np.float32(v))
            snr_sq += v * v / var[f]
    active = nt > 0
    it_start = int(it0[active].min())
    it_end = int((it0 + nt)[active].max())
    it0[~active] = it_start
    scale = snr / np.sqrt(snr_sq)
    data = (np.array(vals, np.float64) * scale).astype(np.float32)
    return it0, nt, off, data, it_start, it_end
