"""Simulated FRB pulses, with the names of pirate's pirate_frb.simpulse (SinglePulse,
dispersion_delay, scattering_time; src_pybind11/pirate_pybind11_simpulse.cpp, include/pirate/simpulse.hpp),
plus SinglePulse.inject, which adds the pulse to a chunk of device samples with one CUDA kernel."""

import ctypes

import numpy as np

from . import _check, _stream_ptr, lib

__all__ = ["SinglePulse", "dispersion_delay", "scattering_time", "config_freq_edges"]


class _PulseParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in (
        "dm", "sm", "intrinsic_width", "spectral_index", "undispersed_arrival_time_sec", "time_sample_ms", "snr",
        "subband_freq_lo_mhz", "subband_freq_hi_mhz")] + [("internal_nt", ctypes.c_long)]


def _sigs():
    L = lib()
    if getattr(L, "_pulse_sigs", False):
        return L
    vp, lp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_double)
    for name, res, args in [
            ("pb2_dispersion_delay", ctypes.c_int, [ctypes.c_double, ctypes.c_double, dp]),
            ("pb2_scattering_time", ctypes.c_int, [ctypes.c_double, ctypes.c_double, dp]),
            ("pb2_pulse_create", ctypes.c_int, [ctypes.POINTER(_PulseParams), vp, vp, ctypes.c_long, ctypes.POINTER(vp)]),
            ("pb2_pulse_destroy", None, [vp]),
            ("pb2_pulse_range", ctypes.c_int, [vp, lp, lp, lp]),
            ("pb2_pulse_sparse", ctypes.c_int, [vp, vp, vp, vp, vp]),
            ("pb2_pulse_add_to_timestream", ctypes.c_int, [vp, vp, ctypes.c_long, ctypes.c_long, ctypes.c_long,
                                                           ctypes.c_long, ctypes.c_float]),
            ("pb2_pulse_shift_samples", ctypes.c_int, [vp, ctypes.c_long]),
            ("pb2_pulse_inject", ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_long,
                                                ctypes.c_long, ctypes.c_float, vp])]:
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    L._pulse_sigs = True
    return L


def dispersion_delay(dm, freq_MHz):
    """Dispersion delay in seconds (include/pirate/simpulse.hpp:27)."""
    out = ctypes.c_double()
    _check(_sigs().pb2_dispersion_delay(float(dm), float(freq_MHz), ctypes.byref(out)))
    return out.value


def scattering_time(sm, freq_MHz):
    """Scattering time in seconds; sm is the scattering time in ms at 1 GHz (include/pirate/simpulse.hpp:31)."""
    out = ctypes.c_double()
    _check(_sigs().pb2_scattering_time(float(sm), float(freq_MHz), ctypes.byref(out)))
    return out.value


def config_freq_edges(config):
    """Channel edges in MHz (nfreq + 1, increasing) of a DedispersionConfig: each zone's band split
    into zone_nfreq equal channels, input channel 0 at the bottom of the band."""
    d = config.to_dict() if hasattr(config, "to_dict") else config
    nz, ze = d["zone_nfreq"], d["zone_freq_edges"]
    parts = [np.linspace(ze[z], ze[z + 1], int(nz[z]) + 1)[:-1] for z in range(len(nz))]
    return np.concatenate(parts + [np.array([ze[-1]], dtype=np.float64)])


class SinglePulse:
    """pirate's simpulse.SinglePulse: one dispersed, scattered pulse on a fixed channelization
    (freq_edges_MHz, low to high) and a zero-based sample grid (sample i spans
    [i * dt, (i + 1) * dt], dt = time_sample_ms / 1000), normalized to matched-filter SNR 'snr' for
    per-channel noise variances freq_variances."""

    def __init__(self, dm, sm, intrinsic_width, spectral_index, undispersed_arrival_time_sec, time_sample_ms, snr,
                 freq_edges_MHz, freq_variances, subband_freq_lo_MHz=0.0, subband_freq_hi_MHz=1.0e9, internal_nt=1024):
        L = _sigs()
        self._edges = np.ascontiguousarray(freq_edges_MHz, dtype=np.float64)
        self._var = np.ascontiguousarray(freq_variances, dtype=np.float64)
        if self._edges.ndim != 1 or self._var.ndim != 1 or self._var.size != self._edges.size - 1:
            raise RuntimeError("SinglePulse: freq_edges_MHz (nfreq + 1) and freq_variances (nfreq) must be 1-d")
        p = _PulseParams(dm, sm, intrinsic_width, spectral_index, undispersed_arrival_time_sec, time_sample_ms, snr,
                         subband_freq_lo_MHz, subband_freq_hi_MHz, int(internal_nt))
        h = ctypes.c_void_p()
        _check(L.pb2_pulse_create(ctypes.byref(p), self._edges.ctypes.data, self._var.ctypes.data,
                                  self._var.size, ctypes.byref(h)))
        self._h = h
        self.dm, self.sm, self.intrinsic_width, self.spectral_index = dm, sm, intrinsic_width, spectral_index
        self.time_sample_ms, self.snr, self.internal_nt = time_sample_ms, snr, int(internal_nt)
        self.undispersed_arrival_time_sec = float(undispersed_arrival_time_sec)
        self.subband_freq_lo_MHz, self.subband_freq_hi_MHz = subband_freq_lo_MHz, subband_freq_hi_MHz
        self.nfreq = self._var.size
        self._refresh()

    def _refresh(self):
        a, b, n = ctypes.c_long(), ctypes.c_long(), ctypes.c_long()
        _check(_sigs().pb2_pulse_range(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(n)))
        self.it_start, self.it_end = a.value, b.value
        self.freq_it0 = np.zeros(self.nfreq, np.int64)
        self.freq_nt = np.zeros(self.nfreq, np.int64)
        self.freq_sd_off = np.zeros(self.nfreq, np.int64)
        self.sparse_data = np.zeros(n.value, np.float32)
        _check(_sigs().pb2_pulse_sparse(self._h, self.freq_it0.ctypes.data, self.freq_nt.ctypes.data,
                                        self.freq_sd_off.ctypes.data, self.sparse_data.ctypes.data))

    @property
    def freq_edges_MHz(self):
        return self._edges

    @property
    def freq_variances(self):
        return self._var

    @property
    def freq_lo_MHz(self):
        return float(self._edges[0])

    @property
    def freq_hi_MHz(self):
        return float(self._edges[-1])

    def add_to_timestream(self, out, out_it0, weight=1.0):
        """out: float32 numpy array (nfreq, out_nt), time-contiguous, spanning samples
        [out_it0, out_it0 + out_nt), which must cover [it_start, it_end). Adds weight * pulse."""
        if not isinstance(out, np.ndarray) or out.dtype != np.float32 or out.ndim != 2 or out.strides[1] != 4:
            raise RuntimeError("SinglePulse.add_to_timestream: out must be a 2-d float32 array with contiguous rows")
        _check(_sigs().pb2_pulse_add_to_timestream(self._h, out.ctypes.data, out.shape[0], out.shape[1],
                                                   out.strides[0] // 4, int(out_it0), float(weight)))

    def shift_samples(self, delta_it):
        _check(_sigs().pb2_pulse_shift_samples(self._h, int(delta_it)))
        self.undispersed_arrival_time_sec += 1.0e-3 * int(delta_it) * self.time_sample_ms
        self._refresh()

    def inject(self, chunk, chunk_it0, weight=1.0, stream=None):
        """Adds weight * pulse to a CUDA tensor chunk (nfreq, nt) of float32/float16/bfloat16 holding
        samples [chunk_it0, chunk_it0 + nt), e.g. one beam of GpuDedisperser.get_input()'s array
        (chunk_it0 = ichunk * nt_in). Samples outside the chunk are skipped."""
        import torch
        codes = {torch.float32: 0, torch.float16: 1, torch.bfloat16: 2}
        if chunk.dtype not in codes or chunk.dim() != 2 or chunk.stride(1) != 1 or not chunk.is_cuda:
            raise RuntimeError("SinglePulse.inject: chunk must be a 2-d CUDA tensor with contiguous rows")
        with torch.cuda.device(chunk.device):
            _check(_sigs().pb2_pulse_inject(self._h, chunk.data_ptr(), codes[chunk.dtype], chunk.shape[0],
                                            chunk.shape[1], chunk.stride(0), int(chunk_it0), float(weight),
                                            _stream_ptr(stream)))

    def __str__(self):
        return ("SinglePulse(nfreq=%d, dm=%g, sm=%g, intrinsic_width=%g, spectral_index=%g, "
                "undispersed_arrival_time_sec=%g, snr=%g, time_sample_ms=%g, samples=[%d, %d))"
                % (self.nfreq, self.dm, self.sm, self.intrinsic_width, self.spectral_index,
                   self.undispersed_arrival_time_sec, self.snr, self.time_sample_ms, self.it_start, self.it_end))

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                lib().pb2_pulse_destroy(self._h)
            except Exception:
                pass
            self._h = None
