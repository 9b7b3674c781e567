/*
 * pirate_b200.h -- C ABI of the B200 real-time dedispersion path.
 *
 * This is the drop-in boundary for pirate's dedispersion hot path: tree gridding, lagged
 * downsampling, two-stage tree dedispersion, lag staging and peak finding on one GPU. Each entry
 * point names the pirate interface it replaces (file:line in the pirate source tree).
 *
 * Conventions: every function returns 0 on success and a nonzero status on error; the message of the
 * most recent error on the calling thread is returned by pb2_last_error(). Handles are opaque.
 * CUDA streams are passed as `void *` (a cudaStream_t; NULL is the legacy default stream).
 * A pb2_dedisperser is thread safe in the same sense as pirate's GpuDedisperser: calls are
 * serialized internally; seq_id cursors must advance 0, 1, 2, ... per cursor.
 */
#ifndef PIRATE_B200_H
#define PIRATE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PB2_MAX_TREES 64

typedef struct pb2_config pb2_config;
typedef struct pb2_plan pb2_plan;
typedef struct pb2_dedisperser pb2_dedisperser;

/* Message of the last failed call on this thread ("" if none). */
const char *pb2_last_error(void);

/* Library version string. */
const char *pb2_version(void);

/* ---- DedispersionConfig (include/pirate/DedispersionConfig.hpp:21-194) ---- */

/* DedispersionConfig::from_yaml(filename), src_lib/DedispersionConfig.cpp:651 */
int pb2_config_from_yaml(const char *path, pb2_config **out);
/* DedispersionConfig::from_yaml(YamlFile) on an in-memory document, src_lib/DedispersionConfig.cpp:659 */
int pb2_config_from_yaml_string(const char *text, pb2_config **out);
/* DedispersionConfig::to_yaml_string(), src_lib/DedispersionConfig.cpp:638. Writes at most buflen bytes
 * (NUL-terminated); *needed receives the full length + 1. */
int pb2_config_to_yaml(const pb2_config *cfg, char *buf, long buflen, long *needed);
/* DedispersionConfig::make_channel_map(), src_lib/DedispersionConfig.cpp:239; out has 2^rank + 1 doubles. */
int pb2_config_channel_map(const pb2_config *cfg, double *out, long n);
/* DedispersionConfig::{delay_to_frequency, frequency_to_delay, dm_per_unit_delay}, src_lib/DedispersionConfig.cpp:135-214 */
int pb2_config_delay_to_frequency(const pb2_config *cfg, double delay, double *freq);
int pb2_config_frequency_to_delay(const pb2_config *cfg, double freq, double *delay);
int pb2_config_dm_per_unit_delay(const pb2_config *cfg, double *dm);
void pb2_config_destroy(pb2_config *cfg);

/* ---- DedispersionPlan (include/pirate/DedispersionPlan.hpp:33-225) ---- */

typedef struct pb2_tree_info {
    long primary_tree_index, early_trigger_level, amb_rank, dd_rank, nt_ds;
    long ndm_out, nt_out, ndm_wt, nt_wt, nprofiles, Dcore;
    long max_width, dm_downsampling, time_downsampling, wt_dm_downsampling, wt_time_downsampling;
    long nsubbands /* N */, nmultiplets /* M */, pf_rank;
    double dm_min, dm_max, trigger_frequency;
} pb2_tree_info;

/* DedispersionPlan(config), src_lib/DedispersionPlan.cpp:29 */
int pb2_plan_create(const pb2_config *cfg, pb2_plan **out);
void pb2_plan_destroy(pb2_plan *plan);
/* DedispersionPlan::to_yaml_string(), src_lib/DedispersionPlan.cpp:900 (tree section; no MegaRingbuf zones) */
int pb2_plan_to_yaml(const pb2_plan *plan, char *buf, long buflen, long *needed);
/* DedispersionPlan::ntrees / trees[i] (include/pirate/DedispersionTree.hpp:19-59) */
int pb2_plan_ntrees(const pb2_plan *plan, long *ntrees);
int pb2_plan_tree_info(const pb2_plan *plan, long itree, pb2_tree_info *out);
/* DedispersionTree::frequency_subbands.n_to_flo / n_to_fhi (include/pirate/FrequencySubbands.hpp):
 * the peak-finding frequency-band range [flo, fhi) of each of the tree's n == N subbands. */
int pb2_plan_tree_subbands(const pb2_plan *plan, long itree, long *n_to_flo, long *n_to_fhi, long n);
/* PfAvarApproximation(plan, freq_variances).tree_variance, include/pirate/PfVariance.hpp:86-120,
 * src_lib/PfVariance.cpp:236-337: analytic variance of each peak-finding trial under unit weights
 * for white-noise input of per-channel variance freq_variances[nfreq] (all > 0). out[itree] receives
 * tree itree's (N, ndm_wt, nprofiles) doubles, out_len[itree] = N * ndm_wt * nprofiles. */
int pb2_plan_pf_variances(const pb2_plan *plan, const double *freq_variances, long nfreq, double *const *out,
                          const long *out_len, long ntrees);
/* DedispersionPlan::stage1_dd_rank / stage1_amb_rank (length num_primary_trees) */
int pb2_plan_stage1_ranks(const pb2_plan *plan, long *dd_rank, long *amb_rank, long n);
/* DedispersionPlan::decode_argmax, src_lib/DedispersionPlan.cpp:481; out5 = (fmin, fmax, tlo, thi, p) */
int pb2_plan_decode_argmax(const pb2_plan *plan, uint32_t token, long itree, long idm, long itime, long *out5);
/* DedispersionPlan::decode_argmax2, src_lib/DedispersionPlan.cpp:544; out5 = (freq_lo, freq_hi, dm, time, width) */
int pb2_plan_decode_argmax2(const pb2_plan *plan, long itree, const long *in5, double *out5);
/* DedispersionPlan.decode_argmax_batch / decode_argmax2_batch (src_pybind11/pirate_pybind11.cpp:396-409):
 * decode_argmax / decode_argmax2 over n >= 1 events, element by element (the first bad element fails
 * the call). Host arrays of length n. */
int pb2_plan_decode_argmax_batch(const pb2_plan *plan, long n, const uint32_t *tokens, const long *itrees,
                                 const long *idms, const long *itimes, long *fmins, long *fmaxs, long *tlos,
                                 long *this_, long *ps);
int pb2_plan_decode_argmax2_batch(const pb2_plan *plan, long n, const long *itrees, const long *fmins,
                                  const long *fmaxs, const long *tlos, const long *this_, const long *ps,
                                  double *freqs_lo, double *freqs_hi, double *dms, double *times, double *widths);
/* DedispersionPlan::compute_steady_state_it0, src_lib/DedispersionPlan.cpp:634; out has ndm_out entries */
int pb2_plan_steady_state_it0(const pb2_plan *plan, long itree, long *out, long n);

/* ---- GpuDedisperser (include/pirate/Dedisperser.hpp:45-254) ---- */

/* GpuDedisperser::Params, include/pirate/Dedisperser.hpp:47-86 (the stream pool is internal). */
typedef struct pb2_dd_params {
    int cuda_device_id;
    long nbatches_out;      /* 0 -> num_active_batches */
    long nbatches_wt;       /* 0 -> nbatches_out */
    long num_consumers;
    int synchronous;
    long initial_chunk;
    /* pb2_dd_release_input blocks until every consumer has released seq_id - nbatches_out (pirate's
     * blocking wait on the release-output event ring, src_lib/GpuDedisperser.cpp:1078-1081), and
     * pb2_dd_acquire_output blocks until seq_id has been launched (src_lib/GpuDedisperser.cpp:932);
     * after this many milliseconds they fail instead (0 -> 60000). */
    long release_timeout_ms;
} pb2_dd_params;

/* GpuDedisperser::Outputs, include/pirate/Dedisperser.hpp:98-125. out_max[i] and out_argmax[i] are
 * device pointers to (nbeams, ndm_out[i], nt_out[i]) arrays; out_max has the config dtype. */
typedef struct pb2_outputs {
    int dtype;              /* 0 float32, 1 float16, 2 bfloat16 */
    long nbeams, ichunk_zero_based, ichunk_fpga_based, ibeam, ntrees;
    long ndm_out[PB2_MAX_TREES], nt_out[PB2_MAX_TREES];
    void *out_max[PB2_MAX_TREES];
    uint32_t *out_argmax[PB2_MAX_TREES];
    /* Candidate stage (pb2_dd_enable_sifter), else null. Device arrays of nbeams entries: each beam's
     * strongest output over every tree (the toy grouper's reduction, pirate_frb/run_toy_grouper.py:79-116):
     * cand_peak, cand_tree, cand_idm, cand_itime, cand_token; cand_valid = (peak >= threshold); the
     * fp16 patch (nbeams, 1728) around the peak; and the score (the sifter's logit, or the peak when no
     * sifter is attached; -inf where not valid). */
    float *cand_peak;
    int *cand_tree, *cand_idm, *cand_itime, *cand_valid;
    uint32_t *cand_token;
    uint16_t *patches;
    float *scores;
} pb2_outputs;

/* The toy grouper's per-chunk reduction (pirate_frb/run_toy_grouper.py:79-116), as one kernel on
 * 'stream' over an acquired batch of outputs: per beam b < outs->nbeams, the largest out_max over
 * every tree, dm and time (a tree whose maximum is NaN is passed over; ties go to the first tree, then
 * the first (dm, time) in row-major order), with its tree, dm and time indices and the out_argmax
 * token there. Device arrays of outs->nbeams entries; peak = -inf and tree = idm = itime = -1 when no
 * tree qualifies. Call it while the outputs are acquired. */
int pb2_beam_peaks(const pb2_outputs *outs, float *peak, int32_t *tree, int32_t *idm, int32_t *itime, uint32_t *token,
                   void *stream);

/* Simulated FRB pulses: pirate::simpulse (include/pirate/simpulse.hpp:24-119, src_lib/simpulse.cpp).
 * dispersion_delay / scattering_time in seconds (simpulse.hpp:27,31). */
int pb2_dispersion_delay(double dm, double freq_mhz, double *seconds);
int pb2_scattering_time(double sm, double freq_mhz, double *seconds);

/* SinglePulse::Params (include/pirate/simpulse.hpp:42-66) without the two arrays, which are passed
 * separately: freq_edges_mhz (nfreq + 1, increasing) and freq_variances (nfreq). */
typedef struct pb2_pulse_params {
    double dm, sm, intrinsic_width, spectral_index, undispersed_arrival_time_sec, time_sample_ms, snr;
    double subband_freq_lo_mhz, subband_freq_hi_mhz;    /* pirate's defaults: 0 and 1e9 */
    long internal_nt;                                   /* pirate's default: 1024 */
} pb2_pulse_params;
typedef struct pb2_pulse pb2_pulse;

/* SinglePulse(params), src_lib/simpulse.cpp:131-320 */
int pb2_pulse_create(const pb2_pulse_params *params, const double *freq_edges_mhz, const double *freq_variances,
                     long nfreq, pb2_pulse **out);
void pb2_pulse_destroy(pb2_pulse *pulse);
/* SinglePulse::it_start, it_end and the number of stored samples (sum of freq_nt). */
int pb2_pulse_range(const pb2_pulse *pulse, long *it_start, long *it_end, long *nsamples);
/* SinglePulse::freq_it0, freq_nt, freq_sd_off (nfreq each) and sparse_data (nsamples), copied out. */
int pb2_pulse_sparse(const pb2_pulse *pulse, long *freq_it0, long *freq_nt, long *freq_sd_off, float *sparse_data);
/* SinglePulse::add_to_timestream(out, out_it0, weight), src_lib/simpulse.cpp:323-360: host float32
 * array of nfreq rows (row_stride elements apart) spanning samples [out_it0, out_it0 + out_nt). */
int pb2_pulse_add_to_timestream(const pb2_pulse *pulse, float *out, long nfreq, long out_nt, long row_stride,
                                long out_it0, float weight);
/* SinglePulse::shift_samples(delta_it), src_lib/simpulse.cpp:363-373 */
int pb2_pulse_shift_samples(pb2_pulse *pulse, long delta_it);
/* Injection on the GPU, one kernel on 'stream': adds weight * pulse to a device chunk of nfreq rows
 * (row_stride elements apart, dtype 0/1/2 = float32/float16/bfloat16) holding samples
 * [chunk_it0, chunk_it0 + nt); pulse samples outside the chunk are skipped (the analogue of pirate's
 * inject_single_pulse clipping). Copies the pulse to the current device on first use. */
int pb2_pulse_inject(pb2_pulse *pulse, void *chunk, int dtype, long nfreq, long nt, long row_stride, long chunk_it0,
                     float weight, void *stream);

/* GpuDedisperser::create(params), src_lib/GpuDedisperser.cpp:84 */
int pb2_dd_create(const pb2_plan *plan, const pb2_dd_params *params, pb2_dedisperser **out);
/* GpuDedisperser::allocate(gpu_allocator, host_allocator), src_lib/GpuDedisperser.cpp:390 (allocates internally) */
int pb2_dd_allocate(pb2_dedisperser *dd);
/* Device bytes held by the dedisperser after allocate(). */
int pb2_dd_device_bytes(const pb2_dedisperser *dd, long *nbytes);
/* Pinned host bytes of the stage-1 delay lines spilled to host memory: rows whose stage-2 readers are
 * more than the config's max_gpu_clag chunks behind (pirate's MegaRingbuf host zones,
 * src_lib/MegaRingbuf.cpp:155-183); 0 when nothing is spilled (max_gpu_clag 10000, the default). */
int pb2_dd_host_bytes(const pb2_dedisperser *dd, long *nbytes);
/* GpuDedisperser::acquire_input, src_lib/GpuDedisperser.cpp:796; shape3 = (beams_per_batch, nfreq, nt_in) */
int pb2_dd_acquire_input(pb2_dedisperser *dd, long seq_id, void *stream, void **ptr, long *shape3);
/* int4 input, the raw format GpuDedisperser::time dequantizes into the input before dedispersing
 * (src_lib/GpuDedisperser.cpp:1617-1660, GpuDequantizationKernel): acquires the next input slot as
 * packed int4 data (beams_per_batch, nfreq, nt_in/2) bytes (two samples per byte, low nibble first)
 * and fp16 (scale, offset) pairs (beams_per_batch, nfreq, nt_in/256, 2); same seq_id cursor as
 * pb2_dd_acquire_input. pb2_dd_release_input then dequantizes inside the gridding kernel, with the
 * same values pb2_dequantize would write in the config dtype. nt_in must be a multiple of 256. */
int pb2_dd_acquire_input_int4(pb2_dedisperser *dd, long seq_id, void *stream, void **data, void **scales_offsets,
                              long *shape3);
/* GpuDequantizationKernel::launch (include/pirate/GpuDequantizationKernel.hpp:53-70) with
 * ReferenceDequantizationKernel::apply's arithmetic (src_lib/GpuDequantizationKernel.cu:326-380):
 * out = 0 where the int4 value is -8, else scale * value + offset in fp32, rounded once to out_dtype
 * (0 float32, 1 float16, 2 bfloat16). Device arrays: out (nbeams, nfreq, ntime), scales_offsets
 * (nbeams, nfreq, ntime/256, 2) fp16, data (nbeams, nfreq, ntime/2) bytes; ntime a multiple of 256. */
int pb2_dequantize(void *out, int out_dtype, const void *scales_offsets, const void *data, long nbeams, long nfreq,
                   long ntime, void *stream);
/* GpuDedisperser::release_input_and_launch_dd_kernels, src_lib/GpuDedisperser.cpp:830 */
int pb2_dd_release_input(pb2_dedisperser *dd, long seq_id, void *stream);
/* GpuDedisperser::acquire_output, src_lib/GpuDedisperser.cpp:890 (sync != 0 blocks the host) */
int pb2_dd_acquire_output(pb2_dedisperser *dd, long consumer_id, long seq_id, void *stream, int sync, pb2_outputs *out);
/* GpuDedisperser::release_output, src_lib/GpuDedisperser.cpp:945 */
int pb2_dd_release_output(pb2_dedisperser *dd, long consumer_id, long seq_id, void *stream);
/* GpuDedisperser::fill_all_weights, src_lib/GpuDedisperser.cpp:1240; host array
 * (nbatches_wt, beams_per_batch, ndm_wt, nt_wt, nprofiles, N) float32 */
int pb2_dd_fill_weights(pb2_dedisperser *dd, long itree, const float *host, long nelts);
/* GpuDedisperser::fill_analytic_weights, include/pirate/Dedisperser.hpp:237-244,
 * src_lib/GpuDedisperser.cpp:1162-1238: every weight slot and beam of every tree gets
 * 1/sqrt(variance) of PfAvarApproximation (see pb2_plan_pf_variances) for the per-channel input
 * variances freq_variances[nfreq] (all > 0). Blocks until the weights are on the GPU. */
int pb2_dd_fill_analytic_weights(pb2_dedisperser *dd, const double *freq_variances, long nfreq);
/* GpuDedisperser::stop, src_lib/GpuDedisperser.cpp:735 */
int pb2_dd_stop(pb2_dedisperser *dd);
/* GpuDedisperser::time, src_lib/GpuDedisperser.cpp:1573-1665: pirate's timing loop over niterations
 * batches. Each copies one batch of int4 data and fp16 (scale, offset) pairs from pinned host memory into
 * the acquired int4 input slot on a copy stream, launches the kernels (dequantization fused into
 * gridding) and acquires and releases the output as consumer 0. rtb[i] (niterations doubles) receives
 * iteration i's real-time beams, beams_per_batch * chunk seconds / (time between the completions of
 * iterations i-1 and i); rtb[0] = 0. pirate prints the same figure per iteration. Needs num_consumers 1,
 * time_samples_per_chunk a multiple of 256, niterations > 2 * num_active_batches, and no acquired
 * batch left unreleased; the seq_id cursors advance by niterations. */
int pb2_dd_time(pb2_dedisperser *dd, long niterations, double *rtb);
/* Clears every delay line and tree state (and the input and output slots) on 'stream', after waiting for
 * the batches already launched: later chunks see zeros as their history, as at the start of a stream.
 * The seq_id cursors are unchanged. (No pirate counterpart; used to separate synthetic events.) */
int pb2_dd_zero_state(pb2_dedisperser *dd, void *stream);
/* Kernel launches per (chunk, batch), and algorithmic HBM bytes per (chunk, batch) for the
 * kernel classes [grid+lds (one fused kernel), candidates+sifter, stage1, stage2, pf]. */
int pb2_dd_kernels_per_batch(const pb2_dedisperser *dd, long *n);
int pb2_dd_algorithmic_bytes(const pb2_dedisperser *dd, double *out5);
/* Per-kernel-class CUDA-event timing on the dedisperser's compute streams (the analogue of pirate's
 * KernelTimer / ResourceTracker reporting, src_lib/GpuDedisperser.cpp:1674-1681). kernel_times()
 * synchronizes and returns accumulated milliseconds and launch counts for [grid+lds (one fused kernel), candidates+sifter, stage1, stage2, pf]. */
int pb2_dd_enable_timing(pb2_dedisperser *dd, int on);
int pb2_dd_kernel_times(pb2_dedisperser *dd, double *ms5, long *counts5);
void pb2_dd_destroy(pb2_dedisperser *dd);

/* ---- Learned candidate sifter (no counterpart in pirate: a learned stage behind the threshold peak
 * finder, which stays the fallback and the yardstick of its recall) ----
 *
 * Patch: 9 fine DMs (the peak's +-4) x 32 output times x 6 trailing boxcar widths (1..32) of the
 * dedispersed data around a candidate, each boxcar sum / sqrt(width), fp16, layout (dm, time, width).
 * MLP: 1728 -> 256 -> 128 -> 1 with ReLU, bf16 weights (fp32 master copy), FP32 accumulation on the
 * tensor cores; trained on the mean binary cross-entropy of its logit with Adam. Parameters are fp32 in
 * the order W1 (256, 1728), b1, W2 (128, 256), b2, W3 (1, 128), b3 (weights (out, in) row-major). */
typedef struct pb2_sifter pb2_sifter;
int pb2_sifter_create(int cuda_device_id, long max_batch, uint64_t seed, pb2_sifter **out);
void pb2_sifter_destroy(pb2_sifter *s);
int pb2_sifter_nparams(long *n);
int pb2_sifter_set_params(pb2_sifter *s, const float *host_params);
int pb2_sifter_get_params(const pb2_sifter *s, float *host_params);
/* logits[n] (device) of n device patches (n, 1728) fp16, n <= max_batch, on 'stream'. */
int pb2_sifter_forward(pb2_sifter *s, const void *patches, long n, float *logits, void *stream);
/* Gradients of the mean binary cross-entropy over a batch (device labels 0/1) into host grad[nparams];
 * *loss = the batch loss. Synchronizes 'stream'. */
int pb2_sifter_gradients(pb2_sifter *s, const void *patches, const float *labels, long n, float *grad, double *loss,
                         void *stream);
/* One Adam step (0.9, 0.999, 1e-8) with learning rate lr; *loss = the batch loss. Synchronizes. */
int pb2_sifter_train_step(pb2_sifter *s, const void *patches, const float *labels, long n, float lr, double *loss,
                          void *stream);
/* Adds the candidate stage to every later batch of 'dd' (after pb2_dd_allocate): per-beam peak over the
 * trees, patches of peaks >= threshold (sigma), and scores by 'sifter' (may be null: scores are then the
 * peaks). The results appear in pb2_outputs. The sifter then runs on the dedisperser's compute streams
 * and must neither be trained meanwhile nor destroyed before the dedisperser. */
int pb2_dd_enable_sifter(pb2_dedisperser *dd, float threshold, pb2_sifter *sifter);

/* ---- Many beams with uneven plans, one CUDA graph per chunk (pirate: one GpuDedisperser per plan on a
 * pool of compute streams, src_lib/GpuDedisperser.cpp:990-1000) ----
 *
 * One group per plan; each group's beams form one batch (beams_per_gpu == beams_per_batch). A step is
 * one chunk of every group, run as one replayed CUDA graph whose kernels read the chunk index from a
 * device counter. Inputs: the group's input slot (pb2_batched_input) written before the step, on the
 * step's stream or ordered before it; outputs (pb2_batched_outputs, no candidate arrays) valid after it.
 * pb2_batched_autotune times the schedule choices (per group: merged stage-2 grids, peak-finder
 * variant, gridding block size; branch concurrency), keeps the fastest, clears the state and writes a
 * JSON record of the trials (copy_out convention of pb2_config_to_yaml). */
typedef struct pb2_batched pb2_batched;
int pb2_batched_create(const pb2_plan *const *plans, long nplans, int cuda_device_id, pb2_batched **out);
int pb2_batched_allocate(pb2_batched *b);
int pb2_batched_ngroups(const pb2_batched *b, long *n);
int pb2_batched_device_bytes(const pb2_batched *b, long *nbytes);
int pb2_batched_fill_weights(pb2_batched *b, long group, long itree, const float *host, long nelts);
int pb2_batched_fill_analytic_weights(pb2_batched *b, long group, const double *freq_variances, long nfreq);
int pb2_batched_input(pb2_batched *b, long group, void **ptr, long *shape3);
int pb2_batched_outputs(pb2_batched *b, long group, pb2_outputs *out);
int pb2_batched_step(pb2_batched *b, void *stream);
int pb2_batched_reset(pb2_batched *b, void *stream);
int pb2_batched_set_schedule(pb2_batched *b, const int *merge_stage2, const int *pf_general, const int *grid_block,
                             int concurrent);
int pb2_batched_autotune(pb2_batched *b, int reps, char *buf, long buflen, long *needed);
int pb2_batched_time_steps(pb2_batched *b, int nsteps, void *stream, double *ms_per_step);
int pb2_batched_kernels_per_step(const pb2_batched *b, long *n);
void pb2_batched_destroy(pb2_batched *b);

/* ---- Allocation-free single-chunk dedispersion (no counterpart in pirate) ----
 *
 * For callers that cannot allocate device memory, for example a real-time thread that must not
 * stall on cudaMalloc's device-wide synchronization, or code inside a host framework whose memory
 * pool must own every device allocation. Dedisperses one chunk of beams_per_batch beams as the first
 * chunk of a fresh stream (zero history), through the same kernels as the GpuDedisperser, and
 * allocates nothing: all scratch lives in a static device array of PB2_NOALLOC_SCRATCH_BYTES that
 * every GPU loading the library holds until exit. Plans whose scratch exceeds it are rejected.
 *   in:          device (beams_per_batch, nfreq, nt_in) in the config dtype
 *   weights[i]:  device (beams_per_batch, ndm_wt, nt_wt, nprofiles, N) float32, per tree
 *   out_max[i], out_argmax[i]: device (beams_per_batch, ndm_out, nt_out), config dtype / uint32
 * The array is shared by all calls: calls that overlap on the GPU race and must be serialized.
 * The first call on a device looks up the array's address (cudaGetSymbolAddress); make that first
 * call before any stream capture. The stream must belong to the current device. The plan's lookup
 * tables are copied from pageable host memory on the first call on a device and whenever the plan
 * differs from the previous call's, so such a call may wait for earlier work on the stream; calls
 * that repeat the previous plan copy nothing from the host. */
#define PB2_NOALLOC_SCRATCH_BYTES (32L << 20)
int pb2_dedisperse_chunk_noalloc(const pb2_plan *plan, const void *in, const float *const *weights,
                                 void *const *out_max, uint32_t *const *out_argmax, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PIRATE_B200_H */
