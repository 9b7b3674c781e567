// dedisperser.hpp -- the B200 GpuDedisperser (host side).
//
// Mirrors pirate's GpuDedisperser (include/pirate/Dedisperser.hpp:45-254): sequential seq_id
// cursors (seq_id = ichunk * nbatches + ibatch), acquire_input / release_input_and_launch_dd_kernels /
// acquire_output / release_output with CUDA-event stream fencing, per-consumer output back-pressure,
// and the "stoppable" error model (any failing entry point stops the object; later calls rethrow).
//
// Device memory layout (all allocated and zeroed by allocate()):
//   inputs    nslots_in x (B, nfreq, nt_in)                     storage dtype
//   int4 in   nslots_in x (B, nfreq, nt_in/2) bytes + (B, nfreq, nt_in/256, 2) fp16 scales/offsets
//   tree0     nstreams x (B, 2^rank, nt_in) level-0 tree         storage dtype
//   lds[p]    (total_beams, 2^(rank-1), cap_p) delay lines       storage dtype, cap_p = 2^k >= nt_p + 2^s1dd - 1
//   ring[p]   per stage-1 output row (a, dm_brev): a delay line of capacity max_lag(row) + nt_p (rounded to 32)
//   pfring[i] (total_beams, ndm_out, M, cap_i) subband rows       storage dtype, cap_i = 2^k >= nt + tpad + Dout
//   state     per-block tree state of the stage-1/stage-2 kernels (fp32): phase delay line + histories
//   outputs   nbatches_out x per-tree (B, ndm_out, nt_out) out_max (storage dtype) + out_argmax (uint32)
//   weights   nbatches_wt x per-tree (B, ndm_wt, nt_wt, P, N) fp32

#pragma once

#include "kernels.cuh"
#include "plan.hpp"
#include "sifter.hpp"

#include <condition_variable>
#include <exception>
#include <memory>
#include <mutex>
#include <vector>

namespace pb2 {

struct DeviceBuffer
{
    void *ptr = nullptr;
    size_t nbytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    DeviceBuffer(DeviceBuffer &&o) noexcept : ptr(o.ptr), nbytes(o.nbytes) { o.ptr = nullptr; o.nbytes = 0; }
    ~DeviceBuffer();
    void alloc(size_t n);   // cudaMalloc + cudaMemset(0)
    void upload(const void *host, size_t n);
    template<typename T> T *as() const { return (T *) ptr; }
};

// Schedule knobs of one dedisperser's kernel sequence (chosen per plan by BatchedDedisperser::autotune).
struct GroupTuning
{
    bool merge_stage2 = true;   // one stage-2 grid for consecutive trees with the same kernel
    bool pf_general = false;    // the general peak-finding kernel even where the fast one applies
    int grid_block = 128;       // threads per gridding block (a multiple of the windows per row; <= 512)
};

class GpuDedisperser
{
public:
    struct Params
    {
        int cuda_device_id = 0;
        long nbatches_out = 0;      // 0 -> num_active_batches
        long nbatches_wt = 0;       // 0 -> nbatches_out
        long num_consumers = 1;
        bool synchronous = true;
        long initial_chunk = 0;
        // release_input_and_launch_dd_kernels(seq_id) waits (host side) until every consumer has
        // released seq_id - nbatches_out, and acquire_output(seq_id) until seq_id has been launched,
        // as pirate's blocking event-ring waits do (src_lib/GpuDedisperser.cpp:932, 1078-1081); they
        // fail after this many ms (0 -> 60000).
        long release_timeout_ms = 0;
    };

    struct Outputs
    {
        Dtype dtype;
        long nbeams = 0, ichunk_zero_based = 0, ichunk_fpga_based = 0, ibeam = 0;
        std::vector<long> ndm_out, nt_out;
        std::vector<void *> out_max;
        std::vector<uint32_t *> out_argmax;
        // Candidate stage (enable_sifter), device arrays of nbeams entries, else null: each beam's
        // strongest output over every tree (peak, tree, idm, itime, token), valid = peak >= threshold,
        // its fp16 patch (nbeams, 1728) and score (sifter logit, or the peak without a sifter; -inf if
        // not valid).
        float *cand_peak = nullptr;
        int *cand_tree = nullptr, *cand_idm = nullptr, *cand_itime = nullptr, *cand_valid = nullptr;
        uint32_t *cand_token = nullptr;
        uint16_t *patches = nullptr;
        float *scores = nullptr;
    };

    GpuDedisperser(const DedispersionPlan &plan, const Params &params);
    ~GpuDedisperser();
    GpuDedisperser(const GpuDedisperser &) = delete;
    GpuDedisperser &operator=(const GpuDedisperser &) = delete;

    void allocate();
    void *acquire_input(long seq_id, cudaStream_t stream);
    // The next input slot as int4 data (B, nfreq, nt/2) bytes; *scales_offsets receives its fp16
    // (scale, offset) pairs (B, nfreq, nt/256, 2). Same cursor as acquire_input. The gridding kernel
    // then dequantizes while it reads (nt must be a multiple of 256).
    void *acquire_input_int4(long seq_id, cudaStream_t stream, void **scales_offsets);
    void release_input_and_launch_dd_kernels(long seq_id, cudaStream_t stream);
    Outputs acquire_output(long consumer_id, long seq_id, cudaStream_t stream, bool sync);
    void release_output(long consumer_id, long seq_id, cudaStream_t stream);
    void fill_all_weights(long itree, const float *host, long nelts);
    // Fills every weight slot and beam of every tree with the analytic SNR weights made from the
    // per-channel input variances (nfreq values > 0), and waits until they are on the GPU.
    void fill_analytic_weights(const double *freq_variances, long nfreq);
    void stop(std::exception_ptr e = nullptr);
    // Adds the candidate stage to every later batch, on its compute stream after peak finding: the
    // per-beam peak over the trees, the candidate patch of peaks >= threshold, and (if 'sifter' is not
    // null) its MLP score. Requires allocate(). The sifter is used on the compute streams from then on
    // and must not be trained at the same time; it must outlive the dedisperser or a later
    // enable_sifter() call.
    void enable_sifter(float threshold, Sifter *sifter);

    // Batched use (BatchedDedisperser): enqueues one chunk of the single batch (needs beams_per_gpu ==
    // beams_per_batch) on 'stream', every kernel reading the chunk index from the device counter
    // *chunk_ctr; input slot 0, output slot 0, weight slot 0; no events and no back-pressure (the caller
    // orders the chunks). It makes no host-side waits, so it can be captured in a CUDA graph.
    void enqueue_chunk(cudaStream_t stream, const long *chunk_ctr, const GroupTuning &tune);
    void *input_ptr(long slot) const;
    Outputs outputs_ptr(long slot) const;
    // Clears every delay line, tree state, input and output slot on 'stream' (a fresh stream of chunks:
    // later chunks see zeros as their history). Waits for this object's launched batches first.
    void zero_state(cudaStream_t stream);

    // pirate's timing loop (GpuDedisperser::time, src_lib/GpuDedisperser.cpp:1573-1665): niterations
    // batches, each copying one batch of int4 data and fp16 (scale, offset) pairs from pinned host
    // memory into the acquired int4 input slot on a copy stream, launching the kernels (dequantization
    // fused into gridding), and acquiring and releasing the output as consumer 0. rtb[i] receives the
    // real-time beams of iteration i: beams_per_batch * chunk seconds / (time between the completions
    // of iterations i-1 and i); rtb[0] = 0. Needs num_consumers == 1, nt_in a multiple of 256,
    // niterations > 2 * num_active_batches, and every cursor caught up (nothing acquired and unreleased).
    void time(long niterations, double *rtb);

    // Device bytes held by allocate() (for reporting).
    size_t device_bytes() const { return total_bytes; }
    // Pinned host bytes of the spilled delay lines (rows whose readers are more than the config's
    // max_gpu_clag chunks behind).
    size_t host_bytes() const { return host_total; }
    // Number of kernels launched per (chunk, batch).
    int kernels_per_batch() const;
    int stage2_launches() const;
    // Bytes of HBM traffic per (chunk, batch) of each kernel class (algorithmic: each element read or
    // written once, following pirate's ResourceTracker model):
    // [grid+lds (one fused kernel), candidates+sifter, stage1, stage2, pf].
    std::vector<double> algorithmic_bytes() const;

    // Kernel timing: when enabled, CUDA events bracket each kernel class
    // [grid+lds (one fused kernel), candidates+sifter, stage1, stage2, pf] on the batch's compute stream; kernel_times() synchronizes and returns
    // the accumulated milliseconds and launch counts since the last reset.
    void enable_timing(bool on);
    void kernel_times(double *ms5, long *counts5);

    const DedispersionPlan plan;
    const Params params;
    long nbatches = 0, B = 0, total_beams = 0, nslots_in = 0, nbatches_out = 0, nbatches_wt = 0;
    long num_compute_streams() const { return nstreams; }

private:
    void check_alive() const;
    template<typename F> auto entry(F &&f) -> decltype(f());
    void launch_batch(long seq_id);
    void launch_kernels(long ichunk, long ibatch, long slot_in, long slot_out, long slot_wt, cudaStream_t s,
                        long istream, const long *chunk_ctr, const GroupTuning &tune, bool fences);
    void sync_compute();

    std::mutex mtx;
    std::condition_variable cv;                     // signalled by release_output() and stop()
    std::unique_lock<std::mutex> *cur_lock = nullptr;   // the lock held by the running entry point
    std::exception_ptr error;
    bool stopped = false;
    bool allocated = false;
    long next_acq_in = 0, next_rel_in = 0;
    std::vector<long> next_acq_out, next_rel_out;

    int dtype_code = 0;
    size_t esize = 4;
    size_t total_bytes = 0;
    size_t host_total = 0;
    // Compute streams, one per active batch (pirate's CudaStreamPool compute streams,
    // include/pirate/CudaStreamPool.hpp:27-39): batch seq_id runs on computes[seq_id % nstreams] with
    // its own level-0 tree and reduction scratch; batches of the same beams are ordered by
    // ev_beams_done[ibatch] (pirate's cdd2 event-ring wait on seq_id - nbatches,
    // src_lib/GpuDedisperser.cpp:1008-1011), and the sifter's forward passes by ev_sifter.
    std::vector<cudaStream_t> computes;
    cudaStream_t compute = nullptr;   // computes[0]: weight uploads and clears, after sync_compute()
    long nstreams = 1;
    std::vector<cudaEvent_t> ev_beams_done;
    std::vector<bool> beams_done_recorded;
    cudaEvent_t ev_sifter = nullptr;
    bool sifter_recorded = false;

    // Per-slot events.
    std::vector<cudaEvent_t> ev_in_acquired, ev_in_free, ev_out_done;
    std::vector<bool> slot_int4;   // input slot holds int4 data (acquire_input_int4)
    std::vector<std::vector<cudaEvent_t>> ev_out_released;   // [consumer][slot]
    std::vector<bool> in_free_recorded, out_done_recorded;
    std::vector<std::vector<bool>> out_released_recorded;

    // Static device tables.
    DeviceBuffer d_grid_f0, d_grid_cnt, d_grid_woff, d_grid_w;
    struct Stage1
    {
        DeviceBuffer ring, ring_off, ring_cap, state;
        // stage-2 read tables (the same as ring_off/ring_cap except for spilled rows: their read rings),
        // the spilled-row table, and the rows' host zones (mapped pinned memory)
        DeviceBuffer ring_off_r, ring_cap_r, spill_rows;
        void *host = nullptr, *host_dev = nullptr;
        size_t host_bytes = 0;
        int nspill = 0;
        long ring_beam_stride = 0, state_per_block = 0;
        int nblocks = 0, nt = 0, rank = 0;
        long lds_cap = 0;
        DeviceBuffer lds;
    };
    struct Stage2
    {
        DeviceBuffer state, pfring, m_to_n, out_max, out_argmax, wt;
        long pf_cap = 0, state_per_block = 0;
        int nblocks = 0, M = 0, N = 0, P = 0, L = 0, tpad = 0, Dout = 0;
        int sb_count[5] = {0, 0, 0, 0, 0}, sb_mbase[5] = {0, 0, 0, 0, 0};
    };
    bool timing = false;
    std::vector<std::vector<std::pair<cudaEvent_t, cudaEvent_t>>> tev;   // per class, pending event pairs
    double tms[5] = {0, 0, 0, 0, 0};
    long tcount[5] = {0, 0, 0, 0, 0};
    std::vector<cudaEvent_t> ev_pool;
    cudaEvent_t tick(int cls, cudaEvent_t start, cudaStream_t s);
    void drain_timing();

    std::vector<Stage1> s1;
    std::vector<Stage2> s2;
    DeviceBuffer d_inputs, d_tree0, d_lds_state;
    DeviceBuffer d_qdata, d_qscoff;   // int4 input slots (allocated when nt is a multiple of 256)
    // Candidate stage: per output slot, 8 arrays of B 4-byte entries (peak, tree, idm, itime, token,
    // valid, logits, scores) and B patches.
    bool sift = false;
    float sift_threshold = 0.0f;
    Sifter *sifter = nullptr;
    DeviceBuffer d_cand, d_patches, d_peak_scratch;
    int peak_split = 1;
    PatchArgs patch_args;
    void *acquire_slot(long seq_id, cudaStream_t stream, void **int4);
};

}  // namespace pb2
