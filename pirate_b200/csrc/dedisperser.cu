// dedisperser.cu -- host driver of the B200 dedispersion path (see dedisperser.hpp).

#include "dedisperser.hpp"
#include "avar.hpp"

#include <algorithm>
#include <limits>
#include <map>
#include <chrono>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>

namespace pb2 {

using std::runtime_error;
using std::vector;

#define CUDA_CHECK(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { \
    std::stringstream _ss; _ss << #x << ": " << cudaGetErrorString(_e); throw runtime_error(_ss.str()); } } while (0)

static long next_pow2(long n) { long p = 1; while (p < n) p <<= 1; return p; }
static long round_up(long n, long k) { return ((n + k - 1) / k) * k; }


DeviceBuffer::~DeviceBuffer() { if (ptr) cudaFree(ptr); }

void DeviceBuffer::alloc(size_t n)
{
    if (ptr) { cudaFree(ptr); ptr = nullptr; }
    nbytes = n;
    if (n == 0) return;
    CUDA_CHECK(cudaMalloc(&ptr, n));
    CUDA_CHECK(cudaMemset(ptr, 0, n));
}

void DeviceBuffer::upload(const void *host, size_t n)
{
    alloc(n);
    if (n) CUDA_CHECK(cudaMemcpy(ptr, host, n, cudaMemcpyHostToDevice));
}


// -------------------------------------------------------------------------------------------------
// GpuDedisperser


GpuDedisperser::GpuDedisperser(const DedispersionPlan &plan_, const Params &params_) : plan(plan_), params(params_)
{
    B = plan.beams_per_batch;
    total_beams = plan.beams_per_gpu;
    nbatches = total_beams / B;
    nslots_in = plan.num_active_batches;
    nstreams = plan.num_active_batches;
    nbatches_out = params.nbatches_out ? params.nbatches_out : plan.num_active_batches;
    nbatches_wt = params.nbatches_wt ? params.nbatches_wt : nbatches_out;
    if (params.num_consumers < 0) throw runtime_error("GpuDedisperser: num_consumers must be >= 0");
    if (params.cuda_device_id < 0) throw runtime_error("GpuDedisperser: cuda_device_id must be >= 0");
    if (nbatches_out <= 0 || nbatches_wt <= 0) throw runtime_error("GpuDedisperser: nbatches_out/nbatches_wt must be > 0");
    dtype_code = int(plan.dtype);
    esize = (plan.dtype == Dtype::f32) ? 4 : 2;
    next_acq_out.assign(params.num_consumers, 0);
    next_rel_out.assign(params.num_consumers, 0);
}

GpuDedisperser::~GpuDedisperser()
{
    int dev = 0;
    cudaGetDevice(&dev);
    cudaSetDevice(params.cuda_device_id);
    for (cudaStream_t c : computes) cudaStreamSynchronize(c);
    for (Stage1 &st : s1) if (st.host) cudaFreeHost(st.host);
    for (auto &v : tev) for (auto &pr : v) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    auto kill = [](vector<cudaEvent_t> &v) { for (cudaEvent_t e : v) if (e) cudaEventDestroy(e); v.clear(); };
    kill(ev_in_acquired);
    kill(ev_in_free);
    kill(ev_out_done);
    for (auto &v : ev_out_released) kill(v);
    kill(ev_beams_done);
    if (ev_sifter) cudaEventDestroy(ev_sifter);
    for (cudaStream_t c : computes) cudaStreamDestroy(c);
    cudaSetDevice(dev);
}

void GpuDedisperser::check_alive() const
{
    if (error) std::rethrow_exception(error);
    if (stopped) throw runtime_error("GpuDedisperser: entry point called after stop()");
}

template<typename F>
auto GpuDedisperser::entry(F &&f) -> decltype(f())
{
    std::unique_lock<std::mutex> lk(mtx);
    struct Scope {
        std::unique_lock<std::mutex> *&slot;
        Scope(std::unique_lock<std::mutex> *&s, std::unique_lock<std::mutex> *l) : slot(s) { slot = l; }
        ~Scope() { slot = nullptr; }
    } scope(cur_lock, &lk);
    check_alive();
    try {
        return f();
    } catch (...) {
        error = std::current_exception();
        stopped = true;
        throw;
    }
}

void GpuDedisperser::sync_compute()
{
    for (cudaStream_t c : computes) CUDA_CHECK(cudaStreamSynchronize(c));
}

void GpuDedisperser::stop(std::exception_ptr e)
{
    std::lock_guard<std::mutex> lk(mtx);
    if (!error && e) error = e;
    stopped = true;
    cv.notify_all();
}

int GpuDedisperser::kernels_per_batch() const
{
    // candidate stage: beam peaks, patches, then the MLP (3 GEMMs) and the score mask, or the mask alone
    const int cand = sift ? (3 + (sifter ? 4 : 1)) : 0;
    int spill = 0;
    for (const Stage1 &st : s1) spill += st.nspill ? 2 : 0;
    return 1 + int(plan.num_primary_trees) + spill + stage2_launches() + int(plan.ntrees) + cand;
}

void GpuDedisperser::enable_sifter(float threshold, Sifter *sf)
{
    entry([&]() {
        if (!allocated) throw runtime_error("GpuDedisperser::enable_sifter(): allocate() was not called");
        if (plan.ntrees > kPatchMaxTrees) throw runtime_error("GpuDedisperser::enable_sifter(): too many trees");
        if (sf && (sf->device != params.cuda_device_id || sf->max_batch < B))
            throw runtime_error("GpuDedisperser::enable_sifter(): the sifter must be on this device with max_batch >= beams_per_batch");
        CUDA_CHECK(cudaSetDevice(params.cuda_device_id));
        sync_compute();
        if (!d_cand.ptr) {
            d_cand.alloc(size_t(nbatches_out) * 8 * B * 4);
            d_patches.alloc(size_t(nbatches_out) * B * kPatchLen * sizeof(uint16_t));
            // split beam-peak reduction: about four waves of blocks over the (tree, beam) pairs
            peak_split = int(std::max(1L, std::min(256L, (4L * 148 + plan.ntrees * B - 1) / (plan.ntrees * B))));
            d_peak_scratch.alloc(size_t(nstreams) * B * plan.ntrees * peak_split * 16);
        }
        memset(&patch_args, 0, sizeof(patch_args));
        patch_args.ntrees = int(plan.ntrees);
        for (long i = 0; i < plan.ntrees; i++) {
            const DedispersionTree &t = plan.trees[i];
            const FrequencySubbands &fs = t.frequency_subbands;
            PatchTree &pt = patch_args.t[i];
            if (fs.pf_rank > 4) throw runtime_error("GpuDedisperser::enable_sifter(): peak-finding rank above 4");
            if (s2[i].pf_cap < 64) throw runtime_error("GpuDedisperser::enable_sifter(): subband rows hold fewer than 64 samples");
            pt.pf = s2[i].pfring.ptr;
            pt.pf_cap = s2[i].pf_cap;
            pt.M = int(fs.M);
            pt.ndm_out = int(t.ndm_out);
            pt.nt_ds = int(t.nt_ds);
            pt.Dout = int(t.pf.time_downsampling);
            pt.Dcore = int(t.Dcore);
            pt.pf_rank = int(fs.pf_rank);
            for (int d = 0; d < 16; d++) pt.d_to_m[d] = -1;
            pt.nfull = -1;
            for (long m = 0; m < fs.M; m++) {
                long n = fs.m_to_n[m];
                if (fs.n_to_flo[n] == 0 && fs.n_to_fhi[n] == pow2(fs.pf_rank)) {
                    pt.d_to_m[fs.m_to_d[m]] = int(m);
                    pt.nfull = int(n);
                }
            }
            if (pt.nfull < 0) throw runtime_error("GpuDedisperser::enable_sifter(): a tree without a full-band search");
            pt.ndm_wt = int(t.ndm_wt);
            pt.nt_wt = int(t.nt_wt);
            pt.nt_out = int(t.nt_out);
            pt.P = int(t.nprofiles);
            pt.N = int(fs.N);
        }
        patch_args.threshold = threshold;
        patch_args.B = int(B);
        sift = true;
        sift_threshold = threshold;
        sifter = sf;
    });
}

// Stage-2 launches per batch: runs of consecutive output trees with the same stage-2 kernel (same dd
// rank and staggered-subband flag), at most kStage2MaxTrees per launch.
int GpuDedisperser::stage2_launches() const
{
    int n = 0;
    for (long i0 = 0; i0 < plan.ntrees;) {
        long i1 = i0 + 1;
        auto stag = [&](long i) {
            const FrequencySubbands &fs = plan.trees[i].frequency_subbands;
            bool x = false;
            for (long l = 1; l <= fs.pf_rank && l < 5; l++) x = x || (fs.subband_counts[l] >= 2);
            return x;
        };
        while (i1 < plan.ntrees && i1 - i0 < kStage2MaxTrees && plan.trees[i1].dd_rank == plan.trees[i0].dd_rank && stag(i1) == stag(i0)) i1++;
        n++;
        i0 = i1;
    }
    return n;
}

std::vector<double> GpuDedisperser::algorithmic_bytes() const
{
    // Compulsory bytes each kernel must move per (chunk, batch): every element it reads or writes
    // once (the reference's ResourceTracker model, src_lib/TreeGriddingKernel.cu:117,
    // GpuLaggedDownsamplingKernel.cu:767-774, DedispersionKernel.cu:514-516, CoalescedDdKernel2.cu:128-135).
    double S = double(esize);
    long rank = plan.config.toplevel_tree_rank, nt = plan.nt_in;
    // Fused gridding + lagged downsampling: read the input, write the level-0 tree and every level's rows.
    double grid = double(B) * (plan.nfreq + pow2(rank)) * nt * S;
    double lds = 0, st1 = 0, st2 = 0, pf = 0;
    for (long p = 1; p < plan.num_primary_trees; p++) grid += double(B) * pow2(rank - 1) * (nt >> p) * S;
    for (long p = 0; p < plan.num_primary_trees; p++) {
        long rk = plan.stage1_dd_rank[p] + plan.stage1_amb_rank[p];
        st1 += 2.0 * B * pow2(rk) * (nt >> p) * S;
    }
    for (const DedispersionTree &t : plan.trees) {
        long M = t.frequency_subbands.M;
        st2 += double(B) * pow2(t.total_rank()) * t.nt_ds * S + double(B) * t.ndm_out * M * t.nt_ds * S;
        pf += double(B) * t.ndm_out * M * t.nt_ds * S + double(B) * t.ndm_out * t.nt_out * (S + 4);
    }
    return {grid, lds, st1, st2, pf};
}

void GpuDedisperser::enable_timing(bool on)
{
    entry([&]() {
        timing = on;
        tev.assign(5, {});
        for (int i = 0; i < 5; i++) { tms[i] = 0; tcount[i] = 0; }
    });
}

// Records an event on the compute stream. With start == nullptr returns a fresh start event;
// otherwise closes the interval (start, now) for class 'cls'.
cudaEvent_t GpuDedisperser::tick(int cls, cudaEvent_t start, cudaStream_t s)
{
    if (!timing) return nullptr;
    cudaEvent_t e;
    if (!ev_pool.empty()) { e = ev_pool.back(); ev_pool.pop_back(); }
    else CUDA_CHECK(cudaEventCreate(&e));
    CUDA_CHECK(cudaEventRecord(e, s));
    if (start) {
        tev[cls].push_back({start, e});
        if (tev[cls].size() > 256) drain_timing();
    }
    return e;
}

void GpuDedisperser::drain_timing()
{
    for (int c = 0; c < 5; c++) {
        for (auto &pr : tev[c]) {
            CUDA_CHECK(cudaEventSynchronize(pr.second));
            float ms = 0;
            CUDA_CHECK(cudaEventElapsedTime(&ms, pr.first, pr.second));
            tms[c] += ms;
            tcount[c]++;
            ev_pool.push_back(pr.first);
            ev_pool.push_back(pr.second);
        }
        tev[c].clear();
    }
}

void GpuDedisperser::kernel_times(double *ms5, long *counts5)
{
    entry([&]() {
        if (timing) drain_timing();
        for (int i = 0; i < 5; i++) { ms5[i] = tms[i]; counts5[i] = tcount[i]; }
    });
}

void GpuDedisperser::allocate()
{
    entry([&]() {
        if (allocated) throw runtime_error("GpuDedisperser::allocate() called twice");
        CUDA_CHECK(cudaSetDevice(params.cuda_device_id));
        computes.resize(nstreams);
        for (auto &c : computes) CUDA_CHECK(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking));
        compute = computes[0];
        CUDA_CHECK(cudaEventCreateWithFlags(&ev_sifter, cudaEventDisableTiming));
        auto mk = [](vector<cudaEvent_t> &v, long n) {
            v.resize(n);
            for (auto &e : v) CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        };
        mk(ev_in_acquired, nslots_in);
        mk(ev_in_free, nslots_in);
        mk(ev_out_done, nbatches_out);
        mk(ev_beams_done, nbatches);
        beams_done_recorded.assign(nbatches, false);
        ev_out_released.resize(params.num_consumers);
        for (auto &v : ev_out_released) mk(v, nbatches_out);
        in_free_recorded.assign(nslots_in, false);
        out_done_recorded.assign(nbatches_out, false);
        out_released_recorded.assign(params.num_consumers, vector<bool>(nbatches_out, false));

        const long rank = plan.config.toplevel_tree_rank, nt = plan.nt_in, F = plan.nfreq, N = pow2(rank);
        const long npri = plan.num_primary_trees;
        total_bytes = 0;
        host_total = 0;
        auto add = [&](DeviceBuffer &d, size_t n) { d.alloc(n); total_bytes += n; };

        // Tree gridding table (src_lib/TreeGriddingKernel.cu:80-97): channel n covers input channels
        // [floor(cm[n+1]), floor(cm[n])] with overlap weights float(w) in ascending order.
        vector<double> cm = plan.config.make_channel_map();
        vector<int> f0(N), cnt(N), woff(N);
        vector<float> w;
        for (long n = 0; n < N; n++) {
            double a0 = cm[n + 1], a1 = cm[n];
            long if0 = std::max(long(a0), 0L), if1 = std::min(long(a1) + 1, F);
            f0[n] = int(if0);
            cnt[n] = int(std::max(if1 - if0, 0L));
            woff[n] = int(w.size());
            for (long f = if0; f < if1; f++) {
                double lo = std::max(a0, double(f)), hi = std::min(a1, double(f) + 1);
                w.push_back(float(std::max(hi - lo, 0.0)));
            }
        }
        d_grid_f0.upload(f0.data(), f0.size() * 4);
        d_grid_cnt.upload(cnt.data(), cnt.size() * 4);
        d_grid_woff.upload(woff.data(), woff.size() * 4);
        d_grid_w.upload(w.data(), w.size() * 4);

        add(d_inputs, size_t(nslots_in) * B * F * nt * esize);
        if (nt % 256 == 0) {
            add(d_qdata, size_t(nslots_in) * B * F * (nt / 2));
            add(d_qscoff, size_t(nslots_in) * B * F * (nt / 256) * 2 * sizeof(uint16_t));
        }
        slot_int4.assign(nslots_in, false);
        add(d_tree0, size_t(nstreams) * B * N * nt * esize);
        if (npri > 1) add(d_lds_state, size_t(2) * total_beams * (npri - 1) * (N / 2) * sizeof(float));

        s1.clear();
        s1.resize(npri);
        for (long p = 0; p < npri; p++) {
            Stage1 &st = s1[p];
            int R1 = plan.stage1_dd_rank[p], A1 = plan.stage1_amb_rank[p];
            if (R1 < 1 || R1 > 8) throw runtime_error("GpuDedisperser: stage-1 dd rank must be in [1, 8]");
            st.rank = R1;
            st.nblocks = 1 << A1;
            st.nt = int(nt >> p);
            st.state_per_block = stage1_state_floats(R1);
            add(st.state, size_t(total_beams) * st.nblocks * st.state_per_block * sizeof(float));

            long nrows = pow2(R1 + A1);
            // Chunk offsets d = ceil((lag + 1) / nt) of every row's readers (this primary tree's stage-2
            // trees). A row whose readers all have the same d >= 2, above the config's max_gpu_clag, is
            // spilled to host memory (MegaRingbuf's host zones, src_lib/MegaRingbuf.cpp:155-183).
            vector<long> dlo(nrows, std::numeric_limits<long>::max()), dhi(nrows, -1);
            for (const DedispersionTree &t : plan.trees) {
                if (t.primary_tree_index != p) continue;
                for (long a = 0; a < pow2(t.dd_rank); a++)
                    for (long d = 0; d < pow2(t.amb_rank); d++) {
                        long row = a * pow2(t.amb_rank) + d;
                        long dc = (rb_lag(a, d, t.amb_rank, t.dd_rank, p > 0) + st.nt) / st.nt;   // ceil((lag + 1) / nt)
                        dlo[row] = std::min(dlo[row], dc);
                        dhi[row] = std::max(dhi[row], dc);
                    }
            }
            vector<char> spill(nrows, 0);
            for (long row = 0; row < nrows; row++)
                spill[row] = (dhi[row] >= 2 && dlo[row] == dhi[row] && dlo[row] > plan.config.max_gpu_clag);

            // Per beam: block by block, the block's resident lines then its spilled rows' write slots
            // (nt samples); then every spilled row's read ring (2 nt samples).
            vector<long> off(nrows), off_r(nrows);
            vector<int> cap(nrows), cap_r(nrows);
            long tot = 0;
            for (long blk = 0; blk < st.nblocks; blk++) {
                for (long r = 0; r < pow2(R1); r++) {
                    long row = blk * pow2(R1) + r;
                    if (spill[row]) continue;
                    // one sample more than the lags need: stage 2 also reads the sample before its first
                    cap[row] = cap_r[row] = int(round_up(plan.max_row_lag[p][row] + st.nt + 1, 32));
                    off[row] = off_r[row] = tot;
                    tot += cap[row];
                }
                for (long r = 0; r < pow2(R1); r++) {
                    long row = blk * pow2(R1) + r;
                    if (!spill[row]) continue;
                    cap[row] = st.nt;
                    off[row] = tot;
                    tot += st.nt;
                }
            }
            std::map<long, std::vector<long>> zones;   // d -> spilled rows
            for (long row = 0; row < nrows; row++)
                if (spill[row]) {
                    cap_r[row] = 2 * st.nt;
                    off_r[row] = tot;
                    tot += 2 * st.nt;
                    zones[dlo[row]].push_back(row);
                }
            st.ring_beam_stride = tot;
            // The stage-1 kernel indexes a block's 2^R1 delay lines with 32-bit offsets.
            for (long blk = 0; blk < st.nblocks; blk++) {
                long lo = std::numeric_limits<long>::max(), hi = 0;
                for (long r = 0; r < pow2(R1); r++) {
                    long row = blk * pow2(R1) + r;
                    lo = std::min(lo, off[row]);
                    hi = std::max(hi, off[row] + cap[row]);
                }
                if (hi - lo >= (1L << 31) || off[blk * pow2(R1)] != lo)
                    throw runtime_error("GpuDedisperser::allocate(): stage-1 delay lines of one block exceed 2^31 samples");
            }
            st.ring_off.upload(off.data(), off.size() * sizeof(long));
            st.ring_cap.upload(cap.data(), cap.size() * sizeof(int));
            st.ring_off_r.upload(off_r.data(), off_r.size() * sizeof(long));
            st.ring_cap_r.upload(cap_r.data(), cap_r.size() * sizeof(int));
            add(st.ring, size_t(total_beams) * tot * esize);

            // Host zones: zone d holds S = d + 1 chunk slots of its rows for every beam.
            vector<SpillRow> srows;
            long hb = 0;
            for (auto &z : zones) {
                const long d = z.first, nz = long(z.second.size());
                for (long k = 0; k < nz; k++) {
                    long row = z.second[k];
                    SpillRow sr;
                    sr.w_off = off[row];
                    sr.r_off = off_r[row];
                    sr.h_base = hb;
                    sr.n_z = int(nz);
                    sr.k = int(k);
                    sr.S = int(d + 1);
                    sr.d = int(d);
                    srows.push_back(sr);
                }
                hb += (d + 1) * total_beams * nz * st.nt;
            }
            st.nspill = int(srows.size());
            if (st.nspill) {
                st.spill_rows.upload(srows.data(), srows.size() * sizeof(SpillRow));
                st.host_bytes = size_t(hb) * esize;
                CUDA_CHECK(cudaHostAlloc(&st.host, st.host_bytes, cudaHostAllocMapped | cudaHostAllocPortable));
                memset(st.host, 0, st.host_bytes);
                CUDA_CHECK(cudaHostGetDevicePointer(&st.host_dev, st.host, 0));
                host_total += st.host_bytes;
            }

            if (p > 0) {
                st.lds_cap = next_pow2(st.nt + (1L << R1) - 1);
                add(st.lds, size_t(total_beams) * (N / 2) * st.lds_cap * esize);
            }
        }

        s2.clear();
        s2.resize(plan.ntrees);
        for (long i = 0; i < plan.ntrees; i++) {
            const DedispersionTree &t = plan.trees[i];
            Stage2 &st = s2[i];
            const FrequencySubbands &fs = t.frequency_subbands;
            if (t.dd_rank < 1 || t.dd_rank > 8) throw runtime_error("GpuDedisperser: stage-2 dd rank must be in [1, 8]");
            if (fs.pf_rank != split_rb(t.dd_rank)) throw runtime_error("GpuDedisperser: unexpected peak-finding rank");
            st.nblocks = 1 << t.amb_rank;
            st.M = fs.M;
            st.N = fs.N;
            st.P = t.nprofiles;
            st.L = std::max(integer_log2(t.pf.max_width), 1);
            st.tpad = int(std::max(2 * t.pf.max_width, 4L));
            st.Dout = int(t.pf.time_downsampling);
            st.state_per_block = stage2_state_floats(t.dd_rank);
            add(st.state, size_t(total_beams) * st.nblocks * st.state_per_block * sizeof(float));
            int mb = 0;
            for (int l = 0; l <= fs.pf_rank; l++) {
                st.sb_count[l] = int(fs.subband_counts[l]);
                st.sb_mbase[l] = mb;
                mb += int(fs.subband_counts[l]) << l;
            }
            if (mb != st.M) throw runtime_error("GpuDedisperser: multiplet count mismatch");

            // The stage-2 kernel emits subband rows already delayed by their alignment lag
            // (see regtree.cuh), so the peak finder reads every row at the same time.
            vector<int> m2n(st.M);
            for (int m = 0; m < st.M; m++) m2n[m] = int(fs.m_to_n[m]);
            st.m_to_n.upload(m2n.data(), m2n.size() * sizeof(int));
            st.pf_cap = next_pow2(t.nt_ds + st.tpad + st.Dout);
            add(st.pfring, size_t(total_beams) * t.ndm_out * st.M * st.pf_cap * esize);
            add(st.out_max, size_t(nbatches_out) * B * t.ndm_out * t.nt_out * esize);
            add(st.out_argmax, size_t(nbatches_out) * B * t.ndm_out * t.nt_out * sizeof(uint32_t));
            add(st.wt, size_t(nbatches_wt) * B * t.ndm_wt * t.nt_wt * t.nprofiles * fs.N * sizeof(float));
        }
        CUDA_CHECK(cudaDeviceSynchronize());
        allocated = true;
    });
}

void *GpuDedisperser::acquire_input(long seq_id, cudaStream_t stream)
{
    return acquire_slot(seq_id, stream, nullptr);
}

void *GpuDedisperser::acquire_input_int4(long seq_id, cudaStream_t stream, void **scales_offsets)
{
    if (!scales_offsets) throw runtime_error("GpuDedisperser::acquire_input_int4(): null scales_offsets");
    return acquire_slot(seq_id, stream, scales_offsets);
}

// int4 != nullptr: acquire the slot's int4 buffers (data returned, scales/offsets in *int4).
void *GpuDedisperser::acquire_slot(long seq_id, cudaStream_t stream, void **int4)
{
    return entry([&]() -> void * {
        if (!allocated) throw runtime_error("GpuDedisperser::acquire_input(): allocate() was not called");
        if (seq_id != next_acq_in)
            throw runtime_error("GpuDedisperser::acquire_input(): expected seq_id=" + std::to_string(next_acq_in) + ", got " + std::to_string(seq_id));
        if (int4 && !d_qdata.ptr)
            throw runtime_error("GpuDedisperser::acquire_input_int4(): time_samples_per_chunk must be a multiple of 256");
        long slot = seq_id % nslots_in;
        if (in_free_recorded[slot]) CUDA_CHECK(cudaStreamWaitEvent(stream, ev_in_free[slot], 0));
        next_acq_in++;
        slot_int4[slot] = (int4 != nullptr);
        if (int4) {
            *int4 = d_qscoff.as<char>() + size_t(slot) * B * plan.nfreq * (plan.nt_in / 256) * 2 * sizeof(uint16_t);
            return d_qdata.as<char>() + size_t(slot) * B * plan.nfreq * (plan.nt_in / 2);
        }
        return d_inputs.as<char>() + size_t(slot) * B * plan.nfreq * plan.nt_in * esize;
    });
}

void GpuDedisperser::release_input_and_launch_dd_kernels(long seq_id, cudaStream_t stream)
{
    entry([&]() {
        if (seq_id != next_rel_in || seq_id >= next_acq_in)
            throw runtime_error("GpuDedisperser::release_input_and_launch_dd_kernels(): expected seq_id=" + std::to_string(next_rel_in) + ", got " + std::to_string(seq_id));
        // Output back-pressure: the batch writes output slot seq_id % nbatches_out, which every consumer
        // must have released (as seq_id - nbatches_out) first. Like pirate's blocking wait on its
        // release-output event ring, wait for that release on the host (other threads release while
        // this one waits), with a bound.
        if (seq_id >= nbatches_out && params.num_consumers > 0) {
            const long need = seq_id - nbatches_out;
            auto released = [&] {
                if (stopped) return true;
                for (long c = 0; c < params.num_consumers; c++)
                    if (next_rel_out[c] <= need) return false;
                return true;
            };
            const long tmo = params.release_timeout_ms > 0 ? params.release_timeout_ms : 60000;
            if (!cv.wait_for(*cur_lock, std::chrono::milliseconds(tmo), released)) {
                long c = 0;
                while (next_rel_out[c] > need) c++;
                throw runtime_error("GpuDedisperser::release_input_and_launch_dd_kernels(): consumer " + std::to_string(c) +
                                    " has not released seq_id=" + std::to_string(need) + " within " + std::to_string(tmo) +
                                    " ms (output slots are reused every nbatches_out=" + std::to_string(nbatches_out) + " batches)");
            }
            if (stopped) throw runtime_error("GpuDedisperser: stopped while waiting for an output release");
        }
        long slot = seq_id % nslots_in;
        CUDA_CHECK(cudaSetDevice(params.cuda_device_id));
        CUDA_CHECK(cudaEventRecord(ev_in_acquired[slot], stream));
        CUDA_CHECK(cudaStreamWaitEvent(computes[seq_id % nstreams], ev_in_acquired[slot], 0));
        launch_batch(seq_id);
        next_rel_in++;
        cv.notify_all();
    });
}

void GpuDedisperser::launch_batch(long seq_id)
{
    const long ichunk = seq_id / nbatches, ibatch = seq_id % nbatches, istream = seq_id % nstreams;
    cudaStream_t s = computes[istream];
    // The previous chunk of these beams may have run on another compute stream: its delay lines and
    // tree state must be complete.
    if (beams_done_recorded[ibatch]) CUDA_CHECK(cudaStreamWaitEvent(s, ev_beams_done[ibatch], 0));
    launch_kernels(ichunk, ibatch, seq_id % nslots_in, seq_id % nbatches_out, seq_id % nbatches_wt, s, istream, nullptr,
                   GroupTuning(), true);
    CUDA_CHECK(cudaEventRecord(ev_beams_done[ibatch], s));
    beams_done_recorded[ibatch] = true;
}

void GpuDedisperser::enqueue_chunk(cudaStream_t stream, const long *chunk_ctr, const GroupTuning &tune)
{
    entry([&]() {
        if (!allocated) throw runtime_error("GpuDedisperser::enqueue_chunk(): allocate() was not called");
        if (nbatches != 1) throw runtime_error("GpuDedisperser::enqueue_chunk(): needs beams_per_gpu == beams_per_batch");
        if (!chunk_ctr) throw runtime_error("GpuDedisperser::enqueue_chunk(): null chunk counter");
        launch_kernels(0, 0, 0, 0, 0, stream, 0, chunk_ctr, tune, false);
    });
}

void *GpuDedisperser::input_ptr(long slot) const
{
    if (slot < 0 || slot >= nslots_in || !allocated) throw runtime_error("GpuDedisperser::input_ptr(): bad slot");
    return d_inputs.as<char>() + size_t(slot) * B * plan.nfreq * plan.nt_in * esize;
}

GpuDedisperser::Outputs GpuDedisperser::outputs_ptr(long slot) const
{
    if (slot < 0 || slot >= nbatches_out || !allocated) throw runtime_error("GpuDedisperser::outputs_ptr(): bad slot");
    Outputs o;
    o.dtype = plan.dtype;
    o.nbeams = B;
    for (long i = 0; i < plan.ntrees; i++) {
        const DedispersionTree &t = plan.trees[i];
        size_t osz = size_t(B) * t.ndm_out * t.nt_out;
        o.ndm_out.push_back(t.ndm_out);
        o.nt_out.push_back(t.nt_out);
        o.out_max.push_back(s2[i].out_max.as<char>() + size_t(slot) * osz * esize);
        o.out_argmax.push_back(s2[i].out_argmax.as<uint32_t>() + size_t(slot) * osz);
    }
    return o;
}

void GpuDedisperser::zero_state(cudaStream_t s)
{
    entry([&]() {
        if (!allocated) throw runtime_error("GpuDedisperser::zero_state(): allocate() was not called");
        CUDA_CHECK(cudaSetDevice(params.cuda_device_id));
        sync_compute();   // no batch of this object may still be running
        auto z = [&](const DeviceBuffer &d) { if (d.ptr) CUDA_CHECK(cudaMemsetAsync(d.ptr, 0, d.nbytes, s)); };
        z(d_inputs); z(d_tree0); z(d_lds_state); z(d_qdata); z(d_qscoff); z(d_cand); z(d_patches);
        for (auto &st : s1) { z(st.ring); z(st.state); z(st.lds); }
        for (auto &st : s2) { z(st.state); z(st.pfring); z(st.out_max); z(st.out_argmax); }
    });
}

void GpuDedisperser::launch_kernels(long ichunk, long ibatch, long slot_in, long slot_out, long slot_wt, cudaStream_t s,
                                    long istream, const long *ctr, const GroupTuning &tune, bool fences)
{
    const long rank = plan.config.toplevel_tree_rank, nt = plan.nt_in, F = plan.nfreq, N = pow2(rank);
    const long npri = plan.num_primary_trees;
    const int beam0 = int(ibatch * B);
    const bool tk = (ctr == nullptr);   // kernel timing ticks only on the compute streams
    char *tree0 = d_tree0.as<char>() + size_t(istream) * B * N * nt * esize;

    GridLdsArgs g;
    memset(&g, 0, sizeof(g));
    g.in = d_inputs.as<char>() + size_t(slot_in) * B * F * nt * esize;
    if (slot_int4[slot_in]) {
        g.q_data = d_qdata.as<char>() + size_t(slot_in) * B * F * (nt / 2);
        g.q_scoff = d_qscoff.as<char>() + size_t(slot_in) * B * F * (nt / 256) * 2 * sizeof(uint16_t);
    }
    g.tree0 = tree0;
    g.chan_f0 = d_grid_f0.as<int>();
    g.chan_cnt = d_grid_cnt.as<int>();
    g.chan_woff = d_grid_woff.as<int>();
    g.chan_w = d_grid_w.as<float>();
    g.F = int(F); g.rank = int(rank); g.T = int(nt); g.nlev = int(npri - 1);
    for (long p = 1; p < npri; p++) {
        g.ring[p - 1] = s1[p].lds.ptr;
        g.cap_mask[p - 1] = s1[p].lds_cap - 1;
    }
    g.state = d_lds_state.as<float>();
    g.lag_rank = (npri > 1) ? int(plan.stage1_dd_rank[1]) : 0;
    g.ichunk = ichunk;
    g.chunk_ctr = ctr;
    g.block_target = tune.grid_block;
    g.beam0 = beam0; g.B = int(B); g.total_beams = int(total_beams);
    cudaEvent_t t0 = tk ? tick(0, nullptr, s) : nullptr;
    launch_grid_lds(g, dtype_code, s);
    if (tk) tick(0, t0, s);
    if (fences) {
        CUDA_CHECK(cudaEventRecord(ev_in_free[slot_in], s));
        in_free_recorded[slot_in] = true;
    }

    for (long p = 0; p < npri; p++) {
        Stage1 &st = s1[p];
        Stage1Args a;
        memset(&a, 0, sizeof(a));
        a.rank = st.rank;
        a.state_per_block = st.state_per_block;
        a.state = st.state.as<float>();
        if (p == 0) {
            a.in = tree0;
            a.in_beam_stride = N * nt;
            a.in_row_stride = nt;
            a.in_mask = -1;
            a.in_s0 = 0;
            a.in_lag0 = a.in_lag1 = 0;
            a.in_beam0 = 0;
        } else {
            a.in = st.lds.ptr;
            a.in_beam_stride = (N / 2) * st.lds_cap;
            a.in_row_stride = st.lds_cap;
            a.in_mask = st.lds_cap - 1;
            a.in_s0 = ichunk * st.nt;
            a.in_lag0 = a.in_lag1 = 0;   // the lagged-downsampling kernel wrote the rows already delayed
            a.in_beam0 = beam0;
        }
        a.ring = st.ring.ptr;
        a.ring_off = st.ring_off.as<long>();
        a.ring_cap = st.ring_cap.as<int>();
        a.ring_beam_stride = st.ring_beam_stride;
        a.s0 = ichunk * st.nt;
        a.nt = st.nt;
        a.beam0 = beam0;
        a.chunk_ctr = ctr;
        cudaEvent_t t2 = tk ? tick(2, nullptr, s) : nullptr;
        launch_stage1(a, dtype_code, st.nblocks, int(B), s);
        if (st.nspill) {
            // host spill: this chunk of the spilled rows to their host zones, and the chunk that
            // stage 2 reads next from the host into the read rings
            SpillArgs sa;
            memset(&sa, 0, sizeof(sa));
            sa.ring = st.ring.ptr;
            sa.ring_beam_stride = st.ring_beam_stride;
            sa.host = st.host_dev;
            sa.rows = st.spill_rows.as<SpillRow>();
            sa.nrows = st.nspill;
            sa.nt = st.nt;
            sa.esize = int(esize);
            sa.total_beams = int(total_beams);
            sa.beam0 = beam0;
            sa.B = int(B);
            sa.ichunk = ichunk;
            sa.chunk_ctr = ctr;
            launch_spill_g2h(sa, s);
            launch_spill_h2g(sa, s);
        }
        if (tk) tick(2, t2, s);
    }

    std::vector<Stage2Args> a2(plan.ntrees);
    std::vector<int> nb2(plan.ntrees);
    for (long i = 0; i < plan.ntrees; i++) {
        const DedispersionTree &t = plan.trees[i];
        Stage2 &st = s2[i];
        Stage1 &src = s1[t.primary_tree_index];
        Stage2Args &a = a2[i];
        memset(&a, 0, sizeof(a));
        a.rank = t.dd_rank;
        a.state_per_block = st.state_per_block;
        a.state = st.state.as<float>();
        a.ring = src.ring.ptr;
        a.ring_off = src.ring_off_r.as<long>();   // spilled rows are read from their read rings
        a.ring_cap = src.ring_cap_r.as<int>();
        a.ring_beam_stride = src.ring_beam_stride;
        a.amb_rank = t.amb_rank;
        a.uflag = (t.primary_tree_index > 0) ? 1 : 0;
        for (int l = 0; l < 5; l++) { a.sb_count[l] = st.sb_count[l]; a.sb_mbase[l] = st.sb_mbase[l]; }
        a.pf = st.pfring.ptr;
        a.M = st.M;
        a.ndm_out = int(t.ndm_out);
        a.pf_cap = st.pf_cap;
        a.s0 = ichunk * t.nt_ds;
        a.nt = t.nt_ds;
        a.beam0 = beam0;
        a.chunk_ctr = ctr;
        nb2[i] = int(st.nblocks);
    }
    // Consecutive output trees that use the same stage-2 kernel share one launch.
    for (long i0 = 0; i0 < plan.ntrees;) {
        long i1 = i0 + 1;
        while (tune.merge_stage2 && i1 < plan.ntrees && i1 - i0 < kStage2MaxTrees && stage2_same_kernel(a2[i0], a2[i1])) i1++;
        cudaEvent_t t3 = tk ? tick(3, nullptr, s) : nullptr;
        launch_stage2_multi(&a2[i0], &nb2[i0], int(i1 - i0), dtype_code, int(B), s);
        if (tk) tick(3, t3, s);
        i0 = i1;
    }

    // Output back-pressure: slot_out is reusable once every consumer released seq_id - nbatches_out.
    if (fences)
        for (long c = 0; c < params.num_consumers; c++)
            if (out_released_recorded[c][slot_out])
                CUDA_CHECK(cudaStreamWaitEvent(s, ev_out_released[c][slot_out], 0));

    for (long i = 0; i < plan.ntrees; i++) {
        const DedispersionTree &t = plan.trees[i];
        Stage2 &st = s2[i];
        PfArgs a;
        memset(&a, 0, sizeof(a));
        a.pf = st.pfring.ptr;
        a.pf_cap = st.pf_cap;
        size_t wsz = size_t(B) * t.ndm_wt * t.nt_wt * t.nprofiles * st.N;
        a.wt = st.wt.as<float>() + size_t(slot_wt) * wsz;
        size_t osz = size_t(B) * t.ndm_out * t.nt_out;
        a.out_max = st.out_max.as<char>() + size_t(slot_out) * osz * esize;
        a.out_argmax = st.out_argmax.as<uint32_t>() + size_t(slot_out) * osz;
        a.m_to_n = st.m_to_n.as<int>();
        a.M = st.M; a.N = st.N; a.P = st.P; a.L = st.L;
        a.ndm_out = int(t.ndm_out); a.nt_out = int(t.nt_out);
        a.ndm_wt = int(t.ndm_wt); a.nt_wt = int(t.nt_wt);
        a.Dout = st.Dout; a.Dcore = int(t.Dcore); a.tpad = st.tpad;
        a.s0 = ichunk * t.nt_ds;
        a.beam0 = beam0;
        a.chunk_ctr = ctr;
        a.nt_chunk = int(t.nt_ds);
        a.force_general = tune.pf_general ? 1 : 0;
        cudaEvent_t t4 = tk ? tick(4, nullptr, s) : nullptr;
        launch_pf(a, dtype_code, int(B), s);
        if (tk) tick(4, t4, s);
    }
    if (sift) {
        // Candidate stage: per-beam peak over the trees, patches of the peaks >= threshold, scores.
        cudaEvent_t t1 = tk ? tick(1, nullptr, s) : nullptr;
        float *cb = (float *) d_cand.ptr + size_t(slot_out) * 8 * B;
        BeamPeakArgs ba;
        memset(&ba, 0, sizeof(ba));
        ba.ntrees = int(plan.ntrees);
        for (long i = 0; i < plan.ntrees; i++) {
            const DedispersionTree &t = plan.trees[i];
            size_t osz = size_t(B) * t.ndm_out * t.nt_out;
            ba.ndm[i] = t.ndm_out;
            ba.nt[i] = t.nt_out;
            ba.out_max[i] = s2[i].out_max.as<char>() + size_t(slot_out) * osz * esize;
            ba.out_argmax[i] = s2[i].out_argmax.as<uint32_t>() + size_t(slot_out) * osz;
        }
        ba.peak = cb;
        ba.tree = (int *) (cb + B);
        ba.idm = (int *) (cb + 2 * B);
        ba.itime = (int *) (cb + 3 * B);
        ba.token = (uint32_t *) (cb + 4 * B);
        launch_beam_peaks_split(ba, dtype_code, B, d_peak_scratch.as<char>() + size_t(istream) * B * plan.ntrees * peak_split * 16,
                                peak_split, s);
        PatchArgs pa = patch_args;
        for (long i = 0; i < plan.ntrees; i++) {
            const DedispersionTree &t = plan.trees[i];
            pa.t[i].wt = s2[i].wt.as<float>() + size_t(slot_wt) * size_t(B) * t.ndm_wt * t.nt_wt * t.nprofiles * s2[i].N;
        }
        pa.peak = ba.peak; pa.tree = ba.tree; pa.idm = ba.idm; pa.itime = ba.itime; pa.token = ba.token;
        pa.valid = (int *) (cb + 5 * B);
        pa.ichunk = ichunk;
        pa.chunk_ctr = ctr;
        pa.beam0 = beam0;
        pa.patches = d_patches.as<uint16_t>() + size_t(slot_out) * B * kPatchLen;
        launch_patches(pa, dtype_code, s);
        float *logits = cb + 6 * B, *scores = cb + 7 * B;
        if (sifter) {
            // one forward pass at a time: the sifter's activations are shared by the compute streams
            if (sifter_recorded) CUDA_CHECK(cudaStreamWaitEvent(s, ev_sifter, 0));
            sifter->forward(pa.patches, B, logits, s);
            CUDA_CHECK(cudaEventRecord(ev_sifter, s));
            sifter_recorded = true;
            launch_mask_scores(logits, pa.valid, scores, int(B), s);
        } else {
            launch_mask_scores(ba.peak, pa.valid, scores, int(B), s);
        }
        if (tk) tick(1, t1, s);
    }
    if (fences) {
        CUDA_CHECK(cudaEventRecord(ev_out_done[slot_out], s));
        out_done_recorded[slot_out] = true;
    }
}

GpuDedisperser::Outputs GpuDedisperser::acquire_output(long consumer_id, long seq_id, cudaStream_t stream, bool sync)
{
    return entry([&]() -> Outputs {
        if (consumer_id < 0 || consumer_id >= params.num_consumers) throw runtime_error("GpuDedisperser::acquire_output(): bad consumer_id");
        if (seq_id != next_acq_out[consumer_id])
            throw runtime_error("GpuDedisperser::acquire_output(): expected seq_id=" + std::to_string(next_acq_out[consumer_id]) + ", got " + std::to_string(seq_id));
        if (seq_id >= next_rel_in) {
            // As pirate's blocking wait on its cdd2 event ring (src_lib/GpuDedisperser.cpp:932): wait on
            // the host, bounded, until another thread has launched seq_id.
            const long tmo = params.release_timeout_ms > 0 ? params.release_timeout_ms : 60000;
            if (!cv.wait_for(*cur_lock, std::chrono::milliseconds(tmo), [&] { return stopped || seq_id < next_rel_in; }))
                throw runtime_error("GpuDedisperser::acquire_output(): seq_id=" + std::to_string(seq_id) +
                                    " has not been launched within " + std::to_string(tmo) + " ms");
            if (stopped) throw runtime_error("GpuDedisperser: stopped while waiting for a launch");
        }
        if (params.synchronous && next_rel_out[consumer_id] != seq_id)
            throw runtime_error("GpuDedisperser::acquire_output(): synchronous consumer must release before acquiring the next batch");
        if (seq_id - next_rel_out[consumer_id] >= nbatches_out)
            throw runtime_error("GpuDedisperser::acquire_output(): too many unreleased output batches");
        long slot = seq_id % nbatches_out;
        if (sync) CUDA_CHECK(cudaEventSynchronize(ev_out_done[slot]));
        else CUDA_CHECK(cudaStreamWaitEvent(stream, ev_out_done[slot], 0));
        Outputs o;
        o.dtype = plan.dtype;
        o.nbeams = B;
        o.ichunk_zero_based = seq_id / nbatches;
        o.ichunk_fpga_based = o.ichunk_zero_based + params.initial_chunk;
        o.ibeam = (seq_id % nbatches) * B;
        for (long i = 0; i < plan.ntrees; i++) {
            const DedispersionTree &t = plan.trees[i];
            size_t osz = size_t(B) * t.ndm_out * t.nt_out;
            o.ndm_out.push_back(t.ndm_out);
            o.nt_out.push_back(t.nt_out);
            o.out_max.push_back(s2[i].out_max.as<char>() + size_t(slot) * osz * esize);
            o.out_argmax.push_back(s2[i].out_argmax.as<uint32_t>() + size_t(slot) * osz);
        }
        if (sift) {
            float *cb = (float *) d_cand.ptr + size_t(slot) * 8 * B;
            o.cand_peak = cb;
            o.cand_tree = (int *) (cb + B);
            o.cand_idm = (int *) (cb + 2 * B);
            o.cand_itime = (int *) (cb + 3 * B);
            o.cand_token = (uint32_t *) (cb + 4 * B);
            o.cand_valid = (int *) (cb + 5 * B);
            o.scores = cb + 7 * B;
            o.patches = d_patches.as<uint16_t>() + size_t(slot) * B * kPatchLen;
        }
        next_acq_out[consumer_id]++;
        return o;
    });
}

void GpuDedisperser::release_output(long consumer_id, long seq_id, cudaStream_t stream)
{
    entry([&]() {
        if (consumer_id < 0 || consumer_id >= params.num_consumers) throw runtime_error("GpuDedisperser::release_output(): bad consumer_id");
        if (seq_id != next_rel_out[consumer_id] || seq_id >= next_acq_out[consumer_id])
            throw runtime_error("GpuDedisperser::release_output(): expected seq_id=" + std::to_string(next_rel_out[consumer_id]) + ", got " + std::to_string(seq_id));
        long slot = seq_id % nbatches_out;
        CUDA_CHECK(cudaEventRecord(ev_out_released[consumer_id][slot], stream));
        out_released_recorded[consumer_id][slot] = true;
        next_rel_out[consumer_id]++;
        cv.notify_all();
    });
}

void GpuDedisperser::fill_all_weights(long itree, const float *host, long nelts)
{
    entry([&]() {
        if (!allocated) throw runtime_error("GpuDedisperser::fill_all_weights(): allocate() was not called");
        if (itree < 0 || itree >= plan.ntrees) throw runtime_error("GpuDedisperser::fill_all_weights(): itree out of range");
        const DedispersionTree &t = plan.trees[itree];
        long expect = nbatches_wt * B * t.ndm_wt * t.nt_wt * t.nprofiles * t.frequency_subbands.N;
        if (nelts != expect)
            throw runtime_error("GpuDedisperser::fill_all_weights(): expected " + std::to_string(expect) + " elements "
                                "(nbatches_wt, beams_per_batch, ndm_wt, nt_wt, nprofiles, N), got " + std::to_string(nelts));
        sync_compute();   // no launched batch may still read the weights
        CUDA_CHECK(cudaMemcpyAsync(s2[itree].wt.ptr, host, nelts * sizeof(float), cudaMemcpyHostToDevice, compute));
        CUDA_CHECK(cudaStreamSynchronize(compute));
    });
}

void GpuDedisperser::time(long niterations, double *rtb)
{
    const long seq0 = entry([&]() -> long {
        if (!allocated) throw runtime_error("GpuDedisperser::time(): allocate() was not called");
        if (!d_qdata.ptr) throw runtime_error("GpuDedisperser::time(): time_samples_per_chunk must be a multiple of 256");
        if (params.num_consumers != 1) throw runtime_error("GpuDedisperser::time(): needs num_consumers == 1");
        if (niterations <= 2 * nstreams)
            throw runtime_error("GpuDedisperser::time(): niterations must be > 2 * num_active_batches");
        if (!rtb) throw runtime_error("GpuDedisperser::time(): null output array");
        if (next_acq_in != next_rel_in || next_acq_out[0] != next_rel_in || next_rel_out[0] != next_rel_in)
            throw runtime_error("GpuDedisperser::time(): every launched batch must have been consumed first");
        return next_acq_in;
    });
    CUDA_CHECK(cudaSetDevice(params.cuda_device_id));
    const long S = nstreams, K = nstreams + 2;
    const size_t data_bytes = size_t(B) * plan.nfreq * (plan.nt_in / 2);
    const size_t so_bytes = size_t(B) * plan.nfreq * (plan.nt_in / 256) * 2 * sizeof(uint16_t);
    const double chunk_seconds = 1.0e-3 * plan.nt_in * plan.config.time_sample_ms;

    // Resources of the loop, released on every exit path.
    struct Res
    {
        std::vector<void *> host;
        cudaStream_t h2g = nullptr, tstream = nullptr;
        std::vector<cudaEvent_t> ev;
        ~Res()
        {
            if (h2g) cudaStreamSynchronize(h2g);
            if (tstream) cudaStreamSynchronize(tstream);
            for (void *p : host) cudaFreeHost(p);
            for (cudaEvent_t e : ev) cudaEventDestroy(e);
            if (h2g) cudaStreamDestroy(h2g);
            if (tstream) cudaStreamDestroy(tstream);
        }
    } r;
    CUDA_CHECK(cudaStreamCreateWithFlags(&r.h2g, cudaStreamNonBlocking));
    CUDA_CHECK(cudaStreamCreateWithFlags(&r.tstream, cudaStreamNonBlocking));
    r.ev.assign(K, nullptr);
    for (auto &e : r.ev) CUDA_CHECK(cudaEventCreate(&e));
    // One host copy of the raw data per compute stream, as pirate's multi_raw_cpu: seeded pseudo-random
    // nibbles (values -8..7, the missing-sample code among them), scale 0.5 and offset 0 per 256
    // samples. (Timing depends a little on the data: the peak finder does more work where maxima move.)
    uint64_t x = 0x9e3779b97f4a7c15ULL;
    for (long i = 0; i < S; i++) {
        void *d = nullptr, *so = nullptr;
        CUDA_CHECK(cudaHostAlloc(&d, data_bytes, cudaHostAllocDefault));
        r.host.push_back(d);
        CUDA_CHECK(cudaHostAlloc(&so, so_bytes, cudaHostAllocDefault));
        r.host.push_back(so);
        uint64_t *w = (uint64_t *) d;
        for (size_t j = 0; j < data_bytes / 8; j++) {
            x ^= x << 13; x ^= x >> 7; x ^= x << 17;
            w[j] = x;
        }
        uint16_t *h = (uint16_t *) so;
        for (size_t j = 0; j < so_bytes / 2; j += 2) { h[j] = 0x3800; h[j + 1] = 0; }   // fp16 0.5, 0
    }

    for (long i = 0; i < niterations; i++) {
        const long seq = seq0 + i;
        void *so = nullptr;
        void *data = acquire_input_int4(seq, r.h2g, &so);
        CUDA_CHECK(cudaMemcpyAsync(data, r.host[2 * (i % S)], data_bytes, cudaMemcpyHostToDevice, r.h2g));
        CUDA_CHECK(cudaMemcpyAsync(so, r.host[2 * (i % S) + 1], so_bytes, cudaMemcpyHostToDevice, r.h2g));
        release_input_and_launch_dd_kernels(seq, r.h2g);
        acquire_output(0, seq, r.tstream, false);
        release_output(0, seq, r.tstream);
        CUDA_CHECK(cudaEventRecord(r.ev[i % K], r.tstream));
        // Completion times lag the launches by S iterations, as pirate's KernelTimer.
        const long j = i - S;
        if (j >= 1) {
            CUDA_CHECK(cudaEventSynchronize(r.ev[j % K]));
            float ms = 0;
            CUDA_CHECK(cudaEventElapsedTime(&ms, r.ev[(j - 1) % K], r.ev[j % K]));
            rtb[j] = B * chunk_seconds / (1.0e-3 * ms);
        }
    }
    rtb[0] = 0.0;
    for (long j = std::max(1L, niterations - S); j < niterations; j++) {
        CUDA_CHECK(cudaEventSynchronize(r.ev[j % K]));
        float ms = 0;
        CUDA_CHECK(cudaEventElapsedTime(&ms, r.ev[(j - 1) % K], r.ev[j % K]));
        rtb[j] = B * chunk_seconds / (1.0e-3 * ms);
    }
}

// GpuDedisperser::fill_analytic_weights (src_lib/GpuDedisperser.cpp:1162-1238): one beam's weights
// per tree from the analytic variances, copied to every (weight batch, beam) slot on the compute stream.
void GpuDedisperser::fill_analytic_weights(const double *freq_variances, long nfreq)
{
    entry([&]() {
        if (!allocated) throw runtime_error("GpuDedisperser::fill_analytic_weights(): allocate() was not called");
        std::vector<std::vector<double>> var = pf_analytic_variances(plan, freq_variances, nfreq);
        sync_compute();   // no launched batch may still read the weights
        for (long itree = 0; itree < plan.ntrees; itree++) {
            std::vector<float> w = pf_weights_from_variances(plan.trees[itree], var[itree]);
            const size_t nb = w.size() * sizeof(float);
            char *dst = (char *) s2[itree].wt.ptr;
            for (long slot = 0; slot < nbatches_wt * B; slot++)
                CUDA_CHECK(cudaMemcpyAsync(dst + slot * nb, w.data(), nb, cudaMemcpyHostToDevice, compute));
            CUDA_CHECK(cudaStreamSynchronize(compute));
        }
    });
}

}  // namespace pb2
