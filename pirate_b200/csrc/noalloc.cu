// noalloc.cu -- single-chunk dedispersion that allocates no device memory.
//
// Some callers cannot call cudaMalloc. Examples are a real-time thread that must not stall on
// cudaMalloc's implicit device-wide synchronization, and code embedded in a host framework whose
// device-memory pool must see every allocation. pb2_dedisperse_chunk_noalloc() serves them: it
// dedisperses one chunk of beams_per_batch beams, as the first chunk of a fresh stream (zero
// history), through the same kernels as GpuDedisperser. All scratch (lookup tables, the gridded
// tree, the lagged-downsampling lines, the stage-1 delay lines, the tree states and the
// peak-finder lines) lives in the file-scope array g_noalloc_scratch below, of fixed size
// PB2_NOALLOC_SCRATCH_BYTES. Every GPU that loads the library holds that array until the process
// exits. Plans whose scratch does not fit are rejected with an error.
//
// The array is shared by all calls and keeps the last call's contents; each call clears it on its
// stream before use. Calls that overlap on the GPU (on different streams, or from different host
// threads) race on the array and give wrong results: serialize them.
//
// On the first call on a device, the address of the array on that device is looked up with
// cudaGetSymbolAddress() (with that device current) and cached. That first call should come
// before any stream capture. The stream must belong to the current device.
//
// Lookup tables. The plan's tables (channel weights, delay-line offsets) sit at the start of the
// array. A call uploads them only when its tables differ from the last ones uploaded on this device,
// i.e. on the first call and whenever the plan changes; the copy is then from pageable host memory,
// so that call may wait for earlier work on its stream. Calls that repeat the previous plan copy
// nothing from the host: they clear the rest of the array and launch the kernels.

#include "../../include/pirate_b200.h"
#include "kernels.cuh"
#include "plan.hpp"

#include <algorithm>
#include <cstring>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace pb2 {

static constexpr long kNoallocBytes = PB2_NOALLOC_SCRATCH_BYTES;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

#define NA_CHECK(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { \
    std::stringstream _ss; _ss << #x << ": " << cudaGetErrorString(_e); throw std::runtime_error(_ss.str()); } } while (0)

static long na_pow2_ceil(long n) { long p = 1; while (p < n) p <<= 1; return p; }
static long na_round_up(long n, long k) { return ((n + k - 1) / k) * k; }

static std::mutex g_noalloc_mtx;

// Scratch address of the current device (looked up once per device).
static unsigned char *noalloc_scratch(int dev)
{
    static std::vector<unsigned char *> addr;
    std::lock_guard<std::mutex> lk(g_noalloc_mtx);
    if ((int) addr.size() <= dev) addr.resize(dev + 1, nullptr);
    if (!addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            throw std::runtime_error(std::string("pb2_dedisperse_chunk_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        addr[dev] = (unsigned char *) p;
    }
    return addr[dev];
}

// Carves 256-byte aligned regions out of the scratch array.
struct Carver
{
    long used = 0;
    long take(long nbytes) { long o = used; used = na_round_up(used + std::max(nbytes, 1L), 256); return o; }
};

struct HostBlob
{
    std::vector<unsigned char> bytes;
    long put(const void *p, long n)
    {
        long o = na_round_up(long(bytes.size()), 256);
        bytes.resize(o + n);
        memcpy(bytes.data() + o, p, n);
        return o;
    }
};

void dedisperse_chunk_noalloc(const DedispersionPlan &plan, const void *in, const float *const *weights,
                              void *const *out_max, uint32_t *const *out_argmax, cudaStream_t stream)
{
    const long B = plan.beams_per_batch, rank = plan.config.toplevel_tree_rank, nt = plan.nt_in;
    const long F = plan.nfreq, N = pow2(rank), npri = plan.num_primary_trees;
    const int dtype_code = int(plan.dtype);
    const long es = (plan.dtype == Dtype::f32) ? 4 : 2;

    // Lookup tables, built on the host and copied into the scratch array.
    HostBlob tab;
    std::vector<double> cm = plan.config.make_channel_map();
    std::vector<int> f0(N), cnt(N), woff(N);
    std::vector<float> w;
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
    long t_f0 = tab.put(f0.data(), N * 4), t_cnt = tab.put(cnt.data(), N * 4), t_woff = tab.put(woff.data(), N * 4);
    long t_w = tab.put(w.data(), std::max<long>(w.size(), 1) * 4);

    struct S1 { long ring_off_t, ring_cap_t, ring, state, lds, lds_cap, ring_stride, state_pb; int rank, nblocks, nt; };
    struct S2 { long m2n_t, state, pf, pf_cap, state_pb; int M, N, P, L, tpad, Dout; int cnt[5], mb[5]; };
    std::vector<S1> s1(npri);
    std::vector<S2> s2(plan.ntrees);

    for (long p = 0; p < npri; p++) {
        int R1 = plan.stage1_dd_rank[p], A1 = plan.stage1_amb_rank[p];
        if (R1 < 1 || R1 > 8) throw std::runtime_error("pb2_dedisperse_chunk_noalloc: stage-1 dd rank must be in [1, 8]");
        S1 &st = s1[p];
        st.rank = R1;
        st.nblocks = 1 << A1;
        st.nt = int(nt >> p);
        long nrows = pow2(R1 + A1);
        std::vector<long> off(nrows);
        std::vector<int> cap(nrows);
        long tot = 0;
        for (long row = 0; row < nrows; row++) {
            // one sample more than the lags need: stage 2 also reads the sample before its first
            cap[row] = int(na_round_up(plan.max_row_lag[p][row] + st.nt + 1, 32));
            off[row] = tot;
            tot += cap[row];
        }
        st.ring_stride = tot;
        for (long blk = 0; blk < st.nblocks; blk++) {   // 32-bit offsets within a block's delay lines
            long end = (blk + 1 < st.nblocks) ? off[(blk + 1) * (1L << R1)] : tot;
            if (end - off[blk * (1L << R1)] >= (1L << 31))
                throw std::runtime_error("pb2_dedisperse_chunk_noalloc: stage-1 delay lines of one block exceed 2^31 samples");
        }
        st.ring_off_t = tab.put(off.data(), nrows * sizeof(long));
        st.ring_cap_t = tab.put(cap.data(), nrows * sizeof(int));
        st.state_pb = stage1_state_floats(R1);
        st.lds_cap = (p > 0) ? na_pow2_ceil(st.nt + (1L << R1) - 1) : 0;
    }
    for (long i = 0; i < plan.ntrees; i++) {
        const DedispersionTree &t = plan.trees[i];
        const FrequencySubbands &fs = t.frequency_subbands;
        if (t.dd_rank < 1 || t.dd_rank > 8) throw std::runtime_error("pb2_dedisperse_chunk_noalloc: stage-2 dd rank must be in [1, 8]");
        if (fs.pf_rank != split_rb(t.dd_rank) || fs.pf_rank < 0 || fs.pf_rank >= 5)
            throw std::runtime_error("pb2_dedisperse_chunk_noalloc: unexpected peak-finding rank");
        S2 &st = s2[i];
        st.M = int(fs.M);
        st.N = int(fs.N);
        st.P = int(t.nprofiles);
        st.L = std::max(integer_log2(t.pf.max_width), 1);
        st.tpad = int(std::max(2 * t.pf.max_width, 4L));
        st.Dout = int(t.pf.time_downsampling);
        st.state_pb = stage2_state_floats(t.dd_rank);
        int mb = 0;
        for (int l = 0; l < 5; l++) { st.cnt[l] = 0; st.mb[l] = 0; }
        for (int l = 0; l <= fs.pf_rank; l++) { st.cnt[l] = int(fs.subband_counts[l]); st.mb[l] = mb; mb += int(fs.subband_counts[l]) << l; }
        if (mb != st.M) throw std::runtime_error("pb2_dedisperse_chunk_noalloc: multiplet count mismatch");
        std::vector<int> m2n(st.M);
        for (int m = 0; m < st.M; m++) m2n[m] = int(fs.m_to_n[m]);
        st.m2n_t = tab.put(m2n.data(), st.M * sizeof(int));
        st.pf_cap = na_pow2_ceil(t.nt_ds + st.tpad + st.Dout);
    }
    // Layout: [tables | cleared scratch]. Tables are rewritten by every call; the rest is zeroed.
    Carver cv;
    const long tab_at = cv.take(long(tab.bytes.size()));
    const long zero_from = cv.used;
    long tree0 = cv.take(B * N * nt * es);
    long lds_state = cv.take(npri > 1 ? 2 * B * (npri - 1) * (N / 2) * 4 : 0);
    for (long p = 0; p < npri; p++) {
        S1 &st = s1[p];
        st.ring = cv.take(B * st.ring_stride * es);
        st.state = cv.take(B * st.nblocks * st.state_pb * 4);
        st.lds = (p > 0) ? cv.take(B * (N / 2) * st.lds_cap * es) : 0;
    }
    for (long i = 0; i < plan.ntrees; i++) {
        const DedispersionTree &t = plan.trees[i];
        S2 &st = s2[i];
        st.state = cv.take(B * (1L << t.amb_rank) * st.state_pb * 4);
        st.pf = cv.take(B * t.ndm_out * st.M * st.pf_cap * es);
    }
    if (cv.used > kNoallocBytes) {
        std::stringstream ss;
        ss << "pb2_dedisperse_chunk_noalloc: this plan needs " << cv.used << " bytes of scratch, more than the "
           << kNoallocBytes << " bytes (PB2_NOALLOC_SCRATCH_BYTES) of the static scratch array";
        throw std::runtime_error(ss.str());
    }

    int dev = 0;
    NA_CHECK(cudaGetDevice(&dev));
    if (stream) {
        int sdev = -1;
        NA_CHECK(cudaStreamGetDevice(stream, &sdev));
        if (sdev != dev)
            throw std::runtime_error("pb2_dedisperse_chunk_noalloc: the stream belongs to another device than the current one");
    }
    unsigned char *base = noalloc_scratch(dev);
    {
        // Upload the tables only if they differ from the last ones uploaded on this device.
        static std::vector<std::vector<unsigned char>> last;
        std::lock_guard<std::mutex> lk(g_noalloc_mtx);
        if ((int) last.size() <= dev) last.resize(dev + 1);
        if (last[dev] != tab.bytes) {
            last[dev].clear();   // a failed upload leaves no stale record
            NA_CHECK(cudaMemcpyAsync(base + tab_at, tab.bytes.data(), tab.bytes.size(), cudaMemcpyHostToDevice, stream));
            last[dev] = tab.bytes;
        }
    }
    NA_CHECK(cudaMemsetAsync(base + zero_from, 0, cv.used - zero_from, stream));
    auto T = [&](long o) { return base + tab_at + o; };
    auto P = [&](long o) { return base + o; };

    GridLdsArgs g;
    memset(&g, 0, sizeof(g));
    g.in = in;
    g.tree0 = P(tree0);
    g.chan_f0 = (const int *) T(t_f0);
    g.chan_cnt = (const int *) T(t_cnt);
    g.chan_woff = (const int *) T(t_woff);
    g.chan_w = (const float *) T(t_w);
    g.F = int(F); g.rank = int(rank); g.T = int(nt); g.nlev = int(npri - 1);
    for (long p = 1; p < npri; p++) { g.ring[p - 1] = P(s1[p].lds); g.cap_mask[p - 1] = s1[p].lds_cap - 1; }
    g.state = (float *) P(lds_state);
    g.lag_rank = (npri > 1) ? int(plan.stage1_dd_rank[1]) : 0;
    g.ichunk = 0;
    g.beam0 = 0; g.B = int(B); g.total_beams = int(B);
    launch_grid_lds(g, dtype_code, stream);

    for (long p = 0; p < npri; p++) {
        S1 &st = s1[p];
        Stage1Args a;
        memset(&a, 0, sizeof(a));
        a.rank = st.rank;
        a.state_per_block = st.state_pb;
        a.state = (float *) P(st.state);
        if (p == 0) {
            a.in = P(tree0); a.in_beam_stride = N * nt; a.in_row_stride = nt; a.in_mask = -1;
        } else {
            a.in = P(st.lds); a.in_beam_stride = (N / 2) * st.lds_cap; a.in_row_stride = st.lds_cap;
            a.in_mask = st.lds_cap - 1; a.in_s0 = 0;
        }
        a.ring = P(st.ring);
        a.ring_off = (const long *) T(st.ring_off_t);
        a.ring_cap = (const int *) T(st.ring_cap_t);
        a.ring_beam_stride = st.ring_stride;
        a.s0 = 0; a.nt = st.nt; a.beam0 = 0;
        launch_stage1(a, dtype_code, st.nblocks, int(B), stream);
    }

    for (long i = 0; i < plan.ntrees; i++) {
        const DedispersionTree &t = plan.trees[i];
        S2 &st = s2[i];
        S1 &src = s1[t.primary_tree_index];
        Stage2Args a;
        memset(&a, 0, sizeof(a));
        a.rank = t.dd_rank;
        a.state_per_block = st.state_pb;
        a.state = (float *) P(st.state);
        a.ring = P(src.ring);
        a.ring_off = (const long *) T(src.ring_off_t);
        a.ring_cap = (const int *) T(src.ring_cap_t);
        a.ring_beam_stride = src.ring_stride;
        a.amb_rank = t.amb_rank;
        a.uflag = (t.primary_tree_index > 0) ? 1 : 0;
        for (int l = 0; l < 5; l++) { a.sb_count[l] = st.cnt[l]; a.sb_mbase[l] = st.mb[l]; }
        a.pf = P(st.pf);
        a.M = st.M;
        a.ndm_out = int(t.ndm_out);
        a.pf_cap = st.pf_cap;
        a.s0 = 0; a.nt = t.nt_ds; a.beam0 = 0;
        launch_stage2(a, dtype_code, 1 << t.amb_rank, int(B), stream);

        PfArgs f;
        memset(&f, 0, sizeof(f));
        f.pf = P(st.pf);
        f.pf_cap = st.pf_cap;
        f.wt = weights[i];
        f.out_max = out_max[i];
        f.out_argmax = out_argmax[i];
        f.m_to_n = (const int *) T(st.m2n_t);
        f.M = st.M; f.N = st.N; f.P = st.P; f.L = st.L;
        f.ndm_out = int(t.ndm_out); f.nt_out = int(t.nt_out);
        f.ndm_wt = int(t.ndm_wt); f.nt_wt = int(t.nt_wt);
        f.Dout = st.Dout; f.Dcore = int(t.Dcore); f.tpad = st.tpad;
        f.s0 = 0; f.beam0 = 0;
        launch_pf(f, dtype_code, int(B), stream);
    }
}

}  // namespace pb2
