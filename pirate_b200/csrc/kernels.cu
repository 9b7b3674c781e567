// kernels.cu -- sm_100a kernels of the B200 dedispersion path.
//
//   grid_kernel    tree gridding                 (replaces GpuTreeGriddingKernel, src_lib/TreeGriddingKernel.cu:108-279)
//   lds_kernel     lagged downsampling           (replaces GpuLaggedDownsamplingKernel, src_lib/GpuLaggedDownsamplingKernel.cu:668-918)
//   stage1_kernel  stage-1 tree -> delay lines   (replaces GpuDedispersionKernel outrb, src_lib/DedispersionKernel.cu:492-653)
//   stage2_kernel  delay lines -> stage-2 tree
//                  with subband outputs          (replaces the dd half of CoalescedDdKernel2, src_lib/CoalescedDdKernel2.cu:79-269)
//   pf_kernel      peak finding, max/argmax      (replaces the pf half of CoalescedDdKernel2 / GpuPeakFindingKernel)
//
// All arithmetic is fp32 in registers with explicit round-to-nearest intrinsics (no FMA contraction),
// performing the same sequence of fp32 operations as the reference CPU dedisperser, so that a float32
// plan reproduces its outputs bit for bit. Storage (inputs, tree intermediates, delay lines,
// out_max) is float32, float16 or bfloat16.

#include "kernels.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdexcept>
#include <string>

namespace pb2 {

constexpr float kRsqrt2 = 0.7071067811865476f;

template<typename T> __device__ __forceinline__ float to_f(T x);
template<> __device__ __forceinline__ float to_f<float>(float x) { return x; }
template<> __device__ __forceinline__ float to_f<__half>(__half x) { return __half2float(x); }
template<> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }

template<typename T> __device__ __forceinline__ T from_f(float x);
template<> __device__ __forceinline__ float from_f<float>(float x) { return x; }
template<> __device__ __forceinline__ __half from_f<__half>(float x) { return __float2half_rn(x); }
template<> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }

__device__ __forceinline__ float bfly(float x, float y) { return __fmul_rn(kRsqrt2, __fadd_rn(x, y)); }

__device__ __forceinline__ int brev_bits(int x, int nbits) { return nbits ? int(__brev(unsigned(x)) >> (32 - nbits)) : 0; }

static void check_launch(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}


// -------------------------------------------------------------------------------------------------
// Tree gridding: out[b,n,t] = sum_f w[n,f] in[b,f,t], summed in ascending f from zero.
// One warp per tree channel, 4 consecutive samples per lane.


template<typename Ts>
__global__ void __launch_bounds__(256) grid_kernel(GridArgs a)
{
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int n = blockIdx.y * 8 + warp;
    int t = (blockIdx.x * 32 + lane) * 4;
    int b = blockIdx.z;
    if (n >= a.N || t >= a.T)
        return;

    const Ts *in = (const Ts *) a.in + (long) b * a.F * a.T + t;
    int f0 = a.chan_f0[n], cnt = a.chan_cnt[n], woff = a.chan_woff[n];
    float acc0 = 0.0f, acc1 = 0.0f, acc2 = 0.0f, acc3 = 0.0f;

    for (int k = 0; k < cnt; k++) {
        float w = a.chan_w[woff + k];
        const Ts *p = in + (long) (f0 + k) * a.T;
        float x0, x1, x2, x3;
        if constexpr (sizeof(Ts) == 4) {
            float4 v = *(const float4 *) p;
            x0 = v.x; x1 = v.y; x2 = v.z; x3 = v.w;
        } else {
            uint2 v = *(const uint2 *) p;
            const Ts *h = (const Ts *) &v;
            x0 = to_f(h[0]); x1 = to_f(h[1]); x2 = to_f(h[2]); x3 = to_f(h[3]);
        }
        acc0 = __fadd_rn(acc0, __fmul_rn(w, x0));
        acc1 = __fadd_rn(acc1, __fmul_rn(w, x1));
        acc2 = __fadd_rn(acc2, __fmul_rn(w, x2));
        acc3 = __fadd_rn(acc3, __fmul_rn(w, x3));
    }

    Ts *out = (Ts *) a.out + ((long) b * a.N + n) * a.T + t;
    if constexpr (sizeof(Ts) == 4) {
        *(float4 *) out = make_float4(acc0, acc1, acc2, acc3);
    } else {
        uint2 v;
        Ts *h = (Ts *) &v;
        h[0] = from_f<Ts>(acc0); h[1] = from_f<Ts>(acc1); h[2] = from_f<Ts>(acc2); h[3] = from_f<Ts>(acc3);
        *(uint2 *) out = v;
    }
}


// -------------------------------------------------------------------------------------------------
// Lagged downsampling. For each level p = 1..nlev:
//   ds_p[ch][u]  = (ds_{p-1}[ch][2u] + ds_{p-1}[ch][2u+1]) / sqrt2          (ds_0 = level-0 tree)
//   out_p[c][u]  = (ds_p[2c][u-1] + ds_p[2c+1][u]) / sqrt2                     (one-sample lag on even channels)
// out_p goes to a per-row delay line; the per-row "large" lag is applied by the stage-1 reader.
// Each thread owns one output row c and a window of W0 level-0 samples.


template<typename Ts, int NLEV>
__global__ void __launch_bounds__(128) lds_kernel(LdsArgs a)
{
    constexpr int W0 = ((1 << NLEV) > 8) ? (1 << NLEV) : 8;
    constexpr int WE = 1 << NLEV;           // level-0 samples feeding one level-NLEV sample

    long nhalf = 1L << (a.rank - 1);
    long nwin = a.T / W0;
    long g = (long) blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nwin * nhalf * a.B)
        return;
    int win = int(g % nwin);
    long c = (g / nwin) % nhalf;
    int b = int(g / (nwin * nhalf));
    int bt = a.beam0 + b;
    int parity = int(a.ichunk & 1);

    const Ts *row0 = (const Ts *) a.in + ((long) b * (2 * nhalf) + 2 * c) * a.T;
    const Ts *row1 = row0 + a.T;
    long t0 = (long) win * W0;

    float r0[W0], r1[W0], e[WE];
#pragma unroll
    for (int i = 0; i < W0; i++) {
        r0[i] = to_f(row0[t0 + i]);
        r1[i] = to_f(row1[t0 + i]);
    }
    if (win > 0) {
#pragma unroll
        for (int i = 0; i < WE; i++)
            e[i] = to_f(row0[t0 - WE + i]);
    }

#pragma unroll
    for (int p = 1; p <= NLEV; p++) {
        constexpr int dummy = 0; (void) dummy;
        const int len = W0 >> p;
        const int elen = WE >> p;
#pragma unroll
        for (int u = 0; u < (W0 >> 1); u++) {
            if (u < len) {
                r0[u] = bfly(r0[2 * u], r0[2 * u + 1]);
                r1[u] = bfly(r1[2 * u], r1[2 * u + 1]);
            }
        }
        float prev;
        if (win > 0) {
#pragma unroll
            for (int u = 0; u < (WE >> 1); u++)
                if (u < elen) e[u] = bfly(e[2 * u], e[2 * u + 1]);
            prev = e[elen - 1];
        } else {
            prev = a.state[(((long) parity * a.total_beams + bt) * a.nlev + (p - 1)) * nhalf + c];
        }

        long cap = a.cap_mask[p - 1] + 1;
        Ts *ring = (Ts *) a.ring[p - 1] + ((long) bt * nhalf + c) * cap;
        long nt_p = a.T >> p;
        long s_base = a.ichunk * nt_p + (long) win * len;
#pragma unroll
        for (int u = 0; u < (W0 >> 1); u++) {
            if (u < len) {
                float lagged = (u == 0) ? prev : r0[u - 1];
                ring[(s_base + u) & a.cap_mask[p - 1]] = from_f<Ts>(bfly(lagged, r1[u]));
            }
        }
        if (win == nwin - 1)
            a.state[(((long) (1 - parity) * a.total_beams + bt) * a.nlev + (p - 1)) * nhalf + c] = r0[len - 1];
    }
}


// -------------------------------------------------------------------------------------------------
// Tree programs (see TreeOp in kernels.cuh). 'cur' holds the tile (nrows x kTreeTile) at the start
// of each phase; butterflies write the next state into 'nxt'. Returns the buffer holding the result.


template<typename OutF>
__device__ __forceinline__ float *run_program(float *cur, float *nxt, const TreeOp *__restrict__ ops,
                                              const int *__restrict__ phase_begin, int nphases, int nsteps,
                                              float *__restrict__ hist, long s_tile, OutF out)
{
    constexpr int TT = kTreeTile;
    const int tid = threadIdx.x, nthr = blockDim.x;

    for (int ph = 0; ph < nphases; ph++) {
        int ob = phase_begin[ph], oe = phase_begin[ph + 1];
        int nitems = (oe - ob) * TT;

        for (int it = tid; it < nitems; it += nthr) {
            const TreeOp op = ops[ob + it / TT];
            int t = it % TT;
            if (op.kind == 2) {
                out(op.out0, t, cur[op.row0 * TT + t]);
                continue;
            }
            float y = cur[op.row1 * TT + t];
            int ta = t - op.lag, tb = ta - 1;
            float xa = (ta >= 0) ? cur[op.row0 * TT + ta] : hist[op.hist_off + ((s_tile + ta) & op.hist_mask)];
            float xb = (tb >= 0) ? cur[op.row0 * TT + tb] : hist[op.hist_off + ((s_tile + tb) & op.hist_mask)];
            float o0 = bfly(xa, y);
            float o1 = bfly(xb, y);
            if (op.kind == 0) {
                nxt[op.row0 * TT + t] = o0;
                nxt[op.row1 * TT + t] = o1;
            }
            if (op.out0 >= 0) out(op.out0, t, o0);
            if (op.out1 >= 0) out(op.out1, t, o1);
        }
        __syncthreads();

        // Save the newest samples of each butterfly's row0 input for the following tiles.
        for (int it = tid; it < nitems; it += nthr) {
            const TreeOp op = ops[ob + it / TT];
            int t = it % TT;
            if (op.kind == 2) continue;
            if (t >= TT - (op.hist_mask + 1))
                hist[op.hist_off + ((s_tile + t) & op.hist_mask)] = cur[op.row0 * TT + t];
        }
        __syncthreads();

        if (ph < nsteps) {
            float *tmp = cur; cur = nxt; nxt = tmp;
        }
    }
    return cur;
}


struct NoOut { __device__ void operator()(int, int, float) const { } };


template<typename Ts>
__global__ void __launch_bounds__(kTreeThreads) stage1_kernel(Stage1Args a)
{
    constexpr int TT = kTreeTile;
    extern __shared__ float sm[];
    const int nrows = a.nrows, tid = threadIdx.x, nthr = blockDim.x;
    float *bufA = sm, *bufB = sm + nrows * TT;
    int *rowpos = (int *) (bufB + nrows * TT);

    const int blk = blockIdx.x, b = blockIdx.y, bt = a.beam0 + b;
    float *hist = a.hist + ((long) bt * gridDim.x + blk) * a.hist_per_block;
    const Ts *in = (const Ts *) a.in + (long) (a.in_beam0 + b) * a.in_beam_stride;
    Ts *ring = (Ts *) a.ring + (long) bt * a.ring_beam_stride;

    for (int n = tid; n < nrows; n += nthr)
        rowpos[n] = int(a.s0 % (long) a.ring_cap[blk * nrows + n]);
    __syncthreads();

    const int ntiles = a.nt / TT;
    for (int tile = 0; tile < ntiles; tile++) {
        long s_tile = a.s0 + (long) tile * TT;
        long s_in = a.in_s0 + (long) tile * TT;

        for (int it = tid; it < nrows * TT; it += nthr) {
            int n = it / TT, t = it % TT;
            long c = (long) blk * nrows + n;
            int lag = a.in_lag0 - a.in_lag1 * n;
            bufA[it] = to_f(in[c * a.in_row_stride + ((s_in + t - lag) & a.in_mask)]);
        }
        __syncthreads();

        float *res = run_program(bufA, bufB, a.ops, a.phase_begin, a.nphases, a.nphases, hist, s_tile, NoOut());

        for (int it = tid; it < nrows * TT; it += nthr) {
            int n = it / TT, t = it % TT;
            int row = blk * nrows + n;
            int cap = a.ring_cap[row];
            int p = rowpos[n] + t;
            if (p >= cap) p -= cap;
            ring[a.ring_off[row] + p] = from_f<Ts>(res[it]);
        }
        __syncthreads();

        for (int n = tid; n < nrows; n += nthr) {
            int cap = a.ring_cap[blk * nrows + n];
            int p = rowpos[n] + TT;
            rowpos[n] = (p >= cap) ? (p - cap) : p;
        }
        __syncthreads();
    }
}


template<typename Ts>
struct PfRingOut
{
    Ts *pf;
    long rowbase, cap_mask, s_tile, cap;
    __device__ void operator()(int o, int t, float v) const
    {
        pf[(rowbase + o) * cap + ((s_tile + t) & cap_mask)] = from_f<Ts>(v);
    }
};


template<typename Ts>
__global__ void __launch_bounds__(kTreeThreads) stage2_kernel(Stage2Args a)
{
    constexpr int TT = kTreeTile;
    extern __shared__ float sm[];
    const int nrows = a.nrows, tid = threadIdx.x, nthr = blockDim.x;
    float *bufA = sm, *bufB = sm + nrows * TT;
    int *rowpos = (int *) (bufB + nrows * TT);

    const int d = blockIdx.x, b = blockIdx.y, bt = a.beam0 + b;
    float *hist = a.hist + ((long) bt * gridDim.x + d) * a.hist_per_block;
    const Ts *ring = (const Ts *) a.ring + (long) bt * a.ring_beam_stride;

    const long dm = brev_bits(d, a.amb_rank) + (a.uflag ? (1L << a.amb_rank) : 0L);
    for (int r = tid; r < nrows; r += nthr) {
        long lag = (long) (nrows - 1 - r) * dm;
        long cap = a.ring_cap[(long) r * (1L << a.amb_rank) + d];
        long p = (a.s0 - lag) % cap;
        rowpos[r] = int(p < 0 ? p + cap : p);
    }
    __syncthreads();

    PfRingOut<Ts> out;
    out.pf = (Ts *) a.pf;
    out.rowbase = ((long) bt * a.ndm_out + ((long) brev_bits(d, a.amb_rank) << a.pf_shift)) * a.M;
    out.cap = a.pf_cap;
    out.cap_mask = a.pf_cap - 1;

    const int ntiles = a.nt / TT;
    for (int tile = 0; tile < ntiles; tile++) {
        long s_tile = a.s0 + (long) tile * TT;
        out.s_tile = s_tile;

        for (int it = tid; it < nrows * TT; it += nthr) {
            int r = it / TT, t = it % TT;
            long row = (long) r * (1L << a.amb_rank) + d;
            int cap = a.ring_cap[row];
            int p = rowpos[r] + t;
            if (p >= cap) p -= cap;
            bufA[it] = to_f(ring[a.ring_off[row] + p]);
        }
        __syncthreads();

        run_program(bufA, bufB, a.ops, a.phase_begin, a.nphases, a.dd_rank, hist, s_tile, out);

        for (int r = tid; r < nrows; r += nthr) {
            int cap = a.ring_cap[(long) r * (1L << a.amb_rank) + d];
            int p = rowpos[r] + TT;
            rowpos[r] = (p >= cap) ? (p - cap) : p;
        }
        __syncthreads();
    }
}


// -------------------------------------------------------------------------------------------------
// Peak finding. One warp per (beam, coarse dm, 32 consecutive output times). For each multiplet m
// the warp stages the input window in shared memory and builds the boxcar levels with the reference's
// recursion  B_{l+1}[u] = B_l[r u] + B_l[r u + s]  (so every boxcar sum has the reference's rounding);
// each lane then scans the trials of its output time. The running maximum breaks ties by the
// reference's scan order (level, multiplet, fine time, profile), reproducing its out_argmax tokens.


constexpr int kPfWarps = 4;
constexpr int kPfMaxLevels = 6;

struct PfLevels
{
    int L;
    int dt[kPfMaxLevels], n[kPfMaxLevels], off[kPfMaxLevels], r[kPfMaxLevels], s[kPfMaxLevels];
    int total;
};

__device__ __forceinline__ void pf_levels(const PfArgs &a, int len0, PfLevels &lv)
{
    lv.L = a.L;
    int off = 0;
    for (int l = 0; l < a.L; l++) {
        int dt = min(a.Dcore, 1 << l);
        lv.dt[l] = dt;
        lv.n[l] = (len0 - (1 << l)) / dt + 1;
        lv.off[l] = off;
        off += lv.n[l];
    }
    for (int l = 0; l + 1 < a.L; l++) {
        lv.r[l] = lv.dt[l + 1] / lv.dt[l];
        lv.s[l] = (1 << l) / lv.dt[l];
    }
    lv.total = off;
}

struct PfBest
{
    float v;
    int key;
    uint32_t tok;
    __device__ __forceinline__ void update(float val, int k, uint32_t t)
    {
        if ((val > v) || (val == v && k < key)) { v = val; key = k; tok = t; }
    }
};

template<typename Ts>
__global__ void __launch_bounds__(kPfWarps * 32) pf_kernel(PfArgs a, int warp_floats)
{
    extern __shared__ float sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int dm = blockIdx.y * kPfWarps + warp;
    const int b = blockIdx.z, bt = a.beam0 + b;
    const int tout0 = blockIdx.x * 32;
    if (dm >= a.ndm_out)
        return;   // whole warp exits; warps never synchronize across the block

    const int ntw = min(32, a.nt_out - tout0);
    const int R0 = tout0 * a.Dout - a.tpad;
    const int len0 = ntw * a.Dout + a.tpad;
    float *lev = sm + warp * warp_floats;

    PfLevels lv;
    pf_levels(a, len0, lv);

    const int tout = tout0 + lane;
    const bool active = (lane < ntw);
    const int pf_dm = dm & ((1 << a.pf_shift) - 1);
    const int Wds = a.ndm_out / a.ndm_wt, Tds = a.nt_out / a.nt_wt;
    const float *wp = a.wt + ((((long) b * a.ndm_wt + dm / Wds) * a.nt_wt + (active ? tout / Tds : 0)) * a.P) * a.N;
    const Ts *pfrows = (const Ts *) a.pf + ((long) bt * a.ndm_out + dm) * a.M * a.pf_cap;
    const long mask = a.pf_cap - 1;

    PfBest best;
    best.v = -1.0e30f;
    best.key = -1;
    best.tok = 0xffffffffu;

    for (int m = 0; m < a.M; m++) {
        const Ts *row = pfrows + (long) m * a.pf_cap;
        long s_base = a.s0 + R0 - a.final_lag[pf_dm * a.M + m];
        for (int u = lane; u < len0; u += 32)
            lev[u] = to_f(row[(s_base + u) & mask]);
        __syncwarp();
        for (int l = 0; l + 1 < lv.L; l++) {
            const float *src = lev + lv.off[l];
            float *dst = lev + lv.off[l + 1];
            int rr = lv.r[l], ss = lv.s[l];
            for (int u = lane; u < lv.n[l + 1]; u += 32)
                dst[u] = __fadd_rn(src[rr * u], src[rr * u + ss]);
            __syncwarp();
        }

        if (active) {
            int n = a.m_to_n[m];
            for (int l = 0; l < lv.L; l++) {
                const int dt = lv.dt[l], S = (1 << l) / dt, nsamp = a.Dout / dt;
                const int I = (a.tpad + dt - (1 << l)) / dt;
                const float *x = lev + lv.off[l] + I + lane * nsamp;
                float w0 = (l == 0) ? wp[n] : 0.0f;
                float w1 = 0.0f, w2 = 0.0f, w3 = 0.0f;
                if (a.P > 1) {
                    w1 = wp[(3 * l + 1) * a.N + n];
                    w2 = wp[(3 * l + 2) * a.N + n];
                    w3 = wp[(3 * l + 3) * a.N + n];
                }
                const int kbase = (l * a.M + m) * 64;
                for (int is = 0; is < nsamp; is++) {
                    float x0 = x[is - 3 * S], x1 = x[is - 2 * S], x2 = x[is - S], x3 = x[is];
                    uint32_t tk0 = (uint32_t(m) << 16) | uint32_t(is * dt);
                    int k = (kbase + is) * 4;
                    if (l == 0)
                        best.update(__fmul_rn(w0, x3), k, tk0);
                    if (a.P > 1) {
                        float y1 = __fadd_rn(x2, x3);
                        float y2 = __fadd_rn(__fadd_rn(__fmul_rn(0.5f, x1), x2), __fmul_rn(0.5f, x3));
                        float y3 = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(0.5f, x0), x1), x2), __fmul_rn(0.5f, x3));
                        best.update(__fmul_rn(w1, y1), k + 1, tk0 | (uint32_t(3 * l + 1) << 8));
                        best.update(__fmul_rn(w2, y2), k + 2, tk0 | (uint32_t(3 * l + 2) << 8));
                        best.update(__fmul_rn(w3, y3), k + 3, tk0 | (uint32_t(3 * l + 3) << 8));
                    }
                }
            }
        }
        __syncwarp();
    }

    if (active) {
        long o = ((long) b * a.ndm_out + dm) * a.nt_out + tout;
        ((Ts *) a.out_max)[o] = from_f<Ts>(best.v);
        a.out_argmax[o] = best.tok;
    }
}


// -------------------------------------------------------------------------------------------------
// Host launchers.


template<typename Ts>
static void launch_grid_t(const GridArgs &a, int B, cudaStream_t s)
{
    dim3 grid((a.T / 4 + 31) / 32, (a.N + 7) / 8, B);
    grid_kernel<Ts><<<grid, 256, 0, s>>>(a);
    check_launch("grid_kernel");
}

void launch_grid(const GridArgs &a, int dtype, int B, cudaStream_t s)
{
    if (dtype == 0) launch_grid_t<float>(a, B, s);
    else if (dtype == 1) launch_grid_t<__half>(a, B, s);
    else launch_grid_t<__nv_bfloat16>(a, B, s);
}

template<typename Ts, int NLEV>
static void launch_lds_t(const LdsArgs &a, cudaStream_t s)
{
    constexpr int W0 = ((1 << NLEV) > 8) ? (1 << NLEV) : 8;
    if (a.T % W0) throw std::runtime_error("lds_kernel: chunk length not a multiple of the window");
    long nthr = (long) (a.T / W0) * (1L << (a.rank - 1)) * a.B;
    lds_kernel<Ts, NLEV><<<(unsigned) ((nthr + 127) / 128), 128, 0, s>>>(a);
    check_launch("lds_kernel");
}

template<typename Ts>
static void launch_lds_d(const LdsArgs &a, cudaStream_t s)
{
    switch (a.nlev) {
    case 1: launch_lds_t<Ts, 1>(a, s); break;
    case 2: launch_lds_t<Ts, 2>(a, s); break;
    case 3: launch_lds_t<Ts, 3>(a, s); break;
    case 4: launch_lds_t<Ts, 4>(a, s); break;
    case 5: launch_lds_t<Ts, 5>(a, s); break;
    case 6: launch_lds_t<Ts, 6>(a, s); break;
    default: throw std::runtime_error("lds_kernel: unsupported number of levels");
    }
}

void launch_lds(const LdsArgs &a, int dtype, cudaStream_t s)
{
    if (dtype == 0) launch_lds_d<float>(a, s);
    else if (dtype == 1) launch_lds_d<__half>(a, s);
    else launch_lds_d<__nv_bfloat16>(a, s);
}

static size_t tree_smem(int nrows) { return (size_t) 2 * nrows * kTreeTile * sizeof(float) + nrows * sizeof(int); }

template<typename K>
static void set_smem(K kernel, size_t bytes)
{
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bytes);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
}

template<typename Ts>
static void launch_stage1_t(const Stage1Args &a, int nblocks, int B, cudaStream_t s)
{
    size_t sm = tree_smem(a.nrows);
    set_smem(stage1_kernel<Ts>, sm);
    stage1_kernel<Ts><<<dim3(nblocks, B), kTreeThreads, sm, s>>>(a);
    check_launch("stage1_kernel");
}

void launch_stage1(const Stage1Args &a, int dtype, int nblocks, int B, cudaStream_t s)
{
    if (dtype == 0) launch_stage1_t<float>(a, nblocks, B, s);
    else if (dtype == 1) launch_stage1_t<__half>(a, nblocks, B, s);
    else launch_stage1_t<__nv_bfloat16>(a, nblocks, B, s);
}

template<typename Ts>
static void launch_stage2_t(const Stage2Args &a, int nblocks, int B, cudaStream_t s)
{
    size_t sm = tree_smem(a.nrows);
    set_smem(stage2_kernel<Ts>, sm);
    stage2_kernel<Ts><<<dim3(nblocks, B), kTreeThreads, sm, s>>>(a);
    check_launch("stage2_kernel");
}

void launch_stage2(const Stage2Args &a, int dtype, int nblocks, int B, cudaStream_t s)
{
    if (dtype == 0) launch_stage2_t<float>(a, nblocks, B, s);
    else if (dtype == 1) launch_stage2_t<__half>(a, nblocks, B, s);
    else launch_stage2_t<__nv_bfloat16>(a, nblocks, B, s);
}

int pf_warp_floats(int Dout, int tpad, int Dcore, int L)
{
    int len0 = 32 * Dout + tpad, tot = 0;
    for (int l = 0; l < L; l++) {
        int dt = (Dcore < (1 << l)) ? Dcore : (1 << l);
        tot += (len0 - (1 << l)) / dt + 1;
    }
    return tot;
}

template<typename Ts>
static void launch_pf_t(const PfArgs &a, int B, cudaStream_t s)
{
    int wf = pf_warp_floats(a.Dout, a.tpad, a.Dcore, a.L);
    size_t sm = (size_t) kPfWarps * wf * sizeof(float);
    set_smem(pf_kernel<Ts>, sm);
    dim3 grid((a.nt_out + 31) / 32, (a.ndm_out + kPfWarps - 1) / kPfWarps, B);
    pf_kernel<Ts><<<grid, kPfWarps * 32, sm, s>>>(a, wf);
    check_launch("pf_kernel");
}

void launch_pf(const PfArgs &a, int dtype, int B, cudaStream_t s)
{
    if (a.L > kPfMaxLevels) throw std::runtime_error("pf_kernel: too many boxcar levels");
    if (dtype == 0) launch_pf_t<float>(a, B, s);
    else if (dtype == 1) launch_pf_t<__half>(a, B, s);
    else launch_pf_t<__nv_bfloat16>(a, B, s);
}

}  // namespace pb2
