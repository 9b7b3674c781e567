// kernels.cu -- sm_100a kernels of the B200 dedispersion path.
//
//   grid_lds_kernel  tree gridding + lagged downsampling (replaces GpuTreeGriddingKernel,
//                    src_lib/TreeGriddingKernel.cu:108-279, and GpuLaggedDownsamplingKernel,
//                    src_lib/GpuLaggedDownsamplingKernel.cu:668-918)
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
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>

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

// Tree butterflies with (NORM) or without the per-step 1/sqrt2. float32 storage normalizes at every
// step, as the reference does, so that its outputs are bitwise the reference's. 16-bit storage keeps
// its in-register fp32 sums unnormalized and scales once, by tree_scale(steps) = 2^(-steps/2), where a
// value leaves the registers (a stored row or an emitted subband): one rounding instead of one per
// step, and one multiply per stored value instead of one per butterfly.
template<bool NORM>
__device__ __forceinline__ float bfly_n(float x, float y) { return NORM ? bfly(x, y) : __fadd_rn(x, y); }

__host__ __device__ constexpr float tree_scale(int steps)
{
    float s = (steps & 1) ? kRsqrt2 : 1.0f;
    for (int i = 0; i < steps / 2; i++) s *= 0.5f;
    return s;
}

// A value leaving the registers after n unnormalized butterflies (n is a compile-time constant at
// every call site once the step loops are unrolled).
__device__ __forceinline__ float tree_out(float v, int n) { return n ? __fmul_rn(v, tree_scale(n)) : v; }

// Two fp32 additions (multiplications) in one sm_100 packed f32x2 instruction; each element is
// rounded to nearest like __fadd_rn (__fmul_rn).
__device__ __forceinline__ unsigned long long f2pack(float2 a)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 f2unpack(unsigned long long r)
{
    float2 d;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(r));
    return d;
}
__device__ __forceinline__ float2 f2add(float2 a, float2 b)
{
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2pack(a)), "l"(f2pack(b)));
    return f2unpack(d);
}
__device__ __forceinline__ float2 f2mul(float2 a, float2 b)
{
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2pack(a)), "l"(f2pack(b)));
    return f2unpack(d);
}

__device__ __forceinline__ int brev_bits(int x, int nbits) { return nbits ? int(__brev(unsigned(x)) >> (32 - nbits)) : 0; }

static void check_launch(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}


// -------------------------------------------------------------------------------------------------
// Tree gridding fused with lagged downsampling.
//
// Gridding: tree channel n = sum_f w[n,f] in[f], summed in ascending f from zero with float(w)
// overlap weights (ReferenceTreeGriddingKernel::apply, src_lib/TreeGriddingKernel.cu:62-102).
// Lagged downsampling, for each level p = 1..nlev:
//   ds_p[ch][u]  = (ds_{p-1}[ch][2u] + ds_{p-1}[ch][2u+1]) / sqrt2          (ds_0 = level-0 tree)
//   out_p[c][u]  = (ds_p[2c][u-1] + ds_p[2c+1][u]) / sqrt2                     (one-sample lag on even channels)
// out_p goes to a per-row delay line, written delayed by the per-row "large" lag
// 2^s1dd - 1 - (c mod 2^s1dd) (ReferenceLaggedDownsamplingKernel.cpp:46-57), so that the stage-1
// kernel reads aligned rows.
//
// One thread per (beam, tree-channel pair (2c, 2c+1), window of W0 level-0 samples); consecutive
// threads take consecutive windows, so every load and store is a contiguous run across the warp.
// The thread grids both channels of its window (and writes them as the level-0 tree), builds every
// level in registers, and gets the even channel's predecessor sample at each level by gridding the
// 2^nlev samples before its window (at the chunk start: from a parity double-buffered state).


// Loads W consecutive samples starting at p (16-byte vectors when W*sizeof(Ts) allows; p must then be
// 16-byte aligned).
template<typename Ts, int W>
__device__ __forceinline__ void load_run(const Ts *p, float (&o)[W])
{
    if constexpr ((W * sizeof(Ts)) % 16 == 0) {
        constexpr int PER = 16 / sizeof(Ts);
#pragma unroll
        for (int v = 0; v < W / PER; v++) {
            uint4 q = ((const uint4 *) p)[v];
            const Ts *h = (const Ts *) &q;
#pragma unroll
            for (int k = 0; k < PER; k++) o[v * PER + k] = to_f(h[k]);
        }
    } else {
#pragma unroll
        for (int i = 0; i < W; i++) o[i] = to_f(p[i]);
    }
}

template<typename Ts, int W>
__device__ __forceinline__ void store_run(Ts *p, const float (&o)[W])
{
    if constexpr ((W * sizeof(Ts)) % 16 == 0) {
        constexpr int PER = 16 / sizeof(Ts);
#pragma unroll
        for (int v = 0; v < W / PER; v++) {
            uint4 q;
            Ts *h = (Ts *) &q;
#pragma unroll
            for (int k = 0; k < PER; k++) h[k] = from_f<Ts>(o[v * PER + k]);
            ((uint4 *) p)[v] = q;
        }
    } else {
#pragma unroll
        for (int i = 0; i < W; i++) p[i] = from_f<Ts>(o[i]);
    }
}

// int4 dequantization, restating pirate's ReferenceDequantizationKernel::apply
// (src_lib/GpuDequantizationKernel.cu:326-380): nibble -> signed value v in [-8, 7]; v = -8 is the
// "missing sample" sentinel and gives 0; otherwise scale * v + offset, one fp32 multiply and one fp32
// add with (scale, offset) converted from fp16. The result is then rounded once to the output type.
__device__ __forceinline__ float dq_value(uint32_t nib, float scale, float offset)
{
    // u = v + 8 in [0, 15]; 2^23 + u is exact in fp32, so subtracting 2^23 + 8 gives v exactly.
    const uint32_t u = (nib & 0xf) ^ 8u;
    const float fv = __fsub_rn(__uint_as_float(0x4B000000u + u), 8388616.0f);
    return (u == 0) ? 0.0f : __fadd_rn(__fmul_rn(scale, fv), offset);
}

// W consecutive samples from t0 of one int4 row (row = the row's bytes, so = its (scale, offset)
// pairs), dequantized, rounded to Ts and returned as floats. The W samples lie in one 256-sample
// scale block; for W >= 8, t0 is a multiple of 8 (32-bit nibble words).
template<typename Ts, int W>
__device__ __forceinline__ void load_run_q(const uint8_t *row, const __half2 *so_row, long t0, float (&o)[W])
{
    const float2 so = __half22float2(so_row[t0 >> 8]);
    if constexpr (W % 8 == 0) {
#pragma unroll
        for (int w = 0; w < W / 8; w++) {
            const uint32_t word = ((const uint32_t *) (row + (t0 >> 1)))[w];
#pragma unroll
            for (int k = 0; k < 8; k++) o[8 * w + k] = to_f(from_f<Ts>(dq_value(word >> (4 * k), so.x, so.y)));
        }
    } else {
#pragma unroll
        for (int i = 0; i < W; i++) {
            const long t = t0 + i;
            const uint32_t byte = row[t >> 1];
            o[i] = to_f(from_f<Ts>(dq_value((t & 1) ? (byte >> 4) : byte, so.x, so.y)));
        }
    }
}

// Grids tree channel n over samples [t0, t0+W) of batch beam b's input. With Q the input rows are
// int4 (dequantized on load exactly as the standalone dequantization kernel would write them).
template<typename Ts, int W, bool Q>
__device__ __forceinline__ void grid_run(const GridLdsArgs &a, int b, long n, long t0, float (&o)[W])
{
#pragma unroll
    for (int i = 0; i < W; i++) o[i] = 0.0f;
    const int f0 = a.chan_f0[n], cnt = a.chan_cnt[n], woff = a.chan_woff[n];
    for (int k = 0; k < cnt; k++) {
        const float w = a.chan_w[woff + k];
        const long row = (long) b * a.F + f0 + k;
        float x[W];
        if constexpr (Q)
            load_run_q<Ts, W>((const uint8_t *) a.q_data + row * (a.T >> 1), (const __half2 *) a.q_scoff + row * (a.T >> 8), t0, x);
        else
            load_run<Ts, W>((const Ts *) a.in + row * a.T + t0, x);
#pragma unroll
        for (int i = 0; i < W; i++) o[i] = __fadd_rn(o[i], __fmul_rn(w, x[i]));
    }
}

// int4 gridding through per-warp lookup tables. A warp's 32 windows of one tree-channel pair read the
// same few input rows, each input sample once per tree channel that overlaps its row (about 2.5 times
// at rank 16 from 16384 channels). Instead of dequantizing on every read, the warp first tabulates,
// per (row, 256-sample scale block), the 16 values its nibbles can take, rounded to Ts exactly as
// load_run_q rounds them; each read is then a nibble extract and a shared-memory lookup.
constexpr int kLutRows = 8;   // input rows per channel pair served by the tables

// Table of the warp: lut[(r * NBLK + blk) * 16 + u] = sample value of nibble u in row rlo + r, scale
// block blk0 + blk.
template<typename Ts, int NBLK>
__device__ __forceinline__ void lut_build(const GridLdsArgs &a, int b, int rlo, int nrows, long blk0, float *lut, int lane)
{
    const __half2 *so = (const __half2 *) a.q_scoff;
    const long nsb = a.T >> 8;
    for (int e = lane; e < nrows * NBLK * 16; e += 32) {
        const int r = e / (NBLK * 16), blk = (e / 16) % NBLK, u = e & 15;
        const float2 sc = __half22float2(so[((long) b * a.F + rlo + r) * nsb + blk0 + blk]);
        lut[e] = to_f(from_f<Ts>(dq_value(uint32_t(u), sc.x, sc.y)));
    }
    __syncwarp();
}

// The nibble words of a window of W samples (W / 8 words) of input row 'row' (t0 a multiple of 8).
template<int W>
__device__ __forceinline__ void lut_words(const GridLdsArgs &a, long row, long t0, uint32_t (&q)[W / 8])
{
    const uint32_t *p = (const uint32_t *) ((const uint8_t *) a.q_data + row * (a.T >> 1) + (t0 >> 1));
#pragma unroll
    for (int v = 0; v < W / 8; v++) q[v] = p[v];
}

// o += w * (row's samples), the samples looked up in table L.
template<int W>
__device__ __forceinline__ void lut_accum(float (&o)[W], float w, const uint32_t (&q)[W / 8], const float *L)
{
#pragma unroll
    for (int v = 0; v < W / 8; v++)
#pragma unroll
        for (int k8 = 0; k8 < 8; k8++) o[8 * v + k8] = __fadd_rn(o[8 * v + k8], __fmul_rn(w, L[(q[v] >> (4 * k8)) & 15]));
}

// grid_run<Ts, W, true> of tree channel n through the warp's tables (W a multiple of 8, t0 in scale
// block blk0 + myblk), summed in ascending input channel. q0 holds the words of the channel's first
// input row (loaded by the caller before the tables were built); later rows are loaded here.
template<typename Ts, int W, int NBLK>
__device__ __forceinline__ void grid_run_lut(const GridLdsArgs &a, int b, int f0, int cnt, int woff, long t0, float (&o)[W],
                                             const uint32_t (&q0)[W / 8], const float *lut, int rlo, int myblk)
{
#pragma unroll
    for (int i = 0; i < W; i++) o[i] = 0.0f;
    if (cnt > 0)
        lut_accum<W>(o, a.chan_w[woff], q0, lut + ((f0 - rlo) * NBLK + myblk) * 16);
    for (int k = 1; k < cnt; k++) {
        uint32_t q[W / 8];
        lut_words<W>(a, (long) b * a.F + f0 + k, t0, q);
        lut_accum<W>(o, a.chan_w[woff + k], q, lut + ((f0 + k - rlo) * NBLK + myblk) * 16);
    }
}

// Standalone dequantization: one thread per 32 samples (16 input bytes, 16-byte output stores).
template<typename To>
__global__ void __launch_bounds__(256) dequant_kernel(To *out, const uint8_t *data, const __half2 *scoff, long rows, int T)
{
    const long nper = T / 32;
    const long g = (long) blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= rows * nper)
        return;
    const long row = g / nper;
    const long t0 = (g - row * nper) * 32;
    float o[32];
    load_run_q<To, 32>(data + row * (T >> 1), scoff + row * (T >> 8), t0, o);
    store_run<To, 32>(out + row * T + t0, o);
}

void launch_dequantize(void *out, int out_dtype, const void *data, const void *scales_offsets, long nbeams, long nfreq,
                       long ntime, cudaStream_t s)
{
    if (ntime <= 0 || ntime % 256) throw std::runtime_error("dequantize: ntime must be a positive multiple of 256");
    if (!out || !data || !scales_offsets) throw std::runtime_error("dequantize: null pointer");
    const long rows = nbeams * nfreq;
    const long nthr = rows * (ntime / 32);
    if (nthr == 0) return;
    const unsigned grid = (unsigned) ((nthr + 255) / 256);
    const uint8_t *d = (const uint8_t *) data;
    const __half2 *so = (const __half2 *) scales_offsets;
    if (out_dtype == 0) dequant_kernel<float><<<grid, 256, 0, s>>>((float *) out, d, so, rows, int(ntime));
    else if (out_dtype == 1) dequant_kernel<__half><<<grid, 256, 0, s>>>((__half *) out, d, so, rows, int(ntime));
    else dequant_kernel<__nv_bfloat16><<<grid, 256, 0, s>>>((__nv_bfloat16 *) out, d, so, rows, int(ntime));
    check_launch("dequant_kernel");
}

// ---------------------------------------------------------------------------------------------
// Per-beam peak over a batch's outputs (the toy grouper's reduction, see BeamPeakArgs).
// One 1024-thread block per beam scans every tree of that beam with 16-byte loads where the beam's
// slice is aligned, keeping per thread the largest value and its first index; the block then
// reduces with ties going to the smaller index, and thread 0 merges the trees in order.

// 16 bytes of out_max as raw words; element k of them as fp32.
template<typename T> struct PeakVec;
template<> struct PeakVec<float>
{
    static constexpr int N = 4;
    __device__ static float get(const uint4 &q, int k)
    {
        return __uint_as_float(k == 0 ? q.x : k == 1 ? q.y : k == 2 ? q.z : q.w);
    }
};
template<> struct PeakVec<__half>
{
    static constexpr int N = 8;
    __device__ static float get(const uint4 &q, int k)
    {
        const uint32_t w = (k < 2) ? q.x : (k < 4) ? q.y : (k < 6) ? q.z : q.w;
        return __half2float(__ushort_as_half((unsigned short) ((k & 1) ? (w >> 16) : (w & 0xffff))));
    }
};
template<> struct PeakVec<__nv_bfloat16>
{
    static constexpr int N = 8;
    __device__ static float get(const uint4 &q, int k)
    {
        const uint32_t w = (k < 2) ? q.x : (k < 4) ? q.y : (k < 6) ? q.z : q.w;
        return __uint_as_float((k & 1) ? (w & 0xffff0000u) : (w << 16));
    }
};

__device__ __forceinline__ void peak_take(float v, long i, float &bv, long &bi)
{
    if (v > bv || (v == bv && i < bi)) { bv = v; bi = i; }
}

template<typename T>
__global__ void __launch_bounds__(1024) beam_peak_kernel(BeamPeakArgs a)
{
    constexpr int V = PeakVec<T>::N;
    constexpr long kNone = 0x7fffffffffffffffL;
    __shared__ float rv[32];
    __shared__ long ri[32];
    __shared__ int rn[32];
    const int b = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;

    float gv = -INFINITY;            // thread 0: best over the trees so far
    int gt = -1;
    long gi = 0;

    for (int t = 0; t < a.ntrees; t++) {
        const long n = a.ndm[t] * a.nt[t];
        const T *x = (const T *) a.out_max[t] + (long) b * n;
        float bv = -INFINITY;
        long bi = kNone;
        bool nan = false;
        if (n % V == 0 && ((uintptr_t) x & 15) == 0) {
            const long nv = n / V;
            const uint4 *xv = (const uint4 *) x;
            for (long j = threadIdx.x; j < nv; j += 4L * blockDim.x) {
                uint4 q[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const long jj = j + (long) u * blockDim.x;
                    if (jj < nv) q[u] = __ldg(xv + jj);
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const long jj = j + (long) u * blockDim.x;
                    if (jj < nv) {
#pragma unroll
                        for (int k = 0; k < V; k++) {
                            const float v = PeakVec<T>::get(q[u], k);
                            nan |= (v != v);
                            if (v > bv) { bv = v; bi = jj * V + k; }
                        }
                    }
                }
            }
        } else {
            for (long i = threadIdx.x; i < n; i += blockDim.x) {
                const float v = to_f(x[i]);
                nan |= (v != v);
                if (v > bv) { bv = v; bi = i; }
            }
        }

#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            peak_take(__shfl_down_sync(0xffffffffu, bv, o), __shfl_down_sync(0xffffffffu, bi, o), bv, bi);
        const bool wnan = __any_sync(0xffffffffu, nan);
        if (lane == 0) { rv[warp] = bv; ri[warp] = bi; rn[warp] = wnan; }
        __syncthreads();
        if (warp == 0) {
            bv = (lane < nwarps) ? rv[lane] : -INFINITY;
            bi = (lane < nwarps) ? ri[lane] : kNone;
            const bool tnan = __any_sync(0xffffffffu, (lane < nwarps) && rn[lane]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                peak_take(__shfl_down_sync(0xffffffffu, bv, o), __shfl_down_sync(0xffffffffu, bi, o), bv, bi);
            if (lane == 0 && !tnan && bv > gv) { gv = bv; gt = t; gi = bi; }
        }
        __syncthreads();
    }

    if (threadIdx.x == 0) {
        a.peak[b] = gv;
        a.tree[b] = gt;
        if (gt >= 0) {
            const long nt = a.nt[gt];
            a.idm[b] = int(gi / nt);
            a.itime[b] = int(gi % nt);
            a.token[b] = a.out_argmax[gt][(long) b * a.ndm[gt] * nt + gi];
        } else {
            a.idm[b] = -1;
            a.itime[b] = -1;
            a.token[b] = 0;
        }
    }
}

struct PeakPartial
{
    float v;      // maximum of the slice (-inf if empty)
    int nan;      // the slice holds a NaN
    long i;       // first position of the maximum in the tree (kNone if none)
};

// Grid (nsplit, ntrees, nbeams): block (s, t, b) reduces slice s of tree t of beam b.
template<typename T>
__global__ void __launch_bounds__(256) beam_peak_split_kernel(BeamPeakArgs a, PeakPartial *part, int nsplit)
{
    constexpr int V = PeakVec<T>::N;
    constexpr long kNone = 0x7fffffffffffffffL;
    __shared__ float rv[8];
    __shared__ long ri[8];
    __shared__ int rn[8];
    const int s = blockIdx.x, t = blockIdx.y, b = blockIdx.z;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long n = a.ndm[t] * a.nt[t];
    const T *x = (const T *) a.out_max[t] + (long) b * n;
    float bv = -INFINITY;
    long bi = kNone;
    bool nan = false;
    if (n % V == 0 && ((uintptr_t) x & 15) == 0) {
        const long nv = n / V, per = (nv + nsplit - 1) / nsplit;
        const long lo = (long) s * per, hi = min(nv, lo + per);
        const uint4 *xv = (const uint4 *) x;
        for (long j = lo + threadIdx.x; j < hi; j += blockDim.x) {
            const uint4 q = __ldg(xv + j);
#pragma unroll
            for (int k = 0; k < V; k++) {
                const float v = PeakVec<T>::get(q, k);
                nan |= (v != v);
                if (v > bv) { bv = v; bi = j * V + k; }
            }
        }
    } else {
        const long per = (n + nsplit - 1) / nsplit;
        const long lo = (long) s * per, hi = min(n, lo + per);
        for (long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const float v = to_f(x[i]);
            nan |= (v != v);
            if (v > bv) { bv = v; bi = i; }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        peak_take(__shfl_down_sync(0xffffffffu, bv, o), __shfl_down_sync(0xffffffffu, bi, o), bv, bi);
    const bool wnan = __any_sync(0xffffffffu, nan);
    if (lane == 0) { rv[warp] = bv; ri[warp] = bi; rn[warp] = wnan; }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        bv = (lane < nw) ? rv[lane] : -INFINITY;
        bi = (lane < nw) ? ri[lane] : kNone;
        const bool tn = __any_sync(0xffffffffu, (lane < nw) && rn[lane]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            peak_take(__shfl_down_sync(0xffffffffu, bv, o), __shfl_down_sync(0xffffffffu, bi, o), bv, bi);
        if (lane == 0) {
            PeakPartial &p = part[((long) b * a.ntrees + t) * nsplit + s];
            p.v = bv;
            p.nan = tn ? 1 : 0;
            p.i = bi;
        }
    }
}

// One warp per beam: per tree (in order) the slices' maximum with the first position, a tree holding a
// NaN passed over, then the first tree with the strictly largest maximum (beam_peak_kernel's rules).
__global__ void beam_peak_final_kernel(BeamPeakArgs a, const PeakPartial *part, int nsplit)
{
    constexpr long kNone = 0x7fffffffffffffffL;
    const int b = blockIdx.x, lane = threadIdx.x;
    float gv = -INFINITY;
    int gt = -1;
    long gi = 0;
    for (int t = 0; t < a.ntrees; t++) {
        float bv = -INFINITY;
        long bi = kNone;
        bool nan = false;
        for (int s = lane; s < nsplit; s += 32) {
            const PeakPartial p = part[((long) b * a.ntrees + t) * nsplit + s];
            nan |= (p.nan != 0);
            peak_take(p.v, p.i, bv, bi);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            peak_take(__shfl_down_sync(0xffffffffu, bv, o), __shfl_down_sync(0xffffffffu, bi, o), bv, bi);
        const bool tnan = __any_sync(0xffffffffu, nan);
        if (lane == 0 && !tnan && bv > gv) { gv = bv; gt = t; gi = bi; }
    }
    if (lane == 0) {
        a.peak[b] = gv;
        a.tree[b] = gt;
        if (gt >= 0) {
            const long nt = a.nt[gt];
            a.idm[b] = int(gi / nt);
            a.itime[b] = int(gi % nt);
            a.token[b] = a.out_argmax[gt][(long) b * a.ndm[gt] * nt + gi];
        } else {
            a.idm[b] = -1;
            a.itime[b] = -1;
            a.token[b] = 0;
        }
    }
}

void launch_beam_peaks_split(const BeamPeakArgs &a, int dtype, long nbeams, void *scratch, int nsplit, cudaStream_t s)
{
    if (a.ntrees <= 0 || a.ntrees > kBeamPeakMaxTrees) throw std::runtime_error("beam_peaks: bad number of trees");
    if (!scratch || nsplit < 1 || nsplit > 1024) throw std::runtime_error("beam_peaks: bad split scratch");
    if (nbeams <= 0) return;
    if (nbeams > 65535) throw std::runtime_error("beam_peaks: too many beams for the split reduction");
    dim3 grid((unsigned) nsplit, (unsigned) a.ntrees, (unsigned) nbeams);
    PeakPartial *part = (PeakPartial *) scratch;
    if (dtype == 0) beam_peak_split_kernel<float><<<grid, 256, 0, s>>>(a, part, nsplit);
    else if (dtype == 1) beam_peak_split_kernel<__half><<<grid, 256, 0, s>>>(a, part, nsplit);
    else if (dtype == 2) beam_peak_split_kernel<__nv_bfloat16><<<grid, 256, 0, s>>>(a, part, nsplit);
    else throw std::runtime_error("beam_peaks: bad dtype");
    check_launch("beam_peak_split_kernel");
    beam_peak_final_kernel<<<(unsigned) nbeams, 32, 0, s>>>(a, part, nsplit);
    check_launch("beam_peak_final_kernel");
}

void launch_beam_peaks(const BeamPeakArgs &a, int dtype, long nbeams, cudaStream_t s)
{
    if (a.ntrees < 0 || a.ntrees > kBeamPeakMaxTrees) throw std::runtime_error("beam_peaks: bad number of trees");
    if (!a.peak || !a.tree || !a.idm || !a.itime || !a.token) throw std::runtime_error("beam_peaks: null output pointer");
    for (int t = 0; t < a.ntrees; t++) {
        if (!a.out_max[t] || !a.out_argmax[t]) throw std::runtime_error("beam_peaks: null output array");
        if (a.ndm[t] <= 0 || a.nt[t] <= 0 || a.ndm[t] * a.nt[t] >= (1L << 31))
            throw std::runtime_error("beam_peaks: tree shape out of range");
    }
    if (nbeams <= 0) return;
    if (nbeams > 0x7fffffffL) throw std::runtime_error("beam_peaks: too many beams");
    const unsigned grid = (unsigned) nbeams;
    if (dtype == 0) beam_peak_kernel<float><<<grid, 1024, 0, s>>>(a);
    else if (dtype == 1) beam_peak_kernel<__half><<<grid, 1024, 0, s>>>(a);
    else if (dtype == 2) beam_peak_kernel<__nv_bfloat16><<<grid, 1024, 0, s>>>(a);
    else throw std::runtime_error("beam_peaks: dtype must be 0 (float32), 1 (float16) or 2 (bfloat16)");
    check_launch("beam_peak_kernel");
}

// ---------------------------------------------------------------------------------------------
// Pulse injection into a chunk (see launch_pulse_inject): one warp per channel, in the storage
// dtype, as out = round(out + weight * value) with one fp32 multiply and one fp32 add.

template<typename T>
__global__ void pulse_inject_kernel(T *out, long nfreq, long nt, long row_stride, long chunk_it0, const long *it0,
                                    const long *cnt, const long *off, const float *data, float weight)
{
    const long f = (long) blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (f >= nfreq) return;
    const long a = it0[f] - chunk_it0;
    const long jlo = (a < 0) ? -a : 0;
    const long jhi = (cnt[f] < nt - a) ? cnt[f] : nt - a;
    const float *src = data + off[f];
    T *row = out + f * row_stride + a;
    for (long j = jlo + (threadIdx.x & 31); j < jhi; j += 32)
        row[j] = from_f<T>(__fadd_rn(to_f(row[j]), __fmul_rn(weight, src[j])));
}

void launch_pulse_inject(void *out, int dtype, long nfreq, long nt, long row_stride, long chunk_it0, const long *it0,
                         const long *cnt, const long *off, const float *data, float weight, cudaStream_t s)
{
    if (!out || !it0 || !cnt || !off || !data) throw std::runtime_error("pulse_inject: null pointer");
    if (nfreq <= 0 || nt <= 0 || row_stride < nt) throw std::runtime_error("pulse_inject: bad chunk shape");
    const unsigned grid = (unsigned) ((nfreq + 7) / 8);
    if (dtype == 0) pulse_inject_kernel<float><<<grid, 256, 0, s>>>((float *) out, nfreq, nt, row_stride, chunk_it0, it0, cnt, off, data, weight);
    else if (dtype == 1) pulse_inject_kernel<__half><<<grid, 256, 0, s>>>((__half *) out, nfreq, nt, row_stride, chunk_it0, it0, cnt, off, data, weight);
    else if (dtype == 2) pulse_inject_kernel<__nv_bfloat16><<<grid, 256, 0, s>>>((__nv_bfloat16 *) out, nfreq, nt, row_stride, chunk_it0, it0, cnt, off, data, weight);
    else throw std::runtime_error("pulse_inject: dtype must be 0 (float32), 1 (float16) or 2 (bfloat16)");
    check_launch("pulse_inject_kernel");
}

// ---------------------------------------------------------------------------------------------
// Host spill copies (see SpillArgs): one warp per (beam, spilled row), 16-byte vectors (a chunk row is
// nt * esize bytes, a multiple of 64; every offset is a multiple of 32 samples).

__device__ __forceinline__ long spill_mod(long x, long m) { long r = x % m; return r < 0 ? r + m : r; }

template<bool G2H>
__global__ void __launch_bounds__(256) spill_kernel(SpillArgs a)
{
    const long w = (long) blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= (long) a.nrows * a.B) return;
    const int j = int(w % a.nrows), b = int(w / a.nrows), bt = a.beam0 + b;
    const SpillRow r = a.rows[j];
    const long c = a.chunk_ctr ? *a.chunk_ctr : a.ichunk;
    const long q = G2H ? c : c - r.d + 1;   // chunk moved this step
    const long slot = spill_mod(q, r.S);
    char *dev = (char *) a.ring + ((long) bt * a.ring_beam_stride + (G2H ? r.w_off : r.r_off + spill_mod(q, 2) * a.nt)) * a.esize;
    char *host = (char *) a.host + (r.h_base + ((slot * a.total_beams + bt) * r.n_z + r.k) * (long) a.nt) * a.esize;
    const int nv = a.nt * a.esize / 16;
    const uint4 *src = (const uint4 *) (G2H ? dev : host);
    uint4 *dst = (uint4 *) (G2H ? host : dev);
    for (int i = lane; i < nv; i += 32) dst[i] = src[i];
}

static void launch_spill(const SpillArgs &a, bool g2h, cudaStream_t s)
{
    if (a.nrows <= 0 || a.B <= 0) return;
    if (!a.ring || !a.host || !a.rows) throw std::runtime_error("spill: null pointer");
    if ((a.nt * a.esize) % 64) throw std::runtime_error("spill: chunk rows must be a multiple of 64 bytes");
    const long warps = (long) a.nrows * a.B;
    const unsigned grid = (unsigned) ((warps + 7) / 8);
    if (g2h) spill_kernel<true><<<grid, 256, 0, s>>>(a);
    else spill_kernel<false><<<grid, 256, 0, s>>>(a);
    check_launch("spill_kernel");
}

void launch_spill_g2h(const SpillArgs &a, cudaStream_t s) { launch_spill(a, true, s); }
void launch_spill_h2g(const SpillArgs &a, cudaStream_t s) { launch_spill(a, false, s); }

constexpr int kGridMaxThreads = 512;

template<typename Ts, int NLEV, bool Q>
__global__ void __launch_bounds__(kGridMaxThreads) grid_lds_kernel(GridLdsArgs a)
{
    constexpr int W0 = ((1 << NLEV) > 8) ? (1 << NLEV) : 8;
    constexpr int WE = 1 << NLEV;           // level-0 samples feeding one level-NLEV sample
    __shared__ float xch[(NLEV > 0) ? NLEV : 1][kGridMaxThreads];
    // int4 lookup tables (grid_run_lut): for windows of at most 16 samples, NBLK scale blocks per warp.
    constexpr bool LUT = Q && (W0 <= 16);
    constexpr int NBLK = LUT ? (32 * W0) / 256 : 1;
    __shared__ float lut_sh[LUT ? (kGridMaxThreads / 32) * kLutRows * NBLK * 16 : 1];

    const long nhalf = 1L << (a.rank - 1);
    const long nwin = a.T / W0;
    const long g = (long) blockIdx.x * blockDim.x + threadIdx.x;
    // Threads past the end take part in the block barrier only.
    const bool live = g < nwin * nhalf * a.B;
    const long gg = live ? g : 0;
    const int win = int(gg % nwin);
    const long c = (gg / nwin) % nhalf;
    const int b = int(gg / (nwin * nhalf));
    const int bt = a.beam0 + b;
    const long ichunk = a.chunk_ctr ? *a.chunk_ctr : a.ichunk;
    const int parity = int(ichunk & 1);
    const long t0 = (long) win * W0;

    float r0[W0], r1[W0];
    // A warp uses the tables when its 32 threads are live windows of one channel pair (nwin a multiple
    // of 32; blocks start at window 0) whose input rows fit; the choice is uniform across the warp.
    bool use_lut = false;
    if constexpr (LUT) {
        if (live && (nwin & 31) == 0) {
            const int fa = a.chan_f0[2 * c], ca = a.chan_cnt[2 * c], fb = a.chan_f0[2 * c + 1], cb = a.chan_cnt[2 * c + 1];
            const int rlo = min(ca ? fa : fb, cb ? fb : fa);
            const int rhi = max(fa + ca, fb + cb);
            use_lut = (rhi - rlo) <= kLutRows;
            if (use_lut) {
                // The first input row of each channel is loaded before the tables are built, so that its
                // latency overlaps that of the (scale, offset) loads.
                uint32_t qa[W0 / 8], qb[W0 / 8];
                lut_words<W0>(a, (long) b * a.F + (ca ? fa : rlo), t0, qa);
                lut_words<W0>(a, (long) b * a.F + (cb ? fb : rlo), t0, qb);
                const int wa = a.chan_woff[2 * c], wb = a.chan_woff[2 * c + 1];
                const int lane = threadIdx.x & 31;
                const long blk0 = ((long) (win - lane) * W0) >> 8;
                float *lut = lut_sh + (threadIdx.x >> 5) * (kLutRows * NBLK * 16);
                lut_build<Ts, NBLK>(a, b, rlo, rhi - rlo, blk0, lut, lane);
                const int myblk = int((t0 >> 8) - blk0);
                grid_run_lut<Ts, W0, NBLK>(a, b, fa, ca, wa, t0, r0, qa, lut, rlo, myblk);
                grid_run_lut<Ts, W0, NBLK>(a, b, fb, cb, wb, t0, r1, qb, lut, rlo, myblk);
            }
        }
    }
    if (live && !use_lut) {
        grid_run<Ts, W0, Q>(a, b, 2 * c, t0, r0);
        grid_run<Ts, W0, Q>(a, b, 2 * c + 1, t0, r1);
    }
    if (live) {
        Ts *lev0 = (Ts *) a.tree0 + ((long) b * (2 * nhalf) + 2 * c) * a.T + t0;
        store_run<Ts, W0>(lev0, r0);
        store_run<Ts, W0>(lev0 + a.T, r1);
    }

    if constexpr (NLEV > 0) {
        // Level p of each channel: in place, r[u] = (r[2u] + r[2u+1]) / sqrt2. The odd channel's output
        // sample u pairs with the even channel's sample u-1; for u = 0 that is the last sample of the
        // previous window at this level (the thread before, exchanged through shared memory), or at
        // the chunk start the saved state.
        float first[NLEV], last[NLEV];
#pragma unroll
        for (int p = 1; p <= NLEV; p++) {
            const int len = W0 >> p;
#pragma unroll
            for (int u = 0; u < (W0 >> 1); u++) {
                if (u < len) {
                    r0[u] = bfly(r0[2 * u], r0[2 * u + 1]);
                    r1[u] = bfly(r1[2 * u], r1[2 * u + 1]);
                }
            }
            first[p - 1] = r1[0];
            last[p - 1] = r0[len - 1];
            xch[p - 1][threadIdx.x] = r0[len - 1];

            if (live) {
                const long cap = a.cap_mask[p - 1] + 1;
                Ts *ring = (Ts *) a.ring[p - 1] + ((long) bt * nhalf + c) * cap;
                const long nt_p = a.T >> p;
                const long s_base = ichunk * nt_p + (long) win * len + ((1L << a.lag_rank) - 1 - (c & ((1L << a.lag_rank) - 1)));
#pragma unroll
                for (int u = 1; u < (W0 >> 1); u++)
                    if (u < len)
                        ring[(s_base + u) & a.cap_mask[p - 1]] = from_f<Ts>(bfly(r0[u - 1], r1[u]));
                if (win == nwin - 1)
                    a.state[(((long) (1 - parity) * a.total_beams + bt) * a.nlev + (p - 1)) * nhalf + c] = last[p - 1];
            }
        }
        __syncthreads();

        if (live) {
            float prev[NLEV];
            if (win == 0) {
#pragma unroll
                for (int p = 1; p <= NLEV; p++)
                    prev[p - 1] = a.state[(((long) parity * a.total_beams + bt) * a.nlev + (p - 1)) * nhalf + c];
            } else if (threadIdx.x > 0) {
#pragma unroll
                for (int p = 1; p <= NLEV; p++)
                    prev[p - 1] = xch[p - 1][threadIdx.x - 1];
            } else {
                // The previous window belongs to the previous block: grid its WE samples again.
                float e[WE];
                grid_run<Ts, WE, Q>(a, b, 2 * c, t0 - WE, e);
#pragma unroll
                for (int p = 1; p <= NLEV; p++) {
#pragma unroll
                    for (int u = 0; u < (WE >> 1); u++)
                        if (u < (WE >> p)) e[u] = bfly(e[2 * u], e[2 * u + 1]);
                    prev[p - 1] = e[(WE >> p) - 1];
                }
            }
#pragma unroll
            for (int p = 1; p <= NLEV; p++) {
                const long cap = a.cap_mask[p - 1] + 1;
                Ts *ring = (Ts *) a.ring[p - 1] + ((long) bt * nhalf + c) * cap;
                const long nt_p = a.T >> p;
                const long s_base = ichunk * nt_p + (long) win * (W0 >> p) + ((1L << a.lag_rank) - 1 - (c & ((1L << a.lag_rank) - 1)));
                ring[s_base & a.cap_mask[p - 1]] = from_f<Ts>(bfly(prev[p - 1], first[p - 1]));
            }
        }
    }
}


// -------------------------------------------------------------------------------------------------
// Two-phase register trees (see regtree.cuh). Lane = time sample within a 32-sample tile.


constexpr unsigned kFull = 0xffffffffu;

// Row 'x' of the current tile lagged by L (< 32) samples, with 'p' = the same row in the previous
// tile: the lane that holds the wanted sample offers x or p, and one shuffle delivers it.
__device__ __forceinline__ float lagged(float x, float p, int L, int lane)
{
    return __shfl_sync(kFull, (lane < 32 - L) ? x : p, (lane - L) & 31);
}

template<int K> struct RT
{
    static constexpr int N = 1 << K;
    static constexpr int NP = (K > 0) ? (1 << (K - 1)) : 1;
    static constexpr int NS = (K > 0) ? K : 1;
};

// Butterfly of a lag-0 pair whose history (the previous tile's row0 at lane 31, the only lane that
// needs it) lives in shared memory at *h instead of a register: lane 0 takes it for the lag-1
// operand, then lane 31 stores this tile's row0. The load precedes the store in the warp's program
// order, and the loop's __syncwarp() orders the store before the next tile's load.
template<bool NORM>
__device__ __forceinline__ void bfly_l0_shared(float &v0, float &v1, float *h, int lane)
{
    const float x = v0, y = v1, hp = *h;
    float b = __shfl_sync(kFull, x, lane - 1);
    b = (lane == 0) ? hp : b;
    v0 = bfly_n<NORM>(x, y);
    v1 = bfly_n<NORM>(b, y);
    if (lane == 31) *h = x;
}

// Two butterflies of the same lag L at once: pair A (rows a0, a1, history pa) and pair B (rows b0, b1,
// history pb). Row pairs (i0, i0 + 2^r) and (i0 + N/2, i0 + N/2 + 2^r) of a rank-K register tree have
// the same lag at every step r <= K - 2, so one sm_100 packed f32x2 add does the work of two scalar
// adds with the same rounding. The NORM multiplies stay scalar: packed multiplies by 1/sqrt2 here gave
// outputs a few ulp from the scalar sequence on the GPU (the float32 parity tests at rank 16).
template<bool NORM>
__device__ __forceinline__ void bfly_x2(float &a0, float &a1, float &pa, float &b0, float &b1, float &pb, int L, int lane)
{
    const float xa = a0, xb = b0;
    const float2 Y = make_float2(a1, b1);
    const float2 A = (L == 0) ? make_float2(xa, xb) : make_float2(lagged(xa, pa, L, lane), lagged(xb, pb, L, lane));
    const float2 Bl = make_float2(lagged(xa, pa, L + 1, lane), lagged(xb, pb, L + 1, lane));
    float2 o0 = f2add(A, Y), o1 = f2add(Bl, Y);
    if (NORM) {
        o0 = make_float2(__fmul_rn(kRsqrt2, o0.x), __fmul_rn(kRsqrt2, o0.y));
        o1 = make_float2(__fmul_rn(kRsqrt2, o1.x), __fmul_rn(kRsqrt2, o1.y));
    }
    a0 = o0.x; b0 = o0.y; a1 = o1.x; b1 = o1.y;
    pa = xa; pb = xb;
}

// Step 0 with caller-supplied lag-1 operands (EXT0) for two pairs at once: (x, y) -> (x + y, e + y).
template<bool NORM>
__device__ __forceinline__ void bfly_ext0_x2(float &a0, float &a1, float ea, float &b0, float &b1, float eb)
{
    const float2 Y = make_float2(a1, b1);
    float2 o0 = f2add(make_float2(a0, b0), Y), o1 = f2add(make_float2(ea, eb), Y);
    if (NORM) {
        o0 = make_float2(__fmul_rn(kRsqrt2, o0.x), __fmul_rn(kRsqrt2, o0.y));
        o1 = make_float2(__fmul_rn(kRsqrt2, o1.x), __fmul_rn(kRsqrt2, o1.y));
    }
    a0 = o0.x; b0 = o0.y; a1 = o1.x; b1 = o1.y;
}

// All K steps of a register tree, in place. pv[r][q] holds pair q's row0 input of the previous tile.
// With HS, the lag-0 pairs keep that history in shared memory (hs[slot], one float per pair, in
// (r, q) order), which frees their registers. With EXT0, step 0 (all lags 0) takes its lag-1
// operands from b0[q] = row 2q one sample earlier, supplied by the caller, and keeps no history;
// with F0 the caller has already done step 0 itself (from rows it can read one sample earlier).
// NORM: butterflies with the 1/sqrt2 (bfly_n).
template<int K, bool HS = false, bool EXT0 = false, bool F0 = false, bool NORM = true>
__device__ __forceinline__ void rt_steps(float (&v)[RT<K>::N], float (&pv)[RT<K>::NS][RT<K>::NP], int lane, float *hs = nullptr,
                                         const float *b0 = nullptr)
{
    static_assert(!F0 || EXT0, "a caller-done step 0 keeps no history (EXT0 layout)");
    constexpr int NP = RT<K>::NP, NH = RT<K>::N / 2;
    int slot = 0;
#pragma unroll
    for (int r = 0; r < K; r++) {
#pragma unroll
        for (int q = 0; q < NP; q++) {
            const int h = 1 << r;
            const int i0 = ((q >> r) << (r + 1)) | (q & (h - 1));
            const int L = rt_lag(r, q);
            if (F0 && r == 0)
                continue;
            // Packed: pair q < NP/2 with pair q + NP/2 (rows i0 + N/2), same lag, at steps r <= K - 2.
            const bool PK = (K >= 2) && (r <= K - 2) && !(HS && L == 0 && !(EXT0 && r == 0));
            if (PK && q >= NP / 2)
                continue;   // done with its partner
            if (EXT0 && r == 0) {
                if (PK) {
                    bfly_ext0_x2<NORM>(v[i0], v[i0 + 1], b0[q], v[i0 + NH], v[i0 + NH + 1], b0[q + NP / 2]);
                } else {
                    const float x = v[i0], y = v[i0 + 1];
                    v[i0] = bfly_n<NORM>(x, y);
                    v[i0 + 1] = bfly_n<NORM>(b0[q], y);
                }
                continue;
            }
            if (HS && L == 0) {
                bfly_l0_shared<NORM>(v[i0], v[i0 + h], hs + slot, lane);
                slot++;
                continue;
            }
            if (PK) {
                bfly_x2<NORM>(v[i0], v[i0 + h], pv[r][q], v[i0 + NH], v[i0 + NH + h], pv[r][q + NP / 2], L, lane);
                continue;
            }
            float x = v[i0], y = v[i0 + h];
            float a = (L == 0) ? x : lagged(x, pv[r][q], L, lane);
            float b = lagged(x, pv[r][q], L + 1, lane);
            v[i0] = bfly_n<NORM>(a, y);
            v[i0 + h] = bfly_n<NORM>(b, y);
            pv[r][q] = x;
        }
    }
}

// Persistent histories: pair (r, q) needs its previous-tile row0 only in lanes >= 31 - lag.
// With HS the lag-0 pairs' single value goes to or comes from hs[slot].
template<int K, bool HS = false, bool EXT0 = false>
__device__ __forceinline__ void rt_load(float (&pv)[RT<K>::NS][RT<K>::NP], const float *st, int lane, float *hs = nullptr)
{
    int off = 0, slot = 0;
#pragma unroll
    for (int r = 0; r < K; r++)
#pragma unroll
        for (int q = 0; q < RT<K>::NP; q++) {
            const int L = rt_lag(r, q);
            if (EXT0 && r == 0) {
                // no history (its state slot stays unused)
            } else if (HS && L == 0) {
                if (lane == 0) hs[slot] = st[off];
                slot++;
            } else {
                int i = lane - (31 - L);
                pv[r][q] = (i >= 0) ? st[off + i] : 0.0f;
            }
            off += L + 1;
        }
    if (HS) __syncwarp();
}

template<int K, bool HS = false, bool EXT0 = false>
__device__ __forceinline__ void rt_save(const float (&pv)[RT<K>::NS][RT<K>::NP], float *st, int lane, const float *hs = nullptr)
{
    if (HS) __syncwarp();
    int off = 0, slot = 0;
#pragma unroll
    for (int r = 0; r < K; r++)
#pragma unroll
        for (int q = 0; q < RT<K>::NP; q++) {
            const int L = rt_lag(r, q);
            if (EXT0 && r == 0) {
            } else if (HS && L == 0) {
                if (lane == 0) st[off] = hs[slot];
                slot++;
            } else {
                int i = lane - (31 - L);
                if (i >= 0) st[off + i] = pv[r][q];
            }
            off += L + 1;
        }
}

// Phase b of a stage-2 (subband) tree: before step r' (r' = 0..RB-1) and after it, subband rows of
// pf level r'+1 are emitted (FrequencySubbands multiplet order), reproducing ReferenceTree::dedisperse_2d
// (src_lib/ReferenceTree.cpp:120-300): even band pairs coincide with the in-place butterflies, odd
// ("staggered") pairs (2k+1, 2k+2) are extra butterflies with their own histories ps[r'][u].
// With F0 the caller has done the level-0 emission and step 0's butterflies (not its emission).
// SA: unnormalized butterfly steps the rows have had before phase b (phase a's, or 0); NORM as in
// rt_steps. Each emitted value is scaled by tree_scale of its unnormalized step count.
template<int RB, bool STAG, bool HS, bool EXT0, bool F0, int SA, bool NORM, typename Emit>
__device__ __forceinline__ void phase_b_subbands(float (&v)[1 << RB], float (&pv)[RT<RB>::NS][RT<RB>::NP],
                                                 float (&ps)[RT<RB>::NS][RT<RB>::NP], const Stage2Args &a,
                                                 int lane, Emit emit, float *hs, const float *b0)
{
    static_assert(!F0 || (EXT0 && !STAG), "a caller-done step 0: no history, no staggered pairs");
    constexpr int NB = 1 << RB;
    int slot = 0;   // HS: lag-0 in-place pairs keep their history in hs[slot] (see rt_steps)
    // Band counts are the same for every tile: each level's emission is skipped as a whole when empty.
    if (!F0 && a.sb_count[0] > 0) {
#pragma unroll
        for (int f = 0; f < NB; f++)
            if (f < a.sb_count[0]) emit(a.sb_mbase[0] + f, tree_out(v[f], SA));
    }

#pragma unroll
    for (int r = 0; r < RB; r++) {
        const int cnt = a.sb_count[r + 1], mb = a.sb_mbase[r + 1];
        const int h = 1 << r;
        if (STAG && cnt >= 2) {
#pragma unroll
            for (int u = 0; u < (STAG ? st_count(RB, r) : 0); u++) {
                const int k = u >> r, j = u & (h - 1);
                if (2 * k + 1 < cnt) {
                    const int qa = ((2 * k + 1) << r) | j, qb = ((2 * k + 2) << r) | j;
                    const int L = rt_lag(r, j);
                    float x = v[qa], y = v[qb];
                    float aa = (L == 0) ? x : lagged(x, ps[r][u], L, lane);
                    float bb = lagged(x, ps[r][u], L + 1, lane);
                    int m = mb + (2 * k + 1) * (2 << r) + 2 * bitrev_c(j, r);
                    emit(m, tree_out(bfly_n<NORM>(aa, y), SA + (NORM ? 0 : r + 1)));
                    emit(m + 1, tree_out(bfly_n<NORM>(bb, y), SA + (NORM ? 0 : r + 1)));
                    ps[r][u] = x;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < RT<RB>::NP; q++) {
            constexpr int NP = RT<RB>::NP, NH = NB / 2;
            const int i0 = ((q >> r) << (r + 1)) | (q & (h - 1));
            const int L = rt_lag(r, q);
            // packed pairs (q, q + NP/2) as in rt_steps
            const bool PK = (RB >= 2) && (r <= RB - 2) && !(HS && L == 0 && !(EXT0 && r == 0)) && !(F0 && r == 0);
            if (PK && q >= NP / 2) {
                // done with its partner
            } else if (F0 && r == 0) {
                // done by the caller
            } else if (EXT0 && r == 0) {
                if (PK) {
                    bfly_ext0_x2<NORM>(v[i0], v[i0 + 1], b0[q], v[i0 + NH], v[i0 + NH + 1], b0[q + NP / 2]);
                } else {
                    const float x = v[i0], y = v[i0 + 1];
                    v[i0] = bfly_n<NORM>(x, y);
                    v[i0 + 1] = bfly_n<NORM>(b0[q], y);
                }
            } else if (PK) {
                bfly_x2<NORM>(v[i0], v[i0 + h], pv[r][q], v[i0 + NH], v[i0 + NH + h], pv[r][q + NP / 2], L, lane);
            } else if (HS && L == 0) {
                bfly_l0_shared<NORM>(v[i0], v[i0 + h], hs + slot, lane);
                slot++;
            } else {
                float x = v[i0], y = v[i0 + h];
                float aa = (L == 0) ? x : lagged(x, pv[r][q], L, lane);
                float bb = lagged(x, pv[r][q], L + 1, lane);
                v[i0] = bfly_n<NORM>(aa, y);
                v[i0 + h] = bfly_n<NORM>(bb, y);
                pv[r][q] = x;
            }
        }
        // Even band pairs are step r's in-place outputs.
        if (cnt > 0) {
#pragma unroll
            for (int q = 0; q < RT<RB>::NP; q++) {
                const int i0 = ((q >> r) << (r + 1)) | (q & (h - 1));
                const int k = q >> r, j = q & (h - 1);
                if (2 * k < cnt) {
                    const int m = mb + (2 * k) * (2 << r) + 2 * bitrev_c(j, r);
                    emit(m, tree_out(v[i0], SA + (NORM ? 0 : r + 1)));
                    emit(m + 1, tree_out(v[i0 + h], SA + (NORM ? 0 : r + 1)));
                }
            }
        }
    }
}

template<int K>
__device__ __forceinline__ void st_load(float (&ps)[RT<K>::NS][RT<K>::NP], const float *st, int lane)
{
    int off = 0;
#pragma unroll
    for (int r = 0; r < K; r++)
#pragma unroll
        for (int u = 0; u < RT<K>::NP; u++) {
            if (u < st_count(K, r)) {
                const int L = rt_lag(r, u & ((1 << r) - 1));
                int i = lane - (31 - L);
                ps[r][u] = (i >= 0) ? st[off + i] : 0.0f;
                off += L + 1;
            } else {
                ps[r][u] = 0.0f;
            }
        }
}

template<int K>
__device__ __forceinline__ void st_save(const float (&ps)[RT<K>::NS][RT<K>::NP], float *st, int lane)
{
    int off = 0;
#pragma unroll
    for (int r = 0; r < K; r++)
#pragma unroll
        for (int u = 0; u < RT<K>::NP; u++) {
            if (u < st_count(K, r)) {
                const int L = rt_lag(r, u & ((1 << r) - 1));
                int i = lane - (31 - L);
                if (i >= 0) st[off + i] = ps[r][u];
                off += L + 1;
            }
        }
}

template<typename Ts>
struct PfEmit
{
    Ts *row0;   // multiplet 0 of this warp's coarse dm, at the current tile's slot + lane
    int cap;    // delay line capacity (multiplet stride)
    __device__ __forceinline__ void operator()(int m, float v) const
    {
        row0[m * cap] = from_f<Ts>(v);
    }
};

// Shared-memory delay line between the phases: row rr = f * 2^RA + d (f < 2^RB) starts at float
// off(rr) and has capacity cap(rr) = ring_cap(f, d), a multiple of 32. Phase a writes tile k at
// wpos, phase b reads tile k-1 at rpos - P(f, d); positions are multiples of 32, so a write never
// wraps and a read wraps at most once. Per row the tables hold
//   wb[f * 2^RA + d] = off + wpos                 (phase a: write index of lane 0)
//   rt[d * 2^RB + f] = {off + rpos - P, off | cap << 16}   (phase b: read index of lane 0, wrap bounds)
// so that each warp's rows are consecutive (128-bit table loads).
template<int RA, int RB>
__device__ __forceinline__ int ring_lag(int f, int d) { return ((1 << RB) - 1 - f) * brev_bits(d, RA); }

__device__ __forceinline__ int wrap_add(int p, int cap) { return (p >= cap) ? (p - cap) : ((p < 0) ? (p + cap) : p); }

// Entry i of a warp's consecutive table row (16-byte aligned base; four ints or two int2 per 128-bit
// shared load, the fields selected at compile time in the unrolled loops that call these).
// N = entries per row: 128-bit loads need N a multiple of 4 (int) or 2 (int2), which keeps every
// row base 16-byte aligned; smaller rows use plain loads.
template<int N>
__device__ __forceinline__ int tab_int(const int *base, int i)
{
    if constexpr (N % 4 != 0) {
        return base[i];
    } else {
        const int4 t = ((const int4 *) base)[i >> 2];
        return ((i & 3) == 0) ? t.x : ((i & 3) == 1) ? t.y : ((i & 3) == 2) ? t.z : t.w;
    }
}
template<int N>
__device__ __forceinline__ int2 tab_int2(const int2 *base, int i)
{
    if constexpr (N % 2 != 0) {
        return base[i];
    } else {
        const int4 t = ((const int4 *) base)[i >> 1];
        return (i & 1) ? make_int2(t.z, t.w) : make_int2(t.x, t.y);
    }
}

// Fills wb[] and rt[] for stream time s0 (a multiple of 32). Uses ioff[NR] as scratch; ends with
// __syncthreads().
template<int RA, int RB>
__device__ void ring_init(int *wb, int2 *rt, int *ioff, long s0)
{
    constexpr int NR = 1 << (RA + RB);
    const int rr = threadIdx.x;
    const int f = rr >> RA, d = rr & ((1 << RA) - 1);
    if (rr < NR)
        ioff[rr] = ring_cap(RA, RB, f, d);
    __syncthreads();
    if (threadIdx.x == 0) {
        int o = 0;
        for (int i = 0; i < NR; i++) {
            const int c = ioff[i];
            ioff[i] = o;
            o += c;
        }
    }
    __syncthreads();
    if (rr < NR) {
        const int off = ioff[rr], cap = ring_cap(RA, RB, f, d), P = ring_lag<RA, RB>(f, d);
        const int pos = int(s0 % cap);
        wb[rr] = off + pos;
        rt[d * (1 << RB) + f] = make_int2(off + pos - P, off | (cap << 16));
    }
    __syncthreads();
}

template<int BYTES>
__device__ __forceinline__ void cp_async_bytes(void *smem, const void *gmem)
{
    unsigned s = (unsigned) __cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" :: "r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Staging of one tile of a phase-a warp's NA input rows: 32-bit words copied with cp.async.
// float: 32 words per row; 16-bit types: 17 words (34 samples) starting at an even sample.
// Staging of one tile of input rows with 16-byte cp.async copies of EPC samples. Stage-1 rows are
// read aligned (32 samples); a stage-2 row starts at an arbitrary sample p and is copied as the
// EPC-aligned run of 32 + EPC samples from p & ~(EPC-1) (SPR samples per staged row).
template<typename Ts> struct Stage
{
    static constexpr int EPC = 16 / sizeof(Ts);
    static constexpr int SPR = 32 + EPC;
};

// Shared-memory layout of a two-phase tree kernel (byte offsets; host and device agree).
template<typename Ts, int RA, int RB>
struct TreeSmem
{
    static constexpr int NR = 1 << (RA + RB);
    static_assert(NR >= 2 && ring_floats(RA, RB) < 65536, "delay-line tables pack offset and capacity in 16 bits");
    static constexpr size_t in_tab = 0;                       // int4[NR]
    static constexpr size_t out_base = in_tab + 16 * NR;      // int[NR]
    static constexpr size_t out_off = out_base + 4 * NR;      // int[NR]
    static constexpr size_t rt = out_off + 4 * NR;            // int2[NR]
    static constexpr size_t wb = rt + 8 * NR;                 // int[NR]
    static constexpr size_t in_cap = wb + 4 * NR;             // int[NR]
    static constexpr size_t hist = in_cap + 4 * NR;           // float[warps][16]: lag-0 histories
    static constexpr size_t staging = (hist + 4 * 16 * ((1 << RA) + (1 << RB)) + 15) & ~size_t(15);
    static constexpr size_t ring = (staging + 2 * (1 << RB) * (1 << RA) * Stage<Ts>::SPR * sizeof(Ts) + 15) & ~size_t(15);
    static constexpr size_t total = ring + sizeof(float) * ring_floats(RA, RB);
};

// Lag-0 histories in shared memory (HS in rt_steps) for the rank-7 and rank-8 trees, whose register
// budgets (64 and 80 per thread in 1024- and 768-thread blocks) are the tightest.
__host__ __device__ constexpr bool tree_hs(int RA, int RB, int STAGE) { return RA + RB >= 7; }

template<int STAGE>
struct TreeArgsOf;
template<> struct TreeArgsOf<1> { using type = Stage1Args; };
template<> struct TreeArgsOf<2> { using type = Stage2Args; };

// Launch parameter: one stage-1 tree, or a grid of stage-2 trees (Stage2Multi).
template<int STAGE>
struct TreeParamOf;
template<> struct TreeParamOf<1> { using type = Stage1Args; };
template<> struct TreeParamOf<2> { using type = Stage2Multi; };

template<int STAGE, typename PT>
__device__ __forceinline__ const typename TreeArgsOf<STAGE>::type &tree_args(const PT &P, int ti)
{
    if constexpr (STAGE == 1) return P;
    else return P.t[ti];
}

// Two-phase tree kernel. Warps [0, NB) run phase a on tile k while warps [NB, NB+NA) run phase b on
// tile k-1; one block barrier per tile.
//   STAGE 1: input = level-p tree rows (aligned), output = per-row stage-1 delay lines.
//   STAGE 2: input = stage-1 delay lines read at lag rb_lag (misaligned), output = subband rows.
template<typename Ts, int RA, int RB, int STAGE, bool STAG, bool HS = tree_hs(RA, RB, STAGE)>
__global__ void __launch_bounds__(32 * ((1 << RA) + (1 << RB)), 1) tree_kernel(const __grid_constant__ typename TreeParamOf<STAGE>::type P)
{
    // Stage 2: this block's tree ti and its block index blk among that tree's nblk blocks.
    int ti = 0, blk = blockIdx.x, nblk = gridDim.x;
    if constexpr (STAGE == 2) {
        while (ti + 1 < P.n && blk >= P.blk0[ti + 1]) ti++;
        nblk = P.blk0[ti + 1] - P.blk0[ti];
        blk -= P.blk0[ti];
    }
    const auto &a = tree_args<STAGE>(P, ti);
    constexpr int NA = 1 << RA, NB = 1 << RB, NR = 1 << (RA + RB);
    constexpr int RING = ring_floats(RA, RB);
    // Staging row stride: stage-1 rows are 32 aligned samples; stage-2 rows take one more chunk.
    constexpr int SPRK = (STAGE == 1) ? 32 : Stage<Ts>::SPR;
    using Lay = TreeSmem<Ts, RA, RB>;
    extern __shared__ __align__(16) unsigned char sm_raw[];

    // stage 2, per input row: {read position, capacity, offset low and high words} of its delay line
    int4 *in_tab = (int4 *) (sm_raw + Lay::in_tab);
    // stage 1, per output row (f, d) at [d * NB + f]: index of lane 0 and start of its delay line,
    // relative to the block's first line
    int *out_base = (int *) (sm_raw + Lay::out_base);
    int *out_off = (int *) (sm_raw + Lay::out_off);
    int2 *rt = (int2 *) (sm_raw + Lay::rt);
    int *wb = (int *) (sm_raw + Lay::wb);
    int *in_cap = (int *) (sm_raw + Lay::in_cap);         // stage 1: output delay line capacities
    Ts *staging = (Ts *) (sm_raw + Lay::staging);
    float *ring = (float *) (sm_raw + Lay::ring);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *hs = (float *) (sm_raw + Lay::hist) + warp * 16;   // this warp's lag-0 histories (HS)
    // Step 0 (all lags 0) without shuffles or histories. Stage 1, phase b: the lag-1 operands are read
    // from the shared delay line. Stage 2: each phase does step 0 while it loads its rows, phase a
    // reading each row from one sample earlier in the staging buffer (rows are staged from p - 1)
    // and phase b from the delay line, so no extra values stay live.
    constexpr bool E0 = (STAGE == 1);
    constexpr bool FA = (STAGE == 2) && (RA >= 1);
    constexpr bool FB = (STAGE == 2) && !STAG && (RB >= 1);
    constexpr bool EB = E0 || FB;
    // bfly_n per phase: float32 storage normalizes every step. 16-bit storage skips the 1/sqrt2 in both
    // phases of both stages (measured 4%, 2% and, with the packed adds, 2% faster in stage 2's phase b)
    // and scales by tree_scale(SU) where values leave the registers.
    constexpr bool NORM_A = (sizeof(Ts) == 4);
    constexpr bool NORM_B = (sizeof(Ts) == 4);
    constexpr int SA = NORM_A ? 0 : RA;                 // unnormalized steps before phase b
    constexpr int SU = SA + (NORM_B ? 0 : RB);          // ... and after it
    const int b = blockIdx.y, bt = a.beam0 + b;
    float *st = a.state + ((long) bt * nblk + blk) * a.state_per_block;

    // The shared delay line comes back from HBM with 16-byte cp.async copies (RING is a multiple of 32
    // floats, and each block's state starts on a 16-byte boundary), overlapping the table setup below;
    // each thread waits for its copies before the block barrier that ends the setup.
    const bool st16 = ((reinterpret_cast<uintptr_t>(st) & 15) == 0);
    if (st16) {
        for (int i = threadIdx.x; i < RING / 4; i += blockDim.x)
            cp_async_bytes<16>(ring + 4 * i, st + 4 * i);
        cp_async_commit();
    } else {
        for (int i = threadIdx.x; i < RING; i += blockDim.x)
            ring[i] = st[i];
    }
    const long s0 = a.chunk_ctr ? *a.chunk_ctr * (long) a.nt : a.s0;
    ring_init<RA, RB>(wb, rt, in_cap, s0);

    const Ts *in;
    int pos1 = 0;   // stage 1: read position of every input row (rows are read aligned)
    if constexpr (STAGE == 1) {
        in = (const Ts *) a.in + (long) (a.in_beam0 + b) * a.in_beam_stride + (long) blk * NR * a.in_row_stride;
        pos1 = int(((a.chunk_ctr && a.in_mask != -1) ? s0 : a.in_s0) & a.in_mask);
        const long off0 = a.ring_off[(long) blk * NR];   // the host checks that a block's lines span < 2^31
        for (int r = threadIdx.x; r < NR; r += blockDim.x) {
            const int cap = a.ring_cap[(long) blk * NR + r];   // capacity of output delay line r (a multiple of 32)
            const int off = int(a.ring_off[(long) blk * NR + r] - off0);
            const int j = (r & (NA - 1)) * NB + (r >> RA);      // row (f, d) = r at [d * NB + f]
            in_cap[j] = cap;
            out_off[j] = off;
            out_base[j] = off + int(s0 % cap);
        }
    } else {
        in = (const Ts *) a.ring + (long) bt * a.ring_beam_stride;
        const long dm1 = brev_bits(blk, a.amb_rank) + (a.uflag ? (1L << a.amb_rank) : 0L);
        for (int r = threadIdx.x; r < NR; r += blockDim.x) {
            long row = ((long) r << a.amb_rank) + blk;
            long lag = (long) (NR - 1 - r) * dm1;
            long cap = a.ring_cap[row];
            long p = (s0 - lag) % cap;
            const long off = a.ring_off[row];
            in_tab[r] = make_int4(int(p < 0 ? p + cap : p), int(cap), int(off & 0xffffffffL), int(off >> 32));
        }
    }

    const bool is_a = warp < NB;
    const int g = is_a ? warp : (warp - NB);   // phase-a group (f) or phase-b group (d)
    const int ntiles = a.nt / 32;
    cp_async_wait0();
    __syncthreads();
    // Register splits between the warp roles (whole warpgroups: phase a is warps 0-15). Each block is
    // launched with the kernel's allocation, and the split adds up to exactly that, so the increasing
    // role's request is always satisfied once the other role has decreased, which each of its warps
    // does here before any barrier:
    //   4+4 (1024 threads, 64 registers): 72 x 512 (phase a) + 56 x 512 (phase b) = 64 x 1024, or
    //        56 x 512 + 72 x 512 for stage 2 with staggered subband pairs (phase b's extra histories);
    //   3+4 (768 threads, 80 registers): 72 x 512 (phase a) + 96 x 256 (phase b) = 80 x 768.
    if constexpr (RA == 4 && RB == 4 && !(STAGE == 2 && STAG)) {
        if (is_a) asm volatile("setmaxnreg.inc.sync.aligned.u32 72;");
        else asm volatile("setmaxnreg.dec.sync.aligned.u32 56;");
    }
    if constexpr (RA == 4 && RB == 4 && STAGE == 2 && STAG) {
        if (is_a) asm volatile("setmaxnreg.dec.sync.aligned.u32 56;");
        else asm volatile("setmaxnreg.inc.sync.aligned.u32 72;");
    }
    if constexpr (RA == 3 && RB == 4) {
        if (is_a) asm volatile("setmaxnreg.dec.sync.aligned.u32 72;");
        else asm volatile("setmaxnreg.inc.sync.aligned.u32 96;");
    }

    // The two warp roles run separate loops (so each holds only its own histories in registers);
    // they meet once per tile at named barrier 1.
    if (is_a) {
        float pva[RT<RA>::NS][RT<RA>::NP];
        float *sta = st + RING + g * rt_state(RA);
        // Phase a keeps its lag-0 histories in registers where the split gives it the room (measured
        // faster); with staggered subbands it has 56 registers and keeps them in shared memory.
        constexpr bool HSA = HS && !(RB == 4 && (RA == 4 || RA == 3) && !(STAGE == 2 && STAG));
        rt_load<RA, HSA, FA>(pva, sta, lane, hs);

        // Issues the cp.async copies of this warp's NA rows for one tile into staging buffer 'buf',
        // then advances the rows' read positions by 32 samples.
        Ts *my_stage = staging + g * NA * SPRK;
        auto issue = [&](int buf) {
            Ts *dst = my_stage + buf * NB * NA * SPRK;
            if constexpr (STAGE == 1) {
                // Aligned rows at a common position: 16-byte copies, CH per row.
                constexpr int EPC = 16 / sizeof(Ts), CH = 32 / EPC;
                for (int c = lane; c < NA * CH; c += 32) {
                    const int i = c / CH, k = c % CH;
                    cp_async_bytes<16>(dst + i * SPRK + k * EPC, in + (long) (g * NA + i) * a.in_row_stride + pos1 + k * EPC);
                }
                pos1 = int((pos1 + 32) & a.in_mask);
            } else {
                // Rows at their own positions: CPR consecutive 16-byte chunks from p & ~(EPC-1), consecutive
                // lanes on consecutive chunks of a row. Capacities are multiples of 32 samples, so a chunk
                // never straddles the end of a delay line and wraps at most once.
                // With FA the run starts at p - 1 (32 + 1 samples fit in the same CPR chunks).
                constexpr int EPC = Stage<Ts>::EPC, CPR = 32 / EPC + 1;
                for (int c = lane; c < NA * CPR; c += 32) {
                    const int i = c / CPR, k = c - i * CPR, r = g * NA + i;
                    const int4 t = in_tab[r];
                    const int cap = t.y;
                    const int p0 = FA ? ((t.x == 0) ? (cap - 1) : (t.x - 1)) : t.x;
                    int q = (p0 & ~(EPC - 1)) + k * EPC;
                    q = (q >= cap) ? (q - cap) : q;
                    cp_async_bytes<16>(dst + i * SPRK + k * EPC, in + ((long) t.w << 32 | (unsigned) t.z) + q);
                }
                __syncwarp();
                if (lane < NA) {
                    const int rr = g * NA + lane;
                    in_tab[rr].x = wrap_add(in_tab[rr].x + 32, in_tab[rr].y);
                }
            }
            __syncwarp();
        };

        // Stage 2: bits [OB i, OB i + OB) = offset in its staged run of the first staged sample of row i,
        // (p - FA) & (EPC-1) (constant: positions advance by 32 and capacities are multiples of 32).
        constexpr int OB = (sizeof(Ts) == 4) ? 2 : 3;
        unsigned long long offs = 0;
        if (STAGE == 2) {
#pragma unroll
            for (int i = 0; i < NA; i++)
                offs |= (unsigned long long) ((in_tab[g * NA + i].x - (FA ? 1 : 0)) & (Stage<Ts>::EPC - 1)) << (OB * i);
        }
        issue(0);
        cp_async_commit();

        for (int it = 0; it <= ntiles; it++) {
            if (it < ntiles) {
                if (it + 1 < ntiles) issue((it + 1) & 1);
                cp_async_commit();
                cp_async_wait1();
                __syncwarp();
                const Ts *sb = my_stage + (it & 1) * NB * NA * SPRK;
                float v[NA];
                if constexpr (FA) {
                    // Step 0 while loading: pair (2q, 2q + 1), lag-1 operand = row 2q one sample earlier.
#pragma unroll
                    for (int q = 0; q < NA / 2; q++) {
                        const Ts *r0 = sb + 2 * q * SPRK + lane + int((offs >> (OB * 2 * q)) & ((1u << OB) - 1));
                        const Ts *r1 = sb + (2 * q + 1) * SPRK + lane + int((offs >> (OB * (2 * q + 1))) & ((1u << OB) - 1));
                        const float xm = to_f(r0[0]), x = to_f(r0[1]), y = to_f(r1[1]);
                        v[2 * q] = bfly_n<NORM_A>(x, y);
                        v[2 * q + 1] = bfly_n<NORM_A>(xm, y);
                    }
                    rt_steps<RA, HSA, true, true, NORM_A>(v, pva, lane, hs);
                } else {
#pragma unroll
                    for (int i = 0; i < NA; i++)
                        v[i] = to_f(sb[i * SPRK + lane + int((offs >> (OB * i)) & ((1u << OB) - 1))]);
                    rt_steps<RA, HSA, false, false, NORM_A>(v, pva, lane, hs);
                }
#pragma unroll
                for (int i = 0; i < NA; i++)
                    ring[tab_int<NA>(wb + g * NA, i) + lane] = v[i];
                __syncwarp();
                if (lane < NA) {
                    const int rr = g * NA + lane;
                    const int y = rt[lane * NB + g].y;   // phase b updates only rt[].x
                    const int lo = y & 0xffff, cap = y >> 16;
                    const int w = wb[rr] + 32;
                    wb[rr] = (w == lo + cap) ? lo : w;
                }
            }
            asm volatile("bar.sync 1, %0;" :: "r"(blockDim.x) : "memory");
        }
        cp_async_wait0();
        rt_save<RA, HSA, FA>(pva, sta, lane, hs);
    } else {
        float pvb[RT<RB>::NS][RT<RB>::NP], psb[RT<RB>::NS][RT<RB>::NP];
        float *stb = st + RING + NB * rt_state(RA) + g * (rt_state(RB) + (STAGE == 2 ? st_state(RB) : 0));
        // Phase b keeps its lag-0 histories in shared memory (56 registers, or 72 with staggered pairs,
        // whose own histories take the room), except in the 3+4 trees, where it has 96.
        constexpr bool HSB = HS && !(RA == 3 && RB == 4);
        rt_load<RB, HSB, EB>(pvb, stb, lane, hs);
        if (STAG) st_load<RB>(psb, stb + rt_state(RB), lane);

        PfEmit<Ts> emit;
        Ts *pf_rows = nullptr;   // stage 2: multiplet 0 of this warp's coarse dm
        int pf_slot = 0;         // stage 2: delay-line slot of this lane's sample in the current tile
        if constexpr (STAGE == 2) {
            const int pf_dm = brev_bits(g, RA);
            const long rowbase = ((long) bt * a.ndm_out + ((long) brev_bits(blk, a.amb_rank) << RA) + pf_dm) * a.M;
            pf_rows = (Ts *) a.pf + rowbase * a.pf_cap;
            pf_slot = int((s0 + lane) & (a.pf_cap - 1));
            emit.cap = int(a.pf_cap);
        }

        for (int it = 0; it <= ntiles; it++) {
            if (it >= 1) {
                // Phase-b rows, and (E0) for step 0 (lag 0) each even row one sample earlier: the delay
                // line holds it (capacity >= P + 65), so no shuffle and no history are needed.
                float v[NB], b0[RT<RB>::NP];
                if constexpr (FB || (STAGE == 1 && RB >= 1)) {
                    // Step 0 while loading (pair (f, f + 1), lag-1 operand = row f one sample earlier,
                    // from the delay line), and in stage 2 the level-0 emission.
                    int cnt0 = 0, mb0 = 0;
                    if constexpr (STAGE == 2) {
                        emit.row0 = pf_rows + pf_slot;
                        pf_slot = (pf_slot + 32) & int(a.pf_cap - 1);
                        cnt0 = a.sb_count[0];
                        mb0 = a.sb_mbase[0];
                    }
#pragma unroll
                    for (int f = 0; f < NB; f += 2) {
                        const int2 t0 = tab_int2<NB>(rt + g * NB, f), t1 = tab_int2<NB>(rt + g * NB, f + 1);
                        const int lo0 = t0.y & 0xffff, cap0 = t0.y >> 16, lo1 = t1.y & 0xffff, cap1 = t1.y >> 16;
                        int q0 = t0.x + lane, q1 = t1.x + lane;
                        q0 = (q0 < lo0) ? (q0 + cap0) : q0;
                        q1 = (q1 < lo1) ? (q1 + cap1) : q1;
                        const int qm = (q0 == lo0) ? (q0 + cap0 - 1) : (q0 - 1);
                        const float x = ring[q0], y = ring[q1], xm = ring[qm];
                        if (STAGE == 2 && cnt0 > 0) {
                            if (f < cnt0) emit(mb0 + f, tree_out(x, SA));
                            if (f + 1 < cnt0) emit(mb0 + f + 1, tree_out(y, SA));
                        }
                        v[f] = bfly_n<NORM_B>(x, y);
                        v[f + 1] = bfly_n<NORM_B>(xm, y);
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < NB; f++) {
                        const int2 t = tab_int2<NB>(rt + g * NB, f);
                        const int lo = t.y & 0xffff, cap = t.y >> 16;
                        int q = t.x + lane;
                        q = (q < lo) ? (q + cap) : q;
                        v[f] = ring[q];
                        if (E0 && (f & 1) == 0 && RB > 0) {
                            const int qm = (q == lo) ? (q + cap - 1) : (q - 1);
                            b0[f >> 1] = ring[qm];
                        }
                    }
                }
                __syncwarp();
                if (lane < NB) {
                    const int rr = g * NB + lane;   // row (f = lane, d = g)
                    const int2 t = rt[rr];
                    const int lo = t.y & 0xffff, cap = t.y >> 16;
                    const int x = t.x + 32;
                    rt[rr].x = (x >= lo + cap - ring_lag<RA, RB>(lane, g)) ? (x - cap) : x;
                }
                if constexpr (STAGE == 1) {
                    if constexpr (RB >= 1)
                        rt_steps<RB, HSB, true, true, NORM_B>(v, pvb, lane, hs);
                    else
                        rt_steps<RB, HSB, E0, false, NORM_B>(v, pvb, lane, hs, b0);
                    Ts *out = (Ts *) a.ring + (long) bt * a.ring_beam_stride + a.ring_off[(long) blk * NR];
#pragma unroll
                    for (int f = 0; f < NB; f++)
                        out[tab_int<NB>(out_base + g * NB, f) + lane] = from_f<Ts>(tree_out(v[f], SU));
                    __syncwarp();
                    if (lane < NB) {
                        const int i = g * NB + lane;
                        const int ob = out_base[i] + 32;
                        out_base[i] = (ob == out_off[i] + in_cap[i]) ? out_off[i] : ob;
                    }
                } else if constexpr (FB) {
                    phase_b_subbands<RB, STAG, HSB, true, true, SA, NORM_B>(v, pvb, psb, a, lane, emit, hs, b0);
                } else {
                    emit.row0 = pf_rows + pf_slot;
                    pf_slot = (pf_slot + 32) & int(a.pf_cap - 1);
                    phase_b_subbands<RB, STAG, HSB, E0, false, SA, NORM_B>(v, pvb, psb, a, lane, emit, hs, b0);
                }
            }
            asm volatile("bar.sync 1, %0;" :: "r"(blockDim.x) : "memory");
        }
        rt_save<RB, HSB, EB>(pvb, stb, lane, hs);
        if (STAG) st_save<RB>(psb, stb + rt_state(RB), lane);
    }
    __syncthreads();

    if (st16) {
        for (int i = threadIdx.x; i < RING / 4; i += blockDim.x)
            reinterpret_cast<float4 *>(st)[i] = reinterpret_cast<const float4 *>(ring)[i];
    } else {
        for (int i = threadIdx.x; i < RING; i += blockDim.x)
            st[i] = ring[i];
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
constexpr int kPfMaxProfiles = 16;   // 1 + 3 log2(max_width), max_width <= 32

// Number of entries of boxcar level l in a window of len0 samples (level 0 = samples).
__device__ __forceinline__ int pf_nlev(int len0, int l, int dt) { return (len0 - (1 << l)) / dt + 1; }

template<typename Ts>
__device__ __forceinline__ float ld_f(const Ts *p) { return to_f(*p); }

// Loads multiplet row 'row' over the warp's window into lev[0..len0) and builds boxcar levels
// 1..L-1 after it with the reference recursion B_{l+1}[u] = B_l[r u] + B_l[r u + s].
template<typename Ts, int L>
__device__ __forceinline__ void pf_build(float *lev, int len0, int lane, int Dcore, const Ts *row, long s_base, long mask)
{
    for (int u = lane; u < len0; u += 32)
        lev[u] = to_f(row[(s_base + u) & mask]);
    __syncwarp();
    int off = 0;
#pragma unroll
    for (int l = 0; l + 1 < L; l++) {
        const int dt = min(Dcore, 1 << l), dt1 = min(Dcore, 1 << (l + 1));
        const int n = pf_nlev(len0, l, dt), n1 = pf_nlev(len0, l + 1, dt1);
        const int rr = dt1 / dt, ss = (1 << l) / dt;
        const float *src = lev + off;
        float *dst = lev + off + n;
        for (int u = lane; u < n1; u += 32)
            dst[u] = __fadd_rn(src[rr * u], src[rr * u + ss]);
        __syncwarp();
        off += n;
    }
}

// Group (level l, multiplet m) of one output time: the reference scans fine times 'is' and, per fine
// time, profiles p = 0 (level 0 only), 3l+1, 3l+2, 3l+3. Keeps the first maximum of the group.
template<bool P0>
__device__ __forceinline__ void pf_group(const float *x, int nsamp, int S, float w0, float w1, float w2, float w3,
                                         bool full, float &gmax, int &gidx)
{
    gmax = -1.0e30f;
    gidx = -1;
    if (S == 1) {
        float x0 = x[-3], x1 = x[-2], x2 = x[-1];
        for (int is = 0; is < nsamp; is++) {
            float x3 = x[is];
            if (P0) { float v = __fmul_rn(w0, x3); if (v > gmax) { gmax = v; gidx = 4 * is; } }
            if (full) {
                float hx3 = __fmul_rn(0.5f, x3);
                float v1 = __fmul_rn(w1, __fadd_rn(x2, x3));
                float v2 = __fmul_rn(w2, __fadd_rn(__fadd_rn(__fmul_rn(0.5f, x1), x2), hx3));
                float v3 = __fmul_rn(w3, __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(0.5f, x0), x1), x2), hx3));
                if (v1 > gmax) { gmax = v1; gidx = 4 * is + 1; }
                if (v2 > gmax) { gmax = v2; gidx = 4 * is + 2; }
                if (v3 > gmax) { gmax = v3; gidx = 4 * is + 3; }
            }
            x0 = x1; x1 = x2; x2 = x3;
        }
    } else {
        for (int is = 0; is < nsamp; is++) {
            float x0 = x[is - 3 * S], x1 = x[is - 2 * S], x2 = x[is - S], x3 = x[is];
            if (P0) { float v = __fmul_rn(w0, x3); if (v > gmax) { gmax = v; gidx = 4 * is; } }
            if (full) {
                float hx3 = __fmul_rn(0.5f, x3);
                float v1 = __fmul_rn(w1, __fadd_rn(x2, x3));
                float v2 = __fmul_rn(w2, __fadd_rn(__fadd_rn(__fmul_rn(0.5f, x1), x2), hx3));
                float v3 = __fmul_rn(w3, __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(0.5f, x0), x1), x2), hx3));
                if (v1 > gmax) { gmax = v1; gidx = 4 * is + 1; }
                if (v2 > gmax) { gmax = v2; gidx = 4 * is + 2; }
                if (v3 > gmax) { gmax = v3; gidx = 4 * is + 3; }
            }
        }
    }
}

// One warp per (beam, coarse dm, 32 consecutive output times). For each multiplet the warp stages
// the input window in shared memory and builds the boxcar levels (every boxcar sum has the
// reference's rounding); each lane then scans the trials of its output time. Across groups the
// winner is the first group, in the reference's scan order (level, multiplet), whose maximum equals
// the overall maximum; within a group the first trial reaching it. This reproduces
// ReferencePeakFindingKernel::apply's strict-'>' sequential scan (src_lib/PeakFindingKernel.cu:339-420).
template<typename Ts, int L>
__global__ void __launch_bounds__(kPfWarps * 32) pf_kernel(PfArgs a, int warp_floats)
{
    const long s0 = a.chunk_ctr ? *a.chunk_ctr * (long) a.nt_chunk : a.s0;
    extern __shared__ float sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int dm = blockIdx.y * kPfWarps + warp;
    const int b = blockIdx.z, bt = a.beam0 + b;
    const int tout0 = blockIdx.x * 32;
    if (dm >= a.ndm_out)
        return;   // whole warp exits; warps never synchronize across the block

    const int ntw = min(32, a.nt_out - tout0);
    const int len0 = ntw * a.Dout + a.tpad;
    float *lev = sm + warp * warp_floats;

    const int tout = tout0 + lane;
    const bool active = (lane < ntw);
    const int Wds = a.ndm_out / a.ndm_wt, Tds = a.nt_out / a.nt_wt;
    const float *wp = a.wt + ((((long) b * a.ndm_wt + dm / Wds) * a.nt_wt + (active ? tout / Tds : 0)) * a.P) * a.N;
    const Ts *pfrows = (const Ts *) a.pf + ((long) bt * a.ndm_out + dm) * a.M * a.pf_cap;
    const long mask = a.pf_cap - 1;
    const long s_base = s0 + (long) tout0 * a.Dout - a.tpad;
    const bool full = (a.P > 1);

    float best = -1.0e30f;
    int win = 0x7fffffff;     // (l * M + m) * 256 + in-group index of the winning trial

    for (int m = 0; m < a.M; m++) {
        pf_build<Ts, L>(lev, len0, lane, a.Dcore, pfrows + (long) m * a.pf_cap, s_base, mask);
        if (active) {
            const int n = a.m_to_n[m];
            int off = 0;
#pragma unroll
            for (int l = 0; l < L; l++) {
                const int dt = min(a.Dcore, 1 << l), S = (1 << l) / dt, nsamp = a.Dout / dt;
                const int I = (a.tpad + dt - (1 << l)) / dt;
                const float *x = lev + off + I + lane * nsamp;
                float w0 = (l == 0) ? wp[n] : 0.0f, w1 = 0.0f, w2 = 0.0f, w3 = 0.0f;
                if (full) {
                    w1 = wp[(3 * l + 1) * a.N + n];
                    w2 = wp[(3 * l + 2) * a.N + n];
                    w3 = wp[(3 * l + 3) * a.N + n];
                }
                float gmax;
                int gidx;
                if (l == 0) pf_group<true>(x, nsamp, S, w0, w1, w2, w3, full, gmax, gidx);
                else pf_group<false>(x, nsamp, S, w0, w1, w2, w3, full, gmax, gidx);
                const int g = ((l * a.M + m) << 8) + gidx;
                if (gidx >= 0 && (gmax > best || (gmax == best && g < win))) { best = gmax; win = g; }
                off += pf_nlev(len0, l, dt);
            }
        }
        __syncwarp();
    }

    if (active) {
        uint32_t tok = 0xffffffffu;
        if (win != 0x7fffffff) {
            const int gi = win & 255, grp = win >> 8;
            const int l = grp / a.M, m = grp % a.M;
            const int dt = min(a.Dcore, 1 << l);
            const int is = gi >> 2, q = gi & 3;
            const int p = (q == 0) ? 0 : (3 * l + q);
            tok = (uint32_t(m) << 16) | (uint32_t(p) << 8) | uint32_t(is * dt);
        }
        long o = ((long) b * a.ndm_out + dm) * a.nt_out + tout;
        ((Ts *) a.out_max)[o] = from_f<Ts>(best);
        a.out_argmax[o] = tok;
    }
}


// -------------------------------------------------------------------------------------------------
// Fast peak finding (output time downsampling Dout >= 4; the general kernel above covers the rest).
//
// Same work split (one warp per beam, coarse dm and 32 output times; lane = output time) and the same
// results, organised around four changes:
//
//  1. Bank-conflict-free shared memory. Level l of the boxcar window is stored in blocks of nsamp_l
//     entries (one block per lane: its output time's fine samples). Levels scanned in pairs with
//     blocks of >= 4 entries pad each block with 2 floats, so the 32 blocks fall on distinct banks
//     for 8-byte loads; the other levels are contiguous and are read in pairs or single floats.
//  2. Levels are built while they are scanned: while a lane scans its fine samples at level l two at
//     a time, the pair's sum is its level-(l+1) entry (B_{l+1}[u] = B_l[2u] + B_l[2u+1] while
//     dt doubles), so only the pad region before the first output time and the levels with
//     saturated time step (dt = Dcore) are built in a separate pass.
//  3. Max-only trial loop. The scan keeps, per group (level, multiplet), the maximum trial value
//     (fmaxf and the three-input max, which ignore NaN as the reference's strict '>' does) and the
//     first fine sample (pair) reaching it; across groups, the first group in the reference's
//     (level, multiplet) order whose maximum equals the overall one. After each multiplet, a lane
//     whose maximum moved into it recomputes that fine sample's (pair's) trials from shared memory
//     and takes the first, in (fine time, profile) order, equal to the maximum: its value and token
//     are the outputs.
//  4. The next multiplet's window is staged in shared memory with cp.async while the current one is
//     scanned.

// Per-level constants of the fast peak finder (host-computed; level l has time step dt, boxcar
// length 2^l = S*dt, and nsamp = Dout/dt fine samples per output time).
enum { kPfU = 1, kPfPairs = 2, kPfNextU = 4 };
struct PfGeom
{
    int off[kPfMaxLevels];   // first float of level l in a warp's region (even)
    int e[kPfMaxLevels];     // entry i lies in block (i + e) >> k
    int k[kPfMaxLevels];     // log2(nsamp_l)
    int pad[kPfMaxLevels];   // floats after each block
    int I[kPfMaxLevels];     // entry of the warp's first output time's first fine sample
    int n[kPfMaxLevels];     // entries of level l in the window of 32 output times
    int dt[kPfMaxLevels], S[kPfMaxLevels], nsamp[kPfMaxLevels];
    int rr[kPfMaxLevels], ss[kPfMaxLevels];   // B_l[u] = B_{l-1}[rr u] + B_{l-1}[rr u + ss]
    int flags[kPfMaxLevels]; // kPfU: dt = 2^l; kPfPairs: scanned two fine samples at a time;
                             // kPfNextU: level l+1 has dt = 2^(l+1) and is built by this level's scan
    int raw_off;             // two staging buffers of the window's raw samples (16-byte aligned), one per
    int raw_floats;          // multiplet in flight, raw_floats apart; level 0 is read from them directly
    int w_off;               // the warp's weights of one subband, [profile < 16][weight time < 32]
    int warp_floats;
};

// max(a, b, c) ignoring NaN inputs (sm_100 three-input max).
__device__ __forceinline__ float pf_max3(float a, float b, float c)
{
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

__device__ __forceinline__ int pf_phys(const PfGeom &g, int l, int i)
{
    const int t = i + g.e[l];
    return g.off[l] + t + g.pad[l] * (t >> g.k[l]);
}

template<typename Ts> __device__ __forceinline__ void pf_load4(const Ts *p, float (&v)[4]);
template<> __device__ __forceinline__ void pf_load4<float>(const float *p, float (&v)[4])
{
    const float4 q = *(const float4 *) p;
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
template<> __device__ __forceinline__ void pf_load4<__half>(const __half *p, float (&v)[4])
{
    const uint2 q = *(const uint2 *) p;
    const float2 a = __half22float2(*(const __half2 *) &q.x), b = __half22float2(*(const __half2 *) &q.y);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
template<> __device__ __forceinline__ void pf_load4<__nv_bfloat16>(const __nv_bfloat16 *p, float (&v)[4])
{
    const uint2 q = *(const uint2 *) p;
    const float2 a = __bfloat1622float2(*(const __nv_bfloat162 *) &q.x), b = __bfloat1622float2(*(const __nv_bfloat162 *) &q.y);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
// Eight samples from a 16-byte-aligned address (two 4-sample loads for fp32).
template<typename Ts> __device__ __forceinline__ void pf_load8(const Ts *p, float (&v)[8])
{
    if constexpr (sizeof(Ts) == 4) {
        float a[4], b[4];
        pf_load4<Ts>(p, a);
        pf_load4<Ts>(p + 4, b);
#pragma unroll
        for (int i = 0; i < 4; i++) { v[i] = a[i]; v[4 + i] = b[i]; }
    } else {
        const uint4 q = *(const uint4 *) p;
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            float2 f;
            if constexpr (std::is_same<Ts, __half>::value) f = __half22float2(*(const __half2 *) &w[i]);
            else f = __bfloat1622float2(*(const __nv_bfloat162 *) &w[i]);
            v[2 * i] = f.x; v[2 * i + 1] = f.y;
        }
    }
}

// Shared-memory layout of the fast peak finder for one warp (see PfGeom).
// LW: output times (lanes) per coarse DM in a warp (32, or 16 and 8 for trees with that few output
// times per chunk: 32 / LW coarse DMs then share a warp).
__host__ __device__ constexpr PfGeom pf_geom(int Dout, int Dcore, int tpad, int L, int esize, int LW = 32)
{
    PfGeom g{};
    int off = 0;
    for (int l = 0; l < L; l++) {
        const int dt = (Dcore < (1 << l)) ? Dcore : (1 << l);
        const int nsamp = Dout / dt;
        const bool pairs = ((1 << l) <= Dcore) && nsamp >= 2;
        const int I = (tpad + dt - (1 << l)) / dt;
        int k = 0;
        while ((1 << k) < nsamp) k++;
        g.off[l] = off;
        g.e[l] = (nsamp - I % nsamp) % nsamp;
        g.k[l] = k;
        // Levels scanned in pairs from per-lane blocks: 2 floats after each block of >= 4 (the
        // blocks then fall on distinct banks for 8-byte loads); the others are stored contiguously.
        g.pad[l] = (pairs && nsamp >= 4) ? 2 : 0;
        g.I[l] = I;
        g.n[l] = LW * nsamp + I;
        g.dt[l] = dt;
        g.S[l] = (1 << l) / dt;
        g.nsamp[l] = nsamp;
        if (l > 0) {
            const int dtp = (Dcore < (1 << (l - 1))) ? Dcore : (1 << (l - 1));
            g.rr[l] = dt / dtp;
            g.ss[l] = (1 << (l - 1)) / dtp;
        }
        g.flags[l] = (((1 << l) <= Dcore) ? kPfU : 0) | (pairs ? kPfPairs : 0)
                   | ((l + 1 < L && (2 << l) <= Dcore) ? kPfNextU : 0);
        const int t = g.n[l] - 1 + g.e[l];
        const int size = t + g.pad[l] * (t >> k) + 1;
        if (l > 0)   // level 0 lives only in the raw staging buffer
            off += (size + 1) & ~1;
    }
    g.raw_off = (off + 3) & ~3;
    g.raw_floats = ((LW * Dout + tpad) * esize + 15) / 16 * 4;
    g.w_off = g.raw_off + 2 * g.raw_floats;
    g.warp_floats = g.w_off + kPfMaxProfiles * 32;
    return g;
}

// Peak-finder constants fixed by the plan rules: Dcore = min(Dout, 8) and tpad = max(2 Wmax, 4) with
// L = max(log2 Wmax, 1), i.e. tpad = max(2^(L+1), 4).
__host__ __device__ constexpr int pf_dcore_of(int Dout) { return Dout < 8 ? Dout : 8; }
__host__ __device__ constexpr int pf_tpad_of(int L) { return (2 << L) > 4 ? (2 << L) : 4; }

// The kernel body. g holds the per-level constants (a compile-time constant object when DOUT > 0, so
// the unrolled level loop sees them as immediates); gr is the same geometry passed at launch, used
// where the level is only known at run time.
// CTR: the chunk index comes from the device counter (replayed CUDA graphs). It is a template flag
// because reading it costs the kernel about 26 registers, which the direct launches should not pay.
template<typename Ts, int L, int DOUT, bool CTR, int LW>
__device__ __forceinline__ void pf_fast_body(const PfArgs &a, const PfGeom &g, const PfGeom &gr)
{
    static_assert(LW == 32 || LW == 16 || LW == 8, "lanes per coarse DM");
    constexpr int G = 32 / LW;   // coarse DMs per warp, each on LW consecutive lanes
    extern __shared__ float sm[];
    const int warp = threadIdx.x >> 5, sub = (threadIdx.x & 31) / LW, lane = threadIdx.x & (LW - 1);
    const int dm0 = (blockIdx.y * kPfWarps + warp) * G;
    const int b = blockIdx.z, bt = a.beam0 + b;
    const int tout0 = blockIdx.x * LW;
    if (dm0 >= a.ndm_out)
        return;   // whole warp exits; warps never synchronize across the block
    // A sub-group past the last coarse DM computes the last one again and stores nothing.
    const bool dm_ok = dm0 + sub < a.ndm_out;
    const int dm = dm_ok ? dm0 + sub : a.ndm_out - 1;

    const int ntw = min(LW, a.nt_out - tout0);
    const int tout = tout0 + lane;
    const bool active = (lane < ntw) && dm_ok;
    float *lev = sm + (warp * G + sub) * g.warp_floats;

    const int Dout = (DOUT > 0) ? DOUT : a.Dout;
    const int tpad = (DOUT > 0) ? pf_tpad_of(L) : a.tpad;
    const int Wds = a.ndm_out / a.ndm_wt, Tds = a.nt_out / a.nt_wt;
    // Weights of one subband for the warp's weight times tw0 .. tw0 + NT - 1, staged in shared memory
    // as wsm[p * 32 + j] (lanes of one weight time read the same word, consecutive weight times
    // consecutive words), and reloaded only when a multiplet's subband differs from the previous one.
    const float *wrow = a.wt + ((long) b * a.ndm_wt + dm / Wds) * a.nt_wt * a.P * a.N;
    const int tw0 = tout0 / Tds, NT = (Tds >= LW) ? 1 : LW / Tds;
    const int tl = (lane < ntw) ? (tout / Tds - tw0) : 0;
    float *wsm = lev + g.w_off;
    int wsm_n = -1;
    const Ts *pfrows = (const Ts *) a.pf + ((long) bt * a.ndm_out + dm) * a.M * a.pf_cap;
    const int mask = int(a.pf_cap - 1);
    // Window sample 0 (stream time s0 + 32 tile * Dout - tpad, a multiple of 4), as a delay-line slot.
    long s0 = a.s0;
    if constexpr (CTR) s0 = *a.chunk_ctr * (long) a.nt_chunk;
    const int sbm = int((s0 + (long) tout0 * Dout - tpad) & (a.pf_cap - 1));
    const bool full = (L > 1) || (a.P > 1);
    const int nq0 = (ntw * Dout + tpad) >> 2;   // samples the active lanes read (a partial last tile reads fewer)

    float best = -1.0e30f;
    int winG = -1;            // group l * M + m of the first maximum; -1: no trial above -1e30
    float outv = best;        // value and token of the first maximal trial
    uint32_t tok = 0xffffffffu;
    // Inputs of the winning group's first maximal pair, saved when the maximum moves, so that the
    // token is found once at the end: x[j - 3S .. j] of its samples is = winP (a) and winP + 1 (b),
    // the level's weights, and the pair's level, multiplet and start.
    float xa0 = 0, xa1 = 0, xa2 = 0, xa3 = 0, xb0 = 0, xb1 = 0, xb2 = 0, xb3 = 0;
    float sw0 = 0, sw1 = 0, sw2 = 0, sw3 = 0;
    int winL = 0, winM = 0, winP = 0;

    // The window's raw samples are staged with cp.async one multiplet ahead into alternating buffers
    // (4-sample runs: a 4-aligned run never wraps the delay line). Level 0 is read from them.
    Ts *raw0 = (Ts *) (lev + g.raw_off);
    const int raw_ts = g.raw_floats * int(sizeof(float) / sizeof(Ts));
    auto stage = [&](int m) {
        const Ts *row = pfrows + (long) m * a.pf_cap;
        Ts *raw = raw0 + (m & 1) * raw_ts;
        for (int q = lane; q < nq0; q += LW)
            cp_async_bytes<4 * sizeof(Ts)>(raw + 4 * q, row + ((sbm + 4 * q) & mask));
        cp_async_commit();
    };
    stage(0);

    for (int m = 0; m < a.M; m++) {
        // Wait for this multiplet's samples; then stage the next one into the other buffer (every
        // lane is past its reads of that buffer: they came before this loop's previous barriers).
        cp_async_wait0();
        __syncwarp();
        if (m + 1 < a.M)
            stage(m + 1);
        const Ts *rawc = raw0 + (m & 1) * raw_ts;

        const int n = a.m_to_n[m];
        if (n != wsm_n) {
            for (int idx = lane; idx < a.P * NT; idx += LW) {
                const int p = idx / NT, j = idx - p * NT, t = tw0 + j;
                wsm[p * 32 + j] = (t < a.nt_wt) ? wrow[((long) t * a.P + p) * a.N + n] : 0.0f;
            }
            __syncwarp();
            wsm_n = n;
        }
#pragma unroll
        for (int l = 0; l < L; l++) {
            const int S = g.S[l], nsamp = g.nsamp[l];
            const bool U = g.flags[l] & kPfU;
            const bool nextU = (l + 1 < L) && (g.flags[l] & kPfNextU);

            if (l > 0 && !U) {
                // Saturated level (dt = Dcore): B_l[u] = B_{l-1}[rr u] + B_{l-1}[rr u + ss].
                const int rr = g.rr[l], ss = g.ss[l];
                for (int u = lane; u < g.n[l]; u += LW)
                    lev[pf_phys(g, l, u)] = __fadd_rn(lev[pf_phys(g, l - 1, rr * u)], lev[pf_phys(g, l - 1, rr * u + ss)]);
                __syncwarp();
            }
            if (nextU) {
                // Entries of level l+1 before the first output time.
                for (int u = lane; u < g.I[l + 1]; u += LW)
                    lev[pf_phys(g, l + 1, u)] = (l == 0) ? __fadd_rn(to_f(rawc[2 * u]), to_f(rawc[2 * u + 1]))
                                                        : __fadd_rn(lev[pf_phys(g, l, 2 * u)], lev[pf_phys(g, l, 2 * u + 1)]);
            }

            float w0 = 0.0f, w1 = 0.0f, w2 = 0.0f, w3 = 0.0f;
            if (l == 0) w0 = wsm[tl];
            if (full) {
                w1 = wsm[(3 * l + 1) * 32 + tl];
                w2 = wsm[(3 * l + 2) * 32 + tl];
                w3 = wsm[(3 * l + 3) * 32 + tl];
            }

            const int j0 = g.I[l] + lane * nsamp;
            float gmax = -1.0e30f;
            int gp = 0;   // first fine sample (pair start) whose trials reach gmax
            if (g.flags[l] & kPfPairs) {
                // x0..x3 = x[is-3..is]; carried: x2, hx1 = x[is-2]/2, hx2 = x[is-1]/2, Ap = x[is-3]/2 + x[is-2].
                // Level 0 comes from the raw staging buffer (entry i = raw sample i; j0 is a multiple of 4).
                float x2, x1, x0;
                if (l == 0) {
                    float q[4];
                    pf_load4<Ts>(rawc + j0 - 4, q);
                    x0 = q[1]; x1 = q[2]; x2 = q[3];
                } else {
                    x2 = lev[pf_phys(g, l, j0 - 1)];
                    x1 = lev[pf_phys(g, l, j0 - 2)];
                    x0 = lev[pf_phys(g, l, j0 - 3)];
                }
                float2 H = make_float2(__fmul_rn(0.5f, x1), __fmul_rn(0.5f, x2));   // x[is-2]/2, x[is-1]/2
                float Ap = __fadd_rn(__fmul_rn(0.5f, x0), x1);
                const float *xs = lev + ((l > 0) ? pf_phys(g, l, j0) : 0);
                float *ys = lev + (nextU ? pf_phys(g, l + 1, g.I[l + 1] + lane * (nsamp >> 1)) : 0);
                const float2 W0 = make_float2(w0, w0), W1 = make_float2(w1, w1);
                const float2 W2 = make_float2(w2, w2), W3 = make_float2(w3, w3);

                // The trials of fine samples is (xa) and is + 1 (xb).
                auto pair = [&](const float xa, const float xb, const int is) {
                    const float2 X = make_float2(xa, xb);
                    float mx;
                    if (full) {
                        // Fine samples is (xa) and is+1 (xb), in packed pairs (a, b): profiles
                        // y1 = x2+x3, y2 = (x1/2+x2)+x3/2, y3 = ((x0/2+x1)+x2)+x3/2 with the reference's
                        // association; A = x1/2+x2 of each sample, and y3's (x0/2+x1) is the previous A.
                        const float2 Hn = f2mul(make_float2(0.5f, 0.5f), X);
                        const float2 Pr = make_float2(x2, xa);       // x[is-1], x[is]
                        const float2 A = f2add(H, Pr);
                        const float2 V1 = f2mul(W1, f2add(Pr, X));
                        const float2 V2 = f2mul(W2, f2add(A, Hn));
                        const float2 V3 = f2mul(W3, f2add(f2add(make_float2(Ap, A.x), Pr), Hn));
                        if (l == 0) {
                            const float2 V0 = f2mul(W0, X);
                            mx = fmaxf(pf_max3(V0.x, V1.x, V2.x), pf_max3(V3.x, V0.y, V1.y));
                            mx = pf_max3(mx, V2.y, V3.y);
                        } else {
                            mx = fmaxf(pf_max3(V1.x, V2.x, V3.x), pf_max3(V1.y, V2.y, V3.y));
                        }
                        H = Hn; x2 = xb; Ap = A.y;
                    } else {
                        mx = fmaxf(__fmul_rn(w0, xa), __fmul_rn(w0, xb));
                    }
                    if (mx > gmax) { gmax = mx; gp = is; }
                    if (nextU) ys[is >> 1] = __fadd_rn(xa, xb);
                };
                if (l == 0) {
                    // 16-byte loads when runs of 8 stay 16-byte aligned (tpad and Dout multiples of 8)
                    if (DOUT > 0 && nsamp % 8 == 0 && pf_tpad_of(L) % 8 == 0) {
                        for (int is = 0; is < nsamp; is += 8) {
                            float q[8];
                            pf_load8<Ts>(rawc + j0 + is, q);
                            pair(q[0], q[1], is);
                            pair(q[2], q[3], is + 2);
                            pair(q[4], q[5], is + 4);
                            pair(q[6], q[7], is + 6);
                        }
                    } else {
                        for (int is = 0; is < nsamp; is += 4) {
                            float q[4];
                            pf_load4<Ts>(rawc + j0 + is, q);
                            pair(q[0], q[1], is);
                            pair(q[2], q[3], is + 2);
                        }
                    }
                } else {
#pragma unroll 2
                    for (int is = 0; is < nsamp; is += 2) {
                        const float2 X = *(const float2 *) (xs + is);
                        pair(X.x, X.y, is);
                    }
                }
            } else {
                // Levels stored without padding (contiguous across lanes): x[j - k S] = xb[is - k S].
                const float *xb = lev + pf_phys(g, l, j0);
                if (nsamp >= 2) {
                    // Two fine samples at a time (S and nsamp even: 8-byte aligned pairs).
                    for (int is = 0; is < nsamp; is += 2) {
                        const float2 p3 = *(const float2 *) (xb + is), p2 = *(const float2 *) (xb + is - S);
                        const float2 p1 = *(const float2 *) (xb + is - 2 * S), p0 = *(const float2 *) (xb + is - 3 * S);
                        float mx;
                        if (full) {
                            const float ha = __fmul_rn(0.5f, p3.x), hb = __fmul_rn(0.5f, p3.y);
                            const float v1a = __fmul_rn(w1, __fadd_rn(p2.x, p3.x));
                            const float v2a = __fmul_rn(w2, __fadd_rn(__fadd_rn(__fmul_rn(0.5f, p1.x), p2.x), ha));
                            const float v3a = __fmul_rn(w3, __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(0.5f, p0.x), p1.x), p2.x), ha));
                            const float v1b = __fmul_rn(w1, __fadd_rn(p2.y, p3.y));
                            const float v2b = __fmul_rn(w2, __fadd_rn(__fadd_rn(__fmul_rn(0.5f, p1.y), p2.y), hb));
                            const float v3b = __fmul_rn(w3, __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(0.5f, p0.y), p1.y), p2.y), hb));
                            mx = fmaxf(pf_max3(v1a, v2a, v3a), pf_max3(v1b, v2b, v3b));
                            if (l == 0) mx = pf_max3(mx, __fmul_rn(w0, p3.x), __fmul_rn(w0, p3.y));
                        } else {
                            mx = fmaxf(__fmul_rn(w0, p3.x), __fmul_rn(w0, p3.y));
                        }
                        if (mx > gmax) { gmax = mx; gp = is; }
                    }
                } else {
                    const float x3 = xb[0];
                    float v = (l == 0) ? __fmul_rn(w0, x3) : -1.0e30f;
                    if (full) {
                        const float x0 = xb[-3 * S], x1 = xb[-2 * S], x2 = xb[-S];
                        const float hx3 = __fmul_rn(0.5f, x3);
                        const float y1 = __fadd_rn(x2, x3);
                        const float y2 = __fadd_rn(__fadd_rn(__fmul_rn(0.5f, x1), x2), hx3);
                        const float y3 = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(0.5f, x0), x1), x2), hx3);
                        v = fmaxf(v, pf_max3(__fmul_rn(w1, y1), __fmul_rn(w2, y2), __fmul_rn(w3, y3)));
                    }
                    if (v > gmax) { gmax = v; gp = 0; }
                }
            }
            __syncwarp();

            const int G = l * a.M + m;
            if (gmax > best || (gmax == best && G < winG)) {
                best = gmax;
                winG = G;
                winL = l;
                winM = m;
                winP = gp;
                const int S = g.S[l];
                const int j = g.I[l] + lane * nsamp + gp;
                // level l's entry i (level 0: the raw sample)
                auto X = [&](int i) { return (l == 0) ? to_f(rawc[i]) : lev[pf_phys(g, l, i)]; };
                xa3 = X(j);
                if (full) {
                    xa2 = X(j - S);
                    xa1 = X(j - 2 * S);
                    xa0 = X(j - 3 * S);
                }
                if (gp + 1 < nsamp) {
                    xb3 = X(j + 1);
                    if (full) {
                        xb2 = X(j + 1 - S);
                        xb1 = X(j + 1 - 2 * S);
                        xb0 = X(j + 1 - 3 * S);
                    }
                }
                sw0 = w0; sw1 = w1; sw2 = w2; sw3 = w3;
            }
        }

    }

    // The first trial of the winning pair, in the reference's order (fine time, then profile 0, 3l+1,
    // 3l+2, 3l+3), equal to the maximum gives the output value and token.
    if (winG >= 0) {
        const int l = winL;
        const uint32_t dt = uint32_t(gr.dt[l]);
        const int nsamp = gr.nsamp[l];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            if (k == 1 && winP + 1 >= nsamp) break;
            const float x3 = k ? xb3 : xa3, x2 = k ? xb2 : xa2, x1 = k ? xb1 : xa1, x0 = k ? xb0 : xa0;
            const uint32_t tk0 = (uint32_t(winM) << 16) | (uint32_t(winP + k) * dt);
            if (l == 0) {
                const float v0 = __fmul_rn(sw0, x3);
                if (v0 == best) { outv = v0; tok = tk0; break; }
            }
            if (full) {
                const float hx3 = __fmul_rn(0.5f, x3);
                const float v1 = __fmul_rn(sw1, __fadd_rn(x2, x3));
                const float v2 = __fmul_rn(sw2, __fadd_rn(__fadd_rn(__fmul_rn(0.5f, x1), x2), hx3));
                const float v3 = __fmul_rn(sw3, __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(0.5f, x0), x1), x2), hx3));
                if (v1 == best) { outv = v1; tok = tk0 | (uint32_t(3 * l + 1) << 8); break; }
                if (v2 == best) { outv = v2; tok = tk0 | (uint32_t(3 * l + 2) << 8); break; }
                if (v3 == best) { outv = v3; tok = tk0 | (uint32_t(3 * l + 3) << 8); break; }
            }
        }
    }

    if (!active)
        return;
    const long o = ((long) b * a.ndm_out + dm) * a.nt_out + tout;
    ((Ts *) a.out_max)[o] = from_f<Ts>(outv);
    a.out_argmax[o] = tok;
}

// DOUT > 0: compiled for that output time downsampling (with Dcore = min(DOUT, 8) and the plan's tpad
// for L levels); DOUT = 0: any Dout >= 4, geometry read from the launch arguments.
template<typename Ts, int L, int DOUT, bool CTR, int LW = 32>
__global__ void __launch_bounds__(kPfWarps * 32) pf_fast_kernel(PfArgs a, PfGeom gr)
{
    if constexpr (DOUT > 0) {
        constexpr PfGeom gc = pf_geom(DOUT, pf_dcore_of(DOUT), pf_tpad_of(L), L, sizeof(Ts), LW);
        pf_fast_body<Ts, L, DOUT, CTR, LW>(a, gc, gr);
    } else {
        pf_fast_body<Ts, L, 0, CTR, LW>(a, gr, gr);
    }
}


// -------------------------------------------------------------------------------------------------
// Host launchers.


template<typename Ts, int NLEV>
static void launch_grid_lds_t(const GridLdsArgs &a, cudaStream_t s)
{
    constexpr int W0 = ((1 << NLEV) > 8) ? (1 << NLEV) : 8;
    if (a.T % W0) throw std::runtime_error("grid_lds_kernel: chunk length not a multiple of the window");
    const long nwin = a.T / W0;
    long nthr = nwin * (1L << (a.rank - 1)) * a.B;
    // Blocks start at a window 0 (a multiple of nwin threads, about 128), so that every other window's
    // predecessor is computed in the same block.
    const int target = (a.block_target > 0) ? std::min(a.block_target, kGridMaxThreads) : 128;
    int bd = (nwin <= target) ? int(nwin * (target / nwin)) : (nwin <= kGridMaxThreads ? int(nwin) : kGridMaxThreads);
    if (a.q_data) {
        if (a.T % 256) throw std::runtime_error("grid_lds_kernel: int4 input needs a chunk length that is a multiple of 256");
        grid_lds_kernel<Ts, NLEV, true><<<(unsigned) ((nthr + bd - 1) / bd), bd, 0, s>>>(a);
    } else {
        grid_lds_kernel<Ts, NLEV, false><<<(unsigned) ((nthr + bd - 1) / bd), bd, 0, s>>>(a);
    }
    check_launch("grid_lds_kernel");
}

template<typename Ts>
static void launch_grid_lds_d(const GridLdsArgs &a, cudaStream_t s)
{
    switch (a.nlev) {
    case 0: launch_grid_lds_t<Ts, 0>(a, s); break;
    case 1: launch_grid_lds_t<Ts, 1>(a, s); break;
    case 2: launch_grid_lds_t<Ts, 2>(a, s); break;
    case 3: launch_grid_lds_t<Ts, 3>(a, s); break;
    case 4: launch_grid_lds_t<Ts, 4>(a, s); break;
    case 5: launch_grid_lds_t<Ts, 5>(a, s); break;
    case 6: launch_grid_lds_t<Ts, 6>(a, s); break;
    default: throw std::runtime_error("grid_lds_kernel: unsupported number of levels");
    }
}

void launch_grid_lds(const GridLdsArgs &a, int dtype, cudaStream_t s)
{
    if (a.rank < 1) throw std::runtime_error("grid_lds_kernel: tree rank must be >= 1");
    if (dtype == 0) launch_grid_lds_d<float>(a, s);
    else if (dtype == 1) launch_grid_lds_d<__half>(a, s);
    else launch_grid_lds_d<__nv_bfloat16>(a, s);
}

template<typename Ts, int RA, int RB>
static size_t tree_smem()
{
    return TreeSmem<Ts, RA, RB>::total;
}

template<typename K>
static void set_smem(K kernel, size_t bytes)
{
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) bytes);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
}

template<typename Ts, int R, int STAGE, bool STAG, typename A>
static void launch_tree_r(const A &a, int nblocks, int B, cudaStream_t s)
{
    constexpr int RA = split_ra(R), RB = split_rb(R);
    size_t sm = tree_smem<Ts, RA, RB>();
    set_smem(tree_kernel<Ts, RA, RB, STAGE, STAG>, sm);
    tree_kernel<Ts, RA, RB, STAGE, STAG><<<dim3(nblocks, B), tree_threads(R), sm, s>>>(a);
    check_launch(STAGE == 1 ? "stage1 tree_kernel" : "stage2 tree_kernel");
}

template<typename Ts, int STAGE, bool STAG, typename A>
static void launch_tree_t(const A &a, int rank, int nblocks, int B, cudaStream_t s)
{
    switch (rank) {
    case 1: launch_tree_r<Ts, 1, STAGE, STAG>(a, nblocks, B, s); break;
    case 2: launch_tree_r<Ts, 2, STAGE, STAG>(a, nblocks, B, s); break;
    case 3: launch_tree_r<Ts, 3, STAGE, STAG>(a, nblocks, B, s); break;
    case 4: launch_tree_r<Ts, 4, STAGE, STAG>(a, nblocks, B, s); break;
    case 5: launch_tree_r<Ts, 5, STAGE, STAG>(a, nblocks, B, s); break;
    case 6: launch_tree_r<Ts, 6, STAGE, STAG>(a, nblocks, B, s); break;
    case 7: launch_tree_r<Ts, 7, STAGE, STAG>(a, nblocks, B, s); break;
    case 8: launch_tree_r<Ts, 8, STAGE, STAG>(a, nblocks, B, s); break;
    default: throw std::runtime_error("tree_kernel: unsupported dd rank " + std::to_string(rank));
    }
}

void launch_stage1(const Stage1Args &a, int dtype, int nblocks, int B, cudaStream_t s)
{
    if (a.in_lag0 != 0 || a.in_lag1 != 0) throw std::runtime_error("launch_stage1: input rows must be aligned (no read lag)");
    if (dtype == 0) launch_tree_t<float, 1, false>(a, a.rank, nblocks, B, s);
    else if (dtype == 1) launch_tree_t<__half, 1, false>(a, a.rank, nblocks, B, s);
    else launch_tree_t<__nv_bfloat16, 1, false>(a, a.rank, nblocks, B, s);
}

static bool stage2_staggered(const Stage2Args &a)
{
    bool stag = false;
    for (int l = 1; l < 5; l++) stag = stag || (a.sb_count[l] >= 2);
    return stag;
}

bool stage2_same_kernel(const Stage2Args &x, const Stage2Args &y)
{
    return x.rank == y.rank && stage2_staggered(x) == stage2_staggered(y);
}

void launch_stage2_multi(const Stage2Args *a, const int *nblocks, int n, int dtype, int B, cudaStream_t s)
{
    if (n < 1 || n > kStage2MaxTrees) throw std::runtime_error("launch_stage2_multi: bad tree count " + std::to_string(n));
    Stage2Multi m;
    memset(&m, 0, sizeof(m));
    m.n = n;
    long tot = 0;
    for (int i = 0; i < n; i++) {
        if (!stage2_same_kernel(a[0], a[i])) throw std::runtime_error("launch_stage2_multi: trees need different kernels");
        if (nblocks[i] < 1) throw std::runtime_error("launch_stage2_multi: bad block count");
        m.t[i] = a[i];
        m.blk0[i] = int(tot);
        tot += nblocks[i];
    }
    if (tot > (1L << 30)) throw std::runtime_error("launch_stage2_multi: grid too large");
    m.blk0[n] = int(tot);
    if (stage2_staggered(a[0])) {
        if (dtype == 0) launch_tree_t<float, 2, true>(m, a[0].rank, int(tot), B, s);
        else if (dtype == 1) launch_tree_t<__half, 2, true>(m, a[0].rank, int(tot), B, s);
        else launch_tree_t<__nv_bfloat16, 2, true>(m, a[0].rank, int(tot), B, s);
    } else {
        if (dtype == 0) launch_tree_t<float, 2, false>(m, a[0].rank, int(tot), B, s);
        else if (dtype == 1) launch_tree_t<__half, 2, false>(m, a[0].rank, int(tot), B, s);
        else launch_tree_t<__nv_bfloat16, 2, false>(m, a[0].rank, int(tot), B, s);
    }
}

void launch_stage2(const Stage2Args &a, int dtype, int nblocks, int B, cudaStream_t s)
{
    launch_stage2_multi(&a, &nblocks, 1, dtype, B, s);
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


// The fast kernel needs 4-sample runs of the window (Dout >= 4, tpad and s0 multiples of 4).
static bool pf_fast_ok(const PfArgs &a)
{
    const long s0 = a.chunk_ctr ? (long) a.nt_chunk : a.s0;   // with a counter, s0 is a multiple of nt_chunk
    return !a.force_general && a.Dout >= 4 && (a.tpad % 4) == 0 && (s0 % 4) == 0 && (a.pf_cap % 4) == 0 && a.L <= 5 && a.P <= kPfMaxProfiles;
}

template<typename Ts, int L, int DOUT, int LW = 32>
static void launch_pf_fast(const PfArgs &a, const PfGeom &g, int B, cudaStream_t s)
{
    // g: the geometry for LW lanes per coarse DM
    constexpr int G = 32 / LW;
    size_t sm = (size_t) kPfWarps * G * g.warp_floats * sizeof(float);
    dim3 grid((a.nt_out + LW - 1) / LW, (a.ndm_out + kPfWarps * G - 1) / (kPfWarps * G), B);
    if (a.chunk_ctr) {
        set_smem(pf_fast_kernel<Ts, L, DOUT, true, LW>, sm);
        pf_fast_kernel<Ts, L, DOUT, true, LW><<<grid, kPfWarps * 32, sm, s>>>(a, g);
    } else {
        set_smem(pf_fast_kernel<Ts, L, DOUT, false, LW>, sm);
        pf_fast_kernel<Ts, L, DOUT, false, LW><<<grid, kPfWarps * 32, sm, s>>>(a, g);
    }
    check_launch("pf_fast_kernel");
}

template<typename Ts, int L>
static void launch_pf_l(const PfArgs &a, int B, cudaStream_t s)
{
    if (pf_fast_ok(a)) {
        const PfGeom g = pf_geom(a.Dout, a.Dcore, a.tpad, L, (int) sizeof(Ts));
        // Compiled geometries for the usual output downsamplings (pirate's default Dout = 2^pf_rank).
        const bool std_geom = (a.Dcore == pf_dcore_of(a.Dout)) && (a.tpad == pf_tpad_of(L));
        // Trees with 16 or 8 output times per chunk (the most downsampled primary trees) share a warp
        // between 2 or 4 coarse DMs, so that no lane idles (compiled for the benchmark's Dout 16, widths
        // to 32).
        if constexpr (L == 5) {
            if (std_geom && a.Dout == 16 && a.nt_out <= 8) {
                launch_pf_fast<Ts, L, 16, 8>(a, pf_geom(a.Dout, a.Dcore, a.tpad, L, (int) sizeof(Ts), 8), B, s);
                return;
            }
            if (std_geom && a.Dout == 16 && a.nt_out <= 16) {
                launch_pf_fast<Ts, L, 16, 16>(a, pf_geom(a.Dout, a.Dcore, a.tpad, L, (int) sizeof(Ts), 16), B, s);
                return;
            }
        }
        if (std_geom && a.Dout == 16) launch_pf_fast<Ts, L, 16>(a, g, B, s);
        else if (std_geom && a.Dout == 8) launch_pf_fast<Ts, L, 8>(a, g, B, s);
        else if (std_geom && a.Dout == 4) launch_pf_fast<Ts, L, 4>(a, g, B, s);
        else launch_pf_fast<Ts, L, 0>(a, g, B, s);
        return;
    }
    int wf = pf_warp_floats(a.Dout, a.tpad, a.Dcore, a.L);
    size_t sm = (size_t) kPfWarps * wf * sizeof(float);
    set_smem(pf_kernel<Ts, L>, sm);
    dim3 grid((a.nt_out + 31) / 32, (a.ndm_out + kPfWarps - 1) / kPfWarps, B);
    pf_kernel<Ts, L><<<grid, kPfWarps * 32, sm, s>>>(a, wf);
    check_launch("pf_kernel");
}

template<typename Ts>
static void launch_pf_t(const PfArgs &a, int B, cudaStream_t s)
{
    switch (a.L) {
    case 1: launch_pf_l<Ts, 1>(a, B, s); break;
    case 2: launch_pf_l<Ts, 2>(a, B, s); break;
    case 3: launch_pf_l<Ts, 3>(a, B, s); break;
    case 4: launch_pf_l<Ts, 4>(a, B, s); break;
    case 5: launch_pf_l<Ts, 5>(a, B, s); break;
    default: throw std::runtime_error("pf_kernel: unsupported number of boxcar levels");
    }
}

void launch_pf(const PfArgs &a, int dtype, int B, cudaStream_t s)
{
    if (a.Dout > 64 || a.Dout < 1) throw std::runtime_error("pf_kernel: time downsampling must be in [1, 64]");
    if (dtype == 0) launch_pf_t<float>(a, B, s);
    else if (dtype == 1) launch_pf_t<__half>(a, B, s);
    else launch_pf_t<__nv_bfloat16>(a, B, s);
}

}  // namespace pb2
