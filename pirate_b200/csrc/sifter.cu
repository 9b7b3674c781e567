// sifter.cu -- candidate patches and the sifter MLP (see sifter.hpp).

#include "sifter.hpp"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>

namespace pb2 {

#define SF_CHECK(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) \
    throw std::runtime_error(std::string("sifter: " #x ": ") + cudaGetErrorString(_e)); } while (0)

static void sf_check_launch(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": launch failed: " + cudaGetErrorString(e));
}

template<typename T> __device__ __forceinline__ float sf_to_f(T x);
template<> __device__ __forceinline__ float sf_to_f<float>(float x) { return x; }
template<> __device__ __forceinline__ float sf_to_f<__half>(__half x) { return __half2float(x); }
template<> __device__ __forceinline__ float sf_to_f<__nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }

// ---------------------------------------------------------------------------------------------
// Patches. One block per batch beam; thread (w, j) = (threadIdx.x / 32, threadIdx.x % 32) computes the
// width-2^w trailing boxcar ending at window time j for the 9 fine DMs.

template<typename Ts>
__global__ void __launch_bounds__(kPatchW * 32) patch_kernel(PatchArgs a)
{
    const int b = blockIdx.x;
    const int w = threadIdx.x >> 5, j = threadIdx.x & 31;
    __half *out = (__half *) a.patches + (long) b * kPatchLen;
    const float pk = a.peak[b];
    const int it = a.tree[b];
    const bool ok = (pk >= a.threshold) && (it >= 0) && (it < a.ntrees);
    if (threadIdx.x == 0) a.valid[b] = ok ? 1 : 0;
    if (!ok) {
        for (int d = 0; d < kPatchDm; d++) out[(d * kPatchT + j) * kPatchW + w] = __float2half_rn(0.0f);
        return;
    }
    const PatchTree &t = a.t[it];
    const uint32_t tok = a.token[b];
    const int m = (tok >> 16) & 0xffff, p = (tok >> 8) & 0xff, tf = tok & 0xff;
    const int l = p ? (p - 1) / 3 : 0;
    const int dt = min(t.Dcore, 1 << l);
    const long s0 = (a.chunk_ctr ? *a.chunk_ctr : a.ichunk) * t.nt_ds;
    // Last sample of the winning trial (the decode_argmax convention), placed at window time 23,
    // shifted so that the window ends inside the chunk.
    const long tend = s0 + (long) a.itime[b] * t.Dout + tf + dt - 1;
    long last = tend + (kPatchT - 1 - kPatchPeakAt);
    if (last > s0 + t.nt_ds - 1) last = s0 + t.nt_ds - 1;
    const long sj = last - (kPatchT - 1) + j;
    const int R = t.pf_rank;
    // Fine DM of the winning multiplet: coarse dm * 2^pf_rank + its fine offset (full band).
    int d0 = 0;
    for (int dd = 0; dd < (1 << R); dd++)
        if (t.d_to_m[dd] == m) d0 = dd;
    const long f0 = (long) a.idm[b] * (1 << R) + d0;
    const long nfine = (long) t.ndm_out << R;
    const long mask = t.pf_cap - 1;
    const int width = 1 << w;
    const float norm = rsqrtf((float) width);
    const int itw = a.itime[b] / (t.nt_out / t.nt_wt);
    const int dwds = t.ndm_out / t.ndm_wt;
    for (int d = 0; d < kPatchDm; d++) {
        const long f = f0 - kPatchDm / 2 + d;
        float v = 0.0f;
        if (f >= 0 && f < nfine) {
            const int mm = t.d_to_m[f & ((1 << R) - 1)];
            if (mm >= 0) {
                const Ts *row = (const Ts *) t.pf + (((long) (a.beam0 + b) * t.ndm_out + (f >> R)) * t.M + mm) * t.pf_cap;
                const float scale = t.wt[(((long) b * t.ndm_wt + (f >> R) / dwds) * t.nt_wt + itw) * t.P * t.N + t.nfull];
                float s = 0.0f;
                for (int k = 0; k < width; k++) s += sf_to_f(row[(sj - k) & mask]);
                v = 8.0f * asinhf(s * scale * norm * 0.125f);
            }
        }
        out[(d * kPatchT + j) * kPatchW + w] = __float2half_rn(v);
    }
}

void launch_patches(const PatchArgs &a, int dtype, cudaStream_t s)
{
    if (a.B <= 0) return;
    if (a.ntrees <= 0 || a.ntrees > kPatchMaxTrees) throw std::runtime_error("patches: bad number of trees");
    if (dtype == 0) patch_kernel<float><<<a.B, kPatchW * 32, 0, s>>>(a);
    else if (dtype == 1) patch_kernel<__half><<<a.B, kPatchW * 32, 0, s>>>(a);
    else if (dtype == 2) patch_kernel<__nv_bfloat16><<<a.B, kPatchW * 32, 0, s>>>(a);
    else throw std::runtime_error("patches: bad dtype");
    sf_check_launch("patch_kernel");
}

__global__ void mask_scores_kernel(const float *logits, const int *valid, float *scores, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) scores[i] = valid[i] ? logits[i] : -INFINITY;
}

void launch_mask_scores(const float *logits, const int *valid, float *scores, int n, cudaStream_t s)
{
    if (n <= 0) return;
    mask_scores_kernel<<<(n + 127) / 128, 128, 0, s>>>(logits, valid, scores, n);
    sf_check_launch("mask_scores_kernel");
}

// ---------------------------------------------------------------------------------------------
// GEMM on the tensor cores: C = A B^T (+ bias), bf16 operands, FP32 accumulation.
// A element (m, k) at A[m*sam + k*sak], B element (n, k) at B[n*sbn + k*sbk], either stored as float,
// fp16 or bf16 (rounded to bf16 while staged in shared memory). 64x64 block tiles, K steps of 32,
// four warps of 32x32, each issuing mma.sync.m16n8k16 (row.col, bf16 -> f32).
// Outputs: C (f32, optional) = acc; Cb (bf16, optional) = relu ? max(acc, 0) : acc.

struct GemmArgs
{
    int M, N, K;
    const void *A; long sam, sak;
    const void *B; long sbn, sbk;
    const float *bias;
    int relu;
    float *C; long ldc;
    uint16_t *Cb; long ldcb;
};

constexpr int kGBM = 64, kGBN = 64, kGBK = 32, kGPad = 8;

__device__ __forceinline__ void mma_bf16(float *c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

template<typename TA, typename TB>
__global__ void __launch_bounds__(128) gemm_kernel(GemmArgs g)
{
    __shared__ __align__(16) __nv_bfloat16 As[kGBM][kGBK + kGPad];
    __shared__ __align__(16) __nv_bfloat16 Bs[kGBN][kGBK + kGPad];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;
    const int gid = lane >> 2, tig = lane & 3;
    const int m0 = blockIdx.y * kGBM, n0 = blockIdx.x * kGBN;
    const TA *A = (const TA *) g.A;
    const TB *B = (const TB *) g.B;

    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int jj = 0; jj < 4; jj++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][jj][q] = 0.0f;

    for (int k0 = 0; k0 < g.K; k0 += kGBK) {
#pragma unroll 4
        for (int e = tid; e < kGBM * kGBK; e += 128) {
            const int r = e / kGBK, c = e % kGBK;
            const int m = m0 + r, k = k0 + c;
            const float va = (m < g.M && k < g.K) ? sf_to_f(A[(long) m * g.sam + (long) k * g.sak]) : 0.0f;
            As[r][c] = __float2bfloat16_rn(va);
            const int n = n0 + r;
            const float vb = (n < g.N && k < g.K) ? sf_to_f(B[(long) n * g.sbn + (long) k * g.sbk]) : 0.0f;
            Bs[r][c] = __float2bfloat16_rn(vb);
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < kGBK; ks += 16) {
            uint32_t af[2][4], bfr[4][2];
#pragma unroll
            for (int mt = 0; mt < 2; mt++) {
                const int r0 = wm * 32 + mt * 16 + gid;
                const int c0 = ks + tig * 2;
                af[mt][0] = *(const uint32_t *) &As[r0][c0];
                af[mt][1] = *(const uint32_t *) &As[r0 + 8][c0];
                af[mt][2] = *(const uint32_t *) &As[r0][c0 + 8];
                af[mt][3] = *(const uint32_t *) &As[r0 + 8][c0 + 8];
            }
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
                const int n = wn * 32 + nt * 8 + gid;
                const int k = ks + tig * 2;
                bfr[nt][0] = *(const uint32_t *) &Bs[n][k];
                bfr[nt][1] = *(const uint32_t *) &Bs[n][k + 8];
            }
#pragma unroll
            for (int mt = 0; mt < 2; mt++)
#pragma unroll
                for (int nt = 0; nt < 4; nt++)
                    mma_bf16(acc[mt][nt], af[mt][0], af[mt][1], af[mt][2], af[mt][3], bfr[nt][0], bfr[nt][1]);
        }
        __syncthreads();
    }

#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int m = m0 + wm * 32 + mt * 16 + gid + ((q >> 1) ? 8 : 0);
                const int n = n0 + wn * 32 + nt * 8 + tig * 2 + (q & 1);
                if (m < g.M && n < g.N) {
                    float v = acc[mt][nt][q] + (g.bias ? g.bias[n] : 0.0f);
                    if (g.C) g.C[(long) m * g.ldc + n] = v;
                    if (g.Cb) {
                        const float r = (g.relu && v < 0.0f) ? 0.0f : v;
                        __nv_bfloat16 h = __float2bfloat16_rn(r);
                        g.Cb[(long) m * g.ldcb + n] = *(const uint16_t *) &h;
                    }
                }
            }
}

enum { kF32 = 0, kF16 = 1, kBF16 = 2 };

static void gemm(const GemmArgs &g, int ta, int tb, cudaStream_t s)
{
    if (g.M <= 0 || g.N <= 0 || g.K <= 0) throw std::runtime_error("sifter gemm: empty shape");
    dim3 grid((g.N + kGBN - 1) / kGBN, (g.M + kGBM - 1) / kGBM);
    if (ta == kF16 && tb == kBF16) gemm_kernel<__half, __nv_bfloat16><<<grid, 128, 0, s>>>(g);
    else if (ta == kBF16 && tb == kBF16) gemm_kernel<__nv_bfloat16, __nv_bfloat16><<<grid, 128, 0, s>>>(g);
    else if (ta == kF32 && tb == kBF16) gemm_kernel<float, __nv_bfloat16><<<grid, 128, 0, s>>>(g);
    else if (ta == kF32 && tb == kF16) gemm_kernel<float, __half><<<grid, 128, 0, s>>>(g);
    else throw std::runtime_error("sifter gemm: unsupported operand types");
    sf_check_launch("gemm_kernel");
}

// ---------------------------------------------------------------------------------------------
// Loss, elementwise and optimizer kernels.

// Mean binary cross-entropy of the logits z against labels y; g[i] = (sigmoid(z_i) - y_i) / n.
// One block of 1024 threads (n <= max_batch); loss[0] = mean loss.
__global__ void __launch_bounds__(1024) bce_kernel(const float *z, const float *y, int n, float *g, float *loss)
{
    __shared__ float red[32];
    float s = 0.0f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float zi = z[i], yi = y[i];
        const float sig = 1.0f / (1.0f + expf(-zi));
        g[i] = (sig - yi) / (float) n;
        s += fmaxf(zi, 0.0f) - zi * yi + log1pf(expf(-fabsf(zi)));
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) loss[0] = s / (float) n;
    }
}

// out = in * (z > 0), elementwise over count values.
__global__ void relu_grad_kernel(const float *in, const float *z, float *out, long count)
{
    const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = (z[i] > 0.0f) ? in[i] : 0.0f;
}

// out[c] = sum_i g[i * H + c] (bias gradients).
__global__ void colsum_kernel(const float *g, int n, int H, float *out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= H) return;
    float s = 0.0f;
    for (int i = 0; i < n; i++) s += g[(long) i * H + c];
    out[c] = s;
}

__global__ void adam_kernel(float *w, const float *g, float *m, float *v, long count, float lr, float c1, float c2)
{
    const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1.0e-8f);
}

__global__ void to_bf16_kernel(const float *src, uint16_t *dst, long count)
{
    const long i = (long) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    __nv_bfloat16 h = __float2bfloat16_rn(src[i]);
    dst[i] = *(const uint16_t *) &h;
}

static unsigned blocks(long count, int t) { return (unsigned) ((count + t - 1) / t); }

// ---------------------------------------------------------------------------------------------
// Parameter layout.

static constexpr long kW1 = long(kMlpH1) * kMlpIn, kB1 = kMlpH1, kW2 = long(kMlpH2) * kMlpH1, kB2 = kMlpH2, kW3 = kMlpH2, kB3 = 1;
static constexpr long oW1 = 0, oB1 = oW1 + kW1, oW2 = oB1 + kB1, oB2 = oW2 + kW2, oW3 = oB2 + kB2, oB3 = oW3 + kW3;
static constexpr long kNparams = oB3 + kB3;
static constexpr long bW1 = 0, bW2 = kW1, bW3 = kW1 + kW2, kNbf16 = kW1 + kW2 + kW3;

long Sifter::nparams() { return kNparams; }

Sifter::Sifter(int device_, long max_batch_, uint64_t seed) : device(device_), max_batch(max_batch_)
{
    if (max_batch < 1 || max_batch > 1024) throw std::runtime_error("Sifter: max_batch must be in [1, 1024]");
    SF_CHECK(cudaSetDevice(device));
    SF_CHECK(cudaMalloc(&master, kNparams * sizeof(float)));
    SF_CHECK(cudaMalloc(&grad, kNparams * sizeof(float)));
    SF_CHECK(cudaMalloc(&adam_m, kNparams * sizeof(float)));
    SF_CHECK(cudaMalloc(&adam_v, kNparams * sizeof(float)));
    SF_CHECK(cudaMalloc(&wb, kNbf16 * sizeof(uint16_t)));
    SF_CHECK(cudaMalloc(&z1, max_batch * kMlpH1 * sizeof(float)));
    SF_CHECK(cudaMalloc(&z2, max_batch * kMlpH2 * sizeof(float)));
    SF_CHECK(cudaMalloc(&z3, max_batch * sizeof(float)));
    SF_CHECK(cudaMalloc(&g, max_batch * sizeof(float)));
    SF_CHECK(cudaMalloc(&loss, sizeof(float)));
    SF_CHECK(cudaMalloc(&h1, max_batch * kMlpH1 * sizeof(uint16_t)));
    SF_CHECK(cudaMalloc(&h2, max_batch * kMlpH2 * sizeof(uint16_t)));
    SF_CHECK(cudaMalloc(&g1, max_batch * kMlpH1 * sizeof(float)));
    SF_CHECK(cudaMalloc(&g2, max_batch * kMlpH2 * sizeof(float)));
    SF_CHECK(cudaMemset(adam_m, 0, kNparams * sizeof(float)));
    SF_CHECK(cudaMemset(adam_v, 0, kNparams * sizeof(float)));
    // He-uniform initial weights, zero biases.
    std::vector<float> p(kNparams, 0.0f);
    std::mt19937_64 rng(seed);
    auto fill = [&](long off, long count, long fan_in) {
        std::uniform_real_distribution<double> u(-std::sqrt(6.0 / fan_in), std::sqrt(6.0 / fan_in));
        for (long i = 0; i < count; i++) p[off + i] = float(u(rng));
    };
    fill(oW1, kW1, kMlpIn);
    fill(oW2, kW2, kMlpH1);
    fill(oW3, kW3, kMlpH2);
    set_params(p.data());
}

Sifter::~Sifter()
{
    cudaSetDevice(device);
    for (void *q : {(void *) master, (void *) grad, (void *) adam_m, (void *) adam_v, (void *) wb, (void *) z1, (void *) z2,
                    (void *) z3, (void *) g, (void *) loss, (void *) h1, (void *) h2, (void *) g1, (void *) g2})
        if (q) cudaFree(q);
}

void Sifter::refresh_bf16(cudaStream_t s)
{
    to_bf16_kernel<<<blocks(kW1, 256), 256, 0, s>>>(master + oW1, wb + bW1, kW1);
    to_bf16_kernel<<<blocks(kW2, 256), 256, 0, s>>>(master + oW2, wb + bW2, kW2);
    to_bf16_kernel<<<blocks(kW3, 256), 256, 0, s>>>(master + oW3, wb + bW3, kW3);
    sf_check_launch("to_bf16_kernel");
}

void Sifter::set_params(const float *host)
{
    SF_CHECK(cudaSetDevice(device));
    SF_CHECK(cudaMemcpy(master, host, kNparams * sizeof(float), cudaMemcpyHostToDevice));
    refresh_bf16(nullptr);
    SF_CHECK(cudaDeviceSynchronize());
}

void Sifter::get_params(float *host) const
{
    SF_CHECK(cudaSetDevice(device));
    SF_CHECK(cudaMemcpy(host, master, kNparams * sizeof(float), cudaMemcpyDeviceToHost));
}

void Sifter::forward(const uint16_t *patches, long n, float *logits, cudaStream_t s)
{
    if (n < 1 || n > max_batch) throw std::runtime_error("Sifter::forward: batch size out of range");
    if (!patches || !logits) throw std::runtime_error("Sifter::forward: null pointer");
    GemmArgs a;
    memset(&a, 0, sizeof(a));
    // Z1 = X W1^T + b1, H1 = bf16(relu(Z1))
    a.M = int(n); a.N = kMlpH1; a.K = kMlpIn;
    a.A = patches; a.sam = kMlpIn; a.sak = 1;
    a.B = wb + bW1; a.sbn = kMlpIn; a.sbk = 1;
    a.bias = master + oB1; a.relu = 1;
    a.C = z1; a.ldc = kMlpH1; a.Cb = h1; a.ldcb = kMlpH1;
    gemm(a, kF16, kBF16, s);
    // Z2 = H1 W2^T + b2, H2 = bf16(relu(Z2))
    a.N = kMlpH2; a.K = kMlpH1;
    a.A = h1; a.sam = kMlpH1; a.sak = 1;
    a.B = wb + bW2; a.sbn = kMlpH1; a.sbk = 1;
    a.bias = master + oB2;
    a.C = z2; a.ldc = kMlpH2; a.Cb = h2; a.ldcb = kMlpH2;
    gemm(a, kBF16, kBF16, s);
    // logit = H2 W3^T + b3
    a.N = 1; a.K = kMlpH2;
    a.A = h2; a.sam = kMlpH2; a.sak = 1;
    a.B = wb + bW3; a.sbn = kMlpH2; a.sbk = 1;
    a.bias = master + oB3; a.relu = 0;
    a.C = logits; a.ldc = 1; a.Cb = nullptr;
    gemm(a, kBF16, kBF16, s);
}

// Gradients of the mean binary cross-entropy into 'grad' (after forward() into z3).
void Sifter::backward(const uint16_t *patches, const float *labels, long n, cudaStream_t s)
{
    bce_kernel<<<1, 1024, 0, s>>>(z3, labels, int(n), g, loss);
    sf_check_launch("bce_kernel");
    GemmArgs a;
    memset(&a, 0, sizeof(a));
    // dW3 = g^T H2 (1 x 128)
    a.M = 1; a.N = kMlpH2; a.K = int(n);
    a.A = g; a.sam = 0; a.sak = 1;
    a.B = h2; a.sbn = 1; a.sbk = kMlpH2;
    a.C = grad + oW3; a.ldc = kMlpH2;
    gemm(a, kF32, kBF16, s);
    colsum_kernel<<<1, 32, 0, s>>>(g, int(n), 1, grad + oB3);
    // gH2 = g W3 (n x 128), g2 = gH2 * (Z2 > 0)
    a.M = int(n); a.N = kMlpH2; a.K = 1;
    a.A = g; a.sam = 1; a.sak = 1;
    a.B = wb + bW3; a.sbn = 1; a.sbk = kMlpH2;
    a.C = g2; a.ldc = kMlpH2;
    gemm(a, kF32, kBF16, s);
    relu_grad_kernel<<<blocks(n * kMlpH2, 256), 256, 0, s>>>(g2, z2, g2, n * kMlpH2);
    // dW2 = g2^T H1 (128 x 256), db2
    a.M = kMlpH2; a.N = kMlpH1; a.K = int(n);
    a.A = g2; a.sam = 1; a.sak = kMlpH2;
    a.B = h1; a.sbn = 1; a.sbk = kMlpH1;
    a.C = grad + oW2; a.ldc = kMlpH1;
    gemm(a, kF32, kBF16, s);
    colsum_kernel<<<blocks(kMlpH2, 128), 128, 0, s>>>(g2, int(n), kMlpH2, grad + oB2);
    // gH1 = g2 W2 (n x 256), g1 = gH1 * (Z1 > 0)
    a.M = int(n); a.N = kMlpH1; a.K = kMlpH2;
    a.A = g2; a.sam = kMlpH2; a.sak = 1;
    a.B = wb + bW2; a.sbn = 1; a.sbk = kMlpH1;
    a.C = g1; a.ldc = kMlpH1;
    gemm(a, kF32, kBF16, s);
    relu_grad_kernel<<<blocks(n * kMlpH1, 256), 256, 0, s>>>(g1, z1, g1, n * kMlpH1);
    // dW1 = g1^T X (256 x 1728), db1
    a.M = kMlpH1; a.N = kMlpIn; a.K = int(n);
    a.A = g1; a.sam = 1; a.sak = kMlpH1;
    a.B = patches; a.sbn = 1; a.sbk = kMlpIn;
    a.C = grad + oW1; a.ldc = kMlpIn;
    gemm(a, kF32, kF16, s);
    colsum_kernel<<<blocks(kMlpH1, 128), 128, 0, s>>>(g1, int(n), kMlpH1, grad + oB1);
    sf_check_launch("sifter backward");
}

double Sifter::gradients(const uint16_t *patches, const float *labels, long n, float *grad_host, cudaStream_t s)
{
    if (!labels || !grad_host) throw std::runtime_error("Sifter::gradients: null pointer");
    SF_CHECK(cudaSetDevice(device));
    forward(patches, n, z3, s);
    backward(patches, labels, n, s);
    float l = 0.0f;
    SF_CHECK(cudaMemcpyAsync(grad_host, grad, kNparams * sizeof(float), cudaMemcpyDeviceToHost, s));
    SF_CHECK(cudaMemcpyAsync(&l, loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    SF_CHECK(cudaStreamSynchronize(s));
    return l;
}

double Sifter::train_step(const uint16_t *patches, const float *labels, long n, float lr, cudaStream_t s)
{
    if (!labels) throw std::runtime_error("Sifter::train_step: null pointer");
    SF_CHECK(cudaSetDevice(device));
    forward(patches, n, z3, s);
    backward(patches, labels, n, s);
    step++;
    const float c1 = 1.0f - std::pow(0.9f, float(step)), c2 = 1.0f - std::pow(0.999f, float(step));
    adam_kernel<<<blocks(kNparams, 256), 256, 0, s>>>(master, grad, adam_m, adam_v, kNparams, lr, c1, c2);
    sf_check_launch("adam_kernel");
    refresh_bf16(s);
    float l = 0.0f;
    SF_CHECK(cudaMemcpyAsync(&l, loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    SF_CHECK(cudaStreamSynchronize(s));
    return l;
}

}  // namespace pb2
