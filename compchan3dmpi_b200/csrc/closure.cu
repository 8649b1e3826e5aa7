// closure.cu -- tensor-core (tcgen05) kernels of the learned subgrid closure.
//
// This translation unit holds the BF16 tensor-core GEMM path the closure's
// MLP runs on, and a self-test entry point that checks it against a host
// product through the C ABI.
#include "chanrhs.h"
#include "chan_internal.h"
#include "umma.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace {

// mbarrier polls before a kernel gives up waiting for its own MMAs, records
// an error and frees its tensor memory (a few seconds at most)
constexpr uint32_t kWaitLimit = 1u << 24;

std::string g_cl_error;

// D[128][N] = A[128][K] * B[N][K]^T on the tensor cores; one CTA of 128 threads
__global__ void __launch_bounds__(128, 1)
    k_umma_selftest(const __nv_bfloat16 *A, const __nv_bfloat16 *B, float *D, int K, int N, int *err)
{
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned char *sA = sm;                       // 128 x K
    unsigned char *sB = sm + 128 * K * 2;         // N x K
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int e = tid; e < 128 * K; e += 128)
        *(__nv_bfloat16 *)(sA + umma::kmaj_off(e / K, e % K, K)) = A[e];
    for (int e = tid; e < N * K; e += 128)
        *(__nv_bfloat16 *)(sB + umma::kmaj_off(e / K, e % K, K)) = B[e];
    if (warp == 0) umma::tmem_alloc(&tbase, 256);
    if (tid == 0) umma::mbar_init(&mbar, 1);
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tb = tbase;
    if (tid == 0) {
        umma::gemm_kmajor(tb, sA, sB, K, N, false);
        umma::commit(&mbar);
    }
    const bool ok = umma::mbar_wait(&mbar, 0, kWaitLimit);
    if (!ok) {
        // give the MMA one more bounded wait before its tensor memory is freed
        if (tid == 0) {
            atomicExch(err, 1);
            umma::mbar_wait(&mbar, 0, kWaitLimit);
        }
    } else {
        umma::fence_after_sync();
        for (int c = 0; c < N; c += 16) {
            float v[16];
            umma::tmem_ld16(umma::lane_addr(tb, warp, c), v);
#pragma unroll
            for (int i = 0; i < 16; i++) D[(size_t)tid * N + c + i] = v[i];
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_free(tb, 256);
}

// ---------------------------------------------------------------------------
// The closure MLP: 13 inputs (padded to 16) -> 64 -> 64 -> 9 outputs (padded
// to 16), GELU activations, BF16 weights and activations on the tensor cores,
// F32 accumulation in tensor memory, F32 biases, F32 master weights.
constexpr int kIn = 13, kInP = 16, kHid = 64, kOut = 9, kOutP = 16, kTile = 128;

// BF16 weight images in the shared-memory layout (K-major core matrices):
// W1 [64][16], W2 [64][64], W3 [16][64] (rows 9..15 zero), and the
// transposes used by the backward pass W2t [64][64], W3t [64][16].
struct WImages {
    static constexpr int w1 = 0, w2 = w1 + kHid * kInP * 2, w3 = w2 + kHid * kHid * 2, w2t = w3 + kOutP * kHid * 2,
                         w3t = w2t + kHid * kHid * 2, bytes = w3t + kHid * kOutP * 2;
};

struct MlpParams {
    const unsigned char *wimg;   // WImages::bytes of BF16 images
    const float *b1, *b2, *b3;   // biases (64, 64, 9)
    const float *X;              // inputs (raw): X[row * xr + f * xc]
    const float *T;              // [n][9] targets (raw), training only
    const float *xmu, *xsd;      // input normalisation (13 each)
    const float *ymu, *ysd;      // output normalisation (9 each)
    long long n;                 // samples
    long long perm_a, perm_b;    // sample of batch row r: (perm_a * (row0 + r) + perm_b) mod n
    long long row0, rows;        // batch rows [row0, row0 + rows)
    float *Y;                    // outputs (raw units), inference only: Y[row * yr + o * yc]
    long long xr, xc, yr, yc;    // element strides of X and Y (rows, columns)
    float *gW1, *gW2, *gW3, *gb1, *gb2, *gb3;   // gradient sums (training)
    float *loss;                 // sum of squared normalised errors (training)
    float inv_count;             // 2 / (9 * rows): d loss / d y factor
    float out_limit;             // inference: |normalised output| above this sets *flag
    int *flag;
    int *err;
};

// GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), on
// the hardware tanh approximation (tanh.approx.f32), and its derivative
__device__ __forceinline__ float tanh_hw(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kGeluA = 0.7978845608028654f, kGeluB = 0.044715f;
__device__ __forceinline__ float gelu(float z)
{
    const float t = tanh_hw(kGeluA * (z + kGeluB * z * z * z));
    return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ float gelu_d(float z)
{
    const float t = tanh_hw(kGeluA * (z + kGeluB * z * z * z));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluA * (1.0f + 3.0f * kGeluB * z * z);
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void st_bf16(unsigned char *base, uint32_t off, float v)
{
    *(__nv_bfloat16 *)(base + off) = __float2bfloat16_rn(v);
}

// 8 consecutive K elements of one row as one 16-byte store
__device__ __forceinline__ void st_bf16x8(unsigned char *base, uint32_t off, const float *v)
{
    __nv_bfloat162 h[4];
#pragma unroll
    for (int i = 0; i < 4; i++) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    *(uint4 *)(base + off) = *(uint4 *)h;
}

// Shared memory of the MLP kernel (bytes)
struct MlpSmem {
    static constexpr int w = 0;                                      // weight images
    static constexpr int x = w + WImages::bytes;                     // X   [128][16]
    static constexpr int h1 = x + kTile * kInP * 2;                  // H1  [128][64]
    static constexpr int h2 = h1 + kTile * kHid * 2;                 // H2  [128][64]
    static constexpr int dy = h2 + kTile * kHid * 2;                 // dY  [128][16]
    static constexpr int dz2 = dy + kTile * kOutP * 2;               // dZ2 [128][64]
    static constexpr int xt = dz2 + kTile * kHid * 2;                // X^T  [16][128]
    static constexpr int h1t = xt + kInP * kTile * 2;                // H1^T [64][128]
    static constexpr int h2t = h1t + kHid * kTile * 2;               // H2^T [64][128]
    static constexpr int gt = h2t + kHid * kTile * 2;                // dY^T / dZ2^T / dZ1^T [128][128]
    static constexpr int fl = gt + kTile * kTile * 2;                // floats: b1 b2 b3 db1 db2 db3 loss
    static constexpr int bytes = fl + (64 + 64 + 16 + 64 + 64 + 16 + 4) * 4;
};

// Shared memory of the inference-only kernel: the forward weight images, X, H1, H2
struct InferSmem {
    static constexpr int wbytes = WImages::w2t;                      // W1, W2, W3 images
    static constexpr int x = wbytes;
    static constexpr int h1 = x + kTile * kInP * 2;
    static constexpr int h2 = h1 + kTile * kHid * 2;
    static constexpr int fl = h2 + kTile * kHid * 2;
    static constexpr int bytes = fl + (64 + 64 + 16 + 64 + 64 + 16 + 4) * 4;
};

// tensor-memory columns: training holds all 512 (one CTA per SM); inference
// needs Z1, Z2 and Y, with Y over Z1's columns (128, four CTAs per SM)
constexpr int cZ1 = 0, cZ2 = 64, cdH2 = 192, cdH1 = 256, cdW3 = 320, cdW2 = 384, cdW1 = 448;
template <bool TRAIN>
struct MlpCfg {
    static constexpr int cY = TRAIN ? 128 : 0, tmem = TRAIN ? 512 : 128, minb = TRAIN ? 1 : 4;
    static constexpr int wbytes = TRAIN ? WImages::bytes : InferSmem::wbytes;
    static constexpr int x = TRAIN ? MlpSmem::x : InferSmem::x, h1 = TRAIN ? MlpSmem::h1 : InferSmem::h1,
                         h2 = TRAIN ? MlpSmem::h2 : InferSmem::h2, fl = TRAIN ? MlpSmem::fl : InferSmem::fl,
                         bytes = TRAIN ? MlpSmem::bytes : InferSmem::bytes;
};

// Forward (and for TRAIN the backward) pass over the batch rows, 128 per
// tile, tiles strided over the grid; one CTA of 128 threads per SM (the CTA
// holds all 512 tensor-memory columns).  Thread t owns row t of each tile.
template <bool TRAIN>
__global__ void __launch_bounds__(128, MlpCfg<TRAIN>::minb) k_mlp(const MlpParams P)
{
    using G = MlpCfg<TRAIN>;
    constexpr int cY = G::cY;
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5;
    float *fb1 = (float *)(sm + G::fl), *fb2 = fb1 + 64, *fb3 = fb2 + 64;
    float *db1 = fb3 + 16, *db2 = db1 + 64, *db3 = db2 + 64, *sloss = db3 + 16;
    {   // weight images and biases
        const uint4 *src = (const uint4 *)P.wimg;
        uint4 *dst = (uint4 *)(sm + MlpSmem::w);
        for (int e = tid; e < G::wbytes / 16; e += 128) dst[e] = src[e];
        if (tid < 64) { fb1[tid] = P.b1[tid]; fb2[tid] = P.b2[tid]; db1[tid] = 0.f; db2[tid] = 0.f; }
        if (tid < 16) { fb3[tid] = tid < kOut ? P.b3[tid] : 0.f; db3[tid] = 0.f; }
        if (tid == 0) sloss[0] = 0.f;
    }
    if (warp == 0) umma::tmem_alloc(&tbase, G::tmem);
    if (tid == 0) umma::mbar_init(&mbar, 1);
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tb = tbase;
    unsigned char *sW = sm + MlpSmem::w;
    unsigned char *sX = sm + G::x, *sH1 = sm + G::h1, *sH2 = sm + G::h2;
    unsigned char *sdY = sm + MlpSmem::dy, *sdZ2 = sm + MlpSmem::dz2;
    unsigned char *sXt = sm + MlpSmem::xt, *sH1t = sm + MlpSmem::h1t, *sH2t = sm + MlpSmem::h2t;
    unsigned char *sGt = sm + MlpSmem::gt;
    uint32_t phase = 0;
    bool ok = true;
    // issue by thread 0 after the smem writes of every thread; then wait
    auto sync_issue_wait = [&](auto &&issue) {
        umma::fence_async_smem();
        umma::fence_before_sync();
        __syncthreads();
        if (tid == 0 && ok) {
            umma::fence_after_sync();
            issue();
            umma::commit(&mbar);
        }
        if (ok) {
            ok = umma::mbar_wait(&mbar, phase, kWaitLimit);
            if (ok) phase ^= 1u;
        }
        ok = __syncthreads_and(ok) != 0;   // one verdict for the whole CTA
        umma::fence_after_sync();
    };
    const long long ntiles = (P.rows + kTile - 1) / kTile;
    bool first = true;
    for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long long row = tile * kTile + tid;
        const bool live = row < P.rows;
        long long sample = 0;
        if (live) sample = (long long)(((__int128)P.perm_a * (P.row0 + row) + P.perm_b) % P.n);
        // ---- inputs, normalised, as X and X^T
        float xin[kInP], tgt[kOut];
#pragma unroll
        for (int f = 0; f < kInP; f++)
            xin[f] = (live && f < kIn) ? (P.X[sample * P.xr + f * P.xc] - P.xmu[f]) / P.xsd[f] : 0.f;
        if (TRAIN) {
#pragma unroll
            for (int o = 0; o < kOut; o++) tgt[o] = live ? (P.T[sample * kOut + o] - P.ymu[o]) / P.ysd[o] : 0.f;
        }
        st_bf16x8(sX, umma::kmaj_off(tid, 0, kInP), xin);
        st_bf16x8(sX, umma::kmaj_off(tid, 8, kInP), xin + 8);
        if (TRAIN) {
#pragma unroll
            for (int f = 0; f < kInP; f++) st_bf16(sXt, umma::kmaj_off(f, tid, kTile), xin[f]);
        }
        // ---- F1: Z1 = X W1^T
        sync_issue_wait([&] { umma::gemm_kmajor(tb + cZ1, sX, sW + WImages::w1, kInP, kHid, false); });
        if (!ok) break;
        for (int c = 0; c < kHid; c += 16) {
            float z[16], h[16];
            umma::tmem_ld16(umma::lane_addr(tb, warp, cZ1 + c), z);
#pragma unroll
            for (int i = 0; i < 16; i++) h[i] = gelu(z[i] + fb1[c + i]);
            st_bf16x8(sH1, umma::kmaj_off(tid, c, kHid), h);
            st_bf16x8(sH1, umma::kmaj_off(tid, c + 8, kHid), h + 8);
            if (TRAIN) {
#pragma unroll
                for (int i = 0; i < 16; i++) st_bf16(sH1t, umma::kmaj_off(c + i, tid, kTile), h[i]);
            }
        }
        // ---- F2: Z2 = H1 W2^T
        sync_issue_wait([&] { umma::gemm_kmajor(tb + cZ2, sH1, sW + WImages::w2, kHid, kHid, false); });
        if (!ok) break;
        for (int c = 0; c < kHid; c += 16) {
            float z[16], h[16];
            umma::tmem_ld16(umma::lane_addr(tb, warp, cZ2 + c), z);
#pragma unroll
            for (int i = 0; i < 16; i++) h[i] = gelu(z[i] + fb2[c + i]);
            st_bf16x8(sH2, umma::kmaj_off(tid, c, kHid), h);
            st_bf16x8(sH2, umma::kmaj_off(tid, c + 8, kHid), h + 8);
            if (TRAIN) {
#pragma unroll
                for (int i = 0; i < 16; i++) st_bf16(sH2t, umma::kmaj_off(c + i, tid, kTile), h[i]);
            }
        }
        // ---- F3: Y = H2 W3^T
        sync_issue_wait([&] { umma::gemm_kmajor(tb + cY, sH2, sW + WImages::w3, kHid, kOutP, false); });
        if (!ok) break;
        float y[16];
        umma::tmem_ld16(umma::lane_addr(tb, warp, cY), y);
#pragma unroll
        for (int o = 0; o < kOutP; o++) y[o] += fb3[o];
        if (!TRAIN) {
            if (live) {
                bool big = false;
#pragma unroll
                for (int o = 0; o < kOut; o++) {
                    big = big || !(fabsf(y[o]) <= P.out_limit);
                    P.Y[row * P.yr + o * P.yc] = y[o] * P.ysd[o] + P.ymu[o];
                }
                if (big && P.flag) atomicOr(P.flag, 1);
            }
            continue;
        }
        // ---- loss and dY = 2 (y - t) / (9 rows)
        float dy[16], l = 0.f;
#pragma unroll
        for (int o = 0; o < kOutP; o++) {
            const float e = (live && o < kOut) ? y[o] - tgt[o] : 0.f;
            l += e * e;
            dy[o] = e * P.inv_count;
        }
        st_bf16x8(sdY, umma::kmaj_off(tid, 0, kOutP), dy);
        st_bf16x8(sdY, umma::kmaj_off(tid, 8, kOutP), dy + 8);
#pragma unroll
        for (int o = 0; o < kOutP; o++) st_bf16(sGt, umma::kmaj_off(o, tid, kTile), dy[o]);
        {
            const float ls = warp_sum(l);
            if ((tid & 31) == 0) atomicAdd(sloss, ls);
#pragma unroll
            for (int o = 0; o < kOut; o++) {
                const float s3 = warp_sum(dy[o]);
                if ((tid & 31) == 0) atomicAdd(&db3[o], s3);
            }
        }
        // ---- B3: dH2 = dY W3 ; G3: dW3 += dY^T H2
        const bool acc = !first;
        sync_issue_wait([&] {
            umma::gemm_kmajor(tb + cdH2, sdY, sW + WImages::w3t, kOutP, kHid, false);
            umma::gemm_kmajor(tb + cdW3, sGt, sH2t, kTile, kHid, acc);
        });
        if (!ok) break;
        for (int c = 0; c < kHid; c += 16) {
            float g[16], z[16], d[16];
            umma::tmem_ld16(umma::lane_addr(tb, warp, cdH2 + c), g);
            umma::tmem_ld16(umma::lane_addr(tb, warp, cZ2 + c), z);
#pragma unroll
            for (int i = 0; i < 16; i++) d[i] = live ? g[i] * gelu_d(z[i] + fb2[c + i]) : 0.f;
            st_bf16x8(sdZ2, umma::kmaj_off(tid, c, kHid), d);
            st_bf16x8(sdZ2, umma::kmaj_off(tid, c + 8, kHid), d + 8);
#pragma unroll
            for (int i = 0; i < 16; i++) {
                st_bf16(sGt, umma::kmaj_off(c + i, tid, kTile), d[i]);
                const float s2 = warp_sum(d[i]);
                if ((tid & 31) == 0) atomicAdd(&db2[c + i], s2);
            }
        }
        // ---- B2: dH1 = dZ2 W2 ; G2: dW2 += dZ2^T H1
        sync_issue_wait([&] {
            umma::gemm_kmajor(tb + cdH1, sdZ2, sW + WImages::w2t, kHid, kHid, false);
            umma::gemm_kmajor(tb + cdW2, sGt, sH1t, kTile, kHid, acc);
        });
        if (!ok) break;
        for (int c = 0; c < kHid; c += 16) {
            float g[16], z[16];
            umma::tmem_ld16(umma::lane_addr(tb, warp, cdH1 + c), g);
            umma::tmem_ld16(umma::lane_addr(tb, warp, cZ1 + c), z);
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const float d = live ? g[i] * gelu_d(z[i] + fb1[c + i]) : 0.f;
                st_bf16(sGt, umma::kmaj_off(c + i, tid, kTile), d);
                const float s1 = warp_sum(d);
                if ((tid & 31) == 0) atomicAdd(&db1[c + i], s1);
            }
        }
        // ---- G1: dW1 += dZ1^T X
        sync_issue_wait([&] { umma::gemm_kmajor(tb + cdW1, sGt, sXt, kTile, kInP, acc); });
        first = false;
    }
    if (TRAIN && ok && !first) {
        // weight-gradient sums out of tensor memory: lane = output feature
        const int o = tid;
        for (int c = 0; c < kHid; c += 16) {
            float v[16];
            umma::tmem_ld16(umma::lane_addr(tb, warp, cdW3 + c), v);
            if (o < kOut) {
#pragma unroll
                for (int i = 0; i < 16; i++) atomicAdd(&P.gW3[o * kHid + c + i], v[i]);
            }
            umma::tmem_ld16(umma::lane_addr(tb, warp, cdW2 + c), v);
            if (o < kHid) {
#pragma unroll
                for (int i = 0; i < 16; i++) atomicAdd(&P.gW2[o * kHid + c + i], v[i]);
            }
        }
        float v[16];
        umma::tmem_ld16(umma::lane_addr(tb, warp, cdW1), v);
        if (o < kHid) {
#pragma unroll
            for (int i = 0; i < kIn; i++) atomicAdd(&P.gW1[o * kIn + i], v[i]);
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (TRAIN) {
        if (tid < 64) { atomicAdd(&P.gb1[tid], db1[tid]); atomicAdd(&P.gb2[tid], db2[tid]); }
        if (tid < kOut) atomicAdd(&P.gb3[tid], db3[tid]);
        if (tid == 0) atomicAdd(P.loss, sloss[0]);
    }
    if (!ok) {
        // an MMA did not signal completion: give it one more bounded wait
        // before the tensor memory it writes is released
        if (tid == 0) {
            umma::mbar_wait(&mbar, phase, kWaitLimit);
            atomicExch(P.err, 1);
        }
        __syncthreads();
    }
    if (warp == 0) umma::tmem_free(tb, G::tmem);
}

// Adam on the F32 master parameters, then the BF16 weight images.
// Parameter vector: W1[64][13] b1[64] W2[64][64] b2[64] W3[9][64] b3[9].
constexpr int kNW1 = kHid * kIn, kNW2 = kHid * kHid, kNW3 = kOut * kHid;
constexpr int kOffB1 = kNW1, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kNW2, kOffW3 = kOffB2 + kHid,
              kOffB3 = kOffW3 + kNW3, kNParam = kOffB3 + kOut;

__global__ void k_adam(float *w, float *m, float *v, const float *g, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// BF16 images of the F32 master weights (padding stays zero from the memset)
__global__ void k_weight_images(const float *w, unsigned char *img)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kNW1) {
        const int o = i / kIn, f = i % kIn;
        st_bf16(img + WImages::w1, umma::kmaj_off(o, f, kInP), w[i]);
    } else if (i < kNW1 + kNW2) {
        const int j = i - kNW1, o = j / kHid, f = j % kHid;
        const float x = w[kOffW2 + j];
        st_bf16(img + WImages::w2, umma::kmaj_off(o, f, kHid), x);
        st_bf16(img + WImages::w2t, umma::kmaj_off(f, o, kHid), x);
    } else if (i < kNW1 + kNW2 + kNW3) {
        const int j = i - kNW1 - kNW2, o = j / kHid, f = j % kHid;
        const float x = w[kOffW3 + j];
        st_bf16(img + WImages::w3, umma::kmaj_off(o, f, kHid), x);
        st_bf16(img + WImages::w3t, umma::kmaj_off(f, o, kOutP), x);
    }
}

// column sums and sums of squares of an [n][ncol] array (double atomics)
__global__ void k_colstats(const float *A, long long n, int ncol, double *sum, double *sumsq)
{
    double s[16], s2[16];
    for (int c = 0; c < ncol; c++) s[c] = s2[c] = 0.0;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
        for (int c = 0; c < ncol; c++) {
            const double v = A[r * ncol + c];
            s[c] += v;
            s2[c] += v * v;
        }
    for (int c = 0; c < ncol; c++) {
        double a = s[c], b = s2[c];
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&sum[c], a);
            atomicAdd(&sumsq[c], b);
        }
    }
}

uint64_t splitmix(uint64_t &x)
{
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

long long gcd_ll(long long a, long long b)
{
    while (b) { const long long t = a % b; a = b; b = t; }
    return a;
}

}  // namespace

// Dataset, parameters, optimiser state and weight images of one closure.
struct chan_closure {
    int dev = 0;
    cudaStream_t stream = nullptr;
    float *X = nullptr, *T = nullptr;       // [cap][13], [cap][9] samples
    long long cap = 0, count = 0;
    float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;   // kNParam each
    unsigned char *img = nullptr;           // BF16 weight images
    float *norm = nullptr;                  // xmu[13] xsd[13] ymu[9] ysd[9]
    float *loss = nullptr;
    int *err = nullptr;
    long long adam_t = 0;
    float out_limit = 50.f;
    int sms = 148;
    std::string msg;
};

namespace {

int cfail(chan_closure *m, const char *what, cudaError_t e)
{
    if (m) m->msg = std::string(what) + ": " + cudaGetErrorString(e);
    else g_cl_error = std::string(what) + ": " + cudaGetErrorString(e);
    return CHAN_ECUDA;
}

#define CLK(m, call)                                    \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cfail((m), #call, e_); \
    } while (0)

MlpParams base_params(chan_closure *m)
{
    MlpParams P{};
    P.wimg = m->img;
    P.b1 = m->w + kOffB1; P.b2 = m->w + kOffB2; P.b3 = m->w + kOffB3;
    P.xmu = m->norm; P.xsd = m->norm + 13; P.ymu = m->norm + 26; P.ysd = m->norm + 35;
    P.gW1 = m->g; P.gb1 = m->g + kOffB1; P.gW2 = m->g + kOffW2; P.gb2 = m->g + kOffB2;
    P.gW3 = m->g + kOffW3; P.gb3 = m->g + kOffB3;
    P.loss = m->loss;
    P.err = m->err;
    P.out_limit = m->out_limit;
    P.perm_a = 1; P.perm_b = 0;
    P.xr = kIn; P.xc = 1; P.yr = kOut; P.yc = 1;
    return P;
}

int refresh_images(chan_closure *m)
{
    k_weight_images<<<(kNW1 + kNW2 + kNW3 + 255) / 256, 256, 0, m->stream>>>(m->w, m->img);
    CLK(m, cudaGetLastError());
    return CHAN_OK;
}

int launch_mlp(chan_closure *m, const MlpParams &P, bool train, cudaStream_t st)
{
    const long long ntiles = (P.rows + kTile - 1) / kTile;
    const long long slots = (long long)m->sms * (train ? MlpCfg<true>::minb : MlpCfg<false>::minb);
    const int grid = (int)(ntiles < slots ? ntiles : slots);
    if (grid < 1) return CHAN_OK;
    if (train) k_mlp<true><<<grid, 128, MlpCfg<true>::bytes, st>>>(P);
    else k_mlp<false><<<grid, 128, MlpCfg<false>::bytes, st>>>(P);
    CLK(m, cudaGetLastError());
    return CHAN_OK;
}

int check_err(chan_closure *m)
{
    int h = 0;
    CLK(m, cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    CLK(m, cudaStreamSynchronize(m->stream));
    if (h) { m->msg = "tensor-core wait gave up"; return CHAN_ECUDA; }
    return CHAN_OK;
}

}  // namespace

int chan_internal_infer(chan_closure *m, const float *X, float *Y, long long n, bool soa, cudaStream_t stream,
                        int *flag)
{
    MlpParams P = base_params(m);
    P.X = X; P.Y = Y; P.n = n; P.rows = n; P.row0 = 0; P.flag = flag;
    if (soa) { P.xr = 1; P.xc = n; P.yr = 1; P.yc = n; }
    return launch_mlp(m, P, false, stream);
}

int chan_internal_closure_device(chan_closure *m) { return m ? m->dev : -1; }

extern "C" {

int chan_selftest_umma(const uint16_t *A, const uint16_t *B, float *D, int32_t K, int32_t N, int32_t device)
{
    if (!A || !B || !D || K < 16 || K > 256 || K % 16 || N < 16 || N > 256 || N % 16) return CHAN_EINVAL;
    cudaError_t e = cudaSetDevice(device);
    __nv_bfloat16 *dA = nullptr, *dB = nullptr;
    float *dD = nullptr;
    int *derr = nullptr, herr = 0;
    const size_t smem = (size_t)(128 + N) * K * 2;
    if (e == cudaSuccess) e = cudaMalloc((void **)&dA, (size_t)128 * K * 2);
    if (e == cudaSuccess) e = cudaMalloc((void **)&dB, (size_t)N * K * 2);
    if (e == cudaSuccess) e = cudaMalloc((void **)&dD, (size_t)128 * N * 4);
    if (e == cudaSuccess) e = cudaMalloc((void **)&derr, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(dA, A, (size_t)128 * K * 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dB, B, (size_t)N * K * 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(derr, 0, sizeof(int));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_umma_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
        k_umma_selftest<<<1, 128, smem>>>(dA, dB, dD, K, N, derr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(D, dD, (size_t)128 * N * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
    if (dA) cudaFree(dA);
    if (dB) cudaFree(dB);
    if (dD) cudaFree(dD);
    if (derr) cudaFree(derr);
    if (e != cudaSuccess) {
        g_cl_error = cudaGetErrorString(e);
        return CHAN_ECUDA;
    }
    return herr ? CHAN_ECUDA : CHAN_OK;
}

int chan_closure_create(int32_t device, int64_t capacity, chan_closure **out)
{
    if (!out || capacity < 0) return CHAN_EINVAL;
    *out = nullptr;
    chan_closure *m = new chan_closure;
    m->dev = device;
    m->cap = capacity;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess && capacity > 0) e = cudaMalloc((void **)&m->X, (size_t)capacity * kIn * sizeof(float));
    if (e == cudaSuccess && capacity > 0) e = cudaMalloc((void **)&m->T, (size_t)capacity * kOut * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->w, 4 * (size_t)kNParam * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->img, WImages::bytes);
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->norm, 44 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&m->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(m->w, 0, 4 * (size_t)kNParam * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(m->img, 0, WImages::bytes);
    if (e == cudaSuccess) e = cudaMemset(m->err, 0, sizeof(int));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, MlpSmem::bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, MlpCfg<false>::bytes);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&m->sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        g_cl_error = std::string("chan_closure_create: ") + cudaGetErrorString(e);
        chan_closure_free(m);
        return CHAN_ECUDA;
    }
    m->m = m->w + kNParam;
    m->v = m->m + kNParam;
    m->g = m->v + kNParam;
    // identity normalisation until one is fitted or set
    float nrm[44];
    for (int i = 0; i < 44; i++) nrm[i] = (i >= 13 && i < 26) || i >= 35 ? 1.f : 0.f;
    cudaMemcpy(m->norm, nrm, sizeof(nrm), cudaMemcpyHostToDevice);
    *out = m;
    return CHAN_OK;
}

int chan_closure_sample(chan_closure *m, chan_ctx *dns, int32_t sx, int32_t sy, int32_t sz, int32_t fw,
                        int64_t *added)
{
    if (!m || !dns) return CHAN_EINVAL;
    long long a = 0;
    int r = chan_internal_sample(dns, m->X + m->count * kIn, m->T + m->count * kOut, m->cap - m->count, sx, sy, sz,
                                 fw, &a);
    if (r) { m->msg = "sampling failed (see chan_last_error of the context)"; return r; }
    m->count += a;
    if (added) *added = a;
    return CHAN_OK;
}

int chan_closure_add_data(chan_closure *m, const float *X, const float *T, int64_t n)
{
    if (!m || !X || !T || n < 0 || m->count + n > m->cap) return CHAN_EINVAL;
    CLK(m, cudaSetDevice(m->dev));
    CLK(m, cudaMemcpy(m->X + m->count * kIn, X, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice));
    CLK(m, cudaMemcpy(m->T + m->count * kOut, T, (size_t)n * kOut * sizeof(float), cudaMemcpyHostToDevice));
    m->count += n;
    return CHAN_OK;
}

int chan_closure_count(chan_closure *m, int64_t *count)
{
    if (!m || !count) return CHAN_EINVAL;
    *count = m->count;
    return CHAN_OK;
}

int chan_closure_get_data(chan_closure *m, int64_t first, int64_t n, float *X, float *T)
{
    if (!m || first < 0 || n < 0 || first + n > m->count) return CHAN_EINVAL;
    CLK(m, cudaSetDevice(m->dev));
    if (X) CLK(m, cudaMemcpy(X, m->X + first * kIn, (size_t)n * kIn * sizeof(float), cudaMemcpyDeviceToHost));
    if (T) CLK(m, cudaMemcpy(T, m->T + first * kOut, (size_t)n * kOut * sizeof(float), cudaMemcpyDeviceToHost));
    return CHAN_OK;
}

int chan_closure_fit_normalization(chan_closure *m, float *norm_out)
{
    if (!m || m->count < 2) return CHAN_EINVAL;
    CLK(m, cudaSetDevice(m->dev));
    double *acc = nullptr;
    CLK(m, cudaMalloc((void **)&acc, 44 * sizeof(double)));
    CLK(m, cudaMemsetAsync(acc, 0, 44 * sizeof(double), m->stream));
    k_colstats<<<4 * m->sms, 256, 0, m->stream>>>(m->X, m->count, kIn, acc, acc + 13);
    k_colstats<<<4 * m->sms, 256, 0, m->stream>>>(m->T, m->count, kOut, acc + 26, acc + 35);
    double h[44];
    cudaError_t e = cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    cudaFree(acc);
    if (e != cudaSuccess) return cfail(m, "normalization", e);
    float nrm[44];
    const double n = (double)m->count;
    for (int c = 0; c < 13; c++) {
        const double mu = h[c] / n, var = h[13 + c] / n - mu * mu;
        nrm[c] = (float)mu;
        nrm[13 + c] = var > 1e-24 ? (float)std::sqrt(var) : 1.f;
    }
    for (int c = 0; c < 9; c++) {
        const double mu = h[26 + c] / n, var = h[35 + c] / n - mu * mu;
        nrm[26 + c] = (float)mu;
        nrm[35 + c] = var > 1e-24 ? (float)std::sqrt(var) : 1.f;
    }
    CLK(m, cudaMemcpy(m->norm, nrm, sizeof(nrm), cudaMemcpyHostToDevice));
    if (norm_out) std::memcpy(norm_out, nrm, sizeof(nrm));
    return CHAN_OK;
}

int chan_closure_set_normalization(chan_closure *m, const float *norm)
{
    if (!m || !norm) return CHAN_EINVAL;
    CLK(m, cudaSetDevice(m->dev));
    CLK(m, cudaMemcpy(m->norm, norm, 44 * sizeof(float), cudaMemcpyHostToDevice));
    return CHAN_OK;
}

int chan_closure_get_normalization(chan_closure *m, float *norm)
{
    if (!m || !norm) return CHAN_EINVAL;
    CLK(m, cudaSetDevice(m->dev));
    CLK(m, cudaMemcpy(norm, m->norm, 44 * sizeof(float), cudaMemcpyDeviceToHost));
    return CHAN_OK;
}

int chan_closure_nparams(void) { return kNParam; }

int chan_closure_init(chan_closure *m, uint64_t seed)
{
    if (!m) return CHAN_EINVAL;
    std::vector<float> w(kNParam, 0.f);
    uint64_t st = seed;
    auto uni = [&](double lim) { return (float)(((splitmix(st) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0) * lim); };
    const double l1 = std::sqrt(6.0 / (kIn + kHid)), l2 = std::sqrt(6.0 / (kHid + kHid)), l3 = std::sqrt(6.0 / (kHid + kOut));
    for (int i = 0; i < kNW1; i++) w[i] = uni(l1);
    for (int i = 0; i < kNW2; i++) w[kOffW2 + i] = uni(l2);
    for (int i = 0; i < kNW3; i++) w[kOffW3 + i] = uni(l3);
    return chan_closure_set_params(m, w.data());
}

int chan_closure_set_params(chan_closure *m, const float *params)
{
    if (!m || !params) return CHAN_EINVAL;
    CLK(m, cudaSetDevice(m->dev));
    CLK(m, cudaMemcpy(m->w, params, (size_t)kNParam * sizeof(float), cudaMemcpyHostToDevice));
    CLK(m, cudaMemset(m->m, 0, 2 * (size_t)kNParam * sizeof(float)));
    m->adam_t = 0;
    int r = refresh_images(m);
    if (r) return r;
    CLK(m, cudaStreamSynchronize(m->stream));
    return CHAN_OK;
}

int chan_closure_get_params(chan_closure *m, float *params)
{
    if (!m || !params) return CHAN_EINVAL;
    CLK(m, cudaSetDevice(m->dev));
    CLK(m, cudaMemcpy(params, m->w, (size_t)kNParam * sizeof(float), cudaMemcpyDeviceToHost));
    return CHAN_OK;
}

int chan_closure_train(chan_closure *m, int32_t epochs, int32_t batch, double lr, uint64_t seed, double *losses)
{
    if (!m || epochs < 0 || batch < kTile || batch % kTile || !(lr > 0)) return CHAN_EINVAL;
    if (m->count < batch) { m->msg = "fewer samples than one batch"; return CHAN_EINVAL; }
    CLK(m, cudaSetDevice(m->dev));
    CLK(m, cudaMemsetAsync(m->err, 0, sizeof(int), m->stream));
    const long long n = m->count, nb = n / batch;
    uint64_t st = seed;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs; ep++) {
        // this epoch's order of the samples: row -> (a*row + b) mod n, a coprime to n
        long long a = (long long)(splitmix(st) % (uint64_t)n) | 1;
        while (gcd_ll(a, n) != 1) a = (a + 2) % n;
        const long long b = (long long)(splitmix(st) % (uint64_t)n);
        CLK(m, cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream));
        for (long long bi = 0; bi < nb; bi++) {
            CLK(m, cudaMemsetAsync(m->g, 0, (size_t)kNParam * sizeof(float), m->stream));
            MlpParams P = base_params(m);
            P.X = m->X; P.T = m->T; P.n = n;
            P.perm_a = a; P.perm_b = b;
            P.row0 = bi * batch; P.rows = batch;
            P.inv_count = 2.f / (9.f * (float)batch);
            int r = launch_mlp(m, P, true, m->stream);
            if (r) return r;
            m->adam_t++;
            const float c1 = 1.f - std::pow(b1, (float)m->adam_t), c2 = 1.f - std::pow(b2, (float)m->adam_t);
            k_adam<<<(kNParam + 255) / 256, 256, 0, m->stream>>>(m->w, m->m, m->v, m->g, kNParam, (float)lr, b1, b2,
                                                                   eps, c1, c2);
            CLK(m, cudaGetLastError());
            r = refresh_images(m);
            if (r) return r;
        }
        float l = 0.f;
        CLK(m, cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
        CLK(m, cudaStreamSynchronize(m->stream));
        if (losses) losses[ep] = (double)l / (9.0 * (double)batch * (double)nb);
        int r = check_err(m);
        if (r) return r;
    }
    return CHAN_OK;
}

int chan_closure_grad(chan_closure *m, const float *X, const float *T, int64_t n, float *grads, double *loss_sum)
{
    if (!m || !X || !T || n < 1) return CHAN_EINVAL;
    CLK(m, cudaSetDevice(m->dev));
    float *dX = nullptr, *dT = nullptr;
    CLK(m, cudaMalloc((void **)&dX, (size_t)n * kIn * sizeof(float)));
    CLK(m, cudaMalloc((void **)&dT, (size_t)n * kOut * sizeof(float)));
    CLK(m, cudaMemcpy(dX, X, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice));
    CLK(m, cudaMemcpy(dT, T, (size_t)n * kOut * sizeof(float), cudaMemcpyHostToDevice));
    CLK(m, cudaMemsetAsync(m->g, 0, (size_t)kNParam * sizeof(float), m->stream));
    CLK(m, cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream));
    CLK(m, cudaMemsetAsync(m->err, 0, sizeof(int), m->stream));
    MlpParams P = base_params(m);
    P.X = dX; P.T = dT; P.n = n; P.rows = n;
    P.inv_count = 2.f / (9.f * (float)n);
    int r = launch_mlp(m, P, true, m->stream);
    float l = 0.f;
    if (!r) r = check_err(m);
    if (!r && grads) CLK(m, cudaMemcpy(grads, m->g, (size_t)kNParam * sizeof(float), cudaMemcpyDeviceToHost));
    if (!r) CLK(m, cudaMemcpy(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
    cudaFree(dX);
    cudaFree(dT);
    if (loss_sum) *loss_sum = l;
    return r;
}

int chan_closure_infer(chan_closure *m, const float *X, int64_t n, float *Y)
{
    if (!m || !X || !Y || n < 1) return CHAN_EINVAL;
    CLK(m, cudaSetDevice(m->dev));
    float *dX = nullptr, *dY = nullptr;
    CLK(m, cudaMalloc((void **)&dX, (size_t)n * kIn * sizeof(float)));
    CLK(m, cudaMalloc((void **)&dY, (size_t)n * kOut * sizeof(float)));
    CLK(m, cudaMemcpy(dX, X, (size_t)n * kIn * sizeof(float), cudaMemcpyHostToDevice));
    CLK(m, cudaMemsetAsync(m->err, 0, sizeof(int), m->stream));
    int r = chan_internal_infer(m, dX, dY, n, false, m->stream, nullptr);
    if (!r) r = check_err(m);
    if (!r) CLK(m, cudaMemcpy(Y, dY, (size_t)n * kOut * sizeof(float), cudaMemcpyDeviceToHost));
    cudaFree(dX);
    cudaFree(dY);
    return r;
}

const char *chan_closure_last_error(chan_closure *m) { return m ? m->msg.c_str() : g_cl_error.c_str(); }

void chan_closure_free(chan_closure *m)
{
    if (!m) return;
    cudaSetDevice(m->dev);
    if (m->stream) cudaStreamSynchronize(m->stream);
    if (m->X) cudaFree(m->X);
    if (m->T) cudaFree(m->T);
    if (m->w) cudaFree(m->w);
    if (m->img) cudaFree(m->img);
    if (m->norm) cudaFree(m->norm);
    if (m->loss) cudaFree(m->loss);
    if (m->err) cudaFree(m->err);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
}

}  // extern "C"
