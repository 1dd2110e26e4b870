// lpc.cuh — kernels of the learned preconditioner: its network (inference and training) and
// the patch-level SGN operator the training loss is measured with.
//
// No counterpart in the reference. Tensors are NCHW FP32; weights are [Co][Ci][K][K] and are
// used as stored (the training loop stores BF16-rounded copies for the forward pass, so the
// arithmetic is BF16 weights with FP32 accumulation). Zero padding at tensor edges.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace wcb {

enum ConvMode { CM_DIRECT = 0, CM_POOL = 1, CM_UP = 2 };
enum ConvAct { ACT_NONE = 0, ACT_RELU = 1, ACT_SIG2 = 2 };

struct ConvArgs {
    const float* a;  // first input: ca channels; CM_POOL: at 2H x 2W (2x2 mean), CM_UP: at H/2 x W/2
    int ca, amode;
    const float* b;  // second input (concatenated after a), at H x W, or null
    int cb;
    const float* w;     // [co][ca + cb][k][k]
    const unsigned short* wre;  // the same as BF16 in the tensor-core kernel's [8 tiles][k k CP] order, or null
    const float* bias;  // [co] or null
    const float* gate;  // [n][co][H][W] or null: y = act(conv + bias) * gate
    float* y;           // [n][co][H][W]
    int co, H, W, N, act;
};

constexpr int CV_TH = 16;  // threads per tile edge (16 x 16 = 256 threads)
constexpr int CV_COB = 8;  // output channels per block
constexpr int CV_CIB = 8;  // input channels staged per pass

__device__ __forceinline__ float conv_input(const ConvArgs& p, int n, int c, int y, int x) {
    if ((unsigned)y >= (unsigned)p.H || (unsigned)x >= (unsigned)p.W) return 0.f;
    if (c < p.ca) {
        if (p.amode == CM_DIRECT) return p.a[(((size_t)n * p.ca + c) * p.H + y) * p.W + x];
        if (p.amode == CM_POOL) {
            const int W2 = 2 * p.W;
            const float* q = p.a + (((size_t)n * p.ca + c) * (2 * p.H) + 2 * y) * W2 + 2 * x;
            return 0.25f * ((q[0] + q[1]) + (q[W2] + q[W2 + 1]));
        }
        const int Hh = p.H / 2, Wh = p.W / 2;
        return p.a[(((size_t)n * p.ca + c) * Hh + y / 2) * Wh + x / 2];
    }
    return p.b[(((size_t)n * p.cb + (c - p.ca)) * p.H + y) * p.W + x];
}

// Direct convolution, register-blocked: a block computes a (16 P) x (16 P) tile of 8 output
// channels; each thread a P x P patch of all 8, from a (P + K - 1)^2 window of every staged input
// channel held in registers and the 8 weights of a tap read as two float4 (broadcast). P = 2 on
// large maps; P = 1 on the coarse levels, where a 32 x 32 tile would leave most SMs idle.
template <int K, int P>
__global__ void __launch_bounds__(CV_TH* CV_TH) conv_fwd_kernel(ConvArgs p) {
    constexpr int T = CV_TH * P, R = K / 2, TE = T + 2 * R, WIN = P + K - 1;
    __shared__ float tile[CV_CIB][TE][TE + 1];
    __shared__ __align__(16) float wsm[CV_CIB][K * K][CV_COB];
    const int ncog = (p.co + CV_COB - 1) / CV_COB;
    const int n = blockIdx.z / ncog, cog = blockIdx.z % ncog;
    const int x0 = blockIdx.x * T, y0 = blockIdx.y * T;
    const int tx = threadIdx.x % CV_TH, ty = threadIdx.x / CV_TH;
    const int ci_total = p.ca + p.cb;
    float acc[P][P][CV_COB];
#pragma unroll
    for (int a = 0; a < P; a++)
#pragma unroll
        for (int b = 0; b < P; b++)
#pragma unroll
            for (int o = 0; o < CV_COB; o++) acc[a][b][o] = 0.f;
    for (int c0 = 0; c0 < ci_total; c0 += CV_CIB) {
        const int nc = min(CV_CIB, ci_total - c0);
        for (int q = threadIdx.x; q < nc * TE * TE; q += CV_TH * CV_TH) {
            const int c = q / (TE * TE), r = q % (TE * TE);
            const int yy = y0 + r / TE - R, xx = x0 + r % TE - R;
            tile[c][r / TE][r % TE] = conv_input(p, n, c0 + c, yy, xx);
        }
        for (int q = threadIdx.x; q < CV_COB * CV_CIB * K * K; q += CV_TH * CV_TH) {
            const int o = q % CV_COB, r = q / CV_COB;
            const int c = r / (K * K), t = r % (K * K);
            const int co = cog * CV_COB + o, ci = c0 + c;
            wsm[c][t][o] = (co < p.co && ci < ci_total) ? p.w[((size_t)co * ci_total + ci) * K * K + t] : 0.f;
        }
        __syncthreads();
        for (int c = 0; c < nc; c++) {
            float win[WIN][WIN];
#pragma unroll
            for (int a = 0; a < WIN; a++)
#pragma unroll
                for (int b = 0; b < WIN; b++) win[a][b] = tile[c][P * ty + a][P * tx + b];
#pragma unroll
            for (int t = 0; t < K * K; t++) {
                const float4 w0 = *reinterpret_cast<const float4*>(&wsm[c][t][0]);
                const float4 w1 = *reinterpret_cast<const float4*>(&wsm[c][t][4]);
                const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
                for (int a = 0; a < P; a++)
#pragma unroll
                    for (int b = 0; b < P; b++) {
                        const float v = win[a + t / K][b + t % K];
#pragma unroll
                        for (int o = 0; o < CV_COB; o++) acc[a][b][o] = fmaf(v, wv[o], acc[a][b][o]);
                    }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < P; a++)
#pragma unroll
        for (int b = 0; b < P; b++) {
            const int x = x0 + P * tx + b, y = y0 + P * ty + a;
            if (x >= p.W || y >= p.H) continue;
#pragma unroll
            for (int o = 0; o < CV_COB; o++) {
                const int co = cog * CV_COB + o;
                if (co >= p.co) break;
                float v = acc[a][b][o] + (p.bias ? p.bias[co] : 0.f);
                if (p.act == ACT_RELU) v = fmaxf(v, 0.f);
                else if (p.act == ACT_SIG2) v = 2.f / (1.f + expf(-v));
                const size_t k = (((size_t)n * p.co + co) * p.H + y) * p.W + x;
                if (p.gate) v *= p.gate[k];
                p.y[k] = v;
            }
        }
}

// ---- inference convolution on the tensor cores ------------------------------------------------
//
// The same convolution as conv_fwd_kernel as an implicit GEMM on BF16 tensor-core MMAs
// (mma.sync m16n8k16, FP32 accumulation): M = pixels (one row of 16 per MMA), N = output channels
// (tiles of 8), K = taps x input channels (k = tap * CP + c, channels padded to CP, a multiple of
// 16, so one K step is 16 channels of one tap). The block stages its 16 x 8 pixel tile plus halo
// with the channels innermost (pixel stride CP + 2 halves: conflict-free 32-bit reads of channel
// pairs) and all weights reordered to the same K, BF16, in shared memory; each warp owns two
// pixel rows. The small channel counts of this network leave it memory-bound: the tensor cores
// take the arithmetic off the FMA pipes.
constexpr int CM_TX = 16, CM_TY = 16, CM_NT = 256, CM_NMAX = 8;  // N tiles of 8: up to 64 channels

__device__ __forceinline__ unsigned short bf16_bits(float x) {  // nearest, ties to even (finite x)
    const unsigned a = __float_as_uint(x);
    return (unsigned short)((a + 0x7FFFu + ((a >> 16) & 1u)) >> 16);
}

__device__ __forceinline__ void mma_bf16_16816(float* d, const unsigned* a, const unsigned* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__host__ __device__ inline int conv_mma_cp(int ci) { return (ci + 15) / 16 * 16; }

// Shared memory of one block (bytes): inputs [TY + 2R][TX + 2R][CP + 2], weights [8 nt][KK CP].
__host__ __device__ inline size_t conv_mma_smem(int ci, int co, int kk) {
    const int r = kk == 9 ? 1 : 0, cp = conv_mma_cp(ci);
    return ((size_t)(CM_TY + 2 * r) * (CM_TX + 2 * r) * (cp + 2) + (size_t)((co + 7) / 8) * 8 * kk * cp) * 2;
}

// The weights [co][ci][tap] (FP32 holding BF16 values) as BF16 in the order [8 ntl][tap CP + c].
__global__ void conv_mma_weights_kernel(const float* __restrict__ w, int co_n, int ci_n, int kk, int ntl,
                                        unsigned short* __restrict__ out) {
    const int cp = conv_mma_cp(ci_n), kp = kk * cp;
    const int total = ntl * 8 * kp;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
        const int co = q / kp, k = q % kp;
        const int tap = k / cp, c = k - tap * cp;
        out[q] = (co < co_n && c < ci_n) ? (unsigned short)(__float_as_uint(w[((size_t)co * ci_n + c) * kk + tap]) >> 16)
                                        : (unsigned short)0;
    }
}

template <int KK, int NTL>  // taps: 9 (3x3) or 1 (1x1); N tiles of 8 channels: 1, 2, 4 or 8
__global__ void __launch_bounds__(CM_NT) conv_mma_kernel(ConvArgs p) {
    constexpr int R = KK == 9 ? 1 : 0, EW = CM_TX + 2 * R, EH = CM_TY + 2 * R;
    extern __shared__ __align__(16) unsigned short cm_smem[];
    const int ci_total = p.ca + p.cb;
    const int CP = conv_mma_cp(ci_total), PS = CP + 2, Kp = KK * CP;
    constexpr int ntiles = NTL;
    unsigned short* in_s = cm_smem;                         // [EH][EW][PS]
    unsigned short* w_s = cm_smem + (size_t)EH * EW * PS;   // [8 ntiles][Kp]
    const int n = blockIdx.z;
    const int x0 = blockIdx.x * CM_TX, y0 = blockIdx.y * CM_TY;
    for (int q = threadIdx.x; q < ci_total * EH * EW; q += CM_NT) {  // x fastest: coalesced reads
        const int c = q / (EH * EW), r = q % (EH * EW);
        const int yy = y0 + r / EW - R, xx = x0 + r % EW - R;
        float v = 0.f;
        if ((unsigned)yy < (unsigned)p.H && (unsigned)xx < (unsigned)p.W) {
            if (c >= p.ca) v = __ldg(p.b + (((size_t)n * p.cb + (c - p.ca)) * p.H + yy) * p.W + xx);
            else if (p.amode == CM_UP) v = __ldg(p.a + (((size_t)n * p.ca + c) * (p.H / 2) + yy / 2) * (p.W / 2) + xx / 2);
            else v = conv_input(p, n, c, yy, xx);
        }
        in_s[r * PS + c] = bf16_bits(v);
    }
    for (int q = threadIdx.x; q < (CP - ci_total) * EH * EW; q += CM_NT)  // padding channels
        in_s[(q % (EH * EW)) * PS + ci_total + q / (EH * EW)] = 0;
    {  // the weights, already in this kernel's order: 16-byte copies (8 tiles x Kp is a multiple of 8)
        const uint4* src = reinterpret_cast<const uint4*>(p.wre);
        uint4* dst = reinterpret_cast<uint4*>(w_s);
        for (int q = threadIdx.x; q < ntiles * Kp; q += CM_NT) dst[q] = __ldg(src + q);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane >> 2, tig = lane & 3;
    float acc[2][NTL][4];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
        for (int t = 0; t < NTL; t++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[r][t][e] = 0.f;
    for (int kb = 0; kb < Kp; kb += 16) {
        const int tap = kb / CP, c0 = kb - tap * CP + tig * 2;
        const int dy = KK == 9 ? tap / 3 : 0, dx = KK == 9 ? tap - 3 * (tap / 3) : 0;
        unsigned b[NTL][2];
#pragma unroll
        for (int t = 0; t < NTL; t++) {
            const unsigned* wrow = reinterpret_cast<const unsigned*>(w_s + (size_t)(t * 8 + grp) * Kp + kb + tig * 2);
            b[t][0] = wrow[0];
            b[t][1] = wrow[4];  // k + 8
        }
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int row = warp * 2 + r + dy;
            const unsigned* lo = reinterpret_cast<const unsigned*>(in_s + ((size_t)row * EW + grp + dx) * PS + c0);
            const unsigned* hi = reinterpret_cast<const unsigned*>(in_s + ((size_t)row * EW + grp + 8 + dx) * PS + c0);
            const unsigned a[4] = {lo[0], hi[0], lo[4], hi[4]};  // (pixel, k..k+1), (pixel+8, ..), (+8 channels)
#pragma unroll
            for (int t = 0; t < NTL; t++) mma_bf16_16816(acc[r][t], a, b[t]);
        }
    }
    // D[pixel][channel]: pixels grp and grp + 8 of the warp's two rows, channels tig * 2 + {0, 1}
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int y = y0 + warp * 2 + r;
#pragma unroll
        for (int t = 0; t < NTL; t++) {
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int x = x0 + grp + (e >= 2 ? 8 : 0);
                const int co = t * 8 + tig * 2 + (e & 1);
                if (x >= p.W || y >= p.H || co >= p.co) continue;
                float v = acc[r][t][e] + (p.bias ? p.bias[co] : 0.f);
                if (p.act == ACT_RELU) v = fmaxf(v, 0.f);
                else if (p.act == ACT_SIG2) v = 2.f / (1.f + expf(-v));
                const size_t kidx = (((size_t)n * p.co + co) * p.H + y) * p.W + x;
                if (p.gate) v *= p.gate[kidx];
                p.y[kidx] = v;
            }
        }
    }
}

// ---- the solver's inference path: channels-innermost BF16 activations ----------------------
//
// The same implicit GEMM as conv_mma_kernel on activations stored NHWC in BF16 (a pixel's
// channels contiguous, channel stride = the channel count, 2 or a multiple of 8): the staging
// moves 16-byte groups of 8 channels (one load and one shared store each, instead of one scalar
// load per element from NCHW FP32), a pooled input is the mean of four such groups, and the
// epilogue writes each thread's channel pairs as 32-bit words, contiguous across the warp. The
// numerics are those of conv_mma_kernel: every input is a BF16 number, products accumulate in
// FP32, and the output is rounded to BF16 once (the network's last layer writes FP32).
struct ConvH {
    const unsigned short* a;  // ca channels, NHWC; CM_POOL: at 2H x 2W (2x2 mean), CM_UP: at H/2 x W/2
    int ca, amode;
    const unsigned short* b;  // cb channels at H x W (concatenated after a), or null
    int cb;
    const unsigned short* wre;  // weights, BF16, [8 ntiles][k k CP] (conv_mma_weights_kernel)
    const float* bias;          // [co] or null
    const unsigned short* gate; // co channels, NHWC, or null: y = act(conv + bias) * gate
    unsigned short* y;          // co channels, NHWC BF16 ...
    float* yf;                  // ... or FP32 (non-null: the network's output)
    const int* done;            // or null: the solve this application serves has ended, skip it
    const float* out_w;         // or null: an 8-channel layer followed by the 2 x 8 1x1 output layer,
                                // applied in the epilogue; yf then gets its FP32 output
    const unsigned short* wre2; // conv_enc0_kernel: the second layer's weights (wre: the first's)
    int co, H, W, N, act;
};

__host__ __device__ inline int conv_h_ps(int cp) { return cp + 8; }  // pixel stride in halves: 16-byte rows

__device__ __forceinline__ float bf16_lo(unsigned v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi(unsigned v) { return __uint_as_float(v & 0xFFFF0000u); }
__device__ __forceinline__ unsigned bf16_pack(float lo, float hi) {  // cvt.rn.bf16x2.f32: nearest, ties to even
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned*>(&v);
}
// the mean of four groups of 8 BF16 channels, in conv_input's order, rounded to BF16
__device__ __forceinline__ unsigned pool_word(unsigned a, unsigned b, unsigned c, unsigned d) {
    const float lo = 0.25f * ((bf16_lo(a) + bf16_lo(b)) + (bf16_lo(c) + bf16_lo(d)));
    const float hi = 0.25f * ((bf16_hi(a) + bf16_hi(b)) + (bf16_hi(c) + bf16_hi(d)));
    return bf16_pack(lo, hi);
}

// 16-byte global -> shared copy that does not hold a register (src_bytes 0: zero fill)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}
// Four 8x8 BF16 matrices from shared memory, one 16-byte row address per lane
__device__ __forceinline__ void ldmatrix_x4(unsigned* r, const void* row) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(row);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(sa));
}
__device__ __forceinline__ void ldmatrix_x2(unsigned* r, const void* row) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(row);
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r[0]), "=r"(r[1]) : "r"(sa));
}

// The layer's weights ([8 NTL rows][KP], BF16) into shared memory with rows padded to KP + 8
// halves: row starts then fall 4 banks apart, so the B-fragment reads are conflict-free.
template <int NTL, int KP>
__device__ __forceinline__ void stage_weights(unsigned short* w_s, const unsigned short* wre) {
    constexpr int G = KP / 8;  // 16-byte groups a row
    const uint4* src = reinterpret_cast<const uint4*>(wre);
    for (int q = threadIdx.x; q < 8 * NTL * G; q += CM_NT) {
        const int row = q / G, c = q - row * G;
        cp_async16(w_s + row * (KP + 8) + c * 8, src + q, 16);
    }
}

// B fragments of the NTL output tiles at K offset kb: ldmatrix on the [n][k] weight rows gives
// (k = 2 tig, 2 tig + 1; n = grp) and its k + 8 partner directly; one x4 covers two tiles.
template <int NTL, int KP>
__device__ __forceinline__ void load_b(unsigned (&b)[NTL][2], const unsigned short* w_s, int kb, int lane) {
    constexpr int WS = KP + 8;
    const int koff = ((lane >> 3) & 1) * 8;
    if constexpr (NTL == 1) {
        ldmatrix_x2(b[0], w_s + (lane & 7) * WS + kb + koff);
    } else {
#pragma unroll
        for (int t = 0; t < NTL; t += 2) {
            unsigned r[4];
            ldmatrix_x4(r, w_s + (t * 8 + ((lane >> 4) & 1) * 8 + (lane & 7)) * WS + kb + koff);
            b[t][0] = r[0];
            b[t][1] = r[1];
            b[t + 1][0] = r[2];
            b[t + 1][1] = r[3];
        }
    }
}

// Rows of 16 pixels per warp: tall tiles for the 8-channel layers (fewer halo cells and less
// fixed work per pixel); shorter ones as the output widens, so that the accumulators leave room
// for more resident blocks and the coarse levels still give every SM several tiles.
__host__ __device__ constexpr int conv_h_rows(int ntl) { return ntl == 1 ? 4 : 2; }
// The decoder's concat(up(a), b) kernel stages a quarter-size coarse box, so taller tiles pay
// there up to two output tiles (measured).
__host__ __device__ constexpr int conv_up_rows(int ntl) { return ntl <= 2 ? 4 : 2; }

// Shared memory of the channels-innermost convolution (bytes): the input box, the weights and,
// for a gated layer, the gate tile ([pixel][co]).
__host__ __device__ inline size_t conv_h_smem2(int ci, int co, int kk, bool gated, int rw = 0) {
    const int r = kk == 9 ? 1 : 0, cp = conv_mma_cp(ci), ntl = (co + 7) / 8;
    const int th = 8 * (rw ? rw : conv_h_rows(ntl));
    const size_t box = (size_t)(th + 2 * r) * (CM_TX + 2 * r) * conv_h_ps(cp);
    return (box + (size_t)ntl * 8 * (kk * cp + 8) + (gated ? (size_t)th * CM_TX * ntl * 8 : 0)) * 2;
}

// The convolution's epilogue: bias, activation, gate (from the staged gate tile), and the BF16
// (or FP32, or fused 1x1 output) store of the warp's RW rows of 16 pixels of the tile at (x0, y0).
template <int NTL, int RW>
__device__ __forceinline__ void conv_h_epilogue(const ConvH& p, float (&acc)[RW][NTL][4], const unsigned short* g_s,
                                                int n, int x0, int y0) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane >> 2, tig = lane & 3;
    // D[pixel][channel]: pixels grp and grp + 8 of the warp's rows, channels t * 8 + tig * 2 + {0, 1}
    float bias[NTL][2];
#pragma unroll
    for (int t = 0; t < NTL; t++) {
        const int co = t * 8 + tig * 2;
        bias[t][0] = p.bias && co < p.co ? __ldg(p.bias + co) : 0.f;
        bias[t][1] = p.bias && co < p.co ? __ldg(p.bias + co + 1) : 0.f;
    }
    if constexpr (NTL == 1) {
        if (p.out_w) {  // the output layer on this layer's 8 gated channels: a dot over the lane quad
            const int co = tig * 2;
            const float w00 = __ldg(p.out_w + co), w01 = __ldg(p.out_w + co + 1);
            const float w10 = __ldg(p.out_w + 8 + co), w11 = __ldg(p.out_w + 8 + co + 1);
#pragma unroll
            for (int r = 0; r < RW; r++) {
                const int y = y0 + warp * RW + r;
#pragma unroll
                for (int half = 0; half < 2; half++) {
                    const int x = x0 + grp + 8 * half;
                    float v0 = acc[r][0][2 * half] + bias[0][0];
                    float v1 = acc[r][0][2 * half + 1] + bias[0][1];
                    if (p.act == ACT_RELU) {
                        v0 = fmaxf(v0, 0.f);
                        v1 = fmaxf(v1, 0.f);
                    }
                    if (p.gate) {  // the gate tile covers every pixel of the tile (zero outside)
                        const int lp = (warp * RW + r) * CM_TX + grp + 8 * half;
                        const unsigned gw = *reinterpret_cast<const unsigned*>(g_s + lp * p.co + co);
                        v0 *= bf16_lo(gw);
                        v1 *= bf16_hi(gw);
                    }
                    float o0 = w00 * v0 + w01 * v1, o1 = w10 * v0 + w11 * v1;
                    o0 += __shfl_xor_sync(0xffffffffu, o0, 1);
                    o1 += __shfl_xor_sync(0xffffffffu, o1, 1);
                    o0 += __shfl_xor_sync(0xffffffffu, o0, 2);
                    o1 += __shfl_xor_sync(0xffffffffu, o1, 2);
                    if (tig == 0 && y < p.H && x < p.W)
                        *reinterpret_cast<float2*>(p.yf + ((n * p.H + y) * p.W + x) * 2) = make_float2(o0, o1);
                }
            }
            return;
        }
    }
#pragma unroll
    for (int r = 0; r < RW; r++) {
        const int y = y0 + warp * RW + r;
        if (y >= p.H) continue;
        const int row = (n * p.H + y) * p.W;
#pragma unroll
        for (int half = 0; half < 2; half++) {
            const int x = x0 + grp + 8 * half;
            if (x >= p.W) continue;
            const int pix = (row + x) * p.co;
#pragma unroll
            for (int t = 0; t < NTL; t++) {
                const int co = t * 8 + tig * 2;
                if (co >= p.co) continue;
                float v0 = acc[r][t][2 * half] + bias[t][0];
                float v1 = acc[r][t][2 * half + 1] + bias[t][1];
                if (p.act == ACT_RELU) {
                    v0 = fmaxf(v0, 0.f);
                    v1 = fmaxf(v1, 0.f);
                } else if (p.act == ACT_SIG2) {
                    v0 = 2.f / (1.f + expf(-v0));
                    v1 = 2.f / (1.f + expf(-v1));
                }
                if (p.gate) {
                    const int lp = (warp * RW + r) * CM_TX + grp + 8 * half;
                    const unsigned gw = *reinterpret_cast<const unsigned*>(g_s + lp * p.co + co);
                    v0 *= bf16_lo(gw);
                    v1 *= bf16_hi(gw);
                }
                if (p.yf) *reinterpret_cast<float2*>(p.yf + pix + co) = make_float2(v0, v1);
                else *reinterpret_cast<unsigned*>(p.y + pix + co) = bf16_pack(v0, v1);
            }
        }
    }
}

// KK taps (9 or 1), NTL tiles of 8 output channels, CP input channels padded to 16: all index
// arithmetic is compile-time and 32-bit (a map of up to 2^31 values). A block computes a tile of
// 16 x (8 RW) pixels, each warp RW rows of 16 (RW = 1 for maps too small to give every SM two
// blocks of the usual height); its halo box is staged with cp.async (pooled inputs through
// registers), A fragments are read with ldmatrix, and values are rounded to BF16 by the hardware
// conversion (round to nearest even, as bf16_bits).
template <int KK, int NTL, int CP, int RW = conv_h_rows(NTL)>
__global__ void __launch_bounds__(CM_NT, 2) conv_h_kernel(ConvH p) {
    if (p.done && *p.done) return;
    constexpr int TH = 8 * RW;
    constexpr int R = KK == 9 ? 1 : 0, EW = CM_TX + 2 * R, EH = TH + 2 * R;
    constexpr int PS = CP + 8, KP = KK * CP, GROUPS = CP / 8, UNITS = EH * EW * GROUPS;
    constexpr int PER = (UNITS + CM_NT - 1) / CM_NT;
    extern __shared__ __align__(16) unsigned short cm_smem[];
    unsigned short* in_s = cm_smem;             // [EH][EW][PS]
    unsigned short* w_s = cm_smem + EH * EW * PS;  // [8 NTL][KP]
    unsigned short* g_s = w_s + 8 * NTL * (KP + 8);      // gated layers: [TH][16][co]
    const int ci_total = p.ca + p.cb;
    const int n = blockIdx.z;
    const int x0 = blockIdx.x * CM_TX, y0 = blockIdx.y * TH;
    const bool two = p.ca == 2;
    stage_weights<NTL, KP>(w_s, p.wre);
    if (p.gate) {  // the tile's gate, in flight with the input box
        const int gg = p.co / 8;
        for (int q = threadIdx.x; q < TH * CM_TX * gg; q += CM_NT) {
            const int pix = q / gg, c0 = (q - pix * gg) * 8;
            const int y = y0 + pix / CM_TX, x = x0 + pix % CM_TX;
            const bool in = y < p.H && x < p.W;
            cp_async16(g_s + pix * p.co + c0, in ? p.gate + ((n * p.H + y) * p.W + x) * p.co + c0 : p.gate, in ? 16 : 0);
        }
    }
    const int Hs = p.amode == CM_POOL ? 2 * p.H : p.amode == CM_UP ? p.H / 2 : p.H;  // a's map
    const int Ws = p.amode == CM_POOL ? 2 * p.W : p.amode == CM_UP ? p.W / 2 : p.W;
    const int abase = n * Hs * Ws, bbase = n * p.H * p.W;
#pragma unroll 4
    for (int u = 0; u < PER; u++) {
        const int q = threadIdx.x + u * CM_NT;
        if (UNITS % CM_NT != 0 && q >= UNITS) break;
        const int r = q / GROUPS, c0 = (q % GROUPS) * 8;
        const int yy = y0 + r / EW - R, xx = x0 + r % EW - R;
        unsigned short* dst = in_s + r * PS + c0;
        const bool inside = (unsigned)yy < (unsigned)p.H && (unsigned)xx < (unsigned)p.W && c0 < ci_total;
        if (inside && c0 < p.ca && (p.amode == CM_POOL || two)) {
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (p.amode == CM_POOL) {
                const int at = abase + (2 * yy) * Ws + 2 * xx;
                if (two) {
                    const unsigned* w = reinterpret_cast<const unsigned*>(p.a);
                    v.x = pool_word(__ldg(w + at), __ldg(w + at + 1), __ldg(w + at + Ws), __ldg(w + at + Ws + 1));
                } else {
                    const uint4* w = reinterpret_cast<const uint4*>(p.a);
                    const int g = p.ca / 8, o = c0 / 8;
                    const uint4 a0 = __ldg(w + at * g + o), a1 = __ldg(w + (at + 1) * g + o);
                    const uint4 a2 = __ldg(w + (at + Ws) * g + o), a3 = __ldg(w + (at + Ws + 1) * g + o);
                    v = make_uint4(pool_word(a0.x, a1.x, a2.x, a3.x), pool_word(a0.y, a1.y, a2.y, a3.y),
                                   pool_word(a0.z, a1.z, a2.z, a3.z), pool_word(a0.w, a1.w, a2.w, a3.w));
                }
            } else {
                const int at = abase + (p.amode == CM_UP ? (yy / 2) * Ws + xx / 2 : yy * Ws + xx);
                v.x = __ldg(reinterpret_cast<const unsigned*>(p.a) + at);
            }
            *reinterpret_cast<uint4*>(dst) = v;
        } else {
            const unsigned short* src = p.a;  // a valid address when nothing is read
            if (inside) {
                if (c0 >= p.ca) src = p.b + (bbase + yy * p.W + xx) * p.cb + (c0 - p.ca);
                else src = p.a + (abase + (p.amode == CM_UP ? (yy / 2) * Ws + xx / 2 : yy * Ws + xx)) * p.ca + c0;
            }
            cp_async16(dst, src, inside ? 16 : 0);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int lpix = (lane & 7) + ((lane >> 3) & 1) * 8, lk = (lane >> 4) * 8;  // ldmatrix row of this lane
    float acc[RW][NTL][4];
#pragma unroll
    for (int r = 0; r < RW; r++)
#pragma unroll
        for (int t = 0; t < NTL; t++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[r][t][e] = 0.f;
#pragma unroll 3
    for (int tap = 0; tap < KK; tap++) {
        const int dy = KK == 9 ? tap / 3 : 0, dx = KK == 9 ? tap % 3 : 0;
#pragma unroll
        for (int cb = 0; cb < CP; cb += 16) {
            const int kb = tap * CP + cb;
            unsigned b[NTL][2];
            load_b<NTL, KP>(b, w_s, kb, lane);
#pragma unroll
            for (int r = 0; r < RW; r++) {
                unsigned a[4];
                ldmatrix_x4(a, in_s + ((warp * RW + r + dy) * EW + lpix + dx) * PS + cb + lk);
#pragma unroll
                for (int t = 0; t < NTL; t++) mma_bf16_16816(acc[r][t], a, b[t]);
            }
        }
    }
    conv_h_epilogue<NTL, RW>(p, acc, g_s, n, x0, y0);
}

// A decoder convolution over concat(up(a), b) (3x3; a at half resolution with CPA channels, a
// multiple of 16; b with the rest of the CP input channels, zero-padded): the a-part is staged
// once per coarse pixel of the tile (a quarter of the fine halo box) and its A fragments are read
// by ldmatrix straight from the coarse box, each lane addressing the coarse pixel its fine pixel
// repeats; the b-part is staged and read as in conv_h_kernel. Same arithmetic and K order as
// conv_h_kernel on the upsampled map.
__host__ __device__ inline size_t conv_up_smem(int cpa, int cp, int co, bool gated) {
    const int ntl = (co + 7) / 8, th = 8 * conv_up_rows(ntl);
    const size_t abox = (size_t)(th / 2 + 2) * (CM_TX / 2 + 2) * (cpa + 8);
    const size_t bbox = (size_t)(th + 2) * (CM_TX + 2) * (cp - cpa + 8);
    return (abox + bbox + (size_t)ntl * 8 * (9 * cp + 8) + (gated ? (size_t)th * CM_TX * ntl * 8 : 0)) * 2;
}

template <int NTL, int CP, int CPA>
__global__ void __launch_bounds__(CM_NT, 2) conv_up_kernel(ConvH p) {
    if (p.done && *p.done) return;
    constexpr int RW = conv_up_rows(NTL), TH = 8 * RW;
    constexpr int EW = CM_TX + 2, EH = TH + 2, CEW = CM_TX / 2 + 2, CEH = TH / 2 + 2;
    constexpr int CPB = CP - CPA, PSA = CPA + 8, PSB = CPB + 8, KP = 9 * CP;
    constexpr int GA = CPA / 8, GB = CPB / 8, UA = CEH * CEW * GA, UB = EH * EW * GB;
    extern __shared__ __align__(16) unsigned short cm_smem[];
    unsigned short* a_s = cm_smem;               // [CEH][CEW][PSA]
    unsigned short* b_s = a_s + CEH * CEW * PSA;  // [EH][EW][PSB]
    unsigned short* w_s = b_s + EH * EW * PSB;    // [8 NTL][KP]
    unsigned short* g_s = w_s + 8 * NTL * (KP + 8);     // gated layers: [TH][16][co]
    const int n = blockIdx.z;
    const int x0 = blockIdx.x * CM_TX, y0 = blockIdx.y * TH;
    const int Hc = p.H / 2, Wc = p.W / 2;
    const int cx0 = (x0 >> 1) - 1, cy0 = (y0 >> 1) - 1;
    stage_weights<NTL, KP>(w_s, p.wre);
    if (p.gate) {
        const int gg = p.co / 8;
        for (int q = threadIdx.x; q < TH * CM_TX * gg; q += CM_NT) {
            const int pix = q / gg, c0 = (q - pix * gg) * 8;
            const int y = y0 + pix / CM_TX, x = x0 + pix % CM_TX;
            const bool in = y < p.H && x < p.W;
            cp_async16(g_s + pix * p.co + c0, in ? p.gate + ((n * p.H + y) * p.W + x) * p.co + c0 : p.gate, in ? 16 : 0);
        }
    }
    for (int q = threadIdx.x; q < UA; q += CM_NT) {  // the coarse box of a
        const int r = q / GA, c0 = (q % GA) * 8;
        const int cy = cy0 + r / CEW, cx = cx0 + r % CEW;
        const bool in = (unsigned)cy < (unsigned)Hc && (unsigned)cx < (unsigned)Wc;
        cp_async16(a_s + r * PSA + c0, in ? p.a + ((n * Hc + cy) * Wc + cx) * p.ca + c0 : p.a, in ? 16 : 0);
    }
    for (int q = threadIdx.x; q < UB; q += CM_NT) {  // the fine box of b (channels past cb: zero)
        const int r = q / GB, c0 = (q % GB) * 8;
        const int yy = y0 + r / EW - 1, xx = x0 + r % EW - 1;
        const bool in = (unsigned)yy < (unsigned)p.H && (unsigned)xx < (unsigned)p.W && c0 < p.cb;
        cp_async16(b_s + r * PSB + c0, in ? p.b + ((n * p.H + yy) * p.W + xx) * p.cb + c0 : p.b, in ? 16 : 0);
    }
    cp_async_wait_all();
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int lpix = (lane & 7) + ((lane >> 3) & 1) * 8, lk = (lane >> 4) * 8;
    float acc[RW][NTL][4];
#pragma unroll
    for (int r = 0; r < RW; r++)
#pragma unroll
        for (int t = 0; t < NTL; t++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[r][t][e] = 0.f;
#pragma unroll 3
    for (int tap = 0; tap < 9; tap++) {
        const int dy = tap / 3, dx = tap % 3;
        const int ccol = (lpix + dx + 1) >> 1;  // the coarse column of this lane's fine pixel (box coordinates)
#pragma unroll
        for (int cb = 0; cb < CP; cb += 16) {
            const int kb = tap * CP + cb;
            unsigned b[NTL][2];
            load_b<NTL, KP>(b, w_s, kb, lane);
#pragma unroll
            for (int r = 0; r < RW; r++) {
                const int frow = warp * RW + r + dy;  // fine box row
                unsigned a[4];
                if (cb < CPA) ldmatrix_x4(a, a_s + (((frow + 1) >> 1) * CEW + ccol) * PSA + cb + lk);
                else ldmatrix_x4(a, b_s + (frow * EW + lpix + dx) * PSB + (cb - CPA) + lk);
#pragma unroll
                for (int t = 0; t < NTL; t++) mma_bf16_16816(acc[r][t], a, b[t]);
            }
        }
    }
    conv_h_epilogue<NTL, RW>(p, acc, g_s, n, x0, y0);
}

// ---- 3x3 convolutions of an 8-channel input: two taps per K step ---------------------------
//
// (A two-channel input, the network's own and the gates' features, takes the same kernel with
// its channels zero-padded to 8 in the box: 5 K steps instead of 9 channel-padded ones.)
//
// With 8 input channels a K step of 16 holds two taps (k = tap * 8 + c; the ninth tap's partner
// has zero weights), so the halo box needs no channel padding (16 bytes a pixel) and a layer
// takes 5 K steps instead of 9: ldmatrix lanes 0-15 address the pixels of the first tap, lanes
// 16-31 those of the second. Same products and FP32 accumulation as conv_h_kernel, in another
// order of the sum.
constexpr int P8_KP = 80;  // 9 taps x 8 channels, padded to a multiple of 16

__global__ void conv_p8_weights_kernel(const float* __restrict__ w, int co_n, int ci_n, int ntl,
                                       unsigned short* __restrict__ out) {  // ci_n: 8, or 2 (zero-padded)
    const int total = ntl * 8 * P8_KP;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
        const int co = q / P8_KP, k = q % P8_KP, tap = k / 8, c = k % 8;
        out[q] = (co < co_n && tap < 9 && c < ci_n)
                     ? (unsigned short)(__float_as_uint(w[((size_t)co * ci_n + c) * 9 + tap]) >> 16)
                     : (unsigned short)0;
    }
}

__host__ __device__ inline size_t conv_p8_smem(int co, bool gated) {
    const int ntl = (co + 7) / 8, th = 8 * conv_h_rows(ntl);
    return ((size_t)(th + 2) * (CM_TX + 2) * 8 + (size_t)ntl * 8 * (P8_KP + 8) + (gated ? (size_t)th * CM_TX * ntl * 8 : 0)) * 2;
}

template <int NTL>
__global__ void __launch_bounds__(CM_NT, 2) conv_p8_kernel(ConvH p) {
    if (p.done && *p.done) return;
    constexpr int RW = conv_h_rows(NTL), TH = 8 * RW, EW = CM_TX + 2, EH = TH + 2, UNITS = EH * EW;
    extern __shared__ __align__(16) unsigned short cm_smem[];
    unsigned short* in_s = cm_smem;           // [EH][EW][8]
    unsigned short* w_s = in_s + UNITS * 8;   // [8 NTL][P8_KP]
    unsigned short* g_s = w_s + 8 * NTL * (P8_KP + 8);
    const int n = blockIdx.z;
    const int x0 = blockIdx.x * CM_TX, y0 = blockIdx.y * TH;
    stage_weights<NTL, P8_KP>(w_s, p.wre);
    if (p.gate) {
        const int gg = p.co / 8;
        for (int q = threadIdx.x; q < TH * CM_TX * gg; q += CM_NT) {
            const int pix = q / gg, c0 = (q - pix * gg) * 8;
            const int y = y0 + pix / CM_TX, x = x0 + pix % CM_TX;
            const bool in = y < p.H && x < p.W;
            cp_async16(g_s + pix * p.co + c0, in ? p.gate + ((n * p.H + y) * p.W + x) * p.co + c0 : p.gate, in ? 16 : 0);
        }
    }
    const bool pool = p.amode == CM_POOL;
    const int Ws = pool ? 2 * p.W : p.W;
    const int abase = n * (pool ? 2 * p.H : p.H) * Ws;
    for (int q = threadIdx.x; q < UNITS; q += CM_NT) {
        const int yy = y0 + q / EW - 1, xx = x0 + q % EW - 1;
        const bool in = (unsigned)yy < (unsigned)p.H && (unsigned)xx < (unsigned)p.W;
        uint4* dst = reinterpret_cast<uint4*>(in_s + q * 8);
        if (p.ca == 2) {  // a two-channel input, zero-padded to 8 in the box
            *dst = make_uint4(in ? __ldg(reinterpret_cast<const unsigned*>(p.a) + abase + yy * Ws + xx) : 0u, 0u, 0u, 0u);
        } else if (pool) {
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (in) {
                const uint4* w = reinterpret_cast<const uint4*>(p.a);
                const int at = abase + (2 * yy) * Ws + 2 * xx;
                const uint4 a0 = __ldg(w + at), a1 = __ldg(w + at + 1), a2 = __ldg(w + at + Ws), a3 = __ldg(w + at + Ws + 1);
                v = make_uint4(pool_word(a0.x, a1.x, a2.x, a3.x), pool_word(a0.y, a1.y, a2.y, a3.y),
                               pool_word(a0.z, a1.z, a2.z, a3.z), pool_word(a0.w, a1.w, a2.w, a3.w));
            }
            *dst = v;
        } else {
            cp_async16(dst, in ? p.a + (abase + yy * Ws + xx) * 8 : p.a, in ? 16 : 0);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int lpix = (lane & 7) + ((lane >> 3) & 1) * 8, second = lane >> 4;  // ldmatrix row: pixel, which tap
    float acc[RW][NTL][4];
#pragma unroll
    for (int r = 0; r < RW; r++)
#pragma unroll
        for (int t = 0; t < NTL; t++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[r][t][e] = 0.f;
#pragma unroll
    for (int j = 0; j < 5; j++) {
        const int tap = min(2 * j + second, 8);  // the ninth tap's partner: zero weights
        const int dy = tap / 3, dx = tap - 3 * (tap / 3);
        unsigned b[NTL][2];
        load_b<NTL, P8_KP>(b, w_s, j * 16, lane);
#pragma unroll
        for (int r = 0; r < RW; r++) {
            unsigned a[4];
            ldmatrix_x4(a, in_s + ((warp * RW + r + dy) * EW + lpix + dx) * 8);
#pragma unroll
            for (int t = 0; t < NTL; t++) mma_bf16_16816(acc[r][t], a, b[t]);
        }
    }
    conv_h_epilogue<NTL, RW>(p, acc, g_s, n, x0, y0);
}

// The network's first two layers in one launch: a = conv3x3(x) over the 2-channel input (no bias,
// no activation, 8 channels out) and y = conv3x3(a) * gate (8 -> 8). A block stages x over its
// tile plus a halo of 2, computes a over the tile plus a halo of 1 into shared memory (rounded to
// BF16, zero outside the map, exactly what the two-launch path stores and re-reads), then the
// second layer from there: the 8-channel map a never goes through HBM. Both layers take two taps
// per K step in conv_p8_kernel's order, so the result is bit-identical to the two launches.
__host__ __device__ inline size_t conv_enc0_smem() {
    constexpr int th = 8 * conv_h_rows(1);
    return ((size_t)(th + 4) * (CM_TX + 4) * 8 + (size_t)(th + 2) * (CM_TX + 2) * 8 + 2 * (size_t)8 * (P8_KP + 8) +
            (size_t)th * CM_TX * 8) * 2;
}

__global__ void __launch_bounds__(CM_NT, 2) conv_enc0_kernel(ConvH p) {
    if (p.done && *p.done) return;
    constexpr int RW = conv_h_rows(1), TH = 8 * RW;
    constexpr int XW = CM_TX + 4, XH = TH + 4;  // x: tile + halo 2
    constexpr int AW = CM_TX + 2, AH = TH + 2;  // a: tile + halo 1
    constexpr int NA = AW * AH, MB = (NA + 15) / 16;
    extern __shared__ __align__(16) unsigned short cm_smem[];
    unsigned short* x_s = cm_smem;                  // [XH][XW][8], channels 2-7 zero
    unsigned short* a_s = x_s + XH * XW * 8;        // [AH][AW][8]
    unsigned short* w1_s = a_s + AH * AW * 8;       // [8][P8_KP + 8]
    unsigned short* w2_s = w1_s + 8 * (P8_KP + 8);  // [8][P8_KP + 8]
    unsigned short* g_s = w2_s + 8 * (P8_KP + 8);   // [TH CM_TX][8]
    const int n = blockIdx.z;
    const int x0 = blockIdx.x * CM_TX, y0 = blockIdx.y * TH;
    stage_weights<1, P8_KP>(w1_s, p.wre);
    stage_weights<1, P8_KP>(w2_s, p.wre2);
    for (int q = threadIdx.x; q < TH * CM_TX; q += CM_NT) {
        const int y = y0 + q / CM_TX, x = x0 + q % CM_TX;
        const bool in = y < p.H && x < p.W;
        cp_async16(g_s + q * 8, in ? p.gate + ((n * p.H + y) * p.W + x) * 8 : p.gate, in ? 16 : 0);
    }
    const unsigned* xa = reinterpret_cast<const unsigned*>(p.a);  // a pixel's two BF16 channels
    for (int q = threadIdx.x; q < XH * XW; q += CM_NT) {
        const int yy = y0 + q / XW - 2, xx = x0 + q % XW - 2;
        const bool in = (unsigned)yy < (unsigned)p.H && (unsigned)xx < (unsigned)p.W;
        *reinterpret_cast<uint4*>(x_s + q * 8) = make_uint4(in ? __ldg(xa + (n * p.H + yy) * p.W + xx) : 0u, 0u, 0u, 0u);
    }
    cp_async_wait_all();
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, grp = lane >> 2, tig = lane & 3;
    const int lpix = (lane & 7) + ((lane >> 3) & 1) * 8, second = lane >> 4;  // ldmatrix row: pixel, which tap
    {  // the first layer over the a box, 16 box pixels (row-major, across box rows) an MMA row block
        unsigned b1[5][1][2];
#pragma unroll
        for (int j = 0; j < 5; j++) load_b<1, P8_KP>(b1[j], w1_s, j * 16, lane);
        for (int mb = warp; mb < MB; mb += CM_NT / 32) {
            const int m = min(mb * 16 + lpix, NA - 1);  // rows past the box repeat its last pixel
            const int py = m / AW, px = m - py * AW;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int j = 0; j < 5; j++) {
                const int tap = min(2 * j + second, 8);
                const int dy = tap / 3, dx = tap - 3 * (tap / 3);
                unsigned fa[4];
                ldmatrix_x4(fa, x_s + ((py + dy) * XW + px + dx) * 8);
                mma_bf16_16816(acc, fa, b1[j][0]);
            }
#pragma unroll
            for (int half = 0; half < 2; half++) {
                const int mo = mb * 16 + grp + 8 * half;
                if (mo >= NA) continue;
                const int oy = y0 - 1 + mo / AW, ox = x0 - 1 + mo % AW;
                const bool in = (unsigned)oy < (unsigned)p.H && (unsigned)ox < (unsigned)p.W;
                // + 0: the epilogue's bias-free sum (a -0 sum stored as +0, as the two launches do)
                reinterpret_cast<unsigned*>(a_s + mo * 8)[tig] =
                    in ? bf16_pack(acc[2 * half] + 0.f, acc[2 * half + 1] + 0.f) : 0u;
            }
        }
    }
    __syncthreads();
    float acc[RW][1][4];
#pragma unroll
    for (int r = 0; r < RW; r++)
#pragma unroll
        for (int e = 0; e < 4; e++) acc[r][0][e] = 0.f;
#pragma unroll
    for (int j = 0; j < 5; j++) {
        const int tap = min(2 * j + second, 8);
        const int dy = tap / 3, dx = tap - 3 * (tap / 3);
        unsigned b[1][2];
        load_b<1, P8_KP>(b, w2_s, j * 16, lane);
#pragma unroll
        for (int r = 0; r < RW; r++) {
            unsigned fa[4];
            ldmatrix_x4(fa, a_s + ((warp * RW + r + dy) * AW + lpix + dx) * 8);
            mma_bf16_16816(acc[r][0], fa, b[0]);
        }
    }
    conv_h_epilogue<1, RW>(p, acc, g_s, n, x0, y0);
}

// conv_up_kernel for an 8-channel skip map b: the b-part takes two taps per K step as in
// conv_p8_kernel (its box unpadded, 16 bytes a pixel), after the coarse a-part. Weights in the
// order [co][9 CPA + P8_KP]: the a-part by tap and channel, then the b-part's tap pairs.
__global__ void conv_up8_weights_kernel(const float* __restrict__ w, int co_n, int cpa, int ntl,
                                        unsigned short* __restrict__ out) {
    const int kp = 9 * cpa + P8_KP, ci = cpa + 8;
    const int total = ntl * 8 * kp;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
        const int co = q / kp, k = q % kp;
        int tap, c;
        if (k < 9 * cpa) {
            tap = k / cpa;
            c = k % cpa;
        } else {
            tap = (k - 9 * cpa) / 8;
            c = cpa + (k - 9 * cpa) % 8;
        }
        out[q] = (co < co_n && tap < 9) ? (unsigned short)(__float_as_uint(w[((size_t)co * ci + c) * 9 + tap]) >> 16)
                                        : (unsigned short)0;
    }
}

__host__ __device__ inline size_t conv_up8_smem(int cpa, int co, bool gated) {
    const int ntl = (co + 7) / 8, th = 8 * conv_up_rows(ntl);
    const size_t abox = (size_t)(th / 2 + 2) * (CM_TX / 2 + 2) * (cpa + 8);
    const size_t bbox = (size_t)(th + 2) * (CM_TX + 2) * 8;
    return (abox + bbox + (size_t)ntl * 8 * (9 * cpa + P8_KP + 8) + (gated ? (size_t)th * CM_TX * ntl * 8 : 0)) * 2;
}

template <int NTL, int CPA>
__global__ void __launch_bounds__(CM_NT, 2) conv_up8_kernel(ConvH p) {
    if (p.done && *p.done) return;
    constexpr int RW = conv_up_rows(NTL), TH = 8 * RW;
    constexpr int EW = CM_TX + 2, EH = TH + 2, CEW = CM_TX / 2 + 2, CEH = TH / 2 + 2;
    constexpr int PSA = CPA + 8, KP = 9 * CPA + P8_KP, GA = CPA / 8, UA = CEH * CEW * GA, UB = EH * EW;
    extern __shared__ __align__(16) unsigned short cm_smem[];
    unsigned short* a_s = cm_smem;                // [CEH][CEW][PSA]
    unsigned short* b_s = a_s + CEH * CEW * PSA;   // [EH][EW][8]
    unsigned short* w_s = b_s + EH * EW * 8;       // [8 NTL][KP]
    unsigned short* g_s = w_s + 8 * NTL * (KP + 8);      // gated layers: [TH][16][co]
    const int n = blockIdx.z;
    const int x0 = blockIdx.x * CM_TX, y0 = blockIdx.y * TH;
    const int Hc = p.H / 2, Wc = p.W / 2;
    const int cx0 = (x0 >> 1) - 1, cy0 = (y0 >> 1) - 1;
    stage_weights<NTL, KP>(w_s, p.wre);
    if (p.gate) {
        const int gg = p.co / 8;
        for (int q = threadIdx.x; q < TH * CM_TX * gg; q += CM_NT) {
            const int pix = q / gg, c0 = (q - pix * gg) * 8;
            const int y = y0 + pix / CM_TX, x = x0 + pix % CM_TX;
            const bool in = y < p.H && x < p.W;
            cp_async16(g_s + pix * p.co + c0, in ? p.gate + ((n * p.H + y) * p.W + x) * p.co + c0 : p.gate, in ? 16 : 0);
        }
    }
    for (int q = threadIdx.x; q < UA; q += CM_NT) {  // the coarse box of a
        const int r = q / GA, c0 = (q % GA) * 8;
        const int cy = cy0 + r / CEW, cx = cx0 + r % CEW;
        const bool in = (unsigned)cy < (unsigned)Hc && (unsigned)cx < (unsigned)Wc;
        cp_async16(a_s + r * PSA + c0, in ? p.a + ((n * Hc + cy) * Wc + cx) * p.ca + c0 : p.a, in ? 16 : 0);
    }
    for (int q = threadIdx.x; q < UB; q += CM_NT) {  // the fine box of b, 8 channels
        const int yy = y0 + q / EW - 1, xx = x0 + q % EW - 1;
        const bool in = (unsigned)yy < (unsigned)p.H && (unsigned)xx < (unsigned)p.W;
        cp_async16(b_s + q * 8, in ? p.b + ((n * p.H + yy) * p.W + xx) * 8 : p.b, in ? 16 : 0);
    }
    cp_async_wait_all();
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int lpix = (lane & 7) + ((lane >> 3) & 1) * 8, lk = (lane >> 4) * 8, second = lane >> 4;
    float acc[RW][NTL][4];
#pragma unroll
    for (int r = 0; r < RW; r++)
#pragma unroll
        for (int t = 0; t < NTL; t++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[r][t][e] = 0.f;
    auto step = [&](int kb, auto addr) {
        unsigned b[NTL][2];
        load_b<NTL, KP>(b, w_s, kb, lane);
#pragma unroll
        for (int r = 0; r < RW; r++) {
            unsigned a[4];
            ldmatrix_x4(a, addr(r));
#pragma unroll
            for (int t = 0; t < NTL; t++) mma_bf16_16816(acc[r][t], a, b[t]);
        }
    };
#pragma unroll 3
    for (int tap = 0; tap < 9; tap++) {  // a: the upsampled coarse map
        const int dy = tap / 3, dx = tap % 3;
        const int ccol = (lpix + dx + 1) >> 1;
#pragma unroll
        for (int cb = 0; cb < CPA; cb += 16)
            step(tap * CPA + cb, [&](int r) { return a_s + (((warp * RW + r + dy + 1) >> 1) * CEW + ccol) * PSA + cb + lk; });
    }
#pragma unroll
    for (int j = 0; j < 5; j++) {  // b: two taps per K step
        const int tap = min(2 * j + second, 8);
        const int dy = tap / 3, dx = tap - 3 * (tap / 3);
        step(9 * CPA + j * 16, [&](int r) { return b_s + ((warp * RW + r + dy) * EW + lpix + dx) * 8; });
    }
    conv_h_epilogue<NTL, RW>(p, acc, g_s, n, x0, y0);
}

// The network's last two layers at the first level in one launch: DA = conv3x3(concat(up(a), b))
// (a: CPA channels at the coarse level, b: the 8-channel skip; no bias, no activation) and
// y = out(conv3x3(DA) * gate), the 1x1 output layer in the epilogue. A block stages the coarse box
// of a (as conv_up8_kernel does: the tile plus a halo of 2 at the fine level needs the same
// TH/2 + 2 coarse rows), the skip box with a halo of 2, computes DA over the tile plus a halo of 1
// into shared memory (rounded to BF16, zero outside the map, what the two launches store and
// re-read) and the second layer from there. Same K order as conv_up8_kernel and conv_p8_kernel:
// bit-identical to the two launches, and DA never reaches HBM.
template <int CPA>
__host__ __device__ inline size_t conv_dec0_smem() {
    constexpr int th = 8 * conv_h_rows(1);
    return ((size_t)(th / 2 + 2) * (CM_TX / 2 + 2) * (CPA + 8) + (size_t)(th + 4) * (CM_TX + 4) * 8 +
            (size_t)(th + 2) * (CM_TX + 2) * 8 + (size_t)8 * (9 * CPA + P8_KP + 8) + (size_t)8 * (P8_KP + 8) +
            (size_t)th * CM_TX * 8) * 2;
}

template <int CPA>
__global__ void __launch_bounds__(CM_NT, 2) conv_dec0_kernel(ConvH p) {
    if (p.done && *p.done) return;
    constexpr int RW = conv_h_rows(1), TH = 8 * RW;
    constexpr int CEW = CM_TX / 2 + 2, CEH = TH / 2 + 2, PSA = CPA + 8, GA = CPA / 8, UA = CEH * CEW * GA;
    constexpr int BW = CM_TX + 4, BH = TH + 4;  // skip: tile + halo 2
    constexpr int DW = CM_TX + 2, DH = TH + 2;  // DA: tile + halo 1
    constexpr int ND = DW * DH, MB = (ND + 15) / 16;
    constexpr int KP1 = 9 * CPA + P8_KP, KS1 = KP1 / 16;  // the first layer's K steps
    extern __shared__ __align__(16) unsigned short cm_smem[];
    unsigned short* a_s = cm_smem;                   // [CEH][CEW][PSA]
    unsigned short* b_s = a_s + CEH * CEW * PSA;     // [BH][BW][8]
    unsigned short* d_s = b_s + BH * BW * 8;         // [DH][DW][8]
    unsigned short* w1_s = d_s + DH * DW * 8;        // [8][KP1 + 8]
    unsigned short* w2_s = w1_s + 8 * (KP1 + 8);     // [8][P8_KP + 8]
    unsigned short* g_s = w2_s + 8 * (P8_KP + 8);    // [TH CM_TX][8]
    const int n = blockIdx.z;
    const int x0 = blockIdx.x * CM_TX, y0 = blockIdx.y * TH;
    const int Hc = p.H / 2, Wc = p.W / 2;
    const int cx0 = (x0 >> 1) - 1, cy0 = (y0 >> 1) - 1;
    stage_weights<1, KP1>(w1_s, p.wre);
    stage_weights<1, P8_KP>(w2_s, p.wre2);
    for (int q = threadIdx.x; q < TH * CM_TX; q += CM_NT) {
        const int y = y0 + q / CM_TX, x = x0 + q % CM_TX;
        const bool in = y < p.H && x < p.W;
        cp_async16(g_s + q * 8, in ? p.gate + ((n * p.H + y) * p.W + x) * 8 : p.gate, in ? 16 : 0);
    }
    for (int q = threadIdx.x; q < UA; q += CM_NT) {  // the coarse box of a
        const int r = q / GA, c0 = (q % GA) * 8;
        const int cy = cy0 + r / CEW, cx = cx0 + r % CEW;
        const bool in = (unsigned)cy < (unsigned)Hc && (unsigned)cx < (unsigned)Wc;
        cp_async16(a_s + r * PSA + c0, in ? p.a + ((n * Hc + cy) * Wc + cx) * CPA + c0 : p.a, in ? 16 : 0);
    }
    for (int q = threadIdx.x; q < BH * BW; q += CM_NT) {  // the skip box
        const int yy = y0 + q / BW - 2, xx = x0 + q % BW - 2;
        const bool in = (unsigned)yy < (unsigned)p.H && (unsigned)xx < (unsigned)p.W;
        cp_async16(b_s + q * 8, in ? p.b + ((n * p.H + yy) * p.W + xx) * 8 : p.b, in ? 16 : 0);
    }
    cp_async_wait_all();
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, grp = lane >> 2, tig = lane & 3;
    const int lpix = (lane & 7) + ((lane >> 3) & 1) * 8, lk = (lane >> 4) * 8, second = lane >> 4;
    {  // the first layer over the DA box, 16 box pixels (row-major, across box rows) an MMA row block
        unsigned b1[KS1][1][2];
#pragma unroll
        for (int k = 0; k < KS1; k++) load_b<1, KP1>(b1[k], w1_s, k * 16, lane);
        for (int mb = warp; mb < MB; mb += CM_NT / 32) {
            const int m = min(mb * 16 + lpix, ND - 1);  // rows past the box repeat its last pixel
            const int py = m / DW, px = m - py * DW;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int tap = 0; tap < 9; tap++) {  // up(a): the fine pixel (py + dy, px + dx) - 2 repeats
                const int dy = tap / 3, dx = tap % 3;  // coarse box pixel ((py + dy) / 2, (px + dx) / 2)
#pragma unroll
                for (int cb = 0; cb < CPA; cb += 16) {
                    unsigned fa[4];
                    ldmatrix_x4(fa, a_s + (((py + dy) >> 1) * CEW + ((px + dx) >> 1)) * PSA + cb + lk);
                    mma_bf16_16816(acc, fa, b1[(tap * CPA + cb) / 16][0]);
                }
            }
#pragma unroll
            for (int j = 0; j < 5; j++) {  // b: two taps per K step
                const int tap = min(2 * j + second, 8);
                const int dy = tap / 3, dx = tap - 3 * (tap / 3);
                unsigned fa[4];
                ldmatrix_x4(fa, b_s + ((py + dy) * BW + px + dx) * 8);
                mma_bf16_16816(acc, fa, b1[9 * CPA / 16 + j][0]);
            }
#pragma unroll
            for (int half = 0; half < 2; half++) {
                const int mo = mb * 16 + grp + 8 * half;
                if (mo >= ND) continue;
                const int oy = y0 - 1 + mo / DW, ox = x0 - 1 + mo % DW;
                const bool in = (unsigned)oy < (unsigned)p.H && (unsigned)ox < (unsigned)p.W;
                // + 0: the epilogue's bias-free sum (a -0 sum stored as +0, as the two launches do)
                reinterpret_cast<unsigned*>(d_s + mo * 8)[tig] =
                    in ? bf16_pack(acc[2 * half] + 0.f, acc[2 * half + 1] + 0.f) : 0u;
            }
        }
    }
    __syncthreads();
    float acc[RW][1][4];
#pragma unroll
    for (int r = 0; r < RW; r++)
#pragma unroll
        for (int e = 0; e < 4; e++) acc[r][0][e] = 0.f;
#pragma unroll
    for (int j = 0; j < 5; j++) {
        const int tap = min(2 * j + second, 8);
        const int dy = tap / 3, dx = tap - 3 * (tap / 3);
        unsigned b[1][2];
        load_b<1, P8_KP>(b, w2_s, j * 16, lane);
#pragma unroll
        for (int r = 0; r < RW; r++) {
            unsigned fa[4];
            ldmatrix_x4(fa, d_s + ((warp * RW + r + dy) * DW + lpix + dx) * 8);
            mma_bf16_16816(acc[r][0], fa, b[0]);
        }
    }
    conv_h_epilogue<1, RW>(p, acc, g_s, n, x0, y0);
}

// NCHW FP32 maps -> NHWC BF16 (c channels, 2 or a multiple of 2).
__global__ void to_h_kernel(const float* __restrict__ x, int N, int C, int H, int W, unsigned short* __restrict__ y) {
    const size_t plane = (size_t)H * W, total = (size_t)N * plane * (C / 2);
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const size_t pix = q / (C / 2);
        const int c = 2 * (int)(q % (C / 2));
        const size_t n = pix / plane, r = pix % plane;
        const float* s = x + (n * C + c) * plane + r;
        reinterpret_cast<unsigned*>(y)[q] = bf16_pack(s[0], s[plane]);
    }
}

// NHWC FP32 two-channel output -> NCHW planes.
__global__ void from_h_kernel(const float* __restrict__ y, int N, int H, int W, float* __restrict__ out) {
    const size_t plane = (size_t)H * W, total = (size_t)N * plane;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const size_t n = q / plane, r = q % plane;
        const float2 v = reinterpret_cast<const float2*>(y)[q];
        out[n * 2 * plane + r] = v.x;
        out[(n * 2 + 1) * plane + r] = v.y;
    }
}

// The features of level l (the 2^l x 2^l block means of the level-0 NCHW FP32 features), NHWC BF16.
__global__ void features_h_kernel(const float* __restrict__ f0, int N, int H0, int W0, int l,
                                  unsigned short* __restrict__ fl) {
    const int S = 1 << l, H = H0 >> l, W = W0 >> l;
    const size_t plane0 = (size_t)H0 * W0, total = (size_t)N * H * W;
    const float inv = 1.f / (float)(S * S);
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const size_t n = q / ((size_t)H * W);
        const int r = (int)(q % ((size_t)H * W)), yy = r / W, xx = r % W;
        float a = 0.f, b = 0.f;
        for (int u = 0; u < S; u++)
            for (int v = 0; v < S; v++) {
                const size_t k = (size_t)(yy * S + u) * W0 + (xx * S + v);
                a += f0[n * 2 * plane0 + k];
                b += f0[(n * 2 + 1) * plane0 + k];
            }
        reinterpret_cast<unsigned*>(fl)[q] = bf16_pack(a * inv, b * inv);
    }
}

// dw[co][ci][t] = sum over samples and pixels of dy[co] * x[ci] shifted by tap t; one block per
// (co, ci) pair. x is the concatenation of xa (ca channels) and xb, both at H x W.
template <int K>
__global__ void __launch_bounds__(256) conv_wgrad_kernel(const float* __restrict__ dy, const float* __restrict__ xa,
                                                         int ca, const float* __restrict__ xb, int cb, int co_n,
                                                         int H, int W, int N, float* __restrict__ dw) {
    constexpr int R = K / 2;
    const int ci_total = ca + cb;
    const int co = blockIdx.x / ci_total, ci = blockIdx.x % ci_total;
    float acc[K * K];
#pragma unroll
    for (int t = 0; t < K * K; t++) acc[t] = 0.f;
    const size_t plane = (size_t)H * W;
    for (size_t q = threadIdx.x; q < (size_t)N * plane; q += blockDim.x) {
        const int n = (int)(q / plane);
        const int r = (int)(q % plane);
        const int y = r / W, x = r % W;
        const float g = dy[((size_t)n * co_n + co) * plane + r];
        const float* src = ci < ca ? xa + ((size_t)n * ca + ci) * plane : xb + ((size_t)n * cb + (ci - ca)) * plane;
#pragma unroll
        for (int t = 0; t < K * K; t++) {
            const int yy = y + t / K - R, xx = x + t % K - R;
            if ((unsigned)yy < (unsigned)H && (unsigned)xx < (unsigned)W) acc[t] = fmaf(g, src[yy * W + xx], acc[t]);
        }
    }
    __shared__ float red[K * K][8];
#pragma unroll
    for (int t = 0; t < K * K; t++) {
        float v = acc[t];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[t][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < K * K) {
        float v = 0.f;
        for (int w8 = 0; w8 < (int)(blockDim.x / 32); w8++) v += red[threadIdx.x][w8];
        dw[((size_t)co * ci_total + ci) * K * K + threadIdx.x] += v;
    }
}

__global__ void bias_grad_kernel(const float* __restrict__ dy, int co_n, int H, int W, int N, float* __restrict__ db) {
    const int co = blockIdx.x;
    const size_t plane = (size_t)H * W;
    float s = 0.f;
    for (size_t q = threadIdx.x; q < (size_t)N * plane; q += blockDim.x) {
        const int n = (int)(q / plane);
        s += dy[((size_t)n * co_n + co) * plane + q % plane];
    }
    __shared__ float red[8];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float v = 0.f;
        for (int w8 = 0; w8 < (int)(blockDim.x / 32); w8++) v += red[w8];
        db[co] += v;
    }
}

// wt[ci][co][K-1-ty][K-1-tx] = w[co][ci][ty][tx]: the input gradient of a convolution is the
// convolution of the output gradient with these weights.
__global__ void transpose_weights_kernel(const float* __restrict__ w, int co_n, int ci_n, int K, float* __restrict__ wt) {
    const int total = co_n * ci_n * K * K;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
        const int t = q % (K * K), r = q / (K * K);
        const int ci = r % ci_n, co = r / ci_n;
        const int ty = t / K, tx = t % K;
        wt[((size_t)ci * co_n + co) * K * K + (K - 1 - ty) * K + (K - 1 - tx)] = w[q];
    }
}

// 2x2 mean pooling and nearest upsampling, their adjoints (pool_bwd = up / 4, up_bwd = sum).
__global__ void pool2_kernel(const float* __restrict__ x, int NC, int H, int W, float* __restrict__ y, float scale,
                             int add) {
    // y at H/2 x W/2: scale * sum of the 2x2 block (scale 0.25: mean pooling; 1: the adjoint of up)
    const int Hh = H / 2, Wh = W / 2;
    const size_t total = (size_t)NC * Hh * Wh;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int xx = (int)(q % Wh), yy = (int)((q / Wh) % Hh);
        const size_t c = q / ((size_t)Hh * Wh);
        const float* s = x + (c * H + 2 * yy) * W + 2 * xx;
        const float v = scale * ((s[0] + s[1]) + (s[W] + s[W + 1]));
        y[q] = add ? y[q] + v : v;
    }
}

__global__ void up2_kernel(const float* __restrict__ x, int NC, int Hh, int Wh, float* __restrict__ y, float scale,
                           int add) {
    // y at 2Hh x 2Wh: scale * nearest value (scale 1: upsampling; 0.25: the adjoint of pooling)
    const int H = 2 * Hh, W = 2 * Wh;
    const size_t total = (size_t)NC * H * W;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int xx = (int)(q % W), yy = (int)((q / W) % H);
        const size_t c = q / ((size_t)H * W);
        const float v = scale * x[(c * Hh + yy / 2) * Wh + xx / 2];
        y[q] = add ? y[q] + v : v;
    }
}

// Gate backward: u * g -> du = dy g, dg = dy u (dg accumulated); then through g = 2 sigmoid(z):
// dz = dg * g (1 - g / 2).
__global__ void gate_bwd_kernel(const float* __restrict__ dy, const float* __restrict__ u, const float* __restrict__ g,
                                float* __restrict__ du, float* __restrict__ dg, size_t n) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        du[q] = dy[q] * g[q];
        dg[q] += dy[q] * u[q];
    }
}

__global__ void sig2_relu_bwd_kernel(float* __restrict__ d, const float* __restrict__ y, size_t n, int act) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        if (act == ACT_SIG2) d[q] *= y[q] * (1.f - 0.5f * y[q]);
        else d[q] = y[q] > 0.f ? d[q] : 0.f;
    }
}

// The network can run on a grid S times coarser than the solver's: its input is the S x S block
// mean, its output is read back at the block's every cell (nearest). Their adjoints: the block
// sum times `scale` (1: the adjoint of nearest upsampling), nearest upsampling times `scale`.
__global__ void pool_s_kernel(const float* __restrict__ x, int NC, int H, int W, int S, float* __restrict__ y,
                              float scale) {
    const int Hc = H / S, Wc = W / S;
    const size_t total = (size_t)NC * Hc * Wc;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int xx = (int)(q % Wc), yy = (int)((q / Wc) % Hc);
        const size_t c = q / ((size_t)Hc * Wc);
        const float* s = x + (c * H + (size_t)yy * S) * W + (size_t)xx * S;
        float v = 0.f;
        for (int a = 0; a < S; a++)
            for (int b = 0; b < S; b++) v += s[(size_t)a * W + b];
        y[q] = scale * v;
    }
}

__global__ void up_s_kernel(const float* __restrict__ x, int NC, int Hc, int Wc, int S, float* __restrict__ y) {
    const int H = Hc * S, W = Wc * S;
    const size_t total = (size_t)NC * H * W;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int xx = (int)(q % W), yy = (int)((q / W) % H);
        const size_t c = q / ((size_t)H * W);
        y[q] = x[(c * Hc + yy / S) * Wc + xx / S];
    }
}

// ---- the SGN operator on training patches (zero outside the patch) ------------------------

struct PatchOp {
    const float* c;     // [n][H][W]
    const float* heff;  // [n][H][W]
    const float* mask;  // [n][H][W]
    int H, W, N;
    float ix, iy, dx2i, dy2i;  // 0.5/dx, 0.5/dy, 0.25/dx^2, 0.25/dy^2
};

// out = A p on every patch cell (dispersion.rs:269-317 with zero values outside the patch).
__global__ void patch_matvec_kernel(PatchOp op, const float* __restrict__ p, float* __restrict__ out) {
    const size_t plane = (size_t)op.H * op.W;
    const size_t total = (size_t)op.N * plane;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int n = (int)(q / plane);
        const int r = (int)(q % plane);
        const int y = r / op.W, x = r % op.W;
        const float* px = p + (size_t)n * 2 * plane;
        const float* py = px + plane;
        const float* c = op.c + (size_t)n * plane;
        auto P = [&](const float* a, int yy, int xx) {
            return ((unsigned)yy < (unsigned)op.H && (unsigned)xx < (unsigned)op.W) ? a[yy * op.W + xx] : 0.f;
        };
        auto f = [&](int yy, int xx) {
            if ((unsigned)yy >= (unsigned)op.H || (unsigned)xx >= (unsigned)op.W) return 0.f;
            return c[yy * op.W + xx] * ((P(px, yy, xx + 1) - P(px, yy, xx - 1)) * op.ix + (P(py, yy + 1, xx) - P(py, yy - 1, xx)) * op.iy);
        };
        const float m = op.mask[q], he = op.heff[q];
        out[(size_t)n * 2 * plane + r] = m * (he * px[r] - (f(y, x + 1) - f(y, x - 1)) * op.ix);
        out[(size_t)n * 2 * plane + plane + r] = m * (he * py[r] - (f(y + 1, x) - f(y - 1, x)) * op.iy);
    }
}

// The Jacobi diagonal on patches (dispersion.rs:441-457), two planes per sample.
__global__ void patch_diag_kernel(PatchOp op, float* __restrict__ d) {
    const size_t plane = (size_t)op.H * op.W;
    const size_t total = (size_t)op.N * plane;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int n = (int)(q / plane);
        const int r = (int)(q % plane);
        const int y = r / op.W, x = r % op.W;
        const float* c = op.c + (size_t)n * plane;
        auto C = [&](int yy, int xx) {
            return ((unsigned)yy < (unsigned)op.H && (unsigned)xx < (unsigned)op.W) ? c[yy * op.W + xx] : 0.f;
        };
        float dxv = 1.f, dyv = 1.f;
        if (op.mask[q] != 0.f) {
            dxv = op.heff[q] + (C(y, x + 1) + C(y, x - 1)) * op.dx2i;
            dyv = op.heff[q] + (C(y + 1, x) + C(y - 1, x)) * op.dy2i;
        }
        d[(size_t)n * 2 * plane + r] = dxv;
        d[(size_t)n * 2 * plane + plane + r] = dyv;
    }
}

// Generic elementwise update on 2-plane fields: out = a * x + b * y * (mask?) / d^e ...
// kept explicit: each use below names what it computes.
__global__ void lincomb_kernel(float* __restrict__ out, const float* __restrict__ x, float ax,
                               const float* __restrict__ y, float ay, const float* __restrict__ div_by,
                               const float* __restrict__ mask, int mask_planes, size_t n, size_t plane) {
    // out = ax * x + ay * y [/ div_by] [* mask (broadcast over 2 planes)]
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        float v = ay * (y ? y[q] : 0.f);
        if (div_by) v /= div_by[q];
        if (mask) v *= mask[(q / (mask_planes * plane)) * plane + q % plane];
        out[q] = (x ? ax * x[q] : 0.f) + v;
    }
}

// Per-sample dots <a, b> over 2-plane fields, accumulated in FP64.
__global__ void sample_dot_kernel(const float* __restrict__ a, const float* __restrict__ b, size_t per_sample,
                                  double* __restrict__ out) {
    const int n = blockIdx.y;
    double s = 0.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < per_sample; q += (size_t)gridDim.x * blockDim.x)
        s += (double)a[n * per_sample + q] * b[n * per_sample + q];
    __shared__ double red[8];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w8 = 0; w8 < (int)(blockDim.x / 32); w8++) v += red[w8];
        atomicAdd(out + n, v);
    }
}

// grad = -2 / (N E_n) * Ad  (the gradient of mean_n <d, A d>_n / E_n with respect to z, d = e - z;
// a patch without a wet cell has E_n = 0 and contributes nothing)
__global__ void loss_grad_kernel(const float* __restrict__ ad, const double* __restrict__ energy, int N,
                                 size_t per_sample, float* __restrict__ g) {
    const size_t total = (size_t)N * per_sample;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int n = (int)(q / per_sample);
        g[q] = energy[n] > 0.0 ? (float)(-2.0 / ((double)N * energy[n])) * ad[q] : 0.f;
    }
}

// Random error fields for training: white noise of a per-sample weight plus value noise at
// scales 1..32 cells (bilinear between hashed lattice values), masked.
__device__ __forceinline__ float hash_unit(unsigned long long k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (float)(k >> 40) * (1.0f / 16777216.0f) * 2.f - 1.f;
}

__global__ void random_field_kernel(float* __restrict__ e, const float* __restrict__ mask, int N, int H, int W,
                                    unsigned long long seed, float rough) {
    const size_t plane = (size_t)H * W;
    const size_t total = (size_t)N * 2 * plane;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int n = (int)(q / (2 * plane));
        const int comp = (int)((q / plane) % 2);
        const int r = (int)(q % plane);
        const int y = r / W, x = r % W;
        const unsigned long long base = seed * 1000003ull + (unsigned long long)(n * 2 + comp) * 7919ull;
        const float wr = rough * 0.5f * (hash_unit(base ^ 0x51ull) + 1.f);
        float v = wr * 1.7320508f * hash_unit(base * 31ull + (unsigned long long)r * 2654435761ull + 17ull);
        for (int sc = 1, li = 0; sc <= 32; sc *= 2, li++) {
            const float fy = (float)y / sc, fx = (float)x / sc;
            const int iy = (int)floorf(fy), ixx = (int)floorf(fx);
            const float ty = fy - iy, tx = fx - ixx;
            auto L = [&](int a, int b) {
                return hash_unit(base * 131ull + (unsigned long long)li * 1000003ull + (unsigned long long)(a + 64) * 92821ull +
                                 (unsigned long long)(b + 64) * 68917ull);
            };
            const float lv = (1 - ty) * ((1 - tx) * L(iy, ixx) + tx * L(iy, ixx + 1)) + ty * ((1 - tx) * L(iy + 1, ixx) + tx * L(iy + 1, ixx + 1));
            v += sqrtf((float)sc) * 1.7320508f * lv;
        }
        e[q] = v * mask[(size_t)n * plane + r];
    }
}

// Nearest bfloat16 (ties to even) as a float: keep the top 16 bits after adding half an ulp of
// the kept part (plus one if the kept part is odd). Finite inputs only (weights are finite).
__device__ __forceinline__ float bf16_round(float x) {
    const unsigned a = __float_as_uint(x);
    return __uint_as_float((a + 0x7FFFu + ((a >> 16) & 1u)) & 0xFFFF0000u);
}

__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ wq, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float c1, float c2, float eps,
                            int round_bf16) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const float gg = g[q];
        m[q] = b1 * m[q] + (1.f - b1) * gg;
        v[q] = b2 * v[q] + (1.f - b2) * gg * gg;
        w[q] -= lr * (m[q] * c1) / (sqrtf(v[q] * c2) + eps);
        wq[q] = round_bf16 ? bf16_round(w[q]) : w[q];
    }
}

__global__ void round_copy_kernel(const float* __restrict__ w, float* __restrict__ wq, int n, int round_bf16) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        wq[q] = round_bf16 ? bf16_round(w[q]) : w[q];
}

}  // namespace wcb

namespace wcb {

// ---- flexible CG with the learned preconditioner, on the solver's arrays ------------------
//
// Vectors are float2 (x, y components) over the interior with the solver's pitch; halo reads go
// through the boundary mapping (vector ghosts: the wall-normal component flips sign), as in the
// Jacobi solve. Scalars live on the device so that iterations chain without the host.


// A v (dispersion.rs:269-317) one cell per thread, halo through the mapping.
__global__ void fcg_matvec_kernel(DevGrid g, const float2* __restrict__ v, const float* __restrict__ cc,
                                  const float* __restrict__ heff, float2* __restrict__ out,
                                  const FcgScalars* __restrict__ sc) {
    if (sc && sc->done) return;
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % g.nx, j = c / g.nx;
        auto V = [&](int a, int b) {
            const Mapped m = map_cell(g, a, b);
            const float2 t = v[m.k];
            return make_float2(t.x * m.sx, t.y * m.sy);
        };
        auto F = [&](int a, int b) {
            const Mapped m = map_cell(g, a, b);
            return cc[m.k] * ((V(a + 1, b).x - V(a - 1, b).x) * g.ix + (V(a, b + 1).y - V(a, b - 1).y) * g.iy);
        };
        const int k = j * g.pitch + i;
        const float he = heff[k];
        const float mask = he >= H_DISP_MIN ? 1.f : 0.f;
        const float2 own = v[k];
        float2 r;
        r.x = mask * (he * own.x - (F(i + 1, j) - F(i - 1, j)) * g.ix);
        r.y = mask * (he * own.y - (F(i, j + 1) - F(i, j - 1)) * g.iy);
        out[k] = r;
    }
}

// The inverse of the Jacobi diagonal (dispersion.rs:441-457) and the warm start masked (:480-490).
__global__ void fcg_setup_kernel(DevGrid g, const float* __restrict__ cc, const float* __restrict__ heff,
                                 float2* __restrict__ diag, float2* __restrict__ w) {
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % g.nx, j = c / g.nx;
        const int k = j * g.pitch + i;
        const float he = heff[k];
        float2 d = make_float2(1.f, 1.f);
        if (he >= H_DISP_MIN) {
            auto C = [&](int a, int b) { return cc[map_cell(g, a, b).k]; };
            d.x = 1.f / (he + (C(i + 1, j) + C(i - 1, j)) * 0.25f / (g.dx * g.dx));
            d.y = 1.f / (he + (C(i, j + 1) + C(i, j - 1)) * 0.25f / (g.dy * g.dy));
        } else {
            w[k] = make_float2(0.f, 0.f);
        }
        diag[k] = d;  // inverted: the passes multiply
    }
}

// Up to three dot products of float2 fields, per-block FP64 partials (fixed partition), then
// one block adds them in block order: reproducible.
__global__ void fcg_dot_partial_kernel(DevGrid g, const float2* a0, const float2* b0, const float2* a1,
                                       const float2* b1, const float2* a2, const float2* b2, double* part,
                                       const FcgScalars* __restrict__ sc) {
    if (sc && sc->done) return;
    double s[3] = {0.0, 0.0, 0.0};
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int k = (c / g.nx) * g.pitch + c % g.nx;
        const float2 x0 = a0[k], y0 = b0[k];
        s[0] += (double)x0.x * y0.x + (double)x0.y * y0.y;
        if (a1) {
            const float2 x1 = a1[k], y1 = b1[k];
            s[1] += (double)x1.x * y1.x + (double)x1.y * y1.y;
        }
        if (a2) {
            const float2 x2 = a2[k], y2 = b2[k];
            s[2] += (double)x2.x * y2.x + (double)x2.y * y2.y;
        }
    }
    __shared__ double red[100];
    block_sum3<256>(s[0], s[1], s[2], red);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = s[0];
        part[3 * blockIdx.x + 1] = s[1];
        part[3 * blockIdx.x + 2] = s[2];
    }
}

enum FcgStep { FCG_INIT = 0, FCG_ALPHA = 1, FCG_RESID = 2, FCG_BETA = 3 };

// Totals of the partials and the scalar logic of one point of the iteration. With `cond` set the
// kernel also steers the graph's while-node: it continues while the solve is not done.
__global__ void fcg_scalars_kernel(const double* part, int nblocks, FcgScalars* sc, int step, double tol,
                                   long long max_it, cudaGraphConditionalHandle handle, int cond) {
    if (sc->done && step != FCG_INIT) {
        if (cond && threadIdx.x == 0) cudaGraphSetConditional(handle, 0u);
        return;
    }
    double s[3] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += 256)
        for (int q = 0; q < 3; q++) s[q] += part[3 * b + q];
    __shared__ double red[100];
    block_sum3<256>(s[0], s[1], s[2], red);
    if (threadIdx.x != 0) return;
    if (step == FCG_INIT) {  // <b, b>, <r, r>
        sc->bb = s[0];
        sc->rr = s[1];
        sc->target = tol * sqrt(s[0]) + 1e-10;
        sc->iterations = 0;
        sc->pq = 0.0;
        sc->converged = sqrt(s[1]) <= sc->target;
        sc->done = sc->converged || max_it <= 0;
    } else if (step == FCG_ALPHA) {  // <p, q>, <r, p>
        sc->pq = s[0];
        sc->rp = s[1];
        sc->alpha = s[1] / s[0];
        if (!(s[0] > 0.0)) {  // breakdown: the solve stops unconverged (Jacobi PCG takes over)
            sc->alpha = 0.0;
            sc->done = 1;
        }
    } else if (step == FCG_RESID) {  // <r, r>
        sc->rr = s[0];
        sc->iterations += 1;
        sc->converged = sqrt(s[0]) <= sc->target;
        sc->done = sc->converged || sc->iterations >= max_it;
    } else {  // <z, q>: the new direction is A-orthogonal to the previous one (none at first)
        sc->zq = s[0];
        sc->beta = sc->iterations == 0 ? 0.0 : -s[0] / sc->pq;
    }
    if (cond && (step == FCG_INIT || step == FCG_RESID)) cudaGraphSetConditional(handle, sc->done ? 0u : 1u);
}

// r = b - t (the initial residual)
__global__ void fcg_residual_kernel(DevGrid g, const float2* b, const float2* t, float2* r) {
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int k = (c / g.nx) * g.pitch + c % g.nx;
        const float2 bb = b[k], tt = t[k];
        r[k] = make_float2(bb.x - tt.x, bb.y - tt.y);
    }
}

// ---- the iteration as four passes -------------------------------------------------------
//
// One flexible-CG iteration touches every cell four times instead of once per vector operation:
//   pre   z1 = w r / D, and the network's input (r - A z1) / D        (A z1 from z1 of the stencil)
//   post  z = z2 + w (r - A z2) / D with z2 = z1 + m y, and <z, q>     (A z2 likewise)
//   dir   p = z + beta p, q = A p, <p, q>, <r, p>                       (p from the other bank)
//   upd   w += alpha p, r -= alpha q, <r, r>
// A vector at a stencil neighbour is recomputed from the inputs it is made of, so no pass waits
// for another's output of the same iteration. Dot partials use the fixed partition of
// fcg_dot_partial_kernel (grid-stride over cells, block_sum3), so runs are reproducible.

// A v at interior cell (i, j) (dispersion.rs:269-317), v given at any padded position by V(a, b)
// with its wall-normal components already sign-flipped.
template <typename VF>
__device__ __forceinline__ float2 apply_a(const DevGrid& g, int i, int j, const float* __restrict__ cc,
                                          const float* __restrict__ heff, VF V) {
    auto F = [&](int a, int b) {
        const Mapped m = map_cell(g, a, b);
        return cc[m.k] * ((V(a + 1, b).x - V(a - 1, b).x) * g.ix + (V(a, b + 1).y - V(a, b - 1).y) * g.iy);
    };
    const float he = heff[j * g.pitch + i];
    const float mask = he >= H_DISP_MIN ? 1.f : 0.f;
    const float2 own = V(i, j);
    return make_float2(mask * (he * own.x - (F(i + 1, j) - F(i - 1, j)) * g.ix),
                       mask * (he * own.y - (F(i, j + 1) - F(i, j - 1)) * g.iy));
}

// pre: per network pixel (S x S cells): z1 of its cells, and the block mean of (r - A z1) / D as
// the network input (NHWC BF16 pairs in xh, else 2 planes in x); zero outside the interior. d
// holds the inverse diagonal.
__global__ void fcg_pre_kernel(DevGrid g, const float2* __restrict__ r, const float2* __restrict__ d,
                               const float* __restrict__ cc, const float* __restrict__ heff, float2* __restrict__ z1,
                               float omega, float* __restrict__ x, unsigned* __restrict__ xh, int Hp, int Wp, int S,
                               const FcgScalars* __restrict__ sc) {
    if (sc->done) return;
    const size_t plane = (size_t)Hp * Wp;
    const float inv = 1.f / (float)(S * S);
    auto Z = [&](int a, int b) {  // d holds the inverse diagonal
        const Mapped m = map_cell(g, a, b);
        const float2 rr = r[m.k], dd = d[m.k];
        return make_float2(omega * rr.x * dd.x * m.sx, omega * rr.y * dd.y * m.sy);
    };
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < plane; q += (size_t)gridDim.x * blockDim.x) {
        const int i0 = (int)(q % Wp) * S, j0 = (int)(q / Wp) * S;
        float vx = 0.f, vy = 0.f;
        for (int a = 0; a < S; a++)
            for (int b = 0; b < S; b++) {
                const int i = i0 + b, j = j0 + a;
                if (i >= g.nx || j >= g.ny) continue;
                const int k = j * g.pitch + i;
                const float2 t = apply_a(g, i, j, cc, heff, Z);
                const float2 rr = r[k], dd = d[k];
                z1[k] = make_float2(omega * rr.x * dd.x, omega * rr.y * dd.y);
                vx += (rr.x - t.x) * dd.x;
                vy += (rr.y - t.y) * dd.y;
            }
        if (xh) {
            xh[q] = bf16_pack(vx * inv, vy * inv);
        } else {
            x[q] = vx * inv;
            x[plane + q] = vy * inv;
        }
    }
}

// The same passes on 32 x 8-cell tiles through shared memory: the derived vector is formed once
// per cell of the tile's box (halo 2, wall-normal signs applied), c once per cell of its halo-1
// box, and A v of every own cell read from there. A block walks tiles b, b + nb, ... (a fixed
// partition, so the dots stay reproducible).
constexpr int FT_X = 32, FT_Y = 8, FT_NT = FT_X * FT_Y;
constexpr int FB_W = FT_X + 4, FB_H = FT_Y + 4, FB_N = FB_W * FB_H;
constexpr int FC_W = FT_X + 2, FC_H = FT_Y + 2, FC_N = FC_W * FC_H;

struct FcgTile {
    float2 v[FB_N];
    float c[FC_N];
};

// box of VF(mapped cell) (the unsigned vector there) and of c; ends with a barrier
template <typename VF>
__device__ __forceinline__ void fcg_tile_stage(const DevGrid& g, int i0, int j0, const float* __restrict__ cc,
                                               FcgTile& sm, VF vf) {
    __syncthreads();  // the previous tile's box is read
    for (int q = threadIdx.x; q < FB_N; q += FT_NT) {
        const Mapped m = map_cell(g, i0 - 2 + q % FB_W, j0 - 2 + q / FB_W);
        const float2 v = vf(m);
        sm.v[q] = make_float2(v.x * m.sx, v.y * m.sy);
    }
    for (int q = threadIdx.x; q < FC_N; q += FT_NT) sm.c[q] = cc[map_cell(g, i0 - 1 + q % FC_W, j0 - 1 + q / FC_W).k];
    __syncthreads();
}

// A v at the own cell (tx, ty) of the staged tile (apply_a's arithmetic)
__device__ __forceinline__ float2 fcg_tile_apply(const DevGrid& g, const FcgTile& sm, int tx, int ty, float he) {
    auto V = [&](int a, int b) { return sm.v[(ty + 2 + b) * FB_W + tx + 2 + a]; };
    auto F = [&](int a, int b) {
        return sm.c[(ty + 1 + b) * FC_W + tx + 1 + a] *
               ((V(a + 1, b).x - V(a - 1, b).x) * g.ix + (V(a, b + 1).y - V(a, b - 1).y) * g.iy);
    };
    const float mask = he >= H_DISP_MIN ? 1.f : 0.f;
    const float2 own = V(0, 0);
    return make_float2(mask * (he * own.x - (F(1, 0) - F(-1, 0)) * g.ix), mask * (he * own.y - (F(0, 1) - F(0, -1)) * g.iy));
}

// pre on tiles, network on the solver's grid (stride 1): z1 and (r - A z1) / D as the input
__global__ void __launch_bounds__(FT_NT) fcg_pre_tile_kernel(DevGrid g, const float2* __restrict__ r,
                                                             const float2* __restrict__ d, const float* __restrict__ cc,
                                                             const float* __restrict__ heff, float2* __restrict__ z1,
                                                             float omega, float* __restrict__ x,
                                                             unsigned* __restrict__ xh, int Hp, int Wp,
                                                             const FcgScalars* __restrict__ sc) {
    if (sc->done) return;
    __shared__ FcgTile sm;
    const int tx = threadIdx.x % FT_X, ty = threadIdx.x / FT_X;
    const int ntx = (g.nx + FT_X - 1) / FT_X, ntiles = ntx * ((g.ny + FT_Y - 1) / FT_Y);
    const size_t plane = (size_t)Hp * Wp;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i0 = (t % ntx) * FT_X, j0 = (t / ntx) * FT_Y;
        fcg_tile_stage(g, i0, j0, cc, sm, [&](const Mapped& m) {
            const float2 rr = r[m.k], dd = d[m.k];
            return make_float2(omega * rr.x * dd.x, omega * rr.y * dd.y);
        });
        const int i = i0 + tx, j = j0 + ty;
        if (i >= g.nx || j >= g.ny) continue;
        const int k = j * g.pitch + i;
        const float2 tv = fcg_tile_apply(g, sm, tx, ty, heff[k]);
        const float2 rr = r[k], dd = d[k];
        z1[k] = make_float2(omega * rr.x * dd.x, omega * rr.y * dd.y);
        const float vx = (rr.x - tv.x) * dd.x, vy = (rr.y - tv.y) * dd.y;
        const size_t q = (size_t)j * Wp + i;
        if (xh) {
            xh[q] = bf16_pack(vx, vy);
        } else {
            x[q] = vx;
            x[plane + q] = vy;
        }
    }
}

// post on tiles: z = z2 + w (r - A z2) / D, z2 = z1 + m y; partial <z, q>
__global__ void __launch_bounds__(FT_NT) fcg_post_tile_kernel(DevGrid g, const float2* __restrict__ z1,
                                                              const float* __restrict__ y, int nhwc,
                                                              const float2* __restrict__ r, const float2* __restrict__ d,
                                                              const float* __restrict__ cc, const float* __restrict__ heff,
                                                              float2* __restrict__ z, const float2* __restrict__ qv,
                                                              float omega, int Hp, int Wp, int lgS,
                                                              double* __restrict__ part,
                                                              const FcgScalars* __restrict__ sc) {
    if (sc->done) return;
    __shared__ FcgTile sm;
    const int tx = threadIdx.x % FT_X, ty = threadIdx.x / FT_X;
    const int ntx = (g.nx + FT_X - 1) / FT_X, ntiles = ntx * ((g.ny + FT_Y - 1) / FT_Y);
    const size_t plane = (size_t)Hp * Wp;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i0 = (t % ntx) * FT_X, j0 = (t / ntx) * FT_Y;
        fcg_tile_stage(g, i0, j0, cc, sm, [&](const Mapped& m) {
            const int q = (m.j >> lgS) * Wp + (m.i >> lgS);
            const float2 yv = nhwc ? reinterpret_cast<const float2*>(y)[q] : make_float2(y[q], y[plane + q]);
            const float mk = heff[m.k] >= H_DISP_MIN ? 1.f : 0.f;
            const float2 a1 = z1[m.k];
            return make_float2(a1.x + mk * yv.x, a1.y + mk * yv.y);
        });
        const int i = i0 + tx, j = j0 + ty;
        if (i >= g.nx || j >= g.ny) continue;
        const int k = j * g.pitch + i;
        const float2 tv = fcg_tile_apply(g, sm, tx, ty, heff[k]);
        const float2 a2 = sm.v[(ty + 2) * FB_W + tx + 2], rr = r[k], dd = d[k];
        const float2 zz = make_float2(a2.x + omega * (rr.x - tv.x) * dd.x, a2.y + omega * (rr.y - tv.y) * dd.y);
        z[k] = zz;
        const float2 qq = qv[k];
        s0 += (double)zz.x * qq.x + (double)zz.y * qq.y;
    }
    __shared__ double red[100];
    block_sum3<FT_NT>(s0, s1, s2, red);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = s0;
        part[3 * blockIdx.x + 1] = 0.0;
        part[3 * blockIdx.x + 2] = 0.0;
    }
}

// dir on tiles: p = z + beta p_old (first: p = z), q = A p; partials <p, q>, <r, p>
__global__ void __launch_bounds__(FT_NT) fcg_dir_tile_kernel(DevGrid g, const float2* __restrict__ z,
                                                             const float2* __restrict__ p_old,
                                                             float2* __restrict__ p_new, const float* __restrict__ cc,
                                                             const float* __restrict__ heff, float2* __restrict__ qv,
                                                             const float2* __restrict__ r, double* __restrict__ part,
                                                             const FcgScalars* __restrict__ sc) {
    if (sc->done) return;
    __shared__ FcgTile sm;
    const bool first = sc->iterations == 0;
    const float beta = first ? 0.f : (float)sc->beta;
    const int tx = threadIdx.x % FT_X, ty = threadIdx.x / FT_X;
    const int ntx = (g.nx + FT_X - 1) / FT_X, ntiles = ntx * ((g.ny + FT_Y - 1) / FT_Y);
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i0 = (t % ntx) * FT_X, j0 = (t / ntx) * FT_Y;
        fcg_tile_stage(g, i0, j0, cc, sm, [&](const Mapped& m) {
            const float2 zz = z[m.k];
            const float2 pp = first ? make_float2(0.f, 0.f) : p_old[m.k];
            return make_float2(zz.x + beta * pp.x, zz.y + beta * pp.y);
        });
        const int i = i0 + tx, j = j0 + ty;
        if (i >= g.nx || j >= g.ny) continue;
        const int k = j * g.pitch + i;
        const float2 qq = fcg_tile_apply(g, sm, tx, ty, heff[k]);
        const float2 pp = sm.v[(ty + 2) * FB_W + tx + 2], rr = r[k];
        p_new[k] = pp;
        qv[k] = qq;
        s0 += (double)pp.x * qq.x + (double)pp.y * qq.y;
        s1 += (double)rr.x * pp.x + (double)rr.y * pp.y;
    }
    __shared__ double red[100];
    block_sum3<FT_NT>(s0, s1, s2, red);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = s0;
        part[3 * blockIdx.x + 1] = s1;
        part[3 * blockIdx.x + 2] = 0.0;
    }
}

// upd: w += alpha p, r -= alpha q; partial <r, r>.
__global__ void fcg_upd_kernel(DevGrid g, float2* __restrict__ w, float2* __restrict__ r, const float2* __restrict__ p,
                               const float2* __restrict__ qv, double* __restrict__ part, const FcgScalars* __restrict__ sc) {
    if (sc->done) return;
    const float a = (float)sc->alpha;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int k = (c / g.nx) * g.pitch + c % g.nx;
        float2 ww = w[k], rr = r[k];
        const float2 pp = p[k], qq = qv[k];
        ww.x += a * pp.x;
        ww.y += a * pp.y;
        rr.x -= a * qq.x;
        rr.y -= a * qq.y;
        w[k] = ww;
        r[k] = rr;
        s0 += (double)rr.x * rr.x + (double)rr.y * rr.y;
    }
    __shared__ double red[100];
    block_sum3<256>(s0, s1, s2, red);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = s0;
        part[3 * blockIdx.x + 1] = 0.0;
        part[3 * blockIdx.x + 2] = 0.0;
    }
}

// the features (h / H0, b / H0) as 2 planes (S x S block means, zero outside the interior)
__global__ void lpc_features_kernel(DevGrid g, const float* heff, const float* bed, float* f, int Hp, int Wp, int S) {
    const size_t plane = (size_t)Hp * Wp;
    const float inv = 1.f / (20.0f * (float)(S * S));
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < plane; q += (size_t)gridDim.x * blockDim.x) {
        const int i0 = (int)(q % Wp) * S, j0 = (int)(q / Wp) * S;
        float a = 0.f, b = 0.f;
        for (int u = 0; u < S; u++)
            for (int v = 0; v < S; v++) {
                const int i = i0 + v, j = j0 + u;
                if (i < g.nx && j < g.ny) {
                    const int k = j * g.pitch + i;
                    a += heff[k];
                    b += bed[k];
                }
            }
        f[q] = a * inv;
        f[plane + q] = b * inv;
    }
}

}  // namespace wcb
