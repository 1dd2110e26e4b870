// lpc_host.cuh — host side of the learned preconditioner: the network (forward, backward, Adam)
// over the kernels of lpc.cuh, and its training loop on SGN systems harvested from solves.
//
// No counterpart in the reference. The parameter layout is the one of wavesim_b200/lpc.py
// (UNetSpec.layers): encoder convolutions, decoder convolutions, the 1x1 output, then per level
// the gate network's 3x3 (with bias) and 1x1 (with bias) convolutions.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "common.cuh"
#include "lpc.cuh"

namespace wcb {

constexpr int LPC_LEVELS = 4;
constexpr float LPC_H0 = 20.0f;
// Damping of the cycle's Jacobi sweeps. The Jacobi-scaled operator's spectrum lies in (0, 4) for
// square cells (Gershgorin: the width-2 x-x couplings and the x-y cross couplings add up to at
// most 3 diagonals), so with w = 0.5 the zero network's cycle 2wD^-1 - w^2 D^-1 A D^-1 stays
// positive definite; w = 0.8 is not (eigenvalues near 3 occur on real beds).
constexpr float LPC_OMEGA = 0.5f;

struct LpcLayer {
    int w, b, co, ci, k;  // offsets into the parameter vector (b = -1: no bias)
};

constexpr size_t CONV_MMA_SMEM_MAX = 160 * 1024;

// The tensor-core convolution's shared-memory limit, set once per process before any capture.
// Every instantiation of the channels-innermost convolution: taps x output tiles x padded inputs.
#define CONV_H_FOR_ALL(X)                                                                          \
    X(9, 1, 16) X(9, 1, 32) X(9, 1, 48) X(9, 1, 64) X(9, 2, 16) X(9, 2, 32) X(9, 2, 48) X(9, 2, 64) \
    X(9, 4, 16) X(9, 4, 32) X(9, 4, 48) X(9, 4, 64) X(9, 8, 16) X(9, 8, 32) X(9, 8, 48) X(9, 8, 64) \
    X(1, 1, 16) X(1, 1, 32) X(1, 1, 48) X(1, 1, 64) X(1, 2, 16) X(1, 2, 32) X(1, 2, 48) X(1, 2, 64) \
    X(1, 4, 16) X(1, 4, 32) X(1, 4, 48) X(1, 4, 64) X(1, 8, 16) X(1, 8, 32) X(1, 8, 48) X(1, 8, 64)
constexpr int CONV_H_CP_MAX = 64;
// Instantiations with one row of 16 pixels per warp (16 x 8 tiles), for 32-channel outputs on maps
// whose usual tiles would give fewer than two blocks per SM (the coarse levels): taps x padded inputs.
#define CONV_H1_FOR_ALL(X) X(9, 16) X(9, 32)
constexpr int CONV_H1_MIN_BLOCKS = 2 * 148;
// The decoder convolutions over concat(up(a), b) with the coarse-box staging: output tiles x
// padded inputs x channels of a.
#define CONV_UP_FOR_ALL(X) X(1, 32, 16) X(2, 32, 16) X(2, 48, 32) X(4, 48, 32) X(4, 64, 32) X(8, 64, 32)
// The 8-channel-input convolutions with two taps per K step: output tiles.
#define CONV_P8_FOR_ALL(X) X(1) X(2) X(4)
// The decoder kernels over concat(up(a), an 8-channel b): output tiles x channels of a.
#define CONV_UP8_FOR_ALL(X) X(1, 16) X(1, 32) X(2, 16)

// Once per process (a function-local static is initialised once, also when several host threads
// reach it together); every call returns the first status.
inline cudaError_t conv_mma_configure() {
    static const cudaError_t status = [] {
        cudaError_t st = cudaSuccess;
        const void* ks[] = {(const void*)conv_mma_kernel<9, 1>, (const void*)conv_mma_kernel<9, 2>,
                            (const void*)conv_mma_kernel<9, 4>, (const void*)conv_mma_kernel<9, 8>,
                            (const void*)conv_mma_kernel<1, 1>, (const void*)conv_mma_kernel<1, 2>,
                            (const void*)conv_mma_kernel<1, 4>, (const void*)conv_mma_kernel<1, 8>,
#define CONV_H_PTR(KK_, NT_, CP_) (const void*)conv_h_kernel<KK_, NT_, CP_>,
                            CONV_H_FOR_ALL(CONV_H_PTR)
#undef CONV_H_PTR
#define CONV_H1_PTR(KK_, CP_) (const void*)conv_h_kernel<KK_, 4, CP_, 1>,
                            CONV_H1_FOR_ALL(CONV_H1_PTR)
#undef CONV_H1_PTR
#define CONV_UP_PTR(NT_, CP_, CPA_) (const void*)conv_up_kernel<NT_, CP_, CPA_>,
                            CONV_UP_FOR_ALL(CONV_UP_PTR)
#undef CONV_UP_PTR
#define CONV_P8_PTR(NT_) (const void*)conv_p8_kernel<NT_>,
                            CONV_P8_FOR_ALL(CONV_P8_PTR)
#undef CONV_P8_PTR
#define CONV_UP8_PTR(NT_, CPA_) (const void*)conv_up8_kernel<NT_, CPA_>,
                            CONV_UP8_FOR_ALL(CONV_UP8_PTR)
#undef CONV_UP8_PTR
                            (const void*)conv_enc0_kernel, (const void*)conv_dec0_kernel<16>,
        };
        for (const void* k : ks)
            if (st == cudaSuccess)
                st = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_MMA_SMEM_MAX);
        return st;
    }();
    return status;
}

inline dim3 ew_grid(size_t n) {
    size_t b = (n + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    if (b < 1) b = 1;
    return dim3((unsigned)b);
}

// Device buffer that frees itself.
struct DBuf {
    float* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    cudaError_t alloc(size_t count) {
        if (p) cudaFree(p);
        n = count;
        cudaError_t e = cudaMalloc(&p, (count ? count : 1) * sizeof(float));
        if (e == cudaSuccess) e = cudaMemset(p, 0, (count ? count : 1) * sizeof(float));
        // the memset runs on the legacy stream; the users of the buffer run on non-blocking ones
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
        return e;
    }
    ~DBuf() {
        if (p) cudaFree(p);
    }
};

struct LpcNet {
    int ch[LPC_LEVELS] = {8, 16, 32, 32};
    int hidden = 8;
    int nparams = 0;
    std::vector<LpcLayer> enc_a, enc_b, dec_a, dec_b, gate_a, gate_b;
    LpcLayer out{};
    const float* wq = nullptr;  // the weights the forward pass uses (owned by the model)
    float* gw = nullptr;        // where backward accumulates the weight gradient
    bool tensor = false;        // inference on the tensor cores (BF16 activations), not FP32 FMA
    DBuf wre;                   // tensor-core weights of every layer (BF16 pairs in floats)
    std::vector<size_t> wre_off;  // per layer, in BF16 elements, keyed by the layer's weight offset
    std::vector<int> wre_key;
    std::vector<size_t> wp8_off;  // 3x3 layers of 8 input channels: the two-taps-per-step order
    std::vector<int> wp8_key;
    std::vector<size_t> wu8_off;  // decoder layers over concat(up(a), 8-channel b): the up8 order
    std::vector<int> wu8_key, wu8_cpa;

    // Inference on NHWC BF16 activations (conv_h_kernel): every channel count a multiple of 8
    // and every layer's tile within the shared-memory limit; set by configure_nhwc.
    bool nhwc = false;
    bool fuse_level0 = true;    // the first level's fused launches (conv_enc0_kernel, conv_dec0_kernel)
    bool small_tiles = true;    // 16 x 8 tiles for 32-channel layers on maps too small for two blocks per SM
    const int* done = nullptr;  // the flexible CG's end flag: applications after it are skipped
    DBuf Xh, Yh, Fh[LPC_LEVELS], HIDh[LPC_LEVELS], Gh[LPC_LEVELS], Ah[LPC_LEVELS], Eh[LPC_LEVELS],
        DAh[LPC_LEVELS], Dh[LPC_LEVELS];

    // activations for one batch shape
    int N = 0, H = 0, W = 0;
    DBuf F[LPC_LEVELS], HID[LPC_LEVELS], G[LPC_LEVELS];    // features, gate hidden, gates
    DBuf X[LPC_LEVELS], A[LPC_LEVELS], U[LPC_LEVELS], E[LPC_LEVELS];  // encoder
    DBuf UP[LPC_LEVELS], DA[LPC_LEVELS], DU[LPC_LEVELS], D[LPC_LEVELS];  // decoder
    DBuf Y;
    // gradients
    DBuf dE[LPC_LEVELS], dD[LPC_LEVELS], dG[LPC_LEVELS], t0, t1, t2, wt;

    void layout(const int* channels, int hid) {
        for (int l = 0; l < LPC_LEVELS; l++) ch[l] = channels[l];
        hidden = hid;
        int off = 0;
        auto add = [&](int co, int ci, int k, bool bias) {
            LpcLayer L{off, -1, co, ci, k};
            off += co * ci * k * k;
            if (bias) {
                L.b = off;
                off += co;
            }
            return L;
        };
        enc_a.clear(); enc_b.clear(); dec_a.clear(); dec_b.clear(); gate_a.clear(); gate_b.clear();
        int cin = 2;
        for (int l = 0; l < LPC_LEVELS; l++) {
            enc_a.push_back(add(ch[l], cin, 3, false));
            enc_b.push_back(add(ch[l], ch[l], 3, false));
            cin = ch[l];
        }
        dec_a.resize(LPC_LEVELS);
        dec_b.resize(LPC_LEVELS);
        for (int l = LPC_LEVELS - 2; l >= 0; l--) {
            dec_a[l] = add(ch[l], ch[l + 1] + ch[l], 3, false);
            dec_b[l] = add(ch[l], ch[l], 3, false);
        }
        out = add(2, ch[0], 1, false);
        for (int l = 0; l < LPC_LEVELS; l++) {
            gate_a.push_back(add(hidden, 2, 3, true));
            gate_b.push_back(add(ch[l], hidden, 1, true));
        }
        nparams = off;
    }

    static int mma_tiles(int co) {
        const int nt0 = (co + 7) / 8;
        return nt0 == 1 ? 1 : nt0 == 2 ? 2 : nt0 <= 4 ? 4 : 8;
    }

    // The tensor-core kernel's copy of the forward weights (call again after they change).
    cudaError_t prepare_tensor(cudaStream_t st) {
        wre_off.clear();
        wre_key.clear();
        size_t total = 0;
        std::vector<const LpcLayer*> all;
        for (auto* L : {&enc_a, &enc_b, &dec_a, &dec_b, &gate_a, &gate_b})
            for (auto& l : *L)
                if (l.co > 0) all.push_back(&l);
        all.push_back(&out);
        for (auto* l : all) {
            wre_key.push_back(l->w);
            wre_off.push_back(total);
            total += (size_t)mma_tiles(l->co) * 8 * l->k * l->k * conv_mma_cp(l->ci);
        }
        wp8_off.clear();
        wp8_key.clear();
        for (auto* l : all)
            if ((l->ci == 8 || l->ci == 2) && l->k == 3) {
                wp8_key.push_back(l->w);
                wp8_off.push_back(total);
                total += (size_t)mma_tiles(l->co) * 8 * P8_KP;
            }
        wu8_off.clear();
        wu8_key.clear();
        wu8_cpa.clear();
        for (int l = 0; l + 1 < LPC_LEVELS; l++) {  // dec_a[l]: ch[l + 1] upsampled channels, then ch[l]
            const LpcLayer& d = dec_a[l];
            if (d.co > 0 && ch[l] == 8 && ch[l + 1] % 16 == 0) {
                wu8_key.push_back(d.w);
                wu8_cpa.push_back(ch[l + 1]);
                wu8_off.push_back(total);
                total += (size_t)mma_tiles(d.co) * 8 * (9 * ch[l + 1] + P8_KP);
            }
        }
        cudaError_t e = wre.alloc((total + 1) / 2 + 8);
        if (e != cudaSuccess) return e;
        auto* base = reinterpret_cast<unsigned short*>(wre.p);
        for (size_t n = 0; n < wu8_key.size(); n++) {
            const LpcLayer* l = nullptr;
            for (auto* c : all)
                if (c->w == wu8_key[n]) l = c;
            const int cnt = mma_tiles(l->co) * 8 * (9 * wu8_cpa[n] + P8_KP);
            conv_up8_weights_kernel<<<ew_grid(cnt), 256, 0, st>>>(wq + l->w, l->co, wu8_cpa[n], mma_tiles(l->co),
                                                                  base + wu8_off[n]);
        }
        for (size_t n = 0; n < all.size(); n++) {
            const LpcLayer* l = all[n];
            const int cnt = mma_tiles(l->co) * 8 * l->k * l->k * conv_mma_cp(l->ci);
            conv_mma_weights_kernel<<<ew_grid(cnt), 256, 0, st>>>(wq + l->w, l->co, l->ci, l->k * l->k, mma_tiles(l->co),
                                                                  base + wre_off[n]);
        }
        for (size_t n = 0; n < wp8_key.size(); n++) {
            const LpcLayer* l = nullptr;
            for (auto* c : all)
                if (c->w == wp8_key[n]) l = c;
            conv_p8_weights_kernel<<<ew_grid(mma_tiles(l->co) * 8 * P8_KP), 256, 0, st>>>(wq + l->w, l->co, l->ci,
                                                                                          mma_tiles(l->co), base + wp8_off[n]);
        }
        return cudaGetLastError();
    }

    const unsigned short* wre_of(const LpcLayer& L) const {
        for (size_t n = 0; n < wre_key.size(); n++)
            if (wre_key[n] == L.w) return reinterpret_cast<const unsigned short*>(wre.p) + wre_off[n];
        return nullptr;
    }
    const unsigned short* wu8_of(const LpcLayer& L) const {
        for (size_t n = 0; n < wu8_key.size(); n++)
            if (wu8_key[n] == L.w) return reinterpret_cast<const unsigned short*>(wre.p) + wu8_off[n];
        return nullptr;
    }
    const unsigned short* wp8_of(const LpcLayer& L) const {
        for (size_t n = 0; n < wp8_key.size(); n++)
            if (wp8_key[n] == L.w) return reinterpret_cast<const unsigned short*>(wre.p) + wp8_off[n];
        return nullptr;
    }

    bool configure_nhwc() {
        nhwc = false;
        if (!tensor || hidden % 8) return false;
        for (int l = 0; l < LPC_LEVELS; l++)
            if (ch[l] % 8 || ch[l] > 8 * CM_NMAX) return false;
        for (auto* L : {&enc_a, &enc_b, &dec_a, &dec_b, &gate_a, &gate_b})
            for (auto& l : *L)
                if (l.co > 0 && (conv_mma_cp(l.ci) > CONV_H_CP_MAX ||
                                 conv_h_smem2(l.ci, 8 * mma_tiles(l.co), l.k * l.k, true) > CONV_MMA_SMEM_MAX))
                    return false;
        nhwc = true;
        return true;
    }

    size_t max_weights() const {
        size_t maxw = 0;
        for (auto* L : {&enc_a, &enc_b, &dec_a, &dec_b, &gate_a, &gate_b})
            for (auto& l : *L) maxw = std::max(maxw, (size_t)l.co * l.ci * l.k * l.k);
        return maxw;
    }

    int h_of(int l) const { return H >> l; }
    int w_of(int l) const { return W >> l; }
    size_t sz(int l, int c) const { return (size_t)N * c * h_of(l) * w_of(l); }

    // Activations for batch N of H x W (H, W divisible by 2^(levels-1)); `training` keeps the
    // buffers the backward pass needs.
    cudaError_t shape(int n, int h, int wd, bool training) {
        N = n;
        H = h;
        W = wd;
        cudaError_t e = cudaSuccess;
        auto A_ = [&](DBuf& b, size_t c) {
            if (e == cudaSuccess && b.n != c) e = b.alloc(c);
        };
        for (int l = 0; l < LPC_LEVELS; l++) {
            A_(F[l], sz(l, 2));
            A_(HID[l], sz(l, hidden));
            A_(G[l], sz(l, ch[l]));
            if (l == 0 || training) A_(X[l], sz(l, l == 0 ? 2 : ch[l - 1]));
            A_(A[l], sz(l, ch[l]));
            if (training) A_(U[l], sz(l, ch[l]));
            A_(E[l], sz(l, ch[l]));
            if (l < LPC_LEVELS - 1) {
                if (training) A_(UP[l], sz(l, ch[l + 1]));
                A_(DA[l], sz(l, ch[l]));
                if (training) A_(DU[l], sz(l, ch[l]));
                A_(D[l], sz(l, ch[l]));
            }
            if (training) {
                A_(dE[l], sz(l, ch[l]));
                A_(dD[l], sz(l, ch[l]));
                A_(dG[l], sz(l, ch[l]));
            }
        }
        A_(Y, sz(0, 2));
        if (nhwc && !training) {  // BF16 halves, two per float of the buffer
            auto H_ = [&](DBuf& b, size_t halves) { A_(b, (halves + 1) / 2); };
            H_(Xh, sz(0, 2));
            A_(Yh, sz(0, 2));
            for (int l = 0; l < LPC_LEVELS; l++) {
                H_(Fh[l], sz(l, 2));
                H_(HIDh[l], sz(l, hidden));
                H_(Gh[l], sz(l, ch[l]));
                H_(Ah[l], sz(l, ch[l]));
                H_(Eh[l], sz(l, ch[l]));
                if (l < LPC_LEVELS - 1) {
                    H_(DAh[l], sz(l, ch[l]));
                    H_(Dh[l], sz(l, ch[l]));
                }
            }
        }
        if (training) {
            size_t big = 0;
            for (int l = 0; l < LPC_LEVELS; l++) big = std::max(big, sz(l, ch[l] + (l + 1 < LPC_LEVELS ? ch[l + 1] : 0) + hidden + 2));
            A_(t0, big);
            A_(t1, big);
            A_(t2, big);
            A_(wt, max_weights());
        }
        return e;
    }

    cudaError_t conv(const float* a, int ca, int amode, const float* b, int cb, const LpcLayer& L, const float* weights,
                     const float* gate, float* y, int level, int act, cudaStream_t st) const {
        ConvArgs p{};
        p.a = a;
        p.ca = ca;
        p.amode = amode;
        p.b = b;
        p.cb = cb;
        p.w = weights + L.w;
        p.bias = L.b >= 0 ? weights + L.b : nullptr;
        p.gate = gate;
        p.y = y;
        p.co = L.co;
        p.H = h_of(level);
        p.W = w_of(level);
        p.N = N;
        p.act = act;
        p.wre = tensor ? wre_of(L) : nullptr;
        if (p.wre && L.co <= 8 * CM_NMAX) {
            const int nt = mma_tiles(L.co);  // the instantiation's tiles
            const size_t smem = conv_mma_smem(L.ci, 8 * nt, L.k * L.k);
            if (smem <= CONV_MMA_SMEM_MAX) {
                dim3 grid((p.W + CM_TX - 1) / CM_TX, (p.H + CM_TY - 1) / CM_TY, N);
#define CONV_MMA_LAUNCH(KK_, NT_) conv_mma_kernel<KK_, NT_><<<grid, CM_NT, smem, st>>>(p)
                if (L.k == 3) {
                    if (nt == 1) CONV_MMA_LAUNCH(9, 1);
                    else if (nt == 2) CONV_MMA_LAUNCH(9, 2);
                    else if (nt <= 4) CONV_MMA_LAUNCH(9, 4);
                    else CONV_MMA_LAUNCH(9, 8);
                } else {
                    if (nt == 1) CONV_MMA_LAUNCH(1, 1);
                    else if (nt == 2) CONV_MMA_LAUNCH(1, 2);
                    else if (nt <= 4) CONV_MMA_LAUNCH(1, 4);
                    else CONV_MMA_LAUNCH(1, 8);
                }
#undef CONV_MMA_LAUNCH
                return cudaGetLastError();
            }
        }
        // 32 x 32 tiles while they give every SM a few blocks, 16 x 16 below
        const int groups = N * ((L.co + CV_COB - 1) / CV_COB);
        const bool big = (size_t)((p.W + 31) / 32) * ((p.H + 31) / 32) * groups >= 4 * 148;
        const int T = big ? 2 * CV_TH : CV_TH;
        dim3 grid((p.W + T - 1) / T, (p.H + T - 1) / T, groups);
        if (L.k == 3) {
            if (big) conv_fwd_kernel<3, 2><<<grid, CV_TH * CV_TH, 0, st>>>(p);
            else conv_fwd_kernel<3, 1><<<grid, CV_TH * CV_TH, 0, st>>>(p);
        } else {
            if (big) conv_fwd_kernel<1, 2><<<grid, CV_TH * CV_TH, 0, st>>>(p);
            else conv_fwd_kernel<1, 1><<<grid, CV_TH * CV_TH, 0, st>>>(p);
        }
        return cudaGetLastError();
    }

    static const unsigned short* hp(const DBuf& b) { return reinterpret_cast<const unsigned short*>(b.p); }
    static unsigned short* hp(DBuf& b) { return reinterpret_cast<unsigned short*>(b.p); }

    // One convolution on NHWC BF16 activations (conv_h_kernel); yf: FP32 output instead of y.
    cudaError_t conv_h(const unsigned short* a, int ca, int amode, const unsigned short* b, int cb, const LpcLayer& L,
                       const unsigned short* gate, unsigned short* y, float* yf, int level, int act,
                       cudaStream_t st, const float* out_w = nullptr) const {
        ConvH p{};
        p.a = a;
        p.ca = ca;
        p.amode = amode;
        p.b = b;
        p.cb = cb;
        p.wre = wre_of(L);
        p.bias = L.b >= 0 ? wq + L.b : nullptr;
        p.gate = gate;
        p.y = y;
        p.yf = yf;
        p.done = done;
        p.out_w = out_w;
        p.co = L.co;
        p.H = h_of(level);
        p.W = w_of(level);
        p.N = N;
        p.act = act;
        const int nt = mma_tiles(L.co);
        const int th = 8 * conv_h_rows(nt);
        dim3 grid((p.W + CM_TX - 1) / CM_TX, (p.H + th - 1) / th, N);
        const int kk = L.k * L.k, cp = conv_mma_cp(L.ci);
        bool launched = false;
        if (kk == 9 && (ca == 8 || (ca == 2 && amode == CM_DIRECT)) && cb == 0 && amode != CM_UP &&
            wp8_of(L)) {  // two taps per K step
            const size_t smem = conv_p8_smem(8 * nt, gate != nullptr);
            p.wre = wp8_of(L);
#define CONV_P8_LAUNCH(NT_)                                               \
            if (!launched && nt == NT_) {                                  \
                conv_p8_kernel<NT_><<<grid, CM_NT, smem, st>>>(p);         \
                launched = true;                                           \
            }
            CONV_P8_FOR_ALL(CONV_P8_LAUNCH)
#undef CONV_P8_LAUNCH
            if (launched) return cudaGetLastError();
            p.wre = wre_of(L);
        }
        if (amode == CM_UP && kk == 9 && ca % 16 == 0 && cb == 8 && b && wu8_of(L)) {  // 8-channel skip
            const size_t smem = conv_up8_smem(ca, 8 * nt, gate != nullptr);
            const int thu = 8 * conv_up_rows(nt);
            const dim3 grid_up((p.W + CM_TX - 1) / CM_TX, (p.H + thu - 1) / thu, N);
            p.wre = wu8_of(L);
#define CONV_UP8_LAUNCH(NT_, CPA_)                                              \
            if (!launched && nt == NT_ && ca == CPA_ && smem <= CONV_MMA_SMEM_MAX) {  \
                conv_up8_kernel<NT_, CPA_><<<grid_up, CM_NT, smem, st>>>(p);     \
                launched = true;                                                 \
            }
            CONV_UP8_FOR_ALL(CONV_UP8_LAUNCH)
#undef CONV_UP8_LAUNCH
            if (launched) return cudaGetLastError();
            p.wre = wre_of(L);
        }
        if (amode == CM_UP && kk == 9 && ca % 16 == 0 && b) {  // the coarse-box decoder kernel
            const size_t smem = conv_up_smem(ca, cp, 8 * nt, gate != nullptr);
            const int thu = 8 * conv_up_rows(nt);
            const dim3 grid_up((p.W + CM_TX - 1) / CM_TX, (p.H + thu - 1) / thu, N);
#define CONV_UP_LAUNCH(NT_, CP_, CPA_)                                          \
            if (!launched && nt == NT_ && cp == CP_ && ca == CPA_ && smem <= CONV_MMA_SMEM_MAX) { \
                conv_up_kernel<NT_, CP_, CPA_><<<grid_up, CM_NT, smem, st>>>(p); \
                launched = true;                                                 \
            }
            CONV_UP_FOR_ALL(CONV_UP_LAUNCH)
#undef CONV_UP_LAUNCH
            if (launched) return cudaGetLastError();
        }
        if (nt == 4 && (size_t)grid.x * grid.y * grid.z < CONV_H1_MIN_BLOCKS && small_tiles) {
            const size_t smem1 = conv_h_smem2(L.ci, 8 * nt, L.k * L.k, gate != nullptr, 1);
            const dim3 grid1(grid.x, (p.H + 7) / 8, N);
#define CONV_H1_LAUNCH(KK_, CP_)                                                   \
            if (!launched && kk == KK_ && cp == CP_) {                              \
                conv_h_kernel<KK_, 4, CP_, 1><<<grid1, CM_NT, smem1, st>>>(p);     \
                launched = true;                                                    \
            }
            CONV_H1_FOR_ALL(CONV_H1_LAUNCH)
#undef CONV_H1_LAUNCH
            if (launched) return cudaGetLastError();
        }
        const size_t smem = conv_h_smem2(L.ci, 8 * nt, L.k * L.k, gate != nullptr);
#define CONV_H_LAUNCH(KK_, NT_, CP_)                                          \
        if (!launched && kk == KK_ && nt == NT_ && cp == CP_) {                 \
            conv_h_kernel<KK_, NT_, CP_><<<grid, CM_NT, smem, st>>>(p);        \
            launched = true;                                                   \
        }
        CONV_H_FOR_ALL(CONV_H_LAUNCH)
#undef CONV_H_LAUNCH
        if (!launched) return cudaErrorInvalidConfiguration;
        return cudaGetLastError();
    }

    // The gates on NHWC BF16 from the level-0 features F[0] (NCHW FP32): 3 launches a level.
    cudaError_t gates_h(cudaStream_t st) {
        cudaError_t e = cudaSuccess;
        for (int l = 0; l < LPC_LEVELS && e == cudaSuccess; l++) {
            features_h_kernel<<<ew_grid(sz(l, 1)), 256, 0, st>>>(F[0].p, N, H, W, l, hp(Fh[l]));
            e = conv_h(hp(Fh[l]), 2, CM_DIRECT, nullptr, 0, gate_a[l], nullptr, hp(HIDh[l]), nullptr, l, ACT_RELU, st);
            if (e == cudaSuccess)
                e = conv_h(hp(HIDh[l]), hidden, CM_DIRECT, nullptr, 0, gate_b[l], nullptr, hp(Gh[l]), nullptr, l, ACT_SIG2, st);
        }
        return e;
    }

    // The output layer rides in dec_b[0]'s epilogue when that layer has one tile of 8 channels.
    bool fused_out() const { return ch[0] == 8 && out.co == 2 && out.k == 1; }
    // The first level's two encoder layers in one launch (conv_enc0_kernel) when both are 8-channel
    // 3x3 layers in the two-taps order and the first has no bias (the network's form: linear, the
    // second gated). The fused kernel applies no activation to the first layer's map: forward_h
    // runs every layer with ACT_NONE, and a network with activations would need the per-layer path.
    bool fused_enc0() const {
        return fuse_level0 && ch[0] == 8 && enc_a[0].k == 3 && enc_a[0].ci == 2 && enc_a[0].b < 0 && enc_b[0].k == 3 && enc_b[0].ci == 8 &&
               wp8_of(enc_a[0]) && wp8_of(enc_b[0]);
    }
    // The first level's two decoder layers and the output layer in one launch (conv_dec0_kernel)
    // when the output layer is fused, the first decoder layer has no bias and takes 16 coarse
    // channels in the up8 order, and the second is an 8-channel 3x3 layer in the two-taps order.
    // As for fused_enc0, the first layer's map gets no activation, matching forward_h's ACT_NONE.
    bool fused_dec0() const {
        return fuse_level0 && LPC_LEVELS > 2 && fused_out() && ch[1] == 16 && dec_a[0].k == 3 && dec_a[0].b < 0 && dec_b[0].k == 3 &&
               dec_b[0].ci == 8 && wu8_of(dec_a[0]) && wp8_of(dec_b[0]);
    }
    // launches of forward_h()
    int forward_h_launches() const {
        return 2 * LPC_LEVELS + 2 * (LPC_LEVELS - 1) + (fused_out() ? 0 : 1) - (fused_enc0() ? 1 : 0) -
               (fused_dec0() ? 1 : 0);
    }

    // The first level's decoder through conv_dec0_kernel: Yh = out(conv(conv(concat(up(Dh[1]), Eh[0]))) * Gh[0]).
    cudaError_t dec0_h(cudaStream_t st) {
        ConvH p{};
        p.a = hp(Dh[1]);
        p.ca = 16;
        p.amode = CM_UP;
        p.b = hp(Eh[0]);
        p.cb = 8;
        p.wre = wu8_of(dec_a[0]);
        p.wre2 = wp8_of(dec_b[0]);
        p.bias = dec_b[0].b >= 0 ? wq + dec_b[0].b : nullptr;
        p.gate = hp(Gh[0]);
        p.yf = Yh.p;
        p.out_w = wq + out.w;
        p.done = done;
        p.co = 8;
        p.H = H;
        p.W = W;
        p.N = N;
        p.act = ACT_NONE;
        const dim3 grid((W + CM_TX - 1) / CM_TX, (H + 8 * conv_h_rows(1) - 1) / (8 * conv_h_rows(1)), N);
        conv_dec0_kernel<16><<<grid, CM_NT, conv_dec0_smem<16>(), st>>>(p);
        return cudaGetLastError();
    }

    // The first level's encoder through conv_enc0_kernel: Eh[0] = conv(conv(Xh)) * Gh[0].
    cudaError_t enc0_h(cudaStream_t st) {
        ConvH p{};
        p.a = hp(Xh);
        p.ca = 2;
        p.amode = CM_DIRECT;
        p.wre = wp8_of(enc_a[0]);
        p.wre2 = wp8_of(enc_b[0]);
        p.bias = enc_b[0].b >= 0 ? wq + enc_b[0].b : nullptr;
        p.gate = hp(Gh[0]);
        p.y = hp(Eh[0]);
        p.done = done;
        p.co = 8;
        p.H = H;
        p.W = W;
        p.N = N;
        p.act = ACT_NONE;
        const dim3 grid((W + CM_TX - 1) / CM_TX, (H + 8 * conv_h_rows(1) - 1) / (8 * conv_h_rows(1)), N);
        conv_enc0_kernel<<<grid, CM_NT, conv_enc0_smem(), st>>>(p);
        return cudaGetLastError();
    }

    // Yh = N(Xh) on NHWC BF16 activations with the gates already in Gh: the launches of forward()
    // (the output layer fused into the last when fused_out()).
    cudaError_t forward_h(cudaStream_t st) {
        cudaError_t e = cudaSuccess;
        for (int l = 0; l < LPC_LEVELS && e == cudaSuccess; l++) {
            if (l == 0 && fused_enc0()) {
                e = enc0_h(st);
                continue;
            }
            const int cin = l == 0 ? 2 : ch[l - 1];
            const unsigned short* in = l == 0 ? hp(Xh) : hp(Eh[l - 1]);
            e = conv_h(in, cin, l == 0 ? CM_DIRECT : CM_POOL, nullptr, 0, enc_a[l], nullptr, hp(Ah[l]), nullptr, l,
                       ACT_NONE, st);
            if (e == cudaSuccess)
                e = conv_h(hp(Ah[l]), ch[l], CM_DIRECT, nullptr, 0, enc_b[l], hp(Gh[l]), hp(Eh[l]), nullptr, l, ACT_NONE, st);
        }
        for (int l = LPC_LEVELS - 2; l >= 0 && e == cudaSuccess; l--) {
            if (l == 0 && fused_dec0()) {
                e = dec0_h(st);
                break;
            }
            const unsigned short* below = (l == LPC_LEVELS - 2) ? hp(Eh[l + 1]) : hp(Dh[l + 1]);
            e = conv_h(below, ch[l + 1], CM_UP, hp(Eh[l]), ch[l], dec_a[l], nullptr, hp(DAh[l]), nullptr, l, ACT_NONE, st);
            if (e != cudaSuccess) break;
            if (l == 0 && fused_out())  // dec_b[0] with the 1x1 output layer in its epilogue
                e = conv_h(hp(DAh[0]), ch[0], CM_DIRECT, nullptr, 0, dec_b[0], hp(Gh[0]), nullptr, Yh.p, 0, ACT_NONE, st,
                           wq + out.w);
            else
                e = conv_h(hp(DAh[l]), ch[l], CM_DIRECT, nullptr, 0, dec_b[l], hp(Gh[l]), hp(Dh[l]), nullptr, l, ACT_NONE, st);
        }
        if (e == cudaSuccess && !fused_out())
            e = conv_h(hp(Dh[0]), ch[0], CM_DIRECT, nullptr, 0, out, nullptr, nullptr, Yh.p, 0, ACT_NONE, st);
        return e;
    }

    // Gates of every level from the features F[0] (h / H0, b / H0): constant within a solve.
    cudaError_t gates(cudaStream_t st) {
        cudaError_t e = cudaSuccess;
        for (int l = 0; l < LPC_LEVELS && e == cudaSuccess; l++) {
            if (l > 0) pool2_kernel<<<ew_grid(sz(l, 2)), 256, 0, st>>>(F[l - 1].p, N * 2, h_of(l - 1), w_of(l - 1), F[l].p, 0.25f, 0);
            e = conv(F[l].p, 2, CM_DIRECT, nullptr, 0, gate_a[l], wq, nullptr, HID[l].p, l, ACT_RELU, st);
            if (e == cudaSuccess) e = conv(HID[l].p, hidden, CM_DIRECT, nullptr, 0, gate_b[l], wq, nullptr, G[l].p, l, ACT_SIG2, st);
        }
        return e;
    }

    // Y = N(X[0]) with the gates already in G. `keep`: materialise what backward needs
    // (pooled inputs, upsampled skips, pre-gate maps); otherwise pooling and upsampling are read
    // on the fly by the convolutions and the gate is applied in their epilogue.
    cudaError_t forward(cudaStream_t st, bool keep) {
        cudaError_t e = cudaSuccess;
        for (int l = 0; l < LPC_LEVELS && e == cudaSuccess; l++) {
            const int cin = l == 0 ? 2 : ch[l - 1];
            const float* in = l == 0 ? X[0].p : E[l - 1].p;
            int mode = l == 0 ? CM_DIRECT : CM_POOL;
            if (keep && l > 0) {
                pool2_kernel<<<ew_grid(sz(l, cin)), 256, 0, st>>>(E[l - 1].p, N * cin, h_of(l - 1), w_of(l - 1), X[l].p, 0.25f, 0);
                in = X[l].p;
                mode = CM_DIRECT;
            }
            e = conv(in, cin, mode, nullptr, 0, enc_a[l], wq, nullptr, A[l].p, l, ACT_NONE, st);
            if (e != cudaSuccess) break;
            if (keep) {
                e = conv(A[l].p, ch[l], CM_DIRECT, nullptr, 0, enc_b[l], wq, nullptr, U[l].p, l, ACT_NONE, st);
                if (e == cudaSuccess) e = product(E[l].p, U[l].p, G[l].p, sz(l, ch[l]), st);  // E = U * G
            } else {
                e = conv(A[l].p, ch[l], CM_DIRECT, nullptr, 0, enc_b[l], wq, G[l].p, E[l].p, l, ACT_NONE, st);
            }
        }
        for (int l = LPC_LEVELS - 2; l >= 0 && e == cudaSuccess; l--) {
            const float* below = (l == LPC_LEVELS - 2) ? E[l + 1].p : D[l + 1].p;
            const float* a_in = below;
            int mode = CM_UP;
            if (keep) {
                up2_kernel<<<ew_grid(sz(l, ch[l + 1])), 256, 0, st>>>(below, N * ch[l + 1], h_of(l + 1), w_of(l + 1), UP[l].p, 1.f, 0);
                a_in = UP[l].p;
                mode = CM_DIRECT;
            }
            e = conv(a_in, ch[l + 1], mode, E[l].p, ch[l], dec_a[l], wq, nullptr, DA[l].p, l, ACT_NONE, st);
            if (e != cudaSuccess) break;
            if (keep) {
                e = conv(DA[l].p, ch[l], CM_DIRECT, nullptr, 0, dec_b[l], wq, nullptr, DU[l].p, l, ACT_NONE, st);
                if (e == cudaSuccess) e = product(D[l].p, DU[l].p, G[l].p, sz(l, ch[l]), st);  // D = DU * G
            } else {
                e = conv(DA[l].p, ch[l], CM_DIRECT, nullptr, 0, dec_b[l], wq, G[l].p, D[l].p, l, ACT_NONE, st);
            }
        }
        if (e == cudaSuccess) e = conv(D[0].p, ch[0], CM_DIRECT, nullptr, 0, out, wq, nullptr, Y.p, 0, ACT_NONE, st);
        return e;
    }

    static cudaError_t product(float* y, const float* u, const float* g, size_t n, cudaStream_t st);
    static cudaError_t accumulate(float* y, const float* x, size_t n, cudaStream_t st);

    // dx = input gradient of the convolution L (weights transposed into wt), dW accumulated.
    cudaError_t conv_bwd(const float* dy, const float* xa, int ca, const float* xb, int cb, const LpcLayer& L,
                         float* dx, int level, cudaStream_t st) {
        const int ci = ca + cb;
        if (dx) {
            transpose_weights_kernel<<<ew_grid((size_t)L.co * ci * L.k * L.k), 256, 0, st>>>(wq + L.w, L.co, ci, L.k, wt.p);
            LpcLayer T{0, -1, ci, L.co, L.k};
            cudaError_t e = conv(dy, L.co, CM_DIRECT, nullptr, 0, T, wt.p, nullptr, dx, level, ACT_NONE, st);
            if (e != cudaSuccess) return e;
        }
        if (L.k == 3)
            conv_wgrad_kernel<3><<<L.co * ci, 256, 0, st>>>(dy, xa, ca, xb, cb, L.co, h_of(level), w_of(level), N, gw + L.w);
        else
            conv_wgrad_kernel<1><<<L.co * ci, 256, 0, st>>>(dy, xa, ca, xb, cb, L.co, h_of(level), w_of(level), N, gw + L.w);
        if (L.b >= 0) bias_grad_kernel<<<L.co, 256, 0, st>>>(dy, L.co, h_of(level), w_of(level), N, gw + L.b);
        return cudaGetLastError();
    }

    // Gradients of sum(dY * Y) into g (which the caller zeroes) and, if dX0 is given, into X[0].
    cudaError_t backward(const float* dY, float* dX0, cudaStream_t st) {
        cudaError_t e;
        for (int l = 0; l < LPC_LEVELS; l++) {
            cudaMemsetAsync(dE[l].p, 0, dE[l].n * sizeof(float), st);
            cudaMemsetAsync(dG[l].p, 0, dG[l].n * sizeof(float), st);
        }
        if ((e = conv_bwd(dY, D[0].p, ch[0], nullptr, 0, out, dD[0].p, 0, st)) != cudaSuccess) return e;
        for (int l = 0; l < LPC_LEVELS - 1; l++) {
            const size_t n = sz(l, ch[l]);
            gate_bwd_kernel<<<ew_grid(n), 256, 0, st>>>(dD[l].p, DU[l].p, G[l].p, t0.p, dG[l].p, n);  // t0 = dDU
            if ((e = conv_bwd(t0.p, DA[l].p, ch[l], nullptr, 0, dec_b[l], t1.p, l, st)) != cudaSuccess) return e;  // t1 = dDA
            if ((e = conv_bwd(t1.p, UP[l].p, ch[l + 1], E[l].p, ch[l], dec_a[l], t2.p, l, st)) != cudaSuccess) return e;  // t2 = dcat
            // dE[l] += dcat[:, C_{l+1}:]; dD[l+1] = up_bwd(dcat[:, :C_{l+1}])
            const size_t plane = (size_t)h_of(l) * w_of(l);
            for (int n_ = 0; n_ < N; n_++) {
                const float* src = t2.p + ((size_t)n_ * (ch[l + 1] + ch[l]) + ch[l + 1]) * plane;
                float* dst = dE[l].p + (size_t)n_ * ch[l] * plane;
                if ((e = accumulate(dst, src, (size_t)ch[l] * plane, st)) != cudaSuccess) return e;
                float* dbelow = (l + 1 == LPC_LEVELS - 1) ? dE[l + 1].p : dD[l + 1].p;
                pool2_kernel<<<ew_grid((size_t)ch[l + 1] * plane / 4), 256, 0, st>>>(
                    t2.p + (size_t)n_ * (ch[l + 1] + ch[l]) * plane, ch[l + 1], h_of(l), w_of(l),
                    dbelow + (size_t)n_ * ch[l + 1] * plane / 4, 1.f, (l + 1 == LPC_LEVELS - 1) ? 1 : 0);
            }
        }
        for (int l = LPC_LEVELS - 1; l >= 0; l--) {
            const size_t n = sz(l, ch[l]);
            gate_bwd_kernel<<<ew_grid(n), 256, 0, st>>>(dE[l].p, U[l].p, G[l].p, t0.p, dG[l].p, n);  // t0 = dU
            if ((e = conv_bwd(t0.p, A[l].p, ch[l], nullptr, 0, enc_b[l], t1.p, l, st)) != cudaSuccess) return e;  // t1 = dA
            const int cin = l == 0 ? 2 : ch[l - 1];
            float* dx = (l == 0) ? dX0 : t2.p;
            if ((e = conv_bwd(t1.p, X[l].p, cin, nullptr, 0, enc_a[l], dx, l, st)) != cudaSuccess) return e;
            if (l > 0)  // dE[l-1] += pool_bwd(dX[l]) = up(dX[l]) / 4
                up2_kernel<<<ew_grid(sz(l - 1, cin)), 256, 0, st>>>(t2.p, N * cin, h_of(l), w_of(l), dE[l - 1].p, 0.25f, 1);
        }
        for (int l = 0; l < LPC_LEVELS; l++) {
            const size_t n = sz(l, ch[l]);
            sig2_relu_bwd_kernel<<<ew_grid(n), 256, 0, st>>>(dG[l].p, G[l].p, n, ACT_SIG2);  // dG -> dZ
            if ((e = conv_bwd(dG[l].p, HID[l].p, hidden, nullptr, 0, gate_b[l], t1.p, l, st)) != cudaSuccess) return e;
            const size_t nh = sz(l, hidden);
            sig2_relu_bwd_kernel<<<ew_grid(nh), 256, 0, st>>>(t1.p, HID[l].p, nh, ACT_RELU);
            if ((e = conv_bwd(t1.p, F[l].p, 2, nullptr, 0, gate_a[l], nullptr, l, st)) != cudaSuccess) return e;
        }
        return cudaGetLastError();
    }
};

__global__ void product_kernel(float* __restrict__ y, const float* __restrict__ u, const float* __restrict__ g, size_t n) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        y[q] = u[q] * g[q];
}

__global__ void accumulate_kernel(float* __restrict__ y, const float* __restrict__ x, size_t n) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) y[q] += x[q];
}

inline cudaError_t LpcNet::product(float* y, const float* u, const float* g, size_t n, cudaStream_t st) {
    product_kernel<<<ew_grid(n), 256, 0, st>>>(y, u, g, n);
    return cudaGetLastError();
}

inline cudaError_t LpcNet::accumulate(float* y, const float* x, size_t n, cudaStream_t st) {
    accumulate_kernel<<<ew_grid(n), 256, 0, st>>>(y, x, n);
    return cudaGetLastError();
}

// ---- training --------------------------------------------------------------------------

// A patch of a harvested system: c, heff and the bed cropped into the batch tensors, the mask
// (h >= 5 cm) and the features (h / H0, b / H0).
// (c may be oc and heff oheff: every element is read before it is written.)
__global__ void crop_kernel(const float* c, const float* heff, const float* __restrict__ bed, int pitch, int x0, int y0,
                            int H, int W, float* oc, float* oheff, float* __restrict__ omask, float* __restrict__ ofeat) {
    const int plane = H * W;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < plane; q += gridDim.x * blockDim.x) {
        const int y = q / W, x = q % W;
        const size_t k = (size_t)(y0 + y) * pitch + (x0 + x);
        const float he = heff[k];
        oc[q] = c[k];
        oheff[q] = he;
        omask[q] = he >= H_DISP_MIN ? 1.f : 0.f;
        ofeat[q] = he / LPC_H0;
        ofeat[plane + q] = bed[k] / LPC_H0;
    }
}

struct LpcSystem {
    int nx, ny, pitch;
    float dx, dy;
    DBuf c, heff, bed;
};

struct LpcTrainer {
    int N = 0, H = 0, W = 0;
    float dx = 1.f, dy = 1.f;
    int S = 1;  // the network's grid is S times coarser
    DBuf c, heff, mask, e, r, dg, z1, tmp, zj, z2, z, dd, ad, feat, yf, gz, gz2, dyc;
    double* sums = nullptr;  // [2][N]: <d, A d>, <e, A e>
    ~LpcTrainer() {
        if (sums) cudaFree(sums);
    }
    cudaError_t shape(int n, int h, int w) {
        N = n;
        H = h;
        W = w;
        const size_t one = (size_t)n * h * w, two = 2 * one;
        cudaError_t er = cudaSuccess;
        for (DBuf* b : {&c, &heff, &mask}) if (er == cudaSuccess && b->n != one) er = b->alloc(one);
        for (DBuf* b : {&e, &r, &dg, &z1, &tmp, &zj, &z2, &z, &dd, &ad, &feat, &yf, &gz, &gz2})
            if (er == cudaSuccess && b->n != two) er = b->alloc(two);
        if (er == cudaSuccess && dyc.n != two / (S * S)) er = dyc.alloc(two / (S * S));
        if (er == cudaSuccess) {
            if (sums) cudaFree(sums);
            er = cudaMalloc(&sums, 2 * n * sizeof(double));
        }
        return er;
    }
    PatchOp op() const {
        PatchOp o;
        o.c = c.p;
        o.heff = heff.p;
        o.mask = mask.p;
        o.H = H;
        o.W = W;
        o.N = N;
        o.ix = 0.5f / dx;
        o.iy = 0.5f / dy;
        o.dx2i = 0.25f / (dx * dx);
        o.dy2i = 0.25f / (dy * dy);
        return o;
    }
};

// out = ax * x + ay * y / d * mask over 2-plane fields of N samples (any of y's modifiers null).
inline void fld(float* out, const float* x, float ax, const float* y, float ay, const float* d, const float* mask, int N,
                size_t plane, cudaStream_t st) {
    const size_t n = (size_t)N * 2 * plane;
    lincomb_kernel<<<ew_grid(n), 256, 0, st>>>(out, x, ax, y, ay, d, mask, 2, n, plane);
}


// loss[step] = mean over samples of <d, A d> / <e, A e>
__global__ void lpc_loss_kernel(const double* __restrict__ sums, int N, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double l = 0.0;
    for (int n = 0; n < N; n++) l += sums[N + n] > 0.0 ? sums[n] / sums[N + n] : 0.0;  // all-dry patch: 0
    *out = l / N;
}

// The trained network and what training needs: parameters with Adam moments, harvested systems,
// the batch buffers.
struct LpcModel {
    LpcNet net;      // layout; activations of the training batch
    DBuf w, wq, g, m, v;
    int adam_t = 0;
    int round_bf16 = 1;
    int stride = 1;  // the network runs on a grid this many times coarser than the solver's
    std::vector<LpcSystem*> systems;
    LpcTrainer tr;
    double* dloss = nullptr;  // the loss of every step of a training call
    size_t dloss_n = 0;
    unsigned long long rng = 0x9e3779b97f4a7c15ull;
    cudaStream_t st = nullptr;

    ~LpcModel() {
        for (auto* q : systems) delete q;
        if (dloss) cudaFree(dloss);
        if (st) cudaStreamDestroy(st);
    }

    cudaError_t init(const int* channels, int hidden, int S) {
        stride = S;
        tr.S = S;
        net.layout(channels, hidden);
        cudaError_t e;
        for (DBuf* b : {&w, &wq, &g, &m, &v})
            if ((e = b->alloc(net.nparams)) != cudaSuccess) return e;
        net.wq = wq.p;
        net.gw = g.p;
        return cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    }

    // The forward copy from the master weights (BF16-rounded unless rounding is off).
    cudaError_t refresh() {
        round_copy_kernel<<<ew_grid(net.nparams), 256, 0, st>>>(w.p, wq.p, net.nparams, round_bf16);
        return cudaGetLastError();
    }

    unsigned long long next() {
        rng ^= rng << 13;
        rng ^= rng >> 7;
        rng ^= rng << 17;
        return rng;
    }

    cudaError_t shape_batch(int N, int H, int W) {
        cudaError_t e;
        if (tr.N != N || tr.H != H || tr.W != W)
            if ((e = tr.shape(N, H, W)) != cudaSuccess) return e;
        return net.shape(N, H / stride, W / stride, true);
    }

    // where crops put the features: the network's input directly, or the fine-grid buffer
    float* fine_features() { return stride == 1 ? net.F[0].p : tr.feat.p; }

    // the network's features from the fine ones (block means)
    cudaError_t pool_features() {
        if (stride == 1) return cudaSuccess;
        const size_t nc = (size_t)tr.N * 2 * (tr.H / stride) * (tr.W / stride);
        pool_s_kernel<<<ew_grid(nc), 256, 0, st>>>(tr.feat.p, tr.N * 2, tr.H, tr.W, stride, net.F[0].p,
                                                   1.f / (float)(stride * stride));
        return cudaGetLastError();
    }

    // A training batch: N patches of H x W from random systems and offsets (all of one grid
    // spacing), one random error field each.
    cudaError_t sample_batch(int N, int H, int W, float rough) {
        cudaError_t e;
        if ((e = shape_batch(N, H, W)) != cudaSuccess) return e;
        const size_t plane = (size_t)H * W, per = 2 * plane;
        const LpcSystem* s0 = systems[next() % systems.size()];
        std::vector<const LpcSystem*> pool;
        for (auto* q : systems)
            if (q->dx == s0->dx && q->dy == s0->dy && q->nx >= W && q->ny >= H) pool.push_back(q);
        if (pool.empty()) return cudaErrorInvalidValue;
        for (int n = 0; n < N; n++) {
            const LpcSystem* sy = pool[next() % pool.size()];
            const int x0 = (int)(next() % (unsigned long long)(sy->nx - W + 1));
            const int y0 = (int)(next() % (unsigned long long)(sy->ny - H + 1));
            crop_kernel<<<ew_grid(plane), 256, 0, st>>>(sy->c.p, sy->heff.p, sy->bed.p, sy->pitch, x0, y0, H, W,
                                                        tr.c.p + n * plane, tr.heff.p + n * plane,
                                                        tr.mask.p + n * plane, fine_features() + n * per);
        }
        tr.dx = s0->dx;
        tr.dy = s0->dy;
        random_field_kernel<<<ew_grid((size_t)N * per), 256, 0, st>>>(tr.e.p, tr.mask.p, N, H, W, next(), rough);
        return pool_features();
    }

    // The loss mean_n <d, A d>_n / <e, A e>_n of the cycle's error d = e - M A e on the batch in
    // tr (c, heff, mask, e) and net.F[0] (features), into *loss_slot; with `grad`, its gradient
    // through the cycle and the network into g.
    cudaError_t loss_grad(double* loss_slot, bool grad) {
        cudaError_t e;
        const int N = tr.N, H = tr.H, W = tr.W;
        const size_t plane = (size_t)H * W, per = 2 * plane, tot = (size_t)N * per;
        const PatchOp op = tr.op();
        const float om = LPC_OMEGA;
        patch_matvec_kernel<<<ew_grid(N * plane), 256, 0, st>>>(op, tr.e.p, tr.r.p);   // r = A e
        patch_diag_kernel<<<ew_grid(N * plane), 256, 0, st>>>(op, tr.dg.p);
        fld(tr.z1.p, nullptr, 0.f, tr.r.p, om, tr.dg.p, nullptr, N, plane, st);       // z1 = w r / D
        patch_matvec_kernel<<<ew_grid(N * plane), 256, 0, st>>>(op, tr.z1.p, tr.tmp.p);
        fld(tr.zj.p, tr.r.p, 1.f, tr.tmp.p, -1.f, nullptr, nullptr, N, plane, st);      // r - A z1
        const int S = stride;
        const size_t coarse = tot / (S * S);
        if (S == 1) {
            fld(net.X[0].p, nullptr, 0.f, tr.zj.p, 1.f, tr.dg.p, nullptr, N, plane, st);  // / D
        } else {
            fld(tr.z2.p, nullptr, 0.f, tr.zj.p, 1.f, tr.dg.p, nullptr, N, plane, st);
            pool_s_kernel<<<ew_grid(coarse), 256, 0, st>>>(tr.z2.p, N * 2, H, W, S, net.X[0].p, 1.f / (float)(S * S));
        }
        if ((e = net.gates(st)) != cudaSuccess) return e;
        if ((e = net.forward(st, true)) != cudaSuccess) return e;
        const float* yfine = net.Y.p;
        if (S > 1) {
            up_s_kernel<<<ew_grid(tot), 256, 0, st>>>(net.Y.p, N * 2, H / S, W / S, S, tr.yf.p);
            yfine = tr.yf.p;
        }
        fld(tr.z2.p, tr.z1.p, 1.f, yfine, 1.f, nullptr, tr.mask.p, N, plane, st);       // z2 = z1 + m Y
        patch_matvec_kernel<<<ew_grid(N * plane), 256, 0, st>>>(op, tr.z2.p, tr.tmp.p);
        fld(tr.dd.p, tr.r.p, 1.f, tr.tmp.p, -1.f, nullptr, nullptr, N, plane, st);      // r - A z2
        fld(tr.z.p, tr.z2.p, 1.f, tr.dd.p, om, tr.dg.p, nullptr, N, plane, st);         // z
        fld(tr.dd.p, tr.e.p, 1.f, tr.z.p, -1.f, nullptr, nullptr, N, plane, st);        // d = e - z
        patch_matvec_kernel<<<ew_grid(N * plane), 256, 0, st>>>(op, tr.dd.p, tr.ad.p);  // A d
        cudaMemsetAsync(tr.sums, 0, 2 * N * sizeof(double), st);
        const dim3 dg((unsigned)std::min<size_t>((per + 255) / 256, 64), (unsigned)N);
        sample_dot_kernel<<<dg, 256, 0, st>>>(tr.dd.p, tr.ad.p, per, tr.sums);
        sample_dot_kernel<<<dg, 256, 0, st>>>(tr.e.p, tr.r.p, per, tr.sums + N);
        lpc_loss_kernel<<<1, 32, 0, st>>>(tr.sums, N, loss_slot);
        if (!grad) return cudaGetLastError();
        // dL/dz = -2 A d / (N E_n); through z = z2 + w (r - A z2) / D: dz2 = dz - w A (dz / D);
        // through z2 = z1 + m Y: dY = m dz2.
        loss_grad_kernel<<<ew_grid(tot), 256, 0, st>>>(tr.ad.p, tr.sums + N, N, per, tr.gz.p);
        fld(tr.tmp.p, nullptr, 0.f, tr.gz.p, 1.f, tr.dg.p, nullptr, N, plane, st);
        patch_matvec_kernel<<<ew_grid(N * plane), 256, 0, st>>>(op, tr.tmp.p, tr.zj.p);
        fld(tr.gz2.p, tr.gz.p, 1.f, tr.zj.p, -om, nullptr, nullptr, N, plane, st);
        fld(tr.gz2.p, nullptr, 0.f, tr.gz2.p, 1.f, nullptr, tr.mask.p, N, plane, st);
        const float* dy = tr.gz2.p;
        if (S > 1) {  // through the nearest upsampling: block sums
            pool_s_kernel<<<ew_grid(coarse), 256, 0, st>>>(tr.gz2.p, N * 2, H, W, S, tr.dyc.p, 1.f);
            dy = tr.dyc.p;
        }
        cudaMemsetAsync(g.p, 0, g.n * sizeof(float), st);
        if ((e = net.backward(dy, nullptr, st)) != cudaSuccess) return e;
        return cudaGetLastError();
    }

    cudaError_t adam_step(float lr) {
        adam_t += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = (float)(1.0 / (1.0 - pow((double)b1, adam_t)));
        const float c2 = (float)(1.0 / (1.0 - pow((double)b2, adam_t)));
        adam_kernel<<<ew_grid(net.nparams), 256, 0, st>>>(w.p, wq.p, g.p, m.p, v.p, net.nparams, lr, b1, b2, c1, c2,
                                                          1e-8f, round_bf16);
        return cudaGetLastError();
    }

    // One step of training: a batch, the loss and its gradient, an Adam update.
    cudaError_t train_step(int N, int H, int W, float lr, double* loss_slot, float rough) {
        cudaError_t e;
        if ((e = sample_batch(N, H, W, rough)) != cudaSuccess) return e;
        if ((e = loss_grad(loss_slot, lr > 0.f)) != cudaSuccess) return e;
        return lr > 0.f ? adam_step(lr) : cudaSuccess;
    }
};

}  // namespace wcb
