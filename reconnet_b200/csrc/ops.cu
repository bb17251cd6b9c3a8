// Ramp filter, TV surrogate, OS-SQS update and the reference-named host
// entry points (synchronous, host pointers).
#include <cuda_runtime.h>
#include <limits.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <list>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "rn_internal.h"

namespace rn {

// PI as the reference defines it (ReconNet4D/Projector.h:5); the filter
// constants below use it so the ramp matches the reference's definition.
static const double kRefPi = 3.141592657;

// ---------------------------------------------------------------------------
// Ramp filter kernel h[0..2nu-2] (offset k = i - (nu-1)): the spatial-domain
// result of getRamp (Filter.cu:66-214): RL ramp (equiangular sin^2 or
// equispaced k^2 form), optionally windowed in the DFT domain
// (Hamming / Hann / cosine), transformed back, real part.
// ---------------------------------------------------------------------------
static std::vector<double> ramp_kernel(int nu, double da, int typeFilter, bool equispace) {
    const int L = 2 * nu - 1;
    std::vector<std::complex<double>> r(L);
    for (int i = 0; i < L; i++) {
        int k = i - (nu - 1);
        double v = 0;
        if (k == 0) v = 1.0 / (4 * da * da);
        else if (k % 2 != 0) {
            if (equispace) v = -1.0 / (kRefPi * kRefPi * (double)k * k * da * da);
            else {
                double s = std::sin(k * da);
                v = -1.0 / (kRefPi * kRefPi * s * s);
            }
        }
        r[i] = v;
    }
    if (typeFilter >= 1 && typeFilter <= 3) {
        // DFT with a twiddle table (exact index arithmetic mod L)
        std::vector<std::complex<double>> tw(L);
        for (int i = 0; i < L; i++) tw[i] = std::polar(1.0, -2.0 * M_PI * i / L);
        std::vector<std::complex<double>> F(L);
        for (int k = 0; k < L; k++) {
            std::complex<double> acc = 0;
            long long idx = 0;
            for (int j = 0; j < L; j++) {
                acc += r[j] * tw[idx];
                idx += k;
                if (idx >= L) idx -= L;
            }
            F[k] = acc;
        }
        for (int i = 0; i < L; i++) {
            double w;
            if (typeFilter == 1) w = 0.54 + 0.46 * std::cos(2 * kRefPi * i / (double)(L - 1));
            else if (typeFilter == 2) w = 0.5 + 0.5 * std::cos(2 * kRefPi * i / (double)(L - 1));
            else w = std::fabs(std::cos(kRefPi * i / (double)(L - 1)));
            F[i] *= w;
        }
        for (int j = 0; j < L; j++) {
            std::complex<double> acc = 0;
            long long idx = 0;
            for (int k = 0; k < L; k++) {
                acc += F[k] * std::conj(tw[idx]);
                idx += j;
                if (idx >= L) idx -= L;
            }
            r[j] = acc / (double)L;
        }
    }
    std::vector<double> h(L);
    for (int i = 0; i < L; i++) h[i] = r[i].real();
    return h;
}

// Device copy of the filter kernel, cached per (device, nu, da, type, geometry).
struct FilterKey {
    int dev, nu, type, fan;
    float da, off_a;
    bool operator<(const FilterKey& o) const {
        return std::tie(dev, nu, type, fan, da, off_a) < std::tie(o.dev, o.nu, o.type, o.fan, o.da, o.off_a);
    }
};
struct FilterVal {
    float* d_h = nullptr;   // [2nu-1]
    float* d_pw = nullptr;  // [nu] pre-weights
    // FFT form (0 = direct convolution only): transform length N = 2^logN >=
    // 2nu - 1, the kernel's spectrum (scaled by 1/N) and the twiddles
    int logN = 0;
    float2* d_H = nullptr;  // [N]
    float2* d_tw = nullptr; // [N/2] exp(-2 pi i q / N)
    // register four-step form (N = 512, 1024, 2048, run as two transforms of
    // M = N/2 points): the even- and odd-frequency halves of the spectrum in
    // the registers' order, [2][M/32][32] (entry [half][r][lane]; at M = 1024
    // in the order of the transposing kernel); then the
    // M-point middle twiddles [M/32][32] followed by the odd half's
    // pre-twiddles exp(-2 pi i n / N), n = lane + 32 r < M
    float2* d_Hp = nullptr;
    float2* d_Tw = nullptr;
};

// In-place radix-2 FFT in FP64 (host; the filter spectrum).
static void fft64(std::vector<std::complex<double>>& a) {
    const size_t n = a.size();
    for (size_t i = 1, j = 0; i < n; i++) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1)
        for (size_t i = 0; i < n; i += len)
            for (size_t j = 0; j < len / 2; j++) {
                const std::complex<double> w = std::polar(1.0, -2.0 * M_PI * (double)j / (double)len);
                const std::complex<double> u = a[i + j], v = a[i + j + len / 2] * w;
                a[i + j] = u + v;
                a[i + j + len / 2] = u - v;
            }
}

// Largest transform the FFT filter stages in shared memory (one signal).
constexpr int kFilterMaxLogN = 14;
static std::mutex g_filter_mu;
static std::map<FilterKey, FilterVal> g_filters;

static int get_filter(int nu, float da, float off_a, int typeFilter, int fan, cudaStream_t st, FilterVal& out) {
    int dev = 0;
    cudaGetDevice(&dev);
    FilterKey key{dev, nu, typeFilter, fan, da, off_a};
    std::lock_guard<std::mutex> lk(g_filter_mu);
    auto it = g_filters.find(key);
    if (it != g_filters.end()) {
        out = it->second;
        return RN_OK;
    }
    std::vector<double> h = ramp_kernel(nu, da, typeFilter, !fan);
    std::vector<float> hf(h.begin(), h.end());
    std::vector<float> pw(nu, 1.f);
    if (fan)
        for (int i = 0; i < nu; i++) pw[i] = (float)std::cos(((i - (nu - 1) / 2.0) - off_a) * (double)da);
    FilterVal v;
    RN_CUDA_TRY(cudaMalloc(&v.d_h, sizeof(float) * hf.size()));
    RN_CUDA_TRY(cudaMalloc(&v.d_pw, sizeof(float) * nu));
    RN_CUDA_TRY(cudaMemcpyAsync(v.d_h, hf.data(), sizeof(float) * hf.size(), cudaMemcpyHostToDevice, st));
    RN_CUDA_TRY(cudaMemcpyAsync(v.d_pw, pw.data(), sizeof(float) * nu, cudaMemcpyHostToDevice, st));
    // FFT form: the kernel placed circularly (offset k = i - (nu-1) at index
    // k mod N), transformed in FP64; the circular convolution of length N >=
    // 2nu - 1 equals the linear one on outputs 0 .. nu-1
    int logN = 1;
    while ((1 << logN) < 2 * nu - 1) logN++;
    std::vector<float2> Hf, twf;
    if (logN <= kFilterMaxLogN) {
        const int N = 1 << logN;
        std::vector<std::complex<double>> hc(N, 0.0);
        for (int i = 0; i < 2 * nu - 1; i++) hc[((i - (nu - 1)) % N + N) % N] += h[i];
        fft64(hc);
        Hf.resize(N);
        for (int f = 0; f < N; f++) Hf[f] = make_float2((float)(hc[f].real() / N), (float)(hc[f].imag() / N));
        twf.resize(N / 2);
        for (int q = 0; q < N / 2; q++) {
            const std::complex<double> w = std::polar(1.0, -2.0 * M_PI * (double)q / (double)N);
            twf[q] = make_float2((float)w.real(), (float)w.imag());
        }
        v.logN = logN;
        if (N >= 512 && N <= 2048) {
            // the signal occupies n < nu <= M = N/2, so the N-point spectrum
            // splits into X[2k] = FFT_M(x)[k] and X[2k+1] = FFT_M(x
            // exp(-2 pi i n / N))[k].  Lane l, register r of the M-point
            // four-step transform holds frequency bitrev(r) + (M/32) bitrev5(l)
            // after the forward pass; its middle twiddle is
            // exp(-2 pi i l bitrev(r) / M)
            const int M = N / 2, L = M / 32, bits = logN - 6;
            auto brev = [](int x, int nb) {
                int r = 0;
                for (int i = 0; i < nb; i++) r = (r << 1) | ((x >> i) & 1);
                return r;
            };
            std::vector<float2> Hp((size_t)N), Tw((size_t)N);
            for (int r = 0; r < L; r++)
                for (int l = 0; l < 32; l++) {
                    const int k2 = brev(r, bits), k = k2 + L * brev(l, 5);
                    // at M = 1024 the transposing kernel holds frequency k2 +
                    // 32 k1 in lane bitrev5^-1(k2), register bitrev5^-1(k1)
                    const size_t at = M == 1024 ? (size_t)l * 32 + r : (size_t)r * 32 + l;
                    Hp[at] = Hf[2 * k];
                    Hp[(size_t)M + at] = Hf[2 * k + 1];
                    const std::complex<double> w = std::polar(1.0, -2.0 * M_PI * (double)(l * k2) / (double)M);
                    Tw[(size_t)r * 32 + l] = make_float2((float)w.real(), (float)w.imag());
                    const std::complex<double> q = std::polar(1.0, -2.0 * M_PI * (double)(l + 32 * r) / (double)N);
                    Tw[(size_t)M + r * 32 + l] = make_float2((float)q.real(), (float)q.imag());
                }
            RN_CUDA_TRY(cudaMalloc(&v.d_Hp, sizeof(float2) * N));
            RN_CUDA_TRY(cudaMalloc(&v.d_Tw, sizeof(float2) * N));
            RN_CUDA_TRY(cudaMemcpyAsync(v.d_Hp, Hp.data(), sizeof(float2) * N, cudaMemcpyHostToDevice, st));
            RN_CUDA_TRY(cudaMemcpyAsync(v.d_Tw, Tw.data(), sizeof(float2) * N, cudaMemcpyHostToDevice, st));
        }
        RN_CUDA_TRY(cudaMalloc(&v.d_H, sizeof(float2) * N));
        RN_CUDA_TRY(cudaMalloc(&v.d_tw, sizeof(float2) * (N / 2)));
        RN_CUDA_TRY(cudaMemcpyAsync(v.d_H, Hf.data(), sizeof(float2) * N, cudaMemcpyHostToDevice, st));
        RN_CUDA_TRY(cudaMemcpyAsync(v.d_tw, twf.data(), sizeof(float2) * (N / 2), cudaMemcpyHostToDevice, st));
    }
    RN_CUDA_TRY(cudaStreamSynchronize(st));
    g_filters[key] = v;
    out = v;
    return RN_OK;
}

// Toeplitz product per sinogram plane: out[view][iu] = scale * sum_j
// (prj[view][j] * pw[j]) * h[nu-1+iu-j].  CTA tile 64 views x 64 outputs,
// 4x4 per thread, inputs staged 32 at a time in shared memory.
__global__ void __launch_bounds__(256) filter_kernel(float* __restrict__ out, const float* __restrict__ prj,
                                                     const float* __restrict__ h, const float* __restrict__ pw,
                                                     const float* __restrict__ sw, int nu, int nview, int nv,
                                                     int nc, int nplane_total, float scale) {
    __shared__ float Xs[32][64 + 4];
    __shared__ float Hs[96];
    const int nplanes = nplane_total;
    for (int plane = blockIdx.z; plane < nplanes; plane += gridDim.z) {
    const int b = plane / (nv * nc);
    const int rem = plane - b * nv * nc;
    const long long off = (long long)b * nu * nview * nv * nc + rem;   // (iv, c) folded: rem = iv*nc + c
    const long long su = (long long)nview * nv * nc, sview = (long long)nv * nc;
    const int v0 = blockIdx.x * 64, i0 = blockIdx.y * 64;
    const int tid = threadIdx.x;
    const int tv = tid & 15, to = tid >> 4;
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[a][c] = 0.f;
    for (int j0 = 0; j0 < nu; j0 += 32) {
        for (int e = tid; e < 32 * 64; e += 256) {
            int jj = e >> 6, vv = e & 63;
            int j = j0 + jj, v = v0 + vv;
            float x = 0.f;
            if (j < nu && v < nview) {
                x = prj[off + (long long)j * su + (long long)v * sview] * pw[j];
                if (sw) x *= sw[(long long)j * nview + v];
            }
            Xs[jj][vv] = x;
        }
        if (tid < 96) {
            int k = nu - 1 + i0 - j0 + tid - 31;
            Hs[tid] = (k >= 0 && k <= 2 * nu - 2) ? h[k] : 0.f;
        }
        __syncthreads();
#pragma unroll 8
        for (int jj = 0; jj < 32; jj++) {
            float4 xv = *reinterpret_cast<const float4*>(&Xs[jj][tv * 4]);
            float hv[4];
#pragma unroll
            for (int c = 0; c < 4; c++) hv[c] = Hs[to * 4 + c - jj + 31];
            float xa[4] = {xv.x, xv.y, xv.z, xv.w};
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[a][c] = fmaf(xa[a], hv[c], acc[a][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
            int v = v0 + tv * 4 + a, i = i0 + to * 4 + c;
            if (v < nview && i < nu) out[off + (long long)i * su + (long long)v * sview] = acc[a][c] * scale;
        }
    __syncthreads();   // the next plane refills Xs / Hs
    }
}

// FFT filter: the same product as filter_kernel as a circular convolution of
// length N = 2^logN >= 2nu - 1.  A CTA holds S complex signals in shared
// memory, each carrying two views (real and imaginary parts: the kernel is
// real, so their convolutions separate again); views run along the threads
// for the loads and stores.  Pre-weighted samples go to bit-reversed
// positions, a radix-2 decimation-in-time pass gives the spectrum in natural
// order, the product with the kernel's spectrum (which carries 1/N) is taken
// in its last pass, and a decimation-in-frequency pass with conjugate
// twiddles returns the outputs in bit-reversed order, scaled on the way out.  N / 2 log2(N) butterflies per
// view pair instead of nu^2 multiply-adds per view.
constexpr int kFftThreads = 512;

__device__ __forceinline__ float2 c_mul(float2 a, float2 w) {
    return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}
__device__ __forceinline__ float2 c_mulc(float2 a, float2 w) {   // a * conj(w)
    return make_float2(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
}
__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// Radix-2 levels s .. s + T - 1 of every signal in one pass over groups of
// 2^T elements held in registers: decimation in time (levels ascending) or,
// kInv, decimation in frequency with conjugate twiddles (levels descending).
// The arithmetic is that of T separate radix-2 passes.  kMul (the last
// forward pass, whose outputs are in natural order): multiply by H on the
// way out.
template <int T, bool kInv, bool kMul = false>
__device__ __forceinline__ void fft_pass(float2* zs, const float2* tws, int Np, int S, int logN, int s,
                                         const float2* __restrict__ H = nullptr) {
    constexpr int R = 1 << T;
    const int h = 1 << s, groups = (1 << logN) >> T;
    for (int gb = threadIdx.x; gb < S * groups; gb += blockDim.x) {
        const int p = gb >> (logN - T), gi = gb & (groups - 1);
        const int j = gi & (h - 1), k = ((gi >> s) << (s + T)) + j;
        float2* z = zs + p * Np + k;
        float2 a[R];
#pragma unroll
        for (int m = 0; m < R; m++) a[m] = z[m * h];
#pragma unroll
        for (int tt = 0; tt < T; tt++) {
            const int t = kInv ? T - 1 - tt : tt;
            const int st = 1 << t;
#pragma unroll
            for (int m = 0; m < R; m++) {
                if (m & st) continue;
                const float2 w = tws[(j + (m & (st - 1)) * h) << (logN - 1 - s - t)];
                if (!kInv) {
                    const float2 x = c_mul(a[m + st], w);
                    a[m + st] = c_sub(a[m], x);
                    a[m] = c_add(a[m], x);
                } else {
                    const float2 u = a[m], v = a[m + st];
                    a[m] = c_add(u, v);
                    a[m + st] = c_mulc(c_sub(u, v), w);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < R; m++) z[m * h] = kMul ? c_mul(a[m], __ldg(H + k + m * h)) : a[m];
    }
}

__global__ void __launch_bounds__(kFftThreads, 2) filter_fft_kernel(float* __restrict__ out, const float* __restrict__ prj,
                                                         const float2* __restrict__ H, const float2* __restrict__ tw,
                                                         const float* __restrict__ pw, const float* __restrict__ sw,
                                                         int nu, int nview, int nv, int nc, int nplane_total, int logN,
                                                         int S, float scale) {
    extern __shared__ float2 zs[];   // S signals, stride N + 1 (one pad entry against bank conflicts), then the twiddles
    const int N = 1 << logN, Np = N + 1, halfN = N >> 1;
    float2* tws = zs + S * Np;
    for (int q = threadIdx.x; q < halfN; q += blockDim.x) tws[q] = __ldg(tw + q);
    const int nplanes = nplane_total;
    for (int plane = blockIdx.y; plane < nplanes; plane += gridDim.y) {
    const int b = plane / (nv * nc);
    const int rem = plane - b * nv * nc;
    const long long off = (long long)b * nu * nview * nv * nc + rem;
    const long long su = (long long)nview * nv * nc, sview = (long long)nv * nc;
    const int v0 = blockIdx.x * 2 * S;
    const int tid = threadIdx.x;
    for (int e = tid; e < S * N; e += blockDim.x) {
        const int p = e % S, n = e / S;
        float a = 0.f, c = 0.f;
        if (n < nu) {
            const int va = v0 + 2 * p;
            const float w = pw[n];
            const float* src = prj + off + (long long)n * su;
            if (va < nview) a = src[(long long)va * sview] * w;
            if (va + 1 < nview) c = src[(long long)(va + 1) * sview] * w;
            if (sw) {   // short-scan weights [nu][nview]
                const float* wr = sw + (long long)n * nview;
                if (va < nview) a *= wr[va];
                if (va + 1 < nview) c *= wr[va + 1];
            }
        }
        zs[p * Np + (int)(__brev((unsigned)n) >> (32 - logN))] = make_float2(a, c);
    }
    __syncthreads();
    // decimation in time: radix-2 levels fused three at a time (then two or
    // one for the remainder), ascending
    // (the last pass also multiplies by the kernel's spectrum)
    int s = 0;
    for (; s + 2 < logN; s += 3) {
        if (s + 3 == logN) fft_pass<3, false, true>(zs, tws, Np, S, logN, s, H);
        else fft_pass<3, false>(zs, tws, Np, S, logN, s);
        __syncthreads();
    }
    if (s + 1 < logN) {
        if (s + 2 == logN) fft_pass<2, false, true>(zs, tws, Np, S, logN, s, H);
        else fft_pass<2, false>(zs, tws, Np, S, logN, s);
        __syncthreads();
        s += 2;
    }
    if (s < logN) {
        fft_pass<1, false, true>(zs, tws, Np, S, logN, s, H);
        __syncthreads();
    }
    // decimation in frequency with conjugate twiddles (the inverse): three
    // levels per pass from the top, then the remaining two or one
    for (s = logN - 3; s >= 0; s -= 3) {
        fft_pass<3, true>(zs, tws, Np, S, logN, s);
        __syncthreads();
    }
    if (s + 3 == 2) {
        fft_pass<2, true>(zs, tws, Np, S, logN, 0);
        __syncthreads();
    } else if (s + 3 == 1) {
        fft_pass<1, true>(zs, tws, Np, S, logN, 0);
        __syncthreads();
    }
    for (int e = tid; e < S * nu; e += blockDim.x) {
        const int p = e % S, n = e / S;
        const float2 r = zs[p * Np + (int)(__brev((unsigned)n) >> (32 - logN))];
        const int va = v0 + 2 * p;
        float* dst = out + off + (long long)n * su;
        if (va < nview) dst[(long long)va * sview] = r.x * scale;
        if (va + 1 < nview) dst[(long long)(va + 1) * sview] = r.y * scale;
    }
    __syncthreads();   // the next plane reuses the signal buffers
    }
}

// Register four-step FFT filter.  The zero-padded signal of N points (N =
// 512, 1024, 2048) is nonzero on its first half only, so its spectrum is two
// M = N/2 point transforms: the even frequencies are FFT_M(x) and the odd ones
// FFT_M(x w), w = exp(-2 pi i n / N).  Each is filtered by its half of the
// kernel's spectrum and inverted, and the outputs (needed for n < nu <= M
// only) are y = y_even + conj(w) y_odd.  A warp runs both halves in turn on
// one complex signal (two views as real and imaginary parts), element n =
// lane + 32 r in register r of its lane (M = 32 L).  An M-point transform:
// an L-point decimation-in-frequency transform in each lane's registers, the
// middle twiddles exp(-2 pi i lane k2 / M), and a 32-point
// decimation-in-frequency transform across the lanes by shuffles; the
// spectrum then sits in bit-reversed order in both indices, where it is
// multiplied by the kernel's spectrum stored in that order.  The inverse runs
// the same steps backwards (decimation in time, conjugate twiddles) and
// returns the signal in its original registers.  No shared-memory passes: a
// CTA stages 16 views of its sinogram plane through shared memory only to
// load and store them coalesced.
constexpr int kRegViews = 16;   // views per CTA (8 warps, two views each)

template <int L>
struct RegFftTw {
    float2 local[L / 2];   // exp(-2 pi i k / L), k < L/2
    float2 w32[16];        // exp(-2 pi i k / 32), k < 16
};

template <int L>
__device__ __forceinline__ void reg_local_dif(float2 (&v)[L], const RegFftTw<L>& t) {
#pragma unroll
    for (int h = L / 2; h >= 1; h >>= 1) {
#pragma unroll
        for (int i = 0; i < L; i++) {
            if (i & h) continue;
            const float2 a = v[i], b = v[i + h];
            v[i] = c_add(a, b);
            const int k = (i & (h - 1)) * (L / (2 * h));
            const float2 d = c_sub(a, b);
            // exp(-2 pi i k / L): 1 at k = 0, -i at k = L/4
            v[i + h] = k == 0 ? d : 4 * k == L ? make_float2(d.y, -d.x) : c_mul(d, t.local[k]);
        }
    }
}

template <int L>
__device__ __forceinline__ void reg_local_dit_inv(float2 (&v)[L], const RegFftTw<L>& t) {
#pragma unroll
    for (int h = 1; h < L; h <<= 1) {
#pragma unroll
        for (int i = 0; i < L; i++) {
            if (i & h) continue;
            const int k = (i & (h - 1)) * (L / (2 * h));
            const float2 c = v[i + h];
            const float2 a = v[i], b = k == 0 ? c : 4 * k == L ? make_float2(-c.y, c.x) : c_mulc(c, t.local[k]);
            v[i] = c_add(a, b);
            v[i + h] = c_sub(a, b);
        }
    }
}

__device__ __forceinline__ float2 shfl_xor2(float2 a, int m) {
    return make_float2(__shfl_xor_sync(0xffffffffu, a.x, m), __shfl_xor_sync(0xffffffffu, a.y, m));
}

// Tiles of 16 views x nu channels of one sinogram plane pass through shared
// memory so that global loads and stores stay coalesced.  The kernels are
// persistent: a CTA walks work items (plane, block of 16 views) with a stride
// of the grid, and while it transforms one item the next item's tile arrives
// by cp.async (4-byte copies, zero-filled beyond the last view) in the other
// of two tile buffers, so the load latency is hidden behind the arithmetic.
__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(valid ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

struct FiltTiles {
    const float* prj;
    float* out;
    const float* pw;
    const float* sw;
    int nu, nview, nvb;      // nvb: view blocks per plane
    long long su, sview, plane_elems;
    int nv, nc;
};

// element offset of work item `it` (plane it / nvb, first view 16 (it % nvb))
__device__ __forceinline__ long long filt_item(const FiltTiles& f, long long it, int& v0) {
    const long long plane = it / f.nvb;
    v0 = (int)(it - plane * f.nvb) * kRegViews;
    const long long b = plane / ((long long)f.nv * f.nc), rem = plane - b * f.nv * f.nc;
    return b * f.plane_elems + rem;
}

__device__ __forceinline__ void filt_issue(const FiltTiles& f, float* tile, long long it) {
    constexpr int TS = kRegViews + 1;
    int v0;
    const long long off = filt_item(f, it, v0);
#pragma unroll 4
    for (int e = threadIdx.x; e < f.nu * kRegViews; e += blockDim.x) {
        const int n = e / kRegViews, vv = e - n * kRegViews, view = v0 + vv;
        const bool ok = view < f.nview;
        cp_async4(tile + n * TS + vv, ok ? f.prj + off + (long long)n * f.su + (long long)view * f.sview : f.prj, ok);
    }
}

__device__ __forceinline__ void filt_store(const FiltTiles& f, const float* tile, long long it) {
    constexpr int TS = kRegViews + 1;
    int v0;
    const long long off = filt_item(f, it, v0);
#pragma unroll 4
    for (int e = threadIdx.x; e < f.nu * kRegViews; e += blockDim.x) {
        const int n = e / kRegViews, vv = e - n * kRegViews, view = v0 + vv;
        if (view < f.nview) f.out[off + (long long)n * f.su + (long long)view * f.sview] = tile[n * TS + vv];
    }
}

// channel n of this warp's two views (columns 2 warp, 2 warp + 1 of the tile),
// pre-weighted (and short-scan weighted) as the filter's input
__device__ __forceinline__ float2 filt_input(const FiltTiles& f, const float* tile, int n, int warp, int v0) {
    constexpr int TS = kRegViews + 1;
    const float p = __ldg(f.pw + n);
    float a = tile[n * TS + 2 * warp] * p, b = tile[n * TS + 2 * warp + 1] * p;
    if (f.sw) {
        const int va = v0 + 2 * warp;
        a *= va < f.nview ? __ldg(f.sw + (long long)n * f.nview + va) : 0.f;
        b *= va + 1 < f.nview ? __ldg(f.sw + (long long)n * f.nview + va + 1) : 0.f;
    }
    return make_float2(a, b);
}

// Per work item, each warp transforms one complex signal (its two views)
// through both halves.  The even half's output y0 is parked in the tile in
// place of the input, which the odd half no longer needs once it has read it.
template <int L>
__global__ void __launch_bounds__(256, 1) filter_reg_kernel(FiltTiles f, const float2* __restrict__ Hp,
                                                           const float2* __restrict__ Tw, long long nitems,
                                                           float scale, RegFftTw<L> tw) {
    extern __shared__ float tiles[];           // two tiles of [nu][kRegViews + 1]
    constexpr int TS = kRegViews + 1, M = 32 * L;
    const float2* __restrict__ Pre = Tw + M;   // exp(-2 pi i n / N), n < M
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile_floats = (f.nu * TS + 1) & ~1;
    const int nu = f.nu;
    // this lane's twiddle in each cross-lane stage: exp(-2 pi i (lane mod h) / 2h)
    float2 wl[5];
#pragma unroll
    for (int s = 0; s < 5; s++) {
        const int h = 1 << s;
        wl[s] = tw.w32[(lane & (h - 1)) * (16 / h)];
    }
    auto forward = [&](float2 (&v)[L], int half) {
        reg_local_dif<L>(v, tw);
#pragma unroll
        for (int r = 0; r < L; r++) v[r] = c_mul(v[r], __ldg(Tw + r * 32 + lane));
#pragma unroll
        for (int s = 4; s >= 0; s--) {
            const int h = 1 << s;
            const bool up = (lane & h) != 0;
#pragma unroll
            for (int r = 0; r < L; r++) {
                const float2 p = shfl_xor2(v[r], h);
                v[r] = up ? c_mul(c_sub(p, v[r]), wl[s]) : c_add(v[r], p);
            }
        }
        // this half of the kernel's spectrum (scaled by 1/N), then the inverse
#pragma unroll
        for (int r = 0; r < L; r++) v[r] = c_mul(v[r], __ldg(Hp + half * M + r * 32 + lane));
#pragma unroll
        for (int s = 0; s < 5; s++) {
            const int h = 1 << s;
            const bool up = (lane & h) != 0;
#pragma unroll
            for (int r = 0; r < L; r++) {
                const float2 t = up ? c_mulc(v[r], wl[s]) : v[r];
                const float2 p = shfl_xor2(t, h);
                v[r] = up ? c_sub(p, t) : c_add(v[r], p);
            }
        }
#pragma unroll
        for (int r = 0; r < L; r++) v[r] = c_mulc(v[r], __ldg(Tw + r * 32 + lane));
        reg_local_dit_inv<L>(v, tw);
    };
    long long it = blockIdx.x;
    if (it < nitems) filt_issue(f, tiles, it);
    cp_async_commit();
    for (int b = 0; it < nitems; it += gridDim.x, b ^= 1) {
        float* tile = tiles + b * tile_floats;
        if (it + gridDim.x < nitems) filt_issue(f, tiles + (b ^ 1) * tile_floats, it + gridDim.x);
        cp_async_commit();
        cp_async_wait_prev();
        __syncthreads();
        int v0;
        filt_item(f, it, v0);
        float2 v[L];
#pragma unroll
        for (int r = 0; r < L; r++) {
            const int n = lane + 32 * r;
            v[r] = n < nu ? filt_input(f, tile, n, warp, v0) : make_float2(0.f, 0.f);
        }
#pragma unroll 1
        for (int half = 0; half < 2; half++) {
            forward(v, half);
            if (half == 0) {
                // park y0 in the tile, take the odd half's input
#pragma unroll
                for (int r = 0; r < L; r++) {
                    const int n = lane + 32 * r;
                    if (n < nu) {
                        const float2 x = filt_input(f, tile, n, warp, v0);
                        tile[n * TS + 2 * warp] = v[r].x;
                        tile[n * TS + 2 * warp + 1] = v[r].y;
                        v[r] = c_mul(x, __ldg(Pre + r * 32 + lane));
                    } else {
                        v[r] = make_float2(0.f, 0.f);
                    }
                }
            } else {
#pragma unroll
                for (int r = 0; r < L; r++) {
                    const int n = lane + 32 * r;
                    if (n < nu) {
                        const float2 y0 = make_float2(tile[n * TS + 2 * warp], tile[n * TS + 2 * warp + 1]);
                        const float2 y = c_add(y0, c_mulc(v[r], __ldg(Pre + r * 32 + lane)));
                        tile[n * TS + 2 * warp] = y.x * scale;
                        tile[n * TS + 2 * warp + 1] = y.y * scale;
                    }
                }
            }
        }
        __syncthreads();
        filt_store(f, tile, it);
        __syncthreads();   // the item after next refills this tile
    }
}

// The N = 2048 case (M = 1024 = 32 x 32) with both 32-point stages in
// registers: lane l first transforms its 32 registers (n2 -> k2, register r
// holding k2 = bitrev(r)), applies the middle twiddle exp(-2 pi i l k2 / M),
// and the warp transposes the 32 x 32 block through shared memory, after which
// lane l holds row k2 = bitrev(l) and transforms n1 -> k1 in its registers
// (register c holding k1 = bitrev(c)); frequency k2 + 32 k1 then sits in lane
// l, register c.  The inverse runs the same steps backwards.  Two transposes
// (64 conflict-free shared-memory accesses per lane) replace ten cross-lane
// shuffle stages.
constexpr int kTrStride = 33;   // float2 row stride of a warp's transpose block

__global__ void __launch_bounds__(256, 1) filter_tr_kernel(FiltTiles f, const float2* __restrict__ Hq,
                                                          const float2* __restrict__ Tw, long long nitems,
                                                          float scale, RegFftTw<32> tw) {
    constexpr int L = 32, M = 1024, TS = kRegViews + 1;
    // two tiles of [nu][kRegViews + 1] floats, then [8 warps][32][33] float2
    // (the transpose blocks)
    extern __shared__ float tiles[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nu = f.nu;
    const float2* __restrict__ Pre = Tw + M;
    const int tile_floats = (nu * TS + 1) & ~1;
    float2* tr = reinterpret_cast<float2*>(tiles + 2 * tile_floats) + warp * (32 * kTrStride);
    auto forward = [&](float2 (&v)[L], int half) {
        reg_local_dif<L>(v, tw);
#pragma unroll
        for (int r = 0; r < L; r++) tr[r * kTrStride + lane] = c_mul(v[r], __ldg(Tw + r * 32 + lane));
        __syncwarp();
#pragma unroll
        for (int c = 0; c < L; c++) v[c] = tr[lane * kTrStride + c];
        reg_local_dif<L>(v, tw);
        // this half of the kernel's spectrum (scaled by 1/N), then the inverse
#pragma unroll
        for (int c = 0; c < L; c++) v[c] = c_mul(v[c], __ldg(Hq + half * M + c * 32 + lane));
        reg_local_dit_inv<L>(v, tw);
        __syncwarp();   // every lane has read its row of the block
#pragma unroll
        for (int c = 0; c < L; c++) tr[lane * kTrStride + c] = v[c];
        __syncwarp();
#pragma unroll
        for (int r = 0; r < L; r++) v[r] = c_mulc(tr[r * kTrStride + lane], __ldg(Tw + r * 32 + lane));
        reg_local_dit_inv<L>(v, tw);
        __syncwarp();   // the block is free for the next half
    };
    long long it = blockIdx.x;
    if (it < nitems) filt_issue(f, tiles, it);
    cp_async_commit();
    for (int b = 0; it < nitems; it += gridDim.x, b ^= 1) {
        float* tile = tiles + b * tile_floats;
        if (it + gridDim.x < nitems) filt_issue(f, tiles + (b ^ 1) * tile_floats, it + gridDim.x);
        cp_async_commit();
        cp_async_wait_prev();
        __syncthreads();
        int v0;
        filt_item(f, it, v0);
        float2 v[L];
#pragma unroll
        for (int r = 0; r < L; r++) {
            const int n = lane + 32 * r;
            v[r] = n < nu ? filt_input(f, tile, n, warp, v0) : make_float2(0.f, 0.f);
        }
#pragma unroll 1
        for (int half = 0; half < 2; half++) {
            forward(v, half);
            if (half == 0) {
                // park y0 in the tile, take the odd half's input
#pragma unroll
                for (int r = 0; r < L; r++) {
                    const int n = lane + 32 * r;
                    if (n < nu) {
                        const float2 x = filt_input(f, tile, n, warp, v0);
                        tile[n * TS + 2 * warp] = v[r].x;
                        tile[n * TS + 2 * warp + 1] = v[r].y;
                        v[r] = c_mul(x, __ldg(Pre + r * 32 + lane));
                    } else {
                        v[r] = make_float2(0.f, 0.f);
                    }
                }
            } else {
#pragma unroll
                for (int r = 0; r < L; r++) {
                    const int n = lane + 32 * r;
                    if (n < nu) {
                        const float2 y0 = make_float2(tile[n * TS + 2 * warp], tile[n * TS + 2 * warp + 1]);
                        const float2 y = c_add(y0, c_mulc(v[r], __ldg(Pre + r * 32 + lane)));
                        tile[n * TS + 2 * warp] = y.x * scale;
                        tile[n * TS + 2 * warp + 1] = y.y * scale;
                    }
                }
            }
        }
        __syncthreads();
        filt_store(f, tile, it);
        __syncthreads();   // the item after next refills this tile
    }
}

static int sm_count_cached() {
    static int sms[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && sms[dev] > 0) return sms[dev];
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    if (dev < 64) sms[dev] = n;
    return n;
}

static FiltTiles filt_tiles(float* d_out, const float* d_prj, const FilterVal& fv, const float* d_sw, int nu,
                            int nview, int nv, int nc) {
    FiltTiles f;
    f.prj = d_prj;
    f.out = d_out;
    f.pw = fv.d_pw;
    f.sw = d_sw;
    f.nu = nu;
    f.nview = nview;
    f.nvb = (nview + kRegViews - 1) / kRegViews;
    f.su = (long long)nview * nv * nc;
    f.sview = (long long)nv * nc;
    f.plane_elems = (long long)nu * nview * nv * nc;
    f.nv = nv;
    f.nc = nc;
    return f;
}

template <class K>
static int launch_persistent(K kernel, size_t smem, long long nitems, unsigned& grid) {
    RN_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    RN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem));
    if (per_sm <= 0) return set_error(RN_ERR_ARG, "filter: sinogram rows too long for shared memory");
    grid = (unsigned)std::min<long long>(nitems, (long long)per_sm * sm_count_cached());
    return RN_OK;
}

template <int L>
static int launch_filter_reg(float* d_out, const float* d_prj, const FilterVal& fv, const float* d_sw, int nu,
                             int nview, int nv, int nc, long long nplanes, float scale, cudaStream_t st) {
    RegFftTw<L> tw;
    for (int k = 0; k < L / 2; k++) {
        const std::complex<double> w = std::polar(1.0, -2.0 * M_PI * k / (double)L);
        tw.local[k] = make_float2((float)w.real(), (float)w.imag());
    }
    for (int k = 0; k < 16; k++) {
        const std::complex<double> w = std::polar(1.0, -2.0 * M_PI * k / 32.0);
        tw.w32[k] = make_float2((float)w.real(), (float)w.imag());
    }
    const FiltTiles f = filt_tiles(d_out, d_prj, fv, d_sw, nu, nview, nv, nc);
    const long long nitems = (long long)f.nvb * nplanes;
    const size_t smem = sizeof(float) * 2 * (((size_t)nu * (kRegViews + 1) + 1) & ~(size_t)1);
    unsigned grid = 0;
    RN_TRY(launch_persistent(filter_reg_kernel<L>, smem, nitems, grid));
    filter_reg_kernel<L><<<grid, 256, smem, st>>>(f, fv.d_Hp, fv.d_Tw, nitems, scale, tw);
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

static int launch_filter_tr(float* d_out, const float* d_prj, const FilterVal& fv, const float* d_sw, int nu,
                            int nview, int nv, int nc, long long nplanes, float scale, cudaStream_t st) {
    RegFftTw<32> tw;
    for (int k = 0; k < 16; k++) {
        const std::complex<double> w = std::polar(1.0, -2.0 * M_PI * k / 32.0);
        tw.local[k] = tw.w32[k] = make_float2((float)w.real(), (float)w.imag());
    }
    const FiltTiles f = filt_tiles(d_out, d_prj, fv, d_sw, nu, nview, nv, nc);
    const long long nitems = (long long)f.nvb * nplanes;
    const size_t smem = sizeof(float) * 2 * (((size_t)nu * (kRegViews + 1) + 1) & ~(size_t)1) +
                        sizeof(float2) * 8 * 32 * kTrStride;
    unsigned grid = 0;
    RN_TRY(launch_persistent(filter_tr_kernel, smem, nitems, grid));
    filter_tr_kernel<<<grid, 256, smem, st>>>(f, fv.d_Hp, fv.d_Tw, nitems, scale, tw);
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

// 0 = the register four-step kernel where it applies (the default), 1 = the
// shared-memory FFT kernel, 2 = the direct product (for comparisons)
static int g_filter_form = 0;

int filter_device(float* d_out, const float* d_prj, int nb, int nc, int nu, int nview, int nv, float da,
                  float off_a, float dsd, float dso, int typeFilter, int fan, cudaStream_t st,
                  const float* d_sw = nullptr) {
    (void)dsd;
    if (nb <= 0 || nc <= 0 || nu <= 0 || nview <= 0 || nv <= 0 || !(da > 0))
        return set_error(RN_ERR_ARG, "filter: sizes and pitch must be positive");
    if (d_out == d_prj) return set_error(RN_ERR_ARG, "filter: output must not alias input");
    FilterVal fv;
    RN_TRY(get_filter(nu, da, off_a, typeFilter, fan, st, fv));
    // scale of cFilterFan::Filter (Filter.cu:294-302) without the FFT length factor
    double scale = fan ? kRefPi / nview * da / dso : kRefPi / nview * da;
    // planes (batch, detector row, channel) beyond the 65,535 grid rows are
    // taken by the kernels' plane loops
    const long long nplanes = (long long)nb * nv * nc;
    if (nplanes > INT_MAX) return set_error(RN_ERR_ARG, "filter: too many sinogram planes");
    const unsigned grid_planes = (unsigned)std::min<long long>(nplanes, 65535);
    if (g_filter_form == 0 && fv.d_Hp) {
        const int N = 1 << fv.logN;
        if (N == 2048) return launch_filter_tr(d_out, d_prj, fv, d_sw, nu, nview, nv, nc, nplanes, (float)scale, st);
        if (N == 1024) return launch_filter_reg<16>(d_out, d_prj, fv, d_sw, nu, nview, nv, nc, nplanes, (float)scale, st);
        return launch_filter_reg<8>(d_out, d_prj, fv, d_sw, nu, nview, nv, nc, nplanes, (float)scale, st);
    }
    if (fv.logN > 0 && g_filter_form <= 1) {
        // S signals (2S views) per CTA: ~64 KB of shared memory at N = 2048
        const int N = 1 << fv.logN;
        const int S = std::max(1, std::min(16, 8192 / N));
        const size_t smem = sizeof(float2) * ((size_t)S * (N + 1) + N / 2);
        RN_CUDA_TRY(cudaFuncSetAttribute(filter_fft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        dim3 grid((unsigned)((nview + 2 * S - 1) / (2 * S)), grid_planes);
        filter_fft_kernel<<<grid, kFftThreads, smem, st>>>(d_out, d_prj, fv.d_H, fv.d_tw, fv.d_pw, d_sw, nu, nview, nv,
                                                           nc, (int)nplanes, fv.logN, S, (float)scale);
        RN_CUDA_TRY(cudaGetLastError());
        return RN_OK;
    }
    dim3 grid((nview + 63) / 64, (nu + 63) / 64, grid_planes);
    filter_kernel<<<grid, 256, 0, st>>>(d_out, d_prj, fv.d_h, fv.d_pw, d_sw, nu, nview, nv, nc, (int)nplanes,
                                        (float)scale);
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

// ---------------------------------------------------------------------------
// TV surrogate (TVSQSKernel, TotalVariation.cu:9-68) on planes of an image
// with strides (isx, isy); plane p at img + plane_off(p).  FP64 TV sums.
// ---------------------------------------------------------------------------
struct TvTerms {
    float grad, norm, var;
};

__device__ __forceinline__ TvTerms tv_terms(const float* __restrict__ img, int ix, int iy, int nx, int ny,
                                            long long isx, long long isy) {
    const float* p = img + ix * isx + iy * isy;
    float x = *p;
    float dx0 = ix == 0 ? x : x - p[-isx];
    float dx1 = ix == nx - 1 ? x : x - p[isx];
    float dy0 = iy == 0 ? x : x - p[-isy];
    float dy1 = iy == ny - 1 ? x : x - p[isy];
    const float eps = 1e-6f;
    float t0 = sqrtf(dx0 * dx0 + eps), t1 = sqrtf(dx1 * dx1 + eps);
    float t2 = sqrtf(dy0 * dy0 + eps), t3 = sqrtf(dy1 * dy1 + eps);
    // one correctly rounded reciprocal per difference instead of two divides
    const float r0 = __frcp_rn(t0), r1 = __frcp_rn(t1), r2 = __frcp_rn(t2), r3 = __frcp_rn(t3);
    TvTerms r;
    r.grad = (dx0 * r0 + dx1 * r1 + dy0 * r2 + dy1 * r3) / 2;
    r.norm = r0 + r1 + r2 + r3;
    r.var = (t0 + t1 + t2 + t3) / 2;
    return r;
}

__global__ void tv_kernel(float* grad, float* norm, double* tv, const float* __restrict__ img, int nx, int ny) {
    const int s = blockIdx.y;
    const long long base = (long long)s * nx * ny;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < nx * ny) {
        int ix = i / ny, iy = i - (i / ny) * ny;
        TvTerms t = tv_terms(img + base, ix, iy, nx, ny, ny, 1);
        if (grad) grad[base + i] = t.grad;
        if (norm) norm[base + i] = t.norm;
        v = (double)t.var;
    }
    if (tv) {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        __shared__ double ws[32];
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) ws[w] = v;
        __syncthreads();
        if (w == 0) {
            v = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) atomicAdd(&tv[s], v);
        }
    }
}

// r = (fp - prj) * w   (Minus2D + Multiply2D of ossqs.cu:106-122)
__global__ void residual_kernel(float* __restrict__ r, const float* __restrict__ prj, const float* __restrict__ w,
                                long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < n; i += stride) r[i] = (r[i] - prj[i]) * w[i];
}

// x_out = clamp(x_in - lam * (M*bp + beta*grad)/(norm + beta*norm_tv + 1e-6))
// (Divide2D / Minus2D / ValueCrop2D of ossqs.cu:135-146 plus the TV terms);
// image [B][nx][ny][nz][C], TV within each (b, z, c) plane.  Grid: x over the
// ny * nz * nc run of one image row, y = ix, z = b, so no thread divides a
// 64-bit index.
__global__ void sqs_update_kernel(float* __restrict__ xo, const float* __restrict__ xi, const float* __restrict__ bp,
                                  const float* __restrict__ nimg, int nx, int ny, int nzc, float lam, float beta,
                                  float M, float lb, float ub, int clamp) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ny * nzc) return;
    const int ix = blockIdx.y, bb = blockIdx.z;
    const long long isx = (long long)ny * nzc;
    const long long i = ((long long)bb * nx + ix) * isx + j;
    // numerator and denominator of the surrogate step in FP64
    double num = (double)M * bp[i];
    double den = (double)nimg[i] + 1e-6;
    if (beta != 0.f) {
        const int iy = nzc == 1 ? j : j / nzc;
        const int zc = j - iy * nzc;
        const float* plane = xi + (long long)bb * nx * isx + zc;
        TvTerms t = tv_terms(plane, ix, iy, nx, ny, isx, nzc);
        num += (double)beta * t.grad;
        den += (double)beta * t.norm;
    }
    float v = (float)((double)xi[i] - (double)lam * num / den);
    if (clamp) v = fminf(fmaxf(v, lb), ub);
    xo[i] = v;
}

int sqs_update(rn_fan_plan* p, float* x_out, const float* x_in, const float* prj_s, const float* w_s,
               const float* norm_img, float lam, float beta, int M, float lb, float ub, int type, cudaStream_t st) {
    if (!p || !x_out || !x_in || !prj_s || !w_s || !norm_img) return set_error(RN_ERR_ARG, "null argument");
    if (x_out == x_in) return set_error(RN_ERR_ARG, "sqs update: x_out must not alias x_in");
    {
        const RnFanGeom& g = p->g;
        const long long nzc = p->ragged ? 1 : (long long)g.nz * g.nChannels;
        if (g.nBatches > 65535 || (long long)g.ny * nzc >= (1LL << 31))
            return set_error(RN_ERR_ARG, "sqs update: more than 65535 batches, or an image row above 2^31 elements");
    }
    RN_TRY(fan_project(p, p->d_tmp_prj, x_in, st, type == RN_TYPE_SIDDON));
    long long n = p->prj_elems;
    residual_kernel<<<(unsigned)std::min<long long>((n + 255) / 256, 148 * 16), 256, 0, st>>>(p->d_tmp_prj, prj_s,
                                                                                               w_s, n);
    RN_CUDA_TRY(cudaGetLastError());
    RN_TRY(fan_backproject(p, p->d_tmp_img, p->d_tmp_prj, type, 0, st));
    const RnFanGeom& g = p->g;
    const int nzc = p->ragged ? 1 : g.nz * g.nChannels;
    const dim3 grid((unsigned)(((long long)g.ny * nzc + 255) / 256), (unsigned)g.nx, (unsigned)g.nBatches);
    sqs_update_kernel<<<grid, 256, 0, st>>>(x_out, x_in, p->d_tmp_img, norm_img, g.nx, g.ny, nzc, lam, beta, (float)M,
                                            lb, ub, lb < ub ? 1 : 0);
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

// ---------------------------------------------------------------------------
// Host-pointer (reference-named) entry points.
// ---------------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    int ensure(size_t bytes) {
        if (bytes <= n) return RN_OK;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) return set_cuda_error(e, "cudaMalloc");
        n = bytes;
        return RN_OK;
    }
    template <class T>
    T* as() {
        return reinterpret_cast<T*>(p);
    }
};

// Host arrays cross PCIe through a pinned staging buffer in chunks, so the
// host's copy of one chunk into (or out of) the staging buffer overlaps the
// DMA of another; pageable copies of the same arrays run at about half the
// rate (the driver stages them itself, one piece after the other).
constexpr int kStageChunksMax = 32;
constexpr size_t kStageChunkMin = (size_t)512 << 10;

// One cached plan and a set of grow-only device buffers per device, guarded
// by a mutex: repeated host calls with the same geometry and angles reuse the
// geometry tables and scratch instead of rebuilding them.
struct HostCtx {
    std::mutex mu;
    cudaStream_t st = nullptr;
    rn_fan_plan* plan = nullptr;    // the plan of the current call (owned by `cache`)
    // plans of recent (geometry, angles) pairs, most recent first: a caller
    // that cycles through the same slices (each with its own angles) finds
    // its plans here instead of rebuilding one per call
    struct Cached {
        RnFanGeom key;
        std::vector<float> deg;
        uint64_t hash;
        rn_fan_plan* plan;
    };
    std::list<Cached> cache;
    size_t cache_bytes = 0;
    DevBuf a, b, c, d, e;
    // pinned staging for the host arrays of a call, and one event per chunk
    void* pin = nullptr;
    size_t pin_n = 0;
    cudaEvent_t ev[kStageChunksMax] = {};
};
constexpr size_t kHostPlanCacheCount = 128;
constexpr size_t kHostPlanCacheBytes = (size_t)4 << 30;
static std::mutex g_ctx_mu;
static std::map<int, HostCtx*> g_ctx;

static HostCtx* host_ctx() {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    HostCtx*& c = g_ctx[dev];
    if (!c) {
        c = new HostCtx();
        cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    }
    return c;
}

static int stage_ensure(HostCtx* c, size_t bytes) {
    if (!c->ev[0])
        for (int k = 0; k < kStageChunksMax; k++)
            RN_CUDA_TRY(cudaEventCreateWithFlags(&c->ev[k], cudaEventDisableTiming));
    if (bytes <= c->pin_n) return RN_OK;
    if (c->pin) cudaFreeHost(c->pin);
    c->pin = nullptr;
    c->pin_n = 0;
    RN_CUDA_TRY(cudaHostAlloc(&c->pin, bytes, cudaHostAllocDefault));
    c->pin_n = bytes;
    return RN_OK;
}

static size_t stage_chunk(size_t bytes) {
    size_t ch = (bytes + kStageChunksMax - 1) / kStageChunksMax;
    ch = std::max(ch, kStageChunkMin);
    return (ch + 255) & ~(size_t)255;
}

// host -> device through the staging buffer: the host copies chunk k while
// the DMA of chunk k - 1 runs.  The staging buffer is free on entry (every
// call ends with its stream synchronised).
static int h2d_staged(HostCtx* c, void* dst, const void* src, size_t bytes) {
    RN_TRY(stage_ensure(c, bytes));
    const size_t ch = stage_chunk(bytes);
    for (size_t off = 0; off < bytes; off += ch) {
        const size_t n = std::min(ch, bytes - off);
        memcpy(static_cast<char*>(c->pin) + off, static_cast<const char*>(src) + off, n);
        RN_CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(dst) + off, static_cast<char*>(c->pin) + off, n,
                                    cudaMemcpyHostToDevice, c->st));
    }
    return RN_OK;
}

// device -> host: every chunk's DMA is queued behind the stream's work with an
// event after it; the host copies chunk k out as soon as its event completes,
// while the later chunks are still crossing.
static int d2h_staged(HostCtx* c, void* dst, const void* src, size_t bytes) {
    RN_TRY(stage_ensure(c, bytes));
    const size_t ch = stage_chunk(bytes);
    int k = 0;
    for (size_t off = 0; off < bytes; off += ch, k++) {
        const size_t n = std::min(ch, bytes - off);
        RN_CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(c->pin) + off, static_cast<const char*>(src) + off, n,
                                    cudaMemcpyDeviceToHost, c->st));
        RN_CUDA_TRY(cudaEventRecord(c->ev[k], c->st));
    }
    k = 0;
    for (size_t off = 0; off < bytes; off += ch, k++) {
        const size_t n = std::min(ch, bytes - off);
        RN_CUDA_TRY(cudaEventSynchronize(c->ev[k]));
        memcpy(static_cast<char*>(dst) + off, static_cast<char*>(c->pin) + off, n);
    }
    return RN_OK;
}

static uint64_t angle_hash(const RnFanGeom& g, const float* deg, int nview) {
    uint64_t h = 1469598103934665603ull;   // FNV-1a over the geometry and the angle bits
    auto mix = [&](const void* d, size_t n) {
        const unsigned char* q = static_cast<const unsigned char*>(d);
        for (size_t i = 0; i < n; i++) {
            h ^= q[i];
            h *= 1099511628211ull;
        }
    };
    mix(&g, sizeof(g));
    mix(deg, sizeof(float) * (size_t)nview);
    return h;
}

static int ctx_plan(HostCtx* c, const RnFanGeom& g, const float* deg, int nview) {
    const uint64_t h = angle_hash(g, deg, nview);
    for (auto it = c->cache.begin(); it != c->cache.end(); ++it) {
        if (it->hash == h && memcmp(&it->key, &g, sizeof(g)) == 0 && (int)it->deg.size() == nview &&
            memcmp(it->deg.data(), deg, sizeof(float) * nview) == 0) {
            c->cache.splice(c->cache.begin(), c->cache, it);   // most recently used first
            c->plan = it->plan;
            return RN_OK;
        }
    }
    rn_fan_plan* p = nullptr;
    RN_TRY(rn_fan_plan_create(&p, &g, deg, c->st));
    c->cache.push_front(HostCtx::Cached{g, std::vector<float>(deg, deg + nview), h, p});
    c->cache_bytes += p->arena_bytes;
    while (c->cache.size() > 1 && (c->cache.size() > kHostPlanCacheCount || c->cache_bytes > kHostPlanCacheBytes)) {
        c->cache_bytes -= c->cache.back().plan->arena_bytes;
        rn_fan_plan_destroy(c->cache.back().plan);
        c->cache.pop_back();
    }
    c->plan = p;
    return RN_OK;
}

static RnFanGeom fan_geom(int nb, int nc, int nx, int ny, int nz, float dx, float dy, float dz, int nu, int nview,
                          int nv, float da, float dv, float off_a, float off_v, float dsd, float dso) {
    RnFanGeom g;
    memset(&g, 0, sizeof(g));
    g.nBatches = nb;
    g.nChannels = nc;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.dx = dx;
    g.dy = dy;
    g.dz = dz;
    g.nu = nu;
    g.nview = nview;
    g.nv = nv;
    g.du = da;
    g.dv = dv;
    g.off_u = off_a;
    g.off_v = off_v;
    g.dsd = dsd;
    g.dso = dso;
    return g;
}

static int finish_sync(HostCtx* c, rn_fan_plan* p) {
    RN_CUDA_TRY(cudaStreamSynchronize(c->st));
    if (p) RN_TRY(rn_fan_plan_check(p, c->st));
    return RN_OK;
}

static int host_fan_fp(float* prj, const float* img, const float* deg, const RnFanGeom& g, bool siddon = false) {
    HostCtx* c = host_ctx();
    std::lock_guard<std::mutex> lk(c->mu);
    RN_TRY(ctx_plan(c, g, deg, g.nview));
    size_t ni = (size_t)c->plan->img_elems, np = (size_t)c->plan->prj_elems;
    RN_TRY(c->a.ensure(ni * 4));
    RN_TRY(c->b.ensure(np * 4));
    RN_TRY(h2d_staged(c, c->a.p, img, ni * 4));
    RN_TRY(fan_project(c->plan, c->b.as<float>(), c->a.as<float>(), c->st, siddon));
    RN_TRY(d2h_staged(c, prj, c->b.p, np * 4));
    return finish_sync(c, c->plan);
}

static int host_fan_bp(float* img, const float* prj, const float* deg, const RnFanGeom& g, int type) {
    HostCtx* c = host_ctx();
    std::lock_guard<std::mutex> lk(c->mu);
    RN_TRY(ctx_plan(c, g, deg, g.nview));
    size_t ni = (size_t)c->plan->img_elems, np = (size_t)c->plan->prj_elems;
    RN_TRY(c->a.ensure(ni * 4));
    RN_TRY(c->b.ensure(np * 4));
    RN_TRY(h2d_staged(c, c->b.p, prj, np * 4));
    RN_TRY(fan_backproject(c->plan, c->a.as<float>(), c->b.as<float>(), type, 0, c->st));
    RN_TRY(d2h_staged(c, img, c->a.p, ni * 4));
    return finish_sync(c, c->plan);
}

}  // namespace rn

using namespace rn;

extern "C" {

int SetDevice(int device) { return (int)cudaSetDevice(device); }

void cDistanceDrivenFanProjection(float* prj, const float* img, const float* deg, int nBatches, int nChannels, int nx,
                                  int ny, int nz, float dx, float dy, float dz, int nu, int nview, int nv, float da,
                                  float dv, float off_a, float off_v, float dsd, float dso, int typeProjector) {
    (void)typeProjector;
    clear_error();
    if (!prj || !img || !deg) {
        set_error(RN_ERR_ARG, "null argument");
        return;
    }
    host_fan_fp(prj, img, deg, fan_geom(nBatches, nChannels, nx, ny, nz, dx, dy, dz, nu, nview, nv, da, dv, off_a,
                                        off_v, dsd, dso));
}

void cSiddonFanProjection(float* prj, const float* img, const float* deg, int nBatches, int nChannels, int nx, int ny,
                          int nz, float dx, float dy, float dz, int nu, int nview, int nv, float da, float dv,
                          float off_a, float off_v, float dsd, float dso, int typeProjector) {
    (void)typeProjector;
    clear_error();
    if (!prj || !img || !deg) {
        set_error(RN_ERR_ARG, "null argument");
        return;
    }
    host_fan_fp(prj, img, deg,
                fan_geom(nBatches, nChannels, nx, ny, nz, dx, dy, dz, nu, nview, nv, da, dv, off_a, off_v, dsd, dso),
                true);
}

void cSiddonFanBackprojection(float* img, const float* prj, const float* deg, int nBatches, int nChannels, int nx,
                              int ny, int nz, float dx, float dy, float dz, int nu, int nview, int nv, float da,
                              float dv, float off_a, float off_v, float dsd, float dso, int typeProjector) {
    (void)typeProjector;
    clear_error();
    if (!prj || !img || !deg) {
        set_error(RN_ERR_ARG, "null argument");
        return;
    }
    host_fan_bp(img, prj, deg,
                fan_geom(nBatches, nChannels, nx, ny, nz, dx, dy, dz, nu, nview, nv, da, dv, off_a, off_v, dsd, dso),
                RN_TYPE_SIDDON);
}

// PixelDriven.cu:73-141: pixel-driven FBP backprojection (typeProjector is
// ignored there: cPixelDrivenFan always runs the FBP weight); the output is
// overwritten.
void cPixelDrivenFanBackprojection(float* img, const float* prj, const float* deg, int nBatches, int nChannels, int nx,
                                   int ny, int nz, float dx, float dy, float dz, int nu, int nview, int nv, float da,
                                   float dv, float off_a, float off_v, float dsd, float dso, int typeProjector) {
    (void)typeProjector;
    clear_error();
    if (!prj || !img || !deg) {
        set_error(RN_ERR_ARG, "null argument");
        return;
    }
    host_fan_bp(img, prj, deg,
                fan_geom(nBatches, nChannels, nx, ny, nz, dx, dy, dz, nu, nview, nv, da, dv, off_a, off_v, dsd, dso),
                RN_TYPE_PIXEL);
}

void cDistanceDrivenFanBackprojection(float* img, const float* prj, const float* deg, int nBatches, int nChannels,
                                      int nx, int ny, int nz, float dx, float dy, float dz, int nu, int nview, int nv,
                                      float da, float dv, float off_a, float off_v, float dsd, float dso,
                                      int typeProjector) {
    clear_error();
    if (typeProjector < 0 || typeProjector > 3) typeProjector = 0;   // the reference treats any non-1 type as iterative
    if (!prj || !img || !deg) {
        set_error(RN_ERR_ARG, "null argument");
        return;
    }
    host_fan_bp(img, prj, deg,
                fan_geom(nBatches, nChannels, nx, ny, nz, dx, dy, dz, nu, nview, nv, da, dv, off_a, off_v, dsd, dso),
                typeProjector);
}

int rn_filter(float* d_out, const float* d_prj, int nBatches, int nChannels, int nu, int nview, int nv, float da,
              float off_a, float dsd, float dso, int typeFilter, int fan, void* stream) {
    clear_error();
    if (!d_out || !d_prj) return set_error(RN_ERR_ARG, "null argument");
    return filter_device(d_out, d_prj, nBatches, nChannels, nu, nview, nv, da, off_a, dsd, dso, typeFilter, fan,
                         (cudaStream_t)stream);
}

int rn_filter_set_form(int form) {
    clear_error();
    if (form < 0 || form > 2) return set_error(RN_ERR_ARG, "filter form must be 0, 1 or 2");
    g_filter_form = form;
    return RN_OK;
}

int rn_filter_weighted(float* d_out, const float* d_prj, const float* d_w, int nBatches, int nChannels, int nu,
                       int nview, int nv, float da, float off_a, float dsd, float dso, int typeFilter, int fan,
                       void* stream) {
    clear_error();
    if (!d_out || !d_prj || !d_w) return set_error(RN_ERR_ARG, "null argument");
    return filter_device(d_out, d_prj, nBatches, nChannels, nu, nview, nv, da, off_a, dsd, dso, typeFilter, fan,
                         (cudaStream_t)stream, d_w);
}

static void host_filter(float* out, const float* prj, int nb, int nc, int nu, int nview, int nv, float da,
                        float off_a, float dsd, float dso, int typeFilter, int fan) {
    clear_error();
    if (!out || !prj) {
        set_error(RN_ERR_ARG, "null argument");
        return;
    }
    HostCtx* c = host_ctx();
    std::lock_guard<std::mutex> lk(c->mu);
    size_t n = (size_t)nb * nu * nview * nv * nc;
    if (c->c.ensure(n * 4) != RN_OK || c->d.ensure(n * 4) != RN_OK) return;
    if (cudaMemcpyAsync(c->c.p, prj, n * 4, cudaMemcpyHostToDevice, c->st) != cudaSuccess) {
        set_error(RN_ERR_CUDA, "filter: host to device copy failed");
        return;
    }
    if (filter_device(c->d.as<float>(), c->c.as<float>(), nb, nc, nu, nview, nv, da, off_a, dsd, dso, typeFilter,
                      fan, c->st) != RN_OK)
        return;
    if (cudaMemcpyAsync(out, c->d.p, n * 4, cudaMemcpyDeviceToHost, c->st) != cudaSuccess) {
        set_error(RN_ERR_CUDA, "filter: device to host copy failed");
        return;
    }
    finish_sync(c, nullptr);
}

void cFilterFanFilter(float* pFPrj, const float* pPrj, int nBatches, int nChannels, int nu, int nview, int nv,
                      float da, float dv, float off_a, float off_v, float dsd, float dso, int typeFilter,
                      int typeProjector) {
    (void)dv;
    (void)off_v;
    (void)typeProjector;
    host_filter(pFPrj, pPrj, nBatches, nChannels, nu, nview, nv, da, off_a, dsd, dso, typeFilter, 1);
}

void cFilterParallelFilter(float* pFPrj, const float* pPrj, int nBatches, int nChannels, int nu, int nview, int nv,
                           float da, float dv, float off_a, float off_v, float dsd, float dso, int typeFilter,
                           int typeProjector) {
    (void)dv;
    (void)off_v;
    (void)typeProjector;
    host_filter(pFPrj, pPrj, nBatches, nChannels, nu, nview, nv, da, off_a, dsd, dso, typeFilter, 0);
}

int rn_tv_sqs(float* d_grad, float* d_norm, double* d_tv, const float* d_img, int nslices, int nx, int ny,
              void* stream) {
    clear_error();
    if (!d_img || nslices <= 0 || nx <= 0 || ny <= 0) return set_error(RN_ERR_ARG, "tv: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (d_tv) RN_CUDA_TRY(cudaMemsetAsync(d_tv, 0, sizeof(double) * nslices, st));
    dim3 grid((unsigned)((nx * ny + 255) / 256), nslices);
    tv_kernel<<<grid, 256, 0, st>>>(d_grad, d_norm, d_tv, d_img, nx, ny);
    RN_CUDA_TRY(cudaGetLastError());
    return RN_OK;
}

float cTVSQS2D(float* grad, float* norm, const float* img, int nx, int ny) {
    clear_error();
    if (!grad || !norm || !img || nx <= 0 || ny <= 0) {
        set_error(RN_ERR_ARG, "cTVSQS2D: bad argument");
        return 0.f;
    }
    HostCtx* c = host_ctx();
    std::lock_guard<std::mutex> lk(c->mu);
    size_t n = (size_t)nx * ny;
    // scratch d: grad [n] | norm [n] | tv (8-byte aligned double)
    size_t tv_off = (n * 8 + 7) & ~size_t(7);
    if (c->c.ensure(n * 4) != RN_OK || c->d.ensure(tv_off + 8) != RN_OK) return 0.f;
    float* dimg = c->c.as<float>();
    float* dgrad = c->d.as<float>();
    float* dnorm = dgrad + n;
    double* dtv = reinterpret_cast<double*>(reinterpret_cast<char*>(c->d.p) + tv_off);
    if (cudaMemcpyAsync(dimg, img, n * 4, cudaMemcpyHostToDevice, c->st) != cudaSuccess) {
        set_error(RN_ERR_CUDA, "cTVSQS2D: copy failed");
        return 0.f;
    }
    if (rn_tv_sqs(dgrad, dnorm, dtv, dimg, 1, nx, ny, c->st) != RN_OK) return 0.f;
    double tv = 0;
    cudaMemcpyAsync(grad, dgrad, n * 4, cudaMemcpyDeviceToHost, c->st);
    cudaMemcpyAsync(norm, dnorm, n * 4, cudaMemcpyDeviceToHost, c->st);
    cudaMemcpyAsync(&tv, dtv, 8, cudaMemcpyDeviceToHost, c->st);
    if (finish_sync(c, nullptr) != RN_OK) return 0.f;
    return (float)tv;
}

int rn_fan_sqs_update(rn_fan_plan* subset_plan, float* d_x_out, const float* d_x_in, const float* d_prj_s,
                      const float* d_w_s, const float* d_norm_img, float lambda, float beta, int nSubsets, float lb,
                      float ub, int typeProjector, void* stream) {
    clear_error();
    if (typeProjector < 0 || typeProjector > 3) return set_error(RN_ERR_ARG, "typeProjector must be 0, 1, 2 or 3");
    return sqs_update(subset_plan, d_x_out, d_x_in, d_prj_s, d_w_s, d_norm_img, lambda, beta, nSubsets, lb, ub,
                      typeProjector, (cudaStream_t)stream);
}

}  // extern "C"

// Host OS-SQS loop shared by cOSSQS (Siddon pair) and cDDFanOSSQS (DD pair,
// type = typeProjector): contiguous subsets of nviewPerSubset views, the
// last one holding the remaining views.
static void host_ossqs(const char* name, float* res, const float* img, const float* prj, const float* normImg,
                       const float* wprj, const float* degs, float lb, float ub, int nviewPerSubset, int nSubsets,
                       int nBatches, int nChannels, int nx, int ny, int nz, float dx, float dy, float dz, int nu,
                       int nview, int nv, float da, float dv, float off_a, float off_v, float dsd, float dso,
                       int typeProjector, float lambda) {
    clear_error();
    if (!res || !img || !prj || !normImg || !wprj || !degs || nviewPerSubset <= 0 || nSubsets <= 0) {
        set_error(RN_ERR_ARG, std::string(name) + ": bad argument");
        return;
    }
    HostCtx* c = host_ctx();
    std::lock_guard<std::mutex> lk(c->mu);
    const size_t ni = (size_t)nBatches * nx * ny * nz * nChannels;
    const size_t rowC = (size_t)nv * nChannels;   // floats per (u, view)
    if (c->a.ensure(ni * 4 * 3) != RN_OK) return;
    float* x0 = c->a.as<float>();
    float* x1 = x0 + ni;
    float* dn = x1 + ni;
    cudaMemcpyAsync(x0, img, ni * 4, cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(dn, normImg, ni * 4, cudaMemcpyHostToDevice, c->st);
    std::vector<float> hs, hw;
    int start = 0;
    for (int k = 0; k < nSubsets && start < nview; k++) {
        int cnt = std::min(nviewPerSubset, nview - start);
        RnFanGeom g = fan_geom(nBatches, nChannels, nx, ny, nz, dx, dy, dz, nu, cnt, nv, da, dv, off_a, off_v, dsd,
                               dso);
        rn_fan_plan* sp = nullptr;
        if (rn_fan_plan_create(&sp, &g, degs + start, c->st) != RN_OK) return;
        size_t ns = (size_t)nBatches * nu * cnt * rowC;
        hs.resize(ns);
        hw.resize(ns);
        for (int b = 0; b < nBatches; b++)
            for (int u = 0; u < nu; u++) {
                size_t src = (((size_t)b * nu + u) * nview + start) * rowC;
                size_t dst = ((size_t)b * nu + u) * cnt * rowC;
                memcpy(&hs[dst], prj + src, sizeof(float) * cnt * rowC);
                memcpy(&hw[dst], wprj + src, sizeof(float) * cnt * rowC);
            }
        if (c->b.ensure(ns * 8) != RN_OK) {
            rn_fan_plan_destroy(sp);
            return;
        }
        float* dps = c->b.as<float>();
        float* dws = dps + ns;
        cudaMemcpyAsync(dps, hs.data(), ns * 4, cudaMemcpyHostToDevice, c->st);
        cudaMemcpyAsync(dws, hw.data(), ns * 4, cudaMemcpyHostToDevice, c->st);
        int s = sqs_update(sp, x1, x0, dps, dws, dn, lambda, 0.f, nSubsets, lb, ub, typeProjector, c->st);
        if (s == RN_OK) s = finish_sync(c, sp);
        rn_fan_plan_destroy(sp);
        if (s != RN_OK) return;
        std::swap(x0, x1);
        start += cnt;
    }
    cudaMemcpyAsync(res, x0, ni * 4, cudaMemcpyDeviceToHost, c->st);
    finish_sync(c, nullptr);
}

extern "C" {

// ossqs.cu:12-161: the reference runs its Siddon pair whatever typeProjector
// says (SiddonFan ignores it).
void cOSSQS(float* res, const float* img, const float* prj, const float* normImg, const float* wprj,
            const float* degs, float lb, float ub, int nviewPerSubset, int nSubsets, int nBatches, int nChannels,
            int nx, int ny, int nz, float dx, float dy, float dz, int nu, int nview, int nv, float da, float dv,
            float off_a, float off_v, float dsd, float dso, int typeProjector, float lambda) {
    (void)typeProjector;
    host_ossqs("cOSSQS", res, img, prj, normImg, wprj, degs, lb, ub, nviewPerSubset, nSubsets, nBatches, nChannels,
               nx, ny, nz, dx, dy, dz, nu, nview, nv, da, dv, off_a, off_v, dsd, dso, RN_TYPE_SIDDON, lambda);
}

void cDDFanOSSQS(float* res, const float* img, const float* prj, const float* normImg, const float* wprj,
                 const float* degs, float lb, float ub, int nviewPerSubset, int nSubsets, int nBatches,
                 int nChannels, int nx, int ny, int nz, float dx, float dy, float dz, int nu, int nview, int nv,
                 float da, float dv, float off_a, float off_v, float dsd, float dso, int typeProjector,
                 float lambda) {
    if (typeProjector < 0 || typeProjector > 2) typeProjector = 0;
    host_ossqs("cDDFanOSSQS", res, img, prj, normImg, wprj, degs, lb, ub, nviewPerSubset, nSubsets, nBatches,
               nChannels, nx, ny, nz, dx, dy, dz, nu, nview, nv, da, dv, off_a, off_v, dsd, dso, typeProjector,
               lambda);
}

}  // extern "C"
