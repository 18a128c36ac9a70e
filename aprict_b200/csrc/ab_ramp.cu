// ab_ramp.cu -- weighted 1-D convolution along the detector u axis (ramp /
// Hilbert filtering for FBP): a direct convolution from the taps, and an FFT
// convolution in shared memory from tables built once per filter.
//
// Replaces RampFilterer._filter_chunk_axis1 (src/aprict/cb/ramp_filter.py:139-240):
// zero-pad each detector row to next_fast_len(2 nu - 1), cuFFT rfft, multiply
// by the kernel spectrum, irfft, crop -- i.e. an exact linear convolution of
// the (cosine-weighted, :685-689) row with taps h[n], |n| <= nu-1. From the
// taps the same linear convolution is evaluated directly:
//     out[row][m] = scale * sum_j h[m - j] * w[j][v] * in[row][j].
//
// B200 layout: a CTA stages R rows (times the weights; R = 8 while the Q x R
// accumulators fit, else 4) and all 2 nu - 1 taps in shared memory with
// coalesced loads, then each thread produces Q outputs per row (m = t, t+T,
// ...), reading the weighted rows as R/4 float4 broadcasts and the taps
// conflict-free: each tap read feeds R multiply-adds. Pure Ram-Lak taps vanish at even
// nonzero offsets (src/aprict/ramp_kernels.py:43-59), so in ODD mode only
// taps of odd offset are visited plus the centre tap: half the FMAs.
#include <cuda_runtime.h>

#include "ab_common.cuh"
#include "ab_host.h"

namespace {

constexpr int kThreads = 256;
constexpr int kR = 4;  // rows per CTA for Q >= 8 (one float4 of a column)

struct RampParams {
    const float *in;
    float *out;
    const float *taps;     // 2*nu-1, centre at nu-1
    const float *weights;  // (nu, nv) element strides (wsu, wsv), or null
    int64_t wsu, wsv;
    int n_views, nu, nv;
    int64_t is_view, is_u, is_v;  // input strides (elements)
    int64_t os_view, os_u, os_v;  // output strides
    float scale;
    int odd;  // taps at even nonzero offsets are all zero
};

__device__ __forceinline__ void row_of(const RampParams &P, int64_t r, int &m, int &v) {
    m = (int)(r / P.nv);
    v = (int)(r % P.nv);
}

template <int Q, int R>
__global__ void __launch_bounds__(kThreads) k_ramp(RampParams P, int64_t n_rows) {
    constexpr int kG = R / 4;  // float4 groups of rows
    extern __shared__ float4 smem4[];
    float4 *xs = smem4;                                      // [nu][kG] x 4 rows
    float *hs = reinterpret_cast<float *>(smem4 + (size_t)P.nu * kG);  // [2 nu - 1]
    const int64_t r0 = (int64_t)blockIdx.x * R;
    const int nu = P.nu;

    for (int k = threadIdx.x; k < 2 * nu - 1; k += kThreads) hs[k] = P.taps[k];
    // Stage the weighted rows. Rows of a CTA are consecutive row indices
    // (view-major, v fastest): when the v stride is 1 the R rows of one u are
    // adjacent in memory, otherwise each row is contiguous along u.
    float *xf = reinterpret_cast<float *>(xs);
    const bool v_contig = P.is_v == 1 && P.nv >= R;
    for (int e = threadIdx.x; e < R * nu; e += kThreads) {
        int q, j;
        if (v_contig) {
            q = e % R;
            j = e / R;
        } else {
            q = e / nu;
            j = e % nu;
        }
        const int64_t r = r0 + q;
        float val = 0.f;
        if (r < n_rows) {
            int m, v;
            row_of(P, r, m, v);
            val = P.in[(int64_t)m * P.is_view + (int64_t)j * P.is_u + (int64_t)v * P.is_v];
            if (P.weights) val *= P.weights[(int64_t)j * P.wsu + (int64_t)v * P.wsv];
        }
        xf[j * R + q] = val;
    }
    __syncthreads();

    float acc[Q][R];
#pragma unroll
    for (int a = 0; a < Q; ++a)
#pragma unroll
        for (int q = 0; q < R; ++q) acc[a][q] = 0.f;

    const int t = threadIdx.x;
    // Taps index: h[m - j] lives at hs[m - j + nu - 1].
    if (P.odd) {
        // m shares the parity of t (kThreads is even); visit j of the other parity.
        const int j0 = 1 - (t & 1);
        for (int j = j0; j < nu; j += 2) {
            float4 x[kG];
#pragma unroll
            for (int g = 0; g < kG; ++g) x[g] = xs[j * kG + g];
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                const int m = t + a * kThreads;
                const float h = (m < nu) ? hs[m - j + nu - 1] : 0.f;
#pragma unroll
                for (int g = 0; g < kG; ++g) {
                    acc[a][4 * g + 0] = fmaf(h, x[g].x, acc[a][4 * g + 0]);
                    acc[a][4 * g + 1] = fmaf(h, x[g].y, acc[a][4 * g + 1]);
                    acc[a][4 * g + 2] = fmaf(h, x[g].z, acc[a][4 * g + 2]);
                    acc[a][4 * g + 3] = fmaf(h, x[g].w, acc[a][4 * g + 3]);
                }
            }
        }
        const float hc = hs[nu - 1];
#pragma unroll
        for (int a = 0; a < Q; ++a) {
            const int m = t + a * kThreads;
            if (m < nu) {
#pragma unroll
                for (int g = 0; g < kG; ++g) {
                    const float4 x = xs[m * kG + g];
                    acc[a][4 * g + 0] = fmaf(hc, x.x, acc[a][4 * g + 0]);
                    acc[a][4 * g + 1] = fmaf(hc, x.y, acc[a][4 * g + 1]);
                    acc[a][4 * g + 2] = fmaf(hc, x.z, acc[a][4 * g + 2]);
                    acc[a][4 * g + 3] = fmaf(hc, x.w, acc[a][4 * g + 3]);
                }
            }
        }
    } else {
        for (int j = 0; j < nu; ++j) {
            float4 x[kG];
#pragma unroll
            for (int g = 0; g < kG; ++g) x[g] = xs[j * kG + g];
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                const int m = t + a * kThreads;
                const float h = (m < nu) ? hs[m - j + nu - 1] : 0.f;
#pragma unroll
                for (int g = 0; g < kG; ++g) {
                    acc[a][4 * g + 0] = fmaf(h, x[g].x, acc[a][4 * g + 0]);
                    acc[a][4 * g + 1] = fmaf(h, x[g].y, acc[a][4 * g + 1]);
                    acc[a][4 * g + 2] = fmaf(h, x[g].z, acc[a][4 * g + 2]);
                    acc[a][4 * g + 3] = fmaf(h, x[g].w, acc[a][4 * g + 3]);
                }
            }
        }
    }

#pragma unroll
    for (int a = 0; a < Q; ++a) {
        const int mo = t + a * kThreads;
        if (mo >= nu) continue;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const int64_t r = r0 + q;
            if (r >= n_rows) continue;
            int m, v;
            row_of(P, r, m, v);
            P.out[(int64_t)m * P.os_view + (int64_t)mo * P.os_u + (int64_t)v * P.os_v] = acc[a][q] * P.scale;
        }
    }
}

// ---------------------------------------------------------------------------
// FFT form of the same convolution (aprict_b200_ramp_filter_fft), for rows of
// kFftMinNu to kFftMaxNu samples, with the filter given as its FFT tables
// (built once per filter by aprict_b200_ramp_fft_tables, as the reference
// keeps the kernel spectrum of a RampFilterer, ramp_filter.py:83-137).
// With N = 2^p >= 2 nu - 1 the circular convolution of the zero-padded row
// with the wrapped taps equals the linear one on the first nu outputs, so
//     out = scale/N * IDFT'_N(H . DFT_N(x)),  H[k] = sum_n h[n] e^{-2 pi i k n/N}
// (IDFT' unnormalised). Two real rows ride as the real and imaginary parts of
// one complex signal: h is real, so h * (a + i b) = h*a + i h*b and the parts
// separate after the inverse, taken as conj(DFT(conj(Y))).
//
// Precision: a ramp filter suppresses the low frequencies that carry most of
// a projection row's energy, so rounding errors of the forward transform
// (white, on the scale of |x|) would be amplified against the filtered
// output: an FP32 forward transform doubles the rel L2 error of the FP32
// inputs themselves (9e-6 against 4.5e-6 on fan-beam sinogram rows with
// Ram-Lak taps). The forward transform therefore runs in FP64 (half the FP32
// rate on B200), Y = H . Z is rounded to FP32, and the inverse, whose
// rounding is relative to the already filtered spectrum, runs in FP32.
//
// Each transform is a mixed-radix Stockham FFT (radix 8, then 4 or 2;
// Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC 2008) in shared memory, one radix-8 butterfly per
// thread and stage, in place (a stage's values are read into registers,
// then a barrier, then written back), rows padded by one slot every 16 (no
// bank conflict except a 2-way one on the second stage's stores), the FP32
// signals of the inverse over the FP64 ones. In place, a CTA needs half the
// shared memory of ping-pong buffers, which leaves the tables in L1 and lets
// four CTAs of 256 threads share an SM at 64 registers (A/B on one box:
// 0.59 -> 0.53 ms for 46080 rows of 1024, 2.63 -> 2.15 ms for 360 x 384 rows
// of 1024 along v). A stage loads one twiddle w per
// butterfly from the tables and forms w^2 .. w^7 by products (FP64 in the
// forward transform; FP32 in the inverse, about 1e-7 relative to the filtered
// output). The first stage's upper half of inputs is the zero padding
// (nu <= N/2). A CTA holds S signals (2 S rows), staged with the weights by
// coalesced loads whichever of u or v is the contiguous axis, and written
// back the same way.
constexpr int kFftMinNu = 128;
constexpr int kFftMaxNu = 2048;

int fft_logn(int64_t nu) {
    int logp = 8;
    while ((int64_t)1 << logp < 2 * nu - 1) ++logp;
    return logp;
}

// Table layout (byte offsets, N = 2^logp): H at 0 (N float2), the FP64
// twiddles e^{-2 pi i m/N} at 8 N (N double2), the FP32 ones at 24 N.
size_t fft_tables_bytes(int logp) { return (size_t)32 << logp; }

struct RampFftParams {
    const float *in;
    float *out;
    const float *weights;
    int64_t wsu, wsv;
    int nu, nv;
    int64_t is_view, is_u, is_v;
    int64_t os_view, os_u, os_v;
    const float2 *H;      // N
    const double2 *tw64;  // N: e^{-2 pi i m / N}
    const float2 *tw32;   // N: the same, rounded
    double hscale;        // scale / N
    int64_t n_rows;
    int in_vc, out_vc;  // rows of a CTA adjacent along v (coalesced staging)
};

__device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }

template <typename V> struct Cx;
template <> struct Cx<float2> {
    using S = float;
    static __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
};
template <> struct Cx<double2> {
    using S = double;
    static __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
};

template <typename V>
__device__ __forceinline__ V cmul(V a, V b) {
    return Cx<V>::mk(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
template <typename V>
__device__ __forceinline__ V cadd(V a, V b) { return Cx<V>::mk(a.x + b.x, a.y + b.y); }
template <typename V>
__device__ __forceinline__ V csub(V a, V b) { return Cx<V>::mk(a.x - b.x, a.y - b.y); }

template <typename V>
__device__ __forceinline__ void dft4(V &c0, V &c1, V &c2, V &c3) {
    const V d0 = cadd(c0, c2), d2 = csub(c0, c2), d1 = cadd(c1, c3);
    const V d3 = Cx<V>::mk(c1.y - c3.y, c3.x - c1.x);  // -i (c1 - c3)
    c0 = cadd(d0, d1);
    c2 = csub(d0, d1);
    c1 = cadd(d2, d3);
    c3 = csub(d2, d3);
}

// In-register DFT of size R, natural order in and out; HALF: v[R/2 ..] are
// zero (radix 8 only).
template <int R, bool HALF, typename V>
__device__ __forceinline__ void dft(V (&v)[R]) {
    using S = typename Cx<V>::S;
    if constexpr (R == 2) {
        const V a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        dft4(v[0], v[1], v[2], v[3]);
    } else {
        // X[2m] = DFT4(a_r + a_{r+4})[m], X[2m+1] = DFT4((a_r - a_{r+4}) W8^r)[m]
        const S kS = (S)0.70710678118654752440;
        V b[8];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            b[r] = HALF ? v[r] : cadd(v[r], v[r + 4]);
            b[r + 4] = HALF ? v[r] : csub(v[r], v[r + 4]);
        }
        b[5] = Cx<V>::mk((b[5].x + b[5].y) * kS, (b[5].y - b[5].x) * kS);   // W8^1 = (1 - i)/sqrt 2
        b[6] = Cx<V>::mk(b[6].y, -b[6].x);                                  // W8^2 = -i
        b[7] = Cx<V>::mk((b[7].y - b[7].x) * kS, -(b[7].x + b[7].y) * kS);  // W8^3 = (-1 - i)/sqrt 2
        dft4(b[0], b[1], b[2], b[3]);
        dft4(b[4], b[5], b[6], b[7]);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            v[2 * m] = b[m];
            v[2 * m + 1] = b[m + 4];
        }
    }
}

// One Stockham stage of radix R after NS points have been combined: butterfly
// j reads x[j + r N/R], twiddles by W_{NS R}^{(j mod NS) r}, and writes
// x'[(j - j mod NS) R + j mod NS + r NS], in place (src and dst are the same
// signal, as FP64 or, from the H stage on, as FP32). FIRST: the upper half of the
// inputs is zero padding; SPEC (end of the forward transform): outputs times
// H scale/N, conjugated, rounded to FP32.
template <int N, int NS, int R, bool FIRST, bool SPEC, typename VI, typename VO>
__device__ __forceinline__ void fft_stage(const VI *src, VO *dst, const VI *__restrict__ tw, int lt, const RampFftParams &P) {
    constexpr int B = N / R, Q8 = 8 / R;
    constexpr bool HALF = FIRST && R == 8;
    VI v[Q8][R];
    int dd[Q8];
#pragma unroll
    for (int q = 0; q < Q8; ++q) {
        const int j = lt + q * (N / 8);
#pragma unroll
        for (int r = 0; r < R; ++r) v[q][r] = (HALF && r >= R / 2) ? Cx<VI>::mk(0, 0) : src[fpad(j + r * B)];
        const int k = j & (NS - 1);
        if constexpr (NS > 1) {
            const VI w1 = __ldg(tw + k * (N / (NS * R)));
            VI w = w1;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                v[q][r] = cmul(v[q][r], w);
                if (r + 1 < R) w = cmul(w, w1);
            }
        }
        dft<R, HALF>(v[q]);
        dd[q] = (j - k) * R + k;
    }
    __syncthreads();  // every read of this stage before any write
#pragma unroll
    for (int q = 0; q < Q8; ++q) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if constexpr (SPEC) {
                const float2 h = __ldg(P.H + dd[q] + r * NS);
                const VI o = cmul(v[q][r], Cx<VI>::mk(h.x * P.hscale, h.y * P.hscale));
                dst[fpad(dd[q] + r * NS)] = make_float2((float)o.x, -(float)o.y);
            } else {
                dst[fpad(dd[q] + r * NS)] = v[q][r];
            }
        }
    }
}

// The stages of one transform in the shared buffer a: FWD in FP64 ending in
// the H stage, else FP32.
template <int N, int NS, bool FWD>
__device__ __forceinline__ void fft_run(char *a, int s, int lt, const RampFftParams &P) {
    if constexpr (NS < N) {
        constexpr int R = N / NS >= 8 ? 8 : N / NS, NP = N + N / 16;
        constexpr bool LAST = NS * R == N;
        if constexpr (FWD && LAST)
            fft_stage<N, NS, R, NS == 1, true>(reinterpret_cast<const double2 *>(a) + s * NP,
                                               reinterpret_cast<float2 *>(a) + s * NP, P.tw64, lt, P);
        else if constexpr (FWD)
            fft_stage<N, NS, R, NS == 1, false>(reinterpret_cast<const double2 *>(a) + s * NP,
                                                reinterpret_cast<double2 *>(a) + s * NP, P.tw64, lt, P);
        else
            fft_stage<N, NS, R, false, false>(reinterpret_cast<const float2 *>(a) + s * NP,
                                              reinterpret_cast<float2 *>(a) + s * NP, P.tw32, lt, P);
        __syncthreads();
        fft_run<N, NS * R, FWD>(a, s, lt, P);
    }
}

template <int LOGP> struct FftCfg {
    static constexpr int N = 1 << LOGP;
    static constexpr int S = N >= 1024 ? 1 : 1024 / N;  // signals per CTA
    static constexpr int T = S * N / 8;                 // threads
    static constexpr int NP = N + N / 16;
    static constexpr int MINB = T >= 512 ? 2 : 1024 / T;  // 64 registers a thread
    static constexpr size_t SMEM = (size_t)S * NP * sizeof(double2);
};

template <int LOGP>
__global__ void __launch_bounds__(FftCfg<LOGP>::T, FftCfg<LOGP>::MINB) k_ramp_fft(RampFftParams P) {
    using C = FftCfg<LOGP>;
    constexpr int N = C::N, S = C::S, T = C::T, NP = C::NP, Q = 2 * S;
    extern __shared__ double2 fsm[];
    __shared__ int64_t rin[Q], rout[Q], rw[Q];
    const int nu = P.nu;
    if (threadIdx.x < Q) {
        // per-row offsets; rows past the end are marked by a negative input offset
        const int64_t r = (int64_t)blockIdx.x * Q + threadIdx.x;
        const int64_t m = r / P.nv, v = r % P.nv;
        rin[threadIdx.x] = r < P.n_rows ? m * P.is_view + v * P.is_v : -1;
        rout[threadIdx.x] = m * P.os_view + v * P.os_v;
        rw[threadIdx.x] = v * P.wsv;
    }
    __syncthreads();
    // stage the rows into the lower half of each signal, zero-pad the upper
    double *bd = reinterpret_cast<double *>(fsm);
    auto stage_in = [&](int q, int j) {
        const int64_t o = rin[q];
        float val = 0.f;
        if (o >= 0 && j < nu) {
            val = __ldg(P.in + o + (int64_t)j * P.is_u);
            if (P.weights) val *= __ldg(P.weights + rw[q] + (int64_t)j * P.wsu);
        }
        bd[2 * ((q >> 1) * NP + fpad(j)) + (q & 1)] = (double)val;
    };
    if (P.in_vc) {
        for (int e = threadIdx.x; e < Q * (N / 2); e += T) stage_in(e & (Q - 1), e / Q);
    } else {
        for (int q = 0; q < Q; ++q)
            for (int j = threadIdx.x; j < N / 2; j += T) stage_in(q, j);
    }
    __syncthreads();
    const int s = threadIdx.x / (N / 8), lt = threadIdx.x % (N / 8);
    char *a = reinterpret_cast<char *>(fsm);
    fft_run<N, 1, true>(a, s, lt, P);
    fft_run<N, 1, false>(a, s, lt, P);
    // the buffer holds conj(IDFT'(Y)) of every signal (FP32, signal stride NP)
    const float *res = reinterpret_cast<const float *>(a);
    auto store_out = [&](int q, int j) {
        if (rin[q] < 0) return;
        const float val = res[2 * ((q >> 1) * NP + fpad(j)) + (q & 1)];
        P.out[rout[q] + (int64_t)j * P.os_u] = (q & 1) ? -val : val;
    };
    if (P.out_vc) {
        for (int e = threadIdx.x; e < Q * nu; e += T) store_out(e & (Q - 1), e / Q);
    } else {
        for (int q = 0; q < Q; ++q)
            for (int j = threadIdx.x; j < nu; j += T) store_out(q, j);
    }
}

// Twiddles e^{-2 pi i m / N}: FP64 from sincospi, and rounded to FP32.
__global__ void __launch_bounds__(256) k_fft_twiddles(int logp, double2 *tw64, float2 *tw32) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= (1 << logp)) return;
    double sn, cs;
    sincospi(2.0 * (double)m / (double)(1 << logp), &sn, &cs);
    tw64[m] = make_double2(cs, -sn);
    tw32[m] = make_float2((float)cs, (float)-sn);
}

// H[k] = sum_{|n| < nu} h[n] e^{-2 pi i k n / N} in FP64, one warp per k.
__global__ void __launch_bounds__(256) k_ramp_spectrum(const float *taps, int nu, int logp, const double2 *tw64,
                                                       float2 *H) {
    const int N = 1 << logp;
    const int k = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (k >= N) return;
    // h[n] e^{-i t} + h[-n] e^{i t} = (h[n] + h[-n]) cos t - i (h[n] - h[-n]) sin t
    double re = 0.0, im = 0.0;
    for (int n = 1 + lane; n < nu; n += 32) {
        const double2 w = tw64[(int)(((int64_t)k * n) & (N - 1))];
        const double hp = (double)__ldg(taps + nu - 1 + n), hm = (double)__ldg(taps + nu - 1 - n);
        re = fma(hp + hm, w.x, re);
        im = fma(hp - hm, w.y, im);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane == 0) H[k] = make_float2((float)(re + (double)taps[nu - 1]), (float)im);
}

template <int LOGP>
int launch_ramp_fft(RampFftParams P, cudaStream_t st) {
    using C = FftCfg<LOGP>;
    P.in_vc = P.is_v == 1 && P.nv >= 2 * C::S;
    P.out_vc = P.os_v == 1 && P.nv >= 2 * C::S;
    const int64_t blocks = (P.n_rows + 2 * C::S - 1) / (2 * C::S);
    if (blocks > 0x7fffffff) return ab_fail(APRICT_ERR_TOO_LARGE, "ramp filter: too many rows");
    int rc = ab_cuda_check(
        cudaFuncSetAttribute(k_ramp_fft<LOGP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM),
        "ramp filter smem");
    if (rc != APRICT_OK) return rc;
    k_ramp_fft<LOGP><<<(unsigned)blocks, C::T, C::SMEM, st>>>(P);
    return ab_cuda_check(cudaGetLastError(), "ramp_filter_fft launch");
}

int check_ramp_io(const aprict_proj_desc *in_desc, const float *in_dev, const aprict_proj_desc *out_desc,
                  const float *out_dev) {
    int rc;
    if ((rc = ab_check_projs(in_desc, in_dev, "ramp input")) != APRICT_OK) return rc;
    if ((rc = ab_check_projs(out_desc, out_dev, "ramp output")) != APRICT_OK) return rc;
    if (in_desc->n_views != out_desc->n_views || in_desc->nu != out_desc->nu || in_desc->nv != out_desc->nv)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ramp filter: input and output shapes differ");
    if (in_dev == out_dev) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ramp filter: in-place filtering is not supported");
    return APRICT_OK;
}

}  // namespace

extern "C" int aprict_b200_ramp_filter(const aprict_proj_desc *in_desc, const float *in_dev,
                                       const aprict_proj_desc *out_desc, float *out_dev, const float *taps_dev,
                                       int odd_taps_only, const float *weights_dev, int64_t w_stride_u,
                                       int64_t w_stride_v, float scale, aprict_stream_t stream) {
    int rc;
    if ((rc = check_ramp_io(in_desc, in_dev, out_desc, out_dev)) != APRICT_OK) return rc;
    if (in_desc->n_views == 0 || in_desc->nu == 0 || in_desc->nv == 0) return APRICT_OK;
    if (taps_dev == nullptr) return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ramp filter: null taps");
    const int nu = (int)in_desc->nu;
    const int q = (nu + kThreads - 1) / kThreads;
    // rows per CTA: 8 while the accumulators fit (Q <= 4), else 4
    const int rows = q <= 4 ? 8 : kR;
    const size_t smem = (size_t)nu * rows * sizeof(float) + (size_t)(2 * nu - 1) * sizeof(float);
    if (smem > 200 * 1024) return ab_fail(APRICT_ERR_TOO_LARGE, "ramp filter: nu = %d exceeds shared memory", nu);
    RampParams P;
    P.in = in_dev;
    P.out = out_dev;
    P.taps = taps_dev;
    P.weights = weights_dev;
    P.wsu = w_stride_u;
    P.wsv = w_stride_v;
    P.n_views = (int)in_desc->n_views;
    P.nu = nu;
    P.nv = (int)in_desc->nv;
    P.is_view = in_desc->stride_view;
    P.is_u = in_desc->stride_u;
    P.is_v = in_desc->stride_v;
    P.os_view = out_desc->stride_view;
    P.os_u = out_desc->stride_u;
    P.os_v = out_desc->stride_v;
    P.scale = scale;
    P.odd = odd_taps_only ? 1 : 0;
    const int64_t n_rows = (int64_t)in_desc->n_views * in_desc->nv;
    const int64_t blocks = (n_rows + rows - 1) / rows;
    if (blocks > 0x7fffffff) return ab_fail(APRICT_ERR_TOO_LARGE, "ramp filter: too many rows");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
#define AB_RAMP_LAUNCH(QQ, RR)                                                                                \
    do {                                                                                                      \
        if (smem > 48 * 1024) cudaFuncSetAttribute(k_ramp<QQ, RR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        k_ramp<QQ, RR><<<(unsigned)blocks, kThreads, smem, st>>>(P, n_rows);                                  \
    } while (0)
    if (q <= 1)
        AB_RAMP_LAUNCH(1, 8);
    else if (q <= 2)
        AB_RAMP_LAUNCH(2, 8);
    else if (q <= 4)
        AB_RAMP_LAUNCH(4, 8);
    else if (q <= 8)
        AB_RAMP_LAUNCH(8, 4);
    else if (q <= 16)
        AB_RAMP_LAUNCH(16, 4);
    else
        return ab_fail(APRICT_ERR_TOO_LARGE, "ramp filter: nu = %d exceeds 4096", nu);
#undef AB_RAMP_LAUNCH
    return ab_cuda_check(cudaGetLastError(), "ramp_filter launch");
}

extern "C" int64_t aprict_b200_ramp_fft_tables_bytes(int64_t nu) {
    if (nu < kFftMinNu || nu > kFftMaxNu) return 0;
    return (int64_t)fft_tables_bytes(fft_logn(nu));
}

extern "C" int aprict_b200_ramp_fft_tables(const float *taps_dev, int64_t nu, void *tables_dev, aprict_stream_t stream) {
    if (nu < kFftMinNu || nu > kFftMaxNu)
        return ab_fail(APRICT_ERR_UNSUPPORTED, "ramp fft tables: rows of %lld samples are filtered directly (FFT: %d..%d)",
                       (long long)nu, kFftMinNu, kFftMaxNu);
    if (taps_dev == nullptr || tables_dev == nullptr)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ramp fft tables: null taps or tables");
    if (reinterpret_cast<uintptr_t>(tables_dev) % 16 != 0)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ramp fft tables: tables must be 16-byte aligned");
    const int logp = fft_logn(nu), N = 1 << logp;
    char *t = static_cast<char *>(tables_dev);
    float2 *H = reinterpret_cast<float2 *>(t);
    double2 *tw64 = reinterpret_cast<double2 *>(t + 8 * (size_t)N);
    float2 *tw32 = reinterpret_cast<float2 *>(t + 24 * (size_t)N);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_fft_twiddles<<<(unsigned)(N / 256), 256, 0, st>>>(logp, tw64, tw32);
    int rc = ab_cuda_check(cudaGetLastError(), "ramp fft twiddles launch");
    if (rc != APRICT_OK) return rc;
    k_ramp_spectrum<<<(unsigned)(N / 8), 256, 0, st>>>(taps_dev, (int)nu, logp, tw64, H);
    return ab_cuda_check(cudaGetLastError(), "ramp spectrum launch");
}

extern "C" int aprict_b200_ramp_filter_fft(const aprict_proj_desc *in_desc, const float *in_dev,
                                           const aprict_proj_desc *out_desc, float *out_dev, const void *tables_dev,
                                           const float *weights_dev, int64_t w_stride_u, int64_t w_stride_v, float scale,
                                           aprict_stream_t stream) {
    int rc;
    if ((rc = check_ramp_io(in_desc, in_dev, out_desc, out_dev)) != APRICT_OK) return rc;
    const int64_t nu = in_desc->nu;
    if (nu < kFftMinNu || nu > kFftMaxNu)
        return ab_fail(APRICT_ERR_UNSUPPORTED, "ramp filter fft: rows of %lld samples are filtered directly (FFT: %d..%d)",
                       (long long)nu, kFftMinNu, kFftMaxNu);
    if (tables_dev == nullptr || reinterpret_cast<uintptr_t>(tables_dev) % 16 != 0)
        return ab_fail(APRICT_ERR_INVALID_ARGUMENT, "ramp filter fft: null or misaligned tables");
    if (in_desc->n_views == 0 || in_desc->nv == 0) return APRICT_OK;
    const int logp = fft_logn(nu), N = 1 << logp;
    const char *t = static_cast<const char *>(tables_dev);
    RampFftParams P;
    P.in = in_dev;
    P.out = out_dev;
    P.weights = weights_dev;
    P.wsu = w_stride_u;
    P.wsv = w_stride_v;
    P.nu = (int)nu;
    P.nv = (int)in_desc->nv;
    P.is_view = in_desc->stride_view;
    P.is_u = in_desc->stride_u;
    P.is_v = in_desc->stride_v;
    P.os_view = out_desc->stride_view;
    P.os_u = out_desc->stride_u;
    P.os_v = out_desc->stride_v;
    P.H = reinterpret_cast<const float2 *>(t);
    P.tw64 = reinterpret_cast<const double2 *>(t + 8 * (size_t)N);
    P.tw32 = reinterpret_cast<const float2 *>(t + 24 * (size_t)N);
    P.hscale = (double)scale / (double)N;
    P.n_rows = in_desc->n_views * in_desc->nv;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    switch (logp) {
        case 8: return launch_ramp_fft<8>(P, st);
        case 9: return launch_ramp_fft<9>(P, st);
        case 10: return launch_ramp_fft<10>(P, st);
        case 11: return launch_ramp_fft<11>(P, st);
        default: return launch_ramp_fft<12>(P, st);
    }
}
