// kw_fft.cuh -- shared-memory Stockham FFT building blocks for sm_100a.
//
// The spectral operators of the k-space loop (kspaceFirstOrder3D.m:792-803,
// 907-909, 977-978, 1040: fftn / ifftn of every field) are computed here as
// batched 1-D transforms of tiles held in shared memory.  A tile is a batch of
// `nl` lines of length `n`; element (line l, position i) lives at
// s[l * ls + i * es].  One transform pass reads a tile from HBM once, runs all
// radix stages in shared memory and writes it back once.
//
// Algorithm: the Stockham autosort formulation (natural-order input and
// output, no bit reversal), radices 2/3/4/5/7 in registers and any other
// prime factor as a direct sum (fft_stage_any).  Stage with radix R and
// current sub-transform length Ns: butterfly j reads x[j + t*n/R]
// (t = 0..R-1), multiplies by w^(t*k) with k = j mod Ns and
// w = exp(-2 pi i / (Ns R)), runs an R-point DFT and writes
// y[(j / Ns) * Ns * R + k + t * Ns].  Twiddles come from a per-axis table
// tw[m] = exp(-2 pi i m / n) built in FP64 on the host and stored FP32.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace kw {

constexpr int kThreads = 256;                // threads per block of every pass
constexpr int kVPT = 16;                     // complex values per thread per tile
constexpr int kCap = kThreads * kVPT;        // complex values per tile (32 KB)
constexpr int kMaxStages = 16;

struct AxisFFT {
    int n;                 // transform length
    int nstages;
    int radix[kMaxStages];
    const float2 *tw;      // device table, n entries
};

// (a.x b.x - a.y b.y, a.x b.y + a.y b.x) as a packed multiply and a packed
// fused multiply-add (each component rounds as fmaf(a.x, b.*, a.y * (+-b.*)))
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    const float2 t = __fmul2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x));
    return __ffma2_rn(make_float2(a.x, a.x), b, t);
}
// complex add / subtract as one packed FP32 instruction (sm_100 FADD2 /
// FFMA2); a - b = b * (-1) + a rounds exactly like a scalar subtraction
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// ---------------------------------------------------------------------------
// small DFTs in registers (forward: exp(-2 pi i jk/R); inverse: conjugate)
// ---------------------------------------------------------------------------
template <int R, bool INV> struct Dft;

template <bool INV> struct Dft<2, INV> {
    static __device__ __forceinline__ void run(float2 *v) {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <bool INV> struct Dft<4, INV> {
    static __device__ __forceinline__ void run(float2 *v) {
        float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        float2 t2 = cadd(v[1], v[3]), t3 = mul_mi<INV>(csub(v[1], v[3]));
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    }
};

template <bool INV> struct Dft<3, INV> {
    static __device__ __forceinline__ void run(float2 *v) {
        const float s3 = 0.86602540378443864676f;   // sin(2 pi / 3)
        float2 s = cadd(v[1], v[2]);
        float2 d = mul_mi<INV>(csub(v[1], v[2]));    // -i(v1-v2) forward
        float2 m = make_float2(v[0].x - 0.5f * s.x, v[0].y - 0.5f * s.y);
        v[0] = cadd(v[0], s);
        v[1] = make_float2(m.x + s3 * d.x, m.y + s3 * d.y);
        v[2] = make_float2(m.x - s3 * d.x, m.y - s3 * d.y);
    }
};

// Odd prime R: X_k = v0 + sum_j a_j cos(2 pi jk/R) -/+ i sum_j b_j sin(2 pi jk/R)
// with a_j = v_j + v_{R-j}, b_j = v_j - v_{R-j}, j = 1..(R-1)/2.
template <int R> struct OddTab;
template <> struct OddTab<5> {
    static __device__ __forceinline__ float c(int m) {
        const float t[5] = {1.0f, 0.30901699437494742f, -0.80901699437494742f, -0.80901699437494742f, 0.30901699437494742f};
        return t[m];
    }
    static __device__ __forceinline__ float s(int m) {
        const float t[5] = {0.0f, 0.95105651629515357f, 0.58778525229247313f, -0.58778525229247313f, -0.95105651629515357f};
        return t[m];
    }
};
template <> struct OddTab<7> {
    static __device__ __forceinline__ float c(int m) {
        const float t[7] = {1.0f, 0.62348980185873353f, -0.22252093395631440f, -0.90096886790241913f,
                            -0.90096886790241913f, -0.22252093395631440f, 0.62348980185873353f};
        return t[m];
    }
    static __device__ __forceinline__ float s(int m) {
        const float t[7] = {0.0f, 0.78183148246802981f, 0.97492791218182361f, 0.43388373911755812f,
                            -0.43388373911755812f, -0.97492791218182361f, -0.78183148246802981f};
        return t[m];
    }
};

template <int R, bool INV> struct DftOdd {
    static __device__ __forceinline__ void run(float2 *v) {
        constexpr int H = (R - 1) / 2;
        float2 a[H], b[H];
#pragma unroll
        for (int j = 1; j <= H; ++j) {
            a[j - 1] = cadd(v[j], v[R - j]);
            b[j - 1] = csub(v[j], v[R - j]);
        }
        float2 v0 = v[0];
        float2 sum = v0;
#pragma unroll
        for (int j = 0; j < H; ++j) sum = cadd(sum, a[j]);
        float2 out[R];
        out[0] = sum;
#pragma unroll
        for (int k = 1; k <= H; ++k) {
            float2 re = v0, im = make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 1; j <= H; ++j) {
                const int m = (j * k) % R;
                const float c = OddTab<R>::c(m), s = OddTab<R>::s(m);
                re.x = fmaf(c, a[j - 1].x, re.x);
                re.y = fmaf(c, a[j - 1].y, re.y);
                im.x = fmaf(s, b[j - 1].x, im.x);
                im.y = fmaf(s, b[j - 1].y, im.y);
            }
            // forward: X_k = re - i*im, X_{R-k} = re + i*im
            float2 mi = mul_mi<INV>(im);   // -i*im forward, +i*im inverse
            out[k] = cadd(re, mi);
            out[R - k] = csub(re, mi);
        }
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = out[k];
    }
};
template <bool INV> struct Dft<5, INV> {
    static __device__ __forceinline__ void run(float2 *v) { DftOdd<5, INV>::run(v); }
};
template <bool INV> struct Dft<7, INV> {
    static __device__ __forceinline__ void run(float2 *v) { DftOdd<7, INV>::run(v); }
};

// Radix-16 and radix-8 DFTs as 4x4 and 4x2 Cooley-Tukey splits in registers:
// n = N2*n1 + n2, k = k1 + N1*k2; inner DFT over n1, twiddle w_N^(n2 k1),
// outer DFT over n2.
__device__ __forceinline__ float c16(int m) {
    const float t[10] = {1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f, 0.0f,
                         -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f, -1.0f,
                         -0.92387953251128674f};
    return t[m];
}
__device__ __forceinline__ float s16(int m) {
    const float t[10] = {0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f, 1.0f,
                         0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f, 0.0f,
                         -0.38268343236508977f};
    return t[m];
}
// multiply by exp(-+ 2 pi i m / 16)
template <bool INV>
__device__ __forceinline__ float2 w16mul(float2 x, int m) {
    const float c = c16(m), s = INV ? s16(m) : -s16(m);
    return make_float2(x.x * c - x.y * s, x.x * s + x.y * c);
}

template <bool INV> struct Dft<16, INV> {
    static __device__ __forceinline__ void run(float2 *v) {
        float2 y[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
            float2 a[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
            Dft<4, INV>::run(a);
#pragma unroll
            for (int k1 = 0; k1 < 4; ++k1) y[n2][k1] = a[k1];
        }
#pragma unroll
        for (int n2 = 1; n2 < 4; ++n2)
#pragma unroll
            for (int k1 = 1; k1 < 4; ++k1) {
                const int m = n2 * k1;
                y[n2][k1] = (m == 4) ? mul_mi<INV>(y[n2][k1]) : w16mul<INV>(y[n2][k1], m);
            }
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            float2 b[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
            Dft<4, INV>::run(b);
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = b[k2];
        }
    }
};

template <bool INV> struct Dft<8, INV> {
    static __device__ __forceinline__ void run(float2 *v) {
        float2 a[4] = {v[0], v[2], v[4], v[6]};
        float2 b[4] = {v[1], v[3], v[5], v[7]};
        Dft<4, INV>::run(a);
        Dft<4, INV>::run(b);
        b[1] = w16mul<INV>(b[1], 2);
        b[2] = mul_mi<INV>(b[2]);
        b[3] = w16mul<INV>(b[3], 6);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            v[k1] = cadd(a[k1], b[k1]);
            v[k1 + 4] = csub(a[k1], b[k1]);
        }
    }
};

// ---------------------------------------------------------------------------
// one Stockham stage over a shared-memory tile
// ---------------------------------------------------------------------------
// lines_fast: consecutive threads take consecutive lines (tiles whose lines
// are interleaved, es == nl); otherwise consecutive butterflies of one line
// (tiles whose lines are contiguous, es == 1).
template <int R, bool INV>
__device__ __forceinline__ void fft_stage(float2 *s, int n, int Ns, int nl, int es, int ls,
                                          bool lines_fast, const float2 *__restrict__ tw) {
    constexpr int MAXB = (kVPT + R - 1) / R;
    const int nb = n / R;
    const int total = nb * nl;
    const int twstride = n / (Ns * R);
    float2 v[MAXB][R];
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
        const int g = threadIdx.x + b * kThreads;
        if (g < total) {
            int l, j;
            if (lines_fast) { l = g % nl; j = g / nl; } else { j = g % nb; l = g / nb; }
            const int k = j % Ns;
            const float2 *line = s + l * ls;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                float2 x = line[(j + t * nb) * es];
                if (t > 0 && k > 0) {
                    float2 w = __ldg(tw + t * k * twstride);
                    if (INV) w.y = -w.y;
                    x = cmul(x, w);
                }
                v[b][t] = x;
            }
            Dft<R, INV>::run(v[b]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
        const int g = threadIdx.x + b * kThreads;
        if (g < total) {
            int l, j;
            if (lines_fast) { l = g % nl; j = g / nl; } else { j = g % nb; l = g / nb; }
            const int k = j % Ns;
            const int base = (j / Ns) * Ns * R + k;
            float2 *line = s + l * ls;
#pragma unroll
            for (int t = 0; t < R; ++t) line[(base + t * Ns) * es] = v[b][t];
        }
    }
    __syncthreads();
}

// One Stockham stage of any radix R (the prime factors above 7): every output
// is a direct R-term sum.  Output q of butterfly j (k = j mod Ns) is
//   sum_t x[j + t n/R] w^(t k) w_R^(t q) = sum_t x[j + t n/R] tw[t e mod n],
// e = k n/(Ns R) + q n/R, written to (j / Ns) Ns R + k + q Ns.  The sums run
// in FP64 (R can be in the thousands); a thread owns at most kVPT outputs of
// the tile, held in registers until every thread has read its inputs.
template <bool INV>
__device__ __noinline__ void fft_stage_any(float2 *s, int n, int R, int Ns, int nl, int es, int ls,
                                           const float2 *__restrict__ tw) {
    const int nb = n / R;
    const int total = n * nl;
    const int twstride = n / (Ns * R);
    float2 out[kVPT];
#pragma unroll
    for (int b = 0; b < kVPT; ++b) {
        const int g = threadIdx.x + b * kThreads;
        if (g < total) {
            const int l = g / n, r = g % n;
            const int j = r % nb, q = r / nb;
            const int k = j % Ns;
            const int e = (int)(((long long)k * twstride + (long long)q * nb) % n);
            const float2 *line = s + l * ls;
            double re = 0.0, im = 0.0;
            int m = 0;
            for (int t = 0; t < R; ++t) {
                const float2 x = line[(j + t * nb) * es];
                float2 w = __ldg(tw + m);
                if (INV) w.y = -w.y;
                re = fma((double)x.x, (double)w.x, fma(-(double)x.y, (double)w.y, re));
                im = fma((double)x.x, (double)w.y, fma((double)x.y, (double)w.x, im));
                m += e;
                if (m >= n) m -= n;
            }
            out[b] = make_float2((float)re, (float)im);
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < kVPT; ++b) {
        const int g = threadIdx.x + b * kThreads;
        if (g < total) {
            const int l = g / n, r = g % n;
            const int j = r % nb, q = r / nb;
            const int k = j % Ns;
            s[l * ls + ((j / Ns) * Ns * R + k + q * Ns) * es] = out[b];
        }
    }
    __syncthreads();
}

// Full transform of every line of the tile (unnormalised in both directions).
// Must be called by all threads of the block; the caller synchronises before.
template <bool INV>
__device__ void fft_tile(float2 *s, const AxisFFT &ax, int nl, int es, int ls, bool lines_fast) {
    int Ns = 1;
    for (int st = 0; st < ax.nstages; ++st) {
        const int R = ax.radix[st];
        switch (R) {
            case 4: fft_stage<4, INV>(s, ax.n, Ns, nl, es, ls, lines_fast, ax.tw); break;
            case 2: fft_stage<2, INV>(s, ax.n, Ns, nl, es, ls, lines_fast, ax.tw); break;
            case 3: fft_stage<3, INV>(s, ax.n, Ns, nl, es, ls, lines_fast, ax.tw); break;
            case 5: fft_stage<5, INV>(s, ax.n, Ns, nl, es, ls, lines_fast, ax.tw); break;
            case 7: fft_stage<7, INV>(s, ax.n, Ns, nl, es, ls, lines_fast, ax.tw); break;
            default: fft_stage_any<INV>(s, ax.n, R, Ns, nl, es, ls, ax.tw); break;
        }
        Ns *= R;
    }
}

// ---------------------------------------------------------------------------
// compile-time transforms: the axis length N and the tile's line count are
// template parameters, so every index split, stride and loop count below is a
// constant.  Radix plan: 16, 8, 4, 2 while they divide, then 3, 5, 7.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int plan_next(int n) {
    return n % 16 == 0 ? 16 : n % 8 == 0 ? 8 : n % 4 == 0 ? 4 : n % 2 == 0 ? 2 : n % 3 == 0 ? 3
         : n % 5 == 0 ? 5 : n % 7 == 0 ? 7 : 0;
}
__host__ __device__ constexpr bool plan_ok(int n) {
    return n == 1 ? true : (plan_next(n) == 0 ? false : plan_ok(n / plan_next(n)));
}
__host__ __device__ constexpr int pow2_floor(int v) { return v < 2 ? 1 : 2 * pow2_floor(v / 2); }

// padded contiguous line layout: one pad slot after every 16 elements
template <int N> struct Padded {
    static constexpr int LS = N + (N + 15) / 16;
    static __device__ __forceinline__ int at(int l, int i) { return l * LS + i + (i >> 4); }
};

// One stage; IL: lines interleaved (element (l, i) at s[i*NL + l], consecutive
// threads take consecutive lines), else padded contiguous lines (consecutive
// threads take consecutive butterflies of one line).
template <int R, bool INV, int N, int NS, int NL, bool IL>
__device__ __forceinline__ void stage_c(float2 *s, const float2 *__restrict__ tw) {
    constexpr int NB = N / R;
    constexpr int TOTAL = NB * NL;
    constexpr int TWS = N / (NS * R);
    constexpr int MAXB = (TOTAL + kThreads - 1) / kThreads;
    float2 v[MAXB][R];
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
        const int g = threadIdx.x + b * kThreads;
        if (TOTAL % kThreads == 0 || g < TOTAL) {
            const int l = IL ? g % NL : g / NB;
            const int j = IL ? g / NL : g % NB;
            const int k = j % NS;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int i = j + t * NB;
                float2 x = IL ? s[i * NL + l] : s[Padded<N>::at(l, i)];
                if (NS > 1 && t > 0) {
                    float2 w = __ldg(tw + t * k * TWS);
                    if (INV) w.y = -w.y;
                    x = cmul(x, w);
                }
                v[b][t] = x;
            }
            Dft<R, INV>::run(v[b]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
        const int g = threadIdx.x + b * kThreads;
        if (TOTAL % kThreads == 0 || g < TOTAL) {
            const int l = IL ? g % NL : g / NB;
            const int j = IL ? g / NL : g % NB;
            const int k = j % NS;
            const int base = (j / NS) * NS * R + k;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int i = base + t * NS;
                if (IL) s[i * NL + l] = v[b][t];
                else s[Padded<N>::at(l, i)] = v[b][t];
            }
        }
    }
    __syncthreads();
}

template <int N, int NL, bool INV, bool IL, int REM = N, int NS = 1>
__device__ __forceinline__ void fft_static(float2 *s, const float2 *__restrict__ tw) {
    if constexpr (REM > 1) {
        constexpr int R = plan_next(REM);
        static_assert(R > 0, "axis length has a prime factor above 7");
        stage_c<R, INV, N, NS, NL, IL>(s, tw);
        fft_static<N, NL, INV, IL, REM / R, NS * R>(s, tw);
    }
}

}  // namespace kw
