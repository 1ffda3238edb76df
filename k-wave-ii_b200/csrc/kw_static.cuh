// kw_static.cuh -- register-staged transform passes for compile-time axis lengths.
//
// Same algorithms as kw_kernels.cuh (Stockham transforms, fused physics
// stages), organised so that data crosses shared memory as little as
// possible:
//   * the first radix stage of every transform loads its butterfly inputs
//     straight from global memory (or from registers), the last stage hands
//     its outputs to a consumer in registers; only the stages in between
//     exchange through shared memory (one exchange for N <= 256);
//   * an inverse transform runs the forward radix plan reversed, so the
//     inverse's last stage and a following forward's first stage own the same
//     elements in the same thread: "inverse -> physics -> forward" (z-stages)
//     and "forward -> operator -> inverse" (x-pass) stay in registers.
#pragma once

#include <type_traits>

#include "kw_kernels.cuh"

namespace kw {

__host__ __device__ constexpr int rs_stages(int n) {
    int m = 0;
    while (n > 1) { n /= plan_next(n); ++m; }
    return m;
}
__host__ __device__ constexpr int rs_radix(int n, int s) {
    for (int k = 0; k < s; ++k) n /= plan_next(n);
    return plan_next(n);
}

template <int N, bool INV> struct RPlan {
    static constexpr int M = rs_stages(N);
    __host__ __device__ static constexpr int R(int s) { return INV ? rs_radix(N, M - 1 - s) : rs_radix(N, s); }
    __host__ __device__ static constexpr int NS(int s) {
        int p = 1;
        for (int k = 0; k < s; ++k) p *= R(k);
        return p;
    }
};

// element (l, i) of a tile: interleaved lines (i*NL + l) or padded rows
template <int N, int NL, bool IL>
__device__ __forceinline__ int tat(int l, int i) {
    if constexpr (IL) return i * NL + l;
    else return Padded<N>::at(l, i);
}

// butterfly g of a stage with NB butterflies per line -> (line, butterfly)
template <int NB, int NL, bool IL>
__device__ __forceinline__ void bmap(int g, int &l, int &j) {
    if constexpr (IL) { l = g % NL; j = g / NL; }
    else { j = g % NB; l = g / NB; }
}

// Contiguous lines (not interleaved) with NT / NL threads per line, a divisor
// of 32, and every stage's butterflies per line a multiple of it: thread u of
// line l (l = tid / T, u = tid % T) takes butterflies u, u + T, ... of its
// line in every stage, so a line never leaves its warp and the exchanges
// between stages need only warp barriers (N = 64, 128, 256, 512 x-passes).
template <int N, int NL, int NT, bool IL>
__host__ __device__ constexpr bool line_in_warp() {
    if (IL || NL <= 0 || NT % NL != 0) return false;
    constexpr int T = NT / NL;
    if (T <= 0 || 32 % T != 0) return false;
    int n = N;
    while (n > 1) {
        const int r = plan_next(n);
        if (r == 0 || (N / r) % T != 0) return false;
        n /= r;
    }
    return true;
}

// butterfly slot b of this thread at a stage with NB butterflies per line ->
// (line, butterfly): the line-in-warp map, or butterfly g = tid + b NT of
// the tile in the order of bmap
template <int NB, int NL, bool IL, int NT, bool LW>
__device__ __forceinline__ void bslot(int b, int &l, int &j) {
    if constexpr (LW) {
        constexpr int T = NT / NL;
        l = threadIdx.x / T;
        j = threadIdx.x % T + T * b;
    } else {
        bmap<NB, NL, IL>(threadIdx.x + b * NT, l, j);
    }
}

// Registers a thread owns after stage S of plan (N, INV) in a block of NT
// threads: MAXB butterflies of R values.
template <int N, int NL, bool INV, int S, int NT = kThreads> struct StageShape {
    static constexpr int R = RPlan<N, INV>::R(S);
    static constexpr int NB = N / R;
    static constexpr int TOT = NB * NL;
    static constexpr int MAXB = (TOT + NT - 1) / NT;
};
// the shape of the registers handed between an inverse's last stage and a
// forward's first stage (identical by construction)
template <int N, int NL, int NT = kThreads> using HandShape = StageShape<N, NL, false, 0, NT>;

// Twiddle table access: a global table through the read-only path, or a
// copy the block keeps in shared memory (SmemTable).
struct SmemTable {
    const float2 *p;
};
__device__ __forceinline__ float2 tw_at(const float2 *__restrict__ tw, int i) { return __ldg(tw + i); }
__device__ __forceinline__ float2 tw_at(const SmemTable &tw, int i) { return tw.p[i]; }

// Per-stage twiddle table in shared memory for contiguous-line passes: the
// multipliers of stage S >= 1 of plan (N, INV) at [off(S) + (t - 1) NS + k]
// (k = butterfly index within its group of NS, t = 1 .. R-1), conjugated
// already for an inverse plan.  Threads with consecutive k read consecutive
// entries, where the shared N-entry table (index t k N / (NS R)) puts them
// 2 t words apart and so into the same banks for even t.
struct StageTable {
    const float2 *p;
};
template <int N, bool INV>
__host__ __device__ constexpr int stage_table_off(int S) {
    int o = 0;
    for (int s = 1; s < S; ++s) o += (RPlan<N, INV>::R(s) - 1) * RPlan<N, INV>::NS(s);
    return o;
}
template <int N, bool INV> __host__ __device__ constexpr int stage_table_size() {
    return stage_table_off<N, INV>(RPlan<N, INV>::M);
}
// fill the table of plan (N, INV) from the N-entry forward table tw (block-wide)
template <int N, bool INV, int NT>
__device__ __forceinline__ void stage_table_fill(float2 *dst, const float2 *__restrict__ tw) {
    constexpr int M = RPlan<N, INV>::M;
    for (int e = threadIdx.x; e < stage_table_size<N, INV>(); e += NT) {
        int S = 1;
        while (S + 1 < M && e >= stage_table_off<N, INV>(S + 1)) ++S;
        const int NS = RPlan<N, INV>::NS(S), R = RPlan<N, INV>::R(S);
        const int r = e - stage_table_off<N, INV>(S);
        const int t = r / NS + 1, k = r % NS;
        float2 w = __ldg(tw + t * k * (N / (NS * R)));
        if (INV) w.y = -w.y;
        dst[e] = w;
    }
}

template <int N, int NL, bool IL, bool INV, int S, int NT, class TW, class Ld, class St>
__device__ __forceinline__ void rs_stage(float2 *sm, const TW &tw, Ld &ld, St &st) {
    using P = RPlan<N, INV>;
    using SH = StageShape<N, NL, INV, S, NT>;
    constexpr int M = P::M, R = SH::R, NS = P::NS(S), NB = SH::NB;
    constexpr int TOT = SH::TOT, MAXB = SH::MAXB;
    constexpr int TWS = N / (NS * R);
    // a line that stays in one warp through every stage is exchanged under a
    // warp barrier (no block barrier)
    constexpr bool WL = line_in_warp<N, NL, NT, IL>();
    float2 v[MAXB][R];
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
        const int g = threadIdx.x + b * NT;
        if (WL || TOT % NT == 0 || g < TOT) {
            int l, j;
            bslot<NB, NL, IL, NT, WL>(b, l, j);
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int i = j + t * NB;
                if constexpr (S == 0) v[b][t] = ld(b, t, l, i);
                else v[b][t] = sm[tat<N, NL, IL>(l, i)];
            }
            if constexpr (NS > 1) {
                const int k = j % NS;
#pragma unroll
                for (int t = 1; t < R; ++t) {
                    float2 w;
                    if constexpr (std::is_same<TW, StageTable>::value) {
                        w = tw.p[stage_table_off<N, INV>(S) + (t - 1) * NS + k];
                    } else {
                        w = tw_at(tw, t * k * TWS);
                        if (INV) w.y = -w.y;
                    }
                    v[b][t] = cmul(v[b][t], w);
                }
            }
            Dft<R, INV>::run(v[b]);
        }
    }
    if constexpr (S == M - 1) {
#pragma unroll
        for (int b = 0; b < MAXB; ++b) {
            const int g = threadIdx.x + b * NT;
            if (WL || TOT % NT == 0 || g < TOT) {
                int l, j;
                bslot<NB, NL, IL, NT, WL>(b, l, j);
                const int base = (j / NS) * NS * R + j % NS;
#pragma unroll
                for (int t = 0; t < R; ++t) st(b, t, l, base + t * NS, v[b][t]);
            }
        }
    } else {
        // earlier readers of the tile are done
        if constexpr (WL) __syncwarp();
        else __syncthreads();
#pragma unroll
        for (int b = 0; b < MAXB; ++b) {
            const int g = threadIdx.x + b * NT;
            if (WL || TOT % NT == 0 || g < TOT) {
                int l, j;
                bslot<NB, NL, IL, NT, WL>(b, l, j);
                const int base = (j / NS) * NS * R + j % NS;
#pragma unroll
                for (int t = 0; t < R; ++t) sm[tat<N, NL, IL>(l, base + t * NS)] = v[b][t];
            }
        }
        if constexpr (WL) __syncwarp();
        else __syncthreads();
    }
}

template <int N, int NL, bool IL, bool INV, int S = 0, int NT = kThreads, class TW, class Ld, class St>
__device__ __forceinline__ void rs_fft(float2 *sm, const TW &tw, Ld &ld, St &st) {
    rs_stage<N, NL, IL, INV, S, NT>(sm, tw, ld, st);
    if constexpr (S + 1 < RPlan<N, INV>::M) rs_fft<N, NL, IL, INV, S + 1, NT>(sm, tw, ld, st);
}

// (line, element) owned by hand-off register (b, t)
template <int N, int NL, bool IL, int NT = kThreads>
__device__ __forceinline__ bool hand_pos(int b, int t, int &l, int &i) {
    using SH = HandShape<N, NL, NT>;
    const int g = threadIdx.x + b * NT;
    if (!(SH::TOT % NT == 0 || g < SH::TOT)) return false;
    int j;
    bmap<SH::NB, NL, IL>(g, l, j);
    i = j + t * SH::NB;
    return true;
}

// (line, first element) of hand-off slot b: element (b, t) is element
// j + t * NB of line l (hand_pos)
template <int N, int NL, bool IL, int NT = kThreads>
__device__ __forceinline__ bool hand_line(int b, int &l, int &j) {
    using SH = HandShape<N, NL, NT>;
    const int g = threadIdx.x + b * NT;
    if (!(SH::TOT % NT == 0 || g < SH::TOT)) return false;
    bmap<SH::NB, NL, IL>(g, l, j);
    return true;
}

// sinc(a) = sin(a)/a and cos(a) from their Taylor series in a^2 (Horner form).
// The k-space argument is a = c_ref |k| dt / 2 <= (CFL c_ref / c_max) pi sqrt(3) / 2,
// below 2.8 for any CFL <= 1; the first omitted terms (a^16/17! and
// a^18/18!) are then below 1e-7 and 1.7e-8.
__device__ __forceinline__ float sinc_series(float a2) {
    // sin(a)/a = sum_n (-1)^n a^(2n) / (2n+1)!, n = 0..7
    float r = -1.0f / 1307674368000.0f;           // n = 7: -1/15!
    r = fmaf(r, a2, 1.0f / 6227020800.0f);        // n = 6: +1/13!
    r = fmaf(r, a2, -1.0f / 39916800.0f);         // n = 5: -1/11!
    r = fmaf(r, a2, 1.0f / 362880.0f);            // n = 4: +1/9!
    r = fmaf(r, a2, -1.0f / 5040.0f);             // n = 3: -1/7!
    r = fmaf(r, a2, 1.0f / 120.0f);               // n = 2: +1/5!
    r = fmaf(r, a2, -1.0f / 6.0f);                // n = 1: -1/3!
    r = fmaf(r, a2, 1.0f);                        // n = 0
    return r;
}
// The same series to a^10, for plans with a^2 <= 1 (OpParams::short_series):
// the first omitted terms, a^12 / 13! and a^12 / 12!, are then below 2.1e-9.
__device__ __forceinline__ float sinc_series_short(float a2) {
    float r = -1.0f / 39916800.0f;                // n = 5: -1/11!
    r = fmaf(r, a2, 1.0f / 362880.0f);            // n = 4: +1/9!
    r = fmaf(r, a2, -1.0f / 5040.0f);             // n = 3: -1/7!
    r = fmaf(r, a2, 1.0f / 120.0f);               // n = 2: +1/5!
    r = fmaf(r, a2, -1.0f / 6.0f);                // n = 1: -1/3!
    r = fmaf(r, a2, 1.0f);                        // n = 0
    return r;
}
__device__ __forceinline__ float cos_series_short(float a2) {
    float r = -1.0f / 3628800.0f;                 // n = 5: -1/10!
    r = fmaf(r, a2, 1.0f / 40320.0f);             // n = 4: +1/8!
    r = fmaf(r, a2, -1.0f / 720.0f);              // n = 3: -1/6!
    r = fmaf(r, a2, 1.0f / 24.0f);                // n = 2: +1/4!
    r = fmaf(r, a2, -0.5f);                       // n = 1: -1/2!
    r = fmaf(r, a2, 1.0f);                        // n = 0
    return r;
}
__device__ __forceinline__ float cos_series(float a2) {
    // cos(a) = sum_n (-1)^n a^(2n) / (2n)!, n = 0..8
    float r = 1.0f / 20922789888000.0f;           // n = 8: +1/16!
    r = fmaf(r, a2, -1.0f / 87178291200.0f);      // n = 7: -1/14!
    r = fmaf(r, a2, 1.0f / 479001600.0f);         // n = 6: +1/12!
    r = fmaf(r, a2, -1.0f / 3628800.0f);          // n = 5: -1/10!
    r = fmaf(r, a2, 1.0f / 40320.0f);             // n = 4: +1/8!
    r = fmaf(r, a2, -1.0f / 720.0f);              // n = 3: -1/6!
    r = fmaf(r, a2, 1.0f / 24.0f);                // n = 2: +1/4!
    r = fmaf(r, a2, -0.5f);                       // n = 1: -1/2!
    r = fmaf(r, a2, 1.0f);                        // n = 0
    return r;
}

// Tile widths of the compile-time kernels.  x-pass: as many lines as fill
// one 4096-element tile of 256 threads, so every thread owns one radix-R
// butterfly (the lines are contiguous rows, so the width does not change how
// HBM is accessed).
__host__ __device__ constexpr int ks_xlines(int n) {
    return pow2_floor(kCap / n) < 64 ? pow2_floor(kCap / n) : 64;
}
// z-stages and y-pass, whose tile width is the length of every row segment
// they move: the same, except that 512-point axes take 16 lines (8192
// elements, 512 threads) so that rows of real fields are 64 bytes and rows of
// spectra 128 bytes, not half that.
__host__ __device__ constexpr int ks_lines(int n) { return n == 512 ? 16 : ks_xlines(n); }
// Narrower tiles (pl lines, for grids too small to fill the GPU with full
// tiles) keep the per-thread share of a full tile, so the block shrinks with
// the tile: ks_threads(n, pl) threads.
__host__ __device__ constexpr int ks_threads(int n, int pl) { return kThreads * pl / ks_xlines(n); }
// the narrow tile widths used when full tiles give less than one wave of blocks
__host__ __device__ constexpr int ks_narrow(int n) { return ks_lines(n) / 4; }
__host__ __device__ constexpr int ks_xnarrow(int n) { return ks_xlines(n) / 4; }
// half-width tiles, between the two: a choice of the autotuner for grids
// whose full tiles leave a ragged last wave of blocks
__host__ __device__ constexpr int ks_half(int n) { return ks_lines(n) / 2; }
__host__ __device__ constexpr int ks_xhalf(int n) { return ks_xlines(n) / 2; }

// ---------------------------------------------------------------------------
// y-pass (C2C along axis 1, in place).  grid = (ceil(N0/TY), N2h, nfields),
// ks_threads(N1, TY) threads, N1 * TY float2 of dynamic shared memory
// ---------------------------------------------------------------------------
template <bool INV, int N1, int TY>
__global__ void __launch_bounds__(ks_threads(N1, TY), (4 * kThreads + ks_threads(N1, TY) - 1) / ks_threads(N1, TY))
    ks_ypass(Spec4 bufs, Geom g, const float2 *__restrict__ tw, int kz0) {
    constexpr int NT = ks_threads(N1, TY);
    static_assert(RPlan<N1, false>::M >= 2, "in-place pass needs two stages");
    extern __shared__ float2 sm[];   // N1 * TY
    // fields in reverse order: blocks start on the field the previous pass
    // (x-pass or z-stage, which walk them in order) wrote last, still in L2
    float2 *buf = pick(bufs.p, gridDim.z - 1 - blockIdx.z);
    const int x0 = blockIdx.x * TY;
    const long long base = (long long)(blockIdx.y + kz0) * N1 * g.N0 + x0;
    const int N0 = g.N0;
    auto ld = [&](int, int, int l, int i) -> float2 {
        return x0 + l < N0 ? buf[base + (long long)i * N0 + l] : make_float2(0.f, 0.f);
    };
    auto st = [&](int, int, int l, int i, float2 v) {
        if (x0 + l < N0) buf[base + (long long)i * N0 + l] = v;
    };
    // twiddles from shared memory (first read after the first stage's barrier)
    __shared__ float2 s_tw[N1];
    for (int i = threadIdx.x; i < N1; i += NT) s_tw[i] = __ldg(tw + i);
    rs_fft<N1, TY, true, INV, 0, NT>(sm, SmemTable{s_tw}, ld, st);
}

// ---------------------------------------------------------------------------
// Inverse y-pass of the 3-D gradient fan-out.  The x-pass left the axis-0
// output in bufs.p[0] and, in bufs.p[1], the inverse x-transform B shared by
// the axis-1 and axis-2 outputs, whose multipliers dd_y(k_y) and dd_z(k_z)
// are constant along x.  blockIdx.z = 0 transforms bufs.p[0] in place;
// blockIdx.z = 1 reads B twice (the second time from L2) and writes
// dd_z(k_z) IFFT_y(B) to bufs.p[2], then IFFT_y(dd_y(k_y) B) in place to
// bufs.p[1].  One read of B replaces the x-pass's write and this pass's read
// of a third field.  grid = (ceil(N0/TY), N2h, 2).
// ---------------------------------------------------------------------------
template <int N1, int TY>
__global__ void __launch_bounds__(ks_threads(N1, TY), (4 * kThreads + ks_threads(N1, TY) - 1) / ks_threads(N1, TY))
    ks_ypass_fan(Spec4 bufs, Geom g, const float2 *__restrict__ tw, int kz0, const float2 *__restrict__ ddy,
                 const float2 *__restrict__ ddz) {
    constexpr int NT = ks_threads(N1, TY);
    static_assert(RPlan<N1, false>::M >= 2, "in-place pass needs two stages");
    extern __shared__ float2 sm[];   // N1 * TY
    const int x0 = blockIdx.x * TY;
    const int kz = blockIdx.y + kz0;
    const long long base = (long long)kz * N1 * g.N0 + x0;
    const int N0 = g.N0;
    __shared__ float2 s_tw[N1], s_dy[N1];
    for (int i = threadIdx.x; i < N1; i += NT) {
        s_tw[i] = __ldg(tw + i);
        s_dy[i] = __ldg(ddy + i);
    }
    const SmemTable stw{s_tw};
    if (blockIdx.z == 0) {
        float2 *buf = bufs.p[0];
        auto ld = [&](int, int, int l, int i) -> float2 {
            return x0 + l < N0 ? buf[base + (long long)i * N0 + l] : make_float2(0.f, 0.f);
        };
        auto st = [&](int, int, int l, int i, float2 v) {
            if (x0 + l < N0) buf[base + (long long)i * N0 + l] = v;
        };
        rs_fft<N1, TY, true, true, 0, NT>(sm, stw, ld, st);
        return;
    }
    float2 *B = bufs.p[1], *out_z = bufs.p[2];
    const float2 mz = __ldg(ddz + kz);
    auto ldb = [&](int, int, int l, int i) -> float2 {
        return x0 + l < N0 ? B[base + (long long)i * N0 + l] : make_float2(0.f, 0.f);
    };
    auto stz = [&](int, int, int l, int i, float2 v) {
        if (x0 + l < N0) out_z[base + (long long)i * N0 + l] = cmul(v, mz);
    };
    rs_fft<N1, TY, true, true, 0, NT>(sm, stw, ldb, stz);
    // the first stage's loads of the second transform come after every
    // thread's loads of the first (its stores went to out_z, not B)
    auto ldy = [&](int, int, int l, int i) -> float2 {
        return x0 + l < N0 ? cmul(B[base + (long long)i * N0 + l], s_dy[i]) : make_float2(0.f, 0.f);
    };
    auto sty = [&](int, int, int l, int i, float2 v) {
        if (x0 + l < N0) B[base + (long long)i * N0 + l] = v;
    };
    rs_fft<N1, TY, true, true, 0, NT>(sm, stw, ldy, sty);
}

// ---------------------------------------------------------------------------
// x-pass: forward C2C along axis 0, operator, inverse C2C, in place.
// grid = (ceil(N1*N2h/NL), 1, fanout ? 1 : nfields), ks_threads(N0, NL) threads.
// FAN: 0 the single-output variant (four blocks per SM); 1 the general
// fan-out (ops.n outputs from one forward transform, kept in registers across
// the inverse transforms); 2 the fan-out of the 3-D gradient ahead of
// ks_ypass_fan (output 0 along x with its own inverse transform, outputs 1
// and 2 sharing one stored unscaled in bufs.p[1]).  The fan-out variants run
// three blocks per SM.  The operator class and, for FAN 0 and 2, the inverse
// transform's input multiplier are chosen once per block, outside the
// per-value loops.
// ---------------------------------------------------------------------------

// operator classes of the x-pass's common factor (times 1/N); the _SHORT
// forms take the shorter k-space series (OpParams::short_series)
enum { XOP_ONE = 0, XOP_SINC = 1, XOP_NABLA = 2, XOP_COS = 3, XOP_SINC_SHORT = 4, XOP_COS_SHORT = 5 };

__device__ __forceinline__ int xop_class(int kind, const OpParams &P) {
    if (kind == OP_GRAD_POS || kind == OP_GRAD_NEG)
        return P.use_kspace ? (P.short_series ? XOP_SINC_SHORT : XOP_SINC) : XOP_ONE;
    if (kind == OP_NABLA1 || kind == OP_NABLA2) return XOP_NABLA;
    if (kind == OP_SRC_KAPPA) return P.use_kspace ? (P.short_series ? XOP_COS_SHORT : XOP_COS) : XOP_ONE;
    return XOP_ONE;
}

// spec <- spec * fac(k) / N for the values this thread holds after the
// forward transform's last stage
template <int N0, int NL, int NT, int CLS, class SPEC>
__device__ __forceinline__ void xpass_operator(SPEC &spec, const OpParams &P, int kind0, const float *s_kx2,
                                               const float *kyz2, int line0, int lines_total) {
    using SH = StageShape<N0, NL, false, RPlan<N0, false>::M - 1, NT>;
    constexpr bool LW = line_in_warp<N0, NL, NT, false>();
    constexpr int NSL = RPlan<N0, false>::NS(RPlan<N0, false>::M - 1);
#pragma unroll
    for (int b = 0; b < SH::MAXB; ++b) {
        const int gg = threadIdx.x + b * NT;
        if (!(LW || SH::TOT % NT == 0 || gg < SH::TOT)) continue;
        int l, j;
        bslot<SH::NB, NL, false, NT, LW>(b, l, j);
        const float ky = kyz2[l];
#pragma unroll
        for (int t = 0; t < SH::R; ++t) {
            const int ix = j + t * NSL;
            const float k2 = s_kx2[ix] + ky;
            float fac;
            if constexpr (CLS == XOP_SINC) {
                fac = sinc_series(P.kappa_a * P.kappa_a * k2);
            } else if constexpr (CLS == XOP_SINC_SHORT) {
                fac = sinc_series_short(P.kappa_a * P.kappa_a * k2);
            } else if constexpr (CLS == XOP_COS_SHORT) {
                fac = cos_series_short(P.kappa_a * P.kappa_a * k2);
            } else if constexpr (CLS == XOP_NABLA) {
                const float e = kind0 == OP_NABLA1 ? P.nabla1_exp : P.nabla2_exp;
                fac = k2 == 0.f ? (e > 0.f ? 0.f : (e == 0.f ? 1.f : 0.f)) : pow_pos(k2, 0.5f * e);
                if (P.filt) fac *= __ldg(P.filt + (long long)min(line0 + l, lines_total - 1) * N0 + ix);
            } else if constexpr (CLS == XOP_COS) {
                fac = cos_series(P.kappa_a * P.kappa_a * k2);
            } else {
                fac = 1.f;
            }
            spec[b][t] = cscale(spec[b][t], fac * P.scale);
        }
    }
}

template <int N0, int NL, int FAN>
__global__ void __launch_bounds__(ks_threads(N0, NL), (FAN ? 3 : 4) * kThreads / ks_threads(N0, NL))
    ks_xpass(Spec4 bufs, Geom g, const float2 *__restrict__ tw, OpParams P, OpSet ops, int fanout_arg, int kz0,
             int nkz) {
    constexpr int NT = ks_threads(N0, NL);
    const int fanout = FAN == 0 ? 0 : (FAN == 2 ? 2 : fanout_arg);
    static_assert(RPlan<N0, false>::M >= 2, "in-place pass needs two stages");
    __shared__ float2 sm[NL * Padded<N0>::LS];
    __shared__ float kyz2[NL];
    // per-line multiplier of each output whose operator table runs along y
    // or z (constant along an x line); 1 for the others
    __shared__ float2 s_lm[3][NL];
    // per-x tables read on the transforms' dependency chains, kept in shared
    // memory: twiddles, k_x^2 and the x-derivative table of an axis-0 output.
    // Stage twiddles: per-stage tables for contiguous lines of up to 256
    // points (conflict-free reads), else the N0-entry table (512 points would
    // take the static shared memory past 48 KB)
    constexpr bool STAB = line_in_warp<N0, NL, NT, false>() && N0 <= 256;
    __shared__ float2 s_tw[STAB ? 1 : N0], s_ddx[N0];
    __shared__ float2 s_stf[STAB ? stage_table_size<N0, false>() : 1], s_sti[STAB ? stage_table_size<N0, true>() : 1];
    __shared__ float s_kx2[N0];
    // lines (y, kz) of kz planes kz0 .. kz0+nkz-1
    const int lines_total = (kz0 + nkz) * g.N1;
    const int line0 = kz0 * g.N1 + blockIdx.x * NL;
    const int f = fanout ? 0 : blockIdx.z;
    const float2 *ddx = nullptr;
    for (int o = 0; o < (fanout ? ops.n : 1); ++o) {
        const int oi = fanout ? o : f;
        const int ko = pick(ops.kind, oi);
        if (pick(ops.axis, oi) == 0 && (ko == OP_GRAD_POS || ko == OP_GRAD_NEG || ko == OP_SHIFT_NEG))
            ddx = ko == OP_GRAD_POS ? P.dd_pos[0] : (ko == OP_GRAD_NEG ? P.dd_neg[0] : P.sh_neg[0]);
    }
    for (int i = threadIdx.x; i < N0; i += NT) {
        if constexpr (!STAB) s_tw[i] = __ldg(tw + i);
        s_kx2[i] = __ldg(P.k2[0] + i);
        if (ddx) s_ddx[i] = __ldg(ddx + i);
    }
    if constexpr (STAB) {
        stage_table_fill<N0, false, NT>(s_stf, tw);
        stage_table_fill<N0, true, NT>(s_sti, tw);
    }
    using TT = std::conditional_t<STAB, StageTable, SmemTable>;
    const TT twf{STAB ? s_stf : s_tw}, twi{STAB ? s_sti : s_tw};
    for (int l = threadIdx.x; l < NL; l += NT) {
        const int line = min(line0 + l, lines_total - 1);
        const int iy = line % g.N1, iz = line / g.N1;
        kyz2[l] = __ldg(P.k2[1] + iy) + __ldg(P.k2[2] + iz);
#pragma unroll
        for (int o = 0; o < 3; ++o) {
            float2 m = make_float2(1.f, 0.f);
            if (o < ops.n && ops.axis[o] != 0) {
                const int ko = ops.kind[o], ax = ops.axis[o];
                const float2 *dd = ko == OP_GRAD_POS ? pick(P.dd_pos, ax)
                                                     : (ko == OP_GRAD_NEG ? pick(P.dd_neg, ax) : pick(P.sh_neg, ax));
                if (ko == OP_GRAD_POS || ko == OP_GRAD_NEG || ko == OP_SHIFT_NEG) m = __ldg(dd + (ax == 1 ? iy : iz));
            }
            s_lm[o][l] = m;
        }
    }
    __syncthreads();
    const float2 *in = pick(bufs.p, f) + (long long)line0 * N0;
    auto ld = [&](int, int, int l, int i) -> float2 {
        return line0 + l < lines_total ? in[l * N0 + i] : make_float2(0.f, 0.f);
    };
    using SH = StageShape<N0, NL, false, RPlan<N0, false>::M - 1, NT>;   // forward last stage
    float2 spec[SH::MAXB][SH::R];
    auto keep = [&](int b, int t, int, int, float2 v) { spec[b][t] = v; };
    rs_fft<N0, NL, false, false, 0, NT>(sm, twf, ld, keep);

    // common factor of the operator (kappa, |k|^e or cos), times 1/N
    const int kind0 = pick(ops.kind, f);
    switch (xop_class(kind0, P)) {
    case XOP_SINC: xpass_operator<N0, NL, NT, XOP_SINC>(spec, P, kind0, s_kx2, kyz2, line0, lines_total); break;
    case XOP_SINC_SHORT:
        xpass_operator<N0, NL, NT, XOP_SINC_SHORT>(spec, P, kind0, s_kx2, kyz2, line0, lines_total);
        break;
    case XOP_COS_SHORT:
        xpass_operator<N0, NL, NT, XOP_COS_SHORT>(spec, P, kind0, s_kx2, kyz2, line0, lines_total);
        break;
    case XOP_NABLA: xpass_operator<N0, NL, NT, XOP_NABLA>(spec, P, kind0, s_kx2, kyz2, line0, lines_total); break;
    case XOP_COS: xpass_operator<N0, NL, NT, XOP_COS>(spec, P, kind0, s_kx2, kyz2, line0, lines_total); break;
    default: xpass_operator<N0, NL, NT, XOP_ONE>(spec, P, kind0, s_kx2, kyz2, line0, lines_total); break;
    }
    auto store_to = [&](float2 *outb) {
        float2 *out = outb + (long long)line0 * N0;
        return [=](int, int, int l, int i, float2 v) {
            if (line0 + l < lines_total) out[l * N0 + i] = v;
        };
    };
    auto plain = [&](int b, int t, int, int) -> float2 { return spec[b][t]; };
    auto by_ddx = [&](int b, int t, int, int i) -> float2 { return cmul(spec[b][t], s_ddx[i]); };

    if constexpr (FAN == 2) {
        // output 0: its own inverse transform of spec dd_x(k_x); outputs 1
        // and 2: one inverse transform of spec, stored unscaled to bufs.p[1]
        // (the inverse y-pass applies their y and z multipliers)
        auto st0 = store_to(bufs.p[0]);
        rs_fft<N0, NL, false, true, 0, NT>(sm, twi, by_ddx, st0);
        auto st1 = store_to(bufs.p[1]);
        rs_fft<N0, NL, false, true, 0, NT>(sm, twi, plain, st1);
    } else if constexpr (FAN == 0) {
        const int axis = pick(ops.axis, f);
        const bool mul_dd = kind0 == OP_GRAD_POS || kind0 == OP_GRAD_NEG || kind0 == OP_SHIFT_NEG;
        auto st = store_to(pick(bufs.p, f));
        if constexpr (!line_in_warp<N0, NL, NT, false>()) {
            // other lengths (several butterflies of different lines per
            // thread) keep one inverse with the choice made per value: their
            // registers are already near the limit
            auto ld2 = [&](int b, int t, int l, int i) -> float2 {
                if (!mul_dd) return spec[b][t];
                if (axis != 0) return cmul(spec[b][t], s_lm[f][l]);
                return cmul(spec[b][t], s_ddx[i]);
            };
            rs_fft<N0, NL, false, true, 0, NT>(sm, twi, ld2, st);
        } else if (!mul_dd) {
            rs_fft<N0, NL, false, true, 0, NT>(sm, twi, plain, st);
        } else {
            // multiplier dd_x(k_x) (axis 0) or the line's constant (axis 1, 2)
            const float2 *tab = axis == 0 ? s_ddx : s_lm[f];
            const int xs = axis == 0 ? 1 : 0, ls = axis == 0 ? 0 : 1;
            auto by_tab = [&](int b, int t, int l, int i) -> float2 { return cmul(spec[b][t], tab[i * xs + l * ls]); };
            rs_fft<N0, NL, false, true, 0, NT>(sm, twi, by_tab, st);
        }
    } else {
        // FAN == 1.  An output whose operator table runs along x gets its own
        // inverse transform.  Every other output is the inverse transform of
        // spec times a constant per x line (s_lm): they share one inverse
        // transform and are scaled as they are stored.
        int shared_mask = 0;
        for (int o = 0; o < ops.n; ++o) {
            const int axis = pick(ops.axis, o);
            const int ko = pick(ops.kind, o);
            const bool mul_dd = ko == OP_GRAD_POS || ko == OP_GRAD_NEG || ko == OP_SHIFT_NEG;
            if (!(mul_dd && axis == 0)) {
                shared_mask |= 1 << o;
                continue;
            }
            auto st2 = store_to(pick(bufs.p, o));
            rs_fft<N0, NL, false, true, 0, NT>(sm, twi, by_ddx, st2);
        }
        if (shared_mask) {
            auto st3 = [&](int, int, int l, int i, float2 v) {
                if (line0 + l >= lines_total) return;
#pragma unroll
                for (int o = 0; o < 3; ++o)
                    if (shared_mask & (1 << o))
                        (bufs.p[o] + (long long)line0 * N0)[l * N0 + i] = cmul(v, s_lm[o][l]);
            };
            rs_fft<N0, NL, false, true, 0, NT>(sm, twi, plain, st3);
        }
    }
}

// ---------------------------------------------------------------------------
// z-tiles: TX = 2*PL consecutive x at one y, all z; hand-off register (b, t)
// holds packed element (l, z) = (f(x0+2l), f(x0+2l+1)).
// ---------------------------------------------------------------------------
template <int N2, int PL_>
struct ZTile {
    static constexpr int PL = PL_;
    static constexpr int TX = 2 * PL;
    static constexpr int NT = ks_threads(N2, PL);
    using SH = HandShape<N2, PL, NT>;
};

// packed C2R input: element z of packed line l from the z-half spectrum
template <int N2>
__device__ __forceinline__ float2 zpack_load(const float2 *__restrict__ H, const Geom &g, int x0, int y, int l, int z) {
    constexpr int N2h = N2 / 2 + 1;
    int k = z;
    bool cj = false;
    if (z >= N2h) { k = N2 - z; cj = true; }
    const int xa = x0 + 2 * l;
    const float2 *h = H + ((long long)k * g.N1 + y) * g.N0;
    float2 A, B;
    if (g.vec2 && xa + 1 < g.N0) {
        const float4 q = *reinterpret_cast<const float4 *>(h + xa);
        A = make_float2(q.x, q.y);
        B = make_float2(q.z, q.w);
    } else {
        A = xa < g.N0 ? h[xa] : make_float2(0.f, 0.f);
        B = xa + 1 < g.N0 ? h[xa + 1] : make_float2(0.f, 0.f);
    }
    if (cj) { A.y = -A.y; B.y = -B.y; }
    if (k == 0 || 2 * k == N2) { A.y = 0.f; B.y = 0.f; }
    return make_float2(A.x - B.y, A.y + B.x);
}

// Rows kz = 0 .. N2/2 of the z-half spectra of the tile's packed lines
// (packed layout z*PL + l in s), unpacked into the two real columns' spectra
// as zstore_r2c does and stored as one 16-byte pair per (row, line).  Thread
// q keeps line q % PL and takes rows q / PL + it KS (KS = NT / PL rows per
// sweep), so its column and row stride are fixed and only the last sweep is
// partial.  N0 is even on this path: a pair is in range whole or not at all.
template <int N2, int PL>
__device__ __forceinline__ void zstore_r2c_tile(const float2 *s, float2 *__restrict__ H, const Geom &g, int x0, int y) {
    constexpr int NT = ZTile<N2, PL>::NT, ROWS = N2 / 2 + 1;
    static_assert(NT % PL == 0, "whole rows per sweep");
    constexpr int KS = NT / PL, SWEEPS = (ROWS + KS - 1) / KS;
    const int l = threadIdx.x % PL, k0 = threadIdx.x / PL;
    const int xa = x0 + 2 * l;
    if (xa >= g.N0) return;
    float2 *h = H + ((long long)k0 * g.N1 + y) * g.N0 + xa;
    const long long step = (long long)KS * g.N1 * g.N0;
#pragma unroll
    for (int it = 0; it < SWEEPS; ++it) {
        const int k = k0 + it * KS;
        if ((it + 1) * KS > ROWS && k >= ROWS) break;
        const float2 Zk = s[k * PL + l];
        const int nk = k == 0 ? 0 : N2 - k;
        const float2 Zn = s[nk * PL + l];
        const float2 A = make_float2(0.5f * (Zk.x + Zn.x), 0.5f * (Zk.y - Zn.y));
        const float2 B = make_float2(0.5f * (Zk.y + Zn.y), -0.5f * (Zk.x - Zn.x));
        *reinterpret_cast<float4 *>(h + it * step) = make_float4(A.x, A.y, B.x, B.y);
    }
}

// forward transform of the hand-off registers, then unpack and store the
// z-half spectrum (two real columns per packed line)
template <int N2, int PL, class Hold>
__device__ __forceinline__ void zforward_store(float2 *sm, const float2 *__restrict__ tw, Hold &hold, float2 *H,
                                               const Geom &g, int x0, int y) {
    constexpr int NT = ZTile<N2, PL>::NT;
    using SL = StageShape<N2, PL, false, RPlan<N2, false>::M - 1, NT>;   // forward last stage
    float2 outv[SL::MAXB][SL::R];
    int outi[SL::MAXB];
    auto ld = [&](int b, int t, int, int) -> float2 { return hold[b][t]; };
    auto st = [&](int b, int t, int l, int i, float2 v) {
        outv[b][t] = v;
        if (t == 0) outi[b] = i * PL + l;   // element i + t*NS of line l sits at outi + t*NS*PL
    };
    rs_fft<N2, PL, true, false, 0, NT>(sm, tw, ld, st);
    __syncthreads();   // every thread has read its last-stage inputs from the tile
    constexpr int NSL = RPlan<N2, false>::NS(RPlan<N2, false>::M - 1);
#pragma unroll
    for (int b = 0; b < SL::MAXB; ++b) {
        const int gg = threadIdx.x + b * NT;
        if (!(SL::TOT % NT == 0 || gg < SL::TOT)) continue;
#pragma unroll
        for (int t = 0; t < SL::R; ++t) sm[outi[b] + t * NSL * PL] = outv[b][t];
    }
    __syncthreads();
    zstore_r2c_tile<N2, PL>(sm, H, g, x0, y);
}

// write hand-off registers into the tile (packed layout z*PL + l)
template <int N2, int PL, class Hold>
__device__ __forceinline__ void hold_to_smem(float2 *sm, Hold &hold) {
    constexpr int NT = ZTile<N2, PL>::NT;
    using SH = typename ZTile<N2, PL>::SH;
#pragma unroll
    for (int b = 0; b < SH::MAXB; ++b)
#pragma unroll
        for (int t = 0; t < SH::R; ++t) {
            int l, i;
            if (hand_pos<N2, PL, true, NT>(b, t, l, i)) sm[i * PL + l] = hold[b][t];
        }
}
template <int N2, int PL, class Hold>
__device__ __forceinline__ void smem_to_hold(const float2 *sm, Hold &hold) {
    constexpr int NT = ZTile<N2, PL>::NT;
    using SH = typename ZTile<N2, PL>::SH;
#pragma unroll
    for (int b = 0; b < SH::MAXB; ++b)
#pragma unroll
        for (int t = 0; t < SH::R; ++t) {
            int l, i;
            if (hand_pos<N2, PL, true, NT>(b, t, l, i)) hold[b][t] = sm[i * PL + l];
        }
}

// ---------------------------------------------------------------------------
// Asynchronous staging of read-only physics inputs: every thread copies the
// values of the cells it will update into a thread-private slice of shared
// memory (index (b*R + t)*NT + tid) before the inverse transform, so
// the loads are in flight while the transform computes.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// wait until at most N of this thread's most recent commit groups are pending
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---------------------------------------------------------------------------
// Tensor-memory-accelerator (TMA) staging: one thread issues a bulk tensor
// copy of a whole tile (a real field's TX x N2 cells at one y, or the N2/2+1
// half-spectrum rows of TX columns) into shared memory; the block waits on
// an mbarrier for the bytes to land.  The copy takes no registers, address
// arithmetic or load instructions from the other threads.  Tensor maps
// cover this GPU's own memory only; no multicast.
//
// Every wait is bounded: after kTmaSpinLimit polls it gives up, sets bit 1
// of *err (the host turns that into KW_ERR_TIMEOUT) and lets the block run
// on, so the kernel always finishes.
// ---------------------------------------------------------------------------
constexpr unsigned kTmaSpinLimit = 1u << 22;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// generic-proxy accesses of a shared-memory region, ordered before an
// async-proxy (TMA) write of it
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
            smem_u32(dst)),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
// wait for phase `phase` of *bar to complete, at most kTmaSpinLimit polls
__device__ __forceinline__ void mbar_wait(uint64_t *bar, unsigned phase, int *err) {
    const unsigned a = smem_u32(bar);
    for (unsigned i = 0; i < kTmaSpinLimit; ++i) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return;
    }
    if (err) atomicOr(err, 2);
}
// one real field's tile (TX x N2 cells at row y) into dst, [z][x] order
template <int N2, int TX>
__device__ __forceinline__ void tma_field(float2 *dst, const CUtensorMap *map, int zbox, int x0, int y, uint64_t *bar) {
    mbar_expect_tx(bar, (unsigned)(TX * N2 * sizeof(float)));
    for (int z = 0; z < N2; z += zbox) tma_load_3d(reinterpret_cast<float *>(dst) + z * TX, map, x0, y, z, bar);
}
// half-spectrum rows kz = 0 .. N2/2 of TX columns at row y into dst, [kz][x],
// in tma_row_boxes(N2) boxes (every box's bytes count, filled rows included)
template <int N2, int TX>
__device__ __forceinline__ void tma_rows(float2 *dst, const CUtensorMap *map, int x0, int y, uint64_t *bar) {
    constexpr int NB = tma_row_boxes(N2), BR = tma_row_box(N2);
    mbar_expect_tx(bar, (unsigned)(NB * BR * TX * sizeof(float2)));
#pragma unroll
    for (int k = 0; k < NB; ++k) tma_load_3d(dst + k * BR * TX, map, x0, y, k * BR, bar);
}

template <int N2, int PL_> struct ZStage {
    using ZT = ZTile<N2, PL_>;
    using SH = typename ZT::SH;
    static constexpr int PL = ZT::PL, TX = ZT::TX, NT = ZT::NT;
    // float2 of the transform tile; it also holds the raw half-spectrum rows of
    // a prefetched input, (N2/2 + 1) rows of TX values (whole TMA boxes of
    // rows, tma_row_boxes(N2) x tma_row_box(N2)).  Rounded up to 128 bytes,
    // so the slices after it can be TMA destinations (128-byte aligned
    // shared-memory addresses).
    static constexpr int ROWS = tma_row_boxes(N2) * tma_row_box(N2) > N2 / 2 + 1 ? tma_row_boxes(N2) * tma_row_box(N2)
                                                                                 : N2 / 2 + 1;
    static constexpr int TILE = (ROWS * TX + 15) / 16 * 16;
    // the TMA path: every box of rows starts on a 128-byte boundary
    static constexpr bool TMA_OK =
        (tma_row_boxes(N2) == 1 || (tma_row_box(N2) * TX * 8) % 128 == 0) && (TX * 4) % 16 == 0;
    static constexpr int SLICE = SH::MAXB * SH::R * NT;   // float2 of one staged field
    static __device__ __forceinline__ int sidx(int b, int t) { return (b * SH::R + t) * NT + threadIdx.x; }
};

// stage one real field (pairs of cells) of this thread's hand-off elements
template <int N2, int PL>
__device__ __forceinline__ void stage_field(float2 *slice, const float *field, const Geom &g, int x0, int y) {
    using Z = ZStage<N2, PL>;
    using SH = typename Z::SH;
#pragma unroll
    for (int b = 0; b < SH::MAXB; ++b)
#pragma unroll
        for (int t = 0; t < SH::R; ++t) {
            int l, z;
            if (!hand_pos<N2, PL, true, Z::NT>(b, t, l, z)) continue;
            const int xa = x0 + 2 * l;
            if (xa >= g.N0) continue;
            cp_async8(slice + Z::sidx(b, t), field + xa + (long long)g.N0 * (y + (long long)g.N1 * z));
        }
}

// Prefetch of one z-tile's input half spectrum: rows kz = 0 .. N2/2 of the
// TX columns x0 .. x0+TX-1 at this y, into raw[kz * TX + x - x0], with
// 16-byte cp.async (two complex values; N0 is even on this path).  Issued
// while the previous component is processed, so the next inverse transform
// reads its inputs from shared memory.
template <int N2, int PL>
__device__ __forceinline__ void zraw_prefetch(float2 *raw, const float2 *__restrict__ H, const Geom &g, int x0, int y) {
    constexpr int TX = 2 * PL, CH = TX / 2, ROWS = N2 / 2 + 1;
    constexpr int NT = ks_threads(N2, PL);
    for (int q = threadIdx.x; q < ROWS * CH; q += NT) {
        const int k = q / CH, c = q - k * CH;
        const int xa = x0 + 2 * c;
        if (xa >= g.N0) continue;
        cp_async16(raw + k * TX + 2 * c, H + ((long long)k * g.N1 + y) * g.N0 + xa);
    }
}
// packed C2R input (as zpack_load) from prefetched raw rows
// Element z = j + t NB (0 <= j < NB) of the inverse transform's first stage:
// for all but at most two values of t (constants once the stage loop is
// unrolled) the row's half and the DC / Nyquist tests are known without z.
template <int N2, int PL>
__device__ __forceinline__ float2 zpack_raw(const float2 *raw, const Geom &g, int x0, int l, int z, int t) {
    constexpr int TX = 2 * PL, N2h = N2 / 2 + 1;
    constexpr int NB = N2 / RPlan<N2, true>::R(0);
    const int zlo = t * NB, zhi = t * NB + NB - 1;
    bool cj;
    if (zhi < N2h) cj = false;
    else if (zlo >= N2h) cj = true;
    else cj = z >= N2h;
    const int k = cj ? N2 - z : z;
    if (x0 + 2 * l >= g.N0) return make_float2(0.f, 0.f);
    const float4 q = *reinterpret_cast<const float4 *>(raw + k * TX + 2 * l);
    float2 A = make_float2(q.x, q.y), B = make_float2(q.z, q.w);
    if (cj) { A.y = -A.y; B.y = -B.y; }
    // k == 0 (z == 0) or 2 k == N2 (z == N2 / 2): the Hermitian part is real
    const bool edge = (zlo == 0 && z == 0) || (N2 % 2 == 0 && zlo <= N2 / 2 && N2 / 2 <= zhi && z == N2 / 2);
    if (edge) { A.y = 0.f; B.y = 0.f; }
    return make_float2(A.x - B.y, A.y + B.x);
}

// ---------------------------------------------------------------------------
// Stage U (momentum, velocity sources, forward z-transform of u); see k_stage_u.
// u is double-buffered (read a.u, write a.u_out).  grid = (ceil(N0/TX), N1, D);
// dynamic shared memory: tile + 2 staged fields.
// ---------------------------------------------------------------------------
template <int N2, int PL, bool TMA>
__global__ void __launch_bounds__(ks_threads(N2, PL), 2 * kThreads / ks_threads(N2, PL))
    ks_stage_u(StageU a, const float2 *__restrict__ tw, const __grid_constant__ StageUMaps m) {
    using Z = ZStage<N2, PL>;
    using SH = typename Z::SH;
    constexpr int TX = Z::TX, NT = Z::NT;
    static_assert(RPlan<N2, false>::M >= 2, "z-stages need two stages");
    static_assert(!TMA || ((Z::TILE * 8) % 128 == 0 && (Z::SLICE * 8) % 128 == 0 && TX * N2 / 2 <= Z::SLICE &&
                           TX * (N2 / 2 + 1) <= Z::TILE && (TX * 4) % 16 == 0),
                  "TMA staging layout");
    extern __shared__ __align__(128) float2 dsm_raw[];
    // TMA destinations must be 128-byte aligned (128 bytes of launch slack)
    float2 *dsm = TMA ? reinterpret_cast<float2 *>(dsm_raw + ((128u - (smem_u32(dsm_raw) & 127u)) & 127u) / 8)
                      : dsm_raw;
    float2 *sm = dsm;
    float2 *s_u = dsm + Z::TILE;
    float2 *s_r = s_u + Z::SLICE;
    const Geom &g = a.g;
    const int f = blockIdx.z;
    const int x0 = blockIdx.x * TX, y = blockIdx.y;
    const int t = *a.d_t;
    float *uout = a.u_out[f];
    const int ax = a.comp_axis[f];
    const float *pmlv = a.pml_sg[ax];
    const float2 *H = a.spec.p[f];
    const Med rsi = a.rho_sg_inv[f];
    auto slot = [&](int b, int tt, int l, int z) -> int { return TMA ? z * PL + l : Z::sidx(b, tt); };

    float2 hold[SH::MAXB][SH::R];
    if constexpr (TMA) {
        // spectrum rows into the tile, old u and 1/rho_sg into their slices:
        // three bulk copies issued by one thread; the transform reads the rows
        // from shared memory.  A block whose destinations fail the 128-byte
        // alignment self-check records bit 2 of *err and returns.
        __shared__ __align__(8) uint64_t bars[2];
        __shared__ int misaligned;
        const bool lead = threadIdx.x == 0;
        if (lead) {
            misaligned = ((smem_u32(sm) | smem_u32(s_u) | smem_u32(s_r)) & 127u) != 0;
            if (misaligned && m.err) atomicOr(m.err, 4);
            mbar_init(&bars[0], 1);
            mbar_init(&bars[1], 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (misaligned) return;
        const bool any_field = !a.init || rsi.arr;
        if (lead) {
            tma_rows<N2, TX>(sm, &m.spec[0] + f, x0, y, &bars[0]);
            if (any_field) {
                // one barrier for both slices: their bytes are expected together
                const unsigned bytes = (unsigned)(TX * N2 * sizeof(float)) * ((!a.init ? 1u : 0u) + (rsi.arr ? 1u : 0u));
                mbar_expect_tx(&bars[1], bytes);
                for (int z = 0; z < N2; z += m.zbox) {
                    if (!a.init) tma_load_3d(reinterpret_cast<float *>(s_u) + z * TX, &m.u[0] + f, x0, y, z, &bars[1]);
                    if (rsi.arr) tma_load_3d(reinterpret_cast<float *>(s_r) + z * TX, &m.rsi[0] + f, x0, y, z, &bars[1]);
                }
            }
        }
        mbar_wait(&bars[0], 0, m.err);
        auto ld = [&](int, int t, int l, int z) -> float2 { return zpack_raw<N2, PL>(sm, g, x0, l, z, t); };
        auto st = [&](int b, int tt, int, int, float2 v) { hold[b][tt] = v; };
        rs_fft<N2, PL, true, true, 0, NT>(sm, tw, ld, st);
        if (any_field) mbar_wait(&bars[1], 0, m.err);
    } else {
        // the first transform stage's inputs are loaded before the per-cell
        // staging is issued, so they are not queued behind it
        using S0 = StageShape<N2, PL, true, 0, NT>;
        float2 in0[S0::MAXB][S0::R];
#pragma unroll
        for (int b = 0; b < S0::MAXB; ++b) {
            const int gg = threadIdx.x + b * NT;
            if (!(S0::TOT % NT == 0 || gg < S0::TOT)) continue;
            int l, j;
            bmap<S0::NB, PL, true>(gg, l, j);
#pragma unroll
            for (int tt = 0; tt < S0::R; ++tt) in0[b][tt] = zpack_load<N2>(H, g, x0, y, l, j + tt * S0::NB);
        }
        if (!a.init) stage_field<N2, PL>(s_u, a.u[f], g, x0, y);
        if (rsi.arr) stage_field<N2, PL>(s_r, rsi.arr, g, x0, y);
        cp_async_commit();
        auto ld = [&](int b, int tt, int, int) -> float2 { return in0[b][tt]; };
        auto st = [&](int b, int tt, int, int, float2 v) { hold[b][tt] = v; };
        rs_fft<N2, PL, true, true, 0, NT>(sm, tw, ld, st);
        cp_async_wait_all();
    }

    float dscale = 0.f;
    const bool dense = dense_active(a.dense[f], t, dscale);
    const float pml_y = ax == 1 ? __ldg(pmlv + y) : 1.f;
    // cell index of element (b, t): that of its first row plus t row strides
    const long long dz = (long long)g.N0 * g.N1 * SH::NB;
#pragma unroll
    for (int b = 0; b < SH::MAXB; ++b) {
        int l, j;
        if (!hand_line<N2, PL, true, NT>(b, l, j)) continue;
        const int xa = x0 + 2 * l;
        if (xa >= g.N0) {
#pragma unroll
            for (int tt = 0; tt < SH::R; ++tt) hold[b][tt] = make_float2(0.f, 0.f);
            continue;
        }
        // the x and y PML factors are constant along this thread's line
        const float2 pmc = ax == 0 ? __ldg(reinterpret_cast<const float2 *>(pmlv + xa))   // xa even, N0 even
                                   : make_float2(pml_y, pml_y);
        const long long gi0 = xa + (long long)g.N0 * (y + (long long)g.N1 * j);
#pragma unroll
        for (int tt = 0; tt < SH::R; ++tt) {
            const int z = j + tt * SH::NB;
            const long long gi = gi0 + tt * dz;
            const float2 gr = hold[b][tt];
            const float2 ri = rsi.arr ? s_r[slot(b, tt, l, z)] : make_float2(rsi.val, rsi.val);
            float2 un;
            if (a.init) {
                un = make_float2(0.5f * a.dt * ri.x * gr.x, 0.5f * a.dt * ri.y * gr.y);
            } else {
                float2 pm = pmc;
                if (ax == 2) { const float q = __ldg(pmlv + z); pm = make_float2(q, q); }
                const float2 uo = s_u[slot(b, tt, l, z)];
                un.x = pm.x * (pm.x * uo.x - a.dt * ri.x * gr.x);
                un.y = pm.y * (pm.y * uo.y - a.dt * ri.y * gr.y);
                if (dense) {
                    const float2 F = __ldg(reinterpret_cast<const float2 *>(a.dense[f].F + gi));
                    un.x = fmaf(dscale, F.x, un.x);
                    un.y = fmaf(dscale, F.y, un.y);
                }
            }
            *reinterpret_cast<float2 *>(uout + gi) = un;
            hold[b][tt] = un;
        }
    }
    if (a.init || !a.write_spec) return;
    if (a.sparse.off && a.sparse.sig[f] && t <= a.sparse.T[f]) {
        const int tile = blockIdx.x + gridDim.x * blockIdx.y;
        const int e0 = a.sparse.off[tile], e1 = a.sparse.off[tile + 1];
        if (e1 > e0) {
            __syncthreads();
            hold_to_smem<N2, PL>(sm, hold);
            __syncthreads();
            for (int e = e0 + threadIdx.x; e < e1; e += NT) {
                const int c = a.sparse.cell[e];
                const int z = c / TX, xl = c - z * TX;
                const float v = __ldg(a.sparse.sig[f] + a.sparse.row[e] + (long long)a.sparse.nsig * (t - 1));
                float *slot = reinterpret_cast<float *>(sm + z * PL + (xl >> 1)) + (xl & 1);
                const float nv = a.sparse.mode == 0 ? v : *slot + v;
                *slot = nv;
                uout[x0 + xl + (long long)g.N0 * (y + (long long)g.N1 * z)] = nv;
            }
            __syncthreads();
            smem_to_hold<N2, PL>(sm, hold);
        }
    }
    zforward_store<N2, PL>(sm, tw, hold, a.spec.p[f], g, x0, y);
}

// ---------------------------------------------------------------------------
// Stage R (mass conservation, pressure sources, equation of state); see
// k_stage_r.  rho is double-buffered (read a.rho, write a.rho_out).  The old
// rho of every component is staged into shared memory at the start; the
// nonlinear coefficient 2 sum(rho_old) + rho0 is formed from the staged values
// during component 0 and kept in component 0's slice.
// TMA: the staged fields and the spectrum rows are brought in by bulk tensor
// copies that one thread issues (slices then hold cells in [z][x] order);
// otherwise by per-thread cp.async into thread-private slots.
// grid = (ceil(N0/TX), N1, 1); dynamic shared memory: tile + D staged fields.
// ---------------------------------------------------------------------------
template <int N2, int PL, bool TMA>
__global__ void __launch_bounds__(ks_threads(N2, PL), 2 * kThreads / ks_threads(N2, PL))
    ks_stage_r(StageR a, const float2 *__restrict__ tw, const __grid_constant__ StageRMaps m) {
    using Z = ZStage<N2, PL>;
    using SH = typename Z::SH;
    constexpr int TX = Z::TX, NT = Z::NT;
    extern __shared__ __align__(128) float2 dsm_raw[];
    // TMA destinations must be 128-byte aligned: the dynamic shared memory
    // carries 128 bytes of slack (ZStage launch size) for this
    float2 *dsm = TMA ? reinterpret_cast<float2 *>(dsm_raw + ((128u - (smem_u32(dsm_raw) & 127u)) & 127u) / 8)
                      : dsm_raw;
    float2 *sm = dsm;
    float2 *s_c = dsm + Z::TILE;        // staged mass coefficient (q or rho0)
    float2 *s_a = s_c + Z::SLICE;       // staged rho_old of the current component
    const Geom &g = a.g;
    const int x0 = blockIdx.x * TX, y = blockIdx.y;
    const int t = *a.d_t;
    const int D = a.D;
    const bool r0arr = a.rho0.arr != nullptr;
    // TMA layout invariants: the tile and each slice are whole 128-byte
    // units, a real-field box set fits a slice and the tile, the spectrum rows
    // fit the tile, and every box row is a multiple of 16 bytes
    static_assert(!TMA || ((Z::TILE * 8) % 128 == 0 && (Z::SLICE * 8) % 128 == 0 && TX * N2 / 2 <= Z::SLICE &&
                           TX * N2 / 2 <= Z::TILE && TX * (N2 / 2 + 1) <= Z::TILE && (TX * 4) % 16 == 0),
                  "TMA staging layout");
    // slot of this thread's cell (l, z) in a staged slice
    auto slot = [&](int b, int tt, int l, int z) -> int { return TMA ? z * PL + l : Z::sidx(b, tt); };
    // TMA barriers: tile (spectrum rows, rho0), slice a, slice c; phases
    __shared__ __align__(8) uint64_t bars[3];
    unsigned ph_t = 0, ph_a = 0, ph_c = 0;
    const bool lead = threadIdx.x == 0;
    const bool coef_staged = a.nonlinear || r0arr;
    // mass coefficient: q = 2 sum(rho_old) + rho0, carried between steps
    // (nonlinear), or rho0 (linear)
    if constexpr (TMA) {
        // self-check of the alignment every TMA destination needs; a block
        // that fails it records bit 2 of *err and returns without copying
        __shared__ int misaligned;
        if (lead) {
            misaligned = ((smem_u32(sm) | smem_u32(s_c) | smem_u32(s_a)) & 127u) != 0;
            if (misaligned && m.err) atomicOr(m.err, 4);
            for (int k = 0; k < 3; ++k) mbar_init(&bars[k], 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (misaligned) return;
        if (lead) {
            if (coef_staged) tma_field<N2, TX>(s_c, &m.coef, m.zbox, x0, y, &bars[2]);
            tma_field<N2, TX>(s_a, &m.rho[0], m.zbox, x0, y, &bars[1]);
            tma_rows<N2, TX>(sm, &m.spec[0], x0, y, &bars[0]);
        }
    } else {
        if (a.nonlinear) stage_field<N2, PL>(s_c, a.srho, g, x0, y);
        else if (r0arr) stage_field<N2, PL>(s_c, a.rho0.arr, g, x0, y);
        stage_field<N2, PL>(s_a, a.rho[0], g, x0, y);
        zraw_prefetch<N2, PL>(sm, a.spec.p[0], g, x0, y);
        cp_async_commit();
    }
    float dscale = 0.f;
    const bool dense = dense_active(a.dense, t, dscale);
    int e0 = 0, e1 = 0;
    if (a.sparse.off && t <= a.sparse.T[0]) {
        const int tile = blockIdx.x + gridDim.x * blockIdx.y;
        e0 = a.sparse.off[tile];
        e1 = a.sparse.off[tile + 1];
    }
    // nonlinear: rho0 for the equation of state is staged into the free
    // transform tile after the last inverse transform (unless a sparse source
    // needs the tile first)
    const bool r0_tile = Z::SLICE <= Z::TILE && a.nonlinear && r0arr && e1 <= e0;
    const bool c0_staged = a.c0.arr != nullptr;
    const bool bona_staged = a.nonlinear && a.BonA.arr != nullptr;

    float2 acc_r[SH::MAXB][SH::R], acc_d[SH::MAXB][SH::R];
#pragma unroll
    for (int b = 0; b < SH::MAXB; ++b)
#pragma unroll
        for (int tt = 0; tt < SH::R; ++tt) {
            acc_r[b][tt] = make_float2(0.f, 0.f);
            acc_d[b][tt] = make_float2(0.f, 0.f);
        }
#pragma unroll 1
    // commit groups, oldest first: {srho, rho_0, rows_0}, then per component
    // {rows_i+1} before its physics and {rho_i+1} after it; after the last
    // component's physics {c0, B/A} for the equation of state
    for (int i = 0; i < D; ++i) {
        float2 hold[SH::MAXB][SH::R];
        if constexpr (TMA) {
            mbar_wait(&bars[0], ph_t, m.err);   // rows_i in the tile
            ph_t ^= 1;
            if (i == 0 && coef_staged) {
                mbar_wait(&bars[2], ph_c, m.err);
                ph_c ^= 1;
            }
        } else {
            if (i == 0) cp_async_wait_all();
            else cp_async_wait_group<1>();   // rows_i landed; rho_i may be in flight
            __syncthreads();                 // the prefetched rows of every thread are in the tile
        }
        auto ld = [&](int, int t, int l, int z) -> float2 { return zpack_raw<N2, PL>(sm, g, x0, l, z, t); };
        auto st = [&](int b, int tt, int, int, float2 v) { hold[b][tt] = v; };
        rs_fft<N2, PL, true, true, 0, NT>(sm, tw, ld, st);
        if constexpr (TMA) {
            mbar_wait(&bars[1], ph_a, m.err);   // rho_i in slice a
            ph_a ^= 1;
        } else {
            cp_async_wait_all();             // staged rho_i (this thread's own slots)
        }
        if (i + 1 < D) {
            __syncthreads();   // every thread has read the tile
            if constexpr (TMA) {
                if (lead) {
                    fence_proxy_async();
                    tma_rows<N2, TX>(sm, &m.spec[i + 1], x0, y, &bars[0]);
                }
            } else {
                zraw_prefetch<N2, PL>(sm, a.spec.p[i + 1], g, x0, y);
                cp_async_commit();
            }
        } else if (r0_tile) {
            __syncthreads();   // every thread has read the tile
            if constexpr (TMA) {
                if (lead) {
                    fence_proxy_async();
                    tma_field<N2, TX>(sm, &m.rho0, m.zbox, x0, y, &bars[0]);
                }
            } else {
                stage_field<N2, PL>(sm, a.rho0.arr, g, x0, y);
                cp_async_commit();
            }
        }
        const int ax = a.comp_axis[i];
        const float *pmlv = a.pml[ax];
        const float pml_y = ax == 1 ? __ldg(pmlv + y) : 1.f;
        float *rout = a.rho_out[i];
        // cell index of element (b, t): that of its first row plus t row strides
        const long long dz = (long long)g.N0 * g.N1 * SH::NB;
#pragma unroll
        for (int b = 0; b < SH::MAXB; ++b) {
            int l, j;
            if (!hand_line<N2, PL, true, NT>(b, l, j)) continue;
            const int xa = x0 + 2 * l;
            if (xa >= g.N0) continue;
            const long long gi0 = xa + (long long)g.N0 * (y + (long long)g.N1 * j);
#pragma unroll
            for (int tt = 0; tt < SH::R; ++tt) {
                const int z = j + tt * SH::NB;
                const long long gi = gi0 + tt * dz;
                const int si = slot(b, tt, l, z);
                const float2 du = hold[b][tt];
                const float2 ro = s_a[si];
                const float2 coef = (a.nonlinear || r0arr) ? s_c[si] : make_float2(a.rho0.val, a.rho0.val);
                float2 pm;
                if (ax == 0) pm = __ldg(reinterpret_cast<const float2 *>(pmlv + xa));   // xa even, N0 even
                else if (ax == 1) pm = make_float2(pml_y, pml_y);
                else { const float q = __ldg(pmlv + z); pm = make_float2(q, q); }
                float2 rn;
                rn.x = pm.x * (pm.x * ro.x - a.dt * coef.x * du.x);
                rn.y = pm.y * (pm.y * ro.y - a.dt * coef.y * du.y);
                if (dense) {
                    const float2 F = __ldg(reinterpret_cast<const float2 *>(a.dense.F + gi));
                    rn.x = fmaf(dscale, F.x, rn.x);
                    rn.y = fmaf(dscale, F.y, rn.y);
                }
                *reinterpret_cast<float2 *>(rout + gi) = rn;
                acc_r[b][tt].x += rn.x;
                acc_r[b][tt].y += rn.y;
                acc_d[b][tt].x += du.x;
                acc_d[b][tt].y += du.y;
            }
        }
        // cp.async: every thread reads only its own slots, so the next
        // component (or, after the last one, c0 for the equation of state) is
        // staged into the same slice right away; TMA rewrites the whole slice,
        // so it waits until every thread has read it
        if constexpr (TMA) {
            if (i + 1 < D || c0_staged || bona_staged) __syncthreads();
            if (lead) {
                fence_proxy_async();
                if (i + 1 < D) {
                    tma_field<N2, TX>(s_a, &m.rho[i + 1], m.zbox, x0, y, &bars[1]);
                } else {
                    if (c0_staged) tma_field<N2, TX>(s_a, &m.c0, m.zbox, x0, y, &bars[1]);
                    // q is read by the mass updates only: its slice takes B/A
                    if (bona_staged) tma_field<N2, TX>(s_c, &m.bona, m.zbox, x0, y, &bars[2]);
                }
            }
        } else {
            if (i + 1 < D) {
                stage_field<N2, PL>(s_a, a.rho[i + 1], g, x0, y);
                cp_async_commit();
            } else {
                if (c0_staged) stage_field<N2, PL>(s_a, a.c0.arr, g, x0, y);
                // q is read by the mass updates only: its slice takes B/A
                if (bona_staged) stage_field<N2, PL>(s_c, a.BonA.arr, g, x0, y);
                cp_async_commit();
            }
        }
    }
    // sparse pressure sources act on every rho component (:930-962)
    {
        if (e1 > e0) {
            __syncthreads();
            hold_to_smem<N2, PL>(sm, acc_r);
            __syncthreads();
            for (int e = e0 + threadIdx.x; e < e1; e += NT) {
                const int c = a.sparse.cell[e];
                const int z = c / TX, xl = c - z * TX;
                const float v = __ldg(a.sparse.sig[0] + a.sparse.row[e] + (long long)a.sparse.nsig * (t - 1));
                const long long gi = x0 + xl + (long long)g.N0 * (y + (long long)g.N1 * z);
                float s = 0.f;
                for (int i = 0; i < D; ++i) {
                    const float nv = a.sparse.mode == 0 ? v : a.rho_out[i][gi] + v;
                    a.rho_out[i][gi] = nv;
                    s += nv;
                }
                *(reinterpret_cast<float *>(sm + z * PL + (xl >> 1)) + (xl & 1)) = s;
            }
            __syncthreads();
            smem_to_hold<N2, PL>(sm, acc_r);
        }
    }
    // equation of state (c0^2 applied to the non-spectral terms here; the
    // absorbing terms are finished in Stage P)
    const bool absorbing = a.eos == 1;
    if constexpr (TMA) {
        if (r0_tile) mbar_wait(&bars[0], ph_t, m.err);
        if (c0_staged) mbar_wait(&bars[1], ph_a, m.err);
        if (bona_staged) mbar_wait(&bars[2], ph_c, m.err);
    } else {
        if (r0_tile || c0_staged || bona_staged) cp_async_wait_all();
    }
    auto r0_at = [&](int si, long long gi) -> float2 {
        if (r0_tile) return sm[si];
        if (!a.nonlinear && r0arr) return s_c[si];
        return med2(a.rho0, gi, true, true);
    };
#pragma unroll
    for (int b = 0; b < SH::MAXB; ++b)
#pragma unroll
        for (int tt = 0; tt < SH::R; ++tt) {
            int l, z;
            if (!hand_pos<N2, PL, true, NT>(b, tt, l, z)) continue;
            const int xa = x0 + 2 * l;
            float2 pv = make_float2(0.f, 0.f);
            float2 rd = make_float2(0.f, 0.f);
            if (xa < g.N0) {
                const long long gi = xa + (long long)g.N0 * (y + (long long)g.N1 * z);
                const int si = slot(b, tt, l, z);
                const float2 sr = acc_r[b][tt];
                const float2 c = c0_staged ? s_a[si] : med2(a.c0, gi, true, true);
                pv = sr;
                if (a.nonlinear) {
                    const float2 r0 = r0_at(si, gi);
                    // next step's mass coefficient q = 2 sum(rho) + rho0
                    *reinterpret_cast<float2 *>(a.srho + gi) = make_float2(fmaf(2.f, sr.x, r0.x), fmaf(2.f, sr.y, r0.y));
                    const float2 bn = bona_staged ? s_c[si] : med2(a.BonA, gi, true, true);
                    pv.x += bona_term(bn.x, sr.x, r0.x);
                    pv.y += bona_term(bn.y, sr.y, r0.y);
                }
                pv.x *= c.x * c.x;
                pv.y *= c.y * c.y;
                if (a.eos == 2 || (absorbing && a.has_tau)) {
                    const float2 r0 = r0_at(si, gi);
                    const float2 sd = acc_d[b][tt];
                    rd = make_float2(r0.x * sd.x, r0.y * sd.y);
                }
                if (a.eos == 2) {
                    const float2 ct = med2(a.c2tau, gi, true, true);
                    pv.x = fmaf(ct.x, rd.x, pv.x);
                    pv.y = fmaf(ct.y, rd.y, pv.y);
                }
                *reinterpret_cast<float2 *>(a.p + gi) = pv;
            } else {
                acc_r[b][tt] = make_float2(0.f, 0.f);
            }
            acc_d[b][tt] = absorbing ? rd : pv;   // next forward input
        }
    if (!absorbing) {
        if (a.tr.off) {
            __syncthreads();
            hold_to_smem<N2, PL>(sm, acc_d);
            __syncthreads();
            apply_tr(sm, a.tr, g, PL, x0, y, t, a.rho_out[0], a.rho_out[1], a.rho_out[2], D, a.c0, a.p,
                     a.nonlinear ? a.srho : nullptr, a.rho0);
            __syncthreads();
            smem_to_hold<N2, PL>(sm, acc_d);
        }
        if (a.write_spec) zforward_store<N2, PL>(sm, tw, acc_d, a.spec.p[0], g, x0, y);
        return;
    }
    // absorbing: forward transforms of rho0 * sum(du) (tau term) and sum(rho)
    // (eta term).  sum(rho) waits in this thread's slots of the freed slice,
    // so only one set of values is held in registers during each transform.
#pragma unroll
    for (int b = 0; b < SH::MAXB; ++b)
#pragma unroll
        for (int tt = 0; tt < SH::R; ++tt) {
            int l = 0, z = 0;
            if (TMA && !hand_pos<N2, PL, true, NT>(b, tt, l, z)) continue;
            s_a[slot(b, tt, l, z)] = acc_r[b][tt];
        }
    int out = 0;
#pragma unroll 1
    for (int term = 0; term < 2; ++term) {
        if ((term == 0 && !a.has_tau) || (term == 1 && !a.has_eta)) continue;
        float2 src[SH::MAXB][SH::R];
#pragma unroll
        for (int b = 0; b < SH::MAXB; ++b)
#pragma unroll
            for (int tt = 0; tt < SH::R; ++tt) {
                int l = 0, z = 0;
                if (TMA && !hand_pos<N2, PL, true, NT>(b, tt, l, z)) { src[b][tt] = make_float2(0.f, 0.f); continue; }
                src[b][tt] = term == 0 ? acc_d[b][tt] : s_a[slot(b, tt, l, z)];
            }
        zforward_store<N2, PL>(sm, tw, src, pick(a.spec.p, out++), g, x0, y);
    }
}

// ---------------------------------------------------------------------------
// Stage P: p = p_partial + c0^2 tau A1 - c0^2 eta A2, time reversal, forward z of p.
// ---------------------------------------------------------------------------
template <int N2, int PL, bool TMA>
__global__ void __launch_bounds__(ks_threads(N2, PL), 2 * kThreads / ks_threads(N2, PL))
    ks_stage_p(StageP a, const float2 *__restrict__ tw, const __grid_constant__ StagePMaps m) {
    using Z = ZStage<N2, PL>;
    using SH = typename Z::SH;
    constexpr int TX = Z::TX, NT = Z::NT;
    static_assert(!TMA || ((Z::TILE * 8) % 128 == 0 && (Z::SLICE * 8) % 128 == 0 && TX * N2 / 2 <= Z::SLICE &&
                           TX * (N2 / 2 + 1) <= Z::TILE && (TX * 4) % 16 == 0),
                  "TMA staging layout");
    extern __shared__ __align__(128) float2 dsm_raw[];
    // TMA destinations must be 128-byte aligned (128 bytes of launch slack)
    float2 *dsm = TMA ? reinterpret_cast<float2 *>(dsm_raw + ((128u - (smem_u32(dsm_raw) & 127u)) & 127u) / 8)
                      : dsm_raw;
    float2 *sm = dsm;
    float2 *const s_w0 = dsm + Z::TILE, *const s_w1 = dsm + Z::TILE + Z::SLICE;
    const Geom &g = a.g;
    const int x0 = blockIdx.x * TX, y = blockIdx.y;
    const int t = *a.d_t;
    auto slot = [&](int b, int tt, int l, int z) -> int { return TMA ? z * PL + l : Z::sidx(b, tt); };
    // TMA barriers: tile rows, slice 0, slice 1, and their phases
    __shared__ __align__(8) uint64_t bars[3];
    __shared__ int misaligned;
    unsigned ph_t = 0, ph_0 = 0, ph_1 = 0;
    const bool lead = threadIdx.x == 0;
    // the terms' spectra are spec[0 .. nterm-1]; term k's per-cell weight
    // (c0^2 tau or c0^2 eta) is staged into slice k at the start, its rows
    // are prefetched into the tile while term k-1 is applied, and p is staged
    // into the slice that is free first
    // terms in order tau, eta; term k's weight is w0 / w1 in slice s_w0 /
    // s_w1 (selects, not arrays, so nothing is indexed at run time)
    const int nterm = (a.has_tau ? 1 : 0) + (a.has_eta ? 1 : 0);
    const Med w0 = a.has_tau ? a.c2tau : a.c2eta, w1 = a.c2eta;
    float2 *s_p = nterm == 2 ? s_w0 : s_w1;
    if constexpr (TMA) {
        // a block whose destinations fail the 128-byte alignment self-check
        // records bit 2 of *err and returns
        if (lead) {
            misaligned = ((smem_u32(sm) | smem_u32(s_w0) | smem_u32(s_w1)) & 127u) != 0;
            if (misaligned && m.err) atomicOr(m.err, 4);
            for (int k = 0; k < 3; ++k) mbar_init(&bars[k], 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (misaligned) return;
        if (lead) {
            if (nterm > 0 && w0.arr) tma_field<N2, TX>(s_w0, &m.w0, m.zbox, x0, y, &bars[1]);
            if (nterm > 1 && w1.arr) tma_field<N2, TX>(s_w1, &m.w1, m.zbox, x0, y, &bars[2]);
            if (nterm < 2) tma_field<N2, TX>(s_p, &m.p, m.zbox, x0, y, &bars[2]);
            if (nterm > 0) tma_rows<N2, TX>(sm, &m.spec[0], x0, y, &bars[0]);
        }
    } else {
        if (nterm > 0 && w0.arr) stage_field<N2, PL>(s_w0, w0.arr, g, x0, y);
        if (nterm > 1 && w1.arr) stage_field<N2, PL>(s_w1, w1.arr, g, x0, y);
        if (nterm < 2) stage_field<N2, PL>(s_p, a.p, g, x0, y);
        if (nterm > 0) zraw_prefetch<N2, PL>(sm, a.spec.p[0], g, x0, y);
        cp_async_commit();
    }
    float2 acc[SH::MAXB][SH::R];
#pragma unroll
    for (int b = 0; b < SH::MAXB; ++b)
#pragma unroll
        for (int tt = 0; tt < SH::R; ++tt) acc[b][tt] = make_float2(0.f, 0.f);
    // commit groups, oldest first: {weights, p (one term), rows_0},
    // {rows_1}, {p (two terms)}
#pragma unroll 1
    for (int k = 0; k < nterm; ++k) {
        const int term = (k == 0 && a.has_tau) ? 0 : 1;
        float2 hold[SH::MAXB][SH::R];
        if constexpr (TMA) {
            mbar_wait(&bars[0], ph_t, m.err);   // rows_k in the tile
            ph_t ^= 1;
        } else {
            if (k == 0) cp_async_wait_all();
            else cp_async_wait_group<1>();   // rows_1 landed; p may be in flight
            __syncthreads();                 // the prefetched rows of every thread are in the tile
        }
        auto ld = [&](int, int t, int l, int z) -> float2 { return zpack_raw<N2, PL>(sm, g, x0, l, z, t); };
        auto st = [&](int b, int tt, int, int, float2 v) { hold[b][tt] = v; };
        rs_fft<N2, PL, true, true, 0, NT>(sm, tw, ld, st);
        if (k + 1 < nterm) {
            __syncthreads();   // every thread has read the tile
            if constexpr (TMA) {
                if (lead) {
                    fence_proxy_async();
                    tma_rows<N2, TX>(sm, &m.spec[1], x0, y, &bars[0]);
                }
            } else {
                zraw_prefetch<N2, PL>(sm, a.spec.p[k + 1], g, x0, y);
                cp_async_commit();
            }
        }
        if constexpr (TMA) {
            // term k's weights in slice k
            if (k == 0 && w0.arr) { mbar_wait(&bars[1], ph_0, m.err); ph_0 ^= 1; }
            if (k == 1 && w1.arr) { mbar_wait(&bars[2], ph_1, m.err); ph_1 ^= 1; }
        }
        const Med w = k == 0 ? w0 : w1;
        const float2 *sw = k == 0 ? s_w0 : s_w1;
        const float sg = term == 0 ? 1.f : -1.f;
#pragma unroll
        for (int b = 0; b < SH::MAXB; ++b)
#pragma unroll
            for (int tt = 0; tt < SH::R; ++tt) {
                int l, z;
                if (!hand_pos<N2, PL, true, NT>(b, tt, l, z)) continue;
                const int xa = x0 + 2 * l;
                if (xa >= g.N0) continue;
                const float2 wv = w.arr ? sw[slot(b, tt, l, z)] : make_float2(w.val, w.val);
                acc[b][tt].x = fmaf(sg * wv.x, hold[b][tt].x, acc[b][tt].x);
                acc[b][tt].y = fmaf(sg * wv.y, hold[b][tt].y, acc[b][tt].y);
            }
        if (k == 0 && nterm == 2) {
            if constexpr (TMA) {
                // slice 0's weights are consumed by every thread: p goes there
                __syncthreads();
                if (lead) {
                    fence_proxy_async();
                    tma_field<N2, TX>(s_p, &m.p, m.zbox, x0, y, &bars[1]);
                }
            } else {
                // slice 0's weights are consumed (this thread's own slots): p goes there
                stage_field<N2, PL>(s_p, a.p, g, x0, y);
                cp_async_commit();
            }
        }
    }
    if constexpr (TMA) {
        if (nterm == 2) mbar_wait(&bars[1], ph_0, m.err);
        else mbar_wait(&bars[2], ph_1, m.err);
    } else {
        cp_async_wait_all();
    }
    const long long dz = (long long)g.N0 * g.N1 * SH::NB;
#pragma unroll
    for (int b = 0; b < SH::MAXB; ++b) {
        int l, j;
        if (!hand_line<N2, PL, true, NT>(b, l, j)) continue;
        const int xa = x0 + 2 * l;
        const long long gi0 = xa + (long long)g.N0 * (y + (long long)g.N1 * j);
#pragma unroll
        for (int tt = 0; tt < SH::R; ++tt) {
            const int z = j + tt * SH::NB;
            float2 pv = make_float2(0.f, 0.f);
            if (xa < g.N0) {
                const float2 pp = s_p[slot(b, tt, l, z)];
                pv.x = pp.x + acc[b][tt].x;
                pv.y = pp.y + acc[b][tt].y;
                *reinterpret_cast<float2 *>(a.p + gi0 + tt * dz) = pv;
            }
            acc[b][tt] = pv;
        }
    }
    if (a.tr.off) {
        __syncthreads();
        hold_to_smem<N2, PL>(sm, acc);
        __syncthreads();
        apply_tr(sm, a.tr, g, PL, x0, y, t, a.rho[0], a.rho[1], a.rho[2], a.D, a.c0, a.p, a.srho, a.rho0);
        __syncthreads();
        smem_to_hold<N2, PL>(sm, acc);
    }
    if (a.write_spec) zforward_store<N2, PL>(sm, tw, acc, a.spec.p[0], g, x0, y);
}

// ---------------------------------------------------------------------------
// plain z-transforms (N2 * PL float2 of dynamic shared memory)
// ---------------------------------------------------------------------------
template <int N2, int PL>
__global__ void __launch_bounds__(ks_threads(N2, PL), 2 * kThreads / ks_threads(N2, PL))
    ks_zr2c(const float *__restrict__ R, float2 *H, Geom g, const float2 *__restrict__ tw) {
    using ZT = ZTile<N2, PL>;
    using SH = typename ZT::SH;
    constexpr int TX = ZT::TX, NT = ZT::NT;
    extern __shared__ float2 sm[];   // N2 * PL
    const int x0 = blockIdx.x * TX, y = blockIdx.y;
    float2 hold[SH::MAXB][SH::R];
#pragma unroll
    for (int b = 0; b < SH::MAXB; ++b)
#pragma unroll
        for (int tt = 0; tt < SH::R; ++tt) {
            int l, z;
            hold[b][tt] = make_float2(0.f, 0.f);
            if (!hand_pos<N2, PL, true, NT>(b, tt, l, z)) continue;
            const int xa = x0 + 2 * l;
            if (xa >= g.N0) continue;
            const long long gi = xa + (long long)g.N0 * (y + (long long)g.N1 * z);
            hold[b][tt] = ld2(R, gi, xa + 1 < g.N0, g.vec2);
        }
    zforward_store<N2, PL>(sm, tw, hold, H, g, x0, y);
}

template <int N2, int PL>
__global__ void __launch_bounds__(ks_threads(N2, PL), 2 * kThreads / ks_threads(N2, PL))
    ks_zc2r(const float2 *__restrict__ H, float *R, Geom g, const float2 *__restrict__ tw) {
    using ZT = ZTile<N2, PL>;
    constexpr int TX = ZT::TX, NT = ZT::NT;
    extern __shared__ float2 sm[];   // N2 * PL
    const int x0 = blockIdx.x * TX, y = blockIdx.y;
    auto ld = [&](int, int, int l, int z) -> float2 { return zpack_load<N2>(H, g, x0, y, l, z); };
    auto st = [&](int, int, int l, int z, float2 v) {
        const int xa = x0 + 2 * l;
        if (xa >= g.N0) return;
        const long long gi = xa + (long long)g.N0 * (y + (long long)g.N1 * z);
        st2(R, gi, v, xa + 1 < g.N0, g.vec2);
    };
    rs_fft<N2, PL, true, true, 0, NT>(sm, tw, ld, st);
}

}  // namespace kw
