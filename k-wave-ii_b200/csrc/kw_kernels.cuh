// kw_kernels.cuh -- transform passes and fused physics stages of the k-space loop.
//
// Layout in HBM.  Internally every grid is 3-D (N0, N1, N2) with axis 0
// contiguous (MATLAB column-major x).  A 3-D problem maps (Nx, Ny, Nz) to
// (N0, N1, N2); a 2-D problem maps (Nx, Ny) to (Nx, 1, Ny) so the same code
// serves both.  Real fields hold N0*N1*N2 floats.  Spectra are "z-half"
// spectra: the real-to-complex axis is axis 2, so a spectrum holds
// N0*N1*N2h complex values, N2h = N2/2 + 1, element (x, y, kz) at
// x + N0*(y + N1*kz).  Axis 0 stays contiguous in every layout, so every
// pass reads and writes whole rows of axis 0.
//
// One spectral operator application real(ifftn(op .* fftn(f))) is:
//   z-stage (R2C along axis 2, fused into the kernel that produces f)
//   y-pass forward (C2C along axis 1)
//   x-pass: forward C2C along axis 0, multiply by op (and 1/N), inverse C2C
//   y-pass inverse
//   z-stage (C2R along axis 2, fused into the kernel that consumes the result)
//
// Real-to-complex and complex-to-real along axis 2 pack two neighbouring
// axis-0 columns into one complex line (z = a + i b) so every line transform
// is a full complex transform.
#pragma once

#include <cuda.h>   // CUtensorMap (the type only; maps are encoded through the runtime's driver entry point)

#include "kw_fft.cuh"

namespace kw {

struct Geom {
    int N0, N1, N2, N2h;
    long long N;      // N0*N1*N2
    long long Nh;     // N0*N1*N2h
    int vec2;         // N0 even: pairs (x, x+1) with x even are 8/16-byte aligned
};

struct Spec4 { float2 *p[4]; };

// Element i of a small kernel-parameter array, read with constant indices
// only.  A run-time index into a parameter array makes every thread copy the
// whole parameter struct to local memory at kernel start; a chain of selects
// reads the parameter bank directly.
template <class T, int K>
__device__ __forceinline__ T pick(const T (&a)[K], int i) {
    T r = a[0];
#pragma unroll
    for (int k = 1; k < K; ++k)
        if (i == k) r = a[k];
    return r;
}

// Tile transform in the interleaved layout (element (l, i) at s[i*nl + l]):
// compile-time plan when the axis length N is a template argument, the
// runtime radix loop otherwise (N == 0).
template <int N, int NL, bool INV>
__device__ __forceinline__ void tile_fft_il(float2 *s, const AxisFFT &ax, int nl) {
    if constexpr (N > 0) fft_static<N, NL, INV, true>(s, ax.tw);
    else fft_tile<INV>(s, ax, nl, nl, 1, true);
}

// ---- scalar-or-array medium quantity -------------------------------------
struct Med {
    const float *arr;
    float val;
};
__device__ __forceinline__ float2 med2(const Med &m, long long gi, bool two, bool vec) {
    if (!m.arr) return make_float2(m.val, m.val);
    if (two && vec) return __ldg(reinterpret_cast<const float2 *>(m.arr + gi));
    return make_float2(__ldg(m.arr + gi), two ? __ldg(m.arr + gi + 1) : 0.f);
}
__device__ __forceinline__ float2 ld2(const float *p, long long gi, bool two, bool vec) {
    if (two && vec) return *reinterpret_cast<const float2 *>(p + gi);
    return make_float2(p[gi], two ? p[gi + 1] : 0.f);
}
__device__ __forceinline__ void st2(float *p, long long gi, float2 v, bool two, bool vec) {
    if (two && vec) { *reinterpret_cast<float2 *>(p + gi) = v; return; }
    p[gi] = v.x;
    if (two) p[gi + 1] = v.y;
}

// TMA copies of half-spectrum rows: a box holds at most 256 rows, so the
// N2/2 + 1 rows of one z-tile come in tma_row_boxes(N2) boxes of
// tma_row_box(N2) rows each (the last may reach past the spectrum; its
// out-of-range rows are filled and never read)
__host__ __device__ constexpr int tma_row_boxes(int n2) { return (n2 / 2 + 1 + 255) / 256; }
__host__ __device__ constexpr int tma_row_box(int n2) {
    return (n2 / 2 + 1 + tma_row_boxes(n2) - 1) / tma_row_boxes(n2);
}

// ---- spectral operators ----------------------------------------------------
// OP_SHIFT_NEG: exp(-i k d / 2) along one axis, no kappa -- the shift of a
// staggered velocity component onto the regular grid
enum OpKind {
    OP_GRAD_POS = 0, OP_GRAD_NEG = 1, OP_NABLA1 = 2, OP_NABLA2 = 3, OP_SRC_KAPPA = 4, OP_IDENT = 5, OP_SHIFT_NEG = 6
};

struct OpParams {
    const float2 *dd_pos[3];   // i k exp(+i k d/2) per axis, FFT order, Hermitian part
    const float2 *dd_neg[3];   // i k exp(-i k d/2)
    const float2 *sh_neg[3];   // exp(-i k d/2) (1 without staggering), Hermitian part
    const float *k2[3];        // k_i^2 per axis, FFT order
    float kappa_a;             // c_ref * dt / 2
    int use_kspace;
    // kappa_a^2 max |k|^2 <= 1: the k-space series to a^10 are exact to FP32
    // (first omitted terms a^12 / 13! and a^12 / 12! below 2.1e-9)
    int short_series;
    float nabla1_exp, nabla2_exp;  // alpha_power - 2, alpha_power - 1
    float scale;               // 1 / (N0 N1 N2)
    // medium.alpha_filter on the z-half spectrum (Hermitian part, FFT order,
    // element (x, y, kz) at x + N0 (y + N1 kz)) multiplying both absorption
    // operators; NULL when absent
    const float *filt;
    int n0, n1;
};

struct OpSet {
    int n;
    int kind[3];
    int axis[3];
};

// x^e for x > 0 as 2^(e log2 x) with the PTX approximate base-2 logarithm
// and exponential.  The logarithm's absolute error (about 2^-22) is
// independent of the magnitude of x, so the result's relative error stays
// near 1e-6 over the whole wavenumber range, far inside the 1e-4 parity
// bound, at a handful of instructions instead of a full powf.
__device__ __forceinline__ float pow_pos(float x, float e) {
    float l, r;
    asm("lg2.approx.f32 %0, %1;" : "=f"(l) : "f"(x));
    asm("ex2.approx.f32 %0, %1;" : "=f"(r) : "f"(e * l));
    return r;
}
// B/A (sum rho)^2 / (2 rho0), the nonlinear term of the equation of state
// (kspaceFirstOrder3D.m:996-1015).  The quotient uses the approximate
// division (reciprocal and multiply, within 2 ulp), whose error is far below
// the 1e-4 parity bound and which avoids the IEEE division sequence.
__device__ __forceinline__ float bona_term(float bona, float sr, float r0) {
    return __fdividef(bona * sr * sr, 2.f * r0);
}
__device__ __forceinline__ float pow_k(float km, float e) {
    // MATLAB: k.^e with inf -> 0 (createAbsorptionVariables.m:40-52)
    if (km == 0.f) return e > 0.f ? 0.f : (e == 0.f ? 1.f : 0.f);
    return pow_pos(km, e);
}

__device__ __forceinline__ float2 eval_op(const OpParams &P, int kind, int axis, int ix, int iy, int iz) {
    const float k2 = __ldg(P.k2[0] + ix) + __ldg(P.k2[1] + iy) + __ldg(P.k2[2] + iz);
    const float km = sqrtf(k2);
    switch (kind) {
        case OP_GRAD_POS:
        case OP_GRAD_NEG: {
            float kap = 1.f;
            if (P.use_kspace && km > 0.f) {
                const float a = P.kappa_a * km;
                kap = sinf(a) / a;
            }
            const int i = axis == 0 ? ix : (axis == 1 ? iy : iz);
            const float2 d = __ldg((kind == OP_GRAD_POS ? P.dd_pos[axis] : P.dd_neg[axis]) + i);
            return cscale(d, kap * P.scale);
        }
        case OP_SHIFT_NEG: {
            const int i = axis == 0 ? ix : (axis == 1 ? iy : iz);
            return cscale(__ldg(P.sh_neg[axis] + i), P.scale);
        }
        case OP_NABLA1:
        case OP_NABLA2: {
            float v = pow_k(km, kind == OP_NABLA1 ? P.nabla1_exp : P.nabla2_exp) * P.scale;
            if (P.filt) v *= __ldg(P.filt + ix + (long long)P.n0 * (iy + (long long)P.n1 * iz));
            return make_float2(v, 0.f);
        }
        case OP_SRC_KAPPA: {
            const float c = P.use_kspace ? cosf(P.kappa_a * km) : 1.f;
            return make_float2(c * P.scale, 0.f);
        }
        default: return make_float2(P.scale, 0.f);
    }
}

// ---------------------------------------------------------------------------
// y-pass: C2C along axis 1 of a spectrum, in place.  Tile = TY consecutive x
// at one kz; lines interleaved (x fastest) so loads are coalesced rows.
// grid = (ceil(N0/TY), N2h, nfields)
// ---------------------------------------------------------------------------
template <bool INV, int N1S, int TYS>
__global__ void __launch_bounds__(kThreads, 3) k_ypass(Spec4 bufs, Geom g, AxisFFT ax, int TYrt) {
    extern __shared__ float2 sm[];
    const int N1 = N1S ? N1S : g.N1;
    const int TY = TYS ? TYS : TYrt;
    float2 *buf = bufs.p[blockIdx.z];
    const int x0 = blockIdx.x * TY;
    const long long base = (long long)blockIdx.y * N1 * g.N0;
    const bool vec = g.vec2 && (TY % 2 == 0) && (x0 + TY <= g.N0);
    if (vec) {
        const int half = TY / 2, tot2 = half * N1;
#pragma unroll 4
        for (int q = threadIdx.x; q < tot2; q += kThreads) {
            const int c2 = q % half, y = q / half;
            *reinterpret_cast<float4 *>(sm + y * TY + 2 * c2) =
                *reinterpret_cast<const float4 *>(buf + base + (long long)y * g.N0 + x0 + 2 * c2);
        }
    } else {
        const int tot = TY * N1;
        for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
            const int l = idx % TY, y = idx / TY, x = x0 + l;
            sm[idx] = x < g.N0 ? buf[base + (long long)y * g.N0 + x] : make_float2(0.f, 0.f);
        }
    }
    __syncthreads();
    tile_fft_il<N1S, TYS, INV>(sm, ax, TY);
    if (vec) {
        const int half = TY / 2, tot2 = half * N1;
#pragma unroll 4
        for (int q = threadIdx.x; q < tot2; q += kThreads) {
            const int c2 = q % half, y = q / half;
            *reinterpret_cast<float4 *>(buf + base + (long long)y * g.N0 + x0 + 2 * c2) =
                *reinterpret_cast<const float4 *>(sm + y * TY + 2 * c2);
        }
    } else {
        const int tot = TY * N1;
        for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
            const int l = idx % TY, y = idx / TY, x = x0 + l;
            if (x < g.N0) buf[base + (long long)y * g.N0 + x] = sm[idx];
        }
    }
}

// ---------------------------------------------------------------------------
// x-pass: forward C2C along axis 0, operator, inverse C2C, in place.
// Lines (y, kz) are contiguous rows of N0 complex values.
//   fanout == 0: field f = blockIdx.z gets operator ops[f]
//   fanout == 1: field 0 is transformed once and ops[0..n-1] write fields 0..n-1
// grid = (ceil(N1*N2h / NL), 1, fanout ? 1 : nfields)
// ---------------------------------------------------------------------------
template <int N0S, int NLS>
__global__ void __launch_bounds__(kThreads, 3) k_xpass(Spec4 bufs, Geom g, AxisFFT ax, int NLrt, OpParams P,
                                                        OpSet ops, int fanout) {
    extern __shared__ float2 sm[];
    const int N0 = N0S ? N0S : g.N0;
    const int NL = NLS ? NLS : NLrt;
    // static sizes use padded contiguous lines; the runtime path plain ones
    const int LS = N0S ? Padded<N0S>::LS : N0;
    auto at = [&](int l, int i) { return N0S ? Padded<N0S>::at(l, i) : l * N0 + i; };
    const int lines_total = g.N1 * g.N2h;
    const int line0 = blockIdx.x * NL;
    const int nl = min(NL, lines_total - line0);
    const int f = fanout ? 0 : blockIdx.z;
    float2 *A = sm;
    float2 *B = sm + NL * LS;
    const long long off = (long long)line0 * N0;
    {
        const float2 *in = bufs.p[f] + off;
        if (N0 % 2 == 0) {
            const int tot2 = NL * N0 / 2, valid2 = nl * N0 / 2;
#pragma unroll 4
            for (int q = threadIdx.x; q < tot2; q += kThreads) {
                const int e = 2 * q, l = e / N0, i = e - l * N0;
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (q < valid2) v = *reinterpret_cast<const float4 *>(in + e);
                A[at(l, i)] = make_float2(v.x, v.y);
                A[at(l, i + 1)] = make_float2(v.z, v.w);
            }
        } else {
            const int tot = NL * N0, valid = nl * N0;
            for (int e = threadIdx.x; e < tot; e += kThreads) {
                const int l = e / N0, i = e - l * N0;
                A[at(l, i)] = e < valid ? in[e] : make_float2(0.f, 0.f);
            }
        }
    }
    __syncthreads();
    if constexpr (N0S > 0) fft_static<N0S, NLS, false, false>(A, ax.tw);
    else fft_tile<false>(A, ax, NL, 1, N0, false);
    const int nout = fanout ? ops.n : 1;
    for (int o = 0; o < nout; ++o) {
        const int oi = fanout ? o : f;
        float2 *W = fanout ? B : A;
        const int tot = NL * N0;
        for (int e = threadIdx.x; e < tot; e += kThreads) {
            const int l = e / N0, ix = e - l * N0;
            const int line = line0 + l;
            const int iy = line % g.N1, iz = line / g.N1;
            const int a = at(l, ix);
            W[a] = line < lines_total ? cmul(A[a], eval_op(P, ops.kind[oi], ops.axis[oi], ix, iy, iz))
                                      : make_float2(0.f, 0.f);
        }
        __syncthreads();
        if constexpr (N0S > 0) fft_static<N0S, NLS, true, false>(W, ax.tw);
        else fft_tile<true>(W, ax, NL, 1, N0, false);
        float2 *out = bufs.p[oi] + off;
        if (N0 % 2 == 0) {
            const int valid2 = nl * N0 / 2;
#pragma unroll 4
            for (int q = threadIdx.x; q < valid2; q += kThreads) {
                const int e = 2 * q, l = e / N0, i = e - l * N0;
                const float2 a0 = W[at(l, i)], a1 = W[at(l, i + 1)];
                *reinterpret_cast<float4 *>(out + e) = make_float4(a0.x, a0.y, a1.x, a1.y);
            }
        } else {
            const int valid = nl * N0;
            for (int e = threadIdx.x; e < valid; e += kThreads) {
                const int l = e / N0, i = e - l * N0;
                out[e] = W[at(l, i)];
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// z-line tile helpers.  A tile is TX = 2*PL consecutive x at one y and every
// z; packed element (l, z) at s[z*PL + l] holds (f(x0+2l), f(x0+2l+1)).
// ---------------------------------------------------------------------------
template <int N2S, int PLS>
__device__ __forceinline__ void zload_c2r(float2 *s, const float2 *__restrict__ H, const Geom &g, int x0, int y,
                                          int PLrt) {
    const int N2 = N2S ? N2S : g.N2, N0 = g.N0;
    const int N2h = N2 / 2 + 1;
    const int PL = PLS ? PLS : PLrt;
    const int tot = PL * N2;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
        const int l = idx % PL, z = idx / PL;
        int k = z;
        bool cj = false;
        if (z >= N2h) { k = N2 - z; cj = true; }
        const int xa = x0 + 2 * l;
        const float2 *h = H + ((long long)k * g.N1 + y) * N0;
        float2 A, B;
        if (g.vec2 && xa + 1 < N0) {
            const float4 q = *reinterpret_cast<const float4 *>(h + xa);
            A = make_float2(q.x, q.y);
            B = make_float2(q.z, q.w);
        } else {
            A = xa < N0 ? h[xa] : make_float2(0.f, 0.f);
            B = xa + 1 < N0 ? h[xa + 1] : make_float2(0.f, 0.f);
        }
        if (cj) { A.y = -A.y; B.y = -B.y; }
        if (k == 0 || 2 * k == N2) { A.y = 0.f; B.y = 0.f; }   // Hermitian projection
        s[idx] = make_float2(A.x - B.y, A.y + B.x);
    }
}

template <int N2S, int PLS>
__device__ __forceinline__ void zstore_r2c(const float2 *s, float2 *__restrict__ H, const Geom &g, int x0, int y,
                                           int PLrt) {
    const int N0 = g.N0;
    const int N2 = N2S ? N2S : g.N2;
    const int PL = PLS ? PLS : PLrt;
    const int tot = PL * (N2 / 2 + 1);
#pragma unroll 4
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const int l = idx % PL, k = idx / PL;
        const float2 Zk = s[k * PL + l];
        const int nk = k == 0 ? 0 : N2 - k;
        const float2 Zn = s[nk * PL + l];
        const float2 A = make_float2(0.5f * (Zk.x + Zn.x), 0.5f * (Zk.y - Zn.y));
        const float2 B = make_float2(0.5f * (Zk.y + Zn.y), -0.5f * (Zk.x - Zn.x));
        const int xa = x0 + 2 * l;
        float2 *h = H + ((long long)k * g.N1 + y) * N0;
        if (g.vec2 && xa + 1 < N0) {
            *reinterpret_cast<float4 *>(h + xa) = make_float4(A.x, A.y, B.x, B.y);
        } else {
            if (xa < N0) h[xa] = A;
            if (xa + 1 < N0) h[xa + 1] = B;
        }
    }
}

template <int N2S, int PLS>
__device__ __forceinline__ void zload_real(float2 *s, const float *__restrict__ R, const Geom &g, int x0, int y,
                                           int PLrt) {
    const int PL = PLS ? PLS : PLrt;
    const int tot = PL * (N2S ? N2S : g.N2);
#pragma unroll 4
    for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
        const int l = idx % PL, z = idx / PL;
        const int xa = x0 + 2 * l;
        const long long gi = xa + (long long)g.N0 * (y + (long long)g.N1 * z);
        const bool two = xa + 1 < g.N0;
        s[idx] = xa < g.N0 ? ld2(R, gi, two, g.vec2) : make_float2(0.f, 0.f);
    }
}

// ---------------------------------------------------------------------------
// source descriptions used inside the fused z-stages
// ---------------------------------------------------------------------------
// Dense additive source: field += scale * F, scale = sig[t-1] (one signal
// for every source point) or 1 (F already holds this step's filtered source).
struct DenseSrc {
    const float *F;
    const float *sig;
    int T;
};
__device__ __forceinline__ bool dense_active(const DenseSrc &d, int t, float &scale) {
    if (!d.F || t > d.T) return false;
    scale = d.sig ? __ldg(d.sig + (t - 1)) : 1.f;
    return true;
}

// Sparse point source (dirichlet / additive-no-correction), CSR per z-tile.
struct SparseSrc {
    const int *off;       // [ntiles + 1], tile = blockIdx.x + gridDim.x * blockIdx.y
    const int *cell;      // tile-local cell: z * TX + (x - x0)
    const int *row;       // signal row of the entry
    const float *sig[3];  // [nsig x T] column-major per field component
    int T[3];             // signal length per component
    int nsig, mode;       // mode: 0 dirichlet, 1 additive-no-correction
};

// Time-reversal overwrite of p on the sensor mask, CSR per z-tile.
struct TRSrc {
    const int *off;
    const int *cell;
    const int *row;       // sensor row
    const float *data;    // [M x Nt] as given (not flipped)
    int M, Nt;
};

// ---------------------------------------------------------------------------
// Stage U: momentum conservation (kspaceFirstOrder3D.m:792-803), velocity
// sources (:806-886) and the forward z-transform of the new velocity.
// Input spec[f] = z-half spectrum of dd_pos_f kappa p_k after the inverse x/y
// passes; output spec[f] = z-half spectrum of u_f.
// grid = (ceil(N0/TX), N1, D); blockIdx.z = velocity component.
// ---------------------------------------------------------------------------
struct StageU {
    Geom g;
    AxisFFT axz;
    int PL;
    Spec4 spec;
    float *u[3];              // velocity before this step's update
    float *u_out[3];          // updated velocity (double-buffered)
    Med rho_sg_inv[3];
    const float *pml_sg[3];   // per internal axis
    float dt;
    int init;                 // p0 start: u = dt/2 rho_sg_inv grad, no PML, no output spectrum
    int write_spec;
    DenseSrc dense[3];
    SparseSrc sparse;
    const int *d_t;
    int comp_axis[3];         // internal axis of velocity component f
};

template <int N2S, int PLS>
__global__ void __launch_bounds__(kThreads, 2) k_stage_u(StageU a) {
    extern __shared__ float2 sm[];
    const Geom &g = a.g;
    const int f = blockIdx.z;
    const int PL = PLS ? PLS : a.PL, TX = 2 * PL;
    const int N2 = N2S ? N2S : g.N2;
    const int x0 = blockIdx.x * TX, y = blockIdx.y;
    const int t = *a.d_t;
    const float *u = a.u[f];
    float *uo_ = a.u_out[f];
    const int ax = a.comp_axis[f];
    const float *pmlv = a.pml_sg[ax];

    zload_c2r<N2S, PLS>(sm, a.spec.p[f], g, x0, y, PL);
    __syncthreads();
    tile_fft_il<N2S, PLS, true>(sm, a.axz, PL);

    float dscale = 0.f;
    const bool dense = dense_active(a.dense[f], t, dscale);
    const float pml_y = ax == 1 ? __ldg(pmlv + y) : 1.f;
    const int tot = PL * N2;
#pragma unroll 2
    for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
        const int l = idx % PL, z = idx / PL;
        const int xa = x0 + 2 * l;
        if (xa >= g.N0) continue;
        const bool two = xa + 1 < g.N0;
        const long long gi = xa + (long long)g.N0 * (y + (long long)g.N1 * z);
        const float2 gr = sm[idx];
        const float2 ri = med2(a.rho_sg_inv[f], gi, two, g.vec2);
        float2 un;
        if (a.init) {
            un = make_float2(0.5f * a.dt * ri.x * gr.x, 0.5f * a.dt * ri.y * gr.y);
        } else {
            float2 pm;
            if (ax == 0) pm = make_float2(__ldg(pmlv + xa), two ? __ldg(pmlv + xa + 1) : 1.f);
            else if (ax == 1) pm = make_float2(pml_y, pml_y);
            else { const float q = __ldg(pmlv + z); pm = make_float2(q, q); }
            const float2 uo = ld2(u, gi, two, g.vec2);
            un.x = pm.x * (pm.x * uo.x - a.dt * ri.x * gr.x);
            un.y = pm.y * (pm.y * uo.y - a.dt * ri.y * gr.y);
            if (dense) {
                const float2 F = ld2(a.dense[f].F, gi, two, g.vec2);
                un.x = fmaf(dscale, F.x, un.x);
                un.y = fmaf(dscale, F.y, un.y);
            }
        }
        st2(uo_, gi, un, two, g.vec2);
        sm[idx] = make_float2(un.x, two ? un.y : 0.f);
    }
    __syncthreads();
    if (!a.init && a.sparse.off && a.sparse.sig[f] && t <= a.sparse.T[f]) {
        const int tile = blockIdx.x + gridDim.x * blockIdx.y;
        const int e0 = a.sparse.off[tile], e1 = a.sparse.off[tile + 1];
        for (int e = e0 + threadIdx.x; e < e1; e += kThreads) {
            const int c = a.sparse.cell[e];
            const int z = c / TX, xl = c - z * TX;
            const float v = __ldg(a.sparse.sig[f] + a.sparse.row[e] + (long long)a.sparse.nsig * (t - 1));
            float *slot = reinterpret_cast<float *>(sm + z * PL + (xl >> 1)) + (xl & 1);
            const float nv = a.sparse.mode == 0 ? v : *slot + v;
            *slot = nv;
            uo_[x0 + xl + (long long)g.N0 * (y + (long long)g.N1 * z)] = nv;
        }
        __syncthreads();
    }
    if (!a.init && a.write_spec) {
        tile_fft_il<N2S, PLS, false>(sm, a.axz, PL);
        zstore_r2c<N2S, PLS>(sm, a.spec.p[f], g, x0, y, PL);
    }
}

// ---------------------------------------------------------------------------
// Stage R: mass conservation (kspaceFirstOrder3D.m:912-927), pressure sources
// (:930-962) and the equation of state (:965-1019).
//   lossless / stokes: p complete; output spec[0] = R2C(p)
//   absorbing: p holds the non-spectral part; outputs R2C(rho0 * sum du) and
//   R2C(sum rho) for the absorption / dispersion operators
// Input spec[0..D-1] = z-half spectra of the velocity divergence terms.
// grid = (ceil(N0/TX), N1, 1)
// ---------------------------------------------------------------------------
struct StageR {
    Geom g;
    AxisFFT axz;
    int PL;
    int D;
    Spec4 spec;
    float *rho[3];            // values before this step's update
    float *rho_out[3];        // updated values (double-buffered)
    float *srho;              // nonlinear mass coefficient q = 2 sum(rho) + rho0: read (old), rewritten (new)
    float *p;
    Med rho0, c0, BonA;
    Med c2tau;                // c0^2 * absorb_tau (stokes equation of state)
    const float *pml[3];      // per internal axis
    int comp_axis[3];
    float dt;
    int nonlinear;
    int eos;                  // 0 lossless, 1 absorbing, 2 stokes
    int has_tau, has_eta;
    DenseSrc dense;
    SparseSrc sparse;
    TRSrc tr;
    int write_spec;
    const int *d_t;
};

// Tensor maps of one stage U launch with TMA staging (component f = the
// block's z index): the current velocity, 1 / rho_sg and the spectrum of
// each component.
struct StageUMaps {
    CUtensorMap u[3];
    CUtensorMap rsi[3];
    CUtensorMap spec[3];
    int zbox;
    int *err;
};

// Tensor maps of one stage P launch with TMA staging: the term weights
// (c0^2 tau, c0^2 eta), p and the terms' spectra.
struct StagePMaps {
    CUtensorMap w0, w1, p;
    CUtensorMap spec[2];
    int zbox;
    int *err;
};

// Tensor maps of one stage R launch with TMA staging, filled per launch by
// the host (rho[] name the current input buffers).  Real fields: 3-D FP32
// maps of (N0, N1, N2) with a (TX, 1, zbox) box; spectra: 3-D 8-byte maps
// of (N0, N1, N2/2+1) with a (TX, 1, N2/2+1) box.
struct StageRMaps {
    CUtensorMap rho[3];    // staged rho_i
    CUtensorMap coef;      // mass coefficient: q (nonlinear) or rho0 (linear)
    CUtensorMap rho0;      // rho0 for the equation of state (nonlinear)
    CUtensorMap c0;
    CUtensorMap bona;
    CUtensorMap spec[3];   // spectra (rows prefetch)
    int zbox;              // z extent of a real-field box (N2 / zbox boxes per field)
    int *err;              // bit 1: a staged copy did not arrive in time
};

__device__ __forceinline__ void apply_tr(float2 *sm, const TRSrc &tr, const Geom &g, int PL, int x0, int y, int t,
                                         float *rho0_, float *rho1_, float *rho2_, int D, const Med &c0, float *p,
                                         float *qnl, const Med &rho0m) {
    // Dirichlet overwrite of p on the mask with the flipped data for step t+1
    // (kspaceFirstOrder3D.m:772-788; 2D :715-729) and the matching rho.
    if (!tr.off) return;
    const int col = tr.Nt - t - 1;       // flipped column t+1 (1-based) -> original column
    if (col < 0) return;
    const int TX = 2 * PL;
    const int tile = blockIdx.x + gridDim.x * blockIdx.y;
    const int e0 = tr.off[tile], e1 = tr.off[tile + 1];
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int c = tr.cell[e];
        const int z = c / TX, xl = c - z * TX;
        const float v = __ldg(tr.data + tr.row[e] + (long long)tr.M * col);
        const long long gi = x0 + xl + (long long)g.N0 * (y + (long long)g.N1 * z);
        float *slot = reinterpret_cast<float *>(sm + z * PL + (xl >> 1)) + (xl & 1);
        *slot = v;
        p[gi] = v;
        const float cc = c0.arr ? __ldg(c0.arr + gi) : c0.val;
        const float r = v / ((float)D * cc * cc);
        rho0_[gi] = r;
        rho1_[gi] = r;
        if (D == 3) rho2_[gi] = r;
        if (qnl) qnl[gi] = fmaf(2.f * (float)D, r, rho0m.arr ? __ldg(rho0m.arr + gi) : rho0m.val);
    }
}

template <int N2S, int PLS>
__global__ void __launch_bounds__(kThreads, 2) k_stage_r(StageR a) {
    extern __shared__ float2 sm[];
    const Geom &g = a.g;
    const int PL = PLS ? PLS : a.PL, TX = 2 * PL;
    const int N2 = N2S ? N2S : g.N2;
    const int tot = PL * N2;
    float2 *tile = sm;
    float2 *acc_old = sm + tot;
    float2 *acc_rho = sm + 2 * tot;
    float2 *acc_du = sm + 3 * tot;
    const int x0 = blockIdx.x * TX, y = blockIdx.y;
    const int t = *a.d_t;
    float dscale = 0.f;
    const bool dense = dense_active(a.dense, t, dscale);

    // sum of rho before the update (nonlinear mass conservation, :921)
    for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
        const int l = idx % PL, z = idx / PL;
        const int xa = x0 + 2 * l;
        float2 so = make_float2(0.f, 0.f);
        if (a.nonlinear && xa < g.N0) {
            const bool two = xa + 1 < g.N0;
            const long long gi = xa + (long long)g.N0 * (y + (long long)g.N1 * z);
            for (int i = 0; i < a.D; ++i) {
                const float2 r = ld2(a.rho[i], gi, two, g.vec2);
                so.x += r.x;
                so.y += r.y;
            }
        }
        acc_old[idx] = so;
        acc_rho[idx] = make_float2(0.f, 0.f);
        acc_du[idx] = make_float2(0.f, 0.f);
    }
    for (int i = 0; i < a.D; ++i) {
        __syncthreads();
        zload_c2r<N2S, PLS>(tile, a.spec.p[i], g, x0, y, PL);
        __syncthreads();
        tile_fft_il<N2S, PLS, true>(tile, a.axz, PL);
        const int ax = a.comp_axis[i];
        const float *pmlv = a.pml[ax];
        const float pml_y = ax == 1 ? __ldg(pmlv + y) : 1.f;
        const float *rho = a.rho[i];
        float *rho_new = a.rho_out[i];
        for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
            const int l = idx % PL, z = idx / PL;
            const int xa = x0 + 2 * l;
            if (xa >= g.N0) continue;
            const bool two = xa + 1 < g.N0;
            const long long gi = xa + (long long)g.N0 * (y + (long long)g.N1 * z);
            const float2 du = tile[idx];
            float2 coef = med2(a.rho0, gi, two, g.vec2);
            if (a.nonlinear) {
                const float2 so = acc_old[idx];
                coef.x = 2.f * so.x + coef.x;
                coef.y = 2.f * so.y + coef.y;
            }
            float2 pm;
            if (ax == 0) pm = make_float2(__ldg(pmlv + xa), two ? __ldg(pmlv + xa + 1) : 1.f);
            else if (ax == 1) pm = make_float2(pml_y, pml_y);
            else { const float q = __ldg(pmlv + z); pm = make_float2(q, q); }
            const float2 ro = ld2(rho, gi, two, g.vec2);
            float2 rn;
            rn.x = pm.x * (pm.x * ro.x - a.dt * coef.x * du.x);
            rn.y = pm.y * (pm.y * ro.y - a.dt * coef.y * du.y);
            if (dense) {
                const float2 F = ld2(a.dense.F, gi, two, g.vec2);
                rn.x = fmaf(dscale, F.x, rn.x);
                rn.y = fmaf(dscale, F.y, rn.y);
            }
            st2(rho_new, gi, rn, two, g.vec2);
            float2 ar = acc_rho[idx], ad = acc_du[idx];
            ar.x += rn.x; ar.y += rn.y;
            ad.x += du.x; ad.y += du.y;
            acc_rho[idx] = ar;
            acc_du[idx] = ad;
        }
    }
    __syncthreads();
    // sparse pressure sources act on every rho component (:930-962)
    if (a.sparse.off && t <= a.sparse.T[0]) {
        const int tile_id = blockIdx.x + gridDim.x * blockIdx.y;
        const int e0 = a.sparse.off[tile_id], e1 = a.sparse.off[tile_id + 1];
        for (int e = e0 + threadIdx.x; e < e1; e += kThreads) {
            const int c = a.sparse.cell[e];
            const int z = c / TX, xl = c - z * TX;
            const float v = __ldg(a.sparse.sig[0] + a.sparse.row[e] + (long long)a.sparse.nsig * (t - 1));
            const long long gi = x0 + xl + (long long)g.N0 * (y + (long long)g.N1 * z);
            float s = 0.f;
            for (int i = 0; i < a.D; ++i) {
                const float nv = a.sparse.mode == 0 ? v : a.rho_out[i][gi] + v;
                a.rho_out[i][gi] = nv;
                s += nv;
            }
            float *slot = reinterpret_cast<float *>(acc_rho + z * PL + (xl >> 1)) + (xl & 1);
            *slot = s;
        }
        __syncthreads();
    }
    // equation of state
    const bool absorbing = a.eos == 1;
    for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
        const int l = idx % PL, z = idx / PL;
        const int xa = x0 + 2 * l;
        float2 pv = make_float2(0.f, 0.f);
        if (xa < g.N0) {
            const bool two = xa + 1 < g.N0;
            const long long gi = xa + (long long)g.N0 * (y + (long long)g.N1 * z);
            const float2 sr = acc_rho[idx];
            const float2 c = med2(a.c0, gi, two, g.vec2);
            const float2 c2 = make_float2(c.x * c.x, c.y * c.y);
            pv = sr;
            if (a.nonlinear) {
                const float2 r0 = med2(a.rho0, gi, two, g.vec2);
                const float2 bn = med2(a.BonA, gi, two, g.vec2);
                pv.x += bona_term(bn.x, sr.x, r0.x);
                pv.y += bona_term(bn.y, sr.y, r0.y);
            }
            pv.x *= c2.x;
            pv.y *= c2.y;
            if (a.eos == 2) {
                const float2 r0 = med2(a.rho0, gi, two, g.vec2);
                const float2 ct = med2(a.c2tau, gi, two, g.vec2);
                const float2 sd = acc_du[idx];
                pv.x += ct.x * r0.x * sd.x;
                pv.y += ct.y * r0.y * sd.y;
            }
            st2(a.p, gi, pv, two, g.vec2);
            if (a.srho && a.nonlinear) {
                const float2 r0 = med2(a.rho0, gi, two, g.vec2);
                st2(a.srho, gi, make_float2(fmaf(2.f, sr.x, r0.x), fmaf(2.f, sr.y, r0.y)), two, g.vec2);
            }
            if (absorbing && a.has_tau) {
                const float2 r0 = med2(a.rho0, gi, two, g.vec2);
                const float2 sd = acc_du[idx];
                acc_old[idx] = make_float2(r0.x * sd.x, two ? r0.y * sd.y : 0.f);
            }
            if (!two) pv.y = 0.f;
        }
        tile[idx] = pv;
    }
    __syncthreads();
    if (!absorbing) {
        apply_tr(tile, a.tr, g, PL, x0, y, t, a.rho_out[0], a.rho_out[1], a.rho_out[2], a.D, a.c0, a.p,
                 a.nonlinear ? a.srho : nullptr, a.rho0);
        __syncthreads();
        if (a.write_spec) {
            tile_fft_il<N2S, PLS, false>(tile, a.axz, PL);
            zstore_r2c<N2S, PLS>(tile, a.spec.p[0], g, x0, y, PL);
        }
        return;
    }
    int out = 0;
    if (a.has_tau) {
        tile_fft_il<N2S, PLS, false>(acc_old, a.axz, PL);
        zstore_r2c<N2S, PLS>(acc_old, a.spec.p[out++], g, x0, y, PL);
    }
    if (a.has_eta) {
        for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
            const int l = idx % PL;
            const int xa = x0 + 2 * l;
            float2 sr = acc_rho[idx];
            if (xa + 1 >= g.N0) sr.y = 0.f;
            if (xa >= g.N0) sr.x = 0.f;
            tile[idx] = sr;
        }
        __syncthreads();
        tile_fft_il<N2S, PLS, false>(tile, a.axz, PL);
        zstore_r2c<N2S, PLS>(tile, a.spec.p[out++], g, x0, y, PL);
    }
}

// ---------------------------------------------------------------------------
// Stage P: finish the absorbing equation of state (kspaceFirstOrder3D.m:972-979)
//   p = p_partial + c0^2 (tau A1 - eta A2)
// with A1 = real(ifftn(nabla1 fftn(rho0 sum du))), A2 = real(ifftn(nabla2 fftn(sum rho))),
// then the forward z-transform of p.  grid = (ceil(N0/TX), N1, 1)
// ---------------------------------------------------------------------------
struct StageP {
    Geom g;
    AxisFFT axz;
    int PL;
    int D;
    Spec4 spec;
    float *p;
    float *rho[3];
    float *srho;              // nonlinear mass coefficient q (time-reversal overwrite)
    Med c0, rho0;
    Med c2tau, c2eta;         // c0^2 * absorb_tau, c0^2 * absorb_eta
    int has_tau, has_eta;
    TRSrc tr;
    int write_spec;
    const int *d_t;
};

template <int N2S, int PLS>
__global__ void __launch_bounds__(kThreads, 2) k_stage_p(StageP a) {
    extern __shared__ float2 sm[];
    const Geom &g = a.g;
    const int PL = PLS ? PLS : a.PL, TX = 2 * PL;
    const int N2 = N2S ? N2S : g.N2;
    const int tot = PL * N2;
    float2 *tile = sm;
    float2 *acc = sm + tot;
    const int x0 = blockIdx.x * TX, y = blockIdx.y;
    const int t = *a.d_t;
    for (int idx = threadIdx.x; idx < tot; idx += kThreads) acc[idx] = make_float2(0.f, 0.f);
    int in = 0;
    for (int term = 0; term < 2; ++term) {
        if (term == 0 && !a.has_tau) continue;
        if (term == 1 && !a.has_eta) continue;
        __syncthreads();
        zload_c2r<N2S, PLS>(tile, a.spec.p[in++], g, x0, y, PL);
        __syncthreads();
        tile_fft_il<N2S, PLS, true>(tile, a.axz, PL);
        for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
            const int l = idx % PL, z = idx / PL;
            const int xa = x0 + 2 * l;
            if (xa >= g.N0) continue;
            const bool two = xa + 1 < g.N0;
            const long long gi = xa + (long long)g.N0 * (y + (long long)g.N1 * z);
            const float2 v = tile[idx];
            const float2 w = term == 0 ? med2(a.c2tau, gi, two, g.vec2) : med2(a.c2eta, gi, two, g.vec2);
            const float sg = term == 0 ? 1.f : -1.f;
            float2 ac = acc[idx];
            ac.x = fmaf(sg * w.x, v.x, ac.x);
            ac.y = fmaf(sg * w.y, v.y, ac.y);
            acc[idx] = ac;
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
        const int l = idx % PL, z = idx / PL;
        const int xa = x0 + 2 * l;
        float2 pv = make_float2(0.f, 0.f);
        if (xa < g.N0) {
            const bool two = xa + 1 < g.N0;
            const long long gi = xa + (long long)g.N0 * (y + (long long)g.N1 * z);
            const float2 pp = ld2(a.p, gi, two, g.vec2);
            const float2 ac = acc[idx];
            pv.x = pp.x + ac.x;
            pv.y = pp.y + ac.y;
            st2(a.p, gi, pv, two, g.vec2);
            if (!two) pv.y = 0.f;
        }
        tile[idx] = pv;
    }
    __syncthreads();
    apply_tr(tile, a.tr, g, PL, x0, y, t, a.rho[0], a.rho[1], a.rho[2], a.D, a.c0, a.p, a.srho, a.rho0);
    __syncthreads();
    if (a.write_spec) {
        tile_fft_il<N2S, PLS, false>(tile, a.axz, PL);
        zstore_r2c<N2S, PLS>(tile, a.spec.p[0], g, x0, y, PL);
    }
}

// ---------------------------------------------------------------------------
// plain z-transforms (setup, p0 start, time-reversal start, source filtering)
// ---------------------------------------------------------------------------
template <int N2S, int PLS>
__global__ void __launch_bounds__(kThreads, 2) k_zr2c(const float *__restrict__ R, float2 *H, Geom g, AxisFFT axz,
                                                    int PLrt) {
    extern __shared__ float2 sm[];
    const int PL = PLS ? PLS : PLrt;
    const int x0 = blockIdx.x * 2 * PL, y = blockIdx.y;
    zload_real<N2S, PLS>(sm, R, g, x0, y, PL);
    __syncthreads();
    tile_fft_il<N2S, PLS, false>(sm, axz, PL);
    zstore_r2c<N2S, PLS>(sm, H, g, x0, y, PL);
}

template <int N2S, int PLS>
__global__ void __launch_bounds__(kThreads, 2) k_zc2r(const float2 *__restrict__ H, float *R, Geom g, AxisFFT axz,
                                                    int PLrt) {
    extern __shared__ float2 sm[];
    const int PL = PLS ? PLS : PLrt;
    const int N2 = N2S ? N2S : g.N2;
    const int x0 = blockIdx.x * 2 * PL, y = blockIdx.y;
    zload_c2r<N2S, PLS>(sm, H, g, x0, y, PL);
    __syncthreads();
    tile_fft_il<N2S, PLS, true>(sm, axz, PL);
    const int tot = PL * N2;
#pragma unroll 2
    for (int idx = threadIdx.x; idx < tot; idx += kThreads) {
        const int l = idx % PL, z = idx / PL;
        const int xa = x0 + 2 * l;
        if (xa >= g.N0) continue;
        const bool two = xa + 1 < g.N0;
        const long long gi = xa + (long long)g.N0 * (y + (long long)g.N1 * z);
        st2(R, gi, sm[idx], two, g.vec2);
    }
}
}  // namespace kw
