// kw_aux.cuh -- sensor gathers, start-of-loop and set-up kernels, and the
// elementwise kernels of the adjoint.  Included by the library's main
// translation unit only; the transform and stage kernels live in
// kw_kernels.cuh / kw_static.cuh and are instantiated per axis length in
// kw_inst.cu.
#pragma once

#include "kw_kernels.cuh"

namespace kw {

// ---------------------------------------------------------------------------
// sensors (kspaceFirstOrder_extractSensorData.m:63-123): gather at the mask
// and running reductions.  p_rms is accumulated as sum p^2 and finished as
// sqrt(sum / n), equal to the reference recurrence in exact arithmetic.
// ---------------------------------------------------------------------------
struct SensorArgs {
    int M;
    int K;                     // grid cells per point (> 1: weighted, column-major M x K)
    const long long *idx;      // 0-based linear indices; NULL: every cell, in order
    const float *w;            // weights (K > 1)
    const float *field[4];     // p, u0, u1, u2
    float *series[4];          // [M x num_rec] or NULL
    float *vmax[4], *vmin[4], *vsq[4];
    int nfield;
    int record_start;
    int ring;                  // > 0: the series hold `ring` columns, column = step mod ring
    const int *d_t;
};

// one sensor point: field at its cell, or sum_k w[m + M k] field[idx[m + M k]];
// idx NULL: the mask holds every cell, so point m is cell m
__device__ __forceinline__ float sensor_value(const float *field, const long long *idx, const float *w, int M, int K,
                                              int m) {
    if (K <= 1) return field[idx ? idx[m] : m];
    float v = 0.f;
    for (int k = 0; k < K; ++k) v = fmaf(w[m + (long long)M * k], field[idx[m + (long long)M * k]], v);
    return v;
}

__global__ void k_sensor(SensorArgs a) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= a.M) return;
    const int t = *a.d_t;
    const int fi = t - a.record_start;   // 0-based column
    if (fi < 0) return;
    // unrolled: constant indices into the parameter arrays
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if (f >= a.nfield || !a.field[f]) continue;
        const float v = sensor_value(a.field[f], a.idx, a.w, a.M, a.K, m);
        if (a.series[f]) a.series[f][m + (long long)a.M * (a.ring ? fi % a.ring : fi)] = v;
        if (a.vmax[f]) a.vmax[f][m] = fi == 0 ? v : fmaxf(a.vmax[f][m], v);
        if (a.vmin[f]) a.vmin[f][m] = fi == 0 ? v : fminf(a.vmin[f][m], v);
        if (a.vsq[f]) a.vsq[f][m] = fi == 0 ? v * v : fmaf(v, v, a.vsq[f][m]);
    }
}

// The same for a mask that holds every cell (point m is cell m): four
// consecutive points per thread with 16-byte loads and stores, so each thread
// keeps four times the bytes in flight.  Needs M % 4 == 0 (every array then
// starts each column on a 16-byte boundary).
__global__ void k_sensor_all(SensorArgs a) {
    const long long m = 4 * ((long long)blockIdx.x * blockDim.x + threadIdx.x);
    if (m >= a.M) return;
    const int t = *a.d_t;
    const int fi = t - a.record_start;
    if (fi < 0) return;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if (f >= a.nfield || !a.field[f]) continue;
        const float4 v = *reinterpret_cast<const float4 *>(a.field[f] + m);
        if (a.series[f]) *reinterpret_cast<float4 *>(a.series[f] + m + (long long)a.M * (a.ring ? fi % a.ring : fi)) = v;
        if (a.vmax[f]) {
            float4 *q = reinterpret_cast<float4 *>(a.vmax[f] + m);
            if (fi == 0) *q = v;
            else { const float4 o = *q; *q = make_float4(fmaxf(o.x, v.x), fmaxf(o.y, v.y), fmaxf(o.z, v.z), fmaxf(o.w, v.w)); }
        }
        if (a.vmin[f]) {
            float4 *q = reinterpret_cast<float4 *>(a.vmin[f] + m);
            if (fi == 0) *q = v;
            else { const float4 o = *q; *q = make_float4(fminf(o.x, v.x), fminf(o.y, v.y), fminf(o.z, v.z), fminf(o.w, v.w)); }
        }
        if (a.vsq[f]) {
            float4 *q = reinterpret_cast<float4 *>(a.vsq[f] + m);
            if (fi == 0) *q = make_float4(v.x * v.x, v.y * v.y, v.z * v.z, v.w * v.w);
            else {
                const float4 o = *q;
                *q = make_float4(fmaf(v.x, v.x, o.x), fmaf(v.y, v.y, o.y), fmaf(v.z, v.z, o.z), fmaf(v.w, v.w, o.w));
            }
        }
    }
}

// running max / min over the inside region (extractSensorData.m:464-569)
struct RegionArgs {
    const float *field[4];
    float *vmax[4], *vmin[4];
    int nfield;
    int lo[3], n[3];          // inside region (0-based start, extent) per internal axis
    Geom g;
    int record_start;
    const int *d_t;
};

__global__ void k_region(RegionArgs a) {
    const long long tot = (long long)a.n[0] * a.n[1] * a.n[2];
    const int t = *a.d_t;
    const int fi = t - a.record_start;
    if (fi < 0) return;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < tot;
         r += (long long)gridDim.x * blockDim.x) {
        const int i0 = r % a.n[0];
        const long long q = r / a.n[0];
        const int i1 = q % a.n[1];
        const int i2 = q / a.n[1];
        const long long gi = (i0 + a.lo[0]) + (long long)a.g.N0 * ((i1 + a.lo[1]) + (long long)a.g.N1 * (i2 + a.lo[2]));
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if (f >= a.nfield || !a.field[f]) continue;
            const float v = a.field[f][gi];
            if (a.vmax[f]) a.vmax[f][r] = fi == 0 ? v : fmaxf(a.vmax[f][r], v);
            if (a.vmin[f]) a.vmin[f][r] = fi == 0 ? v : fminf(a.vmin[f][r], v);
        }
    }
}

// copy the inside region of a field into a compact array (p_final, u_final)
__global__ void k_crop(const float *__restrict__ src, float *dst, Geom g, int lo0, int lo1, int lo2, int n0, int n1,
                       int n2) {
    const long long tot = (long long)n0 * n1 * n2;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < tot;
         r += (long long)gridDim.x * blockDim.x) {
        const int i0 = r % n0;
        const long long q = r / n0;
        const int i1 = q % n1;
        const int i2 = q / n1;
        dst[r] = src[(i0 + lo0) + (long long)g.N0 * ((i1 + lo1) + (long long)g.N1 * (i2 + lo2))];
    }
}

__global__ void k_rms_finish(float *sq, int M, float inv_n) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < M) sq[m] = sqrtf(sq[m] * inv_n);
}

// rho_i = p0 / (D c0^2) on every cell (kspaceFirstOrder3D.m:1027-1030);
// q = 2 sum(rho) + rho0 for the nonlinear mass update
__global__ void k_init_rho(const float *__restrict__ p0, Med c0, Med rho0, float *r0, float *r1, float *r2, float *srho,
                           long long N, int D) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const float c = c0.arr ? c0.arr[i] : c0.val;
        const float v = p0[i] / ((float)D * c * c);
        r0[i] = v;
        r1[i] = v;
        if (D == 3) r2[i] = v;
        srho[i] = fmaf(2.f * (float)D, v, rho0.arr ? rho0.arr[i] : rho0.val);
    }
}

// time-reversal start: p(mask) = data(:, flipped column 1), rho(mask) = p/(D c0^2)
__global__ void k_tr_start(const long long *idx, int M, const float *data, int Nt, Med c0, Med rho0, float *p,
                           float *r0, float *r1, float *r2, float *srho, int D) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const long long gi = idx[m];
    const float v = data[m + (long long)M * (Nt - 1)];
    p[gi] = v;
    const float c = c0.arr ? c0.arr[gi] : c0.val;
    const float r = v / ((float)D * c * c);
    r0[gi] = r;
    r1[gi] = r;
    if (D == 3) r2[gi] = r;
    srho[gi] = fmaf(2.f * (float)D, r, rho0.arr ? rho0.arr[gi] : rho0.val);
}

// final time-reversal assignment p(mask) = data(:, flipped column Nt) (:1211-1213)
__global__ void k_tr_final(const long long *idx, int M, const float *data, float *p) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < M) p[idx[m]] = data[m];
}

// source_mat(index) = values(sig_index, t) into a zero field (general additive path)
__global__ void k_scatter_source(const long long *pos, const int *row, int npts, const float *sig, int nsig,
                                 float *field, const int *d_t, int T) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npts) return;
    const int t = *d_t;
    if (t > T) return;
    field[pos[i]] = sig[row[i] + (long long)nsig * (t - 1)];
}

__global__ void k_set_points(const long long *pos, int npts, float v, float *field) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < npts) field[pos[i]] = v;
}

__global__ void k_step_advance(int *d_t) { *d_t += 1; }

// series[m + M (t - record_start)] = src[idx[m]], t from the device step counter
__global__ void k_gather_series(const float *__restrict__ src, const long long *__restrict__ idx,
                                const float *__restrict__ w, int M, int K, float *series, const int *d_t,
                                int record_start) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    series[m + (long long)M * (*d_t - record_start)] = sensor_value(src, idx, w, M, K, m);
}

// dst[i] = m (array or scalar)
__global__ void k_fill_med(float *dst, Med m, long long N) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        dst[i] = m.arr ? m.arr[i] : m.val;
}

// ---------------------------------------------------------------------------
// set-up kernels (run once per plan)
// ---------------------------------------------------------------------------

// Row-major (C order) grid of shape (A, B, C) -> the column-major layout:
// in[(x B + y) C + z] -> out[x + A (y + B z)].  32 x 32 tiles over (z, x)
// per y; block (32, 8), grid (ceil(C/32), ceil(A/32), B).
__global__ void k_rowmajor_to_col(const float *__restrict__ in, float *__restrict__ out, int A, int B, int C) {
    __shared__ float t[32][33];
    const int y = blockIdx.z;
    const int z0 = blockIdx.x * 32, x0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int x = x0 + i, z = z0 + threadIdx.x;
        if (x < A && z < C) t[i][threadIdx.x] = in[((long long)x * B + y) * C + z];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int z = z0 + i, x = x0 + threadIdx.x;
        if (x < A && z < C) out[x + (long long)A * (y + (long long)B * z)] = t[threadIdx.x][i];
    }
}

// 1 / rho0_sg along internal axis `axis` (stride `s`, extent `n`): with
// derive != 0 the staggered density is the midpoint average of rho0 and its
// +1 neighbour (rho0 on the last plane) rounded to FP32, as the set-up
// forms it; without, in holds rho0_sg already.  The reciprocal is taken in
// FP64 and rounded once.
__global__ void k_inv_rho_sg(const float *in, float *out, Geom g, int axis, int derive) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    float r = in[i];
    if (derive) {
        const int x = (int)(i % g.N0);
        const long long q = i / g.N0;
        const int y = (int)(q % g.N1), z = (int)(q / g.N1);
        const int c = axis == 0 ? x : (axis == 1 ? y : z);
        const int n = axis == 0 ? g.N0 : (axis == 1 ? g.N1 : g.N2);
        const long long s = axis == 0 ? 1 : (axis == 1 ? (long long)g.N0 : (long long)g.N0 * g.N1);
        if (c + 1 < n) r = (float)(0.5 * ((double)in[i] + (double)in[i + s]));
    }
    out[i] = (float)(1.0 / (double)r);
}

// c0^2 absorb_tau and c0^2 absorb_eta (createAbsorptionVariables.m:29-101)
// in FP64: tau = -2 a c^(y-1), eta = 2 a c^y tan(pi y / 2) for the power
// law, tau = -2 a c, eta = 0 for stokes; a = alpha_coeff * np_per_db
// (db2neper with the frequency power folded in).
__global__ void k_absorb_coeffs(const float *__restrict__ c0, double c0s, const float *__restrict__ alpha, double alphas,
                                long long N, double y, double np_per_db, int stokes, double tanv, double sg0, double sg1,
                                float *__restrict__ c2tau, float *__restrict__ c2eta) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double c = c0 ? (double)c0[i] : c0s;
    const double anp = (alpha ? (double)alpha[i] : alphas) * np_per_db;
    const double tau = stokes ? -2.0 * anp * c : -2.0 * anp * pow(c, y - 1.0);
    const double eta = stokes ? 0.0 : 2.0 * anp * pow(c, y) * tanv;
    c2tau[i] = (float)(c * c * tau * sg0);
    if (c2eta) c2eta[i] = (float)(c * c * eta * sg1);
}

// ---------------------------------------------------------------------------
// adjoint kernels (gradient entry point).  One thread per cell, grid-stride;
// the discrete adjoint of the lossless linear step, component by component:
//   w_i     = rho_sg_i^-1 pml_sg_i lambda_u_i                  (k_adj_w)
//   mu      = S^T r(t) + dt sum_i D_i w_i
//   lambda_rho_i = c0^2 mu + pml_i^2 lambda_rho_i, v_i = rho0 pml_i lambda_rho_i,
//   dJ/dc0 += 2 c0 mu sum_i rho_i(t)                           (k_adj_mid)
//   dJ/drho0 += sum_i lambda_rho_i (-dt pml_i D_i u_i(t))      (k_adj_grho)
//   lambda_u_i = pml_sg_i^2 lambda_u_i + dt G_i v_i            (k_adj_u)
//   dJ/drho_sg_i^-1 += lambda_u_i (-dt pml_sg_i G_i p(t-1))    (k_adj_gR)
// Gradients accumulate in FP64.
// ---------------------------------------------------------------------------
struct AdjArgs {
    Geom g;
    int D;
    float dt;
    int axis[3];                 // internal axis of each component
    const float *pml[3];         // mass PML profile along that axis
    const float *pml_sg[3];      // momentum PML profile along that axis
    Med rsi[3];                  // 1 / rho_sg_i
    Med c0, rho0;
    float *lu[3], *lr[3];        // adjoint velocity / density
    float *A[3];                 // work fields
    const float *B[3];           // spectral results
    const float *mu;             // scattered residual S^T r(t)
    const float *rho_t[3];       // forward rho after step t
    double *g_c, *g_r0, *g_R[3];
};

__device__ __forceinline__ int adj_coord(const Geom &g, long long i, int axis) {
    if (axis == 0) return (int)(i % g.N0);
    const long long q = i / g.N0;
    return axis == 1 ? (int)(q % g.N1) : (int)(q / g.N1);
}
__device__ __forceinline__ float med1(const Med &m, long long i) { return m.arr ? __ldg(m.arr + i) : m.val; }

__global__ void k_adj_w(AdjArgs a) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.g.N; i += (long long)gridDim.x * blockDim.x)
        for (int c = 0; c < a.D; ++c) {
            const float pu = __ldg(a.pml_sg[c] + adj_coord(a.g, i, a.axis[c]));
            a.A[c][i] = med1(a.rsi[c], i) * pu * a.lu[c][i];
        }
}

__global__ void k_adj_mid(AdjArgs a) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.g.N; i += (long long)gridDim.x * blockDim.x) {
        float mu = a.mu[i];
        for (int c = 0; c < a.D; ++c) mu = fmaf(a.dt, a.B[c][i], mu);
        const float cc = med1(a.c0, i), r0 = med1(a.rho0, i);
        float srho = 0.f;
        for (int c = 0; c < a.D; ++c) {
            const float pr = __ldg(a.pml[c] + adj_coord(a.g, i, a.axis[c]));
            const float lr = fmaf(cc * cc, mu, pr * pr * a.lr[c][i]);
            a.lr[c][i] = lr;
            a.A[c][i] = r0 * pr * lr;
            srho += a.rho_t[c][i];
        }
        a.g_c[i] += 2.0 * (double)cc * (double)mu * (double)srho;
    }
}

__global__ void k_adj_grho(AdjArgs a) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.g.N; i += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < a.D; ++c) {
            const float pr = __ldg(a.pml[c] + adj_coord(a.g, i, a.axis[c]));
            s += (double)a.lr[c][i] * (double)(-a.dt * pr * a.B[c][i]);
        }
        a.g_r0[i] += s;
    }
}

__global__ void k_adj_u(AdjArgs a) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.g.N; i += (long long)gridDim.x * blockDim.x)
        for (int c = 0; c < a.D; ++c) {
            const float pu = __ldg(a.pml_sg[c] + adj_coord(a.g, i, a.axis[c]));
            a.lu[c][i] = fmaf(pu * pu, a.lu[c][i], a.dt * a.B[c][i]);
        }
}

__global__ void k_adj_gR(AdjArgs a) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.g.N; i += (long long)gridDim.x * blockDim.x)
        for (int c = 0; c < a.D; ++c) {
            const float pu = __ldg(a.pml_sg[c] + adj_coord(a.g, i, a.axis[c]));
            a.g_R[c][i] += (double)a.lu[c][i] * (double)(-a.dt * pu * a.B[c][i]);
        }
}

// mu[sidx[m]] = res[m + M col] (sensor cells are distinct) for the residual
// column col = *d_col, nothing when col < 0 (steps before record_start).  The
// column lives on the device, so a captured backward step replays unchanged.
__global__ void k_adj_scatter(float *mu, const long long *sidx, int M, const float *res, const int *d_col) {
    const int col = *d_col;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= 0 && m < M) mu[sidx[m]] = res[m + (long long)M * col];
}
__global__ void k_adj_set_col(int *d_col, int col) { *d_col = col; }
__global__ void k_adj_col_back(int *d_col) { *d_col -= 1; }

// dJ/drho0 = direct term + the chain through rho_sg_i^-1 = 1 / rho_sg_i:
// h_i = dJ/drho_sg_i = -rho_sg_i^-2 dJ/drho_sg_i^-1; with derive != 0 the
// staggered density is the midpoint average of rho0 at x and x + e_i (rho0
// itself on the last plane), otherwise rho_sg_i = rho0.
__global__ void k_adj_rho_chain(AdjArgs a, int derive, double *out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.g.N; i += (long long)gridDim.x * blockDim.x) {
        double s = a.g_r0[i];
        for (int c = 0; c < a.D; ++c) {
            const int ax = a.axis[c];
            const int n = ax == 0 ? a.g.N0 : (ax == 1 ? a.g.N1 : a.g.N2);
            const long long st = ax == 0 ? 1 : (ax == 1 ? (long long)a.g.N0 : (long long)a.g.N0 * a.g.N1);
            const int k = adj_coord(a.g, i, ax);
            const double r = med1(a.rsi[c], i);
            const double h = -r * r * a.g_R[c][i];
            if (!derive || k == n - 1) {
                s += h;
            } else {
                s += 0.5 * h;
            }
            if (derive && k >= 1) {
                const double rm = med1(a.rsi[c], i - st);
                s += 0.5 * (-rm * rm * a.g_R[c][i - st]);
            }
        }
        out[i] = s;
    }
}

// flags |= bit where a value is not strictly positive (or NaN)
__global__ void k_check_positive(const float *__restrict__ a, long long N, int *flags, int bit) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N && !(a[i] > 0.f)) atomicOr(flags, bit);
}

}  // namespace kw
