// kwave_b200.cu -- host side of the B200 k-space first-order time loop and its C ABI.
//
// The entry points declared in include/kwave_b200.h replace the external
// native solver that k-Wave's kspaceFirstOrder3DC / 3DG / 2DG launch after
// the MATLAB setup (+kwave/+legacy/kspaceFirstOrder3DC.m:530-546): the same
// variable set (private/kspaceFirstOrder_saveToDisk.m:46-353) comes in as
// host pointers, the loop of kspaceFirstOrder3D.m:769-1208 runs on the
// device, and the sensor outputs come back into caller buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <cstdlib>
#include <array>
#include <map>
#include <mutex>
#include <vector>

#include <cudaTypedefs.h>

#include "kw_plan.cuh"
#include "kw_aux.cuh"
#include "kw_static.cuh"
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <thread>

using namespace kw;

namespace {
thread_local std::string g_err;
}  // namespace

namespace kw {

kw_status fail(kw_status s, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

kw_status set_smem(const void *fn, size_t bytes) {
    if (bytes > 48 * 1024) KW_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return KW_OK;
}

kw_status launched(kw_plan *P) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(KW_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
    P->launches += 1;
    return KW_OK;
}

}  // namespace kw

namespace {

// cuTensorMapEncodeTiled from the driver, through the runtime's entry-point
// query (no link-time dependency on the driver library)
PFN_cuTensorMapEncodeTiled_v12000 g_encode_tiled = nullptr;
std::once_flag g_encode_once;
bool have_encode_tiled() {
    std::call_once(g_encode_once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode_tiled = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        cudaGetLastError();
    });
    return g_encode_tiled != nullptr;
}

// 3-D tensor map of a grid array of (d0, d1, d2) elements of `elem` bytes
// (4: a real field, 8: a half spectrum), x fastest, box (b0, 1, b2)
kw_status encode_map(CUtensorMap *m, const void *base, int elem, int d0, int d1, int d2, int b0, int b2) {
    const cuuint64_t dims[3] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2};
    const cuuint64_t strides[2] = {(cuuint64_t)d0 * elem, (cuuint64_t)d0 * d1 * elem};
    const cuuint32_t box[3] = {(cuuint32_t)b0, 1u, (cuuint32_t)b2};
    const cuuint32_t es[3] = {1u, 1u, 1u};
    const CUresult r = g_encode_tiled(m, elem == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT64, 3,
                                      const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(KW_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return KW_OK;
}

}  // namespace

namespace kw {

// tensor map of a plan buffer (elem 4: a real field, 8: a half spectrum) for
// tiles TX wide, cached per (buffer, box width); buffers never move during a
// plan's life
kw_status plan_map(kw_plan *P, const void *ptr, int elem, int TX, CUtensorMap *dst) {
    if (!ptr) return KW_OK;
    const Geom &g = P->g;
    const auto key = std::make_pair(ptr, TX * elem);
    auto it = P->tmaps.find(key);
    if (it == P->tmaps.end()) {
        CUtensorMap t;
        if (elem == 4) KW_TRY(encode_map(&t, ptr, 4, g.N0, g.N1, g.N2, TX, g.N2 <= 256 ? g.N2 : g.N2 / 2));
        else KW_TRY(encode_map(&t, ptr, 8, g.N0, g.N1, g.N2h, TX, tma_row_box(g.N2)));
        it = P->tmaps.emplace(key, t).first;
    }
    *dst = it->second;
    return KW_OK;
}

kw_status stage_u_maps(kw_plan *P, const StageU &a, int TX, StageUMaps *m, bool *use) {
    *use = P->tma_r;
    if (!*use) return KW_OK;
    std::memset(m, 0, sizeof(*m));
    for (int i = 0; i < P->D; ++i) {
        KW_TRY(plan_map(P, a.u[i], 4, TX, &m->u[i]));
        KW_TRY(plan_map(P, a.rho_sg_inv[i].arr, 4, TX, &m->rsi[i]));
        KW_TRY(plan_map(P, a.spec.p[i], 8, TX, &m->spec[i]));
    }
    m->zbox = P->g.N2 <= 256 ? P->g.N2 : P->g.N2 / 2;
    m->err = P->d_err;
    return KW_OK;
}

kw_status stage_p_maps(kw_plan *P, const StageP &a, int TX, StagePMaps *m, bool *use) {
    *use = P->tma_r;
    if (!*use) return KW_OK;
    std::memset(m, 0, sizeof(*m));
    const int nterm = (a.has_tau ? 1 : 0) + (a.has_eta ? 1 : 0);
    const Med w0 = a.has_tau ? a.c2tau : a.c2eta;
    KW_TRY(plan_map(P, nterm > 0 ? w0.arr : nullptr, 4, TX, &m->w0));
    KW_TRY(plan_map(P, nterm > 1 ? a.c2eta.arr : nullptr, 4, TX, &m->w1));
    KW_TRY(plan_map(P, a.p, 4, TX, &m->p));
    for (int k = 0; k < nterm && k < 2; ++k) KW_TRY(plan_map(P, a.spec.p[k], 8, TX, &m->spec[k]));
    m->zbox = P->g.N2 <= 256 ? P->g.N2 : P->g.N2 / 2;
    m->err = P->d_err;
    return KW_OK;
}

kw_status stage_r_maps(kw_plan *P, const StageR &a, int TX, StageRMaps *m, bool *use) {
    *use = P->tma_r;
    if (!*use) return KW_OK;
    const Geom &g = P->g;
    const int zbox = g.N2 <= 256 ? g.N2 : g.N2 / 2;
    auto map_of = [&](const void *ptr, int elem, CUtensorMap *dst) -> kw_status { return plan_map(P, ptr, elem, TX, dst); };
    std::memset(m, 0, sizeof(*m));
    for (int i = 0; i < a.D; ++i) {
        KW_TRY(map_of(a.rho[i], 4, &m->rho[i]));
        KW_TRY(map_of(a.spec.p[i], 8, &m->spec[i]));
    }
    KW_TRY(map_of(a.nonlinear ? (const void *)a.srho : (const void *)a.rho0.arr, 4, &m->coef));
    KW_TRY(map_of(a.rho0.arr, 4, &m->rho0));
    KW_TRY(map_of(a.c0.arr, 4, &m->c0));
    KW_TRY(map_of(a.nonlinear ? a.BonA.arr : nullptr, 4, &m->bona));
    m->zbox = zbox;
    m->err = P->d_err;
    return KW_OK;
}

}  // namespace kw

namespace {

// --------------------------------------------------------------------------
// FP64 host precompute
// --------------------------------------------------------------------------
bool factorize(int n, std::vector<int> &radix) {
    radix.clear();
    while (n % 4 == 0) { radix.push_back(4); n /= 4; }
    while (n % 2 == 0) { radix.push_back(2); n /= 2; }
    const int primes[3] = {3, 5, 7};
    for (int p : primes)
        while (n % p == 0) { radix.push_back(p); n /= p; }
    // any other prime factor: a direct-sum stage (fft_stage_any)
    for (int p = 11; n > 1 && (long long)p * p <= n; p += 2)
        while (n % p == 0) { radix.push_back(p); n /= p; }
    if (n > 1) radix.push_back(n);
    return radix.size() <= (size_t)kMaxStages;
}

// kWaveGrid.makeDim (kWaveGrid.m:779-797) in FFT order (ifftshift applied)
std::vector<double> kvec_fft(int n, double d) {
    std::vector<double> nat(n), out(n);
    for (int i = 0; i < n; ++i) {
        const int m = (n % 2 == 0) ? i - n / 2 : i - (n - 1) / 2;
        nat[i] = (2.0 * M_PI / d) * ((double)m / n);
    }
    nat[n / 2] = 0.0;
    // ifftshift: out[i] = nat[(i + n/2) % n]
    for (int i = 0; i < n; ++i) out[i] = nat[(i + n / 2) % n];
    return out;
}

// getPML.m:52-87
std::vector<double> get_pml(int n, double d, double dt, double c, int size, double alpha, bool staggered) {
    std::vector<double> pml(n, 1.0);
    for (int x = 1; x <= size; ++x) {
        const double xs = staggered ? x + 0.5 : x;
        const double left = alpha * (c / d) * std::pow((xs - size - 1) / (0.0 - size), 4);
        const double right = alpha * (c / d) * std::pow(xs / size, 4);
        pml[x - 1] = std::exp(-left * dt / 2);
        pml[n - size + x - 1] = std::exp(-right * dt / 2);
    }
    return pml;
}

// db2neper.m:52
double db2neper(double a, double y) { return 100.0 * a * std::pow(1e-6 / (2 * M_PI), y) / (20.0 * std::log10(std::exp(1.0))); }

}  // namespace

// --------------------------------------------------------------------------
// plan memory (the plan itself is defined in kw_plan.cuh)
// --------------------------------------------------------------------------

namespace {

// Plan memory is stream-ordered (cudaMallocAsync / cudaFreeAsync on the plan's
// stream), so creating and destroying plans never synchronises other plans'
// work on the device (the serving loop relies on this).
template <typename T>
kw_status palloc(kw_plan *P, T **p, size_t count) {
    *p = nullptr;
    if (count == 0) return KW_OK;
    {
        cudaError_t e = cudaMallocAsync((void **)p, count * sizeof(T), P->stream);
        if (e != cudaSuccess) {
            *p = nullptr;
            return fail(e == cudaErrorMemoryAllocation ? KW_ERR_NOMEM : KW_ERR_CUDA,
                        "device allocation of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
        }
    }
    if (*p) {
        P->allocs.push_back((void *)*p);
        P->bytes += count * sizeof(T);
        cudaError_t e = cudaMemsetAsync(*p, 0, count * sizeof(T), P->stream);
        if (e != cudaSuccess) return fail(KW_ERR_CUDA, "cudaMemset failed: %s", cudaGetErrorString(e));
    }
    return KW_OK;
}

template <typename T>
kw_status pupload(kw_plan *P, T **p, const T *host, size_t count) {
    KW_TRY(palloc(P, p, count));
    if (count) KW_CUDA(cudaMemcpyAsync(*p, host, count * sizeof(T), cudaMemcpyHostToDevice, P->stream));
    KW_CUDA(cudaStreamSynchronize(P->stream));
    return KW_OK;
}

// Device buffers needed only while a plan is set up; released (stream
// ordered) when the set-up returns, on success or failure.
struct TempDev {
    cudaStream_t stream;
    std::vector<void *> ptrs;
    template <typename T>
    kw_status get(T **p, size_t count) {
        *p = nullptr;
        const cudaError_t e = cudaMallocAsync((void **)p, count * sizeof(T), stream);
        if (e != cudaSuccess) {
            *p = nullptr;
            return fail(e == cudaErrorMemoryAllocation ? KW_ERR_NOMEM : KW_ERR_CUDA,
                        "device allocation of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
        }
        ptrs.push_back((void *)*p);
        return KW_OK;
    }
    ~TempDev() {
        for (void *a : ptrs) cudaFreeAsync(a, stream);
    }
};

// ---- timing ---------------------------------------------------------------
kw_status timer_flush(kw_plan *P) {
    if (P->timers.empty()) return KW_OK;
    KW_CUDA(cudaStreamSynchronize(P->stream));
    for (auto &r : P->timers) {
        float ms = 0.f;
        KW_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        P->t_ms[r.cls] += ms;
        P->t_count[r.cls] += 1;
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    P->timers.clear();
    return KW_OK;
}

struct Scope {
    kw_plan *P;
    int cls;
    bool on;
    TimerRec r{};
    Scope(kw_plan *P_, int cls_) : P(P_), cls(cls_), on((P_->timing_mask >> cls_) & 1u) {
        if (on) {
            cudaEventCreate(&r.a);
            cudaEventCreate(&r.b);
            r.cls = cls;
            cudaEventRecord(r.a, P->stream);
        }
    }
    ~Scope() {
        if (on) {
            cudaEventRecord(r.b, P->stream);
            P->timers.push_back(r);
            if (P->timers.size() > 8192) timer_flush(P);
        }
    }
};


bool is_static(int n) {
    switch (n) {
#define KW_CASE(N) case N:
        KW_STATIC_SIZES(KW_CASE)
#undef KW_CASE
        return true;
        default: return false;
    }
}
template <template <int> class L, typename... A>
kw_status dispatch(int n, A... args) {
    switch (n) {
#define KW_CASE(N) case N: return L<N>::run(args...);
        KW_STATIC_SIZES(KW_CASE)
#undef KW_CASE
        default: return L<0>::run(args...);
    }
}

// ---- transform passes -----------------------------------------------------

// kz planes [kz0, kz0 + nkz) only (static kernels); the runtime kernels
// always take every plane and must be called with the full range
kw_status ypass(kw_plan *P, bool inv, Spec4 bufs, int nf, int kz0 = 0, int nkz = -1) {
    if (P->g.N1 == 1 || nf == 0) return KW_OK;
    if (P->static_y && !P->tw[1]) return fail(KW_ERR_INVALID, "internal: axis-1 twiddle table missing");
    Scope s(P, KW_KCLASS_YPASS);
    if (nkz < 0) { kz0 = 0; nkz = P->g.N2h; }
    return dispatch<YLaunch>(P->static_y ? P->g.N1 : 0, P, inv, bufs, nf, kz0, nkz);
}


kw_status xpass(kw_plan *P, Spec4 bufs, OpSet ops, int fanout, int nf, int kz0 = 0, int nkz = -1) {
    if (P->static_x && !P->tw[0]) return fail(KW_ERR_INVALID, "internal: axis-0 twiddle table missing");
    Scope s(P, KW_KCLASS_XPASS);
    if (nkz < 0) { kz0 = 0; nkz = P->g.N2h; }
    return dispatch<XLaunch>(P->static_x ? P->g.N0 : 0, P, bufs, ops, fanout, nf, kz0, nkz);
}

// y / x / y passes of one spectral group, chunked over kz planes so that a
// chunk's half spectrum written by one pass is still in L2 when the next pass
// reads it.  fanout: buffer 0 is transformed once and ops 0..n-1 write
// buffers 0..n-1; otherwise the n buffers each get their own operator.
kw_status yxy_group(kw_plan *P, Spec4 bufs, int n, OpSet ops, bool fanout) {
    const int nch = (P->static_x && (P->static_y || P->g.N1 == 1)) ? P->kz_chunks : 1;
    const int N2h = P->g.N2h;
    for (int c = 0; c < nch; ++c) {
        const int kz0 = (int)((long long)N2h * c / nch), kz1 = (int)((long long)N2h * (c + 1) / nch);
        const int nkz = nch > 1 ? kz1 - kz0 : -1;
        KW_TRY(ypass(P, false, bufs, fanout ? 1 : n, kz0, nkz));
        KW_TRY(xpass(P, bufs, ops, fanout ? 1 : 0, fanout ? 1 : n, kz0, nkz));
        KW_TRY(ypass(P, true, bufs, n, kz0, nkz));
    }
    return KW_OK;
}


kw_status zr2c(kw_plan *P, const float *R, float2 *H) {
    if (P->static_z && !P->tw[2]) return fail(KW_ERR_INVALID, "internal: axis-2 twiddle table missing");
    return dispatch<ZR2CLaunch>(P->static_z ? P->g.N2 : 0, P, R, H);
}

kw_status zc2r(kw_plan *P, const float2 *H, float *R) {
    if (P->static_z && !P->tw[2]) return fail(KW_ERR_INVALID, "internal: axis-2 twiddle table missing");
    return dispatch<ZC2RLaunch>(P->static_z ? P->g.N2 : 0, P, H, R);
}

Spec4 specs(kw_plan *P, int a, int b = -1, int c = -1) {
    Spec4 s{};
    s.p[0] = P->spec[a];
    s.p[1] = b >= 0 ? P->spec[b] : nullptr;
    s.p[2] = c >= 0 ? P->spec[c] : nullptr;
    s.p[3] = nullptr;
    return s;
}

// gradient spectra of p for the next momentum update: spec[0] holds the
// z-half spectrum of p on entry; spec[0..D-1] hold dd_pos_i kappa p_k after
// the inverse x and y passes on exit.
template <int N> struct YFan {
    static kw_status run(kw_plan *P, Spec4 bufs, int kz0, int nkz) {
        return YLaunch<N>::run_fan(P, bufs, kz0, nkz, P->dd_pos[1], P->dd_pos[2]);
    }
};

kw_status grad_group(kw_plan *P) {
    OpSet ops{};
    ops.n = P->D;
    for (int i = 0; i < P->D; ++i) { ops.kind[i] = OP_GRAD_POS; ops.axis[i] = P->comp_axis[i]; }
    const bool fan3 = P->static_x && P->static_y && P->g.N1 > 1 && P->D == 3 && P->comp_axis[0] == 0 &&
                      P->comp_axis[1] == 1 && P->comp_axis[2] == 2 && P->tw[0] && P->tw[1];
    if (!fan3) return yxy_group(P, specs(P, 0, 1, 2), P->D, ops, true);
    // 3-D: the y and z outputs share one inverse x-transform (their
    // multipliers are constant along x) and one read of it in the inverse
    // y-pass (ks_ypass_fan)
    const Spec4 bufs = specs(P, 0, 1, 2);
    const int nch = P->kz_chunks;
    const int N2h = P->g.N2h;
    for (int c = 0; c < nch; ++c) {
        const int kz0 = (int)((long long)N2h * c / nch), kz1 = (int)((long long)N2h * (c + 1) / nch);
        KW_TRY(ypass(P, false, bufs, 1, kz0, kz1 - kz0));
        KW_TRY(xpass(P, bufs, ops, 2, 1, kz0, kz1 - kz0));
        Scope s(P, KW_KCLASS_YPASS);
        KW_TRY(dispatch<YFan>(P->g.N1, P, bufs, kz0, kz1 - kz0));
    }
    return KW_OK;
}

// real(ifftn(source_kappa .* fftn(field))) into out, via spec[3]
kw_status source_filter(kw_plan *P, const float *field, float *out) {
    {
        Scope s(P, KW_KCLASS_SOURCE);
        KW_TRY(zr2c(P, field, P->spec[3]));
    }
    Spec4 b{};
    b.p[0] = P->spec[3];
    OpSet ops{};
    ops.n = 1;
    ops.kind[0] = OP_SRC_KAPPA;
    KW_TRY(yxy_group(P, b, 1, ops, false));
    Scope s(P, KW_KCLASS_SOURCE);
    KW_TRY(zc2r(P, P->spec[3], out));
    return KW_OK;
}

// general additive sources: this step's filtered source field
kw_status general_source(kw_plan *P, SourceDev &S, int comp, int t) {
    if (!S.dense_general || t > S.T[comp] || !S.sig[comp]) return KW_OK;
    {
        Scope s(P, KW_KCLASS_SOURCE);
        k_scatter_source<<<(S.npts + 255) / 256, 256, 0, P->stream>>>(S.pos, S.row, S.npts, S.sig[comp], S.nsig,
                                                                      S.scratch, P->d_t, S.T[comp]);
        KW_TRY(launched(P));
    }
    return source_filter(P, S.scratch, S.Ft[comp]);
}

DenseSrc dense_of(const SourceDev &S, int comp) {
    DenseSrc d{};
    if (S.dense_fast && S.sig[comp]) {
        d.F = S.F;
        d.sig = S.sig[comp];
        d.T = S.T[comp];
    } else if (S.dense_general && S.sig[comp]) {
        d.F = S.Ft[comp];
        d.sig = nullptr;
        d.T = S.T[comp];
    }
    return d;
}

SparseSrc sparse_of(const SourceDev &S) {
    SparseSrc s{};
    if (!S.present || S.dense_fast || S.dense_general) return s;
    s.off = S.csr_off;
    s.cell = S.csr_cell;
    s.row = S.csr_row;
    for (int i = 0; i < 3; ++i) s.sig[i] = S.sig[i];
    s.nsig = S.nsig;
    for (int i = 0; i < 3; ++i) s.T[i] = S.T[i];
    s.mode = S.mode == KW_SOURCE_DIRICHLET ? 0 : 1;
    return s;
}

TRSrc tr_of(kw_plan *P) {
    TRSrc r{};
    if (!P->time_rev) return r;
    r.off = P->tr_off;
    r.cell = P->tr_cell;
    r.row = P->tr_row;
    r.data = P->tr_data;
    r.M = P->M;
    r.Nt = P->Nt;
    return r;
}


kw_status stage_u(kw_plan *P, int init, int t) {
    StageU a{};
    a.g = P->g;
    a.axz = P->fft[2];
    a.PL = P->PL_u;
    for (int i = 0; i < 3; ++i) {
        a.spec.p[i] = P->spec[i];
        a.u[i] = P->u[i];
        a.u_out[i] = P->u_b[i];
        a.rho_sg_inv[i] = P->rsi[i];
        a.pml_sg[i] = P->pml_sg[i];
        a.comp_axis[i] = P->comp_axis[i];
        a.dense[i] = dense_of(P->usrc, i);
    }
    a.dt = (float)P->prob.dt;
    a.init = init;
    a.write_spec = 1;
    a.sparse = sparse_of(P->usrc);
    // components without a signal take no sparse input
    a.d_t = P->d_t;
    (void)t;
    Scope s(P, KW_KCLASS_ZSTAGE_U);
    KW_TRY(dispatch<ULaunch>(P->static_z ? P->g.N2 : 0, P, a));
    for (int i = 0; i < 3; ++i) std::swap(P->u[i], P->u_b[i]);   // the new velocity becomes current
    return KW_OK;
}

kw_status stage_r(kw_plan *P, int write_spec) {
    StageR a{};
    a.g = P->g;
    a.axz = P->fft[2];
    a.PL = P->PL_r;
    a.D = P->D;
    for (int i = 0; i < 3; ++i) {
        a.spec.p[i] = P->spec[i];
        a.rho[i] = P->rho[i];
        a.rho_out[i] = P->rho_b[i];
        a.pml[i] = P->pml[i];
        a.comp_axis[i] = P->comp_axis[i];
    }
    a.p = P->p;
    a.srho = P->srho;
    a.rho0 = P->rho0;
    a.c0 = P->c0;
    a.BonA = P->bona;
    a.c2tau = P->c2tau;
    a.dt = (float)P->prob.dt;
    a.nonlinear = P->prob.nonlinear_flag ? 1 : 0;
    a.eos = P->prob.absorbing_flag;
    a.has_tau = P->has_tau;
    a.has_eta = P->has_eta;
    a.dense = dense_of(P->psrc, 0);
    a.sparse = sparse_of(P->psrc);
    a.tr = P->absorbing ? TRSrc{} : tr_of(P);
    a.write_spec = write_spec;
    a.d_t = P->d_t;
    Scope s(P, KW_KCLASS_ZSTAGE_R);
    KW_TRY(dispatch<RLaunch>(P->static_z ? P->g.N2 : 0, P, a));
    for (int i = 0; i < 3; ++i) std::swap(P->rho[i], P->rho_b[i]);   // the new values become current
    return KW_OK;
}

kw_status stage_p(kw_plan *P, int write_spec) {
    StageP a{};
    a.g = P->g;
    a.axz = P->fft[2];
    a.PL = P->PL_p;
    a.D = P->D;
    for (int i = 0; i < 3; ++i) {
        a.spec.p[i] = P->spec[i];
        a.rho[i] = P->rho[i];
    }
    a.p = P->p;
    a.srho = P->srho;
    a.c0 = P->c0;
    a.rho0 = P->rho0;
    a.c2tau = P->c2tau;
    a.c2eta = P->c2eta;
    a.has_tau = P->has_tau;
    a.has_eta = P->has_eta;
    a.tr = tr_of(P);
    a.write_spec = write_spec;
    a.d_t = P->d_t;
    Scope s(P, KW_KCLASS_ZSTAGE_P);
    return dispatch<PLaunch>(P->static_z ? P->g.N2 : 0, P, a);
}

kw_status sensors(kw_plan *P, int t) {
    if (P->no_record || P->time_rev || t < P->record_start) return KW_OK;
    if (P->M > 0) {
        SensorArgs a{};
        a.M = P->M;
        a.K = P->K;
        a.idx = P->sidx_all ? nullptr : P->sidx;
        a.w = P->sw;
        a.nfield = 1 + P->D;
        a.field[0] = P->p;
        for (int i = 0; i < P->D; ++i) a.field[1 + i] = P->u[i];
        bool any = false;
        for (int f = 0; f < 4; ++f) {
            a.series[f] = P->o_series[f];
            a.vmax[f] = P->o_max[f];
            a.vmin[f] = P->o_min[f];
            a.vsq[f] = P->o_sq[f];
            // a field without outputs is not read
            if (!(a.series[f] || a.vmax[f] || a.vmin[f] || a.vsq[f])) a.field[f] = nullptr;
            any = any || a.field[f];
        }
        if (any) {
            Scope s(P, KW_KCLASS_SENSOR);
            a.record_start = P->record_start;
            a.ring = P->stream_cols;
            a.d_t = P->d_t;
            if (P->sidx_all && P->M % 4 == 0)
                k_sensor_all<<<(P->M / 4 + 255) / 256, 256, 0, P->stream>>>(a);
            else
                k_sensor<<<(P->M + 255) / 256, 256, 0, P->stream>>>(a);
            KW_TRY(launched(P));
        }
        if (P->o_uns[0]) {
            // velocity on the regular grid: real(ifft(shift_neg_i fft(u_i)))
            // along the component's own axis (extractSensorData.m:41-57),
            // applied as a spectral operator that depends on k_i only
            for (int i = 0; i < P->D; ++i) {
                const float *src = P->u[i];
                if (P->prob.use_sg) {
                    KW_TRY(zr2c(P, P->u[i], P->spec[3]));
                    Spec4 b{};
                    b.p[0] = P->spec[3];
                    OpSet ops{};
                    ops.n = 1;
                    ops.kind[0] = OP_SHIFT_NEG;
                    ops.axis[0] = P->comp_axis[i];
                    KW_TRY(yxy_group(P, b, 1, ops, false));
                    KW_TRY(zc2r(P, P->spec[3], P->ush));
                    src = P->ush;
                }
                Scope s(P, KW_KCLASS_SENSOR);
                k_gather_series<<<(P->M + 255) / 256, 256, 0, P->stream>>>(src, P->sidx_all ? nullptr : P->sidx,
                                                                          P->sw, P->M, P->K, P->o_uns[i],
                                                                          P->d_t, P->record_start);
                KW_TRY(launched(P));
            }
        }
    }
    bool any_all = false;
    for (int f = 0; f < 4; ++f) any_all = any_all || P->o_amax[f] || P->o_amin[f];
    if (any_all) {
        RegionArgs r{};
        r.nfield = 1 + P->D;
        r.field[0] = P->p;
        for (int i = 0; i < P->D; ++i) r.field[1 + i] = P->u[i];
        for (int f = 0; f < 4; ++f) {
            r.vmax[f] = P->o_amax[f];
            r.vmin[f] = P->o_amin[f];
        }
        for (int a = 0; a < 3; ++a) {
            r.lo[a] = P->in_lo[a];
            r.n[a] = P->in_n[a];
        }
        r.g = P->g;
        r.record_start = P->record_start;
        r.d_t = P->d_t;
        Scope s(P, KW_KCLASS_SENSOR);
        const long long blocks = std::min<long long>((P->in_count + 255) / 256, 148 * 16);
        k_region<<<(int)blocks, 256, 0, P->stream>>>(r);
        KW_TRY(launched(P));
    }
    return KW_OK;
}

// ---- start of the loop ------------------------------------------------------
kw_status zero_state(kw_plan *P) {
    const size_t N = (size_t)P->g.N, Nh = (size_t)P->g.Nh;
    KW_CUDA(cudaMemsetAsync(P->p, 0, N * sizeof(float), P->stream));
    // nonlinear mass coefficient q = 2 sum(rho) + rho0 of the zero state
    k_fill_med<<<(unsigned)std::min<size_t>((N + 255) / 256, 148 * 16), 256, 0, P->stream>>>(P->srho, P->rho0, (long long)N);
    KW_TRY(launched(P));
    for (int i = 0; i < P->D; ++i) {
        KW_CUDA(cudaMemsetAsync(P->rho[i], 0, N * sizeof(float), P->stream));
        KW_CUDA(cudaMemsetAsync(P->u[i], 0, N * sizeof(float), P->stream));
    }
    for (int i = 0; i < 4; ++i)
        if (P->spec[i]) KW_CUDA(cudaMemsetAsync(P->spec[i], 0, Nh * sizeof(float2), P->stream));
    const int one = 1;
    KW_CUDA(cudaMemcpyAsync(P->d_t, &one, sizeof(int), cudaMemcpyHostToDevice, P->stream));
    P->t = 1;
    P->started = false;
    P->ck_saved = 0;
    P->ck_valid = false;
    return KW_OK;
}

kw_status save_state(kw_plan *P, float *dst);

kw_status start(kw_plan *P) {
    if (P->time_rev) {
        // kspaceFirstOrder3D.m:772-788 at t = 1
        k_tr_start<<<(P->M + 255) / 256, 256, 0, P->stream>>>(P->sidx, P->M, P->tr_data, P->Nt, P->c0, P->rho0, P->p,
                                                              P->rho[0], P->rho[1], P->rho[2], P->srho, P->D);
        KW_TRY(launched(P));
        KW_TRY(zr2c(P, P->p, P->spec[0]));
        KW_TRY(grad_group(P));
    }
    P->started = true;
    return KW_OK;
}

// one time step t (1-based); steps counted on the device by d_t as well
kw_status run_step(kw_plan *P) {
    const int t = P->t;
    const bool need_grad = t < P->index_end;
    if (t == 1 && P->p0) {
        // p0 initial condition (kspaceFirstOrder3D.m:1023-1040): the first
        // step's update is overwritten, so the state is set directly.
        KW_CUDA(cudaMemcpyAsync(P->p, P->p0_dev, (size_t)P->g.N * sizeof(float), cudaMemcpyDeviceToDevice, P->stream));
        k_init_rho<<<1024, 256, 0, P->stream>>>(P->p0_dev, P->c0, P->rho0, P->rho[0], P->rho[1], P->rho[2], P->srho,
                                                P->g.N, P->D);
        KW_TRY(launched(P));
        KW_TRY(zr2c(P, P->p, P->spec[0]));
        KW_TRY(grad_group(P));
        KW_TRY(stage_u(P, 1, t));
    } else {
        for (int c = 0; c < P->D; ++c) KW_TRY(general_source(P, P->usrc, c, t));
        KW_TRY(stage_u(P, 0, t));
        // divergence: real(ifftn(dd_neg_i kappa fftn(u_i))), every component in
        // one launch per pass
        {
            OpSet ops{};
            ops.n = P->D;
            for (int i = 0; i < P->D; ++i) { ops.kind[i] = OP_GRAD_NEG; ops.axis[i] = P->comp_axis[i]; }
            KW_TRY(yxy_group(P, specs(P, 0, 1, 2), P->D, ops, false));
        }
        KW_TRY(general_source(P, P->psrc, 0, t));
        if (!P->absorbing) {
            KW_TRY(stage_r(P, need_grad ? 1 : 0));
        } else {
            KW_TRY(stage_r(P, 0));
            OpSet o2{};
            if (P->has_tau) o2.kind[o2.n++] = OP_NABLA1;
            if (P->has_eta) o2.kind[o2.n++] = OP_NABLA2;
            if (o2.n) KW_TRY(yxy_group(P, specs(P, 0, 1), o2.n, o2, false));
            KW_TRY(stage_p(P, need_grad ? 1 : 0));
        }
        if (need_grad) KW_TRY(grad_group(P));
    }
    KW_TRY(sensors(P, t));
    k_step_advance<<<1, 1, 0, P->stream>>>(P->d_t);
    KW_TRY(launched(P));
    P->t += 1;
    return KW_OK;
}

// CSR of points per z-tile of width TX = 2*PL (tile = x/TX + ntx*y)
kw_status build_csr(kw_plan *P, const std::vector<long long> &pos, const std::vector<int> &row, int PL, int **off,
                    int **cell, int **rowd) {
    const int TX = 2 * PL;
    const int ntx = (P->g.N0 + TX - 1) / TX;
    const int ntiles = ntx * P->g.N1;
    std::vector<int> cnt(ntiles + 1, 0);
    std::vector<int> tile_of(pos.size()), cell_of(pos.size());
    for (size_t i = 0; i < pos.size(); ++i) {
        const long long gi = pos[i];
        const int x = (int)(gi % P->g.N0);
        const long long q = gi / P->g.N0;
        const int y = (int)(q % P->g.N1);
        const int z = (int)(q / P->g.N1);
        tile_of[i] = x / TX + ntx * y;
        cell_of[i] = z * TX + (x % TX);
        cnt[tile_of[i] + 1]++;
    }
    for (int i = 0; i < ntiles; ++i) cnt[i + 1] += cnt[i];
    std::vector<int> fill(cnt.begin(), cnt.end() - 1), cells(pos.size()), rows(pos.size());
    for (size_t i = 0; i < pos.size(); ++i) {
        const int k = fill[tile_of[i]]++;
        cells[k] = cell_of[i];
        rows[k] = row[i];
    }
    KW_TRY(pupload(P, off, cnt.data(), cnt.size()));
    KW_TRY(pupload(P, cell, cells.data(), cells.size()));
    KW_TRY(pupload(P, rowd, rows.data(), rows.size()));
    return KW_OK;
}

kw_status setup_source(kw_plan *P, SourceDev &S, const kw_source *src, int ncomp, int PL) {
    // src[0..ncomp-1] share mode, points and signal index (u_mask is shared)
    int first = -1;
    for (int c = 0; c < ncomp; ++c)
        if (src[c].num_time_samples > 0) { first = c; break; }
    if (first < 0) return KW_OK;
    const kw_source &s0 = src[first];
    S.present = true;
    S.mode = s0.mode;
    if (S.mode < 0 || S.mode > 2) return fail(KW_ERR_INVALID, "source mode must be 0 (dirichlet), 1 (additive-no-correction) or 2 (additive)");
    S.npts = (int)s0.num_points;
    if (S.npts <= 0 || !s0.index) return fail(KW_ERR_INVALID, "source mask must have at least one element set to 1.");
    std::vector<long long> pos(S.npts);
    for (int i = 0; i < S.npts; ++i) {
        const uint64_t v = s0.index[i];
        if (v < 1 || v > (uint64_t)P->g.N) return fail(KW_ERR_INVALID, "source index %llu outside the grid", (unsigned long long)v);
        if (i > 0 && v <= s0.index[i - 1]) return fail(KW_ERR_INVALID, "source indices must be increasing (find(mask) order)");
        pos[i] = (long long)v - 1;
    }
    // components may differ in row count when the mask is binary: one row
    // drives every point (MATLAB's source.ux(':', t) scalar expansion), or one
    // row per point (kspaceFirstOrder_inputChecking.m:966-984)
    S.nsig = 1;
    for (int c = 0; c < ncomp; ++c)
        if (src[c].num_time_samples > 0) S.nsig = std::max(S.nsig, (int)src[c].num_signals);
    std::vector<int> row(S.npts);
    for (int i = 0; i < S.npts; ++i) {
        if (s0.signal_index) {
            const uint64_t r = s0.signal_index[i];
            if (r < 1 || r > (uint64_t)S.nsig) return fail(KW_ERR_INVALID, "source signal index out of range");
            row[i] = (int)r - 1;
        } else if (S.nsig == 1) {
            row[i] = 0;
        } else if (S.nsig == S.npts) {
            row[i] = i;
        } else {
            return fail(KW_ERR_INVALID, "The number of time series in the source must match the number of source elements in the mask.");
        }
    }
    bool one_row = true;
    for (int i = 1; i < S.npts; ++i) one_row = one_row && row[i] == row[0];
    const bool fast = S.mode == KW_SOURCE_ADDITIVE && one_row;
    for (int c = 0; c < ncomp; ++c) {
        if (src[c].num_time_samples == 0) continue;
        const int ns = (int)src[c].num_signals;
        if (!src[c].input || (ns != S.nsig && (ns != 1 || s0.signal_index)))
            return fail(KW_ERR_INVALID, "velocity source components must share the mask and the number of signals");
        S.T[c] = (int)std::min<uint64_t>(src[c].num_time_samples, (uint64_t)P->Nt);
        const size_t len = src[c].num_time_samples;
        if (fast) {
            // one signal drives every point: keep that row only
            std::vector<float> h(S.T[c]);
            for (int tt = 0; tt < S.T[c]; ++tt) h[tt] = src[c].input[(ns == 1 ? 0 : row[0]) + (size_t)ns * tt];
            KW_TRY(pupload(P, &S.sig[c], h.data(), h.size()));
        } else if (ns == S.nsig) {
            KW_TRY(pupload(P, &S.sig[c], src[c].input, (size_t)S.nsig * len));
        } else {
            // a one-row component beside per-point ones: the row for every point
            std::vector<float> h((size_t)S.nsig * len);
            for (size_t tt = 0; tt < len; ++tt)
                for (int r = 0; r < S.nsig; ++r) h[r + (size_t)S.nsig * tt] = src[c].input[tt];
            KW_TRY(pupload(P, &S.sig[c], h.data(), h.size()));
        }
    }
    KW_TRY(pupload(P, &S.pos, pos.data(), pos.size()));
    KW_TRY(pupload(P, &S.row, row.data(), row.size()));
    const size_t N = (size_t)P->g.N;
    if (S.mode == KW_SOURCE_ADDITIVE) {
        if (fast) {
            // rho += s(t) real(ifftn(source_kappa fftn(mask))) -- the source
            // matrix is s(t) times the mask, so filtering the mask once is the
            // same linear operation (kspaceFirstOrder3D.m:941-952)
            S.dense_fast = true;
            KW_TRY(palloc(P, &S.F, N));
            float *m = nullptr;
            KW_CUDA(cudaMallocAsync((void **)&m, N * sizeof(float), P->stream));
            KW_CUDA(cudaMemsetAsync(m, 0, N * sizeof(float), P->stream));
            k_set_points<<<(S.npts + 255) / 256, 256, 0, P->stream>>>(S.pos, S.npts, 1.0f, m);
            KW_TRY(launched(P));
            kw_status st = source_filter(P, m, S.F);
            cudaFreeAsync(m, P->stream);
            KW_TRY(st);
        } else {
            S.dense_general = true;
            KW_TRY(palloc(P, &S.scratch, N));
            for (int c = 0; c < ncomp; ++c)
                if (S.sig[c]) KW_TRY(palloc(P, &S.Ft[c], N));
        }
    } else {
        KW_TRY(build_csr(P, pos, row, PL, &S.csr_off, &S.csr_cell, &S.csr_row));
    }
    return KW_OK;
}

int choose_pl(int cap, int N0, int N1, int N2) {
    int pl = std::max(1, std::min(16, cap / N2));
    // keep at least two blocks per SM where the grid allows it
    while (pl > 1 && (long long)((N0 + 2 * pl - 1) / (2 * pl)) * N1 < 2 * 148) pl /= 2;
    return pl;
}

void plan_tiles(kw_plan *P) {
    const Geom &g = P->g;
    // compile-time kernels where the axis length has one; their tiles are
    // ks_lines(n) lines wide, or ks_narrow(n) when full tiles would give less
    // than one block per SM (small grids)
    constexpr long long kWave = 148;
    P->static_z = g.vec2 && is_static(g.N2);
    if (P->static_z) {
        int pl = ks_lines(g.N2);
        if ((long long)((g.N0 + 2 * pl - 1) / (2 * pl)) * g.N1 < kWave) pl = ks_narrow(g.N2);
        P->PL_u = P->PL_z = P->PL_p = P->PL_r = pl;
    } else {
        P->PL_u = choose_pl(kCap, g.N0, g.N1, g.N2);
        P->PL_z = P->PL_u;
        P->PL_r = choose_pl(kCap / 2, g.N0, g.N1, g.N2);
        P->PL_p = choose_pl(kCap, g.N0, g.N1, g.N2);
    }
    P->static_y = g.N1 > 1 && is_static(g.N1);
    if (P->static_y) {
        P->TY = ks_lines(g.N1);
        if ((long long)((g.N0 + P->TY - 1) / P->TY) * g.N2h < kWave) P->TY = ks_narrow(g.N1);
    } else {
        int ty = 1;
        while (ty * 2 <= 32 && ty * 2 * g.N1 <= kCap) ty *= 2;
        P->TY = ty;
    }
    const int lines = g.N1 * g.N2h;
    P->static_x = is_static(g.N0);
    if (P->static_x) {
        P->NL = ks_xlines(g.N0);
        if ((lines + P->NL - 1) / P->NL < kWave) P->NL = ks_xnarrow(g.N0);
    } else {
        P->NL = std::max(1, kCap / g.N0);
        if (P->NL > lines) P->NL = lines;
        while (P->NL > 1 && (lines + P->NL - 1) / P->NL < 2 * kWave) P->NL /= 2;
    }
    {
        // chunk the y / x / y groups so one chunk of a half spectrum (written
        // and re-read in place) stays well inside the 126 MB L2
        // measured on B200 at 256^3: smaller chunks only add launches and
        // tail waves, so the default is one chunk (KW_KZ_CHUNK_MB > 0 sets a size)
        double mb = 0.0;
        if (const char *e = getenv("KW_KZ_CHUNK_MB")) mb = atof(e);
        const double bytes = (double)g.Nh * sizeof(float2);
        int nch = mb > 0 ? (int)std::ceil(bytes / (mb * 1e6)) : 1;
        nch = std::max(1, std::min(nch, g.N2h));
        // every chunk must still fill the GPU
        while (nch > 1 && (long long)(g.N2h / nch) * g.N1 / std::max(1, P->NL) < kWave) --nch;
        P->kz_chunks = nch;
    }
}

// ---- tile autotuner ------------------------------------------------------
// The compile-time kernels of each pass class (z-stages, y-pass, x-pass)
// exist with a full tile (ks_lines(n) lines), a half one (ks_half(n)) and a
// narrow one (ks_narrow(n), a quarter).  plan_tiles picks by a rule (narrow
// when full tiles give fewer blocks than SMs); the autotuner then times a few
// steps with each other width of one class at a time and keeps what is
// faster, once per grid shape and tile-relevant structure per process.  Tile widths change how lines are grouped into blocks, never the
// arithmetic of a line, so results are identical whichever is chosen.
// z-tile widths of stages U, R and P (each chooses its own), y and x widths
struct TileChoice {
    int PLu, PLr, PLp, TY, NL;
};
std::mutex g_tune_mu;
std::map<std::array<int, 5>, TileChoice> g_tune;

TileChoice tiles_of(const kw_plan *P) { return TileChoice{P->PL_u, P->PL_r, P->PL_p, P->TY, P->NL}; }
void set_tiles(kw_plan *P, const TileChoice &c) {
    P->PL_u = P->PL_z = c.PLu;
    P->PL_r = c.PLr;
    P->PL_p = c.PLp;
    P->TY = c.TY;
    P->NL = c.NL;
}

// device milliseconds per step of the current tiles (steps run directly,
// not recording; the state is reset by the caller)
kw_status time_steps(kw_plan *P, int n, float *ms) {
    KW_TRY(zero_state(P));
    P->started = true;
    KW_TRY(run_step(P));   // warm-up (and the t = 1 special cases)
    cudaEvent_t a, b;
    KW_CUDA(cudaEventCreate(&a));
    KW_CUDA(cudaEventCreate(&b));
    KW_CUDA(cudaEventRecord(a, P->stream));
    kw_status st = KW_OK;
    for (int k = 0; k < n && st == KW_OK; ++k) st = run_step(P);
    cudaEventRecord(b, P->stream);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    KW_TRY(st);
    *ms = t / (float)n;
    return KW_OK;
}

kw_status autotune_tiles(kw_plan *P) {
    if (const char *e = getenv("KW_AUTOTUNE"))
        if (atoi(e) == 0) return KW_OK;
    const Geom &g = P->g;
    // z tiles fix the per-tile lists of sparse sources and time reversal, so
    // those plans keep the rule's z tiles
    const bool tune_z = P->static_z && !P->time_rev && !(P->psrc.present && !P->psrc.dense_fast && !P->psrc.dense_general) &&
                        !(P->usrc.present && !P->usrc.dense_fast && !P->usrc.dense_general);
    const bool tune_y = P->static_y;
    const bool tune_x = P->static_x;
    if (!tune_z && !tune_y && !tune_x) return KW_OK;
    if (P->Nt < 4 || P->time_rev) return KW_OK;
    const std::array<int, 5> key = {g.N0, g.N1, g.N2, P->absorbing ? 1 : 0, tune_z ? 1 : 0};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            set_tiles(P, it->second);
            return KW_OK;
        }
    }
    const bool keep_no_record = P->no_record;
    P->no_record = true;
    TileChoice best = tiles_of(P);
    float best_ms = 0.f;
    kw_status st = time_steps(P, 2, &best_ms);
    // the other widths of one class at a time (full, half, quarter): stage U,
    // stage R, stage P, y-pass, x-pass
    for (int cls = 0; cls < 5 && st == KW_OK; ++cls) {
        int widths[3];
        int *slot = nullptr;
        TileChoice base = best;
        if (cls <= 2 && tune_z) {
            widths[0] = ks_lines(g.N2); widths[1] = ks_half(g.N2); widths[2] = ks_narrow(g.N2);
            slot = cls == 0 ? &base.PLu : (cls == 1 ? &base.PLr : &base.PLp);
        } else if (cls == 3 && tune_y) {
            widths[0] = ks_lines(g.N1); widths[1] = ks_half(g.N1); widths[2] = ks_narrow(g.N1);
            slot = &base.TY;
        } else if (cls == 4 && tune_x) {
            widths[0] = ks_xlines(g.N0); widths[1] = ks_xhalf(g.N0); widths[2] = ks_xnarrow(g.N0);
            slot = &base.NL;
        } else {
            continue;
        }
        const int current = *slot;
        for (int w : widths) {
            if (w == current || st != KW_OK) continue;
            TileChoice c = base;
            *(cls == 0 ? &c.PLu : cls == 1 ? &c.PLr : cls == 2 ? &c.PLp : cls == 3 ? &c.TY : &c.NL) = w;
            set_tiles(P, c);
            float ms = 0.f;
            st = time_steps(P, 2, &ms);
            if (st == KW_OK && ms < 0.97f * best_ms) {
                best = c;
                best_ms = ms;
            }
        }
    }
    set_tiles(P, best);
    P->no_record = keep_no_record;
    KW_TRY(st);
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = best;
    return KW_OK;
}

// medium.alpha_filter multiplies both absorption operators in natural
// wavenumber order: nabla <- ifftshift(fftshift(nabla) .* alpha_filter)
// (createAbsorptionVariables.m:56-76), i.e. the operator in FFT order times
// ifftshift(alpha_filter).  real(ifftn(op X)) of a real field sees only the
// Hermitian part of a real op, (f(k) + f(-k)) / 2, which is tabulated on the
// z-half spectrum (element (x, y, kz) at x + N0 (y + N1 kz)) in FP64 and
// stored FP32.
kw_status build_alpha_filter(kw_plan *P, const kw_problem &q, const int *phys_of_int) {
    const Geom &g = P->g;
    const uint64_t dims[3] = {q.Nx, q.Ny, q.dim == 3 ? q.Nz : 1};
    // user array element at physical (x, y, z), natural order
    auto at = [&](long long x, long long y, long long z) -> double {
        long long i;
        if (q.array_order == KW_ROW_MAJOR)
            i = q.dim == 3 ? z + (long long)dims[2] * (y + (long long)dims[1] * x) : y + (long long)dims[1] * x;
        else
            i = x + (long long)dims[0] * (y + (long long)dims[1] * z);
        return (double)q.alpha_filter[i];
    };
    const int n[3] = {g.N0, g.N1, g.N2};
    std::vector<float> h((size_t)g.Nh);
    for (int i2 = 0; i2 < g.N2h; ++i2)
        for (int i1 = 0; i1 < g.N1; ++i1)
            for (int i0 = 0; i0 < g.N0; ++i0) {
                const int fi[3] = {i0, i1, i2};
                long long pos[3] = {0, 0, 0}, neg[3] = {0, 0, 0};   // physical (x, y, z), natural order
                for (int a = 0; a < 3; ++a) {
                    const int pa = phys_of_int[a];
                    if (pa < 0) continue;
                    pos[pa] = (fi[a] + n[a] / 2) % n[a];
                    neg[pa] = ((n[a] - fi[a]) % n[a] + n[a] / 2) % n[a];
                }
                const double v = 0.5 * (at(pos[0], pos[1], pos[2]) + at(neg[0], neg[1], neg[2]));
                h[(size_t)i0 + (size_t)g.N0 * (i1 + (size_t)g.N1 * i2)] = (float)v;
            }
    float *d = nullptr;
    KW_TRY(pupload(P, &d, h.data(), h.size()));
    P->op.filt = d;
    P->op.n0 = g.N0;
    P->op.n1 = g.N1;
    return KW_OK;
}

// The transducer's delayed, apodised drive (kspaceFirstOrder3D.m:888-904):
// point i adds apodization[i] * s[delay[i] + t - 1] to ux while
// t <= L - max(delay), which is an additive-no-correction ux source whose
// row i is that delayed series; the rows are formed here and run through
// the sparse source path of the momentum stage.
kw_status transducer_as_source(kw_plan *P, const kw_problem &q, kw_source us[3], std::vector<float> &sig) {
    const kw_transducer_source &ts = q.transducer_source;
    for (int c = 0; c < 3; ++c) us[c] = kw_source{};
    if (q.dim != 3) return fail(KW_ERR_INVALID, "Transducer inputs are only compatible with 3D simulations.");
    for (int c = 0; c < 3; ++c)
        if (q.u_source[c].num_time_samples)
            return fail(KW_ERR_INVALID, "a transducer source excludes source.ux / uy / uz");
    if (!ts.index || !ts.delay || !ts.input_signal || ts.signal_length == 0)
        return fail(KW_ERR_INVALID, "transducer source: index, delay and input_signal must be given");
    uint64_t dmax = 0;
    for (uint64_t i = 0; i < ts.num_points; ++i) dmax = std::max(dmax, ts.delay[i]);
    if (dmax >= ts.signal_length) return KW_OK;   // never active (flags.transducer_source <= 0)
    const uint64_t T = std::min<uint64_t>(ts.signal_length - dmax, (uint64_t)P->Nt);
    const uint64_t n = ts.num_points;
    sig.assign((size_t)(n * T), 0.f);
    for (uint64_t t = 0; t < T; ++t)
        for (uint64_t i = 0; i < n; ++i)
            sig[i + n * t] = (ts.apodization ? ts.apodization[i] : 1.f) * ts.input_signal[ts.delay[i] + t];
    us[0].num_time_samples = T;
    us[0].mode = KW_SOURCE_ADDITIVE_NO_CORRECTION;
    us[0].num_points = n;
    us[0].index = ts.index;
    us[0].num_signals = n;
    us[0].signal_index = nullptr;
    us[0].input = sig.data();
    (void)P;
    return KW_OK;
}

kw_status create(const kw_problem *pr, kw_plan *P) {
    if (!pr) return fail(KW_ERR_INVALID, "problem is NULL");
    if (pr->abi_version != KW_ABI_VERSION) return fail(KW_ERR_INVALID, "abi_version %u, library expects %d", pr->abi_version, KW_ABI_VERSION);
    P->prob = *pr;
    const kw_problem &q = *pr;
    if (q.dim != 2 && q.dim != 3) return fail(KW_ERR_INVALID, "dim must be 2 or 3");
    P->D = q.dim;
    const uint64_t shp[3] = {q.Nx, q.Ny, q.dim == 3 ? q.Nz : 1};
    for (int a = 0; a < q.dim; ++a)
        if (shp[a] < 2 || shp[a] > 4096) return fail(KW_ERR_UNSUPPORTED, "grid size %llu along axis %d outside 2..4096", (unsigned long long)shp[a], a);
    if (q.dim == 3 && q.Nz < 2) return fail(KW_ERR_INVALID, "Nz must be >= 2 in 3D");
    if (q.Nt < 1) return fail(KW_ERR_INVALID, "Nt must be a positive integer.");
    if (!(q.dt > 0)) return fail(KW_ERR_INVALID, "dt must be positive.");
    if (!(q.dx > 0) || !(q.dy > 0) || (q.dim == 3 && !(q.dz > 0))) return fail(KW_ERR_INVALID, "grid spacing must be positive");
    const uint64_t pmls[3] = {q.pml_x_size, q.pml_y_size, q.pml_z_size};
    const double pmla[3] = {q.pml_x_alpha, q.pml_y_alpha, q.pml_z_alpha};
    for (int a = 0; a < q.dim; ++a)
        if (pmls[a] * 2 > shp[a]) return fail(KW_ERR_INVALID, "The size of the PML must be smaller than the size of the grid.");
    if (q.absorbing_flag < 0 || q.absorbing_flag > 2) return fail(KW_ERR_INVALID, "absorbing_flag must be 0, 1 or 2");
    if (q.absorbing_flag == KW_ABSORBING) {
        if (!(q.alpha_power >= 0 && q.alpha_power < 3)) return fail(KW_ERR_INVALID, "medium.alpha_power must be a real number between 0 and 3.");
        if (q.alpha_power == 1 && q.alpha_mode != KW_ALPHA_NO_DISPERSION)
            return fail(KW_ERR_INVALID, "The power law dispersion term in the equation of state is not valid for medium.alpha_power = 1.");
    }
    if (q.record_start_index < 1 || q.record_start_index > q.Nt) return fail(KW_ERR_INVALID, "sensor.record_start_index must be between 1 and the number of time steps.");

    // internal geometry: 2D (Nx, Ny) -> (Nx, 1, Ny)
    const double sp[3] = {q.dx, q.dy, q.dz};
    int phys_of_int[3];
    if (q.dim == 3) {
        for (int a = 0; a < 3; ++a) { P->N[a] = (int)shp[a]; P->d[a] = sp[a]; phys_of_int[a] = a; }
        P->comp_axis[0] = 0; P->comp_axis[1] = 1; P->comp_axis[2] = 2;
    } else {
        P->N[0] = (int)shp[0]; P->d[0] = sp[0]; phys_of_int[0] = 0;
        P->N[1] = 1; P->d[1] = 1.0; phys_of_int[1] = -1;
        P->N[2] = (int)shp[1]; P->d[2] = sp[1]; phys_of_int[2] = 1;
        P->comp_axis[0] = 0; P->comp_axis[1] = 2; P->comp_axis[2] = 1;
    }
    Geom &g = P->g;
    g.N0 = P->N[0]; g.N1 = P->N[1]; g.N2 = P->N[2];
    g.N2h = g.N2 / 2 + 1;
    g.N = (long long)g.N0 * g.N1 * g.N2;
    g.Nh = (long long)g.N0 * g.N1 * g.N2h;
    g.vec2 = (g.N0 % 2 == 0) ? 1 : 0;
    if (g.N > (1LL << 31) - 1) return fail(KW_ERR_UNSUPPORTED, "grid larger than 2^31 cells");

    P->Nt = (int)q.Nt;
    P->time_rev = q.time_reversal_input != nullptr;
    P->index_end = P->time_rev ? P->Nt - 1 : P->Nt;
    P->record_start = (int)q.record_start_index;
    P->num_rec = P->Nt - P->record_start + 1;
    P->p0 = q.p0_source_input != nullptr;
    if (P->p0 && q.p_source.num_time_samples > 0) return fail(KW_ERR_INVALID, "source.p0 and source.p can't be defined in the same simulation.");
    P->absorbing = q.absorbing_flag == KW_ABSORBING;

    P->device = q.device;
    {
        int ndev = 0;
        KW_CUDA(cudaGetDeviceCount(&ndev));
        if (q.device < 0 || q.device >= ndev) return fail(KW_ERR_INVALID, "device %d not present (%d devices)", q.device, ndev);
    }
    KW_CUDA(cudaSetDevice(P->device));
    {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, P->device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    KW_CUDA(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking));

    // FFT plans and operator tables (FP64 -> FP32)
    for (int a = 0; a < 3; ++a) {
        const int n = P->N[a];
        std::vector<int> rad;
        if (!factorize(n, rad)) return fail(KW_ERR_UNSUPPORTED, "grid size %d needs more than %d transform stages", n, kMaxStages);
        AxisFFT &f = P->fft[a];
        f.n = n;
        f.nstages = (int)rad.size();
        for (size_t s = 0; s < rad.size(); ++s) f.radix[s] = rad[s];
        std::vector<float2> tw(n);
        for (int m = 0; m < n; ++m) {
            const double ang = -2.0 * M_PI * (double)m / n;
            tw[m] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        }
        KW_TRY(pupload(P, &P->tw[a], tw.data(), tw.size()));
        f.tw = P->tw[a];

        std::vector<float2> dp(n), dn(n), sn(n, make_float2(1.f, 0.f));
        std::vector<float> k2(n);
        std::vector<float> pml(n, 1.f), pmlsg(n, 1.f);
        if (phys_of_int[a] >= 0) {
            const int pa = phys_of_int[a];
            const std::vector<double> k = kvec_fft(n, P->d[a]);
            std::vector<std::complex<double>> cp(n), cn(n);
            for (int i = 0; i < n; ++i) {
                const std::complex<double> ik(0.0, k[i]);
                if (q.use_sg) {
                    cp[i] = ik * std::exp(std::complex<double>(0.0, k[i] * P->d[a] / 2));
                    cn[i] = ik * std::exp(std::complex<double>(0.0, -k[i] * P->d[a] / 2));
                } else {
                    cp[i] = ik;
                    cn[i] = ik;
                }
                k2[i] = (float)(k[i] * k[i]);
            }
            // Hermitian part: real(ifftn(op X)) for real input X equals the
            // inverse transform of (op(k) + conj(op(-k)))/2 times X
            for (int i = 0; i < n; ++i) {
                const int j = (n - i) % n;
                const std::complex<double> hp = 0.5 * (cp[i] + std::conj(cp[j]));
                const std::complex<double> hn = 0.5 * (cn[i] + std::conj(cn[j]));
                dp[i] = make_float2((float)hp.real(), (float)hp.imag());
                dn[i] = make_float2((float)hn.real(), (float)hn.imag());
                if (q.use_sg) {
                    // record.x_shift_neg (createStorageVariables.m:89-114)
                    const std::complex<double> si = std::exp(std::complex<double>(0.0, -k[i] * P->d[a] / 2));
                    const std::complex<double> sj = std::exp(std::complex<double>(0.0, -k[j] * P->d[a] / 2));
                    const std::complex<double> hs = 0.5 * (si + std::conj(sj));
                    sn[i] = make_float2((float)hs.real(), (float)hs.imag());
                }
            }
            const std::vector<double> pr1 = get_pml(n, P->d[a], q.dt, q.c_ref, (int)pmls[pa], pmla[pa], false);
            const std::vector<double> pr2 = get_pml(n, P->d[a], q.dt, q.c_ref, (int)pmls[pa], pmla[pa], q.use_sg != 0);
            for (int i = 0; i < n; ++i) { pml[i] = (float)pr1[i]; pmlsg[i] = (float)pr2[i]; }
        } else {
            for (int i = 0; i < n; ++i) { dp[i] = make_float2(0, 0); dn[i] = make_float2(0, 0); k2[i] = 0.f; }
        }
        KW_TRY(pupload(P, &P->dd_pos[a], dp.data(), dp.size()));
        KW_TRY(pupload(P, &P->dd_neg[a], dn.data(), dn.size()));
        KW_TRY(pupload(P, &P->sh_neg[a], sn.data(), sn.size()));
        KW_TRY(pupload(P, &P->k2[a], k2.data(), k2.size()));
        KW_TRY(pupload(P, &P->pml[a], pml.data(), pml.size()));
        KW_TRY(pupload(P, &P->pml_sg[a], pmlsg.data(), pmlsg.size()));
        P->op.dd_pos[a] = P->dd_pos[a];
        P->op.dd_neg[a] = P->dd_neg[a];
        P->op.sh_neg[a] = P->sh_neg[a];
        P->op.k2[a] = P->k2[a];
    }
    P->op.kappa_a = (float)(q.c_ref * q.dt / 2.0);
    P->op.use_kspace = q.use_kspace ? 1 : 0;
    {
        // largest |k|^2 of the grid: the sum of each axis's largest k_i^2
        double kmax2 = 0.0;
        for (int a = 0; a < 3; ++a)
            if (phys_of_int[a] >= 0) {
                double m = 0.0;
                for (double k : kvec_fft(P->N[a], P->d[a])) m = std::max(m, k * k);
                kmax2 += m;
            }
        const double ka = q.c_ref * q.dt / 2.0;
        P->op.short_series = ka * ka * kmax2 <= 1.0 ? 1 : 0;
    }
    P->op.nabla1_exp = (float)(q.alpha_power - 2.0);
    P->op.nabla2_exp = (float)(q.alpha_power - 1.0);
    P->op.scale = (float)(1.0 / (double)g.N);

    plan_tiles(P);
    // one packed line of the real-to-complex axis fills at most one transform
    // tile (the runtime stage R then holds four such tiles, 128 KB)
    if (g.N2 > kCap) return fail(KW_ERR_UNSUPPORTED, "axis length %d above %d", g.N2, kCap);
    const size_t N = (size_t)g.N, Nh = (size_t)g.Nh;
    KW_TRY(palloc(P, &P->d_t, 1));
    KW_TRY(palloc(P, &P->d_err, 1));
    // the stage kernels stage their fields with TMA when the boxes fit the
    // rules: FP32 rows of 16-byte multiples (N0 % 4), a compile-time z length
    // (the half spectrum's rows come in boxes of at most 256 rows, each
    // 128-byte aligned: the launchers check that per tile width); KW_TMA=0
    // keeps the cp.async path
    {
        const char *e = getenv("KW_TMA");
        P->tma_r = P->static_z && g.N2 <= 512 && g.N0 % 4 == 0 && !(e && atoi(e) == 0) && have_encode_tiled();
    }
    KW_TRY(palloc(P, &P->p, N));
    for (int i = 0; i < P->D; ++i) {
        KW_TRY(palloc(P, &P->rho[i], N));
        KW_TRY(palloc(P, &P->rho_b[i], N));
        KW_TRY(palloc(P, &P->u[i], N));
        KW_TRY(palloc(P, &P->u_b[i], N));
    }
    KW_TRY(palloc(P, &P->srho, N));
    {
        // KW_BLOCK_GRAPHS=0: one graph per step on every grid
        const char *e = getenv("KW_BLOCK_GRAPHS");
        P->block_graphs = !(e && atoi(e) == 0);
    }
    P->rho_first = P->rho[0];
    P->u_first = P->u[0];
    if (const char *e = getenv("KW_GRAPHS")) P->use_graphs = atoi(e) != 0;
    const int nspec = 4;
    for (int i = 0; i < nspec; ++i) KW_TRY(palloc(P, &P->spec[i], Nh));

    // medium.  Grid arrays reach the device in column-major order (row-major
    // input is staged and transposed there); the derived arrays (1/rho0_sg,
    // c0^2 tau, c0^2 eta) are formed on the device in FP64, and the
    // positivity checks run there too
    const bool row_major = q.array_order == KW_ROW_MAJOR;
    if (q.array_order != KW_COLUMN_MAJOR && !row_major)
        return fail(KW_ERR_INVALID, "array_order must be %d (column-major) or %d (row-major)", KW_COLUMN_MAJOR, KW_ROW_MAJOR);
    TempDev tmp{P->stream, {}};
    float *stage_buf = nullptr;
    int *flags = nullptr;
    KW_TRY(tmp.get(&flags, 1));
    KW_CUDA(cudaMemsetAsync(flags, 0, sizeof(int), P->stream));
    const unsigned ew_blocks = (unsigned)((N + 255) / 256);
    auto put_grid = [&](float *dst, const float *host) -> kw_status {
        if (!row_major) {
            KW_CUDA(cudaMemcpyAsync(dst, host, N * sizeof(float), cudaMemcpyHostToDevice, P->stream));
            return KW_OK;
        }
        if (!stage_buf) KW_TRY(tmp.get(&stage_buf, N));
        KW_CUDA(cudaMemcpyAsync(stage_buf, host, N * sizeof(float), cudaMemcpyHostToDevice, P->stream));
        const int A = (int)shp[0], B = q.dim == 3 ? (int)shp[1] : 1, Cn = q.dim == 3 ? (int)shp[2] : (int)shp[1];
        k_rowmajor_to_col<<<dim3((Cn + 31) / 32, (A + 31) / 32, B), dim3(32, 8), 0, P->stream>>>(stage_buf, dst, A, B, Cn);
        return launched(P);
    };
    auto upload_grid = [&](float **dst, const float *host) -> kw_status {
        KW_TRY(palloc(P, dst, N));
        return put_grid(*dst, host);
    };
    if (q.c0) {
        KW_TRY(upload_grid(&P->c0_arr, q.c0));
        P->c0.arr = P->c0_arr;
        k_check_positive<<<ew_blocks, 256, 0, P->stream>>>(P->c0_arr, (long long)N, flags, 1);
        KW_TRY(launched(P));
    } else {
        P->c0.val = (float)q.c0_scalar;
        if (!(q.c0_scalar > 0)) return fail(KW_ERR_INVALID, "medium.sound_speed must be positive");
    }
    if (q.rho0) {
        KW_TRY(upload_grid(&P->rho0_arr, q.rho0));
        P->rho0.arr = P->rho0_arr;
        k_check_positive<<<ew_blocks, 256, 0, P->stream>>>(P->rho0_arr, (long long)N, flags, 2);
        KW_TRY(launched(P));
    } else {
        P->rho0.val = (float)q.rho0_scalar;
        if (!(q.rho0_scalar > 0)) return fail(KW_ERR_INVALID, "medium.density must be positive");
    }
    const float *sg[3] = {q.rho0_sgx, q.rho0_sgy, q.rho0_sgz};
    if (q.derive_rho0_sg && (!q.rho0 || sg[0] || sg[1] || sg[2]))
        return fail(KW_ERR_INVALID, "derive_rho0_sg needs an rho0 array and NULL rho0_sg pointers");
    for (int c = 0; c < P->D; ++c) {
        if (sg[c]) {
            KW_TRY(upload_grid(&P->rsi_arr[c], sg[c]));
            k_inv_rho_sg<<<ew_blocks, 256, 0, P->stream>>>(P->rsi_arr[c], P->rsi_arr[c], g, P->comp_axis[c], 0);
        } else if (q.rho0) {
            KW_TRY(palloc(P, &P->rsi_arr[c], N));
            k_inv_rho_sg<<<ew_blocks, 256, 0, P->stream>>>(P->rho0_arr, P->rsi_arr[c], g, P->comp_axis[c],
                                                          q.derive_rho0_sg ? 1 : 0);
        } else {
            P->rsi[c].val = (float)(1.0 / q.rho0_scalar);
            continue;
        }
        KW_TRY(launched(P));
        P->rsi[c].arr = P->rsi_arr[c];
    }
    if (q.nonlinear_flag) {
        if (q.BonA) {
            KW_TRY(upload_grid(&P->bona_arr, q.BonA));
            P->bona.arr = P->bona_arr;
        } else {
            P->bona.val = (float)q.BonA_scalar;
        }
    }
    if (q.absorbing_flag != KW_LOSSLESS) {
        // absorb_tau / absorb_eta of createAbsorptionVariables.m:29-101 in
        // FP64, multiplied by c0^2 so the equation of state needs no powers
        const bool stokes = q.absorbing_flag == KW_STOKES;
        const double y = stokes ? 2.0 : q.alpha_power;
        const double s0 = q.alpha_sign[0], s1 = q.alpha_sign[1];
        const double sg0 = s0 > 0 ? 1 : (s0 < 0 ? -1 : 0), sg1 = s1 > 0 ? 1 : (s1 < 0 ? -1 : 0);
        const double tanv = stokes ? 0.0 : std::tan(M_PI * q.alpha_power / 2.0);
        if (q.absorbing_flag == KW_ABSORBING) {
            P->has_tau = q.alpha_mode != KW_ALPHA_NO_ABSORPTION;
            P->has_eta = q.alpha_mode != KW_ALPHA_NO_DISPERSION;
        }
        if (q.c0 || q.alpha_coeff) {
            float *a_dev = nullptr;
            if (q.alpha_coeff) {
                KW_TRY(tmp.get(&a_dev, N));
                KW_TRY(put_grid(a_dev, q.alpha_coeff));
            }
            KW_TRY(palloc(P, &P->c2tau_arr, N));
            P->c2tau.arr = P->c2tau_arr;
            if (!stokes) {
                KW_TRY(palloc(P, &P->c2eta_arr, N));
                P->c2eta.arr = P->c2eta_arr;
            }
            k_absorb_coeffs<<<ew_blocks, 256, 0, P->stream>>>(P->c0_arr, q.c0_scalar, a_dev, q.alpha_coeff_scalar,
                                                             (long long)N, y, db2neper(1.0, y), stokes ? 1 : 0, tanv,
                                                             sg0, sg1, P->c2tau_arr, P->c2eta_arr);
            KW_TRY(launched(P));
        } else {
            const double anp = db2neper(q.alpha_coeff_scalar, y), c = q.c0_scalar;
            const double tau = stokes ? -2.0 * anp * c : -2.0 * anp * std::pow(c, y - 1.0);
            const double eta = stokes ? 0.0 : 2.0 * anp * std::pow(c, y) * tanv;
            P->c2tau.val = (float)(c * c * tau * sg0);
            P->c2eta.val = (float)(c * c * eta * sg1);
        }
    }
    if (q.alpha_filter) {
        if (q.absorbing_flag != KW_ABSORBING)
            return fail(KW_ERR_INVALID, "Input option medium.alpha_filter is not supported with medium.alpha_mode = 'stokes' "
                        "or without absorption.");
        KW_TRY(build_alpha_filter(P, q, phys_of_int));
    }
    if (P->p0) KW_TRY(upload_grid(&P->p0_dev, q.p0_source_input));
    {
        int hf = 0;
        KW_CUDA(cudaMemcpyAsync(&hf, flags, sizeof(int), cudaMemcpyDeviceToHost, P->stream));
        KW_CUDA(cudaStreamSynchronize(P->stream));
        if (hf & 1) return fail(KW_ERR_INVALID, "medium.sound_speed must be positive");
        if (hf & 2) return fail(KW_ERR_INVALID, "medium.density must be positive");
    }

    // sources
    KW_TRY(setup_source(P, P->psrc, &q.p_source, 1, P->PL_r));
    if (q.transducer_source.num_points) {
        kw_source us[3];
        std::vector<float> sig;
        KW_TRY(transducer_as_source(P, q, us, sig));
        KW_TRY(setup_source(P, P->usrc, us, P->D, P->PL_u));
    } else {
        KW_TRY(setup_source(P, P->usrc, q.u_source, P->D, P->PL_u));
    }

    // sensors
    P->rec = q.record;
    P->M = (int)q.sensor_num;
    P->K = q.sensor_vertices > 1 ? (int)q.sensor_vertices : 1;
    if (P->K > 8) return fail(KW_ERR_INVALID, "sensor_vertices must be at most 8");
    if (P->K > 1 && P->time_rev) return fail(KW_ERR_INVALID, "interpolated sensor points cannot drive time reversal");
    if (P->M > 0) {
        if (!q.sensor_mask_index) return fail(KW_ERR_INVALID, "sensor_mask_index is NULL");
        if (P->K > 1 && !q.sensor_weights) return fail(KW_ERR_INVALID, "sensor_weights is NULL");
        const size_t MK = (size_t)P->M * P->K;
        std::vector<long long> idx(MK);
        for (size_t m = 0; m < MK; ++m) {
            const uint64_t v = q.sensor_mask_index[m];
            if (v < 1 || v > (uint64_t)g.N) return fail(KW_ERR_INVALID, "sensor index %llu outside the grid", (unsigned long long)v);
            if (P->K == 1 && m > 0 && v <= q.sensor_mask_index[m - 1])
                return fail(KW_ERR_INVALID, "sensor indices must be increasing (find(mask) order)");
            idx[m] = (long long)v - 1;
        }
        KW_TRY(pupload(P, &P->sidx, idx.data(), idx.size()));
        // increasing indices in [0, N) number N only when they are 0 .. N-1
        P->sidx_all = P->K == 1 && (long long)P->M == g.N;
        if (P->K > 1) KW_TRY(pupload(P, &P->sw, q.sensor_weights, MK));
        if (P->time_rev) {
            KW_TRY(pupload(P, &P->tr_data, q.time_reversal_input, (size_t)P->M * P->Nt));
            std::vector<int> rows(P->M);
            for (int m = 0; m < P->M; ++m) rows[m] = m;
            const int PLf = P->absorbing ? P->PL_p : P->PL_r;
            KW_TRY(build_csr(P, idx, rows, PLf, &P->tr_off, &P->tr_cell, &P->tr_row));
        }
    } else if (P->time_rev) {
        return fail(KW_ERR_INVALID, "time reversal needs a sensor mask");
    }
    // inside region per internal axis
    {
        int lo[3] = {0, 0, 0}, n[3] = {P->N[0], P->N[1], P->N[2]};
        for (int a = 0; a < 3; ++a) {
            const int pa = phys_of_int[a];
            if (pa < 0) continue;
            const uint64_t l = q.inside_lo[pa], h = q.inside_hi[pa];
            if (l == 0 && h == 0) continue;
            if (l < 1 || h < l || h > (uint64_t)P->N[a]) return fail(KW_ERR_INVALID, "inside region out of range on axis %d", pa);
            lo[a] = (int)l - 1;
            n[a] = (int)(h - l + 1);
        }
        for (int a = 0; a < 3; ++a) { P->in_lo[a] = lo[a]; P->in_n[a] = n[a]; }
        P->in_count = (long long)n[0] * n[1] * n[2];
    }
    const bool tr = P->time_rev;
    const size_t ser = (size_t)P->M * P->num_rec;
    if (q.stream_to_disk) {
        // kspaceFirstOrder_inputChecking.m:1369-1375, checkOptionalInputs.m:353-374
        if (q.dim != 3) return fail(KW_ERR_INVALID, "Optional input 'StreamToDisk' is currently only compatible with 3D fluid simulations.");
        if (tr || P->M == 0)
            return fail(KW_ERR_INVALID, "The optional input 'StreamToDisk' is currently only compatible with forward "
                        "simulations using a non-zero sensor mask.");
        if (P->rec != KW_REC_P)
            return fail(KW_ERR_INVALID, "The optional input 'StreamToDisk' is currently only compatible with sensor.record = {'p'} (the default).");
        if (q.sensor_vertices > 1)
            return fail(KW_ERR_UNSUPPORTED, "StreamToDisk needs a binary (or nearest-neighbour Cartesian) sensor mask");
        P->stream_cols = (int)std::min<uint64_t>(q.stream_to_disk, (uint64_t)P->num_rec);
    }
    if (!tr && P->M > 0) {
        if (P->rec & KW_REC_P) KW_TRY(palloc(P, &P->o_series[0], P->stream_cols ? (size_t)P->M * P->stream_cols : ser));
        if (P->rec & KW_REC_P_MAX) KW_TRY(palloc(P, &P->o_max[0], P->M));
        if (P->rec & KW_REC_P_MIN) KW_TRY(palloc(P, &P->o_min[0], P->M));
        if (P->rec & KW_REC_P_RMS) KW_TRY(palloc(P, &P->o_sq[0], P->M));
        for (int i = 0; i < P->D; ++i) {
            if (P->rec & KW_REC_U) KW_TRY(palloc(P, &P->o_series[1 + i], ser));
            if (P->rec & KW_REC_U_MAX) KW_TRY(palloc(P, &P->o_max[1 + i], P->M));
            if (P->rec & KW_REC_U_MIN) KW_TRY(palloc(P, &P->o_min[1 + i], P->M));
            if (P->rec & KW_REC_U_RMS) KW_TRY(palloc(P, &P->o_sq[1 + i], P->M));
        }
    }
    if ((P->rec & KW_REC_U_NON_STAGGERED) && !tr && P->M > 0) {
        for (int i = 0; i < P->D; ++i) KW_TRY(palloc(P, &P->o_uns[i], ser));
        KW_TRY(palloc(P, &P->ush, N));
    }
    if (!tr) {
        if (P->rec & KW_REC_P_MAX_ALL) KW_TRY(palloc(P, &P->o_amax[0], P->in_count));
        if (P->rec & KW_REC_P_MIN_ALL) KW_TRY(palloc(P, &P->o_amin[0], P->in_count));
        for (int i = 0; i < P->D; ++i) {
            if (P->rec & KW_REC_U_MAX_ALL) KW_TRY(palloc(P, &P->o_amax[1 + i], P->in_count));
            if (P->rec & KW_REC_U_MIN_ALL) KW_TRY(palloc(P, &P->o_amin[1 + i], P->in_count));
        }
    }
    KW_TRY(palloc(P, &P->o_tmp, std::max<size_t>(std::max<size_t>(P->in_count, P->M), 1)));
    KW_CUDA(cudaStreamSynchronize(P->stream));
    KW_TRY(autotune_tiles(P));
    KW_TRY(zero_state(P));
    return KW_OK;
}

kw_status copy_dev(kw_plan *P, float *dst, const float *src, size_t n) {
    if (!dst || !src || n == 0) return KW_OK;
    KW_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyDeviceToHost, P->stream));
    return KW_OK;
}

kw_status crop_out(kw_plan *P, float *dst, const float *field) {
    if (!dst) return KW_OK;
    k_crop<<<std::min<long long>((P->in_count + 255) / 256, 148 * 16), 256, 0, P->stream>>>(
        field, P->o_tmp, P->g, P->in_lo[0], P->in_lo[1], P->in_lo[2], P->in_n[0], P->in_n[1], P->in_n[2]);
    KW_TRY(launched(P));
    KW_TRY(copy_dev(P, dst, P->o_tmp, P->in_count));
    KW_CUDA(cudaStreamSynchronize(P->stream));
    return KW_OK;
}

kw_status rms_out(kw_plan *P, float *dst, const float *sq) {
    if (!dst || !sq) return KW_OK;
    const int done = std::max(0, std::min(P->t - 1, P->Nt) - P->record_start + 1);
    KW_CUDA(cudaMemcpyAsync(P->o_tmp, sq, (size_t)P->M * sizeof(float), cudaMemcpyDeviceToDevice, P->stream));
    k_rms_finish<<<(P->M + 255) / 256, 256, 0, P->stream>>>(P->o_tmp, P->M, done > 0 ? 1.f / done : 0.f);
    KW_TRY(launched(P));
    KW_TRY(copy_dev(P, dst, P->o_tmp, P->M));
    KW_CUDA(cudaStreamSynchronize(P->stream));
    return KW_OK;
}

// A steady-state step always launches the same kernels with the same
// arguments, except for: which of the double buffers is current, whether a
// general (filtered) source is active, whether sensors record, and whether
// the next step's gradient is needed.  Each combination is captured once as a
// CUDA graph (on its second occurrence; the first runs directly) and replayed.
// structure of step t as the graph cache sees it: buffer parity, general
// source activity, recording, next-step gradient
uint32_t step_key(const kw_plan *P, int t, bool parity_first) {
    uint32_t key = 0;
    key |= parity_first ? 1u : 0u;
    key |= (P->u[0] == P->u_first) ? 2u : 0u;
    bool usrc = false;
    for (int c = 0; c < P->D; ++c) usrc = usrc || (P->usrc.dense_general && P->usrc.sig[c] && t <= P->usrc.T[c]);
    key |= usrc ? 4u : 0u;
    key |= (P->psrc.dense_general && t <= P->psrc.T[0]) ? 8u : 0u;
    key |= (!P->no_record && !P->time_rev && t >= P->record_start) ? 16u : 0u;
    key |= (t < P->index_end) ? 32u : 0u;
    return key;
}

kw_status run_step_graphed(kw_plan *P) {
    const int t = P->t;
    if (!P->use_graphs || P->timing_mask || (t == 1 && P->p0)) return run_step(P);
    const uint32_t key = step_key(P, t, P->rho[0] == P->rho_first);
    kw_plan::GraphEntry &e = P->graphs[key];
    if (e.exec) {
        KW_CUDA(cudaGraphLaunch(e.exec, P->stream));
        for (int i = 0; i < 3; ++i) {
            std::swap(P->u[i], P->u_b[i]);
            std::swap(P->rho[i], P->rho_b[i]);
        }
        P->launches += e.launches;
        P->t += 1;
        return KW_OK;
    }
    if (e.seen == 0) {
        e.seen = 1;
        return run_step(P);
    }
    const uint64_t l0 = P->launches;
    KW_CUDA(cudaStreamBeginCapture(P->stream, cudaStreamCaptureModeThreadLocal));
    const kw_status st = run_step(P);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(P->stream, &graph);
    if (st != KW_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (ce != cudaSuccess) return fail(KW_ERR_CUDA, "step capture failed: %s", cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&e.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return fail(KW_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ie));
    e.launches = P->launches - l0;
    KW_CUDA(cudaGraphLaunch(e.exec, P->stream));   // the captured step has not run yet
    return KW_OK;
}

// Small grids: kBlockSteps consecutive steps of one structure (an even
// number, so the double buffers end where they started) captured as one
// graph, which removes the gaps between per-step graph launches.  Used when a
// step moves fewer than kBlockCells cells; larger grids gain nothing from it.
constexpr int kBlockSteps = 8;
constexpr long long kBlockCells = 1LL << 20;

// kBlockSteps if steps t .. t + kBlockSteps - 1 can run as one block graph
int block_steps(const kw_plan *P, uint64_t remaining) {
    if (!P->use_graphs || !P->block_graphs || P->timing_mask || P->ck_on || P->g.N > kBlockCells || remaining < (uint64_t)kBlockSteps)
        return 0;
    const int t = P->t, G = kBlockSteps;
    if ((t == 1 && P->p0) || t + G - 1 >= P->index_end) return 0;
    // every step of the block has the structure of the first (parity aside)
    const uint32_t k0 = step_key(P, t, true) & ~1u;
    for (int s = 1; s < G; ++s)
        if ((step_key(P, t + s, true) & ~1u) != k0) return 0;
    return G;
}

kw_status run_block_graphed(kw_plan *P, int G) {
    const uint32_t key = step_key(P, P->t, P->rho[0] == P->rho_first) | ((uint32_t)G << 8);
    kw_plan::GraphEntry &e = P->graphs[key];
    if (e.exec) {
        KW_CUDA(cudaGraphLaunch(e.exec, P->stream));   // G even: the buffers end where they started
        P->launches += e.launches;
        P->t += G;
        return KW_OK;
    }
    if (e.seen == 0) {
        e.seen = 1;
        for (int s = 0; s < G; ++s) KW_TRY(run_step_graphed(P));
        return KW_OK;
    }
    const uint64_t l0 = P->launches;
    KW_CUDA(cudaStreamBeginCapture(P->stream, cudaStreamCaptureModeThreadLocal));
    kw_status st = KW_OK;
    for (int s = 0; s < G && st == KW_OK; ++s) st = run_step(P);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(P->stream, &graph);
    if (st != KW_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (ce != cudaSuccess) return fail(KW_ERR_CUDA, "step block capture failed: %s", cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&e.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return fail(KW_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ie));
    e.launches = P->launches - l0;
    KW_CUDA(cudaGraphLaunch(e.exec, P->stream));   // the captured steps have not run yet
    return KW_OK;
}

kw_status run_steps(kw_plan *P, uint64_t n) {
    if (!P->started) KW_TRY(start(P));
    for (uint64_t k = 0; k < n && P->t <= P->index_end; ++k) {
        if (const int G = block_steps(P, n - k)) {
            KW_TRY(run_block_graphed(P, G));
            k += G - 1;
            continue;
        }
        KW_TRY(run_step_graphed(P));
        if (P->ck_on) {
            // kept adjoint checkpoints: the state after step done = j K
            const int done = P->t - 1;
            if (done % P->ck_K == 0 && done / P->ck_K == P->ck_saved + 1 && P->ck_saved + 1 < P->ck_nseg) {
                const size_t snap = (size_t)(2 * P->D + 1) * (size_t)P->g.N;
                KW_TRY(save_state(P, P->ck_buf + (size_t)P->ck_saved * snap));
                P->ck_saved += 1;
            }
            P->ck_valid = P->t > P->Nt && P->ck_saved + 1 == P->ck_nseg;
        }
    }
    if (P->time_rev && P->t > P->index_end) {
        k_tr_final<<<(P->M + 255) / 256, 256, 0, P->stream>>>(P->sidx, P->M, P->tr_data, P->p);
        KW_TRY(launched(P));
    }
    return KW_OK;
}

kw_status use_device(const kw_plan *P) {
    KW_CUDA(cudaSetDevice(P->device));
    return KW_OK;
}

// ---- streamed series outputs ------------------------------------------------
// kw_run copies the recorded time series to the caller's host buffers while
// the loop runs: after every chunk of recorded steps a copy stream moves the
// chunk's columns into one half of a pinned host ring, and the host thread
// moves the previous chunk from the ring into the caller's buffers while the
// GPU computes the next one.  Pinned rings are kept in a process-wide pool,
// since pinning host memory costs about as much as the copy it saves.
constexpr size_t kStreamChunkBytes = (size_t)16 << 20;     // per ring half
constexpr size_t kStreamMinBytes = (size_t)64 << 20;       // smaller series are copied after the loop

std::mutex g_pinned_mutex;
std::vector<std::pair<void *, size_t>> g_pinned_free;

kw_status pinned_get(size_t bytes, void **p, size_t *got) {
    {
        std::lock_guard<std::mutex> lock(g_pinned_mutex);
        for (size_t k = 0; k < g_pinned_free.size(); ++k)
            if (g_pinned_free[k].second >= bytes) {
                *p = g_pinned_free[k].first;
                *got = g_pinned_free[k].second;
                g_pinned_free.erase(g_pinned_free.begin() + k);
                return KW_OK;
            }
    }
    void *q = nullptr;
    cudaError_t e = cudaHostAlloc(&q, bytes, cudaHostAllocPortable);
    if (e != cudaSuccess) return fail(KW_ERR_NOMEM, "pinned host allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    *p = q;
    *got = bytes;
    return KW_OK;
}
void pinned_put(void *p, size_t bytes) {
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    g_pinned_free.push_back({p, bytes});
}

struct SeriesOut {
    float *dst;          // caller's buffer, M x num_rec, column-major
    const float *src;    // device series
};

kw_status run_streamed(kw_plan *P, const std::vector<SeriesOut> &ser) {
    const size_t M = (size_t)P->M, S = ser.size();
    const int C = (int)std::max<size_t>(1, kStreamChunkBytes / (S * M * sizeof(float)));
    const size_t half = kStreamChunkBytes / sizeof(float);   // floats per ring half (holds C steps)
    if (!P->copy_stream) KW_CUDA(cudaStreamCreateWithFlags(&P->copy_stream, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) {
        if (!P->ev_comp[k]) KW_CUDA(cudaEventCreateWithFlags(&P->ev_comp[k], cudaEventDisableTiming));
        if (!P->ev_copy[k]) KW_CUDA(cudaEventCreateWithFlags(&P->ev_copy[k], cudaEventDisableTiming));
    }
    void *ring_v = nullptr;
    size_t ring_bytes = 0;
    KW_TRY(pinned_get(2 * kStreamChunkBytes, &ring_v, &ring_bytes));
    float *ring = (float *)ring_v;
    // drain chunk [c0, c1) from ring half `slot` into the caller's buffers
    auto drain = [&](int slot, int c0, int c1) -> kw_status {
        KW_CUDA(cudaEventSynchronize(P->ev_copy[slot]));
        const float *h = ring + (size_t)slot * half;
        const size_t n = M * (size_t)(c1 - c0);
        for (size_t s = 0; s < S; ++s) std::memcpy(ser[s].dst + M * (size_t)c0, h + s * M * C, n * sizeof(float));
        return KW_OK;
    };
    kw_status st = KW_OK;
    int prev_slot = -1, prev_c0 = 0, prev_c1 = 0, k = 0;
    for (int c0 = 0; c0 < P->num_rec && st == KW_OK; c0 += C, ++k) {
        const int c1 = std::min(P->num_rec, c0 + C);
        const int slot = k & 1;
        // column c is recorded at step record_start + c
        const long long target = (long long)P->record_start + c1;   // next step after the chunk
        if (target > P->t) st = run_steps(P, (uint64_t)(target - P->t));
        if (st != KW_OK) break;
        cudaError_t e = cudaEventRecord(P->ev_comp[slot], P->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(P->copy_stream, P->ev_comp[slot], 0);
        float *h = ring + (size_t)slot * half;
        for (size_t s = 0; s < S && e == cudaSuccess; ++s)
            e = cudaMemcpyAsync(h + s * M * C, ser[s].src + M * (size_t)c0, M * (size_t)(c1 - c0) * sizeof(float),
                                cudaMemcpyDeviceToHost, P->copy_stream);
        if (e == cudaSuccess) e = cudaEventRecord(P->ev_copy[slot], P->copy_stream);
        if (e != cudaSuccess) {
            st = fail(KW_ERR_CUDA, "streamed output copy failed: %s", cudaGetErrorString(e));
            break;
        }
        // the previous chunk's half is drained while the GPU runs this chunk
        if (prev_slot >= 0) st = drain(prev_slot, prev_c0, prev_c1);
        prev_slot = slot;
        prev_c0 = c0;
        prev_c1 = c1;
    }
    if (st == KW_OK && prev_slot >= 0) st = drain(prev_slot, prev_c0, prev_c1);
    if (st == KW_OK && P->t <= P->index_end) st = run_steps(P, (uint64_t)P->index_end);
    // no copy may still target the ring when it goes back to the pool
    cudaStreamSynchronize(P->copy_stream);
    pinned_put(ring_v, ring_bytes);
    return st;
}

// The device error word: bit 1, a TMA-staged copy of stage R did not land
// within its poll limit (KW_ERR_TIMEOUT); bit 2, a TMA destination was not
// 128-byte aligned and the block skipped its work (KW_ERR_CUDA).  The word is
// cleared for the next call.
kw_status check_dev_err(kw_plan *P) {
    if (!P->d_err) return KW_OK;
    int e = 0;
    KW_CUDA(cudaMemcpyAsync(&e, P->d_err, sizeof(int), cudaMemcpyDeviceToHost, P->stream));
    KW_CUDA(cudaStreamSynchronize(P->stream));
    if (e == 0) return KW_OK;
    cudaMemsetAsync(P->d_err, 0, sizeof(int), P->stream);
    if (e & 4) return fail(KW_ERR_CUDA, "internal: a TMA staging buffer was misaligned (device error word %d)", e);
    return fail(KW_ERR_TIMEOUT, "a staged tensor copy did not complete within its wait limit (device error word %d)", e);
}

// StreamToDisk (kspaceFirstOrder3D.m:1101-1146, 1235-1295): the loop runs in
// chunks of stream_cols recorded steps; after each chunk the ring of p
// columns is copied to pinned host memory and appended to the file (FP32,
// column-major, as MATLAB's fwrite) -- or copied into out->p when no file is
// named -- while the next chunk computes.  After the loop the file is read
// back into out->p and deleted, and the other outputs are copied.
kw_status run_to_disk(kw_plan *P, kw_outputs *o) {
    const size_t M = (size_t)P->M, C = (size_t)P->stream_cols;
    const char *path = P->prob.stream_to_disk_file;
    if (P->t != 1 || P->started) KW_TRY(zero_state(P));
    if (!P->copy_stream) KW_CUDA(cudaStreamCreateWithFlags(&P->copy_stream, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) {
        if (!P->ev_comp[k]) KW_CUDA(cudaEventCreateWithFlags(&P->ev_comp[k], cudaEventDisableTiming));
        if (!P->ev_copy[k]) KW_CUDA(cudaEventCreateWithFlags(&P->ev_copy[k], cudaEventDisableTiming));
    }
    std::FILE *fp = nullptr;
    if (path) {
        fp = std::fopen(path, "w+b");
        if (!fp) return fail(KW_ERR_INVALID, "Error in writing file using 'StreamToDisk': cannot open %s", path);
    }
    float *host = nullptr;
    if (cudaMallocHost((void **)&host, 2 * M * C * sizeof(float)) != cudaSuccess) {
        if (fp) {
            std::fclose(fp);
            std::remove(path);
        }
        return fail(KW_ERR_NOMEM, "StreamToDisk: pinned host buffer of %zu bytes failed", 2 * M * C * sizeof(float));
    }
    kw_status st = KW_OK;
    // write chunk [c0, c1) held in ring half `slot`
    auto drain = [&](int slot, int c0, int c1) -> kw_status {
        KW_CUDA(cudaEventSynchronize(P->ev_copy[slot]));
        const float *h = host + (size_t)slot * M * C;
        const size_t n = M * (size_t)(c1 - c0);
        if (fp) {
            if (std::fwrite(h, sizeof(float), n, fp) != n)
                return fail(KW_ERR_INVALID, "Error in writing file using 'StreamToDisk'");
        } else if (o->p) {
            std::memcpy(o->p + M * (size_t)c0, h, n * sizeof(float));
        }
        return KW_OK;
    };
    int prev = -1, pc0 = 0, pc1 = 0, k = 0;
    for (int c0 = 0; c0 < P->num_rec && st == KW_OK; c0 += (int)C, ++k) {
        const int c1 = std::min(P->num_rec, c0 + (int)C);
        const int slot = k & 1;
        const long long target = (long long)P->record_start + c1;   // next step after the chunk
        if (target > P->t) st = run_steps(P, (uint64_t)(target - P->t));
        if (st != KW_OK) break;
        // columns c0 .. c1-1 sit at ring columns 0 .. c1-c0-1 (c0 is a multiple of C)
        cudaError_t e = cudaEventRecord(P->ev_comp[slot], P->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(P->copy_stream, P->ev_comp[slot], 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(host + (size_t)slot * M * C, P->o_series[0], M * (size_t)(c1 - c0) * sizeof(float),
                                cudaMemcpyDeviceToHost, P->copy_stream);
        if (e == cudaSuccess) e = cudaEventRecord(P->ev_copy[slot], P->copy_stream);
        // the compute stream may overwrite this half's device columns only
        // after the copy: the next chunk waits for it
        if (e == cudaSuccess) e = cudaStreamWaitEvent(P->stream, P->ev_copy[slot], 0);
        if (e != cudaSuccess) {
            st = fail(KW_ERR_CUDA, "streamed output copy failed: %s", cudaGetErrorString(e));
            break;
        }
        if (prev >= 0) st = drain(prev, pc0, pc1);
        prev = slot;
        pc0 = c0;
        pc1 = c1;
    }
    if (st == KW_OK && prev >= 0) st = drain(prev, pc0, pc1);
    if (st == KW_OK && P->t <= P->index_end) st = run_steps(P, (uint64_t)P->index_end);
    cudaStreamSynchronize(P->copy_stream);
    cudaStreamSynchronize(P->stream);
    cudaFreeHost(host);
    if (fp) {
        // reload the complete streamed series and remove the file
        if (st == KW_OK && o->p) {
            std::fflush(fp);
            std::rewind(fp);
            const size_t n = M * (size_t)P->num_rec;
            if (std::fread(o->p, sizeof(float), n, fp) != n)
                st = fail(KW_ERR_INVALID, "StreamToDisk: short read of %s", path);
        }
        std::fclose(fp);
        std::remove(path);
    }
    KW_TRY(st);
    kw_outputs rest = *o;
    rest.p = nullptr;
    return kw_copy_outputs(P, &rest);
}

}  // namespace

// --------------------------------------------------------------------------
// Allocation-free spectral gradient (kw_gradient_noalloc)
//
// Some callers cannot let this library call cudaMalloc: a MATLAB MEX function
// working on gpuArray data whose device memory belongs to MATLAB's pool, a
// PyTorch extension that must draw every byte from the framework's caching
// allocator, or a long-running service that forbids device allocation after
// start-up because an allocation can block, fragment the heap or fail late.
// kw_gradient_noalloc serves them: the caller passes device input and output
// buffers, and the only other device memory it touches is the file-scope
// array below.  That array is part of the module image, so every GPU that
// loads this library holds it until the process exits.
// --------------------------------------------------------------------------
#define KW_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[KW_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
void *g_noalloc_base[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mutex;

// Device address of the scratch array on the current device (resolved once
// per device; host code may not use the symbol name as a device address).
kw_status noalloc_base(int dev, void **base) {
    if (dev < 0 || dev >= kMaxDevices) return fail(KW_ERR_UNSUPPORTED, "device ordinal %d above %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_base[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(KW_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed: %s", cudaGetErrorString(e));
        g_noalloc_base[dev] = p;
    }
    *base = g_noalloc_base[dev];
    return KW_OK;
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

// --------------------------------------------------------------------------
// C ABI
// --------------------------------------------------------------------------
extern "C" {

const char *kw_last_error(void) { return g_err.c_str(); }

int kw_abi_version(void) { return KW_ABI_VERSION; }

kw_status kw_plan_create(const kw_problem *problem, kw_plan **plan) {
    if (!plan) return fail(KW_ERR_INVALID, "plan pointer is NULL");
    *plan = nullptr;
    kw_plan *P = new (std::nothrow) kw_plan();
    if (!P) return fail(KW_ERR_NOMEM, "host allocation failed");
    kw_status s = create(problem, P);
    if (s != KW_OK) {
        std::string keep = g_err;
        kw_plan_destroy(P);
        g_err = keep;
        return s;
    }
    *plan = P;
    g_err.clear();
    return KW_OK;
}

kw_status kw_plan_outputs(const kw_plan *P, kw_output_desc *d) {
    if (!P || !d) return fail(KW_ERR_INVALID, "NULL argument");
    d->sensor_num = (uint64_t)P->M;
    d->num_time_points = (uint64_t)P->num_rec;
    const int D = P->D;
    if (D == 3) {
        for (int a = 0; a < 3; ++a) { d->inside_shape[a] = P->in_n[a]; d->grid_shape[a] = P->N[a]; }
    } else {
        d->inside_shape[0] = P->in_n[0]; d->inside_shape[1] = P->in_n[2]; d->inside_shape[2] = 1;
        d->grid_shape[0] = P->N[0]; d->grid_shape[1] = P->N[2]; d->grid_shape[2] = 1;
    }
    return KW_OK;
}

kw_status kw_reset(kw_plan *P) {
    if (!P) return fail(KW_ERR_INVALID, "plan is NULL");
    KW_TRY(use_device(P));
    return zero_state(P);
}

kw_status kw_step(kw_plan *P, uint64_t n) {
    if (!P) return fail(KW_ERR_INVALID, "plan is NULL");
    KW_TRY(use_device(P));
    KW_TRY(run_steps(P, n));
    KW_CUDA(cudaStreamSynchronize(P->stream));
    return check_dev_err(P);
}

kw_status kw_run_device(kw_plan *P) {
    if (!P) return fail(KW_ERR_INVALID, "plan is NULL");
    KW_TRY(use_device(P));
    if (P->t != 1 || P->started) KW_TRY(zero_state(P));
    KW_TRY(run_steps(P, (uint64_t)P->index_end));
    KW_CUDA(cudaStreamSynchronize(P->stream));
    return check_dev_err(P);
}

kw_status kw_copy_outputs(kw_plan *P, kw_outputs *o) {
    if (!P || !o) return fail(KW_ERR_INVALID, "NULL argument");
    KW_TRY(use_device(P));
    if (P->stream_cols && o->p)
        return fail(KW_ERR_UNSUPPORTED, "the p series of a StreamToDisk plan is written out by kw_run only");
    const size_t ser = (size_t)P->M * P->num_rec;
    KW_TRY(copy_dev(P, o->p, P->o_series[0], ser));
    KW_TRY(copy_dev(P, o->p_max, P->o_max[0], P->M));
    KW_TRY(copy_dev(P, o->p_min, P->o_min[0], P->M));
    KW_TRY(rms_out(P, o->p_rms, P->o_sq[0]));
    KW_TRY(copy_dev(P, o->p_max_all, P->o_amax[0], P->in_count));
    KW_TRY(copy_dev(P, o->p_min_all, P->o_amin[0], P->in_count));
    if ((P->rec & KW_REC_P_FINAL) || P->time_rev) KW_TRY(crop_out(P, o->p_final, P->p));
    for (int i = 0; i < P->D; ++i) {
        KW_TRY(copy_dev(P, o->u[i], P->o_series[1 + i], ser));
        KW_TRY(copy_dev(P, o->u_max[i], P->o_max[1 + i], P->M));
        KW_TRY(copy_dev(P, o->u_min[i], P->o_min[1 + i], P->M));
        KW_TRY(rms_out(P, o->u_rms[i], P->o_sq[1 + i]));
        KW_TRY(copy_dev(P, o->u_max_all[i], P->o_amax[1 + i], P->in_count));
        KW_TRY(copy_dev(P, o->u_min_all[i], P->o_amin[1 + i], P->in_count));
        if (P->rec & KW_REC_U_FINAL) KW_TRY(crop_out(P, o->u_final[i], P->u[i]));
        KW_TRY(copy_dev(P, o->u_non_staggered[i], P->o_uns[i], ser));
    }
    KW_CUDA(cudaStreamSynchronize(P->stream));
    return KW_OK;
}

kw_status kw_run(kw_plan *P, kw_outputs *o) {
    if (!P || !o) return fail(KW_ERR_INVALID, "NULL argument");
    KW_TRY(use_device(P));
    if (P->stream_cols) {
        KW_TRY(run_to_disk(P, o));
        return check_dev_err(P);
    }
    // time series large enough to be worth streaming to the host during the loop
    std::vector<SeriesOut> ser;
    if (!P->time_rev && P->M > 0) {
        if (o->p && P->o_series[0]) ser.push_back({o->p, P->o_series[0]});
        for (int i = 0; i < P->D; ++i) {
            if (o->u[i] && P->o_series[1 + i]) ser.push_back({o->u[i], P->o_series[1 + i]});
            if (o->u_non_staggered[i] && P->o_uns[i]) ser.push_back({o->u_non_staggered[i], P->o_uns[i]});
        }
    }
    const size_t col_bytes = ser.size() * (size_t)P->M * sizeof(float);   // one recorded step
    const size_t ser_bytes = col_bytes * P->num_rec;
    // stream when the series are large and one recorded step fits a chunk
    // (the ring is two chunks); otherwise, or when no pinned ring can be had,
    // copy after the loop
    void *ring = nullptr;
    size_t ring_bytes = 0;
    bool stream = ser_bytes >= kStreamMinBytes && col_bytes <= kStreamChunkBytes;
    if (stream && pinned_get(2 * kStreamChunkBytes, &ring, &ring_bytes) != KW_OK) {
        g_err.clear();   // not an error: the copy after the loop needs no pinned memory
        stream = false;
    }
    if (!stream) {
        KW_TRY(kw_run_device(P));
        return kw_copy_outputs(P, o);
    }
    pinned_put(ring, ring_bytes);   // run_streamed takes it back from the pool
    if (P->t != 1 || P->started) KW_TRY(zero_state(P));
    KW_TRY(run_streamed(P, ser));
    KW_CUDA(cudaStreamSynchronize(P->stream));
    KW_TRY(check_dev_err(P));
    // the remaining (non-series) outputs after the loop
    kw_outputs rest = *o;
    rest.p = nullptr;
    for (int i = 0; i < 3; ++i) {
        rest.u[i] = nullptr;
        rest.u_non_staggered[i] = nullptr;
    }
    return kw_copy_outputs(P, &rest);
}

kw_status kw_plan_destroy(kw_plan *P) {
    if (!P) return KW_OK;
    cudaSetDevice(P->device);
    if (P->stream) cudaStreamSynchronize(P->stream);
    for (auto &kv : P->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    for (auto &r : P->timers) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    if (P->copy_stream) {
        cudaStreamSynchronize(P->copy_stream);
        cudaStreamDestroy(P->copy_stream);
    }
    for (int k = 0; k < 2; ++k) {
        if (P->ev_comp[k]) cudaEventDestroy(P->ev_comp[k]);
        if (P->ev_copy[k]) cudaEventDestroy(P->ev_copy[k]);
    }
    for (void *a : P->allocs) cudaFreeAsync(a, P->stream);
    if (P->stream) {
        cudaStreamSynchronize(P->stream);
        cudaStreamDestroy(P->stream);
    }
    delete P;
    return KW_OK;
}

kw_status kw_set_timing(kw_plan *P, uint32_t mask) {
    if (!P) return fail(KW_ERR_INVALID, "plan is NULL");
    KW_TRY(timer_flush(P));
    P->timing_mask = mask;
    for (int c = 0; c < KW_KCLASS_COUNT; ++c) { P->t_ms[c] = 0; P->t_count[c] = 0; }
    return KW_OK;
}

kw_status kw_get_timing(const kw_plan *Pc, int cls, double *ms, uint64_t *n) {
    kw_plan *P = const_cast<kw_plan *>(Pc);
    if (!P || cls < 0 || cls >= KW_KCLASS_COUNT) return fail(KW_ERR_INVALID, "bad argument");
    KW_TRY(timer_flush(P));
    if (ms) *ms = P->t_ms[cls];
    if (n) *n = P->t_count[cls];
    return KW_OK;
}

kw_status kw_run_timed(kw_plan *P, uint32_t n, double *device_ms) {
    if (!P || !device_ms) return fail(KW_ERR_INVALID, "NULL argument");
    KW_TRY(use_device(P));
    cudaEvent_t a, b;
    KW_CUDA(cudaEventCreate(&a));
    KW_CUDA(cudaEventCreate(&b));
    KW_CUDA(cudaStreamSynchronize(P->stream));
    KW_CUDA(cudaEventRecord(a, P->stream));
    kw_status st = KW_OK;
    for (uint32_t k = 0; k < n && st == KW_OK; ++k) {
        st = zero_state(P);
        if (st == KW_OK) st = run_steps(P, (uint64_t)P->index_end);
    }
    cudaEventRecord(b, P->stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    KW_TRY(st);
    KW_CUDA(cudaGetLastError());
    *device_ms = ms;
    return check_dev_err(P);
}

kw_status kw_launch_count(const kw_plan *P, uint64_t *launches) {
    if (!P || !launches) return fail(KW_ERR_INVALID, "NULL argument");
    *launches = P->launches;
    return KW_OK;
}

kw_status kw_gradient_noalloc(int32_t dim, const uint64_t shape[3], const double spacing[3], int32_t axis,
                              int32_t shift_sign, double c_ref, double dt, int32_t use_kspace,
                              const float *field, float *out, void *stream) {
    if (dim != 2 && dim != 3) return fail(KW_ERR_INVALID, "dim must be 2 or 3");
    if (!shape || !spacing || !field || !out) return fail(KW_ERR_INVALID, "NULL argument");
    if (axis < 0 || axis >= dim) return fail(KW_ERR_INVALID, "axis must be 0..dim-1");
    if (shift_sign != 1 && shift_sign != -1 && shift_sign != 0) return fail(KW_ERR_INVALID, "shift_sign must be +1, -1 or 0");
    int n[3] = {1, 1, 1};
    double d[3] = {1, 1, 1};
    int phys_of_int[3] = {0, -1, 1};
    if (dim == 3) {
        for (int a = 0; a < 3; ++a) { n[a] = (int)shape[a]; d[a] = spacing[a]; phys_of_int[a] = a; }
    } else {
        n[0] = (int)shape[0]; d[0] = spacing[0];
        n[2] = (int)shape[1]; d[2] = spacing[1];
    }
    for (int a = 0; a < dim; ++a) {
        if (shape[a] < 2 || shape[a] > 4096) return fail(KW_ERR_UNSUPPORTED, "grid size outside 2..4096");
        if (!(spacing[a] > 0)) return fail(KW_ERR_INVALID, "grid spacing must be positive");
    }
    if (n[2] > kCap / 2) return fail(KW_ERR_UNSUPPORTED, "axis length %d above %d", n[2], kCap / 2);
    const int iaxis = dim == 3 ? axis : (axis == 0 ? 0 : 2);

    kw_plan P;   // launch context only: no plan memory is allocated
    P.D = dim;
    for (int a = 0; a < 3; ++a) { P.N[a] = n[a]; P.d[a] = d[a]; }
    Geom &g = P.g;
    g.N0 = n[0]; g.N1 = n[1]; g.N2 = n[2];
    g.N2h = g.N2 / 2 + 1;
    g.N = (long long)g.N0 * g.N1 * g.N2;
    g.Nh = (long long)g.N0 * g.N1 * g.N2h;
    g.vec2 = (g.N0 % 2 == 0) ? 1 : 0;

    // scratch layout: spectrum, then per-axis twiddles, wavenumbers^2 and the
    // derivative operator of the requested axis
    size_t off = 0;
    const size_t o_spec = off; off = align256(off + (size_t)g.Nh * sizeof(float2));
    size_t o_tw[3], o_k2[3];
    for (int a = 0; a < 3; ++a) { o_tw[a] = off; off = align256(off + (size_t)n[a] * sizeof(float2)); }
    for (int a = 0; a < 3; ++a) { o_k2[a] = off; off = align256(off + (size_t)n[a] * sizeof(float)); }
    const size_t o_dd = off; off = align256(off + (size_t)n[iaxis] * sizeof(float2));
    if (off > KW_NOALLOC_SCRATCH_BYTES)
        return fail(KW_ERR_UNSUPPORTED, "grid needs %zu bytes of scratch; kw_gradient_noalloc is limited to %zu bytes "
                    "(the half spectrum of about 8.3 million cells)", off, (size_t)KW_NOALLOC_SCRATCH_BYTES);

    // the call copies its tables from host memory and synchronizes the
    // stream, neither of which a stream capture can record
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    KW_CUDA(cudaStreamIsCapturing((cudaStream_t)stream, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(KW_ERR_UNSUPPORTED, "kw_gradient_noalloc cannot run while its stream is being captured");

    int dev = 0;
    KW_CUDA(cudaGetDevice(&dev));
    void *basev = nullptr;
    KW_TRY(noalloc_base(dev, &basev));
    unsigned char *base = (unsigned char *)basev;
    P.stream = (cudaStream_t)stream;

    for (int a = 0; a < 3; ++a) {
        std::vector<int> rad;
        if (!factorize(n[a], rad)) return fail(KW_ERR_UNSUPPORTED, "grid size %d needs more than %d transform stages", n[a], kMaxStages);
        AxisFFT &f = P.fft[a];
        f.n = n[a];
        f.nstages = (int)rad.size();
        for (size_t s2 = 0; s2 < rad.size(); ++s2) f.radix[s2] = rad[s2];
        std::vector<float2> tw(n[a]);
        for (int m = 0; m < n[a]; ++m) {
            const double ang = -2.0 * M_PI * (double)m / n[a];
            tw[m] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        }
        std::vector<float> k2(n[a], 0.f);
        if (phys_of_int[a] >= 0) {
            const std::vector<double> k = kvec_fft(n[a], d[a]);
            for (int i = 0; i < n[a]; ++i) k2[i] = (float)(k[i] * k[i]);
        }
        KW_CUDA(cudaMemcpyAsync(base + o_tw[a], tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, P.stream));
        KW_CUDA(cudaMemcpyAsync(base + o_k2[a], k2.data(), k2.size() * sizeof(float), cudaMemcpyHostToDevice, P.stream));
        // both kernel families read the twiddles: the runtime-radix ones
        // through fft[a], the compile-time ones through tw[a]
        P.tw[a] = (float2 *)(base + o_tw[a]);
        f.tw = P.tw[a];
        P.op.k2[a] = (const float *)(base + o_k2[a]);
        P.op.dd_pos[a] = P.op.dd_neg[a] = (const float2 *)(base + o_dd);
    }
    {
        // i k exp(+-i k d/2) (kspaceFirstOrder3D.m:629-636), Hermitian part
        const int na = n[iaxis];
        const double da = d[iaxis];
        const std::vector<double> k = kvec_fft(na, da);
        std::vector<std::complex<double>> c(na);
        for (int i = 0; i < na; ++i)
            c[i] = std::complex<double>(0.0, k[i]) * std::exp(std::complex<double>(0.0, shift_sign * k[i] * da / 2));
        std::vector<float2> dd(na);
        for (int i = 0; i < na; ++i) {
            const std::complex<double> h = 0.5 * (c[i] + std::conj(c[(na - i) % na]));
            dd[i] = make_float2((float)h.real(), (float)h.imag());
        }
        KW_CUDA(cudaMemcpyAsync(base + o_dd, dd.data(), dd.size() * sizeof(float2), cudaMemcpyHostToDevice, P.stream));
    }
    P.op.kappa_a = (float)(c_ref * dt / 2.0);
    P.op.use_kspace = use_kspace ? 1 : 0;
    P.op.scale = (float)(1.0 / (double)g.N);
    plan_tiles(&P);
    float2 *spec = (float2 *)(base + o_spec);
    // the spectrum is fully written by the forward z-transform, so nothing
    // left in the scratch by an earlier call is read
    KW_TRY(zr2c(&P, field, spec));
    Spec4 b{};
    b.p[0] = spec;
    OpSet ops{};
    ops.n = 1;
    ops.kind[0] = OP_GRAD_POS;
    ops.axis[0] = iaxis;
    KW_TRY(ypass(&P, false, b, 1));
    KW_TRY(xpass(&P, b, ops, 1, 1));
    KW_TRY(ypass(&P, true, b, 1));
    KW_TRY(zc2r(&P, spec, out));
    KW_CUDA(cudaStreamSynchronize(P.stream));
    return KW_OK;
}

kw_status kw_plan_tiles(const kw_plan *P, int32_t tiles[3]) {
    if (!P || !tiles) return fail(KW_ERR_INVALID, "NULL argument");
    tiles[0] = P->static_z ? P->PL_z : 0;
    tiles[1] = P->static_y ? P->TY : 0;
    tiles[2] = P->static_x ? P->NL : 0;
    return KW_OK;
}

kw_status kw_set_tiles(kw_plan *P, const int32_t tiles[3]) {
    if (!P || !tiles) return fail(KW_ERR_INVALID, "NULL argument");
    const Geom &g = P->g;
    auto ok = [](int v, int n) { return v == ks_lines(n) || v == ks_half(n) || v == ks_narrow(n); };
    if (P->static_z && !ok(tiles[0], g.N2))
        return fail(KW_ERR_INVALID, "z tile width must be %d, %d or %d", ks_lines(g.N2), ks_half(g.N2), ks_narrow(g.N2));
    if (P->static_y && !ok(tiles[1], g.N1))
        return fail(KW_ERR_INVALID, "y tile width must be %d, %d or %d", ks_lines(g.N1), ks_half(g.N1), ks_narrow(g.N1));
    if (P->static_x && tiles[2] != ks_xlines(g.N0) && tiles[2] != ks_xhalf(g.N0) && tiles[2] != ks_xnarrow(g.N0))
        return fail(KW_ERR_INVALID, "x tile width must be %d, %d or %d", ks_xlines(g.N0), ks_xhalf(g.N0), ks_xnarrow(g.N0));
    const bool z_fixed = P->time_rev || (P->psrc.present && !P->psrc.dense_fast && !P->psrc.dense_general) ||
                         (P->usrc.present && !P->usrc.dense_fast && !P->usrc.dense_general);
    if (P->static_z && z_fixed && tiles[0] != P->PL_z)
        return fail(KW_ERR_INVALID, "the z tiles of this plan are fixed by its sparse source or time-reversal lists");
    KW_TRY(use_device(P));
    KW_CUDA(cudaStreamSynchronize(P->stream));
    TileChoice c = tiles_of(P);
    if (P->static_z) c.PLu = c.PLr = c.PLp = tiles[0];
    if (P->static_y) c.TY = tiles[1];
    if (P->static_x) c.NL = tiles[2];
    set_tiles(P, c);
    // graphs captured with the old tiles are stale
    for (auto &kv : P->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    P->graphs.clear();
    return KW_OK;
}

kw_status kw_plan_device_bytes(const kw_plan *P, uint64_t *bytes) {
    if (!P || !bytes) return fail(KW_ERR_INVALID, "NULL argument");
    *bytes = P->bytes;
    return KW_OK;
}

}  // extern "C"

#include "kw_server.inc"
#include "kw_adjoint.inc"
