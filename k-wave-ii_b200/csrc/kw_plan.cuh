// kw_plan.cuh -- the plan object and the launch interface shared by the
// library's translation units.
//
// kwave_b200.cu holds the host side (set-up, time loop, C ABI); kw_inst.cu is
// compiled once per compile-time axis length (and once for the runtime-radix
// kernels) and holds the kernel launchers of that length, so the transform
// kernels of each length compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <vector>

#include "kw_kernels.cuh"
#include "../../include/kwave_b200.h"

namespace kw {
// sets the calling thread's error message (kw_last_error) and returns s
kw_status fail(kw_status s, const char *fmt, ...);
}  // namespace kw

#define KW_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            return fail(e_ == cudaErrorMemoryAllocation ? KW_ERR_NOMEM : KW_ERR_CUDA,          \
                        "CUDA error %s at %s:%d (%s)", cudaGetErrorName(e_), __FILE__, __LINE__, \
                        cudaGetErrorString(e_));                                               \
        }                                                                                      \
    } while (0)

#define KW_TRY(call)                   \
    do {                               \
        kw_status s_ = (call);         \
        if (s_ != KW_OK) return s_;    \
    } while (0)

// --------------------------------------------------------------------------
// the plan
// --------------------------------------------------------------------------
using kw::AxisFFT;
using kw::Geom;
using kw::Med;
using kw::OpParams;

struct SourceDev {
    bool present = false;
    int mode = 0;
    int T[3] = {0, 0, 0};
    int nsig = 0;
    int npts = 0;
    bool dense_fast = false;      // additive, one signal: rho += s(t) F
    bool dense_general = false;   // additive, several signals: F_t each step
    float *sig[3] = {nullptr, nullptr, nullptr};
    long long *pos = nullptr;     // 0-based linear indices
    int *row = nullptr;           // 0-based signal row per point
    float *F = nullptr;           // filtered mask (fast path)
    float *Ft[3] = {nullptr, nullptr, nullptr};  // filtered source of this step (general path)
    float *scratch = nullptr;     // zero field holding the scattered source (general path)
    int *csr_off = nullptr, *csr_cell = nullptr, *csr_row = nullptr;  // sparse modes
};

struct TimerRec {
    cudaEvent_t a, b;
    int cls;
};

struct kw_plan {
    kw_problem prob;               // scalars (pointers are not retained)
    int D = 3;
    Geom g{};
    int N[3] = {1, 1, 1};          // internal shape
    double d[3] = {1, 1, 1};       // internal spacing
    int comp_axis[3] = {0, 1, 2};
    int Nt = 0, index_end = 0, record_start = 1, num_rec = 0;
    bool time_rev = false, p0 = false, absorbing = false, has_tau = false, has_eta = false;
    cudaStream_t stream = nullptr;

    AxisFFT fft[3]{};
    float2 *tw[3] = {nullptr, nullptr, nullptr};
    float2 *dd_pos[3] = {nullptr, nullptr, nullptr}, *dd_neg[3] = {nullptr, nullptr, nullptr};
    float2 *sh_neg[3] = {nullptr, nullptr, nullptr};
    float *k2[3] = {nullptr, nullptr, nullptr};
    float *pml[3] = {nullptr, nullptr, nullptr}, *pml_sg[3] = {nullptr, nullptr, nullptr};
    OpParams op{};

    // fields
    float *p = nullptr, *rho[3] = {nullptr, nullptr, nullptr}, *u[3] = {nullptr, nullptr, nullptr};
    float *rho_b[3] = {nullptr, nullptr, nullptr};   // second rho buffer (Stage R writes it, then they swap)
    float *u_b[3] = {nullptr, nullptr, nullptr};     // second velocity buffer (Stage U writes it, then they swap)
    float *srho = nullptr;                           // nonlinear mass coefficient q = 2 sum(rho) + rho0
    float2 *spec[4] = {nullptr, nullptr, nullptr, nullptr};
    float *p0_dev = nullptr;
    int *d_t = nullptr;

    // medium
    float *c0_arr = nullptr, *rho0_arr = nullptr, *rsi_arr[3] = {nullptr, nullptr, nullptr};
    float *bona_arr = nullptr;
    Med c0{}, rho0{}, rsi[3]{}, bona{};
    float *c2tau_arr = nullptr, *c2eta_arr = nullptr;
    Med c2tau{}, c2eta{};           // c0^2 * absorb_tau, c0^2 * absorb_eta

    SourceDev psrc, usrc;

    // tiles
    int PL_u = 1, PL_r = 1, PL_p = 1, PL_z = 1, TY = 1, NL = 1;
    bool static_x = false, static_y = false, static_z = false;
    int kz_chunks = 1;               // kz chunks of the y / x / y groups (L2 reuse)

    // sensors / outputs
    int M = 0;
    int K = 1;                     // grid cells per sensor point (interpolated points: K > 1)
    long long *sidx = nullptr;     // [M x K] column-major
    bool sidx_all = false;         // the mask holds every cell (sidx[m] == m): gathers read cell m directly
    float *sw = nullptr;           // [M x K] weights (K > 1)
    float *tr_data = nullptr;
    int *tr_off = nullptr, *tr_cell = nullptr, *tr_row = nullptr;
    uint32_t rec = 0;
    float *o_series[4] = {nullptr, nullptr, nullptr, nullptr};
    float *o_max[4] = {nullptr, nullptr, nullptr, nullptr}, *o_min[4] = {nullptr, nullptr, nullptr, nullptr};
    float *o_sq[4] = {nullptr, nullptr, nullptr, nullptr};
    float *o_amax[4] = {nullptr, nullptr, nullptr, nullptr}, *o_amin[4] = {nullptr, nullptr, nullptr, nullptr};
    float *o_tmp = nullptr;        // crop / rms staging
    float *o_uns[3] = {nullptr, nullptr, nullptr};   // u_non_staggered series
    float *ush = nullptr;          // one unstaggered velocity component
    int in_lo[3] = {0, 0, 0}, in_n[3] = {1, 1, 1};
    int stream_cols = 0;           // StreamToDisk: columns of the p series ring (0: whole record)

    // TMA staging of stage R: usable for this plan's shapes, tensor maps by
    // (device pointer, box width), device error word of bounded waits
    bool tma_r = false;
    std::map<std::pair<const void *, int>, CUtensorMap> tmaps;
    int *d_err = nullptr;
    // adjoint checkpoints kept by the plan's own runs (kw_keep_checkpoints):
    // the state after steps K, 2K, ..., (nseg - 1) K; valid after a complete run
    float *ck_buf = nullptr;
    int ck_K = 0, ck_nseg = 0, ck_saved = 0;
    bool ck_on = false, ck_valid = false;
    long long in_count = 1;

    int t = 1;                     // next step to run (1-based)
    bool started = false;
    bool no_record = false;        // steps re-run by the gradient do not record

    // timing
    uint32_t timing_mask = 0;
    std::vector<TimerRec> timers;
    double t_ms[KW_KCLASS_COUNT] = {0};
    uint64_t t_count[KW_KCLASS_COUNT] = {0};

    // CUDA graphs of steady-state steps, keyed by the step's structure
    struct GraphEntry {
        cudaGraphExec_t exec = nullptr;
        uint64_t launches = 0;
        int seen = 0;
    };
    std::map<uint32_t, GraphEntry> graphs;
    bool use_graphs = true;
    bool block_graphs = true;   // small grids: several steps per graph (run_steps)
    float *rho_first = nullptr, *u_first = nullptr;   // buffer identity for the key

    // streamed series outputs of kw_run: copy stream and per-slot events
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_comp[2] = {nullptr, nullptr}, ev_copy[2] = {nullptr, nullptr};

    std::vector<void *> allocs;
    size_t bytes = 0;
    uint64_t launches = 0;
    int device = 0;
};

namespace kw {

// raise the dynamic shared-memory limit of a kernel when it needs more than 48 KB
kw_status set_smem(const void *fn, size_t bytes);
// tensor maps of a stage R launch with tile width TX; *use is false when
// the plan stages with cp.async instead
kw_status stage_r_maps(kw_plan *P, const StageR &a, int TX, StageRMaps *m, bool *use);
kw_status stage_u_maps(kw_plan *P, const StageU &a, int TX, StageUMaps *m, bool *use);
kw_status stage_p_maps(kw_plan *P, const StageP &a, int TX, StagePMaps *m, bool *use);
// check the last launch and count it in the plan
kw_status launched(kw_plan *P);

// Axis lengths with compile-time kernels; every other length uses the
// runtime-radix kernels.  Tile shapes of both are shared with the planner.
#define KW_STATIC_SIZES(X) X(64) X(96) X(128) X(160) X(192) X(256) X(320) X(384) X(512)

// Kernel launchers of one axis length N (N = 0: the runtime-radix kernels).
// Defined in kw_launch.cuh and instantiated per length in kw_inst.cu.
template <int N> struct YLaunch {
    static kw_status run(kw_plan *P, bool inv, Spec4 bufs, int nf, int kz0, int nkz);
    // inverse y-pass of the 3-D gradient fan-out (ks_ypass_fan); N > 0 only
    static kw_status run_fan(kw_plan *P, Spec4 bufs, int kz0, int nkz, const float2 *ddy, const float2 *ddz);
};
template <int N> struct XLaunch {
    static kw_status run(kw_plan *P, Spec4 bufs, OpSet ops, int fanout, int nf, int kz0, int nkz);
};
template <int N> struct ZR2CLaunch {
    static kw_status run(kw_plan *P, const float *R, float2 *H);
};
template <int N> struct ZC2RLaunch {
    static kw_status run(kw_plan *P, const float2 *H, float *R);
};
template <int N> struct ULaunch {
    static kw_status run(kw_plan *P, StageU a);
};
template <int N> struct RLaunch {
    static kw_status run(kw_plan *P, StageR a);
};
template <int N> struct PLaunch {
    static kw_status run(kw_plan *P, StageP a);
};

}  // namespace kw
