/*
 * kwave_b200.h -- C ABI of the B200 k-space first-order acoustic time loop.
 *
 * This library replaces the time loop of k-Wave's kspaceFirstOrder2D /
 * kspaceFirstOrder3D (+kwave/+legacy/kspaceFirstOrder3D.m:769-1208,
 * +kwave/+legacy/kspaceFirstOrder2D.m:712-1044).  The caller runs the
 * reference's setup (input checking, p0 smoothing, Cartesian->grid sensor
 * conversion, source scaling, staggered density interpolation) and hands over
 * exactly the variable set that the reference serialises for its external
 * native solver at the SaveToDisk hand-off point
 * (+kwave/+legacy/private/kspaceFirstOrder_saveToDisk.m:46-353,
 * +kwave/+legacy/kspaceFirstOrder3D.m:669-687), as plain host pointers.
 *
 * Conventions
 *   - Arrays are MATLAB column-major (x fastest), FP32, Nx*Ny*Nz elements.
 *   - Index arrays are 1-based MATLAB linear indices (as saved by saveToDisk).
 *   - Signal matrices are column-major [rows x time] like MATLAB's source.p.
 *   - Every entry point returns kw_status; kw_last_error() gives the message
 *     of the last failure on the calling thread.  No C++ exception crosses
 *     the ABI.  The library owns all device memory of a plan.
 *   - A plan is used by one host thread at a time; plans are independent.
 */
#ifndef KWAVE_B200_H
#define KWAVE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int kw_status;
#define KW_OK              0
#define KW_ERR_INVALID     1   /* bad argument: mirrors MATLAB error(...) in inputChecking */
#define KW_ERR_CUDA        2   /* CUDA runtime failure */
#define KW_ERR_NOMEM       3   /* device allocation failed */
#define KW_ERR_UNSUPPORTED 4   /* valid reference input this build does not handle */
#define KW_ERR_TIMEOUT     5   /* a bounded wait gave up, or a served request passed its deadline */

#define KW_ABI_VERSION 3

/* sensor.record bit mask (inputChecking.m:340-400 list of record flags) */
#define KW_REC_P               (1u << 0)
#define KW_REC_P_MAX           (1u << 1)
#define KW_REC_P_MIN           (1u << 2)
#define KW_REC_P_RMS           (1u << 3)
#define KW_REC_P_MAX_ALL       (1u << 4)
#define KW_REC_P_MIN_ALL       (1u << 5)
#define KW_REC_P_FINAL         (1u << 6)
#define KW_REC_U               (1u << 7)
#define KW_REC_U_MAX           (1u << 8)
#define KW_REC_U_MIN           (1u << 9)
#define KW_REC_U_RMS           (1u << 10)
#define KW_REC_U_MAX_ALL       (1u << 11)
#define KW_REC_U_MIN_ALL       (1u << 12)
#define KW_REC_U_FINAL         (1u << 13)
#define KW_REC_U_NON_STAGGERED (1u << 14)

/* source modes: saveToDisk.m p_source_mode / u_source_mode */
#define KW_SOURCE_DIRICHLET              0
#define KW_SOURCE_ADDITIVE_NO_CORRECTION 1
#define KW_SOURCE_ADDITIVE               2

/* array_order */
#define KW_COLUMN_MAJOR 0
#define KW_ROW_MAJOR    1

/* absorbing_flag: saveToDisk.m (0 lossless, 1 power-law absorbing, 2 stokes) */
#define KW_LOSSLESS  0
#define KW_ABSORBING 1
#define KW_STOKES    2

/* alpha_mode (createAbsorptionVariables.m:37-71) */
#define KW_ALPHA_NORMAL        0
#define KW_ALPHA_NO_ABSORPTION 1
#define KW_ALPHA_NO_DISPERSION 2

/*
 * One time-varying source field (p, ux, uy or uz).  Mirrors
 * {p,u}_source_flag / _mode / _many / _index / _input of saveToDisk.m:142-265
 * plus the labelled-mask signal index of inputChecking.m:853-887.
 */
typedef struct kw_source {
    uint64_t num_time_samples;   /* *_source_flag: signal length, 0 = field absent */
    int32_t  mode;               /* KW_SOURCE_* */
    uint64_t num_points;         /* number of source grid points */
    const uint64_t *index;       /* [num_points] 1-based linear indices, increasing */
    uint64_t num_signals;        /* rows of input (1 = one signal for all points) */
    const uint64_t *signal_index;/* [num_points] 1-based row per point, or NULL
                                    (NULL: row i for point i when num_signals ==
                                    num_points, row 1 for all when num_signals == 1) */
    const float *input;          /* [num_signals x num_time_samples], already scaled
                                    by scaleSourceTerms.m */
} kw_source;

/*
 * The velocity source of a transducer (kWaveTransducer as `source`):
 * kspaceFirstOrder_inputChecking.m:1160-1209 and the loop hook of
 * kspaceFirstOrder3D.m:888-904.  While t <= signal_length - max(delay),
 * ux at point i gains apodization[i] * input_signal[delay[i] + t - 1]
 * (additive, no k-space correction).  3-D only; excludes u_source.
 */
typedef struct kw_transducer_source {
    uint64_t num_points;         /* active element grid points, 0 = none */
    const uint64_t *index;       /* [num_points] 1-based, increasing: find(active_elements_mask) */
    const uint64_t *delay;       /* [num_points] beamforming delay in samples (delay_mask, 0-based) */
    const float *apodization;    /* [num_points] transmit apodization, or NULL ('Rectangular') */
    uint64_t signal_length;      /* samples of input_signal */
    const float *input_signal;   /* already scaled by 2 c0 dt / dx (scaleSourceTerms.m:377-390) */
} kw_transducer_source;

typedef struct kw_problem {
    uint32_t abi_version;        /* KW_ABI_VERSION */
    int32_t  dim;                /* 2 or 3 */
    uint64_t Nx, Ny, Nz;         /* Nz = 1 in 2D (saveToDisk.m:146-149) */
    uint64_t Nt;                 /* kgrid.Nt */
    double   dx, dy, dz, dt;
    double   c_ref;              /* setSoundSpeedRef.m result */

    /* medium: pointer to N values, or NULL to use the scalar */
    const float *c0;        double c0_scalar;
    const float *rho0;      double rho0_scalar;
    /* staggered densities rho0_sg{x,y,z} (kspaceFirstOrder3D.m:585-601);
       NULL -> rho0 */
    const float *rho0_sgx, *rho0_sgy, *rho0_sgz;

    uint64_t pml_x_size, pml_y_size, pml_z_size;
    double   pml_x_alpha, pml_y_alpha, pml_z_alpha;

    int32_t  use_kspace;         /* 'UsekSpace' (default 1) */
    int32_t  use_sg;             /* 'UseSG' (default 1) */

    int32_t  nonlinear_flag;
    const float *BonA;      double BonA_scalar;

    int32_t  absorbing_flag;     /* KW_LOSSLESS / KW_ABSORBING / KW_STOKES */
    const float *alpha_coeff; double alpha_coeff_scalar;  /* dB/(MHz^y cm) */
    double   alpha_power;
    int32_t  alpha_mode;         /* KW_ALPHA_* */
    double   alpha_sign[2];      /* medium.alpha_sign, {1,1} when absent */

    kw_source p_source;
    kw_source u_source[3];       /* ux, uy, uz; share mode/index/signal_index */
    const float *p0_source_input;/* smoothed p0 (N values) or NULL */

    /* sensor (binary mask, find(mask) order); time reversal when
       time_reversal_input != NULL */
    uint64_t sensor_num;
    const uint64_t *sensor_mask_index;  /* [sensor_num] 1-based, increasing */
    uint64_t record_start_index;        /* >= 1 */
    uint32_t record;                    /* KW_REC_* mask */
    const float *time_reversal_input;   /* [sensor_num x Nt] as given (not flipped) */

    /* region kept by *_all and *_final outputs (record.x1_inside...), 1-based
       inclusive, per axis */
    uint64_t inside_lo[3], inside_hi[3];

    int32_t  device;             /* CUDA device ordinal of the plan ('DeviceNum') */

    /* Memory order of the grid-sized arrays (c0, rho0, rho0_sg*, BonA,
       alpha_coeff, p0_source_input): KW_COLUMN_MAJOR as MATLAB stores them,
       or KW_ROW_MAJOR (C / numpy order, last axis fastest), which the library
       transposes on the device.  Linear indices (source and sensor) are
       column-major in both cases. */
    int32_t  array_order;
    /* Non-zero: form rho0_sg{x,y,z} on the device as the midpoint average of
       rho0 with its +1 neighbour along each axis, rho0 itself on the last
       plane (the linear interpolation at x + dx/2 of
       kspaceFirstOrder3D.m:585-601, NaN edge replaced by rho0); the rho0_sg*
       pointers must then be NULL and rho0 an array. */
    int32_t  derive_rho0_sg;

    /* Interpolated sensor points (Cartesian sensor masks with 'CartInterp'
       'linear', createStorageVariables.m:376-400): 0 or 1 = one grid cell
       per point (sensor_mask_index as above); K > 1 = each of the sensor_num
       points is sum_k sensor_weights[m + M k] * field(sensor_mask_index[m + M k])
       (extractSensorData.m:301-352), both arrays column-major M x K, indices
       1-based in any order.  Time reversal and the gradient need K <= 1. */
    uint32_t sensor_vertices;
    const float *sensor_weights;

    /* medium.alpha_filter (createAbsorptionVariables.m:56-76): N values in
       natural (fftshift-ed) wavenumber order, laid out like the other grid
       arrays (array_order), multiplying both absorption operators; NULL when
       absent.  Power-law absorption only (absorbing_flag KW_ABSORBING). */
    const float *alpha_filter;

    /* transducer velocity source; num_points 0 when absent */
    kw_transducer_source transducer_source;

    /* 'StreamToDisk' (kspaceFirstOrder3D.m:1101-1146, 1235-1295): 0 = off;
       otherwise the p time series is recorded through a device buffer of
       this many time steps, and kw_run writes each filled buffer out during
       the loop -- appended to stream_to_disk_file (FP32, column-major
       sensor_num x steps blocks, as fwrite writes them), which is read back
       into out->p after the loop and deleted, or, with no file, straight
       into out->p.  3-D forward runs recording p only.  The device holds
       sensor_num x stream_to_disk values of the series instead of the whole
       record; kw_copy_outputs cannot return a streamed p. */
    uint64_t stream_to_disk;
    const char *stream_to_disk_file;
} kw_problem;

/* Output sizes (createStorageVariables.m:58-88). */
typedef struct kw_output_desc {
    uint64_t sensor_num;          /* rows of time-series outputs */
    uint64_t num_time_points;     /* Nt - record_start_index + 1 */
    uint64_t inside_shape[3];     /* shape of *_all / *_final outputs */
    uint64_t grid_shape[3];
} kw_output_desc;

/* Caller-allocated host buffers; NULL for outputs not recorded. */
typedef struct kw_outputs {
    float *p, *p_max, *p_min, *p_rms, *p_max_all, *p_min_all, *p_final;
    float *u[3], *u_max[3], *u_min[3], *u_rms[3], *u_max_all[3], *u_min_all[3];
    float *u_final[3], *u_non_staggered[3];
} kw_outputs;

typedef struct kw_plan kw_plan;

/* Last error message of the calling thread ("" if none). */
const char *kw_last_error(void);

/* Library / ABI version. */
int kw_abi_version(void);

/* Validate *problem, upload it and build every operator on the device.
   Replaces the external binary's read of the HDF5 input file
   (kspaceFirstOrder3DC.m:530-546). */
kw_status kw_plan_create(const kw_problem *problem, kw_plan **plan);

/* Sizes of every output of this plan. */
kw_status kw_plan_outputs(const kw_plan *plan, kw_output_desc *desc);

/* Run the whole time loop and copy the recorded outputs to *out.
   Synchronous.  Equivalent of running the binary and reading its HDF5
   outputs (kspaceFirstOrder3DC.m:546-780).  Recorded time series of 64 MB or
   more are copied into *out chunk by chunk while the loop runs (through a
   pinned host ring the library keeps for reuse); the results are the same as
   kw_run_device followed by kw_copy_outputs. */
kw_status kw_run(kw_plan *plan, kw_outputs *out);

/* Split form of kw_run: kw_run_device leaves every output on the device;
   kw_copy_outputs copies them to the host.  kw_reset restores the initial
   state so the plan can run again. */
kw_status kw_reset(kw_plan *plan);
kw_status kw_run_device(kw_plan *plan);
kw_status kw_copy_outputs(kw_plan *plan, kw_outputs *out);

/* Advance the loop by n steps (n <= remaining); used by step-wise callers. */
kw_status kw_step(kw_plan *plan, uint64_t n);

/* Free every resource of the plan. */
kw_status kw_plan_destroy(kw_plan *plan);

/*
 * Kernel timing: when enabled, each launch of the kernel classes selected by
 * class_mask is bracketed by CUDA events on the plan's stream; kw_get_timing
 * returns the summed device milliseconds and the launch count for one class.
 */
#define KW_KCLASS_ZSTAGE_U   0   /* momentum update + z transforms */
#define KW_KCLASS_ZSTAGE_R   1   /* mass conservation / equation of state + z transforms */
#define KW_KCLASS_ZSTAGE_P   2   /* absorbing pressure finish + z transform */
#define KW_KCLASS_YPASS      3   /* y-axis FFT passes */
#define KW_KCLASS_XPASS      4   /* x-axis fused forward/operator/inverse passes */
#define KW_KCLASS_SENSOR     5   /* sensor gather / reduction */
#define KW_KCLASS_SOURCE     6   /* source scatter / injection */
#define KW_KCLASS_COUNT      7
kw_status kw_set_timing(kw_plan *plan, uint32_t class_mask);
kw_status kw_get_timing(const kw_plan *plan, int kclass, double *total_ms, uint64_t *launches);

/* Device bytes held by the plan. */
kw_status kw_plan_device_bytes(const kw_plan *plan, uint64_t *bytes);

/* Run the whole loop n times back to back (each from the initial state) on
   the plan's stream between two CUDA events; *device_ms is the elapsed device
   time.  Outputs of the last run stay on the device. */
kw_status kw_run_timed(kw_plan *plan, uint32_t n, double *device_ms);

/* Number of kernels the plan has launched since creation. */
kw_status kw_launch_count(const kw_plan *plan, uint64_t *launches);

/*
 * Serving: continuous batching of independent simulations on one GPU.  A
 * persistent worker thread admits submitted problems in arrival order
 * whenever the HBM budget and the slot limit allow, keeps every admitted
 * simulation's fields and operators resident, and advances all of them in
 * slices of steps on their own streams so their kernels overlap on the
 * device; finished simulations release their memory and slot at once.  No
 * reference counterpart (the reference runs one simulation per call).
 */
typedef struct kw_server kw_server;

typedef struct kw_server_config {
    int32_t  device;             /* CUDA device ordinal */
    uint64_t hbm_budget_bytes;   /* admission budget; 0 = 80% of free memory */
    int32_t  max_active;         /* simulations resident at once; 0 = 32 */
    int32_t  steps_per_slice;    /* steps issued per simulation per round; 0 = 64 */
    /* Watchdog: a request still running this many milliseconds after its
       admission is stopped -- no further steps are issued, the work already
       issued drains, its memory and slot are released -- and its waiter gets
       KW_ERR_TIMEOUT.  0 = no deadline. */
    uint32_t request_timeout_ms;
    /* Grid cells that fill the GPU: a resident request of this many cells
       or more has its slices issued alone, smaller ones share the device in
       proportion to their size (in-flight cells summed up to this); the
       oldest waiting request goes first.  0 = 4 Mi cells. */
    uint64_t fill_cells;
} kw_server_config;

typedef struct kw_server_stats {
    uint64_t submitted, admitted, completed, failed;
    uint64_t active, pending;
    double   p50_ms, p99_ms, mean_ms;   /* submit -> result latency of completed requests */
    double   cell_steps;                /* cell-steps of completed requests */
    double   busy_seconds;              /* first admission -> last completion */
    /* worker thread time: plan set-up, issuing step slices, retiring
       (outputs to host, release), waiting with every run in flight */
    double   setup_seconds, issue_seconds, retire_seconds, wait_seconds;
} kw_server_stats;

kw_status kw_server_create(const kw_server_config *config, kw_server **server);
/* Copies every array of *problem; the caller may free them on return. */
kw_status kw_server_submit(kw_server *server, const kw_problem *problem, uint64_t *ticket);
/* Blocks until the request is done; copies its outputs (like kw_copy_outputs). */
kw_status kw_server_wait(kw_server *server, uint64_t ticket, kw_outputs *out, double *latency_ms);
/* kw_server_wait bounded by timeout_ms of host time: returns KW_ERR_TIMEOUT
   if the request has not finished by then; the ticket stays valid and a
   later wait returns its result. */
kw_status kw_server_wait_for(kw_server *server, uint64_t ticket, uint32_t timeout_ms, kw_outputs *out,
                             double *latency_ms);
kw_status kw_server_get_stats(kw_server *server, kw_server_stats *stats);
/* Stops the worker after the admitted and pending requests finish. */
kw_status kw_server_destroy(kw_server *server);

/*
 * Tile widths of the compile-time transform kernels (lines per block of the
 * z-stages, the y-pass and the x-pass; 0 for a class that runs the runtime
 * kernels).  Plan creation picks them by rule and then by timing (the
 * autotuner, which may give the three z-stages different widths;
 * environment variable KW_AUTOTUNE=0 turns it off).  kw_plan_tiles reports
 * the momentum stage's z width.  kw_set_tiles accepts, per class, the full
 * width, half of it or a quarter of it, sets every z-stage to tiles[0] and
 * rejects anything else; results do not depend on the choice.
 */
kw_status kw_plan_tiles(const kw_plan *plan, int32_t tiles[3]);
kw_status kw_set_tiles(kw_plan *plan, const int32_t tiles[3]);

/*
 * Gradient of a sensor misfit with respect to the sound speed and the density
 * (the adjoint form).  No counterpart in the reference, which offers time
 * reversal only: this is the exact discrete adjoint of the plan's own time
 * loop for lossless linear media with additive pressure sources and a binary
 * sensor mask (kspaceFirstOrder3D.m:792-1040 run backwards).
 *
 * residual[m + M * (t - record_start_index)] = dJ/dp_m(t), in the layout of
 * the p output (M = sensor_num rows, Nt - record_start_index + 1 columns);
 * for J = 1/2 sum (p - d)^2 it is p - d.  grad_c and grad_rho (either may be
 * NULL) receive dJ/dc0 and dJ/drho0 at every grid cell, column-major.  c_ref,
 * dt, the PML and the (already scaled) source signals are held fixed; the
 * density gradient includes the chain through rho0_sg{x,y,z} when they are
 * formed from rho0 (derive_rho0_sg, or a scalar density).
 *
 * Memory: sqrt(Nt) checkpointing -- the state (u_i, rho_i, p) is kept after
 * every checkpoint_interval-th step (0: round(sqrt(Nt))) and each segment is
 * re-run once, so about (Nt / K + K) (2 D + 1) N floats of device memory are
 * used for the call.  The plan's recorded outputs are left as they were; the
 * plan is reset on return.  Other media or sources: KW_ERR_UNSUPPORTED.
 */
kw_status kw_adjoint_gradient(kw_plan *plan, const float *residual, uint32_t checkpoint_interval, double *grad_c,
                              double *grad_rho);

/*
 * Keep the adjoint's checkpoints from the plan's own runs.  No counterpart in
 * the reference.  With enable != 0, every later complete run of the loop
 * (kw_run, kw_run_device, or kw_step up to Nt from a fresh start) also keeps
 * the state after every checkpoint_interval-th step (0: round(sqrt(Nt))), so
 * a kw_adjoint_gradient that follows it with the same interval skips its own
 * forward pass: the misfit's forward run is the checkpointing run.  The
 * states are the ones kw_adjoint_gradient would compute, so its result is
 * unchanged.  Costs (Nt / K - 1) (2 D + 1) N floats of device memory, held
 * until enable = 0 or kw_plan_destroy; any reset, or an incomplete run,
 * discards the kept states.  Time reversal plans: KW_ERR_UNSUPPORTED.
 */
kw_status kw_keep_checkpoints(kw_plan *plan, int32_t enable, uint32_t checkpoint_interval);

/*
 * Allocation-free staggered spectral gradient.  No counterpart in the
 * reference: it exists for callers that must not have this library allocate
 * device memory -- a MEX function working on gpuArray data owned by MATLAB's
 * memory pool, a PyTorch extension that takes every byte from the
 * framework's caching allocator, or a service that forbids device
 * allocation after start-up.
 *
 * Computes out = real(ifftn(d_k * kappa * fftn(field))) on the calling
 * thread's current device, where d_k = i k exp(shift_sign * i k d / 2) along
 * `axis` (0 = x, 1 = y, 2 = z; shift_sign +1 / -1 / 0 gives the reference's
 * ddx_k_shift_pos / ddx_k_shift_neg / unstaggered operator,
 * kspaceFirstOrder3D.m:629-650) and kappa = sinc(c_ref |k| dt / 2) when
 * use_kspace is non-zero, else 1.  field and out are device pointers to
 * column-major FP32 grids of shape[0] x shape[1] (x shape[2] in 3-D); they
 * may alias.  `stream` is a cudaStream_t (NULL: the default stream); the
 * call returns after the result is written.
 *
 * It calls no cudaMalloc or cudaFree.  Its only other device memory is one
 * file-scope array of 32 MiB, held by every GPU that loads the library until
 * the process exits.  The array holds the half spectrum, shape[0] *
 * shape[1] * (floor(shape[2] / 2) + 1) complex FP32 values in 3-D
 * (shape[0] * (floor(shape[1] / 2) + 1) in 2-D), plus a few kilobytes of
 * operator tables, so grids of up to about 8.3 million cells fit: 200^3 is
 * accepted, 256 x 256 x 128 is rejected with KW_ERR_UNSUPPORTED.  The first
 * call on each device looks up the array's device address with that device
 * current.  No call may be made while its stream is being captured: each call
 * copies operator tables from host memory and synchronizes the stream, so a
 * call on a capturing stream returns KW_ERR_UNSUPPORTED.  The address is
 * kept for the life of the process: after cudaDeviceReset it is stale, so do
 * not call this entry point again in a process that has reset the device.
 * Every call shares the array, so calls that overlap on the GPU (other host
 * threads, other streams) race; issue them one at a time.
 */
kw_status kw_gradient_noalloc(int32_t dim, const uint64_t shape[3], const double spacing[3], int32_t axis,
                              int32_t shift_sign, double c_ref, double dt, int32_t use_kspace,
                              const float *field, float *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* KWAVE_B200_H */
