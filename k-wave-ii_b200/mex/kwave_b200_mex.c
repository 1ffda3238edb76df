/*
 * kwave_b200_mex.c -- MATLAB MEX gateway of the B200 k-space time loop.
 *
 *   sensor_data = kwave_b200_mex(vars)
 *
 * `vars` is a struct holding the variables that k-Wave's setup writes for its
 * external native solver at the SaveToDisk hand-off
 * (+kwave/+legacy/private/kspaceFirstOrder_saveToDisk.m:46-376,
 * +kwave/+legacy/kspaceFirstOrder3D.m:669-687), under the same names:
 *
 *   Nx Ny Nz Nt dx dy dz dt c_ref c0 rho0 rho0_sgx rho0_sgy rho0_sgz
 *   pml_x_size pml_y_size pml_z_size pml_x_alpha pml_y_alpha pml_z_alpha
 *   nonlinear_flag BonA absorbing_flag alpha_coeff alpha_power
 *   p_source_flag p_source_mode p_source_many p_source_index p_source_input
 *   ux_source_flag uy_source_flag uz_source_flag u_source_mode u_source_many
 *   u_source_index ux_source_input uy_source_input uz_source_input
 *   p0_source_flag p0_source_input
 *   sensor_mask_type sensor_mask_index sensor_mask_corners
 *
 * plus what the reference passes to the native binary on its command line or
 * keeps in the MATLAB workspace (kspaceFirstOrder3DC.m:465-554):
 *
 *   record              cell array of sensor.record names (default {'p'})
 *   record_start_index  (default 1)
 *   device              CUDA device ordinal (default 0)
 *   dim                 2 or 3 (default: 3 when Nz > 1, else 2)
 *   alpha_mode          'no_absorption' / 'no_dispersion' (optional)
 *   alpha_sign          [sign_tau, sign_eta] (optional)
 *   use_kspace use_sg   'UsekSpace' / 'UseSG' (default 1)
 *   time_reversal_boundary_data   (optional; returns p_final)
 *   x1_inside x2_inside y1_inside y2_inside z1_inside z2_inside
 *                       region of the _all / _final outputs (default: grid)
 *
 * Numeric fields may be of any numeric class; grid arrays are column-major
 * as MATLAB stores them and are passed to the library without a copy when
 * they are single.  The result has the reference's output layout: the p
 * matrix alone when `record` is absent, a struct of outputs otherwise, and a
 * 1 x n struct array (fields reshaped to [X, Y, (Z,) T]) for cuboid-corner
 * masks (kspaceFirstOrder_reorderCuboidCorners.m).  Failures raise a MATLAB
 * error with the library's message (kw_last_error).
 *
 * Build: mex -I<repo>/include kwave_b200_mex.c -L<repo>/k-wave-ii_b200/kwave_b200 -lkwave_b200
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"
#include "kwave_b200.h"

#define ERR_ID "kwave_b200:mex"

/* ---- numeric field access ------------------------------------------------ */

static const mxArray *field(const mxArray *v, const char *name) { return mxGetField(v, 0, name); }

static int has(const mxArray *v, const char *name) {
    const mxArray *f = field(v, name);
    return f != NULL && mxGetNumberOfElements(f) > 0;
}

static double scalar(const mxArray *v, const char *name, double dflt) {
    return has(v, name) ? mxGetScalar(field(v, name)) : dflt;
}

/* element i of a numeric array of any class, as double */
static double elem(const mxArray *a, size_t i) {
    const void *d = mxGetData(a);
    switch (mxGetClassID(a)) {
        case mxDOUBLE_CLASS: return ((const double *)d)[i];
        case mxSINGLE_CLASS: return ((const float *)d)[i];
        case mxLOGICAL_CLASS: return ((const unsigned char *)d)[i];
        case mxINT8_CLASS: return ((const int8_t *)d)[i];
        case mxUINT8_CLASS: return ((const uint8_t *)d)[i];
        case mxINT16_CLASS: return ((const int16_t *)d)[i];
        case mxUINT16_CLASS: return ((const uint16_t *)d)[i];
        case mxINT32_CLASS: return ((const int32_t *)d)[i];
        case mxUINT32_CLASS: return ((const uint32_t *)d)[i];
        case mxINT64_CLASS: return (double)((const int64_t *)d)[i];
        case mxUINT64_CLASS: return (double)((const uint64_t *)d)[i];
        default: mexErrMsgIdAndTxt(ERR_ID, "numeric input expected");
    }
    return 0.0;
}

/* Allocations made while the problem is assembled; freed on every exit. */
typedef struct {
    void *p[64];
    int n;
} Pool;

static void *pool_alloc(Pool *pool, size_t bytes) {
    void *p;
    if (pool->n >= 64) mexErrMsgIdAndTxt(ERR_ID, "internal: allocation pool exhausted");
    p = calloc(bytes ? bytes : 1, 1);
    if (!p) mexErrMsgIdAndTxt(ERR_ID, "host allocation of %zu bytes failed", bytes);
    pool->p[pool->n++] = p;
    return p;
}

static void pool_free(Pool *pool) {
    int i;
    for (i = 0; i < pool->n; ++i) free(pool->p[i]);
    pool->n = 0;
}

/* FP32 view of a numeric field: the data itself when single, else a copy */
static const float *f32(Pool *pool, const mxArray *v, const char *name, size_t *count) {
    const mxArray *a = field(v, name);
    size_t n, i;
    float *out;
    *count = 0;
    if (!a || mxGetNumberOfElements(a) == 0) return NULL;
    n = mxGetNumberOfElements(a);
    *count = n;
    if (mxGetClassID(a) == mxSINGLE_CLASS) return (const float *)mxGetData(a);
    out = (float *)pool_alloc(pool, n * sizeof(float));
    for (i = 0; i < n; ++i) out[i] = (float)elem(a, i);
    return out;
}

/* a medium quantity: a grid array, or a scalar */
static void medium(Pool *pool, const mxArray *v, const char *name, const float **arr, double *val, double dflt) {
    size_t n = 0;
    const float *a = f32(pool, v, name, &n);
    *arr = NULL;
    *val = dflt;
    if (n == 1) *val = a[0];
    else if (n > 1) *arr = a;
}

static const uint64_t *u64(Pool *pool, const mxArray *v, const char *name, size_t *count) {
    const mxArray *a = field(v, name);
    size_t n, i;
    uint64_t *out;
    *count = 0;
    if (!a || mxGetNumberOfElements(a) == 0) return NULL;
    n = mxGetNumberOfElements(a);
    *count = n;
    if (mxGetClassID(a) == mxUINT64_CLASS) return (const uint64_t *)mxGetData(a);
    out = (uint64_t *)pool_alloc(pool, n * sizeof(uint64_t));
    for (i = 0; i < n; ++i) out[i] = (uint64_t)elem(a, i);
    return out;
}

/* ---- sensor.record ------------------------------------------------------- */

static const struct {
    const char *name;
    uint32_t bit;
} kRecord[] = {
    {"p", KW_REC_P}, {"p_max", KW_REC_P_MAX}, {"p_min", KW_REC_P_MIN}, {"p_rms", KW_REC_P_RMS},
    {"p_max_all", KW_REC_P_MAX_ALL}, {"p_min_all", KW_REC_P_MIN_ALL}, {"p_final", KW_REC_P_FINAL},
    {"u", KW_REC_U}, {"u_max", KW_REC_U_MAX}, {"u_min", KW_REC_U_MIN}, {"u_rms", KW_REC_U_RMS},
    {"u_max_all", KW_REC_U_MAX_ALL}, {"u_min_all", KW_REC_U_MIN_ALL}, {"u_final", KW_REC_U_FINAL},
    {"u_non_staggered", KW_REC_U_NON_STAGGERED},
};

static uint32_t record_bits(const mxArray *v) {
    const mxArray *r = field(v, "record");
    uint32_t bits = 0;
    size_t i, k;
    if (!r) return KW_REC_P;
    if (!mxIsCell(r)) mexErrMsgIdAndTxt(ERR_ID, "sensor.record must be given as a cell array, e.g., {'p', 'u'}.");
    for (i = 0; i < mxGetNumberOfElements(r); ++i) {
        char *s = mxArrayToString(mxGetCell(r, i));
        int found = 0;
        if (!s) mexErrMsgIdAndTxt(ERR_ID, "sensor.record entries must be strings.");
        for (k = 0; k < sizeof kRecord / sizeof kRecord[0]; ++k)
            if (strcmp(s, kRecord[k].name) == 0) { bits |= kRecord[k].bit; found = 1; }
        if (!found) {
            char msg[128];
            snprintf(msg, sizeof msg, "'%s' is not a valid input for sensor.record.", s);
            mxFree(s);
            mexErrMsgIdAndTxt(ERR_ID, "%s", msg);
        }
        mxFree(s);
    }
    return bits;
}

/* ---- sources ------------------------------------------------------------- */

static void source(Pool *pool, const mxArray *v, kw_source *s, const char *flag, const char *mode, const char *many,
                   const char *index, const char *input) {
    size_t n = 0, nin = 0;
    memset(s, 0, sizeof *s);
    s->num_time_samples = (uint64_t)scalar(v, flag, 0);
    if (!s->num_time_samples) return;
    s->mode = (int32_t)scalar(v, mode, KW_SOURCE_ADDITIVE);
    s->index = u64(pool, v, index, &n);
    s->num_points = n;
    s->input = f32(pool, v, input, &nin);
    s->num_signals = scalar(v, many, 0) != 0 ? n : 1;
    if (!s->index || !s->input || nin != s->num_signals * s->num_time_samples)
        mexErrMsgIdAndTxt(ERR_ID, "source %s: index or input missing or of the wrong size", input);
}

/* ---- cuboid corners (sensor_mask_type 1) --------------------------------- */

typedef struct {
    size_t n;               /* cuboids */
    uint64_t *lo, *hi;      /* [3 n], 1-based inclusive */
    uint64_t *rows;         /* per concatenated point: its row in the sorted index list */
    size_t total;           /* concatenated points */
} Cuboids;

static int cmp_u64(const void *a, const void *b) {
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

/* Every cuboid's find() in order, concatenated (inputChecking.m:1610-1633);
   the library takes the sorted distinct indices, and `rows` maps each
   concatenated point to its row there. */
static const uint64_t *cuboid_index(Pool *pool, const mxArray *v, const kw_problem *pr, Cuboids *cb, size_t *num) {
    const mxArray *c = field(v, "sensor_mask_corners");
    const uint64_t N[3] = {pr->Nx, pr->Ny, pr->Nz};
    size_t i, a, k, m = 0, u = 0;
    uint64_t *all, *uniq;
    if (!c || mxGetM(c) != 6) mexErrMsgIdAndTxt(ERR_ID, "sensor_mask_corners must be 6 x n");
    cb->n = mxGetN(c);
    cb->lo = (uint64_t *)pool_alloc(pool, 3 * cb->n * sizeof(uint64_t));
    cb->hi = (uint64_t *)pool_alloc(pool, 3 * cb->n * sizeof(uint64_t));
    cb->total = 0;
    for (i = 0; i < cb->n; ++i) {
        size_t cnt = 1;
        for (a = 0; a < 3; ++a) {
            cb->lo[3 * i + a] = (uint64_t)elem(c, 6 * i + a);
            cb->hi[3 * i + a] = (uint64_t)elem(c, 6 * i + 3 + a);
            if (cb->lo[3 * i + a] < 1 || cb->hi[3 * i + a] < cb->lo[3 * i + a] || cb->hi[3 * i + a] > N[a])
                mexErrMsgIdAndTxt(ERR_ID, "sensor.mask cuboid corners must be within the grid.");
            cnt *= (size_t)(cb->hi[3 * i + a] - cb->lo[3 * i + a] + 1);
        }
        cb->total += cnt;
    }
    all = (uint64_t *)pool_alloc(pool, cb->total * sizeof(uint64_t));
    for (i = 0; i < cb->n; ++i) {
        uint64_t x, y, z;
        for (z = cb->lo[3 * i + 2]; z <= cb->hi[3 * i + 2]; ++z)
            for (y = cb->lo[3 * i + 1]; y <= cb->hi[3 * i + 1]; ++y)
                for (x = cb->lo[3 * i]; x <= cb->hi[3 * i]; ++x) all[m++] = x + N[0] * ((y - 1) + N[1] * (z - 1));
    }
    uniq = (uint64_t *)pool_alloc(pool, cb->total * sizeof(uint64_t));
    memcpy(uniq, all, cb->total * sizeof(uint64_t));
    qsort(uniq, cb->total, sizeof(uint64_t), cmp_u64);
    for (k = 0; k < cb->total; ++k)
        if (k == 0 || uniq[k] != uniq[u - 1]) uniq[u++] = uniq[k];
    cb->rows = (uint64_t *)pool_alloc(pool, cb->total * sizeof(uint64_t));
    for (k = 0; k < cb->total; ++k) {
        const uint64_t *hit = (const uint64_t *)bsearch(&all[k], uniq, u, sizeof(uint64_t), cmp_u64);
        cb->rows[k] = (uint64_t)(hit - uniq);
    }
    *num = u;
    return uniq;
}

/* ---- outputs ------------------------------------------------------------- */

typedef struct {
    const char *name;
    float **slot;
    int kind;               /* 0: M x T series, 1: M vector, 2: region array */
} OutSpec;

static mxArray *new_single(size_t ndim, const mwSize *dims) {
    return mxCreateNumericArray(ndim, dims, mxSINGLE_CLASS, mxREAL);
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    const mxArray *v;
    Pool pool;
    kw_problem pr;
    kw_plan *plan = NULL;
    kw_output_desc d;
    kw_outputs o;
    Cuboids cb;
    OutSpec spec[32];
    mxArray *arrays[32];
    int nspec = 0, i, cuboid = 0, given_record;
    size_t n, ns = 0;
    kw_status st;
    char err[1024];
    static const char *comp[3] = {"ux", "uy", "uz"};
    static char names[3][7][24];

    (void)nlhs;
    if (nrhs != 1 || !mxIsStruct(prhs[0])) mexErrMsgIdAndTxt(ERR_ID, "usage: sensor_data = kwave_b200_mex(vars)");
    v = prhs[0];
    pool.n = 0;
    memset(&pr, 0, sizeof pr);
    memset(&cb, 0, sizeof cb);
    pr.abi_version = KW_ABI_VERSION;
    pr.Nx = (uint64_t)scalar(v, "Nx", 0);
    pr.Ny = (uint64_t)scalar(v, "Ny", 1);
    pr.Nz = (uint64_t)scalar(v, "Nz", 1);
    pr.dim = (int32_t)scalar(v, "dim", pr.Nz > 1 ? 3 : 2);
    pr.Nt = (uint64_t)scalar(v, "Nt", 0);
    pr.dx = scalar(v, "dx", 0);
    pr.dy = scalar(v, "dy", 0);
    pr.dz = scalar(v, "dz", 0);
    pr.dt = scalar(v, "dt", 0);
    pr.c_ref = scalar(v, "c_ref", 0);
    n = (size_t)(pr.Nx * pr.Ny * pr.Nz);

    medium(&pool, v, "c0", &pr.c0, &pr.c0_scalar, 0);
    medium(&pool, v, "rho0", &pr.rho0, &pr.rho0_scalar, 1);
    pr.rho0_sgx = f32(&pool, v, "rho0_sgx", &ns);
    if (ns == 1) pr.rho0_sgx = NULL;
    pr.rho0_sgy = f32(&pool, v, "rho0_sgy", &ns);
    if (ns == 1) pr.rho0_sgy = NULL;
    pr.rho0_sgz = f32(&pool, v, "rho0_sgz", &ns);
    if (ns == 1) pr.rho0_sgz = NULL;
    pr.pml_x_size = (uint64_t)scalar(v, "pml_x_size", 0);
    pr.pml_y_size = (uint64_t)scalar(v, "pml_y_size", 0);
    pr.pml_z_size = (uint64_t)scalar(v, "pml_z_size", 0);
    pr.pml_x_alpha = scalar(v, "pml_x_alpha", 2);
    pr.pml_y_alpha = scalar(v, "pml_y_alpha", 2);
    pr.pml_z_alpha = scalar(v, "pml_z_alpha", 2);
    pr.use_kspace = (int32_t)scalar(v, "use_kspace", 1);
    pr.use_sg = (int32_t)scalar(v, "use_sg", 1);
    pr.nonlinear_flag = (int32_t)scalar(v, "nonlinear_flag", 0);
    medium(&pool, v, "BonA", &pr.BonA, &pr.BonA_scalar, 0);
    pr.absorbing_flag = (int32_t)scalar(v, "absorbing_flag", KW_LOSSLESS);
    medium(&pool, v, "alpha_coeff", &pr.alpha_coeff, &pr.alpha_coeff_scalar, 0);
    pr.alpha_power = scalar(v, "alpha_power", 0);
    pr.alpha_mode = KW_ALPHA_NORMAL;
    if (has(v, "alpha_mode")) {
        char *m = mxArrayToString(field(v, "alpha_mode"));
        if (m && strcmp(m, "no_absorption") == 0) pr.alpha_mode = KW_ALPHA_NO_ABSORPTION;
        else if (m && strcmp(m, "no_dispersion") == 0) pr.alpha_mode = KW_ALPHA_NO_DISPERSION;
        if (m) mxFree(m);
    }
    pr.alpha_sign[0] = pr.alpha_sign[1] = 1.0;
    if (has(v, "alpha_sign")) {
        if (mxGetNumberOfElements(field(v, "alpha_sign")) != 2)
            mexErrMsgIdAndTxt(ERR_ID, "medium.alpha_sign must be given as a 2 element numerical array.");
        pr.alpha_sign[0] = elem(field(v, "alpha_sign"), 0);
        pr.alpha_sign[1] = elem(field(v, "alpha_sign"), 1);
    }

    source(&pool, v, &pr.p_source, "p_source_flag", "p_source_mode", "p_source_many", "p_source_index",
           "p_source_input");
    source(&pool, v, &pr.u_source[0], "ux_source_flag", "u_source_mode", "u_source_many", "u_source_index",
           "ux_source_input");
    source(&pool, v, &pr.u_source[1], "uy_source_flag", "u_source_mode", "u_source_many", "u_source_index",
           "uy_source_input");
    source(&pool, v, &pr.u_source[2], "uz_source_flag", "u_source_mode", "u_source_many", "u_source_index",
           "uz_source_input");
    if (scalar(v, "p0_source_flag", has(v, "p0_source_input")) != 0) {
        pr.p0_source_input = f32(&pool, v, "p0_source_input", &ns);
        if (ns != n) mexErrMsgIdAndTxt(ERR_ID, "p0_source_input must hold Nx*Ny*Nz values");
    }

    /* sensor */
    given_record = field(v, "record") != NULL;
    pr.record = record_bits(v);
    pr.record_start_index = (uint64_t)scalar(v, "record_start_index", 1);
    if (scalar(v, "sensor_mask_type", 0) == 1) {
        cuboid = 1;
        pr.sensor_mask_index = cuboid_index(&pool, v, &pr, &cb, &ns);
        pr.sensor_num = ns;
    } else {
        pr.sensor_mask_index = u64(&pool, v, "sensor_mask_index", &ns);
        pr.sensor_num = ns;
    }
    if (has(v, "time_reversal_boundary_data")) {
        pr.time_reversal_input = f32(&pool, v, "time_reversal_boundary_data", &ns);
        if (ns != pr.sensor_num * pr.Nt) mexErrMsgIdAndTxt(ERR_ID, "time_reversal_boundary_data must be sensor_num x Nt");
        pr.record = KW_REC_P_FINAL;
    }
    pr.inside_lo[0] = (uint64_t)scalar(v, "x1_inside", 1);
    pr.inside_hi[0] = (uint64_t)scalar(v, "x2_inside", (double)pr.Nx);
    pr.inside_lo[1] = (uint64_t)scalar(v, "y1_inside", 1);
    pr.inside_hi[1] = (uint64_t)scalar(v, "y2_inside", (double)pr.Ny);
    pr.inside_lo[2] = (uint64_t)scalar(v, "z1_inside", 1);
    pr.inside_hi[2] = (uint64_t)scalar(v, "z2_inside", (double)pr.Nz);
    pr.device = (int32_t)scalar(v, "device", 0);
    pr.array_order = KW_COLUMN_MAJOR;
    pr.derive_rho0_sg = (pr.rho0 && !pr.rho0_sgx && !pr.rho0_sgy && !pr.rho0_sgz) ? 1 : 0;

    if (kw_plan_create(&pr, &plan) != KW_OK) {
        snprintf(err, sizeof err, "%s", kw_last_error());
        pool_free(&pool);
        mexErrMsgIdAndTxt(ERR_ID, "%s", err);
    }
    kw_plan_outputs(plan, &d);

    /* one host array per recorded output, written by kw_run in place */
    memset(&o, 0, sizeof o);
#define ADD(nm, sl, k) do { spec[nspec].name = (nm); spec[nspec].slot = (sl); spec[nspec].kind = (k); ++nspec; } while (0)
    if (pr.record & KW_REC_P) ADD("p", &o.p, 0);
    if (pr.record & KW_REC_P_MAX) ADD("p_max", &o.p_max, 1);
    if (pr.record & KW_REC_P_MIN) ADD("p_min", &o.p_min, 1);
    if (pr.record & KW_REC_P_RMS) ADD("p_rms", &o.p_rms, 1);
    if (pr.record & KW_REC_P_MAX_ALL) ADD("p_max_all", &o.p_max_all, 2);
    if (pr.record & KW_REC_P_MIN_ALL) ADD("p_min_all", &o.p_min_all, 2);
    if (pr.record & KW_REC_P_FINAL) ADD("p_final", &o.p_final, 2);
    for (i = 0; i < pr.dim; ++i) {
        snprintf(names[i][0], 24, "%s", comp[i]);
        snprintf(names[i][1], 24, "%s_max", comp[i]);
        snprintf(names[i][2], 24, "%s_min", comp[i]);
        snprintf(names[i][3], 24, "%s_rms", comp[i]);
        snprintf(names[i][4], 24, "%s_max_all", comp[i]);
        snprintf(names[i][5], 24, "%s_min_all", comp[i]);
        snprintf(names[i][6], 24, "%s_final", comp[i]);
        if (pr.record & KW_REC_U) ADD(names[i][0], &o.u[i], 0);
        if (pr.record & KW_REC_U_MAX) ADD(names[i][1], &o.u_max[i], 1);
        if (pr.record & KW_REC_U_MIN) ADD(names[i][2], &o.u_min[i], 1);
        if (pr.record & KW_REC_U_RMS) ADD(names[i][3], &o.u_rms[i], 1);
        if (pr.record & KW_REC_U_MAX_ALL) ADD(names[i][4], &o.u_max_all[i], 2);
        if (pr.record & KW_REC_U_MIN_ALL) ADD(names[i][5], &o.u_min_all[i], 2);
        if (pr.record & KW_REC_U_FINAL) ADD(names[i][6], &o.u_final[i], 2);
    }
#undef ADD
    for (i = 0; i < nspec; ++i) {
        mwSize dims[3];
        if (spec[i].kind == 0) {
            dims[0] = (mwSize)d.sensor_num;
            dims[1] = (mwSize)d.num_time_points;
            arrays[i] = new_single(2, dims);
        } else if (spec[i].kind == 1) {
            dims[0] = (mwSize)d.sensor_num;
            dims[1] = 1;
            arrays[i] = new_single(2, dims);
        } else {
            dims[0] = (mwSize)d.inside_shape[0];
            dims[1] = (mwSize)d.inside_shape[1];
            dims[2] = (mwSize)d.inside_shape[2];
            arrays[i] = new_single(pr.dim, dims);
        }
        *spec[i].slot = (float *)mxGetData(arrays[i]);
    }
    st = kw_run(plan, &o);
    if (st != KW_OK) snprintf(err, sizeof err, "%s", kw_last_error());
    kw_plan_destroy(plan);
    if (st != KW_OK) {
        pool_free(&pool);
        mexErrMsgIdAndTxt(ERR_ID, "%s", err);
    }

    if (pr.time_reversal_input) {
        plhs[0] = arrays[0];                                   /* p_final */
    } else if (!cuboid && !given_record) {
        plhs[0] = arrays[0];                                   /* the p matrix */
    } else if (!cuboid) {
        plhs[0] = mxCreateStructMatrix(1, 1, 0, NULL);
        for (i = 0; i < nspec; ++i) {
            mxAddField(plhs[0], spec[i].name);
            mxSetField(plhs[0], 0, spec[i].name, arrays[i]);
        }
    } else {
        /* kspaceFirstOrder_reorderCuboidCorners.m: per cuboid, its rows
           reshaped to [X, Y, (Z,) T]; whole-grid outputs on the first only */
        size_t c, start = 0;
        plhs[0] = mxCreateStructMatrix(1, cb.n, 0, NULL);
        for (i = 0; i < nspec; ++i) mxAddField(plhs[0], spec[i].name);
        for (c = 0; c < cb.n; ++c) {
            mwSize dims[4];
            size_t npts = 1, a;
            for (a = 0; a < (size_t)pr.dim; ++a) {
                const size_t ax = (pr.dim == 2 && a == 1) ? 1 : a;
                dims[a] = (mwSize)(cb.hi[3 * c + ax] - cb.lo[3 * c + ax] + 1);
                npts *= dims[a];
            }
            for (i = 0; i < nspec; ++i) {
                const float *src = (const float *)mxGetData(arrays[i]);
                const size_t T = spec[i].kind == 0 ? (size_t)d.num_time_points : 1;
                mxArray *dst;
                float *dp;
                size_t r, t;
                if (spec[i].kind == 2) {
                    if (c == 0) mxSetField(plhs[0], 0, spec[i].name, arrays[i]);
                    continue;
                }
                dims[pr.dim] = (mwSize)T;
                dst = new_single((size_t)pr.dim + (spec[i].kind == 0), dims);
                dp = (float *)mxGetData(dst);
                for (t = 0; t < T; ++t)
                    for (r = 0; r < npts; ++r) dp[r + npts * t] = src[cb.rows[start + r] + d.sensor_num * t];
                mxSetField(plhs[0], c, spec[i].name, dst);
            }
            start += npts;
        }
    }
    pool_free(&pool);
}
