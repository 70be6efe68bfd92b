/*
 * plategpu_napi.c -- Node-API addon exposing the plate solver's C ABI
 * (include/plategpu.h) to the reference's TypeScript GPU-solver module.
 *
 *   solve(problem) -> Promise<result>   pg_solve on a libuv worker thread
 *   isAvailable() -> boolean            pg_is_available
 *   clearCache() -> undefined           pg_clear_cache
 *
 * `problem` carries typed arrays (nodes: Float32Array, elements:
 * Uint32Array, colorOffsets / elementsByColor: Uint32Array, F: Float32Array,
 * constrained: Uint8Array, elemT: Float32Array | undefined) and numbers
 * (nodeCount, elementCount, nodesPerElement, E, nu, t, tolerance,
 * maxIterations, precision, preconditioner, smoother, stopRule).  The
 * inputs are copied before the work is queued, so the caller may reuse its arrays at once; the result's
 * `solution` is a fresh Float64Array.  A non-OK pg_status rejects the
 * promise with an Error carrying pg_last_error() and the status name.
 *
 * node_api.h is not needed to build this file: it declares the stable
 * Node-API C functions it calls (ABI version 8), which the node binary
 * provides when it loads the addon.
 */
#include <pthread.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "plategpu.h"

/* ---- the subset of the Node-API C ABI this addon uses ---- */
typedef struct napi_env__* napi_env;
typedef struct napi_value__* napi_value;
typedef struct napi_callback_info__* napi_callback_info;
typedef struct napi_deferred__* napi_deferred;
typedef struct napi_async_work__* napi_async_work;
typedef int napi_status; /* napi_ok == 0 */
typedef napi_value (*napi_callback)(napi_env env, napi_callback_info info);
typedef void (*napi_async_execute_callback)(napi_env env, void* data);
typedef void (*napi_async_complete_callback)(napi_env env, napi_status status, void* data);
typedef enum {
    napi_int8_array,
    napi_uint8_array,
    napi_uint8_clamped_array,
    napi_int16_array,
    napi_uint16_array,
    napi_int32_array,
    napi_uint32_array,
    napi_float32_array,
    napi_float64_array
} napi_typedarray_type;
typedef enum { napi_undefined, napi_null, napi_boolean, napi_number } napi_valuetype_prefix;

napi_status napi_get_cb_info(napi_env, napi_callback_info, size_t*, napi_value*, napi_value*, void**);
napi_status napi_get_named_property(napi_env, napi_value, const char*, napi_value*);
napi_status napi_has_named_property(napi_env, napi_value, const char*, bool*);
napi_status napi_typeof(napi_env, napi_value, int*);
napi_status napi_get_typedarray_info(napi_env, napi_value, napi_typedarray_type*, size_t*, void**,
                                     napi_value*, size_t*);
napi_status napi_get_value_double(napi_env, napi_value, double*);
napi_status napi_create_promise(napi_env, napi_deferred*, napi_value*);
napi_status napi_resolve_deferred(napi_env, napi_deferred, napi_value);
napi_status napi_reject_deferred(napi_env, napi_deferred, napi_value);
napi_status napi_create_async_work(napi_env, napi_value, napi_value, napi_async_execute_callback,
                                   napi_async_complete_callback, void*, napi_async_work*);
napi_status napi_queue_async_work(napi_env, napi_async_work);
napi_status napi_delete_async_work(napi_env, napi_async_work);
napi_status napi_create_object(napi_env, napi_value*);
napi_status napi_create_double(napi_env, double, napi_value*);
napi_status napi_get_boolean(napi_env, bool, napi_value*);
napi_status napi_get_undefined(napi_env, napi_value*);
napi_status napi_create_arraybuffer(napi_env, size_t, void**, napi_value*);
napi_status napi_create_typedarray(napi_env, napi_typedarray_type, size_t, napi_value, size_t,
                                   napi_value*);
napi_status napi_create_string_utf8(napi_env, const char*, size_t, napi_value*);
napi_status napi_create_error(napi_env, napi_value, napi_value, napi_value*);
napi_status napi_set_named_property(napi_env, napi_value, const char*, napi_value);
napi_status napi_create_function(napi_env, const char*, size_t, napi_callback, void*, napi_value*);
napi_status napi_throw_error(napi_env, const char*, const char*);
napi_status napi_create_array_with_length(napi_env, size_t, napi_value*);
napi_status napi_set_element(napi_env, napi_value, uint32_t, napi_value);
#define NAPI_AUTO_LENGTH ((size_t)-1)

/* ---- one solver context per CUDA device, created on first use ---- */
#define MAX_DEVICES 16
static pthread_mutex_t g_ctx_mu = PTHREAD_MUTEX_INITIALIZER;
static pg_ctx* g_ctx[MAX_DEVICES];
static int g_ctx_status[MAX_DEVICES];

static pg_ctx* shared_ctx(int device, int* status) {
    if (device < 0 || device >= MAX_DEVICES) {
        *status = PG_EINVAL;
        return NULL;
    }
    pthread_mutex_lock(&g_ctx_mu);
    if (!g_ctx[device] && g_ctx_status[device] == PG_OK)
        g_ctx_status[device] = pg_create(device, &g_ctx[device]);
    *status = g_ctx[device] ? PG_OK : g_ctx_status[device];
    pg_ctx* c = g_ctx[device];
    pthread_mutex_unlock(&g_ctx_mu);
    return c;
}

static const char* status_name(int st) {
    static const char* n[] = {"PG_OK", "PG_EINVAL", "PG_ENOMEM", "PG_ECUDA",
                              "PG_ETIMEOUT", "PG_ENONFINITE", "PG_EUNSUPPORTED"};
    return st >= 0 && st <= 6 ? n[st] : "PG_UNKNOWN";
}

typedef struct {
    napi_deferred deferred;
    napi_async_work work;
    pg_problem prob;
    pg_options opt;
    pg_info info;
    void* owned[7]; /* copies of the input arrays */
    double* x;
    int cases;       /* > 0: a load-case job (pg_solve_load_cases), F holds `cases` loads */
    int device;      /* CUDA device of the job's context */
    pg_info* infos;  /* [cases] */
    int status;
    char error[512];
} SolveJob;

static void job_free(SolveJob* j) {
    for (int i = 0; i < 7; i++) free(j->owned[i]);
    free(j->x);
    free(j->infos);
    free(j);
}

/* Copies a typed array property (NULL when absent and optional). */
static int copy_array(napi_env env, napi_value obj, const char* name, napi_typedarray_type want,
                      size_t elem, size_t expect, int optional, void** out) {
    bool has = false;
    *out = NULL;
    if (napi_has_named_property(env, obj, name, &has) != 0) return -1;
    napi_value v;
    if (has && napi_get_named_property(env, obj, name, &v) != 0) return -1;
    int type = 0;
    if (has && napi_typeof(env, v, &type) != 0) return -1;
    if (!has || type == napi_undefined || type == napi_null) return optional ? 0 : -1;
    napi_typedarray_type t;
    size_t len = 0, off = 0;
    void* data = NULL;
    napi_value ab;
    if (napi_get_typedarray_info(env, v, &t, &len, &data, &ab, &off) != 0 || t != want) return -1;
    if (len != expect) return -1;
    *out = malloc(len * elem > 0 ? len * elem : 1);
    if (!*out) return -1;
    if (len) memcpy(*out, data, len * elem);
    return 0;
}

static int get_number(napi_env env, napi_value obj, const char* name, double def, double* out) {
    bool has = false;
    *out = def;
    if (napi_has_named_property(env, obj, name, &has) != 0) return -1;
    if (!has) return 0;
    napi_value v;
    int type = 0;
    if (napi_get_named_property(env, obj, name, &v) != 0 || napi_typeof(env, v, &type) != 0) return -1;
    if (type == napi_undefined || type == napi_null) return 0;
    return napi_get_value_double(env, v, out) == 0 ? 0 : -1;
}

static void solve_execute(napi_env env, void* data) {
    (void)env;
    SolveJob* j = (SolveJob*)data;
    int st = PG_OK;
    pg_ctx* ctx = shared_ctx(j->device, &st);
    if (!ctx) {
        j->status = st;
        strncpy(j->error, st == PG_EINVAL ? "device index out of range" : pg_last_error(NULL),
                sizeof j->error - 1);
        return;
    }
    if (j->cases > 0)
        j->status = pg_solve_load_cases(ctx, &j->prob, j->cases, j->prob.F, &j->opt, 0, j->x, j->infos);
    else
        j->status = pg_solve(ctx, &j->prob, &j->opt, j->x, &j->info);
    if (j->status != PG_OK) strncpy(j->error, pg_last_error(ctx), sizeof j->error - 1);
}

static void set_num(napi_env env, napi_value o, const char* k, double v) {
    napi_value n;
    napi_create_double(env, v, &n);
    napi_set_named_property(env, o, k, n);
}

/* The result object of case k of a load-case job, or of the one solve (k < 0). */
static napi_value result_object(napi_env env, const SolveJob* j, int k) {
    const size_t n = 3 * (size_t)j->prob.node_count;
    const pg_info* in = k < 0 ? &j->info : &j->infos[k];
    void* buf = NULL;
    napi_value ab, arr, res, b;
    napi_create_arraybuffer(env, n * sizeof(double), &buf, &ab);
    if (n) memcpy(buf, j->x + (k < 0 ? 0 : (size_t)k * n), n * sizeof(double));
    napi_create_typedarray(env, napi_float64_array, n, ab, 0, &arr);
    napi_create_object(env, &res);
    napi_set_named_property(env, res, "solution", arr);
    set_num(env, res, "iterations", in->iterations);
    set_num(env, res, "finalResidual", in->final_residual);
    napi_get_boolean(env, in->converged != 0, &b);
    napi_set_named_property(env, res, "converged", b);
    set_num(env, res, "gpuTimeMs", in->total_ms);
    set_num(env, res, "trueRelResidual", in->true_rel_residual);
    set_num(env, res, "setupMs", in->setup_ms);
    set_num(env, res, "solveMs", in->solve_ms);
    set_num(env, res, "stopReason", in->stop_reason);
    return res;
}

static void solve_complete(napi_env env, napi_status status, void* data) {
    SolveJob* j = (SolveJob*)data;
    if (status != 0 || j->status != PG_OK) {
        napi_value code, msg, err;
        napi_create_string_utf8(env, status_name(j->status), NAPI_AUTO_LENGTH, &code);
        napi_create_string_utf8(env, j->error[0] ? j->error : "solve failed", NAPI_AUTO_LENGTH, &msg);
        napi_create_error(env, code, msg, &err);
        napi_reject_deferred(env, j->deferred, err);
    } else if (j->cases > 0) {
        napi_value list;
        napi_create_array_with_length(env, (size_t)j->cases, &list);
        for (int k = 0; k < j->cases; k++)
            napi_set_element(env, list, (uint32_t)k, result_object(env, j, k));
        napi_resolve_deferred(env, j->deferred, list);
    } else {
        napi_resolve_deferred(env, j->deferred, result_object(env, j, -1));
    }
    napi_delete_async_work(env, j->work);
    job_free(j);
}

/* solve(problem) and solveLoadCases(problem): problem.F holds one load, or
 * problem.cases loads back to back. */
static napi_value start_job(napi_env env, napi_callback_info info, int load_cases) {
    size_t argc = 1;
    napi_value argv[1], promise, name;
    if (napi_get_cb_info(env, info, &argc, argv, NULL, NULL) != 0 || argc < 1) {
        napi_throw_error(env, "PG_EINVAL", "solve(problem) needs one argument");
        return NULL;
    }
    SolveJob* j = (SolveJob*)calloc(1, sizeof(SolveJob));
    if (!j) {
        napi_throw_error(env, "PG_ENOMEM", "out of memory");
        return NULL;
    }
    double nn, ne, npe, E, nu, t, tol, maxit, prec, pre, smo, stop, cases, device;
    napi_value o = argv[0];
    int bad = get_number(env, o, "nodeCount", -1, &nn) | get_number(env, o, "elementCount", -1, &ne) |
              get_number(env, o, "nodesPerElement", 4, &npe) | get_number(env, o, "E", 0, &E) |
              get_number(env, o, "nu", 0, &nu) | get_number(env, o, "t", 0, &t) |
              get_number(env, o, "tolerance", 1e-6, &tol) |
              get_number(env, o, "maxIterations", 1000, &maxit) |
              get_number(env, o, "precision", PG_PREC_FP64, &prec) |
              get_number(env, o, "preconditioner", PG_PRECOND_BLOCK_JACOBI, &pre) |
              get_number(env, o, "smoother", PG_SMOOTHER_BLOCK_JACOBI, &smo) |
              get_number(env, o, "stopRule", PG_STOP_REFERENCE, &stop) |
              get_number(env, o, "cases", 1, &cases) | get_number(env, o, "device", 0, &device);
    if (!load_cases) cases = 1;
    if (bad || nn < 0 || ne < 0 || nn > 67108864.0 || ne > 67108864.0 || cases < 1 || cases > 65536.0 ||
        !(device >= 0 && device < MAX_DEVICES) || device != (double)(int)device) {
        job_free(j);
        napi_throw_error(env, "PG_EINVAL", "problem needs nodeCount, elementCount, E, nu, t");
        return NULL;
    }
    const size_t Nn = (size_t)nn, Ne = (size_t)ne, k = (size_t)npe;
    napi_value col_obj;
    size_t ncolors = 0;
    {
        napi_typedarray_type ty;
        size_t len = 0, off = 0;
        void* d = NULL;
        napi_value ab;
        if (napi_get_named_property(env, o, "colorOffsets", &col_obj) == 0 &&
            napi_get_typedarray_info(env, col_obj, &ty, &len, &d, &ab, &off) == 0 && len > 0)
            ncolors = len - 1;
    }
    if (copy_array(env, o, "nodes", napi_float32_array, 4, 2 * Nn, 0, &j->owned[0]) ||
        copy_array(env, o, "elements", napi_uint32_array, 4, k * Ne, 0, &j->owned[1]) ||
        copy_array(env, o, "colorOffsets", napi_uint32_array, 4, ncolors + 1, 1, &j->owned[2]) ||
        copy_array(env, o, "elementsByColor", napi_uint32_array, 4, Ne, 1, &j->owned[3]) ||
        copy_array(env, o, "elemT", napi_float32_array, 4, Ne, 1, &j->owned[4]) ||
        copy_array(env, o, "F", napi_float32_array, 4, 3 * Nn * (size_t)cases, 0, &j->owned[5]) ||
        copy_array(env, o, "constrained", napi_uint8_array, 1, 3 * Nn, 0, &j->owned[6])) {
        job_free(j);
        napi_throw_error(env, "PG_EINVAL", "problem arrays missing or of the wrong type / length");
        return NULL;
    }
    j->cases = load_cases ? (int)cases : 0;
    j->device = (int)device;
    j->x = (double*)malloc(3 * Nn * (size_t)cases * sizeof(double) + 8);
    if (load_cases) j->infos = (pg_info*)calloc((size_t)cases, sizeof(pg_info));
    if (!j->x || (load_cases && !j->infos)) {
        job_free(j);
        napi_throw_error(env, "PG_ENOMEM", "out of memory");
        return NULL;
    }
    j->prob.node_count = (uint32_t)Nn;
    j->prob.element_count = (uint32_t)Ne;
    j->prob.nodes_per_element = (uint32_t)k;
    j->prob.nodes = (const float*)j->owned[0];
    j->prob.elements = (const uint32_t*)j->owned[1];
    j->prob.color_count = j->owned[2] && j->owned[3] ? (uint32_t)ncolors : 0;
    j->prob.color_offsets = (const uint32_t*)j->owned[2];
    j->prob.elements_by_color = (const uint32_t*)j->owned[3];
    j->prob.E = E;
    j->prob.nu = nu;
    j->prob.t = t;
    j->prob.elem_t = (const float*)j->owned[4];
    j->prob.F = (const float*)j->owned[5];
    j->prob.constrained = (const uint8_t*)j->owned[6];
    pg_options_default(&j->opt);
    j->opt.tolerance = tol;
    j->opt.max_iterations = (int32_t)maxit;
    j->opt.precision = (int32_t)prec;
    j->opt.preconditioner = (int32_t)pre;
    j->opt.smoother = (int32_t)smo;
    j->opt.stop_rule = (int32_t)stop;
    napi_create_promise(env, &j->deferred, &promise);
    napi_create_string_utf8(env, "plategpu.solve", NAPI_AUTO_LENGTH, &name);
    if (napi_create_async_work(env, NULL, name, solve_execute, solve_complete, j, &j->work) != 0 ||
        napi_queue_async_work(env, j->work) != 0) {
        job_free(j);
        napi_throw_error(env, "PG_ECUDA", "could not queue the solve");
        return NULL;
    }
    return promise;
}

static napi_value js_solve(napi_env env, napi_callback_info info) { return start_job(env, info, 0); }

static napi_value js_solve_load_cases(napi_env env, napi_callback_info info) {
    return start_job(env, info, 1);
}

static napi_value js_is_available(napi_env env, napi_callback_info info) {
    (void)info;
    napi_value b;
    napi_get_boolean(env, pg_is_available() != 0, &b);
    return b;
}

static napi_value js_clear_cache(napi_env env, napi_callback_info info) {
    (void)info;
    /* every context created so far */
    pthread_mutex_lock(&g_ctx_mu);
    for (int d = 0; d < MAX_DEVICES; d++)
        if (g_ctx[d]) pg_clear_cache(g_ctx[d]);
    pthread_mutex_unlock(&g_ctx_mu);
    napi_value u;
    napi_get_undefined(env, &u);
    return u;
}

/* Module entry point looked up by Node for Node-API addons. */
napi_value napi_register_module_v1(napi_env env, napi_value exports) {
    napi_value f;
    napi_create_function(env, "solve", NAPI_AUTO_LENGTH, js_solve, NULL, &f);
    napi_set_named_property(env, exports, "solve", f);
    napi_create_function(env, "solveLoadCases", NAPI_AUTO_LENGTH, js_solve_load_cases, NULL, &f);
    napi_set_named_property(env, exports, "solveLoadCases", f);
    napi_create_function(env, "isAvailable", NAPI_AUTO_LENGTH, js_is_available, NULL, &f);
    napi_set_named_property(env, exports, "isAvailable", f);
    napi_create_function(env, "clearCache", NAPI_AUTO_LENGTH, js_clear_cache, NULL, &f);
    napi_set_named_property(env, exports, "clearCache", f);
    return exports;
}

int32_t node_api_module_get_api_version_v1(void) { return 8; }
