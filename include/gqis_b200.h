/*
 * gqis_b200.h - C ABI of the B200 sweep engine behind mesolve_2D / odesolve_2D.
 *
 * The reference launches one NVRTC-compiled CuPy RawKernel per model variant:
 *     cp.RawKernel(kernel_code, "time_evolution_kernel").compile()   gqis/solver.py:2237-2241
 *     time_evolution_kernel(grid, block, args)                        gqis/solver.py:2340
 * with the positional argument list of gqis/solver.py:2322-2339
 * (dt, t_in, num_ParX, num_ParY, num_steps, warmup_steps, ParX*, ParY*, [Const_arr*],
 *  [Rho0_arr*], [solver_param0..k], [adaptive_steps*], results*, [trace*, stride, offset, n]).
 *
 * Here every model variant is a shared library built by nvcc for sm_100a from the project's
 * CUDA templates. Each such "model module" exports the functions below. The caller (the
 * Python front end through ctypes, or any C/C++ host) owns every buffer: the library never
 * allocates or frees caller memory, and no exception crosses the ABI. All entry points return
 * an int status (GQIS_OK on success); gqis_last_error() gives a thread-local message.
 *
 * Buffers are device pointers of the current CUDA device; "stream" is a cudaStream_t
 * (NULL = legacy default stream). Launches are asynchronous on that stream.
 */
#ifndef GQIS_B200_H
#define GQIS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GQIS_ABI_VERSION 1

/* status codes */
#define GQIS_OK 0
#define GQIS_ERR_INVALID 1       /* bad descriptor: sizes, pointers, ABI version */
#define GQIS_ERR_CUDA 2          /* a CUDA runtime call failed (message has the CUDA error) */
#define GQIS_ERR_UNSUPPORTED 3   /* variant not compiled into this module */
#define GQIS_ERR_TOO_LARGE 4     /* request exceeds a stated maximum */
#define GQIS_ERR_CANCELLED 5     /* serving: request cancelled */
#define GQIS_ERR_TIMEOUT 6       /* serving: a bounded wait ran out */
#define GQIS_ERR_BUSY 7          /* serving: no free slot / memory right now */

/* precision forms */
#define GQIS_FORM_FP64 0         /* plain FP64: everything in double (parity form) */
#define GQIS_FORM_FP32 1         /* FP32 state and RHS; FP64 time, drive phase and averages */

/* integrators (names of gqis/cuda_solvers.py:1001-1013, plus dop853a) */
#define GQIS_SOLVER_RK4 0
#define GQIS_SOLVER_LSERK4 1
#define GQIS_SOLVER_LSERK4F 2
#define GQIS_SOLVER_DP5 3
#define GQIS_SOLVER_AB5 4
#define GQIS_SOLVER_ANAS5 5
#define GQIS_SOLVER_TSIT5 6
#define GQIS_SOLVER_ALSHINA6 7
#define GQIS_SOLVER_DOP853 8
#define GQIS_SOLVER_TSIT5A 9
#define GQIS_SOLVER_DOP853A 10

/* output modes (gqis/solver.py:2126-2196) */
#define GQIS_OUT_MEAN 0          /* time average of <O> after warmup: (P, 2) re/im */
#define GQIS_OUT_FINAL 1         /* <O> at the last step: (P, 2) */
#define GQIS_OUT_FINAL_STATE 2   /* reduced state at the last step: (P, S) */
#define GQIS_OUT_MEAN_STATE 3    /* time average of the state: (P, S) */

/* trace modes (gqis/solver.py:2175-2188) */
#define GQIS_TRACE_NONE 0
#define GQIS_TRACE_OBSERVABLE 1  /* (P, num_trace, 2) */
#define GQIS_TRACE_STATE 2       /* (P, num_trace, S) */

/* Static description of one compiled model module. */
typedef struct gqis_model_info {
    int32_t abi_version;
    int32_t state_size;          /* S: real state variables per point */
    int32_t num_consts;          /* length of the Const_arr the module reads */
    int32_t form;                /* GQIS_FORM_* */
    int32_t solver;              /* GQIS_SOLVER_* */
    int32_t output_mode;         /* GQIS_OUT_* */
    int32_t trace_mode;          /* GQIS_TRACE_* */
    int32_t init_from_array;     /* 1: the launch reads rho0 */
    int32_t block_threads;       /* threads per CTA of the sweep kernel */
    int32_t registers_per_thread;
    int32_t sm_count;            /* SMs of the current device */
    int32_t ctas_per_sm;         /* resident CTAs per SM (occupancy) */
    uint64_t model_hash;         /* hash of the emitted model text */
} gqis_model_info;

/* One sweep launch: the flattened grid point p = ix * num_y + iy, p in
 * [point_begin, point_begin + point_count). Per-point buffers (rho0, results, trace,
 * step_counts) are indexed by the LOCAL index p - point_begin, so a shard or a serving
 * chunk passes pointers to its own slice. Real buffers use the form's type (double for
 * GQIS_FORM_FP64, float for GQIS_FORM_FP32); par_x, par_y and consts are always double. */
typedef struct gqis_sweep_desc {
    int32_t abi_version;         /* GQIS_ABI_VERSION */
    int32_t num_x, num_y;        /* sweep axes (num_y = 1 for one axis) */
    int32_t num_steps;           /* output intervals: len(tlist) - 1 */
    int32_t warmup_steps;        /* steps excluded from MEAN / MEAN_STATE */
    int32_t trace_stride;        /* trace: one sample every trace_stride steps ... */
    int32_t trace_offset;        /* ... starting after step trace_offset (0-based) */
    int32_t num_trace;           /* samples per point */
    int64_t point_begin;
    int64_t point_count;
    double dt;                   /* uniform output step of tlist */
    double t_in;                 /* absolute start time */
    const double* par_x;         /* [num_x] */
    const double* par_y;         /* [num_y] */
    const double* consts;        /* [num_consts] runtime constants, or NULL if none */
    const void* rho0;            /* [point_count, S] initial states, or NULL */
    void* results;               /* MEAN/FINAL: [point_count, 2]; state modes: [point_count, S] */
    void* trace;                 /* [point_count, num_trace, 2 or S], or NULL */
    int32_t* step_counts;        /* adaptive: [point_count, 2] accepted/rejected, or NULL */
    uint32_t* work_counter;      /* adaptive: one zeroed uint32 of device scratch (work stealing) */
    double solver_params[8];     /* tsit5a/dop853a: rtol, atol, max_substeps; anas5: fitted value */
} gqis_sweep_desc;

/* Replaces cp.RawKernel(...).compile() metadata (gqis/solver.py:2237-2263): what the
 * module was built for. */
int gqis_model_info_get(gqis_model_info* out);

/* Replaces time_evolution_kernel(grid, block, args) (gqis/solver.py:2322-2340). */
int gqis_sweep_launch(const gqis_sweep_desc* desc, void* stream);

/* Thread-local text of the last error of this module (never NULL). */
const char* gqis_last_error(void);

/* No counterpart in the reference: a launch that allocates nothing, for callers that cannot
 * call cudaMalloc - a host whose caching allocator owns the device memory (a PyTorch or JAX
 * process near its memory cap), a real-time loop where cudaMalloc/cudaFree would synchronize
 * the device, a plugin that is handed only its input and output buffers.
 *
 * Same as gqis_sweep_launch, except that the adaptive kernels take their scratch - the
 * work-stealing point counter - from a file-scope device array of this module
 * (GQIS_NOALLOC_SCRATCH_BYTES, held on every device that loads the module until exit) instead
 * of desc->work_counter, which is ignored. The caller still passes inputs and outputs.
 * Fixed-step modules use no scratch and behave exactly like gqis_sweep_launch.
 *  - At most GQIS_NOALLOC_MAX_POINTS points per call (the counter's range); larger requests
 *    return GQIS_ERR_TOO_LARGE.
 *  - The first call on a device looks up the array's device address (once per device, with
 *    that device current); make that first call before any stream capture. The address is
 *    kept per device ordinal for the life of the process: this entry point supports the
 *    device's primary context only, and not a device reset (cudaDeviceReset) between calls.
 *  - Each call clears the counter on its stream before the kernel. All calls share the one
 *    array: calls whose kernels overlap on the GPU (other streams, other threads) race. */
#define GQIS_NOALLOC_SCRATCH_BYTES 256
#define GQIS_NOALLOC_MAX_POINTS 2147483647LL
int gqis_sweep_launch_noalloc(const gqis_sweep_desc* desc, void* stream);

/* No counterpart in the reference, which launches one sweep per kernel: up to GQIS_BATCH_MAX
 * sweeps of this module (different grids, steps, dt, parameters and buffers; one model, solver,
 * form and output mode) in ONE grid. Replaces a series of time_evolution_kernel launches
 * (gqis/solver.py:2340), e.g. every candidate step count of one calibrate_timesteps search
 * (gqis/solver.py:1131-1180) or point chunks of several serving requests.
 *  - descs: a host array of count descriptors, each valid for gqis_sweep_launch; they travel as
 *    the kernel's parameter, so the call needs no device scratch and makes no copy.
 *  - Fixed-step modules: each sweep's points run as in a launch of their own.
 *  - Adaptive modules: the points of all sweeps share one persistent grid and one work counter
 *    (work_counter: one zeroed uint32 of device scratch; the descriptors' own counters are
 *    ignored), so a lane that finishes a point of one sweep continues with any sweep's next
 *    point; each point's result is the same as in a launch of its own.
 *  - The density-matrix modules have no batch launch (GQIS_ERR_UNSUPPORTED). */
#define GQIS_BATCH_MAX 64
int gqis_sweep_launch_batch(const gqis_sweep_desc* descs, int32_t count, uint32_t* work_counter, void* stream);

/* ---------------------------------------------------------------------------------------
 * Gradients (adjoint modules). No counterpart in the reference, which has no derivatives: a
 * module built with an adjoint (gqis.adjoint) also exports the functions below. For every point
 * they return <O>_avg (the RK4 right-endpoint time average, FP64, bit-identical to the sweep's
 * mean output) and its exact derivative with respect to the module's P parameters (runtime
 * constants and/or sweep parameters), by the discrete adjoint of the RK4 steps with checkpoints.
 * --------------------------------------------------------------------------------------- */
typedef struct gqis_adjoint_desc {
    gqis_sweep_desc sweep;          /* grid, steps, warmup, dt, t_in, inputs; results = [points, 2] FP64:
                                       <O>_avg, or the final <O> in a module built for the final output */
    int32_t num_params;             /* P; must equal the module's */
    int32_t checkpoint_every;       /* steps between stored states (ceil(sqrt(num_steps)) balances memory and time) */
    const double* adjoint_consts;   /* full runtime-constant array in the adjoint's order, or NULL */
    double* grad;                   /* [point_count, P] d<O>_avg / dtheta (or d<O>_final / dtheta) */
    double* scratch;                /* gqis_adjoint_scratch_bytes() bytes of device memory (checkpoints) */
    int64_t scratch_bytes;
} gqis_adjoint_desc;

/* Parameters and state size of the module's adjoint (GQIS_ERR_UNSUPPORTED if it has none). */
int gqis_adjoint_info(int32_t* num_params, int32_t* state_size);

/* Device scratch needed by gqis_adjoint_launch for this many points, steps and checkpoint interval. */
int gqis_adjoint_scratch_bytes(int64_t point_count, int32_t num_steps, int32_t checkpoint_every, int64_t* bytes);

/* Mean (or final) map and its parameter gradient; asynchronous on stream. */
int gqis_adjoint_launch(const gqis_adjoint_desc* desc, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GQIS_B200_H */
