// gqis_module.cuh - the C-ABI entry points of one model module (include/gqis_b200.h).
//
// The generated translation unit defines, before including this file:
//   GQ_MODEL        the emitted model struct
//   GQ_FORM         FormFP64 or FormFP32
//   GQ_SOLVER       an integrator type of gqis_fixed.cuh / gqis_adaptive.cuh
//   GQ_SOLVER_ID    its GQIS_SOLVER_* number
//   GQ_ADAPTIVE     1 for the persistent work-stealing adaptive kernels
//   GQ_OUT, GQ_TRACE  output and trace mode
//   GQ_MODEL_HASH   64-bit hash of the model text
#pragma once

#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "gqis_fixed.cuh"
#include "gqis_adaptive.cuh"
#include "gqis_adjoint.cuh"

#include <type_traits>

#ifndef GQ_WITH_ADJOINT
#define GQ_WITH_ADJOINT 0
#endif
#ifndef GQ_MATRIX
#define GQ_MATRIX 0
#endif
#ifndef GQ_ADJOINT_FINAL
#define GQ_ADJOINT_FINAL 0  // adjoint of the final <O> instead of the time average
#endif
#ifndef GQ_PACK2
#define GQ_PACK2 0  // FP32 RK4 with two points per thread in packed f32x2 arithmetic
#endif
#if GQ_PACK2
#include "gqis_packed.cuh"
#endif

namespace {

thread_local char g_last_error[1024] = "";

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(GQIS_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

using Model = GQ_MODEL;
using Form = GQ_FORM;

#if GQ_MATRIX == 2
// Density-matrix form on the tensor cores (gqis_matrix_tc.cuh): one CTA (N <= 32) or one cluster of
// two CTAs (N = 64) per tile of 128 / N points.
constexpr auto kKernel = gqmatrix_tc::matrix_tc_kernel<Model, GQ_OUT, GQ_TRACE>;
constexpr int kBlock = gqmatrix_tc::TcShape<Model>::THREADS;
constexpr size_t kSmem = gqmatrix_tc::TcShape<Model>::SMEM;
constexpr int kPointsPerCta = gqmatrix_tc::TcShape<Model>::P;
constexpr int kCluster = gqmatrix_tc::TcShape<Model>::CL;
static_assert(Form::id == GQIS_FORM_FP32, "the tensor-core form is an FP32 form");
#elif GQ_MATRIX
// Density-matrix form (gqis_matrix.cuh, included by the generated source): one CTA per point.
constexpr auto kKernel = gqmatrix::matrix_rk4_kernel<Model, Form, GQ_OUT, GQ_TRACE>;
constexpr int kBlock = Model::THREADS;
constexpr size_t kSmem = gqmatrix::smem_bytes<Model, typename Form::real>();
constexpr int kPointsPerCta = 1;
constexpr int kCluster = 1;
static_assert(std::is_same<typename Model::real, typename Form::real>::value, "model data type");
#elif GQ_ADAPTIVE
constexpr auto kKernel = gqadaptive::sweep_adaptive_kernel<GQ_SOLVER, Model, Form, GQ_OUT, GQ_TRACE>;
constexpr int kBlock = GQ_BLOCK;
constexpr size_t kSmem = 0;
#elif GQ_PACK2
constexpr auto kKernel = gqpacked::sweep_pair_kernel<Model, GQ_OUT, GQ_TRACE>;
constexpr int kBlock = GQ_BLOCK;
constexpr size_t kSmem = 0;
static_assert(Form::id == GQIS_FORM_FP32 && GQ_SOLVER_ID == GQIS_SOLVER_RK4,
              "the packed two-point kernel is the FP32 form of RK4");
#else
constexpr auto kKernel = gqfixed::sweep_fixed_kernel<GQ_SOLVER, Model, Form, GQ_OUT, GQ_TRACE>;
constexpr int kBlock = GQ_BLOCK;
constexpr size_t kSmem = 0;
#endif

int check_desc(const gqis_sweep_desc* d) {
    if (!d) return fail(GQIS_ERR_INVALID, "descriptor is NULL");
    if (d->abi_version != GQIS_ABI_VERSION)
        return fail(GQIS_ERR_INVALID, "descriptor ABI version %d, module expects %d", d->abi_version,
                    GQIS_ABI_VERSION);
    if (d->num_x < 1 || d->num_y < 1) return fail(GQIS_ERR_INVALID, "sweep axes must be non-empty");
    const int64_t total = (int64_t)d->num_x * d->num_y;
    if (d->point_begin < 0 || d->point_count < 0 || d->point_begin + d->point_count > total)
        return fail(GQIS_ERR_INVALID, "point range [%lld, %lld) outside the %lld-point grid",
                    (long long)d->point_begin, (long long)(d->point_begin + d->point_count),
                    (long long)total);
    if (d->num_steps < 1) return fail(GQIS_ERR_INVALID, "num_steps must be at least 1");
    if (d->warmup_steps < 0 || d->warmup_steps > d->num_steps)
        return fail(GQIS_ERR_INVALID, "warmup_steps must lie in [0, num_steps]");
    if ((GQ_OUT == GQIS_OUT_MEAN || GQ_OUT == GQIS_OUT_MEAN_STATE) && d->warmup_steps >= d->num_steps)
        return fail(GQIS_ERR_INVALID, "a mean output needs at least one step after warmup");
    if (!(d->dt > 0.0) || !(d->dt < 1e300)) return fail(GQIS_ERR_INVALID, "dt must be positive and finite");
    if (d->point_count == 0) return GQIS_OK;
    if (!d->par_x || !d->par_y || !d->results) return fail(GQIS_ERR_INVALID, "par_x, par_y and results are required");
    if (Model::kInitFromArray && !d->rho0) return fail(GQIS_ERR_INVALID, "this module reads rho0, which is NULL");
    if (GQ_TRACE != GQIS_TRACE_NONE) {
        if (!d->trace || d->num_trace < 0 || d->trace_stride < 1 || d->trace_offset < 0)
            return fail(GQIS_ERR_INVALID, "trace buffer/stride/offset invalid");
    }
#if GQ_ADAPTIVE
    if (!d->work_counter) return fail(GQIS_ERR_INVALID, "adaptive kernels need a zeroed work_counter");
    if (!(d->solver_params[0] >= 0.0) || !(d->solver_params[1] >= 0.0) ||
        !(d->solver_params[0] + d->solver_params[1] > 0.0) || !(d->solver_params[2] >= 1.0))
        return fail(GQIS_ERR_INVALID, "adaptive parameters rtol/atol/max_substeps invalid");
#endif
    return GQIS_OK;
}

#if GQ_ADAPTIVE
// The persistent work-stealing launch shared by gqis_sweep_launch and gqis_sweep_launch_noalloc:
// the grid is every resident CTA slot of the device, and lanes take point indices from the 32-bit
// counter d.work_counter. Its range bounds a launch to GQIS_NOALLOC_MAX_POINTS points (2^31 - 1):
// beyond that the counter would wrap and no lane would ever see the grid exhausted. The check
// comes before any CUDA call.
int launch_adaptive(const gqis_sweep_desc& d, cudaStream_t st) {
    if (d.point_count > GQIS_NOALLOC_MAX_POINTS)
        return fail(GQIS_ERR_TOO_LARGE, "adaptive launch: %lld points exceed the maximum of %lld per call",
                    (long long)d.point_count, (long long)GQIS_NOALLOC_MAX_POINTS);
    int dev = 0, sms = 0, ctas = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return cuda_fail(e, "cudaDeviceGetAttribute");
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas, kKernel, GQ_BLOCK, 0)) != cudaSuccess)
        return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (ctas < 1) ctas = 1;
    const int64_t needed = (d.point_count + GQ_BLOCK - 1) / GQ_BLOCK;
    int64_t grid = GQ_STATIC_SCHEDULE ? needed : (int64_t)sms * ctas;
    if (grid > needed) grid = needed;
    if (grid > 0x7fffffffLL) return fail(GQIS_ERR_TOO_LARGE, "too many points for one launch");
    kKernel<<<(unsigned)grid, GQ_BLOCK, 0, st>>>(d);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "adaptive sweep kernel launch");
    return GQIS_OK;
}
#endif

}  // namespace

extern "C" {

__attribute__((visibility("default"))) const char* gqis_last_error(void) { return g_last_error; }

__attribute__((visibility("default"))) int gqis_model_info_get(gqis_model_info* out) {
    if (!out) return fail(GQIS_ERR_INVALID, "info pointer is NULL");
    out->abi_version = GQIS_ABI_VERSION;
    out->state_size = Model::S;
    out->num_consts = Model::NCONST;
    out->form = Form::id;
    out->solver = GQ_SOLVER_ID;
    out->output_mode = GQ_OUT;
    out->trace_mode = GQ_TRACE;
    out->init_from_array = Model::kInitFromArray ? 1 : 0;
    out->block_threads = kBlock;
    out->model_hash = (uint64_t)GQ_MODEL_HASH;
    out->registers_per_thread = 0;
    out->sm_count = 0;
    out->ctas_per_sm = 0;
    cudaFuncAttributes attr;
    cudaError_t e = cudaFuncGetAttributes(&attr, kKernel);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncGetAttributes");
    out->registers_per_thread = attr.numRegs;
    int dev = 0, sms = 0, ctas = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return cuda_fail(e, "cudaDeviceGetAttribute");
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas, kKernel, kBlock, kSmem)) != cudaSuccess)
        return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    out->sm_count = sms;
    out->ctas_per_sm = ctas;
    return GQIS_OK;
}

__attribute__((visibility("default"))) int gqis_sweep_launch(const gqis_sweep_desc* d, void* stream) {
    int rc = check_desc(d);
    if (rc != GQIS_OK || d->point_count == 0) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
#if GQ_MATRIX
    cudaError_t e;
    if (kSmem > 48 * 1024 &&
        (e = cudaFuncSetAttribute(kKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem)) != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(max dynamic shared memory)");
    const int64_t grid = (d->point_count + kPointsPerCta - 1) / kPointsPerCta * kCluster;
    if (grid > 0x7fffffffLL) return fail(GQIS_ERR_TOO_LARGE, "too many points for one launch");
    if (kCluster > 1) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)grid, 1, 1);
        cfg.blockDim = dim3(kBlock, 1, 1);
        cfg.dynamicSmemBytes = kSmem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kCluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if ((e = cudaLaunchKernelEx(&cfg, kKernel, *d)) != cudaSuccess) return cuda_fail(e, "cluster launch");
    } else {
        kKernel<<<(unsigned)grid, kBlock, kSmem, st>>>(*d);
    }
#elif GQ_ADAPTIVE
    return launch_adaptive(*d, st);
#else
    const int64_t threads = GQ_PACK2 ? (d->point_count + 1) / 2 : d->point_count;  // packed: a pair per thread
    const int64_t grid = (threads + GQ_BLOCK - 1) / GQ_BLOCK;
    if (grid > 0x7fffffffLL) return fail(GQIS_ERR_TOO_LARGE, "too many points for one launch");
    kKernel<<<(unsigned)grid, GQ_BLOCK, 0, st>>>(*d);
#endif
#if GQ_MATRIX || !GQ_ADAPTIVE
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return cuda_fail(err, "sweep kernel launch");
    return GQIS_OK;
#endif
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Allocation-free launch (gqis_sweep_launch_noalloc): the adaptive kernels' work counter lives
// in this file-scope device array instead of caller-provided scratch. Host code only ever
// uses the array's device address, looked up once per device with cudaGetSymbolAddress.
// ---------------------------------------------------------------------------------------
static __device__ __align__(256) unsigned int g_noalloc_scratch[GQIS_NOALLOC_SCRATCH_BYTES / sizeof(unsigned int)];

namespace {
constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned int* g_noalloc_address[kNoallocMaxDevices] = {};

int noalloc_scratch_address(unsigned int** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kNoallocMaxDevices)
        return fail(GQIS_ERR_UNSUPPORTED, "device %d is beyond the %d devices the no-alloc launch tracks", dev,
                    kNoallocMaxDevices);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_address[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_address[dev] = static_cast<unsigned int*>(p);
    }
    *out = g_noalloc_address[dev];
    return GQIS_OK;
}
}  // namespace

extern "C" {

__attribute__((visibility("default"))) int gqis_sweep_launch_noalloc(const gqis_sweep_desc* d, void* stream) {
#if GQ_ADAPTIVE
    if (!d) return fail(GQIS_ERR_INVALID, "descriptor is NULL");
    if (d->point_count > GQIS_NOALLOC_MAX_POINTS)
        return fail(GQIS_ERR_TOO_LARGE, "no-alloc launch: %lld points exceed the maximum of %lld per call",
                    (long long)d->point_count, (long long)GQIS_NOALLOC_MAX_POINTS);
    unsigned int* counter = nullptr;
    int rc = noalloc_scratch_address(&counter);
    if (rc != GQIS_OK) return rc;
    gqis_sweep_desc local = *d;
    local.work_counter = counter;
    rc = check_desc(&local);
    if (rc != GQIS_OK || local.point_count == 0) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(no-alloc work counter)");
    return launch_adaptive(local, st);
#else
    return gqis_sweep_launch(d, stream);  // fixed-step kernels use no scratch
#endif
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Batch launch (gqis_sweep_launch_batch): several sweeps of this module in one grid.
// ---------------------------------------------------------------------------------------
#if !GQ_MATRIX
namespace {
#if GQ_ADAPTIVE
constexpr auto kBatchKernel = gqadaptive::sweep_adaptive_batch_kernel<GQ_SOLVER, Model, Form, GQ_OUT, GQ_TRACE>;
#elif GQ_PACK2
constexpr auto kBatchKernel = gqpacked::sweep_pair_batch_kernel<Model, GQ_OUT, GQ_TRACE>;
#else
constexpr auto kBatchKernel = gqfixed::sweep_fixed_batch_kernel<GQ_SOLVER, Model, Form, GQ_OUT, GQ_TRACE>;
#endif

// Global work units of one sweep in a batch: points (adaptive), or threads padded to whole warps
// (one point, or one pair of points for the packed kernel, per thread).
int64_t batch_units(const gqis_sweep_desc& d) {
#if GQ_ADAPTIVE
    return d.point_count;
#elif GQ_PACK2
    return ((d.point_count + 1) / 2 + 31) / 32 * 32;
#else
    return (d.point_count + 31) / 32 * 32;
#endif
}
}  // namespace
#endif

extern "C" {

__attribute__((visibility("default"))) int gqis_sweep_launch_batch(const gqis_sweep_desc* descs, int32_t count,
                                                                    uint32_t* work_counter, void* stream) {
#if GQ_MATRIX
    (void)descs;
    (void)count;
    (void)work_counter;
    (void)stream;
    return fail(GQIS_ERR_UNSUPPORTED, "the density-matrix kernels have no batch launch");
#else
    if (!descs || count < 1) return fail(GQIS_ERR_INVALID, "batch: descs is NULL or count < 1");
    if (count > GQIS_BATCH_MAX)
        return fail(GQIS_ERR_TOO_LARGE, "batch of %d sweeps exceeds the maximum of %d", count, GQIS_BATCH_MAX);
    static_assert(sizeof(BatchParams) <= 32000, "a batch must fit the kernel parameter space");
    BatchParams b;
    memset(&b, 0, sizeof(b));
    b.count = count;
    b.counter = work_counter;
    int64_t total = 0;
    for (int i = 0; i < count; ++i) {
        b.items[i] = descs[i];
#if GQ_ADAPTIVE
        b.items[i].work_counter = work_counter;  // the batch's one counter
#endif
        const int rc = check_desc(&b.items[i]);
        if (rc != GQIS_OK) {
            char why[sizeof(g_last_error)];
            snprintf(why, sizeof(why), "%s", g_last_error);
            return fail(rc, "batch item %d: %s", i, why);
        }
        b.starts[i] = total;
        total += batch_units(b.items[i]);
    }
    b.starts[count] = total;
    if (total == 0) return GQIS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int64_t grid = (total + GQ_BLOCK - 1) / GQ_BLOCK;
#if GQ_ADAPTIVE
    if (total > GQIS_NOALLOC_MAX_POINTS)
        return fail(GQIS_ERR_TOO_LARGE, "batch: %lld points exceed the maximum of %lld per launch", (long long)total,
                    (long long)GQIS_NOALLOC_MAX_POINTS);
    {
        int dev = 0, sms = 0, ctas = 0;
        cudaError_t e;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
            return cuda_fail(e, "cudaDeviceGetAttribute");
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas, kBatchKernel, GQ_BLOCK, 0)) != cudaSuccess)
            return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        const int64_t resident = (int64_t)sms * (ctas < 1 ? 1 : ctas);
        if (grid > resident) grid = resident;  // persistent: every resident CTA slot, lanes refill
    }
#endif
    if (grid > 0x7fffffffLL) return fail(GQIS_ERR_TOO_LARGE, "too many points for one launch");
    kBatchKernel<<<(unsigned)grid, GQ_BLOCK, 0, st>>>(b);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "batch sweep kernel launch");
    return GQIS_OK;
#endif
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Adjoint entry points (modules generated with an adjoint struct gqmodel::Adjoint).
// ---------------------------------------------------------------------------------------
extern "C" {

__attribute__((visibility("default"))) int gqis_adjoint_info(int32_t* num_params, int32_t* state_size) {
#if GQ_WITH_ADJOINT
    if (num_params) *num_params = gqmodel::Adjoint::P;
    if (state_size) *state_size = Model::S;
    return GQIS_OK;
#else
    (void)num_params;
    (void)state_size;
    return fail(GQIS_ERR_UNSUPPORTED, "this module was built without an adjoint");
#endif
}

__attribute__((visibility("default"))) int gqis_adjoint_scratch_bytes(int64_t point_count, int32_t num_steps,
                                                                       int32_t checkpoint_every, int64_t* bytes) {
    if (!bytes || point_count < 0 || num_steps < 1 || checkpoint_every < 1)
        return fail(GQIS_ERR_INVALID, "adjoint scratch: invalid sizes");
    const int64_t nck = (num_steps + checkpoint_every - 1) / checkpoint_every;
    *bytes = (nck + checkpoint_every) * (int64_t)Model::S * point_count * (int64_t)sizeof(double);
    return GQIS_OK;
}

__attribute__((visibility("default"))) int gqis_adjoint_launch(const gqis_adjoint_desc* a, void* stream) {
#if GQ_WITH_ADJOINT
    if (!a) return fail(GQIS_ERR_INVALID, "adjoint descriptor is NULL");
    if (Form::id != GQIS_FORM_FP64) return fail(GQIS_ERR_UNSUPPORTED, "the adjoint runs in the FP64 form");
    int rc = check_desc(&a->sweep);
    if (rc != GQIS_OK) return rc;
    if (!GQ_ADJOINT_FINAL && a->sweep.warmup_steps >= a->sweep.num_steps)
        return fail(GQIS_ERR_INVALID, "the adjoint differentiates a mean: needs steps after warmup");
    if (a->num_params != gqmodel::Adjoint::P)
        return fail(GQIS_ERR_INVALID, "num_params %d, module has %d", a->num_params, gqmodel::Adjoint::P);
    if (a->checkpoint_every < 1) return fail(GQIS_ERR_INVALID, "checkpoint_every must be positive");
    int64_t need = 0;
    rc = gqis_adjoint_scratch_bytes(a->sweep.point_count, a->sweep.num_steps, a->checkpoint_every, &need);
    if (rc != GQIS_OK) return rc;
    if (!a->scratch || a->scratch_bytes < need)
        return fail(GQIS_ERR_INVALID, "adjoint scratch of %lld bytes needed, %lld given", (long long)need,
                    (long long)a->scratch_bytes);
    if (gqmodel::Adjoint::P > 0 && !a->grad) return fail(GQIS_ERR_INVALID, "grad buffer is NULL");
    if (a->sweep.point_count == 0) return GQIS_OK;
    const int64_t grid = (a->sweep.point_count + GQ_BLOCK - 1) / GQ_BLOCK;
    gqadjoint::adjoint_rk4_kernel<Model, gqmodel::Adjoint, GQ_ADJOINT_FINAL>
        <<<(unsigned)grid, GQ_BLOCK, 0, static_cast<cudaStream_t>(stream)>>>(*a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "adjoint kernel launch");
    return GQIS_OK;
#else
    (void)a;
    (void)stream;
    return fail(GQIS_ERR_UNSUPPORTED, "this module was built without an adjoint");
#endif
}

}  // extern "C"
