// C ABI entry points (include/ehgp.h): context lifetime, argument checks,
// device error word -> status code, poisoning, timing.
#include "ehgp_internal.cuh"

#include <cstdio>
#include <cstring>
#include <new>

using ehgp::Ctx;

namespace ehgp {

cudaError_t ctx_alloc(Ctx& ctx, void** ptr, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(ptr, bytes);
  if (e == cudaSuccess) {
    ctx.allocations.push_back(*ptr);
    ctx.device_bytes += bytes;
  }
  return e;
}

void ctx_free(Ctx& ctx, void* ptr, size_t bytes) {
  if (!ptr) return;
  for (size_t i = 0; i < ctx.allocations.size(); ++i)
    if (ctx.allocations[i] == ptr) {
      ctx.allocations[i] = ctx.allocations.back();
      ctx.allocations.pop_back();
      cudaFree(ptr);
      ctx.device_bytes -= bytes ? bytes : 16;
      return;
    }
}

}  // namespace ehgp

namespace {

int fail(Ctx* ctx, int status, const char* msg);
int cuda_fail(Ctx* ctx, cudaError_t e, const char* where);
int device_status(Ctx* ctx, uint32_t err);

}  // namespace

namespace ehgp {
int abi_fail(Ctx* ctx, int status, const char* msg) { return fail(ctx, status, msg); }
int abi_cuda_fail(Ctx* ctx, cudaError_t e, const char* where) { return cuda_fail(ctx, e, where); }
int abi_device_status(Ctx* ctx, uint32_t err) { return device_status(ctx, err); }
}  // namespace ehgp

namespace {

int fail(Ctx* ctx, int status, const char* msg) {
  if (ctx) ctx->last_error = msg;
  return status;
}

int cuda_fail(Ctx* ctx, cudaError_t e, const char* where) {
  if (ctx) {
    ctx->poisoned = true;
    ctx->last_error = std::string(where) + ": " + cudaGetErrorString(e);
  }
  return EHGP_ERR_CUDA;
}

// Maps the device error word to a status code (most specific first).
int device_status(Ctx* ctx, uint32_t err) {
  if (err == 0) return EHGP_OK;
  if (err & ehgp::kErrNonFinite) return fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "binary64 coordinates must be finite");
  if (err & ehgp::kErrDuplicate)
    return fail(ctx, EHGP_ERR_DUPLICATE_POINT, "a canonical point cloud cannot contain duplicate geometric points");
  if (err & ehgp::kErrNumericRange)
    return fail(ctx, EHGP_ERR_NUMERIC_RANGE, "an exact evaluation left the supported binary64 range");
  if (err & ehgp::kErrTimeout) return fail(ctx, EHGP_ERR_TIMEOUT, "a bounded device wait ran out");
  if (err & ehgp::kErrCapacity) return fail(ctx, EHGP_ERR_CAPACITY, "a device buffer capacity was exceeded");
  return fail(ctx, EHGP_ERR_CUDA, "internal consistency check failed on the device");
}

// Shared body of the three LBVH build entry points.  `src` is a host or
// device pointer according to `where` (0 host f64, 1 host f32, 2 device f64).
int lbvh_build_common(Ctx* ctx, const void* src, uint64_t n, const ehgp_lbvh_out* out, int where) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->last_error.clear();
  if (ctx->poisoned) return fail(ctx, EHGP_ERR_POISONED, "the context is poisoned by an earlier CUDA failure");
  if (!src || !out) return fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "null input or output descriptor");
  if (n == 0) return fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "a canonical point cloud cannot be empty");
  if (n > ctx->max_points) return fail(ctx, EHGP_ERR_CAPACITY, "the point count exceeds the context capacity");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  ehgp::LbvhBuffers& b = ctx->lb;
  const uint32_t n32 = (uint32_t)n;
  ctx->built_n = 0;
  ctx->geom_ready = false;
  ctx->emst_ready = false;
  ctx->pb.witness_ready = false;
  ctx->pb.resident = false;
  ctx->pb.K = 0;  // supports are resident for one cloud and one K
  ctx->hb.K = 0;
  if (where == 0) {
    e = cudaMemcpyAsync(b.xyz_in, src, 3 * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  } else if (where == 1) {
    e = cudaMemcpyAsync(b.xyz_in_f32, src, 3 * n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
  } else {
    e = cudaMemcpyAsync(b.xyz_in, src, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "input copy");
  if ((e = cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream)) != cudaSuccess)
    return cuda_fail(ctx, e, "cudaMemsetAsync");
  cudaEventRecord(ctx->ev0, ctx->stream);
  ctx->last_launches = ehgp::lbvh_enqueue(*ctx, n32, where == 1 ? 1 : 0);
  cudaEventRecord(ctx->ev1, ctx->stream);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "LBVH kernel launch");
  cudaMemcpyAsync(ctx->h_status, ctx->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(ctx->h_status + 1, b.stats, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream);
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "LBVH build");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_ms = ms;
  const int st = device_status(ctx, ctx->h_status[0]);
  if (st != EHGP_OK) return st;
  if ((e = ehgp::lbvh_export(*ctx, n32, out)) != cudaSuccess) return cuda_fail(ctx, e, "LBVH export");
  ctx->built_n = n;
  return EHGP_OK;
}

}  // namespace

extern "C" {

int ehgp_ctx_create(int device, const ehgp_limits* limits, ehgp_ctx** out_ctx) {
  if (!limits || !out_ctx || limits->max_points == 0 || limits->max_points > 0x7fffffffull)
    return EHGP_ERR_INVALID_ARGUMENT;
  *out_ctx = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return EHGP_ERR_INVALID_ARGUMENT;
  ehgp_ctx* ctx = new (std::nothrow) ehgp_ctx();
  if (!ctx) return EHGP_ERR_OUT_OF_MEMORY;
  ctx->device = device;
  ctx->max_points = limits->max_points;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->evk0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->evk1);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->evs0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->evs1);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&ctx->h_status, 64 * sizeof(uint32_t));
  if (e == cudaSuccess) e = ehgp::ctx_alloc(*ctx, (void**)&ctx->d_err, sizeof(uint32_t));
  if (e == cudaSuccess) {
    // admission: the context's resident buffers must fit the HBM fraction
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const double frac = (limits->hbm_fraction > 0.0 && limits->hbm_fraction <= 1.0) ? limits->hbm_fraction : 0.8;
    const double estimate = 900.0 * (double)limits->max_points;  // bytes per point of the resident stages
    if (estimate > frac * (double)total_b || estimate > (double)free_b) e = cudaErrorMemoryAllocation;
  }
  if (e == cudaSuccess) e = ehgp::lbvh_alloc(*ctx);
  if (e == cudaSuccess) e = ehgp::geom_alloc(*ctx);
  if (e == cudaSuccess) e = ehgp::pairs_alloc(*ctx);
  if (e == cudaSuccess) e = ehgp::higher_alloc(*ctx);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    const int st = (e == cudaErrorMemoryAllocation) ? EHGP_ERR_OUT_OF_MEMORY : EHGP_ERR_CUDA;
    cudaGetLastError();
    ehgp_ctx_destroy(ctx);
    return st;
  }
  *out_ctx = ctx;
  return EHGP_OK;
}

int ehgp_ctx_destroy(ehgp_ctx* ctx) {
  if (!ctx) return EHGP_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ehgp::hier_free(*ctx);
  for (void* p : ctx->allocations) cudaFree(p);
  if (ctx->h_status) cudaFreeHost(ctx->h_status);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  for (cudaEvent_t ev : {ctx->evk0, ctx->evk1, ctx->evs0, ctx->evs1})
    if (ev) cudaEventDestroy(ev);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return EHGP_OK;
}

const char* ehgp_last_error(const ehgp_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

const char* ehgp_status_string(int status) {
  switch (status) {
    case EHGP_OK: return "EHGP_OK";
    case EHGP_ERR_INVALID_ARGUMENT: return "EHGP_ERR_INVALID_ARGUMENT";
    case EHGP_ERR_DUPLICATE_POINT: return "EHGP_ERR_DUPLICATE_POINT";
    case EHGP_ERR_CAPACITY: return "EHGP_ERR_CAPACITY";
    case EHGP_ERR_OUT_OF_MEMORY: return "EHGP_ERR_OUT_OF_MEMORY";
    case EHGP_ERR_TIMEOUT: return "EHGP_ERR_TIMEOUT";
    case EHGP_ERR_DEGENERATE: return "EHGP_ERR_DEGENERATE";
    case EHGP_ERR_NUMERIC_RANGE: return "EHGP_ERR_NUMERIC_RANGE";
    case EHGP_ERR_CUDA: return "EHGP_ERR_CUDA";
    case EHGP_ERR_POISONED: return "EHGP_ERR_POISONED";
    case EHGP_ERR_NOT_BUILT: return "EHGP_ERR_NOT_BUILT";
    default: return "EHGP_ERR_UNKNOWN";
  }
}

uint64_t ehgp_ctx_device_bytes(const ehgp_ctx* ctx) { return ctx ? ctx->device_bytes : 0; }

int ehgp_ctx_reserve(ehgp_ctx* ctx, uint32_t stage, uint64_t records) {
  if (!ctx || stage > 1 || records == 0 || records >= 0xffff0000ull) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->last_error.clear();
  if (ctx->poisoned) return fail(ctx, EHGP_ERR_POISONED, "the context is poisoned by an earlier CUDA failure");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamSynchronize");
  // the resident records (if any) are dropped with the buffers
  if (stage == 0) {
    ctx->pb.K = 0;
    ctx->pb.count = 0;
    ctx->pb.witness_ready = false;
    ctx->pb.resident = false;
    e = ehgp::pairs_records_alloc(*ctx, records);
  } else {
    ctx->hb.K = 0;
    ctx->hb.count = 0;
    e = ehgp::higher_records_alloc(*ctx, records);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, EHGP_ERR_OUT_OF_MEMORY, "the reserved record buffers do not fit the device");
  }
  return EHGP_OK;
}

uint64_t ehgp_ctx_regrowths(const ehgp_ctx* ctx) { return ctx ? ctx->regrowths : 0; }

int ehgp_ctx_counters(const ehgp_ctx* ctx, uint64_t* out, uint32_t count) {
  if (!ctx || !out) return EHGP_ERR_INVALID_ARGUMENT;
  const uint64_t v[4] = {ctx->device_bytes, ctx->regrowths, ctx->pair_runs, ctx->higher_runs};
  for (uint32_t i = 0; i < count && i < 4; ++i) out[i] = v[i];
  return EHGP_OK;
}

int ehgp_tune(ehgp_ctx* ctx, uint32_t knob, uint64_t value) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  switch (knob) {
    case EHGP_TUNE_HIGHER_LIST:
      if (value < 1 || value > 1024) return fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "list capacity must be in [1, 1024]");
      ctx->hb.list_cap = (uint32_t)value;
      return EHGP_OK;
    default:
      return fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "unknown tuning knob");
  }
}

int ehgp_lbvh_build(ehgp_ctx* ctx, const double* xyz, uint64_t n, const ehgp_lbvh_out* out) {
  return lbvh_build_common(ctx, xyz, n, out, 0);
}
int ehgp_lbvh_build_f32(ehgp_ctx* ctx, const float* xyz, uint64_t n, const ehgp_lbvh_out* out) {
  return lbvh_build_common(ctx, xyz, n, out, 1);
}
int ehgp_lbvh_build_device(ehgp_ctx* ctx, const double* d_xyz, uint64_t n, const ehgp_lbvh_out* out) {
  return lbvh_build_common(ctx, d_xyz, n, out, 2);
}

int ehgp_step_begin(ehgp_ctx* ctx) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  return cudaEventRecord(ctx->evs0, ctx->stream) == cudaSuccess ? EHGP_OK : EHGP_ERR_CUDA;
}

int ehgp_step_end(ehgp_ctx* ctx, double* elapsed_ms) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (cudaEventRecord(ctx->evs1, ctx->stream) != cudaSuccess || cudaEventSynchronize(ctx->evs1) != cudaSuccess)
    return EHGP_ERR_CUDA;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ctx->evs0, ctx->evs1) != cudaSuccess) return EHGP_ERR_CUDA;
  if (elapsed_ms) *elapsed_ms = ms;
  return EHGP_OK;
}

int ehgp_kernel_stats(const ehgp_ctx* ctx, double* kernel_ms, uint64_t* stats, uint32_t count) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  if (kernel_ms) *kernel_ms = ctx->kernel_ms;
  for (uint32_t i = 0; stats && i < count && i < 8; ++i) stats[i] = ctx->kernel_stats[i];
  return EHGP_OK;
}

int ehgp_last_timing(const ehgp_ctx* ctx, double* device_ms, uint64_t* kernel_launches) {
  if (!ctx) return EHGP_ERR_INVALID_ARGUMENT;
  if (device_ms) *device_ms = ctx->last_ms;
  if (kernel_launches) *kernel_launches = ctx->last_launches;
  return EHGP_OK;
}

}  // extern "C"
