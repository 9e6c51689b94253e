// Checkpoint and resume of a request after its support stages.
//
// The reference streams its supports in transactional chunks (chunk -> checkpoint ->
// commit, morsehgp3d/include/morsehgp3d/hierarchy/pair_support_stream.hpp:421-470) and plans a
// preemption manifest for long runs (morsehgp3d/docs/GPU_G4_ARCHITECTURE.md:239-252).  Here the
// unit of work that is worth keeping is the support catalogue: a checkpoint holds the canonical
// cloud (binary64 coordinates in PointId order), K and the pair and triple/quad records, so
// that a request preempted after its supports resumes with the hierarchy alone.
//
// File: a 64-byte header (magic "EHGPCKP1", format version, point count, K, the two record
// counts, payload bytes, FNV-1a 64 of the payload), then the payload: x, y, z of the points,
// the pair records (64 B each), the triple/quad records (64 B each).  A load checks the magic,
// the version, the sizes against the file and the checksum before touching the context.
#include "ehgp_internal.cuh"

#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

namespace {

constexpr char kMagic[8] = {'E', 'H', 'G', 'P', 'C', 'K', 'P', '1'};
constexpr uint32_t kVersion = 1;

struct Header {
  char magic[8];
  uint32_t version, K;
  uint64_t n, pairs, higher, payload_bytes, checksum;
  uint64_t reserved[1];
};
static_assert(sizeof(Header) == 64, "checkpoint header is 64 bytes");

uint64_t fnv1a(const unsigned char* p, uint64_t len, uint64_t h = 1469598103934665603ull) {
  for (uint64_t i = 0; i < len; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

struct FileCloser {
  void operator()(FILE* f) const {
    if (f) std::fclose(f);
  }
};

}  // namespace

extern "C" {

int ehgp_checkpoint_save(ehgp_ctx* ctx, uint32_t K, const char* path) {
  if (!ctx || !path || K == 0 || K > 10) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mutex);
  ctx->last_error.clear();
  if (ctx->poisoned) return ehgp::abi_fail(ctx, EHGP_ERR_POISONED, "the context is poisoned by an earlier CUDA failure");
  if (ctx->built_n == 0) return ehgp::abi_fail(ctx, EHGP_ERR_NOT_BUILT, "ehgp_checkpoint_save needs a resident cloud");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "cudaSetDevice");
  if (!ctx->geom_ready) {
    ehgp::geom_prepare(*ctx, (uint32_t)ctx->built_n);
    if ((e = cudaGetLastError()) != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "traversal preparation");
  }
  if (!ctx->scale_valid)
    return ehgp::abi_fail(ctx, EHGP_ERR_NUMERIC_RANGE, "the cloud exceeds the exact fixed-point range");
  cudaMemsetAsync(ctx->d_err, 0, sizeof(uint32_t), ctx->stream);
  uint32_t m = 0;
  int s = EHGP_OK;
  if (!(ctx->pb.K == K && ctx->pb.resident) && (s = ehgp::pairs_run(*ctx, K, &m)) != EHGP_OK) return s;
  if (ctx->hb.K != K && (s = ehgp::higher_run(*ctx, K, &m)) != EHGP_OK) return s;
  const uint64_t n = ctx->built_n, np = ctx->pb.count, nh = ctx->hb.count;
  const uint64_t bytes = 3 * n * 8 + (np + nh) * 64;
  std::vector<unsigned char> payload(bytes);
  unsigned char* q = payload.data();
  if ((e = cudaMemcpy(q, ctx->lb.px, n * 8, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(q + n * 8, ctx->lb.py, n * 8, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(q + 2 * n * 8, ctx->lb.pz, n * 8, cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (np && (e = cudaMemcpy(q + 3 * n * 8, ctx->pb.sorted, np * 64, cudaMemcpyDeviceToHost)) != cudaSuccess) ||
      (nh && (e = cudaMemcpy(q + 3 * n * 8 + np * 64, ctx->hb.sorted, nh * 64, cudaMemcpyDeviceToHost)) != cudaSuccess))
    return ehgp::abi_cuda_fail(ctx, e, "checkpoint copy");
  Header h{};
  std::memcpy(h.magic, kMagic, 8);
  h.version = kVersion;
  h.K = K;
  h.n = n;
  h.pairs = np;
  h.higher = nh;
  h.payload_bytes = bytes;
  h.checksum = fnv1a(payload.data(), bytes);
  std::unique_ptr<FILE, FileCloser> f(std::fopen(path, "wb"));
  if (!f) return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "the checkpoint file cannot be created");
  if (std::fwrite(&h, sizeof h, 1, f.get()) != 1 || std::fwrite(payload.data(), 1, bytes, f.get()) != bytes)
    return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "the checkpoint file cannot be written");
  if (std::fflush(f.get()) != 0) return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "the checkpoint file cannot be written");
  return EHGP_OK;
}

int ehgp_checkpoint_load(ehgp_ctx* ctx, const char* path, uint32_t* K_out) {
  if (!ctx || !path) return EHGP_ERR_INVALID_ARGUMENT;
  Header h{};
  std::vector<unsigned char> payload;
  {
    std::unique_ptr<FILE, FileCloser> f(std::fopen(path, "rb"));
    if (!f) return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "the checkpoint file cannot be opened");
    if (std::fread(&h, sizeof h, 1, f.get()) != 1 || std::memcmp(h.magic, kMagic, 8) != 0 || h.version != kVersion)
      return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "not a checkpoint of this format");
    if (h.K == 0 || h.K > 10 || h.n == 0 || h.n > ctx->max_points || h.pairs > 0xffff0000ull ||
        h.higher > 0xffff0000ull || h.payload_bytes != 3 * h.n * 8 + (h.pairs + h.higher) * 64)
      return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "the checkpoint header is inconsistent");
    payload.resize(h.payload_bytes);
    if (std::fread(payload.data(), 1, h.payload_bytes, f.get()) != h.payload_bytes || std::fgetc(f.get()) != EOF)
      return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "the checkpoint file is truncated or too long");
  }
  if (fnv1a(payload.data(), h.payload_bytes) != h.checksum)
    return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "the checkpoint payload fails its checksum");
  // the cloud again (canonical order in, so PointIds are the saved ones), then the records
  const uint64_t n = h.n;
  std::vector<double> xyz(3 * n);
  const double* px = reinterpret_cast<const double*>(payload.data());
  for (uint64_t i = 0; i < n; ++i) {
    xyz[3 * i] = px[i];
    xyz[3 * i + 1] = px[n + i];
    xyz[3 * i + 2] = px[2 * n + i];
  }
  ehgp_lbvh_out none{};
  std::vector<uint64_t> src(n);
  none.source_index = src.data();
  int s = ehgp_lbvh_build(ctx, xyz.data(), n, &none);
  if (s != EHGP_OK) return s;
  for (uint64_t i = 0; i < n; ++i)
    if (src[i] != i) return ehgp::abi_fail(ctx, EHGP_ERR_INVALID_ARGUMENT, "the checkpoint cloud is not canonical");
  std::lock_guard<std::mutex> lock(ctx->mutex);
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "cudaSetDevice");
  if (!ctx->geom_ready) {
    ehgp::geom_prepare(*ctx, (uint32_t)n);
    if ((e = cudaGetLastError()) != cudaSuccess) return ehgp::abi_cuda_fail(ctx, e, "traversal preparation");
  }
  if (h.pairs > ctx->pb.capacity && (e = ehgp::pairs_records_alloc(*ctx, ehgp::grown_capacity(h.pairs))) != cudaSuccess)
    return ehgp::abi_fail(ctx, EHGP_ERR_OUT_OF_MEMORY, "the checkpoint's pair records do not fit the device");
  if (h.higher > ctx->hb.capacity &&
      (e = ehgp::higher_records_alloc(*ctx, ehgp::grown_capacity(h.higher))) != cudaSuccess)
    return ehgp::abi_fail(ctx, EHGP_ERR_OUT_OF_MEMORY, "the checkpoint's higher records do not fit the device");
  const unsigned char* rec = payload.data() + 3 * n * 8;
  if ((h.pairs && (e = cudaMemcpy(ctx->pb.sorted, rec, h.pairs * 64, cudaMemcpyHostToDevice)) != cudaSuccess) ||
      (h.higher && (e = cudaMemcpy(ctx->hb.sorted, rec + h.pairs * 64, h.higher * 64, cudaMemcpyHostToDevice)) !=
                       cudaSuccess))
    return ehgp::abi_cuda_fail(ctx, e, "checkpoint records");
  ctx->pb.count = (uint32_t)h.pairs;
  ctx->pb.K = h.K;
  ctx->pb.resident = true;     // the hierarchy reads these records
  ctx->pb.witness_ready = false;  // the witness lists are not kept (a new triple/quad run redoes them)
  ctx->hb.count = (uint32_t)h.higher;
  ctx->hb.K = h.K;
  if (K_out) *K_out = h.K;
  return EHGP_OK;
}

}  // extern "C"
