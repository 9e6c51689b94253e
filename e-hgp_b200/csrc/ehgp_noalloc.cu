// Allocation-free variant of the LBVH build (ehgp_lbvh_build_noalloc).
//
// Who needs it: callers that may not call cudaMalloc at all.  Examples are a
// host process whose framework owns every byte of device memory through its
// own pool and refuses allocations outside it, and a latency-critical caller
// for which cudaMalloc is off limits because it can synchronise the whole
// device.  Such a caller cannot create an ehgp context, since
// ehgp_ctx_create allocates the context's buffers.
//
// What it does: the same device pipeline as ehgp_lbvh_build, with every byte
// of scratch taken from one file-scope __device__ array of fixed size,
// sized for kNoAllocMaxPoints points.  The array exists on every GPU that
// loads this library and is held until the process exits.  Nothing here calls
// cudaMalloc, cudaMallocHost, cudaFree or an allocating library routine.
//
// Set-up: the first call on a device (with that device current) looks up the
// device address of the array with cudaGetSymbolAddress and caches it for
// that device.
//
// Streams: every call copies its status words back and synchronises its
// stream, which a capturing stream does not allow, so the entry point must
// never be called on a stream that is being captured into a CUDA graph; it
// checks cudaStreamIsCapturing and refuses such a stream with
// EHGP_ERR_INVALID_ARGUMENT.
//
// Sharing: every call on a device uses the same array and it keeps the last
// call's contents; everything that must start at zero is cleared by each
// call.  Calls are serialised by a process-wide mutex, but calls whose GPU
// work overlaps (for example from two processes sharing a GPU) race on the
// array and must not be issued.
#include "ehgp_internal.cuh"

#include <cstring>
#include <mutex>

namespace {

constexpr uint64_t kNoAllocMaxPoints = 16384;

// Byte layout of the scratch array for kNoAllocMaxPoints points; every block
// starts on a 256-byte boundary.
struct NoAllocLayout {
  uint64_t off = 0;
  __host__ __device__ constexpr uint64_t take(uint64_t bytes) {
    const uint64_t at = off;
    off += (bytes + 255) / 256 * 256;
    return at;
  }
};

constexpr uint64_t scratch_bytes() {
  const uint64_t n = kNoAllocMaxPoints;
  NoAllocLayout L;
  L.take(3 * n * 8);            // xyz_in
  L.take(3 * n * 8);            // cin
  L.take(n * 8); L.take(n * 8); L.take(n * 8);  // px py pz
  L.take(n * 4);                // source_index
  L.take(n * 8);                // code
  L.take(n * 4); L.take(n * 4); // vals0 vals1
  L.take(n * 4);                // leaf_pid
  L.take(n * 8);                // leaf_code
  L.take(n * 4);                // group_of
  L.take(ehgp::lbvh_scan_block_sums(n) * 4);  // block_sums
  L.take((n + 1) * 4);          // gstart
  L.take(n * 8);                // gcode
  for (int i = 0; i < 6; ++i) L.take(n * 4);   // top_left/right, parents, grp_root_idx, grp_depth
  L.take(3 * n * 4);            // top split/gmin/gmax
  for (int i = 0; i < 5; ++i) L.take(2 * n * 4);  // n_left/right/begin/end/parent
  L.take(3 * 2 * n * 4); L.take(3 * 2 * n * 4);   // n_lo n_hi
  L.take(2 * n * 4);            // n_flag
  L.take(12 * 8);               // frame
  L.take(12 * ehgp::kLbvhFrameBlocks * 8);  // frame_partial
  L.take(4);                    // frame_done
  L.take(8 * 4);                // stats
  L.take(2 * n * sizeof(ehgp_lbvh_node) + n * sizeof(ehgp_lbvh_leaf) + n * 8);  // export
  L.take(256ull * ((n + ehgp::kRadixTile - 1) / ehgp::kRadixTile) * 4);         // radix counts
  L.take(ehgp::kRadixStateWords * 4);  // radix state
  L.take(4);                    // error word
  return L.off;
}

constexpr uint64_t kScratchBytes = scratch_bytes();
static_assert(kScratchBytes <= (uint64_t{8} << 20), "the fixed scratch array stays below 8 MiB per GPU");

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Points the context's buffers into the scratch array (same order as
// scratch_bytes()).
void carve(ehgp::Ctx& c, unsigned char* base) {
  const uint64_t n = kNoAllocMaxPoints;
  NoAllocLayout L;
  auto at = [&](uint64_t bytes) { return (void*)(base + L.take(bytes)); };
  ehgp::LbvhBuffers& b = c.lb;
  b.xyz_in = (double*)at(3 * n * 8);
  b.xyz_in_f32 = nullptr;
  b.cin = (uint64_t*)at(3 * n * 8);
  b.px = (double*)at(n * 8);
  b.py = (double*)at(n * 8);
  b.pz = (double*)at(n * 8);
  b.source_index = (uint32_t*)at(n * 4);
  b.code = (uint64_t*)at(n * 8);
  b.vals0 = (uint32_t*)at(n * 4);
  b.vals1 = (uint32_t*)at(n * 4);
  b.leaf_pid = (uint32_t*)at(n * 4);
  b.leaf_code = (uint64_t*)at(n * 8);
  b.group_of = (uint32_t*)at(n * 4);
  b.block_sums = (uint32_t*)at(ehgp::lbvh_scan_block_sums(n) * 4);
  b.gstart = (uint32_t*)at((n + 1) * 4);
  b.gcode = (uint64_t*)at(n * 8);
  b.top_left = (uint32_t*)at(n * 4);
  b.top_right = (uint32_t*)at(n * 4);
  b.top_parent_int = (uint32_t*)at(n * 4);
  b.top_parent_grp = (uint32_t*)at(n * 4);
  b.grp_root_idx = (uint32_t*)at(n * 4);
  b.grp_depth = (uint32_t*)at(n * 4);
  uint32_t* topx = (uint32_t*)at(3 * n * 4);
  c.lb_top_split = topx;
  c.lb_top_gmin = topx + n;
  c.lb_top_gmax = topx + 2 * n;
  b.n_left = (uint32_t*)at(2 * n * 4);
  b.n_right = (uint32_t*)at(2 * n * 4);
  b.n_begin = (uint32_t*)at(2 * n * 4);
  b.n_end = (uint32_t*)at(2 * n * 4);
  b.n_parent = (uint32_t*)at(2 * n * 4);
  b.n_lo = (uint32_t*)at(3 * 2 * n * 4);
  b.n_hi = (uint32_t*)at(3 * 2 * n * 4);
  b.n_flag = (uint32_t*)at(2 * n * 4);
  b.frame = (uint64_t*)at(12 * 8);
  b.frame_partial = (unsigned long long*)at(12 * ehgp::kLbvhFrameBlocks * 8);
  b.frame_done = (uint32_t*)at(4);
  b.stats = (uint32_t*)at(8 * 4);
  b.export_bytes = 2 * n * sizeof(ehgp_lbvh_node) + n * sizeof(ehgp_lbvh_leaf) + n * 8;
  b.export_buf = at(b.export_bytes);
  c.radix.max_tiles = (uint32_t)((n + ehgp::kRadixTile - 1) / ehgp::kRadixTile);
  c.radix.counts = (uint32_t*)at(256ull * c.radix.max_tiles * 4);
  c.radix.state = (uint32_t*)at(ehgp::kRadixStateWords * 4);
  c.d_err = (uint32_t*)at(4);
  c.max_points = n;
  // the carve takes exactly the blocks that scratch_bytes() sized
  if (L.off != kScratchBytes) c.max_points = 0;
}

}  // namespace

extern "C" {

uint64_t ehgp_lbvh_noalloc_max_points(void) { return kNoAllocMaxPoints; }

uint64_t ehgp_lbvh_noalloc_scratch_bytes(void) { return kScratchBytes; }

int ehgp_lbvh_build_noalloc(const double* xyz, uint64_t n, const ehgp_lbvh_out* out, void* stream) {
  if (!xyz || !out) return EHGP_ERR_INVALID_ARGUMENT;
  if (n == 0) return EHGP_ERR_INVALID_ARGUMENT;
  if (n > kNoAllocMaxPoints) return EHGP_ERR_CAPACITY;
  {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing((cudaStream_t)stream, &cap) != cudaSuccess) return EHGP_ERR_CUDA;
    if (cap != cudaStreamCaptureStatusNone) return EHGP_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return EHGP_ERR_CUDA;
  if (!g_scratch_addr[device]) {
    void* addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess || addr == nullptr) return EHGP_ERR_CUDA;
    g_scratch_addr[device] = (unsigned char*)addr;
  }
  // A stack context: pointers only, no device or pinned allocation.
  ehgp::Ctx c;
  c.device = device;
  c.stream = (cudaStream_t)stream;
  carve(c, g_scratch_addr[device]);
  if (c.max_points != kNoAllocMaxPoints) return EHGP_ERR_CUDA;  // layout and carve disagree
  uint32_t status[64] = {0};  // pageable host words: a copy into them allocates nothing
  c.h_status = status;
  const uint32_t n32 = (uint32_t)n;
  cudaError_t e = cudaMemcpyAsync(c.lb.xyz_in, xyz, 3 * n * sizeof(double), cudaMemcpyHostToDevice, c.stream);
  // clear what must start at zero: the error word and the frame's arrival counter
  if (e == cudaSuccess) e = cudaMemsetAsync(c.d_err, 0, sizeof(uint32_t), c.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.lb.frame_done, 0, sizeof(uint32_t), c.stream);
  if (e != cudaSuccess) return EHGP_ERR_CUDA;
  ehgp::lbvh_enqueue(c, n32, 0);
  if (cudaGetLastError() != cudaSuccess) return EHGP_ERR_CUDA;
  if (cudaMemcpyAsync(status, c.d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
      cudaMemcpyAsync(status + 1, c.lb.stats, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(c.stream) != cudaSuccess)
    return EHGP_ERR_CUDA;
  // same mapping of the device error word as the context path
  if (status[0]) return ehgp::abi_device_status(nullptr, status[0]);
  if (ehgp::lbvh_export(c, n32, out) != cudaSuccess) return EHGP_ERR_CUDA;
  return EHGP_OK;
}

}  // extern "C"
