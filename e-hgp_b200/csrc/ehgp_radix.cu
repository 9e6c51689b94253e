// Stable LSD radix sort of 32-bit indices by indirect 64-bit keys (sm_100a).
//
// Used twice on the LBVH path:
//  * the canonical PointId order: lexicographic (x, y, z) binary64 total-order
//    keys, i.e. the std::sort of src/cpu/spatial/point_cloud.cpp:58-62;
//  * the Morton leaf order: (code, PointId), i.e. std::sort with
//    morton_leaf_less (src/cpu/spatial/lbvh.cpp:93-100,512) -- stability of
//    the LSD passes over an input in PointId order gives the PointId tie-break.
//
// Each 8-bit pass is four kernels: a per-tile histogram (upsweep), a row scan
// of the histogram (one block per digit), a digit-base scan that also detects a
// pass in which every key has the same digit, and a stable scatter (downsweep).  Trivial passes are skipped on the
// device (the scatter returns at once and the ping-pong buffer is not
// flipped), so the host never synchronises inside a sort and the whole
// sequence can be captured in a CUDA graph.
#include "ehgp_internal.cuh"

namespace ehgp {
namespace {

__device__ __forceinline__ uint32_t digit_of(const IndirectKey& k, uint32_t v, int shift) {
  uint64_t w = __ldg(k.words + v);
  if (k.order) w = order_key(w);
  return (uint32_t)(w >> shift) & 0xffu;
}

__global__ void __launch_bounds__(kRadixThreads)
k_radix_upsweep(uint32_t n, const uint32_t* __restrict__ vals0, const uint32_t* __restrict__ vals1,
                IndirectKey key, int shift, const uint32_t* __restrict__ state, int pass,
                uint32_t* __restrict__ counts, uint32_t tiles) {
  __shared__ uint32_t hist[256];
  const uint32_t tile = blockIdx.x;
  hist[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t* in = state[2 * pass] ? vals1 : vals0;
  const uint32_t base = tile * kRadixTile;
#pragma unroll
  for (int r = 0; r < kRadixItems; ++r) {
    const uint32_t i = base + r * kRadixThreads + threadIdx.x;
    if (i < n) atomicAdd(&hist[digit_of(key, in[i], shift)], 1u);
  }
  __syncthreads();
  counts[threadIdx.x * tiles + tile] = hist[threadIdx.x];
}

// Row scan: block d turns row d of the tile histogram (counts[d * tiles ..]) into
// exclusive offsets within the digit and stores the digit total (coalesced, one
// block per digit).
__global__ void __launch_bounds__(256)
k_radix_rowscan(uint32_t* __restrict__ counts, uint32_t tiles, uint32_t* __restrict__ state) {
  __shared__ uint32_t warp_tot[8];
  __shared__ uint32_t carry;
  const uint32_t d = blockIdx.x, tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  uint32_t* row = counts + (uint64_t)d * tiles;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < tiles; base += 256) {
    const uint32_t t = base + tid;
    const uint32_t v = t < tiles ? row[t] : 0u;
    uint32_t x = v;  // inclusive warp scan
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
      if ((int)lane >= off) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    uint32_t wbase = 0;
    for (uint32_t w = 0; w < warp; ++w) wbase += warp_tot[w];
    const uint32_t c0 = carry;
    if (t < tiles) row[t] = c0 + wbase + x - v;
    __syncthreads();
    if (tid == 255) carry = c0 + wbase + x;
    __syncthreads();
  }
  if (tid == 0) state[2 * (kRadixMaxPasses + 1) + d] = carry;
}

// Digit bases: exclusive scan of the 256 digit totals; a pass whose keys share one
// digit is marked trivial (its scatter is skipped and the buffers do not flip).
__global__ void __launch_bounds__(256)
k_radix_digits(uint32_t n, uint32_t* __restrict__ state, int pass) {
  __shared__ uint32_t totals[256];
  __shared__ uint32_t trivial;
  const uint32_t d = threadIdx.x;
  if (d == 0) trivial = 0;
  const uint32_t sum = state[2 * (kRadixMaxPasses + 1) + d];
  totals[d] = sum;
  __syncthreads();
  if (sum == n) trivial = 1;
  uint32_t v = sum;
  for (int off = 1; off < 256; off <<= 1) {
    __syncthreads();
    const uint32_t add = (d >= (uint32_t)off) ? totals[d - off] : 0u;
    __syncthreads();
    v += add;
    totals[d] = v;
  }
  __syncthreads();
  state[2 * (kRadixMaxPasses + 1) + d] = v - sum;  // exclusive base of digit d
  __syncthreads();
  if (d == 0) {
    const uint32_t cur = state[2 * pass];
    state[2 * pass + 1] = trivial;
    state[2 * (pass + 1)] = trivial ? cur : (cur ^ 1u);
  }
}

__global__ void __launch_bounds__(kRadixThreads)
k_radix_downsweep(uint32_t n, uint32_t* __restrict__ vals0, uint32_t* __restrict__ vals1,
                  IndirectKey key, int shift, const uint32_t* __restrict__ state, int pass,
                  const uint32_t* __restrict__ counts, uint32_t tiles) {
  if (state[2 * pass + 1]) return;  // every key has the same digit: order unchanged
  constexpr int kWarps = kRadixThreads / 32;
  __shared__ uint32_t base[256];
  __shared__ uint32_t warp_cnt[kWarps][256];
  const uint32_t tile = blockIdx.x;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t* in = state[2 * pass] ? vals1 : vals0;
  uint32_t* out = state[2 * pass] ? vals0 : vals1;
  base[tid] = counts[tid * tiles + tile] + state[2 * (kRadixMaxPasses + 1) + tid];
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  for (int r = 0; r < kRadixItems; ++r) {
    const uint32_t i = tile * kRadixTile + r * kRadixThreads + tid;
    const bool valid = i < n;
    const uint32_t v = valid ? in[i] : 0u;
    const uint32_t dig = valid ? digit_of(key, v, shift) : 256u;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) warp_cnt[w][tid] = 0;
    __syncthreads();
    const uint32_t peers = __match_any_sync(0xffffffffu, dig);
    const uint32_t rank = __popc(peers & lanemask_lt);
    if (valid && rank == 0) warp_cnt[warp][dig] = __popc(peers);
    __syncthreads();
    // exclusive prefix over warps, per digit (thread tid owns digit tid)
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t c = warp_cnt[w][tid];
      warp_cnt[w][tid] = run;
      run += c;
    }
    __syncthreads();
    if (valid) out[base[dig] + warp_cnt[warp][dig] + rank] = v;
    __syncthreads();
    base[tid] += run;
    __syncthreads();
  }
}

// Key-value variant: the 64-bit keys move with the indices (keys0/keys1 ping-pong with
// vals0/vals1 under the same pass state), so every pass reads and writes both coalesced
// instead of gathering the key of each index.
__global__ void __launch_bounds__(kRadixThreads)
k_radix_upsweep_kv(uint32_t n, const uint64_t* __restrict__ keys0, const uint64_t* __restrict__ keys1, int shift,
                   const uint32_t* __restrict__ state, int pass, uint32_t* __restrict__ counts, uint32_t tiles) {
  __shared__ uint32_t hist[256];
  const uint32_t tile = blockIdx.x;
  hist[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t* in = state[2 * pass] ? keys1 : keys0;
  const uint32_t base = tile * kRadixTile;
#pragma unroll
  for (int r = 0; r < kRadixItems; ++r) {
    const uint32_t i = base + r * kRadixThreads + threadIdx.x;
    if (i < n) atomicAdd(&hist[(uint32_t)(in[i] >> shift) & 0xffu], 1u);
  }
  __syncthreads();
  counts[threadIdx.x * tiles + tile] = hist[threadIdx.x];
}

__global__ void __launch_bounds__(kRadixThreads)
k_radix_downsweep_kv(uint32_t n, uint32_t* __restrict__ vals0, uint32_t* __restrict__ vals1,
                     uint64_t* __restrict__ keys0, uint64_t* __restrict__ keys1, int shift,
                     const uint32_t* __restrict__ state, int pass, const uint32_t* __restrict__ counts,
                     uint32_t tiles) {
  if (state[2 * pass + 1]) return;  // every key has the same digit: order unchanged
  constexpr int kWarps = kRadixThreads / 32;
  __shared__ uint32_t base[256];
  __shared__ uint32_t warp_cnt[kWarps][256];
  const uint32_t tile = blockIdx.x;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const bool flip = state[2 * pass] != 0;
  const uint32_t* in = flip ? vals1 : vals0;
  uint32_t* out = flip ? vals0 : vals1;
  const uint64_t* kin = flip ? keys1 : keys0;
  uint64_t* kout = flip ? keys0 : keys1;
  base[tid] = counts[tid * tiles + tile] + state[2 * (kRadixMaxPasses + 1) + tid];
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  for (int r = 0; r < kRadixItems; ++r) {
    const uint32_t i = tile * kRadixTile + r * kRadixThreads + tid;
    const bool valid = i < n;
    const uint32_t v = valid ? in[i] : 0u;
    const uint64_t key = valid ? kin[i] : 0u;
    const uint32_t dig = valid ? (uint32_t)(key >> shift) & 0xffu : 256u;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) warp_cnt[w][tid] = 0;
    __syncthreads();
    const uint32_t peers = __match_any_sync(0xffffffffu, dig);
    const uint32_t rank = __popc(peers & lanemask_lt);
    if (valid && rank == 0) warp_cnt[warp][dig] = __popc(peers);
    __syncthreads();
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t c = warp_cnt[w][tid];
      warp_cnt[w][tid] = run;
      run += c;
    }
    __syncthreads();
    if (valid) {
      const uint32_t at = base[dig] + warp_cnt[warp][dig] + rank;
      out[at] = v;
      kout[at] = key;
    }
    __syncthreads();
    base[tid] += run;
    __syncthreads();
  }
}

__global__ void k_radix_init(uint32_t* state) {
  if (threadIdx.x == 0) state[0] = 0;
}

}  // namespace

int radix_sort_indirect(cudaStream_t stream, uint32_t n, uint32_t* vals0, uint32_t* vals1,
                        const IndirectKey* stages, const int* stage_bits, int stage_count,
                        RadixScratch& scratch, uint64_t* launches) {
  const uint32_t tiles = (n + kRadixTile - 1) / kRadixTile;
  k_radix_init<<<1, 32, 0, stream>>>(scratch.state);
  *launches += 1;
  int pass = 0;
  for (int s = 0; s < stage_count; ++s) {
    for (int shift = 0; shift < stage_bits[s]; shift += 8) {
      k_radix_upsweep<<<tiles, kRadixThreads, 0, stream>>>(n, vals0, vals1, stages[s], shift, scratch.state,
                                                           pass, scratch.counts, tiles);
      k_radix_rowscan<<<256, 256, 0, stream>>>(scratch.counts, tiles, scratch.state);
      k_radix_digits<<<1, 256, 0, stream>>>(n, scratch.state, pass);
      k_radix_downsweep<<<tiles, kRadixThreads, 0, stream>>>(n, vals0, vals1, stages[s], shift, scratch.state,
                                                             pass, scratch.counts, tiles);
      *launches += 4;
      ++pass;
    }
  }
  return pass;
}

// Stable LSD sort of (keys0[i], vals0[i]) pairs by the low `bits` bits of the keys; the
// result is in the buffer that radix_result(state, passes, vals0, vals1) selects (the keys
// end beside it, in keys0 or keys1 under the same selection).
int radix_sort_kv(cudaStream_t stream, uint32_t n, uint32_t* vals0, uint32_t* vals1, uint64_t* keys0,
                  uint64_t* keys1, int bits, RadixScratch& scratch, uint64_t* launches) {
  const uint32_t tiles = (n + kRadixTile - 1) / kRadixTile;
  k_radix_init<<<1, 32, 0, stream>>>(scratch.state);
  *launches += 1;
  int pass = 0;
  for (int shift = 0; shift < bits; shift += 8) {
    k_radix_upsweep_kv<<<tiles, kRadixThreads, 0, stream>>>(n, keys0, keys1, shift, scratch.state, pass,
                                                            scratch.counts, tiles);
    k_radix_rowscan<<<256, 256, 0, stream>>>(scratch.counts, tiles, scratch.state);
    k_radix_digits<<<1, 256, 0, stream>>>(n, scratch.state, pass);
    k_radix_downsweep_kv<<<tiles, kRadixThreads, 0, stream>>>(n, vals0, vals1, keys0, keys1, shift, scratch.state,
                                                              pass, scratch.counts, tiles);
    *launches += 4;
    ++pass;
  }
  return pass;
}

}  // namespace ehgp
