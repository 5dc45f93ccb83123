// kf_compare.cu - Comparator::compare on the device (comparison.cpp:12-81):
// voxel-by-voxel deviation of two volumes of one geometry and pixel-by-pixel
// deviation of two sets of surface maps, for the pipeline-set ablations.
//
// The reference downloads both volumes (Pipeline::host_view) and walks them on
// one host core; here both stay in HBM, and one pass reads once each brick
// that either volume may have observed and skips the others by their
// observed bits or block allocation.  Counts and maxima are order-independent
// and come out exact; the means divide a double sum of the float deviations
// by the compared count, as Deviation does (comparison.hpp:64-83), with the
// sum taken per thread, then over warps, CTAs and a final fixed-order pass:
// deterministic for a given grid, and equal to the reference's sequential
// double sum to well under one float ulp of the mean.
#include <mutex>

#include "kf_internal.h"

namespace kf {
namespace {

constexpr unsigned kCompareThreads = 256;
constexpr unsigned kCompareCtas = 148 * 4;

// One CTA's share of a comparison.  Volumes: sum[0] / max[0] = |tsdf delta|,
// max[1] = |weight delta|.  Maps: sum[0] / max[0] = point distance, sum[1] /
// max[1] = normal angle.
struct ComparePartial {
  unsigned long long compared, only_primary, only_reference;
  double sum[2];
  float max[2];
};

// PairTally::classify (comparison.hpp:43-58)
__device__ __forceinline__ bool classify(bool primary_valid, bool reference_valid, ComparePartial& t) {
  if (primary_valid && reference_valid) {
    ++t.compared;
    return true;
  }
  if (primary_valid) {
    ++t.only_primary;
  } else if (reference_valid) {
    ++t.only_reference;
  }
  return false;
}

// std::max(max_, value) of Deviation::add: a NaN value leaves the maximum.
__device__ __forceinline__ float keep_max(float current, float value) { return current < value ? value : current; }

__device__ __forceinline__ void clear(ComparePartial& t) {
  t.compared = t.only_primary = t.only_reference = 0;
  t.sum[0] = t.sum[1] = 0.0;
  t.max[0] = t.max[1] = 0.0f;
}

__device__ __forceinline__ void combine(ComparePartial& a, const ComparePartial& b) {
  a.compared += b.compared;
  a.only_primary += b.only_primary;
  a.only_reference += b.only_reference;
  a.sum[0] += b.sum[0];
  a.sum[1] += b.sum[1];
  a.max[0] = keep_max(a.max[0], b.max[0]);
  a.max[1] = keep_max(a.max[1], b.max[1]);
}

__device__ __forceinline__ void warp_combine(ComparePartial& t) {
  for (int off = 16; off > 0; off >>= 1) {
    ComparePartial o;
    o.compared = __shfl_down_sync(0xFFFFFFFFu, t.compared, off);
    o.only_primary = __shfl_down_sync(0xFFFFFFFFu, t.only_primary, off);
    o.only_reference = __shfl_down_sync(0xFFFFFFFFu, t.only_reference, off);
    o.sum[0] = __shfl_down_sync(0xFFFFFFFFu, t.sum[0], off);
    o.sum[1] = __shfl_down_sync(0xFFFFFFFFu, t.sum[1], off);
    o.max[0] = __shfl_down_sync(0xFFFFFFFFu, t.max[0], off);
    o.max[1] = __shfl_down_sync(0xFFFFFFFFu, t.max[1], off);
    combine(t, o);
  }
}

// The CTA's total into `out` (thread 0 writes it); fixed order throughout.
__device__ __forceinline__ void cta_combine(ComparePartial& t, ComparePartial* out) {
  __shared__ ComparePartial warps[kCompareThreads / 32];
  warp_combine(t);
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  if (lane == 0) warps[warp] = t;
  __syncthreads();
  if (warp == 0) {
    if (lane < kCompareThreads / 32) {
      t = warps[lane];
    } else {
      clear(t);
    }
    warp_combine(t);
    if (lane == 0) *out = t;
  }
}

// Two consecutive voxels (storage offsets 2t, 2t+1 of a brick) in one load.
template <int Kind>
__device__ __forceinline__ void load_pair(const void* voxels, uint32_t slot, uint32_t t,
                                          typename VoxelTraits<Kind>::Raw& r0, typename VoxelTraits<Kind>::Raw& r1) {
  using VT = VoxelTraits<Kind>;
  if (slot == kUnallocated) {
    r0 = r1 = VT::unobserved();
    return;
  }
  if constexpr (Kind == KF_VOXEL_FLOAT) {
    const float4 q = __ldcs(reinterpret_cast<const float4*>(voxels) + static_cast<size_t>(slot) * 256 + t);
    r0 = make_float2(q.x, q.y);
    r1 = make_float2(q.z, q.w);
  } else {
    const uint2 q = __ldcs(reinterpret_cast<const uint2*>(voxels) + static_cast<size_t>(slot) * 256 + t);
    r0 = q.x;
    r1 = q.y;
  }
}

template <int KindA, int KindB>
__device__ __forceinline__ void compare_voxel(typename VoxelTraits<KindA>::Raw a, typename VoxelTraits<KindB>::Raw b,
                                              ComparePartial& t) {
  using TA = VoxelTraits<KindA>;
  using TB = VoxelTraits<KindB>;
  const float wa = TA::weight(a), wb = TB::weight(b);
  if (!classify(wa > 0.0f, wb > 0.0f, t)) return;
  const float distance = fabsf(TA::tsdf(a) - TB::tsdf(b));
  t.sum[0] += static_cast<double>(distance);
  t.max[0] = keep_max(t.max[0], distance);
  t.max[1] = keep_max(t.max[1], fabsf(wa - wb));
}

// Where one volume's observed voxels can be.  A dense volume carries the
// integration's per-voxel `observed` bits (8 uint4 per brick, one per z
// layer, .z/.w = the layer's observed bits): every voxel an integration wrote
// has its bit set, so a brick without bits holds no voxel of weight > 0.  A
// sparse volume holds observed voxels only in allocated blocks.  A dense
// volume that no integration touched yet (no bits allocated) holds none.
struct CompareSide {
  const unsigned long long* table;  // sparse: the voxel-block hash (block -> slot)
  uint32_t table_mask;
  const uint4* observed;  // dense
  uint32_t fresh;         // dense, never integrated
};

__device__ __forceinline__ uint32_t slot_of(const CompareSide& s, uint32_t blk) {
  if (s.fresh) return kUnallocated;  // every voxel reads as unobserved
  return s.table == nullptr ? blk : block_table_lookup(s.table, s.table_mask, blk);
}

__device__ __forceinline__ bool may_hold_observed(const CompareSide& s, uint32_t blk) {
  if (s.fresh) return false;
  if (s.table != nullptr) return block_table_lookup(s.table, s.table_mask, blk) != kUnallocated;
  // the upper 8 bytes of each layer's 16: its two observed words
  const uint2* layers = reinterpret_cast<const uint2*>(s.observed + static_cast<size_t>(blk) * 8u);
  uint32_t any = 0u;
#pragma unroll
  for (int z = 0; z < 8; ++z) {
    const uint2 q = __ldg(layers + 2 * z + 1);
    any |= q.x | q.y;
  }
  return any != 0u;
}

constexpr uint32_t kChunkBricks = 32;                      // blocks per live-mask word
constexpr uint32_t kChunksPerCta = kCompareThreads / 32;  // one chunk per warp

// The live blocks (where either volume may hold an observed voxel) as a list
// in block order, built in three passes: masks, a scan of the per-CTA counts,
// a scatter.  The comparison then spreads the list evenly over all warps.
//
// Pass 1: one warp per chunk of 32 consecutive blocks (x-major block index).
__global__ void __launch_bounds__(kCompareThreads)
    live_mask_kernel(CompareSide side_a, CompareSide side_b, uint32_t blocks, uint32_t* __restrict__ masks,
                     uint32_t* __restrict__ cta_counts) {
  __shared__ uint32_t warp_counts[kChunksPerCta];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t chunk = blockIdx.x * kChunksPerCta + warp;
  const uint32_t blk = chunk * kChunkBricks + lane;
  const bool live = blk < blocks && (may_hold_observed(side_a, blk) || may_hold_observed(side_b, blk));
  const uint32_t mask = __ballot_sync(0xFFFFFFFFu, live);
  if (lane == 0) {
    if (chunk * kChunkBricks < blocks) masks[chunk] = mask;
    warp_counts[warp] = static_cast<uint32_t>(__popc(mask));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t n = 0;
    for (uint32_t w = 0; w < kChunksPerCta; ++w) n += warp_counts[w];
    cta_counts[blockIdx.x] = n;
  }
}

// Pass 2 (one CTA): exclusive prefix sums of the CTA counts; offsets[ctas]
// receives the number of live blocks.
__global__ void __launch_bounds__(1024)
    live_scan_kernel(const uint32_t* __restrict__ counts, uint32_t ctas, uint32_t* __restrict__ offsets) {
  __shared__ uint32_t partial[1024];
  const uint32_t per = (ctas + 1023u) / 1024u;
  const uint32_t begin = min(threadIdx.x * per, ctas), end = min(begin + per, ctas);
  uint32_t sum = 0;
  for (uint32_t i = begin; i < end; ++i) sum += counts[i];
  partial[threadIdx.x] = sum;
  __syncthreads();
  for (uint32_t off = 1; off < 1024u; off <<= 1) {
    const uint32_t v = threadIdx.x >= off ? partial[threadIdx.x - off] : 0u;
    __syncthreads();
    partial[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = partial[threadIdx.x] - sum;
  for (uint32_t i = begin; i < end; ++i) {
    offsets[i] = run;
    run += counts[i];
  }
  if (threadIdx.x == 1023u) offsets[ctas] = partial[1023];
}

// Pass 3: every live block's index at its rank.
__global__ void __launch_bounds__(kCompareThreads)
    live_list_kernel(const uint32_t* __restrict__ masks, uint32_t chunks, const uint32_t* __restrict__ offsets,
                     uint32_t* __restrict__ list) {
  __shared__ uint32_t warp_counts[kChunksPerCta];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t chunk = blockIdx.x * kChunksPerCta + warp;
  const uint32_t mask = chunk < chunks ? masks[chunk] : 0u;
  if (lane == 0) warp_counts[warp] = static_cast<uint32_t>(__popc(mask));
  __syncthreads();
  uint32_t base = offsets[blockIdx.x];
  for (uint32_t w = 0; w < warp; ++w) base += warp_counts[w];
  if ((mask >> lane) & 1u) {
    list[base + static_cast<uint32_t>(__popc(mask & ((1u << lane) - 1u)))] = chunk * kChunkBricks + lane;
  }
}

// Pass 4: a warp per live block, grid-strided over the list; each lane reads
// pairs j * 32 + lane (j = 0..7) of the brick in two batches of four, one
// 16-byte (float) or 8-byte load per pair and volume, so every lane keeps
// eight loads in flight.  Voxels of the padding of edge bricks (outside the
// resolution) are left out.
template <int KindA, int KindB>
__global__ void __launch_bounds__(kCompareThreads)
    compare_volumes_kernel(VolumeDev a, VolumeDev b, CompareSide side_a, CompareSide side_b,
                           const uint32_t* __restrict__ list, const uint32_t* __restrict__ list_count,
                           ComparePartial* __restrict__ partials) {
  using RawA = typename VoxelTraits<KindA>::Raw;
  using RawB = typename VoxelTraits<KindB>::Raw;
  ComparePartial t;
  clear(t);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warps = gridDim.x * kChunksPerCta;
  const uint32_t live = __ldg(list_count);
  for (uint32_t i = blockIdx.x * kChunksPerCta + (threadIdx.x >> 5); i < live; i += warps) {
    const uint32_t blk = __ldg(list + i);
    const uint32_t sa = slot_of(side_a, blk), sb = slot_of(side_b, blk);
    const uint32_t bxi = blk % a.bx, byi = (blk / a.bx) % a.by, bzi = blk / (a.bx * a.by);
#pragma unroll
    for (uint32_t half = 0; half < 2; ++half) {
      RawA a0[4], a1[4];
      RawB b0[4], b1[4];
#pragma unroll
      for (uint32_t j = 0; j < 4; ++j) {
        const uint32_t pair = (half * 4u + j) * 32u + lane;
        load_pair<KindA>(a.voxels, sa, pair, a0[j], a1[j]);
        load_pair<KindB>(b.voxels, sb, pair, b0[j], b1[j]);
      }
#pragma unroll
      for (uint32_t j = 0; j < 4; ++j) {
        const uint32_t o0 = 2u * ((half * 4u + j) * 32u + lane);
        const uint32_t x = bxi * 8u + (o0 & 7u), y = byi * 8u + ((o0 >> 3) & 7u), z = bzi * 8u + (o0 >> 6);
        if (y < a.ry && z < a.rz) {
          if (x < a.rx) compare_voxel<KindA, KindB>(a0[j], b0[j], t);
          if (x + 1u < a.rx) compare_voxel<KindA, KindB>(a1[j], b1[j], t);
        }
      }
    }
  }
  cta_combine(t, partials + blockIdx.x);
}

// Surface maps (x, y, z floats per pixel).  A pixel is valid when its point
// and normal are finite (valid_surface_pixel, comparison.hpp:86-90); the
// normal angle is angle_between (vector.hpp:177-185) with the host branch of
// normalized, and its atan2 evaluated in double and rounded once to float.
__global__ void __launch_bounds__(kCompareThreads)
    compare_maps_kernel(const float* __restrict__ pp, const float* __restrict__ pn, const float* __restrict__ rp,
                        const float* __restrict__ rn, uint64_t pixels, ComparePartial* __restrict__ partials) {
  ComparePartial t;
  clear(t);
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < pixels; i += stride) {
    const f3 p_point = ldg3(pp + 3 * i), p_normal = ldg3(pn + 3 * i);
    const f3 r_point = ldg3(rp + 3 * i), r_normal = ldg3(rn + 3 * i);
    if (!classify(finite3(p_point) && finite3(p_normal), finite3(r_point) && finite3(r_normal), t)) continue;
    const float distance = norm(p_point - r_point);
    const f3 source = normalized(p_normal), target = normalized(r_normal);
    const float angle = static_cast<float>(
        atan2(static_cast<double>(norm(cross(source, target))), static_cast<double>(dot(source, target))));
    t.sum[0] += static_cast<double>(distance);
    t.max[0] = keep_max(t.max[0], distance);
    t.sum[1] += static_cast<double>(angle);
    t.max[1] = keep_max(t.max[1], angle);
  }
  cta_combine(t, partials + blockIdx.x);
}

// The CTA partials summed in index order by one CTA.
__global__ void __launch_bounds__(kCompareThreads)
    compare_finish_kernel(const ComparePartial* __restrict__ partials, unsigned count, ComparePartial* __restrict__ out) {
  ComparePartial t;
  clear(t);
  for (unsigned i = threadIdx.x; i < count; i += blockDim.x) combine(t, partials[i]);
  cta_combine(t, out);
}

// Partials of the running comparison, per device; one comparison at a time.
struct CompareScratch {
  std::mutex lock;
  int device = -1;
  DeviceArray<ComparePartial> partials;
  DeviceArray<float> maps;     // staging of host surface maps
  DeviceArray<uint32_t> live;  // live-block masks, CTA counts, offsets, list
  PinnedArray<ComparePartial> result;
};
CompareScratch& compare_scratch() {
  static CompareScratch* s = new CompareScratch();  // never destroyed: lives past static teardown
  return *s;
}

void prepare(CompareScratch& s) {
  int device = 0;
  check(cudaGetDevice(&device), "compare device");
  if (s.device != device) {  // another device: start over (the arrays belong to the old one)
    s.partials = DeviceArray<ComparePartial>();
    s.maps = DeviceArray<float>();
    s.live = DeviceArray<uint32_t>();
    s.device = device;
  }
  if (s.partials.count == 0) s.partials.resize(kCompareCtas + 1);
  s.result.resize(1);
}

ComparePartial finish(CompareScratch& s, cudaStream_t stream) {
  compare_finish_kernel<<<1, kCompareThreads, 0, stream>>>(s.partials.ptr, kCompareCtas, s.partials.ptr + kCompareCtas);
  check(cudaGetLastError(), "compare_finish_kernel launch");
  check(cudaMemcpyAsync(s.result.ptr, s.partials.ptr + kCompareCtas, sizeof(ComparePartial), cudaMemcpyDeviceToHost,
                        stream),
        "comparison download");
  check(cudaStreamSynchronize(stream), "comparison");
  return *s.result.ptr;
}

// Deviation::mean (comparison.hpp:73-78)
float mean_of(double sum, unsigned long long count) {
  return count == 0 ? 0.0f : static_cast<float>(sum / static_cast<double>(count));
}

CompareSide side_of(const Pipeline& p) {
  CompareSide side{};
  side.table = p.view.table;
  side.table_mask = p.view.table_mask;
  if (p.view.table == nullptr) {
    // the bits exist from the first integration on (prepare_blocks runs
    // before every integration of a dense volume)
    side.observed = p.voxel_bits.count ? reinterpret_cast<const uint4*>(p.voxel_bits.ptr) : nullptr;
    side.fresh = p.voxel_bits.count ? 0u : 1u;
  }
  return side;
}

template <int KindA>
void launch_compare_volumes_as(const Pipeline& a, const Pipeline& b, const CompareSide& sa, const CompareSide& sb,
                               const uint32_t* list, const uint32_t* count, ComparePartial* partials, cudaStream_t s) {
  switch (b.config.voxel) {
    case KF_VOXEL_QUANTIZED:
      compare_volumes_kernel<KindA, KF_VOXEL_QUANTIZED>
          <<<kCompareCtas, kCompareThreads, 0, s>>>(a.view, b.view, sa, sb, list, count, partials);
      break;
    case KF_VOXEL_BF16:
      compare_volumes_kernel<KindA, KF_VOXEL_BF16>
          <<<kCompareCtas, kCompareThreads, 0, s>>>(a.view, b.view, sa, sb, list, count, partials);
      break;
    default:
      compare_volumes_kernel<KindA, KF_VOXEL_FLOAT>
          <<<kCompareCtas, kCompareThreads, 0, s>>>(a.view, b.view, sa, sb, list, count, partials);
      break;
  }
}

void launch_compare_volumes(const Pipeline& a, const Pipeline& b, CompareScratch& scratch, cudaStream_t s) {
  const CompareSide sa = side_of(a), sb = side_of(b);
  const uint32_t blocks = a.view.bx * a.view.by * a.view.bz;
  const uint32_t chunks = ceil_div(blocks, kChunkBricks);
  const uint32_t ctas = ceil_div(chunks, kChunksPerCta);
  // [masks: chunks][counts: ctas][offsets: ctas + 1][list: blocks]
  const size_t words = static_cast<size_t>(chunks) + 2u * ctas + 1u + blocks;
  if (scratch.live.count < words) scratch.live.resize(words);
  uint32_t* masks = scratch.live.ptr;
  uint32_t* counts = masks + chunks;
  uint32_t* offsets = counts + ctas;
  uint32_t* list = offsets + ctas + 1;
  live_mask_kernel<<<ctas, kCompareThreads, 0, s>>>(sa, sb, blocks, masks, counts);
  check(cudaGetLastError(), "live_mask_kernel launch");
  live_scan_kernel<<<1, 1024, 0, s>>>(counts, ctas, offsets);
  check(cudaGetLastError(), "live_scan_kernel launch");
  live_list_kernel<<<ctas, kCompareThreads, 0, s>>>(masks, chunks, offsets, list);
  check(cudaGetLastError(), "live_list_kernel launch");
  switch (a.config.voxel) {
    case KF_VOXEL_QUANTIZED:
      launch_compare_volumes_as<KF_VOXEL_QUANTIZED>(a, b, sa, sb, list, offsets + ctas, scratch.partials.ptr, s);
      break;
    case KF_VOXEL_BF16:
      launch_compare_volumes_as<KF_VOXEL_BF16>(a, b, sa, sb, list, offsets + ctas, scratch.partials.ptr, s);
      break;
    default:
      launch_compare_volumes_as<KF_VOXEL_FLOAT>(a, b, sa, sb, list, offsets + ctas, scratch.partials.ptr, s);
      break;
  }
  check(cudaGetLastError(), "compare_volumes_kernel launch");
}

bool same_geometry(const kf_volume_geometry& a, const kf_volume_geometry& b) {
  return a.res_x == b.res_x && a.res_y == b.res_y && a.res_z == b.res_z && a.voxel_size == b.voxel_size &&
         a.origin[0] == b.origin[0] && a.origin[1] == b.origin[1] && a.origin[2] == b.origin[2] &&
         a.truncation_distance == b.truncation_distance;
}

}  // namespace
}  // namespace kf

using namespace kf;

extern "C" {

kf_status kf_compare_volumes(kf_pipeline* primary, kf_pipeline* reference, kf_volume_comparison* out) {
  return guarded([&] {
    require(primary != nullptr && reference != nullptr && out != nullptr, "kf_compare_volumes: null argument");
    Pipeline& a = primary->impl;
    Pipeline& b = reference->impl;
    require(same_geometry(a.config.volume, b.config.volume), "Volume comparison requires matching geometry");
    CompareScratch& s = compare_scratch();
    std::lock_guard<std::mutex> hold(s.lock);
    prepare(s);
    // the reference's volume is read on the primary's stream after its own work
    if (&a != &b) check(cudaStreamSynchronize(b.stream), "comparison order");
    launch_compare_volumes(a, b, s, a.stream);
    const ComparePartial r = finish(s, a.stream);
    out->compared_voxels = r.compared;
    out->only_primary = r.only_primary;
    out->only_reference = r.only_reference;
    out->max_distance_delta = r.max[0];
    out->mean_distance_delta = mean_of(r.sum[0], r.compared);
    out->max_weight_delta = r.max[1];
  });
}

kf_status kf_compare_surface_maps(const kf_surface_maps* primary, const kf_surface_maps* reference,
                                  kf_surface_maps_comparison* out) {
  return guarded([&] {
    require(primary != nullptr && reference != nullptr && out != nullptr, "kf_compare_surface_maps: null argument");
    require(primary->points != nullptr && primary->normals != nullptr && reference->points != nullptr &&
                reference->normals != nullptr,
            "kf_compare_surface_maps: null map");
    require(primary->width == reference->width && primary->height == reference->height,
            "Surface map comparison requires matching dimensions");
    require((primary->memory == KF_MEMORY_HOST || primary->memory == KF_MEMORY_DEVICE) &&
                (reference->memory == KF_MEMORY_HOST || reference->memory == KF_MEMORY_DEVICE),
            "kf_compare_surface_maps: unknown memory space");
    const uint64_t pixels = static_cast<uint64_t>(primary->width) * primary->height;
    CompareScratch& s = compare_scratch();
    std::lock_guard<std::mutex> hold(s.lock);
    prepare(s);
    const cudaStream_t stream = nullptr;  // legacy stream: after the device work of every blocking stream
    // host maps are staged in device memory: [primary points, normals, reference points, normals]
    const size_t floats = 3 * pixels;
    const bool stage = primary->memory == KF_MEMORY_HOST || reference->memory == KF_MEMORY_HOST;
    if (stage && s.maps.count < 4 * floats) s.maps.resize(4 * floats);
    const float* view[4] = {primary->points, primary->normals, reference->points, reference->normals};
    const int32_t memory[4] = {primary->memory, primary->memory, reference->memory, reference->memory};
    if (pixels != 0) {
      for (int i = 0; i < 4; ++i) {
        if (memory[i] != KF_MEMORY_HOST) continue;
        float* dst = s.maps.ptr + i * floats;
        check(cudaMemcpyAsync(dst, view[i], floats * sizeof(float), cudaMemcpyHostToDevice, stream), "map upload");
        view[i] = dst;
      }
    }
    check(cudaDeviceSynchronize(), "comparison order");  // device maps may come from any stream
    compare_maps_kernel<<<kCompareCtas, kCompareThreads, 0, stream>>>(view[0], view[1], view[2], view[3], pixels,
                                                                       s.partials.ptr);
    check(cudaGetLastError(), "compare_maps_kernel launch");
    const ComparePartial r = finish(s, stream);
    out->compared_pixels = r.compared;
    out->only_primary = r.only_primary;
    out->only_reference = r.only_reference;
    out->max_point_distance = r.max[0];
    out->mean_point_distance = mean_of(r.sum[0], r.compared);
    out->max_normal_angle = r.max[1];
    out->mean_normal_angle = mean_of(r.sum[1], r.compared);
  });
}

}  // extern "C"
