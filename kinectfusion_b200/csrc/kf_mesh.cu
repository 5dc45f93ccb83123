// kf_mesh.cu - marching cubes on the device (MarchingCubes::extract and
// MeshBuilder, marching_cubes.cpp:311-485), dense and sparse volumes.
//
// The mesh is the one the host builder makes, element for element: the same
// cells in the same order (x fastest over the (res-1)^3 cells; sparse:
// allocated blocks in block order, x fastest within each), the same
// welded vertices numbered in order of first use, the same positions,
// normals and colours.  The triangulation table is this library's generated
// one (kf_mc_tables.h).  Passes:
//  1. per row of cells (fixed y, z; sparse: per allocated block), classify
//     the cells: a cell whose corners are all observed, finite and at least
//     min_weight has a sign case; set a bit per crossed edge (key = near
//     voxel's storage index * 3 + axis) and count the unit's triangles.  Cells whose stencil the raycast's stencil
//     bits decide (no observed corner, or all corners exactly 1) cannot cross
//     the surface and are not read;
//  2. exclusive scans give each row its first triangle and each crossed edge
//     a compact id;
//  3. per row again, write every triangle corner's edge id and record each
//     edge's first use (smallest triangle-corner position, atomicMin);
//  4. a bitmap of first-use positions, scanned, numbers the vertices in
//     order of first use; one thread per edge word computes its vertices;
//  5. triangle corners are mapped to vertex numbers; the face-normal fill
//     for vertices without a gradient normal runs on the host, in triangle
//     order, as the host builder does.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "kf_internal.h"
#include "kf_mc_tables.h"
#include "kf_sampler.cuh"

namespace kf {
namespace {

__constant__ uint16_t c_edge_mask[256];
__constant__ int8_t c_triangles[256][16];
__constant__ uint8_t c_corner[8][3];
__constant__ uint8_t c_edge[12][3];

constexpr int kRowThreads = 256;
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;  // elements per thread of a scan block
constexpr unsigned kScanBlock = kScanThreads * kScanItems;

// Sign case of cell (x, y, z), or -1 when a corner is unobserved, not finite
// or lighter than min_weight (MeshBuilder::add_cell, marching_cubes.cpp:369-384).
template <int Kind>
__device__ __forceinline__ int cell_case(const VolumeDev& v, uint32_t x, uint32_t y, uint32_t z, float min_weight) {
  using VT = VoxelTraits<Kind>;
  const auto* voxels = reinterpret_cast<const typename VT::Raw*>(v.voxels);
  int cube = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const long long i = storage_index(v, x + c_corner[c][0], y + c_corner[c][1], z + c_corner[c][2]);
    if (i < 0) return -1;
    const typename VT::Raw r = __ldg(voxels + i);
    if (!VT::observed(r) || !VT::finite(r) || VT::weight(r) < min_weight) return -1;
    if (VT::tsdf(r) < 0.0f) cube |= 1 << c;
  }
  return cube;
}

__device__ __forceinline__ bool stencil_undecided(const uint4* __restrict__ stencil_bits, const VolumeDev& v,
                                                  uint32_t x, uint32_t y, uint32_t z) {
  if (stencil_bits == nullptr) return true;
  const uint32_t record = (((z >> 3) * v.by + (y >> 3)) * v.bx + (x >> 3)) * 8u + (z & 7u);
  const uint32_t bit = (y & 7u) * 8u + (x & 7u);
  const uint4 r = __ldg(stencil_bits + record);
  return (((bit < 32u ? r.x >> bit : r.y >> (bit - 32u))) & 1u) != 0u;
}

// Weld key of cube edge `edge` of cell (x, y, z): the near voxel's storage
// index * 3 + axis (unique per edge; the near voxel is stored whenever a
// cell using the edge is meshed).
__device__ __forceinline__ unsigned long long edge_key(const VolumeDev& v, uint32_t x, uint32_t y, uint32_t z,
                                                       int edge) {
  const int near = c_edge[edge][0];
  const long long i = storage_index(v, x + c_corner[near][0], y + c_corner[near][1], z + c_corner[near][2]);
  return static_cast<unsigned long long>(i) * 3ull + c_edge[edge][2];
}

__device__ __forceinline__ uint32_t triangle_count(int cube) {
  uint32_t n = 0;
  while (n < 5 && c_triangles[cube][3 * n] >= 0) ++n;
  return n;
}

// Exclusive scan of n values over a CTA of kRowThreads; returns the total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t value, uint32_t& prefix, uint32_t* s_warp) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t incl = value;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t up = __shfl_up_sync(0xFFFFFFFFu, incl, off);
    if (lane >= static_cast<unsigned>(off)) incl += up;
  }
  if (lane == 31u) s_warp[warp] = incl;
  __syncthreads();
  uint32_t warp_base = 0, total = 0;
  for (unsigned w = 0; w < blockDim.x / 32u; ++w) {
    if (w < warp) warp_base += s_warp[w];
    total += s_warp[w];
  }
  __syncthreads();
  prefix = warp_base + incl - value;
  return total;
}

// Pass 1 (Write = false): the crossed-edge bits of an active cell.  Pass 3
// (Write = true): its triangle corners' edge ids from `first` on, and each
// edge's first use.
template <bool Write>
__device__ __forceinline__ void emit_cell(const VolumeDev& v, uint32_t x, uint32_t y, uint32_t z, int cube,
                                          uint32_t tris, uint32_t first, uint32_t* __restrict__ edge_words,
                                          const uint32_t* __restrict__ word_first, uint32_t* __restrict__ corner_edge,
                                          uint32_t* __restrict__ first_use) {
  if constexpr (!Write) {
    const uint32_t mask = c_edge_mask[cube];
    for (int e = 0; e < 12; ++e) {
      if (!((mask >> e) & 1u)) continue;
      const unsigned long long key = edge_key(v, x, y, z, e);
      atomicOr(edge_words + (key >> 5), 1u << (key & 31u));
    }
  } else {
    for (uint32_t t = 0; t < tris; ++t) {
      for (int k = 0; k < 3; ++k) {
        const unsigned long long key = edge_key(v, x, y, z, c_triangles[cube][3 * t + k]);
        const uint32_t w = static_cast<uint32_t>(key >> 5), b = static_cast<uint32_t>(key & 31u);
        const uint32_t id = word_first[w] + __popc(edge_words[w] & ((1u << b) - 1u));
        const uint32_t position = 3u * (first + t) + static_cast<uint32_t>(k);
        corner_edge[position] = id;
        atomicMin(first_use + id, position);
      }
    }
  }
}

// Dense volumes: one CTA per row of cells (fixed y, z), x fastest (the host
// builder's GridIndices order).  Pass 1 counts the row's triangles.
template <int Kind, bool Write>
__global__ void __launch_bounds__(kRowThreads)
    mc_rows_kernel(VolumeDev v, const uint4* __restrict__ stencil_bits, float min_weight,
                   uint32_t* __restrict__ edge_words, uint32_t* __restrict__ row_tris,
                   const uint32_t* __restrict__ row_first, const uint32_t* __restrict__ word_first,
                   uint32_t* __restrict__ corner_edge, uint32_t* __restrict__ first_use) {
  __shared__ uint32_t s_warp[kRowThreads / 32];
  const uint32_t cx = v.rx - 1, cy = v.ry - 1;
  const uint32_t row = blockIdx.x;
  const uint32_t y = row % cy, z = row / cy;
  uint32_t base = Write ? row_first[row] : 0u;
  for (uint32_t x0 = 0; x0 < cx; x0 += kRowThreads) {
    const uint32_t x = x0 + threadIdx.x;
    int cube = -1;
    uint32_t tris = 0;
    if (x < cx && stencil_undecided(stencil_bits, v, x, y, z)) {
      cube = cell_case<Kind>(v, x, y, z, min_weight);
      if (cube >= 0 && c_edge_mask[cube] != 0) tris = triangle_count(cube);
    }
    uint32_t prefix;
    const uint32_t total = block_exclusive_scan(tris, prefix, s_warp);
    if (tris != 0u) emit_cell<Write>(v, x, y, z, cube, tris, base + prefix, edge_words, word_first, corner_edge,
                                     first_use);
    base += total;
  }
  if (!Write && threadIdx.x == 0) row_tris[row] = base;
}

// Sparse volumes: one CTA of 512 threads per allocated block, in block order,
// its cells x fastest, then y, then z (BlockVoxels order, clipped to the
// cells of the volume).  Pass 1 counts the block's triangles.
template <int Kind, bool Write>
__global__ void __launch_bounds__(512)
    mc_blocks_kernel(VolumeDev v, const uint32_t* __restrict__ blocks, float min_weight,
                     uint32_t* __restrict__ edge_words, uint32_t* __restrict__ unit_tris,
                     const uint32_t* __restrict__ unit_first, const uint32_t* __restrict__ word_first,
                     uint32_t* __restrict__ corner_edge, uint32_t* __restrict__ first_use) {
  __shared__ uint32_t s_warp[512 / 32];
  const uint32_t block = blocks[blockIdx.x];
  const uint32_t x = (block % v.bx) * 8u + (threadIdx.x & 7u);
  const uint32_t y = ((block / v.bx) % v.by) * 8u + ((threadIdx.x >> 3) & 7u);
  const uint32_t z = (block / (v.bx * v.by)) * 8u + (threadIdx.x >> 6);
  int cube = -1;
  uint32_t tris = 0;
  if (x < v.rx - 1 && y < v.ry - 1 && z < v.rz - 1) {
    cube = cell_case<Kind>(v, x, y, z, min_weight);
    if (cube >= 0 && c_edge_mask[cube] != 0) tris = triangle_count(cube);
  }
  uint32_t prefix;
  const uint32_t total = block_exclusive_scan(tris, prefix, s_warp);
  if (tris != 0u) {
    emit_cell<Write>(v, x, y, z, cube, tris, (Write ? unit_first[blockIdx.x] : 0u) + prefix, edge_words, word_first,
                     corner_edge, first_use);
  }
  if (!Write && threadIdx.x == 0) unit_tris[blockIdx.x] = total;
}

// Allocated blocks of a sparse grid, in block order.
// Sparse storage: flag the block of every used pool slot (the slots are
// handed out in order, min(attempts, capacity) of them).
__global__ void allocated_flags_kernel(const uint32_t* __restrict__ slot_block,
                                       const unsigned long long* __restrict__ allocated, unsigned long long capacity,
                                       uint32_t* __restrict__ flags) {
  const unsigned long long used = allocated[0] < capacity ? allocated[0] : capacity;
  for (unsigned long long s = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; s < used;
       s += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    flags[slot_block[s]] = 1u;
  }
}

__global__ void allocated_list_kernel(const uint32_t* __restrict__ flags, const uint32_t* __restrict__ position,
                                      uint32_t blocks, uint32_t* __restrict__ list) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < blocks && flags[b] != 0u) list[position[b]] = b;
}

// Exclusive scan of n values (or of their popcounts) in blocks of
// kScanBlock; block totals to `sums`.
template <bool Popc>
__global__ void __launch_bounds__(kScanThreads)
    scan_block_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t* __restrict__ sums,
                      uint32_t n) {
  __shared__ uint32_t s_warp[kScanThreads / 32];
  const uint32_t first = blockIdx.x * kScanBlock + threadIdx.x * kScanItems;
  uint32_t v[kScanItems], local = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const uint32_t e = first + i;
    const uint32_t raw = e < n ? in[e] : 0u;
    v[i] = Popc ? static_cast<uint32_t>(__popc(raw)) : raw;
    local += v[i];
  }
  uint32_t prefix;
  const uint32_t total = block_exclusive_scan(local, prefix, s_warp);
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const uint32_t e = first + i;
    if (e < n) out[e] = prefix;
    prefix += v[i];
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void scan_add_kernel(uint32_t* __restrict__ out, const uint32_t* __restrict__ offsets, uint32_t n) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) out[e] += offsets[e / kScanBlock];
}

// Exclusive scan of `n` device values (popcounts when `popc`) into `out`;
// returns the total.  Recursive over the block totals.
uint32_t exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, bool popc, cudaStream_t s) {
  if (n == 0) return 0;
  const uint32_t blocks = ceil_div(n, kScanBlock);
  DeviceArray<uint32_t> sums(blocks), offsets(blocks);
  if (popc) {
    scan_block_kernel<true><<<blocks, kScanThreads, 0, s>>>(in, out, sums.ptr, n);
  } else {
    scan_block_kernel<false><<<blocks, kScanThreads, 0, s>>>(in, out, sums.ptr, n);
  }
  check(cudaGetLastError(), "scan_block_kernel launch");
  uint32_t total = 0;
  if (blocks == 1) {
    check(cudaMemcpyAsync(&total, sums.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "scan total");
    check(cudaStreamSynchronize(s), "scan total");
    return total;
  }
  total = exclusive_scan(sums.ptr, offsets.ptr, blocks, false, s);
  scan_add_kernel<<<ceil_div(n, 256), 256, 0, s>>>(out, offsets.ptr, n);
  check(cudaGetLastError(), "scan_add_kernel launch");
  check(cudaStreamSynchronize(s), "scan");  // before the scratch arrays go
  return total;
}

// Bit of every edge's first use.
__global__ void mark_first_use_kernel(const uint32_t* __restrict__ first_use, uint32_t* __restrict__ use_words,
                                      uint32_t vertices) {
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= vertices) return;
  const uint32_t p = first_use[id];
  atomicOr(use_words + (p >> 5), 1u << (p & 31u));
}

// MeshBuilder::vertex_on_edge (marching_cubes.cpp:403-437) for every crossed
// edge of one bitmap word; vertex number = rank of the edge's first use.
template <int Kind>
__global__ void __launch_bounds__(256)
    mc_vertex_kernel(VolumeDev v, const uint32_t* __restrict__ slot_block, const uint32_t* __restrict__ edge_words,
                     const uint32_t* __restrict__ word_first,
                     const uint32_t* __restrict__ first_use, const uint32_t* __restrict__ use_words,
                     const uint32_t* __restrict__ use_first, uint32_t words, float* __restrict__ positions,
                     float* __restrict__ normals, float* __restrict__ colors, uint32_t* __restrict__ vertex_of) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= words) return;
  uint32_t word = edge_words[w];
  if (word == 0u) return;
  using VT = VoxelTraits<Kind>;
  const auto* voxels = reinterpret_cast<const typename VT::Raw*>(v.voxels);
  const Sampler<Kind> s{v};
  uint32_t id = word_first[w];
  while (word != 0u) {
    const uint32_t b = static_cast<uint32_t>(__ffs(word) - 1);
    word &= word - 1u;
    const unsigned long long key = (static_cast<unsigned long long>(w) << 5) | b;
    const uint32_t axis = static_cast<uint32_t>(key % 3ull);
    const unsigned long long stored = key / 3ull;
    const uint32_t slot = static_cast<uint32_t>(stored >> 9), local = static_cast<uint32_t>(stored & 511ull);
    const uint32_t block = slot_block != nullptr ? slot_block[slot] : slot;
    const uint32_t nx = (block % v.bx) * 8u + (local & 7u), ny = ((block / v.bx) % v.by) * 8u + ((local >> 3) & 7u),
                   nz = (block / (v.bx * v.by)) * 8u + (local >> 6);
    const uint32_t fx = nx + (axis == 0), fy = ny + (axis == 1), fz = nz + (axis == 2);
    const float near_value = VT::tsdf(__ldg(voxels + storage_index(v, nx, ny, nz)));
    const float far_value = VT::tsdf(__ldg(voxels + storage_index(v, fx, fy, fz)));
    const f3 near_point = cell_center(v, nx, ny, nz);
    const f3 far_point = cell_center(v, fx, fy, fz);
    const float fraction = -near_value / (far_value - near_value);
    const f3 position = near_point + ((far_point - near_point) * fraction);
    f3 normal;
    if (!s.central_normal(position, KF_CORNERS_SKIP_MISSING, normal)) normal = make(0.0f, 0.0f, 0.0f);
    f3 color;
    if (!s.color(position, color)) color = make(255.0f, 255.0f, 255.0f);
    const uint32_t p = first_use[id];
    const uint32_t vi = use_first[p >> 5] + __popc(use_words[p >> 5] & ((1u << (p & 31u)) - 1u));
    store3(positions + static_cast<size_t>(vi) * 3, position);
    store3(normals + static_cast<size_t>(vi) * 3, normal);
    store3(colors + static_cast<size_t>(vi) * 3, color);
    vertex_of[id] = vi;
    ++id;
  }
}

__global__ void mc_triangle_kernel(const uint32_t* __restrict__ corner_edge, const uint32_t* __restrict__ vertex_of,
                                   uint32_t* __restrict__ triangles, uint32_t corners) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < corners) triangles[q] = vertex_of[corner_edge[q]];
}

// MeshBuilder::fill_missing_normals (marching_cubes.cpp:441-456), in
// triangle order with the host builder's float arithmetic.
void fill_missing_normals(kf_mesh& m) {
  std::vector<uint8_t> missing(m.vertex_count);
  std::vector<float> acc(m.vertex_count * 3, 0.0f);
  for (uint64_t i = 0; i < m.vertex_count; ++i) {
    missing[i] = m.normals[i * 3] == 0.0f && m.normals[i * 3 + 1] == 0.0f && m.normals[i * 3 + 2] == 0.0f;
  }
  for (uint64_t t = 0; t < m.triangle_count; ++t) {
    const uint32_t* tr = m.triangles + t * 3;
    const float* p0 = m.positions + static_cast<size_t>(tr[0]) * 3;
    const float* p1 = m.positions + static_cast<size_t>(tr[1]) * 3;
    const float* p2 = m.positions + static_cast<size_t>(tr[2]) * 3;
    const float a[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    const float b[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    const float face[3] = {(a[1] * b[2]) - (a[2] * b[1]), (a[2] * b[0]) - (a[0] * b[2]), (a[0] * b[1]) - (a[1] * b[0])};
    for (int k = 0; k < 3; ++k) {
      if (!missing[tr[k]]) continue;
      float* s = acc.data() + static_cast<size_t>(tr[k]) * 3;
      s[0] = s[0] + face[0];
      s[1] = s[1] + face[1];
      s[2] = s[2] + face[2];
    }
  }
  for (uint64_t i = 0; i < m.vertex_count; ++i) {
    if (!missing[i]) continue;
    const float* s = acc.data() + i * 3;
    const float length = std::sqrt((s[0] * s[0]) + (s[1] * s[1]) + (s[2] * s[2]));
    float* n = m.normals + i * 3;
    if (length > 0.0f) {
      n[0] = s[0] / length;
      n[1] = s[1] / length;
      n[2] = s[2] / length;
    } else {
      n[0] = n[1] = n[2] = 0.0f;
    }
  }
}

template <int Kind>
void extract_typed(Pipeline& p, float min_weight, kf_mesh& out, cudaStream_t s) {
  const VolumeDev& v = p.view;
  const bool sparse = v.table != nullptr;
  // edge keys: storage index of the near voxel * 3 + axis
  const unsigned long long keys = static_cast<unsigned long long>(p.voxel_count) * 3ull;
  const unsigned long long words64 = (keys + 31ull) / 32ull;
  if (words64 > 0xFFFFFFFFull) throw Unsupported("volume too large for the device mesher");
  const uint32_t words = static_cast<uint32_t>(words64);
  const uint4* stencil = p.brick_class.count ? reinterpret_cast<const uint4*>(p.stencil_bits.ptr) : nullptr;

  // units: rows of cells (dense) or allocated blocks in block order (sparse)
  uint32_t units = (v.ry - 1) * (v.rz - 1);
  DeviceArray<uint32_t> block_list;
  if (sparse) {
    const uint32_t blocks = v.bx * v.by * v.bz;
    DeviceArray<uint32_t> flags(blocks), position(blocks);
    check(cudaMemsetAsync(flags.ptr, 0, flags.bytes(), s), "allocated flags");
    allocated_flags_kernel<<<148 * 4, 256, 0, s>>>(p.slot_block.ptr, p.allocated.ptr, p.sparse_capacity, flags.ptr);
    check(cudaGetLastError(), "allocated_flags_kernel launch");
    units = exclusive_scan(flags.ptr, position.ptr, blocks, false, s);
    if (units == 0) return;
    block_list.resize(units);
    allocated_list_kernel<<<ceil_div(blocks, 256), 256, 0, s>>>(flags.ptr, position.ptr, blocks, block_list.ptr);
    check(cudaGetLastError(), "allocated_list_kernel launch");
  }
  DeviceArray<uint32_t> edge_words(words), word_first(words), unit_tris(units), unit_first(units);
  check(cudaMemsetAsync(edge_words.ptr, 0, edge_words.bytes(), s), "mesh edge bits");
  if (sparse) {
    mc_blocks_kernel<Kind, false><<<units, 512, 0, s>>>(v, block_list.ptr, min_weight, edge_words.ptr,
                                                         unit_tris.ptr, nullptr, nullptr, nullptr, nullptr);
  } else {
    mc_rows_kernel<Kind, false><<<units, kRowThreads, 0, s>>>(v, stencil, min_weight, edge_words.ptr, unit_tris.ptr,
                                                              nullptr, nullptr, nullptr, nullptr);
  }
  check(cudaGetLastError(), "mesh cell pass launch");
  const uint32_t triangles = exclusive_scan(unit_tris.ptr, unit_first.ptr, units, false, s);
  const uint32_t vertices = exclusive_scan(edge_words.ptr, word_first.ptr, words, true, s);
  if (triangles == 0 || vertices == 0) return;
  if (static_cast<unsigned long long>(triangles) * 3ull > 0xFFFFFFFFull) throw Unsupported("mesh too large");
  const uint32_t corners = triangles * 3u;
  DeviceArray<uint32_t> corner_edge(corners), first_use(vertices), vertex_of(vertices), tris(corners);
  check(cudaMemsetAsync(first_use.ptr, 0xFF, first_use.bytes(), s), "mesh first use");
  if (sparse) {
    mc_blocks_kernel<Kind, true><<<units, 512, 0, s>>>(v, block_list.ptr, min_weight, edge_words.ptr, nullptr,
                                                        unit_first.ptr, word_first.ptr, corner_edge.ptr,
                                                        first_use.ptr);
  } else {
    mc_rows_kernel<Kind, true><<<units, kRowThreads, 0, s>>>(v, stencil, min_weight, edge_words.ptr, nullptr,
                                                             unit_first.ptr, word_first.ptr, corner_edge.ptr,
                                                             first_use.ptr);
  }
  check(cudaGetLastError(), "mesh corner pass launch");
  const uint32_t use_words_n = ceil_div(corners, 32u);
  DeviceArray<uint32_t> use_words(use_words_n), use_first(use_words_n);
  check(cudaMemsetAsync(use_words.ptr, 0, use_words.bytes(), s), "mesh use bits");
  mark_first_use_kernel<<<ceil_div(vertices, 256), 256, 0, s>>>(first_use.ptr, use_words.ptr, vertices);
  check(cudaGetLastError(), "mark_first_use_kernel launch");
  exclusive_scan(use_words.ptr, use_first.ptr, use_words_n, true, s);
  DeviceArray<float> positions(static_cast<size_t>(vertices) * 3), normals(static_cast<size_t>(vertices) * 3),
      colors(static_cast<size_t>(vertices) * 3);
  mc_vertex_kernel<Kind><<<ceil_div(words, 256), 256, 0, s>>>(
      v, sparse ? p.slot_block.ptr : nullptr, edge_words.ptr, word_first.ptr, first_use.ptr, use_words.ptr,
      use_first.ptr, words, positions.ptr, normals.ptr, colors.ptr, vertex_of.ptr);
  check(cudaGetLastError(), "mc_vertex_kernel launch");
  mc_triangle_kernel<<<ceil_div(corners, 256), 256, 0, s>>>(corner_edge.ptr, vertex_of.ptr, tris.ptr, corners);
  check(cudaGetLastError(), "mc_triangle_kernel launch");
  // host copies
  out.vertex_count = vertices;
  out.triangle_count = triangles;
  out.positions = static_cast<float*>(std::malloc(positions.bytes()));
  out.normals = static_cast<float*>(std::malloc(normals.bytes()));
  out.colors = static_cast<float*>(std::malloc(colors.bytes()));
  out.triangles = static_cast<uint32_t*>(std::malloc(tris.bytes()));
  if (!out.positions || !out.normals || !out.colors || !out.triangles) throw CudaError("host allocation failed");
  check(cudaMemcpyAsync(out.positions, positions.ptr, positions.bytes(), cudaMemcpyDeviceToHost, s), "mesh copy");
  check(cudaMemcpyAsync(out.normals, normals.ptr, normals.bytes(), cudaMemcpyDeviceToHost, s), "mesh copy");
  check(cudaMemcpyAsync(out.colors, colors.ptr, colors.bytes(), cudaMemcpyDeviceToHost, s), "mesh copy");
  check(cudaMemcpyAsync(out.triangles, tris.ptr, tris.bytes(), cudaMemcpyDeviceToHost, s), "mesh copy");
  check(cudaStreamSynchronize(s), "mesh copy");
  fill_missing_normals(out);
}

void upload_tables() {
  check(cudaMemcpyToSymbol(c_edge_mask, kMcEdgeMask, sizeof(kMcEdgeMask)), "mesh tables");
  check(cudaMemcpyToSymbol(c_triangles, kMcTriangles, sizeof(kMcTriangles)), "mesh tables");
  check(cudaMemcpyToSymbol(c_corner, kMcCorner, sizeof(kMcCorner)), "mesh tables");
  check(cudaMemcpyToSymbol(c_edge, kMcEdge, sizeof(kMcEdge)), "mesh tables");
}

}  // namespace

void extract_mesh(Pipeline& p, float min_weight, kf_mesh& out) {
  std::memset(&out, 0, sizeof(out));
  if (p.view.rx < 2 || p.view.ry < 2 || p.view.rz < 2) return;
  upload_tables();
  const cudaStream_t s = p.stream;
  try {
    switch (p.config.voxel) {
      case KF_VOXEL_QUANTIZED:
        extract_typed<KF_VOXEL_QUANTIZED>(p, min_weight, out, s);
        break;
      case KF_VOXEL_BF16:
        extract_typed<KF_VOXEL_BF16>(p, min_weight, out, s);
        break;
      default:
        extract_typed<KF_VOXEL_FLOAT>(p, min_weight, out, s);
        break;
    }
  } catch (...) {
    std::free(out.positions);
    std::free(out.normals);
    std::free(out.colors);
    std::free(out.triangles);
    std::memset(&out, 0, sizeof(out));
    throw;
  }
}

}  // namespace kf
