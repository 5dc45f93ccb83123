// kf_gemm.cu - bf16 GEMM on the 5th-generation tensor cores (tcgen05), the
// matrix engine of the learned ICP warm-start (no counterpart in the
// reference).
//
//   C[M x N] (fp32) = A[M x K] (bf16, row-major) * B[N x K]^T (bf16, row-major)
//                     (+ bias[N]) (ReLU)
//
// One CTA of 128 threads computes a 128 x BN tile of C.  The A and B tiles
// move by TMA (cp.async.bulk.tensor, 128-byte swizzle: one 64-element K slab
// of a row is one 128-byte line) into a ring of kStages shared-memory stages.
// Warp 1 issues the copies, warp 0 the tcgen05.mma.kind::f16 (M = 128,
// N = BN, K = 16, FP32 accumulator in tensor memory): a stage's "full"
// mbarrier completes when its bytes have landed, its "empty" mbarrier when
// the MMAs reading it are done (tcgen05.commit), so the copies run up to
// kStages slabs ahead of the tensor core.  The epilogue reads the accumulator with
// tcgen05.ld (each warp its 32 TMEM lanes = 32 rows of the tile).  Every wait
// is bounded: past the limit the kernel records an error, waits (bounded) for
// its own MMAs, frees its tensor memory and returns.
#include <cuda.h>  // CUtensorMap and its enums (the encoder comes through the runtime)
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>

#include "kf_internal.h"

namespace kf {
namespace {

constexpr int kGemmThreads = 128;
constexpr int kGemmBM = 128;
constexpr int kGemmBK = 64;
constexpr unsigned long long kWaitCycles = 2000000000ull;  // ~1 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Stages per tile width: at most about 97 KB of stages, two CTAs per SM.
template <int BN>
constexpr int stages_for() {
  return BN >= 256 ? 2 : 3;
}
constexpr int kGroupM = 16;  // row tiles per group of the CTA order

// Shared-memory matrix descriptor of a K-major operand in the 128-byte
// swizzle layout TMA writes: rows of 128 bytes (one 64-element K slab),
// 8-row groups 1024 bytes apart (SBO), version 1 (sm_100) at bit 46, layout
// type SWIZZLE_128B (2) at bits 61-63.  The K step of 16 elements (32 bytes)
// inside the swizzle atom moves the start address.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>(1u) << 16;              // leading byte offset: unused by swizzled K-major
  d |= static_cast<uint64_t>((1024u >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;
  d |= 2ull << 61;
  return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t m, uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  const unsigned long long start = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (done) return true;
    if (clock64() - start > kWaitCycles) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

template <int BN>
constexpr size_t gemm_smem_bytes() {
  return static_cast<size_t>(stages_for<BN>()) * (kGemmBM + BN) * kGemmBK * 2u + 1024u;  // + alignment slack
}

// One CTA computes a 128 x BN tile of C over the K slabs [blockIdx.z * slabs,
// (blockIdx.z + 1) * slabs).  With gridDim.z == 1 the epilogue adds the bias
// and applies the ReLU into C; otherwise it stores the raw partial tile into
// C + blockIdx.z * M * ldc (split K, summed by gemm_splitk_reduce_kernel).
// TMA coordinates: x = the K element (a multiple of 64, so 128-byte aligned),
// y = the row; rows and K past the matrix read as zeros.
template <int BN>
__global__ void __launch_bounds__(kGemmThreads)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                     float* __restrict__ C, int M, int N, int K, int ldc, const float* __restrict__ bias, int relu,
                     int slabs, int gm, int gn, int* __restrict__ error) {
  constexpr uint32_t kCols = BN < 32 ? 32 : BN;  // tensor-memory columns (a power of two >= 32)
  constexpr uint32_t kStageA = kGemmBM * kGemmBK * 2, kStageB = BN * kGemmBK * 2;
  constexpr uint32_t kStageBytes = kStageA + kStageB;  // a multiple of 1024 for every BN
  constexpr int kStages = stages_for<BN>();
  extern __shared__ uint8_t s_dyn[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(s_dyn) + 1023u) & ~uintptr_t(1023u));
  __shared__ __align__(8) unsigned long long s_full[3], s_empty[3], s_done;
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // Grouped tile order: consecutive CTAs walk kGroupM row tiles down one
  // column tile before moving right, so a wave of CTAs shares its A rows and
  // B columns in L2 instead of streaming all of A once per column of tiles.
  const int id = static_cast<int>(blockIdx.x);
  const int per_group = kGroupM * gn;
  const int first_m = (id / per_group) * kGroupM;
  const int group_rows = min(gm - first_m, kGroupM);
  const int tile_m = (first_m + (id % per_group) % group_rows) * kGemmBM;
  const int tile_n = ((id % per_group) / group_rows) * BN;
  const int total_slabs = (K + kGemmBK - 1) / kGemmBK;
  const int slab0 = blockIdx.z * slabs;
  const int nslabs = min(slabs, total_slabs - slab0);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int st = 0; st < kStages; ++st) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_full[st])), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_empty[st])), "r"(1));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_done)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_a)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_b)) : "memory");
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s_tmem;
  const uint32_t idesc = instr_desc(kGemmBM, BN);

  if (nslabs > 0 && tid == 32) {
    // producer (warp 1): refill a stage once the MMAs that read it are done
    for (int i = 0; i < nslabs; ++i) {
      const int st = i % kStages;
      if (i >= kStages &&
          !mbar_wait(smem_u32(&s_empty[st]), static_cast<uint32_t>(((i - kStages) / kStages) & 1))) {
        s_fail = 1;
        break;
      }
      const uint32_t full = smem_u32(&s_full[st]);
      const uint32_t dst = smem_u32(base + st * kStageBytes);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(full), "r"(kStageBytes)
                   : "memory");
      const int k0 = (slab0 + i) * kGemmBK;
      tma_load_2d(dst, &map_a, k0, tile_m, full);
      tma_load_2d(dst + kStageA, &map_b, k0, tile_n, full);
    }
  } else if (nslabs > 0 && tid == 0) {
    // MMA issuer (warp 0): one slab's four MMAs per full stage
    for (int j = 0; j < nslabs; ++j) {
      const int st = j % kStages;
      if (!mbar_wait(smem_u32(&s_full[st]), static_cast<uint32_t>((j / kStages) & 1))) {
        s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = smem_u32(base + st * kStageBytes), b0 = a0 + kStageA;
#pragma unroll
      for (int kk = 0; kk < kGemmBK / 16; ++kk) {
        const uint64_t da = smem_desc_sw128(a0 + kk * 32);
        const uint64_t db = smem_desc_sw128(b0 + kk * 32);
        const uint32_t accumulate = (j > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   ::"r"(smem_u32(&s_empty[st]))
                   : "memory");
    }
    // arrives once every MMA issued before it is complete
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(&s_done))
                 : "memory");
  }
  __syncthreads();
  bool ok = s_fail == 0;
  if (nslabs > 0) ok = __syncthreads_and(mbar_wait(smem_u32(&s_done), 0u)) && ok;
  if (!ok) {
    if (tid == 0) atomicExch(error, 1);
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;");
    const bool split = gridDim.z > 1;
    float* out = C + (split ? static_cast<size_t>(blockIdx.z) * M * ldc : 0u);
    const int row = tile_m + warp * 32 + lane;
#pragma unroll
    for (int c = 0; c < BN; c += 16) {
      uint32_t r[16];
      const uint32_t addr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(addr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = tile_n + c + j;
          if (col >= N) continue;
          float v = nslabs > 0 ? __uint_as_float(r[j]) : 0.0f;
          if (!split) {
            if (bias != nullptr) v += bias[col];
            if (relu && v < 0.0f) v = 0.0f;
          }
          out[static_cast<size_t>(row) * ldc + col] = v;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// C = sum over the split partials (in split order) (+ bias) (ReLU).
__global__ void gemm_splitk_reduce_kernel(const float* __restrict__ partial, int splits, int M, int N, int ldp,
                                          float* __restrict__ C, int ldc, const float* __restrict__ bias, int relu) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<size_t>(M) * N) return;
  const int row = static_cast<int>(i / N), col = static_cast<int>(i % N);
  float v = 0.0f;
  for (int z = 0; z < splits; ++z) v += partial[(static_cast<size_t>(z) * M + row) * ldp + col];
  if (bias != nullptr) v += bias[col];
  if (relu && v < 0.0f) v = 0.0f;
  C[static_cast<size_t>(row) * ldc + col] = v;
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    check(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q), "tensor map encoder");
    require(q == cudaDriverEntryPointSuccess && p != nullptr, "gemm: the driver has no cuTensorMapEncodeTiled");
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

// A rows x K bf16 row-major matrix (leading dimension ld) read in boxes of
// 64 K elements x box_rows rows, 128-byte swizzle, zeros outside.
CUtensorMap tensor_map(const void* base, int rows, int K, int ld, int box_rows) {
  CUtensorMap map;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(K), static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * 2u};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(kGemmBK), static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t elem[2] = {1u, 1u};
  const CUresult r = encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box,
                               elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  require(r == CUDA_SUCCESS, "gemm: tensor map encoding failed");
  return map;
}

template <int BN>
void launch_tiles(const __nv_bfloat16* a, const __nv_bfloat16* b, float* c, int M, int N, int K, int lda, int ldb,
                  int ldc, const float* bias, int relu, int slabs, unsigned splits, int* error, cudaStream_t s) {
  static bool configured = false;  // per process: every device gets the same attribute
  if (!configured) {
    check(cudaFuncSetAttribute(gemm_bf16_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(gemm_smem_bytes<BN>())),
          "gemm attribute");
    configured = true;
  }
  const CUtensorMap ma = tensor_map(a, M, K, lda, kGemmBM);
  const CUtensorMap mb = tensor_map(b, N, K, ldb, BN);
  const unsigned gm = ceil_div(static_cast<unsigned>(M), static_cast<unsigned>(kGemmBM));
  const unsigned gn = ceil_div(static_cast<unsigned>(N), static_cast<unsigned>(BN));
  gemm_bf16_kernel<BN><<<dim3(gm * gn, 1, splits), kGemmThreads, gemm_smem_bytes<BN>(), s>>>(
      ma, mb, c, M, N, K, ldc, bias, relu, slabs, static_cast<int>(gm), static_cast<int>(gn), error);
}

}  // namespace

void launch_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K, int lda, int ldb, int ldc,
                      const float* bias, int relu, int* error, cudaStream_t s, float* workspace,
                      size_t workspace_floats) {
  require(M > 0 && N > 0 && K > 0, "gemm: empty shape");
  require(lda % 8 == 0 && ldb % 8 == 0 && K % 8 == 0, "gemm: K and the leading dimensions must be multiples of 8");
  require(reinterpret_cast<uintptr_t>(A) % 16 == 0 && reinterpret_cast<uintptr_t>(B) % 16 == 0,
          "gemm: operands must be 16-byte aligned");
  const auto* a = static_cast<const __nv_bfloat16*>(A);
  const auto* b = static_cast<const __nv_bfloat16*>(B);
  // 256-wide tiles halve the A traffic per flop, but only pay when there are
  // enough of them to fill the GPU twice over; small products keep 128
  const unsigned wide_tiles = ceil_div(static_cast<unsigned>(M), static_cast<unsigned>(kGemmBM)) *
                              ceil_div(static_cast<unsigned>(N), 256u);
  const int bn = N <= 16 ? 16 : (N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 || wide_tiles < 296u ? 128 : 256)));
  const unsigned tiles = ceil_div(static_cast<unsigned>(M), static_cast<unsigned>(kGemmBM)) *
                         ceil_div(static_cast<unsigned>(N), static_cast<unsigned>(bn));
  const int total_slabs = (K + kGemmBK - 1) / kGemmBK;
  // split K when the tiles leave most SMs idle and each split keeps >= 8 slabs
  unsigned splits = 1;
  if (workspace != nullptr && tiles < 148u && total_slabs >= 16) {
    splits = std::min<unsigned>(ceil_div(296u, tiles), static_cast<unsigned>(total_slabs / 8));
    splits = std::min<unsigned>(splits, static_cast<unsigned>(workspace_floats / (static_cast<size_t>(M) * N)));
    if (splits < 2) splits = 1;
  }
  const int slabs = (total_slabs + static_cast<int>(splits) - 1) / static_cast<int>(splits);
  splits = static_cast<unsigned>((total_slabs + slabs - 1) / slabs);  // no empty split
  float* out = splits > 1 ? workspace : C;
  const int ldo = splits > 1 ? N : ldc;
  switch (bn) {
    case 16: launch_tiles<16>(a, b, out, M, N, K, lda, ldb, ldo, bias, relu, slabs, splits, error, s); break;
    case 32: launch_tiles<32>(a, b, out, M, N, K, lda, ldb, ldo, bias, relu, slabs, splits, error, s); break;
    case 64: launch_tiles<64>(a, b, out, M, N, K, lda, ldb, ldo, bias, relu, slabs, splits, error, s); break;
    case 128: launch_tiles<128>(a, b, out, M, N, K, lda, ldb, ldo, bias, relu, slabs, splits, error, s); break;
    default: launch_tiles<256>(a, b, out, M, N, K, lda, ldb, ldo, bias, relu, slabs, splits, error, s); break;
  }
  check(cudaGetLastError(), "gemm_bf16_kernel launch");
  if (splits > 1) {
    const size_t n = static_cast<size_t>(M) * N;
    gemm_splitk_reduce_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(workspace, static_cast<int>(splits),
                                                                                  M, N, N, C, ldc, bias, relu);
    check(cudaGetLastError(), "gemm_splitk_reduce_kernel launch");
  }
}

}  // namespace kf

namespace {
// Per-process scratch of kf_gemm_bf16, allocated on the first call that
// needs it and kept: the error flag and the split-K partials.  Calls are
// serialised by the lock (each call waits for its GEMM anyway).
struct GemmScratch {
  std::mutex lock;
  int device = -1;
  kf::DeviceArray<int> error;
  kf::DeviceArray<float> workspace;
};
GemmScratch& gemm_scratch() {
  static GemmScratch* s = new GemmScratch();  // never destroyed: lives past static teardown
  return *s;
}
}  // namespace

extern "C" kf_status kf_gemm_bf16(const void* a, const void* b, float* c, int32_t m, int32_t n, int32_t k,
                                  const float* bias, int32_t relu, void* stream) {
  return kf::guarded([&] {
    kf::require(a != nullptr && b != nullptr && c != nullptr, "kf_gemm_bf16: null argument");
    GemmScratch& g = gemm_scratch();
    std::lock_guard<std::mutex> hold(g.lock);
    int device = 0;
    kf::check(cudaGetDevice(&device), "gemm device");
    if (g.device != device) {  // another device: start over (the arrays belong to the old one)
      g.error = kf::DeviceArray<int>();
      g.workspace = kf::DeviceArray<float>();
      g.device = device;
    }
    if (g.error.count == 0) g.error.resize(1);
    // split-K partials for GEMMs of few output tiles (at most 16 MB)
    const size_t want = std::min<size_t>(static_cast<size_t>(m) * n * 64, size_t{1} << 22);
    const unsigned tiles = kf::ceil_div(static_cast<unsigned>(m), 128u) * kf::ceil_div(static_cast<unsigned>(n), 16u);
    if (tiles < 148u * 8u && g.workspace.count < want) g.workspace.resize(want);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    kf::check(cudaMemsetAsync(g.error.ptr, 0, sizeof(int), s), "gemm error flag");
    kf::launch_gemm_bf16(a, b, c, m, n, k, k, k, n, bias, relu, g.error.ptr, s, g.workspace.ptr, g.workspace.count);
    int flag = 0;
    kf::check(cudaMemcpyAsync(&flag, g.error.ptr, sizeof(int), cudaMemcpyDeviceToHost, s), "gemm error flag");
    kf::check(cudaStreamSynchronize(s), "gemm");
    if (flag) throw kf::CudaError("kf_gemm_bf16: tensor-core wait timed out");
  });
}
