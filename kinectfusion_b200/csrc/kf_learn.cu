// kf_learn.cu - the learned ICP warm start (no counterpart in the reference).
//
// A small CNN reads two 60 x 80 maps - the current depth at 1/8 resolution
// and the model depth rendered at the constant-velocity pose - and proposes
// the SE(3) twist from that pose to the tracked pose.  Every layer is a GEMM
// on the tcgen05 tensor cores (kf_gemm.cu): the convolutions as im2col GEMMs,
// forward and backward, with bf16 operands and FP32 accumulation; ReLU and
// bias ride in the GEMM epilogue; transposes, col2im, the loss and Adam are
// plain CUDA kernels.  Activations are NHWC: row (b, y, x), column channel.
//
//   conv1  2 -> 32, 3x3 stride 2 pad 1: 60x80 -> 30x40  (im2col width 18, padded to 24)
//   conv2 32 -> 32:                      30x40 -> 15x20  (288)
//   conv3 32 -> 64:                      15x20 ->  8x10  (288)
//   conv4 64 -> 64:                       8x10 ->  4x5   (576)
//   fc1  1280 -> 256, ReLU;  fc2  256 -> 6 (the twist, scaled)
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <random>
#include <vector>

#include "kf_internal.h"

namespace kf {
namespace {

struct Conv {
  int cin, cout, hin, win, hout, wout, k, kpad;
};
constexpr Conv kConv[4] = {{2, 32, 60, 80, 30, 40, 18, 24},
                           {32, 32, 30, 40, 15, 20, 288, 288},
                           {32, 64, 15, 20, 8, 10, 288, 288},
                           {64, 64, 8, 10, 4, 5, 576, 576}};
constexpr int kFlat = 64 * 4 * 5;  // 1280
constexpr int kHidden = 256;
constexpr int kOut = 6;
constexpr int kOutPad = 8;  // K of the twist layer's input-gradient GEMM

// Offsets of each tensor in the flat FP32 parameter vector: per layer the
// weights [rows][cols] then the bias, every offset a multiple of 8 floats.
struct Layout {
  size_t w[6], b[6], total;
  int rows[6], cols[6];
};
Layout layout() {
  Layout l{};
  size_t off = 0;
  for (int i = 0; i < 6; ++i) {
    l.rows[i] = i < 4 ? kConv[i].cout : (i == 4 ? kHidden : kOut);
    l.cols[i] = i < 4 ? kConv[i].kpad : (i == 4 ? kFlat : kHidden);
    l.w[i] = off;
    off += static_cast<size_t>(l.rows[i]) * l.cols[i];
    l.b[i] = off;
    off += (l.rows[i] + 7) / 8 * 8;
  }
  l.total = off;
  return l;
}

unsigned blocks_for(size_t n) { return static_cast<unsigned>((n + 255) / 256); }

// ---- small kernels ----------------------------------------------------------
// im2col of an NHWC bf16 map: row (b, oy, ox), column c*9 + ky*3 + kx (zero
// outside the image and in the columns past k).
__global__ void im2col_kernel(const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ col, int batch,
                              Conv c) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const size_t total = static_cast<size_t>(batch) * c.hout * c.wout * c.kpad;
  if (i >= total) return;
  const int kk = static_cast<int>(i % c.kpad);
  const size_t row = i / c.kpad;
  const int ox = static_cast<int>(row % c.wout), oy = static_cast<int>((row / c.wout) % c.hout);
  const int b = static_cast<int>(row / (static_cast<size_t>(c.wout) * c.hout));
  __nv_bfloat16 v = __float2bfloat16(0.0f);
  if (kk < c.k) {
    const int ch = kk / 9, ky = (kk / 3) % 3, kx = kk % 3;
    const int y = oy * 2 - 1 + ky, xx = ox * 2 - 1 + kx;
    if (y >= 0 && y < c.hin && xx >= 0 && xx < c.win) {
      v = x[((static_cast<size_t>(b) * c.hin + y) * c.win + xx) * c.cin + ch];
    }
  }
  col[i] = v;
}

// col2im in gather form (one thread per input element, fixed order): dx = the
// sum of dcol over the output positions whose 3x3 window holds the element.
__global__ void col2im_kernel(const float* __restrict__ dcol, float* __restrict__ dx, int batch, Conv c) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const size_t total = static_cast<size_t>(batch) * c.hin * c.win * c.cin;
  if (i >= total) return;
  const int ch = static_cast<int>(i % c.cin);
  const size_t p = i / c.cin;
  const int x = static_cast<int>(p % c.win), y = static_cast<int>((p / c.win) % c.hin);
  const int b = static_cast<int>(p / (static_cast<size_t>(c.win) * c.hin));
  float s = 0.0f;
  for (int ky = 0; ky < 3; ++ky) {
    const int ty = y + 1 - ky;
    if (ty < 0 || (ty & 1)) continue;
    const int oy = ty / 2;
    if (oy >= c.hout) continue;
    for (int kx = 0; kx < 3; ++kx) {
      const int tx = x + 1 - kx;
      if (tx < 0 || (tx & 1)) continue;
      const int ox = tx / 2;
      if (ox >= c.wout) continue;
      s += dcol[((static_cast<size_t>(b) * c.hout + oy) * c.wout + ox) * c.kpad + ch * 9 + ky * 3 + kx];
    }
  }
  dx[i] = s;
}

__global__ void to_bf16_kernel(const float* __restrict__ in, __nv_bfloat16* __restrict__ out, size_t n) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __float2bfloat16(in[i]);
}

// out[c][r] = bf16(in[r][c]) for an R x C fp32 matrix (leading dimension
// in_ld); rows r >= R of each output line (up to out_ld) are zero.
__global__ void transpose_bf16_kernel(const float* __restrict__ in, int rows, int cols, int in_ld,
                                      __nv_bfloat16* __restrict__ out, int out_ld) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<size_t>(cols) * out_ld) return;
  const int r = static_cast<int>(i % out_ld), c = static_cast<int>(i / out_ld);
  out[i] = __float2bfloat16(r < rows ? in[static_cast<size_t>(r) * in_ld + c] : 0.0f);
}

// the same for a bf16 matrix
__global__ void transpose_bf16_bf16_kernel(const __nv_bfloat16* __restrict__ in, int rows, int cols, int in_ld,
                                           __nv_bfloat16* __restrict__ out, int out_ld) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<size_t>(cols) * out_ld) return;
  const int r = static_cast<int>(i % out_ld), c = static_cast<int>(i / out_ld);
  out[i] = r < rows ? in[static_cast<size_t>(r) * in_ld + c] : __float2bfloat16(0.0f);
}

// dz = dy where the layer's ReLU output was positive, else 0 (in place)
__global__ void relu_back_kernel(float* __restrict__ dy, const float* __restrict__ a, size_t n) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n && !(a[i] > 0.0f)) dy[i] = 0.0f;
}

// Column sums of an R x C fp32 matrix (bias gradients) in two fixed-order
// stages: CTA (x, y) sums rows [256 y, 256 y + 256) of columns [32 x, 32 x +
// 32) into partial[y][c]; colsum_finish adds the partials in order.
constexpr int kColsumRows = 256;
__global__ void colsum_partial_kernel(const float* __restrict__ m, int rows, int cols, float* __restrict__ partial) {
  __shared__ float s[8][33];
  const int c = blockIdx.x * 32 + threadIdx.x;
  const int r0 = blockIdx.y * kColsumRows;
  float acc = 0.0f;
  if (c < cols) {
    const int r1 = min(rows, r0 + kColsumRows);
    for (int r = r0 + threadIdx.y; r < r1; r += 8) acc += m[static_cast<size_t>(r) * cols + c];
  }
  s[threadIdx.y][threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.y == 0 && c < cols) {
    float t = 0.0f;
    for (int j = 0; j < 8; ++j) t += s[j][threadIdx.x];
    partial[static_cast<size_t>(blockIdx.y) * cols + c] = t;
  }
}
__global__ void colsum_finish_kernel(const float* __restrict__ partial, int chunks, int cols, float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float t = 0.0f;
  for (int j = 0; j < chunks; ++j) t += partial[static_cast<size_t>(j) * cols + c];
  out[c] = t;
}

// d_out = 2 (out - target) / B into a B x 8 matrix (columns 6, 7 zero); the
// loss (the batch mean of the squared error) into loss[0].  One CTA of 256.
__global__ void loss_kernel(const float* __restrict__ out, const float* __restrict__ target, int batch,
                            float* __restrict__ d_out, float* __restrict__ loss) {
  __shared__ float s_sum[256];
  float acc = 0.0f;
  for (int i = threadIdx.x; i < batch * kOutPad; i += blockDim.x) {
    const int b = i / kOutPad, j = i % kOutPad;
    float g = 0.0f;
    if (j < kOut) {
      const float e = out[b * kOut + j] - target[b * kOut + j];
      acc += e * e;
      g = 2.0f * e / static_cast<float>(batch);
    }
    d_out[i] = g;
  }
  s_sum[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) s_sum[threadIdx.x] += s_sum[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss[0] = s_sum[0] / static_cast<float>(batch);
}

// Adam (Kingma & Ba 2015) on the flat parameter vector; c1, c2 are the bias
// corrections 1 - beta^t.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace

// ---- the learner -----------------------------------------------------------
struct Learner {
  Layout lay = layout();
  int capacity = 0;  // largest batch
  DeviceArray<float> params, grads, adam_m, adam_v;
  DeviceArray<__nv_bfloat16> wbf;   // bf16 weights [rows][cols] per layer (the forward GEMMs' B)
  DeviceArray<__nv_bfloat16> wtbf;  // bf16 transposed weights [cols][rows_pad] (the input-gradient GEMMs' B)
  size_t wt_off[6] = {};
  int rows_pad[6] = {};
  DeviceArray<__nv_bfloat16> col[4], xbf[6], t_a, t_b;
  DeviceArray<float> act[5], dact[5], dcol, dout8, loss, out, partial;
  DeviceArray<float> workspace;  // split-K partials of the weight-gradient GEMMs
  DeviceArray<int> error;
  int steps = 0;

  void init(int batch, uint32_t seed) {
    capacity = batch;
    params.resize(lay.total);
    grads.resize(lay.total);
    adam_m.resize(lay.total);
    adam_v.resize(lay.total);
    wbf.resize(lay.total);
    size_t wt = 0;
    for (int i = 0; i < 6; ++i) {
      rows_pad[i] = (lay.rows[i] + 7) / 8 * 8;
      wt_off[i] = wt;
      wt += static_cast<size_t>(lay.cols[i]) * rows_pad[i];
    }
    wtbf.resize(wt);
    // He-uniform weights (zero in conv1's padded columns; the last layer
    // scaled by 0.1), zero biases
    std::vector<float> h(lay.total, 0.0f);
    std::mt19937 rng(seed);
    for (int i = 0; i < 6; ++i) {
      const int fan_in = i < 4 ? kConv[i].k : lay.cols[i];
      const float bound = std::sqrt(6.0f / static_cast<float>(fan_in)) * (i == 5 ? 0.1f : 1.0f);
      std::uniform_real_distribution<float> u(-bound, bound);
      for (int r = 0; r < lay.rows[i]; ++r) {
        for (int c = 0; c < lay.cols[i]; ++c) {
          const bool real = i >= 4 || c < kConv[i].k;
          h[lay.w[i] + static_cast<size_t>(r) * lay.cols[i] + c] = real ? u(rng) : 0.0f;
        }
      }
    }
    check(cudaMemcpy(params.ptr, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice), "learner init");
    check(cudaMemset(adam_m.ptr, 0, adam_m.bytes()), "learner init");
    check(cudaMemset(adam_v.ptr, 0, adam_v.bytes()), "learner init");
    size_t dcol_max = static_cast<size_t>(batch) * kFlat, t_max = static_cast<size_t>(batch) * kFlat;
    for (int i = 0; i < 4; ++i) {
      const Conv& c = kConv[i];
      const size_t rows = static_cast<size_t>(batch) * c.hout * c.wout;
      col[i].resize(rows * c.kpad);
      act[i].resize(rows * c.cout);
      dact[i].resize(rows * c.cout);
      xbf[i].resize(static_cast<size_t>(batch) * c.hin * c.win * c.cin);
      dcol_max = std::max(dcol_max, rows * c.kpad);
      t_max = std::max(t_max, rows * std::max(c.kpad, c.cout));
    }
    xbf[4].resize(static_cast<size_t>(batch) * kFlat);
    xbf[5].resize(static_cast<size_t>(batch) * kHidden);
    act[4].resize(static_cast<size_t>(batch) * kHidden);
    dact[4].resize(act[4].count);
    dcol.resize(dcol_max);
    t_a.resize(t_max);
    t_b.resize(t_max);
    dout8.resize(static_cast<size_t>(batch) * kOutPad);
    partial.resize(static_cast<size_t>((batch * kConv[0].hout * kConv[0].wout + kColsumRows - 1) / kColsumRows) *
                   kHidden);
    loss.resize(1);
    workspace.resize(size_t{1} << 22);  // 16 MB
    out.resize(static_cast<size_t>(batch) * kOut);
    error.resize(1);
    check(cudaMemset(error.ptr, 0, sizeof(int)), "learner init");
    refresh_weights(nullptr);
    check(cudaDeviceSynchronize(), "learner init");
  }

  // the bf16 copies of the weights and of their transposes
  void refresh_weights(cudaStream_t s) {
    to_bf16_kernel<<<blocks_for(lay.total), 256, 0, s>>>(params.ptr, wbf.ptr, lay.total);
    for (int i = 0; i < 6; ++i) {
      transpose_bf16_kernel<<<blocks_for(static_cast<size_t>(lay.cols[i]) * rows_pad[i]), 256, 0, s>>>(
          params.ptr + lay.w[i], lay.rows[i], lay.cols[i], lay.cols[i], wtbf.ptr + wt_off[i], rows_pad[i]);
    }
    check(cudaGetLastError(), "learner weights");
  }

  void gemm(const __nv_bfloat16* a, const __nv_bfloat16* b, float* c, int m, int n, int k, int lda, int ldb,
            int ldc, const float* bias, int relu, cudaStream_t s) {
    launch_gemm_bf16(a, b, c, m, n, k, lda, ldb, ldc, bias, relu, error.ptr, s, workspace.ptr, workspace.count);
  }

  void colsum(const float* m, int rows, int cols, float* sums, cudaStream_t s) {
    const int chunks = (rows + kColsumRows - 1) / kColsumRows;
    colsum_partial_kernel<<<dim3((cols + 31) / 32, chunks), dim3(32, 8), 0, s>>>(m, rows, cols, partial.ptr);
    colsum_finish_kernel<<<(cols + 63) / 64, 64, 0, s>>>(partial.ptr, chunks, cols, sums);
  }

  // inputs: bf16 NHWC [batch][60][80][2] -> out [batch][6]
  void forward(const __nv_bfloat16* x0, int batch, cudaStream_t s) {
    const __nv_bfloat16* x = x0;
    for (int i = 0; i < 4; ++i) {
      const Conv& c = kConv[i];
      const size_t rows = static_cast<size_t>(batch) * c.hout * c.wout;
      im2col_kernel<<<blocks_for(rows * c.kpad), 256, 0, s>>>(x, col[i].ptr, batch, c);
      gemm(col[i].ptr, wbf.ptr + lay.w[i], act[i].ptr, static_cast<int>(rows), c.cout, c.kpad, c.kpad, c.kpad,
           c.cout, params.ptr + lay.b[i], 1, s);
      __nv_bfloat16* next = i < 3 ? xbf[i + 1].ptr : xbf[4].ptr;
      to_bf16_kernel<<<blocks_for(rows * c.cout), 256, 0, s>>>(act[i].ptr, next, rows * c.cout);
      x = next;
    }
    gemm(xbf[4].ptr, wbf.ptr + lay.w[4], act[4].ptr, batch, kHidden, kFlat, kFlat, kFlat, kHidden,
         params.ptr + lay.b[4], 1, s);
    to_bf16_kernel<<<blocks_for(static_cast<size_t>(batch) * kHidden), 256, 0, s>>>(
        act[4].ptr, xbf[5].ptr, static_cast<size_t>(batch) * kHidden);
    gemm(xbf[5].ptr, wbf.ptr + lay.w[5], out.ptr, batch, kOut, kHidden, kHidden, kHidden, kOut,
         params.ptr + lay.b[5], 0, s);
    check(cudaGetLastError(), "learner forward");
  }

  // dW [n_out][k] = bf16(dz)^T . in for dz [m][n_out] fp32 and in [m][k] bf16:
  // C = A B^T with A = dz^T [n_out][m], B = in^T [k][m].
  void weight_grad(const float* dz, int m, int n_out, const __nv_bfloat16* in, int k, float* dw, cudaStream_t s) {
    const int mp = (m + 7) / 8 * 8;
    transpose_bf16_kernel<<<blocks_for(static_cast<size_t>(n_out) * mp), 256, 0, s>>>(dz, m, n_out, n_out, t_a.ptr,
                                                                                     mp);
    transpose_bf16_bf16_kernel<<<blocks_for(static_cast<size_t>(k) * mp), 256, 0, s>>>(in, m, k, k, t_b.ptr, mp);
    gemm(t_a.ptr, t_b.ptr, dw, n_out, k, mp, mp, mp, k, nullptr, 0, s);
  }

  // gradients of the batch-mean squared twist error into grads (after forward)
  void backward(const float* target, int batch, cudaStream_t s) {
    loss_kernel<<<1, 256, 0, s>>>(out.ptr, target, batch, dout8.ptr, loss.ptr);
    // fc2: dW = d_out^T x5 (the first 6 rows of an 8-row product), db, dx5 = d_out W
    weight_grad(dout8.ptr, batch, kOutPad, xbf[5].ptr, kHidden, dcol.ptr, s);
    check(cudaMemcpyAsync(grads.ptr + lay.w[5], dcol.ptr, sizeof(float) * kOut * kHidden, cudaMemcpyDeviceToDevice,
                          s),
          "learner grads");
    colsum(dout8.ptr, batch, kOutPad, dcol.ptr, s);
    check(cudaMemcpyAsync(grads.ptr + lay.b[5], dcol.ptr, sizeof(float) * kOut, cudaMemcpyDeviceToDevice, s),
          "learner grads");
    to_bf16_kernel<<<blocks_for(static_cast<size_t>(batch) * kOutPad), 256, 0, s>>>(
        dout8.ptr, t_a.ptr, static_cast<size_t>(batch) * kOutPad);
    gemm(t_a.ptr, wtbf.ptr + wt_off[5], dact[4].ptr, batch, kHidden, kOutPad, kOutPad, rows_pad[5], kHidden,
         nullptr, 0, s);
    // fc1
    relu_back_kernel<<<blocks_for(static_cast<size_t>(batch) * kHidden), 256, 0, s>>>(
        dact[4].ptr, act[4].ptr, static_cast<size_t>(batch) * kHidden);
    weight_grad(dact[4].ptr, batch, kHidden, xbf[4].ptr, kFlat, grads.ptr + lay.w[4], s);
    colsum(dact[4].ptr, batch, kHidden, grads.ptr + lay.b[4], s);
    to_bf16_kernel<<<blocks_for(static_cast<size_t>(batch) * kHidden), 256, 0, s>>>(
        dact[4].ptr, t_a.ptr, static_cast<size_t>(batch) * kHidden);
    // dx4 = the gradient of conv4's output, [batch*20][64] = [batch][1280]
    gemm(t_a.ptr, wtbf.ptr + wt_off[4], dact[3].ptr, batch, kFlat, kHidden, kHidden, rows_pad[4], kFlat, nullptr, 0,
         s);
    for (int i = 3; i >= 0; --i) {
      const Conv& c = kConv[i];
      const size_t rows = static_cast<size_t>(batch) * c.hout * c.wout;
      relu_back_kernel<<<blocks_for(rows * c.cout), 256, 0, s>>>(dact[i].ptr, act[i].ptr, rows * c.cout);
      weight_grad(dact[i].ptr, static_cast<int>(rows), c.cout, col[i].ptr, c.kpad, grads.ptr + lay.w[i], s);
      colsum(dact[i].ptr, static_cast<int>(rows), c.cout, grads.ptr + lay.b[i], s);
      if (i == 0) break;
      to_bf16_kernel<<<blocks_for(rows * c.cout), 256, 0, s>>>(dact[i].ptr, t_a.ptr, rows * c.cout);
      gemm(t_a.ptr, wtbf.ptr + wt_off[i], dcol.ptr, static_cast<int>(rows), c.kpad, c.cout, c.cout, rows_pad[i],
           c.kpad, nullptr, 0, s);
      col2im_kernel<<<blocks_for(static_cast<size_t>(batch) * c.hin * c.win * c.cin), 256, 0, s>>>(
          dcol.ptr, dact[i - 1].ptr, batch, c);
    }
    check(cudaGetLastError(), "learner backward");
  }

  void adam(float lr, cudaStream_t s) {
    ++steps;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, static_cast<float>(steps));
    const float c2 = 1.0f - std::pow(b2, static_cast<float>(steps));
    adam_kernel<<<blocks_for(lay.total), 256, 0, s>>>(params.ptr, grads.ptr, adam_m.ptr, adam_v.ptr, lay.total, lr,
                                                      b1, b2, 1e-8f, c1, c2);
    refresh_weights(s);
  }

  void check_batch(uint32_t batch, const char* what) const {
    require(batch > 0 && static_cast<int>(batch) <= capacity && batch % 8 == 0, what);
  }
};

// ---- the warm start --------------------------------------------------------
namespace {

constexpr int kNetW = 80, kNetH = 60, kNetPixels = kNetW * kNetH;
constexpr int kNetDown = 8;  // 640 x 480 -> 80 x 60

struct Pose34 {
  float m[12];  // row-major 3 x 4 camera_to_world
};

Pose34 pose34(const kf_rigid& r) {
  Pose34 p;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) p.m[4 * i + j] = r.r[3 * i + j];
    p.m[4 * i + 3] = r.t[i];
  }
  return p;
}

// Current depth at the net's resolution: the mean of the valid depths of
// each 8 x 8 block (0 when it has none), in metres.
__global__ void net_depth_kernel(const uint16_t* __restrict__ depth, uint32_t width, uint32_t height,
                                 float inv_scale, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kNetPixels) return;
  const int bx = i % kNetW, by = i / kNetW;
  float sum = 0.0f;
  int n = 0;
  const int y1 = min(static_cast<int>(height), by * kNetDown + kNetDown);
  const int x1 = min(static_cast<int>(width), bx * kNetDown + kNetDown);
  for (int y = by * kNetDown; y < y1; ++y) {
    for (int x = bx * kNetDown; x < x1; ++x) {
      const uint16_t d = depth[static_cast<size_t>(y) * width + x];
      if (d != 0) {
        sum += static_cast<float>(d) * inv_scale;
        ++n;
      }
    }
  }
  out[i] = n ? sum / static_cast<float>(n) : 0.0f;
}

// The net input of one sample, NHWC bf16 [60][80][2]:
//   channel 0: current depth minus the mean predicted depth (0 where invalid);
//   channel 1: (current - predicted) * kDiffGain clamped to [-1, 1] (0 where
//              either is invalid).
// The second channel is the difference of the two maps rather than the
// predicted depth itself so that millimetre offsets survive bf16 rounding.
// The predicted depth is the camera-frame z of the model surface rendered at
// `pose`.  One CTA of 1024 threads.
constexpr float kDiffGain = 10.0f;
__global__ void net_input_kernel(const float* __restrict__ current, const float* __restrict__ points, Pose34 pose_arg,
                                 const Pose34* __restrict__ pose_dev, __nv_bfloat16* __restrict__ out,
                                 float* __restrict__ predicted) {
  // the render pose: a kernel argument, or device memory when pose_dev is set
  const Pose34 pose = pose_dev != nullptr ? *pose_dev : pose_arg;
  __shared__ float s_sum[1024];
  __shared__ int s_n[1024];
  float sum = 0.0f;
  int n = 0;
  for (int i = threadIdx.x; i < kNetPixels; i += blockDim.x) {
    const float px = points[3 * i], py = points[3 * i + 1], pz = points[3 * i + 2];
    float z = 0.0f;
    if (isfinite(px) && isfinite(py) && isfinite(pz)) {
      // z = (R^T (p - t)).z = column 2 of R dotted with p - t
      const float dx = px - pose.m[3], dy = py - pose.m[7], dz = pz - pose.m[11];
      z = pose.m[2] * dx + pose.m[6] * dy + pose.m[10] * dz;
      if (!(z > 0.0f)) z = 0.0f;
    }
    predicted[i] = z;
    if (z > 0.0f) {
      sum += z;
      ++n;
    }
  }
  s_sum[threadIdx.x] = sum;
  s_n[threadIdx.x] = n;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      s_sum[threadIdx.x] += s_sum[threadIdx.x + st];
      s_n[threadIdx.x] += s_n[threadIdx.x + st];
    }
    __syncthreads();
  }
  const float mean = s_n[0] ? s_sum[0] / static_cast<float>(s_n[0]) : 0.0f;
  for (int i = threadIdx.x; i < kNetPixels; i += blockDim.x) {
    const float c = current[i], z = predicted[i];
    const float c0 = c > 0.0f ? c - mean : 0.0f;
    float c1 = 0.0f;
    if (c > 0.0f && z > 0.0f) c1 = fminf(1.0f, fmaxf(-1.0f, (c - z) * kDiffGain));
    out[2 * i] = __float2bfloat16(c0);
    out[2 * i + 1] = __float2bfloat16(c1);
  }
}

// Truncated point-to-plane cost of the current depth (back-projected at the
// net's resolution) placed at camera_to_world poses[blockIdx.x], against the
// model surface rendered at `render` (projective association into the
// rendered maps): per valid pixel min(r^2, cap^2) with r the point-to-plane
// distance to the matched model point, and cap^2 where no model point lies
// within `cap` metres.  costs[2 j] = the cost, costs[2 j + 1] = the matches.
__global__ void warm_cost_kernel(const float* __restrict__ current, const float* __restrict__ points,
                                 const float* __restrict__ normals, Pose34 render, const Pose34* __restrict__ poses,
                                 Intr k, float cap, float* __restrict__ costs) {
  __shared__ float s_cost[256];
  __shared__ float s_match[256];
  const Pose34 p = poses[blockIdx.x];
  float cost = 0.0f, matched = 0.0f;
  for (int i = threadIdx.x; i < kNetPixels; i += blockDim.x) {
    const float d = current[i];
    if (!(d > 0.0f)) continue;
    const int u = i % kNetW, v = i / kNetW;
    const float cx = (static_cast<float>(u) - k.cx) / k.fx * d, cy = (static_cast<float>(v) - k.cy) / k.fy * d;
    const float wx = p.m[0] * cx + p.m[1] * cy + p.m[2] * d + p.m[3];
    const float wy = p.m[4] * cx + p.m[5] * cy + p.m[6] * d + p.m[7];
    const float wz = p.m[8] * cx + p.m[9] * cy + p.m[10] * d + p.m[11];
    const float ex = wx - render.m[3], ey = wy - render.m[7], ez = wz - render.m[11];
    const float rx = render.m[0] * ex + render.m[4] * ey + render.m[8] * ez;
    const float ry = render.m[1] * ex + render.m[5] * ey + render.m[9] * ez;
    const float rz = render.m[2] * ex + render.m[6] * ey + render.m[10] * ez;
    float c = cap * cap;
    if (rz > 0.0f) {
      const float fu = k.fx * rx / rz + k.cx, fv = k.fy * ry / rz + k.cy;
      if (fu > -0.5f && fu < kNetW - 0.5f && fv > -0.5f && fv < kNetH - 0.5f) {
        const int mu = min(kNetW - 1, max(0, __float2int_rn(fu)));
        const int mv = min(kNetH - 1, max(0, __float2int_rn(fv)));
        const int j = mv * kNetW + mu;
        const float mx = points[3 * j], my = points[3 * j + 1], mz = points[3 * j + 2];
        const float nx = normals[3 * j], ny = normals[3 * j + 1], nz = normals[3 * j + 2];
        if (isfinite(mx) && isfinite(nx)) {
          const float qx = wx - mx, qy = wy - my, qz = wz - mz;
          if (qx * qx + qy * qy + qz * qz < cap * cap) {
            const float r = qx * nx + qy * ny + qz * nz;
            c = fminf(r * r, cap * cap);
            matched += 1.0f;
          }
        }
      }
    }
    cost += c;
  }
  s_cost[threadIdx.x] = cost;
  s_match[threadIdx.x] = matched;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      s_cost[threadIdx.x] += s_cost[threadIdx.x + st];
      s_match[threadIdx.x] += s_match[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    costs[2 * blockIdx.x] = s_cost[0];
    costs[2 * blockIdx.x + 1] = s_match[0];
  }
}

// pose * exp(twist) with the decoupled exponential: the translation (tx, ty,
// tz) is added in the pose's frame and the rotation (wx, wy, wz) applied by
// Rodrigues' formula; in double.
kf_rigid apply_twist(const kf_rigid& pose, const double tw[6]) {
  const double wx = tw[3], wy = tw[4], wz = tw[5];
  const double th = std::sqrt(wx * wx + wy * wy + wz * wz);
  double d[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (th > 1e-15) {
    const double kx = wx / th, ky = wy / th, kz = wz / th, sn = std::sin(th), cs = 1.0 - std::cos(th);
    const double K[9] = {0, -kz, ky, kz, 0, -kx, -ky, kx, 0};
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j) {
        double k2 = 0;
        for (int q = 0; q < 3; ++q) k2 += K[3 * i + q] * K[3 * q + j];
        d[3 * i + j] += sn * K[3 * i + j] + cs * k2;
      }
    }
  }
  kf_rigid out;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      double a = 0;
      for (int q = 0; q < 3; ++q) a += static_cast<double>(pose.r[3 * i + q]) * d[3 * q + j];
      out.r[3 * i + j] = static_cast<float>(a);
    }
    double t = pose.t[i];
    for (int q = 0; q < 3; ++q) t += static_cast<double>(pose.r[3 * i + q]) * tw[q];
    out.t[i] = static_cast<float>(t);
  }
  return out;
}

// ---- the asynchronous warm start: every step on the device ---------------
// Row-major 3x4 rigid transforms in double.
__device__ void rigid_mul(const double* a, const double* b, double* out) {
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 4; ++j) {
      double v = a[i * 4 + 0] * b[0 * 4 + j] + a[i * 4 + 1] * b[1 * 4 + j] + a[i * 4 + 2] * b[2 * 4 + j];
      if (j == 3) v += a[i * 4 + 3];
      out[i * 4 + j] = v;
    }
  }
}
// Inverse of [A | t] as [A^-1 | -A^-1 t], A^-1 by cofactors: the inverse of
// the float pose as stored, whose rotation is orthonormal only to float
// precision (the transpose would compound that error through the
// prediction).
__device__ void rigid_inv(const double* a, double* out) {
  const double a00 = a[0], a01 = a[1], a02 = a[2], a10 = a[4], a11 = a[5], a12 = a[6];
  const double a20 = a[8], a21 = a[9], a22 = a[10];
  const double c00 = a11 * a22 - a12 * a21, c01 = a12 * a20 - a10 * a22, c02 = a10 * a21 - a11 * a20;
  const double det = a00 * c00 + a01 * c01 + a02 * c02;
  const double inv_det = 1.0 / det;
  double m[9];
  m[0] = c00 * inv_det;
  m[1] = (a02 * a21 - a01 * a22) * inv_det;
  m[2] = (a01 * a12 - a02 * a11) * inv_det;
  m[3] = c01 * inv_det;
  m[4] = (a00 * a22 - a02 * a20) * inv_det;
  m[5] = (a02 * a10 - a00 * a12) * inv_det;
  m[6] = c02 * inv_det;
  m[7] = (a01 * a20 - a00 * a21) * inv_det;
  m[8] = (a00 * a11 - a01 * a10) * inv_det;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) out[i * 4 + j] = m[i * 3 + j];
    out[i * 4 + 3] = -(m[i * 3 + 0] * a[3] + m[i * 3 + 1] * a[7] + m[i * 3 + 2] * a[11]);
  }
}

// Device state of the asynchronous warm start.
struct WarmDevice {
  double history[12];  // the pose the previous call saw (camera_to_world)
  int known;           // calls so far (the history holds a pose once >= 1)
  Pose34 predicted;    // this call's constant-velocity pose (floats)
  Pose34 poses[2];     // predicted, proposal: the two candidate starts
  float twist[6];
  float costs[4];
  int used_proposal;
  int lost;            // the previous frame lost track: no velocity, no net
};

// Pushes the tracker's pose (the previous frame's result, rounded to float
// as each frame starts from the float pose), predicts the constant-velocity
// pose T1 (T0^-1 T1) from it and the previous push (T1 itself after a frame
// that lost track), and points the render state at the prediction.
__global__ void warm_predict_kernel(const IcpState* __restrict__ st, WarmDevice* w, IcpState* render) {
  if (threadIdx.x != 0) return;
  double t1[12], pred[12];
  for (int i = 0; i < 12; ++i) t1[i] = static_cast<double>(static_cast<float>(st->pose[i]));
  // after a frame that lost track the last motion says nothing: no velocity
  w->lost = st->failed ? 1 : 0;
  if (w->known >= 1 && !st->failed) {
    double inv0[12], delta[12];
    rigid_inv(w->history, inv0);
    rigid_mul(inv0, t1, delta);
    rigid_mul(t1, delta, pred);
  } else {
    for (int i = 0; i < 12; ++i) pred[i] = t1[i];
  }
  for (int i = 0; i < 12; ++i) w->history[i] = t1[i];
  w->known += 1;
  for (int i = 0; i < 12; ++i) w->predicted.m[i] = static_cast<float>(pred[i]);
  // render state: camera = kf_rigid layout (rotation rows, then translation)
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) render->camera[i * 3 + j] = w->predicted.m[i * 4 + j];
    render->camera[9 + i] = w->predicted.m[i * 4 + 3];
  }
  render->failed = 0;
}

// pose * exp(twist) as apply_twist, on the device.
__device__ void apply_twist_dev(const Pose34& pose, const double* tw, Pose34& out) {
  const double wx = tw[3], wy = tw[4], wz = tw[5];
  const double th = sqrt(wx * wx + wy * wy + wz * wz);
  double d[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (th > 1e-15) {
    const double kx = wx / th, ky = wy / th, kz = wz / th, sn = sin(th), cs = 1.0 - cos(th);
    const double K[9] = {0, -kz, ky, kz, 0, -kx, -ky, kx, 0};
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j) {
        double k2 = 0;
        for (int q = 0; q < 3; ++q) k2 += K[3 * i + q] * K[3 * q + j];
        d[3 * i + j] += sn * K[3 * i + j] + cs * k2;
      }
    }
  }
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      double a = 0;
      for (int q = 0; q < 3; ++q) a += static_cast<double>(pose.m[4 * i + q]) * d[3 * q + j];
      out.m[4 * i + j] = static_cast<float>(a);
    }
    double t = pose.m[4 * i + 3];
    for (int q = 0; q < 3; ++q) t += static_cast<double>(pose.m[4 * i + q]) * tw[q];
    out.m[4 * i + 3] = static_cast<float>(t);
  }
}

// The proposal from the net's output (or none), both candidates' truncated
// costs (the warm_cost_kernel arithmetic, one CTA), the choice, and the
// chosen start written into the tracker as kf_frame_set_pose would.
__global__ void __launch_bounds__(256)
    warm_choose_kernel(const float* __restrict__ current, const float* __restrict__ points,
                       const float* __restrict__ normals, const float* __restrict__ net_out, float scale, Intr k,
                       float cap, int use_net, WarmDevice* w, IcpState* st) {
  __shared__ float s_cost[256];
  __shared__ float s_match[256];
  use_net = use_net && !w->lost;
  if (threadIdx.x == 0) {
    w->poses[0] = w->predicted;
    if (use_net) {
      double tw[6];
      for (int i = 0; i < 6; ++i) {
        tw[i] = static_cast<double>(net_out[i]) / static_cast<double>(scale);
        w->twist[i] = static_cast<float>(tw[i]);
      }
      apply_twist_dev(w->predicted, tw, w->poses[1]);
    } else {
      w->poses[1] = w->predicted;
      for (int i = 0; i < 6; ++i) w->twist[i] = 0.0f;
    }
  }
  __syncthreads();
  const Pose34 render = w->predicted;
  for (int cand = 0; cand < 2; ++cand) {
    const Pose34 p = w->poses[cand];
    float cost = 0.0f, matched = 0.0f;
    for (int i = threadIdx.x; i < kNetPixels; i += blockDim.x) {
      const float d = current[i];
      if (!(d > 0.0f)) continue;
      const int u = i % kNetW, v = i / kNetW;
      const float cx = (static_cast<float>(u) - k.cx) / k.fx * d, cy = (static_cast<float>(v) - k.cy) / k.fy * d;
      const float wx = p.m[0] * cx + p.m[1] * cy + p.m[2] * d + p.m[3];
      const float wy = p.m[4] * cx + p.m[5] * cy + p.m[6] * d + p.m[7];
      const float wz = p.m[8] * cx + p.m[9] * cy + p.m[10] * d + p.m[11];
      const float ex = wx - render.m[3], ey = wy - render.m[7], ez = wz - render.m[11];
      const float rx = render.m[0] * ex + render.m[4] * ey + render.m[8] * ez;
      const float ry = render.m[1] * ex + render.m[5] * ey + render.m[9] * ez;
      const float rz = render.m[2] * ex + render.m[6] * ey + render.m[10] * ez;
      float c = cap * cap;
      if (rz > 0.0f) {
        const float fu = k.fx * rx / rz + k.cx, fv = k.fy * ry / rz + k.cy;
        if (fu > -0.5f && fu < kNetW - 0.5f && fv > -0.5f && fv < kNetH - 0.5f) {
          const int mu = min(kNetW - 1, max(0, __float2int_rn(fu)));
          const int mv = min(kNetH - 1, max(0, __float2int_rn(fv)));
          const int j = mv * kNetW + mu;
          const float mx = points[3 * j], my = points[3 * j + 1], mz = points[3 * j + 2];
          const float nx = normals[3 * j], ny = normals[3 * j + 1], nz = normals[3 * j + 2];
          if (isfinite(mx) && isfinite(nx)) {
            const float qx = wx - mx, qy = wy - my, qz = wz - mz;
            if (qx * qx + qy * qy + qz * qz < cap * cap) {
              const float r = qx * nx + qy * ny + qz * nz;
              c = fminf(r * r, cap * cap);
              matched += 1.0f;
            }
          }
        }
      }
      cost += c;
    }
    s_cost[threadIdx.x] = cost;
    s_match[threadIdx.x] = matched;
    __syncthreads();
    for (int sh = blockDim.x / 2; sh > 0; sh >>= 1) {
      if (threadIdx.x < sh) {
        s_cost[threadIdx.x] += s_cost[threadIdx.x + sh];
        s_match[threadIdx.x] += s_match[threadIdx.x + sh];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      w->costs[2 * cand] = s_cost[0];
      w->costs[2 * cand + 1] = s_match[0];
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  w->used_proposal = use_net && w->costs[2] <= w->costs[0] ? 1 : 0;
  const Pose34& start = w->poses[w->used_proposal];
  // icp_set_pose_kernel with reset_frame = 1
  for (int i = 0; i < 12; ++i) st->pose[i] = static_cast<double>(start.m[i]);
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) st->camera[i * 3 + j] = start.m[i * 4 + j];
    st->camera[9 + i] = start.m[i * 4 + 3];
  }
  // world_to_camera = {R^T, -R^T t} as icp_set_pose_kernel writes it
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) st->world_to_camera[i * 3 + j] = static_cast<float>(st->pose[j * 4 + i]);
    st->world_to_camera[9 + i] = static_cast<float>(
        -(st->pose[0 * 4 + i] * st->pose[3] + st->pose[1 * 4 + i] * st->pose[7] + st->pose[2 * 4 + i] * st->pose[11]));
  }
  st->failed = 0;
  st->status = KF_ICP_NOT_RUN;
  for (int l = 0; l < 4; ++l) {
    st->level_status[l] = KF_ICP_NOT_RUN;
    st->level_iterations[l] = 0;
    st->level_correspondences[l] = 0;
  }
}

}  // namespace

struct WarmStart {
  float depth_scale = 5000.0f;
  float cost_cap = 0.05f;
  DeviceArray<uint16_t> staged;  // host depth frames are copied here
  DeviceArray<float> current, predicted, points, normals, costs;
  DeviceArray<uint32_t> colors;
  DeviceArray<Pose34> poses;
  DeviceArray<__nv_bfloat16> input;  // 8 samples (the smallest batch); only the first is filled
  DeviceArray<WarmDevice> dev;       // the asynchronous warm start's state
  DeviceArray<IcpState> render;      // the render pose of the asynchronous warm start
  PinnedArray<WarmDevice> staging;

  void init() {
    dev.resize(1);
    render.resize(1);
    staging.resize(1);
    check(cudaMemset(dev.ptr, 0, dev.bytes()), "warm start init");
    check(cudaMemset(render.ptr, 0, render.bytes()), "warm start init");
    current.resize(kNetPixels);
    predicted.resize(kNetPixels);
    points.resize(kNetPixels * 3);
    normals.resize(kNetPixels * 3);
    colors.resize(kNetPixels);
    costs.resize(4);
    poses.resize(2);
    input.resize(static_cast<size_t>(8) * kNetPixels * 2);
    check(cudaMemset(input.ptr, 0, input.bytes()), "warm start init");
  }

  // the centre of each 8 x 8 block maps to the centre of its net pixel
  static kf_intrinsics net_intrinsics(const kf_intrinsics& k) {
    const float f = 1.0f / kNetDown;
    return kf_intrinsics{k.fx * f, k.fy * f, (k.cx + 0.5f) * f - 0.5f, (k.cy + 0.5f) * f - 0.5f};
  }

  // current depth + the model rendered at render_pose -> the net input `out`
  void build(Pipeline& p, const uint16_t* depth, uint32_t width, uint32_t height, int memory,
             const kf_intrinsics& k, const kf_rigid& render_pose, __nv_bfloat16* out) {
    require(width == kNetW * kNetDown && height == kNetH * kNetDown, "warm start: depth frames must be 640 x 480");
    require(k.fx > 0.0f && k.fy > 0.0f, "warm start: intrinsics must have positive focal lengths");
    const cudaStream_t s = p.stream;
    const uint16_t* d = depth;
    if (memory != KF_MEMORY_DEVICE) {
      staged.resize(static_cast<size_t>(width) * height);
      check(cudaMemcpyAsync(staged.ptr, depth, staged.bytes(), cudaMemcpyHostToDevice, s), "warm start depth");
      d = staged.ptr;
    }
    net_depth_kernel<<<(kNetPixels + 255) / 256, 256, 0, s>>>(d, width, height, 1.0f / depth_scale, current.ptr);
    kf_raycast_camera cam{};
    cam.intrinsics = net_intrinsics(k);
    cam.width = kNetW;
    cam.height = kNetH;
    cam.camera_to_world = render_pose;
    launch_raycast(p, cam, points.ptr, normals.ptr, colors.ptr, nullptr, s);
    net_input_kernel<<<1, 1024, 0, s>>>(current.ptr, points.ptr, pose34(render_pose), nullptr, out, predicted.ptr);
    check(cudaGetLastError(), "warm start input");
  }

  // The asynchronous step: prediction from the tracker's pose, render, net,
  // choice, and the start written into the tracker; no host round trip.
  void enqueue(Pipeline& p, Learner* l, IcpState* st, const uint16_t* depth, uint32_t width, uint32_t height,
               int memory, const kf_intrinsics& k, bool use_net) {
    require(width == kNetW * kNetDown && height == kNetH * kNetDown, "warm start: depth frames must be 640 x 480");
    require(k.fx > 0.0f && k.fy > 0.0f, "warm start: intrinsics must have positive focal lengths");
    const cudaStream_t s = p.stream;
    warm_predict_kernel<<<1, 32, 0, s>>>(st, dev.ptr, render.ptr);
    check(cudaGetLastError(), "warm start predict");
    const uint16_t* d = depth;
    if (memory != KF_MEMORY_DEVICE) {
      staged.resize(static_cast<size_t>(width) * height);
      check(cudaMemcpyAsync(staged.ptr, depth, staged.bytes(), cudaMemcpyHostToDevice, s), "warm start depth");
      d = staged.ptr;
    }
    net_depth_kernel<<<(kNetPixels + 255) / 256, 256, 0, s>>>(d, width, height, 1.0f / depth_scale, current.ptr);
    kf_raycast_camera cam{};
    cam.intrinsics = net_intrinsics(k);
    cam.width = kNetW;
    cam.height = kNetH;
    std::memset(&cam.camera_to_world, 0, sizeof(cam.camera_to_world));  // the render state holds the pose
    launch_raycast(p, cam, points.ptr, normals.ptr, colors.ptr, render.ptr, s);
    const Pose34* pred = reinterpret_cast<const Pose34*>(reinterpret_cast<const char*>(dev.ptr) +
                                                         offsetof(WarmDevice, predicted));
    net_input_kernel<<<1, 1024, 0, s>>>(current.ptr, points.ptr, Pose34{}, pred, input.ptr, predicted.ptr);
    check(cudaGetLastError(), "warm start input");
    if (use_net) l->forward(input.ptr, 8, s);
    warm_choose_kernel<<<1, 256, 0, s>>>(current.ptr, points.ptr, normals.ptr, use_net ? l->out.ptr : nullptr,
                                         static_cast<float>(KF_WARM_START_TWIST_SCALE),
                                         intr_from(net_intrinsics(k)), cost_cap, use_net ? 1 : 0, dev.ptr, st);
    check(cudaGetLastError(), "warm start choose");
  }
};

}  // namespace kf

struct kf_learner {
  kf::Learner impl;
};
struct kf_warm_start {
  kf::WarmStart impl;
};

using namespace kf;

extern "C" {

kf_status kf_learner_create(uint32_t batch_capacity, uint32_t seed, kf_learner** out) {
  return guarded([&] {
    require(out != nullptr && batch_capacity > 0 && batch_capacity % 8 == 0,
            "kf_learner_create: batch capacity must be a positive multiple of 8");
    auto* l = new kf_learner();
    try {
      l->impl.init(static_cast<int>(batch_capacity), seed);
    } catch (...) {
      delete l;
      throw;
    }
    *out = l;
  });
}

kf_status kf_learner_destroy(kf_learner* learner) {
  return guarded([&] { delete learner; });
}

kf_status kf_learner_param_count(kf_learner* learner, uint64_t* count) {
  return guarded([&] {
    require(learner && count, "kf_learner_param_count: null argument");
    *count = learner->impl.lay.total;
  });
}

kf_status kf_learner_get_params(kf_learner* learner, float* host) {
  return guarded([&] {
    require(learner && host, "kf_learner_get_params: null argument");
    check(cudaDeviceSynchronize(), "params");
    check(cudaMemcpy(host, learner->impl.params.ptr, learner->impl.params.bytes(), cudaMemcpyDeviceToHost), "params");
  });
}

kf_status kf_learner_set_params(kf_learner* learner, const float* host) {
  return guarded([&] {
    require(learner && host, "kf_learner_set_params: null argument");
    check(cudaDeviceSynchronize(), "params");
    check(cudaMemcpy(learner->impl.params.ptr, host, learner->impl.params.bytes(), cudaMemcpyHostToDevice), "params");
    learner->impl.refresh_weights(nullptr);
    check(cudaDeviceSynchronize(), "params");
  });
}

kf_status kf_learner_forward(kf_learner* learner, const void* inputs, uint32_t batch, float* out, void* stream) {
  return guarded([&] {
    require(learner && inputs && out, "kf_learner_forward: null argument");
    Learner& l = learner->impl;
    l.check_batch(batch, "kf_learner_forward: batch must be a multiple of 8 within the capacity");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    l.forward(static_cast<const __nv_bfloat16*>(inputs), static_cast<int>(batch), s);
    check(cudaMemcpyAsync(out, l.out.ptr, sizeof(float) * batch * kOut, cudaMemcpyDeviceToDevice, s), "forward out");
  });
}

kf_status kf_learner_gradients(kf_learner* learner, const void* inputs, const float* targets, uint32_t batch,
                               float* host_grads, float* loss, void* stream) {
  return guarded([&] {
    require(learner && inputs && targets, "kf_learner_gradients: null argument");
    Learner& l = learner->impl;
    l.check_batch(batch, "kf_learner_gradients: batch must be a multiple of 8 within the capacity");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    check(cudaMemsetAsync(l.grads.ptr, 0, l.grads.bytes(), s), "grads");
    l.forward(static_cast<const __nv_bfloat16*>(inputs), static_cast<int>(batch), s);
    l.backward(targets, static_cast<int>(batch), s);
    if (host_grads) {
      check(cudaMemcpyAsync(host_grads, l.grads.ptr, l.grads.bytes(), cudaMemcpyDeviceToHost, s), "grads");
    }
    if (loss) check(cudaMemcpyAsync(loss, l.loss.ptr, sizeof(float), cudaMemcpyDeviceToHost, s), "loss");
    int err = 0;
    check(cudaMemcpyAsync(&err, l.error.ptr, sizeof(int), cudaMemcpyDeviceToHost, s), "learner error");
    check(cudaStreamSynchronize(s), "gradients");
    if (err) throw CudaError("kf_learner_gradients: tensor-core wait timed out");
  });
}

kf_status kf_learner_train_step(kf_learner* learner, const void* inputs, const float* targets, uint32_t batch,
                                float learning_rate, float* loss, void* stream) {
  return guarded([&] {
    require(learner && inputs && targets, "kf_learner_train_step: null argument");
    Learner& l = learner->impl;
    l.check_batch(batch, "kf_learner_train_step: batch must be a multiple of 8 within the capacity");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    check(cudaMemsetAsync(l.grads.ptr, 0, l.grads.bytes(), s), "grads");
    l.forward(static_cast<const __nv_bfloat16*>(inputs), static_cast<int>(batch), s);
    l.backward(targets, static_cast<int>(batch), s);
    if (loss) check(cudaMemcpyAsync(loss, l.loss.ptr, sizeof(float), cudaMemcpyDeviceToDevice, s), "loss");
    l.adam(learning_rate, s);
  });
}

kf_status kf_learner_error(kf_learner* learner, int32_t* timed_out) {
  return guarded([&] {
    require(learner && timed_out, "kf_learner_error: null argument");
    int err = 0;
    check(cudaDeviceSynchronize(), "learner error");
    check(cudaMemcpy(&err, learner->impl.error.ptr, sizeof(int), cudaMemcpyDeviceToHost), "learner error");
    *timed_out = err;
  });
}

kf_status kf_warm_start_create(float depth_scale, kf_warm_start** out) {
  return guarded([&] {
    require(out != nullptr && depth_scale > 0.0f, "kf_warm_start_create: bad argument");
    auto* w = new kf_warm_start();
    try {
      w->impl.depth_scale = depth_scale;
      w->impl.init();
    } catch (...) {
      delete w;
      throw;
    }
    *out = w;
  });
}

kf_status kf_warm_start_destroy(kf_warm_start* warm) {
  return guarded([&] { delete warm; });
}

kf_status kf_warm_start_input(kf_warm_start* warm, kf_pipeline* pipeline, const uint16_t* depth, uint32_t width,
                              uint32_t height, kf_intrinsics intrinsics, int32_t memory, const kf_rigid* render_pose,
                              void* input) {
  return guarded([&] {
    require(warm && pipeline && depth && render_pose && input, "kf_warm_start_input: null argument");
    require(reinterpret_cast<uintptr_t>(input) % 16 == 0, "kf_warm_start_input: input must be 16-byte aligned");
    warm->impl.build(pipeline->impl, depth, width, height, memory, intrinsics, *render_pose,
                     static_cast<__nv_bfloat16*>(input));
  });
}

kf_status kf_warm_start_reset(kf_warm_start* warm) {
  return guarded([&] {
    require(warm != nullptr, "kf_warm_start_reset: null argument");
    check(cudaMemset(warm->impl.dev.ptr, 0, warm->impl.dev.bytes()), "warm start reset");
  });
}

kf_status kf_warm_start_enqueue(kf_warm_start* warm, kf_learner* learner, kf_pipeline* pipeline, kf_tracker* tracker,
                                const uint16_t* depth, uint32_t width, uint32_t height, kf_intrinsics intrinsics,
                                int32_t memory, int32_t use_net) {
  return guarded([&] {
    require(warm && pipeline && tracker && depth, "kf_warm_start_enqueue: null argument");
    require(!use_net || learner != nullptr, "kf_warm_start_enqueue: the net's proposal needs a learner");
    if (use_net) learner->impl.check_batch(8, "kf_warm_start_enqueue: the learner's capacity is below 8");
    warm->impl.enqueue(pipeline->impl, use_net ? &learner->impl : nullptr, tracker->impl.state.ptr, depth, width,
                       height, memory, intrinsics, use_net != 0);
  });
}

kf_status kf_warm_start_fetch(kf_warm_start* warm, kf_pipeline* pipeline, kf_warm_start_result* result) {
  return guarded([&] {
    require(warm && pipeline && result, "kf_warm_start_fetch: null argument");
    WarmStart& w = warm->impl;
    const cudaStream_t s = pipeline->impl.stream;
    check(cudaMemcpyAsync(w.staging.ptr, w.dev.ptr, sizeof(WarmDevice), cudaMemcpyDeviceToHost, s), "warm fetch");
    check(cudaStreamSynchronize(s), "warm fetch");
    const WarmDevice& d = *w.staging.ptr;
    auto rigid = [](const Pose34& p) {
      kf_rigid r;
      for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) r.r[i * 3 + j] = p.m[i * 4 + j];
        r.t[i] = p.m[i * 4 + 3];
      }
      return r;
    };
    result->proposal = rigid(d.poses[1]);
    result->start = rigid(d.poses[d.used_proposal]);
    for (int i = 0; i < 6; ++i) result->twist[i] = d.twist[i];
    result->cost_predicted = d.costs[0];
    result->matches_predicted = d.costs[1];
    result->cost_proposal = d.costs[2];
    result->matches_proposal = d.costs[3];
    result->used_proposal = d.used_proposal;
  });
}

kf_status kf_warm_start_propose(kf_warm_start* warm, kf_learner* learner, kf_pipeline* pipeline,
                                const uint16_t* depth, uint32_t width, uint32_t height, kf_intrinsics intrinsics,
                                int32_t memory, const kf_rigid* predicted, kf_warm_start_result* result) {
  return guarded([&] {
    require(warm && learner && pipeline && depth && predicted && result, "kf_warm_start_propose: null argument");
    WarmStart& w = warm->impl;
    Learner& l = learner->impl;
    Pipeline& p = pipeline->impl;
    l.check_batch(8, "kf_warm_start_propose: the learner's capacity is below 8");
    const cudaStream_t s = p.stream;
    w.build(p, depth, width, height, memory, intrinsics, *predicted, w.input.ptr);
    l.forward(w.input.ptr, 8, s);
    float tw[kOut];
    int err = 0;
    check(cudaMemcpyAsync(tw, l.out.ptr, sizeof(tw), cudaMemcpyDeviceToHost, s), "warm start twist");
    check(cudaMemcpyAsync(&err, l.error.ptr, sizeof(int), cudaMemcpyDeviceToHost, s), "warm start error");
    check(cudaStreamSynchronize(s), "warm start forward");
    if (err) throw CudaError("kf_warm_start_propose: tensor-core wait timed out");
    double twist[kOut];
    for (int i = 0; i < kOut; ++i) twist[i] = static_cast<double>(tw[i]) / KF_WARM_START_TWIST_SCALE;
    const kf_rigid proposal = apply_twist(*predicted, twist);
    const Pose34 host_poses[2] = {pose34(*predicted), pose34(proposal)};
    check(cudaMemcpyAsync(w.poses.ptr, host_poses, sizeof(host_poses), cudaMemcpyHostToDevice, s), "warm start");
    warm_cost_kernel<<<2, 256, 0, s>>>(w.current.ptr, w.points.ptr, w.normals.ptr, host_poses[0], w.poses.ptr,
                                       intr_from(WarmStart::net_intrinsics(intrinsics)), w.cost_cap, w.costs.ptr);
    check(cudaGetLastError(), "warm start cost");
    float costs[4];
    check(cudaMemcpyAsync(costs, w.costs.ptr, sizeof(costs), cudaMemcpyDeviceToHost, s), "warm start cost");
    check(cudaStreamSynchronize(s), "warm start cost");
    result->proposal = proposal;
    for (int i = 0; i < kOut; ++i) result->twist[i] = static_cast<float>(twist[i]);
    result->cost_predicted = costs[0];
    result->matches_predicted = costs[1];
    result->cost_proposal = costs[2];
    result->matches_proposal = costs[3];
    // constant velocity stays the start whenever the proposal's residual is higher
    result->used_proposal = costs[2] <= costs[0] ? 1 : 0;
    result->start = result->used_proposal ? proposal : *predicted;
  });
}

}  // extern "C"
