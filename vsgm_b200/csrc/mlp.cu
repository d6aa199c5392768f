// The learned planner's network: a 3-layer MLP (in -> hidden -> hidden -> out)
// with BF16 GEMM inputs and FP32 accumulation, trained and evaluated by the
// kernels below (no library GEMM).  The network only ranks execution orders;
// counts never depend on it.
//
// GEMMs use the warp-level mma.sync.m16n8k16 BF16 instruction: the matrices are
// a few hundred wide, far too small for tcgen05/TMEM tiles to pay off, and
// every call is latency-bound.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "vsgm.h"

namespace {

constexpr int kTile = 64;  // block tile (M and N)
constexpr int kK = 16;     // mma K

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// C[M,N] = op(A)[M,K] * op(B)[K,N]  (+ bias[N]) (ReLU)
// A element (m,k) = transA ? A[k*lda + m] : A[m*lda + k]; B element (k,n) = transB ? B[n*ldb + k] : B[k*ldb + n]
// Inputs are FP32 in memory and rounded to BF16 when staged (the BF16 operand
// copy), accumulation is FP32.  Outputs: C (FP32, may be null), relu mask applied if relu.
__global__ void __launch_bounds__(256) k_gemm(const float* __restrict__ A, const float* __restrict__ B, float* __restrict__ C, int M, int N, int K,
                                              int lda, int ldb, int ldc, int transA, int transB, const float* __restrict__ bias, int relu,
                                              int accumulate) {
  __shared__ uint32_t As[kTile][kK / 2 + 1];  // bf16 pairs along k, row m
  __shared__ uint32_t Bs[kTile][kK / 2 + 1];  // bf16 pairs along k, column n
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp & 3, wn = warp >> 2;  // 4 x 2 warps; warp tile 16 x 32
  const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
  const int g = lane >> 2, t = lane & 3;
  float acc[4][4];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) acc[i][j] = 0.f;

  for (int k0 = 0; k0 < K; k0 += kK) {
    // stage 64 x 16 of A and 16 x 64 of B as bf16 pairs (one pair per thread each... 512 pairs per tile)
    for (int idx = threadIdx.x; idx < kTile * kK / 2; idx += blockDim.x) {
      int r = idx / (kK / 2), kp = (idx % (kK / 2)) * 2;
      int m = m0 + r, k = k0 + kp;
      float a0 = 0.f, a1 = 0.f;
      if (m < M) {
        if (k < K) a0 = transA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
        if (k + 1 < K) a1 = transA ? A[(size_t)(k + 1) * lda + m] : A[(size_t)m * lda + k + 1];
      }
      As[r][kp / 2] = pack_bf16(a0, a1);
      int n = n0 + r;
      float b0 = 0.f, b1 = 0.f;
      if (n < N) {
        if (k < K) b0 = transB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n];
        if (k + 1 < K) b1 = transB ? B[(size_t)n * ldb + k + 1] : B[(size_t)(k + 1) * ldb + n];
      }
      Bs[r][kp / 2] = pack_bf16(b0, b1);
    }
    __syncthreads();
    // A fragment (row-major 16x16): rows g and g+8, k pairs t and t+4
    const int ar = wm * 16;
    uint32_t a[4];
    a[0] = As[ar + g][t];
    a[1] = As[ar + g + 8][t];
    a[2] = As[ar + g][t + 4];
    a[3] = As[ar + g + 8][t + 4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      // B fragment (16x8, column-major): column g of the n-subtile, k pairs t and t+4
      const int bc = wn * 32 + j * 8 + g;
      uint32_t b0 = Bs[bc][t], b1 = Bs[bc][t + 4];
      asm volatile(
          "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
          : "+f"(acc[j][0]), "+f"(acc[j][1]), "+f"(acc[j][2]), "+f"(acc[j][3])
          : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    }
    __syncthreads();
  }
  // epilogue: C fragment rows g, g+8; columns 2t, 2t+1
#pragma unroll
  for (int j = 0; j < 4; j++) {
#pragma unroll
    for (int h = 0; h < 4; h++) {
      int m = m0 + wm * 16 + g + (h >= 2 ? 8 : 0);
      int n = n0 + wn * 32 + j * 8 + 2 * t + (h & 1);
      if (m < M && n < N) {
        float v = acc[j][h];
        if (bias) v += bias[n];
        if (relu) v = v > 0.f ? v : 0.f;
        float* dst = C + (size_t)m * ldc + n;
        *dst = accumulate ? *dst + v : v;
      }
    }
  }
}

// masked MSE: loss = sum(mask * (y - t)^2) / max(1, sum(mask)); dy = 2 mask (y - t) / sum(mask)
__global__ void k_mse(const float* __restrict__ y, const float* __restrict__ t, const float* __restrict__ mask, size_t n, float inv_norm,
                      float* __restrict__ dy, float* __restrict__ loss) {
  float acc = 0.f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float d = (y[i] - t[i]) * mask[i];
    dy[i] = 2.f * d * inv_norm;
    acc += d * d * inv_norm;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

// dh *= (h > 0)
__global__ void k_relu_back(float* __restrict__ dh, const float* __restrict__ h, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (h[i] <= 0.f) dh[i] = 0.f;
}

// db[n] = sum_m d[m, n]
__global__ void k_colsum(const float* __restrict__ d, int M, int N, float* __restrict__ db) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int m = 0; m < M; m++) s += d[(size_t)m * N + n];
  db[n] = s;
}

// Adam on FP32 master parameters
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1, float* __restrict__ m2, size_t n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float gi = g[i];
    float a = m1[i] = b1 * m1[i] + (1.f - b1) * gi;
    float b = m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
    w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
  }
}

}  // namespace

struct vsgm_mlp {
  int device = 0, nin = 0, nh = 0, nout = 0;
  cudaStream_t stream = nullptr;
  size_t nparam = 0;
  float *w = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;  // packed params
  float *W1, *b1, *W2, *b2, *W3, *b3;                              // views into w
  float *gW1, *gb1, *gW2, *gb2, *gW3, *gb3;                        // views into g
  int cap = 0;                                                     // batch capacity
  float *x = nullptr, *h1 = nullptr, *h2 = nullptr, *y = nullptr, *t = nullptr, *mask = nullptr, *dy = nullptr, *dh2 = nullptr, *dh1 = nullptr,
        *loss = nullptr;
  long step = 0;
  std::string err;

  void carve() {
    float* p = w;
    W1 = p, p += (size_t)nin * nh;
    b1 = p, p += nh;
    W2 = p, p += (size_t)nh * nh;
    b2 = p, p += nh;
    W3 = p, p += (size_t)nh * nout;
    b3 = p;
    p = g;
    gW1 = p, p += (size_t)nin * nh;
    gb1 = p, p += nh;
    gW2 = p, p += (size_t)nh * nh;
    gb2 = p, p += nh;
    gW3 = p, p += (size_t)nh * nout;
    gb3 = p;
  }

  cudaError_t ensure(int B) {
    if (B <= cap) return cudaSuccess;
    cudaFree(x);
    size_t per = (size_t)nin + 2 * nh + 4 * (size_t)nout + 2 * nh;
    float* base = nullptr;
    cudaError_t e = cudaMalloc(&base, sizeof(float) * (per * B + 4));
    if (e != cudaSuccess) return e;
    x = base;
    h1 = x + (size_t)B * nin;
    h2 = h1 + (size_t)B * nh;
    y = h2 + (size_t)B * nh;
    t = y + (size_t)B * nout;
    mask = t + (size_t)B * nout;
    dy = mask + (size_t)B * nout;
    dh2 = dy + (size_t)B * nout;
    dh1 = dh2 + (size_t)B * nh;
    loss = dh1 + (size_t)B * nh;
    cap = B;
    return cudaSuccess;
  }

  void gemm(const float* A, const float* B, float* C, int M, int N, int K, int lda, int ldb, int ldc, int tA, int tB, const float* bias, int relu,
            int acc = 0) {
    dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
    k_gemm<<<grid, 256, 0, stream>>>(A, B, C, M, N, K, lda, ldb, ldc, tA, tB, bias, relu, acc);
  }

  void forward(int B) {
    gemm(x, W1, h1, B, nh, nin, nin, nh, nh, 0, 0, b1, 1);
    gemm(h1, W2, h2, B, nh, nh, nh, nh, nh, 0, 0, b2, 1);
    gemm(h2, W3, y, B, nout, nh, nh, nout, nout, 0, 0, b3, 0);
  }

  void backward(int B) {
    // dW3 = h2^T dy ; db3 = colsum(dy) ; dh2 = dy W3^T * relu'(h2)
    gemm(h2, dy, gW3, nh, nout, B, nh, nout, nout, 1, 0, nullptr, 0);
    k_colsum<<<(nout + 255) / 256, 256, 0, stream>>>(dy, B, nout, gb3);
    gemm(dy, W3, dh2, B, nh, nout, nout, nout, nh, 0, 1, nullptr, 0);
    k_relu_back<<<128, 256, 0, stream>>>(dh2, h2, (size_t)B * nh);
    gemm(h1, dh2, gW2, nh, nh, B, nh, nh, nh, 1, 0, nullptr, 0);
    k_colsum<<<(nh + 255) / 256, 256, 0, stream>>>(dh2, B, nh, gb2);
    gemm(dh2, W2, dh1, B, nh, nh, nh, nh, nh, 0, 1, nullptr, 0);
    k_relu_back<<<128, 256, 0, stream>>>(dh1, h1, (size_t)B * nh);
    gemm(x, dh1, gW1, nin, nh, B, nin, nh, nh, 1, 0, nullptr, 0);
    k_colsum<<<(nh + 255) / 256, 256, 0, stream>>>(dh1, B, nh, gb1);
  }
};

namespace {
thread_local std::string g_mlp_err;
int mlp_fail(vsgm_mlp* m, const std::string& s) {
  if (m) m->err = s;
  g_mlp_err = s;
  return VSGM_ECUDA;
}
#define MCK(x)                                                                      \
  do {                                                                              \
    cudaError_t e_ = (x);                                                           \
    if (e_ != cudaSuccess) return mlp_fail(m, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)
}  // namespace

extern "C" {

int vsgm_mlp_create(int device, int n_in, int n_hidden, int n_out, uint64_t seed, vsgm_mlp** out) {
  if (!out || n_in < 1 || n_hidden < 1 || n_out < 1) return VSGM_EINVAL;
  vsgm_mlp* m = new vsgm_mlp();
  m->device = device;
  m->nin = n_in;
  m->nh = n_hidden;
  m->nout = n_out;
  m->nparam = (size_t)n_in * n_hidden + n_hidden + (size_t)n_hidden * n_hidden + n_hidden + (size_t)n_hidden * n_out + n_out;
  MCK(cudaSetDevice(device));
  MCK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  MCK(cudaMalloc(&m->w, sizeof(float) * m->nparam * 4));
  m->g = m->w + m->nparam;
  m->m1 = m->g + m->nparam;
  m->m2 = m->m1 + m->nparam;
  m->carve();
  // He-uniform initialisation from a counter-based hash (host side)
  std::vector<float> h(m->nparam, 0.f);
  auto uni = [&](uint64_t i) {
    uint64_t z = seed * 0x9E3779B97F4A7C15ull + i * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) / 9007199254740992.0 * 2.0 - 1.0;
  };
  size_t at = 0;
  auto fill = [&](size_t n, int fan_in) {
    double s = std::sqrt(6.0 / fan_in);
    for (size_t i = 0; i < n; i++, at++) h[at] = (float)(s * uni(at));
  };
  fill((size_t)n_in * n_hidden, n_in);
  at += n_hidden;
  fill((size_t)n_hidden * n_hidden, n_hidden);
  at += n_hidden;
  fill((size_t)n_hidden * n_out, n_hidden);
  MCK(cudaMemcpy(m->w, h.data(), sizeof(float) * m->nparam, cudaMemcpyHostToDevice));
  MCK(cudaMemset(m->m1, 0, sizeof(float) * m->nparam * 2));
  *out = m;
  return VSGM_OK;
}

uint64_t vsgm_mlp_num_params(vsgm_mlp* m) { return m ? m->nparam : 0; }

int vsgm_mlp_get_params(vsgm_mlp* m, float* host) {
  if (!m || !host) return VSGM_EINVAL;
  MCK(cudaMemcpy(host, m->w, sizeof(float) * m->nparam, cudaMemcpyDeviceToHost));
  return VSGM_OK;
}

int vsgm_mlp_set_params(vsgm_mlp* m, const float* host) {
  if (!m || !host) return VSGM_EINVAL;
  MCK(cudaMemcpy(m->w, host, sizeof(float) * m->nparam, cudaMemcpyHostToDevice));
  return VSGM_OK;
}

int vsgm_mlp_forward(vsgm_mlp* m, const float* x, int B, float* y) {
  if (!m || !x || !y || B < 1) return VSGM_EINVAL;
  MCK(cudaSetDevice(m->device));
  MCK(m->ensure(B));
  MCK(cudaMemcpyAsync(m->x, x, sizeof(float) * (size_t)B * m->nin, cudaMemcpyHostToDevice, m->stream));
  m->forward(B);
  MCK(cudaGetLastError());
  MCK(cudaMemcpyAsync(y, m->y, sizeof(float) * (size_t)B * m->nout, cudaMemcpyDeviceToHost, m->stream));
  MCK(cudaStreamSynchronize(m->stream));
  return VSGM_OK;
}

int vsgm_mlp_gradients(vsgm_mlp* m, const float* x, const float* target, const float* mask, int B, float* loss, float* grads) {
  if (!m || !x || !target || !mask || B < 1) return VSGM_EINVAL;
  MCK(cudaSetDevice(m->device));
  MCK(m->ensure(B));
  const size_t ny = (size_t)B * m->nout;
  MCK(cudaMemcpyAsync(m->x, x, sizeof(float) * (size_t)B * m->nin, cudaMemcpyHostToDevice, m->stream));
  MCK(cudaMemcpyAsync(m->t, target, sizeof(float) * ny, cudaMemcpyHostToDevice, m->stream));
  MCK(cudaMemcpyAsync(m->mask, mask, sizeof(float) * ny, cudaMemcpyHostToDevice, m->stream));
  double msum = 0;
  for (size_t i = 0; i < ny; i++) msum += mask[i];
  m->forward(B);
  MCK(cudaMemsetAsync(m->loss, 0, sizeof(float), m->stream));
  k_mse<<<128, 256, 0, m->stream>>>(m->y, m->t, m->mask, ny, (float)(1.0 / std::max(1.0, msum)), m->dy, m->loss);
  m->backward(B);
  MCK(cudaGetLastError());
  if (loss) MCK(cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  if (grads) MCK(cudaMemcpyAsync(grads, m->g, sizeof(float) * m->nparam, cudaMemcpyDeviceToHost, m->stream));
  MCK(cudaStreamSynchronize(m->stream));
  return VSGM_OK;
}

int vsgm_mlp_train_step(vsgm_mlp* m, const float* x, const float* target, const float* mask, int B, float lr, float* loss) {
  int rc = vsgm_mlp_gradients(m, x, target, mask, B, loss, nullptr);
  if (rc) return rc;
  m->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
  k_adam<<<256, 256, 0, m->stream>>>(m->w, m->g, m->m1, m->m2, m->nparam, lr, b1, b2, 1e-8f, c1, c2);
  MCK(cudaGetLastError());
  MCK(cudaStreamSynchronize(m->stream));
  return VSGM_OK;
}

const char* vsgm_mlp_error(vsgm_mlp* m) { return m ? m->err.c_str() : g_mlp_err.c_str(); }

int vsgm_mlp_destroy(vsgm_mlp* m) {
  if (!m) return VSGM_OK;
  cudaSetDevice(m->device);
  cudaFree(m->w);
  cudaFree(m->x);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return VSGM_OK;
}

}  // extern "C"
