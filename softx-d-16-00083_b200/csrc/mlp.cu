// A small multilayer perceptron trained on the GPU with hand-written kernels: the learned binning
// correction of the coarse-histogram I(q) (no reference counterpart; xns_b200/learned.py drives it).
//
//   h1 = gelu(W1 x + b1),  h2 = gelu(W2 h1 + b2),  y = W3 h2 + b3        (3 linear layers)
//
// Weights are kept as FP32 master copies (Adam state alongside) and used in BF16 by the forward and
// backward products, which accumulate in FP32.  Activations, gradients and losses are FP32.  GELU is
// the erf form, 0.5 x (1 + erf(x / sqrt 2)), with derivative Phi(x) + x phi(x).
//
// Products are small (batch <= a few thousand, widths <= a few thousand), so one SIMT kernel serves
// every GEMM of the forward and backward passes: C[M x N] = A[M x K] B[K x N] (+ bias) with arbitrary
// strides, 64 x 64 output tiles, 16-deep K steps staged in shared memory, 4 x 4 outputs per thread.
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "xns_internal.cuh"

namespace {

constexpr int GT = 64, GK = 16;

// A element (m, k) at A[m * sam + k * sak]; B element (k, n) at B[k * sbk + n * sbn].
template <class TA, class TB>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const TA *__restrict__ A, long sam, long sak,
                                                   const TB *__restrict__ B, long sbk, long sbn, float *__restrict__ C,
                                                   long ldc, const float *__restrict__ bias, float beta) {
  __shared__ float As[GK][GT + 1], Bs[GK][GT + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += GK) {
    for (int e = threadIdx.x; e < GT * GK; e += 256) {
      const int r = e / GK, c = e % GK;  // A: row r of the tile, k c
      const int m = m0 + r, k = k0 + c;
      As[c][r] = (m < M && k < K) ? (float)A[m * sam + k * sak] : 0.f;
      const int n = n0 + r;  // B: column r of the tile, k c
      Bs[c][r] = (n < N && k < K) ? (float)B[k * sbk + n * sbn] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < GK; c++) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[c][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[c][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      float v = acc[i][j] + (bias ? bias[n] : 0.f);
      if (beta != 0.f) v += beta * C[m * ldc + n];
      C[m * ldc + n] = v;
    }
  }
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

__global__ void gelu_kernel(const float *__restrict__ z, float *__restrict__ h, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) h[i] = gelu(z[i]);
}
// dz = dh * gelu'(z)
__global__ void gelu_back_kernel(const float *__restrict__ z, const float *__restrict__ dh, float *__restrict__ dz, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    dz[i] = dh[i] * gelu_grad(z[i]);
}
// loss = mean over all entries of w (y - t)^2 (w: per output column, may be null = 1); dy = d loss / d y
__global__ void mse_kernel(const float *__restrict__ y, const float *__restrict__ t, const float *__restrict__ w, int B,
                           int N, float *__restrict__ dy, double *__restrict__ loss) {
  __shared__ double red[256];
  double s = 0;
  const long n = (long)B * N;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float wi = w ? w[i % N] : 1.f;
    const float d = y[i] - t[i];
    s += (double)wi * d * d;
    dy[i] = 2.f * wi * d / (float)n;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] / (double)n);
}
// db[n] = sum_b dy[b][n]
__global__ void colsum_kernel(const float *__restrict__ dy, int B, int N, float *__restrict__ db) {
  const int nn = blockIdx.x * blockDim.x + threadIdx.x;
  if (nn >= N) return;
  float s = 0.f;
  for (int b = 0; b < B; b++) s += dy[(long)b * N + nn];
  db[nn] = s;
}
// Adam on FP32 masters; refreshes the BF16 copy.
__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                            __nv_bfloat16 *__restrict__ pb, long n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (pb) pb[i] = __float2bfloat16_rn(pi);
  }
}
__global__ void to_bf16_kernel(const float *__restrict__ p, __nv_bfloat16 *__restrict__ pb, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    pb[i] = __float2bfloat16_rn(p[i]);
}

}  // namespace

struct xns_mlp {
  xns_ctx *ctx = nullptr;
  int dims[4] = {};  // in, hidden, hidden, out
  // parameters (FP32 masters, then gradients, Adam m and v), one block each: W1 b1 W2 b2 W3 b3
  float *P = nullptr, *Gr = nullptr, *Mo = nullptr, *Ve = nullptr;
  __nv_bfloat16 *Wb = nullptr;  // BF16 copies of W1, W2, W3 (offsets as in P)
  long off[7] = {};             // W1 b1 W2 b2 W3 b3 | total
  long step = 0;
  // activations for a batch of up to cap rows
  int cap = 0;
  float *X = nullptr, *Z1 = nullptr, *H1 = nullptr, *Z2 = nullptr, *H2 = nullptr, *Y = nullptr, *T = nullptr, *D = nullptr,
        *D2 = nullptr, *Wt = nullptr;
  double *loss = nullptr;
};

namespace {

int grid_for(long n) { return (int)std::min<long>((n + 255) / 256, 4096); }

// C[M x N] (+)= A B, A (M x K) FP32 or BF16 with strides, B likewise.
template <class TA, class TB>
int gemm(xns_ctx *ctx, int M, int N, int K, const TA *A, long sam, long sak, const TB *B, long sbk, long sbn, float *C,
         long ldc, const float *bias, float beta) {
  dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT);
  gemm_kernel<TA, TB><<<grid, 256, 0, ctx->stream>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, bias, beta);
  XNS_LAUNCHED(ctx);
  return XNS_OK;
}

int ensure_batch(xns_mlp *m, int B) {
  if (B <= m->cap) return XNS_OK;
  xns_ctx *ctx = m->ctx;
  float *bufs[] = {m->X, m->Z1, m->H1, m->Z2, m->H2, m->Y, m->T, m->D, m->D2};
  for (float *p : bufs)
    if (p) cudaFree(p);
  const int in = m->dims[0], h = m->dims[1], h2 = m->dims[2], out = m->dims[3];
  const int wmax = std::max(std::max(in, h), std::max(h2, out));
  auto alloc = [&](float **p, long n) -> int {
    XNS_CUDA(ctx, cudaMalloc(p, sizeof(float) * n));
    return XNS_OK;
  };
  int st;
  if ((st = alloc(&m->X, (long)B * in)) || (st = alloc(&m->Z1, (long)B * h)) || (st = alloc(&m->H1, (long)B * h)) ||
      (st = alloc(&m->Z2, (long)B * h2)) || (st = alloc(&m->H2, (long)B * h2)) || (st = alloc(&m->Y, (long)B * out)) ||
      (st = alloc(&m->T, (long)B * out)) || (st = alloc(&m->D, (long)B * wmax)) || (st = alloc(&m->D2, (long)B * wmax)))
    return st;
  m->cap = B;
  return XNS_OK;
}

int forward(xns_mlp *m, int B) {
  xns_ctx *ctx = m->ctx;
  const int in = m->dims[0], h1 = m->dims[1], h2 = m->dims[2], out = m->dims[3];
  int st;
  // Z1 = X W1^T + b1: A = X (B x in), B-operand (k, n) = W1[n][k]
  if ((st = gemm(ctx, B, h1, in, m->X, in, 1, m->Wb + m->off[0], 1, in, m->Z1, h1, m->P + m->off[1], 0.f))) return st;
  gelu_kernel<<<grid_for((long)B * h1), 256, 0, ctx->stream>>>(m->Z1, m->H1, (long)B * h1);
  XNS_LAUNCHED(ctx);
  if ((st = gemm(ctx, B, h2, h1, m->H1, h1, 1, m->Wb + m->off[2], 1, h1, m->Z2, h2, m->P + m->off[3], 0.f))) return st;
  gelu_kernel<<<grid_for((long)B * h2), 256, 0, ctx->stream>>>(m->Z2, m->H2, (long)B * h2);
  XNS_LAUNCHED(ctx);
  return gemm(ctx, B, out, h2, m->H2, h2, 1, m->Wb + m->off[4], 1, h2, m->Y, out, m->P + m->off[5], 0.f);
}

// Gradients of mean w (Y - T)^2 into Gr; the loss into *m->loss.
int backward(xns_mlp *m, int B, const float *d_w) {
  xns_ctx *ctx = m->ctx;
  const int in = m->dims[0], h1 = m->dims[1], h2 = m->dims[2], out = m->dims[3];
  int st;
  XNS_CUDA(ctx, cudaMemsetAsync(m->loss, 0, sizeof(double), ctx->stream));
  mse_kernel<<<grid_for((long)B * out), 256, 0, ctx->stream>>>(m->Y, m->T, d_w, B, out, m->D, m->loss);
  XNS_LAUNCHED(ctx);
  // layer 3: dW3 = dY^T H2 (out x h2), db3 = colsum dY, dH2 = dY W3
  if ((st = gemm(ctx, out, h2, B, m->D, 1, out, m->H2, h2, 1, m->Gr + m->off[4], h2, nullptr, 0.f))) return st;
  colsum_kernel<<<(out + 255) / 256, 256, 0, ctx->stream>>>(m->D, B, out, m->Gr + m->off[5]);
  XNS_LAUNCHED(ctx);
  if ((st = gemm(ctx, B, h2, out, m->D, out, 1, m->Wb + m->off[4], h2, 1, m->D2, h2, nullptr, 0.f))) return st;
  gelu_back_kernel<<<grid_for((long)B * h2), 256, 0, ctx->stream>>>(m->Z2, m->D2, m->D2, (long)B * h2);
  XNS_LAUNCHED(ctx);
  // layer 2
  if ((st = gemm(ctx, h2, h1, B, m->D2, 1, h2, m->H1, h1, 1, m->Gr + m->off[2], h1, nullptr, 0.f))) return st;
  colsum_kernel<<<(h2 + 255) / 256, 256, 0, ctx->stream>>>(m->D2, B, h2, m->Gr + m->off[3]);
  XNS_LAUNCHED(ctx);
  if ((st = gemm(ctx, B, h1, h2, m->D2, h2, 1, m->Wb + m->off[2], h1, 1, m->D, h1, nullptr, 0.f))) return st;
  gelu_back_kernel<<<grid_for((long)B * h1), 256, 0, ctx->stream>>>(m->Z1, m->D, m->D, (long)B * h1);
  XNS_LAUNCHED(ctx);
  // layer 1
  if ((st = gemm(ctx, h1, in, B, m->D, 1, h1, m->X, in, 1, m->Gr + m->off[0], in, nullptr, 0.f))) return st;
  colsum_kernel<<<(h1 + 255) / 256, 256, 0, ctx->stream>>>(m->D, B, h1, m->Gr + m->off[1]);
  XNS_LAUNCHED(ctx);
  return XNS_OK;
}

void mlp_free(xns_mlp *m) {
  if (!m) return;
  float *bufs[] = {m->P, m->Gr, m->Mo, m->Ve, m->X, m->Z1, m->H1, m->Z2, m->H2, m->Y, m->T, m->D, m->D2};
  for (float *p : bufs)
    if (p) cudaFree(p);
  if (m->Wb) cudaFree(m->Wb);
  if (m->loss) cudaFree(m->loss);
  if (m->ctx) xns_destroy(m->ctx);
  delete m;
}

}  // namespace

extern "C" {

// dims: in, hidden, hidden, out.  Weights ~ U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from a seeded
// generator (the host fills them; xns_mlp_set_params replaces them).
int xns_mlp_create(xns_ctx *parent, const int *dims, uint64_t seed, xns_mlp **out) {
  if (!parent || !dims || !out) return XNS_ERR_ARG;
  *out = nullptr;
  for (int i = 0; i < 4; i++)
    if (dims[i] <= 0) return xns_fail(parent, XNS_ERR_ARG, "mlp: non-positive width");
  xns_mlp *m = new xns_mlp();
  int st = xns_create(parent->device, &m->ctx);
  if (st) {
    parent->err = "mlp: " + std::string(xns_last_error(m->ctx));
    mlp_free(m);
    return st;
  }
  memcpy(m->dims, dims, sizeof(m->dims));
  const long sizes[6] = {(long)dims[1] * dims[0], dims[1], (long)dims[2] * dims[1], dims[2], (long)dims[3] * dims[2], dims[3]};
  m->off[0] = 0;
  for (int i = 0; i < 6; i++) m->off[i + 1] = m->off[i] + sizes[i];
  const long n = m->off[6];
  std::vector<float> host(n);
  uint64_t s = seed * 6364136223846793005ull + 1442695040888963407ull;
  const int fan[6] = {dims[0], dims[0], dims[1], dims[1], dims[2], dims[2]};
  for (int i = 0; i < 6; i++) {
    const float a = 1.f / sqrtf((float)fan[i]);
    for (long j = m->off[i]; j < m->off[i + 1]; j++) {
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      host[j] = a * (2.f * (float)((s >> 40) * (1.0 / 16777216.0)) - 1.f);
    }
  }
  xns_ctx *ctx = m->ctx;
  auto fail = [&](cudaError_t e) {
    parent->err = std::string("mlp: ") + cudaGetErrorString(e);
    mlp_free(m);
    return XNS_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaMalloc(&m->P, sizeof(float) * n)) || (e = cudaMalloc(&m->Gr, sizeof(float) * n)) ||
      (e = cudaMalloc(&m->Mo, sizeof(float) * n)) || (e = cudaMalloc(&m->Ve, sizeof(float) * n)) ||
      (e = cudaMalloc(&m->Wb, sizeof(__nv_bfloat16) * n)) || (e = cudaMalloc(&m->loss, sizeof(double))))
    return fail(e);
  if ((e = cudaMemcpy(m->P, host.data(), sizeof(float) * n, cudaMemcpyHostToDevice)) ||
      (e = cudaMemset(m->Mo, 0, sizeof(float) * n)) || (e = cudaMemset(m->Ve, 0, sizeof(float) * n)))
    return fail(e);
  to_bf16_kernel<<<grid_for(n), 256, 0, ctx->stream>>>(m->P, m->Wb, n);
  if ((e = cudaStreamSynchronize(ctx->stream))) return fail(e);
  *out = m;
  return XNS_OK;
}

void xns_mlp_destroy(xns_mlp *m) { mlp_free(m); }

const char *xns_mlp_last_error(const xns_mlp *m) { return m ? xns_last_error(m->ctx) : "null network"; }

long xns_mlp_param_count(const xns_mlp *m) { return m ? m->off[6] : 0; }

// Parameters in the order W1 (hidden x in), b1, W2, b2, W3, b3, as FP32 masters.
int xns_mlp_get_params(xns_mlp *m, float *p) {
  if (!m || !p) return XNS_ERR_ARG;
  XNS_CUDA(m->ctx, cudaMemcpy(p, m->P, sizeof(float) * m->off[6], cudaMemcpyDeviceToHost));
  return XNS_OK;
}

int xns_mlp_set_params(xns_mlp *m, const float *p) {
  if (!m || !p) return XNS_ERR_ARG;
  XNS_CUDA(m->ctx, cudaMemcpy(m->P, p, sizeof(float) * m->off[6], cudaMemcpyHostToDevice));
  to_bf16_kernel<<<grid_for(m->off[6]), 256, 0, m->ctx->stream>>>(m->P, m->Wb, m->off[6]);
  XNS_LAUNCHED(m->ctx);
  XNS_CUDA(m->ctx, cudaStreamSynchronize(m->ctx->stream));
  m->step = 0;
  XNS_CUDA(m->ctx, cudaMemset(m->Mo, 0, sizeof(float) * m->off[6]));
  XNS_CUDA(m->ctx, cudaMemset(m->Ve, 0, sizeof(float) * m->off[6]));
  return XNS_OK;
}

// y (B x out) = network(x (B x in)), host buffers.
int xns_mlp_forward(xns_mlp *m, const float *x, int B, float *y) {
  if (!m || !x || !y || B <= 0) return XNS_ERR_ARG;
  int st;
  if ((st = ensure_batch(m, B))) return st;
  XNS_CUDA(m->ctx, cudaMemcpyAsync(m->X, x, sizeof(float) * B * m->dims[0], cudaMemcpyHostToDevice, m->ctx->stream));
  if ((st = forward(m, B))) return st;
  XNS_CUDA(m->ctx, cudaMemcpyAsync(y, m->Y, sizeof(float) * B * m->dims[3], cudaMemcpyDeviceToHost, m->ctx->stream));
  XNS_CUDA(m->ctx, cudaStreamSynchronize(m->ctx->stream));
  return XNS_OK;
}

// Gradients of mean w (y - t)^2 with respect to every parameter (host buffer, parameter order), and
// the loss.  w: per output column weights (null: 1).
int xns_mlp_gradients(xns_mlp *m, const float *x, const float *t, const float *w, int B, float *grad, double *loss) {
  if (!m || !x || !t || B <= 0) return XNS_ERR_ARG;
  int st;
  if ((st = ensure_batch(m, B))) return st;
  xns_ctx *ctx = m->ctx;
  float *d_w = nullptr;
  if (w) {
    XNS_CUDA(ctx, cudaMalloc(&d_w, sizeof(float) * m->dims[3]));
    XNS_CUDA(ctx, cudaMemcpyAsync(d_w, w, sizeof(float) * m->dims[3], cudaMemcpyHostToDevice, ctx->stream));
  }
  XNS_CUDA(ctx, cudaMemcpyAsync(m->X, x, sizeof(float) * B * m->dims[0], cudaMemcpyHostToDevice, ctx->stream));
  XNS_CUDA(ctx, cudaMemcpyAsync(m->T, t, sizeof(float) * B * m->dims[3], cudaMemcpyHostToDevice, ctx->stream));
  if ((st = forward(m, B)) || (st = backward(m, B, d_w))) return st;
  if (grad) XNS_CUDA(ctx, cudaMemcpyAsync(grad, m->Gr, sizeof(float) * m->off[6], cudaMemcpyDeviceToHost, ctx->stream));
  if (loss) XNS_CUDA(ctx, cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (d_w) cudaFree(d_w);
  return XNS_OK;
}

// steps Adam steps over the given data (n rows), mini-batches of B rows in order (the host shuffles).
// Returns the mean loss of the last epoch's batches in *loss.
int xns_mlp_train(xns_mlp *m, const float *x, const float *t, const float *w, int n, int B, int epochs, float lr,
                  double *loss) {
  if (!m || !x || !t || n <= 0 || B <= 0 || epochs <= 0) return XNS_ERR_ARG;
  xns_ctx *ctx = m->ctx;
  int st;
  if ((st = ensure_batch(m, B))) return st;
  const int in = m->dims[0], out = m->dims[3];
  float *dx = nullptr, *dt = nullptr, *d_w = nullptr;
  XNS_CUDA(ctx, cudaMalloc(&dx, sizeof(float) * (long)n * in));
  XNS_CUDA(ctx, cudaMalloc(&dt, sizeof(float) * (long)n * out));
  XNS_CUDA(ctx, cudaMemcpyAsync(dx, x, sizeof(float) * (long)n * in, cudaMemcpyHostToDevice, ctx->stream));
  XNS_CUDA(ctx, cudaMemcpyAsync(dt, t, sizeof(float) * (long)n * out, cudaMemcpyHostToDevice, ctx->stream));
  if (w) {
    XNS_CUDA(ctx, cudaMalloc(&d_w, sizeof(float) * out));
    XNS_CUDA(ctx, cudaMemcpyAsync(d_w, w, sizeof(float) * out, cudaMemcpyHostToDevice, ctx->stream));
  }
  double sum = 0;
  int batches = 0;
  for (int ep = 0; ep < epochs; ep++) {
    sum = 0;
    batches = 0;
    for (int b0 = 0; b0 + B <= n; b0 += B) {
      XNS_CUDA(ctx, cudaMemcpyAsync(m->X, dx + (long)b0 * in, sizeof(float) * (long)B * in, cudaMemcpyDeviceToDevice,
                                    ctx->stream));
      XNS_CUDA(ctx, cudaMemcpyAsync(m->T, dt + (long)b0 * out, sizeof(float) * (long)B * out, cudaMemcpyDeviceToDevice,
                                    ctx->stream));
      if ((st = forward(m, B)) || (st = backward(m, B, d_w))) return st;
      m->step++;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.f - powf(b1, (float)m->step), c2 = 1.f - powf(b2, (float)m->step);
      adam_kernel<<<grid_for(m->off[6]), 256, 0, ctx->stream>>>(m->P, m->Gr, m->Mo, m->Ve, m->Wb, m->off[6], lr, b1, b2,
                                                                1e-8f, c1, c2);
      XNS_LAUNCHED(ctx);
      double l = 0;
      XNS_CUDA(ctx, cudaMemcpyAsync(&l, m->loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      XNS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      sum += l;
      batches++;
    }
  }
  // biases have BF16 copies too (unused by the products, kept consistent with the masters)
  cudaFree(dx);
  cudaFree(dt);
  if (d_w) cudaFree(d_w);
  if (loss) *loss = batches ? sum / batches : 0.0;
  return XNS_OK;
}

}  // extern "C"
