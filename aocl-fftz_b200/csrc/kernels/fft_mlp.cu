// Learned plan selector: a small MLP (F -> 64 -> 64 -> 1, ReLU) that predicts
// the log execution time of a candidate plan from its features. Forward pass,
// backward pass (parameter gradients of the mean squared error) and the Adam
// update are plain CUDA kernels; every reduction runs in a fixed order, so a
// training run is bitwise reproducible. No transform result depends on it: it
// only ranks candidate plans, and the exhaustive autotuner stays the fallback.
//
// Parameter layout (float32, contiguous): W1[F][H], b1[H], W2[H][H], b2[H],
// w3[H], b3[1], H = 64; y = w3 . relu(W2^T relu(W1^T x + b1) + b2) + b3.
#include <cuda_runtime.h>
#include <stdint.h>

#define FZ_H 64

namespace fftz {

// Y[b][j] = act(bias[j] + sum_i X[b][i] W[i][j])
__global__ void mlp_dense_fwd(const float *__restrict__ X, int B, int I, const float *__restrict__ W,
                              const float *__restrict__ bias, int O, float *__restrict__ Y, int relu) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)B * O) return;
  const int b = (int)(g / O), j = (int)(g - (int64_t)b * O);
  float s = bias[j];
  for (int i = 0; i < I; i++) s = fmaf(X[(int64_t)b * I + i], W[(int64_t)i * O + j], s);
  Y[g] = (relu && s < 0.f) ? 0.f : s;
}

// dW[i][j] = sum_b X[b][i] D[b][j];  dbias[j] = sum_b D[b][j]  (thread per (i, j))
__global__ void mlp_dense_bwd_w(const float *__restrict__ X, const float *__restrict__ D, int B, int I, int O,
                                float *__restrict__ dW, float *__restrict__ dbias) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (I + 1) * O) return;
  const int i = g / O, j = g - i * O;
  float s = 0.f;
  if (i < I) {
    for (int b = 0; b < B; b++) s = fmaf(X[(int64_t)b * I + i], D[(int64_t)b * O + j], s);
    dW[(int64_t)i * O + j] = s;
  } else {
    for (int b = 0; b < B; b++) s += D[(int64_t)b * O + j];
    dbias[j] = s;
  }
}

// DX[b][i] = [A[b][i] > 0] * sum_j D[b][j] W[i][j]  (A: the ReLU output feeding this layer)
__global__ void mlp_dense_bwd_x(const float *__restrict__ D, const float *__restrict__ W, const float *__restrict__ A,
                                int B, int I, int O, float *__restrict__ DX) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)B * I) return;
  const int b = (int)(g / I), i = (int)(g - (int64_t)b * I);
  float s = 0.f;
  for (int j = 0; j < O; j++) s = fmaf(D[(int64_t)b * O + j], W[(int64_t)i * O + j], s);
  DX[g] = A[g] > 0.f ? s : 0.f;
}

// d[b] = 2 (y[b] - t[b]) / B and loss = mean (y - t)^2 (one block, fixed order)
__global__ void mlp_mse(const float *__restrict__ y, const float *__restrict__ t, int B, float *__restrict__ d,
                        float *__restrict__ loss) {
  __shared__ float part[256];
  float s = 0.f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const float e = y[b] - t[b];
    d[b] = 2.f * e / (float)B;
    s = fmaf(e, e, s);
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = part[0] / (float)B;
}

__global__ void mlp_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                         float *__restrict__ v, int n, float lr, float c1, float c2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float b1 = 0.9f, b2 = 0.999f;
  const float mk = b1 * m[k] + (1.f - b1) * g[k];
  const float vk = b2 * v[k] + (1.f - b2) * g[k] * g[k];
  m[k] = mk;
  v[k] = vk;
  p[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + 1e-8f);
}

}  // namespace fftz

static unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

extern "C" {

int aoclfftz_gpu_mlp_nparams(int F) { return F * FZ_H + FZ_H + FZ_H * FZ_H + FZ_H + FZ_H + 1; }

/* work: at least 2 * B * 64 floats */
int aoclfftz_gpu_mlp_forward(const float *params, int F, const float *X, int B, float *y, float *work,
                             void *stream) {
  if (!params || !X || !y || !work || F < 1 || B < 1) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  const float *W1 = params, *b1 = W1 + F * FZ_H, *W2 = b1 + FZ_H, *b2 = W2 + FZ_H * FZ_H, *w3 = b2 + FZ_H,
              *b3 = w3 + FZ_H;
  float *H1 = work, *H2 = work + (int64_t)B * FZ_H;
  fftz::mlp_dense_fwd<<<nblk((int64_t)B * FZ_H, 256), 256, 0, st>>>(X, B, F, W1, b1, FZ_H, H1, 1);
  fftz::mlp_dense_fwd<<<nblk((int64_t)B * FZ_H, 256), 256, 0, st>>>(H1, B, FZ_H, W2, b2, FZ_H, H2, 1);
  fftz::mlp_dense_fwd<<<nblk(B, 256), 256, 0, st>>>(H2, B, FZ_H, w3, b3, 1, y, 0);
  return (int)cudaGetLastError();
}

/* Gradients of the mean squared error over the batch into grads (same layout
 * as params); loss (device float) receives the loss. work: at least
 * 4 * B * 64 + 2 * B floats. */
int aoclfftz_gpu_mlp_grad(const float *params, int F, const float *X, const float *t, int B, float *grads,
                          float *loss, float *work, void *stream) {
  if (!params || !X || !t || !grads || !loss || !work || F < 1 || B < 1) return -1;
  cudaStream_t st = (cudaStream_t)stream;
  const float *W1 = params, *W2 = W1 + F * FZ_H + FZ_H, *w3 = W2 + FZ_H * FZ_H + FZ_H;
  float *gW1 = grads, *gb1 = gW1 + F * FZ_H, *gW2 = gb1 + FZ_H, *gb2 = gW2 + FZ_H * FZ_H, *gw3 = gb2 + FZ_H,
        *gb3 = gw3 + FZ_H;
  float *H1 = work, *H2 = H1 + (int64_t)B * FZ_H, *D2 = H2 + (int64_t)B * FZ_H, *D1 = D2 + (int64_t)B * FZ_H;
  float *y = D1 + (int64_t)B * FZ_H, *dy = y + B;
  int e = aoclfftz_gpu_mlp_forward(params, F, X, B, y, work, stream);
  if (e) return e;
  fftz::mlp_mse<<<1, 256, 0, st>>>(y, t, B, dy, loss);
  fftz::mlp_dense_bwd_w<<<nblk((FZ_H + 1) * 1, 256), 256, 0, st>>>(H2, dy, B, FZ_H, 1, gw3, gb3);
  fftz::mlp_dense_bwd_x<<<nblk((int64_t)B * FZ_H, 256), 256, 0, st>>>(dy, w3, H2, B, FZ_H, 1, D2);
  fftz::mlp_dense_bwd_w<<<nblk((FZ_H + 1) * FZ_H, 256), 256, 0, st>>>(H1, D2, B, FZ_H, FZ_H, gW2, gb2);
  fftz::mlp_dense_bwd_x<<<nblk((int64_t)B * FZ_H, 256), 256, 0, st>>>(D2, W2, H1, B, FZ_H, FZ_H, D1);
  fftz::mlp_dense_bwd_w<<<nblk((int64_t)(F + 1) * FZ_H, 256), 256, 0, st>>>(X, D1, B, F, FZ_H, gW1, gb1);
  return (int)cudaGetLastError();
}

/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8); step counts from 1. */
int aoclfftz_gpu_mlp_adam(float *params, const float *grads, float *m, float *v, int n, float lr, int step,
                          void *stream) {
  if (!params || !grads || !m || !v || n < 1 || step < 1) return -1;
  const float c1 = 1.f - powf(0.9f, (float)step), c2 = 1.f - powf(0.999f, (float)step);
  fftz::mlp_adam<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(params, grads, m, v, n, lr, c1, c2);
  return (int)cudaGetLastError();
}

}  // extern "C"
