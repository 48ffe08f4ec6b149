// es_net.cu -- the learned early-stop network: a 1-D convolutional stack and
// an MLP head over the early port transient, with hand-written training and
// inference kernels.  Weights live as FP32 master values plus BF16 copies; the
// forward and backward passes read the BF16 copies and accumulate in FP32.
//
// Every layer is one GEMM: a convolution is an im2col gather followed by
// out[(b,t)][co] = sum_{k,ci} cols[(b,t)][k*cin+ci] * W[co][k][ci], a dense
// layer is out[b][o] = sum_i in[b][i] * W[o][i].  Activations are stored time
// major with the channel fastest, so a convolution's GEMM output is directly
// the next layer's input.  All reductions run in a fixed order (split sums are
// combined by a second pass, never by atomics), so training is reproducible.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/fdtd_b200.h"
#include "fdtd_internal.h"

namespace {

int es_fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return fdtd_internal_fail(code, buf);
}

#define ES_CK(call)                                                                                    \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess) return es_fail(FDTD_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));     \
  } while (0)

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ float ld(const float* p) { return *p; }
__device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }

constexpr int kTM = 64, kTN = 64, kTK = 16;

// C = op(A) op(B) (+ bias, ReLU).  op(A)[m][k] = TA ? A[k*lda+m] : A[m*lda+k];
// op(B)[k][n] = TB ? B[n*ldb+k] : B[k*ldb+n].  blockIdx.z selects a slice of
// the k range (kchunk wide) whose partial result goes to C + z*c_split; bias
// and ReLU are applied only when there is a single slice.
template <bool TA, bool TB, typename TAe, typename TBe>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const TAe* __restrict__ A, int lda,
                                              const TBe* __restrict__ B, int ldb, float* __restrict__ Cm, int ldc,
                                              long long c_split, int kchunk, const float* __restrict__ bias,
                                              int relu) {
  __shared__ float As[kTK][kTM + 4];
  __shared__ float Bs[kTK][kTN + 4];
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const int m0 = blockIdx.y * kTM, n0 = blockIdx.x * kTN;
  const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
  float acc[4][4];
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) acc[a][b] = 0.f;
  for (int k0 = kbeg; k0 < kend; k0 += kTK) {
    for (int e = tid; e < kTM * kTK; e += 256) {
      int mm, kk;
      if (TA) { mm = e % kTM; kk = e / kTM; } else { kk = e % kTK; mm = e / kTK; }
      const int gm = m0 + mm, gk = k0 + kk;
      float v = 0.f;
      if (gm < M && gk < kend) v = TA ? ld(A + (long long)gk * lda + gm) : ld(A + (long long)gm * lda + gk);
      As[kk][mm] = v;
    }
    for (int e = tid; e < kTN * kTK; e += 256) {
      int nn, kk;
      if (TB) { kk = e % kTK; nn = e / kTK; } else { nn = e % kTN; kk = e / kTN; }
      const int gn = n0 + nn, gk = k0 + kk;
      float v = 0.f;
      if (gn < N && gk < kend) v = TB ? ld(B + (long long)gn * ldb + gk) : ld(B + (long long)gk * ldb + gn);
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTK; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        a[q] = As[kk][ty + 16 * q];
        b[q] = Bs[kk][tx + 16 * q];
      }
#pragma unroll
      for (int p = 0; p < 4; p++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[p][q] = fmaf(a[p], b[q], acc[p][q]);
    }
    __syncthreads();
  }
  float* C = Cm + (long long)blockIdx.z * c_split;
  const bool single = gridDim.z == 1;
#pragma unroll
  for (int p = 0; p < 4; p++) {
    const int m = m0 + ty + 16 * p;
    if (m >= M) continue;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int n = n0 + tx + 16 * q;
      if (n >= N) continue;
      float v = acc[p][q];
      if (single) {
        if (bias) v += bias[n];
        if (relu) v = fmaxf(v, 0.f);
      }
      C[(long long)m * ldc + n] = v;
    }
  }
}

// out[i] = sum over s of part[s*n + i], s in order.
__global__ void k_sum_slices(const float* __restrict__ part, int slices, long long n, float* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int q = 0; q < slices; q++) s += part[(long long)q * n + i];
  out[i] = s;
}

// Column sums of a rows x cols matrix: one block per column, fixed-order tree.
__global__ void __launch_bounds__(256) k_col_sums(const float* __restrict__ x, int rows, int cols,
                                                  float* __restrict__ out) {
  __shared__ float red[256];
  const int c = blockIdx.x;
  float s = 0.f;
  for (int r = threadIdx.x; r < rows; r += 256) s += x[(long long)r * cols + c];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[c] = red[0];
}

// cols[(b*lout + t)][k*cin + c] = in[b][t*stride + k - pad][c] (0 outside).
__global__ void k_im2col(const float* __restrict__ in, int B, int lin, int cin, int lout, int ksz, int stride,
                         int pad, float* __restrict__ cols) {
  const long long w = (long long)ksz * cin;
  const long long n = (long long)B * lout * w;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long row = e / w;
    const int kc = (int)(e % w), k = kc / cin, c = kc % cin;
    const int b = (int)(row / lout), t = (int)(row % lout);
    const int s = t * stride + k - pad;
    cols[e] = (s >= 0 && s < lin) ? in[((long long)b * lin + s) * cin + c] : 0.f;
  }
}

// Adjoint of k_im2col: din[b][s][c] = sum_k dcols[(b*lout + t)][k*cin + c],
// t = (s + pad - k) / stride where that is a whole number in [0, lout).
__global__ void k_col2im(const float* __restrict__ dcols, int B, int lin, int cin, int lout, int ksz, int stride,
                         int pad, float* __restrict__ din) {
  const long long n = (long long)B * lin * cin;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % cin);
    const long long bs = e / cin;
    const int s = (int)(bs % lin), b = (int)(bs / lin);
    float acc = 0.f;
    for (int k = 0; k < ksz; k++) {
      const int num = s + pad - k;
      if (num < 0 || num % stride) continue;
      const int t = num / stride;
      if (t >= lout) continue;
      acc += dcols[((long long)b * lout + t) * ((long long)ksz * cin) + (long long)k * cin + c];
    }
    din[e] = acc;
  }
}

// dpre = dpost * (post > 0), in place.
__global__ void k_relu_back(float* __restrict__ d, const float* __restrict__ post, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !(post[i] > 0.f)) d[i] = 0.f;
}

// Per-sample weighted squared error and dL/dy = 2 w (y - t) / B.
__global__ void k_loss(const float* __restrict__ y, const float* __restrict__ t, const float* __restrict__ w, int B,
                       int D, float* __restrict__ dy, float* __restrict__ per) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  float s = 0.f;
  for (int o = 0; o < D; o++) {
    const float r = y[b * D + o] - t[b * D + o];
    s += w[o] * r * r;
    dy[b * D + o] = 2.f * w[o] * r / (float)B;
  }
  per[b] = s;
}

// Mean of per-sample losses (one block, fixed order).
__global__ void __launch_bounds__(256) k_mean(const float* __restrict__ per, int B, float* __restrict__ out) {
  __shared__ float red[256];
  float s = 0.f;
  for (int b = threadIdx.x; b < B; b += 256) s += per[b];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0] / (float)B;
}

// Adam with decoupled weight decay; refreshes the BF16 compute copy.
__global__ void k_adam(float* __restrict__ p, __nv_bfloat16* __restrict__ p16, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, long long n, float lr, float b1, float b2,
                       float eps, float wd, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float pi = p[i];
  pi -= lr * wd * pi;
  pi -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  p[i] = pi;
  p16[i] = __float2bfloat16_rn(pi);
}

__global__ void k_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ p16, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p16[i] = __float2bfloat16_rn(p[i]);
}

// Minibatch gather from the resident set (block row b = sample b of the batch).
__global__ void k_gather(const float* __restrict__ x, const float* __restrict__ y, const int* __restrict__ idx,
                         int B, int xw, int yw, float* __restrict__ bx, float* __restrict__ by) {
  const int b = blockIdx.y;
  if (b >= B) return;
  const long long s = idx[b];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < xw; e += gridDim.x * blockDim.x)
    bx[(long long)b * xw + e] = x[s * xw + e];
  if (blockIdx.x == 0)
    for (int e = threadIdx.x; e < yw; e += blockDim.x) by[(long long)b * yw + e] = y[s * yw + e];
}

// Network input from the port traces of handle b (block b).
__global__ void __launch_bounds__(256) k_trace_inputs(const double* const* __restrict__ V,
                                                      const double* const* __restrict__ I, int L, int decim,
                                                      float* __restrict__ x, float* __restrict__ scales) {
  __shared__ float red[2][256];
  const int b = blockIdx.x;
  const double* src[2] = {V[b], I[b]};
  float mx[2] = {0.f, 0.f};
  for (int t = threadIdx.x; t < L; t += 256) {
    for (int ch = 0; ch < 2; ch++) {
      double s = 0.0;
      for (int q = 0; q < decim; q++) s += src[ch][(long long)t * decim + q];
      const float v = (float)(s / decim);
      x[((long long)b * L + t) * 2 + ch] = v;
      mx[ch] = fmaxf(mx[ch], fabsf(v));
    }
  }
  red[0][threadIdx.x] = mx[0];
  red[1][threadIdx.x] = mx[1];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      red[0][threadIdx.x] = fmaxf(red[0][threadIdx.x], red[0][threadIdx.x + w]);
      red[1][threadIdx.x] = fmaxf(red[1][threadIdx.x], red[1][threadIdx.x + w]);
    }
    __syncthreads();
  }
  const float s0 = red[0][0] > 0.f ? red[0][0] : 1.f, s1 = red[1][0] > 0.f ? red[1][0] : 1.f;
  for (int t = threadIdx.x; t < L; t += 256) {
    x[((long long)b * L + t) * 2 + 0] /= s0;
    x[((long long)b * L + t) * 2 + 1] /= s1;
  }
  if (threadIdx.x == 0) {
    scales[2 * b] = s0;
    scales[2 * b + 1] = s1;
  }
}

unsigned blocks_for(long long n, int threads = 256) {
  return (unsigned)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 1 << 20));
}

// One GEMM layer of the network.
struct Layer {
  bool conv;
  int cin, cout, lin, lout;  // conv: channels and lengths; dense: lin = lout = 1
  int ksz, stride, pad;
  bool relu;
  long long w_off, b_off;
  long long kdim() const { return conv ? (long long)ksz * cin : cin; }
  long long in_width() const { return (long long)lin * cin; }    // per-sample input values
  long long out_width() const { return (long long)lout * cout; }  // per-sample output values
};

}  // namespace

struct fdtd_es_net {
  FdtdEsConfig cfg{};
  cudaStream_t stream = nullptr;
  std::vector<Layer> layers;
  long long nparam = 0;
  float* p32 = nullptr;
  __nv_bfloat16* p16 = nullptr;
  float *grad = nullptr, *m = nullptr, *v = nullptr;
  std::vector<float*> act;  // act[0] input, act[l+1] output of layer l (max_batch samples)
  float *cols = nullptr, *dcols = nullptr, *da = nullptr, *db = nullptr, *ws = nullptr;
  float *target = nullptr, *wout = nullptr, *dy = nullptr, *per = nullptr, *loss = nullptr;
  float *dset_x = nullptr, *dset_y = nullptr;
  int* d_perm = nullptr;  // shuffled sample order of the current epoch
  long long nsamples = 0;
  float* scales = nullptr;
  const double** d_traces = nullptr;  // [2][max_batch] device pointers
  long long adam_t = 0;
  std::vector<void*> owned;
};

namespace {

int es_alloc(fdtd_es_net* n, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return es_fail(FDTD_ERR_OOM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
  }
  n->owned.push_back(*p);
  e = cudaMemsetAsync(*p, 0, bytes, n->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(n->stream);
  if (e != cudaSuccess) return es_fail(FDTD_ERR_CUDA, "zeroing: %s", cudaGetErrorString(e));
  return FDTD_OK;
}

void es_release(fdtd_es_net* n, void* p) {
  if (!p) return;
  cudaFree(p);
  n->owned.erase(std::remove(n->owned.begin(), n->owned.end(), p), n->owned.end());
}

template <bool TA, bool TB, typename TAe, typename TBe>
void gemm(fdtd_es_net* n, int M, int N, int K, const TAe* A, int lda, const TBe* B, int ldb, float* C, int ldc,
          const float* bias, bool relu, int slices = 1, long long c_split = 0) {
  const int kchunk = ((K + slices - 1) / slices + kTK - 1) / kTK * kTK;
  const dim3 grd((N + kTN - 1) / kTN, (M + kTM - 1) / kTM, slices);
  k_gemm<TA, TB, TAe, TBe><<<grd, 256, 0, n->stream>>>(M, N, K, A, lda, B, ldb, C, ldc, c_split, kchunk, bias,
                                                       relu ? 1 : 0);
}

// Forward pass of B samples already in act[0].
void forward(fdtd_es_net* n, int B) {
  for (size_t l = 0; l < n->layers.size(); l++) {
    const Layer& L = n->layers[l];
    const __nv_bfloat16* W = n->p16 + L.w_off;
    const float* bias = n->p32 + L.b_off;  // biases stay FP32
    if (L.conv) {
      const long long e = (long long)B * L.lout * L.kdim();
      k_im2col<<<blocks_for(e), 256, 0, n->stream>>>(n->act[l], B, L.lin, L.cin, L.lout, L.ksz, L.stride, L.pad,
                                                      n->cols);
      gemm<false, true>(n, B * L.lout, L.cout, (int)L.kdim(), (const float*)n->cols, (int)L.kdim(), W,
                        (int)L.kdim(), n->act[l + 1], L.cout, bias, L.relu);
    } else {
      gemm<false, true>(n, B, L.cout, L.cin, (const float*)n->act[l], L.cin, W, L.cin, n->act[l + 1], L.cout, bias,
                        L.relu);
    }
  }
}

// Number of row slices the weight-gradient reduction over `rows` is split into.
long long grad_slices(long long rows) { return std::max<long long>(1, std::min<long long>(64, rows / 512)); }

// dW (and db) of one layer from dpre (rows x cout) and its input matrix X (rows x kdim).
void weight_grads(fdtd_es_net* n, const Layer& L, const float* dpre, const float* X, int rows) {
  const int N = L.cout, K = (int)L.kdim();
  const int slices = (int)grad_slices(rows);
  float* gW = n->grad + L.w_off;
  if (slices == 1) {
    gemm<true, false>(n, N, K, rows, dpre, N, X, K, gW, K, nullptr, false);
  } else {
    // slice s sums its own range of rows; the slices are then added in order
    gemm<true, false>(n, N, K, rows, dpre, N, X, K, n->ws, K, nullptr, false, slices, (long long)N * K);
    k_sum_slices<<<blocks_for((long long)N * K), 256, 0, n->stream>>>(n->ws, slices, (long long)N * K, gW);
  }
  k_col_sums<<<N, 256, 0, n->stream>>>(dpre, rows, N, n->grad + L.b_off);
}

// Backward pass: dy (B x out_dim) -> n->grad.  Activations of the forward pass
// are still in act[]; the im2col matrix of each convolution is rebuilt.
void backward(fdtd_es_net* n, int B) {
  float* dcur = n->dy;  // gradient with respect to the current layer's output
  float* bufs[2] = {n->da, n->db};
  int flip = 0;
  for (int l = (int)n->layers.size() - 1; l >= 0; l--) {
    const Layer& L = n->layers[l];
    const int rows = L.conv ? B * L.lout : B;
    if (L.relu)
      k_relu_back<<<blocks_for((long long)rows * L.cout), 256, 0, n->stream>>>(dcur, n->act[l + 1],
                                                                               (long long)rows * L.cout);
    const __nv_bfloat16* W = n->p16 + L.w_off;
    float* dnext = bufs[flip];
    if (L.conv) {
      const long long e = (long long)rows * L.kdim();
      k_im2col<<<blocks_for(e), 256, 0, n->stream>>>(n->act[l], B, L.lin, L.cin, L.lout, L.ksz, L.stride, L.pad,
                                                      n->cols);
      weight_grads(n, L, dcur, n->cols, rows);
      if (l > 0) {
        gemm<false, false>(n, rows, (int)L.kdim(), L.cout, (const float*)dcur, L.cout, W, (int)L.kdim(), n->dcols,
                           (int)L.kdim(), nullptr, false);
        k_col2im<<<blocks_for((long long)B * L.lin * L.cin), 256, 0, n->stream>>>(n->dcols, B, L.lin, L.cin, L.lout,
                                                                                   L.ksz, L.stride, L.pad, dnext);
      }
    } else {
      weight_grads(n, L, dcur, n->act[l], rows);
      if (l > 0)
        gemm<false, false>(n, B, L.cin, L.cout, (const float*)dcur, L.cout, W, L.cin, dnext, L.cin, nullptr, false);
    }
    dcur = dnext;
    flip ^= 1;
  }
}

int check_batch(const fdtd_es_net* n, int B) {
  if (B < 1 || B > n->cfg.max_batch)
    return es_fail(FDTD_ERR_BADARG, "batch %d outside 1..%d (max_batch)", B, n->cfg.max_batch);
  return FDTD_OK;
}

long long in_width(const fdtd_es_net* n) { return (long long)n->cfg.in_length * n->cfg.in_channels; }

// Loss of the batch in act[0] against n->target (both on the device).
int loss_and_grad(fdtd_es_net* n, int B, float* loss_host, bool want_grad) {
  forward(n, B);
  const int D = n->cfg.out_dim;
  k_loss<<<(B + 127) / 128, 128, 0, n->stream>>>(n->act.back(), n->target, n->wout, B, D, n->dy, n->per);
  k_mean<<<1, 256, 0, n->stream>>>(n->per, B, n->loss);
  if (want_grad) backward(n, B);
  ES_CK(cudaGetLastError());
  if (loss_host) {
    ES_CK(cudaMemcpyAsync(loss_host, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    ES_CK(cudaStreamSynchronize(n->stream));
  }
  return FDTD_OK;
}

// xorshift64* stream for initialisation and shuffling.
struct Rng {
  unsigned long long s;
  explicit Rng(unsigned long long seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x2545F4914F6CDD1Dull) {
    if (!s) s = 1;
  }
  unsigned long long next() {
    s ^= s >> 12;
    s ^= s << 25;
    s ^= s >> 27;
    return s * 0x2545F4914F6CDD1Dull;
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

int upload_params(fdtd_es_net* n, const float* host) {
  ES_CK(cudaMemcpyAsync(n->p32, host, n->nparam * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  k_to_bf16<<<blocks_for(n->nparam), 256, 0, n->stream>>>(n->p32, n->p16, n->nparam);
  ES_CK(cudaGetLastError());
  ES_CK(cudaStreamSynchronize(n->stream));
  return FDTD_OK;
}

int reset_optimizer(fdtd_es_net* n) {
  n->adam_t = 0;
  ES_CK(cudaMemsetAsync(n->m, 0, n->nparam * sizeof(float), n->stream));
  ES_CK(cudaMemsetAsync(n->v, 0, n->nparam * sizeof(float), n->stream));
  return FDTD_OK;
}

int trace_inputs(fdtd_es_net* n, fdtd_ctx* const* members, int count, int decim, float* scales) {
  if (!members || decim < 1) return es_fail(FDTD_ERR_BADARG, "bad member arguments");
  int rc = check_batch(n, count);
  if (rc) return rc;
  if (n->cfg.in_channels != 2) return es_fail(FDTD_ERR_STATE, "member inputs need in_channels == 2");
  const long long need = (long long)n->cfg.in_length * decim;
  std::vector<const double*> ptr(2 * count);
  for (int b = 0; b < count; b++) {
    if (!members[b]) return es_fail(FDTD_ERR_BADARG, "member %d is NULL", b);
    const double *V, *I;
    int nsteps, steps, dev;
    rc = fdtd_internal_traces(members[b], &V, &I, &nsteps, &steps, &dev);
    if (rc) return rc;
    if (dev != n->cfg.device)
      return es_fail(FDTD_ERR_BADARG, "member %d is on device %d, the network on %d", b, dev, n->cfg.device);
    if (steps < need) return es_fail(FDTD_ERR_STATE, "member %d has run %d steps, the input needs %lld", b, steps, need);
    ptr[b] = V;          // voltage probe 0
    ptr[count + b] = I;  // current probe 0
  }
  ES_CK(cudaMemcpyAsync(n->d_traces, ptr.data(), ptr.size() * sizeof(double*), cudaMemcpyHostToDevice, n->stream));
  k_trace_inputs<<<count, 256, 0, n->stream>>>(n->d_traces, n->d_traces + count, n->cfg.in_length, decim, n->act[0],
                                               n->scales);
  ES_CK(cudaGetLastError());
  if (scales)
    ES_CK(cudaMemcpyAsync(scales, n->scales, 2 * count * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
  ES_CK(cudaStreamSynchronize(n->stream));
  return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_es_create(const FdtdEsConfig* cfg, fdtd_es_net** out) {
  if (!cfg || !out) return es_fail(FDTD_ERR_BADARG, "NULL argument");
  *out = nullptr;
  const FdtdEsConfig& c = *cfg;
  if (c.in_channels < 1 || c.in_length < 1 || c.conv_layers < 0 || c.channels < 1 || c.kernel < 1 ||
      c.kernel % 2 == 0 || c.stride < 1 || c.mlp_layers < 0 || c.mlp_width < 1 || c.out_dim < 1 ||
      c.max_batch < 1 || c.max_batch > 65535)
    return es_fail(FDTD_ERR_BADARG, "invalid network configuration");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || c.device < 0 || c.device >= ndev)
    return es_fail(FDTD_ERR_CUDA, "CUDA device %d not available", c.device);
  fdtd_es_net* n = new fdtd_es_net();
  n->cfg = c;
  long long off = 0;
  int len = c.in_length, ch = c.in_channels;
  for (int l = 0; l < c.conv_layers; l++) {
    Layer L{};
    L.conv = true;
    L.cin = ch;
    L.cout = c.channels;
    L.lin = len;
    L.ksz = c.kernel;
    L.stride = c.stride;
    L.pad = c.kernel / 2;
    L.lout = (len + 2 * L.pad - L.ksz) / L.stride + 1;
    L.relu = true;
    L.w_off = off;
    off += (long long)L.cout * L.ksz * L.cin;
    L.b_off = off;
    off += L.cout;
    n->layers.push_back(L);
    len = L.lout;
    ch = L.cout;
  }
  int feat = len * ch;
  for (int l = 0; l <= c.mlp_layers; l++) {
    Layer L{};
    L.conv = false;
    L.cin = feat;
    L.cout = l < c.mlp_layers ? c.mlp_width : c.out_dim;
    L.lin = L.lout = 1;
    L.ksz = L.stride = 1;
    L.relu = l < c.mlp_layers;
    L.w_off = off;
    off += (long long)L.cout * L.cin;
    L.b_off = off;
    off += L.cout;
    n->layers.push_back(L);
    feat = L.cout;
  }
  n->nparam = off;
  if (cudaSetDevice(c.device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete n;
    return es_fail(FDTD_ERR_CUDA, "cannot create a stream on device %d", c.device);
  }
  const long long B = c.max_batch;
  long long max_act = in_width(n), max_cols = 1, max_ws = 1;
  n->act.assign(n->layers.size() + 1, nullptr);
  for (const Layer& L : n->layers) {
    max_act = std::max(max_act, std::max(L.in_width(), L.out_width()));
    const long long rows = L.conv ? B * L.lout : B;
    if (L.conv) max_cols = std::max(max_cols, rows * L.kdim());
    const long long slices = grad_slices(rows);
    if (slices > 1) max_ws = std::max(max_ws, slices * L.cout * L.kdim());
  }
  int rc = es_alloc(n, (void**)&n->p32, n->nparam * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->p16, n->nparam * sizeof(__nv_bfloat16));
  if (!rc) rc = es_alloc(n, (void**)&n->grad, n->nparam * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->m, n->nparam * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->v, n->nparam * sizeof(float));
  for (size_t l = 0; l <= n->layers.size() && !rc; l++) {
    const long long w = l == 0 ? in_width(n) : n->layers[l - 1].out_width();
    rc = es_alloc(n, (void**)&n->act[l], B * w * sizeof(float));
  }
  if (!rc) rc = es_alloc(n, (void**)&n->cols, max_cols * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->dcols, max_cols * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->da, B * max_act * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->db, B * max_act * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->ws, max_ws * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->target, B * c.out_dim * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->wout, c.out_dim * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->dy, B * c.out_dim * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->per, B * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->loss, sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->scales, 2 * B * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->d_traces, 2 * B * sizeof(double*));
  if (rc) {
    fdtd_es_free(n);
    return rc;
  }
  *out = n;
  return FDTD_OK;
}

void fdtd_es_free(fdtd_es_net* n) {
  if (!n) return;
  cudaSetDevice(n->cfg.device);
  if (n->stream) cudaStreamSynchronize(n->stream);
  for (void* p : n->owned) cudaFree(p);
  if (n->stream) cudaStreamDestroy(n->stream);
  delete n;
}

int fdtd_es_param_count(const fdtd_es_net* n, long* count) {
  if (!n || !count) return es_fail(FDTD_ERR_BADARG, "NULL argument");
  *count = (long)n->nparam;
  return FDTD_OK;
}

int fdtd_es_init_params(fdtd_es_net* n, unsigned long long seed) {
  if (!n) return es_fail(FDTD_ERR_BADARG, "NULL network");
  std::vector<float> h(n->nparam);
  Rng r(seed);
  for (const Layer& L : n->layers) {
    const double bound = 1.0 / std::sqrt((double)L.kdim());
    for (long long q = L.w_off; q < L.b_off + L.cout; q++) h[q] = (float)((2.0 * r.uniform() - 1.0) * bound);
  }
  ES_CK(cudaSetDevice(n->cfg.device));
  int rc = reset_optimizer(n);
  return rc ? rc : upload_params(n, h.data());
}

int fdtd_es_set_params(fdtd_es_net* n, const float* params, long count) {
  if (!n || !params) return es_fail(FDTD_ERR_BADARG, "NULL argument");
  if (count != n->nparam)
    return es_fail(FDTD_ERR_BADARG, "%ld parameters given, the network has %lld", count, n->nparam);
  ES_CK(cudaSetDevice(n->cfg.device));
  int rc = reset_optimizer(n);
  return rc ? rc : upload_params(n, params);
}

int fdtd_es_get_params(fdtd_es_net* n, float* params, long count) {
  if (!n || !params) return es_fail(FDTD_ERR_BADARG, "NULL argument");
  if (count != n->nparam)
    return es_fail(FDTD_ERR_BADARG, "%ld parameters asked, the network has %lld", count, n->nparam);
  ES_CK(cudaSetDevice(n->cfg.device));
  ES_CK(cudaMemcpyAsync(params, n->p32, n->nparam * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
  ES_CK(cudaStreamSynchronize(n->stream));
  return FDTD_OK;
}

int fdtd_es_forward(fdtd_es_net* n, const float* x, int batch, float* y) {
  if (!n || !x || !y) return es_fail(FDTD_ERR_BADARG, "NULL argument");
  int rc = check_batch(n, batch);
  if (rc) return rc;
  ES_CK(cudaSetDevice(n->cfg.device));
  ES_CK(cudaMemcpyAsync(n->act[0], x, batch * in_width(n) * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  forward(n, batch);
  ES_CK(cudaGetLastError());
  ES_CK(cudaMemcpyAsync(y, n->act.back(), (size_t)batch * n->cfg.out_dim * sizeof(float), cudaMemcpyDeviceToHost,
                        n->stream));
  ES_CK(cudaStreamSynchronize(n->stream));
  return FDTD_OK;
}

int fdtd_es_loss_grad(fdtd_es_net* n, const float* x, const float* target, const float* w, int batch, float* loss,
                      float* grad, long count) {
  if (!n || !x || !target || !w || !loss) return es_fail(FDTD_ERR_BADARG, "NULL argument");
  int rc = check_batch(n, batch);
  if (rc) return rc;
  if (grad && count != n->nparam)
    return es_fail(FDTD_ERR_BADARG, "gradient buffer of %ld, the network has %lld", count, n->nparam);
  ES_CK(cudaSetDevice(n->cfg.device));
  const int D = n->cfg.out_dim;
  ES_CK(cudaMemcpyAsync(n->act[0], x, batch * in_width(n) * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  ES_CK(cudaMemcpyAsync(n->target, target, (size_t)batch * D * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  ES_CK(cudaMemcpyAsync(n->wout, w, D * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  rc = loss_and_grad(n, batch, loss, grad != nullptr);
  if (rc) return rc;
  if (grad) {
    ES_CK(cudaMemcpyAsync(grad, n->grad, n->nparam * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    ES_CK(cudaStreamSynchronize(n->stream));
  }
  return FDTD_OK;
}

int fdtd_es_set_data(fdtd_es_net* n, const float* x, const float* target, long count) {
  if (!n || !x || !target || count < 1) return es_fail(FDTD_ERR_BADARG, "bad training set");
  ES_CK(cudaSetDevice(n->cfg.device));
  es_release(n, n->dset_x);
  es_release(n, n->dset_y);
  es_release(n, n->d_perm);
  n->dset_x = n->dset_y = nullptr;
  n->d_perm = nullptr;
  n->nsamples = 0;
  int rc = es_alloc(n, (void**)&n->dset_x, count * in_width(n) * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->dset_y, (size_t)count * n->cfg.out_dim * sizeof(float));
  if (!rc) rc = es_alloc(n, (void**)&n->d_perm, count * sizeof(int));
  if (rc) return rc;
  ES_CK(cudaMemcpyAsync(n->dset_x, x, count * in_width(n) * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  ES_CK(cudaMemcpyAsync(n->dset_y, target, (size_t)count * n->cfg.out_dim * sizeof(float), cudaMemcpyHostToDevice,
                        n->stream));
  ES_CK(cudaStreamSynchronize(n->stream));
  n->nsamples = count;
  return FDTD_OK;
}

int fdtd_es_train(fdtd_es_net* n, int epochs, int batch, const float* w, float lr, float beta1, float beta2,
                  float eps, float weight_decay, unsigned long long seed, float* epoch_loss) {
  if (!n || !w || epochs < 0) return es_fail(FDTD_ERR_BADARG, "bad training arguments");
  int rc = check_batch(n, batch);
  if (rc) return rc;
  if (!n->dset_x) return es_fail(FDTD_ERR_STATE, "no training set (fdtd_es_set_data)");
  if (batch > n->nsamples) return es_fail(FDTD_ERR_BADARG, "batch %d larger than the training set", batch);
  ES_CK(cudaSetDevice(n->cfg.device));
  const int D = n->cfg.out_dim;
  ES_CK(cudaMemcpyAsync(n->wout, w, D * sizeof(float), cudaMemcpyHostToDevice, n->stream));
  const long long steps = n->nsamples / batch;
  std::vector<int> perm(n->nsamples);
  std::vector<float> losses(steps);
  Rng r(seed);
  float* d_losses = nullptr;
  rc = es_alloc(n, (void**)&d_losses, steps * sizeof(float));
  if (rc) return rc;
  for (int ep = 0; ep < epochs && !rc; ep++) {
    for (long long q = 0; q < n->nsamples; q++) perm[q] = (int)q;
    for (long long q = n->nsamples - 1; q > 0; q--) std::swap(perm[q], perm[r.next() % (q + 1)]);
    // the previous epoch ended with a stream wait, so no copy still reads perm
    ES_CK(cudaMemcpyAsync(n->d_perm, perm.data(), n->nsamples * sizeof(int), cudaMemcpyHostToDevice, n->stream));
    for (long long s = 0; s < steps && !rc; s++) {
      const dim3 g((unsigned)std::min<long long>(64, (in_width(n) + 255) / 256), batch);
      k_gather<<<g, 256, 0, n->stream>>>(n->dset_x, n->dset_y, n->d_perm + s * batch, batch, (int)in_width(n), D,
                                          n->act[0], n->target);
      rc = loss_and_grad(n, batch, nullptr, true);
      if (rc) break;
      ES_CK(cudaMemcpyAsync(d_losses + s, n->loss, sizeof(float), cudaMemcpyDeviceToDevice, n->stream));
      n->adam_t++;
      const double c1 = 1.0 / (1.0 - std::pow((double)beta1, (double)n->adam_t));
      const double c2 = 1.0 / (1.0 - std::pow((double)beta2, (double)n->adam_t));
      k_adam<<<blocks_for(n->nparam), 256, 0, n->stream>>>(n->p32, n->p16, n->grad, n->m, n->v, n->nparam, lr, beta1,
                                                           beta2, eps, weight_decay, (float)c1, (float)c2);
      ES_CK(cudaGetLastError());
    }
    if (rc) break;
    ES_CK(cudaMemcpyAsync(losses.data(), d_losses, steps * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    ES_CK(cudaStreamSynchronize(n->stream));
    if (epoch_loss) {
      double s = 0;
      for (float v : losses) s += v;
      epoch_loss[ep] = (float)(s / std::max<long long>(1, steps));
    }
  }
  cudaStreamSynchronize(n->stream);
  es_release(n, d_losses);
  return rc;
}

int fdtd_es_member_inputs(fdtd_es_net* n, fdtd_ctx* const* members, int count, int decim, float* scales,
                          float* x) {
  if (!n) return es_fail(FDTD_ERR_BADARG, "NULL network");
  ES_CK(cudaSetDevice(n->cfg.device));
  int rc = trace_inputs(n, members, count, decim, scales);
  if (rc) return rc;
  if (x) {
    ES_CK(cudaMemcpyAsync(x, n->act[0], count * in_width(n) * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    ES_CK(cudaStreamSynchronize(n->stream));
  }
  return FDTD_OK;
}

int fdtd_es_predict_members(fdtd_es_net* n, fdtd_ctx* const* members, int count, int decim, float* scales,
                            float* y) {
  if (!n || !y) return es_fail(FDTD_ERR_BADARG, "NULL argument");
  ES_CK(cudaSetDevice(n->cfg.device));
  int rc = trace_inputs(n, members, count, decim, scales);
  if (rc) return rc;
  forward(n, count);
  ES_CK(cudaGetLastError());
  ES_CK(cudaMemcpyAsync(y, n->act.back(), (size_t)count * n->cfg.out_dim * sizeof(float), cudaMemcpyDeviceToHost,
                        n->stream));
  ES_CK(cudaStreamSynchronize(n->stream));
  return FDTD_OK;
}

}  // extern "C"
