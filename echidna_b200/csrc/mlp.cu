// The learned importance proposal for sparse STDE: a small MLP
//   x (n_in) -> ReLU(W1 x + b1) (h) -> ReLU(W2 . + b2) (h) -> W3 . + b3 (n_out) -> softmax
// trained on the GPU with BF16 operands and FP32 accumulation.  Every GEMM is
// umma::gemm_bf16_tn (tcgen05.mma, accumulator in TMEM); the rest are small
// elementwise / reduction kernels.  Master weights and Adam moments are FP32;
// the GEMMs read BF16 copies refreshed after every update.
//
// Training target: per point a probability vector q over the n_out
// coordinates (for sparse STDE, q_j = |H_jj| / sum_k |H_kk| from exact tape
// jets); loss = mean over points of -sum_j q_j log p_j.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "abi_internal.h"
#include "umma_gemm.cuh"

namespace {

using bf16 = __nv_bfloat16;
using ech::set_error;

__global__ void to_bf16_kernel(const float* in, bf16* out, size_t n, int relu) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float v = in[i];
  if (relu) v = fmaxf(v, 0.0f);
  out[i] = __float2bfloat16_rn(v);
}

// out[c][r] = in[r][c]
__global__ void transpose_bf16_kernel(const bf16* in, bf16* out, int R, int C) {
  __shared__ bf16 tile[32][33];
  const int c = blockIdx.x * 32 + threadIdx.x;
  for (int k = 0; k < 32; k += 8) {
    const int r = blockIdx.y * 32 + threadIdx.y + k;
    if (r < R && c < C) tile[threadIdx.y + k][threadIdx.x] = in[(size_t)r * C + c];
  }
  __syncthreads();
  const int r2 = blockIdx.y * 32 + threadIdx.x;
  for (int k = 0; k < 32; k += 8) {
    const int c2 = blockIdx.x * 32 + threadIdx.y + k;
    if (c2 < C && r2 < R) out[(size_t)c2 * R + r2] = tile[threadIdx.x][threadIdx.y + k];
  }
}

// One block per row: p = softmax(logits); with a target q, dlogits = (p - q) / rows
// (fp32 and bf16) and the row's cross-entropy -sum q log p added to *loss / rows.
__global__ void softmax_xent_kernel(const float* logits, const float* q, float* p, float* dl, bf16* dlb, int cols,
                                    int rows, float* loss) {
  const int r = blockIdx.x;
  const float* z = logits + (size_t)r * cols;
  __shared__ float red[32];
  float m = -INFINITY;
  for (int c = threadIdx.x; c < cols; c += blockDim.x) m = fmaxf(m, z[c]);
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : -INFINITY;
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  m = red[0];
  __syncthreads();
  float s = 0.0f;
  for (int c = threadIdx.x; c < cols; c += blockDim.x) s += expf(z[c] - m);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  const float lse = m + logf(red[0]);
  __syncthreads();
  float l = 0.0f;
  for (int c = threadIdx.x; c < cols; c += blockDim.x) {
    const float logp = z[c] - lse;
    const float pc = expf(logp);
    p[(size_t)r * cols + c] = pc;
    if (q) {
      const float qc = q[(size_t)r * cols + c];
      const float g = (pc - qc) / (float)rows;
      dl[(size_t)r * cols + c] = g;
      dlb[(size_t)r * cols + c] = __float2bfloat16_rn(g);
      if (qc > 0.0f) l -= qc * logp;
    }
  }
  if (q) {
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l / (float)rows);
  }
}

// dz = dh * (z > 0), fp32 and bf16
__global__ void relu_back_kernel(const float* dh, const float* z, float* dz, bf16* dzb, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = z[i] > 0.0f ? dh[i] : 0.0f;
  dz[i] = g;
  dzb[i] = __float2bfloat16_rn(g);
}

// db[c] = sum_r d[r][c]
__global__ void colsum_kernel(const float* d, float* db, int rows, int cols) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; ++r) s += d[(size_t)r * cols + c];
  db[c] = s;
}

// Adam (Kingma & Ba, 2015) on fp32 master weights; refreshes the bf16 copy.
__global__ void adam_kernel(float* w, const float* g, float* m, float* v, bf16* wb, size_t n, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
}

unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 2-D map of a row-major bf16 matrix [rows][K] (row stride ld elements): boxes of
// 64 K-elements (128 B) x box_rows rows with the 128-byte swizzle, zero fill past
// the edges.
cudaError_t make_operand_map(CUtensorMap* map, const bf16* base, int rows, int K, int ld, int box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return cudaErrorNotSupported;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(bf16)};
  const cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int BN>
cudaError_t gemm_tiles(const bf16* A, const bf16* B, float* C, const float* bias, int M, int N, int K, int lda,
                       int ldb, int ldc, uint32_t* err, cudaStream_t st) {
  using TL = ech::umma::Tile<BN>;
  CUtensorMap ta, tb;
  cudaError_t e = make_operand_map(&ta, A, M, K, lda, ech::umma::kBM);
  if (e == cudaSuccess) e = make_operand_map(&tb, B, N, K, ldb, BN);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ech::umma::gemm_bf16_tn<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TL::kSmemBytes);
  if (e != cudaSuccess) return e;
  dim3 grid((N + BN - 1) / BN, (M + ech::umma::kBM - 1) / ech::umma::kBM);
  ech::umma::gemm_bf16_tn<BN><<<grid, ech::umma::kThreads, TL::kSmemBytes, st>>>(ta, tb, C, bias, M, N, K, ldc, err);
  return cudaGetLastError();
}

// 128 x 256 tiles when they still give each of the 148 SMs one; else 128 x 128,
// or 128 x 64 when the 128-wide grid would cover less than half of the SMs.
cudaError_t gemm(const bf16* A, const bf16* B, float* C, const float* bias, int M, int N, int K, int lda, int ldb,
                 int ldc, uint32_t* err, cudaStream_t st) {
  const long rows = (M + 127) / 128;
  if (rows * ((N + 255) / 256) >= 148) return gemm_tiles<256>(A, B, C, bias, M, N, K, lda, ldb, ldc, err, st);
  if (rows * ((N + 127) / 128) < 74) return gemm_tiles<64>(A, B, C, bias, M, N, K, lda, ldb, ldc, err, st);
  return gemm_tiles<128>(A, B, C, bias, M, N, K, lda, ldb, ldc, err, st);
}

cudaError_t transpose(const bf16* in, bf16* out, int R, int C, cudaStream_t st) {
  dim3 grid((C + 31) / 32, (R + 31) / 32), block(32, 8);
  transpose_bf16_kernel<<<grid, block, 0, st>>>(in, out, R, C);
  return cudaGetLastError();
}

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  ~DBuf() { if (p) cudaFree(p); }
  cudaError_t ensure(size_t m) {
    if (m <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, m * sizeof(T));
    if (e == cudaSuccess) n = m;
    return e;
  }
};

}  // namespace

struct ech_mlp {
  ech_ctx* ctx = nullptr;
  int device = 0;
  int nin = 0, h = 0, nout = 0;
  int step = 0;
  std::mutex mu;
  // parameters: fp32 master, bf16 copy, Adam moments, gradient
  DBuf<float> w1, b1, w2, b2, w3, b3, g_w1, g_b1, g_w2, g_b2, g_w3, g_b3;
  DBuf<float> m_w1, m_b1, m_w2, m_b2, m_w3, m_b3, v_w1, v_b1, v_w2, v_b2, v_w3, v_b3;
  DBuf<bf16> w1b, w2b, w3b, w2bT, w3bT;
  // activations (sized for the largest batch seen)
  DBuf<bf16> xb, xbT, h1b, h1bT, h2b, h2bT, dlb, dlbT, dz2b, dz2bT, dz1b, dz1bT;
  DBuf<float> z1, z2, logits, probs, dl, dh2, dz2, dh1, dz1, loss;
  DBuf<uint32_t> err;
};

namespace {

ech_status cu(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return ECH_OK;
  if (e == cudaErrorMemoryAllocation) return set_error(ECH_ERR_OUT_OF_MEMORY, "GPU out of memory");
  return set_error(ECH_ERR_OTHER, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CUE(call)                                        \
  do {                                                   \
    ech_status s_ = cu((call), #call);                   \
    if (s_ != ECH_OK) return s_;                         \
  } while (0)

ech_status ensure_batch(ech_mlp* m, int B) {
  const size_t b = (size_t)B;
  CUE(m->xb.ensure(b * m->nin));
  CUE(m->xbT.ensure(b * m->nin));
  CUE(m->h1b.ensure(b * m->h));
  CUE(m->h1bT.ensure(b * m->h));
  CUE(m->h2b.ensure(b * m->h));
  CUE(m->h2bT.ensure(b * m->h));
  CUE(m->dlb.ensure(b * m->nout));
  CUE(m->dlbT.ensure(b * m->nout));
  CUE(m->dz2b.ensure(b * m->h));
  CUE(m->dz2bT.ensure(b * m->h));
  CUE(m->dz1b.ensure(b * m->h));
  CUE(m->dz1bT.ensure(b * m->h));
  CUE(m->z1.ensure(b * m->h));
  CUE(m->z2.ensure(b * m->h));
  CUE(m->logits.ensure(b * m->nout));
  CUE(m->probs.ensure(b * m->nout));
  CUE(m->dl.ensure(b * m->nout));
  CUE(m->dh2.ensure(b * m->h));
  CUE(m->dz2.ensure(b * m->h));
  CUE(m->dh1.ensure(b * m->h));
  CUE(m->dz1.ensure(b * m->h));
  return ECH_OK;
}

// forward through the logits and the softmax (and, with q, the loss gradient)
ech_status forward(ech_mlp* m, const float* x, int B, const float* q, cudaStream_t st) {
  const int nin = m->nin, h = m->h, nout = m->nout;
  uint32_t* err = m->err.p;
  const unsigned T = 256;
  to_bf16_kernel<<<blocks_for((size_t)B * nin, T), T, 0, st>>>(x, m->xb.p, (size_t)B * nin, 0);
  CUE(gemm(m->xb.p, m->w1b.p, m->z1.p, m->b1.p, B, h, nin, nin, nin, h, err, st));
  to_bf16_kernel<<<blocks_for((size_t)B * h, T), T, 0, st>>>(m->z1.p, m->h1b.p, (size_t)B * h, 1);
  CUE(gemm(m->h1b.p, m->w2b.p, m->z2.p, m->b2.p, B, h, h, h, h, h, err, st));
  to_bf16_kernel<<<blocks_for((size_t)B * h, T), T, 0, st>>>(m->z2.p, m->h2b.p, (size_t)B * h, 1);
  CUE(gemm(m->h2b.p, m->w3b.p, m->logits.p, m->b3.p, B, nout, h, h, h, nout, err, st));
  softmax_xent_kernel<<<B, 256, 0, st>>>(m->logits.p, q, m->probs.p, m->dl.p, m->dlb.p, nout, B, m->loss.p);
  return cu(cudaGetLastError(), "softmax");
}

ech_status adam_all(ech_mlp* m, float lr, cudaStream_t st) {
  m->step += 1;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.0f - powf(b1, (float)m->step), c2 = 1.0f - powf(b2, (float)m->step);
  const unsigned T = 256;
  struct P {
    float *w, *g, *mm, *vv;
    bf16* wb;
    size_t n;
  } ps[6] = {{m->w1.p, m->g_w1.p, m->m_w1.p, m->v_w1.p, m->w1b.p, (size_t)m->h * m->nin},
             {m->b1.p, m->g_b1.p, m->m_b1.p, m->v_b1.p, nullptr, (size_t)m->h},
             {m->w2.p, m->g_w2.p, m->m_w2.p, m->v_w2.p, m->w2b.p, (size_t)m->h * m->h},
             {m->b2.p, m->g_b2.p, m->m_b2.p, m->v_b2.p, nullptr, (size_t)m->h},
             {m->w3.p, m->g_w3.p, m->m_w3.p, m->v_w3.p, m->w3b.p, (size_t)m->nout * m->h},
             {m->b3.p, m->g_b3.p, m->m_b3.p, m->v_b3.p, nullptr, (size_t)m->nout}};
  for (const P& p : ps)
    adam_kernel<<<blocks_for(p.n, T), T, 0, st>>>(p.w, p.g, p.mm, p.vv, p.wb, p.n, lr, b1, b2, eps, c1, c2);
  CUE(cudaGetLastError());
  CUE(transpose(m->w2b.p, m->w2bT.p, m->h, m->h, st));
  CUE(transpose(m->w3b.p, m->w3bT.p, m->nout, m->h, st));
  return ECH_OK;
}

}  // namespace

extern "C" {

ECH_API ech_status ech_gemm_bf16(ech_ctx* ctx, const void* A, const void* B, float* C, const float* bias, int M,
                                 int N, int K, int lda, int ldb, int ldc, void* stream) {
  if (!ctx || !A || !B || !C) return set_error(ECH_ERR_INVALID_ARG, "null argument");
  if (M <= 0 || N <= 0 || K <= 0 || K % 64 != 0)
    return set_error(ECH_ERR_INVALID_ARG, "M, N > 0 and K a positive multiple of 64 required");
  if (lda % 8 || ldb % 8 || lda < K || ldb < K || ldc < N)
    return set_error(ECH_ERR_INVALID_ARG, "lda, ldb must be multiples of 8 and >= K; ldc >= N");
  if (((uintptr_t)A | (uintptr_t)B) & 15) return set_error(ECH_ERR_INVALID_ARG, "A and B must be 16-byte aligned");
  uint32_t* err = nullptr;
  int device = 0;
  cudaStream_t st = nullptr;
  ech_status s = ech::ctx_basics(ctx, &device, &st, &err);
  if (s != ECH_OK) return s;
  CUE(cudaSetDevice(device));
  return cu(gemm((const bf16*)A, (const bf16*)B, C, bias, M, N, K, lda, ldb, ldc, err,
                 stream ? (cudaStream_t)stream : st),
            "gemm launch");
}

ECH_API ech_status ech_mlp_create(ech_ctx* ctx, int n_in, int hidden, int n_out, const float* w1, const float* b1,
                                  const float* w2, const float* b2, const float* w3, const float* b3,
                                  ech_mlp** out) {
  if (!ctx || !out || !w1 || !b1 || !w2 || !b2 || !w3 || !b3) return set_error(ECH_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (n_in % 64 || hidden % 64 || n_out % 64 || n_in <= 0 || hidden <= 0 || n_out <= 0)
    return set_error(ECH_ERR_INVALID_ARG, "layer sizes must be positive multiples of 64");
  std::unique_ptr<ech_mlp> m(new ech_mlp());
  int device = 0;
  cudaStream_t st = nullptr;
  uint32_t* err = nullptr;
  ech_status s = ech::ctx_basics(ctx, &device, &st, &err);
  if (s != ECH_OK) return s;
  m->ctx = ctx;
  m->device = device;
  m->nin = n_in;
  m->h = hidden;
  m->nout = n_out;
  CUE(cudaSetDevice(device));
  const size_t n1 = (size_t)hidden * n_in, n2 = (size_t)hidden * hidden, n3 = (size_t)n_out * hidden;
  struct S {
    DBuf<float>* d;
    const float* h;
    size_t n;
  } init[6] = {{&m->w1, w1, n1}, {&m->b1, b1, (size_t)hidden}, {&m->w2, w2, n2},
               {&m->b2, b2, (size_t)hidden}, {&m->w3, w3, n3}, {&m->b3, b3, (size_t)n_out}};
  for (const S& e : init) {
    CUE(e.d->ensure(e.n));
    CUE(cudaMemcpy(e.d->p, e.h, e.n * sizeof(float), cudaMemcpyHostToDevice));
  }
  DBuf<float>* zeros[] = {&m->g_w1, &m->g_b1, &m->g_w2, &m->g_b2, &m->g_w3, &m->g_b3, &m->m_w1, &m->m_b1, &m->m_w2,
                          &m->m_b2, &m->m_w3, &m->m_b3, &m->v_w1, &m->v_b1, &m->v_w2, &m->v_b2, &m->v_w3, &m->v_b3};
  const size_t sizes[] = {n1, (size_t)hidden, n2, (size_t)hidden, n3, (size_t)n_out};
  for (int k = 0; k < 18; ++k) {
    CUE(zeros[k]->ensure(sizes[k % 6]));
    CUE(cudaMemset(zeros[k]->p, 0, sizes[k % 6] * sizeof(float)));
  }
  CUE(m->w1b.ensure(n1));
  CUE(m->w2b.ensure(n2));
  CUE(m->w3b.ensure(n3));
  CUE(m->w2bT.ensure(n2));
  CUE(m->w3bT.ensure(n3));
  CUE(m->loss.ensure(1));
  CUE(m->err.ensure(1));
  CUE(cudaMemset(m->err.p, 0, sizeof(uint32_t)));
  const unsigned T = 256;
  to_bf16_kernel<<<blocks_for(n1, T), T>>>(m->w1.p, m->w1b.p, n1, 0);
  to_bf16_kernel<<<blocks_for(n2, T), T>>>(m->w2.p, m->w2b.p, n2, 0);
  to_bf16_kernel<<<blocks_for(n3, T), T>>>(m->w3.p, m->w3b.p, n3, 0);
  CUE(transpose(m->w2b.p, m->w2bT.p, hidden, hidden, nullptr));
  CUE(transpose(m->w3b.p, m->w3bT.p, n_out, hidden, nullptr));
  CUE(cudaDeviceSynchronize());
  *out = m.release();
  return ECH_OK;
}

}  // extern "C"

namespace {

// Forward with the loss and the backward pass of one batch: the parameter
// gradients of the mean cross-entropy land in g_w1 .. g_b3 (fp32).  The
// backward GEMMs read BF16 copies of the loss gradient and the activations,
// as the forward GEMMs read BF16 weights; every GEMM accumulates in FP32.
ech_status forward_backward(ech_mlp* m, const float* x, const float* q, int B, cudaStream_t st) {
  ech_status s = ensure_batch(m, B);
  if (s != ECH_OK) return s;
  const int nin = m->nin, h = m->h, nout = m->nout;
  uint32_t* err = m->err.p;
  const unsigned T = 256;
  CUE(cudaMemsetAsync(m->loss.p, 0, sizeof(float), st));
  s = forward(m, x, B, q, st);
  if (s != ECH_OK) return s;
  // layer 3
  CUE(transpose(m->dlb.p, m->dlbT.p, B, nout, st));
  CUE(transpose(m->h2b.p, m->h2bT.p, B, h, st));
  CUE(gemm(m->dlbT.p, m->h2bT.p, m->g_w3.p, nullptr, nout, h, B, B, B, h, err, st));
  colsum_kernel<<<blocks_for(nout, T), T, 0, st>>>(m->dl.p, m->g_b3.p, B, nout);
  CUE(gemm(m->dlb.p, m->w3bT.p, m->dh2.p, nullptr, B, h, nout, nout, nout, h, err, st));
  relu_back_kernel<<<blocks_for((size_t)B * h, T), T, 0, st>>>(m->dh2.p, m->z2.p, m->dz2.p, m->dz2b.p, (size_t)B * h);
  // layer 2
  CUE(transpose(m->dz2b.p, m->dz2bT.p, B, h, st));
  CUE(transpose(m->h1b.p, m->h1bT.p, B, h, st));
  CUE(gemm(m->dz2bT.p, m->h1bT.p, m->g_w2.p, nullptr, h, h, B, B, B, h, err, st));
  colsum_kernel<<<blocks_for(h, T), T, 0, st>>>(m->dz2.p, m->g_b2.p, B, h);
  CUE(gemm(m->dz2b.p, m->w2bT.p, m->dh1.p, nullptr, B, h, h, h, h, h, err, st));
  relu_back_kernel<<<blocks_for((size_t)B * h, T), T, 0, st>>>(m->dh1.p, m->z1.p, m->dz1.p, m->dz1b.p, (size_t)B * h);
  // layer 1
  CUE(transpose(m->dz1b.p, m->dz1bT.p, B, h, st));
  CUE(transpose(m->xb.p, m->xbT.p, B, nin, st));
  CUE(gemm(m->dz1bT.p, m->xbT.p, m->g_w1.p, nullptr, h, nin, B, B, B, nin, err, st));
  colsum_kernel<<<blocks_for(h, T), T, 0, st>>>(m->dz1.p, m->g_b1.p, B, h);
  return cu(cudaGetLastError(), "backward");
}

// The batch loss into *loss_out (host) and the GEMMs' error word.
ech_status finish_step(ech_mlp* m, float* loss_out) {
  float l = 0.0f;
  uint32_t e = 0;
  CUE(cudaMemcpy(&l, m->loss.p, sizeof l, cudaMemcpyDeviceToHost));
  CUE(cudaMemcpy(&e, m->err.p, sizeof e, cudaMemcpyDeviceToHost));
  if (e) return set_error(ECH_ERR_TIMEOUT, "device-side wait timed out in the MLP GEMM");
  if (loss_out) *loss_out = l;
  return ECH_OK;
}

}  // namespace

extern "C" {

// One Adam step on a batch: x [B][n_in] and q [B][n_out] fp32 device arrays;
// B a positive multiple of 64.  *loss_out (host) receives the batch loss.
ECH_API ech_status ech_mlp_train_step(ech_mlp* m, const float* x, const float* q, int B, float lr, float* loss_out) {
  if (!m || !x || !q) return set_error(ECH_ERR_INVALID_ARG, "null argument");
  if (B <= 0 || B % 64) return set_error(ECH_ERR_INVALID_ARG, "batch must be a positive multiple of 64");
  std::lock_guard<std::mutex> lk(m->mu);
  CUE(cudaSetDevice(m->device));
  cudaStream_t st = nullptr;
  ech_status s = forward_backward(m, x, q, B, st);
  if (s != ECH_OK) return s;
  s = adam_all(m, lr, st);
  if (s != ECH_OK) return s;
  return finish_step(m, loss_out);
}

// The gradients one training step would apply, without applying them: the
// same forward and backward kernels as ech_mlp_train_step, then copies of the
// fp32 parameter gradients (host arrays of the create-time sizes; NULL skips
// one) and the batch loss.  For checking the backward pass against a host
// computation.
ECH_API ech_status ech_mlp_gradients(ech_mlp* m, const float* x, const float* q, int B, float* g_w1, float* g_b1,
                                     float* g_w2, float* g_b2, float* g_w3, float* g_b3, float* loss_out) {
  if (!m || !x || !q) return set_error(ECH_ERR_INVALID_ARG, "null argument");
  if (B <= 0 || B % 64) return set_error(ECH_ERR_INVALID_ARG, "batch must be a positive multiple of 64");
  std::lock_guard<std::mutex> lk(m->mu);
  CUE(cudaSetDevice(m->device));
  cudaStream_t st = nullptr;
  ech_status s = forward_backward(m, x, q, B, st);
  if (s != ECH_OK) return s;
  s = finish_step(m, loss_out);
  if (s != ECH_OK) return s;
  struct S {
    float* h;
    const DBuf<float>* d;
  } o[6] = {{g_w1, &m->g_w1}, {g_b1, &m->g_b1}, {g_w2, &m->g_w2}, {g_b2, &m->g_b2}, {g_w3, &m->g_w3}, {g_b3, &m->g_b3}};
  for (const S& e : o)
    if (e.h) CUE(cudaMemcpy(e.h, e.d->p, e.d->n * sizeof(float), cudaMemcpyDeviceToHost));
  return ECH_OK;
}

// Softmax probabilities for x [B][n_in] into probs [B][n_out] (device arrays);
// B a positive multiple of 64 is not required here.
ECH_API ech_status ech_mlp_forward(ech_mlp* m, const float* x, int B, float* probs, void* stream) {
  if (!m || !x || !probs) return set_error(ECH_ERR_INVALID_ARG, "null argument");
  if (B <= 0) return set_error(ECH_ERR_INVALID_ARG, "batch must be positive");
  std::lock_guard<std::mutex> lk(m->mu);
  CUE(cudaSetDevice(m->device));
  cudaStream_t st = (cudaStream_t)stream;
  ech_status s = ensure_batch(m, B);
  if (s != ECH_OK) return s;
  s = forward(m, x, B, nullptr, st);
  if (s != ECH_OK) return s;
  CUE(cudaMemcpyAsync(probs, m->probs.p, (size_t)B * m->nout * sizeof(float), cudaMemcpyDeviceToDevice, st));
  return ECH_OK;
}

// Copies the fp32 master weights out (host arrays of the create-time sizes).
ECH_API ech_status ech_mlp_get_weights(ech_mlp* m, float* w1, float* b1, float* w2, float* b2, float* w3, float* b3) {
  if (!m) return set_error(ECH_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(m->mu);
  CUE(cudaSetDevice(m->device));
  CUE(cudaDeviceSynchronize());
  struct S {
    float* h;
    const DBuf<float>* d;
  } o[6] = {{w1, &m->w1}, {b1, &m->b1}, {w2, &m->w2}, {b2, &m->b2}, {w3, &m->w3}, {b3, &m->b3}};
  for (const S& e : o)
    if (e.h) CUE(cudaMemcpy(e.h, e.d->p, e.d->n * sizeof(float), cudaMemcpyDeviceToHost));
  return ECH_OK;
}

ECH_API void ech_mlp_destroy(ech_mlp* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  cudaDeviceSynchronize();
  delete m;
}

}  // extern "C"
