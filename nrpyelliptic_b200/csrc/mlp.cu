// Learned initial guess: a small MLP (puncture parameters -> POD coefficients
// of uu) trained and evaluated on the GPU with BF16 matrix products on the
// fifth-generation tensor cores (tcgen05.mma, FP32 accumulators in tensor
// memory), FP32 master weights and Adam; plus the POD reconstruction of the
// guess.
//
// Every matrix product of the network -- forward Z = H W, backward
// dH = dZ W^T and dW = H^T dZ -- is one kernel, k_gemm_tc: 128 x 32 output
// tiles, operands read with arbitrary strides (so the transposes are free),
// rounded to BF16 into shared memory in the tensor cores' layout and
// multiplied by tcgen05.mma issued from one thread, with the bias and tanh
// of the forward pass fused into the epilogue that reads the accumulator
// back with tcgen05.ld.
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "common.cuh"

namespace nrpyell {

namespace {

// ------------------------------------------------------------------ GEMM
// C[M x N] = alpha * A[M x K] B[K x N] (+ bias[N]) (then tanh), with
// A(m,k) = A[m*sam + k*sak] and B(k,n) = B[k*sbk + n*sbn]; FP32 in and out.
//
// One CTA of 128 threads computes a 128 x 32 tile of C on the fifth-
// generation tensor cores: the operands are rounded to BF16 and written to
// shared memory in the tensor cores' no-swizzle K-major layout (8 x 8
// core matrices of 128 contiguous bytes), one thread issues
// tcgen05.mma.cta_group::1.kind::f16 (M = 128, N = 32, K = 16) with the
// FP32 accumulator in tensor memory, tcgen05.commit signals an mbarrier when
// the products of a 64-deep K chunk are done (the next chunk may then
// overwrite shared memory), and each warp reads its 32 rows of the
// accumulator back with tcgen05.ld for the epilogue (alpha, bias, tanh).
constexpr int TC_M = 128, TC_N = 32, TC_KC = 64;      // CTA tile and K chunk
constexpr int TC_B_OFF = 32 * 1024;                   // B tile at 32 KB (the 16 KB A tile at 0)
constexpr int TC_SMEM = 64 * 1024;                    // dynamic shared memory per CTA
constexpr int TC_TMEM_COLS = 128;                     // tensor-memory columns allocated (N = 32 used)
constexpr int EPI_NONE = 0, EPI_BIAS = 1, EPI_BIAS_TANH = 2;
constexpr long long kTcWaitLimit = 1ll << 22;         // bounded mbarrier wait (iterations)

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat16 l = __float2bfloat16_rn(lo), h = __float2bfloat16_rn(hi);
  return (uint32_t)__bfloat16_as_ushort(l) | ((uint32_t)__bfloat16_as_ushort(h) << 16);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of a no-swizzle K-major operand: start
// address, leading-dimension byte offset (between core matrices adjacent in
// K), stride-dimension byte offset (between core matrices adjacent in M/N),
// descriptor version 1, layout type 0 (no swizzle).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A
// and B (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bit
// 17, M >> 4 at bit 24.
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

// Byte offset of element (r, k) (r: M or N row, k: K index, even) of a tile
// with R rows: core matrix (r/8, k/8) at ((k/8) * (R/8) + r/8) * 128, row r%8
// at 16 bytes, element k%8 at 2 bytes.
template <int R>
__device__ __forceinline__ uint32_t tile_off(int r, int k) {
  return (uint32_t)((((k >> 3) * (R / 8) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (long long it = 0; it < kTcWaitLimit; it++) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__global__ void __launch_bounds__(128) k_gemm_tc(int M, int N, int K, const float* __restrict__ A, long long sam,
                                                long long sak, const float* __restrict__ B, long long sbk,
                                                long long sbn, float* __restrict__ Cm, long long ldc,
                                                const float* __restrict__ bias, int epi, float alpha, int* err) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * TC_M, n0 = blockIdx.x * TC_N;
  unsigned char* As = tc_smem;
  unsigned char* Bs = tc_smem + TC_B_OFF;
  const uint32_t mb = smem_addr(&mbar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(&tmem_base)),
                 "n"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb) : "memory");
    failed = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_base;
  const int nchunks = (K + TC_KC - 1) / TC_KC;
  for (int c = 0; c < nchunks; c++) {
    const int k0 = c * TC_KC;
    // A chunk: 128 rows x 32 k-pairs; B chunk: TC_N rows (n) x 32 k-pairs.
    // Consecutive threads take consecutive k where the operand is contiguous
    // along k, else consecutive rows, so the global loads coalesce.
    const bool a_kfast = sak == 1, b_kfast = sbk == 1;
    for (int e = tid; e < TC_M * TC_KC / 2; e += 128) {
      const int r = a_kfast ? e / (TC_KC / 2) : e % TC_M;
      const int k = 2 * (a_kfast ? e % (TC_KC / 2) : e / TC_M);
      const int m = m0 + r, kk = k0 + k;
      float a0 = 0.f, a1 = 0.f;
      if (m < M) {
        if (kk < K) a0 = A[m * sam + kk * sak];
        if (kk + 1 < K) a1 = A[m * sam + (kk + 1) * sak];
      }
      *reinterpret_cast<uint32_t*>(As + tile_off<TC_M>(r, k)) = pack_bf16(a0, a1);
    }
    for (int e = tid; e < TC_N * TC_KC / 2; e += 128) {
      const int r = b_kfast ? e / (TC_KC / 2) : e % TC_N;
      const int k = 2 * (b_kfast ? e % (TC_KC / 2) : e / TC_N);
      const int n = n0 + r, kk = k0 + k;
      float b0 = 0.f, b1 = 0.f;
      if (n < N) {
        if (kk < K) b0 = B[kk * sbk + n * sbn];
        if (kk + 1 < K) b1 = B[(kk + 1) * sbk + n * sbn];
      }
      *reinterpret_cast<uint32_t*>(Bs + tile_off<TC_N>(r, k)) = pack_bf16(b0, b1);
    }
    // make the generic-proxy writes visible to the tensor cores
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
      for (int s = 0; s < TC_KC / 16; s++) {
        // K sub-block s: core-matrix columns 2s and 2s+1
        const uint64_t ad = smem_desc(smem_addr(As) + s * 2 * (TC_M / 8) * 128, (TC_M / 8) * 128, 128);
        const uint64_t bd = smem_desc(smem_addr(Bs) + s * 2 * (TC_N / 8) * 128, (TC_N / 8) * 128, 128);
        const uint32_t acc = (c > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mb)
                   : "memory");
    }
    // the chunk's products are done before shared memory is rewritten
    if (!mbar_wait(mb, (uint32_t)(c & 1))) failed = 1;
    __syncthreads();
    if (failed) break;
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (!failed) {
    // warp w reads accumulator rows 32w..32w+31 (tensor-memory lanes), TC_N columns
    const int m = m0 + 32 * warp + lane;
    const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll
    for (int half = 0; half < TC_N / 32; half++) {
      uint32_t v[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
          "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(taddr + 32 * half));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (m < M) {
#pragma unroll
        for (int j = 0; j < 32; j++) {
          const int n = n0 + 32 * half + j;
          if (n < N) {
            float x = alpha * __uint_as_float(v[j]);
            if (epi != EPI_NONE) x += bias[n];
            if (epi == EPI_BIAS_TANH) x = tanhf(x);
            Cm[m * ldc + n] = x;
          }
        }
      }
    }
  } else {
    // a wait gave up: record it, let the products in flight finish (again
    // bounded) before the tensor memory is released
    if (tid == 0) atomicExch(err, 1);
    mbar_wait(mb, (uint32_t)((nchunks - 1) & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "n"(TC_TMEM_COLS) : "memory");
  }
}

int* g_tc_err = nullptr;  // set by k_gemm_tc when a bounded wait gave up

void gemm(int M, int N, int K, const float* A, long long sam, long long sak, const float* B, long long sbk,
          long long sbn, float* C, long long ldc, const float* bias, int epi, float alpha = 1.f) {
  static unsigned long long opted = 0;
  int dev = 0;
  NRPYELL_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !(opted >> dev & 1ull)) {
    NRPYELL_CUDA(cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    opted |= 1ull << dev;
  }
  if (!g_tc_err) {
    NRPYELL_CUDA(dev_alloc(&g_tc_err, sizeof(int)));
    NRPYELL_CUDA(cudaMemset(g_tc_err, 0, sizeof(int)));
  }
  if (M <= 0 || N <= 0 || K <= 0) {
    NRPYELL_FAIL("k_gemm_tc: empty matrix product");
    return;
  }
  dim3 grid((N + TC_N - 1) / TC_N, (M + TC_M - 1) / TC_M);
  NRPYELL_LAUNCH(k_gemm_tc, grid, 128, TC_SMEM, M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, bias, epi, alpha, g_tc_err);
}

// Reports (once) a bounded wait of the tensor-core GEMM that gave up.
bool gemm_ok() {
  if (!g_tc_err) return true;
  int e = 0;
  NRPYELL_CUDA(cudaMemcpy(&e, g_tc_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    NRPYELL_CUDA(cudaMemset(g_tc_err, 0, sizeof(int)));
    NRPYELL_FAIL("k_gemm_tc: a bounded wait for the tensor-core products gave up");
    return false;
  }
  return status_ok();
}

// ------------------------------------------------------ elementwise pieces
// dZ = dH * (1 - H^2) (tanh layers), in place on dH.
__global__ void k_tanh_back(float* dh, const float* __restrict__ h, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dh[i] *= 1.f - h[i] * h[i];
}
// db[n] = sum over rows of dZ[:, n].
__global__ void k_colsum(const float* __restrict__ dz, int rows, int cols, float* db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; r++) s += dz[(long long)r * cols + n];
  db[n] = s;
}
// dY = 2 (Y - T) * scale; adds the block's sum of (Y - T)^2 to *loss.
__global__ void k_mse(const float* __restrict__ y, const float* __restrict__ tgt, long long n, float scale, float* dy,
                      double* loss) {
  __shared__ double sh[8];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (i < n) {
    const float d = y[i] - tgt[i];
    dy[i] = 2.f * d * scale;
    l = (double)d * d;
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
    atomicAdd(loss, s);
  }
}
// Adam on FP32 master parameters.
__global__ void k_adam(float* p, const float* __restrict__ gr, float* m, float* v, long long n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = gr[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}
// Rows of src selected by idx -> dst (minibatch gather).
__global__ void k_gather_rows(const float* __restrict__ src, const int* __restrict__ idx, int rows, int cols,
                              float* dst) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)rows * cols) return;
  const int r = (int)(i / cols), c = (int)(i % cols);
  dst[i] = src[(long long)idx[r] * cols + c];
}

unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

// ------------------------------------------------------------------- MLP

struct Mlp {
  int n_in, width, depth, n_out, batch_max;
  // layer l: dims[l] -> dims[l+1]; W_l [in x out] row-major, then b_l
  std::vector<int> dims;
  std::vector<long long> woff, boff;  // offsets into the parameter vector
  long long n_params = 0;
  float *p = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  std::vector<float*> h;  // output of layer l [batch_max x dims[l+1]]
  float* x = nullptr;     // minibatch inputs
  float* t = nullptr;     // minibatch targets
  float* dbuf[2] = {nullptr, nullptr};
  double* loss = nullptr;
  int* idx = nullptr;
  long long step = 0;
};

static Mlp* mlp_new(int n_in, int width, int depth, int n_out, int batch_max, unsigned seed) {
  Mlp* q = new Mlp();
  q->n_in = n_in;
  q->width = width;
  q->depth = depth;
  q->n_out = n_out;
  q->batch_max = batch_max;
  q->dims.push_back(n_in);
  for (int i = 0; i < depth; i++) q->dims.push_back(width);
  q->dims.push_back(n_out);
  const int L = (int)q->dims.size() - 1;
  for (int l = 0; l < L; l++) {
    q->woff.push_back(q->n_params);
    q->n_params += (long long)q->dims[l] * q->dims[l + 1];
    q->boff.push_back(q->n_params);
    q->n_params += q->dims[l + 1];
  }
  // Glorot-uniform weights from a fixed 64-bit LCG, zero biases
  std::vector<float> host(q->n_params, 0.f);
  unsigned long long s = 0x9E3779B97F4A7C15ull ^ seed;
  for (int l = 0; l < L; l++) {
    const float a = sqrtf(6.f / (q->dims[l] + q->dims[l + 1]));
    for (long long i = 0; i < (long long)q->dims[l] * q->dims[l + 1]; i++) {
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      const float u = (float)((s >> 11) * (1.0 / 9007199254740992.0));
      host[q->woff[l] + i] = a * (2.f * u - 1.f);
    }
  }
  const size_t pb = sizeof(float) * q->n_params;
  NRPYELL_CUDA(dev_alloc(&q->p, pb));
  NRPYELL_CUDA(dev_alloc(&q->grad, pb));
  NRPYELL_CUDA(dev_alloc(&q->m, pb));
  NRPYELL_CUDA(dev_alloc(&q->v, pb));
  NRPYELL_CUDA(cudaMemcpyAsync(q->p, host.data(), pb, cudaMemcpyHostToDevice, stream()));
  NRPYELL_CUDA(cudaMemsetAsync(q->m, 0, pb, stream()));
  NRPYELL_CUDA(cudaMemsetAsync(q->v, 0, pb, stream()));
  int wmax = n_out > width ? n_out : width;
  if (n_in > wmax) wmax = n_in;
  for (int l = 0; l < L; l++) {
    float* b = nullptr;
    NRPYELL_CUDA(dev_alloc(&b, sizeof(float) * (size_t)batch_max * q->dims[l + 1]));
    q->h.push_back(b);
  }
  NRPYELL_CUDA(dev_alloc(&q->x, sizeof(float) * (size_t)batch_max * n_in));
  NRPYELL_CUDA(dev_alloc(&q->t, sizeof(float) * (size_t)batch_max * n_out));
  NRPYELL_CUDA(dev_alloc(&q->dbuf[0], sizeof(float) * (size_t)batch_max * wmax));
  NRPYELL_CUDA(dev_alloc(&q->dbuf[1], sizeof(float) * (size_t)batch_max * wmax));
  NRPYELL_CUDA(dev_alloc(&q->loss, sizeof(double)));
  NRPYELL_CUDA(dev_alloc(&q->idx, sizeof(int) * batch_max));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  return q;
}

static void mlp_free(Mlp* q) {
  if (!q) return;
  cudaStreamSynchronize(stream());
  cudaFree(q->p);
  cudaFree(q->grad);
  cudaFree(q->m);
  cudaFree(q->v);
  for (float* b : q->h) cudaFree(b);
  cudaFree(q->x);
  cudaFree(q->t);
  cudaFree(q->dbuf[0]);
  cudaFree(q->dbuf[1]);
  cudaFree(q->loss);
  cudaFree(q->idx);
  delete q;
}

// Forward pass of `rows` inputs x [rows x n_in]; output in q->h.back().
static void mlp_forward(Mlp* q, const float* x, int rows) {
  const int L = (int)q->dims.size() - 1;
  const float* in = x;
  for (int l = 0; l < L; l++) {
    const int K = q->dims[l], N = q->dims[l + 1];
    gemm(rows, N, K, in, K, 1, q->p + q->woff[l], N, 1, q->h[l], N, q->p + q->boff[l],
         l + 1 < L ? EPI_BIAS_TANH : EPI_BIAS);
    in = q->h[l];
  }
}

// Gradient of the mean squared error against t [rows x n_out] into q->grad
// (after mlp_forward on the same x); adds the loss sum to *q->loss.
static void mlp_backward(Mlp* q, const float* x, const float* t, int rows) {
  const int L = (int)q->dims.size() - 1;
  const long long nout = (long long)rows * q->n_out;
  float* dz = q->dbuf[0];
  NRPYELL_LAUNCH(k_mse, blocks_for(nout, 256), 256, 0, q->h[L - 1], t, nout, 1.f / (float)nout, dz, q->loss);
  for (int l = L - 1; l >= 0; l--) {
    const int K = q->dims[l], N = q->dims[l + 1];
    const float* hin = (l == 0) ? x : q->h[l - 1];
    // dW = hin^T dZ [K x N]: A(kk, r) = hin[r*K + kk], B(r, n) = dz[r*N + n]
    gemm(K, N, rows, hin, 1, K, dz, N, 1, q->grad + q->woff[l], N, nullptr, EPI_NONE);
    NRPYELL_LAUNCH(k_colsum, blocks_for(N, 128), 128, 0, dz, rows, N, q->grad + q->boff[l]);
    if (l > 0) {
      // dH_{l-1} = dZ W^T [rows x K]: B(n, kk) = W[kk*N + n]
      float* dh = q->dbuf[(L - l) & 1];
      gemm(rows, K, N, dz, N, 1, q->p + q->woff[l], 1, N, dh, K, nullptr, EPI_NONE);
      NRPYELL_LAUNCH(k_tanh_back, blocks_for((long long)rows * K, 256), 256, 0, dh, q->h[l - 1], (long long)rows * K);
      dz = dh;
    }
  }
}

static void mlp_adam(Mlp* q, float lr) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  q->step++;
  const float c1 = 1.f - powf(b1, (float)q->step), c2 = 1.f - powf(b2, (float)q->step);
  NRPYELL_LAUNCH(k_adam, blocks_for(q->n_params, 256), 256, 0, q->p, q->grad, q->m, q->v, q->n_params, lr, b1, b2,
                 eps, c1, c2);
}

// ------------------------------------------------------------ POD guess
// y[0..Ntot) = mean + sum_k c[k] basis[k][.] (uu), y[Ntot..2 Ntot) = eta uu (vv).
__global__ void k_pod_guess(const float* __restrict__ mean, const float* __restrict__ basis, int K, long long ntot,
                            const float* __restrict__ c, double eta, double* y) {
  extern __shared__ float cs[];
  for (int k = threadIdx.x; k < K; k += blockDim.x) cs[k] = c[k];
  __syncthreads();
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntot) return;
  double u = (double)mean[i];
  for (int k = 0; k < K; k++) u += (double)cs[k] * (double)basis[(long long)k * ntot + i];
  y[i] = u;
  y[ntot + i] = eta * u;
}

}  // namespace nrpyell

using namespace nrpyell;

extern "C" {

void* nrpyell_mlp_create(int n_in, int width, int depth, int n_out, int batch_max, unsigned seed) {
  if (n_in <= 0 || width <= 0 || depth < 0 || n_out <= 0 || batch_max <= 0) {
    NRPYELL_FAIL("nrpyell_mlp_create: sizes must be positive");
    return nullptr;
  }
  Mlp* q = mlp_new(n_in, width, depth, n_out, batch_max, seed);
  if (!status_ok()) {
    mlp_free(q);
    return nullptr;
  }
  return q;
}

void nrpyell_mlp_destroy(void* mlp) { mlp_free((Mlp*)mlp); }

long long nrpyell_mlp_num_params(void* mlp) { return mlp ? ((Mlp*)mlp)->n_params : 0; }

int nrpyell_mlp_get_params(void* mlp, float* host) {
  Mlp* q = (Mlp*)mlp;
  NRPYELL_CUDA(cudaMemcpyAsync(host, q->p, sizeof(float) * q->n_params, cudaMemcpyDeviceToHost, stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  return status_ok() ? 0 : -1;
}
int nrpyell_mlp_set_params(void* mlp, const float* host) {
  Mlp* q = (Mlp*)mlp;
  NRPYELL_CUDA(cudaMemcpyAsync(q->p, host, sizeof(float) * q->n_params, cudaMemcpyHostToDevice, stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  return status_ok() ? 0 : -1;
}

int nrpyell_mlp_predict(void* mlp, const float* x, int n, float* y) {
  Mlp* q = (Mlp*)mlp;
  for (int r0 = 0; r0 < n; r0 += q->batch_max) {
    const int rows = (n - r0 < q->batch_max) ? n - r0 : q->batch_max;
    mlp_forward(q, x + (long long)r0 * q->n_in, rows);
    NRPYELL_CUDA(cudaMemcpyAsync(y + (long long)r0 * q->n_out, q->h.back(), sizeof(float) * rows * q->n_out,
                                 cudaMemcpyDeviceToDevice, stream()));
  }
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  return gemm_ok() ? 0 : -1;
}

double nrpyell_mlp_loss_grad(void* mlp, const float* x, const float* t, int rows, float* grad_host) {
  Mlp* q = (Mlp*)mlp;
  if (rows > q->batch_max || rows <= 0) {
    NRPYELL_FAIL("nrpyell_mlp_loss_grad: need 0 < rows <= batch_max");
    return NAN;
  }
  NRPYELL_CUDA(cudaMemsetAsync(q->loss, 0, sizeof(double), stream()));
  mlp_forward(q, x, rows);
  mlp_backward(q, x, t, rows);
  double loss = NAN;
  NRPYELL_CUDA(cudaMemcpyAsync(&loss, q->loss, sizeof(double), cudaMemcpyDeviceToHost, stream()));
  if (grad_host)
    NRPYELL_CUDA(cudaMemcpyAsync(grad_host, q->grad, sizeof(float) * q->n_params, cudaMemcpyDeviceToHost, stream()));
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  if (!gemm_ok()) return NAN;
  return loss / ((double)rows * q->n_out);
}

double nrpyell_mlp_train(void* mlp, const float* x, const float* t, int n, int batch, int epochs, float lr,
                         unsigned seed, double* loss_history) {
  Mlp* q = (Mlp*)mlp;
  if (batch > q->batch_max || batch <= 0 || n < batch || epochs < 1) {
    NRPYELL_FAIL("nrpyell_mlp_train: need 0 < batch <= batch_max, batch <= n and epochs >= 1");
    return NAN;
  }
  std::vector<int> perm(n);
  for (int i = 0; i < n; i++) perm[i] = i;
  unsigned long long s = 0xD1B54A32D192ED03ull ^ seed;
  const int per_epoch = n / batch;
  const long long total = (long long)per_epoch * epochs;
  long long it = 0;
  double last = NAN;
  for (int e = 0; e < epochs && status_ok(); e++) {
    // the previous epoch's index copies read perm: let them finish first
    NRPYELL_CUDA(cudaStreamSynchronize(stream()));
    for (int i = n - 1; i > 0; i--) {  // Fisher-Yates
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      const int j = (int)((s >> 33) % (unsigned long long)(i + 1));
      const int tmp = perm[i];
      perm[i] = perm[j];
      perm[j] = tmp;
    }
    NRPYELL_CUDA(cudaMemsetAsync(q->loss, 0, sizeof(double), stream()));
    for (int b = 0; b < per_epoch; b++, it++) {
      NRPYELL_CUDA(cudaMemcpyAsync(q->idx, perm.data() + (long long)b * batch, sizeof(int) * batch,
                                   cudaMemcpyHostToDevice, stream()));
      NRPYELL_LAUNCH(k_gather_rows, blocks_for((long long)batch * q->n_in, 256), 256, 0, x, q->idx, batch, q->n_in,
                     q->x);
      NRPYELL_LAUNCH(k_gather_rows, blocks_for((long long)batch * q->n_out, 256), 256, 0, t, q->idx, batch,
                     q->n_out, q->t);
      mlp_forward(q, q->x, batch);
      mlp_backward(q, q->x, q->t, batch);
      const float lr_t = lr * (0.01f + 0.99f * 0.5f * (1.f + cosf(3.14159265f * (float)it / (float)total)));
      mlp_adam(q, lr_t);
    }
    double sum = 0.0;
    NRPYELL_CUDA(cudaMemcpyAsync(&sum, q->loss, sizeof(double), cudaMemcpyDeviceToHost, stream()));
    NRPYELL_CUDA(cudaStreamSynchronize(stream()));
    if (!gemm_ok()) return NAN;
    last = sum / ((double)per_epoch * batch * q->n_out);
    if (loss_history) loss_history[e] = last;
  }
  return last;
}

int nrpyell_pod_guess(const float* mean, const float* basis, int K, long long ntot, const float* c, double eta,
                      double* y_n) {
  if (K <= 0 || K > 4096 || ntot <= 0) {
    NRPYELL_FAIL("nrpyell_pod_guess: need 0 < K <= 4096 and ntot > 0");
    return -1;
  }
  NRPYELL_LAUNCH(k_pod_guess, blocks_for(ntot, 256), 256, sizeof(float) * K, mean, basis, K, ntot, c, eta, y_n);
  NRPYELL_CUDA(cudaStreamSynchronize(stream()));
  return status_ok() ? 0 : -1;
}

}  // extern "C"
