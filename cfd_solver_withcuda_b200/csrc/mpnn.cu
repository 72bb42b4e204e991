// Kernels of the warm-start surrogate (a message-passing network on the cell/face graph of a
// mesh): the graph operations are deterministic segment sums over CSR lists (aggregation of the
// face messages into cells, and the backward pass of the per-edge gathers), and the optimiser is
// one fused Adam step.  The dense layers are plain BF16 GEMMs done by the caller.  No reference
// counterpart.
#include <cuda_runtime.h>

#include <string>

#include "cfd_b200.h"

namespace cfdb {
void set_last_error(const std::string &msg);
}

namespace {

// out[r, :] = sum over j in [ptr[r], ptr[r+1]) of x[idx[j], :], in list order (one warp per row,
// lanes over columns), so the sums are the same on every run.
__global__ void k_segment_sum(const float *__restrict__ x, const int *__restrict__ ptr, const int *__restrict__ idx,
                              int n_rows, int width, float *__restrict__ out) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n_rows) return;
  const int b = ptr[row], e = ptr[row + 1];
  for (int col = lane; col < width; col += 32) {
    float acc = 0.f;
    for (int j = b; j < e; j++) acc += x[(size_t)idx[j] * width + col];
    out[(size_t)row * width + col] = acc;
  }
}

// One Adam step (bias-corrected moments) over n parameters.
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int n, float lr, float b1, float b2, float eps, float bc1, float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

cfd_status launch_status(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return CFD_OK;
  cfdb::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return CFD_ERR_CUDA;
}

}  // namespace

extern "C" {

cfd_status cfd_mpnn_segment_sum(const float *x, const int *ptr, const int *idx, int n_rows, int width, float *out,
                                void *stream) {
  if (n_rows < 0 || width < 1 || (n_rows > 0 && (!x || !ptr || !idx || !out))) {
    cfdb::set_last_error("cfd_mpnn_segment_sum: bad argument");
    return CFD_ERR_BAD_ARG;
  }
  if (n_rows == 0) return CFD_OK;
  const int threads = 256, rows_per_block = threads / 32;
  k_segment_sum<<<(n_rows + rows_per_block - 1) / rows_per_block, threads, 0, static_cast<cudaStream_t>(stream)>>>(
      x, ptr, idx, n_rows, width, out);
  return launch_status("cfd_mpnn_segment_sum");
}

cfd_status cfd_mpnn_adam(float *param, const float *grad, float *m, float *v, int n, float lr, float beta1,
                         float beta2, float eps, int step, void *stream) {
  if (n < 0 || step < 1 || (n > 0 && (!param || !grad || !m || !v))) {
    cfdb::set_last_error("cfd_mpnn_adam: bad argument");
    return CFD_ERR_BAD_ARG;
  }
  if (n == 0) return CFD_OK;
  float bc1 = 1.f, bc2 = 1.f;
  for (int i = 0; i < step; i++) {
    bc1 *= beta1;
    bc2 *= beta2;
  }
  bc1 = 1.f - bc1;
  bc2 = 1.f - bc2;
  k_adam<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(param, grad, m, v, n, lr, beta1, beta2, eps,
                                                                         bc1, bc2);
  return launch_status("cfd_mpnn_adam");
}

}  // extern "C"
