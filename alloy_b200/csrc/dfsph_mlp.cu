// SPDX-License-Identifier: Apache-2.0
// C ABI of the warm-start network (include/alloy_dfsph.h, adf_mlp_*): its parameters on the device, tcgen05 inference
// over rows of normalised features, and Adam training steps whose forward and backward passes run on the tensor
// cores (dfsph_mlp.cuh). The solver takes a trained network with adf_set_warm_model.
#include <algorithm>
#include <cstring>
#include <string>

#include "../../include/alloy_dfsph.h"
#define ADF_MLP_STANDALONE
#include "dfsph_mlp.cuh"

namespace adf {
void set_last_error(const std::string& msg);
}

using namespace adf::mlp;

namespace {

int fail(int code, const std::string& msg) {
  adf::set_last_error(msg);
  return code;
}

#define CKM(x)                                                                                          \
  do {                                                                                                  \
    cudaError_t e_ = (x);                                                                               \
    if (e_ != cudaSuccess) return fail(ADF_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

Net net_of(const adf_mlp* m) { return Net{m->w1b, m->w2b, m->w, nullptr, m->error, m->wait_limit}; }

int set_params(adf_mlp* m, const float* host) {
  CKM(cudaMemcpy(m->w, host, sizeof(float) * N_PARAMS, cudaMemcpyHostToDevice));
  CKM(cudaMemset(m->m, 0, sizeof(float) * N_PARAMS));
  CKM(cudaMemset(m->v, 0, sizeof(float) * N_PARAMS));
  k_mlp_to_bf16<<<(NH * NH + 255) / 256, 256>>>(m->w, m->w1b, m->w2b);
  CKM(cudaGetLastError());
  CKM(cudaDeviceSynchronize());
  m->step = 0;
  return ADF_OK;
}

int grad_launch(adf_mlp* m, const float* x, const float* y, const int32_t* idx, int batch, cudaStream_t st,
                int* grid_out) {
  const int tiles = (batch + TILE - 1) / TILE;
  const int grid = std::max(1, std::min(tiles, m->sms));
  k_mlp_grad<<<grid, TILE, TR_SMEM, st>>>(net_of(m), x, y, idx, batch, m->part);
  CKM(cudaGetLastError());
  *grid_out = grid;
  return ADF_OK;
}

}  // namespace

extern "C" {

int adf_mlp_create(const float* params, int device, adf_mlp** out) {
  if (!params || !out) return fail(ADF_ERR_VALUE, "adf_mlp_create: null argument");
  *out = nullptr;
  CKM(cudaSetDevice(device));
  adf_mlp* m = new adf_mlp();
  m->device = device;
  cudaDeviceGetAttribute(&m->sms, cudaDevAttrMultiProcessorCount, device);
  m->sms = std::max(m->sms, 1);
  cudaError_t e = cudaSuccess;
  auto al = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
  };
  al((void**)&m->w, sizeof(float) * N_PARAMS);
  al((void**)&m->m, sizeof(float) * N_PARAMS);
  al((void**)&m->v, sizeof(float) * N_PARAMS);
  al((void**)&m->w1b, sizeof(__nv_bfloat16) * NH * NF);
  al((void**)&m->w2b, sizeof(__nv_bfloat16) * NH * NH);
  al((void**)&m->part, sizeof(float) * (size_t)m->sms * (N_PARAMS + 1));
  al((void**)&m->grad, sizeof(float) * N_PARAMS);
  al((void**)&m->loss, sizeof(float));
  al((void**)&m->error, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(m->error, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, TR_SMEM);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, FW_SMEM);
  if (e != cudaSuccess) {
    adf_mlp_destroy(m);
    return fail(ADF_ERR_CUDA, std::string("adf_mlp_create: ") + cudaGetErrorString(e));
  }
  int rc = set_params(m, params);
  if (rc) {
    adf_mlp_destroy(m);
    return rc;
  }
  *out = m;
  return ADF_OK;
}

void adf_mlp_destroy(adf_mlp* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  cudaDeviceSynchronize();
  void* ps[] = {m->w, m->m, m->v, m->w1b, m->w2b, m->part, m->grad, m->loss, m->error};
  for (void* p : ps)
    if (p) cudaFree(p);
  delete m;
}

int adf_mlp_set_params(adf_mlp* m, const float* params) {
  if (!m || !params) return fail(ADF_ERR_VALUE, "adf_mlp_set_params: null argument");
  CKM(cudaSetDevice(m->device));
  return set_params(m, params);
}

int adf_mlp_get_params(adf_mlp* m, float* params) {
  if (!m || !params) return fail(ADF_ERR_VALUE, "adf_mlp_get_params: null argument");
  CKM(cudaSetDevice(m->device));
  CKM(cudaDeviceSynchronize());
  CKM(cudaMemcpy(params, m->w, sizeof(float) * N_PARAMS, cudaMemcpyDeviceToHost));
  return ADF_OK;
}

int adf_mlp_forward(adf_mlp* m, const float* x, int n, float* y, void* stream) {
  if (!m || (n > 0 && (!x || !y))) return fail(ADF_ERR_VALUE, "adf_mlp_forward: null argument");
  if (n <= 0) return ADF_OK;
  CKM(cudaSetDevice(m->device));
  const int tiles = (n + TILE - 1) / TILE;
  const int grid = std::max(1, std::min(tiles, 4 * m->sms));
  k_mlp_forward<<<grid, TILE, FW_SMEM, (cudaStream_t)stream>>>(net_of(m), x, y, n);
  CKM(cudaGetLastError());
  return ADF_OK;
}

int adf_mlp_gradient(adf_mlp* m, const float* x, const float* y, const int32_t* idx, int batch, float* grad,
                     float* loss, void* stream) {
  if (!m || !x || !y || !idx || batch <= 0) return fail(ADF_ERR_VALUE, "adf_mlp_gradient: bad argument");
  CKM(cudaSetDevice(m->device));
  cudaStream_t st = (cudaStream_t)stream;
  int grid = 0;
  int rc = grad_launch(m, x, y, idx, batch, st, &grid);
  if (rc) return rc;
  k_mlp_adam<<<(N_PARAMS + 256) / 256, 256, 0, st>>>(m->part, grid, batch, m->w, m->m, m->v, m->w1b, m->w2b, 0.0f,
                                                      0.9f, 0.999f, 1e-8f, 1, 0, m->grad, m->loss);
  CKM(cudaGetLastError());
  CKM(cudaStreamSynchronize(st));
  if (grad) CKM(cudaMemcpy(grad, m->grad, sizeof(float) * N_PARAMS, cudaMemcpyDeviceToHost));
  if (loss) CKM(cudaMemcpy(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
  return ADF_OK;
}

int adf_mlp_train_step(adf_mlp* m, const float* x, const float* y, const int32_t* idx, int batch, float lr,
                       float* loss, void* stream) {
  if (!m || !x || !y || !idx || batch <= 0) return fail(ADF_ERR_VALUE, "adf_mlp_train_step: bad argument");
  if (!(lr > 0.0f)) return fail(ADF_ERR_VALUE, "adf_mlp_train_step: learning rate must be > 0");
  CKM(cudaSetDevice(m->device));
  cudaStream_t st = (cudaStream_t)stream;
  int grid = 0;
  int rc = grad_launch(m, x, y, idx, batch, st, &grid);
  if (rc) return rc;
  ++m->step;
  k_mlp_adam<<<(N_PARAMS + 256) / 256, 256, 0, st>>>(m->part, grid, batch, m->w, m->m, m->v, m->w1b, m->w2b, lr,
                                                      0.9f, 0.999f, 1e-8f, m->step, 1, nullptr, m->loss);
  CKM(cudaGetLastError());
  if (loss) {
    CKM(cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    CKM(cudaStreamSynchronize(st));
  }
  return ADF_OK;
}

int adf_mlp_set_wait_limit(adf_mlp* m, uint32_t polls) {
  if (!m) return fail(ADF_ERR_VALUE, "adf_mlp_set_wait_limit: null argument");
  m->wait_limit = polls;
  return ADF_OK;
}

int adf_mlp_clear_status(adf_mlp* m) {
  if (!m) return fail(ADF_ERR_VALUE, "adf_mlp_clear_status: null argument");
  CKM(cudaSetDevice(m->device));
  CKM(cudaDeviceSynchronize());
  CKM(cudaMemset(m->error, 0, sizeof(int)));
  return ADF_OK;
}

int adf_mlp_status(adf_mlp* m) {
  if (!m) return fail(ADF_ERR_VALUE, "adf_mlp_status: null argument");
  CKM(cudaSetDevice(m->device));
  int e = 0;
  CKM(cudaMemcpy(&e, m->error, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) return fail(ADF_ERR_STATE, "warm-start network: a tensor-core wait expired (results invalid)");
  return ADF_OK;
}

}  // extern "C"
