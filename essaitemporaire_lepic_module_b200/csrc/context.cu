// Per-device context: error word, scratch buffers, status helpers.
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "lepic_internal.cuh"

namespace lepic {

namespace {
std::mutex g_mu;
std::map<int, Ctx> g_ctx;
struct Buf {
  void *p = nullptr;
  size_t bytes = 0;
};
std::map<std::pair<int, std::string>, Buf> g_scratch;
thread_local int g_last_cuda_error = 0;
}  // namespace

int cuda_status(cudaError_t e, const char *what) {
  g_last_cuda_error = (int)e;
  fprintf(stderr, "lepic_gpu: CUDA error %d (%s) in %s\n", (int)e, cudaGetErrorString(e), what);
  return LEPIC_ERR_CUDA;
}

Ctx &ctx() {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_mu);
  Ctx &c = g_ctx[dev];
  if (c.device < 0) {
    c.device = dev;
    cudaGetDeviceProperties(&c.prop, dev);
    c.sms = c.prop.multiProcessorCount;
    cudaMalloc(&c.d_err, 2 * sizeof(int));
    cudaMemset(c.d_err, 0, 2 * sizeof(int));
    cudaMallocHost(&c.h_err, 2 * sizeof(int));
    c.h_err[0] = c.h_err[1] = 0;
  }
  return c;
}

void *scratch(const char *name, size_t bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_mu);
  Buf &b = g_scratch[{dev, std::string(name)}];
  if (b.bytes < bytes) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    size_t want = bytes + bytes / 8 + 256;
    if (cudaMalloc(&b.p, want) != cudaSuccess) {
      b.p = nullptr;
      return nullptr;
    }
    b.bytes = want;
  }
  return b.p;
}

// Synchronise the stream, read and clear the device error word.
int check_err(cudaStream_t s) {
  Ctx &c = ctx();
  cudaError_t e = cudaMemcpyAsync(c.h_err, c.d_err, 2 * sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return cuda_status(e, "read error word");
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "stream synchronize");
  int code = c.h_err[0];
  if (code) {
    fprintf(stderr, "lepic_gpu: device status %d (detail %d)\n", code, c.h_err[1]);
    cudaMemsetAsync(c.d_err, 0, 2 * sizeof(int), s);
    cudaStreamSynchronize(s);
  }
  return code;
}

}  // namespace lepic
