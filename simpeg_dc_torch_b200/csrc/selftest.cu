// Self-test of the bounded device waits (failure detection without a GPU
// fault).  Every spin of the tensor-core kernels on an mbarrier is bounded:
// after its poll limit the waiting CTA records DCT_ERR_DEVICE_TIMEOUT in the
// plan's status words and returns, so the host sees an error status and the
// context stays usable.  dct_selftest_wait_timeout runs that same wait
// (tc_wait) on an mbarrier that nothing ever arrives on, with a short limit,
// and reports the status it left -- the path a hung MMA or bulk copy would
// take, made to run out on purpose without any asynchronous operation in
// flight.
#include <cuda_runtime.h>

#include "dct_internal.h"
#include "tc_common.cuh"

namespace dct {
namespace {

__global__ void k_wait_timeout(uint32_t polls, int* status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) mbar_init(&bar);   // one arrival expected, none comes
  __syncthreads();
  const bool ok = tc_wait(&bar, 0u, status, DCT_ERR_DEVICE_TIMEOUT, -1, 0, polls);
  if (threadIdx.x == 0) status[3] = ok ? 1 : 0;   // the wait's own verdict
}

}  // namespace
}  // namespace dct

extern "C" int dct_selftest_wait_timeout(int32_t polls, int32_t* code, int32_t* completed,
                                         void* stream) {
  if (polls < 1 || polls > (1 << 16) || !code) return DCT_ERR_ARG;
  int* d = nullptr;
  cudaError_t e = cudaMalloc(&d, 4 * sizeof(int));
  if (e != cudaSuccess) return DCT_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int h[4] = {0, 0, 0, 0};
  e = cudaMemsetAsync(d, 0, 4 * sizeof(int), st);
  if (e == cudaSuccess) {
    dct::k_wait_timeout<<<1, 128, 0, st>>>(static_cast<uint32_t>(polls), d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d);
  if (e != cudaSuccess) return DCT_ERR_CUDA;
  *code = h[0];
  if (completed) *completed = h[3];
  return DCT_OK;
}
