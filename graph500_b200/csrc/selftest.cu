// Device self-test of the failure path of the grid barrier.  Every persistent
// kernel here waits for all of its blocks at grid barriers with bounded polls;
// a block that never arrives (a fault elsewhere, a block that returned early)
// must make the others give up, set the error flag and return, so that the
// call reports G500_E_TIMEOUT and the CUDA context stays usable.  This test
// makes exactly that happen on purpose and safely: one block of a cooperative
// launch returns before the barrier, the others wait with a short poll limit.
// No counterpart in the reference.
#include "g500_internal.cuh"
#include "device_common.cuh"

namespace g500 {

__global__ void barrier_timeout_kernel(GridBarrier* bar, unsigned long long spin_limit, unsigned* passed) {
  __shared__ unsigned long long sh_cnt[1], sh_acc[1];
  __shared__ unsigned sh_flag;
  if (threadIdx.x == 0) sh_acc[0] = 0;
  __syncthreads();
  if (blockIdx.x == 0) return;  // the block that never arrives
  if (grid_sync<1>(bar, nullptr, sh_acc, nullptr, sh_cnt, &sh_flag, spin_limit) && threadIdx.x == 0)
    atomicAdd(passed, 1u);  // must not happen
}

__global__ void barrier_pass_kernel(GridBarrier* bar, unsigned* passed) {
  __shared__ unsigned long long sh_cnt[1], sh_acc[1];
  __shared__ unsigned sh_flag;
  if (threadIdx.x == 0) sh_acc[0] = 0;
  __syncthreads();
  if (grid_sync<1>(bar, nullptr, sh_acc, nullptr, sh_cnt, &sh_flag) && threadIdx.x == 0) atomicAdd(passed, 1u);
}

}  // namespace g500

using namespace g500;

extern "C" int g500_selftest_barrier_timeout(int device, int* timed_out, int* recovered) {
  if (!timed_out || !recovered) return set_error(G500_E_INVAL, "null argument");
  *timed_out = *recovered = 0;
  G500_CUDA(cudaSetDevice(device));
  GridBarrier* bar = nullptr;
  unsigned* passed = nullptr;
  G500_TRY(dev_alloc_n(&bar, 1, "barrier"));
  int st = dev_alloc_n(&passed, 1, "counter");
  const unsigned blocks = 8;  // far below the device's co-resident limit
  unsigned long long limit = 1ull << 14;  // a few milliseconds of polls
  GridBarrier hb{};
  unsigned hp = 0;
  if (st == G500_OK) {
    cudaError_t e = cudaMemset(bar, 0, sizeof(GridBarrier));
    if (e == cudaSuccess) e = cudaMemset(passed, 0, sizeof(unsigned));
    void* args[] = {&bar, &limit, &passed};
    if (e == cudaSuccess) e = cudaLaunchCooperativeKernel((const void*)barrier_timeout_kernel, blocks, 64, args, 0, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&hb, bar, sizeof(hb), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&hp, passed, sizeof(hp), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = cuda_error(e, "barrier timeout test", __FILE__, __LINE__);
    *timed_out = (st == G500_OK && (hb.err & GRID_ERR_TIMEOUT) && hp == 0) ? 1 : 0;
  }
  // the context is still usable: a full barrier on fresh state completes
  if (st == G500_OK) {
    cudaError_t e = cudaMemset(bar, 0, sizeof(GridBarrier));
    if (e == cudaSuccess) e = cudaMemset(passed, 0, sizeof(unsigned));
    void* args[] = {&bar, &passed};
    if (e == cudaSuccess) e = cudaLaunchCooperativeKernel((const void*)barrier_pass_kernel, blocks, 64, args, 0, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&hb, bar, sizeof(hb), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&hp, passed, sizeof(hp), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = cuda_error(e, "barrier recovery test", __FILE__, __LINE__);
    *recovered = (st == G500_OK && hb.err == 0 && hp == blocks) ? 1 : 0;
  }
  dev_free(bar);
  dev_free(passed);
  return st;
}
