// Cost of a grid-wide barrier on this GPU, with and without the fixed-order reduction of block
// partials that the cooperative Krylov kernels perform after each barrier. Not part of the
// library: it measured the launch geometry of the cooperative kernels (one block per SM).
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o grid_barrier gputest_b200/csrc/probes/grid_barrier.cu
#include <cooperative_groups.h>
#include <cstdio>
namespace cg = cooperative_groups;
__global__ void k_sync(int ns, double* part, double* out) {
  cg::grid_group g = cg::this_grid();
  double acc = 0.0;
  for (int i = 0; i < ns; ++i) {
    if (threadIdx.x == 0) part[(i & 1) * gridDim.x + blockIdx.x] = (double)i;
    g.sync();
    if (threadIdx.x < 32) {
      double s = 0.0;
      for (int b = threadIdx.x; b < gridDim.x; b += 32) s += part[(i & 1) * gridDim.x + b];
      acc += s;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = acc;
}
__global__ void k_plain(int ns, double* out) {
  cg::grid_group g = cg::this_grid();
  for (int i = 0; i < ns; ++i) g.sync();
  if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = 1.0;
}
int main() {
  int sms = 0; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  double *part, *out; cudaMalloc(&part, 2 * 4096 * sizeof(double)); cudaMalloc(&out, 8);
  cudaEvent_t a, b; cudaEventCreate(&a); cudaEventCreate(&b);
  int threads_list[] = {128, 256, 512, 1024};
  for (int ti = 0; ti < 4; ++ti) {
    int th = threads_list[ti];
    int per = 0; cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sync, th, 0);
    for (int bp = 1; bp <= per && bp <= 8; bp *= 2) {
      int g = sms * bp; int ns = 2000;
      void* args[] = {&ns, &part, &out};
      cudaLaunchCooperativeKernel((void*)k_sync, g, th, args, 0, 0);  // warm
      cudaEventRecord(a);
      cudaLaunchCooperativeKernel((void*)k_sync, g, th, args, 0, 0);
      cudaEventRecord(b); cudaEventSynchronize(b);
      float ms = 0; cudaEventElapsedTime(&ms, a, b);
      void* args2[] = {&ns, &out};
      cudaLaunchCooperativeKernel((void*)k_plain, g, th, args2, 0, 0);
      cudaEventRecord(a);
      cudaLaunchCooperativeKernel((void*)k_plain, g, th, args2, 0, 0);
      cudaEventRecord(b); cudaEventSynchronize(b);
      float ms2 = 0; cudaEventElapsedTime(&ms2, a, b);
      printf("threads %4d blocks %4d (%d/SM): sync+reduce %.3f us, bare sync %.3f us\n", th, g, bp, 1e3 * ms / ns, 1e3 * ms2 / ns);
    }
  }
  cudaError_t e = cudaGetLastError(); printf("status %s\n", cudaGetErrorString(e));
  return 0;
}
