// Jacobi-BiCGSTAB without any allocation by the caller: the work space lives in this library's
// own static device memory.
//
// Some callers cannot allocate device memory: a host code that reaches the solver only through
// this C ABI and owns no CUDA allocator (for instance a C or Fortran CFD code that is handed
// device pointers by another component and must not create allocations outside that
// component's memory pool), or an embedding application whose device-memory budget is fixed and
// fully handed out before the solver runs. b2s_bicgstab_jacobi_d needs a work array from its
// caller; this entry point takes the same inputs and outputs without one.
//
// The scratch is a file-scope __device__ array sized for B2S_NOALLOC_MAX_UNKNOWNS unknowns
// (n * nrhs); every GPU that loads the library holds it until the process exits. In host code
// the array's name is only a host-side stand-in, so its device address is looked up with
// cudaGetSymbolAddress, once per device, with that device current, on the first call on that
// device (make that first call before any stream capture). Every call on a device shares the
// one array, so calls that overlap on the GPU (concurrent streams, or several host threads)
// race on it: serialise them. The solve initialises every scratch value it reads before reading
// it (r, r_hat, u, p, v and w are set in its first phase, the rest are written before use), so the
// contents left by the previous call do not matter.
#include <mutex>

#include "b2s_common.cuh"

namespace {

constexpr int64_t kScratchDoubles =
    (int64_t)b2s::kBicgVectors * B2S_NOALLOC_MAX_UNKNOWNS + (int64_t)2 * b2s::kMaxCoopBlocks * 3 * 3;

__device__ __align__(256) double g_bicgstab_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

}  // namespace

extern "C" int b2s_bicgstab_jacobi_noalloc_d(int32_t n, int nrhs, const int32_t* rowptr, const int32_t* col,
                                             const double* val, const double* b, const double* inv_diag, double* x,
                                             double tol, int maxiter, int relative_to_initial, b2s_solve_info* info,
                                             b2s_stream_t s) {
  if (n <= 0 || nrhs < 1 || nrhs > 3) return B2S_ERR_ARG;
  if ((int64_t)n * nrhs > B2S_NOALLOC_MAX_UNKNOWNS) return B2S_ERR_TOO_LARGE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return B2S_ERR_DEVICE;
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
      void* addr = nullptr;
      if (cudaGetSymbolAddress(&addr, g_bicgstab_scratch) != cudaSuccess || !addr) return B2S_ERR_DEVICE;
      g_scratch_addr[dev] = (double*)addr;
    }
    scratch = g_scratch_addr[dev];
  }
  const int64_t need = b2s_bicgstab_workspace_bytes(n, nrhs);
  if (need < 0 || need > (int64_t)sizeof(double) * kScratchDoubles) return B2S_ERR_TOO_LARGE;
  return b2s_bicgstab_jacobi_d(n, nrhs, rowptr, col, val, b, inv_diag, x, tol, maxiter, relative_to_initial, scratch,
                               (int64_t)sizeof(double) * kScratchDoubles, info, s);
}
