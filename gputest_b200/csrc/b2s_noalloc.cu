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
// (n * nrhs): 11 vectors of 131,072 doubles plus 2 x 1184 x 9 doubles of block partials,
// 11,704,832 bytes, which every GPU that loads the library holds until the process exits. In
// host code the array's name is only a host-side stand-in, so its device address is looked up
// with cudaGetSymbolAddress with the device current, on the first call in each CUDA context of a
// device (the primary context that the runtime and torch use, or a context the caller made with
// the driver API): the address is kept per device together with the id of the context it was
// looked up in, and looked up again when the current context differs (after a
// cudaDeviceReset, for instance). Make the first call on a device before any stream capture.
// Every call on a device shares the one array, so calls that overlap on the GPU (concurrent
// streams, or several host threads) race on it: serialise them. The solve initialises every scratch value it reads before reading
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
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // id of the context each address belongs to

// The id of the current CUDA context (cuCtxGetCurrent + cuCtxGetId, reached through the
// runtime's driver entry points so the library does not link the driver library itself).
// 0 when either call is unavailable: the address is then looked up on every call.
typedef int (*ctx_get_current_fn)(void**);
typedef int (*ctx_get_id_fn)(void*, unsigned long long*);

unsigned long long current_context_id() {
  static ctx_get_current_fn get_current = nullptr;
  static ctx_get_id_fn get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (ctx_get_current_fn)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (ctx_get_id_fn)f;
    looked_up = true;
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

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
    const unsigned long long ctx = current_context_id();
    if (!g_scratch_addr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
      // the lookup also makes the device's primary context current when no context is yet
      void* addr = nullptr;
      if (cudaGetSymbolAddress(&addr, g_bicgstab_scratch) != cudaSuccess || !addr) return B2S_ERR_DEVICE;
      g_scratch_addr[dev] = (double*)addr;
      g_scratch_ctx[dev] = current_context_id();
    }
    scratch = g_scratch_addr[dev];
  }
  const int64_t need = b2s_bicgstab_workspace_bytes(n, nrhs);
  if (need < 0 || need > (int64_t)sizeof(double) * kScratchDoubles) return B2S_ERR_TOO_LARGE;
  return b2s_bicgstab_jacobi_d(n, nrhs, rowptr, col, val, b, inv_diag, x, tol, maxiter, relative_to_initial, scratch,
                               (int64_t)sizeof(double) * kScratchDoubles, info, s);
}
