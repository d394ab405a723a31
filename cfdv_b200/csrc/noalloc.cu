// cfdv_ebe_matvec_static: the EBE product for callers that may not allocate device memory.
//
// A context allocates its element-product buffer with cudaMalloc.  Some callers cannot let
// a library do that: an application whose memory pool already holds the GPU's free memory
// (a cudaMalloc from here would fail), or one that cannot afford the device-wide
// synchronisation of cudaFree between its other streams' work.  This entry point takes all
// inputs and the output as the caller's device pointers and keeps the one intermediate it
// needs, the element products Y_e = R_e x_e, in a static device array compiled into the
// library.  The kernels are the ones cfdv_matvec launches (solver.cu), so results agree.
//
// Host code must not hand the array's name to a kernel: on the host that name is a
// stand-in object, not the device address.  The device address is looked up once per
// device with cudaGetSymbolAddress while that device is current, checked, and cached.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "../../include/cfdv_gpu.h"
#include "kernels.h"

// Element products of the last call (shared by every call; nothing in it needs clearing:
// the element pass writes every entry the node pass then reads).
static __device__ __align__(256) double cfdv_static_elem_products[CFDV_STATIC_SCRATCH_DOUBLES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
std::atomic<double*> g_scratch[kMaxDevices];  // static storage: starts as nullptr

// is `p` device memory of device `dev` (the runtime's view)?
bool on_device(const void* p, int dev) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice && at.device == dev;
}

// device address of the scratch array on the current device `dev`.  The address found at
// the first call is kept; a later call checks that it still names memory of this device
// (a cudaDeviceReset unloads the library's module and the array moves when it is loaded
// again) and looks it up again when it does not.
int scratch_on_device(int dev, double** out) {
  double* p = g_scratch[dev].load(std::memory_order_acquire);
  if (p && on_device(p, dev)) {
    *out = p;
    return CFDV_OK;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  p = g_scratch[dev].load(std::memory_order_relaxed);
  if (!p || !on_device(p, dev)) {
    void* addr = nullptr;
    if (cudaGetSymbolAddress(&addr, cfdv_static_elem_products) != cudaSuccess || !addr) {
      cudaGetLastError();
      return CFDV_ERR_CUDA;
    }
    p = static_cast<double*>(addr);
    g_scratch[dev].store(p, std::memory_order_release);
  }
  *out = p;
  return CFDV_OK;
}

// The kernels run on device `dev`: accept its own device memory and managed memory, and
// reject everything else -- pageable host memory, pinned host memory (reachable over the
// bus, but not what this entry point promises to read) and another GPU's memory, whose
// loads would fault instead of returning an error here.
bool device_reachable(const void* p, int dev) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (at.type == cudaMemoryTypeManaged) return true;
  return at.type == cudaMemoryTypeDevice && at.device == dev;
}

}  // namespace

extern "C" int cfdv_ebe_matvec_static(int ndim, int n_nodes, int n_elements, const int* conn, const int* node_ptr,
                                      const int* node_idx, const double* R, const double* x, double* y,
                                      int transpose, void* stream) {
  if ((ndim != 2 && ndim != 3) || n_nodes <= 0 || n_elements <= 0) return CFDV_ERR_ARG;
  if (!conn || !node_ptr || !node_idx || !R || !x || !y) return CFDV_ERR_ARG;
  const int nnod = ndim == 2 ? 4 : 8, neqn = ndim + 2, Ke = nnod * neqn;
  if ((size_t)n_elements * (size_t)Ke > (size_t)CFDV_STATIC_SCRATCH_DOUBLES) return CFDV_ERR_TOO_LARGE;
  if ((size_t)n_nodes * (size_t)neqn > (size_t)0x7fffffff) return CFDV_ERR_TOO_LARGE;
  const int n_dof = n_nodes * neqn;
  if (x == y) return CFDV_ERR_ARG;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return CFDV_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return CFDV_ERR_ARG;
  const void* ptrs[] = {conn, node_ptr, node_idx, R, x, y};
  for (const void* p : ptrs)
    if (!device_reachable(p, dev)) return CFDV_ERR_ARG;
  double* scratch = nullptr;
  if (int rc = scratch_on_device(dev, &scratch)) return rc;

  cfdv::EbeArgs a;
  a.ndim = ndim; a.nnod = nnod; a.neqn = neqn; a.n_elements = n_elements; a.n_dof = n_dof;
  a.conn = conn; a.csr_ptr = node_ptr; a.csr_idx = node_idx;
  a.R64 = R; a.R32 = nullptr; a.Y64 = scratch; a.Y32 = nullptr;
  const cudaError_t err = cfdv::launch_ebe(a, 0, transpose ? 1 : 0, x, y, 0, nullptr, nullptr, nullptr,
                                           static_cast<cudaStream_t>(stream));
  return err == cudaSuccess ? CFDV_OK : CFDV_ERR_CUDA;
}
