// fj_rhs_noalloc.cu -- fj_rhs_noalloc_f64: the block RHS for callers that must
// not allocate device memory.
//
// Who needs it: a caller whose device memory belongs to someone else.  The
// typical case is this library bound into JAX as an XLA custom call: XLA
// reserves most of the GPU's memory for its own pool when the process starts,
// so a cudaMalloc issued from inside a custom call can fail for lack of
// memory, and in any case takes memory the framework believes it owns.
// Solver loops that fix their memory budget at start-up and forbid allocation
// afterwards are in the same position.  fj_rhs_f64 cannot serve them: its
// context grows its scratch with cudaMalloc on first use.
//
// How: the RHS intermediates (primitives, viscous flux components, the three
// face-flux arrays) live in the file-scope device array below instead of
// context scratch.  Host code must not pass the array's name to a kernel: on
// the host that name denotes a host-side placeholder, not device memory.  The
// device address is looked up once per device with cudaGetSymbolAddress (with
// that device current) and cached for the life of the process: a
// cudaDeviceReset while the library is in use (which would recreate the
// context and could move the array) is not supported.
//
// Error attribution: a call finds the runtime's last-error state clear or
// returns FJ_ERR_CUDA at once, leaving that earlier error for its owner to
// read; a failure reported after the launches is then this call's own.
#include <mutex>

#include "fj_common.cuh"
#include "fj_rhs.cuh"

namespace {

// Capacity of the shared scratch: FJ_NOALLOC_SCRATCH_BYTES (64 MiB).  The
// array is reserved on a device when this file's module is loaded there: at
// its first use under lazy module loading (the CUDA default), or at context
// creation on every device under CUDA_MODULE_LOADING=EAGER, whether or not
// the entry point runs there.  It is held until the process exits.
static __device__ __align__(256) unsigned char g_rhs_scratch[FJ_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_addr[kMaxDevices] = {};

}  // namespace

using namespace fj;

extern "C" int fj_rhs_noalloc_f64(const double* q, const double* kxyz, const double* vol,
                                  double* rhs, int ni, int nj, int nk, const fj_params* p,
                                  void* stream) {
  int s = check_params(nullptr, p);
  if (s != FJ_OK) return s;
  s = check_dims(nullptr, ni, nj, nk);
  if (s != FJ_OK) return s;
  if (!q || !kxyz || !vol || !rhs) return FJ_ERR_INVALID_ARGUMENT;
  const size_t need = p->precision == FJ_PREC_F32FLUX ? staged_ws_bytes<float>(ni, nj, nk)
                                                      : staged_ws_bytes<double>(ni, nj, nk);
  if (need > (size_t)FJ_NOALLOC_SCRATCH_BYTES) return FJ_ERR_SCRATCH_LIMIT;
  // an error left by an earlier, unrelated call stays for its owner to read
  if (cudaPeekAtLastError() != cudaSuccess) return FJ_ERR_CUDA;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return FJ_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return FJ_ERR_INVALID_ARGUMENT;
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
      void* addr = nullptr;
      if (cudaGetSymbolAddress(&addr, g_rhs_scratch) != cudaSuccess || !addr) {
        cudaGetLastError();
        return FJ_ERR_CUDA;
      }
      g_scratch_addr[dev] = addr;
    }
    scratch = g_scratch_addr[dev];
  }
  // Every scratch element a call reads is written earlier in the same call, so
  // nothing needs clearing between calls.
  const Phys ph = make_phys(p);
  cudaError_t e =
      p->precision == FJ_PREC_F32FLUX
          ? staged_rhs_noctx<float>(q, kxyz, vol, rhs, ni, nj, nk, ph, scratch, (cudaStream_t)stream)
          : staged_rhs_noctx<double>(q, kxyz, vol, rhs, ni, nj, nk, ph, scratch, (cudaStream_t)stream);
  return e == cudaSuccess ? FJ_OK : FJ_ERR_CUDA;
}
