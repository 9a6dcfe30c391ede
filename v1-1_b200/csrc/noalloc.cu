// Allocation-free form of the Toeplitz/FFT Coulomb solve (op_tinv).
//
// Some callers cannot call cudaMalloc when they need the solve: a process whose
// device memory is partitioned once at start-up by its own memory manager (a
// serving process that sizes its pools to fill HBM and forbids later library
// allocations), or a latency-critical loop that cannot accept the device-wide
// synchronisation cudaMalloc and cudaFree may cause.  The regular entry point
// grows its workspace with cudaMalloc on first use; this one keeps the FFT
// scratch of the solve in a fixed device array owned by the library, so the
// call itself allocates nothing.  The caller passes the inputs and outputs.
//
// The array has a fixed size (kScratchBytes, 64 MiB) and lives on every GPU
// that loads this library until the process exits.  Every call on a device
// shares it and it keeps the contents of the last call; the solve writes every
// scratch element before it reads it, so nothing has to be cleared.  Calls that
// overlap on the GPU (two streams, two host threads) race on the array:
// serialise them.  The first call on each device looks up the array's device
// address (cudaGetSymbolAddress); make that first call before any stream capture.
#include <mutex>
#include "context.hpp"
#include "../../include/sincgpu.h"

namespace sincgpu {

int coulomb_dens_scratch(Ctx& c, const double2* dens, int m, double2* red, double2* scratch,
                         size_t scratch_bytes);  // coulomb.cu

namespace {

constexpr size_t kScratchBytes = 64ull << 20;  // 64 MiB
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_scratch on the current device.  In host code the symbol
// name is only a host-side stand-in, never a device address, so the address is
// looked up once per device with that device current.
int scratch_address(int device, void** out) {
  SG_CHECK(device >= 0 && device < kMaxDevices, SINCGPU_ERANGE, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    SG_CHECK(e == cudaSuccess && p, SINCGPU_ECUDA, "cudaGetSymbolAddress of the fixed scratch failed: %s",
             cudaGetErrorString(e));
    g_scratch_addr[device] = p;
  }
  *out = g_scratch_addr[device];
  return SINCGPU_OK;
}

}  // namespace
}  // namespace sincgpu

using namespace sincgpu;

extern "C" int sincgpu_op_tinv_noalloc_dev(sincgpu_ctx* h, const double* twoeden03, double* twoereduced,
                                           int allsize) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(twoeden03 && twoereduced, SINCGPU_EINVAL, "null argument");
  SG_CHECK(allsize >= 0, SINCGPU_EINVAL, "allsize %d < 0", allsize);
  if (allsize == 0) return SINCGPU_OK;
  void* scratch = nullptr;
  SG_TRY(scratch_address(c.device, &scratch));
  const bool prof = c.prof.on;  // the per-kernel timer creates events; keep it out of this path
  c.prof.on = false;
  int rc = coulomb_dens_scratch(c, (const double2*)twoeden03, allsize, (double2*)twoereduced,
                                (double2*)scratch, kScratchBytes);
  c.prof.on = prof;
  return rc;
}
