// ddc_noalloc.cu -- efld for callers that cannot allocate device memory.
//
// Some host programs own all of the GPU's memory: a QM/MM or molecular
// dynamics code that reserves the HBM for its own pool at start-up and
// accounts for every byte, so that a cudaMalloc issued by a library in the
// middle of a time step either fails or stalls the whole device while it
// synchronises.  ddc_efld_noalloc gives such callers the electric field of
// efld.f90 with no allocation at all: the caller passes device buffers for
// the inputs and the output, and the per-chunk partial sums of the field
// kernel live in a fixed array compiled into this library.
//
// The scratch array below is part of this library's device code.  CUDA loads
// a library's device code lazily by default, so the array (with the field
// kernels that use it) is put on a GPU by the first call made for that
// device, and stays there until the process exits.  That first call also
// looks up the array's device address with cudaGetSymbolAddress (with the
// device current).  A caller whose memory pool will take the whole GPU
// therefore makes one call with ntrg = 0 at start-up, before the pool claims
// the memory and outside any stream capture: it does this one-time set-up
// and nothing else.  All calls share the array: two calls whose kernels
// overlap on the GPU (different streams, or different host threads on the
// same device) race on it, so callers must order them.  Nothing in the
// array has to start at zero: every partial that the reduction reads is
// written by the same call first.
#include <mutex>

#include "ddc_internal.h"

namespace {

// 1 Mi doubles = 8 MiB: up to 349,525 targets with one source chunk, more
// chunks (better parallelism) for fewer targets.
constexpr long long kScratchDoubles = 1LL << 20;
__device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array for `device` (made current by the
// caller); resolved once per device.
cudaError_t scratch_for(int device, double** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

}  // namespace

extern "C" int ddc_efld_noalloc(int device, int nsrc, const double* src, const double* csrc,
                                int ntrg, const double* ctrg, double* ef, void* stream) {
  if (device < 0 || device >= kMaxDevices || nsrc < 0 || ntrg < 0) return DDC_ERR_PARAM;
  if (ntrg > 0 && (!ctrg || !ef)) return DDC_ERR_PARAM;
  if (nsrc > 0 && (!src || !csrc)) return DDC_ERR_PARAM;
  if (3LL * ntrg > kScratchDoubles) return DDC_ERR_CAPACITY;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return DDC_ERR_CUDA;
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return DDC_ERR_CUDA;
  double* scratch = nullptr;
  int rc = DDC_OK;
  // one-time set-up first, so that a call with ntrg = 0 does it: the scratch
  // address and the field kernels' code on this device
  if (scratch_for(device, &scratch) != cudaSuccess || ddc::preload_efield() != cudaSuccess) {
    rc = DDC_ERR_CUDA;
  } else {
    // a stream of another device would make the launch fail and leave a
    // sticky error behind; reject it up front
    int sdev = -1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) {
      cudaGetLastError();
      rc = DDC_ERR_PARAM;
    } else if (sdev != device) {
      rc = DDC_ERR_PARAM;
    } else if (ntrg > 0) {
      // as many source chunks as the fixed scratch holds, up to what fills the GPU
      long long fit = kScratchDoubles / (3LL * ntrg);
      int nchunk = ddc::efield_chunks(nsrc, ntrg);
      if (nchunk > fit) nchunk = (int)fit;
      long long launches = 0;
      ddc::Launch L{st, &launches};
      if (ddc::launch_efield(L, nsrc, src, csrc, ntrg, ctrg, ef, scratch, nchunk, nullptr) !=
          cudaSuccess)
        rc = DDC_ERR_CUDA;
    }
  }
  if (prev != device) cudaSetDevice(prev);
  return rc;
}
