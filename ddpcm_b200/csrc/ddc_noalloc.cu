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
// The scratch array below is allocated once per GPU when the library is
// loaded and stays resident until the process exits.  Its device address is
// looked up with cudaGetSymbolAddress on the first call made for a device
// (with that device current); that first call therefore also does this
// one-time set-up.  All calls share the array: two calls whose kernels
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
  if (ntrg == 0) return DDC_OK;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return DDC_ERR_CUDA;
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return DDC_ERR_CUDA;
  double* scratch = nullptr;
  int rc = DDC_OK;
  if (scratch_for(device, &scratch) != cudaSuccess) {
    rc = DDC_ERR_CUDA;
  } else {
    // as many source chunks as the fixed scratch holds, up to what fills the GPU
    long long fit = kScratchDoubles / (3LL * ntrg);
    int nchunk = ddc::efield_chunks(nsrc, ntrg);
    if (nchunk > fit) nchunk = (int)fit;
    long long launches = 0;
    ddc::Launch L{static_cast<cudaStream_t>(stream), &launches};
    if (ddc::launch_efield(L, nsrc, src, csrc, ntrg, ctrg, ef, scratch, nchunk, nullptr) !=
        cudaSuccess)
      rc = DDC_ERR_CUDA;
  }
  if (prev != device) cudaSetDevice(prev);
  return rc;
}
