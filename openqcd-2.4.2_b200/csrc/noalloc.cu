// Allocation-free variant of the FP64 even-odd preconditioned operator
// (b200_dev_Dwhat_dble_noalloc, declared in include/openqcd_b200.h).
//
// Dwhat needs an odd-site intermediate field between its two kernels.  The
// regular entry point (b200_dev_dirac, op 5) keeps it in a buffer obtained
// with cudaMalloc on first use.  Some callers cannot let a library allocate:
// applications whose own memory pool has already reserved the device (a
// framework's caching allocator, a fixed arena sized at start-up), where a
// further cudaMalloc fails or fragments that pool, and services that must
// keep the device footprint fixed after initialisation.  This variant keeps
// the intermediate in a file-scope device array instead; every GPU that
// loads the library holds it (12 MiB) until the process exits.  Like the
// other b200_dev_* operators it returns once the result is complete (it
// synchronises the library's stream).
#include <mutex>
#include "lib.h"
#include "../../include/openqcd_b200.h"
#include <string>

namespace qcd {

// Largest lattice served: the odd half of an FP64 spinor field of this many
// sites fills the array (65536 sites x 12 double2 = 12 MiB).
static const int NOALLOC_MAX_SITES = 131072;
static __device__ __align__(256) double2 g_dwhat_scratch[(NOALLOC_MAX_SITES / 2) * 12];

// In host code g_dwhat_scratch names a host-side shadow, not device memory:
// the device address is looked up once per device, with that device current
// (the library's device, c.dev, which may differ from the caller's current
// one), under a lock so that concurrent first calls resolve it once.
static const int MAX_DEVICES = 64;
static void *g_scratch_addr[MAX_DEVICES];
static std::mutex g_scratch_lock;

static int scratch_address(int dev, void **p) {
  if (dev < 0 || dev >= MAX_DEVICES) return fail("Dwhat_dble_noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_scratch_lock);
  if (!g_scratch_addr[dev]) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return fail("Dwhat_dble_noalloc: no usable CUDA device");
    if (cur != dev && cudaSetDevice(dev) != cudaSuccess) return fail("Dwhat_dble_noalloc: cannot select the device");
    void *a = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&a, g_dwhat_scratch);
    if (cur != dev) cudaSetDevice(cur);
    if (e != cudaSuccess || !a)
      return fail(std::string("Dwhat_dble_noalloc: cannot resolve the static scratch: ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = a;
  }
  *p = g_scratch_addr[dev];
  return 0;
}

}  // namespace qcd

extern "C" int b200_dev_Dwhat_dble_noalloc(double mu, const void *s, void *r) {
  qcd::Ctx &c = qcd::ctx();
  if (!c.ready) return qcd::fail("Dwhat_dble_noalloc: geometry not set (call b200_geometry first)");
  if (c.g.vol > qcd::NOALLOC_MAX_SITES)
    return qcd::fail("Dwhat_dble_noalloc: the lattice has " + std::to_string(c.g.vol) +
                     " sites, the static scratch serves at most " + std::to_string(qcd::NOALLOC_MAX_SITES));
  if (!c.have_ud || !c.have_sw) return qcd::fail("Dwhat_dble_noalloc: gauge or SW field missing on the device");
  if (qcd::dd_unsupported(c, "Dwhat_dble_noalloc")) return -1;
  void *scratch = nullptr;
  if (qcd::scratch_address(c.dev, &scratch)) return -1;
  // the first kernel writes every odd site the second one reads: nothing to clear
  if (qcd::dwhat_dble_halfscratch(c, mu, s, r, scratch, c.stream)) return qcd::fail("Dwhat_dble_noalloc: launch failed");
  return cudaStreamSynchronize(c.stream) == cudaSuccess ? 0 : qcd::fail("Dwhat_dble_noalloc: CUDA error");
}
