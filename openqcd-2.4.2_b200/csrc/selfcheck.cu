// Self-check of the bounded-wait path that the bulk-copy kernels rely on
// (b200_selfcheck_bounded_wait, no counterpart in the reference).
//
// One CTA arms an mbarrier that no copy and no thread will ever complete and
// waits on it with a caller-given iteration limit.  The wait gives up,
// records the error in the library's mapped error flag and the kernel
// returns; nothing is in flight, so the CUDA context stays usable.  The host
// then sees the flag exactly as it would after a real timed-out copy (the
// next b200_sync fails with the flag's message and clears it).
#include "lib.h"
#include "tma.cuh"
#include "../../include/openqcd_b200.h"

namespace qcd {

__global__ void k_wait_unarmed(int limit, int *err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_wait_st_lim(&bar, 0u, err, limit);
}

}  // namespace qcd

extern "C" int b200_selfcheck_bounded_wait(int limit) {
  qcd::Ctx &c = qcd::ctx();
  if (!c.ready || !c.d_kerr) return qcd::fail("selfcheck_bounded_wait: geometry not set (call b200_geometry first)");
  if (limit < 1 || limit > (1 << 22)) return qcd::fail("selfcheck_bounded_wait: limit must be in [1, 2^22]");
  if (b200_sync()) return -1;   // an older flag would be mistaken for this one
  qcd::k_wait_unarmed<<<1, 32, 0, c.stream>>>(limit, c.d_kerr);
  if (cudaGetLastError() != cudaSuccess) return qcd::fail("selfcheck_bounded_wait: launch failed");
  return b200_sync();
}
