// Allocation-free variant of the batched mesh signed-distance query.
//
// Who needs it: callers that cannot let a library allocate device memory.  The reference's main
// callers are adaptive-mesh codes (AMReX, Chombo) that evaluate value(point) while they build their
// embedded boundaries; AMReX reserves most of the GPU's memory for its own arena when it starts, so
// a cudaMalloc (or a stream-ordered allocation) issued by a library it calls can fail for lack of
// memory, and codes with their own memory managers or hard latency budgets forbid allocations in
// the query loop altogether.  ebg_mesh_signed_distance takes its per-call workspace (sort keys,
// the point order, the near-surface flags and list, counters) from the device's memory pool; this
// entry point takes it from one array of fixed size compiled into the library instead.
//
// The scratch array below is a file-scope __device__ variable.  In host code the name
// g_noallocScratch is only a stand-in for the device variable, not a device address; the address a
// kernel may use is obtained once per device with cudaGetSymbolAddress (with that device current)
// and cached.  With lazy module loading (the CUDA default since 12.2) the array is only created on
// a device when that lookup first loads this module, so the first call on a device -- a call with
// n = 0 is enough -- should come before the caller reserves its memory arena, and before any stream
// capture on that device.  The array then stays on that device until the process exits.
// cudaDeviceReset destroys it; the cached address is then stale, so a process that resets a device
// must not call this entry point on it again.
//
// All calls on a device share the one array and it keeps the contents of the last call: the
// counters are cleared at the start of every call, and two calls whose work overlaps on the GPU
// (different streams, or different threads without ordering) race on it and must be serialised by
// the caller.  The call itself allocates nothing: no cudaMalloc, cudaMallocAsync, cudaFree or
// allocating library routine (the radix sort and the band-list compaction are given their
// temporary storage from the same array).
#include <cstdint>
#include <mutex>
#include <string>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <cuda_runtime.h>
#include <thrust/iterator/counting_iterator.h>

#include "capi_common.h"
#include "capi_internal.h"
#include "ebg_device.cuh"
#include "mesh_kernels.h"
#include "seed_kernels.h"

// Largest point count one allocation-free call accepts, and the scratch that covers it: five
// uint32 arrays (the Morton ordering and the near-surface list), one flag byte per point, two
// counters, and the temporary storage of the radix sort and of the compaction (under 5 MiB together
// at this size on sm_100a; checked at every call).
#define EBG_NOALLOC_MAX_POINTS (int64_t(1) << 19)
#define EBG_NOALLOC_SCRATCH_BYTES (size_t(24) << 20)

static __device__ __align__(256) unsigned char g_noallocScratch[EBG_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex    g_mutex;
void*         g_scratch[kMaxDevices] = {nullptr};

// Device address of the scratch array on `device` (the current device), looked up once.
ebg_status scratchAddress(int device, unsigned char** out)
{
  if (device < 0 || device >= kMaxDevices) {
    return ebg::setError(EBG_ERR_NOT_FOUND, "device ordinal out of range for the allocation-free entry point");
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (g_scratch[device] == nullptr) {
    void*             p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return ebg::setError(EBG_ERR_CUDA, std::string("cannot resolve the scratch array's device address: ") +
                                            cudaGetErrorString(e));
    }
    g_scratch[device] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch[device]);
  return EBG_OK;
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

ebg_status cudaFailed(const char* what)
{
  return ebg::setError(EBG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(cudaGetLastError()));
}

} // namespace

extern "C" {

ebg_status ebg_mesh_signed_distance_noalloc(const ebg_mesh*       m,
                                            const float*          points_dev,
                                            int64_t               n,
                                            float*                dist_dev,
                                            int32_t*              closest_tri_dev,
                                            const ebg_query_opts* opts,
                                            void*                 stream)
{
  using namespace ebg;
  if (m == nullptr || n < 0 || (n > 0 && (points_dev == nullptr || dist_dev == nullptr))) {
    return setError(EBG_ERR_INVALID, "null mesh/buffer or negative count");
  }
  if (n > EBG_NOALLOC_MAX_POINTS) {
    return setError(EBG_ERR_TOO_LARGE, "ebg_mesh_signed_distance_noalloc accepts at most " +
                                         std::to_string(EBG_NOALLOC_MAX_POINTS) + " points per call (got " +
                                         std::to_string(n) + "); split the batch or use ebg_mesh_signed_distance");
  }
  const ebg_seed* seed = opts ? opts->seed : nullptr;
  if (seed && seed->device != m->device) {
    return setError(EBG_ERR_INVALID, "seed model lives on another device than the mesh");
  }
  if (seed && !(m->cellsSeed == seed && m->dCellCount != nullptr)) {
    return setError(EBG_ERR_INVALID, "the seed model is not attached to this mesh (ebg_seed_attach)");
  }
  DeviceGuard guard;
  if (cudaSetDevice(m->device) != cudaSuccess) {
    return setError(EBG_ERR_NOT_FOUND, "cannot select the mesh's device");
  }
  // set-up first, so that an empty call prepares the array on this device
  unsigned char* base = nullptr;
  ebg_status     rc   = scratchAddress(m->device, &base);
  if (rc != EBG_OK || n == 0) {
    return rc;
  }
  cudaStream_t s        = static_cast<cudaStream_t>(stream);
  const bool   sort     = !(opts && opts->no_sort);
  const bool   b64      = !(opts && opts->no_fp64_band);
  const int    wpb      = (opts && opts->warps_per_block > 0) ? opts->warps_per_block
                                                              : (m->tunedWpb > 0 ? m->tunedWpb : 4);
  const int    occ      = (opts && opts->occupancy > 0) ? opts->occupancy : m->tunedOccupancy;
  const double band     = (opts && opts->band > 0) ? opts->band : 1e-4 * fp32ErrorScale(m);

  // carve the scratch
  const size_t u32n = align256(size_t(n) * sizeof(uint32_t));
  size_t       off  = 0;
  auto         take = [&](size_t bytes) {
    unsigned char* p = base + off;
    off += align256(bytes);
    return p;
  };
  auto* counters = reinterpret_cast<unsigned long long*>(take(2 * sizeof(unsigned long long)));
  auto* keysIn   = reinterpret_cast<uint32_t*>(take(u32n));
  auto* keysOut  = reinterpret_cast<uint32_t*>(take(u32n));
  auto* idsIn    = reinterpret_cast<uint32_t*>(take(u32n));
  auto* order    = reinterpret_cast<uint32_t*>(take(u32n));
  auto* bandList = reinterpret_cast<uint32_t*>(take(u32n));
  auto* bandFlag = reinterpret_cast<uint8_t*>(take(size_t(n)));
  auto* bandCnt  = reinterpret_cast<uint32_t*>(counters + 1);
  size_t sortBytes = 0, selBytes = 0;
  if (sort) {
    cub::DeviceRadixSort::SortPairs(nullptr, sortBytes, keysIn, keysOut, idsIn, order, int(n), 0, 30, s);
  }
  if (b64) {
    cub::DeviceSelect::Flagged(nullptr, selBytes, thrust::counting_iterator<uint32_t>(0u), bandFlag, bandList, bandCnt,
                               int(n), s);
  }
  void* sortTemp = take(sortBytes);
  void* selTemp  = take(selBytes);
  if (off > EBG_NOALLOC_SCRATCH_BYTES) {
    return setError(EBG_ERR_TOO_LARGE, "allocation-free scratch too small for this call (" + std::to_string(off) +
                                         " of " + std::to_string(size_t(EBG_NOALLOC_SCRATCH_BYTES)) + " bytes)");
  }

  // the array keeps the previous call's contents: clear what must start at zero (a stale packet
  // counter would make the traversal skip every packet)
  if (cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), s) != cudaSuccess) {
    return cudaFailed("clearing the allocation-free counters");
  }
  if (sort) {
    launchQueryKeys(points_dev, n, m->view.morton_lo, m->view.morton_scale, keysIn, idsIn, s);
    if (cudaGetLastError() != cudaSuccess) {
      return setError(EBG_ERR_CUDA, "query key launch failed");
    }
    if (cub::DeviceRadixSort::SortPairs(sortTemp, sortBytes, keysIn, keysOut, idsIn, order, int(n), 0, 30, s) !=
        cudaSuccess) {
      return cudaFailed("query sort");
    }
  }
  MeshQueryArgs a{};
  a.mesh       = m->view;
  a.points     = points_dev;
  a.order      = sort ? order : nullptr;
  a.hint       = (seed == nullptr && opts) ? opts->radius_hint : nullptr;
  a.n          = n;
  a.out_d      = dist_dev;
  a.out_tri    = closest_tri_dev;
  a.band       = float(band);
  a.band_list  = b64 ? bandList : nullptr;
  a.band_count = bandCnt;
  a.band_d32   = nullptr;
  a.band_flag  = b64 ? bandFlag : nullptr;
  a.work       = counters;
  a.status     = m->dStatus;
  a.stats      = nullptr;
  a.chunk      = (opts && opts->queue_chunk > 0) ? opts->queue_chunk : (m->tunedChunk > 0 ? m->tunedChunk : 1);
  if (seed) {
    a.cells = m->cellsView; // the attached model's entry cuts live with the mesh
  }
  a.top_nodes = topNodesFor(m, opts, seed != nullptr);
  if (launchMeshSdf32(a, wpb, m->numSms, s, occ) != cudaSuccess) {
    return cudaFailed("traversal launch");
  }
  if (b64) {
    // the band list in position (Morton) order, as the allocating entry point builds it
    if (cub::DeviceSelect::Flagged(selTemp, selBytes, thrust::counting_iterator<uint32_t>(0u), bandFlag, bandList,
                                   bandCnt, int(n), s) != cudaSuccess) {
      return cudaFailed("band list compaction");
    }
    if (launchMeshBand64(a, float(2e-6 * fp32ErrorScale(m)) + 1e-30f, m->numSms, s) != cudaSuccess) {
      return cudaFailed("band launch");
    }
  }
  return EBG_OK;
}

} // extern "C"
