// Merkle root of device-resident leaves without allocating any memory.
//
// Who needs this: callers that are not allowed to allocate device memory at
// the point where they want a commitment root — for example a real-time or
// embedded host whose device memory is all reserved up front (an allocation
// there may fail or stall for an unbounded time), or a plugin that only
// receives buffers from an outer framework which owns every allocation and
// its accounting.  They already hold the leaves and a 32-byte output slot in
// device-accessible memory; everything else this entry point needs lives in
// the fixed array below.
//
// The intermediate tree (all 2n - 1 nodes) is kept in a file-scope device
// array sized for at most kMaxLeaves leaves.  Every GPU that loads the library
// holds this array until the process exits.  Host code cannot use the array's
// name as a device address, so the address is looked up once per device with
// cudaGetSymbolAddress while that device is current, and passed to the
// kernels.  The first call on each device does that lookup; make that first
// call before beginning any stream capture.  All calls share the one array and
// it keeps the previous call's contents: every node is written before it is
// read, so nothing needs clearing, but two calls whose work overlaps on the
// GPU (different streams, or different host threads on one device) race on the
// array and must be serialised by the caller.  The address is cached for the
// life of the process, so resetting a device (cudaDeviceReset) after its first
// call is not supported.  A CUDA error already pending on the calling thread
// is left in place for its owner and the call returns FLOCK_ERR_CUDA without
// doing any work.
#include "../../include/flock_gpu.h"
#include "kernels.cuh"
#include <mutex>

namespace {
constexpr size_t kMaxLeaves = size_t(1) << 15;               // 32768 leaves
constexpr size_t kMaxNodes = 2 * kMaxLeaves - 1;              // 2 MiB of nodes
static __device__ __align__(256) uint32_t g_tree_scratch[8 * kMaxNodes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_scratch_addr[kMaxDevices] = {};

// device address of g_tree_scratch on the current device (looked up once)
int scratch_for_current_device(uint32_t** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FLOCK_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_tree_scratch) != cudaSuccess || !p) return FLOCK_ERR_CUDA;
    g_scratch_addr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_scratch_addr[dev];
  return FLOCK_OK;
}
}  // namespace

extern "C" int flock_merkle_root_noalloc(const void* leaves, size_t n_leaves, size_t leaf_size, void* root_out,
                                         void* stream) {
  if (!leaves || !root_out || n_leaves == 0 || (n_leaves & (n_leaves - 1)) || leaf_size == 0 ||
      leaf_size > 1024 || (leaf_size % 16))
    return FLOCK_ERR_ARG;
  if (n_leaves > kMaxLeaves) return FLOCK_ERR_CAPACITY;  // the fixed array holds 2^15 leaves at most
  // an earlier, unrelated error stays pending for its owner: this call neither
  // clears it nor reports it as its own launch failure
  if (cudaPeekAtLastError() != cudaSuccess) return FLOCK_ERR_CUDA;
  uint32_t* tree = nullptr;
  int rc = scratch_for_current_device(&tree);
  if (rc) return rc;
  try {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    merkle_build(leaves, n_leaves, leaf_size, tree, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(root_out, tree + 8 * (2 * n_leaves - 2), 32, cudaMemcpyDeviceToDevice, s));
  } catch (const CudaError&) {
    return FLOCK_ERR_CUDA;
  }
  return FLOCK_OK;
}
