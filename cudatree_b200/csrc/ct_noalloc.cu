// ct_split_nodes_noalloc: the split search of ct_split_nodes for callers
// that cannot allocate device memory.
//
// Some callers have no way to hand the library a workspace: a process whose
// device memory is already claimed by another allocator's pool (so a fresh
// cudaMalloc fails), a serving loop that must not pay for cudaMalloc /
// cudaFree (they can synchronize the device and stall other streams), or a
// host that binds the library through a bare C FFI and owns no device
// buffers of its own.  This entry point needs only the inputs and the output
// array: its scratch is one file-scope __device__ array of
// NOALLOC_SCRATCH_BYTES, which every GPU that loads the library holds until
// the process exits.
//
// The array's name is not a device address on the host, so each call looks
// the device address up with cudaGetSymbolAddress, with the caller's device
// current, and passes it to the kernels.  The lookup allocates nothing and
// issues no stream work; because it is repeated every call, a device reset
// between calls leaves no stale address behind.  The first call on a device
// may load the library's device code (lazy module loading), so that first
// call should come before any stream capture.  All calls share the array and
// it keeps the previous call's contents: the work-list counters are zeroed at
// the start of every call, and every other scratch word is written before it
// is read.  Calls that overlap on the GPU (different streams or threads, same
// device) race on the array and must be serialized by the caller.
#include "ct_internal.cuh"

namespace ct {

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(16) << 20;  // 16 MiB per device

__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch on the current device.
int noalloc_scratch(void** out) {
  void* p = nullptr;
  CT_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  *out = p;
  return CT_OK;
}

}  // namespace

}  // namespace ct

using namespace ct;

extern "C" int ct_split_nodes_noalloc(const ct_problem* p, const ct_lists* lists, const ct_node* nodes,
                                      const uint32_t* totals, uint32_t n_nodes, uint64_t total_samples,
                                      ct_split_result* out, void* stream) {
  CT_GUARD({
    CT_TRY(check_problem(p));
    CT_ARG_CHECK(lists && lists->si0 && lists->si1 && nodes && totals && out, "NULL argument");
    if (n_nodes == 0) return CT_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const View v = make_view(p, lists);
    const LevelBounds b{n_nodes, total_samples};
    const LevelCaps caps = level_caps(v, DEFAULT_SCAN_PIECE, b);
    const size_t need = level_scratch_bytes(v, caps);
    if (need > NOALLOC_SCRATCH_BYTES) {
      set_last_error("ct_split_nodes_noalloc: these nodes need " + std::to_string(need) +
                     " bytes of scratch but the static scratch holds " + std::to_string(NOALLOC_SCRATCH_BYTES) +
                     "; split the batch or use ct_split_nodes with a workspace");
      return CT_ERR_ARG;
    }
    void* base = nullptr;
    CT_TRY(noalloc_scratch(&base));
    Arena a{reinterpret_cast<char*>(base), NOALLOC_SCRATCH_BYTES, 0};
    LevelScratch s;
    if (!carve_level_scratch(a, v, caps, &s)) {
      set_last_error("ct_split_nodes_noalloc: static scratch too small");
      return CT_ERR_ARG;
    }
    s.result = out;
    CT_CUDA_TRY(cudaMemsetAsync(s.ctr, 0, sizeof(Counters), st));
    CT_TRY(launch_reset_step(s, n_nodes, StepLists{nodes, totals, nullptr, nullptr, nullptr, nullptr, DEFAULT_SCAN_PIECE}, st));
    CT_TRY(launch_split(v, p->index_bytes, p->label_bytes, s, b, DEFAULT_SCAN_PIECE, false, st));
    Counters h;
    CT_CUDA_TRY(cudaMemcpyAsync(&h, s.ctr, sizeof(h), cudaMemcpyDeviceToHost, st));
    CT_CUDA_TRY(cudaStreamSynchronize(st));
    if (h.error) {
      set_last_error("ct_split_nodes_noalloc: work lists overflowed (total_samples smaller than the nodes' sizes?)");
      return CT_ERR_CAPACITY;
    }
    return CT_OK;
  })
}
