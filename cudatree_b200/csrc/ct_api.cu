// extern "C" entry points of libcudatree_b200.so (declared in
// include/cudatree_b200.h).  Each one validates its arguments on the host,
// launches on the caller's stream and returns a status code.
#include <cstring>
#include <string>
#include <vector>

#include "ct_internal.cuh"

namespace ct {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }
const std::string& last_error_text() { return g_last_error; }

size_t bootstrap_scratch_bytes(uint32_t n_rows, uint32_t n_features, uint32_t n_slots);
int bootstrap_compact(const ct_problem* p, const ct_lists* l, uint32_t slot, uint32_t tree,
                      uint32_t* n_in_dev, void* ws, size_t wsb, cudaStream_t st);
size_t fit_workspace_bytes(const ct_problem* p, uint32_t n_trees, const ct_fit_options* o);
size_t fit_queue_workspace_bytes(const ct_fit_job* jobs, uint32_t n_jobs, const ct_fit_options* o);
int fit_queue(const ct_fit_job* jobs, uint32_t n_jobs, const ct_fit_options* o, const ct_tree_buffers* trees,
              void* ws, size_t wsb, cudaStream_t st);
int fit(const ct_problem* p, const ct_lists* l, uint32_t first_tree, uint32_t n_trees,
        const ct_fit_options* o, const ct_tree_buffers* trees, void* ws, size_t wsb, cudaStream_t st);
int canonicalize(const uint32_t* left, const uint32_t* right, const uint32_t* feature, const float* threshold,
                 const uint32_t* value, uint32_t n, uint32_t* ol, uint32_t* orr, uint16_t* of, float* ot,
                 uint32_t* ov);
size_t autotune_workspace_bytes(const ct_problem* p, uint32_t n_trees, uint32_t mode);
int autotune(const ct_problem* p, const ct_lists* l, uint32_t n_trees, uint32_t mode, const ct_tree_buffers* trees,
             void* ws, size_t wsb, ct_fit_options* best, float* best_ms, cudaStream_t st);
size_t fetch_trees_scratch(uint64_t total_nodes, uint32_t n_trees);
int fetch_trees(const ct_tree_buffers* tb, uint32_t n_trees, const uint32_t* counts, void* scratch,
                size_t scratch_bytes, uint32_t* ol, uint32_t* orr, uint16_t* of, float* ot, uint32_t* ov,
                cudaStream_t st);
int predict(const void* nodes, uint32_t n_nodes, uint32_t fbits, const uint32_t* tree_off, uint32_t n_trees,
            const float* x, uint32_t n_rows, uint32_t n_features, uint32_t n_classes, uint32_t* votes,
            uint32_t* pred, cudaStream_t st);
uint32_t compact_feature_bits(uint32_t n_features);
bool compact_fits(uint32_t n_features, uint64_t max_tree_nodes);
int compact_forest(const ct_packed_node* nodes, uint32_t n_nodes, uint32_t n_features, uint32_t max_tree_nodes,
                   ct_compact_node* out, cudaStream_t st);
size_t presort_workspace_bytes(uint32_t n_rows, uint32_t n_features);
int presort(const float* x_fm, uint32_t n_rows, uint32_t n_features, uint32_t index_bytes, void* out, void* ws,
            size_t wsb, cudaStream_t st);

}  // namespace ct

using namespace ct;

extern "C" {

const char* ct_version(void) { return "cudatree_b200 0.1.0 (sm_100a)"; }

int ct_last_error(char* buf, size_t len) {
  const std::string& s = g_last_error;
  if (buf && len) {
    const size_t n = s.size() < len - 1 ? s.size() : len - 1;
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return (int)s.size();
}

int ct_mark_bytes(uint32_t n_rows, uint32_t n_slots, size_t* bytes) {
  CT_ARG_CHECK(bytes, "bytes is NULL");
  *bytes = mark_bits_offset(n_rows, n_slots) + (size_t)n_slots * mark_bit_words(n_rows) * sizeof(uint32_t) + 64;
  return CT_OK;
}

int ct_presort_workspace_size(uint32_t n_rows, uint32_t n_features, size_t* bytes) {
  CT_ARG_CHECK(bytes, "bytes is NULL");
  *bytes = presort_workspace_bytes(n_rows, n_features);
  return CT_OK;
}

int ct_presort(const float* x_fm, uint32_t n_rows, uint32_t n_features, uint32_t index_bytes, void* out,
               void* workspace, size_t workspace_bytes, void* stream) {
  CT_GUARD(return presort(x_fm, n_rows, n_features, index_bytes, out, workspace, workspace_bytes,
                          (cudaStream_t)stream);)
}

int ct_bootstrap_workspace_size(const ct_problem* p, size_t* bytes) {
  CT_ARG_CHECK(p && bytes, "NULL argument");
  *bytes = bootstrap_scratch_bytes(p->n_rows, p->n_features, 1);
  return CT_OK;
}

int ct_bootstrap_compact(const ct_problem* p, const ct_lists* lists, uint32_t slot, uint32_t tree,
                         uint32_t* n_in_dev, void* workspace, size_t workspace_bytes, void* stream) {
  CT_GUARD({
    CT_TRY(check_problem(p));
    CT_ARG_CHECK(lists && lists->si0 && lists->mark && n_in_dev, "NULL argument");
    if (p->bootstrap) CT_ARG_CHECK(workspace, "workspace is NULL");
    cudaStream_t st = (cudaStream_t)stream;
    if (workspace) CT_CUDA_TRY(cudaMemsetAsync(workspace, 0, 16, st));
    CT_TRY(bootstrap_compact(p, lists, slot, tree, n_in_dev, workspace, workspace_bytes, st));
    if (p->bootstrap) {
      uint32_t words[2];
      words[1] = 0;
      CT_CUDA_TRY(cudaMemcpyAsync(words, workspace, sizeof(words), cudaMemcpyDeviceToHost, st));
      CT_CUDA_TRY(cudaStreamSynchronize(st));
      if (words[1]) {
        set_last_error("bootstrap compaction flagged a device error");
        return CT_ERR_TIMEOUT;
      }
    }
    return CT_OK;
  })
}

int ct_split_workspace_size(const ct_problem* p, uint32_t n_nodes, uint64_t total_samples, size_t* bytes) {
  CT_ARG_CHECK(p && bytes, "NULL argument");
  View v = make_view(p, nullptr);
  *bytes = level_scratch_bytes(v, level_caps(v, DEFAULT_SCAN_PIECE, LevelBounds{n_nodes, total_samples}));
  return CT_OK;
}

static int carve_api_scratch(const ct_problem* p, const ct_lists* l, uint32_t n_nodes, uint64_t total,
                             void* ws, size_t wsb, View* v, LevelScratch* s) {
  *v = make_view(p, l);
  Arena a{reinterpret_cast<char*>(ws), wsb, 0};
  if (!carve_level_scratch(a, *v, level_caps(*v, DEFAULT_SCAN_PIECE, LevelBounds{n_nodes, total}), s)) {
    set_last_error("workspace too small");
    return CT_ERR_OOM;
  }
  return CT_OK;
}

static int node_total(const ct_node* nodes, uint32_t n_nodes, uint64_t* total, cudaStream_t st) {
  // total samples bound: read the node sizes (API path only; the fit keeps it on the host)
  std::vector<ct_node> h(n_nodes);
  CT_CUDA_TRY(cudaMemcpyAsync(h.data(), nodes, n_nodes * sizeof(ct_node), cudaMemcpyDeviceToHost, st));
  CT_CUDA_TRY(cudaStreamSynchronize(st));
  uint64_t t = 0;
  for (auto& n : h) t += n.n;
  *total = t;
  return CT_OK;
}

int ct_split_nodes(const ct_problem* p, const ct_lists* lists, const ct_node* nodes, const uint32_t* totals,
                   uint32_t n_nodes, ct_split_result* out, uint32_t* selected, void* workspace,
                   size_t workspace_bytes, void* stream) {
  CT_GUARD({
    CT_TRY(check_problem(p));
    CT_ARG_CHECK(lists && lists->si0 && lists->si1 && nodes && totals && out, "NULL argument");
    if (n_nodes == 0) return CT_OK;
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t total = 0;
    CT_TRY(node_total(nodes, n_nodes, &total, st));
    View v;
    LevelScratch s;
    CT_TRY(carve_api_scratch(p, lists, n_nodes, total, workspace, workspace_bytes, &v, &s));
    s.result = out;
    CT_CUDA_TRY(cudaMemsetAsync(s.ctr, 0, sizeof(Counters), st));
    CT_TRY(launch_reset_step(s, n_nodes, StepLists{nodes, totals, nullptr, nullptr, nullptr, nullptr, DEFAULT_SCAN_PIECE}, st));
    CT_TRY(launch_split(v, p->index_bytes, p->label_bytes, s, LevelBounds{n_nodes, total}, DEFAULT_SCAN_PIECE, false,
                        st));
    if (selected)
      CT_CUDA_TRY(cudaMemcpyAsync(selected, s.sel, (size_t)n_nodes * p->max_features * sizeof(uint32_t),
                                  cudaMemcpyDeviceToDevice, st));
    Counters h;
    CT_CUDA_TRY(cudaMemcpyAsync(&h, s.ctr, sizeof(h), cudaMemcpyDeviceToHost, st));
    CT_CUDA_TRY(cudaStreamSynchronize(st));
    if (h.error) {
      set_last_error("split scan: device capacity check failed");
      return CT_ERR_CAPACITY;
    }
    return CT_OK;
  })
}

int ct_partition_workspace_size(const ct_problem* p, uint32_t n_nodes, uint64_t total_samples, size_t* bytes) {
  return ct_split_workspace_size(p, n_nodes, total_samples, bytes);
}

int ct_partition_nodes(const ct_problem* p, const ct_lists* lists, const ct_node* nodes,
                       const ct_split_result* splits, uint32_t n_nodes, void* workspace, size_t workspace_bytes,
                       void* stream) {
  CT_GUARD({
    CT_TRY(check_problem(p));
    CT_ARG_CHECK(lists && lists->si0 && lists->si1 && lists->mark && nodes && splits, "NULL argument");
    if (n_nodes == 0) return CT_OK;
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t total = 0;
    CT_TRY(node_total(nodes, n_nodes, &total, st));
    View v;
    LevelScratch s;
    CT_TRY(carve_api_scratch(p, lists, n_nodes, total, workspace, workspace_bytes, &v, &s));
    s.result = const_cast<ct_split_result*>(splits);
    CT_CUDA_TRY(cudaMemsetAsync(s.ctr, 0, sizeof(Counters), st));
    CT_TRY(launch_reset_step(s, n_nodes, StepLists{nodes, nullptr, nullptr, nullptr, nullptr, nullptr, DEFAULT_SCAN_PIECE}, st));
    TreeView tv;
    std::memset(&tv, 0, sizeof(tv));
    CT_TRY(launch_partition(v, p->index_bytes, p->label_bytes, s, LevelBounds{n_nodes, total}, tv, false, st));
    Counters h;
    CT_CUDA_TRY(cudaMemcpyAsync(&h, s.ctr, sizeof(h), cudaMemcpyDeviceToHost, st));
    CT_CUDA_TRY(cudaStreamSynchronize(st));
    if (h.error & DEV_ERR_TIMEOUT) {
      set_last_error("partition look-back wait gave up");
      return CT_ERR_TIMEOUT;
    }
    if (h.error) {
      set_last_error("partition: device capacity check failed");
      return CT_ERR_CAPACITY;
    }
    return CT_OK;
  })
}

int ct_fit_workspace_size(const ct_problem* p, uint32_t n_trees, const ct_fit_options* opt, size_t* bytes) {
  CT_ARG_CHECK(p && opt && bytes, "NULL argument");
  *bytes = fit_workspace_bytes(p, n_trees, opt);
  return CT_OK;
}

int ct_fit(const ct_problem* p, const ct_lists* lists, uint32_t first_tree, uint32_t n_trees,
           const ct_fit_options* opt, const ct_tree_buffers* trees, void* workspace, size_t workspace_bytes,
           void* stream) {
  CT_GUARD(return fit(p, lists, first_tree, n_trees, opt, trees, workspace, workspace_bytes,
                      (cudaStream_t)stream);)
}

int ct_fit_queue_workspace_size(const ct_fit_job* jobs, uint32_t n_jobs, const ct_fit_options* opt,
                                size_t* bytes) {
  CT_ARG_CHECK(jobs && n_jobs >= 1 && opt && bytes, "NULL argument");
  CT_GUARD(*bytes = fit_queue_workspace_bytes(jobs, n_jobs, opt); return CT_OK;)
}

int ct_fit_queue(const ct_fit_job* jobs, uint32_t n_jobs, const ct_fit_options* opt, const ct_tree_buffers* trees,
                 void* workspace, size_t workspace_bytes, void* stream) {
  CT_GUARD(return fit_queue(jobs, n_jobs, opt, trees, workspace, workspace_bytes, (cudaStream_t)stream);)
}

int ct_fit_stats(ct_kernel_stats* out) {
  CT_ARG_CHECK(out, "NULL argument");
  *out = current_prof()->stats;
  return CT_OK;
}

int ct_tree_canonicalize(const uint32_t* left, const uint32_t* right, const uint32_t* feature,
                         const float* threshold, const uint32_t* value, uint32_t n_nodes, uint32_t* out_left,
                         uint32_t* out_right, uint16_t* out_feature, float* out_threshold, uint32_t* out_value) {
  CT_ARG_CHECK(left && right && feature && threshold && value && out_left && out_right && out_feature &&
                   out_threshold && out_value,
               "NULL argument");
  CT_GUARD(return canonicalize(left, right, feature, threshold, value, n_nodes, out_left, out_right, out_feature,
                               out_threshold, out_value);)
}


int ct_autotune_workspace_size(const ct_problem* p, uint32_t n_trees, uint32_t mode, size_t* bytes) {
  CT_ARG_CHECK(p && bytes && n_trees >= 1, "NULL argument");
  CT_TRY(check_problem(p));
  CT_GUARD(*bytes = autotune_workspace_bytes(p, n_trees, mode); return CT_OK;)
}

int ct_autotune(const ct_problem* p, const ct_lists* lists, uint32_t n_trees, uint32_t mode,
                const ct_tree_buffers* trees, void* workspace, size_t workspace_bytes, ct_fit_options* best,
                float* best_ms, void* stream) {
  CT_GUARD(return autotune(p, lists, n_trees, mode, trees, workspace, workspace_bytes, best, best_ms,
                           (cudaStream_t)stream);)
}

int ct_transpose_rows(const float* x_rm, uint32_t n_rows, uint32_t n_cols, float* x_cm, uint32_t* nan_flag,
                      void* stream) {
  CT_GUARD(return transpose_rows(x_rm, n_rows, n_cols, x_cm, (cudaStream_t)stream, nan_flag);)
}

size_t ct_fetch_trees_scratch(uint64_t total_nodes, uint32_t n_trees) {
  return fetch_trees_scratch(total_nodes, n_trees);
}

int ct_fetch_trees(const ct_tree_buffers* trees, uint32_t n_trees, const uint32_t* counts, void* scratch,
                   size_t scratch_bytes, uint32_t* out_left, uint32_t* out_right, uint16_t* out_feature,
                   float* out_threshold, uint32_t* out_value, void* stream) {
  CT_GUARD(return fetch_trees(trees, n_trees, counts, scratch, scratch_bytes, out_left, out_right, out_feature,
                              out_threshold, out_value, (cudaStream_t)stream);)
}

int ct_predict(const ct_packed_node* nodes, uint32_t n_nodes, const uint32_t* tree_offset, uint32_t n_trees,
               const float* x, uint32_t n_rows, uint32_t n_features, uint32_t n_classes, uint32_t* votes,
               uint32_t* pred, void* stream) {
  CT_GUARD(return predict(nodes, n_nodes, 0, tree_offset, n_trees, x, n_rows, n_features, n_classes, votes, pred,
                          (cudaStream_t)stream);)
}

int ct_compact_fits(uint32_t n_features, uint32_t max_tree_nodes) {
  return n_features >= 1 && compact_fits(n_features, max_tree_nodes) ? 1 : 0;
}

int ct_compact_forest(const ct_packed_node* nodes, uint32_t n_nodes, uint32_t n_features, uint32_t max_tree_nodes,
                      ct_compact_node* out, void* stream) {
  CT_GUARD(return compact_forest(nodes, n_nodes, n_features, max_tree_nodes, out, (cudaStream_t)stream);)
}

int ct_check_forest(const ct_packed_node* nodes, uint32_t n_nodes, const uint32_t* tree_offset, uint32_t n_trees,
                    uint32_t n_features, uint32_t n_classes) {
  CT_ARG_CHECK(nodes && tree_offset, "check forest: NULL argument");
  CT_ARG_CHECK(n_trees >= 1 && n_nodes >= n_trees, "check forest: empty forest");
  CT_ARG_CHECK(n_classes >= 1 && n_classes <= CT_MAX_CLASSES, "check forest: n_classes out of range");
  CT_GUARD(return check_forest_host(nodes, n_nodes, tree_offset, n_trees, n_features, n_classes);)
}

int ct_predict_compact(const ct_compact_node* nodes, uint32_t n_nodes, const uint32_t* tree_offset,
                       uint32_t n_trees, const float* x, uint32_t n_rows, uint32_t n_features, uint32_t n_classes,
                       uint32_t* votes, uint32_t* pred, void* stream) {
  CT_GUARD(return predict(nodes, n_nodes, compact_feature_bits(n_features), tree_offset, n_trees, x, n_rows,
                          n_features, n_classes, votes, pred, (cudaStream_t)stream);)
}

}  // extern "C"
