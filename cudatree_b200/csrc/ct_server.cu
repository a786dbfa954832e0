// Serving engine: resident forests, continuous batching of predict
// requests, small fit jobs, admission by an HBM budget, latency percentiles.
//
// The reference has no serving path (its predict re-uploads X and every tree
// per call, base_tree.py:57-62).  Here:
//   * forests stay resident on the device as breadth-first nodes, in the
//     8-byte compact form whenever the trees fit it;
//   * two predict lanes, each a worker thread with its own CUDA stream: small
//     requests (<= small_rows rows) on a high-priority stream, larger ones on
//     a low-priority stream, so a 65k-row request does not hold back 1-row
//     requests;
//   * small requests whose host buffers are page-locked and mapped are
//     zero-copy: the kernel stages their rows from host memory and writes the
//     predictions back, so they never wait behind bulk copies in the copy
//     engines (a 100 MB request copy takes ~2 ms);
//   * a lane takes every request that has arrived (up to its staging
//     capacity) into one multi-request predict launch; with two staging
//     slots a lane launches the next batch while the previous one runs, and
//     requests that arrive meanwhile join the next batch (continuous
//     batching);
//   * fit jobs (host arrays in, a new resident forest out) run on fit-worker
//     threads with their own low-priority streams and device arenas, so
//     their kernels overlap the predict batches;
//   * every device allocation is made at creation, against the byte budget:
//     forests are carved from a pool reserved there (a device allocation
//     issued while requests run would serialize all streams), and a request
//     or forest that does not fit is rejected with CT_ERR_OOM;
//   * a removed forest's pool bytes return once the batches launched on it
//     have completed (per-forest reference counts).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "ct_internal.cuh"

namespace ct {

size_t fit_workspace_bytes(const ct_problem* p, uint32_t n_trees, const ct_fit_options* o);
int fit(const ct_problem* p, const ct_lists* l, uint32_t first_tree, uint32_t n_trees, const ct_fit_options* o,
        const ct_tree_buffers* trees, void* ws, size_t wsb, cudaStream_t st);
size_t fetch_trees_scratch(uint64_t total_nodes, uint32_t n_trees);
int fetch_trees_reserve(uint64_t total_nodes);
int fetch_trees(const ct_tree_buffers* tb, uint32_t n_trees, const uint32_t* counts, void* scratch,
                size_t scratch_bytes, uint32_t* ol, uint32_t* orr, uint16_t* of, float* ot, uint32_t* ov,
                cudaStream_t st);
size_t presort_workspace_bytes(uint32_t n_rows, uint32_t n_features);
int presort(const float* x_fm, uint32_t n_rows, uint32_t n_features, uint32_t index_bytes, void* out, void* ws,
            size_t wsb, cudaStream_t st);

namespace {


// Page-locked host memory mapped at the same address on the device.
bool device_addressable(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost && a.devicePointer == p;
}

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Forest {
  std::shared_ptr<std::vector<ct_packed_node>> host;  // exact packed copy (read-back)
  std::shared_ptr<std::vector<uint32_t>> host_off;
  void* nodes = nullptr;  // compact nodes when fbits != 0, else packed
  uint32_t fbits = 0;
  uint32_t* off = nullptr;
  uint32_t n_nodes = 0, n_trees = 0, n_features = 0, n_classes = 0;
  uint32_t group = 0;  // trees per L2-sized group
  size_t bytes = 0;     // pool bytes
  size_t pool_off = 0;
  uint32_t refs = 0;    // launched batches not yet completed
  bool removed = false;
};

// First-fit allocator over one device region, 256-byte granules, coalescing.
class Pool {
 public:
  static constexpr size_t NO_ROOM = ~size_t(0);
  void reset(size_t bytes) {
    total_ = bytes;
    used_ = 0;
    free_.clear();
    if (bytes) free_[0] = bytes;
  }
  size_t alloc(size_t bytes) {
    bytes = round(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      const size_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > bytes) free_[off + bytes] = len - bytes;
      used_ += bytes;
      return off;
    }
    return NO_ROOM;
  }
  void release(size_t off, size_t bytes) {
    bytes = round(bytes);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  static size_t round(size_t b) { return (b + 255) & ~size_t(255); }
  size_t used() const { return used_; }
  size_t total() const { return total_; }

 private:
  std::map<size_t, size_t> free_;
  size_t total_ = 0, used_ = 0;
};

struct Job {
  ct_request* req = nullptr;
  double t_start = 0;
  bool done = false;
};

struct Slot {
  float* x_dev = nullptr;
  uint32_t* pred_dev = nullptr;
  uint32_t* votes_dev = nullptr;  // [rows][classes] tables of grouped requests
  BatchReq* req_dev = nullptr;
  BatchReq* req_host = nullptr;  // pinned
  cudaEvent_t ev = nullptr;
  std::vector<Job*> jobs;
  std::vector<uint8_t> direct;  // per job: rows and predictions in host memory, no copies
  double launched = 0;
};

struct Lane {
  cudaStream_t st = nullptr;
  std::deque<Job*> q;
  Slot slot[2];
  std::thread th;
  uint64_t cap_rows = 0, cap_floats = 0;
};

struct FitWorker {
  cudaStream_t st = nullptr;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  std::thread th;
};

}  // namespace

class Server {
 public:
  ct_server_config cfg{};
  int device = 0;
  size_t budget = 0, used = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::vector<Forest> forests;
  char* pool_base = nullptr;
  Pool pool;
  cudaStream_t upload_st = nullptr;
  Lane lanes[2];
  std::deque<Job*> fit_q;
  std::vector<FitWorker> fit_workers;
  // statistics
  std::vector<double> lat_small, lat_large, lat_fit;
  uint64_t n_req = 0, n_rows = 0, n_batches = 0, n_fit = 0, n_rejected = 0, n_zero_copy = 0;
  double t_first = 0, t_last = 0;
  std::string error;

  ~Server() { shutdown(); }

  int take(size_t bytes, void** out) {
    if (used + bytes > budget) {
      set_last_error("server: HBM budget exhausted (" + std::to_string(used + bytes) + " > " +
                     std::to_string(budget) + " bytes)");
      return CT_ERR_OOM;
    }
    CT_CUDA_TRY(cudaMalloc(out, bytes));
    used += bytes;
    return CT_OK;
  }

  int init(const ct_server_config* c) {
    cfg = *c;
    if (!cfg.max_batch_rows) cfg.max_batch_rows = 131072;
    if (!cfg.max_features) cfg.max_features = 512;
    if (!cfg.small_rows) cfg.small_rows = 4096;
    if (!cfg.max_fit_rows) cfg.max_fit_rows = 20000;
    if (!cfg.max_fit_trees) cfg.max_fit_trees = 10;
    if (!cfg.max_classes) cfg.max_classes = 64;
    CT_CUDA_TRY(cudaGetDevice(&device));
    size_t free_b = 0, total_b = 0;
    CT_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    budget = cfg.hbm_budget_bytes ? cfg.hbm_budget_bytes : (size_t)(free_b * 0.8);
    int prio_lo = 0, prio_hi = 0;
    CT_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    for (int l = 0; l < 2; ++l) {
      Lane& ln = lanes[l];
      CT_CUDA_TRY(cudaStreamCreateWithPriority(&ln.st, cudaStreamNonBlocking, l == 0 ? prio_hi : prio_lo));
      ln.cap_rows = l == 0 ? std::max<uint64_t>(cfg.small_rows * 8ull, 32768) : cfg.max_batch_rows;
      ln.cap_floats = ln.cap_rows * cfg.max_features;
      for (auto& s : ln.slot) {
        CT_TRY(take(ln.cap_floats * sizeof(float), (void**)&s.x_dev));
        CT_TRY(take(ln.cap_rows * sizeof(uint32_t), (void**)&s.pred_dev));
        CT_TRY(take(ln.cap_rows * cfg.max_classes * sizeof(uint32_t), (void**)&s.votes_dev));
        CT_TRY(take(4096 * sizeof(BatchReq), (void**)&s.req_dev));
        CT_CUDA_TRY(cudaMallocHost((void**)&s.req_host, 4096 * sizeof(BatchReq)));
        CT_CUDA_TRY(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
      }
    }
    const uint32_t nfw = cfg.fit_workers;
    fit_workers.resize(nfw);
    // page-locked read-back staging for the largest fit job, taken now: a
    // page-locked allocation while requests run would stall every stream
    if (nfw) CT_TRY(fetch_trees_reserve((uint64_t)cfg.max_fit_trees * 2 * cfg.max_fit_rows));
    const size_t arena = fit_arena_bytes();
    for (auto& fw : fit_workers) {
      CT_CUDA_TRY(cudaStreamCreateWithPriority(&fw.st, cudaStreamNonBlocking, prio_lo));
      CT_TRY(take(arena, (void**)&fw.arena));
      fw.arena_bytes = arena;
    }
    size_t pool_bytes = cfg.forest_pool_bytes ? cfg.forest_pool_bytes : std::min<size_t>(4ull << 30, budget / 4);
    pool_bytes = Pool::round(pool_bytes);
    CT_TRY(take(pool_bytes, (void**)&pool_base));
    pool.reset(pool_bytes);
    CT_CUDA_TRY(cudaStreamCreateWithFlags(&upload_st, cudaStreamNonBlocking));
    for (int l = 0; l < 2; ++l) lanes[l].th = std::thread([this, l] { lane_loop(l); });
    for (auto& fw : fit_workers) fw.th = std::thread([this, &fw] { fit_loop(fw); });
    return CT_OK;
  }

  // Device bytes of one fit job at the configured maximum size.
  size_t fit_arena_bytes() const { return job_bytes(cfg.max_fit_rows, cfg.max_features, 255, cfg.max_fit_trees); }

  static size_t job_bytes(uint32_t n, uint32_t f, uint32_t c, uint32_t t) {
    ct_problem p{};
    p.n_rows = n;
    p.n_features = f;
    p.n_classes = c;
    p.index_bytes = n <= 0xFFFF ? 2 : 4;
    p.label_bytes = c <= 255 ? 1 : 2;
    p.max_features = 1;
    p.min_samples_split = 1;
    ct_fit_options o{};
    o.mode = CT_FIT_BATCHED;
    o.subtree_cutoff = 32;
    o.flags = CT_FIT_HOST_LOOP;  // as the job fit below
    const size_t ib = p.index_bytes, nf = (size_t)n * f;
    size_t mb = 0;
    mb = (((size_t)t * n + 255) & ~size_t(255)) + (size_t)t * mark_bit_words(n) * 4 + 64;
    size_t b = 0;
    auto add = [&](size_t x) { b += (x + 511) & ~size_t(511); };
    add(nf * 4);                       // x row-major
    add(nf * 4);                       // x feature-major
    add((size_t)n * 2);                // labels
    add(nf * ib + 64);                 // presort
    add(presort_workspace_bytes(n, f));
    add((size_t)t * nf * ib + 64);     // si0
    add((size_t)t * nf * ib + 64);     // si1
    add(mb);                           // marks
    add((size_t)t * 2 * n * 4 * 5);    // raw trees
    add((size_t)t * 4);                // node counts
    add(fetch_trees_scratch((uint64_t)t * 2 * n, t));  // tree read-back
    add(fit_workspace_bytes(&p, t, &o));
    return b + 4096;
  }

  void shutdown() {
    {
      std::lock_guard<std::mutex> lk(mu);
      if (stop) return;
      stop = true;
    }
    cv_work.notify_all();
    for (auto& ln : lanes)
      if (ln.th.joinable()) ln.th.join();
    for (auto& fw : fit_workers)
      if (fw.th.joinable()) fw.th.join();
    cudaSetDevice(device);
    for (auto& ln : lanes) {
      for (auto& s : ln.slot) {
        if (s.x_dev) cudaFree(s.x_dev);
        if (s.pred_dev) cudaFree(s.pred_dev);
        if (s.votes_dev) cudaFree(s.votes_dev);
        if (s.req_dev) cudaFree(s.req_dev);
        if (s.req_host) cudaFreeHost(s.req_host);
        if (s.ev) cudaEventDestroy(s.ev);
      }
      if (ln.st) cudaStreamDestroy(ln.st);
    }
    for (auto& fw : fit_workers) {
      if (fw.arena) cudaFree(fw.arena);
      if (fw.st) cudaStreamDestroy(fw.st);
    }
    if (pool_base) cudaFree(pool_base);
    if (upload_st) cudaStreamDestroy(upload_st);
  }

  // Pool bytes are taken under the lock; the upload runs outside it (on the
  // caller's stream), so the predict lanes are never held up by a forest
  // being added.
  int add_forest(const ct_packed_node* nodes, uint32_t n_nodes, const uint32_t* off, uint32_t n_trees,
                 uint32_t n_features, uint32_t n_classes, uint32_t* id, cudaStream_t st = nullptr) {
    CT_ARG_CHECK(nodes && off && id && n_nodes && n_trees, "server: empty forest");
    CT_ARG_CHECK(n_features <= cfg.max_features, "server: forest has more features than max_features");
    CT_ARG_CHECK(n_classes >= 1 && n_classes <= CT_MAX_CLASSES, "server: n_classes out of range");
    CT_TRY(check_forest_host(nodes, n_nodes, off, n_trees, n_features, n_classes));
    if (!st) st = upload_st;
    Forest f;
    f.n_nodes = n_nodes;
    f.n_trees = n_trees;
    f.n_features = n_features;
    f.n_classes = n_classes;
    uint32_t max_tree = 0;
    for (uint32_t t = 0; t < n_trees; ++t) {
      const uint32_t end = t + 1 < n_trees ? off[t + 1] : n_nodes;
      CT_ARG_CHECK(off[t] < end && end <= n_nodes, "server: tree offsets out of order");
      max_tree = std::max(max_tree, end - off[t]);
    }
    std::vector<ct_compact_node> compact;
    const void* src = nodes;
    size_t elem = sizeof(ct_packed_node);
    if (compact_fits(n_features, max_tree)) {
      f.fbits = compact_feature_bits(n_features);
      compact.resize(n_nodes);
      compact_host(nodes, n_nodes, f.fbits, compact.data());
      src = compact.data();
      elem = sizeof(ct_compact_node);
    }
    const size_t node_bytes = Pool::round((size_t)n_nodes * elem), off_bytes = (size_t)n_trees * 4;
    f.bytes = Pool::round(node_bytes + off_bytes);
    f.group = n_classes <= cfg.max_classes ? predict_group_size(n_trees, n_nodes, elem) : n_trees;
    {
      std::lock_guard<std::mutex> lk(mu);
      f.pool_off = pool.alloc(f.bytes);
      if (f.pool_off == Pool::NO_ROOM) {
        set_last_error("server: forest pool full (" + std::to_string(pool.used()) + " of " +
                       std::to_string(pool.total()) + " bytes held, " + std::to_string(f.bytes) + " asked)");
        return CT_ERR_OOM;
      }
    }
    f.nodes = pool_base + f.pool_off;
    f.off = reinterpret_cast<uint32_t*>(pool_base + f.pool_off + node_bytes);
    if (cudaMemcpyAsync(f.nodes, src, (size_t)n_nodes * elem, cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(f.off, off, off_bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      std::lock_guard<std::mutex> lk(mu);
      pool.release(f.pool_off, f.bytes);
      set_last_error("server: forest upload failed");
      return CT_ERR_CUDA;
    }
    f.host = std::make_shared<std::vector<ct_packed_node>>(nodes, nodes + n_nodes);
    f.host_off = std::make_shared<std::vector<uint32_t>>(off, off + n_trees);
    std::lock_guard<std::mutex> lk(mu);
    forests.push_back(f);
    *id = (uint32_t)(forests.size() - 1);
    return CT_OK;
  }

  int forest_info(uint32_t id, uint32_t* n_nodes, uint32_t* n_trees, uint32_t* n_features, uint32_t* n_classes) {
    std::lock_guard<std::mutex> lk(mu);
    CT_ARG_CHECK(id < forests.size() && !forests[id].removed, "server: unknown forest id");
    const Forest& f = forests[id];
    if (n_nodes) *n_nodes = f.n_nodes;
    if (n_trees) *n_trees = f.n_trees;
    if (n_features) *n_features = f.n_features;
    if (n_classes) *n_classes = f.n_classes;
    return CT_OK;
  }

  int read_forest(uint32_t id, ct_packed_node* nodes, uint32_t* off) {
    std::shared_ptr<std::vector<ct_packed_node>> h;
    std::shared_ptr<std::vector<uint32_t>> o;
    {
      std::lock_guard<std::mutex> lk(mu);
      CT_ARG_CHECK(id < forests.size() && !forests[id].removed, "server: unknown forest id");
      h = forests[id].host;
      o = forests[id].host_off;
    }
    CT_ARG_CHECK(nodes && off, "server: NULL output");
    std::copy(h->begin(), h->end(), nodes);
    std::copy(o->begin(), o->end(), off);
    return CT_OK;
  }

  int remove_forest(uint32_t id) {
    std::lock_guard<std::mutex> lk(mu);
    CT_ARG_CHECK(id < forests.size() && !forests[id].removed, "server: unknown forest id");
    Forest& f = forests[id];
    f.removed = true;
    f.host.reset();
    f.host_off.reset();
    if (f.refs == 0) pool.release(f.pool_off, f.bytes);
    return CT_OK;
  }

  // caller holds mu
  void unref(uint32_t id) {
    Forest& f = forests[id];
    if (--f.refs == 0 && f.removed) pool.release(f.pool_off, f.bytes);
  }

  int submit(ct_request* r) {
    CT_ARG_CHECK(r && r->x && r->n_rows, "server: empty request");
    std::unique_lock<std::mutex> lk(mu);
    r->status = CT_OK;
    r->latency_ms = -1.0;
    auto* j = new Job();
    j->req = r;
    j->t_start = now_s();
    if (t_first == 0) t_first = j->t_start;
    if (r->kind == CT_REQ_FIT) {
      if (fit_workers.empty()) {
        delete j;
        set_last_error("server: no fit workers");
        return CT_ERR_ARG;
      }
      fit_q.push_back(j);
    } else {
      if (r->forest >= forests.size() || forests[r->forest].removed) {
        delete j;
        set_last_error("server: unknown forest id");
        return CT_ERR_ARG;
      }
      const Forest& f = forests[r->forest];
      const int l = r->n_rows <= cfg.small_rows ? 0 : 1;
      if ((uint64_t)r->n_rows * f.n_features > lanes[l].cap_floats || r->n_rows > lanes[l].cap_rows) {
        // admission: a request larger than the lane's staging never fits
        r->status = CT_ERR_OOM;
        r->latency_ms = 0;
        ++n_rejected;
        delete j;
        set_last_error("server: request larger than the staging capacity");
        return CT_ERR_OOM;
      }
      lanes[l].q.push_back(j);
    }
    r->pending_ = j;
    lk.unlock();
    cv_work.notify_all();
    return CT_OK;
  }

  int wait(ct_request* r, double timeout_s) {
    std::unique_lock<std::mutex> lk(mu);
    Job* j = reinterpret_cast<Job*>(r->pending_);
    if (!j) return r->status;
    const bool ok = cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return j->done; });
    if (!ok) {
      set_last_error("server: wait timed out");
      return CT_ERR_TIMEOUT;
    }
    r->pending_ = nullptr;
    delete j;
    return r->status;
  }

  void finish(Job* j, double t, int status) {
    // caller holds mu
    ct_request* r = j->req;
    r->status = status;
    r->latency_ms = (t - j->t_start) * 1000.0;
    j->done = true;
    t_last = std::max(t_last, t);
    if (r->kind == CT_REQ_FIT) {
      lat_fit.push_back(r->latency_ms);
      ++n_fit;
    } else if (status == CT_OK) {
      (r->n_rows <= 4096 ? lat_small : lat_large).push_back(r->latency_ms);
      ++n_req;
      n_rows += r->n_rows;
    }
  }

  void complete_slot(Slot& s) {
    const double t = now_s();
    std::lock_guard<std::mutex> lk(mu);
    for (Job* j : s.jobs) {
      unref(j->req->forest);
      finish(j, t, CT_OK);
    }
    s.jobs.clear();
    cv_done.notify_all();
  }

  void lane_loop(int l) {
    cudaSetDevice(device);
    Lane& ln = lanes[l];
    int next = 0;
    while (true) {
      // retire finished batches
      for (auto& s : ln.slot)
        if (!s.jobs.empty() && cudaEventQuery(s.ev) == cudaSuccess) complete_slot(s);
      std::vector<Job*> batch;
      {
        std::unique_lock<std::mutex> lk(mu);
        if (ln.q.empty()) {
          Slot* oldest = nullptr;
          for (auto& s : ln.slot)
            if (!s.jobs.empty() && (!oldest || s.launched < oldest->launched)) oldest = &s;
          if (oldest) {
            lk.unlock();
            cudaEventSynchronize(oldest->ev);
            complete_slot(*oldest);
            continue;
          }
          if (stop) break;
          cv_work.wait(lk, [&] { return stop || !ln.q.empty(); });
          if (ln.q.empty()) continue;
        }
        uint64_t rows = 0, floats = 0;
        while (!ln.q.empty() && batch.size() < 4096) {
          Job* j = ln.q.front();
          const Forest& f = forests[j->req->forest];
          const uint64_t fl = (uint64_t)j->req->n_rows * f.n_features;
          if (!batch.empty() && (rows + j->req->n_rows > ln.cap_rows || floats + fl > ln.cap_floats)) break;
          rows += j->req->n_rows;
          floats += fl;
          batch.push_back(j);
          ln.q.pop_front();
        }
      }
      Slot& s = ln.slot[next];
      if (!s.jobs.empty()) {  // both slots busy: wait for this one
        cudaEventSynchronize(s.ev);
        complete_slot(s);
      }
      next ^= 1;
      launch(ln, s, batch);
    }
  }

  void launch(Lane& ln, Slot& s, std::vector<Job*>& batch) {
    const bool small_lane = &ln == &lanes[0];
    uint64_t xoff = 0, roff = 0, voff = 0, zero = 0;
    size_t smem = 0;
    uint32_t blocks = 0, max_c = 1;
    bool grouped = false;
    std::vector<Forest> fs;
    {
      // a forest removed after the request was queued: the request fails;
      // the others hold a reference until their batch completes
      std::lock_guard<std::mutex> lk(mu);
      size_t kept = 0;
      for (Job* j : batch) {
        Forest& f = forests[j->req->forest];
        if (f.removed) {
          finish(j, now_s(), CT_ERR_ARG);
          continue;
        }
        ++f.refs;
        fs.push_back(f);
        max_c = std::max(max_c, f.n_classes);
        batch[kept++] = j;
      }
      if (kept < batch.size()) cv_done.notify_all();
      batch.resize(kept);
    }
    if (batch.empty()) return;
    int err = 0;
    s.direct.assign(batch.size(), 0);
    for (size_t i = 0; i < batch.size(); ++i) {
      ct_request* r = batch[i]->req;
      const Forest& f = fs[i];
      BatchReq& br = s.req_host[i];
      const uint32_t rpb = predict_rows_per_block(f.n_classes, f.n_features);
      smem = std::max(smem, predict_tile_smem(rpb, f.n_classes, f.n_features));
      // small requests whose rows are staged whole read and answer host
      // memory directly when the device can address it
      s.direct[i] = small_lane && predict_tile_smem(rpb, f.n_classes, f.n_features) >
                                      (size_t)rpb * f.n_classes * sizeof(uint32_t) &&
                    device_addressable(r->x) && device_addressable(r->pred);
      br.nodes = f.nodes;
      br.fbits = f.fbits;
      br.rpb = rpb;
      br.tree_off = f.off;
      br.x = s.direct[i] ? r->x : s.x_dev + xoff;
      br.pred = s.direct[i] ? r->pred : s.pred_dev + roff;
      br.n_rows = r->n_rows;
      br.n_features = f.n_features;
      br.n_classes = f.n_classes;
      br.n_trees = f.n_trees;
      br.block0 = blocks;
      br.tiles = ceil_div(r->n_rows, rpb);
      br.group = f.group;
      br.row0 = (uint32_t)roff;
      br.votes = nullptr;  // a single-group request votes directly and must not touch the table
      if (f.group < f.n_trees) {
        grouped = true;
        br.votes = s.votes_dev + voff;
        voff += (uint64_t)r->n_rows * f.n_classes;
      }
      blocks += br.tiles * ceil_div(f.n_trees, f.group);
      if (s.direct[i]) {
        ++zero;
      } else {
        if (cudaMemcpyAsync(s.x_dev + xoff, r->x, (size_t)r->n_rows * f.n_features * sizeof(float),
                            cudaMemcpyHostToDevice, ln.st) != cudaSuccess)
          err = 1;
        xoff += (uint64_t)r->n_rows * f.n_features;
      }
      roff += r->n_rows;
    }
    if (voff && cudaMemsetAsync(s.votes_dev, 0, voff * sizeof(uint32_t), ln.st) != cudaSuccess) err = 1;
    if (cudaMemcpyAsync(s.req_dev, s.req_host, batch.size() * sizeof(BatchReq), cudaMemcpyHostToDevice, ln.st) !=
        cudaSuccess)
      err = 1;
    if (predict_batch(s.req_dev, (uint32_t)batch.size(), blocks, (uint32_t)roff, smem, grouped, ln.st) != CT_OK)
      err = 1;
    for (size_t i = 0; i < batch.size(); ++i) {
      ct_request* r = batch[i]->req;
      if (s.direct[i]) continue;
      if (cudaMemcpyAsync(r->pred, s.pred_dev + s.req_host[i].row0, (size_t)r->n_rows * 4, cudaMemcpyDeviceToHost,
                          ln.st) != cudaSuccess)
        err = 1;
    }
    cudaEventRecord(s.ev, ln.st);
    s.launched = now_s();
    s.jobs = batch;
    {
      std::lock_guard<std::mutex> lk(mu);
      ++n_batches;
      n_zero_copy += zero;
    }
    if (err) {
      cudaEventSynchronize(s.ev);
      std::lock_guard<std::mutex> lk(mu);
      for (Job* j : s.jobs) {
        unref(j->req->forest);
        finish(j, now_s(), CT_ERR_CUDA);
      }
      s.jobs.clear();
      cv_done.notify_all();
    }
  }

  void fit_loop(FitWorker& fw) {
    cudaSetDevice(device);
    while (true) {
      Job* j = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || !fit_q.empty(); });
        if (fit_q.empty()) {
          if (stop) break;
          continue;
        }
        j = fit_q.front();
        fit_q.pop_front();
      }
      uint32_t fid = NONE;
      int st = run_fit(fw, j->req, &fid);
      std::lock_guard<std::mutex> lk(mu);
      j->req->result_forest = fid;
      if (st == CT_ERR_OOM) ++n_rejected;
      finish(j, now_s(), st);
      cv_done.notify_all();
    }
  }

  // Host arrays -> new resident forest, on the worker's stream and arena.
  int run_fit(FitWorker& fw, ct_request* r, uint32_t* fid) {
    const uint32_t n = r->n_rows, F = r->n_features, C = r->n_classes, T = r->n_trees;
    CT_ARG_CHECK(r->y && n && F && C && T && C <= CT_MAX_CLASSES, "fit job: bad arguments");
    CT_ARG_CHECK(F <= cfg.max_features, "fit job: more features than the server's max_features");
    if (job_bytes(n, F, C, T) > fw.arena_bytes) {
      set_last_error("fit job larger than the fit arena (admission)");
      return CT_ERR_OOM;
    }
    cudaStream_t st = fw.st;
    Arena a{fw.arena, fw.arena_bytes, 0};
    const uint32_t ib = n <= 0xFFFF ? 2 : 4, lb = C <= 255 ? 1 : 2;
    const size_t nf = (size_t)n * F;
    float* x_rm = a.take<float>(nf);
    float* x_fm = a.take<float>(nf);
    char* labels = a.take<char>((size_t)n * 2);
    char* pre = a.take<char>(nf * ib + 64);
    const size_t pws_b = presort_workspace_bytes(n, F);
    char* pws = a.take<char>(pws_b);
    char* si0 = a.take<char>((size_t)T * nf * ib + 64);
    char* si1 = a.take<char>((size_t)T * nf * ib + 64);
    const size_t mb = mark_bits_offset(n, T) + (size_t)T * mark_bit_words(n) * 4 + 64;
    uint8_t* mark = a.take<uint8_t>(mb);
    const uint32_t cap = 2 * n;
    uint32_t* raw = a.take<uint32_t>((size_t)T * cap * 5);
    uint32_t* counts = a.take<uint32_t>(T);
    const size_t fsb = fetch_trees_scratch((uint64_t)T * 2 * n, T);
    char* fscratch = a.take<char>(fsb);
    ct_problem p{};
    p.x_fm = x_fm;
    p.labels = labels;
    p.presort = pre;
    p.n_rows = n;
    p.n_features = F;
    p.n_classes = C;
    p.index_bytes = ib;
    p.label_bytes = lb;
    p.max_features = r->max_features ? std::min(r->max_features, F) : (uint32_t)std::ceil(std::sqrt((double)F));
    p.min_samples_split = 1;
    p.bootstrap = 1;
    p.seed = r->seed;
    ct_fit_options o{};
    o.mode = CT_FIT_BATCHED;
    o.subtree_cutoff = 32;
    // each job has its own shape and arena, so a loop graph would be built
    // for one fit and dropped: host-driven levels cost less here
    o.flags = CT_FIT_HOST_LOOP;
    const size_t wsb = fit_workspace_bytes(&p, T, &o);
    char* ws = a.take<char>(wsb);
    if (!ws || !a.ok()) {
      set_last_error("fit job: arena carve failed");
      return CT_ERR_OOM;
    }
    std::vector<uint8_t> lab_host((size_t)n * lb);
    for (uint32_t i = 0; i < n; ++i) {
      if (r->y[i] >= C) {
        set_last_error("fit job: label out of range");
        return CT_ERR_ARG;
      }
      if (lb == 1) lab_host[i] = (uint8_t)r->y[i];
      else reinterpret_cast<uint16_t*>(lab_host.data())[i] = (uint16_t)r->y[i];
    }
    CT_CUDA_TRY(cudaMemcpyAsync(x_rm, r->x, nf * 4, cudaMemcpyHostToDevice, st));
    CT_CUDA_TRY(cudaMemcpyAsync(labels, lab_host.data(), lab_host.size(), cudaMemcpyHostToDevice, st));
    CT_TRY(transpose_rows(x_rm, n, F, x_fm, st));
    CT_TRY(presort(x_fm, n, F, ib, pre, pws, pws_b, st));
    ct_lists l{si0, si1, mark, n, T};
    ct_tree_buffers tb{raw, raw + (size_t)T * cap, raw + 2 * (size_t)T * cap,
                       reinterpret_cast<float*>(raw + 3 * (size_t)T * cap), raw + 4 * (size_t)T * cap, counts, cap};
    CT_TRY(fit(&p, &l, 0, T, &o, &tb, ws, wsb, st));
    std::vector<uint32_t> cnt(T);
    CT_CUDA_TRY(cudaMemcpyAsync(cnt.data(), counts, T * 4, cudaMemcpyDeviceToHost, st));
    CT_CUDA_TRY(cudaStreamSynchronize(st));
    uint64_t total = 0;
    std::vector<uint32_t> offs(T);
    for (uint32_t t = 0; t < T; ++t) {
      offs[t] = (uint32_t)total;
      total += cnt[t];
    }
    std::vector<uint32_t> ol(total), orr(total), ov(total);
    std::vector<uint16_t> of(total);
    std::vector<float> ot(total);
    CT_TRY(fetch_trees(&tb, T, cnt.data(), fscratch, fsb, ol.data(), orr.data(), of.data(), ot.data(), ov.data(),
                       st));
    std::vector<ct_packed_node> packed(total);
    for (uint64_t i = 0; i < total; ++i) packed[i] = ct_packed_node{ot[i], of[i], ol[i], ov[i]};
    return add_forest(packed.data(), (uint32_t)total, offs.data(), T, F, C, fid, st);
  }

  static double pct(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    const size_t k = std::min(v.size() - 1, (size_t)std::ceil(q * v.size()) - (q > 0 ? 1 : 0));
    std::nth_element(v.begin(), v.begin() + k, v.end());
    return v[k];
  }

  void stats(ct_server_stats* out) {
    std::lock_guard<std::mutex> lk(mu);
    std::vector<double> all = lat_small;
    all.insert(all.end(), lat_large.begin(), lat_large.end());
    out->requests = n_req;
    out->rows = n_rows;
    out->batches = n_batches;
    out->fit_jobs = n_fit;
    out->rejected = n_rejected;
    out->p50_ms = pct(all, 0.50);
    out->p99_ms = pct(all, 0.99);
    out->p50_small_ms = pct(lat_small, 0.50);
    out->p99_small_ms = pct(lat_small, 0.99);
    out->p50_fit_ms = pct(lat_fit, 0.50);
    out->p99_fit_ms = pct(lat_fit, 0.99);
    out->max_ms = all.empty() ? 0.0 : *std::max_element(all.begin(), all.end());
    out->wall_s = t_last > t_first ? t_last - t_first : 0.0;
    out->rows_per_s = out->wall_s > 0 ? n_rows / out->wall_s : 0.0;
    out->hbm_used_bytes = used;
    out->hbm_budget_bytes = budget;
    out->zero_copy_requests = n_zero_copy;
    out->forest_bytes = pool.used();
    out->forest_pool_bytes = pool.total();
  }

  void reset_stats() {
    std::lock_guard<std::mutex> lk(mu);
    lat_small.clear();
    lat_large.clear();
    lat_fit.clear();
    n_req = n_rows = n_batches = n_fit = n_rejected = n_zero_copy = 0;
    t_first = t_last = 0;
  }
};

}  // namespace ct

using namespace ct;

extern "C" {

int ct_server_create(const ct_server_config* cfg, void** handle) {
  CT_ARG_CHECK(cfg && handle, "NULL argument");
  try {
    auto s = std::make_unique<Server>();
    const int st = s->init(cfg);
    if (st != CT_OK) return st;  // destructor frees what init allocated
    *handle = s.release();
    return CT_OK;
  } catch (const std::exception& e) {
    set_last_error(std::string("server create: ") + e.what());
    return CT_ERR_INTERNAL;
  }
}

int ct_server_destroy(void* handle) {
  CT_GUARD({
    delete reinterpret_cast<Server*>(handle);
    return CT_OK;
  })
}

int ct_server_add_forest(void* handle, const ct_packed_node* nodes, uint32_t n_nodes, const uint32_t* tree_offset,
                         uint32_t n_trees, uint32_t n_features, uint32_t n_classes, uint32_t* forest_id) {
  CT_ARG_CHECK(handle, "NULL server");
  CT_GUARD({
    return reinterpret_cast<Server*>(handle)->add_forest(nodes, n_nodes, tree_offset, n_trees, n_features, n_classes,
                                                          forest_id);
  })
}

int ct_server_forest_info(void* handle, uint32_t forest_id, uint32_t* n_nodes, uint32_t* n_trees,
                          uint32_t* n_features, uint32_t* n_classes) {
  CT_ARG_CHECK(handle, "NULL server");
  CT_GUARD({
    return reinterpret_cast<Server*>(handle)->forest_info(forest_id, n_nodes, n_trees, n_features, n_classes);
  })
}

int ct_server_read_forest(void* handle, uint32_t forest_id, ct_packed_node* nodes, uint32_t* tree_offset) {
  CT_ARG_CHECK(handle, "NULL server");
  CT_GUARD({
    return reinterpret_cast<Server*>(handle)->read_forest(forest_id, nodes, tree_offset);
  })
}

int ct_server_remove_forest(void* handle, uint32_t forest_id) {
  CT_ARG_CHECK(handle, "NULL server");
  CT_GUARD({
    return reinterpret_cast<Server*>(handle)->remove_forest(forest_id);
  })
}

int ct_server_submit(void* handle, ct_request* req) {
  CT_ARG_CHECK(handle, "NULL server");
  CT_GUARD({
    return reinterpret_cast<Server*>(handle)->submit(req);
  })
}

int ct_server_wait(void* handle, ct_request* req, double timeout_s) {
  CT_ARG_CHECK(handle && req, "NULL argument");
  CT_GUARD({
    return reinterpret_cast<Server*>(handle)->wait(req, timeout_s);
  })
}

int ct_server_replay(void* handle, ct_request* reqs, uint32_t n, double timeout_s, ct_server_stats* stats) {
  CT_ARG_CHECK(handle && (reqs || n == 0), "NULL argument");
  CT_GUARD({
    Server* s = reinterpret_cast<Server*>(handle);
    s->reset_stats();
    const double t0 = now_s();
    for (uint32_t i = 0; i < n; ++i) {
      const double due = t0 + reqs[i].arrival_s;
      while (now_s() < due) {
        const double left = due - now_s();
        if (left > 200e-6) std::this_thread::sleep_for(std::chrono::duration<double>(left - 100e-6));
      }
      const int st = s->submit(&reqs[i]);
      if (st != CT_OK && st != CT_ERR_OOM) return st;
    }
    int worst = CT_OK;
    for (uint32_t i = 0; i < n; ++i) {
      if (!reqs[i].pending_) continue;
      const int st = s->wait(&reqs[i], timeout_s);
      if (st == CT_ERR_TIMEOUT) return st;
      if (st != CT_OK) worst = st;
    }
    if (stats) s->stats(stats);
    (void)worst;
    return CT_OK;
  })
}

int ct_server_get_stats(void* handle, ct_server_stats* out) {
  CT_ARG_CHECK(handle && out, "NULL argument");
  CT_GUARD({
    reinterpret_cast<Server*>(handle)->stats(out);
    return CT_OK;
  })
}

}  // extern "C"
