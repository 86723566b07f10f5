// The extern "C" boundary (include/fgkl_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/fgkl_b200.h"
#include "adjoint_engine.h"
#include "engine.h"
#include "planner.h"
#include "sw_engine.h"
#include "synthetic.h"
#include "tables.h"

namespace {

thread_local std::string t_error;

int set_error(int code, const std::string& msg) {
  t_error = msg;
  return code;
}

// The device this process computes on: FGKL_DEVICE, else 0. An sm_100 part is required; there is
// no CPU path.
int pick_device(int* device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return set_error(FGKL_E_NO_DEVICE, "no CUDA device is visible");
  int d = 0;
  if (const char* env = std::getenv("FGKL_DEVICE")) d = std::atoi(env);
  if (d < 0 || d >= n) return set_error(FGKL_E_NO_DEVICE, "FGKL_DEVICE names no visible device");
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, d) != cudaSuccess) return set_error(FGKL_E_NO_DEVICE, "cannot query the CUDA device");
  if (prop.major != 10 || prop.minor != 0)
    return set_error(FGKL_E_NO_DEVICE, std::string("the kernels are built for sm_100a; device is ") + prop.name);
  *device = d;
  return FGKL_OK;
}

// One engine per calling thread for the per-call entry points. Engines are never destroyed: a
// thread that exits hands its engine to a pool, from which the next new thread on that device takes
// it. So no CUDA call runs from a destructor -- at a thread's exit, or at the process's exit, when
// the main thread's thread-local objects are destroyed while the CUDA runtime's own teardown may
// already be under way -- and a caller whose threads come and go (a JVM thread pool) reuses the
// engines' device buffers instead of allocating new ones.
struct EnginePool {
  std::mutex mu;
  std::vector<std::pair<int, fgkl::Engine*>> idle;  // (device, engine)
};
EnginePool& engine_pool() {
  static EnginePool* pool = new EnginePool;  // never destroyed, like its engines
  return *pool;
}

struct ThreadEngine {
  fgkl::Engine* engine = nullptr;
  int device = -1;
  ~ThreadEngine() {
    if (!engine) return;
    EnginePool& p = engine_pool();
    std::lock_guard<std::mutex> lock(p.mu);
    try {
      p.idle.emplace_back(device, engine);
    } catch (...) {
      // Out of host memory at thread exit: the engine is left unreferenced rather than destroyed.
    }
  }
};

fgkl::Engine* thread_engine(int* rc) {
  thread_local ThreadEngine te;
  if (!te.engine) {
    int d = 0;
    if ((*rc = pick_device(&d)) != FGKL_OK) return nullptr;
    {
      EnginePool& p = engine_pool();
      std::lock_guard<std::mutex> lock(p.mu);
      for (size_t i = 0; i < p.idle.size(); ++i)
        if (p.idle[i].first == d) {
          te.engine = p.idle[i].second;
          p.idle.erase(p.idle.begin() + static_cast<std::ptrdiff_t>(i));
          break;
        }
    }
    if (!te.engine) te.engine = new fgkl::Engine(d);
    te.device = d;
  }
  *rc = FGKL_OK;
  return te.engine;
}

// The calling thread's Smith-Waterman engine, pooled and never destroyed like the PairHMM engines.
struct SwPool {
  std::mutex mu;
  std::vector<std::pair<int, fgkl::SwEngine*>> idle;
};
SwPool& sw_pool() {
  static SwPool* pool = new SwPool;
  return *pool;
}
struct ThreadSw {
  fgkl::SwEngine* engine = nullptr;
  int device = -1;
  ~ThreadSw() {
    if (!engine) return;
    SwPool& p = sw_pool();
    std::lock_guard<std::mutex> lock(p.mu);
    try {
      p.idle.emplace_back(device, engine);
    } catch (...) {
    }
  }
};
fgkl::SwEngine* thread_sw(int* rc) {
  thread_local ThreadSw ts;
  if (!ts.engine) {
    int d = 0;
    if ((*rc = pick_device(&d)) != FGKL_OK) return nullptr;
    {
      SwPool& p = sw_pool();
      std::lock_guard<std::mutex> lock(p.mu);
      for (size_t i = 0; i < p.idle.size(); ++i)
        if (p.idle[i].first == d) {
          ts.engine = p.idle[i].second;
          p.idle.erase(p.idle.begin() + static_cast<std::ptrdiff_t>(i));
          break;
        }
    }
    if (!ts.engine) ts.engine = new fgkl::SwEngine(d);
    ts.device = d;
  }
  *rc = FGKL_OK;
  return ts.engine;
}

// Offset table -> (start, end) checks of crates/jni/src/lib.rs:343-363.
int check_offsets(const int32_t* offsets, int64_t n, int64_t total, const char* what) {
  if (n < 1 || offsets == nullptr || offsets[0] != 0)
    return set_error(FGKL_E_BAD_OFFSETS, std::string(what) + " offset table must start at zero");
  if (offsets[n - 1] < 0 || static_cast<int64_t>(offsets[n - 1]) != total)
    return set_error(FGKL_E_BAD_OFFSETS, std::string(what) + " offset table must end at the array length");
  for (int64_t i = 1; i < n; ++i)
    if (offsets[i] < offsets[i - 1]) return set_error(FGKL_E_BAD_OFFSETS, std::string(what) + " offset table must be non-decreasing");
  return FGKL_OK;
}

void to_stats(const fgkl::BatchStats& bs, fgkl_stats* s);

// One validated per-call request.
struct CallRequest {
  const fgkl_reads* reads = nullptr;
  const fgkl_haplotypes* haps = nullptr;
  bool pd = false;
  fgkl::EngineConfig ec;
  double* out = nullptr;
  int64_t n_reads = 0, n_haps = 0;
  enum State { kQueued, kTaken, kDone, kAlone } state = kQueued;  // guarded by the combiner's mutex
};

// Runs one request on engine `e`; an error is reported on the calling thread.
int run_on(fgkl::Engine* e, const CallRequest& q, fgkl_stats* stats) try {
  int rc;
  std::vector<int64_t> roff(static_cast<size_t>(q.n_reads) + 1), hoff(static_cast<size_t>(q.n_haps) + 1);
  for (int64_t i = 0; i <= q.n_reads; ++i) roff[i] = q.reads->offsets[i];
  for (int64_t i = 0; i <= q.n_haps; ++i) hoff[i] = q.haps->offsets[i];
  const int32_t nr = static_cast<int32_t>(q.n_reads), nh = static_cast<int32_t>(q.n_haps);
  fgkl::BatchInput in;
  in.num_regions = 1;
  in.region_reads = &nr;
  in.region_haps = &nh;
  in.bases = q.reads->bases;
  in.quals = q.reads->quals;
  in.ins = q.reads->ins_gop;
  in.del = q.reads->del_gop;
  in.gcp = q.reads->gcp;
  in.read_off = roff.data();
  in.hap_bases = q.haps->bases;
  in.hap_flags = q.pd ? q.haps->flags : nullptr;
  in.hap_off = hoff.data();
  fgkl::BatchStats bs;
  rc = e->compute(in, q.ec, q.out, q.n_reads * q.n_haps, &bs);
  if (rc) return set_error(rc, e->error());
  if (stats) to_stats(bs, stats);
  return FGKL_OK;
} catch (const std::bad_alloc&) {
  return set_error(FGKL_E_OUT_OF_MEMORY, "host memory allocation failed");
} catch (...) {
  return set_error(FGKL_E_CUDA, "internal error in the per-call path");
}

// Runs one request on the calling thread's engine.
int run_alone(const CallRequest& q, fgkl_stats* stats) try {
  int rc;
  fgkl::Engine* e = thread_engine(&rc);
  if (!e) return rc;
  return run_on(e, q, stats);
} catch (const std::bad_alloc&) {
  return set_error(FGKL_E_OUT_OF_MEMORY, "host memory allocation failed");
} catch (...) {
  return set_error(FGKL_E_CUDA, "internal error in the per-call path");
}

// ---------------------------------------------------------------------------------------------
// Combining of concurrent per-call requests.
//
// GATK calls the native PairHMM once per region from several threads. One region's tasks occupy a
// fraction of the SMs, and the launch chains of separate calls queue behind one another on the
// driver's hardware queues, so separate calls from 8 threads reach about the throughput of one and
// a half. A call therefore joins the calls waiting when it arrives. The first caller to find fewer
// than g_max_in_flight batches running takes a free slot, its own request and every waiting one of
// its kind, concatenates them into one batch on the slot's engine and writes each caller's results;
// the others sleep until theirs are written. Each slot keeps one engine, so its buffers grow to the
// largest combined batch once instead of once per calling thread. A region's program and a read's
// arithmetic do not depend on the batch around them, so the results are bit-identical to separate
// calls. A combined batch that fails is retried as separate calls, each on its caller's thread, so
// that every caller gets its own status and message.
// ---------------------------------------------------------------------------------------------

constexpr int kMaxSlots = 8;                         // batches in flight at most
std::atomic<int> g_max_in_flight{2};
constexpr size_t kMaxCombined = 64;                  // requests in one combined batch
constexpr int64_t kMaxCombinedReadBytes = 64 << 20;  // read bytes of one combined batch

struct Combiner {
  std::mutex mu;
  std::condition_variable cv;
  std::vector<CallRequest*> queue;  // waiting requests, in arrival order
  int in_flight = 0;                // batches running
  bool slot_busy[kMaxSlots] = {};
  // Created on a slot's first batch and kept for the life of the process (never destroyed: their
  // destructors would run after the CUDA runtime at exit).
  fgkl::Engine* engines[kMaxSlots] = {};
};
Combiner g_combiner;
std::atomic<uint64_t> g_combined_batches{0}, g_combined_requests{0};

bool same_kind(const CallRequest& a, const CallRequest& b) {
  return a.pd == b.pd && a.ec.double_precision == b.ec.double_precision && a.ec.double_fallback == b.ec.double_fallback &&
         a.ec.share_suffixes == b.ec.share_suffixes;
}

int64_t read_bytes(const CallRequest& q) { return q.reads->bases_len; }

// Concatenation buffers of a leading thread, kept between its batches.
struct CombinedBuffers {
  std::vector<uint8_t> bases, quals, ins, del, gcp, hap_bases, hap_flags;
  std::vector<int64_t> read_off, hap_off;
  std::vector<int32_t> region_reads, region_haps;
  std::vector<double> out;
};

// Runs the n requests of `batch` as one batch on engine `e` and scatters the results to their
// callers; false when the batch failed (nothing is written then that a retry would not overwrite).
bool run_combined(fgkl::Engine* e, CallRequest* const* batch, size_t n_batch) {
  try {
    thread_local CombinedBuffers b;
    int64_t rbytes = 0, hbytes = 0, nreads = 0, nhaps = 0, nout = 0;
    for (size_t g = 0; g < n_batch; ++g) {
      const CallRequest* q = batch[g];
      rbytes += q->reads->bases_len;
      hbytes += q->haps->bases_len;
      nreads += q->n_reads;
      nhaps += q->n_haps;
      nout += q->n_reads * q->n_haps;
    }
    const bool pd = batch[0]->pd;
    for (auto* v : {&b.bases, &b.quals, &b.ins, &b.del, &b.gcp}) v->resize(static_cast<size_t>(rbytes));
    b.hap_bases.resize(static_cast<size_t>(hbytes));
    b.hap_flags.resize(pd ? static_cast<size_t>(hbytes) : 0);
    b.read_off.resize(static_cast<size_t>(nreads) + 1);
    b.hap_off.resize(static_cast<size_t>(nhaps) + 1);
    b.region_reads.resize(n_batch);
    b.region_haps.resize(n_batch);
    b.out.resize(static_cast<size_t>(nout));
    int64_t ro = 0, ho = 0, ri = 0, hi = 0;
    b.read_off[0] = 0;
    b.hap_off[0] = 0;
    for (size_t g = 0; g < n_batch; ++g) {
      const CallRequest& q = *batch[g];
      const size_t n = static_cast<size_t>(q.reads->bases_len), m = static_cast<size_t>(q.haps->bases_len);
      if (n) {
        std::memcpy(b.bases.data() + ro, q.reads->bases, n);
        std::memcpy(b.quals.data() + ro, q.reads->quals, n);
        std::memcpy(b.ins.data() + ro, q.reads->ins_gop, n);
        std::memcpy(b.del.data() + ro, q.reads->del_gop, n);
        std::memcpy(b.gcp.data() + ro, q.reads->gcp, n);
      }
      if (m) {
        std::memcpy(b.hap_bases.data() + ho, q.haps->bases, m);
        if (pd) std::memcpy(b.hap_flags.data() + ho, q.haps->flags, m);
      }
      for (int64_t r = 1; r <= q.n_reads; ++r) b.read_off[ri + r] = ro + q.reads->offsets[r];
      for (int64_t h = 1; h <= q.n_haps; ++h) b.hap_off[hi + h] = ho + q.haps->offsets[h];
      b.region_reads[g] = static_cast<int32_t>(q.n_reads);
      b.region_haps[g] = static_cast<int32_t>(q.n_haps);
      ro += static_cast<int64_t>(n);
      ho += static_cast<int64_t>(m);
      ri += q.n_reads;
      hi += q.n_haps;
    }
    fgkl::BatchInput in;
    in.num_regions = static_cast<int32_t>(n_batch);
    in.region_reads = b.region_reads.data();
    in.region_haps = b.region_haps.data();
    in.bases = b.bases.data();
    in.quals = b.quals.data();
    in.ins = b.ins.data();
    in.del = b.del.data();
    in.gcp = b.gcp.data();
    in.read_off = b.read_off.data();
    in.hap_bases = b.hap_bases.data();
    in.hap_flags = pd ? b.hap_flags.data() : nullptr;
    in.hap_off = b.hap_off.data();
    if (e->compute(in, batch[0]->ec, b.out.data(), nout, nullptr) != FGKL_OK) return false;
    g_combined_batches.fetch_add(1, std::memory_order_relaxed);
    g_combined_requests.fetch_add(n_batch, std::memory_order_relaxed);
    int64_t o = 0;
    for (size_t g = 0; g < n_batch; ++g) {
      const CallRequest* q = batch[g];
      const int64_t k = q->n_reads * q->n_haps;
      std::memcpy(q->out, b.out.data() + o, static_cast<size_t>(k) * sizeof(double));
      o += k;
    }
    return true;
  } catch (...) {
    return false;
  }
}

int combined_call(CallRequest& q) {
  Combiner& c = g_combiner;
  std::unique_lock<std::mutex> lk(c.mu);
  try {
    c.queue.push_back(&q);
  } catch (...) {
    lk.unlock();
    return run_alone(q, nullptr);
  }
  for (;;) {
    if (q.state == CallRequest::kDone) return FGKL_OK;
    if (q.state == CallRequest::kAlone) {
      lk.unlock();
      return run_alone(q, nullptr);
    }
    if (q.state == CallRequest::kQueued &&
        c.in_flight < std::min(kMaxSlots, std::max(1, g_max_in_flight.load(std::memory_order_relaxed)))) {
      int slot = 0;
      while (c.slot_busy[slot]) ++slot;
      if (!c.engines[slot]) {
        int d = 0;
        int rc = pick_device(&d);
        if (rc == FGKL_OK) {
          try {
            c.engines[slot] = new fgkl::Engine(d);
          } catch (...) {
            rc = set_error(FGKL_E_OUT_OF_MEMORY, "host memory allocation failed");
          }
        }
        if (rc != FGKL_OK) {
          // This request leaves the queue with the error; the others meet the same.
          c.queue.erase(std::find(c.queue.begin(), c.queue.end(), &q));
          return rc;
        }
      }
      // Lead: this request first, then the waiting ones of its kind in arrival order (no
      // allocation here, so nothing can throw while requests are moved out of the queue).
      CallRequest* batch[kMaxCombined];
      size_t n_batch = 0;
      batch[n_batch++] = &q;
      int64_t bytes = read_bytes(q);
      size_t keep = 0;
      for (CallRequest* r : c.queue) {
        if (r != &q && same_kind(*r, q) && n_batch < kMaxCombined && bytes + read_bytes(*r) <= kMaxCombinedReadBytes) {
          batch[n_batch++] = r;
          bytes += read_bytes(*r);
        } else if (r != &q) {
          c.queue[keep++] = r;
        }
      }
      c.queue.resize(keep);
      for (size_t k = 0; k < n_batch; ++k) batch[k]->state = CallRequest::kTaken;
      ++c.in_flight;
      c.slot_busy[slot] = true;
      fgkl::Engine* const e = c.engines[slot];
      lk.unlock();
      if (n_batch == 1) {
        // Alone after all: the error, if any, is set on this thread directly.
        const int rc = run_on(e, q, nullptr);
        lk.lock();
        --c.in_flight;
        c.slot_busy[slot] = false;
        c.cv.notify_all();
        return rc;
      }
      const bool ok = run_combined(e, batch, n_batch);
      lk.lock();
      --c.in_flight;
      c.slot_busy[slot] = false;
      for (size_t k = 0; k < n_batch; ++k) batch[k]->state = ok ? CallRequest::kDone : CallRequest::kAlone;
      c.cv.notify_all();
      continue;
    }
    c.cv.wait(lk);
  }
}

int per_call(const fgkl_reads* reads, const fgkl_haplotypes* haps, const fgkl_config* cfg, bool pd, double* out, int64_t out_len,
             fgkl_stats* stats) {
  t_error.clear();
  if (!reads || !haps || !cfg || (out_len > 0 && !out) || out_len < 0) return set_error(FGKL_E_INVALID_ARGUMENT, "null argument");
  // ReadBatch::fetch (jni/src/lib.rs:104-133): the five read arrays must have one total length.
  const int64_t n = reads->bases_len;
  if (reads->quals_len != n || reads->ins_gop_len != n || reads->del_gop_len != n || reads->gcp_len != n)
    return set_error(FGKL_E_MISMATCHED_READ_ARRAYS, "read bases, qualities and penalties differ in total length");
  if (n < 0 || haps->bases_len < 0) return set_error(FGKL_E_INVALID_ARGUMENT, "negative array length");
  int rc;
  if ((rc = check_offsets(reads->offsets, reads->offsets_len, n, "read"))) return rc;
  if (pd && haps->flags_len != haps->bases_len)
    return set_error(FGKL_E_MISMATCHED_HAPLOTYPE_ARRAYS, "haplotype bases and PD flags differ in total length");
  if ((rc = check_offsets(haps->offsets, haps->offsets_len, haps->bases_len, "haplotype"))) return rc;
  const int64_t n_reads = reads->offsets_len - 1, n_haps = haps->offsets_len - 1;
  const int64_t expected = n_reads * n_haps;
  if (out_len != expected)
    return set_error(FGKL_E_OUTPUT_LENGTH,
                     "output has " + std::to_string(out_len) + " elements but reads x haplotypes is " + std::to_string(expected));
  // PairHmm::compute_log10_likelihoods validation order (lib.rs:278-290).
  for (int64_t r = 0; r < n_reads; ++r)
    if (reads->offsets[r + 1] == reads->offsets[r]) return set_error(FGKL_E_EMPTY_READ, "read " + std::to_string(r) + " has no bases");
  for (int64_t h = 0; h < n_haps; ++h)
    if (haps->offsets[h + 1] == haps->offsets[h])
      return set_error(FGKL_E_EMPTY_HAPLOTYPE, "haplotype " + std::to_string(h) + " has no bases");
  if (stats) std::memset(stats, 0, sizeof *stats);
  if (expected == 0) return FGKL_OK;
  CallRequest q;
  q.reads = reads;
  q.haps = haps;
  q.pd = pd;
  q.ec.double_precision = cfg->double_precision != 0;
  q.ec.double_fallback = cfg->double_fallback != 0;
  q.ec.share_suffixes = cfg->share_suffixes != 0;
  q.out = out;
  q.n_reads = n_reads;
  q.n_haps = n_haps;
  if (stats || g_max_in_flight.load(std::memory_order_relaxed) == 0) return run_alone(q, stats);
  return combined_call(q);
}

fgkl_config default_config(int32_t double_precision) {
  fgkl_config c;
  c.double_precision = double_precision;
  c.double_fallback = 1;
  c.share_suffixes = 1;
  return c;
}

void to_stats(const fgkl::BatchStats& bs, fgkl_stats* s) {
  s->fallback_pairs = bs.fallback_pairs;
  s->rescue_reads = bs.rescue_reads;
  s->nominal_cells = bs.nominal_cells;
  s->computed_cells = bs.computed_cells;
  s->forward_cells = bs.forward_cells;
  s->backward_cells = bs.backward_cells;
  s->prefix_only_cells = bs.prefix_only_cells;
  s->kernel_launches = bs.kernel_launches;
  s->host_plan_ms = bs.host_plan_ms;
  s->host_pack_ms = bs.host_pack_ms;
  s->host_upload_ms = bs.host_upload_ms;
  s->host_fetch_ms = bs.host_fetch_ms;
}


// Allocation-free entry: per-device state, set up by the first call on each device.
constexpr int kNoAllocMaxDevices = 64;
fgkl::NoAllocDevice g_noalloc[kNoAllocMaxDevices];
std::mutex g_noalloc_mutex;

int noalloc_device(fgkl::NoAllocDevice** out) {
  int d = -1;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0) return set_error(FGKL_E_NO_DEVICE, "no current CUDA device");
  if (d >= kNoAllocMaxDevices) return set_error(FGKL_E_NO_DEVICE, "device ordinal beyond the 64 the entry tracks");
  fgkl::NoAllocDevice& dev = g_noalloc[d];
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  // The array's address is looked up on every call (a host-side query): after a device reset the
  // primary context, and with it the array and the uploaded tables, are new, so the set-up is redone.
  char* scratch = nullptr;
  if (cudaError_t e = fgkl::noalloc_scratch_address(&scratch); e != cudaSuccess)
    return set_error(FGKL_E_CUDA, std::string("allocation-free entry: ") + cudaGetErrorString(e));
  if (!dev.ready || scratch != dev.scratch) {
    dev.ready = false;
    int major = 0, minor = 0, sms = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d) != cudaSuccess ||
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, d) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d) != cudaSuccess)
      return set_error(FGKL_E_NO_DEVICE, "cannot query the current CUDA device");
    if (major != 10 || minor != 0) return set_error(FGKL_E_NO_DEVICE, "the kernels are built for sm_100a");
    uint8_t codes[256];
    for (int b = 0; b < 256; ++b) codes[b] = static_cast<uint8_t>(b == 'N' ? fgkl::kCodeN : (b == fgkl::kCodeN ? 'N' : b));
    const fgkl::Tables& t = fgkl::tables();
    const cudaError_t e = fgkl::noalloc_setup(&dev, t.error_prob.data(), t.error_prob.size(), t.m2m.data(), t.m2m.size(), codes);
    if (e != cudaSuccess) return set_error(FGKL_E_CUDA, std::string("allocation-free setup: ") + cudaGetErrorString(e));
    dev.sms = sms;
    dev.ready = true;
  }
  *out = &dev;
  return FGKL_OK;
}

}  // namespace

struct fgkl_context {
  std::unique_ptr<fgkl::Engine> engine;
  std::unique_ptr<fgkl::AdjointEngine> adjoint;  // created on the first adjoint call
  std::unique_ptr<fgkl::SwEngine> sw;            // created on the first Smith-Waterman call
  // The executable graph of the last batch run. A new batch re-captures its launch sequence and
  // updates this graph in place when the topology allows: destroying an executable graph waits for
  // the whole device, which would stall a caller streaming batches through several contexts.
  cudaGraphExec_t graph = nullptr;
  bool graph_current = false;  // holds the prepared batch's launches
  bool prepared = false;
  bool adjoint_prepared = false;
  int device = 0;
  cudaStream_t stream = nullptr;
};

extern "C" {

int fgkl_pairhmm_compute(const fgkl_reads* reads, const fgkl_haplotypes* haps, int32_t double_precision, double* out,
                         int64_t out_len) {
  const fgkl_config c = default_config(double_precision);
  return per_call(reads, haps, &c, false, out, out_len, nullptr);
}

int fgkl_pairhmm_compute_config(const fgkl_reads* reads, const fgkl_haplotypes* haps, const fgkl_config* config, double* out,
                                int64_t out_len, fgkl_stats* stats) {
  return per_call(reads, haps, config, false, out, out_len, stats);
}

int fgkl_pdhmm_compute(const fgkl_reads* reads, const fgkl_haplotypes* haps, int32_t double_precision, double* out,
                       int64_t out_len) {
  const fgkl_config c = default_config(double_precision);
  return per_call(reads, haps, &c, true, out, out_len, nullptr);
}

int fgkl_pdhmm_compute_config(const fgkl_reads* reads, const fgkl_haplotypes* haps, const fgkl_config* config, double* out,
                              int64_t out_len, fgkl_stats* stats) {
  return per_call(reads, haps, config, true, out, out_len, stats);
}

int fgkl_set_call_combining(int32_t max_batches) {
  t_error.clear();
  if (max_batches < 0 || max_batches > kMaxSlots) return set_error(FGKL_E_INVALID_ARGUMENT, "max_batches must be 0 to 8");
  return g_max_in_flight.exchange(max_batches);
}

int fgkl_call_combining_stats(uint64_t* batches, uint64_t* requests) {
  t_error.clear();
  if (!batches || !requests) return set_error(FGKL_E_INVALID_ARGUMENT, "null argument");
  *batches = g_combined_batches.load(std::memory_order_relaxed);
  *requests = g_combined_requests.load(std::memory_order_relaxed);
  return FGKL_OK;
}

int64_t fgkl_set_allocation_limit(int64_t bytes) {
  t_error.clear();
  if (bytes < 0) return set_error(FGKL_E_INVALID_ARGUMENT, "the allocation limit must not be negative");
  return fgkl::set_allocation_limit(bytes);
}

const char* fgkl_backend(void) { return "cuda-sm100a"; }

const char* fgkl_last_error(void) { return t_error.c_str(); }

fgkl_context* fgkl_context_create(int32_t device, void* stream) {
  t_error.clear();
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    set_error(FGKL_E_NO_DEVICE, "no such CUDA device");
    return nullptr;
  }
  auto* ctx = new fgkl_context;
  ctx->engine = std::make_unique<fgkl::Engine>(device, static_cast<cudaStream_t>(stream));
  ctx->device = device;
  ctx->stream = ctx->engine->stream();
  return ctx;
}

void fgkl_context_destroy(fgkl_context* ctx) {
  if (!ctx) return;
  fgkl::DeviceGuard device_guard(ctx->device);
  if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
  delete ctx;
}

int fgkl_batch_prepare(fgkl_context* ctx, const fgkl_batch* b, const fgkl_config* config) {
  t_error.clear();
  if (!ctx || !b || !config) return set_error(FGKL_E_INVALID_ARGUMENT, "null argument");
  ctx->graph_current = false;
  fgkl::BatchInput in;
  in.num_regions = b->num_regions;
  in.region_reads = b->region_reads;
  in.region_haps = b->region_haps;
  in.bases = b->bases;
  in.quals = b->quals;
  in.ins = b->ins_gop;
  in.del = b->del_gop;
  in.gcp = b->gcp;
  in.read_off = b->read_offsets;
  in.hap_bases = b->hap_bases;
  in.hap_flags = b->hap_flags;
  in.hap_off = b->hap_offsets;
  fgkl::EngineConfig ec;
  ec.double_precision = config->double_precision != 0;
  ec.double_fallback = config->double_fallback != 0;
  ec.share_suffixes = config->share_suffixes != 0;
  const int rc = ctx->engine->prepare(in, ec);
  ctx->prepared = rc == FGKL_OK;
  return rc ? set_error(rc, ctx->engine->error()) : FGKL_OK;
}

int fgkl_batch_run(fgkl_context* ctx) {
  t_error.clear();
  if (!ctx || !ctx->prepared) return set_error(FGKL_E_INVALID_ARGUMENT, "no prepared batch");
  fgkl::DeviceGuard device_guard(ctx->device);  // capture and graph launch on the context's device
  fgkl::Engine& e = *ctx->engine;
  if (e.output_len() == 0) return FGKL_OK;
  cudaStream_t s = e.stream();
  int rc0 = e.begin_run();
  if (rc0) return set_error(rc0, e.error());
  if (e.profiling()) {
    // Timed launches: direct, so their events can be read back.
    const int rc = e.run();
    if (rc) return set_error(rc, e.error());
    return (rc0 = e.end_run()) ? set_error(rc0, e.error()) : FGKL_OK;
  }
  if (!ctx->graph_current) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return set_error(FGKL_E_CUDA, "cannot capture the launch sequence");
    const int rc = e.run();
    const cudaError_t end = cudaStreamEndCapture(s, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return set_error(rc, e.error());
    }
    if (end != cudaSuccess) return set_error(FGKL_E_CUDA, std::string("capture: ") + cudaGetErrorString(end));
    bool updated = false;
    if (ctx->graph) {
      cudaGraphExecUpdateResultInfo info;
      updated = cudaGraphExecUpdate(ctx->graph, g, &info) == cudaSuccess;
      if (!updated) {
        cudaGetLastError();  // a refused update leaves no sticky error; clear the last-error slot
        cudaGraphExecDestroy(ctx->graph);
        ctx->graph = nullptr;
      }
    }
    cudaError_t inst = cudaSuccess;
    if (!updated) inst = cudaGraphInstantiate(&ctx->graph, g, 0);
    cudaGraphDestroy(g);
    if (inst != cudaSuccess) {
      ctx->graph = nullptr;
      return set_error(FGKL_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(inst));
    }
    ctx->graph_current = true;
  }
  const cudaError_t err = cudaGraphLaunch(ctx->graph, s);
  if (err != cudaSuccess) return set_error(FGKL_E_CUDA, std::string("graph launch: ") + cudaGetErrorString(err));
  return (rc0 = e.end_run()) ? set_error(rc0, e.error()) : FGKL_OK;
}

int fgkl_batch_fetch(fgkl_context* ctx, double* out, int64_t out_len, fgkl_stats* stats) {
  t_error.clear();
  if (!ctx || !ctx->prepared) return set_error(FGKL_E_INVALID_ARGUMENT, "no prepared batch");
  fgkl::BatchStats bs;
  const int rc = ctx->engine->fetch(out, out_len, &bs);
  if (rc) return set_error(rc, ctx->engine->error());
  if (stats) to_stats(bs, stats);
  return FGKL_OK;
}

int fgkl_batch_compute(fgkl_context* ctx, const fgkl_batch* batch, const fgkl_config* config, double* out, int64_t out_len,
                       fgkl_stats* stats) {
  int rc = fgkl_batch_prepare(ctx, batch, config);
  if (rc) return rc;
  if (out_len != ctx->engine->output_len())
    return set_error(FGKL_E_OUTPUT_LENGTH, "output has " + std::to_string(out_len) + " elements but the batch produces " +
                                               std::to_string(ctx->engine->output_len()));
  if ((rc = fgkl_batch_run(ctx))) return rc;
  return fgkl_batch_fetch(ctx, out, out_len, stats);
}

int64_t fgkl_batch_output_len(const fgkl_context* ctx) { return ctx && ctx->prepared ? ctx->engine->output_len() : 0; }

int fgkl_context_set_tuning(fgkl_context* ctx, const fgkl_tuning* t) {
  t_error.clear();
  if (!ctx || !t) return set_error(FGKL_E_INVALID_ARGUMENT, "null argument");
  if (t->streams < 1 || t->streams > 8 || t->grid_percent < 10 || t->grid_percent > 100 ||
      (t->reads_per_warp != 1 && t->reads_per_warp != 2) || (t->rows_extra != 0 && t->rows_extra != 1) ||
      (t->warps_per_block != 1 && t->warps_per_block != 2 && t->warps_per_block != 4))
    return set_error(FGKL_E_INVALID_ARGUMENT,
                     "streams must be 1-8, grid_percent 10-100, reads_per_warp 1 or 2, rows_extra 0 or 1 and "
                     "warps_per_block 1, 2 or 4");
  ctx->engine->set_tuning(fgkl::Engine::Tuning{t->streams, t->grid_percent, t->reads_per_warp, t->rows_extra, t->warps_per_block});
  ctx->graph_current = false;
  return FGKL_OK;
}

int fgkl_context_get_tuning(const fgkl_context* ctx, fgkl_tuning* t) {
  t_error.clear();
  if (!ctx || !t) return set_error(FGKL_E_INVALID_ARGUMENT, "null argument");
  const auto& k = ctx->engine->tuning();
  t->streams = k.streams;
  t->grid_percent = k.grid_percent;
  t->reads_per_warp = k.reads_per_warp;
  t->rows_extra = k.rows_extra;
  t->warps_per_block = k.warps_per_block;
  t->ms = 0.0;
  return FGKL_OK;
}

int fgkl_context_autotune(fgkl_context* ctx, const fgkl_batch* batch, const fgkl_config* config, int32_t repeats,
                          fgkl_tuning* chosen, fgkl_tuning* tried, int32_t tried_cap, int32_t* n_tried) {
  t_error.clear();
  if (!ctx || !batch || !config) return set_error(FGKL_E_INVALID_ARGUMENT, "null argument");
  if (repeats < 1 || tried_cap < 0) return set_error(FGKL_E_INVALID_ARGUMENT, "repeats must be >= 1");
  fgkl::Engine& e = *ctx->engine;
  const bool was_profiling = e.profiling();
  const fgkl::Engine::Tuning before = e.tuning();
  e.set_profiling(false);
  // Candidates: every streams x grid pair with two reads per warp, then, for an FP32 PD-HMM batch,
  // one read per warp at 4 and 8 streams with full grids; then the tile shapes around the fastest.
  std::vector<fgkl::Engine::Tuning> cands;
  for (int gp : {100, 90, 75, 60})
    for (int st : {1, 2, 4, 8}) cands.push_back(fgkl::Engine::Tuning{st, gp, 2, 0, 4});
  const bool fp32_pd = batch->hap_flags && !config->double_precision;
  if (fp32_pd)
    for (int st : {4, 8}) cands.push_back(fgkl::Engine::Tuning{st, 100, 1, 0, 4});
  fgkl::Engine::Tuning best{};
  double best_ms = -1.0;
  int n = 0, rc = FGKL_OK;
  auto try_one = [&](const fgkl::Engine::Tuning& c) {
    e.set_tuning(c);
    if ((rc = fgkl_batch_prepare(ctx, batch, config))) return;
    double ms = 0.0;
    if ((rc = e.time_run(repeats, &ms))) {
      rc = set_error(rc, e.error());
      return;
    }
    if (tried && n < tried_cap) tried[n] = fgkl_tuning{c.streams, c.grid_percent, c.reads_per_warp, c.rows_extra, c.warps_per_block, ms};
    ++n;
    if (best_ms < 0 || ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  };
  for (const auto& c : cands) {
    try_one(c);
    if (rc) break;
  }
  if (!rc && !config->double_precision) {
    const fgkl::Engine::Tuning base = best;
    std::vector<fgkl::Engine::Tuning> shapes;
    for (int w : {1, 2}) shapes.push_back(fgkl::Engine::Tuning{base.streams, base.grid_percent, base.reads_per_warp, 0, w});
    if (!batch->hap_flags) shapes.push_back(fgkl::Engine::Tuning{base.streams, base.grid_percent, base.reads_per_warp, 1, 4});
    for (const auto& c : shapes) {
      try_one(c);
      if (rc) break;
    }
  }
  e.set_profiling(was_profiling);
  if (n_tried) *n_tried = n;
  if (rc) {
    // A failed search leaves the context as it found it (its batch is no longer prepared).
    e.set_tuning(before);
    ctx->prepared = false;
    ctx->graph_current = false;
    return rc;
  }
  e.set_tuning(best);
  if ((rc = fgkl_batch_prepare(ctx, batch, config))) return rc;
  if (chosen) *chosen = fgkl_tuning{best.streams, best.grid_percent, best.reads_per_warp, best.rows_extra, best.warps_per_block, best_ms};
  return FGKL_OK;
}

// ---------------------------------------------------------------------------------------------
// Synthetic workloads and planner diagnostics (test and benchmark support).
// ---------------------------------------------------------------------------------------------

struct fgkl_synth {
  fgkl::SynthBatch batch;
};

fgkl_synth* fgkl_synth_config(int32_t which, uint64_t seed, int32_t regions, int32_t threads) {
  try {
    auto* s = new fgkl_synth;
    s->batch = fgkl::config_batch(which, seed, regions, threads);
    return s;
  } catch (const std::exception& e) {
    set_error(FGKL_E_INVALID_ARGUMENT, e.what());
    return nullptr;
  }
}

fgkl_synth* fgkl_synth_reference_region(uint64_t seed, int64_t reads, int64_t read_len, int64_t haps, int64_t hap_len, int32_t pd) {
  auto* s = new fgkl_synth;
  const auto r = pd ? fgkl::reference_pd_region(seed, reads, read_len, haps, hap_len)
                    : fgkl::reference_region(seed, reads, read_len, haps, hap_len);
  s->batch.append(r);
  s->batch.pd = pd != 0;
  return s;
}

void fgkl_synth_view(const fgkl_synth* s, fgkl_batch* out, int64_t sizes[4]) {
  const auto& b = s->batch;
  out->num_regions = static_cast<int32_t>(b.region_reads.size());
  out->region_reads = b.region_reads.data();
  out->region_haps = b.region_haps.data();
  out->bases = b.bases.data();
  out->quals = b.quals.data();
  out->ins_gop = b.ins.data();
  out->del_gop = b.del.data();
  out->gcp = b.gcp.data();
  out->read_offsets = b.read_off.data();
  out->hap_bases = b.hap_bases.data();
  out->hap_flags = b.pd ? b.hap_flags.data() : nullptr;
  out->hap_offsets = b.hap_off.data();
  sizes[0] = static_cast<int64_t>(b.read_off.size()) - 1;
  sizes[1] = static_cast<int64_t>(b.bases.size());
  sizes[2] = static_cast<int64_t>(b.hap_off.size()) - 1;
  sizes[3] = static_cast<int64_t>(b.hap_bases.size());
}

void fgkl_synth_free(fgkl_synth* s) { delete s; }

// Sorted order, LCP, duplicate flags, cuts, node count and SharedColumns of one haplotype set;
// sweeps are reported through fgkl_plan_sweeps. Arrays are num_haps long.
int fgkl_plan_describe(const uint8_t* hap_bases, const int32_t* hap_offsets, int32_t num_haps, int32_t share_suffixes,
                       int32_t* order, int32_t* lcp, uint8_t* dup, int32_t* cut_column, int32_t* cut_node, int32_t* num_sweeps,
                       int32_t* num_nodes, uint64_t columns[3]) {
  try {
    std::vector<fgkl::HapView> views(static_cast<size_t>(num_haps));
    for (int h = 0; h < num_haps; ++h) views[h] = fgkl::HapView{hap_bases + hap_offsets[h], hap_offsets[h + 1] - hap_offsets[h]};
    const auto s = fgkl::SortedHaps::make(views, share_suffixes != 0);
    for (int k = 0; k < num_haps; ++k) {
      order[k] = s.order[k];
      lcp[k] = s.lcp[k];
      dup[k] = s.dup[k];
      cut_column[k] = s.plan.cuts[k].column;
      cut_node[k] = s.plan.cuts[k].node;
    }
    *num_sweeps = static_cast<int32_t>(s.plan.sweeps.size());
    *num_nodes = s.plan.nodes;
    const auto c = s.columns();
    columns[0] = c.prefix_only;
    columns[1] = c.forward;
    columns[2] = c.backward;
    return FGKL_OK;
  } catch (const std::exception& e) {
    return set_error(FGKL_E_INVALID_ARGUMENT, e.what());
  }
}

int fgkl_plan_region_cells(const fgkl_batch* b, const fgkl_config* config, uint64_t* cells) {
  t_error.clear();
  if (!b || !config || (b->num_regions > 0 && (!cells || !b->region_reads || !b->region_haps || !b->read_offsets || !b->hap_offsets)))
    return set_error(FGKL_E_INVALID_ARGUMENT, "null argument");
  try {
    fgkl::BatchInput in;
    in.num_regions = b->num_regions;
    in.region_reads = b->region_reads;
    in.region_haps = b->region_haps;
    in.bases = b->bases;
    in.quals = b->quals;
    in.ins = b->ins_gop;
    in.del = b->del_gop;
    in.gcp = b->gcp;
    in.read_off = b->read_offsets;
    in.hap_bases = b->hap_bases;
    in.hap_flags = b->hap_flags;
    in.hap_off = b->hap_offsets;
    fgkl::EngineConfig ec;
    ec.double_precision = config->double_precision != 0;
    ec.double_fallback = config->double_fallback != 0;
    ec.share_suffixes = config->share_suffixes != 0;
    std::string err;
    const int rc = fgkl::plan_region_cells(in, ec, cells, &err);
    return rc ? set_error(rc, err) : FGKL_OK;
  } catch (const std::bad_alloc&) {
    return set_error(FGKL_E_OUT_OF_MEMORY, "host memory allocation failed");
  }
}

// The sweeps of a plan: per sweep (hap, resume, need, start, first write, write count) in
// `sweeps` (6 ints each) and the (depth, node) writes in `writes` (2 ints each).
int fgkl_plan_sweeps(const uint8_t* hap_bases, const int32_t* hap_offsets, int32_t num_haps, int32_t* sweeps, int32_t max_sweeps,
                     int32_t* writes, int32_t max_writes) {
  try {
    std::vector<fgkl::HapView> views(static_cast<size_t>(num_haps));
    for (int h = 0; h < num_haps; ++h) views[h] = fgkl::HapView{hap_bases + hap_offsets[h], hap_offsets[h + 1] - hap_offsets[h]};
    const auto s = fgkl::SortedHaps::make(views, true);
    if (static_cast<int32_t>(s.plan.sweeps.size()) > max_sweeps) return set_error(FGKL_E_INVALID_ARGUMENT, "too many sweeps");
    int w = 0;
    for (size_t i = 0; i < s.plan.sweeps.size(); ++i) {
      const auto& sw = s.plan.sweeps[i];
      int32_t* o = sweeps + 6 * i;
      o[0] = sw.hap;
      o[1] = sw.resume;
      o[2] = sw.need;
      o[3] = sw.start;
      o[4] = w;
      o[5] = static_cast<int32_t>(sw.writes.size());
      for (const auto& wr : sw.writes) {
        if (w >= max_writes) return set_error(FGKL_E_INVALID_ARGUMENT, "too many writes");
        writes[2 * w] = wr.first;
        writes[2 * w + 1] = wr.second;
        ++w;
      }
    }
    return FGKL_OK;
  } catch (const std::exception& e) {
    return set_error(FGKL_E_INVALID_ARGUMENT, e.what());
  }
}

int fgkl_context_profile(fgkl_context* ctx, int32_t on) {
  t_error.clear();
  if (!ctx) return set_error(FGKL_E_INVALID_ARGUMENT, "null context");
  ctx->engine->set_profiling(on != 0);
  return FGKL_OK;
}

int fgkl_batch_launch_profile(fgkl_context* ctx, fgkl_launch_profile* out, int32_t max, int32_t* count) {
  t_error.clear();
  if (!ctx || !count || (max > 0 && !out)) return set_error(FGKL_E_INVALID_ARGUMENT, "null argument");
  std::vector<fgkl::Engine::BinProfile> bins;
  const int rc = ctx->engine->bin_profile(&bins);
  if (rc) return set_error(rc, ctx->engine->error());
  *count = static_cast<int32_t>(bins.size());
  for (int32_t i = 0; i < max && i < *count; ++i) {
    const auto& b = bins[i];
    out[i] = fgkl_launch_profile{b.kind, b.rows, b.n_tasks, b.blocks, b.rescue, b.fwd_cells, b.bwd_cells, b.ms};
  }
  return FGKL_OK;
}

int fgkl_adjoint_prepare(fgkl_context* ctx, const fgkl_adjoint_batch* b, int32_t double_precision) {
  t_error.clear();
  if (!ctx || !b) return set_error(FGKL_E_INVALID_ARGUMENT, "null argument");
  if (!ctx->adjoint) ctx->adjoint = std::make_unique<fgkl::AdjointEngine>(ctx->device, ctx->stream);
  fgkl::AdjointInput in;
  in.num_regions = b->num_regions;
  in.region_reads = b->region_reads;
  in.region_haps = b->region_haps;
  in.bases = b->bases;
  in.read_off = b->read_offsets;
  in.d_ins = b->gap_open_ins;
  in.d_del = b->gap_open_del;
  in.eps = b->gap_continuation;
  in.err = b->base_error;
  in.hap_bases = b->hap_bases;
  in.hap_off = b->hap_offsets;
  const int rc = ctx->adjoint->prepare(in, double_precision != 0);
  ctx->adjoint_prepared = rc == FGKL_OK;
  return rc ? set_error(rc, ctx->adjoint->error()) : FGKL_OK;
}

int fgkl_adjoint_run(fgkl_context* ctx, uint64_t* launches) {
  t_error.clear();
  if (!ctx || !ctx->adjoint || !ctx->adjoint_prepared) return set_error(FGKL_E_INVALID_ARGUMENT, "no prepared adjoint batch");
  const int rc = ctx->adjoint->run();
  if (launches) *launches = ctx->adjoint->launches();
  return rc ? set_error(rc, ctx->adjoint->error()) : FGKL_OK;
}

int fgkl_adjoint_fetch(fgkl_context* ctx, double* log10_out, int64_t out_len, double* grad_gap_open_ins,
                       double* grad_gap_open_del, double* grad_gap_continuation, double* grad_base_error, int64_t grad_len,
                       uint64_t* fp64_reads) {
  t_error.clear();
  if (!ctx || !ctx->adjoint || !ctx->adjoint_prepared) return set_error(FGKL_E_INVALID_ARGUMENT, "no prepared adjoint batch");
  if ((out_len > 0 && !log10_out) || (grad_len > 0 && (!grad_gap_open_ins || !grad_gap_open_del || !grad_gap_continuation || !grad_base_error)))
    return set_error(FGKL_E_INVALID_ARGUMENT, "null output");
  const int rc = ctx->adjoint->fetch(log10_out, out_len, grad_gap_open_ins, grad_gap_open_del, grad_gap_continuation, grad_base_error,
                                     grad_len, fp64_reads);
  return rc ? set_error(rc, ctx->adjoint->error()) : FGKL_OK;
}

int fgkl_adjoint_compute(fgkl_context* ctx, const fgkl_adjoint_batch* b, int32_t double_precision, double* log10_out,
                         int64_t out_len, double* grad_gap_open_ins, double* grad_gap_open_del, double* grad_gap_continuation,
                         double* grad_base_error, int64_t grad_len, uint64_t* fp64_reads) {
  int rc = fgkl_adjoint_prepare(ctx, b, double_precision);
  if (rc) return rc;
  if (out_len != ctx->adjoint->output_len() || grad_len != ctx->adjoint->grad_len())
    return set_error(FGKL_E_OUTPUT_LENGTH, "outputs must hold reads x haplotypes likelihoods and one gradient per read position");
  if ((rc = fgkl_adjoint_run(ctx, nullptr))) return rc;
  return fgkl_adjoint_fetch(ctx, log10_out, out_len, grad_gap_open_ins, grad_gap_open_del, grad_gap_continuation, grad_base_error,
                            grad_len, fp64_reads);
}

int64_t fgkl_adjoint_output_len(const fgkl_context* ctx) { return ctx && ctx->adjoint ? ctx->adjoint->output_len() : 0; }
int64_t fgkl_adjoint_grad_len(const fgkl_context* ctx) { return ctx && ctx->adjoint ? ctx->adjoint->grad_len() : 0; }

int fgkl_pd_row_states(const uint8_t* flags, int32_t len, int32_t start_state, uint8_t* states) {
  if (len < 0 || (len > 0 && (!flags || !states)) || start_state < 0 || start_state > 2)
    return set_error(FGKL_E_INVALID_ARGUMENT, "bad PD row");
  return fgkl::pd_row_states(flags, len, static_cast<uint8_t>(start_state), states);
}

int fgkl_pd_plan_describe(const uint8_t* hap_bases, const uint8_t* hap_flags, const int32_t* hap_offsets, int32_t num_haps,
                          int32_t* order, int32_t* lcp, uint8_t* dup, uint8_t* end_state, int32_t* num_codes) {
  try {
    std::vector<fgkl::HapView> views(static_cast<size_t>(num_haps));
    std::vector<const uint8_t*> flags(static_cast<size_t>(num_haps));
    for (int h = 0; h < num_haps; ++h) {
      views[h] = fgkl::HapView{hap_bases + hap_offsets[h], hap_offsets[h + 1] - hap_offsets[h]};
      flags[h] = hap_flags + hap_offsets[h];
    }
    const auto s = fgkl::SortedHaps::make_pd(views, flags);
    for (int k = 0; k < num_haps; ++k) {
      order[k] = s.order[k];
      lcp[k] = s.lcp[k];
      dup[k] = s.dup[k];
      end_state[k] = s.end_state[k];
    }
    *num_codes = s.num_codes();
    return FGKL_OK;
  } catch (const std::exception& e) {
    return set_error(FGKL_E_INVALID_ARGUMENT, e.what());
  }
}

int fgkl_pd_match_accepts(uint8_t base, uint8_t flag, uint8_t read_base) {
  return fgkl::MatchSet::of(base, flag).accepts(read_base) ? 1 : 0;
}

int fgkl_sw_align(const uint8_t* ref, int64_t ref_len, const uint8_t* alt, int64_t alt_len, const fgkl_sw_params* params,
                  int32_t strategy, char* cigar, int64_t cigar_cap, int32_t* offset) try {
  t_error.clear();
  if (!params || !cigar || !offset || ref_len < 0 || alt_len < 0 || (ref_len > 0 && !ref) || (alt_len > 0 && !alt))
    return set_error(FGKL_E_INVALID_ARGUMENT, "null argument or negative length");
  if (strategy < FGKL_SW_SOFTCLIP || strategy > FGKL_SW_IGNORE)
    return set_error(FGKL_E_INVALID_ARGUMENT, "unknown overhang strategy code " + std::to_string(strategy));
  if (ref_len == 0 || alt_len == 0) return set_error(FGKL_E_EMPTY_SEQUENCE, "Smith-Waterman needs non-empty sequences");
  int rc;
  fgkl::SwEngine* e = thread_sw(&rc);
  if (!e) return rc;
  const int64_t roff[2] = {0, ref_len}, aoff[2] = {0, alt_len};
  fgkl::SwBatch in{1, ref, roff, alt, aoff};
  std::vector<uint32_t> elems(static_cast<size_t>(fgkl::sw_cigar_slot(ref_len, alt_len)));
  int32_t count = 0, off = 0;
  rc = e->align(in, fgkl::SwScores{params->match_value, params->mismatch_penalty, params->gap_open_penalty, params->gap_extend_penalty},
                strategy, elems.data(), static_cast<int64_t>(elems.size()), &count, &off);
  if (rc) return set_error(rc, e->error());
  std::string text;
  static const char kOps[] = {'M', 'I', 'D', 'N', 'S'};
  for (int32_t i = 0; i < count; ++i) {
    text += std::to_string(elems[i] >> 4);
    text += kOps[elems[i] & 0xF];
  }
  if (static_cast<int64_t>(text.size()) + 1 > cigar_cap)
    return set_error(FGKL_E_OUTPUT_LENGTH, "the CIGAR string needs " + std::to_string(text.size() + 1) + " bytes");
  std::memcpy(cigar, text.c_str(), text.size() + 1);
  *offset = off;
  return FGKL_OK;
} catch (const std::bad_alloc&) {
  return set_error(FGKL_E_OUT_OF_MEMORY, "host memory allocation failed");
}

int64_t fgkl_sw_cigar_capacity(const fgkl_sw_batch* b) {
  if (!b || b->num_pairs < 0 || (b->num_pairs > 0 && (!b->ref_offsets || !b->alt_offsets))) return 0;
  return b->ref_offsets[b->num_pairs] + b->alt_offsets[b->num_pairs] + 2 * b->num_pairs;
}

int fgkl_sw_align_batch(fgkl_context* ctx, const fgkl_sw_batch* b, const fgkl_sw_params* params, int32_t strategy, uint32_t* cigar,
                        int64_t cigar_len, int32_t* counts, int32_t* offsets) try {
  t_error.clear();
  if (!ctx || !b || !params) return set_error(FGKL_E_INVALID_ARGUMENT, "null argument");
  if (!ctx->sw) ctx->sw = std::make_unique<fgkl::SwEngine>(ctx->device, ctx->stream);
  fgkl::SwBatch in{b->num_pairs, b->ref_bases, b->ref_offsets, b->alt_bases, b->alt_offsets};
  const int rc = ctx->sw->align(in, fgkl::SwScores{params->match_value, params->mismatch_penalty, params->gap_open_penalty,
                                                   params->gap_extend_penalty},
                                strategy, cigar, cigar_len, counts, offsets);
  return rc ? set_error(rc, ctx->sw->error()) : FGKL_OK;
} catch (const std::bad_alloc&) {
  return set_error(FGKL_E_OUT_OF_MEMORY, "host memory allocation failed");
}

int fgkl_sw_last_kernel_ms(fgkl_context* ctx, float* ms) {
  t_error.clear();
  if (!ctx || !ms) return set_error(FGKL_E_INVALID_ARGUMENT, "null argument");
  if (!ctx->sw || ctx->sw->last_kernel_ms() < 0.f) return set_error(FGKL_E_INVALID_ARGUMENT, "no Smith-Waterman batch has run on this context");
  *ms = ctx->sw->last_kernel_ms();
  return FGKL_OK;
}

int fgkl_pairhmm_compute_device_noalloc(const fgkl_device_region* region, double* out, void* stream) {
  t_error.clear();
  if (!region) return set_error(FGKL_E_INVALID_ARGUMENT, "null region");
  const int64_t n_reads = region->num_reads, n_haps = region->num_haplotypes;
  if (n_reads < 0 || n_haps < 0) return set_error(FGKL_E_INVALID_ARGUMENT, "negative read or haplotype count");
  const int64_t pairs = n_reads * n_haps;
  if (pairs > FGKL_NOALLOC_MAX_PAIRS)
    return set_error(FGKL_E_INVALID_ARGUMENT, "the allocation-free entry takes at most 2^31 - 1 pairs per call; split the region");
  if (region->max_read_len < 1 || region->max_read_len > FGKL_NOALLOC_MAX_READ_LEN)
    return set_error(FGKL_E_UNSUPPORTED, "max_read_len must lie in 1..620 for the allocation-free entry");
  if (pairs == 0) return FGKL_OK;
  if (!out || !region->bases || !region->quals || !region->ins_quals || !region->del_quals || !region->gcp ||
      !region->read_offsets || !region->hap_bases || !region->hap_offsets)
    return set_error(FGKL_E_INVALID_ARGUMENT, "null device array");
  fgkl::NoAllocDevice* dev = nullptr;
  int rc;
  if ((rc = noalloc_device(&dev)) != FGKL_OK) return rc;
  const int rows = fgkl::noalloc_rows(region->max_read_len);
  // A persistent grid: the device's resident blocks, or fewer when the pairs do not fill it, and
  // never more warps than the file-scope scratch holds.
  const int64_t warps_fit = static_cast<int64_t>((dev->scratch_bytes - dev->header_bytes) / dev->per_warp_bytes);
  int64_t blocks = static_cast<int64_t>(dev->blocks_per_sm[rows]) * dev->sms;
  blocks = std::min<int64_t>(blocks, (pairs + 3) / 4);
  blocks = std::min<int64_t>(blocks, warps_fit / 4);
  fgkl::NoAllocCall c{region->bases, region->quals, region->ins_quals, region->del_quals, region->gcp, region->read_offsets,
                      region->hap_bases, region->hap_offsets, static_cast<int>(n_reads), static_cast<int>(n_haps), out};
  const cudaError_t e = fgkl::noalloc_launch(*dev, c, rows, static_cast<int>(blocks), static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return set_error(FGKL_E_CUDA, std::string("allocation-free launch: ") + cudaGetErrorString(e));
  return FGKL_OK;
}

}  // extern "C"
