// api.cu -- C ABI of libemmahydro: device context, resident tree, level
// schedule (host-driven or a captured CUDA graph) and the drop-in entries with
// the reference's names.
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <fcntl.h>
#include <pthread.h>
#include <unistd.h>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include "emma_hydro.h"
#ifdef EMMA_WGRAV
#include "emma_hydro_grav.h"
#endif
#include "mirror.h"
#include "plan_types.h"
#include "schedule.h"

namespace emma {
cudaError_t launch_level_fp64(const BatchArgs &a, unsigned shapes, int nsm, int ctas_per_sm, cudaStream_t s,
                              int *occupancy);
cudaError_t launch_level_f32(const BatchArgs &a, unsigned shapes, int nsm, int ctas_per_sm, cudaStream_t s,
                             int *occupancy);
cudaError_t launch_column_f32(const ColumnArgs &a, cudaStream_t s);
cudaError_t launch_step_f32(const StepArgs &a, unsigned variant, int groups, int nsm, cudaStream_t s, int *grid,
                            int *threads);
cudaError_t launch_step_fp64(const StepArgs &a, unsigned variant, int groups, int nsm, cudaStream_t s, int *grid,
                             int *threads);
int step_groups_f32(unsigned variant, int groups);
int step_groups_fp64(unsigned variant, int groups);
cudaError_t launch_cfl(const LevelArgs *lv, int slot, long long n8, const int *gate, unsigned long long *out, int nsm,
                       cudaStream_t s);
cudaError_t launch_interp(const LevelArgs *lv, int slot, long long nv, const int *gate, int nsm, cudaStream_t s,
                          bool grav);
cudaError_t launch_dropin_base(const double *wb, double *base, long long n8, const double *exc, long long nexc, int nsm,
                               cudaStream_t s, int np, int rec);
bool resident_level(struct OCT **firstoct, int level, const HostLevel **h, const double **W, const uint8_t **split,
                    cudaStream_t *stream, int *nsm);
void release_dump_staging();
}  // namespace emma

using namespace emma;

namespace {

constexpr double kG = 5. / 3.;
constexpr long long kWaitLimit = 1LL << 24;  // ~1 s of __nanosleep(64) polls
constexpr unsigned kMaxHostThreads = 64;      // host threads of the drop-in's parallel passes
constexpr unsigned kDefaultHostThreads = 32;  // without EMMA_HYDRO_HOST_THREADS

struct DevLevel {
  int L = 0, noct = 0, ntiles = 0;
  long long n8 = 0, leaf = 0;
  double *W0 = nullptr, *W1 = nullptr, *C = nullptr, *B = nullptr;
  double *WB = nullptr;  // drop-in levels: one allocation of W0 (5 planes), E (, dX), then B (d,u,v,w,p,E (, dX))
  double *X = nullptr, *Xn = nullptr;  // tracer builds: dX of the level's field and the new dX
  uint8_t *split = nullptr;
  int *child = nullptr;
  TileDesc *tiles = nullptr;
  uint32_t *keys = nullptr;
  int *work = nullptr;  // (L << 24) | tile for every tile of the level
  int *vcell = nullptr;    // transmissive or gravity build: interpolated coarser cells and their slope neighbours
  double *Wv = nullptr;    // their 8 interpolated (gravity build: injected) sub-cells
  double *F = nullptr;     // gravity build: acceleration planes fx,fy,fz of the level's cells
  double *Fv = nullptr;    // gravity build: interpolated accelerations of the listed coarser cells
  uint8_t *az = nullptr;   // dual energy: per cell, a split cell whose stored sound speed is 0
  // column kernel (column_kernel.cuh): a complete periodic level without split cells of a
  // resident plain-variant tree has the oct index of every oct position; col_nz is the
  // planes per work item the autotuner chose (0: the brick kernel was faster)
  int *octidx = nullptr;
  int col_n = 0;  // octs per side, 0 when the level is not eligible
  // device-side refinement (refine_impl.cuh, resident levels): the oct of this level
  // across each face of every oct (-1: none), and the refinement mark of every cell
  int *nb6 = nullptr;
  int *marks = nullptr;
  int col_nz = 0;
  double col_sweep_ms[6] = {};  // planes per item 2, 4, 8, 16, 32, 64 (0 = not tried)
  int col_xs = 0;               // the autotuner's x sweep: 1 warp shuffles, 0 shared memory
  double col_xs_ms[2] = {};     // its times of the two at col_nz (0 = not timed)
  int col_bal = 0;              // the autotuner's work split: 1 balanced runs, 0 items
  double col_bal_ms[2] = {};    // its times of the two (0 = not timed)
  long long nv = 0;
  int shape = 0;        // brick shape of the plan (kShapes)
  int ctas = 0;         // CTAs per SM of its launches (0: the occupancy limit)
  // autotuner record: chosen shape/CTAs and the swept times (ms per launch, 0 = not run)
  bool tuned = false;
  double sweep_ms[kNumShapes][4] = {};
};

struct TimedLaunch {
  cudaEvent_t a, b;
  long long cells;
  int level;  // the resident level a single-level launch advances, -1 for a batched launch
};

struct Tree {
  bool valid = false;
  int lcoarse = 0, lmax = 0;
  HostTree host;
  std::vector<DevLevel> lev;
  LevelArgs *d_lv = nullptr;  // kMaxLevels slots, indexed by level
};

struct Ctx {
  bool ready = false;
  EmmaHydroOptions opt;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  int nsm = 148;
  unsigned *d_status = nullptr;
  long long wait_limit = kWaitLimit;  // polls of a bounded device-side wait
  unsigned *d_done = nullptr;    // kMaxLevels completion counters
  SchedState *d_S = nullptr;
  SchedState *h_S = nullptr;     // pinned staging of the schedule state
  StepCtl *d_ctl = nullptr;      // control block of the fused coarse step
  StepJobRecord *d_jobt = nullptr;  // release times of its jobs (kStepJobLog)
  bool c_dirty = false;          // a level's corrections may hold values (read or not) that the
                                 // fused step, which clears what it reads, would not expect:
                                 // after separate launches; cleared before a fused step
  int step_grid = 0, step_threads = 0;  // CTAs and threads per CTA of the last fused step launch
  // coarse-step mode of the resident tree's subcycled graph: -2 not decided yet,
  // 0 the level schedule's separate launches, k > 0 the fused kernel with k tile
  // groups per CTA; the autotuner's times (ms per step; [0] separate launches,
  // [k] k groups, 0 = not tried) and the nsub and precision it timed
  int step_groups = -2;
  double step_sweep[5] = {};
  int step_tuned_nsub = -1, step_tuned_prec = -1;
  unsigned status = 0;
  std::string last_error;
  Tree res;                      // resident tree
  struct OCT **res_first = nullptr;  // the firstoct array it was uploaded from
  int *d_work_all = nullptr;     // batched work list, finest level first
  int nwork_all = 0;
  cudaGraphExec_t graph = nullptr;
  int graph_nsub = -1, graph_prec = -1, graph_col = -2, graph_colx = -2, graph_colb = -2, graph_groups = -3;
  bool graph_is_fused = false;   // the captured coarse step is one fused kernel
  int graph_kernels = 0;         // kernel nodes of the captured coarse step
  // drop-in cache: one mirror of levels L-1..L+1 per advanced level L, so that a
  // driver cycling through its levels does not rebuild one on every call
  struct DropCache {
    struct OCT **first = nullptr;
    std::vector<unsigned long long> sig;
    Tree t;
  };
  DropCache drop[kMaxLevels];
  std::vector<struct OCT *> lists[kMaxLevels];  // last walk of each level's oct list
  uintptr_t list_lo[kMaxLevels] = {}, list_hi[kMaxLevels] = {};  // lowest, highest oct address in it
  std::vector<struct OCT *> list_tmp;
  // pinned staging
  double *pin = nullptr;
  size_t pin_bytes = 0;
  // counters and timing
  long long updates = 0;
  long long kernel_launches = 0;
  long long h2d_bytes = 0, d2h_bytes = 0;  // host<->device state copies
  double dropin_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // phases of the last drop-in call
  std::vector<cudaEvent_t> range_ev;        // per host thread and sub-range of a drop-in download
  std::vector<double> exc[kMaxHostThreads];  // per host thread: drop-in cells whose fieldnew differs
  double *pin_exc = nullptr;                // their pinned staging
  size_t pin_exc_bytes = 0;
  double *d_exc = nullptr;                  // and device copy
  size_t d_exc_bytes = 0;
  bool timing = true;
  std::vector<TimedLaunch> launches;
  std::vector<cudaEvent_t> free_events;
};

Ctx g;
using Clock = std::chrono::steady_clock;

// The drop-in entries of a library built for the reference's -DWGRAV cell layout
// (libemmahydro_grav.so) run the gravity-coupled advance: the cells carry f[3].
#ifdef EMMA_WGRAV
constexpr int kDropinGrav = 1;
#else
constexpr int kDropinGrav = 0;
#endif
// ... and those of a library built for its -DWRADHYD layout (libemmahydro_rh.so)
// advance the ionised density dX too, and with -DHELIUM (libemmahydro_he.so) the
// helium densities dXHE, dXXHE as well (in the resident mode planes 6.. of every
// level state).  kDropinTracer: the number of tracers.
#if defined(EMMA_HELIUM)
constexpr int kDropinTracer = 3;
#elif defined(EMMA_WRADHYD)
constexpr int kDropinTracer = 1;
#else
constexpr int kDropinTracer = 0;
#endif
// the kernel variant of the tracer builds
constexpr unsigned kLaunchTracers = kDropinTracer == 3 ? kLaunchHelium : (kDropinTracer == 1 ? kLaunchTracer : 0u);
#ifdef EMMA_WRADHYD
// tracer t of a state: dX, then (-DHELIUM) dXHE, dXXHE, which follow it in struct Wtype
inline double &tracer(struct Wtype &W, int t) { return (&W.dX)[t]; }
inline double tracer(const struct Wtype &W, int t) { return (&W.dX)[t]; }
#endif

// Planes of a correction buffer: d, du, dv, dw, E, with dual energy eint, in a
// tracer build the tracers (planes kXPlane..; the tracer builds have no dual energy).
inline long long cplanes() { return (g.opt.dual_energy ? 6 : 5) + kDropinTracer; }
// Planes of a drop-in level's `field` upload and of its base fieldnew: d,u,v,w,p,E (+ tracers)
constexpr int kFieldPlanes = 6 + kDropinTracer;
// doubles per record of a drop-in cell whose fieldnew differs: the cell, then the
// kFieldPlanes values (at least 8, the record of the builds without tracers)
constexpr int kExcRec = kFieldPlanes + 1 > 8 ? kFieldPlanes + 1 : 8;
static_assert(!kDropinTracer || kXPlane == 5, "tracer corrections follow the five conserved planes");

void fail(unsigned bit, const std::string &msg) {
  g.status |= bit;
  g.last_error = msg;
  static const bool abort_on_error = [] {
    const char *e = std::getenv("EMMA_HYDRO_ABORT");
    return e != nullptr && e[0] == '1';
  }();
  if (abort_on_error) {
    std::fprintf(stderr, "libemmahydro: %s\n", msg.c_str());
    std::abort();
  }
}

bool ck(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  fail(EMMA_ST_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return false;
}
#define CK(call) \
  if (!ck((call), #call)) return (int)EMMA_ST_CUDA

cudaEvent_t get_event() {
  if (!g.free_events.empty()) {
    cudaEvent_t e = g.free_events.back();
    g.free_events.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

bool ensure_pin(size_t bytes) {
  if (bytes <= g.pin_bytes) return true;
  if (g.pin) cudaFreeHost(g.pin);
  g.pin = nullptr;
  g.pin_bytes = 0;
  if (!ck(cudaMallocHost(&g.pin, bytes), "cudaMallocHost")) return false;
  g.pin_bytes = bytes;
  return true;
}

// Persistent host workers for the drop-in's parallel passes over the caller's
// tree (packing, unpacking, hashing, clean_new_hydro): several passes run per
// call, so threads are started once instead of per pass.  run(nt, job) runs
// job(t) for t in [0, nt), t = 0 on the calling thread, and returns when all
// are done; workers make the caller's CUDA device current before their share.
// Never destroyed: the workers sleep on the condition variable until exit.
class HostPool {
 public:
  explicit HostPool(unsigned n) : n_(n) {
    for (unsigned i = 1; i < n; i++) std::thread([this, i] { loop(i); }).detach();
  }
  unsigned size() const { return n_; }
  void run(unsigned nt, const std::function<void(unsigned)> &job) {
    int dev = 0;
    cudaGetDevice(&dev);
    {
      std::lock_guard<std::mutex> lk(m_);
      job_ = &job;
      nt_ = nt;
      dev_ = dev;
      pending_ = nt - 1;
      gen_++;
    }
    cv_.notify_all();
    job(0);
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  void loop(unsigned i) {
    unsigned long long seen = 0;
    int dev_set = -1;
    for (;;) {
      const std::function<void(unsigned)> *job = nullptr;
      int dev = 0;
      {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (i >= nt_) continue;
        job = job_;
        dev = dev_;
      }
      if (dev != dev_set && cudaSetDevice(dev) == cudaSuccess) dev_set = dev;
      (*job)(i);
      std::lock_guard<std::mutex> lk(m_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  const unsigned n_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  const std::function<void(unsigned)> *job_ = nullptr;
  unsigned nt_ = 0, pending_ = 0;
  int dev_ = 0;
  unsigned long long gen_ = 0;
};

// Host threads of the parallel passes: EMMA_HYDRO_HOST_THREADS if set, else the
// hardware threads, at most kMaxHostThreads (and kDefaultHostThreads by default).
// A child process forked after the pool started has none of its workers: it
// starts a pool of its own (the parent's pool object is abandoned in the child).
std::atomic<bool> g_pool_forked{false};
HostPool &host_pool() {
  static HostPool *pool = nullptr;
  static bool atfork = false;
  if (pool == nullptr || g_pool_forked.exchange(false)) {
    if (!atfork) {
      pthread_atfork(nullptr, nullptr, [] { g_pool_forked = true; });
      atfork = true;
    }
    unsigned n = std::min(kDefaultHostThreads, std::max(1u, std::thread::hardware_concurrency()));
    if (const char *e = std::getenv("EMMA_HYDRO_HOST_THREADS")) {
      const long v = std::strtol(e, nullptr, 10);
      if (v >= 1) n = (unsigned)std::min<long>(v, (long)kMaxHostThreads);
    }
    pool = new HostPool(n);
  }
  return *pool;
}

// Host threads of a parallel pass over n items: the pool, one for small passes.
unsigned range_threads(long long n) { return n < 4096 ? 1u : host_pool().size(); }

// Runs f(t, a, b) over [0, n) split into contiguous ranges, one per host
// thread t; every range start is a multiple of `align`.
template <class F>
void parallel_ranges(long long n, F f, long long align = 1) {
  const unsigned nt = range_threads(n);
  if (nt == 1) {
    f(0, 0LL, n);
    return;
  }
  long long chunk = (n + nt - 1) / nt;
  chunk = (chunk + align - 1) / align * align;
  const std::function<void(unsigned)> job = [&](unsigned t) {
    const long long a = t * chunk, b = std::min(n, a + chunk);
    if (a < b) f((int)t, a, b);
  };
  host_pool().run(nt, job);
}

template <class F>
void parallel_for(long long n, F f, long long align = 1) {
  parallel_ranges(n, [&](int, long long a, long long b) { f(a, b); }, align);
}

void drop_graph() {
  if (g.graph) cudaGraphExecDestroy(g.graph);
  g.graph = nullptr;
  g.graph_nsub = g.graph_prec = -1;
  g.graph_col = -2;
  g.graph_colx = -2;
  g.graph_colb = -2;
  g.graph_groups = -3;
  g.graph_is_fused = false;
  g.graph_kernels = 0;
}

void free_level(DevLevel &d) {
  if (d.WB != nullptr) {
    cudaFree(d.WB);
  } else {
    cudaFree(d.W0);
    cudaFree(d.B);
  }
  cudaFree(d.W1);
  cudaFree(d.C);
  cudaFree(d.split);
  cudaFree(d.child);
  cudaFree(d.tiles);
  cudaFree(d.keys);
  cudaFree(d.work);
  cudaFree(d.vcell);
  cudaFree(d.Wv);
  cudaFree(d.F);
  cudaFree(d.Fv);
  cudaFree(d.az);
  cudaFree(d.octidx);
  cudaFree(d.nb6);
  cudaFree(d.marks);
  d = DevLevel();
}

void free_tree(Tree &t) {
  for (auto &d : t.lev) free_level(d);
  t.lev.clear();
  cudaFree(t.d_lv);
  t.d_lv = nullptr;
  t.valid = false;
}

void drop_all() {
  for (auto &c : g.drop) {
    free_tree(c.t);
    c.first = nullptr;
    c.sig.clear();
  }
}

template <class T>
bool upload_vec(T **dst, const std::vector<T> &v) {
  *dst = nullptr;
  if (v.empty()) return true;
  if (!ck(cudaMalloc(dst, v.size() * sizeof(T)), "cudaMalloc")) return false;
  return ck(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy plan");
}

// Allocate device arrays of the mirrored levels, copy topology + plans, and
// initialise the device level slots.
int column_default_nz(const DevLevel &d);

bool alloc_tree(const HostTree &H, Tree &t, bool with_base) {
  t.lev.assign(H.lev.size(), DevLevel());
  t.lcoarse = H.lcoarse;
  t.lmax = H.lmax;
  if (!with_base) g.step_groups = -2;  // a new resident tree: its coarse-step mode is chosen again
  if (!ck(cudaMalloc(&t.d_lv, sizeof(LevelArgs) * kMaxLevels), "cudaMalloc level slots")) return false;
  if (!ck(cudaMemset(t.d_lv, 0, sizeof(LevelArgs) * kMaxLevels), "cudaMemset level slots")) return false;
  for (int L = H.lcoarse; L <= H.lmax; L++) {
    const HostLevel &h = H.lev[L];
    DevLevel &d = t.lev[L];
    d.L = L;
    d.noct = h.noct;
    d.n8 = 8LL * h.noct;
    d.leaf = h.leaf;
    d.ntiles = (int)h.tiles.size();
    d.shape = h.shape;
    // state planes d,u,v,w,p (tracer builds: + dX)
    const size_t bytes = sizeof(double) * (5 + kDropinTracer) * (size_t)std::max<long long>(d.n8, 1);
    if (with_base && !h.tiles.empty()) {
      // drop-in levels: W0 (5 planes), E (and dX) of `field` in one block, uploaded
      // by one pitched copy per oct range, then the base B (the same planes of
      // fieldnew), built on the device from them and the cells where fieldnew differs
      if (!ck(cudaMalloc(&d.WB, sizeof(double) * 2 * kFieldPlanes * (size_t)d.n8), "cudaMalloc W+B")) return false;
      d.W0 = d.WB;
      d.B = d.WB + kFieldPlanes * d.n8;
      if (kDropinTracer) d.X = d.WB + 6 * d.n8;
    } else if (!ck(cudaMalloc(&d.W0, bytes), "cudaMalloc W")) {
      return false;
    } else if (kDropinTracer) {
      d.X = d.W0 + 5 * d.n8;
    }
    if (!ck(cudaMalloc(&d.W1, bytes), "cudaMalloc Wn")) return false;
    if (kDropinTracer) d.Xn = d.W1 + 5 * d.n8;
    // corrections arrive only from the finer level: a level without split cells has none
    bool has_split = false;
    for (uint8_t m : h.split) has_split = has_split || m != 0;
    if (has_split) {
      const size_t cb = sizeof(double) * cplanes() * (size_t)std::max<long long>(d.n8, 1);
      if (!ck(cudaMalloc(&d.C, cb), "cudaMalloc C")) return false;
      if (!ck(cudaMemset(d.C, 0, cb), "cudaMemset C")) return false;
    }
    if (!upload_vec(&d.split, h.split)) return false;
    if (!upload_vec(&d.child, h.child)) return false;
    if (!upload_vec(&d.tiles, h.tiles)) return false;
    if (!upload_vec(&d.keys, h.keys)) return false;
    d.nv = (long long)h.interp.size() / 7;
    if (d.nv > 0) {
      if (!upload_vec(&d.vcell, h.interp)) return false;
      // transmissive builds interpolate the states, gravity builds the forces
      if (!H.grav && !ck(cudaMalloc(&d.Wv, sizeof(double) * 5 * 8 * (size_t)d.nv), "cudaMalloc Wv")) return false;
      if (H.grav && !ck(cudaMalloc(&d.Fv, sizeof(double) * 3 * 8 * (size_t)d.nv), "cudaMalloc Fv")) return false;
    }
    if (g.opt.dual_energy) {
      if (!ck(cudaMalloc(&d.az, (size_t)std::max<long long>(d.n8, 1)), "cudaMalloc az") ||
          !ck(cudaMemset(d.az, 0, (size_t)std::max<long long>(d.n8, 1)), "cudaMemset az"))
        return false;
    }
    if (H.grav) {  // accelerations start at zero until the caller sets them
      const size_t fb = sizeof(double) * 3 * (size_t)std::max<long long>(d.n8, 1);
      if (!ck(cudaMalloc(&d.F, fb), "cudaMalloc F") || !ck(cudaMemset(d.F, 0, fb), "cudaMemset F")) return false;
    }
    std::vector<int> work((size_t)d.ntiles);
    for (int i = 0; i < d.ntiles; i++) work[i] = (L << kWorkSlotShift) | i;
    if (!upload_vec(&d.work, work)) return false;
    LevelArgs a;
    std::memset(&a, 0, sizeof(a));
    a.L = L;
    a.noct = d.noct;
    a.W = d.W0;
    a.Wn = d.W1;
    a.C = d.C;
    a.B = nullptr;
    a.nc8 = (L > H.lcoarse) ? 8LL * H.lev[L - 1].noct : 0;
    a.nf8 = (L < H.lmax) ? 8LL * H.lev[L + 1].noct : 0;
    a.split = d.split;
    a.child = d.child;
    a.tiles = d.tiles;
    a.keys = d.keys;
    a.shape = h.shape;
    a.Wv = d.Wv;
    a.vcell = d.vcell;
    a.nv = d.nv;
    a.dx = std::pow(0.5, L);
    a.ntiles = d.ntiles;
    a.wait_slot = -1;
    a.leaf = d.leaf;
    a.F = d.F;
    a.Fc = (L > H.lcoarse) ? t.lev[L - 1].F : nullptr;
    a.Fv = d.Fv;
    a.gcorr = H.grav;
    a.wv_inject = H.grav;
    a.az = d.az;
    a.azall = (!with_base && g.opt.dual_energy) ? &g.d_S->azall[L] : nullptr;  // resident levels only
    if (!with_base) {  // refinement topology and the cells' marks
      if (!upload_vec(&d.nb6, h.nb6)) return false;
      std::vector<int> m((size_t)d.n8);
      for (int i = 0; i < h.noct; i++)
        for (int c = 0; c < 8; c++) m[8 * (size_t)i + c] = (int)h.octs[i]->cell[c].marked;
      if (!upload_vec(&d.marks, m)) return false;
    }
    // the column kernel: a complete periodic level without split cells of a resident
    // plain-variant tree (its oct at every position, so no tile plan is read)
    const long long nside = 1LL << (L - 1);
    if (!with_base && !has_split && !H.trans && !H.grav && !g.opt.dual_energy && !kDropinTracer && L >= 4 &&
        h.noct == h.nown && (long long)h.noct == nside * nside * nside && (2 * nside) % kColumnWidth == 0) {
      std::vector<int> idx((size_t)h.noct, -1);
      bool full = true;
      for (int i = 0; i < h.noct && full; i++) {
        const long long k = ((long long)h.pos[3 * i + 2] * nside + h.pos[3 * i + 1]) * nside + h.pos[3 * i];
        full = idx[(size_t)k] < 0;
        idx[(size_t)k] = i;
      }
      if (full) {
        if (!upload_vec(&d.octidx, idx)) return false;
        d.col_n = (int)nside;
        d.col_nz = column_default_nz(d);
      }
    }
    k_set_args<<<1, 1, 0, g.stream>>>(t.d_lv, L, a);
    if (!ck(cudaGetLastError(), "k_set_args")) return false;
  }
  t.valid = true;
  return ck(cudaStreamSynchronize(g.stream), "sync after tree allocation");
}

// Pack `field` (which=0) or `fieldnew` (which=1, 6 planes incl. E) of a level.
void pack_level(const HostLevel &h, int which, double *out) {
  const long long n8 = 8LL * h.noct;
  parallel_for(h.noct, [&](long long a, long long b) {
    for (long long i = a; i < b; i++) {
      const struct OCT *o = h.octs[i];
      for (int c = 0; c < 8; c++) {
        const struct Wtype &W = which ? o->cell[c].fieldnew : o->cell[c].field;
        const long long k = 8 * i + c;
        out[k] = W.d;
        out[n8 + k] = W.u;
        out[2 * n8 + k] = W.v;
        out[3 * n8 + k] = W.w;
        out[4 * n8 + k] = W.p;
        if (which) out[5 * n8 + k] = W.E;
      }
    }
  });
}

#ifdef EMMA_WGRAV
// Pack the accelerations f[3] of octs [a, b) of a level into 3 planes of 8*noct.
void pack_force(const HostLevel &h, long long a, long long b, double *out) {
  const long long n8 = 8LL * h.noct;
  for (long long i = a; i < b; i++) {
    const struct OCT *o = h.octs[i];
    for (int c = 0; c < 8; c++) {
      const long long k = 8 * i + c;
      out[k] = o->cell[c].f[0];
      out[n8 + k] = o->cell[c].f[1];
      out[2 * n8 + k] = o->cell[c].f[2];
    }
  }
}
#endif

// Dual energy: az[8i+c] = 1 for a split cell whose stored sound speed is 0 (the
// reference's averaging leaves it so), octs [a, b) of a level.
void pack_az(const HostLevel &h, long long a, long long b, uint8_t *az) {
  for (long long i = a; i < b; i++) {
    const struct OCT *o = h.octs[i];
    for (int c = 0; c < 8; c++) az[8 * i + c] = (o->cell[c].child != nullptr && o->cell[c].field.a == 0.) ? 1 : 0;
  }
}

inline void finish_prims(struct Wtype &W) {
  W.a = std::sqrt(kG * W.p / W.d);
  W.E = W.p / (kG - 1.) + 0.5 * W.d * (W.u * W.u + W.v * W.v + W.w * W.w);
}

// Packs octs [a, b) of a level in one pass over their cells: `field` with E into
// the 6 planes of pw (planes of 8*noct); every cell whose `fieldnew` differs from
// `field` (after clean_new_hydro: the cells a finer level corrected) appends
// {cell, d, u, v, w, p, E, tracers} of its fieldnew to exc (kExcRec values).
// The OR of the bitwise differences of n doubles: 0 exactly when every bit
// matches (a memcmp equality test without the call and its branches).
inline uint64_t bits_xor(const double *a, const double *b, int n) {
  uint64_t d = 0;
  for (int k = 0; k < n; k++) {
    uint64_t x, y;
    std::memcpy(&x, a + k, sizeof(x));
    std::memcpy(&y, b + k, sizeof(y));
    d |= x ^ y;
  }
  return d;
}

void pack_cells(const HostLevel &h, long long a, long long b, double *pw, std::vector<double> &exc) {
  const long long n8 = 8LL * h.noct;
  for (long long i = a; i < b; i++) {
    const struct OCT *o = h.octs[i];
    for (int c = 0; c < 8; c++) {
      const struct Wtype &W = o->cell[c].field, &N = o->cell[c].fieldnew;
      const long long k = 8 * i + c;
      pw[k] = W.d;
      pw[n8 + k] = W.u;
      pw[2 * n8 + k] = W.v;
      pw[3 * n8 + k] = W.w;
      pw[4 * n8 + k] = W.p;
      pw[5 * n8 + k] = W.E;
      // fieldnew differs from field in d, u, v, w, p, E or a tracer (a is recomputed)
      uint64_t diff = bits_xor(&W.d, &N.d, 5) | bits_xor(&W.E, &N.E, 1);
#ifdef EMMA_WRADHYD
      for (int t = 0; t < kDropinTracer; t++) pw[(6 + t) * n8 + k] = tracer(W, t);
      diff |= bits_xor(&W.dX, &N.dX, kDropinTracer);
#endif
      if (diff != 0) {
        double e[kExcRec] = {(double)k, N.d, N.u, N.v, N.w, N.p, N.E};
#ifdef EMMA_WRADHYD
        for (int t = 0; t < kDropinTracer; t++) e[7 + t] = tracer(N, t);
#endif
        exc.insert(exc.end(), e, e + kExcRec);
      }
    }
  }
}

// Writes the 5 planes of p (planes of 8*noct) into `fieldnew` of the leaf cells
// of octs [a, b), with a and E; `also_field` copies the result into `field`.
void unpack_cells(const HostLevel &h, long long a, long long b, const double *p, bool also_field) {
  const long long n8 = 8LL * h.noct;
  for (long long i = a; i < b; i++) {
    struct OCT *o = h.octs[i];
    for (int c = 0; c < 8; c++) {
      if (o->cell[c].child != nullptr) continue;
      const long long k = 8 * i + c;
      struct Wtype &W = o->cell[c].fieldnew;
      W.d = p[k];
      W.u = p[n8 + k];
      W.v = p[2 * n8 + k];
      W.w = p[3 * n8 + k];
      W.p = p[4 * n8 + k];
#ifdef EMMA_WRADHYD
      for (int t = 0; t < kDropinTracer; t++) tracer(W, t) = p[(5 + t) * n8 + k];
#endif
      finish_prims(W);
      if (also_field) o->cell[c].field = W;
    }
  }
}

// Sub-ranges of one host thread's oct range in a drop-in transfer: each is
// packed (unpacked) while the copy engine moves another.
constexpr int kSubRanges = 8;
long long dropin_subrange(long long noct) {
  const long long per_thread = (noct + range_threads(noct) - 1) / range_threads(noct);
  return std::max<long long>(1024, (per_thread + kSubRanges - 1) / kSubRanges);
}

bool ensure_range_events() {
  while (g.range_ev.size() < kMaxHostThreads * (size_t)kSubRanges) {
    cudaEvent_t e;
    if (!ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate")) return false;
    g.range_ev.push_back(e);
  }
  return true;
}

// The level's state changed outside the device schedule: its next CFL step
// comes from the reduction kernel again.
cudaError_t mark_stale(int level) {
  cudaError_t e = cudaMemsetAsync(&g.d_S->fresh[level], 0, sizeof(int), g.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(&g.d_S->smax[level], 0, sizeof(unsigned long long), g.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(&g.d_S->stale[level], 1, sizeof(int), g.stream);  // nonzero
  return e;
}

// Column kernel: planes per work item (the autotuner's candidates).
constexpr int kColNz[6] = {2, 4, 8, 16, 32, 64};

bool column_nz_ok(const DevLevel &d, int nz) {
  const int nc = 2 * d.col_n;
  return d.col_n > 0 && nz >= 2 && nz % 2 == 0 && nz <= nc && nc % nz == 0;
}

long long column_items(const DevLevel &d, int nz) {
  const long long ncol = 2LL * d.col_n / kColumnWidth;
  return ncol * ncol * (2LL * d.col_n / nz);
}

// the largest candidate that still gives every SM four work items (two CTAs per SM,
// two waves), else the smallest valid one
int column_default_nz(const DevLevel &d) {
  int best = 0;
  for (int nz : kColNz) {
    if (!column_nz_ok(d, nz)) continue;
    if (best == 0 || column_items(d, nz) >= 4LL * g.nsm) best = nz;
  }
  return best;
}

// planes per item of a launch of resident level L on the column kernel; 0: the
// brick kernel (FP64 path, ineligible level, option column < 0, or the
// autotuner found the brick kernel faster)
int column_nz(int L) {
  if (L < 0 || !g.res.valid || L < g.res.lcoarse || L > g.res.lmax) return 0;
  const DevLevel &d = g.res.lev[L];
  if (d.col_n == 0 || g.opt.precision != EMMA_PREC_MIXED || g.opt.column < 0) return 0;
  if (g.opt.column > 0) return column_nz_ok(d, g.opt.column) ? g.opt.column : 0;
  return d.col_nz;
}

// x sweep of the column-kernel launches of resident level L (ColumnArgs::xshfl)
int column_xs(int L) {
  if (g.opt.column_xshfl != 0) return g.opt.column_xshfl > 0 ? 1 : 0;
  return g.opt.column > 0 ? 0 : g.res.lev[L].col_xs;
}

// work split of the column-kernel launches of resident level L (ColumnArgs::balanced)
int column_bal(int L) {
  if (g.opt.column_balanced != 0) return g.opt.column_balanced > 0 ? 1 : 0;
  return g.opt.column > 0 ? 0 : g.res.lev[L].col_bal;
}

cudaError_t launch_column(int L, int nz, const int *gate, bool fuse_cfl, int xs = -1, int bal = -1) {
  const DevLevel &d = g.res.lev[L];
  ColumnArgs c;
  c.lv = g.res.d_lv + L;
  c.L = L;
  c.octidx = d.octidx;
  c.n = d.col_n;
  c.nz = nz;
  c.ncol = 2 * d.col_n / kColumnWidth;
  c.balanced = bal >= 0 ? bal : column_bal(L);
  if (c.balanced) {  // the kernel's two CTAs per SM, runs of at least 16 column-planes
    const long long ncol = 2LL * d.col_n / kColumnWidth, planes = ncol * ncol * 2LL * d.col_n;
    c.nitems = (int)std::max(1LL, std::min(2LL * g.nsm, planes / 16));
  } else {
    c.nitems = (int)column_items(d, nz);
  }
  c.gate = gate;
  c.status = g.d_status;
  c.smax = fuse_cfl ? g.d_S->smax_next : nullptr;
  c.xshfl = xs >= 0 ? xs : column_xs(L);
  return launch_column_f32(c, g.stream);
}

// fuse_cfl: the launch also accumulates each level's max signal speed of the
// state it writes (the device schedule's next CFL step, SchedState::smax_next).
// col_level: the launch advances resident level col_level alone, which may then
// run on the column kernel (column_nz).
bool launch_batch(LevelArgs *d_lv, const int *work, int nwork, const int *gate, long long cells, unsigned shapes,
                  int ctas, bool fuse_cfl = false, bool grav = false, int col_level = -1) {
  BatchArgs a{};
  a.lv = d_lv;
  a.work = work;
  a.nwork = nwork;
  a.done = g.d_done;
  a.gate = gate;
  a.status = g.d_status;
  a.wait_limit = g.wait_limit;
  a.smax = fuse_cfl ? g.d_S->smax_next : nullptr;
  a.ticket = g.d_S->ticket;
  a.zero_c = 0;  // the level schedule clears a level's corrections when its iteration starts
  TimedLaunch tl{};
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(g.stream, &cap);
  const bool timed = g.timing && cap == cudaStreamCaptureStatusNone;
  if (timed) {
    tl.a = get_event();
    tl.b = get_event();
    cudaEventRecord(tl.a, g.stream);
  }
  // the levels of a gravity build run the gravity-coupled variant; dual energy and the
  // tracer build their own
  if (grav || (d_lv == g.res.d_lv && g.res.host.grav)) shapes |= kLaunchGrav;
  if (g.opt.dual_energy) shapes |= kLaunchDual;
  shapes |= kLaunchTracers;
  const int cnz = (d_lv == g.res.d_lv && !(shapes & (kLaunchGrav | kLaunchDual | kLaunchTracer | kLaunchHelium)))
                      ? column_nz(col_level) : 0;
  cudaError_t e = (cnz > 0) ? launch_column(col_level, cnz, gate, fuse_cfl)
                  : (g.opt.precision == EMMA_PREC_MIXED)
                      ? launch_level_f32(a, shapes, g.nsm, ctas, g.stream, nullptr)
                      : launch_level_fp64(a, shapes, g.nsm, ctas, g.stream, nullptr);
  if (nwork > 0) g.kernel_launches++;
  if (timed) {
    cudaEventRecord(tl.b, g.stream);
    tl.cells = cells;
    tl.level = col_level;
    g.launches.push_back(tl);
  }
  return ck(e, "level kernel launch");
}

int level_ok(int level) {
  if (!g.res.valid || level < g.res.lcoarse || level > g.res.lmax) {
    fail(EMMA_ST_ARG, "level " + std::to_string(level) + " is not mirrored");
    return 0;
  }
  return 1;
}

// current state buffer of a resident level (the device slot is authoritative)
double *current_state(int level) {
  double *p = nullptr;
  if (!ck(cudaMemcpyAsync(&p, &g.res.d_lv[level].W, sizeof(double *), cudaMemcpyDeviceToHost, g.stream),
          "read level slot") ||
      !ck(cudaStreamSynchronize(g.stream), "sync"))
    return nullptr;
  return p;
}

// ------------------------------------------------------------ host schedule
// hydro-only Advance_level schedule (src/advanceamr.c:243-1299), host driven
struct Sched {
  double dt_param, time_max;
  int nsub;
  double *adt;
  int err;
};

double advance_level(Sched &S, int level, double tloc) {
  double dt = 0., dtnew, dthydro, dtfine;
  double *adt = S.adt;
  int is = 0;
  do {
    S.err |= emma_hydro_clean_new(level);
    dtnew = S.dt_param;
    dtnew = ((S.time_max - tloc) < dtnew ? (S.time_max - tloc) : dtnew);
    S.err |= emma_hydro_comptstep(level, &dthydro);
    dtnew = (dthydro < dtnew ? dthydro : dtnew);
    adt[level - 1] = dtnew;
    if (level == g.res.lcoarse) adt[level - 2] = adt[level - 1];
    if (adt[level - 2] < adt[level - 1]) adt[level - 1] = adt[level - 2];
    else adt[level - 1] = std::fmin(adt[level - 1], adt[level - 2] - dt);
    if (level < g.res.lmax && g.res.lev[level + 1].noct > 0) {
      dtfine = advance_level(S, level + 1, tloc);
      adt[level - 1] = dtfine;
      if (level == g.res.lcoarse) adt[level - 2] = adt[level - 1];
    }
    S.err |= emma_hydro_advance_level(level, adt[level - 1]);
    dt += adt[level - 1];
    tloc += adt[level - 1];
    is++;
  } while ((dt < adt[level - 2]) && (is < S.nsub) && S.err == 0);
  return dt;
}

// --------------------------------------------------------- device schedule
int finest_level() {
  int lf = g.res.lcoarse;
  while (lf < g.res.lmax && g.res.lev[lf + 1].noct > 0) lf++;
  return lf;
}

// emit one Advance_level(L) call: nsub gated iterations (schedule.cu)
bool emit_level(int L, int nsub) {
  const Tree &t = g.res;
  const DevLevel &d = t.lev[L];
  const int lf = finest_level();
  const bool has_fine = L < lf;
  SchedState *S = g.d_S;
  for (int it = 0; it < nsub; it++) {
    k_sub_begin<<<1, 1, 0, g.stream>>>(S, L, it);
    const int *gate = &S->active[L];
    const long long n5 = cplanes() * d.n8;
    if (d.C != nullptr)
      k_clear<<<(unsigned)std::max<long long>(1, std::min<long long>((n5 + 255) / 256, 4LL * g.nsm)), 256, 0,
                g.stream>>>(d.C, n5, gate);
    // the separate CFL reduction runs only when the level's state was not written by the level kernel
    if (!ck(launch_cfl(t.d_lv, L, d.n8, &S->cfl_gate[L], &S->smax[L], g.nsm, g.stream), "cfl launch")) return false;
    k_sub_dt<<<1, 1, 0, g.stream>>>(S, L);
    if (has_fine && !emit_level(L + 1, nsub)) return false;
    k_sub_prelaunch<<<1, 1, 0, g.stream>>>(S, t.d_lv, L, has_fine ? 1 : 0);
    if (!ck(launch_interp(t.d_lv, L, d.nv, gate, g.nsm, g.stream, t.host.grav), "interpolation launch")) return false;
    if (!launch_batch(t.d_lv, d.work, d.ntiles, gate, d.leaf, 1u << d.shape, d.ctas, true, false, L)) return false;
    k_sub_end<<<1, 1, 0, g.stream>>>(S, t.d_lv, L);
    if (!ck(cudaGetLastError(), "schedule kernel")) return false;
  }
  return true;
}

// The subcycled coarse step runs as one fused kernel (step_kernel.cuh) unless the
// option turns it off or the tree needs work that kernel does not do: the
// interpolation of coarser neighbours (gravity and transmissive trees) or a level
// on the column kernel.
bool fused_step_ok() {
  if (g.opt.fused_step < 0 || g.res.host.grav || g.opt.trans_flags != 0) return false;
  if (g.opt.dual_energy && kLaunchTracers != 0u) return false;
  for (int L = g.res.lcoarse; L <= finest_level(); L++)
    if (g.res.lev[L].nv > 0 || column_nz(L) > 0) return false;
  return true;
}

// one coarse step, all on the device
bool emit_coarse_step(int nsub) {
  const Tree &t = g.res;
  SchedState *S = g.d_S;
  const int lc = t.lcoarse, lf = finest_level();
  if (nsub == 1 || lf == lc) {
    // one dt for every level: CFL per level (from the previous launch's fused maxima, or a
    // reduction kernel where the state was set from the host), then all levels in one launch
    for (int L = lc; L <= lf; L++) {
      const DevLevel &d = t.lev[L];
      if (d.C != nullptr && !ck(cudaMemsetAsync(d.C, 0, sizeof(double) * cplanes() * d.n8, g.stream), "memset C"))
        return false;
      if (!ck(launch_cfl(t.d_lv, L, d.n8, &S->stale[L], &S->smax[L], g.nsm, g.stream), "cfl launch"))
        return false;
    }
    k_batch_begin<<<1, 1, 0, g.stream>>>(S, t.d_lv, g.d_done);
    for (int L = lc; L <= lf; L++)
      if (!ck(launch_interp(t.d_lv, L, t.lev[L].nv, nullptr, g.nsm, g.stream, t.host.grav), "interpolation launch"))
        return false;
    long long cells = 0;
    unsigned shapes = 0;
    int ctas = 0, most = -1;
    for (int L = lc; L <= lf; L++) {
      cells += t.lev[L].leaf;
      shapes |= 1u << t.lev[L].shape;
      if (t.lev[L].ntiles > most) {  // CTAs per SM tuned for the level with the most tiles
        most = t.lev[L].ntiles;
        ctas = t.lev[L].ctas;
      }
    }
    if (!launch_batch(t.d_lv, g.d_work_all, g.nwork_all, nullptr, cells, shapes, ctas, true, false,
                      lf == lc ? lc : -1))
      return false;
    k_batch_end<<<1, 1, 0, g.stream>>>(S, t.d_lv);
    return ck(cudaGetLastError(), "schedule kernel");
  }
  if (g.step_groups > 0 && fused_step_ok()) {
    // the whole recursion in one persistent kernel (step_kernel.cuh)
    if (!ck(cudaMemsetAsync(g.d_ctl, 0, sizeof(StepCtl), g.stream), "memset step control")) return false;
    StepArgs a{};
    a.lv = t.d_lv;
    a.S = S;
    a.ctl = g.d_ctl;
    a.done = g.d_done;
    a.status = g.d_status;
    a.wait_limit = g.wait_limit;
    a.lfine = lf;
    a.jobt = g.d_jobt;
    const unsigned variant = (g.opt.dual_energy ? kLaunchDual : 0u) | kLaunchTracers;
    const cudaError_t e = (g.opt.precision == EMMA_PREC_MIXED)
                              ? launch_step_f32(a, variant, g.step_groups, g.nsm, g.stream, &g.step_grid,
                                                &g.step_threads)
                              : launch_step_fp64(a, variant, g.step_groups, g.nsm, g.stream, &g.step_grid,
                                                 &g.step_threads);
    g.kernel_launches++;
    g.graph_is_fused = true;
    return ck(e, "fused coarse step");
  }
  if (!emit_level(lc, nsub)) return false;
  k_sub_final<<<1, 1, 0, g.stream>>>(S);
  return ck(cudaGetLastError(), "schedule kernel");
}

bool ensure_graph(int nsub) {
  if (g.graph && g.graph_nsub == nsub && g.graph_prec == g.opt.precision && g.graph_col == g.opt.column &&
      g.graph_colx == g.opt.column_xshfl && g.graph_colb == g.opt.column_balanced &&
      g.graph_groups == g.step_groups)
    return true;
  drop_graph();
  cudaGraph_t graph = nullptr;
  if (!ck(cudaStreamBeginCapture(g.stream, cudaStreamCaptureModeThreadLocal), "begin capture")) return false;
  const bool ok = emit_coarse_step(nsub);
  cudaError_t e = cudaStreamEndCapture(g.stream, &graph);
  if (!ok || !ck(e, "end capture")) {
    if (graph) cudaGraphDestroy(graph);
    return false;
  }
  size_t nn = 0;
  int kn = 0;
  if (cudaGraphGetNodes(graph, nullptr, &nn) == cudaSuccess && nn > 0) {
    std::vector<cudaGraphNode_t> nodes(nn);
    if (cudaGraphGetNodes(graph, nodes.data(), &nn) == cudaSuccess)
      for (size_t i = 0; i < nn; i++) {
        cudaGraphNodeType ty;
        if (cudaGraphNodeGetType(nodes[i], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) kn++;
      }
  }
  e = cudaGraphInstantiate(&g.graph, graph, 0);
  cudaGraphDestroy(graph);
  if (!ck(e, "graph instantiate")) {
    g.graph = nullptr;
    return false;
  }
  g.graph_nsub = nsub;
  g.graph_prec = g.opt.precision;
  g.graph_col = g.opt.column;
  g.graph_colx = g.opt.column_xshfl;
  g.graph_colb = g.opt.column_balanced;
  g.graph_groups = g.step_groups;
  g.graph_kernels = kn;
  return true;
}

bool write_sched_params(double dt_param, double time_max, int nsub, const double *tsim, const double *adt) {
  SchedState &h = *g.h_S;
  if (!ck(cudaStreamSynchronize(g.stream), "sync")) return false;
  h.dt_param = dt_param;
  h.time_max = time_max;
  h.cfl = g.opt.cfl;
  if (!ck(cudaMemcpyAsync(&g.d_S->dt_param, &h.dt_param, 3 * sizeof(double), cudaMemcpyHostToDevice, g.stream),
          "write schedule parameters"))
    return false;
  h.nsub = nsub;
  if (!ck(cudaMemcpyAsync(&g.d_S->nsub, &h.nsub, sizeof(int), cudaMemcpyHostToDevice, g.stream), "write nsub"))
    return false;
  if (tsim != nullptr) {
    h.tsim = *tsim;
    if (!ck(cudaMemcpyAsync(&g.d_S->tsim, &h.tsim, sizeof(double), cudaMemcpyHostToDevice, g.stream), "write tsim"))
      return false;
  }
  if (adt != nullptr) {
    for (int l = 0; l < g.res.lmax && l < kMaxLevels; l++) h.adt[l] = adt[l];
    if (!ck(cudaMemcpyAsync(g.d_S->adt, h.adt, sizeof(double) * std::min(g.res.lmax, kMaxLevels),
                            cudaMemcpyHostToDevice, g.stream),
            "write adt"))
      return false;
  }
  return ck(cudaStreamSynchronize(g.stream), "sync");
}

#include "refine_impl.cuh"

}  // namespace

// The resident tree's mirror of a level and the level's current device state (5
// planes), for the field dumps; false unless `firstoct` is the resident tree's.
bool emma::resident_level(struct OCT **firstoct, int level, const HostLevel **h, const double **W,
                          const uint8_t **split, cudaStream_t *stream, int *nsm) {
  if (!(g.ready && g.res.valid && firstoct != nullptr && g.res_first == firstoct)) return false;
  if (level < g.res.lcoarse || level > g.res.lmax) return false;
  *h = &g.res.host.lev[level];
  *W = current_state(level);
  *split = g.res.lev[level].split;
  *stream = g.stream;
  *nsm = g.nsm;
  return *W != nullptr;
}

extern "C" {

int emma_hydro_status(void) {
  if (g.ready) {
    unsigned h = 0;
    if (cudaStreamSynchronize(g.stream) != cudaSuccess) g.status |= EMMA_ST_CUDA;
    if (cudaMemcpy(&h, g.d_status, sizeof(unsigned), cudaMemcpyDeviceToHost) == cudaSuccess) g.status |= h;
  }
  return (int)g.status;
}

void emma_hydro_clear_status(void) {
  g.status = 0;
  g.last_error.clear();
  if (g.ready) {
    cudaStreamSynchronize(g.stream);
    cudaMemset(g.d_status, 0, sizeof(unsigned));
  }
}

const char *emma_hydro_last_error(void) { return g.last_error.c_str(); }

void emma_hydro_default_options(struct EmmaHydroOptions *opt) {
  if (opt == nullptr) return;
  opt->precision = EMMA_PREC_FP64;
  opt->trans_flags = 0;
  opt->cfl = 0.85;
  opt->tile_octs = 0;
  opt->device = 0;
  opt->use_graph = 1;
  opt->gravity = 0;
  opt->dual_energy = 0;
  opt->column = 0;
  opt->fused_step = 0;
  opt->column_xshfl = 0;
  opt->column_balanced = 0;
}

int emma_hydro_init(const struct EmmaHydroOptions *opt) {
  if (g.ready) {
    if (opt) return emma_hydro_set_options(opt);
    return 0;
  }
  emma_hydro_default_options(&g.opt);
  if (opt) g.opt = *opt;
  CK(cudaSetDevice(g.opt.device));
  CK(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
  CK(cudaDeviceGetAttribute(&g.nsm, cudaDevAttrMultiProcessorCount, g.opt.device));
  CK(cudaMalloc(&g.d_status, sizeof(unsigned)));
  CK(cudaMemset(g.d_status, 0, sizeof(unsigned)));
  CK(cudaMalloc(&g.d_done, sizeof(unsigned) * kMaxLevels));
  CK(cudaMemset(g.d_done, 0, sizeof(unsigned) * kMaxLevels));
  CK(cudaMalloc(&g.d_S, sizeof(SchedState)));
  CK(cudaMemset(g.d_S, 0, sizeof(SchedState)));
  CK(cudaMalloc(&g.d_ctl, sizeof(StepCtl)));
  CK(cudaMemset(g.d_ctl, 0, sizeof(StepCtl)));
  CK(cudaMalloc(&g.d_jobt, sizeof(StepJobRecord) * kStepJobLog));
  CK(cudaMemset(g.d_jobt, 0, sizeof(StepJobRecord) * kStepJobLog));
  CK(cudaMallocHost(&g.h_S, sizeof(SchedState)));
  std::memset(g.h_S, 0, sizeof(SchedState));
  g.ready = true;
  return 0;
}

int emma_hydro_set_options(const struct EmmaHydroOptions *opt) {
  if (opt == nullptr) return EMMA_ST_ARG;
  if (!g.ready) return emma_hydro_init(opt);
  const int old_trans = g.opt.trans_flags, old_grav = g.opt.gravity, old_dual = g.opt.dual_energy;
  g.opt = *opt;
  g.step_groups = -2;  // the coarse-step mode is chosen again for the new options
  if (old_trans != opt->trans_flags || old_grav != opt->gravity || old_dual != opt->dual_energy) {
    // the tile plans encode the boundary ghosts and the gravity interpolation lists:
    // a resident tree must be uploaded again
    cudaStreamSynchronize(g.stream);
    drop_graph();
    free_tree(g.res);
    drop_all();
  }
  return 0;
}

void emma_hydro_shutdown(void) {
  if (!g.ready) return;
  cudaStreamSynchronize(g.stream);
  drop_graph();
  free_tree(g.res);
  drop_all();
  cudaFree(g.d_work_all);
  for (auto &t : g.launches) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  for (auto e : g.free_events) cudaEventDestroy(e);
  for (auto e : g.range_ev) cudaEventDestroy(e);
  g.range_ev.clear();
  if (g.pin_exc) cudaFreeHost(g.pin_exc);
  cudaFree(g.d_exc);
  cudaFree(g.d_status);
  cudaFree(g.d_done);
  cudaFree(g.d_S);
  cudaFree(g.d_ctl);
  cudaFree(g.d_jobt);
  cudaFreeHost(g.h_S);
  if (g.pin) cudaFreeHost(g.pin);
  if (g.own_stream) cudaStreamDestroy(g.stream);
  release_dump_staging();
  g = Ctx();
}

int emma_hydro_set_stream(void *stream) {
  if (!g.ready && emma_hydro_init(nullptr) != 0) return EMMA_ST_CUDA;
  CK(cudaStreamSynchronize(g.stream));
  drop_graph();
  if (g.own_stream) CK(cudaStreamDestroy(g.stream));
  // NULL selects a stream owned by the library (a caller wanting the legacy
  // default stream passes cudaStreamLegacy)
  if (stream == nullptr) {
    CK(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
    g.own_stream = true;
  } else {
    g.stream = static_cast<cudaStream_t>(stream);
    g.own_stream = false;
  }
  return 0;
}

// ------------------------------------------------------------ resident path
// Brick shape requested by the options: -1 = autotuned, else an index into kShapes.
int requested_shape(int tile_octs) {
  if (tile_octs == 0) return -1;
  for (int i = 0; i < kNumShapes; i++)
    if (kShapes[i].octs() == tile_octs) return i;
  return -2;
}

// Point a level slot at a plan (tiles, keys, brick shape, interpolation list).
bool bind_plan(LevelArgs *slot, TileDesc *tiles, uint32_t *keys, int shape, int ntiles, double *Wv, int *vcell,
               long long nv, double *Fv) {
  return ck(cudaMemcpyAsync(&slot->tiles, &tiles, sizeof(tiles), cudaMemcpyHostToDevice, g.stream), "bind") &&
         ck(cudaMemcpyAsync(&slot->keys, &keys, sizeof(keys), cudaMemcpyHostToDevice, g.stream), "bind") &&
         ck(cudaMemcpyAsync(&slot->shape, &shape, sizeof(int), cudaMemcpyHostToDevice, g.stream), "bind") &&
         ck(cudaMemcpyAsync(&slot->ntiles, &ntiles, sizeof(int), cudaMemcpyHostToDevice, g.stream), "bind") &&
         ck(cudaMemcpyAsync(&slot->Wv, &Wv, sizeof(Wv), cudaMemcpyHostToDevice, g.stream), "bind") &&
         ck(cudaMemcpyAsync(&slot->vcell, &vcell, sizeof(vcell), cudaMemcpyHostToDevice, g.stream), "bind") &&
         ck(cudaMemcpyAsync(&slot->nv, &nv, sizeof(nv), cudaMemcpyHostToDevice, g.stream), "bind") &&
         ck(cudaMemcpyAsync(&slot->Fv, &Fv, sizeof(Fv), cudaMemcpyHostToDevice, g.stream), "bind") &&
         ck(cudaStreamSynchronize(g.stream), "bind");
}

// Autotuner.  For every level of the resident tree it times single-level
// launches of the level kernel on the level's own state (dt = 0: the arithmetic
// of a real step, no change of state) for each candidate brick shape (4x4x2
// octs x 1 brick, 2x2x2 octs x 4 bricks: the stencil-batch size and octs per
// tile) and each number of co-resident CTAs per SM (1 .. occupancy: how many
// tiles are staged in flight per SM), and keeps the fastest.  Complete levels
// only try the 4x4x2 brick (every brick is full).  Side effects of the trial
// launches (corrections added to the coarser level, completion counters,
// status bits) are undone afterwards.
bool autotune_tree(Tree &t, int shape_req) {
  unsigned status0 = 0;
  if (!ck(cudaStreamSynchronize(g.stream), "sync") ||
      !ck(cudaMemcpy(&status0, g.d_status, sizeof(unsigned), cudaMemcpyDeviceToHost), "status"))
    return false;
  const bool timing0 = g.timing;
  const long long launches0 = g.kernel_launches;
  g.timing = false;
  cudaEvent_t e0 = get_event(), e1 = get_event();
  bool ok = true;
  for (int L = t.lcoarse; L <= t.lmax && ok; L++) {
    DevLevel &d = t.lev[L];
    HostLevel &h = t.host.lev[L];
    if (d.ntiles == 0) continue;
    const bool complete = h.noct == (1LL << (3 * (L - 1)));
    double best = 0;
    int best_shape = d.shape, best_ctas = 0;
    for (int s = 0; s < kNumShapes && ok; s++) {
      if (shape_req >= 0 && s != shape_req) continue;
      if (shape_req < 0 && complete && s != 0) continue;
      // the candidate plan on the device (the current one, or a re-plan with its
      // own interpolation list and buffer)
      TileDesc *tiles = d.tiles;
      uint32_t *keys = d.keys;
      int *work = d.work, *vcell = d.vcell;
      double *Wv = d.Wv, *Fv = d.Fv;
      long long nv = d.nv;
      int ntiles = d.ntiles;
      HostLevel alt;
      if (s != d.shape) {
        std::string err;
        HostLevel saved = h;
        const int rc = replan_level(t.host, L, s, err);
        alt = h;
        h = saved;
        if (rc != 0) continue;  // shape not plannable here: skip the candidate
        ntiles = (int)alt.tiles.size();
        nv = (long long)alt.interp.size() / 7;
        std::vector<int> wl((size_t)ntiles);
        for (int i = 0; i < ntiles; i++) wl[i] = (L << kWorkSlotShift) | i;
        vcell = nullptr;
        Wv = nullptr;
        Fv = nullptr;
        if (!upload_vec(&tiles, alt.tiles) || !upload_vec(&keys, alt.keys) || !upload_vec(&work, wl) ||
            (nv > 0 && (!upload_vec(&vcell, alt.interp) ||
                        (!t.host.grav && !ck(cudaMalloc(&Wv, sizeof(double) * 5 * 8 * (size_t)nv), "cudaMalloc Wv")))) ||
            (nv > 0 && t.host.grav && !ck(cudaMalloc(&Fv, sizeof(double) * 3 * 8 * (size_t)nv), "cudaMalloc Fv"))) {
          ok = false;
          break;
        }
      }
      ok = bind_plan(t.d_lv + L, tiles, keys, s, ntiles, Wv, vcell, nv, Fv);
      k_bind_level<<<1, 1, 0, g.stream>>>(t.d_lv, L, t.lcoarse, t.lmax, 0.);
      if (ok) ok = ck(launch_interp(t.d_lv, L, nv, nullptr, g.nsm, g.stream, t.host.grav), "interpolation launch");
      int occ = 0;
      BatchArgs probe{};
      if (ok)
        ok = ck((g.opt.precision == EMMA_PREC_MIXED)
                    ? launch_level_f32(probe, (1u << s) | kLaunchTracers | (t.host.grav ? kLaunchGrav : 0u) |
                                                  (g.opt.dual_energy ? kLaunchDual : 0u), g.nsm, 0, g.stream, &occ)
                    : launch_level_fp64(probe, (1u << s) | kLaunchTracers | (t.host.grav ? kLaunchGrav : 0u) |
                                                   (g.opt.dual_energy ? kLaunchDual : 0u), g.nsm, 0, g.stream, &occ),
                "occupancy");
      for (int c = 1; ok && c <= std::min(occ, 4); c++) {
        double ms = 0;
        for (int rep = 0; rep < 4 && ok; rep++) {  // one warm-up, three timed
          ok = ck(cudaEventRecord(e0, g.stream), "event");
          ok = ok && launch_batch(t.d_lv, work, ntiles, nullptr, 0, 1u << s, c);
          ok = ok && ck(cudaEventRecord(e1, g.stream), "event") && ck(cudaEventSynchronize(e1), "event");
          float f = 0;
          if (ok && rep > 0 && cudaEventElapsedTime(&f, e0, e1) == cudaSuccess) ms += f / 3.;
        }
        d.sweep_ms[s][c - 1] = ms;
        if (ok && (best == 0 || ms < best)) {
          best = ms;
          best_shape = s;
          best_ctas = c;
        }
      }
      if (s != d.shape) {
        cudaStreamSynchronize(g.stream);
        if (ok && best_shape == s) {
          // the re-plan wins so far: it becomes the level's plan
          cudaFree(d.tiles);
          cudaFree(d.keys);
          cudaFree(d.work);
          cudaFree(d.vcell);
          cudaFree(d.Wv);
          cudaFree(d.Fv);
          d.tiles = tiles;
          d.keys = keys;
          d.work = work;
          d.vcell = vcell;
          d.Wv = Wv;
          d.Fv = Fv;
          d.nv = nv;
          d.ntiles = ntiles;
          d.shape = s;
          h = alt;
        } else {
          cudaFree(tiles);
          cudaFree(keys);
          cudaFree(work);
          cudaFree(vcell);
          cudaFree(Wv);
          cudaFree(Fv);
        }
      }
    }
    // bind the kept plan
    ok = ok && bind_plan(t.d_lv + L, d.tiles, d.keys, d.shape, d.ntiles, d.Wv, d.vcell, d.nv, d.Fv) &&
         ck(cudaStreamSynchronize(g.stream), "tune");
    d.ctas = best_ctas;
    d.tuned = ok;
    // the column kernel against the best brick launch, over its planes per work item
    if (ok && d.col_n > 0 && g.opt.precision == EMMA_PREC_MIXED && g.opt.column == 0 && shape_req < 0) {
      int best_nz = 0;
      double best_col = 0;
      for (int i = 0; i < 6 && ok; i++) {
        const int nz = kColNz[i];
        d.col_sweep_ms[i] = 0;
        if (!column_nz_ok(d, nz)) continue;
        double ms = 0;
        for (int rep = 0; rep < 4 && ok; rep++) {  // one warm-up, three timed
          ok = ck(cudaEventRecord(e0, g.stream), "event") && ck(launch_column(L, nz, nullptr, false, 0), "column") &&
               ck(cudaEventRecord(e1, g.stream), "event") && ck(cudaEventSynchronize(e1), "event");
          float f = 0;
          if (ok && rep > 0 && cudaEventElapsedTime(&f, e0, e1) == cudaSuccess) ms += f / 3.;
        }
        d.col_sweep_ms[i] = ms;
        if (ok && (best_col == 0 || ms < best_col)) {
          best_col = ms;
          best_nz = nz;
        }
      }
      // the warp-shuffle x sweep at the best depth against the shared-memory one
      d.col_xs = 0;
      d.col_xs_ms[0] = best_col;
      d.col_xs_ms[1] = 0;
      if (ok && best_nz > 0) {
        double ms = 0;
        for (int rep = 0; rep < 4 && ok; rep++) {
          ok = ck(cudaEventRecord(e0, g.stream), "event") &&
               ck(launch_column(L, best_nz, nullptr, false, 1), "column") && ck(cudaEventRecord(e1, g.stream), "event") &&
               ck(cudaEventSynchronize(e1), "event");
          float f = 0;
          if (ok && rep > 0 && cudaEventElapsedTime(&f, e0, e1) == cudaSuccess) ms += f / 3.;
        }
        d.col_xs_ms[1] = ms;
        if (ok && ms > 0 && ms < best_col) {
          d.col_xs = 1;
          best_col = ms;
        }
      }
      // balanced runs of column-planes (the chosen x sweep) against the items
      d.col_bal = 0;
      d.col_bal_ms[0] = best_col;
      d.col_bal_ms[1] = 0;
      if (ok && best_nz > 0) {
        double ms = 0;
        for (int rep = 0; rep < 4 && ok; rep++) {
          ok = ck(cudaEventRecord(e0, g.stream), "event") &&
               ck(launch_column(L, best_nz, nullptr, false, d.col_xs, 1), "column") &&
               ck(cudaEventRecord(e1, g.stream), "event") && ck(cudaEventSynchronize(e1), "event");
          float f = 0;
          if (ok && rep > 0 && cudaEventElapsedTime(&f, e0, e1) == cudaSuccess) ms += f / 3.;
        }
        d.col_bal_ms[1] = ms;
        if (ok && ms > 0 && ms < best_col) {
          d.col_bal = 1;
          best_col = ms;
        }
      }
      d.col_nz = (ok && best_col > 0 && (best == 0 || best_col < best)) ? best_nz : 0;
    }
  }
  // undo the trial launches: corrections, completion counters, status
  for (int L = t.lcoarse; L <= t.lmax && ok; L++) {
    const DevLevel &d = t.lev[L];
    if (d.C != nullptr) ok = ck(cudaMemsetAsync(d.C, 0, sizeof(double) * cplanes() * d.n8, g.stream), "memset C");
  }
  ok = ok && ck(cudaMemsetAsync(g.d_done, 0, sizeof(unsigned) * kMaxLevels, g.stream), "memset done") &&
       ck(cudaMemcpyAsync(g.d_status, &status0, sizeof(unsigned), cudaMemcpyHostToDevice, g.stream), "status") &&
       ck(cudaStreamSynchronize(g.stream), "sync");
  g.free_events.push_back(e0);
  g.free_events.push_back(e1);
  g.timing = timing0;
  g.kernel_launches = launches0;
  return ok;
}

int emma_hydro_is_resident(struct OCT **firstoct) {
  return (g.ready && g.res.valid && firstoct != nullptr && g.res_first == firstoct) ? 1 : 0;
}

int emma_hydro_tree_release(struct OCT **firstoct) {
  if (!emma_hydro_is_resident(firstoct)) return 0;
  const cudaError_t e = cudaStreamSynchronize(g.stream);
  drop_graph();
  free_tree(g.res);
  cudaFree(g.d_work_all);
  g.d_work_all = nullptr;
  g.nwork_all = 0;
  g.res_first = nullptr;
  return e == cudaSuccess ? 0 : EMMA_ST_CUDA;
}

int emma_hydro_tree_upload(struct OCT **firstoct, int lcoarse, int lmax, int rank) {
  if (!g.ready && emma_hydro_init(nullptr) != 0) return EMMA_ST_CUDA;
  if (kDropinTracer && (g.opt.dual_energy || g.opt.trans_flags || g.opt.gravity)) {
    fail(EMMA_ST_ARG, "the -DWRADHYD library has neither dual energy, transmissive boundaries nor gravity");
    return EMMA_ST_ARG;
  }
  if (firstoct == nullptr || lcoarse < 2 || lmax < lcoarse || lmax >= kMaxLevels) {
    fail(EMMA_ST_ARG, "bad tree arguments");
    return EMMA_ST_ARG;
  }
  CK(cudaStreamSynchronize(g.stream));
  drop_graph();
  free_tree(g.res);
  cudaFree(g.d_work_all);
  g.d_work_all = nullptr;
  g.nwork_all = 0;
  std::string err;
  const int shape_req = requested_shape(g.opt.tile_octs);
  if (shape_req < -1) {
    fail(EMMA_ST_ARG, "tile_octs must be 0 (autotuned), 32 or 8");
    return EMMA_ST_ARG;
  }
  std::vector<int> shapes((size_t)lmax + 1, shape_req);
  int rc = build_host_tree(firstoct, lcoarse, lmax, rank, g.opt.trans_flags, lcoarse, lmax, g.res.host, err,
                           shapes.data(), g.opt.gravity, g.opt.dual_energy);
  if (rc != 0) {
    fail((unsigned)rc, err);
    return rc;
  }
  if (g.res.host.ghosts) {
    // a resident tree is advanced for many levels and steps without the host: the
    // boundary octs of a multi-rank run would never be refreshed between solves
    g.res.host = HostTree();
    fail(EMMA_ST_ARG, "the level lists hold octs of other ranks: a multi-rank run advances through the drop-in "
                      "entries, between the exchanges of its boundary octs");
    return EMMA_ST_ARG;
  }
  if (!alloc_tree(g.res.host, g.res, false)) return EMMA_ST_CUDA;
  g.res_first = firstoct;
  // schedule constants
  SchedState &h = *g.h_S;
  std::memset(&h, 0, sizeof(h));
  h.lcoarse = lcoarse;
  h.lmax = lmax;
  h.cfl = g.opt.cfl;
  h.dt_param = 1e9;
  h.time_max = 1e9;
  h.nsub = 2;
  for (int L = 0; L < kMaxLevels; L++) h.dx[L] = std::pow(0.5, L);
  CK(cudaMemcpy(g.d_S, &h, sizeof(SchedState), cudaMemcpyHostToDevice));
  rc = emma_hydro_fields_upload(firstoct);
  if (rc != 0) return rc;
  // EMMA_HYDRO_AUTOTUNE=0: no timing pass (plans by the cost model, CTAs at the
  // occupancy limit), e.g. under a profiler, whose overhead distorts the timings
  const char *tune = std::getenv("EMMA_HYDRO_AUTOTUNE");
  if (!(tune != nullptr && tune[0] == '0') && !autotune_tree(g.res, shape_req)) return EMMA_ST_CUDA;
  // batched work list: finest level first, each level's tiles in order
  std::vector<int> all;
  for (int L = lmax; L >= lcoarse; L--)
    for (int i = 0; i < g.res.lev[L].ntiles; i++) all.push_back((L << kWorkSlotShift) | i);
  if (!upload_vec(&g.d_work_all, all)) return EMMA_ST_CUDA;
  g.nwork_all = (int)all.size();
  return 0;
}

int emma_hydro_fields_upload(struct OCT **firstoct) {
  (void)firstoct;
  if (!g.res.valid) {
    fail(EMMA_ST_ARG, "no tree uploaded");
    return EMMA_ST_ARG;
  }
  for (int L = g.res.lcoarse; L <= g.res.lmax; L++) {
    const HostLevel &h = g.res.host.lev[L];
    if (h.noct == 0) continue;
    double *W = current_state(L);
    if (W == nullptr) return EMMA_ST_CUDA;
    // d,u,v,w,p (tracer builds: and the tracers, planes 6.. of a resident state)
    const size_t bytes = sizeof(double) * (5 + kDropinTracer) * 8 * (size_t)h.noct;
    if (!ensure_pin(bytes)) return EMMA_ST_CUDA;
    pack_level(h, 0, g.pin);
#ifdef EMMA_WRADHYD
    for (int t = 0; t < kDropinTracer; t++) {
      double *px = g.pin + (5 + t) * 8LL * h.noct;
      parallel_for(h.noct, [&](long long a0, long long b0) {
        for (long long i = a0; i < b0; i++)
          for (int c = 0; c < 8; c++) px[8 * i + c] = tracer(h.octs[i]->cell[c].field, t);
      });
    }
#endif
    CK(cudaMemcpyAsync(W, g.pin, bytes, cudaMemcpyHostToDevice, g.stream));
    g.h2d_bytes += (long long)bytes;
    CK(mark_stale(L));
    CK(cudaStreamSynchronize(g.stream));
    const DevLevel &dl = g.res.lev[L];
    if (dl.az != nullptr) {  // dual energy: split cells with a stored sound speed of 0
      uint8_t *pz = reinterpret_cast<uint8_t *>(g.pin);
      parallel_for(h.noct, [&](long long a0, long long b0) { pack_az(h, a0, b0, pz); });
      CK(cudaMemcpyAsync(dl.az, pz, (size_t)dl.n8, cudaMemcpyHostToDevice, g.stream));
      CK(cudaMemsetAsync(&g.d_S->azall[L], 0, sizeof(int), g.stream));
      CK(cudaStreamSynchronize(g.stream));
    }
#ifdef EMMA_WGRAV
    // the cells' accelerations, when the tree was uploaded with gravity coupling
    const DevLevel &d = g.res.lev[L];
    if (d.F != nullptr) {
      if (!ensure_pin(3 * bytes / 5)) return EMMA_ST_CUDA;
      parallel_for(h.noct, [&](long long a0, long long b0) { pack_force(h, a0, b0, g.pin); });
      CK(cudaMemcpyAsync(d.F, g.pin, 3 * bytes / 5, cudaMemcpyHostToDevice, g.stream));
      g.h2d_bytes += (long long)(3 * bytes / 5);
      CK(cudaStreamSynchronize(g.stream));
    }
#endif
  }
  return 0;
}

int emma_hydro_tree_download(struct OCT **firstoct) {
  (void)firstoct;
  if (!g.res.valid) {
    fail(EMMA_ST_ARG, "no tree uploaded");
    return EMMA_ST_ARG;
  }
  for (int L = g.res.lcoarse; L <= g.res.lmax; L++) {
    const HostLevel &h = g.res.host.lev[L];
    if (h.noct == 0) continue;
    double *W = current_state(L);
    if (W == nullptr) return EMMA_ST_CUDA;
    const long long n8 = 8LL * h.noct;
    const size_t bytes = sizeof(double) * (5 + kDropinTracer) * (size_t)n8;
    if (!ensure_pin(bytes)) return EMMA_ST_CUDA;
    CK(cudaMemcpyAsync(g.pin, W, bytes, cudaMemcpyDeviceToHost, g.stream));
    g.d2h_bytes += (long long)bytes;
    CK(cudaStreamSynchronize(g.stream));
    const double *p = g.pin;
    parallel_for(h.noct, [&](long long a, long long b) {
      for (long long i = a; i < b; i++) {
        struct OCT *o = h.octs[i];
        for (int c = 0; c < 8; c++) {
          const long long k = 8 * i + c;
          struct Wtype &W = o->cell[c].field;
          W.d = p[k];
          W.u = p[n8 + k];
          W.v = p[2 * n8 + k];
          W.w = p[3 * n8 + k];
          W.p = p[4 * n8 + k];
#ifdef EMMA_WRADHYD
          for (int t = 0; t < kDropinTracer; t++) tracer(W, t) = p[(5 + t) * n8 + k];
#endif
          finish_prims(W);
          if (o->cell[c].child != nullptr) W.a = 0.;  // split cells: as the reference's averaging leaves them
          o->cell[c].fieldnew = W;
        }
      }
    });
  }
  return 0;
}

int emma_hydro_level_noct(int level) {
  if (!g.res.valid || level < g.res.lcoarse || level > g.res.lmax) return 0;
  return g.res.lev[level].noct;
}

long long emma_hydro_level_leaf_cells(int level) {
  if (!g.res.valid || level < g.res.lcoarse || level > g.res.lmax) return 0;
  return g.res.lev[level].leaf;
}

int emma_hydro_get_level_state(int level, double *host_out) {
  if (!level_ok(level) || host_out == nullptr) return EMMA_ST_ARG;
  const DevLevel &d = g.res.lev[level];
  double *W = current_state(level);
  if (W == nullptr) return EMMA_ST_CUDA;
  CK(cudaMemcpyAsync(host_out, W, sizeof(double) * 5 * d.n8, cudaMemcpyDeviceToHost, g.stream));
  g.d2h_bytes += (long long)sizeof(double) * 5 * d.n8;
  CK(cudaStreamSynchronize(g.stream));
  return 0;
}

int emma_hydro_set_level_state(int level, const double *host_in) {
  if (!level_ok(level) || host_in == nullptr) return EMMA_ST_ARG;
  const DevLevel &d = g.res.lev[level];
  double *W = current_state(level);
  if (W == nullptr) return EMMA_ST_CUDA;
  CK(cudaMemcpyAsync(W, host_in, sizeof(double) * 5 * d.n8, cudaMemcpyHostToDevice, g.stream));
  g.h2d_bytes += (long long)sizeof(double) * 5 * d.n8;
  CK(mark_stale(level));
  if (d.az != nullptr) {  // a state set from primitives: every sound speed follows from p and rho
    CK(cudaMemsetAsync(d.az, 0, (size_t)d.n8, g.stream));
    CK(cudaMemsetAsync(&g.d_S->azall[level], 0, sizeof(int), g.stream));
  }
  CK(cudaStreamSynchronize(g.stream));
  return 0;
}

int emma_hydro_set_level_force(int level, const double *host_f) {
  if (!level_ok(level) || host_f == nullptr) return EMMA_ST_ARG;
  const DevLevel &d = g.res.lev[level];
  if (d.F == nullptr) {
    fail(EMMA_ST_ARG, "emma_hydro_set_level_force: the tree was uploaded without gravity coupling");
    return EMMA_ST_ARG;
  }
  CK(cudaMemcpyAsync(d.F, host_f, sizeof(double) * 3 * d.n8, cudaMemcpyHostToDevice, g.stream));
  g.h2d_bytes += (long long)sizeof(double) * 3 * d.n8;
  CK(cudaStreamSynchronize(g.stream));
  return 0;
}

int emma_hydro_set_level_force_device(int level, const double *dev_f) {
  if (!level_ok(level) || dev_f == nullptr) return EMMA_ST_ARG;
  const DevLevel &d = g.res.lev[level];
  if (d.F == nullptr) {
    fail(EMMA_ST_ARG, "emma_hydro_set_level_force_device: the tree was uploaded without gravity coupling");
    return EMMA_ST_ARG;
  }
  CK(cudaMemcpyAsync(d.F, dev_f, sizeof(double) * 3 * d.n8, cudaMemcpyDeviceToDevice, g.stream));
  return 0;
}

int emma_hydro_clean_new(int level) {
  if (!level_ok(level)) return EMMA_ST_ARG;
  const DevLevel &d = g.res.lev[level];
  if (d.n8 == 0 || d.C == nullptr) return 0;
  CK(cudaMemsetAsync(d.C, 0, sizeof(double) * cplanes() * d.n8, g.stream));
  return 0;
}

int emma_hydro_comptstep(int level, double *dt_out) {
  if (!level_ok(level) || dt_out == nullptr) return EMMA_ST_ARG;
  const DevLevel &d = g.res.lev[level];
  double dt = 1e9;
  if (d.n8 > 0) {
    unsigned long long *slot = &g.d_S->smax[level];
    CK(cudaMemsetAsync(slot, 0, sizeof(unsigned long long), g.stream));
    CK(launch_cfl(g.res.d_lv, level, d.n8, nullptr, slot, g.nsm, g.stream));
    g.kernel_launches++;
    CK(cudaMemcpyAsync(&g.h_S->smax[level], slot, sizeof(unsigned long long), cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    double smax;
    std::memcpy(&smax, &g.h_S->smax[level], sizeof(double));
    const double dxcur = std::pow(0.5, level);
    if (smax > 0.) dt = std::fmin(dxcur * g.opt.cfl / (smax * 3.), dt);
  }
  *dt_out = dt;
  return 0;
}

int emma_hydro_advance_level(int level, double dt) {
  if (!level_ok(level)) return EMMA_ST_ARG;
  DevLevel &d = g.res.lev[level];
  if (d.noct == 0) return 0;
  k_bind_level<<<1, 1, 0, g.stream>>>(g.res.d_lv, level, g.res.lcoarse, g.res.lmax, dt);
  CK(cudaGetLastError());
  CK(launch_interp(g.res.d_lv, level, d.nv, nullptr, g.nsm, g.stream, g.res.host.grav));
  if (!launch_batch(g.res.d_lv, d.work, d.ntiles, nullptr, d.leaf, 1u << d.shape, d.ctas, false, false, level))
    return EMMA_ST_CUDA;
  g.c_dirty = true;  // the coarser level's corrections wait for an update of that level
  k_swap_level<<<1, 1, 0, g.stream>>>(g.res.d_lv, level, nullptr);
  CK(cudaGetLastError());
  CK(mark_stale(level));
  if (d.az != nullptr) CK(cudaMemsetAsync(&g.d_S->azall[level], 1, sizeof(int), g.stream));  // nonzero
  g.updates += d.leaf;
  return 0;
}

}  // extern "C"

namespace {

// tile groups the fused kernel of this build runs with `groups` requested (0 = as
// many as fit), 0 if that count is not built
int step_groups_for(int groups) {
  const unsigned variant = (g.opt.dual_energy ? kLaunchDual : 0u) | kLaunchTracers;
  return (g.opt.precision == EMMA_PREC_MIXED) ? step_groups_f32(variant, groups) : step_groups_fp64(variant, groups);
}

// Coarse-step mode of a subcycled resident tree on the graph.  EmmaHydroOptions.
// fused_step -1: separate launches; k > 0: the fused kernel with k tile groups (or
// as many as fit); 0: the autotuner runs five coarse steps in each mode (separate
// launches; the fused kernel with every built group count) from a snapshot of the
// tree's state (level states, level slots, schedule state), restores it after
// each, and keeps the mode whose fastest step (of the last four) is the fastest.
bool choose_step_mode(int nsub) {
  Tree &t = g.res;
  const int lc = t.lcoarse, lf = finest_level();
  if (nsub == 1 || lf == lc || !fused_step_ok()) {
    g.step_groups = 0;
    return true;
  }
  if (g.opt.fused_step > 0) {
    const int k = step_groups_for(g.opt.fused_step);
    g.step_groups = k > 0 ? k : step_groups_for(0);
    return true;
  }
  if (g.step_groups != -2 && g.step_tuned_nsub == nsub && g.step_tuned_prec == g.opt.precision) return true;
  // snapshot
  if (!ck(cudaStreamSynchronize(g.stream), "sync")) return false;
  std::vector<LevelArgs> lv(kMaxLevels);
  SchedState hs;
  unsigned status0 = 0;
  if (!ck(cudaMemcpy(lv.data(), t.d_lv, sizeof(LevelArgs) * kMaxLevels, cudaMemcpyDeviceToHost), "read slots") ||
      !ck(cudaMemcpy(&hs, g.d_S, sizeof(SchedState), cudaMemcpyDeviceToHost), "read schedule") ||
      !ck(cudaMemcpy(&status0, g.d_status, sizeof(unsigned), cudaMemcpyDeviceToHost), "read status"))
    return false;
  std::vector<double *> snap(kMaxLevels, nullptr);
  std::vector<size_t> bytes(kMaxLevels, 0);
  bool ok = true;
  for (int L = lc; L <= lf && ok; L++) {
    bytes[L] = sizeof(double) * (5 + kDropinTracer) * (size_t)t.lev[L].n8;
    ok = ck(cudaMalloc(&snap[L], bytes[L]), "cudaMalloc snapshot") &&
         ck(cudaMemcpyAsync(snap[L], lv[L].W, bytes[L], cudaMemcpyDeviceToDevice, g.stream), "snapshot");
  }
  auto restore = [&]() {
    bool r = ck(cudaMemcpyAsync(t.d_lv, lv.data(), sizeof(LevelArgs) * kMaxLevels, cudaMemcpyHostToDevice, g.stream),
                "restore slots") &&
             ck(cudaMemcpyAsync(g.d_S, &hs, sizeof(SchedState), cudaMemcpyHostToDevice, g.stream), "restore schedule") &&
             ck(cudaMemcpyAsync(g.d_status, &status0, sizeof(unsigned), cudaMemcpyHostToDevice, g.stream), "status") &&
             ck(cudaMemsetAsync(g.d_done, 0, sizeof(unsigned) * kMaxLevels, g.stream), "memset done");
    for (int L = lc; L <= lf && r; L++) {
      r = ck(cudaMemcpyAsync(lv[L].W, snap[L], bytes[L], cudaMemcpyDeviceToDevice, g.stream), "restore state");
      const DevLevel &d = t.lev[L];
      if (r && d.C != nullptr) r = ck(cudaMemsetAsync(d.C, 0, sizeof(double) * cplanes() * d.n8, g.stream), "memset C");
    }
    return r && ck(cudaStreamSynchronize(g.stream), "sync");
  };
  ok = ok && restore();  // also clears corrections left by host-driven calls
  g.c_dirty = false;
  const long long launches0 = g.kernel_launches;
  constexpr int kTimed = 4;
  cudaEvent_t ev[kTimed + 1];
  for (int i = 0; i <= kTimed; i++) ev[i] = get_event();
  for (int k = 0; k < 5; k++) g.step_sweep[k] = 0.;
  int best = 0;
  double best_ms = 0.;
  for (int cand = 0; cand <= 4 && ok; cand++) {
    if (cand > 0 && step_groups_for(cand) != cand) continue;  // this group count is not built
    g.step_groups = cand;
    drop_graph();
    if (!ensure_graph(nsub)) {
      ok = false;
      break;
    }
    // one step to warm up, four timed one by one, from the snapshot each time
    ok = ck(cudaGraphLaunch(g.graph, g.stream), "graph launch") && ck(cudaEventRecord(ev[0], g.stream), "event");
    for (int i = 0; i < kTimed && ok; i++)
      ok = ck(cudaGraphLaunch(g.graph, g.stream), "graph launch") && ck(cudaEventRecord(ev[i + 1], g.stream), "event");
    ok = ok && ck(cudaEventSynchronize(ev[kTimed]), "event");
    double ms = 0.;
    unsigned bits = 0;
    for (int i = 0; i < kTimed && ok; i++) {
      float m = 0.f;
      ok = ck(cudaEventElapsedTime(&m, ev[i], ev[i + 1]), "event time");
      if (i == 0 || m < ms) ms = m;
    }
    if (ok) ok = ck(cudaMemcpy(&bits, g.d_status, sizeof(unsigned), cudaMemcpyDeviceToHost), "status");
    ok = ok && restore();
    if (!ok) break;
    if ((bits & ~status0) != 0) continue;  // a mode that raised a status is not kept
    g.step_sweep[cand] = ms;
    if (best_ms == 0. || ms < best_ms) {
      best_ms = ms;
      best = cand;
    }
  }
  for (int i = 0; i <= kTimed; i++) g.free_events.push_back(ev[i]);
  for (int L = lc; L <= lf; L++) cudaFree(snap[L]);
  g.kernel_launches = launches0;
  drop_graph();
  g.step_groups = ok ? best : 0;
  g.step_tuned_nsub = nsub;
  g.step_tuned_prec = g.opt.precision;
  return ok;
}

}  // namespace

extern "C" {

int emma_hydro_step_tuning(int *groups, double *sweep_ms) {
  if (groups) *groups = g.step_groups;
  if (sweep_ms)
    for (int k = 0; k < 5; k++) sweep_ms[k] = g.step_sweep[k];
  return 0;
}

int emma_hydro_advance_coarse_step(double dt_param, double time_max, int nsub, double *tsim, double *adt) {
  if (!g.res.valid || tsim == nullptr || adt == nullptr) {
    fail(EMMA_ST_ARG, "advance_coarse_step: no tree or null pointer");
    return EMMA_ST_ARG;
  }
  if (!g.opt.use_graph) {
    Sched S{dt_param, time_max, nsub, adt, 0};
    advance_level(S, g.res.lcoarse, *tsim);
    *tsim += adt[g.res.lcoarse - 1];
    return S.err;
  }
  if (!write_sched_params(dt_param, time_max, nsub, tsim, adt)) return EMMA_ST_CUDA;
  int rc = emma_hydro_advance_coarse_step_async(dt_param, time_max, nsub);
  if (rc != 0) return rc;
  return emma_hydro_get_time(tsim, adt);
}

int emma_hydro_advance_coarse_step_async(double dt_param, double time_max, int nsub) {
  if (!g.res.valid || nsub < 1) {
    fail(EMMA_ST_ARG, "advance_coarse_step_async: no tree or nsub < 1");
    return EMMA_ST_ARG;
  }
  SchedState &h = *g.h_S;
  if (h.dt_param != dt_param || h.time_max != time_max || h.nsub != nsub || h.cfl != g.opt.cfl)
    if (!write_sched_params(dt_param, time_max, nsub, nullptr, nullptr)) return EMMA_ST_CUDA;
  if (!choose_step_mode(nsub)) return EMMA_ST_CUDA;
  if (!ensure_graph(nsub)) return EMMA_ST_CUDA;
  if (g.graph_is_fused && g.c_dirty) {  // the fused step expects every correction at zero
    for (int L = g.res.lcoarse; L <= g.res.lmax; L++) {
      const DevLevel &d = g.res.lev[L];
      if (d.C != nullptr) CK(cudaMemsetAsync(d.C, 0, sizeof(double) * cplanes() * d.n8, g.stream));
    }
    g.c_dirty = false;
  }
  CK(cudaGraphLaunch(g.graph, g.stream));
  if (!g.graph_is_fused) g.c_dirty = true;
  return 0;
}

int emma_hydro_get_time(double *tsim, double *adt) {
  if (!g.res.valid) return EMMA_ST_ARG;
  CK(cudaMemcpyAsync(g.h_S, g.d_S, sizeof(SchedState), cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  if (tsim) *tsim = g.h_S->tsim;
  if (adt)
    for (int l = 0; l < g.res.lmax && l < kMaxLevels; l++) adt[l] = g.h_S->adt[l];
  return 0;
}

int emma_hydro_set_time(double tsim, const double *adt) {
  if (!g.res.valid) return EMMA_ST_ARG;
  SchedState &h = *g.h_S;
  return write_sched_params(h.dt_param == 0. ? 1e9 : h.dt_param, h.time_max == 0. ? 1e9 : h.time_max,
                            h.nsub == 0 ? 2 : h.nsub, &tsim, adt)
             ? 0
             : EMMA_ST_CUDA;
}

long long emma_hydro_cell_updates(void) {
  long long dev = 0;
  if (g.ready && g.res.valid) {
    long long *p = &g.h_S->updates;
    cudaMemcpyAsync(p, &g.d_S->updates, sizeof(long long), cudaMemcpyDeviceToHost, g.stream);
    cudaStreamSynchronize(g.stream);
    dev = *p;
  }
  return g.updates + dev;
}

long long emma_hydro_kernel_launches(void) { return g.kernel_launches; }

int emma_hydro_dropin_profile(double *ms8) {
  if (ms8 == nullptr) return EMMA_ST_ARG;
  for (int i = 0; i < 8; i++) ms8[i] = g.dropin_ms[i];
  return 0;
}

int emma_hydro_transfer_bytes(long long *h2d, long long *d2h) {
  if (h2d == nullptr || d2h == nullptr) return EMMA_ST_ARG;
  *h2d = g.h2d_bytes;
  *d2h = g.d2h_bytes;
  return 0;
}

void emma_hydro_reset_counters(void) {
  g.updates = 0;
  g.kernel_launches = 0;
  g.h2d_bytes = g.d2h_bytes = 0;
  if (g.ready) {
    cudaStreamSynchronize(g.stream);
    if (g.d_S) cudaMemsetAsync(&g.d_S->updates, 0, sizeof(long long), g.stream);
    cudaStreamSynchronize(g.stream);
  }
  for (auto &t : g.launches) {
    g.free_events.push_back(t.a);
    g.free_events.push_back(t.b);
  }
  g.launches.clear();
}

int emma_hydro_probe_wait_timeout(long long polls) {
  if (!g.res.valid) {
    fail(EMMA_ST_ARG, "no tree uploaded");
    return EMMA_ST_ARG;
  }
  if (polls < 0) return EMMA_ST_ARG;
  const int L = g.res.lcoarse;
  const DevLevel &d = g.res.lev[L];
  if (d.ntiles == 0) return EMMA_ST_ARG;
  unsigned status0 = 0, bits = 0;
  CK(cudaStreamSynchronize(g.stream));
  CK(cudaMemcpy(&status0, g.d_status, sizeof(unsigned), cudaMemcpyDeviceToHost));
  CK(cudaMemset(g.d_status, 0, sizeof(unsigned)));
  CK(cudaMemset(g.d_done, 0, sizeof(unsigned) * kMaxLevels));
  // dt = 0, then the level's update waits for all of the level's own tiles:
  // a count that no tile can reach before its own wait ends
  k_bind_level<<<1, 1, 0, g.stream>>>(g.res.d_lv, L, g.res.lcoarse, g.res.lmax, 0.);
  const int self = L;
  CK(cudaMemcpyAsync(&g.res.d_lv[L].wait_slot, &self, sizeof(int), cudaMemcpyHostToDevice, g.stream));
  const long long limit0 = g.wait_limit;
  const bool timing0 = g.timing;
  g.wait_limit = polls;
  g.timing = false;
  const bool ok = launch_batch(g.res.d_lv, d.work, d.ntiles, nullptr, 0, 1u << d.shape, d.ctas);
  g.wait_limit = limit0;
  g.timing = timing0;
  k_bind_level<<<1, 1, 0, g.stream>>>(g.res.d_lv, L, g.res.lcoarse, g.res.lmax, 0.);  // wait_slot back to -1
  CK(cudaStreamSynchronize(g.stream));
  if (!ok) return EMMA_ST_CUDA;
  CK(cudaMemcpy(&bits, g.d_status, sizeof(unsigned), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(g.d_status, &status0, sizeof(unsigned), cudaMemcpyHostToDevice));
  CK(cudaMemset(g.d_done, 0, sizeof(unsigned) * kMaxLevels));
  return (int)bits;
}

int emma_hydro_graph_info(int *fused, int *ctas, int *groups, int *kernel_nodes) {
  if (fused) *fused = g.graph_is_fused ? 1 : 0;
  if (ctas) *ctas = g.graph_is_fused ? g.step_grid : 0;
  if (groups) *groups = g.graph_is_fused ? g.step_threads / kThreads : 0;
  if (kernel_nodes) *kernel_nodes = g.graph ? g.graph_kernels : 0;
  return 0;
}

int emma_hydro_timed_coarse_steps(double dt_param, double time_max, int nsub, int nsteps, double *ms) {
  if (ms == nullptr || nsteps < 1) return EMMA_ST_ARG;
  cudaEvent_t a = get_event(), b = get_event();
  int rc = 0;
  CK(cudaEventRecord(a, g.stream));
  for (int i = 0; i < nsteps && rc == 0; i++) rc = emma_hydro_advance_coarse_step_async(dt_param, time_max, nsub);
  CK(cudaEventRecord(b, g.stream));
  CK(cudaEventSynchronize(b));
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, a, b));
  *ms = f;
  g.free_events.push_back(a);
  g.free_events.push_back(b);
  return rc;
}

int emma_hydro_fused_job_log(int max, int *kinds, int *levels, double *release_us, double *schedule_us) {
  if (!g.ready || max < 0) return -EMMA_ST_ARG;
  std::vector<StepJobRecord> rec(kStepJobLog);
  if (cudaStreamSynchronize(g.stream) != cudaSuccess ||
      cudaMemcpy(rec.data(), g.d_jobt, sizeof(StepJobRecord) * kStepJobLog, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -EMMA_ST_CUDA;
  int n = 0;
  while (n < (int)kStepJobLog && rec[n].kind >= kJobLevel && rec[n].kind <= kJobDone) {
    if (n < max) {
      if (kinds) kinds[n] = rec[n].kind;
      if (levels) levels[n] = rec[n].L;
      if (release_us) release_us[n] = (double)(long long)(rec[n].t - rec[0].t) * 1e-3;
      if (schedule_us) schedule_us[n] = (double)(long long)(rec[n].t - rec[n].t_all) * 1e-3;
    }
    if (rec[n++].kind == kJobDone) break;
  }
  return n;
}

int emma_hydro_column_tuning(int level, int *planes, double *sweep_ms) {
  if (!level_ok(level)) return EMMA_ST_ARG;
  const DevLevel &d = g.res.lev[level];
  if (planes) *planes = column_nz(level);
  if (sweep_ms)
    for (int i = 0; i < 6; i++) sweep_ms[i] = d.col_sweep_ms[i];
  return 0;
}

int emma_hydro_column_xshfl(int level, int *xshfl, double *ms) {
  if (!level_ok(level)) return EMMA_ST_ARG;
  const DevLevel &d = g.res.lev[level];
  if (xshfl) *xshfl = column_nz(level) > 0 ? column_xs(level) : 0;
  if (ms) {
    ms[0] = d.col_xs_ms[0];
    ms[1] = d.col_xs_ms[1];
  }
  return 0;
}

int emma_hydro_column_balanced(int level, int *balanced, double *ms) {
  if (!level_ok(level)) return EMMA_ST_ARG;
  const DevLevel &d = g.res.lev[level];
  if (balanced) *balanced = column_nz(level) > 0 ? column_bal(level) : 0;
  if (ms) {
    ms[0] = d.col_bal_ms[0];
    ms[1] = d.col_bal_ms[1];
  }
  return 0;
}

int emma_hydro_tuning(int level, int *tile_octs, int *ctas_per_sm, double *sweep_ms) {
  if (!level_ok(level)) return EMMA_ST_ARG;
  const DevLevel &d = g.res.lev[level];
  if (tile_octs) *tile_octs = kShapes[d.shape].octs();
  if (ctas_per_sm) *ctas_per_sm = d.ctas;
  if (sweep_ms)
    for (int s = 0; s < kNumShapes; s++)
      for (int c = 0; c < 4; c++) sweep_ms[4 * s + c] = d.sweep_ms[s][c];
  return d.tuned ? 0 : EMMA_ST_ARG;
}

int emma_hydro_kernel_timing(double *avg_ms, long long *launches, long long *cells) {
  if (!g.ready) return EMMA_ST_ARG;
  CK(cudaStreamSynchronize(g.stream));
  double tot = 0.;
  long long nc = 0;
  for (auto &t : g.launches) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t.a, t.b);
    tot += ms;
    nc += t.cells;
  }
  if (avg_ms) *avg_ms = g.launches.empty() ? 0. : tot / (double)g.launches.size();
  if (launches) *launches = (long long)g.launches.size();
  if (cells) *cells = nc;
  return 0;
}

int emma_hydro_kernel_timing_level(int level, double *total_ms, long long *launches, long long *cells) {
  if (!g.ready) return EMMA_ST_ARG;
  CK(cudaStreamSynchronize(g.stream));
  double tot = 0.;
  long long n = 0, nc = 0;
  for (auto &t : g.launches) {
    if (t.level != level) continue;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t.a, t.b);
    tot += ms;
    nc += t.cells;
    n++;
  }
  if (total_ms) *total_ms = tot;
  if (launches) *launches = n;
  if (cells) *cells = nc;
  return 0;
}

// Host-only planning diagnostics (no GPU needed): builds and validates the tile
// plans of levels lcoarse..lmax and reports, per level, {octs, tiles, max staged
// octs per tile, staged octs of all tiles, leaf cells}.  Returns the status bits
// of the planning.
int emma_hydro_plan_stats(struct OCT **firstoct, int lcoarse, int lmax, int trans, long long *stats5) {
  HostTree H;
  std::string err;
  int rc = build_host_tree(firstoct, lcoarse, lmax, 0, trans, lcoarse, lmax, H, err);
  if (rc != 0) {
    fail((unsigned)rc, err);
    return rc;
  }
  for (int L = lcoarse; L <= lmax; L++) {
    const HostLevel &h = H.lev[L];
    long long ms = 0, mh = 0;
    for (size_t t = 0; t < h.tiles.size(); t++) {
      long long s = 0;
      const int ns = kShapes[h.shape].tile_slots();
      for (int i = 0; i < ns; i++) s += (h.keys[t * ns + i] != kKeyNone);
      ms = std::max(ms, s);
      mh += s;
    }
    long long *o = stats5 + 5 * (L - lcoarse);
    o[0] = h.nown;
    o[1] = (long long)h.tiles.size();
    o[2] = ms;
    o[3] = mh;
    o[4] = h.leaf;
  }
  return 0;
}

// ------------------------------------------------------------- drop-in path
// The drop-in entries work on the caller's host tree on every call: mirror the
// level's neighbourhood (levels L-1..L+1, cached while the tree is unchanged),
// upload field/fieldnew, run the level kernel, write fieldnew back and apply
// the fine->coarse corrections to the coarser neighbours' fieldnew.

static int dropin_rank(struct CPUINFO *cpu) { return cpu ? *reinterpret_cast<const int *>(cpu) : 0; }

// [lo, hi) lies in mappings of this process that are readable (/proc/self/maps,
// whose entries come sorted by address); false when it cannot tell.
static bool range_readable(uintptr_t lo, uintptr_t hi) {
  const int fd = open("/proc/self/maps", O_RDONLY | O_CLOEXEC);
  if (fd < 0) return false;
  std::string text;
  char buf[1 << 16];
  for (;;) {
    const ssize_t r = read(fd, buf, sizeof(buf));
    if (r < 0) {
      close(fd);
      return false;
    }
    if (r == 0) break;
    text.append(buf, (size_t)r);
  }
  close(fd);
  uintptr_t cur = lo;  // [lo, cur) is covered
  const char *s = text.c_str();
  while (*s != '\0' && cur < hi) {
    char *e = nullptr;
    const uintptr_t a = (uintptr_t)std::strtoull(s, &e, 16);
    if (e == nullptr || *e != '-') return false;
    const uintptr_t b = (uintptr_t)std::strtoull(e + 1, &e, 16);
    if (e == nullptr || *e != ' ') return false;
    const bool readable = e[1] == 'r';
    if (a > cur) return false;  // a gap before the next mapping
    if (b > cur) {
      if (!readable) return false;
      cur = b;
    }
    const char *nl = std::strchr(e, '\n');
    if (nl == nullptr) break;
    s = nl + 1;
  }
  return cur >= hi;
}

// Oct pointers of level `level` in list order (firstoct[level-1] on).  The
// result stays valid until the next walk of the level.
//
// A list unchanged since the previous walk is confirmed in parallel: every
// oct's `next` is the following oct of that walk and the last one's is NULL.
// The confirmation reads the cached octs only when all of them lie in readable
// mappings of this process (the caller's oct pool), so it cannot fault whatever
// the caller did to its tree since; a list that changed fails it.  Otherwise
// (or when it fails) the serial walk follows `next` (one cache line per oct),
// prefetching those lines along the previous walk (a prefetch never faults).
static const std::vector<struct OCT *> &walk_level(struct OCT **firstoct, int level) {
  std::vector<struct OCT *> &prev = g.lists[level];
  const size_t np = prev.size();
  constexpr size_t kParallelConfirm = 1 << 15;
  if (np >= kParallelConfirm && prev[0] == firstoct[level - 1] &&
      range_readable(g.list_lo[level], g.list_hi[level] + sizeof(struct OCT))) {
    std::atomic<bool> same{true};
    parallel_for((long long)np, [&](long long a, long long b) {
      for (long long i = a; i < b; i++) {
        const struct OCT *nx = (size_t)i + 1 < np ? prev[(size_t)i + 1] : nullptr;
        if (prev[(size_t)i]->next != nx) {
          same.store(false, std::memory_order_relaxed);
          return;
        }
        if ((i & 4095) == 0 && !same.load(std::memory_order_relaxed)) return;
      }
    });
    if (same.load()) return prev;
  }
  std::vector<struct OCT *> &out = g.list_tmp;
  out.clear();
  constexpr size_t kAhead = 24;
  size_t i = 0;
  uintptr_t lo = UINTPTR_MAX, hi = 0;
  for (struct OCT *o = firstoct[level - 1]; o != nullptr; o = o->next, i++) {
    if (i + kAhead < np) __builtin_prefetch(&prev[i + kAhead]->next);
    out.push_back(o);
    lo = std::min(lo, (uintptr_t)o);
    hi = std::max(hi, (uintptr_t)o);
  }
  prev.swap(out);
  g.list_lo[level] = lo;
  g.list_hi[level] = hi;
  return prev;
}

static inline unsigned long long mix64(unsigned long long z) {  // SplitMix64 finaliser
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// Order-sensitive hash of a level's oct addresses, child-presence bits and
// ownership (cpu == rank): the parts of the tree a drop-in mirror depends on;
// `*split` = a cell has a child.
static unsigned long long level_hash(const std::vector<struct OCT *> &v, int rank, bool *split) {
  const long long n = (long long)v.size();
  const long long chunk = 8192;
  const long long nchunk = (n + chunk - 1) / chunk;
  std::vector<unsigned long long> part((size_t)nchunk, 0);
  std::vector<char> any((size_t)nchunk, 0);
  // chunk-wise partial sums: the total does not depend on the thread count
  parallel_for(n, [&](long long a, long long b) {
    for (long long j = (a + chunk - 1) / chunk; j * chunk < b; j++) {
      unsigned long long s = 0;
      bool f = false;
      const long long e = std::min(n, (j + 1) * chunk);
      for (long long i = j * chunk; i < e; i++) {
        const struct OCT *o = v[i];
        unsigned long long bits = 0;
        for (int c = 0; c < 8; c++) bits |= (unsigned long long)(o->cell[c].child != nullptr) << c;
        f = f || bits != 0;
        bits |= (unsigned long long)(o->cpu == rank) << 8;
        s += mix64((unsigned long long)(uintptr_t)o ^ (bits << 56) ^ ((unsigned long long)i * 0x9e3779b97f4a7c15ULL));
      }
      part[j] = s;
      any[j] = f;
    }
  }, chunk);
  unsigned long long h = (unsigned long long)n;
  bool f = false;
  for (long long j = 0; j < nchunk; j++) {
    h += part[j];
    f = f || any[j];
  }
  *split = f;
  return h;
}

// One drop-in advance of `level` on the host tree.  With `final_update` it also
// performs HydroSolver's closing loop on the level (field := fieldnew on
// leaves, primitive mean of the children on split cells), the leaf copy fused
// into the download.  Returns the number of octs advanced (0 on error).
static int dropin_advance(struct OCT **firstoct, int level, struct CPUINFO *cpu, double dtnew, bool final_update) {
  if (!g.ready && emma_hydro_init(nullptr) != 0) return 0;
  if (firstoct == nullptr || level < 2 || level >= kMaxLevels - 1 || firstoct[level - 1] == nullptr) return 0;
  if (kDropinTracer && (g.opt.dual_energy || g.opt.trans_flags)) {
    fail(EMMA_ST_ARG, "the -DWRADHYD library has neither dual energy nor transmissive boundaries");
    return 0;
  }
  const int rank = dropin_rank(cpu);
  const auto t0 = Clock::now();
  // levels present around `level`: L-1 always exists; L+1 only if a cell is split
  bool split_l = false, unused = false;
  const std::vector<struct OCT *> &wl = walk_level(firstoct, level);
  const std::vector<struct OCT *> &wc = walk_level(firstoct, level - 1);
  std::vector<unsigned long long> sig;
  sig.push_back((unsigned long long)(uintptr_t)firstoct);
  sig.push_back(level_hash(wc, rank, &unused));
  sig.push_back(level_hash(wl, rank, &split_l));
  if (split_l) sig.push_back(level_hash(walk_level(firstoct, level + 1), rank, &unused));
  const int lo = level - 1, hi = split_l ? level + 1 : level;
  const auto tw = Clock::now();
  Ctx::DropCache &cache = g.drop[level];
  if (cache.first != firstoct || sig != cache.sig || !cache.t.valid) {
    cudaStreamSynchronize(g.stream);
    free_tree(cache.t);
    cache.first = nullptr;
    cache.sig.clear();
    std::string err;
    std::vector<int> shapes((size_t)hi + 1, std::max(-1, requested_shape(g.opt.tile_octs)));
    int rc = build_host_tree(firstoct, lo, hi, rank, g.opt.trans_flags, level, level, cache.t.host, err,
                             shapes.data(), kDropinGrav, g.opt.dual_energy);
    if (rc != 0) {
      fail((unsigned)rc, err);
      return 0;
    }
    if (!alloc_tree(cache.t.host, cache.t, true)) return 0;
    cache.first = firstoct;
    cache.sig = sig;
  }
  Tree &T = cache.t;
  HostTree &H = T.host;
  const HostLevel &h = H.lev[level];
  const HostLevel &hc = H.lev[level - 1];
  DevLevel &d = T.lev[level];
  DevLevel &dc = T.lev[level - 1];
  if (h.nown == 0) return 0;
  const long long n8 = d.n8, nc8 = dc.n8;
  const bool coarse = nc8 > 0 && h.reads_coarse && dc.C != nullptr;
  // pinned staging: level field with E (and dX) (kFieldPlanes planes; the new state on
  // the way back) | coarser level (5 planes, and dX) | gravity builds: level and
  // coarser accelerations (3 + 3 planes) | device status word
  const long long nf = kDropinGrav ? 3 * (n8 + nc8) : 0, ncp = cplanes();
  // (+ n8 bytes for the dual-energy sound-speed flags after the status word)
  if (!ensure_pin(sizeof(double) * (kFieldPlanes * n8 + ncp * nc8 + nf + 2) + (size_t)n8) || !ensure_range_events())
    return 0;
  double *pw = g.pin, *pc = g.pin + kFieldPlanes * n8;
  [[maybe_unused]] double *pf = pc + ncp * nc8, *pfc = pf + 3 * n8;
  unsigned *pst = reinterpret_cast<unsigned *>(pc + ncp * nc8 + nf);
  const auto t1 = Clock::now();
  // upload: each host thread packs its oct range in sub-ranges (field and the
  // cells whose fieldnew differs, in one pass over the cells) and queues one
  // pitched copy of the 6 planes of each sub-range as soon as it is packed, so the
  // copy engine runs while the rest is still being packed
  if (d.WB == nullptr) {
    fail(EMMA_ST_TREE, "drop-in level without staging block");
    return 0;
  }
  const size_t pitch = sizeof(double) * (size_t)n8;
  const long long sub = dropin_subrange(h.noct);
  std::atomic<bool> copies_ok{true};
  for (auto &e : g.exc) e.clear();
  parallel_ranges(h.noct, [&](int t, long long a0, long long b0) {
    for (long long s0 = a0; s0 < b0; s0 += sub) {
      const long long s1 = std::min(b0, s0 + sub);
      pack_cells(h, s0, s1, pw, g.exc[t]);
      if (cudaMemcpy2DAsync(d.WB + 8 * s0, pitch, pw + 8 * s0, pitch, sizeof(double) * 8 * (s1 - s0), kFieldPlanes,
                            cudaMemcpyHostToDevice, g.stream) != cudaSuccess)
        copies_ok = false;
#ifdef EMMA_WGRAV
      pack_force(h, s0, s1, pf);
      if (d.F == nullptr || cudaMemcpy2DAsync(d.F + 8 * s0, pitch, pf + 8 * s0, pitch, sizeof(double) * 8 * (s1 - s0),
                                              3, cudaMemcpyHostToDevice, g.stream) != cudaSuccess)
        copies_ok = false;
#endif
    }
  });
  if (!copies_ok) return ck(cudaGetLastError(), "H2D level state"), 0;
  {
    // the base fieldnew: field, then the cells where it differs
    size_t nexc = 0;
    for (auto &e : g.exc) nexc += e.size() / kExcRec;
    const size_t eb = sizeof(double) * kExcRec * std::max<size_t>(nexc, 1);
    if (eb > g.pin_exc_bytes) {
      if (g.pin_exc) cudaFreeHost(g.pin_exc);
      g.pin_exc = nullptr;
      g.pin_exc_bytes = 0;
      if (!ck(cudaMallocHost(&g.pin_exc, eb), "cudaMallocHost exceptions")) return 0;
      g.pin_exc_bytes = eb;
    }
    if (eb > g.d_exc_bytes) {
      cudaFree(g.d_exc);
      g.d_exc = nullptr;
      g.d_exc_bytes = 0;
      if (!ck(cudaMalloc(&g.d_exc, eb), "cudaMalloc exceptions")) return 0;
      g.d_exc_bytes = eb;
    }
    size_t at = 0;
    for (auto &e : g.exc) {
      std::memcpy(g.pin_exc + at, e.data(), sizeof(double) * e.size());
      at += e.size();
    }
    if (nexc > 0 &&
        !ck(cudaMemcpyAsync(g.d_exc, g.pin_exc, sizeof(double) * kExcRec * nexc, cudaMemcpyHostToDevice, g.stream),
            "H2D exceptions"))
      return 0;
    if (!ck(launch_dropin_base(d.WB, d.B, n8, g.d_exc, (long long)nexc, g.nsm, g.stream, kFieldPlanes, kExcRec),
            "base launch"))
      return 0;
    g.h2d_bytes += (long long)(sizeof(double) * kExcRec * nexc);
  }
  if (d.az != nullptr) {  // dual energy: the split cells' stored sound speeds of 0
    uint8_t *pz = reinterpret_cast<uint8_t *>(pst + 4);
    parallel_for(h.noct, [&](long long a0, long long b0) { pack_az(h, a0, b0, pz); });
    if (!ck(cudaMemcpyAsync(d.az, pz, (size_t)n8, cudaMemcpyHostToDevice, g.stream), "H2D az")) return 0;
  }
  g.h2d_bytes += (long long)sizeof(double) * (kFieldPlanes + 3 * kDropinGrav) * n8;
  if (coarse) {
    pack_level(hc, 0, pc);
    if (!ck(cudaMemcpyAsync(dc.W0, pc, sizeof(double) * 5 * nc8, cudaMemcpyHostToDevice, g.stream), "H2D Wc"))
      return 0;
    g.h2d_bytes += (long long)sizeof(double) * 5 * nc8;
#ifdef EMMA_WRADHYD
    // the coarser level's tracers, for the fractions of its injected cells
    double *px = pc + 5 * nc8;
    parallel_for(hc.noct, [&](long long a0, long long b0) {
      for (long long i = a0; i < b0; i++)
        for (int c = 0; c < 8; c++)
          for (int t = 0; t < kDropinTracer; t++) px[t * nc8 + 8 * i + c] = tracer(hc.octs[i]->cell[c].field, t);
    });
    if (dc.X == nullptr || !ck(cudaMemcpyAsync(dc.X, px, sizeof(double) * kDropinTracer * nc8, cudaMemcpyHostToDevice,
                                               g.stream),
                               "H2D Xc"))
      return 0;
    g.h2d_bytes += (long long)sizeof(double) * kDropinTracer * nc8;
#endif
    if (!ck(cudaMemsetAsync(dc.C, 0, sizeof(double) * ncp * nc8, g.stream), "memset Cc")) return 0;
  }
#ifdef EMMA_WGRAV
  // the coarser level's accelerations, for the forces of its injected cells
  if (d.nv > 0 && dc.F != nullptr) {
    parallel_for(hc.noct, [&](long long a0, long long b0) { pack_force(hc, a0, b0, pfc); });
    if (!ck(cudaMemcpyAsync(dc.F, pfc, sizeof(double) * 3 * nc8, cudaMemcpyHostToDevice, g.stream), "H2D Fc"))
      return 0;
    g.h2d_bytes += (long long)sizeof(double) * 3 * nc8;
  }
#endif
  const auto t2 = Clock::now();
  LevelArgs a;
  std::memset(&a, 0, sizeof(a));
  a.L = level;
  a.noct = d.noct;
  a.W = d.W0;
  a.Wn = d.W1;
  a.C = nullptr;
  a.B = d.B;
  a.Wc = coarse ? dc.W0 : nullptr;
  a.Cc = coarse ? dc.C : nullptr;
  a.nc8 = nc8;
  a.Wf = nullptr;
  a.split = d.split;
  a.child = d.child;
  a.tiles = d.tiles;
  a.keys = d.keys;
  a.shape = h.shape;
  a.Wv = d.Wv;
  a.vcell = d.vcell;
  a.nv = d.nv;
  a.dt = dtnew;
  a.dx = std::pow(0.5, level);
  a.ntiles = d.ntiles;
  a.wait_slot = -1;
  a.leaf = d.leaf;
  // gravity builds: the caller applies grav_correction itself (src/advanceamr.c:999)
  a.F = d.F;
  a.Fc = dc.F;
  a.Fv = d.Fv;
  a.gcorr = 0;
  a.wv_inject = H.grav;
  a.az = d.az;  // dual energy: from the caller's cells, every call
  a.azall = nullptr;
  if (kDropinTracer) {  // the tracer planes (the union slots of gravity and dual energy)
    a.X = d.X;
    a.Xc = coarse ? dc.X : nullptr;
    a.Xn = d.Xn;
    a.BX = d.B + 6 * n8;
  }
  k_set_args<<<1, 1, 0, g.stream>>>(T.d_lv, level, a);
  if (!ck(cudaGetLastError(), "k_set_args")) return 0;
  if (!ck(launch_interp(T.d_lv, level, d.nv, nullptr, g.nsm, g.stream, H.grav != 0), "interpolation launch"))
    return 0;
  if (!launch_batch(T.d_lv, d.work, d.ntiles, nullptr, d.leaf, 1u << d.shape, d.ctas, false, H.grav != 0)) return 0;
  // device status and the corrections first, then the level's new state range by
  // range: each host thread waits for its own range and unpacks it into fieldnew
  // (and field, for HydroSolver) while later ranges are still being copied
  *pst = 0;
  if (!ck(cudaMemcpyAsync(pst, g.d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, g.stream), "D2H status"))
    return 0;
  if (coarse) {
    if (!ck(cudaMemcpyAsync(pc, dc.C, sizeof(double) * ncp * nc8, cudaMemcpyDeviceToHost, g.stream), "D2H Cc"))
      return 0;
    g.d2h_bytes += (long long)sizeof(double) * ncp * nc8;
  }
  const auto t3 = Clock::now();
  std::atomic<bool> wait_ok{true};
  std::atomic<long long> wait_ns{0};
  const unsigned bad = EMMA_ST_TREE | EMMA_ST_CUDA;
  // this rank's octs only (the first nown): octs of other ranks are not advanced
  const long long sub_own = dropin_subrange(h.nown);
  parallel_ranges(h.nown, [&](int t, long long a0, long long b0) {
    // queue the copies of all sub-ranges of this thread, each followed by an event
    cudaEvent_t *ev = &g.range_ev[(size_t)t * kSubRanges];
    int nq = 0;
    for (long long s0 = a0; s0 < b0 && nq < kSubRanges; s0 += sub_own, nq++) {
      const long long s1 = std::min(b0, s0 + sub_own);
      if (cudaMemcpy2DAsync(pw + 8 * s0, pitch, d.W1 + 8 * s0, pitch, sizeof(double) * 8 * (s1 - s0),
                            5 + kDropinTracer, cudaMemcpyDeviceToHost, g.stream) != cudaSuccess ||
          cudaEventRecord(ev[nq], g.stream) != cudaSuccess) {
        wait_ok = false;
        return;
      }
    }
    // then unpack each as it lands
    int k = 0;
    for (long long s0 = a0; s0 < b0 && k < nq; s0 += sub_own, k++) {
      const auto w0 = Clock::now();
      const bool ok = cudaEventSynchronize(ev[k]) == cudaSuccess;
      wait_ns += std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - w0).count();
      if (!ok) {
        wait_ok = false;
        return;
      }
      // a kernel that found an invalid state leaves the host tree as it was
      if ((g.status | *reinterpret_cast<volatile unsigned *>(pst)) & bad) return;
      unpack_cells(h, s0, std::min(b0, s0 + sub_own), pw, final_update);
    }
  });
  if (!wait_ok) return ck(cudaStreamSynchronize(g.stream), "D2H level state"), ck(cudaGetLastError(), "D2H"), 0;
  g.d2h_bytes += (long long)sizeof(double) * (5 + kDropinTracer) * 8 * h.nown;
  g.status |= *pst;
  if (g.status & bad) return 0;
  const auto t4 = Clock::now();
  g.dropin_ms[3] = std::chrono::duration<double, std::milli>(t4 - t2).count();
  g.dropin_ms[4] = 1e-6 * (double)wait_ns.load() / (double)std::max<size_t>(1, range_threads(h.nown));
  // fine -> coarse corrections: fieldnew = U2W(W2U(fieldnew) + dU) per coarse cell
  if (coarse) {
    const double *p = pc;
    const bool dual = g.opt.dual_energy != 0;
    for (int32_t k : h.inj_cells) {
      struct Wtype &W = hc.octs[k >> 3]->cell[k & 7].fieldnew;
      double Ud = W.d, Udu = W.d * W.u, Udv = W.d * W.v, Udw = W.d * W.w, UE = W.E, Ue = W.p / (kG - 1.);
      Ud += p[k];
      Udu += p[nc8 + k];
      Udv += p[2 * nc8 + k];
      Udw += p[3 * nc8 + k];
      UE += p[4 * nc8 + k];
      if (dual) Ue += p[5 * nc8 + k];
      const double dl = (Ud == 0. ? 10. : Ud);
      W.d = Ud;
      W.u = Udu / dl;
      W.v = Udv / dl;
      W.w = Udw / dl;
      // U2W: the pressure from E - Ekin, or from the tracked eint (-DDUAL_E)
      W.p = dual ? Ue * (kG - 1.) : (kG - 1.) * (UE - ((Udu) * (Udu) + (Udv) * (Udv) + (Udw) * (Udw)) / (dl)*0.5);
      W.E = UE;
      W.a = std::sqrt(kG * W.p / dl);
#ifdef EMMA_WRADHYD
      for (int t = 0; t < kDropinTracer; t++)  // U.dT = W.dT, corrected, U2W (src/hydro_utils.c:3277-3281)
        tracer(W, t) = tracer(W, t) + p[(kXPlane + t) * nc8 + k];
#endif
    }
  }
  g.updates += d.leaf;
  const auto t5 = Clock::now();
  // the rest of the final update: split cells of this rank's octs (the octs of
  // other ranks are left to the caller's exchange, src/hydro_utils.c:3408-3483)
  if (final_update && split_l) {
    parallel_for((long long)wl.size(), [&](long long a0, long long b0) {
      for (long long i = a0; i < b0; i++) {
        struct OCT *o = wl[i];
        if (o->cpu != rank) continue;
        for (int c = 0; c < 8; c++) {
          struct CELL *cell = &o->cell[c];
          if (cell->child == nullptr) continue;
          struct Wtype W;
          std::memset(&W, 0, sizeof(W));
          for (int j = 0; j < 8; j++) {
            const struct Wtype &Wc = cell->child->cell[j].field;
            W.d += Wc.d * 0.125;
            W.u += Wc.u * 0.125;
            W.v += Wc.v * 0.125;
            W.w += Wc.w * 0.125;
            W.p += Wc.p * 0.125;
#ifdef EMMA_WRADHYD
            for (int t = 0; t < kDropinTracer; t++) tracer(W, t) += tracer(Wc, t) * 0.125;  // src/hydro_utils.c:3446-3460
#endif
          }
          W.E = W.p / (kG - 1.) + 0.5 * W.d * (W.u * W.u + W.v * W.v + W.w * W.w);
          cell->field = W;
        }
      }
    });
  }
  const auto t6 = Clock::now();
  auto ms = [](Clock::time_point x, Clock::time_point y) { return std::chrono::duration<double, std::milli>(y - x).count(); };
  g.dropin_ms[0] = ms(t0, tw);
  g.dropin_ms[1] = ms(tw, t1);
  g.dropin_ms[2] = ms(t1, t2);
  g.dropin_ms[5] = ms(t4, t5);
  g.dropin_ms[6] = ms(t5, t6);
  g.dropin_ms[7] = ms(t0, t6);
  return h.nown;
}

int advancehydroGPU(struct OCT **firstoct, int level, struct CPUINFO *cpu, struct HGRID *stencil, int stride,
                    REAL dxcur, REAL dtnew) {
  (void)stencil;
  (void)stride;
  (void)dxcur;
  return dropin_advance(firstoct, level, cpu, dtnew, false);
}

void HydroSolver(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct CPUINFO *cpu,
                 struct HGRID *stencil, int stride, REAL dtnew) {
  (void)param;
  (void)stencil;
  (void)stride;
  dropin_advance(firstoct, level, cpu, dtnew, true);
}

// The leading members of the reference's struct RUNPARAMS (src/prototypes.h,
// npartmax..lmax, REAL = double); clean_new_hydro reads lcoarse.
struct RunParamsHead {
  int npartmax, ngridmax, nbuff, ndumps;
  double dt_dump;
  int nsteps, lcoarse, lmax;
};
static_assert(offsetof(RunParamsHead, lcoarse) == 28, "RUNPARAMS head layout");

// fieldnew := field on every cell of the level (src/hydro_utils.c:3501-3522).
// A multi-rank run (-DWMPI, :3524-3544) also zeroes fieldnew of the octs of
// other ranks one level coarser when level > lcoarse, so that they collect only
// this rank's fine->coarse corrections (src/communication.c:2959 sends them to
// their owners).  Ranks of a single-rank tree are all cpu->rank: nothing is
// zeroed.  Without `param` every level above 1 counts as finer than lcoarse.
void clean_new_hydro(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct CPUINFO *cpu) {
  if (firstoct == nullptr || level < 1) return;
  if (level >= kMaxLevels) return;
  const std::vector<struct OCT *> &v = walk_level(firstoct, level);
  // written only where the bytes differ: after HydroSolver's final update most
  // cells already hold fieldnew == field, and a cache line left clean is not
  // written back to memory (the pass then costs one read of the cells)
  parallel_for((long long)v.size(), [&](long long a0, long long b0) {
    for (long long i = a0; i < b0; i++)
      for (int c = 0; c < 8; c++) {
        struct CELL &cl = v[i]->cell[c];
        if (bits_xor(&cl.fieldnew.d, &cl.field.d, (int)(sizeof(struct Wtype) / sizeof(double))) != 0)
          cl.fieldnew = cl.field;
      }
  });
  const int rank = dropin_rank(cpu);
  const int lcoarse = param ? reinterpret_cast<const RunParamsHead *>(param)->lcoarse : 1;
  if (level > lcoarse && level >= 2) {
    const std::vector<struct OCT *> &vc = walk_level(firstoct, level - 1);
    parallel_for((long long)vc.size(), [&](long long a0, long long b0) {
      for (long long i = a0; i < b0; i++)
        if (vc[i]->cpu != rank)
          for (int c = 0; c < 8; c++) std::memset(&vc[i]->cell[c].fieldnew, 0, sizeof(struct Wtype));
    });
  }
}

// ------------------------------------------------ device-side refinement
int emma_hydro_mark_cells(int level, struct RUNPARAMS *param, struct OCT **firstoct, int nsmooth, REAL threshold,
                          struct CPUINFO *cpu) {
  (void)param;
  (void)cpu;
  int rc = refine_ok(firstoct, level, false);
  if (rc != 0) return rc;
  if (nsmooth < 1) return EMMA_ST_ARG;
  rc = device_mark_cells(level, nsmooth, threshold);
  if (rc != 0) return rc;
  CK(cudaStreamSynchronize(g.stream));
  return 0;
}

int emma_hydro_check_rule(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct CPUINFO *cpu) {
  (void)param;
  (void)cpu;
  int rc = refine_ok(firstoct, level, false);
  if (rc != 0) return rc;
  rc = device_check_rule(level);
  if (rc != 0) return rc;
  CK(cudaStreamSynchronize(g.stream));
  return 0;
}

int emma_hydro_marks_to_host(struct OCT **firstoct, int level) {
  const int rc = refine_ok(firstoct, level, false);
  return rc != 0 ? rc : marks_to_host(level);
}

struct OCT *emma_hydro_refine_cells(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct OCT **lastoct,
                                    struct OCT *freeoct, struct CPUINFO *cpu, struct OCT *limit, REAL aexp) {
  (void)aexp;
  (void)cpu;
  if (refine_ok(firstoct, level, true) != 0) return nullptr;
  if (lastoct == nullptr || freeoct == nullptr || limit == nullptr) {
    fail(EMMA_ST_ARG, "refine_cells: null lastoct, freeoct or limit");
    return nullptr;
  }
  const int lcoarse = param ? reinterpret_cast<const RunParamsHead *>(param)->lcoarse : g.res.lcoarse;
  if (marks_to_host(level) != 0) return nullptr;
  if (cudaStreamSynchronize(g.stream) != cudaSuccess) return nullptr;
  std::vector<struct OCT *> created;
  std::string err;
  struct OCT *f = refine_sweep(level, lcoarse, firstoct, lastoct, freeoct, limit, created, err);
  if (f == nullptr) {
    // the host tree may be partly refined: the resident mirror no longer matches it
    fail(EMMA_ST_TREE, "refine_cells: " + err);
    emma_hydro_tree_release(firstoct);
    return nullptr;
  }
  if (rebuild_after_refine(firstoct, level, created) != 0) {
    emma_hydro_tree_release(firstoct);
    return nullptr;
  }
  return f;
}

#ifdef EMMA_WGRAV
// grav_correction (src/hydro_utils.c:2388-2444, PRIMITIVE): after HydroSolver,
// the leaf cells of rank cpu->rank get the full-step kick u += -f dt, then E;
// `a` is left as it was, as in the reference.  A negative pressure (an abort in
// the reference) sets EMMA_ST_NAN.
void grav_correction(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct CPUINFO *cpu, REAL dt) {
  (void)param;
  if (firstoct == nullptr || level < 1 || level >= kMaxLevels) return;
  const int rank = dropin_rank(cpu);
  const std::vector<struct OCT *> &v = walk_level(firstoct, level);
  std::atomic<bool> neg{false};
  parallel_for((long long)v.size(), [&](long long a0, long long b0) {
    for (long long i = a0; i < b0; i++) {
      struct OCT *o = v[i];
      if (o->cpu != rank) continue;
      for (int c = 0; c < 8; c++) {
        struct CELL *cell = &o->cell[c];
        if (cell->child != nullptr) continue;
        struct Wtype W = cell->field;
        W.u += (-cell->f[0] * dt);
        W.v += (-cell->f[1] * dt);
        W.w += (-cell->f[2] * dt);
        W.E = W.p / (kG - 1.) + 0.5 * W.d * (W.u * W.u + W.v * W.v + W.w * W.w);
        if (W.p < 0) neg = true;
        cell->field = W;
      }
    }
  });
  if (neg) fail(EMMA_ST_NAN, "grav_correction: negative pressure");
}
#endif

void create_hydstencil_GPU(struct CPUINFO *cpu, int stride) {
  (void)cpu;
  (void)stride;
  emma_hydro_init(nullptr);
}

void destroy_hydstencil_GPU(struct CPUINFO *cpu, int stride) {
  (void)cpu;
  (void)stride;
  if (!g.ready) return;
  cudaStreamSynchronize(g.stream);
  drop_all();
}

void create_pinned_stencil(struct HGRID **stencil, int stride) {
  if (stencil == nullptr) return;
  void *p = nullptr;
  if (cudaMallocHost(&p, (size_t)EMMA_SIZEOF_HGRID * (size_t)std::max(stride, 1)) != cudaSuccess) {
    fail(EMMA_ST_CUDA, "create_pinned_stencil: cudaMallocHost failed");
    p = nullptr;
  }
  *stencil = static_cast<struct HGRID *>(p);
}

void destroy_pinned_stencil(struct HGRID **stencil, int stride) {
  (void)stride;
  if (stencil == nullptr || *stencil == nullptr) return;
  cudaFreeHost(*stencil);
  *stencil = nullptr;
}

}  // extern "C"
