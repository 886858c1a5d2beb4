// api.cu -- C ABI of libemmahydro: device context, resident tree, level
// schedule and the drop-in entries with the reference's names.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include "emma_hydro.h"
#include "mirror.h"
#include "plan_types.h"

namespace emma {
cudaError_t launch_level_fp64(const LevelArgs &a, cudaStream_t s);
cudaError_t launch_level_f32(const LevelArgs &a, cudaStream_t s);
cudaError_t launch_cfl(const double *W, long long n8, unsigned long long *out, int nsm, cudaStream_t s);
}  // namespace emma

using namespace emma;

namespace {

constexpr double kG = 5. / 3.;

struct DevLevel {
  int L = 0, noct = 0, ntiles = 0;
  long long n8 = 0, leaf = 0;
  double *W = nullptr, *Wn = nullptr, *C = nullptr, *B = nullptr;
  uint8_t *split = nullptr;
  int *child = nullptr;
  TileDesc *tiles = nullptr;
  uint32_t *keys = nullptr;
  uint8_t *graph = nullptr;
  uint16_t *halo = nullptr;
  uint16_t *bface = nullptr;
};

struct TimedLaunch {
  cudaEvent_t a, b;
  long long cells;
};

struct Ctx {
  bool ready = false;
  EmmaHydroOptions opt;
  cudaStream_t stream = nullptr;
  int nsm = 148;
  unsigned *d_status = nullptr;
  unsigned long long *d_smax = nullptr;
  unsigned long long *h_smax = nullptr;
  unsigned status = 0;
  std::string last_error;
  // resident tree
  bool have_tree = false;
  int lcoarse = 0, lmax = 0;
  HostTree host;
  std::vector<DevLevel> lev;
  // drop-in cache
  struct OCT **drop_first = nullptr;
  int drop_level = -1, drop_lo = 0, drop_hi = 0;
  std::vector<long long> drop_sig;
  HostTree drop_host;
  std::vector<DevLevel> drop_lev;
  // pinned staging
  double *pin = nullptr;
  size_t pin_bytes = 0;
  bool own_stream = true;
  // counters and timing
  long long updates = 0;
  long long kernel_launches = 0;
  bool timing = true;
  std::vector<TimedLaunch> launches;
  std::vector<cudaEvent_t> free_events;
};

Ctx g;

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

template <class F>
void parallel_for(long long n, F f) {
  unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (n < 4096 || nt == 1) {
    f(0LL, n);
    return;
  }
  std::vector<std::thread> th;
  long long chunk = (n + nt - 1) / nt;
  for (unsigned t = 0; t < nt; t++) {
    long long a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    th.emplace_back([=] { f(a, b); });
  }
  for (auto &t : th) t.join();
}

void free_level(DevLevel &d) {
  cudaFree(d.W);
  cudaFree(d.Wn);
  cudaFree(d.C);
  cudaFree(d.B);
  cudaFree(d.split);
  cudaFree(d.child);
  cudaFree(d.tiles);
  cudaFree(d.keys);
  cudaFree(d.graph);
  cudaFree(d.halo);
  cudaFree(d.bface);
  d = DevLevel();
}

template <class T>
bool upload_vec(T **dst, const std::vector<T> &v) {
  *dst = nullptr;
  if (v.empty()) return true;
  if (!ck(cudaMalloc(dst, v.size() * sizeof(T)), "cudaMalloc")) return false;
  return ck(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy plan");
}

// Allocate device arrays of the mirrored levels and copy topology + plans.
bool alloc_levels(const HostTree &H, std::vector<DevLevel> &dl, bool with_base) {
  dl.assign(H.lev.size(), DevLevel());
  for (int L = H.lcoarse; L <= H.lmax; L++) {
    const HostLevel &h = H.lev[L];
    DevLevel &d = dl[L];
    d.L = L;
    d.noct = h.noct;
    d.n8 = 8LL * h.noct;
    d.leaf = h.leaf;
    d.ntiles = (int)h.tiles.size();
    const size_t bytes = sizeof(double) * 5 * (size_t)std::max<long long>(d.n8, 1);
    if (!ck(cudaMalloc(&d.W, bytes), "cudaMalloc W")) return false;
    if (!ck(cudaMalloc(&d.Wn, bytes), "cudaMalloc Wn")) return false;
    if (!ck(cudaMalloc(&d.C, bytes), "cudaMalloc C")) return false;
    if (!ck(cudaMemset(d.C, 0, bytes), "cudaMemset C")) return false;
    if (with_base && !h.tiles.empty())
      if (!ck(cudaMalloc(&d.B, sizeof(double) * 6 * (size_t)std::max<long long>(d.n8, 1)), "cudaMalloc B"))
        return false;
    if (!upload_vec(&d.split, h.split)) return false;
    if (!upload_vec(&d.child, h.child)) return false;
    if (!upload_vec(&d.tiles, h.tiles)) return false;
    if (!upload_vec(&d.keys, h.keys)) return false;
    if (!upload_vec(&d.graph, h.graph)) return false;
    if (!upload_vec(&d.halo, h.halo)) return false;
    if (!upload_vec(&d.bface, h.bface)) return false;
  }
  return true;
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

inline void finish_prims(struct Wtype &W) {
  W.a = std::sqrt(kG * W.p / W.d);
  W.E = W.p / (kG - 1.) + 0.5 * W.d * (W.u * W.u + W.v * W.v + W.w * W.w);
}

bool launch_level(const DevLevel *Lc, DevLevel &Ld, const DevLevel *Lf, double dt, bool dropin) {
  LevelArgs a;
  std::memset(&a, 0, sizeof(a));
  a.L = Ld.L;
  a.noct = Ld.noct;
  a.W = Ld.W;
  a.Wn = Ld.Wn;
  a.C = dropin ? nullptr : Ld.C;
  a.B = dropin ? Ld.B : nullptr;
  if (Lc != nullptr && Lc->noct > 0) {
    a.Wc = Lc->W;
    a.Cc = Lc->C;
    a.nc8 = Lc->n8;
  }
  if (Lf != nullptr && Lf->noct > 0 && !dropin) {
    a.Wf = Lf->W;
    a.nf8 = Lf->n8;
  }
  a.split = Ld.split;
  a.child = Ld.child;
  a.tiles = Ld.tiles;
  a.keys = Ld.keys;
  a.graph = Ld.graph;
  a.halo = Ld.halo;
  a.bface = Ld.bface;
  a.dt = dt;
  a.dx = std::pow(0.5, Ld.L);
  a.status = g.d_status;
  a.ntiles = Ld.ntiles;
  TimedLaunch tl{};
  if (g.timing) {
    tl.a = get_event();
    tl.b = get_event();
    cudaEventRecord(tl.a, g.stream);
  }
  cudaError_t e = (g.opt.precision == EMMA_PREC_MIXED) ? launch_level_f32(a, g.stream) : launch_level_fp64(a, g.stream);
  if (Ld.ntiles > 0) g.kernel_launches++;
  if (g.timing) {
    cudaEventRecord(tl.b, g.stream);
    tl.cells = Ld.leaf;
    g.launches.push_back(tl);
  }
  return ck(e, "level kernel launch");
}

int level_ok(int level) {
  if (!g.have_tree || level < g.lcoarse || level > g.lmax) {
    fail(EMMA_ST_ARG, "level " + std::to_string(level) + " is not mirrored");
    return 0;
  }
  return 1;
}

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
    if (level == g.lcoarse) adt[level - 2] = adt[level - 1];
    if (adt[level - 2] < adt[level - 1]) adt[level - 1] = adt[level - 2];
    else adt[level - 1] = std::fmin(adt[level - 1], adt[level - 2] - dt);
    if (level < g.lmax && g.lev[level + 1].noct > 0) {
      dtfine = advance_level(S, level + 1, tloc);
      adt[level - 1] = dtfine;
      if (level == g.lcoarse) adt[level - 2] = adt[level - 1];
    }
    S.err |= emma_hydro_advance_level(level, adt[level - 1]);
    dt += adt[level - 1];
    tloc += adt[level - 1];
    is++;
  } while ((dt < adt[level - 2]) && (is < S.nsub) && S.err == 0);
  return dt;
}

}  // namespace

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
}

int emma_hydro_init(const struct EmmaHydroOptions *opt) {
  if (g.ready) {
    if (opt) g.opt = *opt;
    return 0;
  }
  emma_hydro_default_options(&g.opt);
  if (opt) g.opt = *opt;
  CK(cudaSetDevice(g.opt.device));
  CK(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
  CK(cudaDeviceGetAttribute(&g.nsm, cudaDevAttrMultiProcessorCount, g.opt.device));
  CK(cudaMalloc(&g.d_status, sizeof(unsigned)));
  CK(cudaMemset(g.d_status, 0, sizeof(unsigned)));
  CK(cudaMalloc(&g.d_smax, sizeof(unsigned long long)));
  CK(cudaMallocHost(&g.h_smax, sizeof(unsigned long long)));
  g.ready = true;
  return 0;
}

int emma_hydro_set_options(const struct EmmaHydroOptions *opt) {
  if (opt == nullptr) return EMMA_ST_ARG;
  if (!g.ready) return emma_hydro_init(opt);
  const int old_trans = g.opt.trans_flags;
  g.opt = *opt;
  if (g.have_tree && old_trans != opt->trans_flags) {
    fail(EMMA_ST_ARG, "transmissive flags changed: upload the tree again");
    return EMMA_ST_ARG;
  }
  return 0;
}

void emma_hydro_shutdown(void) {
  if (!g.ready) return;
  cudaStreamSynchronize(g.stream);
  for (auto &d : g.lev) free_level(d);
  for (auto &d : g.drop_lev) free_level(d);
  g.lev.clear();
  g.drop_lev.clear();
  for (auto &t : g.launches) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  for (auto e : g.free_events) cudaEventDestroy(e);
  g.launches.clear();
  g.free_events.clear();
  cudaFree(g.d_status);
  cudaFree(g.d_smax);
  cudaFreeHost(g.h_smax);
  if (g.pin) cudaFreeHost(g.pin);
  if (g.own_stream) cudaStreamDestroy(g.stream);
  g = Ctx();
}

// ------------------------------------------------------------ resident path
int emma_hydro_tree_upload(struct OCT **firstoct, int lcoarse, int lmax, int rank) {
  if (!g.ready && emma_hydro_init(nullptr) != 0) return EMMA_ST_CUDA;
  if (firstoct == nullptr || lcoarse < 2 || lmax < lcoarse) {
    fail(EMMA_ST_ARG, "bad tree arguments");
    return EMMA_ST_ARG;
  }
  CK(cudaStreamSynchronize(g.stream));
  for (auto &d : g.lev) free_level(d);
  g.have_tree = false;
  std::string err;
  int rc = build_host_tree(firstoct, lcoarse, lmax, rank, g.opt.trans_flags, lcoarse, lmax, g.host, err);
  if (rc != 0) {
    fail((unsigned)rc, err);
    return rc;
  }
  if (!alloc_levels(g.host, g.lev, false)) return EMMA_ST_CUDA;
  g.lcoarse = lcoarse;
  g.lmax = lmax;
  g.have_tree = true;
  return emma_hydro_fields_upload(firstoct);
}

int emma_hydro_fields_upload(struct OCT **firstoct) {
  (void)firstoct;
  if (!g.have_tree) {
    fail(EMMA_ST_ARG, "no tree uploaded");
    return EMMA_ST_ARG;
  }
  for (int L = g.lcoarse; L <= g.lmax; L++) {
    const HostLevel &h = g.host.lev[L];
    if (h.noct == 0) continue;
    const size_t bytes = sizeof(double) * 5 * 8 * (size_t)h.noct;
    if (!ensure_pin(bytes)) return EMMA_ST_CUDA;
    pack_level(h, 0, g.pin);
    CK(cudaMemcpyAsync(g.lev[L].W, g.pin, bytes, cudaMemcpyHostToDevice, g.stream));
    CK(cudaStreamSynchronize(g.stream));
  }
  return 0;
}

int emma_hydro_tree_download(struct OCT **firstoct) {
  (void)firstoct;
  if (!g.have_tree) {
    fail(EMMA_ST_ARG, "no tree uploaded");
    return EMMA_ST_ARG;
  }
  for (int L = g.lcoarse; L <= g.lmax; L++) {
    const HostLevel &h = g.host.lev[L];
    if (h.noct == 0) continue;
    const long long n8 = 8LL * h.noct;
    const size_t bytes = sizeof(double) * 5 * (size_t)n8;
    if (!ensure_pin(bytes)) return EMMA_ST_CUDA;
    CK(cudaMemcpyAsync(g.pin, g.lev[L].W, bytes, cudaMemcpyDeviceToHost, g.stream));
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
  if (!g.have_tree || level < g.lcoarse || level > g.lmax) return 0;
  return g.lev[level].noct;
}

long long emma_hydro_level_leaf_cells(int level) {
  if (!g.have_tree || level < g.lcoarse || level > g.lmax) return 0;
  return g.lev[level].leaf;
}

int emma_hydro_get_level_state(int level, double *host_out) {
  if (!level_ok(level) || host_out == nullptr) return EMMA_ST_ARG;
  const DevLevel &d = g.lev[level];
  CK(cudaMemcpyAsync(host_out, d.W, sizeof(double) * 5 * d.n8, cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  return 0;
}

int emma_hydro_set_level_state(int level, const double *host_in) {
  if (!level_ok(level) || host_in == nullptr) return EMMA_ST_ARG;
  const DevLevel &d = g.lev[level];
  CK(cudaMemcpyAsync(d.W, host_in, sizeof(double) * 5 * d.n8, cudaMemcpyHostToDevice, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  return 0;
}

int emma_hydro_clean_new(int level) {
  if (!level_ok(level)) return EMMA_ST_ARG;
  const DevLevel &d = g.lev[level];
  if (d.n8 == 0) return 0;
  CK(cudaMemsetAsync(d.C, 0, sizeof(double) * 5 * d.n8, g.stream));
  return 0;
}

int emma_hydro_comptstep(int level, double *dt_out) {
  if (!level_ok(level) || dt_out == nullptr) return EMMA_ST_ARG;
  const DevLevel &d = g.lev[level];
  double dt = 1e9;
  if (d.n8 > 0) {
    CK(cudaMemsetAsync(g.d_smax, 0, sizeof(unsigned long long), g.stream));
    CK(launch_cfl(d.W, d.n8, g.d_smax, g.nsm, g.stream));
    g.kernel_launches++;
    CK(cudaMemcpyAsync(g.h_smax, g.d_smax, sizeof(unsigned long long), cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    double smax;
    std::memcpy(&smax, g.h_smax, sizeof(double));
    const double dxcur = std::pow(0.5, level);
    if (smax > 0.) dt = std::fmin(dxcur * g.opt.cfl / (smax * 3.), dt);
  }
  *dt_out = dt;
  return 0;
}

int emma_hydro_advance_level(int level, double dt) {
  if (!level_ok(level)) return EMMA_ST_ARG;
  DevLevel &d = g.lev[level];
  if (d.noct == 0) return 0;
  const DevLevel *Lc = (level > g.lcoarse) ? &g.lev[level - 1] : nullptr;
  const DevLevel *Lf = (level < g.lmax) ? &g.lev[level + 1] : nullptr;
  if (!launch_level(Lc, d, Lf, dt, false)) return EMMA_ST_CUDA;
  std::swap(d.W, d.Wn);
  g.updates += d.leaf;
  return 0;
}

int emma_hydro_advance_coarse_step(double dt_param, double time_max, int nsub, double *tsim, double *adt) {
  if (!g.have_tree || tsim == nullptr || adt == nullptr) {
    fail(EMMA_ST_ARG, "advance_coarse_step: no tree or null pointer");
    return EMMA_ST_ARG;
  }
  Sched S{dt_param, time_max, nsub, adt, 0};
  advance_level(S, g.lcoarse, *tsim);
  *tsim += adt[g.lcoarse - 1];
  return S.err;
}

long long emma_hydro_cell_updates(void) { return g.updates; }

long long emma_hydro_kernel_launches(void) { return g.kernel_launches; }

int emma_hydro_set_stream(void *stream) {
  if (!g.ready && emma_hydro_init(nullptr) != 0) return EMMA_ST_CUDA;
  CK(cudaStreamSynchronize(g.stream));
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

void emma_hydro_reset_counters(void) {
  g.updates = 0;
  g.kernel_launches = 0;
  if (g.ready) cudaStreamSynchronize(g.stream);
  for (auto &t : g.launches) {
    g.free_events.push_back(t.a);
    g.free_events.push_back(t.b);
  }
  g.launches.clear();
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

// Host-only planning diagnostics (no GPU needed): builds and validates the tile
// plans of levels lcoarse..lmax and reports, per level, {octs, tiles, max staged
// octs, max halo cells, leaf cells}.  Returns the status bits of the planning.
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
    for (const TileDesc &t : h.tiles) {
      ms = std::max<long long>(ms, t.S);
      mh = std::max<long long>(mh, t.H);
    }
    long long *o = stats5 + 5 * (L - lcoarse);
    o[0] = h.noct;
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

static std::vector<long long> tree_signature(struct OCT **firstoct, int lo, int hi) {
  std::vector<long long> sig;
  sig.push_back((long long)(uintptr_t)firstoct);
  for (int L = lo; L <= hi; L++) {
    long long n = 0, h = 1469598103934665603LL;
    for (struct OCT *o = firstoct[L - 1]; o != nullptr; o = o->next) {
      n++;
      h = (h ^ (long long)(uintptr_t)o) * 1099511628211LL;
      for (int c = 0; c < 8; c++) h = (h ^ (o->cell[c].child != nullptr)) * 1099511628211LL;
    }
    sig.push_back(n);
    sig.push_back(h);
  }
  return sig;
}

int advancehydroGPU(struct OCT **firstoct, int level, struct CPUINFO *cpu, struct HGRID *stencil, int stride,
                    REAL dxcur, REAL dtnew) {
  (void)stencil;
  (void)stride;
  (void)dxcur;
  if (!g.ready && emma_hydro_init(nullptr) != 0) return 0;
  if (firstoct == nullptr || level < 2 || firstoct[level - 1] == nullptr) return 0;
  const int rank = dropin_rank(cpu);
  // levels present around `level`: L-1 always exists; L+1 only if a cell is split
  bool has_fine = false;
  for (struct OCT *o = firstoct[level - 1]; o != nullptr && !has_fine; o = o->next)
    for (int c = 0; c < 8; c++)
      if (o->cell[c].child != nullptr) has_fine = true;
  const int lo = level - 1, hi = has_fine ? level + 1 : level;
  std::vector<long long> sig = tree_signature(firstoct, lo, hi);
  if (g.drop_first != firstoct || g.drop_level != level || sig != g.drop_sig) {
    cudaStreamSynchronize(g.stream);
    for (auto &d : g.drop_lev) free_level(d);
    g.drop_lev.clear();
    g.drop_level = -1;
    std::string err;
    int rc = build_host_tree(firstoct, lo, hi, rank, g.opt.trans_flags, level, level, g.drop_host, err);
    if (rc != 0) {
      fail((unsigned)rc, err);
      return 0;
    }
    if (!alloc_levels(g.drop_host, g.drop_lev, true)) return 0;
    g.drop_first = firstoct;
    g.drop_level = level;
    g.drop_lo = lo;
    g.drop_hi = hi;
    g.drop_sig = sig;
  }
  HostTree &H = g.drop_host;
  const HostLevel &h = H.lev[level];
  const HostLevel &hc = H.lev[level - 1];
  DevLevel &d = g.drop_lev[level];
  DevLevel &dc = g.drop_lev[level - 1];
  if (h.noct == 0) return 0;
  const long long n8 = d.n8, nc8 = dc.n8;
  const size_t need = sizeof(double) * std::max<long long>(11 * n8, 5 * nc8);
  if (!ensure_pin(need)) return 0;
  // upload: level field (5 planes) + fieldnew (6 planes), coarser field
  pack_level(h, 0, g.pin);
  pack_level(h, 1, g.pin + 5 * n8);
  if (!ck(cudaMemcpyAsync(d.W, g.pin, sizeof(double) * 5 * n8, cudaMemcpyHostToDevice, g.stream), "H2D W")) return 0;
  if (!ck(cudaMemcpyAsync(d.B, g.pin + 5 * n8, sizeof(double) * 6 * n8, cudaMemcpyHostToDevice, g.stream), "H2D B"))
    return 0;
  if (nc8 > 0 && !h.inj_cells.empty()) {
    if (!ck(cudaStreamSynchronize(g.stream), "sync")) return 0;
    pack_level(hc, 0, g.pin);
    if (!ck(cudaMemcpyAsync(dc.W, g.pin, sizeof(double) * 5 * nc8, cudaMemcpyHostToDevice, g.stream), "H2D Wc"))
      return 0;
    if (!ck(cudaMemsetAsync(dc.C, 0, sizeof(double) * 5 * nc8, g.stream), "memset Cc")) return 0;
  }
  if (!launch_level(nc8 > 0 ? &dc : nullptr, d, nullptr, dtnew, true)) return 0;
  // download the level's new state into fieldnew (leaf cells)
  if (!ck(cudaMemcpyAsync(g.pin, d.Wn, sizeof(double) * 5 * n8, cudaMemcpyDeviceToHost, g.stream), "D2H Wn")) return 0;
  if (!ck(cudaStreamSynchronize(g.stream), "sync")) return 0;
  {
    const double *p = g.pin;
    parallel_for(h.noct, [&](long long a, long long b) {
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
          finish_prims(W);
        }
      }
    });
  }
  // fine -> coarse corrections: fieldnew = U2W(W2U(fieldnew) + dU) per coarse cell
  if (nc8 > 0 && !h.inj_cells.empty()) {
    if (!ck(cudaMemcpyAsync(g.pin, dc.C, sizeof(double) * 5 * nc8, cudaMemcpyDeviceToHost, g.stream), "D2H Cc"))
      return 0;
    if (!ck(cudaStreamSynchronize(g.stream), "sync")) return 0;
    const double *p = g.pin;
    for (int32_t k : h.inj_cells) {
      struct Wtype &W = hc.octs[k >> 3]->cell[k & 7].fieldnew;
      double Ud = W.d, Udu = W.d * W.u, Udv = W.d * W.v, Udw = W.d * W.w, UE = W.E;
      Ud += p[k];
      Udu += p[nc8 + k];
      Udv += p[2 * nc8 + k];
      Udw += p[3 * nc8 + k];
      UE += p[4 * nc8 + k];
      const double dl = (Ud == 0. ? 10. : Ud);
      W.d = Ud;
      W.u = Udu / dl;
      W.v = Udv / dl;
      W.w = Udw / dl;
      W.p = (kG - 1.) * (UE - ((Udu) * (Udu) + (Udv) * (Udv) + (Udw) * (Udw)) / (dl)*0.5);
      W.E = UE;
      W.a = std::sqrt(kG * W.p / dl);
    }
  }
  g.updates += d.leaf;
  if (emma_hydro_status() & (EMMA_ST_TREE | EMMA_ST_CUDA)) return 0;
  return h.noct;
}

void HydroSolver(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct CPUINFO *cpu,
                 struct HGRID *stencil, int stride, REAL dtnew) {
  (void)param;
  const double dxcur = std::pow(0.5, level);
  const int nread = advancehydroGPU(firstoct, level, cpu, stencil, stride, dxcur, dtnew);
  if (nread <= 0) return;
  // field := fieldnew on leaves; split cells := primitive mean of the children
  // (src/hydro_utils.c:3408-3483)
  for (struct OCT *o = firstoct[level - 1]; o != nullptr; o = o->next)
    for (int c = 0; c < 8; c++) {
      struct CELL *cell = &o->cell[c];
      if (cell->child == nullptr) {
        cell->field = cell->fieldnew;
      } else {
        struct Wtype W;
        std::memset(&W, 0, sizeof(W));
        for (int i = 0; i < 8; i++) {
          const struct Wtype &Wc = cell->child->cell[i].field;
          W.d += Wc.d * 0.125;
          W.u += Wc.u * 0.125;
          W.v += Wc.v * 0.125;
          W.w += Wc.w * 0.125;
          W.p += Wc.p * 0.125;
        }
        W.E = W.p / (kG - 1.) + 0.5 * W.d * (W.u * W.u + W.v * W.v + W.w * W.w);
        cell->field = W;
      }
    }
}

void clean_new_hydro(int level, struct RUNPARAMS *param, struct OCT **firstoct, struct CPUINFO *cpu) {
  (void)param;
  (void)cpu;
  if (firstoct == nullptr || level < 1) return;
  for (struct OCT *o = firstoct[level - 1]; o != nullptr; o = o->next)
    for (int c = 0; c < 8; c++) o->cell[c].fieldnew = o->cell[c].field;
}

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
  for (auto &d : g.drop_lev) free_level(d);
  g.drop_lev.clear();
  g.drop_level = -1;
  g.drop_first = nullptr;
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
