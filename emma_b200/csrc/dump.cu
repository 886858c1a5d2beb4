// dump.cu -- field dumps in the reference's ALLOCT format (dumpalloct_serial,
// src/io.c:1233-1358).
//
// One file per selected field, <folder>grid_<name>/<name>.<ndumps %05d>.p<rank %05d>:
// a header of int n_cell and seven 4-byte words (tsim, xmin, xmax, ymin, ymax,
// zmin, zmax; the reference hands fwrite the address of its double tsim with
// sizeof(float), so the word is the first 4 bytes of that double), then one
// float per dumped cell: the cells without a child (every cell at lmax) of the
// octs of `rank`, levels lcoarse..lmax, octs in list order (cpu->octList,
// src/oct.c:250-270), cells 0..7.  Values are assign_grid_field's
// (src/io.c:32-104) for the ids this cell layout has.
//
// For a tree resident on the GPU the hydro fields (ids 13-17) come from the
// device state: a gather kernel compacts the dumped cells of each level into
// FP32 planes (the reference's float conversion) and only those floats cross
// PCIe; every other id is read from the host tree.
#include <cuda_runtime.h>
#include <sys/stat.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "emma_hydro.h"
#ifdef EMMA_WGRAV
#include "emma_hydro_grav.h"
#endif
#include "mirror.h"

namespace emma {
bool resident_level(struct OCT **firstoct, int level, const HostLevel **h, const double **W, const uint8_t **split,
                    cudaStream_t *stream, int *nsm);
void release_dump_staging();
}

using namespace emma;

namespace {

constexpr int kMaxDumpFields = 32;

struct Planes {
  int plane[5];  // state plane (0..4 = d,u,v,w,p) of each device field
  int n;
};

// One thread per cell of the level: a dumped cell (no split bit, or every cell
// when `all`) goes to slot off[oct] + (dumped cells before it in its oct) of
// each requested plane, converted to float; a slot outside the oct's range
// [off[oct], off[oct+1]) (split bits that disagree with the offsets) is skipped.
__global__ void alloct_gather_kernel(const double *__restrict__ W, long long n8, const uint8_t *__restrict__ split,
                                     const int *__restrict__ off, int all, Planes pl, float *__restrict__ out,
                                     long long nd, int *__restrict__ bad) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n8; i += (long long)gridDim.x * blockDim.x) {
    const long long o = i >> 3;
    const unsigned c = (unsigned)(i & 7);
    const unsigned sp = all ? 0u : (unsigned)split[o];
    // the host's per-oct counts come from the tree's child pointers, the cells picked
    // here from the device's split bits: a tree refined after its upload disagrees
    if (c == 0 && __popc(~sp & 0xffu) != off[o + 1] - off[o]) atomicAdd(bad, 1);
    if ((sp >> c) & 1u) continue;
    const long long j = off[o] + __popc(~sp & ((1u << c) - 1u));
    if (j >= off[o + 1]) continue;
    for (int f = 0; f < pl.n; f++) out[f * nd + j] = (float)W[(long long)pl.plane[f] * n8 + i];
  }
}

// assign_grid_field (src/io.c:32-104) for the ids of this cell layout
bool grid_field(int id, const struct OCT *o, const struct CELL *c, float *v) {
  const double dxc = std::pow(0.5, o->level);
  switch (id) {
    case 0: *v = (float)(o->x + (double)(c->idx & 1) * dxc); return true;
    case 1: *v = (float)(o->y + (double)((c->idx >> 1) & 1) * dxc); return true;
    case 2: *v = (float)(o->z + (double)(c->idx >> 2) * dxc); return true;
    case 3: *v = (float)o->level; return true;
    case 4: *v = (float)o->cpu; return true;
#ifdef EMMA_WGRAV
    case 5: *v = (float)c->gdata.d; return true;
    case 7: *v = (float)c->gdata.p; return true;
    case 8: *v = (float)c->res; return true;
    case 9: case 10: case 11: *v = (float)c->f[id - 9]; return true;
#endif
    case 12: *v = (float)c->marked; return true;
    case 13: *v = (float)c->field.d; return true;
    case 14: *v = (float)c->field.u; return true;
    case 15: *v = (float)c->field.v; return true;
    case 16: *v = (float)c->field.w; return true;
    case 17: *v = (float)c->field.p; return true;
    default: return false;
  }
}

bool supported(int id) {
  struct OCT o;
  std::memset(&o, 0, sizeof(o));
  float v;
  return grid_field(id, &o, &o.cell[0], &v);
}

void header(FILE *f, int n, double tsim, const float b[6]) {
  std::fwrite(&n, sizeof(int), 1, f);
  std::fwrite(&tsim, 4, 1, f);  // the first 4 bytes of the double, as the reference writes them
  std::fwrite(b, sizeof(float), 6, f);
}

// Staging of the device gathers, kept between dumps (allocating pinned memory
// costs more than a dump's copies): offsets and floats on the device, floats in
// pinned host memory.  Grown on demand; dropped when the current device changes
// and by emma_hydro_shutdown.
struct Staging {
  int *d_off = nullptr;
  float *d_out = nullptr;
  float *pin = nullptr;
  size_t off_bytes = 0, out_bytes = 0, pin_bytes = 0;
  int device = -1;
  void release() {
    if (d_off) cudaFree(d_off);
    if (d_out) cudaFree(d_out);
    if (pin) cudaFreeHost(pin);
    *this = Staging();
  }
};
Staging g_stage;

bool grow(void **p, size_t *have, size_t need, bool pinned) {
  if (need <= *have) return true;
  if (*p) pinned ? cudaFreeHost(*p) : cudaFree(*p);
  *p = nullptr;
  *have = 0;
  if ((pinned ? cudaMallocHost(p, need) : cudaMalloc(p, need)) != cudaSuccess) {
    *p = nullptr;
    return false;
  }
  *have = need;
  return true;
}

struct Files {
  std::vector<FILE *> f;
  ~Files() {
    for (FILE *x : f)
      if (x) std::fclose(x);
  }
};

}  // namespace

void emma::release_dump_staging() { g_stage.release(); }

extern "C" int emma_hydro_dump_alloct(const char *folder, struct OCT **firstoct, int lcoarse, int lmax, int rank,
                                      int ndumps, double tsim, int nfields, const int *ids,
                                      const char *const *names) {
  if (folder == nullptr || firstoct == nullptr || ids == nullptr || names == nullptr || nfields < 1 ||
      nfields > kMaxDumpFields || lcoarse < 1 || lmax < lcoarse)
    return EMMA_ST_ARG;
  for (int i = 0; i < nfields; i++)
    if (names[i] == nullptr || !supported(ids[i])) return EMMA_ST_ARG;
  Files files;
  float b[6] = {2.f, -1.f, 2.f, -1.f, 2.f, -1.f};  // xmin, xmax, ymin, ymax, zmin, zmax
  for (int i = 0; i < nfields; i++) {
    const std::string dir = std::string(folder) + "grid_" + names[i] + "/";
    mkdir(dir.c_str(), 0755);
    char tail[64];
    std::snprintf(tail, sizeof(tail), ".%05d.p%05d", ndumps, rank);
    FILE *f = std::fopen((dir + names[i] + tail).c_str(), "wb");
    if (f == nullptr) return EMMA_ST_ARG;
    files.f.push_back(f);
    header(f, 0, tsim, b);
  }
  // the hydro fields of a resident tree come from the device
  std::vector<int> dev_field(nfields, -1);
  Planes pl{};
  for (int i = 0; i < nfields; i++)
    if (ids[i] >= 13 && ids[i] <= 17) dev_field[i] = ids[i] - 13;
  int n_cell = 0;
  std::vector<float> vals;
  std::vector<struct OCT *> octs;
  std::vector<int> off;
  Staging &S = g_stage;
  int rc = 0;
  for (int level = lcoarse; level <= lmax && rc == 0; level++) {
    const double dx = std::pow(0.5, level - 1);
    const HostLevel *h = nullptr;
    const double *W = nullptr;
    const uint8_t *split = nullptr;
    cudaStream_t stream = nullptr;
    int nsm = 0;
    // (a resident tree holds the octs of one rank: another rank's dump has none of them)
    const bool resident = resident_level(firstoct, level, &h, &W, &split, &stream, &nsm) && h->nown == h->noct &&
                          (h->octs.empty() || h->octs[0]->cpu == rank);
    octs.clear();
    if (resident) {
      octs.assign(h->octs.begin(), h->octs.end());
    } else {
      for (struct OCT *o = firstoct[level - 1]; o != nullptr; o = o->next)
        if (o->cpu == rank) octs.push_back(o);
    }
    // dumped cells per oct, their offsets, and the bounds of the dumped octs
    off.assign(octs.size() + 1, 0);
    for (size_t k = 0; k < octs.size(); k++) {
      const struct OCT *o = octs[k];
      int nd = 0;
      for (int c = 0; c < 8; c++) nd += (o->cell[c].child == nullptr || o->level == lmax);
      off[k + 1] = off[k] + nd;
      if (nd == 0) continue;
      if (o->x < b[0]) b[0] = (float)o->x;
      if (o->y < b[2]) b[2] = (float)o->y;
      if (o->z < b[4]) b[4] = (float)o->z;
      if (o->x + dx > b[1]) b[1] = (float)(o->x + dx);
      if (o->y + dx > b[3]) b[3] = (float)(o->y + dx);
      if (o->z + dx > b[5]) b[5] = (float)(o->z + dx);
    }
    const long long nd = off[octs.size()];
    n_cell += (int)nd;
    if (nd == 0) continue;
    vals.assign((size_t)nfields * nd, 0.f);
    // device fields: gather on the GPU, one copy of the compacted floats
    pl.n = 0;
    std::vector<int> slot(nfields, -1);
    int slot_of_plane[5] = {-1, -1, -1, -1, -1};
    if (resident)
      for (int i = 0; i < nfields; i++)
        if (dev_field[i] >= 0) {
          int &sp = slot_of_plane[dev_field[i]];
          if (sp < 0) {
            sp = pl.n;
            pl.plane[pl.n++] = dev_field[i];
          }
          slot[i] = sp;
        }
    if (pl.n > 0) {
      int dev = -1;
      cudaGetDevice(&dev);
      if (dev != S.device) {
        S.release();
        S.device = dev;
      }
      // offsets, then one counter of octs whose device split bits disagree with the host tree
      const size_t ob = sizeof(int) * (octs.size() + 2), vb = sizeof(float) * (size_t)pl.n * nd;
      bool ok = grow(reinterpret_cast<void **>(&S.d_off), &S.off_bytes, ob, false) &&
                grow(reinterpret_cast<void **>(&S.d_out), &S.out_bytes, vb, false) &&
                grow(reinterpret_cast<void **>(&S.pin), &S.pin_bytes, vb, true);
      const long long n8 = 8LL * (long long)octs.size();
      const int grid = std::max(1, std::min((int)((n8 + 255) / 256), 8 * std::max(nsm, 1)));
      int *d_bad = S.d_off + octs.size() + 1;
      int nbad = 0;
      ok = ok &&
           cudaMemcpyAsync(S.d_off, off.data(), sizeof(int) * (octs.size() + 1), cudaMemcpyHostToDevice, stream) ==
               cudaSuccess &&
           cudaMemsetAsync(d_bad, 0, sizeof(int), stream) == cudaSuccess;
      if (ok) {
        alloct_gather_kernel<<<grid, 256, 0, stream>>>(W, n8, split, S.d_off, level == lmax ? 1 : 0, pl, S.d_out,
                                                       nd, d_bad);
        ok = cudaGetLastError() == cudaSuccess;
      }
      ok = ok && cudaMemcpyAsync(S.pin, S.d_out, vb, cudaMemcpyDeviceToHost, stream) == cudaSuccess &&
           cudaMemcpyAsync(&nbad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, stream) == cudaSuccess &&
           cudaStreamSynchronize(stream) == cudaSuccess;
      if (!ok) {
        rc = EMMA_ST_CUDA;
        break;
      }
      if (nbad != 0) {  // refined or coarsened since the upload: upload the tree again
        rc = EMMA_ST_TREE;
        break;
      }
      for (int i = 0; i < nfields; i++)
        if (slot[i] >= 0) std::memcpy(&vals[(size_t)i * nd], S.pin + (size_t)slot[i] * nd, sizeof(float) * nd);
    }
    // host fields
    for (int i = 0; i < nfields; i++) {
      if (slot[i] >= 0) continue;
      float *v = &vals[(size_t)i * nd];
      long long j = 0;
      for (const struct OCT *o : octs)
        for (int c = 0; c < 8; c++)
          if (o->cell[c].child == nullptr || o->level == lmax) grid_field(ids[i], o, &o->cell[c], &v[j++]);
    }
    for (int i = 0; i < nfields; i++)
      if (std::fwrite(&vals[(size_t)i * nd], sizeof(float), (size_t)nd, files.f[i]) != (size_t)nd) rc = EMMA_ST_ARG;
  }
  if (rc != 0) return rc;
  for (int i = 0; i < nfields; i++) {
    std::rewind(files.f[i]);
    header(files.f[i], n_cell, tsim, b);
    if (std::ferror(files.f[i])) rc = EMMA_ST_ARG;
    if (std::fclose(files.f[i]) != 0) rc = EMMA_ST_ARG;
    files.f[i] = nullptr;
  }
  return rc;
}
