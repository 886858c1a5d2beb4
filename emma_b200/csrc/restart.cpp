// restart.cpp -- checkpoints in the reference's raw-OCT restart format.
//
// save_amr (src/restart.c:12-103, -DWHYDRO2 build): header (tsim, tinit,
// nsteps, ndumps, lcoarse, lmax), the level time steps adt[0..lmax-1], the 7
// unit scales, the addresses of the root oct, of its cell 0 and of the particle
// root, then every oct of levels 1..lmax in `next`-list order as its address
// followed by its bytes.  restore_amr (src/restart.c:108-328) puts each oct back
// at the same offset from the first oct of the caller's pool, shifts every
// pointer by the pool offset, rebuilds firstoct/lastoct and chains the unused
// octs (level 0) of the pool into the free list.  With a resident tree uploaded
// from the same firstoct, a save first downloads the device state into it, and a
// restore releases it (the pool it mirrored is overwritten).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include "emma_hydro.h"

namespace {

struct File {
  FILE *f = nullptr;
  explicit File(FILE *p) : f(p) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

template <class T>
bool put(FILE *f, const T &v) {
  return std::fwrite(&v, sizeof(T), 1, f) == 1;
}
template <class T>
bool get(FILE *f, T &v) {
  return std::fread(&v, sizeof(T), 1, f) == 1;
}

// p - from + to, in bytes (the reference's relocation of a snapshot address)
template <class T>
T *moved(T *p, const void *from, const void *to) {
  if (p == nullptr) return nullptr;
  return reinterpret_cast<T *>(reinterpret_cast<uintptr_t>(p) - reinterpret_cast<uintptr_t>(from) +
                               reinterpret_cast<uintptr_t>(to));
}

}  // namespace

extern "C" {

int emma_hydro_save_amr(const char *filename, struct OCT **firstoct, double tsim, double tinit, int nsteps,
                        int ndumps, int lcoarse, int lmax, const double *adt, const double *units7,
                        const void *proot) {
  if (filename == nullptr || firstoct == nullptr || adt == nullptr || units7 == nullptr || lmax < 1)
    return EMMA_ST_ARG;
  // a device-resident run: its current state goes into the tree first
  if (emma_hydro_is_resident(firstoct)) {
    const int rc = emma_hydro_tree_download(firstoct);
    if (rc != 0) return rc;
  }
  File fp(std::fopen(filename, "wb"));
  if (fp.f == nullptr) return EMMA_ST_ARG;
  bool ok = put(fp.f, tsim) && put(fp.f, tinit) && put(fp.f, nsteps) && put(fp.f, ndumps) && put(fp.f, lcoarse) &&
            put(fp.f, lmax);
  for (int l = 1; l <= lmax && ok; l++) ok = put(fp.f, adt[l - 1]);
  for (int i = 0; i < 7 && ok; i++) ok = put(fp.f, units7[i]);  // unit_l, _v, _t, _n, _mass, _d, _N
  struct OCT *root = firstoct[0];
  struct CELL *rootcell = root ? &root->cell[0] : nullptr;
  ok = ok && put(fp.f, root) && put(fp.f, rootcell) && put(fp.f, proot);
  for (int l = 1; l <= lmax && ok; l++)
    for (struct OCT *o = firstoct[l - 1]; o != nullptr && ok; o = o->next) ok = put(fp.f, o) && put(fp.f, *o);
  return ok ? 0 : EMMA_ST_ARG;
}

int emma_hydro_restore_amr(const char *filename, struct OCT **firstoct, struct OCT **lastoct, int levelmax,
                           long long ngridmax, struct CELL *root, double *tsim, double *tinit, int *nsteps,
                           int *ndumps, int *lcoarse, int *lmax, double *adt, double *units7,
                           struct OCT **freeoct) {
  if (filename == nullptr || firstoct == nullptr || lastoct == nullptr || firstoct[0] == nullptr || tsim == nullptr ||
      tinit == nullptr || nsteps == nullptr || ndumps == nullptr || lcoarse == nullptr || lmax == nullptr ||
      adt == nullptr || units7 == nullptr || levelmax < 1 || ngridmax < 1)
    return EMMA_ST_ARG;
  // the pool is overwritten: a resident tree uploaded from it no longer describes
  // it (its cached oct pointers would write stale device state into the restored
  // octs at the next download), so it is released; upload the restored tree again
  const int rel = emma_hydro_tree_release(firstoct);
  if (rel != 0) return rel;
  struct OCT *root_mem = firstoct[0];  // the pool's first oct
  struct CELL *rootcell_mem = &root_mem->cell[0];
  for (int l = 1; l <= levelmax; l++) firstoct[l - 1] = lastoct[l - 1] = nullptr;
  File fp(std::fopen(filename, "rb"));
  if (fp.f == nullptr) return EMMA_ST_ARG;
  bool ok = get(fp.f, *tsim) && get(fp.f, *tinit) && get(fp.f, *nsteps) && get(fp.f, *ndumps) &&
            get(fp.f, *lcoarse) && get(fp.f, *lmax) && *lmax >= 1 && *lmax <= levelmax;
  for (int l = 1; ok && l <= *lmax; l++) ok = get(fp.f, adt[l - 1]);
  for (int i = 0; ok && i < 7; i++) ok = get(fp.f, units7[i]);
  struct OCT *root_sna = nullptr;
  struct CELL *rootcell_sna = nullptr;
  void *rootpart_sna = nullptr;
  ok = ok && get(fp.f, root_sna) && get(fp.f, rootcell_sna) && get(fp.f, rootpart_sna);
  if (!ok) return EMMA_ST_ARG;
  struct OCT *oct_ad = nullptr;
  std::vector<unsigned char> buf(sizeof(struct OCT));
  while (get(fp.f, oct_ad) && std::fread(buf.data(), sizeof(struct OCT), 1, fp.f) == 1) {
    const long long off = (long long)(reinterpret_cast<intptr_t>(oct_ad) - reinterpret_cast<intptr_t>(root_sna)) /
                          (long long)sizeof(struct OCT);
    if (off < 0 || off >= ngridmax) return EMMA_ST_TREE;  // outside the caller's pool
    struct OCT *o = root_mem + off;
    std::memcpy(o, buf.data(), sizeof(struct OCT));
    o->next = moved(o->next, root_sna, root_mem);
    o->prev = moved(o->prev, root_sna, root_mem);
    o->nexthash = moved(o->nexthash, root_sna, root_mem);
    for (int c = 0; c < 8; c++) o->cell[c].child = moved(o->cell[c].child, root_sna, root_mem);
    for (int k = 0; k < 6; k++) o->nei[k] = moved(o->nei[k], rootcell_sna, rootcell_mem);
    if (o->parent != nullptr) o->parent = (o->level > 1) ? moved(o->parent, rootcell_sna, rootcell_mem) : root;
    if (o->level < 1 || o->level > levelmax) return EMMA_ST_TREE;
    if (firstoct[o->level - 1] == nullptr && o->prev == nullptr) firstoct[o->level - 1] = o;
    if (lastoct[o->level - 1] == nullptr && o->next == nullptr) lastoct[o->level - 1] = o;
  }
  // the unused octs of the pool (level 0), chained in address order
  struct OCT *free_head = nullptr, *last = nullptr;
  for (struct OCT *o = root_mem; o < root_mem + ngridmax; o++) {
    if (o->level != 0) continue;
    o->next = nullptr;
    o->prev = last;
    if (last) last->next = o;
    else free_head = o;
    last = o;
  }
  if (freeoct) *freeoct = free_head;
  return 0;
}

}  // extern "C"
