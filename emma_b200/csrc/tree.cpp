// tree.cpp -- host oct-tree construction with EMMA's ordering.
//
// Callers that have no EMMA tree (the benchmark, the tests) build one here.
// The construction order is the reference's, because the oct order of each
// level (the `next` list) is part of the contract of the hydro path:
//   - levels 1..lcoarse are complete, created level by level, parent oct by
//     parent oct in list order, cell 0..7 inside each parent, octs taken from
//     the array sequentially (build_initial_grid, src/amr.c:1507-1661);
//   - periodic boundaries come from the root oct's neighbours being a stand-in
//     cell whose child is the root oct (src/amr.c:1529);
//   - refinement of marked cells appends the new octs to the end of the finer
//     level's list in the same parent/cell order and copies the parent state
//     into the eight children (L_refine_cells, src/amr.c:286-735);
//   - a refinement whose face neighbour at the parent level is not split is
//     refused (the reference aborts with "ERROR ouhla", src/amr.c:480-497).
// The result is checked against the reference's own builder in
// tests/test_tree.py (positions, levels, neighbour and child links).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>
#include "emma_hydro.h"
#ifdef EMMA_WGRAV
#include "emma_hydro_grav.h"
#endif
#ifdef EMMA_WRADHYD
#include "emma_hydro_rh.h"
#endif
#ifdef EMMA_HELIUM
#include "emma_hydro_he.h"
#endif

struct EmmaTree {
  // octs live in fixed-size blocks so that pointers stay valid as the tree grows
  std::vector<struct OCT *> blocks;
  long long ngridmax = 0, nused = 0;
  int lcoarse = 0, lmax = 0;
  std::vector<struct OCT *> first, last;
  struct CELL root;  // stand-in parent-level cell of the root oct
};

namespace {

// face neighbour k (0:-x 1:+x 2:-y 3:+y 4:-z 5:+z) of cell ic: inside the oct?
inline bool nei_inside(int ic, int k) {
  int bit = 1 << (k >> 1);
  return (k & 1) ? !(ic & bit) : (ic & bit);
}

constexpr long long kBlockOcts = 1 << 16;

struct OCT *new_oct(EmmaTree *t) {
  if (t->ngridmax > 0 && t->nused >= t->ngridmax) return nullptr;
  const long long b = t->nused / kBlockOcts, i = t->nused % kBlockOcts;
  if (b >= (long long)t->blocks.size()) {
    struct OCT *blk = static_cast<struct OCT *>(std::calloc((size_t)kBlockOcts, sizeof(struct OCT)));
    if (blk == nullptr) return nullptr;
    t->blocks.push_back(blk);
  }
  t->nused++;
  return &t->blocks[b][i];
}

void append(EmmaTree *t, int level, struct OCT *o) {
  o->next = nullptr;
  if (t->first[level - 1] == nullptr) {
    t->first[level - 1] = o;
    o->prev = nullptr;
  } else {
    o->prev = t->last[level - 1];
    t->last[level - 1]->next = o;
  }
  t->last[level - 1] = o;
}

// Create the child oct of cell `icell` of `cur` (shared by the initial build
// and by refinement).  Returns nullptr when out of octs or when a face
// neighbour at the parent level is missing.
struct OCT *make_child(EmmaTree *t, struct OCT *cur, int icell, bool copy_field) {
  for (int k = 0; k < 6; k++)
    if (!nei_inside(icell, k) && (cur->nei[k] == nullptr || cur->nei[k]->child == nullptr)) return nullptr;
  struct OCT *o = new_oct(t);
  if (o == nullptr) return nullptr;
  const double dxcur = 1. / std::pow(2., cur->level);
  o->parent = &cur->cell[icell];
  o->level = cur->level + 1;
  o->x = cur->x + (icell % 2) * dxcur;
  o->y = cur->y + ((icell / 2) % 2) * dxcur;
  o->z = cur->z + (icell / 4) * dxcur;
  o->cpu = cur->cpu < 0 ? 0 : cur->cpu;
  o->nexthash = nullptr;
  for (int ii = 0; ii < 8; ii++) {
    struct CELL *c = &o->cell[ii];
    c->child = nullptr;
    c->marked = 0.;
    c->idx = ii;
    if (copy_field) {
      c->field = cur->cell[icell].field;
      c->fieldnew = cur->cell[icell].field;
    } else {
      std::memset(&c->field, 0, sizeof(c->field));
      std::memset(&c->fieldnew, 0, sizeof(c->fieldnew));
    }
  }
  for (int k = 0; k < 6; k++) {
    int vc = icell ^ (1 << (k >> 1));
    o->nei[k] = nei_inside(icell, k) ? &cur->cell[vc] : &cur->nei[k]->child->cell[vc];
  }
  cur->cell[icell].child = o;
  append(t, o->level, o);
  return o;
}

}  // namespace

extern "C" {

// ngridmax <= 0: no limit on the number of octs.
struct EmmaTree *emma_tree_create(int lcoarse, int lmax, long long ngridmax) {
  if (lcoarse < 2 || lmax < lcoarse) return nullptr;
  long long need = 0;
  for (int l = 1; l <= lcoarse; l++) need += 1LL << (3 * (l - 1));
  if (ngridmax > 0 && need > ngridmax) return nullptr;
  EmmaTree *t = new EmmaTree();
  t->ngridmax = ngridmax;
  t->lcoarse = lcoarse;
  t->lmax = lmax;
  t->first.assign(lmax, nullptr);
  t->last.assign(lmax, nullptr);
  std::memset(&t->root, 0, sizeof(t->root));
  struct OCT *root = new_oct(t);
  t->root.child = root;
  root->level = 1;
  root->cpu = -1;
  root->parent = nullptr;
  for (int k = 0; k < 6; k++) root->nei[k] = &t->root;
  for (int ic = 0; ic < 8; ic++) root->cell[ic].idx = ic;
  append(t, 1, root);
  for (int level = 1; level < lcoarse; level++)
    for (struct OCT *cur = t->first[level - 1]; cur != nullptr; cur = cur->next)
      for (int ic = 0; ic < 8; ic++) make_child(t, cur, ic, false);
  return t;
}

void emma_tree_destroy(struct EmmaTree *t) {
  if (t == nullptr) return;
  for (struct OCT *b : t->blocks) std::free(b);
  delete t;
}

int emma_tree_refine(struct EmmaTree *t, int level, const signed char *mark) {
  if (t == nullptr || level < t->lcoarse || level >= t->lmax || mark == nullptr) return -1;
  long long i = 0;
  int refused = 0;
  for (struct OCT *cur = t->first[level - 1]; cur != nullptr; cur = cur->next, i++)
    for (int ic = 0; ic < 8; ic++)
      if (mark[8 * i + ic] && cur->cell[ic].child == nullptr)
        if (make_child(t, cur, ic, true) == nullptr) refused++;
  return refused ? -refused : emma_tree_noct(t, level + 1);
}

struct OCT **emma_tree_firstoct(struct EmmaTree *t) { return t ? t->first.data() : nullptr; }

int emma_tree_noct(struct EmmaTree *t, int level) {
  if (t == nullptr || level < 1 || level > t->lmax) return 0;
  int n = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next) n++;
  return n;
}

void emma_tree_oct_xyz(struct EmmaTree *t, int level, double *xyz) {
  long long i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++) {
    xyz[3 * i] = o->x;
    xyz[3 * i + 1] = o->y;
    xyz[3 * i + 2] = o->z;
  }
}

// Primitive fields of a level (list order, oct*8+cell); a and E follow the
// reference's formulas (U2W src/hydro_utils.c:64, getE :29).
void emma_tree_set_field(struct EmmaTree *t, int level, const double *d, const double *u, const double *v,
                         const double *w, const double *p) {
  const double g = 5. / 3.;
  long long i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++)
    for (int c = 0; c < 8; c++) {
      long long k = 8 * i + c;
      struct Wtype *W = &o->cell[c].field;
      W->d = d[k];
      W->u = u[k];
      W->v = v[k];
      W->w = w[k];
      W->p = p[k];
      W->a = std::sqrt(g * W->p / W->d);
      W->E = W->p / (g - 1.) + 0.5 * W->d * (W->u * W->u + W->v * W->v + W->w * W->w);
      o->cell[c].fieldnew = *W;
    }
}

void emma_tree_get_field(struct EmmaTree *t, int level, int which, double *out7) {
  long long n = 8LL * emma_tree_noct(t, level), i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++)
    for (int c = 0; c < 8; c++) {
      const struct Wtype *W = which ? &o->cell[c].fieldnew : &o->cell[c].field;
      long long k = 8 * i + c;
      out7[k] = W->d;
      out7[n + k] = W->u;
      out7[2 * n + k] = W->v;
      out7[3 * n + k] = W->w;
      out7[4 * n + k] = W->p;
      out7[5 * n + k] = W->a;
      out7[6 * n + k] = W->E;
    }
}

void emma_tree_put_field(struct EmmaTree *t, int level, int which, const double *in7) {
  long long n = 8LL * emma_tree_noct(t, level), i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++)
    for (int c = 0; c < 8; c++) {
      struct Wtype *W = which ? &o->cell[c].fieldnew : &o->cell[c].field;
      long long k = 8 * i + c;
      W->d = in7[k];
      W->u = in7[n + k];
      W->v = in7[2 * n + k];
      W->w = in7[3 * n + k];
      W->p = in7[4 * n + k];
      W->a = in7[5 * n + k];
      W->E = in7[6 * n + k];
    }
}

void emma_tree_set_cpu(struct EmmaTree *t, int level, const int *cpu) {
  long long i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++) o->cpu = cpu[i];
}

#ifdef EMMA_WRADHYD
void emma_tree_set_tracer(struct EmmaTree *t, int level, const double *dX) {
  long long i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++)
    for (int c = 0; c < 8; c++) o->cell[c].field.dX = o->cell[c].fieldnew.dX = dX[8 * i + c];
}

void emma_tree_put_tracer(struct EmmaTree *t, int level, int which, const double *dX) {
  long long i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++)
    for (int c = 0; c < 8; c++) (which ? o->cell[c].fieldnew : o->cell[c].field).dX = dX[8 * i + c];
}

void emma_tree_get_tracer(struct EmmaTree *t, int level, int which, double *out) {
  long long i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++)
    for (int c = 0; c < 8; c++) out[8 * i + c] = which ? o->cell[c].fieldnew.dX : o->cell[c].field.dX;
}
#endif

#ifdef EMMA_HELIUM
// tracer `tr` (0: dX, 1: dXHE, 2: dXXHE, consecutive in struct Wtype)
void emma_tree_set_tracer_n(struct EmmaTree *t, int level, int tr, const double *x) {
  if (tr < 0 || tr > 2) return;
  long long i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++)
    for (int c = 0; c < 8; c++) (&o->cell[c].field.dX)[tr] = (&o->cell[c].fieldnew.dX)[tr] = x[8 * i + c];
}

void emma_tree_put_tracer_n(struct EmmaTree *t, int level, int tr, int which, const double *x) {
  if (tr < 0 || tr > 2) return;
  long long i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++)
    for (int c = 0; c < 8; c++) (&(which ? o->cell[c].fieldnew : o->cell[c].field).dX)[tr] = x[8 * i + c];
}

void emma_tree_get_tracer_n(struct EmmaTree *t, int level, int tr, int which, double *out) {
  if (tr < 0 || tr > 2) return;
  long long i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++)
    for (int c = 0; c < 8; c++) out[8 * i + c] = (&(which ? o->cell[c].fieldnew : o->cell[c].field).dX)[tr];
}
#endif

#ifdef EMMA_WGRAV
void emma_tree_set_force(struct EmmaTree *t, int level, const double *fx, const double *fy, const double *fz) {
  long long i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++)
    for (int c = 0; c < 8; c++) {
      o->cell[c].f[0] = fx[8 * i + c];
      o->cell[c].f[1] = fy[8 * i + c];
      o->cell[c].f[2] = fz[8 * i + c];
    }
}
#endif

// Same encoding as the oracle driver's export: cell code = (oct index in its
// level list)*8 + cell index; -2 for the root stand-in cell; -1 for NULL.
void emma_tree_topology(struct EmmaTree *t, int level, int *nei, int *parent, int *child, int *lev) {
  std::unordered_map<const struct OCT *, int> idx;
  idx.reserve((size_t)t->nused);
  for (int l = 1; l <= t->lmax; l++) {
    int i = 0;
    for (struct OCT *o = t->first[l - 1]; o != nullptr; o = o->next) idx[o] = i++;
  }
  auto code = [&](struct CELL *c) -> int {
    if (c == nullptr) return -1;
    if (c == &t->root) return -2;
    struct OCT *o = reinterpret_cast<struct OCT *>(reinterpret_cast<char *>(c) - (size_t)c->idx * sizeof(struct CELL));
    return idx[o] * 8 + c->idx;
  };
  int i = 0;
  for (struct OCT *o = t->first[level - 1]; o != nullptr; o = o->next, i++) {
    for (int k = 0; k < 6; k++) nei[6 * i + k] = code(o->nei[k]);
    parent[i] = code(o->parent);
    for (int c = 0; c < 8; c++) child[8 * i + c] = o->cell[c].child ? idx[o->cell[c].child] : -1;
    lev[i] = o->level;
  }
}

}  // extern "C"
