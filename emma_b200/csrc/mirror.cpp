// mirror.cpp -- builds the per-level device mirror and tile plans from an EMMA
// oct tree (struct OCT, include/emma_oct.h).
//
// Neighbourhood semantics (what a tile stages).  For a level-L oct O the
// reference gathers a 3x3x3 block of octs (src/hydro_utils.c:2852-2967): slot
// (i,j,k) holds the children of the level-(L-1) cell at parent(O)+(i,j,k) if that
// cell is split, or the cell's state injected into all 8 cells otherwise.  The
// walk always lands on the geometric level-(L-1) cell, so the block is a window
// of one "virtual level-L grid" in which every position holds either a real
// level-L cell or an injected coarser leaf.  vnbr() below steps through that
// virtual grid one oct at a time.  A brick is a block of level-L oct positions
// (4x4x2 or 2x2x2, kShapes); it stages, at their grid positions in a slot box
// one oct wider on every side, the union of the windows of its octs (faces and
// edges: MUSCL never reads the corners).  A tile is one or more bricks.
//
// With transmissive boundaries (the reference's -DHYDROTEST -DTRANS*), the
// face slot across a boundary is the mirror of the boundary oct through the
// reference's face maps (src/hydro_utils.c:2504-2610).  The staged ghost's
// tangential neighbours are the mirrors of the boundary oct's tangential
// neighbours; this equals the reference for states that are uniform along the
// boundary (the Sod tube) and is the zero-gradient ghost layer elsewhere.
#include "mirror.h"
#include <cmath>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include "emma_hydro.h"

namespace emma {
namespace {

// open-addressing pointer -> int map (oct -> index in its level list)
struct PtrMap {
  std::vector<const void *> k;
  std::vector<int> v;
  size_t mask = 0;
  void init(size_t n) {
    size_t cap = 16;
    while (cap < 2 * n + 16) cap <<= 1;
    k.assign(cap, nullptr);
    v.assign(cap, -1);
    mask = cap - 1;
  }
  static size_t h(const void *p) {
    uint64_t x = (uint64_t)(uintptr_t)p;
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    return (size_t)x;
  }
  void put(const void *p, int val) {
    size_t i = h(p) & mask;
    while (k[i] != nullptr && k[i] != p) i = (i + 1) & mask;
    k[i] = p;
    v[i] = val;
  }
  int get(const void *p) const {
    if (mask == 0) return -1;
    size_t i = h(p) & mask;
    while (k[i] != nullptr) {
      if (k[i] == p) return v[i];
      i = (i + 1) & mask;
    }
    return -1;
  }
};

inline int pos_floor(int p, int b) { return p / b * b; }
inline bool inside(int c, int k) {
  const int bit = 1 << (k >> 1);
  return (k & 1) ? !(c & bit) : (c & bit);
}
inline struct OCT *oct_of(struct CELL *c) {
  return reinterpret_cast<struct OCT *>(reinterpret_cast<char *>(c) - (size_t)c->idx * sizeof(struct CELL));
}
bool at_boundary(const struct OCT *o, int k) {
  const double dx = std::pow(0.5, o->level);
  switch (k) {
    case 0: return o->x == 0.;
    case 1: return (o->x + 2. * dx) == 1.;
    case 2: return o->y == 0.;
    case 3: return (o->y + 2. * dx) == 1.;
    case 4: return o->z == 0.;
    default: return (o->z + 2. * dx) == 1.;
  }
}

struct Planner {
  HostTree &H;
  std::vector<PtrMap> idx;              // per level: oct -> index
  std::vector<std::vector<uint32_t>> face;  // per level: 6 keys per oct (vnbr of the real oct)
  unsigned err = 0;
  std::string msg;
  explicit Planner(HostTree &h) : H(h) {}

  uint32_t cell_key(int L, struct CELL *C) {
    // key of the virtual oct filled from level-(L-1) cell C
    if (C->child != nullptr) {
      const int i = idx[L].get(C->child);
      return i < 0 ? kKeyNone : key_make(kKeyReal, (uint32_t)i);
    }
    if (L - 1 < H.lcoarse) return kKeyNone;
    const int io = idx[L - 1].get(oct_of(C));
    return io < 0 ? kKeyNone : key_make(kKeyInj, (uint32_t)(8 * io + C->idx));
  }

  uint32_t real_nbr(int L, int o, int k) {
    struct OCT *oc = H.lev[L].octs[o];
    if ((H.trans >> k) & 1) {
      if (at_boundary(oc, k)) return key_make(kKeyGhost0 + k, (uint32_t)o);
    }
    struct CELL *C = oc->nei[k];
    if (C == nullptr) return kKeyNone;
    return cell_key(L, C);
  }

  uint32_t vnbr(int L, uint32_t key, int k) {
    if (key == kKeyNone) return kKeyNone;
    const uint32_t kind = key >> 28, i = key & 0x0FFFFFFFu;
    if (kind == kKeyReal) return face[L][6 * i + k];
    if (kind == kKeyInj) {
      struct OCT *oc = H.lev[L - 1].octs[i >> 3];
      const int c = (int)(i & 7);
      struct CELL *C2;
      if (inside(c, k)) {
        C2 = &oc->cell[c ^ (1 << (k >> 1))];
      } else {
        if (((H.trans >> k) & 1) && at_boundary(oc, k)) return kKeyNone;  // ghost of a coarse cell: not staged
        struct CELL *X = oc->nei[k];
        if (X == nullptr || X->child == nullptr) return kKeyNone;
        C2 = &X->child->cell[c ^ (1 << (k >> 1))];
      }
      return cell_key(L, C2);
    }
    // ghost across face k0 of oct i
    const int k0 = (int)kind - (int)kKeyGhost0;
    if (k == (k0 ^ 1)) return key_make(kKeyReal, i);
    if (k == k0) return kKeyNone;
    const uint32_t t = face[L][6 * i + k];
    if (t == kKeyNone || (t >> 28) != kKeyReal) return kKeyNone;
    return key_make(kKeyGhost0 + k0, t & 0x0FFFFFFFu);
  }
};

// mirror map of the transmissive ghost octs (src/hydro_utils.c:2504-2610):
// ghost cell c across face k takes cell kMirror[k][c] of the boundary oct
constexpr uint8_t kMirror[6][8] = {{0, 0, 2, 2, 4, 4, 6, 6}, {1, 1, 3, 3, 5, 5, 7, 7}, {0, 1, 0, 1, 4, 5, 4, 5},
                                   {2, 3, 2, 3, 7, 6, 6, 7}, {0, 1, 2, 3, 0, 1, 2, 3}, {4, 5, 6, 7, 4, 5, 6, 7}};
constexpr int kDir[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

// cell flags of the staged box, as the level kernel derives them
enum : uint8_t { kFPresent = 1, kFSplit = 2, kFTile = 4, kFInj = 8 };
inline bool f_ok(uint8_t f) { return (f & (kFPresent | kFSplit)) == kFPresent; }
inline bool f_tileleaf(uint8_t f) { return (f & (kFPresent | kFSplit | kFTile)) == (kFPresent | kFTile); }

// derived sizes of one brick of a shape
struct Box {
  int bx, by, bz, sx, sy, sz, xx, xy, xz, slots, cells;
  explicit Box(const BrickShape &s)
      : bx(s.bx), by(s.by), bz(s.bz), sx(s.bx + 2), sy(s.by + 2), sz(s.bz + 2), xx(2 * sx), xy(2 * sy),
        xz(2 * sz), slots(sx * sy * sz), cells(xx * xy * xz) {}
  int stride(int a) const { return a == 0 ? 1 : (a == 1 ? xx : xx * xy); }
};

// Slot keys of the brick at oct origin (ox,oy,oz) holding `octs` (level list
// indices, positions in `pos`).  Fills keys[slots] and the brick's mask.
bool plan_brick(Planner &P, int L, const Box &G, const std::vector<int> &octs, const std::vector<int32_t> &pos,
                int ox, int oy, int oz, uint32_t *keys, uint32_t &mask) {
  std::fill(keys, keys + G.slots, kKeyNone);
  mask = 0;
  auto put = [&](int sx, int sy, int sz, uint32_t key) -> bool {
    if (key == kKeyNone) return true;
    if (sx < 0 || sx >= G.sx || sy < 0 || sy >= G.sy || sz < 0 || sz >= G.sz) return false;
    uint32_t &k = keys[sx + G.sx * (sy + G.sy * sz)];
    if (k == kKeyNone) k = key;
    return k == key;
  };
  auto bad = [&](const std::string &m) {
    P.err |= EMMA_ST_TREE;
    P.msg = m + " (level " + std::to_string(L) + ", brick at oct " + std::to_string(ox) + "," + std::to_string(oy) +
            "," + std::to_string(oz) + ")";
    return false;
  };
  for (int o : octs) {
    const int ix = pos[3 * o] - ox, iy = pos[3 * o + 1] - oy, iz = pos[3 * o + 2] - oz;
    mask |= 1u << (ix + G.bx * (iy + G.by * iz));
    if (!put(ix + 1, iy + 1, iz + 1, key_make(kKeyReal, (uint32_t)o))) return bad("two octs at one brick position");
  }
  for (int o : octs) {
    const int sx = pos[3 * o] - ox + 1, sy = pos[3 * o + 1] - oy + 1, sz = pos[3 * o + 2] - oz + 1;
    const uint32_t self = key_make(kKeyReal, (uint32_t)o);
    for (int k = 0; k < 6; k++) {
      const uint32_t f = P.vnbr(L, self, k);
      if (f == kKeyNone) return bad("missing face neighbour of an oct");
      if (!put(sx + kDir[k][0], sy + kDir[k][1], sz + kDir[k][2], f)) return bad("inconsistent face neighbour");
      for (int j = 0; j < 6; j++) {
        if ((j >> 1) == (k >> 1)) continue;
        if (!put(sx + kDir[k][0] + kDir[j][0], sy + kDir[k][1] + kDir[j][1], sz + kDir[k][2] + kDir[j][2],
                 P.vnbr(L, f, j)))
          return bad("inconsistent edge neighbour");
      }
    }
  }
  return true;
}

// Cell flags of a planned brick and the checks that every stencil the kernel
// evaluates reads staged cells only.  Marks the level L-1 cells that receive
// fine->coarse corrections.
bool check_brick(Planner &P, int L, const Box &G, const uint32_t *keys, uint32_t mask,
                 std::vector<uint8_t> *corrected) {
  const HostLevel &lv = P.H.lev[L];
  std::vector<uint8_t> fl((size_t)G.cells, 0);
  for (int s = 0; s < G.slots; s++) {
    const int sz = s / (G.sx * G.sy), sy = (s / G.sx) % G.sy, sx = s % G.sx;
    const bool inner = sx >= 1 && sx <= G.bx && sy >= 1 && sy <= G.by && sz >= 1 && sz <= G.bz;
    for (int c = 0; c < 8; c++) {
      const int b = (2 * sx + (c & 1)) + G.xx * ((2 * sy + ((c >> 1) & 1)) + G.xy * (2 * sz + (c >> 2)));
      const uint32_t key = keys[s];
      uint8_t f = 0;
      if (key != kKeyNone) {
        const uint32_t kind = key >> 28, idx = key & 0x0FFFFFFFu;
        f = kFPresent;
        if (kind == kKeyReal) {
          if ((lv.split[idx] >> c) & 1) f |= kFSplit;
          if (inner && ((mask >> ((sx - 1) + G.bx * ((sy - 1) + G.by * (sz - 1)))) & 1)) f |= kFTile;
        } else if (kind == kKeyInj) {
          f |= kFInj;
        } else {
          if ((lv.split[idx] >> kMirror[kind - kKeyGhost0][c]) & 1) f |= kFSplit;
        }
      }
      fl[b] = f;
    }
  }
  // cells whose face states the kernel builds (dual energy: split cells too)
  auto recon = [&](uint8_t f) { return P.H.dual ? (f & kFPresent) != 0 : f_ok(f); };
  auto all_nbrs = [&](int b) {
    for (int a = 0; a < 3; a++)
      if (!(fl[b - G.stride(a)] & kFPresent) || !(fl[b + G.stride(a)] & kFPresent)) return false;
    return true;
  };
  auto fail = [&](const char *m) {
    P.err |= EMMA_ST_TREE;
    P.msg = std::string(m) + " (level " + std::to_string(L) + ")";
    return false;
  };
  const int x0 = 2, x1 = 2 + 2 * G.bx, y0 = 2, y1 = 2 + 2 * G.by, z0 = 2, z1 = 2 + 2 * G.bz;
  // brick cells: reconstructed if a leaf of the tile or face-adjacent to one
  for (int z = z0; z < z1; z++)
    for (int y = y0; y < y1; y++)
      for (int x = x0; x < x1; x++) {
        const int b = x + G.xx * (y + G.xy * z);
        bool near = f_tileleaf(fl[b]);
        for (int a = 0; a < 3; a++)
          near = near || f_tileleaf(fl[b - G.stride(a)]) || f_tileleaf(fl[b + G.stride(a)]);
        if (recon(fl[b]) && near && !all_nbrs(b)) return fail("unstaged neighbour of a reconstructed cell");
        if (!f_tileleaf(fl[b])) continue;
        for (int a = 0; a < 3; a++)
          for (int sgn = -1; sgn <= 1; sgn += 2) {
            const int b2 = b + sgn * G.stride(a);
            if (!(fl[b2] & kFPresent)) return fail("unstaged face neighbour of a leaf cell");
            if (corrected && (fl[b2] & kFInj)) {
              const int xb = b2 % G.xx, yb = (b2 / G.xx) % G.xy, zb = b2 / (G.xx * G.xy);
              (*corrected)[keys[(xb >> 1) + G.sx * ((yb >> 1) + G.sy * (zb >> 1))] & 0x0FFFFFFFu] = 1;
            }
          }
      }
  // ring cells face-adjacent to a leaf of the tile: reconstructed too
  for (int z = 1; z < G.xz - 1; z++)
    for (int y = 1; y < G.xy - 1; y++)
      for (int x = 1; x < G.xx - 1; x++) {
        const bool ix = x >= x0 && x < x1, iy = y >= y0 && y < y1, iz = z >= z0 && z < z1;
        if ((int)ix + (int)iy + (int)iz != 2) continue;  // face layer of the brick, not an edge
        const int b = x + G.xx * (y + G.xy * z);
        int bin = b;
        if (!ix) bin = b + (x < x0 ? 1 : -1);
        if (!iy) bin = b + (y < y0 ? G.xx : -G.xx);
        if (!iz) bin = b + (z < z0 ? G.xx * G.xy : -G.xx * G.xy);
        if (recon(fl[b]) && f_tileleaf(fl[bin]) && !all_nbrs(b)) return fail("unstaged neighbour of a ring cell");
      }
  return true;
}

// Bricks of a shape holding the first `noct` octs of the level (this rank's), in
// order of their first oct.
std::vector<std::vector<int>> group_bricks(const std::vector<int32_t> &pos, int noct, const BrickShape &sh) {
  std::unordered_map<uint64_t, int> brick;
  std::vector<std::vector<int>> members;
  brick.reserve((size_t)noct / 4 + 16);
  for (int i = 0; i < noct; i++) {
    const uint64_t bk = ((uint64_t)(pos[3 * i] / sh.bx) << 42) | ((uint64_t)(pos[3 * i + 1] / sh.by) << 21) |
                        (uint64_t)(pos[3 * i + 2] / sh.bz);
    auto it = brick.find(bk);
    if (it == brick.end()) {
      it = brick.emplace(bk, (int)members.size()).first;
      members.emplace_back();
    }
    members[it->second].push_back(i);
  }
  return members;
}

// Relative cost of one tile of each shape (a 2x2x2-oct brick stages and
// reconstructs more ring cells per cell); used when a level is planned without
// measurement.
constexpr double kTileCost[kNumShapes] = {1.0, 1.3};

int plan_level(Planner &P, HostTree &H, int L, int shape_req, std::string &err) {
  HostLevel &lv = H.lev[L];
  lv.tiles.clear();
  lv.keys.clear();
  lv.inj_cells.clear();
  lv.interp.clear();
  lv.reads_coarse = false;
  lv.shape = 0;
  if (lv.nown == 0) return 0;
  int shape = shape_req;
  std::vector<std::vector<int>> members;
  if (shape < 0 || shape >= kNumShapes) {
    // without a requested shape: the cheaper by tiles x tile cost
    double best = 0;
    for (int s = 0; s < kNumShapes; s++) {
      auto m = group_bricks(lv.pos, lv.nown, kShapes[s]);
      const double c = kTileCost[s] * (double)((m.size() + kShapes[s].nb - 1) / kShapes[s].nb);
      if (s == 0 || c < best) {
        best = c;
        shape = s;
        members = std::move(m);
      }
    }
  } else {
    members = group_bricks(lv.pos, lv.nown, kShapes[shape]);
  }
  const BrickShape &sh = kShapes[shape];
  const Box G(sh);
  lv.shape = shape;
  std::vector<uint8_t> corrected;
  if (L > H.lcoarse) corrected.assign((size_t)8 * H.lev[L - 1].noct, 0);
  const size_t ntiles = (members.size() + sh.nb - 1) / sh.nb;
  lv.tiles.resize(ntiles);
  lv.keys.assign(ntiles * (size_t)sh.tile_slots(), kKeyNone);
  for (size_t t = 0; t < ntiles; t++) {
    TileDesc &td = lv.tiles[t];
    std::memset(&td, 0, sizeof(td));
    for (int nb = 0; nb < sh.nb; nb++) {
      const size_t m = t * sh.nb + nb;
      if (m >= members.size()) break;
      const int o0 = members[m][0];
      const int ox = pos_floor(lv.pos[3 * o0], sh.bx), oy = pos_floor(lv.pos[3 * o0 + 1], sh.by),
                oz = pos_floor(lv.pos[3 * o0 + 2], sh.bz);
      if (nb == 0) {
        td.ox = ox;
        td.oy = oy;
        td.oz = oz;
      }
      uint32_t *keys = &lv.keys[t * sh.tile_slots() + (size_t)nb * sh.slots()];
      uint32_t bmask = 0;
      if (!plan_brick(P, L, G, members[m], lv.pos, ox, oy, oz, keys, bmask) ||
          !check_brick(P, L, G, keys, bmask, corrected.empty() ? nullptr : &corrected)) {
        err = P.msg;
        return (int)P.err;
      }
      td.mask |= bmask << (nb * sh.octs());
      td.noct += (int)members[m].size();
    }
  }
  for (size_t i = 0; i < corrected.size(); i++)
    if (corrected[i]) lv.inj_cells.push_back((int32_t)i);
  for (uint32_t key : lv.keys)
    if (key != kKeyNone && (key >> 28) == kKeyInj) lv.reads_coarse = true;
  if (lv.reads_coarse && (H.trans != 0 || H.grav != 0)) {
    // The reference's transmissive build (-DHYDROTEST) fills a coarser neighbour
    // by limited-slope interpolation (coarse2fine_hydro2, src/hydro_utils.c:311)
    // instead of injection: every injected slot becomes an interpolated one, with
    // the coarse cell and the 6 cells its slopes are taken from.  A gravity build
    // keeps the injected field but spreads the coarse cell's force over the 8
    // sub-cells from the same 6 neighbours (coarse2fine_forcelin,
    // src/poisson_utils.c:315), which dereferences every neighbour: none may miss.
    const HostLevel &lc = H.lev[L - 1];
    std::unordered_map<uint32_t, int> jof;
    for (uint32_t &key : lv.keys) {
      if (key == kKeyNone || (key >> 28) != kKeyInj) continue;
      const uint32_t cell = key & 0x0FFFFFFFu;
      auto it = jof.find(cell);
      if (it == jof.end()) {
        const int j = (int)jof.size();
        it = jof.emplace(cell, j).first;
        const int io = (int)(cell >> 3), c = (int)(cell & 7);
        struct OCT *oc = lc.octs[io];
        const double dxcur = std::pow(0.5, oc->level);
        int nb[6];
        int wm = -1, wp = -1;  // like the reference, a missing neighbour keeps the previous one
        for (int dir = 0; dir < 3; dir++) {
          if (H.grav) wm = wp = -1;
          for (int side = 0; side < 2; side++) {
            const int k = 2 * dir + side;
            int &w = side ? wp : wm;
            const int c2 = c ^ (1 << dir);
            if (inside(c, k)) {
              w = 8 * io + c2;
            } else if (oc->nei[k] != nullptr && oc->nei[k]->child != nullptr) {
              const int jo = P.idx[L - 1].get(oc->nei[k]->child);
              if (jo >= 0) w = 8 * jo + c2;
            }
            const bool bnd = side ? ((k == 1 && oc->x + 2. * dxcur == 1.) || (k == 3 && oc->y + 2. * dxcur == 1.) ||
                                     (k == 5 && oc->z + 2. * dxcur == 1.))
                                  : ((k == 0 && oc->x == 0.) || (k == 2 && oc->y == 0.) || (k == 4 && oc->z == 0.));
            if (((H.trans >> k) & 1) && bnd) w = (int)cell;
            if (w < 0) {
              err = "coarse cell without a slope neighbour at level " + std::to_string(L - 1);
              return EMMA_ST_TREE;
            }
            nb[k] = w;
          }
        }
        lv.interp.push_back((int32_t)cell);
        for (int k = 0; k < 6; k++) lv.interp.push_back(nb[k]);
      }
      key = key_make(kKeyInterp, (uint32_t)it->second);
    }
  }
  return 0;
}

}  // namespace

int validate_host_tree(const HostTree &H, int plan_lo, int plan_hi, std::string &err);

int build_host_tree(struct OCT **firstoct, int lcoarse, int lmax, int rank, int trans, int plan_lo, int plan_hi,
                    HostTree &H, std::string &err, const int *shapes, int grav, int dual) {
  H = HostTree();
  H.dual = dual ? 1 : 0;
  if (grav && trans) {
    err = "gravity coupling with transmissive boundaries is not supported";
    return EMMA_ST_ARG;
  }
  H.grav = grav ? 1 : 0;
  H.lcoarse = lcoarse;
  H.lmax = lmax;
  H.rank = rank;
  H.trans = trans;
  H.lev.assign((size_t)lmax + 1, HostLevel());
  Planner P(H);
  P.idx.resize((size_t)lmax + 2);
  P.face.resize((size_t)lmax + 1);
  for (int L = lcoarse; L <= lmax; L++) {
    HostLevel &lv = H.lev[L];
    lv.L = L;
    for (struct OCT *o = firstoct[L - 1]; o != nullptr; o = o->next)
      if (o->cpu == rank) lv.octs.push_back(o);
    lv.nown = (int)lv.octs.size();
    // octs of other ranks (the boundary octs of a multi-rank run, refreshed by the
    // caller's exchange before each solve): staged as neighbours, never advanced;
    // their coarser cells collect fine->coarse corrections in fieldnew like this
    // rank's (src/hydro_utils.c:2997,3124,3417 skip them; src/communication.c:510
    // sends those fieldnew back to the owners)
    for (struct OCT *o = firstoct[L - 1]; o != nullptr; o = o->next)
      if (o->cpu != rank) lv.octs.push_back(o);
    lv.noct = (int)lv.octs.size();
    if (lv.noct > lv.nown) H.ghosts = 1;
    if (lv.noct >= (1 << 25)) {
      err = "level too large for 28-bit keys";
      return EMMA_ST_ARG;
    }
    P.idx[L].init(lv.octs.size());
    for (int i = 0; i < lv.noct; i++) P.idx[L].put(lv.octs[i], i);
  }
  for (int L = lcoarse; L <= lmax; L++) {
    HostLevel &lv = H.lev[L];
    lv.split.assign(lv.noct, 0);
    lv.child.assign((size_t)8 * lv.noct, -1);
    lv.leaf = 0;
    for (int i = 0; i < lv.noct; i++)
      for (int c = 0; c < 8; c++) {
        struct OCT *ch = lv.octs[i]->cell[c].child;
        if (ch != nullptr) {
          lv.split[i] |= (uint8_t)(1 << c);
          const int j = (L + 1 <= lmax) ? P.idx[L + 1].get(ch) : -1;
          lv.child[8 * i + c] = j;
        } else if (i < lv.nown) {
          lv.leaf++;
        }
      }
    P.face[L].assign((size_t)6 * lv.noct, kKeyNone);
    for (int i = 0; i < lv.noct; i++)
      for (int k = 0; k < 6; k++) P.face[L][6 * i + k] = P.real_nbr(L, i, k);
    lv.nb6.assign((size_t)6 * lv.noct, -1);
    for (size_t j = 0; j < lv.nb6.size(); j++) {
      const uint32_t key = P.face[L][j], kind = key >> 28;
      if (key == kKeyNone) continue;
      if (kind == kKeyReal) lv.nb6[j] = (int32_t)(key & 0x0FFFFFFFu);
      else if (kind >= kKeyGhost0 && kind < kKeyGhost0 + 6) lv.nb6[j] = -2;
    }
    // integer oct positions on the level grid
    const double scale = std::ldexp(1.0, L - 1);
    const int n = 1 << (L - 1);
    lv.pos.assign((size_t)3 * lv.noct, 0);
    for (int i = 0; i < lv.noct; i++) {
      const struct OCT *o = lv.octs[i];
      const double q[3] = {o->x * scale, o->y * scale, o->z * scale};
      for (int a = 0; a < 3; a++) {
        const double r = std::floor(q[a] + 0.5);
        if (r != q[a] || r < 0 || r >= n) {
          err = "oct position off the level grid at level " + std::to_string(L);
          return EMMA_ST_TREE;
        }
        lv.pos[3 * i + a] = (int32_t)r;
      }
    }
  }
  for (int L = std::max(lcoarse, plan_lo); L <= std::min(lmax, plan_hi); L++) {
    const int rc = plan_level(P, H, L, shapes ? shapes[L] : -1, err);
    if (rc != 0) return rc;
  }
  return validate_host_tree(H, plan_lo, plan_hi, err);
}

int replan_level(HostTree &H, int L, int shape, std::string &err) {
  if (L < H.lcoarse || L > H.lmax) {
    err = "level outside the mirrored tree";
    return EMMA_ST_ARG;
  }
  Planner P(H);
  P.idx.resize((size_t)H.lmax + 2);
  P.face.resize((size_t)H.lmax + 1);
  for (int l = std::max(H.lcoarse, L - 1); l <= L; l++) {
    const HostLevel &lv = H.lev[l];
    P.idx[l].init(lv.octs.size());
    for (int i = 0; i < lv.noct; i++) P.idx[l].put(lv.octs[i], i);
  }
  HostLevel &lv = H.lev[L];
  P.face[L].assign((size_t)6 * lv.noct, kKeyNone);
  for (int i = 0; i < lv.noct; i++)
    for (int k = 0; k < 6; k++) P.face[L][6 * i + k] = P.real_nbr(L, i, k);
  const int rc = plan_level(P, H, L, shape, err);
  if (rc != 0) return rc;
  return validate_host_tree(H, L, L, err);
}

// Every index a level kernel dereferences comes from these arrays; check them
// all against their buffers before anything is uploaded.
int validate_host_tree(const HostTree &H, int plan_lo, int plan_hi, std::string &err) {
  for (int L = std::max(H.lcoarse, plan_lo); L <= std::min(H.lmax, plan_hi); L++) {
    const HostLevel &lv = H.lev[L];
    const long long ncoarse8 = (L > H.lcoarse) ? 8LL * H.lev[L - 1].noct : 0;
    const long long nfine = (L < H.lmax) ? H.lev[L + 1].noct : 0;
    if (lv.shape < 0 || lv.shape >= kNumShapes) {
      err = "invalid brick shape at level " + std::to_string(L);
      return EMMA_ST_TREE;
    }
    const BrickShape &sh = kShapes[lv.shape];
    if (lv.keys.size() != lv.tiles.size() * (size_t)sh.tile_slots()) {
      err = "slot keys do not match the tiles at level " + std::to_string(L);
      return EMMA_ST_TREE;
    }
    std::vector<uint8_t> seen((size_t)lv.noct, 0);
    long long covered = 0;
    for (size_t t = 0; t < lv.tiles.size(); t++) {
      const TileDesc &td = lv.tiles[t];
      if (td.mask == 0 || td.noct != __builtin_popcount(td.mask)) {
        err = "invalid tile descriptor at level " + std::to_string(L);
        return EMMA_ST_TREE;
      }
      const uint32_t *keys = &lv.keys[t * (size_t)sh.tile_slots()];
      for (int s = 0; s < sh.tile_slots(); s++) {
        const uint32_t key = keys[s];
        if (key == kKeyNone) continue;
        const uint32_t kind = key >> 28, idx = key & 0x0FFFFFFFu;
        const bool ok = (kind == kKeyReal || (kind >= kKeyGhost0 && kind < kKeyGhost0 + 6)) ? (idx < (uint32_t)lv.noct)
                        : (kind == kKeyInj) ? ((long long)idx < ncoarse8)
                        : (kind == kKeyInterp) ? ((size_t)idx < lv.interp.size() / 7)
                                               : false;
        if (!ok) {
          err = "invalid staged key at level " + std::to_string(L);
          return EMMA_ST_TREE;
        }
      }
      for (int m = 0; m < sh.nb * sh.octs(); m++) {
        if (!((td.mask >> m) & 1)) continue;
        const int nb = m / sh.octs(), i = m % sh.octs();
        const int sx = 1 + i % sh.bx, sy = 1 + (i / sh.bx) % sh.by, sz = 1 + i / (sh.bx * sh.by);
        const uint32_t key = keys[nb * sh.slots() + sx + (sh.bx + 2) * (sy + (sh.by + 2) * sz)];
        if ((key >> 28) != kKeyReal || (key & 0x0FFFFFFFu) >= (uint32_t)lv.nown || seen[key & 0x0FFFFFFFu]) {
          err = "tile oct missing or advanced twice at level " + std::to_string(L);
          return EMMA_ST_TREE;
        }
        seen[key & 0x0FFFFFFFu] = 1;
        covered++;
      }
    }
    if (covered != lv.nown) {
      err = "tiles do not cover level " + std::to_string(L);
      return EMMA_ST_TREE;
    }
    for (size_t i = 0; i < 8 * (size_t)lv.nown; i++) {  // children of this rank's octs
      const bool split = (lv.split[i >> 3] >> (i & 7)) & 1;
      if (split && (lv.child[i] < 0 || lv.child[i] >= nfine) && L < H.lmax) {
        err = "split cell without a mirrored child at level " + std::to_string(L);
        return EMMA_ST_TREE;
      }
    }
    for (int32_t c : lv.inj_cells)
      if (c < 0 || c >= ncoarse8) {
        err = "invalid injected cell at level " + std::to_string(L);
        return EMMA_ST_TREE;
      }
    if (lv.interp.size() % 7 != 0) {
      err = "invalid interpolation list at level " + std::to_string(L);
      return EMMA_ST_TREE;
    }
    for (int32_t c : lv.interp)
      if (c < 0 || c >= ncoarse8) {
        err = "invalid interpolated cell at level " + std::to_string(L);
        return EMMA_ST_TREE;
      }
  }
  return 0;
}

}  // namespace emma
