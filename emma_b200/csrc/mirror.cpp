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
// virtual grid one oct at a time; a tile stages the union of the windows of
// its octs (faces and edges; MUSCL never reads the corners) without duplicates.
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

struct TileBuild {
  std::vector<uint32_t> keys;
  std::vector<uint8_t> graph;
  std::vector<uint16_t> halo;
  std::vector<uint16_t> bface;
  int S = 0, H = 0, B = 0;
};

// Stage list, neighbour graph and halo of the tile [o0, o0+n).  Returns false
// if a needed neighbour is missing (error bit set in the planner).
bool build_tile(Planner &P, int L, int o0, int n, TileBuild &tb) {
  std::unordered_map<uint32_t, int> pos;
  pos.reserve(256);
  tb.keys.clear();
  auto add = [&](uint32_t key) {
    if (key == kKeyNone) return;
    if (pos.find(key) == pos.end()) {
      pos.emplace(key, (int)tb.keys.size());
      tb.keys.push_back(key);
    }
  };
  for (int t = 0; t < n; t++) add(key_make(kKeyReal, (uint32_t)(o0 + t)));
  for (int t = 0; t < n; t++) {
    const uint32_t self = key_make(kKeyReal, (uint32_t)(o0 + t));
    for (int k = 0; k < 6; k++) {
      const uint32_t f = P.vnbr(L, self, k);
      if (f == kKeyNone) {
        P.err |= EMMA_ST_TREE;
        P.msg = "missing face neighbour of a level-" + std::to_string(L) + " oct";
        return false;
      }
      add(f);
    }
  }
  // edges: neighbours of the face neighbours off the face axis
  for (int t = 0; t < n; t++) {
    const uint32_t self = key_make(kKeyReal, (uint32_t)(o0 + t));
    for (int k = 0; k < 6; k++) {
      const uint32_t f = P.vnbr(L, self, k);
      for (int j = 0; j < 6; j++) {
        if ((j >> 1) == (k >> 1)) continue;
        add(P.vnbr(L, f, j));
      }
    }
  }
  tb.S = (int)tb.keys.size();
  tb.H = 0;
  if (tb.S > kSMax) return true;  // too many staged octs: the caller shrinks the tile
  tb.graph.assign((size_t)tb.S * 6, 255);
  for (int s = 0; s < tb.S; s++)
    for (int k = 0; k < 6; k++) {
      const uint32_t g = P.vnbr(L, tb.keys[s], k);
      auto it = (g == kKeyNone) ? pos.end() : pos.find(g);
      if (it != pos.end() && it->second < 255) tb.graph[6 * s + k] = (uint8_t)it->second;
    }
  // halo entries: (cell of a non-tile staged oct, its face toward a tile oct)
  tb.halo.clear();
  for (int s = n; s < tb.S; s++)
    for (int c = 0; c < 8; c++)
      for (int k = 0; k < 6; k++) {
        if (inside(c, k)) continue;
        const int g = tb.graph[6 * s + k];
        if (g != 255 && g < n) tb.halo.push_back((uint16_t)(((8 * s + c) << 3) | k));
      }
  tb.H = (int)tb.halo.size();
  if (tb.H > kHMax) return true;  // too many halo entries: the caller shrinks the tile
  // + faces of tile cells that border a non-tile staged oct
  tb.bface.clear();
  for (int t = 0; t < 8 * n; t++)
    for (int d = 0; d < 3; d++) {
      const int k = 2 * d + 1, c = t & 7;
      if (inside(c, k)) continue;
      const int g = tb.graph[6 * (t >> 3) + k];
      if (g == 255 || g >= n) tb.bface.push_back((uint16_t)(4 * t + d));
    }
  tb.B = (int)tb.bface.size();
  if (tb.B > kBMax) return true;
  // every neighbour a reconstruction reads must be staged
  auto need = [&](int s, int c) -> bool {
    for (int k = 0; k < 6; k++) {
      if (inside(c, k)) continue;
      if (tb.graph[6 * s + k] == 255) return false;
    }
    return true;
  };
  for (int s = 0; s < n; s++)
    for (int c = 0; c < 8; c++)
      if (!need(s, c)) {
        P.err |= EMMA_ST_TREE;
        P.msg = "unstaged neighbour of a tile cell";
        return false;
      }
  for (uint16_t e16 : tb.halo)
    if (!need(e16 >> 6, (e16 >> 3) & 7)) {
      const int e = e16 >> 3;
      P.err |= EMMA_ST_TREE;
      const uint32_t key = tb.keys[e >> 3];
      if (std::getenv("EMMA_PLAN_DEBUG")) {
        std::fprintf(stderr, "tile o0=%d n=%d S=%d H=%d failing staged %d cell %d\n", o0, n, tb.S, tb.H, e >> 3, e & 7);
        for (int s = 0; s < tb.S; s++) {
          std::fprintf(stderr, "  s=%3d kind=%u idx=%u g=", s, tb.keys[s] >> 28, tb.keys[s] & 0x0FFFFFFFu);
          for (int k = 0; k < 6; k++) {
            uint32_t vk = P.vnbr(L, tb.keys[s], k);
            std::fprintf(stderr, " %3d(%u:%u)", tb.graph[6 * s + k], vk == kKeyNone ? 9 : vk >> 28, vk & 0x0FFFFFFFu);
          }
          std::fprintf(stderr, "\n");
        }
      }
      P.msg = "unstaged neighbour of a halo cell (level " + std::to_string(L) + ", tile at oct " +
              std::to_string(o0) + ", staged kind " + std::to_string(key >> 28) + " index " +
              std::to_string(key & 0x0FFFFFFFu) + ", cell " + std::to_string(e & 7) + ")";
      return false;
    }
  return true;
}

}  // namespace

int validate_host_tree(const HostTree &H, int plan_lo, int plan_hi, std::string &err);

int build_host_tree(struct OCT **firstoct, int lcoarse, int lmax, int rank, int trans, int plan_lo, int plan_hi,
                    HostTree &H, std::string &err) {
  H = HostTree();
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
    lv.noct = (int)lv.octs.size();
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
        } else {
          lv.leaf++;
        }
      }
    P.face[L].assign((size_t)6 * lv.noct, kKeyNone);
    for (int i = 0; i < lv.noct; i++)
      for (int k = 0; k < 6; k++) P.face[L][6 * i + k] = P.real_nbr(L, i, k);
  }
  for (int L = std::max(lcoarse, plan_lo); L <= std::min(lmax, plan_hi); L++) {
    HostLevel &lv = H.lev[L];
    std::unordered_map<std::string, int> gdedup, hdedup, bdedup;
    std::vector<uint8_t> injmark;
    if (L > lcoarse) injmark.assign((size_t)8 * H.lev[L - 1].noct, 0);
    TileBuild tb;
    int o0 = 0;
    while (o0 < lv.noct) {
      int n = std::min(kTileOcts, lv.noct - o0);
      for (;;) {
        if (!build_tile(P, L, o0, n, tb)) {
          err = P.msg;
          return (int)P.err;
        }
        if ((tb.S <= kSMax && tb.H <= kHMax && tb.B <= kBMax) || n == 1) break;
        n = (n > 8) ? n - 4 : n - 1;
      }
      if (tb.S > kSMax || tb.H > kHMax || tb.B > kBMax) {
        err = "single-oct tile exceeds the staging limits";
        return EMMA_ST_TREE;
      }
      TileDesc td;
      std::memset(&td, 0, sizeof(td));
      td.oct0 = o0;
      td.noct = n;
      td.S = tb.S;
      td.H = tb.H;
      td.B = tb.B;
      td.keys_off = (int)lv.keys.size();
      lv.keys.insert(lv.keys.end(), tb.keys.begin(), tb.keys.end());
      for (uint32_t key : tb.keys)
        if ((key >> 28) == kKeyInj && !injmark.empty()) injmark[key & 0x0FFFFFFFu] = 1;
      std::string gk(reinterpret_cast<const char *>(tb.graph.data()), tb.graph.size());
      auto git = gdedup.find(gk);
      if (git == gdedup.end()) {
        td.graph_off = (int)lv.graph.size();
        lv.graph.insert(lv.graph.end(), tb.graph.begin(), tb.graph.end());
        gdedup.emplace(std::move(gk), td.graph_off);
      } else {
        td.graph_off = git->second;
      }
      std::string hk(reinterpret_cast<const char *>(tb.halo.data()), tb.halo.size() * sizeof(uint16_t));
      auto hit = hdedup.find(hk);
      if (hit == hdedup.end()) {
        td.halo_off = (int)lv.halo.size();
        lv.halo.insert(lv.halo.end(), tb.halo.begin(), tb.halo.end());
        hdedup.emplace(std::move(hk), td.halo_off);
      } else {
        td.halo_off = hit->second;
      }
      std::string bk(reinterpret_cast<const char *>(tb.bface.data()), tb.bface.size() * sizeof(uint16_t));
      auto bit = bdedup.find(bk);
      if (bit == bdedup.end()) {
        td.bface_off = (int)lv.bface.size();
        lv.bface.insert(lv.bface.end(), tb.bface.begin(), tb.bface.end());
        bdedup.emplace(std::move(bk), td.bface_off);
      } else {
        td.bface_off = bit->second;
      }
      lv.tiles.push_back(td);
      o0 += n;
    }
    for (size_t i = 0; i < injmark.size(); i++)
      if (injmark[i]) lv.inj_cells.push_back((int32_t)i);
  }
  return validate_host_tree(H, plan_lo, plan_hi, err);
}

// Every index a level kernel dereferences comes from these arrays; check them
// all against their buffers before anything is uploaded.
int validate_host_tree(const HostTree &H, int plan_lo, int plan_hi, std::string &err) {
  for (int L = std::max(H.lcoarse, plan_lo); L <= std::min(H.lmax, plan_hi); L++) {
    const HostLevel &lv = H.lev[L];
    const long long ncoarse8 = (L > H.lcoarse) ? 8LL * H.lev[L - 1].noct : 0;
    const long long nfine = (L < H.lmax) ? H.lev[L + 1].noct : 0;
    long long covered = 0;
    for (const TileDesc &t : lv.tiles) {
      if (t.noct < 1 || t.noct > kTileOcts || t.oct0 != covered || t.S < t.noct || t.S > kSMax || t.H < 0 ||
          t.H > kHMax || t.keys_off < 0 || (size_t)t.keys_off + t.S > lv.keys.size() || t.graph_off < 0 ||
          (size_t)t.graph_off + 6 * (size_t)t.S > lv.graph.size() || t.halo_off < 0 ||
          (size_t)t.halo_off + t.H > lv.halo.size()) {
        err = "invalid tile descriptor at level " + std::to_string(L);
        return EMMA_ST_TREE;
      }
      covered += t.noct;
      for (int s = 0; s < t.S; s++) {
        const uint32_t key = lv.keys[t.keys_off + s];
        const uint32_t kind = key >> 28, idx = key & 0x0FFFFFFFu;
        const bool ok = (kind == kKeyReal || (kind >= kKeyGhost0 && kind < kKeyGhost0 + 6)) ? (idx < (uint32_t)lv.noct)
                        : (kind == kKeyInj) ? ((long long)idx < ncoarse8)
                                            : false;
        if (!ok || (s < t.noct && key != key_make(kKeyReal, (uint32_t)(t.oct0 + s)))) {
          err = "invalid staged key at level " + std::to_string(L);
          return EMMA_ST_TREE;
        }
        for (int k = 0; k < 6; k++) {
          const int g = lv.graph[t.graph_off + 6 * s + k];
          if (g != 255 && g >= t.S) {
            err = "invalid graph entry at level " + std::to_string(L);
            return EMMA_ST_TREE;
          }
        }
      }
      if (t.B < 0 || t.B > kBMax || t.bface_off < 0 || (size_t)t.bface_off + t.B > lv.bface.size()) {
        err = "invalid boundary-face range at level " + std::to_string(L);
        return EMMA_ST_TREE;
      }
      for (int h = 0; h < t.H; h++) {
        const int e = lv.halo[t.halo_off + h] >> 3, k = lv.halo[t.halo_off + h] & 7;
        if (e < 8 * t.noct || e >= 8 * t.S || k > 5) {
          err = "invalid halo entry at level " + std::to_string(L);
          return EMMA_ST_TREE;
        }
      }
      for (int b = 0; b < t.B; b++) {
        const int e = lv.bface[t.bface_off + b];
        if ((e >> 2) >= 8 * t.noct || (e & 3) > 2) {
          err = "invalid boundary face at level " + std::to_string(L);
          return EMMA_ST_TREE;
        }
      }
    }
    if (covered != lv.noct) {
      err = "tiles do not cover level " + std::to_string(L);
      return EMMA_ST_TREE;
    }
    for (size_t i = 0; i < lv.child.size(); i++) {
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
  }
  return 0;
}

}  // namespace emma
