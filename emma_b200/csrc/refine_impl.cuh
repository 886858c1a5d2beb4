// refine_impl.cuh -- device-side refinement of the resident tree: the
// reference's marking (L_mark_cells, src/amr.c:883-1445), 2:1 check rule
// (L_check_rule, :746-868) and refinement (L_refine_cells, :286-735).
// Included by api.cu inside its internal namespace (it uses the resident
// context).
//
// Marks live on the device, one int per cell of every resident level (uploaded
// from the cells' `marked` with the tree).  Every marking pass is a kernel over
// the level's cells: a pass only turns unmarked cells into the pass's marker
// and reads marks of earlier passes, so its result does not depend on the
// order the reference sweeps the list in.  Refinement then needs the level's
// marks on the host once (a few bytes per cell): the octs are created and
// destroyed in the caller's struct OCT tree in the reference's sweep order,
// from the caller's free-oct chain, so every list keeps the reference's order
// and every pointer the reference's value; the fields never leave the GPU --
// the new finer level's state is gathered on the device from its surviving
// octs and from the parent cells the new octs are injected from
// (src/hydro_utils.c:512-520: every child cell copies the parent's field).

// cell across face k (-x,+x,-y,+y,-z,+z) of cell c of oct o at the same level,
// or -1 where the level has no oct there (getcellnei, src/oct.c:116-185)
__device__ __forceinline__ long long same_level_nbr(const int *__restrict__ nb6, long long o, int c, int k) {
  const int bit = 1 << (k >> 1);
  const bool inside = (k & 1) ? !(c & bit) : (c & bit);
  if (inside) return 8 * o + (c ^ bit);
  const int no = nb6[6 * o + k];
  return no >= 0 ? 8LL * no + (c ^ bit) : -1;
}

// pass 0: an unmarked split cell whose child holds a marked or split cell keeps
// its child (src/amr.c:937-949)
__global__ void k_mark_keep(int *marks, const int *__restrict__ child, const int *__restrict__ fmarks,
                            const int *__restrict__ fchild, long long n8, int marker) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n8; i += (long long)gridDim.x * blockDim.x) {
    const int ch = child[i];
    if (ch < 0 || marks[i] != 0) continue;
    int s = 0;
    for (int j = 0; j < 8; j++) s += (fmarks[8LL * ch + j] != 0) || (fchild[8LL * ch + j] >= 0);
    if (s != 0) marks[i] = marker;
  }
}

// pass 1: every cell marked by an earlier pass marks the cells of its 3x3x3 block
// it reaches through existing cells: its 6 face neighbours, their 4 side
// neighbours, their 2 corner neighbours (src/amr.c:951-1129)
__global__ void k_mark_spread(int *marks, const int *__restrict__ nb6, long long n8, int marker) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n8; i += (long long)gridDim.x * blockDim.x) {
    const int m = marks[i];
    if (!(m > 0 && m < marker)) continue;
    auto put = [&](long long x) {
      if (marks[x] == 0) marks[x] = marker;  // every writer writes the same value
    };
    for (int ii = 0; ii < 6; ii++) {
      const long long n1 = same_level_nbr(nb6, i >> 3, (int)(i & 7), ii);
      if (n1 < 0) continue;
      put(n1);
      for (int il = 0; il < 6; il++) {
        if (il / 2 == ii / 2) continue;
        const long long n2 = same_level_nbr(nb6, n1 >> 3, (int)(n1 & 7), il);
        if (n2 < 0) continue;
        put(n2);
        for (int ip = 0; ip < 6; ip++) {
          if (ip / 2 == il / 2 || ip / 2 == ii / 2) continue;
          const long long n3 = same_level_nbr(nb6, n2 >> 3, (int)(n2 & 7), ip);
          if (n3 >= 0) put(n3);
        }
      }
    }
  }
}

// pass 2, first smoothing iteration only: the density criterion (the reference's
// -DSNTEST branch, src/amr.c:1330-1354, with the threshold a parameter)
__global__ void k_mark_density(int *marks, const double *__restrict__ d, long long n8, double threshold, int marker) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n8; i += (long long)gridDim.x * blockDim.x)
    if (marks[i] == 0 && d[i] > threshold) marks[i] = marker;
}

// 2:1 rule: the marks of an oct whose 26 neighbours (faces, then edges, then
// corners) do not all exist at its level are cancelled with 10
// (src/amr.c:746-868)
__global__ void k_check_rule(int *marks, const int *__restrict__ nb6, long long noct) {
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < noct; o += (long long)gridDim.x * blockDim.x) {
    bool any = false;
    for (int c = 0; c < 8; c++) any = any || marks[8 * o + c] != 0;
    if (!any) continue;
    bool bad = false;
    for (int ii = 0; ii < 6; ii++) {
      const int f = nb6[6 * o + ii];
      if (f < 0) {
        bad = true;
        continue;
      }
      for (int i2 = 0; i2 < 6; i2++) {
        if (i2 / 2 == ii / 2) continue;
        const int e = nb6[6LL * f + i2];
        if (e < 0) {
          bad = true;
          continue;
        }
        for (int i3 = 0; i3 < 6; i3++) {
          if (i3 / 2 == ii / 2 || i3 / 2 == i2 / 2) continue;
          if (nb6[6LL * e + i3] < 0) bad = true;
        }
      }
    }
    if (bad)
      for (int c = 0; c < 8; c++)
        if (marks[8 * o + c] != 0) marks[8 * o + c] = 10;
  }
}

// state (5 planes) and marks of the refined level's finer level in its new list
// order: src[o] >= 0 is a surviving oct's old index, -(parent cell + 1) a new oct
// whose 8 cells take the parent cell's state
__global__ void k_refine_gather(double *__restrict__ dst, int *__restrict__ dmarks, long long n8, const int *__restrict__ src,
                                const double *__restrict__ oldW, const int *__restrict__ oldmarks, long long n8old,
                                const double *__restrict__ parW, long long n8par) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n8; i += (long long)gridDim.x * blockDim.x) {
    const int s = src[i >> 3];
    const long long j = (s >= 0) ? 8LL * s + (i & 7) : (long long)(-s - 1);
    for (int v = 0; v < 5; v++) dst[v * n8 + i] = (s >= 0) ? oldW[v * n8old + j] : parW[v * n8par + j];
    dmarks[i] = (s >= 0) ? oldmarks[j] : 0;
  }
}

unsigned grid_for(long long n) { return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 8LL * g.nsm)); }

// the resident tree uploaded from firstoct whose level `level` can be marked and
// refined on the device (plain variant, periodic)
int refine_ok(struct OCT **firstoct, int level, bool need_finer) {
  if (!(g.ready && g.res.valid && firstoct != nullptr && g.res_first == firstoct)) {
    fail(EMMA_ST_ARG, "device refinement needs the resident tree uploaded from this firstoct");
    return EMMA_ST_ARG;
  }
  if (level < g.res.lcoarse || level > g.res.lmax || (need_finer && level >= g.res.lmax)) {
    fail(EMMA_ST_ARG, "level " + std::to_string(level) + " cannot be refined in the resident tree");
    return EMMA_ST_ARG;
  }
  if (g.opt.trans_flags || g.res.host.grav || g.opt.dual_energy || kDropinTracer) {
    fail(EMMA_ST_ARG, "device refinement is built for periodic trees of the plain variant");
    return EMMA_ST_ARG;
  }
  return 0;
}

// L_mark_cells on the device after L_clean_marks (the reference's driver clears
// the level's marks before marking it, src/advanceamr.c:1230-1236)
int device_mark_cells(int level, int nsmooth, double threshold) {
  DevLevel &d = g.res.lev[level];
  if (d.n8 == 0) return 0;
  CK(cudaMemsetAsync(d.marks, 0, sizeof(int) * d.n8, g.stream));
  const double *W = current_state(level);
  if (W == nullptr) return EMMA_ST_CUDA;
  const bool finer = level < g.res.lmax && g.res.lev[level + 1].n8 > 0;
  const int *fmarks = finer ? g.res.lev[level + 1].marks : nullptr;
  const int *fchild = finer ? g.res.lev[level + 1].child : nullptr;
  int marker = 0;
  for (int is = 0; is < nsmooth; is++) {
    ++marker;
    if (finer) k_mark_keep<<<grid_for(d.n8), 256, 0, g.stream>>>(d.marks, d.child, fmarks, fchild, d.n8, marker);
    ++marker;
    k_mark_spread<<<grid_for(d.n8), 256, 0, g.stream>>>(d.marks, d.nb6, d.n8, marker);
    ++marker;
    if (is == 0) k_mark_density<<<grid_for(d.n8), 256, 0, g.stream>>>(d.marks, W, d.n8, threshold, marker);
  }
  CK(cudaGetLastError());
  return 0;
}

int device_check_rule(int level) {
  DevLevel &d = g.res.lev[level];
  if (d.noct == 0) return 0;
  k_check_rule<<<grid_for(d.noct), 256, 0, g.stream>>>(d.marks, d.nb6, d.noct);
  CK(cudaGetLastError());
  return 0;
}

// the device marks of a level into the cells' `marked` of the host tree
int marks_to_host(int level) {
  const DevLevel &d = g.res.lev[level];
  const HostLevel &h = g.res.host.lev[level];
  if (d.n8 == 0) return 0;
  std::vector<int> m((size_t)d.n8);
  CK(cudaMemcpyAsync(m.data(), d.marks, sizeof(int) * d.n8, cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  g.d2h_bytes += (long long)(sizeof(int) * d.n8);
  for (int i = 0; i < h.noct; i++)
    for (int c = 0; c < 8; c++) h.octs[i]->cell[c].marked = (REAL)m[8 * (size_t)i + c];
  return 0;
}

// L_refine_cells' sweep on the host tree (src/amr.c:330-710): in list order, an
// unmarked split cell of a level >= lcoarse loses its child oct (unlinked from
// the finer list, pushed on the free chain), a marked leaf with a mark below 10
// gets a new child oct (popped from the free chain, appended to the finer list,
// linked to its neighbours, its cells' fields copied from the parent).  Returns
// the new head of the free chain, or nullptr with `err` set where the reference
// aborts.  `created` receives the new octs in creation order.
struct OCT *refine_sweep(int level, int lcoarse, struct OCT **firstoct, struct OCT **lastoct, struct OCT *freeoct,
                         struct OCT *limit, std::vector<struct OCT *> &created, std::string &err) {
  struct OCT *newoct = freeoct;
  const double dxcur = 1. / std::pow(2., level);
  for (struct OCT *cur = firstoct[level - 1], *next = nullptr; cur != nullptr; cur = next) {
    next = cur->next;
    for (int icell = 0; icell < 8; icell++) {
      if (newoct == nullptr || newoct->level != 0) {
        err = "the free-oct chain does not start with a free oct";
        return nullptr;
      }
      struct CELL &cell = cur->cell[icell];
      if (cell.child != nullptr && cell.marked == 0. && cur->level >= lcoarse) {
        struct OCT *des = cell.child;
        for (int c = 0; c < 8; c++)
          if (des->cell[c].child != nullptr) {
            err = "an oct to destroy has children of its own";
            return nullptr;
          }
        cell.child = nullptr;
        des->parent = nullptr;
        if (des->prev != nullptr) des->prev->next = des->next;
        else firstoct[level] = des->next;
        if (des->next != nullptr) des->next->prev = des->prev;
        else lastoct[level] = des->prev;
        des->level = 0;
        des->prev = nullptr;
        freeoct->prev = des;
        des->next = freeoct;
        freeoct = des;
        newoct = freeoct;
      }
      if (cell.child == nullptr && cell.marked != 0. && cell.marked < 10.) {
        // neighbours of the new oct: the parent level's cells across its faces
        // (the reference aborts when the 2:1 rule left one missing)
        struct CELL *nei[6];
        for (int k = 0; k < 6; k++) {
          const int bit = 1 << (k >> 1);
          const bool inside = (k & 1) ? !(icell & bit) : (icell & bit);
          if (inside) {
            nei[k] = &cur->cell[icell ^ bit];
          } else {
            struct CELL *nc = cur->nei[k];
            if (nc == nullptr || nc->child == nullptr) {
              err = "refinement would break the 2:1 rule (a neighbour oct is missing)";
              return nullptr;
            }
            nei[k] = &nc->child->cell[icell ^ bit];
          }
        }
        newoct->parent = &cell;
        newoct->level = cur->level + 1;
        newoct->x = cur->x + (icell % 2) * dxcur;
        newoct->y = cur->y + ((icell / 2) % 2) * dxcur;
        newoct->z = cur->z + (icell / 4) * dxcur;
        cell.child = newoct;
        newoct->cpu = cur->cpu;
        for (int k = 0; k < 6; k++) newoct->nei[k] = nei[k];
        for (int c = 0; c < 8; c++) {
          struct CELL &nc = newoct->cell[c];
          nc.marked = 0.;
          nc.child = nullptr;
          nc.idx = c;
          nc.field = cell.field;
          nc.fieldnew = cell.field;
        }
        freeoct = newoct->next;
        if (freeoct == nullptr) {
          err = "the free-oct chain is exhausted";
          return nullptr;
        }
        freeoct->prev = nullptr;
        newoct->next = nullptr;
        if (firstoct[level] == nullptr) {
          firstoct[level] = newoct;
          newoct->prev = nullptr;
        } else {
          newoct->prev = lastoct[level];
          lastoct[level]->next = newoct;
        }
        lastoct[level] = newoct;
        created.push_back(newoct);
        newoct = freeoct;
        if (newoct >= limit - 1) {
          err = "the oct pool is full (the reference's ngridmax)";
          return nullptr;
        }
      }
    }
  }
  return freeoct;
}

// After a refinement sweep of `level`: a new mirror of the host tree, the device
// states of every level carried over (the refined level's finer level gathered
// into its new list order), the old device tree released.
int rebuild_after_refine(struct OCT **firstoct, int level, const std::vector<struct OCT *> &created) {
  Tree &old = g.res;
  const int lc = old.lcoarse, lm = old.lmax;
  Tree nt;
  std::string err;
  // the brick shape the options request (a forced one), else the planner's cost model
  int shape = -1;
  for (int i = 0; i < kNumShapes; i++)
    if (g.opt.tile_octs != 0 && kShapes[i].octs() == g.opt.tile_octs) shape = i;
  std::vector<int> shapes((size_t)lm + 1, shape);
  int rc = build_host_tree(firstoct, lc, lm, old.host.rank, g.opt.trans_flags, lc, lm, nt.host, err, shapes.data(), 0, 0);
  if (rc != 0) {
    fail((unsigned)rc, "re-planning after refinement: " + err);
    return rc;
  }
  if (!alloc_tree(nt.host, nt, false)) return EMMA_ST_CUDA;
  const int fl = level + 1;
  // where each oct of the finer level comes from
  std::unordered_set<const struct OCT *> fresh(created.begin(), created.end());
  std::unordered_map<const struct OCT *, int> old_idx;
  const HostLevel &ho = old.host.lev[fl];
  for (int i = 0; i < ho.noct; i++) old_idx[ho.octs[i]] = i;
  const HostLevel &hn = nt.host.lev[fl];
  const HostLevel &hp = nt.host.lev[level];
  std::vector<int> src((size_t)hn.noct, 0);
  for (int i = 0; i < hp.noct; i++)
    for (int c = 0; c < 8; c++) {
      const int j = hp.child[8 * (size_t)i + c];
      if (j >= 0) src[j] = -(8 * i + c) - 1;
    }
  for (int i = 0; i < hn.noct; i++) {
    if (fresh.count(hn.octs[i])) continue;
    const auto it = old_idx.find(hn.octs[i]);
    if (it == old_idx.end()) {
      fail(EMMA_ST_TREE, "an oct of the refined level's finer level is neither old nor new");
      free_tree(nt);
      return EMMA_ST_TREE;
    }
    src[i] = it->second;
  }
  bool ok = true;
  int *d_src = nullptr;
  for (int L = lc; L <= lm && ok; L++) {
    const DevLevel &dn = nt.lev[L], &dold = old.lev[L];
    if (dn.n8 == 0) continue;
    if (L != fl) {  // same octs in the same order
      double *W = current_state(L);
      ok = W != nullptr && dn.n8 == dold.n8 &&
           ck(cudaMemcpyAsync(dn.W0, W, sizeof(double) * 5 * dn.n8, cudaMemcpyDeviceToDevice, g.stream), "state") &&
           ck(cudaMemcpyAsync(dn.marks, dold.marks, sizeof(int) * dn.n8, cudaMemcpyDeviceToDevice, g.stream), "marks");
    } else {
      double *Wold = dold.n8 > 0 ? current_state(L) : nullptr;
      const double *Wp = current_state(level);
      ok = Wp != nullptr && upload_vec(&d_src, src);
      if (ok) {
        k_refine_gather<<<grid_for(dn.n8), 256, 0, g.stream>>>(dn.W0, dn.marks, dn.n8, d_src, Wold, dold.marks,
                                                              dold.n8, Wp, old.lev[level].n8);
        ok = ck(cudaGetLastError(), "refine gather");
      }
    }
  }
  ok = ok && ck(cudaStreamSynchronize(g.stream), "sync after refinement");
  cudaFree(d_src);
  if (!ok) {
    free_tree(nt);
    return EMMA_ST_CUDA;
  }
  drop_graph();
  free_tree(old);
  g.res = std::move(nt);
  // the finer level's state changed outside the schedule: its next CFL step comes
  // from the reduction kernel; the batched work list follows the new plans
  if (mark_stale(fl) != cudaSuccess) return EMMA_ST_CUDA;
  cudaFree(g.d_work_all);
  g.d_work_all = nullptr;
  std::vector<int> all;
  for (int L = lm; L >= lc; L--)
    for (int i = 0; i < g.res.lev[L].ntiles; i++) all.push_back((L << kWorkSlotShift) | i);
  if (!upload_vec(&g.d_work_all, all)) return EMMA_ST_CUDA;
  g.nwork_all = (int)all.size();
  return 0;
}
