// Device schedule builder (see plan.hpp).
#include "plan.hpp"

#include <algorithm>
#include <map>
#include <set>
#include <stdexcept>

namespace amp {

namespace {

// Offline first-fit allocator over one arena (offsets in doubles, 256-byte aligned blocks).
class ArenaPlanner {
 public:
  // best fit among the free blocks (smallest that fits, lowest offset among equals), else the top
  int64_t alloc(int64_t size) {
    size = (size + 31) & ~int64_t(31);
    auto b = bySize_.lower_bound({size, INT64_MIN});
    if (b != bySize_.end()) {
      const int64_t bsize = b->first, off = b->second, rest = bsize - size;
      bySize_.erase(b);
      free_.erase(off);
      if (rest > 0) add_free(off + size, rest);
      used_[off] = size;
      return off;
    }
    int64_t off = top_;
    top_ += size;
    used_[off] = size;
    return off;
  }
  void release(int64_t off) {
    auto u = used_.find(off);
    if (u == used_.end()) throw std::logic_error("arena planner: double free");
    int64_t size = u->second;
    used_.erase(u);
    // merge with the free neighbours
    auto nx = free_.lower_bound(off);
    if (nx != free_.end() && off + size == nx->first) {
      size += nx->second;
      remove_free(nx->first);
    }
    auto pv = free_.lower_bound(off);
    if (pv != free_.begin()) {
      --pv;
      if (pv->first + pv->second == off) {
        off = pv->first;
        size += pv->second;
        remove_free(off);
      }
    }
    if (off + size == top_)  // shrink the top
      top_ = off;
    else
      add_free(off, size);
    peak_ = std::max(peak_, top_);
  }
  int64_t peak() const { return std::max(peak_, top_); }
  void note() { peak_ = std::max(peak_, top_); }

 private:
  void add_free(int64_t off, int64_t size) {
    free_[off] = size;
    bySize_.insert({size, off});
  }
  void remove_free(int64_t off) {
    auto it = free_.find(off);
    bySize_.erase({it->second, off});
    free_.erase(it);
  }
  std::map<int64_t, int64_t> free_, used_;      // offset -> size
  std::set<std::pair<int64_t, int64_t>> bySize_;  // (size, offset) of the free blocks
  int64_t top_ = 0, peak_ = 0;
};

}  // namespace

// An assembly task of front columns [j0, j0 + kAsmCols) of supernode s, with the columns [b0, b1) of each child's
// update matrix that map into them (a child's map is increasing, so they form one range), in the child order.
static void add_asm_task(const Plan &P, int s, int j0, std::vector<AsmTask> &tasks, std::vector<ChildRange> &ranges) {
  const int jend = std::min(j0 + kAsmCols, P.snM[s]);
  tasks.push_back({s, j0, (int)ranges.size()});
  for (int q = P.chPtr[s]; q < P.chPtr[s + 1]; q++) {
    const int c = P.chList[q], muc = std::max(0, P.snM[c] - P.snNc[c]);
    const int *map = P.eaMap.data() + P.eaPtr[c];
    const int b0 = (int)(std::lower_bound(map, map + muc, j0) - map);
    const int b1 = (int)(std::lower_bound(map, map + muc, jend) - map);
    ranges.push_back({b0, b1});
  }
}

// The one-vector forward task list in critical-path order: a topological order of its tasks (a supernode's tasks
// after every task that completes a child's pass-up vector, its diagonal blocks in order, its blocks below after its
// last diagonal block) that lists, among the tasks whose predecessors are already listed, the one with the longest
// estimated path to the end of the sweep first (ties: the level order). The persistent CTAs take tasks in list
// order, so the chains under the large separators start as soon as their inputs allow instead of level by level.
// kinds(s): 0 one-warp supernode (in a group task), 1 whole-supernode task, 2 block tasks.
static void order_forward_by_path(const Plan &P, const std::vector<int> &kinds, std::vector<int> &tasks) {
  constexpr int B = 64;
  constexpr double cDiag = 2.7, cBelow = 3.0, cWhole = 7.0, cSmall = 5.0;  // estimated task times (microseconds)
  const int ns = (int)P.snNc.size(), nt = (int)(tasks.size() / 4);
  auto span = [&](int s) {  // from s's children complete to s's pass-up vector complete
    if (kinds[s] == 0) return cSmall;
    if (kinds[s] == 1) return cWhole;
    return ((P.snNc[s] + B - 1) / B) * cDiag + (P.snM[s] > P.snNc[s] ? cBelow : 0.0);
  };
  std::vector<double> tail(ns, 0.0);  // from s's pass-up vector complete to the end of the sweep
  for (int L = P.nlevels - 1; L >= 0; L--)
    for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
      const int s = P.lvlSn[q], par = P.snParent[s];
      tail[s] = par < 0 ? 0.0 : span(par) + tail[par];
    }
  // nodes: tasks [0, nt), "s complete" [nt, nt + ns), "s ready" (children complete) [nt + ns, nt + 2 ns)
  const int nn = nt + 2 * ns;
  std::vector<std::vector<int>> succ(nn);
  std::vector<int> indeg(nn, 0);
  std::vector<double> prio(nt, 0.0);
  auto edge = [&](int a, int b) {
    succ[a].push_back(b);
    indeg[b]++;
  };
  std::vector<int> diagAt(P.nflags, -1), lastDiag(ns, -1);
  for (int t = 0; t < nt; t++) {
    const int x = tasks[4 * t], y = tasks[4 * t + 1], k = tasks[4 * t + 2];
    if (k == 0) {
      diagAt[P.blkOff[x] + y] = t;
      if (y == P.blkOff[x + 1] - P.blkOff[x] - 1) lastDiag[x] = t;
    }
  }
  for (int t = 0; t < nt; t++) {
    const int x = tasks[4 * t], y = tasks[4 * t + 1], k = tasks[4 * t + 2];
    if (k == 2) {  // one-warp supernodes P.solveSmall[x .. x + y)
      for (int i = x; i < x + y; i++) {
        const int s = P.solveSmall[i];
        edge(nt + ns + s, t);
        edge(t, nt + s);
        prio[t] = std::max(prio[t], cSmall + tail[s]);
      }
    } else if (k == 3) {
      edge(nt + ns + x, t);
      edge(t, nt + x);
      prio[t] = cWhole + tail[x];
    } else if (k == 0) {
      const int nb = P.blkOff[x + 1] - P.blkOff[x];
      edge(y == 0 ? nt + ns + x : diagAt[P.blkOff[x] + y - 1], t);
      prio[t] = (nb - y) * cDiag + (P.snM[x] > P.snNc[x] ? cBelow : 0.0) + tail[x];
    } else {
      edge(lastDiag[x], t);
      edge(t, nt + x);
      prio[t] = cBelow + tail[x];
    }
  }
  for (int s = 0; s < ns; s++)
    if (P.snParent[s] >= 0) edge(nt + s, nt + ns + P.snParent[s]);
  // Kahn's algorithm: virtual nodes pass through at once, tasks leave the heap by priority
  std::vector<std::pair<double, int>> heap;  // (priority, -index)
  auto cmp = [](const std::pair<double, int> &a, const std::pair<double, int> &b) { return a < b; };
  std::vector<int> stack;
  auto release = [&](int v) {
    if (v < nt) {
      heap.push_back({prio[v], -v});
      std::push_heap(heap.begin(), heap.end(), cmp);
    } else {
      stack.push_back(v);
    }
  };
  auto drain = [&]() {
    while (!stack.empty()) {
      const int v = stack.back();
      stack.pop_back();
      for (int w : succ[v])
        if (--indeg[w] == 0) release(w);
    }
  };
  for (int v = 0; v < nn; v++)
    if (indeg[v] == 0) release(v);
  drain();
  std::vector<int> out;
  out.reserve(tasks.size());
  while (!heap.empty()) {
    std::pop_heap(heap.begin(), heap.end(), cmp);
    const int t = -heap.back().second;
    heap.pop_back();
    out.insert(out.end(), tasks.begin() + 4 * (size_t)t, tasks.begin() + 4 * (size_t)t + 4);
    for (int w : succ[t])
      if (--indeg[w] == 0) release(w);
    drain();
  }
  if (out.size() != tasks.size()) throw std::logic_error("forward task order: the dependency graph has a cycle");
  tasks.swap(out);
}

// The backward task list in critical-path order, as the forward one: a topological order (a supernode's tasks after
// all of its parent's, its diagonal blocks from the last down) listing first, among the tasks whose predecessors are
// listed, the one with the longest estimated path to the end of the sweep (its remaining blocks, then the longest
// chain of descendants below it). small(s): a one-warp supernode (in a group task).
static void order_backward_by_path(const Plan &P, const std::vector<char> &small, std::vector<int> &tasks) {
  constexpr double cDiag = 2.7, cSmall = 5.0;  // estimated task times (microseconds)
  const int ns = (int)P.snNc.size(), nt = (int)(tasks.size() / 4);
  auto span = [&](int s) { return small[s] ? cSmall : (P.blkOff[s + 1] - P.blkOff[s]) * cDiag; };
  std::vector<double> tail(ns, 0.0);  // from s's solution complete to the end of the sweep (its descendants)
  for (int L = 0; L < P.nlevels; L++)
    for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
      const int s = P.lvlSn[q], par = P.snParent[s];
      if (par >= 0) tail[par] = std::max(tail[par], span(s) + tail[s]);
    }
  // nodes: tasks [0, nt), "s solved" [nt, nt + ns)
  const int nn = nt + ns;
  std::vector<std::vector<int>> succ(nn);
  std::vector<int> indeg(nn, 0);
  std::vector<double> prio(nt, 0.0);
  auto edge = [&](int a, int b) {
    succ[a].push_back(b);
    indeg[b]++;
  };
  std::vector<int> blkAt(P.nflags, -1);
  for (int t = 0; t < nt; t++)
    if (tasks[4 * t + 2] == 0) blkAt[P.blkOff[tasks[4 * t]] + tasks[4 * t + 1]] = t;
  for (int t = 0; t < nt; t++) {
    const int x = tasks[4 * t], y = tasks[4 * t + 1], k = tasks[4 * t + 2];
    if (k == 2) {  // one-warp supernodes P.solveSmall[x .. x + y)
      for (int i = x; i < x + y; i++) {
        const int s = P.solveSmall[i];
        if (P.snParent[s] >= 0) edge(nt + P.snParent[s], t);
        edge(t, nt + s);
        prio[t] = std::max(prio[t], cSmall + tail[s]);
      }
    } else {
      const int nb = P.blkOff[x + 1] - P.blkOff[x];
      if (y == nb - 1) {
        if (P.snParent[x] >= 0) edge(nt + P.snParent[x], t);
      } else {
        edge(blkAt[P.blkOff[x] + y + 1], t);
      }
      if (y == 0) edge(t, nt + x);
      prio[t] = (y + 1) * cDiag + tail[x];
    }
  }
  std::vector<std::pair<double, int>> heap;  // (priority, -index)
  std::vector<int> stack;
  auto release = [&](int v) {
    if (v < nt) {
      heap.push_back({prio[v], -v});
      std::push_heap(heap.begin(), heap.end());
    } else {
      stack.push_back(v);
    }
  };
  auto drain = [&]() {
    while (!stack.empty()) {
      const int v = stack.back();
      stack.pop_back();
      for (int w : succ[v])
        if (--indeg[w] == 0) release(w);
    }
  };
  for (int v = 0; v < nn; v++)
    if (indeg[v] == 0) release(v);
  drain();
  std::vector<int> out;
  out.reserve(tasks.size());
  while (!heap.empty()) {
    std::pop_heap(heap.begin(), heap.end());
    const int t = -heap.back().second;
    heap.pop_back();
    out.insert(out.end(), tasks.begin() + 4 * (size_t)t, tasks.begin() + 4 * (size_t)t + 4);
    for (int w : succ[t])
      if (--indeg[w] == 0) release(w);
    drain();
  }
  if (out.size() != tasks.size()) throw std::logic_error("backward task order: the dependency graph has a cycle");
  tasks.swap(out);
}

void build_plan(const Symbolic &S, Plan &P, const Tuning &tune) {
  P = Plan();
  if (tune.groupBlocks < 1 || tune.groupBlocks > 16 || tune.smallCut < kTinyFront || tune.smallCut > kSmallFront ||
      tune.deferB < 1 || tune.deferB > 8)
    throw std::invalid_argument(
        "schedule parameters out of range (group blocks 1..16, small fronts 32..128, deferred updates 1..8)");
  P.tune = tune;
  const int GW = tune.groupBlocks * kPanel;  // group width
  const int n = S.n, ns = S.nsuper;
  P.n = n;
  P.nsuper = ns;
  P.maxFront = S.maxFront;
  P.nnzLStored = S.nnzLStored;
  P.nnzA = S.nnzA;
  P.patNnz = S.patNnz;
  P.flops = S.flops;
  P.perm = S.perm;
  P.Sp = S.Sp;
  P.Si = S.Si;
  if (ns == 0) {
    P.lvlPtr.assign(1, 0);
    P.asmLvlPtr.assign(1, 0);
    P.lvlStepPtr.assign(1, 0);
    P.asmPtr.assign(1, 0);
    return;
  }
  P.snF.resize(ns);
  P.snNc.resize(ns);
  P.snM.resize(ns);
  P.snLevel.assign(ns, 0);
  P.snParent = S.superParent;
  P.snLxp.assign(S.Lxp.begin(), S.Lxp.begin() + ns);
  P.snUoff.assign(ns, -1);
  for (int s = 0; s < ns; s++) {
    P.snF[s] = S.superStart[s];
    P.snNc[s] = S.superStart[s + 1] - S.superStart[s];
    P.snM[s] = S.Sp[s + 1] - S.Sp[s];
  }
  // height levels: children always have a smaller index (postorder)
  for (int s = 0; s < ns; s++)
    if (S.superParent[s] >= 0) P.snLevel[S.superParent[s]] = std::max(P.snLevel[S.superParent[s]], P.snLevel[s] + 1);
  P.nlevels = 1 + *std::max_element(P.snLevel.begin(), P.snLevel.end());
  P.lvlPtr.assign(P.nlevels + 1, 0);
  for (int s = 0; s < ns; s++) P.lvlPtr[P.snLevel[s] + 1]++;
  for (int L = 0; L < P.nlevels; L++) P.lvlPtr[L + 1] += P.lvlPtr[L];
  P.lvlSn.resize(ns);
  {
    std::vector<int> fill(P.lvlPtr.begin(), P.lvlPtr.end() - 1);
    for (int s = 0; s < ns; s++) P.lvlSn[fill[P.snLevel[s]]++] = s;
  }
  // children in the reference's order (childHead: decreasing index)
  P.chPtr.assign(ns + 1, 0);
  for (int s = 0; s < ns; s++)
    for (int c = S.childHead[s]; c != -1; c = S.childNext[c]) P.chPtr[s + 1]++;
  for (int s = 0; s < ns; s++) P.chPtr[s + 1] += P.chPtr[s];
  P.chList.resize(P.chPtr[ns]);
  for (int s = 0; s < ns; s++) {
    int q = P.chPtr[s];
    for (int c = S.childHead[s]; c != -1; c = S.childNext[c]) P.chList[q++] = c;
  }
  // assembly and extend-add maps
  std::vector<int> rel(n, -1);
  P.asmPtr.assign(ns + 1, 0);
  P.asmDst.resize(S.nnzA);
  P.asmSrc.resize(S.nnzA);
  P.asmColPtr = S.lowerP;
  P.eaPtr.assign(ns + 1, 0);
  for (int s = 0; s < ns; s++) P.eaPtr[s + 1] = P.eaPtr[s] + (P.snParent[s] >= 0 ? P.snM[s] - P.snNc[s] : 0);
  P.eaMap.resize(P.eaPtr[ns]);
  for (int s = 0; s < ns; s++) {
    const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s], r0 = S.Sp[s];
    for (int r = 0; r < m; r++) rel[S.Si[r0 + r]] = r;
    P.asmPtr[s] = S.lowerP[f];
    for (int c = 0; c < nc; c++)
      for (int p = S.lowerP[f + c]; p < S.lowerP[f + c + 1]; p++) {
        P.asmDst[p] = rel[S.lowerI[p]] + c * m;
        P.asmSrc[p] = S.lowerSrc[p];
      }
    for (int q = P.chPtr[s]; q < P.chPtr[s + 1]; q++) {
      int c = P.chList[q];
      int cr0 = S.Sp[c] + P.snNc[c], mu = P.snM[c] - P.snNc[c];
      for (int a = 0; a < mu; a++) P.eaMap[P.eaPtr[c] + a] = rel[S.Si[cr0 + a]];
    }
  }
  P.asmPtr[ns] = S.lowerP[n];
  // U arena by level lifetimes
  {
    ArenaPlanner ar;
    for (int L = 0; L < P.nlevels; L++) {
      for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
        int s = P.lvlSn[q];
        int64_t mu = P.snM[s] - P.snNc[s];
        if (mu > 0) P.snUoff[s] = ar.alloc(mu * mu);
      }
      ar.note();
      for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
        int s = P.lvlSn[q];
        for (int k = P.chPtr[s]; k < P.chPtr[s + 1]; k++) {
          int c = P.chList[k];
          if (P.snUoff[c] >= 0) ar.release(P.snUoff[c]);
        }
      }
    }
    P.arenaDoubles = ar.peak();
  }
  // BF16 split storage of the pivot columns (mixed precision): ld = round_up(m, 8), 16-byte aligned columns
  P.snSp.assign(ns + 1, 0);
  for (int s = 0; s < ns; s++) P.snSp[s + 1] = P.snSp[s] + (int64_t)((P.snM[s] + 7) & ~7) * P.snNc[s];
  P.splitElems = P.snSp[ns];
  // mixed-precision tiles (128 x 256, starts aligned down to 8, masked by ilo / jlo / jend) of a region
  auto emitMix = [&](std::vector<MixTask> &out, int s, int rlo, int clo, int chi, int kc0, int kw, int width = 256) {
    const int m = P.snM[s], nc = P.snNc[s];
    for (int j0 = clo & ~7; j0 < chi; j0 += width)
      for (int i0 = std::max(rlo, j0) & ~7; i0 < m; i0 += 128)
        out.push_back({(long long)P.snLxp[s], (long long)P.snUoff[s], (long long)P.snSp[s], m, nc, (m + 7) & ~7, kc0,
                       kw, i0, j0, rlo, clo, chi, s});
  };
  P.mixULvlPtr.assign(1, 0);
  // task lists per level
  P.asmLvlPtr.assign(P.nlevels + 1, 0);
  P.asmLvlBytes.assign(P.nlevels, 0.0);
  P.uLvlPtr.assign(1, 0);
  P.lvlStepPtr.assign(P.nlevels + 1, 0);
  P.tinyPtr.assign(1, 0);
  P.tinyMid.clear();
  P.smallPtr.assign(1, 0);
  auto isSmall = [&](int s) { return P.snM[s] <= tune.smallCut; };
  std::vector<int> appliedB(ns, 0);  // per front: pivot columns whose update every column beyond the next group has
  for (int L = 0; L < P.nlevels; L++) {
    // small fronts: the whole front in one kernel; the rest go through the steps below
    int maxM = 0;
    double ff = 0, fb = 0;
    for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
      const int s = P.lvlSn[q];
      if (!isSmall(s)) continue;
      const double m = P.snM[s], nc = P.snNc[s], mu = m - nc;
      ff += nc * nc * nc / 3.0 + nc * nc * mu + nc * mu * mu;
      fb += 16.0 * (S.lowerP[P.snF[s] + P.snNc[s]] - S.lowerP[P.snF[s]]) + 8.0 * (m * nc + mu * (mu + 1) / 2);
      for (int k = P.chPtr[s]; k < P.chPtr[s + 1]; k++) {
        const double muc = P.snM[P.chList[k]] - P.snNc[P.chList[k]];
        fb += 8.0 * muc * (muc + 1) / 2;
      }
      if (P.snM[s] <= kTinyFront) {
        P.tinySn.push_back(s);
      } else {
        P.smallSn.push_back(s);
        maxM = std::max(maxM, P.snM[s]);
      }
    }
    {
      auto t0 = P.tinySn.begin() + P.tinyPtr.back();
      std::stable_sort(t0, P.tinySn.end(), [&](int a, int b) { return P.snM[a] < P.snM[b]; });
      P.tinyMid.push_back(std::partition_point(t0, P.tinySn.end(), [&](int a) { return P.snM[a] <= kTinyMid; }) -
                          P.tinySn.begin());
    }
    P.tinyPtr.push_back((int64_t)P.tinySn.size());
    P.smallPtr.push_back((int64_t)P.smallSn.size());
    P.smallMaxM.push_back(maxM);
    P.frontLvlFlops.push_back(ff);
    P.frontLvlBytes.push_back(fb);
    int maxSteps = 0;
    for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
      int s = P.lvlSn[q];
      if (isSmall(s)) continue;
      for (int j0 = 0; j0 < P.snM[s]; j0 += kAsmCols) add_asm_task(P, s, j0, P.asmTasks, P.asmCh);
      maxSteps = std::max(maxSteps, (P.snNc[s] + GW - 1) / (GW));
      // bytes: value + lowerI + lowerSrc per A entry (16); read U + read/write the parent entry per child entry (24)
      double b = 16.0 * (S.lowerP[P.snF[s] + P.snNc[s]] - S.lowerP[P.snF[s]]);
      for (int k = P.chPtr[s]; k < P.chPtr[s + 1]; k++) {
        double mu = P.snM[P.chList[k]] - P.snNc[P.chList[k]];
        b += 24.0 * mu * (mu + 1) / 2;
      }
      P.asmLvlBytes[L] += b;
    }
    P.asmLvlPtr[L + 1] = (int64_t)P.asmTasks.size();
    const int defer = std::max(1, tune.deferB);
    for (int k = 0; k < maxSteps; k++) {
      const bool doB = (k + 1) % defer == 0;  // part B at this step (every deferB steps)
      StepRange sr;
      sr.panelFlops = sr.updateFlopsA = sr.updateFlopsB = 0;
      sr.item0 = (int64_t)P.groupItems.size();
      sr.strip0 = (int64_t)P.strips.size();
      sr.ticket = P.nGroupTickets++;
      // Group k of every front of the level (pivot columns [g0, g1), up to kGroup pivot blocks) in one group-panel
      // launch; then the columns right of the group receive the updates of the groups since the last part B
      // (K = [appliedB, g1), the group alone when deferB = 1): part A the next group's columns, part B the rest.
      struct Region {
        int s, lo, hi, kc0, kw;
      };
      std::vector<Region> regions;
      // lower entries of columns [a, b) of an m-row front
      auto trap = [](double m, double a, double b) { return (b - a) * m - (a + b - 1) * (b - a) / 2; };
      for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
        int s = P.lvlSn[q];
        const int nc = P.snNc[s], m = P.snM[s], g0 = k * GW;
        if (g0 >= nc || isSmall(s)) continue;
        const int g1 = std::min(g0 + GW, nc), nb = (g1 - g0 + kPanel - 1) / kPanel;
        P.groupItems.push_back({s, g0, g1, P.nGroupFlags});
        P.nGroupFlags += 2 * nb;
        for (int c0 = g0; c0 < g1; c0 += kPanel) {
          const double w = std::min(kPanel, g1 - c0), c1 = c0 + w;
          sr.panelFlops += w * w * w / 3.0 + (m - c1) * w * w + 2.0 * w * trap(m, c1, g1);
        }
        if (g1 < nc) regions.push_back({s, g1, nc, appliedB[s], g1 - appliedB[s]});
      }
      const int64_t i0 = sr.item0, i1 = (int64_t)P.groupItems.size();
      for (int64_t it = i0; it < i1; it++) {  // the diagonal strips of every item first (they take the first tickets)
        const GroupItem &gi = P.groupItems[it];
        for (int c0 = gi.g0, j = 0; c0 < gi.g1; c0 += kPanel, j++)
          P.strips.push_back({(int)it, c0, std::min(c0 + kPanel, gi.g1), j});
      }
      for (int64_t it = i0; it < i1; it++) {  // then the strips below the groups
        const GroupItem &gi = P.groupItems[it];
        const int m = P.snM[gi.s];
        for (int r0 = gi.g1; r0 < m; r0 += kPanel) P.strips.push_back({(int)it, r0, std::min(r0 + kPanel, m), -1});
      }
      sr.item1 = i1;
      sr.strip1 = (int64_t)P.strips.size();
      // part A (the next group's columns, which start on a group boundary) runs tiles as wide as the group when
      // it is 64 or 128 columns: no masked part of a 128 x 256 tile
      sr.mixWidthA = GW <= 128 ? GW : 256;
      auto emit = [&](const Region &g, int lo, int hi, double &flops, int width) {
        if (lo >= hi) return;
        const int m = P.snM[g.s], nc = P.snNc[g.s];
        flops += 2.0 * g.kw * trap(m, lo, hi);
        emitMix(P.mixTiles, g.s, lo, lo, hi, g.kc0, g.kw, width);
        for (int j0 = lo; j0 < hi; j0 += kTile)
          for (int i0 = lo + ((j0 - lo) / kTileM) * kTileM; i0 < m; i0 += kTileM)
            P.tileTasks.push_back({(long long)P.snLxp[g.s], (long long)P.snUoff[g.s], m, nc, g.kc0, g.kw, i0, j0, hi, 0});
      };
      sr.tile0 = (int64_t)P.tileTasks.size();
      sr.mix0 = (int64_t)P.mixTiles.size();
      for (const Region &g : regions) emit(g, g.lo, std::min(g.lo + GW, g.hi), sr.updateFlopsA, sr.mixWidthA);
      sr.tileMid = (int64_t)P.tileTasks.size();
      sr.mixMid = (int64_t)P.mixTiles.size();
      if (doB)
        for (const Region &g : regions) {
          emit(g, g.lo + GW, g.hi, sr.updateFlopsB, 256);
          appliedB[g.s] = g.lo;  // every column right of the next group now has the groups before g.lo
        }
      sr.tile1 = (int64_t)P.tileTasks.size();
      sr.mix1 = (int64_t)P.mixTiles.size();
      P.steps.push_back(sr);
    }
    P.lvlStepPtr[L + 1] = (int)P.steps.size();
    // update blocks of the level's fronts: one long-K pass each
    double uf = 0;
    for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
      int s = P.lvlSn[q];
      const int nc = P.snNc[s], m = P.snM[s];
      if (m <= nc || isSmall(s)) continue;
      const double mu = m - nc;
      uf += (double)nc * mu * (mu + 1);
      for (int j0 = nc; j0 < m; j0 += kTile)
        for (int i0 = nc + ((j0 - nc) / kTileM) * kTileM; i0 < m; i0 += kTileM)
          P.uTasks.push_back({(long long)P.snLxp[s], (long long)P.snUoff[s], m, nc, 0, nc, i0, j0, m, 0});
      emitMix(P.mixUTasks, s, nc, nc, m, 0, nc);
    }
    P.mixULvlPtr.push_back((int64_t)P.mixUTasks.size());
    P.uLvlPtr.push_back((int64_t)P.uTasks.size());
    P.uLvlFlops.push_back(uf);
  }
  // forward-solve update vectors
  P.snTOff.assign(ns + 1, 0);
  for (int s = 0; s < ns; s++) P.snTOff[s + 1] = P.snTOff[s] + (P.snM[s] - P.snNc[s]);
  P.solveBufDoubles = P.snTOff[ns];
  // solve block tasks per level (each task only waits for tasks listed before it)
  constexpr int B = 64;
  P.blkOff.assign(ns + 1, 0);
  for (int s = 0; s < ns; s++) P.blkOff[s + 1] = P.blkOff[s] + (P.snNc[s] + B - 1) / B;
  P.nflags = P.blkOff[ns];
  P.rowBlk.assign(S.n, 0);
  for (int s = 0; s < ns; s++)
    for (int c = 0; c < P.snNc[s]; c++) P.rowBlk[P.snF[s] + c] = P.blkOff[s] + c / B;
  P.diagSlot.clear();
  for (int j = 0; j < S.n; j++)
    for (int p = S.lowerP[j]; p < S.lowerP[j + 1]; p++)
      if (S.lowerI[p] == j) P.diagSlot.push_back(S.lowerSrc[p]);
  P.invOff.assign(P.nflags + 1, 0);
  for (int s = 0; s < ns; s++)
    for (int b = 0; b * B < P.snNc[s]; b++) {
      const int64_t w = std::min(B, P.snNc[s] - b * B);
      P.invOff[P.blkOff[s] + b + 1] = P.invOff[P.blkOff[s] + b] + w * w;
    }
  P.fwdLvlPtr.assign(P.nlevels + 1, 0);
  P.bwdLvlPtr.assign(P.nlevels + 1, 0);
  auto push = [](std::vector<int> &v, int a, int b, int c) {
    v.push_back(a);
    v.push_back(b);
    v.push_back(c);
    v.push_back(0);
  };
  for (int s = 0; s < ns; s++)
    for (int b = 0; P.snNc[s] > B && b * B < P.snNc[s]; b++) {
      P.chainTasks.push_back(s);
      P.chainTasks.push_back(b);
    }
  // Supernodes with m <= kTinyFront are solved whole by one warp: tasks {first, count, 2} over solveSmall, up to
  // kSolveGroup supernodes of one level per task, listed before the level's block tasks.
  auto solveSmall = [&](int s) { return P.snM[s] <= kTinyFront; };
  auto whole = [&](int s) { return !solveSmall(s) && P.snNc[s] <= B && P.snM[s] <= kWholeFront; };
  P.fwdTasks1.clear();
  for (int s = 0; s < ns; s++)
    if (!solveSmall(s))
      for (int b = P.blkOff[s]; b < P.blkOff[s + 1]; b++) P.invBlocks.push_back(b);
  for (int L = 0; L < P.nlevels; L++) {
    const int64_t g0 = (int64_t)P.solveSmall.size();
    for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++)
      if (solveSmall(P.lvlSn[q])) P.solveSmall.push_back(P.lvlSn[q]);
    const int64_t g1 = (int64_t)P.solveSmall.size();
    for (int64_t g = g0; g < g1; g += kSolveGroup) {
      push(P.fwdTasks, (int)g, (int)std::min<int64_t>(kSolveGroup, g1 - g), 2);
      push(P.fwdTasks1, (int)g, (int)std::min<int64_t>(kSolveGroup, g1 - g), 2);
      push(P.bwdTasks, (int)g, (int)std::min<int64_t>(kSolveGroup, g1 - g), 2);
    }
    // one-vector forward: a supernode with one pivot block and m <= kWholeFront is one task (kind 3) doing its
    // diagonal block and all of its rows below
    for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++)
      if (whole(P.lvlSn[q])) push(P.fwdTasks1, P.lvlSn[q], 0, 3);
    int maxNb = 0;
    for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++)
      if (!solveSmall(P.lvlSn[q])) maxNb = std::max(maxNb, (P.snNc[P.lvlSn[q]] + B - 1) / B);
    for (int blk = 0; blk < maxNb; blk++)
      for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
        int s = P.lvlSn[q];
        if (!solveSmall(s) && blk < (P.snNc[s] + B - 1) / B) {
          push(P.fwdTasks, s, blk, 0);
          if (!whole(s)) push(P.fwdTasks1, s, blk, 0);
        }
      }
    for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
      int s = P.lvlSn[q], mu = P.snM[s] - P.snNc[s];
      if (solveSmall(s)) continue;
      for (int j = 0; j * B < mu; j++) {
        push(P.fwdTasks, s, j, 1);
        if (!whole(s)) push(P.fwdTasks1, s, j, 1);
      }
    }
    P.fwdLvlPtr[L + 1] = (int)(P.fwdTasks.size() / 4);
    for (int d = 0; d < maxNb; d++)
      for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
        int s = P.lvlSn[q], nb = (P.snNc[s] + B - 1) / B;
        if (!solveSmall(s) && d < nb) push(P.bwdTasks, s, nb - 1 - d, 0);
      }
    P.bwdLvlPtr[L + 1] = (int)(P.bwdTasks.size() / 4);
  }
  {
    std::vector<int> kinds(ns);
    for (int s = 0; s < ns; s++) kinds[s] = solveSmall(s) ? 0 : whole(s) ? 1 : 2;
    order_forward_by_path(P, kinds, P.fwdTasks1);
  }
  // the whole backward sweep in one launch: levels top-down, then in critical-path order
  P.bwdAll.clear();
  for (int L = P.nlevels - 1; L >= 0; L--)
    P.bwdAll.insert(P.bwdAll.end(), P.bwdTasks.begin() + 4 * (size_t)P.bwdLvlPtr[L],
                    P.bwdTasks.begin() + 4 * (size_t)P.bwdLvlPtr[L + 1]);
  {
    std::vector<char> small(ns);
    for (int s = 0; s < ns; s++) small[s] = solveSmall(s);
    order_backward_by_path(P, small, P.bwdAll);
  }
}

void build_dense_all(const Plan &P, DenseSched &D) {
  D = DenseSched();
  const int GW = P.tune.groupBlocks * kPanel;  // group width
  D.asmLvlPtr.assign(P.nlevels + 1, 0);
  D.lvlStepPtr.assign(P.nlevels + 1, 0);
  D.uLvlPtr.assign(1, 0);
  auto trap = [](double m, double a, double b) { return (b - a) * m - (a + b - 1) * (b - a) / 2; };
  for (int L = 0; L < P.nlevels; L++) {
    int maxSteps = 0;
    for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
      const int s = P.lvlSn[q];
      for (int j0 = 0; j0 < P.snM[s]; j0 += kAsmCols) add_asm_task(P, s, j0, D.asmTasks, D.asmCh);
      maxSteps = std::max(maxSteps, (P.snNc[s] + GW - 1) / (GW));
    }
    D.asmLvlPtr[L + 1] = (int64_t)D.asmTasks.size();
    for (int k = 0; k < maxSteps; k++) {
      StepRange sr{};
      sr.item0 = (int64_t)D.groupItems.size();
      sr.strip0 = (int64_t)D.strips.size();
      sr.ticket = D.nGroupTickets++;
      struct Region {
        int s, lo, hi, kc0, kw;
      };
      std::vector<Region> regions;
      for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
        const int s = P.lvlSn[q], nc = P.snNc[s], m = P.snM[s], g0 = k * GW;
        if (g0 >= nc) continue;
        const int g1 = std::min(g0 + GW, nc), nb = (g1 - g0 + kPanel - 1) / kPanel;
        D.groupItems.push_back({s, g0, g1, D.nGroupFlags});
        D.nGroupFlags += 2 * nb;
        for (int c0 = g0; c0 < g1; c0 += kPanel) {
          const double w = std::min(kPanel, g1 - c0), c1 = c0 + w;
          sr.panelFlops += w * w * w / 3.0 + (m - c1) * w * w + 2.0 * w * trap(m, c1, g1);
        }
        if (g1 < nc) regions.push_back({s, g1, nc, g0, g1 - g0});
      }
      const int64_t i0 = sr.item0, i1 = (int64_t)D.groupItems.size();
      for (int64_t it = i0; it < i1; it++) {  // the diagonal strips of every item take the first tickets
        const GroupItem &gi = D.groupItems[it];
        for (int c0 = gi.g0, j = 0; c0 < gi.g1; c0 += kPanel, j++)
          D.strips.push_back({(int)it, c0, std::min(c0 + kPanel, gi.g1), j});
      }
      for (int64_t it = i0; it < i1; it++) {
        const GroupItem &gi = D.groupItems[it];
        const int m = P.snM[gi.s];
        for (int r0 = gi.g1; r0 < m; r0 += kPanel) D.strips.push_back({(int)it, r0, std::min(r0 + kPanel, m), -1});
      }
      sr.item1 = i1;
      sr.strip1 = (int64_t)D.strips.size();
      auto emit = [&](const Region &g, int lo, int hi, double &flops) {
        if (lo >= hi) return;
        const int m = P.snM[g.s], nc = P.snNc[g.s];
        flops += 2.0 * g.kw * trap(m, lo, hi);
        for (int j0 = lo; j0 < hi; j0 += kTile)
          for (int i0 = lo + ((j0 - lo) / kTileM) * kTileM; i0 < m; i0 += kTileM)
            D.tileTasks.push_back({(long long)P.snLxp[g.s], (long long)P.snUoff[g.s], m, nc, g.kc0, g.kw, i0, j0, hi, 0});
      };
      sr.tile0 = (int64_t)D.tileTasks.size();
      for (const Region &g : regions) emit(g, g.lo, std::min(g.lo + GW, g.hi), sr.updateFlopsA);
      sr.tileMid = (int64_t)D.tileTasks.size();
      for (const Region &g : regions) emit(g, g.lo + GW, g.hi, sr.updateFlopsB);
      sr.tile1 = (int64_t)D.tileTasks.size();
      D.steps.push_back(sr);
    }
    D.lvlStepPtr[L + 1] = (int)D.steps.size();
    for (int q = P.lvlPtr[L]; q < P.lvlPtr[L + 1]; q++) {
      const int s = P.lvlSn[q], nc = P.snNc[s], m = P.snM[s];
      if (m <= nc) continue;
      for (int j0 = nc; j0 < m; j0 += kTile)
        for (int i0 = nc + ((j0 - nc) / kTileM) * kTileM; i0 < m; i0 += kTileM)
          D.uTasks.push_back({(long long)P.snLxp[s], (long long)P.snUoff[s], m, nc, 0, nc, i0, j0, m, 0});
    }
    D.uLvlPtr.push_back((int64_t)D.uTasks.size());
  }
}

}  // namespace amp
