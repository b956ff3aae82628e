// Device schedule of one symbolic structure: everything the numeric factor and the solves need on the GPU, computed
// once per pattern on the host (the analogue of the reference's reusable `sym`, sparse.mjs:666-902).
//
// Layout in HBM:
//   Lx       the factor, exactly the reference's layout: supernode s is an m x nc column-major block at Lxp[s]
//            (rows Si[Sp[s] ..], ld = m). The first nc columns of every frontal matrix live here in place, so no copy
//            of the factor out of the front is ever made.
//   U arena  the trailing mu x mu block (mu = m - nc, column-major, ld = mu, lower part used) of every front: the
//            update (contribution) matrix. Offsets are assigned offline by level lifetimes (allocated at the
//            supernode's level, released after its parent's level has assembled it).
// Front entry (i, j), i >= j, of supernode s is Lx[Lxp[s] + j m + i] for j < nc, else U[Uoff[s] + (j-nc) mu + (i-nc)].
#pragma once
#include <cstdint>
#include <vector>

#include "symbolic.hpp"

namespace amp {

constexpr int kPanel = 64;     // pivot block width of the dense partial factorization
constexpr int kGroup = 4;      // pivot blocks whose update of the columns right of them is applied together
constexpr int kTile = 64;      // trailing-update tile columns
constexpr int kTileM = 128;    // trailing-update tile rows
constexpr int kAsmCols = 8;    // front columns per assembly task (one per warp)
constexpr int kTrsmRows = 64;  // panel rows per TRSM task
constexpr int kTinyFront = 32;    // fronts with m <= 32: one warp per front does the whole front (front_small.cu)
constexpr int kTinyMid = 16;      // the smaller tiny class (m <= 16: 16 x 16 tiles, eight fronts per CTA)
constexpr int kSmallFront = 128;  // fronts with 32 < m <= 128: one CTA per front does the whole front
constexpr int kSolveGroup = 4;    // supernodes with m <= kTinyFront per solve task (one warp each)
constexpr int kWholeFront = 512;  // one-vector forward: supernodes with nc <= 64 and m <= 512 are one task each

struct GroupItem {  // pivot columns [g0, g1) (up to kGroup pivot blocks) of supernode s, factored by one group-panel
                    // launch; its flags start at flag0: one POTRF flag per pivot block, then one TRSM counter per
                    // diagonal strip
  int s, g0, g1, flag0;
};
struct StripTask {  // rows [r0, r1) of the item's front; diag >= 0: the rows of the item's pivot block `diag`
  int item, r0, r1, diag;
};
struct TileTask {  // update tile: rows [i0, i0+128) x cols [j0, min(j0+64, jend)) of a front, K = columns [c0, c0+w)
  long long lp, up;      // offsets of the front's L panel (Lx) and update block (U arena, -1 if none)
  int m, nc, c0, w, i0, j0, jend, pad;
};
struct MixTask {  // mixed-precision update tile (128 x 256, 8-aligned start) of a front with FP32 storage
  long long lp, up, sp;      // FP32 L panel, FP32 update block (-1 if none), BF16 split columns (ld per front)
  int m, nc, ld, c0, w;      // K = pivot columns [c0, c0 + w)
  int i0, j0;                // tile origin (multiples of 8)
  int ilo, jlo, jend;        // rows >= ilo, columns in [jlo, jend) are updated
  int s;                     // supernode (selects the front's TMA descriptors of the split columns)
};
struct AsmTask {  // zero + assemble + extend-add front columns [j0, j0 + kAsmCols) of supernode s; the update-matrix
                  // columns [b0, b1) of each child that map into them (static) are asmCh[ch0 + q], q in child order
  int s, j0, ch0;
};
struct ChildRange {
  int b0, b1;
};

// One group step of a level: the group-panel launch over its items (the level's fronts with a group at this index),
// then the update of the columns right of each group with K = the group: part A = the next group's columns (on the
// factor's stream: the next group panel reads them), part B = the rest (side stream, overlapping the next panel).
struct StepRange {
  int64_t item0, item1, strip0, strip1;  // group items and strip tasks of the panel launch
  int ticket;                            // the launch's ticket counter (index into the group tickets)
  int64_t tile0, tileMid, tile1;  // FP64 update tiles: part A [tile0, tileMid), part B [tileMid, tile1)
  int64_t mix0, mixMid, mix1;     // the same for the mixed-precision tiles
  int mixWidthA;                  // columns of part A's mixed tiles: the group width when it is 64 or 128, else 256
  double panelFlops, updateFlopsA, updateFlopsB;  // algorithmic flops of the step's launches
};
// The update block of every front receives its whole Schur update once, after the group steps of its level:
// U -= L21 L21^T with K = nc (tiles over the lower triangle of [nc, m)^2).

// The dense path for every front, small ones included (the complex-symmetric factor, which has no whole-front
// kernels): assembly tasks, group steps and FP64-layout update tiles per level, with the same meaning as the main
// schedule's fields of Plan.
struct DenseSched {
  std::vector<AsmTask> asmTasks;
  std::vector<ChildRange> asmCh;
  std::vector<int64_t> asmLvlPtr;
  std::vector<GroupItem> groupItems;
  std::vector<StripTask> strips;
  int nGroupFlags = 0, nGroupTickets = 0;
  std::vector<StepRange> steps;
  std::vector<int> lvlStepPtr;
  std::vector<TileTask> tileTasks, uTasks;
  std::vector<int64_t> uLvlPtr;
};

// Tunable schedule parameters (the autotuner's search space, amp_plan_autotune): pivot blocks per group (the width
// of a group panel and the K of the group's update: 64 x groupBlocks columns) and the largest front factored whole
// by one CTA (the small-front kernel; larger fronts take the group path).
struct Tuning {
  int groupBlocks = kGroup;
  int smallCut = kSmallFront;
  // The update of the columns beyond the next group (part B) is applied every deferB group steps, with K = the
  // groups since the last one (the next group's columns still receive every group's update at once, part A): larger
  // K per pass over the trailing matrix, fewer passes. 1 = every step.
  int deferB = 1;
};

struct Plan {
  Tuning tune;
  int n = 0, nsuper = 0, nlevels = 0, maxFront = 0;
  int64_t nnzLStored = 0, arenaDoubles = 0, nnzA = 0, patNnz = 0;
  // per supernode
  std::vector<int> snF, snNc, snM, snLevel, snParent;
  std::vector<int64_t> snLxp, snUoff;
  std::vector<int> chPtr, chList;  // children of s in the reference's extend-add order (childHead chain)
  // assembly of A: entries of supernode s are [asmPtr[s], asmPtr[s+1]) (= lowerP over its columns)
  std::vector<int64_t> asmPtr;
  std::vector<int> asmDst, asmSrc;  // offset in the L panel of s; CSR slot of the value
  std::vector<int> asmColPtr;       // lowerP relative: column j of s has entries [asmColPtr[f+j], asmColPtr[f+j+1])
  // extend-add: child c's rows below its block map to parent front positions eaMap[eaPtr[c] + a]
  std::vector<int64_t> eaPtr;
  std::vector<int> eaMap;
  // supernodes by level
  std::vector<int> lvlPtr, lvlSn;
  // task lists
  std::vector<AsmTask> asmTasks;
  std::vector<ChildRange> asmCh;  // per assembly task and child: the child's columns that map into the task's
  std::vector<int64_t> asmLvlPtr;  // per level
  std::vector<double> asmLvlBytes;  // algorithmic bytes of each level's assembly (A entries + extend-add)
  std::vector<GroupItem> groupItems;
  std::vector<StripTask> strips;
  int nGroupFlags = 0, nGroupTickets = 0;  // flags of all items, ticket counters of all group steps
  std::vector<TileTask> tileTasks;
  std::vector<int> lvlStepPtr;  // per level: steps [lvlStepPtr[L], lvlStepPtr[L+1])
  std::vector<TileTask> uTasks;  // long-K update-block tiles, per level [uLvlPtr[L], uLvlPtr[L+1])
  // mixed precision: the same steps with 128 x 256 tiles; BF16 split storage of the pivot columns
  std::vector<MixTask> mixTiles, mixUTasks;
  std::vector<int64_t> mixULvlPtr;  // per level
  std::vector<int64_t> snSp;  // split-column offset of supernode s (ld = round_up(m, 8) per front)
  int64_t splitElems = 0;
  std::vector<int64_t> uLvlPtr;
  std::vector<double> uLvlFlops;
  std::vector<StepRange> steps;
  // small fronts of each level, done whole by one warp (tiny) or one CTA (small) per front: tiny fronts of level L
  // are tinySn[tinyPtr[L] .. tinyPtr[L + 1]), small ones smallSn[smallPtr[L] ..], the largest m of those smallMaxM[L]
  std::vector<int> tinySn, smallSn, smallMaxM;
  std::vector<int64_t> tinyPtr, smallPtr;
  std::vector<int64_t> tinyMid;  // each level's tiny fronts are sorted by m; those from tinyMid[L] on have m > kTinyMid
  std::vector<double> frontLvlFlops, frontLvlBytes;  // algorithmic work of each level's small fronts
  // solve: rows below of each supernode (Si[Sp[s] + nc ..]) and the perm
  std::vector<int> perm, Sp, Si;
  int64_t solveBufDoubles = 0;      // sum of mu (per RHS) for the forward update vectors
  std::vector<int64_t> snTOff;      // offset of supernode s's forward update vector (per RHS)
  // block tasks of the solves ({supernode, block, kind, 0}); ready flags per 64-row pivot block
  std::vector<int> blkOff;          // first flag of supernode s
  std::vector<int> rowBlk;          // flag (64-column diagonal block) holding each column, permuted order (n)
  int nflags = 0;
  std::vector<int64_t> invOff;      // per diagonal block (flag index): offset of its w x w inverse; [nflags] = total
  std::vector<int> diagSlot;        // CSR slot of each diagonal entry of A (LDL^T pivot scale)
  std::vector<int> fwdTasks, bwdTasks;  // int4 records, flattened
  std::vector<int> fwdTasks1;           // the one-vector forward's list: fwdTasks with kind 3 (whole supernode) tasks
  std::vector<int> solveSmall;          // supernodes solved whole by one warp, grouped by level (tasks of kind 2)
  std::vector<int> invBlocks;           // diagonal blocks (flag index) whose inverse the block-task solves use
  std::vector<int> chainTasks;          // {s, b} pairs: every diagonal block of a supernode with two or more
  std::vector<int> fwdLvlPtr, bwdLvlPtr;
  std::vector<int> bwdAll;  // backward tasks of all levels, top-down (one launch)
  double flops = 0;
};

void build_plan(const Symbolic &S, Plan &P, const Tuning &tune = Tuning());
// the dense schedule of every front (built on demand, by the first complex factor of a plan)
void build_dense_all(const Plan &P, DenseSched &D);

}  // namespace amp
