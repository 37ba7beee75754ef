// factor.hpp — one-time sparse Cholesky factorisation of the global-step
// matrix M + dt^2 A^T A and its device layout.
//
// Replaces Eigen::SimplicialLLT::compute (include/physics/SimulationSpeed.hpp:102,
// src/physics/SimulationSpeed.cpp:53).  The matrix is constant for the whole run
// (the reference never refactorises in the shipped path), so the factor is
// computed once on the host in FP64 and then re-laid out for the device
// triangular sweeps:
//
//  * ordering: nested dissection by recursive coordinate bisection of the rest
//    positions with vertex separators taken from the matrix graph;
//  * supernodes = the nested-dissection tree nodes (leaf domains and
//    separators), each a dense column block [c0, c0+ns) with row set R_s;
//  * numeric factorisation: multifrontal, supernode by supernode in postorder;
//  * partitioned inverse: per supernode W_s = [D_s^-1 ; L_Rs D_s^-1] where D_s
//    is the diagonal block.  The forward sweep is then y_s = D^-1 b_s,
//    b_R -= (L_R D^-1) b_s and the backward sweep x_s = W_s^T [y_s ; -x_R]:
//    both are plain matrix-vector products with no dependency inside a
//    supernode, so a supernode can be split across any number of warps.
//  * W_s is stored twice in 32-lane tiles, one copy per sweep, so that a warp
//    streams a tile with one coalesced load per step:
//      forward tile t  = rows [32t, 32t+m) of W_s, m = min(32, ns+nr-32t),
//                        columns 0..w_t-1 (w_t = min(ns, 32t+32): the zero
//                        upper part of D^-1 is not stored beyond the tile's
//                        diagonal block); element (row 32t+l, col j) at
//                        off + m j + l;
//      backward tile t = columns [32t, 32t+mc) of W_s, mc = min(32, ns-32t),
//                        rows 32t..ns-1 of D^-1 then the nr rows of L_R D^-1
//                        (h_t = ns - 32t + nr); element (local row i, col
//                        32t+l) at off + mc i + l.
//    Only the last tile of a supernode is narrower than 32; no rows or lanes
//    of zeros are stored (each tile is padded to a multiple of kTilePad
//    elements).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "model.hpp"

namespace pdfb {

constexpr int kTile = 32;
// Every tile of the tiled copies starts on a multiple of kTilePad elements
// (16 bytes in FP32 and FP64), the alignment bulk asynchronous copies need;
// the arrays end with kTilePad elements of zeros, so that a copy rounded up
// to 16 bytes stays inside them.
constexpr int kTilePad = 4;
inline int64_t pad_tile(int64_t elems) { return (elems + kTilePad - 1) / kTilePad * kTilePad; }

struct Factor {
  int N = 0;
  std::vector<int> perm, iperm;  // perm[k] = vertex at pivot position k
  int n_sn = 0;
  std::vector<int> sn_c0, sn_ns, sn_nr, sn_parent, sn_level;
  std::vector<int64_t> sn_roff;  // offset into rows
  std::vector<int> rows;         // R_s, permuted indices, ascending
  std::vector<int64_t> sn_woff;  // offset of W_s in the packed row-major form
  // tiled copies (see above); forward tiles of supernode s are
  // [sn_ftile0[s], sn_ftile0[s+1]), backward tiles [sn_btile0[s], sn_btile0[s+1])
  std::vector<int64_t> sn_ftile0, sn_btile0;
  std::vector<int64_t> ftile_off, btile_off;  // per tile, +1 sentinel
  std::vector<double> Wf, Wb;
  int n_levels = 0;
  int64_t nnz_w = 0;             // sum ns(ns+1)/2 + nr ns
  int64_t nnz_l_true = 0;        // structural nnz of L (diagonal included)
  int64_t tiled_w = 0;           // stored elements per tiled copy (upper triangles of the diagonal blocks included)
  double factor_ms = 0;
};

// Returns false (and sets err) if the matrix is not positive definite.
bool factorize(const Model& m, double dt, int leaf_size, Factor& f, std::string& err);

// One warp's work item of a supernodal sweep: tile `tile` of supernode `sn`
// (rows 32 tile.. of W_s for the forward sweep, columns for the backward one),
// restricted to the chunk [a0, a1) of columns (forward) or local rows
// (backward); `off` is the tile's offset in the tiled W copy.
struct SweepTask {
  int sn, tile, a0, a1;
  int64_t off;
};
struct SnInfo {
  int c0, ns, nr, parent;
  int64_t roff;
  int nchild, ntf, ntb, pad;  // children, forward / backward work items
};

// Work items of both sweeps in elimination-tree order (forward: levels
// bottom-up; backward: top-down), at most 32 x chunk elements each, and the
// per-supernode dependency record.
void build_sweep_tasks(const Factor& f, int chunk, std::vector<SweepTask>& fwd, std::vector<SweepTask>& bwd,
                       std::vector<SnInfo>& sn);

// ---- subtree blocks ------------------------------------------------------
// The lower part of the elimination tree is cut into subtrees that one CTA
// solves alone: the subtree's columns are contiguous in the pivot order, so
// its slice of the vector lives in shared memory, the levels inside it are
// separated by CTA barriers, and the factor streams in through bulk
// asynchronous copies.  The rows a subtree touches outside itself are exactly
// its root's row set R_root (a child's rows beyond its parent's columns are
// rows of the parent), so they live in shared memory too ("ext" rows): the
// forward sweep accumulates their updates there and adds them to b once per
// block, the backward sweep loads their x once per block.  Supernodes in no
// block ("upper" supernodes) keep the dependency-driven per-warp work items.
constexpr int kMaxBlockLevels = 16;
constexpr int kMaxBlockCols = 1536;
constexpr int kMaxBlockExt = 1024;
constexpr int kMaxBlockItems = 768;  // work items per block and sweep (staged in shared memory)
// columns (forward) / rows (backward) per bulk copy: 16 in FP64, 32 in FP32
// (4 KB either way); item starts and the backward index lists are aligned to
// the larger
constexpr int kSlab = 16;
constexpr int kSlabMax = 32;
// A tile longer than its sweep's span (forward columns, backward rows) is
// split into items of that span whose partial sums meet in atomics, so that
// long tiles do not hold one warp while the others wait at the level
// barrier.  Backward tiles run over the supernode's rows below it (often
// several times its width), so their span is short: per level, the longest
// warp's work comes within 1.3x of an even split on the 500 x 500 cloth.
constexpr int kBlockSpanF = 128;  // multiples of kSlabMax
constexpr int kBlockSpanB = 32;

struct SweepBlock {
  int c0, c1;    // columns [c0, c1) of the subtree
  int parent;    // supernode above the subtree root, -1 if none
  int nlev;      // levels inside the block
  int item0;     // first item of the block in the item array
  int ext0;      // its ext rows are Factor::rows[ext0, ext0 + next) (R of the root)
  int next;
  int lev[kMaxBlockLevels + 1];  // item offsets (from item0) per level, in sweep order
};
// One work item of a tile of a supernode inside a block: forward, rows
// [32 tile, 32 tile + m) of W_s over its columns [a0, a1) of
// w = min(ns, 32 tile + 32); backward, columns [32 tile, 32 tile + mc) over
// its rows [a0, a1) of h = ns - 32 tile + nr.  a0 is a multiple of kSlabMax.
// The small fields are 16-bit (a block has at most kMaxBlockCols columns and
// kMaxBlockExt ext rows), so that an item is 32 bytes of shared memory.
struct BlockItem {
  int64_t off;   // tile offset in the forward (backward) tiled copy
  int roff;      // offset of the supernode's row set in Factor::rows (and rows_loc)
  int idx0;      // backward: offset of the tile's row-index list in bidx (multiple of kSlabMax)
  int16_t c0l;   // first column of the supernode, relative to the block
  int16_t ns, nr;
  int16_t tile;
  int16_t a0, a1;
  int16_t pad[2];
};
static_assert(sizeof(BlockItem) == 32, "BlockItem is 32 bytes");
static_assert(kBlockSpanF % kSlabMax == 0 && kBlockSpanB % kSlabMax == 0, "items start on a slab");

// An upper work item as the device reads it: the SweepTask with the fields
// of its supernode it needs and its dependency targets per solve, so that one
// 64-byte load replaces the task load and the dependent supernode load.
struct alignas(16) UpperItem {
  int64_t off;     // tile offset in the tiled copy
  int sn, tile, a0, a1;
  int c0, ns, nr, roff;
  int parent;      // parent supernode, -1 if none
  int wait;        // forward: upper children of sn; backward: work items of the parent
  int ntf;         // forward: work items of sn
  int child0;      // forward: its upper children are SweepPlan::child[child0, child0 + wait)
  int pad[2];
};
static_assert(sizeof(UpperItem) == 64, "UpperItem is one 64-byte record");

struct SweepPlan {
  int cut_level = 0, chunk = 0;
  std::vector<SweepTask> fup, bup;     // upper work items, forward / backward
  std::vector<SnInfo> sn;              // dependency record (upper supernodes)
  std::vector<SweepBlock> fblk, bblk;  // blocks, item offsets in forward / backward order
  std::vector<BlockItem> fitem, bitem;
  std::vector<UpperItem> fupi, bupi;   // the upper items as the device reads them
  // the upper items by elimination-tree level, in sweep order: forward level
  // k is fupi[fup_lev[k], fup_lev[k+1]), backward level k bupi[bup_lev[k], ...)
  std::vector<int> fup_lev, bup_lev;
  std::vector<int> upper_cols;         // pivot positions of the upper supernodes' columns
  // per upper supernode with upper children: (child, forward work items of
  // the child), the counters a forward item polls before it starts
  std::vector<int> child;              // pairs, flattened
  // per entry of Factor::rows of a block supernode: the row's place in the
  // block's shared vector (column - c0 inside the block, nc + ext index outside)
  std::vector<int> rows_loc;
  // backward tiles of blocks: per row of the tile, padded to kSlabMax rows, where
  // its vector entry is: >= 0 the shared vector (x), < 0 the shared y slice
  // (entry -1 - k is column k of the block)
  std::vector<int> bidx;
  int max_block_cols = 0, max_block_ext = 0, max_block_items = 0;
  int64_t block_elems = 0, upper_elems = 0;  // stored W elements per sweep copy
};

// Blocks are the largest subtrees whose root is at most cut_level and whose
// columns are contiguous, at most kMaxBlockCols, with at most kMaxBlockExt
// rows outside and at most kMaxBlockItems tiles per sweep; the rest is upper.
void build_sweep_plan(const Factor& f, int chunk, int cut_level, SweepPlan& plan);

// Host emulation of the two device sweeps of a plan on the tiled layout (same
// blocks and work items, same index arithmetic, every index bounds-checked):
// solves (M + dt^2 A^T A) x = b for three right-hand sides given vertex-major
// (3N), result vertex-major.  Returns false with err on an out-of-range index.
bool emulate_sweeps(const Factor& f, const SweepPlan& plan, const std::vector<double>& b, std::vector<double>& x,
                    std::string& err);

// W column offset inside a supernode: column j starts at colstart(j).
inline int64_t w_colstart(int64_t j, int64_t ns, int64_t nr) { return j * (ns + nr) - j * (j - 1) / 2; }
// W row offset: rows i < ns start at i(i+1)/2, rows ns+r at ns(ns+1)/2 + r ns.
inline int64_t w_rowstart(int64_t i, int64_t ns) {
  return i < ns ? i * (i + 1) / 2 : ns * (ns + 1) / 2 + (i - ns) * ns;
}

}  // namespace pdfb
