// pk_levels.h -- the vertical (fine/coarse) couplings of a refined, fully
// periodic domain on one device, planned on the host.  Pure C++ so that the
// tests can build it without CUDA.
//
// Refinement factor 2 between consecutive levels (constants.F90:331).  A block
// of level L sits at an offset on the level-L cell grid, which is the base
// grid refined L times.  Three couplings follow from the layout:
//
//  * prolongation of fine guard cells from the coarser level
//    (cg_level_connected.F90:1150-1359 prolong_bnd_from_coarser, with the
//    target areas of vertical_b_prep :422-704): every guard cell of a level
//    L >= 1 block whose position lies in no interior of its own level takes
//    its value from the level L-1 cell containing it;
//  * the fine->coarse flux correction (fc_fluxes.F90:55-233,
//    grid_container_fcflx.F90:148-259, cg_level_connected.F90:714-825
//    vertical_bf_prep): the flux a fine block computes through a boundary face
//    that borders the coarser level replaces, restricted (the mean of the 2 x 2
//    fine faces), the coarse block's own flux through that face;
//  * leaf cells (cg%leafmap): the CFL reduction skips cells covered by a finer
//    block (timestep.F90:463).
#pragma once
#include <string>
#include <vector>

#include "pk_exchange.h"

namespace pk {

struct LBlock {
    int level;
    int n[3];
    int g[3];
    long long off[3];          // first interior cell on the level's grid
};

// A row of fine guard cells filled from one coarse block: fine block fb,
// guard-inclusive storage cells (fx + i, fy, fz) for i in [0, len); cell i
// has x parity (px + i) & 1 inside its coarse parent and the parent
// (cx + ((px + i) >> 1), cy, cz) in the coarse block cb's storage.
struct PRun {
    int fb, cb;
    int fx, fy, fz, len;
    int cx, cy, cz;
    int px, py, pz;
};

// The flux couplings of one sweep direction.  Pencils of a block are
// numbered i1 + n[o1] * i2 with (o1, o2) = ({1,0,0}[d], {2,2,1}[d]).
struct FcDir {
    // per block: [2][npencil] slot numbers (-1: none) or empty when the block
    // has no slot of that kind along d
    std::vector<std::vector<int>> in_slot, out_slot;
    std::vector<int> in_face;         // per in slot: storage index along the pencil of the
                                      // cell whose right face takes the restricted flux
    std::vector<int> src;             // per in slot: 4 out slots (-1: none), summed in this order
    std::vector<int> in_level_beg;    // max_level + 1 entries: in slots of coarse level L are
                                      // [in_level_beg[L], in_level_beg[L+1])
    int n_out = 0;
};

// Coarse cells [lo, hi) (coarse block cb's storage coordinates) covered by
// fine block fb: the targets of restriction (cg_level_connected.F90:1480-1721)
struct RBox {
    int fb, cb;
    int lo[3], hi[3];
    int flo[3];          // fine block fb's storage cell of the first child of lo
};

struct LevelPlan {
    int max_level = 0;
    int eff_dim = 0;
    std::vector<PRun> runs;               // ordered by the fine block's level
    std::vector<long long> run_level_beg; // runs of fine level L: [run_level_beg[L], run_level_beg[L+1])
    FcDir fc[3];
    std::vector<std::vector<unsigned char>> leaf;   // per block: interior leaf mask (1 = leaf) or empty (all leaf)
    std::vector<long long> leaf_cells;              // per block: number of leaf cells
    std::vector<RBox> rboxes;                       // restriction targets, by the fine block's level
    std::vector<int> rbox_level_beg;                // boxes of fine level L: [rbox_level_beg[L], rbox_level_beg[L+1])
};

// dom: base-level cells per direction (1 where the domain has no extent);
// every direction with extent is periodic.  Checks: blocks of one level do
// not overlap, level 0 covers the domain, blocks of level >= 1 have even
// offsets and extents, every coarse cell a fine block reads lies in an
// interior of the next coarser level, and no coarse pencil borders two fine
// regions on the same side.
bool build_levels(const std::vector<LBlock>& blocks, const long long dom[3], LevelPlan& plan, std::string& err);

// Rows prolonging every interior cell of block `target` from the next coarser
// level, as the refinement update fills a new block (cg_level_connected.F90:
// 870-920 prolong, 1059-1093 the fine block's ijkse): fails if a parent lies
// in no interior of that level.
bool build_fill_runs(const std::vector<LBlock>& blocks, const long long dom[3], int target, std::vector<PRun>& runs,
                     std::string& err);

// The guard refresh one RK stage of the interior-trimmed stage kernel needs
// before it sweeps direction dir: that kernel reads, of each block, only the
// two guard layers on either side of the interior along dir, across the
// interior (the slabs), and a prolonged slab cell reads the coarser block's
// cells within the stencil range r of its parent, guard cells included,
// which must be refreshed too (closed downwards level by level).  Every
// other guard cell may stay stale until a full refresh.  From the full
// plan (same-level segments segs, prolongation rows plan.runs) keeps the
// segment pieces and row pieces that write needed cells: slab pieces as
// boxes, the few other needed cells as rows.
struct PartialRefresh {
    std::vector<XSeg> segs;
    std::vector<PRun> runs;                 // by the fine block's level
    std::vector<long long> run_level_beg;   // as LevelPlan::run_level_beg
};
void build_partial_refresh(const std::vector<LBlock>& blocks, const LevelPlan& plan, const std::vector<XSeg>& segs,
                           int dir, int r, PartialRefresh& out);

}  // namespace pk
