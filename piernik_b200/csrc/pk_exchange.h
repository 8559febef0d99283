// pk_exchange.h -- guard-cell exchange between blocks of one refinement level
// on one device (cg_list_bnd.F90:251-324, internal_boundaries_local): the plan
// of box-to-box copies, built on the host.  Pure C++ so that the tests can
// build it without CUDA.
#pragma once
#include <string>
#include <vector>

namespace pk {

// One block as the exchange sees it: interior extent n, guard width g (0 in
// directions without extent), offset of its first interior cell on the
// level's global cell grid.
struct XBlock {
    int n[3];
    int g[3];
    long long off[3];
};

// One box of guard cells of block dst filled from the interior of block src:
// dst cells lo..hi-1 (in dst's guard-inclusive coordinates) take src cell
// (i + shift[0], j + shift[1], k + shift[2]) (in src's guard-inclusive
// coordinates).
struct XSeg {
    int dst, src;
    int lo[3], hi[3];
    int shift[3];
};

// Every guard cell of every block whose position (wrapped into the domain
// along periodic directions) lies in the interior of some block gets one
// segment cell.  dom: cells of the level along each direction; periodic: wrap
// flags.  Fails (returns false, err set) when two interiors overlap or a
// block leaves a non-periodic domain.
bool build_exchange(const std::vector<XBlock>& blocks, const long long dom[3], const int periodic[3],
                    std::vector<XSeg>& segs, std::string& err);

// Segments between this rank and one peer, in an order both ranks derive
// alike: by the destination block's offset, the segment's first cell, the
// source block's offset and the shift -- positions on the level's grid, not
// block numbers, which differ between ranks.
void sort_canonical(const std::vector<XBlock>& blocks, std::vector<XSeg>& segs);

// The direction along which segment s's box is a face box of block dst's
// guard region -- outside dst's interior along exactly that direction, inside
// along the other two -- or -1 for an edge or corner box.  A fused sweep along
// d reads guard cells of face boxes along d only, so the exchange before it
// needs those alone.  (A segment is a source interior's image clipped to dst's
// guard-inclusive box, so along each direction it lies wholly inside the
// interior or wholly in one guard layer.)
int seg_face_dir(const XBlock& dst, const XSeg& s);

// Split the segments of blocks[0..nlocal) (this rank's) and of the remote
// blocks (owner[i] >= 0 for i >= nlocal) into the local copies, and per peer
// rank the copies received (destination local) and sent (source local).
struct XPeer {
    int rank;
    std::vector<XSeg> recv, send;
};
void split_by_owner(const std::vector<XBlock>& blocks, const std::vector<int>& owner, int nlocal,
                    const std::vector<XSeg>& segs, std::vector<XSeg>& local, std::vector<XPeer>& peers);

}  // namespace pk
