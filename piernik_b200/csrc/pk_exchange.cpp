// pk_exchange.cpp -- plan of the same-level guard-cell exchange (see
// pk_exchange.h).  The reference walks, per block, the list of neighbour
// segments found when the level was built (cg_list_bnd.F90:286-314) and
// copies each one; here every (destination, source, periodic image) triple is
// intersected once on the host and the copies run as one kernel.
#include "pk_exchange.h"

#include <algorithm>
#include <cstdio>
#include <map>
#include <tuple>

namespace pk {

namespace {

struct Box {
    long long lo[3], hi[3];
    bool empty() const { return lo[0] >= hi[0] || lo[1] >= hi[1] || lo[2] >= hi[2]; }
};

Box intersect(const Box& a, const Box& b)
{
    Box r;
    for (int d = 0; d < 3; ++d) {
        r.lo[d] = a.lo[d] > b.lo[d] ? a.lo[d] : b.lo[d];
        r.hi[d] = a.hi[d] < b.hi[d] ? a.hi[d] : b.hi[d];
    }
    return r;
}

Box interior(const XBlock& b, const long long shift[3])
{
    Box r;
    for (int d = 0; d < 3; ++d) {
        r.lo[d] = b.off[d] + shift[d];
        r.hi[d] = b.off[d] + b.n[d] + shift[d];
    }
    return r;
}

}  // namespace

bool build_exchange(const std::vector<XBlock>& blocks, const long long dom[3], const int periodic[3],
                    std::vector<XSeg>& segs, std::string& err)
{
    segs.clear();
    const int nb = (int)blocks.size();
    char msg[200];
    for (int i = 0; i < nb; ++i)
        for (int d = 0; d < 3; ++d) {
            const XBlock& b = blocks[i];
            if (b.n[d] < 1 || b.g[d] < 0 || dom[d] < 1) {
                err = "block extents, guard widths and the domain must be positive";
                return false;
            }
            if (b.off[d] < 0 || b.off[d] + b.n[d] > dom[d]) {
                std::snprintf(msg, sizeof msg, "block %d leaves the domain along direction %d", i, d);
                err = msg;
                return false;
            }
            if (periodic[d] && b.g[d] > dom[d]) {
                err = "periodic domain narrower than the guard width";
                return false;
            }
        }
    // periodic images considered along each direction
    int kmin[3], kmax[3];
    for (int d = 0; d < 3; ++d) {
        kmin[d] = periodic[d] ? -1 : 0;
        kmax[d] = periodic[d] ? 1 : 0;
    }
    for (int i = 0; i < nb; ++i) {
        const XBlock& t = blocks[i];
        const long long zero[3] = {0, 0, 0};
        const Box own = interior(t, zero);
        Box ext;
        for (int d = 0; d < 3; ++d) {
            ext.lo[d] = t.off[d] - t.g[d];
            ext.hi[d] = t.off[d] + t.n[d] + t.g[d];
        }
        for (int j = 0; j < nb; ++j) {
            const XBlock& s = blocks[j];
            for (int kz = kmin[2]; kz <= kmax[2]; ++kz)
                for (int ky = kmin[1]; ky <= kmax[1]; ++ky)
                    for (int kx = kmin[0]; kx <= kmax[0]; ++kx) {
                        const long long sh[3] = {kx * dom[0], ky * dom[1], kz * dom[2]};
                        const Box src = interior(s, sh);
                        if (!intersect(src, own).empty()) {
                            if (i == j && kx == 0 && ky == 0 && kz == 0) continue;   // the block itself
                            std::snprintf(msg, sizeof msg, "blocks %d and %d overlap (periodic image %d,%d,%d)", i, j,
                                          kx, ky, kz);
                            err = msg;
                            return false;
                        }
                        const Box r = intersect(src, ext);
                        if (r.empty()) continue;
                        XSeg g;
                        g.dst = i;
                        g.src = j;
                        for (int d = 0; d < 3; ++d) {
                            const long long base_t = t.off[d] - t.g[d];
                            const long long base_s = s.off[d] + sh[d] - s.g[d];
                            g.lo[d] = (int)(r.lo[d] - base_t);
                            g.hi[d] = (int)(r.hi[d] - base_t);
                            g.shift[d] = (int)(base_t - base_s);
                        }
                        segs.push_back(g);
                    }
        }
    }
    return true;
}

void sort_canonical(const std::vector<XBlock>& blocks, std::vector<XSeg>& segs)
{
    auto key = [&](const XSeg& s) {
        const XBlock& d = blocks[s.dst];
        const XBlock& q = blocks[s.src];
        return std::make_tuple(d.off[2], d.off[1], d.off[0], s.lo[2], s.lo[1], s.lo[0], q.off[2], q.off[1], q.off[0],
                               s.shift[2], s.shift[1], s.shift[0]);
    };
    std::stable_sort(segs.begin(), segs.end(), [&](const XSeg& a, const XSeg& b) { return key(a) < key(b); });
}

int seg_face_dir(const XBlock& dst, const XSeg& s)
{
    int dir = -1, out = 0;
    for (int d = 0; d < 3; ++d) {
        const bool inside = s.lo[d] >= dst.g[d] && s.hi[d] <= dst.g[d] + dst.n[d];
        if (!inside) {
            dir = d;
            ++out;
        }
    }
    return out == 1 ? dir : -1;
}

void split_by_owner(const std::vector<XBlock>& blocks, const std::vector<int>& owner, int nlocal,
                    const std::vector<XSeg>& segs, std::vector<XSeg>& local, std::vector<XPeer>& peers)
{
    local.clear();
    peers.clear();
    std::map<int, XPeer> by;
    for (const XSeg& s : segs) {
        const bool dl = s.dst < nlocal, sl = s.src < nlocal;
        if (dl && sl) local.push_back(s);
        else if (dl) {
            XPeer& p = by[owner[s.src]];
            p.rank = owner[s.src];
            p.recv.push_back(s);
        } else if (sl) {
            XPeer& p = by[owner[s.dst]];
            p.rank = owner[s.dst];
            p.send.push_back(s);
        }
    }
    for (auto& kv : by) {
        sort_canonical(blocks, kv.second.recv);
        sort_canonical(blocks, kv.second.send);
        peers.push_back(kv.second);
    }
}

}  // namespace pk
