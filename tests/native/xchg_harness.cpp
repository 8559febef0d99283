// Host harness around the exchange planner (piernik_b200/csrc/pk_exchange.cpp)
// for the CPU tests: flat arrays in, flat segment records out.
#include <cstring>
#include <string>
#include <vector>

#include "../../piernik_b200/csrc/pk_exchange.h"

extern "C" int xchg_plan(int nb, const int* n, const int* g, const long long* off, const long long* dom,
                         const int* periodic, int* segs, int max_segs, char* err, int errlen)
{
    std::vector<pk::XBlock> b(nb);
    for (int i = 0; i < nb; ++i)
        for (int d = 0; d < 3; ++d) {
            b[i].n[d] = n[3 * i + d];
            b[i].g[d] = g[3 * i + d];
            b[i].off[d] = off[3 * i + d];
        }
    std::vector<pk::XSeg> s;
    std::string e;
    if (!pk::build_exchange(b, dom, periodic, s, e)) {
        std::strncpy(err, e.c_str(), errlen - 1);
        err[errlen - 1] = 0;
        return -1;
    }
    if ((int)s.size() > max_segs) return -2;
    for (size_t k = 0; k < s.size(); ++k) {
        int* r = segs + 11 * k;
        r[0] = s[k].dst;
        r[1] = s[k].src;
        for (int d = 0; d < 3; ++d) {
            r[2 + d] = s[k].lo[d];
            r[5 + d] = s[k].hi[d];
            r[8 + d] = s[k].shift[d];
        }
    }
    return (int)s.size();
}

// Per-rank split: blocks listed this rank's first (nlocal of them), owner[i]
// for the rest.  Writes, for peer `peer`, the received (which = 0) or sent
// (which = 1) segments in their canonical order as records of 12 ints:
// dst offset (3), lo (3), hi (3) and 3 more: the source offset, folded
// through the shift into the source's first guard-inclusive cell.
extern "C" int xchg_peer(int nb, int nlocal, const int* owner, const int* n, const int* g, const long long* off,
                         const long long* dom, const int* periodic, int peer, int which, long long* out, int max_out)
{
    std::vector<pk::XBlock> b(nb);
    for (int i = 0; i < nb; ++i)
        for (int d = 0; d < 3; ++d) {
            b[i].n[d] = n[3 * i + d];
            b[i].g[d] = g[3 * i + d];
            b[i].off[d] = off[3 * i + d];
        }
    std::vector<pk::XSeg> s, local;
    std::vector<pk::XPeer> peers;
    std::string e;
    if (!pk::build_exchange(b, dom, periodic, s, e)) return -1;
    std::vector<int> own(owner, owner + nb);
    pk::split_by_owner(b, own, nlocal, s, local, peers);
    for (const auto& p : peers) {
        if (p.rank != peer) continue;
        const auto& l = which ? p.send : p.recv;
        if ((int)l.size() > max_out) return -2;
        for (size_t k = 0; k < l.size(); ++k) {
            long long* r = out + 12 * k;
            for (int d = 0; d < 3; ++d) {
                r[d] = b[l[k].dst].off[d];
                r[3 + d] = l[k].lo[d];
                r[6 + d] = l[k].hi[d];
                // global coordinate of the source cell under dst cell lo: dst base + lo - (dst base - src base - image)
                r[9 + d] = (b[l[k].dst].off[d] - b[l[k].dst].g[d]) + l[k].lo[d] - l[k].shift[d];
            }
        }
        return (int)l.size();
    }
    return 0;
}

// Per-rank segment lists with the device copy's own fields: for peer `peer`,
// the received (which = 0) or sent (which = 1) segments in canonical order,
// restricted to the face boxes along dir (seg_face_dir; dir = -1: all), as
// records of 11 ints: dst, src (this rank's numbering), lo (3), hi (3),
// shift (3).  which = 2 gives this rank's local copies (no peer).
extern "C" int xchg_peer_segs(int nb, int nlocal, const int* owner, const int* n, const int* g, const long long* off,
                              const long long* dom, const int* periodic, int peer, int which, int dir, int* out,
                              int max_out)
{
    std::vector<pk::XBlock> b(nb);
    for (int i = 0; i < nb; ++i)
        for (int d = 0; d < 3; ++d) {
            b[i].n[d] = n[3 * i + d];
            b[i].g[d] = g[3 * i + d];
            b[i].off[d] = off[3 * i + d];
        }
    std::vector<pk::XSeg> s, local;
    std::vector<pk::XPeer> peers;
    std::string e;
    if (!pk::build_exchange(b, dom, periodic, s, e)) return -1;
    std::vector<int> own(owner, owner + nb);
    pk::split_by_owner(b, own, nlocal, s, local, peers);
    const std::vector<pk::XSeg>* l = nullptr;
    if (which == 2) l = &local;
    for (const auto& p : peers)
        if (p.rank == peer) l = which ? &p.send : &p.recv;
    if (!l) return 0;
    int k = 0;
    for (const auto& x : *l) {
        if (dir >= 0 && pk::seg_face_dir(b[x.dst], x) != dir) continue;
        if (k >= max_out) return -2;
        int* r = out + 11 * k++;
        r[0] = x.dst;
        r[1] = x.src;
        for (int d = 0; d < 3; ++d) {
            r[2 + d] = x.lo[d];
            r[5 + d] = x.hi[d];
            r[8 + d] = x.shift[d];
        }
    }
    return k;
}
