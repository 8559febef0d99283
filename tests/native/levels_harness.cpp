// Host harness of the refined-domain planner (pk_levels.cpp) for the CPU
// tests: builds a plan and hands its tables out through plain C calls.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../piernik_b200/csrc/pk_levels.h"

static pk::LevelPlan g_plan;
static std::vector<pk::PRun> g_fill;
static pk::PartialRefresh g_part;
static std::vector<pk::LBlock> g_blocks;

static std::vector<pk::LBlock> blocks_of(int nb, const int* level, const int* n, const int* g, const long long* off)
{
    std::vector<pk::LBlock> b(nb);
    for (int i = 0; i < nb; ++i) {
        b[i].level = level[i];
        for (int d = 0; d < 3; ++d) {
            b[i].n[d] = n[3 * i + d];
            b[i].g[d] = g[3 * i + d];
            b[i].off[d] = off[3 * i + d];
        }
    }
    return b;
}

extern "C" {

// rows filling the interior of block target from the coarser level; -1 on error
long long lv_fill(int nb, const int* level, const int* n, const int* g, const long long* off, const long long* dom,
                  int target, char* err, int errlen)
{
    std::string e;
    if (!pk::build_fill_runs(blocks_of(nb, level, n, g, off), dom, target, g_fill, e)) {
        if (err && errlen > 0) {
            std::strncpy(err, e.c_str(), errlen - 1);
            err[errlen - 1] = 0;
        }
        return -1;
    }
    return (long long)g_fill.size();
}

void lv_fill_run(long long i, int* out)
{
    const pk::PRun& r = g_fill[i];
    const int v[12] = {r.fb, r.cb, r.fx, r.fy, r.fz, r.len, r.cx, r.cy, r.cz, r.px, r.py, r.pz};
    std::memcpy(out, v, sizeof(v));
}

int lv_build(int nb, const int* level, const int* n, const int* g, const long long* off, const long long* dom,
             char* err, int errlen)
{
    std::vector<pk::LBlock> b = blocks_of(nb, level, n, g, off);
    g_blocks = b;
    std::string e;
    if (!pk::build_levels(b, dom, g_plan, e)) {
        if (err && errlen > 0) {
            std::strncpy(err, e.c_str(), errlen - 1);
            err[errlen - 1] = 0;
        }
        return -1;
    }
    return 0;
}

long long lv_nruns() { return (long long)g_plan.runs.size(); }

static std::vector<pk::XSeg> g_segs;

// same-level segments of every level of the blocks of the last lv_build
// (periodic in every direction with extent), as the library plans them
long long lv_segs(const long long* dom)
{
    g_segs.clear();
    int maxl = 0;
    for (const pk::LBlock& b : g_blocks) maxl = std::max(maxl, b.level);
    const int per[3] = {1, 1, 1};
    for (int L = 0; L <= maxl; ++L) {
        std::vector<int> ids;
        std::vector<pk::XBlock> xb;
        for (int i = 0; i < (int)g_blocks.size(); ++i) {
            if (g_blocks[i].level != L) continue;
            pk::XBlock x;
            for (int d = 0; d < 3; ++d) {
                x.n[d] = g_blocks[i].n[d];
                x.g[d] = g_blocks[i].g[d];
                x.off[d] = g_blocks[i].off[d];
            }
            ids.push_back(i);
            xb.push_back(x);
        }
        long long dl[3];
        for (int d = 0; d < 3; ++d) dl[d] = dom[d] > 1 ? dom[d] << L : 1;
        std::vector<pk::XSeg> segs;
        std::string err;
        if (!pk::build_exchange(xb, dl, per, segs, err)) return -1;
        for (pk::XSeg s : segs) {
            s.dst = ids[s.dst];
            s.src = ids[s.src];
            g_segs.push_back(s);
        }
    }
    return (long long)g_segs.size();
}

void lv_seg(long long i, int* out)
{
    const pk::XSeg& s = g_segs[i];
    const int v[11] = {s.dst, s.src, s.lo[0], s.lo[1], s.lo[2], s.hi[0], s.hi[1], s.hi[2], s.shift[0], s.shift[1], s.shift[2]};
    std::memcpy(out, v, sizeof(v));
}

// the partial refresh of direction dir over the plan and segments built last
long long lv_partial(int dir, int r)
{
    pk::build_partial_refresh(g_blocks, g_plan, g_segs, dir, r, g_part);
    return (long long)g_part.segs.size();
}

long long lv_partial_nruns() { return (long long)g_part.runs.size(); }

void lv_partial_seg(long long i, int* out)
{
    const pk::XSeg& s = g_part.segs[i];
    const int v[11] = {s.dst, s.src, s.lo[0], s.lo[1], s.lo[2], s.hi[0], s.hi[1], s.hi[2], s.shift[0], s.shift[1], s.shift[2]};
    std::memcpy(out, v, sizeof(v));
}

void lv_partial_run(long long i, int* out)
{
    const pk::PRun& r = g_part.runs[i];
    const int v[12] = {r.fb, r.cb, r.fx, r.fy, r.fz, r.len, r.cx, r.cy, r.cz, r.px, r.py, r.pz};
    std::memcpy(out, v, sizeof(v));
}

void lv_run(long long i, int* out)
{
    const pk::PRun& r = g_plan.runs[i];
    const int v[12] = {r.fb, r.cb, r.fx, r.fy, r.fz, r.len, r.cx, r.cy, r.cz, r.px, r.py, r.pz};
    std::memcpy(out, v, sizeof(v));
}

long long lv_run_level_beg(int L) { return g_plan.run_level_beg[L]; }

int lv_fc_nin(int d) { return (int)g_plan.fc[d].in_face.size(); }

// face, then the 4 out slots summed into in slot s
void lv_fc_in(int d, int s, int* out)
{
    out[0] = g_plan.fc[d].in_face[s];
    for (int q = 0; q < 4; ++q) out[1 + q] = g_plan.fc[d].src[4 * s + q];
}

int lv_fc_in_level_beg(int d, int L) { return g_plan.fc[d].in_level_beg[L]; }

// slot of block b's pencil pen on side (kind 0: in, 1: out); -2 when the block has no table
int lv_fc_slot(int d, int b, int kind, int side, long long pen)
{
    const std::vector<int>& t = kind == 0 ? g_plan.fc[d].in_slot[b] : g_plan.fc[d].out_slot[b];
    if (t.empty()) return -2;
    return t[(size_t)side * (t.size() / 2) + pen];
}

long long lv_leaf_cells(int b) { return g_plan.leaf_cells[b]; }

int lv_leaf(int b, long long c)
{
    if (g_plan.leaf[b].empty()) return 1;
    return g_plan.leaf[b][c];
}

}  // extern "C"
