// pk_levels.cpp -- host planner of the fine/coarse couplings (pk_levels.h).
#include "pk_levels.h"

#include <algorithm>
#include <map>

namespace pk {

namespace {

// ortho directions of a sweep in the kernels' pencil numbering
constexpr int GO1[3] = {1, 0, 0};
constexpr int GO2[3] = {2, 2, 1};
// pdims (constants.F90:127-128): ORTHO1 / ORTHO2 of the reference, the loop
// order of the fine->coarse flux sum (fc_fluxes.F90:213-222)
constexpr int RO1[3] = {1, 2, 0};
constexpr int RO2[3] = {2, 0, 1};

long long floordiv2(long long x) { return x >= 0 ? x / 2 : -((-x + 1) / 2); }

// blocks of one level by position: which interior holds a cell
struct LevelIndex {
    long long D[3];
    long long nbk[3];
    static constexpr int BS = 16;
    std::vector<std::vector<int>> bucket;
    const std::vector<LBlock>* blocks = nullptr;

    void init(const std::vector<LBlock>& b, const long long dom[3], int level)
    {
        blocks = &b;
        for (int d = 0; d < 3; ++d) {
            D[d] = dom[d] > 1 ? dom[d] << level : 1;
            nbk[d] = (D[d] + BS - 1) / BS;
        }
        bucket.assign((size_t)(nbk[0] * nbk[1] * nbk[2]), {});
    }
    size_t bidx(long long x, long long y, long long z) const { return (size_t)((z * nbk[1] + y) * nbk[0] + x); }
    void add(int id)
    {
        const LBlock& b = (*blocks)[id];
        long long lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {
            lo[d] = b.off[d] / BS;
            hi[d] = (b.off[d] + b.n[d] - 1) / BS;
        }
        for (long long z = lo[2]; z <= hi[2]; ++z)
            for (long long y = lo[1]; y <= hi[1]; ++y)
                for (long long x = lo[0]; x <= hi[0]; ++x) bucket[bidx(x, y, z)].push_back(id);
    }
    bool wrap(long long p[3]) const
    {
        for (int d = 0; d < 3; ++d) {
            if (D[d] == 1) {
                if (p[d] != 0) return false;
                continue;
            }
            p[d] %= D[d];
            if (p[d] < 0) p[d] += D[d];
        }
        return true;
    }
    // the block whose interior holds cell p (wrapped in place), -1 if none
    int owner(long long p[3]) const
    {
        if (!wrap(p)) return -1;
        for (int id : bucket[bidx(p[0] / BS, p[1] / BS, p[2] / BS)]) {
            const LBlock& b = (*blocks)[id];
            bool in = true;
            for (int d = 0; d < 3; ++d) in = in && p[d] >= b.off[d] && p[d] < b.off[d] + b.n[d];
            if (in) return id;
        }
        return -1;
    }
};

std::string where(int id, const LBlock& b)
{
    return "block " + std::to_string(id) + " (level " + std::to_string(b.level) + ")";
}

}  // namespace

bool build_levels(const std::vector<LBlock>& blocks, const long long dom[3], LevelPlan& plan, std::string& err)
{
    plan = LevelPlan();
    const int nb = (int)blocks.size();
    int maxl = 0;
    for (const LBlock& b : blocks) {
        if (b.level < 0 || b.level > 8) {
            err = "levels must lie in 0..8";
            return false;
        }
        maxl = std::max(maxl, b.level);
    }
    plan.max_level = maxl;
    bool has[3];
    for (int d = 0; d < 3; ++d) {
        has[d] = dom[d] > 1;
        plan.eff_dim += has[d];
    }
    std::vector<LevelIndex> idx(maxl + 1);
    std::vector<std::vector<int>> of_level(maxl + 1);
    for (int i = 0; i < nb; ++i) of_level[blocks[i].level].push_back(i);
    for (int L = 0; L <= maxl; ++L) {
        idx[L].init(blocks, dom, L);
        long long cells = 0;
        for (int i : of_level[L]) {
            const LBlock& b = blocks[i];
            for (int d = 0; d < 3; ++d) {
                if (b.off[d] < 0 || b.off[d] + b.n[d] > idx[L].D[d] || (!has[d] && b.n[d] != 1)) {
                    err = where(i, b) + " leaves its level's grid";
                    return false;
                }
                if (L > 0 && has[d] && ((b.off[d] & 1) || (b.n[d] & 1))) {
                    err = where(i, b) + ": blocks of refined levels need even offsets and extents";
                    return false;
                }
                if (has[d] && b.g[d] < 2) {
                    err = where(i, b) + ": refined domains need at least 2 guard cells";
                    return false;
                }
            }
            // overlap with an earlier block of the level
            for (int j : of_level[L]) {
                if (j >= i) break;
                const LBlock& o = blocks[j];
                bool ov = true;
                for (int d = 0; d < 3; ++d) ov = ov && b.off[d] < o.off[d] + o.n[d] && o.off[d] < b.off[d] + b.n[d];
                if (ov) {
                    err = where(i, b) + " overlaps block " + std::to_string(j);
                    return false;
                }
            }
            idx[L].add(i);
            cells += (long long)b.n[0] * b.n[1] * b.n[2];
        }
        if (L == 0 && cells != dom[0] * dom[1] * dom[2]) {
            err = "the base level must cover the domain";
            return false;
        }
    }

    // prolongation targets: guard cells of refined blocks outside every interior of their level
    plan.run_level_beg.assign(maxl + 2, 0);
    for (int L = 1; L <= maxl; ++L) {
        plan.run_level_beg[L] = (long long)plan.runs.size();
        for (int i : of_level[L]) {
            const LBlock& b = blocks[i];
            int ext[3];
            for (int d = 0; d < 3; ++d) ext[d] = b.n[d] + 2 * b.g[d];
            for (int z = 0; z < ext[2]; ++z)
                for (int y = 0; y < ext[1]; ++y) {
                    PRun run{};
                    run.len = 0;
                    for (int x = 0; x < ext[0]; ++x) {
                        const int s[3] = {x, y, z};
                        bool interior = true;
                        for (int d = 0; d < 3; ++d) interior = interior && s[d] >= b.g[d] && s[d] < b.g[d] + b.n[d];
                        int cb = -1, cs[3] = {0, 0, 0}, par[3] = {0, 0, 0};
                        if (!interior) {
                            long long f[3];
                            for (int d = 0; d < 3; ++d) f[d] = s[d] - b.g[d] + b.off[d];
                            long long fw[3] = {f[0], f[1], f[2]};
                            if (idx[L].owner(fw) < 0) {
                                long long p[3];
                                for (int d = 0; d < 3; ++d) {
                                    p[d] = has[d] ? floordiv2(f[d]) : 0;
                                    par[d] = has[d] ? (int)(f[d] - 2 * floordiv2(f[d])) : 0;
                                }
                                cb = idx[L - 1].owner(p);
                                if (cb < 0) {
                                    err = where(i, b) + " is not nested in level " + std::to_string(L - 1);
                                    return false;
                                }
                                const LBlock& c = blocks[cb];
                                for (int d = 0; d < 3; ++d) cs[d] = (int)(p[d] - c.off[d]) + c.g[d];
                            }
                        }
                        const bool cont = run.len > 0 && cb == run.cb && cs[1] == run.cy && cs[2] == run.cz &&
                                          par[1] == run.py && par[2] == run.pz &&
                                          cs[0] == run.cx + ((run.px + run.len) >> 1) && par[0] == ((run.px + run.len) & 1);
                        if (cont) {
                            ++run.len;
                            continue;
                        }
                        if (run.len > 0) plan.runs.push_back(run);
                        run.len = 0;
                        if (cb >= 0) {
                            run = PRun{i, cb, x, y, z, 1, cs[0], cs[1], cs[2], par[0], par[1], par[2]};
                        }
                    }
                    if (run.len > 0) plan.runs.push_back(run);
                }
        }
    }
    plan.run_level_beg[maxl + 1] = (long long)plan.runs.size();
    if (maxl == 0) plan.run_level_beg.assign(2, 0);

    // fine->coarse flux couplings per direction
    for (int d = 0; d < 3; ++d) {
        FcDir& F = plan.fc[d];
        F.in_slot.assign(nb, {});
        F.out_slot.assign(nb, {});
        F.in_level_beg.assign(maxl + 1, 0);
        if (!has[d] || maxl == 0) continue;
        const int o1 = GO1[d], o2 = GO2[d];
        // in slots grouped by coarse level: build per level, then number
        std::vector<std::map<std::pair<int, long long>, int>> in_of(maxl);   // (coarse block, side*np+pen) -> local slot
        std::vector<std::vector<int>> face_of(maxl), src_of(maxl);
        std::vector<std::vector<std::pair<int, int>>> pending(maxl);   // (local in slot, 4-position) per out slot
        struct OutRec {
            int lvl, local, pos, slot;
        };
        std::vector<OutRec> outs;
        for (int L = 1; L <= maxl; ++L)
            for (int i : of_level[L]) {
                const LBlock& b = blocks[i];
                const long long np = (long long)b.n[o1] * b.n[o2];
                for (int side = 0; side < 2; ++side)
                    for (int i2 = 0; i2 < b.n[o2]; ++i2)
                        for (int i1 = 0; i1 < b.n[o1]; ++i1) {
                            long long f[3];
                            f[d] = side == 0 ? b.off[d] - 1 : b.off[d] + b.n[d];
                            f[o1] = b.off[o1] + i1;
                            f[o2] = b.off[o2] + i2;
                            long long fw[3] = {f[0], f[1], f[2]};
                            if (idx[L].owner(fw) >= 0) continue;
                            long long p[3];
                            for (int e = 0; e < 3; ++e) p[e] = has[e] ? floordiv2(f[e]) : 0;
                            const int cb = idx[L - 1].owner(p);
                            if (cb < 0) {
                                err = where(i, b) + " is not nested in level " + std::to_string(L - 1);
                                return false;
                            }
                            const LBlock& c = blocks[cb];
                            const int s_out = (int)(p[d] - c.off[d]) + c.g[d];
                            const long long cpen = (p[o1] - c.off[o1]) + (long long)c.n[o1] * (p[o2] - c.off[o2]);
                            const int face = side == 0 ? s_out : s_out - 1;
                            auto key = std::make_pair(cb, side * ((long long)c.n[o1] * c.n[o2]) + cpen);
                            int local;
                            auto it = in_of[L - 1].find(key);
                            if (it == in_of[L - 1].end()) {
                                local = (int)face_of[L - 1].size();
                                in_of[L - 1][key] = local;
                                face_of[L - 1].push_back(face);
                                src_of[L - 1].insert(src_of[L - 1].end(), 4, -1);
                            } else {
                                local = it->second;
                                if (face_of[L - 1][local] != face) {
                                    err = "block " + std::to_string(cb) + " has two fine regions on one side of a pencil";
                                    return false;
                                }
                            }
                            const int a = has[RO1[d]] ? (int)(f[RO1[d]] & 1) : 0;
                            const int q = has[RO2[d]] ? (int)(f[RO2[d]] & 1) : 0;
                            const int pos = 2 * a + q;
                            if (src_of[L - 1][4 * local + pos] != -1) {
                                err = "two fine faces restrict to one coarse face position";
                                return false;
                            }
                            if (F.out_slot[i].empty()) F.out_slot[i].assign(2 * np, -1);
                            const int slot = F.n_out++;
                            F.out_slot[i][side * np + i1 + (long long)b.n[o1] * i2] = slot;
                            src_of[L - 1][4 * local + pos] = slot;
                        }
            }
        // number the in slots level by level and fill the per-pencil tables
        const int need = 1 << (plan.eff_dim - 1);
        for (int Lc = 0; Lc < maxl; ++Lc) {
            F.in_level_beg[Lc] = (int)F.in_face.size();
            const int base = (int)F.in_face.size();
            for (size_t k = 0; k < face_of[Lc].size(); ++k) {
                int cnt = 0;
                for (int q = 0; q < 4; ++q) cnt += src_of[Lc][4 * k + q] >= 0;
                if (cnt != need) {
                    err = "a coarse face is covered by " + std::to_string(cnt) + " fine faces instead of " + std::to_string(need);
                    return false;
                }
            }
            F.in_face.insert(F.in_face.end(), face_of[Lc].begin(), face_of[Lc].end());
            F.src.insert(F.src.end(), src_of[Lc].begin(), src_of[Lc].end());
            for (const auto& kv : in_of[Lc]) {
                const int cb = kv.first.first;
                const LBlock& c = blocks[cb];
                const long long np = (long long)c.n[o1] * c.n[o2];
                if (F.in_slot[cb].empty()) F.in_slot[cb].assign(2 * np, -1);
                F.in_slot[cb][kv.first.second] = base + kv.second;
            }
        }
        F.in_level_beg[maxl] = (int)F.in_face.size();
    }

    // leaf cells: paint each refined block's coarse shadow into the next coarser level
    // (the same intersections are the restriction targets)
    plan.leaf.assign(nb, {});
    plan.leaf_cells.assign(nb, 0);
    plan.rbox_level_beg.assign(maxl + 2, 0);
    for (int i = 0; i < nb; ++i) plan.leaf_cells[i] = (long long)blocks[i].n[0] * blocks[i].n[1] * blocks[i].n[2];
    for (int L = 1; L <= maxl; ++L) {
        plan.rbox_level_beg[L] = (int)plan.rboxes.size();
        for (int fi : of_level[L]) {
            const LBlock& f = blocks[fi];
            long long lo[3], hi[3];
            for (int d = 0; d < 3; ++d) {
                lo[d] = has[d] ? f.off[d] / 2 : 0;
                hi[d] = has[d] ? (f.off[d] + f.n[d]) / 2 : 1;
            }
            for (int ci : of_level[L - 1]) {
                const LBlock& c = blocks[ci];
                long long a[3], e[3];
                bool ov = true;
                for (int d = 0; d < 3; ++d) {
                    a[d] = std::max(lo[d], c.off[d]);
                    e[d] = std::min(hi[d], c.off[d] + c.n[d]);
                    ov = ov && a[d] < e[d];
                }
                if (!ov) continue;
                RBox rb;
                rb.fb = fi;
                rb.cb = ci;
                for (int d = 0; d < 3; ++d) {
                    rb.lo[d] = (int)(a[d] - c.off[d]) + c.g[d];
                    rb.hi[d] = (int)(e[d] - c.off[d]) + c.g[d];
                    rb.flo[d] = has[d] ? (int)(2 * a[d] - f.off[d]) + f.g[d] : 0;
                }
                plan.rboxes.push_back(rb);
                std::vector<unsigned char>& m = plan.leaf[ci];
                if (m.empty()) m.assign((size_t)c.n[0] * c.n[1] * c.n[2], 1);
                for (long long z = a[2]; z < e[2]; ++z)
                    for (long long y = a[1]; y < e[1]; ++y)
                        for (long long x = a[0]; x < e[0]; ++x) {
                            unsigned char& v = m[(size_t)(((z - c.off[2]) * c.n[1] + (y - c.off[1])) * c.n[0] + (x - c.off[0]))];
                            if (v) {
                                v = 0;
                                --plan.leaf_cells[ci];
                            }
                        }
            }
        }
    }
    plan.rbox_level_beg[maxl + 1] = (int)plan.rboxes.size();
    return true;
}

bool build_fill_runs(const std::vector<LBlock>& blocks, const long long dom[3], int target, std::vector<PRun>& runs,
                     std::string& err)
{
    runs.clear();
    if (target < 0 || target >= (int)blocks.size()) {
        err = "no such block";
        return false;
    }
    const LBlock& b = blocks[target];
    const int L = b.level;
    if (L < 1) {
        err = "a base-level block has no coarser level to be filled from";
        return false;
    }
    bool has[3];
    for (int d = 0; d < 3; ++d) has[d] = dom[d] > 1;
    LevelIndex coarse;
    coarse.init(blocks, dom, L - 1);
    for (int i = 0; i < (int)blocks.size(); ++i)
        if (blocks[i].level == L - 1) coarse.add(i);
    for (int z = b.g[2]; z < b.g[2] + b.n[2]; ++z)
        for (int y = b.g[1]; y < b.g[1] + b.n[1]; ++y) {
            PRun run{};
            run.len = 0;
            for (int x = b.g[0]; x < b.g[0] + b.n[0]; ++x) {
                const int s[3] = {x, y, z};
                long long p[3];
                int par[3], cs[3];
                for (int d = 0; d < 3; ++d) {
                    const long long f = s[d] - b.g[d] + b.off[d];
                    p[d] = has[d] ? floordiv2(f) : 0;
                    par[d] = has[d] ? (int)(f - 2 * floordiv2(f)) : 0;
                }
                const int cb = coarse.owner(p);
                if (cb < 0) {
                    err = where(target, b) + " reaches outside its coarser level";
                    return false;
                }
                const LBlock& c = blocks[cb];
                for (int d = 0; d < 3; ++d) cs[d] = (int)(p[d] - c.off[d]) + c.g[d];
                const bool cont = run.len > 0 && cb == run.cb && cs[1] == run.cy && cs[2] == run.cz &&
                                  par[1] == run.py && par[2] == run.pz &&
                                  cs[0] == run.cx + ((run.px + run.len) >> 1) && par[0] == ((run.px + run.len) & 1);
                if (cont) {
                    ++run.len;
                    continue;
                }
                if (run.len > 0) runs.push_back(run);
                run = PRun{target, cb, x, y, z, 1, cs[0], cs[1], cs[2], par[0], par[1], par[2]};
            }
            if (run.len > 0) runs.push_back(run);
        }
    return true;
}

void build_partial_refresh(const std::vector<LBlock>& blocks, const LevelPlan& plan, const std::vector<XSeg>& segs,
                           int dir, int r, PartialRefresh& out)
{
    const int nb = (int)blocks.size();
    bool has[3];
    for (int d = 0; d < 3; ++d) has[d] = blocks[0].n[d] > 1;
    // per block: 0 not needed, 1 in a slab, 2 needed by a prolongation stencil only
    std::vector<std::vector<unsigned char>> need(nb);
    std::vector<int> ext(3 * nb);
    std::vector<char> extra(nb, 0);
    auto at = [&](int b, int x, int y, int z) -> unsigned char& {
        return need[b][((size_t)z * ext[3 * b + 1] + y) * ext[3 * b] + x];
    };
    for (int b = 0; b < nb; ++b) {
        const LBlock& B = blocks[b];
        for (int d = 0; d < 3; ++d) ext[3 * b + d] = B.n[d] + 2 * B.g[d];
        need[b].assign((size_t)ext[3 * b] * ext[3 * b + 1] * ext[3 * b + 2], 0);
        for (int side = 0; side < 2; ++side) {
            int lo[3], hi[3];
            for (int d = 0; d < 3; ++d) {
                lo[d] = B.g[d];
                hi[d] = B.g[d] + B.n[d];
            }
            lo[dir] = side == 0 ? B.g[dir] - 2 : B.g[dir] + B.n[dir];
            hi[dir] = lo[dir] + 2;
            for (int z = lo[2]; z < hi[2]; ++z)
                for (int y = lo[1]; y < hi[1]; ++y)
                    for (int x = lo[0]; x < hi[0]; ++x) at(b, x, y, z) = 1;
        }
    }
    // prolongation rows, finest level first: keep the needed pieces, mark their stencils' coarse cells
    out.runs.clear();
    out.run_level_beg.assign(plan.max_level + 2, 0);
    std::vector<std::vector<PRun>> by_level(plan.max_level + 1);
    for (int L = plan.max_level; L >= 1; --L) {
        for (long long q = plan.run_level_beg[L]; q < plan.run_level_beg[L + 1]; ++q) {
            const PRun& R = plan.runs[q];
            int i = 0;
            while (i < R.len) {
                if (!at(R.fb, R.fx + i, R.fy, R.fz)) {
                    ++i;
                    continue;
                }
                int e = i;
                while (e < R.len && at(R.fb, R.fx + e, R.fy, R.fz)) ++e;
                PRun p = R;
                p.fx = R.fx + i;
                p.len = e - i;
                p.px = (R.px + i) & 1;
                p.cx = R.cx + ((R.px + i) >> 1);
                by_level[L].push_back(p);
                const int rx = has[0] ? r : 0, ry = has[1] ? r : 0, rz = has[2] ? r : 0;
                const int x0 = p.cx - rx, x1 = R.cx + ((R.px + e - 1) >> 1) + rx;
                const int c = R.cb;
                for (int z = std::max(0, R.cz - rz); z <= std::min(ext[3 * c + 2] - 1, R.cz + rz); ++z)
                    for (int y = std::max(0, R.cy - ry); y <= std::min(ext[3 * c + 1] - 1, R.cy + ry); ++y)
                        for (int x = std::max(0, x0); x <= std::min(ext[3 * c] - 1, x1); ++x) {
                            unsigned char& m = at(c, x, y, z);
                            if (!m) {
                                m = 2;
                                extra[c] = 1;
                            }
                        }
                i = e;
            }
        }
    }
    for (int L = 1; L <= plan.max_level; ++L) {
        out.run_level_beg[L] = (long long)out.runs.size();
        out.runs.insert(out.runs.end(), by_level[L].begin(), by_level[L].end());
    }
    out.run_level_beg[plan.max_level + 1] = (long long)out.runs.size();
    // same-level segments: slab pieces as boxes, other needed cells as rows.
    // Along x the slab pieces take the whole guard depth: two-cell rows would
    // leave every memory sector half used, and the extra cells receive the
    // values a complete refresh gives them.
    auto slab = [&](int b, int side, int lo[3], int hi[3]) {
        const LBlock& B = blocks[b];
        for (int d = 0; d < 3; ++d) {
            lo[d] = B.g[d];
            hi[d] = B.g[d] + B.n[d];
        }
        const int w = dir == 0 ? B.g[0] : 2;
        lo[dir] = side == 0 ? B.g[dir] - w : B.g[dir] + B.n[dir];
        hi[dir] = lo[dir] + w;
    };
    auto in_slab = [&](int b, int x, int y, int z) {
        const int c[3] = {x, y, z};
        for (int side = 0; side < 2; ++side) {
            int lo[3], hi[3];
            slab(b, side, lo, hi);
            bool in = true;
            for (int d = 0; d < 3; ++d) in = in && c[d] >= lo[d] && c[d] < hi[d];
            if (in) return true;
        }
        return false;
    };
    out.segs.clear();
    for (const XSeg& s : segs) {
        for (int side = 0; side < 2; ++side) {
            XSeg p = s;
            int lo[3], hi[3];
            slab(s.dst, side, lo, hi);
            bool ok = true;
            for (int d = 0; d < 3; ++d) {
                p.lo[d] = std::max(s.lo[d], lo[d]);
                p.hi[d] = std::min(s.hi[d], hi[d]);
                ok = ok && p.lo[d] < p.hi[d];
            }
            if (ok) out.segs.push_back(p);
        }
        if (!extra[s.dst]) continue;
        auto closure_only = [&](int x, int y, int z) { return at(s.dst, x, y, z) == 2 && !in_slab(s.dst, x, y, z); };
        for (int z = s.lo[2]; z < s.hi[2]; ++z)
            for (int y = s.lo[1]; y < s.hi[1]; ++y) {
                int x = s.lo[0];
                while (x < s.hi[0]) {
                    if (!closure_only(x, y, z)) {
                        ++x;
                        continue;
                    }
                    int e = x;
                    while (e < s.hi[0] && closure_only(e, y, z)) ++e;
                    XSeg p = s;
                    p.lo[0] = x;
                    p.hi[0] = e;
                    p.lo[1] = y;
                    p.hi[1] = y + 1;
                    p.lo[2] = z;
                    p.hi[2] = z + 1;
                    out.segs.push_back(p);
                    x = e;
                }
            }
    }
}

}  // namespace pk
