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
