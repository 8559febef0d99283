// Host-side harness exposing the sweep's per-face and per-cell functions and
// their adjoints (piernik_b200/csrc/pk_adjoint.cuh) to the CPU tests, which
// check every vector-Jacobian product against central finite differences.
#include "../../piernik_b200/csrc/pk_adjoint.cuh"

using namespace pk;
using PhM = Phys<K_ION, K_NONE, K_NONE, true>;
using PhH = Phys<K_NEU, K_NONE, K_NONE, false>;
using PhM3 = Phys<K_ION, K_NEU, K_DST, true>;

static PhysParams params(double gamma, int lim, int limb)
{
    PhysParams pp{};
    for (int f = 0; f < 3; ++f) {
        pp.gam[f] = f == 2 ? -1.0 : (f == 1 ? 1.4 : gamma);
        pp.gam_1[f] = pp.gam[f] - 1.0;
    }
    pp.smalld = 1e-3;
    pp.smallei = 1e-4;
    pp.use_smalld = 1;
    pp.use_smallei = 1;
    pp.disallow_negatives = 1;
    pp.lim = lim;
    pp.limb = limb;
    return pp;
}

template <class PH>
static void riemann_f(const double* ql, const double* qr, double ch, double gamma, double* f)
{
    double a[PH::NV], b[PH::NV], o[PH::NV];
    for (int v = 0; v < PH::NV; ++v) { a[v] = ql[v]; b[v] = qr[v]; }
    PhysParams pp = params(gamma, 0, 0);
    riemann<PH>(a, b, ch, pp, o);
    for (int v = 0; v < PH::NV; ++v) f[v] = o[v];
}

template <class PH>
static void riemann_b(const double* ql, const double* qr, double ch, double gamma, const double* fb, double* gl, double* gr)
{
    double a[PH::NV], b[PH::NV], fbb[PH::NV], l[PH::NV], r[PH::NV];
    for (int v = 0; v < PH::NV; ++v) { a[v] = ql[v]; b[v] = qr[v]; fbb[v] = fb[v]; }
    PhysParams pp = params(gamma, 0, 0);
    riemann_adj<PH>(a, b, ch, pp, fbb, l, r);
    for (int v = 0; v < PH::NV; ++v) { gl[v] = l[v]; gr[v] = r[v]; }
}

template <class PH>
static void utoq_f(const double* u, double gamma, double* q)
{
    double a[PH::NV], o[PH::NV];
    for (int v = 0; v < PH::NV; ++v) a[v] = u[v];
    PhysParams pp = params(gamma, 0, 0);
    utoq<PH>(a, o, pp);
    for (int v = 0; v < PH::NV; ++v) q[v] = o[v];
}

template <class PH>
static void utoq_b(const double* u, double gamma, const double* qb, double* ub)
{
    double a[PH::NV], b[PH::NV], o[PH::NV];
    for (int v = 0; v < PH::NV; ++v) { a[v] = u[v]; b[v] = qb[v]; o[v] = 0.0; }
    PhysParams pp = params(gamma, 0, 0);
    utoq_adj<PH>(a, b, o, pp);
    for (int v = 0; v < PH::NV; ++v) ub[v] = o[v];
}

template <class PH>
static void floors_f(const double* u, double gamma, double* out, unsigned* rec2)
{
    double a[PH::NV];
    for (int v = 0; v < PH::NV; ++v) a[v] = u[v];
    PhysParams pp = params(gamma, 0, 0);
    unsigned st = 0;
    FloorRec r;
    floors_rec<PH>(a, pp, st, r);
    for (int v = 0; v < PH::NV; ++v) out[v] = a[v];
    rec2[0] = r.dn;
    rec2[1] = r.en;
}

template <class PH>
static void floors_b(const double* u, double gamma, const double* lb, double* out)
{
    double a[PH::NV], l[PH::NV];
    for (int v = 0; v < PH::NV; ++v) { a[v] = u[v]; l[v] = lb[v]; }
    PhysParams pp = params(gamma, 0, 0);
    unsigned st = 0;
    FloorRec r;
    floors_rec<PH>(a, pp, st, r);
    floors_adj<PH>(a, r, l);
    for (int v = 0; v < PH::NV; ++v) out[v] = l[v];
}

extern "C" {
int h_nv(int phys) { return phys == 0 ? PhH::NV : (phys == 1 ? PhM::NV : PhM3::NV); }

void h_riemann(int phys, const double* ql, const double* qr, double ch, double gamma, double* f)
{
    if (phys == 0) riemann_f<PhH>(ql, qr, ch, gamma, f);
    else if (phys == 1) riemann_f<PhM>(ql, qr, ch, gamma, f);
    else riemann_f<PhM3>(ql, qr, ch, gamma, f);
}
void h_riemann_adj(int phys, const double* ql, const double* qr, double ch, double gamma, const double* fb,
                   double* gl, double* gr)
{
    if (phys == 0) riemann_b<PhH>(ql, qr, ch, gamma, fb, gl, gr);
    else if (phys == 1) riemann_b<PhM>(ql, qr, ch, gamma, fb, gl, gr);
    else riemann_b<PhM3>(ql, qr, ch, gamma, fb, gl, gr);
}
void h_utoq(int phys, const double* u, double gamma, double* q)
{
    if (phys == 0) utoq_f<PhH>(u, gamma, q);
    else if (phys == 1) utoq_f<PhM>(u, gamma, q);
    else utoq_f<PhM3>(u, gamma, q);
}
void h_utoq_adj(int phys, const double* u, double gamma, const double* qb, double* ub)
{
    if (phys == 0) utoq_b<PhH>(u, gamma, qb, ub);
    else if (phys == 1) utoq_b<PhM>(u, gamma, qb, ub);
    else utoq_b<PhM3>(u, gamma, qb, ub);
}
void h_floors(int phys, const double* u, double gamma, double* out, unsigned* rec)
{
    if (phys == 0) floors_f<PhH>(u, gamma, out, rec);
    else if (phys == 1) floors_f<PhM>(u, gamma, out, rec);
    else floors_f<PhM3>(u, gamma, out, rec);
}
void h_floors_adj(int phys, const double* u, double gamma, const double* lb, double* out)
{
    if (phys == 0) floors_b<PhH>(u, gamma, lb, out);
    else if (phys == 1) floors_b<PhM>(u, gamma, lb, out);
    else floors_b<PhM3>(u, gamma, lb, out);
}
double h_slope(int lim, double dl, double dr) { return slope_interior(lim, dl, dr); }
void h_slope_adj(int lim, double dl, double dr, double sb, double* dlb, double* drb) { slope_adj(lim, dl, dr, sb, *dlb, *drb); }
}
