// pk_device.cuh -- per-cell and per-interface FP64 physics of the split sweep.
//
// Device restatement of PIERNIK's RIEMANN_SPLIT building blocks.  Every
// expression keeps the reference's evaluation order so that, compiled with
// --fmad=false (no contraction) and IEEE double division/sqrt, results are
// bit-identical to the Fortran (gfortran -O2, SSE2, no FMA) arithmetic:
//   utoq                 src/scheme/Riemann_Solver/interpolations.F90:69-106
//   limiters             src/scheme/Riemann_Solver/fluxlimiters.F90:109-216
//   linear               src/scheme/Riemann_Solver/interpolations.F90:170-204
//   riemann_hlld (+GLM)  src/scheme/Riemann_Solver/hlld.F90:161-609
//   riemann_hlld_u       src/scheme/Riemann_Solver/hlld.F90:615-841
//   internal_sources     src/fluids/sources.F90:151-244 (adds +0: -0.0 -> +0.0)
//   care_for_positives   src/fluids/sources.F90:299-433
//   ion_cs/neu_cs        src/fluids/ionized/initionized.F90:89-145,
//                        src/fluids/neutral/initneutral.F90:82-109
//
// A cell state is a register array in *swept* order: for each fluid
// [dn, m_n, m_t1, m_t2, (en)], then [B_n, B_t1, B_t2, psi] when magnetised,
// where (n, t1, t2) = (x,y,z), (y,x,z), (z,y,x) for sweeps along x, y, z
// (iarr_all_swp, fluids/fluidtypes.F90:318-320; iarr_mag_swp,
// fluids/fluidindex.F90:190-192).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#define PK_DEV __device__ __forceinline__
#define PK_HD __host__ __device__ __forceinline__
// physics functions compile for the host too (unit tests of the adjoints)
#define PK_PHYS __host__ __device__ __forceinline__

namespace pk {

enum FluidKind { K_ION = 0, K_NEU = 1, K_DST = 2, K_NONE = 3 };
enum Limiter { L_VANLEER = 0, L_MINMOD = 1, L_MONCEN = 2, L_SUPERBEE = 3 };

// -------------------------------------------------------------------------
// Fortran intrinsics
// -------------------------------------------------------------------------

// SPACING(x) for real(8): 2**max(exponent(x)-53, -1022), TINY(x) at zero.
PK_PHYS unsigned long long f_bits(double x)
{
#ifdef __CUDA_ARCH__
    return (unsigned long long)__double_as_longlong(x);
#else
    unsigned long long b;
    memcpy(&b, &x, sizeof b);
    return b;
#endif
}
PK_PHYS double f_from_bits(unsigned long long b)
{
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
#endif
}
PK_PHYS double f_spacing(double x)
{
    const unsigned long long bits = f_bits(x);
    const int be = (int)((bits >> 52) & 0x7ffu);
    if (be == 0x7ff) return f_from_bits(0x7ff8000000000000ULL);
    if (be >= 53) return f_from_bits((unsigned long long)(be - 52) << 52);
    return 2.2250738585072014e-308;
}
PK_PHYS double f_sign1(double x) { return copysign(1.0, x); }
PK_PHYS double f_min(double a, double b) { return (b < a) ? b : a; }
PK_PHYS double f_max(double a, double b) { return (b > a) ? b : a; }

// -------------------------------------------------------------------------
// Compile-time description of the fluid set (flind order: ion, neu, dst)
// -------------------------------------------------------------------------

template <int K0, int K1, int K2, bool MAG>
struct Phys {
    PK_HD static constexpr int kind(int f) { return f == 0 ? K0 : (f == 1 ? K1 : K2); }
    static constexpr int NFL = (K0 != K_NONE) + (K1 != K_NONE) + (K2 != K_NONE);
    static constexpr bool MHD = MAG;
    PK_HD static constexpr int ncomp(int k) { return k == K_NONE ? 0 : (k == K_DST ? 4 : 5); }
    PK_HD static constexpr int beg(int f) { return f == 0 ? 0 : (f == 1 ? ncomp(K0) : ncomp(K0) + ncomp(K1)); }
    static constexpr int NVF = ncomp(K0) + ncomp(K1) + ncomp(K2);   // fluid components
    static constexpr int IB = NVF;                                 // first B component
    static constexpr int NV = NVF + (MAG ? 4 : 0);                 // with Bx,By,Bz,psi
    PK_HD static constexpr bool has_en(int f) { return kind(f) != K_DST; }
    PK_HD static constexpr bool magn(int f) { return MAG && kind(f) == K_ION; }
};

struct PhysParams {
    double gam[3];      // adiabatic index per fluid (dust: -1)
    double gam_1[3];    // gam - 1
    double rgam_1[3];   // 1 / (gam - 1), 1 / gam: the tolerance-mode kernels multiply by these
    double rgam[3];
    double smalld, smallei;
    int use_smalld, use_smallei, disallow_negatives;
    int lim, limb;      // flimiter, blimiter
    int weno3;          // interpol_str = 'weno3': WENO3 face states instead of limited linear ones
    double w_epsilon;   // WENO3 weight regulariser (global.F90:255)
};

// status bits written by kernels (never traps)
enum StatusBits : unsigned {
    ST_DN_NEGATIVE = 1u,   // dn_negative (sources.F90:349-350)
    ST_EI_NEGATIVE = 2u,   // ei_negative (sources.F90:422)
};

// -------------------------------------------------------------------------
// utoq: conservative -> primitive, one cell (interpolations.F90:69-106)
// -------------------------------------------------------------------------
template <class PH>
PK_PHYS void utoq(const double (&u)[PH::NV], double (&q)[PH::NV], const PhysParams& pp)
{
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {
        const int b = PH::beg(f);
        const double dn = u[b], mx = u[b + 1], my = u[b + 2], mz = u[b + 3];
        q[b] = dn;
        q[b + 1] = mx / dn;
        q[b + 2] = my / dn;
        q[b + 3] = mz / dn;
        if (PH::has_en(f)) {
            const double ek = (0.5 * ((mx * mx + my * my) + mz * mz)) / dn;
            double p = pp.gam_1[f] * (u[b + 4] - ek);
            if (PH::magn(f)) {
                const double bx = u[PH::IB], by = u[PH::IB + 1], bz = u[PH::IB + 2];
                p = p - (0.5 * pp.gam_1[f]) * ((bx * bx + by * by) + bz * bz);
            }
            q[b + 4] = p;
        }
    }
    if (PH::MHD) {
#pragma unroll
        for (int c = 0; c < 4; ++c) q[PH::IB + c] = u[PH::IB + c];   // B and psi go to blimiter as they are
    }
}

// -------------------------------------------------------------------------
// Limited slopes.  Interior cell: dl = q(i)-q(i-1), dr = q(i+1)-q(i).
// Pencil end cells use the reference's one-sided rules (dl = dr, vanleer 0).
// -------------------------------------------------------------------------
PK_PHYS double slope_interior(int lim, double dl, double dr)
{
    if (lim == L_VANLEER) {                       // fluxlimiters.F90:122-133
        const double dcen = dl * dr;
        return (dcen > 0.0) ? (2.0 * dcen) / (dl + dr) : 0.0;
    }
    const double s = f_sign1(dl) + f_sign1(dr);
    if (lim == L_MINMOD) return (s * f_min(fabs(dl), fabs(dr))) * 0.5;                        // :158
    if (lim == L_MONCEN) return (s * f_min(f_min(2.0 * fabs(dl), 2.0 * fabs(dr)), 0.5 * fabs(dl + dr))) * 0.5;  // :185
    const double m = (fabs(dl) > fabs(dr)) ? f_min(fabs(dl), fabs(2.0 * dr)) : f_min(fabs(2.0 * dl), fabs(dr)); // :211-212
    return (s * 0.5) * m;
}

// WENO3 face states of cell c from q(c-1), q(c), q(c+1) (interpolations.F90:
// 210-337, Yamaleev & Carpenter 2009): ql = the left state of the right face,
// qr = the right state of the left face, in the reference's operation order.
PK_PHYS void weno3_faces(double qm, double qc, double qp, double weps, double& ql, double& qr)
{
    const double d0 = 2.0 / 3.0, d1 = 1.0 / 3.0;                              // Eq. 19 (twot, onet)
    const double b0 = (qp - qc) * (qp - qc);                                    // Eq. 20
    const double b1 = (qc - qm) * (qc - qm);
    const double tt = ((qp - 2.0 * qc) + qm);                                   // Eq. 22
    const double tau = tt * tt;
    double a0 = d0 * (1.0 + tau / (weps + b0));                                 // Eq. 21
    double a1 = d1 * (1.0 + tau / (weps + b1));
    double w0 = a0 / (a0 + a1), w1 = a1 / (a0 + a1);                            // Eq. 18
    double f0 = 0.5 * (qc + qp), f1 = 0.5 * (-qm + 3.0 * qc);                   // Eq. 15
    ql = w0 * f0 + w1 * f1;                                                     // Eq. 14
    a0 = d0 * (1.0 + tau / (weps + b1));                                        // the mirrored stencil
    a1 = d1 * (1.0 + tau / (weps + b0));
    w0 = a0 / (a0 + a1);
    w1 = a1 / (a0 + a1);
    f0 = 0.5 * (qc + qm);
    f1 = 0.5 * (-qp + 3.0 * qc);
    qr = w0 * f0 + w1 * f1;
}

PK_PHYS double slope_end(int lim, double d)
{
    if (lim == L_VANLEER) return 0.0;             // "sanitizing endpoints" (:119-120)
    return slope_interior(lim, d, d);
}

// -------------------------------------------------------------------------
// Riemann solvers on one interface.  ql/qr: primitive swept states of one
// fluid; bl/br: swept B (zero for unmagnetised fluids); f: fluid fluxes;
// bf: transverse B fluxes.
// -------------------------------------------------------------------------

// Physical flux of one side (hlld.F90:296-308): fluid part f[0..nc) and the
// transverse B fluxes bf[1..2].  Computed where needed so that neither side's
// flux is held in registers through the star-state algebra.
PK_PHYS void side_flux(bool has_energy, const double* u, const double* b, double pr, double en, double* f)
{
    f[0] = u[0] * u[1];
    f[1] = ((u[0] * (u[1] * u[1])) + pr) - (b[0] * b[0]);
    f[2] = ((u[0] * u[2]) * u[1]) - (b[0] * b[1]);
    f[3] = ((u[0] * u[3]) * u[1]) - (b[0] * b[2]);
    if (has_energy) f[4] = ((en + pr) * u[1]) - (b[0] * ((u[1] * b[0] + u[2] * b[1]) + u[3] * b[2]));
}

PK_PHYS double side_bflux(const double* u, const double* b, int c)
{
    return (b[c] * u[1]) - (b[0] * u[1 + c]);     // b_cclf(ydim:zdim), hlld.F90:301,309
}

// [ u(idn), u(idn)*u(imx:imz), en ] of one side
PK_PHYS double side_cons(const double* u, double en, int c)
{
    return c == 0 ? u[0] : (c == 4 ? en : u[0] * u[c]);
}

PK_PHYS void hlld_iface(bool has_energy, double gamma, const double* ul, const double* ur, const double* bl,
                       const double* br, double* f, double* bf)
{
    const int nc = has_energy ? 5 : 4;
    double prl, prr, c_fastm;
    double enl = 1.7976931348623157e308, enr = 1.7976931348623157e308, ue = 0.0;

    const double magprl = 0.5 * ((bl[0] * bl[0] + bl[1] * bl[1]) + bl[2] * bl[2]);   // hlld.F90:239-240
    const double magprr = 0.5 * ((br[0] * br[0] + br[1] * br[1]) + br[2] * br[2]);
    if (gamma < 0.0) {                                                               // :245-249
        prl = 0.0;
        prr = 0.0;
        c_fastm = 0.0;
    } else {
        prl = ul[4] + magprl;                                                         // :258-259
        prr = ur[4] + magprr;
        const double bbl = (bl[0] * bl[0] + bl[1] * bl[1]) + bl[2] * bl[2];
        const double bbr = (br[0] * br[0] + br[1] * br[1]) + br[2] * br[2];
        enl = ((ul[4] / (gamma - 1.0)) + ((0.5 * ul[0]) * ((ul[1] * ul[1] + ul[2] * ul[2]) + ul[3] * ul[3]))) + (0.5 * bbl);
        enr = ((ur[4] / (gamma - 1.0)) + ((0.5 * ur[0]) * ((ur[1] * ur[1] + ur[2] * ur[2]) + ur[3] * ur[3]))) + (0.5 * bbr);
        const double gampr_l = gamma * ul[4];
        const double gampr_r = gamma * ur[4];
        const double al = gampr_l + bbl, ar = gampr_r + bbr;                         // :272-274
        const double cl = (al + sqrt(al * al - ((4.0 * gampr_l) * (bl[0] * bl[0])))) / ul[0];
        const double cr = (ar + sqrt(ar * ar - ((4.0 * gampr_r) * (br[0] * br[0])))) / ur[0];
        c_fastm = sqrt(0.5 * f_max(cl, cr));
    }
    const double sl = f_min(ul[1], ur[1]) - c_fastm;                                // :291-292
    const double sr = f_max(ul[1], ur[1]) + c_fastm;

    if (sl >= 0.0 || sr <= 0.0) {                                                    // :312-319
        const bool left = sl >= 0.0;
        const double* u = left ? ul : ur;
        const double* b = left ? bl : br;
        side_flux(has_energy, u, b, left ? prl : prr, left ? enl : enr, f);
        bf[0] = side_bflux(u, b, 1);
        bf[1] = side_bflux(u, b, 2);
        return;
    }

    double sm;                                                                       // :323-330
    {
        const double auxr = (sr - ur[1]) * ur[0];
        const double auxl = (sl - ul[1]) * ul[0];
        if (fabs(auxr - auxl) < f_spacing(auxr + auxl)) sm = (sl + sr) / 2.0;
        else sm = ((auxr * ur[1] - prr) - (auxl * ul[1] - prl)) / (auxr - auxl);
    }
    const double slsm = sl - sm, srsm = sr - sm;                                    // :334-340
    const double slvxl = sl - ul[1], srvxr = sr - ur[1];
    const double srmsl = sr - sl;
    const double dn_l = ul[0] * slvxl, dn_r = ur[0] * srvxr;                        // :344-347
    const double b_lr = bl[0] * br[0];
    const double b_lrgam = b_lr / gamma;
    const double prt_star = 0.5 * ((prl + dn_l * (sm - ul[1])) + (prr + dn_r * (sm - ur[1])));

    // transverse B of the star states, with the HLL fallback (:362-378)
    double bsl[3], bsr[3];
    bsl[0] = bl[0];
    bsr[0] = br[0];
    {
        const double bclf1 = side_bflux(ul, bl, 1), bclf2 = side_bflux(ul, bl, 2);
        const double bcrf1 = side_bflux(ur, br, 1), bcrf2 = side_bflux(ur, br, 2);
        double coeff_1 = dn_l * slsm - b_lr;
        if (has_energy) ue = ul[4];
        if ((fabs(coeff_1) > f_spacing(b_lr)) && b_lrgam <= ue) {
            const double a = dn_l * slvxl - b_lr;
            bsl[1] = (bl[1] * a) / coeff_1;
            bsl[2] = (bl[2] * a) / coeff_1;
        } else {
            bsl[1] = ((sr * br[1] - sl * bl[1]) - (bcrf1 - bclf1)) / srmsl;
            bsl[2] = ((sr * br[2] - sl * bl[2]) - (bcrf2 - bclf2)) / srmsl;
        }
        coeff_1 = dn_r * srsm - b_lr;
        if (has_energy) ue = ur[4];
        if ((fabs(coeff_1) > f_spacing(b_lr)) && b_lrgam <= ue) {
            const double a = dn_r * srvxr - b_lr;
            bsr[1] = (br[1] * a) / coeff_1;
            bsr[2] = (br[2] * a) / coeff_1;
        } else {
            bsr[1] = ((sr * br[1] - sl * bl[1]) - (bcrf1 - bclf1)) / srmsl;
            bsr[2] = ((sr * br[2] - sl * bl[2]) - (bcrf2 - bclf2)) / srmsl;
        }
    }
    double vsl[3], vsr[3];                                                           // :354-355, :381-382
    vsl[0] = sm;
    vsr[0] = sm;
    {
        const double bxl_dnl = bl[0] / dn_l, bxr_dnr = br[0] / dn_r;
        vsl[1] = ul[2] + (bxl_dnl * (bl[1] - bsl[1]));
        vsl[2] = ul[3] + (bxl_dnl * (bl[2] - bsl[2]));
        vsr[1] = ur[2] + (bxr_dnr * (br[1] - bsr[1]));
        vsr[2] = ur[3] + (bxr_dnr * (br[2] - bsr[2]));
    }
    const double vb_starl = (vsl[0] * bsl[0] + vsl[1] * bsl[1]) + vsl[2] * bsl[2];  // :388-389
    const double vb_starr = (vsr[0] * bsr[0] + vsr[1] * bsr[1]) + vsr[2] * bsr[2];

    double usl[5], usr[5];                                                           // :393-404
    usl[0] = dn_l / slsm;
    usr[0] = dn_r / srsm;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        usl[1 + c] = usl[0] * vsl[c];
        usr[1 + c] = usr[0] * vsr[c];
    }
    if (has_energy) {
        const double vb_l = (ul[1] * bl[0] + ul[2] * bl[1]) + ul[3] * bl[2];
        const double vb_r = (ur[1] * br[0] + ur[2] * br[1]) + ur[3] * br[2];
        usl[4] = ((((slvxl * enl) - (prl * ul[1])) + (prt_star * sm)) + (bl[0] * (vb_l - vb_starl))) / slsm;
        usr[4] = ((((srvxr * enr) - (prr * ur[1])) + (prt_star * sm)) + (br[0] * (vb_r - vb_starr))) / srsm;
    }

    // flux through the outer (star) state of one side: fl + s*(u_star - u) (Eq. 64)
    auto star_flux = [&](bool left, double* out, double* bout) {
        const double* u = left ? ul : ur;
        const double* b = left ? bl : br;
        const double* us = left ? usl : usr;
        const double* bs = left ? bsl : bsr;
        const double s = left ? sl : sr;
        const double en = left ? enl : enr;
        double fs[5];
        side_flux(has_energy, u, b, left ? prl : prr, en, fs);
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) out[c] = fs[c] + s * (us[c] - side_cons(u, en, c));
        bout[0] = side_bflux(u, b, 1) + s * (bs[1] - b[1]);
        bout[1] = side_bflux(u, b, 2) + s * (bs[2] - b[2]);
    };

    if (fabs(bl[0]) > 0.0) {                                                         // :410
        const double dn_lsqt = sqrt(usl[0]);                                        // :414-418
        const double dn_rsqt = sqrt(usr[0]);
        const double alfven_l = sm - fabs(bl[0]) / dn_lsqt;
        const double alfven_r = sm + fabs(br[0]) / dn_rsqt;
        if (alfven_l > 0.0 || alfven_r < 0.0) {                                      // :422-448
            star_flux(alfven_l > 0.0, f, bf);
            return;
        }
        const double b_sig = (bl[0] >= 0.0) ? 1.0 : -1.0;                            // :452-456
        const double add_dnsq = dn_lsqt + dn_rsqt;                                   // :460-461
        const double mul_dnsq = dn_lsqt * dn_rsqt;
        double v2[3], b2[3];                                                         // :465-470
        v2[0] = sm;
        v2[1] = ((dn_lsqt * vsl[1] + dn_rsqt * vsr[1]) + b_sig * (bsr[1] - bsl[1])) / add_dnsq;
        v2[2] = ((dn_lsqt * vsl[2] + dn_rsqt * vsr[2]) + b_sig * (bsr[2] - bsl[2])) / add_dnsq;
        b2[0] = 0.5 * (bl[0] + br[0]);
        const double bsm = b_sig * mul_dnsq;
        b2[1] = ((dn_lsqt * bsr[1] + dn_rsqt * bsl[1]) + bsm * (vsr[1] - vsl[1])) / add_dnsq;
        b2[2] = ((dn_lsqt * bsr[2] + dn_rsqt * bsl[2]) + bsm * (vsr[2] - vsl[2])) / add_dnsq;
        const double vb_2star = (v2[0] * b2[0] + v2[1] * b2[1]) + v2[2] * b2[2];   // :474

        // flux through the Alfven (2-star) state of one side (Eq. 65, :478-522)
        auto alfven_flux = [&](bool left, double* out, double* bout) {
            const double* u = left ? ul : ur;
            const double* b = left ? bl : br;
            const double* us = left ? usl : usr;
            const double* bs = left ? bsl : bsr;
            const double s = left ? sl : sr;
            const double en = left ? enl : enr;
            const double a = left ? alfven_l : alfven_r;
            double u2[5], fs[5];
            u2[0] = us[0];
#pragma unroll
            for (int c = 0; c < 3; ++c) u2[1 + c] = us[0] * v2[c];
            if (has_energy)
                u2[4] = left ? us[4] - (b_sig * dn_lsqt) * (vb_starl - vb_2star)
                             : us[4] + (b_sig * dn_rsqt) * (vb_starr - vb_2star);
            side_flux(has_energy, u, b, left ? prl : prr, en, fs);
#pragma unroll
            for (int c = 0; c < 5; ++c)
                if (c < nc) out[c] = ((fs[c] + a * u2[c]) - (a - s) * us[c]) - s * side_cons(u, en, c);
#pragma unroll
            for (int c = 1; c < 3; ++c)
                bout[c - 1] = ((side_bflux(u, b, c) + a * b2[c]) - (a - s) * bs[c]) - s * b[c];
        };
        if (sm > 0.0 || sm < 0.0) {                                                  // :496-522
            alfven_flux(sm > 0.0, f, bf);
        } else {                                                                     // :524-544
            double fl2[5], fr2[5], bl2[2], br2[2];
            alfven_flux(true, fl2, bl2);
            alfven_flux(false, fr2, br2);
#pragma unroll
            for (int c = 0; c < 5; ++c)
                if (c < nc) f[c] = 0.5 * (fl2[c] + fr2[c]);
            bf[0] = 0.5 * (bl2[0] + br2[0]);
            bf[1] = 0.5 * (bl2[1] + br2[1]);
        }
    } else {                                                                         // :548-599, B_x = 0
        if (sm > 0.0 || sm < 0.0) {
            star_flux(sm > 0.0, f, bf);
        } else {
            // half * (fl + sl*(usl-ucl) + fr + sr*(usr-ucr)), summed left to right
            double fsl[5], fsr[5];
            side_flux(has_energy, ul, bl, prl, enl, fsl);
            side_flux(has_energy, ur, br, prr, enr, fsr);
#pragma unroll
            for (int c = 0; c < 5; ++c)
                if (c < nc)
                    f[c] = 0.5 * (((fsl[c] + sl * (usl[c] - side_cons(ul, enl, c))) + fsr[c]) +
                                  sr * (usr[c] - side_cons(ur, enr, c)));
#pragma unroll
            for (int c = 1; c < 3; ++c)
                bf[c - 1] = 0.5 * (((side_bflux(ul, bl, c) + sl * (bsl[c] - bl[c])) + side_bflux(ur, br, c)) +
                                   sr * (bsr[c] - br[c]));
        }
    }
}

PK_PHYS void hllc_iface(bool has_energy, double gamma, const double* ul, const double* ur, double* f)
{
    double fl[5], fr[5], usl[5], usr[5];
    double prl, prr, c_fastm;
    double enl = 1.7976931348623157e308, enr = 1.7976931348623157e308;
    const int nc = has_energy ? 5 : 4;
    if (gamma < 0.0) {                                                               // hlld.F90:673-677
        prl = 0.0;
        prr = 0.0;
        c_fastm = 0.0;
    } else {                                                                         // :689-703
        prl = ul[4];
        prr = ur[4];
        enl = (ul[4] / (gamma - 1.0)) + ((0.5 * ul[0]) * ((ul[1] * ul[1] + ul[2] * ul[2]) + ul[3] * ul[3]));
        enr = (ur[4] / (gamma - 1.0)) + ((0.5 * ur[0]) * ((ur[1] * ur[1] + ur[2] * ur[2]) + ur[3] * ur[3]));
        const double gampr_l = gamma * ul[4];
        const double gampr_r = gamma * ur[4];
        c_fastm = sqrt(f_max(gampr_l / ul[0], gampr_r / ur[0]));
    }
    const double sl = f_min(ul[1], ur[1]) - c_fastm;                                // :719-720
    const double sr = f_max(ul[1], ur[1]) + c_fastm;
    fl[0] = ul[0] * ul[1];                                                           // :724-734
    fl[1] = (ul[0] * (ul[1] * ul[1])) + prl;
    fl[2] = (ul[0] * ul[2]) * ul[1];
    fl[3] = (ul[0] * ul[3]) * ul[1];
    if (has_energy) fl[4] = (enl + prl) * ul[1];
    fr[0] = ur[0] * ur[1];
    fr[1] = (ur[0] * (ur[1] * ur[1])) + prr;
    fr[2] = (ur[0] * ur[2]) * ur[1];
    fr[3] = (ur[0] * ur[3]) * ur[1];
    if (has_energy) fr[4] = (enr + prr) * ur[1];
    if (sl >= 0.0) {                                                                 // :738-743
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) f[c] = fl[c];
        return;
    }
    if (sr <= 0.0) {
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) f[c] = fr[c];
        return;
    }
    double sm;                                                                       // :747-754
    {
        const double auxr = (sr - ur[1]) * ur[0];
        const double auxl = (sl - ul[1]) * ul[0];
        if (fabs(auxr - auxl) < f_spacing(auxr + auxl)) sm = (sl + sr) / 2.0;
        else sm = ((auxr * ur[1] - prr) - (auxl * ul[1] - prl)) / (auxr - auxl);
    }
    const double slvxl = sl - ul[1], srvxr = sr - ur[1];                            // :758-764
    const double dn_l = ul[0] * slvxl, dn_r = ur[0] * srvxr;
    const double prt_star = 0.5 * ((prl + dn_l * (sm - ul[1])) + (prr + dn_r * (sm - ur[1])));
    if (sm >= 0.0) {                                                                 // :771-784
        const double slsm = sl - sm;
        usl[0] = dn_l / slsm;
        usl[1] = usl[0] * sm;
        usl[2] = usl[0] * ul[2];
        usl[3] = usl[0] * ul[3];
        if (has_energy) usl[4] = (((slvxl * enl) - (prl * ul[1])) + (prt_star * sm)) / slsm;
    }
    if (sm <= 0.0) {                                                                 // :786-796
        const double srsm = sr - sm;
        usr[0] = dn_r / srsm;
        usr[1] = usr[0] * sm;
        usr[2] = usr[0] * ur[2];
        usr[3] = usr[0] * ur[3];
        if (has_energy) usr[4] = (((srvxr * enr) - (prr * ur[1])) + (prt_star * sm)) / srsm;
    }
    double ucl[5], ucr[5];
    ucl[0] = ul[0];
    ucr[0] = ur[0];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        ucl[1 + c] = ul[0] * ul[1 + c];
        ucr[1 + c] = ur[0] * ur[1 + c];
    }
    ucl[4] = enl;
    ucr[4] = enr;
    if (sm > 0.0) {                                                                  // :798-806
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) f[c] = fl[c] + sl * (usl[c] - ucl[c]);
    } else if (sm < 0.0) {                                                           // :808-815
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) f[c] = fr[c] + sr * (usr[c] - ucr[c]);
    } else {                                                                         // :817-829
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) f[c] = 0.5 * (((fl[c] + sl * (usl[c] - ucl[c])) + fr[c]) + sr * (usr[c] - ucr[c]));
    }
}

// riemann_wrap / riemann_wrap_u (hlld.F90:62-155) for one interface of the
// whole state: fluid fluxes, then (MHD) fluxes of Bx, By, Bz, psi.
template <class PH>
PK_PHYS void riemann(const double (&ql)[PH::NV], const double (&qr)[PH::NV], double ch, const PhysParams& pp,
                    double (&fx)[PH::NV])
{
    if (PH::MHD) {
        const double bxl = ql[PH::IB], bxr = qr[PH::IB], psl = ql[PH::IB + 3], psr = qr[PH::IB + 3];
        fx[PH::IB + 3] = ((ch * ch) * 0.5) * ((bxr + bxl) - (psr - psl) / ch);       // hlld.F90:229 (Dedner eq. 42)
        fx[PH::IB] = 0.5 * ((psr + psl) - ch * (bxr - bxl));                          // :230
    }
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {
        const int b = PH::beg(f);
        double fv[5];
        if (PH::MHD) {
            double blv[3] = {0.0, 0.0, 0.0}, brv[3] = {0.0, 0.0, 0.0}, bf[2];
            if (PH::magn(f)) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    blv[c] = ql[PH::IB + c];
                    brv[c] = qr[PH::IB + c];
                }
            }
            hlld_iface(PH::has_en(f), pp.gam[f], &ql[b], &qr[b], blv, brv, fv, bf);
            if (PH::magn(f)) {
                fx[PH::IB + 1] = bf[0];
                fx[PH::IB + 2] = bf[1];
            }
        } else {
            hllc_iface(PH::has_en(f), pp.gam[f], &ql[b], &qr[b], fv);
        }
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < PH::ncomp(PH::kind(f))) fx[b + c] = fv[c];
    }
}

// The same for a tile in shared memory: left states at L[v*PT + me], right
// states at R[v*PT + me + st], fluxes written to F[v*PT + me].  Each fluid's
// states are loaded just before its solve, so the register footprint does not
// grow with the number of fluids.
template <class PH>
PK_DEV void riemann_tile(const double* __restrict__ L, const double* __restrict__ R, double* __restrict__ F, int PT,
                         int me, int st, double ch, const PhysParams& pp)
{
    double blv[3] = {0.0, 0.0, 0.0}, brv[3] = {0.0, 0.0, 0.0};
    if (PH::MHD) {
        const double bxl = L[PH::IB * PT + me], bxr = R[PH::IB * PT + me + st];
        const double psl = L[(PH::IB + 3) * PT + me], psr = R[(PH::IB + 3) * PT + me + st];
        F[(PH::IB + 3) * PT + me] = ((ch * ch) * 0.5) * ((bxr + bxl) - (psr - psl) / ch);   // hlld.F90:229
        F[PH::IB * PT + me] = 0.5 * ((psr + psl) - ch * (bxr - bxl));                      // :230
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            blv[c] = L[(PH::IB + c) * PT + me];
            brv[c] = R[(PH::IB + c) * PT + me + st];
        }
    }
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {
        const int b = PH::beg(f);
        const int nc = PH::ncomp(PH::kind(f));
        double ul[5] = {0, 0, 0, 0, 0}, ur[5] = {0, 0, 0, 0, 0}, fv[5];
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) {
                ul[c] = L[(b + c) * PT + me];
                ur[c] = R[(b + c) * PT + me + st];
            }
        if (PH::MHD) {
            const double zero[3] = {0.0, 0.0, 0.0};
            double bf[2];
            hlld_iface(PH::has_en(f), pp.gam[f], ul, ur, PH::magn(f) ? blv : zero, PH::magn(f) ? brv : zero, fv, bf);
            if (PH::magn(f)) {
                F[(PH::IB + 1) * PT + me] = bf[0];
                F[(PH::IB + 2) * PT + me] = bf[1];
            }
        } else {
            hllc_iface(PH::has_en(f), pp.gam[f], ul, ur, fv);
        }
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) F[(b + c) * PT + me] = fv[c];
    }
}

// internal_sources (+0 added to every fluid component) and care_for_positives
// on one updated cell; B used for emag is the updated one (b1).
template <class PH>
PK_PHYS void sources_and_floors(double (&u)[PH::NV], const PhysParams& pp, unsigned& status)
{
#pragma unroll
    for (int c = 0; c < PH::NVF; ++c) u[c] = u[c] + 0.0;
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {                                   // limit_minimal_density
        const int b = PH::beg(f);
        if (u[b] < 0.0) status |= ST_DN_NEGATIVE;
        if (pp.use_smalld) u[b] = f_max(u[b], pp.smalld);
    }
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {                                   // limit_minimal_intener
        if (!PH::has_en(f)) continue;
        const int b = PH::beg(f);
        const double kin = (0.5 * ((u[b + 1] * u[b + 1] + u[b + 2] * u[b + 2]) + u[b + 3] * u[b + 3])) / u[b];
        double mag = 0.0, eint;
        if (PH::magn(f)) {
            const double bx = u[PH::IB], by = u[PH::IB + 1], bz = u[PH::IB + 2];
            mag = 0.5 * ((bx * bx + by * by) + bz * bz);
            eint = (u[b + 4] - kin) - mag;
        } else {
            eint = u[b + 4] - kin;
        }
        if (pp.disallow_negatives && eint < 0.0) status |= ST_EI_NEGATIVE;
        if (pp.use_smallei) eint = f_max(eint, pp.smallei);
        double e = eint + kin;
        if (PH::magn(f)) e = e + mag;
        u[b + 4] = e;
    }
}

// ---------------------------------------------------------------------------
// internal_sources + care_for_positives with a record of the floors taken
// ---------------------------------------------------------------------------
struct FloorRec {
    unsigned dn;   // bit f: the density floor of fluid f clipped
    unsigned en;   // bit f: the internal-energy floor of fluid f clipped
};

template <class PH>
PK_PHYS void floors_rec(double (&u)[PH::NV], const PhysParams& pp, unsigned& status, FloorRec& rec)
{
    rec.dn = 0;
    rec.en = 0;
#pragma unroll
    for (int c = 0; c < PH::NVF; ++c) u[c] = u[c] + 0.0;
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {
        const int b = PH::beg(f);
        if (u[b] < 0.0) status |= ST_DN_NEGATIVE;
        if (pp.use_smalld) {
            if (pp.smalld > u[b]) rec.dn |= 1u << f;
            u[b] = f_max(u[b], pp.smalld);
        }
    }
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {
        if (!PH::has_en(f)) continue;
        const int b = PH::beg(f);
        const double kin = (0.5 * ((u[b + 1] * u[b + 1] + u[b + 2] * u[b + 2]) + u[b + 3] * u[b + 3])) / u[b];
        double mag = 0.0, eint;
        if (PH::magn(f)) {
            const double bx = u[PH::IB], by = u[PH::IB + 1], bz = u[PH::IB + 2];
            mag = 0.5 * ((bx * bx + by * by) + bz * bz);
            eint = (u[b + 4] - kin) - mag;
        } else {
            eint = u[b + 4] - kin;
        }
        if (pp.disallow_negatives && eint < 0.0) status |= ST_EI_NEGATIVE;
        if (pp.use_smallei) {
            if (pp.smallei > eint) rec.en |= 1u << f;
            eint = f_max(eint, pp.smallei);
        }
        double e = eint + kin;
        if (PH::magn(f)) e = e + mag;
        u[b + 4] = e;
    }
}

}  // namespace pk
