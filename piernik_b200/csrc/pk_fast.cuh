// pk_fast.cuh -- the tolerance-mode arithmetic of the split sweep.
//
// The same algorithms as pk_device.cuh's utoq, riemann_hlld and
// riemann_hlld_u (interpolations.F90:69-106, hlld.F90:161-841) with the same
// branch structure, but rounding is not the reference's: the kernels that use
// these functions are compiled with multiply-add contraction (--fmad=true), and
// divisions by a common denominator are replaced by one reciprocal and
// products (1/rho in utoq; 1/(gamma-1) and 1/gamma from PhysParams; 1/slsm,
// 1/srsm, 1/(coeff_1), 1/(add_dnsq) and 1/ch in the Riemann solver; the two
// Alfven divisions by sqrt(rho*) through the reciprocal square root), and
// the remaining quotients, reciprocals and square roots of the solver and of
// utoq are the branch-free refinements below (rcp_nr, div_nr, rsqrt_nr).  Each replaced operation
// changes a result by a few units in the last place, so a time step agrees
// with the bit-exact path to ~1e-15 relative; the tests hold it to 1e-12 per
// step and 1e-9 after 100 steps.
#pragma once
#include "pk_device.cuh"

namespace pk {

// Reciprocal, quotient and reciprocal square root without the IEEE
// sequences' special-case branches: the hardware's approximate FP64
// reciprocal and reciprocal square root (PTX rcp.approx.ftz.f64,
// rsqrt.approx.ftz.f64, about 20 correct bits) refined by Newton-Raphson
// iterations (r' = r + r(1 - x r) and y' = y(3/2 - x y^2/2): each doubles the
// correct bits, two reach the double precision), the quotient finished with
// one residual correction (Markstein, IBM J. Res. Dev. 34 (1990) 111-119).
// Results are within about an ulp of the correctly rounded ones for normal
// finite operands, which is all the tolerance arithmetic asks; subnormal
// operands are flushed to zero by the seeds and are not expected in the
// states.  Square roots keep the IEEE operation: a Newton-refined root
// (tried) moved a three-fluid blast beyond the 1e-12 per-step bound.
PK_DEV double rcp_nr(double x)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

PK_DEV double div_nr(double a, double b)
{
    const double r = rcp_nr(b);
    const double q = a * r;
    return fma(r, fma(-b, q, a), q);
}

PK_DEV double rsqrt_nr(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double hx = 0.5 * x;
    y = y * fma(-hx * y, y, 1.5);
    return y * fma(-hx * y, y, 1.5);
}


template <class PH>
PK_DEV void utoq_fast(const double (&u)[PH::NV], double (&q)[PH::NV], const PhysParams& pp)
{
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {
        const int b = PH::beg(f);
        const double dn = u[b], mx = u[b + 1], my = u[b + 2], mz = u[b + 3];
        const double rdn = rcp_nr(dn);
        q[b] = dn;
        q[b + 1] = mx * rdn;
        q[b + 2] = my * rdn;
        q[b + 3] = mz * rdn;
        if (PH::has_en(f)) {
            const double ek = (0.5 * ((mx * mx + my * my) + mz * mz)) * rdn;
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
        for (int c = 0; c < 4; ++c) q[PH::IB + c] = u[PH::IB + c];
    }
}

// HLLD of one interface (hlld.F90:161-609); rgam_1 = 1/(gamma-1), rgam = 1/gamma
PK_DEV void hlld_iface_fast(bool has_energy, double gamma, double rgam_1, double rgam, const double* ul,
                            const double* ur, const double* bl, const double* br, double* f, double* bf)
{
    const int nc = has_energy ? 5 : 4;
    double prl, prr, c_fastm;
    double enl = 1.7976931348623157e308, enr = 1.7976931348623157e308, ue = 0.0;

    const double bbl = (bl[0] * bl[0] + bl[1] * bl[1]) + bl[2] * bl[2];
    const double bbr = (br[0] * br[0] + br[1] * br[1]) + br[2] * br[2];
    if (gamma < 0.0) {
        prl = 0.0;
        prr = 0.0;
        c_fastm = 0.0;
    } else {
        prl = ul[4] + 0.5 * bbl;
        prr = ur[4] + 0.5 * bbr;
        enl = ((ul[4] * rgam_1) + ((0.5 * ul[0]) * ((ul[1] * ul[1] + ul[2] * ul[2]) + ul[3] * ul[3]))) + (0.5 * bbl);
        enr = ((ur[4] * rgam_1) + ((0.5 * ur[0]) * ((ur[1] * ur[1] + ur[2] * ur[2]) + ur[3] * ur[3]))) + (0.5 * bbr);
        const double gampr_l = gamma * ul[4];
        const double gampr_r = gamma * ur[4];
        const double al = gampr_l + bbl, ar = gampr_r + bbr;
        const double nl = al + sqrt(al * al - ((4.0 * gampr_l) * (bl[0] * bl[0])));
        const double nr = ar + sqrt(ar * ar - ((4.0 * gampr_r) * (br[0] * br[0])));
        // max(nl/rho_l, nr/rho_r) with one division (densities are positive)
        const double cmax = (nl * ur[0] >= nr * ul[0]) ? div_nr(nl, ul[0]) : div_nr(nr, ur[0]);
        c_fastm = sqrt(0.5 * cmax);
    }
    const double sl = f_min(ul[1], ur[1]) - c_fastm;
    const double sr = f_max(ul[1], ur[1]) + c_fastm;

    if (sl >= 0.0 || sr <= 0.0) {
        const bool left = sl >= 0.0;
        const double* u = left ? ul : ur;
        const double* b = left ? bl : br;
        side_flux(has_energy, u, b, left ? prl : prr, left ? enl : enr, f);
        bf[0] = side_bflux(u, b, 1);
        bf[1] = side_bflux(u, b, 2);
        return;
    }

    double sm;
    {
        const double auxr = (sr - ur[1]) * ur[0];
        const double auxl = (sl - ul[1]) * ul[0];
        if (fabs(auxr - auxl) < f_spacing(auxr + auxl)) sm = (sl + sr) * 0.5;
        else sm = div_nr((auxr * ur[1] - prr) - (auxl * ul[1] - prl), auxr - auxl);
    }
    const double slsm = sl - sm, srsm = sr - sm;
    const double rslsm = rcp_nr(slsm), rsrsm = rcp_nr(srsm);
    const double slvxl = sl - ul[1], srvxr = sr - ur[1];
    const double srmsl = sr - sl;
    const double dn_l = ul[0] * slvxl, dn_r = ur[0] * srvxr;
    const double b_lr = bl[0] * br[0];
    const double b_lrgam = b_lr * rgam;
    const double prt_star = 0.5 * ((prl + dn_l * (sm - ul[1])) + (prr + dn_r * (sm - ur[1])));

    double bsl[3], bsr[3];
    bsl[0] = bl[0];
    bsr[0] = br[0];
    {
        double coeff_1 = dn_l * slsm - b_lr;
        if (has_energy) ue = ul[4];
        const bool star_l = (fabs(coeff_1) > f_spacing(b_lr)) && b_lrgam <= ue;
        double coeff_r = dn_r * srsm - b_lr;
        if (has_energy) ue = ur[4];
        const bool star_r = (fabs(coeff_r) > f_spacing(b_lr)) && b_lrgam <= ue;
        if (star_l) {
            const double t = div_nr(dn_l * slvxl - b_lr, coeff_1);
            bsl[1] = bl[1] * t;
            bsl[2] = bl[2] * t;
        }
        if (star_r) {
            const double t = div_nr(dn_r * srvxr - b_lr, coeff_r);
            bsr[1] = br[1] * t;
            bsr[2] = br[2] * t;
        }
        if (!star_l || !star_r) {                  // the HLL state of the transverse field
            const double r = rcp_nr(srmsl);
            const double h1 = ((sr * br[1] - sl * bl[1]) - (side_bflux(ur, br, 1) - side_bflux(ul, bl, 1))) * r;
            const double h2 = ((sr * br[2] - sl * bl[2]) - (side_bflux(ur, br, 2) - side_bflux(ul, bl, 2))) * r;
            if (!star_l) {
                bsl[1] = h1;
                bsl[2] = h2;
            }
            if (!star_r) {
                bsr[1] = h1;
                bsr[2] = h2;
            }
        }
    }
    double vsl[3], vsr[3];
    vsl[0] = sm;
    vsr[0] = sm;
    {
        const double bxl_dnl = div_nr(bl[0], dn_l), bxr_dnr = div_nr(br[0], dn_r);
        vsl[1] = ul[2] + (bxl_dnl * (bl[1] - bsl[1]));
        vsl[2] = ul[3] + (bxl_dnl * (bl[2] - bsl[2]));
        vsr[1] = ur[2] + (bxr_dnr * (br[1] - bsr[1]));
        vsr[2] = ur[3] + (bxr_dnr * (br[2] - bsr[2]));
    }
    const double vb_starl = (vsl[0] * bsl[0] + vsl[1] * bsl[1]) + vsl[2] * bsl[2];
    const double vb_starr = (vsr[0] * bsr[0] + vsr[1] * bsr[1]) + vsr[2] * bsr[2];

    double usl[5], usr[5];
    usl[0] = dn_l * rslsm;
    usr[0] = dn_r * rsrsm;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        usl[1 + c] = usl[0] * vsl[c];
        usr[1 + c] = usr[0] * vsr[c];
    }
    if (has_energy) {
        const double vb_l = (ul[1] * bl[0] + ul[2] * bl[1]) + ul[3] * bl[2];
        const double vb_r = (ur[1] * br[0] + ur[2] * br[1]) + ur[3] * br[2];
        usl[4] = ((((slvxl * enl) - (prl * ul[1])) + (prt_star * sm)) + (bl[0] * (vb_l - vb_starl))) * rslsm;
        usr[4] = ((((srvxr * enr) - (prr * ur[1])) + (prt_star * sm)) + (br[0] * (vb_r - vb_starr))) * rsrsm;
    }

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

    if (fabs(bl[0]) > 0.0) {
        const double rl = rsqrt_nr(usl[0]), rr = rsqrt_nr(usr[0]);
        const double dn_lsqt = usl[0] * rl;            // sqrt(rho*_l)
        const double dn_rsqt = usr[0] * rr;
        const double alfven_l = sm - fabs(bl[0]) * rl;
        const double alfven_r = sm + fabs(br[0]) * rr;
        if (alfven_l > 0.0 || alfven_r < 0.0) {
            star_flux(alfven_l > 0.0, f, bf);
            return;
        }
        const double b_sig = (bl[0] >= 0.0) ? 1.0 : -1.0;
        const double radd = rcp_nr(dn_lsqt + dn_rsqt);
        const double mul_dnsq = dn_lsqt * dn_rsqt;
        double v2[3], b2[3];
        v2[0] = sm;
        v2[1] = ((dn_lsqt * vsl[1] + dn_rsqt * vsr[1]) + b_sig * (bsr[1] - bsl[1])) * radd;
        v2[2] = ((dn_lsqt * vsl[2] + dn_rsqt * vsr[2]) + b_sig * (bsr[2] - bsl[2])) * radd;
        b2[0] = 0.5 * (bl[0] + br[0]);
        const double bsm = b_sig * mul_dnsq;
        b2[1] = ((dn_lsqt * bsr[1] + dn_rsqt * bsl[1]) + bsm * (vsr[1] - vsl[1])) * radd;
        b2[2] = ((dn_lsqt * bsr[2] + dn_rsqt * bsl[2]) + bsm * (vsr[2] - vsl[2])) * radd;
        const double vb_2star = (v2[0] * b2[0] + v2[1] * b2[1]) + v2[2] * b2[2];

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
        if (sm > 0.0 || sm < 0.0) {
            alfven_flux(sm > 0.0, f, bf);
        } else {
            double fl2[5], fr2[5], bl2[2], br2[2];
            alfven_flux(true, fl2, bl2);
            alfven_flux(false, fr2, br2);
#pragma unroll
            for (int c = 0; c < 5; ++c)
                if (c < nc) f[c] = 0.5 * (fl2[c] + fr2[c]);
            bf[0] = 0.5 * (bl2[0] + br2[0]);
            bf[1] = 0.5 * (bl2[1] + br2[1]);
        }
    } else {
        if (sm > 0.0 || sm < 0.0) {
            star_flux(sm > 0.0, f, bf);
        } else {
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

// HLLC of one interface (riemann_hlld_u, hlld.F90:615-841)
PK_DEV void hllc_iface_fast(bool has_energy, double gamma, double rgam_1, const double* ul, const double* ur,
                            double* f)
{
    double fl[5], fr[5], usl[5], usr[5];
    double prl, prr, c_fastm;
    double enl = 1.7976931348623157e308, enr = 1.7976931348623157e308;
    const int nc = has_energy ? 5 : 4;
    if (gamma < 0.0) {
        prl = 0.0;
        prr = 0.0;
        c_fastm = 0.0;
    } else {
        prl = ul[4];
        prr = ur[4];
        enl = (ul[4] * rgam_1) + ((0.5 * ul[0]) * ((ul[1] * ul[1] + ul[2] * ul[2]) + ul[3] * ul[3]));
        enr = (ur[4] * rgam_1) + ((0.5 * ur[0]) * ((ur[1] * ur[1] + ur[2] * ur[2]) + ur[3] * ur[3]));
        const double gampr_l = gamma * ul[4];
        const double gampr_r = gamma * ur[4];
        const double cmax = (gampr_l * ur[0] >= gampr_r * ul[0]) ? div_nr(gampr_l, ul[0]) : div_nr(gampr_r, ur[0]);
        c_fastm = sqrt(cmax);
    }
    const double sl = f_min(ul[1], ur[1]) - c_fastm;
    const double sr = f_max(ul[1], ur[1]) + c_fastm;
    fl[0] = ul[0] * ul[1];
    fl[1] = (ul[0] * (ul[1] * ul[1])) + prl;
    fl[2] = (ul[0] * ul[2]) * ul[1];
    fl[3] = (ul[0] * ul[3]) * ul[1];
    if (has_energy) fl[4] = (enl + prl) * ul[1];
    fr[0] = ur[0] * ur[1];
    fr[1] = (ur[0] * (ur[1] * ur[1])) + prr;
    fr[2] = (ur[0] * ur[2]) * ur[1];
    fr[3] = (ur[0] * ur[3]) * ur[1];
    if (has_energy) fr[4] = (enr + prr) * ur[1];
    if (sl >= 0.0) {
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
    double sm;
    {
        const double auxr = (sr - ur[1]) * ur[0];
        const double auxl = (sl - ul[1]) * ul[0];
        if (fabs(auxr - auxl) < f_spacing(auxr + auxl)) sm = (sl + sr) * 0.5;
        else sm = div_nr((auxr * ur[1] - prr) - (auxl * ul[1] - prl), auxr - auxl);
    }
    const double slvxl = sl - ul[1], srvxr = sr - ur[1];
    const double dn_l = ul[0] * slvxl, dn_r = ur[0] * srvxr;
    const double prt_star = 0.5 * ((prl + dn_l * (sm - ul[1])) + (prr + dn_r * (sm - ur[1])));
    if (sm >= 0.0) {
        const double r = rcp_nr(sl - sm);
        usl[0] = dn_l * r;
        usl[1] = usl[0] * sm;
        usl[2] = usl[0] * ul[2];
        usl[3] = usl[0] * ul[3];
        if (has_energy) usl[4] = (((slvxl * enl) - (prl * ul[1])) + (prt_star * sm)) * r;
    }
    if (sm <= 0.0) {
        const double r = rcp_nr(sr - sm);
        usr[0] = dn_r * r;
        usr[1] = usr[0] * sm;
        usr[2] = usr[0] * ur[2];
        usr[3] = usr[0] * ur[3];
        if (has_energy) usr[4] = (((srvxr * enr) - (prr * ur[1])) + (prt_star * sm)) * r;
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
    if (sm > 0.0) {
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) f[c] = fl[c] + sl * (usl[c] - ucl[c]);
    } else if (sm < 0.0) {
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) f[c] = fr[c] + sr * (usr[c] - ucr[c]);
    } else {
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) f[c] = 0.5 * (((fl[c] + sl * (usl[c] - ucl[c])) + fr[c]) + sr * (usr[c] - ucr[c]));
    }
}

}  // namespace pk

namespace pk {

// riemann_tile (pk_device.cuh) with the tolerance-mode solvers: the GLM flux
// of psi multiplies by 1/ch instead of dividing
template <class PH>
PK_DEV void riemann_tile_fast(const double* __restrict__ L, const double* __restrict__ R, double* __restrict__ F,
                              int PT, int me, int st, double ch, double rch, const PhysParams& pp)
{
    double blv[3] = {0.0, 0.0, 0.0}, brv[3] = {0.0, 0.0, 0.0};
    if (PH::MHD) {
        const double bxl = L[PH::IB * PT + me], bxr = R[PH::IB * PT + me + st];
        const double psl = L[(PH::IB + 3) * PT + me], psr = R[(PH::IB + 3) * PT + me + st];
        F[(PH::IB + 3) * PT + me] = ((ch * ch) * 0.5) * ((bxr + bxl) - (psr - psl) * rch);   // hlld.F90:229
        F[PH::IB * PT + me] = 0.5 * ((psr + psl) - ch * (bxr - bxl));                       // :230
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
            hlld_iface_fast(PH::has_en(f), pp.gam[f], pp.rgam_1[f], pp.rgam[f], ul, ur, PH::magn(f) ? blv : zero,
                            PH::magn(f) ? brv : zero, fv, bf);
            if (PH::magn(f)) {
                F[(PH::IB + 1) * PT + me] = bf[0];
                F[(PH::IB + 2) * PT + me] = bf[1];
            }
        } else {
            hllc_iface_fast(PH::has_en(f), pp.gam[f], pp.rgam_1[f], ul, ur, fv);
        }
#pragma unroll
        for (int c = 0; c < 5; ++c)
            if (c < nc) F[(b + c) * PT + me] = fv[c];
    }
}

}  // namespace pk
