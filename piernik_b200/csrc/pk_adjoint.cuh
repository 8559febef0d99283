// pk_adjoint.cuh -- reverse-mode (vector-Jacobian) counterparts of the sweep's
// building blocks, for the differentiable path.
//
// Each *_adj function recomputes the primal quantities it needs and
// accumulates (+=) the adjoints of its inputs from the adjoints of its
// outputs, differentiating the branch the primal takes (min/max pass the
// derivative to the selected argument, floors that clip pass none, spacing()
// is piecewise constant).  Evaluation order of the recomputed primal follows
// pk_device.cuh exactly wherever a branch decision depends on it (the wave
// speeds, sm, rho* and the Alfven speeds, the star-state test), so the
// branches taken match the forward kernels.  Quotients that only feed
// derivative values, and every quotient of the reverse accumulation, use one
// reciprocal per denominator (arcp) and products: derivatives agree with the
// dual-number tangent to ~1e-15 relative, and the kernels avoid ~60 IEEE
// division sequences per face.
#pragma once
#include <type_traits>

#include "pk_device.cuh"
#include "pk_fast.cuh"

namespace pk {

// 1/x for derivative values: the branch-free Newton-refined reciprocal on
// the device (within about an ulp of the correctly rounded one), the IEEE
// quotient on the host.
PK_PHYS double arcp(double x)
{
#ifdef __CUDA_ARCH__
    return rcp_nr(x);
#else
    return 1.0 / x;
#endif
}

// a*b + c in one rounding: the multiply-accumulates of the reverse pass (the
// translation unit keeps --fmad=false for the primal recompute, so the fused
// operation is written out).
PK_PHYS double fm(double a, double b, double c) { return fma(a, b, c); }

// Compile-time side of a Riemann interface.  The adjoints below pick the left
// or right state's arrays with it, so that no array has to live in local
// memory for a run-time pointer choice.
template <bool B>
using Side = std::integral_constant<bool, B>;

// ---------------------------------------------------------------------------
// utoq (interpolations.F90:69-106): ub += (dq/du)^T qb
// ---------------------------------------------------------------------------
template <class PH>
PK_PHYS void utoq_adj(const double (&u)[PH::NV], const double (&qb)[PH::NV], double (&ub)[PH::NV],
                      const PhysParams& pp)
{
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {
        const int b = PH::beg(f);
        const double dn = u[b], mx = u[b + 1], my = u[b + 2], mz = u[b + 3];
        const double rdn = arcp(dn);
        const double qv = fm(qb[b + 3], mz, fm(qb[b + 2], my, qb[b + 1] * mx));   // qb . m
        double u0 = fm(-qv, rdn * rdn, ub[b] + qb[b]);
        ub[b + 1] = fm(qb[b + 1], rdn, ub[b + 1]);
        ub[b + 2] = fm(qb[b + 2], rdn, ub[b + 2]);
        ub[b + 3] = fm(qb[b + 3], rdn, ub[b + 3]);
        if (PH::has_en(f)) {
            const double g1 = pp.gam_1[f], pb = qb[b + 4];
            ub[b + 4] = fm(g1, pb, ub[b + 4]);
            const double ekb = -g1 * pb;                       // p = g1*(E - ek)
            const double ek = (0.5 * fm(mz, mz, fm(my, my, mx * mx))) * rdn;
            u0 = fm(-ekb * ek, rdn, u0);
            const double sqb2 = ekb * rdn;                     // d(ek)/dm = m/rho
            ub[b + 1] = fm(sqb2, mx, ub[b + 1]);
            ub[b + 2] = fm(sqb2, my, ub[b + 2]);
            ub[b + 3] = fm(sqb2, mz, ub[b + 3]);
            if (PH::magn(f)) {                                 // p -= (0.5*g1)*|B|^2
                const double t = -g1 * pb;
#pragma unroll
                for (int c = 0; c < 3; ++c) ub[PH::IB + c] = fm(t, u[PH::IB + c], ub[PH::IB + c]);
            }
        }
        ub[b] = u0;
    }
    if (PH::MHD) {
#pragma unroll
        for (int c = 0; c < 4; ++c) ub[PH::IB + c] += qb[PH::IB + c];
    }
}

// ---------------------------------------------------------------------------
// limited slope of an interior cell (fluxlimiters.F90:109-216):
// (dlb, drb) = sb * d(slope)/d(dl, dr)
// ---------------------------------------------------------------------------
PK_PHYS void slope_adj(int lim, double dl, double dr, double sb, double& dlb, double& drb)
{
    dlb = 0.0;
    drb = 0.0;
    if (lim == L_VANLEER) {
        const double dcen = dl * dr;
        if (dcen > 0.0) {
            const double den = dl + dr;
            const double r2 = arcp(den * den);
            dlb = sb * (2.0 * dr * dr) * r2;
            drb = sb * (2.0 * dl * dl) * r2;
        }
        return;
    }
    const double S = f_sign1(dl) + f_sign1(dr);
    const double adl = fabs(dl), adr = fabs(dr);
    if (lim == L_MINMOD) {
        const double mb = sb * 0.5 * S;
        if (adr < adl) drb = mb * f_sign1(dr);
        else dlb = mb * f_sign1(dl);
        return;
    }
    if (lim == L_MONCEN) {
        const double a = 2.0 * adl, b = 2.0 * adr, c = 0.5 * fabs(dl + dr);
        const bool right = b < a;
        const double inner = right ? b : a;
        const double mb = sb * 0.5 * S;
        if (c < inner) {
            const double t = mb * 0.5 * f_sign1(dl + dr);
            dlb = t;
            drb = t;
        } else if (right) {
            drb = mb * 2.0 * f_sign1(dr);
        } else {
            dlb = mb * 2.0 * f_sign1(dl);
        }
        return;
    }
    const double mb = sb * S * 0.5;                            // superbee
    if (adl > adr) {
        if (fabs(2.0 * dr) < adl) drb = mb * 2.0 * f_sign1(dr);
        else dlb = mb * f_sign1(dl);
    } else {
        if (adr < fabs(2.0 * dl)) drb = mb * f_sign1(dr);
        else dlb = mb * 2.0 * f_sign1(dl);
    }
}

// lam: adjoint of the post-floor state in, adjoint of the pre-floor state out.
// uout is the post-floor state (the floors do not change m or B).
template <class PH>
PK_PHYS void floors_adj(const double (&uout)[PH::NV], const FloorRec& rec, double (&lam)[PH::NV])
{
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {
        if (!PH::has_en(f) || !(rec.en & (1u << f))) continue;   // unclipped: E' = E exactly
        const int b = PH::beg(f);
        const double lE = lam[b + 4];
        lam[b + 4] = 0.0;                                          // E' = smallei + kin + mag
        const double rdn = arcp(uout[b]);
        const double kin = (0.5 * ((uout[b + 1] * uout[b + 1] + uout[b + 2] * uout[b + 2]) + uout[b + 3] * uout[b + 3])) * rdn;
        lam[b + 1] += lE * uout[b + 1] * rdn;
        lam[b + 2] += lE * uout[b + 2] * rdn;
        lam[b + 3] += lE * uout[b + 3] * rdn;
        lam[b] += -lE * kin * rdn;
        if (PH::magn(f)) {
#pragma unroll
            for (int c = 0; c < 3; ++c) lam[PH::IB + c] += lE * uout[PH::IB + c];
        }
    }
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f)
        if (rec.dn & (1u << f)) lam[PH::beg(f)] = 0.0;
}

// ---------------------------------------------------------------------------
// helpers for the Riemann adjoints
// ---------------------------------------------------------------------------

// adjoint of side_flux + side_bflux (hlld.F90:296-309); fb has nc entries, bfb 2
PK_PHYS void side_flux_adj(bool has_energy, const double* u, const double* b, double pr, double en, const double* fb,
                           const double* bfb, double* ub, double* bb, double& prb, double& enb)
{
    const double vb = fm(u[3], b[2], fm(u[2], b[1], u[1] * b[0]));
    const double f4 = has_energy ? fb[4] : 0.0;
    const double mv = fm(fb[3], u[3], fm(fb[2], u[2], fm(fb[1], u[1], fb[0])));   // fb[0..3] . (1, u1, u2, u3)
    const double u0u1 = u[0] * u[1], f4b0 = f4 * b[0];
    ub[0] = fm(mv, u[1], ub[0]);
    ub[1] = fm(u[0], fm(fb[1], u[1], mv), fm(f4, fm(-b[0], b[0], en + pr), fm(bfb[1], b[2], fm(bfb[0], b[1], ub[1]))));
    ub[2] = fm(fb[2], u0u1, fm(-f4b0, b[1], fm(-bfb[0], b[0], ub[2])));
    ub[3] = fm(fb[3], u0u1, fm(-f4b0, b[2], fm(-bfb[1], b[0], ub[3])));
    prb += fm(f4, u[1], fb[1]);
    enb = fm(f4, u[1], enb);
    bb[0] -= fm(2.0 * fb[1], b[0], fm(fb[2], b[1], fm(fb[3], b[2], fm(f4, fm(b[0], u[1], vb), fm(bfb[0], u[2], bfb[1] * u[3])))));
    bb[1] += fm(-fb[2], b[0], fm(-f4b0, u[2], bfb[0] * u[1]));
    bb[2] += fm(-fb[3], b[0], fm(-f4b0, u[3], bfb[1] * u[1]));
}

// adjoint of pr = p + |B|^2/2 and en = p/(g-1) + rho v^2/2 + |B|^2/2 (hlld.F90:258-269)
PK_PHYS void pr_en_adj(bool mhd, double gamma, const double* u, const double* b, double prb, double enb, double* ub,
                       double* bb)
{
    ub[4] = fm(enb, arcp(gamma - 1.0), ub[4] + prb);
    const double vv = fm(u[3], u[3], fm(u[2], u[2], u[1] * u[1]));
    ub[0] = fm(enb * 0.5, vv, ub[0]);
    const double eu = enb * u[0];
    ub[1] = fm(eu, u[1], ub[1]);
    ub[2] = fm(eu, u[2], ub[2]);
    ub[3] = fm(eu, u[3], ub[3]);
    if (mhd) {
        const double t = prb + enb;
#pragma unroll
        for (int c = 0; c < 3; ++c) bb[c] = fm(t, b[c], bb[c]);
    }
}

// adjoint of cons = [u0, u0*u1, u0*u2, u0*u3, en] given consb
PK_PHYS void cons_adj(bool has_energy, const double* u, const double* consb, double* ub, double& enb)
{
    ub[0] = fm(consb[3], u[3], fm(consb[2], u[2], fm(consb[1], u[1], ub[0] + consb[0])));
    ub[1] = fm(consb[1], u[0], ub[1]);
    ub[2] = fm(consb[2], u[0], ub[2]);
    ub[3] = fm(consb[3], u[0], ub[3]);
    if (has_energy) enb += consb[4];
}

// ---------------------------------------------------------------------------
// HLLC (riemann_hlld_u, hlld.F90:615-841): given fb (nc), accumulate ulb, urb
// ---------------------------------------------------------------------------
PK_PHYS void hllc_adj(bool has_energy, double gamma, const double* ul, const double* ur, const double* fb, double* ulb,
                      double* urb)
{
    const int nc = has_energy ? 5 : 4;
    const bool dust = gamma < 0.0;
    double prl = 0.0, prr = 0.0, cf = 0.0, enl = 0.0, enr = 0.0, cl = 0.0, cr = 0.0;
    if (!dust) {
        prl = ul[4];
        prr = ur[4];
        const double rg1 = arcp(gamma - 1.0);
        enl = (ul[4] * rg1) + ((0.5 * ul[0]) * ((ul[1] * ul[1] + ul[2] * ul[2]) + ul[3] * ul[3]));
        enr = (ur[4] * rg1) + ((0.5 * ur[0]) * ((ur[1] * ur[1] + ur[2] * ur[2]) + ur[3] * ur[3]));
        cl = (gamma * ul[4]) / ul[0];
        cr = (gamma * ur[4]) / ur[0];
        cf = sqrt(f_max(cl, cr));
    }
    const bool minr = ur[1] < ul[1], maxr = ur[1] > ul[1];
    const double sl = f_min(ul[1], ur[1]) - cf;
    const double sr = f_max(ul[1], ur[1]) + cf;
    double prlb = 0.0, prrb = 0.0, enlb = 0.0, enrb = 0.0, slb = 0.0, srb = 0.0, smb = 0.0;
    const double zb[2] = {0.0, 0.0}, zbv[3] = {0.0, 0.0, 0.0};
    double bdump[3] = {0.0, 0.0, 0.0};
    if (sl >= 0.0 || sr <= 0.0) {
        double fb5[5] = {0, 0, 0, 0, 0};
        for (int c = 0; c < nc; ++c) fb5[c] = fb[c];
        if (sl >= 0.0) side_flux_adj(has_energy, ul, zbv, prl, enl, fb5, zb, ulb, bdump, prlb, enlb);
        else side_flux_adj(has_energy, ur, zbv, prr, enr, fb5, zb, urb, bdump, prrb, enrb);
    } else {
        const double auxr = (sr - ur[1]) * ur[0];
        const double auxl = (sl - ul[1]) * ul[0];
        const bool deg = fabs(auxr - auxl) < f_spacing(auxr + auxl);
        const double num = (auxr * ur[1] - prr) - (auxl * ul[1] - prl);
        const double den = auxr - auxl;
        const double sm = deg ? (sl + sr) / 2.0 : num / den;
        const double slvxl = sl - ul[1], srvxr = sr - ur[1];
        const double dn_l = ul[0] * slvxl, dn_r = ur[0] * srvxr;
        const double prt = 0.5 * ((prl + dn_l * (sm - ul[1])) + (prr + dn_r * (sm - ur[1])));
        double prtb = 0.0, dn_lb = 0.0, dn_rb = 0.0, slvxlb = 0.0, srvxrb = 0.0;
        // one side's star flux f = fs + s*(us - cons), scaled by w (1 or 1/2)
        auto side = [&](auto sd, double w) {
            constexpr bool left = decltype(sd)::value;
            const double* u = left ? ul : ur;
            double* ub = left ? ulb : urb;
            const double s = left ? sl : sr;
            const double ssm = s - sm;
            const double dn = left ? dn_l : dn_r;
            const double svx = left ? slvxl : srvxr;
            const double pr = left ? prl : prr;
            const double en = left ? enl : enr;
            const double rssm = arcp(ssm);
            double us[5];
            us[0] = dn * rssm;
            us[1] = us[0] * sm;
            us[2] = us[0] * u[2];
            us[3] = us[0] * u[3];
            us[4] = has_energy ? (((svx * en) - (pr * u[1])) + (prt * sm)) * rssm : 0.0;
            double cons[5] = {u[0], u[0] * u[1], u[0] * u[2], u[0] * u[3], en};
            double fsb[5] = {0, 0, 0, 0, 0}, usb[5] = {0, 0, 0, 0, 0}, consb[5] = {0, 0, 0, 0, 0};
            double sb = 0.0;
            for (int c = 0; c < nc; ++c) {
                const double g = w * fb[c];
                fsb[c] = g;
                sb = fm(g, us[c] - cons[c], sb);
                usb[c] = g * s;
                consb[c] = -g * s;
            }
            double prb = 0.0, enb = 0.0;
            side_flux_adj(has_energy, u, zbv, pr, en, fsb, zb, ub, bdump, prb, enb);
            cons_adj(has_energy, u, consb, ub, enb);
            // us
            double us0b = fm(usb[3], u[3], fm(usb[2], u[2], fm(usb[1], sm, usb[0])));
            smb = fm(usb[1], us[0], smb);
            ub[2] = fm(usb[2], us[0], ub[2]);
            ub[3] = fm(usb[3], us[0], ub[3]);
            double ssmb = 0.0;
            if (has_energy) {
                const double n4b = usb[4] * rssm;
                ssmb = -n4b * us[4];
                if (left) slvxlb = fm(n4b, en, slvxlb); else srvxrb = fm(n4b, en, srvxrb);
                enb = fm(n4b, svx, enb);
                prb = fm(-n4b, u[1], prb);
                ub[1] = fm(-n4b, pr, ub[1]);
                prtb = fm(n4b, sm, prtb);
                smb = fm(n4b, prt, smb);
            }
            const double t0 = us0b * rssm;
            if (left) dn_lb += t0; else dn_rb += t0;
            ssmb = fm(-t0, us[0], ssmb);
            sb += ssmb;
            smb -= ssmb;
            if (left) { slb += sb; prlb += prb; enlb += enb; }
            else { srb += sb; prrb += prb; enrb += enb; }
        };
        if (sm > 0.0) side(Side<true>{}, 1.0);
        else if (sm < 0.0) side(Side<false>{}, 1.0);
        else { side(Side<true>{}, 0.5); side(Side<false>{}, 0.5); }
        // prt
        const double hp = 0.5 * prtb;
        prlb += hp;
        prrb += hp;
        dn_lb = fm(hp, sm - ul[1], dn_lb);
        dn_rb = fm(hp, sm - ur[1], dn_rb);
        smb = fm(hp, dn_l + dn_r, smb);
        ulb[1] = fm(-hp, dn_l, ulb[1]);
        urb[1] = fm(-hp, dn_r, urb[1]);
        // dn = u0 * svx
        ulb[0] = fm(dn_lb, slvxl, ulb[0]);
        slvxlb = fm(dn_lb, ul[0], slvxlb);
        urb[0] = fm(dn_rb, srvxr, urb[0]);
        srvxrb = fm(dn_rb, ur[0], srvxrb);
        slb += slvxlb;
        ulb[1] -= slvxlb;
        srb += srvxrb;
        urb[1] -= srvxrb;
        // sm
        double auxrb = 0.0, auxlb = 0.0;
        if (deg) {
            slb += smb / 2.0;
            srb += smb / 2.0;
        } else {
            const double rden = arcp(den);
            const double numb = smb * rden, denb = -numb * sm;
            auxrb = fm(numb, ur[1], denb);
            urb[1] = fm(numb, auxr, urb[1]);
            prrb -= numb;
            auxlb = fm(-numb, ul[1], -denb);
            ulb[1] = fm(-numb, auxl, ulb[1]);
            prlb += numb;
        }
        srb = fm(auxrb, ur[0], srb);
        urb[1] = fm(-auxrb, ur[0], urb[1]);
        urb[0] = fm(auxrb, sr - ur[1], urb[0]);
        slb = fm(auxlb, ul[0], slb);
        ulb[1] = fm(-auxlb, ul[0], ulb[1]);
        ulb[0] = fm(auxlb, sl - ul[1], ulb[0]);
    }
    // sl = min(ul1, ur1) - cf ; sr = max(ul1, ur1) + cf
    if (minr) urb[1] += slb; else ulb[1] += slb;
    if (maxr) urb[1] += srb; else ulb[1] += srb;
    if (!dust) {
        const double cfb = srb - slb;
        if (cf > 0.0) {
            const double cmb = cfb * 0.5 * arcp(cf);
            if (cr > cl) {
                const double r0 = arcp(ur[0]);
                urb[4] += cmb * gamma * r0;
                urb[0] -= cmb * cr * r0;
            } else {
                const double r0 = arcp(ul[0]);
                ulb[4] += cmb * gamma * r0;
                ulb[0] -= cmb * cl * r0;
            }
        }
        pr_en_adj(false, gamma, ul, zbv, prlb, enlb, ulb, bdump);
        pr_en_adj(false, gamma, ur, zbv, prrb, enrb, urb, bdump);
    }
}

// ---------------------------------------------------------------------------
// HLLD (riemann_hlld, hlld.F90:161-609): given fb (nc) and bfb (transverse B
// flux adjoints), accumulate ulb, urb (primitive states) and blb, brb (B).
// ---------------------------------------------------------------------------
PK_PHYS void hlld_adj(bool has_energy, double gamma, const double* ul, const double* ur, const double* bl,
                      const double* br, const double* fb, const double* bfb, double* ulb, double* urb, double* blb,
                      double* brb)
{
    const int nc = has_energy ? 5 : 4;
    const bool dust = gamma < 0.0;
    double prl = 0.0, prr = 0.0, cf = 0.0, enl = 0.0, enr = 0.0, cl = 0.0, cr = 0.0;
    double al = 0.0, ar = 0.0, rootl = 0.0, rootr = 0.0, gpl = 0.0, gpr = 0.0;
    if (!dust) {
        const double magprl = 0.5 * ((bl[0] * bl[0] + bl[1] * bl[1]) + bl[2] * bl[2]);
        const double magprr = 0.5 * ((br[0] * br[0] + br[1] * br[1]) + br[2] * br[2]);
        prl = ul[4] + magprl;
        prr = ur[4] + magprr;
        const double bbl = (bl[0] * bl[0] + bl[1] * bl[1]) + bl[2] * bl[2];
        const double bbr = (br[0] * br[0] + br[1] * br[1]) + br[2] * br[2];
        const double rg1 = arcp(gamma - 1.0);
        enl = ((ul[4] * rg1) + ((0.5 * ul[0]) * ((ul[1] * ul[1] + ul[2] * ul[2]) + ul[3] * ul[3]))) + (0.5 * bbl);
        enr = ((ur[4] * rg1) + ((0.5 * ur[0]) * ((ur[1] * ur[1] + ur[2] * ur[2]) + ur[3] * ur[3]))) + (0.5 * bbr);
        gpl = gamma * ul[4];
        gpr = gamma * ur[4];
        al = gpl + bbl;
        ar = gpr + bbr;
        rootl = sqrt(al * al - ((4.0 * gpl) * (bl[0] * bl[0])));
        rootr = sqrt(ar * ar - ((4.0 * gpr) * (br[0] * br[0])));
        cl = (al + rootl) / ul[0];
        cr = (ar + rootr) / ur[0];
        cf = sqrt(0.5 * f_max(cl, cr));
    }
    const bool minr = ur[1] < ul[1], maxr = ur[1] > ul[1];
    const double sl = f_min(ul[1], ur[1]) - cf;
    const double sr = f_max(ul[1], ur[1]) + cf;
    double prlb = 0.0, prrb = 0.0, enlb = 0.0, enrb = 0.0, slb = 0.0, srb = 0.0;
    double fb5[5] = {0, 0, 0, 0, 0};
    for (int c = 0; c < nc; ++c) fb5[c] = fb[c];

    if (sl >= 0.0 || sr <= 0.0) {                                        // :312-319
        if (sl >= 0.0) side_flux_adj(has_energy, ul, bl, prl, enl, fb5, bfb, ulb, blb, prlb, enlb);
        else side_flux_adj(has_energy, ur, br, prr, enr, fb5, bfb, urb, brb, prrb, enrb);
    } else {
        // ---- primal of the star / Alfven states (hlld.F90:323-474) ----
        const double auxr = (sr - ur[1]) * ur[0];
        const double auxl = (sl - ul[1]) * ul[0];
        const bool deg = fabs(auxr - auxl) < f_spacing(auxr + auxl);
        const double num = (auxr * ur[1] - prr) - (auxl * ul[1] - prl);
        const double den = auxr - auxl;
        const double sm = deg ? (sl + sr) / 2.0 : num / den;
        const double slsm = sl - sm, srsm = sr - sm;
        const double slvxl = sl - ul[1], srvxr = sr - ur[1];
        const double srmsl = sr - sl;
        const double dn_l = ul[0] * slvxl, dn_r = ur[0] * srvxr;
        const double b_lr = bl[0] * br[0];
        const double b_lrgam = b_lr / gamma;
        const double prt = 0.5 * ((prl + dn_l * (sm - ul[1])) + (prr + dn_r * (sm - ur[1])));
        const double bclf1 = side_bflux(ul, bl, 1), bclf2 = side_bflux(ul, bl, 2);
        const double bcrf1 = side_bflux(ur, br, 1), bcrf2 = side_bflux(ur, br, 2);
        const double ue_l = has_energy ? ul[4] : 0.0, ue_r = has_energy ? ur[4] : 0.0;
        const double coeffL = dn_l * slsm - b_lr, coeffR = dn_r * srsm - b_lr;
        const bool starL = (fabs(coeffL) > f_spacing(b_lr)) && b_lrgam <= ue_l;
        const bool starR = (fabs(coeffR) > f_spacing(b_lr)) && b_lrgam <= ue_r;
        const double aL = dn_l * slvxl - b_lr, aR = dn_r * srvxr - b_lr;
        double bsl[3], bsr[3];
        bsl[0] = bl[0];
        bsr[0] = br[0];
        const double rsrmsl = arcp(srmsl);
        const double hll1 = ((sr * br[1] - sl * bl[1]) - (bcrf1 - bclf1)) * rsrmsl;
        const double hll2 = ((sr * br[2] - sl * bl[2]) - (bcrf2 - bclf2)) * rsrmsl;
        const double rcL = starL ? arcp(coeffL) : 0.0, rcR = starR ? arcp(coeffR) : 0.0;
        if (starL) { bsl[1] = (bl[1] * aL) * rcL; bsl[2] = (bl[2] * aL) * rcL; }
        else { bsl[1] = hll1; bsl[2] = hll2; }
        if (starR) { bsr[1] = (br[1] * aR) * rcR; bsr[2] = (br[2] * aR) * rcR; }
        else { bsr[1] = hll1; bsr[2] = hll2; }
        const double rdnl = arcp(dn_l), rdnr = arcp(dn_r);
        const double kl = bl[0] * rdnl, kr = br[0] * rdnr;
        double vsl[3], vsr[3];
        vsl[0] = sm;
        vsr[0] = sm;
        vsl[1] = ul[2] + (kl * (bl[1] - bsl[1]));
        vsl[2] = ul[3] + (kl * (bl[2] - bsl[2]));
        vsr[1] = ur[2] + (kr * (br[1] - bsr[1]));
        vsr[2] = ur[3] + (kr * (br[2] - bsr[2]));
        const double vbsl = (vsl[0] * bsl[0] + vsl[1] * bsl[1]) + vsl[2] * bsl[2];
        const double vbsr = (vsr[0] * bsr[0] + vsr[1] * bsr[1]) + vsr[2] * bsr[2];
        const double vbl = (ul[1] * bl[0] + ul[2] * bl[1]) + ul[3] * bl[2];
        const double vbr = (ur[1] * br[0] + ur[2] * br[1]) + ur[3] * br[2];
        double usl[5], usr[5];
        usl[0] = dn_l / slsm;
        usr[0] = dn_r / srsm;
        for (int c = 0; c < 3; ++c) {
            usl[1 + c] = usl[0] * vsl[c];
            usr[1 + c] = usr[0] * vsr[c];
        }
        const double n4l = (((slvxl * enl) - (prl * ul[1])) + (prt * sm)) + (bl[0] * (vbl - vbsl));
        const double n4r = (((srvxr * enr) - (prr * ur[1])) + (prt * sm)) + (br[0] * (vbr - vbsr));
        const double rslsm = arcp(slsm), rsrsm = arcp(srsm);
        usl[4] = has_energy ? n4l * rslsm : 0.0;
        usr[4] = has_energy ? n4r * rsrsm : 0.0;
        const bool bx_nz = fabs(bl[0]) > 0.0;
        const double sql = sqrt(usl[0]), sqr = sqrt(usr[0]);
        const double alfl = sm - fabs(bl[0]) / sql, alfr = sm + fabs(br[0]) / sqr;
        const double b_sig = (bl[0] >= 0.0) ? 1.0 : -1.0;
        const double add = sql + sqr, mul = sql * sqr, bsm = b_sig * mul;
        const double radd = arcp(add);
        double v2[3], b2[3];
        v2[0] = sm;
        v2[1] = ((sql * vsl[1] + sqr * vsr[1]) + b_sig * (bsr[1] - bsl[1])) * radd;
        v2[2] = ((sql * vsl[2] + sqr * vsr[2]) + b_sig * (bsr[2] - bsl[2])) * radd;
        b2[0] = 0.5 * (bl[0] + br[0]);
        b2[1] = ((sql * bsr[1] + sqr * bsl[1]) + bsm * (vsr[1] - vsl[1])) * radd;
        b2[2] = ((sql * bsr[2] + sqr * bsl[2]) + bsm * (vsr[2] - vsl[2])) * radd;
        const double vb2 = (v2[0] * b2[0] + v2[1] * b2[1]) + v2[2] * b2[2];

        // ---- adjoint accumulators of the intermediates ----
        double smb = 0.0, prtb = 0.0, dn_lb = 0.0, dn_rb = 0.0, slvxlb = 0.0, srvxrb = 0.0, slsmb = 0.0,
               srsmb = 0.0, srmslb = 0.0;
        double bslb[3] = {0, 0, 0}, bsrb[3] = {0, 0, 0}, vslb[3] = {0, 0, 0}, vsrb[3] = {0, 0, 0};
        double uslb[5] = {0, 0, 0, 0, 0}, usrb[5] = {0, 0, 0, 0, 0};
        double vbslb = 0.0, vbsrb = 0.0, sqlb = 0.0, sqrb = 0.0, alflb = 0.0, alfrb = 0.0;
        double v2b[3] = {0, 0, 0}, b2b[3] = {0, 0, 0}, vb2b = 0.0;

        // star flux of one side (Eq. 64), weight w
        auto star_adj = [&](auto sd, double w) {
            constexpr bool left = decltype(sd)::value;
            const double* u = left ? ul : ur;
            const double* b = left ? bl : br;
            double* ub = left ? ulb : urb;
            double* bb = left ? blb : brb;
            const double s = left ? sl : sr;
            const double en = left ? enl : enr;
            const double* us = left ? usl : usr;
            const double* bs = left ? bsl : bsr;
            double* usb = left ? uslb : usrb;
            double* bsb = left ? bslb : bsrb;
            const double cons[5] = {u[0], u[0] * u[1], u[0] * u[2], u[0] * u[3], en};
            double fsb[5] = {0, 0, 0, 0, 0}, consb[5] = {0, 0, 0, 0, 0}, bfsb[2];
            double sb = 0.0;
            for (int c = 0; c < nc; ++c) {
                const double g = w * fb5[c];
                fsb[c] = g;
                sb = fm(g, us[c] - cons[c], sb);
                usb[c] = fm(g, s, usb[c]);
                consb[c] = -g * s;
            }
            for (int c = 1; c < 3; ++c) {
                const double g = w * bfb[c - 1];
                bfsb[c - 1] = g;
                sb = fm(g, bs[c] - b[c], sb);
                bsb[c] = fm(g, s, bsb[c]);
                bb[c] = fm(-g, s, bb[c]);
            }
            double prb = 0.0, enb = 0.0;
            side_flux_adj(has_energy, u, b, left ? prl : prr, en, fsb, bfsb, ub, bb, prb, enb);
            cons_adj(has_energy, u, consb, ub, enb);
            if (left) { slb += sb; prlb += prb; enlb += enb; }
            else { srb += sb; prrb += prb; enrb += enb; }
        };
        // Alfven (2-star) flux of one side (Eq. 65), weight w
        auto alfven_adj = [&](auto sd, double w) {
            constexpr bool left = decltype(sd)::value;
            const double* u = left ? ul : ur;
            const double* b = left ? bl : br;
            double* ub = left ? ulb : urb;
            double* bb = left ? blb : brb;
            const double s = left ? sl : sr;
            const double en = left ? enl : enr;
            const double* us = left ? usl : usr;
            const double* bs = left ? bsl : bsr;
            double* usb = left ? uslb : usrb;
            double* bsb = left ? bslb : bsrb;
            const double a = left ? alfl : alfr;
            const double sq = left ? sql : sqr;
            const double vbs = left ? vbsl : vbsr;
            double u2[5];
            u2[0] = us[0];
            for (int c = 0; c < 3; ++c) u2[1 + c] = us[0] * v2[c];
            u2[4] = has_energy ? (left ? us[4] - (b_sig * sq) * (vbs - vb2) : us[4] + (b_sig * sq) * (vbs - vb2)) : 0.0;
            const double cons[5] = {u[0], u[0] * u[1], u[0] * u[2], u[0] * u[3], en};
            double fsb[5] = {0, 0, 0, 0, 0}, consb[5] = {0, 0, 0, 0, 0}, u2b[5] = {0, 0, 0, 0, 0}, bfsb[2];
            double ab = 0.0, sb = 0.0;
            // out = ((fs + a*u2) - (a - s)*us) - s*cons
            const double ams = a - s;
            for (int c = 0; c < nc; ++c) {
                const double g = w * fb5[c];
                fsb[c] = g;
                ab = fm(g, u2[c] - us[c], ab);
                u2b[c] = g * a;
                usb[c] = fm(-g, ams, usb[c]);
                sb = fm(g, us[c] - cons[c], sb);
                consb[c] = -g * s;
            }
            for (int c = 1; c < 3; ++c) {
                const double g = w * bfb[c - 1];
                bfsb[c - 1] = g;
                ab = fm(g, b2[c] - bs[c], ab);
                b2b[c] = fm(g, a, b2b[c]);
                bsb[c] = fm(-g, ams, bsb[c]);
                sb = fm(g, bs[c] - b[c], sb);
                bb[c] = fm(-g, s, bb[c]);
            }
            double prb = 0.0, enb = 0.0;
            side_flux_adj(has_energy, u, b, left ? prl : prr, en, fsb, bfsb, ub, bb, prb, enb);
            cons_adj(has_energy, u, consb, ub, enb);
            // u2
            usb[0] += u2b[0];
            for (int c = 0; c < 3; ++c) {
                usb[0] = fm(u2b[1 + c], v2[c], usb[0]);
                v2b[c] = fm(u2b[1 + c], us[0], v2b[c]);
            }
            if (has_energy) {
                const double sgn = left ? -1.0 : 1.0;   // us4 -/+ (b_sig*sq)*(vbs - vb2)
                usb[4] += u2b[4];
                const double t = sgn * u2b[4];
                if (left) sqlb += t * b_sig * (vbs - vb2); else sqrb += t * b_sig * (vbs - vb2);
                if (left) vbslb += t * b_sig * sq; else vbsrb += t * b_sig * sq;
                vb2b -= t * b_sig * sq;
            }
            if (left) { alflb += ab; slb += sb; prlb += prb; enlb += enb; }
            else { alfrb += ab; srb += sb; prrb += prb; enrb += enb; }
        };

        if (bx_nz) {
            if (alfl > 0.0 || alfr < 0.0) {
                if (alfl > 0.0) star_adj(Side<true>{}, 1.0);
                else star_adj(Side<false>{}, 1.0);
            } else {
                if (sm > 0.0) alfven_adj(Side<true>{}, 1.0);
                else if (sm < 0.0) alfven_adj(Side<false>{}, 1.0);
                else { alfven_adj(Side<true>{}, 0.5); alfven_adj(Side<false>{}, 0.5); }
                // vb2 = (v2.b2)
                for (int c = 0; c < 3; ++c) {
                    v2b[c] = fm(vb2b, b2[c], v2b[c]);
                    b2b[c] = fm(vb2b, v2[c], b2b[c]);
                }
                // b2[1..2] = ((sql*bsr + sqr*bsl) + bsm*(vsr - vsl))/add
                double addb = 0.0, bsmb = 0.0;
                for (int c = 1; c < 3; ++c) {
                    const double nb = b2b[c] * radd;
                    addb = fm(-nb, b2[c], addb);
                    sqlb = fm(nb, bsr[c], sqlb);
                    bsrb[c] = fm(nb, sql, bsrb[c]);
                    sqrb = fm(nb, bsl[c], sqrb);
                    bslb[c] = fm(nb, sqr, bslb[c]);
                    bsmb = fm(nb, vsr[c] - vsl[c], bsmb);
                    vsrb[c] = fm(nb, bsm, vsrb[c]);
                    vslb[c] = fm(-nb, bsm, vslb[c]);
                }
                // b2[0] = 0.5*(bl0 + br0)
                blb[0] += 0.5 * b2b[0];
                brb[0] += 0.5 * b2b[0];
                // v2[0] = sm
                smb += v2b[0];
                // v2[1..2] = ((sql*vsl + sqr*vsr) + b_sig*(bsr - bsl))/add
                for (int c = 1; c < 3; ++c) {
                    const double nb = v2b[c] * radd;
                    addb = fm(-nb, v2[c], addb);
                    sqlb = fm(nb, vsl[c], sqlb);
                    vslb[c] = fm(nb, sql, vslb[c]);
                    sqrb = fm(nb, vsr[c], sqrb);
                    vsrb[c] = fm(nb, sqr, vsrb[c]);
                    bsrb[c] = fm(nb, b_sig, bsrb[c]);
                    bslb[c] = fm(-nb, b_sig, bslb[c]);
                }
                // bsm = b_sig*mul, mul = sql*sqr, add = sql + sqr
                const double mulb = bsmb * b_sig;
                sqlb += fm(mulb, sqr, addb);
                sqrb += fm(mulb, sql, addb);
            }
            // alfl = sm - |bl0|/sql ; alfr = sm + |br0|/sqr (only the selected branch used them)
            const double rsql = arcp(sql), rsqr = arcp(sqr);
            smb += alflb + alfrb;
            blb[0] = fm(-alflb * f_sign1(bl[0]), rsql, blb[0]);
            sqlb = fm(alflb * fabs(bl[0]), rsql * rsql, sqlb);
            brb[0] = fm(alfrb * f_sign1(br[0]), rsqr, brb[0]);
            sqrb = fm(-alfrb * fabs(br[0]), rsqr * rsqr, sqrb);
            // sql = sqrt(usl0)
            uslb[0] = fm(sqlb * 0.5, rsql, uslb[0]);
            usrb[0] = fm(sqrb * 0.5, rsqr, usrb[0]);
        } else {
            if (sm > 0.0) star_adj(Side<true>{}, 1.0);
            else if (sm < 0.0) star_adj(Side<false>{}, 1.0);
            else { star_adj(Side<true>{}, 0.5); star_adj(Side<false>{}, 0.5); }
        }

        // usl[4] = n4l/slsm with n4l = (((slvxl*enl) - (prl*ul1)) + (prt*sm)) + (bl0*(vbl - vbsl))
        auto us4_adj = [&](auto sd) {
            constexpr bool left = decltype(sd)::value;
            const double ub4 = left ? uslb[4] : usrb[4];
            if (!has_energy || ub4 == 0.0) return;
            const double rssm = left ? rslsm : rsrsm;
            const double n4b = ub4 * rssm;
            if (left) slsmb -= n4b * usl[4]; else srsmb -= n4b * usr[4];
            const double* u = left ? ul : ur;
            const double* b = left ? bl : br;
            double* ub = left ? ulb : urb;
            double* bb = left ? blb : brb;
            const double svx = left ? slvxl : srvxr;
            const double en = left ? enl : enr;
            const double pr = left ? prl : prr;
            const double vbs = left ? vbsl : vbsr;
            const double vb = left ? vbl : vbr;
            if (left) { slvxlb = fm(n4b, en, slvxlb); enlb = fm(n4b, svx, enlb); prlb = fm(-n4b, u[1], prlb); vbslb = fm(-n4b, b[0], vbslb); }
            else { srvxrb = fm(n4b, en, srvxrb); enrb = fm(n4b, svx, enrb); prrb = fm(-n4b, u[1], prrb); vbsrb = fm(-n4b, b[0], vbsrb); }
            prtb = fm(n4b, sm, prtb);
            smb = fm(n4b, prt, smb);
            const double vbb = n4b * b[0];                     // vb = (u1*b0 + u2*b1) + u3*b2
            ub[1] = fm(vbb, b[0], fm(-n4b, pr, ub[1]));
            ub[2] = fm(vbb, b[1], ub[2]);
            ub[3] = fm(vbb, b[2], ub[3]);
            bb[0] = fm(vbb, u[1], fm(n4b, vb - vbs, bb[0]));
            bb[1] = fm(vbb, u[2], bb[1]);
            bb[2] = fm(vbb, u[3], bb[2]);
        };
        us4_adj(Side<true>{});
        us4_adj(Side<false>{});
        // us[1..3] = us0 * vs[0..2]; us0 = dn/ssm
        auto side_part1 = [&](auto sd) {
            constexpr bool left = decltype(sd)::value;
            double* usb = left ? uslb : usrb;
            const double* us = left ? usl : usr;
            const double* vs = left ? vsl : vsr;
            double* vsb = left ? vslb : vsrb;
            const double rssm = left ? rslsm : rsrsm;
            for (int c = 0; c < 3; ++c) {
                usb[0] = fm(usb[1 + c], vs[c], usb[0]);
                vsb[c] = fm(usb[1 + c], us[0], vsb[c]);
            }
            const double t = usb[0] * rssm;
            if (left) { dn_lb += t; slsmb = fm(-t, us[0], slsmb); }
            else { dn_rb += t; srsmb = fm(-t, us[0], srsmb); }
        };
        side_part1(Side<true>{});
        side_part1(Side<false>{});
        // vbs = (vs0*bs0 + vs1*bs1) + vs2*bs2, vs0 = sm, bs0 = b0
        auto side_part2 = [&](auto sd) {
            constexpr bool left = decltype(sd)::value;
            const double vbsb = left ? vbslb : vbsrb;
            const double* vs = left ? vsl : vsr;
            const double* bs = left ? bsl : bsr;
            double* vsb = left ? vslb : vsrb;
            double* bsb = left ? bslb : bsrb;
            double* bb = left ? blb : brb;
            smb = fm(vbsb, bs[0], smb);
            bb[0] = fm(vbsb, vs[0], bb[0]);
            for (int c = 1; c < 3; ++c) {
                vsb[c] = fm(vbsb, bs[c], vsb[c]);
                bsb[c] = fm(vbsb, vs[c], bsb[c]);
            }
            smb += vsb[0];
        };
        side_part2(Side<true>{});
        side_part2(Side<false>{});
        // vs[c] = u[1+c] + k*(b[c] - bs[c]),  k = b0/dn
        auto side_part3 = [&](auto sd) {
            constexpr bool left = decltype(sd)::value;
            const double* b = left ? bl : br;
            double* ub = left ? ulb : urb;
            double* bb = left ? blb : brb;
            const double* bs = left ? bsl : bsr;
            double* vsb = left ? vslb : vsrb;
            double* bsb = left ? bslb : bsrb;
            const double k = left ? kl : kr;
            const double rdn = left ? rdnl : rdnr;
            double kb = 0.0;
            for (int c = 1; c < 3; ++c) {
                ub[1 + c] += vsb[c];
                kb = fm(vsb[c], b[c] - bs[c], kb);
                bb[c] = fm(vsb[c], k, bb[c]);
                bsb[c] = fm(-vsb[c], k, bsb[c]);
            }
            const double t = kb * rdn;
            bb[0] += t;
            if (left) dn_lb = fm(-t, k, dn_lb); else dn_rb = fm(-t, k, dn_rb);
        };
        side_part3(Side<true>{});
        side_part3(Side<false>{});
        // bs[1..2]: star formula or the HLL fallback (shared by both sides)
        double hll1b = 0.0, hll2b = 0.0;
        auto side_part4 = [&](auto sd) {
            constexpr bool left = decltype(sd)::value;
            const bool star = left ? starL : starR;
            double* bsb = left ? bslb : bsrb;
            if (star) {
                const double* b = left ? bl : br;
                const double* bs = left ? bsl : bsr;
                double* bb = left ? blb : brb;
                const double a = left ? aL : aR;
                const double rc = left ? rcL : rcR;
                double ab = 0.0, coeffb = 0.0;
                for (int c = 1; c < 3; ++c) {
                    const double t = bsb[c] * rc;
                    bb[c] = fm(t, a, bb[c]);
                    ab = fm(t, b[c], ab);
                    coeffb = fm(-t, bs[c], coeffb);
                }
                // a = dn*svx - b_lr ; coeff = dn*ssm - b_lr
                const double svx = left ? slvxl : srvxr;
                const double ssm = left ? slsm : srsm;
                const double dn = left ? dn_l : dn_r;
                const double dnb = fm(ab, svx, coeffb * ssm);
                if (left) { dn_lb += dnb; slvxlb = fm(ab, dn, slvxlb); slsmb = fm(coeffb, dn, slsmb); }
                else { dn_rb += dnb; srvxrb = fm(ab, dn, srvxrb); srsmb = fm(coeffb, dn, srsmb); }
                const double blrb = -ab - coeffb;
                blb[0] = fm(blrb, br[0], blb[0]);
                brb[0] = fm(blrb, bl[0], brb[0]);
            } else {
                hll1b += bsb[1];
                hll2b += bsb[2];
            }
        };
        side_part4(Side<true>{});
        side_part4(Side<false>{});
        if (hll1b != 0.0 || hll2b != 0.0) {
            // hll_c = ((sr*br_c - sl*bl_c) - (bcrf_c - bclf_c))/srmsl
            const double hb[3] = {0.0, hll1b, hll2b};
            const double hv[3] = {0.0, hll1, hll2};
            for (int c = 1; c < 3; ++c) {
                const double nb = hb[c] * rsrmsl;
                srmslb = fm(-nb, hv[c], srmslb);
                srb = fm(nb, br[c], srb);
                slb = fm(-nb, bl[c], slb);
                // -(bcrf_c - bclf_c); bcf_c = b_c*u1 - b0*u_{1+c}
                brb[c] = fm(nb, sr - ur[1], brb[c]);
                urb[1] = fm(-nb, br[c], urb[1]);
                brb[0] = fm(nb, ur[1 + c], brb[0]);
                urb[1 + c] = fm(nb, br[0], urb[1 + c]);
                blb[c] = fm(nb, ul[1] - sl, blb[c]);
                ulb[1] = fm(nb, bl[c], ulb[1]);
                blb[0] = fm(-nb, ul[1 + c], blb[0]);
                ulb[1 + c] = fm(-nb, bl[0], ulb[1 + c]);
            }
        }
        // prt = 0.5*((prl + dn_l*(sm - ul1)) + (prr + dn_r*(sm - ur1)))
        const double hp = 0.5 * prtb;
        prlb += hp;
        prrb += hp;
        dn_lb = fm(hp, sm - ul[1], dn_lb);
        dn_rb = fm(hp, sm - ur[1], dn_rb);
        smb = fm(hp, dn_l + dn_r, smb);
        ulb[1] = fm(-hp, dn_l, ulb[1]);
        urb[1] = fm(-hp, dn_r, urb[1]);
        // dn = u0*svx
        ulb[0] = fm(dn_lb, slvxl, ulb[0]);
        slvxlb = fm(dn_lb, ul[0], slvxlb);
        urb[0] = fm(dn_rb, srvxr, urb[0]);
        srvxrb = fm(dn_rb, ur[0], srvxrb);
        // speed differences
        slb += slvxlb + slsmb - srmslb;
        ulb[1] -= slvxlb;
        srb += srvxrb + srsmb + srmslb;
        urb[1] -= srvxrb;
        smb -= slsmb + srsmb;
        // sm
        double auxrb = 0.0, auxlb = 0.0;
        if (deg) {
            slb += smb / 2.0;
            srb += smb / 2.0;
        } else {
            const double rden = arcp(den);
            const double numb = smb * rden, denb = -numb * sm;
            auxrb = fm(numb, ur[1], denb);
            urb[1] = fm(numb, auxr, urb[1]);
            prrb -= numb;
            auxlb = fm(-numb, ul[1], -denb);
            ulb[1] = fm(-numb, auxl, ulb[1]);
            prlb += numb;
        }
        srb = fm(auxrb, ur[0], srb);
        urb[1] = fm(-auxrb, ur[0], urb[1]);
        urb[0] = fm(auxrb, sr - ur[1], urb[0]);
        slb = fm(auxlb, ul[0], slb);
        ulb[1] = fm(-auxlb, ul[0], ulb[1]);
        ulb[0] = fm(auxlb, sl - ul[1], ulb[0]);
    }
    // sl, sr
    if (minr) urb[1] += slb; else ulb[1] += slb;
    if (maxr) urb[1] += srb; else ulb[1] += srb;
    if (!dust) {
        const double cfb = srb - slb;
        if (cf > 0.0) {
            // cf = sqrt(0.5*cmax), c = (a + root)/u0, root = sqrt(a*a - 4*gp*b0^2), a = gp + bb, gp = g*p
            const double cmb = cfb * 0.25 * arcp(cf);
            auto cf_adj = [&](auto sd) {
                constexpr bool right = decltype(sd)::value;
                const double* u = right ? ur : ul;
                const double* b = right ? br : bl;
                double* ub = right ? urb : ulb;
                double* bb = right ? brb : blb;
                const double c = right ? cr : cl;
                const double a = right ? ar : al;
                const double root = right ? rootr : rootl;
                const double gp = right ? gpr : gpl;
                const double numb = cmb * arcp(u[0]);
                ub[0] = fm(-numb, c, ub[0]);
                double abb = numb, rootb = numb;
                double gpb = 0.0;
                if (root > 0.0) {
                    const double rb = rootb * 0.5 * arcp(root);   // d(root^2)
                    abb = fm(rb * 2.0, a, abb);
                    gpb = -rb * 4.0 * (b[0] * b[0]);
                    bb[0] = fm(-rb * (4.0 * gp) * 2.0, b[0], bb[0]);
                }
                gpb += abb;                                    // a = gp + bb
                for (int k = 0; k < 3; ++k) bb[k] = fm(abb * 2.0, b[k], bb[k]);
                ub[4] = fm(gpb, gamma, ub[4]);
            };
            if (cr > cl) cf_adj(Side<true>{});
            else cf_adj(Side<false>{});
        }
        pr_en_adj(true, gamma, ul, bl, prlb, enlb, ulb, blb);
        pr_en_adj(true, gamma, ur, br, prrb, enrb, urb, brb);
    }
}

// ---------------------------------------------------------------------------
// riemann_wrap for one face: gl/gr get the adjoints of the left/right states
// from the flux adjoint fb (all components of the swept state)
// ---------------------------------------------------------------------------
template <class PH>
PK_PHYS void riemann_adj(const double (&ql)[PH::NV], const double (&qr)[PH::NV], double ch, const PhysParams& pp,
                         const double (&fb)[PH::NV], double (&gl)[PH::NV], double (&gr)[PH::NV])
{
#pragma unroll
    for (int v = 0; v < PH::NV; ++v) {
        gl[v] = 0.0;
        gr[v] = 0.0;
    }
    if (PH::MHD) {
        // F_psi = ((ch*ch)*0.5)*((bxr+bxl) - (psr-psl)/ch) ; F_bx = 0.5*((psr+psl) - ch*(bxr-bxl))
        const double fp = fb[PH::IB + 3], fx = fb[PH::IB];
        const double h2 = (ch * ch) * 0.5;
        const double ph = fp * h2 * arcp(ch);
        gl[PH::IB] += fp * h2 + fx * 0.5 * ch;
        gr[PH::IB] += fp * h2 - fx * 0.5 * ch;
        gl[PH::IB + 3] += ph + fx * 0.5;
        gr[PH::IB + 3] += -ph + fx * 0.5;
    }
#pragma unroll
    for (int f = 0; f < PH::NFL; ++f) {
        const int b = PH::beg(f);
        const int nc = PH::ncomp(PH::kind(f));
        double ul[5] = {0, 0, 0, 0, 0}, ur[5] = {0, 0, 0, 0, 0}, ulb[5] = {0, 0, 0, 0, 0}, urb[5] = {0, 0, 0, 0, 0};
        double f5[5] = {0, 0, 0, 0, 0};
        for (int c = 0; c < nc; ++c) {
            ul[c] = ql[b + c];
            ur[c] = qr[b + c];
            f5[c] = fb[b + c];
        }
        if (PH::MHD) {
            double blv[3] = {0, 0, 0}, brv[3] = {0, 0, 0}, blb[3] = {0, 0, 0}, brb[3] = {0, 0, 0}, bfb[2] = {0, 0};
            if (PH::magn(f)) {
                for (int c = 0; c < 3; ++c) {
                    blv[c] = ql[PH::IB + c];
                    brv[c] = qr[PH::IB + c];
                }
                bfb[0] = fb[PH::IB + 1];
                bfb[1] = fb[PH::IB + 2];
            }
            hlld_adj(PH::has_en(f), pp.gam[f], ul, ur, blv, brv, f5, bfb, ulb, urb, blb, brb);
            if (PH::magn(f))
                for (int c = 0; c < 3; ++c) {
                    gl[PH::IB + c] += blb[c];
                    gr[PH::IB + c] += brb[c];
                }
        } else {
            hllc_adj(PH::has_en(f), pp.gam[f], ul, ur, f5, ulb, urb);
        }
        for (int c = 0; c < nc; ++c) {
            gl[b + c] += ulb[c];
            gr[b + c] += urb[c];
        }
    }
}

}  // namespace pk
