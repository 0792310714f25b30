// SGP4 and SDP4 as host/device functions, written from the
// published method: F. R. Hoots and R. L. Roehrich, "Models for Propagation
// of NORAD Element Sets", Spacetrack Report #3 (1980), with the revisions of
// D. A. Vallado, P. Crawford, R. Hujsak and T. S. Kelso, "Revisiting
// Spacetrack Report #3", AIAA 2006-6753: WGS72 constants, the un-Kozai mean
// motion, the perigee-dependent atmospheric parameter s, the Kepler solver
// with its 0.95 step limit, and the error codes 1 (mean eccentricity out of
// [-0.001, 1)), 2 (mean motion not positive), 4 (semi-latus rectum negative)
// and 6 (orbit decayed below the Earth's surface).
//
// Element sets with a period of 225 minutes or more take the deep-space
// branch (SDP4, the report's DEEP section): lunar and solar secular rates and
// long-period periodics, and for 12-hour and one-day orbits the geopotential
// resonance terms integrated from epoch in 720-minute steps (Euler-Maclaurin),
// with the report's revisions above plus the 'a' (AFSPC) operation mode:
// Greenwich sidereal time at epoch by the AFSPC formula and the Lyddane
// node adjustment below 0.2 rad of perturbed inclination.
//
// mizuba propagates element sets with this model in make_sgp4_polyjectory
// (mizuba/make_sgp4_polyjectory.cpp:194-277, :699-745): WGS72, the 'a'
// operation mode, positions in km and velocities in km/s in the TEME frame,
// time in minutes since the element set's epoch, the epoch given to the
// set-up as days from 1950 Jan 0.0 UTC.
#pragma once

#include <cmath>
#include <cstdint>

#ifndef MZB_HD
#ifdef __CUDACC__
#define MZB_HD __host__ __device__
#else
#define MZB_HD
#endif
#endif
// The propagator's large functions are kept out of line on the device: the
// production kernel calls them from several places, and one copy of the code
// keeps the instruction cache and the register budget of its callers small.
#ifndef MZB_OUTLINE
#ifdef __CUDA_ARCH__
#define MZB_OUTLINE __noinline__
#else
#define MZB_OUTLINE
#endif
#endif

namespace mzb
{
namespace sgp4
{

// WGS72 (Spacetrack Report #3, Vallado et al. 2006 table 1).
constexpr double MU = 398600.8;           // km^3 / s^2
constexpr double RE = 6378.135;           // km
constexpr double J2 = 0.001082616;
constexpr double J3 = -0.00000253881;
constexpr double J4 = -0.00000165597;
constexpr double TWO_PI = 6.283185307179586476925286766559;
constexpr double X2O3 = 2.0 / 3.0;

// Mean motion unit: sqrt(mu / RE^3) in radians per minute, and the
// velocity unit RE * XKE / 60 in km/s.
MZB_HD inline double xke() { return 60.0 / std::sqrt(RE * RE * RE / MU); }

// One element set after set-up: the mean elements at epoch (un-Kozai mean
// motion no) and the secular and drag terms SGP4 derives from them.
struct sat {
    double no, ecco, inclo, nodeo, argpo, mo, bstar;
    double mdot, argpdot, nodedot, nodecf, omgcof, xmcof, xlcof, aycof;
    double cc1, cc4, cc5, d2, d3, d4, t2cof, t3cof, t4cof, t5cof;
    double eta, delmo, sinmao, con41, x1mth2, x7thm1;
    int isimp;     // 1: perigee below 220 km (or deep space), the simplified drag terms
    int deep;      // 1: period >= 225 min, the deep-space branch
    // Deep space: lunar-solar periodics, secular rates, resonance.
    double e3, ee2, peo, pgho, pho, pinco, plo, se2, se3, sgh2, sgh3, sgh4, sh2, sh3, si2, si3, sl2, sl3, sl4;
    double xgh2, xgh3, xgh4, xh2, xh3, xi2, xi3, xl2, xl3, xl4, zmol, zmos;
    double gsto, dedt, didt, dmdt, dnodt, domdt, del1, del2, del3, xfact, xlamo;
    double d2201, d2211, d3210, d3222, d4410, d4422, d5220, d5232, d5421, d5433;
    int irez;      // 0 none, 1 one-day (synchronous), 2 half-day resonance
};

// Un-Kozai mean motion (Spacetrack Report #3 eqs. for a1, delta1, a0,
// delta0) from the element set's mean motion n0 [rad/min].
MZB_HD inline double unkozai(double n0, double e0, double cosio)
{
    const double k = xke();
    const double ak = std::pow(k / n0, X2O3);
    const double omeosq = 1.0 - e0 * e0;
    const double rteosq = std::sqrt(omeosq);
    const double d1 = 0.75 * J2 * (3.0 * cosio * cosio - 1.0) / (rteosq * omeosq);
    double del = d1 / (ak * ak);
    const double adel = ak * (1.0 - del * del - del * (1.0 / 3.0 + 134.0 * del * del / 81.0));
    del = d1 / (adel * adel);
    return n0 / (1.0 + del);
}

// Whether an element set is propagated by the deep-space branch: period of
// 225 minutes or more at the un-Kozai mean motion.
MZB_HD inline bool is_deep_space(double n0, double e0, double i0)
{
    return TWO_PI / unkozai(n0, e0, std::cos(i0)) >= 225.0;
}

MZB_HD MZB_OUTLINE inline int propagate(const sat &s, double t, double r[3], double v[3]);

MZB_HD MZB_OUTLINE inline void deep_setup(sat &s, double epoch, double eccsq, double xpidot);

// Set-up of one element set (angles in rad, n0 in rad/min, bstar in 1/RE,
// epoch in days from 1950 Jan 0.0).  Returns 0, or the error code of the
// propagation at the epoch that ends the set-up.
MZB_HD MZB_OUTLINE inline int setup(double n0, double e0, double i0, double node0, double omega0, double m0, double bstar,
                        double epoch, sat &s)
{
    const double k = xke();
    const double cosio = std::cos(i0), sinio = std::sin(i0);
    const double cosio2 = cosio * cosio;
    s = sat{};
    s.ecco = e0;
    s.inclo = i0;
    s.nodeo = node0;
    s.argpo = omega0;
    s.mo = m0;
    s.bstar = bstar;
    s.no = unkozai(n0, e0, cosio);
    const double omeosq = 1.0 - e0 * e0;
    const double rteosq = std::sqrt(omeosq);
    const double ao = std::pow(k / s.no, X2O3);
    const double po = ao * omeosq;
    const double con42 = 1.0 - 5.0 * cosio2;
    s.con41 = -con42 - cosio2 - cosio2;
    const double posq = po * po;
    const double rp = ao * (1.0 - e0);
    // Atmospheric parameter s and (q0 - s)^4 for the perigee height
    // (Vallado et al. 2006 sec. "Initialization").
    s.isimp = rp < (220.0 / RE + 1.0) ? 1 : 0;
    double sfour = 78.0 / RE + 1.0;
    double qzms24 = std::pow((120.0 - 78.0) / RE, 4.0);
    const double perige = (rp - 1.0) * RE;
    if (perige < 156.0) {
        sfour = perige - 78.0;
        if (perige < 98.0) sfour = 20.0;
        qzms24 = std::pow((120.0 - sfour) / RE, 4.0);
        sfour = sfour / RE + 1.0;
    }
    const double pinvsq = 1.0 / posq;
    const double tsi = 1.0 / (ao - sfour);
    s.eta = ao * e0 * tsi;
    const double etasq = s.eta * s.eta;
    const double eeta = e0 * s.eta;
    const double psisq = std::fabs(1.0 - etasq);
    const double coef = qzms24 * std::pow(tsi, 4.0);
    const double coef1 = coef / std::pow(psisq, 3.5);
    const double cc2 = coef1 * s.no *
                       (ao * (1.0 + 1.5 * etasq + eeta * (4.0 + etasq)) +
                        0.375 * J2 * tsi / psisq * s.con41 * (8.0 + 3.0 * etasq * (8.0 + etasq)));
    s.cc1 = bstar * cc2;
    double cc3 = 0.0;
    if (e0 > 1.0e-4) cc3 = -2.0 * coef * tsi * (J3 / J2) * s.no * sinio / e0;
    s.x1mth2 = 1.0 - cosio2;
    s.cc4 = 2.0 * s.no * coef1 * ao * omeosq *
            (s.eta * (2.0 + 0.5 * etasq) + e0 * (0.5 + 2.0 * etasq) -
             J2 * tsi / (ao * psisq) *
                 (-3.0 * s.con41 * (1.0 - 2.0 * eeta + etasq * (1.5 - 0.5 * eeta)) +
                  0.75 * s.x1mth2 * (2.0 * etasq - eeta * (1.0 + etasq)) * std::cos(2.0 * omega0)));
    s.cc5 = 2.0 * coef1 * ao * omeosq * (1.0 + 2.75 * (etasq + eeta) + eeta * etasq);
    const double cosio4 = cosio2 * cosio2;
    const double temp1 = 1.5 * J2 * pinvsq * s.no;
    const double temp2 = 0.5 * temp1 * J2 * pinvsq;
    const double temp3 = -0.46875 * J4 * pinvsq * pinvsq * s.no;
    s.mdot = s.no + 0.5 * temp1 * rteosq * s.con41 + 0.0625 * temp2 * rteosq * (13.0 - 78.0 * cosio2 + 137.0 * cosio4);
    s.argpdot = -0.5 * temp1 * con42 + 0.0625 * temp2 * (7.0 - 114.0 * cosio2 + 395.0 * cosio4) +
                temp3 * (3.0 - 36.0 * cosio2 + 49.0 * cosio4);
    const double xhdot1 = -temp1 * cosio;
    s.nodedot = xhdot1 + (0.5 * temp2 * (4.0 - 19.0 * cosio2) + 2.0 * temp3 * (3.0 - 7.0 * cosio2)) * cosio;
    s.omgcof = bstar * cc3 * std::cos(omega0);
    s.xmcof = 0.0;
    if (e0 > 1.0e-4) s.xmcof = -X2O3 * coef * bstar / eeta;
    s.nodecf = 3.5 * omeosq * xhdot1 * s.cc1;
    s.t2cof = 1.5 * s.cc1;
    // Avoid the division by zero of the long-period term at i = 180 deg.
    const double opc = (std::fabs(cosio + 1.0) > 1.5e-12) ? (1.0 + cosio) : 1.5e-12;
    s.xlcof = -0.25 * (J3 / J2) * sinio * (3.0 + 5.0 * cosio) / opc;
    s.aycof = -0.5 * (J3 / J2) * sinio;
    s.delmo = std::pow(1.0 + s.eta * std::cos(m0), 3.0);
    s.sinmao = std::sin(m0);
    s.x7thm1 = 7.0 * cosio2 - 1.0;
    if (TWO_PI / s.no >= 225.0) {
        s.deep = 1;
        s.isimp = 1;
        deep_setup(s, epoch, e0 * e0, s.argpdot + s.nodedot);
    }
    if (s.isimp != 1) {
        const double cc1sq = s.cc1 * s.cc1;
        s.d2 = 4.0 * ao * tsi * cc1sq;
        const double temp = s.d2 * tsi * s.cc1 / 3.0;
        s.d3 = (17.0 * ao + sfour) * temp;
        s.d4 = 0.5 * temp * ao * tsi * (221.0 * ao + 31.0 * sfour) * s.cc1;
        s.t3cof = s.d2 + 2.0 * cc1sq;
        s.t4cof = 0.25 * (3.0 * s.d3 + s.cc1 * (12.0 * s.d2 + 10.0 * cc1sq));
        s.t5cof = 0.2 * (3.0 * s.d4 + 12.0 * s.cc1 * s.d3 + 6.0 * s.d2 * s.d2 + 15.0 * cc1sq * (2.0 * s.d2 + cc1sq));
    }
    double r[3], v[3];
    return propagate(s, 0.0, r, v);
}

// ---- Deep space (Spacetrack Report #3, DEEP; Vallado et al. 2006 dscom,
// dpper, dsinit, dspace).

// Lunar-solar terms of one element set (the report's common deep-space
// initialisation): the periodic coefficients kept in s, and the s*, ss*, z*,
// sz* coefficients dsinit needs, returned in dc.
struct deep_common {
    double s1, s2, s3, s4, s5, ss1, ss2, ss3, ss4, ss5;
    double z1, z3, z11, z13, z21, z23, z31, z33, sz1, sz3, sz11, sz13, sz21, sz23, sz31, sz33;
    double sinim, cosim, emsq, day, gam;
};

MZB_HD inline void deep_lunisolar(sat &s, double epoch, deep_common &dc)
{
    const double zes = 0.01675, zel = 0.05490, c1ss = 2.9864797e-6, c1l = 4.7968065e-7;
    const double zsinis = 0.39785416, zcosis = 0.91744867, zcosgs = 0.1945905, zsings = -0.98088458;
    const double nm = s.no, em = s.ecco;
    const double snodm = std::sin(s.nodeo), cnodm = std::cos(s.nodeo);
    const double sinomm = std::sin(s.argpo), cosomm = std::cos(s.argpo);
    const double sinim = std::sin(s.inclo), cosim = std::cos(s.inclo);
    const double emsq = em * em, betasq = 1.0 - emsq, rtemsq = std::sqrt(betasq);
    s.peo = s.pinco = s.plo = s.pgho = s.pho = 0.0;
    const double day = epoch + 18261.5; // tc = 0 at set-up
    const double xnodce = std::fmod(4.5236020 - 9.2422029e-4 * day, TWO_PI);
    const double stem = std::sin(xnodce), ctem = std::cos(xnodce);
    const double zcosil = 0.91375164 - 0.03568096 * ctem;
    const double zsinil = std::sqrt(1.0 - zcosil * zcosil);
    const double zsinhl = 0.089683511 * stem / zsinil;
    const double zcoshl = std::sqrt(1.0 - zsinhl * zsinhl);
    const double gam = 5.8351514 + 0.0019443680 * day;
    double zx = 0.39785416 * stem / zsinil;
    const double zy = zcoshl * ctem + 0.91744867 * zsinhl * stem;
    zx = std::atan2(zx, zy);
    zx = gam + zx - xnodce;
    const double zcosgl = std::cos(zx), zsingl = std::sin(zx);
    // Solar terms first (lsflg 1), then lunar (lsflg 2).
    double zcosg = zcosgs, zsing = zsings, zcosi = zcosis, zsini = zsinis, zcosh = cnodm, zsinh = snodm;
    double cc = c1ss;
    const double xnoi = 1.0 / nm;
    double s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0, s6 = 0, s7 = 0;
    double z1 = 0, z2 = 0, z3 = 0, z11 = 0, z12 = 0, z13 = 0, z21 = 0, z22 = 0, z23 = 0, z31 = 0, z32 = 0, z33 = 0;
    double ss1 = 0, ss2 = 0, ss3 = 0, ss4 = 0, ss5 = 0, ss6 = 0, ss7 = 0;
    double sz1 = 0, sz2 = 0, sz3 = 0, sz11 = 0, sz12 = 0, sz13 = 0, sz21 = 0, sz22 = 0, sz23 = 0, sz31 = 0,
           sz32 = 0, sz33 = 0;
    for (int lsflg = 1; lsflg <= 2; ++lsflg) {
        const double a1 = zcosg * zcosh + zsing * zcosi * zsinh;
        const double a3 = -zsing * zcosh + zcosg * zcosi * zsinh;
        const double a7 = -zcosg * zsinh + zsing * zcosi * zcosh;
        const double a8 = zsing * zsini;
        const double a9 = zsing * zsinh + zcosg * zcosi * zcosh;
        const double a10 = zcosg * zsini;
        const double a2 = cosim * a7 + sinim * a8;
        const double a4 = cosim * a9 + sinim * a10;
        const double a5 = -sinim * a7 + cosim * a8;
        const double a6 = -sinim * a9 + cosim * a10;
        const double x1 = a1 * cosomm + a2 * sinomm;
        const double x2 = a3 * cosomm + a4 * sinomm;
        const double x3 = -a1 * sinomm + a2 * cosomm;
        const double x4 = -a3 * sinomm + a4 * cosomm;
        const double x5 = a5 * sinomm;
        const double x6 = a6 * sinomm;
        const double x7 = a5 * cosomm;
        const double x8 = a6 * cosomm;
        z31 = 12.0 * x1 * x1 - 3.0 * x3 * x3;
        z32 = 24.0 * x1 * x2 - 6.0 * x3 * x4;
        z33 = 12.0 * x2 * x2 - 3.0 * x4 * x4;
        z1 = 3.0 * (a1 * a1 + a2 * a2) + z31 * emsq;
        z2 = 6.0 * (a1 * a3 + a2 * a4) + z32 * emsq;
        z3 = 3.0 * (a3 * a3 + a4 * a4) + z33 * emsq;
        z11 = -6.0 * a1 * a5 + emsq * (-24.0 * x1 * x7 - 6.0 * x3 * x5);
        z12 = -6.0 * (a1 * a6 + a3 * a5) + emsq * (-24.0 * (x2 * x7 + x1 * x8) - 6.0 * (x3 * x6 + x4 * x5));
        z13 = -6.0 * a3 * a6 + emsq * (-24.0 * x2 * x8 - 6.0 * x4 * x6);
        z21 = 6.0 * a2 * a5 + emsq * (24.0 * x1 * x5 - 6.0 * x3 * x7);
        z22 = 6.0 * (a4 * a5 + a2 * a6) + emsq * (24.0 * (x2 * x5 + x1 * x6) - 6.0 * (x4 * x7 + x3 * x8));
        z23 = 6.0 * a4 * a6 + emsq * (24.0 * x2 * x6 - 6.0 * x4 * x8);
        z1 = z1 + z1 + betasq * z31;
        z2 = z2 + z2 + betasq * z32;
        z3 = z3 + z3 + betasq * z33;
        s3 = cc * xnoi;
        s2 = -0.5 * s3 / rtemsq;
        s4 = s3 * rtemsq;
        s1 = -15.0 * em * s4;
        s5 = x1 * x3 + x2 * x4;
        s6 = x2 * x3 + x1 * x4;
        s7 = x2 * x4 - x1 * x3;
        if (lsflg == 1) {
            ss1 = s1, ss2 = s2, ss3 = s3, ss4 = s4, ss5 = s5, ss6 = s6, ss7 = s7;
            sz1 = z1, sz2 = z2, sz3 = z3, sz11 = z11, sz12 = z12, sz13 = z13;
            sz21 = z21, sz22 = z22, sz23 = z23, sz31 = z31, sz32 = z32, sz33 = z33;
            zcosg = zcosgl;
            zsing = zsingl;
            zcosi = zcosil;
            zsini = zsinil;
            zcosh = zcoshl * cnodm + zsinhl * snodm;
            zsinh = snodm * zcoshl - cnodm * zsinhl;
            cc = c1l;
        }
    }
    s.zmol = std::fmod(4.7199672 + 0.22997150 * day - gam, TWO_PI);
    s.zmos = std::fmod(6.2565837 + 0.017201977 * day, TWO_PI);
    // Solar periodic coefficients.
    s.se2 = 2.0 * ss1 * ss6;
    s.se3 = 2.0 * ss1 * ss7;
    s.si2 = 2.0 * ss2 * sz12;
    s.si3 = 2.0 * ss2 * (sz13 - sz11);
    s.sl2 = -2.0 * ss3 * sz2;
    s.sl3 = -2.0 * ss3 * (sz3 - sz1);
    s.sl4 = -2.0 * ss3 * (-21.0 - 9.0 * emsq) * zes;
    s.sgh2 = 2.0 * ss4 * sz32;
    s.sgh3 = 2.0 * ss4 * (sz33 - sz31);
    s.sgh4 = -18.0 * ss4 * zes;
    s.sh2 = -2.0 * ss2 * sz22;
    s.sh3 = -2.0 * ss2 * (sz23 - sz21);
    // Lunar periodic coefficients.
    s.ee2 = 2.0 * s1 * s6;
    s.e3 = 2.0 * s1 * s7;
    s.xi2 = 2.0 * s2 * z12;
    s.xi3 = 2.0 * s2 * (z13 - z11);
    s.xl2 = -2.0 * s3 * z2;
    s.xl3 = -2.0 * s3 * (z3 - z1);
    s.xl4 = -2.0 * s3 * (-21.0 - 9.0 * emsq) * zel;
    s.xgh2 = 2.0 * s4 * z32;
    s.xgh3 = 2.0 * s4 * (z33 - z31);
    s.xgh4 = -18.0 * s4 * zel;
    s.xh2 = -2.0 * s2 * z22;
    s.xh3 = -2.0 * s2 * (z23 - z21);
    dc = deep_common{s1,  s2,  s3,  s4,  s5,  ss1, ss2,  ss3,  ss4,  ss5,  z1,   z3,   z11,  z13,  z21,   z23,
                     z31, z33, sz1, sz3, sz11, sz13, sz21, sz23, sz31, sz33, sinim, cosim, emsq, day, gam};
}

// Deep-space secular rates and the resonance coefficients (dsinit), with
// Greenwich sidereal time at epoch by the AFSPC formula.
MZB_HD MZB_OUTLINE inline void deep_setup(sat &s, double epoch, double eccsq, double xpidot)
{
    const double k = xke();
    deep_common dc;
    deep_lunisolar(s, epoch, dc);
    // Greenwich sidereal time at epoch, AFSPC ('a' operation mode).
    {
        const double ts70 = epoch - 7305.0;
        const double ds70 = std::floor(ts70 + 1.0e-8);
        const double tfrac = ts70 - ds70;
        const double c1 = 1.72027916940703639e-2, thgr70 = 1.7321343856509374, fk5r = 5.07551419432269442e-15;
        const double c1p2p = c1 + TWO_PI;
        double g = std::fmod(thgr70 + c1 * ds70 + c1p2p * tfrac + ts70 * ts70 * fk5r, TWO_PI);
        if (g < 0.0) g += TWO_PI;
        s.gsto = g;
    }
    const double q22 = 1.7891679e-6, q31 = 2.1460748e-6, q33 = 2.2123015e-7;
    const double root22 = 1.7891679e-6, root44 = 7.3636953e-9, root54 = 2.1765803e-9;
    const double rptim = 4.37526908801129966e-3, root32 = 3.7393792e-7, root52 = 1.1428639e-7;
    const double znl = 1.5835218e-4, zns = 1.19459e-5;
    const double PI = TWO_PI / 2.0;
    const double nm = s.no;
    double em = s.ecco;
    const double inclm = s.inclo;
    const double sinim = dc.sinim, cosim = dc.cosim;
    double emsq = dc.emsq;
    s.irez = 0;
    if (nm < 0.0052359877 && nm > 0.0034906585) s.irez = 1;
    if (nm >= 8.26e-3 && nm <= 9.24e-3 && em >= 0.5) s.irez = 2;
    // Solar terms.
    const double ses = dc.ss1 * zns * dc.ss5;
    const double sis = dc.ss2 * zns * (dc.sz11 + dc.sz13);
    const double sls = -zns * dc.ss3 * (dc.sz1 + dc.sz3 - 14.0 - 6.0 * emsq);
    const double sghs = dc.ss4 * zns * (dc.sz31 + dc.sz33 - 6.0);
    double shs = -zns * dc.ss2 * (dc.sz21 + dc.sz23);
    if (inclm < 5.2359877e-2 || inclm > PI - 5.2359877e-2) shs = 0.0;
    if (sinim != 0.0) shs = shs / sinim;
    const double sgs = sghs - cosim * shs;
    // Lunar terms.
    s.dedt = ses + dc.s1 * znl * dc.s5;
    s.didt = sis + dc.s2 * znl * (dc.z11 + dc.z13);
    s.dmdt = sls - znl * dc.s3 * (dc.z1 + dc.z3 - 14.0 - 6.0 * emsq);
    const double sghl = dc.s4 * znl * (dc.z31 + dc.z33 - 6.0);
    double shll = -znl * dc.s2 * (dc.z21 + dc.z23);
    if (inclm < 5.2359877e-2 || inclm > PI - 5.2359877e-2) shll = 0.0;
    s.domdt = sgs + sghl;
    s.dnodt = shs;
    if (sinim != 0.0) {
        s.domdt = s.domdt - cosim / sinim * shll;
        s.dnodt = s.dnodt + shll / sinim;
    }
    // Resonance (theta at tc = 0).
    const double theta = std::fmod(s.gsto, TWO_PI);
    if (s.irez != 0) {
        const double aonv = std::pow(nm / k, X2O3);
        if (s.irez == 2) {
            // Half-day geopotential resonance.
            const double cosisq = cosim * cosim;
            const double emo = em, emsqo = emsq;
            em = s.ecco;
            emsq = eccsq;
            const double eoc = em * emsq;
            const double g201 = -0.306 - (em - 0.64) * 0.440;
            double g211, g310, g322, g410, g422, g520, g533, g521, g532;
            if (em <= 0.65) {
                g211 = 3.616 - 13.2470 * em + 16.2900 * emsq;
                g310 = -19.302 + 117.3900 * em - 228.4190 * emsq + 156.5910 * eoc;
                g322 = -18.9068 + 109.7927 * em - 214.6334 * emsq + 146.5816 * eoc;
                g410 = -41.122 + 242.6940 * em - 471.0940 * emsq + 313.9530 * eoc;
                g422 = -146.407 + 841.8800 * em - 1629.014 * emsq + 1083.4350 * eoc;
                g520 = -532.114 + 3017.977 * em - 5740.032 * emsq + 3708.2760 * eoc;
            } else {
                g211 = -72.099 + 331.819 * em - 508.738 * emsq + 266.724 * eoc;
                g310 = -346.844 + 1582.851 * em - 2415.925 * emsq + 1246.113 * eoc;
                g322 = -342.585 + 1554.908 * em - 2366.899 * emsq + 1215.972 * eoc;
                g410 = -1052.797 + 4758.686 * em - 7193.992 * emsq + 3651.957 * eoc;
                g422 = -3581.690 + 16178.110 * em - 24462.770 * emsq + 12422.520 * eoc;
                if (em > 0.715) g520 = -5149.66 + 29936.92 * em - 54087.36 * emsq + 31324.56 * eoc;
                else g520 = 1464.74 - 4664.75 * em + 3763.64 * emsq;
            }
            if (em < 0.7) {
                g533 = -919.22770 + 4988.6100 * em - 9064.7700 * emsq + 5542.21 * eoc;
                g521 = -822.71072 + 4568.6173 * em - 8491.4146 * emsq + 5337.524 * eoc;
                g532 = -853.66600 + 4690.2500 * em - 8624.7700 * emsq + 5341.4 * eoc;
            } else {
                g533 = -37995.780 + 161616.52 * em - 229838.20 * emsq + 109377.94 * eoc;
                g521 = -51752.104 + 218913.95 * em - 309468.16 * emsq + 146349.42 * eoc;
                g532 = -40023.880 + 170470.89 * em - 242699.48 * emsq + 115605.82 * eoc;
            }
            const double sini2 = sinim * sinim;
            const double f220 = 0.75 * (1.0 + 2.0 * cosim + cosisq);
            const double f221 = 1.5 * sini2;
            const double f321 = 1.875 * sinim * (1.0 - 2.0 * cosim - 3.0 * cosisq);
            const double f322 = -1.875 * sinim * (1.0 + 2.0 * cosim - 3.0 * cosisq);
            const double f441 = 35.0 * sini2 * f220;
            const double f442 = 39.3750 * sini2 * sini2;
            const double f522 = 9.84375 * sinim *
                                (sini2 * (1.0 - 2.0 * cosim - 5.0 * cosisq) +
                                 0.33333333 * (-2.0 + 4.0 * cosim + 6.0 * cosisq));
            const double f523 = sinim * (4.92187512 * sini2 * (-2.0 - 4.0 * cosim + 10.0 * cosisq) +
                                         6.56250012 * (1.0 + 2.0 * cosim - 3.0 * cosisq));
            const double f542 = 29.53125 * sinim * (2.0 - 8.0 * cosim + cosisq * (-12.0 + 8.0 * cosim + 10.0 * cosisq));
            const double f543 = 29.53125 * sinim * (-2.0 - 8.0 * cosim + cosisq * (12.0 + 8.0 * cosim - 10.0 * cosisq));
            const double xno2 = nm * nm, ainv2 = aonv * aonv;
            double temp1 = 3.0 * xno2 * ainv2;
            double temp = temp1 * root22;
            s.d2201 = temp * f220 * g201;
            s.d2211 = temp * f221 * g211;
            temp1 = temp1 * aonv;
            temp = temp1 * root32;
            s.d3210 = temp * f321 * g310;
            s.d3222 = temp * f322 * g322;
            temp1 = temp1 * aonv;
            temp = 2.0 * temp1 * root44;
            s.d4410 = temp * f441 * g410;
            s.d4422 = temp * f442 * g422;
            temp1 = temp1 * aonv;
            temp = temp1 * root52;
            s.d5220 = temp * f522 * g520;
            s.d5232 = temp * f523 * g532;
            temp = 2.0 * temp1 * root54;
            s.d5421 = temp * f542 * g521;
            s.d5433 = temp * f543 * g533;
            s.xlamo = std::fmod(s.mo + s.nodeo + s.nodeo - theta - theta, TWO_PI);
            s.xfact = s.mdot + s.dmdt + 2.0 * (s.nodedot + s.dnodt - rptim) - s.no;
            em = emo;
            emsq = emsqo;
        }
        if (s.irez == 1) {
            // One-day (synchronous) resonance.
            const double g200 = 1.0 + emsq * (-2.5 + 0.8125 * emsq);
            const double g310 = 1.0 + 2.0 * emsq;
            const double g300 = 1.0 + emsq * (-6.0 + 6.60937 * emsq);
            const double f220 = 0.75 * (1.0 + cosim) * (1.0 + cosim);
            const double f311 = 0.9375 * sinim * sinim * (1.0 + 3.0 * cosim) - 0.75 * (1.0 + cosim);
            double f330 = 1.0 + cosim;
            f330 = 1.875 * f330 * f330 * f330;
            double del1 = 3.0 * nm * nm * aonv * aonv;
            s.del2 = 2.0 * del1 * f220 * g200 * q22;
            s.del3 = 3.0 * del1 * f330 * g300 * q33 * aonv;
            s.del1 = del1 * f311 * g310 * q31 * aonv;
            s.xlamo = std::fmod(s.mo + s.nodeo + s.argpo - theta, TWO_PI);
            s.xfact = s.mdot + xpidot - rptim + s.dmdt + s.domdt + s.dnodt - s.no;
        }
    }
}

// Most Euler-Maclaurin steps of the resonance integration (about 270 years
// from epoch); a time further away is refused (propagate returns 10).
constexpr int MAX_RESONANCE_STEPS = 200000;

// Resonance integration from epoch to t (dspace): the mean motion and the
// mean longitude after Euler-Maclaurin steps of 720 minutes, then the mean
// anomaly.  Started from epoch on every call (the report's integrator keeps
// its state between calls, but restarting gives the same steps).  Returns
// false for a time that is not finite or needs more than
// MAX_RESONANCE_STEPS steps.
MZB_HD MZB_OUTLINE inline bool deep_resonance(const sat &s, double t, double theta, double nodem, double argpm, double &nm,
                                  double &mm)
{
    if (!(std::fabs(t) <= 720.0 * MAX_RESONANCE_STEPS)) return false;
    const double fasx2 = 0.13130908, fasx4 = 2.8843198, fasx6 = 0.37448087;
    const double g22 = 5.7686396, g32 = 0.95240898, g44 = 1.8014998, g52 = 1.0508330, g54 = 4.4108898;
    const double stepp = 720.0, stepn = -720.0, step2 = 259200.0;
    double atime = 0.0, xni = s.no, xli = s.xlamo;
    const double delt = t > 0.0 ? stepp : stepn;
    double xndt = 0, xldot = 0, xnddt = 0, ft = 0;
    // At most |t| / 720 + 1 passes, bounded above.
    for (int pass = 0; pass <= MAX_RESONANCE_STEPS; ++pass) {
        if (s.irez != 2) {
            xndt = s.del1 * std::sin(xli - fasx2) + s.del2 * std::sin(2.0 * (xli - fasx4)) +
                   s.del3 * std::sin(3.0 * (xli - fasx6));
            xldot = xni + s.xfact;
            xnddt = s.del1 * std::cos(xli - fasx2) + 2.0 * s.del2 * std::cos(2.0 * (xli - fasx4)) +
                    3.0 * s.del3 * std::cos(3.0 * (xli - fasx6));
            xnddt = xnddt * xldot;
        } else {
            const double xomi = s.argpo + s.argpdot * atime;
            const double x2omi = xomi + xomi;
            const double x2li = xli + xli;
            xndt = s.d2201 * std::sin(x2omi + xli - g22) + s.d2211 * std::sin(xli - g22) +
                   s.d3210 * std::sin(xomi + xli - g32) + s.d3222 * std::sin(-xomi + xli - g32) +
                   s.d4410 * std::sin(x2omi + x2li - g44) + s.d4422 * std::sin(x2li - g44) +
                   s.d5220 * std::sin(xomi + xli - g52) + s.d5232 * std::sin(-xomi + xli - g52) +
                   s.d5421 * std::sin(xomi + x2li - g54) + s.d5433 * std::sin(-xomi + x2li - g54);
            xldot = xni + s.xfact;
            xnddt = s.d2201 * std::cos(x2omi + xli - g22) + s.d2211 * std::cos(xli - g22) +
                    s.d3210 * std::cos(xomi + xli - g32) + s.d3222 * std::cos(-xomi + xli - g32) +
                    s.d5220 * std::cos(xomi + xli - g52) + s.d5232 * std::cos(-xomi + xli - g52) +
                    2.0 * (s.d4410 * std::cos(x2omi + x2li - g44) + s.d4422 * std::cos(x2li - g44) +
                           s.d5421 * std::cos(xomi + x2li - g54) + s.d5433 * std::cos(-xomi + x2li - g54));
            xnddt = xnddt * xldot;
        }
        if (std::fabs(t - atime) >= stepp) {
            xli = xli + xldot * delt + xndt * step2;
            xni = xni + xndt * delt + xnddt * step2;
            atime = atime + delt;
        } else {
            ft = t - atime;
            break;
        }
    }
    nm = xni + xndt * ft + xnddt * ft * ft * 0.5;
    const double xl = xli + xldot * ft + xndt * ft * ft * 0.5;
    if (s.irez != 1) mm = xl - 2.0 * nodem + 2.0 * theta;
    else mm = xl - nodem - argpm + theta;
    const double dndt = nm - s.no;
    nm = s.no + dndt;
    return true;
}

// Lunar-solar long-period periodics at t (dpper, applied: init = 'n'), with
// the 'a' operation mode's node handling.
MZB_HD MZB_OUTLINE inline void deep_periodics(const sat &s, double t, double &ep, double &inclp, double &nodep, double &argpp,
                                  double &mp)
{
    const double zns = 1.19459e-5, zes = 0.01675, znl = 1.5835218e-4, zel = 0.05490;
    const double PI = TWO_PI / 2.0;
    double zm = s.zmos + zns * t;
    double zf = zm + 2.0 * zes * std::sin(zm);
    double sinzf = std::sin(zf);
    double f2 = 0.5 * sinzf * sinzf - 0.25;
    double f3 = -0.5 * sinzf * std::cos(zf);
    const double ses = s.se2 * f2 + s.se3 * f3;
    const double sis = s.si2 * f2 + s.si3 * f3;
    const double sls = s.sl2 * f2 + s.sl3 * f3 + s.sl4 * sinzf;
    const double sghs = s.sgh2 * f2 + s.sgh3 * f3 + s.sgh4 * sinzf;
    const double shs = s.sh2 * f2 + s.sh3 * f3;
    zm = s.zmol + znl * t;
    zf = zm + 2.0 * zel * std::sin(zm);
    sinzf = std::sin(zf);
    f2 = 0.5 * sinzf * sinzf - 0.25;
    f3 = -0.5 * sinzf * std::cos(zf);
    const double sel = s.ee2 * f2 + s.e3 * f3;
    const double sil = s.xi2 * f2 + s.xi3 * f3;
    const double sll = s.xl2 * f2 + s.xl3 * f3 + s.xl4 * sinzf;
    const double sghl = s.xgh2 * f2 + s.xgh3 * f3 + s.xgh4 * sinzf;
    const double shll = s.xh2 * f2 + s.xh3 * f3;
    double pe = ses + sel, pinc = sis + sil, pl = sls + sll, pgh = sghs + sghl, ph = shs + shll;
    pe = pe - s.peo;
    pinc = pinc - s.pinco;
    pl = pl - s.plo;
    pgh = pgh - s.pgho;
    ph = ph - s.pho;
    inclp = inclp + pinc;
    ep = ep + pe;
    const double sinip = std::sin(inclp), cosip = std::cos(inclp);
    if (inclp >= 0.2) {
        ph = ph / sinip;
        pgh = pgh - cosip * ph;
        argpp = argpp + pgh;
        nodep = nodep + ph;
        mp = mp + pl;
    } else {
        // Lyddane's modification at low inclination.
        const double sinop = std::sin(nodep), cosop = std::cos(nodep);
        double alfdp = sinip * sinop, betdp = sinip * cosop;
        const double dalf = ph * cosop + pinc * cosip * sinop;
        const double dbet = -ph * sinop + pinc * cosip * cosop;
        alfdp = alfdp + dalf;
        betdp = betdp + dbet;
        nodep = std::fmod(nodep, TWO_PI);
        if (nodep < 0.0) nodep = nodep + TWO_PI; // 'a' mode
        double xls = mp + argpp + cosip * nodep;
        const double dls = pl + pgh - pinc * nodep * sinip;
        xls = xls + dls;
        const double xnoh = nodep;
        nodep = std::atan2(alfdp, betdp);
        if (nodep < 0.0) nodep = nodep + TWO_PI; // 'a' mode
        if (std::fabs(xnoh - nodep) > PI) {
            if (nodep < xnoh) nodep = nodep + TWO_PI;
            else nodep = nodep - TWO_PI;
        }
        mp = mp + pl;
        argpp = xls - mp - cosip * nodep;
    }
}

// Position [km] and velocity [km/s] at t minutes from the epoch.  Returns 0
// or an error code (1, 2, 4, 6); r and v are written in every case where
// the model produced them (code 6 is raised after they are computed).
MZB_HD MZB_OUTLINE inline int propagate(const sat &s, double t, double r[3], double v[3])
{
    const double k = xke();
    const double vkmpersec = RE * k / 60.0;
    // Secular gravity and atmospheric drag.
    const double xmdf = s.mo + s.mdot * t;
    const double argpdf = s.argpo + s.argpdot * t;
    const double nodedf = s.nodeo + s.nodedot * t;
    double argpm = argpdf;
    double mm = xmdf;
    const double t2 = t * t;
    double nodem = nodedf + s.nodecf * t2;
    double tempa = 1.0 - s.cc1 * t;
    double tempe = s.bstar * s.cc4 * t;
    double templ = s.t2cof * t2;
    if (s.isimp != 1) {
        const double delomg = s.omgcof * t;
        const double delmtemp = 1.0 + s.eta * std::cos(xmdf);
        const double delm = s.xmcof * (delmtemp * delmtemp * delmtemp - s.delmo);
        const double temp = delomg + delm;
        mm = xmdf + temp;
        argpm = argpdf - temp;
        const double t3 = t2 * t;
        const double t4 = t3 * t;
        tempa = tempa - s.d2 * t2 - s.d3 * t3 - s.d4 * t4;
        tempe = tempe + s.bstar * s.cc5 * (std::sin(mm) - s.sinmao);
        templ = templ + s.t3cof * t3 + t4 * (s.t4cof + t * s.t5cof);
    }
    double nm = s.no;
    double em = s.ecco;
    double inclm = s.inclo;
    if (s.deep) {
        // Secular lunar-solar rates and resonance (dspace).
        const double theta = std::fmod(s.gsto + t * 4.37526908801129966e-3, TWO_PI);
        em = em + s.dedt * t;
        inclm = inclm + s.didt * t;
        argpm = argpm + s.domdt * t;
        nodem = nodem + s.dnodt * t;
        mm = mm + s.dmdt * t;
        if (s.irez != 0 && !deep_resonance(s, t, theta, nodem, argpm, nm, mm)) return 10;
    }
    if (nm <= 0.0) return 2;
    const double am = std::pow(k / nm, X2O3) * tempa * tempa;
    nm = k / std::pow(am, 1.5);
    em = em - tempe;
    if (em >= 1.0 || em < -0.001) return 1;
    if (em < 1.0e-6) em = 1.0e-6;
    mm = mm + s.no * templ;
    double xlm = mm + argpm + nodem;
    nodem = std::fmod(nodem, TWO_PI);
    argpm = std::fmod(argpm, TWO_PI);
    xlm = std::fmod(xlm, TWO_PI);
    mm = std::fmod(xlm - argpm - nodem, TWO_PI);
    // Long-period periodics (plus the lunar-solar ones in deep space).
    double ep = em, xincp = inclm, argpp = argpm, nodep = nodem, mp = mm;
    double sinip = std::sin(inclm), cosip = std::cos(inclm);
    double aycof = s.aycof, xlcof = s.xlcof, con41 = s.con41, x1mth2 = s.x1mth2, x7thm1 = s.x7thm1;
    if (s.deep) {
        deep_periodics(s, t, ep, xincp, nodep, argpp, mp);
        if (xincp < 0.0) {
            xincp = -xincp;
            nodep = nodep + TWO_PI / 2.0;
            argpp = argpp - TWO_PI / 2.0;
        }
        if (ep < 0.0 || ep > 1.0) return 3;
        sinip = std::sin(xincp);
        cosip = std::cos(xincp);
        aycof = -0.5 * (J3 / J2) * sinip;
        const double opc = (std::fabs(cosip + 1.0) > 1.5e-12) ? (1.0 + cosip) : 1.5e-12;
        xlcof = -0.25 * (J3 / J2) * sinip * (3.0 + 5.0 * cosip) / opc;
    }
    const double axnl = ep * std::cos(argpp);
    double temp = 1.0 / (am * (1.0 - ep * ep));
    const double aynl = ep * std::sin(argpp) + temp * aycof;
    const double xl = mp + argpp + nodep + temp * xlcof * axnl;
    // Kepler's equation for the modified eccentric anomaly.
    const double u = std::fmod(xl - nodep, TWO_PI);
    double eo1 = u, tem5 = 9999.9, sineo1 = 0.0, coseo1 = 0.0;
    for (int ktr = 1; std::fabs(tem5) >= 1.0e-12 && ktr <= 10; ++ktr) {
        sineo1 = std::sin(eo1);
        coseo1 = std::cos(eo1);
        tem5 = 1.0 - coseo1 * axnl - sineo1 * aynl;
        tem5 = (u - aynl * coseo1 + axnl * sineo1 - eo1) / tem5;
        if (std::fabs(tem5) >= 0.95) tem5 = tem5 > 0.0 ? 0.95 : -0.95;
        eo1 = eo1 + tem5;
    }
    // Short-period periodics.
    const double ecose = axnl * coseo1 + aynl * sineo1;
    const double esine = axnl * sineo1 - aynl * coseo1;
    const double el2 = axnl * axnl + aynl * aynl;
    const double pl = am * (1.0 - el2);
    if (pl < 0.0) return 4;
    const double rl = am * (1.0 - ecose);
    const double rdotl = std::sqrt(am) * esine / rl;
    const double rvdotl = std::sqrt(pl) / rl;
    const double betal = std::sqrt(1.0 - el2);
    temp = esine / (1.0 + betal);
    const double sinu = am / rl * (sineo1 - aynl - axnl * temp);
    const double cosu = am / rl * (coseo1 - axnl + aynl * temp);
    double su = std::atan2(sinu, cosu);
    const double sin2u = (cosu + cosu) * sinu;
    const double cos2u = 1.0 - 2.0 * sinu * sinu;
    temp = 1.0 / pl;
    const double temp1 = 0.5 * J2 * temp;
    const double temp2 = temp1 * temp;
    if (s.deep) {
        const double cosisq = cosip * cosip;
        con41 = 3.0 * cosisq - 1.0;
        x1mth2 = 1.0 - cosisq;
        x7thm1 = 7.0 * cosisq - 1.0;
    }
    const double mrt = rl * (1.0 - 1.5 * temp2 * betal * con41) + 0.5 * temp1 * x1mth2 * cos2u;
    su = su - 0.25 * temp2 * x7thm1 * sin2u;
    const double xnode = nodep + 1.5 * temp2 * cosip * sin2u;
    const double xinc = xincp + 1.5 * temp2 * cosip * sinip * cos2u;
    const double mvt = rdotl - nm * temp1 * x1mth2 * sin2u / k;
    const double rvdot = rvdotl + nm * temp1 * (x1mth2 * cos2u + 1.5 * con41) / k;
    // Orientation vectors.
    const double sinsu = std::sin(su), cossu = std::cos(su);
    const double snod = std::sin(xnode), cnod = std::cos(xnode);
    const double sini = std::sin(xinc), cosi = std::cos(xinc);
    const double xmx = -snod * cosi, xmy = cnod * cosi;
    const double ux = xmx * sinsu + cnod * cossu;
    const double uy = xmy * sinsu + snod * cossu;
    const double uz = sini * sinsu;
    const double vx = xmx * cossu - cnod * sinsu;
    const double vy = xmy * cossu - snod * sinsu;
    const double vz = sini * cossu;
    r[0] = mrt * ux * RE;
    r[1] = mrt * uy * RE;
    r[2] = mrt * uz * RE;
    v[0] = (mvt * ux + rvdot * vx) * vkmpersec;
    v[1] = (mvt * uy + rvdot * vy) * vkmpersec;
    v[2] = (mvt * uz + rvdot * vz) * vkmpersec;
    if (mrt < 1.0) return 6;
    return 0;
}

} // namespace sgp4
} // namespace mzb
