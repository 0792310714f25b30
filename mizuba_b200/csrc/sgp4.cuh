// SGP4 (near-Earth branch) as host/device functions, written from the
// published method: F. R. Hoots and R. L. Roehrich, "Models for Propagation
// of NORAD Element Sets", Spacetrack Report #3 (1980), with the revisions of
// D. A. Vallado, P. Crawford, R. Hujsak and T. S. Kelso, "Revisiting
// Spacetrack Report #3", AIAA 2006-6753: WGS72 constants, the un-Kozai mean
// motion, the perigee-dependent atmospheric parameter s, the Kepler solver
// with its 0.95 step limit, and the error codes 1 (mean eccentricity out of
// [-0.001, 1)), 2 (mean motion not positive), 4 (semi-latus rectum negative)
// and 6 (orbit decayed below the Earth's surface).
//
// mizuba propagates element sets with this model in make_sgp4_polyjectory
// (mizuba/make_sgp4_polyjectory.cpp:194-277, :699-745): WGS72, positions in
// km and velocities in km/s in the TEME frame, time in minutes since the
// element set's epoch.  Element sets with a period of 225 minutes or more
// belong to the deep-space branch (SDP4), which this header does not
// implement: sgp4_setup classifies them and the caller reports them.
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
    int isimp;     // 1: perigee below 220 km, the simplified drag terms
    int deep;      // 1: period >= 225 min (SDP4, not handled here)
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

MZB_HD inline int propagate(const sat &s, double t, double r[3], double v[3]);

// Set-up of one element set (angles in rad, n0 in rad/min, bstar in 1/RE).
// Returns 0, or the error code of the propagation at the epoch that ends the
// set-up.  Deep-space sets return 0 with s.deep = 1 and nothing else set.
MZB_HD inline int setup(double n0, double e0, double i0, double node0, double omega0, double m0, double bstar, sat &s)
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
    if (TWO_PI / s.no >= 225.0) {
        s.deep = 1;
        return 0;
    }
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

// Position [km] and velocity [km/s] at t minutes from the epoch.  Returns 0
// or an error code (1, 2, 4, 6); r and v are written in every case where
// the model produced them (code 6 is raised after they are computed).
MZB_HD inline int propagate(const sat &s, double t, double r[3], double v[3])
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
    const double inclm = s.inclo;
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
    const double sinim = std::sin(inclm), cosim = std::cos(inclm);
    // Long-period periodics.
    const double ep = em;
    const double axnl = ep * std::cos(argpm);
    double temp = 1.0 / (am * (1.0 - ep * ep));
    const double aynl = ep * std::sin(argpm) + temp * s.aycof;
    const double xl = mm + argpm + nodem + temp * s.xlcof * axnl;
    // Kepler's equation for the modified eccentric anomaly.
    const double u = std::fmod(xl - nodem, TWO_PI);
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
    const double mrt = rl * (1.0 - 1.5 * temp2 * betal * s.con41) + 0.5 * temp1 * s.x1mth2 * cos2u;
    su = su - 0.25 * temp2 * s.x7thm1 * sin2u;
    const double xnode = nodem + 1.5 * temp2 * cosim * sin2u;
    const double xinc = inclm + 1.5 * temp2 * cosim * sinim * cos2u;
    const double mvt = rdotl - nm * temp1 * s.x1mth2 * sin2u / k;
    const double rvdot = rvdotl + nm * temp1 * (s.x1mth2 * cos2u + 1.5 * s.con41) / k;
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
