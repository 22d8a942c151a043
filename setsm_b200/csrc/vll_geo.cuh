// vll_geo.cuh -- map projection on the device, shared by the kernels that
// rasterise orthoimage coordinates.  Includers compile with -fmad=false so the
// arithmetic rounds as the reference's host code does.
#pragma once

#include "vll_ddmath.cuh"
#include "vll_device.cuh"

namespace vll {

// ps2wgs_single, CoordConversion.cpp:396-490, on the device.  Same formulas
// and operation order; the transcendental functions are the correctly
// rounded ones of vll_ddmath.cuh (the host's C library rounds the same way
// for all but about 0.1% of arguments).
static __device__ __noinline__ double2 ps2wgs_dev(const vll_transparam &p, double X, double Y) {
    if (p.projection == 1) {
        const double a = p.a, e = p.e, lambda_0 = p.lambda_0, t_c = p.t_c, m_c = p.m_c;
        const int pm = p.pm;
        const double e2 = e * e, e4 = e2 * e2, e6 = e2 * e4, e8 = e4 * e4;
        const double x = X * pm, y = Y * pm;
        const double rho = sqrt(x * x + y * y);
        const double t = rho * t_c / (a * m_c);
        const double chi = kPi / 2 - 2 * ddm::atan_cr(t);
        double phi = chi + (e2 / 2 + 5 * e4 / 24 + e6 / 12 + 13 * e8 / 360) * ddm::sin_cr(2 * chi) +
                     (7 * e4 / 48 + 29 * e6 / 240 + 811 * e8 / 11520) * ddm::sin_cr(4 * chi) +
                     (7 * e6 / 120 + 81 * e8 / 1120) * ddm::sin_cr(6 * chi) +
                     (4279 * e8 / 161280) * ddm::sin_cr(8 * chi);
        double lambda = lambda_0 + ddm::atan2_cr(x, -y);
        phi = pm * phi;
        lambda = pm * lambda;
        if (lambda > kPi)
            lambda = lambda - 2 * kPi;
        else if (lambda < -kPi)
            lambda = lambda + 2 * kPi;
        return make_double2(180 / kPi * lambda, 180 / kPi * phi);
    }
    const int hemis = p.pm;
    const double e2c = p.e2cuadrada, c = p.c;
    const double X0 = X - 500000;
    double Yv = Y;
    if (hemis < 0) Yv = Yv - 10000000;
    const int S = ((p.utm_zone * 6) - 183);
    const double lat = Yv / (6366197.724 * 0.9996);
    const double cl = ddm::cos_cr(lat);
    const double v = (c / (sqrt(1.0 + (e2c * (cl * cl))))) * 0.9996;
    const double a = X0 / v;
    const double a1 = ddm::sin_cr(2 * lat);
    const double a2 = a1 * (cl * cl);
    const double j2 = lat + (a1 / 2.0);
    const double j4 = ((3 * j2) + a2) / 4.0;
    const double j6 = ((5 * j4) + (a2 * (cl * cl))) / 3;
    const double alfa = (3 / 4.0) * e2c;
    const double beta = (5 / 3.0) * alfa * alfa;
    const double gama = (35 / 27.0) * alfa * alfa * alfa;
    const double Bm = 0.9996 * c * (lat - alfa * j2 + beta * j4 - gama * j6);
    const double b = (Yv - Bm) / v;
    const double Epsi = ((e2c * a * a) / 2.0) * (cl * cl);
    const double Eps = a * (1 - (Epsi / 3.0));
    const double nab = (b * (1 - Epsi)) + lat;
    const double senoheps = (ddm::exp_cr(Eps) - ddm::exp_cr(-Eps)) / 2;
    const double Delt = ddm::atan_cr(senoheps / (ddm::cos_cr(nab)));
    const double TaO = ddm::atan_cr(ddm::cos_cr(Delt) * ddm::tan_cr(nab));
    const double lon_o = (Delt * (180 / kPi)) + S;
    const double lat_o = (lat + (1 + e2c * (cl * cl) - (3 / 2.0) * e2c * ddm::sin_cr(lat) * cl * (TaO - lat)) *
                                    (TaO - lat)) *
                         (180 / kPi);
    return make_double2(lon_o, lat_o);
}

}  // namespace vll
