// sky.cpp -- the procedural daylight environment: the Preetham, Shirley & Smits
// 1999 analytic sky ("A Practical Analytic Model for Daylight") baked into an
// equirectangular RGB map, as the reference packs a procedural-sky environment
// (bakePreethamSkyEquirect, shared-samplers/src/preethamSky.ts:151-313, used by
// pt-webgpu/src/scene/environmentPacking.ts:221-270).
//
// Per texel centre (row 0 at +y, u = atan2(z, x) / 2pi + 0.5) above 0.05 below
// the horizon:
//   sky    luminance Y and chromaticity x, y from the Perez distribution
//          F(theta, gamma) = (1 + A e^(B / cos theta)) (1 + C e^(D gamma) + E cos^2 gamma)
//          relative to its zenith value, with the paper's turbidity-linear
//          coefficients, zenith luminance and zenith chromaticity polynomials;
//          the zenith luminance scaled by `rayleigh` and `intensity`
//   haze   200 * mie_coefficient * HG(cos gamma, g) * 4 pi * Y_zenith
//   sun    a disc of angular radius 0.00436 rad and luminance 500 * Y_zenith,
//          deposited over the texels it covers (covered solid angle measured by
//          sub-texel quadrature, rescaled so the disc's total is exact, divided
//          by the renderer's texel measure dtheta dphi sin(theta_centre))
//   all three fade in over the 0.05 below the horizon, and x, y convert to
//   linear sRGB with the IEC 61966-2-1 matrix.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/vitrum_pt.h"
#include "vt_common.h"

namespace vt {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kSunRadius = 0.00436;  // radians

struct Perez {
  double A, B, C, D, E;
  double operator()(double cos_theta, double gamma) const {
    const double c = std::max(cos_theta, 1e-4);
    const double cg = std::cos(gamma);
    return (1.0 + A * std::exp(B / c)) * (1.0 + C * std::exp(D * gamma) + E * cg * cg);
  }
};

// Preetham 1999, appendix A.2: distribution coefficients linear in turbidity T,
// in the five-digit form the reference uses (preethamSky.ts:67-95)
Perez perez_luminance(double T) {
  return {0.17872 * T - 1.46303, -0.3554 * T + 0.42749, -0.02266 * T + 5.32505, 0.12064 * T - 2.57705,
          -0.06696 * T + 0.37027};
}
Perez perez_x(double T) {
  return {-0.01925 * T - 0.25922, -0.06651 * T + 0.00081, -0.00041 * T + 0.21247, -0.06409 * T - 0.89887,
          -0.00325 * T + 0.04517};
}
Perez perez_y(double T) {
  return {-0.01669 * T - 0.26078, -0.09495 * T + 0.00921, -0.00792 * T + 0.21023, -0.04405 * T - 1.65369,
          -0.01092 * T + 0.05291};
}

double henyey_greenstein(double cos_theta, double g) {
  const double d = 1.0 + g * g - 2.0 * g * std::max(-1.0, std::min(1.0, cos_theta));
  return (1.0 - g * g) / (4.0 * kPi * d * std::sqrt(d));
}

}  // namespace
}  // namespace vt

using namespace vt;

extern "C" vt_status vt_bake_preetham_sky(const vt_sky_desc* sky, int32_t width, int32_t height, float* rgb,
                                          size_t float_capacity) {
  return guard([&] {
    if (!sky || !rgb) fail(VT_ERR_INVALID_ARGUMENT, "null argument");
    if (width < 1 || height < 1 || width > 32768 || height > 32768)
      fail(VT_ERR_RANGE, "sky map dimensions must be in [1, 32768]");
    const size_t px = (size_t)width * (size_t)height;
    if (float_capacity < 3 * px) fail(VT_ERR_RANGE, "sky buffer too small");
    for (float v : {sky->sun_direction[0], sky->sun_direction[1], sky->sun_direction[2], sky->turbidity,
                    sky->rayleigh, sky->mie_coefficient, sky->mie_directional_g, sky->intensity})
      if (!std::isfinite(v)) fail(VT_ERR_RANGE, "sky parameters must be finite");
    double s[3] = {sky->sun_direction[0], sky->sun_direction[1], sky->sun_direction[2]};
    const double sl = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    if (sl < 1e-8) { s[0] = 0.0; s[1] = 1.0; s[2] = 0.0; }
    else for (double& x : s) x /= sl;
    const double T = std::max(1.5, std::min(30.0, (double)sky->turbidity));
    const double rayleigh = std::max(0.0, (double)sky->rayleigh);
    const double mie = 200.0 * std::max(0.0, (double)sky->mie_coefficient);
    const double g = std::max(-0.999999, std::min(0.999999, (double)sky->mie_directional_g));
    const double intensity = std::max(0.0, (double)sky->intensity);

    // zenith values (Preetham 1999, appendix A.2)
    const double ts = std::acos(std::max(-1.0, std::min(1.0, s[1])));
    const double chi = (4.0 / 9.0 - T / 120.0) * (kPi - 2.0 * ts);
    const double yz_raw = (4.0453 * T - 4.9710) * std::tan(chi) - 0.2155 * T + 2.4192;
    const double zenith_Y = std::max(1e-5, yz_raw) * rayleigh * intensity;
    const double ts2 = ts * ts, ts3 = ts2 * ts, T2 = T * T;
    const double zx = (0.00166 * ts3 - 0.00375 * ts2 + 0.00209 * ts) * T2 +
                      (-0.02903 * ts3 + 0.06377 * ts2 - 0.03202 * ts + 0.00394) * T +
                      (0.11693 * ts3 - 0.21196 * ts2 + 0.06052 * ts + 0.25886);
    const double zy = (0.00275 * ts3 - 0.00610 * ts2 + 0.00317 * ts) * T2 +
                      (-0.04214 * ts3 + 0.08970 * ts2 - 0.04153 * ts + 0.00516) * T +
                      (0.15346 * ts3 - 0.26756 * ts2 + 0.06670 * ts + 0.26688);
    const Perez pY = perez_luminance(T), px_ = perez_x(T), py_ = perez_y(T);
    const double nY = pY(1.0, ts), nx = px_(1.0, ts), ny = py_(1.0, ts);

    // sun disc: covered solid angle per texel by a 64 x 64 sub-texel midpoint
    // rule over the texels near the sun, rescaled to the disc's exact solid angle
    const double dth = kPi / height, dph = 2.0 * kPi / width;
    std::vector<double> sun(px, 0.0);
    {
      const double cos_r = std::cos(kSunRadius);
      const int r0 = std::max(0, (int)std::floor((ts - kSunRadius) / dth) - 1);
      const int r1 = std::min(height - 1, (int)std::floor((ts + kSunRadius) / dth) + 1);
      const double sun_u = std::atan2(s[2], s[0]) / (2.0 * kPi) + 0.5;  // texture longitude of the sun
      const double st = std::sin(ts);
      // columns near the sun (all of them when the disc reaches a pole)
      const double span = (st > 1e-9) ? std::min(kPi, kSunRadius / st + dph) : kPi;
      constexpr int kSub = 64;
      double total = 0.0;
      for (int row = r0; row <= r1; ++row) {
        std::vector<int> cols;
        if (span >= kPi) {
          for (int c = 0; c < width; ++c) cols.push_back(c);
        } else {
          const int c0 = (int)std::floor((sun_u - span / (2.0 * kPi)) * width) - 1;
          const int c1 = (int)std::floor((sun_u + span / (2.0 * kPi)) * width) + 1;
          for (int c = c0; c <= c1; ++c) cols.push_back(((c % width) + width) % width);
          std::sort(cols.begin(), cols.end());
          cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        }
        for (int col : cols) {
          double cov = 0.0;
          for (int a = 0; a < kSub; ++a) {
            const double th = (row + (a + 0.5) / kSub) * dth;
            const double sth = std::sin(th), cth = std::cos(th);
            for (int b = 0; b < kSub; ++b) {
              const double ph = ((col + (b + 0.5) / kSub) / width - 0.5) * 2.0 * kPi;
              const double d = sth * std::cos(ph) * s[0] + cth * s[1] + sth * std::sin(ph) * s[2];
              if (d >= cos_r) cov += sth;
            }
          }
          cov *= (dth / kSub) * (dph / kSub);
          sun[(size_t)row * width + col] = cov;
          total += cov;
        }
      }
      const double cap = 2.0 * kPi * (1.0 - cos_r);
      if (total > 0.0)
        for (int row = r0; row <= r1; ++row) {
          const double measure = dth * dph * std::max(std::sin((row + 0.5) * dth), 1e-6);
          for (int col = 0; col < width; ++col) sun[(size_t)row * width + col] *= cap / total / measure;
        }
    }

    for (int row = 0; row < height; ++row) {
      const double th = (row + 0.5) / height * kPi, cth = std::cos(th), sth = std::sin(th);
      for (int col = 0; col < width; ++col) {
        float* out = rgb + 3 * ((size_t)row * width + col);
        out[0] = out[1] = out[2] = 0.0f;
        if (cth < -0.05) continue;
        const double ph = ((col + 0.5) / width - 0.5) * 2.0 * kPi;
        const double cg = std::max(-1.0, std::min(1.0, sth * std::cos(ph) * s[0] + cth * s[1] + sth * std::sin(ph) * s[2]));
        const double gamma = std::acos(cg);
        const double c = std::max(cth, 1e-4);
        const double Y = nY > 1e-12 ? zenith_Y * pY(c, gamma) / nY : 0.0;
        const double x = nx > 1e-12 ? zx * px_(c, gamma) / nx : zx;
        const double y = ny > 1e-12 ? zy * py_(c, gamma) / ny : zy;
        const double fade = std::min(1.0, (cth + 0.05) / 0.05);
        const double sky_Y = std::max(0.0, Y) * fade;
        const double haze = mie * henyey_greenstein(cg, g) * 4.0 * kPi * zenith_Y * fade;
        const double sun_Y = sun[(size_t)row * width + col] * 500.0 * zenith_Y;
        const double total = sky_Y + haze + sun_Y;
        const bool sky_colour = sky_Y > 1e-12 || total < 1e-12;
        const double cx = sky_colour ? x : zx, cy = sky_colour ? y : zy;
        if (cy < 1e-10 || total < 0.0) continue;
        // xyY -> XYZ -> linear sRGB (IEC 61966-2-1, D65)
        const double X = total / cy * cx, Z = total / cy * (1.0 - cx - cy);
        out[0] = (float)std::max(0.0, 3.2406 * X - 1.5372 * total - 0.4986 * Z);
        out[1] = (float)std::max(0.0, -0.9689 * X + 1.8758 * total + 0.0415 * Z);
        out[2] = (float)std::max(0.0, 0.0557 * X - 0.2040 * total + 1.0570 * Z);
      }
    }
  });
}
