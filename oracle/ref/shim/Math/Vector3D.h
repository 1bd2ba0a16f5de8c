// Subset of ROOT's GenVector XYZVector (Math/Vector3D.h) used by the LST
// reference's seed conversion, SDL/LST.cc:9-10,163-174,175-365.  ROOT is not
// available here, so this header restates the published GenVector algorithms
// (ROOT 6.30, the series CMSSW_14_1_0_pre3 builds against):
//   XYZVector        = DisplacementVector3D<Cartesian3D<double>>, double
//                      components, constructible from three scalars
//   Rho()            = sqrt(x*x + y*y)
//   R()              = sqrt(x*x + y*y + z*z)
//   Phi()            = 0 if x == y == 0, else atan2(y, x)
//   Eta()            = Impl::Eta_FromRhoZ(Rho(), z): for rho > 0 and
//                      |z/rho| < eps^-1/4 the exact asinh form
//                      log(z/rho + sqrt((z/rho)^2 + 1)); beyond it the first
//                      order expansion log(2 z/rho + 0.5 rho/z) (z > 0) or
//                      -log(-2 z/rho) (z < 0); for rho == 0: 0 if z == 0,
//                      else z +- etaMax with etaMax the long-double constant
//                      log(LDBL_MAX/256) - log(LDBL_TRUE_MIN*256) + 16 log 2
//   operator-        = componentwise difference
// Test infrastructure for the parity oracle only.
#pragma once

#include <cfloat>
#include <cmath>
#include <limits>

namespace ROOT {
  namespace Math {

    namespace lstref_detail {
      inline double etaMax() {
        return static_cast<double>(std::log(LDBL_MAX / 256.0L) - std::log(LDBL_TRUE_MIN * 256.0L) +
                                   16.0 * std::log(2.0));
      }

      inline double etaFromRhoZ(double rho, double z) {
        if (rho > 0) {
          static const double bigZScaled = std::pow(std::numeric_limits<double>::epsilon(), -0.25);
          const double zs = z / rho;
          if (std::fabs(zs) < bigZScaled)
            return std::log(zs + std::sqrt(zs * zs + 1.0));
          return z > 0 ? std::log(2.0 * zs + 0.5 / zs) : -std::log(-2.0 * zs);
        }
        if (z == 0)
          return 0;
        return z > 0 ? z + etaMax() : z - etaMax();
      }
    }  // namespace lstref_detail

    class XYZVector {
    public:
      XYZVector() = default;
      XYZVector(double x, double y, double z) : fX(x), fY(y), fZ(z) {}

      double x() const { return fX; }
      double y() const { return fY; }
      double z() const { return fZ; }
      double X() const { return fX; }
      double Y() const { return fY; }
      double Z() const { return fZ; }
      double Perp2() const { return fX * fX + fY * fY; }
      double Mag2() const { return fX * fX + fY * fY + fZ * fZ; }
      double rho() const { return std::sqrt(Perp2()); }
      double r() const { return std::sqrt(Mag2()); }
      double phi() const { return (fX == 0.0 && fY == 0.0) ? 0.0 : std::atan2(fY, fX); }
      double eta() const { return lstref_detail::etaFromRhoZ(rho(), fZ); }
      double Rho() const { return rho(); }
      double R() const { return r(); }
      double Phi() const { return phi(); }
      double Eta() const { return eta(); }

      XYZVector operator-(const XYZVector& o) const { return XYZVector(fX - o.fX, fY - o.fY, fZ - o.fZ); }
      XYZVector operator+(const XYZVector& o) const { return XYZVector(fX + o.fX, fY + o.fY, fZ + o.fZ); }

    private:
      double fX = 0, fY = 0, fZ = 0;
    };

  }  // namespace Math
}  // namespace ROOT
