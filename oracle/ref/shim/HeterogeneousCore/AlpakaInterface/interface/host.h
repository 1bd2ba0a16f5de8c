// Host-device accessor of CMSSW AlpakaInterface (serial subset, oracle only).
#pragma once
#include <alpaka/alpaka.hpp>
namespace cms::alpakatools {
  inline alpaka::DevCpu const& host() {
    static alpaka::DevCpu dev;
    return dev;
  }
}  // namespace cms::alpakatools
