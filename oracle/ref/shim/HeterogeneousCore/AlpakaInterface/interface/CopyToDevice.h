// Primary template of CMSSW's CopyToDevice trait (oracle only).
#pragma once
namespace cms::alpakatools {
  template <typename T>
  struct CopyToDevice;
}  // namespace cms::alpakatools
