// Serial-backend subset of CMSSW HeterogeneousCore/AlpakaInterface config.h
// used by the LST reference sources.  Test infrastructure for the parity
// oracle only (see alpaka/alpaka.hpp in this directory).
#pragma once
#include <alpaka/alpaka.hpp>

namespace alpaka_common {
  using Idx = uint32_t;
  using Extent = uint32_t;
  using Dim1D = alpaka::DimInt<1u>;
  using Dim2D = alpaka::DimInt<2u>;
  using Dim3D = alpaka::DimInt<3u>;
  template <typename TDim>
  using Vec = alpaka::Vec<TDim, Idx>;
  using Vec1D = Vec<Dim1D>;
  using Vec3D = Vec<Dim3D>;
  template <typename TDim>
  using WorkDiv = alpaka::WorkDivMembers<TDim, Idx>;
  using WorkDiv1D = WorkDiv<Dim1D>;
  using WorkDiv3D = WorkDiv<Dim3D>;
  using DevHost = alpaka::DevCpu;
  using PlatformHost = alpaka::PlatformCpu;
}  // namespace alpaka_common

namespace alpaka_serial_sync {
  using namespace alpaka_common;
  using Platform = alpaka::PlatformCpu;
  using Device = alpaka::DevCpu;
  using Queue = alpaka::QueueCpuBlocking;
  template <typename TDim>
  using Acc = alpaka::AccCpuSerial<TDim, Idx>;
  using Acc1D = Acc<Dim1D>;
  using Acc3D = Acc<Dim3D>;
}  // namespace alpaka_serial_sync

#define ALPAKA_ACCELERATOR_NAMESPACE alpaka_serial_sync
