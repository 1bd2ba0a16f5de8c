// A caller written against the reference's C++ API (SDL::Event<SDL::Acc>,
// SDL::LST<SDL::Acc>, SDL::loadAndFillES*), as bin/sdl.cc, code/core/
// trkCore.cc:844-904 and CMSSW's LSTProducer use it, compiled against
// include/lst_sdl.hpp.  Test infrastructure for tests/test_adapter.py and
// tests/test_gpu_adapter.py.
//
//   sdl_caller <input> <output>
//
// <input> holds one event twice: the Event-API inputs (5 hit vectors, 18 pLS
// vectors) and the CMSSW seed inputs of LST::run (13 float seed vectors,
// see_q, see_hitIdx as offsets + values, 4 ph2 vectors).  Each vector is a
// u64 element count then its elements.  <output> receives, in the same
// format: the getNumberOf* counters, the track-candidate store of the Event
// run (type, pixel seed index, 14 hit slots per candidate) and the four
// LST::run outputs (flattened hits, len, seedIdx, trackCandidateType).
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "lst_sdl.hpp"

namespace {
  struct Reader {
    std::ifstream f;
    template <typename T>
    std::vector<T> next() {
      uint64_t n = 0;
      if (!f.read(reinterpret_cast<char*>(&n), 8))
        throw std::runtime_error("truncated input");
      std::vector<T> v(n);
      if (n && !f.read(reinterpret_cast<char*>(v.data()), std::streamsize(n * sizeof(T))))
        throw std::runtime_error("truncated input");
      return v;
    }
  };
  struct Writer {
    std::ofstream f;
    template <typename T>
    void put(const std::vector<T>& v) {
      uint64_t n = v.size();
      f.write(reinterpret_cast<const char*>(&n), 8);
      f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(n * sizeof(T)));
    }
  };
}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::cerr << "usage: sdl_caller <input> <output>\n";
    return 2;
  }
  try {
    Reader in{std::ifstream(argv[1], std::ios::binary)};
    auto x = in.next<float>(), y = in.next<float>(), z = in.next<float>();
    auto detId = in.next<unsigned int>(), idx = in.next<unsigned int>();
    auto h0 = in.next<unsigned int>(), h1 = in.next<unsigned int>(), h2 = in.next<unsigned int>(),
         h3 = in.next<unsigned int>();
    auto dPhiChange = in.next<float>(), ptIn = in.next<float>(), ptErr = in.next<float>(), px = in.next<float>(),
         py = in.next<float>(), pz = in.next<float>(), eta = in.next<float>(), etaErr = in.next<float>(),
         phi = in.next<float>();
    auto charge = in.next<int>();
    auto seedIdx = in.next<unsigned int>();
    auto superbin = in.next<int>();
    auto pixelType = in.next<int8_t>();
    auto isQuad = in.next<char>();
    std::vector<std::vector<float>> see(13);
    for (auto& v : see)
      v = in.next<float>();
    auto see_q = in.next<int>();
    auto offsets = in.next<uint32_t>();
    auto flatIdx = in.next<int>();
    auto ph2_detId = in.next<unsigned int>();
    auto ph2_x = in.next<float>(), ph2_y = in.next<float>(), ph2_z = in.next<float>();
    std::vector<std::vector<int>> see_hitIdx;
    for (size_t i = 0; i + 1 < offsets.size(); ++i)
      see_hitIdx.emplace_back(flatIdx.begin() + offsets[i], flatIdx.begin() + offsets[i + 1]);

    // the event setup, as the reference's callers load it
    SDL::QueueAcc queue;
    auto esHost = SDL::loadAndFillESHost();
    auto esDevice = SDL::loadAndFillESDevice(queue, esHost.get());

    // the Event API in bin/sdl.cc's stage order
    SDL::Event<SDL::Acc> event(false, queue, esDevice.get());
    event.addHitToEvent(x, y, z, detId, idx);
    event.addPixelSegmentToEvent(h0, h1, h2, h3, dPhiChange, ptIn, ptErr, px, py, pz, eta, etaErr, phi, charge,
                                 seedIdx, superbin, pixelType, isQuad);
    event.createMiniDoublets();
    event.createSegmentsWithModuleMap();
    event.createTriplets();
    event.createQuintuplets();
    event.pixelLineSegmentCleaning();
    event.createPixelQuintuplets();
    event.createPixelTriplets();
    event.createTrackCandidates();

    Writer out{std::ofstream(argv[2], std::ios::binary)};
    std::vector<int64_t> counts = {event.getNumberOfHits(),
                                   event.getNumberOfMiniDoublets(),
                                   event.getNumberOfSegments(),
                                   event.getNumberOfTriplets(),
                                   event.getNumberOfQuintuplets(),
                                   event.getNumberOfPixelTriplets(),
                                   event.getNumberOfPixelQuintuplets(),
                                   event.getNumberOfTrackCandidates(),
                                   event.getNumberOfPT5TrackCandidates(),
                                   event.getNumberOfPT3TrackCandidates(),
                                   event.getNumberOfT5TrackCandidates(),
                                   event.getNumberOfPLSTrackCandidates()};
    out.put(counts);
    SDL::trackCandidatesBuffer<alpaka::DevCpu>& tc = *event.getTrackCandidates();
    const unsigned int nTC = *tc.nTrackCandidates;
    out.put(std::vector<short>(tc.trackCandidateType, tc.trackCandidateType + nTC));
    out.put(std::vector<int>(tc.pixelSeedIndex, tc.pixelSeedIndex + nTC));
    out.put(std::vector<unsigned int>(tc.hitIndices, tc.hitIndices + 14 * size_t(nTC)));
    SDL::miniDoubletsBuffer<alpaka::DevCpu>& md = *event.getMiniDoublets();
    out.put(std::vector<unsigned int>(md.nMDs, md.nMDs + esDevice->nLowerModules + 1));

    // LST::run on the CMSSW inputs
    SDL::LST<SDL::Acc> lst;
    lst.run(queue, false, esDevice.get(), see[0], see[1], see[2], see[3], see[4], see[5], see[6], see[7], see[8],
            see[9], see[10], see[11], see[12], see_q, see_hitIdx, ph2_detId, ph2_x, ph2_y, ph2_z);
    std::vector<unsigned int> flat;
    for (const auto& h : lst.hits())
      flat.insert(flat.end(), h.begin(), h.end());
    out.put(flat);
    out.put(lst.len());
    out.put(lst.seedIdx());
    out.put(lst.trackCandidateType());
  } catch (const std::exception& e) {
    std::cerr << "sdl_caller: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
