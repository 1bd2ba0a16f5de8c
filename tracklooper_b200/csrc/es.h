// Event setup (ES): the module structure-of-arrays, module connection map,
// pixel-seed module map and endcap strip orientations, built on the host from
// the LST geometry files and then uploaded once per device.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace lst {

  struct EsHost {
    uint16_t nModules = 0;
    uint16_t nLowerModules = 0;
    uint16_t pixelModuleIndex = 0;
    unsigned int nPixels = 0;  // length of connectedPixels
    // pt cut of the module and pixel maps: from the directory name's "_pt<x>"
    // suffix (OT800_IT615_pt0.6 -> 0.6), 0.8 without one
    float ptCut = 0.8f;

    // module arrays (index = re-assigned module index)
    std::vector<unsigned int> detIds;
    std::vector<uint16_t> moduleMap;  // nModules x 40
    std::vector<uint16_t> nConnectedModules;
    std::vector<unsigned int> mapdetId;  // sorted detIds
    std::vector<uint16_t> mapIdx;        // module index of mapdetId[i]
    std::vector<float> drdzs, dxdys, eta, r;
    std::vector<uint16_t> partnerModuleIndices;
    std::vector<short> layers, rings, modules, rods, subdets, sides;
    std::vector<uint8_t> isInverted, isLower, isAnchor, moduleType, moduleLayerType;
    std::vector<int> sdlLayers;
    std::vector<unsigned int> connectedPixels;

    // pixel map (per superbin)
    std::vector<unsigned int> connectedPixelsIndex, connectedPixelsSizes;
    std::vector<unsigned int> connectedPixelsIndexPos, connectedPixelsSizesPos;
    std::vector<unsigned int> connectedPixelsIndexNeg, connectedPixelsSizesNeg;

    // endcap 2S strip orientation, sorted by detId
    std::vector<unsigned int> geoMapDetId;
    std::vector<float> geoMapPhi;
    // per module: position of its detId in geoMapDetId (-1 when absent), so
    // that a hit finds its strip orientation without a search
    std::vector<int> geoMapIndex;

    // static per-module offsets and caps (lower modules + the pixel module)
    std::vector<int> mdOffset, mdCap;    // nLowerModules + 1
    std::vector<int> lsOffset, lsCap;    // nLowerModules + 1
    std::vector<int> t3CapIfUsed;        // nLowerModules: cap when the module has segments
    std::vector<int> t5CapIfEligible;    // nLowerModules: cap when eligible (-1: never eligible)
    // detId -> module index as an open-addressing hash table (linear probing,
    // slot = detId * 2654435761 >> (32 - bits)); value 0xffff marks an empty
    // slot.  Same answers as a binary search of mapdetId, in one or two probes.
    std::vector<unsigned int> detHashKey;
    std::vector<uint16_t> detHashVal;
    unsigned int detHashBits = 0;

    unsigned int nTotalMDs = 0;          // arena size incl. pixel MDs
    unsigned int nTotalSegments = 0;     // arena size incl. pixel segments
    unsigned int maxTriplets = 0;        // upper bound of the triplet arena
    unsigned int maxQuintuplets = 0;     // upper bound of the quintuplet arena
  };

  // Loads the geometry directory (e.g. .../OT800_IT615_pt0.8).  Returns an
  // empty string on success, else an error message.
  std::string loadEsHost(const std::string& geometryDir, EsHost& es);

  // The same event setup built by kernels on `device` from the files' raw
  // records, then copied into `es` (csrc/es_device.cu).  Same arrays, same
  // error messages.
  std::string buildEsOnDevice(const std::string& geometryDir, int device, EsHost& es);

  // The pt cut a geometry directory is built for (the number after its
  // name's last "_pt", 0.8 without one).
  float geometryPtCut(const std::string& dir);

}  // namespace lst
