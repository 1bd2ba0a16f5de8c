// Event-setup loader: restates SDL/ModuleMethods.h:33-416 (module re-indexing,
// derived module quantities, partner modules, module map, pixel map),
// SDL/ModuleConnectionMap.cc:9-50, SDL/EndcapGeometry.cc:13-70 and
// SDL/TiltedGeometry.cc:5-49 on the host, plus the static per-module
// occupancy caps of SDL/MiniDoublet.h:994-1082 and SDL/Segment.h:912-1008.
#include "es.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <fstream>
#include <map>

#include "lst_md.h"

namespace lst {

  namespace {

    template <typename T>
    bool readRecords(const std::string& path, std::vector<T>& out) {
      std::ifstream f(path, std::ios::binary);
      if (!f.is_open())
        return false;
      T rec;
      while (f.read(reinterpret_cast<char*>(&rec), sizeof(T)))
        out.push_back(rec);
      return true;
    }

#pragma pack(push, 1)
    struct CentroidRec {
      uint32_t detId;
      float x, y, z;
      int32_t type;
    };
    struct PairRec {
      uint32_t detId;
      float a, b;
    };
#pragma pack(pop)

    // {u32 key, u32 n, n x u32} records; a later record with the same key
    // replaces an earlier one; a truncated trailing record is ignored, as
    // SDL/ModuleConnectionMap.cc:17-48 drops it at end of file.  A record
    // whose n exceeds what is left of the file is such a record: it is
    // dropped before anything is allocated for it, so a corrupt count cannot
    // ask for gigabytes.
    bool readConnectionMap(const std::string& path, std::map<uint32_t, std::vector<uint32_t>>& out) {
      std::ifstream f(path, std::ios::binary | std::ios::ate);
      if (!f.is_open())
        return false;
      const std::streamoff fileSize = f.tellg();
      f.seekg(0);
      while (true) {
        uint32_t key, n;
        if (!f.read(reinterpret_cast<char*>(&key), 4) || !f.read(reinterpret_cast<char*>(&n), 4))
          break;
        const std::streamoff left = fileSize - std::streamoff(f.tellg());
        if (std::streamoff(n) > left / 4)
          break;
        std::vector<uint32_t> v(n);
        if (n && !f.read(reinterpret_cast<char*>(v.data()), std::streamsize(n) * 4))
          break;
        out[key] = std::move(v);
      }
      return true;
    }

    bool parseIsInverted(short subdet, short side, short module, short layer) {
      if (subdet == Endcap) {
        if (side == NegZ)
          return module % 2 == 1;
        if (side == PosZ)
          return module % 2 == 0;
        return false;
      }
      if (subdet == Barrel) {
        if (side == Center) {
          if (layer <= 3)
            return module % 2 == 1;
          if (layer >= 4)
            return module % 2 == 0;
          return false;
        }
        if (side == NegZ or side == PosZ) {
          if (layer <= 2)
            return module % 2 == 1;
          if (layer == 3)
            return module % 2 == 0;
          return false;
        }
        return false;
      }
      return false;
    }

    bool parseIsLower(bool isInverted, unsigned int detId) { return isInverted ? !(detId & 1) : (detId & 1); }

    unsigned int partnerDetId(unsigned int detId, bool isLower, bool isInverted) {
      return isLower ? (isInverted ? detId - 1 : detId + 1) : (isInverted ? detId + 1 : detId - 1);
    }

  }  // namespace

  // detId -> module index hash of EsHost::detHashKey / detHashVal.
  void buildDetHash(EsHost& es) {
    unsigned int bits = 4;
    while ((1u << bits) < 2u * es.mapdetId.size())
      ++bits;
    es.detHashBits = bits;
    const unsigned int size = 1u << bits, mask = size - 1;
    es.detHashKey.assign(size, 0u);
    es.detHashVal.assign(size, uint16_t(0xffff));
    for (size_t i = 0; i < es.mapdetId.size(); ++i) {
      const unsigned int key = es.mapdetId[i];
      unsigned int slot = (key * 2654435761u) >> (32 - bits);
      while (es.detHashVal[slot] != 0xffff && es.detHashKey[slot] != key)
        slot = (slot + 1) & mask;
      es.detHashKey[slot] = key;
      es.detHashVal[slot] = es.mapIdx[i];
    }
  }

  // The pt cut a geometry directory is built for: the number after the last
  // "_pt" of its name (OT800_IT615_pt0.6 -> 0.6), 0.8 when there is none.
  float geometryPtCut(const std::string& dir) {
    std::string name = dir;
    while (!name.empty() && name.back() == '/')
      name.pop_back();
    const size_t slash = name.find_last_of('/');
    if (slash != std::string::npos)
      name = name.substr(slash + 1);
    const size_t at = name.rfind("_pt");
    if (at == std::string::npos)
      return 0.8f;
    char* end = nullptr;
    const float v = std::strtof(name.c_str() + at + 3, &end);
    return (end != name.c_str() + at + 3 && v > 0.f) ? v : 0.8f;
  }

  std::string loadEsHost(const std::string& dir, EsHost& es) {
    es.ptCut = geometryPtCut(dir);
    std::vector<CentroidRec> cents;
    if (!readRecords(dir + "/sensor_centroids.bin", cents) || cents.empty())
      return "unable to read " + dir + "/sensor_centroids.bin";
    std::vector<PairRec> endcapRecs, tiltedRecs;
    if (!readRecords(dir + "/endcap_orientation.bin", endcapRecs))
      return "unable to read " + dir + "/endcap_orientation.bin";
    if (!readRecords(dir + "/tilted_barrel_orientation.bin", tiltedRecs))
      return "unable to read " + dir + "/tilted_barrel_orientation.bin";
    std::map<uint32_t, std::vector<uint32_t>> connections;
    if (!readConnectionMap(dir + "/module_connection_tracing_merged.bin", connections))
      return "unable to read " + dir + "/module_connection_tracing_merged.bin";

    std::map<uint32_t, float> endcapDxdy, endcapPhi, tiltedDrdz, tiltedDxdy;
    for (auto& r : endcapRecs) {
      endcapDxdy[r.detId] = r.a;
      endcapPhi[r.detId] = r.b;
    }
    for (auto& r : tiltedRecs) {
      tiltedDrdz[r.detId] = r.a;
      tiltedDxdy[r.detId] = r.b;
    }

    std::map<uint32_t, CentroidRec> byDetId;
    for (auto& c : cents)
      byDetId[c.detId] = c;
    if (byDetId.size() != cents.size())
      return "duplicate detIds in sensor_centroids.bin";
    unsigned int nMod = static_cast<unsigned int>(cents.size()) + 1;  // + the pixel module (detId 1)
    if (nMod > 65535)
      return "too many modules";
    es.nModules = static_cast<uint16_t>(nMod);
    es.nLowerModules = static_cast<uint16_t>((nMod - 1) / 2);
    const uint16_t nLower = es.nLowerModules;

    auto resize = [&](auto& v) { v.assign(nMod, {}); };
    resize(es.detIds);
    resize(es.nConnectedModules);
    resize(es.drdzs);
    resize(es.dxdys);
    resize(es.eta);
    resize(es.r);
    resize(es.partnerModuleIndices);
    resize(es.layers);
    resize(es.rings);
    resize(es.modules);
    resize(es.rods);
    resize(es.subdets);
    resize(es.sides);
    resize(es.isInverted);
    resize(es.isLower);
    resize(es.isAnchor);
    resize(es.moduleType);
    resize(es.moduleLayerType);
    resize(es.sdlLayers);
    es.moduleMap.assign(size_t(nMod) * kMaxConnectedModules, 0);

    // Re-index in ascending detId order: lower modules 0..nLower-1, the pixel
    // module nLower, upper modules nLower+1.. (SDL/ModuleMethods.h:285-366).
    std::map<uint32_t, uint16_t> index;
    std::vector<uint32_t> sorted;
    sorted.reserve(nMod);
    sorted.push_back(1u);
    for (auto& kv : byDetId) {
      if (kv.first == 1u)
        return "detId 1 is reserved for the pixel module";
      sorted.push_back(kv.first);
    }
    std::sort(sorted.begin(), sorted.end());
    uint16_t lowerCounter = 0;
    uint16_t upperCounter = nLower + 1;
    for (uint32_t detId : sorted) {
      uint16_t idx;
      if (detId == 1u) {
        idx = nLower;
        es.detIds[idx] = 1u;
        es.moduleType[idx] = PixelModule;
        es.moduleLayerType[idx] = InnerPixelLayer;
        index[detId] = idx;
        continue;
      }
      const CentroidRec& c = byDetId[detId];
      short subdet = static_cast<short>((detId & (7u << 25)) >> 25);
      short side = static_cast<short>(subdet == Endcap ? (detId & (3u << 23)) >> 23 : (detId & (3u << 18)) >> 18);
      short layer = static_cast<short>(subdet == Endcap ? (detId & (7u << 18)) >> 18 : (detId & (7u << 20)) >> 20);
      short ring = static_cast<short>(subdet == Endcap ? (detId & (15u << 12)) >> 12 : 0);
      short module = static_cast<short>((detId & (127u << 2)) >> 2);
      short rod = static_cast<short>(subdet == Endcap ? 0 : (detId & (127u << 10)) >> 10);
      float m_x = c.x, m_y = c.y, m_z = c.z;
      float r = std::sqrt(m_x * m_x + m_y * m_y + m_z * m_z);
      float eta = ((m_z > 0) - (m_z < 0)) * std::acosh(r / std::sqrt(m_x * m_x + m_y * m_y));
      bool inv = parseIsInverted(subdet, side, module, layer);
      bool low = parseIsLower(inv, detId);
      if (low) {
        if (lowerCounter >= nLower)
          return "more lower modules than half of the sensors";
        idx = lowerCounter++;
      } else {
        idx = upperCounter++;
      }
      if (idx >= nMod)
        return "module index out of range";
      index[detId] = idx;
      es.detIds[idx] = detId;
      es.layers[idx] = layer;
      es.rings[idx] = ring;
      es.rods[idx] = rod;
      es.modules[idx] = module;
      es.subdets[idx] = subdet;
      es.sides[idx] = side;
      es.eta[idx] = eta;
      es.r[idx] = r;
      es.isInverted[idx] = inv;
      es.isLower[idx] = low;
      uint8_t mtype = (c.type == 25) ? TwoS : PS;
      uint8_t mltype = (c.type == 23) ? Pixel : Strip;
      es.moduleType[idx] = mtype;
      es.moduleLayerType[idx] = mltype;
      es.isAnchor[idx] = (mtype == PS && mltype == Pixel) || (mtype == TwoS && low);
      if (subdet == Endcap) {
        auto it = endcapDxdy.find(detId);
        es.dxdys[idx] = it == endcapDxdy.end() ? 0.f : it->second;
        es.drdzs[idx] = 0.f;
      } else {
        auto it = tiltedDxdy.find(detId);
        es.dxdys[idx] = it == tiltedDxdy.end() ? 0.f : it->second;
        auto jt = tiltedDrdz.find(detId);
        es.drdzs[idx] = (subdet == Barrel) ? (jt == tiltedDrdz.end() ? 0.f : jt->second) : 0.f;
      }
      es.sdlLayers[idx] = layer + 6 * (subdet == Endcap) + 5 * (subdet == Endcap && mtype == TwoS);
    }
    es.pixelModuleIndex = nLower;

    auto lookup = [&](uint32_t detId, uint16_t& out) {
      auto it = index.find(detId);
      if (it == index.end())
        return false;
      out = it->second;
      return true;
    };

    // Partner modules and drdz/dxdy taken from the partner when missing,
    // in ascending detId order (SDL/ModuleMethods.h:368-382).
    for (uint32_t detId : sorted) {
      if (detId == 1u)
        continue;
      uint16_t idx = index[detId];
      uint16_t partner;
      if (!lookup(partnerDetId(detId, es.isLower[idx], es.isInverted[idx]), partner))
        return "partner sensor missing for detId " + std::to_string(detId);
      es.partnerModuleIndices[idx] = partner;
      if (es.drdzs[idx] == 0)
        es.drdzs[idx] = es.drdzs[partner];
      if (es.dxdys[idx] == 0)
        es.dxdys[idx] = es.dxdys[partner];
    }

    // Pixel map: modules reachable from each pLS superbin, concatenating the
    // charge-inclusive, positive and negative maps (SDL/ModuleMethods.h:33-112).
    static const char* kLayers[4] = {"_layer1_subdet5", "_layer2_subdet5", "_layer1_subdet4", "_layer2_subdet4"};
    std::map<uint32_t, std::vector<uint32_t>> pls[3][4];
    for (int c = 0; c < 3; ++c)
      for (int l = 0; l < 4; ++l) {
        const char* charge = c == 0 ? "" : (c == 1 ? "_pos" : "_neg");
        std::string path = dir + "/pixelmap/pLS_map" + charge + kLayers[l] + ".bin";
        if (!readConnectionMap(path, pls[c][l]))
          return "unable to read " + path;
      }
    es.connectedPixelsIndex.assign(kSizeSuperbins, 0);
    es.connectedPixelsSizes.assign(kSizeSuperbins, 0);
    es.connectedPixelsIndexPos.assign(kSizeSuperbins, 0);
    es.connectedPixelsSizesPos.assign(kSizeSuperbins, 0);
    es.connectedPixelsIndexNeg.assign(kSizeSuperbins, 0);
    es.connectedPixelsSizesNeg.assign(kSizeSuperbins, 0);
    std::vector<uint32_t> det[3];
    unsigned int totals[3] = {0, 0, 0};
    for (unsigned int sb = 0; sb < kSizeSuperbins; ++sb) {
      for (int c = 0; c < 3; ++c) {
        uint32_t key = (c == 0) ? sb + kSizeSuperbins : sb;
        unsigned int sizes = 0;
        for (int l = 0; l < 4; ++l) {
          auto it = pls[c][l].find(key);
          if (it == pls[c][l].end())
            continue;
          det[c].insert(det[c].end(), it->second.begin(), it->second.end());
          sizes += static_cast<unsigned int>(it->second.size());
        }
        auto& idxv = c == 0 ? es.connectedPixelsIndex : (c == 1 ? es.connectedPixelsIndexPos : es.connectedPixelsIndexNeg);
        auto& sizev = c == 0 ? es.connectedPixelsSizes : (c == 1 ? es.connectedPixelsSizesPos : es.connectedPixelsSizesNeg);
        if (sizes > kMaxConnectedModules)
          return "pixel map lists more than " + std::to_string(kMaxConnectedModules) + " modules for superbin " +
                 std::to_string(sb);
        idxv[sb] = totals[c];
        sizev[sb] = sizes;
        totals[c] += sizes;
      }
    }
    es.nPixels = totals[0] + totals[1] + totals[2];
    es.connectedPixels.resize(es.nPixels);
    {
      size_t k = 0;
      for (int c = 0; c < 3; ++c)
        for (uint32_t d : det[c]) {
          uint16_t mi;
          if (!lookup(d, mi))
            return "pixel map references an unknown detId " + std::to_string(d);
          es.connectedPixels[k++] = mi;
        }
    }

    // Module connection map (SDL/ModuleMethods.h:115-141).
    for (uint32_t detId : sorted) {
      uint16_t idx = index[detId];
      auto it = connections.find(detId);
      if (it == connections.end())
        continue;
      if (it->second.size() > kMaxConnectedModules)
        return "more than " + std::to_string(kMaxConnectedModules) + " connected modules for detId " +
               std::to_string(detId);
      es.nConnectedModules[idx] = static_cast<uint16_t>(it->second.size());
      for (size_t i = 0; i < it->second.size(); ++i) {
        uint16_t mi;
        if (!lookup(it->second[i], mi))
          return "module map references an unknown detId " + std::to_string(it->second[i]);
        es.moduleMap[size_t(idx) * kMaxConnectedModules + i] = mi;
      }
    }

    // Sorted detId -> index map for the hit lookup (SDL/ModuleMethods.h:143-166).
    es.mapdetId.assign(sorted.begin(), sorted.end());
    es.mapIdx.resize(nMod);
    for (unsigned int i = 0; i < nMod; ++i)
      es.mapIdx[i] = index[sorted[i]];

    // Endcap strip orientation, ascending detId (SDL/EndcapGeometry.cc:43-70).
    for (auto& kv : endcapPhi) {
      es.geoMapDetId.push_back(kv.first);
      es.geoMapPhi.push_back(kv.second);
    }

    // Static caps and offsets.
    es.mdOffset.assign(nLower + 1, 0);
    es.mdCap.assign(nLower + 1, 0);
    es.lsOffset.assign(nLower + 1, 0);
    es.lsCap.assign(nLower + 1, 0);
    es.t3CapIfUsed.assign(nLower, 0);
    es.t5CapIfEligible.assign(nLower, -1);
    int mdTotal = 0, lsTotal = 0;
    unsigned int t3Total = 0, t5Total = 0;
    for (uint16_t i = 0; i < nLower; ++i) {
      int cat = occupancyCategory(es.layers[i], es.subdets[i], es.rings[i]);
      int etaBin = occupancyEtaBin(std::fabs(es.eta[i]));
      int mdc = mdOccupancy(cat, etaBin);
      es.mdOffset[i] = mdTotal;
      es.mdCap[i] = mdc;
      mdTotal += mdc;
      int lsc = es.nConnectedModules[i] == 0 ? 0 : lsOccupancy(cat, etaBin);
      es.lsOffset[i] = lsTotal;
      es.lsCap[i] = lsc;
      lsTotal += lsc;
      es.t3CapIfUsed[i] = t3Occupancy(cat, etaBin);
      if (es.nConnectedModules[i] != 0)
        t3Total += static_cast<unsigned int>(es.t3CapIfUsed[i]);
      bool eligible = !(es.subdets[i] == Barrel && es.layers[i] >= 3) && !(es.subdets[i] == Endcap && es.layers[i] > 1);
      if (eligible) {
        es.t5CapIfEligible[i] = t5Occupancy(cat, etaBin);
        t5Total += static_cast<unsigned int>(es.t5CapIfEligible[i]);
      }
    }
    es.mdOffset[nLower] = mdTotal;
    es.mdCap[nLower] = static_cast<int>(kMaxPixelMDs);
    es.lsOffset[nLower] = lsTotal;
    es.lsCap[nLower] = 0;
    es.nTotalMDs = static_cast<unsigned int>(mdTotal) + kMaxPixelMDs;
    es.nTotalSegments = static_cast<unsigned int>(lsTotal) + kMaxPixelSegments;
    es.maxTriplets = t3Total;
    es.maxQuintuplets = t5Total;
    buildDetHash(es);
    // geoMapDetId is sorted and unique: the exact match a binary search finds
    es.geoMapIndex.assign(es.detIds.size(), -1);
    for (size_t i = 0; i < es.detIds.size(); ++i) {
      const auto it = std::lower_bound(es.geoMapDetId.begin(), es.geoMapDetId.end(), es.detIds[i]);
      if (it != es.geoMapDetId.end() && *it == es.detIds[i])
        es.geoMapIndex[i] = static_cast<int>(it - es.geoMapDetId.begin());
    }
    return std::string();
  }

}  // namespace lst
