// Table of every per-event device array: store prefix, view member, field,
// element type and length.  The arena carving and the named-field accessor
// both expand this one table, so they cannot disagree.
//
// Length symbols: H = hit capacity, M = modules, L = lower modules,
// MD / LS / T3 / T5 = arena lengths of the mini-doublet, segment, triplet and
// quintuplet stores, P = pixel-segment capacity (50000), P3 / P5 / TC =
// pixel-triplet (5000), pixel-quintuplet (15000) and track-candidate (31000)
// capacities.
#pragma once

#define LST_EVENT_FIELDS(X)                                   \
  X("hits.", hits, xs, float, H)                              \
  X("hits.", hits, ys, float, H)                              \
  X("hits.", hits, zs, float, H)                              \
  X("hits.", hits, moduleIndices, uint16_t, H)                \
  X("hits.", hits, idxs, unsigned int, H)                     \
  X("hits.", hits, detid, unsigned int, H)                    \
  X("hits.", hits, rts, float, H)                             \
  X("hits.", hits, phis, float, H)                            \
  X("hits.", hits, etas, float, H)                            \
  X("hits.", hits, highEdgeXs, float, H)                      \
  X("hits.", hits, highEdgeYs, float, H)                      \
  X("hits.", hits, lowEdgeXs, float, H)                       \
  X("hits.", hits, lowEdgeYs, float, H)                       \
  X("hits.", hits, hitRanges, int, 2 * M)                     \
  X("hits.", hits, hitRangesLower, int, M)                    \
  X("hits.", hits, hitRangesUpper, int, M)                    \
  X("hits.", hits, hitRangesnLower, int8_t, M)                \
  X("hits.", hits, hitRangesnUpper, int8_t, M)                \
  X("md.", md, anchorHitIndices, unsigned int, MD)            \
  X("md.", md, outerHitIndices, unsigned int, MD)             \
  X("md.", md, moduleIndices, uint16_t, MD)                   \
  X("md.", md, nMDs, unsigned int, L + 1)                     \
  X("md.", md, totOccupancyMDs, unsigned int, L + 1)          \
  X("md.", md, dphichanges, float, MD)                        \
  X("md.", md, dzs, float, MD)                                \
  X("md.", md, dphis, float, MD)                              \
  X("md.", md, shiftedXs, float, MD)                          \
  X("md.", md, shiftedYs, float, MD)                          \
  X("md.", md, shiftedZs, float, MD)                          \
  X("md.", md, noShiftedDzs, float, MD)                       \
  X("md.", md, noShiftedDphis, float, MD)                     \
  X("md.", md, noShiftedDphiChanges, float, MD)               \
  X("md.", md, anchorX, float, MD)                            \
  X("md.", md, anchorY, float, MD)                            \
  X("md.", md, anchorZ, float, MD)                            \
  X("md.", md, anchorRt, float, MD)                           \
  X("md.", md, anchorPhi, float, MD)                          \
  X("md.", md, anchorEta, float, MD)                          \
  X("md.", md, anchorHighEdgeX, float, MD)                    \
  X("md.", md, anchorHighEdgeY, float, MD)                    \
  X("md.", md, anchorLowEdgeX, float, MD)                     \
  X("md.", md, anchorLowEdgeY, float, MD)                     \
  X("md.", md, anchorLowEdgePhi, float, MD)                   \
  X("md.", md, anchorHighEdgePhi, float, MD)                  \
  X("md.", md, outerX, float, MD)                             \
  X("md.", md, outerY, float, MD)                             \
  X("md.", md, outerZ, float, MD)                             \
  X("md.", md, outerRt, float, MD)                            \
  X("md.", md, outerPhi, float, MD)                           \
  X("md.", md, outerEta, float, MD)                           \
  X("md.", md, outerHighEdgeX, float, MD)                     \
  X("md.", md, outerHighEdgeY, float, MD)                     \
  X("md.", md, outerLowEdgeX, float, MD)                      \
  X("md.", md, outerLowEdgeY, float, MD)                      \
  X("ls.", ls, dPhis, float, LS)                              \
  X("ls.", ls, dPhiMins, float, LS)                           \
  X("ls.", ls, dPhiMaxs, float, LS)                           \
  X("ls.", ls, dPhiChanges, float, LS)                        \
  X("ls.", ls, dPhiChangeMins, float, LS)                     \
  X("ls.", ls, dPhiChangeMaxs, float, LS)                     \
  X("ls.", ls, innerLowerModuleIndices, uint16_t, LS)         \
  X("ls.", ls, outerLowerModuleIndices, uint16_t, LS)         \
  X("ls.", ls, mdIndices, unsigned int, 2 * LS)               \
  X("ls.", ls, innerMiniDoubletAnchorHitIndices, unsigned int, LS) \
  X("ls.", ls, outerMiniDoubletAnchorHitIndices, unsigned int, LS) \
  X("ls.", ls, nSegments, unsigned int, L + 1)                \
  X("ls.", ls, totOccupancySegments, unsigned int, L + 1)     \
  X("ls.", ls, seedIdx, unsigned int, P)                      \
  X("ls.", ls, charge, int, P)                                \
  X("ls.", ls, superbin, int, P)                              \
  X("ls.", ls, pLSHitsIdxs, unsigned int, 4 * P)              \
  X("ls.", ls, pixelType, int8_t, P)                          \
  X("ls.", ls, isQuad, int8_t, P)                             \
  X("ls.", ls, isDup, int8_t, P)                              \
  X("ls.", ls, partOfPT5, uint8_t, P)                         \
  X("ls.", ls, ptIn, float, P)                                \
  X("ls.", ls, ptErr, float, P)                               \
  X("ls.", ls, px, float, P)                                  \
  X("ls.", ls, py, float, P)                                  \
  X("ls.", ls, pz, float, P)                                  \
  X("ls.", ls, etaErr, float, P)                              \
  X("ls.", ls, eta, float, P)                                 \
  X("ls.", ls, phi, float, P)                                 \
  X("ls.", ls, score, float, P)                               \
  X("ls.", ls, circleCenterX, float, P)                       \
  X("ls.", ls, circleCenterY, float, P)                       \
  X("ls.", ls, circleRadius, float, P)                        \
  X("t3.", t3, segmentIndices, unsigned int, 2 * T3)          \
  X("t3.", t3, lowerModuleIndices, uint16_t, 3 * T3)          \
  X("t3.", t3, nTriplets, unsigned int, L)                    \
  X("t3.", t3, totOccupancyTriplets, unsigned int, L)         \
  X("t3.", t3, logicalLayers, uint8_t, 3 * T3)                \
  X("t3.", t3, hitIndices, unsigned int, 6 * T3)              \
  X("t3.", t3, betaIn, float, T3)                             \
  X("t3.", t3, circleRadius, float, T3)                       \
  X("t3.", t3, circleCenterX, float, T3)                      \
  X("t3.", t3, circleCenterY, float, T3)                      \
  X("t3.", t3, partOfPT5, uint8_t, T3)                        \
  X("t3.", t3, partOfT5, uint8_t, T3)                         \
  X("t3.", t3, partOfPT3, uint8_t, T3)                        \
  X("t5.", t5, tripletIndices, unsigned int, 2 * T5)         \
  X("t5.", t5, lowerModuleIndices, uint16_t, 5 * T5)          \
  X("t5.", t5, nQuintuplets, unsigned int, L)                 \
  X("t5.", t5, totOccupancyQuintuplets, unsigned int, L)      \
  X("t5.", t5, innerRadius, float, T5)                        \
  X("t5.", t5, bridgeRadius, float, T5)                       \
  X("t5.", t5, outerRadius, float, T5)                        \
  X("t5.", t5, pt, float, T5)                                 \
  X("t5.", t5, eta, float, T5)                                \
  X("t5.", t5, phi, float, T5)                                \
  X("t5.", t5, score_rphisum, float, T5)                      \
  X("t5.", t5, layer, uint8_t, T5)                            \
  X("t5.", t5, isDup, int8_t, T5)                             \
  X("t5.", t5, TightCutFlag, uint8_t, T5)                     \
  X("t5.", t5, partOfPT5, uint8_t, T5)                        \
  X("t5.", t5, regressionRadius, float, T5)                   \
  X("t5.", t5, regressionG, float, T5)                        \
  X("t5.", t5, regressionF, float, T5)                        \
  X("t5.", t5, logicalLayers, uint8_t, 5 * T5)                \
  X("t5.", t5, hitIndices, unsigned int, 10 * T5)             \
  X("t5.", t5, rzChiSquared, float, T5)                       \
  X("t5.", t5, chiSquared, float, T5)                         \
  X("t5.", t5, nonAnchorChiSquared, float, T5)                \
  X("pt3.", pt3, pixelSegmentIndices, unsigned int, P3)       \
  X("pt3.", pt3, tripletIndices, unsigned int, P3)            \
  X("pt3.", pt3, nPixelTriplets, unsigned int, 1)             \
  X("pt3.", pt3, totOccupancyPixelTriplets, unsigned int, 1)  \
  X("pt3.", pt3, pixelRadius, float, P3)                      \
  X("pt3.", pt3, tripletRadius, float, P3)                    \
  X("pt3.", pt3, pt, float, P3)                               \
  X("pt3.", pt3, eta, float, P3)                              \
  X("pt3.", pt3, phi, float, P3)                              \
  X("pt3.", pt3, eta_pix, float, P3)                          \
  X("pt3.", pt3, phi_pix, float, P3)                          \
  X("pt3.", pt3, score, float, P3)                            \
  X("pt3.", pt3, isDup, uint8_t, P3)                          \
  X("pt3.", pt3, partOfPT5, uint8_t, P3)                      \
  X("pt3.", pt3, logicalLayers, uint8_t, 5 * P3)              \
  X("pt3.", pt3, hitIndices, unsigned int, 10 * P3)           \
  X("pt3.", pt3, lowerModuleIndices, uint16_t, 5 * P3)        \
  X("pt3.", pt3, centerX, float, P3)                          \
  X("pt3.", pt3, centerY, float, P3)                          \
  X("pt3.", pt3, pixelRadiusError, float, P3)                 \
  X("pt3.", pt3, rPhiChiSquared, float, P3)                   \
  X("pt3.", pt3, rPhiChiSquaredInwards, float, P3)            \
  X("pt3.", pt3, rzChiSquared, float, P3)                     \
  X("pt5.", pt5, pixelIndices, unsigned int, P5)              \
  X("pt5.", pt5, T5Indices, unsigned int, P5)                 \
  X("pt5.", pt5, nPixelQuintuplets, unsigned int, 1)          \
  X("pt5.", pt5, totOccupancyPixelQuintuplets, unsigned int, 1) \
  X("pt5.", pt5, isDup, uint8_t, P5)                          \
  X("pt5.", pt5, score, float, P5)                            \
  X("pt5.", pt5, eta, float, P5)                              \
  X("pt5.", pt5, phi, float, P5)                              \
  X("pt5.", pt5, logicalLayers, uint8_t, 7 * P5)              \
  X("pt5.", pt5, hitIndices, unsigned int, 14 * P5)           \
  X("pt5.", pt5, lowerModuleIndices, uint16_t, 7 * P5)        \
  X("pt5.", pt5, pixelRadius, float, P5)                      \
  X("pt5.", pt5, quintupletRadius, float, P5)                 \
  X("pt5.", pt5, centerX, float, P5)                          \
  X("pt5.", pt5, centerY, float, P5)                          \
  X("pt5.", pt5, rzChiSquared, float, P5)                     \
  X("pt5.", pt5, rPhiChiSquared, float, P5)                   \
  X("pt5.", pt5, rPhiChiSquaredInwards, float, P5)            \
  X("tc.", tc, trackCandidateType, short, TC)                 \
  X("tc.", tc, directObjectIndices, unsigned int, TC)         \
  X("tc.", tc, objectIndices, unsigned int, 2 * TC)           \
  X("tc.", tc, nTrackCandidates, unsigned int, 1)             \
  X("tc.", tc, nTrackCandidatespT3, unsigned int, 1)          \
  X("tc.", tc, nTrackCandidatespT5, unsigned int, 1)          \
  X("tc.", tc, nTrackCandidatespLS, unsigned int, 1)          \
  X("tc.", tc, nTrackCandidatesT5, unsigned int, 1)           \
  X("tc.", tc, logicalLayers, uint8_t, 7 * TC)                \
  X("tc.", tc, hitIndices, unsigned int, 14 * TC)             \
  X("tc.", tc, pixelSeedIndex, int, TC)                       \
  X("tc.", tc, lowerModuleIndices, uint16_t, 7 * TC)          \
  X("tc.", tc, centerX, float, TC)                            \
  X("tc.", tc, centerY, float, TC)                            \
  X("tc.", tc, radius, float, TC)                             \
  X("ranges.", rg, mdRanges, int, 2 * M)                      \
  X("ranges.", rg, segmentRanges, int, 2 * M)                 \
  X("ranges.", rg, tripletRanges, int, 2 * M)                 \
  X("ranges.", rg, quintupletRanges, int, 2 * M)              \
  X("ranges.", rg, nEligibleT5Modules, uint16_t, 1)           \
  X("ranges.", rg, indicesOfEligibleT5Modules, uint16_t, L)   \
  X("ranges.", rg, quintupletModuleIndices, int, L)           \
  X("ranges.", rg, quintupletModuleOccupancy, int, L)         \
  X("ranges.", rg, miniDoubletModuleIndices, int, L + 1)      \
  X("ranges.", rg, miniDoubletModuleOccupancy, int, L + 1)    \
  X("ranges.", rg, segmentModuleIndices, int, L + 1)          \
  X("ranges.", rg, segmentModuleOccupancy, int, L + 1)        \
  X("ranges.", rg, tripletModuleIndices, int, L)              \
  X("ranges.", rg, tripletModuleOccupancy, int, L)            \
  X("ranges.", rg, device_nTotalMDs, unsigned int, 1)         \
  X("ranges.", rg, device_nTotalSegs, unsigned int, 1)        \
  X("ranges.", rg, device_nTotalTrips, unsigned int, 1)       \
  X("ranges.", rg, device_nTotalQuints, unsigned int, 1)

// Work arrays that are not part of the reference's stores.
#define LST_SCRATCH_FIELDS(X)                         \
  X(plsHit0, unsigned int, P)                         \
  X(plsHit1, unsigned int, P)                         \
  X(plsHit2, unsigned int, P)                         \
  X(plsHit3, unsigned int, P)                         \
  X(plsDPhiChange, float, P)                          \
  X(plsConnIndex, unsigned int, P)                    \
  X(plsConnSize, unsigned int, P)                     \
  X(plsCount, unsigned int, P)                        \
  X(plsOffset, unsigned int, P)                       \
  X(moduleCount, unsigned int, L + 1)                 \
  X(moduleOffset, unsigned int, L + 1)                \
  X(t5Flag, uint8_t, T5)                              \
  X(plsFlag, uint8_t, P)                              \
  X(tcOutLen, unsigned int, TC)                       \
  X(tcOutOffset, unsigned int, TC)                    \
  X(lsByMD, uint16_t, LS)                             \
  X(mdLSStart, uint16_t, MD)                          \
  X(mdLSCount, uint16_t, MD)                          \
  X(t3ByMD, uint16_t, T3)                             \
  X(mdT3Start, uint16_t, MD)                          \
  X(mdT3Count, uint16_t, MD)                          \
  X(t5CandPre, unsigned int, T3)                      \
  X(t5ModCand, unsigned int, L)                       \
  X(t5ModOff, unsigned int, L + 1)                    \
  X(t5CandFlag, unsigned int, lst::kT5CandCap)        \
  X(t5PassValues, lst::T5Values, lst::kT5PassCap)     \
  X(t5PassC, unsigned int, lst::kT5PassCap)           \
  X(t5DnnFeat, float, 38 * lst::kT5DnnCap)            \
  X(t5DnnSlot, lst::T5DnnSlotG, lst::kT5DnnCap)      \
  X(plsModPre, unsigned int, P * (lst::kMaxConnectedModules + 1)) \
  X(plsCand, unsigned int, P)                         \
  X(plsCandOff, unsigned int, P + 1)                  \
  X(pixPassC, unsigned int, lst::kPixPassCap)         \
  X(pixPassObj, unsigned int, lst::kPixPassCap)       \
  X(pixPassPLS, unsigned int, lst::kPixPassCap)       \
  X(pixPassV, float, 8 * lst::kPixPassCap)            \
  X(candQueue, unsigned int, lst::kCandQueueCap)        \
  X(pixChunkPLS, unsigned int, lst::kPixChunkCap)       \
  X(t5ChunkMod, unsigned int, lst::kT5CandCap / 32)     \
  X(hitMiniSlope, float, H)                           \
  X(t5Order, unsigned int, lst::kT5SortCap)           \
  X(t5OrderPos, uint16_t, lst::kT5SortCap)            \
  X(t5BinStart, unsigned int, lst::kPLSBins + 2)      \
  X(hitShiftXa, float, H)                             \
  X(hitShiftYa, float, H)                             \
  X(hitShiftZn, float, H)                             \
  X(tcCleanInfo, lst::TCCleanInfo, TC)                \
  X(plsRec, lst::PLSRec, P)                           \
  X(plsHitHead, unsigned int, lst::kPLSHitBuckets)      \
  X(plsHitNext, unsigned int, 4 * P)                   \
  X(plsBinStart, unsigned int, lst::kPLSBins + 2)
