// Test-infrastructure shim (oracle only). Wall.cpp includes the input-data
// header but never dereferences it; PolyBuilding.cpp reads the members below,
// which carry the reference's names (src/winds/WINDSInputData.h and the
// SimulationParameters / BuildingsParams / ESRIShapefile members it reaches).
#pragma once
#include <map>
#include <string>
#include <vector>
#include "util/PolygonVertex.h"

struct ShimSimParams {
  int meshTypeFlag = 0;          // stair-step buildings
  int readCoefficientsFlag = 0;  // coefficients computed, not read
};

struct ShimShapefile {
  std::vector<std::vector<polyVert>> m_polygons;
  std::map<std::string, std::vector<float>> m_features;
};

struct ShimBuildingsParams {
  ShimShapefile *SHPData = nullptr;
  std::string shpHeightField;
  float heightFactor = 1.0f;
};

class WINDSInputData {
public:
  ShimSimParams *simParams = nullptr;
  ShimBuildingsParams *buildingsParams = nullptr;
};
