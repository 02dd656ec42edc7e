// Test-infrastructure shim (oracle only).
//
// The reference's WINDSGeneralData drags in NetCDF, GDAL, OptiX and every
// parameterization. The solver path (src/winds/Solver*.cpp), the wall
// routines (src/winds/Wall.cpp) and the building rasterisation
// (src/winds/PolyBuilding.cpp) only touch the members below, which carry the
// same names and types as src/winds/WINDSGeneralData.h:201-320.
#pragma once
#include <utility>
#include <vector>
#include "qes/Domain.h"
#include "util/QESout.h"  // the reference header reaches it through its own includes

class Wall;

class WINDSGeneralData {
public:
  explicit WINDSGeneralData(qes::Domain d) : domain(std::move(d)) {}

  qes::Domain domain;
  const float vk = 0.4;
  float z0{};

  std::vector<float> e, f, g, h, m, n;
  std::vector<int> icellflag;
  std::vector<int> ibuilding_flag, icellflag_footprint;  // building rasterisation (PolyBuilding.cpp)
  std::vector<float> base_height;
  std::vector<float> building_volume_frac;
  std::vector<float> ni, nj, nk, ti, tj, tk;
  std::vector<float> wall_distance;
  std::vector<int> center_id;
  std::vector<float> u0, v0, w0;
  std::vector<float> u, v, w;

  std::vector<int> wall_right_indices, wall_left_indices, wall_above_indices,
      wall_below_indices, wall_front_indices, wall_back_indices, wall_indices;
};
