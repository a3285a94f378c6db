// Device side of the particle-pair passes (pairs.cu): solid regularisation and heat exchange; internal.
#pragma once
#include <cstddef>

#include "mpm_internal.h"

namespace mpm {

// Neighbour cells of one scene: nc cells per axis from the scene's grid origin, global ids from
// cell_base.
struct RegScene {
  int nc[3];
  int pad;
  long long cell_base;
};

struct RegDev {
  const RegScene* scenes;
  long long cells;        // total over scenes
  float spacing;          // target spacing at volume_unit (m)
  float inv_volume_unit;
  float max_speed;        // displacement budget per second (m/s)
  float rate;             // gain = 1 - exp(-rate dt)
  float eps;              // coincident pairs: r < eps
  float inv_hc;           // 1 / neighbour cell size (cells are two spacings wide)
  const float* dt_scene;  // per-scene dt of the substep just taken, or null: dt
  float dt;
};

struct RegBufs {
  unsigned *cell_of, *count, *start, *cursor, *sorted, *block_sums, *largest;
  float *target, *inv_mass;
  float4* shift;
  uint4* pos_sorted;             // cell order: (qx, qy, qz, target bits)
  uint2* inv_sorted;             // cell order: (inverse mass bits, caller index)
  unsigned short* mat_sorted;    // cell order: material (multi-material scenes)
};

size_t reg_scan_blocks(long long cells);
void launch_regularize(const Ctx& c, const RegDev& r, const RegBufs& b, cudaStream_t st);

// Particle-pair heat exchange: neighbour cells one radius wide (RegScene layout), conductance
// factor geometry * heat_rate, optional ambient loss.
struct HeatDev {
  const RegScene* scenes;
  long long cells;
  float inv_hc;         // 1 / radius
  float radius, eps;    // pairs with eps < r < radius
  float geom_rate;      // geometry * heat_rate
  float dt;
  int ambient;
  float ambient_T, ambient_rate;
};

struct HeatBufs {
  unsigned *cell_of, *count, *start, *cursor, *sorted, *block_sums;
  uint4* pos_sorted;    // cell order: (qx, qy, qz, T bits)
  float2* prop_sorted;  // cell order: (conductivity, m cp)
  float* budget;        // cell order
  double* exchanged;    // 1: sum over pairs of |Q|
};

void launch_exchange_heat(const Ctx& c, const HeatDev& hd, const HeatBufs& b, cudaStream_t st);

}  // namespace mpm
