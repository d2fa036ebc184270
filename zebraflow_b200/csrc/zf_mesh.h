// Host-side membrane mesh shared by every cell (internal, not part of the ABI).
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/zf.h"

namespace zf {

struct MeshHost {
  int n_node = 0, n_tri = 0, n_edge = 0;
  std::vector<int32_t> tri;          // [n_tri][3], 0-based
  std::vector<int32_t> edge;         // [n_edge][6] n1 n2 n3 n4 tri1 tri2, 0-based
  std::vector<uint8_t> area_first;   // [n_edge] bit0: first visitor of tri1, bit1: of tri2
  std::vector<float> lmax, plength, kp, sin0, cos0;  // [n_edge]
  std::vector<float> tri_area_eq;    // [n_tri]
  std::vector<double> rest;          // [n_node][3] um
  int n_node_n = 0, n_edge_n = 0;
  std::vector<int32_t> edge_n;       // [n_edge_n][2], 0-based
  std::vector<float> lmax_n, plength_n, kp_n;
  std::vector<double> rest_n;        // [n_node_n][3] um
  double area0 = 0, volume0 = 0;     // m^2, m^3
};

uint64_t pair_key(int a, int b);
int mesh_build(MeshHost& m, const zf_params& P);

}  // namespace zf
