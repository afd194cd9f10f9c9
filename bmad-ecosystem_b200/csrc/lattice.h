// lattice.h -- host packer interface (see lattice.cpp).
#pragma once
#include <string>
#include <vector>

#include "../../include/bmadgpu.h"
#include "table.h"

namespace bmadgpu {

struct PackedLattice {
  std::vector<uint8_t> image;          // [EleHdr x n][ApRec x n_ap][double pool], 16-byte aligned
  TableInfo info;
  std::vector<int> n_step;             // resolved integration steps per element
  std::vector<double> ds_step;         // resolved ds_step per element
  std::vector<double> ref_time_prefix; // sum of delta_ref_time over elements [0, i)
};

int pack_lattice(const bmadgpu_element* eles, int n_ele, const bmadgpu_param& p, PackedLattice& out,
                 std::string& err);

}  // namespace bmadgpu
