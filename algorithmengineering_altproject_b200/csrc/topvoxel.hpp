// TopVoxel domain files (the MATLAB original's external-model input, TOP3D_XL.m:458-586): a voxelised
// design domain with its fixations, loads and passive elements.  Host code.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace t3d {

// One TopVoxel model in the file's own (unpadded) index spaces, 0-based:
//   voxel k = y + nely * (x + nelx * z)                  (MATLAB column-major [nely, nelx, nelz])
//   node  m = y + (nely+1) * (x + (nelx+1) * z)          (column-major [nely+1, nelx+1, nelz+1])
// Duplicate node rows keep their first occurrence (MATLAB unique(), TOP3D_XL.m:531,541).
struct VoxelModel {
    int nelx = 0, nely = 0, nelz = 0;
    std::vector<uint8_t> voxel;        // [nelx*nely*nelz]: 0 void, 1 solid, 2 passive solid
    std::vector<int64_t> fix_node;     // nodes with at least one fixed DOF, ascending
    std::vector<uint8_t> fix_bits;     // bit c = DOF c fixed
    std::vector<int64_t> load_node;    // loaded nodes, ascending
    std::vector<double> load_f;        // 3 per loaded node
    int64_t num_solid = 0, num_passive = 0;
    int num_additional_loads = 0;      // load cases after the first
    // load cases 2.. (file indices 2..K+1, in that order): loaded nodes ascending, 3 forces per node
    std::vector<std::vector<int64_t>> case_node;
    std::vector<std::vector<double>> case_f;
    bool has_densities = false;        // per-voxel densities were listed (read and not used)
};

// Parses a TopVoxel file of format version 1.0.  On failure returns false with *err set.
bool parse_topvoxel(const char* path, VoxelModel* out, std::string* err);

}  // namespace t3d
