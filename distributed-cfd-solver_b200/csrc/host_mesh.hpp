// Host-side mesh container and set-up routines (synthetic generation,
// reverse Cuthill-McKee renumbering, geometry, connectivity).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "cfdg.h"

namespace cfdg {

// Single-partition mesh in the SoA layout of mesh::MeshPart
// (include/cfd/mesh/localmesh.hpp:17-102), owned cells only (n_own == n_cells).
struct HostMesh {
    int32_t n_cells = 0, n_faces = 0, n_inner = 0, n_nodes = 0, n_patches = 0;
    std::vector<uint8_t> cell_type;
    std::vector<int32_t> cell_nodes_off, cell_nodes;
    std::vector<double> node_x, node_y, node_z;
    std::vector<double> ccx, ccy, ccz, vol;
    std::vector<int32_t> owner, neigh, patch, fn_off, fn;
    std::vector<double> fcx, fcy, fcz, fnx, fny, fnz, area;

    void view(cfdg_mesh_host& v) const;
    void from_view(const cfdg_mesh_host& v);
};

// Synthetic generators (compression ramp, flat plate, tetrahedral bump).
int generate_mesh(const cfdg_mesh_spec& spec, HostMesh& out, std::string& err);

// Cell/face geometry by tetrahedral / fan decomposition; returns false and
// fills err on a non-positive volume or area.
bool compute_geometry(HostMesh& m, std::string& err);

// Compressed-row adjacency.
struct Csr {
    std::vector<int32_t> off, val;
    int32_t rows() const { return off.empty() ? 0 : static_cast<int32_t>(off.size()) - 1; }
};

// cell -> faces (ascending face index, boundary faces included),
// aux_connectivity.cpp:11-86.
Csr build_cell_faces(const HostMesh& m);
// cell -> face-sharing cells (sorted), aux_connectivity.cpp:88-187.
Csr build_cell_cells_face(const HostMesh& m);
// cell -> vertex-sharing cells (sorted, self excluded), aux_connectivity.cpp:348-445.
Csr build_cell_cells_node(const HostMesh& m);

// Reverse Cuthill-McKee order (new -> old) of a symmetric graph.
std::vector<int32_t> rcm_order(const Csr& g);

}  // namespace cfdg
