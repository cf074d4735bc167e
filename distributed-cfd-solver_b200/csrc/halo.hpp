// Partition of a mesh over ranks and the halo plan of one rank: the halo
// fields of mesh::MeshPart (include/cfd/mesh/localmesh.hpp:30-32, 79-83)
// that HaloExchanger (src/fields/halo.cpp:212-330) exchanges, and the
// device pack/unpack of those exchanges.
#pragma once

#include <cstdint>
#include <vector>

#include "host_mesh.hpp"
#include "solver.hpp"

namespace cfdg {

struct HaloPlan {
    int32_t nparts = 1, rank = 0;
    int32_t n_own = 0, n_local = 0;          // owned cells; owned + ghost cells
    std::vector<int32_t> local_to_global;    // n_local: owned (ascending global), then ghosts
    std::vector<int32_t> nb_ranks;           // neighbour ranks, ascending
    // one group per neighbour, in nb_ranks order; each group ascending in
    // global cell id, so a sender's group for rank r and r's group for the
    // sender list the same cells in the same order
    std::vector<int32_t> send_offsets, send_owned_local;   // local indices in [0, n_own)
    std::vector<int32_t> recv_offsets, recv_ghost_local;   // local indices in [n_own, n_local)
    // device copies of the two index lists, uploaded on first pack/unpack
    DevArray<int32_t> send_d, recv_d;
    int device = -1;
};

// part[c]: owning rank of global cell c, or null for nparts contiguous
// ranges of the cell order (compact slabs on an RCM-ordered mesh).
void build_halo_plan(const HostMesh& m, int32_t nparts, const int32_t* part, int32_t rank, HaloPlan& out);

// msg[i * nvars + v] = fields[v][idx[i]] (AoS per cell, as pack_soa_to_aos,
// src/fields/halo.cpp:26-75) and the inverse scatter; nvars <= kHaloMaxVars.
constexpr int kHaloMaxVars = 32;
struct HaloFields {
    double* p[kHaloMaxVars];
};
void launch_halo_pack(int32_t n, const int32_t* idx, const HaloFields& f, int nvars, double* msg, cudaStream_t s);
void launch_halo_unpack(int32_t n, const int32_t* idx, const double* msg, int nvars, const HaloFields& f,
                        cudaStream_t s);
// The same for a block vector x[row * bs + v] (bs <= kHaloMaxVars).
void launch_halo_pack_blocks(int32_t n, const int32_t* idx, const double* x, int bs, double* msg, cudaStream_t s);
void launch_halo_unpack_blocks(int32_t n, const int32_t* idx, const double* msg, int bs, double* x, cudaStream_t s);

}  // namespace cfdg
