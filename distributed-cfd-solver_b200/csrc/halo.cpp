// Halo plan of one rank (mesh::MeshPart's halo fields, built here from a
// single-partition mesh and a cell -> rank map).
#include "halo.hpp"

#include <algorithm>

namespace cfdg {

void build_halo_plan(const HostMesh& m, int32_t nparts, const int32_t* part, int32_t rank, HaloPlan& out) {
    const int32_t n = m.n_cells;
    if (nparts < 1 || rank < 0 || rank >= nparts) throw Failure{CFDG_ERR_INVALID, "halo: rank outside [0, nparts)"};
    if (n < nparts) throw Failure{CFDG_ERR_INVALID, "halo: fewer cells than ranks"};
    std::vector<int32_t> pr(n);
    for (int32_t c = 0; c < n; ++c) {
        pr[c] = part ? part[c] : static_cast<int32_t>((int64_t(c) * nparts) / n);
        if (pr[c] < 0 || pr[c] >= nparts) throw Failure{CFDG_ERR_INVALID, "halo: part entry outside [0, nparts)"};
    }
    out.nparts = nparts;
    out.rank = rank;
    // owned cells in ascending global order
    std::vector<int32_t> g2l(n, -1);
    out.local_to_global.clear();
    for (int32_t c = 0; c < n; ++c)
        if (pr[c] == rank) {
            g2l[c] = static_cast<int32_t>(out.local_to_global.size());
            out.local_to_global.push_back(c);
        }
    out.n_own = static_cast<int32_t>(out.local_to_global.size());
    if (out.n_own == 0) throw Failure{CFDG_ERR_INVALID, "halo: a rank owns no cell"};
    // across every partition face: the other side is a ghost here, and this
    // side is sent to the other side's rank
    std::vector<std::pair<int32_t, int32_t>> ghosts, sends;  // (rank, global cell)
    for (int32_t f = 0; f < m.n_inner; ++f) {
        const int32_t a = m.owner[f], b = m.neigh[f];
        if (pr[a] == pr[b]) continue;
        if (pr[a] == rank) {
            ghosts.emplace_back(pr[b], b);
            sends.emplace_back(pr[b], a);
        } else if (pr[b] == rank) {
            ghosts.emplace_back(pr[a], a);
            sends.emplace_back(pr[a], b);
        }
    }
    auto uniq = [](std::vector<std::pair<int32_t, int32_t>>& v) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
    };
    uniq(ghosts);
    uniq(sends);
    out.nb_ranks.clear();
    for (const auto& g : ghosts)
        if (out.nb_ranks.empty() || out.nb_ranks.back() != g.first) out.nb_ranks.push_back(g.first);
    const std::size_t nnb = out.nb_ranks.size();
    out.recv_offsets.assign(nnb + 1, 0);
    out.send_offsets.assign(nnb + 1, 0);
    out.recv_ghost_local.clear();
    out.send_owned_local.clear();
    std::size_t gi = 0, si = 0;
    for (std::size_t k = 0; k < nnb; ++k) {
        const int32_t r = out.nb_ranks[k];
        for (; gi < ghosts.size() && ghosts[gi].first == r; ++gi) {
            const int32_t c = ghosts[gi].second;
            g2l[c] = static_cast<int32_t>(out.local_to_global.size());
            out.local_to_global.push_back(c);
            out.recv_ghost_local.push_back(g2l[c]);
        }
        for (; si < sends.size() && sends[si].first == r; ++si) out.send_owned_local.push_back(g2l[sends[si].second]);
        out.recv_offsets[k + 1] = static_cast<int32_t>(out.recv_ghost_local.size());
        out.send_offsets[k + 1] = static_cast<int32_t>(out.send_owned_local.size());
    }
    out.n_local = static_cast<int32_t>(out.local_to_global.size());
    out.send_d.release();
    out.recv_d.release();
    out.device = -1;
}

}  // namespace cfdg
