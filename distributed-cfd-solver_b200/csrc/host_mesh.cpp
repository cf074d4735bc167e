// Synthetic meshes, reverse Cuthill-McKee renumbering, geometry and
// connectivity for the single-partition GPU solver.
//
// The reference reads partitioned meshes from an HDF5 container written by
// its CGNS preprocessing app; neither library exists on this machine, so the
// benchmark meshes are generated here in the same MeshPart layout
// (include/cfd/mesh/localmesh.hpp:17-102): 3-zone face order (interior faces
// sorted by (owner, neigh), boundary faces by (patch, owner)), outward face
// node order from the owner, CGNS element node order.
#include "host_mesh.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>

namespace cfdg {

namespace {

// CGNS SIDS local face definitions (0-based), ordered so that the
// right-hand rule gives the outward normal.  These are the element
// conventions of the CGNS standard; the reference tables in
// include/cfd/mesh/cgnstables.hpp:35-75 describe the same faces.
constexpr int kHexFaces[6][4] = {{0, 3, 2, 1}, {0, 1, 5, 4}, {1, 2, 6, 5},
                                 {2, 3, 7, 6}, {0, 4, 7, 3}, {4, 5, 6, 7}};
constexpr int kTetFaces[4][3] = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {2, 0, 3}};

struct Rng {
    std::mt19937_64 g;
    explicit Rng(uint64_t s) : g(s) {}
    double uniform() { return static_cast<double>(g() >> 11) * (1.0 / 9007199254740992.0); }
    double sym() { return 2.0 * uniform() - 1.0; }
};

inline int faces_of(uint8_t t) { return t == CFDG_HEXA ? 6 : 4; }
inline int face_nn(uint8_t t) { return t == CFDG_HEXA ? 4 : 3; }
inline int face_local(uint8_t t, int f, int j) {
    return t == CFDG_HEXA ? kHexFaces[f][j] : kTetFaces[f][j];
}

struct FaceRec {
    int32_t k[4];
    int32_t cell;
    int32_t lf;
};

// Pairs the faces of all cells.  The owner of an interior face is the
// lower-numbered cell; face nodes come from the owner's outward local face.
// classify(face nodes, n) returns the patch id of a boundary face.
template <typename Classify>
bool extract_faces(HostMesh& m, Classify classify, std::string& err) {
    std::vector<FaceRec> recs;
    std::size_t total = 0;
    for (int32_t c = 0; c < m.n_cells; ++c) total += static_cast<std::size_t>(faces_of(m.cell_type[c]));
    recs.resize(total);
    std::size_t w = 0;
    for (int32_t c = 0; c < m.n_cells; ++c) {
        const uint8_t t = m.cell_type[c];
        const int32_t* cn = m.cell_nodes.data() + m.cell_nodes_off[c];
        for (int f = 0; f < faces_of(t); ++f) {
            FaceRec r;
            const int nn = face_nn(t);
            for (int j = 0; j < 4; ++j) r.k[j] = (j < nn) ? cn[face_local(t, f, j)] : INT32_MAX;
            std::sort(r.k, r.k + 4);
            r.cell = c;
            r.lf = f;
            recs[w++] = r;
        }
    }
    std::sort(recs.begin(), recs.end(), [](const FaceRec& a, const FaceRec& b) {
        for (int j = 0; j < 4; ++j)
            if (a.k[j] != b.k[j]) return a.k[j] < b.k[j];
        return a.cell < b.cell;
    });

    struct Face {
        int32_t owner, neigh, lf, patch;
    };
    std::vector<Face> inner, bnd;
    inner.reserve(total / 2);
    for (std::size_t i = 0; i < recs.size();) {
        std::size_t j = i + 1;
        while (j < recs.size() && std::memcmp(recs[j].k, recs[i].k, sizeof(recs[i].k)) == 0) ++j;
        if (j - i == 2) {
            inner.push_back({recs[i].cell, recs[i + 1].cell, recs[i].lf, -1});
        } else if (j - i == 1) {
            const uint8_t t = m.cell_type[recs[i].cell];
            const int32_t* cn = m.cell_nodes.data() + m.cell_nodes_off[recs[i].cell];
            int32_t nodes[4];
            const int nn = face_nn(t);
            for (int q = 0; q < nn; ++q) nodes[q] = cn[face_local(t, recs[i].lf, q)];
            const int32_t p = classify(nodes, nn);
            if (p < 0) {
                err = "boundary face could not be assigned to a patch";
                return false;
            }
            bnd.push_back({recs[i].cell, -1, recs[i].lf, p});
        } else {
            err = "non-manifold face shared by more than two cells";
            return false;
        }
        i = j;
    }
    std::sort(inner.begin(), inner.end(), [](const Face& a, const Face& b) {
        return a.owner != b.owner ? a.owner < b.owner : a.neigh < b.neigh;
    });
    std::stable_sort(bnd.begin(), bnd.end(), [](const Face& a, const Face& b) {
        if (a.patch != b.patch) return a.patch < b.patch;
        if (a.owner != b.owner) return a.owner < b.owner;
        return a.lf < b.lf;
    });

    m.n_inner = static_cast<int32_t>(inner.size());
    m.n_faces = static_cast<int32_t>(inner.size() + bnd.size());
    m.owner.resize(m.n_faces);
    m.neigh.resize(m.n_faces);
    m.patch.resize(m.n_faces);
    m.fn_off.assign(static_cast<std::size_t>(m.n_faces) + 1, 0);
    m.fn.clear();
    m.fn.reserve(static_cast<std::size_t>(m.n_faces) * 4);
    int32_t max_patch = -1;
    auto emit = [&](const Face& f, int32_t idx) {
        m.owner[idx] = f.owner;
        m.neigh[idx] = f.neigh;
        m.patch[idx] = f.patch;
        max_patch = std::max(max_patch, f.patch);
        const uint8_t t = m.cell_type[f.owner];
        const int32_t* cn = m.cell_nodes.data() + m.cell_nodes_off[f.owner];
        for (int q = 0; q < face_nn(t); ++q) m.fn.push_back(cn[face_local(t, f.lf, q)]);
        m.fn_off[idx + 1] = static_cast<int32_t>(m.fn.size());
    };
    int32_t idx = 0;
    for (const Face& f : inner) emit(f, idx++);
    for (const Face& f : bnd) emit(f, idx++);
    m.n_patches = max_patch + 1;
    return true;
}

// Renumbers cells (new -> old permutation) and rebuilds faces.
template <typename Classify>
bool apply_cell_order(HostMesh& m, const std::vector<int32_t>& new2old, Classify classify, std::string& err) {
    std::vector<uint8_t> type(m.n_cells);
    std::vector<int32_t> off(static_cast<std::size_t>(m.n_cells) + 1, 0), nodes;
    nodes.reserve(m.cell_nodes.size());
    for (int32_t c = 0; c < m.n_cells; ++c) {
        const int32_t o = new2old[c];
        type[c] = m.cell_type[o];
        for (int32_t k = m.cell_nodes_off[o]; k < m.cell_nodes_off[o + 1]; ++k) nodes.push_back(m.cell_nodes[k]);
        off[c + 1] = static_cast<int32_t>(nodes.size());
    }
    m.cell_type.swap(type);
    m.cell_nodes_off.swap(off);
    m.cell_nodes.swap(nodes);
    return extract_faces(m, classify, err);
}

// Renumbers nodes by first use in cell order (locality of node data).
void renumber_nodes(HostMesh& m) {
    std::vector<int32_t> old2new(m.n_nodes, -1);
    int32_t next = 0;
    for (int32_t& n : m.cell_nodes) {
        if (old2new[n] < 0) old2new[n] = next++;
        n = old2new[n];
    }
    for (int32_t& n : m.fn) n = old2new[n];
    std::vector<double> x(next), y(next), z(next);
    for (int32_t o = 0; o < m.n_nodes; ++o) {
        const int32_t nw = old2new[o];
        if (nw < 0) continue;
        x[nw] = m.node_x[o];
        y[nw] = m.node_y[o];
        z[nw] = m.node_z[o];
    }
    m.n_nodes = next;
    m.node_x.swap(x);
    m.node_y.swap(y);
    m.node_z.swap(z);
}

Csr face_graph(const HostMesh& m) {
    Csr g;
    g.off.assign(static_cast<std::size_t>(m.n_cells) + 1, 0);
    for (int32_t f = 0; f < m.n_inner; ++f) {
        ++g.off[m.owner[f] + 1];
        ++g.off[m.neigh[f] + 1];
    }
    for (int32_t c = 0; c < m.n_cells; ++c) g.off[c + 1] += g.off[c];
    g.val.resize(g.off.back());
    std::vector<int32_t> cur(g.off.begin(), g.off.end() - 1);
    for (int32_t f = 0; f < m.n_inner; ++f) {
        g.val[cur[m.owner[f]]++] = m.neigh[f];
        g.val[cur[m.neigh[f]]++] = m.owner[f];
    }
    for (int32_t c = 0; c < m.n_cells; ++c) std::sort(g.val.begin() + g.off[c], g.val.begin() + g.off[c + 1]);
    return g;
}

}  // namespace

void HostMesh::view(cfdg_mesh_host& v) const {
    v.n_cells = n_cells;
    v.n_faces = n_faces;
    v.n_inner_faces = n_inner;
    v.n_nodes = n_nodes;
    v.n_patches = n_patches;
    v.cell_type = cell_type.data();
    v.cell_nodes_offsets = cell_nodes_off.data();
    v.cell_nodes = cell_nodes.data();
    v.node_x = node_x.data();
    v.node_y = node_y.data();
    v.node_z = node_z.data();
    v.cell_centroid_x = ccx.data();
    v.cell_centroid_y = ccy.data();
    v.cell_centroid_z = ccz.data();
    v.cell_volume = vol.data();
    v.face_owner = owner.data();
    v.face_neigh = neigh.data();
    v.face_patch = patch.data();
    v.face_nodes_offsets = fn_off.data();
    v.face_nodes = fn.data();
    v.face_centroid_x = fcx.data();
    v.face_centroid_y = fcy.data();
    v.face_centroid_z = fcz.data();
    v.face_normal_x = fnx.data();
    v.face_normal_y = fny.data();
    v.face_normal_z = fnz.data();
    v.face_area = area.data();
}

void HostMesh::from_view(const cfdg_mesh_host& v) {
    n_cells = v.n_cells;
    n_faces = v.n_faces;
    n_inner = v.n_inner_faces;
    n_nodes = v.n_nodes;
    n_patches = v.n_patches;
    auto cp = [](auto* src, std::size_t n, auto& dst) {
        if (src) dst.assign(src, src + n);
        else dst.clear();
    };
    const std::size_t nc = static_cast<std::size_t>(n_cells), nf = static_cast<std::size_t>(n_faces);
    cp(v.cell_type, nc, cell_type);
    cp(v.cell_nodes_offsets, nc + 1, cell_nodes_off);
    cp(v.cell_nodes, v.cell_nodes_offsets ? static_cast<std::size_t>(v.cell_nodes_offsets[nc]) : 0, cell_nodes);
    cp(v.node_x, static_cast<std::size_t>(n_nodes), node_x);
    cp(v.node_y, static_cast<std::size_t>(n_nodes), node_y);
    cp(v.node_z, static_cast<std::size_t>(n_nodes), node_z);
    cp(v.cell_centroid_x, nc, ccx);
    cp(v.cell_centroid_y, nc, ccy);
    cp(v.cell_centroid_z, nc, ccz);
    cp(v.cell_volume, nc, vol);
    cp(v.face_owner, nf, owner);
    cp(v.face_neigh, nf, neigh);
    cp(v.face_patch, nf, patch);
    cp(v.face_nodes_offsets, nf + 1, fn_off);
    cp(v.face_nodes, v.face_nodes_offsets ? static_cast<std::size_t>(v.face_nodes_offsets[nf]) : 0, fn);
    cp(v.face_centroid_x, nf, fcx);
    cp(v.face_centroid_y, nf, fcy);
    cp(v.face_centroid_z, nf, fcz);
    cp(v.face_normal_x, nf, fnx);
    cp(v.face_normal_y, nf, fny);
    cp(v.face_normal_z, nf, fnz);
    cp(v.face_area, nf, area);
}

// Volume and centroid of a cell from tetrahedra with apex at the vertex
// average and bases on the (fan-triangulated) faces; face area vector from
// the fan around the face vertex average, centroid area-weighted.  This is
// the decomposition of compute_poly_cell_metrics / compute_mesh_geometry
// (src/mesh/geometry.cpp:25-140,301-540).
bool compute_geometry(HostMesh& m, std::string& err) {
    const std::size_t nc = static_cast<std::size_t>(m.n_cells), nf = static_cast<std::size_t>(m.n_faces);
    m.ccx.assign(nc, 0.0);
    m.ccy.assign(nc, 0.0);
    m.ccz.assign(nc, 0.0);
    m.vol.assign(nc, 0.0);
    for (std::size_t c = 0; c < nc; ++c) {
        const uint8_t t = m.cell_type[c];
        const int32_t* cn = m.cell_nodes.data() + m.cell_nodes_off[c];
        const int nn = m.cell_nodes_off[c + 1] - m.cell_nodes_off[c];
        double px[8], py[8], pz[8];
        double ax = 0, ay = 0, az = 0;
        for (int i = 0; i < nn; ++i) {
            px[i] = m.node_x[cn[i]];
            py[i] = m.node_y[cn[i]];
            pz[i] = m.node_z[cn[i]];
            ax += px[i];
            ay += py[i];
            az += pz[i];
        }
        ax /= nn;
        ay /= nn;
        az /= nn;
        double V = 0, mx = 0, my = 0, mz = 0;
        auto add_tet = [&](double bx, double by, double bz, double p1x, double p1y, double p1z, double p2x,
                           double p2y, double p2z) {
            // triangle (b, p1, p2) oriented outward, apex at the vertex average
            const double e1x = p1x - bx, e1y = p1y - by, e1z = p1z - bz;
            const double e2x = p2x - bx, e2y = p2y - by, e2z = p2z - bz;
            const double sx = 0.5 * (e1y * e2z - e1z * e2y);
            const double sy = 0.5 * (e1z * e2x - e1x * e2z);
            const double sz = 0.5 * (e1x * e2y - e1y * e2x);
            const double v = (sx * (bx - ax) + sy * (by - ay) + sz * (bz - az)) / 3.0;
            V += v;
            mx += v * 0.25 * (ax + bx + p1x + p2x);
            my += v * 0.25 * (ay + by + p1y + p2y);
            mz += v * 0.25 * (az + bz + p1z + p2z);
        };
        for (int f = 0; f < faces_of(t); ++f) {
            const int fnn = face_nn(t);
            if (fnn == 3) {
                const int i0 = face_local(t, f, 0), i1 = face_local(t, f, 1), i2 = face_local(t, f, 2);
                add_tet(px[i0], py[i0], pz[i0], px[i1], py[i1], pz[i1], px[i2], py[i2], pz[i2]);
            } else {
                double fx = 0, fy = 0, fz = 0;
                for (int j = 0; j < fnn; ++j) {
                    fx += px[face_local(t, f, j)];
                    fy += py[face_local(t, f, j)];
                    fz += pz[face_local(t, f, j)];
                }
                fx /= fnn;
                fy /= fnn;
                fz /= fnn;
                for (int j = 0; j < fnn; ++j) {
                    const int a = face_local(t, f, j), b = face_local(t, f, (j + 1) % fnn);
                    add_tet(fx, fy, fz, px[a], py[a], pz[a], px[b], py[b], pz[b]);
                }
            }
        }
        if (!(V > 1e-15)) {
            err = "non-positive cell volume at cell " + std::to_string(c);
            return false;
        }
        m.vol[c] = V;
        m.ccx[c] = mx / V;
        m.ccy[c] = my / V;
        m.ccz[c] = mz / V;
    }

    m.fcx.assign(nf, 0.0);
    m.fcy.assign(nf, 0.0);
    m.fcz.assign(nf, 0.0);
    m.fnx.assign(nf, 0.0);
    m.fny.assign(nf, 0.0);
    m.fnz.assign(nf, 0.0);
    m.area.assign(nf, 0.0);
    for (std::size_t f = 0; f < nf; ++f) {
        const int32_t* fn = m.fn.data() + m.fn_off[f];
        const int nn = m.fn_off[f + 1] - m.fn_off[f];
        double Sx = 0, Sy = 0, Sz = 0, cx = 0, cy = 0, cz = 0;
        if (nn == 3) {
            const double p0x = m.node_x[fn[0]], p0y = m.node_y[fn[0]], p0z = m.node_z[fn[0]];
            const double p1x = m.node_x[fn[1]], p1y = m.node_y[fn[1]], p1z = m.node_z[fn[1]];
            const double p2x = m.node_x[fn[2]], p2y = m.node_y[fn[2]], p2z = m.node_z[fn[2]];
            const double e1x = p1x - p0x, e1y = p1y - p0y, e1z = p1z - p0z;
            const double e2x = p2x - p0x, e2y = p2y - p0y, e2z = p2z - p0z;
            Sx = 0.5 * (e1y * e2z - e1z * e2y);
            Sy = 0.5 * (e1z * e2x - e1x * e2z);
            Sz = 0.5 * (e1x * e2y - e1y * e2x);
            cx = (p0x + p1x + p2x) / 3.0;
            cy = (p0y + p1y + p2y) / 3.0;
            cz = (p0z + p1z + p2z) / 3.0;
        } else {
            double ox = 0, oy = 0, oz = 0;
            for (int k = 0; k < nn; ++k) {
                ox += m.node_x[fn[k]];
                oy += m.node_y[fn[k]];
                oz += m.node_z[fn[k]];
            }
            ox /= nn;
            oy /= nn;
            oz /= nn;
            double wsum = 0, wx = 0, wy = 0, wz = 0;
            for (int k = 0; k < nn; ++k) {
                const int32_t a = fn[k], b = fn[(k + 1) % nn];
                const double e1x = m.node_x[a] - ox, e1y = m.node_y[a] - oy, e1z = m.node_z[a] - oz;
                const double e2x = m.node_x[b] - ox, e2y = m.node_y[b] - oy, e2z = m.node_z[b] - oz;
                const double tx = 0.5 * (e1y * e2z - e1z * e2y);
                const double ty = 0.5 * (e1z * e2x - e1x * e2z);
                const double tz = 0.5 * (e1x * e2y - e1y * e2x);
                const double ta = std::sqrt(tx * tx + ty * ty + tz * tz);
                Sx += tx;
                Sy += ty;
                Sz += tz;
                wx += ta * (ox + m.node_x[a] + m.node_x[b]) / 3.0;
                wy += ta * (oy + m.node_y[a] + m.node_y[b]) / 3.0;
                wz += ta * (oz + m.node_z[a] + m.node_z[b]) / 3.0;
                wsum += ta;
            }
            if (wsum > 1e-15) {
                cx = wx / wsum;
                cy = wy / wsum;
                cz = wz / wsum;
            } else {
                cx = ox;
                cy = oy;
                cz = oz;
            }
        }
        const double A = std::sqrt(Sx * Sx + Sy * Sy + Sz * Sz);
        if (!(A > 1e-15)) {
            err = "zero-area face " + std::to_string(f);
            return false;
        }
        m.area[f] = A;
        m.fnx[f] = Sx / A;
        m.fny[f] = Sy / A;
        m.fnz[f] = Sz / A;
        m.fcx[f] = cx;
        m.fcy[f] = cy;
        m.fcz[f] = cz;
        // outward from the owner
        const int32_t o = m.owner[f];
        const double dot = m.fnx[f] * (cx - m.ccx[o]) + m.fny[f] * (cy - m.ccy[o]) + m.fnz[f] * (cz - m.ccz[o]);
        if (!(dot > 0.0)) {
            err = "face normal does not point away from its owner at face " + std::to_string(f);
            return false;
        }
    }
    return true;
}

// Reverse Cuthill-McKee (George & Liu): start each component from a
// pseudo-peripheral vertex found by repeated breadth-first search from a
// minimum-degree vertex, visit neighbours in (degree, index) order, reverse.
std::vector<int32_t> rcm_order(const Csr& g) {
    const int32_t n = g.rows();
    std::vector<int32_t> order;
    order.reserve(n);
    std::vector<char> done(n, 0);
    std::vector<int32_t> level(n, -1), queue(n), nbrs;
    auto deg = [&](int32_t v) { return g.off[v + 1] - g.off[v]; };
    auto bfs = [&](int32_t root, int32_t& last_level_min, int32_t& ecc) {
        // returns eccentricity and a min-degree vertex of the last level
        std::vector<int32_t> touched;
        int32_t h = 0, t = 0;
        queue[t++] = root;
        level[root] = 0;
        touched.push_back(root);
        ecc = 0;
        while (h < t) {
            const int32_t v = queue[h++];
            ecc = std::max(ecc, level[v]);
            for (int32_t k = g.off[v]; k < g.off[v + 1]; ++k) {
                const int32_t u = g.val[k];
                if (level[u] < 0 && !done[u]) {
                    level[u] = level[v] + 1;
                    queue[t++] = u;
                    touched.push_back(u);
                }
            }
        }
        last_level_min = -1;
        for (int32_t i = 0; i < t; ++i) {
            const int32_t v = queue[i];
            if (level[v] == ecc && (last_level_min < 0 || deg(v) < deg(last_level_min) ||
                                    (deg(v) == deg(last_level_min) && v < last_level_min)))
                last_level_min = v;
        }
        for (int32_t v : touched) level[v] = -1;
    };
    for (int32_t seed = 0; seed < n; ++seed) {
        if (done[seed]) continue;
        // minimum-degree vertex of this component
        int32_t root = seed;
        {
            int32_t dummy, ecc;
            bfs(seed, dummy, ecc);
        }
        // pseudo-peripheral search
        int32_t ecc = -1;
        for (int iter = 0; iter < 32; ++iter) {
            int32_t cand, e;
            bfs(root, cand, e);
            if (e <= ecc) break;
            ecc = e;
            if (cand == root) break;
            root = cand;
        }
        // Cuthill-McKee from root
        int32_t h = 0, t = 0;
        queue[t++] = root;
        done[root] = 1;
        while (h < t) {
            const int32_t v = queue[h++];
            order.push_back(v);
            nbrs.clear();
            for (int32_t k = g.off[v]; k < g.off[v + 1]; ++k)
                if (!done[g.val[k]]) nbrs.push_back(g.val[k]);
            std::sort(nbrs.begin(), nbrs.end(), [&](int32_t a, int32_t b) {
                return deg(a) != deg(b) ? deg(a) < deg(b) : a < b;
            });
            for (int32_t u : nbrs) {
                done[u] = 1;
                queue[t++] = u;
            }
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}

Csr build_cell_faces(const HostMesh& m) {
    Csr c;
    c.off.assign(static_cast<std::size_t>(m.n_cells) + 1, 0);
    for (int32_t f = 0; f < m.n_faces; ++f) {
        ++c.off[m.owner[f] + 1];
        if (m.neigh[f] >= 0) ++c.off[m.neigh[f] + 1];
    }
    for (int32_t i = 0; i < m.n_cells; ++i) c.off[i + 1] += c.off[i];
    c.val.resize(c.off.back());
    std::vector<int32_t> cur(c.off.begin(), c.off.end() - 1);
    for (int32_t f = 0; f < m.n_faces; ++f) {
        c.val[cur[m.owner[f]]++] = f;
        if (m.neigh[f] >= 0) c.val[cur[m.neigh[f]]++] = f;
    }
    return c;
}

Csr build_cell_cells_face(const HostMesh& m) { return face_graph(m); }

Csr build_cell_cells_node(const HostMesh& m) {
    // node -> cells
    Csr n2c;
    n2c.off.assign(static_cast<std::size_t>(m.n_nodes) + 1, 0);
    for (int32_t n : m.cell_nodes) ++n2c.off[n + 1];
    for (int32_t i = 0; i < m.n_nodes; ++i) n2c.off[i + 1] += n2c.off[i];
    n2c.val.resize(n2c.off.back());
    {
        std::vector<int32_t> cur(n2c.off.begin(), n2c.off.end() - 1);
        for (int32_t c = 0; c < m.n_cells; ++c)
            for (int32_t k = m.cell_nodes_off[c]; k < m.cell_nodes_off[c + 1]; ++k)
                n2c.val[cur[m.cell_nodes[k]]++] = c;
    }
    Csr c2c;
    c2c.off.assign(static_cast<std::size_t>(m.n_cells) + 1, 0);
    std::vector<int32_t> stamp(m.n_cells, -1), buf;
    for (int32_t c = 0; c < m.n_cells; ++c) {
        buf.clear();
        for (int32_t k = m.cell_nodes_off[c]; k < m.cell_nodes_off[c + 1]; ++k) {
            const int32_t n = m.cell_nodes[k];
            for (int32_t j = n2c.off[n]; j < n2c.off[n + 1]; ++j) {
                const int32_t o = n2c.val[j];
                if (o == c || stamp[o] == c) continue;
                stamp[o] = c;
                buf.push_back(o);
            }
        }
        std::sort(buf.begin(), buf.end());
        c2c.val.insert(c2c.val.end(), buf.begin(), buf.end());
        c2c.off[c + 1] = static_cast<int32_t>(c2c.val.size());
    }
    return c2c;
}

// --------------------------------------------------------------- generators
int generate_mesh(const cfdg_mesh_spec& s, HostMesh& m, std::string& err) {
    if (s.nx < 1 || s.ny < 1 || s.nz < 1 || s.kind < 0 || s.kind > 2) {
        err = "invalid mesh spec";
        return CFDG_ERR_INVALID;
    }
    const int64_t NX = s.nx + 1, NY = s.ny + 1, NZ = s.nz + 1;
    const int64_t nn64 = NX * NY * NZ;
    const int64_t ncell64 = int64_t(s.nx) * s.ny * s.nz * (s.kind == 2 ? 6 : 1);
    if (nn64 > INT32_MAX / 2 || ncell64 > INT32_MAX / 8) {
        err = "mesh too large for 32-bit indices";
        return CFDG_ERR_INVALID;
    }
    auto nid = [&](int64_t i, int64_t j, int64_t k) { return static_cast<int32_t>((k * NY + j) * NX + i); };

    // 1. Structured coordinates per kind.
    std::vector<double> xs(NX), ys(NY), zs(NZ);
    for (int64_t i = 0; i < NX; ++i) xs[i] = s.lx * double(i) / double(s.nx);
    for (int64_t k = 0; k < NZ; ++k) zs[k] = s.lz * double(k) / double(s.nz);
    if (s.kind == 1) {
        // geometric wall-normal stretching with optional cap on the spacing
        ys[0] = 0.0;
        double h = s.first_spacing > 0 ? s.first_spacing : s.ly / s.ny;
        for (int64_t j = 1; j < NY; ++j) {
            ys[j] = ys[j - 1] + h;
            double hn = h * (s.stretch > 0 ? s.stretch : 1.0);
            if (s.cap_spacing > 0 && hn > s.cap_spacing) hn = s.cap_spacing;
            h = hn;
        }
    } else {
        for (int64_t j = 0; j < NY; ++j) ys[j] = s.ly * double(j) / double(s.ny);
    }
    auto wall_y = [&](double x) -> double {
        if (s.kind == 0) {
            const double t = std::tan(s.ramp_angle_deg * M_PI / 180.0);
            return std::max(0.0, (x - s.ramp_x) * t);
        }
        if (s.kind == 2 && s.bump_height > 0 && x > s.bump_x0 && x < s.bump_x1) {
            const double half = 0.5 * (s.bump_x1 - s.bump_x0);
            const double h = s.bump_height * (s.bump_x1 - s.bump_x0);
            const double R = (half * half + h * h) / (2.0 * h);
            const double xm = 0.5 * (s.bump_x0 + s.bump_x1);
            return std::sqrt(std::max(0.0, R * R - (x - xm) * (x - xm))) + (h - R);
        }
        return 0.0;
    };
    m.n_nodes = static_cast<int32_t>(nn64);
    m.node_x.resize(nn64);
    m.node_y.resize(nn64);
    m.node_z.resize(nn64);
    for (int64_t k = 0; k < NZ; ++k)
        for (int64_t j = 0; j < NY; ++j)
            for (int64_t i = 0; i < NX; ++i) {
                const int32_t n = nid(i, j, k);
                const double x = xs[i];
                double y;
                if (s.kind == 1) {
                    y = ys[j];
                } else {
                    const double yw = wall_y(x);
                    y = yw + (ys[j] / s.ly) * (s.ly - yw);
                }
                m.node_x[n] = x;
                m.node_y[n] = y;
                m.node_z[n] = zs[k];
            }
    // 2. Seeded node jitter, a fraction of the local spacing.
    //    Plate (wall-normal stretching): every wall-normal grid line moves as
    //    a whole in x and z (by up to `jitter` of the x / z spacing, wall and
    //    top nodes included, which stay on their planes) and every row of
    //    nodes moves as a whole in y (by up to `jitter` of its y spacing).
    //    The cells stay boxes of random size: a cell 1e-5 high whose top
    //    and bottom faces were tilted independently would have its centroid
    //    shifted sideways by ~1e-4, many times its height, and the
    //    least-squares gradients of the stacked cells would mix the
    //    wall-normal derivative into the streamwise one.  Other meshes: each
    //    interior node moves in every coordinate by up to `jitter` of its
    //    shortest edge.
    if (s.jitter > 0) {
        Rng rng(s.seed ^ 0x9e3779b97f4a7c15ULL);
        std::vector<double> x0(m.node_x), y0(m.node_y), z0(m.node_z);
        auto dist = [&](int32_t a, int32_t b) {
            const double dx = x0[a] - x0[b], dy = y0[a] - y0[b], dz = z0[a] - z0[b];
            return std::sqrt(dx * dx + dy * dy + dz * dz);
        };
        if (s.kind == 1) {
            for (int64_t k = 1; k < NZ - 1; ++k)
                for (int64_t i = 1; i < NX - 1; ++i) {
                    const double hx = std::min(xs[i + 1] - xs[i], xs[i] - xs[i - 1]);
                    const double hz = std::min(zs[k + 1] - zs[k], zs[k] - zs[k - 1]);
                    const double ox = s.jitter * hx * rng.sym(), oz = s.jitter * hz * rng.sym();
                    for (int64_t j = 0; j < NY; ++j) {
                        const int32_t n = nid(i, j, k);
                        m.node_x[n] = x0[n] + ox;
                        m.node_z[n] = z0[n] + oz;
                    }
                }
            for (int64_t j = 1; j < NY - 1; ++j) {
                const double oy = s.jitter * std::min(ys[j + 1] - ys[j], ys[j] - ys[j - 1]) * rng.sym();
                for (int64_t k = 0; k < NZ; ++k)
                    for (int64_t i = 0; i < NX; ++i) m.node_y[nid(i, j, k)] = y0[nid(i, j, k)] + oy;
            }
        } else {
            for (int64_t k = 1; k < NZ - 1; ++k)
                for (int64_t j = 1; j < NY - 1; ++j)
                    for (int64_t i = 1; i < NX - 1; ++i) {
                        const int32_t n = nid(i, j, k);
                        const double hx = std::min(dist(n, nid(i + 1, j, k)), dist(n, nid(i - 1, j, k)));
                        const double hy = std::min(dist(n, nid(i, j + 1, k)), dist(n, nid(i, j - 1, k)));
                        const double hz = std::min(dist(n, nid(i, j, k + 1)), dist(n, nid(i, j, k - 1)));
                        const double h = std::min(hx, std::min(hy, hz));
                        m.node_x[n] = x0[n] + s.jitter * h * rng.sym();
                        m.node_y[n] = y0[n] + s.jitter * h * rng.sym();
                        m.node_z[n] = z0[n] + s.jitter * h * rng.sym();
                    }
        }
    }
    // 3. Cells in CGNS order.
    m.cell_type.clear();
    m.cell_nodes_off.assign(1, 0);
    m.cell_nodes.clear();
    for (int64_t k = 0; k < s.nz; ++k)
        for (int64_t j = 0; j < s.ny; ++j)
            for (int64_t i = 0; i < s.nx; ++i) {
                const int32_t v[8] = {nid(i, j, k),         nid(i + 1, j, k),         nid(i + 1, j + 1, k),
                                      nid(i, j + 1, k),     nid(i, j, k + 1),         nid(i + 1, j, k + 1),
                                      nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)};
                if (s.kind != 2) {
                    m.cell_type.push_back(CFDG_HEXA);
                    m.cell_nodes.insert(m.cell_nodes.end(), v, v + 8);
                    m.cell_nodes_off.push_back(static_cast<int32_t>(m.cell_nodes.size()));
                } else {
                    // Kuhn (Freudenthal) split into 6 tetrahedra along the
                    // (0,0,0)-(1,1,1) diagonal; conforming across cubes.
                    static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
                    for (int p = 0; p < 6; ++p) {
                        int bits = 0;
                        int corner[4];
                        corner[0] = 0;
                        for (int q = 0; q < 3; ++q) {
                            bits |= 1 << perm[p][q];
                            corner[q + 1] = bits;
                        }
                        auto vtx = [&](int b) {
                            const int64_t di = b & 1, dj = (b >> 1) & 1, dk = (b >> 2) & 1;
                            return nid(i + di, j + dj, k + dk);
                        };
                        int32_t t4[4] = {vtx(corner[0]), vtx(corner[1]), vtx(corner[2]), vtx(corner[3])};
                        // CGNS TETRA_4: det[n1-n0, n2-n0, n3-n0] > 0
                        auto det = [&](const int32_t* t) {
                            const double ax = m.node_x[t[1]] - m.node_x[t[0]], ay = m.node_y[t[1]] - m.node_y[t[0]],
                                         az = m.node_z[t[1]] - m.node_z[t[0]];
                            const double bx = m.node_x[t[2]] - m.node_x[t[0]], by = m.node_y[t[2]] - m.node_y[t[0]],
                                         bz = m.node_z[t[2]] - m.node_z[t[0]];
                            const double cx = m.node_x[t[3]] - m.node_x[t[0]], cy = m.node_y[t[3]] - m.node_y[t[0]],
                                         cz = m.node_z[t[3]] - m.node_z[t[0]];
                            return ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
                        };
                        if (det(t4) < 0) std::swap(t4[1], t4[2]);
                        m.cell_type.push_back(CFDG_TET);
                        m.cell_nodes.insert(m.cell_nodes.end(), t4, t4 + 4);
                        m.cell_nodes_off.push_back(static_cast<int32_t>(m.cell_nodes.size()));
                    }
                }
            }
    m.n_cells = static_cast<int32_t>(m.cell_type.size());

    // 4. Boundary patches from the structured index of the face nodes.
    //    ramp:  0 inlet(x=0) 1 outlet(x=L) 2 top 3 wall 4 z-planes
    //    plate: 0 inlet 1 outlet 2 top 3 wall (x>=plate_x0) 4 z-planes 5 lower symmetry (x<plate_x0)
    //    bump:  0 inlet 1 outlet 2 top 3 lower wall 4 z-planes
    auto classify = [&](const int32_t* nodes, int nn) -> int32_t {
        bool all_i0 = true, all_iN = true, all_j0 = true, all_jN = true, all_k0 = true, all_kN = true;
        double xc = 0;
        for (int q = 0; q < nn; ++q) {
            const int64_t n = nodes[q];
            const int64_t i = n % NX, j = (n / NX) % NY, k = n / (NX * NY);
            all_i0 &= (i == 0);
            all_iN &= (i == NX - 1);
            all_j0 &= (j == 0);
            all_jN &= (j == NY - 1);
            all_k0 &= (k == 0);
            all_kN &= (k == NZ - 1);
            xc += xs[i];
        }
        xc /= nn;
        if (all_i0) return 0;
        if (all_iN) return 1;
        if (all_jN) return 2;
        if (all_j0) {
            if (s.kind == 1 && xc < s.plate_x0) return 5;
            return 3;
        }
        if (all_k0 || all_kN) return 4;
        return -1;
    };

    // 5. Random permutation, then RCM on the face graph.
    if (!extract_faces(m, classify, err)) return CFDG_ERR_MESH;
    std::vector<int32_t> order(m.n_cells);
    std::iota(order.begin(), order.end(), 0);
    if (s.permute) {
        Rng rng(s.seed);
        for (int32_t i = m.n_cells - 1; i > 0; --i) {
            const int32_t j = static_cast<int32_t>(rng.g() % static_cast<uint64_t>(i + 1));
            std::swap(order[i], order[j]);
        }
        if (!apply_cell_order(m, order, classify, err)) return CFDG_ERR_MESH;
    }
    if (s.reorder_rcm) {
        const Csr g = face_graph(m);
        const std::vector<int32_t> rcm = rcm_order(g);
        if (!apply_cell_order(m, rcm, classify, err)) return CFDG_ERR_MESH;
    }
    // node locality after the final cell order (patch classification above
    // used the structured node ids, which the renumbering destroys)
    renumber_nodes(m);
    // patch count: the plate always has 6 patches, the others 5
    m.n_patches = (s.kind == 1) ? 6 : 5;
    if (!compute_geometry(m, err)) return CFDG_ERR_MESH;
    return CFDG_OK;
}

}  // namespace cfdg
