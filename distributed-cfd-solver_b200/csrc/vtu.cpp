// Solution output as VTK XML unstructured grid, the files of the
// reference's Solver::write_fields (include/cfd/solver/compressible/solver.hpp:856-898)
// through io::vtk::write_solution_vtu (src/io/vtk/vtu.cpp:321-470) at one
// rank: <outdir>/<stem>_00000.vtu (points, cells, CellData rank + fields,
// ASCII) and the <outdir>/<stem>.pvtu collection naming it.  The fields
// are formed on the device from the resident state (k_output_fields) and
// copied to the host once; the mesh comes from the caller, who owns it as
// the reference's MeshPart.
#include <cuda_runtime.h>

#include <cstdio>
#include <filesystem>
#include <memory>
#include <string>
#include <vector>

#include "solver.hpp"

namespace cfdg {
namespace {

// CGNS element type -> VTK cell type (to_vtk_cell_type, vtu.cpp:20-31).
unsigned vtk_type(uint8_t t) {
    switch (t) {
        case CFDG_TRI: return 5;
        case CFDG_QUAD: return 9;
        case CFDG_TET: return 10;
        case CFDG_HEXA: return 12;
        case CFDG_PRISM: return 13;
        case CFDG_PYRA: return 14;
        default: return 0;
    }
}

struct File {
    FILE* f = nullptr;
    std::vector<char> buf;
    explicit File(const std::string& path) : f(std::fopen(path.c_str(), "wb")), buf(1 << 20) {
        if (!f) throw Failure{CFDG_ERR_INVALID, "cannot open " + path + " for writing"};
        std::setvbuf(f, buf.data(), _IOFBF, buf.size());
    }
    ~File() {
        if (f) std::fclose(f);
    }
};

}  // namespace

void Solver::write_vtu(const cfdg_mesh_host& m, const std::string& outdir, const std::string& stem) {
    if (m.n_cells != dm_.n || !m.cell_type || !m.cell_nodes_offsets || !m.cell_nodes || !m.node_x || !m.node_y ||
        !m.node_z)
        throw Failure{CFDG_ERR_INVALID, "write_vtu: the mesh does not match the solver"};
    const int32_t n = dm_.n;
    const int nf = sa_ ? 8 : 6;
    static const char* kNames[8] = {"rho", "u", "v", "w", "pressure", "mach", "nu_tilde", "mu_t"};
    DevArray<double> out;
    alloc_or_throw(out, static_cast<std::size_t>(n) * nf, "output fields");
    launch_output_fields(n, nv_, U_.p, gas_, sap_.cv1, out.p, stream_);
    cuda_check(cudaGetLastError(), "output launch");
    std::vector<double> h(static_cast<std::size_t>(n) * nf);
    cuda_check(cudaMemcpyAsync(h.data(), out.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_), "D2H");
    cuda_check(cudaStreamSynchronize(stream_), "output sync");

    std::error_code ec;
    std::filesystem::create_directories(outdir, ec);
    {
        File file(outdir + "/" + stem + "_00000.vtu");
        FILE* f = file.f;
        std::fprintf(f, "<?xml version=\"1.0\"?>\n");
        std::fprintf(f, "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
        std::fprintf(f, "  <UnstructuredGrid>\n");
        std::fprintf(f, "    <Piece NumberOfPoints=\"%d\" NumberOfCells=\"%d\">\n", m.n_nodes, n);
        std::fprintf(f, "      <Points>\n");
        std::fprintf(f, "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n");
        for (int32_t i = 0; i < m.n_nodes; ++i)
            std::fprintf(f, "          %.16g %.16g %.16g\n", m.node_x[i], m.node_y[i], m.node_z[i]);
        std::fprintf(f, "        </DataArray>\n");
        std::fprintf(f, "      </Points>\n");
        std::fprintf(f, "      <Cells>\n");
        std::fprintf(f, "        <DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n");
        for (int32_t c = 0; c < n; ++c) {
            std::fprintf(f, "          ");
            for (int32_t k = m.cell_nodes_offsets[c]; k < m.cell_nodes_offsets[c + 1]; ++k)
                std::fprintf(f, "%d ", m.cell_nodes[k]);
            std::fprintf(f, "\n");
        }
        std::fprintf(f, "        </DataArray>\n");
        std::fprintf(f, "        <DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n          ");
        for (int32_t c = 0; c < n; ++c) std::fprintf(f, "%d ", m.cell_nodes_offsets[c + 1]);
        std::fprintf(f, "\n        </DataArray>\n");
        std::fprintf(f, "        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n          ");
        for (int32_t c = 0; c < n; ++c) std::fprintf(f, "%u ", vtk_type(m.cell_type[c]));
        std::fprintf(f, "\n        </DataArray>\n");
        std::fprintf(f, "      </Cells>\n");
        std::fprintf(f, "      <CellData>\n");
        std::fprintf(f, "        <DataArray type=\"Int32\" Name=\"rank\" format=\"ascii\">\n          ");
        for (int32_t c = 0; c < n; ++c) std::fprintf(f, "%d ", 0);
        std::fprintf(f, "\n        </DataArray>\n");
        for (int k = 0; k < nf; ++k) {
            std::fprintf(f, "        <DataArray type=\"Float64\" Name=\"%s\" format=\"ascii\">\n          ", kNames[k]);
            const double* v = h.data() + static_cast<std::size_t>(k) * n;
            for (int32_t c = 0; c < n; ++c) std::fprintf(f, "%.10e ", v[c]);
            std::fprintf(f, "\n        </DataArray>\n");
        }
        std::fprintf(f, "      </CellData>\n");
        std::fprintf(f, "    </Piece>\n");
        std::fprintf(f, "  </UnstructuredGrid>\n");
        std::fprintf(f, "</VTKFile>\n");
        if (std::ferror(f)) throw Failure{CFDG_ERR_INVALID, "write_vtu: write error"};
    }
    {
        File file(outdir + "/" + stem + ".pvtu");
        FILE* f = file.f;
        std::fprintf(f, "<?xml version=\"1.0\"?>\n");
        std::fprintf(f, "<VTKFile type=\"PUnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n");
        std::fprintf(f, "  <PUnstructuredGrid GhostLevel=\"0\">\n");
        std::fprintf(f, "    <PCellData>\n");
        std::fprintf(f, "      <PDataArray type=\"Int32\" Name=\"rank\"/>\n");
        for (int k = 0; k < nf; ++k) std::fprintf(f, "      <PDataArray type=\"Float64\" Name=\"%s\"/>\n", kNames[k]);
        std::fprintf(f, "    </PCellData>\n");
        std::fprintf(f, "    <PPoints>\n");
        std::fprintf(f, "      <PDataArray type=\"Float64\" NumberOfComponents=\"3\"/>\n");
        std::fprintf(f, "    </PPoints>\n");
        std::fprintf(f, "    <Piece Source=\"%s_%05d.vtu\"/>\n", stem.c_str(), 0);
        std::fprintf(f, "  </PUnstructuredGrid>\n");
        std::fprintf(f, "</VTKFile>\n");
    }
}

}  // namespace cfdg
