// io.cpp -- visualisation and checkpoint output of a forest and its state.
//
// VTK: the reference writes, per visualisation interval, an unstructured
// VTK file through p4est_vtk (src/amr/src/amr_vtk.c:23-106): one quad cell
// per quadrant, its corners shrunk by 0.99999 towards the quadrant's centre,
// cell data tree / level / MPI rank, and point data rho, rhou, rhov, rhoe
// equal to the patch average at all four corners (interpolate_solution,
// amr_vtk.c:109-217). amrgpu_write_vtk writes the same content as an XML
// UnstructuredGrid (.vtu, ASCII); with `subgrid` set it writes every
// subgrid cell as its own quad with its own values (cell data) instead.
//
// Checkpoint: the reference saves the p4est forest with each quadrant's
// data to WRK/checkpoint/amr_soln_%07d.bin (amr_evolve.c:61-64, p4est_save)
// and has no reader. amrgpu_checkpoint_write saves the host forest, the
// AoS state (the reference's soln layout), the step and the time, and
// amrgpu_checkpoint_read restores them, so a run can restart.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "amrgpu_internal.h"

using namespace amrgpu;

namespace {

constexpr uint64_t kCheckpointMagic = 0x31504b43524d4147ULL;  // "GAMRCKP1"

struct CheckpointHeader {
    uint64_t magic;
    int32_t nquad, n, nfields, istep;
    double time;
    uint64_t forest_bytes, soln_doubles;
};

bool write_all(FILE *fp, const void *p, size_t n) { return n == 0 || std::fwrite(p, 1, n, fp) == n; }

}  // namespace

extern "C" {

int amrgpu_write_vtk(const char *path, const amrgpu_forest_t *forest, int n, const double *soln, int subgrid)
{
    if (!path || !forest || !forest->f || n < 1 || !soln) return AMRGPU_ERR_ARG;
    const std::vector<Leaf> &leaves = forest_leaves(forest->f);
    const size_t nq = leaves.size();
    FILE *fp = std::fopen(path, "w");
    if (!fp) {
        set_error(AMRGPU_ERR_IO, std::string("cannot open ") + path);
        return AMRGPU_ERR_IO;
    }
    const size_t ncell = subgrid ? nq * size_t(n) * size_t(n) : nq;
    std::fprintf(fp,
                 "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" "
                 "byte_order=\"LittleEndian\">\n<UnstructuredGrid>\n<Piece NumberOfPoints=\"%zu\" "
                 "NumberOfCells=\"%zu\">\n<Points>\n<DataArray type=\"Float64\" NumberOfComponents=\"3\" "
                 "format=\"ascii\">\n",
                 4 * ncell, ncell);
    const char *names[4] = {"rho", "rhou", "rhov", "rhoe"};
    const size_t per = 4 * size_t(n) * size_t(n);
    for (size_t q = 0; q < nq; ++q) {
        double g[12];
        forest_quad_corners(forest->f, leaves[q], g);
        if (!subgrid) {
            // corners n1(-,-) n2(+,-) n4(+,+) n3(-,+) in VTK_QUAD order,
            // shrunk by 0.99999 towards the centre as the reference's scale
            const double cx = 0.25 * (g[0] + g[3] + g[6] + g[9]), cy = 0.25 * (g[1] + g[4] + g[7] + g[10]);
            for (int k : {0, 1, 3, 2})
                std::fprintf(fp, "%.17g %.17g 0\n", cx + 0.99999 * (g[3 * k] - cx), cy + 0.99999 * (g[3 * k + 1] - cy));
        } else {
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i)
                    for (int k : {0, 1, 3, 2}) {
                        // bilinear position of sub-cell corner (i + k&1, j + k>>1)
                        const double xi = double(i + (k & 1)) / n, eta = double(j + (k >> 1)) / n;
                        const double x = (1 - xi) * (1 - eta) * g[0] + xi * (1 - eta) * g[3] + (1 - xi) * eta * g[6] +
                                         xi * eta * g[9];
                        const double y = (1 - xi) * (1 - eta) * g[1] + xi * (1 - eta) * g[4] + (1 - xi) * eta * g[7] +
                                         xi * eta * g[10];
                        std::fprintf(fp, "%.17g %.17g 0\n", x, y);
                    }
        }
    }
    std::fprintf(fp, "</DataArray>\n</Points>\n<Cells>\n<DataArray type=\"Int64\" Name=\"connectivity\" "
                     "format=\"ascii\">\n");
    for (size_t c = 0; c < ncell; ++c)
        std::fprintf(fp, "%zu %zu %zu %zu\n", 4 * c, 4 * c + 1, 4 * c + 2, 4 * c + 3);
    std::fprintf(fp, "</DataArray>\n<DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n");
    for (size_t c = 0; c < ncell; ++c) std::fprintf(fp, "%zu\n", 4 * (c + 1));
    std::fprintf(fp, "</DataArray>\n<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n");
    for (size_t c = 0; c < ncell; ++c) std::fprintf(fp, "9\n");  // VTK_QUAD
    std::fprintf(fp, "</DataArray>\n</Cells>\n<CellData Scalars=\"level\">\n");
    std::fprintf(fp, "<DataArray type=\"Int32\" Name=\"treeid\" format=\"ascii\">\n");
    for (size_t c = 0; c < ncell; ++c) std::fprintf(fp, "%d\n", leaves[subgrid ? c / (size_t(n) * n) : c].tree);
    std::fprintf(fp, "</DataArray>\n<DataArray type=\"Int32\" Name=\"level\" format=\"ascii\">\n");
    for (size_t c = 0; c < ncell; ++c) std::fprintf(fp, "%d\n", leaves[subgrid ? c / (size_t(n) * n) : c].level);
    std::fprintf(fp, "</DataArray>\n<DataArray type=\"Int32\" Name=\"mpirank\" format=\"ascii\">\n");
    for (size_t c = 0; c < ncell; ++c) std::fprintf(fp, "0\n");
    std::fprintf(fp, "</DataArray>\n");
    if (subgrid) {
        for (int f = 0; f < 4; ++f) {
            std::fprintf(fp, "<DataArray type=\"Float64\" Name=\"%s\" format=\"ascii\">\n", names[f]);
            for (size_t c = 0; c < ncell; ++c) std::fprintf(fp, "%.17g\n", soln[4 * c + size_t(f)]);
            std::fprintf(fp, "</DataArray>\n");
        }
        std::fprintf(fp, "</CellData>\n<PointData>\n</PointData>\n");
    } else {
        std::fprintf(fp, "</CellData>\n<PointData Scalars=\"rho\">\n");
        // patch averages (interpolate_solution): sum over the patch in
        // row-major order, times 1/(n*n)
        std::vector<double> avg(nq * 4, 0.0);
        const double inv = 1.0 / double(n * n);
        for (size_t q = 0; q < nq; ++q) {
            double u[4] = {0.0, 0.0, 0.0, 0.0};
            for (int c = 0; c < n * n; ++c)
                for (int f = 0; f < 4; ++f) u[f] += soln[q * per + 4 * size_t(c) + size_t(f)];
            for (int f = 0; f < 4; ++f) avg[4 * q + size_t(f)] = u[f] * inv;
        }
        for (int f = 0; f < 4; ++f) {
            std::fprintf(fp, "<DataArray type=\"Float64\" Name=\"%s\" format=\"ascii\">\n", names[f]);
            for (size_t q = 0; q < nq; ++q)
                for (int k = 0; k < 4; ++k) std::fprintf(fp, "%.17g\n", avg[4 * q + size_t(f)]);
            std::fprintf(fp, "</DataArray>\n");
        }
        std::fprintf(fp, "</PointData>\n");
    }
    std::fprintf(fp, "</Piece>\n</UnstructuredGrid>\n</VTKFile>\n");
    const bool ok = std::ferror(fp) == 0;
    if (std::fclose(fp) != 0 || !ok) {
        set_error(AMRGPU_ERR_IO, std::string("write failed: ") + path);
        return AMRGPU_ERR_IO;
    }
    return AMRGPU_OK;
}

int amrgpu_checkpoint_write(const char *path, const amrgpu_forest_t *forest, int n, const double *soln, int istep,
                            double time)
{
    if (!path || !forest || !forest->f || n < 1 || !soln) return AMRGPU_ERR_ARG;
    const std::vector<unsigned char> img = forest_save(forest->f);
    const size_t nq = forest_leaves(forest->f).size();
    CheckpointHeader h{};
    h.magic = kCheckpointMagic;
    h.nquad = int32_t(nq);
    h.n = n;
    h.nfields = 4;
    h.istep = istep;
    h.time = time;
    h.forest_bytes = img.size();
    h.soln_doubles = uint64_t(nq) * 4 * uint64_t(n) * uint64_t(n);
    FILE *fp = std::fopen(path, "wb");
    if (!fp) {
        set_error(AMRGPU_ERR_IO, std::string("cannot open ") + path);
        return AMRGPU_ERR_IO;
    }
    const bool ok = write_all(fp, &h, sizeof(h)) && write_all(fp, img.data(), img.size()) &&
                    write_all(fp, soln, sizeof(double) * size_t(h.soln_doubles));
    if (std::fclose(fp) != 0 || !ok) {
        set_error(AMRGPU_ERR_IO, std::string("write failed: ") + path);
        return AMRGPU_ERR_IO;
    }
    return AMRGPU_OK;
}

int amrgpu_checkpoint_read_header(const char *path, int *nquad, int *n, int *istep, double *time)
{
    if (!path) return AMRGPU_ERR_ARG;
    FILE *fp = std::fopen(path, "rb");
    if (!fp) {
        set_error(AMRGPU_ERR_IO, std::string("cannot open ") + path);
        return AMRGPU_ERR_IO;
    }
    CheckpointHeader h{};
    const bool ok = std::fread(&h, 1, sizeof(h), fp) == sizeof(h) && h.magic == kCheckpointMagic;
    std::fclose(fp);
    if (!ok) {
        set_error(AMRGPU_ERR_IO, std::string("not a checkpoint: ") + path);
        return AMRGPU_ERR_IO;
    }
    if (nquad) *nquad = h.nquad;
    if (n) *n = h.n;
    if (istep) *istep = h.istep;
    if (time) *time = h.time;
    return AMRGPU_OK;
}

int amrgpu_checkpoint_read(const char *path, amrgpu_forest_t **forest, double *soln, long long soln_capacity)
{
    if (!path || !forest || !soln) return AMRGPU_ERR_ARG;
    *forest = nullptr;
    FILE *fp = std::fopen(path, "rb");
    if (!fp) {
        set_error(AMRGPU_ERR_IO, std::string("cannot open ") + path);
        return AMRGPU_ERR_IO;
    }
    CheckpointHeader h{};
    bool ok = std::fread(&h, 1, sizeof(h), fp) == sizeof(h) && h.magic == kCheckpointMagic && h.nfields == 4 &&
              h.n >= 1 && h.nquad >= 1 && h.forest_bytes < (uint64_t(1) << 40) &&
              h.soln_doubles == uint64_t(h.nquad) * 4 * uint64_t(h.n) * uint64_t(h.n);
    if (ok && (long long)h.soln_doubles > soln_capacity) {
        std::fclose(fp);
        set_error(AMRGPU_ERR_ARG, "checkpoint_read: soln buffer too small");
        return AMRGPU_ERR_ARG;
    }
    std::vector<unsigned char> img;
    if (ok) {
        img.resize(size_t(h.forest_bytes));
        ok = std::fread(img.data(), 1, img.size(), fp) == img.size() &&
             std::fread(soln, sizeof(double), size_t(h.soln_doubles), fp) == size_t(h.soln_doubles);
    }
    std::fclose(fp);
    Forest *f = ok ? forest_load(img.data(), img.size()) : nullptr;
    if (!f || forest_num_quads(f) != h.nquad) {
        if (f) forest_destroy(f);
        set_error(AMRGPU_ERR_IO, std::string("corrupt checkpoint: ") + path);
        return AMRGPU_ERR_IO;
    }
    *forest = new amrgpu_forest{f};
    return AMRGPU_OK;
}

}  // extern "C"
