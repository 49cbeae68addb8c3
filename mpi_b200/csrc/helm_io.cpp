// Output writers: the solution on the plan's grid as a Tecplot point file or a
// legacy-VTK structured grid, in the reference's text format (WriteFile of
// NonPeriodic2D_MPI.cpp:571-650, NonPeriodic3D_MPI.cpp:713-795 and their
// Periodic twins): fixed notation with 8 decimals, tab-separated columns,
// points ordered element, GLL node, y, x (x fastest), element boundaries
// written twice (J or K = Ns * N).  Host code: u is a host array in the plan's
// compact layout [Ns][Nx][(Ny)][N].
#include <fstream>
#include <string>

#include "helm_plan.hpp"

using helm::Plan;

namespace {

struct GridPoint {
    double x, y, z, u;
};

// Calls fn(point) in the reference's order, with the point's solution value.
template <typename Fn>
void for_each_point(const Plan& p, const double* u, Fn fn)
{
    const double dx = p.Lx / p.Nx;
    const double dy = p.dim == 3 ? p.Ly / p.Ny : 0.0;
    const int Ny = p.dim == 3 ? p.Ny : 1, N = p.N;
    for (int e = 0; e < p.Ns; ++e)
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < Ny; ++j)
                for (int i = 0; i < p.Nx; ++i) {
                    const double g = p.gll.nodes[(size_t)e * (N - 1) + k];
                    const size_t idx = (((size_t)e * p.Nx + i) * Ny + j) * N + k;
                    GridPoint pt;
                    pt.x = p.xl + i * dx;
                    if (p.dim == 3) { pt.y = p.yl + j * dy; pt.z = g; }
                    else { pt.y = g; pt.z = 0.0; }
                    pt.u = u[idx];
                    fn(pt);
                }
}

}  // namespace

extern "C" {

int helm_write_tecplot(helm_plan_t plan, const double* u, double (*exact)(double, double, double), const char* path)
{
    if (!plan || !u || !path) return HELM_ERR_INVALID;
    const Plan& p = *reinterpret_cast<const Plan*>(plan);
    if (p.fd || p.batch > 1) return HELM_ERR_UNSUPPORTED;
    std::ofstream out(path, std::ios::out);
    if (!out) {
        helm::set_last_error("output file could not be opened");
        return HELM_ERR_INVALID;
    }
    out.flags(std::ios::dec | std::ios::fixed);
    out.precision(8);
    out << "TITLE = \"Helmholtz solver\"" << std::endl;
    if (p.dim == 3) {
        out << "Variables = \"X\",\"Y\",\"Z\",\"U\",\"Exact\"" << std::endl;
        out << "Zone I = " << p.Nx << ", J = " << p.Ny << ", K = " << p.Ns * p.N << ", DATAPACKING=POINT" << std::endl;
    } else {
        out << "Variables = \"X\",\"Y\",\"U\",\"Exact\"" << std::endl;
        out << "Zone I = " << p.Nx << ", J = " << p.Ns * p.N << ", DATAPACKING=POINT" << std::endl;
    }
    for_each_point(p, u, [&](const GridPoint& pt) {
        const double ex = exact ? exact(pt.x, pt.y, pt.z) : 0.0;
        if (p.dim == 3)
            out << pt.x << "\t" << pt.y << "\t" << pt.z << "\t" << pt.u << "\t" << ex << std::endl;
        else
            out << pt.x << "\t" << pt.y << "\t" << pt.u << "\t" << ex << std::endl;
    });
    return out ? HELM_OK : HELM_ERR_INVALID;
}

int helm_write_vtk(helm_plan_t plan, const double* u, const char* path)
{
    if (!plan || !u || !path) return HELM_ERR_INVALID;
    const Plan& p = *reinterpret_cast<const Plan*>(plan);
    if (p.fd || p.batch > 1) return HELM_ERR_UNSUPPORTED;
    std::ofstream out(path, std::ios::out);
    if (!out) {
        helm::set_last_error("output file could not be opened");
        return HELM_ERR_INVALID;
    }
    out.flags(std::ios::dec | std::ios::fixed);
    out.precision(8);
    const long long npts = (long long)p.Nx * (p.dim == 3 ? p.Ny : 1) * p.Ns * p.N;
    out << "# vtk DataFile Version 3.1" << std::endl;
    out << "Helmholtz solver" << std::endl;
    out << "ASCII" << std::endl;
    out << "DATASET STRUCTURED_GRID" << std::endl;
    if (p.dim == 3)
        out << "DIMENSIONS " << p.Nx << " " << p.Ny << " " << p.Ns * p.N << std::endl;
    else
        out << "DIMENSIONS " << p.Nx << " " << p.Ns * p.N << " " << 1 << std::endl;
    out << "POINTS " << npts << " FLOAT" << std::endl;
    for_each_point(p, u, [&](const GridPoint& pt) { out << pt.x << "\t" << pt.y << "\t" << pt.z << std::endl; });
    out << std::endl << "POINT_DATA " << npts << std::endl;
    out << "SCALARS Phi float" << std::endl << "LOOKUP_TABLE default" << std::endl;
    for_each_point(p, u, [&](const GridPoint& pt) { out << pt.u << std::endl; });
    return out ? HELM_OK : HELM_ERR_INVALID;
}

}  // extern "C"
