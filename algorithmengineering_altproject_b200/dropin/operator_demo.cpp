// The reference's operator API driven the way its driver drives it (driver.cpp:47-103), from a program
// written against the reference's headers only, linked to the drop-in library.
//
//   operator_demo nely nelx nelz DIR
//
// Reads from DIR: E.bin (numElements doubles, compact element order), u.bin and r.bin (free-DOF
// doubles), fsrc.bin (numElements floats).  Writes to DIR: Ku.bin = K(E)u; z.bin = M r for the
// multigrid preconditioner of E; x.bin and iters.bin = 50 PCG iterations from zero on the cantilever load;
// C.bin and ce.bin = the compliance of x; fdst.bin = the PDE filter of fsrc; xj.bin and itersj.bin = 30
// PCG iterations with the Jacobi preconditioner; sizes.bin = numElements, free DOFs, numNodes.
#include "core.hpp"
#include "fea.hpp"
#include "filter.hpp"
#include "multigrid/multigrid.hpp"
#include "solver.hpp"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

template <class T>
static std::vector<T> load(const std::string& path, size_t n) {
    std::vector<T> v(n);
    std::ifstream f(path, std::ios::binary);
    if (!f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(T)))) {
        std::cerr << "cannot read " << n << " values from " << path << "\n";
        std::exit(2);
    }
    return v;
}

template <class T>
static void save(const std::string& path, const std::vector<T>& v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
}

int main(int argc, char** argv) {
    if (argc < 5) {
        std::cerr << "usage: operator_demo nely nelx nelz DIR\n";
        return 1;
    }
    using namespace top3d;
    const int nely = std::atoi(argv[1]), nelx = std::atoi(argv[2]), nelz = std::atoi(argv[3]);
    const std::string dir = std::string(argv[4]) + "/";
    Problem pb;
    InitialSettings(pb.params);
    CreateVoxelFEAmodel_Cuboid(pb, nely, nelx, nelz);
    ApplyBoundaryConditions(pb);
    const size_t ne = (size_t)pb.mesh.numElements, nf = pb.freeDofIndex.size();
    save(dir + "sizes.bin", std::vector<int64_t>{(int64_t)ne, (int64_t)nf, (int64_t)pb.mesh.numNodes});
    const auto E = load<double>(dir + "E.bin", ne);
    const auto u = load<double>(dir + "u.bin", nf);
    const auto r = load<double>(dir + "r.bin", nf);
    const auto fsrc = load<float>(dir + "fsrc.bin", ne);

    std::vector<double> Ku;
    K_times_u_finest(pb, E, u, Ku);
    save(dir + "Ku.bin", Ku);

    mg::MGPrecondConfig cfg;
    cfg.nonDyadic = true;
    cfg.maxLevels = 5;
    cfg.weight = 0.6f;
    mg::MGHierarchy H;
    std::vector<std::vector<uint8_t>> masks;
    mg::build_static_once(pb, cfg, H, masks);
    Preconditioner M = mg::make_diagonal_preconditioner_from_static(pb, H, masks, E, cfg);
    std::vector<double> z;
    M(r, z);
    save(dir + "z.bin", z);

    std::vector<double> b;
    restrict_to_free(pb, pb.F, b);
    std::vector<double> x(nf, 0.0);
    PCGFreeWorkspace ws;
    const int it = PCG_free(pb, E, b, x, pb.params.cgTol, 50, M, ws);
    save(dir + "x.bin", x);
    save(dir + "iters.bin", std::vector<int32_t>{it});

    DOFData U;
    U.ux.assign((size_t)pb.mesh.numNodes, 0.0);
    U.uy.assign((size_t)pb.mesh.numNodes, 0.0);
    U.uz.assign((size_t)pb.mesh.numNodes, 0.0);
    scatter_from_free(pb, x, U);
    std::vector<double> ce;
    const double C = ComputeCompliance(pb, E, U, ce);
    save(dir + "C.bin", std::vector<double>{C});
    save(dir + "ce.bin", ce);

    PDEFilter pf = SetupPDEFilter(pb, std::sqrt(3.0f));
    PDEFilterWorkspace fws;
    std::vector<float> fdst;
    ApplyPDEFilter(pb, pf, fsrc, fdst, fws);
    save(dir + "fdst.bin", fdst);

    Preconditioner J = make_jacobi_preconditioner(pb, E);
    std::vector<double> xj(nf, 0.0);
    const int itj = PCG_free(pb, E, b, xj, pb.params.cgTol, 30, J, ws);
    save(dir + "xj.bin", xj);
    save(dir + "itersj.bin", std::vector<int32_t>{itj});
    std::cout << "operator_demo: " << ne << " elements, " << nf << " free DOFs, PCG " << it << " / Jacobi " << itj
              << " iterations, C = " << C << "\n";
    return 0;
}
