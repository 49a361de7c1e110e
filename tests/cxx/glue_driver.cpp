// Test driver of the compiled device binding (cuda_dg_operator.h): reads a mesh, rules, material
// and a vector written by tests/test_cxx_glue.py, builds CudaDGOperator + PetscDGShell, and
//   cpu mode: exercises construction, sizes, the error paths (invalid topology, apply before the
//             material, null arrays) through the C++ exceptions and the shell's PetscErrorCode;
//   gpu mode: MatMult through the shell and the block-Jacobi and multigrid PCSHELL applies on
//             device arrays, writing y = A x and z = D^-1 x for the test to check.
// Every check prints one "name value" line; the process exits non-zero on the first failure.
#include "cuda_dg_operator.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <string>
#include <vector>

namespace {

template <typename T>
std::vector<T> read_bin(std::string const& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot read " + path);
    std::vector<char> raw((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    std::vector<T> out(raw.size() / sizeof(T));
    std::memcpy(out.data(), raw.data(), out.size() * sizeof(T));
    return out;
}

template <typename T>
void write_bin(std::string const& path, std::vector<T> const& v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}

int fails = 0;
void expect(bool ok, const char* what) {
    std::printf("%s %s\n", what, ok ? "ok" : "FAIL");
    if (!ok) ++fails;
}

template <std::size_t D>
int run(std::string const& dir, bool gpu, std::vector<int64_t> const& meta) {
    using namespace tndm;
    const int degree = static_cast<int>(meta[1]), geo_degree = static_cast<int>(meta[2]), kind = static_cast<int>(meta[5]);
    const std::size_t E = static_cast<std::size_t>(meta[3]);
    auto up = read_bin<int64_t>(dir + "/up.bin");
    auto loc = read_bin<int32_t>(dir + "/loc.bin");
    auto bc = read_bin<int32_t>(dir + "/bc.bin");
    auto geo = read_bin<double>(dir + "/geo.bin");
    auto vx = read_bin<double>(dir + "/vx.bin"), vw = read_bin<double>(dir + "/vw.bin");
    auto fx = read_bin<double>(dir + "/fx.bin"), fw = read_bin<double>(dir + "/fw.bin");
    tdg_quadrature rules{static_cast<int32_t>(vw.size()), static_cast<int32_t>(fw.size()), vx.data(), vw.data(),
                         fx.data(), fw.data()};

    // an invalid topology (an element id past the mesh) is reported by the constructor
    {
        auto bad = up;
        bad[0] = static_cast<int64_t>(E) + 5;
        bool threw = false;
        try {
            CudaDGOperator<D> op(degree, geo_degree, E, bad, loc, bc, geo, rules, kind);
        } catch (std::runtime_error const& e) {
            threw = std::string(e.what()).find("tandem_b200") != std::string::npos;
        }
        expect(threw, "invalid_topology_throws");
    }

    CudaDGOperator<D> op(degree, geo_degree, E, up, loc, bc, geo, rules, kind);
    const std::size_t n = op.number_of_local_dofs();
    std::printf("block_size %zu\nnum_local_elements %zu\n", op.block_size(), op.num_local_elements());
    expect(op.num_local_elements() == E, "num_local_elements");
    PetscDGShell<D> shell(op);

    // MatMult before the material: the operator throws, the shell returns PETSC_ERR_LIB and the
    // library keeps the message
    {
        std::vector<double> dx(1), dy(1);  // never dereferenced: the state check comes first
        _p_Vec xv{dx.data(), static_cast<PetscInt>(n)}, yv{dy.data(), static_cast<PetscInt>(n)};
        const PetscErrorCode ierr = MatMult(shell.mat(), &xv, &yv);
        expect(ierr == PETSC_ERR_LIB, "apply_before_material_is_petsc_err_lib");
        expect(std::string(tdg_last_error()).find("tdg_set_material") != std::string::npos,
               "apply_before_material_message");
    }
    // short vectors are rejected before any device work
    {
        std::vector<double> dx(1), dy(1);
        _p_Vec xv{dx.data(), 1}, yv{dy.data(), 1};
        expect(MatMult(shell.mat(), &xv, &yv) == PETSC_ERR_LIB, "short_vector_is_petsc_err_lib");
    }
    auto c0 = read_bin<double>(dir + "/c0.bin");
    std::vector<double> c1;
    if (kind == TDG_ELASTICITY) c1 = read_bin<double>(dir + "/c1.bin");
    op.set_material(c0, kind == TDG_ELASTICITY ? &c1 : nullptr);
    expect(op.flops_apply() > 0, "flops_apply_positive");
    expect(tdg_apply(op.handle(), TDG_FP64, nullptr, nullptr, 1, static_cast<int64_t>(n), nullptr) == TDG_E_INVALID,
           "null_arrays_invalid");
    if (!gpu) return fails;

    // device vectors as VECCUDA holds them
    auto x = read_bin<double>(dir + "/x.bin");
    double *dx = nullptr, *dy = nullptr, *dz = nullptr;
    if (cudaMalloc(&dx, n * sizeof(double)) != cudaSuccess || cudaMalloc(&dy, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dz, n * sizeof(double)) != cudaSuccess)
        throw std::runtime_error("cudaMalloc");
    cudaMemcpy(dx, x.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    _p_Vec xv{dx, static_cast<PetscInt>(n)}, yv{dy, static_cast<PetscInt>(n)}, zv{dz, static_cast<PetscInt>(n)};
    expect(MatMult(shell.mat(), &xv, &yv) == PETSC_SUCCESS, "matmult");
    PC pc = nullptr;
    PCCreateShell(op.handle(), &pc);
    PCShellSetApply(pc, bjacobi_pc_apply);
    tdg_check(tdg_bjacobi_setup(op.handle(), TDG_FP64, nullptr));
    expect(PCApply(pc, &xv, &zv) == PETSC_SUCCESS, "pc_bjacobi");
    cudaDeviceSynchronize();
    std::vector<double> y(n), z(n);
    cudaMemcpy(y.data(), dy, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(z.data(), dz, n * sizeof(double), cudaMemcpyDeviceToHost);
    write_bin(dir + "/y.bin", y);
    write_bin(dir + "/z.bin", z);
    // one V-cycle through the multigrid PCSHELL
    tdg_check(tdg_mg_setup(op.handle(), nullptr, nullptr));
    PCShellSetApply(pc, mg_pc_apply);
    expect(PCApply(pc, &xv, &zv) == PETSC_SUCCESS, "pc_multigrid");
    cudaDeviceSynchronize();
    std::vector<double> zm(n);
    cudaMemcpy(zm.data(), dz, n * sizeof(double), cudaMemcpyDeviceToHost);
    write_bin(dir + "/zm.bin", zm);
    PCDestroy(&pc);
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(dz);
    return fails;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <dir> cpu|gpu\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const bool gpu = std::string(argv[2]) == "gpu";
    try {
        auto meta = read_bin<int64_t>(dir + "/meta.bin");  // dim, degree, geo_degree, E, F, kind
        const int rc = meta[0] == 2 ? run<2>(dir, gpu, meta) : run<3>(dir, gpu, meta);
        std::printf("done %d\n", rc);
        return rc ? 1 : 0;
    } catch (std::exception const& e) {
        std::printf("exception %s\n", e.what());
        return 1;
    }
}
