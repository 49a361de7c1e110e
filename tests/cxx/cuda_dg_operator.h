// The device binding a tandem maintainer adds (INTEGRATION.md sections 1-3), compiled by the
// tests against minimal stand-ins for tandem's AbstractDGOperator and PETSc (tests/cxx/stub):
//
//  * CudaDGOperator<D>: an AbstractDGOperator (src/form/AbstractDGOperator.h:18-52) whose apply
//    forwards device arrays to tdg_apply; built from the FacetInfo arrays of DGOperatorTopo
//    (src/form/FacetInfo.h:17-23) and Curvilinear's geometry nodes;
//  * PetscDGShell: tandem's MatShell (app/common/PetscDGShell.cpp:8-55) with MATOP_MULT on
//    VECCUDA arrays and the C++ exceptions of the operator turned into a PetscErrorCode (tandem's
//    apply returns 0 and lets them propagate);
//  * block Jacobi and one multigrid V-cycle as PCSHELL applies (replacing the assembled-matrix
//    PCs of app/common/PetscLinearSolver.cpp:14-32,53-114).
#pragma once

#include "form/AbstractDGOperator.h"
#include "petsc/petsc_stub.h"
#include "tandem_b200.h"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace tndm {

// Throws on a non-zero tandem_b200 return code, with the library's message.
inline void tdg_check(int rc) {
    if (rc != TDG_OK) throw std::runtime_error(std::string("tandem_b200: ") + tdg_last_error());
}

template <std::size_t D> class CudaDGOperator : public AbstractDGOperator<D> {
public:
    // topology: FacetInfo up[2] / localNo[2] / bc per local facet; geo_nodes: Curvilinear's
    // degree-geo_degree nodes [E][Ngeo][D]; rules: tandem's volRule / fctRule.
    CudaDGOperator(int degree, int geo_degree, std::size_t num_elements, std::vector<int64_t> up,
                   std::vector<int32_t> local_no, std::vector<int32_t> bc, std::vector<double> geo_nodes,
                   tdg_quadrature const& rules, int kind)
        : up_(std::move(up)), loc_(std::move(local_no)), bc_(std::move(bc)), geo_(std::move(geo_nodes)) {
        tdg_mesh_desc m{static_cast<int32_t>(D), degree, geo_degree, 0, static_cast<int64_t>(num_elements),
                        static_cast<int64_t>(bc_.size()), geo_.data(), up_.data(), loc_.data(), bc_.data()};
        tdg_check(tdg_create(&m, &rules, kind, &op_));
        int64_t sizes[8];
        tdg_check(tdg_sizes(op_, sizes));
        bs_ = static_cast<std::size_t>(sizes[0]);
        ne_ = static_cast<std::size_t>(sizes[5]);
    }
    ~CudaDGOperator() override { tdg_destroy(op_); }
    CudaDGOperator(CudaDGOperator const&) = delete;
    CudaDGOperator& operator=(CudaDGOperator const&) = delete;

    std::size_t block_size() const override { return bs_; }
    std::size_t num_local_elements() const override { return ne_; }
    std::size_t flops_apply() const override { return static_cast<std::size_t>(tdg_flops_apply(op_)); }

    // Material at the volume quadrature points (tandem evaluates its functionals at
    // tdg_volume_coords); c1 may be null (Poisson).
    void set_material(std::vector<double> const& c0, std::vector<double> const* c1) {
        tdg_check(tdg_set_material(op_, c0.data(), c1 ? c1->data() : nullptr));
    }
    std::vector<double> volume_coords() const {
        int64_t sizes[8];
        tdg_check(tdg_sizes(op_, sizes));
        std::vector<double> out(static_cast<std::size_t>(sizes[5] * sizes[3] * static_cast<int64_t>(D)));
        tdg_check(tdg_volume_coords(op_, out.data()));
        return out;
    }

    // y = A x on device arrays: no host transfer.
    void apply(BlockVector const& x, BlockVector& y) override {
        const int64_t n = static_cast<int64_t>(this->number_of_local_dofs());
        if (static_cast<int64_t>(x.size()) < n || static_cast<int64_t>(y.size()) < n)
            throw std::invalid_argument("vector shorter than the operator's local dofs");
        tdg_check(tdg_apply(op_, TDG_FP64, x.device_data(), y.device_data(), 1, n, nullptr));
    }

    tdg_op* handle() { return op_; }

private:
    tdg_op* op_ = nullptr;
    std::vector<int64_t> up_;
    std::vector<int32_t> loc_, bc_;
    std::vector<double> geo_;
    std::size_t bs_ = 0, ne_ = 0;
};

// tandem's MatShell around the device operator (PetscDGShell, app/common/PetscDGShell.cpp).
template <std::size_t D> class PetscDGShell {
public:
    explicit PetscDGShell(CudaDGOperator<D>& op) {
        const PetscInt n = static_cast<PetscInt>(op.number_of_local_dofs());
        if (MatCreateShell(n, static_cast<PetscInt>(op.block_size()), &op, &A_) ||
            MatShellSetOperation(A_, MATOP_MULT, reinterpret_cast<void (*)(void)>(apply)))
            throw std::runtime_error("MatShell set-up failed");
    }
    ~PetscDGShell() { MatDestroy(&A_); }
    Mat mat() const { return A_; }

    static PetscErrorCode apply(Mat A, Vec x, Vec y) {
        CudaDGOperator<D>* op = nullptr;
        PetscCall(MatShellGetContext(A, &op));
        const double* xd = nullptr;
        double* yd = nullptr;
        PetscInt nx = 0, ny = 0;
        PetscCall(VecGetLocalSize(x, &nx));
        PetscCall(VecGetLocalSize(y, &ny));
        PetscCall(VecCUDAGetArrayRead(x, &xd));
        PetscCall(VecCUDAGetArrayWrite(y, &yd));
        PetscErrorCode ierr = PETSC_SUCCESS;
        try {
            const BlockVector xv(const_cast<double*>(xd), static_cast<std::size_t>(nx));
            BlockVector yv(yd, static_cast<std::size_t>(ny));
            op->apply(xv, yv);
        } catch (std::exception const&) {
            ierr = PETSC_ERR_LIB;  // the message stays available through tdg_last_error()
        }
        PetscCall(VecCUDARestoreArrayRead(x, &xd));
        PetscCall(VecCUDARestoreArrayWrite(y, &yd));
        return ierr;
    }

private:
    Mat A_ = nullptr;
};

// Block Jacobi (element diagonal blocks inverted on the device) as a PCSHELL apply.
inline PetscErrorCode bjacobi_pc_apply(PC pc, Vec r, Vec z) {
    tdg_op* op = nullptr;
    PetscCall(PCShellGetContext(pc, &op));
    const double* rd = nullptr;
    double* zd = nullptr;
    PetscInt n = 0;
    PetscCall(VecGetLocalSize(r, &n));
    PetscCall(VecCUDAGetArrayRead(r, &rd));
    PetscCall(VecCUDAGetArrayWrite(z, &zd));
    const int rc = tdg_bjacobi_apply(op, TDG_FP64, rd, zd, 1, n, nullptr);
    PetscCall(VecCUDARestoreArrayRead(r, &rd));
    PetscCall(VecCUDARestoreArrayWrite(z, &zd));
    return rc ? PETSC_ERR_LIB : PETSC_SUCCESS;
}

// One p-multigrid V-cycle (tdg_mg_setup done) as a PCSHELL apply, for -ksp_type fgmres / fcg.
inline PetscErrorCode mg_pc_apply(PC pc, Vec r, Vec z) {
    tdg_op* op = nullptr;
    PetscCall(PCShellGetContext(pc, &op));
    const double* rd = nullptr;
    double* zd = nullptr;
    PetscInt n = 0;
    PetscCall(VecGetLocalSize(r, &n));
    PetscCall(VecCUDAGetArrayRead(r, &rd));
    PetscCall(VecCUDAGetArrayWrite(z, &zd));
    const int rc = tdg_mg_apply(op, rd, zd, 1, n, nullptr);
    PetscCall(VecCUDARestoreArrayRead(r, &rd));
    PetscCall(VecCUDARestoreArrayWrite(z, &zd));
    return rc ? PETSC_ERR_LIB : PETSC_SUCCESS;
}

}  // namespace tndm
