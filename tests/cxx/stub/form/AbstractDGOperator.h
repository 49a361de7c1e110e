// Minimal stand-in for tandem's operator interface (src/form/AbstractDGOperator.h:18-52): the
// members the device glue overrides, with tandem's names and signatures; BlockVector stands for a
// device-aware PetscVectorView (app/common/PetscVector.h), the extension the integration adds so
// that apply sees VECCUDA arrays without a host copy.  The rest of the interface (assemble, rhs,
// wave_rhs, project, solution, params, the functional setters) keeps tandem's host implementation
// and is not exercised here.
#pragma once

#include <cstddef>

namespace tndm {

class BlockVector {
public:
    BlockVector(double* device_data, std::size_t size) : data_(device_data), size_(size) {}
    double* device_data() { return data_; }
    double const* device_data() const { return data_; }
    std::size_t size() const { return size_; }

private:
    double* data_;
    std::size_t size_;
};

template <std::size_t D> class AbstractDGOperator {
public:
    virtual ~AbstractDGOperator() {}
    virtual std::size_t block_size() const = 0;
    virtual std::size_t num_local_elements() const = 0;
    virtual std::size_t number_of_local_dofs() const { return block_size() * num_local_elements(); }
    virtual void apply(BlockVector const& x, BlockVector& y) = 0;
    virtual std::size_t flops_apply() const = 0;
};

}  // namespace tndm
