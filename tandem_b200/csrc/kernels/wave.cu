// Launcher of the inverse-mass kernel of the explicit wave operator (wave.cuh).
#include "dispatch.hpp"
#include "wave.cuh"

#include "../../../include/tandem_b200.h"

namespace tdg {

namespace {
template <int D, int N>
int run_imass(WaveData const& wd, int64_t E, int Nq, const double* x, const double* b, double* y, int nrhs, int64_t ld,
              cudaStream_t s) {
    using S = Shape<D, N, kElasticity>;
    const size_t smem = sizeof(double) * (2 * S::BS + static_cast<size_t>(Nq) * S::Q);
    if (E > 0x7fffffff || nrhs > 65535) return TDG_E_INVALID;
    dim3 grid(static_cast<unsigned>(E), static_cast<unsigned>(nrhs));
    inverse_mass_kernel<S><<<grid, kWaveThreads, smem, s>>>(wd, E, Nq, x, b, y, ld);
    return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
}
template <int D>
int imass_deg(int N, WaveData const& wd, int64_t E, int Nq, const double* x, const double* b, double* y, int nrhs,
              int64_t ld, cudaStream_t s) {
    switch (N) {
        case 1: return run_imass<D, 1>(wd, E, Nq, x, b, y, nrhs, ld, s);
        case 2: return run_imass<D, 2>(wd, E, Nq, x, b, y, nrhs, ld, s);
        case 3: return run_imass<D, 3>(wd, E, Nq, x, b, y, nrhs, ld, s);
        case 4: return run_imass<D, 4>(wd, E, Nq, x, b, y, nrhs, ld, s);
        default: return TDG_E_INVALID;
    }
}
}  // namespace

int launch_inverse_mass(int D, int N, WaveData const& wd, int64_t E, int Nq, const double* x, const double* b,
                        double* y, int nrhs, int64_t ld, cudaStream_t s) {
    if (D == 2) return imass_deg<2>(N, wd, E, Nq, x, b, y, nrhs, ld, s);
    if (D == 3) return imass_deg<3>(N, wd, E, Nq, x, b, y, nrhs, ld, s);
    return TDG_E_INVALID;
}

}  // namespace tdg
