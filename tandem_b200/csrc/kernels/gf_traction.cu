// Traction update of the discrete Green's function operator (SeasQDDiscreteGreenOperator::
// update_traction, app/form/SeasQDDiscreteGreenOperator.cpp:115-127: MatMult(G, S) then
// VecAXPY(traction, time, t_boundary)) as one kernel: out[:, j] = G S[:, j] + t * tb for k slip
// states.  G is dense row-major [n][ldg] (n x m used); S, out hold k column vectors at leading
// dimensions lds, ldo.  One warp per row of G: the warp streams the row once (coalesced, four
// loads in flight per lane) and forms the dot products of up to kStates states from shared memory,
// so G is read once per group of kStates states; bandwidth-bound (8 n m bytes per group).
#include "dispatch.hpp"

#include "../../../include/tandem_b200.h"

namespace tdg {

namespace {

constexpr int kStates = 4;
constexpr int kWarps = 8;

template <int KS>
__global__ void __launch_bounds__(kWarps * 32) k_gf_traction(int64_t n, int64_t m, const double* __restrict__ G,
                                                              int64_t ldg, const double* __restrict__ S, int64_t lds,
                                                              const double* __restrict__ tb, double t,
                                                              double* __restrict__ out, int64_t ldo) {
    extern __shared__ double s_states[];  // [KS][m]
    for (int64_t i = threadIdx.x; i < KS * m; i += blockDim.x) {
        const int64_t j = i / m, c = i % m;
        s_states[i] = S[j * lds + c];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t row = static_cast<int64_t>(blockIdx.x) * kWarps + (threadIdx.x >> 5);
    if (row >= n) return;
    const double* g = G + row * ldg;
    double acc[KS];
#pragma unroll
    for (int j = 0; j < KS; ++j) acc[j] = 0.0;
    int64_t c = lane;
    for (; c + 96 < m; c += 128) {
        const double g0 = __ldg(g + c), g1 = __ldg(g + c + 32), g2 = __ldg(g + c + 64), g3 = __ldg(g + c + 96);
#pragma unroll
        for (int j = 0; j < KS; ++j) {
            const double* sj = s_states + j * m;
            acc[j] = fma(g0, sj[c], acc[j]);
            acc[j] = fma(g1, sj[c + 32], acc[j]);
            acc[j] = fma(g2, sj[c + 64], acc[j]);
            acc[j] = fma(g3, sj[c + 96], acc[j]);
        }
    }
    for (; c < m; c += 32) {
        const double gv = __ldg(g + c);
#pragma unroll
        for (int j = 0; j < KS; ++j) acc[j] = fma(gv, s_states[j * m + c], acc[j]);
    }
#pragma unroll
    for (int j = 0; j < KS; ++j) {
        double v = acc[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) out[j * ldo + row] = tb ? fma(t, tb[row], v) : v;
    }
}

template <int KS>
int launch_ks(int64_t n, int64_t m, const double* G, int64_t ldg, const double* S, int64_t lds, const double* tb,
              double t, double* out, int64_t ldo, cudaStream_t s) {
    const size_t smem = static_cast<size_t>(KS) * m * sizeof(double);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(k_gf_traction<KS>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) !=
            cudaSuccess)
        return TDG_E_INVALID;
    const int64_t blocks = (n + kWarps - 1) / kWarps;
    k_gf_traction<KS><<<static_cast<unsigned>(blocks), kWarps * 32, smem, s>>>(n, m, G, ldg, S, lds, tb, t, out, ldo);
    return cudaGetLastError() == cudaSuccess ? 0 : TDG_E_CUDA;
}

}  // namespace

int launch_gf_traction(int64_t n, int64_t m, const double* G, int64_t ldg, const double* S, int64_t lds, int k,
                       const double* tb, double t, double* out, int64_t ldo, cudaStream_t s) {
    // the states of one launch live in shared memory: at most 227 KB
    if (static_cast<int64_t>(kStates) * m * 8 > 227 * 1024 || n > (int64_t(1) << 31) * kWarps) return TDG_E_INVALID;
    for (int j0 = 0; j0 < k; j0 += kStates) {
        const int kk = k - j0 < kStates ? k - j0 : kStates;
        const double* Sj = S + j0 * lds;
        double* oj = out + j0 * ldo;
        int rc = kk == 4   ? launch_ks<4>(n, m, G, ldg, Sj, lds, tb, t, oj, ldo, s)
                 : kk == 3 ? launch_ks<3>(n, m, G, ldg, Sj, lds, tb, t, oj, ldo, s)
                 : kk == 2 ? launch_ks<2>(n, m, G, ldg, Sj, lds, tb, t, oj, ldo, s)
                           : launch_ks<1>(n, m, G, ldg, Sj, lds, tb, t, oj, ldo, s);
        if (rc) return rc;
    }
    return 0;
}

}  // namespace tdg
