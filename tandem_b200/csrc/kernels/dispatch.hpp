// Host-side launchers of the device kernels, dispatched from runtime (dim, degree, kind) to the
// compile-time instances.  Each returns 0 or a TDG_E* code.
#pragma once

#include "common.cuh"

#include <cstdint>
#include <cuda_runtime.h>

namespace tdg {

// Degrees with compiled kernel instances.
constexpr int kMinDegree = 1;
constexpr int kMaxDegree = 4;

template <typename T>
int launch_apply(int D, int N, int kind, DevOp<T> const& op, const T* x, T* y, int nrhs,
                 int64_t ld, cudaStream_t s);
struct MmaTiles;
// FP64 apply on the FP64 tensor pipe over signature-grouped element tiles (apply_mma.cuh);
// TDG_E_INVALID when the instance's tables do not fit in shared memory.
// ctas: persistent CTAs per SM requested (clipped to the occupancy limit); 0 = the default
// (1 for the FP64 tensor kernel, the occupancy limit for the FP32 one).
int launch_apply_mma(int D, int N, int kind, DevOp<double> const& op, MmaTiles const& mt, const double* x, double* y,
                     int nrhs, int64_t ld, cudaStream_t s, int ctas = 0);

// Face-centric FP64 apply (apply_face.cuh): volume kernel (y = volume term) then facet kernel
// (y += facet terms, each facet once for both sides).
struct FaceTiles;
int launch_apply_face(int D, int N, int kind, DevOp<double> const& op, MmaTiles const& mt, FaceTiles const& ft,
                      const double* x, double* y, int nrhs, int64_t ld, cudaStream_t s, int ctas = 0);

// Software-pipelined face-centric FP64 apply (apply_face2.cuh): cp.async double-buffered
// coefficient blocks, tile-ordered geometry (TileGeo), both sides' fluxes from one stress.
struct TileGeo;
// qc: volume points per pass of the volume kernel (the M extent of its GEMM tiles is D x qc rows);
// 0 = every point in one pass where the buffers fit two CTAs per SM, else 24; otherwise a multiple
// of face2_pass_step(D) (TDG_E_INVALID else).
int launch_apply_face2(int D, int N, int kind, DevOp<double> const& op, MmaTiles const& mt, FaceTiles const& ft,
                       TileGeo const& tg, const double* x, double* y, int nrhs, int64_t ld, cudaStream_t s,
                       int ctas = 0, int qc = 0);
// Granularity of qc: passes start on whole 8-row GEMM tiles and on whole point quads.
constexpr int face2_pass_step(int D) { return D == 3 ? 8 : 4; }

// Face-centric FP32 apply (apply_face_tc32.cuh), TX = float or double vectors.
struct Tc32Tiles;
// vol05: the volume term on the 5th-generation tensor cores (apply_tc05.cuh) where the shape allows
// it, else the mma.sync volume kernel.
template <typename TX>
int launch_apply_face_tc32(int D, int N, int kind, DevOp<float> const& op, Tc32Tiles const& mt, FaceTiles const& ft,
                           const TX* x, TX* y, int nrhs, int64_t ld, cudaStream_t s, int ctas = 0, bool vol05 = false,
                           int passes = 3);
// The volume term alone on the 5th-generation tensor cores (stores y); TDG_E_INVALID when the
// shape does not fit (more than 64 volume points).
template <typename TX>
int launch_vol_tc05(int D, int N, int kind, DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y,
                    int nrhs, int64_t ld, cudaStream_t s, int passes = 3);

// FP32 apply on the tensor cores in the 3xTF32 form (apply_tc32.cuh); TDG_E_INVALID when the
// shape's shared-memory layout does not fit (the caller then uses the SIMT kernel).
struct Tc32Tiles;
// TX = float (FP32 vectors) or double (FP64 vectors, FP32 operator arithmetic).
template <typename TX>
int launch_apply_tc32(int D, int N, int kind, DevOp<float> const& op, Tc32Tiles const& mt, const TX* x, TX* y,
                      int nrhs, int64_t ld, cudaStream_t s, int ctas = 0, int passes = 3);
int launch_bjac_assemble(int D, int N, int kind, DevOp<double> const& op, double* blk,
                         cudaStream_t s);
template <typename T>
int launch_bjac_invert(int bs, int64_t E, const double* blk, T* inv, int* status, cudaStream_t s);
// z = D^-1 r with inverses stored as TM and vectors TV (TM = float, TV = double: FP32 inverses
// applied to FP64 vectors).
template <typename TM, typename TV>
int launch_bjac_apply(int bs, int64_t E, const TM* inv, const TV* r, TV* z, int nrhs, int64_t ld,
                      cudaStream_t s);

struct DevFault;
// Poisson fault coupling: traction == false: out += rhs of slip; true: out = traction of (u, slip).
int launch_fault(int D, int N, bool traction, DevOp<double> const& op, DevFault const& fl, const double* u,
                 int64_t ld, const double* slip, int64_t ld_slip, double* out, int64_t ld_out, int nrhs,
                 cudaStream_t s);

// Gradient of J with respect to per-element constant (lambda, mu) from state u and adjoint p
// (adjoint.cuh).  dpen: [F][4] penalty derivatives (d/dlam, d/dmu per side) followed by [E][2]
// element (lam, mu); bcq: [F][D][nq] Dirichlet data or null.
int launch_adjoint_lame(int D, int N, DevOp<double> const& op, const double* u, const double* p, const double* bcq,
                        const double* dpen, double* grad, cudaStream_t s);

// Fixed device scratch of tdg_adjoint_lame_gradient_noalloc: 2^20 doubles (8 MiB) per device, a
// static __device__ array.  adjoint_scratch returns its address on the current device (looked up
// once per device); TDG_E_CUDA when the lookup fails.  adjoint_prepare(D, N) looks the address up
// and loads the gradient kernel of that shape on the current device (both may place code or the
// module image in device memory under lazy loading), so that later calls allocate nothing.
constexpr size_t kAdjointScratchDoubles = size_t(1) << 20;
int adjoint_scratch(double** ptr);
int adjoint_prepare(int D, int N);

// y = Minv_rho (x - b) (elasticity inverse mass of the wave operator, wave.cuh); b may be null,
// y may alias x.
struct WaveData;
int launch_inverse_mass(int D, int N, WaveData const& wd, int64_t E, int Nq, const double* x, const double* b,
                        double* y, int nrhs, int64_t ld, cudaStream_t s);

// out[:, j] = G S[:, j] + t tb for k states (Green's-function traction update, gf_traction.cu);
// G row-major [n][ldg], S / out [k][lds / ldo], tb may be null.
int launch_gf_traction(int64_t n, int64_t m, const double* G, int64_t ldg, const double* S, int64_t lds, int k,
                       const double* tb, double t, double* out, int64_t ldo, cudaStream_t s);

// Number of resident CTAs of a kernel on the current device times the SM count, cached.
int device_sm_count();

}  // namespace tdg
