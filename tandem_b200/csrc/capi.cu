// C ABI of tandem_b200 (include/tandem_b200.h): operator handle, device upload, apply,
// block-Jacobi and the device Krylov drivers.
#include "../../include/tandem_b200.h"
#include "host/setup.hpp"
#include "kernels/apply_mma.cuh"
#include "kernels/apply_tc32.cuh"
#include "kernels/apply_face.cuh"
#include "kernels/apply_face_tc32.cuh"
#include "kernels/apply_face2.cuh"
#include "kernels/wave.cuh"
#include "kernels/dispatch.hpp"
#include "kernels/krylov.cuh"
#include "kernels/gmres.cuh"
#include "kernels/mg.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <cstring>
#include <exception>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

namespace tdg {

__global__ void k_dot_finalize(const double* __restrict__ partial, const int* __restrict__ seg_chunk,
                               double* __restrict__ scal, int slot0, int slot1) {
    const int seg = blockIdx.x;
    double s0 = 0.0, s1 = 0.0;
    for (int i = seg_chunk[seg] + threadIdx.x; i < seg_chunk[seg + 1]; i += blockDim.x) {
        s0 += partial[2 * static_cast<int64_t>(i)];
        s1 += partial[2 * static_cast<int64_t>(i) + 1];
    }
    __shared__ double red[2][32];
    s0 = block_sum(s0, red[0]);
    s1 = block_sum(s1, red[1]);
    if (threadIdx.x == 0) {
        if (slot0 >= 0) scal[seg * kScal + slot0] = s0;
        if (slot1 >= 0) scal[seg * kScal + slot1] = s1;
    }
}

__global__ void k_cg_shift(double* __restrict__ scal, int nseg, int only_replaced) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nseg && scal[r * kScal + kActive] != 0.0 && (!only_replaced || scal[r * kScal + kRepl] != 0.0))
        scal[r * kScal + kRZ] = scal[r * kScal + kRZnew];
}

// ---- device-side loop control (CUDA graph conditional `while` nodes) -------------------------------
//
// A loop whose trip count depends on device data (a Krylov block that ends when a segment asks for a
// reliable update, the coarse CG of the multigrid preconditioner that ends at its tolerance) runs as
// a conditional while node of a CUDA graph: its body ends with one of the control kernels below,
// which sets the loop condition from the Krylov scalars.  Every loop is bounded by an iteration
// limit that the control kernel itself counts, so it ends even when no segment converges.
//
// Loop counters, per operator (long long each): kLoopIts iterations of the current outer block,
// kLoopLimit its limit (written by the host before each launch), kCoarseIts iterations of the
// current coarse solve, kCoarseDiverged set when a coarse column's residual is not finite,
// kCoarseTotal coarse iterations since the multigrid set-up.
enum LoopSlot { kLoopIts = 0, kLoopLimit = 1, kCoarseIts = 2, kCoarseDiverged = 3, kCoarseTotal = 4, kLoopSlots = 8 };
// Krylov scalar slot of the outer block's stopping threshold: max(delta rmax, tol)^2 per segment.
constexpr int kThr = 9;
static_assert(kThr < kScal, "threshold slot inside the scalar row");

// After each iteration of a device-looped Krylov block: counts it and ends the loop when an active
// segment's recurrence residual r.r met its threshold scal[kThr] or is not finite, or when the
// block's limit is reached.  One CTA.
__global__ void k_block_ctl(const double* __restrict__ scal, int nseg, long long* __restrict__ ctl,
                            cudaGraphConditionalHandle h) {
    __shared__ int stop;
    if (threadIdx.x == 0) stop = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < nseg; i += blockDim.x) {
        const double* sc = scal + static_cast<int64_t>(i) * kScal;
        const double rr = sc[kRR];
        if (sc[kActive] != 0.0 && !(rr > sc[kThr] && rr < INFINITY)) stop = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const long long n = ++ctl[kLoopIts];
        cudaGraphSetConditional(h, (stop || n >= ctl[kLoopLimit]) ? 0u : 1u);
    }
}

// Coarse CG control of the multigrid preconditioner, one CTA.  mode 0, before the loop: tolerance
// scal[kThr] = rtol2 r0.r0 per column, columns with r0 = 0 inactive, counter reset.  mode 1, after
// each block of `block` iterations: columns whose r.r met their tolerance stop, a non-finite r.r
// stops its column and raises the divergence flag.  Both set the loop condition: a column is
// active and fewer than max_it iterations ran.  mode 2, after the loop: the solve's iterations
// are added to the running total.
__global__ void k_coarse_ctl(double* __restrict__ scal, int ncol, double rtol2, long long* __restrict__ ctl,
                             int max_it, int block, int mode, cudaGraphConditionalHandle h) {
    if (mode == 2) {
        if (threadIdx.x == 0) ctl[kCoarseTotal] += ctl[kCoarseIts];
        return;
    }
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    int mine = 0;
    for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
        double* sc = scal + static_cast<int64_t>(c) * kScal;
        const double rr = sc[kRR];
        if (mode == 0) {
            sc[kThr] = rtol2 * rr;
            sc[kActive] = rr > 0.0 ? 1.0 : 0.0;
        } else if (sc[kActive] != 0.0) {
            if (!(rr < INFINITY) || rr != rr) {
                sc[kActive] = 0.0;
                ctl[kCoarseDiverged] = 1;
            } else if (rr <= sc[kThr]) {
                sc[kActive] = 0.0;
            }
        }
        mine |= sc[kActive] != 0.0;
    }
    if (mine) any = 1;
    __syncthreads();
    if (threadIdx.x == 0) {
        const long long n = mode == 0 ? 0 : ctl[kCoarseIts] + block;
        ctl[kCoarseIts] = n;
        cudaGraphSetConditional(h, (any && n < max_it) ? 1u : 0u);
    }
}

}  // namespace tdg

using namespace tdg;

namespace {

thread_local std::string g_last_error;

int fail(int code, std::string const& msg) {
    g_last_error = msg;
    return code;
}

#define TDG_CUDA_TRY(expr)                                                                   \
    do {                                                                                     \
        cudaError_t err_ = (expr);                                                           \
        if (err_ != cudaSuccess)                                                             \
            return fail(err_ == cudaErrorMemoryAllocation ? TDG_E_NOMEM : TDG_E_CUDA,        \
                        std::string(#expr) + ": " + cudaGetErrorString(err_));              \
    } while (0)

#define TDG_TRY(expr)                                                                        \
    do {                                                                                     \
        int rc_ = (expr);                                                                    \
        if (rc_ != 0) {                                                                      \
            if (g_last_error.empty()) g_last_error = std::string(#expr) + " failed";         \
            return rc_;                                                                      \
        }                                                                                    \
    } while (0)

// A set of device allocations freed together.
struct DevArena {
    std::vector<void*> ptrs;
    template <typename T>
    cudaError_t alloc(T** p, size_t n) {
        void* v = nullptr;
        cudaError_t e = cudaMalloc(&v, n * sizeof(T) + 16);
        if (e == cudaSuccess) {
            ptrs.push_back(v);
            *p = static_cast<T*>(v);
        }
        return e;
    }
    template <typename T>
    cudaError_t upload(T const** out, std::vector<T> const& h) {
        T* d = nullptr;
        cudaError_t e = alloc(&d, h.size());
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
        *out = d;
        return e;
    }
    void release() {
        for (void* p : ptrs) cudaFree(p);
        ptrs.clear();
    }
    ~DevArena() { release(); }
};

template <typename T>
std::vector<T> conv(std::vector<double> const& v) {
    return std::vector<T>(v.begin(), v.end());
}

}  // namespace

namespace {

// One level of the p-multigrid hierarchy.  Coarse levels hold their Galerkin operator as element
// block-sparse blocks A [E][NB][bs][bs]; the finest level is the matrix-free operator.  ip is the
// interpolation from this level to the next finer one.  x, b are the level's solution and
// right-hand side (the caller's z and r on the finest level), r, d, y, w work vectors; every
// vector holds up to `cap` columns at stride ld (the caller's ld on the finest level, n below).
struct MgLevel {
    int degree = 0, bs = 0;
    int64_t n = 0, ld = 0;
    double* A = nullptr;
    float* A32 = nullptr;  // FP32 copy of A for the smoother under mixed precision (levels below the finest)
    double* dinv = nullptr;
    MgInterp ip{};
    double *x = nullptr, *b = nullptr, *r = nullptr, *d = nullptr, *y = nullptr, *w = nullptr;
    double lmax = 0.0;
};

struct MgHierarchy {
    bool ready = false;
    tdg_mg_opts opts{};
    int fine_prec = TDG_FP64;
    int NB = 0, ncolours = 0;
    std::vector<MgLevel> lv;  // coarsest first; lv.back() is the matrix-free operator
    DevArena arena;           // operators, diagonals, interpolation, topology
    DevArena ws;              // work vectors, sized for cap right-hand sides
    int cap = 0;
    int64_t fine_ld = 0;
    int32_t* nbr = nullptr;
    int32_t* colour = nullptr;
    int* status = nullptr;
    // the coarse system the CG solves: the coarsest DG level, or (aux) the continuous P1 level
    // below it; cn unknowns per right-hand side, block-Jacobi blocks of cbs x cbs, cnb of them
    bool aux = false;
    MgAux ax{};
    double *ab = nullptr, *axv = nullptr;
    int64_t cn = 0, cnb = 0;
    int cbs = 0;
    // coarse CG: block-Jacobi inverses, vectors of cap columns, one segment (own scalars and
    // stopping test) per column, chunk plan (seg_chunk_h: its host copy)
    double* cinv = nullptr;
    double *cr = nullptr, *cz = nullptr, *cp = nullptr, *cq = nullptr;
    double* partial = nullptr;
    double* scal = nullptr;
    Chunk* chunks = nullptr;
    int* seg_chunk = nullptr;
    std::vector<int> seg_chunk_h;
    // the whole coarse CG (start, device loop of kCoarseBlock-iteration blocks) as one graph for
    // graph_nrhs columns of the right-hand side graph_b and the solution graph_x
    cudaGraphExec_t coarse_exec = nullptr;
    int graph_nrhs = 0;
    const double* graph_b = nullptr;
    const double* graph_x = nullptr;
    void reset_graph() {
        if (coarse_exec) cudaGraphExecDestroy(coarse_exec);
        coarse_exec = nullptr;
        graph_nrhs = 0;
        graph_b = graph_x = nullptr;
    }
    ~MgHierarchy() { reset_graph(); }
};

constexpr int kCoarseBlock = 8;

}  // namespace

struct tdg_op {
    HostOperator h;
    bool uploaded64 = false, uploaded32 = false;
    DevArena arena64, arena32, arena_common, arena_pc, arena_ws;
    DevOp<double> op64;
    DevOp<float> op32;
    MmaTiles mma;           // FP64 tensor-pipe apply: packed tables and signature tiles
    Tc32Tiles tc32;         // FP32 tensor-core apply (3xTF32): packed tables and signature tiles
    FaceTiles face;         // face-centric FP64 apply: facet tiles grouped by (l0, l1, mode)
    FaceTiles face32;       // face-centric FP32 apply: the same grouping with the FP32 tile size
    TileGeo tgeo;           // software-pipelined face-centric FP64 apply: tile-ordered geometry
    // explicit wave operator: basis at the volume points, reference inverse mass, -rhoInv W / |J|
    DevArena arena_wave;
    WaveData wave;
    bool wave_uploaded = false;
    bool use_mma = true;
    // per precision (0 = FP64, 1 = FP32): kernel family (0 tensor cores, 1 SIMT) and persistent CTAs
    // per SM (0 = default); set by tdg_autotune
    int family[2] = {0, 0};
    int ctas[2] = {0, 0};
    // volume points per pass of the FP64 face-centric pipelined volume kernel (0 = automatic)
    int tile[2] = {0, 0};
    const double* penalty = nullptr;
    const int4* sides = nullptr;
    // block-Jacobi
    double* blk = nullptr;
    void* inv = nullptr;
    int inv_precision = -1;
    int* status = nullptr;
    // solve workspace
    size_t ws_bytes = 0;
    void* ws = nullptr;
    // p-multigrid hierarchy and the preconditioner the solves use
    MgHierarchy mg;
    int pc = TDG_PC_BJACOBI;
    // device-looped graphs: loop counters (LoopSlot) and two non-blocking streams on which loop
    // bodies (and the stand-alone coarse-solve graph) are captured
    DevArena arena_loop;
    long long* loop = nullptr;
    cudaStream_t side[2] = {nullptr, nullptr};
    // tdg_apply_host: two device buffer pairs, copy-in / apply / copy-out streams and their events
    struct HostStream {
        cudaStream_t s[3] = {nullptr, nullptr, nullptr};
        cudaEvent_t in[2] = {}, out[2] = {}, freed[2] = {}, entry = nullptr, done[2] = {};
        void* xd[2] = {nullptr, nullptr};
        void* yd[2] = {nullptr, nullptr};
        size_t bytes = 0;
        bool ready = false;
        void release() {
            for (int b = 0; b < 2; ++b) {
                if (xd[b]) cudaFree(xd[b]);
                if (yd[b]) cudaFree(yd[b]);
                xd[b] = yd[b] = nullptr;
            }
            bytes = 0;
            if (!ready) return;
            for (int k = 0; k < 3; ++k) cudaStreamDestroy(s[k]);
            for (int b = 0; b < 2; ++b) {
                cudaEventDestroy(in[b]);
                cudaEventDestroy(out[b]);
                cudaEventDestroy(freed[b]);
                cudaEventDestroy(done[b]);
            }
            cudaEventDestroy(entry);
            ready = false;
        }
    } hs;
    ~tdg_op() {
        hs.release();
        for (cudaStream_t& q : side)
            if (q) cudaStreamDestroy(q);
    }
};

namespace {

// Loop counters and side streams of the device-looped graphs (once per operator; outside any
// capture).
int ensure_loop(tdg_op* op) {
    if (op->loop) return 0;
    for (cudaStream_t& q : op->side)
        if (!q) TDG_CUDA_TRY(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
    long long* c = nullptr;
    TDG_CUDA_TRY(op->arena_loop.alloc(&c, kLoopSlots));
    TDG_CUDA_TRY(cudaMemset(c, 0, kLoopSlots * sizeof(long long)));
    op->loop = c;
    return 0;
}

// The side stream on which the body of a loop emitted from stream s is captured.
cudaStream_t side_for(tdg_op* op, cudaStream_t s) { return s == op->side[0] ? op->side[1] : op->side[0]; }

// Emits a device loop into the graph being captured on s: start(h) launches on s what sets the
// first condition through the handle h (the loop runs while it is non-zero; it starts at `first`
// when start sets nothing), a while node follows, and body(b, h) launches one pass of the loop
// body on the side stream b, ending with a kernel that sets the next condition.  Later work on s
// follows the loop.
template <class Start, class Body>
int emit_while(tdg_op* op, cudaStream_t s, unsigned first, Start&& start, Body&& body) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    TDG_CUDA_TRY(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
    if (st != cudaStreamCaptureStatusActive) return fail(TDG_E_CUDA, "device loop outside a stream capture");
    cudaGraphConditionalHandle h{};
    TDG_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, g, first, cudaGraphCondAssignDefault));
    TDG_TRY(start(h));
    TDG_CUDA_TRY(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    TDG_CUDA_TRY(cudaGraphAddNode(&node, g, deps, nd, &p));
    TDG_CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    cudaStream_t b = side_for(op, s);
    TDG_CUDA_TRY(cudaStreamBeginCaptureToGraph(b, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
    const int rc = body(b, h);
    cudaGraph_t done = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(b, &done);
    if (rc) return rc;
    if (ce != cudaSuccess) return fail(TDG_E_CUDA, std::string("device loop body: ") + cudaGetErrorString(ce));
    return 0;
}

// True when s is capturing a graph.
bool capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    return s != nullptr && cudaStreamIsCapturing(s, &st) == cudaSuccess && st == cudaStreamCaptureStatusActive;
}

int upload_common(tdg_op* op) {
    if (op->penalty) return 0;
    auto& h = op->h;
    TDG_CUDA_TRY(op->arena_common.upload(&op->penalty, h.penalty));
    std::vector<int4> sides(h.sides.size());
    for (size_t i = 0; i < sides.size(); ++i) {
        auto const& s = h.sides[i];
        sides[i] = make_int4(s.fct, s.side | (s.bc << 8), s.nb, s.nb_local);
    }
    TDG_CUDA_TRY(op->arena_common.upload(&op->sides, sides));
    return 0;
}

// Tables of the FP64 tensor-pipe apply in its shared-memory layout (apply_mma.cuh): TV[m][k] with
// m = q * D + e the reference derivative e of basis k at volume point q; TF[f][m][k] the same at
// the facet points of local face f followed by the basis values.  Leading dimension mma_ld(MY).
// Tiles group elements by their neighbour-face signature (nb_local per face, 2 bits each).
void signature_tiles(HostOperator const& h, int TE, std::vector<int>& perm, std::vector<int4>& tiles);

// Face-centric apply: every facet with a flux once, grouped by (l0, l1, mode) -- mode 1 interior
// (both sides), 2 boundary Dirichlet / fault (side 0), 3 boundary with code None (side 0, the
// element as its own neighbour, as the element-centric apply treats it) -- and cut into tiles of
// at most TE facets with one key.  finfo[f] = {up0, up1, l0 | l1 << 8, mode}.
void facet_tiles(HostOperator const& h, int TE, std::vector<int4>& finfo, std::vector<int>& fids,
                 std::vector<int4>& ftiles) {
    finfo.assign(static_cast<size_t>(h.F), make_int4(0, 0, 0, 0));
    std::vector<int> fkey(static_cast<size_t>(h.F), 0);
    fids.clear();
    for (int64_t f = 0; f < h.F; ++f) {
        int64_t up0 = h.up[2 * f], up1 = h.up[2 * f + 1];
        int l0 = h.loc[2 * f], l1 = h.loc[2 * f + 1];
        const int bc = h.bc[f];
        const bool interior = up0 != up1;
        int mode;
        if (interior) {
            mode = (bc == 0 || bc == 3 || bc == 5) ? 1 : 0;
        } else {
            mode = (bc == 3 || bc == 5) ? 2 : (bc == 0 ? 3 : 0);
            up1 = up0;
            l1 = l0;
        }
        finfo[f] = make_int4(static_cast<int>(up0), static_cast<int>(up1), l0 | (l1 << 8), mode);
        if (mode) {
            fkey[f] = l0 | (l1 << 2) | (mode << 4);
            fids.push_back(static_cast<int>(f));
        }
    }
    std::stable_sort(fids.begin(), fids.end(), [&](int a, int b) { return fkey[a] < fkey[b]; });
    ftiles.clear();
    for (size_t i = 0; i < fids.size();) {
        size_t j = i;
        while (j < fids.size() && static_cast<int>(j - i) < TE && fkey[fids[j]] == fkey[fids[i]]) ++j;
        ftiles.push_back(make_int4(static_cast<int>(i), static_cast<int>(j - i), fkey[fids[i]], 0));
        i = j;
    }
}

// The face2 facet kernel's geometry rows (see face2_point_swizzle): quads of points with the middle
// two swapped, rows per field rounded up to the quad, for 8-facet tiles.
inline bool face2_swizzle_host(int D, int N, int Q) { return mma_tile_elements(D, N, Q) == 8; }
inline int face2_geo_rows_host(int D, int N, int Q, int nq) { return face2_swizzle_host(D, N, Q) ? (nq + 3) / 4 * 4 : nq; }

// The facet tiles' geometry [tile][field][nq][TE] (n, n_unit, then Poisson K G0, K G1 or
// elasticity G0, G1, lam0, mu0, lam1, mu1; unused slots zero), the penalty [tile][TE] and the facet
// and element ids of every slot {facet, side-0 element, side-1 element (-1 unless mode 1), 0}.
template <typename T>
void tile_facet_geometry(HostOperator const& h, int TE, std::vector<int> const& fids, std::vector<int4> const& ftiles,
                         std::vector<T>& fct, std::vector<double>& pen, std::vector<int4>& tids, int rows = 0,
                         bool swizzle = false) {
    // rows per field (>= nq, zero past nq); point q at row q, or at row face2_point(q) (an involution)
    const int D = h.D, DD = D * D, nq = rows > 0 ? rows : h.nq, nqh = h.nq;
    const bool poisson = h.kind == 0;
    const int ff = 2 * D + 2 * DD + (poisson ? 0 : 4);
    const size_t nft = ftiles.size();
    fct.assign(nft * ff * nq * TE, T(0));
    pen.assign(nft * TE, 0.0);
    tids.assign(nft * TE, make_int4(-1, -1, -1, 0));
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < static_cast<int64_t>(nft); ++t) {
        const int4 td = ftiles[t];
        const bool two = (td.z >> 4) == 1;
        T* base = &fct[static_cast<size_t>(t) * ff * nq * TE];
        for (int te = 0; te < td.y; ++te) {
            const int64_t f = fids[td.x + te];
            auto put = [&](int field, int q, double v) {
                const int row = swizzle ? face2_point(q) : q;
                base[(static_cast<size_t>(field) * nq + row) * TE + te] = static_cast<T>(v);
            };
            for (int q = 0; q < nqh; ++q) {
                for (int i = 0; i < D; ++i) {
                    put(i, q, h.fN[(static_cast<size_t>(f) * D + i) * nqh + q]);
                    put(D + i, q, h.fNunit[(static_cast<size_t>(f) * D + i) * nqh + q]);
                }
                if (poisson) {
                    for (int side = 0; side < 2; ++side)
                        for (int c = 0; c < DD; ++c)
                            put(2 * D + side * DD + c, q, h.fCoef[((static_cast<size_t>(f) * 2 + side) * DD + c) * nqh + q]);
                } else {
                    for (int c = 0; c < DD; ++c) {
                        put(2 * D + c, q, h.fG0[(static_cast<size_t>(f) * DD + c) * nqh + q]);
                        put(2 * D + DD + c, q, h.fG1[(static_cast<size_t>(f) * DD + c) * nqh + q]);
                    }
                    for (int c = 0; c < 4; ++c) put(2 * D + 2 * DD + c, q, h.fCoef[(static_cast<size_t>(f) * 4 + c) * nqh + q]);
                }
            }
            pen[static_cast<size_t>(t) * TE + te] = h.penalty[f];
            tids[static_cast<size_t>(t) * TE + te] = make_int4(static_cast<int>(f), static_cast<int>(h.up[2 * f]),
                                                                two ? static_cast<int>(h.up[2 * f + 1]) : -1, 0);
        }
    }
}

// Geometry and coefficients of the software-pipelined face-centric apply (apply_face2.cuh) in tile
// order: per element tile of TE consecutive elements [field][Nq rows][TE] (J^-1, then the volume
// coefficients), per facet tile [field][nq rows][TE] (n, n_unit, then Poisson K G0, K G1 or
// elasticity G0, G1, lam0, mu0, lam1, mu1) and the penalty [TE]; unused slots and padding rows
// zero; 8-wide tiles hold point q in row face2_point(q) of nq rounded up to 4 rows.  The same values
// as the reference-layout arrays, read with the tile's elements or facets fastest.
int upload_tile_geometry(tdg_op* op, DevArena& arena, std::vector<int> const& fids, std::vector<int4> const& ftiles) {
    auto const& h = op->h;
    const int D = h.D, DD = D * D, Nq = h.Nq;
    const int TE = mma_tile_elements(D, h.N, h.Q);
    const bool poisson = h.kind == 0;
    const int ncoef = poisson ? 1 : 2;
    const int vf = DD + ncoef;
    const int64_t vtiles = (h.E + TE - 1) / TE;
    // rows per field and the row of point q (the volume kernel's point swizzle)
    const bool swz = face2_swizzle_host(D, h.N, h.Q);
    const int Nqg = face2_geo_rows_host(D, h.N, h.Q, Nq);
    std::vector<double> vol(static_cast<size_t>(vtiles) * vf * Nqg * TE, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < h.E; ++e) {
        const int64_t t = e / TE;
        const int te = static_cast<int>(e % TE);
        double* base = &vol[static_cast<size_t>(t) * vf * Nqg * TE];
        for (int c = 0; c < DD; ++c)
            for (int q = 0; q < Nq; ++q)
                base[(static_cast<size_t>(c) * Nqg + (swz ? face2_point(q) : q)) * TE + te] =
                    h.vG[(static_cast<size_t>(e) * DD + c) * Nq + q];
        for (int c = 0; c < ncoef; ++c)
            for (int q = 0; q < Nq; ++q)
                base[(static_cast<size_t>(DD + c) * Nqg + (swz ? face2_point(q) : q)) * TE + te] =
                    h.vCoef[(static_cast<size_t>(e) * ncoef + c) * Nq + q];
    }
    const size_t nft = ftiles.size();
    std::vector<double> fct, pen;
    std::vector<int4> tids;
    tile_facet_geometry(h, TE, fids, ftiles, fct, pen, tids, face2_geo_rows_host(h.D, h.N, h.Q, h.nq),
                        face2_swizzle_host(h.D, h.N, h.Q));
    if (nft) TDG_CUDA_TRY(arena.upload(&op->face.tids, tids));
    {
        const int* st = nullptr;
        TDG_CUDA_TRY(arena.upload(&st, std::vector<int>(1, 0)));
        op->tgeo.status = const_cast<int*>(st);
    }
    TDG_CUDA_TRY(arena.upload(&op->tgeo.vol, vol));
    if (nft) {
        TDG_CUDA_TRY(arena.upload(&op->tgeo.fct, fct));
        TDG_CUDA_TRY(arena.upload(&op->tgeo.pen, pen));
    }
    return 0;
}

int upload_mma(tdg_op* op, DevArena& arena) {
    auto const& h = op->h;
    const int D = h.D, NBF = h.Nbf, Nq = h.Nq, nq = h.nq, NF = h.nfaces;
    const int KP = (NBF + 3) / 4 * 4, LDT = mma_ld(KP);
    const int MV = round8(D * Nq), MF = round8((D + 1) * nq);
    std::vector<double> tab(static_cast<size_t>(MV) * LDT + static_cast<size_t>(NF) * MF * LDT, 0.0);
    for (int q = 0; q < Nq; ++q)
        for (int e = 0; e < D; ++e)
            for (int k = 0; k < NBF; ++k)
                tab[static_cast<size_t>(q * D + e) * LDT + k] = h.Dxi_Q[(static_cast<size_t>(k) * D + e) * Nq + q];
    for (int f = 0; f < NF; ++f) {
        double* T = &tab[static_cast<size_t>(MV) * LDT + static_cast<size_t>(f) * MF * LDT];
        for (int q = 0; q < nq; ++q)
            for (int k = 0; k < NBF; ++k) {
                for (int e = 0; e < D; ++e)
                    T[static_cast<size_t>(q * D + e) * LDT + k] = h.Dxi_qf[f][(static_cast<size_t>(k) * D + e) * nq + q];
                T[static_cast<size_t>(D * nq + q) * LDT + k] = h.E_qf[f](k, q);
            }
    }
    std::vector<int> perm;
    std::vector<int4> tiles;
    signature_tiles(h, mma_tile_elements(h.D, h.N, h.Q), perm, tiles);
    TDG_CUDA_TRY(arena.upload(&op->mma.tables, tab));
    TDG_CUDA_TRY(arena.upload(&op->mma.perm, perm));
    TDG_CUDA_TRY(arena.upload(&op->mma.tiles, tiles));
    op->mma.ntiles = static_cast<int>(tiles.size());
    op->mma.table_doubles = static_cast<int>(tab.size());

    std::vector<int4> finfo, ftiles;
    std::vector<int> fids;
    facet_tiles(h, mma_tile_elements(D, h.N, h.Q), finfo, fids, ftiles);
    if (!fids.empty()) {
        TDG_CUDA_TRY(arena.upload(&op->face.fperm, fids));
        TDG_CUDA_TRY(arena.upload(&op->face.ftiles, ftiles));
    }
    TDG_CUDA_TRY(arena.upload(&op->face.finfo, finfo));
    op->face.nftiles = static_cast<int>(ftiles.size());
    op->face.tables = op->mma.tables + static_cast<size_t>(MV) * LDT;
    TDG_TRY(upload_tile_geometry(op, arena, fids, ftiles));
    return 0;
}

// Elements grouped by the local face numbers their neighbours see them through (2 bits per
// face), cut into tiles of at most TE elements with one signature each.
void signature_tiles(HostOperator const& h, int TE, std::vector<int>& perm, std::vector<int4>& tiles) {
    const int NF = h.nfaces;
    std::vector<int> sig(h.E);
    perm.resize(h.E);
    for (int64_t e = 0; e < h.E; ++e) {
        int sg = 0;
        for (int f = 0; f < NF; ++f) sg |= (h.sides[static_cast<size_t>(e) * NF + f].nb_local & 3) << (2 * f);
        sig[e] = sg;
        perm[e] = static_cast<int>(e);
    }
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return sig[a] < sig[b]; });
    tiles.clear();
    for (int64_t i = 0; i < h.E;) {
        int64_t j = i;
        while (j < h.E && j - i < TE && sig[perm[j]] == sig[perm[i]]) ++j;
        tiles.push_back(make_int4(static_cast<int>(i), static_cast<int>(j - i), sig[perm[i]], 0));
        i = j;
    }
}

// FP32 tensor-core apply: tables as in apply_tc32.cuh (K padded to 8, ld = K + 4, rows padded to
// 16) and signature tiles of tc32_tile_elements elements.
int upload_tc32(tdg_op* op, DevArena& arena) {
    auto const& h = op->h;
    const int D = h.D, NBF = h.Nbf, Nq = h.Nq, nq = h.nq, NF = h.nfaces;
    const int KP = tc_round(NBF, 8), LDT = KP + 4;
    const int MV = tc_round(D * Nq, 16), MF = tc_round((D + 1) * nq, 16);
    std::vector<float> tab(static_cast<size_t>(MV) * LDT + static_cast<size_t>(NF) * MF * LDT, 0.0f);
    for (int q = 0; q < Nq; ++q)
        for (int e = 0; e < D; ++e)
            for (int k = 0; k < NBF; ++k)
                tab[static_cast<size_t>(q * D + e) * LDT + k] =
                    static_cast<float>(h.Dxi_Q[(static_cast<size_t>(k) * D + e) * Nq + q]);
    for (int f = 0; f < NF; ++f) {
        float* T = &tab[static_cast<size_t>(MV) * LDT + static_cast<size_t>(f) * MF * LDT];
        for (int q = 0; q < nq; ++q)
            for (int k = 0; k < NBF; ++k) {
                for (int e = 0; e < D; ++e)
                    T[static_cast<size_t>(q * D + e) * LDT + k] =
                        static_cast<float>(h.Dxi_qf[f][(static_cast<size_t>(k) * D + e) * nq + q]);
                T[static_cast<size_t>(D * nq + q) * LDT + k] = static_cast<float>(h.E_qf[f](k, q));
            }
    }
    std::vector<int> perm;
    std::vector<int4> tiles;
    signature_tiles(h, tc32_tile_elements(D, h.Q), perm, tiles);
    TDG_CUDA_TRY(arena.upload(&op->tc32.tables, tab));
    TDG_CUDA_TRY(arena.upload(&op->tc32.perm, perm));
    TDG_CUDA_TRY(arena.upload(&op->tc32.tiles, tiles));
    op->tc32.ntiles = static_cast<int>(tiles.size());
    op->tc32.table_floats = static_cast<int>(tab.size());
    {
        const int* st = nullptr;
        TDG_CUDA_TRY(arena.upload(&st, std::vector<int>(1, 0)));
        op->tc32.status = const_cast<int*>(st);
    }
    {
        std::vector<int4> finfo, ftiles;
        std::vector<int> fids;
        facet_tiles(h, tc32_tile_elements(D, h.Q), finfo, fids, ftiles);
        if (!fids.empty()) {
            TDG_CUDA_TRY(arena.upload(&op->face32.fperm, fids));
            TDG_CUDA_TRY(arena.upload(&op->face32.ftiles, ftiles));
        }
        TDG_CUDA_TRY(arena.upload(&op->face32.finfo, finfo));
        op->face32.nftiles = static_cast<int>(ftiles.size());
        std::vector<float> fct;
        std::vector<double> pen;
        std::vector<int4> tids;
        // the FP32 facet kernel's point swizzle (kTc32PointSwizzle): 3D elasticity, 16-facet tiles
        const bool swz = D == 3 && h.kind == 1 && tc32_tile_elements(D, h.Q) == 16;
        tile_facet_geometry(h, tc32_tile_elements(D, h.Q), fids, ftiles, fct, pen, tids, swz ? (nq + 3) / 4 * 4 : nq,
                            swz);
        if (!ftiles.empty()) {
            TDG_CUDA_TRY(arena.upload(&op->face32.tids, tids));
            TDG_CUDA_TRY(arena.upload(&op->face32.geo, fct));
            TDG_CUDA_TRY(arena.upload(&op->face32.pen, pen));
        }
    }
    return 0;
}

template <typename T>
int upload_precision(tdg_op* op, DevArena& arena, DevOp<T>& d) {
    auto& h = op->h;
    const int D = h.D, NBF = h.Nbf, Nq = h.Nq, nq = h.nq, NF = h.nfaces;
    TDG_TRY(upload_common(op));
    d.E = h.E;
    d.F = h.F;
    d.Nq = Nq;
    d.nq = nq;
    // basis tables and their transposes
    std::vector<T> Dxi(h.Dxi_Q.begin(), h.Dxi_Q.end()), DxiT(static_cast<size_t>(NBF) * D * Nq);
    for (int k = 0; k < NBF; ++k)
        for (int c = 0; c < D * Nq; ++c) DxiT[static_cast<size_t>(c) * NBF + k] = Dxi[static_cast<size_t>(k) * D * Nq + c];
    std::vector<T> Eq, ETq, Dq, DTq;
    for (int f = 0; f < NF; ++f) {
        for (int k = 0; k < NBF; ++k)
            for (int q = 0; q < nq; ++q) Eq.push_back(static_cast<T>(h.E_qf[f](k, q)));
        for (int q = 0; q < nq; ++q)
            for (int k = 0; k < NBF; ++k) ETq.push_back(static_cast<T>(h.E_qf[f](k, q)));
        auto const& g = h.Dxi_qf[f];
        for (size_t i = 0; i < g.size(); ++i) Dq.push_back(static_cast<T>(g[i]));
        std::vector<T> t(static_cast<size_t>(D) * nq * NBF);
        for (int k = 0; k < NBF; ++k)
            for (int c = 0; c < D * nq; ++c) t[static_cast<size_t>(c) * NBF + k] = static_cast<T>(g[static_cast<size_t>(k) * D * nq + c]);
        DTq.insert(DTq.end(), t.begin(), t.end());
    }
    TDG_CUDA_TRY(arena.upload(&d.Dxi_Q, Dxi));
    TDG_CUDA_TRY(arena.upload(&d.DxiT_Q, DxiT));
    TDG_CUDA_TRY(arena.upload(&d.E_q, Eq));
    TDG_CUDA_TRY(arena.upload(&d.ET_q, ETq));
    TDG_CUDA_TRY(arena.upload(&d.Dxi_q, Dq));
    TDG_CUDA_TRY(arena.upload(&d.DxiT_q, DTq));
    TDG_CUDA_TRY(arena.upload(&d.w, conv<T>(h.w)));
    TDG_CUDA_TRY(arena.upload(&d.vG, conv<T>(h.vG)));
    TDG_CUDA_TRY(arena.upload(&d.vCoef, conv<T>(h.vCoef)));
    TDG_CUDA_TRY(arena.upload(&d.fN, conv<T>(h.fN)));
    TDG_CUDA_TRY(arena.upload(&d.fNunit, conv<T>(h.fNunit)));
    TDG_CUDA_TRY(arena.upload(&d.fNl, conv<T>(h.fNl)));
    TDG_CUDA_TRY(arena.upload(&d.fCoef, conv<T>(h.fCoef)));
    {
        // [F][2][DD][nq]: G0 and G1 interleaved per facet
        const size_t per = static_cast<size_t>(D) * D * nq;
        std::vector<T> fg(static_cast<size_t>(h.F) * 2 * per);
        for (int64_t f = 0; f < h.F; ++f)
            for (size_t i = 0; i < per; ++i) {
                fg[(static_cast<size_t>(f) * 2 + 0) * per + i] = static_cast<T>(h.fG0[static_cast<size_t>(f) * per + i]);
                fg[(static_cast<size_t>(f) * 2 + 1) * per + i] = static_cast<T>(h.fG1[static_cast<size_t>(f) * per + i]);
            }
        TDG_CUDA_TRY(arena.upload(&d.fG, fg));
    }
    d.penalty = op->penalty;
    d.sides = op->sides;
    if constexpr (std::is_same_v<T, double>) TDG_TRY(upload_mma(op, arena));
    if constexpr (std::is_same_v<T, float>) TDG_TRY(upload_tc32(op, arena));
    TDG_CUDA_TRY(cudaDeviceSynchronize());
    return 0;
}

int ensure_uploaded(tdg_op* op, int precision) {
    if (!op->h.has_material) return fail(TDG_E_STATE, "tdg_set_material has not been called");
    if (precision == TDG_FP64) {
        if (!op->uploaded64) {
            TDG_TRY(upload_precision<double>(op, op->arena64, op->op64));
            op->uploaded64 = true;
            // the allocation-free gradient entry point of elasticity operators reads these data:
            // resolve its fixed scratch and load its kernel now, while allocating is allowed (a
            // failure here is reported by that entry point when it repeats the lookup)
            if (op->h.kind == 1 && adjoint_prepare(op->h.D, op->h.N)) cudaGetLastError();
        }
        return 0;
    }
    if (precision == TDG_FP32 || precision == TDG_MIXED || precision == TDG_TF32) {
        if (!op->uploaded32) {
            TDG_TRY(upload_precision<float>(op, op->arena32, op->op32));
            op->uploaded32 = true;
        }
        return 0;
    }
    return fail(TDG_E_INVALID, "precision must be TDG_FP64 or TDG_FP32");
}

// A solve over the owned rows of one rank of a distributed operator (tdg_solve_distributed):
// before every apply the caller's exchange fills the ghost blocks of the apply's input, and every
// dot product's per-rank sum is summed over the ranks by the caller's all-reduce, both enqueued on
// the solve's stream.
struct DistCtx {
    tdg_exchange_fn exchange = nullptr;
    tdg_allreduce_fn allreduce = nullptr;
    void* ctx = nullptr;
};

// Chunk list of a segmented vector (see krylov.cuh), uploaded into solve workspace.
struct SegPlan {
    int nseg = 0, nchunks = 0;
    const Chunk* chunks = nullptr;   // device [nchunks]
    const int* seg_chunk = nullptr;  // device [nseg + 1]
    // operator view of the stacked vectors: apply / precondition with nrhs and leading dimension
    int op_nrhs = 1;
    int64_t op_ld = 0;
    const DistCtx* dist = nullptr;  // distributed solve (one segment: the owned rows), else null
};

// Chunk length: about four chunks per SM over all segments (so short vectors still occupy the
// whole GPU), a multiple of the CTA size, between kChunkMin and kChunk entries.
void plan_chunks(std::vector<int64_t> const& seg_begin, std::vector<int64_t> const& seg_end, std::vector<Chunk>& chunks,
                 std::vector<int>& seg_chunk) {
    int64_t total = 0;
    for (size_t sgi = 0; sgi < seg_begin.size(); ++sgi) total += seg_end[sgi] - seg_begin[sgi];
    const int64_t target = (total / (4 * static_cast<int64_t>(device_sm_count())) + kVecThreads - 1) / kVecThreads * kVecThreads;
    const int64_t len = std::max<int64_t>(kChunkMin, std::min<int64_t>(kChunk, target));
    chunks.clear();
    seg_chunk.assign(1, 0);
    for (size_t sgi = 0; sgi < seg_begin.size(); ++sgi) {
        for (int64_t b = seg_begin[sgi]; b < seg_end[sgi]; b += len) {
            Chunk c;
            c.begin = b;
            c.end = std::min(seg_end[sgi], b + len);
            c.seg = static_cast<int>(sgi);
            c.pad = 0;
            chunks.push_back(c);
        }
        seg_chunk.push_back(static_cast<int>(chunks.size()));
    }
}

// scal[seg][slot0] = a.b, scal[seg][slot1] = c.d
template <typename T>
int dots(SegPlan const& sp, const T* a, const T* b, const T* c, const T* d, double* partial, double* scal, int slot0,
         int slot1, cudaStream_t s) {
    k_dot2<T><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, a, b, c, d, partial);
    k_dot_finalize<<<sp.nseg, 256, 0, s>>>(partial, sp.seg_chunk, scal, slot0, slot1);
    if (cudaGetLastError() != cudaSuccess) return fail(TDG_E_CUDA, "dot kernels");
    if (sp.dist) {  // one segment: sum the slots over the ranks (adjacent slots in one call)
        const bool pair = slot0 >= 0 && slot1 == slot0 + 1;
        for (int slot : {slot0, slot1}) {
            if (slot < 0 || (pair && slot == slot1)) continue;
            if (sp.dist->allreduce(sp.dist->ctx, scal + slot, pair ? 2 : 1, s) != 0)
                return fail(TDG_E_STATE, "the all-reduce callback of the distributed solve failed");
        }
    }
    return 0;
}

// The apply of the Krylov drivers: y = A x, with the ghost exchange of x in front for a
// distributed solve.
int krylov_apply(tdg_op* op, int prec, SegPlan const& sp, void* x, void* y, cudaStream_t s) {
    if (sp.dist && sp.dist->exchange(sp.dist->ctx, static_cast<double*>(x), s) != 0)
        return fail(TDG_E_STATE, "the exchange callback of the distributed solve failed");
    return tdg_apply(op, prec, x, y, sp.op_nrhs, sp.op_ld, s);
}

// ---- block-Jacobi diagonal blocks ---------------------------------------------------------------

// Assembles the element diagonal blocks once (block Jacobi, and the point-Jacobi diagonal of the
// finest multigrid level).
int ensure_blocks(tdg_op* op, cudaStream_t s) {
    if (op->blk) return 0;
    TDG_TRY(ensure_uploaded(op, TDG_FP64));
    auto const& h = op->h;
    TDG_CUDA_TRY(op->arena_pc.alloc(&op->blk, static_cast<size_t>(h.E) * h.bs * h.bs));
    TDG_CUDA_TRY(op->arena_pc.alloc(&op->status, 1));
    int rc = launch_bjac_assemble(h.D, h.N, h.kind, op->op64, op->blk, s);
    if (rc) {
        op->blk = nullptr;
        return fail(rc, "block assembly launch failed");
    }
    return 0;
}

// ---- p-multigrid (PCMG with Chebyshev / point-Jacobi smoothing) ---------------------------------

int mgk(int rc, const char* what) { return rc ? fail(rc, std::string("multigrid: ") + what) : 0; }

// y = A_l x, or y = b - A_l x when b != nullptr, for nrhs columns at the level's stride.
int mg_level_apply(tdg_op* op, int l, const double* x, double* y, const double* b, int nrhs, cudaStream_t s) {
    auto& mg = op->mg;
    auto const& L = mg.lv[static_cast<size_t>(l)];
    if (l + 1 == static_cast<int>(mg.lv.size())) {
        TDG_TRY(tdg_apply(op, mg.fine_prec, x, y, nrhs, L.ld, s));
        if (b) TDG_TRY(mgk(launch_vec_rsub_cols(L.n, nrhs, L.ld, b, y, s), "residual"));
        return 0;
    }
    if (L.A32) return mgk(launch_mg_bsr_apply(op->h.E, mg.NB, L.bs, mg.nbr, L.A32, x, b, y, nrhs, L.ld, s), "level apply");
    return mgk(launch_mg_bsr_apply(op->h.E, mg.NB, L.bs, mg.nbr, L.A, x, b, y, nrhs, L.ld, s), "level apply");
}

// Chebyshev smoothing of A_l x = b on [esteig_lo, esteig_hi] x lambda_max(D^-1 A_l), smooth_its
// steps (Saad, Alg. 12.1, with the point-Jacobi preconditioner), from x = 0 or from the given x.
int mg_smooth(tdg_op* op, int l, const double* b, double* x, bool x_zero, int nrhs, cudaStream_t s) {
    auto& mg = op->mg;
    auto& L = mg.lv[static_cast<size_t>(l)];
    const double emax = mg.opts.esteig_hi * L.lmax, emin = mg.opts.esteig_lo * L.lmax;
    const double theta = 0.5 * (emax + emin), delta = 0.5 * (emax - emin), sigma = theta / delta;
    double rho = 1.0 / sigma;
    if (x_zero)
        TDG_TRY(mgk(launch_vec_copy_cols(L.n, nrhs, L.ld, b, L.r, s), "copy"));
    else
        TDG_TRY(mg_level_apply(op, l, x, L.r, b, nrhs, s));
    TDG_TRY(mgk(launch_cheb_first(L.n, nrhs, L.ld, L.dinv, L.r, L.d, x, 1.0 / theta, x_zero ? 1 : 0, s), "Chebyshev"));
    for (int k = 1; k < mg.opts.smooth_its; ++k) {
        TDG_TRY(mg_level_apply(op, l, L.d, L.y, nullptr, nrhs, s));
        const double rho1 = 1.0 / (2.0 * sigma - rho);
        TDG_TRY(mgk(launch_cheb_step(L.n, nrhs, L.ld, L.dinv, L.y, L.r, L.d, x, rho1 * rho, 2.0 * rho1 / delta, s),
                    "Chebyshev"));
        rho = rho1;
    }
    return 0;
}

// kCoarseBlock CG iterations of the coarse system with device-resident scalars, nrhs columns.
int mg_coarse_block(tdg_op* op, SegPlan const& sp, double* x, int nrhs, cudaStream_t s) {
    auto& mg = op->mg;
    auto const& L = mg.lv[0];
    for (int k = 0; k < kCoarseBlock; ++k) {
        if (mg.aux)
            TDG_TRY(mgk(launch_aux_apply(mg.ax, mg.cp, nullptr, mg.cq, nrhs, s), "coarse A"));
        else
            TDG_TRY(mgk(launch_mg_bsr_apply(op->h.E, mg.NB, L.bs, mg.nbr, L.A, mg.cp, nullptr, mg.cq, nrhs, mg.cn, s),
                        "coarse A"));
        TDG_TRY(dots<double>(sp, mg.cp, mg.cq, nullptr, nullptr, mg.partial, mg.scal, kPQ, -1, s));
        k_cg_xr<double><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, x, mg.cr, mg.cp, mg.cq, mg.scal);
        TDG_TRY(mgk(launch_bjac_apply<double, double>(mg.cbs, mg.cnb, mg.cinv, mg.cr, mg.cz, nrhs, mg.cn, s),
                    "coarse PC"));
        TDG_TRY(dots<double>(sp, mg.cr, mg.cz, mg.cr, mg.cr, mg.partial, mg.scal, kRZnew, kRR, s));
        k_cg_p<double><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, mg.cp, mg.cz, mg.scal);
        k_cg_shift<<<(nrhs + 127) / 128, 128, 0, s>>>(mg.scal, nrhs);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : fail(TDG_E_CUDA, "multigrid: coarse CG kernels");
}

// Coarse solve of nrhs columns (contiguous, cn entries each): CG with the block-Jacobi inverses
// from x = 0, one segment per column, until every column has ||r|| <= coarse_rtol ||b|| (checked
// on the device every kCoarseBlock iterations) or coarse_max_it iterations.  The whole solve is a
// device loop (emit_while) with no host synchronisation: emitted into the caller's capture when s
// is capturing (a V-cycle inside a graph-captured Krylov block), else captured once per (nrhs, b,
// x) as a graph of its own and launched on s.  A column whose residual is not finite stops and
// raises the loop counter kCoarseDiverged, which the solve drivers and tdg_mg_apply read.  x is
// always the coarse system's own vector (the coarsest DG level's, or the continuous P1 level's).
int mg_coarse_emit(tdg_op* op, const double* b, double* x, int nrhs, cudaStream_t s) {
    auto& mg = op->mg;
    SegPlan sp;
    sp.nseg = nrhs;
    sp.nchunks = mg.seg_chunk_h[static_cast<size_t>(nrhs)];
    sp.chunks = mg.chunks;
    sp.seg_chunk = mg.seg_chunk;
    sp.op_nrhs = nrhs;
    sp.op_ld = mg.cn;
    const size_t nc = static_cast<size_t>(mg.cn) * nrhs;
    long long* ctl = op->loop;
    const double rtol2 = mg.opts.coarse_rtol * mg.opts.coarse_rtol;
    const int max_it = mg.opts.coarse_max_it;
    TDG_CUDA_TRY(cudaMemsetAsync(x, 0, nc * sizeof(double), s));
    TDG_CUDA_TRY(cudaMemcpyAsync(mg.cr, b, nc * sizeof(double), cudaMemcpyDeviceToDevice, s));
    TDG_CUDA_TRY(cudaMemsetAsync(mg.scal, 0, static_cast<size_t>(nrhs) * kScal * sizeof(double), s));
    TDG_TRY(mgk(launch_bjac_apply<double, double>(mg.cbs, mg.cnb, mg.cinv, mg.cr, mg.cz, nrhs, mg.cn, s), "coarse PC"));
    k_copy<double><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, mg.cz, mg.cp);
    TDG_TRY(dots<double>(sp, mg.cr, mg.cz, mg.cr, mg.cr, mg.partial, mg.scal, kRZ, kRR, s));
    auto start = [&](cudaGraphConditionalHandle h) {
        k_coarse_ctl<<<1, 256, 0, s>>>(mg.scal, nrhs, rtol2, ctl, max_it, kCoarseBlock, 0, h);
        return cudaGetLastError() == cudaSuccess ? 0 : fail(TDG_E_CUDA, "multigrid: coarse CG control");
    };
    auto body = [&](cudaStream_t bs, cudaGraphConditionalHandle h) {
        TDG_TRY(mg_coarse_block(op, sp, x, nrhs, bs));
        k_coarse_ctl<<<1, 256, 0, bs>>>(mg.scal, nrhs, rtol2, ctl, max_it, kCoarseBlock, 1, h);
        return cudaGetLastError() == cudaSuccess ? 0 : fail(TDG_E_CUDA, "multigrid: coarse CG control");
    };
    TDG_TRY(emit_while(op, s, 0u, start, body));
    k_coarse_ctl<<<1, 32, 0, s>>>(mg.scal, nrhs, rtol2, ctl, max_it, kCoarseBlock, 2, cudaGraphConditionalHandle{});
    return cudaGetLastError() == cudaSuccess ? 0 : fail(TDG_E_CUDA, "multigrid: coarse CG control");
}

int mg_coarse_solve(tdg_op* op, const double* b, double* x, int nrhs, cudaStream_t s) {
    auto& mg = op->mg;
    if (capturing(s)) return mg_coarse_emit(op, b, x, nrhs, s);
    TDG_TRY(ensure_loop(op));
    if (!mg.coarse_exec || mg.graph_nrhs != nrhs || mg.graph_b != b || mg.graph_x != x) {
        mg.reset_graph();
        cudaStream_t cs = op->side[0];
        cudaGraph_t graph = nullptr;
        TDG_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        const int rc = mg_coarse_emit(op, b, x, nrhs, cs);
        const cudaError_t ce = cudaStreamEndCapture(cs, &graph);
        cudaError_t ci = cudaSuccess;
        if (rc == 0 && ce == cudaSuccess) ci = cudaGraphInstantiate(&mg.coarse_exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (rc) return rc;
        if (ce != cudaSuccess || ci != cudaSuccess) {
            mg.coarse_exec = nullptr;
            return fail(TDG_E_CUDA, std::string("multigrid: coarse CG graph: ") +
                                        cudaGetErrorString(ce != cudaSuccess ? ce : ci));
        }
        mg.graph_nrhs = nrhs;
        mg.graph_b = b;
        mg.graph_x = x;
    }
    TDG_CUDA_TRY(cudaGraphLaunch(mg.coarse_exec, s));
    return 0;
}

// Reads and clears the coarse CG's divergence flag (synchronises s).
int mg_check_coarse(tdg_op* op, cudaStream_t s) {
    if (!op->loop) return 0;
    long long flag = 0;
    TDG_CUDA_TRY(cudaMemcpyAsync(&flag, op->loop + kCoarseDiverged, sizeof flag, cudaMemcpyDeviceToHost, s));
    TDG_CUDA_TRY(cudaStreamSynchronize(s));
    if (!flag) return 0;
    TDG_CUDA_TRY(cudaMemsetAsync(op->loop + kCoarseDiverged, 0, sizeof flag, s));
    return fail(TDG_E_DIVERGED, "multigrid: coarse CG diverged");
}

// One V-cycle on level l for nrhs columns: x = M_l b.  Below the coarsest DG level sits either the
// coarse solve itself or, with the auxiliary space, a smoothed DG level corrected from the
// continuous P1 level.
int mg_vcycle(tdg_op* op, int l, const double* b, double* x, int nrhs, cudaStream_t s) {
    auto& mg = op->mg;
    if (l == 0 && !mg.aux) return mg_coarse_solve(op, b, x, nrhs, s);
    auto& L = mg.lv[static_cast<size_t>(l)];
    const int64_t E = op->h.E;
    TDG_TRY(mg_smooth(op, l, b, x, true, nrhs, s));
    TDG_TRY(mg_level_apply(op, l, x, L.r, b, nrhs, s));
    if (l == 0) {
        TDG_TRY(mgk(launch_aux_restrict(mg.ax, L.r, L.ld, mg.ab, nrhs, s), "restriction to P1"));
        TDG_TRY(mg_coarse_solve(op, mg.ab, mg.axv, nrhs, s));
        TDG_TRY(mgk(launch_aux_prolong_add(mg.ax, E, mg.axv, x, L.ld, nrhs, s), "prolongation from P1"));
    } else {
        auto& C = mg.lv[static_cast<size_t>(l - 1)];
        TDG_TRY(mgk(launch_mg_restrict(E, C.ip, L.r, L.ld, C.b, C.ld, nrhs, s), "restriction"));
        TDG_TRY(mg_vcycle(op, l - 1, C.b, C.x, nrhs, s));
        TDG_TRY(mgk(launch_mg_prolong_add(E, C.ip, C.x, C.ld, x, L.ld, nrhs, s), "prolongation"));
    }
    return mg_smooth(op, l, b, x, false, nrhs, s);
}

// Work vectors for nrhs right-hand sides with the finest level's leading dimension ld (grown on
// demand; reallocation waits for the stream and drops the coarse CG graph).
int mg_ensure_ws(tdg_op* op, int nrhs, int64_t ld, cudaStream_t s) {
    auto& mg = op->mg;
    if (nrhs <= mg.cap && ld == mg.fine_ld) return 0;
    TDG_CUDA_TRY(cudaStreamSynchronize(s));
    const int cap = std::max(nrhs, mg.cap);
    // until every vector is in place the hierarchy has no work space (a failed allocation must not
    // leave stale pointers that a later call with the same shape would reuse)
    mg.reset_graph();
    mg.ws.release();
    mg.cap = 0;
    mg.fine_ld = 0;
    const int nl = static_cast<int>(mg.lv.size());
    for (int l = 0; l < nl; ++l) {
        auto& L = mg.lv[static_cast<size_t>(l)];
        L.ld = (l + 1 == nl) ? ld : L.n;
        const size_t sz = static_cast<size_t>(cap) * static_cast<size_t>(L.ld);
        if (l + 1 < nl) {
            TDG_CUDA_TRY(mg.ws.alloc(&L.x, sz));
            TDG_CUDA_TRY(mg.ws.alloc(&L.b, sz));
        }
        for (double** v : {&L.r, &L.d, &L.y, &L.w}) TDG_CUDA_TRY(mg.ws.alloc(v, sz));
    }
    const size_t csz = static_cast<size_t>(cap) * static_cast<size_t>(mg.cn);
    for (double** v : {&mg.cr, &mg.cz, &mg.cp, &mg.cq}) TDG_CUDA_TRY(mg.ws.alloc(v, csz));
    if (mg.aux) {
        TDG_CUDA_TRY(mg.ws.alloc(&mg.ab, csz));
        TDG_CUDA_TRY(mg.ws.alloc(&mg.axv, csz));
    }
    std::vector<int64_t> sb(static_cast<size_t>(cap)), se(static_cast<size_t>(cap));
    for (int c = 0; c < cap; ++c) {
        sb[static_cast<size_t>(c)] = c * mg.cn;
        se[static_cast<size_t>(c)] = c * mg.cn + mg.cn;
    }
    std::vector<Chunk> hc;
    plan_chunks(sb, se, hc, mg.seg_chunk_h);
    const Chunk* dch = nullptr;
    const int* dsc = nullptr;
    TDG_CUDA_TRY(mg.ws.upload(&dch, hc));
    TDG_CUDA_TRY(mg.ws.upload(&dsc, mg.seg_chunk_h));
    mg.chunks = const_cast<Chunk*>(dch);
    mg.seg_chunk = const_cast<int*>(dsc);
    TDG_CUDA_TRY(mg.ws.alloc(&mg.scal, static_cast<size_t>(cap) * kScal));
    // dot partials: the level dots (kDotBlocks + a result slot) and the coarse CG's chunk pairs
    TDG_CUDA_TRY(mg.ws.alloc(&mg.partial, std::max<size_t>(kDotBlocks + 8, 2 * hc.size())));
    mg.cap = cap;
    mg.fine_ld = ld;
    return 0;
}

// Largest eigenvalue of the symmetric tridiagonal matrix (a diagonal, c off-diagonal) by Sturm
// bisection.
double tridiag_lmax(std::vector<double> const& a, std::vector<double> const& c) {
    const size_t m = a.size();
    double lo = std::numeric_limits<double>::max(), hi = -lo;
    for (size_t i = 0; i < m; ++i) {
        const double r = (i > 0 ? std::fabs(c[i - 1]) : 0.0) + (i + 1 < m ? std::fabs(c[i]) : 0.0);
        lo = std::min(lo, a[i] - r);
        hi = std::max(hi, a[i] + r);
    }
    auto count_below = [&](double x) {  // eigenvalues < x
        int cnt = 0;
        double d = 1.0;
        for (size_t i = 0; i < m; ++i) {
            d = a[i] - x - (i > 0 ? c[i - 1] * c[i - 1] / d : 0.0);
            if (d == 0.0) d = -1e-300;
            if (d < 0.0) ++cnt;
        }
        return cnt;
    };
    for (int it = 0; it < 200 && hi - lo > 1e-14 * std::max(1.0, std::fabs(hi)); ++it) {
        const double mid = 0.5 * (lo + hi);
        if (count_below(mid) >= static_cast<int>(m)) hi = mid;
        else lo = mid;
    }
    return hi;
}

// lambda_max(D^-1 A_l) from esteig_steps Jacobi-preconditioned CG (Lanczos) steps on a seeded
// random right-hand side: the Lanczos tridiagonal T has diagonal 1/alpha_k + beta_{k-1}/alpha_{k-1}
// and off-diagonal sqrt(beta_k)/alpha_k.
int mg_estimate_lmax(tdg_op* op, int l, cudaStream_t s) {
    auto& mg = op->mg;
    auto& L = mg.lv[static_cast<size_t>(l)];
    const int64_t n = L.n;
    double* r = L.r;
    double* p = L.d;
    double* q = L.y;
    double* z = L.w;
    double* dsc = mg.partial + kDotBlocks;
    auto dot = [&](const double* a, const double* b, double* out) -> int {
        TDG_TRY(mgk(launch_vec_dot(n, a, b, mg.partial, dsc, s), "dot"));
        TDG_CUDA_TRY(cudaMemcpyAsync(out, dsc, sizeof(double), cudaMemcpyDeviceToHost, s));
        TDG_CUDA_TRY(cudaStreamSynchronize(s));
        return 0;
    };
    TDG_TRY(mgk(launch_vec_random(n, 0x7a6d3c1b5e9f2d41ull + static_cast<uint64_t>(l), r, s), "random"));
    TDG_TRY(mgk(launch_vec_mul(n, L.dinv, r, z, s), "jacobi"));
    TDG_TRY(mgk(launch_vec_axpby(n, 1.0, z, 0.0, p, s), "copy"));
    double rz = 0.0;
    TDG_TRY(dot(r, z, &rz));
    std::vector<double> alpha, beta;
    for (int k = 0; k < mg.opts.esteig_steps && rz > 0.0; ++k) {
        TDG_TRY(mg_level_apply(op, l, p, q, nullptr, 1, s));
        double pq = 0.0;
        TDG_TRY(dot(p, q, &pq));
        if (!(pq > 0.0)) break;
        const double a = rz / pq;
        TDG_TRY(mgk(launch_vec_axpby(n, -a, q, 1.0, r, s), "axpy"));
        TDG_TRY(mgk(launch_vec_mul(n, L.dinv, r, z, s), "jacobi"));
        double rz1 = 0.0;
        TDG_TRY(dot(r, z, &rz1));
        const double bta = rz1 / rz;
        alpha.push_back(a);
        beta.push_back(bta);
        TDG_TRY(mgk(launch_vec_axpby(n, 1.0, z, bta, p, s), "xpay"));
        rz = rz1;
    }
    if (alpha.empty()) return fail(TDG_E_NOT_SPD, "multigrid: the level operator is not positive definite");
    const size_t m = alpha.size();
    std::vector<double> a(m), c(m > 1 ? m - 1 : 0);
    for (size_t k = 0; k < m; ++k) {
        a[k] = 1.0 / alpha[k] + (k > 0 ? beta[k - 1] / alpha[k - 1] : 0.0);
        if (k + 1 < m) c[k] = std::sqrt(beta[k]) / alpha[k];
    }
    L.lmax = tridiag_lmax(a, c);
    if (!(L.lmax > 0.0) || !std::isfinite(L.lmax)) return fail(TDG_E_NOT_SPD, "multigrid: bad eigenvalue estimate");
    return 0;
}

// The first coarse level's Galerkin operator I^T A I by probing the matrix-free operator: for each
// colour and each coarse basis column j, one multi-RHS apply of the interpolated unit columns on
// all elements of that colour.
int mg_probe(tdg_op* op, cudaStream_t s) {
    auto& mg = op->mg;
    const size_t nl = mg.lv.size();
    auto& C = mg.lv[nl - 2];
    const int64_t nf = mg.lv[nl - 1].n, E = op->h.E;
    const int nj = std::min(C.bs, 16);
    double *V = nullptr, *Y = nullptr;
    TDG_CUDA_TRY(cudaMalloc(&V, sizeof(double) * nj * nf));
    cudaError_t ce = cudaMalloc(&Y, sizeof(double) * nj * nf);
    if (ce != cudaSuccess) {
        cudaFree(V);
        return fail(TDG_E_NOMEM, "multigrid: probe vectors");
    }
    int rc = 0;
    for (int c = 0; c < mg.ncolours && rc == 0; ++c)
        for (int j0 = 0; j0 < C.bs && rc == 0; j0 += nj) {
            const int nb = std::min(nj, C.bs - j0);
            if (cudaMemsetAsync(V, 0, sizeof(double) * nb * nf, s) != cudaSuccess) rc = fail(TDG_E_CUDA, "memset");
            if (!rc) rc = mgk(launch_mg_probe_fill(E, mg.colour, c, C.ip, j0, nb, V, nf, s), "probe fill");
            if (!rc) rc = tdg_apply(op, TDG_FP64, V, Y, nb, nf, s);
            if (!rc)
                rc = mgk(launch_mg_probe_extract(E, mg.NB, mg.nbr, mg.colour, c, C.ip, j0, nb, Y, nf, C.A, s),
                         "probe extract");
        }
    cudaStreamSynchronize(s);
    cudaFree(V);
    cudaFree(Y);
    return rc;
}

// Continuous P1 level below the coarsest DG level: vertex numbering, the Galerkin operator
// R^T A_0 R assembled on the host from the coarsest DG level's blocks, its Q x Q diagonal blocks
// inverted for the block-Jacobi CG.
int mg_setup_aux(tdg_op* op, cudaStream_t s) {
    auto& h = op->h;
    auto& mg = op->mg;
    auto& L0 = mg.lv[0];
    const int64_t E = h.E;
    const int NVe = h.D + 1, Nbf0 = L0.bs / h.Q;
    std::vector<double> A0(static_cast<size_t>(E) * mg.NB * L0.bs * L0.bs);
    TDG_CUDA_TRY(cudaMemcpyAsync(A0.data(), L0.A, A0.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    std::vector<int32_t> nbr(static_cast<size_t>(E) * mg.NB);
    TDG_CUDA_TRY(cudaMemcpyAsync(nbr.data(), mg.nbr, nbr.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    TDG_CUDA_TRY(cudaStreamSynchronize(s));
    int64_t nv = 0;
    std::vector<int32_t> vid = vertex_numbering(h, &nv);
    Dense T = linear_to_space(h.D, h.kind, L0.degree);
    VertexCsr c = vertex_galerkin(A0, nbr, E, mg.NB, h.D, Nbf0, h.Q, T, vid, nv);
    A0.clear();
    A0.shrink_to_fit();
    const int64_t* dptr = nullptr;
    const int32_t *dcol = nullptr, *dvinc = nullptr, *dvid = nullptr;
    const double *dval = nullptr, *dT = nullptr;
    const int64_t* dvp = nullptr;
    TDG_CUDA_TRY(mg.arena.upload(&dptr, c.ptr));
    TDG_CUDA_TRY(mg.arena.upload(&dcol, c.col));
    TDG_CUDA_TRY(mg.arena.upload(&dval, c.val));
    TDG_CUDA_TRY(mg.arena.upload(&dvp, c.vinc_ptr));
    TDG_CUDA_TRY(mg.arena.upload(&dvinc, c.vinc));
    TDG_CUDA_TRY(mg.arena.upload(&dvid, vid));
    TDG_CUDA_TRY(mg.arena.upload(&dT, T.a));
    mg.ax.ptr = dptr;
    mg.ax.col = dcol;
    mg.ax.val = dval;
    mg.ax.vinc_ptr = dvp;
    mg.ax.vinc = dvinc;
    mg.ax.vid = dvid;
    mg.ax.T = dT;
    mg.ax.nv = nv;
    mg.ax.Q = h.Q;
    mg.ax.Nbf = Nbf0;
    mg.ax.NV = NVe;
    mg.cn = nv * h.Q;
    mg.cbs = h.Q;
    mg.cnb = nv;
    // diagonal blocks, column-major, for the block-Jacobi inversion
    const int Q = h.Q;
    std::vector<double> diag(static_cast<size_t>(nv) * Q * Q, 0.0);
    for (int64_t v = 0; v < nv; ++v) {
        const int32_t* c0 = c.col.data() + c.ptr[static_cast<size_t>(v)];
        const int32_t* c1 = c.col.data() + c.ptr[static_cast<size_t>(v) + 1];
        const int32_t* it = std::lower_bound(c0, c1, static_cast<int32_t>(v));
        if (it == c1 || *it != v) return fail(TDG_E_NOT_SPD, "multigrid: a P1 vertex without a diagonal block");
        const double* blk = &c.val[static_cast<size_t>(it - c.col.data()) * Q * Q];
        for (int p = 0; p < Q; ++p)
            for (int q = 0; q < Q; ++q) diag[static_cast<size_t>(v) * Q * Q + q * Q + p] = blk[p * Q + q];
    }
    const double* ddiag = nullptr;
    TDG_CUDA_TRY(mg.arena.upload(&ddiag, diag));
    TDG_CUDA_TRY(mg.arena.alloc(&mg.cinv, diag.size()));
    return mgk(launch_bjac_invert<double>(Q, nv, ddiag, mg.cinv, mg.status, s), "P1 block inversion");
}

int mg_setup(tdg_op* op, tdg_mg_opts o, cudaStream_t s) {
    auto& h = op->h;
    auto& mg = op->mg;
    if (o.smooth_its <= 0) o.smooth_its = 10;
    if (!(o.esteig_lo > 0.0)) o.esteig_lo = 0.01;
    if (!(o.esteig_hi > 0.0)) o.esteig_hi = 1.1;
    if (o.esteig_steps <= 0) o.esteig_steps = 10;
    if (!(o.coarse_rtol > 0.0)) o.coarse_rtol = 0.1;
    if (o.coarse_max_it <= 0) o.coarse_max_it = 1000;
    if (o.coarse_degree < 0) o.coarse_degree = 1;
    if (o.smooth_precision != TDG_MIXED && o.smooth_precision != TDG_TF32) o.smooth_precision = TDG_FP64;
    if (o.strategy < 0 || o.strategy > 2) return fail(TDG_E_INVALID, "multigrid: unknown strategy");
    if (!(o.esteig_lo < o.esteig_hi)) return fail(TDG_E_INVALID, "multigrid: esteig_lo must be below esteig_hi");
    if (!h.has_material) return fail(TDG_E_STATE, "multigrid: tdg_set_material first");
    std::vector<int> deg;
    try {
        deg = mg_level_degrees(o.strategy, o.coarse_degree, h.N);
    } catch (std::exception const& e) {
        return fail(TDG_E_INVALID, e.what());
    }
    if (deg.size() < 2) return fail(TDG_E_INVALID, "multigrid: needs at least two levels");
    // a fresh hierarchy
    mg.reset_graph();
    mg.ws.release();
    mg.arena.release();
    mg.lv.clear();
    mg.ready = false;
    TDG_TRY(ensure_loop(op));
    TDG_CUDA_TRY(cudaMemset(op->loop + kCoarseIts, 0, 3 * sizeof(long long)));  // its, diverged, total
    mg.opts = o;
    mg.fine_prec = o.smooth_precision;
    // the continuous P1 level embeds in the coarsest DG level only from degree 1 on
    mg.aux = o.coarse_space == TDG_MG_COARSE_P1 && deg[0] >= 1;
    TDG_TRY(ensure_uploaded(op, TDG_FP64));
    if (mg.fine_prec != TDG_FP64) TDG_TRY(ensure_uploaded(op, TDG_FP32));
    TDG_TRY(ensure_blocks(op, s));
    const int64_t E = h.E;
    mg.NB = 1 + h.nfaces;
    std::vector<int32_t> nbr = element_neighbours(h);
    std::vector<int32_t> col = distance2_colouring(nbr, E, mg.NB, &mg.ncolours);
    const int32_t* dn = nullptr;
    const int32_t* dc = nullptr;
    TDG_CUDA_TRY(mg.arena.upload(&dn, nbr));
    TDG_CUDA_TRY(mg.arena.upload(&dc, col));
    mg.nbr = const_cast<int32_t*>(dn);
    mg.colour = const_cast<int32_t*>(dc);
    const int nl = static_cast<int>(deg.size());
    mg.lv.resize(static_cast<size_t>(nl));
    for (int l = 0; l < nl; ++l) {
        auto& L = mg.lv[static_cast<size_t>(l)];
        L.degree = deg[static_cast<size_t>(l)];
        L.bs = num_basis(h.D, L.degree) * h.Q;
        L.n = E * L.bs;
        if (l + 1 < nl) {
            TDG_CUDA_TRY(mg.arena.alloc(&L.A, static_cast<size_t>(E) * mg.NB * L.bs * L.bs));
            TDG_CUDA_TRY(cudaMemsetAsync(L.A, 0, sizeof(double) * E * mg.NB * L.bs * L.bs, s));
            Dense I = interpolation_matrix(h.D, h.kind, deg[static_cast<size_t>(l + 1)], L.degree);
            const double* dI = nullptr;
            TDG_CUDA_TRY(mg.arena.upload(&dI, I.a));
            L.ip = MgInterp{dI, I.rows, I.cols, h.Q};
        }
        TDG_CUDA_TRY(mg.arena.alloc(&L.dinv, static_cast<size_t>(L.n)));
    }
    TDG_CUDA_TRY(mg.arena.alloc(&mg.status, 1));
    TDG_CUDA_TRY(cudaMemsetAsync(mg.status, 0, sizeof(int), s));
    // Galerkin operators: probing below the finest level, triple products further down
    TDG_TRY(mg_probe(op, s));
    for (int l = nl - 3; l >= 0; --l)
        TDG_TRY(mgk(launch_mg_triple(E, mg.NB, mg.nbr, mg.lv[static_cast<size_t>(l)].ip,
                                     mg.lv[static_cast<size_t>(l + 1)].A, mg.lv[static_cast<size_t>(l)].A, s),
                    "Galerkin triple product"));
    // point-Jacobi diagonals
    for (int l = 0; l < nl; ++l) {
        auto& L = mg.lv[static_cast<size_t>(l)];
        if (l + 1 == nl)
            TDG_TRY(mgk(launch_mg_diag_inv(E, L.bs, static_cast<int64_t>(L.bs) * L.bs, op->blk, L.dinv, mg.status, s),
                        "diagonal"));
        else
            TDG_TRY(mgk(launch_mg_diag_inv(E, L.bs, static_cast<int64_t>(mg.NB) * L.bs * L.bs, L.A, L.dinv, mg.status, s),
                        "diagonal"));
    }
    // the coarse system: block-Jacobi inverses, CG vectors and plan
    auto& L0 = mg.lv[0];
    if (mg.aux) {
        TDG_TRY(mg_setup_aux(op, s));
    } else {
        mg.cn = L0.n;
        mg.cbs = L0.bs;
        mg.cnb = E;
        double* blk0 = nullptr;
        TDG_CUDA_TRY(cudaMalloc(&blk0, sizeof(double) * E * L0.bs * L0.bs));
        int rc = mgk(launch_mg_self_blocks(E, mg.NB, L0.bs, L0.A, blk0, s), "coarse blocks");
        if (!rc) {
            cudaError_t ce = mg.arena.alloc(&mg.cinv, static_cast<size_t>(E) * L0.bs * L0.bs);
            rc = ce == cudaSuccess ? 0 : fail(TDG_E_NOMEM, "multigrid: coarse inverses");
        }
        if (!rc) rc = mgk(launch_bjac_invert<double>(L0.bs, E, blk0, mg.cinv, mg.status, s), "coarse inversion");
        cudaStreamSynchronize(s);
        cudaFree(blk0);
        if (rc) return rc;
    }
    int st = 0;
    TDG_CUDA_TRY(cudaMemcpyAsync(&st, mg.status, sizeof(int), cudaMemcpyDeviceToHost, s));
    TDG_CUDA_TRY(cudaStreamSynchronize(s));
    if (st) return fail(TDG_E_NOT_SPD, "multigrid: a level diagonal or coarse block is not positive definite");
    // work vectors for one right-hand side (grown by tdg_mg_apply on demand)
    mg.cap = 0;
    mg.fine_ld = 0;
    TDG_TRY(mg_ensure_ws(op, 1, mg.lv.back().n, s));
    // mixed precision: the smoothed levels below the finest apply FP32 copies of their blocks
    // (half the bytes of the HBM-bound block-sparse apply; vectors and accumulation stay FP64)
    if (mg.fine_prec != TDG_FP64)
        for (int l = mg.aux ? 0 : 1; l + 1 < nl; ++l) {
            auto& L = mg.lv[static_cast<size_t>(l)];
            const int64_t nb = E * mg.NB * L.bs * L.bs;
            TDG_CUDA_TRY(mg.arena.alloc(&L.A32, static_cast<size_t>(nb)));
            TDG_TRY(mgk(launch_round_to_float(nb, L.A, L.A32, s), "FP32 level blocks"));
        }
    // Chebyshev bounds of the smoothed levels
    for (int l = mg.aux ? 0 : 1; l < nl; ++l) TDG_TRY(mg_estimate_lmax(op, l, s));
    mg.ready = true;
    return 0;
}

int mg_apply(tdg_op* op, const double* r, double* z, int nrhs, int64_t ld, cudaStream_t s) {
    auto& mg = op->mg;
    if (!mg.ready) return fail(TDG_E_STATE, "tdg_mg_setup not called");
    if (nrhs < 1 || ld < mg.lv.back().n) return fail(TDG_E_INVALID, "nrhs < 1 or ld < E * bs");
    TDG_TRY(mg_ensure_ws(op, nrhs, ld, s));
    return mg_vcycle(op, static_cast<int>(mg.lv.size()) - 1, r, z, nrhs, s);
}

// z = M r with the preconditioner the solves use (multigrid for FP64 vectors when selected).
template <typename T>
int precondition(tdg_op* op, int prec, const T* r, T* z, int nrhs, int64_t ld, cudaStream_t s) {
    if constexpr (std::is_same_v<T, double>) {
        if (op->pc == TDG_PC_MG) return mg_apply(op, r, z, nrhs, ld, s);
    }
    return tdg_bjacobi_apply(op, prec, r, z, nrhs, ld, s);
}

}  // namespace

// ------------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------------

extern "C" {

const char* tdg_last_error(void) { return g_last_error.c_str(); }

int tdg_create(const tdg_mesh_desc* mesh, const tdg_quadrature* quad, int kind, tdg_op** out) {
    g_last_error.clear();
    if (!mesh || !quad || !out) return fail(TDG_E_INVALID, "null argument");
    if (!mesh->geo_nodes || !mesh->facet_up || !mesh->facet_local_no || !mesh->facet_bc)
        return fail(TDG_E_INVALID, "mesh arrays missing");
    if (!quad->vol_points || !quad->vol_weights || !quad->fct_points || !quad->fct_weights)
        return fail(TDG_E_INVALID, "quadrature arrays missing");
    if (mesh->degree < kMinDegree || mesh->degree > kMaxDegree)
        return fail(TDG_E_INVALID, "degree outside the compiled range [1, 4]");
    try {
        auto* op = new tdg_op();
        const char* kv = std::getenv("TDG_APPLY_KERNEL");
        op->use_mma = !(kv && std::string(kv) == "simt");
        op->h.build(mesh->dim, mesh->degree, mesh->geo_degree, kind, mesh->num_elements, mesh->num_facets,
                    mesh->geo_nodes, mesh->facet_up, mesh->facet_local_no, mesh->facet_bc,
                    quad->num_vol_points, quad->vol_points, quad->vol_weights, quad->num_fct_points,
                    quad->fct_points, quad->fct_weights);
        *out = op;
        return 0;
    } catch (std::exception const& e) {
        return fail(TDG_E_INVALID, e.what());
    }
}

void tdg_destroy(tdg_op* op) { delete op; }

int tdg_sizes(const tdg_op* op, int64_t out[8]) {
    if (!op || !out) return fail(TDG_E_INVALID, "null argument");
    auto const& h = op->h;
    out[0] = h.bs;
    out[1] = h.Nbf;
    out[2] = h.Q;
    out[3] = h.Nq;
    out[4] = h.nq;
    out[5] = h.E;
    out[6] = h.F;
    out[7] = h.D;
    return 0;
}

int tdg_volume_coords(const tdg_op* op, double* out) {
    if (!op || !out) return fail(TDG_E_INVALID, "null argument");
    std::memcpy(out, op->h.vCoords.data(), op->h.vCoords.size() * sizeof(double));
    return 0;
}

int tdg_facet_coords(const tdg_op* op, double* out) {
    if (!op || !out) return fail(TDG_E_INVALID, "null argument");
    std::memcpy(out, op->h.fCoords.data(), op->h.fCoords.size() * sizeof(double));
    return 0;
}

int tdg_facet_normals(const tdg_op* op, double* out) {
    if (!op || !out) return fail(TDG_E_INVALID, "null argument");
    auto const& h = op->h;
    for (int64_t f = 0; f < h.F; ++f)
        for (int q = 0; q < h.nq; ++q)
            for (int i = 0; i < h.D; ++i)
                out[(static_cast<size_t>(f) * h.nq + q) * h.D + i] = h.fN[(static_cast<size_t>(f) * h.D + i) * h.nq + q];
    return 0;
}

int tdg_set_material(tdg_op* op, const double* c0_Q, const double* c1_Q) {
    if (!op) return fail(TDG_E_INVALID, "null operator");
    try {
        op->h.set_material(c0_Q, c1_Q);
    } catch (std::exception const& e) {
        return fail(TDG_E_INVALID, e.what());
    }
    op->arena64.release();
    op->arena32.release();
    op->arena_common.release();
    op->arena_pc.release();
    op->uploaded64 = op->uploaded32 = false;
    op->penalty = nullptr;
    op->sides = nullptr;
    op->blk = nullptr;
    op->inv = nullptr;
    op->inv_precision = -1;
    op->mg.ready = false;  // the hierarchy's Galerkin operators and bounds belong to the old material
    op->status = nullptr;
    return 0;
}

int tdg_update_material(tdg_op* op, const double* c0_Q, const double* c1_Q) {
    if (!op) return fail(TDG_E_INVALID, "null operator");
    const bool pc_ready = op->inv != nullptr || op->mg.ready;
    if (!op->h.has_material || !pc_ready)
        return fail(TDG_E_STATE, "tdg_update_material needs a material and a preconditioner set up for it");
    try {
        op->h.set_material(c0_Q, c1_Q);
    } catch (std::exception const& e) {
        return fail(TDG_E_INVALID, e.what());
    }
    // the operator's own data (both precisions, the penalty) follow the new material on the next
    // upload; the block-Jacobi inverses (arena_pc) and the multigrid hierarchy stay as they are
    op->arena64.release();
    op->arena32.release();
    op->arena_common.release();
    op->uploaded64 = op->uploaded32 = false;
    op->penalty = nullptr;
    op->sides = nullptr;
    return 0;
}

int tdg_material_nodal(const tdg_op* op, int c, double* out) {
    if (!op || !out || c < 0 || c > 1) return fail(TDG_E_INVALID, "bad argument");
    auto const& h = op->h;
    if (!h.has_material) return fail(TDG_E_STATE, "no material");
    int nm = h.mat_space.num_basis();
    for (int64_t e = 0; e < h.E; ++e)
        std::memcpy(out + e * nm, &h.mat_nodal[(static_cast<size_t>(e) * 2 + c) * nm], nm * sizeof(double));
    return 0;
}

int tdg_penalty(const tdg_op* op, double* out) {
    if (!op || !out) return fail(TDG_E_INVALID, "bad argument");
    if (!op->h.has_material) return fail(TDG_E_STATE, "no material");
    std::memcpy(out, op->h.penalty.data(), op->h.penalty.size() * sizeof(double));
    return 0;
}

int tdg_apply(tdg_op* op, int precision, const void* x, void* y, int nrhs, int64_t ld, void* stream) {
    if (!op || !x || !y) return fail(TDG_E_INVALID, "null argument");
    auto const& h = op->h;
    if (nrhs < 1 || ld < h.E * h.bs) return fail(TDG_E_INVALID, "nrhs < 1 or ld < E * bs");
    if (x == y) return fail(TDG_E_INVALID, "x and y must not alias");
    TDG_TRY(ensure_uploaded(op, precision));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = TDG_E_INVALID;
    const int pi = precision == TDG_FP64 ? 0 : 1;
    const bool tensor = op->use_mma && op->family[pi] == 0;
    if (precision == TDG_FP64 && op->use_mma && op->family[0] == 3)
        rc = launch_apply_face2(h.D, h.N, h.kind, op->op64, op->mma, op->face, op->tgeo,
                                static_cast<const double*>(x), static_cast<double*>(y), nrhs, ld, s, op->ctas[0],
                                op->tile[0]);
    // family 3 falls back to family 2 only where its automatic layout does not fit; an explicit
    // points-per-pass that does not fit is the caller's error
    if (precision == TDG_FP64 && op->family[0] == 3 && op->tile[0] != 0 && rc == TDG_E_INVALID)
        return fail(rc, "points per pass do not fit this shape");
    if (precision == TDG_FP64 && op->use_mma && (op->family[0] == 2 || (op->family[0] == 3 && rc == TDG_E_INVALID)))
        rc = launch_apply_face(h.D, h.N, h.kind, op->op64, op->mma, op->face, static_cast<const double*>(x),
                               static_cast<double*>(y), nrhs, ld, s, op->ctas[0]);
    else if (precision == TDG_FP64 && tensor)
        rc = launch_apply_mma(h.D, h.N, h.kind, op->op64, op->mma, static_cast<const double*>(x),
                              static_cast<double*>(y), nrhs, ld, s, op->ctas[0]);
    if (precision == TDG_FP64 && rc == TDG_E_INVALID)
        rc = launch_apply<double>(h.D, h.N, h.kind, op->op64, static_cast<const double*>(x),
                                  static_cast<double*>(y), nrhs, ld, s);
    const bool face32 = op->use_mma && op->family[1] >= 2;  // face-centric (the FP32 kernels have one form)
    const bool vol05 = op->family[1] == 4;                    // its volume term on tcgen05
    if (precision == TDG_FP32 && face32)
        rc = launch_apply_face_tc32<float>(h.D, h.N, h.kind, op->op32, op->tc32, op->face32,
                                           static_cast<const float*>(x), static_cast<float*>(y), nrhs, ld, s,
                                           op->ctas[1], vol05);
    else if (precision == TDG_FP32 && tensor)
        rc = launch_apply_tc32<float>(h.D, h.N, h.kind, op->op32, op->tc32, static_cast<const float*>(x),
                                      static_cast<float*>(y), nrhs, ld, s, op->ctas[1]);
    if (precision == TDG_MIXED || precision == TDG_TF32) {
        if (!op->use_mma) return fail(TDG_E_INVALID, "TDG_MIXED / TDG_TF32 need the tensor-core kernels");
        const int passes = precision == TDG_TF32 ? 1 : 3;  // one TF32 pass, or 3xTF32
        // the selected tensor-core family, else the other one (a shape whose element-centric tile
        // does not fit shared memory runs face-centric, and the reverse)
        auto face = [&] {
            return launch_apply_face_tc32<double>(h.D, h.N, h.kind, op->op32, op->tc32, op->face32,
                                                  static_cast<const double*>(x), static_cast<double*>(y), nrhs, ld, s,
                                                  op->ctas[1], vol05, passes);
        };
        auto elem = [&] {
            return launch_apply_tc32<double>(h.D, h.N, h.kind, op->op32, op->tc32, static_cast<const double*>(x),
                                             static_cast<double*>(y), nrhs, ld, s, op->ctas[1], passes);
        };
        rc = face32 ? face() : elem();
        if (rc == TDG_E_INVALID) rc = face32 ? elem() : face();
        if (rc) return fail(rc, std::string("mixed apply launch failed: ") + cudaGetErrorString(cudaGetLastError()));
        return 0;
    }
    if (precision == TDG_FP32 && rc == TDG_E_INVALID)
        rc = launch_apply<float>(h.D, h.N, h.kind, op->op32, static_cast<const float*>(x),
                                 static_cast<float*>(y), nrhs, ld, s);
    if (rc) return fail(rc, std::string("apply launch failed: ") + cudaGetErrorString(cudaGetLastError()));
    return 0;
}

int tdg_apply_host(tdg_op* op, int precision, const void* x_host, void* y_host, int count, int64_t host_stride,
                   void* stream) {
    if (!op || !x_host || !y_host) return fail(TDG_E_INVALID, "null argument");
    if (precision != TDG_FP64 && precision != TDG_FP32 && precision != TDG_MIXED)
        return fail(TDG_E_INVALID, "unknown precision");
    auto const& h = op->h;
    const int64_t n = h.E * h.bs;
    if (count < 1 || (host_stride != 0 && host_stride < n)) return fail(TDG_E_INVALID, "count < 1 or 0 < host_stride < E * bs");
    if (x_host == y_host) return fail(TDG_E_INVALID, "x and y must not alias");
    const size_t esz = precision == TDG_FP32 ? sizeof(float) : sizeof(double);
    const size_t bytes = static_cast<size_t>(n) * esz;
    auto& hs = op->hs;
    if (!hs.ready) {
        for (int k = 0; k < 3; ++k) TDG_CUDA_TRY(cudaStreamCreateWithFlags(&hs.s[k], cudaStreamNonBlocking));
        for (int b = 0; b < 2; ++b) {
            TDG_CUDA_TRY(cudaEventCreateWithFlags(&hs.in[b], cudaEventDisableTiming));
            TDG_CUDA_TRY(cudaEventCreateWithFlags(&hs.out[b], cudaEventDisableTiming));
            TDG_CUDA_TRY(cudaEventCreateWithFlags(&hs.freed[b], cudaEventDisableTiming));
            TDG_CUDA_TRY(cudaEventCreateWithFlags(&hs.done[b], cudaEventDisableTiming));
        }
        TDG_CUDA_TRY(cudaEventCreateWithFlags(&hs.entry, cudaEventDisableTiming));
        hs.ready = true;
    }
    if (hs.bytes < bytes) {
        for (int b = 0; b < 2; ++b) {
            if (hs.xd[b]) cudaFree(hs.xd[b]);
            if (hs.yd[b]) cudaFree(hs.yd[b]);
            hs.xd[b] = hs.yd[b] = nullptr;
        }
        hs.bytes = 0;
        for (int b = 0; b < 2; ++b) {
            if (cudaMalloc(&hs.xd[b], bytes) != cudaSuccess || cudaMalloc(&hs.yd[b], bytes) != cudaSuccess)
                return fail(TDG_E_NOMEM, "tdg_apply_host: device buffers");
        }
        hs.bytes = bytes;
    }
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    cudaStream_t cin = hs.s[0], cmp = hs.s[1], cout = hs.s[2];
    // everything already on the caller's stream comes first
    TDG_CUDA_TRY(cudaEventRecord(hs.entry, user));
    for (int k = 0; k < 3; ++k) TDG_CUDA_TRY(cudaStreamWaitEvent(hs.s[k], hs.entry, 0));
    const char* xb = static_cast<const char*>(x_host);
    char* yb = static_cast<char*>(y_host);
    const size_t hstep = static_cast<size_t>(host_stride) * esz;
    auto step = [&](int i) -> int {
        const int b = i & 1;
        // x buffer b is free once the apply two steps back has read it; y buffer b once that apply's
        // result has been copied out.  Freeing them separately keeps the copy-in stream busy while
        // the copy-out of two steps back still runs.
        if (i >= 2) TDG_CUDA_TRY(cudaStreamWaitEvent(cin, hs.out[b], 0));
        TDG_CUDA_TRY(cudaMemcpyAsync(hs.xd[b], xb + i * hstep, bytes, cudaMemcpyHostToDevice, cin));
        TDG_CUDA_TRY(cudaEventRecord(hs.in[b], cin));
        TDG_CUDA_TRY(cudaStreamWaitEvent(cmp, hs.in[b], 0));
        if (i >= 2) TDG_CUDA_TRY(cudaStreamWaitEvent(cmp, hs.freed[b], 0));
        TDG_TRY(tdg_apply(op, precision, hs.xd[b], hs.yd[b], 1, n, cmp));
        TDG_CUDA_TRY(cudaEventRecord(hs.out[b], cmp));
        TDG_CUDA_TRY(cudaStreamWaitEvent(cout, hs.out[b], 0));
        TDG_CUDA_TRY(cudaMemcpyAsync(yb + i * hstep, hs.yd[b], bytes, cudaMemcpyDeviceToHost, cout));
        TDG_CUDA_TRY(cudaEventRecord(hs.freed[b], cout));
        return 0;
    };
    for (int i = 0; i < count; ++i) {
        if (int rc = step(i)) {
            // nothing of the caller's host buffers stays in flight after an error
            for (int k = 0; k < 3; ++k) cudaStreamSynchronize(hs.s[k]);
            return rc;
        }
    }
    // the caller's stream continues after the last copy out (and after every apply)
    TDG_CUDA_TRY(cudaEventRecord(hs.done[0], cout));
    TDG_CUDA_TRY(cudaEventRecord(hs.done[1], cmp));
    TDG_CUDA_TRY(cudaStreamWaitEvent(user, hs.done[0], 0));
    TDG_CUDA_TRY(cudaStreamWaitEvent(user, hs.done[1], 0));
    return 0;
}

int tdg_set_apply_config(tdg_op* op, int precision, int family, int ctas_per_sm) {
    if (!op || (precision != TDG_FP64 && precision != TDG_FP32) || family < 0 || family > 4 || ctas_per_sm < 0 ||
        (family == 4 && precision != TDG_FP32))
        return fail(TDG_E_INVALID, "bad argument");
    const int pi = precision == TDG_FP64 ? 0 : 1;
    op->family[pi] = family;
    op->ctas[pi] = ctas_per_sm;
    return 0;
}

int tdg_set_apply_tile(tdg_op* op, int precision, int points_per_pass) {
    if (!op || (precision != TDG_FP64 && precision != TDG_FP32) || points_per_pass < 0)
        return fail(TDG_E_INVALID, "bad argument");
    if (points_per_pass != 0 && (precision != TDG_FP64 || points_per_pass % face2_pass_step(op->h.D) != 0))
        return fail(TDG_E_INVALID, "points per pass: FP64 only, a multiple of 8 (3D) or 4 (2D)");
    op->tile[precision == TDG_FP64 ? 0 : 1] = points_per_pass;
    return 0;
}

// Points-per-pass candidates of the FP64 pipelined volume kernel: one pass (0, the automatic
// layout), then the smallest multiple of the step that covers the points in 2, 3 and 4 passes.
static std::vector<int> face2_tile_candidates(int D, int Nq) {
    std::vector<int> t{0};
    const int step = face2_pass_step(D);
    for (int p = 2; p <= 4; ++p) {
        const int qc = ((Nq + p - 1) / p + step - 1) / step * step;
        if (qc < Nq && qc >= step && (t.size() == 1 || t.back() != qc)) t.push_back(qc);
    }
    return t;
}

int tdg_autotune(tdg_op* op, int precision, int nrhs, void* stream, tdg_tune_entry* entries, int max_entries,
                 int* n_entries) {
    if (!op || nrhs < 1 || (precision != TDG_FP64 && precision != TDG_FP32))
        return fail(TDG_E_INVALID, "bad argument");
    TDG_TRY(ensure_uploaded(op, precision));
    auto const& h = op->h;
    const int pi = precision == TDG_FP32 ? 1 : 0;
    const size_t esz = precision == TDG_FP32 ? sizeof(float) : sizeof(double);
    const int64_t ld = h.E * h.bs;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void *x = nullptr, *y = nullptr;
    if (cudaMalloc(&x, esz * ld * nrhs) != cudaSuccess) return fail(TDG_E_NOMEM, "autotune buffers");
    if (cudaMalloc(&y, esz * ld * nrhs) != cudaSuccess) {
        cudaFree(x);
        return fail(TDG_E_NOMEM, "autotune buffers");
    }
    cudaMemsetAsync(x, 0x3f, esz * ld * nrhs, s);
    // candidates: tensor-core kernel at 1..4 persistent CTAs per SM (clipped to the occupancy
    // limit), then the SIMT kernel
    struct Cand {
        int family, ctas, tile;
    };
    std::vector<Cand> cands;
    if (op->use_mma)
        for (int c = 1; c <= 4; ++c) cands.push_back({0, c, 0});
    if (op->use_mma)
        for (int c = 1; c <= 4; ++c) cands.push_back({2, c, 0});
    if (op->use_mma && precision == TDG_FP64)
        for (int c = 1; c <= 2; ++c)
            for (int t : face2_tile_candidates(h.D, h.Nq)) cands.push_back({3, c, t});
    if (op->use_mma && precision == TDG_FP32)  // the facet kernel's CTAs; the tcgen05 volume kernel runs one per SM
        for (int c = 1; c <= 4; ++c) cands.push_back({4, c, 0});
    cands.push_back({1, 0, 0});
    const int fam0 = op->family[pi], ct0 = op->ctas[pi], tl0 = op->tile[pi];
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    int bi = -1, n = 0, rc = 0;
    for (size_t i = 0; i < cands.size() && rc == 0; ++i) {
        op->family[pi] = cands[i].family;
        op->ctas[pi] = cands[i].ctas;
        op->tile[pi] = cands[i].tile;
        for (int w = 0; w < 2 && rc == 0; ++w) rc = tdg_apply(op, precision, x, y, nrhs, ld, stream);
        if (rc == TDG_E_INVALID && cands[i].tile != 0) {  // a points-per-pass that does not fit: skip it
            rc = 0;
            continue;
        }
        if (rc) break;
        constexpr int reps = 5;
        cudaEventRecord(e0, s);
        for (int r = 0; r < reps && rc == 0; ++r) rc = tdg_apply(op, precision, x, y, nrhs, ld, stream);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double per = ms / reps;
        if (entries && n < max_entries) entries[n] = tdg_tune_entry{cands[i].family, cands[i].ctas, cands[i].tile, per};
        ++n;
        if (per < best) {
            best = per;
            bi = static_cast<int>(i);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(x);
    cudaFree(y);
    if (rc || bi < 0) {
        op->family[pi] = fam0;
        op->ctas[pi] = ct0;
        op->tile[pi] = tl0;
        return rc ? rc : fail(TDG_E_CUDA, "autotune found no candidate");
    }
    op->family[pi] = cands[bi].family;
    op->ctas[pi] = cands[bi].ctas;
    op->tile[pi] = cands[bi].tile;
    if (n_entries) *n_entries = n;
    return 0;
}

int64_t tdg_flops_apply(const tdg_op* op) { return op ? op->h.flops_apply() : -1; }

int64_t tdg_bytes_apply(const tdg_op* op, int precision) {
    return op ? op->h.bytes_apply(precision == TDG_FP32 ? 4 : 8) : -1;
}

int tdg_bjacobi_setup(tdg_op* op, int precision, void* stream) {
    if (!op) return fail(TDG_E_INVALID, "null operator");
    if (precision == TDG_MIXED) precision = TDG_FP32;  // FP32 inverses (the lighter mixed preconditioner)
    if (precision != TDG_FP64 && precision != TDG_FP32) return fail(TDG_E_INVALID, "bad precision");
    auto const& h = op->h;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t nblk = static_cast<size_t>(h.E) * h.bs * h.bs;
    TDG_TRY(ensure_blocks(op, s));
    if (op->inv && op->inv_precision == precision) return 0;
    if (op->inv) {
        // switching precision: re-allocate (arena keeps the old buffer until release)
        op->inv = nullptr;
    }
    TDG_CUDA_TRY(cudaMemsetAsync(op->status, 0, sizeof(int), s));
    int rc;
    if (precision == TDG_FP64) {
        double* inv = nullptr;
        TDG_CUDA_TRY(op->arena_pc.alloc(&inv, nblk));
        rc = launch_bjac_invert<double>(h.bs, h.E, op->blk, inv, op->status, s);
        op->inv = inv;
    } else {
        float* inv = nullptr;
        TDG_CUDA_TRY(op->arena_pc.alloc(&inv, nblk));
        rc = launch_bjac_invert<float>(h.bs, h.E, op->blk, inv, op->status, s);
        op->inv = inv;
    }
    if (rc) return fail(rc, "block inversion launch failed");
    op->inv_precision = precision;
    int st = 0;
    TDG_CUDA_TRY(cudaMemcpyAsync(&st, op->status, sizeof(int), cudaMemcpyDeviceToHost, s));
    TDG_CUDA_TRY(cudaStreamSynchronize(s));
    if (st) {
        op->inv = nullptr;
        op->inv_precision = -1;
        return fail(TDG_E_NOT_SPD, "a block-Jacobi diagonal block is not positive definite");
    }
    return 0;
}

int tdg_bjacobi_apply(tdg_op* op, int precision, const void* r, void* z, int nrhs, int64_t ld, void* stream) {
    if (!op || !r || !z) return fail(TDG_E_INVALID, "null argument");
    // FP64 and mixed (FP64 vectors) take FP64 or FP32 inverses; FP32 vectors take FP32 inverses
    if (!op->inv || (precision == TDG_FP32 && op->inv_precision != TDG_FP32))
        return fail(TDG_E_STATE, "tdg_bjacobi_setup not called for this precision");
    auto const& h = op->h;
    if (nrhs < 1 || ld < h.E * h.bs) return fail(TDG_E_INVALID, "nrhs < 1 or ld < E * bs");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc;
    if (precision == TDG_FP32)
        rc = launch_bjac_apply<float, float>(h.bs, h.E, static_cast<const float*>(op->inv),
                                             static_cast<const float*>(r), static_cast<float*>(z), nrhs, ld, s);
    else if (op->inv_precision == TDG_FP32)
        rc = launch_bjac_apply<float, double>(h.bs, h.E, static_cast<const float*>(op->inv),
                                              static_cast<const double*>(r), static_cast<double*>(z), nrhs, ld, s);
    else
        rc = launch_bjac_apply<double, double>(h.bs, h.E, static_cast<const double*>(op->inv),
                                               static_cast<const double*>(r), static_cast<double*>(z), nrhs, ld, s);
    if (rc) return fail(rc, "block-Jacobi apply launch failed");
    return 0;
}

int tdg_bjacobi_blocks(tdg_op* op, double* out) {
    if (!op || !out) return fail(TDG_E_INVALID, "null argument");
    if (!op->blk) return fail(TDG_E_STATE, "tdg_bjacobi_setup not called");
    auto const& h = op->h;
    TDG_CUDA_TRY(cudaDeviceSynchronize());
    TDG_CUDA_TRY(cudaMemcpy(out, op->blk, static_cast<size_t>(h.E) * h.bs * h.bs * sizeof(double),
                            cudaMemcpyDeviceToHost));
    return 0;
}

int tdg_rhs(tdg_op* op, const double* force_Q, const double* bc_q, double* b) {
    if (!op || !b) return fail(TDG_E_INVALID, "null argument");
    try {
        op->h.rhs(force_Q, bc_q, b);
    } catch (std::exception const& e) {
        return fail(TDG_E_STATE, e.what());
    }
    return 0;
}

int tdg_ref_nodes(int dim, int degree, int family, double* out) {
    if (!out || dim < 1 || dim > 3 || degree < 0 || degree > 15) return fail(TDG_E_INVALID, "bad argument");
    try {
        Points p = (family == 0) ? warp_blend_nodes(dim, degree) : equidistant_nodes(dim, degree);
        std::memcpy(out, p.data(), p.size() * sizeof(double));
    } catch (std::exception const& e) {
        return fail(TDG_E_INVALID, e.what());
    }
    return 0;
}

int tdg_ref_basis(int dim, int degree, int family, int np, const double* points, double* E, double* grad) {
    if (!points || dim < 1 || dim > 3 || degree < 0 || degree > 15 || np < 0)
        return fail(TDG_E_INVALID, "bad argument");
    try {
        RefSpace sp = (family < 0) ? RefSpace::modal(dim, degree)
                                   : RefSpace::nodal(dim, degree, family == 0 ? warp_blend_nodes(dim, degree)
                                                                              : equidistant_nodes(dim, degree));
        Points pts(points, points + static_cast<size_t>(np) * dim);
        if (E) {
            Dense e = sp.eval(pts);
            std::memcpy(E, e.a.data(), e.a.size() * sizeof(double));
        }
        if (grad) {
            auto g = sp.grad(pts);
            std::memcpy(grad, g.data(), g.size() * sizeof(double));
        }
    } catch (std::exception const& e) {
        return fail(TDG_E_INVALID, e.what());
    }
    return 0;
}

int tdg_conical_rule(int dim, int order, double* points, double* weights) {
    if (dim < 1 || dim > 3 || order < 0) return fail(TDG_E_INVALID, "bad argument");
    SimplexRule r = conical_product_rule(dim, order);
    if (points) std::memcpy(points, r.x.data(), r.x.size() * sizeof(double));
    if (weights) std::memcpy(weights, r.w.data(), r.w.size() * sizeof(double));
    return r.size();
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Krylov drivers
// ------------------------------------------------------------------------------------------------

namespace {

template <typename T>
struct CgVectors {
    T *r, *z, *p, *q;
};

// One preconditioned CG iteration on (A_T, M_T) with device-resident scalars; with the multigrid
// preconditioner the flexible CG step (beta from z_new . q).
template <typename T>
int cg_iteration(tdg_op* op, int prec, SegPlan const& sp, T* x, CgVectors<T> v, double* partial, double* scal,
                 cudaStream_t s) {
    const bool flexible = op->pc == TDG_PC_MG;
    TDG_TRY(krylov_apply(op, prec, sp, v.p, v.q, s));
    TDG_TRY(dots<T>(sp, v.p, v.q, nullptr, nullptr, partial, scal, kPQ, -1, s));
    k_cg_xr<T><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, x, v.r, v.p, v.q, scal);
    TDG_TRY(precondition<T>(op, prec, v.r, v.z, sp.op_nrhs, sp.op_ld, s));
    TDG_TRY(dots<T>(sp, v.r, v.z, v.r, v.r, partial, scal, kRZnew, kRR, s));
    if (flexible) TDG_TRY(dots<T>(sp, v.z, v.q, nullptr, nullptr, partial, scal, kZQ, -1, s));
    k_cg_p<T><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, v.p, v.z, scal, flexible ? 1 : 0);
    k_cg_shift<<<(sp.nseg + 127) / 128, 128, 0, s>>>(scal, sp.nseg);
    return cudaGetLastError() == cudaSuccess ? 0 : fail(TDG_E_CUDA, "CG update kernels");
}

// r = b - A x (FP64); per-segment ||r|| and ||b|| on the host.
int residual64(tdg_op* op, SegPlan const& sp, const double* b, const double* x, double* r, double* tmp,
               double* partial, double* scal, std::vector<double>& rn, std::vector<double>& bn, cudaStream_t s) {
    TDG_TRY(krylov_apply(op, TDG_FP64, sp, const_cast<double*>(x), tmp, s));
    k_sub<double><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, b, tmp, r);
    TDG_TRY(dots<double>(sp, r, r, b, b, partial, scal, kRR, kBB, s));
    std::vector<double> hs(static_cast<size_t>(sp.nseg) * kScal);
    TDG_CUDA_TRY(cudaMemcpyAsync(hs.data(), scal, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    TDG_CUDA_TRY(cudaStreamSynchronize(s));
    rn.resize(sp.nseg);
    bn.resize(sp.nseg);
    for (int i = 0; i < sp.nseg; ++i) {
        rn[i] = std::sqrt(hs[static_cast<size_t>(i) * kScal + kRR]);
        bn[i] = std::sqrt(hs[static_cast<size_t>(i) * kScal + kBB]);
    }
    return 0;
}

// z = M r, p = z, rz = r.z, rr = r.r, active flags from `active`.
template <typename T>
int cg_start(tdg_op* op, int prec, SegPlan const& sp, CgVectors<T> v, double* partial, double* scal,
             std::vector<double> const& active, std::vector<double> const& thr, cudaStream_t s) {
    std::vector<double> hs(static_cast<size_t>(sp.nseg) * kScal, 0.0);
    for (int i = 0; i < sp.nseg; ++i) {
        hs[static_cast<size_t>(i) * kScal + kActive] = active[i];
        hs[static_cast<size_t>(i) * kScal + kThr] = thr[i];
    }
    TDG_CUDA_TRY(cudaMemcpyAsync(scal, hs.data(), hs.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    TDG_TRY(precondition<T>(op, prec, v.r, v.z, sp.op_nrhs, sp.op_ld, s));
    k_copy<T><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, v.z, v.p);
    TDG_TRY(dots<T>(sp, v.r, v.z, v.r, v.r, partial, scal, kRZ, kRR, s));
    return cudaGetLastError() == cudaSuccess ? 0 : fail(TDG_E_CUDA, "CG start");
}

// Rebuilds the search direction after a residual replacement.  The block ended with
// p = z_old + beta p_prev, beta = rz_old / rz_prev; with the replaced residual the recurrence
// gives p = z_new + (rz_new / rz_prev) p_prev = z_new + (rz_new / rz_old) (p - z_old), and z
// takes z_new.  Segments flagged in scal[seg][kTmp] restart from p = z_new.  rz_new is in slot
// kRZnew, rz_old in kRZ (k_cg_shift then moves rz_new to kRZ).  Only the segments flagged kRepl
// (whose residual was replaced) change.
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_replace_dir(const Chunk* __restrict__ chunks, T* __restrict__ p, T* __restrict__ z, const T* __restrict__ znew,
                  const double* __restrict__ scal) {
    const Chunk ch = chunks[blockIdx.x];
    const double* sc = scal + ch.seg * kScal;
    if (sc[kActive] == 0.0 || sc[kRepl] == 0.0) return;
    const double rz = sc[kRZ];
    const T c = static_cast<T>((sc[kTmp] != 0.0 || rz == 0.0) ? 0.0 : sc[kRZnew] / rz);
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        const T zn = znew[i];
        p[i] = zn + c * (p[i] - z[i]);
        z[i] = zn;
    }
}

// x += (double) xh; xh = 0 (flush of the low-precision correction).
template <typename T>
__global__ void __launch_bounds__(kVecThreads)
    k_flush(const Chunk* __restrict__ chunks, double* __restrict__ x, T* __restrict__ xh) {
    const Chunk ch = chunks[blockIdx.x];
    for (int64_t i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        x[i] += static_cast<double>(xh[i]);
        xh[i] = T(0);
    }
}

// Preconditioned CG with reliable updates (residual replacement; Clark et al., "Solving lattice
// QCD systems of equations using mixed precision solvers on GPUs", 2010; van der Vorst & Ye,
// "Residual replacement strategies for Krylov subspace iterative methods", 2000).  The recurrence
// runs in T (operator, preconditioner and vectors in T, dot products accumulated in FP64) and
// accumulates its correction in xh.  Whenever a segment's recurrence residual has dropped by
// `delta` since the last update, or claims convergence, the correction is flushed into the FP64
// solution x and the true residual b - A x is recomputed in FP64 for every segment.  It replaces
// the recurrence residual of the segments that asked for the update (the others keep their
// recurrence untouched, so one problem of a batch does not disturb the Krylov space of another);
// the search direction is rebuilt from the replaced residual with the CG recurrence
// (k_replace_dir), so the Krylov information is kept -- unless the true residual exceeds the
// recurrence residual by more than 2x (accumulated drift), in which case that segment restarts
// from p = z.  Every segment whose true residual meets its target stops.  A segment within three
// decades of its target whose true residual gains less than 1% over max(2000, iterations / 2)
// iterations has reached the attainable accuracy of the recurrence and stops unconverged; so
// does, for a low-precision recurrence, a segment whose true residual realised less than half of
// the claimed decades at two consecutive replacements that followed a `delta` reduction.
// Convergence is decided on the FP64 residual only.  For T = double xh aliases x and rh aliases
// r64 (the true residual is then formed in q, free between iterations).
template <typename T>
int pcg_reliable(tdg_op* op, int prec, SegPlan const& sp, const double* b, double* x, T* xh, double* r64, T* rh,
                 CgVectors<T> v, double* t64, double* partial, double* scal, double rtol, double delta, int max_it,
                 int max_updates, bool graphs, cudaStream_t s, std::vector<double>& rn, std::vector<double>& bn,
                 int* iters, int* updates, bool* diverged) {
    constexpr bool kLow = !std::is_same_v<T, double>;
    // Iterations run in blocks.  The first block (kCheck iterations) is launched from the host; the
    // later ones replay a captured graph whose device loop (k_block_ctl) ends the block after the
    // iteration at which a segment asks for a reliable update (its recurrence residual met
    // max(delta rmax, tol) or is not finite) or after kBlock iterations; the host then reads the
    // scalars, so the updates happen at the same iterations as with a check after every iteration.
    // Without graphs (no stream, the distributed solve's host callbacks) the host checks after
    // every kCheck iterations.  The multigrid preconditioner is captured with its coarse solve's
    // own device loop inside the block.
    const bool mg = op->pc == TDG_PC_MG;
    const int kCheck = mg ? 1 : 8;
    constexpr int kBlock = 32;
    graphs = graphs && s != nullptr;
    if (graphs) TDG_TRY(ensure_loop(op));
    const int nseg = sp.nseg;
    if (max_updates <= 0) max_updates = 1 << 20;
    std::vector<double> tol(nseg), act(nseg), rmax(nseg), best(nseg), thr(nseg);
    auto threshold = [&](int i) {  // squared recurrence-residual norm that triggers an update
        const double t = std::max(delta * rmax[i], tol[i]);
        return t * t;
    };
    std::vector<int> stall(nseg, 0), poor(nseg, 0);
    std::vector<double> hs(static_cast<size_t>(nseg) * kScal);
    *iters = 0;
    *updates = 0;
    *diverged = false;
    // true residual, activity, recurrence start
    TDG_TRY(residual64(op, sp, b, x, r64, t64, partial, scal, rn, bn, s));
    bool any = false;
    for (int i = 0; i < nseg; ++i) {
        tol[i] = rtol * bn[i];
        act[i] = rn[i] > tol[i] ? 1.0 : 0.0;
        rmax[i] = rn[i];
        best[i] = rn[i];
        thr[i] = threshold(i);
        any = any || act[i] != 0.0;
    }
    if (!any) return 0;
    if constexpr (kLow) {
        k_scale_convert<double, T><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, r64, rh, scal, -1);
        k_fill<T><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, xh, T(0));
    }
    TDG_TRY(cg_start<T>(op, prec, sp, v, partial, scal, act, thr, s));
    cudaGraphExec_t exec = nullptr;
    long long lc[2] = {0, 0};  // kLoopIts, kLoopLimit of the next graph block
    int rc = 0;
    for (;;) {
        // one block of iterations
        const bool use_graph = graphs && *iters >= kCheck;
        if (use_graph && !exec) {
            cudaGraph_t graph = nullptr;
            rc = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess ? 0 : TDG_E_CUDA;
            if (rc == 0)
                rc = emit_while(op, s, 1u, [](cudaGraphConditionalHandle) { return 0; },
                                [&](cudaStream_t bs, cudaGraphConditionalHandle h) {
                                    TDG_TRY(cg_iteration<T>(op, prec, sp, xh, v, partial, scal, bs));
                                    k_block_ctl<<<1, 256, 0, bs>>>(scal, nseg, op->loop, h);
                                    return cudaGetLastError() == cudaSuccess ? 0 : fail(TDG_E_CUDA, "block control");
                                });
            cudaError_t ce = cudaStreamEndCapture(s, &graph);
            if (rc == 0 && ce == cudaSuccess) rc = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess ? 0 : TDG_E_CUDA;
            else if (rc == 0) rc = TDG_E_CUDA;
            if (graph) cudaGraphDestroy(graph);
            if (rc) {
                if (g_last_error.empty()) fail(rc, "capturing the device-looped CG block");
                break;
            }
        }
        int done = kCheck;
        if (exec) {
            lc[kLoopIts] = 0;
            lc[kLoopLimit] = std::min(kBlock, max_it - *iters);
            if (cudaMemcpyAsync(op->loop, lc, sizeof lc, cudaMemcpyHostToDevice, s) != cudaSuccess ||
                cudaGraphLaunch(exec, s) != cudaSuccess ||
                cudaMemcpyAsync(lc, op->loop, sizeof lc, cudaMemcpyDeviceToHost, s) != cudaSuccess) {
                rc = fail(TDG_E_CUDA, "graph launch");
                break;
            }
        } else {
            for (int i = 0; i < kCheck && rc == 0; ++i) rc = cg_iteration<T>(op, prec, sp, xh, v, partial, scal, s);
            if (rc) break;
        }
        // decide on reliable updates from the recurrence residuals
        if (cudaMemcpyAsync(hs.data(), scal, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            rc = fail(TDG_E_CUDA, "reading the Krylov scalars");
            break;
        }
        if (exec) done = static_cast<int>(lc[kLoopIts]);
        *iters += done;
        const bool last = *iters >= max_it;
        bool update = last;
        for (int i = 0; i < nseg; ++i) {
            double* sr = &hs[static_cast<size_t>(i) * kScal];
            sr[kRepl] = 0.0;
            if (sr[kActive] == 0.0) continue;
            const double rr = std::sqrt(sr[kRR]);
            if (last || !std::isfinite(rr) || rr <= delta * rmax[i] || rr <= tol[i]) {
                sr[kRepl] = 1.0;
                update = true;
            }
        }
        if (!update) continue;
        // reliable update: flush, FP64 residual of every segment into rt, replace the recurrence
        // residual of the flagged segments
        ++*updates;
        double* rt;
        if constexpr (kLow) {
            k_flush<T><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, x, xh);
            rt = r64;
        } else {
            rt = v.q;
        }
        if ((rc = residual64(op, sp, b, x, rt, t64, partial, scal, rn, bn, s))) break;
        any = false;
        for (int i = 0; i < nseg; ++i) {
            double* sr = &hs[static_cast<size_t>(i) * kScal];
            sr[kTmp] = 0.0;
            if (sr[kActive] == 0.0) continue;
            if (!std::isfinite(rn[i])) {
                *diverged = true;
                sr[kActive] = 0.0;
                continue;
            }
            if (rn[i] <= tol[i]) {
                sr[kActive] = 0.0;
                continue;
            }
            // stagnation near the target (CG residual norms are not monotone, so only within
            // three decades of it): no 1% gain of the true residual over the last
            // max(2000, iters / 2) iterations -- the attainable accuracy of this recurrence
            if (rn[i] < 0.99 * best[i]) {
                best[i] = rn[i];
                stall[i] = *iters;
            } else if (rn[i] <= 1e3 * tol[i] && *iters - stall[i] > std::max(2000, *iters / 2)) {
                sr[kActive] = 0.0;
                continue;
            }
            if (sr[kRepl] != 0.0) {
                const double rrec = std::sqrt(sr[kRR]);
                if constexpr (kLow) {
                    // twice in a row the recurrence claimed a `delta` reduction while the true
                    // residual realised less than half of its decades: near its attainable
                    // accuracy a low-precision iteration (about half the cost of an FP64 one)
                    // gains less than an FP64 iteration would, so the segment stops here (the
                    // caller continues it in FP64)
                    if (rrec <= delta * rmax[i] && rn[i] > std::sqrt(rrec * rmax[i])) {
                        if (++poor[i] >= 2) {
                            sr[kActive] = 0.0;
                            continue;
                        }
                    } else {
                        poor[i] = 0;
                    }
                }
                // the recurrence residual fell below the true one: its search direction no longer
                // matches the replaced residual, restart it (always with the flexible step, whose
                // direction recurrence the rebuild does not follow)
                if (mg || !(rn[i] <= 2.0 * rrec)) sr[kTmp] = 1.0;
                rmax[i] = rn[i];
                sr[kThr] = threshold(i);
            }
            any = true;
        }
        if (!any || *diverged || last || *updates >= max_updates) break;
        // restore the scalars (alpha / beta state, activity, replace and restart flags) that
        // residual64 overwrote; on the flagged segments replace the residual, recompute
        // z = M rh, rz and rr, and rebuild p (unless the segment restarts)
        if (cudaMemcpyAsync(scal, hs.data(), hs.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess) {
            rc = fail(TDG_E_CUDA, "writing the Krylov scalars");
            break;
        }
        k_replace_residual<double, T><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, rt, rh, scal);
        // z_new = M r into q (free between iterations; for T = double its true residual is
        // consumed above), rz_new, rr; the unflagged segments get z_new = z and are left as is
        if ((rc = precondition<T>(op, prec, rh, v.q, sp.op_nrhs, sp.op_ld, s))) break;
        if ((rc = dots<T>(sp, rh, v.q, rh, rh, partial, scal, kRZnew, kRR, s))) break;
        k_replace_dir<T><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, v.p, v.z, v.q, scal);
        k_cg_shift<<<(nseg + 127) / 128, 128, 0, s>>>(scal, nseg, 1);
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (rc) return rc;
    if constexpr (kLow) k_flush<T><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, x, xh);
    return cudaGetLastError() == cudaSuccess ? 0 : fail(TDG_E_CUDA, "solve kernels");
}

// Restarted flexible GMRES(m) with right preconditioning (gmres.cuh), FP64 vectors; prec selects
// the operator / preconditioner arithmetic (TDG_MIXED: FP32 arithmetic inside FP64 vectors).
// Every cycle starts from the true FP64 residual b - A x, so the Arnoldi process of an inexact
// (mixed) operator acts as an inner solver of an iterative refinement; a cycle of a segment ends
// when its residual estimate meets max(tol, inner * beta) (inner = 1e-6 for TDG_MIXED, about the
// FP32 operator's relative error; 0 for FP64), when its new basis vector vanishes, or after m
// steps.  The host looks at the per-segment activity every kCheck steps (every step under
// multigrid, which synchronises anyway) and ends a cycle early once no segment is active.
struct GmWork {
    double *V, *Z, *w, *dots, *H, *cs, *sn, *g, *y, *st, *gpart;
    int gstride;  // columns of gpart per chunk: m + 2
};

int fgmres(tdg_op* op, int prec, SegPlan const& sp, const double* b, double* x, size_t vec, int m, GmWork const& gw,
           double* r64, double* t64, double* partial, double* scal, double rtol, int max_it, cudaStream_t s,
           std::vector<double>& rn, std::vector<double>& bn, int* iters, int* cycles, bool* diverged) {
    const int nseg = sp.nseg;
    const int kCheck = op->pc == TDG_PC_MG ? 1 : 4;
    const double inner = prec == TDG_MIXED ? 1e-6 : 0.0;
    const int ds = m + 2;  // columns of gw.dots per segment
    std::vector<double> tol(nseg), hst(static_cast<size_t>(nseg) * kGm), hg(static_cast<size_t>(nseg) * (m + 1));
    std::vector<double> last(nseg, HUGE_VAL);
    int stagnant = 0;
    *iters = 0;
    *cycles = 0;
    *diverged = false;
    auto ngroups = [](int nv) { return (nv + kGmGroup - 1) / kGmGroup; };
    for (;;) {
        TDG_TRY(residual64(op, sp, b, x, r64, t64, partial, scal, rn, bn, s));
        bool any = false, progress = false;
        for (int i = 0; i < nseg; ++i) {
            if (!std::isfinite(rn[i])) *diverged = true;
            tol[i] = rtol * bn[i];
            const bool act = rn[i] > tol[i];
            any = any || act;
            if (act && rn[i] < 0.999 * last[i]) progress = true;
            last[i] = rn[i];
            double* sg = &hst[static_cast<size_t>(i) * kGm];
            std::fill(sg, sg + kGm, 0.0);
            sg[kGmBeta] = rn[i];
            sg[kGmActive] = act ? 1.0 : 0.0;
            sg[kGmTol] = std::max(tol[i], inner * rn[i]);
            sg[kGmEst] = rn[i];
            double* gs = &hg[static_cast<size_t>(i) * (m + 1)];
            std::fill(gs, gs + m + 1, 0.0);
            gs[0] = rn[i];
        }
        if (*diverged || !any || *iters >= max_it) break;
        stagnant = progress ? 0 : stagnant + 1;
        if (stagnant >= 3) break;  // three cycles without a 0.1 % gain: the attainable accuracy
        TDG_CUDA_TRY(cudaMemcpyAsync(gw.st, hst.data(), hst.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        TDG_CUDA_TRY(cudaMemcpyAsync(gw.g, hg.data(), hg.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        TDG_CUDA_TRY(cudaMemsetAsync(gw.H, 0, static_cast<size_t>(nseg) * (m + 1) * m * sizeof(double), s));
        k_gm_start<<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, r64, gw.V, gw.st);
        int j = 0;
        while (j < m && *iters < max_it) {
            double* vj = gw.V + static_cast<size_t>(j) * vec;
            double* zj = gw.Z + static_cast<size_t>(j) * vec;
            TDG_TRY(precondition<double>(op, prec, vj, zj, sp.op_nrhs, sp.op_ld, s));
            TDG_TRY(tdg_apply(op, prec, zj, gw.w, sp.op_nrhs, sp.op_ld, s));
            const int nv = j + 1;
            const int ng = ngroups(nv);
            // pass 1: h1 = V^T w, w -= V h1
            for (int q = 0; q < ng; ++q) {
                const int k0 = q * kGmGroup, nk = std::min(kGmGroup, nv - k0);
                k_gm_dots<kGmGroup><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, gw.V + static_cast<size_t>(k0) * vec,
                                                                      static_cast<int64_t>(vec), nk, gw.w, 0, gw.gpart,
                                                                      gw.gstride, k0);
            }
            k_gm_reduce<<<nseg, 64, 0, s>>>(gw.gpart, gw.gstride, sp.seg_chunk, nv, gw.dots, ds);
            k_gm_pass1<<<nseg, 64, 0, s>>>(gw.dots, ds, gw.H, m, j, nseg, gw.st);
            for (int q = 0; q < ng; ++q) {
                const int k0 = q * kGmGroup, nk = std::min(kGmGroup, nv - k0);
                k_gm_update<kGmGroup><<<sp.nchunks, kVecThreads, 0, s>>>(
                    sp.chunks, gw.V + static_cast<size_t>(k0) * vec, static_cast<int64_t>(vec), nk, gw.w, gw.dots + k0,
                    ds, gw.st, nullptr);
            }
            // pass 2: h2 = V^T w and w.w, H[:, j] += h2, rotations; v_{j+1} = (w - V h2) / h_{j+1,j}
            for (int q = 0; q < ng; ++q) {
                const int k0 = q * kGmGroup, nk = std::min(kGmGroup, nv - k0);
                k_gm_dots<kGmGroup><<<sp.nchunks, kVecThreads, 0, s>>>(sp.chunks, gw.V + static_cast<size_t>(k0) * vec,
                                                                      static_cast<int64_t>(vec), nk, gw.w,
                                                                      q == ng - 1 ? 1 : 0, gw.gpart, gw.gstride, k0);
            }
            k_gm_reduce<<<nseg, 64, 0, s>>>(gw.gpart, gw.gstride, sp.seg_chunk, nv + 1, gw.dots, ds);
            k_gm_pass2<<<(nseg + 127) / 128, 128, 0, s>>>(gw.dots, ds, gw.H, gw.cs, gw.sn, gw.g, m, j, nseg, gw.st);
            for (int q = 0; q < ng; ++q) {
                const int k0 = q * kGmGroup, nk = std::min(kGmGroup, nv - k0);
                k_gm_update<kGmGroup><<<sp.nchunks, kVecThreads, 0, s>>>(
                    sp.chunks, gw.V + static_cast<size_t>(k0) * vec, static_cast<int64_t>(vec), nk, gw.w, gw.dots + k0,
                    ds, gw.st, q == ng - 1 ? gw.V + static_cast<size_t>(j + 1) * vec : nullptr);
            }
            TDG_CUDA_TRY(cudaGetLastError());
            ++j;
            ++*iters;
            if (j % kCheck == 0 && j < m) {
                TDG_CUDA_TRY(cudaMemcpyAsync(hst.data(), gw.st, hst.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
                TDG_CUDA_TRY(cudaStreamSynchronize(s));
                bool live = false;
                for (int i = 0; i < nseg; ++i) live = live || hst[static_cast<size_t>(i) * kGm + kGmActive] != 0.0;
                if (!live) break;
            }
        }
        // x += Z y with y = R^-1 g over each segment's steps of this cycle
        k_gm_solve_y<<<(nseg + 127) / 128, 128, 0, s>>>(gw.H, gw.g, gw.y, m, nseg, gw.st);
        for (int q = 0; q < ngroups(j); ++q) {
            const int k0 = q * kGmGroup, nk = std::min(kGmGroup, j - k0);
            k_gm_update_x<kGmGroup><<<sp.nchunks, kVecThreads, 0, s>>>(
                sp.chunks, gw.Z + static_cast<size_t>(k0) * vec, static_cast<int64_t>(vec), nk, x, gw.y + k0, m);
        }
        TDG_CUDA_TRY(cudaGetLastError());
        ++*cycles;
    }
    return 0;
}

// Shared solve driver over a segment plan.  seg_rel (optional) receives each segment's final
// relative residual.
int solve_segments(tdg_op* op, const double* b, double* x, std::vector<int64_t> const& seg_begin,
                   std::vector<int64_t> const& seg_end, int op_nrhs, int64_t op_ld, size_t vec_entries,
                   const tdg_solve_opts* opts, tdg_solve_stats* stats, double* seg_rel, cudaStream_t s,
                   const DistCtx* dist = nullptr) {
    const int prec = opts->precision;
    if (prec != TDG_FP64 && prec != TDG_FP32 && prec != TDG_MIXED) return fail(TDG_E_INVALID, "bad precision");
    const bool gmres = opts->method == TDG_KSP_FGMRES;
    if (opts->method != TDG_KSP_CG && !gmres) return fail(TDG_E_INVALID, "method must be TDG_KSP_CG or TDG_KSP_FGMRES");
    const int m = opts->restart > 0 ? opts->restart : 30;
    if (gmres && prec == TDG_FP32) return fail(TDG_E_INVALID, "FGMRES runs with TDG_FP64 or TDG_MIXED");
    if (gmres && m > kGmMaxRestart) return fail(TDG_E_INVALID, "FGMRES restart length above 64");
    if (op->pc == TDG_PC_MG) {
        if (!op->mg.ready) return fail(TDG_E_STATE, "tdg_mg_setup must be called before a multigrid solve");
        if (prec == TDG_FP32) return fail(TDG_E_INVALID, "the multigrid preconditioner needs TDG_FP64 or TDG_MIXED");
    } else if (!op->inv || (prec != TDG_MIXED && op->inv_precision != prec)) {
        // FP64 needs FP64 inverses, FP32 needs FP32 inverses, MIXED takes either
        return fail(TDG_E_STATE, "tdg_bjacobi_setup must be called with the solve precision");
    }
    TDG_TRY(ensure_uploaded(op, TDG_FP64));
    if (prec != TDG_FP64) TDG_TRY(ensure_uploaded(op, TDG_FP32));
    std::memset(stats, 0, sizeof(*stats));
    if (op->pc == TDG_PC_MG && op->loop)  // a divergence flag left by an earlier failed call
        TDG_CUDA_TRY(cudaMemsetAsync(op->loop + kCoarseDiverged, 0, sizeof(long long), s));

    std::vector<Chunk> hchunks;
    std::vector<int> hseg;
    plan_chunks(seg_begin, seg_end, hchunks, hseg);
    const int nseg = static_cast<int>(seg_begin.size());
    const size_t vec = vec_entries;
    // every carve below is rounded up to 256 bytes: one 256-byte unit of slack per carve (9 FP64
    // carves, 5 more for the FP32 vectors)
    size_t need = 5 * vec * sizeof(double) + hchunks.size() * (2 * sizeof(double) + sizeof(Chunk)) +
                  (hseg.size()) * sizeof(int) + static_cast<size_t>(nseg) * kScal * sizeof(double) + 9 * 256;
    if (prec == TDG_FP32) need += 5 * vec * sizeof(float) + 5 * 256;
    // FGMRES: V (m + 1 vectors), Z (m), w; per segment the dots, H, rotations, g, y, state; chunk
    // partials of the multi-dots (m + 2 columns)
    const size_t gm_seg = static_cast<size_t>(nseg) *
                          ((m + 2) + static_cast<size_t>(m + 1) * m + 2 * m + (m + 1) + m + kGm);
    if (gmres)
        need += (2 * static_cast<size_t>(m) + 2) * vec * sizeof(double) + gm_seg * sizeof(double) +
                hchunks.size() * (m + 2) * sizeof(double) + 12 * 256;
    if (op->ws_bytes < need) {
        op->arena_ws.release();
        op->ws = nullptr;
        op->ws_bytes = 0;
        unsigned char* w = nullptr;
        TDG_CUDA_TRY(op->arena_ws.alloc(&w, need));
        op->ws = w;
        op->ws_bytes = need;
    }
    unsigned char* w = static_cast<unsigned char*>(op->ws);
    auto take = [&](size_t bytes) {
        unsigned char* p = w;
        w += (bytes + 255) / 256 * 256;
        return p;
    };
    double* r64 = reinterpret_cast<double*>(take(vec * sizeof(double)));
    double* z64 = reinterpret_cast<double*>(take(vec * sizeof(double)));
    double* p64 = reinterpret_cast<double*>(take(vec * sizeof(double)));
    double* q64 = reinterpret_cast<double*>(take(vec * sizeof(double)));
    double* t64 = reinterpret_cast<double*>(take(vec * sizeof(double)));
    double* partial = reinterpret_cast<double*>(take(hchunks.size() * 2 * sizeof(double)));
    Chunk* dchunks = reinterpret_cast<Chunk*>(take(hchunks.size() * sizeof(Chunk)));
    int* dseg = reinterpret_cast<int*>(take(hseg.size() * sizeof(int)));
    double* scal = reinterpret_cast<double*>(take(static_cast<size_t>(nseg) * kScal * sizeof(double)));
    TDG_CUDA_TRY(cudaMemcpyAsync(dchunks, hchunks.data(), hchunks.size() * sizeof(Chunk), cudaMemcpyHostToDevice, s));
    TDG_CUDA_TRY(cudaMemcpyAsync(dseg, hseg.data(), hseg.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    SegPlan sp;
    sp.nseg = nseg;
    sp.nchunks = static_cast<int>(hchunks.size());
    sp.chunks = dchunks;
    sp.seg_chunk = dseg;
    sp.op_nrhs = op_nrhs;
    sp.op_ld = op_ld;
    sp.dist = dist;

    cudaEvent_t ev0, ev1;
    TDG_CUDA_TRY(cudaEventCreate(&ev0));
    TDG_CUDA_TRY(cudaEventCreate(&ev1));
    TDG_CUDA_TRY(cudaEventRecord(ev0, s));

    const int max_it = opts->max_iterations > 0 ? opts->max_iterations : 10000;
    const double rtol = opts->rtol > 0 ? opts->rtol : 1e-10;
    const bool graphs = opts->use_graphs != 0 && !dist;  // the callbacks are host code: no capture
    std::vector<double> rn, bn;
    int total_it = 0, updates = 0;
    bool diverged = false;
    auto rel_of = [&](int i) { return bn[i] > 0 ? rn[i] / bn[i] : 0.0; };
    if (gmres) {
        GmWork gw;
        gw.V = reinterpret_cast<double*>(take((m + 1) * vec * sizeof(double)));
        gw.Z = reinterpret_cast<double*>(take(static_cast<size_t>(m) * vec * sizeof(double)));
        gw.w = reinterpret_cast<double*>(take(vec * sizeof(double)));
        gw.dots = reinterpret_cast<double*>(take(static_cast<size_t>(nseg) * (m + 2) * sizeof(double)));
        gw.H = reinterpret_cast<double*>(take(static_cast<size_t>(nseg) * (m + 1) * m * sizeof(double)));
        gw.cs = reinterpret_cast<double*>(take(static_cast<size_t>(nseg) * m * sizeof(double)));
        gw.sn = reinterpret_cast<double*>(take(static_cast<size_t>(nseg) * m * sizeof(double)));
        gw.g = reinterpret_cast<double*>(take(static_cast<size_t>(nseg) * (m + 1) * sizeof(double)));
        gw.y = reinterpret_cast<double*>(take(static_cast<size_t>(nseg) * m * sizeof(double)));
        gw.st = reinterpret_cast<double*>(take(static_cast<size_t>(nseg) * kGm * sizeof(double)));
        gw.gstride = m + 2;
        gw.gpart = reinterpret_cast<double*>(take(hchunks.size() * (m + 2) * sizeof(double)));
        int cycles = 0;
        TDG_TRY(fgmres(op, prec, sp, b, x, vec, m, gw, r64, t64, partial, scal, rtol, max_it, s, rn, bn, &total_it,
                       &cycles, &diverged));
        updates = cycles;
    } else if (prec == TDG_FP64 || prec == TDG_MIXED) {
        // FP64 recurrence: the recurrence residual is r64 itself and x accumulates directly; the
        // mixed mode applies the operator in FP32 arithmetic and the FP32 inverses, so its
        // recurrence residual drifts from the true one and is replaced more often.  Multigrid
        // needs few iterations per decade and restarts at every replacement, so it replaces
        // rarely (FP64: drift-free up to the convergence test)
        const double delta = opts->inner_rtol > 0 ? opts->inner_rtol
                             : op->pc == TDG_PC_MG ? (prec == TDG_FP64 ? 1e-4 : 1e-2)
                                                    : 0.1;
        TDG_TRY((pcg_reliable<double>(op, prec, sp, b, x, x, r64, r64, {r64, z64, p64, q64}, t64, partial, scal,
                                      rtol, delta, max_it, opts->max_outer, graphs, s, rn, bn, &total_it, &updates,
                                      &diverged)));
    } else {
        float* xh = reinterpret_cast<float*>(take(vec * sizeof(float)));
        float* r32 = reinterpret_cast<float*>(take(vec * sizeof(float)));
        float* z32 = reinterpret_cast<float*>(take(vec * sizeof(float)));
        float* p32 = reinterpret_cast<float*>(take(vec * sizeof(float)));
        float* q32 = reinterpret_cast<float*>(take(vec * sizeof(float)));
        const double delta = opts->inner_rtol > 0 ? opts->inner_rtol : 0.1;
        TDG_TRY((pcg_reliable<float>(op, TDG_FP32, sp, b, x, xh, r64, r32, {r32, z32, p32, q32}, t64, partial, scal,
                                     rtol, delta, max_it, opts->max_outer, graphs, s, rn, bn, &total_it, &updates,
                                     &diverged)));
        // problems still above the target (the FP32 recurrence stalled) continue in FP64 with the
        // FP32 inverses as preconditioner
        bool rest = false;
        for (int i = 0; i < nseg && !diverged; ++i) rest = rest || rel_of(i) > rtol;
        if (rest && !diverged && total_it < max_it) {
            int it2 = 0, up2 = 0;
            TDG_TRY((pcg_reliable<double>(op, TDG_FP64, sp, b, x, x, r64, r64, {r64, z64, p64, q64}, t64, partial,
                                          scal, rtol, 1e-2, max_it - total_it, opts->max_outer, graphs, s, rn, bn,
                                          &it2, &up2, &diverged)));
            total_it += it2;
            updates += up2;
            stats->fp64_iterations = it2;
        }
    }
    stats->outer = updates;
    if (!diverged) TDG_TRY(residual64(op, sp, b, x, r64, t64, partial, scal, rn, bn, s));

    TDG_CUDA_TRY(cudaEventRecord(ev1, s));
    TDG_CUDA_TRY(cudaEventSynchronize(ev1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    double worst = 0.0;
    if (!diverged)
        for (int i = 0; i < nseg; ++i) {
            worst = std::max(worst, rel_of(i));
            if (seg_rel) seg_rel[i] = rel_of(i);
        }
    stats->iterations = total_it;
    stats->rel_residual = diverged ? NAN : worst;
    stats->seconds = ms * 1e-3;
    stats->converged = (!diverged && worst <= rtol) ? 1 : 0;
    if (op->pc == TDG_PC_MG) TDG_TRY(mg_check_coarse(op, s));
    if (diverged) return fail(TDG_E_DIVERGED, "non-finite residual in the Krylov iteration");
    for (int* word : {op->tgeo.status, op->tc32.status})
        if (word) {  // a bounded wait of a pipelined kernel that ran out makes the solve invalid
            int st = 0;
            TDG_CUDA_TRY(cudaMemcpy(&st, word, sizeof st, cudaMemcpyDeviceToHost));
            if (st) return fail(TDG_E_TIMEOUT, "a bounded wait of an apply kernel ran out");
        }
    if (!stats->converged) return fail(TDG_E_DIVERGED, "iteration limit reached before the residual target");
    return 0;
}

}  // namespace

extern "C" int tdg_solve(tdg_op* op, const double* b, double* x, int nrhs, int64_t ld, const tdg_solve_opts* opts,
                         tdg_solve_stats* stats, void* stream) {
    if (!op || !b || !x || !opts || !stats) return fail(TDG_E_INVALID, "null argument");
    auto const& h = op->h;
    const int64_t n = h.E * h.bs;
    if (nrhs < 1 || ld < n) return fail(TDG_E_INVALID, "nrhs < 1 or ld < E * bs");
    std::vector<int64_t> sb(nrhs), se(nrhs);
    for (int r = 0; r < nrhs; ++r) {
        sb[r] = r * ld;
        se[r] = r * ld + n;
    }
    return solve_segments(op, b, x, sb, se, nrhs, ld, static_cast<size_t>(nrhs) * ld, opts, stats, nullptr,
                          static_cast<cudaStream_t>(stream));
}

extern "C" int tdg_solve_distributed(tdg_op* op, const double* b, double* x, int64_t owned_elements,
                                     const tdg_solve_opts* opts, tdg_solve_stats* stats, tdg_exchange_fn exchange,
                                     tdg_allreduce_fn allreduce, void* ctx, void* stream) {
    if (!op || !b || !x || !opts || !stats || !exchange || !allreduce) return fail(TDG_E_INVALID, "null argument");
    auto const& h = op->h;
    if (owned_elements < 0 || owned_elements > h.E) return fail(TDG_E_INVALID, "owned_elements outside [0, E]");
    if (opts->precision != TDG_FP64 && opts->precision != TDG_MIXED)
        return fail(TDG_E_INVALID, "a distributed solve runs with TDG_FP64 or TDG_MIXED");
    if (opts->method != TDG_KSP_CG) return fail(TDG_E_INVALID, "a distributed solve runs CG");
    if (op->pc != TDG_PC_BJACOBI)
        return fail(TDG_E_INVALID, "a distributed solve is preconditioned by block Jacobi (element-local)");
    const DistCtx dc{exchange, allreduce, ctx};
    std::vector<int64_t> sb{0}, se{owned_elements * h.bs};
    return solve_segments(op, b, x, sb, se, 1, h.E * h.bs, static_cast<size_t>(h.E) * h.bs, opts, stats, nullptr,
                          static_cast<cudaStream_t>(stream), &dc);
}

extern "C" int tdg_solve_segmented(tdg_op* op, const double* b, double* x, int nseg, const int64_t* seg_elem_offset,
                                   const tdg_solve_opts* opts, tdg_solve_stats* stats, double* seg_rel_residual,
                                   void* stream) {
    if (!op || !b || !x || !opts || !stats || !seg_elem_offset || nseg < 1) return fail(TDG_E_INVALID, "bad argument");
    auto const& h = op->h;
    if (seg_elem_offset[0] != 0 || seg_elem_offset[nseg] != h.E)
        return fail(TDG_E_INVALID, "segments must cover the elements [0, E)");
    std::vector<int64_t> sb(nseg), se(nseg);
    for (int i = 0; i < nseg; ++i) {
        if (seg_elem_offset[i + 1] < seg_elem_offset[i]) return fail(TDG_E_INVALID, "segment offsets must not decrease");
        sb[i] = seg_elem_offset[i] * h.bs;
        se[i] = seg_elem_offset[i + 1] * h.bs;
    }
    return solve_segments(op, b, x, sb, se, 1, h.E * h.bs, static_cast<size_t>(h.E) * h.bs, opts, stats,
                          seg_rel_residual, static_cast<cudaStream_t>(stream));
}

// ---- p-multigrid ---------------------------------------------------------------------------------

extern "C" int tdg_mg_setup(tdg_op* op, const tdg_mg_opts* opts, void* stream) {
    if (!op) return fail(TDG_E_INVALID, "null operator");
    tdg_mg_opts o{};
    if (opts) {
        o = *opts;
    } else {
        o.strategy = TDG_MG_LOGARITHMIC;
        o.coarse_degree = 1;
        o.coarse_space = TDG_MG_COARSE_P1;
    }
    try {
        return mg_setup(op, o, static_cast<cudaStream_t>(stream));
    } catch (std::exception const& e) {
        op->mg.ready = false;
        return fail(TDG_E_INVALID, std::string("multigrid set-up: ") + e.what());
    }
}

extern "C" int tdg_mg_apply(tdg_op* op, const double* r, double* z, int nrhs, int64_t ld, void* stream) {
    if (!op || !r || !z) return fail(TDG_E_INVALID, "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    TDG_TRY(mg_apply(op, r, z, nrhs, ld, s));
    return mg_check_coarse(op, s);
}

extern "C" int tdg_set_preconditioner(tdg_op* op, int pc) {
    if (!op) return fail(TDG_E_INVALID, "null operator");
    if (pc != TDG_PC_BJACOBI && pc != TDG_PC_MG) return fail(TDG_E_INVALID, "unknown preconditioner");
    op->pc = pc;
    return 0;
}

extern "C" int tdg_mg_info(tdg_op* op, int* nlevels, int max_levels, int* degrees, int* block_sizes,
                           double* lambda_max, int64_t* coarse_its) {
    if (!op) return fail(TDG_E_INVALID, "null operator");
    auto const& mg = op->mg;
    if (!mg.ready) return fail(TDG_E_STATE, "tdg_mg_setup not called");
    const int nl = static_cast<int>(mg.lv.size());
    if (nlevels) *nlevels = nl;
    for (int l = 0; l < std::min(nl, max_levels); ++l) {
        if (degrees) degrees[l] = mg.lv[static_cast<size_t>(l)].degree;
        if (block_sizes) block_sizes[l] = mg.lv[static_cast<size_t>(l)].bs;
        if (lambda_max) lambda_max[l] = mg.lv[static_cast<size_t>(l)].lmax;
    }
    if (coarse_its) {
        long long total = 0;
        if (op->loop) TDG_CUDA_TRY(cudaMemcpy(&total, op->loop + kCoarseTotal, sizeof total, cudaMemcpyDeviceToHost));
        *coarse_its = total;
    }
    return 0;
}

extern "C" int tdg_mg_level_matrix(tdg_op* op, int level, double* blocks, int32_t* nbr) {
    if (!op) return fail(TDG_E_INVALID, "null operator");
    auto const& mg = op->mg;
    if (!mg.ready) return fail(TDG_E_STATE, "tdg_mg_setup not called");
    if (level < 0 || level + 1 >= static_cast<int>(mg.lv.size()))
        return fail(TDG_E_INVALID, "level must be a coarse (block-sparse) level");
    auto const& L = mg.lv[static_cast<size_t>(level)];
    const size_t E = static_cast<size_t>(op->h.E);
    TDG_CUDA_TRY(cudaDeviceSynchronize());
    if (blocks)
        TDG_CUDA_TRY(cudaMemcpy(blocks, L.A, sizeof(double) * E * mg.NB * L.bs * L.bs, cudaMemcpyDeviceToHost));
    if (nbr) TDG_CUDA_TRY(cudaMemcpy(nbr, mg.nbr, sizeof(int32_t) * E * mg.NB, cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int tdg_mg_level_degrees(int strategy, int coarse_degree, int degree, int* degrees) {
    try {
        std::vector<int> d = mg_level_degrees(strategy, coarse_degree, degree);
        if (degrees) std::copy(d.begin(), d.end(), degrees);
        return static_cast<int>(d.size());
    } catch (std::exception const& e) {
        return fail(TDG_E_INVALID, e.what());
    }
}

extern "C" int tdg_mg_colouring(const tdg_op* op, int32_t* colour, int* ncolours) {
    if (!op || !colour || !ncolours) return fail(TDG_E_INVALID, "null argument");
    std::vector<int32_t> nbr = element_neighbours(op->h);
    std::vector<int32_t> col = distance2_colouring(nbr, op->h.E, 1 + op->h.nfaces, ncolours);
    std::copy(col.begin(), col.end(), colour);
    return 0;
}

extern "C" int tdg_mg_vertex_numbering(const tdg_op* op, int32_t* vid, int64_t* nv) {
    if (!op || !vid || !nv) return fail(TDG_E_INVALID, "null argument");
    std::vector<int32_t> v = vertex_numbering(op->h, nv);
    std::copy(v.begin(), v.end(), vid);
    return 0;
}

extern "C" int tdg_project(const tdg_op* op, const double* U_Q, double* y) {
    if (!op || !U_Q || !y) return fail(TDG_E_INVALID, "null argument");
    op->h.project(U_Q, y);
    return 0;
}

extern "C" int tdg_evaluate(const tdg_op* op, const double* x, int np, const double* points, double* out) {
    if (!op || !x || !points || !out || np < 1) return fail(TDG_E_INVALID, "bad argument");
    op->h.evaluate(x, np, points, out);
    return 0;
}

extern "C" int tdg_rule_coords(const tdg_op* op, int np, const double* points, double* out) {
    if (!op || !points || !out || np < 1) return fail(TDG_E_INVALID, "bad argument");
    op->h.rule_coords(np, points, out);
    return 0;
}

extern "C" int tdg_error_l2(const tdg_op* op, const double* x, int np, const double* points, const double* weights,
                            const double* ref, double* out) {
    if (!op || !x || !points || !weights || !ref || !out || np < 1) return fail(TDG_E_INVALID, "bad argument");
    *out = op->h.error_l2(x, np, points, weights, ref);
    return 0;
}

extern "C" int tdg_error_h1_semi(const tdg_op* op, const double* x, int np, const double* points,
                                 const double* weights, const double* refgrad, double* out) {
    if (!op || !x || !points || !weights || !refgrad || !out || np < 1) return fail(TDG_E_INVALID, "bad argument");
    *out = op->h.error_h1_semi(x, np, points, weights, refgrad);
    return 0;
}

extern "C" int tdg_mg_p1_embedding(int dim, int kind, int degree, double* out) {
    if (!out || dim < 2 || dim > 3 || degree < 1 || (kind != TDG_POISSON && kind != TDG_ELASTICITY))
        return fail(TDG_E_INVALID, "bad argument");
    try {
        Dense T = linear_to_space(dim, kind, degree);
        std::copy(T.a.begin(), T.a.end(), out);
        return 0;
    } catch (std::exception const& e) {
        return fail(TDG_E_INVALID, e.what());
    }
}

extern "C" int tdg_mg_interpolation(int dim, int kind, int n_to, int n_from, double* out) {
    if (!out || dim < 2 || dim > 3 || (kind != TDG_POISSON && kind != TDG_ELASTICITY))
        return fail(TDG_E_INVALID, "bad argument");
    try {
        Dense I = interpolation_matrix(dim, kind, n_to, n_from);
        std::copy(I.a.begin(), I.a.end(), out);
        return 0;
    } catch (std::exception const& e) {
        return fail(TDG_E_INVALID, e.what());
    }
}

// ------------------------------------------------------------------------------------------------
// fault coupling (Green's functions)
// ------------------------------------------------------------------------------------------------

#include "kernels/fault.cuh"

struct tdg_fault {
    tdg_op* op = nullptr;
    DevArena arena;
    DevFault d;
};

extern "C" int tdg_fault_create(tdg_op* op, int64_t num_fault, const int64_t* fault_facets, const double* ref_normal,
                                tdg_fault** out) {
    if (!op || !fault_facets || !ref_normal || !out || num_fault < 1) return fail(TDG_E_INVALID, "bad argument");
    auto const& h = op->h;
    if (h.kind != 0) return fail(TDG_E_INVALID, "fault coupling is implemented for the Poisson operator");
    if (!h.has_material) return fail(TDG_E_STATE, "tdg_set_material has not been called");
    const int D = h.D, nq = h.nq;
    if (nq > kFaultMaxQ) return fail(TDG_E_INVALID, "too many facet quadrature points for the fault kernels");
    try {
        // fault basis: nodal warp & blend of degree N on the (D-1)-simplex (RateAndStateBase::Space)
        RefSpace fs = RefSpace::nodal(D - 1, h.N, warp_blend_nodes(D - 1, h.N));
        const int nbf = fs.num_basis();
        Dense eq = fs.eval(h.fct_x);  // [nbf][nq]
        std::vector<double> e_q(eq.a.begin(), eq.a.end());
        std::vector<int4> info(num_fault);
        std::vector<double> sign(static_cast<size_t>(num_fault) * nq), normal(static_cast<size_t>(num_fault) * D * nq);
        std::vector<double> minv(static_cast<size_t>(num_fault) * nbf * nbf);
        for (int64_t i = 0; i < num_fault; ++i) {
            const int64_t f = fault_facets[i];
            if (f < 0 || f >= h.F) return fail(TDG_E_INVALID, "fault facet out of range");
            info[i] = make_int4(static_cast<int>(f), static_cast<int>(h.up[2 * f]), static_cast<int>(h.up[2 * f + 1]),
                                h.loc[2 * f] | (h.loc[2 * f + 1] << 8));
            std::vector<double> nl(nq);
            for (int q = 0; q < nq; ++q) {
                double dot = 0.0, n2 = 0.0;
                for (int d = 0; d < D; ++d) {
                    const double v = h.fN[(static_cast<size_t>(f) * D + d) * nq + q];
                    dot += ref_normal[d] * v;
                    n2 += v * v;
                }
                if (std::fabs(dot) < 10000.0 * std::numeric_limits<double>::epsilon())
                    return fail(TDG_E_INVALID, "fault normal and reference normal are almost perpendicular");
                const double s = dot < 0 ? -1.0 : 1.0;
                sign[static_cast<size_t>(i) * nq + q] = s;
                for (int d = 0; d < D; ++d)
                    normal[(static_cast<size_t>(i) * D + d) * nq + q] = s * h.fN[(static_cast<size_t>(f) * D + d) * nq + q];
                nl[q] = std::sqrt(n2);
            }
            Dense m(nbf, nbf);
            for (int a = 0; a < nbf; ++a)
                for (int b = 0; b < nbf; ++b) {
                    double s = 0.0;
                    for (int q = 0; q < nq; ++q) s += h.w[q] * nl[q] * eq(a, q) * eq(b, q);
                    m(a, b) = s;
                }
            Dense mi = invert(m);
            std::copy(mi.a.begin(), mi.a.end(), &minv[static_cast<size_t>(i) * nbf * nbf]);
        }
        TDG_TRY(ensure_uploaded(op, TDG_FP64));
        auto* fl = new tdg_fault();
        fl->op = op;
        fl->d.nfault = static_cast<int>(num_fault);
        fl->d.nbf = nbf;
        cudaError_t e = cudaSuccess;
        if (e == cudaSuccess) e = fl->arena.upload(&fl->d.info, info);
        if (e == cudaSuccess) e = fl->arena.upload(&fl->d.sign, sign);
        if (e == cudaSuccess) e = fl->arena.upload(&fl->d.normal, normal);
        if (e == cudaSuccess) e = fl->arena.upload(&fl->d.minv, minv);
        if (e == cudaSuccess) e = fl->arena.upload(&fl->d.e_q, e_q);
        if (e != cudaSuccess) {
            delete fl;
            return fail(TDG_E_CUDA, std::string("fault upload: ") + cudaGetErrorString(e));
        }
        *out = fl;
        return 0;
    } catch (std::exception const& ex) {
        return fail(TDG_E_INVALID, ex.what());
    }
}

extern "C" void tdg_fault_destroy(tdg_fault* fault) { delete fault; }

extern "C" int tdg_fault_sizes(const tdg_fault* fault, int64_t out[2]) {
    if (!fault || !out) return fail(TDG_E_INVALID, "null argument");
    out[0] = fault->d.nfault;
    out[1] = fault->d.nbf;
    return 0;
}

extern "C" int tdg_fault_slip_rhs(tdg_fault* fault, const double* slip, int64_t ld_slip, double* b, int nrhs,
                                  int64_t ld, void* stream) {
    if (!fault || !slip || !b) return fail(TDG_E_INVALID, "null argument");
    auto const& h = fault->op->h;
    if (ld < h.E * h.bs || ld_slip < static_cast<int64_t>(fault->d.nfault) * fault->d.nbf)
        return fail(TDG_E_INVALID, "leading dimension too small");
    TDG_TRY(ensure_uploaded(fault->op, TDG_FP64));
    int rc = launch_fault(h.D, h.N, false, fault->op->op64, fault->d, nullptr, 0, slip, ld_slip, b, ld, nrhs,
                          static_cast<cudaStream_t>(stream));
    return rc ? fail(rc, "fault rhs launch failed") : 0;
}

extern "C" int tdg_fault_traction(tdg_fault* fault, const double* u, int64_t ld, const double* slip, int64_t ld_slip,
                                  double* traction, int64_t ld_t, int nrhs, void* stream) {
    if (!fault || !u || !traction) return fail(TDG_E_INVALID, "null argument");
    auto const& h = fault->op->h;
    const int64_t nt = static_cast<int64_t>(fault->d.nfault) * fault->d.nbf;
    if (ld < h.E * h.bs || ld_t < nt || (slip && ld_slip < nt)) return fail(TDG_E_INVALID, "leading dimension too small");
    TDG_TRY(ensure_uploaded(fault->op, TDG_FP64));
    int rc = launch_fault(h.D, h.N, true, fault->op->op64, fault->d, u, ld, slip, ld_slip, traction, ld_t, nrhs,
                          static_cast<cudaStream_t>(stream));
    return rc ? fail(rc, "fault traction launch failed") : 0;
}

extern "C" int tdg_gf_traction_update(int64_t n, int64_t m, const double* G, int64_t ldg, const double* S,
                                      int64_t lds, int k, const double* t_boundary, double time, double* out,
                                      int64_t ldo, void* stream) {
    if (!G || !S || !out || n < 0 || m < 0 || k < 0) return fail(TDG_E_INVALID, "null argument or negative size");
    if (n == 0 || k == 0) return 0;
    if (ldg < m || (k > 1 && (lds < m || ldo < n))) return fail(TDG_E_INVALID, "leading dimension too small");
    if (m == 0) return fail(TDG_E_INVALID, "G has no columns");
    if ((out < S + lds * (k - 1) + m && S < out + ldo * (k - 1) + n))
        return fail(TDG_E_INVALID, "out must not overlap the slip states");
    int rc = launch_gf_traction(n, m, G, ldg, S, lds, k, t_boundary, time, out, ldo, static_cast<cudaStream_t>(stream));
    if (rc == TDG_E_INVALID) return fail(rc, "G has too many columns for the shared-memory slip states (m <= 7264)");
    return rc ? fail(rc, std::string("traction update launch failed: ") + cudaGetErrorString(cudaGetLastError())) : 0;
}

// ------------------------------------------------------------------------------------------------
// adjoint gradient with respect to per-element Lame parameters
// ------------------------------------------------------------------------------------------------

namespace {
// Host part of the Lame gradient: checks that the material is constant per element and fills
// dpen = [F][4] penalty derivatives (d/dlam, d/dmu of each side's contribution) followed by
// [E][2] element (lam, mu), the layout adjoint_lame_kernel reads.
int lame_gradient_inputs(tdg_op* op, std::vector<double>& dpen) {
    auto const& h = op->h;
    if (h.kind != 1) return fail(TDG_E_INVALID, "the Lame gradient needs an elasticity operator");
    if (!h.has_material) return fail(TDG_E_STATE, "no material");
    const int nm = h.mat_space.num_basis();
    const int D = h.D;
    // piecewise-constant material: every nodal coefficient of an element equals its mean
    std::vector<double> lam(h.E), mu(h.E);
    for (int64_t e = 0; e < h.E; ++e) {
        const double* a = &h.mat_nodal[(static_cast<size_t>(e) * 2 + 0) * nm];
        const double* b = &h.mat_nodal[(static_cast<size_t>(e) * 2 + 1) * nm];
        double sa = 0.0, sb = 0.0;
        for (int i = 0; i < nm; ++i) {
            sa += a[i];
            sb += b[i];
        }
        lam[e] = sa / nm;
        mu[e] = sb / nm;
        for (int i = 0; i < nm; ++i)
            if (std::fabs(a[i] - lam[e]) > 1e-10 * std::fabs(lam[e]) || std::fabs(b[i] - mu[e]) > 1e-10 * std::fabs(mu[e]))
                return fail(TDG_E_INVALID, "material is not constant per element");
    }
    // penalty derivatives (Elasticity::prepare_penalty with c0 = 2 mu, c1 = D lam + 2 mu):
    // p_s = K_s c1^2 / c0, K_s = (D + 1) c_{N-1} |f| / |E_s|; interior pen = (p0 + p1) / 4
    const double cN1 = h.N * (h.N - 1.0 + D) / static_cast<double>(D);
    dpen.assign(static_cast<size_t>(h.F) * 4 + static_cast<size_t>(h.E) * 2, 0.0);
    for (int64_t f = 0; f < h.F; ++f) {
        const bool interior = h.up[2 * f] != h.up[2 * f + 1];
        for (int s = 0; s < (interior ? 2 : 1); ++s) {
            const int64_t e = h.up[2 * f + s];
            const double K = (D + 1) * cN1 * h.area[f] / h.volume[e];
            const double c0 = 2.0 * mu[e], c1 = D * lam[e] + 2.0 * mu[e];
            const double scale = interior ? 0.25 : 1.0;
            dpen[static_cast<size_t>(f) * 4 + 2 * s + 0] = scale * K * 2.0 * c1 * D / c0;
            dpen[static_cast<size_t>(f) * 4 + 2 * s + 1] = scale * K * (4.0 * c1 / c0 - 2.0 * c1 * c1 / (c0 * c0));
        }
    }
    for (int64_t e = 0; e < h.E; ++e) {
        dpen[static_cast<size_t>(h.F) * 4 + 2 * e] = lam[e];
        dpen[static_cast<size_t>(h.F) * 4 + 2 * e + 1] = mu[e];
    }
    return 0;
}
}  // namespace

extern "C" int tdg_adjoint_lame_gradient(tdg_op* op, const double* u, const double* p, const double* bc_q,
                                         double* grad, void* stream) {
    if (!op || !u || !p || !grad) return fail(TDG_E_INVALID, "null argument");
    auto const& h = op->h;
    std::vector<double> dpen;
    TDG_TRY(lame_gradient_inputs(op, dpen));
    TDG_TRY(ensure_uploaded(op, TDG_FP64));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* d = nullptr;
    TDG_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d), dpen.size() * sizeof(double), s));
    TDG_CUDA_TRY(cudaMemcpyAsync(d, dpen.data(), dpen.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    int rc = launch_adjoint_lame(h.D, h.N, op->op64, u, p, bc_q, d, grad, s);
    cudaFreeAsync(d, s);
    TDG_CUDA_TRY(cudaStreamSynchronize(s));
    return rc ? fail(rc, "adjoint gradient launch failed") : 0;
}

// Allocation-free variant: the penalty derivatives go through the fixed device scratch of
// adjoint.cu, staged in chunks through a static host buffer; the operator's FP64 data must already
// be resident (its upload resolved the scratch address and loaded the kernel).
namespace {
constexpr size_t kNoallocStage = size_t(1) << 16;  // doubles; a multiple of 4 (facet) and 2 (element)
double g_noalloc_stage[kNoallocStage];
std::mutex g_noalloc_mutex;

// lam, mu of element e: the mean of its nodal coefficients (constant per element, checked).
inline void element_lame(HostOperator const& h, int nm, int64_t e, double& lam, double& mu) {
    const double* a = &h.mat_nodal[(static_cast<size_t>(e) * 2 + 0) * nm];
    const double* b = &h.mat_nodal[(static_cast<size_t>(e) * 2 + 1) * nm];
    double sa = 0.0, sb = 0.0;
    for (int i = 0; i < nm; ++i) {
        sa += a[i];
        sb += b[i];
    }
    lam = sa / nm;
    mu = sb / nm;
}
}  // namespace

extern "C" int tdg_adjoint_lame_gradient_noalloc(tdg_op* op, const double* u, const double* p, const double* bc_q,
                                                 double* grad, void* stream) {
    if (!op || !u || !p || !grad) return fail(TDG_E_INVALID, "null argument");
    auto const& h = op->h;
    if (h.kind != 1) return fail(TDG_E_INVALID, "the Lame gradient needs an elasticity operator");
    if (!h.has_material) return fail(TDG_E_STATE, "no material");
    const size_t nfct = static_cast<size_t>(h.F) * 4;
    const size_t need = nfct + static_cast<size_t>(h.E) * 2;
    if (need > kAdjointScratchDoubles) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "mesh needs %zu doubles of scratch (4 per facet + 2 per element), the fixed scratch "
                      "holds %zu (8 MiB); use tdg_adjoint_lame_gradient",
                      need, kAdjointScratchDoubles);
        return fail(TDG_E_INVALID, msg);
    }
    if (!op->uploaded64)
        return fail(TDG_E_STATE, "FP64 operator data not resident: call tdg_apply (FP64) once after tdg_set_material");
    const int nm = h.mat_space.num_basis();
    const int D = h.D;
    for (int64_t e = 0; e < h.E; ++e) {
        double lam, mu;
        element_lame(h, nm, e, lam, mu);
        const double* a = &h.mat_nodal[(static_cast<size_t>(e) * 2 + 0) * nm];
        const double* b = &h.mat_nodal[(static_cast<size_t>(e) * 2 + 1) * nm];
        for (int i = 0; i < nm; ++i)
            if (std::fabs(a[i] - lam) > 1e-10 * std::fabs(lam) || std::fabs(b[i] - mu) > 1e-10 * std::fabs(mu))
                return fail(TDG_E_INVALID, "material is not constant per element");
    }
    double* scratch = nullptr;
    if (adjoint_scratch(&scratch)) return fail(TDG_E_CUDA, "looking up the fixed scratch failed");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the values of lame_gradient_inputs: per facet both sides' penalty derivatives (each side's
    // lam, mu computed once per facet), then per element (lam, mu)
    const double cN1 = h.N * (h.N - 1.0 + D) / static_cast<double>(D);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    for (size_t c0 = 0; c0 < need; c0 += kNoallocStage) {
        const size_t n = std::min(kNoallocStage, need - c0);
        double* st = g_noalloc_stage;
        for (size_t i = c0; i < c0 + n;) {
            if (i < nfct) {  // chunk boundaries are multiples of 4: a facet never straddles two
                const int64_t f = static_cast<int64_t>(i / 4);
                const bool interior = h.up[2 * f] != h.up[2 * f + 1];
                const double scale = interior ? 0.25 : 1.0;
                for (int sd = 0; sd < 2; ++sd) {
                    double dl = 0.0, dm = 0.0;
                    if (sd == 0 || interior) {
                        const int64_t e = h.up[2 * f + sd];
                        double lam, mu;
                        element_lame(h, nm, e, lam, mu);
                        const double K = (D + 1) * cN1 * h.area[f] / h.volume[e];
                        const double c0v = 2.0 * mu, c1v = D * lam + 2.0 * mu;
                        dl = scale * K * 2.0 * c1v * D / c0v;
                        dm = scale * K * (4.0 * c1v / c0v - 2.0 * c1v * c1v / (c0v * c0v));
                    }
                    st[i - c0 + 2 * sd] = dl;
                    st[i - c0 + 2 * sd + 1] = dm;
                }
                i += 4;
            } else {
                const int64_t e = static_cast<int64_t>((i - nfct) / 2);
                double lam, mu;
                element_lame(h, nm, e, lam, mu);
                st[i - c0] = lam;
                st[i - c0 + 1] = mu;
                i += 2;
            }
        }
        TDG_CUDA_TRY(cudaMemcpyAsync(scratch + c0, st, n * sizeof(double), cudaMemcpyHostToDevice, s));
        TDG_CUDA_TRY(cudaStreamSynchronize(s));  // the stage is reused
    }
    int rc = launch_adjoint_lame(h.D, h.N, op->op64, u, p, bc_q, scratch, grad, s);
    TDG_CUDA_TRY(cudaStreamSynchronize(s));  // the scratch is free again when the call returns
    return rc ? fail(rc, "adjoint gradient launch failed") : 0;
}

// ------------------------------------------------------------------------------------------------
// explicit wave operator of elasticity (Elasticity::wave_rhs)
// ------------------------------------------------------------------------------------------------

namespace {
int ensure_wave(tdg_op* op) {
    if (op->wave_uploaded) return 0;
    auto const& h = op->h;
    op->arena_wave.release();
    const double *eq = nullptr, *mi = nullptr, *nr = nullptr;
    TDG_CUDA_TRY(op->arena_wave.upload(&eq, h.E_Q.a));
    TDG_CUDA_TRY(op->arena_wave.upload(&mi, h.Minv_ref.a));
    TDG_CUDA_TRY(op->arena_wave.upload(&nr, h.nrwj));
    op->wave.EQ = eq;
    op->wave.Minv = mi;
    op->wave.nrwj = nr;
    op->wave_uploaded = true;
    return 0;
}
}  // namespace

extern "C" int tdg_set_density(tdg_op* op, const double* rho_Q) {
    if (!op || !rho_Q) return fail(TDG_E_INVALID, "null argument");
    if (op->h.kind != 1) return fail(TDG_E_INVALID, "the density belongs to the elasticity operator");
    try {
        op->h.set_density(rho_Q);
    } catch (std::exception const& e) {
        return fail(TDG_E_INVALID, e.what());
    }
    op->wave_uploaded = false;
    return 0;
}

extern "C" int tdg_apply_inverse_mass(tdg_op* op, const double* x, double* y, int nrhs, int64_t ld, void* stream) {
    if (!op || !x || !y) return fail(TDG_E_INVALID, "null argument");
    auto const& h = op->h;
    if (h.kind != 1) return fail(TDG_E_INVALID, "the wave operator is defined for elasticity");
    if (nrhs < 1 || ld < h.E * h.bs) return fail(TDG_E_INVALID, "nrhs < 1 or ld < E * bs");
    TDG_TRY(ensure_wave(op));
    int rc = launch_inverse_mass(h.D, h.N, op->wave, h.E, h.Nq, x, nullptr, y, nrhs, ld,
                                 static_cast<cudaStream_t>(stream));
    return rc ? fail(rc, "inverse mass launch failed") : 0;
}

extern "C" int tdg_wave_rhs(tdg_op* op, const double* x, const double* b, double* y, int nrhs, int64_t ld,
                            void* stream) {
    if (!op || !x || !y) return fail(TDG_E_INVALID, "null argument");
    auto const& h = op->h;
    if (h.kind != 1) return fail(TDG_E_INVALID, "the wave operator is defined for elasticity");
    if (x == y || (b && b == y)) return fail(TDG_E_INVALID, "y must not alias x or b");
    TDG_TRY(tdg_apply(op, TDG_FP64, x, y, nrhs, ld, stream));
    TDG_TRY(ensure_wave(op));
    int rc = launch_inverse_mass(h.D, h.N, op->wave, h.E, h.Nq, y, b, y, nrhs, ld, static_cast<cudaStream_t>(stream));
    return rc ? fail(rc, "inverse mass launch failed") : 0;
}
