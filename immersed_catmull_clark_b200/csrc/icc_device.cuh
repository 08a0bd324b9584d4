// Device-side declarations: brick geometry, solver state, the operator handle and small
// device helpers shared by the FP64 (icc_op.cu) and tensor-core mixed (icc_mixed.cu) paths.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "icc_internal.h"

namespace icc {

// Brick of elements owned by one CTA and its control-point patch.
constexpr int kBX = 8, kBY = 4, kBZ = 4;
constexpr int kPX = kBX + 2, kPY = kBY + 2, kPZ = kBZ + 2;
constexpr int kPVol = kPX * kPY * kPZ;  // 360 control points per component
constexpr int kEPB = kBX * kBY * kBZ;   // 128 elements per brick

// FP64 DMMA tiling of the 81x81 contraction: K (trial) padded to 84 = 21 x 4, N (test) to 88 = 11 x 8.
constexpr int kKSteps = 21;
constexpr int kNTiles = 11;
constexpr int kFragPerType = kKSteps * kNTiles * 32;
constexpr int kApplyThreads = 256;
constexpr int kApplySmem = (3 * kPVol + kEPB * 81) * 8;

constexpr int kVecThreads = 256;

// PCG stop states (rust/src/solver.rs:40-73)
constexpr int kStatConverged = 1;
constexpr int kStatBreakdown = 2;
constexpr int kStatMaxIter = 3;
constexpr int kStatNan = 4;
constexpr int kStatReplace = 5;   // mixed form: the FP32 recurrence wants an FP64 residual replacement

struct Geom {
    int nx, ny, nz;        // elements per direction
    int cx, cy, cz;        // control points per direction
    long long nsc;         // scalar control points
    int nbx, nby, nbz;     // bricks per direction
    int nbricks;
};

struct PcgState {
    double rz_old, p_ap, alpha, beta, norm_b, rel_res, tol;
    double rz_prev;        // r'z used by the last alpha (the beta of a residual replacement needs it)
    long long iter, max_iter;
    int status;
    int fresh;             // mixed form: rz_old and rr_old are exact (set at the start and at replacements)
    // mixed form: ask for a residual replacement once rel_res < repl_delta * repl_res or after
    // repl_seg iterations since iteration repl_iter (repl_delta = 0: never); the test runs every
    // repl_every iterations (the host's batch), which keeps replacements from coming too often
    double repl_res, repl_delta;
    long long repl_iter, repl_seg, repl_every;   // tested only when iter is a multiple of repl_every
    double rr_old;         // mixed form: r'r of the current residual
};

// A sparse term S added to the operator: CSR with 32-bit row pointers and columns over the
// operator's DOFs, values in the vector type of the path that reads it (FP64 or FP32).
template <class T>
struct Sparse {
    const int *ptr = nullptr, *idx = nullptr;
    const T *val = nullptr;
};

// Boundary extraction.  On open uniform knots the B-splines of every element are a fixed
// recombination of the uniform (translated) quadratic B-splines: along each direction N = E B with
// E the identity except on the first two and the last two control points (knot insertion at the
// ends).  With K_u the element matrix of the uniform basis, which is the same for every element of
// the grid, the operator is K = E (sum_e s_e P_e' K_u P_e) E' (E = E_z (x) E_y (x) E_x per
// component).  The tensor-core apply therefore runs every element on K_u: its input patches are
// transformed by E' on the boundary control planes, and the node sums by E in the node-side pass.
struct Edge {
    int nb[3];          // boundary control points of direction d with a non-identity E (0: E = I)
    int id[3][4];       // their indices among 0, 1, n, n + 1
    float e[3][4][4];   // e[d][a][b] = E[id a][id b]
};

__device__ __forceinline__ int edge_slot(const Edge &E, int d, int i) {
    for (int a = 0; a < E.nb[d]; ++a)
        if (E.id[d][a] == i) return a;
    return -1;
}

struct MixedState;  // tensor-core path (icc_mixed.cu)
struct StateScratch;  // warm-started state solve and element energies (icc_topopt.cu)

struct Op {
    int device = 0, num_sms = 148, vec_blocks = 592;
    Geom g{};
    int64_t nel = 0, ndof = 0;
    int ntypes = 0, ntiles = 0, mask_mode = 0;
    long long scale_version = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // operator data
    double *d_scale = nullptr, *d_kfrag = nullptr, *d_kdiag = nullptr;
    int *d_type_id = nullptr, *d_tile_start = nullptr, *d_tile_type = nullptr;
    uint8_t *d_tile_elem = nullptr, *d_mask = nullptr;
    double *d_patch = nullptr;              // brick patch partial sums [nbricks][3][kPVol]
    // extra sparse term (icc_op_set_extra_triplets): y = mask rule of (K + S)(m .* x)
    int *d_sp_ptr = nullptr, *d_sp_idx = nullptr;
    double *d_sp_val = nullptr, *d_sp_diag = nullptr;
    float *d_sp_val32 = nullptr;
    int64_t sp_nnz = 0;
    Sparse<double> extra64() const {
        Sparse<double> s;
        if (sp_nnz) { s.ptr = d_sp_ptr; s.idx = d_sp_idx; s.val = d_sp_val; }
        return s;
    }
    Sparse<float> extra32() const {
        Sparse<float> s;
        if (sp_nnz) { s.ptr = d_sp_ptr; s.idx = d_sp_idx; s.val = d_sp_val32; }
        return s;
    }
    double *d_x_in = nullptr, *d_y_out = nullptr;
    // PCG
    double *d_x = nullptr, *d_r = nullptr, *d_p = nullptr, *d_ap = nullptr, *d_inv = nullptr, *d_b = nullptr,
           *d_diag = nullptr, *d_partials = nullptr;
    PcgState *d_state = nullptr, *h_state = nullptr;
    unsigned *d_counter = nullptr;          // last-CTA counter of the fused reductions
    cudaGraphExec_t graph_exec = nullptr;
    int graph_batch = 0;
    icc_solve_info last_info{};
    // host copies used by the tensor-core path set-up
    std::vector<double> host_ktypes, host_scale;
    std::vector<int32_t> host_type_id;
    std::vector<int> host_type1d[3];                     // 1-D type of every element position
    std::vector<std::array<double, 9>> host_basis1d[3];  // basis values per 1-D type (Space::basis1d)
    MixedState *mixed = nullptr;
    StateScratch *state = nullptr;

    ~Op();
    int init(const Space &s, const double *ke_types, int nt, const int32_t *type_id, const double *scale,
             const uint8_t *free_mask, int mode);
    int set_scale(const double *scale);
    int set_scale_dev(const double *scale_dev);   // device array, stream-ordered
    int set_mask(const uint8_t *free_mask, int mode);
    int set_extra(int64_t count, const int64_t *rows, const int64_t *cols, const double *vals);
    void enqueue_apply(const double *x, double *y, double *partials, const PcgState *st);
    void enqueue_apply_on(cudaStream_t s, const double *x, double *y);   // y = A x on stream s
    void enqueue_diagonal(double *d, cudaStream_t s);                     // the diagonal on stream s
    int apply_dev(const double *x, double *y);
    int diagonal_dev(double *d);
    int ensure_pcg_buffers();
    void enqueue_pcg_iteration();
    int pcg_fp64(const double *b, const double *diag, double tol, int64_t max_iter, int check_every, double *x,
                 int64_t *iters, double *rel_res);
};

int cuda_fail(cudaError_t e, const char *where);

// tensor-core mixed-precision path (icc_mixed.cu)
void mixed_release(Op &op);
void state_release(Op &op);
int mixed_on_scale_update(Op &op);
int mixed_apply_f32(Op &op, const float *x, float *y);
int mixed_profile_apply(Op &op, const float *x, float *y, int reps, double *contract_ms, double *gather_ms);
int mixed_set_wait_limit(Op &op, long long polls);
struct VecSet;   // the vectors of one system of a mixed solve (icc_mixed.cu)
int mixed_solve_batch(cudaStream_t stream, const std::vector<Op *> &ops, const std::vector<VecSet *> &vsets,
                      const double *const *b, const double *const *diag, const double *tol, const int64_t *max_iter,
                      const icc_solve_opts &opts, double *const *x, int *status, int64_t *iters, double *rel_res,
                      int64_t *replacements);
VecSet *mixed_vecset_create(Op &op);
void mixed_vecset_destroy(VecSet *v);
VecSet *mixed_own_vecset(Op &op);
void mixed_invalidate_graph(Op &op);
int mixed_solve(Op &op, const double *b, const double *diag, double tol, int64_t max_iter,
                const icc_solve_opts &opts, double *x, int64_t *iters, double *rel_res);

// ---- device helpers -------------------------------------------------------------------------

// D[16x8] += A[16x4] * B[4x8] on the FP64 tensor cores.  Fragments (PTX ISA, mma.m16n8k4 .f64):
// a0/a1 = A[gid][tig] / A[gid+8][tig], b0 = B[tig][gid], d0..d3 = D[gid (+8 for d2,d3)][2 tig + (i&1)],
// with gid = lane / 4 and tig = lane % 4.
__device__ __forceinline__ void dmma_m16n8k4(double (&d)[4], double a0, double a1, double b0) {
    asm("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block reduction; the result is valid in warp 0 (thread 0 writes it out).
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double ws[32];
    v = warp_sum(v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

}  // namespace icc

// The C-ABI operator handle.
struct icc_op {
    icc::Op op;
};

// Solve on device arrays with the handle's operator (icc_pcg_solve_dev without the final sync);
// internal, not part of include/icc.h.
extern "C" int icc_solve_common(icc_op *op, const double *b_dev, const double *diag_dev, int64_t n, double tol,
                     int64_t max_iter, const icc_solve_opts *opts, double *x_dev, int64_t *iters, double *rel_res);
