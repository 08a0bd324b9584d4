// Mixed-precision form of the solve: a Jacobi-PCG whose iterations run in FP32 on the
// 5th-generation tensor cores, with FP64 reductions, an FP64 solution and FP64 residual
// replacement (reliable updates).
//
// Tensor-core brick apply (persistent, one CTA per SM, bricks of 8x4x4 elements; element m of a
// brick = row m of the MMA tile = TMEM lane m):
//   A = U [128 elements x 96], the brick's element vectors, component c at columns c*32 + [0,27)
//       after the element-local shift, the scale s_e and the 1-D basis change R^T;
//   B = K_main [96 x 96] (test DOF rows, trial DOF columns, same per-component padding);
//   D[128 x 96] (TMEM, FP32) = A_lo B_hi + A_hi B_lo + A_hi B_hi, a 3-term split-TF32 product
//   (v = hi + lo with hi = tf32(v), lo = tf32(v - hi)): 36 tcgen05.mma kind::tf32, M=128, N=96, K=8.
// The epilogue applies R to each row and sums the element results per patch node in a fixed
// order, and the node-side pass resolves the brick overlaps, as in the FP64 apply: no atomics,
// bitwise reproducible.
//
// Solve (mixed_solve): the FP32 recurrence x, r, p, Ap (FP64 dot products) runs in CUDA graphs;
// the FP64 solution accumulates its updates and the FP64 true residual b - A x (FP64 apply)
// replaces the FP32 residual whenever it has fallen by a factor delta; the solve stops on the
// FP64 true residual.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "icc_device.cuh"
#include "icc_tc.cuh"
#include "icc_vec.cuh"

namespace icc {

#define ICC_CUDA(call, where)                                    \
    do {                                                         \
        cudaError_t _e = (call);                                 \
        if (_e != cudaSuccess) return ::icc::cuda_fail(_e, where); \
    } while (0)

constexpr int kTcM = kEPB;             // 128 rows = the brick's elements
constexpr int kTcN = 96;               // test DOFs: component c at rows c*32 + [0, 27)
constexpr int kTcK = 96;               // trial DOFs: component c at columns c*32 + [0, 27)
constexpr int kTcKSteps = kTcK / 8;    // 12 MMAs of K = 8 per term
constexpr int kBFl = kTcN * kTcK;      // floats per B term
constexpr uint32_t kBLbo = (kTcN / 8) * 128;  // bytes between K-adjacent core matrices of B
constexpr uint32_t kSbo = 128;                // bytes between 8-row groups
constexpr long long kWaitLimit = 1LL << 22;
constexpr long long kGridWaitLimit = 1LL << 22;   // default polls of a grid barrier before it gives up

// offset (floats) of element (row, k) in the canonical K-major no-swizzle layout with `rows` rows
__host__ __device__ __forceinline__ int canon(int row, int k, int rows) {
    return (k >> 2) * (rows / 8) * 32 + (row >> 3) * 32 + (row & 7) * 4 + (k & 3);
}

// One brick of a batch, precomputed on the host so the kernel needs no integer divisions: its
// system, its index within the system, its brick coordinates and extent, and its boundary flags
// (bit d: the brick's patch holds boundary control points of direction d).
struct BrickDesc {
    int inst, local;
    unsigned xyz;   // bx | by << 11 | bz << 22
    unsigned ext;   // ex_n | ey_n << 4 | ez_n << 8 | flags << 12
};
constexpr int kMaxListPerCta = 1024;   // bricks of one persistent CTA in one launch, at most
constexpr int kMaxInst = 1024;         // systems of one batch, at most

// One system of a mixed solve as the kernels see it: the operator data of its handle and its own
// FP32 vectors.  A solve of one system is a batch of one; a batch of several (designs of uneven
// sizes, or load cases of one operator) runs every iteration as one persistent apply over all
// bricks of all systems and one fused vector step whose CTAs are shared out among the systems.
struct TcInst {
    CUtensorMap tmap;            // the apply input pin as a 4-D tensor (x, y, z, component), for TMA
    Geom g;
    int cta0, ncta;              // CTAs of the fused vector step that serve it
    float kfac;                  // the system's K_u = kfac * the batch's K_u (same element shape)
    const float *scale;          // s_e (FP32)
    const Edge *edge;
    float *patch;                // brick partials [nbricks][3][kPVol]
    const uint8_t *mask;         // output rule of the fused vector step (null: none)
    int mask_mode;
    Sparse<float> sp;
    const float *inv;
    float *x, *r, *p, *ap;
    float *pin;                  // the brick apply's input: the masked p, rows padded to cxp
    int cxp;
    double *part;                // [9][ncta] partial sums of the fused vector step
    PcgState *st;                // null for a plain apply: every brick is active
};

// The FP32 and FP64 vectors and the PCG state of one system of a mixed solve.
struct VecSet {
    float *patch32 = nullptr, *rhs32 = nullptr, *x32 = nullptr, *r32 = nullptr, *p32 = nullptr, *ap32 = nullptr,
          *inv32 = nullptr;
    // the brick apply's input [3][cz][cy][cxp] (rows padded to a multiple of 4 floats, so every row
    // starts on 16 bytes as TMA needs) and its tensor map
    float *pin32 = nullptr;
    int cxp = 0;
    CUtensorMap tmap{};
    double *x64 = nullptr, *r64 = nullptr, *y64 = nullptr;
    double *part = nullptr;  // [9][tail CTAs]
    int part_cap = 0;
};

struct MixedState {
    bool ready = false;
    float4 *d_bmat = nullptr;        // K_u split [hi, lo][kBFl] in the canonical layout
    std::vector<double> kunif;       // K_u (host), to compare systems of a batch
    Edge edge{};
    Edge *d_edge = nullptr;          // the same in device memory, for the node-side passes
    std::vector<uint8_t> flags;      // per brick: bit d set when its patch holds boundary points of d
    BrickDesc *d_desc = nullptr;     // the handle's bricks as system 0 of a batch
    float *d_scale32 = nullptr;
    double *d_scalars = nullptr, *h_scalars = nullptr;
    int *d_err = nullptr;
    int *h_err = nullptr;                      // pinned copy of d_err read after every graph batch
    unsigned long long *d_grid_ctr = nullptr;  // grid barrier counter of the fused vector step
    int tail_per_sm = 1;                       // resident CTAs of the fused vector step per SM
    long long grid_wait_limit = kGridWaitLimit;
    VecSet v;                                  // the handle's own system
    TcInst *d_inst = nullptr;                  // its one-entry instance table
    PcgState *d_state = nullptr, *h_state = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_batch = 0;
    long long graph_limit = 0;   // grid_wait_limit the graph was captured with
};

// ------------------------------------------------------------------------------------------
// Kernels
// ------------------------------------------------------------------------------------------

// ---- persistent, warp-specialised tensor-core brick apply ------------------------------------
// One CTA per SM walks the bricks blockIdx.x, blockIdx.x + gridDim.x, ... of the batch's brick
// numbering (all bricks of all systems), skipping systems whose solve has stopped.  Roles
// (26 warps):
//   warps 25-27 (loaders): one thread fetches the input patch of each brick (3 x 6 x 6 x 12
//     control values, zero outside the grid) with one TMA copy, up to four bricks ahead, into one
//     of five patch buffers; warp 25 + c transforms component c of the patches of bricks at the
//     grid's ends by E' (the boundary extraction), and the three warps hand each buffer to the
//     builders through an mbarrier;
//   warps 0-11 (builders, warp 4 c + q: component c of z-layer q): gather each element's 27
//     values of component c from the shared patch, shift them by the element's centre value and
//     scale by s_e, split into TF32 hi/lo and store A_hi into TMEM (row m = element m = lane m)
//     and A_lo into shared memory, in two A slots;
//   warp 24 (MMA, one thread): holds B = K_u hi/lo in shared memory and issues the 36
//     tcgen05.mma of a brick (A_lo B_hi from shared memory, A_hi B_lo and A_hi B_hi with A from
//     TMEM) into one of two TMEM accumulators;
//   warps 12-23 (epilogue, same split): read their 32 accumulator columns with tcgen05.ld and
//     release them, sum the element results per patch node with warp shuffles (x, y) and a
//     shared buffer (z), transform the node partials of bricks at the grid's ends by E, and
//     write the brick partials.
// mbarriers: t_full (TMA copies), p_full/p_empty (patch buffers), a_full/a_empty (A slots),
// d_full/d_empty (kNAcc accumulator buffers), b_full, fin.
// Every wait is bounded.  On time-out the waiting thread raises a shared abort flag; every other
// wait then returns false at once.  The builders and the epilogue decide at a barrier that ORs
// the flag over the role, so all threads of a role leave their loop at the same brick; the MMA
// thread stops issuing, then commits once more and waits (bounded) for that commit, so no MMA
// of the CTA is in flight when TMEM is released.  The host reports ICC_TIMEOUT.
constexpr int kRoleWarps = 12;                  // builders: warps 0-11, epilogue: 12-23, MMA: 24, loaders: 25-27
constexpr int kRoleThreads = kRoleWarps * 32;
constexpr int kLoaderWarp = 2 * kRoleWarps + 1;   // the MMA warp is 2 kRoleWarps
constexpr int kPtThreads = (2 * kRoleWarps + 4) * 32;
constexpr int kColSlot = kTcK;         // A_hi slot s: TMEM columns s*96 + [0,96)
constexpr int kColD = 2 * kColSlot;    // accumulator buffer d: TMEM columns 192 + d*96 + [0,96)
constexpr int kNAcc = 3;              // accumulator buffers: the epilogue may lag the MMA by two bricks
constexpr int kAloFl = kTcM * kTcK;    // A_lo slot (shared memory, canonical K-major): floats
constexpr uint32_t kALbo = (kTcM / 8) * 128;  // bytes between K-adjacent core matrices of A_lo
constexpr uint32_t kPtTmemCols = 512;
static_assert(kColD + kNAcc * kTcN <= (int)kPtTmemCols, "accumulators beyond the TMEM allocation");
constexpr int kZFl = kBZ * 3 * 3 * kPY * kPX;  // per-layer node partials: [lz][az][c][py][px]
constexpr int kPXs = 12;                        // x extent of an input patch row in shared memory (48 B)
constexpr int kPVolS = kPZ * kPY * kPXs;        // per component
constexpr uint32_t kPatchBytes = 3 * kPVolS * 4;   // one TMA box: 5,184 B
constexpr int kPatBuf = 1312;                   // floats per patch buffer (5,248 B: 128-byte aligned)
constexpr int kNPatch = 5;                      // patch buffers (the loaders run up to 4 bricks ahead)
constexpr int kLoadAhead = 3;                   // bricks whose copies are in flight while one is finished
static_assert(kPatBuf * 4 >= (int)kPatchBytes && (kPatBuf * 4) % 128 == 0, "patch buffer");
constexpr int kPtSmem = (2 * kBFl + 2 * kAloFl + kNPatch * kPatBuf + 2 * kZFl + 3 * kPVol) * 4;  // 219,872 B
constexpr uint32_t kBBytes = 2 * kBFl * 4;                         // hi + lo

// A test (mbarrier.try_wait without a time hint) may suspend the thread for a system-dependent
// time; after kWaitLimit tests (~0.1 s if they return at once, a few seconds if each suspends for
// about a microsecond) the wait gives up -- far beyond any wait of a working kernel (a brick takes
// a few microseconds).  Measured on the 128x64x64 apply, the version with a 1 us suspend hint
// took 1% longer.
__device__ __forceinline__ bool pt_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag, int *err) {
    for (long long i = 0; i < kWaitLimit; ++i) {
        if (tc::mbar_try_wait(bar, parity)) return true;
        if (*abort_flag) return false;
    }
    *abort_flag = 1;
    atomicExch(err, 1);
    return false;
}

struct BrickBox {
    int x0, y0, z0, ex_n, ey_n, ez_n;
};


__device__ __forceinline__ BrickBox desc_box(const BrickDesc &d) {
    BrickBox r;
    r.x0 = int(d.xyz & 2047u) * kBX;
    r.y0 = int((d.xyz >> 11) & 2047u) * kBY;
    r.z0 = int(d.xyz >> 22) * kBZ;
    r.ex_n = int(d.ext & 15u);
    r.ey_n = int((d.ext >> 4) & 15u);
    r.ez_n = int((d.ext >> 8) & 15u);
    return r;
}

__device__ __forceinline__ unsigned desc_flags(const BrickDesc &d) { return (d.ext >> 12) & 7u; }

// V = E' u on the boundary control points of direction D inside the patch P (3 x kPZ x kPY x kPXs,
// patch origin o along D, ext of its control points inside the grid); line t along D (t < the
// number of lines) is handled by thread t.  Every control point that a boundary value needs lies
// in the patch: the set-up checks that E couples only control points of a common element.
template <int D>
__device__ __forceinline__ void edge_in(float *P, const Edge &E, int o, int ext, int t) {
    constexpr int LA = D == 0 ? kPY : kPX;   // extent of the line index that runs fastest
    constexpr int LB = D == 2 ? kPY : kPZ;
    constexpr int stride = D == 0 ? 1 : (D == 1 ? kPXs : kPXs * kPY);
    if (t >= 3 * LA * LB) return;
    const int c = t / (LA * LB), w = t - c * (LA * LB), a1 = w % LA, a2 = w / LA;
    const int base = D == 0 ? c * kPVolS + (a2 * kPY + a1) * kPXs
                            : (D == 1 ? c * kPVolS + a2 * (kPY * kPXs) + a1 : c * kPVolS + a2 * kPXs + a1);
    const int nb = E.nb[D];
    float u[4], v[4];
    int loc[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int l = a < nb ? E.id[D][a] - o : -1;
        loc[a] = (l >= 0 && l < ext) ? l : -1;
        u[a] = loc[a] >= 0 ? P[base + loc[a] * stride] : 0.f;
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        float acc = 0.f;
#pragma unroll
        for (int a = 0; a < 4; ++a) acc = fmaf(E.e[D][a][b], u[a], acc);
        v[b] = acc;
    }
#pragma unroll
    for (int b = 0; b < 4; ++b)
        if (loc[b] >= 0) P[base + loc[b] * stride] = v[b];
}

// W <- E W on the boundary control points of direction D of a brick's node partials P (patch
// layout, origin o along D, ext of them inside the grid); line t along D is handled by thread t.
// E couples only control points of a common element, so the partials of one brick transform on
// their own and the transformed partials of all bricks add up to E applied to the node sums.
template <int D>
__device__ __forceinline__ void edge_out(float *P, const Edge &E, int o, int ext, int t) {
    constexpr int LA = D == 0 ? kPY : kPX;
    constexpr int LB = D == 2 ? kPY : kPZ;
    constexpr int stride = D == 0 ? 1 : (D == 1 ? kPX : kPX * kPY);
    if (t >= 3 * LA * LB) return;
    const int c = t / (LA * LB), w = t - c * (LA * LB), a1 = w % LA, a2 = w / LA;
    const int base = D == 0 ? c * kPVol + (a2 * kPY + a1) * kPX
                            : (D == 1 ? c * kPVol + a2 * (kPY * kPX) + a1 : c * kPVol + a2 * kPX + a1);
    const int nb = E.nb[D];
    float u[4], v[4];
    int loc[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int l = a < nb ? E.id[D][a] - o : -1;
        loc[a] = (l >= 0 && l < ext) ? l : -1;
        u[a] = loc[a] >= 0 ? P[base + loc[a] * stride] : 0.f;
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        float acc = 0.f;
#pragma unroll
        for (int b = 0; b < 4; ++b) acc = fmaf(E.e[D][a][b], u[b], acc);
        v[a] = acc;
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
        if (loc[a] >= 0) P[base + loc[a] * stride] = v[a];
}

__device__ __forceinline__ float row_scale(const TcInst &I, const BrickBox &bb, int r) {
    const int lx = r % kBX, ly = (r / kBX) % kBY, lz = r / (kBX * kBY);
    if (lx < bb.ex_n && ly < bb.ey_n && lz < bb.ez_n)
        return I.kfac * I.scale[(long long)(bb.x0 + lx) +
                                (long long)I.g.nx * ((bb.y0 + ly) + (long long)I.g.ny * (bb.z0 + lz))];
    return 0.f;
}

// 28 warps: registers are split over the 4 SM sub-partitions, so 7 warps share 16,384 of them and
// the compiler caps a thread at 72
__global__ void __launch_bounds__(kPtThreads, 1)
apply_tc_kernel(const TcInst *__restrict__ insts, int ninst, int nbricks, const BrickDesc *__restrict__ desc,
                const float4 *__restrict__ bmat, int *__restrict__ err) {
    extern __shared__ __align__(1024) float psm[];
    float *sB = psm;                      // [hi, lo][kBFl]
    float *sAlo = psm + 2 * kBFl;         // [2 slots][kAloFl] A_lo operand
    float *sP = sAlo + 2 * kAloFl;        // [kNPatch][kPatBuf] input patches
    float *sZb = sP + kNPatch * kPatBuf;  // [2][kZFl] per-layer node partials, by brick parity
    float *sW = sZb + 2 * kZFl;           // [3 * kPVol] node partials of a boundary brick (E applied)
    __shared__ __align__(8) uint64_t bars[6 + 2 * kNAcc + 3 * kNPatch];
    __shared__ uint32_t tmem_base;
    __shared__ volatile int s_abort;
    // this CTA's bricks of systems whose solve goes on: bricks blockIdx.x + k gridDim.x in order
    __shared__ int s_list[kMaxListPerCta];
    __shared__ int s_cnt[32];
    __shared__ int s_nlist;
    __shared__ unsigned s_act[kMaxInst / 32];   // bit i: system i's solve goes on
    uint64_t *a_full = bars, *a_empty = bars + 2, *d_full = bars + 4, *d_empty = bars + 4 + kNAcc,
             *b_full = bars + 4 + 2 * kNAcc,
             *fin = bars + 5 + 2 * kNAcc, *p_full = bars + 6 + 2 * kNAcc, *p_empty = p_full + kNPatch,
             *t_full = p_full + 2 * kNPatch;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, kPtTmemCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&a_full[0], kRoleThreads);
        tc::mbar_init(&a_full[1], kRoleThreads);
        tc::mbar_init(&a_empty[0], 1);
        tc::mbar_init(&a_empty[1], 1);
        for (int d = 0; d < kNAcc; ++d) {
            tc::mbar_init(&d_full[d], 1);
            tc::mbar_init(&d_empty[d], kRoleThreads);
        }
        tc::mbar_init(b_full, 1);
        tc::mbar_init(fin, 1);
        for (int b = 0; b < kNPatch; ++b) {
            tc::mbar_init(&p_full[b], 96);
            tc::mbar_init(&p_empty[b], kRoleThreads);
            tc::mbar_init(&t_full[b], 1);
        }
        tc::fence_mbar_init();
        s_abort = 0;
        // B, the same in every launch, is copied before the wait below
        tc::mbar_arrive_expect_tx(b_full, kBBytes);
        tc::bulk_g2s(sB, bmat, kBBytes, b_full);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    // everything below reads or writes what the previous kernel of the stream may still use (the
    // states, the input, the brick partials)
    tc::griddep_wait();
    {
        // stream compaction, kPtThreads candidates per round: each warp ballots its 32, the counts
        // give every warp its offset, the list keeps the order of the bricks
        const int G = gridDim.x, L = (nbricks - (int)blockIdx.x + G - 1) / G;
        constexpr int kW = kPtThreads / 32;
        if (tid == 0) s_nlist = 0;
        for (int i = tid; i < kMaxInst / 32; i += kPtThreads) s_act[i] = 0u;
        __syncthreads();
        for (int i = tid; i < ninst; i += kPtThreads) {
            const PcgState *st = insts[i].st;
            if (!st || __ldcg(&st->status) == 0) atomicOr(&s_act[i >> 5], 1u << (i & 31));
        }
        __syncthreads();
        for (int base = 0; base < L; base += kPtThreads) {
            const int k = base + tid;
            bool a = false;
            if (k < L) {
                const int si = ninst == 1 ? 0 : desc[blockIdx.x + k * G].inst;
                a = (s_act[si >> 5] >> (si & 31)) & 1u;
            }
            const unsigned act = __ballot_sync(0xffffffffu, a);
            if (lane == 0) s_cnt[warp] = __popc(act);
            __syncthreads();
            int off = s_nlist;
            for (int w2 = 0; w2 < warp; ++w2) off += s_cnt[w2];
            if (a) s_list[off + __popc(act & ((1u << lane) - 1u))] = blockIdx.x + k * G;
            __syncthreads();
            if (tid == 0) {
                int t = s_nlist;
                for (int w2 = 0; w2 < kW; ++w2) t += s_cnt[w2];
                s_nlist = t;
            }
            __syncthreads();
        }
        if (s_nlist == 0) {   // nothing for this CTA (the same for all its threads)
            if (tid == 0) tc::mbar_wait_bounded(b_full, 0u, kWaitLimit);   // the B copy has landed
            tc::fence_before_sync();
            __syncthreads();
            if (warp == 0) {
                tc::fence_after_sync();
                tc::tmem_dealloc(tmem_base, kPtTmemCols);
            }
            return;
        }
    }
    const int nmine = s_nlist;
    const uint32_t tmem = tmem_base;

    if (warp < kRoleWarps) {
        // ------------------------------ builders ------------------------------
        // warp = 4 c + q: component c of the 32 elements of z-layer q (TMEM lanes 32 q ..); the
        // builders wait only for their patch buffer and their A slot, never for each other.
        const int c = warp >> 2, q = warp & 3;
        const int lx = lane & 7, ly = lane >> 3;
        const unsigned FULLW = 0xffffffffu;
        const int r = q * 32 + lane;
        // s_e of this thread's element is read one brick ahead, descriptors two
        BrickDesc dn = desc[s_list[0]];
        BrickDesc d1 = nmine > 1 ? desc[s_list[1]] : BrickDesc{};
        float se_next = row_scale(insts[dn.inst], desc_box(dn), r);
        for (int it = 0; it < nmine; ++it) {
            const int s = it & 1, pb = it % kNPatch;
            const float se = se_next;      // s_e k of this thread's element (0 outside the grid)
            const BrickBox bb = desc_box(dn);
            if (it + 1 < nmine) se_next = row_scale(insts[d1.inst], desc_box(d1), r);
            dn = d1;
            d1 = it + 2 < nmine ? desc[s_list[it + 2]] : BrickDesc{};
            const bool valid = lx < bb.ex_n && ly < bb.ey_n && q < bb.ez_n;
            const float vm = valid ? se : 0.f;
            const bool ok = pt_wait(&p_full[pb], uint32_t(it / kNPatch) & 1u, &s_abort, err) &&
                            (it < 2 || pt_wait(&a_empty[s], uint32_t((it >> 1) - 1) & 1u, &s_abort, err));
            // the warp leaves together on abort (nothing of the other warps waits for it here)
            if (!__all_sync(FULLW, ok && s_abort == 0)) break;
            tc::fence_after_sync();
            const float *Pc = sP + pb * kPatBuf + c * kPVolS + q * (kPY * kPXs) + ly * kPXs + lx;
            float v[27];
#pragma unroll
            for (int a = 0; a < 27; ++a) v[a] = Pc[(a / 9) * (kPY * kPXs) + ((a / 3) % 3) * kPXs + a % 3];
            // Element-local shift: K_u maps a constant per-component field to zero, so subtracting
            // the element's centre control value changes nothing in exact arithmetic while the
            // split operands carry only the variation across the element; the TF32 splitting
            // error then scales with that variation instead of with |u| (smooth, low-energy
            // vectors of a converging PCG).
            const float nctr = -v[13] * vm;
#pragma unroll
            for (int a = 0; a < 27; ++a) v[a] = fmaf(v[a], vm, nctr);   // s_e (v - ctr), or 0 outside the grid
            tc::mbar_arrive(&p_empty[pb]);   // this thread's reads of the patch are done
            // A_hi into TMEM (lane = element), A_lo into shared memory in the canonical layout
            const uint32_t col = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(s * kColSlot + c * 32);
            float *alo = sAlo + s * kAloFl + canon(q * 32 + lane, c * 32, kTcM);
#pragma unroll
            for (int q8 = 0; q8 < 4; ++q8) {
                float hi[8], lo[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) tc::split_tf32_raw(q8 * 8 + j < 27 ? v[q8 * 8 + j] : 0.f, hi[j], lo[j]);
                tc::tmem_st8(col + q8 * 8, hi);
                // 4 consecutive k of one row are 16 contiguous bytes; k + 4 is one core-matrix column on
                *reinterpret_cast<float4 *>(alo + (2 * q8) * (kTcM / 8) * 32) = make_float4(lo[0], lo[1], lo[2], lo[3]);
                *reinterpret_cast<float4 *>(alo + (2 * q8 + 1) * (kTcM / 8) * 32) = make_float4(lo[4], lo[5], lo[6], lo[7]);
            }
            tc::fence_proxy_async();   // A_lo (generic-proxy stores) -> visible to the tensor core
            tc::tmem_wait_st();
            tc::fence_before_sync();
            tc::mbar_arrive(&a_full[s]);
        }
    } else if (warp < 2 * kRoleWarps) {
        // ------------------------------ epilogue ------------------------------
        // warp = 12 + 4 c + q: component c of z-layer q; lane = lx + 8 ly = element (lx, ly, q)
        // = TMEM lane 32 q + lane.  Node sums run in registers: along x with shuffles by 1 and 2
        // lanes, along y by 8 and 16 lanes; the 4 layers are combined through shared memory.
        const int et = tid - kRoleThreads;
        const int c = (warp - kRoleWarps) >> 2, q = warp & 3;
        const int lx = lane & 7, ly = lane >> 3;
        const uint32_t dcol0 = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(kColD + c * 32);
        const unsigned FULL = 0xffffffffu;
        // lane masks of the node sums as multipliers (FMA instead of selects)
        const float mx1 = lx >= 1 ? 1.f : 0.f, my1 = ly >= 1 ? 1.f : 0.f;
        // z-sum: this thread's outputs i = et + k * 384 of the brick; the term of layer lz = pz - az
        // sits at sZ[((lz * 3 + az) * 3 + ci) * 60 + pyx] = sZ[zb - 360 az] with zb = 540 pz + 60 ci + pyx
        int zb[3], zpz[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int i = et + k * kRoleThreads;
            const int ci = i / kPVol, rem = i - ci * kPVol;
            const int pz = rem / (kPX * kPY), pyx = rem - pz * (kPX * kPY);
            zb[k] = 9 * (kPY * kPX) * pz + (kPY * kPX) * ci + pyx;
            zpz[k] = pz;
        }
        for (int it = 0, db = 0, dph = 0; it < nmine; ++it) {
            float *sZ = sZb + (it & 1) * kZFl;
            const BrickDesc d = desc[s_list[it]];
            // on a failed wait the values read below are not used: the barrier before the z-sum
            // makes every epilogue thread leave the loop
            const bool ok = pt_wait(&d_full[db], uint32_t(dph), &s_abort, err);
            tc::fence_after_sync();
            uint32_t dv[32];
            tc::tmem_ld32(dcol0 + (uint32_t)(db * kTcN), dv);
            tc::tmem_wait_ld();
            tc::fence_before_sync();
            tc::mbar_arrive(&d_empty[db]);   // accumulator buffer db is free for brick it + kNAcc
            if (++db == kNAcc) {
                db = 0;
                dph ^= 1;
            }
            float res[27];
#pragma unroll
            for (int a = 0; a < 27; ++a) res[a] = __uint_as_float(dv[a]);
            // x, in place: t(lx) = v[ax=1](lx) + v[2](lx-1), then node px = lx gets v[0](lx) + t(lx-1) in
            // res[o]; lanes lx = 7 also carry px = 8 (t(7)) in res[o+1] and px = 9 (v[2](7)) in res[o+2]
#pragma unroll
            for (int az = 0; az < 3; ++az)
#pragma unroll
                for (int ay = 0; ay < 3; ++ay) {
                    const int o = 3 * ay + 9 * az;
                    const float t = fmaf(mx1, __shfl_up_sync(FULL, res[o + 2], 1), res[o + 1]);
                    res[o] = fmaf(mx1, __shfl_up_sync(FULL, t, 1), res[o]);
                    res[o + 1] = t;
                }
            // y, the same along ly (lanes 8 apart): node py = ly gets X[ay=0](ly) + (X[1] + X[2](. - 1))(ly - 1);
            // lanes ly = 3 also carry py = 4 and py = 5.  Results are this layer's partials for z-offset az.
#pragma unroll
            for (int az = 0; az < 3; ++az)
#pragma unroll
                for (int var = 0; var < 3; ++var) {
                    const float a0 = res[9 * az + var], a1 = res[9 * az + 3 + var], a2 = res[9 * az + 6 + var];
                    const float y4 = fmaf(my1, __shfl_up_sync(FULL, a2, 8), a1);
                    const float yv = fmaf(my1, __shfl_up_sync(FULL, y4, 8), a0);
                    const int px = var == 0 ? lx : 7 + var;
                    if (var == 0 || lx == 7) {
                        float *zp = sZ + (((q * 3 + az) * 3 + c) * kPY) * kPX + px;
                        zp[ly * kPX] = yv;
                        if (ly == 3) {
                            zp[4 * kPX] = y4;
                            zp[5 * kPX] = a2;
                        }
                    }
                }
            // all layers of brick it are in sZ[it & 1]; every z-sum of brick it - 1 (which read
            // the other buffer) finished before its thread reached this barrier
            if (tc::named_sync_or(2, kRoleThreads, !ok || s_abort != 0)) break;
            // z: node pz = lz + az; sum the <= 3 layers in increasing az
            const TcInst &I = insts[d.inst];
            const int local = d.local;
            const unsigned fl = desc_flags(d);   // the same for every epilogue thread
            float *ob = I.patch + (size_t)local * 3 * kPVol + et;
            float sums[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                float sum = 0.f;
                if (et + k * kRoleThreads < 3 * kPVol) {
#pragma unroll
                    for (int az = 0; az < 3; ++az)
                        if (zpz[k] - az >= 0 && zpz[k] - az < kBZ) sum += sZ[zb[k] - 2 * 3 * (kPY * kPX) * az];
                }
                sums[k] = sum;
            }
            if (fl) {
                // W <- E W on the boundary planes of this brick's partials, one direction after the
                // other (sW is reused by the next boundary brick only after the next brick's barrier,
                // which every thread reaches after its reads below)
                const BrickBox bb = desc_box(d);
                const Edge &E = *I.edge;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    if (et + k * kRoleThreads < 3 * kPVol) sW[et + k * kRoleThreads] = sums[k];
                tc::named_sync(2, kRoleThreads);
                if (fl & 1u) {
                    edge_out<0>(sW, E, bb.x0, min(kPX, I.g.cx - bb.x0), et);
                    tc::named_sync(2, kRoleThreads);
                }
                if (fl & 2u) {
                    edge_out<1>(sW, E, bb.y0, min(kPY, I.g.cy - bb.y0), et);
                    tc::named_sync(2, kRoleThreads);
                }
                if (fl & 4u) {
                    edge_out<2>(sW, E, bb.z0, min(kPZ, I.g.cz - bb.z0), et);
                    tc::named_sync(2, kRoleThreads);
                }
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    if (et + k * kRoleThreads < 3 * kPVol) sums[k] = sW[et + k * kRoleThreads];
            }
#pragma unroll
            for (int k = 0; k < 3; ++k)
                if (et + k * kRoleThreads < 3 * kPVol) ob[k * kRoleThreads] = sums[k];
        }
    } else if (warp >= kLoaderWarp) {
        // ------------------------------ loaders ------------------------------
        // brick k goes to buffer k % kNPatch once the builders have read brick k - kNPatch from
        // it (warp 25 issues the copy); kLoadAhead bricks later each loader warp waits for the
        // copy, transforms its component and its lanes arrive on the buffer's p_full (their own
        // writes are done).  Every loader warp waits for each copy once, in brick order, so no
        // wait runs a phase ahead of its barrier.
        const unsigned FULLW = 0xffffffffu;
        const int lc = warp - kLoaderWarp;
        int issued = 0, landed = 0, last_inst = -1;
        for (int k = 0; k < nmine + kLoadAhead; ++k) {
            if (k < nmine && lc == 0) {
                const int b = k % kNPatch;
                const bool ok = k < kNPatch || pt_wait(&p_empty[b], uint32_t(k / kNPatch - 1) & 1u, &s_abort, err);
                if (!__all_sync(FULLW, ok && s_abort == 0)) break;
                if (lane == 0) {
                    const BrickDesc d = desc[s_list[k]];
                    const BrickBox bb = desc_box(d);
                    const CUtensorMap *tm = &insts[d.inst].tmap;
                    if ((int)d.inst != last_inst) {
                        tc::fence_tensormap_acquire(tm);
                        last_inst = (int)d.inst;
                    }
                    tc::fence_proxy_async();   // earlier generic accesses of the buffer before the copy
                    tc::mbar_arrive_expect_tx(&t_full[b], kPatchBytes);
                    tc::tma_load_4d(sP + b * kPatBuf, tm, bb.x0, bb.y0, bb.z0, 0, &t_full[b]);
                }
                issued = k + 1;
            }
            const int j = k - kLoadAhead;
            if (j >= 0) {
                const int b = j % kNPatch;
                const bool ok = pt_wait(&t_full[b], uint32_t(j / kNPatch) & 1u, &s_abort, err);
                if (!__all_sync(FULLW, ok && s_abort == 0)) break;
                landed = j + 1;
                const BrickDesc d = desc[s_list[j]];
                const unsigned fl = desc_flags(d);
                float *P = sP + b * kPatBuf;
                if (fl) {   // V = E' u on the boundary control planes, one direction after the other
                    const TcInst &I = insts[d.inst];
                    const Geom &g = I.g;
                    const Edge &E = *I.edge;
                    const BrickBox bb = desc_box(d);
                    if (fl & 1u) {
                        for (int t = lane; t < kPY * kPZ; t += 32)
                            edge_in<0>(P, E, bb.x0, min(kPX, g.cx - bb.x0), lc * (kPY * kPZ) + t);
                        __syncwarp();
                    }
                    if (fl & 2u) {
                        for (int t = lane; t < kPX * kPZ; t += 32)
                            edge_in<1>(P, E, bb.y0, min(kPY, g.cy - bb.y0), lc * (kPX * kPZ) + t);
                        __syncwarp();
                    }
                    if (fl & 4u) {
                        for (int t = lane; t < kPX * kPY; t += 32)
                            edge_in<2>(P, E, bb.z0, min(kPZ, g.cz - bb.z0), lc * (kPX * kPY) + t);
                        __syncwarp();
                    }
                }
                tc::mbar_arrive(&p_full[b]);
            }
        }
        // after an abort: copies still in flight land before the CTA ends
        for (int j = landed; j < issued; ++j)
            tc::mbar_wait_bounded(&t_full[j % kNPatch], uint32_t(j / kNPatch) & 1u, kWaitLimit);
    } else if (lane == 0) {
        // ------------------------------ MMA issuer ------------------------------
        constexpr uint32_t idesc = tc::idesc_tf32(kTcM, kTcN);
        const bool b_ok = pt_wait(b_full, 0u, &s_abort, err);
        bool run = b_ok;
        // descriptors of K step 0 (hi and lo terms); the shared-memory window is below 256 KB,
        // so adding a step's offset never carries out of the address field
        const uint64_t dbh0 = tc::make_desc(sB, kBLbo, kSbo), dbl0 = tc::make_desc(sB + kBFl, kBLbo, kSbo);
        const uint64_t dal0 = tc::make_desc(sAlo, kALbo, kSbo), dal1 = tc::make_desc(sAlo + kAloFl, kALbo, kSbo);
        for (int it = 0, db = 0, dph = 0; it < nmine && run; ++it) {
            const int s = it & 1;
            // slot s holds brick it, and brick it - kNAcc has been drained from accumulator buffer
            // db (brick it is its use number it / kNAcc, dph the parity of that); on a failed wait
            // nothing more is issued
            run = pt_wait(&a_full[s], uint32_t(it >> 1) & 1u, &s_abort, err) &&
                  (it < kNAcc || pt_wait(&d_empty[db], uint32_t(dph ^ 1), &s_abort, err));
            if (!run) break;
            tc::fence_after_sync();
            const uint32_t acol = tmem + (uint32_t)(s * kColSlot);
            const uint32_t dacc = tmem + (uint32_t)(kColD + db * kTcN);
            const uint64_t dal = s ? dal1 : dal0;
#pragma unroll
            for (int ks = 0; ks < kTcKSteps; ++ks) {
                // one K step of 8 = two core-matrix columns: advance the start address fields
                const uint64_t dk = (uint64_t)(ks * 2 * kBLbo) >> 4, dka = (uint64_t)(ks * 2 * kALbo) >> 4;
                const uint64_t dbh = dbh0 + dk, dbl = dbl0 + dk;
                const uint32_t ah = acol + ks * 8;
                tc::mma_tf32(dacc, dal + dka, dbh, idesc, ks > 0 ? 1u : 0u);   // A_lo B_hi
                tc::mma_tf32_ts(dacc, ah, dbl, idesc, 1u);                     // A_hi B_lo
                tc::mma_tf32_ts(dacc, ah, dbh, idesc, 1u);                     // A_hi B_hi
            }
            tc::mma_commit(&d_full[db]);
            tc::mma_commit(&a_empty[s]);
            if (++db == kNAcc) {
                db = 0;
                dph ^= 1;
            }
        }
        if (run)
            for (int it = nmine - kNAcc; it < nmine; ++it)
                if (it >= 0 && !pt_wait(&d_empty[it % kNAcc], uint32_t(it / kNAcc) & 1u, &s_abort, err)) break;
        // every MMA this thread issued has completed once fin arrives; then TMEM may be released.
        // A B copy whose wait failed is waited for again, so it does not land after the CTA ends.
        tc::mma_commit(fin);
        tc::mbar_wait_bounded(fin, 0u, kWaitLimit);
        if (!b_ok) tc::mbar_wait_bounded(b_full, 0u, kWaitLimit);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kPtTmemCols);
    }
}

// sum of per-CTA partials -> out[slot] (one CTA)
__global__ void __launch_bounds__(kVecThreads) sum_partials_kernel(const double *__restrict__ partials, int np,
                                                                   double *__restrict__ out, int slot) {
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partials[i];
    s = block_sum(s);
    if (threadIdx.x == 0) out[slot] = s;
}

// x = 0, r = b; partial b'b
__global__ void __launch_bounds__(kVecThreads)
ir_init_kernel(long long n, const double *__restrict__ b, double *__restrict__ x, double *__restrict__ r,
               double *__restrict__ partials) {
    double bb = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double v = b[i];
        x[i] = 0.0;
        r[i] = v;
        bb += v * v;
    }
    bb = block_sum(bb);
    if (threadIdx.x == 0) partials[blockIdx.x] = bb;
}

// r32 = r / |r| (FP32), |r|^2 in scalars[0] (r = 0 gives r32 = 0)
__global__ void ir_to_f32_kernel(long long n, const double *__restrict__ r, float *__restrict__ r32,
                                 const double *__restrict__ scalars) {
    const double inv = scalars[0] > 0.0 ? 1.0 / sqrt(scalars[0]) : 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        r32[i] = float(r[i] * inv);
}

// r = b - y; partial r'r
__global__ void __launch_bounds__(kVecThreads)
ir_residual_kernel(long long n, const double *__restrict__ b, const double *__restrict__ y, double *__restrict__ r,
                   double *__restrict__ partials) {
    double rr = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double v = b[i] - y[i];
        r[i] = v;
        rr += v * v;
    }
    rr = block_sum(rr);
    if (threadIdx.x == 0) partials[blockIdx.x] = rr;
}

__global__ void to_f32_kernel(long long n, const double *__restrict__ a, float *__restrict__ b) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = float(a[i]);
}

// ---- fused vector step of the FP32 recurrence ------------------------------------------------
constexpr int kTailThreads = 256;

// Grid-wide barrier of a cooperative launch (every CTA resident).  The counter only grows (the
// host clears it before each solve); a CTA waits for the next multiple of gridDim.x above its own
// arrival.  Bounded by `limit` polls: false on time-out (err = 2), so a stuck barrier ends the
// kernel instead of hanging the GPU.
__device__ bool grid_sync(unsigned long long *ctr, int *err, long long limit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned long long old = atomicAdd(ctr, 1ull);
        const unsigned long long target = (old / gridDim.x + 1ull) * gridDim.x;
        int ok = 0;
        for (long long i = 0; i < limit; ++i) {   // each poll is an L2 round trip
            if (*(volatile unsigned long long *)ctr >= target) {
                ok = 1;
                break;
            }
        }
        if (!ok) atomicExch(err, 2);
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Arrival at the grid barrier by a CTA that has nothing after it (its system has stopped): the
// others still count it.
__device__ void grid_arrive(unsigned long long *ctr) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(ctr, 1ull);
    }
}

// Deterministic block reduction of N values at once; the sums are valid in thread 0.
template <int N>
__device__ __forceinline__ void block_sum_n(double (&v)[N]) {
    __shared__ double ws[N][kTailThreads / 32];
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < N; ++k) ws[k][threadIdx.x >> 5] = v[k];
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            double r = threadIdx.x < (blockDim.x >> 5) ? ws[k][threadIdx.x] : 0.0;
            v[k] = warp_sum(r);
        }
    }
}

// One launch for everything of a PCG iteration after the operator (rust/src/solver.rs:38-71),
// with one grid-wide barrier, for every system of the batch: system i is served by CTAs
// [cta0, cta0 + ncta) and reduces its own partials.
//   Phase A, one warp per row (iy, iz) of control points, lanes along x: Ap = the node sum of the
//   brick partials plus the sparse term, output rule applied; and five dot products p'Ap, z'Ap,
//   Ap'D^-1 Ap, r'Ap, Ap'Ap (z = D^-1 r).  The loads of a node (its <= 8 brick partials per
//   component, p, r, D^-1, the mask) are issued together.
//   Barrier.  Every CTA of the system reduces the same partials in the same order: the phase A
//   sums, and the exact r'r and r'z of the current r from the previous launch's phase B (or the
//   state's after an initialisation or replacement).  alpha = r'z / p'Ap, and for
//   r_new = r - alpha Ap, without another reduction,
//       |r_new|^2 = r'r - 2 alpha r'Ap + alpha^2 Ap'Ap,
//       r_new' D^-1 r_new = r'z - 2 alpha z'Ap + alpha^2 Ap'D^-1 Ap,
//   which give the convergence test and beta = r_new'z_new / r'z.  When the FP32 residual has
//   gained the replacement factor (or the segment is long) the state asks the host for an FP64
//   residual replacement instead.
//   Phase B, four elements per thread at a time: x += alpha p, r -= alpha Ap, p = D^-1 r + beta p
//   (when the iteration goes on) with the next apply's input pin (p with the fixed DOFs zeroed,
//   rows padded), and the exact r'r and r'z of the new r as per-CTA partials.  Those partials
//   alternate between two buffers by iteration parity, so a CTA that writes them never meets one
//   that still reads the previous ones.
// The system's first CTA writes its state.  All CTAs of a system take the same branches; the CTAs
// of a stopped system only arrive at the barrier.
__global__ void __launch_bounds__(kTailThreads, 4)
pcg_tail_kernel(const TcInst *__restrict__ insts, int ninst, unsigned long long *ctr, int *err, long long wait_limit) {
    __shared__ PcgState S;
    __shared__ double s_ab[2];
    __shared__ int s_stat, s_inst;
    if (threadIdx.x == 0) {
        int i = 0;
        while (i + 1 < ninst && (int)blockIdx.x >= insts[i + 1].cta0) ++i;
        s_inst = i;
        S = *insts[i].st;
    }
    __syncthreads();
    const TcInst &I = insts[s_inst];
    if (S.status != 0 || (int)blockIdx.x >= I.cta0 + I.ncta) {
        grid_arrive(ctr);
        return;
    }
    const Geom g = I.g;
    const int G = I.ncta, bid = (int)blockIdx.x - I.cta0;
    const uint8_t *__restrict__ mask = I.mask;
    const int mask_mode = I.mask_mode;
    const float *__restrict__ inv = I.inv;
    float *__restrict__ x = I.x;
    float *__restrict__ r = I.r;
    float *__restrict__ p = I.p;
    float *__restrict__ pin = I.pin;
    float *__restrict__ ap = I.ap;
    // partials: phase A [5][G]; exact r'r, r'z [2][G] in two buffers by iteration parity
    const int par = int(S.iter & 1);
    double *pa = I.part, *pb_new = I.part + (5 + 2 * par) * G, *pb_old = I.part + (7 - 2 * par) * G;
    // 32-bit indices: the set-up keeps the padded vectors below 2^31 values
    const int T = G * (int)blockDim.x;
    const int t0 = bid * (int)blockDim.x + (int)threadIdx.x;
    const int n = 3 * (int)g.nsc, nsc = (int)g.nsc;
    // A. Ap at every node and the five dot products
    double dA[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const float *__restrict__ patch = I.patch;
    {
        const int lane = threadIdx.x & 31;
        const int nrows = g.cy * g.cz;
        const int wstride = (G * (int)blockDim.x) >> 5;
        const size_t bstride = (size_t)3 * kPVol;
        for (int row = (bid * (int)blockDim.x + (int)threadIdx.x) >> 5; row < nrows; row += wstride) {
            const int iy = row % g.cy, iz = row / g.cy;
            int by[2], ly[2], bz[2], lz[2];
            const int nby = node_bricks(iy, kBY, g.nby, by, ly);
            const int nbz = node_bricks(iz, kBZ, g.nbz, bz, lz);
            // the row's partial rows in the y bricks (absent ones repeat the first and are not added)
            const size_t ybase0 = (size_t)g.nbx * by[0] * bstride + ly[0] * kPX;
            const size_t ybase1 = (size_t)g.nbx * by[nby - 1] * bstride + ly[nby - 1] * kPX;
            for (int ix = lane; ix < g.cx; ix += 32) {
                const int nd = row * g.cx + ix;
                const int bx1 = min(ix / kBX, g.nbx - 1), lx1 = ix - bx1 * kBX;
                const bool two = lx1 <= 1 && bx1 >= 1;   // also in the previous brick along x
                const int o1 = bx1 * (3 * kPVol) + lx1, o0 = two ? (bx1 - 1) * (3 * kPVol) + lx1 + kBX : o1;
                float sv[3] = {0.f, 0.f, 0.f};
                for (int a = 0; a < nbz; ++a) {   // z bricks, then y bricks, then x bricks: lower first
                    const float *zb = patch + (size_t)g.nbx * g.nby * bz[a] * bstride + lz[a] * (kPY * kPX);
                    float lo[2][3], hi[2][3];
#pragma unroll
                    for (int q2 = 0; q2 < 2; ++q2)
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const float *rb = zb + (q2 ? ybase1 : ybase0) + c * kPVol;
                            lo[q2][c] = rb[o0];
                            hi[q2][c] = rb[o1];
                        }
#pragma unroll
                    for (int q2 = 0; q2 < 2; ++q2)
                        if (q2 < nby)
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                if (two) sv[c] += lo[q2][c];
                                sv[c] += hi[q2][c];
                            }
                }
                float pv[3], rr[3], iv[3];
                bool mk[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int idx = c * nsc + nd;
                    pv[c] = p[idx];
                    rr[c] = r[idx];
                    iv[c] = inv[idx];
                    mk[c] = mask_mode == ICC_MASK_NONE || mask[idx];
                }
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int idx = c * nsc + nd;
                    float v = sv[c];
                    if (I.sp.ptr) v += sparse_row(I.sp, idx, p, mask, mask_mode);
                    if (!mk[c]) v = mask_mode == ICC_MASK_ZERO ? 0.f : pv[c];
                    ap[idx] = v;
                    const double av = double(v);
                    dA[0] += double(pv[c]) * av;
                    dA[1] += double(iv[c] * rr[c]) * av;
                    dA[2] += double(iv[c] * v) * av;
                    dA[3] += double(rr[c]) * av;
                    dA[4] += av * av;
                }
            }
        }
    }
    block_sum_n<5>(dA);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < 5; ++k) pa[k * G + bid] = dA[k];
    if (!grid_sync(ctr, err, wait_limit)) return;
    {
        double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int i = threadIdx.x; i < G; i += blockDim.x) {
#pragma unroll
            for (int k = 0; k < 5; ++k) v[k] += __ldcg(pa + k * G + i);
            if (!S.fresh) {
                v[5] += __ldcg(pb_old + i);
                v[6] += __ldcg(pb_old + G + i);
            }
        }
        block_sum_n<7>(v);
        if (threadIdx.x == 0) {
            // exact r'r and r'z of the current r: from the state after an initialisation or
            // replacement, else from the previous launch's phase B
            const double rr0 = S.fresh ? S.rr_old : v[5], rz0 = S.fresh ? S.rz_old : v[6];
            // rust/src/solver.rs:41-51 (alpha or breakdown), :56-71 (residual test, beta)
            S.iter += 1;
            S.p_ap = v[0];
            S.rz_prev = rz0;
            S.fresh = 0;
            if (!(v[0] > 0.0)) {
                S.status = isfinite(v[0]) ? kStatBreakdown : kStatNan;
            } else {
                const double alpha = rz0 / v[0];
                S.alpha = alpha;
                const double rr1 = fmax(rr0 - 2.0 * alpha * v[3] + alpha * alpha * v[4], 0.0);
                const double rz1 = rz0 - 2.0 * alpha * v[1] + alpha * alpha * v[2];
                const double res = sqrt(rr1) / S.norm_b;
                S.rel_res = res;
                S.rr_old = rr1;
                S.rz_old = rz1;
                if (res < S.tol) S.status = kStatConverged;
                else if (!isfinite(res) || !isfinite(rz1)) S.status = kStatNan;
                else {
                    S.beta = rz1 / rz0;
                    if (S.iter >= S.max_iter) S.status = kStatMaxIter;
                    else if (S.repl_delta > 0.0 && S.iter % S.repl_every == 0 &&
                             (S.rel_res < S.repl_delta * S.repl_res || S.iter - S.repl_iter >= S.repl_seg))
                        S.status = kStatReplace;
                }
            }
            s_stat = S.status;
            s_ab[0] = S.alpha;
            s_ab[1] = S.beta;
            if (bid == 0) *I.st = S;
        }
    }
    __syncthreads();
    tc::griddep_launch_dependents();   // the next apply may be scheduled (it waits for this grid)
    if (s_stat == kStatBreakdown || s_stat == kStatNan) return;
    // B. x += alpha p, r -= alpha Ap; the direction only when the iteration goes on.  Element i of
    // pin sits at i + (i / cx) (cxp - cx); the quotient and remainder are carried along.
    const float alpha = float(s_ab[0]), beta = float(s_ab[1]);
    const bool go = s_stat == 0;
    const bool ident = mask_mode == ICC_MASK_IDENTITY;
    const int pad = I.cxp - g.cx, Tq = T / g.cx, Tr = T % g.cx;
    int qrow = t0 / g.cx, qcol = t0 % g.cx;
    constexpr int kU = 4;
    double v[2] = {0.0, 0.0};
    for (int i0 = t0; i0 < n; i0 += kU * T) {
        float pv[kU], xv[kU], rv[kU], av[kU], iv[kU];
        bool ok[kU], mk[kU];
        int pidx[kU];
#pragma unroll
        for (int k = 0; k < kU; ++k) {
            const int i = i0 + k * T;
            ok[k] = i < n;
            pidx[k] = i + qrow * pad;
            qrow += Tq;
            qcol += Tr;
            if (qcol >= g.cx) {
                qcol -= g.cx;
                ++qrow;
            }
            if (ok[k]) {
                pv[k] = p[i];
                xv[k] = x[i];
                rv[k] = r[i];
                av[k] = ap[i];
                iv[k] = inv[i];
                mk[k] = !mask || mask[i];
            }
        }
#pragma unroll
        for (int k = 0; k < kU; ++k) {
            if (!ok[k]) continue;
            const int i = i0 + k * T;
            x[i] = xv[k] + alpha * pv[k];
            const float ri = rv[k] - alpha * av[k];
            r[i] = ri;
            const float zi = iv[k] * ri;
            v[0] += double(ri) * double(ri);
            v[1] += double(ri) * double(zi);
            if (go) {
                const float w = zi + beta * pv[k];
                const float wm = mk[k] ? w : 0.f;
                p[i] = ident ? w : wm;
                pin[pidx[k]] = wm;
            }
        }
    }
    block_sum_n<2>(v);
    if (threadIdx.x == 0) {
        pb_new[bid] = v[0];
        pb_new[G + bid] = v[1];
    }
}

// arm the replacement trigger after a residual replacement (or at the start)
__global__ void ru_arm_kernel(PcgState *st, double res, double delta, long long seg, long long every) {
    st->repl_res = res;
    st->repl_delta = delta;
    st->repl_iter = st->iter;
    st->repl_seg = seg;
    st->repl_every = every;
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------

static float host_tf32(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) {
        u += 0x1000u;
        u &= 0xffffe000u;
    }
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

template <class T>
static int dalloc(T **p, size_t count, const char *what) {
    *p = nullptr;
    ICC_CUDA(cudaMalloc((void **)p, (count ? count : 1) * sizeof(T)), what);
    return ICC_OK;
}

static bool inv3(const double *a, double *o) {
    const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                       a[2] * (a[3] * a[7] - a[4] * a[6]);
    if (!(std::fabs(det) > 1e-300)) return false;
    o[0] = (a[4] * a[8] - a[5] * a[7]) / det;
    o[1] = (a[2] * a[7] - a[1] * a[8]) / det;
    o[2] = (a[1] * a[5] - a[2] * a[4]) / det;
    o[3] = (a[5] * a[6] - a[3] * a[8]) / det;
    o[4] = (a[0] * a[8] - a[2] * a[6]) / det;
    o[5] = (a[2] * a[3] - a[0] * a[5]) / det;
    o[6] = (a[3] * a[7] - a[4] * a[6]) / det;
    o[7] = (a[1] * a[6] - a[0] * a[7]) / det;
    o[8] = (a[0] * a[4] - a[1] * a[3]) / det;
    return true;
}

// out = (R_z (x) R_y (x) R_x) in per component, on 81-vectors with element strides sin / sout
static void apply_r3(const double *Rx, const double *Ry, const double *Rz, const double *in, int sin, double *out,
                     int sout) {
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 27; ++a) {
            const int ax = a % 3, ay = (a / 3) % 3, az = a / 9;
            double s = 0.0;
            for (int b = 0; b < 27; ++b) {
                const int bx = b % 3, by = (b / 3) % 3, bz = b / 9;
                s += Rz[az * 3 + bz] * Ry[ay * 3 + by] * Rx[ax * 3 + bx] * in[(c * 27 + b) * sin];
            }
            out[(c * 27 + a) * sout] = s;
        }
}

// Values of the three uniform quadratic B-splines of an element at relative position t in [0, 1].
static void uniform_basis(double t, double b[3]) {
    b[0] = 0.5 * (1.0 - t) * (1.0 - t);
    b[1] = 0.5 + t - t * t;
    b[2] = 0.5 * t * t;
}

// Set-up of the tensor-core form:
//  * R of every 1-D element type: its three local B-splines in terms of the uniform ones,
//    N = R B, from the basis values at the element's three Gauss points;
//  * K_u = R_m^-1 K_m R_m^-T from the most frequent element type m, and the check that every
//    element type's matrix equals R K_u R' (to 1e-9 of max |K_u|);
//  * E along each direction, assembled from the elements' R (E[e + a][e + b] = R_e[a][b]), with
//    the checks that overlapping elements agree, that E differs from the identity only among the
//    control points 0, 1, n, n + 1, and that E couples only control points of a common element
//    (so a brick's patch holds what its boundary values need, and the transforms of single
//    bricks add up to the global one).
// Fills edge and kunif (81 x 81 row-major); ICC_BAD_ARG with the error set when the element
// matrices are not of this form.
static int setup_edge(const Op &op, Edge &edge, std::vector<double> &kunif) {
    const Geom &g = op.g;
    const int n[3] = {g.nx, g.ny, g.nz};
    // R per direction and 1-D type
    double xg[3] = {-std::sqrt(0.6), 0.0, std::sqrt(0.6)};
    double vu[9], vuinv[9];
    for (int q = 0; q < 3; ++q) {
        double b[3];
        uniform_basis(0.5 * (xg[q] + 1.0), b);
        for (int i = 0; i < 3; ++i) vu[3 * i + q] = b[i];
    }
    if (!inv3(vu, vuinv)) return set_error(ICC_BAD_ARG, "tensor-core path: singular uniform basis");
    std::vector<std::array<double, 9>> R1[3];
    for (int d = 0; d < 3; ++d) {
        if ((int)op.host_type1d[d].size() != n[d] || op.host_basis1d[d].empty())
            return set_error(ICC_BAD_ARG, "tensor-core path: space without 1-D basis data");
        for (const auto &vt : op.host_basis1d[d]) {
            std::array<double, 9> r;
            for (int i = 0; i < 3; ++i)
                for (int b = 0; b < 3; ++b) {
                    double acc = 0.0;
                    for (int q = 0; q < 3; ++q) acc += vt[3 * i + q] * vuinv[3 * q + b];
                    r[3 * i + b] = std::fabs(acc - (i == b ? 1.0 : 0.0)) < 1e-12 ? (i == b ? 1.0 : 0.0) : acc;
                }
            R1[d].push_back(r);
        }
    }
    // K_u from the most frequent element type
    std::vector<long long> count((size_t)op.ntypes, 0);
    for (int32_t t : op.host_type_id) count[(size_t)t]++;
    int mt = 0;
    for (int t = 1; t < op.ntypes; ++t)
        if (count[(size_t)t] > count[(size_t)mt]) mt = t;
    long long e0 = 0;
    while (op.host_type_id[(size_t)e0] != mt) ++e0;
    const int pos0[3] = {int(e0 % g.nx), int((e0 / g.nx) % g.ny), int(e0 / ((long long)g.nx * g.ny))};
    double Ri[3][9];
    for (int d = 0; d < 3; ++d)
        if (!inv3(R1[d][(size_t)op.host_type1d[d][(size_t)pos0[d]]].data(), Ri[d]))
            return set_error(ICC_BAD_ARG, "tensor-core path: singular 1-D basis");
    {
        const double *Km = op.host_ktypes.data() + (size_t)mt * 81 * 81;
        std::vector<double> t1(81 * 81);
        kunif.assign(81 * 81, 0.0);
        for (int j = 0; j < 81; ++j) apply_r3(Ri[0], Ri[1], Ri[2], Km + j, 81, t1.data() + j, 81);
        for (int i = 0; i < 81; ++i) apply_r3(Ri[0], Ri[1], Ri[2], t1.data() + i * 81, 1, kunif.data() + i * 81, 1);
    }
    double kmax = 0.0;
    for (double v : kunif) kmax = std::fmax(kmax, std::fabs(v));
    // every (element type, 1-D type triple) that occurs must be R K_u R'
    {
        std::vector<std::array<int, 4>> combos;
        for (int ez = 0; ez < g.nz; ++ez)
            for (int ey = 0; ey < g.ny; ++ey)
                for (int ex = 0; ex < g.nx; ++ex) {
                    const std::array<int, 4> k = {
                        op.host_type_id[(size_t)ex + (size_t)g.nx * ((size_t)ey + (size_t)g.ny * ez)],
                        op.host_type1d[0][(size_t)ex], op.host_type1d[1][(size_t)ey], op.host_type1d[2][(size_t)ez]};
                    if (std::find(combos.begin(), combos.end(), k) == combos.end()) combos.push_back(k);
                }
        std::vector<double> t1(81 * 81), t2(81 * 81);
        for (const auto &k : combos) {
            const double *Rx = R1[0][(size_t)k[1]].data(), *Ry = R1[1][(size_t)k[2]].data(), *Rz = R1[2][(size_t)k[3]].data();
            for (int j = 0; j < 81; ++j) apply_r3(Rx, Ry, Rz, kunif.data() + j, 81, t1.data() + j, 81);
            for (int i = 0; i < 81; ++i) apply_r3(Rx, Ry, Rz, t1.data() + i * 81, 1, t2.data() + i * 81, 1);
            const double *Kt = op.host_ktypes.data() + (size_t)k[0] * 81 * 81;
            double dmax = 0.0;
            for (int i = 0; i < 81 * 81; ++i) dmax = std::fmax(dmax, std::fabs(t2[(size_t)i] - Kt[i]));
            if (!(dmax <= 1e-9 * kmax))
                return set_error(ICC_BAD_ARG, "tensor-core path: an element matrix is not the uniform element matrix "
                                              "seen through its B-spline basis (element matrices must come from the "
                                              "space's own bases)");
        }
    }
    // E per direction
    std::memset(&edge, 0, sizeof(edge));
    for (int d = 0; d < 3; ++d) {
        const int nd = n[d];
        std::map<std::pair<int, int>, double> E;
        for (int e = 0; e < nd; ++e) {
            const auto &r = R1[d][(size_t)op.host_type1d[d][(size_t)e]];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    const std::pair<int, int> key(e + a, e + b);
                    const double v = r[(size_t)(3 * a + b)];
                    auto it = E.find(key);
                    if (it == E.end()) E.emplace(key, v);
                    else if (std::fabs(it->second - v) > 1e-12 * std::fmax(1.0, std::fabs(v)))
                        return set_error(ICC_BAD_ARG, "tensor-core path: element bases disagree on a shared B-spline");
                }
        }
        std::vector<int> ids;
        for (int i : {0, 1, nd, nd + 1})
            if (std::find(ids.begin(), ids.end(), i) == ids.end()) ids.push_back(i);
        auto in_ids = [&](int i) { return std::find(ids.begin(), ids.end(), i) != ids.end(); };
        bool identity = true;
        for (const auto &kv : E) {
            const int i = kv.first.first, j = kv.first.second;
            const double dev = std::fabs(kv.second - (i == j ? 1.0 : 0.0));
            if (dev == 0.0) continue;
            identity = false;
            if (!in_ids(i) || !in_ids(j))
                return set_error(ICC_BAD_ARG, "tensor-core path: the B-spline extraction is not confined to the two "
                                              "first and two last control points");
            // every element whose control points include j also includes i
            for (int e = std::max(0, j - 2); e <= std::min(nd - 1, j); ++e)
                if (i < e || i > e + 2)
                    return set_error(ICC_BAD_ARG, "tensor-core path: the B-spline extraction couples control points "
                                                  "of different elements");
        }
        if (identity) continue;
        edge.nb[d] = int(ids.size());
        for (size_t a = 0; a < ids.size(); ++a) {
            edge.id[d][a] = ids[a];
            for (size_t b = 0; b < ids.size(); ++b) {
                auto it = E.find({ids[a], ids[b]});
                edge.e[d][a][b] = float(it == E.end() ? 0.0 : it->second);
            }
        }
    }
    return ICC_OK;
}

// The tensor map of a system's apply input: dimensions (cx, cy, cz, 3) with row pitch cxp, boxes of
// 12 x 6 x 6 x 3 floats (one brick's patch), zero fill outside the grid.  The driver's encoder is
// looked up through the runtime, so the library needs no link to the driver library.
static int encode_input_map(const Op &op, VecSet &v) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return set_error(ICC_CUDA_ERROR, "cuTensorMapEncodeTiled is not available");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[4] = {(cuuint64_t)op.g.cx, (cuuint64_t)op.g.cy, (cuuint64_t)op.g.cz, 3};
    const cuuint64_t strides[3] = {(cuuint64_t)v.cxp * 4, (cuuint64_t)v.cxp * op.g.cy * 4,
                                   (cuuint64_t)v.cxp * op.g.cy * op.g.cz * 4};
    const cuuint32_t box[4] = {kPXs, kPY, kPZ, 3};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = encode(&v.tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, v.pin32, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(ICC_CUDA_ERROR, "tensor map of the apply input: error " + std::to_string((int)r));
    return ICC_OK;
}

static int vecset_alloc(const Op &op, VecSet &v, int part_cap) {
    const size_t n = (size_t)op.ndof;
    int rc;
    if ((rc = dalloc(&v.patch32, (size_t)op.g.nbricks * 3 * kPVol, "alloc mixed"))) return rc;
    float **f32[] = {&v.rhs32, &v.x32, &v.r32, &v.p32, &v.ap32, &v.inv32};
    for (float **p : f32)
        if ((rc = dalloc(p, n, "alloc mixed"))) return rc;
    v.cxp = (op.g.cx + 3) & ~3;
    const size_t npad = (size_t)3 * v.cxp * op.g.cy * op.g.cz;
    if ((rc = dalloc(&v.pin32, npad, "alloc mixed"))) return rc;
    ICC_CUDA(cudaMemset(v.pin32, 0, npad * sizeof(float)), "clear apply input");
    if ((rc = encode_input_map(op, v))) return rc;
    double **f64[] = {&v.x64, &v.r64, &v.y64};
    for (double **p : f64)
        if ((rc = dalloc(p, n, "alloc mixed"))) return rc;
    if ((rc = dalloc(&v.part, (size_t)9 * part_cap, "alloc mixed"))) return rc;
    v.part_cap = part_cap;
    return ICC_OK;
}

static void vecset_free(VecSet &v) {
    void *bufs[] = {v.patch32, v.rhs32, v.x32, v.r32, v.p32, v.ap32, v.inv32, v.pin32, v.x64, v.r64, v.y64, v.part};
    for (void *p : bufs)
        if (p) cudaFree(p);
    v = VecSet();
}

// CTAs of the fused vector step that can be resident at once (its grid barrier needs all of them)
static int tail_capacity(const Op &op) { return op.mixed->tail_per_sm * op.num_sms; }

// The bricks of system `inst` (the handle op) in brick order, for a batch's brick list.
static void append_descs(const Op &op, int inst, std::vector<BrickDesc> &out) {
    const Geom &g = op.g;
    const std::vector<uint8_t> &fl = op.mixed->flags;
    for (int b = 0; b < g.nbricks; ++b) {
        const int bx = b % g.nbx, by = (b / g.nbx) % g.nby, bz = b / (g.nbx * g.nby);
        BrickDesc d;
        d.inst = inst;
        d.local = b;
        d.xyz = unsigned(bx) | unsigned(by) << 11 | unsigned(bz) << 22;
        const unsigned ex = unsigned(std::min(kBX, g.nx - bx * kBX)), ey = unsigned(std::min(kBY, g.ny - by * kBY)),
                       ez = unsigned(std::min(kBZ, g.nz - bz * kBZ));
        d.ext = ex | ey << 4 | ez << 8 | unsigned(fl[(size_t)b]) << 12;
        out.push_back(d);
    }
}

static int mixed_init(Op &op) {
    if (op.mixed && op.mixed->ready) return ICC_OK;
    if (3LL * ((op.g.cx + 3) & ~3) * op.g.cy * op.g.cz + 4LL * kTailThreads * 1024 >= (1LL << 31))
        return set_error(ICC_BAD_ARG, "tensor-core path: more than 2^31 DOF");
    if (op.g.nbx > 2047 || op.g.nby > 2047 || op.g.nbz > 2047)
        return set_error(ICC_BAD_ARG, "tensor-core path: more than 2047 bricks along a direction");
    if (!op.mixed) op.mixed = new MixedState();
    MixedState &ms = *op.mixed;
    int rc = setup_edge(op, ms.edge, ms.kunif);
    if (rc) return rc;
    // the uniform element matrix split into TF32 hi/lo in the canonical layout, component c of
    // the test (row) and trial (column) DOFs at c*32 + [0, 27)
    std::vector<float> bm((size_t)2 * kBFl, 0.f);
    {
        const double *K = ms.kunif.data();
        float *hi = bm.data(), *lo = hi + kBFl;
        for (int n = 0; n < 81; ++n)
            for (int k = 0; k < 81; ++k) {
                const double v = K[n * 81 + k];
                const float h = host_tf32(float(v));
                const float l = host_tf32(float(v - double(h)));
                const int nr = (n / 27) * 32 + n % 27, kc = (k / 27) * 32 + k % 27;
                hi[canon(nr, kc, kTcN)] = h;
                lo[canon(nr, kc, kTcN)] = l;
            }
    }
    if ((rc = dalloc(&ms.d_bmat, bm.size() / 4, "alloc tc matrices"))) return rc;
    ICC_CUDA(cudaMemcpyAsync(ms.d_bmat, bm.data(), bm.size() * 4, cudaMemcpyHostToDevice, op.stream), "copy tc matrices");
    const Geom &g = op.g;
    {
        // bit d of a brick: its patch holds boundary control points of direction d
        std::vector<uint8_t> fl((size_t)g.nbricks, 0);
        const int be[3] = {kBX, kBY, kBZ}, cp[3] = {g.cx, g.cy, g.cz};
        for (int b = 0; b < g.nbricks; ++b) {
            const int bi[3] = {b % g.nbx, (b / g.nbx) % g.nby, b / (g.nbx * g.nby)};
            for (int d = 0; d < 3; ++d) {
                const int o = bi[d] * be[d], ext = std::min(be[d] + 2, cp[d] - o);
                for (int a = 0; a < ms.edge.nb[d]; ++a)
                    if (ms.edge.id[d][a] >= o && ms.edge.id[d][a] < o + ext) fl[(size_t)b] |= uint8_t(1u << d);
            }
        }
        ms.flags = fl;
        if ((g.nbricks + op.num_sms - 1) / op.num_sms > kMaxListPerCta)
            return set_error(ICC_BAD_ARG, "tensor-core path: more than 2048 bricks per SM");
        std::vector<BrickDesc> dv;
        append_descs(op, 0, dv);
        if ((rc = dalloc(&ms.d_desc, dv.size(), "alloc brick list"))) return rc;
        if ((rc = dalloc(&ms.d_edge, 1, "alloc edge"))) return rc;
        ICC_CUDA(cudaMemcpyAsync(ms.d_desc, dv.data(), dv.size() * sizeof(BrickDesc), cudaMemcpyHostToDevice, op.stream),
                 "copy brick list");
        ICC_CUDA(cudaMemcpyAsync(ms.d_edge, &ms.edge, sizeof(Edge), cudaMemcpyHostToDevice, op.stream), "copy edge");
        ICC_CUDA(cudaStreamSynchronize(op.stream), "copy brick list");
    }
    {
        int per_sm = 0;
        ICC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_tail_kernel, kTailThreads, 0),
                 "tail occupancy");
        ms.tail_per_sm = std::max(1, std::min(per_sm, 4));
    }
    if ((rc = dalloc(&ms.d_scale32, (size_t)op.nel, "alloc mixed"))) return rc;
    if ((rc = vecset_alloc(op, ms.v, tail_capacity(op)))) return rc;
    if ((rc = dalloc(&ms.d_scalars, 8, "alloc mixed"))) return rc;
    if ((rc = dalloc(&ms.d_grid_ctr, 1, "alloc mixed"))) return rc;
    if ((rc = dalloc(&ms.d_err, 1, "alloc mixed"))) return rc;
    if ((rc = dalloc(&ms.d_state, 1, "alloc mixed"))) return rc;
    if ((rc = dalloc(&ms.d_inst, 2, "alloc mixed"))) return rc;   // [0] plain apply, [1] the handle's solve
    ICC_CUDA(cudaMallocHost((void **)&ms.h_state, sizeof(PcgState)), "alloc pinned");
    ICC_CUDA(cudaMallocHost((void **)&ms.h_scalars, 8 * sizeof(double)), "alloc pinned");
    ICC_CUDA(cudaMallocHost((void **)&ms.h_err, sizeof(int)), "alloc pinned");
    ICC_CUDA(cudaMemsetAsync(ms.d_err, 0, sizeof(int), op.stream), "clear err");
    ICC_CUDA(cudaMemsetAsync(ms.d_grid_ctr, 0, sizeof(unsigned long long), op.stream), "clear grid counter");
    ICC_CUDA(cudaStreamSynchronize(op.stream), "clear err");
    ICC_CUDA(cudaFuncSetAttribute(apply_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPtSmem),
             "cudaFuncSetAttribute tc");
    ms.ready = true;
    return mixed_on_scale_update(op);
}

void mixed_release(Op &op) {
    if (!op.mixed) return;
    MixedState &ms = *op.mixed;
    if (ms.graph) cudaGraphExecDestroy(ms.graph);
    vecset_free(ms.v);
    void *bufs[] = {ms.d_bmat, ms.d_desc, ms.d_edge, ms.d_scale32, ms.d_scalars, ms.d_err, ms.d_state,
                    ms.d_grid_ctr, ms.d_inst};
    for (void *p : bufs)
        if (p) cudaFree(p);
    if (ms.h_state) cudaFreeHost(ms.h_state);
    if (ms.h_scalars) cudaFreeHost(ms.h_scalars);
    if (ms.h_err) cudaFreeHost(ms.h_err);
    delete op.mixed;
    op.mixed = nullptr;
}

int mixed_on_scale_update(Op &op) {
    if (!op.mixed || !op.mixed->ready) return ICC_OK;
    MixedState &ms = *op.mixed;
    to_f32_kernel<<<op.vec_blocks, kVecThreads, 0, op.stream>>>(op.nel, op.d_scale, ms.d_scale32);
    ICC_CUDA(cudaGetLastError(), "scale to f32");
    return ICC_OK;
}

// xm = mask .* x (the brick apply reads its input unmasked)
// pin = x with the fixed DOFs zeroed (mask given), rows of cx values stored with pitch cxp; one
// warp per row of control points
__global__ void pad_input_kernel(long long rows, int cx, int cxp, const float *__restrict__ x,
                                 const uint8_t *__restrict__ mask, float *__restrict__ pin) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long rw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; rw < rows; rw += warps)
        for (int ix = lane; ix < cx; ix += 32) {
            const long long i = rw * cx + ix;
            pin[rw * cxp + ix] = (mask && !mask[i]) ? 0.f : x[i];
        }
}

static void enqueue_pad_input(const Op &op, const VecSet &v, const float *x, cudaStream_t s) {
    const uint8_t *mask = op.mask_mode != ICC_MASK_NONE ? op.d_mask : nullptr;
    pad_input_kernel<<<op.vec_blocks, kVecThreads, 0, s>>>(3LL * op.g.cy * op.g.cz, op.g.cx, v.cxp, x, mask, v.pin32);
}

// The instance entry of system (op, v) with PCG state st (null: a plain apply of v.pin32).
static TcInst make_inst(const Op &op, const VecSet &v, PcgState *st, int cta0, int ncta, float kfac) {
    const MixedState &ms = *op.mixed;
    TcInst I;
    std::memset(&I, 0, sizeof(I));
    I.g = op.g;
    I.cta0 = cta0;
    I.ncta = ncta;
    I.kfac = kfac;
    I.tmap = v.tmap;
    I.scale = ms.d_scale32;
    I.edge = ms.d_edge;
    I.patch = v.patch32;
    I.mask = op.mask_mode != ICC_MASK_NONE ? op.d_mask : nullptr;
    I.mask_mode = op.mask_mode;
    I.sp = op.extra32();
    I.inv = v.inv32;
    I.x = v.x32;
    I.r = v.r32;
    I.p = v.p32;
    I.pin = v.pin32;
    I.cxp = v.cxp;
    I.ap = v.ap32;
    I.part = v.part;
    I.st = st;
    return I;
}

// The apply may start while the previous kernel of the stream finishes (programmatic dependent
// launch): it sets up TMEM, its barriers and the B copy, then waits for that kernel.
static cudaError_t launch_apply_tc(cudaStream_t s, const TcInst *d_insts, int ninst, int nbricks,
                                   const BrickDesc *d_desc, const float4 *bmat, int *err, int num_sms) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)std::min(num_sms, nbricks));
    cfg.blockDim = dim3(kPtThreads);
    cfg.dynamicSmemBytes = kPtSmem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, apply_tc_kernel, d_insts, ninst, nbricks, d_desc, bmat, err);
}

static cudaError_t launch_tail(cudaStream_t s, const TcInst *d_insts, int ninst, int grid, unsigned long long *ctr,
                               int *err, long long limit) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kTailThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;   // the grid barrier needs every CTA resident
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, pcg_tail_kernel, d_insts, ninst, ctr, err, limit);
}

// enqueue y32 = A x32 with the tensor-core apply: the input goes to the padded apply input (fixed
// DOFs of a masked operator zeroed), the node-side pass applies the output rule
static int enqueue_apply_tc(Op &op, const float *x, float *y) {
    MixedState &ms = *op.mixed;
    enqueue_pad_input(op, ms.v, x, op.stream);
    const TcInst I = make_inst(op, ms.v, nullptr, 0, 0, 1.f);
    ICC_CUDA(cudaMemcpyAsync(ms.d_inst, &I, sizeof(TcInst), cudaMemcpyHostToDevice, op.stream), "instance table");
    ICC_CUDA(launch_apply_tc(op.stream, ms.d_inst, 1, op.g.nbricks, ms.d_desc, ms.d_bmat, ms.d_err, op.num_sms),
             "tc apply launch");
    gather_kernel<float><<<op.vec_blocks, kVecThreads, 0, op.stream>>>(op.g, ms.v.patch32, x, op.d_mask,
                                                                       op.mask_mode, op.extra32(), y, nullptr, nullptr);
    ICC_CUDA(cudaGetLastError(), "tc apply launch");
    return ICC_OK;
}

// Clears the device error flag and the grid-barrier counter before a call, so a handle whose
// previous call timed out starts clean (stream-ordered before the call's kernels).
static int clear_flags(cudaStream_t s, int *d_err, unsigned long long *d_ctr) {
    ICC_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), s), "clear err");
    ICC_CUDA(cudaMemsetAsync(d_ctr, 0, sizeof(unsigned long long), s), "clear grid counter");
    return ICC_OK;
}

static int timeout_error(int err) {
    return set_error(ICC_TIMEOUT, err == 2 ? "fused vector step: grid barrier wait ran out"
                                           : "tensor-core apply: mbarrier wait ran out");
}

// y32 = A x32 on the tensor cores (icc_op_apply_f32).
int mixed_apply_f32(Op &op, const float *x, float *y) {
    int rc = mixed_init(op);
    if (rc) return rc;
    MixedState &ms = *op.mixed;
    if ((rc = clear_flags(op.stream, ms.d_err, ms.d_grid_ctr))) return rc;
    if ((rc = enqueue_apply_tc(op, x, y))) return rc;
    ICC_CUDA(cudaMemcpyAsync(ms.h_err, ms.d_err, sizeof(int), cudaMemcpyDeviceToHost, op.stream), "err");
    ICC_CUDA(cudaStreamSynchronize(op.stream), "tc apply");
    if (*ms.h_err) return timeout_error(*ms.h_err);
    return ICC_OK;
}

// The captured iteration graph holds kernel arguments by value; it is rebuilt after they change.
void mixed_invalidate_graph(Op &op) {
    if (!op.mixed || !op.mixed->graph) return;
    cudaGraphExecDestroy(op.mixed->graph);
    op.mixed->graph = nullptr;
    op.mixed->graph_batch = 0;
}

// Polls of a grid barrier before the fused vector step gives up (ICC_TIMEOUT).
int mixed_set_wait_limit(Op &op, long long polls) {
    int rc = mixed_init(op);
    if (rc) return rc;
    op.mixed->grid_wait_limit = polls;
    return ICC_OK;
}

// Mean device ms of the brick kernel and of the node-side pass over `reps` FP32 applies.
int mixed_profile_apply(Op &op, const float *x, float *y, int reps, double *contract_ms, double *gather_ms) {
    int rc = mixed_init(op);
    if (rc) return rc;
    MixedState &ms = *op.mixed;
    if ((rc = clear_flags(op.stream, ms.d_err, ms.d_grid_ctr))) return rc;
    enqueue_pad_input(op, ms.v, x, op.stream);
    const TcInst I = make_inst(op, ms.v, nullptr, 0, 0, 1.f);
    ICC_CUDA(cudaMemcpyAsync(ms.d_inst, &I, sizeof(TcInst), cudaMemcpyHostToDevice, op.stream), "instance table");
    std::vector<cudaEvent_t> ev(3 * size_t(reps));
    for (auto &e : ev) ICC_CUDA(cudaEventCreate(&e), "event create");
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(ev[3 * r], op.stream);
        ICC_CUDA(launch_apply_tc(op.stream, ms.d_inst, 1, op.g.nbricks, ms.d_desc, ms.d_bmat, ms.d_err, op.num_sms),
                 "tc apply launch");
        cudaEventRecord(ev[3 * r + 1], op.stream);
        gather_kernel<float><<<op.vec_blocks, kVecThreads, 0, op.stream>>>(op.g, ms.v.patch32, x, op.d_mask,
                                                                           ICC_MASK_NONE, op.extra32(), y, nullptr,
                                                                           nullptr);
        cudaEventRecord(ev[3 * r + 2], op.stream);
    }
    cudaError_t e = cudaEventSynchronize(ev.back());
    double a = 0.0, gt = 0.0;
    for (int r = 0; r < reps && e == cudaSuccess; ++r) {
        float t1 = 0.f, t2 = 0.f;
        cudaEventElapsedTime(&t1, ev[3 * r], ev[3 * r + 1]);
        cudaEventElapsedTime(&t2, ev[3 * r + 1], ev[3 * r + 2]);
        a += t1;
        gt += t2;
    }
    for (auto &x2 : ev) cudaEventDestroy(x2);
    ICC_CUDA(e, "profile tc apply");
    ICC_CUDA(cudaMemcpyAsync(ms.h_err, ms.d_err, sizeof(int), cudaMemcpyDeviceToHost, op.stream), "err");
    ICC_CUDA(cudaStreamSynchronize(op.stream), "err");
    if (*ms.h_err) return timeout_error(*ms.h_err);
    *contract_ms = a / reps;
    *gather_ms = gt / reps;
    return ICC_OK;
}

// x64 += sigma * xs32; xs32 = 0
__global__ void ru_accumulate_kernel(long long n, double *__restrict__ x, float *__restrict__ xs, double sigma) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        x[i] += sigma * double(xs[i]);
        xs[i] = 0.f;
    }
}

// r32 = r64 / sigma (the FP64 residual replaces the FP32 recurrence residual); partials r'z, r'r
__global__ void __launch_bounds__(kVecThreads)
ru_replace_kernel(long long n, const double *__restrict__ r64, double inv_sigma, const float *__restrict__ inv,
                  float *__restrict__ r32, double *__restrict__ partials) {
    double rz = 0.0, rr = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float ri = float(r64[i] * inv_sigma);
        r32[i] = ri;
        rz += double(ri) * double(inv[i] * ri);
        rr += double(ri) * double(ri);
    }
    rz = block_sum(rz);
    rr = block_sum(rr);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = rz;
        partials[2 * blockIdx.x + 1] = rr;
    }
}

// continue the FP32 iteration from the replaced residual: the next search direction is
// p = z + beta p with beta = r'z (replaced) / r'z (of the last alpha), as a reliable update does
__global__ void __launch_bounds__(kVecThreads)
ru_replace_finalize(const double *__restrict__ partials, int np, PcgState *st) {
    double rz = 0.0, rr = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        rz += partials[2 * i];
        rr += partials[2 * i + 1];
    }
    rz = block_sum(rz);
    rr = block_sum(rr);
    if (threadIdx.x == 0) {
        st->beta = rz / st->rz_prev;
        st->rz_old = rz;
        st->rr_old = rr;
        st->fresh = 1;   // the next fused step takes r'r and r'z from here
        st->rel_res = sqrt(rr) / st->norm_b;
        st->status = 0;
    }
}

// ---- the mixed-precision solve of one or several systems ------------------------------------

// Per-system inputs, outputs and loop state of a (batched) mixed solve.
struct MixedItem {
    Op *op = nullptr;
    VecSet *v = nullptr;
    const double *b = nullptr, *diag = nullptr;
    double tol = 0.0;
    int64_t max_iter = 0;
    double *x_out = nullptr;
    float kfac = 1.f;
    // results
    int status = ICC_NOT_CONVERGED;
    int64_t iters = 0, updates = 0;
    double rel_res = 1.0;
    // loop state
    double nb = 1.0, res = 1.0, best = INFINITY;
    int no_progress = 0;
    bool done = false;
};

// The device side of a (batched) mixed solve: the instance table, the systems' states (one
// array, read back with one copy per graph batch) and the captured iteration graph.
struct MixedBatch {
    cudaStream_t stream = nullptr;
    TcInst *d_inst = nullptr;
    BrickDesc *d_desc = nullptr;   // all bricks of all systems, system by system
    PcgState *d_state = nullptr, *h_state = nullptr;
    double *d_scalars = nullptr, *h_scalars = nullptr;   // |b|^2 and |r|^2 per system
    int *d_err = nullptr, *h_err = nullptr;
    unsigned long long *d_ctr = nullptr;
    cudaGraphExec_t graph = nullptr;
    int ninst = 0, nbricks = 0, tail_grid = 0, num_sms = 148;
    const float4 *bmat = nullptr;
    long long limit = kGridWaitLimit;
    bool owned = false;   // allocated for this call (a batch), else borrowed from the handle
    ~MixedBatch() {
        if (!owned) return;
        if (graph) cudaGraphExecDestroy(graph);
        void *bufs[] = {d_inst, d_desc, d_state, d_scalars, d_err, d_ctr};
        for (void *p : bufs)
            if (p) cudaFree(p);
        if (h_state) cudaFreeHost(h_state);
        if (h_scalars) cudaFreeHost(h_scalars);
        if (h_err) cudaFreeHost(h_err);
    }
};

// Shares `cap` CTAs of the fused vector step among the systems: every system gets at least one,
// the rest in proportion to its control points (mode 0) or in equal parts (mode 1), never more
// than one per 256 control points.
static std::vector<int> share_ctas(const std::vector<MixedItem> &items, int cap, int mode = 0) {
    const size_t m = items.size();
    std::vector<int> n(m, 1);
    long long tot = 0;
    for (const auto &it : items) tot += it.op->g.nsc;
    for (size_t i = 0; i < m; ++i) {
        const long long need = (items[i].op->g.nsc + kTailThreads - 1) / kTailThreads;
        const double frac = mode == 0 ? (double)items[i].op->g.nsc / (double)tot : 1.0 / (double)m;
        const long long want = (long long)((double)(cap - (int)m) * frac);
        n[i] += (int)std::max(0LL, std::min(need - 1, want));
    }
    return n;
}

// Runs the graph batches of a (batched) mixed solve until every system has stopped.
//
// Reliable-update PCG per system: the Jacobi-PCG recurrence runs in FP32 on the tensor-core
// operator; whenever its residual has fallen by `delta` since the last replacement (or below tol),
// the FP32 solution increment is folded into the FP64 solution, the true residual b - A x is
// recomputed with the FP64 operator, and the FP32 residual is replaced by it while the search
// direction is kept.  A system stops when its FP64 residual meets its tolerance (the reference's
// stopping rule, rust/src/solver.rs:56-58, evaluated on the true residual), on breakdown or NaN,
// or when its iteration budget or progress runs out.
constexpr int64_t kMaxSegment = 512;  // FP32 iterations between residual replacements at most

// Initial state of every system: x = 0, r = b, |b|, the FP32 recurrence armed for residual
// replacement by the factor delta (0: never, as the autotuner runs it), tolerance tol of the
// system (trial: 0, so no system stops while candidates are timed).
static int init_items(MixedBatch &bt, std::vector<MixedItem> &items, double delta, int check_every, bool trial,
                      int64_t &launches) {
    cudaStream_t s = bt.stream;
    const size_t m = items.size();
    int rc;
    if ((rc = clear_flags(s, bt.d_err, bt.d_ctr))) return rc;
    for (size_t i = 0; i < m; ++i) {
        MixedItem &it = items[i];
        Op &op = *it.op;
        VecSet &v = *it.v;
        const double *diag = it.diag;
        if (!diag) {
            op.enqueue_diagonal(op.d_diag, s);
            diag = op.d_diag;
            launches++;
        }
        inv_diag_kernel<float><<<op.vec_blocks, kVecThreads, 0, s>>>(op.ndof, diag, v.inv32);
        ir_init_kernel<<<op.vec_blocks, kVecThreads, 0, s>>>(op.ndof, it.b, v.x64, v.r64, op.d_partials);
        sum_partials_kernel<<<1, kVecThreads, 0, s>>>(op.d_partials, op.vec_blocks, bt.d_scalars, (int)i);
        launches += 3;
    }
    ICC_CUDA(cudaMemcpyAsync(bt.h_scalars, bt.d_scalars, m * sizeof(double), cudaMemcpyDeviceToHost, s), "scalars");
    ICC_CUDA(cudaStreamSynchronize(s), "mixed init");
    for (size_t i = 0; i < m; ++i) {
        MixedItem &it = items[i];
        Op &op = *it.op;
        VecSet &v = *it.v;
        it.nb = std::fmax(std::sqrt(bt.h_scalars[i]), 1e-16);   // FP32 quantities are scaled by 1 / |b|
        if (it.max_iter == 0) {
            it.done = true;
            it.status = ICC_NOT_CONVERGED;
            it.rel_res = 1.0;
            // a stopped state, so the kernels skip the system
            ru_arm_kernel<<<1, 1, 0, s>>>(bt.d_state + i, 1.0, 0.0, kMaxSegment, check_every);
            pcg_init_finalize<<<1, kVecThreads, 0, s>>>(op.d_partials, 0, bt.d_state + i, it.tol, 0);
            launches += 2;
            continue;
        }
        const uint8_t *pm = op.mask_mode == ICC_MASK_ZERO ? op.d_mask : nullptr;
        ir_to_f32_kernel<<<op.vec_blocks, kVecThreads, 0, s>>>(op.ndof, v.r64, v.rhs32, bt.d_scalars + i);
        pcg_init_kernel<float><<<op.vec_blocks, kVecThreads, 0, s>>>(op.ndof, v.rhs32, v.inv32, v.x32, v.r32, v.p32,
                                                                     op.d_partials, pm);
        pcg_init_finalize<<<1, kVecThreads, 0, s>>>(op.d_partials, op.vec_blocks, bt.d_state + i, trial ? 0.0 : it.tol,
                                                    trial ? (1LL << 40) : (long long)it.max_iter);
        ru_arm_kernel<<<1, 1, 0, s>>>(bt.d_state + i, 1.0, trial ? 0.0 : delta, kMaxSegment, check_every);
        launches += 4;
        enqueue_pad_input(op, v, v.p32, s);
        launches++;
    }
    ICC_CUDA(cudaGetLastError(), "mixed init");
    return ICC_OK;
}

static int run_mixed(MixedBatch &bt, std::vector<MixedItem> &items, const icc_solve_opts &opts, int64_t *launches_out) {
    cudaStream_t s = bt.stream;
    const size_t m = items.size();
    // 0.6: a replacement every ~75 iterations at 128x64x64 keeps the FP32 recurrence close to the
    // FP64 iteration count (1,350-1,410 vs 1,337 over four seeds; 0.1 gave up to 1,820)
    const double delta = opts.inner_tol > 0.0 ? opts.inner_tol : 0.6;
    const int max_updates = opts.max_outer > 0 ? opts.max_outer : 1000;
    const int check_every = opts.check_every > 0 ? opts.check_every : 32;
    // give up after the FP32 recurrence has gained eight decades (8 ln 0.1 / ln delta replacements)
    // without a 10% improvement of the true residual
    const int max_no_progress = std::max(8, (int)std::ceil(8.0 * std::log(0.1) / std::log(std::fmin(delta, 0.99))));
    int64_t launches = 0;
    int rc;
    if ((rc = init_items(bt, items, delta, check_every, false, launches))) return rc;

    int64_t launched = 0, max_budget = 0;
    for (const auto &it : items) max_budget = std::max(max_budget, it.max_iter);
    size_t active = 0;
    for (const auto &it : items) active += it.done ? 0 : 1;
    while (active > 0) {
        ICC_CUDA(cudaGraphLaunch(bt.graph, s), "graph launch");
        launches += 2 * int64_t(check_every);
        launched += check_every;
        ICC_CUDA(cudaMemcpyAsync(bt.h_state, bt.d_state, m * sizeof(PcgState), cudaMemcpyDeviceToHost, s), "state");
        ICC_CUDA(cudaMemcpyAsync(bt.h_err, bt.d_err, sizeof(int), cudaMemcpyDeviceToHost, s), "err");
        ICC_CUDA(cudaStreamSynchronize(s), "inner sync");
        if (*bt.h_err) return timeout_error(*bt.h_err);   // a bounded wait ran out in this batch
        // systems that asked for a replacement or stopped: reliable update x += sigma xs, r = b - A x in FP64
        std::vector<size_t> upd;
        for (size_t i = 0; i < m; ++i)
            if (!items[i].done && bt.h_state[i].status != 0) upd.push_back(i);
        if (upd.empty()) {
            if (launched > max_budget + 2 * int64_t(check_every))
                return set_error(ICC_TIMEOUT, "mixed solve: device state did not reach a stop condition");
            continue;
        }
        for (size_t i : upd) {
            MixedItem &it = items[i];
            Op &op = *it.op;
            VecSet &v = *it.v;
            ru_accumulate_kernel<<<op.vec_blocks, kVecThreads, 0, s>>>(op.ndof, v.x64, v.x32, it.nb);
            op.enqueue_apply_on(s, v.x64, v.y64);
            ir_residual_kernel<<<op.vec_blocks, kVecThreads, 0, s>>>(op.ndof, it.b, v.y64, v.r64, op.d_partials);
            sum_partials_kernel<<<1, kVecThreads, 0, s>>>(op.d_partials, op.vec_blocks, bt.d_scalars, (int)i);
            launches += 5;
        }
        ICC_CUDA(cudaMemcpyAsync(bt.h_scalars, bt.d_scalars, m * sizeof(double), cudaMemcpyDeviceToHost, s), "scalars");
        ICC_CUDA(cudaStreamSynchronize(s), "update sync");
        for (size_t i : upd) {
            MixedItem &it = items[i];
            Op &op = *it.op;
            VecSet &v = *it.v;
            const PcgState &hs = bt.h_state[i];
            it.updates++;
            it.iters = hs.iter;
            it.res = std::sqrt(bt.h_scalars[i]) / it.nb;
            bool stop = true;
            if (it.res < it.tol) {
                it.status = ICC_OK;
            } else if (!std::isfinite(it.res) || hs.status == kStatNan) {
                it.status = set_error(ICC_NAN, "mixed solve: non-finite residual (FP64 " + std::to_string(it.res) +
                                                   ", FP32 " + std::to_string(hs.rel_res) + ", p'Ap " +
                                                   std::to_string(hs.p_ap) + ", iteration " + std::to_string(hs.iter) +
                                                   ", update " + std::to_string(it.updates) + ")");
            } else if (hs.status == kStatBreakdown) {
                it.status = ICC_BREAKDOWN;
            } else if (hs.status == kStatMaxIter || hs.iter >= it.max_iter || it.updates >= max_updates) {
                it.status = ICC_NOT_CONVERGED;
            } else {
                if (it.res < 0.9 * it.best) {
                    it.best = it.res;
                    it.no_progress = 0;
                    stop = false;
                } else {
                    stop = ++it.no_progress >= max_no_progress;   // no longer reduces the true residual
                }
                it.status = ICC_NOT_CONVERGED;
            }
            if (stop) {
                it.done = true;   // its state keeps a non-zero status, so the kernels skip it
                active--;
                continue;
            }
            ru_replace_kernel<<<op.vec_blocks, kVecThreads, 0, s>>>(op.ndof, v.r64, 1.0 / it.nb, v.inv32, v.r32,
                                                                    op.d_partials);
            ru_replace_finalize<<<1, kVecThreads, 0, s>>>(op.d_partials, op.vec_blocks, bt.d_state + i);
            ru_arm_kernel<<<1, 1, 0, s>>>(bt.d_state + i, it.res, delta, kMaxSegment, check_every);
            // the direction update of this iteration, with the replaced residual
            pcg_p_kernel<float><<<op.vec_blocks, kVecThreads, 0, s>>>(op.ndof, v.r32, v.inv32, v.p32, bt.d_state + i,
                                                                      op.mask_mode == ICC_MASK_ZERO ? op.d_mask : nullptr);
            enqueue_pad_input(op, v, v.p32, s);
            launches += 5;
        }
        ICC_CUDA(cudaGetLastError(), "replacement");
    }
    for (size_t i = 0; i < m; ++i) {
        MixedItem &it = items[i];
        it.rel_res = it.res;
        ICC_CUDA(cudaMemcpyAsync(it.x_out, it.v->x64, (size_t)it.op->ndof * 8, cudaMemcpyDeviceToDevice, s), "copy x");
    }
    ICC_CUDA(cudaMemcpyAsync(bt.h_state, bt.d_state, m * sizeof(PcgState), cudaMemcpyDeviceToHost, s), "state");
    ICC_CUDA(cudaStreamSynchronize(s), "mixed final");
    for (size_t i = 0; i < m; ++i) items[i].iters = bt.h_state[i].iter;
    if (launches_out) *launches_out = launches;
    return ICC_OK;
}

// Captures the iteration graph of a batch: check_every x (persistent apply, fused vector step).
static int capture_graph(MixedBatch &bt, int check_every) {
    if (bt.graph) cudaGraphExecDestroy(bt.graph);
    bt.graph = nullptr;
    cudaGraph_t graph;
    ICC_CUDA(cudaStreamBeginCapture(bt.stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t ce = cudaSuccess;
    for (int i = 0; i < check_every && ce == cudaSuccess; ++i) {
        ce = launch_apply_tc(bt.stream, bt.d_inst, bt.ninst, bt.nbricks, bt.d_desc, bt.bmat, bt.d_err, bt.num_sms);
        if (ce == cudaSuccess)
            ce = launch_tail(bt.stream, bt.d_inst, bt.ninst, bt.tail_grid, bt.d_ctr, bt.d_err, bt.limit);
    }
    cudaError_t ee = cudaStreamEndCapture(bt.stream, &graph);
    ICC_CUDA(ce, "capture fused vector step");
    ICC_CUDA(ee, "end capture");
    cudaError_t e = cudaGraphInstantiate(&bt.graph, graph, 0);
    cudaGraphDestroy(graph);
    ICC_CUDA(e, "graph instantiate");
    return ICC_OK;
}

// One system: the handle's own vectors, state and cached graph.
int mixed_solve(Op &op, const double *b, const double *diag, double tol, int64_t max_iter, const icc_solve_opts &opts,
                double *x_out, int64_t *iters, double *rel_res) {
    int rc = op.ensure_pcg_buffers();
    if (rc) return rc;
    if ((rc = mixed_init(op))) return rc;
    MixedState &ms = *op.mixed;
    const int check_every = opts.check_every > 0 ? opts.check_every : 32;
    std::vector<MixedItem> items(1);
    items[0].op = &op;
    items[0].v = &ms.v;
    items[0].b = b;
    items[0].diag = diag;
    items[0].tol = tol;
    items[0].max_iter = max_iter;
    items[0].x_out = x_out;
    MixedBatch bt;
    bt.stream = op.stream;
    bt.d_inst = ms.d_inst + 1;
    bt.d_desc = ms.d_desc;
    bt.d_state = ms.d_state;
    bt.h_state = ms.h_state;
    bt.d_scalars = ms.d_scalars;
    bt.h_scalars = ms.h_scalars;
    bt.d_err = ms.d_err;
    bt.h_err = ms.h_err;
    bt.d_ctr = ms.d_grid_ctr;
    bt.ninst = 1;
    bt.nbricks = op.g.nbricks;
    bt.tail_grid = share_ctas(items, tail_capacity(op))[0];
    bt.num_sms = op.num_sms;
    bt.bmat = ms.d_bmat;
    bt.limit = ms.grid_wait_limit;
    bt.graph = ms.graph;
    if (!ms.graph || ms.graph_batch != check_every || ms.graph_limit != ms.grid_wait_limit) {
        const TcInst I = make_inst(op, ms.v, ms.d_state, 0, bt.tail_grid, 1.f);
        ICC_CUDA(cudaMemcpyAsync(bt.d_inst, &I, sizeof(TcInst), cudaMemcpyHostToDevice, op.stream), "instance table");
        bt.graph = ms.graph;
        if ((rc = capture_graph(bt, check_every))) return rc;
        ms.graph = bt.graph;
        ms.graph_batch = check_every;
        ms.graph_limit = ms.grid_wait_limit;
    }
    int64_t launches = 0;
    rc = run_mixed(bt, items, opts, &launches);
    bt.graph = nullptr;   // stays with the handle
    if (rc) return rc;
    *iters = items[0].iters;
    *rel_res = items[0].rel_res;
    op.last_info.iterations = items[0].iters;
    op.last_info.outer_iterations = items[0].updates;
    op.last_info.rel_res = items[0].rel_res;
    op.last_info.fp64_applies = items[0].updates;
    op.last_info.mixed_applies = items[0].iters;
    op.last_info.kernel_launches = launches;
    return items[0].status;
}

// ---- autotuner of the batched solve -------------------------------------------------------------
// The batch's free choices are how many CTAs of the fused vector step run per SM (its grid barrier
// needs them all resident: 1, 2 or 4) and how they are shared among the systems (in proportion to
// their control points, or in equal parts).  Each candidate is timed on the batch itself: the
// systems are initialised with residual replacement off and no tolerance, a graph of kTuneIters
// iterations runs once to warm up and once under CUDA events, and the fastest per iteration wins.
// Choices are kept per batch shape (the systems' grid sizes and mask modes, and the SM count) for
// the process, and in the JSON file named by the environment variable ICC_TUNE_CACHE when it is
// set, so other processes reuse them.
struct TuneChoice {
    int per_sm = 4, share = 0;
    double us_per_iter = 0.0;
};
constexpr int kTuneIters = 16;
static std::mutex g_tune_mu;
static std::map<std::string, TuneChoice> g_tune;
static bool g_tune_loaded = false;

static std::string tune_key(const std::vector<MixedItem> &items, int sms) {
    std::string k = "sms" + std::to_string(sms);
    for (const auto &it : items)
        k += ";" + std::to_string(it.op->g.nx) + "x" + std::to_string(it.op->g.ny) + "x" + std::to_string(it.op->g.nz) +
             "m" + std::to_string(it.op->mask_mode);
    return k;
}

// The cache file: one JSON object {"key": [per_sm, share, us_per_iter], ...}, one entry a line.
static void tune_load() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char *path = std::getenv("ICC_TUNE_CACHE");
    if (!path) return;
    std::FILE *f = std::fopen(path, "r");
    if (!f) return;
    char line[65536];
    while (std::fgets(line, sizeof line, f)) {
        char *q0 = std::strchr(line, '"');
        char *q1 = q0 ? std::strchr(q0 + 1, '"') : nullptr;
        char *br = q1 ? std::strchr(q1, '[') : nullptr;
        if (!br) continue;
        TuneChoice c;
        if (std::sscanf(br + 1, "%d , %d , %lf", &c.per_sm, &c.share, &c.us_per_iter) == 3)
            g_tune[std::string(q0 + 1, q1)] = c;
    }
    std::fclose(f);
}

static void tune_save() {
    const char *path = std::getenv("ICC_TUNE_CACHE");
    if (!path) return;
    std::FILE *f = std::fopen(path, "w");
    if (!f) return;
    std::fprintf(f, "{\n");
    size_t k = 0;
    for (const auto &kv : g_tune)
        std::fprintf(f, "  \"%s\": [%d, %d, %.3f]%s\n", kv.first.c_str(), kv.second.per_sm, kv.second.share,
                     kv.second.us_per_iter, ++k < g_tune.size() ? "," : "");
    std::fprintf(f, "}\n");
    std::fclose(f);
}

static int upload_table(MixedBatch &bt, std::vector<MixedItem> &items, const std::vector<int> &ncta) {
    std::vector<TcInst> tab(items.size());
    int cta = 0;
    for (size_t i = 0; i < items.size(); ++i) {
        if (items[i].v->part_cap < ncta[i]) return set_error(ICC_BAD_ARG, "batched mixed solve: partial buffer too small");
        tab[i] = make_inst(*items[i].op, *items[i].v, bt.d_state + i, cta, ncta[i], items[i].kfac);
        cta += ncta[i];
    }
    bt.tail_grid = cta;
    ICC_CUDA(cudaMemcpyAsync(bt.d_inst, tab.data(), tab.size() * sizeof(TcInst), cudaMemcpyHostToDevice, bt.stream),
             "instance table");
    return ICC_OK;
}

static int autotune(MixedBatch &bt, std::vector<MixedItem> &items, int max_per_sm, TuneChoice &best) {
    cudaEvent_t e0, e1;
    ICC_CUDA(cudaEventCreate(&e0), "event");
    ICC_CUDA(cudaEventCreate(&e1), "event");
    best.us_per_iter = INFINITY;
    int rc = ICC_OK;
    for (int per_sm : {1, 2, 4}) {
        if (per_sm > max_per_sm || rc) continue;
        for (int share = 0; share < 2 && !rc; ++share) {
            const std::vector<int> ncta = share_ctas(items, per_sm * bt.num_sms, share);
            int64_t l = 0;
            if ((rc = upload_table(bt, items, ncta)) || (rc = capture_graph(bt, kTuneIters)) ||
                (rc = init_items(bt, items, 0.0, kTuneIters, true, l)))
                break;
            cudaGraphLaunch(bt.graph, bt.stream);
            cudaEventRecord(e0, bt.stream);
            cudaGraphLaunch(bt.graph, bt.stream);
            cudaEventRecord(e1, bt.stream);
            cudaError_t e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) {
                rc = cuda_fail(e, "autotune");
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double us = 1e3 * ms / kTuneIters;
            if (us < best.us_per_iter) {
                best.us_per_iter = us;
                best.per_sm = per_sm;
                best.share = share;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

// Several systems at once: systems m of the call are (ops[m], vsets[m]) with right-hand side b[m]
// (device), Jacobi diagonal diag[m] (device, null: the operator's own), tolerance tol[m] and
// budget max_iter[m]; solutions into x[m] (device).  All operators must be on one device and have
// element matrices of one shape (their uniform element matrices proportional).  The iterations of
// all systems run in one persistent apply and one fused vector step per iteration, captured in
// one CUDA graph; status[m], iters[m], rel_res[m], replacements[m] per system.  stream: where the
// batch runs (every handle's own work is finished first).
int mixed_solve_batch(cudaStream_t stream, const std::vector<Op *> &ops, const std::vector<VecSet *> &vsets,
                      const double *const *b, const double *const *diag, const double *tol, const int64_t *max_iter,
                      const icc_solve_opts &opts, double *const *x, int *status, int64_t *iters, double *rel_res,
                      int64_t *replacements) {
    const size_t m = ops.size();
    if (m == 0) return ICC_OK;
    int rc;
    for (Op *op : ops) {
        if ((rc = op->ensure_pcg_buffers())) return rc;
        if ((rc = mixed_init(*op))) return rc;
        ICC_CUDA(cudaStreamSynchronize(op->stream), "batch: drain handle");
    }
    // every system's K_u must be the first one's times a factor (elements of one shape)
    const std::vector<double> &K0 = ops[0]->mixed->kunif;
    double k0max = 0.0;
    for (double v : K0) k0max = std::fmax(k0max, std::fabs(v));
    std::vector<float> kfac(m, 1.f);
    for (size_t i = 0; i < m; ++i) {
        const std::vector<double> &Ki = ops[i]->mixed->kunif;
        double num = 0.0, den = 0.0;
        for (size_t k = 0; k < Ki.size(); ++k) {
            num += Ki[k] * K0[k];
            den += K0[k] * K0[k];
        }
        const double f = num / den;
        double dev = 0.0;
        for (size_t k = 0; k < Ki.size(); ++k) dev = std::fmax(dev, std::fabs(Ki[k] - f * K0[k]));
        if (!(dev <= 1e-9 * std::fabs(f) * k0max))
            return set_error(ICC_BAD_ARG, "batched mixed solve: the systems' elements differ in shape (system " +
                                              std::to_string(i) + ")");
        kfac[i] = float(f);
    }
    std::vector<MixedItem> items(m);
    int nbricks = 0;
    std::vector<BrickDesc> descs;
    for (size_t i = 0; i < m; ++i) {
        items[i].op = ops[i];
        items[i].v = vsets[i];
        items[i].b = b[i];
        items[i].diag = diag ? diag[i] : nullptr;
        items[i].tol = tol[i];
        items[i].max_iter = max_iter[i];
        items[i].x_out = x[i];
        items[i].kfac = kfac[i];
        append_descs(*ops[i], (int)i, descs);
        nbricks += ops[i]->g.nbricks;
    }
    if ((nbricks + ops[0]->num_sms - 1) / ops[0]->num_sms > kMaxListPerCta)
        return set_error(ICC_BAD_ARG, "batched mixed solve: more than 2048 bricks per SM");
    const int cap = tail_capacity(*ops[0]);
    if ((int)m > cap || (int)m > kMaxInst)
        return set_error(ICC_BAD_ARG, "batched mixed solve: more systems than resident CTAs of the vector step");
    MixedBatch bt;
    bt.owned = true;
    bt.stream = stream;
    bt.ninst = (int)m;
    bt.nbricks = nbricks;
    bt.num_sms = ops[0]->num_sms;
    bt.bmat = ops[0]->mixed->d_bmat;
    bt.limit = ops[0]->mixed->grid_wait_limit;
    if ((rc = dalloc(&bt.d_inst, m, "alloc batch")) || (rc = dalloc(&bt.d_desc, descs.size(), "alloc batch")) ||
        (rc = dalloc(&bt.d_state, m, "alloc batch")) ||
        (rc = dalloc(&bt.d_scalars, m, "alloc batch")) || (rc = dalloc(&bt.d_err, 1, "alloc batch")) ||
        (rc = dalloc(&bt.d_ctr, 1, "alloc batch")))
        return rc;
    ICC_CUDA(cudaMallocHost((void **)&bt.h_state, m * sizeof(PcgState)), "alloc pinned");
    ICC_CUDA(cudaMallocHost((void **)&bt.h_scalars, m * sizeof(double)), "alloc pinned");
    ICC_CUDA(cudaMallocHost((void **)&bt.h_err, sizeof(int)), "alloc pinned");
    ICC_CUDA(cudaMemcpyAsync(bt.d_desc, descs.data(), descs.size() * sizeof(BrickDesc), cudaMemcpyHostToDevice, stream),
             "brick list");
    // the vector step's CTAs: tuned once per batch shape (a single system takes them all)
    TuneChoice ch;
    ch.per_sm = ops[0]->mixed->tail_per_sm;
    if (m > 1) {
        const std::string key = tune_key(items, bt.num_sms);
        bool have = false;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            tune_load();
            auto it = g_tune.find(key);
            if (it != g_tune.end() && it->second.per_sm <= ops[0]->mixed->tail_per_sm) {
                ch = it->second;
                have = true;
            }
        }
        if (!have) {
            if ((rc = autotune(bt, items, ops[0]->mixed->tail_per_sm, ch))) return rc;
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune[key] = ch;
            tune_save();
        }
    }
    if ((rc = upload_table(bt, items, share_ctas(items, ch.per_sm * bt.num_sms, ch.share)))) return rc;
    const int check_every = opts.check_every > 0 ? opts.check_every : 32;
    if ((rc = capture_graph(bt, check_every))) return rc;
    rc = run_mixed(bt, items, opts, nullptr);
    if (rc) return rc;
    for (size_t i = 0; i < m; ++i) {
        if (status) status[i] = items[i].status;
        if (iters) iters[i] = items[i].iters;
        if (rel_res) rel_res[i] = items[i].rel_res;
        if (replacements) replacements[i] = items[i].updates;
    }
    return ICC_OK;
}

// Extra vector sets for systems that share a handle's operator (load cases).
VecSet *mixed_vecset_create(Op &op) {
    if (mixed_init(op)) return nullptr;
    VecSet *v = new VecSet();
    if (vecset_alloc(op, *v, tail_capacity(op))) {
        vecset_free(*v);
        delete v;
        return nullptr;
    }
    return v;
}

void mixed_vecset_destroy(VecSet *v) {
    if (!v) return;
    vecset_free(*v);
    delete v;
}

VecSet *mixed_own_vecset(Op &op) {
    if (mixed_init(op)) return nullptr;
    return &op.mixed->v;
}

}  // namespace icc
