// Mixed-precision form of the solve: FP64 iterative refinement (defect correction) around an
// inner FP32 Jacobi-PCG whose operator runs on the 5th-generation tensor cores.
//
// Tensor-core brick apply (one CTA per 8x4x4-element brick, 128 threads, thread m = element m =
// row m of the MMA tile and TMEM lane m):
//   A = U^T [128 elements x 88], the brick's gathered element vectors (81 padded to 88);
//   B = K_type [96 x 88] row-major (test DOF n, trial DOF k; 81 padded to 96 x 88);
//   D[128 x 96] (TMEM, FP32) = A_lo B_hi + A_hi B_lo + A_hi B_hi, a 3-term split-TF32 product
//   (v = hi + lo with hi = tf32(v), lo = tf32(v - hi)), 33 tcgen05.mma kind::tf32 of M=128, N=96, K=8.
// Bricks that hold several element types run one MMA pass per type; every row keeps the pass of
// its own type.  Rows are scaled by s_e, staged in shared memory and summed per patch node in a
// fixed order, exactly as the FP64 apply, and the node-side pass resolves the brick overlaps.
//
// Outer loop (FP64): r = b - A x with the FP64 apply, d = inner_PCG(A, r / |r|), x += |r| d.
// FP64 is kept for the outer residual, the solution update and every reduction; the inner
// vectors are FP32 with FP64 dot products.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
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

constexpr int kTcM = kEPB;        // 128 rows = the brick's elements
constexpr int kTcN = 96;          // test DOFs 81 -> 96
constexpr int kTcK = 88;          // trial DOFs 81 -> 88 = 11 MMAs of K = 8
constexpr int kTcKSteps = kTcK / 8;
constexpr int kAFl = kTcM * kTcK;  // floats per A term
constexpr int kBFl = kTcN * kTcK;  // floats per B term
constexpr uint32_t kALbo = (kTcM / 8) * 128;  // bytes between K-adjacent core matrices of A
constexpr uint32_t kBLbo = (kTcN / 8) * 128;
constexpr uint32_t kSbo = 128;                // bytes between 8-row groups
constexpr int kTcThreads = 128;
constexpr int kTcSmemUsed = (2 * kAFl + 2 * kBFl + 3 * kPVol) * 4;
// allocation rounded up to 176 KB: the operand descriptors can never address past the CTA's
// shared memory, even if an 8-row-group stride and a K-chunk stride were interchanged
constexpr int kTcSmem = 176 * 1024;
static_assert(kTcSmemUsed <= kTcSmem, "shared memory budget");
constexpr uint32_t kTmemCols = 256;  // D uses 96; one CTA per SM
constexpr long long kWaitLimit = 1LL << 22;

// offset (floats) of element (row, k) in the canonical K-major no-swizzle layout with `rows` rows
__host__ __device__ __forceinline__ int canon(int row, int k, int rows) {
    return (k >> 2) * (rows / 8) * 32 + (row >> 3) * 32 + (row & 7) * 4 + (k & 3);
}

struct MixedState {
    bool ready = false;
    float4 *d_bmat = nullptr;        // [ntypes][2 terms][kBFl] canonical layout, hi then lo
    float *d_scale32 = nullptr;
    int *d_pass_start = nullptr, *d_pass_type = nullptr;
    float *d_patch32 = nullptr;
    float *d_rhs32 = nullptr, *d_x32 = nullptr, *d_r32 = nullptr, *d_p32 = nullptr, *d_ap32 = nullptr,
          *d_inv32 = nullptr;
    double *d_x64 = nullptr, *d_r64 = nullptr, *d_y64 = nullptr, *d_scalars = nullptr;
    int *d_err = nullptr;
    PcgState *d_state = nullptr, *h_state = nullptr;
    double *h_scalars = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_batch = 0;
};

// ------------------------------------------------------------------------------------------
// Kernels
// ------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(kTcThreads, 1)
apply_tc_kernel(Geom g, const float *__restrict__ x, const uint8_t *__restrict__ mask, int mask_in,
                const float *__restrict__ scale, const int *__restrict__ type_id, const float4 *__restrict__ bmat,
                const int *__restrict__ pass_start, const int *__restrict__ pass_type, float *__restrict__ patch_out,
                int *__restrict__ err, const PcgState *__restrict__ st) {
    if (st && st->status != 0) return;
    extern __shared__ __align__(1024) float tsm[];
    float *sA = tsm;                 // [2][kAFl]  A_hi, A_lo; reused as Y[128][81] after the MMAs
    float *sB = tsm + 2 * kAFl;      // [2][kBFl]  B_hi, B_lo
    float *sP = sB + 2 * kBFl;       // [3][kPVol] input patch
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int b = blockIdx.x;
    const int bxi = b % g.nbx, byi = (b / g.nbx) % g.nby, bzi = b / (g.nbx * g.nby);
    const int x0 = bxi * kBX, y0 = byi * kBY, z0 = bzi * kBZ;
    const int ex_n = min(kBX, g.nx - x0), ey_n = min(kBY, g.ny - y0), ez_n = min(kBZ, g.nz - z0);

    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, kTmemCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&mbar, 1);
        tc::fence_mbar_init();
    }
    for (int i = tid; i < 3 * kPVol; i += kTcThreads) {
        int c = i / kPVol, r = i - c * kPVol;
        int px = r % kPX, py = (r / kPX) % kPY, pz = r / (kPX * kPY);
        int gx = x0 + px, gy = y0 + py, gz = z0 + pz;
        float v = 0.f;
        if (gx < g.cx && gy < g.cy && gz < g.cz) {
            long long idx = (long long)c * g.nsc + ((long long)gz * g.cy + gy) * g.cx + gx;
            v = x[idx];
            if (mask_in && !mask[idx]) v = 0.f;
        }
        sP[i] = v;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;

    // this thread's element (row m of the tile)
    const int m = tid;
    const int lx = m % kBX, ly = (m / kBX) % kBY, lz = m / (kBX * kBY);
    const bool valid = lx < ex_n && ly < ey_n && lz < ez_n;
    int my_type = -1;
    float s = 0.f;
    if (valid) {
        long long eg = (long long)(x0 + lx) + (long long)g.nx * ((y0 + ly) + (long long)g.ny * (z0 + lz));
        my_type = type_id[eg];
        s = scale[eg];
    }
    const int base = (lz * kPY + ly) * kPX + lx;
    // A rows: split each value into hi + lo TF32 parts, 16-byte stores along K
#pragma unroll 1
    for (int ch = 0; ch < kTcK / 4; ++ch) {
        float hi[4], lo[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int k = ch * 4 + q;
            float v = 0.f;
            if (valid && k < 81) {
                int c = k / 27, a = k % 27;
                v = sP[c * kPVol + base + (a / 9) * (kPY * kPX) + ((a / 3) % 3) * kPX + a % 3];
            }
            hi[q] = tc::to_tf32(v);
            lo[q] = tc::to_tf32(v - hi[q]);
        }
        int off = canon(m, ch * 4, kTcM);
        *reinterpret_cast<float4 *>(sA + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<float4 *>(sA + kAFl + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
    }
    tc::fence_proxy_async();

    float res[81];
#pragma unroll
    for (int n = 0; n < 81; ++n) res[n] = 0.f;
    constexpr uint32_t idesc = tc::idesc_tf32(kTcM, kTcN);
    const int p0 = pass_start[b], p1 = pass_start[b + 1];
    bool timed_out = false;
    for (int pi = p0; pi < p1; ++pi) {
        const int t = pass_type[pi];
        const float4 *src = bmat + (size_t)t * (2 * kBFl / 4);
        float4 *dst = reinterpret_cast<float4 *>(sB);
        for (int i = tid; i < 2 * kBFl / 4; i += kTcThreads) dst[i] = src[i];
        tc::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll 1
            for (int ks = 0; ks < kTcKSteps; ++ks) {
                const float *a_hi = sA + ks * 2 * (kTcM / 8) * 32;
                const float *b_hi = sB + ks * 2 * (kTcN / 8) * 32;
                uint64_t ah = tc::make_desc(a_hi, kALbo, kSbo), al = tc::make_desc(a_hi + kAFl, kALbo, kSbo);
                uint64_t bh = tc::make_desc(b_hi, kBLbo, kSbo), bl = tc::make_desc(b_hi + kBFl, kBLbo, kSbo);
                tc::mma_tf32(tmem, al, bh, idesc, ks > 0 ? 1u : 0u);
                tc::mma_tf32(tmem, ah, bl, idesc, 1u);
                tc::mma_tf32(tmem, ah, bh, idesc, 1u);
            }
            tc::mma_commit(&mbar);
        }
        const bool ok = tc::mbar_wait_bounded(&mbar, uint32_t(pi - p0) & 1u, kWaitLimit);
        timed_out = __syncthreads_or(!ok) != 0;  // CTA-uniform decision
        if (timed_out) {
            if (tid == 0) atomicExch(err, 1);
            tc::mbar_wait_bounded(&mbar, uint32_t(pi - p0) & 1u, kWaitLimit);  // let issued MMAs drain
        }
        tc::fence_after_sync();
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
        for (int cc = 0; cc < kTcN / 16; ++cc) {
            uint32_t r[16];
            tc::tmem_ld16(taddr + cc * 16, r);
            tc::tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int n = cc * 16 + j;
                if (n < 81 && my_type == t) res[n] = s * __uint_as_float(r[j]);
            }
        }
        tc::fence_before_sync();
        __syncthreads();
        if (timed_out) break;
    }

    // stage the scaled element results (A is no longer read by the tensor core)
    float *sY = sA;
    if (valid) {
#pragma unroll
        for (int n = 0; n < 81; ++n) sY[m * 81 + n] = res[n];
    }
    __syncthreads();
    float *outb = patch_out + (size_t)b * 3 * kPVol;
    for (int i = tid; i < 3 * kPVol; i += kTcThreads) {
        int c = i / kPVol, r = i - c * kPVol;
        int px = r % kPX, py = (r / kPX) % kPY, pz = r / (kPX * kPY);
        float sum = 0.f;
        if (px < ex_n + 2 && py < ey_n + 2 && pz < ez_n + 2) {
            for (int qz = max(pz - 2, 0); qz <= min(pz, ez_n - 1); ++qz)
                for (int qy = max(py - 2, 0); qy <= min(py, ey_n - 1); ++qy)
                    for (int qx = max(px - 2, 0); qx <= min(px, ex_n - 1); ++qx) {
                        int e = qx + kBX * (qy + kBY * qz);
                        sum += sY[e * 81 + c * 27 + (px - qx) + 3 * (py - qy) + 9 * (pz - qz)];
                    }
        }
        outb[i] = sum;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kTmemCols);
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

// r32 = r / |r| (FP32), |r|^2 in scalars[0]
__global__ void ir_to_f32_kernel(long long n, const double *__restrict__ r, float *__restrict__ r32,
                                 const double *__restrict__ scalars) {
    const double inv = 1.0 / sqrt(scalars[0]);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        r32[i] = float(r[i] * inv);
}

// x += |r| d
__global__ void ir_update_kernel(long long n, double *__restrict__ x, const float *__restrict__ d,
                                 const double *__restrict__ scalars) {
    const double nr = sqrt(scalars[0]);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] += nr * double(d[i]);
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

static int mixed_init(Op &op) {
    if (op.mixed && op.mixed->ready) return ICC_OK;
    if (!op.mixed) op.mixed = new MixedState();
    MixedState &ms = *op.mixed;
    const int nt = op.ntypes;
    // element matrices split into TF32 hi/lo in the canonical layout
    std::vector<float> bm((size_t)nt * 2 * kBFl, 0.f);
    for (int t = 0; t < nt; ++t) {
        const double *K = op.host_ktypes.data() + (size_t)t * 81 * 81;
        float *hi = bm.data() + (size_t)t * 2 * kBFl, *lo = hi + kBFl;
        for (int n = 0; n < 81; ++n)
            for (int k = 0; k < 81; ++k) {
                double v = K[n * 81 + k];
                float h = host_tf32(float(v));
                float l = host_tf32(float(v - double(h)));
                hi[canon(n, k, kTcN)] = h;
                lo[canon(n, k, kTcN)] = l;
            }
    }
    int rc;
    if ((rc = dalloc(&ms.d_bmat, bm.size() / 4, "alloc tc matrices"))) return rc;
    ICC_CUDA(cudaMemcpy(ms.d_bmat, bm.data(), bm.size() * 4, cudaMemcpyHostToDevice), "copy tc matrices");
    // per brick: distinct element types in first-appearance order (one MMA pass each)
    std::vector<int> pstart(1, 0), ptype;
    const Geom &g = op.g;
    for (int b = 0; b < g.nbricks; ++b) {
        int bxi = b % g.nbx, byi = (b / g.nbx) % g.nby, bzi = b / (g.nbx * g.nby);
        std::vector<int> seen;
        for (int lz = 0; lz < kBZ && bzi * kBZ + lz < g.nz; ++lz)
            for (int ly = 0; ly < kBY && byi * kBY + ly < g.ny; ++ly)
                for (int lx = 0; lx < kBX && bxi * kBX + lx < g.nx; ++lx) {
                    int64_t e = (bxi * kBX + lx) + (int64_t)g.nx * ((byi * kBY + ly) + (int64_t)g.ny * (bzi * kBZ + lz));
                    int t = op.host_type_id[(size_t)e];
                    bool found = false;
                    for (int v : seen) found |= v == t;
                    if (!found) seen.push_back(t);
                }
        for (int t : seen) ptype.push_back(t);
        pstart.push_back(int(ptype.size()));
    }
    if ((rc = dalloc(&ms.d_pass_start, pstart.size(), "alloc passes"))) return rc;
    if ((rc = dalloc(&ms.d_pass_type, ptype.size(), "alloc passes"))) return rc;
    ICC_CUDA(cudaMemcpy(ms.d_pass_start, pstart.data(), pstart.size() * 4, cudaMemcpyHostToDevice), "copy passes");
    ICC_CUDA(cudaMemcpy(ms.d_pass_type, ptype.data(), ptype.size() * 4, cudaMemcpyHostToDevice), "copy passes");
    const size_t n = (size_t)op.ndof;
    if ((rc = dalloc(&ms.d_scale32, (size_t)op.nel, "alloc mixed"))) return rc;
    if ((rc = dalloc(&ms.d_patch32, (size_t)g.nbricks * 3 * kPVol, "alloc mixed"))) return rc;
    float **f32[] = {&ms.d_rhs32, &ms.d_x32, &ms.d_r32, &ms.d_p32, &ms.d_ap32, &ms.d_inv32};
    for (float **p : f32)
        if ((rc = dalloc(p, n, "alloc mixed"))) return rc;
    double **f64[] = {&ms.d_x64, &ms.d_r64, &ms.d_y64};
    for (double **p : f64)
        if ((rc = dalloc(p, n, "alloc mixed"))) return rc;
    if ((rc = dalloc(&ms.d_scalars, 8, "alloc mixed"))) return rc;
    if ((rc = dalloc(&ms.d_err, 1, "alloc mixed"))) return rc;
    if ((rc = dalloc(&ms.d_state, 1, "alloc mixed"))) return rc;
    ICC_CUDA(cudaMallocHost((void **)&ms.h_state, sizeof(PcgState)), "alloc pinned");
    ICC_CUDA(cudaMallocHost((void **)&ms.h_scalars, 8 * sizeof(double)), "alloc pinned");
    ICC_CUDA(cudaMemset(ms.d_err, 0, sizeof(int)), "clear err");
    ICC_CUDA(cudaFuncSetAttribute(apply_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem),
             "cudaFuncSetAttribute tc");
    ms.ready = true;
    return mixed_on_scale_update(op);
}

void mixed_release(Op &op) {
    if (!op.mixed) return;
    MixedState &ms = *op.mixed;
    if (ms.graph) cudaGraphExecDestroy(ms.graph);
    void *bufs[] = {ms.d_bmat, ms.d_scale32, ms.d_pass_start, ms.d_pass_type, ms.d_patch32, ms.d_rhs32, ms.d_x32,
                    ms.d_r32, ms.d_p32, ms.d_ap32, ms.d_inv32, ms.d_x64, ms.d_r64, ms.d_y64, ms.d_scalars,
                    ms.d_err, ms.d_state};
    for (void *p : bufs)
        if (p) cudaFree(p);
    if (ms.h_state) cudaFreeHost(ms.h_state);
    if (ms.h_scalars) cudaFreeHost(ms.h_scalars);
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

// enqueue y32 = A p32 with the tensor-core apply (partials: p'Ap per CTA)
static void enqueue_apply_tc(Op &op, const float *x, float *y, double *partials, const PcgState *st) {
    MixedState &ms = *op.mixed;
    apply_tc_kernel<<<op.g.nbricks, kTcThreads, kTcSmem, op.stream>>>(
        op.g, x, op.d_mask, op.mask_mode != ICC_MASK_NONE, ms.d_scale32, op.d_type_id, ms.d_bmat, ms.d_pass_start,
        ms.d_pass_type, ms.d_patch32, ms.d_err, st);
    gather_kernel<float><<<op.vec_blocks, kVecThreads, 0, op.stream>>>(op.g, ms.d_patch32, x, op.d_mask, op.mask_mode,
                                                                       y, partials, st);
}

static void enqueue_inner_iteration(Op &op) {
    MixedState &ms = *op.mixed;
    const int vb = op.vec_blocks;
    enqueue_apply_tc(op, ms.d_p32, ms.d_ap32, op.d_partials, ms.d_state);
    pcg_alpha_kernel<<<1, kVecThreads, 0, op.stream>>>(op.d_partials, vb, ms.d_state);
    pcg_update_kernel<float><<<vb, kVecThreads, 0, op.stream>>>(op.ndof, ms.d_p32, ms.d_ap32, ms.d_inv32, ms.d_x32,
                                                                ms.d_r32, op.d_partials, ms.d_state);
    pcg_beta_kernel<<<1, kVecThreads, 0, op.stream>>>(op.d_partials, vb, ms.d_state);
    pcg_p_kernel<float><<<vb, kVecThreads, 0, op.stream>>>(op.ndof, ms.d_r32, ms.d_inv32, ms.d_p32, ms.d_state);
}

// Diagnostic / test hook: y32 = A x32 on the tensor cores (used by the mixed apply test path).
int mixed_apply_f32(Op &op, const float *x, float *y) {
    int rc = mixed_init(op);
    if (rc) return rc;
    enqueue_apply_tc(op, x, y, nullptr, nullptr);
    ICC_CUDA(cudaGetLastError(), "tc apply launch");
    int err = 0;
    ICC_CUDA(cudaMemcpyAsync(&err, op.mixed->d_err, sizeof(int), cudaMemcpyDeviceToHost, op.stream), "err");
    ICC_CUDA(cudaStreamSynchronize(op.stream), "tc apply");
    if (err) return set_error(ICC_TIMEOUT, "tensor-core apply: mbarrier wait ran out");
    return ICC_OK;
}

int mixed_solve(Op &op, const double *b, const double *diag, double tol, int64_t max_iter, const icc_solve_opts &opts,
                double *x_out, int64_t *iters, double *rel_res) {
    int rc = op.ensure_pcg_buffers();
    if (rc) return rc;
    if ((rc = mixed_init(op))) return rc;
    MixedState &ms = *op.mixed;
    const int vb = op.vec_blocks;
    const long long n = op.ndof;
    const double inner_tol = opts.inner_tol > 0.0 ? opts.inner_tol : 1e-3;
    const int max_outer = opts.max_outer > 0 ? opts.max_outer : 60;
    const int check_every = opts.check_every > 0 ? opts.check_every : 32;
    int64_t launches = 0;

    if (!diag) {
        if ((rc = op.diagonal_dev(op.d_diag))) return rc;
        diag = op.d_diag;
        launches++;
    }
    inv_diag_kernel<float><<<vb, kVecThreads, 0, op.stream>>>(n, diag, ms.d_inv32);
    ir_init_kernel<<<vb, kVecThreads, 0, op.stream>>>(n, b, ms.d_x64, ms.d_r64, op.d_partials);
    sum_partials_kernel<<<1, kVecThreads, 0, op.stream>>>(op.d_partials, vb, ms.d_scalars, 0);
    launches += 3;
    ICC_CUDA(cudaMemcpyAsync(ms.h_scalars, ms.d_scalars, 8, cudaMemcpyDeviceToHost, op.stream), "scalars");
    ICC_CUDA(cudaStreamSynchronize(op.stream), "mixed init");
    const double nb = std::fmax(std::sqrt(ms.h_scalars[0]), 1e-16);
    double rr = ms.h_scalars[0];

    if (!ms.graph || ms.graph_batch != check_every) {
        if (ms.graph) cudaGraphExecDestroy(ms.graph);
        ms.graph = nullptr;
        cudaGraph_t graph;
        ICC_CUDA(cudaStreamBeginCapture(op.stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        for (int i = 0; i < check_every; ++i) enqueue_inner_iteration(op);
        ICC_CUDA(cudaStreamEndCapture(op.stream, &graph), "end capture");
        cudaError_t e = cudaGraphInstantiate(&ms.graph, graph, 0);
        cudaGraphDestroy(graph);
        ICC_CUDA(e, "graph instantiate");
        ms.graph_batch = check_every;
    }

    int64_t total_inner = 0, outer = 0, fp64_applies = 0;
    double res = std::sqrt(rr) / nb, prev_res = INFINITY;
    int status = ICC_NOT_CONVERGED;
    int stall = 0;
    for (;;) {
        res = std::sqrt(rr) / nb;
        if (res < tol) {
            status = ICC_OK;
            break;
        }
        if (!std::isfinite(res)) {
            status = set_error(ICC_NAN, "mixed solve: non-finite residual");
            break;
        }
        if (outer >= max_outer || total_inner >= max_iter) break;
        if (res > 0.5 * prev_res) {
            if (++stall >= 3) break;  // refinement no longer contracts: report NOT_CONVERGED
        } else {
            stall = 0;
        }
        prev_res = res;
        // inner FP32 PCG on A d = r / |r|
        ir_to_f32_kernel<<<vb, kVecThreads, 0, op.stream>>>(n, ms.d_r64, ms.d_rhs32, ms.d_scalars);
        pcg_init_kernel<float><<<vb, kVecThreads, 0, op.stream>>>(n, ms.d_rhs32, ms.d_inv32, ms.d_x32, ms.d_r32,
                                                                  ms.d_p32, op.d_partials);
        pcg_init_finalize<<<1, kVecThreads, 0, op.stream>>>(op.d_partials, vb, ms.d_state, inner_tol,
                                                            (long long)(max_iter - total_inner));
        launches += 3;
        for (;;) {
            ICC_CUDA(cudaMemcpyAsync(ms.h_state, ms.d_state, sizeof(PcgState), cudaMemcpyDeviceToHost, op.stream),
                     "state");
            ICC_CUDA(cudaStreamSynchronize(op.stream), "inner sync");
            if (ms.h_state->status != 0) break;
            ICC_CUDA(cudaGraphLaunch(ms.graph, op.stream), "graph launch");
            launches += 6 * int64_t(check_every);
        }
        int err = 0;
        ICC_CUDA(cudaMemcpy(&err, ms.d_err, sizeof(int), cudaMemcpyDeviceToHost), "err");
        if (err) return set_error(ICC_TIMEOUT, "tensor-core apply: mbarrier wait ran out");
        if (ms.h_state->status == kStatNan) {
            status = set_error(ICC_NAN, "mixed solve: non-finite inner reduction");
            break;
        }
        total_inner += ms.h_state->iter;
        // x += |r| d;  r = b - A x (FP64)
        ir_update_kernel<<<vb, kVecThreads, 0, op.stream>>>(n, ms.d_x64, ms.d_x32, ms.d_scalars);
        op.enqueue_apply(ms.d_x64, ms.d_y64, nullptr, nullptr);
        ir_residual_kernel<<<vb, kVecThreads, 0, op.stream>>>(n, b, ms.d_y64, ms.d_r64, op.d_partials);
        sum_partials_kernel<<<1, kVecThreads, 0, op.stream>>>(op.d_partials, vb, ms.d_scalars, 0);
        launches += 5;
        ICC_CUDA(cudaMemcpyAsync(ms.h_scalars, ms.d_scalars, 8, cudaMemcpyDeviceToHost, op.stream), "scalars");
        ICC_CUDA(cudaStreamSynchronize(op.stream), "outer sync");
        rr = ms.h_scalars[0];
        outer++;
        fp64_applies++;
    }
    ICC_CUDA(cudaMemcpyAsync(x_out, ms.d_x64, (size_t)n * 8, cudaMemcpyDeviceToDevice, op.stream), "copy x");
    *iters = total_inner;
    *rel_res = res;
    op.last_info.iterations = total_inner;
    op.last_info.outer_iterations = outer;
    op.last_info.rel_res = res;
    op.last_info.fp64_applies = fp64_applies;
    op.last_info.mixed_applies = total_inner;
    op.last_info.kernel_launches = launches;
    return status;
}

}  // namespace icc
