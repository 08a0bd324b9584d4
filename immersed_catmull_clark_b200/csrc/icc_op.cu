// Matrix-free p = 2 B-spline elasticity operator, Jacobi diagonal and device PCG for sm_100a.
//
// Work decomposition.  The element grid is cut into bricks of BX x BY x BZ = 8 x 4 x 4
// elements.  One CTA owns one brick:
//   1. it stages the brick's (BX+2)(BY+2)(BZ+2) control-point patch of the input vector, all
//      three components, into shared memory (input mask applied on the fly);
//   2. its warps contract the gathered element vectors with the element matrices on the FP64
//      tensor cores (DMMA, mma.sync m16n8k4 f64): a warp tile is 16 elements of one type,
//      Y^T[16 x 88] = U^T[16 x 84] * K_type^T[84 x 88] (81 padded to 84 / 88);
//   3. rows are scaled by s_e, staged in shared memory, and every patch node sums its <= 27
//      element contributions in a fixed order;
//   4. the brick's patch partial sums go to a scratch buffer; a node-centric pass then adds the
//      <= 8 partials of the bricks that share each node (2-plane overlaps), applies the output
//      mask and, inside PCG, also forms p'Ap.  No atomics anywhere: results are bitwise
//      reproducible run to run.
// The reference computes the same y = sum_e s_e K_e u_e through an assembled CSR matrix
// (rust/src/sparse.rs:128-175 then :60-68).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "icc_internal.h"
#include "icc_device.cuh"
#include "icc_vec.cuh"

namespace icc {

thread_local std::string g_last_error;

int set_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *where) {
    if (e == cudaErrorMemoryAllocation)
        return set_error(ICC_OUT_OF_MEMORY, std::string(where) + ": " + cudaGetErrorString(e));
    return set_error(ICC_CUDA_ERROR, std::string(where) + ": " + cudaGetErrorString(e));
}

#define ICC_CUDA(call, where)                         \
    do {                                              \
        cudaError_t _e = (call);                      \
        if (_e != cudaSuccess) return ::icc::cuda_fail(_e, where); \
    } while (0)

// ------------------------------------------------------------------------------------------
// Device kernels
// ------------------------------------------------------------------------------------------

// FP64 brick apply.  Writes the brick's patch partial sums to patch_out[brick][3][PVOL].
__global__ void __launch_bounds__(kApplyThreads, 2)
apply_f64_kernel(Geom g, const double *__restrict__ x, const uint8_t *__restrict__ mask, int mask_in,
                 const double *__restrict__ scale, const double *__restrict__ kfrag,
                 const int *__restrict__ tile_start, const int *__restrict__ tile_type,
                 const uint8_t *__restrict__ tile_elem, double *__restrict__ patch_out,
                 const PcgState *__restrict__ st) {
    if (st && st->status != 0) return;
    extern __shared__ double smem[];
    double *sx = smem;                  // [3][PVOL]
    double *sy = smem + 3 * kPVol;      // [kEPB][81]
    __shared__ int koff[84];

    const int b = blockIdx.x;
    const int bxi = b % g.nbx, byi = (b / g.nbx) % g.nby, bzi = b / (g.nbx * g.nby);
    const int x0 = bxi * kBX, y0 = byi * kBY, z0 = bzi * kBZ;
    const int ex_n = min(kBX, g.nx - x0), ey_n = min(kBY, g.ny - y0), ez_n = min(kBZ, g.nz - z0);

    if (threadIdx.x < 84) {
        int k = threadIdx.x;
        int kk = k < 81 ? k : 0;  // padded k has a zero B row; any in-range A value works
        int c = kk / 27, a = kk % 27;
        koff[k] = c * kPVol + ((a / 9) * kPY + (a / 3) % 3) * kPX + a % 3;
    }
    for (int i = threadIdx.x; i < 3 * kPVol; i += blockDim.x) {
        int c = i / kPVol, r = i - c * kPVol;
        int px = r % kPX, py = (r / kPX) % kPY, pz = r / (kPX * kPY);
        int gx = x0 + px, gy = y0 + py, gz = z0 + pz;
        double v = 0.0;
        if (gx < g.cx && gy < g.cy && gz < g.cz) {
            long long idx = (long long)c * g.nsc + ((long long)gz * g.cy + gy) * g.cx + gx;
            v = x[idx];
            if (mask_in && !mask[idx]) v = 0.0;
        }
        sx[i] = v;
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    const int t0 = tile_start[b], t1 = tile_start[b + 1];
    for (int t = t0 + warp; t < t1; t += kApplyThreads / 32) {
        const double *kf = kfrag + (size_t)tile_type[t] * kFragPerType;
        const int e0 = tile_elem[t * 16 + gid], e1 = tile_elem[t * 16 + gid + 8];
        const int base0 = e0 < kEPB ? ((e0 / (kBX * kBY)) * kPY + (e0 / kBX) % kBY) * kPX + e0 % kBX : 0;
        const int base1 = e1 < kEPB ? ((e1 / (kBX * kBY)) * kPY + (e1 / kBX) % kBY) * kPX + e1 % kBX : 0;
        double acc[kNTiles][4];
#pragma unroll
        for (int nt = 0; nt < kNTiles; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0;
#pragma unroll 3
        for (int ks = 0; ks < kKSteps; ++ks) {
            const int off = koff[ks * 4 + tig];
            const double a0 = sx[base0 + off];
            const double a1 = sx[base1 + off];
            const double *kk = kf + ks * (kNTiles * 32) + lane;
#pragma unroll
            for (int nt = 0; nt < kNTiles; ++nt) {
                const double bf = __ldg(kk + nt * 32);
                dmma_m16n8k4(acc[nt], a0, a1, bf);
            }
        }
        const int zx0 = (b % g.nbx) * kBX, zy0 = ((b / g.nbx) % g.nby) * kBY, zz0 = (b / (g.nbx * g.nby)) * kBZ;
        double s0 = 0.0, s1 = 0.0;
        if (e0 < kEPB) {
            long long eg = (long long)(zx0 + e0 % kBX) +
                           (long long)g.nx * ((zy0 + (e0 / kBX) % kBY) + (long long)g.ny * (zz0 + e0 / (kBX * kBY)));
            s0 = scale ? scale[eg] : 1.0;
        }
        if (e1 < kEPB) {
            long long eg = (long long)(zx0 + e1 % kBX) +
                           (long long)g.nx * ((zy0 + (e1 / kBX) % kBY) + (long long)g.ny * (zz0 + e1 / (kBX * kBY)));
            s1 = scale ? scale[eg] : 1.0;
        }
#pragma unroll
        for (int nt = 0; nt < kNTiles; ++nt) {
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                int n = nt * 8 + 2 * tig + j;
                if (n < 81) {
                    if (e0 < kEPB) sy[e0 * 81 + n] = s0 * acc[nt][j];
                    if (e1 < kEPB) sy[e1 * 81 + n] = s1 * acc[nt][2 + j];
                }
            }
        }
    }
    __syncthreads();

    // node-side sum over the brick's elements, fixed order (z, y, x ascending)
    double *outb = patch_out + (size_t)b * 3 * kPVol;
    for (int i = threadIdx.x; i < 3 * kPVol; i += blockDim.x) {
        int c = i / kPVol, r = i - c * kPVol;
        int px = r % kPX, py = (r / kPX) % kPY, pz = r / (kPX * kPY);
        double sum = 0.0;
        if (px < ex_n + 2 && py < ey_n + 2 && pz < ez_n + 2) {
            for (int lz = max(pz - 2, 0); lz <= min(pz, ez_n - 1); ++lz)
                for (int ly = max(py - 2, 0); ly <= min(py, ey_n - 1); ++ly)
                    for (int lx = max(px - 2, 0); lx <= min(px, ex_n - 1); ++lx) {
                        int e = lx + kBX * (ly + kBY * lz);
                        sum += sy[e * 81 + c * 27 + (px - lx) + 3 * (py - ly) + 9 * (pz - lz)];
                    }
        }
        outb[i] = sum;
    }
}

// Jacobi diagonal sum_e s_e K_type(e)[a,a]; elements visited in increasing index so the sum
// rounds exactly as the assembled CSR entry (rust/src/sparse.rs:166-172, then :70-78).  With a
// sparse term, its diagonal is added last, as the reference adds the stabilisation's diagonal to
// the stiffness diagonal (rust/src/topopt_immersed.rs:165-167).
__global__ void __launch_bounds__(kVecThreads)
diagonal_kernel(Geom g, const double *__restrict__ scale, const int *__restrict__ type_id,
                const double *__restrict__ kdiag, const double *__restrict__ extra, double *__restrict__ d) {
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < g.nsc;
         n += (long long)gridDim.x * blockDim.x) {
        int ix = int(n % g.cx), iy = int((n / g.cx) % g.cy), iz = int(n / ((long long)g.cx * g.cy));
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int ez = max(iz - 2, 0); ez <= min(iz, g.nz - 1); ++ez)
            for (int ey = max(iy - 2, 0); ey <= min(iy, g.ny - 1); ++ey)
                for (int ex = max(ix - 2, 0); ex <= min(ix, g.nx - 1); ++ex) {
                    long long e = ex + (long long)g.nx * (ey + (long long)g.ny * ez);
                    double s = scale ? scale[e] : 1.0;
                    const double *kd = kdiag + (size_t)type_id[e] * 81;
                    int a = (ix - ex) + 3 * (iy - ey) + 9 * (iz - ez);
                    s0 = __dadd_rn(s0, __dmul_rn(s, kd[a]));
                    s1 = __dadd_rn(s1, __dmul_rn(s, kd[27 + a]));
                    s2 = __dadd_rn(s2, __dmul_rn(s, kd[54 + a]));
                }
        if (extra) {
            s0 += extra[n];
            s1 += extra[g.nsc + n];
            s2 += extra[2 * g.nsc + n];
        }
        d[n] = s0;
        d[g.nsc + n] = s1;
        d[2 * g.nsc + n] = s2;
    }
}

// ---- PCG scalar steps (rust/src/solver.rs:14-76), shared by both precision forms -------------

__global__ void __launch_bounds__(kVecThreads)
pcg_init_finalize(const double *__restrict__ partials, int np, PcgState *st, double tol, long long max_iter) {
    double rz = 0.0, bb = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        rz += partials[2 * i];
        bb += partials[2 * i + 1];
    }
    rz = block_sum(rz);
    bb = block_sum(bb);
    if (threadIdx.x == 0) {
        st->rz_old = rz;
        st->norm_b = fmax(sqrt(bb), 1e-16);
        st->rel_res = 1.0;
        st->tol = tol;
        st->iter = 0;
        st->max_iter = max_iter;
        st->status = max_iter > 0 ? 0 : kStatMaxIter;
        st->alpha = st->beta = st->p_ap = 0.0;
        st->rz_prev = rz;
        st->rr_old = bb;
        st->fresh = 1;
        st->repl_res = 1.0;
        st->repl_delta = 0.0;
        st->repl_iter = 0;
        st->repl_seg = 0;
        st->repl_every = 1;
    }
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------

template <class T>
static int dev_alloc(T **p, size_t count, const char *what) {
    *p = nullptr;
    if (count == 0) count = 1;
    ICC_CUDA(cudaMalloc((void **)p, count * sizeof(T)), what);
    return ICC_OK;
}

Op::~Op() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    void *bufs[] = {d_x_in, d_y_out, d_scale, d_kfrag, d_kdiag, d_type_id, d_tile_start, d_tile_type, d_tile_elem,
                    d_mask, d_patch, d_x, d_r, d_p, d_ap, d_inv, d_b, d_diag, d_partials, d_state, d_counter,
                    d_sp_ptr, d_sp_idx, d_sp_val, d_sp_val32, d_sp_diag};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (h_state) cudaFreeHost(h_state);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
    mixed_release(*this);
    state_release(*this);
}

int Op::init(const Space &s, const double *ke_types, int nt, const int32_t *type_id, const double *scale,
             const uint8_t *free_mask, int mode) {
    if (cudaGetDevice(&device) != cudaSuccess) return set_error(ICC_NO_DEVICE, "no CUDA device");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(ICC_NO_DEVICE, "no CUDA device");
    cudaDeviceProp prop;
    ICC_CUDA(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    if (prop.major < 10) return set_error(ICC_NO_DEVICE, "device is not sm_100 class (B200 required)");
    num_sms = prop.multiProcessorCount;

    g.nx = int(s.nel_dir[0]); g.ny = int(s.nel_dir[1]); g.nz = int(s.nel_dir[2]);
    g.cx = int(s.ncp[0]); g.cy = int(s.ncp[1]); g.cz = int(s.ncp[2]);
    g.nsc = s.nsc;
    g.nbx = (g.nx + kBX - 1) / kBX; g.nby = (g.ny + kBY - 1) / kBY; g.nbz = (g.nz + kBZ - 1) / kBZ;
    g.nbricks = g.nbx * g.nby * g.nbz;
    nel = s.nel;
    ndof = s.ndof;
    ntypes = nt;

    for (int64_t e = 0; e < nel; ++e)
        if (type_id[e] < 0 || type_id[e] >= nt) return set_error(ICC_BAD_ARG, "type_id out of range");

    ICC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ICC_CUDA(cudaEventCreate(&ev0), "cudaEventCreate");
    ICC_CUDA(cudaEventCreate(&ev1), "cudaEventCreate");

    // element matrices in DMMA B-fragment order: kfrag[t][ks][nt][lane] = K[n][k] with
    // k = 4 ks + lane % 4 (trial), n = 8 nt + lane / 4 (test); zero outside 81 x 81.
    std::vector<double> kf((size_t)nt * kFragPerType, 0.0), kd((size_t)nt * 81);
    for (int t = 0; t < nt; ++t) {
        const double *K = ke_types + (size_t)t * 81 * 81;
        for (int ks = 0; ks < kKSteps; ++ks)
            for (int ntile = 0; ntile < kNTiles; ++ntile)
                for (int lane = 0; lane < 32; ++lane) {
                    int k = 4 * ks + (lane & 3), n = 8 * ntile + (lane >> 2);
                    kf[(size_t)t * kFragPerType + (ks * kNTiles + ntile) * 32 + lane] =
                        (k < 81 && n < 81) ? K[n * 81 + k] : 0.0;
                }
        for (int a = 0; a < 81; ++a) kd[(size_t)t * 81 + a] = K[a * 81 + a];
    }
    host_ktypes.assign(ke_types, ke_types + (size_t)nt * 81 * 81);
    int rc;
    if ((rc = dev_alloc(&d_kfrag, kf.size(), "alloc kfrag"))) return rc;
    if ((rc = dev_alloc(&d_kdiag, kd.size(), "alloc kdiag"))) return rc;
    ICC_CUDA(cudaMemcpyAsync(d_kfrag, kf.data(), kf.size() * 8, cudaMemcpyHostToDevice, stream), "copy kfrag");
    ICC_CUDA(cudaMemcpyAsync(d_kdiag, kd.data(), kd.size() * 8, cudaMemcpyHostToDevice, stream), "copy kdiag");
    if ((rc = dev_alloc(&d_type_id, (size_t)nel, "alloc type_id"))) return rc;
    ICC_CUDA(cudaMemcpyAsync(d_type_id, type_id, (size_t)nel * 4, cudaMemcpyHostToDevice, stream), "copy type_id");
    host_type_id.assign(type_id, type_id + nel);
    for (int d = 0; d < 3; ++d) {
        host_type1d[d] = s.type1d[d];
        host_basis1d[d] = s.basis1d[d];
    }

    // brick tile plan: per brick, its elements grouped by type (first-appearance order) and cut
    // into warp tiles of 16 (255 marks an empty row)
    std::vector<int> tstart(1, 0), ttype;
    std::vector<uint8_t> telem;
    std::vector<int> order, types_seen;
    for (int b = 0; b < g.nbricks; ++b) {
        int bxi = b % g.nbx, byi = (b / g.nbx) % g.nby, bzi = b / (g.nbx * g.nby);
        int x0 = bxi * kBX, y0 = byi * kBY, z0 = bzi * kBZ;
        types_seen.clear();
        std::vector<std::vector<int>> groups;
        for (int lz = 0; lz < kBZ && z0 + lz < g.nz; ++lz)
            for (int ly = 0; ly < kBY && y0 + ly < g.ny; ++ly)
                for (int lx = 0; lx < kBX && x0 + lx < g.nx; ++lx) {
                    int64_t e = (x0 + lx) + (int64_t)g.nx * ((y0 + ly) + (int64_t)g.ny * (z0 + lz));
                    int t = type_id[e];
                    size_t gi = std::find(types_seen.begin(), types_seen.end(), t) - types_seen.begin();
                    if (gi == types_seen.size()) {
                        types_seen.push_back(t);
                        groups.emplace_back();
                    }
                    groups[gi].push_back(lx + kBX * (ly + kBY * lz));
                }
        for (size_t gi = 0; gi < groups.size(); ++gi)
            for (size_t k = 0; k < groups[gi].size(); k += 16) {
                ttype.push_back(types_seen[gi]);
                for (size_t j = 0; j < 16; ++j)
                    telem.push_back(k + j < groups[gi].size() ? uint8_t(groups[gi][k + j]) : uint8_t(255));
            }
        tstart.push_back(int(ttype.size()));
    }
    ntiles = int(ttype.size());
    if ((rc = dev_alloc(&d_tile_start, tstart.size(), "alloc tiles"))) return rc;
    if ((rc = dev_alloc(&d_tile_type, ttype.size(), "alloc tiles"))) return rc;
    if ((rc = dev_alloc(&d_tile_elem, telem.size(), "alloc tiles"))) return rc;
    ICC_CUDA(cudaMemcpyAsync(d_tile_start, tstart.data(), tstart.size() * 4, cudaMemcpyHostToDevice, stream), "copy tiles");
    ICC_CUDA(cudaMemcpyAsync(d_tile_type, ttype.data(), ttype.size() * 4, cudaMemcpyHostToDevice, stream), "copy tiles");
    ICC_CUDA(cudaMemcpyAsync(d_tile_elem, telem.data(), telem.size(), cudaMemcpyHostToDevice, stream), "copy tiles");
    // every set-up copy is ordered on the handle's stream (a non-blocking stream is not ordered
    // after copies on the legacy default stream); the host arrays must outlive them
    ICC_CUDA(cudaStreamSynchronize(stream), "set-up copies");

    if ((rc = dev_alloc(&d_scale, (size_t)nel, "alloc scale"))) return rc;
    if ((rc = dev_alloc(&d_mask, (size_t)ndof, "alloc mask"))) return rc;
    if ((rc = dev_alloc(&d_patch, (size_t)g.nbricks * 3 * kPVol, "alloc patch scratch"))) return rc;
    if ((rc = dev_alloc(&d_x_in, (size_t)ndof, "alloc io"))) return rc;
    if ((rc = dev_alloc(&d_y_out, (size_t)ndof, "alloc io"))) return rc;
    vec_blocks = num_sms * 4;
    if ((rc = dev_alloc(&d_partials, (size_t)vec_blocks * 2, "alloc partials"))) return rc;
    if ((rc = dev_alloc(&d_state, 1, "alloc state"))) return rc;
    if ((rc = dev_alloc(&d_counter, 1, "alloc counter"))) return rc;
    ICC_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned), stream), "clear counter");
    ICC_CUDA(cudaStreamSynchronize(stream), "clear counter");
    ICC_CUDA(cudaMallocHost((void **)&h_state, sizeof(PcgState)), "alloc pinned state");
    ICC_CUDA(cudaFuncSetAttribute(apply_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kApplySmem),
             "cudaFuncSetAttribute");
    if ((rc = set_scale(scale))) return rc;
    if ((rc = set_mask(free_mask, mode))) return rc;
    return ICC_OK;
}

int Op::set_scale(const double *scale) {
    std::vector<double> ones;
    const double *src = scale;
    if (!src) {
        ones.assign((size_t)nel, 1.0);
        src = ones.data();
    }
    host_scale.assign(src, src + nel);
    ICC_CUDA(cudaMemcpyAsync(d_scale, src, (size_t)nel * 8, cudaMemcpyHostToDevice, stream), "copy scale");
    ICC_CUDA(cudaStreamSynchronize(stream), "copy scale");
    scale_version++;
    return mixed_on_scale_update(*this);
}

int Op::set_scale_dev(const double *scale_dev) {
    ICC_CUDA(cudaMemcpyAsync(d_scale, scale_dev, (size_t)nel * 8, cudaMemcpyDeviceToDevice, stream), "copy scale");
    scale_version++;
    return mixed_on_scale_update(*this);
}

int Op::set_mask(const uint8_t *free_mask, int mode) {
    if (mode < 0 || mode > 2) return set_error(ICC_BAD_ARG, "mask_mode must be 0, 1 or 2");
    const int new_mode = (mode != ICC_MASK_NONE && free_mask) ? mode : ICC_MASK_NONE;
    if (new_mode != mask_mode) {
        // the iteration graphs hold the mask mode by value: rebuild them on the next solve
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
        graph_batch = 0;
        mixed_invalidate_graph(*this);
    }
    mask_mode = new_mode;
    std::vector<uint8_t> ones;
    const uint8_t *src = free_mask;
    if (!src) {
        ones.assign((size_t)ndof, 1);
        src = ones.data();
    }
    ICC_CUDA(cudaMemcpyAsync(d_mask, src, (size_t)ndof, cudaMemcpyHostToDevice, stream), "copy mask");
    ICC_CUDA(cudaStreamSynchronize(stream), "copy mask");
    return ICC_OK;
}

// The extra sparse term from triplets (duplicates summed in input order, columns sorted per row).
// Replaces any previous term; count = 0 removes it.
int Op::set_extra(int64_t count, const int64_t *rows, const int64_t *cols, const double *vals) {
    for (int64_t k = 0; k < count; ++k)
        if (rows[k] < 0 || rows[k] >= ndof || cols[k] < 0 || cols[k] >= ndof)
            return set_error(ICC_BAD_ARG, "icc_op_set_extra_triplets: index out of range");
    if (count >= (1LL << 31) || ndof >= (1LL << 31))
        return set_error(ICC_BAD_ARG, "icc_op_set_extra_triplets: more than 2^31 entries or DOFs");
    // counting sort by row, then a stable sort by column inside each row, then merge
    std::vector<int> ptr((size_t)ndof + 1, 0);
    for (int64_t k = 0; k < count; ++k) ptr[(size_t)rows[k] + 1]++;
    for (int64_t i = 0; i < ndof; ++i) ptr[(size_t)i + 1] += ptr[(size_t)i];
    std::vector<int64_t> order((size_t)count);
    {
        std::vector<int> next(ptr.begin(), ptr.end() - 1);
        for (int64_t k = 0; k < count; ++k) order[(size_t)next[(size_t)rows[k]]++] = k;
    }
    std::vector<int> mptr((size_t)ndof + 1, 0), midx;
    std::vector<double> mval, diag((size_t)ndof, 0.0);
    midx.reserve((size_t)count);
    mval.reserve((size_t)count);
    for (int64_t i = 0; i < ndof; ++i) {
        auto b = order.begin() + ptr[(size_t)i], e = order.begin() + ptr[(size_t)i + 1];
        std::stable_sort(b, e, [&](int64_t a, int64_t c) { return cols[a] < cols[c]; });
        for (auto it = b; it != e; ++it) {
            if (it != b && cols[*it] == cols[*(it - 1)]) mval.back() += vals[*it];
            else {
                midx.push_back(int(cols[*it]));
                mval.push_back(vals[*it]);
            }
        }
        mptr[(size_t)i + 1] = int(midx.size());
        for (int k = mptr[(size_t)i]; k < mptr[(size_t)i + 1]; ++k)
            if (midx[(size_t)k] == i) diag[(size_t)i] = mval[(size_t)k];
    }
    void *old[] = {d_sp_ptr, d_sp_idx, d_sp_val, d_sp_val32, d_sp_diag};
    ICC_CUDA(cudaStreamSynchronize(stream), "extra term: drain");
    for (void *p : old)
        if (p) cudaFree(p);
    d_sp_ptr = d_sp_idx = nullptr;
    d_sp_val = d_sp_diag = nullptr;
    d_sp_val32 = nullptr;
    sp_nnz = 0;
    if (midx.empty()) return ICC_OK;
    const size_t nnz = midx.size();
    std::vector<float> v32(nnz);
    for (size_t k = 0; k < nnz; ++k) v32[k] = float(mval[k]);
    int rc;
    if ((rc = dev_alloc(&d_sp_ptr, mptr.size(), "alloc extra term")) || (rc = dev_alloc(&d_sp_idx, nnz, "alloc extra term")) ||
        (rc = dev_alloc(&d_sp_val, nnz, "alloc extra term")) || (rc = dev_alloc(&d_sp_val32, nnz, "alloc extra term")) ||
        (rc = dev_alloc(&d_sp_diag, (size_t)ndof, "alloc extra term")))
        return rc;
    ICC_CUDA(cudaMemcpyAsync(d_sp_ptr, mptr.data(), mptr.size() * 4, cudaMemcpyHostToDevice, stream), "copy extra term");
    ICC_CUDA(cudaMemcpyAsync(d_sp_idx, midx.data(), nnz * 4, cudaMemcpyHostToDevice, stream), "copy extra term");
    ICC_CUDA(cudaMemcpyAsync(d_sp_val, mval.data(), nnz * 8, cudaMemcpyHostToDevice, stream), "copy extra term");
    ICC_CUDA(cudaMemcpyAsync(d_sp_val32, v32.data(), nnz * 4, cudaMemcpyHostToDevice, stream), "copy extra term");
    ICC_CUDA(cudaMemcpyAsync(d_sp_diag, diag.data(), diag.size() * 8, cudaMemcpyHostToDevice, stream), "copy extra term");
    ICC_CUDA(cudaStreamSynchronize(stream), "copy extra term");
    sp_nnz = (int64_t)nnz;
    // graphs captured with the previous term's pointers are rebuilt on the next solve
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
    graph_batch = 0;
    mixed_invalidate_graph(*this);
    return ICC_OK;
}

// Enqueue y = A x on the op's stream (FP64).  partials != null also forms p'y per CTA.
void Op::enqueue_apply(const double *x, double *y, double *partials, const PcgState *st) {
    apply_f64_kernel<<<g.nbricks, kApplyThreads, kApplySmem, stream>>>(
        g, x, d_mask, mask_mode != ICC_MASK_NONE, d_scale, d_kfrag, d_tile_start, d_tile_type, d_tile_elem, d_patch,
        st);
    gather_kernel<double><<<vec_blocks, kVecThreads, 0, stream>>>(g, d_patch, x, d_mask, mask_mode, extra64(), y,
                                                                  partials, st);
}

void Op::enqueue_apply_on(cudaStream_t s, const double *x, double *y) {
    apply_f64_kernel<<<g.nbricks, kApplyThreads, kApplySmem, s>>>(
        g, x, d_mask, mask_mode != ICC_MASK_NONE, d_scale, d_kfrag, d_tile_start, d_tile_type, d_tile_elem, d_patch,
        nullptr);
    gather_kernel<double><<<vec_blocks, kVecThreads, 0, s>>>(g, d_patch, x, d_mask, mask_mode, extra64(), y,
                                                             nullptr, nullptr);
}

void Op::enqueue_diagonal(double *d, cudaStream_t s) {
    diagonal_kernel<<<vec_blocks, kVecThreads, 0, s>>>(g, d_scale, d_type_id, d_kdiag, sp_nnz ? d_sp_diag : nullptr, d);
}

int Op::apply_dev(const double *x, double *y) {
    enqueue_apply(x, y, nullptr, nullptr);
    ICC_CUDA(cudaGetLastError(), "apply launch");
    return ICC_OK;
}

int Op::diagonal_dev(double *d) {
    diagonal_kernel<<<vec_blocks, kVecThreads, 0, stream>>>(g, d_scale, d_type_id, d_kdiag, sp_nnz ? d_sp_diag : nullptr,
                                                            d);
    ICC_CUDA(cudaGetLastError(), "diagonal launch");
    return ICC_OK;
}

int Op::ensure_pcg_buffers() {
    if (d_x) return ICC_OK;
    int rc;
    if ((rc = dev_alloc(&d_x, (size_t)ndof, "alloc pcg"))) return rc;
    if ((rc = dev_alloc(&d_r, (size_t)ndof, "alloc pcg"))) return rc;
    if ((rc = dev_alloc(&d_p, (size_t)ndof, "alloc pcg"))) return rc;
    if ((rc = dev_alloc(&d_ap, (size_t)ndof, "alloc pcg"))) return rc;
    if ((rc = dev_alloc(&d_inv, (size_t)ndof, "alloc pcg"))) return rc;
    if ((rc = dev_alloc(&d_b, (size_t)ndof, "alloc pcg"))) return rc;
    if ((rc = dev_alloc(&d_diag, (size_t)ndof, "alloc pcg"))) return rc;
    return ICC_OK;
}

// One PCG iteration (rust/src/solver.rs:40-72) as six launches: p = z + beta p (beta = 0 on the
// first iteration, so p = z), Ap, alpha, x/r update, convergence test and the next beta.  Every
// kernel returns at once when the state says the solve has finished, so a batch may overrun
// harmlessly.
void Op::enqueue_pcg_iteration() {
    pcg_p_kernel<double><<<vec_blocks, kVecThreads, 0, stream>>>(ndof, d_r, d_inv, d_p, d_state);
    apply_f64_kernel<<<g.nbricks, kApplyThreads, kApplySmem, stream>>>(
        g, d_p, d_mask, mask_mode != ICC_MASK_NONE, d_scale, d_kfrag, d_tile_start, d_tile_type, d_tile_elem, d_patch,
        d_state);
    gather_kernel<double><<<vec_blocks, kVecThreads, 0, stream>>>(g, d_patch, d_p, d_mask, mask_mode, extra64(), d_ap,
                                                                  d_partials,
                                                                  d_state, d_state, d_counter);
    pcg_update_kernel<double><<<vec_blocks, kVecThreads, 0, stream>>>(ndof, d_p, d_ap, d_inv, d_x, d_r, d_partials,
                                                                      d_state, d_state, d_counter);
}

int Op::pcg_fp64(const double *b, const double *diag, double tol, int64_t max_iter, int check_every, double *x,
                 int64_t *iters, double *rel_res) {
    int rc;
    if ((rc = ensure_pcg_buffers())) return rc;
    int64_t launches = 3;
    if (!diag) {
        if ((rc = diagonal_dev(d_diag))) return rc;
        diag = d_diag;
        launches += 1;
    }
    inv_diag_kernel<double><<<vec_blocks, kVecThreads, 0, stream>>>(ndof, diag, d_inv);
    pcg_init_kernel<double><<<vec_blocks, kVecThreads, 0, stream>>>(ndof, b, d_inv, d_x, d_r, d_p, d_partials);
    pcg_init_finalize<<<1, kVecThreads, 0, stream>>>(d_partials, vec_blocks, d_state, tol, max_iter);
    ICC_CUDA(cudaGetLastError(), "pcg init");
    if (check_every <= 0) check_every = 32;
    if (!graph_exec || graph_batch != check_every) {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
        cudaGraph_t graph;
        ICC_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        for (int i = 0; i < check_every; ++i) enqueue_pcg_iteration();
        ICC_CUDA(cudaStreamEndCapture(stream, &graph), "end capture");
        cudaError_t e = cudaGraphInstantiate(&graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        ICC_CUDA(e, "graph instantiate");
        graph_batch = check_every;
    }
    int64_t launched = 0;
    for (;;) {
        ICC_CUDA(cudaMemcpyAsync(h_state, d_state, sizeof(PcgState), cudaMemcpyDeviceToHost, stream), "state");
        ICC_CUDA(cudaStreamSynchronize(stream), "pcg sync");
        if (h_state->status != 0) break;
        if (launched > max_iter + 2 * int64_t(check_every))
            return set_error(ICC_TIMEOUT, "pcg: device state did not reach a stop condition");
        ICC_CUDA(cudaGraphLaunch(graph_exec, stream), "graph launch");
        launched += check_every;
        launches += 4 * int64_t(check_every);
    }
    ICC_CUDA(cudaMemcpyAsync(x, d_x, (size_t)ndof * 8, cudaMemcpyDeviceToDevice, stream), "copy x");
    *iters = h_state->iter;
    *rel_res = h_state->rel_res;
    last_info.iterations = h_state->iter;
    last_info.outer_iterations = 0;
    last_info.rel_res = h_state->rel_res;
    last_info.fp64_applies = h_state->iter;
    last_info.mixed_applies = 0;
    last_info.kernel_launches = launches;
    switch (h_state->status) {
        case kStatConverged: return ICC_OK;
        case kStatBreakdown: return ICC_BREAKDOWN;
        case kStatMaxIter: return ICC_NOT_CONVERGED;
        default: return set_error(ICC_NAN, "pcg: non-finite reduction (NaN input or non-SPD operator)");
    }
}

}  // namespace icc

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------
using icc::set_error;

extern "C" {

const char *icc_last_error(void) { return icc::g_last_error.c_str(); }

int icc_op_create(const icc_space *sp, const double *ke_types, int32_t ntypes, const int32_t *type_id,
                  const double *scale, const uint8_t *free_mask, int32_t mask_mode, icc_op **out) {
    if (!sp || !ke_types || !type_id || !out || ntypes <= 0)
        return set_error(ICC_BAD_ARG, "icc_op_create: null argument or ntypes <= 0");
    *out = nullptr;
    auto *h = new (std::nothrow) icc_op();
    if (!h) return set_error(ICC_OUT_OF_MEMORY, "icc_op_create: out of host memory");
    int rc = h->op.init(sp->s, ke_types, ntypes, type_id, scale, free_mask, mask_mode);
    if (rc != ICC_OK) {
        delete h;
        return rc;
    }
    *out = h;
    return ICC_OK;
}

int icc_op_create_lame(const icc_space *sp, double lambda, double mu, const double *scale,
                       const uint8_t *free_mask, int32_t mask_mode, icc_op **out) {
    if (!sp || !out) return set_error(ICC_BAD_ARG, "icc_op_create_lame: null argument");
    std::vector<double> ke;
    std::vector<int32_t> tid;
    std::vector<std::array<int, 3>> combos;
    sp->s.element_types(lambda, mu, ke, tid, combos);
    return icc_op_create(sp, ke.data(), int32_t(combos.size()), tid.data(), scale, free_mask, mask_mode, out);
}

void icc_op_destroy(icc_op *op) {
    if (!op) return;
    cudaSetDevice(op->op.device);
    delete op;
}

int icc_op_update_scale(icc_op *op, const double *scale) {
    if (!op) return set_error(ICC_BAD_ARG, "icc_op_update_scale: null op");
    cudaSetDevice(op->op.device);
    return op->op.set_scale(scale);
}

int icc_op_set_extra_triplets(icc_op *op, int64_t count, const int64_t *rows, const int64_t *cols,
                              const double *vals) {
    if (!op || count < 0 || (count > 0 && (!rows || !cols || !vals)))
        return set_error(ICC_BAD_ARG, "icc_op_set_extra_triplets: bad argument");
    cudaSetDevice(op->op.device);
    return op->op.set_extra(count, rows, cols, vals);
}

int icc_op_update_mask(icc_op *op, const uint8_t *free_mask, int32_t mask_mode) {
    if (!op) return set_error(ICC_BAD_ARG, "icc_op_update_mask: null op");
    cudaSetDevice(op->op.device);
    return op->op.set_mask(free_mask, mask_mode);
}

void *icc_op_stream(icc_op *op) { return op ? (void *)op->op.stream : nullptr; }

int icc_op_apply_dev(icc_op *op, const double *x, double *y, int64_t n) {
    if (!op || !x || !y) return set_error(ICC_BAD_ARG, "icc_op_apply_dev: null argument");
    if (n != op->op.ndof) return set_error(ICC_BAD_ARG, "icc_op_apply_dev: n != ndof");
    cudaSetDevice(op->op.device);
    return op->op.apply_dev(x, y);
}

int icc_op_apply(icc_op *op, const double *x, double *y, int64_t n) {
    if (!op || !x || !y) return set_error(ICC_BAD_ARG, "icc_op_apply: null argument");
    icc::Op &o = op->op;
    if (n != o.ndof) return set_error(ICC_BAD_ARG, "icc_op_apply: n != ndof");
    cudaSetDevice(o.device);
    ICC_CUDA(cudaMemcpyAsync(o.d_x_in, x, (size_t)n * 8, cudaMemcpyHostToDevice, o.stream), "apply h2d");
    int rc = o.apply_dev(o.d_x_in, o.d_y_out);
    if (rc) return rc;
    ICC_CUDA(cudaMemcpyAsync(y, o.d_y_out, (size_t)n * 8, cudaMemcpyDeviceToHost, o.stream), "apply d2h");
    ICC_CUDA(cudaStreamSynchronize(o.stream), "apply sync");
    return ICC_OK;
}

int icc_op_apply_f32_dev(icc_op *op, const float *x, float *y, int64_t n) {
    if (!op || !x || !y) return set_error(ICC_BAD_ARG, "icc_op_apply_f32_dev: null argument");
    if (n != op->op.ndof) return set_error(ICC_BAD_ARG, "icc_op_apply_f32_dev: n != ndof");
    cudaSetDevice(op->op.device);
    return icc::mixed_apply_f32(op->op, x, y);
}

int icc_op_apply_f32(icc_op *op, const float *x, float *y, int64_t n) {
    if (!op || !x || !y) return set_error(ICC_BAD_ARG, "icc_op_apply_f32: null argument");
    icc::Op &o = op->op;
    if (n != o.ndof) return set_error(ICC_BAD_ARG, "icc_op_apply_f32: n != ndof");
    cudaSetDevice(o.device);
    float *xd = reinterpret_cast<float *>(o.d_x_in), *yd = reinterpret_cast<float *>(o.d_y_out);
    ICC_CUDA(cudaMemcpyAsync(xd, x, (size_t)n * 4, cudaMemcpyHostToDevice, o.stream), "apply_f32 h2d");
    int rc = icc::mixed_apply_f32(o, xd, yd);
    if (rc) return rc;
    ICC_CUDA(cudaMemcpyAsync(y, yd, (size_t)n * 4, cudaMemcpyDeviceToHost, o.stream), "apply_f32 d2h");
    ICC_CUDA(cudaStreamSynchronize(o.stream), "apply_f32 sync");
    return ICC_OK;
}

int icc_op_diagonal(icc_op *op, double *d, int64_t n) {
    if (!op || !d) return set_error(ICC_BAD_ARG, "icc_op_diagonal: null argument");
    icc::Op &o = op->op;
    if (n != o.ndof) return set_error(ICC_BAD_ARG, "icc_op_diagonal: n != ndof");
    cudaSetDevice(o.device);
    int rc = o.diagonal_dev(o.d_y_out);
    if (rc) return rc;
    ICC_CUDA(cudaMemcpyAsync(d, o.d_y_out, (size_t)n * 8, cudaMemcpyDeviceToHost, o.stream), "diag d2h");
    ICC_CUDA(cudaStreamSynchronize(o.stream), "diag sync");
    return ICC_OK;
}

int icc_solve_common(icc_op *op, const double *b_dev, const double *diag_dev, int64_t n, double tol,
                        int64_t max_iter, const icc_solve_opts *opts, double *x_dev, int64_t *iters, double *rel_res) {
    icc::Op &o = op->op;
    if (n != o.ndof) return set_error(ICC_BAD_ARG, "icc_pcg_solve: n != ndof");
    if (max_iter < 0 || !(tol >= 0.0)) return set_error(ICC_BAD_ARG, "icc_pcg_solve: bad tol or max_iter");
    icc_solve_opts def = {ICC_FP64, 32, 0.0, 0, 0};
    const icc_solve_opts *op_ = opts ? opts : &def;
    int64_t it = 0;
    double rr = 1.0;
    cudaEventRecord(o.ev0, o.stream);
    int rc;
    if (op_->precision == ICC_FP64) {
        rc = o.pcg_fp64(b_dev, diag_dev, tol, max_iter, op_->check_every, x_dev, &it, &rr);
    } else if (op_->precision == ICC_MIXED) {
        rc = icc::mixed_solve(o, b_dev, diag_dev, tol, max_iter, *op_, x_dev, &it, &rr);
    } else {
        return set_error(ICC_BAD_ARG, "icc_pcg_solve: unknown precision");
    }
    cudaEventRecord(o.ev1, o.stream);
    cudaEventSynchronize(o.ev1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, o.ev0, o.ev1);
    o.last_info.device_ms = ms;
    if (iters) *iters = it;
    if (rel_res) *rel_res = rr;
    return rc;
}

int icc_pcg_solve_dev(icc_op *op, const double *b_dev, const double *diag_dev, int64_t n, double tol,
                      int64_t max_iter, const icc_solve_opts *opts, double *x_dev, int64_t *iters, double *rel_res) {
    if (!op || !b_dev || !x_dev) return set_error(ICC_BAD_ARG, "icc_pcg_solve_dev: null argument");
    cudaSetDevice(op->op.device);
    int rc = icc_solve_common(op, b_dev, diag_dev, n, tol, max_iter, opts, x_dev, iters, rel_res);
    cudaError_t e = cudaStreamSynchronize(op->op.stream);
    if (e != cudaSuccess && rc >= 0) return icc::set_error(ICC_CUDA_ERROR, cudaGetErrorString(e));
    return rc;
}

int icc_pcg_solve(icc_op *op, const double *b, const double *diag, int64_t n, double tol, int64_t max_iter,
                  const icc_solve_opts *opts, double *x, int64_t *iters, double *rel_res) {
    if (!op || !b || !x) return set_error(ICC_BAD_ARG, "icc_pcg_solve: null argument");
    icc::Op &o = op->op;
    if (n != o.ndof) return set_error(ICC_BAD_ARG, "icc_pcg_solve: n != ndof");
    cudaSetDevice(o.device);
    int rc = o.ensure_pcg_buffers();
    if (rc) return rc;
    ICC_CUDA(cudaMemcpyAsync(o.d_b, b, (size_t)n * 8, cudaMemcpyHostToDevice, o.stream), "solve h2d");
    if (diag) ICC_CUDA(cudaMemcpyAsync(o.d_diag, diag, (size_t)n * 8, cudaMemcpyHostToDevice, o.stream), "solve h2d");
    rc = icc_solve_common(op, o.d_b, diag ? o.d_diag : nullptr, n, tol, max_iter, opts, o.d_y_out, iters, rel_res);
    if (rc < 0) return rc;
    ICC_CUDA(cudaMemcpyAsync(x, o.d_y_out, (size_t)n * 8, cudaMemcpyDeviceToHost, o.stream), "solve d2h");
    ICC_CUDA(cudaStreamSynchronize(o.stream), "solve sync");
    return rc;
}

int icc_pcg_solve_batched(int32_t count, icc_op *const *ops, const double *const *b, const double *const *diag,
                          double tol, int64_t max_iter, const icc_solve_opts *opts, double *const *x, int64_t *iters,
                          double *rel_res, int32_t *status) {
    if (count < 0 || (count > 0 && (!ops || !b || !x || !status)))
        return set_error(ICC_BAD_ARG, "icc_pcg_solve_batched: null argument");
    for (int32_t i = 0; i < count; ++i)
        if (!ops[i] || !b[i] || !x[i]) return set_error(ICC_BAD_ARG, "icc_pcg_solve_batched: null instance argument");
    {
        std::vector<const icc_op *> seen(ops, ops + count);
        std::sort(seen.begin(), seen.end());
        if (std::adjacent_find(seen.begin(), seen.end()) != seen.end())
            return set_error(ICC_BAD_ARG, "icc_pcg_solve_batched: a handle appears twice (each instance needs its own)");
    }
    if (opts && opts->precision == ICC_MIXED && count > 0) {
        // one batched solve: every iteration of all instances in one persistent tensor-core apply
        // and one fused vector step, captured in one CUDA graph
        std::vector<icc::Op *> o((size_t)count);
        std::vector<icc::VecSet *> vs((size_t)count);
        std::vector<const double *> bd((size_t)count), dd((size_t)count);
        std::vector<double *> xd((size_t)count);
        std::vector<double> tl((size_t)count, tol);
        std::vector<int64_t> mi((size_t)count, max_iter), reps((size_t)count, 0);
        const int dev = ops[0]->op.device;
        for (int32_t i = 0; i < count; ++i) {
            icc::Op &oi = ops[i]->op;
            if (oi.device != dev) return set_error(ICC_BAD_ARG, "icc_pcg_solve_batched: handles on different devices");
            if (max_iter < 0 || !(tol >= 0.0)) return set_error(ICC_BAD_ARG, "icc_pcg_solve_batched: bad tol or max_iter");
            cudaSetDevice(oi.device);
            int rc = oi.ensure_pcg_buffers();
            if (rc) return rc;
            o[(size_t)i] = &oi;
            if (!(vs[(size_t)i] = icc::mixed_own_vecset(oi))) return ICC_BAD_ARG;
            ICC_CUDA(cudaMemcpyAsync(oi.d_b, b[i], (size_t)oi.ndof * 8, cudaMemcpyHostToDevice, oi.stream), "batch h2d");
            if (diag && diag[i])
                ICC_CUDA(cudaMemcpyAsync(oi.d_diag, diag[i], (size_t)oi.ndof * 8, cudaMemcpyHostToDevice, oi.stream),
                         "batch h2d");
            bd[(size_t)i] = oi.d_b;
            dd[(size_t)i] = (diag && diag[i]) ? oi.d_diag : nullptr;
            xd[(size_t)i] = oi.d_y_out;
        }
        cudaStream_t s = ops[0]->op.stream;
        std::vector<int> st((size_t)count, 0);
        int rc = icc::mixed_solve_batch(s, o, vs, bd.data(), dd.data(), tl.data(), mi.data(), *opts, xd.data(), st.data(),
                                        iters, rel_res, reps.data());
        if (rc) return rc;
        for (int32_t i = 0; i < count; ++i) {
            ICC_CUDA(cudaMemcpyAsync(x[i], o[(size_t)i]->d_y_out, (size_t)o[(size_t)i]->ndof * 8, cudaMemcpyDeviceToHost, s),
                     "batch d2h");
            status[i] = st[(size_t)i];
        }
        ICC_CUDA(cudaStreamSynchronize(s), "batch d2h");
        for (int32_t i = 0; i < count; ++i)
            if (status[i] < 0) return set_error(status[i], "instance " + std::to_string(i) + " failed");
        return ICC_OK;
    }
    // FP64: instances on worker threads, each solving on its handle's own stream: the GPU
    // interleaves the instances' kernels (small grids leave SMs to the others); every solve is
    // deterministic, so the results equal those of sequential calls
    std::atomic<int32_t> next(0);
    std::vector<std::string> errs((size_t)count);
    auto work = [&]() {
        for (;;) {
            const int32_t i = next.fetch_add(1);
            if (i >= count) return;
            icc::Op &o = ops[i]->op;
            cudaSetDevice(o.device);
            int64_t it = 0;
            double rr = 1.0;
            const int rc = icc_pcg_solve(ops[i], b[i], diag ? diag[i] : nullptr, o.ndof, tol, max_iter, opts, x[i], &it,
                                         &rr);
            status[i] = rc;
            if (iters) iters[i] = it;
            if (rel_res) rel_res[i] = rr;
            if (rc < 0) errs[(size_t)i] = icc_last_error();
        }
    };
    const int32_t nthreads = std::max<int32_t>(1, std::min<int32_t>(count, 16));
    std::vector<std::thread> pool;
    for (int32_t t = 1; t < nthreads; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    for (int32_t i = 0; i < count; ++i)
        if (status[i] < 0) return set_error(status[i], "instance " + std::to_string(i) + ": " + errs[(size_t)i]);
    return ICC_OK;
}

int icc_op_profile_apply(icc_op *op, const double *x_dev, double *y_dev, int32_t reps, double *contract_ms,
                         double *gather_ms) {
    if (!op || !x_dev || !y_dev || reps <= 0) return set_error(ICC_BAD_ARG, "icc_op_profile_apply: bad argument");
    icc::Op &o = op->op;
    cudaSetDevice(o.device);
    std::vector<cudaEvent_t> ev(3 * size_t(reps));
    for (auto &e : ev) ICC_CUDA(cudaEventCreate(&e), "event create");
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(ev[3 * r], o.stream);
        icc::apply_f64_kernel<<<o.g.nbricks, icc::kApplyThreads, icc::kApplySmem, o.stream>>>(
            o.g, x_dev, o.d_mask, o.mask_mode != ICC_MASK_NONE, o.d_scale, o.d_kfrag, o.d_tile_start, o.d_tile_type,
            o.d_tile_elem, o.d_patch, nullptr);
        cudaEventRecord(ev[3 * r + 1], o.stream);
        icc::gather_kernel<double><<<o.vec_blocks, icc::kVecThreads, 0, o.stream>>>(
            o.g, o.d_patch, x_dev, o.d_mask, o.mask_mode, o.extra64(), y_dev, nullptr, nullptr);
        cudaEventRecord(ev[3 * r + 2], o.stream);
    }
    cudaError_t e = cudaEventSynchronize(ev.back());
    double a = 0.0, g = 0.0;
    for (int r = 0; r < reps && e == cudaSuccess; ++r) {
        float t1 = 0.f, t2 = 0.f;
        cudaEventElapsedTime(&t1, ev[3 * r], ev[3 * r + 1]);
        cudaEventElapsedTime(&t2, ev[3 * r + 1], ev[3 * r + 2]);
        a += t1;
        g += t2;
    }
    for (auto &x : ev) cudaEventDestroy(x);
    ICC_CUDA(e, "profile apply");
    if (contract_ms) *contract_ms = a / reps;
    if (gather_ms) *gather_ms = g / reps;
    return ICC_OK;
}

int icc_op_profile_apply_f32(icc_op *op, const float *x_dev, float *y_dev, int32_t reps, double *contract_ms,
                             double *gather_ms) {
    if (!op || !x_dev || !y_dev || reps <= 0 || !contract_ms || !gather_ms)
        return set_error(ICC_BAD_ARG, "icc_op_profile_apply_f32: bad argument");
    cudaSetDevice(op->op.device);
    return icc::mixed_profile_apply(op->op, x_dev, y_dev, reps, contract_ms, gather_ms);
}

int icc_op_set_wait_limit(icc_op *op, int64_t grid_polls) {
    if (!op || grid_polls < 0) return set_error(ICC_BAD_ARG, "icc_op_set_wait_limit: bad argument");
    cudaSetDevice(op->op.device);
    return icc::mixed_set_wait_limit(op->op, grid_polls);
}

int icc_op_last_solve_info(const icc_op *op, icc_solve_info *info) {
    if (!op || !info) return set_error(ICC_BAD_ARG, "icc_op_last_solve_info: null argument");
    *info = op->op.last_info;
    return ICC_OK;
}

}  // extern "C"
