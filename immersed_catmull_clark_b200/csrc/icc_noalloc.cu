// FP64 operator apply for callers that cannot allocate device memory.
//
// Some host applications own every byte of device memory: they hand a library device buffers
// carved from their own pool and do not allow it to call cudaMalloc or cudaFree (cudaMalloc can
// synchronize the whole device and would grow a footprint the application budgets itself), and
// some control loops must not allocate anything once they have started.  The handle-based
// operator (icc_op_create) allocates its element data, brick partials and vectors, so it is not
// usable there.  icc_apply_f64_noalloc computes the same y = sum_e s_e K_type(e) x_e from buffers
// the caller already owns and takes the one scratch buffer it needs -- the per-brick partial sums
// that the node-side pass adds up -- from a fixed array in this file.
//
// The scratch array is a file-scope __device__ variable of kNoallocScratchBytes (16 MiB): every
// GPU that loads this library holds it until the process exits.  It fits grids of at most
// kNoallocMaxBricks bricks of 8x4x4 elements (for example 96x48x48 elements); larger grids are
// rejected with ICC_BAD_ARG before any device work.  All calls share it and it keeps the last
// call's contents.  Nothing in it has to start at zero: each call writes every partial it later
// reads.  Calls whose work overlaps on the GPU (two streams, or two host threads) race on the
// array and must be ordered by the caller.
#include <cuda_runtime.h>

#include <climits>
#include <mutex>
#include <string>

#include "icc_device.cuh"
#include "icc_vec.cuh"

namespace icc {

constexpr size_t kNoallocScratchBytes = size_t(16) << 20;
constexpr int kNoallocMaxBricks = int(kNoallocScratchBytes / (sizeof(double) * 3 * kPVol));  // 1941

static __device__ __align__(256) double g_noalloc_scratch[kNoallocScratchBytes / sizeof(double)];

// Same brick contraction as apply_f64_kernel, but it reads the element matrices in the caller's
// row-major [ntypes][81][81] layout and needs no precomputed tile plan: a warp tile is 16
// consecutive elements of the brick, and a tile that holds several element types runs one DMMA
// pass per type (types taken in increasing order), each row keeping its own type's pass.
// Elements whose type id lies outside [0, ntypes) contribute nothing.
__global__ void __launch_bounds__(kApplyThreads, 2)
apply_f64_noalloc_kernel(Geom g, const double *__restrict__ x, const double *__restrict__ scale,
                         const double *__restrict__ ke, int ntypes, const int *__restrict__ type_id,
                         double *__restrict__ patch_out) {
    extern __shared__ double smem[];
    double *sx = smem;               // [3][PVOL]
    double *sy = smem + 3 * kPVol;   // [kEPB][81]
    __shared__ int koff[84];

    const int b = blockIdx.x;
    const int bxi = b % g.nbx, byi = (b / g.nbx) % g.nby, bzi = b / (g.nbx * g.nby);
    const int x0 = bxi * kBX, y0 = byi * kBY, z0 = bzi * kBZ;
    const int ex_n = min(kBX, g.nx - x0), ey_n = min(kBY, g.ny - y0), ez_n = min(kBZ, g.nz - z0);

    if (threadIdx.x < 84) {
        int k = threadIdx.x < 81 ? threadIdx.x : 0;
        int c = k / 27, a = k % 27;
        koff[threadIdx.x] = c * kPVol + ((a / 9) * kPY + (a / 3) % 3) * kPX + a % 3;
    }
    for (int i = threadIdx.x; i < 3 * kPVol; i += blockDim.x) {
        int c = i / kPVol, r = i - c * kPVol;
        int px = r % kPX, py = (r / kPX) % kPY, pz = r / (kPX * kPY);
        int gx = x0 + px, gy = y0 + py, gz = z0 + pz;
        double v = 0.0;
        if (gx < g.cx && gy < g.cy && gz < g.cz) v = x[(long long)c * g.nsc + ((long long)gz * g.cy + gy) * g.cx + gx];
        sx[i] = v;
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    for (int tile = warp; tile < kEPB / 16; tile += kApplyThreads / 32) {
        int er[2], tr[2], base[2];
        double sr[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            int e = tile * 16 + gid + 8 * h;
            int lx = e % kBX, ly = (e / kBX) % kBY, lz = e / (kBX * kBY);
            bool ok = lx < ex_n && ly < ey_n && lz < ez_n;
            er[h] = e;
            base[h] = (lz * kPY + ly) * kPX + lx;
            tr[h] = -1;
            sr[h] = 0.0;
            if (ok) {
                long long eg = (long long)(x0 + lx) + (long long)g.nx * ((y0 + ly) + (long long)g.ny * (z0 + lz));
                int t = type_id[eg];
                if (t >= 0 && t < ntypes) {
                    tr[h] = t;
                    sr[h] = scale ? scale[eg] : 1.0;
                }
            }
        }
        bool done0 = tr[0] < 0, done1 = tr[1] < 0;
        for (;;) {
            int cand = min(done0 ? INT_MAX : tr[0], done1 ? INT_MAX : tr[1]);
            cand = __reduce_min_sync(0xffffffffu, cand);
            if (cand == INT_MAX) break;
            const double *K = ke + (size_t)cand * 81 * 81;
            double acc[kNTiles][4];
#pragma unroll
            for (int nt = 0; nt < kNTiles; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0;
#pragma unroll 3
            for (int ks = 0; ks < kKSteps; ++ks) {
                const int k = ks * 4 + tig;
                const int off = koff[k];
                const double a0 = sx[base[0] + off];
                const double a1 = sx[base[1] + off];
#pragma unroll
                for (int nt = 0; nt < kNTiles; ++nt) {
                    const int n = nt * 8 + gid;
                    const double bf = (k < 81 && n < 81) ? __ldg(K + n * 81 + k) : 0.0;
                    dmma_m16n8k4(acc[nt], a0, a1, bf);
                }
            }
#pragma unroll
            for (int nt = 0; nt < kNTiles; ++nt) {
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    int n = nt * 8 + 2 * tig + j;
                    if (n < 81) {
                        if (!done0 && tr[0] == cand) sy[er[0] * 81 + n] = sr[0] * acc[nt][j];
                        if (!done1 && tr[1] == cand) sy[er[1] * 81 + n] = sr[1] * acc[nt][2 + j];
                    }
                }
            }
            if (tr[0] == cand) done0 = true;
            if (tr[1] == cand) done1 = true;
        }
        // rows of elements that contribute nothing
#pragma unroll
        for (int h = 0; h < 2; ++h)
            if (tr[h] < 0)
                for (int n = 2 * tig; n < 81; n += 8) {
                    sy[er[h] * 81 + n] = 0.0;
                    if (n + 1 < 81) sy[er[h] * 81 + n + 1] = 0.0;
                }
    }
    __syncthreads();

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

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
double *g_noalloc_ptr[kMaxDevices] = {};
}  // namespace

// Once per device, with that device current: resolve the device address of the scratch array
// (in host code its name is only a host-side stand-in) and raise the kernel's shared-memory limit.
static int noalloc_setup(int dev, double **out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        double *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "icc_apply_f64_noalloc: cudaGetSymbolAddress");
        e = cudaFuncSetAttribute(apply_f64_noalloc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kApplySmem);
        if (e != cudaSuccess) return cuda_fail(e, "icc_apply_f64_noalloc: cudaFuncSetAttribute");
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return ICC_OK;
}

}  // namespace icc

extern "C" int icc_apply_f64_noalloc(const int64_t nel_dir[3], const double *ke_types_dev, int32_t ntypes,
                                     const int32_t *type_id_dev, const double *scale_dev, const double *x_dev,
                                     double *y_dev, void *stream) {
    using namespace icc;
    if (!nel_dir || !ke_types_dev || !type_id_dev || !x_dev || !y_dev || ntypes <= 0)
        return set_error(ICC_BAD_ARG, "icc_apply_f64_noalloc: null argument or ntypes <= 0");
    for (int d = 0; d < 3; ++d)
        if (nel_dir[d] < 1 || nel_dir[d] > (1 << 20))
            return set_error(ICC_BAD_ARG, "icc_apply_f64_noalloc: element counts must lie in [1, 2^20]");
    Geom g{};
    g.nx = int(nel_dir[0]); g.ny = int(nel_dir[1]); g.nz = int(nel_dir[2]);
    g.cx = g.nx + 2; g.cy = g.ny + 2; g.cz = g.nz + 2;
    g.nsc = (long long)g.cx * g.cy * g.cz;
    long long nbx = (g.nx + kBX - 1) / kBX, nby = (g.ny + kBY - 1) / kBY, nbz = (g.nz + kBZ - 1) / kBZ;
    long long nb = nbx * nby * nbz;
    if (nb > kNoallocMaxBricks)
        return set_error(ICC_BAD_ARG, "icc_apply_f64_noalloc: grid needs " + std::to_string(nb) +
                                          " bricks of 8x4x4 elements, the fixed scratch holds at most " +
                                          std::to_string(kNoallocMaxBricks));
    g.nbx = int(nbx); g.nby = int(nby); g.nbz = int(nbz);
    g.nbricks = int(nb);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "icc_apply_f64_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return set_error(ICC_BAD_ARG, "icc_apply_f64_noalloc: device index too large");
    double *scratch = nullptr;
    int rc = noalloc_setup(dev, &scratch);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    apply_f64_noalloc_kernel<<<g.nbricks, kApplyThreads, kApplySmem, s>>>(g, x_dev, scale_dev, ke_types_dev, ntypes,
                                                                         type_id_dev, scratch);
    gather_kernel<double><<<sms * 4, kVecThreads, 0, s>>>(g, scratch, x_dev, nullptr, ICC_MASK_NONE, Sparse<double>(), y_dev, nullptr,
                                                          nullptr);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "icc_apply_f64_noalloc: launch");
    return ICC_OK;
}
