// Immersed fictitious-domain set-up on the device: per-cell volume fractions of an analytic solid
// by the reference's rule (rust/src/immersed.rs:88-155 classify_background_cells +
// element_weights): a cell whose 8 vertices are all inside is inside (weight 1), all outside is
// outside (0), otherwise it is cut and its weight is the fraction of sub^3 midpoints inside.  The
// solid is the unit cube minus three orthogonal through-cylinders of radius r about the centre
// lines (the immersed benchmark geometry).  Arithmetic uses explicit round-to-nearest operations
// in the reference's order, so weights are bitwise those of a CPU evaluation of the same rule.
#include <cuda_runtime.h>

#include "icc_device.cuh"

namespace icc {
namespace {

__device__ __forceinline__ int cyl_inside(double qx, double qy, double qz, double r2) {
    if (qx < 0.0 || qx > 1.0 || qy < 0.0 || qy > 1.0 || qz < 0.0 || qz > 1.0) return 0;
    const double x = __dsub_rn(qx, 0.5), y = __dsub_rn(qy, 0.5), z = __dsub_rn(qz, 0.5);
    const double xx = __dmul_rn(x, x), yy = __dmul_rn(y, y), zz = __dmul_rn(z, z);
    if (__dadd_rn(yy, zz) < r2) return 0;   // cylinder along x
    if (__dadd_rn(xx, zz) < r2) return 0;   // along y
    if (__dadd_rn(xx, yy) < r2) return 0;   // along z
    return 1;
}

// vertex i of n + 1 equally spaced points on [0, 1] (the last one exactly 1)
__device__ __forceinline__ double vertex(long long i, long long n, double step) {
    return i == n ? 1.0 : __dmul_rn((double)i, step);
}

__global__ void cylinder_weights_kernel(int nx, int ny, int nz, int sx, int sy, int sz, double radius,
                                        double *__restrict__ w, int8_t *__restrict__ status) {
    const long long ncell = (long long)nx * ny * nz;
    const double r2 = __dmul_rn(radius, radius);
    const double stx = __ddiv_rn(1.0, (double)nx), sty = __ddiv_rn(1.0, (double)ny), stz = __ddiv_rn(1.0, (double)nz);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ncell; e += (long long)gridDim.x * blockDim.x) {
        const long long i = e % nx, j = (e / nx) % ny, k = e / ((long long)nx * ny);
        int s = 0;
        for (int dk = 0; dk < 2; ++dk)
            for (int dj = 0; dj < 2; ++dj)
                for (int di = 0; di < 2; ++di)
                    s += cyl_inside(vertex(i + di, nx, stx), vertex(j + dj, ny, sty), vertex(k + dk, nz, stz), r2);
        const int8_t st = s == 8 ? 1 : (s == 0 ? 0 : -1);
        status[e] = st;
        if (st != -1) {
            w[e] = st == 1 ? 1.0 : 0.0;
            continue;
        }
        // cut cell: midpoints lo + (a + 1/2) dx with lo = idx h, dx = ((idx + 1) h - idx h) / sub
        const double lo0 = __dmul_rn((double)i, stx), lo1 = __dmul_rn((double)j, sty), lo2 = __dmul_rn((double)k, stz);
        const double dx0 = __ddiv_rn(__dsub_rn(__dmul_rn((double)(i + 1), stx), lo0), (double)sx);
        const double dx1 = __ddiv_rn(__dsub_rn(__dmul_rn((double)(j + 1), sty), lo1), (double)sy);
        const double dx2 = __ddiv_rn(__dsub_rn(__dmul_rn((double)(k + 1), stz), lo2), (double)sz);
        long long n_in = 0;
        for (int c = 0; c < sz; ++c) {
            const double qz = __dadd_rn(lo2, __dmul_rn(__dadd_rn((double)c, 0.5), dx2));
            for (int b = 0; b < sy; ++b) {
                const double qy = __dadd_rn(lo1, __dmul_rn(__dadd_rn((double)b, 0.5), dx1));
                for (int a = 0; a < sx; ++a) {
                    const double qx = __dadd_rn(lo0, __dmul_rn(__dadd_rn((double)a, 0.5), dx0));
                    n_in += cyl_inside(qx, qy, qz, r2);
                }
            }
        }
        w[e] = __ddiv_rn((double)n_in, (double)((long long)sx * sy * sz));
    }
}

}  // namespace
}  // namespace icc

extern "C" {

int icc_cylinder_weights(const int64_t res[3], const int32_t sub[3], double radius, double *weights, int8_t *status) {
    if (!res || !sub || !weights || !status) return icc::set_error(ICC_BAD_ARG, "icc_cylinder_weights: null argument");
    for (int d = 0; d < 3; ++d)
        if (res[d] < 1 || res[d] > (1 << 20) || sub[d] < 1 || sub[d] > 64)
            return icc::set_error(ICC_BAD_ARG, "icc_cylinder_weights: bad resolution or sub-sampling");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return icc::set_error(ICC_NO_DEVICE, "no CUDA device");
    const long long ncell = res[0] * res[1] * res[2];
    double *d_w = nullptr;
    int8_t *d_s = nullptr;
    cudaError_t e = cudaMalloc((void **)&d_w, (size_t)ncell * 8);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_s, (size_t)ncell);
    if (e == cudaSuccess) {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        icc::cylinder_weights_kernel<<<sms * 8, 256>>>(int(res[0]), int(res[1]), int(res[2]), sub[0], sub[1], sub[2],
                                                       radius, d_w, d_s);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(weights, d_w, (size_t)ncell * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(status, d_s, (size_t)ncell, cudaMemcpyDeviceToHost);
    cudaFree(d_w);
    cudaFree(d_s);
    if (e != cudaSuccess) return icc::cuda_fail(e, "icc_cylinder_weights");
    return ICC_OK;
}

}  // extern "C"
