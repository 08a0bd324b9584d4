// Node-side sum of brick partials and the PCG vector kernels, templated on the vector type:
// T = double for the FP64 solve, T = float for the inner solve of the mixed form.  Every
// reduction accumulates in double with a fixed-shape two-stage tree (per-CTA partials, then one
// CTA), so results are reproducible run to run.
#pragma once

#include "icc_device.cuh"

namespace icc {

// Bricks containing node j along one direction: the brick min(j / B, nb - 1) and, for the two
// lowest patch planes of that brick, also the previous one.  Lower brick first.
__device__ __forceinline__ int node_bricks(int j, int B, int nb, int *bi, int *li) {
    int i1 = min(j / B, nb - 1);
    int l1 = j - i1 * B;
    if (l1 <= 1 && i1 >= 1) {
        bi[0] = i1 - 1;
        li[0] = l1 + B;
        bi[1] = i1;
        li[1] = l1;
        return 2;
    }
    bi[0] = i1;
    li[0] = l1;
    return 1;
}

// ---- PCG scalar steps (rust/src/solver.rs:41-71), run by one thread ---------------------------

// p'Ap -> alpha, or breakdown (rust/src/solver.rs:41-51)
__device__ __forceinline__ void pcg_alpha_step(PcgState *st, double p_ap) {
    st->iter += 1;
    st->p_ap = p_ap;
    if (!(p_ap > 0.0)) st->status = isfinite(p_ap) ? kStatBreakdown : kStatNan;
    else st->alpha = st->rz_old / p_ap;
}

// relative residual test, then beta (rust/src/solver.rs:56-71)
__device__ __forceinline__ void pcg_beta_step(PcgState *st, double rr, double rz) {
    double res = sqrt(rr) / st->norm_b;
    st->rel_res = res;
    st->rz_prev = st->rz_old;  // the r'z of this iteration's alpha
    if (res < st->tol) {
        st->status = kStatConverged;
    } else if (!isfinite(res)) {
        st->status = kStatNan;
    } else {
        st->beta = rz / st->rz_old;
        st->rz_old = rz;
        if (st->iter >= st->max_iter) st->status = kStatMaxIter;
    }
}

// True in exactly one CTA: the last to finish.  Every CTA has stored its partial before calling;
// the last one then reads all partials (in fixed order, so the result does not depend on which
// CTA is last) and resets the counter for the next use.
__device__ __forceinline__ bool last_block(unsigned *counter) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (is_last) {
        __threadfence();
        if (threadIdx.x == 0) *counter = 0u;
    }
    return is_last;
}

// The <= 8 brick partials of control point (ix, iy, iz) summed in a fixed order (lower bricks
// first along z, then y, then x).
template <class T>
__device__ __forceinline__ void node_partials(const Geom &g, const T *__restrict__ patch, int ix, int iy, int iz, T &s0,
                                              T &s1, T &s2) {
    int bx[2], lx[2], by[2], ly[2], bz[2], lz[2];
    const int nbx = node_bricks(ix, kBX, g.nbx, bx, lx);
    const int nby = node_bricks(iy, kBY, g.nby, by, ly);
    const int nbz = node_bricks(iz, kBZ, g.nbz, bz, lz);
    s0 = s1 = s2 = T(0);
    for (int a = 0; a < nbz; ++a)
        for (int q = 0; q < nby; ++q)
            for (int w = 0; w < nbx; ++w) {
                const size_t brick = (size_t)bx[w] + (size_t)g.nbx * (by[q] + (size_t)g.nby * bz[a]);
                const T *pb = patch + brick * 3 * kPVol + (lz[a] * kPY + ly[q]) * kPX + lx[w];
                s0 += pb[0];
                s1 += pb[kPVol];
                s2 += pb[2 * kPVol];
            }
}

// Row idx of the sparse term applied to the masked input: sum_k S[idx][k] (m .* p)[k].
template <class T>
__device__ __forceinline__ T sparse_row(const Sparse<T> &sp, long long idx, const T *__restrict__ p,
                                        const uint8_t *__restrict__ mask, int mask_mode) {
    T acc = T(0);
    const int k1 = sp.ptr[idx + 1];
    for (int k = sp.ptr[idx]; k < k1; ++k) {
        const int j = sp.idx[k];
        const T xj = (mask_mode != ICC_MASK_NONE && !mask[j]) ? T(0) : p[j];
        acc += sp.val[k] * xj;
    }
    return acc;
}

// y = sum of the brick partials of each node (fixed order) plus the sparse term, output mask
// applied; optionally the CTA partial of p'y (in double), and with `fuse` the alpha step in the
// last CTA.
template <class T>
__global__ void __launch_bounds__(kVecThreads)
gather_kernel(Geom g, const T *__restrict__ patch, const T *__restrict__ p, const uint8_t *__restrict__ mask,
              int mask_mode, Sparse<T> sp, T *__restrict__ y, double *__restrict__ partials, const PcgState *st,
              PcgState *fuse = nullptr, unsigned *counter = nullptr) {
    if (st && st->status != 0) return;
    double dot = 0.0;
    // one warp per row (iy, iz) of control points, lanes along x: the brick partials of
    // neighbouring nodes are neighbouring floats, and the row's divisions are paid once
    const int lane = threadIdx.x & 31;
    const int nrows = g.cy * g.cz;
    const int wstride = (gridDim.x * blockDim.x) >> 5;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nrows; row += wstride) {
        const int iy = row % g.cy, iz = row / g.cy;
        int by[2], ly[2], bz[2], lz[2];
        const int nby = node_bricks(iy, kBY, g.nby, by, ly);
        const int nbz = node_bricks(iz, kBZ, g.nbz, bz, lz);
        for (int ix = lane; ix < g.cx; ix += 32) {
            const long long n = (long long)row * g.cx + ix;
            int bx[2], lx[2];
            const int nbx = node_bricks(ix, kBX, g.nbx, bx, lx);
            T s0 = T(0), s1 = T(0), s2 = T(0);
            for (int a = 0; a < nbz; ++a)
                for (int q = 0; q < nby; ++q)
                    for (int w = 0; w < nbx; ++w) {
                        size_t brick = (size_t)bx[w] + (size_t)g.nbx * (by[q] + (size_t)g.nby * bz[a]);
                        const T *pb = patch + brick * 3 * kPVol + (lz[a] * kPY + ly[q]) * kPX + lx[w];
                        s0 += pb[0];
                        s1 += pb[kPVol];
                        s2 += pb[2 * kPVol];
                    }
            T sv[3] = {s0, s1, s2};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                long long idx = (long long)c * g.nsc + n;
                T v = sv[c];
                if (sp.ptr) v += sparse_row(sp, idx, p, mask, mask_mode);
                if (mask_mode == ICC_MASK_ZERO && !mask[idx]) v = T(0);
                else if (mask_mode == ICC_MASK_IDENTITY && !mask[idx]) v = p[idx];
                y[idx] = v;
                if (partials) dot += double(p[idx]) * double(v);
            }
        }
    }
    if (partials) {
        dot = block_sum(dot);
        if (threadIdx.x == 0) partials[blockIdx.x] = dot;
        if (fuse && last_block(counter)) {
            double s2 = 0.0;
            for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) s2 += __ldcg(partials + i);
            s2 = block_sum(s2);
            if (threadIdx.x == 0) pcg_alpha_step(fuse, s2);
        }
    }
}

// ---- PCG vector kernels (rust/src/solver.rs:14-76) -----------------------------------------

template <class T>
__global__ void inv_diag_kernel(long long n, const double *__restrict__ d, T *__restrict__ inv) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        inv[i] = T(fabs(d[i]) > 1e-12 ? 1.0 / d[i] : 1.0);
}

// x = 0, r = b, z = D^-1 r, p = z; partials: r'z and b'b   (rust/src/solver.rs:15-36)
// pmask != null keeps p zero on fixed DOFs (the mixed form's inner loop, ICC_MASK_ZERO)
template <class T>
__global__ void __launch_bounds__(kVecThreads)
pcg_init_kernel(long long n, const T *__restrict__ b, const T *__restrict__ inv, T *__restrict__ x,
                T *__restrict__ r, T *__restrict__ p, double *__restrict__ partials,
                const uint8_t *__restrict__ pmask = nullptr) {
    double rz = 0.0, bb = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        T bi = b[i], zi = inv[i] * bi;
        x[i] = T(0);
        r[i] = bi;
        p[i] = (pmask && !pmask[i]) ? T(0) : zi;
        rz += double(bi) * double(zi);
        bb += double(bi) * double(bi);
    }
    rz = block_sum(rz);
    bb = block_sum(bb);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = rz;
        partials[2 * blockIdx.x + 1] = bb;
    }
}

__global__ void __launch_bounds__(kVecThreads)
pcg_init_finalize(const double *__restrict__ partials, int np, PcgState *st, double tol, long long max_iter);

// p'Ap -> alpha, or breakdown (rust/src/solver.rs:41-51)
__global__ void __launch_bounds__(kVecThreads) pcg_alpha_kernel(const double *__restrict__ partials, int np, PcgState *st);

// relative residual test, then beta (rust/src/solver.rs:56-71)
__global__ void __launch_bounds__(kVecThreads) pcg_beta_kernel(const double *__restrict__ partials, int np, PcgState *st);

// x += alpha p; r -= alpha Ap; partials: r'r and r'z with z = D^-1 r (rust/src/solver.rs:52-66)
template <class T>
__global__ void __launch_bounds__(kVecThreads)
pcg_update_kernel(long long n, const T *__restrict__ p, const T *__restrict__ ap, const T *__restrict__ inv,
                  T *__restrict__ x, T *__restrict__ r, double *__restrict__ partials,
                  const PcgState *st, PcgState *fuse = nullptr, unsigned *counter = nullptr) {
    if (st->status != 0) return;
    const T alpha = T(st->alpha);
    double rr = 0.0, rz = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        T ri = r[i] - alpha * ap[i];
        r[i] = ri;
        rr += double(ri) * double(ri);
        rz += double(ri) * double(inv[i] * ri);
    }
    rr = block_sum(rr);
    rz = block_sum(rz);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = rr;
        partials[2 * blockIdx.x + 1] = rz;
    }
    if (fuse && last_block(counter)) {
        double a = 0.0, c = 0.0;
        for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
            a += __ldcg(partials + 2 * i);
            c += __ldcg(partials + 2 * i + 1);
        }
        a = block_sum(a);
        c = block_sum(c);
        if (threadIdx.x == 0) pcg_beta_step(fuse, a, c);
    }
}

// p = D^-1 r + beta p (rust/src/solver.rs:64-71).  With pmask: p is kept zero on fixed DOFs, or,
// when pm is given, p stays whole and pm = pmask .* p is written beside it.
template <class T>
__global__ void __launch_bounds__(kVecThreads)
pcg_p_kernel(long long n, const T *__restrict__ r, const T *__restrict__ inv, T *__restrict__ p,
             const PcgState *__restrict__ st, const uint8_t *__restrict__ pmask = nullptr, T *__restrict__ pm = nullptr) {
    if (st->status != 0) return;
    const T beta = T(st->beta);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const T v = inv[i] * r[i] + beta * p[i];
        if (pm) {
            p[i] = v;
            pm[i] = pmask[i] ? v : T(0);
        } else {
            p[i] = (pmask && !pmask[i]) ? T(0) : v;
        }
    }
}

}  // namespace icc
