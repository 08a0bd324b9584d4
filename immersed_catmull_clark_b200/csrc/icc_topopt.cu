// The callers of the hot path in the reference's SIMP cantilever loop, on the device:
//   solve_state      warm-started masked solve (rust/src/topopt_iga.rs:137-162)
//   element_energies u_e^T K_e u_e per element (rust/src/topopt_iga.rs:165-184)
//   run              SIMP scale, state solve, compliance, sensitivities, the radius filter on
//                    element centres and the optimality-criteria bisection with move limit
//                    (rust/src/topopt_iga.rs:73-129, :187-234)
// Reductions are deterministic (fixed-order two-stage sums); every vector stays on the device and
// only scalars (bisection means, compliance, change) come back to the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "icc_device.cuh"
#include "icc_vec.cuh"

namespace icc {

#define ICC_CUDA(call, where)                                      \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) return ::icc::cuda_fail(_e, where); \
    } while (0)

namespace {

constexpr int kTopoThreads = 256;
constexpr int kEnergyWarps = 8;

// ---- element strain energies ------------------------------------------------------------------
// One warp per element: the 81 values of u_e (connectivity from the element position) go to
// shared memory; lane l forms the rows a = l, l + 32, l + 64 of K_type(e) u_e in column order and
// adds u_a * row_a; the warp sum is the energy.
__global__ void __launch_bounds__(kEnergyWarps * 32)
energies_kernel(Geom g, const double *__restrict__ K, const int *__restrict__ type_id, const double *__restrict__ u,
                double *__restrict__ ee, int accumulate) {
    __shared__ double su[kEnergyWarps][81];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long nel = (long long)g.nx * g.ny * g.nz;
    for (long long e = (long long)blockIdx.x * kEnergyWarps + warp; e < nel; e += (long long)gridDim.x * kEnergyWarps) {
        const int ex = int(e % g.nx), ey = int((e / g.nx) % g.ny), ez = int(e / ((long long)g.nx * g.ny));
        for (int k = lane; k < 81; k += 32) {
            const int c = k / 27, a = k % 27;
            const long long node = (long long)(ex + a % 3) + (long long)g.cx * ((ey + (a / 3) % 3) + (long long)g.cy * (ez + a / 9));
            su[warp][k] = u[(long long)c * g.nsc + node];
        }
        __syncwarp();
        const double *Ke = K + (size_t)type_id[e] * 81 * 81;
        double s = 0.0;
        for (int a = lane; a < 81; a += 32) {
            double row = 0.0;
            for (int b = 0; b < 81; ++b) row += Ke[a * 81 + b] * su[warp][b];
            s += su[warp][a] * row;
        }
        s = warp_sum(s);
        if (lane == 0) ee[e] = accumulate ? ee[e] + s : s;
        __syncwarp();
    }
}

// ---- deterministic reductions -------------------------------------------------------------------
__device__ __forceinline__ double block_max(double v) {
    __shared__ double wm[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < (blockDim.x >> 5) ? wm[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
    }
    return r;
}

// part[0 .. np) -> *out, kind 0: sum, 1: max (fixed order)
__global__ void __launch_bounds__(kTopoThreads) finish_kernel(const double *__restrict__ part, int np, int kind,
                                                              double *__restrict__ out) {
    double v = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) v = kind ? fmax(v, part[i]) : v + part[i];
    v = kind ? block_max(v) : block_sum(v);
    if (threadIdx.x == 0) *out = v;
}

// ---- solve_state pieces ----------------------------------------------------------------------
// b = F - K u0 on free DOFs (0 on fixed); partials of |F_free|^2 and |b|^2
__global__ void __launch_bounds__(kTopoThreads)
state_rhs_kernel(long long n, const double *__restrict__ force, const double *__restrict__ ku0,
                 const uint8_t *__restrict__ mask, double *__restrict__ b, double *__restrict__ part) {
    double nf = 0.0, nb = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const bool fr = !mask || mask[i];
        const double bi = fr ? force[i] - ku0[i] : 0.0;
        b[i] = bi;
        if (fr) nf += force[i] * force[i];
        nb += bi * bi;
    }
    nf = block_sum(nf);
    nb = block_sum(nb);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = nf;
        part[gridDim.x + blockIdx.x] = nb;
    }
}

__global__ void clamp_diag_kernel(long long n, double *__restrict__ d, double floor) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] = fmax(d[i], floor);
}

// u = u0 + du on free DOFs, 0 on fixed
__global__ void state_update_kernel(long long n, const double *__restrict__ u0, const double *__restrict__ du,
                                    const uint8_t *__restrict__ mask, double *__restrict__ u) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        u[i] = (!mask || mask[i]) ? u0[i] + du[i] : 0.0;
}

// partial dot products a'b
__global__ void __launch_bounds__(kTopoThreads) dot_kernel(long long n, const double *__restrict__ a,
                                                           const double *__restrict__ b, double *__restrict__ part) {
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += a[i] * b[i];
    s = block_sum(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// ---- SIMP loop pieces ------------------------------------------------------------------------
__global__ void fill_kernel(long long n, double *__restrict__ x, double v) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = v;
}

// s_e = emin + (1 - emin) x_e^penal (rust/src/topopt_iga.rs:132)
__global__ void simp_scale_kernel(long long n, const double *__restrict__ x, double emin, double penal,
                                  double *__restrict__ s) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s[i] = emin + (1.0 - emin) * pow(x[i], penal);
}

// dc_raw = -penal (1 - emin) x^(penal-1) ee (rust/src/topopt_iga.rs:202)
__global__ void sens_kernel(long long n, const double *__restrict__ x, const double *__restrict__ ee, double emin,
                            double penal, double *__restrict__ dc_raw) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dc_raw[i] = -penal * (1.0 - emin) * pow(x[i], penal - 1.0) * ee[i];
}

// Radius filter on element centres as a stencil: the neighbours f of e within r, in increasing
// element index (offsets sorted by dz, dy, dx), weights max(r - |c_e - c_f|, 0)
// (rust/src/topopt_iga.rs:94-120, :203-208).  Partials of max |dc| for the bisection bracket.
__global__ void __launch_bounds__(kTopoThreads)
filter_kernel(Geom g, int nst, const int4 *__restrict__ off, const double *__restrict__ w, const double *__restrict__ x,
              const double *__restrict__ dc_raw, double *__restrict__ dc, double *__restrict__ part) {
    const long long nel = (long long)g.nx * g.ny * g.nz;
    double mx = 0.0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nel; e += (long long)gridDim.x * blockDim.x) {
        const int ex = int(e % g.nx), ey = int((e / g.nx) % g.ny), ez = int(e / ((long long)g.nx * g.ny));
        double sm = 0.0, fs = 0.0;
        for (int k = 0; k < nst; ++k) {
            const int4 o = off[k];
            const int fx = ex + o.x, fy = ey + o.y, fz = ez + o.z;
            if (fx < 0 || fy < 0 || fz < 0 || fx >= g.nx || fy >= g.ny || fz >= g.nz) continue;
            const long long f = fx + (long long)g.nx * (fy + (long long)g.ny * fz);
            sm += w[k] * x[f] * dc_raw[f];
            fs += w[k];
        }
        const double v = sm / (fs * fmax(x[e], 1e-3));
        dc[e] = v;
        mx = fmax(mx, fabs(v));
    }
    mx = block_max(mx);
    if (threadIdx.x == 0) part[blockIdx.x] = mx;
}

// OC candidate for the multiplier lmid and partial sums of it (rust/src/topopt_iga.rs:209-219)
__global__ void __launch_bounds__(kTopoThreads)
oc_kernel(long long n, const double *__restrict__ x_old, const double *__restrict__ dc, double lmid, double move,
          double *__restrict__ cand, double *__restrict__ part) {
    double s = 0.0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double be = sqrt(-dc[e] / lmid);
        const double xo = x_old[e];
        const double c = fmax(fmax(fmin(fmin(xo * be, xo + move), 1.0), xo - move), 0.001);
        cand[e] = c;
        s += c;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// partials of max |a - b|
__global__ void __launch_bounds__(kTopoThreads) maxdiff_kernel(long long n, const double *__restrict__ a,
                                                               const double *__restrict__ b, double *__restrict__ part) {
    double m = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(a[i] - b[i]));
    m = block_max(m);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}

template <class T>
int dalloc(T **p, size_t count, const char *what) {
    *p = nullptr;
    ICC_CUDA(cudaMalloc((void **)p, (count ? count : 1) * sizeof(T)), what);
    return ICC_OK;
}

}  // namespace

// Scratch of the state solve and the energies, owned by the operator (Op::state).  f and u stage
// the host arrays of the C-ABI calls; ktypes holds the row-major element matrices.
struct StateScratch {
    double *ku0 = nullptr, *b = nullptr, *du = nullptr, *diag = nullptr, *part = nullptr, *scal = nullptr;
    double *f = nullptr, *u = nullptr, *ee = nullptr, *ktypes = nullptr;
    int nblocks = 0;
    ~StateScratch() {
        void *p[] = {ku0, b, du, diag, part, scal, f, u, ee, ktypes};
        for (void *q : p)
            if (q) cudaFree(q);
    }
};

void state_release(Op &op) {
    delete op.state;
    op.state = nullptr;
}

static int state_scratch(Op &o, StateScratch &s) {
    int rc;
    if (!s.ku0) {
        s.nblocks = o.num_sms * 4;
        if ((rc = dalloc(&s.ku0, (size_t)o.ndof, "alloc state"))) return rc;
        if ((rc = dalloc(&s.b, (size_t)o.ndof, "alloc state"))) return rc;
        if ((rc = dalloc(&s.du, (size_t)o.ndof, "alloc state"))) return rc;
        if ((rc = dalloc(&s.diag, (size_t)o.ndof, "alloc state"))) return rc;
        if ((rc = dalloc(&s.part, (size_t)2 * s.nblocks, "alloc state"))) return rc;
        if ((rc = dalloc(&s.scal, 8, "alloc state"))) return rc;
        if ((rc = dalloc(&s.f, (size_t)o.ndof, "alloc state"))) return rc;
        if ((rc = dalloc(&s.u, (size_t)o.ndof, "alloc state"))) return rc;
        if ((rc = dalloc(&s.ee, (size_t)o.nel, "alloc state"))) return rc;
    }
    return ICC_OK;
}

static StateScratch &op_scratch(Op &o) {
    if (!o.state) o.state = new StateScratch();
    return *o.state;
}

static int state_ktypes(Op &o, StateScratch &s) {
    if (s.ktypes) return ICC_OK;
    int rc;
    if ((rc = dalloc(&s.ktypes, o.host_ktypes.size(), "alloc element matrices"))) return rc;
    ICC_CUDA(cudaMemcpyAsync(s.ktypes, o.host_ktypes.data(), o.host_ktypes.size() * 8, cudaMemcpyHostToDevice,
                             o.stream),
             "copy element matrices");
    ICC_CUDA(cudaStreamSynchronize(o.stream), "copy element matrices");
    return ICC_OK;
}

// Reduce part[0 .. np) (sum or max) into a host double, stream-ordered.
static int reduce_to_host(Op &o, StateScratch &s, const double *part, int np, int kind, double *out) {
    finish_kernel<<<1, kTopoThreads, 0, o.stream>>>(part, np, kind, s.scal);
    ICC_CUDA(cudaMemcpyAsync(out, s.scal, 8, cudaMemcpyDeviceToHost, o.stream), "reduce d2h");
    ICC_CUDA(cudaStreamSynchronize(o.stream), "reduce sync");
    return ICC_OK;
}

// solve_state on device arrays (rust/src/topopt_iga.rs:137-162)
static int solve_state_dev(icc_op *h, StateScratch &s, const double *force, const double *u0, double pcg_tol,
                           const icc_solve_opts *opts, double *u, int64_t *iters, double *rel_res) {
    Op &o = h->op;
    int rc;
    if ((rc = state_scratch(o, s))) return rc;
    const long long n = o.ndof;
    const int nb = s.nblocks;
    const uint8_t *mask = o.mask_mode != ICC_MASK_NONE ? o.d_mask : nullptr;
    // K u0 on the free rows (the masked operator; u0 vanishes on fixed DOFs)
    o.enqueue_apply(u0, s.ku0, nullptr, nullptr);
    state_rhs_kernel<<<nb, kTopoThreads, 0, o.stream>>>(n, force, s.ku0, mask, s.b, s.part);
    double nf2 = 0.0, rb2 = 0.0;
    if ((rc = reduce_to_host(o, s, s.part, nb, 0, &nf2))) return rc;
    if ((rc = reduce_to_host(o, s, s.part + nb, nb, 0, &rb2))) return rc;
    const double nfree = std::sqrt(nf2), rb = std::sqrt(rb2);
    if ((rc = o.diagonal_dev(s.diag))) return rc;
    clamp_diag_kernel<<<nb, kTopoThreads, 0, o.stream>>>(n, s.diag, 1e-12);
    const double tol = rb > 0.0 ? std::fmin(pcg_tol * nfree / rb, 0.5) : 1.0;
    int64_t it = 0;
    double r0 = 0.0;
    rc = icc_solve_common(h, s.b, s.diag, n, tol, 20 * n, opts, s.du, &it, &r0);
    if (rc < 0) return rc;
    state_update_kernel<<<nb, kTopoThreads, 0, o.stream>>>(n, u0, s.du, mask, u);
    ICC_CUDA(cudaGetLastError(), "state update");
    if (iters) *iters = it;
    if (rel_res) *rel_res = r0 * rb / std::fmax(nfree, 1e-300);
    return rc;
}

// The state solves of several load cases on one operator at once (rust/src/topopt_iga.rs:137-162
// per case): b_k = F_k - K u_k on the free DOFs and its rescaled tolerance, then one batched
// mixed-precision solve of all cases (their iterations share one persistent apply and one fused
// vector step), then u_k += du_k on the free DOFs.  force and u hold nload vectors of n; bk and duk
// are scratch of the same size; vsets[k] are the cases' FP32 vector sets.  iters = the summed
// iterations.
static int solve_states_batched(icc_op *h, StateScratch &s, int nload, const double *force, double *u, double *bk,
                                double *duk, const std::vector<VecSet *> &vsets, double pcg_tol,
                                const icc_solve_opts *opts, int64_t *iters) {
    Op &o = h->op;
    int rc;
    if ((rc = state_scratch(o, s))) return rc;
    const long long n = o.ndof;
    const int nb = s.nblocks;
    const uint8_t *mask = o.mask_mode != ICC_MASK_NONE ? o.d_mask : nullptr;
    std::vector<double> tol((size_t)nload);
    for (int k = 0; k < nload; ++k) {
        const double *fk = force + (size_t)k * n;
        double *uk = u + (size_t)k * n;
        o.enqueue_apply(uk, s.ku0, nullptr, nullptr);
        state_rhs_kernel<<<nb, kTopoThreads, 0, o.stream>>>(n, fk, s.ku0, mask, bk + (size_t)k * n, s.part);
        double nf2 = 0.0, rb2 = 0.0;
        if ((rc = reduce_to_host(o, s, s.part, nb, 0, &nf2))) return rc;
        if ((rc = reduce_to_host(o, s, s.part + nb, nb, 0, &rb2))) return rc;
        const double nfree = std::sqrt(nf2), rb = std::sqrt(rb2);
        tol[(size_t)k] = rb > 0.0 ? std::fmin(pcg_tol * nfree / rb, 0.5) : 1.0;
    }
    if ((rc = o.diagonal_dev(s.diag))) return rc;
    clamp_diag_kernel<<<nb, kTopoThreads, 0, o.stream>>>(n, s.diag, 1e-12);
    ICC_CUDA(cudaStreamSynchronize(o.stream), "state set-up");
    std::vector<Op *> ops((size_t)nload, &o);
    std::vector<const double *> bp((size_t)nload), dp((size_t)nload, s.diag);
    std::vector<double *> xp((size_t)nload);
    std::vector<int64_t> mi((size_t)nload, 20 * n), its((size_t)nload, 0), reps((size_t)nload, 0);
    std::vector<double> res((size_t)nload, 0.0);
    std::vector<int> st((size_t)nload, 0);
    for (int k = 0; k < nload; ++k) {
        bp[(size_t)k] = bk + (size_t)k * n;
        xp[(size_t)k] = duk + (size_t)k * n;
    }
    rc = mixed_solve_batch(o.stream, ops, vsets, bp.data(), dp.data(), tol.data(), mi.data(), *opts, xp.data(),
                           st.data(), its.data(), res.data(), reps.data());
    if (rc) return rc;
    int64_t sum = 0;
    for (int k = 0; k < nload; ++k) {
        if (st[(size_t)k] < 0) return set_error(st[(size_t)k], "load case " + std::to_string(k) + ": state solve failed");
        sum += its[(size_t)k];
        double *uk = u + (size_t)k * n;
        state_update_kernel<<<nb, kTopoThreads, 0, o.stream>>>(n, uk, duk + (size_t)k * n, mask, uk);
    }
    ICC_CUDA(cudaGetLastError(), "state update");
    if (iters) *iters = sum;
    return ICC_OK;
}

// ee = u_e^T K_e u_e, or ee += it (several load cases)
static int energies_dev(Op &o, StateScratch &s, const double *u, double *ee, bool accumulate = false) {
    int rc;
    if ((rc = state_ktypes(o, s))) return rc;
    energies_kernel<<<o.num_sms * 8, kEnergyWarps * 32, 0, o.stream>>>(o.g, s.ktypes, o.d_type_id, u, ee,
                                                                      accumulate ? 1 : 0);
    ICC_CUDA(cudaGetLastError(), "energies");
    return ICC_OK;
}

}  // namespace icc

// ------------------------------------------------------------------------------------------------
// Handles
// ------------------------------------------------------------------------------------------------

struct icc_topopt {
    icc_topopt_cfg cfg{};
    icc_space *sp = nullptr;
    icc_op *op = nullptr;
    long long ne = 0, n = 0;
    double *d_force = nullptr, *d_u = nullptr, *d_un = nullptr, *d_x = nullptr, *d_xold = nullptr,
           *d_cand = nullptr, *d_scale = nullptr, *d_ee = nullptr, *d_dcraw = nullptr, *d_dc = nullptr,
           *d_part = nullptr, *d_w = nullptr;
    int4 *d_off = nullptr;
    int nst = 0, nblocks = 0;
    int nload = 1;   // load cases: d_force and d_u hold nload vectors of n
    // batched mixed-precision state solves of several load cases: their right-hand sides and
    // corrections (nload vectors of n each) and FP32 vector sets (case 0: the operator's own)
    double *d_bk = nullptr, *d_duk = nullptr;
    std::vector<icc::VecSet *> vsets;
    ~icc_topopt() {
        for (size_t k = 1; k < vsets.size(); ++k) icc::mixed_vecset_destroy(vsets[k]);
        void *p[] = {d_force, d_u, d_un, d_x, d_xold, d_cand, d_scale, d_ee, d_dcraw, d_dc, d_part, d_w, d_off,
                     d_bk, d_duk};
        for (void *q : p)
            if (q) cudaFree(q);
        if (op) icc_op_destroy(op);
        if (sp) icc_space_destroy(sp);
    }
};

extern "C" {

int icc_solve_state(icc_op *op, const double *force, const double *u0, int64_t n, double pcg_tol,
                    const icc_solve_opts *opts, double *u, int64_t *iters, double *rel_res) {
    if (!op || !force || !u0 || !u) return icc::set_error(ICC_BAD_ARG, "icc_solve_state: null argument");
    icc::Op &o = op->op;
    if (n != o.ndof) return icc::set_error(ICC_BAD_ARG, "icc_solve_state: n != ndof");
    cudaSetDevice(o.device);
    int rc = o.ensure_pcg_buffers();
    if (rc) return rc;
    icc::StateScratch &s = icc::op_scratch(o);
    if ((rc = icc::state_scratch(o, s))) return rc;
    ICC_CUDA(cudaMemcpyAsync(s.f, force, (size_t)n * 8, cudaMemcpyHostToDevice, o.stream), "state h2d");
    ICC_CUDA(cudaMemcpyAsync(s.u, u0, (size_t)n * 8, cudaMemcpyHostToDevice, o.stream), "state h2d");
    rc = icc::solve_state_dev(op, s, s.f, s.u, pcg_tol, opts, s.u, iters, rel_res);   // u in place of u0
    if (rc < 0) return rc;
    ICC_CUDA(cudaMemcpyAsync(u, s.u, (size_t)n * 8, cudaMemcpyDeviceToHost, o.stream), "state d2h");
    ICC_CUDA(cudaStreamSynchronize(o.stream), "state sync");
    return rc;
}

int icc_op_element_energies(icc_op *op, const double *u, int64_t n, double *ee, int64_t nel) {
    if (!op || !u || !ee) return icc::set_error(ICC_BAD_ARG, "icc_op_element_energies: null argument");
    icc::Op &o = op->op;
    if (n != o.ndof || nel != o.nel) return icc::set_error(ICC_BAD_ARG, "icc_op_element_energies: bad sizes");
    cudaSetDevice(o.device);
    icc::StateScratch &s = icc::op_scratch(o);
    int rc;
    if ((rc = icc::state_scratch(o, s))) return rc;
    ICC_CUDA(cudaMemcpyAsync(s.u, u, (size_t)n * 8, cudaMemcpyHostToDevice, o.stream), "energies h2d");
    if ((rc = icc::energies_dev(o, s, s.u, s.ee))) return rc;
    ICC_CUDA(cudaMemcpyAsync(ee, s.ee, (size_t)nel * 8, cudaMemcpyDeviceToHost, o.stream), "energies d2h");
    ICC_CUDA(cudaStreamSynchronize(o.stream), "energies sync");
    return ICC_OK;
}

int icc_topopt_create(const int64_t nel[3], const icc_topopt_cfg *cfg, icc_topopt **out) {
    if (!nel || !cfg || !out) return icc::set_error(ICC_BAD_ARG, "icc_topopt_create: null argument");
    *out = nullptr;
    if (!(cfg->volfrac > 0.0 && cfg->volfrac <= 1.0) || !(cfg->rmin > 0.0) || !(cfg->move_limit > 0.0))
        return icc::set_error(ICC_BAD_ARG, "icc_topopt_create: bad volfrac, rmin or move_limit");
    auto *t = new (std::nothrow) icc_topopt();
    if (!t) return icc::set_error(ICC_OUT_OF_MEMORY, "icc_topopt_create: out of host memory");
    t->cfg = *cfg;
    const double bounds[6] = {0.0, cfg->size[0], 0.0, cfg->size[1], 0.0, cfg->size[2]};
    int rc = icc_space_create(bounds, nel, 2, &t->sp);
    if (rc) {
        delete t;
        return rc;
    }
    const icc::Space &S = t->sp->s;
    t->ne = S.nel;
    t->n = S.ndof;
    // clamp x = 0; load on control points with i1 = last, |i2 - 1| <= 1, |i3 - ncp3/2| <= 1 (1-based)
    // (rust/src/topopt_iga.rs:78-97)
    std::vector<uint8_t> free_mask((size_t)t->n, 1);
    std::vector<double> force((size_t)t->n, 0.0);
    std::vector<int64_t> load;
    const int64_t *nd = S.ncp;
    for (int64_t i = 0; i < S.nsc; ++i) {
        const int64_t s0 = i % nd[0], s1 = (i / nd[0]) % nd[1], s2 = i / (nd[0] * nd[1]);
        if (s0 == 0)
            for (int c = 0; c < 3; ++c) free_mask[(size_t)(c * S.nsc + i)] = 0;
        const double i2 = double(s1) + 1.0, i3 = double(s2) + 1.0;
        if (s0 + 1 == nd[0] && std::fabs(i2 - 1.0) <= 1.0 && std::fabs(i3 - double(nd[2]) / 2.0) <= 1.0)
            load.push_back(i);
    }
    for (int64_t i : load) force[(size_t)(S.nsc + i)] = -1.0 / double(load.size());
    double lambda, mu;
    icc_lame(cfg->young, cfg->poisson, &lambda, &mu);
    if ((rc = icc_op_create_lame(t->sp, lambda, mu, nullptr, free_mask.data(), ICC_MASK_ZERO, &t->op))) {
        delete t;
        return rc;
    }
    // filter stencil: element-centre offsets within r = rmin * mean(h), in increasing element index
    double h[3];
    for (int d = 0; d < 3; ++d) h[d] = S.len[d] / double(S.nel_dir[d]);
    const double r = cfg->rmin * (h[0] + h[1] + h[2]) / 3.0;
    int reach[3];
    for (int d = 0; d < 3; ++d) reach[d] = int(std::ceil(r / h[d])) + 1;
    std::vector<int4> off;
    std::vector<double> w;
    for (int dz = -reach[2]; dz <= reach[2]; ++dz)
        for (int dy = -reach[1]; dy <= reach[1]; ++dy)
            for (int dx = -reach[0]; dx <= reach[0]; ++dx) {
                const double a = double(dx) * h[0], b = double(dy) * h[1], c = double(dz) * h[2];
                const double d2 = a * a + b * b + c * c;
                if (d2 <= r * r) {
                    off.push_back(make_int4(dx, dy, dz, 0));
                    w.push_back(std::fmax(r - std::sqrt(d2), 0.0));
                }
            }
    t->nst = int(off.size());
    icc::Op &o = t->op->op;
    t->nblocks = o.num_sms * 4;
    auto al = [&](double **p, size_t cnt) { return icc::dalloc(p, cnt, "alloc topopt"); };
    const size_t ne = (size_t)t->ne, n = (size_t)t->n;
    if ((rc = al(&t->d_force, n)) || (rc = al(&t->d_u, n)) || (rc = al(&t->d_un, n)) || (rc = al(&t->d_x, ne)) ||
        (rc = al(&t->d_xold, ne)) || (rc = al(&t->d_cand, ne)) || (rc = al(&t->d_scale, ne)) ||
        (rc = al(&t->d_ee, ne)) || (rc = al(&t->d_dcraw, ne)) || (rc = al(&t->d_dc, ne)) ||
        (rc = al(&t->d_part, (size_t)t->nblocks)) || (rc = al(&t->d_w, w.size())) ||
        (rc = icc::dalloc(&t->d_off, off.size(), "alloc topopt"))) {
        delete t;
        return rc;
    }
    // ordered on the operator's stream, which runs every later kernel of the loop
    cudaError_t e = cudaMemcpyAsync(t->d_force, force.data(), n * 8, cudaMemcpyHostToDevice, o.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t->d_w, w.data(), w.size() * 8, cudaMemcpyHostToDevice, o.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(t->d_off, off.data(), off.size() * sizeof(int4), cudaMemcpyHostToDevice, o.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(o.stream);
    if (e != cudaSuccess) {
        delete t;
        return icc::cuda_fail(e, "copy topopt set-up");
    }
    *out = t;
    return ICC_OK;
}

void icc_topopt_destroy(icc_topopt *t) { delete t; }

int icc_topopt_set_loads(icc_topopt *t, int32_t nload, const double *forces) {
    if (!t || nload < 1 || !forces) return icc::set_error(ICC_BAD_ARG, "icc_topopt_set_loads: bad argument");
    icc::Op &o = t->op->op;
    cudaSetDevice(o.device);
    double *f = nullptr, *u = nullptr;
    const size_t cnt = (size_t)nload * (size_t)t->n;
    int rc;
    if ((rc = icc::dalloc(&f, cnt, "alloc loads"))) return rc;
    if ((rc = icc::dalloc(&u, cnt, "alloc loads"))) {
        cudaFree(f);
        return rc;
    }
    cudaError_t e = cudaMemcpyAsync(f, forces, cnt * 8, cudaMemcpyHostToDevice, o.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(o.stream);
    if (e != cudaSuccess) {
        cudaFree(f);
        cudaFree(u);
        return icc::cuda_fail(e, "copy loads");
    }
    cudaFree(t->d_force);
    cudaFree(t->d_u);
    t->d_force = f;
    t->d_u = u;
    t->nload = nload;
    // batched-solve buffers are sized for the previous number of cases
    for (size_t k = 1; k < t->vsets.size(); ++k) icc::mixed_vecset_destroy(t->vsets[k]);
    t->vsets.clear();
    cudaFree(t->d_bk);
    cudaFree(t->d_duk);
    t->d_bk = t->d_duk = nullptr;
    return ICC_OK;
}

int icc_topopt_run(icc_topopt *t, int32_t max_iter, double *compliance, double *change, int64_t *pcg_iters,
                   double *density, int32_t *iters_run) {
    if (!t || max_iter < 0) return icc::set_error(ICC_BAD_ARG, "icc_topopt_run: bad argument");
    icc::Op &o = t->op->op;
    cudaSetDevice(o.device);
    const icc_topopt_cfg &c = t->cfg;
    const long long ne = t->ne, n = t->n;
    const int nb = t->nblocks;
    icc::StateScratch &s = icc::op_scratch(o);
    int rc;
    if ((rc = o.ensure_pcg_buffers())) return rc;
    if ((rc = icc::state_scratch(o, s))) return rc;
    const icc_solve_opts opts = {c.precision, 32, 0.0, 0, 0};
    icc::fill_kernel<<<nb, icc::kTopoThreads, 0, o.stream>>>(ne, t->d_x, c.volfrac);
    ICC_CUDA(cudaMemsetAsync(t->d_u, 0, (size_t)t->nload * n * 8, o.stream), "zero u");
    int done = 0;
    for (int iter = 1; iter <= max_iter; ++iter) {
        ICC_CUDA(cudaMemcpyAsync(t->d_xold, t->d_x, (size_t)ne * 8, cudaMemcpyDeviceToDevice, o.stream), "x_old");
        icc::simp_scale_kernel<<<nb, icc::kTopoThreads, 0, o.stream>>>(ne, t->d_x, c.emin, c.penal, t->d_scale);
        if ((rc = o.set_scale_dev(t->d_scale))) return rc;
        // every load case: warm-started state, compliance F'u and energies, summed over the cases;
        // with mixed precision and several cases, all their state solves run as one batch
        int64_t it = 0;
        double comp = 0.0;
        const bool batched = t->nload > 1 && c.precision == ICC_MIXED;
        if (batched) {
            if (t->vsets.empty()) {
                t->vsets.push_back(icc::mixed_own_vecset(o));
                for (int k = 1; k < t->nload; ++k) t->vsets.push_back(icc::mixed_vecset_create(o));
                for (auto *v : t->vsets)
                    if (!v) return icc::set_error(ICC_OUT_OF_MEMORY, "icc_topopt_run: load-case vectors");
            }
            if (!t->d_bk) {
                if ((rc = icc::dalloc(&t->d_bk, (size_t)t->nload * n, "alloc loads")) ||
                    (rc = icc::dalloc(&t->d_duk, (size_t)t->nload * n, "alloc loads")))
                    return rc;
            }
            rc = icc::solve_states_batched(t->op, s, t->nload, t->d_force, t->d_u, t->d_bk, t->d_duk, t->vsets,
                                           c.pcg_tol, &opts, &it);
            if (rc < 0) return rc;
        }
        for (int k = 0; k < t->nload; ++k) {
            double *fk = t->d_force + (size_t)k * n, *uk = t->d_u + (size_t)k * n;
            if (!batched) {
                int64_t itk = 0;
                double res = 0.0;
                rc = icc::solve_state_dev(t->op, s, fk, uk, c.pcg_tol, &opts, t->d_un, &itk, &res);
                if (rc < 0) return rc;
                it += itk;
                ICC_CUDA(cudaMemcpyAsync(uk, t->d_un, (size_t)n * 8, cudaMemcpyDeviceToDevice, o.stream), "state copy");
            }
            double ck = 0.0;
            icc::dot_kernel<<<nb, icc::kTopoThreads, 0, o.stream>>>(n, fk, uk, t->d_part);
            if ((rc = icc::reduce_to_host(o, s, t->d_part, nb, 0, &ck))) return rc;
            comp += ck;
            if ((rc = icc::energies_dev(o, s, uk, t->d_ee, k > 0))) return rc;
        }
        icc::sens_kernel<<<nb, icc::kTopoThreads, 0, o.stream>>>(ne, t->d_x, t->d_ee, c.emin, c.penal, t->d_dcraw);
        icc::filter_kernel<<<nb, icc::kTopoThreads, 0, o.stream>>>(o.g, t->nst, t->d_off, t->d_w, t->d_x, t->d_dcraw,
                                                                   t->d_dc, t->d_part);
        double mx = 0.0;
        if ((rc = icc::reduce_to_host(o, s, t->d_part, nb, 1, &mx))) return rc;
        // OC bisection; the update is the candidate of the last bisection step
        double l1 = 0.0, l2 = 2.0 * mx;
        ICC_CUDA(cudaMemcpyAsync(t->d_cand, t->d_xold, (size_t)ne * 8, cudaMemcpyDeviceToDevice, o.stream), "cand");
        int steps = 0;
        while ((l2 - l1) / (l1 + l2 + 1e-10) > 1e-4) {
            if (++steps > 400) return icc::set_error(ICC_NOT_CONVERGED, "icc_topopt_run: OC bisection did not close");
            const double lmid = 0.5 * (l1 + l2);
            icc::oc_kernel<<<nb, icc::kTopoThreads, 0, o.stream>>>(ne, t->d_xold, t->d_dc, lmid, c.move_limit,
                                                                   t->d_cand, t->d_part);
            double sum = 0.0;
            if ((rc = icc::reduce_to_host(o, s, t->d_part, nb, 0, &sum))) return rc;
            if (sum / double(ne) > c.volfrac) l1 = lmid;
            else l2 = lmid;
        }
        std::swap(t->d_x, t->d_cand);
        double chg = 0.0;
        icc::maxdiff_kernel<<<nb, icc::kTopoThreads, 0, o.stream>>>(ne, t->d_x, t->d_xold, t->d_part);
        if ((rc = icc::reduce_to_host(o, s, t->d_part, nb, 1, &chg))) return rc;
        if (compliance) compliance[iter - 1] = std::fabs(comp);
        if (change) change[iter - 1] = chg;
        if (pcg_iters) pcg_iters[iter - 1] = it;
        done = iter;
        if (chg < 0.01 && iter >= 15) break;
    }
    if (density) {
        ICC_CUDA(cudaMemcpyAsync(density, t->d_x, (size_t)ne * 8, cudaMemcpyDeviceToHost, o.stream), "density d2h");
        ICC_CUDA(cudaStreamSynchronize(o.stream), "density sync");
    }
    if (iters_run) *iters_run = done;
    return ICC_OK;
}

}  // extern "C"
