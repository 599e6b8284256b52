// Hand-written discrete adjoint of the BGK duct step, with checkpointing.
//
// The differentiated model is the duct step of the AA kernels (lbm_aa.cu) in
// two-buffer push form, in FP32 or FP64 (template R):
//   f*_q(x) = f_q(x) + w (feq_q(rho, u) - f_q(x)),   rho = sum f, u = j/rho + F
//   f'_q(x + c_q) = f*_q(x)                             streaming link
//   f'_opp(q)(x)  = f*_q(x)                             x + c_q solid (halfway bounce-back)
//   f'_opp(q)(x)  = w_q rho(x) (1 + 3 u_in + 3 u_in^2)  x + c_q before the inlet plane,
//                                                        u_in = u_in(y, z) (the inlet control)
//   f'_opp(q)(x)  = f*_opp(q)(x)                        x + c_q past the outlet plane
// with the drag of a step D = sum over links into obstacle cells of 2 c_qx f*_q.
// The objective is J = mean of D over the steps [window_begin, window_end]
// (1-based, the drag of step n uses the collision of f^{n-1}); the controls are
// the inlet profile u_in(y, z) and the initial velocity field u0 (f^0 =
// feq(1, u0)).
//
// Reverse pass, one kernel per step, gather form (lambda = dJ/df):
//   lambda*_q(x) = lambda'_q(x + c_q)            streaming link
//               = lambda'_opp(q)(x) [+ 2 c_qx / nwin if x + c_q is an obstacle in the window]
//               = 0                                inlet / outlet links (f*_q leaves)
//   outlet copies: lambda*_opp(q)(x) += lambda'_opp(q)(x)
//   lambda_p(x) = (1 - w) lambda*_p + w (A + sum_a B_a (c_pa - (u_a - F_a)) / rho) + A_in
//   A = sum_q lambda*_q feq_q / rho,  B_a = sum_q lambda*_q w_q rho (3 c_qa + 9 (c_q.u) c_qa - 3 u_a)
//   A_in = sum over inlet links lambda'_opp(q)(x) w_q kin   (rho enters the inlet value)
//   dJ/du_in(y,z) += sum over inlet links lambda'_opp(q)(x) w_q rho (3 + 6 u_in)
// and at the end dJ/du0_a = sum_q lambda^0_q w_q (3 c_qa + 9 (c_q.u0) c_qa - 3 u0_a).
// The forward states the reverse pass needs are recomputed segment by segment
// from checkpoints taken every `checkpoint_every` steps.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "lbm_capi.h"
#include "lbm_common.cuh"
#include "lbm_internal.h"

namespace lbm {
void set_error(const std::string& msg);

namespace {

template <class R>
__device__ __forceinline__ R wR(int q) {
    return q == 0 ? R(1) / R(3) : (q <= 6 ? R(1) / R(18) : R(1) / R(36));
}

template <class R>
struct AdjP {
    const uint8_t* flags;
    const uint32_t* links;
    int nx, ny, nz;
    int64_t N;
    R omega, fx, fy, fz;
};

__device__ __forceinline__ int wrapa(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

template <class R>
__device__ __forceinline__ int64_t nbr(const AdjP<R>& p, int x, int y, int z, int q) {
    return ((int64_t)wrapa(z + cz(q), p.nz) * p.ny + wrapa(y + cy(q), p.ny)) * p.nx + wrapa(x + cx(q), p.nx);
}

template <class R>
__global__ void adj_init(AdjP<R> p, const double* __restrict__ u0, R* __restrict__ f) {
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < p.N; id += (int64_t)gridDim.x * blockDim.x) {
        const R ux = (R)u0[id], uy = (R)u0[p.N + id], uz = (R)u0[2 * p.N + id];
        const R uu = ux * ux + uy * uy + uz * uz;
        for (int q = 0; q < 19; ++q) {
            const R cu = (R)cx(q) * ux + (R)cy(q) * uy + (R)cz(q) * uz;
            f[q * p.N + id] = wR<R>(q) * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * uu);
        }
    }
}

// one push step f -> fn; per-block drag partial sums (FP64)
template <class R>
__global__ void __launch_bounds__(256) adj_fwd(AdjP<R> p, const R* __restrict__ f, R* __restrict__ fn,
                                               const double* __restrict__ uin, double* __restrict__ drag_part) {
    double drag = 0.0;
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < p.N; id += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t fl = p.flags[id];
        if (fl & F_SOLID) {
            for (int q = 0; q < 19; ++q) fn[q * p.N + id] = f[q * p.N + id];
            continue;
        }
        const int x = (int)(id % p.nx);
        const int64_t row = id / p.nx;
        const int y = (int)(row % p.ny), z = (int)(row / p.ny);
        R fq[19];
        R rho = 0, jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < 19; ++q) {
            fq[q] = f[q * p.N + id];
            rho += fq[q];
            jx += (R)cx(q) * fq[q]; jy += (R)cy(q) * fq[q]; jz += (R)cz(q) * fq[q];
        }
        const R ux = jx / rho + p.fx, uy = jy / rho + p.fy, uz = jz / rho + p.fz;
        const R uu = ux * ux + uy * uy + uz * uz;
        R fs[19];
        for (int q = 0; q < 19; ++q) {
            const R cu = (R)cx(q) * ux + (R)cy(q) * uy + (R)cz(q) * uz;
            const R feq = wR<R>(q) * rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * uu);
            fs[q] = fq[q] + p.omega * (feq - fq[q]);
        }
        const uint32_t lk = (fl & F_SPECIAL) ? p.links[id] : 0u;
        for (int q = 0; q < 19; ++q) {
            if (!((lk >> q) & 1u)) {
                fn[q * p.N + nbr(p, x, y, z, q)] = fs[q];
                continue;
            }
            const int xt = x + cx(q);
            const int o = opp(q);
            if (xt < 0) {
                const R u = (R)uin[(int64_t)z * p.ny + y];
                fn[o * p.N + id] = wR<R>(q) * rho * (R(1) + R(3) * u + R(3) * u * u);
            } else if (xt >= p.nx) {
                fn[o * p.N + id] = fs[o];
            } else {
                fn[o * p.N + id] = fs[q];
                if (p.flags[nbr(p, x, y, z, q)] & F_OBST) drag += 2.0 * cx(q) * (double)fs[q];
            }
        }
    }
    __shared__ double red[8];
    for (int o = 16; o > 0; o >>= 1) drag += __shfl_down_sync(0xffffffffu, drag, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = drag;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        drag_part[blockIdx.x] = s;
    }
}

// one reverse step: lam0 = (d f'/d f)^T lam1 (+ the drag term when wdrag != 0)
template <class R>
__global__ void __launch_bounds__(256) adj_bwd(AdjP<R> p, const R* __restrict__ f, const R* __restrict__ lam1,
                                               R* __restrict__ lam0, const double* __restrict__ uin,
                                               double* __restrict__ g_uin, R wdrag) {
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < p.N; id += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t fl = p.flags[id];
        if (fl & F_SOLID) {
            for (int q = 0; q < 19; ++q) lam0[q * p.N + id] = R(0);
            continue;
        }
        const int x = (int)(id % p.nx);
        const int64_t row = id / p.nx;
        const int y = (int)(row % p.ny), z = (int)(row / p.ny);
        R fq[19];
        R rho = 0, jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < 19; ++q) {
            fq[q] = f[q * p.N + id];
            rho += fq[q];
            jx += (R)cx(q) * fq[q]; jy += (R)cy(q) * fq[q]; jz += (R)cz(q) * fq[q];
        }
        const R ux = jx / rho + p.fx, uy = jy / rho + p.fy, uz = jz / rho + p.fz;
        const R uu = ux * ux + uy * uy + uz * uz;
        const uint32_t lk = (fl & F_SPECIAL) ? p.links[id] : 0u;
        R ls[19];
        for (int q = 0; q < 19; ++q) ls[q] = R(0);
        R a_in = 0;
        double g_in = 0.0;
        for (int q = 0; q < 19; ++q) {
            if (!((lk >> q) & 1u)) {
                ls[q] += lam1[q * p.N + nbr(p, x, y, z, q)];
                continue;
            }
            const int xt = x + cx(q);
            const int o = opp(q);
            const R lo = lam1[o * p.N + id];
            if (xt < 0) {
                const R u = (R)uin[(int64_t)z * p.ny + y];
                a_in += lo * wR<R>(q) * (R(1) + R(3) * u + R(3) * u * u);
                g_in += (double)(lo * wR<R>(q) * rho * (R(3) + R(6) * u));
            } else if (xt >= p.nx) {
                ls[o] += lo;
            } else {
                ls[q] += lo;
                if (wdrag != R(0) && (p.flags[nbr(p, x, y, z, q)] & F_OBST)) ls[q] += wdrag * R(2 * cx(q));
            }
        }
        if (x == 0 && g_uin) g_uin[(int64_t)z * p.ny + y] += g_in;
        R A = 0, Bx = 0, By = 0, Bz = 0;
        for (int q = 0; q < 19; ++q) {
            const R cu = (R)cx(q) * ux + (R)cy(q) * uy + (R)cz(q) * uz;
            const R w = wR<R>(q);
            A += ls[q] * w * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * uu);
            const R t = ls[q] * w * rho;
            Bx += t * (R(3) * cx(q) + R(9) * cu * cx(q) - R(3) * ux);
            By += t * (R(3) * cy(q) + R(9) * cu * cy(q) - R(3) * uy);
            Bz += t * (R(3) * cz(q) + R(9) * cu * cz(q) - R(3) * uz);
        }
        const R om = p.omega;
        const R vx = ux - p.fx, vy = uy - p.fy, vz = uz - p.fz;
        for (int q = 0; q < 19; ++q) {
            const R du = (Bx * ((R)cx(q) - vx) + By * ((R)cy(q) - vy) + Bz * ((R)cz(q) - vz)) / rho;
            lam0[q * p.N + id] = (R(1) - om) * ls[q] + om * (A + du) + a_in;
        }
    }
}

template <class R>
__global__ void adj_grad_u0(AdjP<R> p, const double* __restrict__ u0, const R* __restrict__ lam, double* __restrict__ g) {
    for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < p.N; id += (int64_t)gridDim.x * blockDim.x) {
        const R ux = (R)u0[id], uy = (R)u0[p.N + id], uz = (R)u0[2 * p.N + id];
        R gx = 0, gy = 0, gz = 0;
        for (int q = 0; q < 19; ++q) {
            const R cu = (R)cx(q) * ux + (R)cy(q) * uy + (R)cz(q) * uz;
            const R t = lam[q * p.N + id] * wR<R>(q);
            gx += t * (R(3) * cx(q) + R(9) * cu * cx(q) - R(3) * ux);
            gy += t * (R(3) * cy(q) + R(9) * cu * cy(q) - R(3) * uy);
            gz += t * (R(3) * cz(q) + R(9) * cu * cz(q) - R(3) * uz);
        }
        g[id] = (double)gx;
        g[p.N + id] = (double)gy;
        g[2 * p.N + id] = (double)gz;
    }
}

int grid_of(int64_t n) {
    const int64_t b = (n + 255) / 256;
    const int64_t cap = (int64_t)num_sms() * 8;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

#define ACK(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            set_error(std::string("lbm_adjoint: ") + #call + ": " + cudaGetErrorString(e_)); \
            return LBM_ERR_CUDA;                                                           \
        }                                                                                  \
    } while (0)

// Device buffers of one run; released by the destructor.
struct AdjBuffers {
    std::vector<void*> ptrs;
    template <class T>
    bool alloc(T** p, size_t n) {
        if (cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)) != cudaSuccess) return false;
        ptrs.push_back(*p);
        return true;
    }
    ~AdjBuffers() {
        for (void* p : ptrs) cudaFree(p);
    }
};

template <class R>
int adjoint_run(const lbm_adj_problem* pr, const uint8_t* flags, const uint32_t* links, const double* h_uin,
                const double* h_u0, double* J, double* h_g_uin, double* h_g_u0, cudaStream_t s) {
    const int64_t N = (int64_t)pr->nx * pr->ny * pr->nz;
    const int64_t NI = (int64_t)pr->ny * pr->nz;
    const int steps = pr->n_steps, K = pr->checkpoint_every;
    const int wb = pr->window_begin, we = pr->window_end;
    const int nwin = we - wb + 1;
    const bool want_grad = h_g_uin || h_g_u0;
    AdjP<R> p{flags, links, pr->nx, pr->ny, pr->nz, N, R(1) / (R)pr->tau, (R)pr->force[0], (R)pr->force[1],
              (R)pr->force[2]};
    const int grid = grid_of(N);
    AdjBuffers B;
    double *d_uin = nullptr, *d_u0 = nullptr, *d_drag = nullptr, *d_guin = nullptr, *d_gu0 = nullptr;
    R *fa = nullptr, *fb = nullptr;
    const int nseg = (steps + K - 1) / K;
    R* ckpt = nullptr;     // f^{kK}, k = 0 .. nseg-1
    R* seg = nullptr;      // f^{sK} .. f^{sK+K-1} of the segment being reversed
    bool ok = B.alloc(&d_uin, NI) && B.alloc(&d_u0, 3 * N) && B.alloc(&d_drag, (size_t)grid * (steps + 1)) &&
              B.alloc(&fa, 19 * N) && B.alloc(&fb, 19 * N);
    if (want_grad)
        ok = ok && B.alloc(&ckpt, (size_t)nseg * 19 * N) && B.alloc(&seg, (size_t)K * 19 * N) &&
             B.alloc(&d_guin, NI) && B.alloc(&d_gu0, 3 * N);
    if (!ok) { set_error("lbm_adjoint: device allocation failed"); return LBM_ERR_ALLOC; }
    ACK(cudaMemcpyAsync(d_uin, h_uin, sizeof(double) * NI, cudaMemcpyHostToDevice, s));
    ACK(cudaMemcpyAsync(d_u0, h_u0, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s));
    adj_init<R><<<grid, 256, 0, s>>>(p, d_u0, fa);
    ACK(cudaGetLastError());
    // forward: f^{n-1} -> f^n, drag of step n in d_drag[n * grid ...]
    for (int n = 1; n <= steps; ++n) {
        if (want_grad && (n - 1) % K == 0)
            ACK(cudaMemcpyAsync(ckpt + (size_t)((n - 1) / K) * 19 * N, fa, sizeof(R) * 19 * N,
                                cudaMemcpyDeviceToDevice, s));
        adj_fwd<R><<<grid, 256, 0, s>>>(p, fa, fb, d_uin, d_drag + (size_t)n * grid);
        ACK(cudaGetLastError());
        std::swap(fa, fb);
    }
    std::vector<double> drag((size_t)grid * (steps + 1));
    ACK(cudaMemcpyAsync(drag.data(), d_drag, sizeof(double) * drag.size(), cudaMemcpyDeviceToHost, s));
    ACK(cudaStreamSynchronize(s));
    double acc = 0.0;
    for (int n = wb; n <= we; ++n)
        for (int b = 0; b < grid; ++b) acc += drag[(size_t)n * grid + b];
    *J = acc / nwin;
    if (!want_grad) return LBM_OK;

    // reverse: lambda^steps = 0; lambda^{n-1} from lambda^n and f^{n-1}
    R* lam1 = fa;
    R* lam0 = fb;
    ACK(cudaMemsetAsync(lam1, 0, sizeof(R) * 19 * N, s));
    ACK(cudaMemsetAsync(d_guin, 0, sizeof(double) * NI, s));
    for (int sgi = nseg - 1; sgi >= 0; --sgi) {
        const int n0 = sgi * K;                          // f^{n0} is the checkpoint
        const int n1 = std::min(steps, n0 + K);          // states f^{n0} .. f^{n1-1} are needed
        ACK(cudaMemcpyAsync(seg, ckpt + (size_t)sgi * 19 * N, sizeof(R) * 19 * N, cudaMemcpyDeviceToDevice, s));
        for (int n = n0 + 1; n < n1; ++n) {
            adj_fwd<R><<<grid, 256, 0, s>>>(p, seg + (size_t)(n - 1 - n0) * 19 * N, seg + (size_t)(n - n0) * 19 * N,
                                            d_uin, d_drag);
            ACK(cudaGetLastError());
        }
        for (int n = n1; n > n0; --n) {
            const R wd = (n >= wb && n <= we) ? R(1) / (R)nwin : R(0);
            adj_bwd<R><<<grid, 256, 0, s>>>(p, seg + (size_t)(n - 1 - n0) * 19 * N, lam1, lam0, d_uin, d_guin, wd);
            ACK(cudaGetLastError());
            std::swap(lam0, lam1);
        }
    }
    adj_grad_u0<R><<<grid, 256, 0, s>>>(p, d_u0, lam1, d_gu0);
    ACK(cudaGetLastError());
    if (h_g_uin) ACK(cudaMemcpyAsync(h_g_uin, d_guin, sizeof(double) * NI, cudaMemcpyDeviceToHost, s));
    if (h_g_u0) ACK(cudaMemcpyAsync(h_g_u0, d_gu0, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, s));
    ACK(cudaStreamSynchronize(s));
    return LBM_OK;
}

}  // namespace

cudaError_t build_duct_flags(const uint8_t* h_mask, int nx, int ny, int nz, uint8_t** d_flags, uint32_t** d_links,
                             cudaStream_t s) {
    const int64_t N = (int64_t)nx * ny * nz;
    uint8_t* mask = nullptr;
    cudaError_t e = cudaMalloc((void**)&mask, (size_t)N);
    if (e == cudaSuccess) e = cudaMalloc((void**)d_flags, (size_t)N);
    if (e == cudaSuccess) e = cudaMalloc((void**)d_links, sizeof(uint32_t) * (size_t)N);
    if (e == cudaSuccess) e = cudaMemcpyAsync(mask, h_mask, (size_t)N, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = launch_build_flags(mask, nullptr, *d_flags, *d_links, nx, ny, nz, 1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(mask);
    return e;
}

}  // namespace lbm

extern "C" int lbm_adjoint_run(const lbm_adj_problem* p, const uint8_t* host_mask, const double* u_inlet,
                               const double* u0, double* objective, double* grad_inlet, double* grad_u0) {
    using lbm::set_error;
    if (!p || !host_mask || !u_inlet || !u0 || !objective) { set_error("lbm_adjoint_run: null argument"); return LBM_ERR_INVALID; }
    if (p->nx < 3 || p->ny < 1 || p->nz < 1 || !(p->tau > 0.5) || p->n_steps < 1 || p->checkpoint_every < 1 ||
        p->window_begin < 1 || p->window_end < p->window_begin || p->window_end > p->n_steps ||
        (p->precision != 0 && p->precision != 1)) {
        set_error("lbm_adjoint_run: bad problem (nx >= 3, tau > 0.5, 1 <= window_begin <= window_end <= n_steps, "
                  "checkpoint_every >= 1, precision 0|1)");
        return LBM_ERR_INVALID;
    }
    if ((int64_t)p->nx * p->ny * p->nz > ((int64_t)1 << 31)) { set_error("lbm_adjoint_run: grid too large"); return LBM_ERR_SIZE; }
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("lbm_adjoint_run: cannot create a stream");
        return LBM_ERR_CUDA;
    }
    uint8_t* flags = nullptr;
    uint32_t* links = nullptr;
    int rc = LBM_OK;
    const cudaError_t e = lbm::build_duct_flags(host_mask, p->nx, p->ny, p->nz, &flags, &links, s);
    if (e != cudaSuccess) {
        set_error(std::string("lbm_adjoint_run: flags: ") + cudaGetErrorString(e));
        rc = LBM_ERR_CUDA;
    } else if (p->precision == 0) {
        rc = lbm::adjoint_run<float>(p, flags, links, u_inlet, u0, objective, grad_inlet, grad_u0, s);
    } else {
        rc = lbm::adjoint_run<double>(p, flags, links, u_inlet, u0, objective, grad_inlet, grad_u0, s);
    }
    cudaStreamSynchronize(s);
    cudaFree(flags);
    cudaFree(links);
    cudaStreamDestroy(s);
    return rc;
}
