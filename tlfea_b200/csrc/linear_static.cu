// linear_static.cu -- LinearStaticSolver<T> (LinearStaticSolver.cu:196-603) on
// sm_100a: deterministic row-wise stiffness assembly into 3x3 node blocks,
// Dirichlet elimination, and an FP64 CG (unpreconditioned like the reference,
// or opt-in block Jacobi) whose dot products are fused into the SpMV / axpy
// kernels and whose scalars never leave the device (CUDA graph of several
// iterations per host check).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "mf_tangent.cuh"
#include "solver.cuh"

namespace tlfea {

// Stiffness, one thread per node row i.  For every incident (element e, slot a)
// in element order and every QP: the SVK tangent blocks K_ab of
// compute_hessian_assemble_csr (FEAT10DataFunc.cuh:512-684; SVK.cuh:41-67) at
// the current positions, scaled by h, plus the Kelvin-Voigt block C_ab
// (:686-768) when damping is set; with MR the Mooney-Rivlin blocks
// sum_JL A[d][J][e][L] gN_aJ gN_bL dV (:607-640).  Block (a,b) is added to row
// i's block for node conn(e,b).  No atomics: each row is owned by one thread.
// K is row-planar: component c of row i's k-th block is K[9*off[i] + c*nb + k].
template <int NPE, int NQP, bool MR>
__global__ void __launch_bounds__(128) k_stiffness_rows(int N, int E, const int* __restrict__ conn,
                                                        const double* __restrict__ x, const double* __restrict__ y,
                                                        const double* __restrict__ z, const int* __restrict__ elem_slot,
                                                        const double* __restrict__ grad64,
                                                        const double* __restrict__ dv64,
                                                        const int* __restrict__ inc_off, const int* __restrict__ inc_e,
                                                        const int* __restrict__ inc_a, const int* __restrict__ off,
                                                        const int* __restrict__ col, double* K, double lambda,
                                                        double mu, double eta_d, double lambda_d, double h,
                                                        double mu10, double mu01, double kappa) {
    constexpr int TE = TILE_ELEMS;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int rb = off[i], re = off[i + 1], nbr = re - rb;
    double* Kr = K + 9LL * rb;
    for (long long k = 0; k < 9LL * nbr; ++k) Kr[k] = 0.0;
    const bool visc = (eta_d != 0.0 || lambda_d != 0.0);
    for (int k = inc_off[i]; k < inc_off[i + 1]; ++k) {
        const int e = inc_e[k], a = inc_a[k];
        const int slot = elem_slot[e];
        const int tile = slot / TE, t = slot % TE;
        int bpos[NPE];
        double X[NPE][3];
        for (int b = 0; b < NPE; ++b) {
            const int nb = conn[e + (size_t)b * E];
            X[b][0] = x[nb];
            X[b][1] = y[nb];
            X[b][2] = z[nb];
            int lo = rb, hi = re - 1, pos = -1;
            while (lo <= hi) {
                const int mid = lo + ((hi - lo) >> 1);
                const int v = col[mid];
                if (v == nb) {
                    pos = mid;
                    break;
                }
                if (v < nb)
                    lo = mid + 1;
                else
                    hi = mid - 1;
            }
            bpos[b] = pos - rb;  // block index within the row (pattern holds every pair)
        }
        for (int q = 0; q < NQP; ++q) {
            const double* gp = grad64 + ((size_t)tile * NQP + q) * (NPE * 3) * TE + t;
            double g[NPE][3];
            for (int b = 0; b < NPE; ++b)
                for (int j = 0; j < 3; ++j) g[b][j] = gp[(size_t)(b * 3 + j) * TE];
            const double dV = dv64[((size_t)tile * NQP + q) * TE + t];
            double F[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int b = 0; b < NPE; ++b)
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) F[r][c] += X[b][r] * g[b][c];
            double C[3][3], FFT[3][3];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) {
                    double s = 0.0, s2 = 0.0;
                    for (int kk = 0; kk < 3; ++kk) {
                        s += F[kk][r] * F[kk][c];
                        s2 += F[r][kk] * F[c][kk];
                    }
                    C[r][c] = s;
                    FFT[r][c] = s2;
                }
            const double trE = 0.5 * ((C[0][0] + C[1][1] + C[2][2]) - 3.0);
            double Fha[3];
            for (int r = 0; r < 3; ++r) {
                double s = 0.0;
                for (int c = 0; c < 3; ++c) s += F[r][c] * g[a][c];
                Fha[r] = s;
            }
            double Bmr[3][3][3];
            if constexpr (MR) mooney_rivlin_tangent_a(F, mu10, mu01, kappa, g[a], Bmr);
            for (int b = 0; b < NPE; ++b) {
                if (bpos[b] < 0) continue;
                double Fhb[3];
                for (int r = 0; r < 3; ++r) {
                    double s = 0.0;
                    for (int c = 0; c < 3; ++c) s += F[r][c] * g[b][c];
                    Fhb[r] = s;
                }
                const double hij = g[b][0] * g[a][0] + g[b][1] * g[a][1] + g[b][2] * g[a][2];
                const double fdf = Fhb[0] * Fha[0] + Fhb[1] * Fha[1] + Fhb[2] * Fha[2];
                double* Kb = Kr + bpos[b];
                for (int d = 0; d < 3; ++d)
                    for (int ee = 0; ee < 3; ++ee) {
                        if constexpr (MR) {
                            const double kb = Bmr[d][ee][0] * g[b][0] + Bmr[d][ee][1] * g[b][1] + Bmr[d][ee][2] * g[b][2];
                            Kb[(size_t)(3 * d + ee) * nbr] += h * (kb * dV);
                            continue;
                        }
                        const double delta = (d == ee) ? 1.0 : 0.0;
                        const double kv = (lambda * Fha[d] * Fhb[ee] + lambda * trE * hij * delta + mu * fdf * delta +
                                           mu * Fhb[d] * Fha[ee] + mu * hij * FFT[d][ee] + (-mu * hij * delta)) *
                                          dV;
                        Kb[(size_t)(3 * d + ee) * nbr] += h * kv;
                    }
                if (visc) {
                    const double hd = g[a][0] * g[b][0] + g[a][1] * g[b][1] + g[a][2] * g[b][2];
                    for (int d = 0; d < 3; ++d)
                        for (int ee = 0; ee < 3; ++ee)
                            Kb[(size_t)(3 * d + ee) * nbr] += (eta_d * (Fhb[d] * Fha[ee]) + eta_d * FFT[d][ee] * hd +
                                               lambda_d * (Fha[d] * Fhb[ee])) *
                                              dV;
                }
            }
        }
    }
}

// Dirichlet elimination (apply_bcs_kernel, LinearStaticSolver.cu:284-306): a
// fixed row becomes the identity row with f = 0; free rows drop fixed columns.
__global__ void k_apply_bcs(int N, const int* __restrict__ off, const int* __restrict__ col,
                            const unsigned char* __restrict__ fixed, double* K, double* f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int rb = off[i], nbr = off[i + 1] - rb;
    double* Kr = K + 9LL * rb;
    for (int k = 0; k < nbr; ++k) {
        const int cn = col[rb + k];
        for (int d = 0; d < 3; ++d) {
            const int row = 3 * i + d;
            for (int e = 0; e < 3; ++e) {
                const int c = 3 * cn + e;
                if (fixed[row])
                    Kr[(size_t)(3 * d + e) * nbr + k] = (c == row) ? 1.0 : 0.0;
                else if (fixed[c])
                    Kr[(size_t)(3 * d + e) * nbr + k] = 0.0;
            }
        }
    }
    for (int d = 0; d < 3; ++d)
        if (fixed[3 * i + d]) f[3 * i + d] = 0.0;
}

__global__ void k_zero_fixed(int n3, const unsigned char* __restrict__ fixed, double* f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n3 && fixed[i]) f[i] = 0.0;
}

__global__ void k_mark_fixed(int nf, const int* __restrict__ nodes, unsigned char* fixed) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf) return;
    const int n = nodes[k];
    fixed[3 * n + 0] = fixed[3 * n + 1] = fixed[3 * n + 2] = 1;
}

__global__ void k_update_positions(int n, double* x, double* y, double* z, const double* __restrict__ u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] += u[3 * i + 0];
    y[i] += u[3 * i + 1];
    z[i] += u[3 * i + 2];
}

// Last-block-done reduction of per-block partials in block order (deterministic
// for a fixed grid).  Returns true in the last block, with the total in `out`
// (valid in thread 0).
__device__ __forceinline__ bool last_block_sum(double part, double* partials, unsigned int* ticket, double* out) {
    __shared__ double red[32];
    __shared__ bool am_last;
    const double bs = block_sum(part, red);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = bs;
        __threadfence();
        const unsigned int tk = atomicAdd(ticket, 1u);
        am_last = (tk == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s += __ldcg(partials + b);
    s = block_sum(s, red);
    if (threadIdx.x == 0) {
        *out = s;
        *ticket = 0;
    }
    return true;
}

// u = 0, r = p = f, rr0 = r.r
__global__ void k_cg_init(int n, const double* __restrict__ f, double* u, double* r, double* p, double* partials,
                          CgCtl* ctl, int max_iter) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double fi = f[i];
        u[i] = 0.0;
        r[i] = fi;
        p[i] = fi;
        s += fi * fi;
    }
    double tot;
    if (last_block_sum(s, partials, &ctl->ticket, &tot) && threadIdx.x == 0) {
        ctl->rr0 = tot;
        ctl->rr = tot;
        ctl->iters = 0;
        ctl->status = 0;
        ctl->rel = 1.0;
        ctl->done = 0;
        if (tot == 0.0) {
            ctl->done = 1;
            ctl->rel = 0.0;
        } else if (max_iter <= 0) {
            ctl->done = 1;
            ctl->status = 2;
        }
    }
}

// q = K p on 3x3 node blocks fused with the p.q reduction; the last block sets
// alpha = rr / p.q (LinearStaticSolver.cu:519-533).  K is stored row-planar:
// node row i owns K[9*rb, 9*(rb+nb)) and component c = 3d+e of its k-th block
// sits at K[9*rb + c*nb + k].  One warp per node row, one lane per block: the
// nine component loads of a lane are coalesced across the warp, independent
// of each other and of the column-index load, and the component index is a
// compile-time constant.  The next row's extent and first 32 column indices
// are fetched while the current row is in flight, so the gather of p does not
// wait behind a load of its own row's indices.
__device__ __forceinline__ void spmv_block(const double* Kr, int nb, int k, int cj, const double* __restrict__ p,
                                           double& a0, double& a1, double& a2) {
    const double* kv = Kr + k;
    double v[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) v[c] = __ldcs(kv + (size_t)c * nb);
    const double p0 = p[3 * cj + 0], p1 = p[3 * cj + 1], p2 = p[3 * cj + 2];
    a0 += v[0] * p0 + v[1] * p1 + v[2] * p2;
    a1 += v[3] * p0 + v[4] * p1 + v[5] * p2;
    a2 += v[6] * p0 + v[7] * p1 + v[8] * p2;
}

__global__ void __launch_bounds__(256) k_cg_spmv_dot(int N, const int* __restrict__ off, const int* __restrict__ col,
                                                     const double* __restrict__ K, const double* __restrict__ p,
                                                     double* q, double* partials, CgCtl* ctl) {
    if (ctl->done) return;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    double pq = 0.0;
    int rb = 0, nb = 0, cj = 0;
    if (warp < N) {
        rb = off[warp];
        nb = off[warp + 1] - rb;
        cj = (lane < nb) ? col[rb + lane] : 0;
    }
    for (int i = warp; i < N; i += nwarps) {
        const int in = i + nwarps;
        int rbn = 0, nbn = 0;
        if (in < N) {
            rbn = off[in];
            nbn = off[in + 1] - rbn;
        }
        const double* Kr = K + 9LL * rb;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        if (lane < nb) spmv_block(Kr, nb, lane, cj, p, a0, a1, a2);
        for (int k = lane + 32; k < nb; k += 32) spmv_block(Kr, nb, k, col[rb + k], p, a0, a1, a2);
        const int cjn = (lane < nbn) ? col[rbn + lane] : 0;
        a0 = warp_sum(a0);
        a1 = warp_sum(a1);
        a2 = warp_sum(a2);
        if (lane == 0) {
            q[3 * i + 0] = a0;
            q[3 * i + 1] = a1;
            q[3 * i + 2] = a2;
            pq += p[3 * i + 0] * a0 + p[3 * i + 1] * a1 + p[3 * i + 2] * a2;
        }
        rb = rbn;
        nb = nbn;
        cj = cjn;
    }
    double tot;
    if (last_block_sum(pq, partials, &ctl->ticket, &tot) && threadIdx.x == 0) {
        ctl->pq = tot;
        if (tot <= 0.0) {
            ctl->status = 1;
            ctl->done = 1;
        } else {
            ctl->alpha = ctl->rr / tot;
        }
    }
}

// u += alpha p; r -= alpha q; rr_new = r.r; convergence test sqrt(rr_new/rr0) < tol;
// beta = rr_new / rr (LinearStaticSolver.cu:534-557).
__global__ void k_cg_axpy_dot(int n, double* u, double* r, const double* __restrict__ p, const double* __restrict__ q,
                              double* partials, CgCtl* ctl, double tol, int max_iter) {
    if (ctl->done) return;
    const double alpha = ctl->alpha;
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        u[i] += alpha * p[i];
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        s += ri * ri;
    }
    double rrn;
    if (last_block_sum(s, partials, &ctl->ticket, &rrn) && threadIdx.x == 0) {
        const double rel = (ctl->rr0 > 0.0) ? sqrt(rrn / ctl->rr0) : sqrt(rrn);
        ctl->iters += 1;
        if (rel < tol) {
            ctl->rel = rel;
            ctl->done = 1;
        } else {
            ctl->beta = rrn / ctl->rr;
            ctl->rr = rrn;
            if (ctl->iters >= max_iter) {
                ctl->rel = rel;
                ctl->status = 2;
                ctl->done = 1;
            }
        }
    }
}

// p = r + beta p  (cublasDscal + cublasDaxpy of LinearStaticSolver.cu:554-555)
__global__ void k_cg_pupdate(int n, const double* __restrict__ r, double* p, const CgCtl* ctl) {
    if (ctl->done) return;
    const double beta = ctl->beta;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = r[i] + beta * p[i];
}

// ---- block-Jacobi preconditioned CG (opt-in; new, no reference counterpart).
// D = the 3x3 diagonal node blocks of K (BCs applied: a fixed DOF's row and
// column are the identity's), inverted once per solve; z = D^-1 r.  The
// stop test stays sqrt(r.r / r0.r0) < tol; alpha = r.z / p.Kp, beta = r.z_new / r.z.

__global__ void k_block_jacobi(int N, const int* __restrict__ off, const int* __restrict__ col,
                               const double* __restrict__ K, double* dinv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int rb = off[i], nb = off[i + 1] - rb;
    int kd = 0;
    for (int k = 0; k < nb; ++k)
        if (col[rb + k] == i) kd = k;
    double a[9];
    for (int c = 0; c < 9; ++c) a[c] = K[9LL * rb + (size_t)c * nb + kd];
    // inverse by cofactors (the block is symmetric positive definite)
    const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    const double id = (det != 0.0) ? 1.0 / det : 0.0;
    double* d = dinv + 9LL * i;
    d[0] = c00 * id;
    d[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    d[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    d[3] = c01 * id;
    d[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    d[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    d[6] = c02 * id;
    d[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    d[8] = (a[0] * a[4] - a[1] * a[3]) * id;
}

// Two last-block-done sums in one pass (partials hold 2 * gridDim.x values).
__device__ __forceinline__ bool last_block_sum2(double a, double b, double* partials, unsigned int* ticket, double* oa,
                                                double* ob) {
    __shared__ double red[32];
    __shared__ bool am_last;
    const double sa = block_sum(a, red);
    const double sb = block_sum(b, red);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = sa;
        partials[gridDim.x + blockIdx.x] = sb;
        __threadfence();
        am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double ta = 0.0, tb = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
        ta += __ldcg(partials + k);
        tb += __ldcg(partials + gridDim.x + k);
    }
    ta = block_sum(ta, red);
    tb = block_sum(tb, red);
    if (threadIdx.x == 0) {
        *oa = ta;
        *ob = tb;
        *ticket = 0;
    }
    return true;
}

__device__ __forceinline__ void apply_dinv(const double* __restrict__ d, const double r[3], double z[3]) {
    z[0] = d[0] * r[0] + d[1] * r[1] + d[2] * r[2];
    z[1] = d[3] * r[0] + d[4] * r[1] + d[5] * r[2];
    z[2] = d[6] * r[0] + d[7] * r[1] + d[8] * r[2];
}

// u = 0, r = f, z = D^-1 f, p = z; rres = r.r (= r0.r0), rr = r.z
__global__ void k_pcg_init(int N, const double* __restrict__ f, const double* __restrict__ dinv, double* u, double* r,
                           double* z, double* p, double* partials, CgCtl* ctl, int max_iter) {
    double srr = 0.0, srz = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        double ri[3], zi[3];
        for (int d = 0; d < 3; ++d) ri[d] = f[3 * i + d];
        apply_dinv(dinv + 9LL * i, ri, zi);
        for (int d = 0; d < 3; ++d) {
            u[3 * i + d] = 0.0;
            r[3 * i + d] = ri[d];
            z[3 * i + d] = zi[d];
            p[3 * i + d] = zi[d];
            srr += ri[d] * ri[d];
            srz += ri[d] * zi[d];
        }
    }
    double trr, trz;
    if (last_block_sum2(srr, srz, partials, &ctl->ticket, &trr, &trz) && threadIdx.x == 0) {
        ctl->rr0 = trr;
        ctl->rres = trr;
        ctl->rr = trz;
        ctl->iters = 0;
        ctl->status = 0;
        ctl->rel = 1.0;
        ctl->done = 0;
        if (trr == 0.0) {
            ctl->done = 1;
            ctl->rel = 0.0;
        } else if (max_iter <= 0) {
            ctl->done = 1;
            ctl->status = 2;
        }
    }
}

// u += alpha p; r -= alpha q; z = D^-1 r; r.r for the stop test, r.z for beta.
__global__ void k_pcg_axpy_dot(int N, const double* __restrict__ dinv, double* u, double* r, double* z,
                               const double* __restrict__ p, const double* __restrict__ q, double* partials,
                               CgCtl* ctl, double tol, int max_iter) {
    if (ctl->done) return;
    const double alpha = ctl->alpha;
    double srr = 0.0, srz = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        double ri[3], zi[3];
        for (int d = 0; d < 3; ++d) {
            u[3 * i + d] += alpha * p[3 * i + d];
            ri[d] = r[3 * i + d] - alpha * q[3 * i + d];
            r[3 * i + d] = ri[d];
        }
        apply_dinv(dinv + 9LL * i, ri, zi);
        for (int d = 0; d < 3; ++d) {
            z[3 * i + d] = zi[d];
            srr += ri[d] * ri[d];
            srz += ri[d] * zi[d];
        }
    }
    double trr, trz;
    if (last_block_sum2(srr, srz, partials, &ctl->ticket, &trr, &trz) && threadIdx.x == 0) {
        const double rel = (ctl->rr0 > 0.0) ? sqrt(trr / ctl->rr0) : sqrt(trr);
        ctl->iters += 1;
        ctl->rres = trr;
        if (rel < tol) {
            ctl->rel = rel;
            ctl->done = 1;
        } else {
            ctl->beta = trz / ctl->rr;
            ctl->rr = trz;
            if (ctl->iters >= max_iter) {
                ctl->rel = rel;
                ctl->status = 2;
                ctl->done = 1;
            }
        }
    }
}

static int cg_grid(const tlfea_solver_s* s) { return s->cg_blocks; }

// The matrix-free product where it applies -- SVK without damping, no preconditioner,
// TET10 -- and, by default, where it pays: with the earlier per-node-gradient product the
// assembled SpMV measured faster on TET4 (few QPs, small K blocks: 7.5 against 5.7
// solves/s at 200x20x20) and on meshes of a few thousand elements (17.4 against 12.7
// solves/s on the 512-instance batch's single-instance solves); from about 10^5 elements
// the product wins (now 0.75 against 0.40 solves/s at 480,000 elements).
constexpr int MF_MIN_ELEMENTS = 100000;

static bool use_matrix_free(const tlfea_solver_s* s) {
    const tlfea_element_s* el = s->el;
    const bool applies = s->precond == 0 && el->npe == 10 && el->material != TLFEA_MATERIAL_MOONEY_RIVLIN &&
                         el->eta_d == 0.0 && el->lambda_d == 0.0;
    if (!applies || s->op_mode == 1) return false;
    return s->op_mode == 2 || el->E >= MF_MIN_ELEMENTS;
}

static MfArgs mf_args(tlfea_solver_s* s, const double* p, double* q, CgCtl* ctl) {
    tlfea_element_s* el = s->el;
    const Tiling& tl = el->tl;
    MfArgs M;
    memset(&M, 0, sizeof(M));
    M.n_tiles = tl.n_tiles;
    M.max_local = tl.max_local_pad;
    M.node_off = tl.node_off;
    M.pad_off = tl.pad_off;
    M.pad_gid = tl.pad_gid;
    M.pad_dst = tl.pad_dst;
    M.pad_iend = tl.pad_iend;
    M.inc = tl.inc;
    M.lconn = tl.lconn;
    M.ji = tl.ji64;
    M.dv = tl.dv64;
    M.tan = s->mf_tan;
    M.x = s->xk;  // the last solve's positions
    M.y = s->yk;
    M.z = s->zk;
    M.p = p;
    M.q = q;
    M.partial = tl.partial64;
    M.is_fixed = s->is_fixed;
    M.prec = s->mf_prec;
    M.pfix = s->mf_pfix;
    M.tile_dot = s->mf_part;
    M.lambda = el->lambda;
    M.mu = el->mu;
    M.qb = qp_bary(el);
    M.ctl = ctl;
    return M;
}

// The matrix-free product's tile kernel and its shared memory (TET10: use_matrix_free
// admits no other element type).
using MfKernel = void (*)(MfArgs, int*);
static MfKernel mf_kernel(const tlfea_solver_s*) { return k_mf_geo<10, 5>; }

static size_t mf_smem(const tlfea_solver_s* s) { return MfLayout<10>(s->el->tl.max_local_pad).total; }

// q = K_bc p matrix-free and p.q, alpha (the SpMV kernel's contract).
static int launch_mf_apply(tlfea_solver_s* s, cudaStream_t st, const double* p, double* q, CgCtl* ctl) {
    tlfea_element_s* el = s->el;
    const MfArgs M = mf_args(s, p, q, ctl);
    const size_t smem = mf_smem(s);
    const long long n_pad = el->tl.n_pad;
    const long long per_block = 256LL * MF_GATHER_ILP;
    k_mf_gather<<<(unsigned)((n_pad + per_block - 1) / per_block), 256, 0, st>>>(n_pad, el->tl.pad_gid, s->mf_pfix, p,
                                                                                s->mf_prec, ctl);
    if (cudaGetLastError() != cudaSuccess) return TLFEA_CUDA_ERROR;
    // the tile kernel and the combine are programmatic dependents: each starts while its
    // predecessor drains and waits (griddepcontrol.wait) before reading its results
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t tcfg = {};
    tcfg.gridDim = dim3((unsigned)el->tl.n_tiles);
    tcfg.blockDim = dim3(TILE_ELEMS);
    tcfg.dynamicSmemBytes = smem;
    tcfg.stream = st;
    tcfg.attrs = attr;
    tcfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&tcfg, mf_kernel(s), M, el->d_err) != cudaSuccess) return TLFEA_CUDA_ERROR;
    const int nb = el->tl.n_bnodes;
    const int cb = std::max(1, (nb + 255) / 256);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cb);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, k_mf_combine_dot, nb, (const int*)el->tl.bnode_gid, (const int*)el->tl.bnode_off, M,
                           s->mf_part + el->tl.n_tiles) != cudaSuccess)
        return TLFEA_CUDA_ERROR;
    return TLFEA_OK;
}

static int launch_cg_iteration(tlfea_solver_s* s, cudaStream_t st) {
    tlfea_element_s* el = s->el;
    const int n = 3 * el->N;
    const int G = cg_grid(s);
    if (use_matrix_free(s)) {
        if (launch_mf_apply(s, st, s->p, s->q, s->ctl)) return TLFEA_CUDA_ERROR;
        k_cg_axpy_dot<<<G, 256, 0, st>>>(n, s->u, s->r, s->p, s->q, s->cg_part, s->ctl, s->tol, s->max_iter);
        if (cudaGetLastError() != cudaSuccess) return TLFEA_CUDA_ERROR;
        k_cg_pupdate<<<G, 256, 0, st>>>(n, s->r, s->p, s->ctl);
        if (cudaGetLastError() != cudaSuccess) return TLFEA_CUDA_ERROR;
        return TLFEA_OK;
    }
    k_cg_spmv_dot<<<G, 256, 0, st>>>(el->N, el->pat_off, el->pat_col, s->K, s->p, s->q, s->cg_part, s->ctl);
    if (cudaGetLastError() != cudaSuccess) return TLFEA_CUDA_ERROR;
    if (s->precond) {
        k_pcg_axpy_dot<<<G, 256, 0, st>>>(el->N, s->dinv, s->u, s->r, s->z, s->p, s->q, s->cg_part, s->ctl, s->tol,
                                          s->max_iter);
        if (cudaGetLastError() != cudaSuccess) return TLFEA_CUDA_ERROR;
        k_cg_pupdate<<<G, 256, 0, st>>>(n, s->z, s->p, s->ctl);  // p = z + beta p
        if (cudaGetLastError() != cudaSuccess) return TLFEA_CUDA_ERROR;
        return TLFEA_OK;
    }
    k_cg_axpy_dot<<<G, 256, 0, st>>>(n, s->u, s->r, s->p, s->q, s->cg_part, s->ctl, s->tol, s->max_iter);
    if (cudaGetLastError() != cudaSuccess) return TLFEA_CUDA_ERROR;
    k_cg_pupdate<<<G, 256, 0, st>>>(n, s->r, s->p, s->ctl);
    if (cudaGetLastError() != cudaSuccess) return TLFEA_CUDA_ERROR;
    return TLFEA_OK;
}

// Captures `iters` CG iterations (3 kernels each) in one CUDA graph.
static int build_cg_graph(tlfea_solver_s* s, int iters) {
    cudaStream_t st = s->el->stream;
    if (s->cg_graph) {
        cudaGraphExecDestroy(s->cg_graph);
        s->cg_graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    TLFEA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = TLFEA_OK;
    for (int k = 0; k < iters && rc == TLFEA_OK; ++k) rc = launch_cg_iteration(s, st);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != TLFEA_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        set_error("CG graph capture failed");
        return TLFEA_CUDA_ERROR;
    }
    e = cudaGraphInstantiate(&s->cg_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        set_error(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
        s->cg_graph = nullptr;
        return TLFEA_CUDA_ERROR;
    }
    s->cg_graph_iters = iters;
    s->cg_graph_precond = s->precond;
    s->cg_graph_mf = use_matrix_free(s) ? 1 : 0;
    return TLFEA_OK;
}

int linear_static_prepare(tlfea_solver_s* s) {
    tlfea_element_s* el = s->el;
    int st = element_build_pattern(el);
    if (st) return st;
    if (!s->K) {
        const size_t n3 = 3 * (size_t)el->N;
        if ((st = dalloc(&s->K, 9 * (size_t)std::max(el->pat_nnz, 1LL)))) return st;
        if ((st = dalloc(&s->u, n3)) || (st = dalloc(&s->f, n3)) || (st = dalloc(&s->r, n3)) ||
            (st = dalloc(&s->p, n3)) || (st = dalloc(&s->q, n3)))
            return st;
        if ((st = dalloc(&s->is_fixed, n3))) return st;
        if ((st = dalloc(&s->ctl, 1))) return st;
        TLFEA_CUDA(cudaMemset(s->ctl, 0, sizeof(CgCtl)));
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        // persistent grid: every CG kernel strides over rows/DOFs with all resident blocks
        int per_sm = 0;
        TLFEA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg_spmv_dot, 256, 0));
        const int rows_warps = (el->N + 7) / 8;
        s->cg_blocks = std::max(1, std::min(rows_warps, std::max(per_sm, 1) * sms));
        if ((st = dalloc(&s->cg_part, 2 * (size_t)s->cg_blocks))) return st;
    }
    return TLFEA_OK;
}

// AssembleLinearStiffness (h = 1) at the given positions, then ApplyDirichletBCs to K
// and f (is_fixed already marked).
static int assemble_k(tlfea_solver_s* s, const double* x, const double* y, const double* z) {
    tlfea_element_s* el = s->el;
    cudaStream_t stream = el->stream;
    const int N = el->N;
    const bool mr = (el->material == TLFEA_MATERIAL_MOONEY_RIVLIN);
    auto kern = (el->npe == 10) ? (mr ? k_stiffness_rows<10, 5, true> : k_stiffness_rows<10, 5, false>)
                                : (mr ? k_stiffness_rows<4, 1, true> : k_stiffness_rows<4, 1, false>);
    kern<<<(N + 127) / 128, 128, 0, stream>>>(N, el->E, el->d_conn, x, y, z, el->tl.elem_slot, el->tl.grad64,
                                               el->tl.dv64, el->inc_off, el->inc_e, el->inc_a, el->pat_off,
                                               el->pat_col, s->K, el->lambda, el->mu, el->eta_d, el->lambda_d, 1.0,
                                               el->mu10, el->mu01, el->kappa);
    TLFEA_CHECK_LAUNCH();
    if (el->n_constraint > 0) {
        k_apply_bcs<<<(N + 255) / 256, 256, 0, stream>>>(N, el->pat_off, el->pat_col, s->is_fixed, s->K, s->f);
        TLFEA_CHECK_LAUNCH();
    }
    s->k_built = true;
    return TLFEA_OK;
}

int linear_static_solve(tlfea_solver_s* s) {
    tlfea_element_s* el = s->el;
    if (!el->is_setup) {
        set_error("element must be set up first");
        return TLFEA_NOT_SETUP;
    }
    int st = linear_static_prepare(s);
    if (st) return st;
    cudaStream_t stream = el->stream;
    const int N = el->N, n3 = 3 * N;
    // the right-hand side and the Dirichlet DOFs
    TLFEA_CUDA(cudaMemcpyAsync(s->f, el->f_ext, sizeof(double) * n3, cudaMemcpyDeviceToDevice, stream));
    TLFEA_CUDA(cudaMemsetAsync(s->is_fixed, 0, n3, stream));
    const int nf = el->n_constraint / 3;
    if (nf > 0) {
        k_mark_fixed<<<(nf + 255) / 256, 256, 0, stream>>>(nf, el->fixed, s->is_fixed);
        TLFEA_CHECK_LAUNCH();
    }
    const bool mf = use_matrix_free(s);
    if (mf) {
        // matrix-free K p at these positions: keep a copy (the products' tangent stream is
        // formed from it, and K can still be assembled at them after the update)
        k_zero_fixed<<<(n3 + 255) / 256, 256, 0, stream>>>(n3, s->is_fixed, s->f);
        TLFEA_CHECK_LAUNCH();
        if (!s->xk && ((st = dalloc(&s->xk, (size_t)N)) || (st = dalloc(&s->yk, (size_t)N)) ||
                       (st = dalloc(&s->zk, (size_t)N))))
            return st;
        TLFEA_CUDA(cudaMemcpyAsync(s->xk, el->x, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream));
        TLFEA_CUDA(cudaMemcpyAsync(s->yk, el->y, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream));
        TLFEA_CUDA(cudaMemcpyAsync(s->zk, el->z, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream));
        TLFEA_CUDA(cudaMemsetAsync(s->q, 0, sizeof(double) * n3, stream));  // nodes of no element stay 0
        const size_t need = (size_t)el->tl.n_tiles + std::max(1, (el->tl.n_bnodes + 255) / 256);
        if (!s->mf_part && (st = dalloc(&s->mf_part, need))) return st;
        const long long n_pad = el->tl.n_pad;
        if (!s->mf_prec && ((st = dalloc(&s->mf_prec, 3 * (size_t)n_pad)) || (st = dalloc(&s->mf_pfix, (size_t)n_pad))))
            return st;
        k_mf_fixbits<<<(unsigned)((n_pad + 255) / 256), 256, 0, stream>>>(n_pad, el->tl.pad_gid, s->is_fixed,
                                                                           s->mf_pfix);
        TLFEA_CHECK_LAUNCH();
        // F and S at every element QP, once for the whole solve
        const size_t ntan = (size_t)el->tl.n_tiles * el->nqp * MF_TAN * TILE_ELEMS;
        if (!s->mf_tan && (st = dalloc(&s->mf_tan, ntan))) return st;
        {
            const MfArgs M = mf_args(s, s->p, s->q, s->ctl);
            k_mf_prep<10, 5><<<el->tl.n_tiles, TILE_ELEMS, 0, stream>>>(M);
            TLFEA_CHECK_LAUNCH();
        }
        const size_t smem = mf_smem(s);
        if (smem > 227 * 1024) {
            set_error("matrix-free stiffness: shared memory exceeds 227 KB (tile touches too many nodes)");
            return TLFEA_UNSUPPORTED;
        }
        if (smem > 48 * 1024)
            TLFEA_CUDA(cudaFuncSetAttribute((const void*)mf_kernel(s), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem));
        s->k_built = false;
        s->mf_last = true;
    } else {
        if ((st = assemble_k(s, el->x, el->y, el->z))) return st;
        s->mf_last = false;
    }
    // SolveLinearSystemCG
    const int G = cg_grid(s);
    if (s->precond) {
        if (!s->dinv && ((st = dalloc(&s->dinv, 9 * (size_t)N)) || (st = dalloc(&s->z, (size_t)n3)))) return st;
        k_block_jacobi<<<(N + 255) / 256, 256, 0, stream>>>(N, el->pat_off, el->pat_col, s->K, s->dinv);
        TLFEA_CHECK_LAUNCH();
        k_pcg_init<<<G, 256, 0, stream>>>(N, s->f, s->dinv, s->u, s->r, s->z, s->p, s->cg_part, s->ctl, s->max_iter);
    } else {
        k_cg_init<<<G, 256, 0, stream>>>(n3, s->f, s->u, s->r, s->p, s->cg_part, s->ctl, s->max_iter);
    }
    TLFEA_CHECK_LAUNCH();
    int chunk = 8;
    long long launched = 0;
    CgCtl h{};
    for (;;) {
        TLFEA_CUDA(cudaMemcpyAsync(&h, s->ctl, sizeof(CgCtl), cudaMemcpyDeviceToHost, stream));
        TLFEA_CUDA(cudaStreamSynchronize(stream));
        if (h.done || launched >= s->max_iter) break;
        if (!s->cg_graph || s->cg_graph_iters != chunk || s->cg_graph_precond != s->precond ||
            s->cg_graph_mf != (mf ? 1 : 0)) {
            if ((st = build_cg_graph(s, chunk))) return st;
        }
        TLFEA_CUDA(cudaGraphLaunch(s->cg_graph, stream));
        TLFEA_LAUNCHED((mf ? 5LL : 3LL) * chunk);  // matrix-free: gather, tiles, combine, axpy, direction
        launched += chunk;
        if (chunk < 64) chunk *= 2;
    }
    if (h.status == 1) set_error("LinearStaticSolver CG: non-positive p*Kp detected; aborting.");
    if (h.status == 1) {
        // the reference leaves last_iter_count = max_iter and residual = 1 on breakdown
        s->last_iters = s->max_iter;
        s->last_res = 1.0;
    } else {
        s->last_iters = h.iters;
        s->last_res = h.rel;
    }
    // UpdatePositions
    k_update_positions<<<(N + 255) / 256, 256, 0, stream>>>(N, el->x, el->y, el->z, s->u);
    positions_changed(el);
    TLFEA_CHECK_LAUNCH();
    TLFEA_CUDA(cudaStreamSynchronize(stream));
    return TLFEA_OK;
}

int linear_static_apply(tlfea_solver_s* s, const double* d_x, double* d_y) {
    tlfea_element_s* el = s->el;
    if (!s->k_built && !s->mf_last) {
        set_error("LinearStaticSolver::Solve has not assembled K yet");
        return TLFEA_NOT_SETUP;
    }
    if (!s->ctl_apply) {
        int st = dalloc(&s->ctl_apply, 1);
        if (st) return st;
        TLFEA_CUDA(cudaMemsetAsync(s->ctl_apply, 0, sizeof(CgCtl), el->stream));
    }
    if (s->mf_last) {
        // matrix-free, at the positions of the last solve (its tangent stream); the
        // product's kernels skip their work once the control block reads done
        // (a p.q <= 0 would set it): start every product from a clear block
        TLFEA_CUDA(cudaMemsetAsync(s->ctl_apply, 0, sizeof(CgCtl), el->stream));
        if (launch_mf_apply(s, el->stream, d_x, d_y, s->ctl_apply)) return TLFEA_CUDA_ERROR;
        TLFEA_LAUNCHED(3);
        if (el->blocking) TLFEA_CUDA(cudaStreamSynchronize(el->stream));
        return TLFEA_OK;
    }
    k_cg_spmv_dot<<<cg_grid(s), 256, 0, el->stream>>>(el->N, el->pat_off, el->pat_col, s->K, d_x, d_y, s->cg_part,
                                                      s->ctl_apply);
    TLFEA_CHECK_LAUNCH();
    if (el->blocking) TLFEA_CUDA(cudaStreamSynchronize(el->stream));
    return TLFEA_OK;
}

int linear_static_retrieve_k(tlfea_solver_s* s, long long* nnz, int* offsets, int* columns, double* values) {
    tlfea_element_s* el = s->el;
    TLFEA_CUDA(cudaStreamSynchronize(el->stream));
    if (!s->k_built && s->mf_last) {
        // the last solve ran matrix-free: assemble K at its positions now
        int st = assemble_k(s, s->xk, s->yk, s->zk);
        if (st) return st;
        TLFEA_CUDA(cudaStreamSynchronize(el->stream));
    }
    if (!s->k_built) {
        if (nnz) *nnz = 0;
        return TLFEA_OK;
    }
    const int N = el->N;
    const long long nb = el->pat_nnz;
    if (nnz) *nnz = 9 * nb;
    if (!offsets && !columns && !values) return TLFEA_OK;
    std::vector<double> Kh((size_t)(9 * nb));
    TLFEA_CUDA(cudaMemcpy(Kh.data(), s->K, sizeof(double) * Kh.size(), cudaMemcpyDeviceToHost));
    const std::vector<int>& off = el->h_pat_off;
    const std::vector<int>& col = el->h_pat_col;
    // Full 3N x 3N CSR: entry (3i+d, 3j+e) is component 3d+e of row i's block for j.
    long long o = 0;
    for (int i = 0; i < N; ++i) {
        const int rb = off[i], nbr = off[i + 1] - rb;
        for (int d = 0; d < 3; ++d) {
            if (offsets) offsets[3 * i + d] = (int)o;
            for (int k = 0; k < nbr; ++k)
                for (int e = 0; e < 3; ++e) {
                    if (columns) columns[o] = 3 * col[rb + k] + e;
                    if (values) values[o] = Kh[9 * (size_t)rb + (size_t)(3 * d + e) * nbr + k];
                    ++o;
                }
        }
    }
    if (offsets) offsets[3 * N] = (int)o;
    return TLFEA_OK;
}

void linear_static_free(tlfea_solver_s* s) {
    if (s->cg_graph) cudaGraphExecDestroy(s->cg_graph);
    s->cg_graph = nullptr;
    dfree(s->K);
    dfree(s->u);
    dfree(s->f);
    dfree(s->r);
    dfree(s->p);
    dfree(s->q);
    dfree(s->is_fixed);
    dfree(s->ctl);
    dfree(s->ctl_apply);
    dfree(s->cg_part);
    dfree(s->dinv);
    dfree(s->z);
    dfree(s->mf_part);
    dfree(s->mf_prec);
    dfree(s->mf_tan);
    dfree(s->mf_pfix);
    dfree(s->xk);
    dfree(s->yk);
    dfree(s->zk);
}

}  // namespace tlfea
