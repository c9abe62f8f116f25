// dynamics.cu -- implicit time steps for a batch of sequences on one mesh, each step
// solved by the SyncedNesterov iteration (new: e.g. 64 load sequences on the 100x10x10
// TET10 cantilever advanced together).
//
// B sequences share one element object's mesh: its tiling and geometry stream, mass
// pattern, fixed nodes, constraint targets and external load (gravity plus a device-side
// time-varying tip load); each sequence has its own material (E, nu), step size and
// state.  A step follows SyncedNesterov's Solve (SyncedNesterov.cu:97-360) for every
// sequence: the outer augmented-Lagrangian loop (v_prev = v, x = x_prev + dt v,
// c = x - x_jac, lambda += rho dt c) around the inner Nesterov loop
// (t' = (1 + sqrt(1 + 4 t^2)) / 2, beta = (t - 1) / t', y = v_k + beta (v_k - v_km1),
// x = x_prev + dt y, g = M (y - v_prev) / dt + f_int(x) - f_ext + dt J^T (lambda + rho c),
// v_next = y - alpha g).  The inner loop of a sequence ends on a relative-residual rule of
// the step, ||g_free|| / ||f_ext|| < rel_tol (g is the step's residual: inertia, internal
// and external force), or after max_inner iterations; with rel_tol = 0 every sequence runs
// exactly max_inner iterations, the reference's iteration with zero inner tolerance.
//
// B200 layout: each inner iteration is three kernels over every sequence still running,
//   k_dyn_force   one block per (tile, sequence), tile-major, so the sequences of a tile
//                 run back to back and its geometry stream is read from HBM once and from
//                 L2 after; fused F -> SVK P -> element forces plus the element-wise mass
//                 term M (y - v_prev) / dt; per-tile partials for shared nodes;
//   k_dyn_grad    one thread per (sequence, node): the node force (partials summed in tile
//                 order), the gradient, ||g_free||^2 partials folded per sequence by the
//                 last block to arrive (ticket; fold in block order, so deterministic),
//                 which also applies the stop rule and marks the sequence done;
//   k_dyn_update  one thread per (sequence, node): v_next = y - alpha g and the next
//                 look-ahead y and positions, fused;
// captured once as a CUDA graph of `chunk` iterations and replayed until every sequence
// is done (the host reads one counter per chunk).  Sequences that are done skip their
// work at block entry.  Warm starts per step: the previous step's velocity (the
// reference's behaviour), linear extrapolation 2 v_n - v_(n-1), or a caller-given
// velocity field (the learned step predictor).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "solver.cuh"

namespace tlfea {

constexpr int DYN_NODE_THREADS = 256;

enum { DYN_RUNNING = 0, DYN_RULE_MET = 1, DYN_OUT_OF_ITERS = 2, DYN_FINISHED = 3 };

struct DynArgs {
    int B, N, n_tiles, n_pslots, blocks_per_seq;
    const int* node_bidx;
    const int* bnode_off;
    const int* bnode_slots;
    const int* jt_off;
    const int* jt_col;
    const unsigned char* node_fixed;
    const double *xjx, *xjy, *xjz;  // constraint targets (x12_jac)
    const double* f_ext;            // 3N, this step's load, shared by the sequences
    const double* fext_norm;        // ||f_ext||
    // per-sequence state: sequence s at offset s*N (positions), s*3N (vectors),
    // s*3*n_pslots (partials), s*nc (multipliers)
    double *x, *y, *z, *xp, *yp, *zp;
    double *vg, *vp, *vk, *g, *f, *partial, *lam;
    int nc;
    const double *lam_s, *mu_s;  // per-sequence Lame parameters
    const double* alpha_s;       // per-sequence step size
    // per-sequence control
    int* done;
    int* inner;
    int* inner_total;
    int* rule_met;
    int* status;
    double* rel;
    double* red;
    unsigned int* ticket;
    int* n_done;
    const double* beta;  // beta[k] for the look-ahead after inner iteration k (beta[0] = 0)
    double rho, dt, rel_tol;
    int max_inner;
    // momentum restart (optional; off = the reference's iteration): per sequence the
    // index into beta, which restarts at 0 when g . (v_next - v_k) > 0 (the gradient
    // restart test of O'Donoghue and Candes, 2015); red2 holds the two dot partials
    int restart;
    int* mom;
    double* red2;
};

// ---------------------------------------------------------------- kernels

// f_ext = f_base + a * f_var (rounded multiply, then rounded add).
__global__ void k_dyn_load(int n3, const double* __restrict__ f_base, const double* __restrict__ f_var, double a,
                           double* __restrict__ f_ext) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n3) f_ext[i] = __dadd_rn(f_base[i], __dmul_rn(a, f_var[i]));
}

// ||f_ext|| of this step (one block, fixed summation order).
__global__ void k_dyn_fext_norm(int n3, const double* __restrict__ f, double* out) {
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < n3; i += blockDim.x) s += f[i] * f[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) *out = sqrt(s);
}

// Start of a step: the warm start of the velocity and x_prev = x.
//   mode 0: v stays the previous step's velocity;  mode 1: v = 2 v_n - v_(n-1);
//   mode 2: v = guess.  v_hist keeps v_n for the next step's extrapolation.
__global__ void k_dyn_begin_step(DynArgs D, double* __restrict__ vhist, const double* __restrict__ guess, int mode) {
    const int s = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.N) return;
    const size_t o = (size_t)s * D.N + i;
    D.xp[o] = D.x[o];
    D.yp[o] = D.y[o];
    D.zp[o] = D.z[o];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const size_t k = (size_t)s * 3 * D.N + 3 * i + d;
        const double v = D.vg[k];
        if (mode == 1) D.vg[k] = 2.0 * v - vhist[k];
        else if (mode == 2) D.vg[k] = guess[k];
        vhist[k] = v;
    }
}

// Control words of an outer iteration: sequences whose outer loop ended stay finished.
__global__ void k_dyn_outer_ctl(DynArgs D, const int* __restrict__ outer_done) {
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < D.B; s += blockDim.x) {
        const int od = outer_done[s];
        D.done[s] = od ? DYN_FINISHED : DYN_RUNNING;
        D.inner[s] = 0;
        D.mom[s] = 0;
        D.ticket[s] = 0u;
        if (od) atomicAdd(&cnt, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) *D.n_done = cnt;
}

// First look-ahead of an outer iteration: v_k = v_km1 = v, so y = v (beta_0 = 0).
__global__ void k_dyn_start(DynArgs D) {
    const int s = blockIdx.y;
    if (D.done[s] != DYN_RUNNING) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.N) return;
    const size_t o = (size_t)s * D.N + i, b3 = (size_t)s * 3 * D.N + 3 * i;
    D.vk[b3 + 0] = D.vg[b3 + 0];
    D.vk[b3 + 1] = D.vg[b3 + 1];
    D.vk[b3 + 2] = D.vg[b3 + 2];
    D.x[o] = D.xp[o] + D.dt * D.vg[b3 + 0];
    D.y[o] = D.yp[o] + D.dt * D.vg[b3 + 1];
    D.z[o] = D.zp[o] + D.dt * D.vg[b3 + 2];
}

// Element forces (and the element-wise mass term) of one tile of one sequence.  TET10
// without damping: 3 blocks per SM (168 registers); the others keep what they need.
template <int NPE, int NQP, bool DAMP>
__global__ void __launch_bounds__(TILE_ELEMS, (DAMP || NPE != 10) ? 1 : 3) k_dyn_force(DynArgs D, TileArgs<double> A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int s = blockIdx.x % D.B, tile = blockIdx.x / D.B;
    const int st = D.done[s];
    if (st != DYN_RUNNING) {
        // an out-of-iterations sequence has had its last velocity update: finished from now on
        // (other blocks of this kernel read either value and skip alike)
        if (st == DYN_OUT_OF_ITERS && tile == 0 && threadIdx.x == 0) D.done[s] = DYN_FINISHED;
        return;
    }
    const size_t oN = (size_t)s * D.N, o3 = 3 * oN;
    // this sequence's arrays and material; A itself stays the (unmodified) kernel parameter
    const TileSeq<double> sq{D.x + oN, D.y + oN, D.z + oN, D.vg + o3, D.vp + o3, D.f + o3,
                             D.partial + (size_t)s * 3 * D.n_pslots, D.lam_s[s], D.mu_s[s]};
    process_tile<double, NPE, NQP, TILE_FORCE, DAMP, false, true, true>(A, tile, smem, &sq);
}

// Node force, gradient, ||g_free||^2 partials; the last block of a sequence folds them and
// applies the stop rule.
__global__ void __launch_bounds__(DYN_NODE_THREADS) k_dyn_grad(DynArgs D) {
    __shared__ double red_sh[32];
    __shared__ bool last;
    const int s = blockIdx.y;
    if (D.done[s] != DYN_RUNNING) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t oN = (size_t)s * D.N, o3 = 3 * oN;
    double sg = 0.0, gdy = 0.0, gg = 0.0;
    if (i < D.N) {
        double fn[3];
        const int b = D.node_bidx[i];
        if (b < 0) {
            fn[0] = D.f[o3 + 3 * i + 0];
            fn[1] = D.f[o3 + 3 * i + 1];
            fn[2] = D.f[o3 + 3 * i + 2];
        } else {
            const double* part = D.partial + (size_t)s * 3 * D.n_pslots;
            double s0 = 0.0, s1 = 0.0, s2 = 0.0;
            for (int k = D.bnode_off[b]; k < D.bnode_off[b + 1]; ++k) {
                const int p = D.bnode_slots[k];
                s0 += part[3 * p + 0];
                s1 += part[3 * p + 1];
                s2 += part[3 * p + 2];
            }
            fn[0] = s0;
            fn[1] = s1;
            fn[2] = s2;
            D.f[o3 + 3 * i + 0] = s0;
            D.f[o3 + 3 * i + 1] = s1;
            D.f[o3 + 3 * i + 2] = s2;
        }
        const bool free_node = !D.node_fixed[i];
        const double xd[3] = {D.x[oN + i], D.y[oN + i], D.z[oN + i]};
        const double xj[3] = {D.xjx[i], D.xjy[i], D.xjz[i]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int t = 3 * i + d;
            double r = fn[d] - D.f_ext[t];  // the mass term is already in fn
            for (int k = D.jt_off[t]; k < D.jt_off[t + 1]; ++k) {
                const int ci = D.jt_col[k];
                r += D.dt * (D.lam[(size_t)s * D.nc + ci] + D.rho * (xd[d] - xj[d]));
            }
            D.g[o3 + t] = r;
            if (free_node) sg += r * r;
            if (D.restart) {
                gdy += r * (D.vg[o3 + t] - D.vk[o3 + t]);  // g . (y - v_k)
                gg += r * r;
            }
        }
    }
    if (D.restart) {
        gdy = block_sum(gdy, red_sh);
        gg = block_sum(gg, red_sh);
        if (threadIdx.x == 0) {
            D.red2[(size_t)s * D.blocks_per_seq + blockIdx.x] = gdy;
            D.red2[((size_t)D.B + s) * D.blocks_per_seq + blockIdx.x] = gg;
        }
    }
    sg = block_sum(sg, red_sh);
    if (threadIdx.x == 0) {
        D.red[(size_t)s * D.blocks_per_seq + blockIdx.x] = sg;
        __threadfence();
        const unsigned int tk = atomicAdd(&D.ticket[s], 1u);
        last = (tk == (unsigned int)D.blocks_per_seq - 1u);
    }
    __syncthreads();
    if (!last) return;
    if (threadIdx.x < 32) {
        __threadfence();
        double a = 0.0;
        double a_dy = 0.0, a_gg = 0.0;
        for (int bb = threadIdx.x; bb < D.blocks_per_seq; bb += 32) {
            a += __ldcg(D.red + (size_t)s * D.blocks_per_seq + bb);
            if (D.restart) {
                a_dy += __ldcg(D.red2 + (size_t)s * D.blocks_per_seq + bb);
                a_gg += __ldcg(D.red2 + ((size_t)D.B + s) * D.blocks_per_seq + bb);
            }
        }
        a = warp_sum(a);
        a_dy = warp_sum(a_dy);
        a_gg = warp_sum(a_gg);
        if (threadIdx.x == 0) {
            D.ticket[s] = 0u;
            // g . (v_next - v_k) = g . (y - v_k) - alpha ||g||^2 > 0: the step works against
            // the momentum, so the next look-ahead starts the beta sequence afresh
            const bool restart_now = D.restart && (a_dy - D.alpha_s[s] * a_gg > 0.0);
            D.mom[s] = restart_now ? 0 : D.mom[s] + 1;
            const double fe = *D.fext_norm;
            const double rel = fe > 0.0 ? sqrt(a) / fe : sqrt(a);
            D.rel[s] = rel;
            const int it = D.inner[s] + 1;
            D.inner[s] = it;
            D.inner_total[s] += 1;
            int nd = DYN_RUNNING;
            if (!isfinite(rel)) {
                D.status[s] = TLFEA_NONFINITE;
                nd = DYN_RULE_MET;  // stop without another update
            } else if (D.rel_tol > 0.0 && rel < D.rel_tol) {
                D.rule_met[s] = 1;
                nd = DYN_RULE_MET;  // keep v = y: the positions the residual was measured at
            } else if (it >= D.max_inner) {
                nd = DYN_OUT_OF_ITERS;  // one more velocity update, no look-ahead
            }
            if (nd != DYN_RUNNING) {
                D.done[s] = nd;
                atomicAdd(D.n_done, 1);
            }
        }
    }
}

// v_next = y - alpha g; then the next look-ahead y' = v_next + beta_k (v_next - v_k) and
// x = x_prev + dt y' (a sequence out of iterations keeps v = v_next).
__global__ void __launch_bounds__(DYN_NODE_THREADS) k_dyn_update(DynArgs D) {
    const int s = blockIdx.y;
    const int st = D.done[s];
    if (st == DYN_RULE_MET || st == DYN_FINISHED) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.N) return;
    const size_t oN = (size_t)s * D.N, o3 = 3 * oN;
    const bool predict = (st == DYN_RUNNING);
    const double beta = predict ? D.beta[D.mom[s]] : 0.0;
    const double alpha = D.alpha_s[s];
    double yv[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const size_t k = o3 + 3 * i + d;
        const double vn = D.vg[k] - alpha * D.g[k];
        const double vko = D.vk[k];
        D.vk[k] = vn;
        yv[d] = predict ? vn + beta * (vn - vko) : vn;
        D.vg[k] = yv[d];
    }
    D.x[oN + i] = D.xp[oN + i] + D.dt * yv[0];
    D.y[oN + i] = D.yp[oN + i] + D.dt * yv[1];
    D.z[oN + i] = D.zp[oN + i] + D.dt * yv[2];
}

// Outer update of the sequences still in their outer loop: v_prev = v, x = x_prev + dt v,
// c = x - x_jac, lambda += rho dt c; ||c|| folded per sequence; a sequence whose stop rule
// was met, or whose ||c|| < outer_tol, has finished its step.
__global__ void __launch_bounds__(DYN_NODE_THREADS) k_dyn_outer(DynArgs D, int* __restrict__ outer_done,
                                                               const int* __restrict__ fixed, int n_fixed,
                                                               double outer_tol, unsigned int* ticket2) {
    __shared__ double red_sh[32];
    __shared__ bool last;
    const int s = blockIdx.y;
    if (outer_done[s]) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t oN = (size_t)s * D.N, o3 = 3 * oN;
    if (i < D.N) {
        double v[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v[d] = D.vg[o3 + 3 * i + d];
            D.vp[o3 + 3 * i + d] = v[d];
        }
        D.x[oN + i] = D.xp[oN + i] + D.dt * v[0];
        D.y[oN + i] = D.yp[oN + i] + D.dt * v[1];
        D.z[oN + i] = D.zp[oN + i] + D.dt * v[2];
    }
    // constraints: this block's share of the fixed nodes (grid-strided over blockIdx.x)
    double sc = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_fixed; k += gridDim.x * blockDim.x) {
        const int n = fixed[k];
        const double v[3] = {D.vg[o3 + 3 * n + 0], D.vg[o3 + 3 * n + 1], D.vg[o3 + 3 * n + 2]};
        const double xn[3] = {D.xp[oN + n] + D.dt * v[0], D.yp[oN + n] + D.dt * v[1], D.zp[oN + n] + D.dt * v[2]};
        const double xj[3] = {D.xjx[n], D.xjy[n], D.xjz[n]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double c = xn[d] - xj[d];
            D.lam[(size_t)s * D.nc + 3 * k + d] += D.rho * D.dt * c;
            sc += c * c;
        }
    }
    sc = block_sum(sc, red_sh);
    if (threadIdx.x == 0) {
        D.red[(size_t)s * D.blocks_per_seq + blockIdx.x] = sc;
        __threadfence();
        const unsigned int tk = atomicAdd(&ticket2[s], 1u);
        last = (tk == (unsigned int)gridDim.x - 1u);
    }
    __syncthreads();
    if (!last) return;
    if (threadIdx.x < 32) {
        __threadfence();
        double a = 0.0;
        for (int bb = threadIdx.x; bb < (int)gridDim.x; bb += 32)
            a += __ldcg(D.red + (size_t)s * D.blocks_per_seq + bb);
        a = warp_sum(a);
        if (threadIdx.x == 0) {
            ticket2[s] = 0u;
            if (D.rule_met[s] || D.status[s] || sqrt(a) < outer_tol) outer_done[s] = 1;
        }
    }
}

__global__ void k_dyn_reset_state(DynArgs D, double* __restrict__ vhist, const double* __restrict__ X0x,
                                  const double* __restrict__ X0y, const double* __restrict__ X0z) {
    const int s = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.N) return;
    const size_t oN = (size_t)s * D.N, o3 = 3 * oN;
    D.x[oN + i] = D.xp[oN + i] = X0x[i];
    D.y[oN + i] = D.yp[oN + i] = X0y[i];
    D.z[oN + i] = D.zp[oN + i] = X0z[i];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const size_t k = o3 + 3 * i + d;
        D.vg[k] = D.vp[k] = D.vk[k] = vhist[k] = 0.0;
    }
}

}  // namespace tlfea

using namespace tlfea;

struct tlfea_dynbatch_s {
    tlfea_element_s* el = nullptr;
    int B = 0;
    int device = 0;
    DynArgs D{};
    // per-sequence arrays
    double *x = nullptr, *y = nullptr, *z = nullptr, *xp = nullptr, *yp = nullptr, *zp = nullptr;
    double *vg = nullptr, *vp = nullptr, *vk = nullptr, *g = nullptr, *f = nullptr, *partial = nullptr;
    double *lam = nullptr, *vhist = nullptr, *lam_s = nullptr, *mu_s = nullptr, *alpha_s = nullptr;
    int *done = nullptr, *inner = nullptr, *inner_total = nullptr, *rule_met = nullptr, *status = nullptr;
    int* outer_done = nullptr;
    int* mom = nullptr;       // momentum index per sequence (restart)
    double* red2 = nullptr;   // restart test partials
    double *rel = nullptr, *red = nullptr, *beta = nullptr, *fext_norm = nullptr;
    unsigned int *ticket = nullptr, *ticket2 = nullptr;
    int* counters = nullptr;    // [n_done]
    int* h_counters = nullptr;  // pinned copy
    int* zero_off = nullptr;    // all-zero J^T offsets of a mesh without constraints
    unsigned char* node_fixed = nullptr;
    double* f_base = nullptr;
    double* f_var = nullptr;
    double amp = 0.0, omega = 0.0, phase = 0.0;
    long long step_index = 0;  // steps taken since the last reset; step k ends at t = k * dt
    tlfea_nesterov_params np{};
    double rel_tol = 0.0;
    bool params_set = false;
    int chunk = 8;
    cudaGraphExec_t graph = nullptr;
    int beta_n = -1;
};

namespace {

// Launch check inside graph capture (the replays are counted where the graph is launched).
#define DYN_CHECK()                                                                       \
    do {                                                                                  \
        cudaError_t e_ = cudaGetLastError();                                              \
        if (e_ != cudaSuccess) {                                                          \
            set_error(std::string("batched dynamics launch: ") + cudaGetErrorString(e_)); \
            return TLFEA_CUDA_ERROR;                                                      \
        }                                                                                 \
    } while (0)

template <int NPE, int NQP, bool DAMP>
size_t force_smem(const tlfea_element_s* el) {
    return tile_smem_bytes<double>(NPE, el->tl.max_local, DAMP, true);
}

// Opt the force kernel into its dynamic shared memory (outside any stream capture).
template <int NPE, int NQP, bool DAMP>
int prepare_force(tlfea_dynbatch_s* b) {
    const size_t smem = force_smem<NPE, NQP, DAMP>(b->el);
    if (smem > 200 * 1024) {
        set_error("batched dynamics: tile shared memory exceeds 200 KB");
        return TLFEA_UNSUPPORTED;
    }
    if (smem > 48 * 1024)
        TLFEA_CUDA(cudaFuncSetAttribute(k_dyn_force<NPE, NQP, DAMP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    return TLFEA_OK;
}

template <int NPE, int NQP, bool DAMP>
int enqueue_force(tlfea_dynbatch_s* b, cudaStream_t stream) {
    tlfea_element_s* el = b->el;
    TileArgs<double> A;
    memset(&A, 0, sizeof(A));
    const Tiling& tl = el->tl;
    A.node_off = tl.node_off;
    A.ln_gid = tl.ln_gid;
    A.ln_pslot = tl.ln_pslot;
    A.ln_inc_end = tl.ln_inc_end;
    A.inc = tl.inc;
    A.lconn = tl.lconn;
    A.tile_elem = tl.tile_elem;
    A.grad = tl.grad64;
    A.ji = tl.ji64;
    A.dv = tl.dv64;
    A.eta = el->eta_d;
    A.lamd = el->lambda_d;
    A.max_local = tl.max_local;
    A.qb = qp_bary(el);
    A.mass_scale = el->rho / b->np.time_step;
    k_dyn_force<NPE, NQP, DAMP><<<tl.n_tiles * b->B, TILE_ELEMS, force_smem<NPE, NQP, DAMP>(el), stream>>>(b->D, A);
    DYN_CHECK();
    return TLFEA_OK;
}

int enqueue_iteration(tlfea_dynbatch_s* b, cudaStream_t stream) {
    tlfea_element_s* el = b->el;
    const bool damp = (el->eta_d != 0.0 || el->lambda_d != 0.0);
    int st;
    if (el->npe == 10)
        st = damp ? enqueue_force<10, 5, true>(b, stream) : enqueue_force<10, 5, false>(b, stream);
    else
        st = damp ? enqueue_force<4, 1, true>(b, stream) : enqueue_force<4, 1, false>(b, stream);
    if (st) return st;
    const dim3 grid(b->D.blocks_per_seq, b->B);
    k_dyn_grad<<<grid, DYN_NODE_THREADS, 0, stream>>>(b->D);
    DYN_CHECK();
    k_dyn_update<<<grid, DYN_NODE_THREADS, 0, stream>>>(b->D);
    DYN_CHECK();
    return TLFEA_OK;
}

// A CUDA graph of `chunk` inner iterations, built on first use after the parameters last
// changed (the kernels' arguments are baked into it).
int ensure_graph(tlfea_dynbatch_s* b) {
    if (b->graph) return TLFEA_OK;
    cudaStream_t stream = b->el->stream;
    const bool damp = (b->el->eta_d != 0.0 || b->el->lambda_d != 0.0);
    int st;
    if (b->el->npe == 10)
        st = damp ? prepare_force<10, 5, true>(b) : prepare_force<10, 5, false>(b);
    else
        st = damp ? prepare_force<4, 1, true>(b) : prepare_force<4, 1, false>(b);
    if (st) return st;
    cudaGraph_t g = nullptr;
    TLFEA_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < b->chunk && !st; ++k) st = enqueue_iteration(b, stream);
    const cudaError_t ec = cudaStreamEndCapture(stream, &g);
    if (st || ec != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (!st) set_error("batched dynamics: graph capture failed");
        return st ? st : TLFEA_CUDA_ERROR;
    }
    const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        b->graph = nullptr;
        set_error(std::string("batched dynamics: graph instantiation: ") + cudaGetErrorString(ei));
        return TLFEA_CUDA_ERROR;
    }
    return TLFEA_OK;
}

void drop_graph(tlfea_dynbatch_s* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

// beta[k] for the look-ahead after inner iteration k (k = 0..max_inner): t_0 = 1,
// t_(k+1) = (1 + sqrt(1 + 4 t_k^2)) / 2, beta_k = (t_k - 1) / t_(k+1)
// (SyncedNesterov.cu:153-156).
int upload_beta(tlfea_dynbatch_s* b) {
    const int n = b->np.max_inner + 1;
    if (b->beta_n == n) return TLFEA_OK;
    std::vector<double> beta((size_t)n);
    double t = 1.0;
    for (int k = 0; k < n; ++k) {
        const double tn = 0.5 * (1.0 + std::sqrt(1.0 + 4.0 * t * t));
        beta[k] = (t - 1.0) / tn;
        t = tn;
    }
    dfree(b->beta);
    int st = dalloc(&b->beta, (size_t)n);
    if (st) return st;
    TLFEA_CUDA(cudaMemcpy(b->beta, beta.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    b->D.beta = b->beta;
    b->beta_n = n;
    return TLFEA_OK;
}

void dyn_free(tlfea_dynbatch_s* b) {
    drop_graph(b);
    dfree(b->x); dfree(b->y); dfree(b->z); dfree(b->xp); dfree(b->yp); dfree(b->zp);
    dfree(b->vg); dfree(b->vp); dfree(b->vk); dfree(b->g); dfree(b->f); dfree(b->partial);
    dfree(b->lam); dfree(b->vhist); dfree(b->lam_s); dfree(b->mu_s); dfree(b->alpha_s);
    dfree(b->done); dfree(b->inner); dfree(b->inner_total); dfree(b->rule_met); dfree(b->status);
    dfree(b->outer_done); dfree(b->rel); dfree(b->red); dfree(b->beta); dfree(b->fext_norm);
    dfree(b->mom); dfree(b->red2);
    dfree(b->ticket); dfree(b->ticket2); dfree(b->counters); dfree(b->node_fixed);
    dfree(b->f_base); dfree(b->f_var); dfree(b->zero_off);
    if (b->h_counters) cudaFreeHost(b->h_counters);
    b->h_counters = nullptr;
}

}  // namespace

#define CHECK_DYN(b)                                   \
    do {                                               \
        if (!(b)) {                                    \
            set_error("null batched-dynamics handle"); \
            return TLFEA_INVALID_ARG;                  \
        }                                              \
        TLFEA_CUDA(cudaSetDevice((b)->device));        \
    } while (0)

extern "C" {

int tlfea_dynbatch_create(tlfea_element mesh, int n_seq, tlfea_dynbatch* out) {
    if (!mesh || !out || n_seq < 1) return TLFEA_INVALID_ARG;
    *out = nullptr;
    tlfea_element_s* el = mesh;
    if (!el->is_setup || !el->precomputed || !el->mass_setup) {
        set_error("batched dynamics: the mesh element needs Setup, CalcDnDuPre and CalcMassMatrix first");
        return TLFEA_NOT_SETUP;
    }
    if (el->tl.n_orphans > 0) {
        set_error("batched dynamics: every node must belong to an element");
        return TLFEA_UNSUPPORTED;
    }
    if (el->material != TLFEA_MATERIAL_SVK) {
        set_error("batched dynamics: SVK material only");
        return TLFEA_UNSUPPORTED;
    }
    int st;
    if (el->n_constraint > 0 && !el->jt_setup && (st = tlfea_element_build_constraint_jact_csr(el))) return st;
    TLFEA_CUDA(cudaSetDevice(el->device));
    auto* b = new tlfea_dynbatch_s();
    b->el = el;
    b->B = n_seq;
    b->device = el->device;
    const size_t N = el->N, B = n_seq, n3 = 3 * N;
    const size_t nc = (size_t)std::max(el->n_constraint, 1);
    const int bps = (int)((N + DYN_NODE_THREADS - 1) / DYN_NODE_THREADS);
    st = 0;
    st |= dalloc(&b->x, B * N) | dalloc(&b->y, B * N) | dalloc(&b->z, B * N);
    st |= dalloc(&b->xp, B * N) | dalloc(&b->yp, B * N) | dalloc(&b->zp, B * N);
    st |= dalloc(&b->vg, B * n3) | dalloc(&b->vp, B * n3) | dalloc(&b->vk, B * n3) | dalloc(&b->g, B * n3);
    st |= dalloc(&b->f, B * n3) | dalloc(&b->vhist, B * n3);
    st |= dalloc(&b->partial, B * 3 * (size_t)std::max(el->tl.n_pslots, 1));
    st |= dalloc(&b->lam, B * nc) | dalloc(&b->lam_s, B) | dalloc(&b->mu_s, B) | dalloc(&b->alpha_s, B);
    st |= dalloc(&b->done, B) | dalloc(&b->inner, B) | dalloc(&b->inner_total, B) | dalloc(&b->rule_met, B);
    st |= dalloc(&b->status, B) | dalloc(&b->outer_done, B) | dalloc(&b->rel, B);
    st |= dalloc(&b->red, B * (size_t)bps) | dalloc(&b->fext_norm, 1);
    st |= dalloc(&b->mom, B) | dalloc(&b->red2, 2 * B * (size_t)bps);
    st |= dalloc(&b->ticket, B) | dalloc(&b->ticket2, B) | dalloc(&b->counters, 1);
    st |= dalloc(&b->node_fixed, N) | dalloc(&b->f_base, n3) | dalloc(&b->f_var, n3);
    if (el->n_constraint == 0) st |= dalloc(&b->zero_off, n3 + 1);
    if (!st && cudaMallocHost((void**)&b->h_counters, sizeof(int)) != cudaSuccess) st = TLFEA_CUDA_ERROR;
    if (st) {
        dyn_free(b);
        delete b;
        set_error("batched dynamics: device allocation failed");
        return TLFEA_CUDA_ERROR;
    }
    std::vector<unsigned char> nf(N, 0);
    for (int n : el->h_fixed) nf[n] = 1;
    cudaStream_t stream = el->stream;
    const cudaError_t e0 = cudaMemcpyAsync(b->node_fixed, nf.data(), N, cudaMemcpyHostToDevice, stream);
    const cudaError_t e1 = cudaMemcpyAsync(b->f_base, el->f_ext, n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream);
    cudaMemsetAsync(b->f_var, 0, n3 * sizeof(double), stream);
    cudaMemsetAsync(b->ticket, 0, B * sizeof(unsigned int), stream);
    cudaMemsetAsync(b->ticket2, 0, B * sizeof(unsigned int), stream);
    cudaMemsetAsync(b->lam, 0, B * nc * sizeof(double), stream);
    if (b->zero_off) cudaMemsetAsync(b->zero_off, 0, (n3 + 1) * sizeof(int), stream);
    std::vector<double> lam_s(B, el->lambda), mu_s(B, el->mu), al(B, 1.0);
    cudaMemcpyAsync(b->lam_s, lam_s.data(), B * sizeof(double), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(b->mu_s, mu_s.data(), B * sizeof(double), cudaMemcpyHostToDevice, stream);
    cudaMemcpyAsync(b->alpha_s, al.data(), B * sizeof(double), cudaMemcpyHostToDevice, stream);
    DynArgs& D = b->D;
    D.B = n_seq;
    D.N = el->N;
    D.n_tiles = el->tl.n_tiles;
    D.n_pslots = el->tl.n_pslots;
    D.blocks_per_seq = bps;
    D.node_bidx = el->tl.node_bidx;
    D.bnode_off = el->tl.bnode_off;
    D.bnode_slots = el->tl.bnode_slots;
    D.jt_off = b->zero_off ? b->zero_off : el->jt_off;
    D.jt_col = b->zero_off ? b->zero_off : el->jt_col;
    D.node_fixed = b->node_fixed;
    D.xjx = el->xj;
    D.xjy = el->yj;
    D.xjz = el->zj;
    D.f_ext = el->f_ext;
    D.fext_norm = b->fext_norm;
    D.x = b->x; D.y = b->y; D.z = b->z; D.xp = b->xp; D.yp = b->yp; D.zp = b->zp;
    D.vg = b->vg; D.vp = b->vp; D.vk = b->vk; D.g = b->g; D.f = b->f; D.partial = b->partial; D.lam = b->lam;
    D.nc = (int)nc;
    D.lam_s = b->lam_s;
    D.mu_s = b->mu_s;
    D.alpha_s = b->alpha_s;
    D.done = b->done; D.inner = b->inner; D.inner_total = b->inner_total; D.rule_met = b->rule_met;
    D.status = b->status; D.rel = b->rel; D.red = b->red; D.ticket = b->ticket; D.n_done = b->counters;
    D.mom = b->mom;
    D.red2 = b->red2;
    D.restart = 0;
    cudaMemsetAsync(b->mom, 0, B * sizeof(int), stream);
    const dim3 grid(bps, n_seq);
    k_dyn_reset_state<<<grid, DYN_NODE_THREADS, 0, stream>>>(D, b->vhist, el->X0x, el->X0y, el->X0z);
    const cudaError_t e2 = cudaGetLastError();
    const cudaError_t e3 = cudaStreamSynchronize(stream);
    if (e0 != cudaSuccess || e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
        dyn_free(b);
        delete b;
        set_error("batched dynamics: set-up copies failed");
        return TLFEA_CUDA_ERROR;
    }
    TLFEA_LAUNCHED(1);
    *out = b;
    return TLFEA_OK;
}

int tlfea_dynbatch_destroy(tlfea_dynbatch b) {
    if (!b) return TLFEA_OK;
    cudaSetDevice(b->device);
    dyn_free(b);
    delete b;
    return TLFEA_OK;
}

int tlfea_dynbatch_set_material(tlfea_dynbatch b, const double* E, const double* nu) {
    CHECK_DYN(b);
    if (!E || !nu) return TLFEA_INVALID_ARG;
    std::vector<double> lam((size_t)b->B), mu((size_t)b->B);
    for (int s = 0; s < b->B; ++s) {
        if (!(E[s] > 0.0) || !(nu[s] > -1.0 && nu[s] < 0.5)) {
            set_error("batched dynamics: E must be positive and -1 < nu < 0.5");
            return TLFEA_INVALID_ARG;
        }
        // SetSVK(E, nu) (FEAT10Data.cuh:553-569)
        mu[s] = E[s] / (2 * (1 + nu[s]));
        lam[s] = (E[s] * nu[s]) / ((1 + nu[s]) * (1 - 2 * nu[s]));
    }
    TLFEA_CUDA(cudaMemcpy(b->lam_s, lam.data(), sizeof(double) * b->B, cudaMemcpyHostToDevice));
    TLFEA_CUDA(cudaMemcpy(b->mu_s, mu.data(), sizeof(double) * b->B, cudaMemcpyHostToDevice));
    return TLFEA_OK;
}

int tlfea_dynbatch_set_parameters(tlfea_dynbatch b, const tlfea_nesterov_params* p, double rel_tol) {
    CHECK_DYN(b);
    if (!p || p->max_inner < 1 || p->max_outer < 1 || !(p->time_step > 0.0) || !(p->alpha > 0.0) || rel_tol < 0.0)
        return TLFEA_INVALID_ARG;
    b->np = *p;
    b->rel_tol = rel_tol;
    std::vector<double> al((size_t)b->B, p->alpha);
    TLFEA_CUDA(cudaMemcpy(b->alpha_s, al.data(), sizeof(double) * b->B, cudaMemcpyHostToDevice));
    b->D.rho = p->rho;
    b->D.dt = p->time_step;
    b->D.rel_tol = rel_tol;
    b->D.max_inner = p->max_inner;
    int st = upload_beta(b);
    if (st) return st;
    drop_graph(b);  // kernel arguments changed
    b->params_set = true;
    return TLFEA_OK;
}

// Per-sequence step sizes (after set_parameters, which gives every sequence p->alpha).
int tlfea_dynbatch_set_step_sizes(tlfea_dynbatch b, const double* alpha) {
    CHECK_DYN(b);
    if (!alpha) return TLFEA_INVALID_ARG;
    for (int s = 0; s < b->B; ++s)
        if (!(alpha[s] > 0.0)) return TLFEA_INVALID_ARG;
    TLFEA_CUDA(cudaMemcpy(b->alpha_s, alpha, sizeof(double) * b->B, cudaMemcpyHostToDevice));
    return TLFEA_OK;
}

// f_ext(t) = f_base + amp * sin(omega * t + phase) * f_var, evaluated on the device at the
// end time of every step; f_base is the element's f_ext when the batch was created
// (e.g. gravity added with AddGravity).
int tlfea_dynbatch_set_load(tlfea_dynbatch b, const double* f_var, int n, double amp, double omega, double phase) {
    CHECK_DYN(b);
    if (n != 3 * b->el->N) return TLFEA_SIZE_MISMATCH;
    if (f_var) TLFEA_CUDA(cudaMemcpy(b->f_var, f_var, sizeof(double) * n, cudaMemcpyHostToDevice));
    else TLFEA_CUDA(cudaMemset(b->f_var, 0, sizeof(double) * n));
    b->amp = amp;
    b->omega = omega;
    b->phase = phase;
    return TLFEA_OK;
}

int tlfea_dynbatch_set_restart(tlfea_dynbatch b, int on) {
    CHECK_DYN(b);
    if (on != 0 && on != 1) return TLFEA_INVALID_ARG;
    if (on != b->D.restart) drop_graph(b);  // kernel arguments changed
    b->D.restart = on;
    return TLFEA_OK;
}

int tlfea_dynbatch_set_chunk(tlfea_dynbatch b, int chunk) {
    CHECK_DYN(b);
    if (chunk < 1 || chunk > 256) return TLFEA_INVALID_ARG;
    if (chunk != b->chunk) drop_graph(b);
    b->chunk = chunk;
    return TLFEA_OK;
}

// Positions back to the reference configuration, velocities and multipliers to zero, t = 0.
int tlfea_dynbatch_reset(tlfea_dynbatch b) {
    CHECK_DYN(b);
    cudaStream_t stream = b->el->stream;
    const dim3 grid(b->D.blocks_per_seq, b->B);
    k_dyn_reset_state<<<grid, DYN_NODE_THREADS, 0, stream>>>(b->D, b->vhist, b->el->X0x, b->el->X0y, b->el->X0z);
    TLFEA_CHECK_LAUNCH();
    TLFEA_CUDA(cudaMemsetAsync(b->lam, 0, sizeof(double) * (size_t)b->B * b->D.nc, stream));
    TLFEA_CUDA(cudaStreamSynchronize(stream));
    b->step_index = 0;
    return TLFEA_OK;
}

// One implicit step of every sequence (see the header).
int tlfea_dynbatch_step(tlfea_dynbatch b, int warm_start, const double* d_v_guess, int* iters, double* rel,
                        int* converged) {
    CHECK_DYN(b);
    if (!b->params_set) {
        set_error("batched dynamics: set_parameters first");
        return TLFEA_NOT_SETUP;
    }
    if (warm_start < 0 || warm_start > 2 || (warm_start == 2 && !d_v_guess)) return TLFEA_INVALID_ARG;
    tlfea_element_s* el = b->el;
    cudaStream_t stream = el->stream;
    int st;
    if ((st = ensure_graph(b))) return st;
    const int n3 = 3 * el->N;
    const dim3 grid(b->D.blocks_per_seq, b->B);
    // this step's load (end time t = k dt) and its norm
    b->step_index += 1;
    const double t_end = (double)b->step_index * b->np.time_step;
    const double a = b->amp * sin(b->omega * t_end + b->phase);
    k_dyn_load<<<(n3 + 255) / 256, 256, 0, stream>>>(n3, b->f_base, b->f_var, a, el->f_ext);
    TLFEA_CHECK_LAUNCH();
    k_dyn_fext_norm<<<1, 1024, 0, stream>>>(n3, el->f_ext, b->fext_norm);
    TLFEA_CHECK_LAUNCH();
    k_dyn_begin_step<<<grid, DYN_NODE_THREADS, 0, stream>>>(b->D, b->vhist, d_v_guess, warm_start);
    TLFEA_CHECK_LAUNCH();
    TLFEA_CUDA(cudaMemsetAsync(b->outer_done, 0, sizeof(int) * b->B, stream));
    TLFEA_CUDA(cudaMemsetAsync(b->inner_total, 0, sizeof(int) * b->B, stream));
    TLFEA_CUDA(cudaMemsetAsync(b->rule_met, 0, sizeof(int) * b->B, stream));
    TLFEA_CUDA(cudaMemsetAsync(b->status, 0, sizeof(int) * b->B, stream));
    std::vector<int> od((size_t)b->B);
    for (int outer = 0; outer < b->np.max_outer; ++outer) {
        k_dyn_outer_ctl<<<1, 1024, 0, stream>>>(b->D, b->outer_done);
        TLFEA_CHECK_LAUNCH();
        k_dyn_start<<<grid, DYN_NODE_THREADS, 0, stream>>>(b->D);
        TLFEA_CHECK_LAUNCH();
        for (int run = 0; run < b->np.max_inner; run += b->chunk) {
            TLFEA_CUDA(cudaGraphLaunch(b->graph, stream));
            TLFEA_LAUNCHED(3 * b->chunk);
            TLFEA_CUDA(cudaMemcpyAsync(b->h_counters, b->counters, sizeof(int), cudaMemcpyDeviceToHost, stream));
            TLFEA_CUDA(cudaStreamSynchronize(stream));
            if (b->h_counters[0] >= b->B) break;
        }
        k_dyn_outer<<<grid, DYN_NODE_THREADS, 0, stream>>>(b->D, b->outer_done, el->fixed, (int)el->h_fixed.size(),
                                                        b->np.outer_tol, b->ticket2);
        TLFEA_CHECK_LAUNCH();
        TLFEA_CUDA(cudaMemcpyAsync(od.data(), b->outer_done, sizeof(int) * b->B, cudaMemcpyDeviceToHost, stream));
        TLFEA_CUDA(cudaStreamSynchronize(stream));
        int n_od = 0;
        for (int v : od) n_od += v;
        if (n_od >= b->B) break;
    }
    std::vector<int> it((size_t)b->B), rm((size_t)b->B), sts((size_t)b->B);
    std::vector<double> rl((size_t)b->B);
    TLFEA_CUDA(cudaMemcpy(it.data(), b->inner_total, sizeof(int) * b->B, cudaMemcpyDeviceToHost));
    TLFEA_CUDA(cudaMemcpy(rm.data(), b->rule_met, sizeof(int) * b->B, cudaMemcpyDeviceToHost));
    TLFEA_CUDA(cudaMemcpy(sts.data(), b->status, sizeof(int) * b->B, cudaMemcpyDeviceToHost));
    TLFEA_CUDA(cudaMemcpy(rl.data(), b->rel, sizeof(double) * b->B, cudaMemcpyDeviceToHost));
    if (iters) std::copy(it.begin(), it.end(), iters);
    if (rel) std::copy(rl.begin(), rl.end(), rel);
    if (converged) std::copy(rm.begin(), rm.end(), converged);
    for (int v : sts)
        if (v) {
            set_error("batched dynamics: non-finite residual");
            return TLFEA_NONFINITE;
        }
    return TLFEA_OK;
}

int tlfea_dynbatch_device_ptrs(tlfea_dynbatch b, double** x, double** y, double** z, double** v, double** v_hist) {
    CHECK_DYN(b);
    if (x) *x = b->x;
    if (y) *y = b->y;
    if (z) *z = b->z;
    if (v) *v = b->vg;
    if (v_hist) *v_hist = b->vhist;
    return TLFEA_OK;
}

int tlfea_dynbatch_retrieve_positions(tlfea_dynbatch b, int seq, double* x, double* y, double* z) {
    CHECK_DYN(b);
    if (seq < 0 || seq >= b->B || !x || !y || !z) return TLFEA_INVALID_ARG;
    const size_t N = b->el->N, o = (size_t)seq * N;
    TLFEA_CUDA(cudaStreamSynchronize(b->el->stream));
    TLFEA_CUDA(cudaMemcpy(x, b->x + o, sizeof(double) * N, cudaMemcpyDeviceToHost));
    TLFEA_CUDA(cudaMemcpy(y, b->y + o, sizeof(double) * N, cudaMemcpyDeviceToHost));
    TLFEA_CUDA(cudaMemcpy(z, b->z + o, sizeof(double) * N, cudaMemcpyDeviceToHost));
    return TLFEA_OK;
}

int tlfea_dynbatch_retrieve_velocity(tlfea_dynbatch b, int seq, double* v) {
    CHECK_DYN(b);
    if (seq < 0 || seq >= b->B || !v) return TLFEA_INVALID_ARG;
    const size_t n3 = 3 * (size_t)b->el->N;
    TLFEA_CUDA(cudaStreamSynchronize(b->el->stream));
    TLFEA_CUDA(cudaMemcpy(v, b->vg + (size_t)seq * n3, sizeof(double) * n3, cudaMemcpyDeviceToHost));
    return TLFEA_OK;
}

}  // extern "C"
