// first_order.cu -- SyncedNesterovSolver, SyncedAdamWSolver and
// SyncedAdamWNocoopSolver (SyncedNesterov.cu:97-414, SyncedAdamW.cu:99-425,
// SyncedAdamWNocoop.cu:97-458) as one persistent cooperative kernel per Solve().
//
// Differences from the reference, none of which changes the iteration:
//   * every phase is grid-strided, so any mesh size runs (the reference
//     Nesterov leaves DOFs beyond its co-resident grid un-updated, and its
//     AdamW refuses such sizes);
//   * the internal force is the fused tile routine (no F/P round trip through
//     HBM, no atomics) and the gradient reads it back per node;
//   * the inertial term M (v - v_prev) / dt is added element by element in the
//     same tiles (the consistent mass from the shape functions at the QPs) when
//     the stop rule is off, instead of an assembled mass-row pass per node;
//   * norms are two-level reductions (block shuffles, then every block folds
//     the per-block partials in block order, so every block takes the same
//     branch without another barrier) instead of one thread's serial loop;
//   * about 4 grid barriers per inner iteration instead of 13.
//   * a non-finite ||g|| ends the solve with TLFEA_NONFINITE;
//   * optional relative-residual stop rule (new): ||(f_int - f_ext)_free|| /
//     ||f_ext|| < rel_tol in FP64 at the positions of the last force evaluation.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "solver.cuh"

namespace cg = cooperative_groups;

namespace tlfea {

struct FOArgs {
    int kind;
    int N, nc, n_fixed, n_tiles;
    const int* fixed;
    double* c;
    const double *xj, *yj, *zj;
    double *x, *y, *z;
    const double *X0x, *X0y, *X0z;
    const int* m_off;
    const int* m_col;
    const double* m_val;
    const double* f_ext;
    double* f_int64;
    float* f_int32;
    const int* node_bidx;
    const int* bnode_off;
    const int* bnode_slots;
    const int* jt_off;
    const int* jt_col;
    double *vg, *vp, *vk, *vkm1, *g, *lam, *m, *va, *xp, *yp, *zp;
    double* red;
    int red_stride;
    int* stat;          // [outer, inner_total, last_inner, status, ||g|| (2 ints), rel (2 ints), rule met]
    double* stat_norm;  // last ||g||
    double* stat_rel;   // last ||(f_int - f_ext)_free|| / ||f_ext|| (stop rule on)
    double rel_tol;     // relative-residual stop rule (0 = off)
    const unsigned char* node_fixed;
    // parameters (SyncedNesterovParams / SyncedAdamWParams)
    double alpha, rho, inner_tol, outer_tol, dt;
    int max_outer, max_inner;
    double lr, beta1, beta2, eps, wd, lr_decay, rtol;
    int check;
};

// Every block folds the per-block partials of slot `k` in block order.
__device__ __forceinline__ double fold_partials(const FOArgs& S, int k, double* sh) {
    __syncthreads();
    if (threadIdx.x < 32) {
        double s = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) s += __ldcg(S.red + (size_t)k * S.red_stride + b);
        s = warp_sum(s);
        if (threadIdx.x == 0) *sh = s;
    }
    __syncthreads();
    return *sh;
}

__device__ __forceinline__ void write_partial(const FOArgs& S, int k, double v, double* red_sh) {
    const double s = block_sum(v, red_sh);
    if (threadIdx.x == 0) S.red[(size_t)k * S.red_stride + blockIdx.x] = s;
}

// x = x_prev + dt * v (FP32 force mode stages x - X0 per tile from these)
template <typename R>
__device__ __forceinline__ void set_node_positions(const FOArgs& S, int i, double v0, double v1, double v2) {
    S.x[i] = S.xp[i] + S.dt * v0;
    S.y[i] = S.yp[i] + S.dt * v1;
    S.z[i] = S.zp[i] + S.dt * v2;
}

// Internal force of node i (boundary nodes: sum of the tile partials in tile
// order, written back so f_int is complete).
template <typename R>
__device__ __forceinline__ void node_force(const FOArgs& S, const TileArgs<R>& A, int i, double f[3]) {
    const int b = S.node_bidx[i];
    if (b < 0) {
        f[0] = (double)A.f_out[3 * i + 0];
        f[1] = (double)A.f_out[3 * i + 1];
        f[2] = (double)A.f_out[3 * i + 2];
    } else {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;  // node sums in FP64 (near equilibrium they cancel)
        for (int k = S.bnode_off[b]; k < S.bnode_off[b + 1]; ++k) {
            const int p = S.bnode_slots[k];
            s0 += A.partial[3 * p + 0];
            s1 += A.partial[3 * p + 1];
            s2 += A.partial[3 * p + 2];
        }
        A.f_out[3 * i + 0] = s0;
        A.f_out[3 * i + 1] = s1;
        A.f_out[3 * i + 2] = s2;
        f[0] = (double)s0;
        f[1] = (double)s1;
        f[2] = (double)s2;
    }
}

// solver_grad_L (SyncedNesterov.cu:32-95) for the 3 DOFs of node i.  With
// MASS the force f already holds M (v - v_prev) / dt (added element by element in
// the force phase) and the mass-row pass is skipped.
template <bool MASS>
__device__ __forceinline__ void grad_node(const FOArgs& S, int i, const double f[3], double gi[3]) {
    const double inv_dt = 1.0 / S.dt;
    double r[3] = {0.0, 0.0, 0.0};
    for (int k = MASS ? 0 : S.m_off[i]; k < (MASS ? 0 : S.m_off[i + 1]); ++k) {
        const int j = S.m_col[k];
        const double mij = S.m_val[k];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double vd = S.vg[3 * j + d] - S.vp[3 * j + d];
            r[d] += mij * vd * inv_dt;
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        r[d] -= (-f[d]);
        r[d] -= S.f_ext[3 * i + d];
        if (S.nc > 0) {
            const int t = 3 * i + d;
            for (int k = S.jt_off[t]; k < S.jt_off[t + 1]; ++k) {
                const int ci = S.jt_col[k];
                r[d] += S.dt * 1.0 * (S.lam[ci] + S.rho * S.c[ci]);
            }
        }
        gi[d] = r[d];
    }
}

template <typename R, int NPE, int NQP, bool DAMP, bool MR, bool MASS>
__device__ __forceinline__ void force_phase(const FOArgs& S, const TileArgs<R>& A, unsigned char* smem) {
    for (int tile = blockIdx.x; tile < S.n_tiles; tile += gridDim.x)
        process_tile<R, NPE, NQP, TILE_FORCE, DAMP, MR, MASS>(A, tile, smem);
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    for (int k = gt; k < S.n_fixed; k += gs) {
        const int n = S.fixed[k];
        S.c[3 * k + 0] = S.x[n] - S.xj[n];
        S.c[3 * k + 1] = S.y[n] - S.yj[n];
        S.c[3 * k + 2] = S.z[n] - S.zj[n];
    }
}

template <typename R, int NPE, int NQP, bool DAMP, bool MR, bool MASS>
__global__ void __launch_bounds__(TILE_ELEMS) k_first_order(FOArgs S, TileArgs<R> A) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double red_sh[32];
    __shared__ double fold_sh;
    cg::grid_group grid = cg::this_grid();
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    const int N = S.N, n3 = 3 * N;
    const bool nesterov = (S.kind == KIND_NESTEROV);
    const bool nocoop = (S.kind == KIND_ADAMW_NOCOOP);
    const int check = S.check > 0 ? S.check : 1;
    const int eff_outer = (nocoop && S.nc == 0) ? 1 : S.max_outer;

    const bool rule = S.rel_tol > 0.0;
    double sf = 0.0;
    for (int i = gt; i < N; i += gs) {
        S.xp[i] = S.x[i];
        S.yp[i] = S.y[i];
        S.zp[i] = S.z[i];
        if (rule)
#pragma unroll
            for (int d = 0; d < 3; ++d) sf += S.f_ext[3 * i + d] * S.f_ext[3 * i + d];
    }
    if (rule) write_partial(S, 5, sf, red_sh);
    grid.sync();
    const double fext_norm = rule ? sqrt(fold_partials(S, 5, &fold_sh)) : 0.0;

    int outer_flag = 0, status = 0, n_outer = 0, inner_total = 0, last_inner = 0, rule_met = 0;
    double last_norm = 0.0, last_rel = -1.0;
    for (int outer = 0; outer < eff_outer && !outer_flag && !status; ++outer) {
        ++n_outer;
        double t = 1.0, prev_norm_g = 0.0, norm_g = 0.0, norm_g0 = -1.0, lr = S.lr;
        int inner_flag = 0, inner_count = 0;
        for (int i = gt; i < n3; i += gs) {
            if (nesterov) {
                S.vk[i] = S.vg[i];
                S.vkm1[i] = S.vg[i];
            } else {
                S.g[i] = 0.0;
                S.m[i] = 0.0;
                S.va[i] = 0.0;
            }
        }
        grid.sync();
        for (int inner = 0; inner < S.max_inner && !inner_flag; ++inner) {
            ++inner_count;
            // ---- P1: new velocity guess and scratch positions
            if (nesterov) {
                const double t_next = 0.5 * (1.0 + sqrt(1.0 + 4.0 * t * t));
                const double beta = (t - 1.0) / t_next;
                for (int i = gt; i < N; i += gs) {
                    double v[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const double vk = S.vk[3 * i + d];
                        v[d] = vk + beta * (vk - S.vkm1[3 * i + d]);
                        S.vg[3 * i + d] = v[d];
                    }
                    set_node_positions<R>(S, i, v[0], v[1], v[2]);
                }
                t = t_next;
            } else {
                double lr_cur, b1t, b2t;
                if (nocoop) {
                    lr_cur = S.lr * pow(S.lr_decay, inner + 1);
                    const double tc = (double)(inner + 2);
                    b1t = 1.0 / (1.0 - pow(S.beta1, tc));
                    b2t = 1.0 / (1.0 - pow(S.beta2, tc));
                } else {
                    lr = lr * S.lr_decay;
                    t += 1;
                    lr_cur = lr;
                    b1t = 1 - pow(S.beta1, t);
                    b2t = 1 - pow(S.beta2, t);
                }
                for (int i = gt; i < N; i += gs) {
                    double v[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const int k = 3 * i + d;
                        const double gk = S.g[k], vgk = S.vg[k];
                        const double mt = S.beta1 * S.m[k] + (1 - S.beta1) * gk;
                        const double vt = S.beta2 * S.va[k] + (1 - S.beta2) * gk * gk;
                        double mh, vh;
                        if (nocoop) {
                            mh = mt * b1t;
                            vh = vt * b2t;
                        } else {
                            mh = mt / b1t;
                            vh = vt / b2t;
                        }
                        v[d] = vgk - lr_cur * (mh / (sqrt(vh) + S.eps) + S.wd * vgk);
                        S.m[k] = mt;
                        S.va[k] = vt;
                        S.vg[k] = v[d];
                    }
                    set_node_positions<R>(S, i, v[0], v[1], v[2]);
                }
            }
            grid.sync();
            // ---- P2: internal force (fused tiles) and constraint values
            force_phase<R, NPE, NQP, DAMP, MR, MASS>(S, A, smem);
            grid.sync();
            // ---- P3: gradient per node and the norm partials
            const bool do_check = nesterov || (inner % check == 0);
            double sg = 0.0, sv = 0.0, sr = 0.0;
            for (int i = gt; i < N; i += gs) {
                double f[3], gi[3];
                node_force<R>(S, A, i, f);
                grad_node<MASS>(S, i, f, gi);
                const bool free_node = rule && !S.node_fixed[i];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    S.g[3 * i + d] = gi[d];
                    sg += gi[d] * gi[d];
                    if (!nesterov) sv += S.vg[3 * i + d] * S.vg[3 * i + d];
                    if (free_node) {
                        const double rd = f[d] - S.f_ext[3 * i + d];
                        sr += rd * rd;
                    }
                }
            }
            if (do_check) {
                write_partial(S, 0, sg, red_sh);
                if (!nesterov) write_partial(S, 1, sv, red_sh);
                if (rule) write_partial(S, 4, sr, red_sh);
            }
            grid.sync();
            bool rule_now = false;
            if (rule && do_check) {
                const double rr = sqrt(fold_partials(S, 4, &fold_sh));
                last_rel = fext_norm > 0.0 ? rr / fext_norm : rr;
                rule_now = last_rel < S.rel_tol;
            }
            if (nesterov) {
                // ---- P4: ||g|| test, v_next = y - alpha g, norm partials of v_next and v_k
                norm_g = sqrt(fold_partials(S, 0, &fold_sh));
                if (!isfinite(norm_g)) status = TLFEA_NONFINITE;
                if (rule_now) {
                    // stop at the positions the residual was measured at (v = y)
                    inner_flag = 1;
                    rule_met = 1;
                    break;
                }
                if (inner > 0 && fabs(norm_g - prev_norm_g) < S.inner_tol) inner_flag = 1;
                double snv = 0.0, snk = 0.0;
                for (int i = gt; i < n3; i += gs) {
                    const double vn = S.vg[i] - S.alpha * S.g[i];
                    const double vk = S.vk[i];
                    snv += vn * vn;
                    snk += vk * vk;
                    S.vkm1[i] = vk;
                    S.vk[i] = vn;
                    S.vg[i] = vn;
                }
                write_partial(S, 1, snv, red_sh);
                write_partial(S, 2, snk, red_sh);
                grid.sync();
                const double nvn = sqrt(fold_partials(S, 1, &fold_sh));
                const double nvk = sqrt(fold_partials(S, 2, &fold_sh));
                if (inner > 0 && fabs(nvn - nvk) < S.inner_tol) inner_flag = 1;
                prev_norm_g = norm_g;
            } else if (do_check) {
                norm_g = sqrt(fold_partials(S, 0, &fold_sh));
                const double nv = sqrt(fold_partials(S, 1, &fold_sh));
                if (!isfinite(norm_g)) status = TLFEA_NONFINITE;
                if (norm_g0 < 0.0) norm_g0 = norm_g;
                const double tol_abs = S.inner_tol * (1.0 + nv);
                const double tol_rel = (S.rtol > 0.0 && norm_g0 > 0.0) ? (S.rtol * norm_g0) : 0.0;
                if (norm_g <= tol_abs || (tol_rel > 0.0 && norm_g <= tol_rel)) inner_flag = 1;
                if (rule_now) {
                    inner_flag = 1;
                    rule_met = 1;
                }
            }
            if (status) break;
        }
        inner_total += inner_count;
        last_inner = inner_count;
        last_norm = norm_g;
        if (status) break;
        // ---- outer update: v_prev, positions, constraints, multipliers
        for (int i = gt; i < N; i += gs) {
            double v[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                v[d] = S.vg[3 * i + d];
                S.vp[3 * i + d] = v[d];
            }
            set_node_positions<R>(S, i, v[0], v[1], v[2]);
        }
        grid.sync();
        double sc = 0.0;
        for (int k = gt; k < S.n_fixed; k += gs) {
            const int n = S.fixed[k];
            const double cc[3] = {S.x[n] - S.xj[n], S.y[n] - S.yj[n], S.z[n] - S.zj[n]};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                S.c[3 * k + d] = cc[d];
                S.lam[3 * k + d] += S.rho * S.dt * cc[d];
                sc += cc[d] * cc[d];
            }
        }
        write_partial(S, 3, sc, red_sh);
        grid.sync();
        const double norm_c = sqrt(fold_partials(S, 3, &fold_sh));
        if (rule_met) {
            outer_flag = 1;
        } else if (nocoop) {
            if (S.nc > 0 && norm_c < S.outer_tol && inner_flag) outer_flag = 1;
        } else if (fabs(norm_c) < S.outer_tol) {
            outer_flag = 1;
        }
    }
    // final positions x = x_prev + dt v
    for (int i = gt; i < N; i += gs) set_node_positions<R>(S, i, S.vg[3 * i], S.vg[3 * i + 1], S.vg[3 * i + 2]);
    if (gt == 0) {
        S.stat[0] = n_outer;
        S.stat[1] = inner_total;
        S.stat[2] = last_inner;
        S.stat[3] = status;
        *S.stat_norm = last_norm;
        *S.stat_rel = last_rel;
        S.stat[8] = rule_met;
    }
}

// ---------------------------------------------------------------------------
// Per-phase solve (mode 0, the default).  The persistent kernel above holds 2
// blocks (8 warps) per SM -- its registers are the force tile routine's -- so its
// node phases run latency-bound.  Here every phase is its own launch at the
// occupancy its code allows, and the control flow of the reference's loops
// (inner stop tests, outer multiplier updates, the stop rule) lives in a small
// device-side state record, FOCtl, advanced by the last block to finish each
// phase (a ticket; the norms are folded in block order, so deterministically).
// A slot of launches -- outer start, velocity guess, forces, gradient, Nesterov
// update, outer update (two), final positions -- covers every state; each kernel
// returns at entry unless the state is its own, so a CUDA graph of a chunk of
// slots is replayed until the state reads FO_DONE.  Per node and per tile the
// arithmetic is the persistent kernel's, so with fixed iteration counts the
// trajectories are bitwise the same; norms group their partials per launch grid.
enum { FO_OUTER_START = 0, FO_INNER = 1, FO_OUTER = 2, FO_FINAL = 3, FO_DONE = 4 };

struct FOCtl {
    int mode, outer, inner, inner_flag, outer_flag, status, n_outer, inner_total, last_inner, rule_met;
    unsigned int ticket;
    int pad;
    double t, lr, prev_norm_g, norm_g, norm_g0, last_norm, last_rel, fext_norm;
    double beta, lr_cur, b1t, b2t;  // scalars of the current inner iteration
};

constexpr int FO_NODE_THREADS = 256;

__device__ __forceinline__ int fo_eff_outer(const FOArgs& S) {
    return (S.kind == KIND_ADAMW_NOCOOP && S.nc == 0) ? 1 : S.max_outer;
}

// True in every thread of the block that finishes the phase last (all other blocks'
// partials and writes are visible to it).
__device__ __forceinline__ bool fo_last_block(FOCtl* C, int* flag_sh) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int tk = atomicAdd(&C->ticket, 1u);
        const int last = (tk == gridDim.x - 1) ? 1 : 0;
        if (last) {
            C->ticket = 0u;
            __threadfence();
        }
        *flag_sh = last;
    }
    __syncthreads();
    return *flag_sh != 0;
}

// The scalars of inner iteration C->inner, as the persistent kernel forms them at
// the top of its inner loop (one thread).
__device__ __forceinline__ void fo_scalars(const FOArgs& S, FOCtl* C) {
    if (S.kind == KIND_NESTEROV) {
        const double t_next = 0.5 * (1.0 + sqrt(1.0 + 4.0 * C->t * C->t));
        C->beta = (C->t - 1.0) / t_next;
        C->t = t_next;
    } else if (S.kind == KIND_ADAMW_NOCOOP) {
        C->lr_cur = S.lr * pow(S.lr_decay, C->inner + 1);
        const double tc = (double)(C->inner + 2);
        C->b1t = 1.0 / (1.0 - pow(S.beta1, tc));
        C->b2t = 1.0 / (1.0 - pow(S.beta2, tc));
    } else {
        C->lr = C->lr * S.lr_decay;
        C->t += 1;
        C->lr_cur = C->lr;
        C->b1t = 1 - pow(S.beta1, C->t);
        C->b2t = 1 - pow(S.beta2, C->t);
    }
}

// End of inner iteration C->inner (one thread): leave the inner loop on a flag, a
// non-finite norm or the iteration cap, else set up the next iteration.
__device__ __forceinline__ void fo_end_inner(const FOArgs& S, FOCtl* C) {
    const int count = C->inner + 1;
    if (C->status || C->inner_flag || count >= S.max_inner) {
        C->inner_total += count;
        C->last_inner = count;
        C->last_norm = C->norm_g;
        C->mode = C->status ? FO_FINAL : FO_OUTER;
    } else {
        C->inner = count;
        fo_scalars(S, C);
    }
}

// x_prev = x, ||f_ext||^2 (stop rule), the start state.
__global__ void __launch_bounds__(FO_NODE_THREADS) k_fo_start(FOArgs S, FOCtl* C) {
    __shared__ double red_sh[32];
    __shared__ double fold_sh;
    __shared__ int flag_sh;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    const bool rule = S.rel_tol > 0.0;
    double sf = 0.0;
    for (int i = gt; i < S.N; i += gs) {
        S.xp[i] = S.x[i];
        S.yp[i] = S.y[i];
        S.zp[i] = S.z[i];
        if (rule)
#pragma unroll
            for (int d = 0; d < 3; ++d) sf += S.f_ext[3 * i + d] * S.f_ext[3 * i + d];
    }
    if (rule) write_partial(S, 5, sf, red_sh);
    if (!fo_last_block(C, &flag_sh)) return;
    const double fn = rule ? sqrt(fold_partials(S, 5, &fold_sh)) : 0.0;
    if (threadIdx.x == 0) {
        C->fext_norm = fn;
        C->outer = C->inner = C->inner_flag = C->outer_flag = C->status = 0;
        C->n_outer = C->inner_total = C->last_inner = C->rule_met = 0;
        C->norm_g = C->last_norm = 0.0;
        C->last_rel = -1.0;
        C->mode = (fo_eff_outer(S) > 0) ? FO_OUTER_START : FO_FINAL;
    }
}

// Start of an outer iteration: the inner loop's vectors and scalars.
__global__ void __launch_bounds__(FO_NODE_THREADS) k_fo_outer_start(FOArgs S, FOCtl* C) {
    __shared__ int flag_sh;
    if (__ldcg(&C->mode) != FO_OUTER_START) return;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    const bool nesterov = (S.kind == KIND_NESTEROV);
    for (int i = gt; i < 3 * S.N; i += gs) {
        if (nesterov) {
            S.vk[i] = S.vg[i];
            S.vkm1[i] = S.vg[i];
        } else {
            S.g[i] = 0.0;
            S.m[i] = 0.0;
            S.va[i] = 0.0;
        }
    }
    if (!fo_last_block(C, &flag_sh) || threadIdx.x != 0) return;
    C->n_outer += 1;
    C->t = 1.0;
    C->prev_norm_g = 0.0;
    C->norm_g = 0.0;
    C->norm_g0 = -1.0;
    C->lr = S.lr;
    C->inner_flag = 0;
    C->inner = 0;
    if (S.max_inner > 0) {
        fo_scalars(S, C);
        C->mode = FO_INNER;
    } else {
        C->last_inner = 0;
        C->last_norm = C->norm_g;
        C->mode = FO_OUTER;
    }
}

// P1: the inner iteration's velocity guess and positions.
template <typename R>
__global__ void __launch_bounds__(FO_NODE_THREADS) k_fo_guess(FOArgs S, const FOCtl* C) {
    if (__ldcg(&C->mode) != FO_INNER) return;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    if (S.kind == KIND_NESTEROV) {
        const double beta = __ldcg(&C->beta);
        for (int i = gt; i < S.N; i += gs) {
            double v[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double vk = S.vk[3 * i + d];
                v[d] = vk + beta * (vk - S.vkm1[3 * i + d]);
                S.vg[3 * i + d] = v[d];
            }
            set_node_positions<R>(S, i, v[0], v[1], v[2]);
        }
        return;
    }
    const bool nocoop = (S.kind == KIND_ADAMW_NOCOOP);
    const double lr_cur = __ldcg(&C->lr_cur), b1t = __ldcg(&C->b1t), b2t = __ldcg(&C->b2t);
    for (int i = gt; i < S.N; i += gs) {
        double v[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int k = 3 * i + d;
            const double gk = S.g[k], vgk = S.vg[k];
            const double mt = S.beta1 * S.m[k] + (1 - S.beta1) * gk;
            const double vt = S.beta2 * S.va[k] + (1 - S.beta2) * gk * gk;
            double mh, vh;
            if (nocoop) {
                mh = mt * b1t;
                vh = vt * b2t;
            } else {
                mh = mt / b1t;
                vh = vt / b2t;
            }
            v[d] = vgk - lr_cur * (mh / (sqrt(vh) + S.eps) + S.wd * vgk);
            S.m[k] = mt;
            S.va[k] = vt;
            S.vg[k] = v[d];
        }
        set_node_positions<R>(S, i, v[0], v[1], v[2]);
    }
}

// P2: internal force, one tile per block (the fused tile routine), and the
// constraint values at the new positions.
// TET10 SVK without damping fits 3 blocks per SM in FP64 (168 registers) and 4 in
// FP32 (128); the other variants keep the registers they need.
template <typename R, int NPE, int NQP, bool DAMP, bool MR, bool MASS>
__global__ void __launch_bounds__(TILE_ELEMS, (DAMP || MR || NPE != 10) ? 1 : (sizeof(R) == 4 ? 4 : 3))
    k_fo_force(FOArgs S, TileArgs<R> A, const FOCtl* C) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (__ldcg(&C->mode) != FO_INNER) return;
    process_tile<R, NPE, NQP, TILE_FORCE, DAMP, MR, MASS>(A, blockIdx.x, smem);
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    for (int k = gt; k < S.n_fixed; k += gs) {
        const int n = S.fixed[k];
        S.c[3 * k + 0] = S.x[n] - S.xj[n];
        S.c[3 * k + 1] = S.y[n] - S.yj[n];
        S.c[3 * k + 2] = S.z[n] - S.zj[n];
    }
}

// P3: the gradient per node and its norm partials; the last block applies the
// stop tests (AdamW: all of them; Nesterov: the stop rule, which skips the update,
// and the ||g|| test).
template <typename R, bool MASS>
__global__ void __launch_bounds__(FO_NODE_THREADS) k_fo_grad(FOArgs S, TileArgs<R> A, FOCtl* C) {
    __shared__ double red_sh[32];
    __shared__ double fold_sh;
    __shared__ int flag_sh;
    if (__ldcg(&C->mode) != FO_INNER) return;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    const bool nesterov = (S.kind == KIND_NESTEROV);
    const bool rule = S.rel_tol > 0.0;
    const int check = S.check > 0 ? S.check : 1;
    const int inner = __ldcg(&C->inner);
    const bool do_check = nesterov || (inner % check == 0);
    double sg = 0.0, sv = 0.0, sr = 0.0;
    for (int i = gt; i < S.N; i += gs) {
        double f[3], gi[3];
        node_force<R>(S, A, i, f);
        grad_node<MASS>(S, i, f, gi);
        const bool free_node = rule && !S.node_fixed[i];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            S.g[3 * i + d] = gi[d];
            sg += gi[d] * gi[d];
            if (!nesterov) sv += S.vg[3 * i + d] * S.vg[3 * i + d];
            if (free_node) {
                const double rd = f[d] - S.f_ext[3 * i + d];
                sr += rd * rd;
            }
        }
    }
    if (do_check) {
        write_partial(S, 0, sg, red_sh);
        if (!nesterov) write_partial(S, 1, sv, red_sh);
        if (rule) write_partial(S, 4, sr, red_sh);
    }
    if (!fo_last_block(C, &flag_sh)) return;
    bool rule_now = false;
    double rr = 0.0, norm_g = 0.0, nv = 0.0;
    if (rule && do_check) rr = sqrt(fold_partials(S, 4, &fold_sh));
    if (nesterov || do_check) norm_g = sqrt(fold_partials(S, 0, &fold_sh));
    if (!nesterov && do_check) nv = sqrt(fold_partials(S, 1, &fold_sh));
    if (threadIdx.x != 0) return;
    if (rule && do_check) {
        C->last_rel = C->fext_norm > 0.0 ? rr / C->fext_norm : rr;
        rule_now = C->last_rel < S.rel_tol;
    }
    if (nesterov) {
        C->norm_g = norm_g;
        if (!isfinite(norm_g)) C->status = TLFEA_NONFINITE;
        if (rule_now) {
            // stop at the positions the residual was measured at (v = y)
            C->inner_flag = 1;
            C->rule_met = 1;
            fo_end_inner(S, C);
            return;
        }
        if (inner > 0 && fabs(norm_g - C->prev_norm_g) < S.inner_tol) C->inner_flag = 1;
        return;  // the update and the rest of the tests follow in k_fo_nesterov
    }
    if (do_check) {
        C->norm_g = norm_g;
        if (!isfinite(norm_g)) C->status = TLFEA_NONFINITE;
        if (C->norm_g0 < 0.0) C->norm_g0 = norm_g;
        const double tol_abs = S.inner_tol * (1.0 + nv);
        const double tol_rel = (S.rtol > 0.0 && C->norm_g0 > 0.0) ? (S.rtol * C->norm_g0) : 0.0;
        if (norm_g <= tol_abs || (tol_rel > 0.0 && norm_g <= tol_rel)) C->inner_flag = 1;
        if (rule_now) {
            C->inner_flag = 1;
            C->rule_met = 1;
        }
    }
    fo_end_inner(S, C);
}

// P4 (Nesterov): v_next = y - alpha g, and the ||v_next|| - ||v_k|| test.
__global__ void __launch_bounds__(FO_NODE_THREADS) k_fo_nesterov(FOArgs S, FOCtl* C) {
    __shared__ double red_sh[32];
    __shared__ double fold_sh;
    __shared__ int flag_sh;
    if (__ldcg(&C->mode) != FO_INNER) return;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    double snv = 0.0, snk = 0.0;
    for (int i = gt; i < 3 * S.N; i += gs) {
        const double vn = S.vg[i] - S.alpha * S.g[i];
        const double vk = S.vk[i];
        snv += vn * vn;
        snk += vk * vk;
        S.vkm1[i] = vk;
        S.vk[i] = vn;
        S.vg[i] = vn;
    }
    write_partial(S, 1, snv, red_sh);
    write_partial(S, 2, snk, red_sh);
    if (!fo_last_block(C, &flag_sh)) return;
    const double nvn = sqrt(fold_partials(S, 1, &fold_sh));
    const double nvk = sqrt(fold_partials(S, 2, &fold_sh));
    if (threadIdx.x != 0) return;
    if (C->inner > 0 && fabs(nvn - nvk) < S.inner_tol) C->inner_flag = 1;
    C->prev_norm_g = C->norm_g;
    fo_end_inner(S, C);
}

// Outer update, part 1: v_prev = v and x = x_prev + dt v.
template <typename R>
__global__ void __launch_bounds__(FO_NODE_THREADS) k_fo_outer_positions(FOArgs S, const FOCtl* C) {
    if (__ldcg(&C->mode) != FO_OUTER) return;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    for (int i = gt; i < S.N; i += gs) {
        double v[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v[d] = S.vg[3 * i + d];
            S.vp[3 * i + d] = v[d];
        }
        set_node_positions<R>(S, i, v[0], v[1], v[2]);
    }
}

// Outer update, part 2: constraints, multipliers and the outer stop test.
__global__ void __launch_bounds__(FO_NODE_THREADS) k_fo_outer_multipliers(FOArgs S, FOCtl* C) {
    __shared__ double red_sh[32];
    __shared__ double fold_sh;
    __shared__ int flag_sh;
    if (__ldcg(&C->mode) != FO_OUTER) return;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    double sc = 0.0;
    for (int k = gt; k < S.n_fixed; k += gs) {
        const int n = S.fixed[k];
        const double cc[3] = {S.x[n] - S.xj[n], S.y[n] - S.yj[n], S.z[n] - S.zj[n]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            S.c[3 * k + d] = cc[d];
            S.lam[3 * k + d] += S.rho * S.dt * cc[d];
            sc += cc[d] * cc[d];
        }
    }
    write_partial(S, 3, sc, red_sh);
    if (!fo_last_block(C, &flag_sh)) return;
    const double norm_c = sqrt(fold_partials(S, 3, &fold_sh));
    if (threadIdx.x != 0) return;
    if (C->rule_met) {
        C->outer_flag = 1;
    } else if (S.kind == KIND_ADAMW_NOCOOP) {
        if (S.nc > 0 && norm_c < S.outer_tol && C->inner_flag) C->outer_flag = 1;
    } else if (fabs(norm_c) < S.outer_tol) {
        C->outer_flag = 1;
    }
    if (C->outer_flag || C->outer + 1 >= fo_eff_outer(S)) {
        C->mode = FO_FINAL;
    } else {
        C->outer += 1;
        C->mode = FO_OUTER_START;
    }
}

// Final positions x = x_prev + dt v and the statistics.
template <typename R>
__global__ void __launch_bounds__(FO_NODE_THREADS) k_fo_final(FOArgs S, FOCtl* C) {
    __shared__ int flag_sh;
    if (__ldcg(&C->mode) != FO_FINAL) return;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    for (int i = gt; i < S.N; i += gs) set_node_positions<R>(S, i, S.vg[3 * i], S.vg[3 * i + 1], S.vg[3 * i + 2]);
    if (!fo_last_block(C, &flag_sh) || threadIdx.x != 0) return;
    S.stat[0] = C->n_outer;
    S.stat[1] = C->inner_total;
    S.stat[2] = C->last_inner;
    S.stat[3] = C->status;
    *S.stat_norm = C->last_norm;
    *S.stat_rel = C->last_rel;
    S.stat[8] = C->rule_met;
    C->mode = FO_DONE;
}

template <typename R, int NPE, int NQP, bool DAMP, bool MR, bool MASS>
static int launch_first_order(tlfea_solver_s* s, FOArgs& S, TileArgs<R>& A) {
    tlfea_element_s* el = s->el;
    auto kern = k_first_order<R, NPE, NQP, DAMP, MR, MASS>;
    const size_t smem = tile_smem_bytes<R>(NPE, el->tl.max_local, DAMP, MASS);
    if (smem > 48 * 1024) TLFEA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, sms = 0;
    TLFEA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TILE_ELEMS, smem));
    TLFEA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, el->device));
    if (per_sm < 1) {
        set_error("persistent solver kernel does not fit on an SM");
        return TLFEA_UNSUPPORTED;
    }
    int blocks = std::min(per_sm * sms, s->max_blocks);
    const int need = std::max((3 * el->N + TILE_ELEMS - 1) / TILE_ELEMS, el->tl.n_tiles);
    blocks = std::max(1, std::min(blocks, need));
    void* args[] = {(void*)&S, (void*)&A};
    TLFEA_CUDA(cudaLaunchCooperativeKernel((const void*)kern, blocks, TILE_ELEMS, args, smem, el->stream));
    TLFEA_LAUNCHED(1);
    return TLFEA_OK;
}

void first_order_drop_graphs(tlfea_solver_s* s);

// One slot of per-phase launches (every state's kernels, each a no-op unless the
// state is its own).
template <typename R, int NPE, int NQP, bool DAMP, bool MR, bool MASS>
static void fo_enqueue_slot(const tlfea_solver_s* s, const FOArgs& S, const TileArgs<R>& A, FOCtl* C,
                            cudaStream_t st) {
    const int gn = std::max(1, std::min(s->max_blocks, (S.N + FO_NODE_THREADS - 1) / FO_NODE_THREADS));
    // the outer-step kernels do their work once per outer iteration and are no-ops in
    // every inner slot: a small grid keeps the no-op launches short
    const int go = std::min(gn, std::max(1, s->max_blocks / 8));  // two blocks per SM
    const size_t smem = tile_smem_bytes<R>(NPE, A.max_local, DAMP, MASS);
    k_fo_outer_start<<<go, FO_NODE_THREADS, 0, st>>>(S, C);
    k_fo_guess<R><<<gn, FO_NODE_THREADS, 0, st>>>(S, C);
    k_fo_force<R, NPE, NQP, DAMP, MR, MASS><<<S.n_tiles, TILE_ELEMS, smem, st>>>(S, A, C);
    k_fo_grad<R, MASS><<<gn, FO_NODE_THREADS, 0, st>>>(S, A, C);
    if (S.kind == KIND_NESTEROV) k_fo_nesterov<<<gn, FO_NODE_THREADS, 0, st>>>(S, C);
    k_fo_outer_positions<R><<<go, FO_NODE_THREADS, 0, st>>>(S, C);
    k_fo_outer_multipliers<<<go, FO_NODE_THREADS, 0, st>>>(S, C);
    k_fo_final<R><<<go, FO_NODE_THREADS, 0, st>>>(S, C);
}

// One Solve() in per-phase launches: the start kernel, then graph chunks of slots
// (8, then 32) until the state reads FO_DONE.  The chunks are captured once per
// (arguments, kernel variant) and kept.
template <typename R, int NPE, int NQP, bool DAMP, bool MR, bool MASS>
static int run_phased(tlfea_solver_s* s, const FOArgs& S, const TileArgs<R>& A, cudaStream_t st) {
    auto kern = k_fo_force<R, NPE, NQP, DAMP, MR, MASS>;
    const size_t smem = tile_smem_bytes<R>(NPE, A.max_local, DAMP, MASS);
    if (smem > 48 * 1024) TLFEA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    FOCtl* C = static_cast<FOCtl*>(s->fo_ctl);
    // the chunks bake in S, A and the kernel variant: recapture when any differs
    const int variant = (sizeof(R) == 4 ? 1 : 0) | (NPE == 10 ? 2 : 0) | (DAMP ? 4 : 0) | (MR ? 8 : 0) | (MASS ? 16 : 0);
    std::vector<unsigned char> key(sizeof(int) + sizeof(FOArgs) + sizeof(TileArgs<R>));
    memcpy(key.data(), &variant, sizeof(int));
    memcpy(key.data() + sizeof(int), &S, sizeof(FOArgs));
    memcpy(key.data() + sizeof(int) + sizeof(FOArgs), &A, sizeof(TileArgs<R>));
    if (key != s->fo_graph_key) {
        first_order_drop_graphs(s);
        const int slots[2] = {8, 32};
        for (int k = 0; k < 2; ++k) {
            cudaGraph_t g = nullptr;
            TLFEA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            for (int j = 0; j < slots[k]; ++j) fo_enqueue_slot<R, NPE, NQP, DAMP, MR, MASS>(s, S, A, C, st);
            const cudaError_t e1 = cudaGetLastError();
            const cudaError_t e2 = cudaStreamEndCapture(st, &g);
            cudaGraphExec_t ge = nullptr;
            const cudaError_t e3 = (e1 == cudaSuccess && e2 == cudaSuccess) ? cudaGraphInstantiate(&ge, g, 0) : e2;
            if (g) cudaGraphDestroy(g);
            if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
                cudaGetLastError();
                first_order_drop_graphs(s);
                set_error("first-order solve: capture of the per-phase chunk failed");
                return TLFEA_CUDA_ERROR;
            }
            s->fo_graph[k] = ge;
        }
        s->fo_graph_key = key;
    }
    const int gn = std::max(1, std::min(s->max_blocks, (S.N + FO_NODE_THREADS - 1) / FO_NODE_THREADS));
    k_fo_start<<<gn, FO_NODE_THREADS, 0, st>>>(S, C);
    TLFEA_CUDA(cudaGetLastError());
    TLFEA_LAUNCHED(1);
    // every slot advances the state by at least one phase: a bound on the replays
    const long long max_slots = 4 + (long long)std::max(S.max_outer, 1) * ((long long)std::max(S.max_inner, 0) + 2);
    long long slots = 0;
    const int per_slot = (S.kind == KIND_NESTEROV) ? 8 : 7;
    for (int k = 0;; k = 1) {
        TLFEA_CUDA(cudaGraphLaunch(s->fo_graph[k], st));
        TLFEA_LAUNCHED(per_slot * (k ? 32 : 8));
        slots += k ? 32 : 8;
        int mode = 0;
        TLFEA_CUDA(cudaMemcpyAsync(&mode, &C->mode, sizeof(int), cudaMemcpyDeviceToHost, st));
        TLFEA_CUDA(cudaStreamSynchronize(st));
        if (mode == FO_DONE) break;
        if (slots > max_slots) {
            set_error("first-order solve: the per-phase loop did not finish within its iteration bounds");
            return TLFEA_CUDA_ERROR;
        }
    }
    return TLFEA_OK;
}

int first_order_alloc(tlfea_solver_s* s) {
    tlfea_element_s* el = s->el;
    const size_t n3 = 3 * (size_t)el->N, N = el->N;
    int st = 0;
    st |= dalloc(&s->v_guess, n3) | dalloc(&s->v_prev, n3) | dalloc(&s->v_k, n3) | dalloc(&s->v_km1, n3);
    st |= dalloc(&s->g, n3) | dalloc(&s->m, n3) | dalloc(&s->va, n3);
    st |= dalloc(&s->lam, (size_t)std::max(s->n_constraints, 1));
    st |= dalloc(&s->xp, N) | dalloc(&s->yp, N) | dalloc(&s->zp, N);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, el->device);
    s->max_blocks = std::max(1, sms * 16);
    st |= dalloc(&s->red, (size_t)6 * s->max_blocks);
    st |= dalloc(&s->dstat, 16);
    st |= dalloc(&s->node_fixed, N);
    if (cudaMalloc(&s->fo_ctl, sizeof(FOCtl)) != cudaSuccess) st = 1;
    else if (cudaMemset(s->fo_ctl, 0, sizeof(FOCtl)) != cudaSuccess) st = 1;
    if (st) return TLFEA_CUDA_ERROR;
    return TLFEA_OK;
}

void first_order_drop_graphs(tlfea_solver_s* s) {
    for (auto& g : s->fo_graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    s->fo_graph_key.clear();
}

void first_order_free(tlfea_solver_s* s) {
    dfree(s->v_guess); dfree(s->v_prev); dfree(s->v_k); dfree(s->v_km1);
    dfree(s->g); dfree(s->m); dfree(s->va); dfree(s->lam);
    dfree(s->xp); dfree(s->yp); dfree(s->zp);
    dfree(s->red); dfree(s->dstat); dfree(s->node_fixed);
    first_order_drop_graphs(s);
    if (s->fo_ctl) cudaFree(s->fo_ctl);
    s->fo_ctl = nullptr;
}

// f_ext = f_base + a * f_var, rounded multiply then rounded add (no fused
// multiply-add), so a host loop computing the same load in FP64 matches bitwise.
__global__ void k_step_load(int n3, const double* __restrict__ f_base, const double* __restrict__ f_var,
                            double a, double* __restrict__ f_ext) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n3) f_ext[i] = __dadd_rn(f_base[i], __dmul_rn(a, f_var[i]));
}

static int first_order_finish(tlfea_solver_s* s, const std::vector<int>& hs, int n_steps, int* inner_iters,
                              float ms, bool fp32);

// One Solve(), or n implicit steps with a time-varying load (new).
int first_order_steps(tlfea_solver_s* s, int steps, const StepLoad* load, int* inner_iters) {
    tlfea_element_s* el = s->el;
    if (!el->is_setup) {
        set_error("element must be set up first");
        return TLFEA_NOT_SETUP;
    }
    if (!s->params_set) {
        set_error("SetParameters must be called before Solve");
        return TLFEA_NOT_SETUP;
    }
    if (!el->mass_setup) {
        set_error("CalcMassMatrix must be called before Solve");
        return TLFEA_NOT_SETUP;
    }
    if (s->n_constraints != el->n_constraint) {
        set_error("solver constraint count differs from the element's");
        return TLFEA_SIZE_MISMATCH;
    }
    int st;
    if (el->n_constraint > 0 && !el->jt_setup) {
        if ((st = tlfea_element_build_constraint_jact_csr(el))) return st;
    }
    const bool fp32 = (el->precision == TLFEA_PRECISION_FP32);
    FOArgs S;
    memset(&S, 0, sizeof(S));
    S.kind = s->kind;
    S.N = el->N;
    S.nc = el->n_constraint;
    S.n_fixed = el->n_constraint / 3;
    S.n_tiles = el->tl.n_tiles;
    S.fixed = el->fixed;
    S.c = el->c;
    S.xj = el->xj; S.yj = el->yj; S.zj = el->zj;
    S.x = el->x; S.y = el->y; S.z = el->z;
    S.X0x = el->X0x; S.X0y = el->X0y; S.X0z = el->X0z;
    S.m_off = el->pat_off; S.m_col = el->pat_col; S.m_val = el->m_val;
    S.f_ext = el->f_ext;
    S.f_int64 = el->f_int;
    S.f_int32 = el->f_int32;
    S.node_bidx = el->tl.node_bidx;
    S.bnode_off = el->tl.bnode_off;
    S.bnode_slots = el->tl.bnode_slots;
    S.jt_off = el->jt_off;
    S.jt_col = el->jt_col;
    S.vg = s->v_guess; S.vp = s->v_prev; S.vk = s->v_k; S.vkm1 = s->v_km1;
    S.g = s->g; S.lam = s->lam; S.m = s->m; S.va = s->va;
    S.xp = s->xp; S.yp = s->yp; S.zp = s->zp;
    S.red = s->red;
    S.red_stride = s->max_blocks;
    S.stat = s->dstat;
    S.stat_norm = (double*)(s->dstat + 4);
    S.stat_rel = (double*)(s->dstat + 6);
    S.rel_tol = s->rel_tol;
    S.node_fixed = s->node_fixed;
    if (s->rel_tol > 0.0) {
        std::vector<unsigned char> nf((size_t)el->N, 0);
        for (int n : el->h_fixed) nf[n] = 1;
        TLFEA_CUDA(cudaMemcpyAsync(s->node_fixed, nf.data(), nf.size(), cudaMemcpyHostToDevice, el->stream));
        TLFEA_CUDA(cudaStreamSynchronize(el->stream));
    }
    if (s->kind == KIND_NESTEROV) {
        S.alpha = s->np.alpha; S.rho = s->np.rho; S.inner_tol = s->np.inner_tol; S.outer_tol = s->np.outer_tol;
        S.max_outer = s->np.max_outer; S.max_inner = s->np.max_inner; S.dt = s->np.time_step;
    } else {
        S.lr = s->ap.lr; S.beta1 = s->ap.beta1; S.beta2 = s->ap.beta2; S.eps = s->ap.eps;
        S.wd = s->ap.weight_decay; S.lr_decay = s->ap.lr_decay; S.inner_tol = s->ap.inner_tol;
        S.outer_tol = s->ap.outer_tol; S.rho = s->ap.rho; S.max_outer = s->ap.max_outer;
        S.max_inner = s->ap.max_inner; S.dt = s->ap.time_step; S.check = s->ap.convergence_check_interval;
        S.rtol = s->ap.inner_rtol;
    }
    const bool damp = (el->eta_d != 0.0 || el->lambda_d != 0.0);
    TileArgs<float> A32;
    TileArgs<double> A64;
    memset(&A32, 0, sizeof(A32));
    memset(&A64, 0, sizeof(A64));
    A32.node_off = A64.node_off = el->tl.node_off;
    A32.ln_gid = A64.ln_gid = el->tl.ln_gid;
    A32.ln_pslot = A64.ln_pslot = el->tl.ln_pslot;
    A32.ln_inc_end = A64.ln_inc_end = el->tl.ln_inc_end;
    A32.inc = A64.inc = el->tl.inc;
    A32.lconn = A64.lconn = el->tl.lconn;
    A32.tile_elem = A64.tile_elem = el->tl.tile_elem;
    A32.v = A64.v = s->v_guess;
    A32.max_local = A64.max_local = el->tl.max_local;
    A32.qb = A64.qb = qp_bary(el);
    A32.mu10 = A64.mu10 = el->mu10;
    A32.mu01 = A64.mu01 = el->mu01;
    A32.kappa = A64.kappa = el->kappa;
    A32.ji = el->tl.ji32;
    A64.ji = el->tl.ji64;
    A32.grad = el->tl.grad32; A32.dv = el->tl.dv32; A32.px = A32.py = A32.pz = nullptr;
    A32.x64 = el->x; A32.y64 = el->y; A32.z64 = el->z; A32.X0x = el->X0x; A32.X0y = el->X0y; A32.X0z = el->X0z;
    A32.f_out = el->f_int32; A32.partial = el->tl.partial32;
    A32.lambda = (float)el->lambda; A32.mu = (float)el->mu; A32.eta = (float)el->eta_d; A32.lamd = (float)el->lambda_d;
    A64.grad = el->tl.grad64; A64.dv = el->tl.dv64; A64.px = el->x; A64.py = el->y; A64.pz = el->z;
    A64.f_out = el->f_int; A64.partial = el->tl.partial64;
    A64.lambda = el->lambda; A64.mu = el->mu; A64.eta = el->eta_d; A64.lamd = el->lambda_d;
    const bool mr = (el->material == TLFEA_MATERIAL_MOONEY_RIVLIN);
    // the element-wise mass term replaces the assembled row pass unless the stop
    // rule needs f_int alone (and for Mooney-Rivlin, which keeps the row pass)
    const bool mass = (s->rel_tol <= 0.0) && !mr;
    A32.vp = A64.vp = s->v_prev;
    A32.mass_scale = A64.mass_scale = el->rho / S.dt;
    auto launch_one = [&](FOArgs& SS) -> int {
#define TLFEA_FO_LAUNCH(R_, NPE_, NQP_, AA)                                                                     \
    (mr ? (damp ? launch_first_order<R_, NPE_, NQP_, true, true, false>(s, SS, AA)                             \
                : launch_first_order<R_, NPE_, NQP_, false, true, false>(s, SS, AA))                           \
        : mass ? (damp ? launch_first_order<R_, NPE_, NQP_, true, false, true>(s, SS, AA)                      \
                       : launch_first_order<R_, NPE_, NQP_, false, false, true>(s, SS, AA))                    \
               : (damp ? launch_first_order<R_, NPE_, NQP_, true, false, false>(s, SS, AA)                     \
                       : launch_first_order<R_, NPE_, NQP_, false, false, false>(s, SS, AA)))
        if (fp32) return (el->npe == 10) ? TLFEA_FO_LAUNCH(float, 10, 5, A32) : TLFEA_FO_LAUNCH(float, 4, 1, A32);
        return (el->npe == 10) ? TLFEA_FO_LAUNCH(double, 10, 5, A64) : TLFEA_FO_LAUNCH(double, 4, 1, A64);
#undef TLFEA_FO_LAUNCH
    };
    cudaStream_t stream = el->stream;
    const int n_steps = std::max(1, steps);
    st = TLFEA_OK;
    // per-phase launches by default from FO_PHASED_MIN_NODES nodes: below it the host
    // round trip of each chunk outweighs the persistent kernel's latency (the 100x10x10
    // beam, 88,641 nodes: 97 against 127 steps/s), above it the phases' occupancy wins
    // (the 200x20x20 beam, 674,081 nodes: 0.287 against 0.425 ms per Nesterov iteration)
    constexpr int FO_PHASED_MIN_NODES = 200000;
    if (s->fo_mode == 2 || (s->fo_mode == 0 && el->N >= FO_PHASED_MIN_NODES)) {
        // per-phase launches: each step's load, then its solve, then its statistics
        auto run_one = [&]() -> int {
#define TLFEA_FO_PHASED(R_, NPE_, NQP_, AA)                                                              \
    (mr ? (damp ? run_phased<R_, NPE_, NQP_, true, true, false>(s, S, AA, stream)                        \
                : run_phased<R_, NPE_, NQP_, false, true, false>(s, S, AA, stream))                      \
        : mass ? (damp ? run_phased<R_, NPE_, NQP_, true, false, true>(s, S, AA, stream)                 \
                       : run_phased<R_, NPE_, NQP_, false, false, true>(s, S, AA, stream))               \
               : (damp ? run_phased<R_, NPE_, NQP_, true, false, false>(s, S, AA, stream)                \
                       : run_phased<R_, NPE_, NQP_, false, false, false>(s, S, AA, stream)))
            if (fp32) return (el->npe == 10) ? TLFEA_FO_PHASED(float, 10, 5, A32) : TLFEA_FO_PHASED(float, 4, 1, A32);
            return (el->npe == 10) ? TLFEA_FO_PHASED(double, 10, 5, A64) : TLFEA_FO_PHASED(double, 4, 1, A64);
#undef TLFEA_FO_PHASED
        };
        std::vector<int> hs(16 * (size_t)n_steps);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, stream);
        for (int k = 0; k < n_steps && !st; ++k) {
            if (load) {
                const double tk = load->t0 + (k + 1) * S.dt;
                const double a = load->amp * sin(load->omega * tk + load->phase);
                const int n3 = 3 * el->N;
                k_step_load<<<(n3 + 255) / 256, 256, 0, stream>>>(n3, load->f_base, load->f_var, a, el->f_ext);
                if (cudaGetLastError() != cudaSuccess) st = TLFEA_CUDA_ERROR;
            }
            if (!st) st = run_one();
            if (!st && cudaMemcpy(hs.data() + 16 * (size_t)k, s->dstat, 16 * sizeof(int), cudaMemcpyDeviceToHost) !=
                           cudaSuccess) {
                set_error("first-order solve: statistics read-back failed");
                st = TLFEA_CUDA_ERROR;
            }
        }
        cudaEventRecord(e1, stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st) return st;
        return first_order_finish(s, hs, n_steps, inner_iters, ms, fp32);
    }
    int* stat_steps = s->dstat;
    if (n_steps > 1 && (st = dalloc(&stat_steps, 16 * (size_t)n_steps))) return st;
    auto release = [&]() {
        if (stat_steps != s->dstat) dfree(stat_steps);
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream);
    // every step: the time-varying load, then one implicit step (Solve); more
    // than one step runs as a single captured graph
    auto enqueue = [&]() -> int {
        for (int k = 0; k < n_steps; ++k) {
            if (load) {
                const double tk = load->t0 + (k + 1) * S.dt;
                const double a = load->amp * sin(load->omega * tk + load->phase);
                const int n3 = 3 * el->N;
                k_step_load<<<(n3 + 255) / 256, 256, 0, stream>>>(n3, load->f_base, load->f_var, a, el->f_ext);
                if (cudaGetLastError() != cudaSuccess) return TLFEA_CUDA_ERROR;
            }
            FOArgs SS = S;
            SS.stat = stat_steps + 16 * k;
            SS.stat_norm = (double*)(SS.stat + 4);
            SS.stat_rel = (double*)(SS.stat + 6);
            const int r = launch_one(SS);
            if (r) return r;
        }
        return TLFEA_OK;
    };
    if (n_steps == 1) {
        st = enqueue();
    } else {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
            release();
            set_error("run_steps: stream capture failed");
            return TLFEA_CUDA_ERROR;
        }
        st = enqueue();
        const cudaError_t ec = cudaStreamEndCapture(stream, &g);
        if (!st && ec == cudaSuccess && cudaGraphInstantiate(&ge, g, 0) == cudaSuccess) {
            if (cudaGraphLaunch(ge, stream) != cudaSuccess) st = TLFEA_CUDA_ERROR;
        } else if (!st) {
            st = TLFEA_CUDA_ERROR;
            set_error("run_steps: graph capture failed");
        }
        if (ge) cudaGraphExecDestroy(ge);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
    }
    cudaEventRecord(e1, stream);
    if (st) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        release();
        return st;
    }
    TLFEA_CUDA(cudaStreamSynchronize(stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::vector<int> hs(16 * (size_t)n_steps);
    if (cudaMemcpy(hs.data(), stat_steps, hs.size() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        release();
        set_error("run_steps: statistics read-back failed");
        return TLFEA_CUDA_ERROR;
    }
    release();
    return first_order_finish(s, hs, n_steps, inner_iters, ms, fp32);
}

// Statistics of the last step (and inner iterations of every step) into the solver.
static int first_order_finish(tlfea_solver_s* s, const std::vector<int>& hs, int n_steps, int* inner_iters,
                              float ms, bool fp32) {
    tlfea_element_s* el = s->el;
    int status = TLFEA_OK;
    for (int k = 0; k < n_steps; ++k) {
        const int* h = hs.data() + 16 * k;
        if (inner_iters) inner_iters[k] = h[1];
        if (h[3]) status = h[3];
    }
    const int* hl = hs.data() + 16 * (n_steps - 1);
    s->stats.outer_iters = hl[0];
    s->stats.inner_iters_total = hl[1];
    s->stats.last_inner_iters = hl[2];
    s->stats.status = status;
    memcpy(&s->stats.last_norm_g, hl + 4, sizeof(double));
    memcpy(&s->stats.rel_residual, hl + 6, sizeof(double));
    s->stats.stop_rule_met = hl[8];
    s->stats.kernel_ms = ms;
    el->f_int_from32 = fp32;
    positions_changed(el);  // the solve moved the positions
    if (status == TLFEA_NONFINITE) {
        set_error("non-finite gradient norm");
        return TLFEA_NONFINITE;
    }
    return TLFEA_OK;
}

int first_order_solve(tlfea_solver_s* s) { return first_order_steps(s, 1, nullptr, nullptr); }

}  // namespace tlfea
