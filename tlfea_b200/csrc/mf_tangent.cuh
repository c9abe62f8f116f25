// mf_tangent.cuh -- the LinearStaticSolver's K p without assembling K (new: the
// reference assembles K, LinearStaticSolver.cu:196-263, and multiplies it with
// cuSPARSE).  K is the SVK tangent at the current positions (the blocks of
// compute_hessian_assemble_csr, FEAT10DataFunc.cuh:512-684 / SVK.cuh:41-67), so
// K p = sum over elements and QPs of dP[dF] gradN_a dV with dF = sum_a p_a (x) gradN_a,
// dP = dF S + F dS, S = lambda tr(E) I + 2 mu E, E = (F^T F - I) / 2,
// dS = lambda tr(dE) I + 2 mu dE, dE = (dF^T F + F^T dF) / 2 -- the directional
// derivative of P whose 3x3 blocks the reference assembles.  Dirichlet DOFs are
// eliminated as apply_bcs_kernel does (LinearStaticSolver.cu:284-306): their columns
// are dropped (p is staged as zero there) and their rows of K_bc p are p itself.
//
// One tile per block: the gradient stream's QP slices by 1-D bulk copies (one stage,
// read twice from shared memory), the tile's node positions, destinations and
// incidence ends by bulk copies of the tile-ordered node record, p gathered per local
// node; the element forces reduce per node in the tile's incidence order (no atomics)
// and the tile's share of p.q over its interior nodes is written per tile, so the
// combine kernel can fold the dot product deterministically.
#pragma once

#include "force_pipe.cuh"
#include "solver.cuh"

namespace tlfea {

struct MfArgs {
    int n_tiles, max_local;  // max_local: the node record's padded tile size
    const int* node_off;
    const int* pad_off;
    const int* pad_gid;
    const int* pad_dst;
    const uint16_t* pad_iend;
    const uint16_t* inc;
    const uint16_t* lconn;
    const double* grad;
    const double* dv;
    const double* sx;
    const double* sy;
    const double* sz;
    const double* p;
    double* q;
    double* partial;  // per partial slot of the nodes shared between tiles
    const unsigned char* is_fixed;  // 3N
    double* tile_dot;  // per tile: p.q over the tile's interior nodes
    double lambda, mu;
    CgCtl* ctl;
};

template <int NPE, int NQP>
__global__ void __launch_bounds__(TILE_ELEMS, 3) k_mf_tile(MfArgs M, int* err) {
    using G = TileTmaGeom<double, NPE>;
    static_assert(G::STAGES == 1, "one stage, read twice");
    constexpr int TE = TILE_ELEMS;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double red_sh[32];
    if (M.ctl->done) return;  // uniform: written by the previous kernel
    const int tile = blockIdx.x, t = threadIdx.x;
    const int ML = M.max_local;
    const TileTmaLayout<double, NPE> L(ML, true);  // the velocity region holds p
    unsigned char* stage0 = smem;
    const uint16_t* lcs = reinterpret_cast<const uint16_t*>(smem + G::STAGE_BYTES);
    const uint16_t* incs = reinterpret_cast<const uint16_t*>(smem + L.inc);
    double* xs = reinterpret_cast<double*>(smem + L.pos);
    double* ys = xs + ML;
    double* zs = ys + ML;
    int* dsts = reinterpret_cast<int*>(smem + L.dst);
    uint16_t* iends = reinterpret_cast<uint16_t*>(smem + L.iend);
    double* ps = reinterpret_cast<double*>(smem + L.vel);
    double* fe = reinterpret_cast<double*>(smem);  // aliases the stage after the QP loop
    const uint32_t bar0 = smem_u32(smem + L.bar), bar_rec = bar0 + 8;

    auto issue = [&](int q) {  // thread 0 only
        const uint32_t extra = (q == 0) ? G::LCONN_BYTES + G::INC_BYTES : 0;
        mbar_expect_tx(bar0, G::STAGE_BYTES + extra);
        bulk_g2s(smem_u32(stage0), M.grad + ((size_t)tile * NQP + q) * (NPE * 3) * TE, G::GRAD_BYTES, bar0);
        bulk_g2s(smem_u32(stage0) + G::GRAD_BYTES, M.dv + ((size_t)tile * NQP + q) * TE, G::DV_BYTES, bar0);
        if (q == 0) {
            bulk_g2s(smem_u32(lcs), M.lconn + (size_t)tile * NPE * TE, G::LCONN_BYTES, bar0);
            bulk_g2s(smem_u32(incs), M.inc + (size_t)tile * NPE * TE, G::INC_BYTES, bar0);
        }
    };
    const int pb = M.pad_off[tile];
    if (t == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar_rec, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(0);
        const int np = M.pad_off[tile + 1] - pb;
        mbar_expect_tx(bar_rec, (uint32_t)np * (3 * sizeof(double) + sizeof(int) + sizeof(uint16_t)));
        bulk_g2s(smem_u32(xs), M.sx + pb, np * sizeof(double), bar_rec);
        bulk_g2s(smem_u32(ys), M.sy + pb, np * sizeof(double), bar_rec);
        bulk_g2s(smem_u32(zs), M.sz + pb, np * sizeof(double), bar_rec);
        bulk_g2s(smem_u32(dsts), M.pad_dst + pb, np * sizeof(int), bar_rec);
        bulk_g2s(smem_u32(iends), M.pad_iend + pb, np * sizeof(uint16_t), bar_rec);
    }
    const int nl = M.node_off[tile + 1] - M.node_off[tile];
#pragma unroll 4
    for (int ln = t; ln < nl; ln += TE) {  // unrolled: several nodes' gathers in flight at once
        const int g = M.pad_gid[pb + ln];
#pragma unroll
        for (int d = 0; d < 3; ++d) ps[3 * ln + d] = M.is_fixed[3 * g + d] ? 0.0 : M.p[3 * g + d];
    }
    __syncthreads();  // barriers initialised, p staged
    if (!mbar_wait(bar_rec, 0)) atomicExch(err, 3);
    auto lc = [&](int a) -> int { return lcs[a * TE + t]; };

    double f[NPE][3];
#pragma unroll
    for (int a = 0; a < NPE; ++a) f[a][0] = f[a][1] = f[a][2] = 0.0;
#pragma unroll 1
    for (int q = 0; q < NQP; ++q) {
        if (!mbar_wait(bar0, q & 1)) atomicExch(err, 3);
        const double* gs = reinterpret_cast<const double*>(stage0);
        const double dv = reinterpret_cast<const double*>(stage0 + G::GRAD_BYTES)[t];
        double F[3][3], Hp[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) F[i][j] = Hp[i][j] = 0.0;
#pragma unroll 2
        for (int a = 0; a < NPE; ++a) {
            const int l = lc(a);
            const double xa[3] = {xs[l], ys[l], zs[l]};
            const double pa[3] = {ps[3 * l + 0], ps[3 * l + 1], ps[3 * l + 2]};
            const double ga[3] = {gs[grad_slot<double>(a, 0, t)], gs[grad_slot<double>(a, 1, t)],
                                  gs[grad_slot<double>(a, 2, t)]};
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    F[i][j] += xa[i] * ga[j];
                    Hp[i][j] += pa[i] * ga[j];
                }
        }
        // E, S at F; dE, dS along dF = Hp; dP = Hp S + F dS (scaled by dV)
        double S[3][3], dS[3][3];
        {
            double E[3][3], dE[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    double e = 0.0, de = 0.0;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        e += F[k][i] * F[k][j];
                        de += Hp[k][i] * F[k][j] + F[k][i] * Hp[k][j];
                    }
                    E[i][j] = 0.5 * (e - (i == j ? 1.0 : 0.0));
                    dE[i][j] = 0.5 * de;
                }
            const double trE = E[0][0] + E[1][1] + E[2][2], trdE = dE[0][0] + dE[1][1] + dE[2][2];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    S[i][j] = 2.0 * M.mu * E[i][j] + (i == j ? M.lambda * trE : 0.0);
                    dS[i][j] = 2.0 * M.mu * dE[i][j] + (i == j ? M.lambda * trdE : 0.0);
                }
        }
        double dP[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double v = 0.0;
#pragma unroll
                for (int k = 0; k < 3; ++k) v += Hp[i][k] * S[k][j] + F[i][k] * dS[k][j];
                dP[i][j] = v * dv;
            }
#pragma unroll
        for (int a = 0; a < NPE; ++a) {
            const double ga[3] = {gs[grad_slot<double>(a, 0, t)], gs[grad_slot<double>(a, 1, t)],
                                  gs[grad_slot<double>(a, 2, t)]};
#pragma unroll
            for (int i = 0; i < 3; ++i) f[a][i] += dP[i][0] * ga[0] + dP[i][1] * ga[1] + dP[i][2] * ga[2];
        }
        if (q + 1 < NQP) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (t == 0) issue(q + 1);
        }
    }
    __syncthreads();  // every thread is done with the stage the force table reuses
#pragma unroll
    for (int a = 0; a < NPE; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) fe[(a * 3 + d) * TE + t] = f[a][d];
    __syncthreads();
    double dot = 0.0;
    for (int ln = t; ln < nl; ln += TE) {
        const int beg = ln ? iends[ln - 1] : 0;
        const int end = iends[ln];
        double s[3] = {0.0, 0.0, 0.0};
        for (int k = beg; k < end; ++k) {
            const int ent = incs[k];
            const int base = (ent >> TILE_SHIFT) * 3 * TE + (ent & (TE - 1));
            s[0] += fe[base];
            s[1] += fe[base + TE];
            s[2] += fe[base + 2 * TE];
        }
        const int dn = dsts[ln];
        if (dn >= 0) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const bool fx = M.is_fixed[3 * dn + d];
                const double pv = fx ? M.p[3 * dn + d] : ps[3 * ln + d];
                const double qv = fx ? pv : s[d];  // eliminated DOF: identity row
                M.q[3 * dn + d] = qv;
                dot += pv * qv;
            }
        } else {
            const int sl = -dn - 1;
            M.partial[3 * sl + 0] = s[0];
            M.partial[3 * sl + 1] = s[1];
            M.partial[3 * sl + 2] = s[2];
        }
    }
    dot = block_sum(dot, red_sh);
    if (t == 0) M.tile_dot[tile] = dot;
    // outputs written: the combine (a programmatic dependent) may be scheduled
    asm volatile("griddepcontrol.launch_dependents;");
}

// The nodes shared between tiles: their partials summed in tile order, then p.q folded
// -- the tiles' interior shares in tile order, the shared nodes' per block in block
// order -- by the last block, which sets alpha = rr / p.q (LinearStaticSolver.cu:519-533).
__global__ void __launch_bounds__(256) k_mf_combine_dot(int nb, const int* __restrict__ bgid,
                                                        const int* __restrict__ boff, MfArgs M, double* part) {
    __shared__ double red[32];
    __shared__ bool am_last;
    // launched as a programmatic dependent of the tile kernel: wait for its results
    asm volatile("griddepcontrol.wait;" ::: "memory");
    CgCtl* ctl = M.ctl;
    if (ctl->done) return;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    double dot = 0.0;
    if (b < nb) {
        double s[3] = {0.0, 0.0, 0.0};
        for (int k = boff[b]; k < boff[b + 1]; ++k) {
            s[0] += M.partial[3 * k + 0];
            s[1] += M.partial[3 * k + 1];
            s[2] += M.partial[3 * k + 2];
        }
        const int g = bgid[b];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double pv = M.p[3 * g + d];
            const double qv = M.is_fixed[3 * g + d] ? pv : s[d];
            M.q[3 * g + d] = qv;
            dot += pv * qv;
        }
    }
    const double bs = block_sum(dot, red);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = bs;
        __threadfence();
        const unsigned int tk = atomicAdd(&ctl->ticket, 1u);
        am_last = (tk == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    double s = 0.0;
    for (int k = threadIdx.x; k < M.n_tiles; k += blockDim.x) s += __ldcg(M.tile_dot + k);
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) s += __ldcg(part + k);
    s = block_sum(s, red);
    if (threadIdx.x == 0) {
        ctl->ticket = 0;
        ctl->pq = s;
        if (s <= 0.0) {
            ctl->status = 1;
            ctl->done = 1;
        } else {
            ctl->alpha = ctl->rr / s;
        }
    }
}

}  // namespace tlfea
