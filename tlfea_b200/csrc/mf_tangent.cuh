// mf_tangent.cuh -- the LinearStaticSolver's K p without assembling K (new: the
// reference assembles K, LinearStaticSolver.cu:196-263, and multiplies it with
// cuSPARSE).  K is the SVK tangent at the solve's positions (the blocks of
// compute_hessian_assemble_csr, FEAT10DataFunc.cuh:512-684 / SVK.cuh:41-67), so
// K p = sum over elements and QPs of dP[dF] gradN_a dV with dF = sum_a p_a (x) gradN_a,
// dP = dF S + F dS, S = lambda tr(E) I + 2 mu E, E = (F^T F - I) / 2,
// dS = lambda tr(dE) I + 2 mu dE, dE = (dF^T F + F^T dF) / 2 -- the directional
// derivative of P whose 3x3 blocks the reference assembles.  Dirichlet DOFs are
// eliminated as apply_bcs_kernel does (LinearStaticSolver.cu:284-306): their columns
// are dropped (p is staged as zero there) and their rows of K_bc p are p itself.
//
// The positions do not change during a solve, so F and S at every QP are formed once
// per solve (k_mf_prep) into a tangent stream beside the compact geometry stream
// (J^-1, dV); each product then needs only dF = (dp/dxi) J^-1, dE, dS, dP and the
// nodal forces Q dN/dxi (Q = dP J^-T).  One tile per block: the QP slices (J^-1, dV,
// F, S) by 1-D bulk copies into two stages, the tile's destinations, incidence ends,
// fixed-DOF flags and p (gathered into the node record's tile order by k_mf_gather)
// by bulk copies; the element forces reduce per node in the tile's incidence order
// (no atomics) and the tile's share of p.q over its interior nodes is written per
// tile, so the combine kernel can fold the dot product deterministically.
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
    const double* ji;  // compact geometry stream: J^-1 per QP
    const double* dv;
    double* tan;       // per element and QP: F (9, row-major) and S (6, symmetric), tile/QP slices
    const double* x;   // positions the tangent is formed at (node order)
    const double* y;
    const double* z;
    const double* p;
    const double* prec;     // p in the node record's tile order (k_mf_gather), fixed DOFs zeroed
    const uint16_t* pfix;   // per padded slot: its node's fixed-DOF flags (bits 0..2)
    double* q;
    double* partial;  // per partial slot of the nodes shared between tiles
    const unsigned char* is_fixed;  // 3N
    double* tile_dot;  // per tile: p.q over the tile's interior nodes
    double lambda, mu;
    QpBary qb;
    CgCtl* ctl;
};

// Values per element and QP in the tangent stream: F (9) then S (6).
constexpr int MF_TAN = 15;
// Symmetric 3x3 storage: index k of (i, j), i <= j: 0 00, 1 11, 2 22, 3 01, 4 02, 5 12.
__host__ __device__ constexpr int sym3(int i, int j) {
    return i == j ? i : (i + j == 1 ? 3 : (i + j == 2 ? 4 : 5));
}

// S = lambda tr(E) I + 2 mu E with E = (F^T F - I) / 2 (six entries).
__device__ __forceinline__ void svk_stress_sym(const double F[3][3], double lambda, double mu, double S[6]) {
    constexpr int SI[6] = {0, 1, 2, 0, 0, 1}, SJ[6] = {0, 1, 2, 1, 2, 2};
    double E[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const int i = SI[k], j = SJ[k];
        double e = 0.0;
#pragma unroll
        for (int m = 0; m < 3; ++m) e += F[m][i] * F[m][j];
        E[k] = 0.5 * (e - (i == j ? 1.0 : 0.0));
    }
    const double trE = E[0] + E[1] + E[2];
#pragma unroll
    for (int k = 0; k < 6; ++k) S[k] = 2.0 * mu * E[k] + (k < 3 ? lambda * trE : 0.0);
}

// dP dV along dF = Hp at (F, S): dE = (Hp^T F + F^T Hp) / 2, dS = lambda tr(dE) I +
// 2 mu dE, dP = Hp S + F dS (the SVK tangent).
__device__ __forceinline__ void svk_tangent_dp(const double F[3][3], const double S[6], const double Hp[3][3],
                                               double lambda, double mu, double dv, double dP[3][3]) {
    constexpr int SI[6] = {0, 1, 2, 0, 0, 1}, SJ[6] = {0, 1, 2, 1, 2, 2};
    double dS[6];
    {
        double dE[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int i = SI[k], j = SJ[k];
            double de = 0.0;
#pragma unroll
            for (int m = 0; m < 3; ++m) de += Hp[m][i] * F[m][j] + F[m][i] * Hp[m][j];
            dE[k] = 0.5 * de;
        }
        const double trdE = dE[0] + dE[1] + dE[2];
#pragma unroll
        for (int k = 0; k < 6; ++k) dS[k] = 2.0 * mu * dE[k] + (k < 3 ? lambda * trdE : 0.0);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double v = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) v += Hp[i][k] * S[sym3(k, j)] + F[i][k] * dS[sym3(k, j)];
            dP[i][j] = v * dv;
        }
}

// Bulk-copy sizes of the product's QP slices (J^-1, dV, F and S of a tile's elements).
template <int NPE>
struct MfGeom {
    static constexpr uint32_t JI_BYTES = 9 * TILE_ELEMS * sizeof(double);
    static constexpr uint32_t DV_BYTES = TILE_ELEMS * sizeof(double);
    static constexpr uint32_t TAN_BYTES = MF_TAN * TILE_ELEMS * sizeof(double);
    static constexpr uint32_t STAGE_BYTES = JI_BYTES + DV_BYTES + TAN_BYTES;
    static constexpr uint32_t LCONN_BYTES = NPE * TILE_ELEMS * sizeof(uint16_t);
    static constexpr uint32_t INC_BYTES = NPE * TILE_ELEMS * sizeof(uint16_t);
    static constexpr uint32_t FE_BYTES = 3 * NPE * TILE_ELEMS * sizeof(double);
    // the two stages, and after the QP loop the element forces of the reduction
    static constexpr uint32_t REGION0 = ((2 * STAGE_BYTES > FE_BYTES ? 2 * STAGE_BYTES : FE_BYTES) + 15u) & ~15u;
    static_assert(STAGE_BYTES % 16 == 0 && LCONN_BYTES % 16 == 0 && INC_BYTES % 16 == 0, "bulk sizes");
};

// The product's shared memory: [stages | element forces][lconn][incidence][destinations]
// [incidence ends][p (3 per local node)][fixed flags][barriers: two stages, the record].
template <int NPE>
struct MfLayout {
    size_t lconn, inc, dst, iend, pvals, fmask, bar, total;
    __host__ __device__ explicit MfLayout(int max_local) {
        using G = MfGeom<NPE>;
        auto al = [](size_t v) { return (v + 15) & ~size_t(15); };
        lconn = G::REGION0;
        inc = lconn + G::LCONN_BYTES;
        dst = inc + G::INC_BYTES;
        iend = al(dst + (size_t)max_local * sizeof(int));
        pvals = al(iend + (size_t)max_local * sizeof(uint16_t));
        fmask = al(pvals + 3 * (size_t)max_local * sizeof(double));
        bar = al(fmask + (size_t)max_local * sizeof(uint16_t));
        total = bar + 3 * sizeof(unsigned long long);
    }
};

// Per padded slot of the node record, its node's fixed-DOF flags (padding: 0); once
// per solve.
__global__ void k_mf_fixbits(long long n_pad, const int* __restrict__ pad_gid,
                             const unsigned char* __restrict__ is_fixed, uint16_t* __restrict__ pfix) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n_pad) return;
    const int g = pad_gid[i];
    unsigned m = 0;
    if (g >= 0)
        for (int d = 0; d < 3; ++d) m |= (unsigned)(is_fixed[3 * (size_t)g + d] != 0) << d;
    pfix[i] = (uint16_t)m;
}

// p in the node record's tile order, per padded slot its node's three components with
// the eliminated DOFs zeroed (their columns dropped from K p), padding 0: a streaming
// gather over all slots, so the product's tiles bulk-copy p like the other record
// arrays.  Each thread takes MF_GATHER_ILP slots (blockDim apart, so every load and
// store stays coalesced across the warp) and issues all their loads before any use.
constexpr int MF_GATHER_ILP = 4;
__global__ void __launch_bounds__(256) k_mf_gather(long long n_pad, const int* __restrict__ pad_gid,
                                                   const uint16_t* __restrict__ pfix, const double* __restrict__ p,
                                                   double* __restrict__ prec, const CgCtl* __restrict__ ctl) {
    // the tile kernel (a programmatic dependent) may start its own copies meanwhile
    asm volatile("griddepcontrol.launch_dependents;");
    if (ctl->done) return;
    const long long base = (long long)blockIdx.x * blockDim.x * MF_GATHER_ILP + threadIdx.x;
    int g[MF_GATHER_ILP];
    unsigned m[MF_GATHER_ILP];
#pragma unroll
    for (int j = 0; j < MF_GATHER_ILP; ++j) {
        const long long i = base + (long long)j * blockDim.x;
        g[j] = (i < n_pad) ? pad_gid[i] : -1;
        m[j] = (i < n_pad) ? pfix[i] : 0u;
    }
    double v[MF_GATHER_ILP][3];
#pragma unroll
    for (int j = 0; j < MF_GATHER_ILP; ++j)
#pragma unroll
        for (int d = 0; d < 3; ++d)
            v[j][d] = (g[j] >= 0 && !((m[j] >> d) & 1)) ? p[3 * (size_t)g[j] + d] : 0.0;
#pragma unroll
    for (int j = 0; j < MF_GATHER_ILP; ++j) {
        const long long i = base + (long long)j * blockDim.x;
        if (i < n_pad) {
#pragma unroll
            for (int d = 0; d < 3; ++d) prec[3 * i + d] = v[j][d];
        }
    }
}

// The tile's element forces f (this thread's element) reduced per node in the
// incidence order: interior nodes write q (identity rows for eliminated DOFs) and
// their share of p.q, shared nodes their partial slot; then the tile's p.q.  Called
// by all threads after the stage region that fe aliases is free.
template <int NPE>
__device__ __forceinline__ void mf_tile_epilogue(const MfArgs& M, const double (&f)[NPE][3], double* fe,
                                                 const uint16_t* incs, const uint16_t* iends, const int* dsts,
                                                 const double* ps, const uint16_t* fmask, int tile, int nl,
                                                 double* red_sh) {
    constexpr int TE = TILE_ELEMS;
    const int t = threadIdx.x;
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
                const bool fx = (fmask[ln] >> d) & 1;  // staged with the node record
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

// F and S of every element and QP at the given positions, into the tangent stream
// (once per solve).  One tile per block, one element per thread: dx/dxi through the
// barycentric structure, F = (dx/dxi) J^-1, S from E.  Padding element slots have a
// zero J^-1 and dV, so they contribute nothing to a product.
template <int NPE, int NQP>
__global__ void __launch_bounds__(TILE_ELEMS) k_mf_prep(MfArgs M) {
    constexpr int TE = TILE_ELEMS;
    const int tile = blockIdx.x, t = threadIdx.x;
    const int pb = M.pad_off[tile];
    int gid[NPE];
#pragma unroll
    for (int a = 0; a < NPE; ++a) gid[a] = M.pad_gid[pb + M.lconn[((size_t)tile * NPE + a) * TE + t]];
    auto x = [&](int a, int d) -> double {
        const int g = gid[a];
        if (g < 0) return 0.0;
        return d == 0 ? M.x[g] : (d == 1 ? M.y[g] : M.z[g]);
    };
#pragma unroll 1
    for (int q = 0; q < NQP; ++q) {
        const size_t sl = (size_t)tile * NQP + q;
        double ji[9];
#pragma unroll
        for (int m = 0; m < 9; ++m) ji[m] = M.ji[(sl * 9 + m) * TE + t];
        const double Lq[4] = {M.qb.L[q][0], M.qb.L[q][1], M.qb.L[q][2], M.qb.L[q][3]};
        double Gx[3][3], F[3][3], S[6];
        tet_dx_dxi_at<double, NPE>(x, Lq, Gx);
        mul_jinv(Gx, ji, F);
        svk_stress_sym(F, M.lambda, M.mu, S);
        double* out = M.tan + sl * MF_TAN * TE + t;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) out[(3 * i + j) * TE] = F[i][j];
#pragma unroll
        for (int k = 0; k < 6; ++k) out[(9 + k) * TE] = S[k];
    }
}

// K_bc p for one tile per block (see the file comment).  The QP slices fill a
// double-buffered ring: a slice is read into registers, then its stage is refilled two
// QPs ahead, so each tile keeps a copy in flight while it computes.
template <int NPE, int NQP>
__global__ void __launch_bounds__(TILE_ELEMS, 3) k_mf_geo(MfArgs M, int* err) {
    using G = MfGeom<NPE>;
    constexpr int TE = TILE_ELEMS;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double red_sh[32];
    if (M.ctl->done) return;  // uniform: written by the previous kernel
    const int tile = blockIdx.x, t = threadIdx.x;
    const MfLayout<NPE> L(M.max_local);
    unsigned char* stage0 = smem;
    const uint16_t* lcs = reinterpret_cast<const uint16_t*>(smem + L.lconn);
    const uint16_t* incs = reinterpret_cast<const uint16_t*>(smem + L.inc);
    int* dsts = reinterpret_cast<int*>(smem + L.dst);
    uint16_t* iends = reinterpret_cast<uint16_t*>(smem + L.iend);
    double* ps = reinterpret_cast<double*>(smem + L.pvals);
    uint16_t* fmask = reinterpret_cast<uint16_t*>(smem + L.fmask);
    double* fe = reinterpret_cast<double*>(smem);  // aliases the stages after the QP loop
    const uint32_t bar0 = smem_u32(smem + L.bar), bar_rec = bar0 + 16;

    auto issue = [&](int q) {  // thread 0 only
        const uint32_t bar = bar0 + 8 * (q & 1);
        const uint32_t dst = smem_u32(stage0 + (size_t)(q & 1) * G::STAGE_BYTES);
        const uint32_t extra = (q == 0) ? G::LCONN_BYTES + G::INC_BYTES : 0;
        const size_t sl = (size_t)tile * NQP + q;
        mbar_expect_tx(bar, G::STAGE_BYTES + extra);
        bulk_g2s(dst, M.ji + sl * 9 * TE, G::JI_BYTES, bar);
        bulk_g2s(dst + G::JI_BYTES, M.dv + sl * TE, G::DV_BYTES, bar);
        bulk_g2s(dst + G::JI_BYTES + G::DV_BYTES, M.tan + sl * MF_TAN * TE, G::TAN_BYTES, bar);
        if (q == 0) {
            bulk_g2s(smem_u32(lcs), M.lconn + (size_t)tile * NPE * TE, G::LCONN_BYTES, bar);
            bulk_g2s(smem_u32(incs), M.inc + (size_t)tile * NPE * TE, G::INC_BYTES, bar);
        }
    };
    const int pb = M.pad_off[tile];
    if (t == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        mbar_init(bar_rec, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(0);
        if (NQP > 1) issue(1);
        const int np = M.pad_off[tile + 1] - pb;
        // destinations, incidence ends, fixed flags and p (3 doubles) per slot
        mbar_expect_tx(bar_rec, (uint32_t)np * (sizeof(int) + 2 * sizeof(uint16_t) + 3 * sizeof(double)));
        bulk_g2s(smem_u32(dsts), M.pad_dst + pb, np * sizeof(int), bar_rec);
        bulk_g2s(smem_u32(iends), M.pad_iend + pb, np * sizeof(uint16_t), bar_rec);
        bulk_g2s(smem_u32(fmask), M.pfix + pb, np * sizeof(uint16_t), bar_rec);
        // p's tile-ordered copy comes from the gather kernel this one depends on
        asm volatile("griddepcontrol.wait;" ::: "memory");
        bulk_g2s(smem_u32(ps), M.prec + 3 * (size_t)pb, np * 3 * sizeof(double), bar_rec);
    }
    const int nl = M.node_off[tile + 1] - M.node_off[tile];
    __syncthreads();  // barriers initialised
    if (!mbar_wait(bar_rec, 0)) atomicExch(err, 3);

    double f[NPE][3];
#pragma unroll
    for (int a = 0; a < NPE; ++a) f[a][0] = f[a][1] = f[a][2] = 0.0;
#pragma unroll 1
    for (int q = 0; q < NQP; ++q) {
        if (!mbar_wait(bar0 + 8 * (q & 1), (q >> 1) & 1)) atomicExch(err, 3);
        const double* st = reinterpret_cast<const double*>(stage0 + (size_t)(q & 1) * G::STAGE_BYTES);
        double ji[9], F[3][3], S[6];
#pragma unroll
        for (int m = 0; m < 9; ++m) ji[m] = st[m * TE + t];
        const double dv = st[9 * TE + t];
#pragma unroll
        for (int m = 0; m < 9; ++m) F[m / 3][m % 3] = st[(10 + m) * TE + t];
#pragma unroll
        for (int k = 0; k < 6; ++k) S[k] = st[(19 + k) * TE + t];
        if (q + 2 < NQP) {
            // every thread's generic reads of this stage precede the bulk refill
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (t == 0) issue(q + 2);
        }
        const double Lq[4] = {M.qb.L[q][0], M.qb.L[q][1], M.qb.L[q][2], M.qb.L[q][3]};
        double Gp[3][3], Hp[3][3], dP[3][3], Q[3][3];
        tet_dx_dxi_at<double, NPE>([&](int a, int d) { return ps[3 * lcs[a * TE + t] + d]; }, Lq, Gp);
        mul_jinv(Gp, ji, Hp);
        svk_tangent_dp(F, S, Hp, M.lambda, M.mu, dv, dP);
        mul_jinv_t(dP, ji, Q);
        tet_scatter<double, NPE>(Q, Lq, [&](int a, int d, double v) { f[a][d] += v; });
    }
    __syncthreads();  // every thread is done with the stages the force table reuses
    mf_tile_epilogue<NPE>(M, f, fe, incs, iends, dsts, ps, fmask, tile, nl, red_sh);
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
