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
// One tile per block: the compact geometry stream's QP slices by 1-D bulk copies
// (two stages), the tile's node positions, destinations, incidence ends, fixed-DOF
// flags and p (gathered into the record's tile order by k_mf_gather) by bulk copies of
// the tile-ordered node record; the element forces reduce per node in the tile's incidence order (no atomics)
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
    const double* ji;  // compact geometry stream: J^-1 per QP
    const double* dv;
    const double* sx;
    const double* sy;
    const double* sz;
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

// dP dV from F and the direction's Hp = dF (the SVK tangent along Hp):
// E = (F^T F - I) / 2, dE = (Hp^T F + F^T Hp) / 2, S = lambda tr(E) I + 2 mu E,
// dS likewise from dE, dP = Hp S + F dS.  E, dE, S and dS are symmetric: their six
// upper entries are formed once (sym index k of (i, j): 0 00, 1 11, 2 22, 3 01, 4 02, 5 12).
__device__ __forceinline__ void svk_tangent_dp(const double F[3][3], const double Hp[3][3], double lambda,
                                               double mu, double dv, double dP[3][3]) {
    constexpr int SI[6] = {0, 1, 2, 0, 0, 1}, SJ[6] = {0, 1, 2, 1, 2, 2};
    double S[6], dS[6];
    {
        double E[6], dE[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int i = SI[k], j = SJ[k];
            double e = 0.0, de = 0.0;
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                e += F[m][i] * F[m][j];
                de += Hp[m][i] * F[m][j] + F[m][i] * Hp[m][j];
            }
            E[k] = 0.5 * (e - (i == j ? 1.0 : 0.0));
            dE[k] = 0.5 * de;
        }
        const double trE = E[0] + E[1] + E[2], trdE = dE[0] + dE[1] + dE[2];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            S[k] = 2.0 * mu * E[k] + (k < 3 ? lambda * trE : 0.0);
            dS[k] = 2.0 * mu * dE[k] + (k < 3 ? lambda * trdE : 0.0);
        }
    }
    auto sym = [](int i, int j) { return i == j ? i : (i + j == 1 ? 3 : (i + j == 2 ? 4 : 5)); };
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double v = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) v += Hp[i][k] * S[sym(k, j)] + F[i][k] * dS[sym(k, j)];
            dP[i][j] = v * dv;
        }
}

// The compact kernel's shared memory: the geometry kernel's layout (the velocity
// region holds p) and per local node its fixed-DOF flags (16 bits).
template <int NPE>
struct MfGeoLayout : TileGeoLayout<double, NPE> {
    size_t fmask, total_mf;
    __host__ __device__ explicit MfGeoLayout(int max_local) : TileGeoLayout<double, NPE>(max_local, true) {
        fmask = (this->total + 15) & ~size_t(15);
        total_mf = fmask + (((size_t)max_local * sizeof(uint16_t) + 15) & ~size_t(15));
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
// gather over all slots, so the product's tiles bulk-copy p like the positions.
__global__ void __launch_bounds__(256) k_mf_gather(long long n_pad, const int* __restrict__ pad_gid,
                                                   const uint16_t* __restrict__ pfix, const double* __restrict__ p,
                                                   double* __restrict__ prec, const CgCtl* __restrict__ ctl) {
    // the tile kernel (a programmatic dependent) may start its own copies meanwhile
    asm volatile("griddepcontrol.launch_dependents;");
    if (ctl->done) return;
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n_pad) return;
    const int g = pad_gid[i];
    const unsigned m = pfix[i];
    double v[3] = {0.0, 0.0, 0.0};
    if (g >= 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d) v[d] = ((m >> d) & 1) ? 0.0 : p[3 * (size_t)g + d];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) prec[3 * i + d] = v[d];
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

// One tile per block on the compact geometry stream (J^-1 and dV per QP, 10 values
// instead of the 3 NPE + 1 of the per-node gradients): F = (dx/dxi) J^-1 and
// dF = (dp/dxi) J^-1 from the staged positions and p through the barycentric
// structure of the shape functions, the nodal forces from Q = dP J^-T (tet_dx_dxi_at
// / tet_scatter).  The 10-value slices fit a double-buffered ring (a slice is read
// into registers, then its stage is refilled two QPs ahead), so each tile keeps a
// copy in flight while it computes.
template <int NPE, int NQP>
__global__ void __launch_bounds__(TILE_ELEMS, 3) k_mf_geo(MfArgs M, int* err) {
    using G = TileGeoGeom<double, NPE>;
    constexpr int TE = TILE_ELEMS;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double red_sh[32];
    if (M.ctl->done) return;  // uniform: written by the previous kernel
    const int tile = blockIdx.x, t = threadIdx.x;
    const int ML = M.max_local;
    const MfGeoLayout<NPE> L(ML);
    unsigned char* stage0 = smem;
    uint16_t* fmask = reinterpret_cast<uint16_t*>(smem + L.fmask);
    const uint16_t* lcs = reinterpret_cast<const uint16_t*>(smem + L.lconn);
    const uint16_t* incs = reinterpret_cast<const uint16_t*>(smem + L.inc);
    double* xs = reinterpret_cast<double*>(smem + L.pos);
    double* ys = xs + ML;
    double* zs = ys + ML;
    int* dsts = reinterpret_cast<int*>(smem + L.dst);
    uint16_t* iends = reinterpret_cast<uint16_t*>(smem + L.iend);
    double* ps = reinterpret_cast<double*>(smem + L.vel);
    double* fe = reinterpret_cast<double*>(smem);  // aliases the stages after the QP loop
    const uint32_t bar0 = smem_u32(smem + L.bar), bar_rec = bar0 + 16;

    auto issue = [&](int q) {  // thread 0 only
        const uint32_t bar = bar0 + 8 * (q & 1);
        const uint32_t dst = smem_u32(stage0 + (size_t)(q & 1) * G::STAGE_BYTES);
        const uint32_t extra = (q == 0) ? G::LCONN_BYTES + G::INC_BYTES : 0;
        mbar_expect_tx(bar, G::STAGE_BYTES + extra);
        bulk_g2s(dst, M.ji + ((size_t)tile * NQP + q) * 9 * TE, G::JI_BYTES, bar);
        bulk_g2s(dst + G::JI_BYTES, M.dv + ((size_t)tile * NQP + q) * TE, G::DV_BYTES, bar);
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
        // positions, destinations, incidence ends, p (3 doubles) and fixed flags per slot
        mbar_expect_tx(bar_rec, (uint32_t)np * (6 * sizeof(double) + sizeof(int) + 2 * sizeof(uint16_t)));
        bulk_g2s(smem_u32(xs), M.sx + pb, np * sizeof(double), bar_rec);
        bulk_g2s(smem_u32(ys), M.sy + pb, np * sizeof(double), bar_rec);
        bulk_g2s(smem_u32(zs), M.sz + pb, np * sizeof(double), bar_rec);
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

    int lc[NPE];
    double f[NPE][3];
#pragma unroll
    for (int a = 0; a < NPE; ++a) f[a][0] = f[a][1] = f[a][2] = 0.0;
#pragma unroll 1
    for (int q = 0; q < NQP; ++q) {
        if (!mbar_wait(bar0 + 8 * (q & 1), (q >> 1) & 1)) atomicExch(err, 3);
        const unsigned char* st = stage0 + (size_t)(q & 1) * G::STAGE_BYTES;
        const double* js = reinterpret_cast<const double*>(st);
        if (q == 0) {
#pragma unroll
            for (int a = 0; a < NPE; ++a) lc[a] = lcs[a * TE + t];
        }
        double ji[9];
#pragma unroll
        for (int m = 0; m < 9; ++m) ji[m] = js[m * TE + t];
        const double dv = reinterpret_cast<const double*>(st + G::JI_BYTES)[t];
        if (q + 2 < NQP) {
            // every thread's generic reads of this stage precede the bulk refill
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (t == 0) issue(q + 2);
        }
        const double Lq[4] = {M.qb.L[q][0], M.qb.L[q][1], M.qb.L[q][2], M.qb.L[q][3]};
        double Gx[3][3], Gp[3][3], F[3][3], Hp[3][3];
        tet_dx_dxi_at<double, NPE>(
            [&](int a, int d) { return d == 0 ? xs[lc[a]] : (d == 1 ? ys[lc[a]] : zs[lc[a]]); }, Lq, Gx);
        tet_dx_dxi_at<double, NPE>([&](int a, int d) { return ps[3 * lc[a] + d]; }, Lq, Gp);
        mul_jinv(Gx, ji, F);
        mul_jinv(Gp, ji, Hp);
        double dP[3][3], Q[3][3];
        svk_tangent_dp(F, Hp, M.lambda, M.mu, dv, dP);
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
