// batch.cu -- batched linear-static solve: hundreds of independent meshes of
// uneven size and material solved by one persistent cooperative launch.
//
// The instances are concatenated into one mesh (instance-contiguous node
// numbering; tiles built instance by instance, so a tile holds one instance
// except where an instance ends mid-tile).  Material is carried per element
// slot, so a tile that straddles two instances is still exact.
//
// Per instance the iteration is the LinearStaticSolver CG (LinearStaticSolver.cu:
// 469-565): u = u0, r = f - K u0, p = r; alpha = rr / p.Kp (stop on p.Kp <= 0);
// u += alpha p; r -= alpha Kp; beta = rr_new / rr; p = r + beta p.  K is the
// linear (small-strain) stiffness at the reference configuration -- the
// tangent of compute_hessian_assemble_csr (FEAT10DataFunc.cuh:512-684) at F = I,
// applied matrix-free from the compact geometry stream (J^-1 and dV per QP),
// with Dirichlet DOFs eliminated as apply_bcs_kernel does
// (LinearStaticSolver.cu:284-306).  Stop rule: ||r|| / ||f_free|| < tol in FP64,
// which equals the reference's sqrt(rr / rr0) for a cold start and does not
// reward a warm start for a smaller initial residual.
//
// One launch runs every iteration of every instance: a grid-stride loop over
// element tiles (K p), then over node chunks, one warp per chunk (segmented FP64
// dots, vector updates); four grid barriers per iteration; the per-instance
// scalars of a phase are folded once, in chunk order, by the warp that posts
// the instance's last chunk partial.
//
// Shared-mesh mode: when every instance is the same mesh (only material and
// loads differ) the batch keeps ONE tiling and one geometry stream, and the
// tile loop runs over (tile, group of instances) items: the tile's tables are
// staged once per group, the geometry stream stays in L2, and HBM carries
// little more than the per-instance vectors.
#include <cooperative_groups.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "element.cuh"

namespace cg = cooperative_groups;

struct tlfea_batch_s {
    int type = TLFEA_TYPE_T10;
    int n_inst = 0;
    int N = 0, E = 0;  // combined mesh
    tlfea_element_s* el = nullptr;
    std::vector<int> node_off, elem_off;
    std::vector<double> inst_E, inst_nu;
    int precision = TLFEA_PRECISION_FP64;
    // device
    double *lam = nullptr, *mu = nullptr;  // per element slot (n_tiles * TILE_ELEMS), shared mode: per instance
    float *lam32 = nullptr, *mu32 = nullptr;
    bool shared = false;                   // every instance is one mesh (el holds it once)
    double* part64 = nullptr;              // shared mode: per-instance partial slots
    float* part32 = nullptr;
    unsigned char* fixed = nullptr;        // per node
    int* chunk_inst = nullptr;             // per chunk
    int* chunk_beg = nullptr;              // n_chunks + 1 node offsets
    int* inst_chunk = nullptr;             // n_inst + 1 chunk offsets
    int* tile_inst = nullptr;              // 2 per tile: first and last instance of its elements
    int n_chunks = 0;
    int chunk_nodes = 256;
    double *u = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *f = nullptr, *u0 = nullptr;
    double *cpa = nullptr, *cpb = nullptr;  // per-chunk partials
    double *rr = nullptr, *fnorm = nullptr, *rel = nullptr;  // rr: 2 * n_inst (iteration parity)
    int *iters = nullptr, *status = nullptr, *done = nullptr;
    int* n_done = nullptr;  // [0] instances done, [1] the per-phase launches' iteration counter
    double *alpha = nullptr, *beta = nullptr;  // per instance, folded once per phase
    int *flag = nullptr, *ticket = nullptr;    // per instance: 0 go, 1 converged, 2 broke down; fold tickets
    bool warm = false;
    bool material_set = false;
    // launch
    int mode = 0;           // 0 = per-phase kernels, 1 = one persistent cooperative launch
    int blocks_per_sm = 0;  // persistent launch: 0 = occupancy maximum
    cudaGraphExec_t graph = nullptr;  // the captured cold-start solve
    cudaGraphExec_t graph_w = nullptr;  // the captured warm-start solve
    double graph_tol = -1.0;
    int graph_max_iter = -1;
    int graph_grid = -1;
    int graph_precision = -1;
    // per-phase launches: captured chunks of iterations, keyed by what they bake in
    struct PhaseGraph {
        int precision, max_iter, iters;
        double tol;
        cudaGraphExec_t exec;
    };
    std::vector<PhaseGraph> phase_graphs;
    // FP32 element work: iterations summed over the refinement passes
    std::vector<int> iters_total;
    bool refined = false;
    double *rhs = nullptr, *uacc = nullptr;  // correction right-hand side, accumulated solution
};

// Captured launches of a batch are rebuilt whenever the launch shape changes.
static void drop_graphs(tlfea_batch_s* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->graph_w) cudaGraphExecDestroy(b->graph_w);
    b->graph = b->graph_w = nullptr;
    for (auto& g : b->phase_graphs) cudaGraphExecDestroy(g.exec);
    b->phase_graphs.clear();
}

namespace tlfea {

template <typename R>
struct BatchArgs {
    // tiling
    const int* node_off;
    const int* ln_gid;
    const int* ln_pslot;
    const uint16_t* ln_inc_end;
    const uint16_t* inc;
    const uint16_t* lconn;
    const R* grad;
    const R* ji;  // J^-1 per (tile, QP): the compact geometry stream
    const R* dv;
    const R* lam;
    const R* mu;
    R* partial;
    const int* node_bidx;
    const int* bnode_off;
    const int* bnode_slots;
    int n_tiles, max_local;  // n_tiles: work items (shared mode: instances x mesh tiles)
    // shared mode: every instance is one mesh of tiles_per_inst tiles, nodes_per_inst
    // nodes and pslots_per_inst partial slots; 0 otherwise
    int tiles_per_inst, nodes_per_inst, pslots_per_inst;
    // nodes and instances
    int N, n_inst, n_chunks;
    const unsigned char* fixed;
    const int* chunk_inst;
    const int* chunk_beg;
    const int* inst_chunk;
    const int* tile_inst;
    double *u, *r, *p, *q;
    const double* f;
    const double* u0;
    double *cpa, *cpb, *rr, *fnorm, *rel;
    int *iters, *status, *done, *n_done;
    double *alpha, *beta;
    int *flag, *ticket;
    int* it_dev;  // per-phase launches: the device-side iteration counter
    QpBary qb;
};

// q = K p on one tile: H = sum_a p_a (x) gradN_a, P = lambda tr(H) I + mu (H + H^T)
// (the SVK tangent at F = I), f_a += P gradN_a dV; element forces reduced per
// node in the tile's fixed incidence order.  Interior nodes are written to q,
// nodes shared with other tiles to their partial slot.
template <typename R, int NPE, int NQP>
__device__ __forceinline__ void linear_tile(const BatchArgs<R>& A, int item, const double* p, double* q,
                                            unsigned char* smem) {
    constexpr int TE = TILE_ELEMS;
    const int t = threadIdx.x;
    // work item -> mesh tile, and the instance's node and partial-slot offsets
    int tile = item, noff = 0, poff = 0, inst = 0;
    if (A.tiles_per_inst) {
        inst = item / A.tiles_per_inst;
        tile = item - inst * A.tiles_per_inst;
        noff = inst * A.nodes_per_inst;
        poff = inst * A.pslots_per_inst;
    }
    // shared memory: p at the local nodes, element forces, then the tile's
    // tables (node destination, incidence ends, incidence list) so the scatter
    // reads no global memory
    R* ps = reinterpret_cast<R*>(smem);  // 3 * max_local, interleaved
    R* fe = ps + 3 * A.max_local;        // 3 * NPE * TE
    int* dsts = reinterpret_cast<int*>(fe + 3 * NPE * TE);  // max_local: node id, or -(slot + 1)
    uint16_t* iends = reinterpret_cast<uint16_t*>(dsts + A.max_local);
    uint16_t* incs = iends + A.max_local;  // NPE * TE
    if (t == 0) {
        // the tile's J^-1 and dV stream (every QP) into L2 now, so the per-QP loads below
        // hit L2 instead of each waiting on DRAM (sizes are multiples of 16 bytes)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(A.ji + (size_t)tile * NQP * 9 * TE),
                     "r"((uint32_t)(NQP * 9 * TE * sizeof(R)))
                     : "memory");
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(A.dv + (size_t)tile * NQP * TE),
                     "r"((uint32_t)(NQP * TE * sizeof(R)))
                     : "memory");
    }
    const int lb = A.node_off[tile], nl = A.node_off[tile + 1] - lb;
    for (int k = t; k < NPE * TE; k += TE) incs[k] = A.inc[(size_t)tile * TE * NPE + k];
    // FP32: p relative to the tile's first node, differenced in FP64: the gradients
    // sum to zero over an element's nodes, so K p is unchanged, but the FP32
    // copy no longer carries the (large, cancelling) common part of p and H =
    // sum_a p_a (x) grad N_a keeps FP32 accuracy relative to the local variation.
    // FP64 stages p as it is (no dependent loads before the gathers).
    double r0 = 0.0, r1 = 0.0, r2 = 0.0;
    if constexpr (sizeof(R) == 4) {
        const int g0 = noff + A.ln_gid[lb];
        r0 = p[3 * g0 + 0];
        r1 = p[3 * g0 + 1];
        r2 = p[3 * g0 + 2];
    }
#pragma unroll 4
    for (int ln = t; ln < nl; ln += TE) {  // unrolled: several nodes' gathers in flight at once
        const int gid = noff + A.ln_gid[lb + ln];
        const int pslot = A.ln_pslot[lb + ln];
        dsts[ln] = (pslot < 0) ? gid : -(poff + pslot + 1);
        iends[ln] = A.ln_inc_end[lb + ln];
        ps[3 * ln + 0] = R(p[3 * gid + 0] - r0);
        ps[3 * ln + 1] = R(p[3 * gid + 1] - r1);
        ps[3 * ln + 2] = R(p[3 * gid + 2] - r2);
    }
    int lc[NPE];
#pragma unroll
    for (int a = 0; a < NPE; ++a) lc[a] = A.lconn[((size_t)tile * NPE + a) * TE + t];
    const R lam = A.tiles_per_inst ? A.lam[inst] : A.lam[(size_t)tile * TE + t];
    const R mu = A.tiles_per_inst ? A.mu[inst] : A.mu[(size_t)tile * TE + t];
#pragma unroll
    for (int a = 0; a < NPE; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) fe[(a * 3 + d) * TE + t] = R(0);
    __syncthreads();
#pragma unroll 1
    for (int qp = 0; qp < NQP; ++qp) {
        R xa[NPE][3];
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
            for (int d = 0; d < 3; ++d) xa[a][d] = ps[3 * lc[a] + d];
        const R* jp = A.ji + ((size_t)tile * NQP + qp) * 9 * TE + t;
        const R* dp = A.dv + ((size_t)tile * NQP + qp) * TE + t;
        R ji[9];
        R dv;
        if (A.tiles_per_inst) {
            // shared mesh: every instance re-reads this geometry, keep it in L2
#pragma unroll
            for (int m = 0; m < 9; ++m) ji[m] = __ldg(jp + m * TE);
            dv = __ldg(dp);
        } else {
            // one instance per tile: a single pass, stream past L2
#pragma unroll
            for (int m = 0; m < 9; ++m) ji[m] = __ldcs(jp + m * TE);
            dv = __ldcs(dp);
        }
        const R L[4] = {R(A.qb.L[qp][0]), R(A.qb.L[qp][1]), R(A.qb.L[qp][2]), R(A.qb.L[qp][3])};
        R G[3][3], H[3][3];
        tet_dx_dxi<R, NPE>(xa, L, G);
        mul_jinv(G, ji, H);
        const R tr = lam * (H[0][0] + H[1][1] + H[2][2]);
        R P[3][3], Q[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) P[i][j] = (mu * (H[i][j] + H[j][i]) + (i == j ? tr : R(0))) * dv;
        mul_jinv_t(P, ji, Q);
        tet_scatter<R, NPE>(Q, L, [&](int a, int d, R v) { fe[(a * 3 + d) * TE + t] += v; });
    }
    __syncthreads();
    for (int ln = t; ln < nl; ln += TE) {
        const int beg = ln ? iends[ln - 1] : 0;
        const int end = iends[ln];
        R s0 = R(0), s1 = R(0), s2 = R(0);
        for (int k = beg; k < end; ++k) {
            const int ent = incs[k];
            const int base = (ent >> TILE_SHIFT) * 3 * TE + (ent & (TE - 1));
            s0 += fe[base];
            s1 += fe[base + TE];
            s2 += fe[base + 2 * TE];
        }
        const int dn = dsts[ln];
        if (dn >= 0) {
            q[3 * dn + 0] = double(s0);
            q[3 * dn + 1] = double(s1);
            q[3 * dn + 2] = double(s2);
        } else {
            R* pt = A.partial + 3 * (size_t)(-dn - 1);
            pt[0] = s0;
            pt[1] = s1;
            pt[2] = s2;
        }
    }
    __syncthreads();  // smem reused by the next tile
}

// Complete K p at node i: boundary nodes sum their tile partials in tile
// order; fixed nodes get 0 (eliminated rows and columns).
template <typename R>
__device__ __forceinline__ void node_kp(const BatchArgs<R>& A, int i, double* q, double out[3]) {
    if (A.fixed[i]) {
        out[0] = out[1] = out[2] = 0.0;
    } else {
        int local = i, poff = 0;
        if (A.tiles_per_inst) {
            const int inst = i / A.nodes_per_inst;
            local = i - inst * A.nodes_per_inst;
            poff = inst * A.pslots_per_inst;
        }
        const int b = A.node_bidx[local];
        if (b < 0) {
            out[0] = q[3 * i + 0];
            out[1] = q[3 * i + 1];
            out[2] = q[3 * i + 2];
        } else {
            R s0 = R(0), s1 = R(0), s2 = R(0);
            for (int k = A.bnode_off[b]; k < A.bnode_off[b + 1]; ++k) {
                const int sl = poff + k;  // partial slots are numbered by shared node
                s0 += __ldcg(A.partial + 3 * sl + 0);
                s1 += __ldcg(A.partial + 3 * sl + 1);
                s2 += __ldcg(A.partial + 3 * sl + 2);
            }
            out[0] = double(s0);
            out[1] = double(s1);
            out[2] = double(s2);
        }
    }
    q[3 * i + 0] = out[0];
    q[3 * i + 1] = out[1];
    q[3 * i + 2] = out[2];
}

// Sum of the chunk partials of instance b, folded by one warp in a fixed order
// (any warp computing it gets the same bits, in every lane).
__device__ __forceinline__ double inst_sum(const double* part, const int* inst_chunk, int b) {
    double s = 0.0;
    for (int c = inst_chunk[b] + (threadIdx.x & 31); c < inst_chunk[b + 1]; c += 32) s += __ldcg(part + c);
    return warp_sum(s);
}

// Shared-mesh mode: one mesh tile for a group of SHARED_GROUP instances.  The
// tile's tables (incidence, node ids, partial slots, local connectivity) are
// staged once for the group; each active instance's p is gathered with cp.async
// into one of two buffers while the previous instance is computed and
// scattered, so the gather latency overlaps the element work.
constexpr int SHARED_GROUP = 8;

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Byte offsets of the group tile's shared memory (16-byte aligned regions).
template <typename R, int NPE>
struct GroupLayout {
    size_t fe, gid, slot, iend, inc, total;
    __host__ __device__ GroupLayout(int ml) {
        auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
        fe = al(2 * 3 * (size_t)ml * sizeof(double));  // two gather buffers first
        gid = al(fe + 3 * (size_t)NPE * TILE_ELEMS * sizeof(R));
        slot = al(gid + (size_t)ml * sizeof(int));
        iend = al(slot + (size_t)ml * sizeof(int));
        inc = al(iend + (size_t)ml * sizeof(uint16_t));
        total = inc + (size_t)NPE * TILE_ELEMS * sizeof(uint16_t);
    }
};

template <typename R, int NPE, int NQP>
__device__ __forceinline__ void shared_group_tile(const BatchArgs<R>& A, int tile, int g0, const double* p, double* q,
                                                  unsigned char* smem, bool skip_done) {
    constexpr int TE = TILE_ELEMS;
    const int t = threadIdx.x;
    const int ml = A.max_local;
    const GroupLayout<R, NPE> L(ml);
    double* psb = reinterpret_cast<double*>(smem);
    R* fe = reinterpret_cast<R*>(smem + L.fe);
    int* gid_s = reinterpret_cast<int*>(smem + L.gid);
    int* slot_s = reinterpret_cast<int*>(smem + L.slot);
    uint16_t* iends = reinterpret_cast<uint16_t*>(smem + L.iend);
    uint16_t* incs = reinterpret_cast<uint16_t*>(smem + L.inc);
    const int g1 = min(g0 + SHARED_GROUP, A.n_inst);
    // next instance of the group to compute (done[] is stable in this phase)
    auto next_active = [&](int from) -> int {
        for (int i = from; i < g1; ++i)
            if (!skip_done || !__ldcg(A.done + i)) return i;
        return -1;
    };
    int cur = next_active(g0);
    if (cur < 0) return;  // uniform: every thread read the same flags
    const int lb = A.node_off[tile], nl = A.node_off[tile + 1] - lb;
    for (int k = t; k < NPE * TE; k += TE) incs[k] = A.inc[(size_t)tile * TE * NPE + k];
    for (int ln = t; ln < nl; ln += TE) {
        const int gid = A.ln_gid[lb + ln];
        gid_s[ln] = gid;
        slot_s[ln] = A.ln_pslot[lb + ln];
        iends[ln] = A.ln_inc_end[lb + ln];
        // this thread's own gathers of the first instance start right away
        const double* src = p + 3 * ((size_t)cur * A.nodes_per_inst + gid);
#pragma unroll
        for (int d = 0; d < 3; ++d) cp_async8(psb + 3 * ln + d, src + d);
    }
    cp_async_commit();
    int lc[NPE];
#pragma unroll
    for (int a = 0; a < NPE; ++a) lc[a] = A.lconn[((size_t)tile * NPE + a) * TE + t];
    __syncthreads();  // node tables staged (the next gathers read gid_s)
    int buf = 0;
    while (cur >= 0) {
        const int nxt = next_active(cur + 1);
        if (nxt >= 0) {
            double* dst = psb + (buf ^ 1) * 3 * ml;
            for (int ln = t; ln < nl; ln += TE) {
                const double* src = p + 3 * ((size_t)nxt * A.nodes_per_inst + gid_s[ln]);
#pragma unroll
                for (int d = 0; d < 3; ++d) cp_async8(dst + 3 * ln + d, src + d);
            }
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();  // instance cur's p visible in buffer buf
        const double* ps = psb + buf * 3 * ml;
        const R lam = A.lam[cur], mu = A.mu[cur];
        // FP32: p relative to the tile's first node, differenced in FP64 (the
        // gradients sum to zero per element, so K p is unchanged)
        double r0 = 0.0, r1 = 0.0, r2 = 0.0;
        if constexpr (sizeof(R) == 4) {
            r0 = ps[0];
            r1 = ps[1];
            r2 = ps[2];
        }
        R f[NPE][3];
        // p at the element's nodes is read from the gather buffer where tet_dx_dxi_at uses
        // it (holding those 30 values in registers beside the element forces cost a third
        // of the resident blocks; accumulating the forces in shared memory instead was
        // slower still)
        const double rr[3] = {r0, r1, r2};
        auto xa = [&](int a, int d) -> R { return R(ps[3 * lc[a] + d] - rr[d]); };
#pragma unroll 1
        for (int qp = 0; qp < NQP; ++qp) {
            const R* jp = A.ji + ((size_t)tile * NQP + qp) * 9 * TE + t;
            R ji[9];
#pragma unroll
            for (int m = 0; m < 9; ++m) ji[m] = __ldg(jp + m * TE);
            const R dv = __ldg(A.dv + ((size_t)tile * NQP + qp) * TE + t);
            const R Lq[4] = {R(A.qb.L[qp][0]), R(A.qb.L[qp][1]), R(A.qb.L[qp][2]), R(A.qb.L[qp][3])};
            R G[3][3], H[3][3];
            tet_dx_dxi_at<R, NPE>(xa, Lq, G);
            mul_jinv(G, ji, H);
            const R tr = lam * (H[0][0] + H[1][1] + H[2][2]);
            R P[3][3], Q[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) P[i][j] = (mu * (H[i][j] + H[j][i]) + (i == j ? tr : R(0))) * dv;
            mul_jinv_t(P, ji, Q);
            if (qp == 0)
                tet_scatter<R, NPE>(Q, Lq, [&](int a, int d, R v) { f[a][d] = v; });
            else
                tet_scatter<R, NPE>(Q, Lq, [&](int a, int d, R v) { f[a][d] += v; });
        }
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
            for (int d = 0; d < 3; ++d) fe[(a * 3 + d) * TE + t] = f[a][d];
        __syncthreads();  // element forces complete
        const size_t noff = (size_t)cur * A.nodes_per_inst, poff = (size_t)cur * A.pslots_per_inst;
        for (int ln = t; ln < nl; ln += TE) {
            const int beg = ln ? iends[ln - 1] : 0;
            const int end = iends[ln];
            R s0 = R(0), s1 = R(0), s2 = R(0);
            for (int k = beg; k < end; ++k) {
                const int ent = incs[k];
                const int base = (ent >> TILE_SHIFT) * 3 * TE + (ent & (TE - 1));
                s0 += fe[base];
                s1 += fe[base + TE];
                s2 += fe[base + 2 * TE];
            }
            const int sl = slot_s[ln];
            if (sl < 0) {
                double* qd = q + 3 * (noff + gid_s[ln]);
                qd[0] = double(s0);
                qd[1] = double(s1);
                qd[2] = double(s2);
            } else {
                R* pt = A.partial + 3 * (poff + sl);
                pt[0] = s0;
                pt[1] = s1;
                pt[2] = s2;
            }
        }
        __syncthreads();  // forces and buffer buf free for reuse
        cur = nxt;
        buf ^= 1;
    }
}

// K p over every tile; with skip_done, tiles whose instances have all
// converged are skipped (their q is never read again).  The done flags do not
// change during this phase, so the skip is uniform across the block.
template <typename R, int NPE, int NQP>
__device__ __forceinline__ void general_tiles(const BatchArgs<R>& A, const double* p, double* q, unsigned char* smem,
                                              bool skip_done) {
    for (int tile = blockIdx.x; tile < A.n_tiles; tile += gridDim.x) {
        if (skip_done) {
            bool all_done = true;
            if (A.tiles_per_inst) {
                all_done = __ldcg(A.done + tile / A.tiles_per_inst) != 0;
            } else {
                for (int i = A.tile_inst[2 * tile]; i <= A.tile_inst[2 * tile + 1] && all_done; ++i)
                    all_done = __ldcg(A.done + i) != 0;
            }
            if (all_done) continue;
        }
        linear_tile<R, NPE, NQP>(A, tile, p, q, smem);
    }
}

// SH: the shared-mesh instantiation (instance groups per tile); the general one
// keeps its lower register count, and so its occupancy, for uneven batches.
template <typename R, int NPE, int NQP, bool SH>
__device__ __forceinline__ void apply_all_tiles(const BatchArgs<R>& A, const double* p, double* q,
                                                unsigned char* smem, bool skip_done) {
    if constexpr (SH) {
        const int T = A.tiles_per_inst;
        const int n_items = T * ((A.n_inst + SHARED_GROUP - 1) / SHARED_GROUP);
        for (int item = blockIdx.x; item < n_items; item += gridDim.x)
            shared_group_tile<R, NPE, NQP>(A, item % T, (item / T) * SHARED_GROUP, p, q, smem, skip_done);
    } else {
        general_tiles<R, NPE, NQP>(A, p, q, smem, skip_done);
    }
}

// ---------------------------------------------------------------------------
// The phases of the batched CG.  Each is a grid-stride loop, so the persistent
// kernel (one cooperative launch, grid barriers between phases) and the
// per-phase kernels (one launch per phase, stream order between them) run the
// same code.  Chunk phases run one block per chunk; node phases of an iteration
// run one warp per chunk (no block barriers): a chunk's partial is the warp's
// lane-strided sum folded by shuffles, so its bits are fixed.

// u = u0 (warm) or 0, r = f_free, p = u; ||f_free||^2 per chunk into cpa.
template <typename R>
__device__ __forceinline__ void bcg_start(const BatchArgs<R>& A, int warm, double* red) {
    const int t = threadIdx.x;
    for (int c = blockIdx.x; c < A.n_chunks; c += gridDim.x) {
        double sf = 0.0;
        for (int i = A.chunk_beg[c] + t; i < A.chunk_beg[c + 1]; i += blockDim.x) {
            const bool fx = A.fixed[i];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double fi = fx ? 0.0 : A.f[3 * i + d];
                const double ui = (warm && !fx) ? A.u0[3 * i + d] : 0.0;
                A.r[3 * i + d] = fi;
                A.u[3 * i + d] = ui;
                A.p[3 * i + d] = ui;
                sf += fi * fi;
            }
        }
        const double s = block_sum(sf, red);
        if (t == 0) A.cpa[c] = s;
    }
}

// r -= K u0 (warm: q holds K p with p = u0), p = r; ||r||^2 per chunk into cpb.
template <typename R>
__device__ __forceinline__ void bcg_start_residual(const BatchArgs<R>& A, int warm, double* red) {
    const int t = threadIdx.x;
    for (int c = blockIdx.x; c < A.n_chunks; c += gridDim.x) {
        double sr = 0.0;
        for (int i = A.chunk_beg[c] + t; i < A.chunk_beg[c + 1]; i += blockDim.x) {
            double kp[3] = {0.0, 0.0, 0.0};
            if (warm) node_kp<R>(A, i, A.q, kp);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double ri = A.r[3 * i + d] - kp[d];
                A.r[3 * i + d] = ri;
                A.p[3 * i + d] = ri;
                sr += ri * ri;
            }
        }
        const double s = block_sum(sr, red);
        if (t == 0) A.cpb[c] = s;
    }
}

// Per instance: ||f_free||, rr_0, the initial relative residual and the start state.
template <typename R>
__device__ __forceinline__ void bcg_init(const BatchArgs<R>& A, double tol) {
    const int t = threadIdx.x;
    for (int b = blockIdx.x; b < A.n_inst; b += gridDim.x) {
        if (t < 32) {
            const double ff = inst_sum(A.cpa, A.inst_chunk, b);
            const double rr0 = inst_sum(A.cpb, A.inst_chunk, b);
            if (t == 0) {
                const double fn = sqrt(ff);
                const double rel = (fn > 0.0) ? sqrt(rr0) / fn : 0.0;
                A.fnorm[b] = fn;
                A.rr[b] = rr0;
                A.rel[b] = rel;
                A.iters[b] = 0;
                A.status[b] = 0;
                A.flag[b] = 0;
                A.ticket[b] = 0;
                const int dn = (fn == 0.0 || rel < tol) ? 1 : 0;
                A.done[b] = dn;
                if (dn) atomicAdd(A.n_done, 1);
            }
        }
    }
}

// Post a chunk's partial; true (in every lane) for the warp whose post completes the
// instance.  The per-instance scalars of a phase are folded once, in chunk order, by
// that warp (a ticket per instance), so their bits do not depend on which warp it is.
template <typename R>
__device__ __forceinline__ bool bcg_post_last(const BatchArgs<R>& A, double* part, int c, int b, double s) {
    const int lane = threadIdx.x & 31;
    int last = 0;
    if (lane == 0) {
        part[c] = s;
        __threadfence();
        const int nch = A.inst_chunk[b + 1] - A.inst_chunk[b];
        const int tk = atomicAdd(A.ticket + b, 1);
        last = (tk == nch - 1);
        if (last) A.ticket[b] = 0;  // every ticket of this phase is taken
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) __threadfence();
    return last != 0;
}

// Complete q = K p at the nodes (partials of shared nodes, zero at fixed ones), p.q
// per chunk; alpha = rr / p.q per instance (iteration `it`).
template <typename R>
__device__ __forceinline__ void bcg_pq(const BatchArgs<R>& A, int it) {
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), n_warps = gridDim.x * (blockDim.x / 32);
    const double* rr_old = A.rr + (size_t)(it & 1) * A.n_inst;
    for (int c = gw; c < A.n_chunks; c += n_warps) {
        const int b = A.chunk_inst[c];
        const int i_end = A.chunk_beg[c + 1];
        if (__ldcg(A.done + b)) continue;
        double s = 0.0;
        // two nodes per lane per step: every load of both is issued before
        // the first use (the chunk's nodes all belong to instance b)
        const int noff = A.tiles_per_inst ? b * A.nodes_per_inst : 0;
        const int poff = A.tiles_per_inst ? b * A.pslots_per_inst : 0;
        for (int i0 = A.chunk_beg[c] + lane; i0 < i_end; i0 += 64) {
            double pv[2][3], qv[2][3];
            int fx[2], bi[2];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int i = i0 + 32 * k;
                const bool ok = i < i_end;
                fx[k] = ok ? A.fixed[i] : 1;
                bi[k] = ok ? A.node_bidx[i - noff] : -1;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    pv[k][d] = ok ? __ldcg(A.p + 3 * i + d) : 0.0;
                    qv[k][d] = ok ? __ldcg(A.q + 3 * i + d) : 0.0;
                }
            }
            int kb[2], ke[2];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                kb[k] = (bi[k] >= 0) ? A.bnode_off[bi[k]] : 0;
                ke[k] = (bi[k] >= 0) ? A.bnode_off[bi[k] + 1] : 0;
            }
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int i = i0 + 32 * k;
                if (bi[k] >= 0) {
                    R s0 = R(0), s1 = R(0), s2 = R(0);
                    for (int m = kb[k]; m < ke[k]; ++m) {
                        const R* pt = A.partial + 3 * (size_t)(poff + m);
                        s0 += __ldcg(pt + 0);
                        s1 += __ldcg(pt + 1);
                        s2 += __ldcg(pt + 2);
                    }
                    qv[k][0] = double(s0);
                    qv[k][1] = double(s1);
                    qv[k][2] = double(s2);
                }
                if (fx[k]) qv[k][0] = qv[k][1] = qv[k][2] = 0.0;
                if (i < i_end) {
#pragma unroll
                    for (int d = 0; d < 3; ++d) A.q[3 * i + d] = qv[k][d];
                }
                s += pv[k][0] * qv[k][0] + pv[k][1] * qv[k][1] + pv[k][2] * qv[k][2];
            }
        }
        s = warp_sum(s);
        if (bcg_post_last(A, A.cpa, c, b, s)) {
            const double pq = inst_sum(A.cpa, A.inst_chunk, b);
            if (lane == 0) {
                // non-positive p.Kp: the reference aborts this solve (flag 2)
                A.alpha[b] = (pq > 0.0) ? __ldcg(rr_old + b) / pq : 0.0;
                A.flag[b] = (pq > 0.0) ? 0 : 2;
            }
        }
    }
}

// u += alpha p; r -= alpha q; r.r per chunk; then rr_new, the test and beta.
template <typename R>
__device__ __forceinline__ void bcg_update(const BatchArgs<R>& A, int it, double tol, int max_iter) {
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), n_warps = gridDim.x * (blockDim.x / 32);
    const double* rr_old = A.rr + (size_t)(it & 1) * A.n_inst;
    double* rr_new_out = A.rr + (size_t)((it + 1) & 1) * A.n_inst;
    for (int c = gw; c < A.n_chunks; c += n_warps) {
        const int b = A.chunk_inst[c];
        const int dn = __ldcg(A.done + b), fl = __ldcg(A.flag + b);  // loads issued together
        const double alpha = __ldcg(A.alpha + b);
        if (dn || fl == 2) continue;
        double s = 0.0;
        // flat over the chunk's 3n values, eight per lane per step with every
        // load issued before the first store
        const int j1 = 3 * A.chunk_beg[c + 1];
        for (int j0 = 3 * A.chunk_beg[c] + lane; j0 < j1; j0 += 256) {
            double uv[8], pv[8], rv[8], qv[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int j = j0 + 32 * k;
                const bool ok = j < j1;
                uv[k] = ok ? __ldcg(A.u + j) : 0.0;
                pv[k] = ok ? __ldcg(A.p + j) : 0.0;
                rv[k] = ok ? __ldcg(A.r + j) : 0.0;
                qv[k] = ok ? __ldcg(A.q + j) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int j = j0 + 32 * k;
                const double rj = rv[k] - alpha * qv[k];
                if (j < j1) {
                    A.u[j] = uv[k] + alpha * pv[k];
                    A.r[j] = rj;
                }
                s += rj * rj;
            }
        }
        s = warp_sum(s);
        if (bcg_post_last(A, A.cpb, c, b, s)) {
            const double rrn = inst_sum(A.cpb, A.inst_chunk, b);
            if (lane == 0) {
                const double rel = sqrt(rrn) / __ldcg(A.fnorm + b);
                const bool conv = rel < tol;
                rr_new_out[b] = rrn;
                A.beta[b] = rrn / __ldcg(rr_old + b);
                A.iters[b] = it + 1;
                A.rel[b] = rel;
                A.flag[b] = conv ? 1 : 0;
                if (!conv && it + 1 >= max_iter) A.status[b] = 2;
            }
        }
    }
}

// p = r + beta p; instances that converged or broke down retire (their first chunk
// sets done; every warp skips them either way).
template <typename R>
__device__ __forceinline__ void bcg_direction(const BatchArgs<R>& A) {
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), n_warps = gridDim.x * (blockDim.x / 32);
    for (int c = gw; c < A.n_chunks; c += n_warps) {
        const int b = A.chunk_inst[c];
        const int dn = __ldcg(A.done + b), fl = __ldcg(A.flag + b);  // loads issued together
        const double beta = __ldcg(A.beta + b);
        if (dn) continue;
        if (fl == 0) {
            const int j1 = 3 * A.chunk_beg[c + 1];
            for (int j0 = 3 * A.chunk_beg[c] + lane; j0 < j1; j0 += 256) {
                double pv[8], rv[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int j = j0 + 32 * k;
                    pv[k] = (j < j1) ? __ldcg(A.p + j) : 0.0;
                    rv[k] = (j < j1) ? __ldcg(A.r + j) : 0.0;
                }
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int j = j0 + 32 * k;
                    if (j < j1) A.p[j] = rv[k] + beta * pv[k];
                }
            }
        } else if (lane == 0 && c == A.inst_chunk[b]) {
            if (fl == 2) A.status[b] = 1;
            A.done[b] = 1;
            atomicAdd(A.n_done, 1);
        }
    }
}

// Instances still running when the iteration cap is reached end with status 2.
template <typename R>
__device__ __forceinline__ void bcg_finish(const BatchArgs<R>& A) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < A.n_inst; b += gridDim.x * blockDim.x)
        if (!A.done[b] && A.status[b] == 0) A.status[b] = 2;
}

// The whole batched solve in one persistent cooperative launch (launch mode 1).
template <typename R, int NPE, int NQP, bool SH>
__global__ void __launch_bounds__(TILE_ELEMS) k_batch_cg(BatchArgs<R> A, double tol, int max_iter, int warm) {
    cg::grid_group grid = cg::this_grid();
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double red[32];
    bcg_start<R>(A, warm, red);
    grid.sync();
    if (warm) {
        apply_all_tiles<R, NPE, NQP, SH>(A, A.p, A.q, smem, false);
        grid.sync();
    }
    bcg_start_residual<R>(A, warm, red);
    grid.sync();
    bcg_init<R>(A, tol);
    grid.sync();
    // done[] changes only in the last phase of an iteration, so every other phase
    // branches on it uniformly
    for (int it = 0; it < max_iter; ++it) {
        if (atomicAdd(A.n_done, 0) >= A.n_inst) break;  // uniform: read after a grid barrier
        apply_all_tiles<R, NPE, NQP, SH>(A, A.p, A.q, smem, true);
        grid.sync();
        bcg_pq<R>(A, it);
        grid.sync();
        bcg_update<R>(A, it, tol, max_iter);
        grid.sync();
        bcg_direction<R>(A);
        grid.sync();
    }
    bcg_finish<R>(A);
}

// ---------------------------------------------------------------------------
// Per-phase kernels (launch mode 0, the default): each phase one launch at the
// occupancy its own registers allow -- the element tiles one item per block, the
// node phases one warp per chunk -- and an iteration is five launches: tiles,
// p.q, update, direction, and a one-thread kernel that advances the device-side
// iteration counter.  Chunks of iterations are captured in a CUDA graph and
// replayed until every instance is done or the cap is reached; a kernel whose
// iteration is past the cap, or that finds every instance done, returns at entry,
// so a replay that overshoots costs a few empty launches.
template <typename R>
__global__ void __launch_bounds__(TILE_ELEMS) k_bcg_start(BatchArgs<R> A, int warm) {
    __shared__ double red[32];
    bcg_start<R>(A, warm, red);
}

template <typename R>
__global__ void __launch_bounds__(TILE_ELEMS) k_bcg_start_residual(BatchArgs<R> A, int warm) {
    __shared__ double red[32];
    bcg_start_residual<R>(A, warm, red);
}

template <typename R>
__global__ void __launch_bounds__(TILE_ELEMS) k_bcg_init(BatchArgs<R> A, double tol) {
    bcg_init<R>(A, tol);
}

__device__ __forceinline__ bool bcg_idle(const int* it_dev, const int* n_done, int n_inst, int max_iter) {
    return __ldcg(n_done) >= n_inst || __ldcg(it_dev) >= max_iter;
}

// skip_done = 0: the warm start's K u0, before the iterations
template <typename R, int NPE, int NQP, bool SH>
__global__ void __launch_bounds__(TILE_ELEMS) k_bcg_tiles(BatchArgs<R> A, int skip_done, int max_iter) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (skip_done && bcg_idle(A.it_dev, A.n_done, A.n_inst, max_iter)) return;
    apply_all_tiles<R, NPE, NQP, SH>(A, A.p, A.q, smem, skip_done != 0);
}

template <typename R>
__global__ void __launch_bounds__(TILE_ELEMS) k_bcg_pq(BatchArgs<R> A, int max_iter) {
    if (bcg_idle(A.it_dev, A.n_done, A.n_inst, max_iter)) return;
    bcg_pq<R>(A, __ldcg(A.it_dev));
}

template <typename R>
__global__ void __launch_bounds__(TILE_ELEMS) k_bcg_update(BatchArgs<R> A, double tol, int max_iter) {
    if (bcg_idle(A.it_dev, A.n_done, A.n_inst, max_iter)) return;
    bcg_update<R>(A, __ldcg(A.it_dev), tol, max_iter);
}

// n_done may reach n_inst while this kernel runs (its own retirements); a block that
// then returns at entry has nothing left to retire
template <typename R>
__global__ void __launch_bounds__(TILE_ELEMS) k_bcg_direction(BatchArgs<R> A, int max_iter) {
    if (bcg_idle(A.it_dev, A.n_done, A.n_inst, max_iter)) return;
    bcg_direction<R>(A);
}

__global__ void k_bcg_next(int* it_dev, const int* n_done, int n_inst, int max_iter) {
    if (*n_done < n_inst && *it_dev < max_iter) ++*it_dev;
}

template <typename R>
__global__ void k_bcg_finish(BatchArgs<R> A) {
    bcg_finish<R>(A);
}

// y = K_bc x for the whole batch: fixed rows are identity rows and fixed
// columns are dropped (the BC-applied K of LinearStaticSolver::Apply).
template <typename R, int NPE, int NQP, bool SH>
__global__ void __launch_bounds__(TILE_ELEMS) k_batch_apply(BatchArgs<R> A, const double* x, double* y) {
    cg::grid_group grid = cg::this_grid();
    extern __shared__ __align__(16) unsigned char smem[];
    const int t = threadIdx.x;
    for (int i = blockIdx.x * blockDim.x + t; i < A.N; i += gridDim.x * blockDim.x)
#pragma unroll
        for (int d = 0; d < 3; ++d) A.p[3 * i + d] = A.fixed[i] ? 0.0 : x[3 * i + d];
    grid.sync();
    apply_all_tiles<R, NPE, NQP, SH>(A, A.p, A.q, smem, false);
    grid.sync();
    for (int i = blockIdx.x * blockDim.x + t; i < A.N; i += gridDim.x * blockDim.x) {
        double kp[3];
        node_kp<R>(A, i, A.q, kp);
#pragma unroll
        for (int d = 0; d < 3; ++d) y[3 * i + d] = A.fixed[i] ? x[3 * i + d] : kp[d];
    }
}

template <typename R>
static BatchArgs<R> batch_args(tlfea_batch_s* b) {
    tlfea_element_s* el = b->el;
    const Tiling& tl = el->tl;
    BatchArgs<R> A;
    A.node_off = tl.node_off;
    A.ln_gid = tl.ln_gid;
    A.ln_pslot = tl.ln_pslot;
    A.ln_inc_end = tl.ln_inc_end;
    A.inc = tl.inc;
    A.lconn = tl.lconn;
    if constexpr (sizeof(R) == 8) {
        A.grad = tl.grad64;
        A.ji = tl.ji64;
        A.dv = tl.dv64;
        A.lam = b->lam;
        A.mu = b->mu;
        A.partial = b->shared ? b->part64 : tl.partial64;
    } else {
        A.grad = tl.grad32;
        A.ji = tl.ji32;
        A.dv = tl.dv32;
        A.lam = b->lam32;
        A.mu = b->mu32;
        A.partial = b->shared ? b->part32 : tl.partial32;
    }
    A.node_bidx = tl.node_bidx;
    A.bnode_off = tl.bnode_off;
    A.bnode_slots = tl.bnode_slots;
    A.qb = qp_bary(el);
    A.n_tiles = b->shared ? tl.n_tiles * b->n_inst : tl.n_tiles;
    A.tiles_per_inst = b->shared ? tl.n_tiles : 0;
    A.nodes_per_inst = b->shared ? el->N : 0;
    A.pslots_per_inst = b->shared ? tl.n_pslots : 0;
    A.max_local = tl.max_local;
    A.N = b->N;
    A.n_inst = b->n_inst;
    A.n_chunks = b->n_chunks;
    A.fixed = b->fixed;
    A.chunk_inst = b->chunk_inst;
    A.chunk_beg = b->chunk_beg;
    A.inst_chunk = b->inst_chunk;
    A.tile_inst = b->tile_inst;
    A.u = b->u;
    A.r = b->r;
    A.p = b->p;
    A.q = b->q;
    A.f = b->f;
    A.u0 = b->u0;
    A.cpa = b->cpa;
    A.cpb = b->cpb;
    A.rr = b->rr;
    A.fnorm = b->fnorm;
    A.rel = b->rel;
    A.iters = b->iters;
    A.status = b->status;
    A.done = b->done;
    A.n_done = b->n_done;
    A.alpha = b->alpha;
    A.beta = b->beta;
    A.flag = b->flag;
    A.ticket = b->ticket;
    A.it_dev = b->n_done + 1;
    return A;
}

template <typename R>
static size_t batch_smem(const tlfea_batch_s* b) {
    const size_t ml = (size_t)b->el->tl.max_local;
    if (b->shared)
        return (b->el->npe == 10) ? GroupLayout<R, 10>((int)ml).total : GroupLayout<R, 4>((int)ml).total;
    return sizeof(R) * (3 * ml + 3 * (size_t)b->el->npe * TILE_ELEMS) + ml * (sizeof(int) + sizeof(uint16_t)) +
           (size_t)b->el->npe * TILE_ELEMS * sizeof(uint16_t);
}

// The kernel instantiation of this batch (shared-mesh or general).
template <typename R, int NPE, int NQP>
static const void* batch_kernel(const tlfea_batch_s* b, bool apply) {
    if (b->shared)
        return apply ? (const void*)k_batch_apply<R, NPE, NQP, true> : (const void*)k_batch_cg<R, NPE, NQP, true>;
    return apply ? (const void*)k_batch_apply<R, NPE, NQP, false> : (const void*)k_batch_cg<R, NPE, NQP, false>;
}

template <typename R, int NPE, int NQP>
static int batch_grid(tlfea_batch_s* b, int blocks_per_sm, int* grid_out, bool apply = false) {
    const void* kern = batch_kernel<R, NPE, NQP>(b, apply);
    const size_t smem = batch_smem<R>(b);
    if (smem > 200 * 1024) {
        set_error("batch: a tile touches too many nodes for shared memory");
        return TLFEA_UNSUPPORTED;
    }
    TLFEA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, sms = 0;
    TLFEA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TILE_ELEMS, smem));
    TLFEA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->el->device));
    if (per_sm < 1) {
        set_error("batch kernel does not fit on an SM");
        return TLFEA_UNSUPPORTED;
    }
    if (blocks_per_sm > 0) per_sm = std::min(per_sm, blocks_per_sm);
    *grid_out = per_sm * sms;
    return TLFEA_OK;
}

template <typename R, int NPE, int NQP>
static int launch_batch_cg(tlfea_batch_s* b, int grid, double tol, int max_iter, bool warm, cudaStream_t st,
                           const double* f_over = nullptr, const double* u0_over = nullptr) {
    BatchArgs<R> A = batch_args<R>(b);
    if (f_over) A.f = f_over;
    if (u0_over) A.u0 = u0_over;
    int w = warm ? 1 : 0;
    void* args[] = {&A, &tol, &max_iter, &w};
    TLFEA_CUDA(cudaLaunchCooperativeKernel(batch_kernel<R, NPE, NQP>(b, false), dim3(grid), dim3(TILE_ELEMS), args,
                                           batch_smem<R>(b), st));
    TLFEA_LAUNCHED(1);
    return TLFEA_OK;
}

static int batch_dispatch_grid(tlfea_batch_s* b, int blocks_per_sm, int* grid, bool apply = false) {
    const bool f32 = b->precision == TLFEA_PRECISION_FP32;
    if (b->el->npe == 10)
        return f32 ? batch_grid<float, 10, 5>(b, blocks_per_sm, grid, apply)
                   : batch_grid<double, 10, 5>(b, blocks_per_sm, grid, apply);
    return f32 ? batch_grid<float, 4, 1>(b, blocks_per_sm, grid, apply)
               : batch_grid<double, 4, 1>(b, blocks_per_sm, grid, apply);
}

static int batch_launch(tlfea_batch_s* b, int grid, double tol, int max_iter, bool warm, cudaStream_t st) {
    const bool f32 = b->precision == TLFEA_PRECISION_FP32;
    if (b->el->npe == 10)
        return f32 ? launch_batch_cg<float, 10, 5>(b, grid, tol, max_iter, warm, st)
                   : launch_batch_cg<double, 10, 5>(b, grid, tol, max_iter, warm, st);
    return f32 ? launch_batch_cg<float, 4, 1>(b, grid, tol, max_iter, warm, st)
               : launch_batch_cg<double, 4, 1>(b, grid, tol, max_iter, warm, st);
}

// ---- per-phase launches (mode 0)

// Work items of the tile kernel (one per block): tiles, or (tile, instance group)
// pairs in shared-mesh mode.
static int bcg_items(const tlfea_batch_s* b) {
    const int T = b->el->tl.n_tiles;
    return b->shared ? T * ((b->n_inst + SHARED_GROUP - 1) / SHARED_GROUP) : T;
}

template <typename R, int NPE, int NQP>
static int bcg_prepare(const tlfea_batch_s* b) {
    const size_t smem = batch_smem<R>(b);
    if (smem > 200 * 1024) {
        set_error("batch: a tile touches too many nodes for shared memory");
        return TLFEA_UNSUPPORTED;
    }
    const void* kern = b->shared ? (const void*)k_bcg_tiles<R, NPE, NQP, true> : (const void*)k_bcg_tiles<R, NPE, NQP, false>;
    TLFEA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return TLFEA_OK;
}

template <typename R, int NPE, int NQP>
static void bcg_enqueue_tiles(const tlfea_batch_s* b, const BatchArgs<R>& A, int skip_done, int max_iter,
                              cudaStream_t st) {
    const size_t smem = batch_smem<R>(b);
    if (b->shared)
        k_bcg_tiles<R, NPE, NQP, true><<<bcg_items(b), TILE_ELEMS, smem, st>>>(A, skip_done, max_iter);
    else
        k_bcg_tiles<R, NPE, NQP, false><<<bcg_items(b), TILE_ELEMS, smem, st>>>(A, skip_done, max_iter);
}

// One CG iteration: five launches in stream order.
template <typename R, int NPE, int NQP>
static void bcg_enqueue_iteration(const tlfea_batch_s* b, const BatchArgs<R>& A, double tol, int max_iter,
                                  cudaStream_t st) {
    const int warps_grid = (b->n_chunks + TILE_ELEMS / 32 - 1) / (TILE_ELEMS / 32);  // one warp per chunk
    bcg_enqueue_tiles<R, NPE, NQP>(b, A, 1, max_iter, st);
    k_bcg_pq<R><<<warps_grid, TILE_ELEMS, 0, st>>>(A, max_iter);
    k_bcg_update<R><<<warps_grid, TILE_ELEMS, 0, st>>>(A, tol, max_iter);
    k_bcg_direction<R><<<warps_grid, TILE_ELEMS, 0, st>>>(A, max_iter);
    k_bcg_next<<<1, 1, 0, st>>>(A.it_dev, A.n_done, A.n_inst, max_iter);
}

// The graph of `iters` iterations for (precision, tol, max_iter), captured once.
template <typename R, int NPE, int NQP>
static int bcg_graph(tlfea_batch_s* b, const BatchArgs<R>& A, double tol, int max_iter, int iters, cudaStream_t st,
                     cudaGraphExec_t* out) {
    const int prec = sizeof(R) == 4 ? TLFEA_PRECISION_FP32 : TLFEA_PRECISION_FP64;
    for (auto& g : b->phase_graphs)
        if (g.precision == prec && g.tol == tol && g.max_iter == max_iter && g.iters == iters) {
            *out = g.exec;
            return TLFEA_OK;
        }
    cudaGraph_t g = nullptr;
    TLFEA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < iters; ++k) bcg_enqueue_iteration<R, NPE, NQP>(b, A, tol, max_iter, st);
    const cudaError_t e1 = cudaGetLastError();
    const cudaError_t e2 = cudaStreamEndCapture(st, &g);
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        set_error("batch_solve: capture of the iteration chunk failed");
        return TLFEA_CUDA_ERROR;
    }
    cudaGraphExec_t ge = nullptr;
    const cudaError_t e3 = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) {
        set_error(std::string("batch_solve: cudaGraphInstantiate: ") + cudaGetErrorString(e3));
        return TLFEA_CUDA_ERROR;
    }
    b->phase_graphs.push_back({prec, max_iter, iters, tol, ge});
    *out = ge;
    return TLFEA_OK;
}

// The whole solve in per-phase launches: the start (u, r, p, the initial residual),
// then chunks of iterations replayed until every instance is done or max_iter is
// reached (the host reads the two control words after each chunk), then the final
// status.  f_over / u0_over replace the batch's load and initial guess.
template <typename R, int NPE, int NQP>
static int run_phased(tlfea_batch_s* b, double tol, int max_iter, bool warm, cudaStream_t st,
                      const double* f_over = nullptr, const double* u0_over = nullptr) {
    int s = bcg_prepare<R, NPE, NQP>(b);
    if (s) return s;
    BatchArgs<R> A = batch_args<R>(b);
    if (f_over) A.f = f_over;
    if (u0_over) A.u0 = u0_over;
    const int w = warm ? 1 : 0;
    const int chunk_grid = std::min(b->n_chunks, 148 * 16);  // one block per chunk, grid-stride beyond
    TLFEA_CUDA(cudaMemsetAsync(b->n_done, 0, 2 * sizeof(int), st));
    k_bcg_start<R><<<chunk_grid, TILE_ELEMS, 0, st>>>(A, w);
    if (warm) bcg_enqueue_tiles<R, NPE, NQP>(b, A, 0, max_iter, st);
    k_bcg_start_residual<R><<<chunk_grid, TILE_ELEMS, 0, st>>>(A, w);
    k_bcg_init<R><<<std::min(b->n_inst, 65535), 32, 0, st>>>(A, tol);
    TLFEA_CUDA(cudaGetLastError());
    TLFEA_LAUNCHED(warm ? 4 : 3);
    int ctl[2] = {0, 0};
    for (int chunk = 16; max_iter > 0; chunk = 64) {
        cudaGraphExec_t ge = nullptr;
        if ((s = bcg_graph<R, NPE, NQP>(b, A, tol, max_iter, chunk, st, &ge))) return s;
        TLFEA_CUDA(cudaGraphLaunch(ge, st));
        TLFEA_LAUNCHED(5 * chunk);
        TLFEA_CUDA(cudaMemcpyAsync(ctl, b->n_done, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
        TLFEA_CUDA(cudaStreamSynchronize(st));
        if (ctl[0] >= b->n_inst || ctl[1] >= max_iter) break;
    }
    k_bcg_finish<R><<<(b->n_inst + 127) / 128, 128, 0, st>>>(A);
    TLFEA_CUDA(cudaGetLastError());
    TLFEA_LAUNCHED(1);
    return TLFEA_OK;
}

// Dispatch on precision and element type; mode 1 keeps the persistent launch.
static int bcg_run(tlfea_batch_s* b, bool f32, int grid, double tol, int max_iter, bool warm, cudaStream_t st,
                   const double* f_over = nullptr, const double* u0_over = nullptr) {
    const bool t10 = (b->el->npe == 10);
    if (b->mode == 0) {
        if (t10)
            return f32 ? run_phased<float, 10, 5>(b, tol, max_iter, warm, st, f_over, u0_over)
                       : run_phased<double, 10, 5>(b, tol, max_iter, warm, st, f_over, u0_over);
        return f32 ? run_phased<float, 4, 1>(b, tol, max_iter, warm, st, f_over, u0_over)
                   : run_phased<double, 4, 1>(b, tol, max_iter, warm, st, f_over, u0_over);
    }
    TLFEA_CUDA(cudaMemsetAsync(b->n_done, 0, sizeof(int), st));
    if (t10)
        return f32 ? launch_batch_cg<float, 10, 5>(b, grid, tol, max_iter, warm, st, f_over, u0_over)
                   : launch_batch_cg<double, 10, 5>(b, grid, tol, max_iter, warm, st, f_over, u0_over);
    return f32 ? launch_batch_cg<float, 4, 1>(b, grid, tol, max_iter, warm, st, f_over, u0_over)
               : launch_batch_cg<double, 4, 1>(b, grid, tol, max_iter, warm, st, f_over, u0_over);
}

// Node chunks of at most `chunk_nodes` nodes that never straddle instances.
static int build_chunks(tlfea_batch_s* b, int chunk_nodes) {
    std::vector<int> cinst, cbeg, ichunk((size_t)b->n_inst + 1, 0);
    for (int i = 0; i < b->n_inst; ++i) {
        ichunk[i] = (int)cinst.size();
        for (int n = b->node_off[i]; n < b->node_off[i + 1]; n += chunk_nodes) {
            cinst.push_back(i);
            cbeg.push_back(n);
        }
    }
    ichunk[b->n_inst] = (int)cinst.size();
    cbeg.push_back(b->N);
    cudaStream_t st = b->el->stream;
    TLFEA_CUDA(cudaStreamSynchronize(st));
    dfree(b->chunk_inst);
    dfree(b->chunk_beg);
    dfree(b->inst_chunk);
    dfree(b->cpa);
    dfree(b->cpb);
    b->n_chunks = (int)cinst.size();
    int s;
    if ((s = dalloc(&b->chunk_inst, cinst.size())) || (s = dalloc(&b->chunk_beg, cbeg.size())) ||
        (s = dalloc(&b->inst_chunk, ichunk.size())) || (s = dalloc(&b->cpa, cinst.size())) ||
        (s = dalloc(&b->cpb, cinst.size())))
        return s;
    TLFEA_CUDA(cudaMemcpy(b->chunk_inst, cinst.data(), cinst.size() * sizeof(int), cudaMemcpyHostToDevice));
    TLFEA_CUDA(cudaMemcpy(b->chunk_beg, cbeg.data(), cbeg.size() * sizeof(int), cudaMemcpyHostToDevice));
    TLFEA_CUDA(cudaMemcpy(b->inst_chunk, ichunk.data(), ichunk.size() * sizeof(int), cudaMemcpyHostToDevice));
    b->chunk_nodes = chunk_nodes;
    drop_graphs(b);
    return TLFEA_OK;
}

// Lame parameters as SetSVK computes them (FEAT10Data.cuh:399-409).
static void lame(double Ey, double nu, double& lam, double& mu) {
    mu = Ey / (2.0 * (1.0 + nu));
    lam = Ey * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
}

static int upload_material(tlfea_batch_s* b) {
    tlfea_element_s* el = b->el;
    const Tiling& tl = el->tl;
    if (b->shared) {  // per instance
        const size_t n = (size_t)b->n_inst;
        std::vector<double> lam(n), mu(n);
        std::vector<float> lam32(n), mu32(n);
        for (size_t i = 0; i < n; ++i) {
            lame(b->inst_E[i], b->inst_nu[i], lam[i], mu[i]);
            lam32[i] = (float)lam[i];
            mu32[i] = (float)mu[i];
        }
        cudaStream_t st = el->stream;
        TLFEA_CUDA(cudaMemcpyAsync(b->lam, lam.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
        TLFEA_CUDA(cudaMemcpyAsync(b->mu, mu.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
        TLFEA_CUDA(cudaMemcpyAsync(b->lam32, lam32.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
        TLFEA_CUDA(cudaMemcpyAsync(b->mu32, mu32.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
        TLFEA_CUDA(cudaStreamSynchronize(st));
        return TLFEA_OK;
    }
    const size_t ns = (size_t)tl.n_tiles * TILE_ELEMS;
    std::vector<int> elem_inst((size_t)b->E);
    for (int i = 0; i < b->n_inst; ++i)
        for (int e = b->elem_off[i]; e < b->elem_off[i + 1]; ++e) elem_inst[e] = i;
    std::vector<double> lam(ns, 0.0), mu(ns, 0.0);
    std::vector<float> lam32(ns, 0.f), mu32(ns, 0.f);
    for (size_t s = 0; s < ns; ++s) {
        const int e = tl.h_tile_elem[s];
        if (e < 0) continue;
        const int i = elem_inst[e];
        lame(b->inst_E[i], b->inst_nu[i], lam[s], mu[s]);
        lam32[s] = (float)lam[s];
        mu32[s] = (float)mu[s];
    }
    cudaStream_t st = el->stream;
    TLFEA_CUDA(cudaMemcpyAsync(b->lam, lam.data(), ns * sizeof(double), cudaMemcpyHostToDevice, st));
    TLFEA_CUDA(cudaMemcpyAsync(b->mu, mu.data(), ns * sizeof(double), cudaMemcpyHostToDevice, st));
    TLFEA_CUDA(cudaMemcpyAsync(b->lam32, lam32.data(), ns * sizeof(float), cudaMemcpyHostToDevice, st));
    TLFEA_CUDA(cudaMemcpyAsync(b->mu32, mu32.data(), ns * sizeof(float), cudaMemcpyHostToDevice, st));
    TLFEA_CUDA(cudaStreamSynchronize(st));
    return TLFEA_OK;
}

// Nodes touched by no element carry no stiffness: they are always held fixed.
static std::vector<unsigned char> untouched_nodes(const tlfea_batch_s* b) {
    const int per = b->shared ? b->el->N : b->N;
    std::vector<unsigned char> base((size_t)per, 1);
    for (int k : b->el->conn) base[k] = 0;
    std::vector<unsigned char> fx((size_t)b->N);
    for (size_t i = 0; i < fx.size(); ++i) fx[i] = base[i % (size_t)per];
    return fx;
}

// Solver state of a batch whose element (tiling, gradients) is set up.
static int batch_alloc_state(tlfea_batch_s* b) {
    const int n_inst = b->n_inst;
    const size_t n3 = 3 * (size_t)b->N;
    const size_t nmat = b->shared ? (size_t)n_inst : (size_t)b->el->tl.n_tiles * TILE_ELEMS;
    int st;
    if ((st = dalloc(&b->lam, nmat)) || (st = dalloc(&b->mu, nmat)) || (st = dalloc(&b->lam32, nmat)) ||
        (st = dalloc(&b->mu32, nmat)) || (st = dalloc(&b->fixed, (size_t)b->N)) || (st = dalloc(&b->u, n3)) ||
        (st = dalloc(&b->r, n3)) || (st = dalloc(&b->p, n3)) || (st = dalloc(&b->q, n3)) ||
        (st = dalloc(&b->f, n3)) || (st = dalloc(&b->u0, n3)) || (st = dalloc(&b->rr, 2 * (size_t)n_inst)) ||
        (st = dalloc(&b->fnorm, (size_t)n_inst)) || (st = dalloc(&b->rel, (size_t)n_inst)) ||
        (st = dalloc(&b->iters, (size_t)n_inst)) || (st = dalloc(&b->status, (size_t)n_inst)) ||
        (st = dalloc(&b->done, (size_t)n_inst)) || (st = dalloc(&b->n_done, 2)) ||
        (st = dalloc(&b->alpha, (size_t)n_inst)) || (st = dalloc(&b->beta, (size_t)n_inst)) ||
        (st = dalloc(&b->flag, (size_t)n_inst)) || (st = dalloc(&b->ticket, (size_t)n_inst)))
        return st;
    if (b->shared) {
        const size_t np = 3 * (size_t)n_inst * (size_t)std::max(b->el->tl.n_pslots, 1);
        if ((st = dalloc(&b->part64, np)) || (st = dalloc(&b->part32, np))) return st;
    }
    cudaStream_t s = b->el->stream;
    const std::vector<unsigned char> fx = untouched_nodes(b);
    TLFEA_CUDA(cudaMemcpyAsync(b->fixed, fx.data(), (size_t)b->N, cudaMemcpyHostToDevice, s));
    TLFEA_CUDA(cudaMemsetAsync(b->f, 0, n3 * sizeof(double), s));
    TLFEA_CUDA(cudaMemsetAsync(b->u, 0, n3 * sizeof(double), s));
    TLFEA_CUDA(cudaMemsetAsync(b->u0, 0, n3 * sizeof(double), s));
    TLFEA_CUDA(cudaMemsetAsync(b->iters, 0, n_inst * sizeof(int), s));
    TLFEA_CUDA(cudaMemsetAsync(b->status, 0, n_inst * sizeof(int), s));
    TLFEA_CUDA(cudaMemsetAsync(b->rel, 0, n_inst * sizeof(double), s));
    TLFEA_CUDA(cudaStreamSynchronize(s));
    return build_chunks(b, 256);
}

}  // namespace tlfea

using namespace tlfea;

#define CHECK_BATCH(b)                \
    do {                              \
        if (!(b)) {                   \
            set_error("null batch");  \
            return TLFEA_INVALID_ARG; \
        }                             \
    } while (0)

extern "C" {

int tlfea_batch_create(int type, int n_inst, const int* node_off, const int* elem_off, const double* qx,
                       const double* qy, const double* qz, const double* qw, int n_qp, const double* x,
                       const double* y, const double* z, const int* conn, tlfea_batch* out) {
    if (!out) return TLFEA_INVALID_ARG;
    *out = nullptr;
    if ((type != TLFEA_TYPE_T10 && type != TLFEA_TYPE_T4) || n_inst <= 0 || !node_off || !elem_off || !x || !y ||
        !z || !conn || !qx || !qy || !qz || !qw) {
        set_error("batch_create: bad arguments");
        return TLFEA_INVALID_ARG;
    }
    const int npe = (type == TLFEA_TYPE_T10) ? T10_NPE : T4_NPE;
    const int nqp = (type == TLFEA_TYPE_T10) ? T10_NQP : T4_NQP;
    if (node_off[0] != 0 || elem_off[0] != 0) {
        set_error("batch_create: offsets must start at 0");
        return TLFEA_INVALID_ARG;
    }
    for (int i = 0; i < n_inst; ++i)
        if (node_off[i + 1] <= node_off[i] || elem_off[i + 1] <= elem_off[i]) {
            set_error("batch_create: every instance needs nodes and elements");
            return TLFEA_INVALID_ARG;
        }
    const long long Nl = node_off[n_inst], El = elem_off[n_inst];
    if (3 * Nl >= (1LL << 31) || El * npe >= (1LL << 31)) {
        set_error("batch_create: batch too large for 32-bit indices");
        return TLFEA_INVALID_ARG;
    }
    const int N = (int)Nl, E = (int)El;
    // combined column-major connectivity with global node ids
    std::vector<int> gconn((size_t)E * npe);
    std::vector<int> group((size_t)E);
    for (int i = 0; i < n_inst; ++i) {
        const int nb = node_off[i], nn = node_off[i + 1] - nb;
        for (int e = elem_off[i]; e < elem_off[i + 1]; ++e) {
            group[e] = i;
            for (int a = 0; a < npe; ++a) {
                const int l = conn[(size_t)e * npe + a];
                if (l < 0 || l >= nn) {
                    set_error("batch_create: connectivity index out of range of its instance");
                    return TLFEA_INVALID_ARG;
                }
                gconn[e + (size_t)a * E] = nb + l;
            }
        }
    }
    tlfea_element el = nullptr;
    int st = tlfea_element_create(type, E, N, &el);
    if (st) return st;
    tlfea_batch_s* b = new tlfea_batch_s();
    b->type = type;
    b->n_inst = n_inst;
    b->N = N;
    b->E = E;
    b->el = el;
    b->node_off.assign(node_off, node_off + n_inst + 1);
    b->elem_off.assign(elem_off, elem_off + n_inst + 1);
    b->inst_E.assign(n_inst, 0.0);
    b->inst_nu.assign(n_inst, 0.0);
    el->elem_group = std::move(group);
    auto fail = [&](int s) {
        tlfea_batch_destroy(b);
        return s;
    };
    if (n_qp != nqp) {
        set_error("batch_create: quadrature size does not match the element type");
        return fail(TLFEA_SIZE_MISMATCH);
    }
    if ((st = tlfea_element_setup(el, qx, qy, qz, qw, n_qp, x, y, z, gconn.data()))) return fail(st);
    if ((st = tlfea_element_calc_dndu_pre(el))) return fail(st);
    {
        std::vector<int> elem_inst((size_t)E), ti(2 * (size_t)el->tl.n_tiles);
        for (int i = 0; i < n_inst; ++i)
            for (int e = elem_off[i]; e < elem_off[i + 1]; ++e) elem_inst[e] = i;
        for (int t = 0; t < el->tl.n_tiles; ++t) {
            int lo = n_inst, hi = -1;
            for (int k = 0; k < TILE_ELEMS; ++k) {
                const int e = el->tl.h_tile_elem[(size_t)t * TILE_ELEMS + k];
                if (e < 0) continue;
                lo = std::min(lo, elem_inst[e]);
                hi = std::max(hi, elem_inst[e]);
            }
            ti[2 * t] = lo;
            ti[2 * t + 1] = hi;
        }
        if ((st = dalloc(&b->tile_inst, ti.size()))) return fail(st);
        if (cudaMemcpy(b->tile_inst, ti.data(), ti.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
            set_error("batch_create: upload failed");
            return fail(TLFEA_CUDA_ERROR);
        }
    }
    if ((st = batch_alloc_state(b))) return fail(st);
    *out = b;
    return TLFEA_OK;
}

int tlfea_batch_create_shared(int type, int n_inst, int n_nodes, int n_elem, const double* qx, const double* qy,
                              const double* qz, const double* qw, int n_qp, const double* x, const double* y,
                              const double* z, const int* conn, tlfea_batch* out) {
    if (!out) return TLFEA_INVALID_ARG;
    *out = nullptr;
    if ((type != TLFEA_TYPE_T10 && type != TLFEA_TYPE_T4) || n_inst <= 0 || n_nodes <= 0 || n_elem <= 0 || !x ||
        !y || !z || !conn || !qx || !qy || !qz || !qw) {
        set_error("batch_create_shared: bad arguments");
        return TLFEA_INVALID_ARG;
    }
    const int npe = (type == TLFEA_TYPE_T10) ? T10_NPE : T4_NPE;
    const int nqp = (type == TLFEA_TYPE_T10) ? T10_NQP : T4_NQP;
    if (3LL * n_nodes * n_inst >= (1LL << 31) || (long long)n_elem * n_inst >= (1LL << 31)) {
        set_error("batch_create_shared: batch too large for 32-bit indices");
        return TLFEA_INVALID_ARG;
    }
    std::vector<int> cm((size_t)n_elem * npe);
    for (int e = 0; e < n_elem; ++e)
        for (int a = 0; a < npe; ++a) {
            const int l = conn[(size_t)e * npe + a];
            if (l < 0 || l >= n_nodes) {
                set_error("batch_create_shared: connectivity index out of range");
                return TLFEA_INVALID_ARG;
            }
            cm[e + (size_t)a * n_elem] = l;
        }
    tlfea_element el = nullptr;
    int st = tlfea_element_create(type, n_elem, n_nodes, &el);
    if (st) return st;
    tlfea_batch_s* b = new tlfea_batch_s();
    b->type = type;
    b->n_inst = n_inst;
    b->shared = true;
    b->N = n_nodes * n_inst;
    b->E = n_elem * n_inst;
    b->el = el;
    b->node_off.resize((size_t)n_inst + 1);
    b->elem_off.resize((size_t)n_inst + 1);
    for (int i = 0; i <= n_inst; ++i) {
        b->node_off[i] = i * n_nodes;
        b->elem_off[i] = i * n_elem;
    }
    b->inst_E.assign(n_inst, 0.0);
    b->inst_nu.assign(n_inst, 0.0);
    auto fail = [&](int s) {
        tlfea_batch_destroy(b);
        return s;
    };
    if (n_qp != nqp) {
        set_error("batch_create_shared: quadrature size does not match the element type");
        return fail(TLFEA_SIZE_MISMATCH);
    }
    if ((st = tlfea_element_setup(el, qx, qy, qz, qw, n_qp, x, y, z, cm.data()))) return fail(st);
    if ((st = tlfea_element_calc_dndu_pre(el))) return fail(st);
    if ((st = batch_alloc_state(b))) return fail(st);
    *out = b;
    return TLFEA_OK;
}

int tlfea_batch_destroy(tlfea_batch b) {
    CHECK_BATCH(b);
    if (b->el) TLFEA_CUDA(cudaSetDevice(b->el->device));
    drop_graphs(b);
    dfree(b->lam); dfree(b->mu); dfree(b->lam32); dfree(b->mu32);
    dfree(b->fixed); dfree(b->chunk_inst); dfree(b->chunk_beg); dfree(b->inst_chunk); dfree(b->tile_inst);
    dfree(b->u); dfree(b->r); dfree(b->p); dfree(b->q); dfree(b->f); dfree(b->u0);
    dfree(b->rhs); dfree(b->uacc);
    dfree(b->cpa); dfree(b->cpb); dfree(b->rr); dfree(b->fnorm); dfree(b->rel);
    dfree(b->alpha); dfree(b->beta); dfree(b->flag); dfree(b->ticket);
    dfree(b->part64); dfree(b->part32);
    dfree(b->iters); dfree(b->status); dfree(b->done); dfree(b->n_done);
    if (b->el) tlfea_element_destroy(b->el);
    delete b;
    return TLFEA_OK;
}

int tlfea_batch_get_counts(tlfea_batch b, int* n_inst, int* n_elem, int* n_nodes, int* n_tiles) {
    CHECK_BATCH(b);
    if (n_inst) *n_inst = b->n_inst;
    if (n_elem) *n_elem = b->E;
    if (n_nodes) *n_nodes = b->N;
    if (n_tiles) *n_tiles = b->shared ? b->el->tl.n_tiles * b->n_inst : b->el->tl.n_tiles;
    return TLFEA_OK;
}

int tlfea_batch_get_stream(tlfea_batch b, void** stream) {
    CHECK_BATCH(b);
    if (!stream) return TLFEA_INVALID_ARG;
    *stream = (void*)b->el->stream;
    return TLFEA_OK;
}

int tlfea_batch_set_material(tlfea_batch b, const double* E, const double* nu) {
    CHECK_BATCH(b);
    if (!E || !nu) return TLFEA_INVALID_ARG;
    for (int i = 0; i < b->n_inst; ++i) {
        if (!(E[i] > 0.0) || !(nu[i] > -1.0 && nu[i] < 0.5)) {
            set_error("batch_set_material: need E > 0 and -1 < nu < 0.5");
            return TLFEA_INVALID_ARG;
        }
        b->inst_E[i] = E[i];
        b->inst_nu[i] = nu[i];
    }
    const int st = upload_material(b);
    if (st) return st;
    b->material_set = true;
    return TLFEA_OK;
}

int tlfea_batch_set_fixed(tlfea_batch b, const int* nodes, int n) {
    CHECK_BATCH(b);
    if (n < 0 || (n > 0 && !nodes)) return TLFEA_INVALID_ARG;
    std::vector<unsigned char> fx = untouched_nodes(b);
    for (int k = 0; k < n; ++k) {
        if (nodes[k] < 0 || nodes[k] >= b->N) {
            set_error("batch_set_fixed: node index out of range");
            return TLFEA_INVALID_ARG;
        }
        fx[nodes[k]] = 1;
    }
    TLFEA_CUDA(cudaMemcpyAsync(b->fixed, fx.data(), (size_t)b->N, cudaMemcpyHostToDevice, b->el->stream));
    TLFEA_CUDA(cudaStreamSynchronize(b->el->stream));
    return TLFEA_OK;
}

int tlfea_batch_set_external_force(tlfea_batch b, const double* f, long long n, int on_device) {
    CHECK_BATCH(b);
    if (!f || n != 3LL * b->N) {
        set_error("batch_set_external_force: need 3 * n_nodes values");
        return TLFEA_SIZE_MISMATCH;
    }
    TLFEA_CUDA(cudaMemcpyAsync(b->f, f, (size_t)n * sizeof(double),
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, b->el->stream));
    TLFEA_CUDA(cudaStreamSynchronize(b->el->stream));
    return TLFEA_OK;
}

int tlfea_batch_set_initial_guess(tlfea_batch b, const double* u0, long long n, int on_device) {
    CHECK_BATCH(b);
    if (!u0) {
        b->warm = false;
        return TLFEA_OK;
    }
    if (n != 3LL * b->N) {
        set_error("batch_set_initial_guess: need 3 * n_nodes values");
        return TLFEA_SIZE_MISMATCH;
    }
    TLFEA_CUDA(cudaMemcpyAsync(b->u0, u0, (size_t)n * sizeof(double),
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, b->el->stream));
    TLFEA_CUDA(cudaStreamSynchronize(b->el->stream));
    b->warm = true;
    return TLFEA_OK;
}

int tlfea_batch_set_precision(tlfea_batch b, int precision) {
    CHECK_BATCH(b);
    if (precision != TLFEA_PRECISION_FP64 && precision != TLFEA_PRECISION_FP32) return TLFEA_INVALID_ARG;
    if (precision != b->precision) drop_graphs(b);
    b->precision = precision;
    return TLFEA_OK;
}

int tlfea_batch_set_launch(tlfea_batch b, int blocks_per_sm, int chunk_nodes) {
    CHECK_BATCH(b);
    if (blocks_per_sm < 0 || (chunk_nodes != 0 && (chunk_nodes < 32 || chunk_nodes > 4096))) return TLFEA_INVALID_ARG;
    if (chunk_nodes != 0 && chunk_nodes != b->chunk_nodes) {
        const int st = build_chunks(b, chunk_nodes);
        if (st) return st;
    }
    if (blocks_per_sm != b->blocks_per_sm) drop_graphs(b);
    b->blocks_per_sm = blocks_per_sm;
    return TLFEA_OK;
}

int tlfea_batch_set_mode(tlfea_batch b, int mode) {
    CHECK_BATCH(b);
    if (mode != 0 && mode != 1) return TLFEA_INVALID_ARG;
    if (mode != b->mode) drop_graphs(b);
    b->mode = mode;
    return TLFEA_OK;
}

int tlfea_batch_get_launch(tlfea_batch b, int* blocks_per_sm, int* chunk_nodes, int* grid) {
    CHECK_BATCH(b);
    if (blocks_per_sm) *blocks_per_sm = b->blocks_per_sm;
    if (chunk_nodes) *chunk_nodes = b->chunk_nodes;
    if (grid) {
        int g = 0;
        const int st = batch_dispatch_grid(b, b->blocks_per_sm, &g);
        if (st) return st;
        *grid = g;
    }
    return TLFEA_OK;
}

// Right-hand side of a correction pass: the FP64 residual of every instance
// not yet converged, zero for the converged ones (their correction is zero).
__global__ void k_batch_rhs(int n_chunks, const int* __restrict__ chunk_beg, const int* __restrict__ chunk_inst,
                            const int* __restrict__ done, const double* __restrict__ r, double* rhs) {
    for (int c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const bool dn = done[chunk_inst[c]] != 0;
        for (int i = 3 * chunk_beg[c] + threadIdx.x; i < 3 * chunk_beg[c + 1]; i += blockDim.x) rhs[i] = dn ? 0.0 : r[i];
    }
}

__global__ void k_batch_accumulate(long long n, const double* __restrict__ d, double* u) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        u[i] += d[i];
}

// One persistent launch of the whole CG (element work in b->precision),
// captured once per (grid, tol, max_iter, precision, warm) and replayed.
static int run_captured(tlfea_batch_s* b, int grid, double tol, int max_iter, bool warm) {
    cudaStream_t st = b->el->stream;
    if (b->graph_tol != tol || b->graph_max_iter != max_iter || b->graph_grid != grid ||
        b->graph_precision != b->precision) {
        drop_graphs(b);
        b->graph_tol = tol;
        b->graph_max_iter = max_iter;
        b->graph_grid = grid;
        b->graph_precision = b->precision;
    }
    cudaGraphExec_t& ge = warm ? b->graph_w : b->graph;
    if (!ge) {
        cudaGraph_t g = nullptr;
        TLFEA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        cudaError_t e1 = cudaMemsetAsync(b->n_done, 0, sizeof(int), st);
        const int rc = (e1 == cudaSuccess) ? batch_launch(b, grid, tol, max_iter, warm, st) : TLFEA_CUDA_ERROR;
        cudaError_t e2 = cudaStreamEndCapture(st, &g);
        if (rc != TLFEA_OK || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            set_error("batch_solve: capture of the persistent launch failed");
            return TLFEA_CUDA_ERROR;
        }
        cudaError_t e3 = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) {
            ge = nullptr;
            set_error(std::string("batch_solve: cudaGraphInstantiate: ") + cudaGetErrorString(e3));
            return TLFEA_CUDA_ERROR;
        }
    }
    TLFEA_CUDA(cudaGraphLaunch(ge, st));
    return TLFEA_OK;
}

int tlfea_batch_solve(tlfea_batch b, double tol, int max_iter) {
    CHECK_BATCH(b);
    if (!b->material_set) {
        set_error("batch_solve: set the material first");
        return TLFEA_NOT_SETUP;
    }
    if (!(tol > 0.0) || max_iter < 0) return TLFEA_INVALID_ARG;
    cudaStream_t st = b->el->stream;
    int grid = 0, s = 0;
    if (b->mode == 1 && (s = batch_dispatch_grid(b, b->blocks_per_sm, &grid))) return s;
    b->refined = false;
    if (b->precision != TLFEA_PRECISION_FP32) {
        if ((s = (b->mode == 1) ? run_captured(b, grid, tol, max_iter, b->warm)
                                : bcg_run(b, false, 0, tol, max_iter, b->warm, st)))
            return s;
        TLFEA_CUDA(cudaStreamSynchronize(st));
        return TLFEA_OK;
    }
    // FP32 element work, FP64 verdict: iterative refinement on the correction
    // equation.  Each pass evaluates the true residual r = f - K u with the FP64
    // operator (the prologue of the FP64 kernel at u, no iterations), solves
    // K d = r with the FP32-element CG to a relative tolerance tau, and adds d
    // to u.  The FP32 rounding then acts on the correction, not on u, so every
    // pass gains a factor of about max(tau, FP32 operator error) on the FP64
    // residual.  The reported residual and stop test are the FP64 ones.
    const size_t n = (size_t)b->n_inst, n3 = 3 * (size_t)b->N;
    if (!b->rhs && (dalloc(&b->rhs, n3) || dalloc(&b->uacc, n3))) return TLFEA_CUDA_ERROR;
    std::vector<int> it(n);
    b->iters_total.assign(n, 0);
    int grid64 = 0;
    if (b->mode == 1) {
        s = (b->el->npe == 10) ? batch_grid<double, 10, 5>(b, 0, &grid64) : batch_grid<double, 4, 1>(b, 0, &grid64);
        if (s) return s;
    }
    auto eval64 = [&](bool at_u, const double* u_at) -> int {  // FP64 residual at u_at (or at 0)
        return bcg_run(b, false, grid64, tol, 0, at_u, st, nullptr, u_at);
    };
    const double tau = std::max(tol, std::min(0.1, std::max(1e-4, 0.5 * std::sqrt(tol))));
    constexpr int MAX_PASSES = 8;
    if ((s = eval64(b->warm, b->u0))) return s;
    for (int pass = 0;; ++pass) {
        int nd = 0;
        TLFEA_CUDA(cudaMemcpyAsync(&nd, b->n_done, sizeof(int), cudaMemcpyDeviceToHost, st));
        TLFEA_CUDA(cudaStreamSynchronize(st));
        if (nd >= b->n_inst || pass == MAX_PASSES) break;
        // u (the FP64 kernel's copy of the evaluation point) is the accumulated solution
        TLFEA_CUDA(cudaMemcpyAsync(b->uacc, b->u, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
        k_batch_rhs<<<std::min(b->n_chunks, 4096), 256, 0, st>>>(b->n_chunks, b->chunk_beg, b->chunk_inst, b->done,
                                                                 b->r, b->rhs);
        TLFEA_CUDA(cudaGetLastError());
        TLFEA_LAUNCHED(1);
        if ((s = bcg_run(b, true, grid, tau, max_iter, false, st, b->rhs, nullptr))) return s;
        TLFEA_CUDA(cudaMemcpyAsync(it.data(), b->iters, n * sizeof(int), cudaMemcpyDeviceToHost, st));
        TLFEA_CUDA(cudaStreamSynchronize(st));
        for (size_t i = 0; i < n; ++i) b->iters_total[i] += it[i];
        k_batch_accumulate<<<1184, 256, 0, st>>>((long long)n3, b->u, b->uacc);
        TLFEA_CUDA(cudaGetLastError());
        TLFEA_LAUNCHED(1);
        if ((s = eval64(true, b->uacc))) return s;
    }
    TLFEA_CUDA(cudaStreamSynchronize(st));
    b->refined = true;
    return TLFEA_OK;
}

int tlfea_batch_get_results(tlfea_batch b, int* iters, double* rel, int* status) {
    CHECK_BATCH(b);
    cudaStream_t st = b->el->stream;
    const size_t n = (size_t)b->n_inst;
    if (iters) {
        if (b->refined)
            std::memcpy(iters, b->iters_total.data(), n * sizeof(int));
        else
            TLFEA_CUDA(cudaMemcpyAsync(iters, b->iters, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    if (rel) TLFEA_CUDA(cudaMemcpyAsync(rel, b->rel, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (status) TLFEA_CUDA(cudaMemcpyAsync(status, b->status, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    TLFEA_CUDA(cudaStreamSynchronize(st));
    return TLFEA_OK;
}

int tlfea_batch_retrieve_displacement(tlfea_batch b, double* u, long long n) {
    CHECK_BATCH(b);
    if (!u || n != 3LL * b->N) {
        set_error("batch_retrieve_displacement: need 3 * n_nodes values");
        return TLFEA_SIZE_MISMATCH;
    }
    TLFEA_CUDA(cudaMemcpyAsync(u, b->u, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, b->el->stream));
    TLFEA_CUDA(cudaStreamSynchronize(b->el->stream));
    return TLFEA_OK;
}

int tlfea_batch_device_ptrs(tlfea_batch b, double** u, double** f, double** u0) {
    CHECK_BATCH(b);
    if (u) *u = b->u;
    if (f) *f = b->f;
    if (u0) *u0 = b->u0;
    return TLFEA_OK;
}

int tlfea_batch_apply(tlfea_batch b, const double* d_x, double* d_y) {
    CHECK_BATCH(b);
    if (!b->material_set) {
        set_error("batch_apply: set the material first");
        return TLFEA_NOT_SETUP;
    }
    if (!d_x || !d_y) return TLFEA_INVALID_ARG;
    int grid = 0;
    int s = batch_dispatch_grid(b, 0, &grid, true);
    if (s) return s;
    cudaStream_t st = b->el->stream;
    const bool f32 = b->precision == TLFEA_PRECISION_FP32;
    const bool t10 = b->el->npe == 10;
    auto go = [&](auto tag, const void* fn, size_t smem) -> int {
        using R = typename decltype(tag)::type;
        BatchArgs<R> A = batch_args<R>(b);
        void* args[] = {&A, (void*)&d_x, (void*)&d_y};
        TLFEA_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(TILE_ELEMS), args, smem, st));
        TLFEA_LAUNCHED(1);
        return TLFEA_OK;
    };
    struct TD { using type = double; };
    struct TF { using type = float; };
    if (f32)
        s = t10 ? go(TF{}, batch_kernel<float, 10, 5>(b, true), batch_smem<float>(b))
                : go(TF{}, batch_kernel<float, 4, 1>(b, true), batch_smem<float>(b));
    else
        s = t10 ? go(TD{}, batch_kernel<double, 10, 5>(b, true), batch_smem<double>(b))
                : go(TD{}, batch_kernel<double, 4, 1>(b, true), batch_smem<double>(b));
    if (s) return s;
    TLFEA_CUDA(cudaStreamSynchronize(st));
    return TLFEA_OK;
}

// Autotuner: times `trial_iters` CG iterations of this batch for every
// (blocks per SM, node-chunk size) candidate and keeps the fastest.  The
// trials overwrite the solution vectors; solve afterwards.
int tlfea_batch_autotune(tlfea_batch b, int trial_iters, int* best_blocks_per_sm, int* best_chunk, float* best_ms) {
    CHECK_BATCH(b);
    if (!b->material_set) {
        set_error("batch_autotune: set the material first");
        return TLFEA_NOT_SETUP;
    }
    if (trial_iters <= 0) trial_iters = 8;
    cudaStream_t st = b->el->stream;
    const int chunks[] = {128, 256, 512, 1024};
    int s = 0;
    if (b->mode == 0) {
        // per-phase launches: every kernel takes the occupancy its registers allow, so
        // the chunk size is the one knob; time trial_iters iterations of each
        const bool f32 = b->precision == TLFEA_PRECISION_FP32;
        float best = 1e30f;
        int bc = b->chunk_nodes;
        for (int c : chunks) {
            if ((s = build_chunks(b, c))) return s;
            float ms = 0.f;
            for (int rep = 0; rep < 2 && !s; ++rep) {  // first run warms up (and captures)
                const auto t0 = std::chrono::steady_clock::now();
                s = bcg_run(b, f32, 0, 1e-300, trial_iters, false, st);
                if (!s && cudaStreamSynchronize(st) != cudaSuccess) s = TLFEA_CUDA_ERROR;
                ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
            }
            if (s) return s;
            if (ms < best) {
                best = ms;
                bc = c;
            }
        }
        if ((s = build_chunks(b, bc))) return s;
        if (best_blocks_per_sm) *best_blocks_per_sm = 0;
        if (best_chunk) *best_chunk = bc;
        if (best_ms) *best_ms = best;
        return TLFEA_OK;
    }
    int max_grid = 0;
    s = batch_dispatch_grid(b, 0, &max_grid);
    if (s) return s;
    int sms = 0;
    TLFEA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->el->device));
    const int max_per_sm = std::max(1, max_grid / std::max(sms, 1));
    cudaEvent_t e0, e1;
    TLFEA_CUDA(cudaEventCreate(&e0));
    TLFEA_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int bb = max_per_sm, bc = b->chunk_nodes;
    for (int c : chunks) {
        if ((s = build_chunks(b, c))) break;
        for (int per_sm = 1; per_sm <= max_per_sm; ++per_sm) {
            const int grid = per_sm * sms;
            float ms = 0.f;
            for (int rep = 0; rep < 2 && !s; ++rep) {  // first run warms up
                if (cudaMemsetAsync(b->n_done, 0, sizeof(int), st) != cudaSuccess) s = TLFEA_CUDA_ERROR;
                cudaEventRecord(e0, st);
                if (!s) s = batch_launch(b, grid, 1e-300, trial_iters, false, st);
                cudaEventRecord(e1, st);
                if (cudaEventSynchronize(e1) != cudaSuccess) s = TLFEA_CUDA_ERROR;
                cudaEventElapsedTime(&ms, e0, e1);
            }
            if (s) break;
            if (ms < best) {
                best = ms;
                bb = per_sm;
                bc = c;
            }
        }
        if (s) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s) return s;
    if ((s = build_chunks(b, bc))) return s;
    drop_graphs(b);
    b->blocks_per_sm = bb;
    if (best_blocks_per_sm) *best_blocks_per_sm = bb;
    if (best_chunk) *best_chunk = bc;
    if (best_ms) *best_ms = best;
    return TLFEA_OK;
}

}  // extern "C"
