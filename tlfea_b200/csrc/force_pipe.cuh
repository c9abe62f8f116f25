// force_pipe.cuh -- TMA-fed fused internal-force kernel (sm_100a).
//
// Persistent CTAs, each a producer warp plus TILE_ELEMS consumer threads (one
// element each).  The producer streams, per (tile, QP), the gradient slice
// [NPE*3][TE] and the dV slice [TE] -- plus, with QP 0, the tile's local
// connectivity [NPE][TE] -- from HBM into a shared-memory ring with 1-D bulk
// copies (cp.async.bulk ... mbarrier::complete_tx, no multicast), so several
// slices are always in flight while the consumers compute.  The consumers
// prefetch the next tile's node positions with per-thread cp.async into a
// second buffer, evaluate F, the SVK stress and the element forces QP by QP from
// the ring, and reduce per node in the fixed incidence order (interior nodes
// written directly, shared nodes as per-tile partials for k_combine).
//
// Every wait is bounded: a wait that runs out sets *err and the kernel carries
// on without the data (no hang); the host turns a set *err into an error status.
#pragma once

#include "element.cuh"

namespace tlfea {

constexpr int PIPE_THREADS = TILE_ELEMS + 32;  // consumers + one producer warp
constexpr long long PIPE_WAIT_LIMIT = 1LL << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Bounded wait for the phase with the given parity; false if the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < PIPE_WAIT_LIMIT; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// 1-D bulk copy global -> shared, completion counted on `bar` (16-byte aligned
// addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(TILE_ELEMS) : "memory"); }

// Ring geometry shared by host and device.  A QP slice is streamed in PARTS
// parts (FP64: two halves, nodes 0..NPE/2-1 and the rest) so that the ring,
// the double-buffered positions and the element forces of two CTAs fit one SM.
template <typename R, int NPE>
struct PipeGeom {
    static constexpr int PARTS = sizeof(R) == 8 ? 2 : 1;
    static constexpr int PART_NODES = NPE / PARTS;
    static constexpr uint32_t GRAD_BYTES = PART_NODES * 3 * TILE_ELEMS * sizeof(R);  // one part
    static constexpr uint32_t DV_BYTES = TILE_ELEMS * sizeof(R);
    static constexpr uint32_t LCONN_BYTES = NPE * TILE_ELEMS * sizeof(uint16_t);
    static constexpr uint32_t STAGE_BYTES = GRAD_BYTES + DV_BYTES + LCONN_BYTES;
    static constexpr int STAGES = sizeof(R) == 4 ? 4 : 3;
    static_assert(NPE % PARTS == 0, "parts split the nodes evenly");
    static_assert(GRAD_BYTES % 16 == 0 && DV_BYTES % 16 == 0 && LCONN_BYTES % 16 == 0, "bulk copy alignment");
};

template <typename R, int NPE>
inline size_t pipe_smem_bytes(int max_local, bool damp) {
    using G = PipeGeom<R, NPE>;
    size_t b = (size_t)G::STAGES * G::STAGE_BYTES;        // ring
    b += 2 * 3 * (size_t)max_local * sizeof(double);      // positions (FP64), double-buffered
    if (damp) b += 2 * 3 * (size_t)max_local * sizeof(double);  // velocities, double-buffered
    b += (size_t)3 * NPE * TILE_ELEMS * sizeof(R);        // element forces
    b = (b + 15) & ~size_t(15);
    b += 2 * G::STAGES * sizeof(unsigned long long);      // full / empty barriers
    return b;
}

// Stage tile `tile`'s node values (and velocities) in FP64: FP64 mode the positions
// by cp.async copies; FP32 mode the displacements (stage_pos), plain loads.
template <typename R, bool DAMP>
__device__ __forceinline__ void prefetch_nodes(const TileArgs<R>& A, int tile, double* xs, double* ys, double* zs,
                                               double* vs) {
    const int lb = A.node_off[tile], nl = A.node_off[tile + 1] - lb;
    for (int ln = threadIdx.x; ln < nl; ln += TILE_ELEMS) {
        const int gid = A.ln_gid[lb + ln];
        if constexpr (sizeof(R) == 8) {
            cp_async<8>(xs + ln, A.px + gid);
            cp_async<8>(ys + ln, A.py + gid);
            cp_async<8>(zs + ln, A.pz + gid);
        } else {
            stage_pos(A, gid, xs[ln], ys[ln], zs[ln]);
        }
        if (DAMP) {
            cp_async<8>(vs + 3 * ln + 0, A.v + 3 * gid + 0);
            cp_async<8>(vs + 3 * ln + 1, A.v + 3 * gid + 1);
            cp_async<8>(vs + 3 * ln + 2, A.v + 3 * gid + 2);
        }
    }
}

template <typename R, int NPE, int NQP, bool DAMP>
__global__ void __launch_bounds__(PIPE_THREADS, 2) k_force_pipe(TileArgs<R> A, int n_tiles, int* err) {
    using G = PipeGeom<R, NPE>;
    constexpr int TE = TILE_ELEMS;
    constexpr int S = G::STAGES;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* ring = smem;
    double* pos = reinterpret_cast<double*>(smem + (size_t)S * G::STAGE_BYTES);
    const int ML = A.max_local;
    double* vel = pos + 6 * ML;
    R* fe = reinterpret_cast<R*>(DAMP ? reinterpret_cast<unsigned char*>(vel + 6 * ML)
                                      : reinterpret_cast<unsigned char*>(vel));
    size_t bar_off = (size_t)S * G::STAGE_BYTES + 2 * 3 * (size_t)ML * sizeof(double) +
                     (DAMP ? 2 * 3 * (size_t)ML * sizeof(double) : 0) + (size_t)3 * NPE * TE * sizeof(R);
    bar_off = (bar_off + 15) & ~size_t(15);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + bar_off);
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + S);

    const int t = threadIdx.x;
    if (t == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, TE);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();

    if (t >= TE) {
        // ------------------------------------------------------------ producer
        if (t == TE) {
            int it = 0;
            for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
                for (int q = 0; q < NQP; ++q) {
                    for (int p = 0; p < G::PARTS; ++p, ++it) {
                        const int s = it % S;
                        const uint32_t full = full0 + 8 * s, empty = empty0 + 8 * s;
                        if (it >= S && !mbar_wait(empty, ((it / S) & 1) ^ 1)) atomicExch(err, 1);
                        const bool last = (p == G::PARTS - 1), first = (q == 0 && p == 0);
                        const uint32_t bytes = G::GRAD_BYTES + (last ? G::DV_BYTES : 0) + (first ? G::LCONN_BYTES : 0);
                        mbar_expect_tx(full, bytes);
                        const uint32_t dst = smem_u32(ring + (size_t)s * G::STAGE_BYTES);
                        bulk_g2s(dst,
                                 A.grad + (((size_t)tile * NQP + q) * (NPE * 3) + (size_t)p * G::PART_NODES * 3) * TE,
                                 G::GRAD_BYTES, full);
                        if (last)
                            bulk_g2s(dst + G::GRAD_BYTES, A.dv + ((size_t)tile * NQP + q) * TE, G::DV_BYTES, full);
                        if (first)
                            bulk_g2s(dst + G::GRAD_BYTES + G::DV_BYTES, A.lconn + (size_t)tile * NPE * TE,
                                     G::LCONN_BYTES, full);
                    }
                }
            }
        }
        return;
    }

    // ---------------------------------------------------------------- consumers
    int it = 0, buf = 0;
    if (blockIdx.x < n_tiles) prefetch_nodes<R, DAMP>(A, blockIdx.x, pos, pos + ML, pos + 2 * ML, vel);
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, buf ^= 1) {
        cp_async_wait_all();
        consumer_sync();  // positions of this tile visible; previous tile's reduction done
        const int next = tile + gridDim.x;
        if (next < n_tiles) {
            double* nx = pos + (buf ^ 1) * 3 * ML;
            prefetch_nodes<R, DAMP>(A, next, nx, nx + ML, nx + 2 * ML, vel + (DAMP ? (buf ^ 1) * 3 * ML : 0));
        }
        const double* xs = pos + buf * 3 * ML;
        const double* ys = xs + ML;
        const double* zs = ys + ML;
        const double* vs = vel + (DAMP ? buf * 3 * ML : 0);

        int lc[NPE];
        R f[NPE][3];
        R ua[NPE][3], va[NPE][3];  // FP32: the element's node values, read once per tile
#pragma unroll
        for (int a = 0; a < NPE; ++a) f[a][0] = f[a][1] = f[a][2] = R(0);
#pragma unroll 1
        for (int q = 0; q < NQP; ++q) {
            R g[NPE][3];
            R dv = R(0);
#pragma unroll
            for (int p = 0; p < G::PARTS; ++p, ++it) {
                const int s = it % S;
                if (!mbar_wait(full0 + 8 * s, (it / S) & 1)) atomicExch(err, 2);
                const unsigned char* st = ring + (size_t)s * G::STAGE_BYTES;
                const R* gs = reinterpret_cast<const R*>(st);
                if (q == 0 && p == 0) {
                    const uint16_t* lcs = reinterpret_cast<const uint16_t*>(st + G::GRAD_BYTES + G::DV_BYTES);
#pragma unroll
                    for (int a = 0; a < NPE; ++a) lc[a] = lcs[a * TE + t];
                }
#pragma unroll
                for (int a = 0; a < G::PART_NODES; ++a)
#pragma unroll
                    for (int j = 0; j < 3; ++j) g[p * G::PART_NODES + a][j] = gs[grad_slot<R>(a, j, t)];
                if (p == G::PARTS - 1) dv = reinterpret_cast<const R*>(st + G::GRAD_BYTES)[t];
                // The producer refills this stage with a bulk copy (async proxy) once
                // every consumer has arrived; order this thread's generic-proxy
                // reads of the stage before that write (without the fence the refill
                // was observed to overtake the reads).
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_arrive(empty0 + 8 * s);  // slice data is in registers now
            }

            R P[3][3];
            if constexpr (sizeof(R) == 8) {
                double F[3][3];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) F[i][j] = 0.0;
#pragma unroll
                for (int a = 0; a < NPE; ++a) {
                    const double xa[3] = {xs[lc[a]], ys[lc[a]], zs[lc[a]]};
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) F[i][j] += xa[i] * g[a][j];
                }
                svk_p_reference(F, A.lambda, A.mu, P);
                if (DAMP) {
                    double Fd[3][3], Pv[3][3];
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) Fd[i][j] = 0.0;
#pragma unroll
                    for (int a = 0; a < NPE; ++a)
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int j = 0; j < 3; ++j) Fd[i][j] += vs[3 * lc[a] + i] * g[a][j];
                    kelvin_voigt<double>(F, Fd, A.eta, A.lamd, Pv);
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) P[i][j] += Pv[i][j];
                }
            } else {
                R H[3][3];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) H[i][j] = R(0);
                if (q == 0) {
                    element_nodes<R, NPE>(xs, ys, zs, lc, ua);
                    if (DAMP) element_velocities<R, NPE>(vs, lc, va);
                }
#pragma unroll
                for (int a = 0; a < NPE; ++a)
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) H[i][j] += ua[a][i] * g[a][j];
                R Em[3][3];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        R sm = H[i][j] + H[j][i];
#pragma unroll
                        for (int k = 0; k < 3; ++k) sm += H[k][i] * H[k][j];
                        Em[i][j] = R(0.5) * sm;
                    }
                const R trE = Em[0][0] + Em[1][1] + Em[2][2];
                R Sm[3][3];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) Sm[i][j] = R(2) * A.mu * Em[i][j] + (i == j ? A.lambda * trE : R(0));
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        R sm = Sm[i][j];
#pragma unroll
                        for (int k = 0; k < 3; ++k) sm += H[i][k] * Sm[k][j];
                        P[i][j] = sm;
                    }
                if (DAMP) {
                    R F[3][3], Fd[3][3], Pv[3][3];
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            F[i][j] = H[i][j] + (i == j ? R(1) : R(0));
                            Fd[i][j] = R(0);
                        }
#pragma unroll
                    for (int a = 0; a < NPE; ++a)
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int j = 0; j < 3; ++j) Fd[i][j] += va[a][i] * g[a][j];
                    kelvin_voigt<R>(F, Fd, A.eta, A.lamd, Pv);
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) P[i][j] += Pv[i][j];
                }
            }
            // f_a += (P grad_a) dV   (FEAT10DataFunc.cuh:417-449)
#pragma unroll
            for (int a = 0; a < NPE; ++a)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    R fc = R(0);
#pragma unroll
                    for (int j = 0; j < 3; ++j) fc += P[i][j] * g[a][j];
                    f[a][i] += fc * dv;
                }
        }
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
            for (int d = 0; d < 3; ++d) fe[(a * 3 + d) * TE + t] = f[a][d];
        consumer_sync();

        const int lb = A.node_off[tile], nl = A.node_off[tile + 1] - lb;
        const uint16_t* inc = A.inc + (size_t)tile * TE * NPE;
        for (int ln = t; ln < nl; ln += TE) {
            const int beg = ln ? A.ln_inc_end[lb + ln - 1] : 0;
            const int end = A.ln_inc_end[lb + ln];
            double s0 = 0.0, s1 = 0.0, s2 = 0.0;  // node sums in FP64 (near equilibrium they cancel)
            for (int k = beg; k < end; ++k) {
                const int ent = inc[k];
                const int base = (ent >> TILE_SHIFT) * 3 * TE + (ent & (TE - 1));
                s0 += fe[base];
                s1 += fe[base + TE];
                s2 += fe[base + 2 * TE];
            }
            const int ps = A.ln_pslot[lb + ln];
            if (ps < 0) {
                const int gid = A.ln_gid[lb + ln];
                A.f_out[3 * gid + 0] = s0;
                A.f_out[3 * gid + 1] = s1;
                A.f_out[3 * gid + 2] = s2;
            } else {
                A.partial[3 * ps + 0] = s0;
                A.partial[3 * ps + 1] = s1;
                A.partial[3 * ps + 2] = s2;
            }
        }
    }
    cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// One tile per CTA (4 CTAs/SM in FP32), with the tile's QP slices double-
// buffered in shared memory by 1-D bulk copies issued from thread 0: QP q+2 is
// requested as soon as every thread has read QP q into registers, so a slice is
// always in flight while the CTA computes.  The node positions are gathered by
// the threads while the first two slices land.

// Stage a tile's block of the tile-ordered node record (values, scatter destinations,
// incidence ends) by bulk copies completing on `bar` (thread 0; `bar` initialised with
// count 1).  The record holds every tile's nodes contiguously, padded to TILE_NODE_PAD
// entries, so the staging is three plus two copies instead of dependent gathers
// (local node -> global id -> value).
template <typename R>
__device__ __forceinline__ void issue_node_record(const TileArgs<R>& A, int tile, uint32_t bar, double* xs,
                                                  double* ys, double* zs, int* dsts, uint16_t* iends) {
    const int pb = A.pad_off[tile], np = A.pad_off[tile + 1] - pb;
    mbar_expect_tx(bar, (uint32_t)np * (3 * sizeof(double) + sizeof(int) + sizeof(uint16_t)));
    bulk_g2s(smem_u32(xs), A.sx + pb, np * sizeof(double), bar);
    bulk_g2s(smem_u32(ys), A.sy + pb, np * sizeof(double), bar);
    bulk_g2s(smem_u32(zs), A.sz + pb, np * sizeof(double), bar);
    bulk_g2s(smem_u32(dsts), A.pad_dst + pb, np * sizeof(int), bar);
    bulk_g2s(smem_u32(iends), A.pad_iend + pb, np * sizeof(uint16_t), bar);
}

// Velocities of a tile's local nodes for the Kelvin-Voigt term (gathered).
template <typename R>
__device__ __forceinline__ void stage_tile_velocities(const TileArgs<R>& A, int tile, int nl, double* vs) {
    const int pb = A.pad_off[tile];
    for (int ln = threadIdx.x; ln < nl; ln += TILE_ELEMS) {
        const int g = A.pad_gid[pb + ln];
        vs[3 * ln + 0] = A.v[3 * g + 0];
        vs[3 * ln + 1] = A.v[3 * g + 1];
        vs[3 * ln + 2] = A.v[3 * g + 2];
    }
}

template <typename R, int NPE>
struct TileTmaGeom {
    static constexpr uint32_t GRAD_BYTES = NPE * 3 * TILE_ELEMS * sizeof(R);
    static constexpr uint32_t DV_BYTES = TILE_ELEMS * sizeof(R);
    static constexpr uint32_t STAGE_BYTES = GRAD_BYTES + DV_BYTES;
    static constexpr uint32_t LCONN_BYTES = NPE * TILE_ELEMS * sizeof(uint16_t);
    static constexpr uint32_t INC_BYTES = NPE * TILE_ELEMS * sizeof(uint16_t);
    // QP-slice stages: FP64 copies a slice into registers before computing it, so one
    // stage suffices (refilled as soon as it is read); FP32 reads a slice twice (H, then
    // the forces) and double-buffers
    static constexpr int STAGES = sizeof(R) == 8 ? 1 : 2;
    // element forces of the scatter reuse the stages once the QP loop is done
    static_assert(3 * NPE * TILE_ELEMS * sizeof(R) <= STAGES * STAGE_BYTES, "force table must fit in the stages");
    static_assert(LCONN_BYTES % 16 == 0 && INC_BYTES % 16 == 0 && STAGE_BYTES % 16 == 0, "bulk sizes");
};

// Byte offsets of the regions of k_tile_force_tma's shared memory, each
// 16-byte aligned: [stage(s), later the element forces][lconn][incidence]
// [x y z][node destination][incidence end][velocities][a barrier per stage, the node
// record's].
template <typename R, int NPE>
struct TileTmaLayout {
    size_t inc, pos, dst, iend, vel, bar, total;
    __host__ __device__ TileTmaLayout(int max_local, bool damp) {
        using G = TileTmaGeom<R, NPE>;
        auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
        inc = G::STAGES * (size_t)G::STAGE_BYTES + G::LCONN_BYTES;
        pos = inc + G::INC_BYTES;
        dst = al(pos + 3 * (size_t)max_local * sizeof(double));
        iend = al(dst + (size_t)max_local * sizeof(int));
        vel = al(iend + (size_t)max_local * sizeof(uint16_t));
        bar = al(vel + (damp ? 3 * (size_t)max_local * sizeof(double) : 0));
        total = bar + (G::STAGES + 1) * sizeof(unsigned long long);
    }
};

template <typename R, int NPE>
inline size_t tile_tma_smem_bytes(int max_local, bool damp) {
    return TileTmaLayout<R, NPE>(max_local, damp).total;
}

template <typename R, int NPE, int NQP, bool DAMP>
__global__ void __launch_bounds__(TILE_ELEMS, sizeof(R) == 4 ? 4 : 3) k_tile_force_tma(TileArgs<R> A, int* err) {
    using G = TileTmaGeom<R, NPE>;
    constexpr int S = G::STAGES;
    constexpr int TE = TILE_ELEMS;
    extern __shared__ __align__(128) unsigned char smem[];
    const int tile = blockIdx.x, t = threadIdx.x;
    const int ML = A.max_local;
    const TileTmaLayout<R, NPE> L(ML, DAMP);
    unsigned char* stage0 = smem;
    const uint16_t* lcs = reinterpret_cast<const uint16_t*>(smem + S * G::STAGE_BYTES);
    const uint16_t* incs = reinterpret_cast<const uint16_t*>(smem + L.inc);
    double* xs = reinterpret_cast<double*>(smem + L.pos);
    double* ys = xs + ML;
    double* zs = ys + ML;
    int* dsts = reinterpret_cast<int*>(smem + L.dst);  // global node id, or -(partial slot + 1)
    uint16_t* iends = reinterpret_cast<uint16_t*>(smem + L.iend);
    double* vs = reinterpret_cast<double*>(smem + L.vel);
    R* fe = reinterpret_cast<R*>(smem);  // aliases the stages after the QP loop
    const uint32_t bar0 = smem_u32(smem + L.bar);

    // slice q goes to stage q % S, completing phase (q / S) of that stage's barrier
    auto issue = [&](int q) {  // thread 0 only
        const uint32_t bar = bar0 + 8 * (q % S);
        const uint32_t dst = smem_u32(stage0 + (size_t)(q % S) * G::STAGE_BYTES);
        const uint32_t extra = (q == 0) ? G::LCONN_BYTES + G::INC_BYTES : 0;
        mbar_expect_tx(bar, G::STAGE_BYTES + extra);
        bulk_g2s(dst, A.grad + ((size_t)tile * NQP + q) * (NPE * 3) * TE, G::GRAD_BYTES, bar);
        bulk_g2s(dst + G::GRAD_BYTES, A.dv + ((size_t)tile * NQP + q) * TE, G::DV_BYTES, bar);
        if (q == 0) {
            bulk_g2s(smem_u32(lcs), A.lconn + (size_t)tile * NPE * TE, G::LCONN_BYTES, bar);
            bulk_g2s(smem_u32(incs), A.inc + (size_t)tile * NPE * TE, G::INC_BYTES, bar);
        }
    };
    if (t == 0) {
        for (int k = 0; k <= S; ++k) mbar_init(bar0 + 8 * k, 1);  // S stages, then the node record
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (int q = 0; q < S && q < NQP; ++q) issue(q);
        issue_node_record(A, tile, bar0 + 8 * S, xs, ys, zs, dsts, iends);
    }
    const int nl = A.node_off[tile + 1] - A.node_off[tile];
    if (DAMP) stage_tile_velocities(A, tile, nl, vs);
    __syncthreads();  // barriers initialised (velocities staged)
    if (!mbar_wait(bar0 + 8 * S, 0)) atomicExch(err, 3);  // the node record

    if constexpr (sizeof(R) == 4) {
        // FP32: paired arithmetic (two nodes per instruction, __ffma2_rn).  The
        // element's node displacements are gathered from shared memory once per tile
        // into registers, node pairs side by side; each QP slice is read as node
        // pairs (grad_slot<float>), H = sum_a u_a (x) gradN_a and the element forces
        // f_a += (P dV) gradN_a accumulate two nodes per instruction.
        constexpr int NP = NPE / 2;
        if (!mbar_wait(bar0, 0)) atomicExch(err, 3);  // stage 0 brings lconn and the incidence
        int lc[NPE];
#pragma unroll
        for (int a = 0; a < NPE; ++a) lc[a] = lcs[a * TE + t];
        float2 up[NP][3], f2[NP][3];
        {
            // element_nodes' values (relative to the element's first node, differenced in
            // FP64, rounded once), formed directly as node pairs
            const double* sv[3] = {xs, ys, zs};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double b = sv[d][lc[0]];
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    up[p][d] = make_float2(float(sv[d][lc[2 * p]] - b), float(sv[d][lc[2 * p + 1]] - b));
                    f2[p][d] = make_float2(0.f, 0.f);
                }
            }
        }

        // velocities relative to the element's first node, differenced per QP (keeping
        // them in registers would spill)
        double vb[3] = {0.0, 0.0, 0.0};
        if constexpr (DAMP) {
#pragma unroll
            for (int d = 0; d < 3; ++d) vb[d] = vs[3 * lc[0] + d];
        }
#pragma unroll 1
        for (int q = 0; q < NQP; ++q) {
            if (q > 0 && !mbar_wait(bar0 + 8 * (q % S), (q / S) & 1)) atomicExch(err, 3);
            const unsigned char* st = stage0 + (size_t)(q % S) * G::STAGE_BYTES;
            const float2* gs2 = reinterpret_cast<const float2*>(st);
            const float dv = reinterpret_cast<const float*>(st + G::GRAD_BYTES)[t];
            float2 h2[3][3], fd2[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) h2[i][j] = fd2[i][j] = make_float2(0.f, 0.f);
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                float2 g[3];
#pragma unroll
                for (int j = 0; j < 3; ++j) g[j] = gs2[(p * 3 + j) * TE + t];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) h2[i][j] = __ffma2_rn(up[p][i], g[j], h2[i][j]);
                if (DAMP) {
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const float2 v2 = make_float2(float(vs[3 * lc[2 * p] + i] - vb[i]),
                                                      float(vs[3 * lc[2 * p + 1] + i] - vb[i]));
#pragma unroll
                        for (int j = 0; j < 3; ++j) fd2[i][j] = __ffma2_rn(v2, g[j], fd2[i][j]);
                    }
                }
            }
            float H[3][3], Fd[3][3], P[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    H[i][j] = h2[i][j].x + h2[i][j].y;
                    Fd[i][j] = fd2[i][j].x + fd2[i][j].y;
                }
            tile_stress<float, DAMP, false>(H, Fd, reinterpret_cast<const TileArgs<float>&>(A), P, float(A.lambda),
                                            float(A.mu));
            // f_a += (P dV) grad_a   (FEAT10DataFunc.cuh:417-449), two nodes per instruction
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                float2 g[3];
#pragma unroll
                for (int j = 0; j < 3; ++j) g[j] = gs2[(p * 3 + j) * TE + t];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const float pij = P[i][j] * dv;
                        f2[p][i] = __ffma2_rn(make_float2(pij, pij), g[j], f2[p][i]);
                    }
            }
            if (q + S < NQP) {
                // every thread's generic reads of this stage precede the bulk refill
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncthreads();
                if (t == 0) issue(q + S);
            }
        }
        __syncthreads();  // every thread is done with the stages the force table reuses
#pragma unroll
        for (int p = 0; p < NP; ++p)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                fe[((2 * p) * 3 + d) * TE + t] = f2[p][d].x;
                fe[((2 * p + 1) * 3 + d) * TE + t] = f2[p][d].y;
            }
        __syncthreads();
    } else {
        int lc[NPE];
        R f[NPE][3];
    #pragma unroll
        for (int a = 0; a < NPE; ++a) f[a][0] = f[a][1] = f[a][2] = R(0);
    #pragma unroll 1
        for (int q = 0; q < NQP; ++q) {
            if (!mbar_wait(bar0 + 8 * (q % S), (q / S) & 1)) atomicExch(err, 3);
            const unsigned char* st = stage0 + (size_t)(q % S) * G::STAGE_BYTES;
            const R* gs = reinterpret_cast<const R*>(st);
            if (q == 0) {
    #pragma unroll
                for (int a = 0; a < NPE; ++a) lc[a] = lcs[a * TE + t];
            }
            R g[NPE][3];
    #pragma unroll
            for (int a = 0; a < NPE; ++a)
    #pragma unroll
                for (int j = 0; j < 3; ++j) g[a][j] = gs[grad_slot<R>(a, j, t)];
            const R dv = reinterpret_cast<const R*>(st + G::GRAD_BYTES)[t];
            if (q + S < NQP) {
                // every thread's generic reads of this stage precede the bulk refill
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncthreads();
                if (t == 0) issue(q + S);
            }
            R P[3][3];
            {
                double F[3][3];
    #pragma unroll
                for (int i = 0; i < 3; ++i)
    #pragma unroll
                    for (int j = 0; j < 3; ++j) F[i][j] = 0.0;
    #pragma unroll
                for (int a = 0; a < NPE; ++a) {
                    const double xa[3] = {xs[lc[a]], ys[lc[a]], zs[lc[a]]};
    #pragma unroll
                    for (int i = 0; i < 3; ++i)
    #pragma unroll
                        for (int j = 0; j < 3; ++j) F[i][j] += xa[i] * g[a][j];
                }
                svk_p_reference(F, A.lambda, A.mu, P);
                if (DAMP) {
                    double Fd[3][3], Pv[3][3];
    #pragma unroll
                    for (int i = 0; i < 3; ++i)
    #pragma unroll
                        for (int j = 0; j < 3; ++j) Fd[i][j] = 0.0;
    #pragma unroll
                    for (int a = 0; a < NPE; ++a)
    #pragma unroll
                        for (int i = 0; i < 3; ++i)
    #pragma unroll
                            for (int j = 0; j < 3; ++j) Fd[i][j] += vs[3 * lc[a] + i] * g[a][j];
                    kelvin_voigt<double>(F, Fd, A.eta, A.lamd, Pv);
    #pragma unroll
                    for (int i = 0; i < 3; ++i)
    #pragma unroll
                        for (int j = 0; j < 3; ++j) P[i][j] += Pv[i][j];
                }
            }
            // f_a += (P dV) grad_a   (FEAT10DataFunc.cuh:417-449)
    #pragma unroll
            for (int i = 0; i < 3; ++i)
    #pragma unroll
                for (int j = 0; j < 3; ++j) P[i][j] *= dv;
    #pragma unroll
            for (int a = 0; a < NPE; ++a)
    #pragma unroll
                for (int i = 0; i < 3; ++i) f[a][i] += P[i][0] * g[a][0] + P[i][1] * g[a][1] + P[i][2] * g[a][2];
        }
        __syncthreads();  // every thread is done with the stages the force table reuses
    #pragma unroll
        for (int a = 0; a < NPE; ++a)
    #pragma unroll
            for (int d = 0; d < 3; ++d) fe[(a * 3 + d) * TE + t] = f[a][d];
        __syncthreads();
    }

    for (int ln = t; ln < nl; ln += TE) {
        const int beg = ln ? iends[ln - 1] : 0;
        const int end = iends[ln];
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;  // node sums in FP64 (near equilibrium they cancel)
        for (int k = beg; k < end; ++k) {
            const int ent = incs[k];
            const int base = (ent >> TILE_SHIFT) * 3 * TE + (ent & (TE - 1));
            s0 += fe[base];
            s1 += fe[base + TE];
            s2 += fe[base + 2 * TE];
        }
        const int dn = dsts[ln];
        if (dn >= 0) {
            A.f_out[3 * dn + 0] = s0;
            A.f_out[3 * dn + 1] = s1;
            A.f_out[3 * dn + 2] = s2;
        } else {
            const int ps = -dn - 1;
            A.partial[3 * ps + 0] = s0;
            A.partial[3 * ps + 1] = s1;
            A.partial[3 * ps + 2] = s2;
        }
    }
    // outputs written: the combine kernel (a programmatic dependent) may be scheduled
    asm volatile("griddepcontrol.launch_dependents;");
}

// ---------------------------------------------------------------------------
// Compact-geometry variant of k_tile_force_tma: the per-QP slices hold J^-1
// (9 values) and dV instead of 3 * NPE gradients, and F = (dx/dxi) J^-1 and the
// nodal forces Q dN/dxi (Q = dV P J^-T) follow the barycentric structure of the
// tetrahedral shape functions (tet_dx_dxi / tet_scatter).  Same forces to
// rounding, 10 / (3 NPE + 1) of the element stream.

template <typename R, int NPE>
struct TileGeoGeom {
    static constexpr uint32_t JI_BYTES = 9 * TILE_ELEMS * sizeof(R);
    static constexpr uint32_t DV_BYTES = TILE_ELEMS * sizeof(R);
    static constexpr uint32_t STAGE_BYTES = JI_BYTES + DV_BYTES;
    static constexpr uint32_t LCONN_BYTES = NPE * TILE_ELEMS * sizeof(uint16_t);
    static constexpr uint32_t INC_BYTES = NPE * TILE_ELEMS * sizeof(uint16_t);
    static constexpr uint32_t FE_BYTES = 3 * NPE * TILE_ELEMS * sizeof(R);
    // the two stages, and after the QP loop the element forces of the scatter
    static constexpr uint32_t REGION0 =
        ((2 * STAGE_BYTES > FE_BYTES ? 2 * STAGE_BYTES : FE_BYTES) + 15u) & ~15u;
    static_assert(LCONN_BYTES % 16 == 0 && INC_BYTES % 16 == 0 && STAGE_BYTES % 16 == 0, "bulk sizes");
};

template <typename R, int NPE>
struct TileGeoLayout {
    size_t lconn, inc, pos, dst, iend, vel, bar, total;
    __host__ __device__ TileGeoLayout(int max_local, bool damp) {
        using G = TileGeoGeom<R, NPE>;
        auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
        lconn = G::REGION0;
        inc = lconn + G::LCONN_BYTES;
        pos = inc + G::INC_BYTES;
        dst = al(pos + 3 * (size_t)max_local * sizeof(double));
        iend = al(dst + (size_t)max_local * sizeof(int));
        vel = al(iend + (size_t)max_local * sizeof(uint16_t));
        bar = al(vel + (damp ? 3 * (size_t)max_local * sizeof(double) : 0));
        total = bar + 3 * sizeof(unsigned long long);  // two stage barriers, the node record's
    }
};

template <typename R, int NPE>
inline size_t tile_geo_smem_bytes(int max_local, bool damp) {
    return TileGeoLayout<R, NPE>(max_local, damp).total;
}

template <typename R, int NPE, int NQP, bool DAMP, bool MR = false>
__global__ void __launch_bounds__(TILE_ELEMS) k_tile_force_geo(TileArgs<R> A, int* err) {
    using G = TileGeoGeom<R, NPE>;
    constexpr int TE = TILE_ELEMS;
    extern __shared__ __align__(128) unsigned char smem[];
    const int tile = blockIdx.x, t = threadIdx.x;
    const int ML = A.max_local;
    const TileGeoLayout<R, NPE> L(ML, DAMP);
    unsigned char* stage0 = smem;
    const uint16_t* lcs = reinterpret_cast<const uint16_t*>(smem + L.lconn);
    const uint16_t* incs = reinterpret_cast<const uint16_t*>(smem + L.inc);
    double* xs = reinterpret_cast<double*>(smem + L.pos);
    double* ys = xs + ML;
    double* zs = ys + ML;
    int* dsts = reinterpret_cast<int*>(smem + L.dst);  // global node id, or -(partial slot + 1)
    uint16_t* iends = reinterpret_cast<uint16_t*>(smem + L.iend);
    double* vs = reinterpret_cast<double*>(smem + L.vel);
    R* fe = reinterpret_cast<R*>(smem);  // aliases the stages after the QP loop
    const uint32_t bar0 = smem_u32(smem + L.bar);

    auto issue = [&](int q) {  // thread 0 only
        const uint32_t bar = bar0 + 8 * (q & 1);
        const uint32_t dst = smem_u32(stage0 + (size_t)(q & 1) * G::STAGE_BYTES);
        const uint32_t extra = (q == 0) ? G::LCONN_BYTES + G::INC_BYTES : 0;
        mbar_expect_tx(bar, G::STAGE_BYTES + extra);
        bulk_g2s(dst, A.ji + ((size_t)tile * NQP + q) * 9 * TE, G::JI_BYTES, bar);
        bulk_g2s(dst + G::JI_BYTES, A.dv + ((size_t)tile * NQP + q) * TE, G::DV_BYTES, bar);
        if (q == 0) {
            bulk_g2s(smem_u32(lcs), A.lconn + (size_t)tile * NPE * TE, G::LCONN_BYTES, bar);
            bulk_g2s(smem_u32(incs), A.inc + (size_t)tile * NPE * TE, G::INC_BYTES, bar);
        }
    };
    if (t == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        mbar_init(bar0 + 16, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(0);
        if (NQP > 1) issue(1);
        issue_node_record(A, tile, bar0 + 16, xs, ys, zs, dsts, iends);
    }
    const int nl = A.node_off[tile + 1] - A.node_off[tile];
    if (DAMP) stage_tile_velocities(A, tile, nl, vs);
    __syncthreads();  // barriers initialised (velocities staged)
    if (!mbar_wait(bar0 + 16, 0)) atomicExch(err, 3);  // the node record

    int lc[NPE];
    R f[NPE][3], xa[NPE][3], va[NPE][3];
#pragma unroll 1
    for (int q = 0; q < NQP; ++q) {
        if (!mbar_wait(bar0 + 8 * (q & 1), (q >> 1) & 1)) atomicExch(err, 3);
        const unsigned char* st = stage0 + (size_t)(q & 1) * G::STAGE_BYTES;
        const R* js = reinterpret_cast<const R*>(st);
        if (q == 0) {
#pragma unroll
            for (int a = 0; a < NPE; ++a) lc[a] = lcs[a * TE + t];
        }
        R ji[9];
#pragma unroll
        for (int m = 0; m < 9; ++m) ji[m] = js[m * TE + t];
        const R dv = reinterpret_cast<const R*>(st + G::JI_BYTES)[t];
        if (q + 2 < NQP) {
            // every thread's generic reads of this stage precede the bulk refill
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (t == 0) issue(q + 2);
        }
        const R Lq[4] = {R(A.qb.L[q][0]), R(A.qb.L[q][1]), R(A.qb.L[q][2]), R(A.qb.L[q][3])};
        if (q == 0 || sizeof(R) == 8) {  // FP32 keeps the element-relative values in registers
            element_nodes<R, NPE>(xs, ys, zs, lc, xa);
            if (DAMP) element_velocities<R, NPE>(vs, lc, va);
        }
        // F (FP64) or H (FP32), the stress, f_a (+)= (dV P J^-T) dN_a/dxi
        // (FEAT10DataFunc.cuh:417-449 with gradN = J^-T dN/dxi)
        if (q == 0)
            compact_qp<R, NPE, DAMP, true, MR>(A, xa, va, ji, dv, Lq, f, A.lambda, A.mu);
        else
            compact_qp<R, NPE, DAMP, false, MR>(A, xa, va, ji, dv, Lq, f, A.lambda, A.mu);
    }
    __syncthreads();  // every thread is done with the stages the force table reuses
#pragma unroll
    for (int a = 0; a < NPE; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) fe[(a * 3 + d) * TE + t] = f[a][d];
    __syncthreads();

    for (int ln = t; ln < nl; ln += TE) {
        const int beg = ln ? iends[ln - 1] : 0;
        const int end = iends[ln];
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;  // node sums in FP64 (near equilibrium they cancel)
        for (int k = beg; k < end; ++k) {
            const int ent = incs[k];
            const int base = (ent >> TILE_SHIFT) * 3 * TE + (ent & (TE - 1));
            s0 += fe[base];
            s1 += fe[base + TE];
            s2 += fe[base + 2 * TE];
        }
        const int dn = dsts[ln];
        if (dn >= 0) {
            A.f_out[3 * dn + 0] = s0;
            A.f_out[3 * dn + 1] = s1;
            A.f_out[3 * dn + 2] = s2;
        } else {
            const int ps = -dn - 1;
            A.partial[3 * ps + 0] = s0;
            A.partial[3 * ps + 1] = s1;
            A.partial[3 * ps + 2] = s2;
        }
    }
    // outputs written: the combine kernel (a programmatic dependent) may be scheduled
    asm volatile("griddepcontrol.launch_dependents;");
}

}  // namespace tlfea
