// element.cu -- TET10 / TET4 element state, precompute, fused internal force,
// mass CSR and constraints behind the C ABI (include/tlfea_b200.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <mutex>
#include <numeric>
#include <tuple>
#include <vector>

#include "element.cuh"
#include "force_pipe.cuh"

namespace tlfea {

std::atomic<long long> g_launches{0};
static thread_local std::string t_last_error;
void set_error(const std::string& msg) { t_last_error = msg; }

// -------------------------------------------------------------- kernels

struct QuadParams {
    double qx[5], qy[5], qz[5], qw[5];
};

// solve_3x3_system (FEAT10DataFunc.cuh:32-84): Gaussian elimination with partial
// pivoting on [A|b]; |pivot| < 1e-14 gives the zero vector.
__device__ __forceinline__ void solve3_pivot(const double A[3][3], const double b[3], double xo[3]) {
    double aug[3][4];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) aug[i][j] = A[i][j];
        aug[i][3] = b[i];
    }
    for (int k = 0; k < 3; ++k) {
        int pr = k;
        double mv = fabs(aug[k][k]);
        for (int i = k + 1; i < 3; ++i)
            if (fabs(aug[i][k]) > mv) {
                mv = fabs(aug[i][k]);
                pr = i;
            }
        if (pr != k)
            for (int j = 0; j < 4; ++j) {
                double tmp = aug[k][j];
                aug[k][j] = aug[pr][j];
                aug[pr][j] = tmp;
            }
        if (fabs(aug[k][k]) < 1e-14) {
            xo[0] = xo[1] = xo[2] = 0.0;
            return;
        }
        for (int i = k + 1; i < 3; ++i) {
            const double f = aug[i][k] / aug[k][k];
            for (int j = k; j < 4; ++j) aug[i][j] -= f * aug[k][j];
        }
    }
    xo[2] = aug[2][3] / aug[2][2];
    xo[1] = (aug[1][3] - aug[1][2] * xo[2]) / aug[1][1];
    xo[0] = (aug[0][3] - aug[0][2] * xo[2] - aug[0][1] * xo[1]) / aug[0][0];
}

__device__ __forceinline__ double det3(const double J[3][3]) {
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

// CalcDnDuPre: one thread per (tile slot, QP).  T10 follows dn_du_pre_kernel
// (FEAT10Data.cu:92-198), T4 follows dn_du_pre_feat4_kernel (FEAT4Data.cu:98-195).
// Writes the tiled FP64 and FP32 gradient streams, dV = detJ*w, and detJ in the
// reference layout.
template <int NPE, int NQP>
__global__ void k_dndu_pre(int n_slots, int E, const int* __restrict__ tile_elem, const int* __restrict__ conn,
                           const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                           QuadParams qp, double* grad64, float* grad32, double* dv64, float* dv32, double* detJ,
                           double* ji64, float* ji32) {
    constexpr int TE = TILE_ELEMS;
    const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gtid >= (long long)n_slots * NQP) return;
    const int slot = (int)(gtid / NQP);
    const int q = (int)(gtid % NQP);
    const int tile = slot / TE, t = slot % TE;
    const int e = tile_elem[slot];
    double gN[NPE][3];
    double Jinv[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};  // dxi/dX
    double dj = 0.0;
    if (e >= 0) {
        double dN[NPE][3];
        if (NPE == 10) {
            const double xi = qp.qx[q], eta = qp.qy[q], zeta = qp.qz[q];
            const double L[4] = {1.0 - xi - eta - zeta, xi, eta, zeta};
            const double dL[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
            const int edges[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
            for (int i = 0; i < 4; ++i) {
                const double f = 4.0 * L[i] - 1.0;
                for (int j = 0; j < 3; ++j) dN[i][j] = f * dL[i][j];
            }
            for (int k = 0; k < 6; ++k) {
                const int i = edges[k][0], j = edges[k][1];
                for (int d = 0; d < 3; ++d) dN[k + 4][d] = 4.0 * (L[i] * dL[j][d] + L[j] * dL[i][d]);
            }
        } else {
            const double d4[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
            for (int a = 0; a < 4; ++a)
                for (int j = 0; j < 3; ++j) dN[a][j] = d4[a][j];
        }
        double J[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
        for (int a = 0; a < NPE; ++a) {
            const int n = conn[e + (size_t)a * E];
            const double X[3] = {x[n], y[n], z[n]};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) J[i][j] += X[i] * dN[a][j];
        }
        dj = det3(J);
        double JT[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) JT[i][j] = J[j][i];
        if (NPE == 10) {
            for (int a = 0; a < NPE; ++a) solve3_pivot(JT, dN[a], gN[a]);
            // row k of J^-1 solves J^T y = e_k by the same elimination, so a
            // degenerate element (tiny pivot) gets a zero inverse, as its
            // gradients are zero
            for (int k = 0; k < 3; ++k) {
                const double ek[3] = {k == 0 ? 1.0 : 0.0, k == 1 ? 1.0 : 0.0, k == 2 ? 1.0 : 0.0};
                solve3_pivot(JT, ek, Jinv[k]);
            }
        } else {
            const double dT = det3(JT);
            const double inv = (dT != 0.0) ? 1.0 / dT : 0.0;
            double Ji[3][3];
            Ji[0][0] = (JT[1][1] * JT[2][2] - JT[1][2] * JT[2][1]) * inv;
            Ji[0][1] = -(JT[0][1] * JT[2][2] - JT[0][2] * JT[2][1]) * inv;
            Ji[0][2] = (JT[0][1] * JT[1][2] - JT[0][2] * JT[1][1]) * inv;
            Ji[1][0] = -(JT[1][0] * JT[2][2] - JT[1][2] * JT[2][0]) * inv;
            Ji[1][1] = (JT[0][0] * JT[2][2] - JT[0][2] * JT[2][0]) * inv;
            Ji[1][2] = -(JT[0][0] * JT[1][2] - JT[0][2] * JT[1][0]) * inv;
            Ji[2][0] = (JT[1][0] * JT[2][1] - JT[1][1] * JT[2][0]) * inv;
            Ji[2][1] = -(JT[0][0] * JT[2][1] - JT[0][1] * JT[2][0]) * inv;
            Ji[2][2] = (JT[0][0] * JT[1][1] - JT[0][1] * JT[1][0]) * inv;
            for (int a = 0; a < NPE; ++a)
                for (int i = 0; i < 3; ++i) {
                    double s = 0.0;
                    for (int j = 0; j < 3; ++j) s += Ji[i][j] * dN[a][j];
                    gN[a][i] = s;
                }
            for (int k = 0; k < 3; ++k)
                for (int j = 0; j < 3; ++j) Jinv[k][j] = Ji[j][k];  // Ji = (J^T)^-1
        }
        detJ[(size_t)e * NQP + q] = dj;
    } else {
        for (int a = 0; a < NPE; ++a) gN[a][0] = gN[a][1] = gN[a][2] = 0.0;
    }
    const size_t gb = ((size_t)tile * NQP + q) * (NPE * 3) * TE;
    for (int a = 0; a < NPE; ++a)
        for (int j = 0; j < 3; ++j) {
            grad64[gb + grad_slot<double>(a, j, t)] = gN[a][j];
            grad32[gb + grad_slot<float>(a, j, t)] = (float)gN[a][j];
        }
    const double dv = (e >= 0) ? dj * qp.qw[q] : 0.0;
    dv64[((size_t)tile * NQP + q) * TE + t] = dv;
    dv32[((size_t)tile * NQP + q) * TE + t] = (float)dv;
    const size_t jb = ((size_t)tile * NQP + q) * 9 * TE + t;
    for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) {
            ji64[jb + (size_t)(3 * k + j) * TE] = Jinv[k][j];
            ji32[jb + (size_t)(3 * k + j) * TE] = (float)Jinv[k][j];
        }
}

template <typename R, int NPE, int NQP, int MODE, bool DAMP, bool MR>
__global__ void __launch_bounds__(TILE_ELEMS) k_tile_force(TileArgs<R> A) {
    extern __shared__ __align__(128) unsigned char smem[];
    process_tile<R, NPE, NQP, MODE, DAMP, MR>(A, blockIdx.x, smem);
}

// Sum of each shared node's per-tile partials, in tile order.  Partial slots
// are numbered by shared node (build_tiling), so node b's partials are the
// contiguous range [boff[b], boff[b+1]) and consecutive threads read
// consecutive memory.
template <typename R, bool ACCUM>
__global__ void k_combine(int nb, const int* __restrict__ bgid, const int* __restrict__ boff,
                          const R* __restrict__ partial, R* f_out) {
    // launched as a programmatic dependent of the force kernel: its blocks may be
    // scheduled while the force kernel drains, and wait here until it has completed
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;  // node sums in FP64 (near equilibrium they cancel)
    for (int k = boff[b]; k < boff[b + 1]; ++k) {
        s0 += partial[3 * k + 0];
        s1 += partial[3 * k + 1];
        s2 += partial[3 * k + 2];
    }
    const int g = bgid[b];
    if (ACCUM) {
        f_out[3 * g + 0] += s0;
        f_out[3 * g + 1] += s1;
        f_out[3 * g + 2] += s2;
    } else {
        f_out[3 * g + 0] = s0;
        f_out[3 * g + 1] = s1;
        f_out[3 * g + 2] = s2;
    }
}

// f_ext[3i+d] += g_d * sum_j M_ij: the body force of a uniform acceleration g on
// the consistent mass (the node pattern's mass rows), one thread per node row.
__global__ void k_add_gravity(int N, const int* __restrict__ off, const double* __restrict__ m, double gx, double gy,
                              double gz, double* f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double s = 0.0;
    for (int k = off[i]; k < off[i + 1]; ++k) s += m[k];
    f[3 * i + 0] += s * gx;
    f[3 * i + 1] += s * gy;
    f[3 * i + 2] += s * gz;
}

// u64[3i + d] = x_d[i] - X0_d[i], node order (coalesced).
__global__ void k_disp64(int n, const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ z, const double* __restrict__ X0x, const double* __restrict__ X0y,
                         const double* __restrict__ X0z, double* __restrict__ u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u[3 * i + 0] = x[i] - X0x[i];
    u[3 * i + 1] = y[i] - X0y[i];
    u[3 * i + 2] = z[i] - X0z[i];
}

__global__ void k_f32_to_f64(long long n, const float* __restrict__ a, double* b) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}

struct MassParams {
    double N[5][10];
    double w[5];
};

// Consistent mass, one thread per node row: for every incident (element, slot a)
// in element order and every slot b, add sum_q rho N_a N_b detJ w_q to the
// (row, conn(e,b)) entry.  Same per-entry formula as mass_matrix_qp_kernel
// (FEAT10Data.cu:200-271; FEAT4Data.cu:197-243); the additions into one entry
// happen in a fixed order instead of atomicAdd.
template <int NPE, int NQP>
__global__ void k_mass_rows(int N, int E, double rho, const int* __restrict__ conn, const double* __restrict__ detJ,
                            const int* __restrict__ inc_off, const int* __restrict__ inc_e,
                            const int* __restrict__ inc_a, const int* __restrict__ off, const int* __restrict__ col,
                            double* val, MassParams mp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int rb = off[i], re = off[i + 1];
    for (int k = rb; k < re; ++k) val[k] = 0.0;
    for (int k = inc_off[i]; k < inc_off[i + 1]; ++k) {
        const int e = inc_e[k], a = inc_a[k];
        for (int b = 0; b < NPE; ++b) {
            const int jg = conn[e + (size_t)b * E];
            double m = 0.0;
            for (int q = 0; q < NQP; ++q) m += rho * mp.N[q][a] * mp.N[q][b] * detJ[(size_t)e * NQP + q] * mp.w[q];
            int lo = rb, hi = re - 1, pos = -1;
            while (lo <= hi) {
                const int mid = lo + ((hi - lo) >> 1);
                const int v = col[mid];
                if (v == jg) {
                    pos = mid;
                    break;
                }
                if (v < jg)
                    lo = mid + 1;
                else
                    hi = mid - 1;
            }
            if (pos >= 0) val[pos] += m;
        }
    }
}

// c = x(fixed) - x_jac(fixed)  (compute_constraint_data, FEAT10DataFunc.cuh:470-481)
__global__ void k_constraint(int n_fixed, const int* __restrict__ fixed, const double* __restrict__ x,
                             const double* __restrict__ y, const double* __restrict__ z, const double* __restrict__ xj,
                             const double* __restrict__ yj, const double* __restrict__ zj, double* c) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_fixed) return;
    const int n = fixed[k];
    c[3 * k + 0] = x[n] - xj[n];
    c[3 * k + 1] = y[n] - yj[n];
    c[3 * k + 2] = z[n] - zj[n];
}

// -------------------------------------------------------------- host helpers

static inline unsigned long long spread3(unsigned long long v) {
    v &= 0x1fffffULL;
    v = (v | (v << 32)) & 0x1f00000000ffffULL;
    v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
    v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
    v = (v | (v << 2)) & 0x1249249249249249ULL;
    return v;
}

static void free_tiling(Tiling& tl) {
    dfree(tl.node_off);
    dfree(tl.ln_gid);
    dfree(tl.ln_pslot);
    dfree(tl.ln_inc_end);
    dfree(tl.inc);
    dfree(tl.lconn);
    dfree(tl.tile_elem);
    dfree(tl.elem_slot);
    dfree(tl.bnode_gid);
    dfree(tl.bnode_off);
    dfree(tl.bnode_slots);
    dfree(tl.node_bidx);
    dfree(tl.pad_off);
    dfree(tl.pad_gid);
    dfree(tl.pad_dst);
    dfree(tl.pad_iend);
    dfree(tl.sx);
    dfree(tl.sy);
    dfree(tl.sz);
    dfree(tl.grad64);
    dfree(tl.dv64);
    dfree(tl.grad32);
    dfree(tl.dv32);
    dfree(tl.ji64);
    dfree(tl.ji32);
    dfree(tl.partial64);
    dfree(tl.partial32);
    tl = Tiling();
}

// Device copy of a host vector, ordered on `stream` and complete on return.
template <typename T>
static int upload(T** d, const std::vector<T>& v, cudaStream_t stream) {
    int st = dalloc(d, v.size());
    if (st) return st;
    if (!v.empty()) {
        TLFEA_CUDA(cudaMemcpyAsync(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
        TLFEA_CUDA(cudaStreamSynchronize(stream));
    }
    return TLFEA_OK;
}

// Host-side construction of the tiles (see element.cuh for the layout).
static int build_tiling(tlfea_element_s* h, const double* x, const double* y, const double* z) {
    Tiling& tl = h->tl;
    const int E = h->E, N = h->N, npe = h->npe, TE = TILE_ELEMS;
    const std::vector<int>& conn = h->conn;

    // 1. Morton order of element centroids (corner nodes), isotropic scaling.
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < N; ++i) {
        const double p[3] = {x[i], y[i], z[i]};
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], p[d]);
            hi[d] = std::max(hi[d], p[d]);
        }
    }
    double ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
    if (!(ext > 0.0)) ext = 1.0;
    // (group, Morton code, element): a batch of meshes sorts instance by instance
    std::vector<std::tuple<int, unsigned long long, int>> key((size_t)E);
    const bool grouped = h->elem_group.size() == (size_t)E;
    for (int e = 0; e < E; ++e) {
        double c[3] = {0, 0, 0};
        for (int a = 0; a < 4; ++a) {
            const int n = conn[e + (size_t)a * E];
            c[0] += x[n];
            c[1] += y[n];
            c[2] += z[n];
        }
        unsigned long long m = 0;
        for (int d = 0; d < 3; ++d) {
            double u = (c[d] * 0.25 - lo[d]) / ext;
            u = std::min(std::max(u, 0.0), 1.0);
            const unsigned long long qd = (unsigned long long)(u * 2097151.0);
            m |= spread3(qd) << d;
        }
        key[e] = {grouped ? h->elem_group[e] : 0, m, e};
    }
    std::sort(key.begin(), key.end());

    // 2. Tiles.
    const int n_tiles = (E + TE - 1) / TE;
    tl.n_tiles = n_tiles;
    std::vector<int> tile_elem((size_t)n_tiles * TE, -1);
    for (int s = 0; s < E; ++s) tile_elem[s] = std::get<2>(key[s]);

    std::vector<int> total_inc((size_t)N, 0);
    for (size_t k = 0; k < conn.size(); ++k) total_inc[conn[k]]++;
    int orphans = 0;
    for (int i = 0; i < N; ++i) orphans += (total_inc[i] == 0);
    tl.n_orphans = orphans;

    std::vector<int> node_off((size_t)n_tiles + 1, 0);
    std::vector<int> ln_gid, ln_pslot;
    std::vector<uint16_t> ln_inc_end;
    std::vector<uint16_t> inc((size_t)n_tiles * TE * npe, 0);
    std::vector<uint16_t> lconn((size_t)n_tiles * npe * TE, 0);
    std::vector<int> stamp((size_t)N, -1), lidx((size_t)N, 0);
    std::vector<std::vector<int>> node_slots;  // per boundary gid: pslots (tile order)
    std::vector<int> gid_to_b((size_t)N, -1);
    std::vector<int> bnode_gid;
    int n_pslots = 0, max_local = 0;
    std::vector<int> nodes, cnt, pos;
    for (int tile = 0; tile < n_tiles; ++tile) {
        nodes.clear();
        for (int t = 0; t < TE; ++t) {
            const int e = tile_elem[(size_t)tile * TE + t];
            if (e < 0) continue;
            for (int a = 0; a < npe; ++a) {
                const int n = conn[e + (size_t)a * E];
                if (stamp[n] != tile) {
                    stamp[n] = tile;
                    nodes.push_back(n);
                }
            }
        }
        std::sort(nodes.begin(), nodes.end());
        const int nl = (int)nodes.size();
        max_local = std::max(max_local, nl);
        for (int l = 0; l < nl; ++l) lidx[nodes[l]] = l;
        cnt.assign((size_t)nl, 0);
        for (int t = 0; t < TE; ++t) {
            const int e = tile_elem[(size_t)tile * TE + t];
            for (int a = 0; a < npe; ++a) {
                int l = 0;
                if (e >= 0) {
                    l = lidx[conn[e + (size_t)a * E]];
                    cnt[l]++;
                }
                lconn[((size_t)tile * npe + a) * TE + t] = (uint16_t)l;
            }
        }
        pos.assign((size_t)nl, 0);
        int run = 0;
        for (int l = 0; l < nl; ++l) {
            pos[l] = run;
            run += cnt[l];
            ln_inc_end.push_back((uint16_t)run);
        }
        for (int t = 0; t < TE; ++t) {
            const int e = tile_elem[(size_t)tile * TE + t];
            if (e < 0) continue;
            for (int a = 0; a < npe; ++a) {
                const int l = lidx[conn[e + (size_t)a * E]];
                inc[(size_t)tile * TE * npe + pos[l]++] = (uint16_t)((a << TILE_SHIFT) | t);
            }
        }
        for (int l = 0; l < nl; ++l) {
            const int g = nodes[l];
            ln_gid.push_back(g);
            if (cnt[l] == total_inc[g]) {
                ln_pslot.push_back(-1);
            } else {
                const int ps = n_pslots++;
                ln_pslot.push_back(ps);
                if (gid_to_b[g] < 0) {
                    gid_to_b[g] = (int)bnode_gid.size();
                    bnode_gid.push_back(g);
                    node_slots.emplace_back();
                }
                node_slots[gid_to_b[g]].push_back(ps);
            }
        }
        node_off[tile + 1] = node_off[tile] + nl;
    }
    // boundary CSR, sorted by node id (slots stay in tile order)
    std::vector<int> border(bnode_gid.size());
    std::iota(border.begin(), border.end(), 0);
    std::sort(border.begin(), border.end(), [&](int a, int b) { return bnode_gid[a] < bnode_gid[b]; });
    std::vector<int> bgid, boff(1, 0), bslots, node_bidx((size_t)N, -1);
    // Partial slots are renumbered by shared node (in node-id order), each node's
    // slots in tile order: a node's partials are one contiguous range, so the
    // combine streams them coalesced; the summation order is unchanged.
    std::vector<int> renum((size_t)std::max(n_pslots, 1), -1);
    for (int k : border) {
        node_bidx[bnode_gid[k]] = (int)bgid.size();
        bgid.push_back(bnode_gid[k]);
        for (int ps : node_slots[k]) {
            renum[ps] = (int)bslots.size();
            bslots.push_back((int)bslots.size());
        }
        boff.push_back((int)bslots.size());
    }
    for (int& ps : ln_pslot)
        if (ps >= 0) ps = renum[ps];
    tl.max_local = std::max(max_local, 1);
    tl.n_local_total = (long long)ln_gid.size();
    tl.n_pslots = n_pslots;
    tl.n_bnodes = (int)bgid.size();
    tl.h_tile_elem = tile_elem;

    // the tile-ordered node record, each tile's block padded to TILE_NODE_PAD entries
    std::vector<int> pad_off((size_t)n_tiles + 1, 0), pad_gid, pad_dst;
    std::vector<uint16_t> pad_iend;
    int max_pad = 0;
    for (int tile = 0; tile < n_tiles; ++tile) {
        const int b = node_off[tile], nl = node_off[tile + 1] - b;
        const int np = (nl + TILE_NODE_PAD - 1) / TILE_NODE_PAD * TILE_NODE_PAD;
        max_pad = std::max(max_pad, np);
        for (int l = 0; l < np; ++l) {
            if (l < nl) {
                const int g = ln_gid[(size_t)b + l], ps = ln_pslot[(size_t)b + l];
                pad_gid.push_back(g);
                pad_dst.push_back(ps < 0 ? g : -(ps + 1));
                pad_iend.push_back(ln_inc_end[(size_t)b + l]);
            } else {
                pad_gid.push_back(-1);
                pad_dst.push_back(0);
                pad_iend.push_back(0);
            }
        }
        pad_off[tile + 1] = pad_off[tile] + np;
    }
    tl.n_pad = (long long)pad_gid.size();
    tl.max_local_pad = std::max(max_pad, TILE_NODE_PAD);

    int st;
    if ((st = upload(&tl.pad_off, pad_off, h->stream))) return st;
    if ((st = upload(&tl.pad_gid, pad_gid, h->stream))) return st;
    if ((st = upload(&tl.pad_dst, pad_dst, h->stream))) return st;
    if ((st = upload(&tl.pad_iend, pad_iend, h->stream))) return st;
    if ((st = dalloc(&tl.sx, (size_t)tl.n_pad)) || (st = dalloc(&tl.sy, (size_t)tl.n_pad)) ||
        (st = dalloc(&tl.sz, (size_t)tl.n_pad)))
        return st;
    h->stage_content = 0;
    if ((st = upload(&tl.node_off, node_off, h->stream))) return st;
    if ((st = upload(&tl.ln_gid, ln_gid, h->stream))) return st;
    if ((st = upload(&tl.ln_pslot, ln_pslot, h->stream))) return st;
    if ((st = upload(&tl.ln_inc_end, ln_inc_end, h->stream))) return st;
    if ((st = upload(&tl.inc, inc, h->stream))) return st;
    if ((st = upload(&tl.lconn, lconn, h->stream))) return st;
    if ((st = upload(&tl.tile_elem, tile_elem, h->stream))) return st;
    std::vector<int> elem_slot((size_t)E);
    for (int s = 0; s < E; ++s) elem_slot[std::get<2>(key[s])] = s;
    if ((st = upload(&tl.elem_slot, elem_slot, h->stream))) return st;
    if ((st = upload(&tl.bnode_gid, bgid, h->stream))) return st;
    if ((st = upload(&tl.bnode_off, boff, h->stream))) return st;
    if ((st = upload(&tl.bnode_slots, bslots, h->stream))) return st;
    if ((st = upload(&tl.node_bidx, node_bidx, h->stream))) return st;
    const size_t ng = (size_t)n_tiles * h->nqp * npe * 3 * TE;
    const size_t nd = (size_t)n_tiles * h->nqp * TE;
    if ((st = dalloc(&tl.grad64, ng))) return st;
    if ((st = dalloc(&tl.grad32, ng))) return st;
    if ((st = dalloc(&tl.dv64, nd))) return st;
    if ((st = dalloc(&tl.dv32, nd))) return st;
    const size_t nj = (size_t)n_tiles * h->nqp * 9 * TE;
    if ((st = dalloc(&tl.ji64, nj))) return st;
    if ((st = dalloc(&tl.ji32, nj))) return st;
    TLFEA_CUDA(cudaMemsetAsync(tl.ji64, 0, nj * sizeof(double), h->stream));
    TLFEA_CUDA(cudaMemsetAsync(tl.ji32, 0, nj * sizeof(float), h->stream));
    if ((st = dalloc(&tl.partial64, (size_t)3 * std::max(n_pslots, 1)))) return st;
    if ((st = dalloc(&tl.partial32, (size_t)3 * std::max(n_pslots, 1)))) return st;
    TLFEA_CUDA(cudaMemsetAsync(tl.grad64, 0, ng * sizeof(double), h->stream));
    TLFEA_CUDA(cudaMemsetAsync(tl.grad32, 0, ng * sizeof(float), h->stream));
    TLFEA_CUDA(cudaMemsetAsync(tl.dv64, 0, nd * sizeof(double), h->stream));
    TLFEA_CUDA(cudaMemsetAsync(tl.dv32, 0, nd * sizeof(float), h->stream));
    return TLFEA_OK;
}

// node -> (element, slot) incidence, element order (BuildNodeIncidence, cpu_utils.cc:97-109)
static int build_incidence(tlfea_element_s* h) {
    const int E = h->E, N = h->N, npe = h->npe;
    h->h_inc_off.assign((size_t)N + 1, 0);
    for (size_t k = 0; k < h->conn.size(); ++k) h->h_inc_off[h->conn[k] + 1]++;
    for (int i = 0; i < N; ++i) h->h_inc_off[i + 1] += h->h_inc_off[i];
    std::vector<int> pos(h->h_inc_off.begin(), h->h_inc_off.end() - 1);
    h->h_inc_e.assign((size_t)E * npe, 0);
    h->h_inc_a.assign((size_t)E * npe, 0);
    for (int e = 0; e < E; ++e)
        for (int a = 0; a < npe; ++a) {
            const int n = h->conn[e + (size_t)a * E];
            h->h_inc_e[pos[n]] = e;
            h->h_inc_a[pos[n]] = a;
            pos[n]++;
        }
    int st;
    if ((st = upload(&h->inc_off, h->h_inc_off, h->stream))) return st;
    if ((st = upload(&h->inc_e, h->h_inc_e, h->stream))) return st;
    if ((st = upload(&h->inc_a, h->h_inc_a, h->stream))) return st;
    return TLFEA_OK;
}

// Node-level pattern: row i = sorted unique nodes of the elements touching i
// (the set BuildMassCSRPattern obtains from its key sort, FEAT10Data.cu:361-417).
int element_build_pattern(tlfea_element_s* h) {
    if (h->pat_off) return TLFEA_OK;
    const int N = h->N, E = h->E, npe = h->npe;
    std::vector<int>& off = h->h_pat_off;
    std::vector<int>& col = h->h_pat_col;
    off.assign((size_t)N + 1, 0);
    col.clear();
    std::vector<int> mark((size_t)N, -1), row;
    for (int i = 0; i < N; ++i) {
        row.clear();
        for (int k = h->h_inc_off[i]; k < h->h_inc_off[i + 1]; ++k) {
            const int e = h->h_inc_e[k];
            for (int b = 0; b < npe; ++b) {
                const int j = h->conn[e + (size_t)b * E];
                if (mark[j] != i) {
                    mark[j] = i;
                    row.push_back(j);
                }
            }
        }
        std::sort(row.begin(), row.end());
        col.insert(col.end(), row.begin(), row.end());
        off[i + 1] = (int)col.size();
    }
    h->pat_nnz = (long long)col.size();
    int st;
    if ((st = upload(&h->pat_off, off, h->stream))) return st;
    if ((st = upload(&h->pat_col, col, h->stream))) return st;
    return TLFEA_OK;
}

template <typename R>
static TileArgs<R> make_args(tlfea_element_s* h, bool fp32) {
    TileArgs<R> A;
    memset(&A, 0, sizeof(A));
    Tiling& tl = h->tl;
    A.node_off = tl.node_off;
    A.ln_gid = tl.ln_gid;
    A.ln_pslot = tl.ln_pslot;
    A.ln_inc_end = tl.ln_inc_end;
    A.inc = tl.inc;
    A.lconn = tl.lconn;
    A.tile_elem = tl.tile_elem;
    A.v = nullptr;
    A.Pst = h->Pst;
    A.lambda = (R)h->lambda;
    A.mu = (R)h->mu;
    A.eta = (R)h->eta_d;
    A.lamd = (R)h->lambda_d;
    A.max_local = tl.max_local_pad;  // staging regions hold a tile's padded record block
    A.pad_off = tl.pad_off;
    A.pad_dst = tl.pad_dst;
    A.pad_iend = tl.pad_iend;
    A.pad_gid = tl.pad_gid;
    A.sx = tl.sx;
    A.sy = tl.sy;
    A.sz = tl.sz;
    if constexpr (sizeof(R) == 8) {
        A.grad = (const R*)tl.grad64;
        A.ji = (const R*)tl.ji64;
        A.dv = (const R*)tl.dv64;
        A.px = (const R*)h->x;
        A.py = (const R*)h->y;
        A.pz = (const R*)h->z;
        A.u64 = A.x64 = A.y64 = A.z64 = A.X0x = A.X0y = A.X0z = nullptr;
        A.f_out = (R*)h->f_int;
        A.partial = (R*)tl.partial64;
    } else {
        A.grad = (const R*)tl.grad32;
        A.ji = (const R*)tl.ji32;
        A.dv = (const R*)tl.dv32;
        A.px = A.py = A.pz = nullptr;  // staged from x64 - X0 relative to each tile's anchor
        A.u64 = h->u64;
        A.x64 = h->x;
        A.y64 = h->y;
        A.z64 = h->z;
        A.X0x = h->X0x;
        A.X0y = h->X0y;
        A.X0z = h->X0z;
        A.f_out = (R*)h->f_int32;
        A.partial = (R*)tl.partial32;
    }
    A.qb = qp_bary(h);
    A.mu10 = h->mu10;
    A.mu01 = h->mu01;
    A.kappa = h->kappa;
    (void)fp32;
    return A;
}

template <typename R, int NPE, int NQP, int MODE, bool DAMP, bool MR = false>
static int launch_tiles(tlfea_element_s* h, const TileArgs<R>& A) {
    const size_t smem = tile_smem_bytes<R>(NPE, h->tl.max_local_pad, DAMP);
    if (smem > 200 * 1024) {
        set_error("tile shared memory exceeds 200 KB");
        return TLFEA_UNSUPPORTED;
    }
    if (smem > 48 * 1024)
        TLFEA_CUDA(cudaFuncSetAttribute(k_tile_force<R, NPE, NQP, MODE, DAMP, MR>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_tile_force<R, NPE, NQP, MODE, DAMP, MR><<<h->tl.n_tiles, TILE_ELEMS, smem, h->stream>>>(A);
    TLFEA_CHECK_LAUNCH();
    return TLFEA_OK;
}

template <typename R, bool ACCUM>
static int launch_combine(tlfea_element_s* h, const R* partial, R* f_out) {
    const int nb = h->tl.n_bnodes;
    if (nb == 0) return TLFEA_OK;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((nb + 255) / 256));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TLFEA_CUDA(cudaLaunchKernelEx(&cfg, k_combine<R, ACCUM>, nb, (const int*)h->tl.bnode_gid,
                                  (const int*)h->tl.bnode_off, partial, f_out));
    TLFEA_CHECK_LAUNCH();
    return TLFEA_OK;
}

// One tile per block, QP slices double-buffered by bulk copies.
template <typename R, int NPE, int NQP, bool DAMP>
static int launch_tile_tma(tlfea_element_s* h, const TileArgs<R>& A) {
    auto kern = k_tile_force_tma<R, NPE, NQP, DAMP>;
    const size_t smem = tile_tma_smem_bytes<R, NPE>(h->tl.max_local_pad, DAMP);
    if (smem > 227 * 1024) {
        set_error("force kernel shared memory exceeds 227 KB (tile touches too many nodes)");
        return TLFEA_UNSUPPORTED;
    }
    static bool configured = false;  // one instantiation per template argument set
    if (!configured) {
        TLFEA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared));
        configured = true;
    }
    if (smem > 48 * 1024) TLFEA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<h->tl.n_tiles, TILE_ELEMS, smem, h->stream>>>(A, h->d_err);
    TLFEA_CHECK_LAUNCH();
    return TLFEA_OK;
}

// One tile per block on the compact geometry stream (J^-1 and dV per QP).
template <typename R, int NPE, int NQP, bool DAMP, bool MR = false>
static int launch_tile_geo(tlfea_element_s* h, const TileArgs<R>& A) {
    auto kern = k_tile_force_geo<R, NPE, NQP, DAMP, MR>;
    const size_t smem = tile_geo_smem_bytes<R, NPE>(h->tl.max_local_pad, DAMP);
    if (smem > 227 * 1024) {
        set_error("force kernel shared memory exceeds 227 KB (tile touches too many nodes)");
        return TLFEA_UNSUPPORTED;
    }
    static bool configured = false;  // one instantiation per template argument set
    if (!configured) {
        TLFEA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared));
        configured = true;
    }
    if (smem > 48 * 1024) TLFEA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<h->tl.n_tiles, TILE_ELEMS, smem, h->stream>>>(A, h->d_err);
    TLFEA_CHECK_LAUNCH();
    return TLFEA_OK;
}

// Persistent TMA-fed force kernel: grid = resident CTAs (occupancy) capped by the tile count.
template <typename R, int NPE, int NQP, bool DAMP>
static int launch_pipe(tlfea_element_s* h, const TileArgs<R>& A) {
    auto kern = k_force_pipe<R, NPE, NQP, DAMP>;
    const size_t smem = pipe_smem_bytes<R, NPE>(h->tl.max_local_pad, DAMP);
    int& grid = h->pipe_grid[(sizeof(R) == 4 ? 2 : 0) + (DAMP ? 1 : 0)];
    if (grid == 0) {
        if (smem > 227 * 1024) {
            set_error("force pipeline shared memory exceeds 227 KB (tile touches too many nodes)");
            return TLFEA_UNSUPPORTED;
        }
        TLFEA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0, sms = 0;
        TLFEA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, PIPE_THREADS, smem));
        TLFEA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
        if (per_sm < 1) {
            set_error("force pipeline does not fit on an SM");
            return TLFEA_UNSUPPORTED;
        }
        grid = std::max(1, std::min(h->tl.n_tiles, per_sm * sms));
        if (h->pipe_grid_limit > 0) grid = std::min(grid, h->pipe_grid_limit);
    }
    kern<<<grid, PIPE_THREADS, smem, h->stream>>>(A, h->tl.n_tiles, h->d_err);
    TLFEA_CHECK_LAUNCH();
    return TLFEA_OK;
}

template <typename R, int NPE, int NQP>
static int force_dispatch(tlfea_element_s* h, const double* d_v, bool fp32) {
    TileArgs<R> A = make_args<R>(h, fp32);
    const bool damp = d_v && (h->eta_d != 0.0 || h->lambda_d != 0.0);
    A.v = d_v;
    if (h->tl.n_orphans)
        TLFEA_CUDA(cudaMemsetAsync(A.f_out, 0, sizeof(R) * 3 * (size_t)h->N, h->stream));
    int st;
    if (h->material == TLFEA_MATERIAL_MOONEY_RIVLIN)  // Mooney-Rivlin runs on the compact-geometry kernel
        st = damp ? launch_tile_geo<R, NPE, NQP, true, true>(h, A) : launch_tile_geo<R, NPE, NQP, false, true>(h, A);
    else if (h->force_kernel == 1)
        st = damp ? launch_tiles<R, NPE, NQP, TILE_FORCE, true>(h, A) : launch_tiles<R, NPE, NQP, TILE_FORCE, false>(h, A);
    else if (h->force_kernel == 2)
        st = damp ? launch_pipe<R, NPE, NQP, true>(h, A) : launch_pipe<R, NPE, NQP, false>(h, A);
    else if (h->force_kernel == 3)
        st = damp ? launch_tile_geo<R, NPE, NQP, true>(h, A) : launch_tile_geo<R, NPE, NQP, false>(h, A);
    else
        st = damp ? launch_tile_tma<R, NPE, NQP, true>(h, A) : launch_tile_tma<R, NPE, NQP, false>(h, A);
    if (st) return st;
    return launch_combine<R, false>(h, A.partial, A.f_out);
}

// The tile-ordered node record's values: FP64 positions (disp = 0) or displacements
// x - X0 (disp = 1, FP32 mode, the same difference as k_disp64); padding entries 0.
__global__ void k_stage_refresh(long long n, const int* __restrict__ gid, const double* __restrict__ x,
                                const double* __restrict__ y, const double* __restrict__ z,
                                const double* __restrict__ X0x, const double* __restrict__ X0y,
                                const double* __restrict__ X0z, int disp, double* __restrict__ sx,
                                double* __restrict__ sy, double* __restrict__ sz) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int g = gid[k];
        double a = 0.0, b = 0.0, c = 0.0;
        if (g >= 0) {
            a = x[g];
            b = y[g];
            c = z[g];
            if (disp) {
                a -= X0x[g];
                b -= X0y[g];
                c -= X0z[g];
            }
        }
        sx[k] = a;
        sy[k] = b;
        sz[k] = c;
    }
}

// Rebuild the tile-ordered node record for the precision about to be evaluated, after
// a change of positions (or every time, once the positions' pointers are exposed).
int element_refresh_record(tlfea_element_s* h, bool fp32) {
    const int want = fp32 ? 2 : 1;
    if (h->stage_content == want && !h->positions_exposed) return TLFEA_OK;
    const long long n = h->tl.n_pad;
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_stage_refresh<<<blocks, 256, 0, h->stream>>>(n, h->tl.pad_gid, h->x, h->y, h->z, h->X0x, h->X0y, h->X0z,
                                                   fp32 ? 1 : 0, h->tl.sx, h->tl.sy, h->tl.sz);
    TLFEA_CHECK_LAUNCH();
    h->stage_content = want;
    return TLFEA_OK;
}

// f_int (FP64) or f_int32 (FP32) = internal force at the current positions.
// Asynchronous on h->stream (the solvers call it inside their loops).
// The interleaved FP64 displacement the FP32 force stages from, after a change of positions.
int element_refresh_u64(tlfea_element_s* h) {
    if (!h->u_dirty && !h->positions_exposed) return TLFEA_OK;
    const int n = h->N;
    k_disp64<<<(n + 255) / 256, 256, 0, h->stream>>>(n, h->x, h->y, h->z, h->X0x, h->X0y, h->X0z, h->u64);
    TLFEA_CHECK_LAUNCH();
    h->u_dirty = false;
    return TLFEA_OK;
}

int element_force(tlfea_element_s* h, const double* d_v, bool fp32) {
    int st;
    // the bulk-copy tile kernels (launch options 0 and 3, and Mooney-Rivlin's) stage the record
    if ((h->force_kernel == 0 || h->force_kernel == 3 || h->material == TLFEA_MATERIAL_MOONEY_RIVLIN) &&
        (st = element_refresh_record(h, fp32)))
        return st;
    if (fp32) {
        if ((st = element_refresh_u64(h))) return st;
        st = (h->npe == 10) ? force_dispatch<float, 10, 5>(h, d_v, true) : force_dispatch<float, 4, 1>(h, d_v, true);
    } else {
        st = (h->npe == 10) ? force_dispatch<double, 10, 5>(h, d_v, false)
                            : force_dispatch<double, 4, 1>(h, d_v, false);
    }
    if (st == TLFEA_OK) h->f_int_from32 = fp32;
    return st;
}

// f_int (FP64) catches up with the last FP32 evaluation.
static int sync_f_int64(tlfea_element_s* h) {
    if (!h->f_int_from32) return TLFEA_OK;
    const long long n = 3LL * h->N;
    k_f32_to_f64<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(n, h->f_int32, h->f_int);
    TLFEA_CHECK_LAUNCH();
    h->f_int_from32 = false;
    return TLFEA_OK;
}

// ------------------------------------------- scratch of the allocation-free entry
//
// The force kernel needs scratch for the per-tile partial sums of nodes shared
// between tiles (3 values per shared-node slot).  The regular entry point keeps
// that buffer in the element; the allocation-free entry point uses this array
// instead.  It is a file-scope device array, so every GPU that loads the
// library holds these 8 MiB until the process exits.
constexpr size_t NOALLOC_SCRATCH_DOUBLES = size_t(1) << 20;  // 8 MiB
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

constexpr int NOALLOC_MAX_DEVICES = 64;
static double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};
static std::mutex g_noalloc_mutex;

// Device address of the scratch array on `device` (which must be current).  In
// host code the array's name is a host-side stand-in, not a device address, so
// the address is looked up once per device with cudaGetSymbolAddress.
static int noalloc_scratch(int device, double** out) {
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) {
        set_error("device index out of range for the static scratch table");
        return TLFEA_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        double* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
            return TLFEA_CUDA_ERROR;
        }
        g_noalloc_ptr[device] = p;
    }
    *out = g_noalloc_ptr[device];
    return TLFEA_OK;
}

// A kernel's bounded wait ran out: report it once and clear the word.
static int check_device_error(tlfea_element_s* h) {
    int e = 0;
    if (cudaMemcpy(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("reading the device error word failed");
        return TLFEA_CUDA_ERROR;
    }
    if (e) {
        cudaMemset(h->d_err, 0, sizeof(int));
        set_error("a pipeline wait in the force kernel ran out (code " + std::to_string(e) + ")");
        return TLFEA_BUDGET_EXCEEDED;
    }
    return TLFEA_OK;
}

static int ensure_pst(tlfea_element_s* h) {
    if (h->Pst) return TLFEA_OK;
    const size_t n = (size_t)h->E * h->nqp * 9;
    int st = dalloc(&h->Pst, n);
    if (st) return st;
    TLFEA_CUDA(cudaMemsetAsync(h->Pst, 0, n * sizeof(double), h->stream));
    return TLFEA_OK;
}

static void fill_mass_params(const tlfea_element_s* h, MassParams& mp) {
    static const int edges[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
    memset(&mp, 0, sizeof(mp));
    for (int q = 0; q < h->nqp; ++q) {
        const double xi = h->qx[q], eta = h->qy[q], zeta = h->qz[q];
        const double L[4] = {1.0 - xi - eta - zeta, xi, eta, zeta};
        if (h->npe == 4) {
            for (int k = 0; k < 4; ++k) mp.N[q][k] = L[k];
        } else {
            for (int k = 0; k < 4; ++k) mp.N[q][k] = L[k] * (2.0 * L[k] - 1.0);
            for (int k = 0; k < 6; ++k) mp.N[q][k + 4] = 4.0 * L[edges[k][0]] * L[edges[k][1]];
        }
        mp.w[q] = h->qw[q];
    }
}

}  // namespace tlfea

using namespace tlfea;

#define CHECK_HANDLE(h)                                  \
    do {                                                 \
        if (!(h)) {                                      \
            set_error("null handle");                    \
            return TLFEA_INVALID_ARG;                    \
        }                                                \
        const cudaError_t dev_e_ = cudaSetDevice((h)->device); \
        if (dev_e_ != cudaSuccess) {                     \
            set_error(std::string("cudaSetDevice: ") + cudaGetErrorString(dev_e_)); \
            return TLFEA_CUDA_ERROR;                     \
        }                                                \
    } while (0)

#define SYNC(h) TLFEA_CUDA(cudaStreamSynchronize((h)->stream))
#define REQUIRE_SETUP(h)                                     \
    do {                                                     \
        if (!(h)->is_setup) {                                \
            set_error("element must be set up first");       \
            return TLFEA_NOT_SETUP;                          \
        }                                                    \
    } while (0)
// compute calls honour the non-blocking mode
#define SYNC_COMPUTE(h)                                            \
    do {                                                           \
        if ((h)->blocking) {                                       \
            TLFEA_CUDA(cudaStreamSynchronize((h)->stream));        \
            int st_err_ = check_device_error(h);                   \
            if (st_err_) return st_err_;                           \
        }                                                          \
    } while (0)
// device -> host copy after the element's stream has drained
#define D2H(dst, src, bytes)                                                      \
    do {                                                                          \
        TLFEA_CUDA(cudaStreamSynchronize(h->stream));                             \
        TLFEA_CUDA(cudaMemcpy((dst), (src), (bytes), cudaMemcpyDeviceToHost));    \
    } while (0)

extern "C" {

const char* tlfea_last_error(void) { return t_last_error.c_str(); }
long long tlfea_launch_count(void) { return g_launches.load(); }
const char* tlfea_version(void) { return "tlfea_b200 0.1 (sm_100a)"; }

int tlfea_element_create(int type, int n_elem, int n_nodes, tlfea_element* out) {
    if (!out) return TLFEA_INVALID_ARG;
    *out = nullptr;
    if ((type != TLFEA_TYPE_T10 && type != TLFEA_TYPE_T4) || n_elem <= 0 || n_nodes <= 0) {
        set_error("element_create: bad type or size");
        return TLFEA_INVALID_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("no CUDA device");
        return TLFEA_NO_CUDA_DEVICE;
    }
    tlfea_element_s* h = new tlfea_element_s();
    cudaGetDevice(&h->device);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("cudaStreamCreate failed");
        delete h;
        return TLFEA_CUDA_ERROR;
    }
    h->own_stream = true;
    h->type = type;
    h->npe = (type == TLFEA_TYPE_T10) ? T10_NPE : T4_NPE;
    h->nqp = (type == TLFEA_TYPE_T10) ? T10_NQP : T4_NQP;
    h->E = n_elem;
    h->N = n_nodes;
    const size_t N = (size_t)n_nodes;
    int st = TLFEA_OK;
    st |= dalloc(&h->x, N) | dalloc(&h->y, N) | dalloc(&h->z, N);
    st |= dalloc(&h->xj, N) | dalloc(&h->yj, N) | dalloc(&h->zj, N);
    st |= dalloc(&h->X0x, N) | dalloc(&h->X0y, N) | dalloc(&h->X0z, N) | dalloc(&h->u64, 3 * (size_t)N);
    st |= dalloc(&h->d_conn, (size_t)n_elem * h->npe);
    st |= dalloc(&h->f_int, 3 * N) | dalloc(&h->f_ext, 3 * N) | dalloc(&h->f_int32, 3 * N);
    st |= dalloc(&h->detJ, (size_t)n_elem * h->nqp);
    st |= dalloc(&h->d_err, 1);
    if (st) {
        tlfea_element_destroy(h);
        return TLFEA_CUDA_ERROR;
    }
    cudaMemsetAsync(h->f_int, 0, 3 * N * sizeof(double), h->stream);
    cudaMemsetAsync(h->f_ext, 0, 3 * N * sizeof(double), h->stream);
    cudaMemsetAsync(h->f_int32, 0, 3 * N * sizeof(float), h->stream);
    cudaMemsetAsync(h->detJ, 0, (size_t)n_elem * h->nqp * sizeof(double), h->stream);
    cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream);
    cudaStreamSynchronize(h->stream);
    *out = h;
    return TLFEA_OK;
}

int tlfea_element_destroy(tlfea_element h) {
    if (!h) return TLFEA_INVALID_ARG;
    TLFEA_CUDA(cudaSetDevice(h->device));
    dfree(h->x); dfree(h->y); dfree(h->z);
    dfree(h->xj); dfree(h->yj); dfree(h->zj);
    dfree(h->X0x); dfree(h->X0y); dfree(h->X0z); dfree(h->u64);
    dfree(h->d_conn); dfree(h->f_int); dfree(h->f_ext); dfree(h->f_int32);
    dfree(h->detJ); dfree(h->Pst); dfree(h->d_err);
    free_tiling(h->tl);
    dfree(h->inc_off); dfree(h->inc_e); dfree(h->inc_a);
    dfree(h->pat_off); dfree(h->pat_col); dfree(h->m_val);
    dfree(h->fixed); dfree(h->c);
    dfree(h->jt_off); dfree(h->jt_col); dfree(h->jt_val);
    dfree(h->j_off); dfree(h->j_col); dfree(h->j_val);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return TLFEA_OK;
}

int tlfea_element_set_stream(tlfea_element h, void* stream) {
    CHECK_HANDLE(h);
    TLFEA_CUDA(cudaStreamSynchronize(h->stream));
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    h->own_stream = false;
    h->stream = (cudaStream_t)stream;
    return TLFEA_OK;
}

int tlfea_element_get_stream(tlfea_element h, void** stream) {
    if (!h || !stream) return TLFEA_INVALID_ARG;
    *stream = (void*)h->stream;
    return TLFEA_OK;
}

int tlfea_element_set_blocking(tlfea_element h, int blocking) {
    CHECK_HANDLE(h);
    h->blocking = (blocking != 0);
    if (h->blocking) SYNC(h);
    return TLFEA_OK;
}

int tlfea_element_reset_positions(tlfea_element h) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    positions_changed(h);
    const size_t nb = (size_t)h->N * sizeof(double);
    TLFEA_CUDA(cudaMemcpyAsync(h->x, h->X0x, nb, cudaMemcpyDeviceToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->y, h->X0y, nb, cudaMemcpyDeviceToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->z, h->X0z, nb, cudaMemcpyDeviceToDevice, h->stream));
    SYNC_COMPUTE(h);
    return TLFEA_OK;
}

int tlfea_element_get_counts(tlfea_element h, int* n_elem, int* n_nodes, int* n_constraint) {
    if (!h) return TLFEA_INVALID_ARG;
    if (n_elem) *n_elem = h->E;
    if (n_nodes) *n_nodes = h->N;
    if (n_constraint) *n_constraint = h->n_constraint;
    return TLFEA_OK;
}

int tlfea_element_setup(tlfea_element h, const double* qx, const double* qy, const double* qz, const double* qw,
                        int n_qp, const double* x, const double* y, const double* z, const int* conn) {
    CHECK_HANDLE(h);
    if (h->is_setup) {
        set_error("element is already set up");
        return TLFEA_ALREADY_SETUP;
    }
    if (!qx || !qy || !qz || !qw || !x || !y || !z || !conn) return TLFEA_INVALID_ARG;
    if (n_qp != h->nqp) {
        set_error("quadrature size does not match the element type");
        return TLFEA_SIZE_MISMATCH;
    }
    const size_t ne = (size_t)h->E * h->npe;
    for (size_t k = 0; k < ne; ++k)
        if (conn[k] < 0 || conn[k] >= h->N) {
            set_error("connectivity index out of range");
            return TLFEA_INVALID_ARG;
        }
    for (int q = 0; q < n_qp; ++q) {
        h->qx[q] = qx[q];
        h->qy[q] = qy[q];
        h->qz[q] = qz[q];
        h->qw[q] = qw[q];
    }
    const size_t nb = (size_t)h->N * sizeof(double);
    TLFEA_CUDA(cudaMemcpyAsync(h->x, x, nb, cudaMemcpyHostToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->y, y, nb, cudaMemcpyHostToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->z, z, nb, cudaMemcpyHostToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->xj, x, nb, cudaMemcpyHostToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->yj, y, nb, cudaMemcpyHostToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->zj, z, nb, cudaMemcpyHostToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->X0x, x, nb, cudaMemcpyHostToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->X0y, y, nb, cudaMemcpyHostToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->X0z, z, nb, cudaMemcpyHostToDevice, h->stream));
    h->conn.assign(conn, conn + ne);
    TLFEA_CUDA(cudaMemcpyAsync(h->d_conn, conn, ne * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    TLFEA_CUDA(cudaMemsetAsync(h->f_int, 0, 3 * nb, h->stream));
    TLFEA_CUDA(cudaMemsetAsync(h->detJ, 0, (size_t)h->E * h->nqp * sizeof(double), h->stream));
    h->rho = h->E_mod = h->nu = h->mu = h->lambda = h->eta_d = h->lambda_d = 0.0;
    h->material = TLFEA_MATERIAL_SVK;
    h->mu10 = h->mu01 = h->kappa = 0.0;
    int st = build_tiling(h, x, y, z);
    if (st) return st;
    if ((st = build_incidence(h))) return st;
    SYNC(h);
    positions_changed(h);
    h->is_setup = true;
    return TLFEA_OK;
}


int tlfea_element_set_density(tlfea_element h, double rho0) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    h->rho = rho0;
    return TLFEA_OK;
}

int tlfea_element_set_damping(tlfea_element h, double eta_damp, double lambda_damp) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    h->eta_d = eta_damp;
    h->lambda_d = lambda_damp;
    return TLFEA_OK;
}

int tlfea_element_set_svk_default(tlfea_element h) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    h->material = TLFEA_MATERIAL_SVK;
    h->mu10 = h->mu01 = h->kappa = 0.0;
    return TLFEA_OK;
}

int tlfea_element_set_svk(tlfea_element h, double E, double nu) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    h->E_mod = E;
    h->nu = nu;
    h->mu = E / (2 * (1 + nu));
    h->lambda = (E * nu) / ((1 + nu) * (1 - 2 * nu));
    return tlfea_element_set_svk_default(h);
}

int tlfea_element_set_mooney_rivlin(tlfea_element h, double mu10, double mu01, double kappa) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    h->material = TLFEA_MATERIAL_MOONEY_RIVLIN;
    h->mu10 = mu10;
    h->mu01 = mu01;
    h->kappa = kappa;
    return TLFEA_OK;
}

int tlfea_element_add_gravity(tlfea_element h, double gx, double gy, double gz) {
    CHECK_HANDLE(h);
    if (!h->mass_setup) {
        set_error("add_gravity: CalcMassMatrix must be called first");
        return TLFEA_NOT_SETUP;
    }
    k_add_gravity<<<(h->N + 255) / 256, 256, 0, h->stream>>>(h->N, h->pat_off, h->m_val, gx, gy, gz, h->f_ext);
    TLFEA_CHECK_LAUNCH();
    SYNC(h);
    return TLFEA_OK;
}

int tlfea_element_set_external_force(tlfea_element h, const double* f, int n) {
    CHECK_HANDLE(h);
    if (!f || n != 3 * h->N) {
        set_error("External force vector size mismatch.");
        return TLFEA_SIZE_MISMATCH;
    }
    TLFEA_CUDA(cudaMemcpyAsync(h->f_ext, f, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    SYNC(h);
    return TLFEA_OK;
}

static int upload_fixed(tlfea_element h, const int* nodes, int n) {
    for (int k = 0; k < n; ++k)
        if (nodes[k] < 0 || nodes[k] >= h->N) {
            set_error("fixed node index out of range");
            return TLFEA_INVALID_ARG;
        }
    dfree(h->fixed);
    dfree(h->c);
    h->h_fixed.assign(nodes, nodes + n);
    h->n_constraint = 3 * n;
    int st = upload(&h->fixed, h->h_fixed, h->stream);
    if (st) return st;
    if ((st = dalloc(&h->c, (size_t)std::max(3 * n, 1)))) return st;
    TLFEA_CUDA(cudaMemsetAsync(h->c, 0, (size_t)std::max(3 * n, 1) * sizeof(double), h->stream));
    dfree(h->jt_off); dfree(h->jt_col); dfree(h->jt_val);
    dfree(h->j_off); dfree(h->j_col); dfree(h->j_val);
    h->jt_setup = h->j_setup = false;
    h->constraints_setup = true;
    return TLFEA_OK;
}

int tlfea_element_set_nodal_fixed(tlfea_element h, const int* nodes, int n) {
    CHECK_HANDLE(h);
    if (n < 0 || (n > 0 && !nodes)) return TLFEA_INVALID_ARG;
    if (h->constraints_setup) {
        set_error("constraint is already set up");
        return TLFEA_ALREADY_SETUP;
    }
    return upload_fixed(h, nodes, n);
}

int tlfea_element_update_nodal_fixed(tlfea_element h, const int* nodes, int n) {
    CHECK_HANDLE(h);
    if (n < 0 || (n > 0 && !nodes)) return TLFEA_INVALID_ARG;
    return upload_fixed(h, nodes, n);
}

static int copy_positions(tlfea_element h, double* dx, double* dy, double* dz, const double* x, const double* y,
                          const double* z, int n) {
    if (!x || !y || !z || n != h->N) {
        set_error("Position vector size mismatch.");
        return TLFEA_SIZE_MISMATCH;
    }
    const size_t nb = (size_t)n * sizeof(double);
    TLFEA_CUDA(cudaMemcpyAsync(dx, x, nb, cudaMemcpyHostToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(dy, y, nb, cudaMemcpyHostToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(dz, z, nb, cudaMemcpyHostToDevice, h->stream));
    SYNC(h);
    return TLFEA_OK;
}

int tlfea_element_update_positions(tlfea_element h, const double* x, const double* y, const double* z, int n) {
    CHECK_HANDLE(h);
    positions_changed(h);
    return copy_positions(h, h->x, h->y, h->z, x, y, z, n);
}

int tlfea_element_update_constraint_targets(tlfea_element h, const double* x, const double* y, const double* z,
                                            int n) {
    CHECK_HANDLE(h);
    return copy_positions(h, h->xj, h->yj, h->zj, x, y, z, n);
}

int tlfea_element_calc_dndu_pre(tlfea_element h) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    QuadParams qp;
    memcpy(qp.qx, h->qx, sizeof(qp.qx));
    memcpy(qp.qy, h->qy, sizeof(qp.qy));
    memcpy(qp.qz, h->qz, sizeof(qp.qz));
    memcpy(qp.qw, h->qw, sizeof(qp.qw));
    const int n_slots = h->tl.n_tiles * TILE_ELEMS;
    const long long nt = (long long)n_slots * h->nqp;
    const unsigned blocks = (unsigned)((nt + 127) / 128);
    Tiling& tl = h->tl;
    if (h->npe == 10)
        k_dndu_pre<10, 5><<<blocks, 128, 0, h->stream>>>(n_slots, h->E, tl.tile_elem, h->d_conn, h->x, h->y, h->z, qp,
                                                        tl.grad64, tl.grad32, tl.dv64, tl.dv32, h->detJ,
                                                        tl.ji64, tl.ji32);
    else
        k_dndu_pre<4, 1><<<blocks, 128, 0, h->stream>>>(n_slots, h->E, tl.tile_elem, h->d_conn, h->x, h->y, h->z, qp,
                                                       tl.grad64, tl.grad32, tl.dv64, tl.dv32, h->detJ,
                                                        tl.ji64, tl.ji32);
    TLFEA_CHECK_LAUNCH();
    const size_t nb = (size_t)h->N * sizeof(double);
    TLFEA_CUDA(cudaMemcpyAsync(h->X0x, h->x, nb, cudaMemcpyDeviceToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->X0y, h->y, nb, cudaMemcpyDeviceToDevice, h->stream));
    TLFEA_CUDA(cudaMemcpyAsync(h->X0z, h->z, nb, cudaMemcpyDeviceToDevice, h->stream));
    positions_changed(h);
    h->precomputed = true;
    SYNC(h);
    return TLFEA_OK;
}

int tlfea_element_calc_mass_matrix(tlfea_element h) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    int st = element_build_pattern(h);
    if (st) return st;
    if (!h->m_val) {
        if ((st = dalloc(&h->m_val, (size_t)std::max(h->pat_nnz, 1LL)))) return st;
    }
    MassParams mp;
    fill_mass_params(h, mp);
    const int N = h->N;
    if (h->npe == 10)
        k_mass_rows<10, 5><<<(N + 127) / 128, 128, 0, h->stream>>>(N, h->E, h->rho, h->d_conn, h->detJ, h->inc_off,
                                                                   h->inc_e, h->inc_a, h->pat_off, h->pat_col,
                                                                   h->m_val, mp);
    else
        k_mass_rows<4, 1><<<(N + 127) / 128, 128, 0, h->stream>>>(N, h->E, h->rho, h->d_conn, h->detJ, h->inc_off,
                                                                  h->inc_e, h->inc_a, h->pat_off, h->pat_col,
                                                                  h->m_val, mp);
    TLFEA_CHECK_LAUNCH();
    h->mass_setup = true;
    SYNC(h);
    return TLFEA_OK;
}

int tlfea_element_calc_p(tlfea_element h) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    int st = ensure_pst(h);
    if (st) return st;
    TileArgs<double> A = make_args<double>(h, false);
    A.Pst = h->Pst;
    if (h->material == TLFEA_MATERIAL_MOONEY_RIVLIN)
        st = (h->npe == 10) ? launch_tiles<double, 10, 5, TILE_STORE_P, false, true>(h, A)
                            : launch_tiles<double, 4, 1, TILE_STORE_P, false, true>(h, A);
    else
        st = (h->npe == 10) ? launch_tiles<double, 10, 5, TILE_STORE_P, false>(h, A)
                            : launch_tiles<double, 4, 1, TILE_STORE_P, false>(h, A);
    if (st) return st;
    SYNC_COMPUTE(h);
    return TLFEA_OK;
}

int tlfea_element_calc_internal_force(tlfea_element h) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    int st = ensure_pst(h);
    if (st) return st;
    if ((st = sync_f_int64(h))) return st;
    TileArgs<double> A = make_args<double>(h, false);
    A.Pst = h->Pst;
    st = (h->npe == 10) ? launch_tiles<double, 10, 5, TILE_FORCE_FROM_P, false>(h, A)
                        : launch_tiles<double, 4, 1, TILE_FORCE_FROM_P, false>(h, A);
    if (st) return st;
    if ((st = launch_combine<double, true>(h, A.partial, A.f_out))) return st;
    SYNC_COMPUTE(h);
    return TLFEA_OK;
}

int tlfea_element_calc_constraint_data(tlfea_element h) {
    CHECK_HANDLE(h);
    if (!h->constraints_setup) {
        set_error("constraint is not set up");
        return TLFEA_NOT_SETUP;
    }
    const int nf = h->n_constraint / 3;
    if (nf == 0) return TLFEA_OK;
    k_constraint<<<(nf + 127) / 128, 128, 0, h->stream>>>(nf, h->fixed, h->x, h->y, h->z, h->xj, h->yj, h->zj, h->c);
    TLFEA_CHECK_LAUNCH();
    SYNC_COMPUTE(h);
    return TLFEA_OK;
}

// J^T: rows = 3N DOFs, one unit entry per constraint k at row 3*fixed[k/3]+k%3,
// columns in increasing k (FEAT10Data.cu:510-562 fills each row in atomic order).
int tlfea_element_build_constraint_jact_csr(tlfea_element h) {
    CHECK_HANDLE(h);
    if (h->jt_setup) return TLFEA_OK;
    if (!h->constraints_setup || h->n_constraint == 0) return TLFEA_OK;
    const int nr = 3 * h->N, nc = h->n_constraint;
    std::vector<int> off((size_t)nr + 1, 0), col((size_t)nc);
    std::vector<double> val((size_t)nc, 1.0);
    for (int k = 0; k < nc; ++k) off[3 * h->h_fixed[k / 3] + k % 3 + 1]++;
    for (int r = 0; r < nr; ++r) off[r + 1] += off[r];
    std::vector<int> pos(off.begin(), off.end() - 1);
    for (int k = 0; k < nc; ++k) col[pos[3 * h->h_fixed[k / 3] + k % 3]++] = k;
    int st;
    if ((st = upload(&h->jt_off, off, h->stream))) return st;
    if ((st = upload(&h->jt_col, col, h->stream))) return st;
    if ((st = upload(&h->jt_val, val, h->stream))) return st;
    h->jt_setup = true;
    return TLFEA_OK;
}

// J: rows = constraints, row k has the unit entry at DOF 3*fixed[k/3]+k%3 (FEAT10Data.cu:420-505).
int tlfea_element_build_constraint_jac_csr(tlfea_element h) {
    CHECK_HANDLE(h);
    if (h->j_setup) return TLFEA_OK;
    if (!h->constraints_setup || h->n_constraint == 0) return TLFEA_OK;
    const int nc = h->n_constraint;
    std::vector<int> off((size_t)nc + 1), col((size_t)nc);
    std::vector<double> val((size_t)nc, 1.0);
    for (int k = 0; k < nc; ++k) {
        off[k] = k;
        col[k] = 3 * h->h_fixed[k / 3] + k % 3;
    }
    off[nc] = nc;
    int st;
    if ((st = upload(&h->j_off, off, h->stream))) return st;
    if ((st = upload(&h->j_col, col, h->stream))) return st;
    if ((st = upload(&h->j_val, val, h->stream))) return st;
    h->j_setup = true;
    return TLFEA_OK;
}

int tlfea_element_compute_internal_force(tlfea_element h, const double* d_v) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    int st = element_force(h, d_v, h->precision == TLFEA_PRECISION_FP32);
    if (st) return st;
    SYNC_COMPUTE(h);
    return TLFEA_OK;
}

int tlfea_element_set_launch_config(tlfea_element h, int force_kernel, int grid_limit) {
    CHECK_HANDLE(h);
    if (force_kernel < 0 || force_kernel > 3 || grid_limit < 0) return TLFEA_INVALID_ARG;
    h->force_kernel = force_kernel;
    h->pipe_grid_limit = grid_limit;
    for (int& g : h->pipe_grid) g = 0;
    return TLFEA_OK;
}

int tlfea_element_set_force_precision(tlfea_element h, int precision) {
    CHECK_HANDLE(h);
    if (precision != TLFEA_PRECISION_FP64 && precision != TLFEA_PRECISION_FP32) return TLFEA_INVALID_ARG;
    h->precision = precision;
    return TLFEA_OK;
}

// Allocation-free variant of tlfea_element_compute_internal_force (FP64): the
// same tile and combine kernels, with the shared-node partials in the static
// scratch array and the result in the caller's buffer.  Calls no cudaMalloc,
// cudaFree or allocating library routine.  The first call on a device looks
// up the scratch address (cudaGetSymbolAddress); make that first call before
// any stream capture.  Every call shares the one array per device and it keeps
// the last call's contents; each call writes every slot it reads before
// reading it, so nothing has to start at zero.  Calls that overlap on the GPU
// (other streams, other elements, other threads) race on the array.
int tlfea_element_compute_internal_force_noalloc(tlfea_element h, const double* d_v, double* d_f_out) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    if (!d_f_out) {
        set_error("output pointer is null");
        return TLFEA_INVALID_ARG;
    }
    if (h->precision != TLFEA_PRECISION_FP64) {
        set_error("the allocation-free internal force runs in FP64 only; this element is in FP32 force mode "
                  "(use tlfea_element_compute_internal_force)");
        return TLFEA_UNSUPPORTED;
    }
    const size_t need = 3 * (size_t)h->tl.n_pslots;
    if (need > NOALLOC_SCRATCH_DOUBLES) {
        set_error("mesh needs " + std::to_string(need) + " doubles of shared-node scratch; the static scratch holds " +
                  std::to_string(NOALLOC_SCRATCH_DOUBLES) + " (use tlfea_element_compute_internal_force)");
        return TLFEA_SIZE_MISMATCH;
    }
    double* scratch = nullptr;
    int st = noalloc_scratch(h->device, &scratch);
    if (st) return st;
    TileArgs<double> A = make_args<double>(h, false);
    A.v = d_v;
    A.f_out = d_f_out;
    A.partial = scratch;
    const bool damp = d_v && (h->eta_d != 0.0 || h->lambda_d != 0.0);
    if (h->tl.n_orphans) TLFEA_CUDA(cudaMemsetAsync(d_f_out, 0, sizeof(double) * 3 * (size_t)h->N, h->stream));
    const bool mr = (h->material == TLFEA_MATERIAL_MOONEY_RIVLIN);
    if (h->npe == 10) {
        if (mr)
            st = damp ? launch_tiles<double, 10, 5, TILE_FORCE, true, true>(h, A)
                      : launch_tiles<double, 10, 5, TILE_FORCE, false, true>(h, A);
        else
            st = damp ? launch_tiles<double, 10, 5, TILE_FORCE, true>(h, A)
                      : launch_tiles<double, 10, 5, TILE_FORCE, false>(h, A);
    } else {
        if (mr)
            st = damp ? launch_tiles<double, 4, 1, TILE_FORCE, true, true>(h, A)
                      : launch_tiles<double, 4, 1, TILE_FORCE, false, true>(h, A);
        else
            st = damp ? launch_tiles<double, 4, 1, TILE_FORCE, true>(h, A)
                      : launch_tiles<double, 4, 1, TILE_FORCE, false>(h, A);
    }
    if (st) return st;
    if ((st = launch_combine<double, false>(h, A.partial, A.f_out))) return st;
    SYNC_COMPUTE(h);
    return TLFEA_OK;
}

int tlfea_element_get_mass_nnz(tlfea_element h, long long* nnz) {
    if (!h || !nnz) return TLFEA_INVALID_ARG;
    *nnz = h->mass_setup ? h->pat_nnz : 0;
    return TLFEA_OK;
}

int tlfea_element_retrieve_mass_csr(tlfea_element h, int* offsets, int* columns, double* values) {
    CHECK_HANDLE(h);
    if (!offsets) return TLFEA_INVALID_ARG;
    if (!h->mass_setup) {
        memset(offsets, 0, sizeof(int) * ((size_t)h->N + 1));
        return TLFEA_OK;
    }
    memcpy(offsets, h->h_pat_off.data(), sizeof(int) * ((size_t)h->N + 1));
    if (columns) memcpy(columns, h->h_pat_col.data(), sizeof(int) * (size_t)h->pat_nnz);
    if (values) D2H(values, h->m_val, sizeof(double) * (size_t)h->pat_nnz);
    return TLFEA_OK;
}

int tlfea_element_retrieve_internal_force(tlfea_element h, double* f, int n) {
    CHECK_HANDLE(h);
    if (!f || n != 3 * h->N) return TLFEA_SIZE_MISMATCH;
    int st = sync_f_int64(h);
    if (st) return st;
    SYNC(h);
    D2H(f, h->f_int, (size_t)n * sizeof(double));
    return TLFEA_OK;
}

int tlfea_element_retrieve_external_force(tlfea_element h, double* f, int n) {
    CHECK_HANDLE(h);
    if (!f || n != 3 * h->N) return TLFEA_SIZE_MISMATCH;
    D2H(f, h->f_ext, (size_t)n * sizeof(double));
    return TLFEA_OK;
}

int tlfea_element_retrieve_positions(tlfea_element h, double* x, double* y, double* z, int n) {
    CHECK_HANDLE(h);
    if (!x || !y || !z || n != h->N) return TLFEA_SIZE_MISMATCH;
    SYNC(h);
    const size_t nb = (size_t)n * sizeof(double);
    D2H(x, h->x, nb);
    D2H(y, h->y, nb);
    D2H(z, h->z, nb);
    return TLFEA_OK;
}

int tlfea_element_retrieve_p(tlfea_element h, double* P, long long n) {
    CHECK_HANDLE(h);
    const long long need = (long long)h->E * h->nqp * 9;
    if (!P || n != need) return TLFEA_SIZE_MISMATCH;
    if (!h->Pst) {
        memset(P, 0, sizeof(double) * (size_t)n);
        return TLFEA_OK;
    }
    D2H(P, h->Pst, sizeof(double) * (size_t)n);
    return TLFEA_OK;
}

int tlfea_element_retrieve_dndu_pre(tlfea_element h, double* g, long long n) {
    CHECK_HANDLE(h);
    const int npe = h->npe, nqp = h->nqp, TE = TILE_ELEMS;
    const long long need = (long long)h->E * nqp * npe * 3;
    if (!g || n != need) return TLFEA_SIZE_MISMATCH;
    const size_t ng = (size_t)h->tl.n_tiles * nqp * npe * 3 * TE;
    std::vector<double> tiled(ng);
    D2H(tiled.data(), h->tl.grad64, ng * sizeof(double));
    for (size_t s = 0; s < h->tl.h_tile_elem.size(); ++s) {
        const int e = h->tl.h_tile_elem[s];
        if (e < 0) continue;
        const size_t tile = s / TE, t = s % TE;
        for (int q = 0; q < nqp; ++q)
            for (int a = 0; a < npe; ++a)
                for (int j = 0; j < 3; ++j)
                    g[((size_t)e * nqp + q) * npe * 3 + a + (size_t)npe * j] =
                        tiled[((tile * nqp + q) * npe * 3 + a * 3 + j) * TE + t];
    }
    return TLFEA_OK;
}

int tlfea_element_retrieve_detj(tlfea_element h, double* detJ, long long n) {
    CHECK_HANDLE(h);
    if (!detJ || n != (long long)h->E * h->nqp) return TLFEA_SIZE_MISMATCH;
    D2H(detJ, h->detJ, sizeof(double) * (size_t)n);
    return TLFEA_OK;
}

int tlfea_element_retrieve_connectivity(tlfea_element h, int* conn, long long n) {
    if (!h || !conn || n != (long long)h->E * h->npe) return TLFEA_SIZE_MISMATCH;
    if (!h->is_setup) return TLFEA_NOT_SETUP;
    memcpy(conn, h->conn.data(), sizeof(int) * (size_t)n);
    return TLFEA_OK;
}

int tlfea_element_retrieve_constraint(tlfea_element h, double* c, int n) {
    CHECK_HANDLE(h);
    if (!c || n != h->n_constraint) return TLFEA_SIZE_MISMATCH;
    if (n == 0) return TLFEA_OK;
    SYNC(h);
    D2H(c, h->c, sizeof(double) * (size_t)n);
    return TLFEA_OK;
}

int tlfea_element_retrieve_constraint_jac_csr(tlfea_element h, int which, int* offsets, int* columns,
                                              double* values) {
    CHECK_HANDLE(h);
    if (which != 0 && which != 1) return TLFEA_INVALID_ARG;
    if (!offsets || !columns || !values) return TLFEA_INVALID_ARG;
    const bool built = which ? h->jt_setup : h->j_setup;
    if (!built) {
        set_error("the constraint Jacobian CSR was not built (ConvertToCSR_ConstraintJac / _ConstraintJacT)");
        return TLFEA_NOT_SETUP;
    }
    const size_t rows = which ? 3 * (size_t)h->N : (size_t)h->n_constraint;
    const size_t nnz = (size_t)h->n_constraint;
    SYNC(h);
    D2H(offsets, which ? h->jt_off : h->j_off, sizeof(int) * (rows + 1));
    D2H(columns, which ? h->jt_col : h->j_col, sizeof(int) * nnz);
    D2H(values, which ? h->jt_val : h->j_val, sizeof(double) * nnz);
    return TLFEA_OK;
}

// Legacy ASCII VTK in the layout of WriteOutputVTK (FEAT10Data.cu:759-794).
int tlfea_element_write_vtk(tlfea_element h, const char* filename) {
    CHECK_HANDLE(h);
    REQUIRE_SETUP(h);
    if (!filename) return TLFEA_INVALID_ARG;
    std::vector<double> x(h->N), y(h->N), z(h->N);
    int st = tlfea_element_retrieve_positions(h, x.data(), y.data(), z.data(), h->N);
    if (st) return st;
    std::ofstream out(filename);
    if (!out) {
        set_error("cannot open VTK output file");
        return TLFEA_INVALID_ARG;
    }
    const int npe = h->npe, E = h->E;
    out << "# vtk DataFile Version 3.0\n" << (npe == 10 ? "T10" : "T4") << " mesh output\nASCII\n"
        << "DATASET UNSTRUCTURED_GRID\n";
    out << "POINTS " << h->N << " float\n";
    for (int i = 0; i < h->N; ++i) out << x[i] << " " << y[i] << " " << z[i] << "\n";
    out << "CELLS " << E << " " << (long long)E * (npe + 1) << "\n";
    for (int e = 0; e < E; ++e) {
        out << npe << " ";
        for (int a = 0; a < npe; ++a) out << h->conn[e + (size_t)a * E] << " ";
        out << "\n";
    }
    out << "CELL_TYPES " << E << "\n";
    for (int e = 0; e < E; ++e) out << (npe == 10 ? 24 : 10) << "\n";
    return TLFEA_OK;
}

int tlfea_element_device_ptrs(tlfea_element h, double** x, double** y, double** z, double** f_ext, double** f_int) {
    CHECK_HANDLE(h);
    // a caller holding the positions may write them without telling the element
    if (x || y || z) h->positions_exposed = true;
    if (x) *x = h->x;
    if (y) *y = h->y;
    if (z) *z = h->z;
    if (f_ext) *f_ext = h->f_ext;
    if (f_int) {
        int st = sync_f_int64(h);
        if (st) return st;
        *f_int = h->f_int;
    }
    return TLFEA_OK;
}

}  // extern "C"
